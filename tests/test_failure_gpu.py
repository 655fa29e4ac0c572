"""GPU: failure detection without a GPU fault.

Every wait of the e-map kernel on its atom-tile copies is bounded; when a wait
expires the kernel records it in the context's status word, lets its own
copies land and returns, and the call fails with AG_E_DEVICE while the
context stays usable.  The test makes a wait expire on purpose through a test
hook: after the first tile has landed, each CTA also waits a few polls on a
barrier that nothing arrives on.  The net-charge checksum is made to fire from
the host side, by offsetting the host's sum of the input weights.  After each
failure the next ordinary call must succeed and match the FP64 oracle.
"""
import numpy as np
import pytest

from conftest import E_TOL, chdir

import fastgrid_b200 as fg
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def job(tmp_path_factory):
    d = tmp_path_factory.mktemp("fail")
    fg.synth_write(str(d), "f", n_atoms=1200, semi_axes=(13, 12, 11), npts=30, seed=31)
    with chdir(str(d)):
        p = fg.Problem("f.gpf", log="f.glg")
    return p, oracle.emap(p.grid, p.xyzw(), p.inv_eps())


def _ok(ctx, p, ref):
    e = ctx.emap(p.grid, p.xyzw(), p.inv_eps())
    assert np.abs(e.astype(np.float64) - ref).max() <= E_TOL


def test_expired_wait_is_reported_and_the_context_recovers(job):
    p, ref = job
    ctx = fg.Context(0)
    try:
        _ok(ctx, p, ref)
        ctx.tune(fg.AG_TUNE_TEST_IDLE_WAIT, 4)
        with pytest.raises(fg.AgError) as ei:
            ctx.emap(p.grid, p.xyzw(), p.inv_eps())
        assert ei.value.code == fg.AG_E_DEVICE
        assert "bounded wait expired" in str(ei.value)
        ctx.tune(fg.AG_TUNE_TEST_IDLE_WAIT, 0)
        _ok(ctx, p, ref)
    finally:
        ctx.close()


def test_checksum_mismatch_is_reported(job):
    p, ref = job
    ctx = fg.Context(0)
    try:
        ctx.tune(fg.AG_TUNE_TEST_CHECKSUM_OFFSET, 0.5)
        with pytest.raises(fg.AgError) as ei:
            ctx.emap(p.grid, p.xyzw(), p.inv_eps())
        assert ei.value.code == fg.AG_E_DEVICE
        assert "checksum mismatch" in str(ei.value)
        ctx.tune(fg.AG_TUNE_TEST_CHECKSUM_OFFSET, 0.0)
        _ok(ctx, p, ref)
    finally:
        ctx.close()


def test_fresh_context_ignores_stale_device_memory():
    """A new context's status word starts clear even when the memory it gets
    last held other data of this process: small device blocks are filled with
    0xFF and freed (through the CUDA runtime), then contexts are created and
    their first call is an e-map, which reads the status word back."""
    from cuda.bindings import runtime as rt

    rng = np.random.default_rng(3)
    eps = np.zeros(8192)
    oracle.lib().oracle_ddd_table(oracle._dp(eps))
    g = fg.Grid(17, 13, 11, 0.375)
    xyzw = np.concatenate([rng.uniform(-6, 6, (300, 3)), rng.normal(0, 0.1, (300, 1))], axis=1)
    ref = oracle.emap(g, xyzw, eps)
    for _ in range(4):
        ptrs = []
        for _ in range(16):
            err, p = rt.cudaMalloc(64)
            assert err == rt.cudaError_t.cudaSuccess
            assert rt.cudaMemset(p, 0xFF, 64)[0] == rt.cudaError_t.cudaSuccess
            ptrs.append(p)
        assert rt.cudaDeviceSynchronize()[0] == rt.cudaError_t.cudaSuccess
        for p in ptrs:
            assert rt.cudaFree(p)[0] == rt.cudaError_t.cudaSuccess
        ctx = fg.Context(0)
        try:
            got = ctx.emap(g, xyzw, eps)
            assert np.abs(got.astype(np.float64) - ref).max() <= E_TOL
        finally:
            ctx.close()
