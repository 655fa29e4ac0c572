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
