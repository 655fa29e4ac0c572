"""GPU: the allocation-free e-map entry point (ag_emap_noalloc).

Callers that cannot call cudaMalloc — hosts that own the GPU's memory in
their own pool or run under a fixed memory budget — pass device buffers and
the library uses its fixed device arrays for scratch.  This checks, through
the C ABI, that two calls in a row (different grids, so the second call runs
over the first call's leftovers in the shared arrays) reproduce the ordinary
entry point ag_emap within the e-map tolerance, 1e-4 kcal/mol/e, and agree
with the FP64 oracle on sampled points within the same tolerance.

Collected last (file name) so that a run stopping at the first failure has
already run every other test; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import E_TOL, chdir

import fastgrid_b200 as fg
import oracle

pytestmark = pytest.mark.gpu


def _case(tmp, stem, n_atoms, npts, seed):
    fg.synth_write(str(tmp), stem, n_atoms=n_atoms, semi_axes=(14, 12, 11), npts=npts, seed=seed)
    with chdir(str(tmp)):
        return fg.Problem(stem + ".gpf", log=stem + ".glg")


def test_noalloc_matches_emap_twice(tmp_path):
    import torch

    ctx = fg.Context(0)
    rng = np.random.default_rng(5)
    # A small grid (the atom-split path, which uses the FP64 partial-sum array)
    # then a larger one (a single split) on the same shared arrays.
    for stem, n_atoms, npts, seed in (("na1", 1500, 40, 21), ("na2", 3000, 64, 22)):
        p = _case(tmp_path, stem, n_atoms, npts, seed)
        xyzw = p.xyzw()
        eps = p.inv_eps()
        ref = ctx.emap(p.grid, xyzw, eps)
        d_xyzw = torch.tensor(xyzw, dtype=torch.float64, device="cuda:0").contiguous()
        d_eps = torch.tensor(eps, dtype=torch.float32, device="cuda:0").contiguous()
        d_out = torch.full((p.npoints,), float("nan"), dtype=torch.float32, device="cuda:0")
        stream = torch.cuda.current_stream().cuda_stream
        rc = fg.lib().ag_emap_noalloc(C.byref(p.grid), xyzw.shape[0], C.c_void_p(d_xyzw.data_ptr()),
                                      C.c_void_p(d_eps.data_ptr()), C.c_void_p(d_out.data_ptr()), C.c_void_p(stream))
        assert rc == fg.AG_OK, fg.lib().ag_last_error()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert np.isfinite(got).all()
        assert np.abs(got.astype(np.float64) - ref).max() <= E_TOL, (stem, np.abs(got - ref).max())
        idx = rng.choice(p.npoints, size=800, replace=False)
        want = oracle.emap_points(p.grid, xyzw, eps, idx)
        assert np.abs(got[idx].astype(np.float64) - want).max() <= E_TOL, stem
    ctx.close()


def test_noalloc_rejects_oversized_grid():
    import torch

    # Rejected by the argument checks, which run before any CUDA call: nothing
    # is read or written on the device.
    out = torch.zeros(16, dtype=torch.float32, device="cuda:0")
    g = fg.Grid(1025, 1025, 1025, 0.375)
    rc = fg.lib().ag_emap_noalloc(C.byref(g), 0, None, None, C.c_void_p(out.data_ptr()), None)
    assert rc == -1
    assert b"too large" in fg.lib().ag_last_error()
