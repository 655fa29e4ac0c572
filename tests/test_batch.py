"""GPU: batches of map sets (persistent kernels under one CUDA graph).

Six receptors of uneven atom counts and grid sizes are computed as one batch;
every map set must match the FP64 oracle (every point of the grids up to
51^3, 2,000 sampled points of the larger ones; the parity tests' tolerances)
and the single-job path, a replay of the captured graph must reproduce the
first run bit for bit, and the autotuner's cache file must round-trip.  Every
batch computation also passes the net-charge checksum of each job's e-map
(ag_batch_compute fails otherwise).
"""
import os

import numpy as np
import pytest

from conftest import AFF_ABS, AFF_REL, E_TOL, chdir

import fastgrid_b200 as fg
import oracle

pytestmark = pytest.mark.gpu

JOBS = [(1200, 41, 11), (5000, 63, 12), (2500, 51, 13), (9000, 45, 14), (1500, 81, 15), (7000, 71, 16)]


def _problems(tmp):
    out = []
    for k, (n, g, seed) in enumerate(JOBS):
        r = 20.0 * (n / 2000.0) ** (1 / 3)
        fg.synth_write(str(tmp), f"b{k}", n_atoms=n, semi_axes=(r, r, r), npts=g - 1, seed=seed)
        with chdir(str(tmp)):
            out.append(fg.Problem(f"b{k}.gpf", log=f"b{k}.glg"))
    return out


def _check_against_oracle(p, got, i):
    nm = p.n_maps
    if p.grid.nx <= 51:
        idx = np.arange(p.npoints)
        om, od = oracle.affinity(p.grid, p.receptor, p.params)
        oe = oracle.emap(p.grid, p.xyzw(), p.inv_eps())
    else:
        idx = np.sort(np.random.default_rng(i).choice(p.npoints, 2000, replace=False))
        om, od = oracle.affinity_points(p.grid, p.receptor, p.params, idx)
        oe = oracle.emap_points(p.grid, p.xyzw(), p.inv_eps(), idx)
    flat = got.reshape(nm + 2, -1)
    for m in range(nm):
        d = np.abs(flat[m, idx] - om[m])
        assert (d <= np.maximum(AFF_ABS, AFF_REL * np.abs(om[m]))).all(), (i, m, d.max())
    assert np.abs(flat[nm, idx] - oe).max() <= E_TOL, (i, np.abs(flat[nm, idx] - oe).max())
    assert (np.abs(flat[nm + 1, idx] - od) <= np.maximum(AFF_ABS, AFF_REL * np.abs(od))).all(), i


def test_batch_matches_oracle_and_single_jobs(tmp_path):
    ctx = fg.Context(0)
    probs = _problems(tmp_path)
    single = []
    for p in probs:
        p.compute(ctx)
        single.append(p.maps())
    b = fg.Batch(ctx, probs)
    b.compute()
    first = [b.maps(i) for i in range(len(probs))]
    b.compute()
    for i, p in enumerate(probs):
        again = b.maps(i)
        assert np.array_equal(again, first[i]), f"graph replay differs for job {i}"
        ref = single[i].astype(np.float64)
        got = first[i].astype(np.float64)
        _check_against_oracle(p, got, i)
        nm = p.n_maps
        d = np.abs(got[:nm] - ref[:nm])
        assert (d <= np.maximum(AFF_ABS, AFF_REL * np.abs(ref[:nm]))).all(), (i, d.max())
        assert np.abs(got[nm] - ref[nm]).max() <= E_TOL, (i, np.abs(got[nm] - ref[nm]).max())
        assert np.abs(got[nm + 1] - ref[nm + 1]).max() <= AFF_ABS
    cache = os.path.join(str(tmp_path), "tune.txt")
    b.autotune(cache)
    assert os.path.exists(cache) and "emap_tile" in open(cache).read()
    b.compute()
    for i, p in enumerate(probs):
        got = b.maps(i).astype(np.float64)
        ref = single[i].astype(np.float64)
        assert np.abs(got[p.n_maps] - ref[p.n_maps]).max() <= E_TOL
    b.autotune(cache)  # second call reads the cache
    b.close()
    ctx.close()
