"""GPU: batches of map sets (persistent kernels under one CUDA graph).

Six receptors of uneven atom counts and grid sizes are computed as one batch;
every map set must match the single-job path (same tolerances as the parity
tests), a replay of the captured graph must reproduce the first run bit for
bit, and the autotuner's cache file must round-trip.
"""
import os

import numpy as np
import pytest

from conftest import AFF_ABS, AFF_REL, E_TOL, chdir

import fastgrid_b200 as fg

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


def test_batch_matches_single_jobs(tmp_path):
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
