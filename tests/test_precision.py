"""GPU: precision study of the e-map (the 60,000-atom configuration).

Receptor: 60,000 atoms in a 55 A globule, charges N(0, 0.25) clipped to
+-0.9 with net charge +12; grid 255^3 at 0.375 A; e-map only, no cutoff.
Kahan-compensated FP32 (the production mode) and plain FP32 are compared with
the FP64 oracle on 4,000 points: 3,000 uniform samples plus the 1,000 points
with the largest |e| (next to atoms, where the terms are largest).  The max
and RMS errors of both modes are printed as one JSON line; the production
mode must stay within 1e-4 kcal/mol/e.
"""
import json
import time

import numpy as np
import pytest

from conftest import E_TOL, chdir

import fastgrid_b200 as fg
import oracle

pytestmark = pytest.mark.gpu


def test_precision_study(tmp_path):
    fg.synth_write(str(tmp_path), "c2", n_atoms=60000, semi_axes=(55, 55, 55), npts=254, seed=31,
                   charge_sigma=0.25, charge_clip=0.9, net_charge=12.0, ligand_types="C")
    with chdir(str(tmp_path)):
        p = fg.Problem("c2.gpf", log="c2.glg")
    ctx = fg.Context(0)
    xyzw, eps = p.xyzw(), p.inv_eps()
    t0 = time.perf_counter()
    kahan = ctx.emap(p.grid, xyzw, eps, mode=fg.AG_EMAP_KAHAN)
    t1 = time.perf_counter()
    plain = ctx.emap(p.grid, xyzw, eps, mode=fg.AG_EMAP_PLAIN)
    t2 = time.perf_counter()
    ctx.close()
    rng = np.random.default_rng(5)
    idx = np.unique(np.concatenate([rng.choice(p.npoints, 3000, replace=False),
                                    np.argsort(-np.abs(kahan))[:1000]]))
    ref = oracle.emap_points(p.grid, xyzw, eps, idx)
    report = {"config": "60000 atoms, r=55 A globule, net charge +12, 255^3 @0.375 A, e-map only",
              "points_checked": int(idx.size), "pairs_per_map": int(xyzw.shape[0]) * p.npoints}
    for name, v, secs in (("fp32_kahan", kahan, t1 - t0), ("fp32_plain", plain, t2 - t1)):
        d = v[idx].astype(np.float64) - ref
        report[name] = {"max_abs_err": float(np.abs(d).max()), "rms_err": float(np.sqrt(np.mean(d * d))),
                        "call_s": secs}
    print("PRECISION " + json.dumps(report))
    assert report["fp32_kahan"]["max_abs_err"] <= E_TOL
    assert report["fp32_kahan"]["rms_err"] <= report["fp32_plain"]["rms_err"] + 1e-7
