"""GPU: the large benchmark configuration, every written value against the
reference's own maps.

The job is the benchmark's: 20,000 synthetic atoms in a 45 x 35 x 30 A
ellipsoid, a 161^3 grid at 0.375 A, ligand types A C HD N NA OA SA S F Cl
(10 affinity maps + e-map + d-map).  FastGrid's CPU build (oracle/_ref/
fastgrid4, compiled from the reference sources: CalculateGridmaps.cpp:433-485,
electrostatics/Cpu.cpp:27-88, writer GridMap.cpp:183-212) and the engine's
fastgrid4 command line both run on the same GPF, and all 12 maps are compared
value by value, with the .xyz file and the .fld file.

Rule (values in written thousandths): equal; or, for the e-map, one thousandth
apart only where the engine's unrounded value lies within 1e-4 kcal/mol/e of
the rounding boundary between the two; for affinity maps and the d-map, within
max(1e-3, 1e-4 |v|) kcal/mol (the affinity tolerance).  The unrounded GPU e-map
is also compared with the FP64 oracle on every grid point (within 1e-4
kcal/mol/e), and the per-map error of the unrounded GPU values against the
FP64 oracle on sampled points is printed.
"""
import os
import shutil
import subprocess
import time

import numpy as np
import pytest

from conftest import AFF_ABS, AFF_REL, E_TOL, REPO, chdir

import fastgrid_b200 as fg
import oracle

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(REPO, "oracle", "_ref", "fastgrid4")
TYPES = "A C HD N NA OA SA S F Cl"


def test_large_config_every_value_vs_fastgrid_cpu(tmp_path):
    if not os.path.exists(REF_BIN):
        pytest.skip("oracle/_ref/fastgrid4 not built (needs the reference sources)")
    ref_dir, cli_dir = tmp_path / "ref", tmp_path / "cli"
    fg.synth_write(str(ref_dir), "c1", n_atoms=20000, semi_axes=(45, 35, 30), npts=160, seed=2, ligand_types=TYPES)
    os.makedirs(cli_dir)
    for f in ("c1.gpf", "c1.pdbqt"):
        shutil.copy(ref_dir / f, cli_dir / f)

    t0 = time.perf_counter()
    r = subprocess.run([REF_BIN, "-p", "c1.gpf", "-l", "ref.glg"], cwd=ref_dir, capture_output=True, text=True)
    t_ref = time.perf_counter() - t0
    assert r.returncode == 0, r.stderr[-2000:]
    t0 = time.perf_counter()
    r = subprocess.run([fg.CLI_PATH, "-p", "c1.gpf", "-l", "cli.glg"], cwd=cli_dir, capture_output=True, text=True)
    t_cli = time.perf_counter() - t0
    assert r.returncode == 0, r.stderr[-2000:]
    print(f"\nwall time: FastGrid CPU {t_ref:.1f} s, engine command line {t_cli:.2f} s")

    # Unrounded GPU values of the same job (for the rounding-boundary rule).
    with chdir(str(cli_dir)):
        p = fg.Problem("c1.gpf", log="p.glg")
    ctx = fg.Context(0)
    try:
        p.compute(ctx)
    finally:
        ctx.close()
    gpu = p.maps().reshape(p.n_maps + 2, -1).astype(np.float64)
    names = [f"c1.{t}.map" for t in TYPES.split()] + ["c1.e.map", "c1.d.map"]
    assert len(names) == p.n_maps + 2

    for m, n in enumerate(names):
        ref = oracle.read_map(str(ref_dir / n))
        mine = oracle.read_map(str(cli_dir / n))
        assert ref.size == mine.size == p.npoints, n
        kr = np.round(ref * 1000).astype(np.int64)
        km = np.round(mine * 1000).astype(np.int64)
        u = gpu[m]
        # The command line writes the rounded unrounded values of the same computation.
        assert np.array_equal(km, np.round(oracle.round3(u) * 1000).astype(np.int64)), n
        diff = np.abs(km - kr)
        if n == "c1.e.map":
            lo = np.minimum(km, kr)
            boundary = (lo + 0.5) / 1000.0
            ok = (diff == 0) | ((diff == 1) & (np.abs(u - boundary) <= E_TOL))
        else:
            tol = np.maximum(AFF_ABS, AFF_REL * np.abs(u))
            ok = diff <= np.maximum(1, np.ceil(tol * 1000))
        bad = np.nonzero(~ok)[0]
        print(f"{n}: {np.count_nonzero(diff == 0)} of {diff.size} equal, {np.count_nonzero(diff == 1)} one "
              f"thousandth apart, max {diff.max()}")
        assert bad.size == 0, f"{n}: {bad.size} values differ beyond the rule, first at {bad[:5]}"

    assert open(ref_dir / "c1.maps.xyz").read() == open(cli_dir / "c1.maps.xyz").read()
    strip = lambda path: [l for l in open(path).read().split("\n") if not l.startswith("# Created by")]
    assert strip(ref_dir / "c1.maps.fld") == strip(cli_dir / "c1.maps.fld")

    # The e-map against the FP64 oracle on every grid point (mid atoms take
    # FP32 round-down bins, whose rare off-by-one events this bounds).
    e_all = gpu[p.n_maps]
    worst, sq = 0.0, 0.0
    for s in range(0, p.npoints, 1 << 21):
        ix = np.arange(s, min(p.npoints, s + (1 << 21)))
        dd = np.abs(e_all[ix] - oracle.emap_points(p.grid, p.xyzw(), p.inv_eps(), ix))
        worst, sq = max(worst, float(dd.max())), sq + float((dd * dd).sum())
    print(f"c1.e.map, every point: max |d| {worst:.3g}, rms {(sq / p.npoints) ** 0.5:.3g} vs the FP64 oracle")
    assert worst <= E_TOL

    # Per-map error of the unrounded GPU values against the FP64 oracle, sampled.
    rng = np.random.default_rng(3)
    idx = np.sort(rng.choice(p.npoints, 2000, replace=False))
    om, od = oracle.affinity_points(p.grid, p.receptor, p.params, idx)
    oe = oracle.emap_points(p.grid, p.xyzw(), p.inv_eps(), idx)
    for m, n in enumerate(names):
        ref = om[m] if m < p.n_maps else (oe if m == p.n_maps else od)
        d = gpu[m, idx] - ref
        print(f"{n}: max |d| {np.abs(d).max():.3g}, rms {np.sqrt((d * d).mean()):.3g} vs the FP64 oracle")
        tol = E_TOL if m == p.n_maps else np.maximum(AFF_ABS, AFF_REL * np.abs(ref))
        assert (np.abs(d) <= tol).all(), n
