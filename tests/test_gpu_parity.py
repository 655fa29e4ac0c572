"""GPU parity: the engine's CUDA path against the pinned FP64 oracle and the
reference's golden maps.

Tolerances (unrounded GPU values against the oracle):
  e-map:               |d| <= 1e-4 kcal/mol/e
  affinity and d-map:  |d| <= max(1e-3 kcal/mol, 1e-4 * |value|)
Written maps (rounded to 3 decimals) against the reference's files: equal, or
one thousandth apart where the unrounded value sits within the tolerance of a
rounding boundary (e-map), or within the affinity tolerance above.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import (AFF_ABS, AFF_REL, CASES, E_TOL, chdir, golden_tol, golden_values, map_names, materialize,
                      thousandths)

import fastgrid_b200 as fg
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = fg.Context(0)
    yield c
    c.close()


def _check_maps(gpu, orc, names, en, dn, label):
    for i, n in enumerate(names):
        ref = orc[n]
        d = np.abs(gpu[i].ravel().astype(np.float64) - ref)
        tol = np.maximum(AFF_ABS, AFF_REL * np.abs(ref))
        bad = np.nonzero(d > tol)[0]
        assert bad.size == 0, f"{label} {n}: {bad.size} points off, worst {d.max():.3g} at {np.argmax(d)}"
    de = np.abs(gpu[len(names)].ravel().astype(np.float64) - orc[en])
    assert de.max() <= E_TOL, f"{label} e-map max |d| {de.max():.3g} > {E_TOL}"
    dd = np.abs(gpu[len(names) + 1].ravel().astype(np.float64) - orc[dn])
    assert (dd <= np.maximum(AFF_ABS, AFF_REL * np.abs(orc[dn]))).all(), f"{label} d-map max |d| {dd.max():.3g}"


@pytest.mark.parametrize("name", CASES)
def test_map_set_matches_oracle_and_golden(name, tmp_path, ctx):
    from test_oracle import oracle_maps
    work, gpf, case = materialize(name, str(tmp_path))
    with chdir(work):
        p = fg.Problem(gpf, v4=case["v4"], log="glg.txt")
    p.compute(ctx)
    gpu = p.maps().reshape(p.n_maps + 2, -1)
    orc = oracle_maps(p, case)
    names, en, dn = map_names(case)
    _check_maps(gpu, orc, names, en, dn, name)
    # Written values against the reference's own maps.
    for i, n in enumerate(names + [en, dn]):
        tol = golden_tol(case["maps"][n])
        if tol is None:  # not pinned by the reference's file (older H-bond model)
            continue
        idx, gv = golden_values(case["maps"][n])
        k = thousandths(gpu[i][idx])
        diff = np.abs(k - gv)
        if n == en:
            ok = diff <= max(1, tol)
        else:
            ok = diff <= np.maximum(max(1, tol), np.ceil(AFF_REL * np.abs(gv)))
        assert ok.all(), f"{name} {n}: written values differ at {idx[~ok][:5]}"


@pytest.mark.parametrize("name", ["colagen2", "hsg1_sm", "synth_disorder_h", "synth_paramfile_v4"])
def test_one_point_affinity_kernel_matches_oracle(name, tmp_path):
    """The one-point affinity kernel (a separate nearest-donor kernel, one
    grid point per thread), still used for passes with more than four H-bond
    maps and by the batch kernel, against the oracle (the default two-point
    kernel is covered by the test above)."""
    from test_oracle import oracle_maps
    work, gpf, case = materialize(name, str(tmp_path))
    with chdir(work):
        p = fg.Problem(gpf, v4=case["v4"], log="glg.txt")
    c = fg.Context(0)
    try:
        c.tune(fg.AG_TUNE_AFFINITY_KERNEL, 1)
        p.compute(c)
    finally:
        c.close()
    names, en, dn = map_names(case)
    _check_maps(p.maps().reshape(p.n_maps + 2, -1), oracle_maps(p, case), names, en, dn, name + " (one-point)")


def test_many_hbond_maps(tmp_path):
    """Seven H-bond probe maps (HD HS NA NS OA OS SA): more than the two-point
    kernel's four H-bond slots, so that pass falls back to the one-point
    kernel; both settings must match the oracle."""
    fg.synth_write(str(tmp_path), "hb", n_atoms=1500, semi_axes=(14, 13, 12), npts=30, seed=17,
                   ligand_types="A C HD HS NA NS OA OS SA")
    with chdir(str(tmp_path)):
        p = fg.Problem("hb.gpf", log="hb.glg")
    om, od = oracle.affinity(p.grid, p.receptor, p.params)
    for k in (2, 1):
        c = fg.Context(0)
        try:
            c.tune(fg.AG_TUNE_AFFINITY_KERNEL, k)
            p.compute(c)
        finally:
            c.close()
        gpu = p.maps().reshape(p.n_maps + 2, -1).astype(np.float64)
        for m in range(p.n_maps):
            d = np.abs(gpu[m] - om[m])
            assert (d <= np.maximum(AFF_ABS, AFF_REL * np.abs(om[m]))).all(), (k, m, d.max())
        assert (np.abs(gpu[p.n_maps + 1] - od) <= np.maximum(AFF_ABS, AFF_REL * np.abs(od))).all(), k


def test_emap_edge_cases(ctx):
    """Atoms on a grid point, within 0.01 A of one, at r = 0.5 A (the 1/r cap),
    beyond 81.91 A (the table clamp), and grids that are not multiples of the
    kernel's tiles."""
    rng = np.random.default_rng(0)
    eps = np.zeros(8192)
    oracle.lib().oracle_ddd_table(oracle._dp(eps))
    for (nx, ny, nz) in [(1, 1, 1), (3, 5, 7), (17, 9, 33), (41, 41, 41)]:
        g = fg.Grid(nx, ny, nz, 0.375)
        pts = []
        for k in range(4):
            x, y, z = rng.integers(0, nx), rng.integers(0, ny), rng.integers(0, nz)
            p = np.array([(x - nx // 2) * 0.375, (y - ny // 2) * 0.375, (z - nz // 2) * 0.375])
            pts += [p, p + [0.004, 0, 0], p + [0.5, 0, 0], p + [0, 0.3, 0.4]]
        pts += [[90.0, 5.0, -3.0], [-60.0, 60.0, 10.0]]
        pts = np.array(pts)
        xyzw = np.concatenate([pts, rng.normal(0, 0.03, (len(pts), 1))], axis=1)
        xyzw = np.concatenate([xyzw, np.concatenate([rng.uniform(-15, 15, (300, 3)),
                                                      rng.normal(0, 0.03, (300, 1))], axis=1)])
        got = ctx.emap(g, xyzw, eps)
        ref = oracle.emap(g, xyzw, eps)
        assert np.abs(got - ref).max() <= E_TOL, (nx, ny, nz, np.abs(got - ref).max())
        got = ctx.emap(g, xyzw, None)
        ref = oracle.emap(g, xyzw, None)
        assert np.abs(got - ref).max() <= E_TOL * max(1.0, np.abs(ref).max() * 1e-3)


# Plain FP32 summation (AG_EMAP_PLAIN) of a few thousand atoms: its rounding
# error stays well inside this bound, and a wrongly scaled packed-table sum
# (a factor 2^16) or a missing term would not.
PLAIN_TOL = 5e-4


@pytest.mark.parametrize("order,tile,packed", [(0, 11616, 1), (1, 11616, 1), (2, 20816, 1), (2, 21608, 1),
                                               (2, 40808, 1), (1, 20816, 0), (2, 20816, 0)])
@pytest.mark.parametrize("mode", [fg.AG_EMAP_KAHAN, fg.AG_EMAP_PLAIN])
def test_emap_item_orders_tiles_and_packed_table(order, tile, packed, mode):
    """Every e-map item order (rows, warp-compact, x-interleaved lane pairs),
    several CTA tiles, and the FP32 table against its packed 16- and 8-bit
    tail copies, against the oracle in both summation modes, on grids whose x
    extent leaves partial and unpaired 8-point columns, with atoms in the
    near, mid, packed-mid (22-55 A from a CTA box) and far (saturated
    dielectric) classes."""
    rng = np.random.default_rng(7)
    eps = np.zeros(8192)
    oracle.lib().oracle_ddd_table(oracle._dp(eps))
    c = fg.Context(0)
    try:
        c.tune(fg.AG_TUNE_EMAP_WARP_COMPACT, order)
        c.tune(fg.AG_TUNE_EMAP_TILE, tile)
        c.tune(fg.AG_TUNE_EMAP_PACKED_TABLE, packed)
        inner = rng.normal(0, 9.0, (2500, 3))
        shell = rng.normal(0, 1.0, (900, 3))
        shell = shell / np.linalg.norm(shell, axis=1, keepdims=True) * rng.uniform(20, 62, (900, 1))
        outer = rng.normal(0, 1.0, (60, 3))
        outer = outer / np.linalg.norm(outer, axis=1, keepdims=True) * rng.uniform(55, 75, (60, 1))
        pts = np.concatenate([inner, shell, outer])
        xyzw = np.concatenate([pts, rng.normal(0, 0.05, (len(pts), 1))], axis=1)
        for (nx, ny, nz) in [(33, 45, 29), (45, 41, 37)]:
            g = fg.Grid(nx, ny, nz, 0.375)
            got = c.emap(g, xyzw, eps, mode=mode)
            ref = oracle.emap(g, xyzw, eps)
            tol = E_TOL if mode == fg.AG_EMAP_KAHAN else PLAIN_TOL
            assert np.abs(got - ref).max() <= tol, (order, tile, packed, (nx, ny, nz), np.abs(got - ref).max())
            if packed == 1 and mode == fg.AG_EMAP_KAHAN:
                got = c.emap(g, xyzw, None)
                ref = oracle.emap(g, xyzw, None)
                assert np.abs(got - ref).max() <= E_TOL * max(1.0, np.abs(ref).max() * 1e-3)
    finally:
        c.close()


@pytest.mark.parametrize("spacing", [1.0, 1.5, 2.0])
def test_emap_coarse_grids(spacing, ctx):
    """Coarse grids, whose CTA boxes are large: from 1.5 A a full box's
    diagonal is long enough that a mid atom's bin can pass the table's end
    (the clamped mid-list path, FP32 table only), while the smaller boxes at
    the grid's edges still read the packed tail tables; atoms spread over
    +-90 A so every class occurs."""
    rng = np.random.default_rng(11)
    eps = np.zeros(8192)
    oracle.lib().oracle_ddd_table(oracle._dp(eps))
    g = fg.Grid(45, 37, 41, spacing)
    pts = np.concatenate([rng.uniform(-35, 35, (2500, 3)), rng.uniform(-90, 90, (700, 3))])
    xyzw = np.concatenate([pts, rng.normal(0, 0.1, (len(pts), 1))], axis=1)
    got = ctx.emap(g, xyzw, eps)
    ref = oracle.emap(g, xyzw, eps)
    assert np.abs(got - ref).max() <= E_TOL, (spacing, np.abs(got - ref).max())


def test_large_config_sampled(tmp_path, ctx):
    """The large benchmark configuration (20,000 atoms, 161^3, 10 ligand maps)
    against the oracle on 1500 sampled points."""
    gpf = fg.synth_write(str(tmp_path), "c1", n_atoms=20000, semi_axes=(45, 35, 30), npts=160, seed=2,
                         ligand_types="A C HD N NA OA SA S F Cl")
    with chdir(str(tmp_path)):
        p = fg.Problem("c1.gpf", log="glg.txt")
    p.compute(ctx)
    gpu = p.maps().reshape(p.n_maps + 2, -1)
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(p.npoints, 1500, replace=False))
    om, od = oracle.affinity_points(p.grid, p.receptor, p.params, idx)
    oe = oracle.emap_points(p.grid, p.xyzw(), p.inv_eps(), idx)
    for m in range(p.n_maps):
        d = np.abs(gpu[m, idx] - om[m])
        assert (d <= np.maximum(AFF_ABS, AFF_REL * np.abs(om[m]))).all(), (m, d.max())
    assert np.abs(gpu[p.n_maps, idx] - oe).max() <= E_TOL
    assert np.abs(gpu[p.n_maps + 1, idx] - od).max() <= AFF_ABS


def test_kahan_vs_plain(tmp_path, ctx):
    """Compensated accumulation is at least as accurate as plain FP32."""
    gpf = fg.synth_write(str(tmp_path), "pk", n_atoms=12000, semi_axes=(30, 30, 30), npts=40, seed=4,
                         charge_sigma=0.25, charge_clip=0.9, net_charge=12.0)
    with chdir(str(tmp_path)):
        p = fg.Problem("pk.gpf", log="glg.txt")
    ref = oracle.emap(p.grid, p.xyzw(), p.inv_eps())
    k = ctx.emap(p.grid, p.xyzw(), p.inv_eps(), mode=fg.AG_EMAP_KAHAN)
    pl = ctx.emap(p.grid, p.xyzw(), p.inv_eps(), mode=fg.AG_EMAP_PLAIN)
    ek, ep = np.abs(k - ref).max(), np.abs(pl - ref).max()
    assert ek <= E_TOL
    assert ek <= ep + 1e-6


def test_cli_writes_reference_maps(tmp_path):
    """The fastgrid4 drop-in on FastGrid's own regression case writes the
    golden maps (and .fld / .xyz)."""
    work, gpf, case = materialize("colagen2", str(tmp_path))
    r = subprocess.run([fg.CLI_PATH, "-p", gpf, "-l", "log.glg", "--v4"], cwd=work, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    names, en, dn = map_names(case)
    for n in names + [en, dn]:
        v = oracle.read_map(os.path.join(work, n))
        idx, gv = golden_values(case["maps"][n])
        k = np.round(v[idx] * 1000).astype(np.int64)
        assert (np.abs(k - gv) <= np.maximum(1, np.ceil(AFF_REL * np.abs(gv)))).all(), n
        head = open(os.path.join(work, n)).read().split("\n")[:6]
        assert head[0] == "GRID_PARAMETER_FILE ../colagen2.gpf" and head[4] == "NELEMENTS 40 40 40"
    assert open(os.path.join(work, "colagen2.maps.xyz")).read() == "44.000 84.000\n-36.000 4.000\n17.000 57.000\n"


def test_cli_covalent_and_floating_grid(tmp_path):
    work, gpf, case = materialize("synth_covalent", str(tmp_path))
    r = subprocess.run([fg.CLI_PATH, "-p", gpf, "-l", "log.glg"], cwd=work, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    names, en, dn = map_names(case)
    for n in names + [en, dn]:
        v = oracle.read_map(os.path.join(work, n))
        idx, gv = golden_values(case["maps"][n])
        k = np.round(v[idx] * 1000).astype(np.int64)
        assert (np.abs(k - gv) <= np.maximum(1, np.ceil(AFF_REL * np.abs(gv)))).all(), n
    fgv = oracle.read_map(os.path.join(work, "synth_covalent.fg.map"))
    idx, gv = golden_values(case["floating_grid"])
    assert (np.abs(np.round(fgv[idx] * 1000).astype(np.int64) - gv) <= 1).all()
    fld = open(os.path.join(work, "synth_covalent.maps.fld")).read().split("\n")
    ref = case["fld"].split("\n")
    assert [l for l in fld if not l.startswith("# Created by")] == [l for l in ref if not l.startswith("# Created by")]


@pytest.mark.parametrize("kernel", [2, 1])
def test_concurrent_passes_equal_sequential(tmp_path, kernel):
    """The map set with the e-map and the affinity pass run concurrently (the
    default; the whole-job call also copies the affinity maps back in z-slab
    chunks) is bit-identical to the passes run one after the other, through
    ag_compute and through the whole-job call, for both affinity kernels."""
    fg.synth_write(str(tmp_path), "cc", n_atoms=2500, semi_axes=(16, 14, 12), npts=44, seed=23,
                   ligand_types="A C HD N NA OA SA")
    with chdir(str(tmp_path)):
        p = fg.Problem("cc.gpf", log="cc.glg")
    out = {}
    for conc in (0, 1):
        c = fg.Context(0)
        try:
            c.tune(fg.AG_TUNE_AFFINITY_KERNEL, kernel)
            c.tune(fg.AG_TUNE_CONCURRENT_PASSES, conc)
            c.upload(p.grid, p.receptor, p.params, p.inv_eps_ptr)
            c.compute(fg.AG_WORK_ALL)
            dev = np.empty((p.n_maps + 2) * p.npoints, dtype=np.float32)
            c.download(dev)
            p.compute(c)
            out[conc] = (dev, p.maps().astype(np.float32).ravel().copy())
        finally:
            c.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[1][0], out[1][1])
