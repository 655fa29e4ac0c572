"""CPU: the oracle (FP64 restatement) fed by the engine's host preprocessing
reproduces every golden map exactly after the reference's rounding.

Pins both the oracle and the C++ loader / parameter library / tables / bond
vectors against FastGrid's and AutoGrid 4.2.1's own outputs.
"""
import re

import numpy as np
import pytest

from conftest import CASES, chdir, golden_tol, golden_values, map_names, materialize, sha, thousandths

import fastgrid_b200 as fg
import oracle


def _covalent(problem, case):
    m = re.search(r"^covalentmap\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)", case["gpf"], re.M)
    hw, barrier, x, y, z = (float(v) for v in m.groups())
    c = problem.info.center
    cov = np.array([x - c[0], y - c[1], z - c[2]])
    g = problem.grid
    ix, iy, iz = np.meshgrid(np.arange(g.nx), np.arange(g.ny), np.arange(g.nz), indexing="ij")
    gx = (ix - g.nx // 2) * g.spacing
    gy = (iy - g.ny // 2) * g.spacing
    gz = (iz - g.nz // 2) * g.spacing
    r = ((cov[0] - gx) ** 2 + (cov[1] - gy) ** 2 + (cov[2] - gz) ** 2) * (1 / hw ** 2)
    r = np.maximum(r, 1e-12)
    e = barrier * (1 - np.exp(-0.69314718055994529 * r))
    return e.transpose(2, 1, 0).ravel()


def oracle_maps(problem, case):
    maps, dmap = oracle.affinity(problem.grid, problem.receptor, problem.params)
    e = oracle.emap(problem.grid, problem.xyzw(), problem.inv_eps())
    names, en, dn = map_names(case)
    out = {}
    for i, n in enumerate(names):
        out[n] = maps[i]
        if problem.params.map_is_covalent[i]:
            out[n] = _covalent(problem, case)
    out[en] = e
    out[dn] = dmap
    return out


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(name, tmp_path):
    work, gpf, case = materialize(name, str(tmp_path))
    with chdir(work):
        p = fg.Problem(gpf, v4=case["v4"], log="glg.txt")
    om = oracle_maps(p, case)
    for m, rec in case["maps"].items():
        k = thousandths(om[m])
        idx, gv = golden_values(rec)
        assert k.size == rec["n"], m
        tol = golden_tol(rec)
        if tol is None:  # written by an older H-bond model: not pinned
            continue
        if tol > 0:
            assert np.abs(k[idx] - gv).max() <= tol, f"{name} {m}: sampled values beyond {tol} thousandths"
            continue
        bad = np.nonzero(k[idx] != gv)[0]
        assert bad.size == 0, f"{name} {m}: {bad.size} sampled values differ, first at {idx[bad[0]]}: {k[idx[bad[0]]]} vs {gv[bad[0]]}"
        assert sha(k) == rec["sha256"], f"{name} {m}: full-map hash differs"


def test_tables_restated(tmp_path):
    work, gpf, case = materialize("synth_c0", str(tmp_path))
    with chdir(work):
        p = fg.Problem(gpf, log="glg.txt")
    eps = np.zeros(8192)
    oracle.lib().oracle_ddd_table(oracle._dp(eps))
    assert np.array_equal(eps, p.inv_eps())
    sol = np.zeros(8192)
    oracle.lib().oracle_sol_table(0.1322, oracle._dp(sol))
    got = np.ctypeslib.as_array(p.params.sol, shape=(8192,))
    assert np.array_equal(sol, got)
    # C-C 12-6 table with the 0.5 A smoothing window; receptor/map parameters
    # from the AD4.1 library: Rij = 4.0, eps = 0.150 * 0.1662.
    t = np.zeros(8192)
    oracle.lib().oracle_pair_table(12, 6, 4.0, np.sqrt(0.150 * 0.1662 * 0.150 * 0.1662), 0.5, oracle._dp(t))
    e = np.ctypeslib.as_array(p.params.energy, shape=(p.info.n_types, 8192, p.n_maps))
    types = [l.split()[-1] for l in open(f"{work}/synth_c0.pdbqt")]
    ctype = list(dict.fromkeys(types)).index("C")  # receptor index = order of first appearance
    cmap = 1  # ligand_types A C HD N OA SA
    assert np.array_equal(t, e[ctype, :, cmap])


def test_brute_force_and_cell_list_oracles_agree(tmp_path):
    work, gpf, case = materialize("synth_c0", str(tmp_path))
    with chdir(work):
        p = fg.Problem(gpf, log="glg.txt")
    rng = np.random.default_rng(3)
    idx = np.sort(rng.choice(p.npoints, 3000, replace=False))
    m1, d1 = oracle.affinity_points(p.grid, p.receptor, p.params, idx)
    m0, d0 = oracle.affinity(p.grid, p.receptor, p.params)
    assert np.array_equal(m1, m0[:, idx])
    assert np.array_equal(d1, d0[idx])
    e0 = oracle.emap(p.grid, p.xyzw(), p.inv_eps())
    e1 = oracle.emap_points(p.grid, p.xyzw(), p.inv_eps(), idx)
    assert np.array_equal(e1, e0[idx])
