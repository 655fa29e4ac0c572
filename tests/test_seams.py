"""GPU: FastGrid's own driver on the engine.

oracle/_ref/fastgrid4_seams is FastGrid's main.cpp, loader, parameter
library, tables, bond vectors and writers, compiled from the reference
sources, with its two map-calculation seams (calculateElectrostaticMapAsync /
synchronizeCalculation, electrostatics/Electrostatics.h:32-36, and
calculateGridmaps, CalculateGridmaps.h:30-31) implemented on the engine's C ABI
by fastgrid_b200/integration/fastgrid_seams.cpp.  On the reference's own
regression cases it must write the golden maps.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import AFF_REL, REPO, golden_tol, golden_values, map_names, materialize

import oracle

pytestmark = pytest.mark.gpu

SEAMS = os.path.join(REPO, "oracle", "_ref", "fastgrid4_seams")


@pytest.mark.parametrize("name", ["colagen2", "hsg1_sm", "1pgp", "x1hpv", "synth_covalent"])
def test_fastgrid_driver_on_the_engine_writes_the_golden_maps(name, tmp_path):
    if not os.path.exists(SEAMS):
        pytest.skip("oracle/_ref/fastgrid4_seams not built (needs the reference sources)")
    work, gpf, case = materialize(name, str(tmp_path))
    args = [SEAMS, "-p", gpf, "-l", "seams.glg"] + (["--v4"] if case["v4"] else [])
    r = subprocess.run(args, cwd=work, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Successful Completion" in open(os.path.join(work, "seams.glg")).read()
    names, en, dn = map_names(case)
    for n in names + [en, dn]:
        rec = case["maps"][n]
        tol = golden_tol(rec)
        if tol is None:
            continue
        v = oracle.read_map(os.path.join(work, n))
        assert v.size == rec["n"], n
        idx, gv = golden_values(rec)
        k = np.round(v[idx] * 1000).astype(np.int64)
        assert (np.abs(k - gv) <= np.maximum(max(1, tol), np.ceil(AFF_REL * np.abs(gv)))).all(), n
