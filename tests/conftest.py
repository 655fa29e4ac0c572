"""Shared test helpers: materialise golden cases into temp dirs, compare maps.

Markers: ``gpu`` — needs a CUDA device (run with ``-m gpu``); everything else
runs on the CPU.
"""
import contextlib
import hashlib
import json
import lzma
import os
import shutil
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
sys.path.insert(0, REPO)

CASES = ["colagen2", "hsg1_sm", "1pgp", "x1hpv", "synth_c0", "synth_const_diel", "synth_covalent",
         "synth_paramfile_v4", "synth_disorder_h"]

# Tolerances (unrounded values against the FP64 oracle):
#   electrostatics: 1e-4 kcal/mol/e absolute
#   affinity and desolvation: 1e-4 relative or 1e-3 kcal/mol absolute, whichever is larger
E_TOL = 1e-4
AFF_REL, AFF_ABS = 1e-4, 1e-3


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    import fastgrid_b200.build as b
    b.build()
    import oracle
    oracle.build()
    yield


def load_case(name):
    return json.load(open(os.path.join(GOLDEN, name + ".json")))


def materialize(name, dest):
    """Write the case's inputs into `dest`; return (workdir, gpf filename, case dict)."""
    case = load_case(name)
    os.makedirs(dest, exist_ok=True)
    if name == "colagen2":
        with open(os.path.join(dest, case["pdbqt_name"]), "wb") as f:
            f.write(lzma.decompress(open(os.path.join(GOLDEN, case["pdbqt"]), "rb").read()))
        work = os.path.join(dest, case["subdir"])
        os.makedirs(work, exist_ok=True)
        with open(os.path.join(dest, "colagen2.gpf"), "w") as f:
            f.write(case["gpf"])
        return work, "../colagen2.gpf", case
    if name == "hsg1_sm":
        for f in case["files"]:
            shutil.copy(os.path.join(GOLDEN, "hsg1_sm", f), os.path.join(dest, f))
            os.chmod(os.path.join(dest, f), 0o644)
        with open(os.path.join(dest, "hsg1_sm.gpf"), "w") as f:
            f.write(case["gpf"])
        return dest, "hsg1_sm.gpf", case
    if "files_dir" in case:  # reference test receptors: files (some xz-compressed) + the GPF
        for f in case["files"]:
            src = os.path.join(GOLDEN, case["files_dir"], f)
            if f.endswith(".xz"):
                with open(os.path.join(dest, f[:-3]), "wb") as o:
                    o.write(lzma.decompress(open(src, "rb").read()))
            else:
                shutil.copy(src, os.path.join(dest, f))
                os.chmod(os.path.join(dest, f), 0o644)
        stem = name + ".gpf"
        with open(os.path.join(dest, stem), "w") as f:
            f.write(case["gpf"])
        return dest, stem, case
    import fastgrid_b200 as fg
    gen = dict(case["gen"])
    gen["semi_axes"] = tuple(gen["semi_axes"])
    if "origin" in gen:
        gen["origin"] = tuple(gen["origin"])
    fg.synth_write(dest, name, **gen)
    with open(os.path.join(dest, name + ".gpf"), "w") as f:
        f.write(case["gpf"])
    for f in case.get("files", []):
        shutil.copy(os.path.join(GOLDEN, "hsg1_sm", f), os.path.join(dest, f))
        os.chmod(os.path.join(dest, f), 0o644)
    return dest, name + ".gpf", case


@contextlib.contextmanager
def chdir(path):
    old = os.getcwd()
    os.chdir(path)
    try:
        yield
    finally:
        os.chdir(old)


def thousandths(values):
    """Map values as written (roundOutput then %.3f) in integer thousandths."""
    a = np.asarray(values, dtype=np.float64)
    r = np.where(np.abs(a) < 0.0005, 0.0, np.floor(a * 1000 + 0.5) * 0.001)
    return np.round(r * 1000.0).astype(np.int64)


def sha(k):
    return hashlib.sha256(np.ascontiguousarray(k, dtype=np.int64).tobytes()).hexdigest()


def golden_values(rec):
    """(indices, values in thousandths) stored for a map record."""
    if "values" in rec:
        v = np.array(rec["values"], dtype=np.int64)
        return np.arange(v.size), v
    return np.array(rec["sample_idx"], dtype=np.int64), np.array(rec["sample_values"], dtype=np.int64)


def golden_tol(rec):
    """Allowed difference in thousandths between a golden map and the reference
    restatement: 0 (exact), k, or None when the map is not pinned."""
    return rec.get("tol", 0)


def map_names(case):
    import re
    g = case["gpf"]
    return (re.findall(r"^map\s+(\S+)", g, re.M), re.findall(r"^elecmap\s+(\S+)", g, re.M)[0],
            re.findall(r"^dsolvmap\s+(\S+)", g, re.M)[0])


def aff_tol(ref):
    return np.maximum(AFF_ABS, AFF_REL * np.abs(ref))
