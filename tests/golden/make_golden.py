"""Regenerate the golden fixtures in tests/golden/ from the reference.

Run in the build container (needs the reference checkout — $FASTGRID_REFERENCE,
default /root/reference — and the reference programs built by
``make -C oracle ref``):

    python tests/golden/make_golden.py

Fixtures written (all small):
  colagen2.json + colagen2.pdbqt.xz  FastGrid's own regression case
      (tests/colagen2.gpf.orig, tests/macromol_1t60_half_prot.pdbqt.orig, golden
      maps tests/original_win32/colagen2.{C,HD,OA,e,d}.map, run with --v4).
  hsg1_sm.json + hsg1_sm/           AutoGrid 4.2.1's test case
      (AG421/Tests/hsg1_sm.gpf, hsg1_sm.pdbqt, AD4.1_bound.dat, golden maps
      py_hsg1_sm.*.map).
  1pgp.json + 1pgp/                 AutoDock 4.0.1's test receptor
      (autogrid_original_r1_tag/autodock-4.0.1/Tests/1pgp.gpf, 1pgp_rec.pdbqt,
      AD4_parameters.dat, golden maps 1pgp_rec.{C,HD,OA,P,e,d}.map, run with
      --v4).  Written by AutoGrid 4.0, so only the e-map and d-map are pinned
      exactly; C and P agree within 8 thousandths (AutoGrid 4.0 rounding of the
      pair-energy tables) and HD and OA follow AutoGrid 4.0's older H-bond
      model, so they are not pinned ("tol": null).
  x1hpv.json + x1hpv/               AutoGrid 4.2.1's GPF tests x1hpv_CASE0..3
      (AG421/Tests/test_autogrid4.py:281-311): CASE0 must complete (golden maps
      = FastGrid's CPU build on it), CASE1-3 lack a map / elecmap / dsolvmap
      line and must fail.
  synth_*.json                      seeded synthetic receptors (regenerated by the
      tests from their parameters) with the maps FastGrid's CPU build
      (oracle/_ref/fastgrid4) writes for them.

For every map a fixture stores the SHA-256 of the values in thousandths
(int64, i.e. exactly what the .map file holds) plus up to 600 sampled
(index, value) pairs; maps of at most 1000 values are stored in full.
"""
import hashlib
import json
import lzma
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
REF = os.environ.get("FASTGRID_REFERENCE", "/root/reference")
FG4 = os.path.join(REPO, "oracle", "_ref", "fastgrid4")

import fastgrid_b200 as fg  # noqa: E402  (generator only)
from oracle import read_map  # noqa: E402


def map_record(values, full_limit=1000, nsample=600, seed=0, tol=0):
    """tol: 0 = pinned exactly (hash and values); k > 0 = pinned within k thousandths;
    None = not pinned (stored for reference only)."""
    k = np.round(np.asarray(values) * 1000.0).astype(np.int64)
    rec = {"n": int(k.size), "sha256": hashlib.sha256(k.tobytes()).hexdigest(), "tol": tol}
    if k.size <= full_limit:
        rec["values"] = k.tolist()
    else:
        rng = np.random.default_rng(seed)
        idx = np.sort(rng.choice(k.size, size=nsample, replace=False))
        rec["sample_idx"] = idx.tolist()
        rec["sample_values"] = k[idx].tolist()
    return rec


def gpf_maps(gpf_text):
    maps = re.findall(r"^map\s+(\S+)", gpf_text, re.M)
    e = re.findall(r"^elecmap\s+(\S+)", gpf_text, re.M)[0]
    d = re.findall(r"^dsolvmap\s+(\S+)", gpf_text, re.M)[0]
    return maps, e, d


def colagen2():
    gpf = open(os.path.join(REF, "tests", "colagen2.gpf.orig")).read()
    pdbqt = open(os.path.join(REF, "tests", "macromol_1t60_half_prot.pdbqt.orig"), "rb").read()
    with open(os.path.join(HERE, "colagen2.pdbqt.xz"), "wb") as f:
        f.write(lzma.compress(pdbqt, preset=9))
    maps, e, d = gpf_maps(gpf)
    gold = os.path.join(REF, "tests", "original_win32")
    out = {"gpf": gpf, "v4": True, "pdbqt": "colagen2.pdbqt.xz",
           "pdbqt_name": "macromol_1t60_half_prot.pdbqt", "subdir": "run",
           "maps": {}, "source": "tests/original_win32 (FastGrid regression golden)"}
    for m in maps + [e, d]:
        out["maps"][m] = map_record(read_map(os.path.join(gold, m)))
    json.dump(out, open(os.path.join(HERE, "colagen2.json"), "w"))


def hsg1_sm():
    t = os.path.join(REF, "autogrid_original_4_2_1_ref", "autogrid", "Tests")
    dst = os.path.join(HERE, "hsg1_sm")
    os.makedirs(dst, exist_ok=True)
    for f in ("hsg1_sm.pdbqt", "AD4.1_bound.dat"):
        shutil.copy(os.path.join(t, f), os.path.join(dst, f))
    gpf = open(os.path.join(t, "hsg1_sm.gpf")).read()
    maps, e, d = gpf_maps(gpf)
    out = {"gpf": gpf, "v4": False, "files": ["hsg1_sm.pdbqt", "AD4.1_bound.dat"], "maps": {},
           "source": "AG421/Tests/py_hsg1_sm.*.map (AutoGrid 4.2.1 test golden)"}
    for m in maps + [e, d]:
        out["maps"][m] = map_record(read_map(os.path.join(t, "py_" + m)))
    json.dump(out, open(os.path.join(HERE, "hsg1_sm.json"), "w"))


def pgp1():
    t = os.path.join(REF, "autogrid_original_r1_tag", "autodock-4.0.1", "Tests")
    dst = os.path.join(HERE, "1pgp")
    os.makedirs(dst, exist_ok=True)
    with open(os.path.join(dst, "1pgp_rec.pdbqt.xz"), "wb") as f:
        f.write(lzma.compress(open(os.path.join(t, "1pgp_rec.pdbqt"), "rb").read(), preset=9))
    shutil.copy(os.path.join(t, "AD4_parameters.dat"), os.path.join(dst, "AD4_parameters.dat"))
    gpf = open(os.path.join(t, "1pgp.gpf")).read()
    maps, e, d = gpf_maps(gpf)
    tol = {"1pgp_rec.C.map": 8, "1pgp_rec.P.map": 8, "1pgp_rec.HD.map": None, "1pgp_rec.OA.map": None}
    out = {"gpf": gpf, "v4": True, "files_dir": "1pgp", "files": ["1pgp_rec.pdbqt.xz", "AD4_parameters.dat"],
           "maps": {}, "source": "autogrid_original_r1_tag/autodock-4.0.1/Tests/1pgp_rec.*.map (AutoGrid 4.0 golden)"}
    for m in maps + [e, d]:
        out["maps"][m] = map_record(read_map(os.path.join(t, m)), tol=tol.get(m, 0))
    json.dump(out, open(os.path.join(HERE, "1pgp.json"), "w"))


def x1hpv():
    t = os.path.join(REF, "autogrid_original_4_2_1_ref", "autogrid", "Tests")
    dst = os.path.join(HERE, "x1hpv")
    os.makedirs(dst, exist_ok=True)
    with open(os.path.join(dst, "x1hpv.pdbqt.xz"), "wb") as f:
        f.write(lzma.compress(open(os.path.join(t, "x1hpv.pdbqt"), "rb").read(), preset=9))
    gpfs = {c: open(os.path.join(t, f"x1hpv_CASE{c}.gpf")).read() for c in range(4)}
    tmp = tempfile.mkdtemp()
    try:
        shutil.copy(os.path.join(t, "x1hpv.pdbqt"), tmp)
        open(os.path.join(tmp, "x1hpv.gpf"), "w").write(gpfs[0])
        r = subprocess.run([FG4, "-p", "x1hpv.gpf", "-l", "ref.glg"], cwd=tmp, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        maps, e, d = gpf_maps(gpfs[0])
        out = {"gpf": gpfs[0], "v4": False, "files_dir": "x1hpv", "files": ["x1hpv.pdbqt.xz"], "maps": {},
               "negative": {f"x1hpv_CASE{c}.gpf": gpfs[c] for c in (1, 2, 3)},
               "source": "AG421/Tests/x1hpv_CASE0.gpf run by oracle/_ref/fastgrid4 (FastGrid CPU build)"}
        for m in maps + [e, d]:
            out["maps"][m] = map_record(read_map(os.path.join(tmp, m)))
        json.dump(out, open(os.path.join(HERE, "x1hpv.json"), "w"))
    finally:
        shutil.rmtree(tmp)


# Synthetic cases: generator parameters + GPF edits; golden = FastGrid CPU.
SYNTH = {
    "synth_c0": dict(gen=dict(n_atoms=2000, semi_axes=(20, 20, 20), npts=60, seed=1, origin=(12.5, -3.25, 7.0)),
                     edits={}, v4=False),
    "synth_const_diel": dict(gen=dict(n_atoms=500, semi_axes=(12, 10, 9), npts=24, seed=7,
                                      ligand_types="A C HD N NA OA SA S F Cl", dielectric=40.0),
                             edits={}, v4=False),
    "synth_covalent": dict(gen=dict(n_atoms=400, semi_axes=(10, 10, 10), npts=20, seed=11,
                                    ligand_types="C HD OA Z"),
                           edits={"smooth 0.5": "smooth 0", "dielectric": None,
                                  "+": ["covalentmap 1.7 1000.0 3.1 -2.2 1.5", "qasp 0.01097",
                                        "fmap synth_covalent.fg.map"]},
                           v4=False),
    "synth_paramfile_v4": dict(gen=dict(n_atoms=600, semi_axes=(11, 11, 11), npts=22, seed=5,
                                        ligand_types="A C HD N NA OA SA"),
                               edits={"+front": ["parameter_file AD4.1_bound.dat"],
                                      "+after_receptor": ["receptor_types A C HD N OA SA"]},
                               v4=True),
    "synth_disorder_h": dict(gen=dict(n_atoms=700, semi_axes=(12, 11, 10), npts=24, seed=13,
                                      ligand_types="A C HD N NA OA SA"),
                             edits={"+": ["disorder_h"]}, v4=False),
}


def synth(name, spec):
    tmp = tempfile.mkdtemp()
    try:
        gpf_path = fg.synth_write(tmp, name, **spec["gen"])
        lines = open(gpf_path).read().splitlines()
        ed = spec["edits"]
        out = []
        for l in lines:
            rep = None
            for k, v in ed.items():
                if k.startswith("+"):
                    continue
                if l.startswith(k):
                    rep = (k, v)
            if rep is None:
                out.append(l)
            elif rep[1] is not None:
                out.append(rep[1])
            else:
                out.append(l)
            if l.startswith("receptor ") and "+after_receptor" in ed:
                out += ed["+after_receptor"]
        if "+front" in ed:
            out = ed["+front"] + out
        if "+" in ed:
            out += ed["+"]
        gpf = "\n".join(out) + "\n"
        open(gpf_path, "w").write(gpf)
        if "+front" in ed:
            shutil.copy(os.path.join(REF, "autogrid_original_4_2_1_ref", "autogrid", "Tests", "AD4.1_bound.dat"), tmp)
        args = [FG4, "-p", name + ".gpf", "-l", "ref.glg"] + (["--v4"] if spec["v4"] else [])
        r = subprocess.run(args, cwd=tmp, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        maps, e, d = gpf_maps(gpf)
        rec = {"gen": spec["gen"], "gpf": gpf, "v4": spec["v4"], "maps": {},
               "files": ["AD4.1_bound.dat"] if "+front" in ed else [],
               "source": "oracle/_ref/fastgrid4 (FastGrid CPU build) on the seeded synthetic receptor"}
        for m in maps + [e, d]:
            rec["maps"][m] = map_record(read_map(os.path.join(tmp, m)))
        fm = re.findall(r"^fmap\s+(\S+)", gpf, re.M)
        if fm:
            rec["floating_grid"] = map_record(read_map(os.path.join(tmp, fm[0])))
        rec["fld"] = open(os.path.join(tmp, name + ".maps.fld")).read()
        rec["xyz"] = open(os.path.join(tmp, name + ".maps.xyz")).read()
        json.dump(rec, open(os.path.join(HERE, name + ".json"), "w"))
    finally:
        shutil.rmtree(tmp)


if __name__ == "__main__":
    colagen2()
    hsg1_sm()
    pgp1()
    x1hpv()
    for n, s in SYNTH.items():
        synth(n, s)
    print("fixtures written to", HERE)
