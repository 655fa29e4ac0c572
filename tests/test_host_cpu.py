"""CPU tests of the host side: the C ABI library loads and exports every
function include/fastgrid_b200.h declares, the command line's exit codes
follow the reference (ProgramParameters.cpp:103-107, ExitProgram(911)), the
synthetic receptor generators keep their promises, and the benchmark's
max-over-ranks timing works across two gloo ranks."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO

import fastgrid_b200 as fg

HEADER = os.path.join(REPO, "include", "fastgrid_b200.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ag_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_function():
    names = header_functions()
    assert len(names) > 40
    lib = fg.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(fg.EXPORTS) == names


def test_cli_exit_codes(tmp_path):
    exe = fg.CLI_PATH
    r = subprocess.run([exe, "--no-such-switch"], capture_output=True, text=True)
    assert r.returncode == 1 and "unknown switch" in r.stderr
    r = subprocess.run([exe, "-p", str(tmp_path / "missing.gpf"), "-l", str(tmp_path / "x.glg")],
                       capture_output=True, text=True)
    assert r.returncode == 911 % 256  # ExitProgram(911), as the shell sees it
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--gpf" in r.stdout + r.stderr


def _read_pdbqt(path):
    xyz, q, t = [], [], []
    for line in open(path):
        if line.startswith("ATOM"):
            xyz.append([float(line[30:38]), float(line[38:46]), float(line[46:54])])
            q.append(float(line[70:76]))
            t.append(line[77:].strip())
    return np.array(xyz), np.array(q), t


def _min_dist(x):
    from scipy.spatial import cKDTree
    d, _ = cKDTree(x).query(x, k=2)
    return d[:, 1].min()


def test_synth_write_properties(tmp_path):
    fg.synth_write(str(tmp_path), "s", n_atoms=1500, semi_axes=(18, 16, 14), npts=40, seed=9, net_charge=2.0)
    x, q, t = _read_pdbqt(tmp_path / "s.pdbqt")
    assert len(x) == 1500
    assert _min_dist(x) >= 1.2 - 2e-3
    assert round(q.sum() * 1000) == 2000
    assert set(t) <= {"C", "OA", "N", "HD", "A", "SA"}
    # every HD sits next to an N/OA/SA within 20 atoms in file order (bond vectors need it)
    for i, ti in enumerate(t):
        if ti == "HD":
            lo, hi = max(0, i - 20), min(len(t), i + 21)
            d = np.linalg.norm(x[lo:hi] - x[i], axis=1)
            assert np.any((d < 1.378) & (d > 0))
    gpf = open(tmp_path / "s.gpf").read()
    assert "npts 40 40 40" in gpf and "gridcenter auto" in gpf and "elecmap" in gpf


def test_surrogate_receptor_generator():
    x = fg.surrogate_receptor(123, 3000)
    assert x.shape == (3000, 4)
    assert abs(x[:, 3].sum()) < 1e-9                       # net charge 0
    assert np.abs(x[:, :3].mean(axis=0)).max() < 1e-9      # centred on the centroid
    assert _min_dist(x[:, :3]) >= 1.2 - 2e-3
    r = 20.0 * (3000 / 2000.0) ** (1 / 3)
    ext = x[:, :3].max(axis=0) - x[:, :3].min(axis=0)
    assert np.all(ext <= 2 * r + 0.01)                     # inside a globule of radius r
    np.testing.assert_array_equal(x, fg.surrogate_receptor(123, 3000))  # seeded


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, REPO)
    import bench
    out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_bench_max_over_ranks_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert dict(out) == {0: 15.0, 1: 15.0}


def test_bench_reference_arm_prints_only_on_rank0(capsys):
    sys.path.insert(0, REPO)
    import bench

    class A:
        steps, warmup, gpus = 1, 3, 2
    assert bench.run_reference(A(), rank=1) is None
    assert capsys.readouterr().out == ""


def test_noalloc_rejects_misaligned_pointers_before_any_cuda_call():
    # ag_emap_noalloc reads atoms by 16-byte bulk copies and the dielectric
    # table as float4; a misaligned pointer is refused by the argument checks,
    # which run before the first CUDA call (so this runs without a GPU, and
    # the fake addresses are never dereferenced).
    import ctypes as C
    g = fg.Grid(9, 9, 9, 0.375)
    L = fg.lib()
    rc = L.ag_emap_noalloc(C.byref(g), 10, C.c_void_p(0x10008), C.c_void_p(0x20000), C.c_void_p(0x30000), None)
    assert rc == -1 and b"16-byte aligned" in L.ag_last_error()
    rc = L.ag_emap_noalloc(C.byref(g), 10, C.c_void_p(0x10000), C.c_void_p(0x20004), C.c_void_p(0x30000), None)
    assert rc == -1 and b"16-byte aligned" in L.ag_last_error()
    rc = L.ag_emap_noalloc(C.byref(g), 10, C.c_void_p(0x10000), C.c_void_p(0x20000), C.c_void_p(0x30002), None)
    assert rc == -1 and b"4-byte aligned" in L.ag_last_error()
    big = fg.Grid(1025, 1025, 1025, 0.375)
    rc = L.ag_emap_noalloc(C.byref(big), 10, C.c_void_p(0x10000), None, C.c_void_p(0x30000), None)
    assert rc == -1 and b"too large" in L.ag_last_error()


@pytest.mark.parametrize("seed,kw", [
    (1, dict(n_atoms=2000, semi_axes=(20, 20, 20), npts=60)),
    (2, dict(n_atoms=20000, semi_axes=(45, 35, 30), npts=160, ligand_types="A C HD N NA OA SA S F Cl")),
    (7000, dict(n_atoms=1800, semi_axes=(17, 17, 17), npts=44, ligand_types="A C HD N OA SA")),
])
def test_python_generator_writes_the_same_files(tmp_path, seed, kw):
    """oracle/synth.py (used by bench.py's reference arm, which must not load
    the engine's library) writes byte-identical PDBQT and GPF files."""
    from oracle import synth
    fg.synth_write(str(tmp_path / "lib"), "s", seed=seed, **kw)
    synth.write(str(tmp_path / "py"), "s", seed=seed, **kw)
    for ext in (".pdbqt", ".gpf"):
        assert open(tmp_path / "lib" / ("s" + ext), "rb").read() == open(tmp_path / "py" / ("s" + ext), "rb").read()


def test_reference_arm_slabs_cover_the_grid_once():
    sys.path.insert(0, REPO)
    import bench
    for k in (1, 2, 3, 5, 20, 25, 161):
        h = bench.slab_plan(k)
        assert len(h) == k and all(x % 2 == 1 for x in h)
        assert 161 <= sum(h) <= 162
    assert "fastgrid_b200" not in open(os.path.join(REPO, "oracle", "synth.py")).read().split('"""')[2]


@pytest.mark.parametrize("gpf,message", [("x1hpv_CASE1.gpf", "Not enough map keywords found"),
                                         ("x1hpv_CASE2.gpf", "No electrostatic map file defined"),
                                         ("x1hpv_CASE3.gpf", "No desolvation map file defined")])
def test_cli_rejects_gpf_missing_a_map_line(tmp_path, gpf, message):
    """AutoGrid 4.2.1's negative GPF tests (Tests/test_autogrid4.py:299-311):
    a GPF with one map / elecmap / dsolvmap line missing must not complete.
    The loader stops before any GPU work, like FastGrid's CPU build (exit
    code -2, as the shell sees it 254)."""
    from conftest import materialize
    work, _, case = materialize("x1hpv", str(tmp_path))
    open(os.path.join(work, gpf), "w").write(case["negative"][gpf])
    r = subprocess.run([fg.CLI_PATH, "-p", gpf, "-l", "neg.glg"], cwd=work, capture_output=True, text=True)
    assert r.returncode == 254, r.stderr
    assert message in r.stderr
    assert "Successful Completion" not in open(os.path.join(work, "neg.glg")).read()


def test_cli_timeout_ends_a_stalled_job(tmp_path):
    """--timeout N (ProgramParameters.cpp:199-220): the job runs in a child
    process; if it has not finished after N seconds the parent kills it,
    prints "Timeout! Process terminated." and exits 0.  The job stalls on the
    host: its receptor file is a FIFO that nobody writes, so it never reaches
    the GPU."""
    fifo = tmp_path / "stall.pdbqt"
    os.mkfifo(fifo)
    (tmp_path / "stall.gpf").write_text("npts 4 4 4\ngridfld stall.maps.fld\nspacing 0.375\n"
                                        "receptor_types A C\nligand_types C\nreceptor stall.pdbqt\n"
                                        "gridcenter 0 0 0\nmap stall.C.map\nelecmap stall.e.map\n"
                                        "dsolvmap stall.d.map\ndielectric -0.1465\n")
    t0 = __import__("time").perf_counter()
    r = subprocess.run([fg.CLI_PATH, "--timeout", "1", "-p", "stall.gpf", "-l", "stall.glg"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=60)
    dt = __import__("time").perf_counter() - t0
    assert r.returncode == 0
    assert "Timeout! Process terminated." in r.stderr
    assert 0.9 <= dt < 20


def test_shipped_surrogate_weights_match_their_training_report():
    """fastgrid_b200/surrogate_weights.bin was written by the training run whose
    report (command, seed, loss per epoch, timings, GPU) is
    fastgrid_b200/surrogate_weights.json; the report's SHA-256 pins the file."""
    import hashlib
    import json
    rep = json.load(open(os.path.join(REPO, "fastgrid_b200", "surrogate_weights.json")))
    data = open(fg.DEFAULT_WEIGHTS, "rb").read()
    assert hashlib.sha256(data).hexdigest() == rep["weights_sha256"]
    assert rep["receptors"] == 200 and rep["epochs"] == 10 and len(rep["loss_per_epoch"]) == 10
    assert rep["last_epoch_loss"] < 0.1 * rep["first_epoch_loss"]
    assert rep["command"].startswith("python -m fastgrid_b200.train_surrogate")


def test_packed_table_tail_reconstructs_the_fp32_table():
    """The e-map's packed copies of the table's saturating tail (capi.cu
    packTableTail, emap.cu mid_packed_atoms), restated: from bin b16 (b8) on
    every FP32 entry is bits(t[8191]) + k with k < 2^16 (2^8), all in
    t[8191]'s binade, and the kernel's one FMA  aws * (k as the subnormal
    k 2^-149) + awg,  awg = 100 w t[8191] 2^-16 and aws = awg * 2^(e+126) /
    t[8191], gives 100 w t[b] 2^-16 to within one FP32 rounding."""
    t = np.asarray(fg.ddd_table(), dtype=np.float64).astype(np.float32)
    u = t.view(np.uint32)
    G = int(u[-1])
    e = G >> 23

    def first(kmax):
        b = t.size
        while b > 0:
            x = int(u[b - 1])
            if (x >> 31) or (x >> 23) != e or x < G or x - G > kmax:
                break
            b -= 1
        return b

    b16, b8 = first(0xFFFF), first(0xFF)
    # About 22 A and 40 A; both parts fit the kernel's 16 KB region.
    assert 2200 <= b16 <= 2300 and 3950 <= b8 <= 4050
    assert ((2 * (8192 - b16) + 15) // 16 + (8192 - b8 + 15) // 16) * 16 <= 16384
    g = np.float32(t[-1])
    k_scale = np.float32(np.ldexp(1.0, e - 127 + 126) / float(g))
    assert np.isfinite(k_scale)
    bins = np.arange(b16, 8192)
    k = (u[bins].astype(np.int64) - G).astype(np.uint32)
    assert np.array_equal(u[bins], (G + k).astype(np.uint32))
    kf = k.view(np.float32).astype(np.float64)  # subnormals k 2^-149
    assert np.array_equal(kf, k.astype(np.float64) * 2.0 ** -149)
    for w in (0.001, -0.137, 0.5, 2.0, -1.9, 300.0):
        lw = np.float32(np.float64(w) * 100.0)
        awg = np.float32(lw * g * np.float32(2.0 ** -16))
        aws = np.float32(awg * k_scale)
        assert np.isfinite(aws)
        got = (np.float64(aws) * kf + np.float64(awg)).astype(np.float32).astype(np.float64)
        want = float(lw) * t[bins].astype(np.float64) * 2.0 ** -16
        assert np.abs(got / want - 1.0).max() <= 2.0 ** -23


def test_python_constants_match_the_header():
    """Every tuning knob and work flag the header defines is bound in Python
    with the same value (a knob added to one side only would pass silently)."""
    txt = open(HEADER).read()
    defs = dict(re.findall(r"#define\s+(AG_(?:TUNE|WORK|EMAP)_[A-Z0-9_]+)\s+(-?\d+)", txt))
    assert any(k.startswith("AG_TUNE_") for k in defs)
    for name, value in defs.items():
        assert hasattr(fg, name), name
        assert getattr(fg, name) == int(value), name


def test_bench_affinity_pair_count_is_exact():
    """bench.py's count of (grid point, atom) pairs within 8 A (the affinity
    pass's algorithmic work in the map set's FP32 roofline) equals a brute
    force count, atoms inside, on and outside the grid."""
    sys.path.insert(0, REPO)
    import bench

    rng = np.random.default_rng(12)
    nx, ny, nz, h = 23, 17, 20, 0.5
    xyz = np.concatenate([rng.uniform(-9, 9, (150, 3)), rng.uniform(-16, 16, (60, 3))])
    xyz[:5] = (np.array([[0, 0, 0], [2, -3, 1], [4, 4, 4], [-5, 0, 2], [1, 1, -1]]) * h)  # on grid points
    g = np.stack(np.meshgrid((np.arange(nx) - nx // 2) * h, (np.arange(ny) - ny // 2) * h,
                             (np.arange(nz) - nz // 2) * h, indexing="ij"), -1).reshape(-1, 3)
    brute = sum(int((((g - a) ** 2).sum(1) <= 64.0).sum()) for a in xyz)
    assert bench.affinity_pairs(xyz, nx, ny, nz, h) == brute
