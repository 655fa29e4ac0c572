#!/usr/bin/env python3
"""Benchmark: one AutoGrid map set (e-map + 10 affinity maps + d-map) for the
large synthetic configuration — 20,000 receptor atoms in a 45 x 35 x 30 A
ellipsoid, 161^3 grid at 0.375 A, ligand types A C HD N NA OA SA S F Cl — on
the B200 engine.

A step is one map set (the e-map and the affinity pass run concurrently, as
the library runs them; each pass is also timed alone for the rooflines).
`value` is point-atom evaluations per second over all ranks (N_atoms x
N_points per map set / map-set seconds), with the inputs resident in HBM; `e2e` is the same metric through the public C ABI with host
buffers (ag_problem_compute: upload, compute, all maps back in host memory).  L2 is flushed (256 MiB
write) between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

At N=1 the line also carries two supplementary measurements:
  "surrogate": the learned far-field e-map surrogate against the direct e-map
    on 20 held-out synthetic receptors (20,000 atoms, 161^3 grid, e-map only):
    device time of both, speed-up, and the surrogate's error against the
    direct sum over every point;
  "batch": 64 receptors of 1,000-30,000 atoms on odd grids of 41^3-161^3
    points with 6 ligand maps each, computed as one batch (persistent kernels
    replayed from one CUDA graph, autotuned e-map tiles);
  "config0": the small configuration (2,000 atoms, 61^3, 6 maps), with FastGrid's
    CPU build (all host threads) and AutoGrid 4.2.1 (one thread) timed on the same
    job in the cpu_baseline object, and the engine's fastgrid4 command line timed
    against AutoGrid 4.2.1's whole program on the same GPF;
  "e2e_cli": the engine's fastgrid4 command line on the large configuration's
    GPF (parse, tables, bond vectors, GPU map set, ASCII .map writing), wall
    time and per-phase times, next to FastGrid's CPU build on the same GPF;
  "cpu_baseline": FastGrid's CPU build on the whole large configuration (its
    own phase times and wall time), and, as the checker, the per-map error of
    the GPU maps against the FP64 oracle on sampled points.

--impl reference times FastGrid's own CPU path (oracle/_ref/fastgrid4, built
from the reference sources, all host threads) on the same workload and reports
the same metric: each step is one y-slab of the 161^3 grid (odd heights, all
161 z-planes and all 20,000 atoms), and the K timed steps together cover every
point of the grid once, so the timed work is the whole map set.  Its inputs are written by
oracle/synth.py, a pure-Python copy of the engine's generator (byte-identical
files), so the reference process never loads the engine's library.
Under torchrun (N > 1) every rank computes its own map set on its own GPU
(replicas; weak scaling); there is no inter-GPU exchange in this path.
"""
import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "map-set sec & point-atom evals/s, direct vs surrogate at stated error"
UNIT = "point-atom evals/s"
WORKLOAD = dict(n_atoms=20000, semi_axes=(45, 35, 30), npts=160, seed=2,
                ligand_types="A C HD N NA OA SA S F Cl")
REF_BIN = os.path.join(HERE, "oracle", "_ref", "fastgrid4")
AG421_BIN = os.path.join(HERE, "oracle", "_ref", "autogrid4")
C0 = dict(n_atoms=2000, semi_axes=(20, 20, 20), npts=60, seed=1)  # 61^3, ligands A C HD N OA SA
SURR_SEEDS = list(range(900001, 900021))   # held out: training uses seeds 1000003 * s + i
# DRAM bytes of one emap_kernel launch on this workload (ncu dram__bytes_read.sum +
# dram__bytes_write.sum of one captured launch).
EMAP_TRAFFIC_BYTES = 3.50e6
CHECK_POINTS = 3000  # sampled grid points of the per-map error against the FP64 oracle


def surrogate_section(fg, torch, ctx, stream, flush, np):
    """Direct vs surrogate e-map on the held-out receptors (device time, error).

    Returns the section and, per receptor, (atoms, sampled point indices,
    surrogate values, direct values) for the FP64-oracle check."""
    import ctypes as C
    g = fg.Grid(161, 161, 161, 0.375)
    npts = g.nx * g.ny * g.nz
    eps = fg.ddd_table()
    eps_ptr = eps.ctypes.data_as(C.POINTER(C.c_double))
    ctx.surrogate_load()
    ctx.surrogate_set()
    buf = np.empty(2 * npts, dtype=np.float32)
    d_ms, s_ms, e2e_ms = [], [], []
    max_err, sq, boxes, fallback, probe_max = 0.0, 0.0, 0, 0, 0.0
    samples = []
    rng = np.random.default_rng(11)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for i, seed in enumerate(SURR_SEEDS):
        x = fg.surrogate_receptor(seed, 20000)
        rec = fg.Receptor()
        rec.n_atoms = x.shape[0]
        rec.xyzw = x.ctypes.data_as(C.POINTER(C.c_double))
        ctx.upload(g, rec, None, eps_ptr)
        for _ in range(3 if i == 0 else 1):  # warm-up
            ctx.compute(fg.AG_WORK_EMAP)
            ctx.compute(fg.AG_WORK_EMAP_SURROGATE)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            flush.fill_(1)
            ev[0].record(stream)
            ctx.compute(fg.AG_WORK_EMAP)
            ev[1].record(stream)
        ctx.download(buf)
        direct = buf[:npts].astype(np.float64)
        with torch.cuda.stream(stream):
            flush.fill_(2)
            ev[2].record(stream)
            ctx.compute(fg.AG_WORK_EMAP_SURROGATE)
            ev[3].record(stream)
        ctx.download(buf)
        st = ctx.surrogate_stats()
        d_ms.append(ev[0].elapsed_time(ev[1]))
        s_ms.append(ev[2].elapsed_time(ev[3]))
        err = np.abs(buf[:npts].astype(np.float64) - direct)
        idx = np.unique(np.concatenate([rng.choice(npts, 200, replace=False), np.argsort(np.abs(direct))[-50:]]))
        samples.append((x, idx, buf[idx].astype(np.float64), direct[idx]))
        max_err = max(max_err, float(err.max()))
        sq += float((err * err).sum())
        boxes += st["boxes"]
        fallback += st["fallback_boxes"]
        probe_max = max(probe_max, st["probe_max_err"])
        if i < 5:  # through the host-buffer entry point (atoms in, map out)
            t0 = time.perf_counter()
            ctx.emap_surrogate(g, x, eps)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    n = len(SURR_SEEDS)
    dm, sm = sum(d_ms) / n, sum(s_ms) / n
    pairs = 20000 * npts
    return {"workload": f"{n} held-out synthetic receptors of 20000 atoms (globules at 0.06 atoms/A^3, charges "
                        "N(0,0.2) clipped at 0.7, net 0), 161^3 grid @0.375 A, e-map only",
            "direct_emap_ms": dm, "surrogate_emap_ms": sm, "speedup": dm / sm,
            "direct_pairs_per_s": pairs / (dm * 1e-3), "surrogate_equiv_pairs_per_s": pairs / (sm * 1e-3),
            "max_abs_err_vs_direct": max_err, "rms_err_vs_direct": (sq / (n * npts)) ** 0.5,
            "stated_error_bound": 0.01, "boxes": boxes, "fallback_boxes": fallback,
            "probe_max_err": probe_max, "e2e_ms_host_buffers": sum(e2e_ms) / len(e2e_ms),
            "method": "exact near field within 10 A + 1.5 A far-field grid, trilinear + 3-layer 32-channel "
                      "BF16 3D-conv corrector (shipped weights), residual probes with direct-sum fallback",
            "l2": "flushed before each timed map"}, samples


def config0_section(fg, torch, ctx, stream, tmp, steps):
    """The small configuration (2,000 atoms, 61^3, 6 maps) on the GPU: device map-set time and the
    whole-job call's wall time."""
    d = os.path.join(tmp, "c0")
    os.makedirs(d, exist_ok=True)
    fg.synth_write(d, "c0", **C0)
    old = os.getcwd()
    os.chdir(d)
    try:
        p = fg.Problem("c0.gpf", log="c0.glg")
    finally:
        os.chdir(old)
    pairs = p.info.n_atoms * p.npoints
    ctx.upload(p.grid, p.receptor, p.params, p.inv_eps_ptr)
    for _ in range(3):
        ctx.compute(fg.AG_WORK_ALL)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for _ in range(steps):
            ctx.compute(fg.AG_WORK_ALL)
        ev[1].record(stream)
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / steps
    p.compute(ctx)
    t0 = time.perf_counter()
    for _ in range(steps):
        p.compute(ctx)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / steps
    return {"workload": "synthetic receptor 2000 atoms (20 A globule), 61^3 grid @0.375 A, ligand types "
                        "A C HD N OA SA (6 maps + e + d)", "pairs": pairs, "map_set_ms": ms,
            "value": pairs / (ms * 1e-3), "unit": UNIT, "e2e_ms": e2e_ms}, d


def config0_cpu(d):
    """FastGrid's CPU build (all host threads) and AutoGrid 4.2.1 (one thread) on the small configuration,
    and the engine's fastgrid4 command line on the same GPF (whole programs, wall time)."""
    out = {}
    if os.path.exists(REF_BIN):
        t0 = time.perf_counter()
        secs, _, _ = fastgrid_cpu_run(d, os.path.join(d, "c0.gpf"))
        out.update(fastgrid_cpu_map_set_s=secs, fastgrid_cpu_wall_s=time.perf_counter() - t0,
                   fastgrid_cpu_threads=os.cpu_count())
    if os.path.exists(AG421_BIN):
        t0 = time.perf_counter()
        r = subprocess.run([AG421_BIN, "-p", "c0.gpf", "-l", "ag421.glg"], cwd=d, capture_output=True, text=True)
        if r.returncode == 0:
            out.update(autogrid421_wall_s=time.perf_counter() - t0, autogrid421_threads=1)
    cli = cli_run(d, "c0.gpf")
    out["engine_cli_wall_s"] = cli["wall_s"]
    if "autogrid421_wall_s" in out:
        out["cli_speedup_vs_autogrid421_wall"] = out["autogrid421_wall_s"] / cli["wall_s"]
    if "fastgrid_cpu_wall_s" in out:
        out["cli_speedup_vs_fastgrid_cpu_wall"] = out["fastgrid_cpu_wall_s"] / cli["wall_s"]
    return out


def cli_run(workdir, gpf):
    """The engine's fastgrid4 command line on `gpf` (a whole program: parse, tables, bond vectors, GPU
    map set, .map/.fld/.xyz writing): wall time and its --benchmark phase times."""
    import fastgrid_b200 as fg
    t0 = time.perf_counter()
    r = subprocess.run([fg.CLI_PATH, "-p", gpf, "-l", "cli.glg", "--benchmark"], cwd=workdir, capture_output=True,
                       text=True)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError("fastgrid4 (engine) failed: " + r.stderr[-500:])
    phases = {m.group(1).strip(): float(m.group(2)) for m in re.finditer(r"^(.+?)\s+Real: ([0-9.]+) ms", r.stderr, re.M)}
    return {"wall_s": wall, "phases_ms": phases}


def batch_section(fg, ctx, tmp, steps, np):
    """64 receptors of uneven size as one batch under a captured CUDA graph."""
    rng = np.random.default_rng(3)
    d = os.path.join(tmp, "batch")
    os.makedirs(d, exist_ok=True)
    probs, atoms, grids = [], [], []
    old = os.getcwd()
    try:
        for k in range(64):
            n = int(round(np.exp(rng.uniform(np.log(1000), np.log(30000)))))
            gsz = 2 * int(rng.integers(20, 81)) + 1
            r = 20.0 * (n / 2000.0) ** (1 / 3)
            fg.synth_write(d, f"j{k}", n_atoms=n, semi_axes=(r, r, r), npts=gsz - 1, seed=7000 + k,
                           ligand_types="A C HD N OA SA")
            os.chdir(d)
            probs.append(fg.Problem(f"j{k}.gpf", log=f"j{k}.glg"))
            os.chdir(old)
            atoms.append(n)
            grids.append(gsz)
    finally:
        os.chdir(old)
    b = fg.Batch(ctx, probs)
    t0 = time.perf_counter()
    b.autotune(None)
    tune_s = time.perf_counter() - t0
    for _ in range(3):
        b.compute()
    ms = []
    for _ in range(steps):
        b.compute()
        ms.append(b.last_ms)
    pairs = b.pairs
    b.close()
    m = sum(ms) / len(ms)
    return {"workload": "64 synthetic receptors, atoms log-uniform 1000-30000 (globules at 0.06 atoms/A^3), odd "
                        "grids uniform 41^3-161^3 @0.375 A, ligand types A C HD N OA SA (6 maps + e + d)",
            "atoms": [min(atoms), max(atoms)], "grid_points_per_axis": [min(grids), max(grids)],
            "pairs": pairs, "ms_per_batch": m, "value": pairs / (m * 1e-3), "unit": UNIT,
            "map_set_sec_mean": m * 1e-3 / 64, "autotune_s": tune_s,
            "launch": "one CUDA graph: per-job cell lists, one persistent e-map kernel and one persistent affinity "
                      "kernel over (job, CTA box) units, largest first"}


def config_dict(n_gpus, extra=None):
    d = {"workload": "synthetic receptor 20000 atoms (45x35x30 A ellipsoid), 161^3 grid @0.375 A, "
                     "10 ligand maps + e-map + d-map, distance-dependent dielectric",
         "n_atoms": WORKLOAD["n_atoms"], "grid": [161, 161, 161], "ligand_types": WORKLOAD["ligand_types"],
         "parallelism": f"replicas x{n_gpus}", "l2": "flushed between steps (256 MiB write)"}
    if extra:
        d.update(extra)
    return d


def make_workload(d):
    import fastgrid_b200 as fg
    return fg.synth_write(d, "bench", **WORKLOAD)


def slab_plan(steps, planes=161):
    """Heights of `steps` consecutive y-slabs of the grid that together cover its `planes` rows once:
    odd heights (a GPF's npts must be even), as equal as possible; when the parities do not add up
    the last slab reaches one plane past the top (its points are counted like the others)."""
    steps = max(1, steps)
    if steps >= planes:
        return [1] * steps
    base = planes // steps
    if base % 2 == 0:
        base -= 1
    h = [base] * steps
    k = 0
    while sum(h) < planes:
        h[k % steps] += 2
        k += 1
    return h


def slab_gpf(src, dst, y0, height, center):
    """Copy of the GPF `src` for rows y0 .. y0+height-1 of the 161^3 grid centred at `center` (all 161
    z-planes, so FastGrid's OpenMP loops, which run over z, keep every host thread busy)."""
    h = 0.375
    cy = center[1] + (y0 + (height - 1) / 2.0 - 80) * h
    txt = open(src).read()
    txt = re.sub(r"^npts .*$", f"npts 160 {height - 1} 160", txt, flags=re.M)
    txt = re.sub(r"^gridcenter .*$", f"gridcenter {center[0]:.6f} {cy:.6f} {center[2]:.6f}", txt, flags=re.M)
    open(dst, "w").write(txt)


def pdbqt_centroid(path):
    xyz = []
    for line in open(path):
        if line.startswith(("ATOM", "HETATM")):
            xyz.append((float(line[30:38]), float(line[38:46]), float(line[46:54])))
    n = len(xyz)
    return [sum(a[k] for a in xyz) / n for k in range(3)]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()
            self.f.close()

    def summary(self):
        if not self.p:
            return None
        rows = [l.split(",") for l in open(self.path).read().splitlines() if l.strip()]
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip() == "Active":
                    reasons.add(n)
        mx = [float(r[2]) for r in rows if len(r) > 2 and r[2].strip().replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def max_over_ranks(value, dist, device):
    """Max of a per-rank float over all ranks (the value itself without a process group)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def affinity_pairs(xyz, nx, ny, nz, h, cutoff=8.0):
    """Exact number of (grid point, atom) pairs within the affinity cutoff
    (r <= 8 A, CalculateGridmaps.cpp:238-316), the affinity pass's algorithmic
    work: per atom and per (z, y) lattice row, the x points inside the sphere
    and the grid, vectorised over atoms."""
    import numpy as np
    u = xyz / h + np.array([nx // 2, ny // 2, nz // 2], dtype=np.float64)
    rr = int(np.ceil(cutoff / h)) + 1
    base = np.floor(u).astype(np.int64)
    total = 0
    for dz in range(-rr, rr + 1):
        iz = base[:, 2] + dz
        zz = (iz - u[:, 2]) * h
        rem_z = cutoff * cutoff - zz * zz
        okz = (iz >= 0) & (iz < nz) & (rem_z >= 0)
        for dy in range(-rr, rr + 1):
            iy = base[:, 1] + dy
            yy = (iy - u[:, 1]) * h
            rem = rem_z - yy * yy
            ok = okz & (iy >= 0) & (iy < ny) & (rem >= 0)
            if not ok.any():
                continue
            half = np.sqrt(np.where(ok, rem, 0.0)) / h
            lo = np.maximum(np.ceil(u[:, 0] - half), 0)
            hi = np.minimum(np.floor(u[:, 0] + half), nx - 1)
            total += int(np.where(ok, np.maximum(hi - lo + 1, 0), 0).sum())
    return total


FG_PHASES = ("Cutoff grid", "KD-tree of hydrogens", "Atom & desolvation maps", "Electrostatic map")


def fastgrid_cpu_run(workdir, gpf):
    """Run FastGrid's CPU build on `gpf`; return (map-set seconds, all its --benchmark phases in ms, wall s).
    The map-set time is the sum of its e-map, cutoff-grid, kd-tree and affinity phases."""
    t0 = time.perf_counter()
    r = subprocess.run([REF_BIN, "-p", os.path.basename(gpf), "-l", "ref.glg", "--benchmark"], cwd=workdir,
                       capture_output=True, text=True)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError("fastgrid4 (reference CPU) failed: " + r.stderr[-500:])
    phases = {m.group(1).strip(): float(m.group(2)) for m in re.finditer(r"^(.+?)\s+Real: (\d+) ms", r.stderr, re.M)}
    return sum(phases.get(k, 0.0) for k in FG_PHASES) / 1e3, phases, wall


def cpu_baseline_leg(tmp, gpf_dir, prob, maps, surr_samples, np):
    """FastGrid's CPU build on the whole large configuration, and the checker: the per-map error of the
    GPU maps against the FP64 oracle on sampled points (and of the surrogate e-maps, if measured)."""
    import oracle
    secs, phases, wall = fastgrid_cpu_run(gpf_dir, os.path.join(gpf_dir, "bench.gpf"))
    pairs = WORKLOAD["n_atoms"] * 161 ** 3
    cpu = {"value": pairs / secs, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
           "sample": f"FastGrid CPU (oracle/_ref/fastgrid4, OpenMP, all host threads) on the whole workload, "
                     f"{pairs:.3g} pairs in {secs:.2f} s of its e-map + cutoff-grid + kd-tree + affinity phases",
           "map_set_s": secs, "wall_s": wall, "phases_ms": phases}
    # Checker: GPU maps against the FP64 oracle on sampled points.
    rng = np.random.default_rng(7)
    npts = prob.npoints
    nm = prob.n_maps
    e_gpu = maps[nm]
    idx = np.unique(np.concatenate([rng.choice(npts, CHECK_POINTS, replace=False),
                                    np.argsort(np.abs(e_gpu))[-200:]]))
    e_ref = oracle.emap_points(prob.grid, prob.xyzw(), prob.inv_eps(), idx)
    a_ref, d_ref = oracle.affinity_points(prob.grid, prob.receptor, prob.params, idx)
    names = WORKLOAD["ligand_types"].split() + ["e", "d"]
    per_map = {}
    for m in range(nm + 2):
        ref = a_ref[m] if m < nm else (e_ref if m == nm else d_ref)
        d = maps[m][idx].astype(np.float64) - ref
        per_map[names[m]] = {"max_abs": float(np.abs(d).max()), "rms": float(np.sqrt((d * d).mean())),
                             "max_rel": float((np.abs(d) / np.maximum(np.abs(ref), 1e-3)).max())}
    check = {"points": int(idx.size), "per_map": per_map,
             "tolerance": "e-map 1e-4 kcal/mol/e; affinity and d-map max(1e-3, 1e-4 |v|) kcal/mol"}
    if surr_samples:
        smax, ssq, dmax, n = 0.0, 0.0, 0.0, 0
        eps = oracle_ddd(np)
        g = prob.grid.__class__(161, 161, 161, 0.375)
        for x, sidx, sval, dval in surr_samples:
            ref = oracle.emap_points(g, x, eps, sidx)
            smax = max(smax, float(np.abs(sval - ref).max()))
            ssq += float(((sval - ref) ** 2).sum())
            dmax = max(dmax, float(np.abs(dval - ref).max()))
            n += sidx.size
        check["surrogate_vs_fp64_oracle"] = {"points": n, "max_abs": smax, "rms": (ssq / n) ** 0.5,
                                             "direct_max_abs": dmax}
    return cpu, check


def oracle_ddd(np):
    """332/eps table of the distance-dependent dielectric, as the oracle computes it."""
    import oracle
    import ctypes as C
    t = np.empty(8192)
    oracle.lib().oracle_ddd_table(t.ctypes.data_as(C.POINTER(C.c_double)))
    return t


def run_reference(args, rank):
    """FastGrid's CPU build on the whole large configuration, one y-slab per step (rank 0 only)."""
    if rank != 0:
        return
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/fastgrid4 was not built "
                          "(build() compiles it from the reference sources when they are present)"}))
        return
    from oracle import synth  # writes the inputs without loading the engine's library
    heights = slab_plan(args.steps)
    with tempfile.TemporaryDirectory() as tmp:
        src = synth.write(tmp, "bench", **WORKLOAD)
        center = pdbqt_centroid(os.path.join(tmp, "bench.pdbqt"))
        gpf = os.path.join(tmp, "slab.gpf")
        for _ in range(args.warmup):  # one row of x-z points through the middle
            slab_gpf(src, gpf, 80, 1, center)
            fastgrid_cpu_run(tmp, gpf)
        times, y0 = [], 0
        for hgt in heights:
            slab_gpf(src, gpf, y0 % 161, hgt, center)
            times.append(fastgrid_cpu_run(tmp, gpf)[0])
            y0 += hgt
    planes = sum(heights)
    pairs = WORKLOAD["n_atoms"] * 161 * 161 * planes
    secs = sum(times)
    value = pairs / secs
    cores = os.cpu_count()
    sample = (f"the whole 161^3 grid in {len(heights)} y-slabs of {min(heights)}-{max(heights)} rows, one per "
              f"step ({planes} rows, all 20000 atoms each step, {pairs:.3g} point-atom pairs); time = FastGrid's "
              "own e-map + cutoff-grid + kd-tree + affinity phase times; inputs written by oracle/synth.py")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "map_set_sec_whole_grid": secs}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-config0", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import numpy as np
    import torch
    import fastgrid_b200 as fg

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    tmp = tempfile.mkdtemp()
    try:
        gpf = make_workload(tmp)
        old = os.getcwd()
        os.chdir(tmp)
        prob = fg.Problem(os.path.basename(gpf), log="bench.glg")
        os.chdir(old)
        n_atoms, npts, nmaps = prob.info.n_atoms, prob.npoints, prob.n_maps
        pairs = n_atoms * npts

        rsqrt_ps, ffma_ps = fg.measure_peaks(local)
        ctx = fg.Context(local)
        stream = torch.cuda.ExternalStream(ctx.stream)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

        # ---- device-resident timing (value) ----
        ctx.upload(prob.grid, prob.receptor, prob.params, prob.inv_eps_ptr)
        for _ in range(args.warmup):
            ctx.compute(fg.AG_WORK_ALL)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        # One step = one map set: the e-map and the affinity pass in one call,
        # which runs them concurrently (the e-map's CTAs first, on a
        # high-priority stream; the affinity pass fills the SMs its last wave
        # leaves free).  Events on the context's stream, which waits for both.
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        launches0 = ctx.launches
        with ClockSampler(local) as clocks:
            for k in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(k & 0xFF)
                    starts[k].record(stream)
                    ctx.compute(fg.AG_WORK_ALL)
                    ends[k].record(stream)
            torch.cuda.synchronize()
        launches = ctx.launches - launches0
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
        tot_ms = max_over_ranks(sum(step_ms), dist, f"cuda:{local}")
        ms_step = tot_ms / args.steps
        value = world * pairs / (ms_step * 1e-3)

        # Each pass alone, K more steps (the e-map kernel's own duration is the
        # roofline's denominator; the affinity pass's is reported beside it).
        e_starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        e_ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        a_ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(k & 0xFF)
                e_starts[k].record(stream)
                ctx.compute(fg.AG_WORK_EMAP)
                e_ends[k].record(stream)
                ctx.compute(fg.AG_WORK_AFFINITY)
                a_ends[k].record(stream)
        torch.cuda.synchronize()
        emap_ms = [s.elapsed_time(e) for s, e in zip(e_starts, e_ends)]
        aff_ms = [s.elapsed_time(e) for s, e in zip(e_ends, a_ends)]
        emap_avg = sum(emap_ms) / len(emap_ms)
        aff_avg = sum(aff_ms) / len(aff_ms)

        # ---- end to end through the whole-job C ABI call (ag_problem_compute):
        # the parsed job's host arrays are uploaded, every map is computed and
        # the map set is copied back to host memory, each step ----
        h2d = n_atoms * (32 + 4 + 4 + 4 + 4 + 48) + 8192 * 4
        h2d += prob.info.n_types * 801 * nmaps * 4
        d2h = (nmaps + 2) * npts * 4
        for _ in range(2):
            prob.compute(ctx)
        if dist:
            dist.barrier()
        e2e_t = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            prob.compute(ctx)
            e2e_t.append(time.perf_counter() - t0)
        maps_all = prob.maps().reshape(nmaps + 2, npts)
        e2e_s = max_over_ranks(sum(e2e_t) / len(e2e_t), dist, f"cuda:{local}")
        e2e_value = world * pairs / e2e_s
        check = float(np.abs(maps_all[nmaps]).max())
        emap_pairs_per_s = pairs / (emap_avg * 1e-3)
        aff_pairs = affinity_pairs(prob.xyzw()[:, :3], prob.grid.nx, prob.grid.ny, prob.grid.nz, prob.grid.spacing)
        mapset_ops = 8 * pairs + (nmaps + 10) * aff_pairs
        ck = clocks.summary()

        # ---- supplementary measurements (N=1) ----
        surr = batch = None
        surr_samples = []
        if world == 1 and not args.no_surrogate:
            surr, surr_samples = surrogate_section(fg, torch, ctx, stream, flush, np)
        if world == 1 and not args.no_batch:
            batch = batch_section(fg, ctx, tmp, args.steps, np)
        c0 = c0dir = None
        if world == 1 and not args.no_config0:
            c0, c0dir = config0_section(fg, torch, ctx, stream, tmp, args.steps)

        # ---- CPU baseline and checker (rank 0, N=1 only), then the command line end to end ----
        cpu = check_maps = e2e_cli = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_BIN):
            cpu, check_maps = cpu_baseline_leg(tmp, tmp, prob, maps_all, surr_samples, np)
            for f in os.listdir(tmp):
                if f.endswith(".map"):
                    os.remove(os.path.join(tmp, f))
            if c0dir is not None:
                cpu["config0"] = config0_cpu(c0dir)
                if c0 is not None and "fastgrid_cpu_map_set_s" in cpu["config0"]:
                    c0["speedup_vs_fastgrid_cpu_map_set"] = (cpu["config0"]["fastgrid_cpu_map_set_s"] /
                                                             (c0["map_set_ms"] * 1e-3))
            if surr is not None and "surrogate_vs_fp64_oracle" in check_maps:
                surr["vs_fp64_oracle"] = check_maps.pop("surrogate_vs_fp64_oracle")
        if rank == 0 and world == 1:
            d = os.path.join(tmp, "cli")
            os.makedirs(d, exist_ok=True)
            for f in ("bench.gpf", "bench.pdbqt"):
                shutil.copy(os.path.join(tmp, f), os.path.join(d, f))
            e2e_cli = cli_run(d, "bench.gpf")
            e2e_cli["workload"] = "the large configuration's GPF through the engine's fastgrid4 command line"
            e2e_cli["value"] = pairs / e2e_cli["wall_s"]
            e2e_cli["unit"] = UNIT
            host = {k: v for k, v in e2e_cli["phases_ms"].items() if k not in ("Total", "Grid maps (GPU)")}
            if host:
                e2e_cli["largest_host_phase"] = max(host, key=host.get)
            if cpu is not None:
                e2e_cli["fastgrid_cpu_wall_s"] = cpu["wall_s"]
                e2e_cli["speedup_vs_fastgrid_cpu_wall"] = cpu["wall_s"] / e2e_cli["wall_s"]
            shutil.rmtree(d, ignore_errors=True)

        if rank == 0:
            line = {
                "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 (FP64 tile sums and exact FP64 bins near edges)",
                "data": "synthetic", "config": config_dict(world),
                "map_set_sec": ms_step * 1e-3, "emap_ms": emap_avg, "affinity_ms": aff_avg,
                "passes": "concurrent: the e-map on a high-priority stream, the affinity pass filling the SMs "
                          "its last wave leaves free; emap_ms and affinity_ms time each pass alone in K more "
                          "steps (their sum is the map set run one pass after the other)",
                "roofline": {"bound": "sfu", "kernel": "emap_kernel",
                             "achieved": emap_pairs_per_s / 1e9, "peak": rsqrt_ps / 1e9, "unit": "Gpair/s",
                             "frac": emap_pairs_per_s / rsqrt_ps, "traffic": EMAP_TRAFFIC_BYTES,
                             "traffic_unit": "DRAM bytes per launch (ncu capture of this workload)",
                             "note": "one SFU rsqrt per point-atom pair; peak = rsqrt/s measured by "
                                     "ag_measure_peaks in this run (MEASURED_PEAKS.json has no SFU figure)"},
                "roofline_fp32": {"achieved_ops": 8 * emap_pairs_per_s / 1e12, "peak": ffma_ps / 1e12,
                                  "unit": "Tinstr/s", "frac": 8 * emap_pairs_per_s / ffma_ps,
                                  "note": "8 algorithmic FP32-pipe ops per pair vs measured FFMA issue rate"},
                "roofline_mapset_fp32": {
                    "emap_pairs": pairs, "affinity_pairs": aff_pairs, "ops": mapset_ops,
                    "achieved_ops": mapset_ops / (ms_step * 1e-3) / 1e12, "peak": ffma_ps / 1e12,
                    "unit": "Tinstr/s", "frac": mapset_ops / (ms_step * 1e-3) / ffma_ps,
                    "note": "the whole map set (e-map + affinity maps + d-map) per map-set time: 8 FP32 ops per "
                            "e-map pair, n_maps + 10 per in-cutoff affinity pair (geometry, bin, one add per map, "
                            "two desolvation FMAs; H-bond angular terms not counted), vs the measured FFMA rate"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": e2e_s * 1e3},
                "gpu_launches": launches, "clocks": ck, "cpu_baseline": cpu, "e2e_cli": e2e_cli,
                "check_vs_fp64_oracle": check_maps,
                "emap_abs_max": check, "surrogate": surr, "batch": batch, "config0": c0,
            }
            print(json.dumps(line))
        ctx.close()
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
