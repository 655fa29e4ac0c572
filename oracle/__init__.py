"""Oracle — TEST INFRASTRUCTURE ONLY.

ctypes wrapper of oracle/oracle.c, the FP64 C restatement of FastGrid's CPU
map calculation.  Imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the checker; the product library never
loads it.  Built by ``make -C oracle oracle`` (or ``build()`` below).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            build()
        from fastgrid_b200 import Grid, Receptor, AffinityParams  # struct layouts only
        L = C.CDLL(SO)
        dp, i64p = C.POINTER(C.c_double), C.POINTER(C.c_int64)
        L.oracle_emap.argtypes = [C.POINTER(Grid), C.c_int, dp, dp, C.c_int, dp]
        L.oracle_emap_points.argtypes = [C.POINTER(Grid), C.c_int, dp, dp, C.c_int, C.c_int, i64p, dp]
        L.oracle_affinity.argtypes = [C.POINTER(Grid), C.POINTER(Receptor), C.POINTER(AffinityParams), dp, dp]
        L.oracle_affinity_points.argtypes = [C.POINTER(Grid), C.POINTER(Receptor), C.POINTER(AffinityParams),
                                             C.c_int, i64p, dp, dp]
        L.oracle_ddd_table.argtypes = [dp]
        L.oracle_sol_table.argtypes = [C.c_double, dp]
        L.oracle_pair_table.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, dp]
        L.oracle_round.argtypes = [C.c_double]
        L.oracle_round.restype = C.c_double
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def emap(grid, xyzw, inv_eps):
    xyzw = np.ascontiguousarray(xyzw, dtype=np.float64)
    out = np.empty(grid.nx * grid.ny * grid.nz)
    eps = np.zeros(8192) if inv_eps is None else np.ascontiguousarray(inv_eps, dtype=np.float64)
    lib().oracle_emap(C.byref(grid), xyzw.shape[0], _dp(xyzw), _dp(eps), 0 if inv_eps is None else 1, _dp(out))
    return out


def emap_points(grid, xyzw, inv_eps, idx):
    xyzw = np.ascontiguousarray(xyzw, dtype=np.float64)
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.empty(idx.shape[0])
    eps = np.zeros(8192) if inv_eps is None else np.ascontiguousarray(inv_eps, dtype=np.float64)
    lib().oracle_emap_points(C.byref(grid), xyzw.shape[0], _dp(xyzw), _dp(eps), 0 if inv_eps is None else 1,
                             idx.shape[0], idx.ctypes.data_as(C.POINTER(C.c_int64)), _dp(out))
    return out


def affinity(grid, receptor, params):
    n = grid.nx * grid.ny * grid.nz
    maps = np.zeros((max(params.n_maps, 1), n))
    dmap = np.zeros(n)
    lib().oracle_affinity(C.byref(grid), C.byref(receptor), C.byref(params), _dp(maps), _dp(dmap))
    return maps[:params.n_maps], dmap


def affinity_points(grid, receptor, params, idx):
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    maps = np.zeros((max(params.n_maps, 1), idx.shape[0]))
    dmap = np.zeros(idx.shape[0])
    lib().oracle_affinity_points(C.byref(grid), C.byref(receptor), C.byref(params), idx.shape[0],
                                 idx.ctypes.data_as(C.POINTER(C.c_int64)), _dp(maps), _dp(dmap))
    return maps[:params.n_maps], dmap


def round3(a):
    """roundOutput (autogrid.h:255-258), vectorised."""
    a = np.asarray(a, dtype=np.float64)
    return np.where(np.abs(a) < 0.0005, 0.0, np.floor(a * 1000 + 0.5) * 0.001)


def read_map(path):
    """Values of an AutoGrid .map file (6 header lines, one value per line)."""
    with open(path, "rb") as f:
        b = f.read().replace(b"\r", b"")
    pos = 0
    for _ in range(6):
        pos = b.index(b"\n", pos) + 1
    return np.fromstring(b[pos:].decode(), dtype=np.float64, sep="\n")
