"""fastgrid_b200 — B200 AutoGrid grid-map engine (Python bindings).

The engine itself is native: CUDA kernels for sm_100a plus C++ host code in
``_lib/libfastgrid_b200.so``, reached through the C ABI declared in
``include/fastgrid_b200.h``.  This module only binds that ABI with ctypes and
moves numpy arrays across it.  There is no Python or CPU implementation of the
map calculation here: if the library is missing, importing the engine raises.

Mirrors the reference's seams (fastgrid_master/fastgrid/):
  * ``Context.emap``      <- calculateElectrostaticMapAsync / synchronizeCalculation
                             (electrostatics/Electrostatics.h:32-36)
  * ``Context.affinity``  <- calculateGridmaps (CalculateGridmaps.h:30-31)
  * ``Problem``           <- InputDataLoader::load + programMain (main.cpp:115-254)
  * ``main``              <- the fastgrid4 / autogrid4 command line
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfastgrid_b200.so")
CLI_PATH = os.path.join(HERE, "_lib", "fastgrid4")

AG_OK = 0
AG_WORK_EMAP, AG_WORK_AFFINITY, AG_WORK_ALL = 1, 2, 3
AG_EMAP_KAHAN, AG_EMAP_PLAIN = 0, 1
AG_TUNE_EMAP_RNEAR, AG_TUNE_EMAP_ANALYTIC_EVERY, AG_TUNE_EMAP_CTAS_PER_SM = 1, 2, 3
TABLE_LEN = 8192


class AgError(RuntimeError):
    pass


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("spacing", C.c_double)]


class Receptor(C.Structure):
    _fields_ = [("n_atoms", C.c_int), ("xyzw", C.POINTER(C.c_double)), ("charge", C.POINTER(C.c_double)),
                ("vol", C.POINTER(C.c_double)), ("solpar", C.POINTER(C.c_double)), ("type", C.POINTER(C.c_int)),
                ("hbond", C.POINTER(C.c_int)), ("disorder", C.POINTER(C.c_ubyte)), ("rexp", C.POINTER(C.c_int)),
                ("rvector", C.POINTER(C.c_double)), ("rvector2", C.POINTER(C.c_double))]


class AffinityParams(C.Structure):
    _fields_ = [("n_maps", C.c_int), ("n_types", C.c_int), ("energy", C.POINTER(C.c_double)),
                ("sol", C.POINTER(C.c_double)), ("map_hbond", C.POINTER(C.c_int)),
                ("map_is_hbonder", C.POINTER(C.c_int)), ("map_is_covalent", C.POINTER(C.c_int)),
                ("solpar_probe", C.POINTER(C.c_double)), ("vol_probe", C.POINTER(C.c_double)),
                ("solpar_q", C.c_double), ("hydrogen", C.c_int)]


class ProblemInfo(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("spacing", C.c_double),
                ("center", C.c_double * 3), ("n_atoms", C.c_int), ("n_maps", C.c_int), ("n_types", C.c_int),
                ("dist_dep_diel", C.c_int), ("has_floating_grid", C.c_int)]


class SynthParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_atoms", C.c_int), ("semi_axes", C.c_double * 3),
                ("origin", C.c_double * 3), ("frac_C", C.c_double), ("frac_OA", C.c_double),
                ("frac_N", C.c_double), ("frac_HD", C.c_double), ("frac_A", C.c_double), ("frac_SA", C.c_double),
                ("charge_sigma", C.c_double), ("charge_clip", C.c_double), ("net_charge", C.c_double),
                ("npts", C.c_int), ("spacing", C.c_double), ("ligand_types", C.c_char_p),
                ("dielectric", C.c_double)]


# Every symbol include/fastgrid_b200.h declares.
EXPORTS = ["ag_ctx_create", "ag_ctx_destroy", "ag_last_error", "ag_ctx_stream", "ag_ctx_launch_count",
           "ag_emap", "ag_emap_mode", "ag_affinity", "ag_upload", "ag_compute", "ag_device_maps", "ag_download",
           "ag_problem_load", "ag_problem_free", "ag_problem_info_get", "ag_problem_views", "ag_problem_compute",
           "ag_problem_maps", "ag_problem_write", "ag_main", "ag_synth_write", "ag_measure_peaks",
           "ag_emap_noalloc", "ag_ctx_tune", "ag_batch_create", "ag_batch_autotune",
           "ag_batch_compute", "ag_batch_download", "ag_batch_pairs", "ag_batch_free"]

_lib = None


def lib():
    """Load libfastgrid_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AgError("libfastgrid_b200.so is not built (run `python -m fastgrid_b200.build`); "
                      "the engine has no CPU fallback")
    L = C.CDLL(LIB_PATH)
    vp, i64 = C.c_void_p, C.c_int64
    dp, fp = C.POINTER(C.c_double), C.POINTER(C.c_float)
    L.ag_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.ag_ctx_destroy.argtypes = [vp]
    L.ag_last_error.restype = C.c_char_p
    L.ag_ctx_stream.argtypes = [vp]
    L.ag_ctx_stream.restype = vp
    L.ag_ctx_launch_count.argtypes = [vp]
    L.ag_ctx_launch_count.restype = i64
    L.ag_emap.argtypes = [vp, C.POINTER(Grid), C.c_int, dp, dp, fp]
    L.ag_emap_mode.argtypes = [vp, C.POINTER(Grid), C.c_int, dp, dp, C.c_int, fp]
    L.ag_affinity.argtypes = [vp, C.POINTER(Grid), C.POINTER(Receptor), C.POINTER(AffinityParams), fp, fp]
    L.ag_upload.argtypes = [vp, C.POINTER(Grid), C.POINTER(Receptor), C.POINTER(AffinityParams), dp]
    L.ag_compute.argtypes = [vp, C.c_int]
    L.ag_device_maps.argtypes = [vp]
    L.ag_device_maps.restype = vp
    L.ag_download.argtypes = [vp, fp]
    L.ag_problem_load.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.POINTER(vp)]
    L.ag_problem_free.argtypes = [vp]
    L.ag_problem_free.restype = None
    L.ag_problem_info_get.argtypes = [vp, C.POINTER(ProblemInfo)]
    L.ag_problem_views.argtypes = [vp, C.POINTER(Grid), C.POINTER(Receptor), C.POINTER(AffinityParams),
                                   C.POINTER(dp)]
    L.ag_problem_compute.argtypes = [vp, vp]
    L.ag_problem_maps.argtypes = [vp]
    L.ag_problem_maps.restype = fp
    L.ag_problem_write.argtypes = [vp]
    L.ag_main.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
    L.ag_synth_write.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(SynthParams)]
    L.ag_measure_peaks.argtypes = [C.c_int, dp, dp]
    L.ag_emap_noalloc.argtypes = [C.POINTER(Grid), C.c_int, vp, vp, vp, vp]
    L.ag_ctx_tune.argtypes = [vp, C.c_int, C.c_double]
    L.ag_batch_create.argtypes = [vp, C.POINTER(vp), C.c_int, C.POINTER(vp)]
    L.ag_batch_autotune.argtypes = [vp, C.c_char_p]
    L.ag_batch_compute.argtypes = [vp]
    L.ag_batch_download.argtypes = [vp, C.c_int, fp]
    L.ag_batch_pairs.argtypes = [vp]
    L.ag_batch_pairs.restype = C.c_double
    L.ag_batch_free.argtypes = [vp]
    _lib = L
    return L


def _check(rc):
    if rc != AG_OK:
        raise AgError(lib().ag_last_error().decode(errors="replace") + f" (code {rc})")


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Context:
    """One GPU context (stream + device buffers).  Not thread-safe."""

    def __init__(self, device=0):
        h = C.c_void_p()
        _check(lib().ag_ctx_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().ag_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return lib().ag_ctx_stream(self.h)

    def tune(self, knob, value):
        _check(lib().ag_ctx_tune(self.h, knob, float(value)))

    @property
    def launches(self):
        return lib().ag_ctx_launch_count(self.h)

    def emap(self, grid, xyzw, inv_eps=None, mode=AG_EMAP_KAHAN):
        """E-map of atoms `xyzw` (n x 4, grid-centred, weights premultiplied)."""
        xyzw = np.ascontiguousarray(xyzw, dtype=np.float64)
        n = xyzw.shape[0]
        out = np.empty(grid.nx * grid.ny * grid.nz, dtype=np.float32)
        eps = None if inv_eps is None else np.ascontiguousarray(inv_eps, dtype=np.float64)
        _check(lib().ag_emap_mode(self.h, C.byref(grid), n, _dp(xyzw), None if eps is None else _dp(eps), mode,
                                  _fp(out)))
        return out

    def affinity(self, grid, receptor, params, n_maps):
        npts = grid.nx * grid.ny * grid.nz
        maps = np.empty((max(n_maps, 1), npts), dtype=np.float32)
        dmap = np.empty(npts, dtype=np.float32)
        _check(lib().ag_affinity(self.h, C.byref(grid), C.byref(receptor), C.byref(params), _fp(maps), _fp(dmap)))
        return maps[:n_maps], dmap

    def upload(self, grid, receptor, params, inv_eps_ptr):
        _check(lib().ag_upload(self.h, C.byref(grid), C.byref(receptor),
                               C.byref(params) if params is not None else None, inv_eps_ptr))

    def compute(self, work=AG_WORK_ALL):
        _check(lib().ag_compute(self.h, work))

    def download(self, out):
        _check(lib().ag_download(self.h, _fp(out)))

    def device_maps(self):
        return lib().ag_device_maps(self.h)


class Problem:
    """A parsed GPF job (receptor, tables, bond vectors) and its map set."""

    def __init__(self, gpf, v4=False, log=None):
        h = C.c_void_p()
        _check(lib().ag_problem_load(gpf.encode(), 1 if v4 else 0, (log or "").encode() if log else None,
                                     C.byref(h)))
        self.h = h
        info = ProblemInfo()
        _check(lib().ag_problem_info_get(h, C.byref(info)))
        self.info = info
        self.grid, self.receptor, self.params = Grid(), Receptor(), AffinityParams()
        self.inv_eps_ptr = C.POINTER(C.c_double)()
        _check(lib().ag_problem_views(h, C.byref(self.grid), C.byref(self.receptor), C.byref(self.params),
                                      C.byref(self.inv_eps_ptr)))

    def __del__(self):
        try:
            if self.h:
                lib().ag_problem_free(self.h)
                self.h = None
        except Exception:
            pass

    @property
    def npoints(self):
        return self.grid.nx * self.grid.ny * self.grid.nz

    @property
    def n_maps(self):
        return self.info.n_maps

    def xyzw(self):
        return np.ctypeslib.as_array(self.receptor.xyzw, shape=(self.info.n_atoms, 4)).copy()

    def inv_eps(self):
        if not self.inv_eps_ptr:
            return None
        return np.ctypeslib.as_array(self.inv_eps_ptr, shape=(TABLE_LEN,)).copy()

    def compute(self, ctx):
        _check(lib().ag_problem_compute(ctx.h, self.h))

    def maps(self):
        """(n_maps + 2, nz, ny, nx) FP32: atom maps, then e-map, then d-map (unrounded)."""
        p = lib().ag_problem_maps(self.h)
        if not p:
            raise AgError("maps not computed")
        g = self.grid
        return np.ctypeslib.as_array(p, shape=(self.n_maps + 2, g.nz, g.ny, g.nx)).copy()

    def write(self):
        _check(lib().ag_problem_write(self.h))


def measure_peaks(device=0):
    """(SFU rsqrt/s, FP32 FMA instructions/s) measured on `device` now."""
    a, b = C.c_double(), C.c_double()
    _check(lib().ag_measure_peaks(device, C.byref(a), C.byref(b)))
    return a.value, b.value


class Batch:
    """Many map sets computed by persistent kernels replayed from one CUDA graph."""

    def __init__(self, ctx, problems):
        self.problems = list(problems)  # keep the problems alive
        arr = (C.c_void_p * len(self.problems))(*[p.h.value for p in self.problems])
        h = C.c_void_p()
        _check(lib().ag_batch_create(ctx.h, arr, len(self.problems), C.byref(h)))
        self.h = h

    def autotune(self, cache_path=None):
        _check(lib().ag_batch_autotune(self.h, cache_path.encode() if cache_path else None))

    def compute(self):
        _check(lib().ag_batch_compute(self.h))

    @property
    def pairs(self):
        return lib().ag_batch_pairs(self.h)

    def maps(self, i):
        p = self.problems[i]
        out = np.empty((p.n_maps + 2) * p.npoints, dtype=np.float32)
        _check(lib().ag_batch_download(self.h, i, _fp(out)))
        return out.reshape(p.n_maps + 2, p.grid.nz, p.grid.ny, p.grid.nx)

    def close(self):
        if self.h:
            lib().ag_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def main(argv):
    """Run the fastgrid4 command line in-process; returns the exit code."""
    arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
    return lib().ag_main(len(argv), arr)


SYNTH_DEFAULTS = dict(frac=(0.45, 0.18, 0.15, 0.15, 0.05, 0.02), charge_sigma=0.2, charge_clip=0.7,
                      net_charge=0.0, spacing=0.375, dielectric=-0.1465)


def synth_write(dirname, stem, n_atoms, semi_axes, npts, ligand_types="A C HD N OA SA", seed=0,
                origin=(0.0, 0.0, 0.0), frac=SYNTH_DEFAULTS["frac"], charge_sigma=0.2, charge_clip=0.7,
                net_charge=0.0, spacing=0.375, dielectric=-0.1465):
    """Write <dir>/<stem>.pdbqt and <stem>.gpf for a seeded synthetic receptor."""
    sp = SynthParams()
    sp.seed = seed
    sp.n_atoms = n_atoms
    for k in range(3):
        sp.semi_axes[k] = semi_axes[k]
        sp.origin[k] = origin[k]
    sp.frac_C, sp.frac_OA, sp.frac_N, sp.frac_HD, sp.frac_A, sp.frac_SA = frac
    sp.charge_sigma, sp.charge_clip, sp.net_charge = charge_sigma, charge_clip, net_charge
    sp.npts, sp.spacing = npts, spacing
    lt = ligand_types.encode()
    sp.ligand_types = lt
    sp.dielectric = dielectric
    os.makedirs(dirname, exist_ok=True)
    _check(lib().ag_synth_write(dirname.encode(), stem.encode(), C.byref(sp)))
    return os.path.join(dirname, stem + ".gpf")
