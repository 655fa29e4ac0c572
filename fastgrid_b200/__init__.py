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
AG_WORK_EMAP_SURROGATE = 4
SURROGATE_WEIGHTS = 35424
DEFAULT_WEIGHTS = os.path.join(HERE, "surrogate_weights.bin")
AG_EMAP_KAHAN, AG_EMAP_PLAIN = 0, 1
AG_TUNE_EMAP_RNEAR, AG_TUNE_EMAP_PACKED_TABLE, AG_TUNE_EMAP_CTAS_PER_SM = 1, 2, 3
AG_TUNE_EMAP_WARP_COMPACT, AG_TUNE_EMAP_TILE, AG_TUNE_SURROGATE_TCGEN05 = 4, 5, 6
AG_TUNE_TEST_IDLE_WAIT, AG_TUNE_TEST_CHECKSUM_OFFSET, AG_TUNE_AFFINITY_KERNEL = 7, 8, 9
AG_TUNE_CONCURRENT_PASSES = 10
AG_E_INVALID, AG_E_CUDA, AG_E_DEVICE, AG_E_HOST, AG_E_NOMEM = -1, -2, -3, -4, -5
TABLE_LEN = 8192


class AgError(RuntimeError):
    """A failed engine call; `code` is the AG_E_* status it returned."""

    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


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


class SurrogateParams(C.Structure):
    _fields_ = [("r_near", C.c_double), ("coarse_spacing", C.c_double), ("probe_tol", C.c_double),
                ("probes_per_box", C.c_int), ("use_corrector", C.c_int)]


class SurrogateStats(C.Structure):
    _fields_ = [("boxes", C.c_int), ("fallback_boxes", C.c_int), ("probe_max_err", C.c_double)]


class SurrogateTrainParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_receptors", C.c_int), ("min_atoms", C.c_int), ("max_atoms", C.c_int),
                ("points", C.c_int), ("spacing", C.c_double), ("epochs", C.c_int), ("lr", C.c_double)]


class SurrogateTrainReport(C.Structure):
    _fields_ = [("gen_seconds", C.c_double), ("train_seconds", C.c_double), ("steps", C.c_int),
                ("first_epoch_loss", C.c_double), ("last_epoch_loss", C.c_double), ("s_in", C.c_double),
                ("s_out", C.c_double)]


# Every symbol include/fastgrid_b200.h declares.
EXPORTS = ["ag_ctx_create", "ag_ctx_destroy", "ag_last_error", "ag_ctx_stream", "ag_ctx_launch_count",
           "ag_emap", "ag_emap_mode", "ag_affinity", "ag_upload", "ag_compute", "ag_device_maps", "ag_download",
           "ag_problem_load", "ag_problem_free", "ag_problem_info_get", "ag_problem_views", "ag_problem_compute",
           "ag_problem_maps", "ag_problem_write", "ag_main", "ag_synth_write", "ag_measure_peaks",
           "ag_emap_noalloc", "ag_ctx_tune", "ag_batch_create", "ag_batch_autotune",
           "ag_batch_compute", "ag_batch_download", "ag_batch_pairs", "ag_batch_last_ms", "ag_batch_free", "ag_surrogate_set",
           "ag_surrogate_load", "ag_surrogate_save", "ag_surrogate_weights", "ag_emap_surrogate",
           "ag_surrogate_last_stats", "ag_surrogate_features", "ag_surrogate_net_grad", "ag_surrogate_train",
           "ag_surrogate_receptor"]

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
    L.ag_batch_last_ms.argtypes = [vp]
    L.ag_batch_last_ms.restype = C.c_double
    L.ag_batch_free.argtypes = [vp]
    L.ag_surrogate_set.argtypes = [vp, C.POINTER(SurrogateParams)]
    L.ag_surrogate_load.argtypes = [vp, C.c_char_p]
    L.ag_surrogate_save.argtypes = [vp, C.c_char_p]
    L.ag_surrogate_weights.argtypes = [vp, fp, dp, fp, dp]
    L.ag_emap_surrogate.argtypes = [vp, C.POINTER(Grid), C.c_int, dp, dp, fp, C.POINTER(SurrogateStats)]
    L.ag_surrogate_last_stats.argtypes = [vp, C.POINTER(SurrogateStats)]
    L.ag_surrogate_features.argtypes = [vp, C.POINTER(Grid), C.c_int, dp, dp, fp, fp]
    L.ag_surrogate_net_grad.argtypes = [vp, C.POINTER(Grid), fp, fp, fp, fp, dp]
    L.ag_surrogate_train.argtypes = [vp, C.POINTER(SurrogateTrainParams), C.POINTER(SurrogateTrainReport), dp]
    L.ag_surrogate_receptor.argtypes = [C.c_uint64, C.c_int, dp]
    _lib = L
    return L


def _check(rc):
    if rc != AG_OK:
        raise AgError(lib().ag_last_error().decode(errors="replace") + f" (code {rc})", rc)


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

    # --- learned far-field surrogate of the e-map ---------------------------
    def surrogate_set(self, r_near=10.0, coarse_spacing=1.5, probe_tol=0.005, probes_per_box=2, use_corrector=True):
        p = SurrogateParams(r_near, coarse_spacing, probe_tol, probes_per_box, 1 if use_corrector else 0)
        _check(lib().ag_surrogate_set(self.h, C.byref(p)))

    def surrogate_load(self, path=DEFAULT_WEIGHTS):
        _check(lib().ag_surrogate_load(self.h, path.encode()))

    def surrogate_save(self, path):
        _check(lib().ag_surrogate_save(self.h, path.encode()))

    def surrogate_weights(self, w=None, scales=None):
        """Set (if given) and return (FP32 weights, (s_in, s_out))."""
        win = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
        sin = None if scales is None else np.ascontiguousarray(scales, dtype=np.float64)
        wout = np.empty(SURROGATE_WEIGHTS, dtype=np.float32)
        sout = np.empty(2, dtype=np.float64)
        _check(lib().ag_surrogate_weights(self.h, None if win is None else _fp(win), None if sin is None else _dp(sin),
                                          _fp(wout), _dp(sout)))
        return wout, (float(sout[0]), float(sout[1]))

    def emap_surrogate(self, grid, xyzw, inv_eps):
        xyzw = np.ascontiguousarray(xyzw, dtype=np.float64)
        eps = np.ascontiguousarray(inv_eps, dtype=np.float64)
        out = np.empty(grid.nx * grid.ny * grid.nz, dtype=np.float32)
        st = SurrogateStats()
        _check(lib().ag_emap_surrogate(self.h, C.byref(grid), xyzw.shape[0], _dp(xyzw), _dp(eps), _fp(out),
                                       C.byref(st)))
        return out, dict(boxes=st.boxes, fallback_boxes=st.fallback_boxes, probe_max_err=st.probe_max_err)

    def surrogate_stats(self):
        st = SurrogateStats()
        _check(lib().ag_surrogate_last_stats(self.h, C.byref(st)))
        return dict(boxes=st.boxes, fallback_boxes=st.fallback_boxes, probe_max_err=st.probe_max_err)

    def surrogate_features(self, grid, xyzw, inv_eps):
        """(features (P, 8) FP32, base map (P,)) of the surrogate before its corrector."""
        xyzw = np.ascontiguousarray(xyzw, dtype=np.float64)
        eps = np.ascontiguousarray(inv_eps, dtype=np.float64)
        n = grid.nx * grid.ny * grid.nz
        feat = np.empty((n, 8), dtype=np.float32)
        base = np.empty(n, dtype=np.float32)
        _check(lib().ag_surrogate_features(self.h, C.byref(grid), xyzw.shape[0], _dp(xyzw), _dp(eps), _fp(feat),
                                           _fp(base)))
        return feat, base

    def surrogate_net_grad(self, grid, features, target=None):
        """(o, grad, loss) of the corrector on features (P, 8)."""
        feat = np.ascontiguousarray(features, dtype=np.float32)
        n = grid.nx * grid.ny * grid.nz
        o = np.empty(n, dtype=np.float32)
        grad = np.empty(SURROGATE_WEIGHTS, dtype=np.float32)
        loss = C.c_double()
        tgt = None if target is None else np.ascontiguousarray(target, dtype=np.float32)
        _check(lib().ag_surrogate_net_grad(self.h, C.byref(grid), _fp(feat), None if tgt is None else _fp(tgt),
                                           _fp(o), _fp(grad), C.byref(loss)))
        return o, (grad if tgt is not None else None), loss.value

    def surrogate_train(self, n_receptors=200, min_atoms=5000, max_atoms=30000, points=161, spacing=0.375,
                        epochs=10, lr=2e-3, seed=1):
        tp = SurrogateTrainParams(seed, n_receptors, min_atoms, max_atoms, points, spacing, epochs, lr)
        rep = SurrogateTrainReport()
        per = np.zeros(epochs, dtype=np.float64)
        _check(lib().ag_surrogate_train(self.h, C.byref(tp), C.byref(rep), _dp(per)))
        return dict(gen_seconds=rep.gen_seconds, train_seconds=rep.train_seconds, steps=rep.steps,
                    first_epoch_loss=rep.first_epoch_loss, last_epoch_loss=rep.last_epoch_loss, s_in=rep.s_in,
                    s_out=rep.s_out, loss_per_epoch=per.tolist())


def surrogate_receptor(seed, n_atoms):
    """(n, 4) atoms of the surrogate's synthetic receptor generator (centred, w = 0.1465 q)."""
    out = np.empty((n_atoms, 4), dtype=np.float64)
    _check(lib().ag_surrogate_receptor(seed, n_atoms, _dp(out)))
    return out


def ddd_table():
    """332/eps(i/100) for i < 8192, the distance-dependent dielectric table (FP64)."""
    d = np.arange(TABLE_LEN, dtype=np.float64) / 100.0
    E = np.exp(-0.3153767175 * d)
    return (332.0 + (332 * 7.7839) * E) / (78.4 + -66.57180475 * E)


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

    @property
    def last_ms(self):
        """Device time of the last compute()'s graph, in ms."""
        return lib().ag_batch_last_ms(self.h)

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
