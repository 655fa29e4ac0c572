/*
 * fastgrid_b200 — C ABI of the B200 AutoGrid grid-map engine.
 *
 * The engine computes an AutoGrid map set on one GPU: the electrostatic map
 * (e-map), one affinity map per ligand atom type and the desolvation map
 * (d-map).  The entry points below are the seams at which the reference
 * (FastGrid, fastgrid_master/fastgrid/) dispatches that work; each declaration
 * names the reference interface it replaces.  All arguments are plain C types
 * and host pointers unless a name says "device"; no exceptions cross this
 * boundary.  Every function returns AG_OK (0) or a negative AG_E* code, and
 * ag_last_error() then describes the failure (thread-local).
 *
 * Coordinates are in the grid-centred frame used by the reference: grid point
 * (i, j, k) sits at ((i - nx/2)*h, (j - ny/2)*h, (k - nz/2)*h) with integer
 * division (autogrid.h:267-286), and receptor atoms have had the grid centre
 * subtracted (InputDataLoader.cpp:466-467).  Map values are written x fastest,
 * then y, then z, as FP32 and unrounded (the writers round to 3 decimals).
 */
#ifndef FASTGRID_B200_H
#define FASTGRID_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AG_OK 0
#define AG_E_INVALID (-1)   /* bad argument */
#define AG_E_CUDA (-2)      /* CUDA runtime error (device, launch, copy) */
#define AG_E_DEVICE (-3)    /* a kernel reported an error status (e.g. a bounded wait expired) */
#define AG_E_HOST (-4)      /* input file / host-side failure */
#define AG_E_NOMEM (-5)     /* allocation failure */

#define AG_TABLE_LEN 8192   /* 0.01 A bins, MAX_DIST (autogrid.h:215) */

typedef struct ag_ctx ag_ctx;
typedef struct ag_problem ag_problem;

/* Grid shape: nx, ny, nz points (odd in AutoGrid GPFs) at `spacing` A. */
typedef struct ag_grid {
  int nx, ny, nz;
  double spacing;
} ag_grid;

/* Receptor, structure of arrays (InputData.h:53-58 + BondVectors.h:27-31). */
typedef struct ag_receptor {
  int n_atoms;
  const double* xyzw;          /* 4 per atom: centred x, y, z and the e-map weight
                                  q*coeff_estat (distance-dependent dielectric) or
                                  q*coeff_estat*332/diel (constant dielectric) */
  const double* charge;        /* partial charge q */
  const double* vol;           /* atomic fragmental volume */
  const double* solpar;        /* atomic solvation parameter */
  const int* type;             /* receptor type index, < n_types */
  const int* hbond;            /* 0 NON, 1 DS, 2 D1, 3 AS, 4 A1, 5 A2 */
  const unsigned char* disorder;
  const int* rexp;             /* 2 (N-H) or 4 (O-H / S-H) for D1 atoms */
  const double* rvector;       /* 3 per atom, unit bond vector */
  const double* rvector2;      /* 3 per atom, unit lone-pair plane normal (A2) */
} ag_receptor;

/* Per-map parameters of the affinity + desolvation pass
 * (GridMap.h:27-57, PairwiseInteractionEnergies.h:31-49, DesolvExpFunc.h). */
typedef struct ag_affinity_params {
  int n_maps;                  /* ligand (atom) maps, <= 14 */
  int n_types;                 /* receptor types, <= 32 */
  const double* energy;        /* [n_types][AG_TABLE_LEN][n_maps] pair energies */
  const double* sol;           /* [AG_TABLE_LEN] coeff_desolv*exp(-r^2/25.92) */
  const int* map_hbond;        /* per map: H-bond character of the probe */
  const int* map_is_hbonder;   /* per map: GridMap::isHBonder */
  const int* map_is_covalent;  /* per map: covalent maps are skipped here */
  const double* solpar_probe;  /* per map */
  const double* vol_probe;     /* per map */
  double solpar_q;             /* charge-dependent solvation coefficient (qasp) */
  int hydrogen;                /* receptor type index of "HD", or -1 */
} ag_affinity_params;

/* ------------------------------------------------------------------------ */
/* Context: one per host thread; owns a CUDA stream and device buffers.     */
/* ------------------------------------------------------------------------ */
int ag_ctx_create(int device, ag_ctx** out);
int ag_ctx_destroy(ag_ctx* ctx);
const char* ag_last_error(void);
/* The cudaStream_t the context launches on (for event timing by callers). */
void* ag_ctx_stream(ag_ctx* ctx);
/* Number of kernel launches issued by this context so far. */
int64_t ag_ctx_launch_count(const ag_ctx* ctx);

/* Tuning knobs of a context (no reference counterpart; the reference's
 * --cuda-* switches played this role for its kernels).  Results stay within
 * the stated tolerances for every allowed value. */
#define AG_TUNE_EMAP_RNEAR 1          /* A, >= 8: atoms nearer the CTA box take the exact-bin path (default 11) */
#define AG_TUNE_EMAP_PACKED_TABLE 2   /* 0/1: mid atoms in the table's saturating tail (from about 22 A) read 16- and 8-bit copies of it (1, default) or the FP32 table (0) */
#define AG_TUNE_EMAP_CTAS_PER_SM 3    /* 1..8: CTAs per SM the atom split aims for on small grids (default 3) */
#define AG_TUNE_EMAP_WARP_COMPACT 4   /* e-map item order: 0 rows, 1 each warp's items form a compact box, 2 as 1 with
                                         neighbouring lanes sharing a 16-point x span alternately (default 2) */
#define AG_TUNE_EMAP_TILE 5           /* direct e-map: TX*10000 + TY*100 + TZ work items per CTA tile, product 256 (default 20816) */
#define AG_TUNE_SURROGATE_TCGEN05 6   /* 0/1: surrogate corrector convolutions on tcgen05 (1, default) or mma.sync (0) */
#define AG_TUNE_AFFINITY_KERNEL 9     /* affinity pass: 2 two grid points per thread, type-major candidates,
                                         nearest donor found in the kernel (default); 1 one point per thread
                                         with a separate nearest-donor kernel (also used for passes with more
                                         than 4 H-bond maps) */
#define AG_TUNE_CONCURRENT_PASSES 10 /* 0/1: a map set's e-map and affinity pass run concurrently, the e-map on a
                                         high-priority stream (1, default), or one after the other (0) */
/* Failure-detection test hooks (default 0 = off).  IDLE_WAIT: 1..64 polls of an
 * extra wait, after each direct e-map CTA's first atom tile has landed, on a
 * barrier nothing arrives on; the wait expires, the kernel records it in its
 * status word, lets its own copies land and returns, and the call fails with
 * AG_E_DEVICE.  CHECKSUM_OFFSET: added to the host's FP64 sum of the input
 * weights before the net-charge checksum comparison, so a nonzero value makes
 * the call fail with AG_E_DEVICE. */
#define AG_TUNE_TEST_IDLE_WAIT 7
#define AG_TUNE_TEST_CHECKSUM_OFFSET 8
int ag_ctx_tune(ag_ctx* ctx, int knob, double value);

/* ------------------------------------------------------------------------ */
/* Electrostatic map.                                                        */
/* Replaces calculateElectrostaticMapAsync + synchronizeCalculation          */
/* (electrostatics/Electrostatics.h:32-36; CPU body Cpu.cpp:27-112, CUDA     */
/* body Cuda.cpp:75-249).  e(p) = sum over all atoms of                       */
/* w * min(1/r, 2) * inv_eps[min(int(100 r), 8191)], no cutoff.             */
/* inv_eps == NULL selects the constant dielectric (w already holds 332/diel).*/
/* `out` receives nx*ny*nz FP32 values.  Synchronous.                        */
/* ------------------------------------------------------------------------ */
int ag_emap(ag_ctx* ctx, const ag_grid* grid, int n_atoms, const double* xyzw, const double* inv_eps,
            float* out);

/* Precision modes of the e-map accumulation (for the precision study). */
#define AG_EMAP_KAHAN 0      /* Kahan-compensated FP32 per atom tile, FP64 across tiles (default) */
#define AG_EMAP_PLAIN 1      /* plain FP32 accumulation over all atoms */
int ag_emap_mode(ag_ctx* ctx, const ag_grid* grid, int n_atoms, const double* xyzw, const double* inv_eps,
                 int mode, float* out);

/* ------------------------------------------------------------------------ */
/* Affinity maps + desolvation map in one fused pass.                        */
/* Replaces calculateGridmaps (CalculateGridmaps.h:30-31, body               */
/* CalculateGridmaps.cpp:433-485).  out_maps receives n_maps*nx*ny*nz FP32   */
/* values (map-major), out_dmap nx*ny*nz.  Covalent maps are left untouched. */
/* ------------------------------------------------------------------------ */
int ag_affinity(ag_ctx* ctx, const ag_grid* grid, const ag_receptor* rec, const ag_affinity_params* par,
                float* out_maps, float* out_dmap);

/* ------------------------------------------------------------------------ */
/* Device-resident form, for callers that keep inputs in HBM between calls:  */
/* ag_upload stages a job into context-owned device memory, ag_compute runs  */
/* the kernels on it (AG_WORK_* bits), ag_download copies the maps back.     */
/* ------------------------------------------------------------------------ */
#define AG_WORK_EMAP 1
#define AG_WORK_AFFINITY 2
#define AG_WORK_ALL 3
int ag_upload(ag_ctx* ctx, const ag_grid* grid, const ag_receptor* rec, const ag_affinity_params* par,
              const double* inv_eps);
int ag_compute(ag_ctx* ctx, int work);
/* Device pointer to the map set [n_maps atom maps][e-map][d-map], FP32. */
float* ag_device_maps(ag_ctx* ctx);
/* out: (n_maps + 2) * nx*ny*nz floats in the same order. */
int ag_download(ag_ctx* ctx, float* out);

/* ------------------------------------------------------------------------ */
/* Whole jobs (the drop-in for programMain, main.cpp:115-254).               */
/* ------------------------------------------------------------------------ */
typedef struct ag_problem_info {
  int nx, ny, nz;
  double spacing;
  double center[3];
  int n_atoms;
  int n_maps;                  /* ligand maps; the set also has the e-map and d-map */
  int n_types;
  int dist_dep_diel;
  int has_floating_grid;
} ag_problem_info;

/* Parse a GPF (and the PDBQT / parameter file it names) and precompute the
 * tables and bond vectors, as InputDataLoader::load + main.cpp:163-193 do.
 * Writes the .xyz file (on the GPF's gridcenter line) and the .fld file. */
int ag_problem_load(const char* gpf_path, int use_v4_params, const char* log_path, ag_problem** out);
void ag_problem_free(ag_problem* p);
int ag_problem_info_get(const ag_problem* p, ag_problem_info* info);
/* Views of the host arrays the GPU consumes (valid while p lives). */
int ag_problem_views(const ag_problem* p, ag_grid* grid, ag_receptor* rec, ag_affinity_params* par,
                     const double** inv_eps);
/* Compute the whole map set on the GPU (also covalent maps and the floating grid).
 * Synchronous: the maps are in host memory (ag_problem_maps) when it returns.
 * The problem keeps a page-locked buffer for the maps, and its atom array is
 * page-locked on the first call; both are released by ag_problem_free. */
int ag_problem_compute(ag_ctx* ctx, ag_problem* p);
/* Host copy of the map set [n_maps][e][d], FP32 unrounded; n*(n_maps+2) floats. */
const float* ag_problem_maps(const ag_problem* p);
/* Write every .map file (and the floating grid) like GridMapList::saveGridMap. */
int ag_problem_write(ag_problem* p);

/* ------------------------------------------------------------------------ */
/* Batches: many map sets (receptors or conformations of uneven atom counts */
/* and grid sizes) computed by persistent e-map and affinity kernels that   */
/* take (job, CTA) work units from a counter, largest first; the first      */
/* ag_batch_compute captures the whole batch in a CUDA graph and later calls*/
/* replay it.  No counterpart in the reference (one job per process).       */
/* Problems must outlive the batch; all use the distance-dependent          */
/* dielectric.                                                               */
/* ------------------------------------------------------------------------ */
typedef struct ag_batch ag_batch;
int ag_batch_create(ag_ctx* ctx, ag_problem* const* problems, int n, ag_batch** out);
/* Choose the e-map CTA tile shape per size class (atom count x grid size) by
 * timing candidates on one job of each class; cache_path (or NULL) names a
 * text file of earlier choices that is read first and rewritten after. */
int ag_batch_autotune(ag_batch* b, const char* cache_path);
int ag_batch_compute(ag_batch* b);
/* Map set of problem i: (n_maps + 2) * nx*ny*nz floats, as ag_download. */
int ag_batch_download(ag_batch* b, int i, float* out);
/* Sum over the batch of n_atoms x n_points (the batch's point-atom pairs). */
double ag_batch_pairs(const ag_batch* b);
/* Device time in ms of the last ag_batch_compute's graph (CUDA events). */
double ag_batch_last_ms(const ag_batch* b);
int ag_batch_free(ag_batch* b);

/* The autogrid4 / fastgrid4 command line (ProgramParameters.cpp:63-112). */
int ag_main(int argc, char** argv);

/* E-map without any device memory allocation.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc/cudaFree — hosts that
 * manage the GPU's memory in their own pool or run under a fixed memory budget
 * where an allocation could synchronise the device or fail mid-run.  Inputs
 * and output are the caller's device buffers: d_xyzw (n_atoms x 4 doubles,
 * as for ag_emap, 16-byte aligned), d_inv_eps (8192 FP32 values of 332/eps,
 * 16-byte aligned, or NULL for the constant dielectric), d_out (nx*ny*nz
 * floats, 4-byte aligned); misaligned pointers are rejected with
 * AG_E_INVALID before any CUDA call.  Work is issued on `stream` (a
 * cudaStream_t, NULL for the default stream) and the call is synchronous: it
 * returns when that work is done, so it cannot be recorded into a stream
 * capture (a call on a capturing stream fails with AG_E_CUDA).  Scratch
 * lives in fixed device arrays of the library (about 21 MiB on each device
 * that loads it, kept until exit): grids above about 8.4 million points
 * (1,048,576 rows of 8 points) are rejected with AG_E_INVALID, also before
 * any CUDA call.  All calls share those arrays and they keep the last call's
 * contents, so calls whose GPU work overlaps race; serialise them.  The first
 * call on a device (and the first after its context is re-created) also
 * performs that device's set-up.  Each call reads the dielectric table back
 * to the host (32 KB) to pack its saturating tail, as ag_emap does.  Like
 * ag_emap it checks the net charge: the
 * kernel's FP64 sum of the weights it consumed must equal the input's, else
 * AG_E_DEVICE. */
int ag_emap_noalloc(const ag_grid* grid, int n_atoms, const double* d_xyzw, const float* d_inv_eps, float* d_out,
                    void* stream);

/* ------------------------------------------------------------------------ */
/* Learned far-field surrogate of the e-map (no reference counterpart; an   */
/* approximate, faster alternative to ag_emap for the distance-dependent    */
/* dielectric).  The map is split exactly into                              */
/*   near field: the exact binned sum over atoms within r_near, minus a     */
/*     smooth kernel psi for those atoms, and                               */
/*   far field: the sum of psi over all atoms, sampled on a coarse grid,    */
/*     interpolated trilinearly and corrected by a 3-layer 3x3x3            */
/*     convolutional network (32 channels, BF16 weights, FP32 accumulation).*/
/* Residual probes (the exact FP64 direct sum at a few points of every CTA  */
/* box) send each box whose error exceeds probe_tol back to the direct sum. */
/* ------------------------------------------------------------------------ */
typedef struct ag_surrogate_params {
  double r_near;               /* A, radius of the exact near field (default 10) */
  double coarse_spacing;       /* A, far-field grid (default 1.5; rounded to a multiple of the map spacing) */
  double probe_tol;            /* kcal/mol/e; <= 0 turns the probes and the fallback off (default 0.005) */
  int probes_per_box;          /* probe points per CTA box (default 2) */
  int use_corrector;           /* 0: trilinear far field only (default 1) */
} ag_surrogate_params;
typedef struct ag_surrogate_stats {
  int boxes;                   /* CTA boxes of the last surrogate e-map */
  int fallback_boxes;          /* boxes recomputed by the direct sum */
  double probe_max_err;        /* largest probe error before the fallback (kcal/mol/e) */
} ag_surrogate_stats;
#define AG_SURROGATE_WEIGHTS 35424 /* W1 [27][8][32] | W2 [27][32][32] | W3 [27][32] */
#define AG_WORK_EMAP_SURROGATE 4   /* ag_compute: the e-map slot by the surrogate */

int ag_surrogate_set(ag_ctx* ctx, const ag_surrogate_params* p); /* NULL restores the defaults */
/* Corrector weights file (BF16 weights and the input/output scales). */
int ag_surrogate_load(ag_ctx* ctx, const char* path);
int ag_surrogate_save(ag_ctx* ctx, const char* path);
/* FP32 copies of the weights in (w_in) and out (w_out), either may be NULL;
 * scales[0] = input scale, scales[1] = output scale, read (scales_in) and
 * written (scales_out), either may be NULL. */
int ag_surrogate_weights(ag_ctx* ctx, const float* w_in, const double* scales_in, float* w_out, double* scales_out);
/* The e-map by the surrogate, host buffers, synchronous (like ag_emap). */
int ag_emap_surrogate(ag_ctx* ctx, const ag_grid* grid, int n_atoms, const double* xyzw, const double* inv_eps,
                      float* out, ag_surrogate_stats* stats);
int ag_surrogate_last_stats(ag_ctx* ctx, ag_surrogate_stats* stats);
/* Test hooks: the corrector's 8 input features per point (FP32 values of the
 * BF16 inputs, scaled) and the map before the corrector (near + trilinear
 * far field) of a job. */
int ag_surrogate_features(ag_ctx* ctx, const ag_grid* grid, int n_atoms, const double* xyzw, const double* inv_eps,
                          float* features, float* base);
/* The network alone on features (P x 8, rounded to BF16 on upload): output
 * o (P, in units of the output scale) and, with a target (P), the loss
 * mean((o - target / s_out)^2) and its gradient with respect to the
 * AG_SURROGATE_WEIGHTS weights.  Outputs may be NULL. */
int ag_surrogate_net_grad(ag_ctx* ctx, const ag_grid* grid, const float* features, const float* target, float* o,
                          float* grad, double* loss);

/* Training on synthetic receptors (globules at 0.06 atoms/A^3, charges
 * N(0, 0.2) clipped at 0.7, net 0), each e-map computed by the direct
 * kernel; Adam on FP32 master weights, forward and backward on the GPU. */
typedef struct ag_surrogate_train_params {
  uint64_t seed;
  int n_receptors;             /* e.g. 200 */
  int min_atoms, max_atoms;    /* log-uniform atom counts, e.g. 5000 .. 30000 */
  int points;                  /* grid points per axis, e.g. 161 */
  double spacing;              /* A, e.g. 0.375 */
  int epochs;
  double lr;                   /* peak Adam learning rate, e.g. 2e-3 */
} ag_surrogate_train_params;
typedef struct ag_surrogate_train_report {
  double gen_seconds;          /* receptors, direct e-maps and features */
  double train_seconds;
  int steps;
  double first_epoch_loss, last_epoch_loss;
  double s_in, s_out;
} ag_surrogate_train_report;
/* loss_per_epoch (or NULL) receives `epochs` mean training losses. */
int ag_surrogate_train(ag_ctx* ctx, const ag_surrogate_train_params* tp, ag_surrogate_train_report* rep,
                       double* loss_per_epoch);
/* Write the atoms of the synthetic training/evaluation receptor generator:
 * xyzw (n_atoms x 4: centred coordinates, q * 0.1465). */
int ag_surrogate_receptor(uint64_t seed, int n_atoms, double* xyzw);

/* Measured issue-rate peaks of a device (no reference counterpart; used for
 * the e-map's roofline): SFU reciprocal square roots per second and FP32 FMA
 * instructions per second, at the clocks the device runs at now. */
int ag_measure_peaks(int device, double* rsqrt_per_s, double* ffma_per_s);

/* ------------------------------------------------------------------------ */
/* Seeded synthetic receptors for tests and benchmarks: a self-avoiding      */
/* chain walk inside a sphere or ellipsoid, AutoDock4 types by fraction,     */
/* charges N(0, sigma) clipped and shifted to a net charge, 3-decimal values.*/
/* Writes <dir>/<stem>.pdbqt and <dir>/<stem>.gpf.                           */
/* ------------------------------------------------------------------------ */
typedef struct ag_synth_params {
  uint64_t seed;
  int n_atoms;
  double semi_axes[3];         /* ellipsoid semi-axes in A (equal: sphere) */
  double origin[3];            /* shape centre */
  double frac_C, frac_OA, frac_N, frac_HD, frac_A, frac_SA;
  double charge_sigma, charge_clip, net_charge;
  int npts;                    /* GPF npts (even): npts+1 points per axis */
  double spacing;
  const char* ligand_types;    /* space-separated, e.g. "A C HD N OA SA" */
  double dielectric;           /* GPF dielectric line value, e.g. -0.1465 */
} ag_synth_params;
int ag_synth_write(const char* dir, const char* stem, const ag_synth_params* sp);

#ifdef __cplusplus
}
#endif
#endif /* FASTGRID_B200_H */
