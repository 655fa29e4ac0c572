// Launch interfaces of the grid-map kernels (host side of the CUDA code).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace agk {

constexpr int kNX = 8;            // e-map: consecutive x points per thread
constexpr int kEmapKahan = 0;
constexpr int kEmapPlain = 1;
constexpr int kItemInterleaved = 1 << 30;  // e-map item flag: x points shared alternately with the partner column
constexpr int kEmapCtasPerSm = 3;  // e-map CTAs resident per SM (register bound 85)
constexpr int kEmapPackedBytes = 16384;  // e-map: shared-memory region of the packed table tail

// A CTA's work in the e-map: items [item0, item0+nitems) of the item list and
// the CTA's box: local origin (grid-centred frame, A) and half extents
// (scaled by 100) that contain every point of those items.
struct EmapBlock {
  int item0, nitems;
  double ox, oy, oz;
  float hx, hy, hz;
  float rfar2;                    // (100 * rFar)^2, rFar >= 50 A
  int clampMid;                   // 1 if rFar + box diagonal can reach 81.9 A: clamp mid-list bins at 8191
  int pad;
};

struct EmapParams {
  const double4* atoms;           // n_atoms (x, y, z, w), grid-centred
  int n_atoms, chunk, nsplit, nblocks;
  const int* items;               // packed (xc | y << 8 | z << 19)
  const EmapBlock* blocks;
  int nx, ny, nz, n2x, n2y, n2z;
  int64_t npoints;
  double h;
  const float* table;             // 8192 entries of 332/eps(r), FP32
  const double* thr;              // thr[k]: least r^2 whose reference bin is >= k
  float rnear2;                   // (100 * rNear)^2
  float delta;                    // guard half-width around bin edges (units of 0.01 A)
  // Packed copies of the table's saturating tail (null: not used).  Entry b
  // of the table, for b >= b16 (b8), is bits(table[8191]) + k with k stored
  // in 16 (8) bits; the 16-bit entries for bins [b16, 8192) come first, then
  // the 8-bit entries for bins [b8, 8192), each part padded to 16 bytes.
  const uint4* packed;
  int packedVecs;                 // 16-byte vectors in `packed`
  int vec8;                       // vector at which the 8-bit part starts
  int b16, b8;
  float r16sq, r8sq;              // (b16 + 2)^2, (b8 + 2)^2: mid atoms at least that far (0.01 A units) from the box
  float kScale;                   // 2^(e + 126) / g, g = table[8191] = 2^e * m: turns 100 w g 2^-16 into 100 w ulp(g) 2^133
  int testIdleWait;               // test hook: > 0 adds a wait of that many polls on a barrier nothing arrives on
  float* out;
  double* partial;                // nsplit * npoints, when nsplit > 1
  unsigned* status;
  double* checksum;               // per split: FP64 sum of the weights the split's first CTA consumed (or null)
  // Near-field mode of the far-field surrogate: only atoms within rcut of a
  // point count, each as w * (exact term - psi(r)), psi(r) = (psi[0] +
  // psi[1] r2 + psi[2] r2^2) / 100 with r2 in (0.01 A)^2 units.
  float rcut2;                    // (100 * rcut)^2
  float psi[3];
  const float4* tileLo;           // near field: per 256-atom tile, bounding box of its atoms (A)
  const float4* tileHi;
};

cudaError_t emap_launch(const EmapParams& P, bool ddd, int mode, int grid, cudaStream_t st);
// Near field of the surrogate e-map (distance-dependent dielectric, Kahan).
cudaError_t emap_near_launch(const EmapParams& P, int grid, cudaStream_t st);
// Direct e-map of the CTA boxes list[0 .. *count) (no atom split), by `grid`
// persistent CTAs; the surrogate's fallback for boxes whose probe failed.
cudaError_t emap_list_launch(const EmapParams& P, const int* list, const int* count, int* counter, int grid,
                             cudaStream_t st);
size_t emap_smem_bytes();
// Persistent e-map over the units (job, CTA box) of many jobs (no atom split, distance-dependent dielectric).
cudaError_t emap_batch_launch(const EmapParams* jobs, const int2* units, int nunits, int* counter, int grid,
                              cudaStream_t st);

// ---------------------------------------------------------------------------
// Affinity + desolvation
// ---------------------------------------------------------------------------
constexpr int kAffTX = 8, kAffTY = 8, kAffTZ = 4;   // points per CTA (one per thread)
constexpr int kAffRows = 801;                       // table rows kept: r <= 8 A
constexpr int kMaxTypes = 32;                       // receptor types
constexpr int kMaxMapsPass = 16;                    // ligand maps per pass
constexpr int kMaxMinMax = 4;                       // maps per pass with H-bond min/max bookkeeping

// Per (receptor type, map) H-bond handling, 2 bits per map in typeModes[t]
// (CalculateGridmaps.cpp:206-228): 0 add E; 1 acceptor probe vs donor atom
// (Hramp, racc weighting); 2 A1 probe vs donor atom (min/max, racc);
// 3 donor probe vs acceptor atom (min/max, rdon).
struct AffParams {
  // receptor (device)
  int n_atoms;
  const double4* xyz;             // FP64 grid-centred x, y, z (w unused)
  const int* info;                // type | hbond << 5 | disorder << 8 | rexp << 9
  const float* vol;
  const float* solq;              // solpar + solparQ * |q|
  const float* rv;                // rvector, 3 per atom (FP32)
  const float* rv2;               // rvector2, 3 per atom (FP32)
  const double* rv64;             // rvector, 3 per atom (FP64, for exact sign decisions)
  // cell list (8 A cells)
  const int* cellStart;           // ncell + 1
  const int* cellAtoms;
  double cellLo[3];
  int ncell[3];
  const int* closestH;            // per point: index of the nearest H donor within 8 A, or -1
  // grid
  int nx, ny, nz, n2x, n2y, n2z;
  int64_t npoints;
  double h;
  // maps of this pass
  int nmaps, nmPad, ntypes, hydrogen;
  const float* table;             // [ntypes][kAffRows][nmPad] FP32
  const float* tableH;            // [kAffRows][nmPad] rows of the "HD" type (disordered donors), or null
  const float* sol;               // kAffRows
  const double* thr;              // thr[k]: least r^2 whose reference bin int(100/(1/sqrt(r^2))) is >= k
  float delta;                    // guard half-width around bin edges (units of 0.01 A)
  int typeHbond[kMaxTypes];
  unsigned typeModes[kMaxTypes];
  int typeNeedsAngular[kMaxTypes];
  int mapMinMaxSlot[kMaxMapsPass];
  int mapCov[kMaxMapsPass];
  float solparProbe[kMaxMapsPass], volProbe[kMaxMapsPass];
  float solparQ;
  float* out;                     // this pass's first map: [nmaps][npoints]
  float* dmap;
  unsigned* status;
};

size_t aff_smem_bytes(int nmPad);
cudaError_t aff_launch(const AffParams& P, cudaStream_t st);
// Persistent affinity pass over the units (job, CTA block) of many jobs.
cudaError_t aff_batch_launch(const AffParams* jobs, const int2* units, int nunits, int* counter, int nmPadMax,
                             int nmapsMax, int grid, cudaStream_t st);

// Cell list build (counting sort of atoms into 8 A cells, file order kept inside each cell).
struct CellBuild {
  const double4* xyz;
  int n_atoms;
  double lo[3];
  int ncell[3];
  int* cellOf;                    // n_atoms scratch
  int* count;                     // ncell + 1 scratch (zeroed by the launcher)
  int* cellStart;                 // ncell + 1
  int* cellAtoms;                 // n_atoms
  int* fill;                      // ncell scratch
  const int* donorMask;           // optional: only atoms with mask[i] != 0 (null = all)
  const int* typeInfo;            // optional: key = cell * ntypes + (typeInfo[i] & 31) (type-major segments)
  int ntypes;
};
// ncellTotal: number of keys (cells, or cells x ntypes with typeInfo).
cudaError_t cells_launch(const CellBuild& C, int ncellTotal, cudaStream_t st);

// ---------------------------------------------------------------------------
// Affinity + desolvation, two grid points per thread (affinity2.cu)
// ---------------------------------------------------------------------------
constexpr int kA2Slots = 4;         // H-bond maps per pass handled by the two-point kernel
enum { A2_SPH = 0, A2_D1 = 1, A2_A1 = 2, A2_A2 = 3 };          // angular class of a receptor type
enum { A2_SLOT_ACC = 0, A2_SLOT_A1 = 1, A2_SLOT_DON = 2 };     // H-bond map kind (probe class)

struct Aff2Params {
  // receptor (device)
  const double4* xyz;             // FP64 grid-centred x, y, z
  const int* info;                // type | hbond << 5 | disorder << 8 | rexp << 9
  const float* vol;
  const float* solq;
  const float* rv;                // rvector (FP32, 3 per atom)
  const float* rv2;               // rvector2 (FP32, 3 per atom)
  const double* rv64;             // rvector (FP64) for exact sign decisions
  // type-major cell list: segment (cell, type) = atoms ctAtoms[ctStart[cell*ntypes+t] .. ctStart[...+1])
  const int* ctStart;
  const int* ctAtoms;
  double cellLo[3];
  int ncell[3];
  // grid
  int nx, ny, nz, n2x, n2y, n2z;
  int64_t npoints;
  double h;
  // maps of this pass
  int nmaps, nmPad, ntypes, hydrogen;
  const float* table;             // [ntypes][kAffRows][nmPad] FP32
  const float* tableH;            // [kAffRows][nmPad] rows of the "HD" type, or null
  const float* sol;               // kAffRows
  int solInRow;                   // the table rows' last column (nmPad - 1 >= nmaps) holds sol
  const double* thr;              // affinity bin thresholds (kAffRows + 1)
  float delta;                    // guard half-width around bin edges (bins)
  int needClosestH;               // some D1 type meets an acceptor-probe slot: find the nearest donor
  int typeAng[kMaxTypes];         // A2_SPH / A2_D1 / A2_A1 / A2_A2
  int typeDonor[kMaxTypes];       // DS or D1 (candidates of the nearest-donor search)
  unsigned typeSlots[kMaxTypes];  // bit k: H-bond slot k applies to this type
  unsigned typePlain[kMaxTypes];  // bit g: map g takes the plain table sum for this type
  int nslots;
  int slotMap[kA2Slots];          // map index of each H-bond slot
  int slotKind[kA2Slots];         // A2_SLOT_*
  int mapCov[kMaxMapsPass];
  float solparProbe[kMaxMapsPass], volProbe[kMaxMapsPass];
  float solparQ;
  float* out;                     // this pass's first map: [nmaps][npoints]
  float* dmap;
  unsigned* status;
  int ctaBase;                    // first CTA block of a launch (0, or a z-slab chunk's first block)
};
size_t aff2_smem_bytes(int nmPad);
cudaError_t aff2_launch(const Aff2Params& P, cudaStream_t st);
// Blocks [b0, b1) of the pass (the grid's CTA blocks run z-slab by z-slab).
cudaError_t aff2_launch_range(const Aff2Params& P, int b0, int b1, cudaStream_t st);
// CTA blocks (work units) of the two-point kernel on an nx x ny x nz grid.
int aff2_ctas(int nx, int ny, int nz);
// Persistent two-point pass over the units (job, CTA block) of many jobs.
cudaError_t aff2_batch_launch(const Aff2Params* jobs, const int2* units, int nunits, int* counter, int nmPadMax,
                              int nmapsMax, int grid, cudaStream_t st);

struct ClosestHParams {
  const double4* xyz;
  const int* cellStart;
  const int* cellAtoms;           // donor-only cell list
  double cellLo[3];
  int ncell[3];
  int nx, ny, nz, n2x, n2y, n2z;
  int64_t npoints;
  double h;
  int* closestH;
};
cudaError_t closest_h_launch(const ClosestHParams& P, cudaStream_t st);

// Covalent map (main.cpp:32-52) and floating grid (main.cpp:54-79).
cudaError_t covalent_launch(float* out, int nx, int ny, int nz, double h, const double cov[3], double hwInv,
                            double barrier, cudaStream_t st);
cudaError_t floating_launch(const double4* xyz, int n_atoms, int nx, int ny, int nz, double h, float* out,
                            cudaStream_t st);

}  // namespace agk
