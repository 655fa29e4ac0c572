// Launch interfaces of the grid-map kernels (host side of the CUDA code).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace agk {

constexpr int kNX = 8;            // e-map: consecutive x points per thread
constexpr int kEmapKahan = 0;
constexpr int kEmapPlain = 1;

// A CTA's work in the e-map: items [item0, item0+nitems) of the item list and
// the CTA's box: local origin (grid-centred frame, A) and half extents
// (scaled by 100) that contain every point of those items.
struct EmapBlock {
  int item0, nitems;
  double ox, oy, oz;
  float hx, hy, hz, pad;
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
  float* out;
  double* partial;                // nsplit * npoints, when nsplit > 1
  unsigned* status;
};

cudaError_t emap_launch(const EmapParams& P, bool ddd, int mode, int grid, cudaStream_t st);
size_t emap_smem_bytes();

// ---------------------------------------------------------------------------
// Affinity + desolvation
// ---------------------------------------------------------------------------
constexpr int kAffTX = 8, kAffTY = 8, kAffTZ = 4;   // points per CTA (one per thread)
constexpr int kAffMaxGroup = 8;                     // maps per pass
constexpr int kAffRows = 801;                       // table rows kept: r <= 8 A

struct AffParams {
  // receptor (device)
  int n_atoms;
  const double4* xyz;             // x, y, z, unused
  const int* info;                // type | hbond << 5 | disorder << 8 | rexp << 9
  const float* vol;
  const float* solq;              // solpar + solparQ * |q|
  const double* rv;               // rvector, 3 per atom
  const double* rv2;              // rvector2, 3 per atom
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
  int m0, G, nmaps, ntypes, hydrogen, doDmap;
  const float* table;             // [ntypes][kAffRows][G] for this pass
  const float* tableH;            // [kAffRows][G] hydrogen rows for this pass, or null
  const float* sol;               // kAffRows
  int mapHbond[kAffMaxGroup], mapIsHB[kAffMaxGroup], mapCov[kAffMaxGroup];
  float solparProbe[kAffMaxGroup], volProbe[kAffMaxGroup];
  float solparQ;
  float* out;                     // [nmaps][npoints]
  float* dmap;
  unsigned* status;
};

size_t aff_smem_bytes(int ntypes, int G);
cudaError_t aff_launch(const AffParams& P, cudaStream_t st);

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
};
cudaError_t cells_launch(const CellBuild& C, int ncellTotal, cudaStream_t st);

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
