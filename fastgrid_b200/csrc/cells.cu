// Helper kernels of the affinity pass and the small per-point maps:
//  * the device cell list (counting sort of atoms into 8 A cells, file order
//    kept inside each cell) that replaces FastGrid's cutoff grid
//    (SpatialGrid.h:50-315),
//  * the nearest H donor of every grid point (the role of FastGrid's ANN
//    kd-tree query, CalculateGridmaps.cpp:246-250, 417-431),
//  * the covalent map (main.cpp:32-52) and the floating grid (main.cpp:54-79).
#include <cuda_runtime.h>

#include <cstdint>

#include "ag_device.cuh"
#include "ag_kernels.h"

namespace agk {

// Exact FP64 squared distance as the reference forms it (Vec3d::MagnitudeSqr
// of atom - gridPos, left to right, separately rounded).
__device__ __forceinline__ double rsq_exact_c(double ax, double ay, double az, double gx, double gy, double gz) {
  const double dx = __dsub_rn(ax, gx), dy = __dsub_rn(ay, gy), dz = __dsub_rn(az, gz);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// ---------------------------------------------------------------------------
// Cell list: counting sort into 8 A cells (or into (cell, type) segments);
// file order inside each cell or segment.
// ---------------------------------------------------------------------------
__global__ void cell_count_kernel(CellBuild C) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n_atoms; i += gridDim.x * blockDim.x) {
    int cell = -1;
    if (!C.donorMask || C.donorMask[i]) {
      const double4 a = C.xyz[i];
      const int cx = (int)floor((a.x - C.lo[0]) / 8.0), cy = (int)floor((a.y - C.lo[1]) / 8.0),
                cz = (int)floor((a.z - C.lo[2]) / 8.0);
      if (cx >= 0 && cy >= 0 && cz >= 0 && cx < C.ncell[0] && cy < C.ncell[1] && cz < C.ncell[2]) {
        cell = (cz * C.ncell[1] + cy) * C.ncell[0] + cx;
        if (C.typeInfo) cell = cell * C.ntypes + (C.typeInfo[i] & 31);
      }
    }
    C.cellOf[i] = cell;
    if (cell >= 0) atomicAdd(&C.count[cell], 1);
  }
}

// Exclusive scan of the counts by one CTA (cells are at most a few hundred thousand).
__global__ void cell_scan_kernel(const int* count, int n, int* start) {
  __shared__ int part[1024];
  const int tid = threadIdx.x;
  const int per = (n + 1023) / 1024;
  const int b = tid * per, e = min(n, b + per);
  int s = 0;
  for (int i = b; i < e; i++) s += count[i];
  part[tid] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  int run = part[tid] - s;
  for (int i = b; i < e; i++) { start[i] = run; run += count[i]; }
  if (tid == 1023) start[n] = part[1023];
}

__global__ void cell_scatter_kernel(CellBuild C) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n_atoms; i += gridDim.x * blockDim.x) {
    const int cell = C.cellOf[i];
    if (cell >= 0) C.cellAtoms[C.cellStart[cell] + atomicAdd(&C.fill[cell], 1)] = i;
  }
}

// Restore file order inside each cell (one warp per cell, rank sort).
__global__ void cell_sort_kernel(const int* cellStart, int ncell, int* cellAtoms, int* tmp) {
  const int warpsPerBlock = blockDim.x / 32;
  const int lane = threadIdx.x & 31;
  for (int c = blockIdx.x * warpsPerBlock + threadIdx.x / 32; c < ncell; c += gridDim.x * warpsPerBlock) {
    const int b = cellStart[c], e = cellStart[c + 1];
    for (int i = b + lane; i < e; i += 32) {
      const int v = cellAtoms[i];
      int rank = 0;
      for (int j = b; j < e; j++) rank += cellAtoms[j] < v;
      tmp[b + rank] = v;
    }
    __syncwarp();
    for (int i = b + lane; i < e; i += 32) cellAtoms[i] = tmp[i];
  }
}

cudaError_t cells_launch(const CellBuild& C, int ncellTotal, cudaStream_t st) {
  cudaMemsetAsync(C.count, 0, sizeof(int) * (ncellTotal + 1), st);
  cudaMemsetAsync(C.fill, 0, sizeof(int) * (ncellTotal + 1), st);
  const int blocks = max(1, min(1184, (C.n_atoms + 255) / 256));
  cell_count_kernel<<<blocks, 256, 0, st>>>(C);
  cell_scan_kernel<<<1, 1024, 0, st>>>(C.count, ncellTotal, C.cellStart);
  cell_scatter_kernel<<<blocks, 256, 0, st>>>(C);
  // cellOf (n_atoms entries) is free after the scatter and serves as the sort's scratch.
  cell_sort_kernel<<<max(1, min(2048, (ncellTotal + 7) / 8)), 256, 0, st>>>(C.cellStart, ncellTotal, C.cellAtoms,
                                                                         C.cellOf);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Nearest H donor per grid point (argmin over DS/D1 atoms within the 27 cells
// around the point's cell, ties to the lower file index), FP64 like the
// reference's kd-tree query (CalculateGridmaps.cpp:246-250).
// ---------------------------------------------------------------------------
__global__ void closest_h_kernel(ClosestHParams P) {
  for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.npoints;
       pt += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(pt % P.nx), iy = (int)((pt / P.nx) % P.ny), iz = (int)(pt / ((int64_t)P.nx * P.ny));
    const double gx = __dmul_rn((double)(ix - P.n2x), P.h), gy = __dmul_rn((double)(iy - P.n2y), P.h),
                 gz = __dmul_rn((double)(iz - P.n2z), P.h);
    const int cx = (int)floor((gx - P.cellLo[0]) / 8.0), cy = (int)floor((gy - P.cellLo[1]) / 8.0),
              cz = (int)floor((gz - P.cellLo[2]) / 8.0);
    int best = -1;
    double bestR = 1e300;
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int x = cx + dx, y = cy + dy, z = cz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= P.ncell[0] || y >= P.ncell[1] || z >= P.ncell[2]) continue;
          const int c = (z * P.ncell[1] + y) * P.ncell[0] + x;
          for (int j = P.cellStart[c]; j < P.cellStart[c + 1]; j++) {
            const int ia = P.cellAtoms[j];
            const double4 a = P.xyz[ia];
            const double r = rsq_exact_c(a.x, a.y, a.z, gx, gy, gz);
            if (r < bestR || (r == bestR && ia < best)) { bestR = r; best = ia; }
          }
        }
    P.closestH[pt] = (bestR <= 64.0) ? best : -1;
  }
}

cudaError_t closest_h_launch(const ClosestHParams& P, cudaStream_t st) {
  const int64_t blocks = (P.npoints + 255) / 256;
  closest_h_kernel<<<(int)(blocks < 65535 * 16 ? blocks : 65535 * 16), 256, 0, st>>>(P);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Covalent map and floating grid
// ---------------------------------------------------------------------------
__global__ void covalent_kernel(float* out, int nx, int ny, int nz, double h, double cx, double cy, double cz,
                                double hwInv, double barrier) {
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < n; pt += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(pt % nx), iy = (int)((pt / nx) % ny), iz = (int)(pt / ((int64_t)nx * ny));
    const double dx = cx - __dmul_rn((double)(ix - nx / 2), h), dy = cy - __dmul_rn((double)(iy - ny / 2), h),
                 dz = cz - __dmul_rn((double)(iz - nz / 2), h);
    double r = __dmul_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)), hwInv);
    if (r < 1.0e-12) r = 1.0e-12;
    out[pt] = (float)(barrier * (1 - exp(-0.69314718055994529 * r)));
  }
}

cudaError_t covalent_launch(float* out, int nx, int ny, int nz, double h, const double cov[3], double hwInv,
                            double barrier, cudaStream_t st) {
  covalent_kernel<<<1184, 256, 0, st>>>(out, nx, ny, nz, h, cov[0], cov[1], cov[2], hwInv, barrier);
  return cudaGetLastError();
}

__global__ void floating_kernel(const double4* xyz, int n, int nx, int ny, int nz, double h, float* out) {
  __shared__ double4 tile[256];
  const int64_t np = (int64_t)nx * ny * nz;
  const int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool valid = pt < np;
  const int ix = (int)(pt % nx), iy = (int)((pt / nx) % ny), iz = (int)(pt / ((int64_t)nx * ny));
  const double gx = (double)(ix - nx / 2) * h, gy = (double)(iy - ny / 2) * h, gz = (double)(iz - nz / 2) * h;
  double best = 1e24;
  for (int t0 = 0; t0 < n; t0 += 256) {
    if (t0 + (int)threadIdx.x < n) tile[threadIdx.x] = xyz[t0 + threadIdx.x];
    __syncthreads();
    const int m = min(256, n - t0);
    for (int j = 0; j < m; j++) {
      const double dx = tile[j].x - gx, dy = tile[j].y - gy, dz = tile[j].z - gz;
      const double r = dx * dx + dy * dy + dz * dz;
      best = r < best ? r : best;
    }
    __syncthreads();
  }
  if (valid) out[pt] = (float)sqrt(best);
}

cudaError_t floating_launch(const double4* xyz, int n, int nx, int ny, int nz, double h, float* out,
                            cudaStream_t st) {
  const int64_t np = (int64_t)nx * ny * nz;
  floating_kernel<<<(int)((np + 255) / 256), 256, 0, st>>>(xyz, n, nx, ny, nz, h, out);
  return cudaGetLastError();
}

}  // namespace agk
