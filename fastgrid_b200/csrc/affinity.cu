// Affinity maps for every ligand type plus the desolvation map, in one fused
// pass over a device-built cell list (FastGrid CalculateGridmaps.cpp:84-316).
//
// For each grid point and each receptor atom within 8 A:
//   r, unit vector, bin int(100 r)   (exactly as the reference: FP64, IEEE
//                                     sqrt and reciprocal, no fused ops)
//   directional H-bond factors racc / rdon / Hramp (FP64; :84-197)
//   per map: E = table[type][bin][map], H-bond weighting or min/max
//            bookkeeping, desolvation                (FP32; :199-236)
//   d-map += solparQ * vol * sol[bin]                (FP32; :302)
// then per map the H-bond min + max are added (:307-313).
//
// The nearest H donor of each point (the reference's kd-tree query,
// :246-250) is found by a separate kernel over a donor-only cell list: it only
// matters for a donor atom within 8 A, so searching the cells that cover the
// 8 A sphere is exact.
//
// Schedule: one CTA per 8x8x4 block of points, one point per thread.  The CTA
// gathers the atoms of the 8 A cells around its box that lie within 8 A of
// the box into shared memory (batches of kCap), and every thread walks that
// list.  The pair-energy tables for the maps of this pass sit in shared memory
// as FP32 (rows for r <= 8 A only); maps are split into passes so that
// ntypes * 801 * G floats fit.
#include <cuda_runtime.h>

#include <cstdint>

#include "ag_device.cuh"
#include "ag_kernels.h"

namespace agk {

using namespace agd;

constexpr int kAffThreads = kAffTX * kAffTY * kAffTZ;  // 256
constexpr int kCap = 256;                              // candidate atoms per batch
enum { NON = 0, DS = 1, D1 = 2, AS = 3, A1 = 4, A2 = 5 };
#define AG_PI 3.14159265358979323846

struct Cand {
  double x, y, z;
  double rv[3], rv2[3];
  int info, idx;
  float vol, solq;
};

struct AffSmemHead {
  Cand cand[kCap];
  float sol[kAffRows + 3];
  int cnt[kAffThreads / 32];
};

size_t aff_smem_bytes(int ntypes, int G) {
  return sizeof(AffSmemHead) + sizeof(float) * (size_t)(ntypes + 1) * kAffRows * G;
}

__device__ __forceinline__ double dot3(const double* a, double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, a[0]), __dmul_rn(y, a[1])), __dmul_rn(z, a[2]));
}
__device__ __forceinline__ double acos_c(double f) { return (f > 1) ? 0.0 : (f < -1) ? AG_PI : acos(f); }

// Directional H-bond factors (CalculateGridmaps.cpp:84-197), FP64.
__device__ void hbond_angular(const Cand& a, int hb, const double* rvClosest, bool isClosest, double ux, double uy,
                              double uz, double& racc, double& rdon, double& Hramp) {
  racc = 1; rdon = 1; Hramp = 1;
  const double cosTheta = -dot3(a.rv, ux, uy, uz);
  if (hb == D1) {
    racc = 0;
    if (cosTheta > 0) {
      double ra = cosTheta;
      const int rexp = (a.info >> 9) & 7;
      if (rexp == 4) ra = ra * ra;
      if (rexp == 4 || rexp == 2) ra = ra * ra;
      racc = ra;
      if (!isClosest && rvClosest) {
        const double c = __dadd_rn(__dadd_rn(__dmul_rn(rvClosest[0], a.rv[0]), __dmul_rn(rvClosest[1], a.rv[1])),
                                   __dmul_rn(rvClosest[2], a.rv[2]));
        const double theta = acos_c(c);
        Hramp = 0.5 - 0.5 * cos(theta * (120.0 / 90.0));
      }
    }
  } else if (hb == A1) {
    rdon = 0;
    if (cosTheta > 0) rdon = cosTheta * cosTheta;
  } else if (hb == A2) {
    rdon = 0;
    if ((a.info >> 8) & 1) {
      racc = 0;
      const double theta = acos_c(cosTheta);
      if (theta <= 1.24791 + (AG_PI / 2)) {
        const double c = cos(theta - 1.24791);
        rdon = (c * c) * (c * c);
        racc = rdon;
      }
    } else {
      double rd = 0;
      if (cosTheta >= 0) {
        // cross(u, rvector2)
        const double cx = __dsub_rn(__dmul_rn(uy, a.rv2[2]), __dmul_rn(uz, a.rv2[1]));
        const double cy = __dsub_rn(__dmul_rn(uz, a.rv2[0]), __dmul_rn(ux, a.rv2[2]));
        const double cz = __dsub_rn(__dmul_rn(ux, a.rv2[1]), __dmul_rn(uy, a.rv2[0]));
        double rd2 = __dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), __dmul_rn(cz, cz));
        if (rd2 < 1.0e-6) rd2 = 1.0e-6;
        const double inv_rd = __drcp_rn(__dsqrt_rn(rd2));
        const double ti = fabs(acos_c(__dmul_rn(inv_rd, dot3(a.rv, cx, cy, cz))) - (AG_PI / 2));
        rd = 0.9 + 0.1 * sin(ti + ti);
      } else if (cosTheta >= -0.34202) {
        const double q = 0.116978 - cosTheta * cosTheta;
        rd = 562.25 * (q * q * q);
      }
      const double t0 = (AG_PI / 2) - acos_c(dot3(a.rv2, ux, uy, uz));
      rdon = rd * cos(t0);
    }
  }
}

__global__ void __launch_bounds__(kAffThreads, 2) affinity_kernel(AffParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  AffSmemHead& S = *reinterpret_cast<AffSmemHead*>(smem_raw);
  float* tab = reinterpret_cast<float*>(smem_raw + sizeof(AffSmemHead));
  float* tabH = tab + (size_t)P.ntypes * kAffRows * P.G;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  // This CTA's block of points and this thread's point.
  const int tbx = (P.nx + kAffTX - 1) / kAffTX, tby = (P.ny + kAffTY - 1) / kAffTY;
  const int bx = blockIdx.x % tbx, by = (blockIdx.x / tbx) % tby, bz = blockIdx.x / (tbx * tby);
  const int x0 = bx * kAffTX, y0 = by * kAffTY, z0 = bz * kAffTZ;
  const int ix = x0 + (tid % kAffTX), iy = y0 + (tid / kAffTX) % kAffTY, iz = z0 + tid / (kAffTX * kAffTY);
  const bool valid = ix < P.nx && iy < P.ny && iz < P.nz;
  const double h = P.h;
  const double gx = __dmul_rn((double)(ix - P.n2x), h), gy = __dmul_rn((double)(iy - P.n2y), h),
               gz = __dmul_rn((double)(iz - P.n2z), h);
  const int64_t pt = ((int64_t)iz * P.ny + iy) * P.nx + ix;

  double lo[3], hi[3];
  lo[0] = (double)(x0 - P.n2x) * h; hi[0] = (double)(min(x0 + kAffTX, P.nx) - 1 - P.n2x) * h;
  lo[1] = (double)(y0 - P.n2y) * h; hi[1] = (double)(min(y0 + kAffTY, P.ny) - 1 - P.n2y) * h;
  lo[2] = (double)(z0 - P.n2z) * h; hi[2] = (double)(min(z0 + kAffTZ, P.nz) - 1 - P.n2z) * h;
  int c0[3], c1[3];
  for (int d = 0; d < 3; d++) {
    c0[d] = max(0, (int)floor((lo[d] - 8.0 - P.cellLo[d]) / 8.0));
    c1[d] = min(P.ncell[d] - 1, (int)floor((hi[d] + 8.0 - P.cellLo[d]) / 8.0));
  }

  // Tables of this pass -> shared memory.
  {
    const int n = P.ntypes * kAffRows * P.G;
    for (int i = tid; i < n; i += kAffThreads) tab[i] = P.table[i];
    if (P.tableH)
      for (int i = tid; i < kAffRows * P.G; i += kAffThreads) tabH[i] = P.tableH[i];
    for (int i = tid; i < kAffRows; i += kAffThreads) S.sol[i] = P.sol[i];
  }

  const int ch = valid ? P.closestH[pt] : -1;
  double rvC[3] = {0, 0, 0};
  if (ch >= 0) { rvC[0] = P.rv[3 * ch]; rvC[1] = P.rv[3 * ch + 1]; rvC[2] = P.rv[3 * ch + 2]; }

  float em[kAffMaxGroup], mn[kAffMaxGroup], mx[kAffMaxGroup];
  unsigned hbFlag = 0;
#pragma unroll
  for (int g = 0; g < kAffMaxGroup; g++) { em[g] = 0.f; mn[g] = 999999.f; mx[g] = -999999.f; }
  float ed = 0.f;

  // Iterate over the cells around the box in fixed order; gather batches.
  const int ncx = c1[0] - c0[0] + 1, ncy = c1[1] - c0[1] + 1, ncz = c1[2] - c0[2] + 1;
  const int ncells = (ncx > 0 && ncy > 0 && ncz > 0) ? ncx * ncy * ncz : 0;
  int ci = 0, pos = 0;
  __syncthreads();
  while (ci < ncells) {
    int nb = 0;
    // Fill one batch.
    while (ci < ncells) {
      const int cx = c0[0] + ci % ncx, cy = c0[1] + (ci / ncx) % ncy, cz = c0[2] + ci / (ncx * ncy);
      const int cell = (cz * P.ncell[1] + cy) * P.ncell[0] + cx;
      const int cbeg = P.cellStart[cell], cend = P.cellStart[cell + 1];
      const int cnt = min(cend - (cbeg + pos), kAffThreads);
      if (cnt <= 0) { ci++; pos = 0; continue; }
      if (nb + cnt > kCap) break;
      bool keep = false;
      int atom = -1;
      if (tid < cnt) {
        atom = P.cellAtoms[cbeg + pos + tid];
        const double4 a = P.xyz[atom];
        const double ddx = fmax(fmax(lo[0] - a.x, a.x - hi[0]), 0.0);
        const double ddy = fmax(fmax(lo[1] - a.y, a.y - hi[1]), 0.0);
        const double ddz = fmax(fmax(lo[2] - a.z, a.z - hi[2]), 0.0);
        keep = ddx * ddx + ddy * ddy + ddz * ddz <= 64.000001;
      }
      const unsigned kb = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) S.cnt[warp] = __popc(kb);
      __syncthreads();
      int total = 0, off = 0;
#pragma unroll
      for (int w = 0; w < kAffThreads / 32; w++) {
        if (w == warp) off = total;
        total += S.cnt[w];
      }
      if (keep) {
        Cand& c = S.cand[nb + off + __popc(kb & ((1u << lane) - 1u))];
        const double4 a = P.xyz[atom];
        c.x = a.x; c.y = a.y; c.z = a.z;
        for (int k = 0; k < 3; k++) { c.rv[k] = P.rv[3 * atom + k]; c.rv2[k] = P.rv2[3 * atom + k]; }
        c.info = P.info[atom];
        c.idx = atom;
        c.vol = P.vol[atom];
        c.solq = P.solq[atom];
      }
      nb += total;
      pos += cnt;
      if (cbeg + pos >= cend) { ci++; pos = 0; }
      __syncthreads();
    }

    // Walk the batch.
    if (valid) {
      for (int j = 0; j < nb; j++) {
        const Cand& a = S.cand[j];
        double dx = a.x - gx, dy = a.y - gy, dz = a.z - gz;
        double rSq = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        if (rSq > 64.0) continue;
        const int t = a.info & 31, hb = (a.info >> 5) & 7, dis = (a.info >> 8) & 1;
        if (t == P.hydrogen && dis) continue;
        if (rSq < 1.0e-24) rSq = 1.0e-24;
        const double invR = __drcp_rn(__dsqrt_rn(rSq));
        dx = __dmul_rn(dx, invR); dy = __dmul_rn(dy, invR); dz = __dmul_rn(dz, invR);
        int iR = (int)__dmul_rn(__drcp_rn(invR), 100.0);
        iR = min(iR, kAffRows - 1);
        double racc, rdon, Hramp;
        hbond_angular(a, hb, ch >= 0 ? rvC : nullptr, a.idx == ch, dx, dy, dz, racc, rdon, Hramp);
        const float fracc = (float)racc, frdon = (float)rdon, fH = (float)Hramp;
        const float s = S.sol[iR];
        const float* row = tab + ((size_t)t * kAffRows + iR) * P.G;
        const bool donorAtom = (hb == DS || hb == D1);
#pragma unroll
        for (int g = 0; g < kAffMaxGroup; g++) {
          if (g >= P.G) break;
          if (P.mapCov[g]) continue;
          const float pwi = row[g];
          if (P.mapIsHB[g]) {
            const float rsph = fminf(fmaxf(pwi * 0.01f, 0.f), 1.f);
            const int mhb = P.mapHbond[g];
            if ((mhb == AS || mhb == A2) && donorAtom) {
              float e = pwi;
              if (dis) e = P.tableH ? tabH[max(0, iR - 110) * P.G + g] : 0.f;
              em[g] += e * fH * (fracc + (1.f - fracc) * rsph);
            } else if (mhb == A1 && donorAtom) {
              const float v = pwi * (fracc + (1.f - fracc) * rsph);
              mn[g] = fminf(mn[g], v); mx[g] = fmaxf(mx[g], v); hbFlag |= 1u << g;
            } else if ((mhb == DS || mhb == D1) && hb >= AS) {
              const float v = pwi * (frdon + (1.f - frdon) * rsph);
              mn[g] = fminf(mn[g], v); mx[g] = fmaxf(mx[g], v); hbFlag |= 1u << g;
            } else {
              em[g] += pwi;
            }
          } else {
            em[g] += pwi;
          }
          em[g] += s * (P.solparProbe[g] * a.vol + a.solq * P.volProbe[g]);
        }
        ed += P.solparQ * a.vol * s;
      }
    }
    __syncthreads();
  }

  if (!valid) return;
#pragma unroll
  for (int g = 0; g < kAffMaxGroup; g++) {
    if (g >= P.G) break;
    if (P.mapCov[g]) continue;
    float e = em[g];
    if (hbFlag & (1u << g)) e += mn[g] + mx[g];
    P.out[(int64_t)(P.m0 + g) * P.npoints + pt] = e;
  }
  if (P.doDmap) P.dmap[pt] = ed;
}

cudaError_t aff_launch(const AffParams& P, cudaStream_t st) {
  const size_t smem = aff_smem_bytes(P.ntypes, P.G);
  cudaError_t e = cudaFuncSetAttribute(affinity_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int tbx = (P.nx + kAffTX - 1) / kAffTX, tby = (P.ny + kAffTY - 1) / kAffTY,
            tbz = (P.nz + kAffTZ - 1) / kAffTZ;
  affinity_kernel<<<tbx * tby * tbz, kAffThreads, smem, st>>>(P);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Cell list: counting sort into 8 A cells; file order inside each cell.
// ---------------------------------------------------------------------------
__global__ void cell_count_kernel(CellBuild C) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n_atoms; i += gridDim.x * blockDim.x) {
    int cell = -1;
    if (!C.donorMask || C.donorMask[i]) {
      const double4 a = C.xyz[i];
      const int cx = (int)floor((a.x - C.lo[0]) / 8.0), cy = (int)floor((a.y - C.lo[1]) / 8.0),
                cz = (int)floor((a.z - C.lo[2]) / 8.0);
      if (cx >= 0 && cy >= 0 && cz >= 0 && cx < C.ncell[0] && cy < C.ncell[1] && cz < C.ncell[2])
        cell = (cz * C.ncell[1] + cy) * C.ncell[0] + cx;
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
  // `count` is free again: reuse it as the sort's scratch (it holds ncell+1 >= n entries only if
  // ncell+1 >= n; use cellOf, which holds n_atoms entries, instead).
  cell_sort_kernel<<<max(1, min(2048, (ncellTotal + 7) / 8)), 256, 0, st>>>(C.cellStart, ncellTotal, C.cellAtoms,
                                                                         C.cellOf);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Nearest H donor per grid point (argmin over DS/D1 atoms within the 27 cells
// around the point's cell, ties to the lower file index).
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
            const double ex = a.x - gx, ey = a.y - gy, ez = a.z - gz;
            const double r = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
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
