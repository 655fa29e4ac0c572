// Affinity maps for every ligand type plus the desolvation map, in one fused
// pass over a device-built cell list (FastGrid CalculateGridmaps.cpp:84-316).
//
// For each grid point and each receptor atom within 8 A (:263-303):
//   r, unit vector, bin = int(100 r)
//   directional H-bond factors racc / rdon / Hramp            (:84-197)
//   per map: E = table[type][bin][map] with the H-bond weighting or the
//            min/max bookkeeping                              (:199-232)
//   desolvation                                               (:234-235, :302)
// then per map the H-bond min + max are added                 (:307-313).
//
// Arithmetic.  Geometry is FP32 in a CTA-local frame (atoms and points within
// ~12 A of the frame origin, so coordinates keep ~1e-6 A).  The three places
// where the reference's FP64 result is a step function of the geometry are
// decided exactly: the 8 A cutoff, the 0.01 A table bin and the sign of
// cos(theta) for D1 and ordered A2 atoms.  When the FP32 value lies within a
// guard band of such an edge, that decision is recomputed in FP64 exactly as
// the reference computes it (same operations, no fused multiply-adds; the bin
// through a table of r^2 thresholds).  Everything else is continuous in the
// geometry and stays FP32.
//
// The desolvation terms are linear in two per-point sums,
//   S1 = sum sol(r) vol_a,  S2 = sum sol(r) (solpar_a + solparQ |q_a|),
// so map m receives solparProbe_m S1 + volProbe_m S2 and the d-map solparQ S1.
//
// Schedule.  One CTA per 8x8x4 block of points, one point per thread.  The CTA
// lists the 8 A cells around its box, prefix-sums their atom counts, and
// gathers the atoms within 8 A of the box 256 at a time into a shared-memory
// batch (up to kCap).  A batch is ordered by receptor type and walked one type
// at a time with that type's FP32 table rows (801 x nmPad) in shared memory,
// fetched by TMA bulk copies into two buffers so the next type's rows load
// while the current type is processed.  Branches on the atom's H-bond class
// and the map's H-bond mode are uniform across the CTA.
#include <cuda_runtime.h>

#include <cstdint>

#include "ag_device.cuh"
#include "ag_kernels.h"

namespace agk {

using namespace agd;

constexpr int kAffThreads = kAffTX * kAffTY * kAffTZ;  // 256
constexpr int kCap = 512;                              // candidate atoms per batch
constexpr int kMaxCells = 128;                         // cells per gather group
enum { NON = 0, DS = 1, D1 = 2, AS = 3, A1 = 4, A2 = 5 };
#define AG_PI 3.14159265358979323846

struct CandF {          // FP32 view, CTA-local coordinates
  float x, y, z;
  int idx;
  float vol, solq;
  int info;
  float pad;
  float rv[3], rv2[3];  // unit vectors
};

struct AffSmem {
  CandF cand[kCap];
  short perm[kCap];
  int typeStart[kMaxTypes + 1];
  int run[kMaxTypes + 1];
  int cnt[kAffThreads / 32];
  int cellBeg[kMaxCells];
  int cellPre[kMaxCells + 1];
  float sol[kAffRows + 3];
  uint64_t bar[2];
};

size_t aff_smem_bytes(int nmPad) {
  return ((sizeof(AffSmem) + 127) / 128) * 128 + 2 * sizeof(float) * (size_t)kAffRows * nmPad;
}

__device__ __forceinline__ float acosf_c(float f) { return (f > 1.f) ? 0.f : (f < -1.f) ? 3.14159265f : acosf(f); }

// Exact FP64 squared distance as the reference forms it (Vec3d::MagnitudeSqr
// of atom - gridPos, left to right, separately rounded).
__device__ __forceinline__ double rsq_exact(double ax, double ay, double az, double gx, double gy, double gz) {
  const double dx = __dsub_rn(ax, gx), dy = __dsub_rn(ay, gy), dz = __dsub_rn(az, gz);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Exact FP64 cos(theta) = -dot(unit(atom - gridPos), rvector) (CalculateGridmaps.cpp:89).
__device__ double costheta_exact(double ax, double ay, double az, double gx, double gy, double gz, const double* rv) {
  const double dx = __dsub_rn(ax, gx), dy = __dsub_rn(ay, gy), dz = __dsub_rn(az, gz);
  double rSq = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  if (rSq < 1.0e-24) rSq = 1.0e-24;
  const double invR = __drcp_rn(__dsqrt_rn(rSq));
  const double ux = __dmul_rn(dx, invR), uy = __dmul_rn(dy, invR), uz = __dmul_rn(dz, invR);
  return -__dadd_rn(__dadd_rn(__dmul_rn(ux, rv[0]), __dmul_rn(uy, rv[1])), __dmul_rn(uz, rv[2]));
}

// One work unit: the CTA block `cta` of job P.  Called once per CTA by
// affinity_kernel and repeatedly by the persistent batch kernel.
template <int NMAX>
__device__ __forceinline__ void aff_unit(const AffParams& P, const int cta, unsigned char* smem_raw) {
  AffSmem& S = *reinterpret_cast<AffSmem*>(smem_raw);
  float* tabBuf = reinterpret_cast<float*>(smem_raw + ((sizeof(AffSmem) + 127) / 128) * 128);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nmPad = P.nmPad;
  const unsigned tabBytes = (unsigned)(kAffRows * nmPad * sizeof(float));
  const float kBias = 8388608.f;  // 2^23: adding it with round-down leaves floor() in the low bits

  // This CTA's block of points and this thread's point.
  const int tbx = (P.nx + kAffTX - 1) / kAffTX, tby = (P.ny + kAffTY - 1) / kAffTY;
  const int bx = cta % tbx, by = (cta / tbx) % tby, bz = cta / (tbx * tby);
  const int x0 = bx * kAffTX, y0 = by * kAffTY, z0 = bz * kAffTZ;
  const int ix = x0 + (tid % kAffTX), iy = y0 + (tid / kAffTX) % kAffTY, iz = z0 + tid / (kAffTX * kAffTY);
  const bool valid = ix < P.nx && iy < P.ny && iz < P.nz;
  const double h = P.h;
  // FP64 point as the reference forms it, and FP32 point in the CTA frame
  // (origin on the lattice point (x0, y0, z0): local coordinates are exact).
  const double gx = __dmul_rn((double)(ix - P.n2x), h), gy = __dmul_rn((double)(iy - P.n2y), h),
               gz = __dmul_rn((double)(iz - P.n2z), h);
  const double ox = __dmul_rn((double)(x0 - P.n2x), h), oy = __dmul_rn((double)(y0 - P.n2y), h),
               oz = __dmul_rn((double)(z0 - P.n2z), h);
  const float px = (float)(gx - ox), py = (float)(gy - oy), pz = (float)(gz - oz);
  const int64_t pt = ((int64_t)iz * P.ny + iy) * P.nx + ix;

  double lo[3], hi[3];
  lo[0] = ox; hi[0] = (double)(min(x0 + kAffTX, P.nx) - 1 - P.n2x) * h;
  lo[1] = oy; hi[1] = (double)(min(y0 + kAffTY, P.ny) - 1 - P.n2y) * h;
  lo[2] = oz; hi[2] = (double)(min(z0 + kAffTZ, P.nz) - 1 - P.n2z) * h;
  int c0[3], c1[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    c0[d] = max(0, (int)floor((lo[d] - 8.0 - P.cellLo[d]) / 8.0));
    c1[d] = min(P.ncell[d] - 1, (int)floor((hi[d] + 8.0 - P.cellLo[d]) / 8.0));
  }

  for (int i = tid; i < kAffRows; i += kAffThreads) S.sol[i] = P.sol[i];
  if (tid == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
    fence_barrier_init();
  }

  const int ch = valid ? P.closestH[pt] : -1;
  float rcx = 0.f, rcy = 0.f, rcz = 0.f;
  if (ch >= 0) { rcx = P.rv[3 * ch]; rcy = P.rv[3 * ch + 1]; rcz = P.rv[3 * ch + 2]; }

  // Map sums in pairs (maps 2i, 2i+1): the table row's float4 halves add with
  // one packed FP32x2 instruction each (add.f32x2, rounded as two scalar adds).
  float2 em[NMAX / 2];
  float mn[kMaxMinMax], mx[kMaxMinMax];
#pragma unroll
  for (int g = 0; g < NMAX / 2; g++) em[g] = make_float2(0.f, 0.f);
#pragma unroll
  for (int s = 0; s < kMaxMinMax; s++) { mn[s] = 999999.f; mx[s] = -999999.f; }
  unsigned mmFlag = 0;
  float S1 = 0.f, S2 = 0.f;
  unsigned phaseBits = 0u;   // phase of the two table buffers' barriers (bit b = buffer b)
  bool aborted = false;
  int nb = 0;                // candidates in the current batch

  // ---- one batch: order by receptor type, walk the types ----
  auto processBatch = [&]() {
    if (warp == 0) {  // stable counting sort by type, one warp
      for (int t = lane; t <= kMaxTypes; t += 32) S.run[t] = 0;
      __syncwarp();
      for (int base = 0; base < nb; base += 32) {
        const int j = base + lane;
        const int key = j < nb ? (S.cand[j].info & 31) : 64 + lane;
        const unsigned grp = __match_any_sync(0xffffffffu, key);
        if (j < nb && lane == __ffs(grp) - 1) S.run[key] += __popc(grp);
        __syncwarp();
      }
      if (lane == 0) {
        int s = 0;
        for (int t = 0; t < P.ntypes; t++) {
          S.typeStart[t] = s;
          s += S.run[t];
          S.run[t] = S.typeStart[t];
        }
        S.typeStart[P.ntypes] = s;
      }
      __syncwarp();
      for (int base = 0; base < nb; base += 32) {
        const int j = base + lane;
        const int key = j < nb ? (S.cand[j].info & 31) : 64 + lane;
        const unsigned grp = __match_any_sync(0xffffffffu, key);
        if (j < nb) S.perm[S.run[key] + __popc(grp & ((1u << lane) - 1u))] = (short)j;
        __syncwarp();
        if (j < nb && lane == __ffs(grp) - 1) S.run[key] += __popc(grp);
        __syncwarp();
      }
    }
    __syncthreads();

    int slot = 0;
    int t = 0;
    while (t < P.ntypes && S.typeStart[t + 1] == S.typeStart[t]) t++;
    if (t < P.ntypes && tid == 0) {
      fence_proxy_async();
      mbar_arrive_expect_tx(&S.bar[0], tabBytes);
      tma_load_1d(tabBuf, P.table + (size_t)t * kAffRows * nmPad, tabBytes, &S.bar[0]);
    }
    while (t < P.ntypes) {
      int tn = t + 1;
      while (tn < P.ntypes && S.typeStart[tn + 1] == S.typeStart[tn]) tn++;
      if (tn < P.ntypes && tid == 0) {
        fence_proxy_async();
        mbar_arrive_expect_tx(&S.bar[slot ^ 1], tabBytes);
        tma_load_1d(tabBuf + (size_t)(slot ^ 1) * kAffRows * nmPad, P.table + (size_t)tn * kAffRows * nmPad, tabBytes,
                    &S.bar[slot ^ 1]);
      }
      const bool ok = mbar_wait_bounded(&S.bar[slot], (phaseBits >> slot) & 1u, P.status);
      phaseBits ^= 1u << slot;
      if (__syncthreads_or(!ok)) {
        if (tid == 0 && tn < P.ntypes) mbar_wait_bounded(&S.bar[slot ^ 1], (phaseBits >> (slot ^ 1)) & 1u, P.status);
        aborted = true;
        return;
      }
      const float* tab = tabBuf + (size_t)slot * kAffRows * nmPad;
      const int hb = P.typeHbond[t];
      const bool skipDisH = (t == P.hydrogen);
      const unsigned modes = P.typeModes[t];  // 2 bits per map
      const bool needAng = P.typeNeedsAngular[t];

      if (valid) {
        for (int jj = S.typeStart[t]; jj < S.typeStart[t + 1]; jj++) {
          const int j = S.perm[jj];
          const CandF& a = S.cand[j];
          const float dx = a.x - px, dy = a.y - py, dz = a.z - pz;
          float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
          if (r2 > 64.0002f) continue;
          const int dis = (a.info >> 8) & 1;
          if (skipDisH && dis) continue;
          double rSq64 = -1.0;
          if (r2 > 63.9998f) {
            const double4 a64 = P.xyz[a.idx];
            rSq64 = rsq_exact(a64.x, a64.y, a64.z, gx, gy, gz);
            if (rSq64 > 64.0) continue;
          }
          r2 = fmaxf(r2, 1.0e-24f);
          const float rs = rsqrt_approx(r2);
          const float rs100 = rs * 100.f;
          const float T = r2 * rs100;
          int iR = __float_as_int(__fmaf_rd(r2, rs100, kBias)) - 0x4B000000;
          iR = min(iR, kAffRows - 1);
          const float kb = T + 12582912.f;  // 1.5 * 2^23: nearest integer in the low bits
          const float kr = kb - 12582912.f;
          if (fabsf(T - kr) < P.delta && kr >= 1.f && kr <= (float)(kAffRows - 1)) {
            if (rSq64 < 0.0) {
              const double4 a64 = P.xyz[a.idx];
              rSq64 = rsq_exact(a64.x, a64.y, a64.z, gx, gy, gz);
            }
            const int k = __float_as_int(kb) - 0x4B400000;
            iR = (rSq64 >= P.thr[k]) ? k : k - 1;
          }
          const float ux = dx * rs, uy = dy * rs, uz = dz * rs;

          // Directional factors (CalculateGridmaps.cpp:84-197).
          float racc = 1.f, rdon = 1.f, Hramp = 1.f;
          if (needAng) {
            float cosT = -(ux * a.rv[0] + uy * a.rv[1] + uz * a.rv[2]);
            bool gt0 = cosT > 0.f, ge0 = cosT >= 0.f;
            if ((hb == D1 || (hb == A2 && !dis)) && fabsf(cosT) < 1.0e-5f) {
              // The D1 and ordered-A2 factors jump where cos(theta) changes sign:
              // take the sign from the reference's FP64 expression.
              const double4 a64 = P.xyz[a.idx];
              const double c64 = costheta_exact(a64.x, a64.y, a64.z, gx, gy, gz, P.rv64 + 3 * a.idx);
              cosT = (float)c64;
              gt0 = c64 > 0.0;
              ge0 = c64 >= 0.0;
            }
            if (hb == D1) {
              racc = 0.f;
              if (gt0) {
                float ra = cosT;
                const int rexp = (a.info >> 9) & 7;
                if (rexp == 4) ra = ra * ra;
                if (rexp == 4 || rexp == 2) ra = ra * ra;
                racc = ra;
                if (a.idx != ch && ch >= 0) {
                  const float c = rcx * a.rv[0] + rcy * a.rv[1] + rcz * a.rv[2];
                  // cos on the SFU (absolute error ~4e-7 on [0, pi]); cos(x) = cos(2 pi - x)
                  // folds 4 theta / 3 in [0, 4 pi / 3] into [0, pi].
                  const float xr = acosf_c(c) * (120.f / 90.f);
                  Hramp = 0.5f - 0.5f * __cosf(fminf(xr, 6.28318531f - xr));
                }
              }
            } else if (hb == A1) {
              rdon = gt0 ? cosT * cosT : 0.f;
            } else if (hb == A2) {
              if (dis) {
                // theta <= 1.24791 + pi/2  <=>  cos(theta) >= -sin(1.24791)
                racc = 0.f;
                rdon = 0.f;
                if (cosT >= -0.94832352f) {
                  const float s = sqrtf(fmaxf(0.f, 1.f - cosT * cosT));
                  const float c = cosT * 0.31730505f + s * 0.94832352f;  // cos(theta - 1.24791)
                  rdon = (c * c) * (c * c);
                  racc = rdon;
                }
              } else {
                float rd = 0.f;
                if (ge0) {
                  // sin(2 ti) with ti = |acos(x) - pi/2| = |asin(x)|:  2 |x| sqrt(1 - x^2)
                  const float cxp = uy * a.rv2[2] - uz * a.rv2[1];
                  const float cyp = uz * a.rv2[0] - ux * a.rv2[2];
                  const float czp = ux * a.rv2[1] - uy * a.rv2[0];
                  const float rd2 = fmaxf(cxp * cxp + cyp * cyp + czp * czp, 1.0e-6f);
                  float x = rsqrt_approx(rd2) * (cxp * a.rv[0] + cyp * a.rv[1] + czp * a.rv[2]);
                  x = fminf(fabsf(x), 1.f);
                  rd = 0.9f + 0.2f * x * sqrtf(fmaxf(0.f, 1.f - x * x));
                } else if (cosT >= -0.34202f) {
                  const float q = 0.116978f - cosT * cosT;
                  rd = 562.25f * (q * q * q);
                }
                // cos(pi/2 - acos(y)) = sqrt(1 - y^2), y = dot(u, rvector2)
                const float y = ux * a.rv2[0] + uy * a.rv2[1] + uz * a.rv2[2];
                rdon = rd * sqrtf(fmaxf(0.f, 1.f - y * y));
              }
            }
          }

          const float sv = S.sol[iR];
          S1 = fmaf(sv, a.vol, S1);
          S2 = fmaf(sv, a.solq, S2);
          const float4* row4 = reinterpret_cast<const float4*>(tab + iR * nmPad);
          if (modes == 0u) {  // no H-bond terms for this receptor type (uniform): plain sums
#pragma unroll
            for (int g4 = 0; g4 < NMAX / 4; g4++) {
              if (4 * g4 >= P.nmaps) break;
              const float4 q = row4[g4];
              em[2 * g4] = __fadd2_rn(em[2 * g4], make_float2(q.x, q.y));
              em[2 * g4 + 1] = __fadd2_rn(em[2 * g4 + 1], make_float2(q.z, q.w));
            }
            continue;
          }
          float4 q4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
          for (int g = 0; g < NMAX; g++) {
            if (g >= P.nmaps) break;
            if ((g & 3) == 0) q4 = row4[g >> 2];
            const float pwi = (g & 3) == 0 ? q4.x : (g & 3) == 1 ? q4.y : (g & 3) == 2 ? q4.z : q4.w;
            const unsigned mode = (modes >> (2 * g)) & 3u;
            float& emg = (g & 1) ? em[g >> 1].y : em[g >> 1].x;
            if (mode == 0u) {
              emg += pwi;
            } else {
              const float rsph = fminf(fmaxf(pwi * 0.01f, 0.f), 1.f);
              if (mode == 1u) {
                const float e = dis ? (P.tableH ? P.tableH[max(0, iR - 110) * nmPad + g] : 0.f) : pwi;
                emg += e * Hramp * (racc + (1.f - racc) * rsph);
              } else {
                const float f = (mode == 2u) ? racc : rdon;
                const float v = pwi * (f + (1.f - f) * rsph);
                const int mslot = P.mapMinMaxSlot[g];
                switch (mslot) {  // uniform across the CTA
                  case 0: mn[0] = fminf(mn[0], v); mx[0] = fmaxf(mx[0], v); break;
                  case 1: mn[1] = fminf(mn[1], v); mx[1] = fmaxf(mx[1], v); break;
                  case 2: mn[2] = fminf(mn[2], v); mx[2] = fmaxf(mx[2], v); break;
                  default: mn[3] = fminf(mn[3], v); mx[3] = fmaxf(mx[3], v); break;
                }
                mmFlag |= 1u << mslot;
              }
            }
          }
        }
      }
      __syncthreads();  // this buffer is free for the type after next
      slot ^= 1;
      t = tn;
    }
    nb = 0;
  };

  // ---- gather: cells around the box, 256 atoms per step ----
  const int ncx = c1[0] - c0[0] + 1, ncy = c1[1] - c0[1] + 1, ncz = c1[2] - c0[2] + 1;
  const int ncells = (ncx > 0 && ncy > 0 && ncz > 0) ? ncx * ncy * ncz : 0;
  for (int cg = 0; cg < ncells; cg += kMaxCells) {
    const int ncg = min(kMaxCells, ncells - cg);
    __syncthreads();  // the previous group's cell ranges are no longer read
    if (warp == 0) {
      constexpr int kPer = kMaxCells / 32;
      int cnts[kPer];
      int mine = 0;
#pragma unroll
      for (int q = 0; q < kPer; q++) {
        const int i = lane * kPer + q;
        int c = 0;
        if (i < ncg) {
          const int ci = cg + i;
          const int cx = c0[0] + ci % ncx, cy = c0[1] + (ci / ncx) % ncy, cz = c0[2] + ci / (ncx * ncy);
          const int cell = (cz * P.ncell[1] + cy) * P.ncell[0] + cx;
          const int beg = P.cellStart[cell];
          c = P.cellStart[cell + 1] - beg;
          S.cellBeg[i] = beg;
        }
        cnts[q] = c;
        mine += c;
      }
      int incl = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      int run = incl - mine;
#pragma unroll
      for (int q = 0; q < kPer; q++) {
        const int i = lane * kPer + q;
        if (i < ncg) S.cellPre[i] = run;
        run += cnts[q];
      }
      if (lane == 31) S.cellPre[ncg] = incl;
    }
    __syncthreads();
    const int total = S.cellPre[ncg];
    for (int v0 = 0; v0 < total; v0 += kAffThreads) {
      if (nb + kAffThreads > kCap) {
        processBatch();
        if (aborted) return;
      }
      const int v = v0 + tid;
      bool keep = false;
      int atom = -1;
      double4 a = make_double4(0, 0, 0, 0);
      if (v < total) {
        int lo_i = 0, hi_i = ncg - 1;  // last cell with cellPre <= v
        while (lo_i < hi_i) {
          const int mid = (lo_i + hi_i + 1) >> 1;
          if (S.cellPre[mid] <= v) lo_i = mid; else hi_i = mid - 1;
        }
        atom = P.cellAtoms[S.cellBeg[lo_i] + (v - S.cellPre[lo_i])];
        a = P.xyz[atom];
        const double ddx = fmax(fmax(lo[0] - a.x, a.x - hi[0]), 0.0);
        const double ddy = fmax(fmax(lo[1] - a.y, a.y - hi[1]), 0.0);
        const double ddz = fmax(fmax(lo[2] - a.z, a.z - hi[2]), 0.0);
        keep = ddx * ddx + ddy * ddy + ddz * ddz <= 64.001;
      }
      const unsigned kbal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) S.cnt[warp] = __popc(kbal);
      __syncthreads();
      int tot = 0, off = 0;
#pragma unroll
      for (int w = 0; w < kAffThreads / 32; w++) {
        if (w == warp) off = tot;
        tot += S.cnt[w];
      }
      if (keep) {
        const int j = nb + off + __popc(kbal & ((1u << lane) - 1u));
        CandF& c = S.cand[j];
        c.x = (float)(a.x - ox); c.y = (float)(a.y - oy); c.z = (float)(a.z - oz);
        c.idx = atom;
        c.vol = P.vol[atom];
        c.solq = P.solq[atom];
        c.info = P.info[atom];
        c.rv[0] = P.rv[3 * atom]; c.rv[1] = P.rv[3 * atom + 1]; c.rv[2] = P.rv[3 * atom + 2];
        c.rv2[0] = P.rv2[3 * atom]; c.rv2[1] = P.rv2[3 * atom + 1]; c.rv2[2] = P.rv2[3 * atom + 2];
      }
      nb += tot;
      __syncthreads();
    }
  }
  if (nb > 0) {
    processBatch();
    if (aborted) return;
  }

  if (!valid) return;
#pragma unroll
  for (int g = 0; g < NMAX; g++) {
    if (g >= P.nmaps) break;
    if (P.mapCov[g]) continue;
    float e = ((g & 1) ? em[g >> 1].y : em[g >> 1].x) + (P.solparProbe[g] * S1 + P.volProbe[g] * S2);
    const int mslot = P.mapMinMaxSlot[g];
#pragma unroll
    for (int s = 0; s < kMaxMinMax; s++)
      if (s == mslot && (mmFlag & (1u << s))) e += mn[s] + mx[s];
    P.out[(int64_t)g * P.npoints + pt] = e;
  }
  P.dmap[pt] = P.solparQ * S1;
}

template <int NMAX>
__global__ void __launch_bounds__(kAffThreads, 2) affinity_kernel(const __grid_constant__ AffParams P) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  aff_unit<NMAX>(P, blockIdx.x, smem_raw);
}

// Persistent kernel over the work units (job, CTA block) of a batch of
// receptors, taken from an atomic counter in the host's (decreasing cost) order.
template <int NMAX>
__global__ void __launch_bounds__(kAffThreads, 2)
    affinity_batch_kernel(const AffParams* __restrict__ jobs, const int2* __restrict__ units, int nunits,
                          int* counter) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int s_unit;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_unit = atomicAdd(counter, 1);
    __syncthreads();
    const int u = s_unit;
    if (u >= nunits) return;
    const int2 w = units[u];
    aff_unit<NMAX>(jobs[w.x], w.y, smem_raw);
  }
}

cudaError_t aff_batch_launch(const AffParams* jobs, const int2* units, int nunits, int* counter, int nmPadMax,
                             int nmapsMax, int grid, cudaStream_t st) {
  const size_t smem = aff_smem_bytes(nmPadMax);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
#define AG_AFFB(N)                                                                                               \
  do {                                                                                                           \
    e = cudaFuncSetAttribute(affinity_batch_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    if (e != cudaSuccess) return e;                                                                              \
    affinity_batch_kernel<N><<<grid, kAffThreads, smem, st>>>(jobs, units, nunits, counter);                     \
  } while (0)
  if (nmapsMax <= 4) AG_AFFB(4);
  else if (nmapsMax <= 8) AG_AFFB(8);
  else if (nmapsMax <= 12) AG_AFFB(12);
  else AG_AFFB(16);
#undef AG_AFFB
  return cudaGetLastError();
}

cudaError_t aff_launch(const AffParams& P, cudaStream_t st) {
  const size_t smem = aff_smem_bytes(P.nmPad);
  const int tbx = (P.nx + kAffTX - 1) / kAffTX, tby = (P.ny + kAffTY - 1) / kAffTY,
            tbz = (P.nz + kAffTZ - 1) / kAffTZ;
  const int grid = tbx * tby * tbz;
  cudaError_t e;
#define AG_AFF(N)                                                                                           \
  do {                                                                                                      \
    e = cudaFuncSetAttribute(affinity_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    if (e != cudaSuccess) return e;                                                                         \
    affinity_kernel<N><<<grid, kAffThreads, smem, st>>>(P);                                                 \
  } while (0)
  if (P.nmaps <= 4) AG_AFF(4);
  else if (P.nmaps <= 8) AG_AFF(8);
  else if (P.nmaps <= 12) AG_AFF(12);
  else AG_AFF(16);
#undef AG_AFF
  return cudaGetLastError();
}

}  // namespace agk
