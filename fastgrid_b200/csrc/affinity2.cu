// Affinity maps for every ligand type plus the desolvation map, two grid
// points per thread (FastGrid CalculateGridmaps.cpp:84-316).
//
// The arithmetic and the exact edge decisions are those of affinity_kernel
// (affinity.cu): FP32 geometry in a CTA-local frame; the 8 A cutoff, the
// 0.01 A table bin and the sign of cos(theta) for D1 and ordered A2 atoms
// decided in FP64 exactly as the reference computes them whenever the FP32
// value lies in a guard band around the edge.  What changes is the
// organisation, for fewer instructions per point-atom pair:
//
//  * each thread holds two z-neighbouring points: one shared-memory record,
//    dx, dy and dx^2 + dy^2 of a candidate atom serve both;
//  * a CTA covers 8 x 8 x 8 points and each warp a 4 x 4 x 4 sub-box; a warp
//    walks only the candidates within 8 A of its own sub-box;
//  * candidates are gathered from a type-major cell list ((cell, type)
//    segments, file order inside each), so a batch arrives sorted by receptor
//    type without a sort, and each type's table rows are loaded once per batch
//    (one TMA bulk copy);
//  * the plain map sums add whole table rows with packed FP32x2 adds (types
//    without an H-bond term) or FMAs with a per-type 0/1 mask; the mask removes
//    the maps whose H-bond term applies to that type (the "slots", at most four
//    per pass), which read their table entry separately; a spare column of the
//    row carries the desolvation value;
//  * a point beyond 8 A of the atom reads an all-zero extra table row, so the
//    plain sums need no branch;
//  * the nearest H donor of each point (the reference's kd-tree query,
//    CalculateGridmaps.cpp:246-250) is found in the kernel from the donors
//    within 8 A of the box, exactly in FP64 with ties to the lower file index,
//    before the map sums need it.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "ag_device.cuh"
#include "ag_kernels.h"

namespace agk {

using namespace agd;

namespace {

constexpr int kT = 256;              // threads per CTA, two points each
constexpr int kW = kT / 32;
constexpr int kCap = 640;            // candidate atoms per batch
constexpr int kCellGroup = 128;      // cells per gather group (a CTA box reaches at most 4^3)
constexpr float kBias = 8388608.f;   // 2^23

struct A2Smem {
  float4 pos[kCap];                  // CTA-local x, y, z; w = info bits
  float2 vs[kCap];                   // vol, solq
  float4 rvA[kCap];                  // rvector x, y, z, rvector2 x
  float2 rvB[kCap];                  // rvector2 y, z
  int idx[kCap];                     // atom index
  unsigned short wlist[kW][kCap];    // per warp: candidates within 8 A of its sub-box
  int wStart[kW][kMaxTypes + 1];     // per warp: first wlist entry of each type
  int typeCount[kMaxTypes];
  int typeStart[kMaxTypes + 1];
  int cellPre[kCellGroup + 1];
  int cellBeg[kCellGroup];
  int cnt[kW];
  float sol[kAffRows + 1];           // + 0 at kAffRows (the out-of-cutoff entry)
  float4 mask4[kMaxMapsPass / 4];    // current type: 1 for maps summed plainly, 0 for its H-bond slot maps
  float4 rch[kT][2];                 // per thread and point: rvector of the nearest H donor
  uint64_t bar;
  // The nearest-donor search keeps each candidate's FP64 record where the map
  // sums keep vs, rvA and rvB (the two phases do not overlap).
  __device__ double4* d64() { return reinterpret_cast<double4*>(vs); }
};
static_assert(offsetof(A2Smem, vs) % 32 == 0 && offsetof(A2Smem, idx) - offsetof(A2Smem, vs) == kCap * sizeof(double4),
              "vs, rvA and rvB must hold kCap FP64 records");

__host__ __device__ constexpr size_t tabOffset() { return ((sizeof(A2Smem) + 127) / 128) * 128; }

__device__ __forceinline__ double rsq64(double ax, double ay, double az, double gx, double gy, double gz) {
  const double dx = __dsub_rn(ax, gx), dy = __dsub_rn(ay, gy), dz = __dsub_rn(az, gz);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Exact FP64 cos(theta) = -dot(unit(atom - gridPos), rvector) (CalculateGridmaps.cpp:89).
__device__ double costheta64(double ax, double ay, double az, double gx, double gy, double gz, const double* rv) {
  const double dx = __dsub_rn(ax, gx), dy = __dsub_rn(ay, gy), dz = __dsub_rn(az, gz);
  double rSq = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  if (rSq < 1.0e-24) rSq = 1.0e-24;
  const double invR = __drcp_rn(__dsqrt_rn(rSq));
  const double ux = __dmul_rn(dx, invR), uy = __dmul_rn(dy, invR), uz = __dmul_rn(dz, invR);
  return -__dadd_rn(__dadd_rn(__dmul_rn(ux, rv[0]), __dmul_rn(uy, rv[1])), __dmul_rn(uz, rv[2]));
}

__device__ __forceinline__ float acos_clamped(float f) { return (f > 1.f) ? 0.f : (f < -1.f) ? 3.14159265f : acosf(f); }

// Per-thread state: two points (p = 0, 1 at z and z + 1) and their sums.
template <int NMAX>
struct Pts {
  float px, py, pz[2];
  int ix, iy, iz0;
  bool valid[2];
  int ch[2];                         // nearest H donor, or -1 (its rvector is in shared memory)
  float2 em[2][NMAX / 2];            // plain map sums, maps (2i, 2i+1)
  float s1[2], s2[2];                // desolvation sums (sol * vol, sol * solq)
  float mn[2][kA2Slots], mx[2][kA2Slots];  // per slot: additive sum (acceptor probes) or min / max
  unsigned fl[2];                    // per slot: a min / max value was recorded
};

// FP64 grid-point coordinate as the reference forms it.
__device__ __forceinline__ double gcoord(int i, int n2, double h) { return __dmul_rn((double)(i - n2), h); }

// One receptor type's candidates in this warp's list, for both points.
// ANG: angular class of the type; ISH: the type is "HD" (disordered ones are skipped).
template <int NMAX, int ANG, bool ISH, bool PLAIN>
__device__ __forceinline__ void run_type(const Aff2Params& P, const A2Smem& S, const float* tab, const int j0,
                                         const int j1, const unsigned short* wl, const unsigned slots,
                                         Pts<NMAX>& q) {
  const int nmPad = P.nmPad;
  const float4* tab4 = reinterpret_cast<const float4*>(tab);
  const int rowQ = nmPad >> 2;       // float4 per row

  // The next candidate's record is read one iteration ahead (its shared-memory
  // latency overlaps the current candidate's arithmetic).
  int cNext = j0 < j1 ? wl[j0] : 0;
  float4 aNext = j0 < j1 ? S.pos[cNext] : make_float4(0.f, 0.f, 0.f, 0.f);
  for (int jj = j0; jj < j1; jj++) {
    const int c = cNext;
    const float4 a = aNext;
    if (jj + 1 < j1) {
      cNext = wl[jj + 1];
      aNext = S.pos[cNext];
    }
    const float dx = a.x - q.px, dy = a.y - q.py;
    const float dxy = fmaf(dy, dy, dx * dx);
    float dz[2], r2[2];
    bool in[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      dz[p] = a.z - q.pz[p];
      r2[p] = fmaf(dz[p], dz[p], dxy);
      in[p] = q.valid[p] && r2[p] <= 64.0002f;
    }
    if (!__any_sync(0xffffffffu, in[0] || in[1])) continue;
    const int info = __float_as_int(a.w);
    const bool dis = (info >> 8) & 1;
    if (ISH && dis) continue;        // the reference skips disordered hydrogens (:280); uniform: one candidate
    // Exact 8 A cutoff near the edge.
#pragma unroll
    for (int p = 0; p < 2; p++)
      if (in[p] && r2[p] > 63.9998f) {
        const double4 a64 = P.xyz[S.idx[c]];
        if (rsq64(a64.x, a64.y, a64.z, gcoord(q.ix, P.n2x, P.h), gcoord(q.iy, P.n2y, P.h),
                  gcoord(q.iz0 + p, P.n2z, P.h)) > 64.0)
          in[p] = false;
      }
    float rs[2];
    int iR[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      const float r2c = fmaxf(r2[p], 1.0e-24f);
      rs[p] = rsqrt_approx(r2c);
      const float rs100 = rs[p] * 100.f;
      const float T = r2c * rs100;
      const float kf = __fmaf_rd(r2c, rs100, kBias);   // 2^23 + floor(100 r) in the low bits
      int b = __float_as_int(kf) - 0x4B000000;
      const float fr = T - (kf - kBias);
      if (in[p] && fabsf(fr - 0.5f) > 0.5f - P.delta) {
        // Within the guard band of a bin edge: the reference's FP64 bin
        // int(100 / (1 / sqrt(r^2))) through the table of r^2 thresholds.
        const int k = min(fr > 0.5f ? b + 1 : b, kAffRows);
        const double4 a64 = P.xyz[S.idx[c]];
        const double r64 = rsq64(a64.x, a64.y, a64.z, gcoord(q.ix, P.n2x, P.h), gcoord(q.iy, P.n2y, P.h),
                                 gcoord(q.iz0 + p, P.n2z, P.h));
        b = (r64 >= P.thr[k]) ? k : k - 1;
      }
      iR[p] = in[p] ? min(max(b, 0), kAffRows - 1) : kAffRows;  // kAffRows: the zero row
    }
    // Plain map sums: whole rows.  PLAIN (no H-bond slot applies to this type)
    // adds them directly, otherwise through the type's 0/1 mask.  When the pass
    // has a spare column the row's last entry holds the desolvation value.
    float solv[2] = {0.f, 0.f};
    const int lastQ = rowQ - 1;
#pragma unroll
    for (int g4 = 0; g4 < NMAX / 4; g4++) {
      if (4 * g4 >= P.nmaps) break;
      float4 m4 = make_float4(1.f, 1.f, 1.f, 1.f);
      if (!PLAIN) m4 = S.mask4[g4];  // same address in every lane: one broadcast for both points
#pragma unroll
      for (int p = 0; p < 2; p++) {
        const float4 e4 = tab4[iR[p] * rowQ + g4];
        if (PLAIN) {
          q.em[p][2 * g4] = __fadd2_rn(q.em[p][2 * g4], make_float2(e4.x, e4.y));
          q.em[p][2 * g4 + 1] = __fadd2_rn(q.em[p][2 * g4 + 1], make_float2(e4.z, e4.w));
        } else {
          q.em[p][2 * g4] = __ffma2_rn(make_float2(e4.x, e4.y), make_float2(m4.x, m4.y), q.em[p][2 * g4]);
          q.em[p][2 * g4 + 1] = __ffma2_rn(make_float2(e4.z, e4.w), make_float2(m4.z, m4.w), q.em[p][2 * g4 + 1]);
        }
        if (g4 == lastQ) solv[p] = e4.w;
      }
    }
    const float2 v = S.vs[c];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      const float sv = P.solInRow ? solv[p] : S.sol[iR[p]];
      q.s1[p] = fmaf(sv, v.x, q.s1[p]);
      q.s2[p] = fmaf(sv, v.y, q.s2[p]);
    }
    if (PLAIN) continue;

    // Directional factors (CalculateGridmaps.cpp:84-197) and the H-bond slots (:199-232).
    float racc[2] = {1.f, 1.f}, rdon[2] = {1.f, 1.f}, hramp[2] = {1.f, 1.f};
    if (ANG != A2_SPH) {
      const int idx = S.idx[c];
      const float4 ra = S.rvA[c];
      const float2 rb = S.rvB[c];
#pragma unroll
      for (int p = 0; p < 2; p++) {
        if (!in[p]) continue;
        const float ux = dx * rs[p], uy = dy * rs[p], uz = dz[p] * rs[p];
        float cosT = -(ux * ra.x + uy * ra.y + uz * ra.z);
        bool gt0 = cosT > 0.f, ge0 = cosT >= 0.f;
        if ((ANG == A2_D1 || (ANG == A2_A2 && !dis)) && fabsf(cosT) < 1.0e-5f) {
          // The D1 and ordered-A2 factors jump where cos(theta) changes sign.
          const double4 a64 = P.xyz[idx];
          const double c64 = costheta64(a64.x, a64.y, a64.z, gcoord(q.ix, P.n2x, P.h), gcoord(q.iy, P.n2y, P.h),
                                        gcoord(q.iz0 + p, P.n2z, P.h), P.rv64 + 3 * (size_t)idx);
          cosT = (float)c64;
          gt0 = c64 > 0.0;
          ge0 = c64 >= 0.0;
        }
        if (ANG == A2_D1) {
          racc[p] = 0.f;
          if (gt0) {
            float ra2 = cosT;
            const int rexp = (info >> 9) & 7;
            if (rexp == 4) ra2 = ra2 * ra2;
            if (rexp == 4 || rexp == 2) ra2 = ra2 * ra2;
            racc[p] = ra2;
            if (idx != q.ch[p] && q.ch[p] >= 0) {
              const float4 rc = S.rch[threadIdx.x][p];
              const float cc = rc.x * ra.x + rc.y * ra.y + rc.z * ra.z;
              // cos on the SFU over [0, pi]; cos(x) = cos(2 pi - x) folds 4 theta / 3.
              const float xr = acos_clamped(cc) * (120.f / 90.f);
              hramp[p] = 0.5f - 0.5f * __cosf(fminf(xr, 6.28318531f - xr));
            }
          }
        } else if (ANG == A2_A1) {
          rdon[p] = gt0 ? cosT * cosT : 0.f;
        } else {  // A2
          if (dis) {
            // theta <= 1.24791 + pi/2  <=>  cos(theta) >= -sin(1.24791)
            racc[p] = 0.f;
            rdon[p] = 0.f;
            if (cosT >= -0.94832352f) {
              const float s = sqrtf(fmaxf(0.f, 1.f - cosT * cosT));
              const float cs = cosT * 0.31730505f + s * 0.94832352f;  // cos(theta - 1.24791)
              rdon[p] = (cs * cs) * (cs * cs);
              racc[p] = rdon[p];
            }
          } else {
            float rd = 0.f;
            if (ge0) {
              // sin(2 ti), ti = |acos(x) - pi/2| = |asin(x)|:  2 |x| sqrt(1 - x^2)
              const float cxp = uy * rb.y - uz * rb.x;
              const float cyp = uz * ra.w - ux * rb.y;
              const float czp = ux * rb.x - uy * ra.w;
              const float rd2 = fmaxf(cxp * cxp + cyp * cyp + czp * czp, 1.0e-6f);
              float x = rsqrt_approx(rd2) * (cxp * ra.x + cyp * ra.y + czp * ra.z);
              x = fminf(fabsf(x), 1.f);
              rd = 0.9f + 0.2f * x * sqrtf(fmaxf(0.f, 1.f - x * x));
            } else if (cosT >= -0.34202f) {
              const float qq = 0.116978f - cosT * cosT;
              rd = 562.25f * (qq * qq * qq);
            }
            // cos(pi/2 - acos(y)) = sqrt(1 - y^2), y = dot(u, rvector2)
            const float y = ux * ra.w + uy * rb.x + uz * rb.y;
            rdon[p] = rd * sqrtf(fmaxf(0.f, 1.f - y * y));
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kA2Slots; k++) {
      if (!((slots >> k) & 1u)) continue;   // uniform
      const int m = P.slotMap[k];
      const int kind = P.slotKind[k];
#pragma unroll
      for (int p = 0; p < 2; p++) {
        if (!in[p]) continue;
        const float E = tab[iR[p] * nmPad + m];
        const float rsph = fminf(fmaxf(E * 0.01f, 0.f), 1.f);
        if (kind == A2_SLOT_ACC) {
          const float e = dis ? (P.tableH ? __ldg(P.tableH + max(0, iR[p] - 110) * nmPad + m) : 0.f) : E;
          q.mn[p][k] += e * hramp[p] * (racc[p] + (1.f - racc[p]) * rsph);
        } else {
          const float f = (kind == A2_SLOT_A1) ? racc[p] : rdon[p];
          const float val = E * (f + (1.f - f) * rsph);
          q.mn[p][k] = fminf(q.mn[p][k], val);
          q.mx[p][k] = fmaxf(q.mx[p][k], val);
          q.fl[p] |= 1u << k;
        }
      }
    }
  }
}

}  // namespace

size_t aff2_smem_bytes(int nmPad) { return tabOffset() + sizeof(float) * (size_t)(kAffRows + 1) * nmPad; }

// The CTA's box in the grid-centred frame, the 8 A cells around it and the
// calling warp's sub-box in the CTA frame.
struct Box {
  double ox, oy, oz;                 // CTA frame origin (its first lattice point)
  double lo[3], hi[3];               // CTA box
  int c0[3], ncx, ncy, ncells;       // cells around the box
  float sblo[3], sbhi[3];            // this warp's sub-box
  bool warpEmpty;
};

// Cell ranges of receptor type t in cell group cg: S.cellBeg / S.cellPre.
// Returns the group's cell count (S.cellPre[ncg] is its atom count).
__device__ __forceinline__ int cell_prefix(const Aff2Params& P, A2Smem& S, const Box& B, const int t, const int cg) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ncg = min(kCellGroup, B.ncells - cg);
  __syncthreads();  // the previous group's ranges are no longer read
  if (warp == 0) {
    constexpr int kPer = kCellGroup / 32;
    int cnts[kPer];
    int mine = 0;
#pragma unroll
    for (int u = 0; u < kPer; u++) {
      const int i = lane * kPer + u;
      int cn = 0;
      if (i < ncg) {
        const int ci = cg + i;
        const int cx = B.c0[0] + ci % B.ncx, cy = B.c0[1] + (ci / B.ncx) % B.ncy, cz = B.c0[2] + ci / (B.ncx * B.ncy);
        const int key = ((cz * P.ncell[1] + cy) * P.ncell[0] + cx) * P.ntypes + t;
        const int beg = P.ctStart[key];
        cn = P.ctStart[key + 1] - beg;
        S.cellBeg[i] = beg;
      }
      cnts[u] = cn;
      mine += cn;
    }
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    int run = incl - mine;
#pragma unroll
    for (int u = 0; u < kPer; u++) {
      const int i = lane * kPer + u;
      if (i < ncg) S.cellPre[i] = run;
      run += cnts[u];
    }
    if (lane == 31) S.cellPre[ncg] = incl;
  }
  __syncthreads();
  return ncg;
}

// Up to kT atoms v0 .. v0 + kT of the current cell group (type t) that lie
// within 8 A of the CTA box, appended to the candidate arrays at slot nb
// (full: with the fields the map sums need).  Returns the new count.
__device__ __forceinline__ int gather_chunk(const Aff2Params& P, A2Smem& S, const Box& B, const int t, const int ncg,
                                            const int total, const int v0, const int nb, const bool full) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
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
    atom = P.ctAtoms[S.cellBeg[lo_i] + (v - S.cellPre[lo_i])];
    a = P.xyz[atom];
    const double ddx = fmax(fmax(B.lo[0] - a.x, a.x - B.hi[0]), 0.0);
    const double ddy = fmax(fmax(B.lo[1] - a.y, a.y - B.hi[1]), 0.0);
    const double ddz = fmax(fmax(B.lo[2] - a.z, a.z - B.hi[2]), 0.0);
    keep = ddx * ddx + ddy * ddy + ddz * ddz <= 64.001;
  }
  const unsigned kbal = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) S.cnt[warp] = __popc(kbal);
  __syncthreads();
  int tot = 0, off = 0;
#pragma unroll
  for (int w = 0; w < kW; w++) {
    if (w == warp) off = tot;
    tot += S.cnt[w];
  }
  if (keep) {
    const int j = nb + off + __popc(kbal & ((1u << lane) - 1u));
    const int inf = P.info[atom];
    S.pos[j] = make_float4((float)(a.x - B.ox), (float)(a.y - B.oy), (float)(a.z - B.oz), __int_as_float(inf));
    S.idx[j] = atom;
    if (full) {
      S.vs[j] = make_float2(P.vol[atom], P.solq[atom]);
      S.rvA[j] = make_float4(P.rv[3 * atom], P.rv[3 * atom + 1], P.rv[3 * atom + 2], P.rv2[3 * atom]);
      S.rvB[j] = make_float2(P.rv2[3 * atom + 1], P.rv2[3 * atom + 2]);
    } else {
      S.d64()[j] = a;
    }
  }
  if (tid == 0) S.typeCount[t] += tot;
  __syncthreads();
  return nb + tot;
}

// Nearest H donor of both points over candidates 0 .. nb (FP64 exact, ties to
// the lower file index), folded into best / bi.  A first FP32 pass finds each
// point's smallest r^2 in the batch; the FP64 distance (from the records in
// shared memory) is formed only for the candidates within 1e-3 A^2 of it,
// which the FP32 error (< 1e-4 A^2) cannot hide.
template <int NMAX>
__device__ __forceinline__ void scan_donors(const Aff2Params& P, A2Smem& S, const int nb, double (&best)[2],
                                            int (&bi)[2], const Pts<NMAX>& q) {
  __syncthreads();
  float lim[2] = {3.0e38f, 3.0e38f};
  for (int j = 0; j < nb; j++) {
    const float4 a = S.pos[j];
    const float dx = a.x - q.px, dy = a.y - q.py;
    const float dxy = fmaf(dy, dy, dx * dx);
#pragma unroll
    for (int p = 0; p < 2; p++) {
      const float dz = a.z - q.pz[p];
      lim[p] = fminf(lim[p], fmaf(dz, dz, dxy));
    }
  }
#pragma unroll
  for (int p = 0; p < 2; p++) lim[p] = fminf(lim[p], (float)best[p]) + 1.0e-3f;
  const double4* d64 = S.d64();
  for (int j = 0; j < nb; j++) {
    const float4 a = S.pos[j];
    const float dx = a.x - q.px, dy = a.y - q.py;
    const float dxy = fmaf(dy, dy, dx * dx);
#pragma unroll
    for (int p = 0; p < 2; p++) {
      const float dz = a.z - q.pz[p];
      if (q.valid[p] && fmaf(dz, dz, dxy) <= lim[p]) {
        const int id = S.idx[j];
        const double4 a64 = d64[j];
        const double r64 = rsq64(a64.x, a64.y, a64.z, gcoord(q.ix, P.n2x, P.h), gcoord(q.iy, P.n2y, P.h),
                                 gcoord(q.iz0 + p, P.n2z, P.h));
        if (r64 < best[p] || (r64 == best[p] && id < bi[p])) {
          best[p] = r64;
          bi[p] = id;
        }
      }
    }
  }
  __syncthreads();
}

// One batch of nb candidates: per-warp lists, then the types one by one.
// Returns false if a table copy's bounded wait expired (status set).
template <int NMAX>
__device__ __forceinline__ bool process_batch(const Aff2Params& P, A2Smem& S, float* tab, const Box& B, const int nb,
                                              unsigned& phase, Pts<NMAX>& q) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nmPad = P.nmPad;
  const unsigned tabBytes = (unsigned)(kAffRows * nmPad * sizeof(float));
  __syncthreads();  // candidate records and counts are complete
  if (tid == 0) {
    int s = 0;
    for (int t = 0; t < P.ntypes; t++) {
      S.typeStart[t] = s;
      s += S.typeCount[t];
      S.typeCount[t] = 0;
    }
    S.typeStart[P.ntypes] = s;
  }
  __syncthreads();
  // This warp's list: the candidates within 8 A of its sub-box (FP32 with margin).
  int nw = 0;
  if (!B.warpEmpty)
    for (int base = 0; base < nb; base += 32) {
      const int j = base + lane;
      bool keep = false;
      if (j < nb) {
        const float4 a = S.pos[j];
        const float ddx = fmaxf(fmaxf(B.sblo[0] - a.x, a.x - B.sbhi[0]), 0.f);
        const float ddy = fmaxf(fmaxf(B.sblo[1] - a.y, a.y - B.sbhi[1]), 0.f);
        const float ddz = fmaxf(fmaxf(B.sblo[2] - a.z, a.z - B.sbhi[2]), 0.f);
        keep = fmaf(ddz, ddz, fmaf(ddy, ddy, ddx * ddx)) <= 64.01f;
      }
      const unsigned b = __ballot_sync(0xffffffffu, keep);
      if (keep) S.wlist[warp][nw + __popc(b & ((1u << lane) - 1u))] = (unsigned short)j;
      nw += __popc(b);
    }
  __syncwarp();
  for (int t = lane; t <= P.ntypes; t += 32) {  // first entry of each type (the list is sorted)
    const int target = S.typeStart[t];
    int a = 0, b = nw;
    while (a < b) {
      const int mid = (a + b) >> 1;
      if ((int)S.wlist[warp][mid] < target) a = mid + 1; else b = mid;
    }
    S.wStart[warp][t] = a;
  }
  __syncwarp();
  for (int t = 0; t < P.ntypes; t++) {
    if (S.typeStart[t + 1] == S.typeStart[t]) continue;  // uniform
    if (tid == 0) {
      fence_proxy_async();
      mbar_arrive_expect_tx(&S.bar, tabBytes);
      tma_load_1d(tab, P.table + (size_t)t * kAffRows * nmPad, tabBytes, &S.bar);
    }
    if (tid < kMaxMapsPass) {  // read after the __syncthreads_or below
      const unsigned plain = P.typePlain[t];
      reinterpret_cast<float*>(S.mask4)[tid] = (plain >> tid) & 1u ? 1.f : 0.f;
    }
    const bool ok = mbar_wait_bounded(&S.bar, phase & 1u, P.status);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) mbar_wait_bounded(&S.bar, phase & 1u, P.status);  // let the copy land before leaving
      return false;
    }
    phase++;
    const int j0 = S.wStart[warp][t], j1 = S.wStart[warp][t + 1];
    const unsigned slots = P.typeSlots[t];
    const unsigned short* wl = S.wlist[warp];
    const bool ish = (t == P.hydrogen);
    if (slots == 0u) {  // uniform: no H-bond term, no angular factors
      if (ish) run_type<NMAX, A2_SPH, true, true>(P, S, tab, j0, j1, wl, slots, q);
      else run_type<NMAX, A2_SPH, false, true>(P, S, tab, j0, j1, wl, slots, q);
    } else {
      switch (P.typeAng[t]) {  // uniform
        case A2_D1:
          if (ish) run_type<NMAX, A2_D1, true, false>(P, S, tab, j0, j1, wl, slots, q);
          else run_type<NMAX, A2_D1, false, false>(P, S, tab, j0, j1, wl, slots, q);
          break;
        case A2_A1: run_type<NMAX, A2_A1, false, false>(P, S, tab, j0, j1, wl, slots, q); break;
        case A2_A2: run_type<NMAX, A2_A2, false, false>(P, S, tab, j0, j1, wl, slots, q); break;
        default:
          if (ish) run_type<NMAX, A2_SPH, true, false>(P, S, tab, j0, j1, wl, slots, q);
          else run_type<NMAX, A2_SPH, false, false>(P, S, tab, j0, j1, wl, slots, q);
          break;
      }
    }
    __syncthreads();  // the table buffer is free for the next type
  }
  return true;
}

// One work unit: the CTA block `cta` of job P.  Called once per CTA by
// affinity2_kernel and repeatedly by the persistent batch kernel.
template <int NMAX>
__device__ __forceinline__ void aff2_unit(const Aff2Params& P, const int cta, unsigned char* smem_raw) {
  A2Smem& S = *reinterpret_cast<A2Smem*>(smem_raw);
  float* tab = reinterpret_cast<float*>(smem_raw + tabOffset());
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nmPad = P.nmPad;

  // This CTA's 8 x 8 x 8 points; this warp's 4 x 4 x 4 sub-box; this thread's two points.
  const int tbx = (P.nx + 7) / 8, tby = (P.ny + 7) / 8;
  const int x0 = (cta % tbx) * 8, y0 = ((cta / tbx) % tby) * 8, z0 = (cta / (tbx * tby)) * 8;
  const int wx = x0 + (warp & 1) * 4, wy = y0 + ((warp >> 1) & 1) * 4, wz = z0 + (warp >> 2) * 4;
  Pts<NMAX> q;
  q.ix = wx + (lane & 3);
  q.iy = wy + ((lane >> 2) & 3);
  q.iz0 = wz + (lane >> 4) * 2;
  q.valid[0] = q.ix < P.nx && q.iy < P.ny && q.iz0 < P.nz;
  q.valid[1] = q.ix < P.nx && q.iy < P.ny && q.iz0 + 1 < P.nz;
  const double h = P.h;
  Box B;
  B.ox = gcoord(x0, P.n2x, h);
  B.oy = gcoord(y0, P.n2y, h);
  B.oz = gcoord(z0, P.n2z, h);
  q.px = (float)(gcoord(q.ix, P.n2x, h) - B.ox);
  q.py = (float)(gcoord(q.iy, P.n2y, h) - B.oy);
  q.pz[0] = (float)(gcoord(q.iz0, P.n2z, h) - B.oz);
  q.pz[1] = (float)(gcoord(q.iz0 + 1, P.n2z, h) - B.oz);

  // CTA box (FP64, grid-centred) and the 8 A cells around it.
  B.lo[0] = B.ox; B.hi[0] = gcoord(min(x0 + 8, P.nx) - 1, P.n2x, h);
  B.lo[1] = B.oy; B.hi[1] = gcoord(min(y0 + 8, P.ny) - 1, P.n2y, h);
  B.lo[2] = B.oz; B.hi[2] = gcoord(min(z0 + 8, P.nz) - 1, P.n2z, h);
  int c1[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    B.c0[d] = max(0, (int)floor((B.lo[d] - 8.0 - P.cellLo[d]) / 8.0));
    c1[d] = min(P.ncell[d] - 1, (int)floor((B.hi[d] + 8.0 - P.cellLo[d]) / 8.0));
  }
  B.ncx = c1[0] - B.c0[0] + 1;
  B.ncy = c1[1] - B.c0[1] + 1;
  const int ncz = c1[2] - B.c0[2] + 1;
  B.ncells = (B.ncx > 0 && B.ncy > 0 && ncz > 0) ? B.ncx * B.ncy * ncz : 0;

  // This warp's sub-box in the CTA frame (empty when it lies past the grid edge).
  B.warpEmpty = wx >= P.nx || wy >= P.ny || wz >= P.nz;
  B.sblo[0] = (float)(gcoord(wx, P.n2x, h) - B.ox); B.sbhi[0] = (float)(gcoord(min(wx + 3, P.nx - 1), P.n2x, h) - B.ox);
  B.sblo[1] = (float)(gcoord(wy, P.n2y, h) - B.oy); B.sbhi[1] = (float)(gcoord(min(wy + 3, P.ny - 1), P.n2y, h) - B.oy);
  B.sblo[2] = (float)(gcoord(wz, P.n2z, h) - B.oz); B.sbhi[2] = (float)(gcoord(min(wz + 3, P.nz - 1), P.n2z, h) - B.oz);

  for (int i = tid; i < kAffRows + 1; i += kT) S.sol[i] = i < kAffRows ? P.sol[i] : 0.f;
  for (int i = tid; i < nmPad; i += kT) tab[kAffRows * nmPad + i] = 0.f;
  for (int t = tid; t < kMaxTypes; t += kT) S.typeCount[t] = 0;
  if (tid == 0) {
    mbar_init(&S.bar, 1);
    fence_barrier_init();
  }

#pragma unroll
  for (int p = 0; p < 2; p++) {
    q.s1[p] = 0.f;
    q.s2[p] = 0.f;
    q.fl[p] = 0u;
    q.ch[p] = -1;
#pragma unroll
    for (int g = 0; g < NMAX / 2; g++) q.em[p][g] = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < kA2Slots; k++) {
      q.mn[p][k] = (P.slotKind[k] == A2_SLOT_ACC) ? 0.f : 999999.f;
      q.mx[p][k] = -999999.f;
    }
  }
  __syncthreads();

  // ---- the nearest H donor of both points, from the donors within 8 A of the box ----
  int nb = 0;
  if (P.needClosestH) {
    double best[2] = {1e300, 1e300};
    int bi[2] = {-1, -1};
    for (int t = 0; t < P.ntypes; t++) {
      if (!P.typeDonor[t]) continue;
      for (int cg = 0; cg < B.ncells; cg += kCellGroup) {
        const int ncg = cell_prefix(P, S, B, t, cg);
        const int total = S.cellPre[ncg];
        for (int v0 = 0; v0 < total; v0 += kT) {
          if (nb + min(kT, total - v0) > kCap) {  // this round keeps at most that many atoms
            scan_donors(P, S, nb, best, bi, q);
            nb = 0;
          }
          nb = gather_chunk(P, S, B, t, ncg, total, v0, nb, false);
        }
      }
    }
    scan_donors(P, S, nb, best, bi, q);
    nb = 0;
    for (int t = tid; t < kMaxTypes; t += kT) S.typeCount[t] = 0;
#pragma unroll
    for (int p = 0; p < 2; p++) {
      q.ch[p] = (best[p] <= 64.0) ? bi[p] : -1;
      S.rch[tid][p] = q.ch[p] >= 0 ? make_float4(P.rv[3 * q.ch[p]], P.rv[3 * q.ch[p] + 1], P.rv[3 * q.ch[p] + 2], 0.f)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
  }

  // ---- map sums: batches of candidates in type-major order, walked type by type ----
  unsigned phase = 0;
  for (int t = 0; t < P.ntypes; t++)
    for (int cg = 0; cg < B.ncells; cg += kCellGroup) {
      const int ncg = cell_prefix(P, S, B, t, cg);
      const int total = S.cellPre[ncg];
      for (int v0 = 0; v0 < total; v0 += kT) {
        if (nb + min(kT, total - v0) > kCap) {  // this round keeps at most that many atoms
          if (!process_batch(P, S, tab, B, nb, phase, q)) return;
          nb = 0;
        }
        nb = gather_chunk(P, S, B, t, ncg, total, v0, nb, true);
      }
    }
  if (nb > 0 && !process_batch(P, S, tab, B, nb, phase, q)) return;

  // ---- results ----
#pragma unroll
  for (int p = 0; p < 2; p++) {
    if (!q.valid[p]) continue;
    const int64_t pt = ((int64_t)(q.iz0 + p) * P.ny + q.iy) * P.nx + q.ix;
#pragma unroll
    for (int g = 0; g < NMAX; g++) {
      if (g >= P.nmaps) break;
      if (P.mapCov[g]) continue;
      float e = ((g & 1) ? q.em[p][g >> 1].y : q.em[p][g >> 1].x) +
                (P.solparProbe[g] * q.s1[p] + P.volProbe[g] * q.s2[p]);
#pragma unroll
      for (int k = 0; k < kA2Slots; k++) {
        if (k < P.nslots && P.slotMap[k] == g) {
          if (P.slotKind[k] == A2_SLOT_ACC) e += q.mn[p][k];
          else if ((q.fl[p] >> k) & 1u) e += q.mn[p][k] + q.mx[p][k];
        }
      }
      P.out[(int64_t)g * P.npoints + pt] = e;
    }
    P.dmap[pt] = P.solparQ * q.s1[p];
  }
}

template <int NMAX>
__global__ void __launch_bounds__(kT, 2) affinity2_kernel(const __grid_constant__ Aff2Params P) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  aff2_unit<NMAX>(P, P.ctaBase + blockIdx.x, smem_raw);
}

// Persistent kernel over the work units (job, CTA block) of a batch of
// receptors, taken from an atomic counter in the host's (decreasing cost) order.
template <int NMAX>
__global__ void __launch_bounds__(kT, 2)
    affinity2_batch_kernel(const Aff2Params* __restrict__ jobs, const int2* __restrict__ units, int nunits,
                           int* counter) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int s_unit;
  for (;;) {
    __syncthreads();  // the previous unit is finished by every thread
    if (threadIdx.x == 0) s_unit = atomicAdd(counter, 1);
    __syncthreads();
    const int u = s_unit;
    if (u >= nunits) return;
    const int2 w = units[u];
    aff2_unit<NMAX>(jobs[w.x], w.y, smem_raw);
  }
}

int aff2_ctas(int nx, int ny, int nz) { return ((nx + 7) / 8) * ((ny + 7) / 8) * ((nz + 7) / 8); }

cudaError_t aff2_batch_launch(const Aff2Params* jobs, const int2* units, int nunits, int* counter, int nmPadMax,
                              int nmapsMax, int grid, cudaStream_t st) {
  const size_t smem = aff2_smem_bytes(nmPadMax);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
#define AG_AFF2B(N)                                                                                               \
  do {                                                                                                            \
    e = cudaFuncSetAttribute(affinity2_batch_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    if (e != cudaSuccess) return e;                                                                               \
    affinity2_batch_kernel<N><<<grid, kT, smem, st>>>(jobs, units, nunits, counter);                              \
  } while (0)
  if (nmapsMax <= 4) AG_AFF2B(4);
  else if (nmapsMax <= 8) AG_AFF2B(8);
  else if (nmapsMax <= 12) AG_AFF2B(12);
  else AG_AFF2B(16);
#undef AG_AFF2B
  return cudaGetLastError();
}

cudaError_t aff2_launch_range(const Aff2Params& P0, int b0, int b1, cudaStream_t st) {
  const int nb = ((P0.nx + 7) / 8) * ((P0.ny + 7) / 8) * ((P0.nz + 7) / 8);
  b0 = max(0, b0);
  b1 = min(nb, b1);
  if (b1 <= b0) return cudaSuccess;
  Aff2Params P = P0;
  P.ctaBase = b0;
  const size_t smem = aff2_smem_bytes(P.nmPad);
  const int grid = b1 - b0;
  cudaError_t e;
#define AG_AFF2(N)                                                                                           \
  do {                                                                                                       \
    e = cudaFuncSetAttribute(affinity2_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    if (e != cudaSuccess) return e;                                                                          \
    affinity2_kernel<N><<<grid, kT, smem, st>>>(P);                                                          \
  } while (0)
  if (P.nmaps <= 4) AG_AFF2(4);
  else if (P.nmaps <= 8) AG_AFF2(8);
  else if (P.nmaps <= 12) AG_AFF2(12);
  else AG_AFF2(16);
#undef AG_AFF2
  return cudaGetLastError();
}

cudaError_t aff2_launch(const Aff2Params& P, cudaStream_t st) { return aff2_launch_range(P, 0, 1 << 30, st); }

}  // namespace agk
