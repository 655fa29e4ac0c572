// Near field of the e-map surrogate: at every grid point, the exact binned
// sum over the atoms within rcut (the direct kernel's near-path arithmetic:
// 1/r capped at 2, the bin decided exactly in FP64 near a bin edge) minus the
// smooth kernel psi(r) for those atoms:
//
//   near(p) = sum_{r < rcut} w (min(1/r, 2) invEps[bin(r)] - psi(r)).
//
// The atoms arrive sorted along a Morton curve, so a 256-atom tile is a
// compact blob; each CTA first lists the tiles whose bounding box lies within
// rcut of its box and streams only those through shared memory (1-D TMA bulk
// copies, two-slot ring, bounded mbarrier waits).  The atoms of those tiles
// within rcut of the CTA box are gathered into one near batch (FP32 local
// coordinates plus the FP64 record for exact bin decisions), which the CTA
// then sums behind a single barrier; each warp skips the atoms farther than
// rcut from its own 32 work items' box.  Terms are summed in plain FP32 over
// chunks of 16 atoms, the chunk sums Kahan-compensated.
#include <cuda_runtime.h>

#include <cstdint>

#include "ag_device.cuh"
#include "ag_kernels.h"

namespace agk {

using namespace agd;

namespace {

constexpr int kThreads = 256;
constexpr int kTile = 256;
constexpr int kTabLen = 8192;
constexpr int kListCap = 1024;    // tiles listed per round (262,144 atoms)
constexpr int kNearCap = 1024;    // near batch capacity (atoms)
constexpr int kChunk = 16;        // atoms per plain-FP32 chunk sum

struct NearSmem {
  float tab[kTabLen];
  double4 ring[2][kTile];
  float4 nearA[kNearCap];         // CTA-local x, y, z scaled by 100 and 100 w
  double4 nearD[kNearCap];        // the FP64 record, for exact bin decisions
  int cnt[kThreads / 32];
  int tileList[kListCap];
  uint64_t bar[2];
};

// This thread's slot among the threads with `flag` set, in thread order;
// `total` receives their count.  Contains two block-wide barriers.
__device__ __forceinline__ int block_compact(bool flag, int* cnt, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, flag);
  if (lane == 0) cnt[warp] = __popc(b);
  __syncthreads();
  int off = 0;
  total = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; w++) {
    if (w == warp) off = total;
    total += cnt[w];
  }
  __syncthreads();
  return off + __popc(b & ((1u << lane) - 1u));
}

__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float lo_hi(const float2& v, int k) { return (k & 1) ? v.y : v.x; }

// Sum the near batch into this thread's points: for each atom within rcut of
// a point, w (min(1/r, 2) invEps[bin] - psi(r)); bins within P.delta of an
// edge are decided exactly in FP64 from the atom's FP64 record.  The point
// pairs (x0, x1), (x2, x3), ... go through Blackwell's packed FP32
// instructions (add/mul/fma .f32x2, each half rounded as the scalar one).
// gxn holds minus the thread's x coordinates in those pairs.
__device__ __forceinline__ void near_batch(const NearSmem& S, const EmapParams& P, int n,
                                           const float2 (&gxn)[kNX / 2], float gy, float gz, int xc, int iy, int iz,
                                           const float (&wlo)[3], const float (&whi)[3], float (&sum)[kNX],
                                           float (&cmp)[kNX]) {
  const float cap = 0.02f;        // min(1/r, 2) in units of 1/(100 r)
  const float kBias = 8388608.f;  // 2^23: adding it with round-down leaves floor() in the low bits
  const float2 bias2 = dup2(kBias), mone2 = dup2(-1.f), mhalf2 = dup2(-0.5f);
  const float2 np0 = dup2(-P.psi[0]), np1 = dup2(-P.psi[1]), np2 = dup2(-P.psi[2]);
  const float edge = 0.5f - P.delta;
  const float rcut2 = P.rcut2;
  const float warpCut2 = rcut2 * 1.0001f;
  const uint32_t tabBiased = smem_u32(S.tab) - 0x2C000000u;  // address(tab) - 4 * bits(2^23)
  const double h = P.h;
#pragma unroll 1
  for (int j0 = 0; j0 < n; j0 += kChunk) {
    float2 cs[kNX / 2];
#pragma unroll
    for (int k = 0; k < kNX / 2; k++) cs[k] = make_float2(0.f, 0.f);
    const int j1 = min(n, j0 + kChunk);
#pragma unroll 1
    for (int j = j0; j < j1; j++) {
      const float4 a = S.nearA[j];
      {  // skip atoms beyond rcut of every point of this warp (warp-uniform)
        const float ex = fmaxf(fmaxf(wlo[0] - a.x, a.x - whi[0]), 0.f);
        const float ey = fmaxf(fmaxf(wlo[1] - a.y, a.y - whi[1]), 0.f);
        const float ez = fmaxf(fmaxf(wlo[2] - a.z, a.z - whi[2]), 0.f);
        if (fmaf(ex, ex, fmaf(ey, ey, ez * ez)) >= warpCut2) continue;
      }
      const float dy = a.y - gy, dz = a.z - gz;
      // The 1e-30 keeps r2 > 0 (an atom on a grid point) without a per-point max.
      const float2 dyz2 = dup2(fmaf(dz, dz, dy * dy) + 1e-30f);
      const float2 ax = dup2(a.x);
      float2 rs[kNX / 2], r2[kNX / 2], npsi[kNX / 2], fr5[kNX / 2];
      uint32_t bits[kNX];
      bool any = false;
#pragma unroll
      for (int k = 0; k < kNX / 2; k++) {
        const float2 dx = __fadd2_rn(ax, gxn[k]);
        r2[k] = __ffma2_rn(dx, dx, dyz2);
        rs[k] = make_float2(rsqrt_approx(r2[k].x), rsqrt_approx(r2[k].y));
        npsi[k] = __ffma2_rn(r2[k], __ffma2_rn(r2[k], np2, np1), np0);
        float2 f = __ffma2_rd(r2[k], rs[k], bias2);
        f.x = fminf(f.x, kBias + (float)(kTabLen - 1));
        f.y = fminf(f.y, kBias + (float)(kTabLen - 1));
        bits[2 * k] = __float_as_uint(f.x);
        bits[2 * k + 1] = __float_as_uint(f.y);
        // fraction of 100 r, minus one half: within delta of a bin edge <=> |fr5| > 0.5 - delta
        fr5[k] = __fadd2_rn(__fadd2_rn(__fmul2_rn(r2[k], rs[k]), __ffma2_rn(f, mone2, bias2)), mhalf2);
        any |= ((r2[k].x < rcut2) & (fabsf(fr5[k].x) > edge)) | ((r2[k].y < rcut2) & (fabsf(fr5[k].y) > edge));
      }
      if (__any_sync(0xffffffffu, any)) {
        if (any) {
          const double4 a64 = S.nearD[j];
          const double gy64 = __dmul_rn((double)(iy - P.n2y), h), gz64 = __dmul_rn((double)(iz - P.n2z), h);
          const double ddz = __dsub_rn(a64.z, gz64), ddy = __dsub_rn(a64.y, gy64);
          const double dydz = __dadd_rn(__dmul_rn(ddy, ddy), __dmul_rn(ddz, ddz));
#pragma unroll
          for (int k = 0; k < kNX; k++) {
            const float r2k = lo_hi(r2[k >> 1], k);
            if (r2k < rcut2 && fabsf(lo_hi(fr5[k >> 1], k)) > edge) {
              // The reference's bin is kmid - 1 or kmid, kmid the integer nearest 100 r.
              const int kmid = min(__float_as_int(r2k * lo_hi(rs[k >> 1], k) + 12582912.f) - 0x4B400000, kTabLen - 1);
              const double gx64 = __dmul_rn((double)(xc * kNX + k - P.n2x), h);
              const double ddx = __dsub_rn(a64.x, gx64);
              const double r2d = __dadd_rn(__dmul_rn(ddx, ddx), dydz);
              const int b = (kmid == 0) ? 0 : ((r2d >= P.thr[kmid]) ? kmid : kmid - 1);
              bits[k] = 0x4B000000u + (uint32_t)b;
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kNX / 2; k++) {
        float2 t;
        asm("ld.shared.f32 %0, [%1];" : "=f"(t.x) : "r"(tabBiased + (bits[2 * k] << 2)));
        asm("ld.shared.f32 %0, [%1];" : "=f"(t.y) : "r"(tabBiased + (bits[2 * k + 1] << 2)));
        const float2 c = make_float2(fminf(rs[k].x, cap), fminf(rs[k].y, cap));
        const float2 wm = make_float2(r2[k].x < rcut2 ? a.w : 0.f, r2[k].y < rcut2 ? a.w : 0.f);
        cs[k] = __ffma2_rn(wm, __ffma2_rn(c, t, npsi[k]), cs[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < kNX; k++) {
      const float y = lo_hi(cs[k >> 1], k) - cmp[k];
      const float s1 = sum[k] + y;
      cmp[k] = (s1 - sum[k]) - y;
      sum[k] = s1;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 2) surr_near_kernel(const __grid_constant__ EmapParams P) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  NearSmem& S = *reinterpret_cast<NearSmem*>(smem_raw);
  const int tid = threadIdx.x;
  const int blk = blockIdx.x % P.nblocks, split = blockIdx.x / P.nblocks;
  const EmapBlock B = P.blocks[blk];
  const int a0 = split * P.chunk;
  const int a1 = min(P.n_atoms, a0 + P.chunk);
  const int tl0 = a0 / kTile, tl1 = (a1 + kTile - 1) / kTile;  // the chunk is a multiple of kTile

  // This thread's points, CTA-local and scaled by 100.
  const bool active = tid < B.nitems;
  const int v = P.items[B.item0 + (active ? tid : 0)];
  const int xc = v & 0xFF, iy = (v >> 8) & 0x7FF, iz = (v >> 19) & 0x7FF;
  const double h = P.h;
  float gx[kNX];
#pragma unroll
  for (int k = 0; k < kNX; k++) gx[k] = (float)(((double)(xc * kNX + k - P.n2x) * h - B.ox) * 100.0);
  float2 gxn[kNX / 2];
#pragma unroll
  for (int k = 0; k < kNX / 2; k++) gxn[k] = make_float2(-gx[2 * k], -gx[2 * k + 1]);
  const float gy = (float)(((double)(iy - P.n2y) * h - B.oy) * 100.0);
  const float gz = (float)(((double)(iz - P.n2z) * h - B.oz) * 100.0);
  // The box of this warp's points.
  float wlo[3] = {gx[0], gy, gz}, whi[3] = {gx[kNX - 1], gy, gz};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      wlo[d] = fminf(wlo[d], __shfl_xor_sync(0xffffffffu, wlo[d], o));
      whi[d] = fmaxf(whi[d], __shfl_xor_sync(0xffffffffu, whi[d], o));
    }

  {
    const float4* src = reinterpret_cast<const float4*>(P.table);
    float4* dst = reinterpret_cast<float4*>(S.tab);
    for (int i = tid; i < kTabLen / 4; i += kThreads) dst[i] = src[i];
  }
  if (tid == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  float sum[kNX], cmp[kNX];
#pragma unroll
  for (int k = 0; k < kNX; k++) { sum[k] = 0.f; cmp[k] = 0.f; }
  const float rc = sqrtf(P.rcut2) * 0.01f + 0.01f;  // tile test radius (A), with a margin
  const float bhx = B.hx * 0.01f, bhy = B.hy * 0.01f, bhz = B.hz * 0.01f;
  unsigned seq = 0;  // tiles consumed: ring slot seq & 1, mbarrier phase (seq >> 1) & 1
  int nBatch = 0;    // atoms in the near batch (block-uniform)

  for (int base = tl0; base < tl1; base += kListCap) {
    const int bend = min(tl1, base + kListCap);
    int ntl = 0;
    for (int k0 = base; k0 < bend; k0 += kThreads) {
      const int k = k0 + tid;
      bool rel = false;
      if (k < bend) {
        const float4 lo = P.tileLo[k], hi = P.tileHi[k];
        const float dx = fmaxf(fabsf(0.5f * (lo.x + hi.x) - (float)B.ox) - (0.5f * (hi.x - lo.x) + bhx), 0.f);
        const float dy = fmaxf(fabsf(0.5f * (lo.y + hi.y) - (float)B.oy) - (0.5f * (hi.y - lo.y) + bhy), 0.f);
        const float dz = fmaxf(fabsf(0.5f * (lo.z + hi.z) - (float)B.oz) - (0.5f * (hi.z - lo.z) + bhz), 0.f);
        rel = dx * dx + dy * dy + dz * dz < rc * rc;
      }
      int tot;
      const int pos = block_compact(rel, S.cnt, tot);
      if (rel) S.tileList[ntl + pos] = k;
      ntl += tot;
    }
    __syncthreads();
    if (tid == 0 && ntl > 0) {
      const int t0 = S.tileList[0] * kTile;
      const unsigned n0 = (unsigned)min(kTile, a1 - t0);
      fence_proxy_async();
      mbar_arrive_expect_tx(&S.bar[seq & 1], n0 * 32u);
      tma_load_1d(S.ring[seq & 1], P.atoms + t0, n0 * 32u, &S.bar[seq & 1]);
    }
    for (int t = 0; t < ntl; t++, seq++) {
      const int slot = seq & 1;
      const int t0 = S.tileList[t] * kTile;
      const int nt = min(kTile, a1 - t0);
      if (tid == 0 && t + 1 < ntl) {
        // The other slot was last read before the barriers that ended the previous tile's compaction.
        const int t1 = S.tileList[t + 1] * kTile;
        const unsigned n1 = (unsigned)min(kTile, a1 - t1);
        fence_proxy_async();
        mbar_arrive_expect_tx(&S.bar[slot ^ 1], n1 * 32u);
        tma_load_1d(S.ring[slot ^ 1], P.atoms + t1, n1 * 32u, &S.bar[slot ^ 1]);
      }
      const bool ok = mbar_wait_bounded(&S.bar[slot], (seq >> 1) & 1u, P.status);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          mbar_wait_bounded(&S.bar[slot], (seq >> 1) & 1u, P.status);
          if (t + 1 < ntl) mbar_wait_bounded(&S.bar[slot ^ 1], ((seq + 1) >> 1) & 1u, P.status);
        }
        return;
      }
      // Atoms within rcut of the CTA box join the near batch.
      bool near = false;
      float4 loc = make_float4(0.f, 0.f, 0.f, 0.f);
      double4 a64 = make_double4(0.0, 0.0, 0.0, 0.0);
      if (tid < nt) {
        a64 = S.ring[slot][tid];
        loc.x = (float)((a64.x - B.ox) * 100.0);
        loc.y = (float)((a64.y - B.oy) * 100.0);
        loc.z = (float)((a64.z - B.oz) * 100.0);
        loc.w = (float)(a64.w * 100.0);
        const float dx = fmaxf(fabsf(loc.x) - B.hx, 0.f), dy = fmaxf(fabsf(loc.y) - B.hy, 0.f),
                    dz = fmaxf(fabsf(loc.z) - B.hz, 0.f);
        near = dx * dx + dy * dy + dz * dz < P.rcut2;
      }
      int nNear;
      const int pos = block_compact(near, S.cnt, nNear);  // ends with a barrier: the ring slot is read
      if (nBatch + nNear > kNearCap) {
        near_batch(S, P, nBatch, gxn, gy, gz, xc, iy, iz, wlo, whi, sum, cmp);
        __syncthreads();
        nBatch = 0;
      }
      if (near) {
        S.nearA[nBatch + pos] = loc;
        S.nearD[nBatch + pos] = a64;
      }
      nBatch += nNear;
    }
  }
  __syncthreads();
  near_batch(S, P, nBatch, gxn, gy, gz, xc, iy, iz, wlo, whi, sum, cmp);

  if (!active) return;
  const int64_t row = ((int64_t)iz * P.ny + iy) * P.nx;
#pragma unroll
  for (int k = 0; k < kNX; k++) {
    const int x = xc * kNX + k;
    if (x >= P.nx) break;
    const double val = (double)sum[k] - (double)cmp[k];
    if (P.nsplit == 1)
      P.out[row + x] = (float)val;
    else
      P.partial[(int64_t)split * P.npoints + row + x] = val;
  }
}

__global__ void surr_near_reduce_kernel(const double* __restrict__ partial, int nsplit, int64_t n,
                                        float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nsplit; k++) s += partial[(int64_t)k * n + i];
    out[i] = (float)s;
  }
}

}  // namespace

cudaError_t emap_near_launch(const EmapParams& P, int grid, cudaStream_t st) {
  const size_t smem = sizeof(NearSmem);
  cudaError_t e =
      cudaFuncSetAttribute(surr_near_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  surr_near_kernel<<<grid, kThreads, smem, st>>>(P);
  e = cudaGetLastError();
  if (e != cudaSuccess || P.nsplit == 1) return e;
  surr_near_reduce_kernel<<<592, 256, 0, st>>>(P.partial, P.nsplit, P.npoints, P.out);
  return cudaGetLastError();
}

}  // namespace agk
