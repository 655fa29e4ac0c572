// Electrostatic map (e-map) by direct summation over all receptor atoms.
//
//   e(p) = sum_a w_a * min(1/r, 2) * invEps[min(int(100 r), 8191)]
//
// (FastGrid electrostatics/Cpu.cpp:27-88; the table is InputDataLoader.cpp:
// 715-742).  There is no cutoff, so the work is N_atoms x N_points pairs and
// the kernel is bound by the SM's instruction issue (one SFU rsqrt, one
// shared-memory table read and ~6 FP32/INT ops per pair), not by HBM.
//
// Layout and schedule
//  * Work item = NX consecutive x points of one (y, z) row; one thread per item,
//    256 items per CTA, items grouped by the host into compact boxes.
//  * Atoms stream through shared memory in tiles of kTile FP64 (x, y, z, w)
//    records, fetched with 1-D TMA bulk copies into a two-slot ring and
//    tracked by mbarriers (no multicast).
//  * Each tile is converted once per CTA to CTA-local coordinates scaled by
//    100 (so 100 r comes straight out of r^2 * rsqrt(r^2)) and split by the
//    atom's distance d to the CTA's box into three lists:
//      near (d < rNear): 1/r capped at 2, Kahan-compensated per pair, and the
//        bin decided exactly in FP64 (squared-distance threshold table) when
//        100 r lies within `delta` of a bin edge.  Decided again per warp:
//        a warp whose own points are all at least rNear away evaluates the
//        atom with the mid arithmetic (each term still compensated), and the
//        cap and the table clamp are dropped where they cannot apply;
//      mid (rNear <= d < rFar): bin by a round-down FMA, table read;
//      far (d >= rFar, at least 50 A): the table has saturated there (its
//        entries differ from entry 8191 by < 2e-6 relative), so the term is
//        w * invEps[8191] / r with no table read.
//    Mid atoms whose every bin lies in the table's saturating tail read a
//    packed copy of it instead: entry b is bits(g) + k_b, g = invEps[8191],
//    with k_b < 2^16 from about 22 A and < 2^8 from about 40 A.  Half- and
//    quarter-width entries put two or four neighbouring bins in one 32-bit
//    shared-memory word, so a warp's reads (its lanes' distances span ~1 A,
//    ~100 bins) touch fewer distinct words per bank: 2.0 and 1.5 wavefronts
//    per read instead of 2.6 (simulated), and those wavefronts are the
//    kernel's binding resource.  Decoding costs no instruction: k_b read as
//    float bits is the subnormal k_b 2^-149, and one packed FMA forms
//    100 w 2^-16 (g + k_b ulp(g)) = 100 w 2^-16 invEps[b] from it.
//    Mid and far terms are summed in plain FP32 over chunks of kChunk atoms
//    and the chunk sums are Kahan-compensated.
//  * When the grid is too small to fill the GPU, atoms are split across CTAs
//    and the per-CTA results are reduced in FP64, in a fixed order, by a
//    second kernel.
#include <cuda_runtime.h>

#include <cstdint>

#include "ag_device.cuh"
#include "ag_kernels.h"

namespace agk {

using namespace agd;

constexpr int kThreads = 256;
constexpr int kTile = 256;        // atoms per shared-memory tile
constexpr int kTabLen = 8192;     // invEps entries
constexpr int kChunk = 32;        // atoms per plain-FP32 chunk sum

// Atom classes of a tile, in their order in EmapSmem::list.
enum { kClsNear = 0, kClsMid = 1, kClsMid16 = 2, kClsMid8 = 3, kClsFar = 4, kNumCls = 5 };

struct EmapSmem {
  float tab[kTabLen];             // 32 KB
  double4 ring[2][kTile];         // 16 KB, TMA destination
  __align__(16) unsigned char packed[kEmapPackedBytes];
  // This tile's atoms grouped by class: local scaled x, y, z and 100*w
  // (near, mid), 100*w*g*2^-16 (packed mid) or 100*w*g (far).
  float4 list[kTile];
  short nearIdx[kTile];           // tile slot of each near atom (for FP64 lookups)
  // Near atom: bit w set if it lies within rNear of warp w's points, bit 8 + w
  // if within 0.51 A of them (the 1/r cap can apply).
  unsigned short nearMask[kTile];
  float4 wlo[kThreads / 32], whi[kThreads / 32];  // each warp's box (local, scaled), widened by 0.01 A
  int cnt[kNumCls][kThreads / 32];
  double wpart[kThreads / 32];
  int unit;                       // persistent batch kernel: the unit being processed
  uint64_t bar[2];
  uint64_t barIdle;               // never arrived on (target of the expiry test hook)
};

__device__ __forceinline__ void unpack_item(int v, int& xc, int& y, int& z) {
  xc = v & 0xFF;
  y = (v >> 8) & 0x7FF;
  z = (v >> 19) & 0x7FF;
}

// Packed FP32 pairs: Blackwell issues one instruction for two lanes of FP32
// arithmetic (add/mul/fma .f32x2), each half rounded exactly as the scalar
// operation, so the pair loops below halve their FP32 instruction count
// without changing a bit of the result.  A thread's kNX points are held as
// the pairs (x0, x1), (x2, x3), ...
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

__device__ __forceinline__ float2 rsqrt2(float2 v) { return make_float2(rsqrt_approx(v.x), rsqrt_approx(v.y)); }

__device__ __forceinline__ float lo_hi(const float2& v, int k) { return (k & 1) ? v.y : v.x; }

// One Kahan step on a pair, (x - c), (s + y), ((s1 - s) - y) each rounded once
// as in the scalar form (a * -1 + b is exact before its single rounding).
__device__ __forceinline__ void kahan2(float2& s, float2& c, float2 x) {
  const float2 m1 = dup2(-1.f);
  const float2 y = __ffma2_rn(c, m1, x);
  const float2 s1 = __fadd2_rn(s, y);
  c = __ffma2_rn(y, m1, __ffma2_rn(s, m1, s1));
  s = s1;
}

// Fold a chunk's plain FP32 sums into the running sums (Kahan), or, in plain
// mode, take them over (the chunk sums started from the running sums).
template <int MODE>
__device__ __forceinline__ void add_chunk(float2 (&sum)[kNX / 2], float2 (&cmp)[kNX / 2],
                                          const float2 (&cs)[kNX / 2]) {
#pragma unroll
  for (int k = 0; k < kNX / 2; k++) {
    if (MODE == kEmapKahan)
      kahan2(sum[k], cmp[k], cs[k]);
    else
      sum[k] = cs[k];
  }
}

// Table read at the bin encoded in the low bits of f = 2^23 + bin: the shared
// address is tabBiased + 4 * bits(f) in 32-bit shared-window arithmetic,
// where tabBiased = address(tab) - 4 * bits(2^23) (mod 2^32).
__device__ __forceinline__ float lds_bin(uint32_t tabBiased, float f) {
  const uint32_t a = tabBiased + ((uint32_t)__float_as_int(f) << 2);
  float v;
  asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}

// Mid-list atoms: bin by a round-down FMA, table read, plain FP32 chunk sums.
// CLAMP: the CTA's box is large enough that a bin can pass the table's end.
// gxn holds minus the thread's x coordinates, in pairs (x0, x1), (x2, x3), ...
template <int MODE, bool CLAMP>
__device__ __forceinline__ void mid_atoms(const float4* __restrict__ list, uint32_t tabBiased, int n,
                                          const float2 (&gxn)[kNX / 2], float gy, float gz, float2 (&sum)[kNX / 2],
                                          float2 (&cmp)[kNX / 2]) {
  const float kBias = 8388608.f;
  const float2 bias2 = dup2(kBias);
#pragma unroll 1
  for (int j0 = 0; j0 < n; j0 += kChunk) {
    float2 cs[kNX / 2];
#pragma unroll
    for (int k = 0; k < kNX / 2; k++)
      cs[k] = (MODE == kEmapKahan) ? make_float2(0.f, 0.f) : sum[k];
    const int j1 = min(n, j0 + kChunk);
    // Unrolled over atoms: the scheduler interleaves several atoms' rsqrt and
    // table-read latencies (3 CTAs x 8 warps per SM alone do not hide them).
#pragma unroll 8
    for (int j = j0; j < j1; j++) {
      const float4 a = list[j];
      const float dy = a.y - gy, dz = a.z - gz;
      const float2 dyz2 = dup2(fmaf(dz, dz, dy * dy));
      const float2 ax = dup2(a.x), aw = dup2(a.w);
#pragma unroll
      for (int k = 0; k < kNX / 2; k++) {
        const float2 dx = __fadd2_rn(ax, gxn[k]);
        const float2 r2 = __ffma2_rn(dx, dx, dyz2);
        const float2 rs = rsqrt2(r2);
        float2 f = __ffma2_rd(r2, rs, bias2);
        if (CLAMP) {
          f.x = fminf(f.x, kBias + (float)(kTabLen - 1));
          f.y = fminf(f.y, kBias + (float)(kTabLen - 1));
        }
        const float2 g = make_float2(lds_bin(tabBiased, f.x), lds_bin(tabBiased, f.y));
        cs[k] = __ffma2_rn(__fmul2_rn(aw, rs), g, cs[k]);
      }
    }
    add_chunk<MODE>(sum, cmp, cs);
  }
}

// Entry k_b of a packed tail table (W = 2: 16-bit, W = 1: 8-bit) at the bin
// encoded in f = 2^23 + bin, returned as float bits (the subnormal k_b 2^-149).
// tabBiased = address(entry 0) - W * (bits(2^23) + first bin), mod 2^32.
template <int W>
__device__ __forceinline__ float lds_packed(uint32_t tabBiased, float f) {
  uint32_t v;
  if (W == 2)
    asm("ld.shared.u16 %0, [%1];" : "=r"(v) : "r"(tabBiased + ((uint32_t)__float_as_int(f) << 1)));
  else
    asm("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(tabBiased + (uint32_t)__float_as_int(f)));
  return __uint_as_float(v);
}

// Mid atoms whose bins all lie in a packed tail table.  With a.w = 100 w g
// 2^-16 and kScale = 2^(e+126) / g (g = 2^e m), aws = a.w kScale = 100 w
// ulp(g) 2^133, so aws * k_b 2^-149 + a.w = 100 w 2^-16 (g + k_b ulp(g)):
// the term's weight times the table entry, scaled by 2^-16 (exact), in one
// FMA whose product is exact for 8-bit k_b and rounded once for 16-bit.  The
// chunk sums run in the same scale and are scaled back by 2^16 (exact).
template <int MODE, int W>
__device__ __forceinline__ void mid_packed_atoms(const float4* __restrict__ list, uint32_t tabBiased, int n,
                                                 const float2 (&gxn)[kNX / 2], float gy, float gz,
                                                 float2 (&sum)[kNX / 2], float2 (&cmp)[kNX / 2], float kScale) {
  const float2 bias2 = dup2(8388608.f);
  const float2 down = dup2(1.0f / 65536.f), up = dup2(65536.f);
#pragma unroll 1
  for (int j0 = 0; j0 < n; j0 += kChunk) {
    float2 cs[kNX / 2];
#pragma unroll
    for (int k = 0; k < kNX / 2; k++)
      cs[k] = (MODE == kEmapKahan) ? make_float2(0.f, 0.f) : __fmul2_rn(sum[k], down);
    const int j1 = min(n, j0 + kChunk);
#pragma unroll 8
    for (int j = j0; j < j1; j++) {
      const float4 a = list[j];
      const float dy = a.y - gy, dz = a.z - gz;
      const float2 dyz2 = dup2(fmaf(dz, dz, dy * dy));
      const float2 ax = dup2(a.x), awg = dup2(a.w), aws = dup2(a.w * kScale);
#pragma unroll
      for (int k = 0; k < kNX / 2; k++) {
        const float2 dx = __fadd2_rn(ax, gxn[k]);
        const float2 r2 = __ffma2_rn(dx, dx, dyz2);
        const float2 rs = rsqrt2(r2);
        const float2 f = __ffma2_rd(r2, rs, bias2);
        const float2 kb = make_float2(lds_packed<W>(tabBiased, f.x), lds_packed<W>(tabBiased, f.y));
        cs[k] = __ffma2_rn(rs, __ffma2_rn(aws, kb, awg), cs[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < kNX / 2; k++) cs[k] = __fmul2_rn(cs[k], up);
    add_chunk<MODE>(sum, cmp, cs);
  }
}

// One near atom against this thread's points, bins decided exactly near an
// edge.  GUARD: cap 1/r at 2 and clamp the bin at the table's end; without it
// the caller has shown that no point of the warp lies within 0.51 A of the
// atom and that no bin can pass the table's end (the CTA box is small enough),
// so neither would change a value.
template <bool DDD, int MODE, bool GUARD>
__device__ __forceinline__ void near_exact(const EmapSmem& S, const EmapParams& P, const int slot, const int j,
                                           const float2 dyz2, const float2 ax, const float2 aw,
                                           const float2 (&gxn)[kNX / 2], const int iy, const int iz, const int xb,
                                           const int xs, float2 (&sum)[kNX / 2], float2 (&cmp)[kNX / 2]) {
  const float cap = 0.02f;        // min(1/r, 2) in units of 1/(100 r)
  const float kBias = 8388608.f;  // 2^23
  const double h = P.h;
  float2 rsv[kNX / 2];
  float2 fT[kNX / 2];   // 100 r (FP32), kept for the rare exact-bin fallback
  float2 fr5[kNX / 2];  // fraction of 100 r minus one half
  uint32_t bits[kNX];   // 2^23 + bin, as float bits
  bool any = false;
#pragma unroll
  for (int k = 0; k < kNX / 2; k++) {
    const float2 dx = __fadd2_rn(ax, gxn[k]);
    const float2 r2 = __ffma2_rn(dx, dx, dyz2);
    rsv[k] = rsqrt2(r2);
    if (DDD) {
      fT[k] = __fmul2_rn(r2, rsv[k]);
      float2 f = __ffma2_rd(r2, rsv[k], dup2(kBias));
      if (GUARD) {
        f.x = fminf(f.x, kBias + (float)(kTabLen - 1));
        f.y = fminf(f.y, kBias + (float)(kTabLen - 1));
      }
      bits[2 * k] = __float_as_uint(f.x);
      bits[2 * k + 1] = __float_as_uint(f.y);
      // Within delta of a bin edge <=> the fraction of T is within delta of 0 or 1.
      fr5[k] = __fadd2_rn(__fadd2_rn(fT[k], __ffma2_rn(f, dup2(-1.f), dup2(kBias))), dup2(-0.5f));
      any |= (fabsf(fr5[k].x) > 0.5f - P.delta) | (fabsf(fr5[k].y) > 0.5f - P.delta);
    }
  }
  if (DDD && __any_sync(0xffffffffu, any)) {
    if (any) {
      const double4 a64 = S.ring[slot][S.nearIdx[j]];
      const double gy64 = __dmul_rn((double)(iy - P.n2y), h), gz64 = __dmul_rn((double)(iz - P.n2z), h);
      const double ddz = __dsub_rn(a64.z, gz64), ddy = __dsub_rn(a64.y, gy64);
      const double dydz = __dadd_rn(__dmul_rn(ddy, ddy), __dmul_rn(ddz, ddz));
#pragma unroll
      for (int k = 0; k < kNX; k++) {
        if (fabsf(lo_hi(fr5[k >> 1], k)) > 0.5f - P.delta) {
          // The reference's bin is kmid - 1 or kmid, kmid the integer nearest 100 r.
          const int kmid = min(__float_as_int(lo_hi(fT[k >> 1], k) + 12582912.f) - 0x4B400000, kTabLen - 1);
          const double gx64 = __dmul_rn((double)(xb + k * xs - P.n2x), h);
          const double ddx = __dsub_rn(a64.x, gx64);
          const double r2d = __dadd_rn(__dmul_rn(ddx, ddx), dydz);
          const int b = (kmid == 0) ? 0 : ((r2d >= P.thr[kmid]) ? kmid : kmid - 1);
          bits[k] = 0x4B000000u + (uint32_t)b;
        }
      }
    }
  }
  const uint32_t tabB = smem_u32(S.tab) - 0x2C000000u;  // address(tab) - 4 * bits(2^23)
#pragma unroll
  for (int k = 0; k < kNX / 2; k++) {
    float2 term = __fmul2_rn(aw, GUARD ? make_float2(fminf(rsv[k].x, cap), fminf(rsv[k].y, cap)) : rsv[k]);
    if (DDD) {
      float2 t;
      asm("ld.shared.f32 %0, [%1];" : "=f"(t.x) : "r"(tabB + (bits[2 * k] << 2)));
      asm("ld.shared.f32 %0, [%1];" : "=f"(t.y) : "r"(tabB + (bits[2 * k + 1] << 2)));
      term = __fmul2_rn(term, t);
    }
    if (MODE == kEmapKahan)
      kahan2(sum[k], cmp[k], term);
    else
      sum[k] = __fadd2_rn(sum[k], term);
  }
}

// One work unit: CTA box `blk` of job P against atom split `split`.  Called
// once per CTA by emap_kernel, and repeatedly by the persistent batch kernel.
template <bool DDD, int MODE>
__device__ __forceinline__ void emap_unit(const EmapParams& P, const int blk, const int split, EmapSmem& S) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const EmapBlock B = P.blocks[blk];
  const int a0 = split * P.chunk;
  const int a1 = min(P.n_atoms, a0 + P.chunk);
  const int ntiles = (a1 - a0 + kTile - 1) / kTile;

  // This thread's points, in the CTA-local frame scaled by 100.
  const bool active = tid < B.nitems;
  int xc = 0, iy = 0, iz = 0;
  const int item = P.items[B.item0 + (active ? tid : 0)];
  unpack_item(item, xc, iy, iz);
  // x of point k = xb + k * xs: NX consecutive points, or every other point of
  // the 2 NX points of an interleaved column pair.
  const bool il = (item & kItemInterleaved) != 0;
  const int xb = il ? (xc >> 1) * (2 * kNX) + (xc & 1) : xc * kNX;
  const int xs = il ? 2 : 1;
  const double h = P.h;
  float gx[kNX];
#pragma unroll
  for (int k = 0; k < kNX; k++)
    gx[k] = (float)(((double)(xb + k * xs - P.n2x) * h - B.ox) * 100.0);
  const float gy = (float)(((double)(iy - P.n2y) * h - B.oy) * 100.0);
  const float gz = (float)(((double)(iz - P.n2z) * h - B.oz) * 100.0);
  float2 gxn[kNX / 2];
#pragma unroll
  for (int k = 0; k < kNX / 2; k++) gxn[k] = make_float2(-gx[2 * k], -gx[2 * k + 1]);

  // Packed tail tables for this box: only when no bin can pass the table's end.
  const bool pk = DDD && P.packed != nullptr && !B.clampMid;
  if (DDD) {
    const float4* src = reinterpret_cast<const float4*>(P.table);
    float4* dst = reinterpret_cast<float4*>(S.tab);
    for (int i = tid; i < kTabLen / 4; i += kThreads) dst[i] = src[i];
    if (pk) {
      uint4* pdst = reinterpret_cast<uint4*>(S.packed);
      for (int i = tid; i < P.packedVecs; i += kThreads) pdst[i] = P.packed[i];
    }
  }
  // This warp's box: the extent of its active lanes' points (an empty box,
  // lo > hi, when no lane has an item), widened by 1 (0.01 A).
  {
    float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    if (active) {
      lo[0] = fminf(gx[0], gx[kNX - 1]);
      hi[0] = fmaxf(gx[0], gx[kNX - 1]);
      lo[1] = hi[1] = gy;
      lo[2] = hi[2] = gz;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int d = 0; d < 3; d++) {
        lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
        hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
      }
    if (lane == 0) {
      S.wlo[warp] = make_float4(lo[0] - 1.f, lo[1] - 1.f, lo[2] - 1.f, 0.f);
      S.whi[warp] = make_float4(hi[0] + 1.f, hi[1] + 1.f, hi[2] + 1.f, 0.f);
    }
  }
  if (tid == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
    mbar_init(&S.barIdle, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const float gFar = DDD ? S.tab[kTabLen - 1] : 1.f;
  if (tid == 0 && ntiles > 0) {
    unsigned n0 = (unsigned)min(kTile, a1 - a0);
    mbar_arrive_expect_tx(&S.bar[0], n0 * 32u);
    tma_load_1d(S.ring[0], P.atoms + a0, n0 * 32u, &S.bar[0]);
  }

  float2 sum[kNX / 2], cmp[kNX / 2];
  double wsum = 0.0;  // FP64 sum of the weights this thread converted (checksum)
#pragma unroll
  for (int k = 0; k < kNX / 2; k++) { sum[k] = make_float2(0.f, 0.f); cmp[k] = make_float2(0.f, 0.f); }

  const float cap = 0.02f;        // min(1/r, 2) in units of 1/(100 r)
  const float kBias = 8388608.f;  // 2^23: adding it with round-down leaves floor() in the low bits

  for (int t = 0; t < ntiles; t++) {
    const int slot = t & 1;
    const int t0 = a0 + t * kTile;
    const int nt = min(kTile, a1 - t0);
    if (tid == 0 && t + 1 < ntiles) {
      // The other slot was released by the __syncthreads() that ended tile t-1.
      const int t1 = t0 + kTile;
      unsigned n1 = (unsigned)min(kTile, a1 - t1);
      fence_proxy_async();
      mbar_arrive_expect_tx(&S.bar[slot ^ 1], n1 * 32u);
      tma_load_1d(S.ring[slot ^ 1], P.atoms + t1, n1 * 32u, &S.bar[slot ^ 1]);
    }
    bool ok = mbar_wait_bounded(&S.bar[slot], (unsigned)(t >> 1) & 1u, P.status);
    // Test hook: after the first tile has landed, wait a few polls on a
    // barrier that nothing arrives on; the wait expires like a lost copy would.
    if (P.testIdleWait > 0 && t == 0) ok = mbar_wait_limit(&S.barIdle, 0u, P.status, P.testIdleWait) && ok;
    if (__syncthreads_or(!ok)) {
      // Give the copies still in flight (this tile's and the prefetched next
      // one) a bounded chance to land before shared memory is released.
      if (tid == 0) {
        mbar_wait_bounded(&S.bar[slot], (unsigned)(t >> 1) & 1u, P.status);
        if (t + 1 < ntiles) mbar_wait_bounded(&S.bar[slot ^ 1], (unsigned)((t + 1) >> 1) & 1u, P.status);
      }
      return;
    }

    // Classify and convert this tile's atoms (one atom per thread).
    int cls = -1;
    unsigned nearBits = 0xFFFFu;
    float4 loc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tid < nt) {
      double4 a = S.ring[slot][tid];
      wsum += a.w;
      loc.x = (float)((a.x - B.ox) * 100.0);
      loc.y = (float)((a.y - B.oy) * 100.0);
      loc.z = (float)((a.z - B.oz) * 100.0);
      loc.w = (float)(a.w * 100.0);
      const float dx = fmaxf(fabsf(loc.x) - B.hx, 0.f), dy = fmaxf(fabsf(loc.y) - B.hy, 0.f),
                  dz = fmaxf(fabsf(loc.z) - B.hz, 0.f);
      const float d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < P.rnear2) {
        cls = kClsNear;
        // The warps whose own points it is near: the others evaluate it as a mid atom.
        unsigned m = 0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; w++) {
          const float4 wl = S.wlo[w], wh = S.whi[w];
          const float ex = fmaxf(fmaxf(wl.x - loc.x, loc.x - wh.x), 0.f);
          const float ey = fmaxf(fmaxf(wl.y - loc.y, loc.y - wh.y), 0.f);
          const float ez = fmaxf(fmaxf(wl.z - loc.z, loc.z - wh.z), 0.f);
          const float e2 = ex * ex + ey * ey + ez * ez;
          m |= ((e2 < P.rnear2 ? 1u : 0u) << w) | ((e2 < 51.f * 51.f ? 1u : 0u) << (8 + w));
        }
        nearBits = m;
      } else if (DDD && d2 < B.rfar2) {
        cls = kClsMid;
        if (pk && d2 >= P.r16sq) {
          cls = d2 >= P.r8sq ? kClsMid8 : kClsMid16;
          loc.w *= gFar * (1.0f / 65536.f);
        }
      } else {
        cls = kClsFar;
        loc.w *= gFar;
      }
    }
    const unsigned lt = (1u << lane) - 1u;
    unsigned myBallot = 0;
#pragma unroll
    for (int c = 0; c < kNumCls; c++) {
      const unsigned b = __ballot_sync(0xffffffffu, cls == c);
      if (cls == c) myBallot = b;
      if (lane == 0) S.cnt[c][warp] = __popc(b);
    }
    __syncthreads();
    // Start of each class in the list, and of this warp's atoms within it.
    int base[kNumCls];
    int run = 0, myPos = 0;
#pragma unroll
    for (int c = 0; c < kNumCls; c++) {
      base[c] = run;
      int off = 0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; w++) {
        const int v = S.cnt[c][w];
        off += (w < warp) ? v : 0;
        run += v;
      }
      if (cls == c) myPos = base[c] + off + __popc(myBallot & lt);
    }
    if (cls >= 0) {
      S.list[myPos] = loc;
      if (cls == kClsNear) {
        S.nearIdx[myPos] = (short)tid;
        S.nearMask[myPos] = (unsigned short)nearBits;
      }
    }
    __syncthreads();
    const int nNear = base[kClsMid];

    // Mid atoms: table read, or a packed tail table.
    if (DDD) {
      const uint32_t tabBiased = smem_u32(S.tab) - 0x2C000000u;
      const int nMid = base[kClsMid16] - base[kClsMid];
      if (B.clampMid)
        mid_atoms<MODE, true>(S.list + base[kClsMid], tabBiased, nMid, gxn, gy, gz, sum, cmp);
      else
        mid_atoms<MODE, false>(S.list + base[kClsMid], tabBiased, nMid, gxn, gy, gz, sum, cmp);
      if (pk) {
        const uint32_t p16 = smem_u32(S.packed) - 2u * (0x4B000000u + (uint32_t)P.b16);
        const uint32_t p8 = smem_u32(S.packed) + 16u * (uint32_t)P.vec8 - (0x4B000000u + (uint32_t)P.b8);
        mid_packed_atoms<MODE, 2>(S.list + base[kClsMid16], p16, base[kClsMid8] - base[kClsMid16], gxn, gy, gz, sum,
                                  cmp, P.kScale);
        mid_packed_atoms<MODE, 1>(S.list + base[kClsMid8], p8, base[kClsFar] - base[kClsMid8], gxn, gy, gz, sum,
                                  cmp, P.kScale);
      }
    }

    // Far atoms: saturated dielectric (or the constant dielectric), no table.
    const int nFar = run - base[kClsFar];
    const float4* farA = S.list + base[kClsFar];
#pragma unroll 1
    for (int j0 = 0; j0 < nFar; j0 += kChunk) {
      float2 cs[kNX / 2];
#pragma unroll
      for (int k = 0; k < kNX / 2; k++)
        cs[k] = (MODE == kEmapKahan) ? make_float2(0.f, 0.f) : sum[k];
      const int j1 = min(nFar, j0 + kChunk);
#pragma unroll 8
      for (int j = j0; j < j1; j++) {
        const float4 a = farA[j];
        const float dy = a.y - gy, dz = a.z - gz;
        const float2 dyz2 = dup2(fmaf(dz, dz, dy * dy));
        const float2 ax = dup2(a.x), aw = dup2(a.w);
#pragma unroll
        for (int k = 0; k < kNX / 2; k++) {
          const float2 dx = __fadd2_rn(ax, gxn[k]);
          cs[k] = __ffma2_rn(aw, rsqrt2(__ffma2_rn(dx, dx, dyz2)), cs[k]);
        }
      }
      add_chunk<MODE>(sum, cmp, cs);
    }

    // Near atoms: clamp 1/r at 2 and decide bins near an edge exactly.
#pragma unroll 1
    for (int j = 0; j < nNear; j++) {
      const float4 a = S.list[j];
      const float dy = a.y - gy, dz = a.z - gz;
      // The 1e-30 keeps r2 > 0 (an atom on a grid point) without a per-point max.
      const float2 dyz2 = dup2(fmaf(dz, dz, dy * dy) + 1e-30f);
      const float2 ax = dup2(a.x), aw = dup2(a.w);
      if (DDD && !((S.nearMask[j] >> warp) & 1u)) {
        // At least rNear from every point of this warp (uniform): the mid-list
        // arithmetic (no cap, round-down bin), each term compensated.  The
        // clamp keeps the bin inside the table for any box size, and for the
        // lanes without an item, whose stand-in points can lie anywhere.
        const uint32_t tabB = smem_u32(S.tab) - 0x2C000000u;
#pragma unroll
        for (int k = 0; k < kNX / 2; k++) {
          const float2 dx = __fadd2_rn(ax, gxn[k]);
          const float2 r2 = __ffma2_rn(dx, dx, dyz2);
          const float2 rs = rsqrt2(r2);
          float2 f = __ffma2_rd(r2, rs, dup2(kBias));
          f.x = fminf(f.x, kBias + (float)(kTabLen - 1));
          f.y = fminf(f.y, kBias + (float)(kTabLen - 1));
          const float2 t = make_float2(lds_bin(tabB, f.x), lds_bin(tabB, f.y));
          const float2 term = __fmul2_rn(__fmul2_rn(aw, rs), t);
          if (MODE == kEmapKahan)
            kahan2(sum[k], cmp[k], term);
          else
            sum[k] = __fadd2_rn(sum[k], term);
        }
        continue;
      }
      if (!B.clampMid && !((S.nearMask[j] >> (8 + warp)) & 1u))  // uniform
        near_exact<DDD, MODE, false>(S, P, slot, j, dyz2, ax, aw, gxn, iy, iz, xb, xs, sum, cmp);
      else
        near_exact<DDD, MODE, true>(S, P, slot, j, dyz2, ax, aw, gxn, iy, iz, xb, xs, sum, cmp);
    }
    __syncthreads();  // ring slot and atom lists are free again
  }

  // Net-charge checksum: the first CTA of each atom split reports, in FP64,
  // the sum of the weights of every atom that went through its tile ring.
  if (blk == 0 && P.checksum) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if (lane == 0) S.wpart[warp] = wsum;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int w = 0; w < kThreads / 32; w++) s += S.wpart[w];
      P.checksum[split] = s;
    }
  }

  if (!active) return;
  const int64_t row = ((int64_t)iz * P.ny + iy) * P.nx;
#pragma unroll
  for (int k = 0; k < kNX; k++) {
    const int x = xb + k * xs;
    if (x >= P.nx) break;
    const double v = (MODE == kEmapKahan) ? (double)lo_hi(sum[k >> 1], k) - (double)lo_hi(cmp[k >> 1], k)
                                          : (double)lo_hi(sum[k >> 1], k);
    if (P.nsplit == 1)
      P.out[row + x] = (float)v;
    else
      P.partial[(int64_t)split * P.npoints + row + x] = v;
  }
}

template <bool DDD, int MODE>
__global__ void __launch_bounds__(kThreads, kEmapCtasPerSm) emap_kernel(const __grid_constant__ EmapParams P) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  EmapSmem& S = *reinterpret_cast<EmapSmem*>(smem_raw);
  emap_unit<DDD, MODE>(P, blockIdx.x % P.nblocks, blockIdx.x / P.nblocks, S);
}

// Persistent kernel over the work units of many jobs (a batch of receptors):
// every CTA takes the next unit (job, CTA box) from an atomic counter until
// none is left; the host orders units by decreasing cost.  Jobs run without
// an atom split and with the distance-dependent dielectric.  Two CTAs per SM:
// at three the per-unit job parameters spill and the batch gains nothing.
template <int MODE>
__global__ void __launch_bounds__(kThreads, 2)
    emap_batch_kernel(const EmapParams* __restrict__ jobs, const int2* __restrict__ units, int nunits, int* counter) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  EmapSmem& S = *reinterpret_cast<EmapSmem*>(smem_raw);
  for (;;) {
    __syncthreads();  // the previous unit is finished by every thread
    if (threadIdx.x == 0) S.unit = atomicAdd(counter, 1);
    __syncthreads();
    const int u = S.unit;
    if (u >= nunits) return;
    const int2 w = units[u];
    emap_unit<true, MODE>(jobs[w.x], w.y, 0, S);
  }
}

cudaError_t emap_batch_launch(const EmapParams* jobs, const int2* units, int nunits, int* counter, int grid,
                              cudaStream_t st) {
  const size_t smem = sizeof(EmapSmem);
  cudaError_t e = cudaFuncSetAttribute(emap_batch_kernel<kEmapKahan>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  emap_batch_kernel<kEmapKahan><<<grid, kThreads, smem, st>>>(jobs, units, nunits, counter);
  return cudaGetLastError();
}

// Persistent direct e-map over a device-side list of CTA boxes.
template <int MODE>
__global__ void __launch_bounds__(kThreads, kEmapCtasPerSm)
    emap_list_kernel(const __grid_constant__ EmapParams P, const int* __restrict__ list, const int* __restrict__ count,
                     int* counter) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  EmapSmem& S = *reinterpret_cast<EmapSmem*>(smem_raw);
  const int n = min(*count, P.nblocks);
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) S.unit = atomicAdd(counter, 1);
    __syncthreads();
    const int u = S.unit;
    if (u >= n) return;
    const int blk = list[u];
    if (blk < 0 || blk >= P.nblocks) {
      if (threadIdx.x == 0) atomicOr(P.status, ST_BAD_INPUT);
      continue;
    }
    emap_unit<true, MODE>(P, blk, 0, S);
  }
}

cudaError_t emap_list_launch(const EmapParams& P, const int* list, const int* count, int* counter, int grid,
                             cudaStream_t st) {
  const size_t smem = sizeof(EmapSmem);
  cudaError_t e = cudaFuncSetAttribute(emap_list_kernel<kEmapKahan>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  emap_list_kernel<kEmapKahan><<<grid, kThreads, smem, st>>>(P, list, count, counter);
  return cudaGetLastError();
}

// Sum the atom-split partials in split order (FP64).
__global__ void emap_reduce_kernel(const double* __restrict__ partial, int nsplit, int64_t n, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nsplit; k++) s += partial[(int64_t)k * n + i];
    out[i] = (float)s;
  }
}

size_t emap_smem_bytes() { return sizeof(EmapSmem); }

cudaError_t emap_launch(const EmapParams& P, bool ddd, int mode, int grid, cudaStream_t st) {
  const size_t smem = sizeof(EmapSmem);
  cudaError_t e = cudaSuccess;
#define AG_LAUNCH(D, M)                                                                               \
  do {                                                                                                \
    e = cudaFuncSetAttribute(emap_kernel<D, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    if (e != cudaSuccess) return e;                                                                   \
    emap_kernel<D, M><<<grid, kThreads, smem, st>>>(P);                                               \
  } while (0)
  if (ddd) {
    if (mode == kEmapKahan) AG_LAUNCH(true, kEmapKahan); else AG_LAUNCH(true, kEmapPlain);
  } else {
    if (mode == kEmapKahan) AG_LAUNCH(false, kEmapKahan); else AG_LAUNCH(false, kEmapPlain);
  }
#undef AG_LAUNCH
  e = cudaGetLastError();
  if (e != cudaSuccess || P.nsplit == 1) return e;
  emap_reduce_kernel<<<592, 256, 0, st>>>(P.partial, P.nsplit, P.npoints, P.out);
  return cudaGetLastError();
}

}  // namespace agk
