// Kernels of the learned far-field surrogate of the e-map: the coarse
// far-field grid, its finite differences, the corrector's input features, the
// corrector network's forward and backward convolutions on the tensor cores
// (BF16 operands, FP32 accumulation), the training loss and optimiser, and
// the residual probes that send badly predicted boxes back to the direct sum.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "ag_device.cuh"
#include "ag_kernels.h"
#include "surr_kernels.h"

namespace agk {

using namespace agd;

namespace {

__device__ __forceinline__ float ex2f_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ---------------------------------------------------------------------------
// Coarse far field: F(node) = sum over all atoms of w psi(|node - atom|).
// Two nodes per thread (node and node + 256 of the CTA's 512), evaluated with
// Blackwell's packed FP32 instructions (add/mul/fma .f32x2, each half rounded
// as the scalar instruction), atoms streamed through shared memory in FP32
// (grid-centred coordinates), plain FP32 sums over 32-atom chunks added in
// FP64.  Atoms are split across blockIdx.y; partials are summed in order.
// ---------------------------------------------------------------------------
constexpr int kCoarseNodes = 512;  // nodes per CTA (256 threads x 2)

__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

__global__ void __launch_bounds__(256) surr_coarse_kernel(const CoarseParams P) {
  __shared__ float4 sA[256];
  const int tid = threadIdx.x;
  const SurrGeom& G = P.G;
  const int64_t NN = (int64_t)G.N[0] * G.N[1] * G.N[2];
  const int64_t node0 = (int64_t)blockIdx.x * kCoarseNodes + tid, node1 = node0 + 256;
  float gc[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int64_t node = q ? node1 : node0;
    if (node < NN) {
      const int I = (int)(node % G.N[0]), J = (int)((node / G.N[0]) % G.N[1]),
                K = (int)(node / ((int64_t)G.N[0] * G.N[1]));
      gc[q][0] = (float)((double)((I - G.halo) * G.R - G.n2x) * G.h);
      gc[q][1] = (float)((double)((J - G.halo) * G.R - G.n2y) * G.h);
      gc[q][2] = (float)((double)((K - G.halo) * G.R - G.n2z) * G.h);
    }
  }
  // Minus the node coordinates, one pair per axis.
  const float2 ngx = make_float2(-gc[0][0], -gc[1][0]), ngy = make_float2(-gc[0][1], -gc[1][1]),
               ngz = make_float2(-gc[0][2], -gc[1][2]);
  const SplitKernel& S = P.K;
  const float2 nl2 = dup2(S.negLambda2), eShift2 = dup2(-S.negLambda2 * S.shift);
  const float2 pA = dup2(S.pA), pB = dup2(S.pB), pC = dup2(S.pC);
  const float2 q0 = dup2(S.poly[0]), q1 = dup2(S.poly[1]), q2 = dup2(S.poly[2]), q3 = dup2(S.poly[3]),
               q4 = dup2(S.poly[4]), q5 = dup2(S.poly[5]);
  const int split = blockIdx.y;
  const int a0 = split * P.chunk, a1 = min(P.n_atoms, a0 + P.chunk);
  double acc0 = 0.0, acc1 = 0.0;
  for (int t0 = a0; t0 < a1; t0 += 256) {
    __syncthreads();
    if (t0 + tid < a1) {
      const double4 a = P.atoms[t0 + tid];
      sA[tid] = make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w);
    }
    __syncthreads();
    const int nt = min(256, a1 - t0);
#pragma unroll 1
    for (int j0 = 0; j0 < nt; j0 += 32) {
      const int j1 = min(nt, j0 + 32);
      float2 s = make_float2(0.f, 0.f);
#pragma unroll 4
      for (int j = j0; j < j1; j++) {
        const float4 a = sA[j];
        const float2 dx = __fadd2_rn(dup2(a.x), ngx), dy = __fadd2_rn(dup2(a.y), ngy),
                     dz = __fadd2_rn(dup2(a.z), ngz);
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        // r2 = 0 (an atom on the node) gives rsqrt = inf and a NaN tail below,
        // but r2 < a2 there, so the select takes the inner polynomial.
        const float2 rs = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
        // E = exp(-lambda (r - shift)); past the table's end (81.91 A) the
        // reference's value stays at bin 8191, which differs from this by < 1e-10.
        const float2 arg = __ffma2_rn(__fmul2_rn(r2, rs), nl2, eShift2);
        const float2 E = make_float2(ex2f_approx(arg.x), ex2f_approx(arg.y));
        float2 tau = __ffma2_rn(E, q5, q4);
        tau = __ffma2_rn(E, tau, q3);
        tau = __ffma2_rn(E, tau, q2);
        tau = __ffma2_rn(E, tau, q1);
        tau = __ffma2_rn(E, tau, q0);
        const float2 inner = __ffma2_rn(r2, __ffma2_rn(r2, pC, pB), pA);
        const float2 outer = __fmul2_rn(tau, rs);
        const float2 psi = make_float2(r2.x < S.a2 ? inner.x : outer.x, r2.y < S.a2 ? inner.y : outer.y);
        s = __ffma2_rn(dup2(a.w), psi, s);
      }
      acc0 += (double)s.x;
      acc1 += (double)s.y;
    }
  }
  if (node0 < NN) P.partial[(int64_t)split * NN + node0] = acc0;
  if (node1 < NN) P.partial[(int64_t)split * NN + node1] = acc1;
}

__global__ void surr_coarse_reduce_kernel(const double* __restrict__ partial, int nsplit, int64_t n,
                                          double* __restrict__ field) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nsplit; k++) s += partial[(int64_t)k * n + i];
    field[i] = s;
  }
}

// Second and fourth central differences of the far field at each node the
// fine grid uses.
__global__ void surr_deriv_kernel(const double* __restrict__ f, const SurrGeom G, float4* __restrict__ rec) {
  const int64_t n = (int64_t)G.nc[0] * G.nc[1] * G.nc[2];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int I = (int)(i % G.nc[0]) + G.halo, J = (int)((i / G.nc[0]) % G.nc[1]) + G.halo,
            K = (int)(i / ((int64_t)G.nc[0] * G.nc[1])) + G.halo;
  const int64_t sx = 1, sy = G.N[0], sz = (int64_t)G.N[0] * G.N[1];
  const int64_t c = K * sz + J * sy + I;
  const double F = f[c];
  double d2[3], d4[3];
  const int64_t st[3] = {sx, sy, sz};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double m2 = f[c - 2 * st[a]], m1 = f[c - st[a]], p1 = f[c + st[a]], p2 = f[c + 2 * st[a]];
    d2[a] = p1 - 2.0 * F + m1;
    d4[a] = p2 - 4.0 * p1 + 6.0 * F - 4.0 * m1 + m2;
  }
  rec[2 * i] = make_float4((float)F, (float)d2[0], (float)d2[1], (float)d2[2]);
  rec[2 * i + 1] = make_float4((float)d4[0], (float)d4[1], (float)d4[2], 0.f);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xFFFF0000u); }

// Fine-grid features: with (u, v, w) the point's fractions inside its coarse
// cell and D2*, D4* the trilinearly interpolated differences,
//   f0..f2 = u(1-u) D2x, v(1-v) D2y, w(1-w) D2z   (leading trilinear error)
//   f3..f5 = D2x, D2y, D2z
//   f6 = sum_a u_a(1-u_a)(2u_a-1) dD2a/du_a       (third-order term)
//   f7 = sum_a u_a(1-u_a) D4a                       (fourth-order term)
__global__ void surr_feature_kernel(const float4* __restrict__ rec, const SurrGeom G, float sIn, float* __restrict__ out,
                                    uint4* __restrict__ feat) {
  const int64_t np = (int64_t)G.nx * G.ny * G.nz;
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int ix = (int)(p % G.nx), iy = (int)((p / G.nx) % G.ny), iz = (int)(p / ((int64_t)G.nx * G.ny));
  const int I = min(ix / G.R, G.nc[0] - 2), J = min(iy / G.R, G.nc[1] - 2), K = min(iz / G.R, G.nc[2] - 2);
  const float invR = 1.0f / (float)G.R;
  const float u = (float)(ix - I * G.R) * invR, v = (float)(iy - J * G.R) * invR, w = (float)(iz - K * G.R) * invR;
  const float wx[2] = {1.f - u, u}, wy[2] = {1.f - v, v}, wz[2] = {1.f - w, w};
  float F = 0.f, Dx = 0.f, Dy = 0.f, Dz = 0.f, Qx = 0.f, Qy = 0.f, Qz = 0.f, gX = 0.f, gY = 0.f, gZ = 0.f;
#pragma unroll
  for (int dk = 0; dk < 2; dk++)
#pragma unroll
    for (int dj = 0; dj < 2; dj++)
#pragma unroll
      for (int di = 0; di < 2; di++) {
        const int64_t idx = ((int64_t)(K + dk) * G.nc[1] + (J + dj)) * G.nc[0] + (I + di);
        const float4 r0 = rec[2 * idx], r1 = rec[2 * idx + 1];
        const float wt = wx[di] * wy[dj] * wz[dk];
        F = fmaf(wt, r0.x, F);
        Dx = fmaf(wt, r0.y, Dx);
        Dy = fmaf(wt, r0.z, Dy);
        Dz = fmaf(wt, r0.w, Dz);
        Qx = fmaf(wt, r1.x, Qx);
        Qy = fmaf(wt, r1.y, Qy);
        Qz = fmaf(wt, r1.z, Qz);
        gX = fmaf((di ? 1.f : -1.f) * wy[dj] * wz[dk], r0.y, gX);
        gY = fmaf((dj ? 1.f : -1.f) * wx[di] * wz[dk], r0.z, gY);
        gZ = fmaf((dk ? 1.f : -1.f) * wx[di] * wy[dj], r0.w, gZ);
      }
  const float bu = u * (1.f - u), bv = v * (1.f - v), bw = w * (1.f - w);
  const float f[8] = {bu * Dx,
                      bv * Dy,
                      bw * Dz,
                      Dx,
                      Dy,
                      Dz,
                      bu * (2.f * u - 1.f) * gX + bv * (2.f * v - 1.f) * gY + bw * (2.f * w - 1.f) * gZ,
                      bu * Qx + bv * Qy + bw * Qz};
  uint4 o;
  o.x = pack_bf16x2(f[0] * sIn, f[1] * sIn);
  o.y = pack_bf16x2(f[2] * sIn, f[3] * sIn);
  o.z = pack_bf16x2(f[4] * sIn, f[5] * sIn);
  o.w = pack_bf16x2(f[6] * sIn, f[7] * sIn);
  feat[p] = o;
  if (out) out[p] += F;
}

// ---------------------------------------------------------------------------
// Tensor-core convolutions (mma.sync m16n8k16, BF16 x BF16 -> FP32).
// Output tile 16 x 4 x 4 points per CTA iteration; each of the 16 warps owns
// one x row of 16 points (the MMA's M), the 3x3x3 taps and input channels
// form K, the output channels N.  The packed weights stay in shared memory
// for the CTA's lifetime; input halos (18 x 6 x 6 points) are double-buffered
// with cp.async, the next tile's halo landing while the current one is
// multiplied.  Fragments come from ldmatrix, whose per-lane row addresses
// read each tap's shifted window in place (no im2col copy); the K loop is
// fully unrolled so every tap offset is an immediate.
// ---------------------------------------------------------------------------
constexpr int kTX = 16, kTY = 4, kTZ = 4;
constexpr int kHX = kTX + 2, kHY = kTY + 2, kHZ = kTZ + 2;
constexpr int kHalo = kHX * kHY * kHZ;     // 648
constexpr int kTilePts = kTX * kTY * kTZ;  // 256
constexpr int kConvThreads = 512;          // 16 warps, one x row each

template <int CIN>
struct ConvShape {
  static constexpr int KS = CIN == 8 ? kKS8 : kKS32;   // weight row stride (BF16)
  static constexpr int NCHUNK = CIN == 8 ? 14 : 54;    // K / 16 (taps paired for CIN 8)
  static constexpr int CS = CIN == 8 ? 8 : CIN + 8;    // halo point stride (BF16)
};

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t (&r)[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t (&r)[4]) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2(uint32_t addr, uint32_t& r0, uint32_t& r1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t addr, uint32_t& r0, uint32_t& r1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// 16-byte asynchronous copy global -> shared; src_bytes 0 fills zeros.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ int tap_base(int t, int y, int z) {
  const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
  return ((z + dz) * kHY + (y + dy)) * kHX + dx;
}

__device__ __forceinline__ void tile_origin(int tile, int nx, int ny, int& x0, int& y0, int& z0) {
  const int ntx = (nx + kTX - 1) / kTX, nty = (ny + kTY - 1) / kTY;
  x0 = (tile % ntx) * kTX;
  y0 = ((tile / ntx) % nty) * kTY;
  z0 = (tile / (ntx * nty)) * kTZ;
}

// Halo of tile (x0, y0, z0) of a [P][CIN] BF16 tensor into sX (zero outside the grid).
template <int CIN, int NTHREADS, bool ASYNC>
__device__ __forceinline__ void load_halo(const uint16_t* __restrict__ in, uint16_t* sX, int x0, int y0, int z0, int nx,
                                          int ny, int nz) {
  constexpr int CH = CIN / 8;
  constexpr int CS = ConvShape<CIN>::CS;
  for (int i = threadIdx.x; i < kHalo * CH; i += NTHREADS) {
    const int pt = i / CH, c = i - pt * CH;
    const int hx = pt % kHX, hy = (pt / kHX) % kHY, hz = pt / (kHX * kHY);
    const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z0 + hz - 1;
    const bool inside = gx >= 0 && gx < nx && gy >= 0 && gy < ny && gz >= 0 && gz < nz;
    const uint4* src = reinterpret_cast<const uint4*>(in) +
                       (inside ? (((int64_t)gz * ny + gy) * nx + gx) * CH + c : 0);
    if (ASYNC) {
      cp_async16(smem_u32(sX + pt * CS + c * 8), src, inside ? 16 : 0);
    } else {
      *reinterpret_cast<uint4*>(sX + pt * CS + c * 8) = inside ? __ldg(src) : make_uint4(0u, 0u, 0u, 0u);
    }
  }
}

template <int CIN, int NT, int EPI>
__global__ void __launch_bounds__(kConvThreads, 1) surr_conv_kernel(const ConvArgs A) {
  using SH = ConvShape<CIN>;
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* sW = reinterpret_cast<uint16_t*>(smem);  // [8 NT][KS]
  uint16_t* sX0 = sW + 8 * NT * SH::KS;              // two halo buffers [kHalo][CS]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ntiles = ((A.nx + kTX - 1) / kTX) * ((A.ny + kTY - 1) / kTY) * ((A.nz + kTZ - 1) / kTZ);
  if ((int)blockIdx.x < ntiles) {
    int x0, y0, z0;
    tile_origin(blockIdx.x, A.nx, A.ny, x0, y0, z0);
    load_halo<CIN, kConvThreads, true>(A.in, sX0, x0, y0, z0, A.nx, A.ny, A.nz);
  }
  cp_async_commit();
  {
    const uint4* src = reinterpret_cast<const uint4*>(A.w);
    uint4* dst = reinterpret_cast<uint4*>(sW);
    for (int i = tid; i < 8 * NT * SH::KS / 8; i += kConvThreads) dst[i] = __ldg(src + i);
  }
  const int q = lane >> 3, r = lane & 7, g = lane >> 2, tig = lane & 3;
  const int wy = warp & 3, wz = warp >> 2;
  const uint32_t sWa = smem_u32(sW);
  // Per-lane byte offsets of the A rows (tap 0) and B rows (chunk 0); the
  // unrolled K loop adds compile-time tap and chunk offsets to them.
  const uint32_t aLane =
      (uint32_t)(((wz * kHY + wy) * kHX + r + ((q & 1) ? 8 : 0)) * SH::CS + (CIN == 32 && (q & 2) ? 8 : 0)) * 2u;
  const bool aTap1 = CIN == 8 && (q & 2);  // CIN 8: lanes 16-31 read the second tap of a pair
  const uint32_t bBase = NT == 1 ? sWa + (uint32_t)(r * SH::KS + (q & 1) * 8) * 2u
                                 : sWa + (uint32_t)((8 * (q >> 1) + r) * SH::KS + (q & 1) * 8) * 2u;
  int it = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
    uint16_t* sX = sX0 + (it & 1) * kHalo * SH::CS;
    const int next = tile + gridDim.x;
    if (next < ntiles) {
      int nx0, ny0, nz0;
      tile_origin(next, A.nx, A.ny, nx0, ny0, nz0);
      load_halo<CIN, kConvThreads, true>(A.in, sX0 + ((it + 1) & 1) * kHalo * SH::CS, nx0, ny0, nz0, A.nx, A.ny,
                                         A.nz);
    }
    cp_async_commit();
    cp_async_wait1();  // this thread's copies of the current halo have landed
    __syncthreads();   // ... and everyone else's (and the weights)
    int x0, y0, z0;
    tile_origin(tile, A.nx, A.ny, x0, y0, z0);
    const uint32_t aBase = smem_u32(sX) + aLane;
    float acc[NT][4];
#pragma unroll
    for (int n = 0; n < NT; n++) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
    for (int j = 0; j < SH::NCHUNK; j++) {
      uint32_t aAddr;
      if (CIN == 32) {
        const int t = j >> 1;
        const int off = ((t / 9) * kHY + (t / 3) % 3) * kHX + t % 3;
        aAddr = aBase + (uint32_t)(off * SH::CS + 16 * (j & 1)) * 2u;
      } else {
        const int t0 = min(2 * j, 26), t1 = min(2 * j + 1, 26);  // tap 27 is padding (zero weights)
        const int off0 = ((t0 / 9) * kHY + (t0 / 3) % 3) * kHX + t0 % 3;
        const int off1 = ((t1 / 9) * kHY + (t1 / 3) % 3) * kHX + t1 % 3;
        aAddr = aBase + (uint32_t)((aTap1 ? off1 : off0) * SH::CS) * 2u;
      }
      uint32_t a[4];
      ldsm_x4(aAddr, a);
      const uint32_t K0b = 32u * j;  // 16 BF16 per chunk
      if (NT == 1) {
        uint32_t b0, b1;
        ldsm_x2(bBase + K0b, b0, b1);
        mma_bf16(acc[0], a, b0, b1);
      } else {
#pragma unroll
        for (int np = 0; np < NT / 2; np++) {
          uint32_t b[4];
          ldsm_x4(bBase + K0b + (uint32_t)(16 * np * SH::KS) * 2u, b);
          mma_bf16(acc[2 * np], a, b[0], b[1]);
          mma_bf16(acc[2 * np + 1], a, b[2], b[3]);
        }
      }
    }
    // Epilogue: rows g and g+8 are points x0+g, x0+g+8 of row (y0+wy, z0+wz).
    const int gy = y0 + wy, gz = z0 + wz;
    if (gy < A.ny && gz < A.nz) {
#pragma unroll
      for (int half = 0; half < 2; half++) {
        const int x = x0 + g + 8 * half;
        if (x >= A.nx) continue;
        const int64_t p = ((int64_t)gz * A.ny + gy) * A.nx + x;
        if (EPI == EPI_STORE || EPI == EPI_ADD) {
          if (tig == 0) {
            const float v = acc[0][2 * half] * A.scale;
            if (EPI == EPI_STORE) A.outF[p] = v;
            else A.outF[p] += v;
          }
        } else {
#pragma unroll
          for (int n = 0; n < NT; n++) {
            float v0 = acc[n][2 * half], v1 = acc[n][2 * half + 1];
            const int co = 8 * n + 2 * tig;
            if (EPI == EPI_LEAKY) {
              v0 = v0 > 0.f ? v0 : v0 * kLeakySlope;
              v1 = v1 > 0.f ? v1 : v1 * kLeakySlope;
            } else {
              const uint32_t m = __ldg(reinterpret_cast<const uint32_t*>(A.act) + ((p * 32 + co) >> 1));
              v0 = bf16_lo(m) > 0.f ? v0 : v0 * kLeakySlope;
              v1 = bf16_hi(m) > 0.f ? v1 : v1 * kLeakySlope;
            }
            reinterpret_cast<uint32_t*>(A.out16)[(p * 32 + co) >> 1] = pack_bf16x2(v0, v1);
          }
        }
      }
    }
    __syncthreads();  // this halo buffer is read; the next iteration's prefetch may overwrite it
  }
}

// Weight gradient: per tap t, dW[t] (CIN x COUT) += X_t^T Y over the tile's
// 256 points (K = points, fragments by transposing ldmatrix).  Units of work
// are (tap, 16 input channels) (CIN 32) or tap pairs (CIN 8), spread over 16
// warps; accumulators stay in registers across all tiles a CTA visits and
// are added to global memory once.
template <int CIN, int NT>
__global__ void __launch_bounds__(512, 1) surr_bwdw_kernel(const BwdwArgs A) {
  using SH = ConvShape<CIN>;
  constexpr int YS = NT == 1 ? 8 : 8 * NT + 8;   // Y tile point stride (BF16)
  constexpr int NU = CIN == 32 ? 54 : 14;
  constexpr int UPW = (NU + 15) / 16;
  constexpr int COUT = NT == 1 ? 1 : 32;
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t* sX = reinterpret_cast<uint16_t*>(smem);  // [kHalo][CS]
  uint16_t* sY = sX + kHalo * SH::CS;                // [kTilePts][YS]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = lane >> 3, r = lane & 7, g = lane >> 2, tig = lane & 3;
  const int ntx = (A.nx + kTX - 1) / kTX, nty = (A.ny + kTY - 1) / kTY, ntz = (A.nz + kTZ - 1) / kTZ;
  const int ntiles = ntx * nty * ntz;
  const uint32_t sXa = smem_u32(sX), sYa = smem_u32(sY);
  float acc[UPW][NT][4];
#pragma unroll
  for (int u = 0; u < UPW; u++)
#pragma unroll
    for (int n = 0; n < NT; n++) acc[u][n][0] = acc[u][n][1] = acc[u][n][2] = acc[u][n][3] = 0.f;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int x0, y0, z0;
    tile_origin(tile, A.nx, A.ny, x0, y0, z0);
    __syncthreads();
    load_halo<CIN, 512, false>(A.x, sX, x0, y0, z0, A.nx, A.ny, A.nz);
    for (int i = tid; i < kTilePts * NT; i += 512) {
      const int pt = i / NT, c = i - pt * NT;
      const int lx = pt % kTX, ly = (pt / kTX) % kTY, lz = pt / (kTX * kTY);
      const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gx < A.nx && gy < A.ny && gz < A.nz)
        v = __ldg(reinterpret_cast<const uint4*>(A.y) + (((int64_t)gz * A.ny + gy) * A.nx + gx) * NT + c);
      *reinterpret_cast<uint4*>(sY + pt * YS + c * 8) = v;
    }
    __syncthreads();
#pragma unroll
    for (int ui = 0; ui < UPW; ui++) {
      const int u = warp + 16 * ui;
      if (u >= NU) continue;
#pragma unroll 2
      for (int kc = 0; kc < kTY * kTZ; kc++) {
        const int ly = kc % kTY, lz = kc / kTY;
        int pt, ch;
        if (CIN == 32) {
          pt = tap_base(u >> 1, ly, lz) + r + ((q & 2) ? 8 : 0);
          ch = 16 * (u & 1) + ((q & 1) ? 8 : 0);
        } else {
          const int t = min(2 * u + (q & 1), 26);
          pt = tap_base(t, ly, lz) + r + ((q & 2) ? 8 : 0);
          ch = 0;
        }
        uint32_t a[4];
        ldsm_x4_t(sXa + (uint32_t)(pt * SH::CS + ch) * 2u, a);
        if (NT == 1) {
          uint32_t b0, b1;
          ldsm_x2_t(sYa + (uint32_t)((kc * 16 + r + (q & 1) * 8) * YS) * 2u, b0, b1);
          mma_bf16(acc[ui][0], a, b0, b1);
        } else {
#pragma unroll
          for (int np = 0; np < NT / 2; np++) {
            uint32_t b[4];
            const int yp = kc * 16 + r + (q & 1) * 8;
            ldsm_x4_t(sYa + (uint32_t)(yp * YS + 8 * (2 * np + (q >> 1))) * 2u, b);
            mma_bf16(acc[ui][2 * np], a, b[0], b[1]);
            mma_bf16(acc[ui][2 * np + 1], a, b[2], b[3]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int ui = 0; ui < UPW; ui++) {
    const int u = warp + 16 * ui;
    if (u >= NU) continue;
#pragma unroll
    for (int n = 0; n < NT; n++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int m = g + ((e & 2) ? 8 : 0);
        const int co = 8 * n + 2 * tig + (e & 1);
        int t, ci;
        if (CIN == 32) {
          t = u >> 1;
          ci = 16 * (u & 1) + m;
        } else {
          t = 2 * u + (m >> 3);
          ci = m & 7;
        }
        if (t < 27 && co < COUT) atomicAdd(&A.dw[((int64_t)t * CIN + ci) * COUT + co], acc[ui][n][e]);
      }
  }
}

// Packed BF16 weight matrices from the FP32 master weights.
__global__ void surr_pack_kernel(const float* __restrict__ w, PackedWeights pw) {
  const float* W1 = w;
  const float* W2 = w + kSurrW1;
  const float* W3 = w + kSurrW1 + kSurrW2;
  const int n1 = 32 * kKS8, n2 = 32 * kKS32, n3 = 8 * kKS32;
  const int total = n1 + n2 + n3 + n2 + n1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    int j = i;
    if (j < n1) {  // wk1[co][t*8+ci] = W1[t][ci][co]
      const int co = j / kKS8, k = j % kKS8;
      const float v = k < 216 ? W1[((k >> 3) * 8 + (k & 7)) * 32 + co] : 0.f;
      pw.wk1[j] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
      continue;
    }
    j -= n1;
    if (j < n2) {  // wk2[co][t*32+ci] = W2[t][ci][co]
      const int co = j / kKS32, k = j % kKS32;
      const float v = k < 864 ? W2[((k >> 5) * 32 + (k & 31)) * 32 + co] : 0.f;
      pw.wk2[j] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
      continue;
    }
    j -= n2;
    if (j < n3) {  // wk3[0][t*32+ci] = W3[t][ci]
      const int row = j / kKS32, k = j % kKS32;
      const float v = (row == 0 && k < 864) ? W3[(k >> 5) * 32 + (k & 31)] : 0.f;
      pw.wk3[j] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
      continue;
    }
    j -= n3;
    if (j < n2) {  // wk2t[ci][t'*32+co] = W2[26-t'][ci][co]
      const int ci = j / kKS32, k = j % kKS32;
      const float v = k < 864 ? W2[((26 - (k >> 5)) * 32 + ci) * 32 + (k & 31)] : 0.f;
      pw.wk2t[j] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
      continue;
    }
    j -= n2;
    {  // wk3t[ci][t'*8] = W3[26-t'][ci]
      const int ci = j / kKS8, k = j % kKS8;
      const float v = (k < 216 && (k & 7) == 0) ? W3[(26 - (k >> 3)) * 32 + ci] : 0.f;
      pw.wk3t[j] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
  }
}

__global__ void surr_loss_kernel(const float* __restrict__ o, const float* __restrict__ y, int64_t n, float invSOut,
                                 float gscale, uint4* __restrict__ do8, double* loss) {
  __shared__ double part[8];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float e = o[i] - y[i] * invSOut;
    s += (double)e * e;
    do8[i] = make_uint4(pack_bf16x2(gscale * e, 0.f), 0u, 0u, 0u);
  }
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += part[k];
    atomicAdd(loss, t);
  }
}

__global__ void surr_adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                                 const float* __restrict__ g, int n, float lr, float b1, float b2, float eps, float bc1,
                                 float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

__global__ void surr_residual_kernel(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ y,
                                     const uint4* __restrict__ feat, int64_t n, double* sums) {
  __shared__ double part[9][8];
  double s[9];
#pragma unroll
  for (int k = 0; k < 9; k++) s[k] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float d = a[i] - b[i];
    y[i] = d;
    s[0] += (double)d * d;
    const uint4 f = feat[i];
    const uint32_t fw[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double lo = bf16_lo(fw[k]), hi = bf16_hi(fw[k]);
      s[1 + 2 * k] += lo * lo;
      s[2 + 2 * k] += hi * hi;
    }
  }
#pragma unroll
  for (int k = 0; k < 9; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    if ((threadIdx.x & 31) == 0) part[k][threadIdx.x >> 5] = s[k];
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[threadIdx.x][w];
    atomicAdd(&sums[threadIdx.x], t);
  }
}

__global__ void surr_scale_kernel(uint4* __restrict__ feat, int64_t n, float s) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint4 f = feat[i];
    uint32_t* fw = reinterpret_cast<uint32_t*>(&f);
#pragma unroll
    for (int k = 0; k < 4; k++) fw[k] = pack_bf16x2(bf16_lo(fw[k]) * s, bf16_hi(fw[k]) * s);
    feat[i] = f;
  }
}

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// One warp per probe point, eight per CTA sharing each 256-atom tile staged
// in shared memory: the direct sum, compared with the map.  Pairs within 6 A
// follow the reference's FP64 arithmetic (Cpu.cpp:59-82); farther pairs, where
// a bin decided one step off moves a term by < 3e-5, run in FP32 with 1/r and
// the bin from one reciprocal square root.
__global__ void __launch_bounds__(256) surr_probe_kernel(const ProbeParams P) {
  __shared__ double4 sA[256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = blockIdx.x * 8 + warp;
  const bool valid = gw < P.nblocks * P.nprobe;
  int b = 0, x = 0, y = 0, z = 0;
  bool ok = false;
  if (valid) {
    b = gw / P.nprobe;
    const int k = gw - b * P.nprobe;
    const EmapBlock B = reinterpret_cast<const EmapBlock*>(P.blocks)[b];
    if (B.nitems > 0) {
      const uint32_t hsh = mix32((uint32_t)b * 7919u + (uint32_t)k * 104729u + 12345u);
      const int seg = max(1, B.nitems / P.nprobe);
      const int it = min(B.nitems - 1, k * seg + (int)(hsh % (uint32_t)seg));
      const int v = P.items[B.item0 + it];
      const int xc = v & 0xFF;
      y = (v >> 8) & 0x7FF;
      z = (v >> 19) & 0x7FF;
      x = min(xc * kNX + (int)((hsh >> 16) % (uint32_t)kNX), P.nx - 1);
      ok = true;
    }
  }
  const double gx = (double)(x - P.n2x) * P.h, gy = (double)(y - P.n2y) * P.h, gz = (double)(z - P.n2z) * P.h;
  double s64 = 0.0;
  float s = 0.f, c = 0.f;
  for (int t0 = 0; t0 < P.n_atoms; t0 += 256) {
    const int nt = min(256, P.n_atoms - t0);
    __syncthreads();
    if ((int)threadIdx.x < nt) sA[threadIdx.x] = P.atoms[t0 + threadIdx.x];
    __syncthreads();
    if (!ok) continue;
    for (int i = lane; i < nt; i += 32) {
      const double4 a = sA[i];
      const double dx = a.x - gx, dy = a.y - gy, dz = a.z - gz;
      const float fx = (float)dx, fy = (float)dy, fz = (float)dz;
      const float r2 = fmaf(fx, fx, fmaf(fy, fy, fz * fz));
      if (r2 < 36.f) {
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double inv = fmin(1.0 / r, 2.0);
        const int bin = min((int)(r * 100.0), 8191);
        s64 += a.w * inv * P.tab[bin];
      } else {
        const float rs = rsqrt_approx(r2);
        const int bin = min((int)(r2 * rs * 100.f), 8191);
        const float term = (float)a.w * rs * (float)P.tab[bin];
        const float yk = term - c;  // Kahan
        const float t = s + yk;
        c = (t - s) - yk;
        s = t;
      }
    }
  }
  s64 += (double)s - (double)c;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s64 += __shfl_xor_sync(0xffffffffu, s64, o);
  if (ok && lane == 0) {
    const int64_t p = ((int64_t)z * P.ny + y) * P.nx + x;
    const float err = (float)fabs((double)P.map[p] - s64);
    atomicMax(P.maxErrBits, __float_as_uint(err));
    if (!(err <= P.tol)) {
      if (atomicExch(&P.flags[b], 1) == 0) P.list[atomicAdd(P.count, 1)] = b;
    }
  }
}

template <int CIN, int NT, int EPI>
cudaError_t conv_go(const ConvArgs& A, int sms, cudaStream_t st) {
  const size_t smem = (size_t)(8 * NT * ConvShape<CIN>::KS + 2 * kHalo * ConvShape<CIN>::CS) * 2;
  cudaError_t e = cudaFuncSetAttribute(surr_conv_kernel<CIN, NT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int ntiles = ((A.nx + kTX - 1) / kTX) * ((A.ny + kTY - 1) / kTY) * ((A.nz + kTZ - 1) / kTZ);
  int per = 1;  // resident CTAs per SM
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, surr_conv_kernel<CIN, NT, EPI>, kConvThreads, smem) !=
          cudaSuccess ||
      per < 1)
    per = 1;
  const int grid = ntiles < per * sms ? ntiles : per * sms;
  surr_conv_kernel<CIN, NT, EPI><<<grid, kConvThreads, smem, st>>>(A);
  return cudaGetLastError();
}

template <int CIN, int NT>
cudaError_t bwdw_go(const BwdwArgs& A, int sms, cudaStream_t st) {
  constexpr int YS = NT == 1 ? 8 : 8 * NT + 8;
  const size_t smem = (size_t)(kHalo * ConvShape<CIN>::CS + kTilePts * YS) * 2;
  cudaError_t e =
      cudaFuncSetAttribute(surr_bwdw_kernel<CIN, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int ntiles = ((A.nx + kTX - 1) / kTX) * ((A.ny + kTY - 1) / kTY) * ((A.nz + kTZ - 1) / kTZ);
  const int grid = ntiles < sms ? ntiles : sms;
  surr_bwdw_kernel<CIN, NT><<<grid, 512, smem, st>>>(A);
  return cudaGetLastError();
}

}  // namespace

cudaError_t surr_coarse_launch(const CoarseParams& P, cudaStream_t st) {
  const int64_t NN = (int64_t)P.G.N[0] * P.G.N[1] * P.G.N[2];
  if (P.n_atoms <= 0) return cudaMemsetAsync(P.field, 0, sizeof(double) * NN, st);
  dim3 grid((unsigned)((NN + kCoarseNodes - 1) / kCoarseNodes), (unsigned)P.nsplit);
  surr_coarse_kernel<<<grid, 256, 0, st>>>(P);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  surr_coarse_reduce_kernel<<<(unsigned)((NN + 255) / 256), 256, 0, st>>>(P.partial, P.nsplit, NN, P.field);
  return cudaGetLastError();
}

cudaError_t surr_deriv_launch(const double* field, const SurrGeom& G, float4* rec, cudaStream_t st) {
  const int64_t n = (int64_t)G.nc[0] * G.nc[1] * G.nc[2];
  surr_deriv_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(field, G, rec);
  return cudaGetLastError();
}

cudaError_t surr_feature_launch(const float4* rec, const SurrGeom& G, float sIn, float* out, uint4* feat,
                                cudaStream_t st) {
  const int64_t n = (int64_t)G.nx * G.ny * G.nz;
  surr_feature_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(rec, G, sIn, out, feat);
  return cudaGetLastError();
}

cudaError_t surr_conv_launch(int cin, int nt, int epi, const ConvArgs& A, int sms, cudaStream_t st) {
  if (cin == 8 && nt == 4 && epi == EPI_LEAKY) return conv_go<8, 4, EPI_LEAKY>(A, sms, st);
  if (cin == 32 && nt == 4 && epi == EPI_LEAKY) return conv_go<32, 4, EPI_LEAKY>(A, sms, st);
  if (cin == 32 && nt == 4 && epi == EPI_GRADMASK) return conv_go<32, 4, EPI_GRADMASK>(A, sms, st);
  if (cin == 8 && nt == 4 && epi == EPI_GRADMASK) return conv_go<8, 4, EPI_GRADMASK>(A, sms, st);
  if (cin == 32 && nt == 1 && epi == EPI_STORE) return conv_go<32, 1, EPI_STORE>(A, sms, st);
  if (cin == 32 && nt == 1 && epi == EPI_ADD) return conv_go<32, 1, EPI_ADD>(A, sms, st);
  return cudaErrorInvalidValue;
}

cudaError_t surr_bwdw_launch(int cin, int nt, const BwdwArgs& A, int sms, cudaStream_t st) {
  if (cin == 32 && nt == 4) return bwdw_go<32, 4>(A, sms, st);
  if (cin == 8 && nt == 4) return bwdw_go<8, 4>(A, sms, st);
  if (cin == 32 && nt == 1) return bwdw_go<32, 1>(A, sms, st);
  return cudaErrorInvalidValue;
}

cudaError_t surr_pack_launch(const float* w, const PackedWeights& pw, cudaStream_t st) {
  surr_pack_kernel<<<148, 256, 0, st>>>(w, pw);
  return cudaGetLastError();
}

cudaError_t surr_loss_launch(const float* o, const float* y, int64_t n, float invSOut, uint4* do8, double* loss,
                             cudaStream_t st) {
  surr_loss_kernel<<<592, 256, 0, st>>>(o, y, n, invSOut, (float)(2.0 / (double)n), do8, loss);
  return cudaGetLastError();
}

cudaError_t surr_adam_launch(float* w, float* m, float* v, const float* g, int n, float lr, float b1, float b2,
                             float eps, int step, cudaStream_t st) {
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  surr_adam_kernel<<<(n + 255) / 256, 256, 0, st>>>(w, m, v, g, n, lr, b1, b2, eps, bc1, bc2);
  return cudaGetLastError();
}

cudaError_t surr_residual_launch(const float* a, const float* b, float* y, const uint4* feat, int64_t n, double* sums,
                                 cudaStream_t st) {
  surr_residual_kernel<<<592, 256, 0, st>>>(a, b, y, feat, n, sums);
  return cudaGetLastError();
}

cudaError_t surr_scale_launch(uint4* feat, int64_t n, float s, cudaStream_t st) {
  surr_scale_kernel<<<592, 256, 0, st>>>(feat, n, s);
  return cudaGetLastError();
}

cudaError_t surr_probe_launch(const ProbeParams& P, cudaStream_t st) {
  const int64_t warps = (int64_t)P.nblocks * P.nprobe;
  if (warps == 0) return cudaSuccess;
  surr_probe_kernel<<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(P);
  return cudaGetLastError();
}

}  // namespace agk
