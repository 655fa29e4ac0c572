// Corrector convolutions of the e-map surrogate on the 5th-generation tensor
// cores (tcgen05.mma, BF16 x BF16 -> FP32 accumulators in tensor memory), fed
// by TMA tile loads.
//
// A 3x3x3 convolution over a channel-last BF16 grid is an implicit GEMM:
//   D[point][co] = sum over taps t and input channels ci of
//                  X[point + off(t)][ci] * W[t][ci][co].
// One output tile is 8 (x) x 16 (y) x 1 (z) = 128 points, the MMA's M.  Its
// input halo (10 x 18 x 3 points) arrives by one 4-D TMA tile load per
// 8-channel plane.  Activations between layers are stored chunk-planar,
// [C/8][z][y][x][8 channels], so that a plane's x run is contiguous: the
// tensor map merges x and the 8 channels into one innermost dimension and a
// box row is 10 points x 16 bytes = 160 bytes (points outside the grid are
// filled with zeros by the copy engine):
//
//   halo[plane c][point p] at  c * kPlane + p * 16,  p = (hz * 18 + hy) * 10 + hx.
//
// In that layout the A operand of every tap is a plain no-swizzle K-major
// matrix: rows are points (8 consecutive x form one 8 x 16-byte core matrix,
// consecutive y rows are 160 bytes apart = SBO) and the two 8-channel halves
// of a 16-channel K step are one plane apart (LBO); a tap only moves the start
// address.  The weights are packed in the matching layout
//
//   W[kchunk][co][8 channels],  kchunk = (tap * CINP + ci) / 8,
//
// (core matrices of 8 output channels, SBO 128 bytes, LBO = NOUT * 16 bytes).
//
// Pipeline (one CTA per SM, persistent over tiles, warp-specialised): warp 5
// keeps up to 8 halo tiles in flight (as many as shared memory holds) (TMA, mbarrier with transaction count);
// warp 4 issues the 27 * CINP / 16 MMAs of each tile, spread over kAcc
// independent accumulators so consecutive MMAs do not wait on each other,
// into one of two tensor-memory buffers and commits them to mbarriers that
// free the halo stage and hand the buffer over; warps 0-3 read finished
// buffers (warp w owns lanes 32w..32w+31), sum the accumulators and write the
// epilogue, then hand the buffer back.  Every wait is bounded.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "ag_device.cuh"
#include "surr_kernels.h"

namespace agk {

using namespace agd;

namespace {

constexpr int kTcX = 8, kTcY = 16;            // output tile (z = 1)
constexpr int kTcHX = kTcX + 2, kTcHY = kTcY + 2, kTcHZ = 3;
constexpr int kTcHalo = kTcHX * kTcHY * kTcHZ;  // 540 points
constexpr int kPlane = 8704;                    // bytes per 8-channel plane: 540 x 16, padded to 128-byte TMA alignment
constexpr int kTcThreads = 192;                 // warps 0-3 epilogue, warp 4 MMA, warp 5 TMA
constexpr int kSmemBudget = 226 * 1024;         // dynamic shared memory per CTA (one CTA per SM)

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = nout, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(int nout) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nout >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns of this thread's TMEM lane (no wait).
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 4-D TMA tile load global -> shared (no multicast), completion on `bar`.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

template <int CINP, int NOUT>
struct TcShape {
  // CINP 16 (8 real input channels): one K step of 16 covers two taps, the
  // first tap's 8 channels and the next tap's 8, so the padding plane is not
  // multiplied; the tap pairs (0,1), (2,3), ..., (24,25), (26, zero plane).
  static constexpr bool kPairTaps = CINP == 16;
  static constexpr int kChunks = kPairTaps ? 28 : 27 * CINP / 8;  // 8-channel K chunks
  static constexpr int kWBytes = kChunks * NOUT * 16;              // packed weights
  static constexpr int kStageBytes = (CINP / 8) * kPlane;
  static constexpr int kMmas = kPairTaps ? 14 : 27 * (CINP / 16);
  // halo tiles in flight: as many as the shared memory left after the weights holds, at most 8
  static constexpr int kStages = (kSmemBudget - kWBytes - 128) / kStageBytes < 8 ? (kSmemBudget - kWBytes - 128) / kStageBytes : 8;
  static constexpr int kAcc = 4;  // independent accumulators per tile (breaks the MMA dependency chain)
  static constexpr int kBufCols = kAcc * NOUT;
  static constexpr int kTmemCols = 2 * kBufCols;  // two tile buffers: 256 columns
};

// Epilogue of one tile: the sum of its NACC accumulators (NOUT columns each,
// starting at column taddr).  The loads of all accumulators are issued before
// one wait, 16 columns at a time.
template <int NOUT, int NACC, int EPI>
__device__ __forceinline__ void tc_epilogue(const ConvArgs& A, uint32_t taddr, int x0, int y0, int z0) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t rowAddr = taddr + ((uint32_t)(32 * warp) << 16);
  const int i = 32 * warp + lane;
  const int x = x0 + (i & 7), y = y0 + (i >> 3);
  const bool inside = x < A.nx && y < A.ny;
  const int64_t p = ((int64_t)z0 * A.ny + y) * A.nx + x;
  static_assert(EPI == EPI_LEAKY, "the 32-output layers write leaky-ReLU BF16 activations");
  {
    const int64_t np = (int64_t)A.nx * A.ny * A.nz;
#pragma unroll
    for (int hcol = 0; hcol < 2; hcol++) {  // channels 16 hcol .. 16 hcol + 15
      uint32_t r[NACC][16];
#pragma unroll
      for (int a = 0; a < NACC; a++) tmem_ld16_nowait(rowAddr + (uint32_t)(a * NOUT + 16 * hcol), r[a]);
      tmem_wait();
      float v[16];
#pragma unroll
      for (int k = 0; k < 16; k++) {
        float t = __uint_as_float(r[0][k]);
#pragma unroll
        for (int a = 1; a < NACC; a++) t += __uint_as_float(r[a][k]);
        v[k] = t > 0.f ? t : t * kLeakySlope;
      }
      if (inside) {
        // chunk-planar output: plane q holds channels 8q..8q+7
#pragma unroll
        for (int q = 0; q < 2; q++) {
          uint4* dst = reinterpret_cast<uint4*>(A.out16 + ((int64_t)(2 * hcol + q) * np + p) * 8);
          const float* e = v + 8 * q;
          *dst = make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]), pack2(e[6], e[7]));
        }
      }
    }
  }
}

__device__ __forceinline__ void tile_xyz(int tile, int ntx, int nty, int& x0, int& y0, int& z0) {
  x0 = (tile % ntx) * kTcX;
  y0 = ((tile / ntx) % nty) * kTcY;
  z0 = tile / (ntx * nty);
}

// CIN: channels of the input tensor in global memory (8 or 32); CINP: channels
// in the halo and K per tap (16 or 32, padding planes are zero); NOUT: MMA N
// (32).  The one-output layer has its own kernel, surr_conv_tc3_kernel.
template <int CIN, int CINP, int NOUT, int EPI>
__global__ void __launch_bounds__(kTcThreads, 1)
    surr_conv_tc_kernel(const __grid_constant__ CUtensorMap tmap, const ConvArgs A, const uint16_t* __restrict__ wtc,
                        unsigned* status) {
  using SH = TcShape<CINP, NOUT>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 128-byte aligned base (TMA destinations); the launch adds 128 bytes of slack.
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  unsigned char* sW = smem;                  // packed weights
  unsigned char* sX = smem + SH::kWBytes;    // kStages halo stages
  constexpr int kStages = SH::kStages;
  __shared__ uint64_t full[8], empty[8], tfull[2], tempty[2];
  __shared__ uint32_t tmemBase;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntx = (A.nx + kTcX - 1) / kTcX, nty = (A.ny + kTcY - 1) / kTcY;
  const int ntiles = ntx * nty * A.nz;
  const int nmine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const uint32_t sXa = smem_u32(sX), sWa = smem_u32(sW);
  constexpr uint32_t txBytes = (uint32_t)(CIN / 8) * (kTcHalo * 16);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmemBase)),
                 "r"(SH::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int k = 0; k < kStages; k++) {
      mbar_init(&full[k], 1);
      mbar_init(&empty[k], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
    }
    fence_barrier_init();
  }
  {
    const uint4* src = reinterpret_cast<const uint4*>(wtc);
    uint4* dst = reinterpret_cast<uint4*>(sW);
    for (int i = tid; i < SH::kWBytes / 16; i += kTcThreads) dst[i] = __ldg(src + i);
    // Padding planes (K beyond the input's channels) stay zero in every stage.
    for (int k = 0; k < kStages; k++)
      for (int c = CIN / 8; c < CINP / 8; c++)
        for (int i = tid; i < kPlane / 16; i += kTcThreads)
          reinterpret_cast<uint4*>(sX + k * SH::kStageBytes + c * kPlane)[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  fence_proxy_async();  // generic-proxy writes above are read by the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmemBase;

  if (warp == 5) {
    // ---- TMA producer ----
    if (lane == 0) {
      for (int j = 0; j < nmine; j++) {
        const int st = j % kStages;
        if (j >= kStages && !mbar_wait_bounded(&empty[st], (unsigned)((j / kStages - 1) & 1), status)) break;
        int x0, y0, z0;
        tile_xyz((int)blockIdx.x + j * (int)gridDim.x, ntx, nty, x0, y0, z0);
        const uint32_t dst = sXa + (uint32_t)(st * SH::kStageBytes);
        mbar_arrive_expect_tx(&full[st], txBytes);
#pragma unroll
        for (int c = 0; c < CIN / 8; c++)
          tma_load_4d(dst + (uint32_t)(c * kPlane), &tmap, 8 * (x0 - 1), y0 - 1, z0 - 1, c, &full[st]);
      }
    }
  } else if (warp == 4) {
    // ---- MMA issuer ----
    if (lane == 0) {
      constexpr uint32_t idesc = instr_desc(NOUT);
      for (int i = 0; i < nmine; i++) {
        const int st = i % kStages, b = i & 1;
        if (i >= 2 && !mbar_wait_bounded(&tempty[b], (unsigned)(((i >> 1) - 1) & 1), status)) break;
        if (!mbar_wait_bounded(&full[st], (unsigned)((i / kStages) & 1), status)) break;
        tc_fence_after();
        const uint32_t dcol = tbase + (uint32_t)(b * SH::kBufCols);
        // Descriptors of the stage's and the weights' first core matrices; a tap
        // or K step only adds its byte offset / 16 to the start-address field
        // (bits 0-13, no carry: shared addresses stay below 256 KB).
        const uint64_t aDesc0 = smem_desc(sXa + (uint32_t)(st * SH::kStageBytes), kPlane, kTcHX * 16);
        const uint64_t aDesc1 = smem_desc(sXa + (uint32_t)(st * SH::kStageBytes), 0, kTcHX * 16);  // LBO per MMA
        const uint64_t bDesc0 = smem_desc(sWa, NOUT * 16, 128);
#pragma unroll
        for (int j = 0; j < SH::kMmas; j++) {
          uint64_t aDesc;
          uint32_t bOff;
          if constexpr (SH::kPairTaps) {
            // K halves: tap 2j's window and tap 2j+1's window of plane 0, LBO bytes
            // apart (the zero plane for the last, unpaired tap).
            const int t = 2 * j, t2 = 2 * j + 1;
            const uint32_t off1 = (uint32_t)((((t / 9) * kTcHY + (t / 3) % 3) * kTcHX + t % 3) * 16);
            const uint32_t off2 = t2 < 27 ? (uint32_t)((((t2 / 9) * kTcHY + (t2 / 3) % 3) * kTcHX + t2 % 3) * 16)
                                          : off1 + (uint32_t)kPlane;
            aDesc = aDesc1 + (off1 >> 4) + ((uint64_t)((off2 - off1) >> 4) << 16);
            bOff = (uint32_t)(2 * j * NOUT * 16);
          } else {
            const int t = j / (CINP / 16), hh = j % (CINP / 16);
            const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
            const uint32_t aOff = (uint32_t)(2 * hh * kPlane + ((dz * kTcHY + dy) * kTcHX + dx) * 16);
            aDesc = aDesc0 + (aOff >> 4);
            bOff = (uint32_t)((t * (CINP / 8) + 2 * hh) * NOUT * 16);
          }
          // MMA j accumulates into accumulator j % kAcc; the first MMA of each overwrites it
          tc_mma(dcol + (uint32_t)((j % SH::kAcc) * NOUT), aDesc, bDesc0 + (bOff >> 4), idesc, j >= SH::kAcc ? 1u : 0u);
        }
        tc_commit(&empty[st]);  // the halo stage is free once these MMAs complete
        tc_commit(&tfull[b]);   // ... and the accumulator buffer holds the tile
      }
    }
  } else {
    // ---- epilogue warps 0-3 ----
    for (int i = 0; i < nmine; i++) {
      const int b = i & 1;
      if (!mbar_wait_bounded(&tfull[b], (unsigned)((i >> 1) & 1), status)) break;
      tc_fence_after();
      int x0, y0, z0;
      tile_xyz((int)blockIdx.x + i * (int)gridDim.x, ntx, nty, x0, y0, z0);
      tc_epilogue<NOUT, SH::kAcc, EPI>(A, tbase + (uint32_t)(b * SH::kBufCols), x0, y0, z0);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(SH::kTmemCols));
}

// ---------------------------------------------------------------------------
// Layer 3 (32 channels -> 1 output) as a GEMM over the taps.  With one output
// channel, the layers' implicit GEMM would spend 27 x 2 MMAs of N 16 per tile
// on one useful column, each re-reading 4 KB of activations.  Instead, for
// every point h of the tile's halo,
//
//   Y[h][t] = sum_ci act[h][ci] W3[t][ci]      (M 128 halo points, N 32 = 27 taps + 5 zero, K 32),
//
// 5 x 2 MMAs per tile, and the epilogue gathers out(q) = sum_t Y[q + off(t)][t]
// through shared memory (the halo point of a tap lives in another TMEM lane).
// The halo planes are padded to 640 points so that the fifth M block stays
// inside its plane; rows 540..639 hold stale data and their Y rows are unused.
// ---------------------------------------------------------------------------
constexpr int kT3Rows = 640;                          // 5 M blocks of 128 halo points
constexpr int kT3Plane = kT3Rows * 16;                // bytes per 8-channel plane
constexpr int kT3StageBytes = 4 * kT3Plane;           // 32 channels
constexpr int kT3WBytes = 4 * 32 * 16;                // W[kchunk 4][tap 32][8 channels] BF16
constexpr int kT3Stride = 27;                         // floats per halo point in the Y array (odd: no bank conflicts on writes)
constexpr int kT3YBytes = kTcHalo * kT3Stride * 4;
constexpr int kT3Stages0 = (kSmemBudget - kT3WBytes - kT3YBytes - 128) / kT3StageBytes;
constexpr int kT3Stages = kT3Stages0 < 8 ? kT3Stages0 : 8;
constexpr int kT3BufCols = 5 * 32;                    // one tile's Y in TMEM
constexpr int kT3TmemCols = 512;                      // two tile buffers (320 columns), a power of two
static_assert(kT3Stages >= 2, "layer-3 halo ring needs two stages");

// The 128 epilogue threads (warps 0-3): named barrier 1, optionally or-reducing a flag.
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
__device__ __forceinline__ bool epi_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, 1, 128, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}

template <int EPI>
__global__ void __launch_bounds__(kTcThreads, 1)
    surr_conv_tc3_kernel(const __grid_constant__ CUtensorMap tmap, const ConvArgs A, const uint16_t* __restrict__ wtc,
                         unsigned* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 128-byte aligned base (TMA destinations); the launch adds 128 bytes of slack.
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  unsigned char* sW = smem;
  unsigned char* sX = smem + kT3WBytes;
  float* sY = reinterpret_cast<float*>(sX + kT3Stages * kT3StageBytes);
  __shared__ uint64_t full[kT3Stages], empty[kT3Stages], tfull[2], tempty[2];
  __shared__ uint32_t tmemBase;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntx = (A.nx + kTcX - 1) / kTcX, nty = (A.ny + kTcY - 1) / kTcY;
  const int ntiles = ntx * nty * A.nz;
  const int nmine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const uint32_t sXa = smem_u32(sX), sWa = smem_u32(sW);
  constexpr uint32_t txBytes = 4u * (kTcHalo * 16);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmemBase)),
                 "r"(kT3TmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int k = 0; k < kT3Stages; k++) {
      mbar_init(&full[k], 1);
      mbar_init(&empty[k], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
    }
    fence_barrier_init();
  }
  {
    const uint4* src = reinterpret_cast<const uint4*>(wtc);
    uint4* dst = reinterpret_cast<uint4*>(sW);
    for (int i = tid; i < kT3WBytes / 16; i += kTcThreads) dst[i] = __ldg(src + i);
  }
  fence_proxy_async();  // the weights written above are read by the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmemBase;

  if (warp == 5) {
    // ---- TMA producer ----
    if (lane == 0) {
      for (int j = 0; j < nmine; j++) {
        const int st = j % kT3Stages;
        if (j >= kT3Stages && !mbar_wait_bounded(&empty[st], (unsigned)((j / kT3Stages - 1) & 1), status)) break;
        int x0, y0, z0;
        tile_xyz((int)blockIdx.x + j * (int)gridDim.x, ntx, nty, x0, y0, z0);
        const uint32_t dst = sXa + (uint32_t)(st * kT3StageBytes);
        mbar_arrive_expect_tx(&full[st], txBytes);
#pragma unroll
        for (int c = 0; c < 4; c++)
          tma_load_4d(dst + (uint32_t)(c * kT3Plane), &tmap, 8 * (x0 - 1), y0 - 1, z0 - 1, c, &full[st]);
      }
    }
  } else if (warp == 4) {
    // ---- MMA issuer: 5 M blocks x 2 K steps per tile ----
    if (lane == 0) {
      constexpr uint32_t idesc = instr_desc(32);
      for (int i = 0; i < nmine; i++) {
        const int st = i % kT3Stages, b = i & 1;
        if (i >= 2 && !mbar_wait_bounded(&tempty[b], (unsigned)(((i >> 1) - 1) & 1), status)) break;
        if (!mbar_wait_bounded(&full[st], (unsigned)((i / kT3Stages) & 1), status)) break;
        tc_fence_after();
        // Start-address field + offset / 16 (no carry: shared addresses stay below 256 KB).
        const uint64_t aDesc0 = smem_desc(sXa + (uint32_t)(st * kT3StageBytes), kT3Plane, 128);
        const uint64_t bDesc0 = smem_desc(sWa, 32 * 16, 128);
#pragma unroll
        for (int mb = 0; mb < 5; mb++)
#pragma unroll
          for (int hh = 0; hh < 2; hh++)
            tc_mma(tbase + (uint32_t)(b * kT3BufCols + 32 * mb),
                   aDesc0 + (uint64_t)((2 * hh * kT3Plane + mb * 128 * 16) >> 4),
                   bDesc0 + (uint64_t)((2 * hh * 32 * 16) >> 4), idesc, hh ? 1u : 0u);
        tc_commit(&empty[st]);
        tc_commit(&tfull[b]);
      }
    }
  } else {
    // ---- epilogue warps 0-3 ----
    const int q = 32 * warp + lane;        // output point of the tile: x = q & 7, y = q >> 3
    const int hc = (q >> 3) * kTcHX + (q & 7);  // its halo index at tap (0, 0, 0)
    for (int i = 0; i < nmine; i++) {
      const int b = i & 1;
      const bool ok = mbar_wait_bounded(&tfull[b], (unsigned)((i >> 1) & 1), status);
      if (epi_any(!ok)) break;  // all four warps leave together
      tc_fence_after();
      // TMEM -> shared: lane 32 warp + lane of block mb is halo point 128 mb + 32 warp + lane.
#pragma unroll 1
      for (int mb = 0; mb < 5; mb++) {
        float v[32];
        tmem_ld32(tbase + (uint32_t)(b * kT3BufCols + 32 * mb) + ((uint32_t)(32 * warp) << 16), v);
        const int h = 128 * mb + q;
        if (h < kTcHalo) {
#pragma unroll
          for (int t = 0; t < 27; t++) sY[h * kT3Stride + t] = v[t];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);  // the TMEM buffer is free again
      epi_sync();                              // Y of the whole halo is in shared memory
      int x0, y0, z0;
      tile_xyz((int)blockIdx.x + i * (int)gridDim.x, ntx, nty, x0, y0, z0);
      float o = 0.f;
#pragma unroll
      for (int t = 0; t < 27; t++) {
        const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
        o += sY[(hc + (dz * kTcHY + dy) * kTcHX + dx) * kT3Stride + t];
      }
      o *= A.scale;
      const int x = x0 + (q & 7), y = y0 + (q >> 3);
      if (x < A.nx && y < A.ny) {
        const int64_t p = ((int64_t)z0 * A.ny + y) * A.nx + x;
        if (EPI == EPI_STORE) A.outF[p] = o;
        else A.outF[p] += o;
      }
      epi_sync();  // every read of Y is done before the next tile overwrites it
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kT3TmemCols));
}

// Master FP32 weights -> the tcgen05 layouts of the three layers.
__global__ void surr_pack_tc_kernel(const float* __restrict__ w, uint16_t* w1, uint16_t* w2, uint16_t* w3) {
  const float* W1 = w;
  const float* W2 = w + kSurrW1;
  const float* W3 = w + kSurrW1 + kSurrW2;
  constexpr int n1 = TcShape<16, 32>::kWBytes / 2, n2 = TcShape<32, 32>::kWBytes / 2, n3 = kT3WBytes / 2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1 + n2 + n3; i += gridDim.x * blockDim.x) {
    // element i of a layout [kchunk][co][8]: k = 8 kchunk + (i % 8), co = (i / 8) % NOUT
    if (i < n1) {  // layer 1: [tap 28][co 32][8 channels], tap 27 zero (the unpaired last K half)
      const int ci = i % 8, co = (i / 8) % 32, t = i / 256;
      w1[i] = __bfloat16_as_ushort(__float2bfloat16_rn(t < 27 ? W1[(t * 8 + ci) * 32 + co] : 0.f));
    } else if (i < n1 + n2) {  // layer 2: CINP 32, NOUT 32
      const int j = i - n1, e = j % 8, co = (j / 8) % 32, kc = j / 256, k = 8 * kc + e, t = k / 32, ci = k % 32;
      w2[j] = __bfloat16_as_ushort(__float2bfloat16_rn(W2[(t * 32 + ci) * 32 + co]));
    } else {  // layer 3 as a GEMM over taps: [kchunk 4][tap 32][8 channels], taps 27..31 zero
      const int j = i - n1 - n2, e = j % 8, t = (j / 8) % 32, kc = j / 256, ci = 8 * kc + e;
      w3[j] = __bfloat16_as_ushort(__float2bfloat16_rn(t < 27 ? W3[t * 32 + ci] : 0.f));
    }
  }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encodeTiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Tensor map of a chunk-planar [C/8][nz][ny][nx][8] BF16 tensor, x and the 8
// channels merged into the innermost dimension; the box is one 8-channel plane
// of a halo (innermost start coordinate 8 (x0 - 1): a multiple of 16 bytes).
cudaError_t halo_map(CUtensorMap* m, const uint16_t* base, int C, int nx, int ny, int nz) {
  EncodeTiledFn fn = encodeTiled();
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[4] = {(cuuint64_t)nx * 8, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)(C / 8)};
  const cuuint64_t strides[3] = {(cuuint64_t)nx * 16, (cuuint64_t)ny * nx * 16, (cuuint64_t)nz * ny * nx * 16};
  const cuuint32_t box[4] = {8 * kTcHX, kTcHY, kTcHZ, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<uint16_t*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int CIN, int CINP, int NOUT, int EPI>
cudaError_t tc_go(const ConvArgs& A, const uint16_t* wtc, unsigned* status, int sms, cudaStream_t st) {
  using SH = TcShape<CINP, NOUT>;
  if ((reinterpret_cast<uintptr_t>(A.in) & 15) != 0) return cudaErrorInvalidValue;  // TMA base alignment
  CUtensorMap map;
  cudaError_t e = halo_map(&map, A.in, CIN, A.nx, A.ny, A.nz);
  if (e != cudaSuccess) return e;
  const size_t smem = (size_t)SH::kWBytes + (size_t)SH::kStages * SH::kStageBytes + 128;
  e = cudaFuncSetAttribute(surr_conv_tc_kernel<CIN, CINP, NOUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess) return e;
  const int ntiles = ((A.nx + kTcX - 1) / kTcX) * ((A.ny + kTcY - 1) / kTcY) * A.nz;
  const int grid = ntiles < sms ? ntiles : sms;  // one CTA per SM
  surr_conv_tc_kernel<CIN, CINP, NOUT, EPI><<<grid, kTcThreads, smem, st>>>(map, A, wtc, status);
  return cudaGetLastError();
}

template <int EPI>
cudaError_t tc3_go(const ConvArgs& A, const uint16_t* wtc, unsigned* status, int sms, cudaStream_t st) {
  if ((reinterpret_cast<uintptr_t>(A.in) & 15) != 0) return cudaErrorInvalidValue;  // TMA base alignment
  CUtensorMap map;
  cudaError_t e = halo_map(&map, A.in, 32, A.nx, A.ny, A.nz);
  if (e != cudaSuccess) return e;
  const size_t smem = (size_t)kT3WBytes + (size_t)kT3Stages * kT3StageBytes + (size_t)kT3YBytes + 128;
  e = cudaFuncSetAttribute(surr_conv_tc3_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int ntiles = ((A.nx + kTcX - 1) / kTcX) * ((A.ny + kTcY - 1) / kTcY) * A.nz;
  const int grid = ntiles < sms ? ntiles : sms;  // one CTA per SM
  surr_conv_tc3_kernel<EPI><<<grid, kTcThreads, smem, st>>>(map, A, wtc, status);
  return cudaGetLastError();
}

}  // namespace

size_t surr_tc_weight_elems(int layer) {
  return layer == 1 ? TcShape<16, 32>::kWBytes / 2 : layer == 2 ? TcShape<32, 32>::kWBytes / 2 : kT3WBytes / 2;
}

cudaError_t surr_pack_tc_launch(const float* w, uint16_t* w1, uint16_t* w2, uint16_t* w3, cudaStream_t st) {
  surr_pack_tc_kernel<<<148, 256, 0, st>>>(w, w1, w2, w3);
  return cudaGetLastError();
}

cudaError_t surr_conv_tc_launch(int layer, int epi, const ConvArgs& A, const uint16_t* wtc, unsigned* status, int sms,
                                cudaStream_t st) {
  if (layer == 1 && epi == EPI_LEAKY) return tc_go<8, 16, 32, EPI_LEAKY>(A, wtc, status, sms, st);
  if (layer == 2 && epi == EPI_LEAKY) return tc_go<32, 32, 32, EPI_LEAKY>(A, wtc, status, sms, st);
  if (layer == 3 && epi == EPI_ADD) return tc3_go<EPI_ADD>(A, wtc, status, sms, st);
  if (layer == 3 && epi == EPI_STORE) return tc3_go<EPI_STORE>(A, wtc, status, sms, st);
  return cudaErrorInvalidValue;
}

}  // namespace agk
