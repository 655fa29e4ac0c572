// Launch interfaces of the learned far-field surrogate of the e-map.
//
// The e-map is split exactly as
//   e(p) = sum_{r < a} w (phi(r) - psi(r))  +  sum_all w psi(r)  +  residual,
// phi the reference's binned kernel min(1/r, 2) * invEps[int(100 r)], psi a
// smooth kernel: tau(r - 0.005) / r beyond a (tau = 332/eps evaluated
// analytically, the 0.005 A shift centring the 0.01 A bins) and an even
// quartic in r inside a that matches it to second order at a.  The residual
// is the binning noise of the atoms beyond a (zero mean, ~1e-4).  The first
// sum is the exact near field (emap_near_launch); the second, the far field,
// is smooth and is sampled on a coarse grid, interpolated trilinearly and
// corrected by a small 3-D convolutional network.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace agk {

constexpr int kSurrIn = 8;        // corrector input features per point
constexpr int kSurrCh = 32;       // hidden channels
constexpr int kSurrW1 = 27 * kSurrIn * kSurrCh;   // [27 taps][8 in][32 out]
constexpr int kSurrW2 = 27 * kSurrCh * kSurrCh;   // [27][32][32]
constexpr int kSurrW3 = 27 * kSurrCh;             // [27][32] (one output channel)
constexpr int kSurrWeights = kSurrW1 + kSurrW2 + kSurrW3;
constexpr float kLeakySlope = 0.125f;             // leaky ReLU of the hidden layers

// Packed BF16 weight matrices for the tensor-core convolutions: rows are
// output channels, K = tap * CIN + input channel, row stride KS (padded so
// ldmatrix row addresses fall in distinct bank groups).
constexpr int kKS8 = 232;         // CIN 8:  K = 216, padded to 224, stride 232
constexpr int kKS32 = 872;        // CIN 32: K = 864, stride 872

// Coarse far-field grid: coarse node I sits on fine index I * R.
struct SurrGeom {
  int nx, ny, nz, n2x, n2y, n2z;
  double h;
  int R;                          // fine intervals per coarse interval
  int nc[3];                      // coarse nodes covering the grid (>= 2 per axis)
  int halo;                       // extra nodes on each side of the far-field array
  int N[3];                       // far-field array extent = nc + 2 halo
};

// psi(r) in A units: r < a: pA + pB r^2 + pC r^4; r >= a: tau(min(r - shift, xmax)) / r,
// tau(x) = sum_n poly[n] E^n, E = 2^(negLambda2 * x).
struct SplitKernel {
  float a2;
  float pA, pB, pC;
  float negLambda2;
  float shift, xmax;
  float poly[6];
};

struct CoarseParams {
  const double4* atoms;
  int n_atoms, chunk, nsplit;
  SurrGeom G;
  SplitKernel K;
  double* partial;                // [nsplit][N0*N1*N2]
  double* field;                  // [N0*N1*N2] (sum of the partials, FP64)
};
cudaError_t surr_coarse_launch(const CoarseParams& P, cudaStream_t st);

// Per coarse node (nc[0]*nc[1]*nc[2]): {F, D2x, D2y, D2z}, {D4x, D4y, D4z, 0}
// (second and fourth central differences of the far field along each axis).
cudaError_t surr_deriv_launch(const double* field, const SurrGeom& G, float4* rec, cudaStream_t st);

// Per fine point: out += trilinear far field; feat = 8 BF16 corrector inputs
// (scaled by sIn).  out may be null (features only).
cudaError_t surr_feature_launch(const float4* rec, const SurrGeom& G, float sIn, float* out, uint4* feat,
                                cudaStream_t st);

// Corrector convolutions (3x3x3, zero padding, channel-last BF16 tensors).
enum ConvEpi { EPI_LEAKY = 0, EPI_GRADMASK = 1, EPI_STORE = 2, EPI_ADD = 3 };
struct ConvArgs {
  const uint16_t* in;             // [P][CIN] BF16
  const uint16_t* w;              // packed [8*NT rows][KS] BF16
  int nx, ny, nz;
  uint16_t* out16;                // EPI_LEAKY / EPI_GRADMASK: [P][32] BF16
  const uint16_t* act;            // EPI_GRADMASK: activation whose leaky-ReLU slope masks the result
  float* outF;                    // EPI_STORE / EPI_ADD: [P] FP32 (channel 0 times scale)
  float scale;
};
// cin 8 or 32; nt 4 (32 outputs) or 1 (one output, EPI_STORE / EPI_ADD).
cudaError_t surr_conv_launch(int cin, int nt, int epi, const ConvArgs& A, int sms, cudaStream_t st);

// dW[t][ci][co] += sum_p X[p + off(t)][ci] * Y[p][co] (FP32 atomics, once per CTA).
struct BwdwArgs {
  const uint16_t* x;              // [P][CIN]
  const uint16_t* y;              // [P][8*NT]
  int nx, ny, nz;
  float* dw;                      // [27][CIN][COUT], COUT = 32 (nt 4) or 1 (nt 1)
};
cudaError_t surr_bwdw_launch(int cin, int nt, const BwdwArgs& A, int sms, cudaStream_t st);

// FP32 master weights (W1 | W2 | W3) -> the five packed BF16 matrices.
struct PackedWeights {
  uint16_t* wk1;                  // [32][kKS8]   forward layer 1
  uint16_t* wk2;                  // [32][kKS32]  forward layer 2
  uint16_t* wk3;                  // [8][kKS32]   forward layer 3 (row 0)
  uint16_t* wk2t;                 // [32][kKS32]  layer 2 input gradient (taps mirrored, transposed)
  uint16_t* wk3t;                 // [32][kKS8]   layer 3 input gradient
};
cudaError_t surr_pack_launch(const float* w, const PackedWeights& pw, cudaStream_t st);

// tcgen05 forward convolutions (surr_tc.cu).  Weights in the tcgen05 layout:
// layer 1 (8 -> 32, K padded to 16 per tap), 2 (32 -> 32), 3 (32 -> 1, N padded
// to 16); surr_tc_weight_elems gives their BF16 element counts.
size_t surr_tc_weight_elems(int layer);
cudaError_t surr_pack_tc_launch(const float* w, uint16_t* w1, uint16_t* w2, uint16_t* w3, cudaStream_t st);
// layer 1 and 2: EPI_LEAKY into out16; layer 3: EPI_ADD / EPI_STORE into outF.
// Activations (in and out16) are chunk-planar [C/8][nz][ny][nx][8] (for the 8
// feature channels the same as [P][8]).
cudaError_t surr_conv_tc_launch(int layer, int epi, const ConvArgs& A, const uint16_t* wtc, unsigned* status, int sms,
                                cudaStream_t st);

// Training: loss = mean (o - y / sOut)^2; dO8[p] = (2 (o - y/sOut) / n, 0 x 7) in BF16.
cudaError_t surr_loss_launch(const float* o, const float* y, int64_t n, float invSOut, uint4* do8, double* loss,
                             cudaStream_t st);
cudaError_t surr_adam_launch(float* w, float* m, float* v, const float* g, int n, float lr, float b1, float b2,
                             float eps, int step, cudaStream_t st);
// y = a - b (FP32), and the sums of squares of y and of each feature channel (FP64, 9 values).
cudaError_t surr_residual_launch(const float* a, const float* b, float* y, const uint4* feat, int64_t n,
                                 double* sums, cudaStream_t st);
// Scale BF16 features in place by a power of two.
cudaError_t surr_scale_launch(uint4* feat, int64_t n, float s, cudaStream_t st);

// Residual probes: per CTA box, nprobe points evaluated by the exact FP64
// direct sum and compared with the surrogate map; boxes off by more than tol
// are appended to list (their direct e-map is then recomputed).
struct ProbeParams {
  const double4* atoms;
  int n_atoms;
  const double* tab;              // 8192 FP64 entries of 332/eps
  const int* items;
  const void* blocks;             // EmapBlock[nblocks]
  int nblocks, nprobe;
  int nx, ny, nz, n2x, n2y, n2z;
  double h;
  const float* map;
  float tol;
  int* flags;                     // nblocks, zeroed
  int* list;                      // nblocks
  int* count;                     // zeroed
  unsigned* maxErrBits;           // float bits of the largest probe error, zeroed
};
cudaError_t surr_probe_launch(const ProbeParams& P, cudaStream_t st);

}  // namespace agk
