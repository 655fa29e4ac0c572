// Host side of the learned far-field surrogate of the e-map: geometry and
// split kernel, the evaluation pipeline (near field, coarse far field,
// features, corrector network, residual probes, direct-sum fallback), the
// training loop on synthetic receptors, and the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/fastgrid_b200.h"
#include "ag_ctx.h"
#include "ag_host.h"
#include "ag_kernels.h"
#include "surr_kernels.h"

namespace agc {

struct SurrState {
  ag_surrogate_params par{10.0, 1.5, 0.005, 2, 1};
  bool haveWeights = false;
  std::vector<float> w;           // FP32 master weights
  float sIn = 1.f, sOut = 1.f;
  bool packedValid = false;
  DevBuf<float> dW, dGrad, dM, dV, o, tgt;
  DevBuf<uint16_t> wk1, wk2, wk3, wk2t, wk3t;
  DevBuf<uint16_t> wtc1, wtc2, wtc3;  // tcgen05 layouts
  bool useTc = true;                  // inference convolutions on tcgen05 (mma.sync when false)
  DevBuf<double> cPartial, field, tab64, loss, sums;
  DevBuf<float4> rec;
  DevBuf<uint4> feat, do8;
  DevBuf<uint16_t> a1, a2, dz1, dz2;
  DevBuf<int> flags, list, count, counter;
  DevBuf<unsigned> maxErr;
  // CTA boxes with warp-compact item order, and the atoms along a Morton curve
  std::vector<int> hItems;
  std::vector<agk::EmapBlock> hBlocks;
  DevBuf<int> dItems;
  DevBuf<agk::EmapBlock> dBlocks;
  int itemsKey[4] = {0, 0, 0, 0};
  double itemsH = 0;
  DevBuf<double4> atomsSorted;
  DevBuf<float4> tileLo, tileHi;
  uint64_t sortedVersion = ~0ull;
  std::vector<double> tab64Host;  // what S.tab64 holds
  int lastBoxes = 0;
  bool statsValid = false;
  void releaseAll() {
    for (auto* b : {&dW, &dGrad, &dM, &dV, &o, &tgt}) b->release();
    for (auto* b : {&wk1, &wk2, &wk3, &wk2t, &wk3t, &a1, &a2, &dz1, &dz2, &wtc1, &wtc2, &wtc3}) b->release();
    for (auto* b : {&cPartial, &field, &tab64, &loss, &sums}) b->release();
    rec.release();
    feat.release();
    do8.release();
    for (auto* b : {&flags, &list, &count, &counter, &dItems}) b->release();
    maxErr.release();
    dBlocks.release();
    atomsSorted.release();
    tileLo.release();
    tileHi.release();
  }
};

void surrUseTc(ag_ctx* c, bool on);

void surrFree(SurrState* s) {
  if (!s) return;
  s->releaseAll();
  delete s;
}

namespace {

SurrState& surrOf(ag_ctx* c) {
  if (!c->surr) c->surr = new SurrState();
  return *c->surr;
}

// ---------------------------------------------------------------------------
// Split kernel psi and coarse geometry
// ---------------------------------------------------------------------------
constexpr double kLambda = 0.3153767175;  // per A (autogrid.h:233-239)
constexpr double kShift = 0.005;          // half a 0.01 A bin
constexpr double kXmax = 81.91;           // the table's last bin (8191)

struct SplitCoeffs {
  double poly[6];
  double A, B, C;                         // psi(r) = A + B r^2 + C r^4 inside a
};

// 332/eps as the series sum_n poly[n] E^n, E = exp(-lambda x):
// 332 (1 + a E) / (78.4 - c E) = (332/78.4)(1 + a E) sum_n (c/78.4)^n E^n.
void seriesCoeffs(double poly[6]) {
  const double a = 7.7839, rho = 66.57180475 / 78.4, g0 = 332.0 / 78.4;
  double rp = 1.0;
  poly[0] = g0;
  for (int n = 1; n < 6; n++) {
    const double prev = rp;
    rp *= rho;
    poly[n] = g0 * (rp + a * prev);
  }
}

double tauOf(double x, const double poly[6]) {
  const double E = std::exp(-kLambda * x);
  double t = poly[5];
  for (int n = 4; n >= 0; n--) t = t * E + poly[n];
  return t;
}

double gOuter(double r, const double poly[6]) { return tauOf(std::min(r - kShift, kXmax), poly) / r; }

SplitCoeffs splitCoeffs(double a) {
  SplitCoeffs s{};
  seriesCoeffs(s.poly);
  const double h = 1e-3;
  const double gm = gOuter(a - h, s.poly), g0 = gOuter(a, s.poly), gp = gOuter(a + h, s.poly);
  const double g1 = (gp - gm) / (2 * h), g2 = (gp - 2 * g0 + gm) / (h * h);
  // psi = A + B r^2 + C r^4 with psi, psi', psi'' equal to g's at r = a.
  s.C = (a * g2 - g1) / (8 * a * a * a);
  s.B = (g2 - 12 * s.C * a * a) / 2;
  s.A = g0 - s.B * a * a - s.C * a * a * a * a;
  return s;
}

agk::SplitKernel splitKernel(double a) {
  const SplitCoeffs s = splitCoeffs(a);
  agk::SplitKernel K{};
  K.a2 = (float)(a * a);
  K.pA = (float)s.A;
  K.pB = (float)s.B;
  K.pC = (float)s.C;
  K.negLambda2 = (float)(-kLambda / std::log(2.0));
  K.shift = (float)kShift;
  K.xmax = (float)kXmax;
  for (int n = 0; n < 6; n++) K.poly[n] = (float)s.poly[n];
  return K;
}

agk::SurrGeom makeGeom(const ag_grid& g, double coarse) {
  agk::SurrGeom G{};
  G.nx = g.nx;
  G.ny = g.ny;
  G.nz = g.nz;
  G.n2x = g.nx / 2;
  G.n2y = g.ny / 2;
  G.n2z = g.nz / 2;
  G.h = g.spacing;
  G.R = std::max(1, (int)std::lround(coarse / g.spacing));
  const int n[3] = {g.nx, g.ny, g.nz};
  G.halo = 2;
  for (int d = 0; d < 3; d++) {
    G.nc[d] = std::max(2, (n[d] - 1 + G.R - 1) / G.R + 1);
    G.N[d] = G.nc[d] + 2 * G.halo;
  }
  return G;
}

int sms(ag_ctx* c) {
  int v = 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, c->device);
  return v;
}

// ---------------------------------------------------------------------------
// Buffers and weights
// ---------------------------------------------------------------------------
int ensureNet(SurrState& S, int64_t np) {
  CK(S.feat.ensure(np));
  CK(S.a1.ensure((size_t)np * 32));
  CK(S.a2.ensure((size_t)np * 32));
  CK(S.o.ensure(np));
  return AG_OK;
}

int ensureTrain(SurrState& S, int64_t np) {
  CK(S.dz1.ensure((size_t)np * 32));
  CK(S.dz2.ensure((size_t)np * 32));
  CK(S.do8.ensure(np));
  CK(S.tgt.ensure(np));
  CK(S.dGrad.ensure(agk::kSurrWeights));
  CK(S.loss.ensure(1));
  return AG_OK;
}

int packWeights(ag_ctx* c, SurrState& S) {
  if (S.packedValid) return AG_OK;
  CK(S.dW.ensure(agk::kSurrWeights));
  CK(S.wk1.ensure(32 * agk::kKS8));
  CK(S.wk2.ensure(32 * agk::kKS32));
  CK(S.wk3.ensure(8 * agk::kKS32));
  CK(S.wk2t.ensure(32 * agk::kKS32));
  CK(S.wk3t.ensure(32 * agk::kKS8));
  CK(cudaMemcpyAsync(S.dW.p, S.w.data(), sizeof(float) * agk::kSurrWeights, cudaMemcpyHostToDevice, c->stream));
  agk::PackedWeights pw{S.wk1.p, S.wk2.p, S.wk3.p, S.wk2t.p, S.wk3t.p};
  CK(agk::surr_pack_launch(S.dW.p, pw, c->stream));
  CK(S.wtc1.ensure(agk::surr_tc_weight_elems(1)));
  CK(S.wtc2.ensure(agk::surr_tc_weight_elems(2)));
  CK(S.wtc3.ensure(agk::surr_tc_weight_elems(3)));
  CK(agk::surr_pack_tc_launch(S.dW.p, S.wtc1.p, S.wtc2.p, S.wtc3.p, c->stream));
  c->launches += 2;
  CK(cudaStreamSynchronize(c->stream));
  S.packedValid = true;
  return AG_OK;
}

// Round to BF16 (nearest, ties to even) and back.
float bf16Round(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  if ((b & 0x7F800000u) != 0x7F800000u) b = (b + 0x7FFFu + ((b >> 16) & 1u)) & 0xFFFF0000u;
  else b &= 0xFFFF0000u;
  float r;
  memcpy(&r, &b, 4);
  return r;
}

// Spread the low 10 bits of v to every third bit (Morton interleave).
uint32_t spread3(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Work items (warp-compact order, CTA tiles of 1 x 16 x 16 items: the near-field
// kernel's box shape) and the Morton-sorted atoms with the bounding box of
// every 256-atom tile, for the staged job.
int surrPrepare(ag_ctx* c, SurrState& S) {
  const ag_grid& g = c->grid;
  static const int kTile[3] = {1, 16, 16};
  const int key[4] = {g.nx, g.ny, g.nz, kTile[0] * 10000 + kTile[1] * 100 + kTile[2]};
  if (memcmp(key, S.itemsKey, sizeof key) != 0 || S.itemsH != g.spacing) {
    makeItems(g, kTile, 1, S.hItems, S.hBlocks);
    CK(S.dItems.ensure(S.hItems.size()));
    CK(S.dBlocks.ensure(S.hBlocks.size()));
    CK(cudaMemcpyAsync(S.dItems.p, S.hItems.data(), sizeof(int) * S.hItems.size(), cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaMemcpyAsync(S.dBlocks.p, S.hBlocks.data(), sizeof(agk::EmapBlock) * S.hBlocks.size(),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    memcpy(S.itemsKey, key, sizeof key);
    S.itemsH = g.spacing;
  }
  if (S.sortedVersion != c->atomsVersion) {
    const int n = c->nAtoms;
    if (c->atomsHostVersion != c->atomsVersion) {  // host copy of the staged atoms, read back once per staging
      c->atomsHost.resize(4 * (size_t)n);
      if (n) CK(cudaMemcpyAsync(c->atomsHost.data(), c->atoms.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost,
                                c->stream));
      CK(cudaStreamSynchronize(c->stream));
      c->atomsHostVersion = c->atomsVersion;
    }
    const double* x = c->atomsHost.data();
    std::vector<std::pair<uint32_t, int>> order(n);
    for (int i = 0; i < n; i++) {
      uint32_t k = 0;
      for (int d = 0; d < 3; d++) {
        const int q = std::min(1023, std::max(0, (int)std::floor((x[4 * (size_t)i + d] + 1024.0) * 0.5)));
        k |= spread3((uint32_t)q) << d;
      }
      order[i] = {k, i};
    }
    std::sort(order.begin(), order.end());
    std::vector<double> sorted(4 * (size_t)n);
    for (int i = 0; i < n; i++) memcpy(&sorted[4 * (size_t)i], &x[4 * (size_t)order[i].second], 4 * sizeof(double));
    const int nt = (n + 255) / 256;
    std::vector<float4> lo(std::max(nt, 1)), hi(std::max(nt, 1));
    for (int t = 0; t < nt; t++) {
      float l[3] = {3e38f, 3e38f, 3e38f}, u[3] = {-3e38f, -3e38f, -3e38f};
      for (int i = 256 * t; i < std::min(n, 256 * t + 256); i++)
        for (int d = 0; d < 3; d++) {
          const double v = sorted[4 * (size_t)i + d];
          l[d] = std::min(l[d], std::nextafter((float)v, -3e38f));
          u[d] = std::max(u[d], std::nextafter((float)v, 3e38f));
        }
      lo[t] = make_float4(l[0], l[1], l[2], 0.f);
      hi[t] = make_float4(u[0], u[1], u[2], 0.f);
    }
    CK(S.atomsSorted.ensure(std::max(n, 1)));
    CK(S.tileLo.ensure(lo.size()));
    CK(S.tileHi.ensure(hi.size()));
    if (n)
      CK(cudaMemcpyAsync(S.atomsSorted.p, sorted.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(S.tileLo.p, lo.data(), sizeof(float4) * lo.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(S.tileHi.p, hi.data(), sizeof(float4) * hi.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    S.sortedVersion = c->atomsVersion;
  }
  return AG_OK;
}

// ---------------------------------------------------------------------------
// Pipeline stages
// ---------------------------------------------------------------------------
// Near field + trilinear far field into dBase, corrector inputs into dFeat.
int surrBase(ag_ctx* c, SurrState& S, float* dBase, uint4* dFeat, float sIn) {
  const ag_grid& g = c->grid;
  const int64_t np = c->npoints();
  const double a = S.par.r_near;
  const agk::SurrGeom G = makeGeom(g, S.par.coarse_spacing);
  const agk::SplitKernel K = splitKernel(a);
  const SplitCoeffs sc = splitCoeffs(a);
  // near field (exact bins, Kahan) with psi subtracted
  if (int e = surrPrepare(c, S)) return e;
  if (c->nAtoms == 0) {
    CK(cudaMemsetAsync(dBase, 0, sizeof(float) * np, c->stream));
  } else {
    agk::EmapParams P;
    if (int e = buildEmapParams(c, dBase, true, P)) return e;
    P.checksum = nullptr;
    P.atoms = S.atomsSorted.p;
    P.items = S.dItems.p;
    P.blocks = S.dBlocks.p;
    P.nblocks = (int)S.hBlocks.size();
    P.tileLo = S.tileLo.p;
    P.tileHi = S.tileHi.p;
    P.rnear2 = (float)((100.0 * a) * (100.0 * a));
    P.rcut2 = P.rnear2;
    P.psi[0] = (float)(sc.A / 100.0);
    P.psi[1] = (float)(sc.B * 1e-6);
    P.psi[2] = (float)(sc.C * 1e-10);
    CK(agk::emap_near_launch(P, P.nblocks * P.nsplit, c->stream));
    c->launches += P.nsplit > 1 ? 2 : 1;
  }
  // coarse far field
  const int64_t NN = (int64_t)G.N[0] * G.N[1] * G.N[2];
  const int64_t nodeBlocks = (NN + 511) / 512;  // surr_coarse_kernel: 512 nodes per CTA
  int nsplit = (int)std::max<int64_t>(1, (8 * (int64_t)sms(c) + nodeBlocks - 1) / nodeBlocks);
  nsplit = std::min(nsplit, std::max(1, (c->nAtoms + 255) / 256));
  int chunk = (c->nAtoms + nsplit - 1) / nsplit;
  chunk = std::max(256, ((chunk + 255) / 256) * 256);
  nsplit = std::max(1, (c->nAtoms + chunk - 1) / chunk);
  CK(S.cPartial.ensure((size_t)nsplit * NN));
  CK(S.field.ensure(NN));
  agk::CoarseParams CP{};
  CP.atoms = c->atoms.p;
  CP.n_atoms = c->nAtoms;
  CP.chunk = chunk;
  CP.nsplit = nsplit;
  CP.G = G;
  CP.K = K;
  CP.partial = S.cPartial.p;
  CP.field = S.field.p;
  CK(agk::surr_coarse_launch(CP, c->stream));
  c->launches += 2;
  const int64_t nc = (int64_t)G.nc[0] * G.nc[1] * G.nc[2];
  CK(S.rec.ensure(2 * nc));
  CK(agk::surr_deriv_launch(S.field.p, G, S.rec.p, c->stream));
  CK(agk::surr_feature_launch(S.rec.p, G, sIn, dBase, dFeat, c->stream));
  c->launches += 2;
  return AG_OK;
}

// Corrector forward: outF = scale * net(feat) (add: += instead of =).
// training: keep the activations in the [P][32] layout the backward kernels
// read (mma.sync forward); otherwise tcgen05 when enabled (chunk-planar).
int surrNet(ag_ctx* c, SurrState& S, const agk::SurrGeom& G, const uint4* feat, float* outF, bool add, float scale,
            bool training) {
  if (int e = packWeights(c, S)) return e;
  const int n = sms(c);
  agk::ConvArgs A{};
  A.nx = G.nx;
  A.ny = G.ny;
  A.nz = G.nz;
  if (S.useTc && !training) {  // tcgen05: accumulators in tensor memory
    A.in = reinterpret_cast<const uint16_t*>(feat);
    A.out16 = S.a1.p;
    CK(agk::surr_conv_tc_launch(1, agk::EPI_LEAKY, A, S.wtc1.p, c->status.p, n, c->stream));
    A.in = S.a1.p;
    A.out16 = S.a2.p;
    CK(agk::surr_conv_tc_launch(2, agk::EPI_LEAKY, A, S.wtc2.p, c->status.p, n, c->stream));
    A.in = S.a2.p;
    A.out16 = nullptr;
    A.outF = outF;
    A.scale = scale;
    CK(agk::surr_conv_tc_launch(3, add ? agk::EPI_ADD : agk::EPI_STORE, A, S.wtc3.p, c->status.p, n, c->stream));
    c->launches += 3;
    return AG_OK;
  }
  A.in = reinterpret_cast<const uint16_t*>(feat);
  A.w = S.wk1.p;
  A.out16 = S.a1.p;
  CK(agk::surr_conv_launch(8, 4, agk::EPI_LEAKY, A, n, c->stream));
  A.in = S.a1.p;
  A.w = S.wk2.p;
  A.out16 = S.a2.p;
  CK(agk::surr_conv_launch(32, 4, agk::EPI_LEAKY, A, n, c->stream));
  A.in = S.a2.p;
  A.w = S.wk3.p;
  A.out16 = nullptr;
  A.outF = outF;
  A.scale = scale;
  CK(agk::surr_conv_launch(32, 1, add ? agk::EPI_ADD : agk::EPI_STORE, A, n, c->stream));
  c->launches += 3;
  return AG_OK;
}

// Corrector backward from S.do8 (after a forward on feat): gradient into S.dGrad.
int surrBackward(ag_ctx* c, SurrState& S, const agk::SurrGeom& G, const uint4* feat) {
  const int n = sms(c);
  CK(cudaMemsetAsync(S.dGrad.p, 0, sizeof(float) * agk::kSurrWeights, c->stream));
  agk::BwdwArgs B{};
  B.nx = G.nx;
  B.ny = G.ny;
  B.nz = G.nz;
  B.x = S.a2.p;
  B.y = reinterpret_cast<const uint16_t*>(S.do8.p);
  B.dw = S.dGrad.p + agk::kSurrW1 + agk::kSurrW2;
  CK(agk::surr_bwdw_launch(32, 1, B, n, c->stream));
  agk::ConvArgs A{};
  A.nx = G.nx;
  A.ny = G.ny;
  A.nz = G.nz;
  A.in = reinterpret_cast<const uint16_t*>(S.do8.p);
  A.w = S.wk3t.p;
  A.act = S.a2.p;
  A.out16 = S.dz2.p;
  CK(agk::surr_conv_launch(8, 4, agk::EPI_GRADMASK, A, n, c->stream));
  B.x = S.a1.p;
  B.y = S.dz2.p;
  B.dw = S.dGrad.p + agk::kSurrW1;
  CK(agk::surr_bwdw_launch(32, 4, B, n, c->stream));
  A.in = S.dz2.p;
  A.w = S.wk2t.p;
  A.act = S.a1.p;
  A.out16 = S.dz1.p;
  CK(agk::surr_conv_launch(32, 4, agk::EPI_GRADMASK, A, n, c->stream));
  B.x = reinterpret_cast<const uint16_t*>(feat);
  B.y = S.dz1.p;
  B.dw = S.dGrad.p;
  CK(agk::surr_bwdw_launch(8, 4, B, n, c->stream));
  c->launches += 5;
  return AG_OK;
}

// ---------------------------------------------------------------------------
// Synthetic receptors for training and evaluation
// ---------------------------------------------------------------------------
// A globule at the C0 density (2000 atoms in 20 A), the C0 type mix, charges
// N(0, 0.2) clipped at 0.7 with net 0; centred on its centroid; w = 0.1465 q.
int makeReceptor(uint64_t seed, int n, std::vector<double>& xyzw) {
  ag_synth_params sp{};
  sp.seed = seed;
  sp.n_atoms = n;
  const double r = 20.0 * std::cbrt(n / 2000.0);
  sp.semi_axes[0] = sp.semi_axes[1] = sp.semi_axes[2] = r;
  sp.frac_C = 0.45;
  sp.frac_OA = 0.18;
  sp.frac_N = 0.15;
  sp.frac_HD = 0.15;
  sp.frac_A = 0.05;
  sp.frac_SA = 0.02;
  sp.charge_sigma = 0.2;
  sp.charge_clip = 0.7;
  sp.net_charge = 0.0;
  std::vector<double> x;
  std::vector<int> t;
  std::vector<long long> k;
  if (int e = ag::synthReceptor(&sp, x, t, k)) return e;
  double cm[3] = {0, 0, 0};
  for (int i = 0; i < n; i++)
    for (int d = 0; d < 3; d++) cm[d] += x[3 * (size_t)i + d];
  for (int d = 0; d < 3; d++) cm[d] /= n;
  xyzw.resize(4 * (size_t)n);
  for (int i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) xyzw[4 * (size_t)i + d] = x[3 * (size_t)i + d] - cm[d];
    xyzw[4 * (size_t)i + 3] = (k[i] / 1000.0) * 0.1465;
  }
  return AG_OK;
}

struct Rng64 {  // splitmix64
  uint64_t s;
  explicit Rng64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {
    const double u1 = std::max(uni(), 1e-300), u2 = uni();
    return std::sqrt(-2 * std::log(u1)) * std::cos(2 * M_PI * u2);
  }
};

std::vector<double> dddTable() {
  std::vector<double> t(8192);
  for (int i = 0; i < 8192; i++) t[i] = ag::distDepDielInv(i / 100.0);
  return t;
}

constexpr char kMagic[8] = {'F', 'G', 'S', 'U', 'R', 'R', '1', 0};

}  // namespace

// The e-map of the staged job by the surrogate, into dOut.
int runEmapSurrogate(ag_ctx* c, float* dOut) {
  if (!c->ddd) return fail(AG_E_INVALID, "the e-map surrogate needs the distance-dependent dielectric");
  SurrState& S = surrOf(c);
  if (S.par.use_corrector && !S.haveWeights)
    return fail(AG_E_INVALID, "no corrector weights: ag_surrogate_load or ag_surrogate_train first "
                              "(or turn the corrector off)");
  const int64_t np = c->npoints();
  const agk::SurrGeom G = makeGeom(c->grid, S.par.coarse_spacing);
  CK(S.feat.ensure(np));
  if (int e = surrBase(c, S, dOut, S.feat.p, S.sIn)) return e;
  if (S.par.use_corrector) {
    if (int e = ensureNet(S, np)) return e;
    if (int e = surrNet(c, S, G, S.feat.p, dOut, true, S.sOut, false)) return e;
  }
  S.lastBoxes = (int)S.hBlocks.size();
  S.statsValid = false;
  if (S.par.probe_tol > 0 && S.par.probes_per_box > 0 && c->nAtoms > 0) {
    const int nb = (int)S.hBlocks.size();
    CK(S.flags.ensure(nb));
    CK(S.list.ensure(nb));
    CK(S.count.ensure(1));
    CK(S.counter.ensure(1));
    CK(S.maxErr.ensure(1));
    if (S.tab64Host != c->epsHost) {
      CK(S.tab64.ensure(8192));
      CK(cudaMemcpyAsync(S.tab64.p, c->epsHost.data(), sizeof(double) * 8192, cudaMemcpyHostToDevice, c->stream));
      S.tab64Host = c->epsHost;
    }
    CK(cudaMemsetAsync(S.flags.p, 0, sizeof(int) * nb, c->stream));
    CK(cudaMemsetAsync(S.count.p, 0, sizeof(int), c->stream));
    CK(cudaMemsetAsync(S.maxErr.p, 0, sizeof(unsigned), c->stream));
    agk::ProbeParams Q{};
    Q.atoms = c->atoms.p;
    Q.n_atoms = c->nAtoms;
    Q.tab = S.tab64.p;
    Q.items = S.dItems.p;
    Q.blocks = S.dBlocks.p;
    Q.nblocks = nb;
    Q.nprobe = S.par.probes_per_box;
    Q.nx = c->grid.nx;
    Q.ny = c->grid.ny;
    Q.nz = c->grid.nz;
    Q.n2x = Q.nx / 2;
    Q.n2y = Q.ny / 2;
    Q.n2z = Q.nz / 2;
    Q.h = c->grid.spacing;
    Q.map = dOut;
    Q.tol = (float)S.par.probe_tol;
    Q.flags = S.flags.p;
    Q.list = S.list.p;
    Q.count = S.count.p;
    Q.maxErrBits = S.maxErr.p;
    CK(agk::surr_probe_launch(Q, c->stream));
    agk::EmapParams P;
    if (int e = buildEmapParams(c, dOut, false, P)) return e;
    P.checksum = nullptr;
    P.items = S.dItems.p;
    P.blocks = S.dBlocks.p;
    P.nblocks = nb;
    CK(agk::emap_list_launch(P, S.list.p, S.count.p, S.counter.p, std::min(nb, agk::kEmapCtasPerSm * sms(c)), c->stream));
    c->launches += 2;
    S.statsValid = true;
  }
  return AG_OK;
}

void surrUseTc(ag_ctx* c, bool on) { surrOf(c).useTc = on; }

}  // namespace agc

using namespace agc;

extern "C" int ag_surrogate_set(ag_ctx* c, const ag_surrogate_params* p) {
  if (!c) return fail(AG_E_INVALID, "null context");
  SurrState& S = surrOf(c);
  if (!p) {
    S.par = ag_surrogate_params{10.0, 1.5, 0.005, 2, 1};
    return AG_OK;
  }
  if (!(p->r_near >= 4.0 && p->r_near <= 30.0)) return fail(AG_E_INVALID, "r_near must be in [4, 30] A");
  if (!(p->coarse_spacing > 0 && p->coarse_spacing <= 4.0)) return fail(AG_E_INVALID, "coarse_spacing must be in (0, 4] A");
  if (p->probes_per_box < 0 || p->probes_per_box > 64) return fail(AG_E_INVALID, "probes_per_box must be 0..64");
  S.par = *p;
  return AG_OK;
}

extern "C" int ag_surrogate_weights(ag_ctx* c, const float* w_in, const double* s_in, float* w_out, double* s_out) {
  if (!c) return fail(AG_E_INVALID, "null context");
  SurrState& S = surrOf(c);
  if (w_in) {
    for (int i = 0; i < agk::kSurrWeights; i++)
      if (!std::isfinite(w_in[i])) return fail(AG_E_INVALID, "non-finite weight %d", i);
    S.w.assign(w_in, w_in + agk::kSurrWeights);
    S.haveWeights = true;
    S.packedValid = false;
  }
  if (s_in) {
    if (!(s_in[0] > 0 && s_in[1] > 0 && std::isfinite(s_in[0]) && std::isfinite(s_in[1])))
      return fail(AG_E_INVALID, "scales must be positive");
    S.sIn = (float)s_in[0];
    S.sOut = (float)s_in[1];
  }
  if (w_out) {
    if (!S.haveWeights) return fail(AG_E_INVALID, "no weights");
    std::copy(S.w.begin(), S.w.end(), w_out);
  }
  if (s_out) {
    s_out[0] = S.sIn;
    s_out[1] = S.sOut;
  }
  return AG_OK;
}

extern "C" int ag_surrogate_save(ag_ctx* c, const char* path) {
  if (!c || !path) return fail(AG_E_INVALID, "null argument");
  SurrState& S = surrOf(c);
  if (!S.haveWeights) return fail(AG_E_INVALID, "no weights to save");
  FILE* f = fopen(path, "wb");
  if (!f) return fail(AG_E_HOST, "cannot write %s", path);
  const uint32_t hdr[4] = {1u, (uint32_t)agk::kSurrW1, (uint32_t)agk::kSurrW2, (uint32_t)agk::kSurrW3};
  const float sc[4] = {S.sIn, S.sOut, (float)S.par.r_near, (float)S.par.coarse_spacing};
  std::vector<uint16_t> b(agk::kSurrWeights);
  for (int i = 0; i < agk::kSurrWeights; i++) {
    const float r = bf16Round(S.w[i]);
    uint32_t u;
    memcpy(&u, &r, 4);
    b[i] = (uint16_t)(u >> 16);
  }
  bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(hdr, 4, 4, f) == 4 && fwrite(sc, 4, 4, f) == 4 &&
            fwrite(b.data(), 2, b.size(), f) == b.size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(AG_E_HOST, "short write to %s", path);
  return AG_OK;
}

extern "C" int ag_surrogate_load(ag_ctx* c, const char* path) {
  if (!c || !path) return fail(AG_E_INVALID, "null argument");
  FILE* f = fopen(path, "rb");
  if (!f) return fail(AG_E_HOST, "cannot open %s", path);
  char magic[8];
  uint32_t hdr[4];
  float sc[4];
  std::vector<uint16_t> b(agk::kSurrWeights);
  const bool ok = fread(magic, 1, 8, f) == 8 && fread(hdr, 4, 4, f) == 4 && fread(sc, 4, 4, f) == 4 &&
                  fread(b.data(), 2, b.size(), f) == b.size();
  fclose(f);
  if (!ok || memcmp(magic, kMagic, 8) != 0 || hdr[0] != 1u || hdr[1] != (uint32_t)agk::kSurrW1 ||
      hdr[2] != (uint32_t)agk::kSurrW2 || hdr[3] != (uint32_t)agk::kSurrW3)
    return fail(AG_E_HOST, "%s is not a corrector weights file of this layout", path);
  if (!(sc[0] > 0 && sc[1] > 0 && std::isfinite(sc[0]) && std::isfinite(sc[1])))
    return fail(AG_E_HOST, "%s: bad scales", path);
  SurrState& S = surrOf(c);
  S.w.resize(agk::kSurrWeights);
  for (int i = 0; i < agk::kSurrWeights; i++) {
    const uint32_t u = (uint32_t)b[i] << 16;
    memcpy(&S.w[i], &u, 4);
    if (!std::isfinite(S.w[i])) return fail(AG_E_HOST, "%s: non-finite weight", path);
  }
  S.sIn = sc[0];
  S.sOut = sc[1];
  S.par.r_near = sc[2];
  S.par.coarse_spacing = sc[3];
  S.haveWeights = true;
  S.packedValid = false;
  return AG_OK;
}

extern "C" int ag_emap_surrogate(ag_ctx* c, const ag_grid* g, int n, const double* xyzw, const double* inv_eps,
                                 float* out, ag_surrogate_stats* stats) {
  if (!c || !out) return fail(AG_E_INVALID, "null argument");
  if (!inv_eps) return fail(AG_E_INVALID, "the e-map surrogate needs the distance-dependent dielectric table");
  c->haveJob = false;
  c->haveAff = false;
  c->nMaps = 0;
  if (int e = stageEmap(c, g, n, xyzw, inv_eps, false)) return e;
  CK(c->maps.ensure((size_t)2 * c->npoints()));
  if (int e = runEmapSurrogate(c, c->maps.p)) return e;
  CK(cudaMemcpyAsync(out, c->maps.p, sizeof(float) * c->npoints(), cudaMemcpyDeviceToHost, c->stream));
  if (int e = checkStatus(c)) return e;
  if (stats) return ag_surrogate_last_stats(c, stats);
  return AG_OK;
}

extern "C" int ag_surrogate_last_stats(ag_ctx* c, ag_surrogate_stats* st) {
  if (!c || !st) return fail(AG_E_INVALID, "null argument");
  SurrState& S = surrOf(c);
  st->boxes = S.lastBoxes;
  st->fallback_boxes = 0;
  st->probe_max_err = 0;
  if (S.statsValid) {
    int cnt = 0;
    unsigned bits = 0;
    CK(cudaMemcpyAsync(&cnt, S.count.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&bits, S.maxErr.p, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    float e;
    memcpy(&e, &bits, 4);
    st->fallback_boxes = cnt;
    st->probe_max_err = e;
  }
  return AG_OK;
}

extern "C" int ag_surrogate_features(ag_ctx* c, const ag_grid* g, int n, const double* xyzw, const double* inv_eps,
                                     float* features, float* base) {
  if (!c || !inv_eps) return fail(AG_E_INVALID, "null argument");
  c->haveJob = false;
  c->haveAff = false;
  c->nMaps = 0;
  if (int e = stageEmap(c, g, n, xyzw, inv_eps, false)) return e;
  SurrState& S = surrOf(c);
  const int64_t np = c->npoints();
  CK(c->maps.ensure((size_t)2 * np));
  CK(S.feat.ensure(np));
  if (int e = surrBase(c, S, c->maps.p, S.feat.p, S.sIn)) return e;
  std::vector<uint4> f(np);
  CK(cudaMemcpyAsync(f.data(), S.feat.p, sizeof(uint4) * np, cudaMemcpyDeviceToHost, c->stream));
  if (base) CK(cudaMemcpyAsync(base, c->maps.p, sizeof(float) * np, cudaMemcpyDeviceToHost, c->stream));
  if (int e = checkStatus(c)) return e;
  if (features)
    for (int64_t i = 0; i < np; i++) {
      const uint32_t w[4] = {f[i].x, f[i].y, f[i].z, f[i].w};
      for (int k = 0; k < 4; k++) {
        const uint32_t lo = w[k] << 16, hi = w[k] & 0xFFFF0000u;
        memcpy(&features[8 * i + 2 * k], &lo, 4);
        memcpy(&features[8 * i + 2 * k + 1], &hi, 4);
      }
    }
  return AG_OK;
}

extern "C" int ag_surrogate_net_grad(ag_ctx* c, const ag_grid* g, const float* features, const float* target, float* o,
                                     float* grad, double* loss) {
  if (!c || !g || !features) return fail(AG_E_INVALID, "null argument");
  if (int e = checkGrid(g)) return e;
  SurrState& S = surrOf(c);
  if (!S.haveWeights) return fail(AG_E_INVALID, "no weights");
  CK(cudaSetDevice(c->device));
  const int64_t np = (int64_t)g->nx * g->ny * g->nz;
  if (int e = ensureNet(S, np)) return e;
  if (target)
    if (int e = ensureTrain(S, np)) return e;
  std::vector<uint4> f(np);
  for (int64_t i = 0; i < np; i++) {
    uint32_t w[4];
    for (int k = 0; k < 4; k++) {
      const float lo = bf16Round(features[8 * i + 2 * k]), hi = bf16Round(features[8 * i + 2 * k + 1]);
      uint32_t a, b;
      memcpy(&a, &lo, 4);
      memcpy(&b, &hi, 4);
      w[k] = (a >> 16) | (b & 0xFFFF0000u);
    }
    f[i] = make_uint4(w[0], w[1], w[2], w[3]);
  }
  CK(cudaMemcpyAsync(S.feat.p, f.data(), sizeof(uint4) * np, cudaMemcpyHostToDevice, c->stream));
  agk::SurrGeom G{};
  G.nx = g->nx;
  G.ny = g->ny;
  G.nz = g->nz;
  if (int e = surrNet(c, S, G, S.feat.p, S.o.p, false, 1.f, true)) return e;
  if (target) {
    CK(cudaMemcpyAsync(S.tgt.p, target, sizeof(float) * np, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(S.loss.p, 0, sizeof(double), c->stream));
    CK(agk::surr_loss_launch(S.o.p, S.tgt.p, np, 1.f / S.sOut, S.do8.p, S.loss.p, c->stream));
    if (int e = surrBackward(c, S, G, S.feat.p)) return e;
    c->launches += 1;
  }
  if (o) CK(cudaMemcpyAsync(o, S.o.p, sizeof(float) * np, cudaMemcpyDeviceToHost, c->stream));
  if (target && grad)
    CK(cudaMemcpyAsync(grad, S.dGrad.p, sizeof(float) * agk::kSurrWeights, cudaMemcpyDeviceToHost, c->stream));
  double L = 0;
  if (target) CK(cudaMemcpyAsync(&L, S.loss.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (loss) *loss = L / (double)np;
  return AG_OK;
}

extern "C" int ag_surrogate_receptor(uint64_t seed, int n, double* xyzw) {
  if (n <= 0 || !xyzw) return fail(AG_E_INVALID, "bad argument");
  std::vector<double> v;
  if (int e = makeReceptor(seed, n, v)) return fail(e, "receptor generation failed");
  std::copy(v.begin(), v.end(), xyzw);
  return AG_OK;
}

extern "C" int ag_surrogate_train(ag_ctx* c, const ag_surrogate_train_params* tp, ag_surrogate_train_report* rep,
                                  double* lossPerEpoch) {
  if (!c || !tp) return fail(AG_E_INVALID, "null argument");
  if (tp->n_receptors < 1 || tp->min_atoms < 1 || tp->max_atoms < tp->min_atoms || tp->points < 2 ||
      tp->points > 513 || !(tp->spacing > 0) || tp->epochs < 1 || !(tp->lr > 0))
    return fail(AG_E_INVALID, "bad training parameters");
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  SurrState& S = surrOf(c);
  CK(cudaSetDevice(c->device));
  const int nr = tp->n_receptors;
  // receptors (host, in parallel; each depends on its seed only)
  std::vector<std::vector<double>> recs(nr);
  std::vector<int> natoms(nr);
  {
    Rng64 rng(tp->seed * 0x2545F4914F6CDD1Dull + 17);
    for (int i = 0; i < nr; i++)
      natoms[i] = (int)std::lround(std::exp(std::log((double)tp->min_atoms) +
                                            rng.uni() * (std::log((double)tp->max_atoms) - std::log((double)tp->min_atoms))));
    std::atomic<int> next{0}, bad{0};
    const int nth = std::max(1, std::min(nr, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (int k = 0; k < nth; k++)
      th.emplace_back([&] {
        for (int i; (i = next++) < nr;)
          if (makeReceptor(tp->seed * 1000003ull + (uint64_t)i, natoms[i], recs[i]) != AG_OK) bad++;
      });
    for (auto& t : th) t.join();
    if (bad) return fail(AG_E_HOST, "synthetic receptor generation failed");
  }
  const ag_grid grid{tp->points, tp->points, tp->points, tp->spacing};
  const int64_t np = (int64_t)grid.nx * grid.ny * grid.nz;
  const std::vector<double> eps = dddTable();
  DevBuf<uint4> featAll;
  DevBuf<float> yAll, direct;
  CK(featAll.ensure((size_t)nr * np));
  CK(yAll.ensure((size_t)nr * np));
  CK(direct.ensure(np));
  CK(S.sums.ensure(9));
  CK(cudaMemsetAsync(S.sums.p, 0, sizeof(double) * 9, c->stream));
  CK(c->maps.ensure((size_t)2 * np));
  const agk::SurrGeom G = makeGeom(grid, S.par.coarse_spacing);
  auto cleanup = [&] {
    featAll.release();
    yAll.release();
    direct.release();
  };
  for (int i = 0; i < nr; i++) {
    c->haveJob = false;
    c->haveAff = false;
    c->nMaps = 0;
    int e = stageEmap(c, &grid, natoms[i], recs[i].data(), eps.data(), false);
    if (!e) e = runEmap(c, direct.p);
    if (!e) e = surrBase(c, S, c->maps.p, featAll.p + (size_t)i * np, 1.f);
    if (!e && agk::surr_residual_launch(direct.p, c->maps.p, yAll.p + (size_t)i * np, featAll.p + (size_t)i * np, np,
                                        S.sums.p, c->stream) != cudaSuccess)
      e = fail(AG_E_CUDA, "residual kernel launch failed");
    if (!e) e = checkStatus(c);
    if (e) {
      cleanup();
      return e;
    }
    c->launches += 1;
  }
  double sums[9];
  CK(cudaMemcpy(sums, S.sums.p, sizeof sums, cudaMemcpyDeviceToHost));
  const double tot = (double)nr * np;
  double msF = 0;
  for (int k = 1; k < 9; k++) msF += sums[k];
  msF /= 8 * tot;
  const double msR = sums[0] / tot;
  S.sIn = (float)std::exp2(std::round(-0.5 * std::log2(std::max(msF, 1e-30))));
  S.sOut = (float)std::exp2(std::round(0.5 * std::log2(std::max(msR, 1e-30))));
  CK(agk::surr_scale_launch(featAll.p, (int64_t)nr * np, S.sIn, c->stream));
  const auto t1 = clk::now();

  // weights: He initialisation for the leaky-ReLU layers, small last layer
  S.w.assign(agk::kSurrWeights, 0.f);
  {
    Rng64 rng(tp->seed * 0x9E3779B97F4A7C15ull + 5);
    const double s1 = std::sqrt(2.0 / ((1 + agk::kLeakySlope * agk::kLeakySlope) * 27 * agk::kSurrIn));
    const double s2 = std::sqrt(2.0 / ((1 + agk::kLeakySlope * agk::kLeakySlope) * 27 * agk::kSurrCh));
    const double s3 = 0.1 * std::sqrt(1.0 / (27 * agk::kSurrCh));
    for (int i = 0; i < agk::kSurrW1; i++) S.w[i] = (float)(s1 * rng.normal());
    for (int i = 0; i < agk::kSurrW2; i++) S.w[agk::kSurrW1 + i] = (float)(s2 * rng.normal());
    for (int i = 0; i < agk::kSurrW3; i++) S.w[agk::kSurrW1 + agk::kSurrW2 + i] = (float)(s3 * rng.normal());
  }
  S.haveWeights = true;
  S.packedValid = false;
  if (int e = ensureNet(S, np)) { cleanup(); return e; }
  if (int e = ensureTrain(S, np)) { cleanup(); return e; }
  if (int e = packWeights(c, S)) { cleanup(); return e; }  // uploads the master weights into S.dW
  CK(S.dM.ensure(agk::kSurrWeights));
  CK(S.dV.ensure(agk::kSurrWeights));
  CK(cudaMemsetAsync(S.dM.p, 0, sizeof(float) * agk::kSurrWeights, c->stream));
  CK(cudaMemsetAsync(S.dV.p, 0, sizeof(float) * agk::kSurrWeights, c->stream));
  const int steps = tp->epochs * nr;
  DevBuf<double> lossSteps;
  CK(lossSteps.ensure(steps));
  CK(cudaMemsetAsync(lossSteps.p, 0, sizeof(double) * steps, c->stream));
  Rng64 shuf(tp->seed * 31 + 7);
  std::vector<int> order(nr);
  const int warm = std::min(50, steps / 10 + 1);
  agk::PackedWeights pw{S.wk1.p, S.wk2.p, S.wk3.p, S.wk2t.p, S.wk3t.p};
  int step = 0;
  for (int ep = 0; ep < tp->epochs; ep++) {
    for (int i = 0; i < nr; i++) order[i] = i;
    for (int i = nr - 1; i > 0; i--) std::swap(order[i], order[(int)(shuf.next() % (uint64_t)(i + 1))]);
    for (int k = 0; k < nr; k++, step++) {
      const int i = order[k];
      const uint4* f = featAll.p + (size_t)i * np;
      if (int e = surrNet(c, S, G, f, S.o.p, false, 1.f, true)) { cleanup(); return e; }
      CK(agk::surr_loss_launch(S.o.p, yAll.p + (size_t)i * np, np, 1.f / S.sOut, S.do8.p, lossSteps.p + step,
                               c->stream));
      if (int e = surrBackward(c, S, G, f)) { cleanup(); return e; }
      const double prog = (double)step / std::max(1, steps - 1);
      double lr = tp->lr * (step < warm ? (step + 1.0) / warm : 0.05 + 0.95 * 0.5 * (1 + std::cos(M_PI * prog)));
      CK(agk::surr_adam_launch(S.dW.p, S.dM.p, S.dV.p, S.dGrad.p, agk::kSurrWeights, (float)lr, 0.9f, 0.999f, 1e-8f,
                               step + 1, c->stream));
      CK(agk::surr_pack_launch(S.dW.p, pw, c->stream));
      c->launches += 3;
    }
  }
  std::vector<double> ls(steps);
  CK(cudaMemcpyAsync(ls.data(), lossSteps.p, sizeof(double) * steps, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(S.w.data(), S.dW.p, sizeof(float) * agk::kSurrWeights, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (auto& v : S.w) v = bf16Round(v);  // the weights the kernels use
  S.packedValid = false;
  cleanup();
  lossSteps.release();
  const auto t2 = clk::now();
  std::vector<double> per(tp->epochs, 0.0);
  for (int s = 0; s < steps; s++) per[s / nr] += ls[s] / (double)np / nr;
  if (lossPerEpoch) std::copy(per.begin(), per.end(), lossPerEpoch);
  if (rep) {
    rep->gen_seconds = std::chrono::duration<double>(t1 - t0).count();
    rep->train_seconds = std::chrono::duration<double>(t2 - t1).count();
    rep->steps = steps;
    rep->first_epoch_loss = per.front();
    rep->last_epoch_loss = per.back();
    rep->s_in = S.sIn;
    rep->s_out = S.sOut;
  }
  return checkStatus(c);
}
