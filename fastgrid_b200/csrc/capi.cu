// C ABI of the grid-map engine: contexts, device buffers, the e-map and
// affinity entry points, whole-job (GPF) entry points and the command line.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <signal.h>
#include <string>
#include <thread>
#include <sys/wait.h>
#include <unistd.h>
#include <vector>

#include "../../include/fastgrid_b200.h"
#include "ag_ctx.h"
#include "ag_host.h"
#include "ag_kernels.h"

namespace agc {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

// Threshold table for the exact e-map bin: thr[k] is the least double r^2
// with int(sqrt(r^2) * 100.0) >= k under IEEE double rounding, i.e. the bin
// the reference's FP64 code (Cpu.cpp:70-75) computes is k-1 below it and k
// at or above it.  Fills thr[0 .. 8192] (found by bisection over doubles).
void emapBinThresholdsInto(double* thr) {
  thr[0] = 0.0;
  for (int k = 1; k <= 8192; k++) {
    double lo = 0.0, hi = (k / 100.0 + 1.0) * (k / 100.0 + 1.0);
    uint64_t a, b;
    memcpy(&a, &lo, 8);
    memcpy(&b, &hi, 8);
    while (b - a > 1) {
      uint64_t m = a + (b - a) / 2;
      double v;
      memcpy(&v, &m, 8);
      if (sqrt(v) * 100.0 >= (double)k) b = m; else a = m;
    }
    memcpy(&thr[k], &b, 8);
  }
}

const std::vector<double>& binThresholds() {
  static std::vector<double> thr;
  static std::once_flag once;
  std::call_once(once, [] {
    thr.assign(8193, 0.0);
    emapBinThresholdsInto(thr.data());
  });
  return thr;
}

// The same for the affinity pass, whose bin is int((1 / (1 / sqrt(r^2))) * 100)
// (CalculateGridmaps.cpp:284-289): thr[k] is the least r^2 with bin >= k.
const std::vector<double>& affinityBinThresholds() {
  static std::vector<double> thr;
  static std::once_flag once;
  std::call_once(once, [] {
    thr.assign(agk::kAffRows + 1, 0.0);
    auto binOf = [](double r2) {
      volatile double inv = 1.0 / sqrt(r2);
      volatile double r = 1.0 / inv;
      return r * 100.0;
    };
    for (int k = 1; k <= agk::kAffRows; k++) {
      double lo = 0.0, hi = (k / 100.0 + 1.0) * (k / 100.0 + 1.0);
      uint64_t a, b;
      memcpy(&a, &lo, 8);
      memcpy(&b, &hi, 8);
      while (b - a > 1) {
        uint64_t m = a + (b - a) / 2;
        double v;
        memcpy(&v, &m, 8);
        if (binOf(v) >= (double)k) b = m; else a = m;
      }
      memcpy(&thr[k], &b, 8);
    }
  });
  return thr;
}

}  // namespace agc

using namespace agc;

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
extern "C" const char* ag_last_error(void) { return g_err.c_str(); }

namespace ag {
// Lets other translation units of the library report through ag_last_error().
void setLastError(const char* msg) { g_err = msg; }
}  // namespace ag

extern "C" int ag_ctx_create(int device, ag_ctx** out) {
  if (!out) return fail(AG_E_INVALID, "null output pointer");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return fail(AG_E_CUDA, "no CUDA device is available; this engine has no CPU fallback");
  if (device < 0 || device >= n) return fail(AG_E_INVALID, "device %d out of range (%d devices)", device, n);
  CK(cudaSetDevice(device));
  auto* c = new ag_ctx();
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(AG_E_CUDA, "cudaStreamCreate failed");
  }
  // The status word must start at zero: cudaMalloc may hand back memory that
  // a freed buffer of this process (another context's maps) left its values
  // in, and kernels only ever set bits in it.
  if (c->status.ensure(4) != cudaSuccess || cudaMemset(c->status.p, 0, sizeof(unsigned)) != cudaSuccess) {
    delete c;
    return fail(AG_E_NOMEM, "cannot allocate the status word");
  }
  const auto& thr = binThresholds();
  if (c->thr.ensure(thr.size()) != cudaSuccess ||
      cudaMemcpy(c->thr.p, thr.data(), thr.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    delete c;
    return fail(AG_E_CUDA, "cannot upload the bin threshold table");
  }
  *out = c;
  return AG_OK;
}

extern "C" int ag_ctx_destroy(ag_ctx* c) {
  if (!c) return AG_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto* b : {&c->epsTab, &c->maps, &c->vol, &c->solq, &c->affTab, &c->affTabH, &c->sol, &c->rv32, &c->rv2_32})
    b->release();
  c->atoms.release();
  c->thr.release();
  c->partial.release();
  c->rv64.release();
  c->thrA.release();
  c->checksum.release();
  agc::surrFree(c->surr);
  c->surr = nullptr;
  c->blocks.release();
  c->status.release();
  for (auto* b : {&c->items, &c->info, &c->cellStart, &c->cellAtoms, &c->cellOf, &c->count, &c->fill, &c->dStart,
                  &c->dAtoms, &c->donorMask, &c->closestH, &c->ctStart, &c->ctAtoms})
    b->release();
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copyStream) cudaStreamDestroy(c->copyStream);
  if (c->evAff) cudaEventDestroy(c->evAff);
  if (c->emapStream) cudaStreamDestroy(c->emapStream);
  if (c->evFork) cudaEventDestroy(c->evFork);
  if (c->evJoin) cudaEventDestroy(c->evJoin);
  for (cudaEvent_t ev : c->evChunk)
    if (ev) cudaEventDestroy(ev);
  delete c;
  return AG_OK;
}

extern "C" int ag_ctx_tune(ag_ctx* c, int knob, double v) {
  if (!c) return fail(AG_E_INVALID, "null context");
  switch (knob) {
    case AG_TUNE_EMAP_RNEAR:
      if (!(v >= 8.0 && v <= 40.0)) return fail(AG_E_INVALID, "rNear must be in [8, 40] A");
      c->rNear = (float)v;
      return AG_OK;
    case AG_TUNE_EMAP_PACKED_TABLE:
      if (!(v == 0.0 || v == 1.0)) return fail(AG_E_INVALID, "packed-table switch must be 0 or 1");
      c->packedTable = (int)v;
      return AG_OK;
    case AG_TUNE_EMAP_WARP_COMPACT:
      if (!(v == 0.0 || v == 1.0 || v == 2.0)) return fail(AG_E_INVALID, "e-map item order must be 0, 1 or 2");
      c->warpCompact = (int)v;
      return AG_OK;
    case AG_TUNE_EMAP_TILE: {
      const int t = (int)v, tx = t / 10000, ty = (t / 100) % 100, tz = t % 100;
      if (v != (double)t || tx < 1 || ty < 1 || tz < 1 || tx * ty * tz != 256)
        return fail(AG_E_INVALID, "tile must be TX*10000 + TY*100 + TZ with TX*TY*TZ = 256 work items");
      c->tile[0] = tx;
      c->tile[1] = ty;
      c->tile[2] = tz;
      return AG_OK;
    }
    case AG_TUNE_SURROGATE_TCGEN05:
      if (!(v == 0.0 || v == 1.0)) return fail(AG_E_INVALID, "tcgen05 switch must be 0 or 1");
      agc::surrUseTc(c, v != 0.0);
      return AG_OK;
    case AG_TUNE_AFFINITY_KERNEL:
      if (!(v == 1.0 || v == 2.0)) return fail(AG_E_INVALID, "affinity kernel must be 1 or 2");
      c->affKernel = (int)v;
      return AG_OK;
    case AG_TUNE_TEST_IDLE_WAIT:
      if (!(v >= 0.0 && v <= 64.0) || v != (double)(int)v) return fail(AG_E_INVALID, "idle-wait polls must be 0..64");
      c->testIdleWait = (int)v;
      return AG_OK;
    case AG_TUNE_TEST_CHECKSUM_OFFSET:
      if (!std::isfinite(v)) return fail(AG_E_INVALID, "checksum offset must be finite");
      c->testChecksumOffset = v;
      return AG_OK;
    case AG_TUNE_CONCURRENT_PASSES:
      if (!(v == 0.0 || v == 1.0)) return fail(AG_E_INVALID, "concurrent-passes switch must be 0 or 1");
      c->concurrentPasses = (int)v;
      return AG_OK;
    case AG_TUNE_EMAP_CTAS_PER_SM:
      if (!(v >= 1.0 && v <= 8.0)) return fail(AG_E_INVALID, "CTAs per SM must be 1..8");
      c->ctasPerSm = (int)v;
      return AG_OK;
    default:
      return fail(AG_E_INVALID, "unknown tuning knob %d", knob);
  }
}

extern "C" void* ag_ctx_stream(ag_ctx* c) { return c ? (void*)c->stream : nullptr; }
extern "C" int64_t ag_ctx_launch_count(const ag_ctx* c) { return c ? c->launches : 0; }

// ---------------------------------------------------------------------------
// Job staging
// ---------------------------------------------------------------------------
namespace agc {

int checkGrid(const ag_grid* g) {
  if (!g) return fail(AG_E_INVALID, "null grid");
  if (g->nx < 1 || g->ny < 1 || g->nz < 1 || g->nx > 1025 || g->ny > 1025 || g->nz > 1025)
    return fail(AG_E_INVALID, "grid %dx%dx%d outside 1..1025 points per axis", g->nx, g->ny, g->nz);
  if (!(g->spacing > 0) || !std::isfinite(g->spacing)) return fail(AG_E_INVALID, "bad grid spacing");
  return AG_OK;
}

// Work items of the e-map (NX points of one row each), grouped into CTAs of
// 256 items walking tiles of TX x TY x TZ items, with each CTA's box.
// warpCompact >= 1: inside a tile, items go in blocks of TX x 4 x 4 (x fastest),
// so each warp's 32 items form a compact box (for kernels that skip atoms
// per warp); otherwise x, then y, then z.
// warpCompact == 2 (TX even): the two items of each pair of x columns, held by
// neighbouring lanes, are marked kItemInterleaved and split the pair's 2 NX
// points between them alternately, so the points a warp visits at one step k
// form a 2 x 4 x 4 block of neighbouring grid points instead of a 1 x 4 x 8
// one with columns NX points apart.  Their distances to an atom then span
// fewer table bins, and the table reads of a warp hit fewer distinct words in
// one shared-memory bank.  A column whose partner is past the grid edge keeps
// its own NX consecutive points.
void makeItems(const ag_grid& g, const int tile[3], int warpCompact, std::vector<int>& items,
               std::vector<agk::EmapBlock>& blocks) {
  const int nxc = (g.nx + agk::kNX - 1) / agk::kNX;
  const int TX = tile[0], TY = tile[1], TZ = tile[2];
  items.clear();
  // Tiles in boustrophedon order (y rows and x columns reverse direction on
  // alternate passes), so a CTA that continues from one tile into the next
  // stays within neighbouring tiles and its box stays compact.
  const int ntx = (nxc + TX - 1) / TX, nty = (g.ny + TY - 1) / TY, ntz = (g.nz + TZ - 1) / TZ;
  const bool compact = warpCompact && TY % 4 == 0 && TZ % 4 == 0;
  int serp = 0;
  for (int kz = 0; kz < ntz; kz++)
    for (int ky0 = 0; ky0 < nty; ky0++) {
      const int ky = (kz & 1) ? nty - 1 - ky0 : ky0;
      for (int kx0 = 0; kx0 < ntx; kx0++, serp++) {
        const int kx = (serp / ntx) & 1 ? ntx - 1 - kx0 : kx0;
        const int tx = kx * TX, ty = ky * TY, tz = kz * TZ;
        if (compact) {
          for (int zb = tz; zb < tz + TZ; zb += 4)
            for (int yb = ty; yb < ty + TY; yb += 4)
              for (int z = zb; z < std::min(g.nz, zb + 4); z++)
                for (int y = yb; y < std::min(g.ny, yb + 4); y++)
                  for (int x = tx; x < std::min(nxc, tx + TX); x++) {
                    const bool il = warpCompact == 2 && TX % 2 == 0 && (x ^ 1) < nxc;
                    items.push_back(x | (y << 8) | (z << 19) | (il ? agk::kItemInterleaved : 0));
                  }
        } else {
          for (int z = tz; z < std::min(g.nz, tz + TZ); z++)
            for (int y = ty; y < std::min(g.ny, ty + TY); y++)
              for (int x = tx; x < std::min(nxc, tx + TX); x++) items.push_back(x | (y << 8) | (z << 19));
        }
      }
    }
  blocks.clear();
  const double h = g.spacing;
  const int n2x = g.nx / 2, n2y = g.ny / 2, n2z = g.nz / 2;
  for (size_t i0 = 0; i0 < items.size(); i0 += 256) {
    agk::EmapBlock b{};
    b.item0 = (int)i0;
    b.nitems = (int)std::min<size_t>(256, items.size() - i0);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < b.nitems; k++) {
      int v = items[i0 + k];
      int xc = v & 0xFF, y = (v >> 8) & 0x7FF, z = (v >> 19) & 0x7FF;  // the pair's union is the same box
      int xa = xc * agk::kNX, xb = std::min(g.nx - 1, xa + agk::kNX - 1);
      double p[2][3] = {{(xa - n2x) * h, (y - n2y) * h, (z - n2z) * h}, {(xb - n2x) * h, (y - n2y) * h, (z - n2z) * h}};
      for (int q = 0; q < 2; q++)
        for (int d = 0; d < 3; d++) {
          lo[d] = std::min(lo[d], p[q][d]);
          hi[d] = std::max(hi[d], p[q][d]);
        }
    }
    b.ox = 0.5 * (lo[0] + hi[0]);
    b.oy = 0.5 * (lo[1] + hi[1]);
    b.oz = 0.5 * (lo[2] + hi[2]);
    b.hx = (float)(50.0 * (hi[0] - lo[0]) + 1.0);
    b.hy = (float)(50.0 * (hi[1] - lo[1]) + 1.0);
    b.hz = (float)(50.0 * (hi[2] - lo[2]) + 1.0);
    // Atoms at least rFar (50-55 A) from the box use the saturated dielectric
    // (table entries past 55 A differ from entry 8191 by < 2.6e-7 relative, past
    // 50 A by < 1.3e-6); nearer ones read the table, whose index then stays
    // below 8191 without clamping.
    const double diag = 2.0 * std::sqrt((double)b.hx * b.hx + (double)b.hy * b.hy + (double)b.hz * b.hz) / 100.0;
    const double rFar = std::max(50.0, std::min(55.0, 81.0 - diag));
    b.rfar2 = (float)((100.0 * rFar) * (100.0 * rFar));
    b.clampMid = rFar + diag >= 81.0 ? 1 : 0;  // mid-list bins may then exceed the table
    blocks.push_back(b);
  }
}

void buildItems(ag_ctx* c) {
  const ag_grid& g = c->grid;
  if (c->itemsFor[0] == g.nx && c->itemsFor[1] == g.ny && c->itemsFor[2] == g.nz && c->itemsH == g.spacing &&
      c->itemsTile == c->tile[0] * 10000 + c->tile[1] * 100 + c->tile[2] && c->itemsCompact == c->warpCompact)
    return;
  makeItems(g, c->tile, c->warpCompact, c->hItems, c->hBlocks);
  c->itemsOnDevice = false;
  c->itemsCompact = c->warpCompact;
  c->itemsFor[0] = g.nx;
  c->itemsFor[1] = g.ny;
  c->itemsFor[2] = g.nz;
  c->itemsH = g.spacing;
  c->itemsTile = c->tile[0] * 10000 + c->tile[1] * 100 + c->tile[2];
}

// 16- and 8-bit copies of the FP32 table's saturating tail.  With g = t[n-1]
// and G = bits(g), entry b is G + k_b, k_b < 2^16 (2^8), for every bin from
// b16 (b8) on, all of them in g's binade, so that k_b counts units in the last
// place of g and g + k_b ulp(g) = t[b] exactly.  The two parts are padded to
// 16 bytes and must fit `cap` bytes; b16 moves up until they do.  Writes the
// parts to raw and returns their size in bytes (0: no usable tail; b16 = b8
// = n).  Allocates nothing.
int packTableTailInto(const float* t, int n, unsigned char* raw, int cap, int& b16, int& b8, int& vec8,
                      float& kScale) {
  b16 = b8 = n;
  vec8 = 0;
  kScale = 0.f;
  if (n <= 0) return 0;
  const float g = t[n - 1];
  if (!(std::isfinite(g) && g >= FLT_MIN)) return 0;
  uint32_t G;
  std::memcpy(&G, &g, 4);
  const uint32_t expG = G >> 23;
  auto first = [&](uint32_t kmax) {
    int b = n;
    while (b > 0) {
      uint32_t u;
      std::memcpy(&u, &t[b - 1], 4);
      if ((u >> 31) || (u >> 23) != expG || u < G || u - G > kmax) break;
      b--;
    }
    return b;
  };
  b16 = first(0xFFFFu);
  b8 = first(0xFFu);
  auto bytes = [&](int b16_) { return ((2 * (n - b16_) + 15) / 16) * 16 + ((n - b8 + 15) / 16) * 16; };
  while (b16 < n && bytes(b16) > cap) b16 += 8;
  if (b16 >= n) {
    b16 = b8 = n;
    return 0;
  }
  const int v16 = (2 * (n - b16) + 15) / 16;
  vec8 = v16;
  const int total = bytes(b16);
  std::memset(raw, 0, (size_t)total);
  for (int b = b16; b < n; b++) {
    uint32_t u;
    std::memcpy(&u, &t[b], 4);
    const uint16_t k = (uint16_t)(u - G);
    std::memcpy(&raw[2 * (size_t)(b - b16)], &k, 2);
  }
  for (int b = b8; b < n; b++) {
    uint32_t u;
    std::memcpy(&u, &t[b], 4);
    raw[16 * (size_t)v16 + (b - b8)] = (unsigned char)(u - G);
  }
  // 2^(e + 126) / g with g = 2^e m, 1 <= m < 2.
  kScale = (float)(std::ldexp(1.0, (int)expG - 127 + 126) / (double)g);
  return total;
}

// The same, into 16-byte vectors (empty: no usable tail).
std::vector<uint4> packTableTail(const std::vector<float>& t, int& b16, int& b8, int& vec8, float& kScale) {
  std::vector<uint4> out(agk::kEmapPackedBytes / 16);
  const int bytes = packTableTailInto(t.data(), (int)t.size(), reinterpret_cast<unsigned char*>(out.data()),
                                      agk::kEmapPackedBytes, b16, b8, vec8, kScale);
  out.resize((size_t)bytes / 16);
  return out;
}

int stageEmap(ag_ctx* c, const ag_grid* g, int n, const double* xyzw, const double* inv_eps, bool deviceInputs) {
  if (int r = checkGrid(g)) return r;
  if (n < 0 || (n > 0 && !xyzw)) return fail(AG_E_INVALID, "bad atom array");
  c->grid = *g;
  c->nAtoms = n;
  c->ddd = inv_eps != nullptr;
  CK(cudaSetDevice(c->device));
  if (!deviceInputs) {
    for (int64_t i = 0; i < 4 * (int64_t)n; i++)
      if (!std::isfinite(xyzw[i])) return fail(AG_E_INVALID, "non-finite atom coordinate or weight at atom %lld", (long long)(i / 4));
    c->wSum = 0;
    c->wAbsSum = 0;
    for (int i = 0; i < n; i++) {
      c->wSum += xyzw[4 * (size_t)i + 3];
      c->wAbsSum += std::fabs(xyzw[4 * (size_t)i + 3]);
    }
    CK(c->atoms.ensure(n));
    if (n) CK(cudaMemcpyAsync(c->atoms.p, xyzw, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, c->stream));
    c->atomsVersion++;  // the surrogate reads the staged atoms back when it needs a host copy
  }
  c->epsHost.clear();
  if (c->ddd) {
    c->epsHost.assign(inv_eps, inv_eps + 8192);
    std::vector<float> t(8192);
    for (int i = 0; i < 8192; i++) t[i] = (float)inv_eps[i];
    CK(c->epsTab.ensure(8192));
    CK(cudaMemcpyAsync(c->epsTab.p, t.data(), sizeof(float) * 8192, cudaMemcpyHostToDevice, c->stream));
    const std::vector<uint4> pk = packTableTail(t, c->pkB16, c->pkB8, c->pkVec8, c->pkScale);
    c->pkVecs = (int)pk.size();
    if (!pk.empty()) {
      CK(c->epsPacked.ensure(pk.size()));
      CK(cudaMemcpyAsync(c->epsPacked.p, pk.data(), sizeof(uint4) * pk.size(), cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
  }
  buildItems(c);
  if (!c->itemsOnDevice) {  // the work items and CTA boxes depend on the grid only
    CK(c->items.ensure(c->hItems.size()));
    CK(c->blocks.ensure(c->hBlocks.size()));
    CK(cudaMemcpyAsync(c->items.p, c->hItems.data(), sizeof(int) * c->hItems.size(), cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaMemcpyAsync(c->blocks.p, c->hBlocks.data(), sizeof(agk::EmapBlock) * c->hBlocks.size(),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->itemsOnDevice = true;
  }
  return AG_OK;
}

// Launch parameters of the e-map of the staged job; allowSplit = false keeps
// every CTA on all atoms (the batch kernel's mode).
int buildEmapParams(ag_ctx* c, float* dOut, bool allowSplit, agk::EmapParams& P) {
  const int64_t np = c->npoints();
  P = agk::EmapParams{};
  P.atoms = c->atoms.p;
  P.n_atoms = c->nAtoms;
  P.nblocks = (int)c->hBlocks.size();
  P.items = c->items.p;
  P.blocks = c->blocks.p;
  P.nx = c->grid.nx; P.ny = c->grid.ny; P.nz = c->grid.nz;
  P.n2x = P.nx / 2; P.n2y = P.ny / 2; P.n2z = P.nz / 2;
  P.npoints = np;
  P.h = c->grid.spacing;
  P.table = c->epsTab.p;
  P.thr = c->thr.p;
  P.rnear2 = (100.f * c->rNear) * (100.f * c->rNear);
  P.delta = c->delta;
  if (c->ddd && c->packedTable && c->pkVecs > 0) {
    P.packed = c->epsPacked.p;
    P.packedVecs = c->pkVecs;
    P.vec8 = c->pkVec8;
    P.b16 = c->pkB16;
    P.b8 = c->pkB8;
    P.r16sq = (float)((c->pkB16 + 2.0) * (c->pkB16 + 2.0));
    P.r8sq = (float)((c->pkB8 + 2.0) * (c->pkB8 + 2.0));
    P.kScale = c->pkScale;
  }
  P.out = dOut;
  P.status = c->status.p;
  P.testIdleWait = c->testIdleWait;
  // Split atoms across CTAs when the grid alone cannot fill the GPU.
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  const int want = 2 * sms * c->ctasPerSm;  // two waves of resident CTAs
  int nsplit = 1;
  if (allowSplit && P.nblocks < want && c->nAtoms > 512)
    nsplit = std::min((want + P.nblocks - 1) / P.nblocks, (c->nAtoms + 255) / 256);
  int chunk = (c->nAtoms + nsplit - 1) / nsplit;
  chunk = ((chunk + 255) / 256) * 256;
  if (chunk == 0) chunk = 256;
  nsplit = std::max(1, (c->nAtoms + chunk - 1) / chunk);
  P.chunk = chunk;
  P.nsplit = nsplit;
  if (nsplit > 1) {
    CK(c->partial.ensure((size_t)nsplit * np));
    P.partial = c->partial.p;
  }
  return AG_OK;
}

int runEmap(ag_ctx* c, float* dOut) {
  const int64_t np = c->npoints();
  agk::EmapParams P;
  if (int e = buildEmapParams(c, dOut, true, P)) return e;
  const int nsplit = P.nsplit;
  if (c->nAtoms == 0) {
    CK(cudaMemsetAsync(dOut, 0, sizeof(float) * np, c->stream));
    return AG_OK;
  }
  CK(c->checksum.ensure(nsplit));
  P.checksum = c->checksum.p;
  c->checksumSplits = nsplit;
  CK(agk::emap_launch(P, c->ddd, c->emapMode, P.nblocks * nsplit, c->stream));
  c->launches += nsplit > 1 ? 2 : 1;
  return AG_OK;
}

int stageAffinity(ag_ctx* c, const ag_receptor* r, const ag_affinity_params* p) {
  const int n = r->n_atoms;
  if (p->n_maps < 0 || p->n_maps > ag::kMaxAtomTypes) return fail(AG_E_INVALID, "n_maps %d outside 0..14", p->n_maps);
  if (p->n_types < 1 || p->n_types > ag::kNumAllTypes) return fail(AG_E_INVALID, "n_types %d outside 1..32", p->n_types);
  std::vector<int> info(n), donor(n);
  std::vector<float> vol(n), solq(n);
  for (int i = 0; i < n; i++) {
    if (r->type[i] < 0 || r->type[i] >= p->n_types) return fail(AG_E_INVALID, "atom %d has type %d outside 0..%d", i, r->type[i], p->n_types - 1);
    if (r->hbond[i] < 0 || r->hbond[i] > 5) return fail(AG_E_INVALID, "atom %d has H-bond class %d", i, r->hbond[i]);
    info[i] = r->type[i] | (r->hbond[i] << 5) | ((r->disorder[i] ? 1 : 0) << 8) | ((r->rexp[i] & 7) << 9);
    donor[i] = (r->hbond[i] == ag::DS || r->hbond[i] == ag::D1) ? 1 : 0;
    vol[i] = (float)r->vol[i];
    solq[i] = (float)(r->solpar[i] + p->solpar_q * fabs(r->charge[i]));
  }
  // The H-bond class is a property of the receptor type; the kernel branches on it per type.
  for (int t = 0; t < agk::kMaxTypes; t++) c->typeHbond[t] = -1;
  for (int i = 0; i < n; i++) {
    int& th = c->typeHbond[r->type[i]];
    if (th < 0) th = r->hbond[i];
    else if (th != r->hbond[i])
      return fail(AG_E_INVALID, "atoms of receptor type %d have different H-bond classes", r->type[i]);
  }
  for (int t = 0; t < agk::kMaxTypes; t++) if (c->typeHbond[t] < 0) c->typeHbond[t] = ag::NON;
  std::vector<float> rv32(3 * (size_t)n), rv2_32(3 * (size_t)n);
  for (size_t i = 0; i < 3 * (size_t)n; i++) { rv32[i] = (float)r->rvector[i]; rv2_32[i] = (float)r->rvector2[i]; }
  CK(c->info.ensure(n)); CK(c->donorMask.ensure(n)); CK(c->vol.ensure(n)); CK(c->solq.ensure(n));
  CK(c->rv32.ensure(3 * (size_t)n)); CK(c->rv2_32.ensure(3 * (size_t)n)); CK(c->rv64.ensure(3 * (size_t)n));
  if (n) {
    CK(cudaMemcpyAsync(c->info.p, info.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->donorMask.p, donor.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->vol.p, vol.data(), sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->solq.p, solq.data(), sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->rv32.p, rv32.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->rv2_32.p, rv2_32.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->rv64.p, r->rvector, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  }
  c->nMaps = p->n_maps;
  c->nTypes = p->n_types;
  c->hydrogen = p->hydrogen;
  c->solparQ = p->solpar_q;
  c->mapHbond.assign(p->map_hbond, p->map_hbond + p->n_maps);
  c->mapIsHB.assign(p->map_is_hbonder, p->map_is_hbonder + p->n_maps);
  c->mapCov.assign(p->map_is_covalent, p->map_is_covalent + p->n_maps);
  c->solparProbe.assign(p->solpar_probe, p->solpar_probe + p->n_maps);
  c->volProbe.assign(p->vol_probe, p->vol_probe + p->n_maps);

  // Split the maps into passes of at most 16 maps and 4 min/max maps.
  const int nm = p->n_maps, nt = p->n_types;
  auto isMinMax = [&](int m) {
    const int hb = c->mapHbond[m];
    return c->mapIsHB[m] && !c->mapCov[m] && (hb == ag::A1 || hb == ag::DS || hb == ag::D1);
  };
  c->passes.clear();
  for (int m0 = 0; m0 < nm;) {
    ag_ctx::Pass ps{};
    ps.m0 = m0;
    int mm = 0, k = 0;
    while (m0 + k < nm && k < agk::kMaxMapsPass) {
      if (isMinMax(m0 + k) && mm == agk::kMaxMinMax) break;
      ps.mapMinMaxSlot[k] = isMinMax(m0 + k) ? mm++ : -1;
      k++;
    }
    ps.nm = k;
    ps.nmPad = ((k + 3) / 4) * 4;
    for (int t = 0; t < nt; t++) {
      unsigned modes = 0;
      const int ahb = c->typeHbond[t];
      const bool donor = ahb == ag::DS || ahb == ag::D1;
      for (int g = 0; g < k; g++) {
        const int m = m0 + g, mhb = c->mapHbond[m];
        unsigned mode = 0;
        if (c->mapIsHB[m] && !c->mapCov[m]) {
          if ((mhb == ag::AS || mhb == ag::A2) && donor) mode = 1;
          else if (mhb == ag::A1 && donor) mode = 2;
          else if ((mhb == ag::DS || mhb == ag::D1) && ahb >= ag::AS) mode = 3;
        }
        modes |= mode << (2 * g);
      }
      ps.typeModes[t] = modes;
      ps.typeNeedsAngular[t] = modes != 0 && (ahb == ag::D1 || ahb == ag::A1 || ahb == ag::A2);
    }
    c->passes.push_back(ps);
    m0 += k;
  }
  // Pair-energy tables, FP32, rows r <= 8 A, per pass [type][row][nmPad].
  size_t tabSize = 0, tabHSize = 0;
  for (auto& ps : c->passes) {
    ps.tabOff = tabSize;
    ps.tabHOff = tabHSize;
    tabSize += (size_t)nt * agk::kAffRows * ps.nmPad;
    tabHSize += (size_t)agk::kAffRows * ps.nmPad;
  }
  std::vector<float> tab(std::max<size_t>(tabSize, 4), 0.f), tabH(std::max<size_t>(tabHSize, 4), 0.f);
  for (auto& ps : c->passes) {
    for (int t = 0; t < nt; t++)
      for (int i = 0; i < agk::kAffRows; i++) {
        for (int g = 0; g < ps.nm; g++)
          tab[ps.tabOff + ((size_t)t * agk::kAffRows + i) * ps.nmPad + g] =
              (float)p->energy[((size_t)t * 8192 + i) * nm + ps.m0 + g];
        // A spare last column carries the desolvation value (read by the two-point kernel).
        if (ps.nm < ps.nmPad) tab[ps.tabOff + ((size_t)t * agk::kAffRows + i) * ps.nmPad + ps.nmPad - 1] = (float)p->sol[i];
      }
    if (p->hydrogen >= 0 && p->hydrogen < nt)
      for (int i = 0; i < agk::kAffRows; i++)
        for (int g = 0; g < ps.nm; g++)
          tabH[ps.tabHOff + (size_t)i * ps.nmPad + g] = (float)p->energy[((size_t)p->hydrogen * 8192 + i) * nm + ps.m0 + g];
  }
  if (!c->thrA.p) {
    const auto& thr = affinityBinThresholds();
    CK(c->thrA.ensure(thr.size()));
    CK(cudaMemcpyAsync(c->thrA.p, thr.data(), sizeof(double) * thr.size(), cudaMemcpyHostToDevice, c->stream));
  }
  std::vector<float> sol(agk::kAffRows);
  for (int i = 0; i < agk::kAffRows; i++) sol[i] = (float)p->sol[i];
  CK(c->affTab.ensure(tab.size())); CK(c->affTabH.ensure(tabH.size())); CK(c->sol.ensure(sol.size()));
  CK(cudaMemcpyAsync(c->affTab.p, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->affTabH.p, tabH.data(), sizeof(float) * tabH.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->sol.p, sol.data(), sizeof(float) * sol.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->haveAff = true;
  return AG_OK;
}

// 8 A cells over the grid box widened by 8 A (atoms further out cannot reach a point).
void cellGrid(const ag_grid& g, double lo[3], int ncell[3]) {
  const double h = g.spacing;
  const int nn[3] = {g.nx, g.ny, g.nz};
  for (int d = 0; d < 3; d++) {
    lo[d] = (double)(0 - nn[d] / 2) * h - 8.0;
    const double hi = (double)(nn[d] - 1 - nn[d] / 2) * h + 8.0;
    ncell[d] = std::max(1, (int)std::ceil((hi - lo[d]) / 8.0));
  }
}

// H-bond slots of a pass for the two-point kernel: the H-bond maps whose term
// differs from a plain table sum for some receptor type
// (CalculateGridmaps.cpp:206-228).  Returns false if the pass has more than
// kA2Slots of them (the one-point kernel then computes it).
bool passSlots(const ag_ctx* c, const ag_ctx::Pass& ps, int& nslots, int slotMap[agk::kA2Slots],
               int slotKind[agk::kA2Slots]) {
  nslots = 0;
  for (int g = 0; g < ps.nm; g++) {
    const int m = ps.m0 + g, mhb = c->mapHbond[m];
    if (!c->mapIsHB[m] || c->mapCov[m]) continue;
    int kind = -1;
    if (mhb == ag::AS || mhb == ag::A2) kind = agk::A2_SLOT_ACC;
    else if (mhb == ag::A1) kind = agk::A2_SLOT_A1;
    else if (mhb == ag::DS || mhb == ag::D1) kind = agk::A2_SLOT_DON;
    if (kind < 0) continue;
    if (nslots == agk::kA2Slots) return false;
    slotMap[nslots] = g;
    slotKind[nslots] = kind;
    nslots++;
  }
  return true;
}

// Whether every affinity pass of the staged job runs on the two-point kernel.
bool useTwoPoint(const ag_ctx* c) {
  if (c->affKernel != 2) return false;
  for (const auto& ps : c->passes) {
    int n, sm[agk::kA2Slots], sk[agk::kA2Slots];
    if (!passSlots(c, ps, n, sm, sk)) return false;
  }
  return true;
}

// Cell lists on stream st.  One-point kernel: all atoms and H donors in 8 A
// cells, and the nearest donor of every point.  Two-point kernel: one list of
// (cell, receptor type) segments (it finds the nearest donor itself).
int prepAffinity(ag_ctx* c, cudaStream_t st) {
  const ag_grid& g = c->grid;
  const int64_t np = c->npoints();
  const int n = c->nAtoms;
  const double h = g.spacing;
  double lo[3];
  int ncell[3];
  cellGrid(g, lo, ncell);
  const int ncellT = ncell[0] * ncell[1] * ncell[2];
  agk::CellBuild C{};
  C.xyz = c->atoms.p; C.n_atoms = n;
  for (int d = 0; d < 3; d++) { C.lo[d] = lo[d]; C.ncell[d] = ncell[d]; }
  if (useTwoPoint(c)) {
    const int nkeys = ncellT * c->nTypes;
    CK(c->ctStart.ensure(nkeys + 1)); CK(c->count.ensure(nkeys + 1)); CK(c->fill.ensure(nkeys + 1));
    CK(c->ctAtoms.ensure(n)); CK(c->cellOf.ensure(n));
    C.cellOf = c->cellOf.p; C.count = c->count.p; C.fill = c->fill.p;
    C.cellStart = c->ctStart.p; C.cellAtoms = c->ctAtoms.p; C.donorMask = nullptr;
    C.typeInfo = c->info.p; C.ntypes = c->nTypes;
    CK(agk::cells_launch(C, nkeys, st));
    c->launches += 4;
    return AG_OK;
  }
  CK(c->cellStart.ensure(ncellT + 1)); CK(c->count.ensure(ncellT + 1)); CK(c->fill.ensure(ncellT + 1));
  CK(c->cellAtoms.ensure(n)); CK(c->cellOf.ensure(n));
  CK(c->dStart.ensure(ncellT + 1)); CK(c->dAtoms.ensure(n));
  CK(c->closestH.ensure(np));
  C.cellOf = c->cellOf.p; C.count = c->count.p; C.fill = c->fill.p;
  C.cellStart = c->cellStart.p; C.cellAtoms = c->cellAtoms.p; C.donorMask = nullptr;
  CK(agk::cells_launch(C, ncellT, st));
  C.cellStart = c->dStart.p; C.cellAtoms = c->dAtoms.p; C.donorMask = c->donorMask.p;
  CK(agk::cells_launch(C, ncellT, st));
  c->launches += 8;
  agk::ClosestHParams H{};
  H.xyz = c->atoms.p; H.cellStart = c->dStart.p; H.cellAtoms = c->dAtoms.p;
  for (int d = 0; d < 3; d++) { H.cellLo[d] = lo[d]; H.ncell[d] = ncell[d]; }
  H.nx = g.nx; H.ny = g.ny; H.nz = g.nz; H.n2x = g.nx / 2; H.n2y = g.ny / 2; H.n2z = g.nz / 2;
  H.npoints = np; H.h = h; H.closestH = c->closestH.p;
  CK(agk::closest_h_launch(H, st));
  c->launches += 1;
  return AG_OK;
}

// Launch parameters of the two-point kernel for the staged job's passes.
int buildAff2Params(ag_ctx* c, float* dMaps, float* dDmap, std::vector<agk::Aff2Params>& out) {
  const ag_grid& g = c->grid;
  double lo[3];
  int ncell[3];
  cellGrid(g, lo, ncell);
  out.clear();
  const int nt = c->nTypes;
  std::vector<ag_ctx::Pass> passes = c->passes;
  if (passes.empty()) {  // no ligand maps: one pass for the d-map alone
    ag_ctx::Pass ps{};
    ps.nmPad = 4;
    passes.push_back(ps);
  }
  for (const auto& ps : passes) {
    agk::Aff2Params P{};
    P.xyz = c->atoms.p; P.info = c->info.p; P.vol = c->vol.p; P.solq = c->solq.p;
    P.rv = c->rv32.p; P.rv2 = c->rv2_32.p; P.rv64 = c->rv64.p;
    P.ctStart = c->ctStart.p; P.ctAtoms = c->ctAtoms.p;
    for (int d = 0; d < 3; d++) { P.cellLo[d] = lo[d]; P.ncell[d] = ncell[d]; }
    P.nx = g.nx; P.ny = g.ny; P.nz = g.nz; P.n2x = g.nx / 2; P.n2y = g.ny / 2; P.n2z = g.nz / 2;
    P.npoints = c->npoints(); P.h = g.spacing;
    P.nmaps = ps.nm; P.nmPad = ps.nmPad; P.ntypes = nt; P.hydrogen = c->hydrogen;
    P.table = c->affTab.p + ps.tabOff;
    P.tableH = (c->hydrogen >= 0 && c->hydrogen < nt) ? c->affTabH.p + ps.tabHOff : nullptr;
    P.sol = c->sol.p;
    P.solInRow = ps.nm < ps.nmPad ? 1 : 0;
    P.thr = c->thrA.p;
    P.delta = 1.0e-3f;
    if (!passSlots(c, ps, P.nslots, P.slotMap, P.slotKind)) return fail(AG_E_INVALID, "too many H-bond maps");
    for (int k = P.nslots; k < agk::kA2Slots; k++) { P.slotMap[k] = -1; P.slotKind[k] = agk::A2_SLOT_ACC; }
    P.needClosestH = 0;
    for (int t = 0; t < agk::kMaxTypes; t++) {
      const int ahb = t < nt ? c->typeHbond[t] : ag::NON;
      const bool donor = ahb == ag::DS || ahb == ag::D1, acceptor = ahb >= ag::AS;
      unsigned slots = 0;
      for (int k = 0; k < P.nslots; k++)
        if (((P.slotKind[k] == agk::A2_SLOT_ACC || P.slotKind[k] == agk::A2_SLOT_A1) && donor) ||
            (P.slotKind[k] == agk::A2_SLOT_DON && acceptor))
          slots |= 1u << k;
      unsigned plain = 0;
      for (int gg = 0; gg < ps.nm; gg++) plain |= 1u << gg;
      for (int k = 0; k < P.nslots; k++)
        if ((slots >> k) & 1u) plain &= ~(1u << P.slotMap[k]);
      P.typeSlots[t] = slots;
      P.typePlain[t] = plain;
      P.typeDonor[t] = donor ? 1 : 0;
      P.typeAng[t] = ahb == ag::D1 ? agk::A2_D1 : ahb == ag::A1 ? agk::A2_A1 : ahb == ag::A2 ? agk::A2_A2 : agk::A2_SPH;
      for (int k = 0; k < P.nslots; k++)
        if (((slots >> k) & 1u) && P.slotKind[k] == agk::A2_SLOT_ACC && ahb == ag::D1) P.needClosestH = 1;
    }
    for (int k = 0; k < agk::kMaxMapsPass; k++) {
      P.mapCov[k] = k < ps.nm ? c->mapCov[ps.m0 + k] : 1;
      P.solparProbe[k] = k < ps.nm ? (float)c->solparProbe[ps.m0 + k] : 0.f;
      P.volProbe[k] = k < ps.nm ? (float)c->volProbe[ps.m0 + k] : 0.f;
    }
    P.solparQ = (float)c->solparQ;
    P.out = dMaps + (size_t)ps.m0 * c->npoints();
    P.dmap = dDmap;
    P.status = c->status.p;
    out.push_back(P);
  }
  return AG_OK;
}

// Launch parameters of the affinity passes of the staged job.
int buildAffParams(ag_ctx* c, float* dMaps, float* dDmap, std::vector<agk::AffParams>& out) {
  const ag_grid& g = c->grid;
  const int64_t np = c->npoints();
  const int n = c->nAtoms;
  const double h = g.spacing;
  double lo[3];
  int ncell[3];
  cellGrid(g, lo, ncell);
  out.clear();
  const int nt = c->nTypes;
  std::vector<ag_ctx::Pass> passes = c->passes;
  if (passes.empty()) {  // no ligand maps: one pass for the d-map alone
    ag_ctx::Pass ps{};
    ps.nmPad = 4;
    for (int k = 0; k < agk::kMaxMapsPass; k++) ps.mapMinMaxSlot[k] = -1;
    passes.push_back(ps);
  }
  for (const auto& ps : passes) {
    agk::AffParams P{};
    P.n_atoms = n; P.xyz = c->atoms.p; P.info = c->info.p; P.vol = c->vol.p; P.solq = c->solq.p;
    P.rv = c->rv32.p; P.rv2 = c->rv2_32.p; P.rv64 = c->rv64.p;
    P.cellStart = c->cellStart.p; P.cellAtoms = c->cellAtoms.p;
    for (int d = 0; d < 3; d++) { P.cellLo[d] = lo[d]; P.ncell[d] = ncell[d]; }
    P.closestH = c->closestH.p;
    P.nx = g.nx; P.ny = g.ny; P.nz = g.nz; P.n2x = g.nx / 2; P.n2y = g.ny / 2; P.n2z = g.nz / 2;
    P.npoints = np; P.h = h;
    P.nmaps = ps.nm; P.nmPad = ps.nmPad; P.ntypes = nt; P.hydrogen = c->hydrogen;
    P.table = c->affTab.p + ps.tabOff;
    P.tableH = (c->hydrogen >= 0 && c->hydrogen < nt) ? c->affTabH.p + ps.tabHOff : nullptr;
    P.sol = c->sol.p;
    P.thr = c->thrA.p;
    P.delta = 1.0e-3f;
    for (int t = 0; t < agk::kMaxTypes; t++) {
      P.typeHbond[t] = c->typeHbond[t];
      P.typeModes[t] = ps.typeModes[t];
      P.typeNeedsAngular[t] = ps.typeNeedsAngular[t];
    }
    for (int k = 0; k < agk::kMaxMapsPass; k++) {
      P.mapMinMaxSlot[k] = k < ps.nm ? ps.mapMinMaxSlot[k] : -1;
      P.mapCov[k] = k < ps.nm ? c->mapCov[ps.m0 + k] : 1;
      P.solparProbe[k] = k < ps.nm ? (float)c->solparProbe[ps.m0 + k] : 0.f;
      P.volProbe[k] = k < ps.nm ? (float)c->volProbe[ps.m0 + k] : 0.f;
    }
    P.solparQ = (float)c->solparQ;
    P.out = dMaps + (size_t)ps.m0 * np;
    P.dmap = dDmap;
    P.status = c->status.p;
    out.push_back(P);
  }
  return AG_OK;
}

int runAffinity(ag_ctx* c, float* dMaps, float* dDmap) {
  if (int e = prepAffinity(c, c->stream)) return e;
  if (useTwoPoint(c)) {
    std::vector<agk::Aff2Params> passes;
    if (int e = buildAff2Params(c, dMaps, dDmap, passes)) return e;
    for (const auto& P : passes) {
      CK(agk::aff2_launch(P, c->stream));
      c->launches += 1;
    }
    return AG_OK;
  }
  std::vector<agk::AffParams> passes;
  if (int e = buildAffParams(c, dMaps, dDmap, passes)) return e;
  for (const auto& P : passes) {
    CK(agk::aff_launch(P, c->stream));
    c->launches += 1;
  }
  return AG_OK;
}

// The two-point affinity pass in z-slab chunks on the context's stream; as
// each chunk finishes, the copy stream moves its rows of every affinity map
// and of the d-map to `host` (page-locked, laid out [nMaps + 2][npoints] like
// the device buffer).  Blocks run z-slab by z-slab, so a chunk of slabs is a
// contiguous range of rows in every map.
int runAffinityChunked(ag_ctx* c, float* host, int nchunks) {
  const int64_t np = c->npoints();
  const int nm = c->nMaps;
  float* dMaps = c->maps.p;
  float* dDmap = dMaps + (size_t)(nm + 1) * np;
  if (int e = prepAffinity(c, c->stream)) return e;
  std::vector<agk::Aff2Params> passes;
  if (int e = buildAff2Params(c, dMaps, dDmap, passes)) return e;
  const ag_grid& g = c->grid;
  const int tbx = (g.nx + 7) / 8, tby = (g.ny + 7) / 8, slabs = (g.nz + 7) / 8;
  const int64_t plane = (int64_t)g.nx * g.ny;
  nchunks = std::max(1, std::min(nchunks, ag_ctx::kMaxChunks));
  CK(c->ensureCopyStream());
  CK(c->ensureEmapStream());
  for (int k = 0; k < nchunks; k++) {
    const int s0 = slabs * k / nchunks, s1 = slabs * (k + 1) / nchunks;
    if (s1 <= s0) continue;
    for (const auto& P : passes) {
      CK(agk::aff2_launch_range(P, s0 * tbx * tby, s1 * tbx * tby, c->stream));
      c->launches += 1;
    }
    CK(cudaEventRecord(c->evChunk[k], c->stream));
    CK(cudaStreamWaitEvent(c->copyStream, c->evChunk[k], 0));
    const int64_t z0 = 8LL * s0, z1 = std::min<int64_t>(8LL * s1, g.nz);
    const size_t off = (size_t)(z0 * plane), cnt = (size_t)((z1 - z0) * plane);
    if (s0 == 0 && s1 == slabs) {  // one chunk: the affinity maps are one contiguous block
      if (nm) CK(cudaMemcpyAsync(host, dMaps, sizeof(float) * nm * np, cudaMemcpyDeviceToHost, c->copyStream));
    } else {
      for (int m = 0; m < nm; m++)
        CK(cudaMemcpyAsync(host + (size_t)m * np + off, dMaps + (size_t)m * np + off, sizeof(float) * cnt,
                           cudaMemcpyDeviceToHost, c->copyStream));
    }
    CK(cudaMemcpyAsync(host + (size_t)(nm + 1) * np + off, dDmap + off, sizeof(float) * cnt,
                       cudaMemcpyDeviceToHost, c->copyStream));
  }
  return AG_OK;
}

int checkStatus(ag_ctx* c) {
  unsigned st = 0;
  CK(cudaMemcpyAsync(&st, c->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (st) {
    cudaMemsetAsync(c->status.p, 0, sizeof(unsigned), c->stream);
    cudaStreamSynchronize(c->stream);
    return fail(AG_E_DEVICE, "a kernel reported error status 0x%x (1 = bounded wait expired, 2 = bad input)", st);
  }
  // Net-charge checksum of the last e-map: the FP64 sum of the weights the
  // kernel consumed must equal the host's sum of the input weights.
  if (c->checksumSplits > 0) {
    std::vector<double> cs(c->checksumSplits);
    CK(cudaMemcpyAsync(cs.data(), c->checksum.p, sizeof(double) * cs.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double s = 0.0;
    for (double v : cs) s += v;
    c->checksumSplits = 0;
    c->lastChecksum = s;
    const double want = c->wSum + c->testChecksumOffset;
    if (!(std::fabs(s - want) <= 1e-9 * c->wAbsSum + 1e-12))
      return fail(AG_E_DEVICE, "net-charge checksum mismatch: kernel summed %.17g, input holds %.17g", s, want);
  }
  return AG_OK;
}

}  // namespace agc

extern "C" int ag_upload(ag_ctx* c, const ag_grid* g, const ag_receptor* r, const ag_affinity_params* p,
                         const double* inv_eps) {
  if (!c || !r) return fail(AG_E_INVALID, "null argument");
  c->haveJob = false;
  c->haveAff = false;
  if (int e = stageEmap(c, g, r->n_atoms, r->xyzw, inv_eps, false)) return e;
  c->nMaps = 0;
  if (p)
    if (int e = stageAffinity(c, r, p)) return e;
  CK(c->maps.ensure((size_t)(c->nMaps + 2) * c->npoints()));
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(unsigned), c->stream));
  c->haveJob = true;
  return AG_OK;
}

extern "C" int ag_compute(ag_ctx* c, int work) {
  if (!c || !c->haveJob) return fail(AG_E_INVALID, "no job uploaded");
  CK(cudaSetDevice(c->device));
  const int64_t np = c->npoints();
  float* maps = c->maps.p;
  if ((work & AG_WORK_EMAP) && (work & AG_WORK_AFFINITY) && c->haveAff && c->concurrentPasses) {
    // Both passes at once: the e-map's CTAs go first on a high-priority
    // stream and the affinity pass, on the context's stream, takes the SMs
    // its last wave leaves free.  The outputs are disjoint; the context's
    // stream waits for both.
    CK(c->ensureEmapStream());
    CK(cudaEventRecord(c->evFork, c->stream));
    CK(cudaStreamWaitEvent(c->emapStream, c->evFork, 0));
    std::swap(c->stream, c->emapStream);
    int e = runEmap(c, maps + (size_t)c->nMaps * np);
    std::swap(c->stream, c->emapStream);
    if (e) return e;
    CK(cudaEventRecord(c->evJoin, c->emapStream));
    e = runAffinity(c, maps, maps + (size_t)(c->nMaps + 1) * np);
    CK(cudaStreamWaitEvent(c->stream, c->evJoin, 0));
    if (e) return e;
    work &= ~(AG_WORK_EMAP | AG_WORK_AFFINITY);
  }
  if (work & AG_WORK_EMAP)
    if (int e = runEmap(c, maps + (size_t)c->nMaps * np)) return e;
  if (work & AG_WORK_EMAP_SURROGATE)
    if (int e = runEmapSurrogate(c, maps + (size_t)c->nMaps * np)) return e;
  if ((work & AG_WORK_AFFINITY) && c->haveAff)
    if (int e = runAffinity(c, maps, maps + (size_t)(c->nMaps + 1) * np)) return e;
  CK(cudaGetLastError());
  return AG_OK;
}

extern "C" float* ag_device_maps(ag_ctx* c) { return c ? c->maps.p : nullptr; }

extern "C" int ag_download(ag_ctx* c, float* out) {
  if (!c || !c->haveJob || !out) return fail(AG_E_INVALID, "nothing to download");
  CK(cudaMemcpyAsync(out, c->maps.p, sizeof(float) * (size_t)(c->nMaps + 2) * c->npoints(), cudaMemcpyDeviceToHost,
                     c->stream));
  return checkStatus(c);
}

extern "C" int ag_emap_mode(ag_ctx* c, const ag_grid* g, int n, const double* xyzw, const double* inv_eps, int mode,
                            float* out) {
  if (!c || !out) return fail(AG_E_INVALID, "null argument");
  if (mode != AG_EMAP_KAHAN && mode != AG_EMAP_PLAIN) return fail(AG_E_INVALID, "unknown e-map mode %d", mode);
  c->haveJob = false;
  c->haveAff = false;
  c->nMaps = 0;
  if (int e = stageEmap(c, g, n, xyzw, inv_eps, false)) return e;
  CK(c->maps.ensure((size_t)2 * c->npoints()));
  c->emapMode = mode;
  int e = runEmap(c, c->maps.p);
  c->emapMode = agk::kEmapKahan;
  if (e) return e;
  CK(cudaMemcpyAsync(out, c->maps.p, sizeof(float) * c->npoints(), cudaMemcpyDeviceToHost, c->stream));
  return checkStatus(c);
}

extern "C" int ag_emap(ag_ctx* c, const ag_grid* g, int n, const double* xyzw, const double* inv_eps, float* out) {
  return ag_emap_mode(c, g, n, xyzw, inv_eps, AG_EMAP_KAHAN, out);
}

extern "C" int ag_affinity(ag_ctx* c, const ag_grid* g, const ag_receptor* r, const ag_affinity_params* p,
                           float* out_maps, float* out_dmap) {
  if (!c || !r || !p || !out_dmap || (p->n_maps > 0 && !out_maps)) return fail(AG_E_INVALID, "null argument");
  if (int e = ag_upload(c, g, r, p, nullptr)) return e;
  if (int e = ag_compute(c, AG_WORK_AFFINITY)) return e;
  const int64_t np = c->npoints();
  if (p->n_maps)
    CK(cudaMemcpyAsync(out_maps, c->maps.p, sizeof(float) * p->n_maps * np, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(out_dmap, c->maps.p + (size_t)(p->n_maps + 1) * np, sizeof(float) * np, cudaMemcpyDeviceToHost,
                     c->stream));
  return checkStatus(c);
}

// ---------------------------------------------------------------------------
// Whole jobs
// ---------------------------------------------------------------------------
struct ag_problem {
  ag::Problem p;
  std::unique_ptr<ag::ParamLib> lib;
  ag::Log log;
  std::vector<int> mapHbond, mapIsHB, mapCov;
  std::vector<double> solparProbe, volProbe;
  float* pinned = nullptr;  // page-locked host copy of the map set (the D2H copies land here)
  size_t pinnedN = 0;
  const void* xyzwLocked = nullptr;  // p.xyzw, page-locked once for fast uploads (it never moves after loading)
  ~ag_problem() {
    if (pinned) cudaFreeHost(pinned);
    if (xyzwLocked) cudaHostUnregister(const_cast<void*>(xyzwLocked));
  }
};

extern "C" int ag_problem_load(const char* gpf, int v4, const char* log_path, ag_problem** out) {
  if (!out) return fail(AG_E_INVALID, "null output pointer");
  auto* P = new ag_problem();
  try {
    P->log.open(log_path);
    P->lib.reset(new ag::ParamLib(v4 != 0));
    ag::loadGPF(P->p, *P->lib, P->log, gpf);
    ag::precompute(P->p, *P->lib, P->log);
    ag::writeFld(P->p, P->log.programName.c_str(), P->log);
  } catch (ag::ExitProgram& e) {
    delete P;
    return fail(AG_E_HOST, "exit %d: %s", e.code, e.msg.c_str());
  }
  for (auto& m : P->p.maps) {
    P->mapHbond.push_back(m.hbond);
    P->mapIsHB.push_back(m.isHBonder ? 1 : 0);
    P->mapCov.push_back(m.isCovalent ? 1 : 0);
    P->solparProbe.push_back(m.solparProbe);
    P->volProbe.push_back(m.volProbe);
  }
  *out = P;
  return AG_OK;
}

extern "C" void ag_problem_free(ag_problem* p) { delete p; }

extern "C" int ag_problem_info_get(const ag_problem* P, ag_problem_info* info) {
  if (!P || !info) return fail(AG_E_INVALID, "null argument");
  const ag::Problem& p = P->p;
  info->nx = p.n[0]; info->ny = p.n[1]; info->nz = p.n[2];
  info->spacing = p.spacing;
  for (int k = 0; k < 3; k++) info->center[k] = p.center[k];
  info->n_atoms = p.numAtoms;
  info->n_maps = p.numMaps();
  info->n_types = p.numReceptorTypes;
  info->dist_dep_diel = p.distDepDiel;
  info->has_floating_grid = p.hasFloatingGrid();
  return AG_OK;
}

extern "C" int ag_problem_views(const ag_problem* P, ag_grid* g, ag_receptor* r, ag_affinity_params* a,
                                const double** inv_eps) {
  if (!P) return fail(AG_E_INVALID, "null problem");
  const ag::Problem& p = P->p;
  if (g) { g->nx = p.n[0]; g->ny = p.n[1]; g->nz = p.n[2]; g->spacing = p.spacing; }
  if (r) {
    r->n_atoms = p.numAtoms;
    r->xyzw = p.xyzw.data();
    r->charge = p.charge.data(); r->vol = p.vol.data(); r->solpar = p.solpar.data();
    r->type = p.atomType.data(); r->hbond = p.hbond.data();
    r->disorder = p.disorder.data(); r->rexp = p.rexp.data();
    r->rvector = p.rvector.data(); r->rvector2 = p.rvector2.data();
  }
  if (a) {
    a->n_maps = p.numMaps();
    a->n_types = std::max(1, p.numReceptorTypes);
    a->energy = p.energy.data();
    a->sol = p.sol.data();
    a->map_hbond = P->mapHbond.data();
    a->map_is_hbonder = P->mapIsHB.data();
    a->map_is_covalent = P->mapCov.data();
    a->solpar_probe = P->solparProbe.data();
    a->vol_probe = P->volProbe.data();
    a->solpar_q = p.solparQ;
    a->hydrogen = p.hydrogen;
  }
  if (inv_eps) *inv_eps = p.distDepDiel ? p.epsilon.data() : nullptr;
  return AG_OK;
}

extern "C" int ag_problem_compute(ag_ctx* c, ag_problem* P) {
  if (!c || !P) return fail(AG_E_INVALID, "null argument");
  ag::Problem& p = P->p;
  ag_grid g;
  ag_receptor r;
  ag_affinity_params a;
  const double* eps = nullptr;
  ag_problem_views(P, &g, &r, &a, &eps);
  // The atoms are this call's largest upload: page-lock them once so that
  // each call copies them by DMA (a failure only leaves the copy slower).
  if (!P->xyzwLocked && !p.xyzw.empty() &&
      cudaHostRegister(p.xyzw.data(), sizeof(double) * p.xyzw.size(), cudaHostRegisterPortable) == cudaSuccess)
    P->xyzwLocked = p.xyzw.data();
  cudaGetLastError();  // clear a failed registration
  const int nm = p.numMaps();
  bool anyCovalent = false;
  for (int m = 0; m < nm; m++) anyCovalent |= p.maps[m].isCovalent;
  const bool conc = c->concurrentPasses && !anyCovalent;
  // Sequential order: everything staged first.  Concurrent order: the e-map
  // is launched as soon as its own inputs are on the device, and the
  // affinity pass's inputs are staged on the host while it runs.
  if (conc) {
    c->haveJob = false;
    c->haveAff = false;
    if (int e = stageEmap(c, &g, r.n_atoms, r.xyzw, eps, false)) return e;
  } else if (int e = ag_upload(c, &g, &r, &a, eps)) {
    return e;
  }
  const int64_t np = c->npoints();
  const size_t total = (size_t)(nm + 2) * np;
  if (P->pinnedN < total) {
    if (P->pinned) cudaFreeHost(P->pinned);
    P->pinned = nullptr;
    P->pinnedN = 0;
    CK(cudaHostAlloc((void**)&P->pinned, sizeof(float) * total, cudaHostAllocDefault));
    P->pinnedN = total;
  }
  CK(c->ensureCopyStream());
  if (conc) {
    // Both passes at once (as ag_compute runs them): the e-map on the
    // high-priority stream, its 17 MB copied back as soon as it is done; the
    // affinity pass, which fills the SMs the e-map's last wave leaves free,
    // in z-slab chunks whose rows are copied back while later chunks run, so
    // that little of the 184 MB of affinity maps (large configuration) is
    // copied after the last kernel.
    c->nMaps = nm;
    CK(c->maps.ensure(total));
    CK(cudaMemsetAsync(c->status.p, 0, sizeof(unsigned), c->stream));
    CK(c->ensureEmapStream());
    CK(cudaEventRecord(c->evFork, c->stream));
    CK(cudaStreamWaitEvent(c->emapStream, c->evFork, 0));
    std::swap(c->stream, c->emapStream);
    int e = runEmap(c, c->maps.p + (size_t)nm * np);
    std::swap(c->stream, c->emapStream);
    if (e) return e;
    CK(cudaMemcpyAsync(P->pinned + (size_t)nm * np, c->maps.p + (size_t)nm * np, sizeof(float) * np,
                       cudaMemcpyDeviceToHost, c->emapStream));
    CK(cudaEventRecord(c->evJoin, c->emapStream));
    e = stageAffinity(c, &r, &a);
    if (!e) {
      c->haveJob = true;
      if (useTwoPoint(c)) {
        // One chunk per 32 MB of affinity maps, at most four (small jobs:
        // one copy, no per-chunk calls).
        const int chunks = (int)std::max<int64_t>(1, std::min<int64_t>(4, (int64_t)nm * np * 4 / (32 << 20)));
        e = runAffinityChunked(c, P->pinned, chunks);
      } else {
        e = runAffinity(c, c->maps.p, c->maps.p + (size_t)(nm + 1) * np);
        if (!e) {
          CK(cudaEventRecord(c->evAff, c->stream));
          CK(cudaStreamWaitEvent(c->copyStream, c->evAff, 0));
          if (nm) CK(cudaMemcpyAsync(P->pinned, c->maps.p, sizeof(float) * nm * np, cudaMemcpyDeviceToHost,
                                     c->copyStream));
          CK(cudaMemcpyAsync(P->pinned + (size_t)(nm + 1) * np, c->maps.p + (size_t)(nm + 1) * np,
                             sizeof(float) * np, cudaMemcpyDeviceToHost, c->copyStream));
        }
      }
    }
    // Joined on every path: no e-map work may outlive the call.
    CK(cudaStreamWaitEvent(c->stream, c->evJoin, 0));
    if (e) {
      cudaStreamSynchronize(c->stream);
      cudaStreamSynchronize(c->copyStream);
      return e;
    }
  } else {
    // Affinity, d-map and covalent maps first; their copy to the host then
    // runs on a second stream while the e-map (most of the time) is computed.
    if (int e = ag_compute(c, AG_WORK_AFFINITY)) return e;
    for (int m = 0; m < nm; m++)
      if (p.maps[m].isCovalent) {
        CK(agk::covalent_launch(c->maps.p + (size_t)m * np, g.nx, g.ny, g.nz, g.spacing, p.covalentPoint,
                                p.covHalfWidthSquaredInv, p.covBarrier, c->stream));
        c->launches++;
      }
    CK(cudaEventRecord(c->evAff, c->stream));
    CK(cudaStreamWaitEvent(c->copyStream, c->evAff, 0));
    if (nm) CK(cudaMemcpyAsync(P->pinned, c->maps.p, sizeof(float) * nm * np, cudaMemcpyDeviceToHost, c->copyStream));
    CK(cudaMemcpyAsync(P->pinned + (size_t)(nm + 1) * np, c->maps.p + (size_t)(nm + 1) * np, sizeof(float) * np,
                       cudaMemcpyDeviceToHost, c->copyStream));
    if (int e = ag_compute(c, AG_WORK_EMAP)) return e;
    CK(cudaMemcpyAsync(P->pinned + (size_t)nm * np, c->maps.p + (size_t)nm * np, sizeof(float) * np,
                       cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->copyStream));
  if (int e = checkStatus(c)) return e;
  p.out.clear();
  p.outView = P->pinned;
  if (p.hasFloatingGrid()) {
    DevBuf<float> fg;
    CK(fg.ensure(np));
    CK(agk::floating_launch(c->atoms.p, p.numAtoms, g.nx, g.ny, g.nz, g.spacing, fg.p, c->stream));
    c->launches++;
    p.floatingGrid.resize(np);
    CK(cudaMemcpyAsync(p.floatingGrid.data(), fg.p, sizeof(float) * np, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    fg.release();
  }
  return AG_OK;
}

extern "C" const float* ag_problem_maps(const ag_problem* P) {
  return P && (P->p.outView || !P->p.out.empty()) ? P->p.mapData() : nullptr;
}

// ---------------------------------------------------------------------------
// Batches: persistent kernels over the work units of many jobs, one CUDA graph
// ---------------------------------------------------------------------------
struct ag_batch {
  ag_ctx* ctx = nullptr;                 // stream and device of the batch
  std::vector<ag_ctx*> sub;              // per job: staged inputs and outputs
  std::vector<ag_problem*> probs;
  DevBuf<agk::EmapParams> ejobs;
  DevBuf<int2> eunits;
  DevBuf<agk::AffParams> ajobs;
  DevBuf<agk::Aff2Params> a2jobs;        // two-point affinity jobs (when every job allows it)
  bool twoPoint = false;
  DevBuf<int2> aunits;
  DevBuf<int> counters;
  DevBuf<double> checks;                 // per job: net-charge checksum of its e-map (FP64 weight sum)
  std::vector<double> hChecks;
  int ne = 0, na = 0, nmPadMax = 4, nmapsMax = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double pairs = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double lastMs = 0;                     // device time of the last graph launch
};

namespace {

void batchDropGraph(ag_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

int restageItems(ag_ctx* c) {
  buildItems(c);
  CK(c->items.ensure(c->hItems.size()));
  CK(c->blocks.ensure(c->hBlocks.size()));
  CK(cudaMemcpy(c->items.p, c->hItems.data(), sizeof(int) * c->hItems.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->blocks.p, c->hBlocks.data(), sizeof(agk::EmapBlock) * c->hBlocks.size(), cudaMemcpyHostToDevice));
  c->itemsOnDevice = true;
  return AG_OK;
}

// Job parameters and work units (largest jobs first) for the current tile shapes.
int batchBuild(ag_batch* b) {
  batchDropGraph(b);
  std::vector<agk::EmapParams> ej;
  std::vector<agk::AffParams> aj;
  std::vector<agk::Aff2Params> a2j;
  std::vector<std::pair<double, int2>> eu, au;
  b->nmPadMax = 4;
  b->nmapsMax = 0;
  b->pairs = 0;
  CK(b->checks.ensure(b->sub.size()));
  for (size_t i = 0; i < b->sub.size(); i++) {
    ag_ctx* c = b->sub[i];
    const int64_t np = c->npoints();
    agk::EmapParams P;
    if (int e = buildEmapParams(c, c->maps.p + (size_t)c->nMaps * np, false, P)) return e;
    P.checksum = b->checks.p + i;  // written by the job's first CTA box (no atom split in a batch)
    const int j = (int)ej.size();
    ej.push_back(P);
    for (int k = 0; k < P.nblocks; k++)
      eu.push_back({(double)c->nAtoms * c->hBlocks[k].nitems, make_int2(j, k)});
    b->pairs += (double)c->nAtoms * (double)np;
    if (b->twoPoint) {
      std::vector<agk::Aff2Params> passes;
      if (int e = buildAff2Params(c, c->maps.p, c->maps.p + (size_t)(c->nMaps + 1) * np, passes)) return e;
      const int ncta = agk::aff2_ctas(c->grid.nx, c->grid.ny, c->grid.nz);
      for (const auto& A : passes) {
        const int ja = (int)a2j.size();
        a2j.push_back(A);
        b->nmPadMax = std::max(b->nmPadMax, A.nmPad);
        b->nmapsMax = std::max(b->nmapsMax, A.nmaps);
        for (int k = 0; k < ncta; k++) au.push_back({(double)c->nAtoms, make_int2(ja, k)});
      }
      continue;
    }
    std::vector<agk::AffParams> passes;
    if (int e = buildAffParams(c, c->maps.p, c->maps.p + (size_t)(c->nMaps + 1) * np, passes)) return e;
    const int ncta = ((c->grid.nx + agk::kAffTX - 1) / agk::kAffTX) * ((c->grid.ny + agk::kAffTY - 1) / agk::kAffTY) *
                     ((c->grid.nz + agk::kAffTZ - 1) / agk::kAffTZ);
    for (const auto& A : passes) {
      const int ja = (int)aj.size();
      aj.push_back(A);
      b->nmPadMax = std::max(b->nmPadMax, A.nmPad);
      b->nmapsMax = std::max(b->nmapsMax, A.nmaps);
      for (int k = 0; k < ncta; k++) au.push_back({(double)c->nAtoms, make_int2(ja, k)});
    }
  }
  auto byCost = [](const std::pair<double, int2>& x, const std::pair<double, int2>& y) {
    return x.first > y.first || (x.first == y.first && (x.second.x < y.second.x ||
                                                         (x.second.x == y.second.x && x.second.y < y.second.y)));
  };
  std::sort(eu.begin(), eu.end(), byCost);
  std::sort(au.begin(), au.end(), byCost);
  std::vector<int2> eul, aul;
  for (auto& u : eu) eul.push_back(u.second);
  for (auto& u : au) aul.push_back(u.second);
  b->ne = (int)eul.size();
  b->na = (int)aul.size();
  CK(b->ejobs.ensure(ej.size()));
  CK(b->ajobs.ensure(std::max<size_t>(aj.size(), 1)));
  CK(b->a2jobs.ensure(std::max<size_t>(a2j.size(), 1)));
  CK(b->eunits.ensure(eul.size()));
  CK(b->aunits.ensure(aul.size()));
  CK(b->counters.ensure(2));
  CK(cudaMemcpy(b->ejobs.p, ej.data(), sizeof(agk::EmapParams) * ej.size(), cudaMemcpyHostToDevice));
  if (!aj.empty()) CK(cudaMemcpy(b->ajobs.p, aj.data(), sizeof(agk::AffParams) * aj.size(), cudaMemcpyHostToDevice));
  if (!a2j.empty())
    CK(cudaMemcpy(b->a2jobs.p, a2j.data(), sizeof(agk::Aff2Params) * a2j.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->eunits.p, eul.data(), sizeof(int2) * eul.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->aunits.p, aul.data(), sizeof(int2) * aul.size(), cudaMemcpyHostToDevice));
  return AG_OK;
}

int batchSizeClass(const ag_ctx* c) {
  const int a = c->nAtoms < 3000 ? 0 : (c->nAtoms < 10000 ? 1 : 2);
  const int64_t np = const_cast<ag_ctx*>(c)->npoints();
  const int g = np < 200000 ? 0 : (np < 1500000 ? 1 : 2);
  return a * 3 + g;
}

}  // namespace

extern "C" int ag_batch_create(ag_ctx* ctx, ag_problem* const* problems, int n, ag_batch** out) {
  if (!ctx || !problems || n <= 0 || !out) return fail(AG_E_INVALID, "bad batch arguments");
  auto* b = new ag_batch();
  b->ctx = ctx;
  for (int i = 0; i < n; i++) {
    if (!problems[i] || !problems[i]->p.distDepDiel) {
      ag_batch_free(b);
      return fail(AG_E_INVALID, "batch job %d is missing or does not use the distance-dependent dielectric", i);
    }
    ag_ctx* c = nullptr;
    if (int e = ag_ctx_create(ctx->device, &c)) { ag_batch_free(b); return e; }
    c->affKernel = ctx->affKernel;
    b->sub.push_back(c);
    b->probs.push_back(problems[i]);
    ag_grid g;
    ag_receptor r;
    ag_affinity_params a;
    const double* eps = nullptr;
    ag_problem_views(problems[i], &g, &r, &a, &eps);
    if (int e = ag_upload(c, &g, &r, &a, eps)) { ag_batch_free(b); return e; }
  }
  // One affinity kernel for the whole batch: the two-point one if every job's
  // passes allow it.
  b->twoPoint = true;
  for (ag_ctx* c : b->sub) b->twoPoint = b->twoPoint && useTwoPoint(c);
  for (ag_ctx* c : b->sub) {
    if (!b->twoPoint) c->affKernel = 1;
    // Allocate every per-job buffer now (the graph capture must not allocate).
    if (int e = prepAffinity(c, c->stream)) { ag_batch_free(b); return e; }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) { ag_batch_free(b); return fail(AG_E_CUDA, "staging failed"); }
  }
  if (int e = batchBuild(b)) { ag_batch_free(b); return e; }
  *out = b;
  return AG_OK;
}

extern "C" double ag_batch_pairs(const ag_batch* b) { return b ? b->pairs : 0.0; }

extern "C" int ag_batch_compute(ag_batch* b) {
  if (!b) return fail(AG_E_INVALID, "null batch");
  cudaStream_t st = b->ctx->stream;
  CK(cudaSetDevice(b->ctx->device));
  if (!b->exec) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->ctx->device);
    // The e-map units and the affinity units are independent: with concurrent
    // passes the graph holds them as two branches, the e-map's on the
    // context's high-priority stream, so the affinity kernel's CTAs take the
    // SMs the e-map kernel's last units leave free.
    ag_ctx* bc = b->ctx;
    const bool conc = bc->concurrentPasses != 0;
    if (conc) CK(bc->ensureEmapStream());
    cudaStream_t est = conc ? bc->emapStream : st;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int err = AG_OK;
    // NaN in every checksum slot until the job's e-map writes it.
    if (cudaMemsetAsync(b->checks.p, 0xFF, sizeof(double) * b->sub.size(), st) != cudaSuccess)
      err = fail(AG_E_CUDA, "batch checksum reset failed");
    if (!err && conc &&
        (cudaEventRecord(bc->evFork, st) != cudaSuccess || cudaStreamWaitEvent(est, bc->evFork, 0) != cudaSuccess))
      err = fail(AG_E_CUDA, "batch graph fork failed");
    if (!err && agk::emap_batch_launch(b->ejobs.p, b->eunits.p, b->ne, b->counters.p, 2 * sms, est) != cudaSuccess)
      err = fail(AG_E_CUDA, "batch e-map launch failed");
    if (!err && conc && cudaEventRecord(bc->evJoin, est) != cudaSuccess)
      err = fail(AG_E_CUDA, "batch graph join failed");
    for (ag_ctx* c : b->sub)
      if (!err) err = prepAffinity(c, st);
    if (!err) {
      const cudaError_t ae =
          b->twoPoint ? agk::aff2_batch_launch(b->a2jobs.p, b->aunits.p, b->na, b->counters.p + 1, b->nmPadMax,
                                               b->nmapsMax, 2 * sms, st)
                      : agk::aff_batch_launch(b->ajobs.p, b->aunits.p, b->na, b->counters.p + 1, b->nmPadMax,
                                              b->nmapsMax, 2 * sms, st);
      if (ae != cudaSuccess) err = fail(AG_E_CUDA, "batch affinity launch failed");
    }
    if (conc && cudaStreamWaitEvent(st, bc->evJoin, 0) != cudaSuccess && !err)
      err = fail(AG_E_CUDA, "batch graph join failed");
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (err) {
      if (g) cudaGraphDestroy(g);
      return err;
    }
    if (ce != cudaSuccess) return fail(AG_E_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
    b->graph = g;
    CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  }
  if (!b->ev[0]) {
    CK(cudaEventCreate(&b->ev[0]));
    CK(cudaEventCreate(&b->ev[1]));
  }
  CK(cudaEventRecord(b->ev[0], st));
  CK(cudaGraphLaunch(b->exec, st));
  CK(cudaEventRecord(b->ev[1], st));
  b->ctx->launches += 2 + 9 * (int64_t)b->sub.size();
  CK(cudaStreamSynchronize(st));
  {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
    b->lastMs = ms;
  }
  for (ag_ctx* c : b->sub) {
    c->checksumSplits = 0;
    if (int e = checkStatus(c)) return e;
  }
  // Net-charge checksum of every job's e-map: the FP64 sum of the weights its
  // kernel consumed must equal the host's sum of the job's input weights.
  b->hChecks.resize(b->sub.size());
  CK(cudaMemcpy(b->hChecks.data(), b->checks.p, sizeof(double) * b->sub.size(), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < b->sub.size(); i++) {
    const ag_ctx* c = b->sub[i];
    if (!(std::fabs(b->hChecks[i] - c->wSum) <= 1e-9 * c->wAbsSum + 1e-12))
      return fail(AG_E_DEVICE, "net-charge checksum mismatch in batch job %d: kernel summed %.17g, input holds %.17g",
                  (int)i, b->hChecks[i], c->wSum);
  }
  return AG_OK;
}

extern "C" double ag_batch_last_ms(const ag_batch* b) { return b ? b->lastMs : 0.0; }

extern "C" int ag_batch_download(ag_batch* b, int i, float* out) {
  if (!b || i < 0 || i >= (int)b->sub.size() || !out) return fail(AG_E_INVALID, "bad batch download");
  ag_ctx* c = b->sub[i];
  CK(cudaMemcpyAsync(out, c->maps.p, sizeof(float) * (size_t)(c->nMaps + 2) * c->npoints(), cudaMemcpyDeviceToHost,
                     b->ctx->stream));
  CK(cudaStreamSynchronize(b->ctx->stream));
  return AG_OK;
}

extern "C" int ag_batch_autotune(ag_batch* b, const char* cache_path) {
  if (!b) return fail(AG_E_INVALID, "null batch");
  static const int kCand[][3] = {{2, 16, 8}, {4, 8, 8}, {1, 16, 16}, {2, 8, 16}, {4, 16, 4}};
  const int ncand = sizeof(kCand) / sizeof(kCand[0]);
  int choice[9];
  for (int k = 0; k < 9; k++) choice[k] = -1;
  if (cache_path && cache_path[0]) {
    if (FILE* f = fopen(cache_path, "r")) {
      int cls, x, y, z;
      while (fscanf(f, "emap_tile class=%d tile=%d,%d,%d\n", &cls, &x, &y, &z) == 4)
        for (int k = 0; k < ncand && cls >= 0 && cls < 9; k++)
          if (kCand[k][0] == x && kCand[k][1] == y && kCand[k][2] == z) choice[cls] = k;
      fclose(f);
    }
  }
  cudaStream_t st = b->ctx->stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int cls = 0; cls < 9; cls++) {
    if (choice[cls] >= 0) continue;
    // The median-sized job of the class stands for it.
    std::vector<std::pair<double, ag_ctx*>> js;
    for (ag_ctx* c : b->sub)
      if (batchSizeClass(c) == cls) js.push_back({(double)c->nAtoms * (double)c->npoints(), c});
    if (js.empty()) continue;
    std::sort(js.begin(), js.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    ag_ctx* c = js[js.size() / 2].second;
    float best = 1e30f;
    for (int k = 0; k < ncand; k++) {
      for (int d = 0; d < 3; d++) c->tile[d] = kCand[k][d];
      if (int e = restageItems(c)) return e;
      agk::EmapParams P;
      if (int e = buildEmapParams(c, c->maps.p + (size_t)c->nMaps * c->npoints(), false, P)) return e;
      float tms = 1e30f;
      for (int rep = 0; rep < 3; rep++) {
        cudaEventRecord(e0, st);
        if (agk::emap_launch(P, true, agk::kEmapKahan, P.nblocks, st) != cudaSuccess) return fail(AG_E_CUDA, "tuning launch failed");
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) tms = std::min(tms, ms);
      }
      if (tms < best) {
        best = tms;
        choice[cls] = k;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (ag_ctx* c : b->sub) {
    const int k = choice[batchSizeClass(c)] >= 0 ? choice[batchSizeClass(c)] : 0;
    for (int d = 0; d < 3; d++) c->tile[d] = kCand[k][d];
    if (int e = restageItems(c)) return e;
  }
  if (cache_path && cache_path[0]) {
    if (FILE* f = fopen(cache_path, "w")) {
      for (int cls = 0; cls < 9; cls++)
        if (choice[cls] >= 0)
          fprintf(f, "emap_tile class=%d tile=%d,%d,%d\n", cls, kCand[choice[cls]][0], kCand[choice[cls]][1],
                  kCand[choice[cls]][2]);
      fclose(f);
    }
  }
  return batchBuild(b);
}

extern "C" int ag_batch_free(ag_batch* b) {
  if (!b) return AG_OK;
  batchDropGraph(b);
  b->ejobs.release();
  b->eunits.release();
  b->ajobs.release();
  b->aunits.release();
  b->counters.release();
  b->checks.release();
  b->a2jobs.release();
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  for (ag_ctx* c : b->sub) ag_ctx_destroy(c);
  delete b;
  return AG_OK;
}

extern "C" int ag_problem_write(ag_problem* P) {
  if (!P || (P->p.out.empty() && !P->p.outView)) return fail(AG_E_INVALID, "no computed maps");
  try {
    ag::writeAllMaps(P->p, P->log);
    ag::writeFloatingGrid(P->p, P->log);
  } catch (ag::ExitProgram& e) {
    return fail(AG_E_HOST, "exit %d: %s", e.code, e.msg.c_str());
  }
  return AG_OK;
}

// ---------------------------------------------------------------------------
// Command line (ProgramParameters.cpp:63-112, main.cpp:115-279)
// ---------------------------------------------------------------------------
namespace {

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double ms() const { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); }
};

void printHelp(const char* prog) {
  fprintf(stderr,
          "Usage: %s [OPTIONS]\n\n"
          "Stream control:\n"
          "  -l, --log FILE    log to FILE, default: standard output\n"
          "  -p, --gpf FILE    read grid parameters from FILE, default: standard input\n\n"
          "Miscellaneous:\n"
          "      --benchmark   print execution times to standard error output\n"
          "      --cuda-enum   enumerate all CUDA devices and exit\n"
          "      --cuda-dev N  use a CUDA device number N, default: 0\n"
          "  -d, --debug       increment debug level\n"
          "  -u, --help        display this help and exit\n"
          "      --timeout N   terminate if calculations does not finish in N seconds\n"
          "      --v4          set the AutoGrid 4.0 default parameter library\n\n"
          "Accepted for compatibility and ignored (the maps are always computed on the GPU):\n"
          "      --no-cuda --omp N --cogrid-mem N --no-cogrid --no-nns\n"
          "      --cuda-ddd=g|c|t|i --cuda-slices=y|n --cuda-thread=y|n --cuda-unroll=y|n\n",
          prog);
}

int runMain(int argc, char** argv) {
  const char* prog = argv[0];
  std::string gpf, logf;
  bool bench = false, v4 = false;
  int dev = 0;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto needArg = [&](void) -> const char* {
      if (i + 1 >= argc) throw ag::ExitProgram{1, "missing argument for " + a};
      return argv[++i];
    };
    auto needInt = [&](void) -> int {
      const char* s = needArg();
      int v;
      if (sscanf(s, "%i", &v) != 1) {
        fprintf(stderr, "%s: '%s' is not a number\n", prog, s);
        throw ag::ExitProgram{1, "not a number"};
      }
      return v;
    };
    if (a == "-l" || a == "--log") logf = needArg();
    else if (a == "-p" || a == "--gpf") gpf = needArg();
    else if (a == "--benchmark") bench = true;
    else if (a == "--cogrid-mem" || a == "--omp") needInt();
    else if (a == "--cuda-enum") {
      int n = 0;
      cudaGetDeviceCount(&n);
      fprintf(stderr, "Found %i CUDA devices:\n\n # | Name                           | MPs | Cap | GlobalMem\n", n);
      for (int d = 0; d < n; d++) {
        cudaDeviceProp pr;
        cudaGetDeviceProperties(&pr, d);
        fprintf(stderr, "%2i | %-31s|%4i |%2i.%-2i|%6lu MiB\n", d, pr.name, pr.multiProcessorCount, pr.major, pr.minor,
                (unsigned long)(pr.totalGlobalMem >> 20));
      }
      return 0;
    } else if (a == "--cuda-dev") dev = needInt();
    else if (a == "-d" || a == "--debug") {}
    else if (a == "-u" || a == "--help") { printHelp(prog); return 0; }
    else if (a == "--no-cuda" || a == "--no-cogrid" || a == "--no-nns" || a.rfind("--cuda-ddd=", 0) == 0 ||
             a.rfind("--cuda-slices=", 0) == 0 || a.rfind("--cuda-thread=", 0) == 0 || a.rfind("--cuda-unroll=", 0) == 0) {}
    else if (a == "--timeout") {
      int secs = needInt();
      pid_t pid = fork();
      if (pid > 0) {
        int status = 0;
        for (int t = 0; t < secs * 10; t++) {
          if (waitpid(pid, &status, WNOHANG) == pid) return 0;
          usleep(100000);
        }
        kill(pid, SIGKILL);
        waitpid(pid, &status, 0);
        fprintf(stderr, "Timeout! Process terminated.\n");
        return 0;
      }
    } else if (a == "--v4") v4 = true;
    else {
      fprintf(stderr, "%s: unknown switch '%s'\n", prog, a.c_str());
      return 1;
    }
  }

  Timer total;
  ag::Problem p;
  ag::Log log;
  log.programName = prog;
  log.open(logf.c_str());
  log.print("%s 4.2.1 (B200 map engine)\n\n", prog);
  ag::ParamLib lib(v4);
  // The CUDA context (the longest host step) is created on a second thread
  // while this one parses the inputs and builds the tables.
  struct CtxStart {
    ag_ctx* ctx = nullptr;
    int rc = AG_OK;
    std::string err;
    std::thread th;
    ~CtxStart() {  // also on the error paths of the host steps
      if (th.joinable()) th.join();
      if (ctx) ag_ctx_destroy(ctx);
    }
  } cs;
  Timer tc;
  cs.th = std::thread([&cs, dev] {
    cs.rc = ag_ctx_create(dev, &cs.ctx);
    if (cs.rc != AG_OK) cs.err = ag_last_error();
  });
  Timer t0;
  ag::loadGPF(p, lib, log, gpf.empty() ? nullptr : gpf.c_str());
  const double parseMs = t0.ms();
  double preMs[2] = {0, 0};
  ag::precompute(p, lib, log, preMs);
  Timer tf;
  ag::writeFld(p, prog, log);
  const double fldMs = tf.ms();
  if (bench) {
    fprintf(stderr, "Parsing GPF and PDBQT    Real: %.1f ms\n", parseMs);
    fprintf(stderr, "Energy tables            Real: %.1f ms\n", preMs[0]);
    fprintf(stderr, "Bond vectors             Real: %.1f ms\n", preMs[1]);
    fprintf(stderr, "Writing .fld             Real: %.1f ms\n", fldMs);
  }

  Timer tw;
  cs.th.join();
  if (cs.rc != AG_OK) log.fatal(-2, "%s", cs.err.c_str());
  ag_ctx* ctx = cs.ctx;
  cs.ctx = nullptr;
  if (bench) {
    fprintf(stderr, "CUDA context             Real: %.1f ms\n", tc.ms());
    fprintf(stderr, "  (waited after the host steps: %.1f ms)\n", tw.ms());
  }
  ag_problem P;
  P.p = std::move(p);
  for (auto& m : P.p.maps) {
    P.mapHbond.push_back(m.hbond);
    P.mapIsHB.push_back(m.isHBonder ? 1 : 0);
    P.mapCov.push_back(m.isCovalent ? 1 : 0);
    P.solparProbe.push_back(m.solparProbe);
    P.volProbe.push_back(m.volProbe);
  }
  Timer t1;
  if (ag_problem_compute(ctx, &P) != AG_OK) {
    std::string e = ag_last_error();
    ag_ctx_destroy(ctx);
    log.fatal(-2, "%s", e.c_str());
  }
  const double gpuMs = t1.ms();
  ag_ctx_destroy(ctx);
  if (bench) {
    fprintf(stderr, "Grid maps (GPU)          Real: %.1f ms\n", gpuMs);
    double pairs = (double)P.p.numAtoms * (double)P.p.numPoints;
    fprintf(stderr, "Electrostatics performance: %i million atoms/s (whole map set)\n", (int)(pairs / (gpuMs * 1e-3) / 1e6));
  }
  Timer t2;
  ag::writeAllMaps(P.p, log);
  ag::writeFloatingGrid(P.p, log);
  if (bench) fprintf(stderr, "Saving maps              Real: %.1f ms\n", t2.ms());

  // Summary of extrema (GridMap.cpp:53-82), over the rounded values.
  log.print("\nGrid\tAtom\tMinimum   \tMaximum\nMap \tType\tEnergy    \tEnergy \n\t\t(kcal/mol)\t(kcal/mol)\n____\t____\t_____________\t_____________\n");
  const int64_t np = P.p.numPoints;
  for (int m = 0; m < P.p.numMaps() + 2; m++) {
    double mn = ag::kBig, mx = -ag::kBig;
    for (int64_t j = 0; j < np; j++) {
      double v = ag::roundOutput(P.p.mapData()[(size_t)m * np + j]);
      mn = std::min(mn, v);
      mx = std::max(mx, v);
    }
    const char* type = m < P.p.numMaps() ? P.p.maps[m].type : (m == P.p.numMaps() ? "e" : "d");
    log.print(" %d\t %s\t  %6.2lf\t%9.2le\n", m + 1, type, mn, mx);
  }
  log.print("\n\n * Note:  Every pairwise-atomic interaction was clamped at %.2f\n\n\n", ag::kEintClamp);
  fprintf(stderr, "\n%s: Successful Completion.\n", prog);
  log.print("%s: Successful Completion.\n", prog);
  if (bench) fprintf(stderr, "Total                    Real: %.1f ms\n", total.ms());
  return 0;
}

}  // namespace

extern "C" int ag_main(int argc, char** argv) {
  try {
    return runMain(argc, argv);
  } catch (ag::ExitProgram& e) {
    return e.code;
  } catch (std::bad_alloc&) {
    fprintf(stderr, "\n%s: FATAL ERROR: Not enough memory!\n", argv[0]);
    return (int)0xBADA110C;
  }
}
