// E-map entry point that performs no device memory allocation.
//
// Who needs it: hosts that embed the map engine in a process whose GPU memory
// they manage themselves — a docking service that reserves the device's memory
// up front in its own pool, or a pipeline stage with a fixed memory budget that
// must not call cudaMalloc/cudaFree mid-run (those calls can synchronise the
// device and fail under memory pressure).  Such callers pass device-resident
// inputs and output buffers; every other buffer the e-map kernel needs lives in
// the fixed-size, file-scope device arrays below.
//
// Limits: at most kNaMaxItems = 1,048,576 work items of 8 x-points (about
// 8.4 million grid points, e.g. 201^3), and the atom-split partial sums are
// limited to kNaMaxPartial = 2,097,152 doubles (the split count is reduced to
// fit).  Larger grids are rejected with AG_E_INVALID.  The arrays take about
// 21 MiB on every device that loads the library, until the process exits.
//
// Sharing: every call, from any thread or stream, uses the same device arrays,
// and they keep the previous call's contents.  Calls whose GPU work overlaps
// race on them; serialise such calls (same stream, or wait between them).
// The per-device set-up (symbol addresses, the bin-threshold table) happens on
// the first call on each device; make that first call before any stream
// capture on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/fastgrid_b200.h"
#include "ag_kernels.h"

namespace ag {
void setLastError(const char* msg);  // capi.cu
}

namespace {

constexpr int kNaMaxItems = 1 << 20;             // 4 MiB of work items
constexpr int kNaMaxBlocks = (kNaMaxItems + 255) / 256;
constexpr int64_t kNaMaxPartial = 1 << 21;       // 16 MiB of FP64 partial sums
constexpr int kNaThr = 8193;

static __device__ __align__(256) double g_naPartial[kNaMaxPartial];
static __device__ __align__(256) int g_naItems[kNaMaxItems];
static __device__ __align__(256) agk::EmapBlock g_naBlocks[kNaMaxBlocks];
static __device__ __align__(256) double g_naThr[kNaThr];
static __device__ __align__(256) unsigned g_naStatus[64];

struct NaDevice {
  bool ready = false;
  double* partial = nullptr;
  int* items = nullptr;
  agk::EmapBlock* blocks = nullptr;
  double* thr = nullptr;
  unsigned* status = nullptr;
};

constexpr int kNaMaxDevices = 64;
NaDevice g_dev[kNaMaxDevices];
std::mutex g_mu;

// Host staging (static, so the entry point allocates nothing on the host either).
int g_hItems[kNaMaxItems];
agk::EmapBlock g_hBlocks[kNaMaxBlocks];
double g_hThr[kNaThr];
bool g_thrReady = false;

int naFail(int code, const char* msg) {
  ag::setLastError(msg);  // read back with ag_last_error()
  return code;
}

// thr[k]: least double r^2 whose bin int(sqrt(r^2) * 100.0) is >= k.
void naThresholds() {
  if (g_thrReady) return;
  g_hThr[0] = 0.0;
  for (int k = 1; k < kNaThr; k++) {
    double lo = 0.0, hi = (k / 100.0 + 1.0) * (k / 100.0 + 1.0);
    uint64_t a, b;
    memcpy(&a, &lo, 8);
    memcpy(&b, &hi, 8);
    while (b - a > 1) {
      const uint64_t m = a + (b - a) / 2;
      double v;
      memcpy(&v, &m, 8);
      if (sqrt(v) * 100.0 >= (double)k) b = m; else a = m;
    }
    memcpy(&g_hThr[k], &b, 8);
  }
  g_thrReady = true;
}

int naSetup(int dev, NaDevice& d) {
  if (d.ready) return AG_OK;
  if (cudaGetSymbolAddress((void**)&d.partial, g_naPartial) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.items, g_naItems) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.blocks, g_naBlocks) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.thr, g_naThr) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.status, g_naStatus) != cudaSuccess)
    return naFail(AG_E_CUDA, "cudaGetSymbolAddress failed for the no-allocation scratch arrays");
  naThresholds();
  if (cudaMemcpy(d.thr, g_hThr, sizeof g_hThr, cudaMemcpyHostToDevice) != cudaSuccess)
    return naFail(AG_E_CUDA, "cannot initialise the bin threshold table");
  (void)dev;
  d.ready = true;
  return AG_OK;
}

// Work items (8 x points of one row) in 2 x 16 x 8 tiles, boustrophedon order,
// 256 per CTA, with each CTA's box; returns the number of CTAs or -1 if the
// grid needs more than kNaMaxItems items.
int naItems(const ag_grid& g, int& nitems) {
  const int nxc = (g.nx + agk::kNX - 1) / agk::kNX;
  const int64_t need = (int64_t)nxc * g.ny * g.nz;
  if (need > kNaMaxItems) return -1;
  const int TX = 2, TY = 16, TZ = 8;
  const int ntx = (nxc + TX - 1) / TX, nty = (g.ny + TY - 1) / TY, ntz = (g.nz + TZ - 1) / TZ;
  int n = 0, serp = 0;
  for (int kz = 0; kz < ntz; kz++)
    for (int ky0 = 0; ky0 < nty; ky0++) {
      const int ky = (kz & 1) ? nty - 1 - ky0 : ky0;
      for (int kx0 = 0; kx0 < ntx; kx0++, serp++) {
        const int kx = (serp / ntx) & 1 ? ntx - 1 - kx0 : kx0;
        for (int z = kz * TZ; z < std::min(g.nz, kz * TZ + TZ); z++)
          for (int y = ky * TY; y < std::min(g.ny, ky * TY + TY); y++)
            for (int x = kx * TX; x < std::min(nxc, kx * TX + TX); x++) g_hItems[n++] = x | (y << 8) | (z << 19);
      }
    }
  nitems = n;
  const double h = g.spacing;
  const int n2x = g.nx / 2, n2y = g.ny / 2, n2z = g.nz / 2;
  int nb = 0;
  for (int i0 = 0; i0 < n; i0 += 256, nb++) {
    agk::EmapBlock b{};
    b.item0 = i0;
    b.nitems = std::min(256, n - i0);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < b.nitems; k++) {
      const int v = g_hItems[i0 + k];
      const int xc = v & 0xFF, y = (v >> 8) & 0x7FF, z = (v >> 19) & 0x7FF;
      const int xa = xc * agk::kNX, xb = std::min(g.nx - 1, xa + agk::kNX - 1);
      const double p[2][3] = {{(xa - n2x) * h, (y - n2y) * h, (z - n2z) * h},
                              {(xb - n2x) * h, (y - n2y) * h, (z - n2z) * h}};
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
    const double diag = 2.0 * std::sqrt((double)b.hx * b.hx + (double)b.hy * b.hy + (double)b.hz * b.hz) / 100.0;
    const double rFar = std::max(50.0, std::min(60.0, 81.0 - diag));
    b.rfar2 = (float)((100.0 * rFar) * (100.0 * rFar));
    b.clampMid = rFar + diag >= 81.0 ? 1 : 0;
    g_hBlocks[nb] = b;
  }
  return nb;
}

}  // namespace

extern "C" int ag_emap_noalloc(const ag_grid* grid, int n_atoms, const double* d_xyzw, const float* d_inv_eps,
                               float* d_out, void* stream) {
  if (!grid || !d_out || n_atoms < 0 || (n_atoms > 0 && !d_xyzw))
    return naFail(AG_E_INVALID, "null argument or negative atom count");
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || grid->nx > 1025 || grid->ny > 1025 || grid->nz > 1025 ||
      !(grid->spacing > 0))
    return naFail(AG_E_INVALID, "grid outside 1..1025 points per axis or bad spacing");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices)
    return naFail(AG_E_CUDA, "no current CUDA device");
  std::lock_guard<std::mutex> lock(g_mu);
  NaDevice& D = g_dev[dev];
  if (int e = naSetup(dev, D)) return e;
  cudaStream_t st = (cudaStream_t)stream;
  int nitems = 0;
  const int nblocks = naItems(*grid, nitems);
  if (nblocks < 0)
    return naFail(AG_E_INVALID, "grid too large for ag_emap_noalloc (more than 1048576 work items of 8 points)");
  const int64_t np = (int64_t)grid->nx * grid->ny * grid->nz;
  if (n_atoms == 0) {
    if (cudaMemsetAsync(d_out, 0, sizeof(float) * np, st) != cudaSuccess) return naFail(AG_E_CUDA, "memset failed");
    return AG_OK;
  }
  if (cudaMemcpyAsync(D.items, g_hItems, sizeof(int) * nitems, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(D.blocks, g_hBlocks, sizeof(agk::EmapBlock) * nblocks, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemsetAsync(D.status, 0, sizeof(unsigned), st) != cudaSuccess)
    return naFail(AG_E_CUDA, "cannot stage the work list");
  // The host staging arrays are reused by the next call: wait for the copies.
  if (cudaStreamSynchronize(st) != cudaSuccess) return naFail(AG_E_CUDA, "stream error");

  agk::EmapParams P{};
  P.atoms = reinterpret_cast<const double4*>(d_xyzw);
  P.n_atoms = n_atoms;
  P.nblocks = nblocks;
  P.items = D.items;
  P.blocks = D.blocks;
  P.nx = grid->nx; P.ny = grid->ny; P.nz = grid->nz;
  P.n2x = P.nx / 2; P.n2y = P.ny / 2; P.n2z = P.nz / 2;
  P.npoints = np;
  P.h = grid->spacing;
  P.table = d_inv_eps;
  P.thr = D.thr;
  P.rnear2 = (100.f * 14.0f) * (100.f * 14.0f);
  P.delta = 2.0e-3f;
  P.out = d_out;
  P.status = D.status;
  // Split atoms across CTAs when the grid alone cannot fill the GPU, within the
  // partial-sum array's capacity.
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int want = 2 * agk::kEmapCtasPerSm * sms;
  int nsplit = 1;
  if (nblocks < want && n_atoms > 512) nsplit = std::min((want + nblocks - 1) / nblocks, (n_atoms + 255) / 256);
  while (nsplit > 1 && (int64_t)nsplit * np > kNaMaxPartial) nsplit--;
  int chunk = ((n_atoms + nsplit - 1) / nsplit + 255) / 256 * 256;
  nsplit = std::max(1, (n_atoms + chunk - 1) / chunk);
  P.chunk = chunk;
  P.nsplit = nsplit;
  P.partial = nsplit > 1 ? D.partial : nullptr;
  if (agk::emap_launch(P, d_inv_eps != nullptr, agk::kEmapKahan, nblocks * nsplit, st) != cudaSuccess)
    return naFail(AG_E_CUDA, "e-map launch failed");
  unsigned status = 0;
  if (cudaMemcpyAsync(&status, D.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return naFail(AG_E_CUDA, "e-map kernel failed");
  if (status) return naFail(AG_E_DEVICE, "the e-map kernel reported an error status (bounded wait expired)");
  return AG_OK;
}
