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
// fit).  Larger grids are rejected with AG_E_INVALID before any CUDA call, and
// so are input pointers that are not 16-byte aligned (the kernel reads atoms
// by 16-byte bulk copies and the table as float4).  The arrays take about
// 21 MiB on every device that loads the library, until the process exits.
//
// Sharing: every call, from any thread or stream, uses the same device arrays,
// and they keep the previous call's contents.  Calls whose GPU work overlaps
// race on them; serialise such calls (same stream, or wait between them).
// The dielectric table is read back to the host on every call (32 KB) and its
// saturating tail packed into 16- and 8-bit copies in a fixed device array, as
// the ordinary entry points do.
//
// The per-device set-up (symbol addresses, the bin-threshold table) happens on
// the first call on each device, and again on the first call after the
// device's context was re-created (e.g. after cudaDeviceReset); make that
// first call before any stream capture on the device.  The call is
// synchronous: it returns when its GPU work has finished.
//
// Net-charge checksum: the e-map kernel's first CTA of every atom split sums,
// in FP64, the weights of the atoms that went through its tile ring; a
// separate one-CTA kernel sums the input weights directly.  The call fails
// with AG_E_DEVICE if the two differ (a lost or duplicated atom tile).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cuda.h>
#include <mutex>

#include "../../include/fastgrid_b200.h"
#include "ag_kernels.h"

namespace ag {
void setLastError(const char* msg);  // capi.cu
}
namespace agc {
void emapBinThresholdsInto(double* thr);  // capi.cu: fills thr[0 .. 8192], no allocation
int packTableTailInto(const float* t, int n, unsigned char* raw, int cap, int& b16, int& b8, int& vec8,
                      float& kScale);  // capi.cu: packed tail tables of the dielectric table, no allocation
}

namespace {

constexpr int kNaMaxItems = 1 << 20;             // 4 MiB of work items
constexpr int kNaMaxBlocks = (kNaMaxItems + 255) / 256;
constexpr int64_t kNaMaxPartial = 1 << 21;       // 16 MiB of FP64 partial sums
constexpr int kNaThr = 8193;
constexpr int kNaMaxSplit = 1024;                // atom splits (checksum slots)

static __device__ __align__(256) double g_naPartial[kNaMaxPartial];
static __device__ __align__(256) int g_naItems[kNaMaxItems];
static __device__ __align__(256) agk::EmapBlock g_naBlocks[kNaMaxBlocks];
static __device__ __align__(256) double g_naThr[kNaThr];
static __device__ __align__(256) unsigned g_naStatus[64];
static __device__ __align__(256) double g_naChecksum[kNaMaxSplit];
static __device__ __align__(256) double g_naWeights[2];  // input sum w, sum |w|
static __device__ __align__(256) uint4 g_naPacked[agk::kEmapPackedBytes / 16];  // packed table tail

struct NaDevice {
  bool ready = false;
  unsigned long long ctxId = 0;  // the context the set-up was done in
  double* partial = nullptr;
  int* items = nullptr;
  agk::EmapBlock* blocks = nullptr;
  double* thr = nullptr;
  unsigned* status = nullptr;
  double* checksum = nullptr;
  double* weights = nullptr;
  uint4* packed = nullptr;
};

constexpr int kNaMaxDevices = 64;
NaDevice g_dev[kNaMaxDevices];
std::mutex g_mu;

// Host staging (static, so the entry point allocates nothing on the host either).
int g_hItems[kNaMaxItems];
agk::EmapBlock g_hBlocks[kNaMaxBlocks];
double g_hThr[kNaThr];
bool g_thrReady = false;
double g_hChecksum[kNaMaxSplit];
double g_hWeights[2];
float g_hTab[8192];
alignas(16) unsigned char g_hPacked[agk::kEmapPackedBytes];

int naFail(int code, const char* msg) {
  ag::setLastError(msg);  // read back with ag_last_error()
  return code;
}

// thr[k]: least double r^2 whose bin int(sqrt(r^2) * 100.0) is >= k (the
// table the ordinary e-map entry points use, written into the static array).
void naThresholds() {
  if (g_thrReady) return;
  agc::emapBinThresholdsInto(g_hThr);
  g_thrReady = true;
}

// Unique id of the calling thread's current CUDA context, through the driver
// entry points the runtime exposes (the library does not link libcuda).
bool naContextId(unsigned long long& id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent getCurrent = nullptr;
  static GetId getId = nullptr;
  if (!getCurrent || !getId) {
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
      return false;
    getCurrent = reinterpret_cast<GetCurrent>(a);
    getId = reinterpret_cast<GetId>(b);
  }
  CUcontext ctx = nullptr;
  if (getCurrent(&ctx) != CUDA_SUCCESS || !ctx) return false;
  return getId(ctx, &id) == CUDA_SUCCESS;
}

// Sum of the input weights (w of every atom) and of their magnitudes, in FP64,
// by one CTA in a fixed order: the reference value of the net-charge checksum.
__global__ void na_weight_sum_kernel(const double4* __restrict__ atoms, int n, double* out) {
  __shared__ double s[2][256];
  double w = 0.0, a = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = atoms[i].w;
    w += v;
    a += fabs(v);
  }
  s[0][threadIdx.x] = w;
  s[1][threadIdx.x] = a;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s[0][threadIdx.x] += s[0][threadIdx.x + o];
      s[1][threadIdx.x] += s[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = s[0][0];
    out[1] = s[1][0];
  }
}

// Symbol addresses of the scratch arrays in the current context, and (once
// per context) the bin-threshold table.
int naSetup(NaDevice& d) {
  if (cudaGetSymbolAddress((void**)&d.partial, g_naPartial) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.items, g_naItems) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.blocks, g_naBlocks) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.thr, g_naThr) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.status, g_naStatus) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.checksum, g_naChecksum) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.weights, g_naWeights) != cudaSuccess ||
      cudaGetSymbolAddress((void**)&d.packed, g_naPacked) != cudaSuccess)
    return naFail(AG_E_CUDA, "cudaGetSymbolAddress failed for the no-allocation scratch arrays");
  unsigned long long id = 0;
  if (!naContextId(id)) return naFail(AG_E_CUDA, "cannot identify the current CUDA context");
  if (d.ready && d.ctxId == id) return AG_OK;
  naThresholds();
  if (cudaMemcpy(d.thr, g_hThr, sizeof g_hThr, cudaMemcpyHostToDevice) != cudaSuccess)
    return naFail(AG_E_CUDA, "cannot initialise the bin threshold table");
  d.ctxId = id;
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
  // Every argument check comes before the first CUDA call: a rejected call
  // touches no device.
  if (!grid || !d_out || n_atoms < 0 || (n_atoms > 0 && !d_xyzw))
    return naFail(AG_E_INVALID, "null argument or negative atom count");
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || grid->nx > 1025 || grid->ny > 1025 || grid->nz > 1025 ||
      !(grid->spacing > 0))
    return naFail(AG_E_INVALID, "grid outside 1..1025 points per axis or bad spacing");
  if ((int64_t)((grid->nx + agk::kNX - 1) / agk::kNX) * grid->ny * grid->nz > kNaMaxItems)
    return naFail(AG_E_INVALID, "grid too large for ag_emap_noalloc (more than 1048576 work items of 8 points)");
  if ((reinterpret_cast<uintptr_t>(d_xyzw) & 15u) || (reinterpret_cast<uintptr_t>(d_inv_eps) & 15u))
    return naFail(AG_E_INVALID, "d_xyzw and d_inv_eps must be 16-byte aligned");
  if (reinterpret_cast<uintptr_t>(d_out) & 3u) return naFail(AG_E_INVALID, "d_out must be 4-byte aligned");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices)
    return naFail(AG_E_CUDA, "no current CUDA device");
  std::lock_guard<std::mutex> lock(g_mu);
  NaDevice& D = g_dev[dev];
  if (int e = naSetup(D)) return e;
  cudaStream_t st = (cudaStream_t)stream;
  int nitems = 0;
  const int nblocks = naItems(*grid, nitems);
  if (nblocks < 0)
    return naFail(AG_E_INVALID, "grid too large for ag_emap_noalloc (more than 1048576 work items of 8 points)");
  const int64_t np = (int64_t)grid->nx * grid->ny * grid->nz;
  if (n_atoms == 0) {
    if (cudaMemsetAsync(d_out, 0, sizeof(float) * np, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return naFail(AG_E_CUDA, "memset failed");
    return AG_OK;
  }
  // Split atoms across CTAs when the grid alone cannot fill the GPU, within the
  // partial-sum array's and the checksum array's capacity.
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int want = 2 * agk::kEmapCtasPerSm * sms;
  int nsplit = 1;
  if (nblocks < want && n_atoms > 512) nsplit = std::min((want + nblocks - 1) / nblocks, (n_atoms + 255) / 256);
  nsplit = std::min(nsplit, kNaMaxSplit);
  while (nsplit > 1 && (int64_t)nsplit * np > kNaMaxPartial) nsplit--;
  const int chunk = ((n_atoms + nsplit - 1) / nsplit + 255) / 256 * 256;
  nsplit = std::max(1, (n_atoms + chunk - 1) / chunk);

  if (cudaMemcpyAsync(D.items, g_hItems, sizeof(int) * nitems, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(D.blocks, g_hBlocks, sizeof(agk::EmapBlock) * nblocks, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemsetAsync(D.status, 0, sizeof(unsigned), st) != cudaSuccess ||
      cudaMemsetAsync(D.checksum, 0xFF, sizeof(double) * nsplit, st) != cudaSuccess)  // NaN until written
    return naFail(AG_E_CUDA, "cannot stage the work list");
  // The dielectric table's packed tail: the caller's table is read back
  // (32 KB) and packed on the host, as for the ordinary entry points.
  int pkBytes = 0, b16 = 8192, b8 = 8192, vec8 = 0;
  float kScale = 0.f;
  if (d_inv_eps) {
    if (cudaMemcpyAsync(g_hTab, d_inv_eps, sizeof g_hTab, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return naFail(AG_E_CUDA, "cannot read the dielectric table");
    pkBytes = agc::packTableTailInto(g_hTab, 8192, g_hPacked, agk::kEmapPackedBytes, b16, b8, vec8, kScale);
    if (pkBytes > 0 &&
        cudaMemcpyAsync(D.packed, g_hPacked, (size_t)pkBytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
      return naFail(AG_E_CUDA, "cannot stage the packed table");
  }
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
  if (pkBytes > 0) {
    P.packed = D.packed;
    P.packedVecs = pkBytes / 16;
    P.vec8 = vec8;
    P.b16 = b16;
    P.b8 = b8;
    P.r16sq = (float)((b16 + 2.0) * (b16 + 2.0));
    P.r8sq = (float)((b8 + 2.0) * (b8 + 2.0));
    P.kScale = kScale;
  }
  P.thr = D.thr;
  P.rnear2 = (100.f * 14.0f) * (100.f * 14.0f);
  P.delta = 2.0e-3f;
  P.out = d_out;
  P.status = D.status;
  P.checksum = D.checksum;
  P.chunk = chunk;
  P.nsplit = nsplit;
  P.partial = nsplit > 1 ? D.partial : nullptr;
  na_weight_sum_kernel<<<1, 256, 0, st>>>(P.atoms, n_atoms, D.weights);
  if (cudaGetLastError() != cudaSuccess) return naFail(AG_E_CUDA, "weight-sum launch failed");
  if (agk::emap_launch(P, d_inv_eps != nullptr, agk::kEmapKahan, nblocks * nsplit, st) != cudaSuccess)
    return naFail(AG_E_CUDA, "e-map launch failed");
  unsigned status = 0;
  if (cudaMemcpyAsync(&status, D.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(g_hChecksum, D.checksum, sizeof(double) * nsplit, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(g_hWeights, D.weights, sizeof g_hWeights, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return naFail(AG_E_CUDA, "e-map kernel failed");
  if (status) return naFail(AG_E_DEVICE, "the e-map kernel reported an error status (bounded wait expired)");
  double s = 0.0;
  for (int k = 0; k < nsplit; k++) s += g_hChecksum[k];
  if (!(std::fabs(s - g_hWeights[0]) <= 1e-9 * g_hWeights[1] + 1e-12))
    return naFail(AG_E_DEVICE, "net-charge checksum mismatch: the e-map kernel did not consume every atom once");
  return AG_OK;
}
