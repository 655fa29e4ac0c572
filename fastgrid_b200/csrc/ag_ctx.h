// Internal: the context object behind the C ABI and the staging helpers that
// the e-map, affinity, batch and surrogate entry points share.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/fastgrid_b200.h"
#include "ag_kernels.h"

namespace agc {

// Set the thread's last-error text and return `code`.
int fail(int code, const char* fmt, ...);

#define CK(call)                                                                                \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return agc::fail(AG_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = std::max<size_t>(n, 1);
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

const std::vector<double>& binThresholds();
// The same table written into thr[0 .. 8192], without allocating.
void emapBinThresholdsInto(double* thr);
const std::vector<double>& affinityBinThresholds();

struct SurrState;                 // learned far-field surrogate (surrogate_host.cu)
void surrFree(SurrState* s);

}  // namespace agc

struct ag_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;
  // e-map
  agc::DevBuf<double4> atoms;
  agc::DevBuf<float> epsTab;
  agc::DevBuf<double> thr;
  agc::DevBuf<int> items;
  agc::DevBuf<agk::EmapBlock> blocks;
  agc::DevBuf<double> partial;
  agc::DevBuf<float> maps;
  agc::DevBuf<unsigned> status;
  std::vector<int> hItems;
  std::vector<agk::EmapBlock> hBlocks;
  int itemsFor[3] = {0, 0, 0};
  double itemsH = 0;
  int itemsTile = 0;
  int tile[3] = {2, 8, 16};   // e-map CTA tile in work items (x chunks of 8 points, y rows, z planes)
  int warpCompact = 2;        // e-map item order: 0 rows, 1 warp-compact, 2 warp-compact with x-interleaved lane pairs
  int itemsCompact = -1;      // the order hItems was built with
  bool itemsOnDevice = false; // items / blocks hold hItems / hBlocks
  std::vector<double> epsHost;  // the staged 332/eps table (FP64), empty for the constant dielectric
  std::vector<double> atomsHost;  // host copy of the staged atoms (x, y, z, w), read back on demand
  uint64_t atomsVersion = 0;      // bumped whenever new atoms are staged
  uint64_t atomsHostVersion = ~0ull;  // the staging atomsHost holds
  // affinity
  agc::DevBuf<int> info, cellStart, cellAtoms, cellOf, count, fill, dStart, dAtoms, donorMask, closestH;
  agc::DevBuf<int> ctStart, ctAtoms;  // type-major cell list ((cell, type) segments) of the two-point kernel
  int affKernel = 2;                  // affinity kernel: 2 two-point (default), 1 one point per thread
  agc::DevBuf<float> vol, solq, affTab, affTabH, sol, rv32, rv2_32;
  agc::DevBuf<double> rv64, thrA;
  struct Pass {
    int m0, nm, nmPad;
    size_t tabOff, tabHOff;
    unsigned typeModes[agk::kMaxTypes];
    int typeNeedsAngular[agk::kMaxTypes];
    int mapMinMaxSlot[agk::kMaxMapsPass];
  };
  std::vector<Pass> passes;
  int typeHbond[agk::kMaxTypes] = {0};
  // job
  bool haveJob = false, haveAff = false, ddd = true;
  ag_grid grid{};
  int nAtoms = 0, nMaps = 0, nTypes = 0, hydrogen = -1;
  double solparQ = 0;
  std::vector<int> mapHbond, mapIsHB, mapCov;
  std::vector<float> solparProbe, volProbe;
  int emapMode = agk::kEmapKahan;
  float rNear = 11.0f;
  float delta = 2.0e-3f;
  int packedTable = 1;              // AG_TUNE_EMAP_PACKED_TABLE
  agc::DevBuf<uint4> epsPacked;     // 16- and 8-bit copies of the staged table's saturating tail
  int pkVecs = 0, pkVec8 = 0, pkB16 = 8192, pkB8 = 8192;  // pkVecs == 0: no packed table
  float pkScale = 0;
  int ctasPerSm = agk::kEmapCtasPerSm;
  agc::DevBuf<double> checksum;
  int checksumSplits = 0;
  int testIdleWait = 0;             // test hook AG_TUNE_TEST_IDLE_WAIT
  double testChecksumOffset = 0;    // test hook AG_TUNE_TEST_CHECKSUM_OFFSET
  double wSum = 0, wAbsSum = 0, lastChecksum = 0;
  agc::SurrState* surr = nullptr;
  cudaStream_t copyStream = nullptr;  // device-to-host copies that overlap compute (whole-job path)
  cudaEvent_t evAff = nullptr;
  cudaError_t ensureCopyStream() {
    if (copyStream) return cudaSuccess;
    cudaError_t e = cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&evAff, cudaEventDisableTiming);
    return e;
  }
  // Map set with both passes: the e-map on a high-priority stream and the
  // affinity pass on `stream`, concurrently (AG_TUNE_CONCURRENT_PASSES).
  int concurrentPasses = 1;
  cudaStream_t emapStream = nullptr;
  cudaEvent_t evFork = nullptr, evJoin = nullptr;
  static constexpr int kMaxChunks = 8;  // z-slab chunks of the whole-job affinity pass
  cudaEvent_t evChunk[kMaxChunks] = {};
  cudaError_t ensureEmapStream() {
    if (emapStream) return cudaSuccess;
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&emapStream, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&evFork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&evJoin, cudaEventDisableTiming);
    for (int k = 0; k < kMaxChunks && e == cudaSuccess; k++)
      e = cudaEventCreateWithFlags(&evChunk[k], cudaEventDisableTiming);
    return e;
  }
  int64_t npoints() const { return (int64_t)grid.nx * grid.ny * grid.nz; }
};

namespace agc {

int checkGrid(const ag_grid* g);
// E-map work items and CTA boxes of a grid for a CTA tile shape.
void makeItems(const ag_grid& g, const int tile[3], int warpCompact, std::vector<int>& items,
               std::vector<agk::EmapBlock>& blocks);
// Stage the e-map inputs of a job (atoms, dielectric table, CTA boxes).
int stageEmap(ag_ctx* c, const ag_grid* g, int n, const double* xyzw, const double* inv_eps, bool deviceInputs);
// Launch parameters of the direct e-map of the staged job.
int buildEmapParams(ag_ctx* c, float* dOut, bool allowSplit, agk::EmapParams& P);
int runEmap(ag_ctx* c, float* dOut);
// Read back the status word (and the net-charge checksum) after a computation.
int checkStatus(ag_ctx* c);
// The e-map of the staged job by the learned far-field surrogate (surrogate_host.cu).
int runEmapSurrogate(ag_ctx* c, float* dOut);
// Run the surrogate's inference convolutions on tcgen05 (true) or mma.sync.
void surrUseTc(ag_ctx* c, bool on);

}  // namespace agc
