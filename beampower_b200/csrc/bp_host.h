// Host-side helpers shared by the library's translation units: error
// recording, launch counting, device attributes, and the staged kernel's
// shape configurations with their launch dispatch.  The dispatch templates
// are instantiated in bp_staged_c*.cu, one file per (config, reduce) pair, so
// that the many kernel variants compile in parallel.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <limits>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "beampower_b200.h"
#include "bp_kernels.cuh"

namespace bp_host {

// Records a printf-style message for bp_last_error() and returns code.
int fail(int code, const char* fmt, ...);
// Maps a CUDA error to BP_ERR_OUT_OF_MEMORY / BP_ERR_CUDA with its text.
int cuda_fail(cudaError_t e, const char* what);
// Kernels launched by the library (bp_launch_count()).
extern std::atomic<uint64_t> g_launches;

// A named range over a public entry point, for timeline profilers (NVTX v3:
// header only; it costs a check when no tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

int device_sm_count(int dev);
int device_smem_optin(int dev);
// Raises the release threshold of the device's default memory pool once, so
// cudaMallocAsync scratch stays mapped between calls.
void retain_pool(int dev);

constexpr long long kMaxInt = std::numeric_limits<int>::max();

// ---- staged-kernel configurations --------------------------------------------
// All use 64-source tiles (the table's tile size).  Config 0: 8 consumer warps
// x 8 sources per thread, 8 samples per lane (256-sample time tiles), 2 blocks
// per SM.  Config 1: 16 consumer warps x 4 sources, 16 samples per lane
// (512-sample time tiles), 1 block per SM: twice the terms per metadata load.
// (A third shape, 16 warps x 4 sources x 8 samples at 2 blocks per SM, was
// measured slower for every storage type: capped at 56 registers it spills.)
#ifndef BP_NSTAGE
#define BP_NSTAGE 4
#endif
template <int ID> struct KCfg;
template <> struct KCfg<0> {
  static constexpr int KS = 8, MT = 8, WS = 8, NSTAGE = BP_NSTAGE, MINB = 2;
};
template <> struct KCfg<1> {
  static constexpr int KS = 4, MT = 16, WS = 16, NSTAGE = BP_NSTAGE, MINB = 1;
};
constexpr int kNumConfigs = 2;
constexpr int kTileSources = 64;
static_assert(KCfg<0>::KS * KCfg<0>::WS == kTileSources, "tile size");
static_assert(KCfg<1>::KS * KCfg<1>::WS == kTileSources, "tile size");


// Launches the staged kernel of config CFG (plain grid of `blocks` blocks, or
// the persistent batch kernel when `batch`), choosing the template variant by
// phase count, storage type and the checked (non-finite weight) rule.
template <int CFG, bool MAXRED>
int launch_window_c(int P, bool checked, int storage, const bp::LaunchArgs& a, bool batch,
                    long long blocks, int dev, cudaStream_t st);

extern template int launch_window_c<0, true>(int, bool, int, const bp::LaunchArgs&, bool,
                                             long long, int, cudaStream_t);
extern template int launch_window_c<0, false>(int, bool, int, const bp::LaunchArgs&, bool,
                                              long long, int, cudaStream_t);
extern template int launch_window_c<1, true>(int, bool, int, const bp::LaunchArgs&, bool,
                                             long long, int, cudaStream_t);
extern template int launch_window_c<1, false>(int, bool, int, const bp::LaunchArgs&, bool,
                                              long long, int, cudaStream_t);

}  // namespace bp_host

#define BP_CUDA(call)                                              \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return ::bp_host::cuda_fail(e_, #call); \
  } while (0)

#define BP_NVTX(name) ::bp_host::NvtxRange bp_nvtx_range_(name)

#define BP_LAUNCHED(what)                                                  \
  do {                                                                     \
    ::bp_host::g_launches.fetch_add(1, std::memory_order_relaxed);         \
    cudaError_t e_ = cudaGetLastError();                                   \
    if (e_ != cudaSuccess) return ::bp_host::cuda_fail(e_, "launch " what); \
  } while (0)
