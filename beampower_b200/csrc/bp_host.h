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
#include <string>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "beampower_b200.h"
#include "bp_kernels.cuh"

namespace bp_host {

// Records a printf-style message for bp_last_error() and returns code.
int fail(int code, const char* fmt, ...);
// The calling thread's last error message (cleared at the start of an entry
// point, set by fail()).
extern thread_local std::string g_last_error;
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
// Each covers the table's 64-source tiles with WS consumer warps x KS sources
// per thread (one block per tile, or two blocks of 32 sources when WS x KS is
// 32), MT samples per lane (time tiles of 32 MT samples), SPS stations per
// ring stage, and MINB blocks per SM.
//   0: 8 x 8, MT 8,  SPS 1, 2/SM     1: 16 x 4, MT 16, SPS 1, 1/SM
//   2: 16 x 4, MT 16, SPS 2, 1/SM    3: 8 x 8, MT 8,  SPS 2, 2/SM
//   4: 16 x 2, MT 32, SPS 1, 1/SM    5: 16 x 2, MT 32, SPS 2, 1/SM
//   6: 8 x 8, MT 16, SPS 2, 1/SM     7: 8 x 8, MT 16, SPS 1, 1/SM
//   8: 16 x 2, MT 16, SPS 2, 1/SM (32 sources per block)
// Registers: a sub-partition holds 16K; 17 warps (16 consumers + producer)
// or 2 x 9 warps put 5 warps on one sub-partition and cap a thread at 96
// registers, 9 warps at one block per SM allow 168 (configs 6 and 7: 8 x 16
// accumulators per thread).
// (A shape of 16 warps x 4 sources x 8 samples at 2 blocks per SM was
// measured slower for every storage type: capped at 56 registers it spills.)
#ifndef BP_NSTAGE
#define BP_NSTAGE 4
#endif
template <int WS_, int KS_, int MT_, int SPS_, int MINB_>
struct KShape {
  static constexpr int WS = WS_, KS = KS_, MT = MT_, SPS = SPS_, MINB = MINB_;
  static constexpr int NSTAGE = BP_NSTAGE;
  static constexpr int K = WS * KS;  // sources per block
};
template <int ID> struct KCfg;
template <> struct KCfg<0> : KShape<8, 8, 8, 1, 2> {};
template <> struct KCfg<1> : KShape<16, 4, 16, 1, 1> {};
template <> struct KCfg<2> : KShape<16, 4, 16, 2, 1> {};
template <> struct KCfg<3> : KShape<8, 8, 8, 2, 2> {};
template <> struct KCfg<4> : KShape<16, 2, 32, 1, 1> {};
template <> struct KCfg<5> : KShape<16, 2, 32, 2, 1> {};
template <> struct KCfg<6> : KShape<8, 8, 16, 2, 1> {};
template <> struct KCfg<7> : KShape<8, 8, 16, 1, 1> {};
template <> struct KCfg<8> : KShape<16, 2, 16, 2, 1> {};
constexpr int kNumConfigs = 9;
constexpr int kTileSources = bp::kTableTile;

// Launches the staged kernel of config CFG (plain grid of `blocks` blocks, or
// the persistent batch kernel when `batch`), choosing the template variant by
// phase count, storage type and the checked (non-finite weight) rule.
template <int CFG, bool MAXRED>
int launch_window_c(int P, bool checked, int storage, const bp::LaunchArgs& a, bool batch,
                    long long blocks, int dev, cudaStream_t st);

#define BP_EXTERN_CFG(C)                                                                  \
  extern template int launch_window_c<C, true>(int, bool, int, const bp::LaunchArgs&, bool, \
                                               long long, int, cudaStream_t);             \
  extern template int launch_window_c<C, false>(int, bool, int, const bp::LaunchArgs&,      \
                                                bool, long long, int, cudaStream_t);
BP_EXTERN_CFG(0)
BP_EXTERN_CFG(1)
BP_EXTERN_CFG(2)
BP_EXTERN_CFG(3)
BP_EXTERN_CFG(4)
BP_EXTERN_CFG(5)
BP_EXTERN_CFG(6)
BP_EXTERN_CFG(7)
BP_EXTERN_CFG(8)
#undef BP_EXTERN_CFG

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
