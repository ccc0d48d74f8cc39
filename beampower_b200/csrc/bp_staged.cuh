// Staged-kernel launch dispatch (template bodies).  Included only by the
// bp_staged_c*.cu files, each of which instantiates one (config, reduce) pair.
#pragma once

#include <algorithm>

#define BP_TEMPLATE_KERNELS_ONLY
#include "bp_host.h"

namespace bp_host {

template <int CFG, int P, bool MAXRED, bool CHECKED, int STORAGE>
int launch_window_p(const bp::LaunchArgs& a, bool batch, long long plain_blocks, int dev,
                    cudaStream_t st) {
  using C = KCfg<CFG>;
  using L = bp::WindowSmem<P, C::KS, C::MT, C::WS, C::NSTAGE, C::SPS, MAXRED>;
  const L lay(a.rowcap, a.max_active, bp::ring_row_factor<STORAGE>(), a.red_rows);
  if (lay.total > (size_t)device_smem_optin(dev))
    return fail(BP_ERR_UNSUPPORTED, "staged kernel needs %zu B of shared memory", lay.total);
  // 16-bit storage addresses ring rows with 16-bit byte offsets
  if (STORAGE != BP_STORAGE_F32 && (long long)a.rowcap * 8 >= 65536)
    return fail(BP_ERR_UNSUPPORTED, "16-bit storage: ring rows of %d samples are too long",
                a.rowcap);
  constexpr int threads = bp::WindowCfg<P, C::KS, C::MT, C::WS>::kThreads;
  if (batch) {
    auto kern = bp::beam_batch_kernel<P, C::KS, C::MT, C::WS, C::NSTAGE, C::SPS, C::MINB,
                                      MAXRED, CHECKED, STORAGE>;
    BP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)lay.total));
    int per_sm = 0;
    BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, lay.total));
    const int grid = std::max(1, per_sm) * std::max(1, device_sm_count(dev));
    kern<<<grid, threads, lay.total, st>>>(a);
    BP_LAUNCHED("beam_batch_kernel");
  } else {
    auto kern = bp::beam_window_kernel<P, C::KS, C::MT, C::WS, C::NSTAGE, C::SPS, C::MINB,
                                       MAXRED, CHECKED, STORAGE>;
    BP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)lay.total));
    if (plain_blocks > kMaxInt) return fail(BP_ERR_UNSUPPORTED, "grid too large");
    if (plain_blocks <= 0) return BP_OK;
    kern<<<(unsigned)plain_blocks, threads, lay.total, st>>>(a);
    BP_LAUNCHED("beam_window_kernel");
  }
  return BP_OK;
}

template <int CFG, bool MAXRED, bool CHECKED, int STORAGE>
int launch_window_s(int P, const bp::LaunchArgs& a, bool batch, long long blocks, int dev,
                    cudaStream_t st) {
  switch (P) {
    case 1: return launch_window_p<CFG, 1, MAXRED, CHECKED, STORAGE>(a, batch, blocks, dev, st);
    case 2: return launch_window_p<CFG, 2, MAXRED, CHECKED, STORAGE>(a, batch, blocks, dev, st);
    case 3: return launch_window_p<CFG, 3, MAXRED, CHECKED, STORAGE>(a, batch, blocks, dev, st);
    case 4: return launch_window_p<CFG, 4, MAXRED, CHECKED, STORAGE>(a, batch, blocks, dev, st);
    default: return fail(BP_ERR_UNSUPPORTED, "staged kernel supports 1..4 phases");
  }
}

template <int CFG, bool MAXRED>
int launch_window_c(int P, bool checked, int storage, const bp::LaunchArgs& a, bool batch,
                    long long blocks, int dev, cudaStream_t st) {
  if (storage == BP_STORAGE_F32)
    return checked
               ? launch_window_s<CFG, MAXRED, true, BP_STORAGE_F32>(P, a, batch, blocks, dev, st)
               : launch_window_s<CFG, MAXRED, false, BP_STORAGE_F32>(P, a, batch, blocks, dev, st);
  if (checked)
    return fail(BP_ERR_UNSUPPORTED,
                "non-finite weights in flexible mode need FP32 trace storage");
  if (storage == BP_STORAGE_BF16)
    return launch_window_s<CFG, MAXRED, false, BP_STORAGE_BF16>(P, a, batch, blocks, dev, st);
  if (storage == BP_STORAGE_F16)
    return launch_window_s<CFG, MAXRED, false, BP_STORAGE_F16>(P, a, batch, blocks, dev, st);
  return fail(BP_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
}

}  // namespace bp_host
