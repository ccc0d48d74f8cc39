// Travel times in seconds to integer sample delays, on the GPU: the
// reference tutorial's sec_to_samp (notebooks/3_beampower.ipynb:378-393),
// which turns the travel-time grid it reads from travel_times.h5 into the
// int32 time_delays of beamform (:394), and the optional shift that makes
// each source's delays relative to its earliest arrival (:396).
//
// The tutorial multiplies float32 seconds by a Python-float sampling rate,
// so the arithmetic is float32: |t * sr| + epsilon, truncated to an integer,
// with the sign of t restored.  Where that value is NaN, infinite or not
// below 2^31 the tutorial's NumPy cast on x86 yields INT_MIN; so does this.
#define BP_TEMPLATE_KERNELS_ONLY
#include <climits>
#include <cstdint>

#include <cuda_runtime.h>

#include "beampower_b200.h"
#include "bp_host.h"

using namespace bp_host;

namespace {

__device__ __forceinline__ int32_t seconds_to_samples(float v, float sr, float eps) {
  const float a = __fadd_rn(fabsf(__fmul_rn(v, sr)), eps);
  if (!(a < 2147483648.0f)) return INT_MIN;
  const int32_t k = (int32_t)a;  // truncation toward zero (a >= 0)
  return v > 0.0f ? k : (v < 0.0f ? -k : 0);
}

__global__ void seconds_to_samples_kernel(const float* __restrict__ t, long long n, float sr,
                                          float eps, int32_t* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = seconds_to_samples(t[i], sr, eps);
}

// One warp per source: convert, then subtract the source's smallest delay
// (int32 arithmetic wraps, as NumPy's in-place subtract does).  The row is
// read twice; the second read comes from cache.
__global__ void relative_delays_kernel(const float* __restrict__ t, long long n_sources, int per,
                                       float sr, float eps, int32_t* __restrict__ d) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= n_sources) return;
  const float* row = t + gw * per;
  int32_t* out = d + gw * per;
  int32_t m = INT_MAX;
  for (int j = lane; j < per; j += 32) m = min(m, seconds_to_samples(row[j], sr, eps));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  for (int j = lane; j < per; j += 32)
    out[j] = (int32_t)((uint32_t)seconds_to_samples(row[j], sr, eps) - (uint32_t)m);
}

}  // namespace

extern "C" int bp_seconds_to_samples_dev(const float* d_seconds, size_t n_sources,
                                         size_t n_per_source, double sampling_rate,
                                         double epsilon, int relative, int32_t* d_delays,
                                         void* stream) {
  BP_NVTX("bp_seconds_to_samples_dev");
  const size_t n = n_sources * n_per_source;
  if (n == 0) return BP_OK;
  if (!d_seconds || !d_delays) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  if (n_per_source > (size_t)INT_MAX)
    return fail(BP_ERR_UNSUPPORTED, "more than 2^31 - 1 delays per source");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const float sr = (float)sampling_rate, eps = (float)epsilon;
  if (relative) {
    const long long threads = (long long)n_sources * 32;
    relative_delays_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
        d_seconds, (long long)n_sources, (int)n_per_source, sr, eps, d_delays);
    BP_LAUNCHED("relative_delays_kernel");
    return BP_OK;
  }
  const long long blocks = std::min<long long>(((long long)n + 255) / 256, 148LL * 16);
  seconds_to_samples_kernel<<<(unsigned)blocks, 256, 0, st>>>(d_seconds, (long long)n, sr, eps,
                                                              d_delays);
  BP_LAUNCHED("seconds_to_samples_kernel");
  return BP_OK;
}
