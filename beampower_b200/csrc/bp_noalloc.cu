// Allocation-free variant of the direct max/argmax beamforming path.
//
// Who needs it: programs that are not allowed to allocate device memory
// while they run -- for example a monitoring service that reserves its GPU
// memory once at start-up and hands every later buffer out of its own pool,
// or a host application whose allocator owns the whole device, so that a
// cudaMalloc from inside a library would fail or would synchronise the device
// in the middle of a real-time stream.  They pass every input and output
// buffer themselves; this entry point takes its working memory (the per-sample
// max keys and the per-source delay range) from a fixed array compiled into
// the library instead of allocating it.
//
// The array below is a file-scope __device__ object of kScratchBytes (8 MiB):
// every GPU that loads the library holds it until the process exits.  In host
// code its name is only a host-side stand-in, never a device address, so its
// device address is looked up once per device with cudaGetSymbolAddress (with
// that device current) and passed to the kernels.  That set-up happens inside
// the first call made on each device; make that first call before any stream
// capture begins.  All calls share the one array and it keeps the last call's
// contents: each call clears the keys it uses before the kernels run, and two
// calls that overlap on the GPU (different streams, or different host threads
// on one device) race on it -- serialise them.
#include <climits>
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "beampower_b200.h"
#include "bp_common.cuh"
// error recording, launch counting and NVTX ranges shared with the other
// entry points (template kernels only: the library's other kernels are
// defined in bp_capi.cu)
#define BP_TEMPLATE_KERNELS_ONLY
#include "bp_host.h"

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;
constexpr size_t kKeyBytes = size_t(4) << 20;  // first half: one uint64 key per sample
constexpr size_t kMaxSamples = kKeyBytes / sizeof(unsigned long long);         // 524,288
constexpr size_t kMaxSources = (kScratchBytes - kKeyBytes) / (2 * sizeof(int32_t));  // 524,288

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Records the reason for bp_last_error() and returns the status code.
inline int noalloc_fail(int code, const char* reason) {
  return bp_host::fail(code, "bp_beamform_max_noalloc: %s", reason);
}

// Device address of g_scratch on the current device (set up once per device).
int scratch_on_current_device(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(BP_ERR_CUDA, "no usable current CUDA device");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
      return noalloc_fail(BP_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return BP_OK;
}

// Per-source (min, max) delay over weighted stations (reference rule,
// beampower/src/beamform.c:10-47) into the scratch array.
__global__ void noalloc_minmax_kernel(const int32_t* __restrict__ delays,
                                      const float* __restrict__ weights, int N, int S, int P,
                                      int32_t* __restrict__ minmax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int mn = INT_MAX, mx = INT_MIN;
  for (int s = 0; s < S; ++s) {
    if (weights[(size_t)i * S + s] == 0.0f) continue;
    for (int p = 0; p < P; ++p) {
      const int v = delays[((size_t)i * S + s) * P + p];
      mn = min(mn, v);
      mx = max(mx, v);
    }
  }
  minmax[2 * i] = mn;
  minmax[2 * i + 1] = mx;
}

// One thread per sample, a group of sources per block, terms in reference
// order (stations, then phases; rounded multiply then rounded add); packed
// (beam, source) keys max-reduced into the scratch array.
__global__ void __launch_bounds__(256)
noalloc_direct_max_kernel(const float* __restrict__ traces, long long pitch, int lpad, int T,
                          const int32_t* __restrict__ delays, const float* __restrict__ weights,
                          const int32_t* __restrict__ minmax, int N, int S, int P, int flexible,
                          int src_per_block, unsigned long long* __restrict__ keys) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * src_per_block;
  const int i1 = min(i0 + src_per_block, N);
  unsigned long long best = 0ull;
  for (int i = i0; i < i1; ++i) {
    const int mn = minmax[2 * i], mx = minmax[2 * i + 1];
    const bool valid =
        t < T && (flexible || (mn <= mx && t + mn >= 0 && t + (long long)mx < T));
    if (!valid) continue;
    float acc = 0.0f;
    for (int s = 0; s < S; ++s) {
      const float w = __ldg(weights + (size_t)i * S + s);
      if (w == 0.0f) continue;
      for (int p = 0; p < P; ++p) {
        const long long tt = t + __ldg(delays + ((size_t)i * S + s) * P + p);
        if (tt < 0 || tt >= T) continue;
        const float u = __ldg(traces + (size_t)(s * P + p) * pitch + lpad + tt);
        acc = __fadd_rn(acc, __fmul_rn(w, u));
      }
    }
    const unsigned long long key = bp::make_key(acc, i);
    best = key > best ? key : best;
  }
  if (best != 0ull) bp::red_max_u64(&keys[t], best);
}

__global__ void noalloc_decode_kernel(const unsigned long long* __restrict__ keys, int T,
                                      float* __restrict__ beam_max, int32_t* __restrict__ argmax) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const unsigned long long k = keys[t];
  if (k != 0ull) {
    beam_max[t] = bp::key_value(k);
    argmax[t] = bp::key_source(k);
  } else {
    argmax[t] = 0;
  }
}

}  // namespace

extern "C" BP_API int bp_beamform_max_noalloc(const float* d_traces, size_t n_samples, size_t lpad,
                                              size_t pitch, const int32_t* d_time_delays,
                                              const float* d_weights_sources, size_t n_sources,
                                              size_t n_stations, size_t n_phases,
                                              int out_of_bounds, float* d_beam_max,
                                              int32_t* d_argmax, void* stream) {
  BP_NVTX("bp_beamform_max_noalloc");
  bp_host::g_last_error.clear();
  if (n_samples > kMaxSamples)
    return noalloc_fail(BP_ERR_SCRATCH_LIMIT,
                        "n_samples exceeds the fixed scratch limit of 524288 samples");
  if (n_sources > kMaxSources)
    return noalloc_fail(BP_ERR_SCRATCH_LIMIT,
                        "n_sources exceeds the fixed scratch limit of 524288 sources");
  if (n_stations == 0 || n_phases == 0 || n_stations > 65535 || n_stations * n_phases > 65535)
    return noalloc_fail(BP_ERR_INVALID_ARGUMENT, "n_stations / n_phases out of range");
  if (out_of_bounds != 0 && out_of_bounds != 1)
    return noalloc_fail(BP_ERR_INVALID_ARGUMENT, "out_of_bounds must be 0 or 1");
  if (pitch < lpad + n_samples)
    return noalloc_fail(BP_ERR_INVALID_ARGUMENT, "pitch < lpad + n_samples");
  if (n_samples == 0) return BP_OK;
  if (!d_traces || !d_beam_max || !d_argmax || (n_sources > 0 && (!d_time_delays ||
                                                                   !d_weights_sources)))
    return noalloc_fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  void* base = nullptr;
  if (int rc = scratch_on_current_device(&base)) return rc;
  auto* keys = static_cast<unsigned long long*>(base);
  auto* minmax = reinterpret_cast<int32_t*>(static_cast<unsigned char*>(base) + kKeyBytes);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int T = (int)n_samples, N = (int)n_sources, S = (int)n_stations, P = (int)n_phases;

  // the previous call's keys are still in the array: clear this call's range
  BP_CUDA(cudaMemsetAsync(keys, 0, n_samples * sizeof(unsigned long long), st));
  if (N > 0) {
    noalloc_minmax_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(
        d_time_delays, d_weights_sources, N, S, P, minmax);
    BP_LAUNCHED("noalloc_minmax_kernel");
    int src_per_block = 64;
    unsigned gy = (unsigned)((N + src_per_block - 1) / src_per_block);
    dim3 grid((unsigned)((T + 255) / 256), gy);
    noalloc_direct_max_kernel<<<grid, 256, 0, st>>>(d_traces, (long long)pitch, (int)lpad, T,
                                                     d_time_delays, d_weights_sources, minmax, N,
                                                     S, P, out_of_bounds, src_per_block, keys);
    BP_LAUNCHED("noalloc_direct_max_kernel");
  }
  noalloc_decode_kernel<<<(unsigned)((T + 255) / 256), 256, 0, st>>>(keys, T, d_beam_max,
                                                                     d_argmax);
  BP_LAUNCHED("noalloc_decode_kernel");
  return BP_OK;
}
