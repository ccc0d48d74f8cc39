// Waveform features on the GPU: the reference tutorial's envelope transform
// (notebooks/3_beampower.ipynb:74-103, `envelope`): the modulus of the
// analytic signal (scipy.signal.hilbert), centred on its median and divided
// by its median absolute deviation (1 when that is 0), clipped above at 1e5.
//
// Per row of samples: a real-to-complex FFT (cuFFT), the Hilbert weights on
// the spectrum (1 at DC and, for even lengths, Nyquist; 2 on the positive
// frequencies; 0 on the negative ones) written as a full-length spectrum, an
// inverse complex FFT, and the modulus scaled by 1/N.  The median and the
// median absolute deviation are exact order statistics of that envelope
// (the radix select shared with the detection code), and the normalisation
// uses NumPy's float32 subtract and divide.
#define BP_TEMPLATE_KERNELS_ONLY
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

#include <cufft.h>

#include "bp_stats.cuh"

namespace {

const char* cufft_name(cufftResult r) {
  switch (r) {
    case CUFFT_SUCCESS: return "success";
    case CUFFT_INVALID_PLAN: return "invalid plan";
    case CUFFT_ALLOC_FAILED: return "allocation failed";
    case CUFFT_INVALID_VALUE: return "invalid value";
    case CUFFT_INTERNAL_ERROR: return "internal error";
    case CUFFT_EXEC_FAILED: return "exec failed";
    case CUFFT_SETUP_FAILED: return "setup failed";
    case CUFFT_INVALID_SIZE: return "invalid size";
    default: return "error";
  }
}

#define BP_CUFFT(call)                                                              \
  do {                                                                              \
    cufftResult r_ = (call);                                                        \
    if (r_ != CUFFT_SUCCESS)                                                        \
      return fail(r_ == CUFFT_ALLOC_FAILED ? BP_ERR_OUT_OF_MEMORY : BP_ERR_CUDA,     \
                  "%s: cuFFT %s", #call, cufft_name(r_));                           \
  } while (0)

// Plans are costly to make: kept per (device, length, batch, kind) for the
// life of the process.  A plan holds one stream at a time, so setting its
// stream and enqueueing its transform happen under the cache's lock.  The
// lock orders the enqueues only: a plan's work area is shared by every stream
// that uses it, so transforms of one shape on different streams must not
// overlap on the GPU (stated in the header; the library's own callers use
// one stream per call).
struct PlanCache {
  std::mutex mu;
  std::map<std::tuple<int, int, int, int>, cufftHandle> plans;
};
PlanCache g_plans;

// Caller holds g_plans.mu.
int get_plan(int n, int batch, cufftType type, cufftHandle* out) {
  int dev = 0;
  BP_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, n, batch, (int)type);
  auto it = g_plans.plans.find(key);
  if (it != g_plans.plans.end()) {
    *out = it->second;
    return BP_OK;
  }
  cufftHandle h;
  BP_CUFFT(cufftCreate(&h));
  size_t work = 0;
  int len = n;
  const int in_dist = n, out_dist = type == CUFFT_R2C ? n / 2 + 1 : n;
  cufftResult r = cufftMakePlanMany(h, 1, &len, nullptr, 1, in_dist, nullptr, 1, out_dist, type,
                                    batch, &work);
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(h);
    return fail(r == CUFFT_ALLOC_FAILED ? BP_ERR_OUT_OF_MEMORY : BP_ERR_CUDA,
                "cufftMakePlanMany(n=%d, batch=%d): %s", n, batch, cufft_name(r));
  }
  g_plans.plans.emplace(key, h);
  *out = h;
  return BP_OK;
}

int fft_forward_r2c(int n, int batch, float* in, cufftComplex* out, cudaStream_t st) {
  std::lock_guard<std::mutex> lock(g_plans.mu);
  cufftHandle h;
  BP_TRY(get_plan(n, batch, CUFFT_R2C, &h));
  BP_CUFFT(cufftSetStream(h, st));
  BP_CUFFT(cufftExecR2C(h, in, out));
  return BP_OK;
}

int fft_inverse_c2c(int n, int batch, cufftComplex* data, cudaStream_t st) {
  std::lock_guard<std::mutex> lock(g_plans.mu);
  cufftHandle h;
  BP_TRY(get_plan(n, batch, CUFFT_C2C, &h));
  BP_CUFFT(cufftSetStream(h, st));
  BP_CUFFT(cufftExecC2C(h, data, data, CUFFT_INVERSE));
  return BP_OK;
}

// Full-length analytic spectrum from the half spectrum of a real row
// (grid: x over the row's bins, y over rows).
__global__ void hilbert_weights_kernel(const cufftComplex* __restrict__ half, int n,
                                       cufftComplex* __restrict__ full) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const size_t r = blockIdx.y;
  const int nh = n / 2 + 1;
  cufftComplex z = make_cuFloatComplex(0.0f, 0.0f);
  if (k == 0 || (n % 2 == 0 && k == n / 2)) {
    z = half[r * nh + k];
  } else if (k < (n + 1) / 2) {
    const cufftComplex x = half[r * nh + k];
    z = make_cuFloatComplex(2.0f * x.x, 2.0f * x.y);
  }
  full[r * n + k] = z;
}

// Envelope = |inverse transform| / n.
__global__ void modulus_kernel(const cufftComplex* __restrict__ z, long long count, float inv_n,
                               float* __restrict__ env) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const cufftComplex v = z[i];
  env[i] = hypotf(v.x * inv_n, v.y * inv_n);
}

// NumPy's minimum against the clip value: NaN stays NaN.
__device__ __forceinline__ float clip_above(float x, float hi) {
  return (isnan(x) || x <= hi) ? x : hi;
}

// (env - median) / (mad, or 1 when it is 0), clipped above (grid: x over
// the row's samples, y over rows).
__global__ void normalise_kernel(const float* __restrict__ env, int n,
                                 const float* __restrict__ med, const float* __restrict__ mad,
                                 float clip_max, long long out_pitch, float* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const size_t r = blockIdx.y;
  const float m = mad[r];
  const float scale = m == 0.0f ? 1.0f : m;
  out[r * out_pitch + k] = clip_above(__fdiv_rn(__fsub_rn(env[r * n + k], med[r]), scale),
                                      clip_max);
}

// Rows per pass so that the two complex buffers stay within a few GB.
int rows_per_pass(size_t n, size_t rows) {
  const size_t per_row = n * sizeof(cufftComplex) * 2 + n * sizeof(float);
  const size_t budget = size_t(6) << 30;
  size_t r = std::max<size_t>(1, budget / std::max<size_t>(per_row, 1));
  return (int)std::min<size_t>(std::min<size_t>(r, rows), 65535);
}

int envelope_rows(const float* x, size_t rows, size_t n, size_t in_pitch, float clip_max,
                  float* out, size_t out_pitch, cudaStream_t st) {
  const int N = (int)n;
  if (N == 1) {  // the analytic signal of one sample is itself: feature 0
    BP_CUDA(cudaMemset2DAsync(out, out_pitch * sizeof(float), 0, sizeof(float), rows, st));
    return BP_OK;
  }
  const int chunk = rows_per_pass(n, rows);
  Scratch sc(st);
  float *re = nullptr, *env = nullptr, *med = nullptr, *mad = nullptr;
  cufftComplex *half = nullptr, *full = nullptr;
  BP_TRY(sc.get(&re, (size_t)chunk * n));
  BP_TRY(sc.get(&half, (size_t)chunk * (n / 2 + 1)));
  BP_TRY(sc.get(&full, (size_t)chunk * n));
  BP_TRY(sc.get(&env, (size_t)chunk * n));
  BP_TRY(sc.get(&med, chunk));
  BP_TRY(sc.get(&mad, chunk));
  for (size_t r0 = 0; r0 < rows; r0 += chunk) {
    const int b = (int)std::min<size_t>(chunk, rows - r0);
    BP_CUDA(cudaMemcpy2DAsync(re, n * sizeof(float), x + r0 * in_pitch, in_pitch * sizeof(float),
                              n * sizeof(float), b, cudaMemcpyDeviceToDevice, st));
    BP_TRY(fft_forward_r2c(N, b, re, half, st));
    const long long count = (long long)b * N;
    const dim3 rows_grid((unsigned)((N + 255) / 256), (unsigned)b);
    hilbert_weights_kernel<<<rows_grid, 256, 0, st>>>(half, N, full);
    BP_LAUNCHED("hilbert_weights_kernel");
    BP_TRY(fft_inverse_c2c(N, b, full, st));
    modulus_kernel<<<grid_for(count, 256), 256, 0, st>>>(full, count, 1.0f / (float)N, env);
    BP_LAUNCHED("modulus_kernel");
    BP_TRY(np_median(env, N, N, b, 0, nullptr, med, sc, st));
    BP_TRY(np_median(env, N, N, b, 1, med, mad, sc, st));
    normalise_kernel<<<rows_grid, 256, 0, st>>>(env, N, med, mad, clip_max, (long long)out_pitch,
                                                out + r0 * out_pitch);
    BP_LAUNCHED("normalise_kernel");
  }
  return BP_OK;
}

}  // namespace

extern "C" {

int bp_envelope_dev(const float* d_x, size_t n_rows, size_t n_samples, float clip_max,
                    float* d_out, void* stream) {
  BP_NVTX("bp_envelope_dev");
  if (n_rows == 0 || n_samples == 0) return BP_OK;
  if (!d_x || !d_out) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  if (n_samples > (size_t)INT_MAX / 2)
    return fail(BP_ERR_UNSUPPORTED, "rows longer than 2^30 samples");
  return envelope_rows(d_x, n_rows, n_samples, n_samples, clip_max, d_out, n_samples,
                       reinterpret_cast<cudaStream_t>(stream));
}

}  // extern "C"

extern "C" {

int bp_prestack_envelope_dev(const float* d_waveforms, const float* d_weights_phases,
                             size_t n_samples, size_t n_stations, size_t n_channels,
                             size_t n_phases, float clip_max, int storage, size_t lpad,
                             size_t pitch, void* d_traces, float* d_scales, void* stream) {
  BP_NVTX("bp_prestack_envelope_dev");
  if (n_samples == 0 || n_stations == 0 || n_channels == 0) return BP_OK;
  if (!d_waveforms || !d_weights_phases || !d_traces)
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  if (n_samples > (size_t)INT_MAX / 2)
    return fail(BP_ERR_UNSUPPORTED, "rows longer than 2^30 samples");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t rows = n_stations * n_channels;
  float* features = nullptr;
  {
    Scratch sc(st);
    BP_TRY(sc.get(&features, rows * n_samples));
    BP_TRY(envelope_rows(d_waveforms, rows, n_samples, n_samples, clip_max, features, n_samples,
                         st));
    BP_TRY(bp_prestack_dev(features, d_weights_phases, n_samples, n_stations, n_channels,
                           n_phases, storage, lpad, pitch, d_traces, d_scales, stream));
  }
  return BP_OK;
}

}  // extern "C"
