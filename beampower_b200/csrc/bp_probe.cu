// Peak microbenchmarks used to state this GPU's rooflines at the clock it is
// running: shared-memory load bandwidth (the binding resource of the staged
// gather-sum) and FP32 FMA throughput.  Each runs ~ms on the given stream.
#include <cuda_runtime.h>

#include "beampower_b200.h"

namespace {

constexpr int kProbeThreads = 512;
constexpr int kSmemWords = 8192;  // 32 KB

// Conflict-free 128-bit shared loads: every warp instruction reads 512
// distinct bytes (4 wavefronts).  The sum is written so nothing is elided.
__global__ void __launch_bounds__(kProbeThreads) smem_probe_kernel(float* out, int iters) {
  __shared__ float4 buf[kSmemWords / 4];
  for (int i = threadIdx.x; i < kSmemWords / 4; i += blockDim.x)
    buf[i] = make_float4(i * 1e-7f, i * 2e-7f, i * 3e-7f, i * 4e-7f);
  __syncthreads();
  float4 a0 = make_float4(0, 0, 0, 0), a1 = a0, a2 = a0, a3 = a0;
  const int lane = threadIdx.x & 31;
  int base = (threadIdx.x >> 5) * 64 + lane;
  constexpr int mask = kSmemWords / 4 - 1;
  for (int it = 0; it < iters; ++it) {
    const float4 v0 = buf[(base) & mask];
    const float4 v1 = buf[(base + 32) & mask];
    const float4 v2 = buf[(base + 64) & mask];
    const float4 v3 = buf[(base + 96) & mask];
    a0.x += v0.x; a0.y += v0.y; a0.z += v0.z; a0.w += v0.w;
    a1.x += v1.x; a1.y += v1.y; a1.z += v1.z; a1.w += v1.w;
    a2.x += v2.x; a2.y += v2.y; a2.z += v2.z; a2.w += v2.w;
    a3.x += v3.x; a3.y += v3.y; a3.z += v3.z; a3.w += v3.w;
    base += 128;
  }
  const float s = a0.x + a0.y + a0.z + a0.w + a1.x + a1.y + a1.z + a1.w + a2.x + a2.y + a2.z +
                  a2.w + a3.x + a3.y + a3.z + a3.w;
  if (s == 12345.678f) out[blockIdx.x] = s;  // practically never true
}

// Independent FMA chains: 16 per thread.
__global__ void __launch_bounds__(kProbeThreads) fma_probe_kernel(float* out, int iters, float x,
                                                                  float y) {
  float a[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) a[j] = threadIdx.x * 1e-3f + j;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int j = 0; j < 16; ++j) a[j] = fmaf(a[j], x, y);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 16; ++j) s += a[j];
  if (s == 12345.678f) out[blockIdx.x] = s;
}

}  // namespace

extern "C" BP_API int bp_measure_peaks(void* stream, double* smem_gbs, double* fp32_tflops) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return BP_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  float* out = nullptr;
  if (cudaMallocAsync(&out, 4 * sms * 4 * sizeof(float), st) != cudaSuccess) return BP_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 4;  // 4 x 512 threads per SM
  const int smem_iters = 4096, fma_iters = 8192;
  float ms = 0.f;
  // warm-up, then timed
  smem_probe_kernel<<<blocks, kProbeThreads, 0, st>>>(out, smem_iters / 8);
  cudaEventRecord(e0, st);
  smem_probe_kernel<<<blocks, kProbeThreads, 0, st>>>(out, smem_iters);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  const double smem_bytes = (double)blocks * kProbeThreads * smem_iters * 4 * 16;
  if (smem_gbs) *smem_gbs = smem_bytes / (ms * 1e-3) / 1e9;
  fma_probe_kernel<<<blocks, kProbeThreads, 0, st>>>(out, fma_iters / 8, 0.999f, 1e-3f);
  cudaEventRecord(e0, st);
  fma_probe_kernel<<<blocks, kProbeThreads, 0, st>>>(out, fma_iters, 0.999f, 1e-3f);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  const double flops = 2.0 * blocks * kProbeThreads * (double)fma_iters * 16;
  if (fp32_tflops) *fp32_tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(out, st);
  cudaError_t e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? BP_OK : BP_ERR_CUDA;
}
