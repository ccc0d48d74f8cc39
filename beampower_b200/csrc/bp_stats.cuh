// Shared device statistics for the detection and feature files: scratch
// memory, NumPy's float32 division of a sum by its count, NumPy's median as
// an exact radix select, and order-preserving flag compaction.  Everything
// is in an unnamed namespace: each including file gets its own copy.
#pragma once

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "beampower_b200.h"
#include "bp_host.h"

namespace {

using namespace bp_host;

constexpr unsigned kFull = 0xFFFFFFFFu;

// ---- stream-ordered scratch, freed at scope exit -----------------------------
struct Scratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit Scratch(cudaStream_t s) : st(s) {}
  ~Scratch() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
  template <class T>
  int get(T** out, size_t count) {
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, std::max<size_t>(count, 1) * sizeof(T), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync (detection scratch)");
    ptrs.push_back(p);
    *out = static_cast<T*>(p);
    return BP_OK;
  }
};

#define BP_TRY(expr)              \
  do {                            \
    if (int rc_ = (expr)) return rc_; \
  } while (0)

template <class T>
int read_back(T* host, const T* dev, cudaStream_t st) {
  BP_CUDA(cudaMemcpyAsync(host, dev, sizeof(T), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  return BP_OK;
}

inline unsigned grid_for(long long n, int threads, long long cap = 0x7FFFFFFFLL) {
  return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, cap));
}

// NumPy divides a float32 sum by its integer count in float64 and stores the
// quotient as float32 (the count is a NumPy integer, which promotes).
__device__ __forceinline__ float np_divide_count(float s, int count) {
  return __double2float_rn(__ddiv_rn((double)s, (double)count));
}

// ---- exact medians by radix select -----------------------------------------
__device__ __forceinline__ uint32_t order_key(float v) {
  const uint32_t u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

struct SelState {
  uint32_t prefix[2];  // decided high bits of the order statistics
  uint32_t rank[2];    // rank still to find below the decided prefix
  uint32_t nan;        // NaN count (NumPy's median is NaN if any)
  int32_t q;           // 1: odd length (one statistic), 2: even (two)
};

__global__ void select_init_kernel(SelState* st, int n_seg, int len) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_seg) return;
  SelState s;
  s.nan = 0;
  s.prefix[0] = s.prefix[1] = 0;
  if (len % 2) {
    s.q = 1;
    s.rank[0] = s.rank[1] = (uint32_t)(len / 2);
  } else {
    s.q = 2;
    s.rank[0] = (uint32_t)(len / 2 - 1);
    s.rank[1] = (uint32_t)(len / 2);
  }
  st[w] = s;
}

// Histogram of the next 8 bits of the values whose higher bits match each
// statistic's prefix.  mode 1 selects among |x - centre[w]| (float32).
__global__ void __launch_bounds__(256)
select_hist_kernel(const float* __restrict__ x, long long seg_stride, int len, int mode,
                   const float* __restrict__ centre, int n_seg, int pass,
                   SelState* __restrict__ st, unsigned* __restrict__ hist) {
  __shared__ unsigned h[2][256];
  __shared__ unsigned nan_count;
  const int shift = 24 - 8 * pass;
  const uint32_t mask = pass == 0 ? 0u : (0xFFFFFFFFu << (32 - 8 * pass));
  for (int w = blockIdx.y; w < n_seg; w += gridDim.y) {
    for (int b = threadIdx.x; b < 512; b += blockDim.x) (&h[0][0])[b] = 0;
    if (threadIdx.x == 0) nan_count = 0;
    __syncthreads();
    const int q = st[w].q;
    const uint32_t p0 = st[w].prefix[0] & mask, p1 = st[w].prefix[1] & mask;
    const float c = mode ? centre[w] : 0.0f;
    const float* base = x + (size_t)w * seg_stride;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len;
         i += (long long)gridDim.x * blockDim.x) {
      float v = base[i];
      if (mode) v = fabsf(__fsub_rn(v, c));
      if (pass == 0 && isnan(v)) atomicAdd(&nan_count, 1u);
      const uint32_t key = order_key(v);
      const uint32_t bin = (key >> shift) & 255u;
      if ((key & mask) == p0) atomicAdd(&h[0][bin], 1u);
      if (q == 2 && (key & mask) == p1) atomicAdd(&h[1][bin], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256 * q; b += blockDim.x) {
      const unsigned v = (&h[0][0])[b];
      if (v) atomicAdd(&hist[(size_t)w * 512 + b], v);
    }
    if (threadIdx.x == 0 && nan_count) atomicAdd(&st[w].nan, nan_count);
    __syncthreads();
  }
}

// One warp per (segment, statistic): the bin that holds the wanted rank
// becomes the next 8 bits of its prefix; the histogram is cleared.
__global__ void select_pick_kernel(SelState* __restrict__ st, unsigned* __restrict__ hist,
                                   int n_seg, int pass) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long w = gw >> 1;
  const int qi = (int)(gw & 1);
  if (w >= n_seg) return;
  unsigned* h = hist + (size_t)w * 512 + qi * 256;
  if (qi < st[w].q) {
    unsigned c[8], tot = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      c[j] = h[lane * 8 + j];
      tot += c[j];
    }
    unsigned incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned v = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += v;
    }
    const unsigned excl = incl - tot;
    const uint32_t r = st[w].rank[qi];
    if (r >= excl && r < incl) {
      unsigned acc = excl;
      for (int j = 0; j < 8; ++j) {
        if (r < acc + c[j]) {
          const int shift = 24 - 8 * pass;
          st[w].prefix[qi] |= (uint32_t)(lane * 8 + j) << shift;
          st[w].rank[qi] = r - acc;
          break;
        }
        acc += c[j];
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 8; ++j) h[lane * 8 + j] = 0;
}

// NumPy's median from the order statistics: NaN if any NaN, else the middle
// value, or the float32 sum of the two middle values divided by 2.
__global__ void select_finish_kernel(const SelState* __restrict__ st, int n_seg, int len,
                                     float* __restrict__ out) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_seg) return;
  const SelState s = st[w];
  float v;
  if (len == 0 || s.nan) {
    v = __uint_as_float(0x7FC00000u);
  } else if (s.q == 1) {
    v = np_divide_count(__fadd_rn(0.0f, key_float(s.prefix[0])), 1);
  } else {
    const float sum = __fadd_rn(key_float(s.prefix[0]), key_float(s.prefix[1]));
    v = np_divide_count(__fadd_rn(0.0f, sum), 2);
  }
  out[w] = v;
}

int np_median(const float* x, long long seg_stride, int len, int n_seg, int mode,
              const float* centre, float* out, Scratch& sc, cudaStream_t st) {
  SelState* state = nullptr;
  unsigned* hist = nullptr;
  BP_TRY(sc.get(&state, n_seg));
  BP_TRY(sc.get(&hist, (size_t)n_seg * 512));
  BP_CUDA(cudaMemsetAsync(hist, 0, (size_t)n_seg * 512 * sizeof(unsigned), st));
  select_init_kernel<<<grid_for(n_seg, 256), 256, 0, st>>>(state, n_seg, len);
  BP_LAUNCHED("select_init_kernel");
  if (len > 0) {
    const unsigned gx = grid_for(len, 256 * 16, 1024);
    dim3 g(gx, (unsigned)std::min(n_seg, 65535));
    for (int pass = 0; pass < 4; ++pass) {
      select_hist_kernel<<<g, 256, 0, st>>>(x, seg_stride, len, mode, centre, n_seg, pass, state,
                                            hist);
      BP_LAUNCHED("select_hist_kernel");
      select_pick_kernel<<<grid_for((long long)n_seg * 64, 256), 256, 0, st>>>(state, hist,
                                                                               n_seg, pass);
      BP_LAUNCHED("select_pick_kernel");
    }
  }
  select_finish_kernel<<<grid_for(n_seg, 256), 256, 0, st>>>(state, n_seg, len, out);
  BP_LAUNCHED("select_finish_kernel");
  return BP_OK;
}

// ---- flag compaction (order preserving) -------------------------------------
// rank = exclusive prefix sum of flags over n + 1 entries (flags[n] == 0), so
// rank[n] is the number of flagged entries.
int scan_flags(const int* flags, int* rank, int n, Scratch& sc, cudaStream_t st) {
  size_t bytes = 0;
  BP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, flags, rank, n + 1, st));
  void* tmp = nullptr;
  BP_TRY(sc.get(reinterpret_cast<char**>(&tmp), bytes));
  BP_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, flags, rank, n + 1, st));
  return BP_OK;
}

}  // namespace
