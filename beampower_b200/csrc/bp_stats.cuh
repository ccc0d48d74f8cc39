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
  explicit Scratch(cudaStream_t s) : st(s) {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) retain_pool(dev);
  }
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

// Radix digits, most significant first.  Wide digits (12 + 10 + 10 bits)
// spread the first pass over many bins -- the values of one row share few
// exponents, and 8-bit first digits put almost all of them in a handful of
// bins whose shared atomics then serialise -- and need one pass fewer; they
// are used while the per-segment histograms (4096 bins) stay small in total.
struct Digit {
  int shift, width;
};
constexpr Digit kWideDigits[3] = {{20, 12}, {10, 10}, {0, 10}};
constexpr Digit kByteDigits[4] = {{24, 8}, {16, 8}, {8, 8}, {0, 8}};
constexpr int kWideBins = 4096;

// Histogram of the current digit of the values whose higher bits match each
// statistic's prefix (dynamic shared memory: 2 x bins counters).  mode 1
// selects among |x - centre[w]| (float32).
__global__ void __launch_bounds__(256)
select_hist_kernel(const float* __restrict__ x, long long seg_stride, int len, int mode,
                   const float* __restrict__ centre, int n_seg, Digit dg, int first,
                   int hist_stride, SelState* __restrict__ st, unsigned* __restrict__ hist) {
  extern __shared__ unsigned h[];  // [2][bins]
  __shared__ unsigned nan_count;
  const int bins = 1 << dg.width;
  const int top = dg.shift + dg.width;
  const uint32_t mask = top >= 32 ? 0u : (0xFFFFFFFFu << top);
  for (int w = blockIdx.y; w < n_seg; w += gridDim.y) {
    const int q = st[w].q;
    for (int b = threadIdx.x; b < bins * q; b += blockDim.x) h[b] = 0;
    if (threadIdx.x == 0) nan_count = 0;
    __syncthreads();
    const uint32_t p0 = st[w].prefix[0] & mask, p1 = st[w].prefix[1] & mask;
    // the two middle ranks of an even length usually share their prefix:
    // then one histogram serves both
    const bool shared_prefix = q == 2 && p0 == p1;
    const bool second = q == 2 && !shared_prefix;
    const float c = mode ? centre[w] : 0.0f;
    const float* base = x + (size_t)w * seg_stride;
    // eight independent loads per thread before the atomics (the atomics
    // would otherwise keep one load in flight per thread)
    constexpr int U = 8;
    const long long step = (long long)gridDim.x * blockDim.x * U;
    for (long long i0 = (long long)blockIdx.x * blockDim.x * U + threadIdx.x; i0 < len;
         i0 += step) {
      float v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const long long i = i0 + (long long)u * blockDim.x;
        v[u] = i < len ? base[i] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (i0 + (long long)u * blockDim.x >= len) break;
        float y = v[u];
        if (mode) y = fabsf(__fsub_rn(y, c));
        if (first && isnan(y)) atomicAdd(&nan_count, 1u);
        const uint32_t key = order_key(y);
        const uint32_t bin = (key >> dg.shift) & (uint32_t)(bins - 1);
        if ((key & mask) == p0) atomicAdd(&h[bin], 1u);
        if (second && (key & mask) == p1) atomicAdd(&h[bins + bin], 1u);
      }
    }
    __syncthreads();
    unsigned* g = hist + (size_t)w * 2 * hist_stride;
    for (int b = threadIdx.x; b < bins * q; b += blockDim.x) {
      const int qi = b / bins, bin = b % bins;
      const unsigned v = (shared_prefix && qi == 1) ? h[bin] : h[b];
      if (v) atomicAdd(&g[(size_t)qi * hist_stride + bin], v);
    }
    if (threadIdx.x == 0 && nan_count) atomicAdd(&st[w].nan, nan_count);
    __syncthreads();
  }
}

// One 256-thread block per (segment, statistic): thread t owns bins
// [t * per, (t + 1) * per); a block-wide exclusive scan of the per-thread
// totals locates the bin that holds the wanted rank, which becomes the next
// digit of the prefix.  The histogram is cleared for the next pass.
__global__ void __launch_bounds__(256)
select_pick_kernel(SelState* __restrict__ st, unsigned* __restrict__ hist, int n_seg, Digit dg,
                   int hist_stride) {
  __shared__ unsigned warp_tot[8];
  const int w = blockIdx.x >> 1, qi = blockIdx.x & 1;
  if (w >= n_seg || qi >= st[w].q) return;  // block-uniform
  const int bins = 1 << dg.width;
  const int per = bins / 256;  // 16 (wide digits) or 1
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  unsigned* h = hist + (size_t)w * 2 * hist_stride + (size_t)qi * hist_stride + (size_t)t * per;
  unsigned c[16];
  unsigned tot = 0;
  for (int j = 0; j < per; ++j) {
    c[j] = h[j];
    tot += c[j];
  }
  unsigned incl = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned v = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  unsigned before = 0;
  for (int k = 0; k < wid; ++k) before += warp_tot[k];
  const unsigned excl = before + incl - tot;
  const uint32_t r = st[w].rank[qi];
  __syncthreads();  // every thread has read rank before it changes
  if (r >= excl && r < excl + tot) {
    unsigned acc = excl;
    for (int j = 0; j < per; ++j) {
      if (r < acc + c[j]) {
        st[w].prefix[qi] |= (uint32_t)(t * per + j) << dg.shift;
        st[w].rank[qi] = r - acc;
        break;
      }
      acc += c[j];
    }
  }
  for (int j = 0; j < per; ++j) h[j] = 0;
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
  const bool wide = (long long)n_seg * 2 * kWideBins <= (1LL << 24);  // <= 64 MB of counters
  const int n_pass = wide ? 3 : 4;
  const Digit* digits = wide ? kWideDigits : kByteDigits;
  const int hist_stride = wide ? kWideBins : 256;
  SelState* state = nullptr;
  unsigned* hist = nullptr;
  BP_TRY(sc.get(&state, n_seg));
  BP_TRY(sc.get(&hist, (size_t)n_seg * 2 * hist_stride));
  BP_CUDA(cudaMemsetAsync(hist, 0, (size_t)n_seg * 2 * hist_stride * sizeof(unsigned), st));
  select_init_kernel<<<grid_for(n_seg, 256), 256, 0, st>>>(state, n_seg, len);
  BP_LAUNCHED("select_init_kernel");
  if (len > 0) {
    const unsigned gx = grid_for(len, 256 * 64, 1024);
    dim3 g(gx, (unsigned)std::min(n_seg, 65535));
    const size_t smem = 2 * (size_t)hist_stride * sizeof(unsigned);
    for (int pass = 0; pass < n_pass; ++pass) {
      select_hist_kernel<<<g, 256, smem, st>>>(x, seg_stride, len, mode, centre, n_seg,
                                               digits[pass], pass == 0 ? 1 : 0, hist_stride,
                                               state, hist);
      BP_LAUNCHED("select_hist_kernel");
      select_pick_kernel<<<(unsigned)(2 * n_seg), 256, 0, st>>>(state, hist, n_seg,
                                                                 digits[pass], hist_stride);
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
