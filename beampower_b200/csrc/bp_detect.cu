// Detection on the beam series, on the GPU: the reference tutorial's
// time-dependent threshold (notebooks/3_beampower.ipynb:497-579) and its
// peak picking -- scipy.signal.find_peaks(beam_max, distance=...) followed by
// the strict threshold test (notebooks/3_beampower.ipynb:618-626) -- with
// results identical to the NumPy / SciPy code.
//
// Exactness rests on three restatements:
//  * NumPy's float32 sum (inside mean and std) is a pairwise sum whose split
//    points depend on the length only.  The split tree is built on the host;
//    its leaves are summed in parallel and its inner nodes level by level,
//    each with the same rounded operations as NumPy's loop.
//  * NumPy's median is an order statistic (the mean of the two middle values
//    for even lengths); a 4-pass 8-bit radix select on the order-preserving
//    integer image of the floats finds it exactly.
//  * SciPy's distance rule is a greedy pass in decreasing height.  Its result
//    is also the fixed point of rounds in which every undecided peak with no
//    higher undecided peak within the distance is kept, and then every
//    undecided peak within the distance of a kept one is dropped.
#define BP_TEMPLATE_KERNELS_ONLY
#include <cmath>
#include <map>
#include <mutex>
#include <utility>

#include "bp_stats.cuh"

namespace {

// ---- NumPy's float32 pairwise summation --------------------------------------
// numpy/_core/src/umath/loops_utils.h.src, pairwise_sum: a run of n values
// sums as: n < 8, in order; n <= 128, eight strided partial sums r[0..7]
// combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)) and then the n % 8 tail in
// order; otherwise sum([0, n2)) + sum([n2, n)) with n2 = n/2 - (n/2) % 8.
// The reduction then adds that sum to its initial +0.0.
constexpr int kPwLeaf = 128;

__host__ __device__ inline float add_rn(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}

template <class Get>
__host__ __device__ inline float pw_leaf(const Get& get, int len) {
  if (len < 8) {
    float r = 0.0f;
    for (int i = 0; i < len; ++i) r = add_rn(r, get(i));
    return r;
  }
  float r0 = get(0), r1 = get(1), r2 = get(2), r3 = get(3);
  float r4 = get(4), r5 = get(5), r6 = get(6), r7 = get(7);
  int i = 8;
  const int lim = len - len % 8;
  for (; i < lim; i += 8) {
    r0 = add_rn(r0, get(i + 0));
    r1 = add_rn(r1, get(i + 1));
    r2 = add_rn(r2, get(i + 2));
    r3 = add_rn(r3, get(i + 3));
    r4 = add_rn(r4, get(i + 4));
    r5 = add_rn(r5, get(i + 5));
    r6 = add_rn(r6, get(i + 6));
    r7 = add_rn(r7, get(i + 7));
  }
  float res = add_rn(add_rn(add_rn(r0, r1), add_rn(r2, r3)), add_rn(add_rn(r4, r5), add_rn(r6, r7)));
  for (; i < len; ++i) res = add_rn(res, get(i));
  return res;
}

// The split tree of a length: leaves {node, begin, len}, inner nodes
// {node, left, right} grouped by height (children always lower).
struct PwTree {
  std::vector<int4> leaves;
  std::vector<int4> inner;
  std::vector<int> level_end;
  int n_nodes = 0;
  int root = 0;
};

int pw_build(int begin, int len, std::vector<int4>& leaves, std::vector<int4>& inner,
             std::vector<int>& height, int& next_id, int* h_out) {
  if (len <= kPwLeaf) {
    const int id = next_id++;
    leaves.push_back(make_int4(id, begin, len, 0));
    *h_out = 0;
    return id;
  }
  int n2 = len / 2;
  n2 -= n2 % 8;
  int hl = 0, hr = 0;
  const int l = pw_build(begin, n2, leaves, inner, height, next_id, &hl);
  const int r = pw_build(begin + n2, len - n2, leaves, inner, height, next_id, &hr);
  const int id = next_id++;
  inner.push_back(make_int4(id, l, r, 0));
  height.push_back(1 + std::max(hl, hr));
  *h_out = height.back();
  return id;
}

PwTree pw_tree(int n) {
  PwTree t;
  std::vector<int4> raw;
  std::vector<int> h;
  int next = 0, top = 0;
  t.root = pw_build(0, n, t.leaves, raw, h, next, &top);
  t.n_nodes = next;
  std::vector<std::vector<int4>> by_level(top + 1);
  for (size_t i = 0; i < raw.size(); ++i) by_level[h[i]].push_back(raw[i]);
  for (int lv = 1; lv <= top; ++lv) {
    t.inner.insert(t.inner.end(), by_level[lv].begin(), by_level[lv].end());
    t.level_end.push_back((int)t.inner.size());
  }
  return t;
}

// Leaves of every segment w (data x + w * seg_stride): mode 0 sums x, mode 1
// sums (x - centre[w])^2 with NumPy's float32 subtract and multiply.
__global__ void pw_leaves_kernel(const float* __restrict__ x, long long seg_stride, int mode,
                                 const float* __restrict__ centre, const int4* __restrict__ leaves,
                                 int n_leaves, int n_nodes, int n_seg, float* __restrict__ vals) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n_leaves) return;
  const int4 lf = leaves[l];
  for (int w = blockIdx.y; w < n_seg; w += gridDim.y) {
    const float* base = x + (size_t)w * seg_stride + lf.y;
    float s;
    if (mode == 0) {
      s = pw_leaf([&](int i) { return base[i]; }, lf.z);
    } else {
      const float c = centre[w];
      s = pw_leaf(
          [&](int i) {
            const float d = __fsub_rn(base[i], c);
            return __fmul_rn(d, d);
          },
          lf.z);
    }
    vals[(size_t)w * n_nodes + lf.x] = s;
  }
}

// Inner nodes of every segment, one block per segment, level by level; then
// out[w] = (0 + root) / count as NumPy's mean / var store it.
__global__ void pw_inner_kernel(const int4* __restrict__ inner, const int* __restrict__ level_end,
                                int n_levels, int n_nodes, int root, int count, int n_seg,
                                float* __restrict__ vals, float* __restrict__ out) {
  for (int w = blockIdx.x; w < n_seg; w += gridDim.x) {
    float* v = vals + (size_t)w * n_nodes;
    int begin = 0;
    for (int lv = 0; lv < n_levels; ++lv) {
      const int end = level_end[lv];
      for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
        const int4 nd = inner[i];
        v[nd.x] = __fadd_rn(v[nd.y], v[nd.z]);
      }
      begin = end;
      __syncthreads();
    }
    if (threadIdx.x == 0) out[w] = np_divide_count(__fadd_rn(0.0f, v[root]), count);
    __syncthreads();
  }
}

// out[w] = mean (mode 0) or population variance (mode 1, given the means) of
// segments of `len` values starting every seg_stride values.
// Split trees of the lengths seen so far, built and uploaded once per device
// and kept for the life of the process (up to kTreeCache lengths; beyond
// that a tree is uploaded into the call's scratch).  The upload is ordered
// on the call's stream and waited for (a plain cudaMemcpy from pageable
// memory may return before its DMA lands), so a cached tree is complete
// before any stream uses it.
struct DevTree {
  int n_leaves = 0, n_inner = 0, n_levels = 0, n_nodes = 0, root = 0;
  const int4* leaves = nullptr;
  const int4* inner = nullptr;
  const int* levels = nullptr;
};
constexpr size_t kTreeCache = 64;
std::mutex g_tree_mu;
std::map<std::pair<int, int>, DevTree> g_trees;

int upload_tree(const PwTree& t, DevTree* d, void* mem, cudaStream_t st) {
  char* p = static_cast<char*>(mem);
  d->n_leaves = (int)t.leaves.size();
  d->n_inner = (int)t.inner.size();
  d->n_levels = (int)t.level_end.size();
  d->n_nodes = t.n_nodes;
  d->root = t.root;
  d->leaves = reinterpret_cast<const int4*>(p);
  d->inner = reinterpret_cast<const int4*>(p + t.leaves.size() * sizeof(int4));
  d->levels = reinterpret_cast<const int*>(p + (t.leaves.size() + t.inner.size()) *
                                                   sizeof(int4));
  BP_CUDA(cudaMemcpyAsync(p, t.leaves.data(), t.leaves.size() * sizeof(int4),
                          cudaMemcpyHostToDevice, st));
  if (!t.inner.empty()) {
    BP_CUDA(cudaMemcpyAsync(p + t.leaves.size() * sizeof(int4), t.inner.data(),
                            t.inner.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    BP_CUDA(cudaMemcpyAsync(p + (t.leaves.size() + t.inner.size()) * sizeof(int4),
                            t.level_end.data(), t.level_end.size() * sizeof(int),
                            cudaMemcpyHostToDevice, st));
  }
  // the host vectors are freed on return and a cached tree is shared by
  // every stream: wait until the copies have landed
  BP_CUDA(cudaStreamSynchronize(st));
  return BP_OK;
}

size_t tree_bytes(const PwTree& t) {
  return (t.leaves.size() + t.inner.size()) * sizeof(int4) + t.level_end.size() * sizeof(int) +
         16;
}

int get_tree(int len, DevTree* out, Scratch& sc) {
  int dev = 0;
  BP_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_pair(dev, len);
  {
    std::lock_guard<std::mutex> lock(g_tree_mu);
    auto it = g_trees.find(key);
    if (it != g_trees.end()) {
      *out = it->second;
      return BP_OK;
    }
  }
  const PwTree t = pw_tree(len);
  std::lock_guard<std::mutex> lock(g_tree_mu);
  auto it = g_trees.find(key);
  if (it != g_trees.end()) {
    *out = it->second;
    return BP_OK;
  }
  void* mem = nullptr;
  if (g_trees.size() < kTreeCache) {
    BP_CUDA(cudaMalloc(&mem, tree_bytes(t)));
    DevTree d;
    if (int rc = upload_tree(t, &d, mem, sc.st)) {
      cudaFree(mem);
      return rc;
    }
    g_trees.emplace(key, d);
    *out = d;
    return BP_OK;
  }
  char* scratch = nullptr;  // cache full: this call's own copy
  BP_TRY(sc.get(&scratch, tree_bytes(t)));
  return upload_tree(t, out, scratch, sc.st);  // ordered after the allocation
}

int pw_mean(const float* x, long long seg_stride, int len, int n_seg, int mode,
            const float* centre, float* out, Scratch& sc, cudaStream_t st) {
  DevTree t;
  BP_TRY(get_tree(len, &t, sc));
  float* vals = nullptr;
  BP_TRY(sc.get(&vals, (size_t)t.n_nodes * n_seg));
  dim3 g1((t.n_leaves + 127) / 128, (unsigned)std::min(n_seg, 65535));
  pw_leaves_kernel<<<g1, 128, 0, st>>>(x, seg_stride, mode, centre, t.leaves, t.n_leaves,
                                       t.n_nodes, n_seg, vals);
  BP_LAUNCHED("pw_leaves_kernel");
  pw_inner_kernel<<<(unsigned)std::min(n_seg, 65535), n_seg == 1 ? 1024 : 256, 0, st>>>(
      t.inner, t.levels, t.n_levels, t.n_nodes, t.root, len, n_seg, vals, out);
  BP_LAUNCHED("pw_inner_kernel");
  return BP_OK;
}

// ---- threshold kernels ---------------------------------------------------------
__global__ void zero_flags_kernel(const float* __restrict__ x, int n, int* __restrict__ flags) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  flags[i] = (i < n && x[i] == 0.0f) ? 1 : 0;
}

// Non-zero samples, in order, into nz.
__global__ void gather_nonzero_kernel(const float* __restrict__ x, int n,
                                      const int* __restrict__ zero_rank, float* __restrict__ nz) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = x[i];
  if (v != 0.0f) nz[i - zero_rank[i]] = v;
}

// SplitMix64 output function (Steele, Lea & Flood, OOPSLA 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Standard normal draws: Box-Muller on two counter-based uniforms.
__global__ void normal_kernel(unsigned long long seed, int n, float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t a = mix64(seed ^ mix64(2ull * (uint64_t)i));
  const uint64_t b = mix64(seed ^ mix64(2ull * (uint64_t)i + 1ull));
  const float u1 = ((float)(a >> 40) + 0.5f) * 0x1p-24f;  // (0, 1)
  const float u2 = (float)(b >> 40) * 0x1p-24f;           // [0, 1)
  out[i] = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// Zeros replaced by noise * deviation + centre (NumPy float32 multiply, add).
__global__ void fill_zeros_kernel(const float* __restrict__ x, int n,
                                  const int* __restrict__ zero_rank,
                                  const float* __restrict__ noise,
                                  const float* __restrict__ centre0,
                                  const float* __restrict__ dev0, float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = x[i];
  out[i] = v != 0.0f ? v : __fadd_rn(__fmul_rn(noise[zero_rank[i]], *dev0), *centre0);
}

// Default centre / deviation for the rms rule: deviation = sqrt(variance);
// both NaN when there is no non-zero sample (NumPy's mean of nothing).
__global__ void finish_stats_kernel(float* __restrict__ stats, int have) {
  if (threadIdx.x != 0) return;
  if (have) {
    stats[1] = __fsqrt_rn(stats[1]);
  } else {
    stats[0] = stats[1] = __uint_as_float(0x7FC00000u);
  }
}

// np.maximum on float32: NaN propagates, equal values give the second operand.
__device__ __forceinline__ float np_maximum(float a, float b) {
  return (a > b || isnan(a)) ? a : b;
}

// thr[w] = centre + num_dev * deviation (rms: deviation = sqrt(variance)).
__global__ void window_threshold_kernel(const float* __restrict__ centre,
                                        const float* __restrict__ spread, int n_win, int is_var,
                                        float num_dev, float* __restrict__ thr) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_win) return;
  const float dev = is_var ? __fsqrt_rn(spread[w]) : spread[w];
  thr[w] = __fadd_rn(centre[w], __fmul_rn(num_dev, dev));
}

// neighbour = -1: out[i] = max(in[i-1], in[i]) for i >= 1 (in[0] kept);
// neighbour = +1: out[i] = max(in[i], in[i+1]) for i < n-1 (in[n-1] kept).
__global__ void neighbour_max_kernel(const float* __restrict__ in, int n_win, int neighbour,
                                     float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_win) return;
  float v = in[i];
  if (neighbour < 0 && i >= 1) v = np_maximum(in[i - 1], in[i]);
  if (neighbour > 0 && i + 1 < n_win) v = np_maximum(in[i], in[i + 1]);
  out[i] = v;
}

// Per-sample threshold: windows' values at (half + j) / shift for the middle
// samples, the first / last middle value repeated at both ends.
__global__ void spread_threshold_kernel(const float* __restrict__ thr, int n_win, int n,
                                        int window, int half, int shift, float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long n_mid = (long long)n - window;
  long long j = i - half;
  if (j < 0) j = 0;
  if (j > n_mid - 1) j = n_mid - 1;
  long long idx = (half + j) / shift;
  if (idx > n_win - 1) idx = n_win - 1;
  out[i] = thr[idx];
}

// ---- peak kernels ----------------------------------------------------------
// Rising edges x[i-1] < x[i]: a peak at i when x[i+1] < x[i]; a plateau to
// measure when x[i+1] == x[i].
__global__ void local_max_kernel(const float* __restrict__ x, int n, int* __restrict__ flags,
                                 int* __restrict__ plateau, int* __restrict__ n_plateau) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 1 || i >= (long long)n - 1) return;
  const float xi = x[i];
  if (!(x[i - 1] < xi)) return;
  const float nx = x[i + 1];
  if (nx < xi) {
    flags[i] = 1;
  } else if (nx == xi) {
    plateau[atomicAdd(n_plateau, 1)] = (int)i;
  }
}

// One warp per plateau starting at i: its end j is the first index > i with
// x[j] != x[i], capped at n - 1; a peak at (i + j - 1) / 2 when x[j] < x[i].
__global__ void plateau_kernel(const float* __restrict__ x, int n, const int* __restrict__ plateau,
                               const int* __restrict__ n_plateau, int* __restrict__ flags) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= *n_plateau) return;
  const int i = plateau[gw];
  const float xi = x[i];
  for (long long base = (long long)i + 1;; base += 32) {
    const long long j = base + lane;
    const bool stop = j >= (long long)n - 1 || x[j] != xi;
    const unsigned b = __ballot_sync(kFull, stop);
    if (b) {
      long long e = base + __ffs(b) - 1;
      if (e > n - 1) e = n - 1;
      if (lane == 0 && x[e] < xi) flags[(i + e - 1) / 2] = 1;
      return;
    }
  }
}

__global__ void scatter_flagged_kernel(const int* __restrict__ flags, const int* __restrict__ rank,
                                       int n, int* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (flags[i]) out[rank[i]] = (int)i;
}

__global__ void gather_heights_kernel(const float* __restrict__ x, const int* __restrict__ pos,
                                      int m, float* __restrict__ val, int* __restrict__ state,
                                      int* __restrict__ undecided) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  val[j] = x[pos[j]];
  state[j] = 0;
  undecided[j] = j;
}

enum : int { kUndecided = 0, kKept = 1, kDropped = 2 };

// Peak k goes before peak j in SciPy's order (decreasing height; the later
// sample first among equal heights, as a stable ascending sort read backwards).
__device__ __forceinline__ bool before(const float* val, int k, int j) {
  return val[k] > val[j] || (val[k] == val[j] && k > j);
}

// Round step 1, one warp per undecided peak: kept when no undecided peak
// within the distance goes before it.
__global__ void distance_keep_kernel(const int* __restrict__ pos, const float* __restrict__ val,
                                     const int* __restrict__ state, int m, long long dist,
                                     const int* __restrict__ undecided, int n_undecided,
                                     int* __restrict__ kept, int* __restrict__ n_kept) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= n_undecided) return;
  const int j = undecided[gw];
  const long long pj = pos[j];
  bool blocked = false;
  for (long long base = (long long)j - 1; base >= 0; base -= 32) {
    const long long k = base - lane;
    const bool in = k >= 0 && pj - pos[k] < dist;
    const bool blk = in && state[k] == kUndecided && before(val, (int)k, j);
    if (__any_sync(kFull, blk)) {
      blocked = true;
      break;
    }
    if (__any_sync(kFull, !in)) break;
  }
  if (!blocked) {
    for (long long base = (long long)j + 1; base < m; base += 32) {
      const long long k = base + lane;
      const bool in = k < m && pos[k] - pj < dist;
      const bool blk = in && state[k] == kUndecided && before(val, (int)k, j);
      if (__any_sync(kFull, blk)) {
        blocked = true;
        break;
      }
      if (__any_sync(kFull, !in)) break;
    }
  }
  if (!blocked && lane == 0) kept[atomicAdd(n_kept, 1)] = j;
}

// Round step 2, one warp per newly kept peak: mark it kept and drop every
// undecided peak within the distance.
__global__ void distance_drop_kernel(const int* __restrict__ pos, int* __restrict__ state, int m,
                                     long long dist, const int* __restrict__ kept,
                                     const int* __restrict__ n_kept) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= *n_kept) return;
  const int j = kept[gw];
  const long long pj = pos[j];
  if (lane == 0) state[j] = kKept;
  for (long long base = (long long)j - 1; base >= 0; base -= 32) {
    const long long k = base - lane;
    const bool in = k >= 0 && pj - pos[k] < dist;
    if (in && state[k] == kUndecided) state[k] = kDropped;
    if (__any_sync(kFull, !in)) break;
  }
  for (long long base = (long long)j + 1; base < m; base += 32) {
    const long long k = base + lane;
    const bool in = k < m && pos[k] - pj < dist;
    if (in && state[k] == kUndecided) state[k] = kDropped;
    if (__any_sync(kFull, !in)) break;
  }
}

// Round step 3: the still undecided peaks form the next work list.
__global__ void distance_next_kernel(const int* __restrict__ state,
                                     const int* __restrict__ undecided, int n_undecided,
                                     int* __restrict__ next, int* __restrict__ n_next) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_undecided) return;
  const int j = undecided[i];
  if (state[j] == kUndecided) next[atomicAdd(n_next, 1)] = j;
}

__global__ void kept_flags_kernel(const int* __restrict__ state, int m, int* __restrict__ flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > m) return;
  flags[j] = (j < m && state[j] == kKept) ? 1 : 0;
}

__global__ void above_flags_kernel(const float* __restrict__ x, const float* __restrict__ thr,
                                   const int* __restrict__ peaks, int m, int* __restrict__ flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > m) return;
  flags[j] = (j < m && x[peaks[j]] > thr[peaks[j]]) ? 1 : 0;
}

__global__ void scatter_detections_kernel(const int* __restrict__ flags,
                                          const int* __restrict__ rank,
                                          const int* __restrict__ peaks, int m,
                                          const float* __restrict__ x,
                                          const int32_t* __restrict__ argmax,
                                          int32_t* __restrict__ out_peaks,
                                          float* __restrict__ out_heights,
                                          int32_t* __restrict__ out_sources) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m || !flags[j]) return;
  const int r = rank[j], p = peaks[j];
  out_peaks[r] = p;
  if (out_heights) out_heights[r] = x[p];
  if (argmax && out_sources) out_sources[r] = argmax[p];
}

// ---- host drivers -------------------------------------------------------------
// Peaks of x into d_peaks (device, ascending); their number into *m_out.
// ---- height and prominence conditions (SciPy's find_peaks options) ----------
// lo <= v_lo and v_hi <= hi in float64; a NaN scalar border is an open side,
// a per-sample border array (float64, read at the peak) compares as SciPy
// does (NaN fails).
__device__ __forceinline__ bool within(double v_lo, double v_hi, double lo, double hi,
                                       const double* lo_arr, const double* hi_arr, int p) {
  bool ok = true;
  if (lo_arr) ok = ok && (lo_arr[p] <= v_lo);
  else if (!isnan(lo)) ok = ok && (lo <= v_lo);
  if (hi_arr) ok = ok && (v_hi <= hi_arr[p]);
  else if (!isnan(hi)) ok = ok && (v_hi <= hi);
  return ok;
}

// SciPy's threshold condition: the peak's rise over each neighbour (float64),
// the smaller rise against the lower border, the larger against the upper.
// A peak's neighbours exist and are never NaN (both are below the peak).
__global__ void threshold_flags_kernel(const float* __restrict__ x, const int* __restrict__ pos,
                                       int m, double lo, double hi,
                                       const double* __restrict__ lo_arr,
                                       const double* __restrict__ hi_arr,
                                       int* __restrict__ flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > m) return;
  int keep = 0;
  if (j < m) {
    const int p = pos[j];
    const double left = (double)x[p] - (double)x[p - 1];
    const double right = (double)x[p] - (double)x[p + 1];
    keep = within(fmin(left, right), fmax(left, right), lo, hi, lo_arr, hi_arr, p) ? 1 : 0;
  }
  flags[j] = keep;
}

__global__ void height_flags_kernel(const float* __restrict__ x, const int* __restrict__ pos,
                                    int m, double lo, double hi, const double* __restrict__ lo_arr,
                                    const double* __restrict__ hi_arr, int* __restrict__ flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > m) return;
  int keep = 0;
  if (j < m) {
    const double v = (double)x[pos[j]];
    keep = within(v, v, lo, hi, lo_arr, hi_arr, pos[j]) ? 1 : 0;
  }
  flags[j] = keep;
}

// One warp per peak: from the peak, walk outwards while the signal is not
// above it (NaN stops the walk), at most `half` samples when half >= 0; the
// base of each side is its lowest sample (the one nearest the peak among
// equals), the prominence the peak minus the higher base, in float64.
__global__ void prominence_kernel(const float* __restrict__ x, int n, const int* __restrict__ pos,
                                  int m, long long half, double* __restrict__ prom,
                                  int* __restrict__ lbase, int* __restrict__ rbase) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= m) return;
  const int p = pos[gw];
  const float xp = x[p];
  const long long lo_end = half >= 0 ? max(0LL, (long long)p - half) : 0LL;
  const long long hi_end = half >= 0 ? min((long long)n - 1, (long long)p + half)
                                     : (long long)n - 1;
  float side_min[2];
  int side_base[2];
  for (int dir = 0; dir < 2; ++dir) {  // 0: left, 1: right
    float best = xp;
    int best_i = p;
    for (long long base = p;; base += dir ? 32 : -32) {
      const long long i = dir ? base + lane : base - lane;
      const bool inside = dir ? i <= hi_end : i >= lo_end;
      const float v = inside ? x[i] : 0.0f;
      const bool walk = inside && v <= xp;  // false past the window, above the peak, NaN
      const unsigned stop = __ballot_sync(kFull, !walk);
      const int n_walk = stop ? __ffs(stop) - 1 : 32;  // lanes before the first stop
      // lowest value among the walked lanes, nearest the peak among equals
      float cv = lane < n_walk ? v : INFINITY;
      int ci = lane < n_walk ? (int)i : INT_MAX;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(kFull, cv, o);
        const int oi = __shfl_xor_sync(kFull, ci, o);
        const bool nearer = dir ? oi < ci : (oi != INT_MAX && (ci == INT_MAX || oi > ci));
        if (ov < cv || (ov == cv && nearer)) {
          cv = ov;
          ci = oi;
        }
      }
      if (n_walk > 0 && cv < best) {  // a strictly lower sample further out
        best = cv;
        best_i = ci;
      }
      if (stop) break;
    }
    side_min[dir] = best;
    side_base[dir] = best_i;
  }
  if (lane == 0) {
    prom[gw] = (double)xp - (double)fmaxf(side_min[0], side_min[1]);
    lbase[gw] = side_base[0];
    rbase[gw] = side_base[1];
  }
}

__global__ void prominence_flags_kernel(const double* __restrict__ prom,
                                        const int* __restrict__ pos, int m, double lo, double hi,
                                        const double* __restrict__ lo_arr,
                                        const double* __restrict__ hi_arr,
                                        int* __restrict__ flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > m) return;
  flags[j] = (j < m && within(prom[j], prom[j], lo, hi, lo_arr, hi_arr, pos[j])) ? 1 : 0;
}

__global__ void compact_peaks_kernel(const int* __restrict__ flags, const int* __restrict__ rank,
                                     int m, const int* __restrict__ pos,
                                     const double* __restrict__ prom, const int* __restrict__ lb,
                                     const int* __restrict__ rb, int* __restrict__ out_pos,
                                     double* __restrict__ out_prom, int* __restrict__ out_lb,
                                     int* __restrict__ out_rb) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m || !flags[j]) return;
  const int r = rank[j];
  out_pos[r] = pos[j];
  if (out_prom) out_prom[r] = prom[j];
  if (out_lb) out_lb[r] = lb[j];
  if (out_rb) out_rb[r] = rb[j];
}

// ---- host driver of the peak finder -----------------------------------------
struct PeakOut {
  int32_t* peaks;
  double* prominences;  // may be NULL
  int32_t* left_bases;  // may be NULL
  int32_t* right_bases; // may be NULL
};

// Keeps the entries of `pos` (m, device) whose flag is set, in order, into a
// new scratch array; returns their number.
int keep_flagged(int* flags, int m, int** pos, Scratch& sc, cudaStream_t st, int* kept) {
  int* rank = nullptr;
  int* out = nullptr;
  BP_TRY(sc.get(&rank, (size_t)m + 1));
  BP_TRY(scan_flags(flags, rank, m, sc, st));
  BP_TRY(read_back(kept, rank + m, st));
  BP_TRY(sc.get(&out, std::max(*kept, 1)));
  compact_peaks_kernel<<<grid_for(m, 256), 256, 0, st>>>(flags, rank, m, *pos, nullptr, nullptr,
                                                         nullptr, out, nullptr, nullptr,
                                                         nullptr);
  BP_LAUNCHED("compact_peaks_kernel");
  *pos = out;
  return BP_OK;
}

// Peaks of x in SciPy's order of conditions: local maxima (plateaus by their
// midpoint), height, distance, prominence.  Writes `*m_out` entries of `out`.
int find_peaks_impl(const float* x, int n, const bp_peak_options& o, const PeakOut& out,
                    int* m_out, Scratch& sc, cudaStream_t st) {
  *m_out = 0;
  if (n < 3) return BP_OK;
  int *flags = nullptr, *rank = nullptr, *plateau = nullptr, *counters = nullptr;
  BP_TRY(sc.get(&flags, (size_t)n + 1));
  BP_TRY(sc.get(&rank, (size_t)n + 1));
  BP_TRY(sc.get(&plateau, n));
  BP_TRY(sc.get(&counters, 4));
  BP_CUDA(cudaMemsetAsync(flags, 0, ((size_t)n + 1) * sizeof(int), st));
  BP_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(int), st));
  local_max_kernel<<<grid_for(n, 256), 256, 0, st>>>(x, n, flags, plateau, counters);
  BP_LAUNCHED("local_max_kernel");
  int n_plateau = 0;
  BP_TRY(read_back(&n_plateau, counters, st));
  if (n_plateau > 0) {
    plateau_kernel<<<grid_for((long long)n_plateau * 32, 256), 256, 0, st>>>(x, n, plateau,
                                                                             counters, flags);
    BP_LAUNCHED("plateau_kernel");
  }
  BP_TRY(scan_flags(flags, rank, n, sc, st));
  int m = 0;
  BP_TRY(read_back(&m, rank + n, st));
  int* pos = nullptr;
  BP_TRY(sc.get(&pos, std::max(m, 1)));
  scatter_flagged_kernel<<<grid_for(n, 256), 256, 0, st>>>(flags, rank, n, pos);
  BP_LAUNCHED("scatter_flagged_kernel");
  // height
  if (o.use_height && m > 0) {
    height_flags_kernel<<<grid_for((long long)m + 1, 256), 256, 0, st>>>(
        x, pos, m, o.height_min, o.height_max, o.d_height_min, o.d_height_max, flags);
    BP_LAUNCHED("height_flags_kernel");
    BP_TRY(keep_flagged(flags, m, &pos, sc, st, &m));
  }
  // threshold
  if (o.use_threshold && m > 0) {
    threshold_flags_kernel<<<grid_for((long long)m + 1, 256), 256, 0, st>>>(
        x, pos, m, o.threshold_min, o.threshold_max, o.d_threshold_min, o.d_threshold_max,
        flags);
    BP_LAUNCHED("threshold_flags_kernel");
    BP_TRY(keep_flagged(flags, m, &pos, sc, st, &m));
  }
  // greedy distance rule, in rounds
  if (o.distance > 0.0 && m > 1) {
    const double dc = std::ceil(o.distance);
    const long long dist = dc > (double)n ? (long long)n + 1 : (long long)dc;
    float* val = nullptr;
    int *state = nullptr, *und = nullptr, *und2 = nullptr, *kept = nullptr;
    BP_TRY(sc.get(&val, m));
    BP_TRY(sc.get(&state, (size_t)m + 1));
    BP_TRY(sc.get(&und, m));
    BP_TRY(sc.get(&und2, m));
    BP_TRY(sc.get(&kept, m));
    gather_heights_kernel<<<grid_for(m, 256), 256, 0, st>>>(x, pos, m, val, state, und);
    BP_LAUNCHED("gather_heights_kernel");
    int u = m;
    for (int round = 0; u > 0; ++round) {
      if (round > m) return fail(BP_ERR_KERNEL, "distance rule did not converge");
      BP_CUDA(cudaMemsetAsync(counters + 1, 0, 2 * sizeof(int), st));
      const unsigned gw = grid_for((long long)u * 32, 256);
      distance_keep_kernel<<<gw, 256, 0, st>>>(pos, val, state, m, dist, und, u, kept,
                                               counters + 1);
      BP_LAUNCHED("distance_keep_kernel");
      distance_drop_kernel<<<gw, 256, 0, st>>>(pos, state, m, dist, kept, counters + 1);
      BP_LAUNCHED("distance_drop_kernel");
      distance_next_kernel<<<grid_for(u, 256), 256, 0, st>>>(state, und, u, und2, counters + 2);
      BP_LAUNCHED("distance_next_kernel");
      BP_TRY(read_back(&u, counters + 2, st));
      std::swap(und, und2);
    }
    kept_flags_kernel<<<grid_for((long long)m + 1, 256), 256, 0, st>>>(state, m, flags);
    BP_LAUNCHED("kept_flags_kernel");
    BP_TRY(keep_flagged(flags, m, &pos, sc, st, &m));
  }
  // prominence
  if (o.use_prominence && m > 0) {
    double* prom = nullptr;
    int *lb = nullptr, *rb = nullptr;
    BP_TRY(sc.get(&prom, m));
    BP_TRY(sc.get(&lb, m));
    BP_TRY(sc.get(&rb, m));
    const long long half = o.wlen > 1.0 ? (long long)std::ceil(o.wlen) / 2 : -1;
    prominence_kernel<<<grid_for((long long)m * 32, 256), 256, 0, st>>>(x, n, pos, m, half,
                                                                        prom, lb, rb);
    BP_LAUNCHED("prominence_kernel");
    prominence_flags_kernel<<<grid_for((long long)m + 1, 256), 256, 0, st>>>(
        prom, pos, m, o.prominence_min, o.prominence_max, o.d_prominence_min,
        o.d_prominence_max, flags);
    BP_LAUNCHED("prominence_flags_kernel");
    int* prank = nullptr;
    BP_TRY(sc.get(&prank, (size_t)m + 1));
    BP_TRY(scan_flags(flags, prank, m, sc, st));
    int k = 0;
    BP_TRY(read_back(&k, prank + m, st));
    compact_peaks_kernel<<<grid_for(m, 256), 256, 0, st>>>(flags, prank, m, pos, prom, lb, rb,
                                                           out.peaks, out.prominences,
                                                           out.left_bases, out.right_bases);
    BP_LAUNCHED("compact_peaks_kernel");
    *m_out = k;
    return BP_OK;
  }
  if (m > 0)
    BP_CUDA(cudaMemcpyAsync(out.peaks, pos, (size_t)m * sizeof(int32_t),
                            cudaMemcpyDeviceToDevice, st));
  *m_out = m;
  return BP_OK;
}

bp_peak_options distance_only(double distance) {
  bp_peak_options o{};
  o.distance = distance;
  o.height_min = o.height_max = NAN;
  o.threshold_min = o.threshold_max = NAN;
  o.prominence_min = o.prominence_max = NAN;
  return o;
}

int check_series(const void* p, size_t n, const char* what) {
  if (!p && n) return fail(BP_ERR_INVALID_ARGUMENT, "%s is NULL", what);
  if (n > (size_t)INT_MAX - 1) return fail(BP_ERR_UNSUPPORTED, "%s longer than 2^31 - 2", what);
  return BP_OK;
}

}  // namespace

extern "C" {

float bp_pairwise_sum_f32(const float* x, size_t n) {
  if (n == 0 || !x || n > (size_t)INT_MAX) return 0.0f;
  const PwTree t = pw_tree((int)n);
  std::vector<float> v(t.n_nodes);
  for (const int4& lf : t.leaves) {
    const float* base = x + lf.y;
    v[lf.x] = pw_leaf([&](int i) { return base[i]; }, lf.z);
  }
  for (const int4& nd : t.inner) v[nd.x] = v[nd.y] + v[nd.z];
  return 0.0f + v[t.root];
}

int bp_threshold_dev(const float* d_series, size_t n_samples, size_t sliding_window,
                     double overlap, int kind, float num_dev, const float* d_white_noise,
                     size_t n_white_noise, unsigned long long seed, float* d_threshold,
                     void* stream) {
  BP_NVTX("bp_threshold_dev");
  BP_TRY(check_series(d_series, n_samples, "series"));
  if (!d_threshold) return fail(BP_ERR_INVALID_ARGUMENT, "threshold output is NULL");
  if (kind != BP_THRESHOLD_RMS && kind != BP_THRESHOLD_MAD)
    return fail(BP_ERR_INVALID_ARGUMENT, "threshold kind must be rms (0) or mad (1)");
  if (sliding_window < 1 || n_samples <= sliding_window)
    return fail(BP_ERR_INVALID_ARGUMENT,
                "the series (%zu samples) must be longer than the sliding window (%zu)",
                n_samples, sliding_window);
  const double step = (1.0 - overlap) * (double)sliding_window;
  if (!(step >= 1.0) || step > (double)INT_MAX)
    return fail(BP_ERR_INVALID_ARGUMENT, "(1 - overlap) * sliding_window must be in [1, 2^31)");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int n = (int)n_samples, W = (int)sliding_window, half = W / 2;
  const int shift = (int)step;  // int() truncation, as in the notebook
  const int n_win = (n - W) / shift + 1;
  Scratch sc(st);
  int *zflags = nullptr, *zrank = nullptr;
  float *nz = nullptr, *filled = nullptr, *stats0 = nullptr;
  BP_TRY(sc.get(&zflags, (size_t)n + 1));
  BP_TRY(sc.get(&zrank, (size_t)n + 1));
  BP_TRY(sc.get(&nz, n));
  BP_TRY(sc.get(&filled, n));
  BP_TRY(sc.get(&stats0, 2));  // default centre, deviation
  zero_flags_kernel<<<grid_for((long long)n + 1, 256), 256, 0, st>>>(d_series, n, zflags);
  BP_LAUNCHED("zero_flags_kernel");
  BP_TRY(scan_flags(zflags, zrank, n, sc, st));
  int n_zeros = 0;
  BP_TRY(read_back(&n_zeros, zrank + n, st));
  if (d_white_noise && n_white_noise < (size_t)n_zeros)
    return fail(BP_ERR_INVALID_ARGUMENT, "white noise holds %zu values for %d zero samples",
                n_white_noise, n_zeros);
  const int m = n - n_zeros;
  gather_nonzero_kernel<<<grid_for(n, 256), 256, 0, st>>>(d_series, n, zrank, nz);
  BP_LAUNCHED("gather_nonzero_kernel");
  // centre and deviation of the non-zero samples (NaN when there are none)
  if (kind == BP_THRESHOLD_RMS) {
    if (m > 0) {
      BP_TRY(pw_mean(nz, 0, m, 1, 0, nullptr, stats0, sc, st));
      BP_TRY(pw_mean(nz, 0, m, 1, 1, stats0, stats0 + 1, sc, st));
    }
    finish_stats_kernel<<<1, 32, 0, st>>>(stats0, m > 0 ? 1 : 0);
    BP_LAUNCHED("finish_stats_kernel");
  } else {
    BP_TRY(np_median(nz, 0, m, 1, 0, nullptr, stats0, sc, st));
    BP_TRY(np_median(nz, 0, m, 1, 1, stats0, stats0 + 1, sc, st));
  }
  const float* noise = d_white_noise;
  if (n_zeros > 0 && !noise) {
    float* gen = nullptr;
    BP_TRY(sc.get(&gen, n_zeros));
    normal_kernel<<<grid_for(n_zeros, 256), 256, 0, st>>>(seed, n_zeros, gen);
    BP_LAUNCHED("normal_kernel");
    noise = gen;
  }
  fill_zeros_kernel<<<grid_for(n, 256), 256, 0, st>>>(d_series, n, zrank, noise, stats0,
                                                       stats0 + 1, filled);
  BP_LAUNCHED("fill_zeros_kernel");
  // per-window centre and spread
  float *centre = nullptr, *spread = nullptr, *thr = nullptr, *thr2 = nullptr;
  BP_TRY(sc.get(&centre, n_win));
  BP_TRY(sc.get(&spread, n_win));
  BP_TRY(sc.get(&thr, n_win));
  BP_TRY(sc.get(&thr2, n_win));
  if (kind == BP_THRESHOLD_RMS) {
    BP_TRY(pw_mean(filled, shift, W, n_win, 0, nullptr, centre, sc, st));
    BP_TRY(pw_mean(filled, shift, W, n_win, 1, centre, spread, sc, st));
  } else {
    BP_TRY(np_median(filled, shift, W, n_win, 0, nullptr, centre, sc, st));
    BP_TRY(np_median(filled, shift, W, n_win, 1, centre, spread, sc, st));
  }
  const unsigned gwin = grid_for(n_win, 256);
  window_threshold_kernel<<<gwin, 256, 0, st>>>(centre, spread, n_win,
                                                kind == BP_THRESHOLD_RMS ? 1 : 0, num_dev, thr);
  BP_LAUNCHED("window_threshold_kernel");
  neighbour_max_kernel<<<gwin, 256, 0, st>>>(thr, n_win, -1, thr2);
  BP_LAUNCHED("neighbour_max_kernel");
  neighbour_max_kernel<<<gwin, 256, 0, st>>>(thr2, n_win, +1, thr);
  BP_LAUNCHED("neighbour_max_kernel");
  spread_threshold_kernel<<<grid_for(n, 256), 256, 0, st>>>(thr, n_win, n, W, half, shift,
                                                            d_threshold);
  BP_LAUNCHED("spread_threshold_kernel");
  return BP_OK;
}

int bp_find_peaks_dev(const float* d_x, size_t n_samples, double distance, int32_t* d_peaks,
                      size_t capacity, size_t* n_peaks, void* stream) {
  BP_NVTX("bp_find_peaks_dev");
  BP_TRY(check_series(d_x, n_samples, "series"));
  if (!n_peaks) return fail(BP_ERR_INVALID_ARGUMENT, "n_peaks is NULL");
  *n_peaks = 0;
  if (distance > 0.0 && distance < 1.0)
    return fail(BP_ERR_INVALID_ARGUMENT, "distance must be greater or equal to 1");
  if (capacity < n_samples / 2 || (!d_peaks && n_samples >= 3))
    return fail(BP_ERR_INVALID_ARGUMENT, "peak capacity must be at least n_samples / 2");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  Scratch sc(st);
  int m = 0;
  BP_TRY(find_peaks_impl(d_x, (int)n_samples, distance_only(distance),
                         PeakOut{d_peaks, nullptr, nullptr, nullptr}, &m, sc, st));
  BP_CUDA(cudaStreamSynchronize(st));
  *n_peaks = (size_t)m;
  return BP_OK;
}

int bp_find_peaks_opt_dev(const float* d_x, size_t n_samples, const bp_peak_options* opt,
                          int32_t* d_peaks, double* d_prominences, int32_t* d_left_bases,
                          int32_t* d_right_bases, size_t capacity, size_t* n_peaks,
                          void* stream) {
  BP_NVTX("bp_find_peaks_opt_dev");
  BP_TRY(check_series(d_x, n_samples, "series"));
  if (!n_peaks || !opt) return fail(BP_ERR_INVALID_ARGUMENT, "n_peaks / options is NULL");
  *n_peaks = 0;
  if (opt->distance > 0.0 && opt->distance < 1.0)
    return fail(BP_ERR_INVALID_ARGUMENT, "distance must be greater or equal to 1");
  if (opt->use_prominence && opt->wlen > 0.0 && std::ceil(opt->wlen) <= 1.0)
    return fail(BP_ERR_INVALID_ARGUMENT, "wlen must be larger than 1");
  if (capacity < n_samples / 2 || (!d_peaks && n_samples >= 3))
    return fail(BP_ERR_INVALID_ARGUMENT, "peak capacity must be at least n_samples / 2");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  Scratch sc(st);
  int m = 0;
  BP_TRY(find_peaks_impl(d_x, (int)n_samples, *opt,
                         PeakOut{d_peaks, d_prominences, d_left_bases, d_right_bases}, &m, sc,
                         st));
  BP_CUDA(cudaStreamSynchronize(st));
  *n_peaks = (size_t)m;
  return BP_OK;
}

int bp_detect_dev(const float* d_beam_max, const int32_t* d_argmax, const float* d_threshold,
                  size_t n_samples, double distance, int32_t* d_peaks, float* d_heights,
                  int32_t* d_sources, size_t capacity, size_t* n_detections, void* stream) {
  BP_NVTX("bp_detect_dev");
  BP_TRY(check_series(d_beam_max, n_samples, "beam_max"));
  BP_TRY(check_series(d_threshold, n_samples, "threshold"));
  if (!n_detections) return fail(BP_ERR_INVALID_ARGUMENT, "n_detections is NULL");
  *n_detections = 0;
  if (distance > 0.0 && distance < 1.0)
    return fail(BP_ERR_INVALID_ARGUMENT, "distance must be greater or equal to 1");
  if (capacity < n_samples / 2 || (!d_peaks && n_samples >= 3))
    return fail(BP_ERR_INVALID_ARGUMENT, "detection capacity must be at least n_samples / 2");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  Scratch sc(st);
  const int n = (int)n_samples;
  int* peaks = nullptr;
  BP_TRY(sc.get(&peaks, n / 2 + 1));
  int m = 0;
  BP_TRY(find_peaks_impl(d_beam_max, n, distance_only(distance),
                         PeakOut{peaks, nullptr, nullptr, nullptr}, &m, sc, st));
  if (m == 0) return BP_OK;
  int *flags = nullptr, *rank = nullptr;
  BP_TRY(sc.get(&flags, (size_t)m + 1));
  BP_TRY(sc.get(&rank, (size_t)m + 1));
  above_flags_kernel<<<grid_for((long long)m + 1, 256), 256, 0, st>>>(d_beam_max, d_threshold,
                                                                      peaks, m, flags);
  BP_LAUNCHED("above_flags_kernel");
  BP_TRY(scan_flags(flags, rank, m, sc, st));
  int k = 0;
  BP_TRY(read_back(&k, rank + m, st));
  scatter_detections_kernel<<<grid_for(m, 256), 256, 0, st>>>(
      flags, rank, peaks, m, d_beam_max, d_argmax, d_peaks, d_heights, d_sources);
  BP_LAUNCHED("scatter_detections_kernel");
  BP_CUDA(cudaStreamSynchronize(st));
  *n_detections = (size_t)k;
  return BP_OK;
}

}  // extern "C"
