// C-ABI of libbeampower_b200.so: table management, launch configuration,
// the stream-ordered device entry points and the host-buffer drop-ins.
// Declarations and their reference counterparts: include/beampower_b200.h.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "beampower_b200.h"
#include "bp_common.cuh"
#include "bp_kernels.cuh"
#include "bp_host.h"

namespace bp_host {

thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation)
    return fail(BP_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return fail(BP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int device_sm_count(int dev) {
  static int cache[64] = {0};
  if (dev >= 0 && dev < 64 && cache[dev]) return cache[dev];
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  if (dev >= 0 && dev < 64) cache[dev] = v;
  return v;
}

int device_smem_optin(int dev) {
  static int cache[64] = {0};
  if (dev >= 0 && dev < 64 && cache[dev]) return cache[dev];
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (dev >= 0 && dev < 64) cache[dev] = v;
  return v;
}

// Keeps the device's default stream-ordered pool from returning memory to
// the driver at every synchronisation (cudaMallocAsync scratch is reused).
void retain_pool(int dev) {
  static std::atomic<uint64_t> done{0};
  if (dev < 0 || dev >= 64) return;
  const uint64_t bit = 1ull << dev;
  if (done.load() & bit) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = std::numeric_limits<uint64_t>::max();
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done.fetch_or(bit);
}

}  // namespace bp_host

using namespace bp_host;

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

struct CfgDesc {
  int ks, mt, ws, nstage, sps, k, minb;
};
template <int ID>
constexpr CfgDesc cfg_desc() {
  using C = KCfg<ID>;
  return {C::KS, C::MT, C::WS, C::NSTAGE, C::SPS, C::K, C::MINB};
}
constexpr CfgDesc kCfgDesc[kNumConfigs] = {cfg_desc<0>(), cfg_desc<1>(), cfg_desc<2>(),
                                           cfg_desc<3>(), cfg_desc<4>(), cfg_desc<5>(),
                                           cfg_desc<6>(), cfg_desc<7>(), cfg_desc<8>()};

inline const CfgDesc& cfg_of(int cfg) {
  return kCfgDesc[(cfg >= 0 && cfg < kNumConfigs) ? cfg : 0];
}
inline int cfg_time_tile(int cfg) { return 32 * cfg_of(cfg).mt; }
// Blocks that share one 64-source table tile.
inline int cfg_blocks_per_tile(int cfg) { return kTileSources / cfg_of(cfg).k; }

// Preferred config per (storage, reduce); -1 = built-in default.
std::atomic<int> g_cfg_choice[3][2] = {{{-1}, {-1}}, {{-1}, {-1}}, {{-1}, {-1}}};

int pick_config(int storage, bool maxred) {
  if (const char* v = std::getenv("BEAMPOWER_B200_KERNEL_CONFIG")) {
    const int c = std::atoi(v);
    if (c >= 0 && c < kNumConfigs) return c;
  }
  if (storage >= 0 && storage < 3) {
    const int c = g_cfg_choice[storage][maxred ? 1 : 0].load();
    if (c >= 0 && c < kNumConfigs) return c;
  }
  // Built-in defaults, measured on B200 (400,000 sources x 60 stations x
  // 180,000 samples, reduce='max'): FP32 storage runs fastest with config 8
  // (32-source blocks, 721 ms; config 3 741 ms, config 0 757 ms), 16-bit
  // storage with config 2 (16 warps x 4 sources x 16 samples, two stations
  // per ring stage; FP16 471 ms, BF16 510 ms).
  return storage == BP_STORAGE_F32 ? 8 : 2;
}

}  // namespace

struct bp_table {
  bp::TableDev dev;
  bp_table_info info;
  int32_t* minmax;   // (N, 2) in source order
  void* mem;         // one device allocation holding everything above
  void* direct_mem;  // copies of delays / weights when the direct kernel is used
  int32_t* delays;   // (N, S, P), direct kernel only
  float* weights;    // (N, S), direct kernel only
  int* status;       // kernel status word
  int device;
  cudaStream_t stream;
};

namespace {

__global__ void init_stats_kernel(int* stats, int* status) {
  if (threadIdx.x == 0) {
    stats[bp::kStatMinDelay] = INT_MAX;
    stats[bp::kStatMaxDelay] = INT_MIN;
    stats[bp::kStatMaxSpread] = 0;
    stats[bp::kStatMaxActive] = 0;
    stats[bp::kStatNonFinite] = 0;
    stats[bp::kStatMinLoAligned] = INT_MAX;
    stats[bp::kStatWideTile] = 0;
    stats[7] = 0;
    *status = 0;
  }
}

template <int P>
int launch_table_build(const int32_t* d, const float* w, bp::TableDev& tb, cudaStream_t st) {
  const size_t smem = (size_t)(2 * tb.S * P + tb.S) * sizeof(int);
  if (smem > 48 * 1024)
    BP_CUDA(cudaFuncSetAttribute(bp::table_build_kernel<P>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  bp::table_build_kernel<P><<<tb.n_tiles, 256, smem, st>>>(d, w, tb);
  BP_LAUNCHED("table_build_kernel");
  return BP_OK;
}

size_t pad256(size_t v) { return (v + 255) / 256 * 256; }

// Keep freed stream-ordered allocations in the device's default pool between
// calls (the default release threshold hands them back to the driver at every
// synchronisation, and re-mapping hundreds of MB costs tens of ms per call).

bool tiling_map_enabled() {
  const char* v = std::getenv("BEAMPOWER_B200_TILING_MAP");
  return !(v && v[0] == '0');
}

// Source order for the tiles (see split_dim_kernel): d_perm[n_tiles * K],
// original indices, -1 past the last source.  Segment boundaries depend only
// on N and K (children split at a multiple of K); the data decide which
// (station, phase) delay orders each segment.
int build_tiling_map(const int32_t* d_delays, const float* d_w, size_t N, size_t S, size_t P,
                     int K, int n_tiles, int* d_perm, cudaStream_t st) {
  const int total = n_tiles * K;
  bp::iota_perm_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(d_perm, (int)N, total);
  BP_LAUNCHED("iota_perm_kernel");
  if ((int)N <= K || !tiling_map_enabled()) return BP_OK;
  // Host: per level, every segment in position order (begin, end, splitting?).
  std::vector<int> seg_b, seg_e, seg_dim0, seg_of_tile;
  std::vector<size_t> level_seg_off, level_tile_off;
  std::vector<std::pair<int, int>> cur = {{0, (int)N}};
  int max_segs = 1;
  while (true) {
    bool any_split = false;
    for (auto& be : cur)
      if (be.second - be.first > K) any_split = true;
    if (!any_split) break;
    level_seg_off.push_back(seg_b.size());
    level_tile_off.push_back(seg_of_tile.size());
    std::vector<std::pair<int, int>> next;
    const int base = (int)seg_b.size();
    for (size_t g = 0; g < cur.size(); ++g) {
      const int b = cur[g].first, e = cur[g].second;
      const bool split = e - b > K;
      seg_b.push_back(b);
      seg_e.push_back(e);
      seg_dim0.push_back(split ? 0 : -1);
      for (int t = b / K; t < (e + K - 1) / K; ++t) seg_of_tile.push_back((int)g);
      if (split) {
        const int left = ((e - b + K - 1) / K / 2) * K;
        next.push_back({b, b + left});
        next.push_back({b + left, e});
      } else {
        next.push_back({b, e});
      }
    }
    max_segs = std::max(max_segs, (int)seg_b.size() - base);
    cur.swap(next);
  }
  if (level_seg_off.empty()) return BP_OK;
  level_seg_off.push_back(seg_b.size());
  level_tile_off.push_back(seg_of_tile.size());
  int seg_bits = 1;
  while ((1 << seg_bits) < max_segs) ++seg_bits;
  size_t temp_bytes = 0;
  {
    cudaError_t e = cub::DeviceRadixSort::SortPairs(
        nullptr, temp_bytes, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
        (const int*)nullptr, (int*)nullptr, (int)N, 0, 32 + seg_bits, st);
    if (e != cudaSuccess) return cuda_fail(e, "radix sort size query");
  }
  const size_t ns = seg_b.size(), nt = seg_of_tile.size();
  const size_t o_b = 0, o_e = o_b + pad256(ns * 4), o_d = o_e + pad256(ns * 4),
               o_t = o_d + pad256(ns * 4), o_ka = o_t + pad256(nt * 4),
               o_kb = o_ka + pad256(N * 8), o_pb = o_kb + pad256(N * 8),
               o_tmp = o_pb + pad256(N * 4), bytes = o_tmp + pad256(temp_bytes);
  char* scratch = nullptr;
  BP_CUDA(cudaMallocAsync(&scratch, bytes, st));
  int* d_b = reinterpret_cast<int*>(scratch + o_b);
  int* d_e = reinterpret_cast<int*>(scratch + o_e);
  int* d_dim = reinterpret_cast<int*>(scratch + o_d);
  int* d_tile = reinterpret_cast<int*>(scratch + o_t);
  auto* d_ka = reinterpret_cast<unsigned long long*>(scratch + o_ka);
  auto* d_kb = reinterpret_cast<unsigned long long*>(scratch + o_kb);
  int* d_pb = reinterpret_cast<int*>(scratch + o_pb);
  cudaError_t e = cudaMemcpyAsync(d_b, seg_b.data(), ns * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_e, seg_e.data(), ns * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_dim, seg_dim0.data(), ns * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_tile, seg_of_tile.data(), nt * 4, cudaMemcpyHostToDevice, st);
  int* p_cur = d_perm;
  int* p_next = d_pb;
  for (size_t L = 0; e == cudaSuccess && L + 1 < level_seg_off.size(); ++L) {
    const int nseg = (int)(level_seg_off[L + 1] - level_seg_off[L]);
    int* ldim = d_dim + level_seg_off[L];
    bp::split_dim_kernel<<<nseg, 128, 0, st>>>(d_delays, d_w, (int)S, (int)P, p_cur,
                                               d_b + level_seg_off[L], d_e + level_seg_off[L],
                                               ldim);
    bp::split_keys_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(
        d_delays, (int)(S * P), (int)N, K, p_cur, d_tile + level_tile_off[L], ldim, d_ka);
    g_launches.fetch_add(2, std::memory_order_relaxed);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      size_t tb = temp_bytes;
      e = cub::DeviceRadixSort::SortPairs(scratch + o_tmp, tb, d_ka, d_kb, p_cur, p_next, (int)N,
                                          0, 32 + seg_bits, st);
    }
    std::swap(p_cur, p_next);
  }
  if (e == cudaSuccess && p_cur != d_perm)
    e = cudaMemcpyAsync(d_perm, p_cur, N * 4, cudaMemcpyDeviceToDevice, st);
  int rc = BP_OK;
  if (e != cudaSuccess) rc = cuda_fail(e, "tiling map");
  cudaFreeAsync(scratch, st);
  return rc;
}

template <bool MAXRED>
int launch_window(int cfg, int P, bool checked, int storage, const bp::LaunchArgs& a,
                  bool batch, long long blocks, int dev, cudaStream_t st) {
  switch (cfg) {
    case 1: return launch_window_c<1, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
    case 2: return launch_window_c<2, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
    case 3: return launch_window_c<3, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
    case 4: return launch_window_c<4, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
    case 5: return launch_window_c<5, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
    case 6: return launch_window_c<6, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
    case 7: return launch_window_c<7, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
    case 8: return launch_window_c<8, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
    default: return launch_window_c<0, MAXRED>(P, checked, storage, a, batch, blocks, dev, st);
  }
}

template <int CFG>
size_t staged_smem_cfg(int P, bool maxred, int rowcap, int max_active, int row_factor,
                       int red_rows) {
  using C = KCfg<CFG>;
  auto f = [&](auto tag) -> size_t {
    constexpr int PP = decltype(tag)::value;
    if (maxred)
      return bp::WindowSmem<PP, C::KS, C::MT, C::WS, C::NSTAGE, C::SPS, true>(
                 rowcap, max_active, row_factor, red_rows)
          .total;
    return bp::WindowSmem<PP, C::KS, C::MT, C::WS, C::NSTAGE, C::SPS, false>(
               rowcap, max_active, row_factor, red_rows)
        .total;
  };
  switch (P) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
  }
  return SIZE_MAX;
}

// Shared memory of the staged kernel; storage < 0: the largest over storages.
size_t staged_smem_bytes(int cfg, int P, bool maxred, int rowcap, int max_active, int storage,
                         int red_rows) {
  const int rf = storage == BP_STORAGE_F32 ? bp::ring_row_factor<BP_STORAGE_F32>()
                                           : bp::ring_row_factor<BP_STORAGE_F16>();
  switch (cfg) {
    case 1: return staged_smem_cfg<1>(P, maxred, rowcap, max_active, rf, red_rows);
    case 2: return staged_smem_cfg<2>(P, maxred, rowcap, max_active, rf, red_rows);
    case 3: return staged_smem_cfg<3>(P, maxred, rowcap, max_active, rf, red_rows);
    case 4: return staged_smem_cfg<4>(P, maxred, rowcap, max_active, rf, red_rows);
    case 5: return staged_smem_cfg<5>(P, maxred, rowcap, max_active, rf, red_rows);
    case 6: return staged_smem_cfg<6>(P, maxred, rowcap, max_active, rf, red_rows);
    case 7: return staged_smem_cfg<7>(P, maxred, rowcap, max_active, rf, red_rows);
    case 8: return staged_smem_cfg<8>(P, maxred, rowcap, max_active, rf, red_rows);
    default: return staged_smem_cfg<0>(P, maxred, rowcap, max_active, rf, red_rows);
  }
}

int rowcap_for(const bp_table* t, int cfg) {
  return (int)bp::align_up_sz((size_t)(cfg_time_tile(cfg) + t->info.max_spread + 1),
                              bp::kAlign);
}

int device_smem_per_sm(int dev) {
  static int cache[64] = {0};
  if (dev >= 0 && dev < 64 && cache[dev]) return cache[dev];
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (dev >= 0 && dev < 64) cache[dev] = v;
  return v;
}

// Rows of the max buffer with which config `c` serves table `t`: one per
// consumer warp when that fits, else a single (atomic) row; 0 when neither
// fits a block, or the blocks per SM the shape is built for do not fit an
// SM (a two-block shape left at one block per SM runs at half its
// occupancy).  Without the max reduction the buffer is empty.
int rows_for(const bp_table* t, int c, int storage, bool maxred) {
  const int ws = cfg_of(c).ws;
  const int minb = cfg_of(c).minb;
  for (int rows : {ws, 1}) {
    const size_t need = staged_smem_bytes(c, t->dev.P, maxred, rowcap_for(t, c),
                                          std::max(1, t->info.max_active), storage, rows);
    if (need <= (size_t)device_smem_optin(t->device) &&
        (need + 1024) * (size_t)minb <= (size_t)device_smem_per_sm(t->device))
      return rows;
    if (!maxred) break;
  }
  return 0;
}

bool config_fits(const bp_table* t, int c, int storage, bool maxred) {
  return rows_for(t, c, storage, maxred) > 0;
}

// Fallback order when the chosen shape does not fit a table, fastest first
// (measured on the 400,000-source workload).
const int kOrderF32[kNumConfigs] = {8, 3, 0, 1, 2, 4, 5, 6, 7};
const int kOrder16[kNumConfigs] = {2, 1, 6, 7, 0, 5, 4, 3, 8};

// The preferred config if it serves this table, else the first one of the
// storage's fallback order that does; config 0 (the smallest) as the last
// resort.
int config_for(const bp_table* t, int storage, bool maxred) {
  const int c = pick_config(storage, maxred);
  if (config_fits(t, c, storage, maxred)) return c;
  const int* order = storage == BP_STORAGE_F32 ? kOrderF32 : kOrder16;
  for (int i = 0; i < kNumConfigs; ++i)
    if (config_fits(t, order[i], storage, maxred)) return order[i];
  return 0;
}

// Whether some staged shape serves table `t` with this storage and reduction
// (tables too wide for every shape's ring run the direct kernel).
bool staged_serves(const bp_table* t, int storage, bool maxred) {
  if (!t->info.uses_window_kernel) return false;
  for (int c = 0; c < kNumConfigs; ++c)
    if (config_fits(t, c, storage, maxred)) return true;
  return false;
}

int choose_tiles_per_chunk(int n_tt, int n_tiles, int dev) {
  // Enough blocks for load balance (>= ~16 per SM), chunks of at most 64 time
  // tiles so that the blocks in flight share an L2-resident stretch of trace.
  const long long want_blocks = 16ll * std::max(1, device_sm_count(dev));
  long long tpc = (long long)n_tt * n_tiles / std::max(1ll, want_blocks);
  tpc = std::max(1ll, std::min(tpc, 64ll));
  return (int)std::min<long long>(tpc, n_tt);
}

int check_layout(const bp_table* t, size_t n_samples, size_t lpad, size_t pitch) {
  size_t need_lpad = 0, need_pitch = 0;
  int rc = bp_trace_layout(t, n_samples, &need_lpad, &need_pitch);
  if (rc) return rc;
  if (lpad < need_lpad || pitch < lpad + n_samples ||
      (t->info.uses_window_kernel && (lpad % bp::kAlign || pitch % bp::kAlign ||
                                      pitch - lpad < need_pitch - need_lpad)))
    return fail(BP_ERR_INVALID_ARGUMENT,
                "trace layout lpad=%zu pitch=%zu too small for this table (need %zu, %zu)", lpad,
                pitch, need_lpad, need_pitch);
  return BP_OK;
}

bp::TableView table_view(const bp_table* t) {
  bp::TableView v{};
  v.src_info = t->dev.src_info;
  v.tile_hdr = t->dev.tile_hdr;
  v.st_s = t->dev.st_s;
  v.st_lo = t->dev.st_lo;
  v.st_spread = t->dev.st_spread;
  v.meta = t->dev.meta;
  v.S = t->dev.S;
  v.n_tiles = t->dev.n_tiles;
  return v;
}

int run_staged(const bp_table* t, const void* traces, int storage, const float* scales,
               size_t T, size_t lpad, size_t pitch, int out_of_bounds, unsigned long long* keys,
               float* beam, size_t ldb, cudaStream_t st) {
  bp::LaunchArgs a{};
  a.tab0 = table_view(t);
  bp::RecordView& r = a.rec0;
  r.traces = traces;
  r.scales = scales;
  r.pitch = (long long)pitch;
  r.t_origin = 0;
  r.lpad = (int)lpad;
  r.T = (int)T;
  r.out0 = 0;
  r.out1 = (int)T;
  r.flexible = out_of_bounds;
  r.keys = keys;
  r.beam = beam;
  r.ldb = (long long)ldb;
  const bool maxred = keys != nullptr;
  const int cfg = config_for(t, storage, maxred);
  const int tt = cfg_time_tile(cfg);
  const int n_tt = (int)((T + tt - 1) / tt);
  const int n_btiles = t->dev.n_tiles * cfg_blocks_per_tile(cfg);
  a.tiles_per_chunk = choose_tiles_per_chunk(n_tt, n_btiles, t->device);
  a.rowcap = rowcap_for(t, cfg);
  a.max_active = std::max(1, t->info.max_active);
  a.red_rows = std::max(1, rows_for(t, cfg, storage, maxred));
  a.status = t->status;
  if (n_tt == 0) return BP_OK;
  const long long blocks =
      (long long)((n_tt + a.tiles_per_chunk - 1) / a.tiles_per_chunk) * n_btiles;
  const bool checked = out_of_bounds && t->info.any_nonfinite;
  if (maxred)
    return launch_window<true>(cfg, t->dev.P, checked, storage, a, false, blocks, t->device, st);
  return launch_window<false>(cfg, t->dev.P, checked, storage, a, false, blocks, t->device, st);
}

int run_direct(const void* traces, int storage, const float* scales, size_t T, size_t lpad,
               size_t pitch, const int32_t* delays, const float* weights, const int32_t* minmax,
               size_t N, size_t S, size_t P, int out_of_bounds, unsigned long long* keys,
               float* beam, size_t ldb, cudaStream_t st, int index_base = 0) {
  if (T == 0 || N == 0) return BP_OK;
  bp::DirectArgs a{};
  a.traces = traces;
  a.scales = scales;
  a.pitch = (long long)pitch;
  a.lpad = (int)lpad;
  a.T = (int)T;
  a.N = (int)N;
  a.S = (int)S;
  a.P = (int)P;
  a.flexible = out_of_bounds;
  a.src_per_block = 64;
  a.delays = delays;
  a.weights = weights;
  a.minmax = minmax;
  a.index_base = index_base;
  a.keys = keys;
  a.beam = beam;
  a.ldb = (long long)ldb;
  dim3 grid((unsigned)((T + 255) / 256), (unsigned)((N + a.src_per_block - 1) / a.src_per_block));
  if (grid.y > 65535) {
    a.src_per_block = (int)((N + 65534) / 65535);
    grid.y = (unsigned)((N + a.src_per_block - 1) / a.src_per_block);
  }
#define BP_DIRECT(STOR)                                                        \
  do {                                                                         \
    if (keys) bp::beam_direct_kernel<STOR, true><<<grid, 256, 0, st>>>(a);     \
    else bp::beam_direct_kernel<STOR, false><<<grid, 256, 0, st>>>(a);         \
  } while (0)
  switch (storage) {
    case BP_STORAGE_F32: BP_DIRECT(BP_STORAGE_F32); break;
    case BP_STORAGE_BF16: BP_DIRECT(BP_STORAGE_BF16); break;
    case BP_STORAGE_F16: BP_DIRECT(BP_STORAGE_F16); break;
    default: return fail(BP_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
  }
#undef BP_DIRECT
  BP_LAUNCHED("beam_direct_kernel");
  return BP_OK;
}

int check_sizes(size_t T, size_t N, size_t S, size_t P) {
  if (S == 0 || P == 0) return fail(BP_ERR_INVALID_ARGUMENT, "n_stations and n_phases must be > 0");
  if (T > (size_t)kMaxInt / 2 || N > (size_t)kMaxInt || S > 65535 || P > 64 ||
      S * P > 65535)
    return fail(BP_ERR_UNSUPPORTED, "sizes out of range (T=%zu N=%zu S=%zu P=%zu)", T, N, S, P);
  return BP_OK;
}

// Per-thread stream for the host-buffer entry points.
cudaStream_t host_stream() {
  thread_local cudaStream_t s = nullptr;
  thread_local int dev_of_s = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!s || dev_of_s != dev) {
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    dev_of_s = dev;
    retain_pool(dev);
  }
  return s;
}

// Per-thread second stream of the host entry points: host-buffer uploads
// (a copy from pageable memory waits for the work already on its own stream,
// so it is kept off the stream that runs the kernels) and the tables built
// from them.  Highest priority: a table build's short kernels take SMs ahead
// of the long kernel running beside them on the other stream.
cudaStream_t upload_stream() {
  thread_local cudaStream_t s = nullptr;
  thread_local int dev_of_s = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!s || dev_of_s != dev) {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest);
    dev_of_s = dev;
  }
  return s;
}

// Scoped stream-ordered device buffers for the host entry points.
struct DevBufs {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit DevBufs(cudaStream_t s) : st(s) {}
  template <class T>
  cudaError_t alloc(T** p, size_t bytes) {
    void* v = nullptr;
    cudaError_t e = cudaMallocAsync(&v, std::max<size_t>(bytes, 16), st);
    if (e == cudaSuccess) ptrs.push_back(v);
    *p = reinterpret_cast<T*>(v);
    return e;
  }
  ~DevBufs() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
  }
};

struct TableGuard {
  bp_table* t = nullptr;
  ~TableGuard() {
    if (t) bp_table_destroy(t);
  }
};

int read_status(const bp_table* t, cudaStream_t st) {
  int status = 0;
  BP_CUDA(cudaMemcpyAsync(&status, t->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  if (status) return fail(BP_ERR_KERNEL, "kernel reported status 0x%x", status);
  return BP_OK;
}

void decode_keys_host(const std::vector<unsigned long long>& keys, float* beam_max,
                      int32_t* argmax) {
  for (size_t t = 0; t < keys.size(); ++t) {
    const unsigned long long k = keys[t];
    if (k) {
      beam_max[t] = bp::key_value(k);
      argmax[t] = bp::key_source(k);
    } else {
      argmax[t] = 0;
    }
  }
}

}  // namespace

extern "C" {

const char* bp_last_error(void) { return g_last_error.c_str(); }
const char* bp_version(void) { return "beampower_b200 0.1.0 (sm_100a)"; }
uint64_t bp_launch_count(void) { return g_launches.load(); }

// ---------------------------------------------------------------------------
// Tables
// ---------------------------------------------------------------------------
// A table whose source indexes start at `index_base` (a table over a block
// of a larger grid's sources, whose keys are then global: the host path's
// source chunks); bp_table_create is the case index_base = 0.
static int table_create_based(const int32_t* d_delays, const float* d_weights, size_t N,
                              size_t S, size_t P, void* stream, int index_base,
                              bp_table** out) {
  g_last_error.clear();
  if (!out) return fail(BP_ERR_INVALID_ARGUMENT, "out_table is NULL");
  *out = nullptr;
  if (int rc = check_sizes(0, N, S, P)) return rc;
  if (N > 0 && (!d_delays || !d_weights))
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL delays or weights");
  cudaStream_t st = as_stream(stream);
  int device = 0;
  BP_CUDA(cudaGetDevice(&device));
  bp_table* t = new bp_table();
  std::memset(t, 0, sizeof(*t));
  t->device = device;
  retain_pool(t->device);
  t->stream = st;
  const int K = kTileSources;
  const long long n_tiles = ((long long)N + K - 1) / K;
  const bool window = P <= 4;
  const size_t meta_elem = (P <= 2) ? sizeof(uint2) : sizeof(uint4);
  // one allocation, 256-byte aligned sub-buffers
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += pad256(std::max<size_t>(bytes, 1));
    return o;
  };
  const size_t o_stats = take(bp::kStatCount * sizeof(int));
  const size_t o_status = take(sizeof(int));
  const size_t o_minmax = take(N * 2 * sizeof(int32_t));
  size_t o_src = 0, o_hdr = 0, o_sts = 0, o_stlo = 0, o_stsp = 0, o_meta = 0, o_perm = 0;
  if (window && n_tiles > 0) {
    o_src = take((size_t)n_tiles * K * sizeof(int4));
    o_hdr = take((size_t)n_tiles * sizeof(int2));
    o_sts = take((size_t)n_tiles * S * sizeof(int));
    o_stlo = take((size_t)n_tiles * S * P * sizeof(int));
    o_stsp = take((size_t)n_tiles * S * P * sizeof(int));
    o_meta = take((size_t)n_tiles * S * K * meta_elem);
    o_perm = take((size_t)n_tiles * K * sizeof(int));
  }
  cudaError_t e = cudaMallocAsync(&t->mem, off, st);
  if (e != cudaSuccess) {
    delete t;
    return cuda_fail(e, "cudaMallocAsync(table)");
  }
  char* base = reinterpret_cast<char*>(t->mem);
  t->dev.N = (int)N;
  t->dev.S = (int)S;
  t->dev.P = (int)P;
  t->dev.K = K;
  t->dev.index_base = index_base;
  t->dev.n_tiles = (int)n_tiles;
  t->dev.stats = reinterpret_cast<int*>(base + o_stats);
  t->status = reinterpret_cast<int*>(base + o_status);
  t->minmax = reinterpret_cast<int32_t*>(base + o_minmax);
  if (window && n_tiles > 0) {
    t->dev.src_info = reinterpret_cast<int4*>(base + o_src);
    t->dev.tile_hdr = reinterpret_cast<int2*>(base + o_hdr);
    t->dev.st_s = reinterpret_cast<int*>(base + o_sts);
    t->dev.st_lo = reinterpret_cast<int*>(base + o_stlo);
    t->dev.st_spread = reinterpret_cast<int*>(base + o_stsp);
    t->dev.meta = base + o_meta;
    t->dev.perm = reinterpret_cast<int*>(base + o_perm);
  }

  auto bail = [&](int rc) {
    bp_table_destroy(t);
    return rc;
  };
  init_stats_kernel<<<1, 32, 0, st>>>(t->dev.stats, t->status);
  g_launches.fetch_add(1);
  if (N > 0) {
    bp::minmax_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(d_delays, d_weights, (int)N,
                                                                  (int)S, (int)P, t->minmax);
    g_launches.fetch_add(1);
  }
  if (cudaError_t le = cudaGetLastError(); le != cudaSuccess)
    return bail(cuda_fail(le, "launch minmax_kernel"));
  int rc = BP_OK;
  if (window && n_tiles > 0) {
    rc = build_tiling_map(d_delays, d_weights, N, S, P, K, (int)n_tiles,
                          const_cast<int*>(t->dev.perm), st);
    if (rc) return bail(rc);
    bp::sort_tile_slots_kernel<<<(unsigned)n_tiles, bp::kTableTile, 0, st>>>(
        const_cast<int*>(t->dev.perm), (int)N);
    g_launches.fetch_add(1);
    if (cudaError_t le = cudaGetLastError(); le != cudaSuccess)
      return bail(cuda_fail(le, "launch sort_tile_slots_kernel"));
    switch (P) {
      case 1: rc = launch_table_build<1>(d_delays, d_weights, t->dev, st); break;
      case 2: rc = launch_table_build<2>(d_delays, d_weights, t->dev, st); break;
      case 3: rc = launch_table_build<3>(d_delays, d_weights, t->dev, st); break;
      case 4: rc = launch_table_build<4>(d_delays, d_weights, t->dev, st); break;
    }
    if (rc) return bail(rc);
  }
  int stats[bp::kStatCount];
  e = cudaMemcpyAsync(stats, t->dev.stats, sizeof(stats), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(cuda_fail(e, "table statistics"));

  bp_table_info& in = t->info;
  in.n_sources = (int64_t)N;
  in.n_stations = (int64_t)S;
  in.n_phases = (int64_t)P;
  in.tile_sources = K;
  in.n_tiles = (int32_t)n_tiles;
  in.min_delay = stats[bp::kStatMinDelay];
  in.max_delay = stats[bp::kStatMaxDelay];
  in.max_spread = stats[bp::kStatMaxSpread];
  in.max_active = stats[bp::kStatMaxActive];
  in.any_nonfinite = stats[bp::kStatNonFinite];
  // The staged kernel serves the table when some shape holds its windows
  // with FP32 storage (the smallest ring).  16-bit storage keeps four copies
  // of every window and may fit no shape where FP32 does; such calls expand
  // their traces to FP32 and run the FP32 shapes (run_staged_expanded).
  in.uses_window_kernel = window && n_tiles > 0 && !stats[bp::kStatWideTile] ? 1 : 0;
  if (in.uses_window_kernel && !staged_serves(t, BP_STORAGE_F32, true)) in.uses_window_kernel = 0;
  const bool use_window = in.uses_window_kernel != 0;
  if (!use_window && N > 0) {
    // The direct kernel reads the raw arrays: keep private copies.
    e = cudaMallocAsync(&t->direct_mem, N * S * P * sizeof(int32_t) + N * S * sizeof(float) + 256,
                        st);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMallocAsync(table copies)"));
    t->delays = reinterpret_cast<int32_t*>(t->direct_mem);
    t->weights = reinterpret_cast<float*>(
        reinterpret_cast<char*>(t->direct_mem) + pad256(N * S * P * sizeof(int32_t)));
    e = cudaMemcpyAsync(t->delays, d_delays, N * S * P * sizeof(int32_t),
                        cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(t->weights, d_weights, N * S * sizeof(float), cudaMemcpyDeviceToDevice,
                          st);
    if (e != cudaSuccess) return bail(cuda_fail(e, "copy table arrays"));
  }
  *out = t;
  return BP_OK;
}

int bp_table_create(const int32_t* d_delays, const float* d_weights, size_t N, size_t S,
                    size_t P, void* stream, bp_table** out) {
  BP_NVTX("bp_table_create");
  return table_create_based(d_delays, d_weights, N, S, P, stream, 0, out);
}

int bp_table_destroy(bp_table* t) {
  if (!t) return BP_OK;
  if (t->mem) cudaFreeAsync(t->mem, t->stream);
  if (t->direct_mem) cudaFreeAsync(t->direct_mem, t->stream);
  cudaStreamSynchronize(t->stream);
  delete t;
  return BP_OK;
}

int bp_table_get_info(const bp_table* t, bp_table_info* info) {
  if (!t || !info) return fail(BP_ERR_INVALID_ARGUMENT, "NULL table or info");
  *info = t->info;
  return BP_OK;
}

int bp_trace_layout(const bp_table* t, size_t T, size_t* lpad, size_t* pitch) {
  if (!t || !lpad || !pitch) return fail(BP_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!t->info.uses_window_kernel) {  // the direct kernel reads [0, T) only
    *lpad = 0;
    *pitch = bp::align_up_sz(std::max<size_t>(T, 1), 64);
    return BP_OK;
  }
  const int mn = t->info.min_delay, mx = t->info.max_delay;
  const bool any = mn <= mx;
  // left pad: the lowest aligned window start below zero
  long long lp = 0;
  if (any && mn < 0) lp = -(long long)bp::floor_align(mn);
  lp = (long long)bp::align_up_sz((size_t)lp, 32);
  const long long right = any ? std::max(0, mx) : 0;
  const long long p = (long long)bp::align_up_sz(
      (size_t)(lp + (long long)bp::align_up_sz(T, bp::kMaxTimeTile) + right + 2 * bp::kAlign), 64);
  *lpad = (size_t)lp;
  *pitch = (size_t)p;
  return BP_OK;
}

// ---------------------------------------------------------------------------
// Device entry points
// ---------------------------------------------------------------------------
int bp_minmax_dev(const int32_t* d, const float* w, size_t N, size_t S, size_t P, int32_t* out,
                  void* stream) {
  g_last_error.clear();
  if (int rc = check_sizes(0, N, S, P)) return rc;
  if (N == 0) return BP_OK;
  if (!d || !w || !out) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  bp::minmax_kernel<<<(unsigned)((N + 255) / 256), 256, 0, as_stream(stream)>>>(
      d, w, (int)N, (int)S, (int)P, out);
  BP_LAUNCHED("minmax_kernel");
  return BP_OK;
}

int bp_prestack_dev(const float* F, const float* alpha, size_t T, size_t S, size_t C, size_t P,
                    int storage, size_t lpad, size_t pitch, void* traces, float* scales,
                    void* stream) {
  BP_NVTX("bp_prestack_dev");
  g_last_error.clear();
  if (int rc = check_sizes(T, 0, S, P)) return rc;
  if (C == 0 || C > 65535) return fail(BP_ERR_INVALID_ARGUMENT, "bad n_channels %zu", C);
  if (pitch < lpad + T) return fail(BP_ERR_INVALID_ARGUMENT, "pitch < lpad + n_samples");
  if (!traces || (T > 0 && (!F || !alpha)))
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  cudaStream_t st = as_stream(stream);
  dim3 grid((unsigned)((pitch + 255) / 256), (unsigned)S);
  if (storage == BP_STORAGE_F32) {
    bp::prestack_f32_kernel<<<grid, 256, 0, st>>>(F, alpha, (int)T, (int)S, (int)C, (int)P,
                                                  (int)lpad, (long long)pitch,
                                                  reinterpret_cast<float*>(traces));
  } else {
    if (!scales) return fail(BP_ERR_INVALID_ARGUMENT, "16-bit storage needs a scales buffer");
    if (lpad % 2) return fail(BP_ERR_INVALID_ARGUMENT, "16-bit storage needs an even lpad");
    unsigned int* sb = reinterpret_cast<unsigned int*>(scales);
    BP_CUDA(cudaMemsetAsync(sb, 0, S * sizeof(float), st));
    dim3 g1((unsigned)((T + 255) / 256), (unsigned)S);
    if (T > 0) bp::prestack_absmax_kernel<<<g1, 256, 0, st>>>(F, alpha, (int)T, (int)S, (int)C,
                                                             (int)P, sb);
    bp::scale_pow2_kernel<<<(unsigned)((S + 255) / 256), 256, 0, st>>>(sb, (int)S);
    g_launches.fetch_add(2, std::memory_order_relaxed);
    if (storage == BP_STORAGE_BF16)
      bp::prestack_h16_kernel<BP_STORAGE_BF16><<<grid, 256, 0, st>>>(
          F, alpha, (int)T, (int)S, (int)C, (int)P, (int)lpad, (long long)pitch, scales,
          reinterpret_cast<__nv_bfloat16*>(traces));
    else if (storage == BP_STORAGE_F16)
      bp::prestack_h16_kernel<BP_STORAGE_F16><<<grid, 256, 0, st>>>(
          F, alpha, (int)T, (int)S, (int)C, (int)P, (int)lpad, (long long)pitch, scales,
          reinterpret_cast<__half*>(traces));
    else
      return fail(BP_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
  }
  BP_LAUNCHED("prestack_f32_kernel");
  return BP_OK;
}

int bp_traces_from_prestacked_dev(const float* U, size_t T, size_t S, size_t P, size_t lpad,
                                  size_t pitch, float* traces, void* stream) {
  g_last_error.clear();
  if (int rc = check_sizes(T, 0, S, P)) return rc;
  if (pitch < lpad + T) return fail(BP_ERR_INVALID_ARGUMENT, "pitch < lpad + n_samples");
  if (!traces || (T > 0 && !U)) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  dim3 grid((unsigned)((pitch + 255) / 256), (unsigned)S);
  bp::traces_from_prestacked_kernel<<<grid, 256, 0, as_stream(stream)>>>(
      U, (int)T, (int)S, (int)P, (int)lpad, (long long)pitch, traces);
  BP_LAUNCHED("traces_from_prestacked_kernel");
  return BP_OK;
}

// 16-bit traces of a table whose four-copy windows fit no staged shape while
// its FP32 windows do are expanded to FP32 rows of the same layout in a
// scratch buffer (value * scale_s, exact), and the FP32 staged kernel runs on
// them.  Per term it forms round(w * (u * scale_s)) and adds it with one
// rounding, stations then phases ascending: the value and order of the direct
// kernel's 16-bit path, at the staged kernel's speed.
struct ScratchF32 {
  float* p = nullptr;
  cudaStream_t s = nullptr;
  ~ScratchF32() {
    if (p) cudaFreeAsync(p, s);
  }
};

static bool expands_to_f32(const bp_table* t, int storage, bool maxred) {
  return storage != BP_STORAGE_F32 && !staged_serves(t, storage, maxred) &&
         staged_serves(t, BP_STORAGE_F32, maxred);
}

static int expand_to_f32(const bp_table* t, const void* traces, int storage,
                         const float* scales, size_t pitch, cudaStream_t st, ScratchF32* out) {
  const int S = t->dev.S, P = t->dev.P;
  out->s = st;
  BP_CUDA(cudaMallocAsync(&out->p, (size_t)S * P * pitch * sizeof(float), st));
  const dim3 grid((unsigned)((pitch + 255) / 256), (unsigned)(S * P));
  if (storage == BP_STORAGE_BF16)
    bp::expand_h16_kernel<BP_STORAGE_BF16><<<grid, 256, 0, st>>>(traces, scales, P,
                                                                 (long long)pitch, out->p);
  else
    bp::expand_h16_kernel<BP_STORAGE_F16><<<grid, 256, 0, st>>>(traces, scales, P,
                                                                (long long)pitch, out->p);
  BP_LAUNCHED("expand_h16_kernel");
  return BP_OK;
}

static int run_staged_expanded(const bp_table* t, const void* traces, int storage,
                               const float* scales, size_t T, size_t lpad, size_t pitch,
                               int out_of_bounds, unsigned long long* keys, float* beam,
                               size_t ldb, cudaStream_t st) {
  ScratchF32 f32;
  if (int rc = expand_to_f32(t, traces, storage, scales, pitch, st, &f32)) return rc;
  return run_staged(t, f32.p, BP_STORAGE_F32, nullptr, T, lpad, pitch, out_of_bounds, keys, beam,
                    ldb, st);
}

// Max-reduces the keys of every (source, sample) of table `t` into `keys`
// (not cleared here), with the table's source index base.
static int max_keys(const bp_table* t, const void* traces, int storage, const float* scales,
                    size_t T, size_t lpad, size_t pitch, int out_of_bounds,
                    unsigned long long* keys, cudaStream_t st) {
  if (staged_serves(t, storage, true))
    return run_staged(t, traces, storage, scales, T, lpad, pitch, out_of_bounds, keys, nullptr,
                      0, st);
  if (expands_to_f32(t, storage, true))
    return run_staged_expanded(t, traces, storage, scales, T, lpad, pitch, out_of_bounds, keys,
                               nullptr, 0, st);
  return run_direct(traces, storage, scales, T, lpad, pitch, t->delays, t->weights, t->minmax,
                    t->info.n_sources, t->info.n_stations, t->info.n_phases, out_of_bounds,
                    keys, nullptr, 0, st, t->dev.index_base);
}

int bp_beamform_max_dev(const bp_table* t, const void* traces, int storage, const float* scales,
                        size_t T, size_t lpad, size_t pitch, int out_of_bounds,
                        unsigned long long* keys, float* beam_max, int32_t* argmax,
                        void* stream) {
  BP_NVTX("bp_beamform_max_dev");
  g_last_error.clear();
  if (!t) return fail(BP_ERR_INVALID_ARGUMENT, "NULL table");
  if (out_of_bounds != 0 && out_of_bounds != 1)
    return fail(BP_ERR_INVALID_ARGUMENT, "out_of_bounds must be 0 or 1");
  if (int rc = check_sizes(T, t->info.n_sources, t->info.n_stations, t->info.n_phases)) return rc;
  if (T == 0) return BP_OK;
  if (!traces || !keys || !beam_max || !argmax)
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  if (storage != BP_STORAGE_F32 && !scales)
    return fail(BP_ERR_INVALID_ARGUMENT, "16-bit storage needs scales");
  if (int rc = check_layout(t, T, lpad, pitch)) return rc;
  cudaStream_t st = as_stream(stream);
  BP_CUDA(cudaMemsetAsync(keys, 0, T * sizeof(unsigned long long), st));
  if (int rc = max_keys(t, traces, storage, scales, T, lpad, pitch, out_of_bounds, keys, st))
    return rc;
  bp::decode_keys_kernel<<<(unsigned)((T + 255) / 256), 256, 0, st>>>(keys, (int)T, beam_max,
                                                                      argmax);
  BP_LAUNCHED("decode_keys_kernel");
  return BP_OK;
}

int bp_beamform_dev(const bp_table* t, const void* traces, int storage, const float* scales,
                    size_t T, size_t lpad, size_t pitch, int out_of_bounds, float* beam,
                    size_t ldb, void* stream) {
  BP_NVTX("bp_beamform_dev");
  g_last_error.clear();
  if (!t) return fail(BP_ERR_INVALID_ARGUMENT, "NULL table");
  if (out_of_bounds != 0 && out_of_bounds != 1)
    return fail(BP_ERR_INVALID_ARGUMENT, "out_of_bounds must be 0 or 1");
  if (int rc = check_sizes(T, t->info.n_sources, t->info.n_stations, t->info.n_phases)) return rc;
  if (T == 0 || t->info.n_sources == 0) return BP_OK;
  if (!traces || !beam) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  if (ldb < T) return fail(BP_ERR_INVALID_ARGUMENT, "ldb < n_samples");
  if (storage != BP_STORAGE_F32 && !scales)
    return fail(BP_ERR_INVALID_ARGUMENT, "16-bit storage needs scales");
  if (int rc = check_layout(t, T, lpad, pitch)) return rc;
  if (staged_serves(t, storage, false))
    return run_staged(t, traces, storage, scales, T, lpad, pitch, out_of_bounds, nullptr, beam,
                      ldb, as_stream(stream));
  if (expands_to_f32(t, storage, false))
    return run_staged_expanded(t, traces, storage, scales, T, lpad, pitch, out_of_bounds,
                               nullptr, beam, ldb, as_stream(stream));
  return run_direct(traces, storage, scales, T, lpad, pitch, t->delays, t->weights, t->minmax,
                    t->info.n_sources, t->info.n_stations, t->info.n_phases, out_of_bounds,
                    nullptr, beam, ldb, as_stream(stream));
}

int bp_beamform_max_direct_dev(const void* traces, int storage, const float* scales, size_t T,
                               size_t lpad, size_t pitch, const int32_t* delays,
                               const float* weights, size_t N, size_t S, size_t P,
                               int out_of_bounds, unsigned long long* keys, float* beam_max,
                               int32_t* argmax, void* stream) {
  BP_NVTX("bp_beamform_max_direct_dev");
  g_last_error.clear();
  if (int rc = check_sizes(T, N, S, P)) return rc;
  if (out_of_bounds != 0 && out_of_bounds != 1)
    return fail(BP_ERR_INVALID_ARGUMENT, "out_of_bounds must be 0 or 1");
  if (T == 0) return BP_OK;
  if (!traces || !keys || !beam_max || !argmax || (N > 0 && (!delays || !weights)))
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  if (pitch < lpad + T) return fail(BP_ERR_INVALID_ARGUMENT, "pitch < lpad + n_samples");
  cudaStream_t st = as_stream(stream);
  BP_CUDA(cudaMemsetAsync(keys, 0, T * sizeof(unsigned long long), st));
  if (N > 0) {
    int32_t* mm = nullptr;
    BP_CUDA(cudaMallocAsync(&mm, N * 2 * sizeof(int32_t), st));
    bp::minmax_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(delays, weights, (int)N,
                                                                  (int)S, (int)P, mm);
    g_launches.fetch_add(1);
    int rc = run_direct(traces, storage, scales, T, lpad, pitch, delays, weights, mm, N, S, P,
                        out_of_bounds, keys, nullptr, 0, st);
    cudaFreeAsync(mm, st);
    if (rc) return rc;
  }
  bp::decode_keys_kernel<<<(unsigned)((T + 255) / 256), 256, 0, st>>>(keys, (int)T, beam_max,
                                                                      argmax);
  BP_LAUNCHED("decode_keys_kernel");
  return BP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Host-buffer entry points
// ---------------------------------------------------------------------------
namespace {

// Runs the hot path on device buffers already uploaded: table, traces,
// kernel, and the download of the results.  `traces_fill` writes the trace
// layout (from prestacked traces or from raw features).
template <class Fill>
int host_path(cudaStream_t st, DevBufs& bufs, const int32_t* d_delays, const float* d_w,
              size_t T, size_t N, size_t S, size_t P, int oob, int reduce, int storage,
              Fill traces_fill, float* beam_max, int32_t* argmax, float* beam) {
  TableGuard tg;
  if (int rc = bp_table_create(d_delays, d_w, N, S, P, st, &tg.t)) return rc;
  size_t lpad = 0, pitch = 0;
  if (int rc = bp_trace_layout(tg.t, T, &lpad, &pitch)) return rc;
  // FP32: S*P rows of 4-byte elements; 16-bit: kHalfCopies*S*P rows of 2 bytes
  void* d_traces = nullptr;
  float* d_scales = nullptr;
  BP_CUDA(bufs.alloc(&d_traces, S * P * pitch * (storage == BP_STORAGE_F32 ? 4 : 2 * bp::kHalfCopies)));
  BP_CUDA(bufs.alloc(&d_scales, S * sizeof(float)));
  if (int rc = traces_fill(d_traces, d_scales, lpad, pitch)) return rc;
  if (reduce == BP_REDUCE_MAX) {
    unsigned long long* d_keys = nullptr;
    float* d_bm = nullptr;
    int32_t* d_am = nullptr;
    BP_CUDA(bufs.alloc(&d_keys, T * sizeof(unsigned long long)));
    BP_CUDA(bufs.alloc(&d_bm, T * sizeof(float)));
    BP_CUDA(bufs.alloc(&d_am, T * sizeof(int32_t)));
    if (int rc = bp_beamform_max_dev(tg.t, d_traces, storage, d_scales, T, lpad, pitch, oob,
                                     d_keys, d_bm, d_am, st))
      return rc;
    std::vector<unsigned long long> keys(T);
    BP_CUDA(cudaMemcpyAsync(keys.data(), d_keys, T * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, st));
    if (int rc = read_status(tg.t, st)) return rc;
    decode_keys_host(keys, beam_max, argmax);
  } else {
    float* d_beam = nullptr;
    BP_CUDA(bufs.alloc(&d_beam, std::max<size_t>(N * T, 1) * sizeof(float)));
    // entries the strict rule leaves alone keep the caller's content
    BP_CUDA(cudaMemcpyAsync(d_beam, beam, N * T * sizeof(float), cudaMemcpyHostToDevice, st));
    if (int rc = bp_beamform_dev(tg.t, d_traces, storage, d_scales, T, lpad, pitch, oob, d_beam,
                                 T, st))
      return rc;
    BP_CUDA(cudaMemcpyAsync(beam, d_beam, N * T * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (int rc = read_status(tg.t, st)) return rc;
  }
  return BP_OK;
}

// Sources per chunk of the host path's pipeline (at least), and chunks at most.
constexpr size_t kChunkMinSources = 65536;
constexpr size_t kMaxChunks = 8;

// reduce='max' from host buffers for many sources, as a pipeline: the sources
// in up to kMaxChunks contiguous chunks; each chunk's delays and weights are
// uploaded, and its table built, on the upload stream while the previous
// chunk's kernel runs; the chunk tables' source indexes start at the chunk's
// first source, and every chunk max-reduces into the same keys, so the result
// is the single table's, bit for bit (the keys' max does not depend on the
// order).  The features are prestacked per chunk (each table has its own
// trace layout; the prestack is a fraction of a millisecond).
int host_max_chunked(const float* F, const float* alpha, const int32_t* delays, const float* w,
                     size_t T, size_t N, size_t S, size_t C, size_t P, int oob, int storage,
                     float* beam_max, int32_t* argmax) {
  cudaStream_t st = host_stream();
  cudaStream_t up = upload_stream();
  DevBufs bufs(st);
  const size_t n_chunks = std::min(kMaxChunks, N / kChunkMinSources);
  size_t chunk = (N + n_chunks - 1) / n_chunks;
  chunk = (chunk + kTileSources - 1) / kTileSources * kTileSources;
  float *d_F = nullptr, *d_a = nullptr, *d_w = nullptr;
  int32_t* d_d = nullptr;
  unsigned long long* d_keys = nullptr;
  BP_CUDA(bufs.alloc(&d_d, N * S * P * sizeof(int32_t)));
  BP_CUDA(bufs.alloc(&d_w, N * S * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_F, S * C * T * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_a, S * C * P * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_keys, T * sizeof(unsigned long long)));
  BP_CUDA(cudaMemsetAsync(d_keys, 0, T * sizeof(unsigned long long), st));
  // the allocations above are ordered on `st`; the upload stream waits for them
  std::vector<cudaEvent_t> ev(n_chunks + 1, nullptr);
  // on every return: the upload stream too is drained before the tables and
  // (after this guard) the buffers go -- an early return can leave a chunk's
  // copies and table build queued there that `st` never waited for
  struct Cleanup {
    std::vector<cudaEvent_t>& ev;
    std::vector<bp_table*> tables;
    cudaStream_t st, up;
    ~Cleanup() {
      cudaStreamSynchronize(up);
      cudaStreamSynchronize(st);
      for (bp_table* t : tables) bp_table_destroy(t);
      for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    }
  } cleanup{ev, {}, st, up};
  for (auto& e : ev) BP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  BP_CUDA(cudaEventRecord(ev[n_chunks], st));
  BP_CUDA(cudaStreamWaitEvent(up, ev[n_chunks], 0));
  BP_CUDA(cudaMemcpyAsync(d_F, F, S * C * T * sizeof(float), cudaMemcpyHostToDevice, up));
  BP_CUDA(cudaMemcpyAsync(d_a, alpha, S * C * P * sizeof(float), cudaMemcpyHostToDevice, up));
  for (size_t k = 0; k < n_chunks; ++k) {
    const size_t lo = k * chunk, n = std::min(N, lo + chunk) - lo;
    if (lo >= N) break;
    // upload and table of chunk k (overlapping the kernel of chunk k - 1)
    BP_CUDA(cudaMemcpyAsync(d_d + lo * S * P, delays + lo * S * P, n * S * P * sizeof(int32_t),
                            cudaMemcpyHostToDevice, up));
    BP_CUDA(cudaMemcpyAsync(d_w + lo * S, w + lo * S, n * S * sizeof(float),
                            cudaMemcpyHostToDevice, up));
    bp_table* t = nullptr;
    if (int rc = table_create_based(d_d + lo * S * P, d_w + lo * S, n, S, P, up, (int)lo, &t))
      return rc;
    cleanup.tables.push_back(t);
    BP_CUDA(cudaEventRecord(ev[k], up));
    // prestack and kernel of chunk k, after its upload and table
    BP_CUDA(cudaStreamWaitEvent(st, ev[k], 0));
    size_t lpad = 0, pitch = 0;
    if (int rc = bp_trace_layout(t, T, &lpad, &pitch)) return rc;
    void* d_traces = nullptr;
    float* d_scales = nullptr;
    BP_CUDA(bufs.alloc(&d_traces,
                       S * P * pitch * (storage == BP_STORAGE_F32 ? 4 : 2 * bp::kHalfCopies)));
    BP_CUDA(bufs.alloc(&d_scales, S * sizeof(float)));
    if (int rc = bp_prestack_dev(d_F, d_a, T, S, C, P, storage, lpad, pitch, d_traces, d_scales,
                                 st))
      return rc;
    if (int rc = max_keys(t, d_traces, storage, d_scales, T, lpad, pitch, oob, d_keys, st))
      return rc;
  }
  std::vector<unsigned long long> keys(T);
  BP_CUDA(cudaMemcpyAsync(keys.data(), d_keys, T * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  for (bp_table* t : cleanup.tables)
    if (int rc = read_status(t, st)) return rc;
  decode_keys_host(keys, beam_max, argmax);
  return BP_OK;
}

int prestacked_entry(const float* U, const int* delays, const float* w, size_t T, size_t N,
                     size_t S, size_t P, int oob, int reduce, float* beam_max, int32_t* argmax,
                     float* beam) {
  g_last_error.clear();
  if (int rc = check_sizes(T, N, S, P)) return rc;
  if (oob != 0 && oob != 1) return fail(BP_ERR_INVALID_ARGUMENT, "out_of_bounds must be 0 or 1");
  if (T == 0) return BP_OK;
  if (!U || (N > 0 && (!delays || !w)))
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL input pointer");
  if (reduce == BP_REDUCE_MAX && (!beam_max || !argmax))
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL output pointer");
  if (reduce == BP_REDUCE_NONE && N > 0 && !beam)
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL output pointer");
  if (N == 0) {
    if (reduce == BP_REDUCE_MAX) std::fill(argmax, argmax + T, 0);
    return BP_OK;
  }
  cudaStream_t st = host_stream();
  DevBufs bufs(st);
  float* d_U = nullptr;
  int32_t* d_d = nullptr;
  float* d_w = nullptr;
  BP_CUDA(bufs.alloc(&d_U, S * T * P * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_d, N * S * P * sizeof(int32_t)));
  BP_CUDA(bufs.alloc(&d_w, N * S * sizeof(float)));
  BP_CUDA(cudaMemcpyAsync(d_U, U, S * T * P * sizeof(float), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_d, delays, N * S * P * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_w, w, N * S * sizeof(float), cudaMemcpyHostToDevice, st));
  auto fill = [&](void* d_traces, float*, size_t lpad, size_t pitch) {
    return bp_traces_from_prestacked_dev(d_U, T, S, P, lpad, pitch,
                                         static_cast<float*>(d_traces), st);
  };
  return host_path(st, bufs, d_d, d_w, T, N, S, P, oob, reduce, BP_STORAGE_F32, fill, beam_max,
                   argmax, beam);
}

}  // namespace

extern "C" {

int beamform(float* waveform_features, int* time_delays, float* weights, size_t n_samples,
             size_t n_sources, size_t n_stations, size_t n_phases, int out_of_bounds,
             float* beam) {
  BP_NVTX("beamform");
  return prestacked_entry(waveform_features, time_delays, weights, n_samples, n_sources,
                          n_stations, n_phases, out_of_bounds, BP_REDUCE_NONE, nullptr, nullptr,
                          beam);
}

int beamform_max(float* waveform_features, int* time_delays, float* weights, size_t n_samples,
                 size_t n_sources, size_t n_stations, size_t n_phases, int out_of_bounds,
                 float* beam_max, int* source_index_beam_max) {
  BP_NVTX("beamform_max");
  return prestacked_entry(waveform_features, time_delays, weights, n_samples, n_sources,
                          n_stations, n_phases, out_of_bounds, BP_REDUCE_MAX, beam_max,
                          source_index_beam_max, nullptr);
}

int prestack_waveform_features(float* F, float* alpha, size_t T, size_t S, size_t C, size_t P,
                               int num_threads, float* out) {
  BP_NVTX("prestack_waveform_features");
  (void)num_threads;
  g_last_error.clear();
  if (int rc = check_sizes(T, 0, S, P)) return rc;
  if (C == 0 || C > 65535) return fail(BP_ERR_INVALID_ARGUMENT, "bad n_channels %zu", C);
  if (T == 0) return BP_OK;
  if (!F || !alpha || !out) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  cudaStream_t st = host_stream();
  DevBufs bufs(st);
  float *d_F = nullptr, *d_a = nullptr, *d_rows = nullptr, *d_U = nullptr;
  BP_CUDA(bufs.alloc(&d_F, S * C * T * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_a, S * C * P * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_rows, S * P * T * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_U, S * T * P * sizeof(float)));
  BP_CUDA(cudaMemcpyAsync(d_F, F, S * C * T * sizeof(float), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_a, alpha, S * C * P * sizeof(float), cudaMemcpyHostToDevice, st));
  if (int rc = bp_prestack_dev(d_F, d_a, T, S, C, P, BP_STORAGE_F32, 0, T, d_rows, nullptr, st))
    return rc;
  // rows (S, P, T) -> (S, T, P), the reference's prestack layout
  dim3 grid((unsigned)((T + 255) / 256), (unsigned)S);
  bp::rows_to_prestacked_kernel<<<grid, 256, 0, st>>>(d_rows, (int)T, (int)S, (int)P, d_U);
  BP_LAUNCHED("rows_to_prestacked_kernel");
  BP_CUDA(cudaMemcpyAsync(out, d_U, S * T * P * sizeof(float), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  return BP_OK;
}

int bp_beamform_host(const float* F, const float* alpha, const int32_t* delays, const float* w,
                     size_t T, size_t N, size_t S, size_t C, size_t P, int oob, int reduce,
                     int storage, float* beam_max, int32_t* argmax, float* beam) {
  BP_NVTX("bp_beamform_host");
  g_last_error.clear();
  if (int rc = check_sizes(T, N, S, P)) return rc;
  if (C == 0 || C > 65535) return fail(BP_ERR_INVALID_ARGUMENT, "bad n_channels %zu", C);
  if (oob != 0 && oob != 1) return fail(BP_ERR_INVALID_ARGUMENT, "out_of_bounds must be 0 or 1");
  if (reduce != BP_REDUCE_MAX && reduce != BP_REDUCE_NONE)
    return fail(BP_ERR_INVALID_ARGUMENT, "reduce must be BP_REDUCE_MAX or BP_REDUCE_NONE");
  if (storage != BP_STORAGE_F32 && storage != BP_STORAGE_BF16 && storage != BP_STORAGE_F16)
    return fail(BP_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
  if (T == 0) return BP_OK;
  if (!F || !alpha || (N > 0 && (!delays || !w)))
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL input pointer");
  if (reduce == BP_REDUCE_MAX && (!beam_max || !argmax))
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL output pointer");
  if (reduce == BP_REDUCE_NONE && N > 0 && !beam)
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL output pointer");
  if (N == 0) {
    if (reduce == BP_REDUCE_MAX) std::fill(argmax, argmax + T, 0);
    return BP_OK;
  }
  if (reduce == BP_REDUCE_MAX && N >= 2 * kChunkMinSources)
    return host_max_chunked(F, alpha, delays, w, T, N, S, C, P, oob, storage, beam_max, argmax);
  cudaStream_t st = host_stream();
  DevBufs bufs(st);
  float *d_F = nullptr, *d_a = nullptr, *d_w = nullptr;
  int32_t* d_d = nullptr;
  BP_CUDA(bufs.alloc(&d_d, N * S * P * sizeof(int32_t)));
  BP_CUDA(bufs.alloc(&d_w, N * S * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_F, S * C * T * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_a, S * C * P * sizeof(float)));
  BP_CUDA(cudaMemcpyAsync(d_d, delays, N * S * P * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_w, w, N * S * sizeof(float), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_F, F, S * C * T * sizeof(float), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_a, alpha, S * C * P * sizeof(float), cudaMemcpyHostToDevice, st));
  auto fill = [&](void* d_traces, float* d_scales, size_t lpad, size_t pitch) {
    return bp_prestack_dev(d_F, d_a, T, S, C, P, storage, lpad, pitch, d_traces, d_scales, st);
  };
  return host_path(st, bufs, d_d, d_w, T, N, S, P, oob, reduce, storage, fill, beam_max, argmax,
                   beam);
}

}  // extern "C"

extern "C" {

int bp_beamform_differential_dev(const float* traces, size_t T, size_t lpad, size_t pitch,
                                 const int32_t* delays, const float* weights, size_t N, size_t S,
                                 size_t P, float* beam, void* stream) {
  BP_NVTX("bp_beamform_differential_dev");
  g_last_error.clear();
  if (int rc = check_sizes(T, N, S, P)) return rc;
  if (N == 0 || T == 0) return BP_OK;
  if (!traces || !delays || !weights || !beam) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  if (pitch < lpad + T) return fail(BP_ERR_INVALID_ARGUMENT, "pitch < lpad + n_samples");
  bp::differential_kernel<<<(unsigned)((N + 127) / 128), 128, 0, as_stream(stream)>>>(
      traces, (long long)pitch, (int)lpad, (int)T, delays, weights, (int)N, (int)S, (int)P, beam);
  BP_LAUNCHED("differential_kernel");
  return BP_OK;
}

int beamform_differential(float* U, int* delays, float* w, size_t T, size_t N, size_t S,
                          size_t P, int num_threads, float* beam) {
  BP_NVTX("beamform_differential");
  (void)num_threads;
  g_last_error.clear();
  if (int rc = check_sizes(T, N, S, P)) return rc;
  if (N == 0 || T == 0) return BP_OK;
  if (!U || !delays || !w || !beam) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  cudaStream_t st = host_stream();
  DevBufs bufs(st);
  float *d_U = nullptr, *d_rows = nullptr, *d_w = nullptr, *d_beam = nullptr;
  int32_t* d_d = nullptr;
  BP_CUDA(bufs.alloc(&d_U, S * T * P * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_rows, S * P * T * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_d, N * S * P * sizeof(int32_t)));
  BP_CUDA(bufs.alloc(&d_w, N * S * sizeof(float)));
  BP_CUDA(bufs.alloc(&d_beam, N * sizeof(float)));
  BP_CUDA(cudaMemcpyAsync(d_U, U, S * T * P * sizeof(float), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_d, delays, N * S * P * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_w, w, N * S * sizeof(float), cudaMemcpyHostToDevice, st));
  BP_CUDA(cudaMemcpyAsync(d_beam, beam, N * sizeof(float), cudaMemcpyHostToDevice, st));
  if (int rc = bp_traces_from_prestacked_dev(d_U, T, S, P, 0, T, d_rows, st)) return rc;
  if (int rc = bp_beamform_differential_dev(d_rows, T, 0, T, d_d, d_w, N, S, P, d_beam, st))
    return rc;
  BP_CUDA(cudaMemcpyAsync(beam, d_beam, N * sizeof(float), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  return BP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches
// ---------------------------------------------------------------------------
struct bp_batch {
  int device;
  int P;
  int storage;
  int n_records;
  int rowcap;
  int cfg;
  int max_active;
  int red_rows;
  bool checked;
  void* mem;                        // device: tables, records, prefix, keys, srcmm, queue, status
  bp::TableView* d_tables;
  bp::RecordView* d_records;
  long long* d_prefix;
  unsigned long long* d_keys;
  size_t n_keys;
  unsigned long long* d_queue;
  int* d_status;
  cudaStream_t stream;
};

namespace {
constexpr int kBatchSamplesPerItem = 16384;  // samples per work item

int masked_minmax(const bp::TableView& tv, int P, const uint32_t* mask, int2* out,
                  cudaStream_t st) {
  const long long slots = (long long)tv.n_tiles * kTileSources;
  const unsigned grid = (unsigned)((slots + 255) / 256);
  switch (P) {
    case 1: bp::masked_minmax_kernel<1><<<grid, 256, 0, st>>>(tv, kTileSources, mask, out); break;
    case 2: bp::masked_minmax_kernel<2><<<grid, 256, 0, st>>>(tv, kTileSources, mask, out); break;
    case 3: bp::masked_minmax_kernel<3><<<grid, 256, 0, st>>>(tv, kTileSources, mask, out); break;
    case 4: bp::masked_minmax_kernel<4><<<grid, 256, 0, st>>>(tv, kTileSources, mask, out); break;
    default: return fail(BP_ERR_UNSUPPORTED, "batches support 1..4 phases");
  }
  BP_LAUNCHED("masked_minmax_kernel");
  return BP_OK;
}
}  // namespace

extern "C" {

int bp_batch_create(const bp_table* const* tables, int n_tables, const bp_record* records,
                    int n_records, int storage, void* stream, bp_batch** out) {
  g_last_error.clear();
  if (!out) return fail(BP_ERR_INVALID_ARGUMENT, "out_batch is NULL");
  *out = nullptr;
  if (!tables || n_tables <= 0 || !records || n_records <= 0)
    return fail(BP_ERR_INVALID_ARGUMENT, "empty batch");
  if (storage != BP_STORAGE_F32 && storage != BP_STORAGE_BF16 && storage != BP_STORAGE_F16)
    return fail(BP_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
  cudaStream_t st = as_stream(stream);
  int dev = 0;
  BP_CUDA(cudaGetDevice(&dev));
  retain_pool(dev);
  const int P = tables[0] ? tables[0]->dev.P : 0;
  // the preferred shape if it serves every table, else the first of the
  // fallback order that does
  int cfg = -1;
  {
    const int pref = pick_config(storage, true);
    const int* order = storage == BP_STORAGE_F32 ? kOrderF32 : kOrder16;
    for (int i = -1; i < kNumConfigs && cfg < 0; ++i) {
      const int c = i < 0 ? pref : order[i];
      bool all = true;
      for (int j = 0; j < n_tables; ++j)
        if (tables[j] && staged_serves(tables[j], storage, true) &&
            !config_fits(tables[j], c, storage, true))
          all = false;
      if (all) cfg = c;
    }
    if (cfg < 0) cfg = 0;
  }
  // one max-buffer row per warp only if every table leaves room for it
  int red_rows = cfg_of(cfg).ws;
  for (int j = 0; j < n_tables; ++j)
    if (tables[j] && staged_serves(tables[j], storage, true))
      red_rows = std::min(red_rows, std::max(1, rows_for(tables[j], cfg, storage, true)));
  const int tt = cfg_time_tile(cfg);
  int rowcap = 0, max_active = 1;
  bool any_nonfinite = false;
  std::vector<bp::TableView> tv(n_tables);
  for (int i = 0; i < n_tables; ++i) {
    const bp_table* t = tables[i];
    if (!t) return fail(BP_ERR_INVALID_ARGUMENT, "NULL table %d", i);
    if (!staged_serves(t, storage, true))
      return fail(BP_ERR_UNSUPPORTED,
                  "table %d needs the direct kernel with this storage; batches use the staged one",
                  i);
    if (t->dev.P != P) return fail(BP_ERR_INVALID_ARGUMENT, "tables of a batch share n_phases");
    if (t->device != dev) return fail(BP_ERR_INVALID_ARGUMENT, "table %d is on another device", i);
    rowcap = std::max(rowcap, rowcap_for(t, cfg));
    max_active = std::max(max_active, t->info.max_active);
    any_nonfinite |= t->info.any_nonfinite != 0;
    tv[i] = table_view(t);
  }
  std::vector<bp::RecordView> rv(n_records);
  std::vector<long long> prefix(n_records + 1, 0);
  size_t n_keys = 0, n_srcmm = 0;
  bool any_flexible = false;
  for (int r = 0; r < n_records; ++r) {
    const bp_record& q = records[r];
    if (q.table < 0 || q.table >= n_tables)
      return fail(BP_ERR_INVALID_ARGUMENT, "record %d: table index %d", r, q.table);
    const bp_table* t = tables[q.table];
    if (q.out_of_bounds != 0 && q.out_of_bounds != 1)
      return fail(BP_ERR_INVALID_ARGUMENT, "record %d: out_of_bounds must be 0 or 1", r);
    if (q.out0 > q.out1 || q.out1 > q.n_samples || q.n_samples > (size_t)kMaxInt / 2)
      return fail(BP_ERR_INVALID_ARGUMENT, "record %d: output range outside the record", r);
    if (!q.traces || !q.beam_max || !q.argmax || (storage != BP_STORAGE_F32 && !q.scales))
      return fail(BP_ERR_INVALID_ARGUMENT, "record %d: NULL pointer", r);
    if (int rc = check_layout(t, q.n_samples, q.lpad, q.pitch)) return rc;
    any_flexible |= q.out_of_bounds != 0;
    bp::RecordView& v = rv[r];
    v = bp::RecordView{};
    v.traces = q.traces;
    v.scales = q.scales;
    v.pitch = (long long)q.pitch;
    v.t_origin = q.t_origin;
    v.lpad = (int)q.lpad;
    v.T = (int)q.n_samples;
    v.out0 = (int)q.out0;
    v.out1 = (int)q.out1;
    v.flexible = q.out_of_bounds;
    v.table = q.table;
    v.tpc = kBatchSamplesPerItem / tt;
    const int tau_first = v.out0 / tt;
    const int tau_end = (v.out1 + tt - 1) / tt;
    v.n_chunks = (tau_end - tau_first + v.tpc - 1) / v.tpc;
    v.station_mask = q.station_mask;
    v.beam_max = q.beam_max;
    v.argmax = q.argmax;
    prefix[r + 1] =
        prefix[r] + (long long)v.n_chunks * t->dev.n_tiles * cfg_blocks_per_tile(cfg);
    n_keys += q.out1 - q.out0;
    if (q.station_mask) n_srcmm += (size_t)t->dev.n_tiles * kTileSources;
  }
  bp_batch* b = new bp_batch();
  b->device = dev;
  b->P = P;
  b->storage = storage;
  b->n_records = n_records;
  b->rowcap = rowcap;
  b->cfg = cfg;
  b->max_active = max_active;
  b->red_rows = red_rows;
  b->checked = any_flexible && any_nonfinite;
  b->stream = st;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += pad256(std::max<size_t>(bytes, 1));
    return o;
  };
  const size_t o_t = take(n_tables * sizeof(bp::TableView));
  const size_t o_r = take(n_records * sizeof(bp::RecordView));
  const size_t o_p = take((n_records + 1) * sizeof(long long));
  const size_t o_k = take(n_keys * sizeof(unsigned long long));
  const size_t o_m = take(n_srcmm * sizeof(int2));
  const size_t o_q = take(sizeof(unsigned long long));
  const size_t o_s = take(sizeof(int));
  cudaError_t e = cudaMallocAsync(&b->mem, off, st);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(e, "cudaMallocAsync(batch)");
  }
  char* base = static_cast<char*>(b->mem);
  b->d_tables = reinterpret_cast<bp::TableView*>(base + o_t);
  b->d_records = reinterpret_cast<bp::RecordView*>(base + o_r);
  b->d_prefix = reinterpret_cast<long long*>(base + o_p);
  b->d_keys = reinterpret_cast<unsigned long long*>(base + o_k);
  b->n_keys = n_keys;
  b->d_queue = reinterpret_cast<unsigned long long*>(base + o_q);
  b->d_status = reinterpret_cast<int*>(base + o_s);
  auto bail = [&](int rc) {
    bp_batch_destroy(b);
    return rc;
  };
  // keys and delay ranges inside the allocation
  size_t koff = 0, moff = 0;
  int2* d_srcmm = reinterpret_cast<int2*>(base + o_m);
  for (int r = 0; r < n_records; ++r) {
    rv[r].keys = b->d_keys + koff;
    koff += (size_t)(rv[r].out1 - rv[r].out0);
    if (records[r].station_mask) {
      rv[r].srcmm = d_srcmm + moff;
      const bp::TableView& t = tv[rv[r].table];
      if (int rc = masked_minmax(t, P, records[r].station_mask, d_srcmm + moff, st))
        return bail(rc);
      moff += (size_t)t.n_tiles * kTileSources;
    }
  }
  e = cudaMemcpyAsync(b->d_tables, tv.data(), n_tables * sizeof(bp::TableView),
                      cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_records, rv.data(), n_records * sizeof(bp::RecordView),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_prefix, prefix.data(), (n_records + 1) * sizeof(long long),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_status, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return bail(cuda_fail(e, "batch descriptors"));
  *out = b;
  return BP_OK;
}

int bp_batch_run(bp_batch* b, void* stream) {
  BP_NVTX("bp_batch_run");
  g_last_error.clear();
  if (!b) return fail(BP_ERR_INVALID_ARGUMENT, "NULL batch");
  cudaStream_t st = as_stream(stream);
  BP_CUDA(cudaMemsetAsync(b->d_keys, 0, std::max<size_t>(b->n_keys, 1) * 8, st));
  BP_CUDA(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned long long), st));
  bp::LaunchArgs a{};
  a.tables = b->d_tables;
  a.records = b->d_records;
  a.rec_prefix = b->d_prefix;
  a.n_records = b->n_records;
  a.next_item = b->d_queue;
  a.rowcap = b->rowcap;
  a.max_active = b->max_active;
  a.red_rows = b->red_rows;
  a.status = b->d_status;
  if (int rc = launch_window<true>(b->cfg, b->P, b->checked, b->storage, a, true, 0, b->device,
                                   st))
    return rc;
  dim3 grid(64, (unsigned)b->n_records);
  bp::batch_decode_kernel<<<grid, 256, 0, st>>>(b->d_records);
  BP_LAUNCHED("batch_decode_kernel");
  return BP_OK;
}

int bp_batch_status(bp_batch* b, void* stream, int* status) {
  if (!b || !status) return fail(BP_ERR_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t st = as_stream(stream);
  BP_CUDA(cudaMemcpyAsync(status, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  return BP_OK;
}

int bp_batch_destroy(bp_batch* b) {
  if (!b) return BP_OK;
  if (b->mem) cudaFreeAsync(b->mem, b->stream);
  cudaStreamSynchronize(b->stream);
  delete b;
  return BP_OK;
}

}  // extern "C"

extern "C" {

int bp_record_beamform_max_dev(const bp_table* t, const bp_record* q, int storage,
                               unsigned long long* keys, void* stream) {
  BP_NVTX("bp_record_beamform_max_dev");
  g_last_error.clear();
  if (!t || !q || !keys) return fail(BP_ERR_INVALID_ARGUMENT, "NULL argument");
  const bool expand = expands_to_f32(t, storage, true);
  if (!expand && !staged_serves(t, storage, true))
    return fail(BP_ERR_UNSUPPORTED, "records need a table that the staged kernel serves");
  if (q->station_mask) return fail(BP_ERR_INVALID_ARGUMENT, "station masks need a batch");
  if (q->out_of_bounds != 0 && q->out_of_bounds != 1)
    return fail(BP_ERR_INVALID_ARGUMENT, "out_of_bounds must be 0 or 1");
  if (q->out0 > q->out1 || q->out1 > q->n_samples || q->n_samples > (size_t)kMaxInt / 2)
    return fail(BP_ERR_INVALID_ARGUMENT, "output range outside the record");
  if (!q->traces || !q->beam_max || !q->argmax || (storage != BP_STORAGE_F32 && !q->scales))
    return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  if (int rc = check_layout(t, q->n_samples, q->lpad, q->pitch)) return rc;
  const size_t n_out = q->out1 - q->out0;
  if (n_out == 0) return BP_OK;
  cudaStream_t st = as_stream(stream);
  BP_CUDA(cudaMemsetAsync(keys, 0, n_out * sizeof(unsigned long long), st));
  ScratchF32 f32;
  if (expand) {
    if (int rc = expand_to_f32(t, q->traces, storage, q->scales, q->pitch, st, &f32)) return rc;
    storage = BP_STORAGE_F32;
  }
  bp::LaunchArgs a{};
  a.tab0 = table_view(t);
  bp::RecordView& r = a.rec0;
  r.traces = expand ? static_cast<const void*>(f32.p) : q->traces;
  r.scales = expand ? nullptr : q->scales;
  r.pitch = (long long)q->pitch;
  r.t_origin = q->t_origin;
  r.lpad = (int)q->lpad;
  r.T = (int)q->n_samples;
  r.out0 = (int)q->out0;
  r.out1 = (int)q->out1;
  r.flexible = q->out_of_bounds;
  r.keys = keys;
  const int cfg = config_for(t, storage, true);
  const int tt = cfg_time_tile(cfg);
  const int tau_first = r.out0 / tt;
  const int n_tt = (r.out1 + tt - 1) / tt - tau_first;
  const int n_btiles = t->dev.n_tiles * cfg_blocks_per_tile(cfg);
  a.tiles_per_chunk = choose_tiles_per_chunk(n_tt, n_btiles, t->device);
  a.rowcap = rowcap_for(t, cfg);
  a.max_active = std::max(1, t->info.max_active);
  a.red_rows = std::max(1, rows_for(t, cfg, storage, true));
  a.status = t->status;
  const long long blocks =
      (long long)((n_tt + a.tiles_per_chunk - 1) / a.tiles_per_chunk) * n_btiles;
  const bool checked = q->out_of_bounds && t->info.any_nonfinite;
  if (int rc = launch_window<true>(cfg, t->dev.P, checked, storage, a, false, blocks, t->device,
                                   st))
    return rc;
  bp::decode_keys_kernel<<<(unsigned)((n_out + 255) / 256), 256, 0, st>>>(
      keys, (int)n_out, q->beam_max, q->argmax);
  BP_LAUNCHED("decode_keys_kernel");
  return BP_OK;
}

}  // extern "C"

extern "C" {

int bp_trace_copies(int storage) {
  if (storage == BP_STORAGE_F32) return 1;
  if (storage == BP_STORAGE_BF16 || storage == BP_STORAGE_F16) return bp::kHalfCopies;
  fail(BP_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
  return -1;
}

int bp_kernel_config_count(void) { return kNumConfigs; }

int bp_kernel_config_describe(int cfg, int* sources_per_thread, int* samples_per_lane,
                              int* consumer_warps, int* stages) {
  if (cfg < 0 || cfg >= kNumConfigs) return fail(BP_ERR_INVALID_ARGUMENT, "no config %d", cfg);
  const CfgDesc& d = kCfgDesc[cfg];
  if (sources_per_thread) *sources_per_thread = d.ks;
  if (samples_per_lane) *samples_per_lane = d.mt;
  if (consumer_warps) *consumer_warps = d.ws;
  if (stages) *stages = d.nstage;
  return BP_OK;
}

int bp_kernel_config_shape(int cfg, int* stations_per_stage, int* sources_per_block,
                           int* blocks_per_sm) {
  if (cfg < 0 || cfg >= kNumConfigs) return fail(BP_ERR_INVALID_ARGUMENT, "no config %d", cfg);
  const CfgDesc& d = kCfgDesc[cfg];
  if (stations_per_stage) *stations_per_stage = d.sps;
  if (sources_per_block) *sources_per_block = d.k;
  if (blocks_per_sm) *blocks_per_sm = d.minb;
  return BP_OK;
}

int bp_set_kernel_config(int storage, int reduce, int cfg) {
  if (storage < 0 || storage > 2 || (reduce != BP_REDUCE_MAX && reduce != BP_REDUCE_NONE))
    return fail(BP_ERR_INVALID_ARGUMENT, "bad storage / reduce");
  if (cfg < -1 || cfg >= kNumConfigs) return fail(BP_ERR_INVALID_ARGUMENT, "no config %d", cfg);
  g_cfg_choice[storage][reduce == BP_REDUCE_MAX ? 1 : 0].store(cfg);
  return BP_OK;
}

int bp_table_kernel_config(const bp_table* t, int storage, int reduce) {
  if (!t) return fail(BP_ERR_INVALID_ARGUMENT, "NULL table");
  if (storage < 0 || storage > 2 || (reduce != BP_REDUCE_MAX && reduce != BP_REDUCE_NONE))
    return fail(BP_ERR_INVALID_ARGUMENT, "bad storage / reduce");
  if (!staged_serves(t, storage, reduce == BP_REDUCE_MAX)) return -1;
  return config_for(t, storage, reduce == BP_REDUCE_MAX);
}

int bp_get_kernel_config(int storage, int reduce) {
  if (storage < 0 || storage > 2) return 0;
  return pick_config(storage, reduce == BP_REDUCE_MAX);
}

}  // extern "C"

namespace {
// A wait that can never complete: an mbarrier expecting one arrival that no
// thread makes.  Every thread gives up after `limit_ns` and the kernel ends.
__global__ void wait_timeout_probe_kernel(unsigned long long limit_ns, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    bp::mbar_init(&bar, 1);
    bp::fence_mbar_init();
  }
  __syncthreads();
  bp::mbar_wait_limit(&bar, 0, limit_ns, status);
}
}  // namespace

extern "C" {

int bp_debug_wait_timeout(unsigned long long limit_ns, void* stream, int* status_out) {
  g_last_error.clear();
  if (!status_out) return fail(BP_ERR_INVALID_ARGUMENT, "NULL status");
  if (limit_ns > 1000000000ull) return fail(BP_ERR_INVALID_ARGUMENT, "limit above 1 s");
  cudaStream_t st = as_stream(stream);
  int* d = nullptr;
  BP_CUDA(cudaMallocAsync(&d, sizeof(int), st));
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    wait_timeout_probe_kernel<<<1, 64, 0, st>>>(limit_ns, d);
    g_launches.fetch_add(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(status_out, d, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "wait timeout probe");
  return BP_OK;
}

}  // extern "C"
