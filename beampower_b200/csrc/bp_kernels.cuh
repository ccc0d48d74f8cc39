// sm_100a kernels of the beamforming hot path.
//
// Data layout in HBM
//   traces   row r = s * P + p holds phase p of station s: element (s, p, t)
//            at traces[r * pitch + lpad + t]; indexes outside [lpad, lpad + T)
//            are zero.  Written once per record by the prestack kernel.
//   table    built once per (time_delays, weights) pair: sources grouped in
//            tiles of K; per tile the active stations (some source of the
//            tile weights them), per (tile, station, phase) the delay window
//            lo .. lo + spread (lo aligned down to kAlign samples), per
//            (tile, station, source) the weight and the delay offsets
//            d - lo as 16-bit integers, per source its min/max delay over
//            weighted stations (the strict validity rule).
//   keys     (T,) uint64 packed (beam, source) keys, max-reduced in place.
#pragma once

#include <cfloat>
#include <climits>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "bp_common.cuh"

namespace bp {

// Window starts are aligned down to this many samples (32 bytes of FP32,
// 16 bytes of 16-bit storage), so every bulk copy starts 16-byte aligned.
constexpr int kAlign = 8;
// 16-bit trace storage keeps this many copies of every row, copy v shifted
// by v samples, so that any run of 4 samples is one 8-byte-aligned pair of
// 32-bit words in one of the copies (one 64-bit shared load per lane).
constexpr int kHalfCopies = 4;
// Checked build (-DBP_DEBUG_CHECKS=1, libbeampower_b200_checked.so): the
// staged kernel checks every bulk copy against the trace buffer and its ring
// row and every shared-memory read against the copied window; a failed check
// records kStatusBadIndex in the status word and skips the access (a skipped
// copy is left out of the stage's expected bytes, so no wait depends on it).
#ifndef BP_DEBUG_CHECKS
#define BP_DEBUG_CHECKS 0
#endif
// 32-bit words of one ring row per sample of window capacity: FP32 1, 16-bit
// 2 (kHalfCopies copies of 2-byte elements).
template <int STORAGE>
constexpr int ring_row_factor() {
  return STORAGE == BP_STORAGE_F32 ? 1 : kHalfCopies / 2;
}
// Largest time tile of any kernel configuration; trace layouts are padded
// for it so that one layout serves every configuration.
constexpr int kMaxTimeTile = 1024;

// ---------------------------------------------------------------------------
// Table (device view)
// ---------------------------------------------------------------------------
struct TableDev {
  int N, S, P, K, n_tiles;
  int4* src_info;    // [n_tiles * K]  {source index or -1, min delay, max delay, 0}
  int2* tile_hdr;    // [n_tiles]      {active stations, 0}
  int* st_s;         // [n_tiles * S]  station of active slot j
  int* st_lo;        // [n_tiles * S * P] window start (aligned)
  int* st_spread;    // [n_tiles * S * P] window span beyond the time tile
  void* meta;        // [n_tiles * S * K] MetaT<P>
  int* stats;        // [kStatCount]
  const int* perm;   // optional [n_tiles * K] source order (nullptr: identity)
  int index_base;    // added to every source index (a table over part of a grid)
};

enum : int {
  kStatMinDelay = 0,   // min delay over weighted terms
  kStatMaxDelay = 1,   // max delay over weighted terms
  kStatMaxSpread = 2,  // max window span (hi - lo_aligned)
  kStatMaxActive = 3,  // max active stations in a tile
  kStatNonFinite = 4,  // a non-zero weight is NaN or inf
  kStatMinLoAligned = 5,
  kStatWideTile = 6,   // a window span does not fit 16-bit offsets
  kStatCount = 8
};

// Per (tile, station, source) metadata: weight bits and 16-bit offsets.
template <int P> struct MetaT;
template <> struct MetaT<1> { using type = uint2; };  // {w, off0}
template <> struct MetaT<2> { using type = uint2; };  // {w, off0 | off1 << 16}
template <> struct MetaT<3> { using type = uint4; };  // {w, off0|off1<<16, off2, 0}
template <> struct MetaT<4> { using type = uint4; };  // {w, off0|off1<<16, off2|off3<<16, 0}

template <int P>
__host__ __device__ __forceinline__ int meta_off(const typename MetaT<P>::type& m, int p) {
  if constexpr (P <= 2) {
    return (p == 0) ? (int)(m.y & 0xFFFFu) : (int)(m.y >> 16);
  } else {
    const uint32_t v = (p < 2) ? m.y : m.z;
    return (p & 1) ? (int)(v >> 16) : (int)(v & 0xFFFFu);
  }
}

__host__ __device__ __forceinline__ int floor_align(int v) {
  return (v >= 0) ? (v / kAlign) * kAlign : -(((-v) + kAlign - 1) / kAlign) * kAlign;
}

// ---------------------------------------------------------------------------
// Table build: one block per source tile.
// Dynamic shared memory: 2 * S * P ints (per-station lo / hi) + S ints.
// ---------------------------------------------------------------------------
template <int P>
__global__ void table_build_kernel(const int32_t* __restrict__ delays,
                                   const float* __restrict__ weights, TableDev tb) {
  using M = typename MetaT<P>::type;
  extern __shared__ int sh[];
  const int S = tb.S, K = tb.K;
  int* lo = sh;               // [S * P]
  int* hi = lo + S * P;       // [S * P]
  int* slot = hi + S * P;     // [S] active slot of station s, or -1
  __shared__ int n_active_sh;
  const int tile = blockIdx.x;

  auto orig_of = [&](int k) -> int {
    const long long idx = (long long)tile * K + k;
    int o = tb.perm ? tb.perm[idx] : (int)idx;
    return (o >= 0 && o < tb.N) ? o : -1;
  };

  // 1. per source: min / max over weighted stations, non-finite weights.
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    const int o = orig_of(k);
    int mn = INT_MAX, mx = INT_MIN, bad = 0;
    if (o >= 0) {
      const int32_t* d = delays + (size_t)o * S * P;
      const float* w = weights + (size_t)o * S;
      for (int s = 0; s < S; ++s) {
        const float ws = w[s];
        if (ws == 0.0f) continue;
        if (!isfinite(ws)) bad = 1;
        for (int p = 0; p < P; ++p) {
          const int v = d[s * P + p];
          mn = min(mn, v);
          mx = max(mx, v);
        }
      }
    }
    tb.src_info[(size_t)tile * K + k] = make_int4(o >= 0 ? o + tb.index_base : o, mn, mx, 0);
    if (bad) atomicOr(&tb.stats[kStatNonFinite], 1);
  }
  // 2. per (station, phase): window over the tile's weighted sources.
  for (int sp = threadIdx.x; sp < S * P; sp += blockDim.x) {
    const int s = sp / P;
    int l = INT_MAX, h = INT_MIN;
    for (int k = 0; k < K; ++k) {
      const int o = orig_of(k);
      if (o < 0) continue;
      if (weights[(size_t)o * S + s] == 0.0f) continue;
      const int v = delays[(size_t)o * S * P + sp];
      l = min(l, v);
      h = max(h, v);
    }
    lo[sp] = l;
    hi[sp] = h;
  }
  __syncthreads();
  // 3. active station list, ascending station index (the summation order).
  if (threadIdx.x == 0) {
    int n = 0, spread_max = 0, mn = INT_MAX, mx = INT_MIN, lo_al_min = INT_MAX, wide = 0;
    for (int s = 0; s < S; ++s) {
      if (lo[s * P] > hi[s * P]) {  // no weighted source in this tile
        slot[s] = -1;
        continue;
      }
      slot[s] = n;
      tb.st_s[(size_t)tile * S + n] = s;
      for (int p = 0; p < P; ++p) {
        const int l = lo[s * P + p], h = hi[s * P + p];
        const int la = floor_align(l);
        const long long span = (long long)h - la;
        if (span > 0xFFFF) wide = 1;
        const int sp32 = (int)min(span, (long long)INT_MAX);
        tb.st_lo[((size_t)tile * S + n) * P + p] = la;
        tb.st_spread[((size_t)tile * S + n) * P + p] = sp32;
        spread_max = max(spread_max, sp32);
        mn = min(mn, l);
        mx = max(mx, h);
        lo_al_min = min(lo_al_min, la);
      }
      ++n;
    }
    n_active_sh = n;
    tb.tile_hdr[tile] = make_int2(n, 0);
    if (n > 0) {
      atomicMin(&tb.stats[kStatMinDelay], mn);
      atomicMax(&tb.stats[kStatMaxDelay], mx);
      atomicMin(&tb.stats[kStatMinLoAligned], lo_al_min);
    }
    atomicMax(&tb.stats[kStatMaxSpread], spread_max);
    atomicMax(&tb.stats[kStatMaxActive], n);
    if (wide) atomicOr(&tb.stats[kStatWideTile], 1);
  }
  __syncthreads();
  // 4. per (active station, source): weight and 16-bit offsets.
  const int n_active = n_active_sh;
  M* meta = reinterpret_cast<M*>(tb.meta) + (size_t)tile * S * K;
  for (int idx = threadIdx.x; idx < n_active * K; idx += blockDim.x) {
    const int j = idx / K, k = idx - j * K;
    const int s = tb.st_s[(size_t)tile * S + j];
    const int o = orig_of(k);
    float w = 0.0f;
    uint32_t off[4] = {0u, 0u, 0u, 0u};
    if (o >= 0) {
      w = weights[(size_t)o * S + s];
      if (w != 0.0f) {
        for (int p = 0; p < P; ++p) {
          const long long v = (long long)delays[(size_t)o * S * P + s * P + p] -
                              tb.st_lo[((size_t)tile * S + j) * P + p];
          off[p] = (uint32_t)min(v, 0xFFFFll);
        }
      }
    }
    M m;
    if constexpr (P <= 2) {
      m.x = __float_as_uint(w);
      m.y = off[0] | (off[1] << 16);
    } else {
      m.x = __float_as_uint(w);
      m.y = off[0] | (off[1] << 16);
      m.z = off[2] | (off[3] << 16);
      m.w = 0u;
    }
    meta[(size_t)j * K + k] = m;
  }
}

// ---------------------------------------------------------------------------
// Staged shift-and-stack kernel.
//
// Block = WS consumer warps + 1 producer warp, one source tile of
// K = WS * KS sources, a contiguous chunk of time tiles of TT = 32 * MT
// samples.  For every (time tile, group of SPS active stations) the producer
// copies the stations' P delay windows, [t0 + lo, t0 + lo + W), from HBM/L2
// into a shared-memory ring of NSTAGE stages with 1-D bulk copies (TMA
// engine, 16-byte aligned, completing on the stage's "full" mbarrier); 16-bit
// storage copies each window four times, shifted by one sample.  Consumer
// warp w owns sources w*KS .. w*KS+KS-1; with FP32 storage lane l owns samples
// t0 + l + 32*m, m < MT, so each warp-wide shared load reads 32 consecutive
// words (one conflict-free wavefront), and the per-(source, station) metadata
// is a broadcast.  FP32 accumulation: acc = acc + w * u, rounded multiply
// then rounded add, stations ascending, phases ascending (reference order).
// After the last station of a time tile: per sample the thread's best
// (value, source) over its KS sources, one packed key per sample, a max over
// the WS warps through shared memory, then one red.global.max.u64 per sample;
// or, for reduce='none', coalesced stores of the tile's beams.
// ---------------------------------------------------------------------------
// A travel-time table as the staged kernel reads it.
struct TableView {
  const int4* src_info;  // [n_tiles * K] {source index or -1, min delay, max delay, 0}
  const int2* tile_hdr;  // [n_tiles] {active stations, 0}
  const int* st_s;       // [n_tiles * S]
  const int* st_lo;      // [n_tiles * S * P]
  const int* st_spread;  // [n_tiles * S * P]
  const void* meta;      // [n_tiles * S * K]
  int S, n_tiles;
};

// One record: a waveform window, or a streamed chunk with its carried halo.
// Sample t of the record is global sample t_origin + t.  Traces hold samples
// [0, T) (zeros outside); results are produced for samples [out0, out1).
struct RecordView {
  const void* traces;   // FP32 rows, or 16-bit rows in kHalfCopies shifted copies
  const float* scales;  // per-station scale of 16-bit storage (unused for FP32)
  long long pitch;      // elements per row
  long long t_origin;   // global index of record sample 0 (strict lower bound)
  int lpad;
  int T;
  int out0, out1;
  int flexible;
  int table;                    // index into the launch's tables
  int tpc;                      // batch launch: time tiles per work item
  int n_chunks;                 // batch launch: work items per source tile
  const uint32_t* station_mask; // bit s set: station s used (nullptr: all)
  const int2* srcmm;            // per tile slot (min, max) over used stations, or nullptr
  unsigned long long* keys;     // [out1 - out0] packed keys (reduce='max')
  float* beam;                  // [N, ldb], column = sample - out0 (reduce='none')
  long long ldb;
  float* beam_max;              // batch launch: decoded outputs [out1 - out0]
  int32_t* argmax;
};

struct LaunchArgs {
  TableView tab0;               // plain launch: the table
  RecordView rec0;              // plain launch: the record
  const TableView* tables;      // batch launch: device arrays
  const RecordView* records;
  const long long* rec_prefix;  // batch launch: work items before record r, [n_records + 1]
  int n_records;
  unsigned long long* next_item;  // batch launch: work-queue head
  int tiles_per_chunk;          // plain launch: time tiles per block
  int rowcap;                   // elements per ring row (per version for 16-bit)
  int max_active;
  // Rows of the cross-warp max buffer (reduce='max'): WS, one per consumer
  // warp (plain stores, then a max over the rows), or 1, a row the warps max
  // into with shared-memory atomics -- the host takes 1 when the per-warp
  // rows would not leave room for the table's ring.
  int red_rows;
  int* status;
};

// Sources of a table tile (the tiling map groups sources by this many).  A
// kernel configuration covers a tile with one block (WS * KS == kTableTile)
// or splits it over kTableTile / (WS * KS) blocks.
constexpr int kTableTile = 64;

template <int P, int KS, int MT, int WS>
struct WindowCfg {
  static constexpr int K = WS * KS;
  static constexpr int TT = 32 * MT;
  static constexpr int kThreads = (WS + 1) * 32;
};

__host__ __device__ inline size_t align_up_sz(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Shared-memory carve-up, used identically by host (size) and device.  A
// ring row holds `rowcap` FP32 elements, or `rowcap` 16-bit elements of
// each of the kHalfCopies copies; a stage holds SPS stations x P rows.
template <int P, int KS, int MT, int WS, int NSTAGE, int SPS, bool MAXRED>
struct WindowSmem {
  using M = typename MetaT<P>::type;
  static constexpr int K = WS * KS;
  static constexpr int TT = 32 * MT;
  size_t ring, meta, red, srci, st_s, st_j, st_lo, st_w, st_sc, bars, misc, total;
  // row_factor: 32-bit words per ring row per sample of capacity
  // (ring_row_factor<STORAGE>()); red_rows: rows of the max buffer (WS or 1)
  __host__ __device__ WindowSmem(int rowcap, int max_active, int row_factor, int red_rows) {
    size_t o = 0;
    ring = o;        o += (size_t)NSTAGE * SPS * P * rowcap * 4 * row_factor;
    o = align_up_sz(o, 16);
    meta = o;        o += (size_t)max_active * K * sizeof(M);
    o = align_up_sz(o, 16);
    red = o;         o += MAXRED ? (size_t)red_rows * TT * sizeof(unsigned long long) : 0;
    o = align_up_sz(o, 16);
    srci = o;        o += (size_t)K * sizeof(int4);
    st_s = o;        o += (size_t)max_active * sizeof(int);
    st_j = o;        o += (size_t)max_active * sizeof(int);
    st_lo = o;       o += (size_t)max_active * P * sizeof(int);
    st_w = o;        o += (size_t)max_active * P * sizeof(int);
    st_sc = o;       o += (size_t)max_active * sizeof(float);
    o = align_up_sz(o, 16);
    bars = o;        o += (size_t)2 * NSTAGE * sizeof(uint64_t);
    o = align_up_sz(o, 16);    // the current item is an int4 at misc + 32
    misc = o;        o += 64;  // abort flag, active count, current item
    total = align_up_sz(o, 128);
  }
};

// Sample of accumulator half h of pair q for this lane, relative to t0.
// FP32: lane owns samples lane + 32 m (pair q = m 2q, 2q+1);
// 16-bit: lane owns runs of 4 samples 4 lane + 128 r (pairs q = 2r, 2r+1).
template <int STORAGE>
__device__ __forceinline__ int pair_sample(int lane, int q, int h) {
  if constexpr (STORAGE == BP_STORAGE_F32) return lane + 64 * q + 32 * h;
  else return 4 * lane + 128 * (q >> 1) + 2 * (q & 1) + h;
}

// ---- 16-bit arithmetic with FP32 accumulation --------------------------------
// Packed FP16 pair add, round to nearest (no multiply precedes it).
__device__ __forceinline__ uint32_t hadd2_rn(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("add.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}

// acc.{x,y} = round_f32(v.{lo,hi} * c.lo + acc.{x,y}) for FP16 v and c: the
// mixed-precision FMA (16-bit sources, FP32 addend and result, one
// rounding), which needs no widening of v.  The product of two FP16 values
// is exact in FP32, so each lane equals fmaf((float)v, (float)c, acc).
__device__ __forceinline__ void fma2_f32_f16(float2& acc, uint32_t v, uint32_t c) {
  asm("{\n\t.reg .b16 vl, vh, cl, ch;\n\t"
      "mov.b32 {vl, vh}, %2;\n\t"
      "mov.b32 {cl, ch}, %3;\n\t"
      "fma.rn.f32.f16 %0, vl, cl, %0;\n\t"
      "fma.rn.f32.f16 %1, vh, cl, %1;\n\t}"
      : "+f"(acc.x), "+f"(acc.y)
      : "r"(v), "r"(c));
}

// The same for BF16 v and c (the product of two BF16 values is exact too).
__device__ __forceinline__ void fma2_f32_bf16(float2& acc, uint32_t v, uint32_t c) {
  asm("{\n\t.reg .b16 vl, vh, cl, ch;\n\t"
      "mov.b32 {vl, vh}, %2;\n\t"
      "mov.b32 {cl, ch}, %3;\n\t"
      "fma.rn.f32.bf16 %0, vl, cl, %0;\n\t"
      "fma.rn.f32.bf16 %1, vh, cl, %1;\n\t}"
      : "+f"(acc.x), "+f"(acc.y)
      : "r"(v), "r"(c));
}

// The factor c = w * scale of one (source, station) as a pair of equal
// 16-bit values, when that is exact: c finite, a normal number of the
// storage format, and no mantissa bits beyond the format's.  Returns false
// otherwise (the kernel then keeps the FP32 factor for the whole item).
template <int STORAGE>
__device__ __forceinline__ bool pack_factor16(float c, uint32_t* packed) {
  if constexpr (STORAGE == BP_STORAGE_F16) {
    const float a = fabsf(c);
    if (!(a >= 6.103515625e-05f && a <= 65504.0f)) return false;  // normal FP16
    const __half h = __float2half_rn(c);
    if (__half2float(h) != c) return false;
    const uint32_t b = (uint32_t)__half_as_ushort(h);
    *packed = b | (b << 16);
    return true;
  } else {
    const float a = fabsf(c);
    if (!(a >= FLT_MIN && a <= FLT_MAX)) return false;  // normal, finite
    const uint32_t b = __float_as_uint(c);
    if (b & 0xFFFFu) return false;
    *packed = (b >> 16) | (b & 0xFFFF0000u);
    return true;
  }
}

// The staged shift-and-stack for one item (record, block tile, time tiles
// [tau0, tau1)), shared by the plain and the persistent kernels.  A block
// tile is one table tile (WS * KS == kTableTile) or a part of one: block
// tile b covers sources (b % H) * K .. + K - 1 of table tile b / H.  A ring
// stage carries SPS consecutive active stations (one mbarrier round trip per
// SPS stations).
template <int P, int KS, int MT, int WS, int NSTAGE, int SPS, bool MAXRED, bool CHECKED,
          int STORAGE>
struct Staged {
  static_assert(MT % 2 == 0 && KS % 2 == 0, "packed pairs");
  static_assert(!(CHECKED && STORAGE != BP_STORAGE_F32), "checked variant is FP32 only");
  using M = typename MetaT<P>::type;
  static constexpr bool F32 = STORAGE == BP_STORAGE_F32;
  static constexpr int K = WS * KS;   // sources per block
  static_assert(kTableTile % K == 0, "a block covers a whole part of a table tile");
  static constexpr int H = kTableTile / K;  // blocks per table tile
  static constexpr int TT = 32 * MT;
  static_assert(TT <= kMaxTimeTile, "time tile beyond the trace layout's padding");
  static constexpr int NCONS = WS * 32;
  static constexpr int ESZ = F32 ? 4 : 2;  // bytes per stored element
  static constexpr int NVER = F32 ? 1 : kHalfCopies;  // stored copies per row
  static constexpr int RF = ring_row_factor<STORAGE>();
  static_assert(F32 || MT % 4 == 0, "16-bit lanes own runs of 4 samples");
  // Samples per lane whose words are loaded before their arithmetic (the
  // whole lane up to 16; longer lanes in groups of 16, to bound registers).
  static constexpr int GS = MT > 16 ? 16 : MT;
  static_assert(MT % GS == 0, "whole groups");
  // 16-bit storage with at most 32 accumulators per thread: the words of both
  // sources of a metadata pair are loaded before either's arithmetic.
  static constexpr bool PAIRLOAD = !F32 && KS * MT <= 32 && MT == GS;
  // Who issues one stage's bulk copies (SPS stations x P phases x NVER row
  // copies): lane 0 alone, or one producer lane per (station, phase) row with
  // its NVER copies.  Rows in parallel pay for 16-bit storage with two
  // stations per stage (16 copies a stage at P = 2; 400k-source workload,
  // config 2 FP16 488 -> 420 ms, config 5 506 -> 445 ms); with one station
  // per stage, or FP32's P x SPS copies, lane 0 alone measured 1-7% faster.
  static constexpr int kIssueLane0 = 0, kIssueRow = 1;
  static constexpr int ISSUE = (!F32 && SPS > 1) ? kIssueRow : kIssueLane0;

  struct Smem {
    unsigned char* ring;
    M* meta_s;
    unsigned long long* red;
    int4* srci;
    int* st_s;
    int* st_j;
    int* st_lo;
    int* st_w;
    float* st_sc;
    uint64_t* full;
    uint64_t* empty;
    volatile int* abort_flag;
    int* n_act;
    int4* cur_item;
    int red_rows;
  };

  __device__ static Smem carve(unsigned char* smem, int rowcap, int max_active, int red_rows) {
    const WindowSmem<P, KS, MT, WS, NSTAGE, SPS, MAXRED> L(rowcap, max_active, RF, red_rows);
    Smem s;
    s.red_rows = red_rows;
    s.ring = smem + L.ring;
    s.meta_s = reinterpret_cast<M*>(smem + L.meta);
    s.red = reinterpret_cast<unsigned long long*>(smem + L.red);
    s.srci = reinterpret_cast<int4*>(smem + L.srci);
    s.st_s = reinterpret_cast<int*>(smem + L.st_s);
    s.st_j = reinterpret_cast<int*>(smem + L.st_j);
    s.st_lo = reinterpret_cast<int*>(smem + L.st_lo);
    s.st_w = reinterpret_cast<int*>(smem + L.st_w);
    s.st_sc = reinterpret_cast<float*>(smem + L.st_sc);
    s.full = reinterpret_cast<uint64_t*>(smem + L.bars);
    s.empty = s.full + NSTAGE;
    s.abort_flag = reinterpret_cast<volatile int*>(smem + L.misc);
    s.n_act = reinterpret_cast<int*>(smem + L.misc + 16);
    s.cur_item = reinterpret_cast<int4*>(smem + L.misc + 32);
    return s;
  }

  // thread 0, once per block
  __device__ static void init_barriers(const Smem& sm) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], WS);
    }
    *sm.abort_flag = 0;
    fence_mbar_init();
  }

  // All threads.  Ends after the item's last epilogue; the caller puts a
  // __syncthreads() between items.  `it0` is the block's stage counter
  // before the item; returns the number of stages the item used.
  __device__ static int run_item(const Smem& sm, const TableView& tb, const RecordView& rc,
                                 int btile, int tau0, int tau1, int rowcap, int* status,
                                 int it0) {
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int row_words = rowcap * RF;  // one ring row (all copies) in 32-bit words
    const int tile = btile / H;         // table tile
    const int k0 = (btile - tile * H) * K;  // first source slot of this block in the tile

    // ---- prologue: the tile's stations (those the record uses) ----------
    if (warp == 0) {
      const int n_tab = tb.tile_hdr[tile].x;
      int n = 0;
      for (int j0 = 0; j0 < n_tab; j0 += 32) {
        const int j = j0 + lane;
        int s = -1;
        bool use = false;
        if (j < n_tab) {
          s = tb.st_s[(size_t)tile * tb.S + j];
          use = !rc.station_mask || ((rc.station_mask[s >> 5] >> (s & 31)) & 1u);
        }
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, use);
        if (use) sm.st_j[n + __popc(bal & ((1u << lane) - 1u))] = j;  // table slot
        n += __popc(bal);
      }
      if (lane == 0) *sm.n_act = n;
    }
    __syncthreads();
    const int n_active = *sm.n_act;
    // per active station: station index, scale, window starts and widths
    for (int i = tid; i < n_active; i += blockDim.x) {
      const int j = sm.st_j[i];
      const int s = tb.st_s[(size_t)tile * tb.S + j];
      sm.st_s[i] = s;
      sm.st_sc[i] = F32 ? 1.0f : rc.scales[s];
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const size_t g = ((size_t)tile * tb.S + j) * P + p;
        sm.st_lo[i * P + p] = tb.st_lo[g];
        const int w = (int)align_up_sz((size_t)(TT + tb.st_spread[g] + 1), kAlign);
        sm.st_w[i * P + p] = w;
        if (w > rowcap) atomicOr(status, kStatusBadWindow);
      }
    }
    if (MAXRED && sm.red_rows == 1)
      for (int i = tid; i < TT; i += blockDim.x) sm.red[i] = 0ull;
    {
      // Per source slot: {source, first, end, 0} with [first, end) the
      // record-local samples the out-of-bounds rule keeps (strict: every
      // delay of the source inside the record, the lower bound in global
      // time); empty for an unused slot.  Bounds are clamped to +-2^30,
      // beyond any sample index of a record.
      constexpr long long kFar = 1ll << 30;
      for (int i = tid; i < K; i += blockDim.x) {
        const size_t slot = (size_t)tile * kTableTile + k0 + i;
        int4 si = tb.src_info[slot];
        if (rc.srcmm) {
          const int2 mm = rc.srcmm[slot];
          si.y = mm.x;
          si.z = mm.y;
        }
        long long first = -kFar, end = kFar;
        if (si.x < 0 || (!rc.flexible && si.y > si.z)) {
          first = kFar;
          end = -kFar;
        } else if (!rc.flexible) {
          first = min(max(-rc.t_origin - (long long)si.y, -kFar), kFar);
          end = min(max((long long)rc.T - (long long)si.z, -kFar), kFar);
        }
        sm.srci[i] = make_int4(si.x, (int)first, (int)end, 0);
      }
    }
    __syncthreads();
    // Per (active station, source): weight and offsets.  16-bit storage: each
    // sample offset becomes the byte offset in the ring row of the copy that
    // starts the run on an 8-byte boundary: 4 (2 (off >> 2) + (off & 3) *
    // rowcap / 2) (copy v starts v * rowcap / 2 words into the row; the host
    // keeps 8 rowcap below 2^16); and when every factor c = w * scale of the item is exact in the
    // 16-bit format, the weight word becomes c packed twice (0 for a zero
    // weight) and the item runs the mixed-precision arithmetic.
    bool fast16 = false;
    {
      const M* gm = reinterpret_cast<const M*>(tb.meta) + (size_t)tile * tb.S * kTableTile;
      const uint32_t copy_words = (uint32_t)rowcap >> 1;  // one 16-bit copy, in words
      int exact = 1;
      for (int i = tid; i < n_active * K; i += blockDim.x) {
        const int jj = i / K, k = i - jj * K;
        M m = gm[(size_t)sm.st_j[jj] * kTableTile + k0 + k];
        if constexpr (!F32) {
          auto wo = [&](uint32_t v) {
            const uint32_t lo = v & 0xFFFFu, hi = v >> 16;
            return (4 * (2 * (lo >> 2) + (lo & 3u) * copy_words)) |
                   ((4 * (2 * (hi >> 2) + (hi & 3u) * copy_words)) << 16);
          };
          m.y = wo(m.y);
          if constexpr (P > 2) m.z = wo(m.z);
          const float w = __uint_as_float(m.x);
          uint32_t pk;
          if (w != 0.0f && !pack_factor16<STORAGE>(w * sm.st_sc[jj], &pk)) exact = 0;
        }
        sm.meta_s[i] = m;
      }
      if constexpr (F32) {
        __syncthreads();
      } else {
        fast16 = __syncthreads_and(exact) != 0;
        if (fast16) {
          for (int i = tid; i < n_active * K; i += blockDim.x) {
            const int jj = i / K;
            const float w = __uint_as_float(sm.meta_s[i].x);
            uint32_t pk = 0u;
            if (w != 0.0f) pack_factor16<STORAGE>(w * sm.st_sc[jj], &pk);
            sm.meta_s[i].x = pk;
          }
          __syncthreads();
        }
      }
    }

    const int n_grp = (n_active + SPS - 1) / SPS;  // stages per time tile
    const int n_stages = (tau1 - tau0) * n_grp;

    // ---- producer warp ----------------------------------------------------
    // Lane 0 waits for the stage to drain and arms its full barrier with the
    // stage's byte count; the stage's copies are then issued as ISSUE says.
    if (warp == WS) {
      if (ISSUE == kIssueLane0 && lane != 0) return n_stages;
      const unsigned char* tr = reinterpret_cast<const unsigned char*>(rc.traces);
      int issued = 0;
      for (int r = 0; r < n_stages; ++r) {
        const int it = it0 + r;
        const int stage = it % NSTAGE;
        int ok = 1;
        if (lane == 0 && it >= NSTAGE)
          ok = mbar_wait_bounded(&sm.empty[stage], ((it / NSTAGE) - 1) & 1, sm.abort_flag,
                                 status) ? 1 : 0;
        if constexpr (ISSUE != kIssueLane0) {
          if (!__shfl_sync(0xFFFFFFFFu, ok, 0)) break;
          // every issuing lane observes the drained phase itself before its
          // copies overwrite the stage (the phase has completed: no wait)
          if (it >= NSTAGE) (void)mbar_try_wait(&sm.empty[stage], ((it / NSTAGE) - 1) & 1);
        } else {
          if (!ok) break;
        }
        const int tau = tau0 + r / n_grp;
        const int j0 = (r - (r / n_grp) * n_grp) * SPS;
        const int nj = min(SPS, n_active - j0);
        const int t0 = tau * TT;
        // copy (jj, p, v) reads trace row (s P + p) NVER + v, columns [col, col + w)
        auto copy_ok = [&](int j, int p) -> bool {
#if BP_DEBUG_CHECKS
          const int s = sm.st_s[j];
          const int w = min(sm.st_w[j * P + p], rowcap);
          const long long col = (long long)rc.lpad + t0 + sm.st_lo[j * P + p];
          return s >= 0 && s < tb.S && w > 0 && col >= 0 && col + w <= rc.pitch &&
                 (col * ESZ) % 16 == 0 && ((long long)w * ESZ) % 16 == 0;
#else
          (void)j;
          (void)p;
          return true;
#endif
        };
        if (lane == 0) {
          uint32_t bytes = 0;
#pragma unroll
          for (int jj = 0; jj < SPS; ++jj) {
            if (jj >= nj) break;
#pragma unroll
            for (int p = 0; p < P; ++p)
              if (copy_ok(j0 + jj, p))
                bytes += (uint32_t)min(sm.st_w[(j0 + jj) * P + p], rowcap) * ESZ * NVER;
              else
                atomicOr(status, kStatusBadIndex);
          }
          mbar_arrive_expect_tx(&sm.full[stage], bytes);
        }
        if constexpr (ISSUE != kIssueLane0) __syncwarp();
        // Row (jj, p): station slot j0 + jj, phase p; its NVER copies go to
        // consecutive ring rows.  The row's index, width and offset are read
        // once: every bulk copy's memory clobber would reload them.
        struct RowSpan {
          unsigned char* dst;
          const unsigned char* src;
          uint32_t bytes;
        };
        auto row_span = [&](int jj, int p) -> RowSpan {
          const int j = j0 + jj;
          const int s = sm.st_s[j];
          const int w = min(sm.st_w[j * P + p], rowcap);
          const long long col = (long long)rc.lpad + t0 + sm.st_lo[j * P + p];
          const size_t row0 = (size_t)(s * P + p) * NVER;
          return {sm.ring + ((size_t)((stage * SPS + jj) * P + p) * row_words) * 4,
                  tr + (row0 * rc.pitch + col) * ESZ, (uint32_t)w * ESZ};
        };
        auto issue = [&](const RowSpan& r, int v) {
          bulk_g2s(r.dst + (size_t)v * rowcap * ESZ, r.src + (size_t)v * rc.pitch * ESZ, r.bytes,
                   &sm.full[stage]);
        };
        if constexpr (ISSUE == kIssueLane0) {
#pragma unroll
          for (int jj = 0; jj < SPS; ++jj) {
            if (jj >= nj) break;
#pragma unroll
            for (int p = 0; p < P; ++p) {
              if (!copy_ok(j0 + jj, p)) continue;
              const RowSpan r = row_span(jj, p);
#pragma unroll
              for (int v = 0; v < NVER; ++v) issue(r, v);
            }
          }
        } else {
          for (int q = lane; q < nj * P; q += 32) {
            const int jj = q / P;
            const int p = q - jj * P;
            if (!copy_ok(j0 + jj, p)) continue;
            const RowSpan r = row_span(jj, p);
#pragma unroll
            for (int v = 0; v < NVER; ++v) issue(r, v);
          }
        }
        ++issued;
      }
      if (lane == 0 && *sm.abort_flag) {
        // Let every copy already issued land before the block moves on.
        volatile int never = 0;
        for (int r = max(0, issued - NSTAGE); r < issued; ++r) {
          const int it = it0 + r;
          mbar_wait_bounded(&sm.full[it % NSTAGE], (it / NSTAGE) & 1, &never, nullptr);
        }
      }
      return n_stages;
    }

    // ---- consumer warps ---------------------------------------------------
    if constexpr (F32) {
      consume<false>(sm, rc, tau0, tau1, n_active, n_grp, rowcap, status, it0);
    } else {
      if (fast16) consume<true>(sm, rc, tau0, tau1, n_active, n_grp, rowcap, status, it0);
      else consume<false>(sm, rc, tau0, tau1, n_active, n_grp, rowcap, status, it0);
    }
    return n_stages;
  }

  // The consumer warps' part of an item: for every time tile, the stages'
  // stations into the accumulators, then the epilogue.  FAST16: the item's
  // weight words hold packed 16-bit factors (block-uniform choice).
  template <bool FAST16>
  __device__ static void consume(const Smem& sm, const RecordView& rc, int tau0, int tau1,
                                 int n_active, int n_grp, int rowcap, int* status, int it0) {
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int row_words = rowcap * RF;
    const int4* my_src = sm.srci + warp * KS;
    int it = it0;
    for (int tau = tau0; tau < tau1; ++tau) {
      float2 acc[KS][MT / 2];  // pair q, half h: sample pair_sample(lane, q, h)
#pragma unroll
      for (int k = 0; k < KS; ++k)
#pragma unroll
        for (int m = 0; m < MT / 2; ++m) acc[k][m] = make_float2(0.0f, 0.0f);
      const int t0 = tau * TT;

      for (int g = 0; g < n_grp; ++g, ++it) {
        const int stage = it % NSTAGE;
        mbar_wait_bounded(&sm.full[stage], (it / NSTAGE) & 1, sm.abort_flag, status);
#pragma unroll
        for (int jj = 0; jj < SPS; ++jj) {
          const int j = g * SPS + jj;
          if (j >= n_active) break;
          // station base in 32-bit words; row p at + p * row_words words
          const int sbase = (stage * SPS + jj) * P * row_words;
          const M* mrow = sm.meta_s + (size_t)j * K + warp * KS;
          station<FAST16>(sm, rc, mrow, sbase, row_words, sm.st_sc[j], j, t0, lane, rowcap,
                          status, acc);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.empty[stage]);
      }

      // ---- epilogue of the time tile ----
      if constexpr (MAXRED) {
        // Per sample, the thread's best (value, source) over its KS slots.
        // The table orders each tile's slots by source index, so ascending
        // slots are ascending sources and a strict `>` keeps the lowest
        // index among equal maxima; seeding with -FLT_MAX makes NaN and
        // -FLT_MAX (and below) lose, as in the reference's running max.
        // Samples outer, so that each pair's accumulators die after use.
        const bool one_row = sm.red_rows == 1;  // block-uniform
        // the key of sample (q, h) into this warp's row of the max buffer, or
        // into the single shared row (zero on entry) by an atomic max
        auto put = [&](int q, int h, float bv, int bi) {
          const int i = pair_sample<STORAGE>(lane, q, h);
          const unsigned long long key = bi >= 0 ? make_key(bv, bi) : 0ull;
          if (!one_row) sm.red[warp * TT + i] = key;
          else if (key) atomicMax(&sm.red[i], key);
        };
        bool all_kept = true;  // warp-uniform: every slot keeps the whole tile
#pragma unroll
        for (int k = 0; k < KS; ++k)
          all_kept = all_kept && my_src[k].y <= t0 && t0 + TT <= my_src[k].z;
        if (all_kept) {
#pragma unroll
          for (int q = 0; q < MT / 2; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              float bv = -FLT_MAX;
              int bi = -1;
#pragma unroll
              for (int k = 0; k < KS; ++k) {
                const float v = h ? acc[k][q].y : acc[k][q].x;
                if (v > bv) {
                  bv = v;
                  bi = my_src[k].x;
                }
              }
              put(q, h, bv, bi);
            }
        } else {
#pragma unroll
          for (int q = 0; q < MT / 2; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int t = t0 + pair_sample<STORAGE>(lane, q, h);
              float bv = -FLT_MAX;
              int bi = -1;
#pragma unroll
              for (int k = 0; k < KS; ++k) {
                const int4 si = my_src[k];
                if (t < si.y || t >= si.z) continue;  // outside the kept samples (or no source)
                const float v = h ? acc[k][q].y : acc[k][q].x;
                if (v > bv) {
                  bv = v;
                  bi = si.x;
                }
              }
              put(q, h, bv, bi);
            }
        }
        named_barrier_sync(1, NCONS);
        for (int i = tid; i < TT; i += NCONS) {
          unsigned long long b = 0ull;
          if (one_row) {
            b = sm.red[i];
            sm.red[i] = 0ull;  // zero again for the next tile
          } else {
#pragma unroll
            for (int w = 0; w < WS; ++w) {
              const unsigned long long v = sm.red[w * TT + i];
              b = v > b ? v : b;
            }
          }
          const int t = t0 + i;
          if (b != 0ull && t >= rc.out0 && t < rc.out1) red_max_u64(&rc.keys[t - rc.out0], b);
        }
        named_barrier_sync(1, NCONS);
      } else {
#pragma unroll
        for (int k = 0; k < KS; ++k) {
          const int4 si = my_src[k];
          if (si.x < 0) continue;
          float* row = rc.beam + (size_t)si.x * rc.ldb - rc.out0;
#pragma unroll
          for (int q = 0; q < MT / 2; ++q) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int t = t0 + pair_sample<STORAGE>(lane, q, h);
              if (t < rc.out0 || t >= rc.out1) continue;
              if (t >= si.y && t < si.z) row[t] = h ? acc[k][q].y : acc[k][q].x;
            }
          }
        }
      }
    }
  }

  // 16-bit storage: a weight word that skips its (source, station).
  template <bool FAST16>
  __device__ static __forceinline__ bool skip16(const M& m) {
    return FAST16 ? (m.x == 0u) : (__uint_as_float(m.x) == 0.0f);
  }

  // 16-bit storage: the words of sample group g0 (runs g0 .. g0 + GS/4 - 1 of
  // 4 samples) of every phase for one (source, station).  Each run is one
  // 64-bit load from the copy that starts it on an 8-byte boundary (byte
  // offsets prepared in the prologue).
  __device__ static __forceinline__ void load16(const Smem& sm, const M& m, int sbase,
                                                int row_words, int lane, int g0, int j,
                                                int rowcap, int* status,
                                                uint32_t (&wd)[P][GS / 2]) {
    (void)j;
    (void)rowcap;
    (void)status;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const uint2* src = reinterpret_cast<const uint2*>(
                             sm.ring + (size_t)(sbase + p * row_words) * 4 + meta_off<P>(m, p)) +
                         lane;
#pragma unroll
      for (int rr = 0; rr < GS / 4; ++rr) {
        const int r = g0 + rr;
#if BP_DEBUG_CHECKS
        {  // the 4 samples of this load inside its copy's window
          const int copy_words = rowcap >> 1;
          const int wi = meta_off<P>(m, p) / 4 + 2 * lane + 64 * r;
          const int cv = wi / copy_words, pos = 2 * (wi - cv * copy_words);
          if (cv >= NVER || pos + 3 >= min(sm.st_w[j * P + p], rowcap)) {
            atomicOr(status, kStatusBadIndex);
            wd[p][2 * rr] = wd[p][2 * rr + 1] = 0u;
            continue;
          }
        }
#endif
        const uint2 v = src[32 * r];  // samples 4 lane + 128 r + 0..3
        wd[p][2 * rr] = v.x;
        wd[p][2 * rr + 1] = v.y;
      }
    }
  }

  // 16-bit storage: acc += c * (phase sum) for the pairs of sample group g0.
  template <bool FAST16>
  __device__ static __forceinline__ void arith16(const M& m, float scale, int g0,
                                                 const uint32_t (&wd)[P][GS / 2],
                                                 float2 (&acc)[MT / 2]) {
    const float c = FAST16 ? 0.0f : __uint_as_float(m.x) * scale;
    const float2 c2 = make_float2(c, c);
    (void)c2;
#pragma unroll
    for (int qq = 0; qq < GS / 2; ++qq) {
      const int q = 2 * g0 + qq;
      if constexpr (STORAGE == BP_STORAGE_F16) {
        // phases summed in FP16 pairs (one extra FP16 rounding of a sum of
        // values in [-P, P])
        uint32_t hs = wd[0][qq];
#pragma unroll
        for (int p = 1; p < P; ++p) hs = hadd2_rn(hs, wd[p][qq]);
        if constexpr (FAST16) {
          fma2_f32_f16(acc[q], hs, m.x);
        } else {
          __half2 hh;
          memcpy(&hh, &hs, 4);
          acc[q] = __ffma2_rn(c2, __half22float2(hh), acc[q]);
        }
      } else {
        // BF16: one FMA per phase and sample, phases ascending
#pragma unroll
        for (int p = 0; p < P; ++p) {
          if constexpr (FAST16) {
            fma2_f32_bf16(acc[q], wd[p][qq], m.x);
          } else {
            const float2 u = make_float2(__uint_as_float(wd[p][qq] << 16),
                                         __uint_as_float(wd[p][qq] & 0xFFFF0000u));
            acc[q] = __ffma2_rn(c2, u, acc[q]);
          }
        }
      }
    }
  }

  // One active station j of the current stage for this warp's KS sources:
  // acc[k][.] += w_k * (sum over phases of the station's shifted samples).
  // FAST16 (16-bit storage, block-uniform): the weight words hold the packed
  // 16-bit factors c = w * scale (see the prologue).
  template <bool FAST16>
  __device__ static __forceinline__ void station(const Smem& sm, const RecordView& rc,
                                                 const M* mrow, int sbase, int row_words,
                                                 float scale, int j, int t0, int lane,
                                                 int rowcap, int* status,
                                                 float2 (&acc)[KS][MT / 2]) {
    (void)rc;
    (void)j;
    (void)t0;
    (void)rowcap;
    (void)status;
    (void)scale;
#pragma unroll
    for (int k2 = 0; k2 < KS; k2 += 2) {
      M mm2[2];
      if constexpr (P <= 2) {
        // two sources' records in one 128-bit broadcast
        const uint4 q4 = *reinterpret_cast<const uint4*>(mrow + k2);
        mm2[0] = make_uint2(q4.x, q4.y);
        mm2[1] = make_uint2(q4.z, q4.w);
      } else {
        mm2[0] = mrow[k2];
        mm2[1] = mrow[k2 + 1];
      }
      if constexpr (!F32 && PAIRLOAD) {
        // both sources' words first, then both sources' arithmetic: two
        // independent load batches in flight per warp
        uint32_t wd0[P][GS / 2], wd1[P][GS / 2];
        const bool u0 = !skip16<FAST16>(mm2[0]), u1 = !skip16<FAST16>(mm2[1]);
        if (u0) load16(sm, mm2[0], sbase, row_words, lane, 0, j, rowcap, status, wd0);
        if (u1) load16(sm, mm2[1], sbase, row_words, lane, 0, j, rowcap, status, wd1);
        if (u0) arith16<FAST16>(mm2[0], scale, 0, wd0, acc[k2]);
        if (u1) arith16<FAST16>(mm2[1], scale, 0, wd1, acc[k2 + 1]);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k = k2 + h;
        const M m = mm2[h];
        if constexpr (!F32) {
          // FAST16: m.x is the packed 16-bit factor c (0: skipped station);
          // otherwise m.x is the FP32 weight and c = w * scale (exact: scale
          // is 2^k).  Both give the same value per sample: c times the phase
          // sum (FP16: summed in half2 first; BF16: one product per phase)
          // added to the FP32 accumulator with one rounding per product.
          if constexpr (PAIRLOAD) continue;  // done above for the pair
          if (skip16<FAST16>(m)) continue;  // warp-uniform
#pragma unroll
          for (int g0 = 0; g0 < MT / 4; g0 += GS / 4) {
            uint32_t wd[P][GS / 2];  // the group's words first
            load16(sm, m, sbase, row_words, lane, g0, j, rowcap, status, wd);
            arith16<FAST16>(m, scale, g0, wd, acc[k]);
          }
        } else if constexpr (CHECKED) {
          const float w = __uint_as_float(m.x);
          if (w == 0.0f) continue;  // warp-uniform: skipped station
#pragma unroll
          for (int p = 0; p < P; ++p) {
            const int off = meta_off<P>(m, p);
            const float* src = reinterpret_cast<const float*>(sm.ring) + sbase +
                               p * row_words + off + lane;
            const long long tb0 = (long long)t0 + lane + sm.st_lo[j * P + p] + off;
#pragma unroll
            for (int mm = 0; mm < MT; ++mm) {
              const long long tt = tb0 + 32 * mm;
              if (tt < 0 || tt >= rc.T) continue;
#if BP_DEBUG_CHECKS
              if (off + lane + 32 * mm >= min(sm.st_w[j * P + p], rowcap)) {
                atomicOr(status, kStatusBadIndex);
                continue;
              }
#endif
              const float v = __fadd_rn((mm & 1) ? acc[k][mm >> 1].y : acc[k][mm >> 1].x,
                                        __fmul_rn(w, src[mm * 32]));
              if (mm & 1) acc[k][mm >> 1].y = v; else acc[k][mm >> 1].x = v;
            }
          }
        } else {
          const float w = __uint_as_float(m.x);
          if (w == 0.0f) continue;  // warp-uniform: skipped station
          // All of this source's words of a group first, then the arithmetic:
          // the loads of one (source, station) are independent, and issuing
          // them together keeps P * GS shared-memory loads in flight.
          const float* sbf = reinterpret_cast<const float*>(sm.ring) + sbase + lane;
#pragma unroll
          for (int g0 = 0; g0 < MT; g0 += GS) {
            float u[P][GS];
#pragma unroll
            for (int p = 0; p < P; ++p) {
              const float* src = sbf + p * row_words + meta_off<P>(m, p);
#pragma unroll
              for (int mm = 0; mm < GS; ++mm) {
#if BP_DEBUG_CHECKS
                if (meta_off<P>(m, p) + lane + 32 * (g0 + mm) >=
                    min(sm.st_w[j * P + p], rowcap)) {
                  atomicOr(status, kStatusBadIndex);
                  u[p][mm] = 0.0f;
                  continue;
                }
#endif
                u[p][mm] = src[32 * (g0 + mm)];
              }
            }
            if (w == 1.0f) {  // warp-uniform: 1 * u == u exactly, skip the multiply
#pragma unroll
              for (int p = 0; p < P; ++p)
#pragma unroll
                for (int qq = 0; qq < GS / 2; ++qq) {
                  const int q = g0 / 2 + qq;
                  acc[k][q] = add2_rn(acc[k][q], make_float2(u[p][2 * qq], u[p][2 * qq + 1]));
                }
            } else {
              // Scalar rounded multiply then rounded add: a packed multiply
              // followed by a packed add can be fused downstream, which would
              // change the last bit against the reference.
#pragma unroll
              for (int p = 0; p < P; ++p)
#pragma unroll
                for (int qq = 0; qq < GS / 2; ++qq) {
                  const int q = g0 / 2 + qq;
                  acc[k][q].x = __fadd_rn(acc[k][q].x, __fmul_rn(w, u[p][2 * qq]));
                  acc[k][q].y = __fadd_rn(acc[k][q].y, __fmul_rn(w, u[p][2 * qq + 1]));
                }
            }
          }
        }
      }
    }
  }
};

// Plain launch: one record, block = (block tile, chunk of time tiles),
// time-chunk major so that the blocks in flight share an L2-resident stretch
// of trace.
template <int P, int KS, int MT, int WS, int NSTAGE, int SPS, int MINB, bool MAXRED,
          bool CHECKED, int STORAGE>
__global__ void __launch_bounds__((WS + 1) * 32, MINB)
beam_window_kernel(const LaunchArgs a) {
  using St = Staged<P, KS, MT, WS, NSTAGE, SPS, MAXRED, CHECKED, STORAGE>;
  extern __shared__ __align__(128) unsigned char smem[];
  const typename St::Smem sm = St::carve(smem, a.rowcap, a.max_active, a.red_rows);
  if (threadIdx.x == 0) St::init_barriers(sm);
  __syncthreads();
  const int n_btiles = a.tab0.n_tiles * St::H;
  const int btile = blockIdx.x % n_btiles;
  const int chunk = blockIdx.x / n_btiles;
  const int tau_first = a.rec0.out0 / St::TT;
  const int tau_end = (a.rec0.out1 + St::TT - 1) / St::TT;
  const int tau0 = tau_first + chunk * a.tiles_per_chunk;
  const int tau1 = min(tau0 + a.tiles_per_chunk, tau_end);
  St::run_item(sm, a.tab0, a.rec0, btile, tau0, tau1, a.rowcap, a.status, 0);
}

// Persistent launch: a fixed grid whose blocks pop work items from a device
// queue until it is empty.  The queue is a counter over the items of all
// records (record r owns items rec_prefix[r] .. rec_prefix[r + 1] - 1, each a
// block tile x a chunk of r.tpc time tiles, time-chunk major).  Records may
// differ in length, station subset and table; storage, phases and reduce are
// the launch's.
template <int P, int KS, int MT, int WS, int NSTAGE, int SPS, int MINB, bool MAXRED,
          bool CHECKED, int STORAGE>
__global__ void __launch_bounds__((WS + 1) * 32, MINB)
beam_batch_kernel(const LaunchArgs a) {
  using St = Staged<P, KS, MT, WS, NSTAGE, SPS, MAXRED, CHECKED, STORAGE>;
  extern __shared__ __align__(128) unsigned char smem[];
  const typename St::Smem sm = St::carve(smem, a.rowcap, a.max_active, a.red_rows);
  if (threadIdx.x == 0) St::init_barriers(sm);
  __syncthreads();
  int it = 0;
  const long long n_items = a.rec_prefix[a.n_records];
  while (true) {
    if (threadIdx.x == 0) {
      const long long i = (long long)atomicAdd(a.next_item, 1ull);
      int4 cur = make_int4(-1, 0, 0, 0);
      if (i < n_items) {
        // record r: rec_prefix[r] <= i < rec_prefix[r + 1]
        int lo = 0, hi = a.n_records - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (a.rec_prefix[mid] <= i) lo = mid; else hi = mid - 1;
        }
        const RecordView& r = a.records[lo];
        const int n_btiles = a.tables[r.table].n_tiles * St::H;
        const long long local = i - a.rec_prefix[lo];
        const int chunk = (int)(local / n_btiles);
        const int btile = (int)(local - (long long)chunk * n_btiles);
        const int tau_first = r.out0 / St::TT;
        const int tau_end = (r.out1 + St::TT - 1) / St::TT;
        const int tau0 = tau_first + chunk * r.tpc;
        cur = make_int4(lo, btile, tau0, min(tau0 + r.tpc, tau_end));
      }
      *sm.cur_item = cur;
    }
    __syncthreads();
    const int4 item = *sm.cur_item;
    if (item.x < 0) break;
    const RecordView rc = a.records[item.x];
    const TableView tb = a.tables[rc.table];
    it += St::run_item(sm, tb, rc, item.y, item.z, item.w, a.rowcap, a.status, it);
    __syncthreads();
    if (*sm.abort_flag) break;
  }
}

// Everything below holds non-template kernels (one definition per program):
// translation units other than bp_capi.cu define BP_TEMPLATE_KERNELS_ONLY and
// leave it out.
#ifndef BP_TEMPLATE_KERNELS_ONLY

// Decode every record's keys of a batch into its outputs.
__global__ void batch_decode_kernel(const RecordView* __restrict__ recs) {
  const RecordView& r = recs[blockIdx.y];
  const int n = r.out1 - r.out0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const unsigned long long k = r.keys[t];
    if (k != 0ull) {
      r.beam_max[t] = key_value(k);
      r.argmax[t] = key_source(k);
    } else {
      r.argmax[t] = 0;
    }
  }
}

// Per tile slot (min, max) delay over the stations a record uses (weighted
// and in its station mask), from the table itself: d = lo + offset.
template <int P>
__global__ void masked_minmax_kernel(TableView tb, int K, const uint32_t* __restrict__ mask,
                                     int2* __restrict__ out) {
  using M = typename MetaT<P>::type;
  const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= (long long)tb.n_tiles * K) return;
  const int tile = (int)(slot / K), k = (int)(slot - (long long)tile * K);
  const int n_act = tb.tile_hdr[tile].x;
  const M* meta = reinterpret_cast<const M*>(tb.meta) + (size_t)tile * tb.S * K;
  int mn = INT_MAX, mx = INT_MIN;
  for (int j = 0; j < n_act; ++j) {
    const int s = tb.st_s[(size_t)tile * tb.S + j];
    if (mask && !((mask[s >> 5] >> (s & 31)) & 1u)) continue;
    const M m = meta[(size_t)j * K + k];
    if (__uint_as_float(m.x) == 0.0f) continue;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const int d = tb.st_lo[((size_t)tile * tb.S + j) * P + p] + meta_off<P>(m, p);
      mn = min(mn, d);
      mx = max(mx, d);
    }
  }
  out[slot] = make_int2(mn, mx);
}

// ---------------------------------------------------------------------------
// Storage element loads (direct kernel).
// ---------------------------------------------------------------------------
template <int STORAGE>
__device__ __forceinline__ float load_trace(const void* base, size_t idx) {
  if constexpr (STORAGE == BP_STORAGE_F32) {
    return __ldg(reinterpret_cast<const float*>(base) + idx);
  } else if constexpr (STORAGE == BP_STORAGE_BF16) {
    return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(base)[idx]);
  } else {
    return __half2float(reinterpret_cast<const __half*>(base)[idx]);
  }
}

// ---------------------------------------------------------------------------
// Direct kernel: no staging, any P, any delay spread.  Block = 256 samples x
// a group of sources; thread = one sample, sources looped in order.  Reads
// the traces through L1 (coalesced along t).  Terms whose sample falls
// outside [0, T) are skipped, which is the flexible rule and, for samples
// the strict rule keeps, never happens.
// ---------------------------------------------------------------------------
struct DirectArgs {
  const void* traces;
  const float* scales;
  long long pitch;
  int lpad;
  int T, N, S, P;
  int flexible;
  int src_per_block;
  const int32_t* delays;
  const float* weights;
  const int32_t* minmax;   // (N, 2)
  int index_base;          // added to the source index of every key
  unsigned long long* keys;
  float* beam;
  long long ldb;
};

template <int STORAGE, bool MAXRED>
__global__ void __launch_bounds__(256) beam_direct_kernel(const DirectArgs a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * a.src_per_block;
  const int i1 = min(i0 + a.src_per_block, a.N);
  unsigned long long best = 0ull;
  for (int i = i0; i < i1; ++i) {
    const int mn = a.minmax[2 * i], mx = a.minmax[2 * i + 1];
    const bool valid =
        t < a.T && (a.flexible || (mn <= mx && t + mn >= 0 && t + (long long)mx < a.T));
    float acc = 0.0f;
    if (valid) {
      const int32_t* d = a.delays + (size_t)i * a.S * a.P;
      const float* wrow = a.weights + (size_t)i * a.S;
      for (int s = 0; s < a.S; ++s) {
        float w = __ldg(wrow + s);
        if (w == 0.0f) continue;
        if constexpr (STORAGE != BP_STORAGE_F32) w = w * a.scales[s];
        for (int p = 0; p < a.P; ++p) {
          const long long tt = t + __ldg(d + s * a.P + p);
          if (tt < 0 || tt >= a.T) continue;
          const size_t row = (STORAGE == BP_STORAGE_F32) ? (size_t)(s * a.P + p)
                                                         : (size_t)(s * a.P + p) * kHalfCopies;
          const float u = load_trace<STORAGE>(a.traces, row * a.pitch + a.lpad + tt);
          acc = __fadd_rn(acc, __fmul_rn(w, u));
        }
      }
    }
    if constexpr (MAXRED) {
      if (valid) {
        const unsigned long long key = make_key(acc, i + a.index_base);
        best = key > best ? key : best;
      }
    } else {
      if (valid) a.beam[(size_t)i * a.ldb + t] = acc;
    }
  }
  if constexpr (MAXRED) {
    if (best != 0ull) red_max_u64(&a.keys[t], best);
  }
}

// ---------------------------------------------------------------------------
// Small kernels.
// ---------------------------------------------------------------------------

// Per-source min/max over weighted stations (beamform.c:10-47).
__global__ void minmax_kernel(const int32_t* __restrict__ delays, const float* __restrict__ weights,
                              int N, int S, int P, int32_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int mn = INT_MAX, mx = INT_MIN;
  const int32_t* d = delays + (size_t)i * S * P;
  const float* w = weights + (size_t)i * S;
  for (int s = 0; s < S; ++s) {
    if (w[s] == 0.0f) continue;
    for (int p = 0; p < P; ++p) {
      const int v = d[s * P + p];
      mn = min(mn, v);
      mx = max(mx, v);
    }
  }
  out[2 * i] = mn;
  out[2 * i + 1] = mx;
}

// FP32 prestack into the trace layout (beamform.c:108-152 arithmetic):
// U = ((0 + a0 * F0) + a1 * F1) + ..., rounded multiply then rounded add.
// grid (ceil(pitch / 256), S); each thread one row index of every phase row.
__global__ void prestack_f32_kernel(const float* __restrict__ F, const float* __restrict__ alpha,
                                    int T, int S, int C, int P, int lpad, long long pitch,
                                    float* __restrict__ out) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (r >= pitch) return;
  const long long t = r - lpad;
  const bool in = t >= 0 && t < T;
  for (int p = 0; p < P; ++p) {
    float acc = 0.0f;
    if (in) {
      for (int c = 0; c < C; ++c)
        acc = __fadd_rn(acc, __fmul_rn(__ldg(alpha + ((size_t)s * C + c) * P + p),
                                       __ldg(F + ((size_t)s * C + c) * T + t)));
    }
    out[(size_t)(s * P + p) * pitch + r] = acc;
  }
}

// Prestacked (S, T, P) -> trace layout, FP32.
__global__ void traces_from_prestacked_kernel(const float* __restrict__ U, int T, int S, int P,
                                              int lpad, long long pitch, float* __restrict__ out) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (r >= pitch) return;
  const long long t = r - lpad;
  const bool in = t >= 0 && t < T;
  for (int p = 0; p < P; ++p)
    out[(size_t)(s * P + p) * pitch + r] = in ? U[((size_t)s * T + t) * P + p] : 0.0f;
}

// Keys -> (beam_max, argmax).  beam_max keeps its content where no source
// was a candidate, argmax gets 0 there (beamform.c:332-334).
__global__ void decode_keys_kernel(const unsigned long long* __restrict__ keys, int T,
                                   float* __restrict__ beam_max, int32_t* __restrict__ argmax) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const unsigned long long k = keys[t];
  if (k != 0ull) {
    beam_max[t] = key_value(k);
    argmax[t] = key_source(k);
  } else {
    argmax[t] = 0;
  }
}

// Trace rows (S, P, T) -> prestacked (S, T, P), the reference's layout.
__global__ void rows_to_prestacked_kernel(const float* __restrict__ rows, int T, int S, int P,
                                          float* __restrict__ U) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (t >= T) return;
  for (int p = 0; p < P; ++p)
    U[((size_t)s * T + t) * P + p] = rows[(size_t)(s * P + p) * T + t];
}

// Differential mode (beamform.c:338-394): one beam per source at the zero lag
// t0 = (T - 1) / 2 of inter-station correlations, strict rule, written only
// where the rule holds.  One thread per source, stations then phases in order.
__global__ void differential_kernel(const float* __restrict__ traces, long long pitch, int lpad,
                                    int T, const int32_t* __restrict__ delays,
                                    const float* __restrict__ weights, int N, int S, int P,
                                    float* __restrict__ beam) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const long long t0 = ((long long)T - 1) / 2;
  const int32_t* d = delays + (size_t)i * S * P;
  const float* w = weights + (size_t)i * S;
  int mn = INT_MAX, mx = INT_MIN;
  for (int s = 0; s < S; ++s) {
    if (w[s] == 0.0f) continue;
    for (int p = 0; p < P; ++p) {
      mn = min(mn, d[s * P + p]);
      mx = max(mx, d[s * P + p]);
    }
  }
  if (mn > mx || t0 + mn < 0 || t0 + (long long)mx >= T) return;
  float acc = 0.0f;
  for (int s = 0; s < S; ++s) {
    const float ws = w[s];
    if (ws == 0.0f) continue;
    for (int p = 0; p < P; ++p) {
      const float u = traces[(size_t)(s * P + p) * pitch + lpad + t0 + d[s * P + p]];
      acc = __fadd_rn(acc, __fmul_rn(ws, u));
    }
  }
  beam[i] = acc;
}

// ---------------------------------------------------------------------------
// Source tiling map: recursive median splits of the sources on their delay
// vectors (a k-d tree over the (station, phase) delays), so that the 64
// sources of a tile are close in delay space and every station's delay
// window inside a tile is short.  Each level: pick per splitting segment the
// (station, phase) whose weighted delays vary most (variance over up to 256
// evenly spaced members), then one global stable radix sort of all sources
// on (segment, delay) keys orders every splitting segment by that delay and
// leaves finished segments in place; children split at a multiple of the
// tile size.  Only the grouping changes: keys and outputs use the original
// source index.
// ---------------------------------------------------------------------------
__global__ void split_dim_kernel(const int32_t* __restrict__ delays,
                                 const float* __restrict__ weights, int S, int P,
                                 const int* __restrict__ perm, const int* __restrict__ seg_begin,
                                 const int* __restrict__ seg_end, int* __restrict__ seg_dim) {
  const int g = blockIdx.x;
  const int b = seg_begin[g], e = seg_end[g];
  const int len = e - b;
  const int D = S * P;
  if (len <= 0 || seg_dim[g] < 0) return;  // finished segment (dim preset to -1)
  const int n_sample = min(len, 256);
  __shared__ double best_v[32];
  __shared__ int best_d[32];
  double bv = -1.0;
  int bd = 0;
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    const int s = d / P;
    double sum = 0.0, sq = 0.0;
    int n = 0;
    for (int j = 0; j < n_sample; ++j) {
      const int o = perm[b + (int)(((long long)len * j) / n_sample)];
      if (weights[(size_t)o * S + s] == 0.0f) continue;
      const double v = (double)delays[(size_t)o * D + d];
      sum += v;
      sq += v * v;
      ++n;
    }
    const double var = n > 1 ? (sq - sum * sum / n) / n : 0.0;
    if (var > bv) {  // ascending d per thread: the lower d wins ties
      bv = var;
      bd = d;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    const double ov = __shfl_down_sync(0xFFFFFFFFu, bv, off);
    const int od = __shfl_down_sync(0xFFFFFFFFu, bd, off);
    if (ov > bv || (ov == bv && od < bd)) {
      bv = ov;
      bd = od;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    best_v[threadIdx.x >> 5] = bv;
    best_d[threadIdx.x >> 5] = bd;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = -1.0;
    int d = 0;
    for (int w = 0; w < (int)((blockDim.x + 31) / 32); ++w)
      if (best_v[w] > v || (best_v[w] == v && best_d[w] < d)) {
        v = best_v[w];
        d = best_d[w];
      }
    seg_dim[g] = d;
  }
}

// Composite sort key of every source position for one level:
// (segment index << 32) | biased delay on the segment's split dimension
// (0 for finished segments, which therefore keep their order).
__global__ void split_keys_kernel(const int32_t* __restrict__ delays, int D, int N, int K,
                                  const int* __restrict__ perm,
                                  const int* __restrict__ seg_of_tile,
                                  const int* __restrict__ seg_dim,
                                  unsigned long long* __restrict__ keys) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= N) return;
  const int g = seg_of_tile[pos / K];
  const int d = seg_dim[g];
  uint32_t low = 0u;
  if (d >= 0) low = (uint32_t)delays[(size_t)perm[pos] * D + d] ^ 0x80000000u;
  keys[pos] = ((unsigned long long)(uint32_t)g << 32) | low;
}

__global__ void iota_perm_kernel(int* __restrict__ perm, int N, int total) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) perm[i] = (i < N) ? i : -1;
}

// Orders the slots of every tile by source index (unused slots last), so
// that ascending slots are ascending sources: the staged kernel's epilogue
// then keeps the lowest source index among equal maxima with a plain `>`.
// One block of kTableTile threads per tile.
__global__ void sort_tile_slots_kernel(int* __restrict__ perm, int N) {
  __shared__ int v[kTableTile];
  const int k = threadIdx.x;
  const size_t base = (size_t)blockIdx.x * kTableTile;
  const int o = perm[base + k];
  v[k] = (o >= 0 && o < N) ? o : INT_MAX;
  __syncthreads();
  const int mine = v[k];
  int rank = 0;
  for (int j = 0; j < kTableTile; ++j) rank += (v[j] < mine) || (v[j] == mine && j < k);
  perm[base + rank] = mine == INT_MAX ? -1 : mine;
}

// ---------------------------------------------------------------------------
// 16-bit trace storage (BF16 / FP16 with a per-station scale).
//
// Each (station, phase) row is stored kHalfCopies = 4 times: version v holds
// x[t + v] at index lpad + t.  Row (s * P + p) * 4 + v of `pitch` 16-bit
// elements.  A run of four consecutive samples x[a .. a + 3] is then always
// one aligned 64-bit word: version a & 3, index lpad + a - (a & 3).
// The stored value is U / scale_s with scale_s a power of two >= max |U| of
// the station (1 for an all-zero station), so the scaling itself is exact and
// only the rounding to 16 bits loses precision.
// ---------------------------------------------------------------------------
template <int STORAGE> struct Half16;
template <> struct Half16<BP_STORAGE_BF16> {
  using T = __nv_bfloat16;
  static __device__ __forceinline__ T from_float(float v) { return __float2bfloat16_rn(v); }
};
template <> struct Half16<BP_STORAGE_F16> {
  using T = __half;
  static __device__ __forceinline__ T from_float(float v) { return __float2half_rn(v); }
};

// Pass 1: max |U| per station (as float bits, non-negative floats order like
// unsigned integers).  scale_bits must be zeroed first.
__global__ void prestack_absmax_kernel(const float* __restrict__ F, const float* __restrict__ alpha,
                                       int T, int S, int C, int P,
                                       unsigned int* __restrict__ scale_bits) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  float m = 0.0f;
  if (t < T) {
    for (int p = 0; p < P; ++p) {
      float acc = 0.0f;
      for (int c = 0; c < C; ++c)
        acc = __fadd_rn(acc, __fmul_rn(__ldg(alpha + ((size_t)s * C + c) * P + p),
                                       __ldg(F + ((size_t)s * C + c) * T + t)));
      m = fmaxf(m, fabsf(acc));  // fmaxf drops NaN
    }
  }
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_down_sync(0xFFFFFFFFu, m, off));
  if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(scale_bits + s, __float_as_uint(m));
}

// max |U| bits -> power-of-two scale (in place, as float).
__global__ void scale_pow2_kernel(unsigned int* __restrict__ scale_bits, int S) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const float m = __uint_as_float(scale_bits[s]);
  float sc = 1.0f;
  if (m > 0.0f && isfinite(m)) {
    int e;
    const float f = frexpf(m, &e);  // m = f * 2^e, f in [0.5, 1)
    sc = ldexpf(1.0f, (f == 0.5f) ? e - 1 : e);
  }
  reinterpret_cast<float*>(scale_bits)[s] = sc;
}

// Pass 2: U / scale rounded to 16 bits, every shifted copy, zero padding.
template <int STORAGE>
__global__ void prestack_h16_kernel(const float* __restrict__ F, const float* __restrict__ alpha,
                                    int T, int S, int C, int P, int lpad, long long pitch,
                                    const float* __restrict__ scales,
                                    typename Half16<STORAGE>::T* __restrict__ out) {
  using H = Half16<STORAGE>;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (r >= pitch) return;
  const float inv = 1.0f / scales[s];  // power of two: exact
  for (int v = 0; v < kHalfCopies; ++v) {
    const long long t = r - lpad + v;
    const bool in = t >= 0 && t < T;
    for (int p = 0; p < P; ++p) {
      float acc = 0.0f;
      if (in) {
        for (int c = 0; c < C; ++c)
          acc = __fadd_rn(acc, __fmul_rn(__ldg(alpha + ((size_t)s * C + c) * P + p),
                                         __ldg(F + ((size_t)s * C + c) * T + t)));
      }
      out[((size_t)(s * P + p) * kHalfCopies + v) * pitch + r] = H::from_float(acc * inv);
    }
  }
}

// 16-bit trace rows back to FP32 rows of the same layout: element x of row
// (s, p) becomes value * scale_s, exact (a 16-bit value times a power of
// two).  Only copy 0 of the four shifted copies is read.  Lets the FP32
// staged kernel serve 16-bit traces whose four-copy windows fit no shape.
template <int STORAGE>
__global__ void expand_h16_kernel(const void* __restrict__ in, const float* __restrict__ scales,
                                  int P, long long pitch, float* __restrict__ out) {
  const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;  // s * P + p
  if (x >= pitch) return;
  const float v = load_trace<STORAGE>(in, (size_t)row * kHalfCopies * pitch + x);
  out[(size_t)row * pitch + x] = v * __ldg(scales + row / P);
}

#endif  // BP_TEMPLATE_KERNELS_ONLY

}  // namespace bp
