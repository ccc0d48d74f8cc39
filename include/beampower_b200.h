/*
 * beampower_b200 -- C-ABI of the sm_100a beamforming library
 * (beampower_b200/lib/libbeampower_b200.so).
 *
 * Four groups of entry points; groups 3 (detection on the beam series) and
 * 4 (inputs: waveform features, travel times in samples) are described at
 * their sections below:
 *
 * 1. Drop-ins for the reference's GPU library.  Same symbol names, argument
 *    order and meaning as beampower/src/beamform_gpu.h:1-2, bound by
 *    beampower/core.py:65-87 ("gpu" entry of LIBRARIES).  They take HOST
 *    buffers, synchronise before returning, and return an int status (0 on
 *    success) where the reference returned void and called exit() on errors.
 *    A caller that ignores the return value (ctypes without restype) keeps
 *    working unchanged.
 *
 * 2. Stream-ordered device entry points (prefix bp_) for callers whose data
 *    already lives in HBM (torch tensors, the batch and stream schedulers).
 *    Pointers are device pointers, `stream` is a cudaStream_t passed as
 *    void*, nothing synchronises, and every function returns an int status.
 *
 * Conventions shared by both groups:
 *   N = n_sources, S = n_stations, C = n_channels, P = n_phases,
 *   T = n_samples.
 *   time_delays (N, S, P) int32, weights (N, S) float32, row-major.
 *   out_of_bounds: 0 = 'strict', 1 = 'flexible' (beampower/beampower.py:85-88).
 *   Results follow the reference's CPU path (beampower/src/beamform.c):
 *   stations ascending, phases ascending, one FP32 accumulator per
 *   (source, sample), each term a rounded multiply then a rounded add,
 *   zero-weight stations skipped; max/argmax keeps the lowest source index
 *   among equal beams.
 */
#ifndef BEAMPOWER_B200_H
#define BEAMPOWER_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define BP_API __attribute__((visibility("default")))
#else
#define BP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define BP_OK 0
#define BP_ERR_INVALID_ARGUMENT 1   /* sizes, pointers or options rejected   */
#define BP_ERR_CUDA 2               /* a CUDA runtime call failed            */
#define BP_ERR_OUT_OF_MEMORY 3      /* device allocation failed              */
#define BP_ERR_UNSUPPORTED 4        /* shape outside what the kernels handle */
#define BP_ERR_KERNEL 5             /* a kernel reported a failure (status)  */
#define BP_ERR_SCRATCH_LIMIT 6      /* size beyond the fixed scratch array of
                                       bp_beamform_max_noalloc              */

/* ---- trace storage types ---------------------------------------------- */
#define BP_STORAGE_F32 0
#define BP_STORAGE_BF16 1
#define BP_STORAGE_F16 2

/* ---- reduce ------------------------------------------------------------ */
#define BP_REDUCE_NONE 0
#define BP_REDUCE_MAX 1

/* ======================================================================= */
/* 1. Drop-in host-buffer entry points                                     */
/* ======================================================================= */

/* Full network response, reduce='none'.
 * Replaces `beamform` of beampower/src/beamform.cu:462-659
 * (declared beamform_gpu.h:1, argtypes core.py:65-75).
 * waveform_features: the PRESTACKED traces (S, T, P) float32, phase fastest,
 * as produced by prestack_waveform_features.  beam: (N, T) float32; entries
 * that the strict rule does not compute keep the caller's content. */
BP_API int beamform(float *waveform_features, int *time_delays, float *weights,
             size_t n_samples, size_t n_sources, size_t n_stations,
             size_t n_phases, int out_of_bounds, float *beam);

/* Max and argmax over sources for every sample, reduce='max'.
 * Replaces `beamform_max` of beampower/src/beamform.cu:207-460
 * (declared beamform_gpu.h:2, argtypes core.py:76-87).
 * beam_max[t] is written only where some source is a candidate; otherwise it
 * keeps the caller's content (the reference front-end passes zeros,
 * beampower/beampower.py:175-176).  source_index_beam_max[t] is always
 * written (0 when there is no candidate). */
BP_API int beamform_max(float *waveform_features, int *time_delays, float *weights,
                 size_t n_samples, size_t n_sources, size_t n_stations,
                 size_t n_phases, int out_of_bounds, float *beam_max,
                 int *source_index_beam_max);

/* Channel -> phase prestack on the GPU, host buffers.
 * Same prototype as the CPU library's prestack_waveform_features
 * (beampower/src/beamform.c:108-111, argtypes core.py:50-59); num_threads is
 * accepted and ignored.  features (S, C, T), weights_phases (S, C, P),
 * prestacked out (S, T, P), all float32. */
BP_API int prestack_waveform_features(float *waveform_features, float *weights_phases,
                               size_t n_samples, size_t n_stations,
                               size_t n_channels, size_t n_phases,
                               int num_threads, float *prestacked_traces);

/* Whole hot path from host buffers in one call: upload, GPU prestack, table
 * build, beamforming, download.  This is what beampower_b200.beamform()
 * calls for numpy inputs (the reference front-end prestacks on the CPU,
 * beampower/beampower.py:103-105; here it runs on the GPU).
 * reduce = BP_REDUCE_MAX: beam_max (T,), argmax (T,) ; beam unused.
 * reduce = BP_REDUCE_NONE: beam (N, T) ; beam_max / argmax unused.
 * storage = BP_STORAGE_F32 / BF16 / F16 (16-bit storage uses a per-station
 * scale and FP32 accumulation). */
BP_API int bp_beamform_host(const float *waveform_features, const float *weights_phases,
                     const int32_t *time_delays, const float *weights_sources,
                     size_t n_samples, size_t n_sources, size_t n_stations,
                     size_t n_channels, size_t n_phases, int out_of_bounds,
                     int reduce, int storage, float *beam_max, int32_t *argmax,
                     float *beam);

/* ======================================================================= */
/* 2. Stream-ordered device entry points                                   */
/* ======================================================================= */

/* A travel-time table made resident in HBM: per source tile, the active
 * stations, each station's delay window, 16-bit delay offsets and weights,
 * and per source the min/max delay over weighted stations.  Built once per
 * (time_delays, weights_sources) pair and reused by every call. */
typedef struct bp_table bp_table;

typedef struct bp_table_info {
  int64_t n_sources, n_stations, n_phases;
  int32_t tile_sources;      /* sources per tile                          */
  int32_t n_tiles;
  int32_t min_delay;         /* min over weighted (source, station, phase) */
  int32_t max_delay;         /* max over weighted (source, station, phase) */
  int32_t max_spread;        /* widest per-tile station delay window - 1   */
  int32_t max_active;        /* most active stations in one tile           */
  int32_t any_nonfinite;     /* some non-zero weight is NaN or +-inf       */
  int32_t uses_window_kernel;/* 1: staged kernel (FP32 windows fit a shape),
                                 0: direct kernel for every storage        */
} bp_table_info;

/* Build a table from device arrays (N, S, P) int32 and (N, S) float32.
 * Allocates device memory (stream-ordered) and synchronises `stream` once to
 * read the table statistics back. */
BP_API int bp_table_create(const int32_t *d_time_delays, const float *d_weights_sources,
                    size_t n_sources, size_t n_stations, size_t n_phases,
                    void *stream, bp_table **out_table);
BP_API int bp_table_destroy(bp_table *table);
BP_API int bp_table_get_info(const bp_table *table, bp_table_info *info);

/* Layout of device trace storage for a table and a record length: element
 * (s, p, t) sits at row (s * P + p) of `pitch` elements, index lpad + t;
 * indexes outside [lpad, lpad + T) must hold zeros.  16-bit storage holds
 * bp_trace_copies(storage) = 4 copies per (s, p): row (s * P + p) * 4 + v,
 * index lpad + t, holds element t + v (copy v shifted by v samples). */
BP_API int bp_trace_layout(const bp_table *table, size_t n_samples, size_t *lpad,
                    size_t *pitch);
/* Rows per (station, phase) of trace storage: 1 for FP32, 4 for BF16 / FP16. */
BP_API int bp_trace_copies(int storage);

/* Prestack on device: features (S, C, T) f32, weights_phases (S, C, P) f32
 * -> traces in the layout above (element type per `storage`; zero padding is
 * written).  For 16-bit storage `d_scales` (S,) receives each station's
 * max |U| (1 where it is 0) and traces hold U / scale. */
BP_API int bp_prestack_dev(const float *d_features, const float *d_weights_phases,
                    size_t n_samples, size_t n_stations, size_t n_channels,
                    size_t n_phases, int storage, size_t lpad, size_t pitch,
                    void *d_traces, float *d_scales, void *stream);

/* Prestacked (S, T, P) f32 on device -> traces in the layout above (f32). */
BP_API int bp_traces_from_prestacked_dev(const float *d_prestacked, size_t n_samples,
                                  size_t n_stations, size_t n_phases, size_t lpad,
                                  size_t pitch, float *d_traces, void *stream);

/* Shift-and-stack with fused max/argmax over sources.  d_keys (T,) uint64 is
 * scratch the caller provides; it is cleared here.  Results go to
 * d_beam_max (T,) and d_argmax (T,) with the drop-in's semantics (beam_max
 * keeps its previous content where no source is a candidate). */
BP_API int bp_beamform_max_dev(const bp_table *table, const void *d_traces, int storage,
                        const float *d_scales, size_t n_samples, size_t lpad,
                        size_t pitch, int out_of_bounds,
                        unsigned long long *d_keys, float *d_beam_max,
                        int32_t *d_argmax, void *stream);

/* Full response (N, T), row stride ldb elements. */
BP_API int bp_beamform_dev(const bp_table *table, const void *d_traces, int storage,
                    const float *d_scales, size_t n_samples, size_t lpad,
                    size_t pitch, int out_of_bounds, float *d_beam, size_t ldb,
                    void *stream);

/* ---- batches of records (waveform windows, streamed chunks) ------------- */

/* One record of a batch: a waveform window, or a streamed chunk together
 * with the samples it carries over from the previous chunk.  Record sample t
 * is global sample t_origin + t; the traces hold record samples
 * [0, n_samples) in the layout of bp_trace_layout(table, n_samples); results
 * are produced for record samples [out0, out1).  The strict rule's lower
 * bound is applied in global time (t_origin + t + min >= 0), its upper bound
 * in record time (t + max < n_samples).  A station mask restricts the record
 * to a subset of the table's stations (as if weights_sources were zero for
 * the others), without rebuilding the table.  No reference counterpart: the
 * reference beamforms one window per call (beampower/beampower.py:10). */
typedef struct bp_record {
  int32_t table;                 /* index into the batch's tables             */
  int32_t out_of_bounds;         /* 0 strict, 1 flexible                      */
  const void *traces;            /* device                                    */
  const float *scales;           /* device (S,), 16-bit storage only          */
  size_t n_samples, lpad, pitch;
  int64_t t_origin;
  size_t out0, out1;
  const uint32_t *station_mask;  /* device, ceil(S / 32) words, or NULL (all) */
  float *beam_max;               /* device [out1 - out0]                      */
  int32_t *argmax;               /* device [out1 - out0]                      */
} bp_record;

typedef struct bp_batch bp_batch;

/* One record alone (no batch): the plain staged launch over the record's
 * output range, global time origin included; this is what a streamed chunk
 * with its carried samples uses.  d_keys: (out1 - out0) uint64 scratch,
 * cleared here.  station_mask must be NULL.  Stream-ordered, no allocation,
 * no synchronisation. */
BP_API int bp_record_beamform_max_dev(const bp_table *table, const bp_record *record,
                                      int storage, unsigned long long *d_keys,
                                      void *stream);

/* Upload the batch's descriptors and per-record delay ranges (stream-ordered
 * device allocations; synchronises `stream` once). */
BP_API int bp_batch_create(const bp_table *const *tables, int n_tables,
                           const bp_record *records, int n_records, int storage,
                           void *stream, bp_batch **out_batch);
/* Beamform every record (reduce='max') in one persistent launch fed by a
 * device work queue, then decode all outputs.  Only memsets and kernel
 * launches on `stream`: it can be captured in a CUDA graph and replayed on
 * new trace data in the same buffers. */
BP_API int bp_batch_run(bp_batch *batch, void *stream);
/* Kernel status bits of the batch's last runs (synchronises `stream`). */
BP_API int bp_batch_status(bp_batch *batch, void *stream, int *status);
BP_API int bp_batch_destroy(bp_batch *batch);

/* Per-source (min, max) delay over weighted stations, (N, 2) int32, the
 * reference's _find_minmax_time_delays (beampower/src/beamform.c:10-47,
 * beamform.cu:28-65). */
BP_API int bp_minmax_dev(const int32_t *d_time_delays, const float *d_weights_sources,
                  size_t n_sources, size_t n_stations, size_t n_phases,
                  int32_t *d_minmax, void *stream);

/* Direct (unstaged) kernel, any P and any delay spread: the path taken when
 * a table's windows do not fit shared memory, and a cross-check. */
BP_API int bp_beamform_max_direct_dev(const void *d_traces, int storage, const float *d_scales,
                               size_t n_samples, size_t lpad, size_t pitch,
                               const int32_t *d_time_delays, const float *d_weights_sources,
                               size_t n_sources, size_t n_stations, size_t n_phases,
                               int out_of_bounds, unsigned long long *d_keys,
                               float *d_beam_max, int32_t *d_argmax, void *stream);

/* Allocation-free max/argmax, for callers that must not allocate device
 * memory while they run (a service that reserves its GPU memory once at
 * start-up, or a host program whose own allocator owns the device, where a
 * cudaMalloc inside a library call would fail or stall the stream).  It has
 * no counterpart in the reference.
 * Same inputs and results as bp_beamform_max_direct_dev (FP32 traces in the
 * row layout above, raw delays and weights), but its working memory -- one
 * uint64 key per sample and a (min, max) delay pair per source -- lives in an
 * 8 MiB array compiled into the library, which every GPU that loads the
 * library keeps until the process exits.  Limits: n_samples <= 524288 and
 * n_sources <= 524288; larger calls return BP_ERR_SCRATCH_LIMIT.  It calls
 * no allocator.  The first call on each device looks up the array's device
 * address (make it before any stream capture starts).  All calls share the
 * array and it keeps the previous call's contents; each call clears what it
 * needs, and calls that overlap on the GPU race with each other. */
BP_API int bp_beamform_max_noalloc(const float *d_traces, size_t n_samples, size_t lpad,
                                   size_t pitch, const int32_t *d_time_delays,
                                   const float *d_weights_sources, size_t n_sources,
                                   size_t n_stations, size_t n_phases, int out_of_bounds,
                                   float *d_beam_max, int32_t *d_argmax, void *stream);

/* Differential mode (reduce over inter-station correlations): one beam per
 * source at the zero lag t0 = (T - 1) / 2, strict rule, written only where
 * the rule holds.  Replaces the CPU-only beamform_differential of
 * beampower/src/beamform.c:338-394 (argtypes core.py:27-37); the reference's
 * GPU branch was a stub (beampower/beampower.py:220-223).  Host buffers;
 * num_threads is accepted and ignored. */
BP_API int beamform_differential(float *waveform_features, int *time_delays,
                                 float *weights, size_t n_samples, size_t n_sources,
                                 size_t n_stations, size_t n_phases, int num_threads,
                                 float *beam);

/* Device version of beamform_differential on traces in the layout above. */
BP_API int bp_beamform_differential_dev(const float *d_traces, size_t n_samples, size_t lpad,
                                        size_t pitch, const int32_t *d_time_delays,
                                        const float *d_weights_sources, size_t n_sources,
                                        size_t n_stations, size_t n_phases, float *d_beam,
                                        void *stream);

/* ======================================================================= */
/* 3. Detection on the beam series (the step after beamform_max)           */
/* ======================================================================= */
/* The reference tutorial turns beam_max into detections in two notebook
 * cells; these entry points restate them on the device with identical
 * results (float32 arithmetic in NumPy's own order, SciPy's peak rules).
 * Each allocates its scratch with cudaMallocAsync on `stream` and
 * synchronises `stream` (it reads counts back), so none of them can be
 * captured in a CUDA graph.  bp_threshold_dev keeps the pairwise-sum split
 * tree of each length it has seen on the device (cudaMalloc, up to 64 lengths
 * per process, freed at exit). */

#define BP_THRESHOLD_RMS 0 /* window mean + num_dev * standard deviation */
#define BP_THRESHOLD_MAD 1 /* window median + num_dev * median |x - median| */

/* Time-dependent detection threshold, one value per sample
 * (notebooks/3_beampower.ipynb:497-579, time_dependent_threshold).  Zero
 * samples are first replaced by noise * deviation + centre of the non-zero
 * samples: d_white_noise holds the standard normal draws in sample order
 * (n_white_noise >= number of zeros); NULL draws them from this library's
 * own generator seeded by `seed` (the notebook draws them from NumPy's global
 * generator).  Windows of sliding_window samples start every
 * int((1 - overlap) * sliding_window) samples.  Rejects n_samples <=
 * sliding_window and a window step below 1 (the notebook raises there). */
BP_API int bp_threshold_dev(const float *d_series, size_t n_samples, size_t sliding_window,
                            double overlap, int kind, float num_dev,
                            const float *d_white_noise, size_t n_white_noise,
                            unsigned long long seed, float *d_threshold, void *stream);

/* Peak sample indexes in increasing order, as
 * scipy.signal.find_peaks(x, distance=distance)[0] (called at
 * notebooks/3_beampower.ipynb:621): local maxima, flat plateaus by their
 * midpoint, then, when distance > 0, the greedy rule that keeps peaks in
 * decreasing height and drops every peak closer than ceil(distance) samples
 * to a kept one (equal heights: the later sample first).  distance <= 0
 * means no distance rule; 0 < distance < 1 is rejected as SciPy does.
 * capacity must be at least n_samples / 2. */
BP_API int bp_find_peaks_dev(const float *d_x, size_t n_samples, double distance,
                             int32_t *d_peaks, size_t capacity, size_t *n_peaks, void *stream);

/* SciPy's other find_peaks conditions used around the tutorial (the
 * prominence / wlen option is shown at notebooks/3_beampower.ipynb:625),
 * applied in SciPy's order: height, threshold, distance, prominence.  Borders
 * are float64 with NaN for an open side; the d_height_* / d_threshold_* /
 * d_prominence_* arrays, when not NULL, give per-sample float64 borders (n_samples values)
 * read at the peak (SciPy's array borders). */
typedef struct bp_peak_options {
  double distance;          /* <= 0: no distance rule                          */
  int32_t use_height;       /* 1: keep height_min <= x[peak] <= height_max      */
  double height_min, height_max;
  const double *d_height_min, *d_height_max;
  int32_t use_threshold;    /* 1: keep threshold_min <= min(x[p] - x[p-1],
                               x[p] - x[p+1]) and max(...) <= threshold_max    */
  double threshold_min, threshold_max;
  const double *d_threshold_min, *d_threshold_max;
  int32_t use_prominence;   /* 1: keep prominence_min <= prominence <= max      */
  double prominence_min, prominence_max;
  const double *d_prominence_min, *d_prominence_max;
  double wlen;              /* > 1: prominence walk limited to ceil(wlen) / 2
                               samples each side; <= 0: whole series            */
} bp_peak_options;

/* Peaks as scipy.signal.find_peaks(x, height=, threshold=, distance=,
 * prominence=, wlen=)
 * (identical indexes; prominences in float64, bases as SciPy's
 * left_bases / right_bases).  d_prominences / d_left_bases / d_right_bases
 * may be NULL and are written only with use_prominence.  Synchronises. */
BP_API int bp_find_peaks_opt_dev(const float *d_x, size_t n_samples, const bp_peak_options *opt,
                                 int32_t *d_peaks, double *d_prominences,
                                 int32_t *d_left_bases, int32_t *d_right_bases,
                                 size_t capacity, size_t *n_peaks, void *stream);

/* Detections (notebooks/3_beampower.ipynb:618-626): the peaks of d_beam_max
 * as above whose height is strictly above d_threshold, with their heights
 * and, when d_argmax is not NULL, the winning source of each. */
BP_API int bp_detect_dev(const float *d_beam_max, const int32_t *d_argmax,
                         const float *d_threshold, size_t n_samples, double distance,
                         int32_t *d_peaks, float *d_heights, int32_t *d_sources,
                         size_t capacity, size_t *n_detections, void *stream);

/* ======================================================================= */
/* 4. Inputs: waveform features and travel times in samples              */
/* ======================================================================= */
/* The reference tutorial's envelope transform (notebooks/3_beampower.ipynb:
 * 74-103, `envelope`, applied to every trace at :145-147): the modulus of the
 * analytic signal (scipy.signal.hilbert), minus its median, divided by its
 * median absolute deviation (1 when that is 0), clipped above at clip_max
 * (1e5 in the tutorial).  The FFTs run in cuFFT (float32), so results match
 * the tutorial's float32 SciPy FFTs to rounding, not bit for bit.  Allocates
 * scratch with cudaMallocAsync on `stream`; cuFFT plans are cached per
 * (device, length, rows) for the life of the process. */

/* d_x: n_rows rows of n_samples float32 (contiguous); d_out: same shape.
 * The FFT plans behind the envelope are cached per (device, length, rows)
 * and shared by every stream: envelope calls of the same shape on different
 * streams must not overlap on the GPU (order them with an event or run them
 * on one stream); calls on one stream are always safe. */
BP_API int bp_envelope_dev(const float *d_x, size_t n_rows, size_t n_samples, float clip_max,
                           float *d_out, void *stream);

/* Raw waveforms (S, C, T) to the beamformer's trace rows in one call: the
 * envelope features of every (station, channel) row, then bp_prestack_dev
 * with the same storage / layout arguments.  Replaces the tutorial's CPU
 * feature loop followed by the reference front-end's CPU prestack
 * (beampower/beampower.py:103-105). */
BP_API int bp_prestack_envelope_dev(const float *d_waveforms, const float *d_weights_phases,
                                    size_t n_samples, size_t n_stations, size_t n_channels,
                                    size_t n_phases, float clip_max, int storage, size_t lpad,
                                    size_t pitch, void *d_traces, float *d_scales,
                                    void *stream);

/* Travel times in seconds to int32 sample delays, as the tutorial's
 * sec_to_samp (notebooks/3_beampower.ipynb:378-394): in float32,
 * sign(t) * trunc(|t * sampling_rate| + epsilon) (epsilon 0.2 there), and
 * INT_MIN where that is NaN, infinite or not below 2^31 (the x86 result of
 * the tutorial's NumPy cast).  d_seconds and d_delays hold n_sources rows of
 * n_per_source values ((S, P) per source); relative != 0 then subtracts each
 * row's minimum, the tutorial's optional relative delays (:396).  Reading
 * the tutorial's travel_times.h5 stays with the caller. */
BP_API int bp_seconds_to_samples_dev(const float *d_seconds, size_t n_sources,
                                     size_t n_per_source, double sampling_rate, double epsilon,
                                     int relative, int32_t *d_delays, void *stream);

/* Host function: NumPy's float32 pairwise sum of x[0..n) (the summation
 * order the threshold kernels reproduce), for checking that order without a
 * GPU.  No reference counterpart. */
BP_API float bp_pairwise_sum_f32(const float *x, size_t n);

/* ---- sources split over GPUs ---------------------------------------------
 * The reference splits sources over the visible GPUs and merges the partial
 * maxima on the host (beampower/src/beamform.cu:227-276, 430-445).  Here each
 * rank runs bp_beamform_max_dev on its block of sources (a table of those
 * sources) and keeps the keys buffer; bp_keys_to_shared_dev rebases the keys
 * to global source indexes (source_offset = the block's first source) and
 * maps them to signed order, an elementwise int64 max all-reduce over the
 * ranks merges them (NCCL, torch.distributed), and bp_keys_from_shared_dev
 * decodes the merged keys.  Results equal the single-GPU call bit for bit. */
BP_API int bp_keys_to_shared_dev(unsigned long long *d_keys, size_t n_samples,
                                 size_t source_offset, void *stream);
BP_API int bp_keys_from_shared_dev(const unsigned long long *d_keys, size_t n_samples,
                                   float *d_beam_max, int32_t *d_argmax, void *stream);

/* ---- staged-kernel configurations (autotuning) -------------------------- */
/* The staged kernel exists in several shapes (sources per thread, samples per
 * lane, consumer warps, ring stages, stations per ring stage, sources per
 * block, blocks per SM), all over the same 64-source tables.
 * bp_set_kernel_config chooses one per (storage, reduce) for every later
 * launch in the process (-1: built-in default); the environment variable
 * BEAMPOWER_B200_KERNEL_CONFIG overrides it.  beampower_b200/autotune.py
 * times the shapes on a workload and stores its choices.  A shape whose
 * shared memory does not fit a table falls back to config 0 for that table.
 * No reference counterpart (the reference has one launch shape,
 * beamform.cu:10). */
BP_API int bp_kernel_config_count(void);
BP_API int bp_kernel_config_describe(int config, int *sources_per_thread,
                                     int *samples_per_lane, int *consumer_warps,
                                     int *stages);
/* The other dimensions of a shape: stations carried by one ring stage (one
 * mbarrier round trip each), sources per block (64: one block per table tile;
 * 32: two blocks share a tile) and the blocks per SM it is built for. */
BP_API int bp_kernel_config_shape(int config, int *stations_per_stage,
                                  int *sources_per_block, int *blocks_per_sm);
BP_API int bp_set_kernel_config(int storage, int reduce, int config);
BP_API int bp_get_kernel_config(int storage, int reduce);
/* The shape a call on this table runs with (storage, reduce): the chosen one
 * when its shared memory and blocks per SM fit the table, else the first
 * that fits in a fixed, measured order; -1 when no shape holds the table's
 * windows in this storage (16-bit calls then expand their traces to FP32 and
 * run the FP32 shape, with the direct kernel's values, when that fits; else,
 * and for tables with uses_window_kernel == 0, the direct kernel runs); a
 * negative error code for bad arguments.  Records expand the same way;
 * batches need a shape for their own storage. */
BP_API int bp_table_kernel_config(const bp_table *table, int storage, int reduce);

/* ---- diagnostics -------------------------------------------------------- */
/* Last error message of the calling thread ("" if none). */
BP_API const char *bp_last_error(void);
/* Measure this GPU's shared-memory load bandwidth (GB/s, whole GPU) and
 * FP32 FMA throughput (TFLOP/s) with short microbenchmarks on `stream`
 * (synchronises it).  These are the rooflines of the staged kernel. */
BP_API int bp_measure_peaks(void *stream, double *smem_gbs, double *fp32_tflops);
/* Failure-path check: launches a kernel whose threads wait on an mbarrier
 * that nothing completes, with a limit of limit_ns (at most 1 s); the wait
 * gives up, the kernel ends, and *status_out receives the status bits
 * (1 = wait timeout).  Shows that a wait which can never finish ends with an
 * error status instead of hanging the GPU.  Synchronises `stream`. */
BP_API int bp_debug_wait_timeout(unsigned long long limit_ns, void *stream, int *status_out);
/* Library version string. */
BP_API const char *bp_version(void);
/* Kernel launches issued by this process since load (all entry points). */
BP_API uint64_t bp_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* BEAMPOWER_B200_H */
