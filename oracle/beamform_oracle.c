/*
 * CPU oracle for the beamforming hot path.  TEST INFRASTRUCTURE ONLY: it is
 * loaded by tests/, by __graft_entry__.smoke() and by the CPU legs of
 * bench.py as the checker, never by the beampower_b200 package.
 *
 * It restates, in plain C99 + OpenMP, the arithmetic of the reference's CPU
 * path (beampower/src/beamform.c).  Every function cites the reference lines
 * it follows.  Floating-point order is the reference's: one FP32 accumulator
 * per (source, sample), stations ascending, phases ascending, zero-weight
 * stations skipped, each term a rounded multiply then a rounded add
 * (compiled with -ffp-contract=off, which the reference gets from -std=c99).
 *
 * Validity rule (N = sources, S = stations, P = phases, T = samples):
 *   strict   (out_of_bounds = 0): sample t of source i is computed iff source
 *            i has at least one station with non-zero weight and
 *            0 <= t + min_i and t + max_i < T, min_i / max_i taken over the
 *            delays of stations with non-zero weight
 *            (beamform.c:10-47, 196-201).
 *   flexible (out_of_bounds = 1): every sample is computed; a term enters the
 *            sum iff 0 <= t + d < T (beamform.c:74-105).
 * One difference from the reference, on purpose: the reference's
 * beamform_max tests `t + min < 0` on size_t operands (beamform.c:281), so
 * that test never fires and a source with a negative minimum delay reads
 * outside its station's trace.  The oracle applies the rule above, which is
 * also what the reference's reduce='none' path does (int t, beamform.c:194).
 * For non-negative delays both agree bit for bit.
 *
 * Max/argmax (beamform.c:269-334): running max seeded with -FLT_MAX and
 * index 0, strict '>' over ascending source index (lowest index wins ties,
 * NaN never wins); beam_max[t] is written only when some source beat
 * -FLT_MAX, otherwise it keeps the caller's value; argmax[t] is always
 * written.
 */
#include <float.h>
#include <limits.h>
#include <stddef.h>
#include <stdint.h>
#include <omp.h>

static void set_threads(int num_threads)
{
    if (num_threads > 0)
        omp_set_num_threads(num_threads);
}

/* Per-source min/max delay over weighted stations: beamform.c:10-47.
 * Sources without a weighted station get {INT_MAX, INT_MIN}. */
void bpo_minmax(const int32_t *delays, const float *weights, size_t n_sources,
                size_t n_stations, size_t n_phases, int num_threads,
                int32_t *minmax)
{
    set_threads(num_threads);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n_sources; i++) {
        int32_t lo = INT_MAX, hi = INT_MIN;
        const int32_t *d = delays + (size_t)i * n_stations * n_phases;
        const float *w = weights + (size_t)i * n_stations;
        for (size_t s = 0; s < n_stations; s++) {
            if (w[s] == 0.0f)
                continue;
            for (size_t p = 0; p < n_phases; p++) {
                int32_t v = d[s * n_phases + p];
                if (v < lo) lo = v;
                if (v > hi) hi = v;
            }
        }
        minmax[2 * i] = lo;
        minmax[2 * i + 1] = hi;
    }
}

/* Channel -> phase prestack: beamform.c:108-152.
 * F (S, C, T), alpha (S, C, P) -> U (S, T, P), phase fastest. */
void bpo_prestack(const float *features, const float *alpha, size_t n_samples,
                  size_t n_stations, size_t n_channels, size_t n_phases,
                  int num_threads, float *prestacked)
{
    set_threads(num_threads);
#pragma omp parallel for schedule(static)
    for (long long s = 0; s < (long long)n_stations; s++) {
        const float *fs = features + (size_t)s * n_channels * n_samples;
        const float *as = alpha + (size_t)s * n_channels * n_phases;
        float *us = prestacked + (size_t)s * n_samples * n_phases;
        for (size_t t = 0; t < n_samples; t++) {
            for (size_t p = 0; p < n_phases; p++) {
                float acc = 0.0f;
                for (size_t c = 0; c < n_channels; c++)
                    acc = acc + as[c * n_phases + p] * fs[c * n_samples + t];
                us[t * n_phases + p] = acc;
            }
        }
    }
}

/* One beam value: beamform.c:49-72 (strict) and 74-105 (flexible). */
static float beam_at(const float *U, const int32_t *d, const float *w,
                     long long t, size_t n_samples, size_t n_stations,
                     size_t n_phases, int flexible)
{
    float acc = 0.0f;
    for (size_t s = 0; s < n_stations; s++) {
        if (w[s] == 0.0f)
            continue;
        const float *us = U + s * n_samples * n_phases;
        for (size_t p = 0; p < n_phases; p++) {
            long long tt = t + (long long)d[s * n_phases + p];
            if (flexible && (tt < 0 || tt >= (long long)n_samples))
                continue;
            acc = acc + w[s] * us[(size_t)tt * n_phases + p];
        }
    }
    return acc;
}

static int strict_valid(const int32_t *mm, long long t, size_t n_samples)
{
    if (mm[0] > mm[1])
        return 0; /* no weighted station */
    return t + (long long)mm[0] >= 0 && t + (long long)mm[1] < (long long)n_samples;
}

/* reduce='none': beamform.c:154-228.  beam (N, T) is only written where the
 * rule above computes a value; other entries keep the caller's content. */
void bpo_beamform(const float *U, const int32_t *delays, const float *weights,
                  size_t n_samples, size_t n_sources, size_t n_stations,
                  size_t n_phases, int out_of_bounds, int num_threads,
                  float *beam)
{
    set_threads(num_threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (long long i = 0; i < (long long)n_sources; i++) {
        const int32_t *d = delays + (size_t)i * n_stations * n_phases;
        const float *w = weights + (size_t)i * n_stations;
        int32_t mm[2] = {INT_MAX, INT_MIN};
        for (size_t s = 0; s < n_stations; s++) {
            if (w[s] == 0.0f) continue;
            for (size_t p = 0; p < n_phases; p++) {
                if (d[s * n_phases + p] < mm[0]) mm[0] = d[s * n_phases + p];
                if (d[s * n_phases + p] > mm[1]) mm[1] = d[s * n_phases + p];
            }
        }
        float *bi = beam + (size_t)i * n_samples;
        for (long long t = 0; t < (long long)n_samples; t++) {
            if (!out_of_bounds && !strict_valid(mm, t, n_samples))
                continue;
            bi[t] = beam_at(U, d, w, t, n_samples, n_stations, n_phases, out_of_bounds);
        }
    }
}

/* reduce='max': beamform.c:230-336. */
void bpo_beamform_max(const float *U, const int32_t *delays, const float *weights,
                      size_t n_samples, size_t n_sources, size_t n_stations,
                      size_t n_phases, int out_of_bounds, int num_threads,
                      float *beam_max, int32_t *argmax, int32_t *minmax_scratch)
{
    bpo_minmax(delays, weights, n_sources, n_stations, n_phases, num_threads,
               minmax_scratch);
    set_threads(num_threads);
#pragma omp parallel for schedule(dynamic, 16)
    for (long long t = 0; t < (long long)n_samples; t++) {
        float best = -FLT_MAX;
        int32_t best_i = 0;
        for (size_t i = 0; i < n_sources; i++) {
            if (!out_of_bounds && !strict_valid(minmax_scratch + 2 * i, t, n_samples))
                continue;
            float b = beam_at(U, delays + i * n_stations * n_phases,
                              weights + i * n_stations, t, n_samples,
                              n_stations, n_phases, out_of_bounds);
            if (b > best) {
                best = b;
                best_i = (int32_t)i;
            }
        }
        if (best > -FLT_MAX)
            beam_max[t] = best;
        argmax[t] = best_i;
    }
}

/* Max/argmax at selected samples only (same rule as bpo_beamform_max), for
 * checking full-size runs at a sample of times. */
void bpo_beamform_max_at(const float *U, const int32_t *delays, const float *weights,
                         size_t n_samples, size_t n_sources, size_t n_stations,
                         size_t n_phases, int out_of_bounds, int num_threads,
                         const int64_t *times, size_t n_times, float *beam_max,
                         int32_t *argmax, int32_t *minmax_scratch)
{
    bpo_minmax(delays, weights, n_sources, n_stations, n_phases, num_threads,
               minmax_scratch);
    set_threads(num_threads);
    for (size_t k = 0; k < n_times; k++) {
        long long t = times[k];
        float best = -FLT_MAX;
        long long best_i = 0;
#pragma omp parallel
        {
            float lbest = -FLT_MAX;
            long long li = 0;
#pragma omp for schedule(static)
            for (long long i = 0; i < (long long)n_sources; i++) {
                if (!out_of_bounds && !strict_valid(minmax_scratch + 2 * i, t, n_samples))
                    continue;
                float b = beam_at(U, delays + (size_t)i * n_stations * n_phases,
                                  weights + (size_t)i * n_stations, t, n_samples,
                                  n_stations, n_phases, out_of_bounds);
                if (b > lbest) { lbest = b; li = i; }
            }
#pragma omp critical
            {
                /* merge: larger value wins, lower index on ties */
                if (lbest > best || (lbest == best && lbest > -FLT_MAX && li < best_i)) {
                    best = lbest;
                    best_i = li;
                }
            }
        }
        beam_max[k] = best > -FLT_MAX ? best : 0.0f;
        argmax[k] = best > -FLT_MAX ? (int32_t)best_i : 0;
    }
}

/* Differential mode: beamform.c:338-394.  One value per source, the beam at
 * the zero lag t0 = (T - 1) / 2 of inter-station correlations, strict rule. */
void bpo_beamform_differential(const float *U, const int32_t *delays,
                               const float *weights, size_t n_samples,
                               size_t n_sources, size_t n_stations,
                               size_t n_phases, int num_threads, float *beam)
{
    set_threads(num_threads);
    long long t0 = ((long long)n_samples - 1) / 2;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n_sources; i++) {
        const int32_t *d = delays + (size_t)i * n_stations * n_phases;
        const float *w = weights + (size_t)i * n_stations;
        int32_t mm[2] = {INT_MAX, INT_MIN};
        for (size_t s = 0; s < n_stations; s++) {
            if (w[s] == 0.0f) continue;
            for (size_t p = 0; p < n_phases; p++) {
                if (d[s * n_phases + p] < mm[0]) mm[0] = d[s * n_phases + p];
                if (d[s * n_phases + p] > mm[1]) mm[1] = d[s * n_phases + p];
            }
        }
        if (!strict_valid(mm, t0, n_samples))
            continue;
        beam[i] = beam_at(U, d, w, t0, n_samples, n_stations, n_phases, 0);
    }
}
