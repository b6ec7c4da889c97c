/*
 * ffa64_oracle.c -- FP64 restatement of the FFA search of one time series
 * (TEST INFRASTRUCTURE: the precision reference the FP32 paths are measured
 * against; gaffa_oracle.c is the bit-exact FP32 restatement).
 *
 * It follows the reference's algorithm step for step but carries every value
 * in double:
 *   downsample_weighted_sum_cpu   time_series.cpp:140-174 (weights and sums)
 *   transform_recursive / merge   ffa.cpp:110-195 (the head/tail split and the
 *                                 row-index arithmetic are kept verbatim,
 *                                 including its float scale: it selects which
 *                                 rows combine, not a value)
 *   emit_transform_rows           ffa.cpp:203-251 (rows_eval rows of the root)
 *   make_boxcar_trials            ffa_detection.cpp:60-80 (height, baseline)
 *   fill_circular_prefix / scan   ffa_detection.cpp:126-170
 *   ffa_task_stdnoise             ffa_detection.cpp:256-264
 * For every evaluated row and every width it reports the best boxcar S/N and
 * the first phase attaining it, with no threshold.
 */
#include "gaffa_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ffa.cpp:110-125: out[i] = lhs[i] + rhs[(i + shift) % n] */
static void rollback_add64(const double* lhs, const double* rhs, uint64_t n, uint64_t shift, double* out) {
  const uint64_t r = shift % n;
  for (uint64_t i = 0; i < n - r; ++i) out[i] = lhs[i] + rhs[i + r];
  for (uint64_t i = 0; i < r; ++i) out[n - r + i] = lhs[n - r + i] + rhs[i];
}

/* ffa.cpp:153-171 */
static void merge_row64(const double* head, uint64_t head_rows, const double* tail, uint64_t tail_rows,
                        uint64_t out_rows, uint64_t shift, uint64_t bins, double* out) {
  const float hsc = (float)(head_rows - 1) / (float)(out_rows - 1);
  const float tsc = (float)(tail_rows - 1) / (float)(out_rows - 1);
  const uint64_t hs = (uint64_t)(hsc * (float)shift + 0.5f);
  const uint64_t ts = (uint64_t)(tsc * (float)shift + 0.5f);
  const uint64_t comp = shift - (hs + ts);
  rollback_add64(head + hs * bins, tail + ts * bins, bins, hs + comp, out);
}

/* ffa.cpp:173-195 */
static void transform_rec64(const double* in, uint64_t rows, uint64_t bins, double* scratch, double* out) {
  if (rows == 1) {
    memcpy(out, in, sizeof(double) * bins);
    return;
  }
  if (rows == 2) {
    for (uint64_t i = 0; i < bins; ++i) out[i] = in[i] + in[bins + i];
    rollback_add64(in, in + bins, bins, 1, out + bins);
    return;
  }
  const uint64_t h = rows / 2, t = rows - h;
  transform_rec64(in, h, bins, out, scratch);
  transform_rec64(in + h * bins, t, bins, out + h * bins, scratch + h * bins);
  for (uint64_t s = 0; s < rows; ++s) merge_row64(scratch, h, scratch + h * bins, t, rows, s, bins, out + s * bins);
}

int gfo64_ffa_transform(const double* in, uint64_t rows, uint64_t bins, double* out) {
  if (rows == 0 || bins <= 1) return GFO_EINVAL;
  double* scratch = (double*)malloc(sizeof(double) * rows * bins);
  if (!scratch) return GFO_ENOMEM;
  transform_rec64(in, rows, bins, scratch, out);
  free(scratch);
  return GFO_OK;
}

/* time_series.cpp:140-174 in double: out[k] = w0 x[first] + sum x[first+1 .. last-1] + w1 x[last] */
int gfo64_downsample(const float* in, uint64_t n, double factor, double* out, uint64_t* nout) {
  if (!(factor > 1.0) || !isfinite(factor) || factor > (double)n) return GFO_EINVAL;
  const uint64_t m = (uint64_t)floor((double)n / factor);
  const double last_index = (double)(n - 1);
  for (uint64_t k = 0; k < m; ++k) {
    const double start = (double)k * factor;
    const double end = start + factor;
    const uint64_t first = (uint64_t)floor(start);
    const double fe = floor(end);
    const uint64_t last = (uint64_t)(fe < last_index ? fe : last_index);
    double sum = ((double)(first + 1) - start) * (double)in[first];
    for (uint64_t i = first + 1; i < last; ++i) sum += (double)in[i];
    sum += (end - (double)last) * (double)in[last];
    out[k] = sum;
  }
  *nout = m;
  return GFO_OK;
}

/* ffa_detection.cpp:126-170 and :60-80 in double, for one row and every
 * width: best S/N and the first phase attaining the best boxcar sum */
static void row_snr64(const double* prof, uint64_t bins, const uint64_t* widths, uint64_t nw, uint64_t max_width,
                      double stdnoise, double* cp, double* snr, uint64_t* phase) {
  cp[0] = 0.0;
  for (uint64_t i = 0; i < bins; ++i) cp[i + 1] = cp[i] + prof[i];
  for (uint64_t i = 0; i < max_width; ++i) cp[bins + i + 1] = cp[bins + i] + prof[i];
  const double psum = cp[bins];
  const double b = (double)bins;
  for (uint64_t k = 0; k < nw; ++k) {
    const double w = (double)widths[k];
    const double h = sqrt((b - w) / (b * w));
    const double beta = w / (b - w) * h;
    double best = -INFINITY;
    uint64_t best_ph = 0;
    for (uint64_t ph = 0; ph < bins; ++ph) {
      const double s = cp[ph + widths[k]] - cp[ph];
      if (s > best) {
        best = s;
        best_ph = ph;
      }
    }
    snr[k] = ((h + beta) * best - beta * psum) / stdnoise;
    phase[k] = best_ph;
  }
}

/* One task of the plan on a normalised series: S/N [rows_eval][nw] and the
 * phases, everything in double from the float series on. */
int gfo64_ffa_task_snr(const float* series, uint64_t n, const gfo_ffa_task* task, const uint64_t* widths,
                       uint64_t nw, double* snr, uint64_t* phase) {
  if (!series || !task || !widths || nw == 0 || !snr || !phase) return GFO_EINVAL;
  const uint64_t rows = task->rows, bins = task->bins, rows_eval = task->rows_eval;
  if (rows == 0 || bins <= 1 || rows_eval == 0 || rows_eval > rows) return GFO_EINVAL;
  uint64_t max_width = 0;
  for (uint64_t k = 0; k < nw; ++k) {
    if (widths[k] == 0 || widths[k] >= bins) return GFO_EINVAL;
    if (widths[k] > max_width) max_width = widths[k];
  }
  double* prepared = (double*)malloc(sizeof(double) * (n > rows * bins ? n : rows * bins));
  double* transform = (double*)malloc(sizeof(double) * rows * bins);
  double* cp = (double*)malloc(sizeof(double) * (bins + max_width + 1));
  int rc = GFO_OK;
  if (!prepared || !transform || !cp) rc = GFO_ENOMEM;
  double var = 1.0;
  if (rc == GFO_OK) {
    if (task->downsample_factor == 1.0) {
      for (uint64_t i = 0; i < rows * bins; ++i) prepared[i] = (double)series[i];
    } else {
      uint64_t m = 0;
      rc = gfo64_downsample(series, n, task->downsample_factor, prepared, &m);
      if (rc == GFO_OK && m < rows * bins) rc = GFO_EINVAL;
      /* time_series.cpp:124-138, the riptide noise model */
      if (rc == GFO_OK) rc = gfo_downsampled_variance(n, task->downsample_factor, &var);
    }
  }
  if (rc == GFO_OK) rc = gfo64_ffa_transform(prepared, rows, bins, transform);
  if (rc == GFO_OK) {
    const double stdnoise = sqrt((double)rows * var);
    for (uint64_t s = 0; s < rows_eval; ++s)
      row_snr64(transform + s * bins, bins, widths, nw, max_width, stdnoise, cp, snr + s * nw, phase + s * nw);
  }
  free(prepared);
  free(transform);
  free(cp);
  return rc;
}
