/*
 * gaffa_oracle.c -- CPU restatement of gaffa's search hot path (TEST
 * INFRASTRUCTURE: the checker for the CUDA product, never part of it).
 *
 * Each function cites the reference source it restates (lintian233/gaffa,
 * paths relative to that project).  Operation order follows the reference so
 * that float/double results are bit-identical; build with -ffp-contract=off
 * (oracle/Makefile) so the compiler cannot fuse multiply-adds.
 */
#include "gaffa_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static _Thread_local char g_error[256];

static int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof g_error, fmt, ap);
  va_end(ap);
  return code;
}

const char* gfo_last_error(void) { return g_error; }
void gfo_free(void* p) { free(p); }

/* ------------------------------------------------------------------------ */
/* dedispersion                                                              */
/* ------------------------------------------------------------------------ */

/* internal/dedispersion_delay.h:37-50 dedispersion_delay_bins.  The constant
 * 4148.808 is in s MHz^2 (named dispersion_delay_ms in the reference). */
int32_t gfo_delay_bins(double dm, double f, double fref, double tsamp) {
  const double f2 = f * f;
  const double ref2 = fref * fref;
  const double delay = 4148.808 * dm * (1.0 / f2 - 1.0 / ref2);
  const double bins = round(delay / tsamp);
  return (int32_t)bins;
}

static int validate_multi(uint64_t nsamples, uint64_t nchans,
                          const double* freq, double dm_low, double dm_step,
                          uint64_t ndm, double fref, double tsamp,
                          uint64_t cb, uint64_t ce) {
  /* dedispersion.cpp:49-130 validate_samples / validate_multi_plan */
  if (nsamples == 0) return fail(GFO_EINVAL, "dedispersion requires at least one sample");
  if (nchans == 0) return fail(GFO_EINVAL, "dedispersion requires at least one channel");
  for (uint64_t c = 0; c < nchans; ++c)
    if (!isfinite(freq[c]) || !(freq[c] > 0.0))
      return fail(GFO_EINVAL, "frequency values must be finite and positive");
  if (!isfinite(fref) || !(fref > 0.0)) return fail(GFO_EINVAL, "reference frequency must be positive");
  if (!isfinite(tsamp) || !(tsamp > 0.0)) return fail(GFO_EINVAL, "tsamp must be positive");
  if (!isfinite(dm_low) || dm_low < 0.0) return fail(GFO_EINVAL, "dm_low must be finite and non-negative");
  if (ndm == 0) return fail(GFO_EINVAL, "dedispersion requires at least one DM");
  if (!isfinite(dm_step) || !(dm_step > 0.0)) return fail(GFO_EINVAL, "dm_step must be positive");
  if (cb >= ce) return fail(GFO_EINVAL, "channel range must be non-empty");
  if (ce > nchans) return fail(GFO_EINVAL, "channel range exceeds sample channel count");
  for (uint64_t c = cb; c < ce; ++c)
    if (freq[c] > fref)
      return fail(GFO_EINVAL, "dedispersion requires selected frequencies <= reference frequency");
  return GFO_OK;
}

/* internal/dedispersion_delay.h:95-110,129-139 multi_dm_max_delay +
 * valid_output_nsamples */
int gfo_multi_dm_output_nsamples(const double* freq, uint64_t nchans,
                                 uint64_t nsamples, double dm_low, double dm_step,
                                 uint64_t ndm, double fref, double tsamp,
                                 uint64_t cb, uint64_t ce, uint64_t* nout) {
  int rc = validate_multi(nsamples, nchans, freq, dm_low, dm_step, ndm, fref,
                          tsamp, cb, ce);
  if (rc) return rc;
  const double max_dm = dm_low + (double)(ndm - 1) * dm_step;
  double fmin = freq[cb];
  for (uint64_t c = cb + 1; c < ce; ++c)
    if (freq[c] < fmin) fmin = freq[c];
  const int32_t max_delay = gfo_delay_bins(max_dm, fmin, fref, tsamp);
  if (max_delay < 0) return fail(GFO_EINVAL, "dedispersion requires non-negative delays");
  if ((uint64_t)max_delay >= nsamples)
    return fail(GFO_EINVAL, "dedispersion valid output range is empty");
  *nout = nsamples - (uint64_t)max_delay;
  return GFO_OK;
}

/* dedispersion.cpp:197-215 direct_sum_at, :291-329 dedisperse_multi_dm_cpu */
int gfo_dedisperse_multi_dm_u8(const uint8_t* in, uint64_t nsamples, uint64_t nchans,
                               const double* freq, double dm_low, double dm_step,
                               uint64_t ndm, double fref, double tsamp, uint64_t cb,
                               uint64_t ce, uint32_t* out) {
  uint64_t nout = 0;
  int rc = gfo_multi_dm_output_nsamples(freq, nchans, nsamples, dm_low, dm_step,
                                        ndm, fref, tsamp, cb, ce, &nout);
  if (rc) return rc;
  const uint64_t nc = ce - cb;
  int32_t* delays = (int32_t*)malloc(sizeof(int32_t) * ndm * nc);
  if (!delays) return fail(GFO_ENOMEM, "out of memory");
  for (uint64_t d = 0; d < ndm; ++d) {
    const double dm = dm_low + (double)d * dm_step;
    for (uint64_t o = 0; o < nc; ++o)
      delays[d * nc + o] = gfo_delay_bins(dm, freq[cb + o], fref, tsamp);
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t d = 0; d < (int64_t)ndm; ++d) {
    for (int64_t t = 0; t < (int64_t)nout; ++t) {
      const int32_t* dd = delays + (uint64_t)d * nc;
      uint32_t sum = 0;
      for (uint64_t o = 0; o < nc; ++o) {
        const int64_t st = t + dd[o];
        if (st >= 0 && st < (int64_t)nsamples)
          sum += in[(uint64_t)st * nchans + cb + o];
      }
      out[(uint64_t)d * nout + (uint64_t)t] = sum;
    }
  }
  free(delays);
  return GFO_OK;
}

/* dedispersion.cpp:141-189 subband delay tables, :331-453 two-stage sum */
int gfo_dedisperse_subband_u8(const uint8_t* in, uint64_t nsamples, uint64_t nchans,
                              const double* freq, double dm_low, double dm_step,
                              uint64_t ndm, double fref, double tsamp, uint64_t cb,
                              uint64_t ce, uint64_t subband_channels,
                              uint64_t ndm_per_nominal, uint32_t* out) {
  uint64_t nout = 0;
  int rc = gfo_multi_dm_output_nsamples(freq, nchans, nsamples, dm_low, dm_step,
                                        ndm, fref, tsamp, cb, ce, &nout);
  if (rc) return rc;
  if (subband_channels == 0) return fail(GFO_EINVAL, "subband_channels must be positive");
  if (ndm_per_nominal == 0) return fail(GFO_EINVAL, "ndm_per_nominal must be positive");
  const uint64_t nc = ce - cb;
  const uint64_t nsb = nc / subband_channels + (nc % subband_channels != 0);
  const uint64_t nnom = ndm / ndm_per_nominal + (ndm % ndm_per_nominal != 0);
  uint64_t* sb_begin = (uint64_t*)malloc(sizeof(uint64_t) * nsb);
  uint64_t* sb_end = (uint64_t*)malloc(sizeof(uint64_t) * nsb);
  double* sb_freq = (double*)malloc(sizeof(double) * nsb);
  int32_t* coarse = (int32_t*)malloc(sizeof(int32_t) * nnom * nc);
  int32_t* resid = (int32_t*)malloc(sizeof(int32_t) * ndm * nsb);
  uint32_t* inter = (uint32_t*)malloc(sizeof(uint32_t) * nnom * nsb * nsamples);
  if (!sb_begin || !sb_end || !sb_freq || !coarse || !resid || !inter) {
    free(sb_begin); free(sb_end); free(sb_freq); free(coarse); free(resid); free(inter);
    return fail(GFO_ENOMEM, "out of memory");
  }
  for (uint64_t b = 0; b < nsb; ++b) {
    const uint64_t begin = cb + b * subband_channels;
    const uint64_t end = begin + subband_channels < ce ? begin + subband_channels : ce;
    sb_begin[b] = begin;
    sb_end[b] = end;
    sb_freq[b] = freq[(begin + end - 1) / 2];
  }
  for (uint64_t n = 0; n < nnom; ++n) {
    const double nominal_dm = dm_low + (double)(n * ndm_per_nominal) * dm_step;
    for (uint64_t o = 0; o < nc; ++o)
      coarse[n * nc + o] = gfo_delay_bins(nominal_dm, freq[cb + o], fref, tsamp);
  }
  for (uint64_t d = 0; d < ndm; ++d) {
    const uint64_t n = d / ndm_per_nominal;
    const double nominal_dm = dm_low + (double)(n * ndm_per_nominal) * dm_step;
    const double final_dm = dm_low + (double)d * dm_step;
    for (uint64_t b = 0; b < nsb; ++b)
      resid[d * nsb + b] = gfo_delay_bins(final_dm - nominal_dm, sb_freq[b], fref, tsamp);
  }
  const uint64_t inter_stride = nsb * nsamples;
#pragma omp parallel for collapse(3) schedule(static)
  for (int64_t n = 0; n < (int64_t)nnom; ++n)
    for (int64_t b = 0; b < (int64_t)nsb; ++b)
      for (int64_t t = 0; t < (int64_t)nsamples; ++t) {
        const int32_t* nd = coarse + (uint64_t)n * nc;
        uint32_t sum = 0;
        for (uint64_t c = sb_begin[b]; c < sb_end[b]; ++c) {
          const int64_t st = t + nd[c - cb];
          if (st >= 0 && st < (int64_t)nsamples) sum += in[(uint64_t)st * nchans + c];
        }
        inter[(uint64_t)n * inter_stride + (uint64_t)b * nsamples + (uint64_t)t] = sum;
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t d = 0; d < (int64_t)ndm; ++d)
    for (int64_t t = 0; t < (int64_t)nout; ++t) {
      const uint64_t n = (uint64_t)d / ndm_per_nominal;
      uint32_t sum = 0;
      for (uint64_t b = 0; b < nsb; ++b) {
        const int64_t st = t + resid[(uint64_t)d * nsb + b];
        if (st >= 0 && st < (int64_t)nsamples)
          sum += inter[n * inter_stride + b * nsamples + (uint64_t)st];
      }
      out[(uint64_t)d * nout + (uint64_t)t] = sum;
    }
  free(sb_begin); free(sb_end); free(sb_freq); free(coarse); free(resid); free(inter);
  return GFO_OK;
}

void gfo_unpack_2bit(const uint8_t* packed, uint64_t nsamples, uint64_t nchans,
                     uint8_t* out) {
  const uint64_t row = nchans / 4;
  for (uint64_t t = 0; t < nsamples; ++t)
    for (uint64_t c = 0; c < nchans; ++c)
      out[t * nchans + c] = (uint8_t)((packed[t * row + c / 4] >> (2 * (c % 4))) & 3u);
}

/* ------------------------------------------------------------------------ */
/* time series                                                               */
/* ------------------------------------------------------------------------ */

/* time_series.cpp:14-23 validate_downsample_factor, :118-122 downsampled_size */
static int check_factor(uint64_t n, double factor) {
  if (n == 0) return fail(GFO_EINVAL, "time series must not be empty");
  if (!isfinite(factor) || factor <= 1.0 || factor > (double)n)
    return fail(GFO_EINVAL, "downsample factor must satisfy 1 < factor <= nsamples");
  return GFO_OK;
}

int gfo_downsampled_size(uint64_t n, double factor, uint64_t* out) {
  int rc = check_factor(n, factor);
  if (rc) return rc;
  *out = (uint64_t)floor((double)n / factor);
  return GFO_OK;
}

/* time_series.cpp:124-138 downsampled_variance (riptide noise model) */
int gfo_downsampled_variance(uint64_t n, double factor, double* out) {
  uint64_t m = 0;
  int rc = gfo_downsampled_size(n, factor, &m);
  if (rc) return rc;
  const double whole = floor(factor);
  const double fractional = factor - whole;
  const double span = (double)m * fractional;
  if (span > 1.0) {
    *out = factor - 1.0 / 3.0;
    return GFO_OK;
  }
  *out = pow(whole - 1.0, 2.0) + (2.0 / 3.0) * pow(span, 2.0) - span + 1.0;
  return GFO_OK;
}

/* time_series.cpp:140-174 downsample_weighted_sum_cpu */
int gfo_downsample_weighted_sum(const float* in, uint64_t n, double factor,
                                float* out) {
  uint64_t m = 0;
  int rc = gfo_downsampled_size(n, factor, &m);
  if (rc) return rc;
  const double last_index = (double)(n - 1);
  for (uint64_t k = 0; k < m; ++k) {
    const double start = (double)k * factor;
    const double end = start + factor;
    const uint64_t first = (uint64_t)floor(start);
    const double fe = floor(end);
    const uint64_t last = (uint64_t)(fe < last_index ? fe : last_index);
    const float w0 = (float)((double)(first + 1) - start);
    const float w1 = (float)(end - (double)last);
    float sum = w0 * in[first];
    for (uint64_t i = first + 1; i < last; ++i) sum += in[i];
    sum += w1 * in[last];
    out[k] = sum;
  }
  return GFO_OK;
}

/* time_series.cpp:50-104 time_series_stats_cpu + normalise_cpu */
int gfo_normalise(const float* in, uint64_t n, int reject_constant, float* out) {
  if (n == 0) return fail(GFO_EINVAL, "normalise input must not be empty");
  for (uint64_t i = 0; i < n; ++i)
    if (!isfinite(in[i])) return fail(GFO_EINVAL, "time series samples must be finite");
  double sum = 0.0, sum_sq = 0.0;
  for (uint64_t i = 0; i < n; ++i) {
    const double s = (double)in[i];
    sum += s;
    sum_sq += s * s;
  }
  const double count = (double)n;
  const double mean = sum / count;
  double var = sum_sq / count - mean * mean;
  if (var < 0.0 && var > -1.0e-12) var = 0.0;
  if (var < 0.0 || !isfinite(var))
    return fail(GFO_EINVAL, "time series variance must be finite and >= 0");
  const double sd = sqrt(var);
  if (!(sd > 0.0) || !isfinite(sd)) {
    if (reject_constant)
      return fail(GFO_EINVAL, "normalise input standard deviation must be finite and > 0");
    for (uint64_t i = 0; i < n; ++i) out[i] = 0.0f;
    return GFO_OK;
  }
  const double scale = 1.0 / sd;
  for (uint64_t i = 0; i < n; ++i) out[i] = (float)(((double)in[i] - mean) * scale);
  return GFO_OK;
}

/* ------------------------------------------------------------------------ */
/* preprocessing                                                             */
/* ------------------------------------------------------------------------ */

/* preprocessing.cpp:164-188 running_median_window_seconds */
int gfo_running_median_window(double seconds, double tsamp, uint64_t* w) {
  if (!(seconds > 0.0) || !isfinite(seconds))
    return fail(GFO_EINVAL, "running median window_seconds must be finite and > 0");
  if (!(tsamp > 0.0) || !isfinite(tsamp))
    return fail(GFO_EINVAL, "running median tsamp must be finite and > 0");
  const double r = round(seconds / tsamp);
  if (!isfinite(r) || r > 18446744073709551615.0 - 1.0)
    return fail(GFO_EINVAL, "running median window_samples is too large");
  uint64_t ws = (uint64_t)(r > 1.0 ? r : 1.0);
  if (ws % 2 == 0) ++ws;
  *w = ws;
  return GFO_OK;
}

/* Upper median of w values (w odd): std::nth_element at w/2 selects the
 * element that a full sort puts at index w/2 (preprocessing.cpp:44-51). */
static int cmp_float(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

/* preprocessing.cpp:53-76 exact_running_median_cpu (edge-value padding) */
static int exact_running_median(const float* in, uint64_t n, uint64_t w, float* out) {
  if (w >= n) return fail(GFO_EINVAL, "running median detrend window_samples must be < input size");
  const uint64_t half = w / 2;
  float* padded = (float*)malloc(sizeof(float) * (n + 2 * half));
  float* win = (float*)malloc(sizeof(float) * w);
  if (!padded || !win) { free(padded); free(win); return fail(GFO_ENOMEM, "out of memory"); }
  for (uint64_t i = 0; i < half; ++i) padded[i] = in[0];
  memcpy(padded + half, in, sizeof(float) * n);
  for (uint64_t i = 0; i < half; ++i) padded[half + n + i] = in[n - 1];
  for (uint64_t i = 0; i < n; ++i) {
    memcpy(win, padded + i, sizeof(float) * w);
    qsort(win, w, sizeof(float), cmp_float);
    out[i] = win[w / 2];
  }
  free(padded);
  free(win);
  return GFO_OK;
}

/* preprocessing.cpp:212-231 detrend_running_median_cpu with
 * :124-145 fast_running_median_cpu, :78-92 mean_scrunch_cpu,
 * :94-122 interpolate_scrunched_median */
int gfo_detrend_running_median(const float* in, uint64_t n, uint64_t window,
                               uint64_t min_points, float* out) {
  if (window == 0 || window % 2 == 0)
    return fail(GFO_EINVAL, "running median detrend window_samples must be odd and > 0");
  if (min_points == 0 || min_points % 2 == 0)
    return fail(GFO_EINVAL, "running median detrend min_points must be odd and > 0");
  if (n == 0) return fail(GFO_EINVAL, "running median detrend input must not be empty");
  for (uint64_t i = 0; i < n; ++i)
    if (!isfinite(in[i])) return fail(GFO_EINVAL, "running median detrend input samples must be finite");
  float* median = (float*)malloc(sizeof(float) * n);
  if (!median) return fail(GFO_ENOMEM, "out of memory");
  double sf = (double)window / (double)min_points;
  uint64_t scrunch = (uint64_t)sf;
  if (scrunch < 1) scrunch = 1;
  int rc = GFO_OK;
  if (scrunch == 1) {
    rc = exact_running_median(in, n, window, median);
  } else {
    const uint64_t m = n / scrunch;
    if (m <= min_points) {
      free(median);
      return fail(GFO_EINVAL, "running median detrend low-resolution sample count must be > min_points");
    }
    float* low = (float*)malloc(sizeof(float) * m);
    float* lowmed = (float*)malloc(sizeof(float) * m);
    if (!low || !lowmed) { free(low); free(lowmed); free(median); return fail(GFO_ENOMEM, "out of memory"); }
    for (uint64_t k = 0; k < m; ++k) {
      double s = 0.0;
      for (uint64_t i = 0; i < scrunch; ++i) s += (double)in[k * scrunch + i];
      low[k] = (float)(s / (double)scrunch);
    }
    rc = exact_running_median(low, m, min_points, lowmed);
    if (rc == GFO_OK) {
      const double offset = 0.5 * (double)(scrunch - 1);
      for (uint64_t i = 0; i < n; ++i) {
        const double pos = ((double)i - offset) / (double)scrunch;
        if (pos <= 0.0) { median[i] = lowmed[0]; continue; }
        const uint64_t lower = (uint64_t)floor(pos);
        if (lower >= m - 1) { median[i] = lowmed[m - 1]; continue; }
        const double frac = pos - (double)lower;
        median[i] = (float)((1.0 - frac) * (double)lowmed[lower] + frac * (double)lowmed[lower + 1]);
      }
    }
    free(low);
    free(lowmed);
  }
  if (rc == GFO_OK)
    for (uint64_t i = 0; i < n; ++i) out[i] = in[i] - median[i];
  free(median);
  return rc;
}

/* preprocessing.cpp:190-210 make_riptide_preprocess_plan followed by
 * :241-257 preprocess_time_series_cpu (steps applied in order) */
int gfo_preprocess_riptide(float* data, uint64_t n, double tsamp,
                           const gfo_preprocess_options* o) {
  if (n == 0) return fail(GFO_EINVAL, "time series data must not be empty");
  if (!(tsamp > 0.0) || !isfinite(tsamp)) return fail(GFO_EINVAL, "time series tsamp must be finite and > 0");
  uint64_t window = 0;
  int rc = gfo_running_median_window(o->window_seconds, tsamp, &window);
  if (rc) return rc;
  float* tmp = (float*)malloc(sizeof(float) * n);
  if (!tmp) return fail(GFO_ENOMEM, "out of memory");
  rc = gfo_detrend_running_median(data, n, window, o->min_points, tmp);
  if (rc == GFO_OK) {
    if (o->normalise) rc = gfo_normalise(tmp, n, o->reject_constant, data);
    else memcpy(data, tmp, sizeof(float) * n);
  }
  free(tmp);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* FFA plan (ffa_plan.cpp)                                                   */
/* ------------------------------------------------------------------------ */

static uint64_t ceil_shift(uint64_t rows, uint64_t bins, double pmax) {
  /* ffa_plan.cpp:47-54 */
  const double v = (double)bins * ((double)rows - 1.0) * (1.0 - (double)bins / pmax);
  return (uint64_t)ceil(v);
}

static double evaluated_period_end(double eff, uint64_t bins, uint64_t rows,
                                   uint64_t rows_eval) {
  /* ffa_plan.cpp:74-86 */
  if (rows == 1 || rows_eval == 1) return eff * (double)bins;
  const double b = (double)bins;
  const double shift = (double)(rows_eval - 1) / (double)(rows - 1);
  return eff * b * b / (b - shift);
}

/* ffa_plan.cpp:18-38 validation, :56-72 widths, :90-170 tasks */
int gfo_make_riptide_ffa_plan(uint64_t nsamples, double tsamp,
                              const gfo_plan_options* o, gfo_ffa_task** tasks_out,
                              uint64_t* ntasks_out, uint64_t** widths_out,
                              uint64_t* nwidths_out) {
  if (!(nsamples > 0)) return fail(GFO_EINVAL, "FFA plan nsamples must be > 0");
  if (!(tsamp > 0.0)) return fail(GFO_EINVAL, "FFA plan tsamp must be > 0");
  if (!(o->period_min > 0.0)) return fail(GFO_EINVAL, "FFA plan period_min must be > 0");
  if (!(o->period_max > o->period_min)) return fail(GFO_EINVAL, "FFA plan period_max must be > period_min");
  if (!(o->bins_min > 1)) return fail(GFO_EINVAL, "FFA plan bins_min must be > 1");
  if (!(o->bins_max >= o->bins_min)) return fail(GFO_EINVAL, "FFA plan bins_max must be >= bins_min");
  if (!(o->min_periods > 0)) return fail(GFO_EINVAL, "FFA plan min_periods must be > 0");
  if (!(o->duty_cycle_max > 0.0 && o->duty_cycle_max < 1.0)) return fail(GFO_EINVAL, "FFA plan duty_cycle_max must be in (0, 1)");
  if (!(o->width_trial_spacing > 1.0)) return fail(GFO_EINVAL, "FFA plan width_trial_spacing must be > 1");
  if (!(o->max_tasks > 0)) return fail(GFO_EINVAL, "FFA plan max_tasks must be > 0");
  if (!(o->period_min >= tsamp * (double)o->bins_min)) return fail(GFO_EINVAL, "FFA plan period_min must be >= tsamp * bins_min");

  const double tobs = (double)nsamples * tsamp;
  const double cap = tobs / (double)o->min_periods;
  const double pmax = o->period_max < cap ? o->period_max : cap;
  if (pmax <= o->period_min) return fail(GFO_EINVAL, "FFA search range is empty after min_periods cap");

  /* widths */
  uint64_t wmax = (uint64_t)floor(o->duty_cycle_max * (double)o->bins_min);
  if (wmax < 1) wmax = 1;
  uint64_t wcap = 16, nw = 0;
  uint64_t* widths = (uint64_t*)malloc(sizeof(uint64_t) * wcap);
  if (!widths) return fail(GFO_ENOMEM, "out of memory");
  for (uint64_t w = 1; w <= wmax;) {
    if (nw == wcap) {
      wcap *= 2;
      uint64_t* nwp = (uint64_t*)realloc(widths, sizeof(uint64_t) * wcap);
      if (!nwp) { free(widths); return fail(GFO_ENOMEM, "out of memory"); }
      widths = nwp;
    }
    widths[nw++] = w;
    const uint64_t scaled = (uint64_t)floor(o->width_trial_spacing * (double)w);
    w = (w + 1 > scaled) ? w + 1 : scaled;
  }

  const double f0 = o->period_min / (tsamp * (double)o->bins_min);
  const double growth = ((double)o->bins_max + 1.0) / (double)o->bins_min;
  const uint64_t cycles = (uint64_t)ceil(log(pmax / o->period_min) / log(growth));

  uint64_t tcap = 64, nt = 0;
  gfo_ffa_task* tasks = (gfo_ffa_task*)malloc(sizeof(gfo_ffa_task) * tcap);
  if (!tasks) { free(widths); return fail(GFO_ENOMEM, "out of memory"); }
  for (uint64_t cycle = 0; cycle < cycles; ++cycle) {
    const double factor = f0 * pow(growth, (double)cycle);
    const double eff = factor * tsamp;
    uint64_t prepared;
    if (factor == 1.0) {
      prepared = nsamples;
    } else {
      int rc = gfo_downsampled_size(nsamples, factor, &prepared);
      if (rc) { free(widths); free(tasks); return rc; }
    }
    const double pmax_samples = pmax / eff;
    uint64_t stop = o->bins_max;
    if (prepared < stop) stop = prepared;
    const uint64_t fl = (uint64_t)floor(pmax_samples);
    if (fl < stop) stop = fl;
    if (stop < o->bins_min) continue;
    for (uint64_t bins = o->bins_min; bins <= stop; ++bins) {
      const uint64_t rows = prepared / bins;
      if (rows < o->min_periods) continue;
      const double pceil = pmax_samples < (double)bins + 1.0 ? pmax_samples : (double)bins + 1.0;
      uint64_t rows_eval = ceil_shift(rows, bins, pceil);
      if (rows < rows_eval) rows_eval = rows;
      if (rows_eval == 0) continue;
      if (nt >= o->max_tasks) {
        free(widths); free(tasks);
        return fail(GFO_ERUNTIME, "FFA search plan exceeds max_tasks");
      }
      if (nt == tcap) {
        tcap *= 2;
        gfo_ffa_task* ntp = (gfo_ffa_task*)realloc(tasks, sizeof(gfo_ffa_task) * tcap);
        if (!ntp) { free(widths); free(tasks); return fail(GFO_ENOMEM, "out of memory"); }
        tasks = ntp;
      }
      gfo_ffa_task* t = &tasks[nt++];
      t->downsample_factor = factor;
      t->effective_tsamp = eff;
      t->input_nsamples = nsamples;
      t->prepared_nsamples = prepared;
      t->bins = bins;
      t->rows = rows;
      t->rows_eval = rows_eval;
      t->period_begin = eff * (double)bins;
      t->period_end = evaluated_period_end(eff, bins, rows, rows_eval);
    }
  }
  *tasks_out = tasks;
  *ntasks_out = nt;
  *widths_out = widths;
  *nwidths_out = nw;
  return GFO_OK;
}

/* ------------------------------------------------------------------------ */
/* FFA transform (ffa.cpp)                                                   */
/* ------------------------------------------------------------------------ */

/* ffa.cpp:110-125 fused_rollback_add: out[i] = lhs[i] + rhs[(i + shift) % n] */
static void rollback_add(const float* lhs, const float* rhs, uint64_t n,
                         uint64_t shift, float* out) {
  const uint64_t r = shift % n;
  for (uint64_t i = 0; i < n - r; ++i) out[i] = lhs[i] + rhs[i + r];
  for (uint64_t i = 0; i < r; ++i) out[n - r + i] = lhs[n - r + i] + rhs[i];
}

/* ffa.cpp:153-171 merge_row: the float index arithmetic is kept verbatim */
static void merge_row(const float* head, uint64_t head_rows, const float* tail,
                      uint64_t tail_rows, uint64_t out_rows, uint64_t shift,
                      uint64_t bins, float* out) {
  const float hsc = (float)(head_rows - 1) / (float)(out_rows - 1);
  const float tsc = (float)(tail_rows - 1) / (float)(out_rows - 1);
  const uint64_t hs = (uint64_t)(hsc * (float)shift + 0.5f);
  const uint64_t ts = (uint64_t)(tsc * (float)shift + 0.5f);
  const uint64_t comp = shift - (hs + ts);
  rollback_add(head + hs * bins, tail + ts * bins, bins, hs + comp, out);
}

/* ffa.cpp:173-195 transform_recursive (input -> output, scratch as work) */
static void transform_rec(const float* in, uint64_t rows, uint64_t bins,
                          float* scratch, float* out) {
  if (rows == 1) {
    memcpy(out, in, sizeof(float) * bins);
    return;
  }
  if (rows == 2) {
    for (uint64_t i = 0; i < bins; ++i) out[i] = in[i] + in[bins + i];
    rollback_add(in, in + bins, bins, 1, out + bins);
    return;
  }
  const uint64_t h = rows / 2, t = rows - h;
  transform_rec(in, h, bins, out, scratch);
  transform_rec(in + h * bins, t, bins, out + h * bins, scratch + h * bins);
  for (uint64_t s = 0; s < rows; ++s)
    merge_row(scratch, h, scratch + h * bins, t, rows, s, bins, out + s * bins);
}

int gfo_ffa_transform(const float* in, uint64_t rows, uint64_t bins, float* out) {
  if (rows == 0) return fail(GFO_EINVAL, "FFA transform rows must be > 0");
  if (bins <= 1) return fail(GFO_EINVAL, "FFA transform bins must be > 1");
  float* scratch = (float*)malloc(sizeof(float) * rows * bins);
  if (!scratch) return fail(GFO_ENOMEM, "out of memory");
  transform_rec(in, rows, bins, scratch, out);
  free(scratch);
  return GFO_OK;
}

/* ffa.cpp:419-439 ffa_trial_periods */
int gfo_ffa_trial_periods(uint64_t rows, uint64_t bins, double tsamp, double* p) {
  if (rows == 0) return fail(GFO_EINVAL, "FFA transform rows must be > 0");
  if (bins <= 1) return fail(GFO_EINVAL, "FFA transform bins must be > 1");
  if (!(tsamp > 0.0)) return fail(GFO_EINVAL, "FFA sampling interval must be > 0");
  if (rows == 1) {
    p[0] = (double)bins * tsamp;
    return GFO_OK;
  }
  const double b = (double)bins, ms = (double)(rows - 1);
  for (uint64_t s = 0; s < rows; ++s) p[s] = b * b / (b - (double)s / ms) * tsamp;
  return GFO_OK;
}

/* ------------------------------------------------------------------------ */
/* detection (ffa_detection.cpp) and peaks (ffa_peak.cpp)                     */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint64_t width, width_index;
  float height, baseline;
  double duty_cycle;
} boxcar;

/* ffa_detection.cpp:60-80 make_boxcar_trials */
static void make_boxcars(const uint64_t* widths, uint64_t nw, uint64_t bins,
                         boxcar* out) {
  const float bf = (float)bins;
  for (uint64_t i = 0; i < nw; ++i) {
    const float wf = (float)widths[i];
    const float h = sqrtf((bf - wf) / (bf * wf));
    out[i].width = widths[i];
    out[i].width_index = i;
    out[i].height = h;
    out[i].baseline = wf / (bf - wf) * h;
    out[i].duty_cycle = (double)widths[i] / (double)bins;
  }
}

/* ffa_detection.cpp:256-264 ffa_task_stdnoise */
float gfo_ffa_task_stdnoise(const gfo_ffa_task* t) {
  double var = 1.0;
  if (t->downsample_factor != 1.0) gfo_downsampled_variance(t->input_nsamples, t->downsample_factor, &var);
  return (float)sqrt((double)t->rows * var);
}

/* ffa_detection.cpp:115-124 trial_period */
static double trial_period(const gfo_ffa_task* t, uint64_t shift) {
  if (t->rows <= 1) return t->effective_tsamp * (double)t->bins;
  const double b = (double)t->bins;
  return t->effective_tsamp * b * b / (b - (double)shift / (double)(t->rows - 1));
}

typedef struct {
  gfo_peak* data;
  uint64_t n, cap, max_peaks;
} peak_vec;

static int push_peak(peak_vec* v, const gfo_peak* p) {
  /* ffa_detection.cpp:286-295 FfaPeakCollector::add */
  if (v->max_peaks != 0 && v->n >= v->max_peaks)
    return fail(GFO_ERUNTIME, "FFA detection peak count exceeded max_peaks safety guard");
  if (v->n == v->cap) {
    uint64_t nc = v->cap ? v->cap * 2 : 256;
    gfo_peak* nd = (gfo_peak*)realloc(v->data, sizeof(gfo_peak) * nc);
    if (!nd) return fail(GFO_ENOMEM, "out of memory");
    v->data = nd;
    v->cap = nc;
  }
  v->data[v->n++] = *p;
  return GFO_OK;
}

/* ffa_detection.cpp:126-170 fill_circular_prefix + scan_boxcar_peak, and
 * :315-372 detect_ffa_row_cpu, :266-284 make_ffa_peak */
static int detect_row(const float* profile, uint64_t shift, const gfo_ffa_task* task,
                      const boxcar* trials, uint64_t nw, uint64_t max_width,
                      float stdnoise, float thr, float* cp, peak_vec* out) {
  const uint64_t bins = task->bins;
  cp[0] = 0.0f;
  for (uint64_t i = 0; i < bins; ++i) cp[i + 1] = cp[i] + profile[i];
  for (uint64_t i = 0; i < max_width; ++i) cp[bins + i + 1] = cp[bins + i] + profile[i];
  const float psum = cp[bins];
  const float inv = 1.0f / stdnoise;
  for (uint64_t k = 0; k < nw; ++k) {
    const boxcar* tr = &trials[k];
    float best = -INFINITY;
    for (uint64_t ph = 0; ph < bins; ++ph) {
      const float s = cp[ph + tr->width] - cp[ph];
      if (s > best) best = s;
    }
    uint64_t best_phase = 0;
    for (uint64_t ph = 0; ph < bins; ++ph) {
      const float s = cp[ph + tr->width] - cp[ph];
      if (s == best) { best_phase = ph; break; }
    }
    const float snr = ((tr->height + tr->baseline) * best - tr->baseline * psum) * inv;
    if (snr >= thr) {
      gfo_peak p;
      memset(&p, 0, sizeof p);
      p.period = trial_period(task, shift);
      p.frequency = 1.0 / p.period;
      p.width = tr->width;
      p.duty_cycle = tr->duty_cycle;
      p.width_index = tr->width_index;
      p.period_index = shift;
      p.phase = best_phase;
      p.shift = shift;
      p.bins = bins;
      p.snr = snr;
      int rc = push_peak(out, &p);
      if (rc) return rc;
    }
  }
  return GFO_OK;
}

/* ffa_peak.cpp:9-41 is_better_ffa_peak, extended by dm_search.cpp:89-100 */
static int finite_peak(const gfo_peak* p) {
  return isfinite(p->snr) && isfinite(p->period) && isfinite(p->frequency);
}

static int better_ffa(const gfo_peak* l, const gfo_peak* r) {
  const int lf = finite_peak(l), rf = finite_peak(r);
  if (lf != rf) return lf;
  if (l->snr != r->snr) return l->snr > r->snr;
  if (l->period != r->period) return l->period < r->period;
  if (l->frequency != r->frequency) return l->frequency < r->frequency;
  if (l->width != r->width) return l->width < r->width;
  if (l->phase != r->phase) return l->phase < r->phase;
  if (l->shift != r->shift) return l->shift < r->shift;
  return l->bins < r->bins;
}

int gfo_is_better_peak(const gfo_peak* l, const gfo_peak* r) {
  if (better_ffa(l, r)) return 1;
  if (better_ffa(r, l)) return 0;
  if (l->dm_index != r->dm_index) return l->dm_index < r->dm_index;
  return l->dm < r->dm;
}

static int cmp_dm_peak(const void* a, const void* b) {
  const gfo_peak* l = (const gfo_peak*)a;
  const gfo_peak* r = (const gfo_peak*)b;
  if (gfo_is_better_peak(l, r)) return -1;
  if (gfo_is_better_peak(r, l)) return 1;
  return 0;
}

void gfo_sort_dm_peaks(gfo_peak* peaks, uint64_t n) {
  qsort(peaks, n, sizeof(gfo_peak), cmp_dm_peak);
}

static uint64_t max_u64(const uint64_t* v, uint64_t n) {
  uint64_t m = 0;
  for (uint64_t i = 0; i < n; ++i) if (v[i] > m) m = v[i];
  return m;
}

static int validate_widths(const uint64_t* widths, uint64_t nw, uint64_t bins) {
  /* ffa_detection.cpp:47-58 */
  if (nw == 0) return fail(GFO_EINVAL, "FFA detection width trials must not be empty");
  for (uint64_t i = 0; i < nw; ++i)
    if (widths[i] == 0 || widths[i] >= bins)
      return fail(GFO_EINVAL, "FFA detection width trials must satisfy 0 < width < bins");
  return GFO_OK;
}

/* ffa_detection.cpp:374-404 find_ffa_peaks_cpu */
int gfo_find_ffa_peaks(const float* transform, uint64_t rows, uint64_t bins,
                       const gfo_ffa_task* task, const uint64_t* widths,
                       uint64_t nw, float stdnoise, float thr, uint64_t max_peaks,
                       gfo_peak** peaks, uint64_t* npeaks) {
  if (rows == 0) return fail(GFO_EINVAL, "FFA detection rows must be > 0");
  if (bins <= 1) return fail(GFO_EINVAL, "FFA detection bins must be > 1");
  if (task->bins != bins) return fail(GFO_EINVAL, "FFA detection task bins must match shape");
  if (task->rows_eval != rows) return fail(GFO_EINVAL, "FFA detection task rows_eval must match shape");
  if (task->rows < task->rows_eval || task->rows == 0) return fail(GFO_EINVAL, "FFA detection task rows must be >= rows_eval and > 0");
  if (!(stdnoise > 0.0f) || !isfinite(stdnoise)) return fail(GFO_EINVAL, "FFA detection stdnoise must be finite and > 0");
  if (!isfinite(thr)) return fail(GFO_EINVAL, "FFA detection S/N threshold must be finite");
  int rc = validate_widths(widths, nw, bins);
  if (rc) return rc;
  boxcar* trials = (boxcar*)malloc(sizeof(boxcar) * nw);
  const uint64_t mw = max_u64(widths, nw);
  float* cp = (float*)calloc(bins + mw + 1, sizeof(float));
  peak_vec v = {NULL, 0, 0, max_peaks};
  if (!trials || !cp) { free(trials); free(cp); return fail(GFO_ENOMEM, "out of memory"); }
  make_boxcars(widths, nw, bins, trials);
  for (uint64_t s = 0; s < rows && rc == GFO_OK; ++s)
    rc = detect_row(transform + s * bins, s, task, trials, nw, mw, stdnoise, thr, cp, &v);
  free(trials);
  free(cp);
  if (rc) { free(v.data); return rc; }
  gfo_sort_dm_peaks(v.data, v.n);
  *peaks = v.data;
  *npeaks = v.n;
  return GFO_OK;
}

/* ffa_executor.cpp:196-245 validate_task */
static int validate_task(const gfo_ffa_task* t, uint64_t n) {
  if (t->input_nsamples != n) return fail(GFO_EINVAL, "FFA executor task input_nsamples must match time series size");
  if (!isfinite(t->downsample_factor) || t->downsample_factor < 1.0) return fail(GFO_EINVAL, "FFA executor task downsample_factor must be finite and >= 1");
  if (!(t->effective_tsamp > 0.0) || !isfinite(t->effective_tsamp)) return fail(GFO_EINVAL, "FFA executor task effective_tsamp must be finite and > 0");
  if (t->bins <= 1) return fail(GFO_EINVAL, "FFA executor task bins must be > 1");
  if (t->rows == 0) return fail(GFO_EINVAL, "FFA executor task rows must be > 0");
  if (t->rows_eval == 0 || t->rows_eval > t->rows) return fail(GFO_EINVAL, "FFA executor task rows_eval must satisfy 0 < rows_eval <= rows");
  if (t->prepared_nsamples == 0) return fail(GFO_EINVAL, "FFA executor task prepared_nsamples must be > 0");
  if (t->rows * t->bins > t->prepared_nsamples) return fail(GFO_EINVAL, "FFA executor task rows * bins must be <= prepared_nsamples");
  if (t->downsample_factor == 1.0) {
    if (t->prepared_nsamples != n) return fail(GFO_EINVAL, "FFA executor no-downsample task prepared_nsamples must match input size");
    return GFO_OK;
  }
  uint64_t m = 0;
  int rc = gfo_downsampled_size(n, t->downsample_factor, &m);
  if (rc) return rc;
  if (t->prepared_nsamples != m) return fail(GFO_EINVAL, "FFA executor task prepared_nsamples must match downsampled_size");
  return GFO_OK;
}

/* ffa_search.cpp:73-108 search_ffa_cpu over ffa_executor.cpp:319-354
 * for_each_ffa_row_cpu and ffa.cpp:203-251 emit_transform_rows */
static int search_series(const float* series, uint64_t n, const gfo_ffa_task* tasks,
                         uint64_t ntasks, const uint64_t* widths, uint64_t nw,
                         float thr, peak_vec* out) {
  if (!isfinite(thr)) return fail(GFO_EINVAL, "FFA search S/N threshold must be finite");
  if (nw == 0) return fail(GFO_EINVAL, "FFA search plan width_trials must not be empty");
  if (n == 0) return fail(GFO_EINVAL, "FFA executor time series must not be empty");
  if (ntasks == 0) return fail(GFO_EINVAL, "FFA executor plan must contain at least one task");
  for (uint64_t i = 0; i < ntasks; ++i) {
    int rc = validate_task(&tasks[i], n);
    if (rc) return rc;
  }
  uint64_t max_full = 0, max_bins = 0;
  for (uint64_t i = 0; i < ntasks; ++i) {
    if (tasks[i].rows * tasks[i].bins > max_full) max_full = tasks[i].rows * tasks[i].bins;
    if (tasks[i].bins > max_bins) max_bins = tasks[i].bins;
  }
  const uint64_t mw = max_u64(widths, nw);
  float* cache = NULL;
  uint64_t cache_n = 0;
  double cache_factor = 0.0;
  int cache_valid = 0;
  float* scratch = (float*)malloc(sizeof(float) * max_full);
  float* work = (float*)malloc(sizeof(float) * max_full);
  float* row = (float*)malloc(sizeof(float) * max_bins);
  float* cp = (float*)calloc(max_bins + mw + 1, sizeof(float));
  boxcar* trials = (boxcar*)malloc(sizeof(boxcar) * nw);
  int rc = GFO_OK;
  if (!scratch || !work || !row || !cp || !trials) rc = fail(GFO_ENOMEM, "out of memory");
  for (uint64_t ti = 0; ti < ntasks && rc == GFO_OK; ++ti) {
    const gfo_ffa_task* t = &tasks[ti];
    const float* prepared = series;
    if (t->downsample_factor != 1.0) {
      /* ffa_executor.cpp:264-280 prepare_task_samples cache */
      if (!cache_valid || cache_factor != t->downsample_factor || cache_n != t->prepared_nsamples) {
        free(cache);
        cache = (float*)malloc(sizeof(float) * t->prepared_nsamples);
        if (!cache) { rc = fail(GFO_ENOMEM, "out of memory"); break; }
        rc = gfo_downsample_weighted_sum(series, n, t->downsample_factor, cache);
        if (rc) break;
        cache_n = t->prepared_nsamples;
        cache_factor = t->downsample_factor;
        cache_valid = 1;
      }
      prepared = cache;
    }
    rc = validate_widths(widths, nw, t->bins);
    if (rc) break;
    make_boxcars(widths, nw, t->bins, trials);
    const float sn = gfo_ffa_task_stdnoise(t);
    const uint64_t rows = t->rows, bins = t->bins;
    if (rows == 1) {
      rc = detect_row(prepared, 0, t, trials, nw, mw, sn, thr, cp, out);
      continue;
    }
    if (rows == 2) {
      for (uint64_t i = 0; i < bins; ++i) row[i] = prepared[i] + prepared[bins + i];
      rc = detect_row(row, 0, t, trials, nw, mw, sn, thr, cp, out);
      if (rc == GFO_OK && t->rows_eval > 1) {
        rollback_add(prepared, prepared + bins, bins, 1, row);
        rc = detect_row(row, 1, t, trials, nw, mw, sn, thr, cp, out);
      }
      continue;
    }
    const uint64_t h = rows / 2, tl = rows - h;
    transform_rec(prepared, h, bins, scratch, work);
    transform_rec(prepared + h * bins, tl, bins, scratch + h * bins, work + h * bins);
    for (uint64_t s = 0; s < t->rows_eval && rc == GFO_OK; ++s) {
      merge_row(work, h, work + h * bins, tl, rows, s, bins, row);
      rc = detect_row(row, s, t, trials, nw, mw, sn, thr, cp, out);
    }
  }
  free(cache); free(scratch); free(work); free(row); free(cp); free(trials);
  return rc;
}

int gfo_ffa_search(const float* series, uint64_t n, const gfo_ffa_task* tasks,
                   uint64_t ntasks, const uint64_t* widths, uint64_t nw, float thr,
                   uint64_t max_peaks, gfo_peak** peaks, uint64_t* npeaks) {
  peak_vec v = {NULL, 0, 0, max_peaks};
  int rc = search_series(series, n, tasks, ntasks, widths, nw, thr, &v);
  if (rc) { free(v.data); return rc; }
  gfo_sort_dm_peaks(v.data, v.n);
  *peaks = v.data;
  *npeaks = v.n;
  return GFO_OK;
}

/* dm_search.cpp:119-199 find_dm_peaks_cpu (composition of dm_time_series_cpu,
 * preprocess_time_series_cpu and search_ffa_cpu per DM, then a global sort).
 * width_override replaces the plan's generated width trials, as a caller of
 * search_ffa_cpu may do with the public FfaSearchPlan struct. */
int gfo_find_dm_peaks_u32(const uint32_t* data, uint64_t ndm, uint64_t nsamples,
                          const double* dms, double tsamp,
                          const gfo_plan_options* po, const gfo_preprocess_options* pre,
                          float thr, uint64_t max_peaks, const uint64_t* wo,
                          uint64_t nwo, gfo_peak** peaks_out, uint64_t* npeaks_out) {
  if (ndm == 0) return fail(GFO_EINVAL, "DM search dedispersed ndm must be > 0");
  if (nsamples == 0) return fail(GFO_EINVAL, "DM search dedispersed nsamples must be > 0");
  if (!(tsamp > 0.0) || !isfinite(tsamp)) return fail(GFO_EINVAL, "DM search tsamp must be finite and > 0");
  for (uint64_t d = 0; d < ndm; ++d)
    if (!isfinite(dms[d])) return fail(GFO_EINVAL, "DM search dms must be finite");
  if (!isfinite(thr)) return fail(GFO_EINVAL, "DM search S/N threshold must be finite");
  gfo_ffa_task* tasks = NULL;
  uint64_t ntasks = 0, nw = 0;
  uint64_t* widths = NULL;
  int rc = gfo_make_riptide_ffa_plan(nsamples, tsamp, po, &tasks, &ntasks, &widths, &nw);
  if (rc) return rc;
  const uint64_t* use_w = widths;
  uint64_t use_nw = nw;
  if (wo && nwo) { use_w = wo; use_nw = nwo; }

  peak_vec all = {NULL, 0, 0, 0};
  int err = GFO_OK;
  char errmsg[256] = {0};
#pragma omp parallel
  {
    peak_vec local = {NULL, 0, 0, 0};
    float* ts = (float*)malloc(sizeof(float) * nsamples);
#pragma omp for schedule(dynamic, 1)
    for (int64_t d = 0; d < (int64_t)ndm; ++d) {
      int lrc;
#pragma omp atomic read
      lrc = err;
      if (lrc) continue;
      if (!ts) { lrc = fail(GFO_ENOMEM, "out of memory"); }
      else {
        const uint32_t* row = data + (uint64_t)d * nsamples;
        for (uint64_t i = 0; i < nsamples; ++i) ts[i] = (float)row[i];
        lrc = pre ? gfo_preprocess_riptide(ts, nsamples, tsamp, pre) : GFO_OK;
        if (lrc == GFO_OK) {
          peak_vec v = {NULL, 0, 0, max_peaks};
          lrc = search_series(ts, nsamples, tasks, ntasks, use_w, use_nw, thr, &v);
          for (uint64_t i = 0; lrc == GFO_OK && i < v.n; ++i) {
            v.data[i].dm = dms[d];
            v.data[i].dm_index = (uint64_t)d;
            lrc = push_peak(&local, &v.data[i]);
          }
          free(v.data);
        }
      }
      if (lrc) {
#pragma omp critical(gfo_dm_error)
        {
          if (!err) { err = lrc; memcpy(errmsg, g_error, sizeof errmsg); }
        }
      }
    }
#pragma omp critical(gfo_dm_peaks)
    {
      for (uint64_t i = 0; i < local.n && !err; ++i)
        if (push_peak(&all, &local.data[i])) err = GFO_ENOMEM;
    }
    free(local.data);
    free(ts);
  }
  free(tasks);
  free(widths);
  if (err) {
    free(all.data);
    memcpy(g_error, errmsg, sizeof errmsg);
    return err;
  }
  gfo_sort_dm_peaks(all.data, all.n);
  *peaks_out = all.data;
  *npeaks_out = all.n;
  return GFO_OK;
}

/* ------------------------------------------------------------------------ */
/* candidates (candidate.cpp)                                                */
/* ------------------------------------------------------------------------ */

static int cmp_peak_order(const void* a, const void* b) {
  /* candidate.cpp:64-75 peak_order */
  const gfo_peak* l = (const gfo_peak*)a;
  const gfo_peak* r = (const gfo_peak*)b;
  if (l->frequency != r->frequency) return l->frequency < r->frequency ? -1 : 1;
  if (l->width != r->width) return l->width < r->width ? -1 : 1;
  if (l->dm_index != r->dm_index) return l->dm_index < r->dm_index ? -1 : 1;
  return cmp_dm_peak(a, b);
}

static int cmp_dm_group(const void* a, const void* b) {
  /* candidate.cpp:77-85 dm_group_order */
  const gfo_peak* l = (const gfo_peak*)a;
  const gfo_peak* r = (const gfo_peak*)b;
  if (l->dm_index != r->dm_index) return l->dm_index < r->dm_index ? -1 : 1;
  if (l->width != r->width) return l->width < r->width ? -1 : 1;
  if (l->frequency != r->frequency) return l->frequency < r->frequency ? -1 : 1;
  return 0;
}

static int cmp_width_dm_group(const void* a, const void* b) {
  /* candidate.cpp:87-92 width_then_dm_group_order */
  const gfo_peak* l = (const gfo_peak*)a;
  const gfo_peak* r = (const gfo_peak*)b;
  if (l->width != r->width) return l->width < r->width ? -1 : 1;
  return cmp_dm_group(a, b);
}

typedef struct {
  gfo_candidate* data;
  uint64_t n, cap;
} cand_vec;

static int push_cand(cand_vec* v, const gfo_candidate* c) {
  if (v->n == v->cap) {
    uint64_t nc = v->cap ? v->cap * 2 : 64;
    gfo_candidate* nd = (gfo_candidate*)realloc(v->data, sizeof(gfo_candidate) * nc);
    if (!nd) return fail(GFO_ENOMEM, "out of memory");
    v->data = nd;
    v->cap = nc;
  }
  v->data[v->n++] = *c;
  return GFO_OK;
}

/* candidate.cpp:101-138 make_candidate */
static void make_candidate(const gfo_peak* b, const gfo_peak* e, gfo_candidate* c) {
  const gfo_peak* best = b;
  uint64_t dmin = UINT64_MAX, dmax = 0;
  double fmin = INFINITY, fmax = -INFINITY;
  for (const gfo_peak* p = b; p != e; ++p) {
    if (gfo_is_better_peak(p, best)) best = p;
    if (p->dm_index < dmin) dmin = p->dm_index;
    if (p->dm_index > dmax) dmax = p->dm_index;
    if (p->frequency < fmin) fmin = p->frequency;
    if (p->frequency > fmax) fmax = p->frequency;
  }
  memset(c, 0, sizeof *c);
  c->dm = best->dm;
  c->dm_index = best->dm_index;
  c->period = best->period;
  c->frequency = best->frequency;
  c->width = best->width;
  c->duty_cycle = best->duty_cycle;
  c->snr = best->snr;
  c->peak_count = (uint64_t)(e - b);
  c->dm_index_min = dmin;
  c->dm_index_max = dmax;
  c->frequency_min = fmin;
  c->frequency_max = fmax;
  c->best_peak = *best;
}

/* candidate.cpp:140-171 append_dm_clusters */
static int append_dm_clusters(gfo_peak* b, gfo_peak* e, const gfo_candidate_options* o,
                              cand_vec* out) {
  if (b == e) return GFO_OK;
  qsort(b, (size_t)(e - b), sizeof(gfo_peak),
        o->cluster_across_widths ? cmp_dm_group : cmp_width_dm_group);
  gfo_peak* cluster = b;
  uint64_t prev_dm = b->dm_index, prev_w = b->width;
  gfo_candidate c;
  for (gfo_peak* p = b + 1; p != e; ++p) {
    const int same_w = o->cluster_across_widths || p->width == prev_w;
    /* candidate.cpp:94-99 same_dm_cluster */
    const int same_dm = p->dm_index <= prev_dm || p->dm_index - prev_dm <= o->dm_cluster_radius;
    if (!same_w || !same_dm) {
      make_candidate(cluster, p, &c);
      if (push_cand(out, &c)) return GFO_ENOMEM;
      cluster = p;
    }
    prev_dm = p->dm_index;
    prev_w = p->width;
  }
  make_candidate(cluster, e, &c);
  return push_cand(out, &c);
}

/* candidate.cpp:48-62 is_better_candidate */
static int cmp_candidate(const void* a, const void* b) {
  const gfo_candidate* l = (const gfo_candidate*)a;
  const gfo_candidate* r = (const gfo_candidate*)b;
  if (gfo_is_better_peak(&l->best_peak, &r->best_peak)) return -1;
  if (gfo_is_better_peak(&r->best_peak, &l->best_peak)) return 1;
  if (l->peak_count != r->peak_count) return l->peak_count > r->peak_count ? -1 : 1;
  if (l->frequency != r->frequency) return l->frequency < r->frequency ? -1 : 1;
  if (l->dm_index != r->dm_index) return l->dm_index < r->dm_index ? -1 : 1;
  return 0;
}

/* candidate.cpp:175-212 select_candidates_cpu */
int gfo_select_candidates(const gfo_peak* peaks, uint64_t n, double tobs,
                          const gfo_candidate_options* o, gfo_candidate** out,
                          uint64_t* nout) {
  if (!(tobs > 0.0) || !isfinite(tobs))
    return fail(GFO_EINVAL, "Candidate selection observation_seconds must be finite and > 0");
  if (o->frequency_cluster_radius < 0.0 || !isfinite(o->frequency_cluster_radius))
    return fail(GFO_EINVAL, "Candidate selection frequency_cluster_radius must be finite and >= 0");
  *out = NULL;
  *nout = 0;
  if (n == 0) return GFO_OK;
  for (uint64_t i = 0; i < n; ++i) {
    const gfo_peak* p = &peaks[i];
    if (!isfinite(p->dm) || !isfinite(p->period) || !isfinite(p->frequency) ||
        !isfinite(p->duty_cycle) || !isfinite(p->snr))
      return fail(GFO_EINVAL, "Candidate selection peaks must contain finite scientific values");
  }
  gfo_peak* sorted = (gfo_peak*)malloc(sizeof(gfo_peak) * n);
  if (!sorted) return fail(GFO_ENOMEM, "out of memory");
  memcpy(sorted, peaks, sizeof(gfo_peak) * n);
  qsort(sorted, n, sizeof(gfo_peak), cmp_peak_order);
  const double radius_hz = o->frequency_cluster_radius / tobs;
  cand_vec cv = {NULL, 0, 0};
  gfo_peak* fb = sorted;
  double prev_f = fb->frequency;
  int rc = GFO_OK;
  for (gfo_peak* p = sorted + 1; p != sorted + n && rc == GFO_OK; ++p) {
    if (p->frequency - prev_f > radius_hz) {
      rc = append_dm_clusters(fb, p, o, &cv);
      fb = p;
    }
    prev_f = p->frequency;
  }
  if (rc == GFO_OK) rc = append_dm_clusters(fb, sorted + n, o, &cv);
  free(sorted);
  if (rc) { free(cv.data); return rc; }
  qsort(cv.data, cv.n, sizeof(gfo_candidate), cmp_candidate);
  if (o->max_candidates != 0 && cv.n > o->max_candidates) cv.n = o->max_candidates;
  *out = cv.data;
  *nout = cv.n;
  return GFO_OK;
}

/* ------------------------------------------------------------------------ */
/* folding (folding.cpp)                                                     */
/* ------------------------------------------------------------------------ */

/* folding.cpp:124-158 accumulate_interval with :115-122 positive_mod */
static void accumulate(double value, double lo, double hi, double* sums,
                       double* expo, uint64_t nbin) {
  const int64_t first = (int64_t)floor(lo);
  const int64_t last = (int64_t)(ceil(hi) - 1.0);
  for (int64_t bin = first; bin <= last; ++bin) {
    const double bl = (double)bin, br = bl + 1.0;
    const double w = (hi < br ? hi : br) - (lo > bl ? lo : bl);
    if (!(w > 0.0)) continue;
    int64_t m = bin % (int64_t)nbin;
    if (m < 0) m += (int64_t)nbin;
    sums[m] += value * w;
    expo[m] += w;
  }
}

static int fold_check(double period, double tsamp, uint64_t nbin, uint64_t n) {
  /* folding.cpp:44-58 validate_fold_shape */
  if (!isfinite(period) || !(period > 0.0)) return fail(GFO_EINVAL, "fold period must be finite and positive");
  if (!isfinite(tsamp) || !(tsamp > 0.0)) return fail(GFO_EINVAL, "fold tsamp must be finite and positive");
  if (nbin == 0) return fail(GFO_EINVAL, "fold nbin must be positive");
  if (n == 0) return fail(GFO_EINVAL, "fold input must not be empty");
  return GFO_OK;
}

/* folding.cpp:452-490 fold_time_series_impl (single-threaded accumulation;
 * the reference reduces per-thread FP64 partial sums in arbitrary order) */
#define FOLD_BODY(VALUE_EXPR)                                                  \
  double* sums = (double*)calloc(nbin, sizeof(double));                       \
  if (!sums) return fail(GFO_ENOMEM, "out of memory");                        \
  for (uint64_t b = 0; b < nbin; ++b) exposure[b] = 0.0;                      \
  const double step = tsamp / period * (double)nbin;                           \
  for (uint64_t i = 0; i < n; ++i) {                                           \
    const double lo = (double)(start + i) * step;                              \
    accumulate((VALUE_EXPR), lo, lo + step, sums, exposure, nbin);             \
  }                                                                            \
  for (uint64_t b = 0; b < nbin; ++b)                                          \
    profile[b] = exposure[b] > 0.0 ? (float)(sums[b] / exposure[b]) : 0.0f;    \
  free(sums);                                                                  \
  return GFO_OK;

int gfo_fold_time_series_f32(const float* in, uint64_t n, double period, double tsamp,
                             uint64_t nbin, uint64_t start, float* profile,
                             double* exposure) {
  int rc = fold_check(period, tsamp, nbin, n);
  if (rc) return rc;
  for (uint64_t i = 0; i < n; ++i)
    if (!isfinite(in[i])) return fail(GFO_EINVAL, "fold input must contain only finite samples");
  FOLD_BODY((double)in[i])
}

int gfo_fold_time_series_u32(const uint32_t* in, uint64_t n, double period,
                             double tsamp, uint64_t nbin, uint64_t start,
                             float* profile, double* exposure) {
  int rc = fold_check(period, tsamp, nbin, n);
  if (rc) return rc;
  FOLD_BODY((double)in[i])
}

/* ------------------------------------------------------------------------ */
/* harmonics: harmonic.cpp:14-311                                            */
/* ------------------------------------------------------------------------ */

typedef struct {
  int32_t num, den;
  double value;
} h_ratio;

static uint64_t gcd_u64(uint64_t a, uint64_t b) {
  while (b) {
    const uint64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

static int cmp_ratio(const void* a, const void* b) {
  const h_ratio* l = (const h_ratio*)a;
  const h_ratio* r = (const h_ratio*)b;
  if (l->value != r->value) return l->value < r->value ? -1 : 1;
  if (l->num != r->num) return l->num < r->num ? -1 : 1;
  if (l->den != r->den) return l->den < r->den ? -1 : 1;
  return 0;
}

/* harmonic.cpp:21-35: S/N desc, peak_count desc, frequency asc, dm_index asc */
static int cmp_harmonic_rank(const void* a, const void* b) {
  const gfo_candidate* l = (const gfo_candidate*)a;
  const gfo_candidate* r = (const gfo_candidate*)b;
  if (l->snr != r->snr) return l->snr > r->snr ? -1 : 1;
  if (l->peak_count != r->peak_count) return l->peak_count > r->peak_count ? -1 : 1;
  if (l->frequency != r->frequency) return l->frequency < r->frequency ? -1 : 1;
  if (l->dm_index != r->dm_index) return l->dm_index < r->dm_index ? -1 : 1;
  return 0;
}

/* nearest ratio to x (harmonic.cpp:137-163): the first ratio with value >= x,
 * replaced by its predecessor only when that is strictly closer */
static const h_ratio* nearest_ratio(double x, const h_ratio* r, uint64_t nr) {
  if (!(x > 0.0) || nr == 0) return NULL;
  uint64_t lo = 0, hi = nr;
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (r[mid].value < x) lo = mid + 1; else hi = mid;
  }
  const h_ratio* best = lo < nr ? &r[lo] : NULL;
  if (lo > 0 && (best == NULL || fabs(r[lo - 1].value - x) < fabs(best->value - x))) best = &r[lo - 1];
  return best;
}

int gfo_flag_harmonics(const gfo_candidate* in, uint64_t n, const gfo_harmonic_context* ctx,
                       const gfo_harmonic_options* o, gfo_candidate* sorted,
                       gfo_harmonic_relation* rel) {
  /* harmonic.cpp:37-92 validation */
  if (!(ctx->observation_seconds > 0.0) || !isfinite(ctx->observation_seconds))
    return fail(GFO_EINVAL, "Harmonic context observation_seconds must be finite and > 0");
  if (!(ctx->frequency_low_mhz > 0.0) || !(ctx->frequency_high_mhz > 0.0) ||
      !isfinite(ctx->frequency_low_mhz) || !isfinite(ctx->frequency_high_mhz))
    return fail(GFO_EINVAL, "Harmonic context frequencies must be finite and > 0 MHz");
  if (o->max_harmonic < 2) return fail(GFO_EINVAL, "Harmonic max_harmonic must be >= 2");
  if (o->denominator_max == 0) return fail(GFO_EINVAL, "Harmonic denominator_max must be > 0");
  if (o->frequency_tolerance_bins < 0.0 || !isfinite(o->frequency_tolerance_bins))
    return fail(GFO_EINVAL, "Harmonic frequency_tolerance_bins must be finite and >= 0");
  if (o->phase_distance_max < 0.0 || !isfinite(o->phase_distance_max))
    return fail(GFO_EINVAL, "Harmonic phase_distance_max must be finite and >= 0");
  if (o->dm_distance_max < 0.0 || !isfinite(o->dm_distance_max))
    return fail(GFO_EINVAL, "Harmonic dm_distance_max must be finite and >= 0");
  if (o->snr_distance_max < 0.0 || !isfinite(o->snr_distance_max))
    return fail(GFO_EINVAL, "Harmonic snr_distance_max must be finite and >= 0");
  if (n == 0) return GFO_OK;
  for (uint64_t i = 0; i < n; ++i) {
    const gfo_candidate* c = &in[i];
    if (!isfinite(c->dm) || !isfinite(c->period) || !isfinite(c->frequency) ||
        !isfinite(c->duty_cycle) || !isfinite(c->snr))
      return fail(GFO_EINVAL, "Harmonic candidates must contain finite scientific values");
    if (!(c->frequency > 0.0) || !(c->period > 0.0) || !(c->duty_cycle > 0.0) || !(c->snr >= 0.0f))
      return fail(GFO_EINVAL, "Harmonic candidate frequency, period, duty_cycle, and snr are invalid");
  }
  memcpy(sorted, in, n * sizeof(gfo_candidate));
  qsort(sorted, n, sizeof(gfo_candidate), cmp_harmonic_rank);
  for (uint64_t i = 0; i < n; ++i) {
    memset(&rel[i], 0, sizeof rel[i]);
    rel[i].parent_index = UINT64_MAX;
    rel[i].numerator = 1;
    rel[i].denominator = 1;
  }
  /* harmonic.cpp:94-135: reduced n/d with n != d, sorted, unique */
  h_ratio* r = (h_ratio*)malloc(o->max_harmonic * o->denominator_max * sizeof(h_ratio));
  if (!r) return fail(GFO_ENOMEM, "out of memory");
  uint64_t nr = 0;
  for (uint64_t a = 1; a <= o->max_harmonic; ++a)
    for (uint64_t b = 1; b <= o->denominator_max; ++b) {
      const uint64_t g = gcd_u64(a, b);
      if (a / g == b / g) continue;
      r[nr].num = (int32_t)(a / g);
      r[nr].den = (int32_t)(b / g);
      r[nr].value = (double)(a / g) / (double)(b / g);
      ++nr;
    }
  qsort(r, nr, sizeof(h_ratio), cmp_ratio);
  uint64_t u = 0;
  for (uint64_t i = 0; i < nr; ++i)
    if (u == 0 || r[i].num != r[u - 1].num || r[i].den != r[u - 1].den) r[u++] = r[i];
  nr = u;
  const double low = fmin(ctx->frequency_low_mhz, ctx->frequency_high_mhz);
  const double high = fmax(ctx->frequency_low_mhz, ctx->frequency_high_mhz);
  for (uint64_t pi = 0; pi < n; ++pi) {
    if (rel[pi].is_harmonic) continue;
    const gfo_candidate* p = &sorted[pi];
    for (uint64_t ci = pi + 1; ci < n; ++ci) {
      if (rel[ci].is_harmonic) continue;
      const gfo_candidate* c = &sorted[ci];
      /* harmonic.cpp:186-243 test_harmonic_relation */
      const h_ratio* hr = nearest_ratio(c->frequency / p->frequency, r, nr);
      if (!hr) continue;
      const double expected = p->frequency * hr->value;
      const double ferr = fabs(c->frequency - expected) * ctx->observation_seconds;
      if (ferr > o->frequency_tolerance_bins) continue;
      const double fast_duty = c->frequency >= p->frequency ? c->duty_cycle : p->duty_cycle;
      const double phase = ferr / fast_duty;
      if (phase > o->phase_distance_max) continue;
      const double delay_ms = fabs(p->dm - c->dm) * 4.148808e3 * fabs(1.0 / (low * low) - 1.0 / (high * high));
      const double wp = p->period * p->duty_cycle, wc = c->period * c->duty_cycle;
      const double dist = (delay_ms / 1000.0) / (wp < wc ? wp : wc);
      if (dist > o->dm_distance_max) continue;
      const double esnr = (double)p->snr / sqrt((double)hr->num * (double)hr->den);
      const double sdist = fabs((double)c->snr - esnr);
      if (o->use_snr_consistency && sdist > o->snr_distance_max) continue;
      rel[ci].is_harmonic = 1;
      rel[ci].parent_index = pi;
      rel[ci].numerator = hr->num;
      rel[ci].denominator = hr->den;
      rel[ci].frequency_error_bins = ferr;
      rel[ci].phase_distance = phase;
      rel[ci].dm_distance = dist;
      rel[ci].expected_snr = esnr;
      rel[ci].snr_distance = sdist;
    }
  }
  free(r);
  return GFO_OK;
}

int gfo_remove_harmonics(const gfo_candidate* sorted, const gfo_harmonic_relation* rel, uint64_t n,
                         uint64_t max_candidates, gfo_candidate* out, uint64_t* nout) {
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (rel[i].is_harmonic) continue;
    out[k++] = sorted[i];
    if (max_candidates != 0 && k >= max_candidates) break;
  }
  *nout = k;
  return GFO_OK;
}

/* ------------------------------------------------------------------------ */
/* aligned spectrum: dedispersion.cpp:249-289                                */
/* ------------------------------------------------------------------------ */

int gfo_dedisperse_spectrum_u8(const uint8_t* in, uint64_t nsamples, uint64_t nchans,
                               const double* freq, double dm, double ref, double tsamp,
                               uint64_t cb, uint64_t ce, uint8_t* out, uint64_t* nout) {
  if (nsamples == 0) return fail(GFO_EINVAL, "dedispersion requires at least one sample");
  if (nchans == 0) return fail(GFO_EINVAL, "dedispersion requires at least one channel");
  if (!(isfinite(ref) && ref > 0.0)) return fail(GFO_EINVAL, "reference frequency must be positive");
  if (!(isfinite(tsamp) && tsamp > 0.0)) return fail(GFO_EINVAL, "tsamp must be positive");
  if (cb >= ce) return fail(GFO_EINVAL, "channel range must be non-empty");
  if (ce > nchans) return fail(GFO_EINVAL, "channel range exceeds sample channel count");
  if (!isfinite(dm) || dm < 0.0) return fail(GFO_EINVAL, "dm must be finite and non-negative");
  double fmin = freq[cb];
  for (uint64_t c = cb; c < ce; ++c) {
    if (!(isfinite(freq[c]) && freq[c] > 0.0))
      return fail(GFO_EINVAL, "frequency values must be finite and positive");
    if (freq[c] > ref)
      return fail(GFO_EINVAL, "dedispersion requires selected frequencies <= reference frequency");
    if (freq[c] < fmin) fmin = freq[c];
  }
  const int32_t maxd = gfo_delay_bins(dm, fmin, ref, tsamp);
  if (maxd < 0) return fail(GFO_EINVAL, "dedispersion requires non-negative delays");
  if ((uint64_t)maxd >= nsamples) return fail(GFO_EINVAL, "dedispersion valid output range is empty");
  *nout = nsamples - (uint64_t)maxd;
  if (!out) return GFO_OK;
  const uint64_t nc = ce - cb;
  for (uint64_t c = 0; c < nc; ++c) {
    const int32_t d = gfo_delay_bins(dm, freq[cb + c], ref, tsamp);
    for (uint64_t t = 0; t < *nout; ++t) out[t * nc + c] = in[(t + (uint64_t)d) * nchans + cb + c];
  }
  return GFO_OK;
}
