/*
 * synth_oracle.c -- the seeded synthetic filterbank of gaffa_b200/synth.py on
 * the host cores (TEST INFRASTRUCTURE: it feeds the CPU baseline and the
 * reference arm of bench.py, which must not load the CUDA product).
 *
 * The reference ships no generator; this one defines the workload.  Every
 * sample is a pure function of (seed, time, channel): noise is an
 * Irwin-Hall(12) deviate from a splitmix64 stream keyed by the flat sample
 * index, the injected pulses and RFI are evaluated in FP64 with the same
 * expressions as the numpy and CUDA generators and rounded to 1/4096 count.
 * Rows are generated in parallel (OpenMP).
 *
 * Speed: a pulse term is exactly 0.0 outside |x| < 12 (x = phase offset /
 * sigma).  Rows are generated in blocks of 64; for every (pulsar, channel) the
 * samples of a block that can lie in a pulse window are found from a
 * multiply-only phase estimate (its error is far inside the 0.001 sigma and
 * one-sample slack of the window), and only those are evaluated with the
 * exact expression.  Pulsars are added in order, so the sums are the same.
 */
#include "gaffa_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* sum of twelve 16-bit words: z = S / 65536 - 6 */
static inline int64_t noise_sum(uint64_t seed, uint64_t idx) {
  const uint64_t base = ((seed & 0xFFFFFull) << 44) ^ (idx * 3ull);
  int64_t s = 0;
  for (int k = 0; k < 3; ++k) {
    const uint64_t h = splitmix(base + (uint64_t)k);
    s += (int64_t)(h & 0xFFFFull) + (int64_t)((h >> 16) & 0xFFFFull) + (int64_t)((h >> 32) & 0xFFFFull) +
         (int64_t)(h >> 48);
  }
  return s;
}

typedef struct {
  double period, dm, sigma, amplitude, phase;
  double inv_period, inv_sigma;
} pulsar_t;

enum { kBlockRows = 64 };

int gfo_synth_generate(const gfo_synth_desc* d, uint64_t t_begin, uint64_t t_end, uint8_t* out) {
  if (!d || !out) return GFO_EINVAL;
  if (d->nbits != 8 && d->nbits != 2) return GFO_EINVAL;
  if (d->nbits == 2 && d->nchans % 4) return GFO_EINVAL;
  if (t_begin > t_end || t_end > d->nsamples || d->nchans == 0 || !(d->tsamp > 0.0)) return GFO_EINVAL;
  const uint64_t nchans = d->nchans;
  double* freq = (double*)malloc(nchans * sizeof(double));
  double* delay = (double*)malloc((size_t)(d->npulsars > 0 ? d->npulsars : 1) * nchans * sizeof(double));
  pulsar_t* ps = (pulsar_t*)malloc((size_t)(d->npulsars > 0 ? d->npulsars : 1) * sizeof(pulsar_t));
  if (!freq || !delay || !ps) {
    free(freq);
    free(delay);
    free(ps);
    return GFO_ENOMEM;
  }
  for (uint64_t c = 0; c < nchans; ++c)
    freq[c] = nchans == 1 ? d->f_high : d->f_low + (d->f_high - d->f_low) * (double)c / (double)(nchans - 1);
  double fref = freq[0];
  for (uint64_t c = 0; c < nchans; ++c)
    if (freq[c] > fref) fref = freq[c];
  for (int k = 0; k < d->npulsars; ++k) {
    const gfo_synth_pulsar q = d->pulsars[k];
    ps[k].period = q.period;
    ps[k].dm = q.dm;
    ps[k].sigma = q.duty_cycle / 2.3548200450309493;
    ps[k].amplitude = q.amplitude;
    ps[k].phase = q.phase;
    ps[k].inv_period = 1.0 / q.period;
    ps[k].inv_sigma = 1.0 / ps[k].sigma;
    for (uint64_t c = 0; c < nchans; ++c) {
      const double f = freq[c];
      delay[(uint64_t)k * nchans + c] = 4148.808 * q.dm * (1.0 / (f * f) - 1.0 / (fref * fref));
    }
  }
  int64_t impulse_period = 0;
  if (d->impulse_hz > 0.0) {
    impulse_period = llround(1.0 / (d->impulse_hz * d->tsamp));
    if (impulse_period < 1) impulse_period = 1;
  }
  const uint64_t row_bytes = d->nbits == 8 ? nchans : nchans / 4;
  const int have_signal = d->npulsars > 0 || d->narrowband_mask != NULL || impulse_period > 0;
  const double two_pi_hz = 2.0 * 3.141592653589793 * d->narrowband_hz;
  const uint64_t nrows = t_end - t_begin;
  const uint64_t nblocks = (nrows + kBlockRows - 1) / kBlockRows;
  int failed = 0;

#pragma omp parallel
  {
    /* signal totals of one block of rows, [row][channel] */
    double* total = have_signal ? (double*)malloc(kBlockRows * nchans * sizeof(double)) : NULL;
    if (have_signal && !total) {
#pragma omp atomic write
      failed = 1;
    }
#pragma omp for schedule(dynamic, 1)
    for (int64_t bi = 0; bi < (int64_t)nblocks; ++bi) {
      if (have_signal && !total) continue;
      const uint64_t t0 = t_begin + (uint64_t)bi * kBlockRows;
      const uint64_t t1 = t0 + kBlockRows < t_end ? t0 + kBlockRows : t_end;
      const uint64_t rows = t1 - t0;
      if (have_signal) {
        memset(total, 0, rows * nchans * sizeof(double));
        /* pulsars in order; a term outside its window is exactly 0.0 */
        for (int k = 0; k < d->npulsars; ++k) {
          const pulsar_t* p = &ps[k];
          const double slope = d->tsamp * p->inv_period;   /* phase per sample */
          const double w = 12.001 * p->sigma;              /* window half-width (phase) */
          for (uint64_t c = 0; c < nchans; ++c) {
            const double dl = delay[(uint64_t)k * nchans + c];
            const double pa0 = ((double)t0 * d->tsamp - dl) * p->inv_period - p->phase;
            const double pa1 = pa0 + (double)rows * slope;
            uint64_t next = 0; /* rows below this one are done for this (pulsar, channel) */
            for (double n = floor(pa0 - w); n <= ceil(pa1 + w) && next < rows; n += 1.0) {
              /* samples whose estimated phase lies within w of pulse n, one
                 sample of slack on each side (every phase when w >= 1/2) */
              uint64_t a = 0, b = rows;
              if (w < 0.5) {
                const double lo = (n - w - pa0) / slope - 1.0, hi = (n + w - pa0) / slope + 1.0;
                if (hi < 0.0 || lo >= (double)rows) continue;
                a = lo <= 0.0 ? 0 : (uint64_t)lo;
                b = hi >= (double)rows ? rows : (uint64_t)hi + 1;
              }
              if (a < next) a = next; /* overlapping windows: each sample once */
              for (uint64_t r = a; r < b; ++r) {
                const double tt = (double)(t0 + r) * d->tsamp;
                double ph = (tt - dl) / p->period - p->phase;
                ph = ph - floor(ph + 0.5);
                const double x = ph / p->sigma;
                if (fabs(x) < 12.0) total[r * nchans + c] = total[r * nchans + c] + p->amplitude * exp(-0.5 * (x * x));
              }
              if (b > next) next = b;
            }
          }
        }
      }
      for (uint64_t r = 0; r < rows; ++r) {
        const uint64_t t = t0 + r;
        const double tt = (double)t * d->tsamp;
        const int impulse = impulse_period > 0 && (int64_t)t % impulse_period == impulse_period / 2;
        const double nb = d->narrowband_mask ? d->narrowband_amplitude * sin(two_pi_hz * tt) : 0.0;
        uint8_t* row = out + (t - t_begin) * row_bytes;
        uint32_t packed = 0;
        for (uint64_t c = 0; c < nchans; ++c) {
          const int64_t s = noise_sum(d->seed, t * nchans + c);
          int64_t sig = 0;
          if (have_signal) {
            double tot = total[r * nchans + c];
            if (d->narrowband_mask && d->narrowband_mask[c]) tot = tot + nb;
            if (impulse) tot = tot + d->impulse_amplitude;
            sig = (int64_t)rint(tot * 4096.0);
          }
          if (d->nbits == 8) {
            int64_t v = (32 * 4096 + s + sig + 2048) >> 12;
            row[c] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
          } else {
            const int64_t zu = (s >> 4) - 24576 + (sig >> 4);
            const uint32_t lvl = (uint32_t)(zu >= -2763) + (uint32_t)(zu >= 0) + (uint32_t)(zu >= 2763);
            packed |= lvl << (2 * (c & 3));
            if ((c & 3) == 3) {
              row[c >> 2] = (uint8_t)packed;
              packed = 0;
            }
          }
        }
      }
    }
    free(total);
  }
  if (failed) {
    free(freq);
    free(delay);
    free(ps);
    return GFO_ENOMEM;
  }
  free(freq);
  free(delay);
  free(ps);
  return GFO_OK;
}
