// The pairwise harmonic test of flag_harmonics_cpu (harmonic.cpp:137-243),
// shared by the host loop (host.cpp) and the device flagging (harmonics.cu)
// so both take identical decisions.  FP64 throughout; on the device every
// operation is an explicitly rounded intrinsic (no contraction), on the host
// the build disables contraction, so the two evaluate the same IEEE
// expressions.
#pragma once

#include <cmath>
#include <cstdint>

#include "gaffa_b200.h"

namespace gf {

#ifdef __CUDA_ARCH__
#define GF_DMUL(a, b) __dmul_rn((a), (b))
#define GF_DDIV(a, b) __ddiv_rn((a), (b))
#define GF_DSUB(a, b) __dsub_rn((a), (b))
#define GF_DSQRT(a) __dsqrt_rn(a)
#else
#define GF_DMUL(a, b) ((a) * (b))
#define GF_DDIV(a, b) ((a) / (b))
#define GF_DSUB(a, b) ((a) - (b))
#define GF_DSQRT(a) std::sqrt(a)
#endif

// A reduced harmonic ratio num/den (harmonic.cpp:94-135).
struct HarmonicRatio {
  int32_t num, den;
  double value;
};

// The candidate fields the test reads.
struct HarmonicInput {
  double frequency, period, duty_cycle, dm;
  float snr;
  uint32_t reserved;
};

// Index of the ratio nearest to x: the first with value >= x unless its
// predecessor is strictly closer (harmonic.cpp:137-163); -1 when none.
__host__ __device__ inline int nearest_harmonic_ratio(double x, const HarmonicRatio* r, int n) {
  if (!(x > 0.0) || n == 0) return -1;
  int lo = 0, hi = n;  // first index with r[i].value >= x
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (r[mid].value < x) lo = mid + 1; else hi = mid;
  }
  int best = lo < n ? lo : -1;
  if (lo > 0) {
    const int prev = lo - 1;
    if (best < 0 || fabs(GF_DSUB(r[prev].value, x)) < fabs(GF_DSUB(r[best].value, x))) best = prev;
  }
  return best;
}

// test_harmonic_relation (harmonic.cpp:186-243): whether child c is a
// harmonic of parent p; fills *rel (when given) on success.  band is
// |1/lo^2 - 1/hi^2| of the observing band.
__host__ __device__ inline bool harmonic_test(const HarmonicInput& p, const HarmonicInput& c,
                                              const HarmonicRatio* ratios, int nratios, double observation_seconds,
                                              double band, const gf_harmonic_options& o, uint64_t parent_index,
                                              gf_harmonic_relation* rel) {
  const int k = nearest_harmonic_ratio(GF_DDIV(c.frequency, p.frequency), ratios, nratios);
  if (k < 0) return false;
  const HarmonicRatio hr = ratios[k];
  const double ferr = GF_DMUL(fabs(GF_DSUB(c.frequency, GF_DMUL(p.frequency, hr.value))), observation_seconds);
  if (ferr > o.frequency_tolerance_bins) return false;
  const double phase = GF_DDIV(ferr, c.frequency >= p.frequency ? c.duty_cycle : p.duty_cycle);
  if (phase > o.phase_distance_max) return false;
  const double delay_s = GF_DDIV(GF_DMUL(GF_DMUL(fabs(GF_DSUB(p.dm, c.dm)), 4.148808e3), band), 1000.0);
  const double wp = GF_DMUL(p.period, p.duty_cycle), wc = GF_DMUL(c.period, c.duty_cycle);
  const double dist = GF_DDIV(delay_s, wp < wc ? wp : wc);
  if (dist > o.dm_distance_max) return false;
  const double esnr = GF_DDIV(static_cast<double>(p.snr),
                              GF_DSQRT(GF_DMUL(static_cast<double>(hr.num), static_cast<double>(hr.den))));
  const double sdist = fabs(GF_DSUB(static_cast<double>(c.snr), esnr));
  if (o.use_snr_consistency && sdist > o.snr_distance_max) return false;
  if (rel) {
    rel->is_harmonic = 1;
    rel->reserved = 0;
    rel->parent_index = parent_index;
    rel->numerator = hr.num;
    rel->denominator = hr.den;
    rel->frequency_error_bins = ferr;
    rel->phase_distance = phase;
    rel->dm_distance = dist;
    rel->expected_snr = esnr;
    rel->snr_distance = sdist;
  }
  return true;
}

inline HarmonicInput harmonic_input(const gf_candidate& c) {
  return HarmonicInput{c.frequency, c.period, c.duty_cycle, c.dm, c.snr, 0u};
}

}  // namespace gf
