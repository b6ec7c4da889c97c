// Host side of the C ABI: error reporting, the riptide FFA planner, peak
// ordering and candidate selection.  These restate the reference's host
// arithmetic (FP64, same operation order) so plans and candidate lists are
// identical to the CPU path.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "harmonic_math.cuh"

namespace gf {

namespace {
thread_local char g_error[512];
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_error, sizeof g_error, fmt, ap);
  va_end(ap);
}

const char* last_error() { return g_error; }

namespace {

// ---- ffa_plan.cpp --------------------------------------------------------

uint64_t ceil_shift(uint64_t rows, uint64_t bins, double pmax_samples) {
  // ffa_plan.cpp:47-54
  const double v = static_cast<double>(bins) * (static_cast<double>(rows) - 1.0) *
                   (1.0 - static_cast<double>(bins) / pmax_samples);
  return static_cast<uint64_t>(std::ceil(v));
}

double evaluated_period_end(double eff, uint64_t bins, uint64_t rows, uint64_t rows_eval) {
  // ffa_plan.cpp:74-86
  if (rows == 1 || rows_eval == 1) return eff * static_cast<double>(bins);
  const double b = static_cast<double>(bins);
  const double shift = static_cast<double>(rows_eval - 1) / static_cast<double>(rows - 1);
  return eff * b * b / (b - shift);
}

void make_plan(uint64_t n, double tsamp, const gf_plan_options& o, std::vector<gf_ffa_task>& tasks,
               std::vector<uint64_t>& widths) {
  // ffa_plan.cpp:18-38 validation
  check_arg(n > 0, "FFA plan nsamples must be > 0");
  check_arg(tsamp > 0.0, "FFA plan tsamp must be > 0");
  check_arg(o.period_min > 0.0, "FFA plan period_min must be > 0");
  check_arg(o.period_max > o.period_min, "FFA plan period_max must be > period_min");
  check_arg(o.bins_min > 1, "FFA plan bins_min must be > 1");
  check_arg(o.bins_max >= o.bins_min, "FFA plan bins_max must be >= bins_min");
  check_arg(o.min_periods > 0, "FFA plan min_periods must be > 0");
  check_arg(o.duty_cycle_max > 0.0 && o.duty_cycle_max < 1.0, "FFA plan duty_cycle_max must be in (0, 1)");
  check_arg(o.width_trial_spacing > 1.0, "FFA plan width_trial_spacing must be > 1");
  check_arg(o.max_tasks > 0, "FFA plan max_tasks must be > 0");
  check_arg(o.period_min >= tsamp * static_cast<double>(o.bins_min),
            "FFA plan period_min must be >= tsamp * bins_min");
  // ffa_plan.cpp:90-170
  const double tobs = static_cast<double>(n) * tsamp;
  const double pmax = std::min(o.period_max, tobs / static_cast<double>(o.min_periods));
  check_arg(pmax > o.period_min, "FFA search range is empty after min_periods cap");
  const uint64_t wmax = std::max<uint64_t>(
      1, static_cast<uint64_t>(std::floor(o.duty_cycle_max * static_cast<double>(o.bins_min))));
  for (uint64_t w = 1; w <= wmax;) {
    widths.push_back(w);
    const uint64_t scaled = static_cast<uint64_t>(std::floor(o.width_trial_spacing * static_cast<double>(w)));
    w = std::max(w + 1, scaled);
  }
  const double f0 = o.period_min / (tsamp * static_cast<double>(o.bins_min));
  const double growth = (static_cast<double>(o.bins_max) + 1.0) / static_cast<double>(o.bins_min);
  const uint64_t cycles = static_cast<uint64_t>(std::ceil(std::log(pmax / o.period_min) / std::log(growth)));
  for (uint64_t cycle = 0; cycle < cycles; ++cycle) {
    const double factor = f0 * std::pow(growth, static_cast<double>(cycle));
    const double eff = factor * tsamp;
    uint64_t prepared;
    if (factor == 1.0) {
      prepared = n;
    } else {
      check_arg(std::isfinite(factor) && factor > 1.0 && factor <= static_cast<double>(n),
                "downsample factor must satisfy 1 < factor <= nsamples");
      prepared = static_cast<uint64_t>(std::floor(static_cast<double>(n) / factor));
    }
    const double pmax_samples = pmax / eff;
    const uint64_t stop = std::min({o.bins_max, prepared, static_cast<uint64_t>(std::floor(pmax_samples))});
    if (stop < o.bins_min) continue;
    for (uint64_t bins = o.bins_min; bins <= stop; ++bins) {
      const uint64_t rows = prepared / bins;
      if (rows < o.min_periods) continue;
      const double pceil = std::min(pmax_samples, static_cast<double>(bins) + 1.0);
      const uint64_t rows_eval = std::min(rows, ceil_shift(rows, bins, pceil));
      if (rows_eval == 0) continue;
      if (tasks.size() >= o.max_tasks) raise(GF_ERUNTIME, "FFA search plan exceeds max_tasks");
      gf_ffa_task t{};
      t.downsample_factor = factor;
      t.effective_tsamp = eff;
      t.input_nsamples = n;
      t.prepared_nsamples = prepared;
      t.bins = bins;
      t.rows = rows;
      t.rows_eval = rows_eval;
      t.period_begin = eff * static_cast<double>(bins);
      t.period_end = evaluated_period_end(eff, bins, rows, rows_eval);
      tasks.push_back(t);
    }
  }
}

// ---- ffa_peak.cpp / dm_search.cpp ordering --------------------------------

bool finite_peak(const gf_peak& p) {
  return std::isfinite(p.snr) && std::isfinite(p.period) && std::isfinite(p.frequency);
}

bool better_ffa(const gf_peak& l, const gf_peak& r) {
  // ffa_peak.cpp:16-41 is_better_ffa_peak
  const bool lf = finite_peak(l), rf = finite_peak(r);
  if (lf != rf) return lf;
  if (l.snr != r.snr) return l.snr > r.snr;
  if (l.period != r.period) return l.period < r.period;
  if (l.frequency != r.frequency) return l.frequency < r.frequency;
  if (l.width != r.width) return l.width < r.width;
  if (l.phase != r.phase) return l.phase < r.phase;
  if (l.shift != r.shift) return l.shift < r.shift;
  return l.bins < r.bins;
}

bool better_dm(const gf_peak& l, const gf_peak& r) {
  // dm_search.cpp:89-100 is_better_dm_peak
  if (better_ffa(l, r)) return true;
  if (better_ffa(r, l)) return false;
  if (l.dm_index != r.dm_index) return l.dm_index < r.dm_index;
  return l.dm < r.dm;
}

// ---- candidate.cpp ---------------------------------------------------------

bool peak_order(const gf_peak& l, const gf_peak& r) {
  if (l.frequency != r.frequency) return l.frequency < r.frequency;
  if (l.width != r.width) return l.width < r.width;
  if (l.dm_index != r.dm_index) return l.dm_index < r.dm_index;
  return better_dm(l, r);
}

bool dm_group_order(const gf_peak& l, const gf_peak& r) {
  if (l.dm_index != r.dm_index) return l.dm_index < r.dm_index;
  if (l.width != r.width) return l.width < r.width;
  return l.frequency < r.frequency;
}

bool width_dm_group_order(const gf_peak& l, const gf_peak& r) {
  if (l.width != r.width) return l.width < r.width;
  return dm_group_order(l, r);
}

gf_candidate make_candidate(const gf_peak* b, const gf_peak* e) {
  // candidate.cpp:101-138
  const gf_peak* best = b;
  uint64_t dmin = std::numeric_limits<uint64_t>::max(), dmax = 0;
  double fmin = std::numeric_limits<double>::infinity(), fmax = -std::numeric_limits<double>::infinity();
  for (const gf_peak* p = b; p != e; ++p) {
    if (better_dm(*p, *best)) best = p;
    dmin = std::min(dmin, p->dm_index);
    dmax = std::max(dmax, p->dm_index);
    fmin = std::min(fmin, p->frequency);
    fmax = std::max(fmax, p->frequency);
  }
  gf_candidate c{};
  c.dm = best->dm;
  c.dm_index = best->dm_index;
  c.period = best->period;
  c.frequency = best->frequency;
  c.width = best->width;
  c.duty_cycle = best->duty_cycle;
  c.snr = best->snr;
  c.peak_count = static_cast<uint64_t>(e - b);
  c.dm_index_min = dmin;
  c.dm_index_max = dmax;
  c.frequency_min = fmin;
  c.frequency_max = fmax;
  c.best_peak = *best;
  return c;
}

void append_dm_clusters(gf_peak* b, gf_peak* e, const gf_candidate_options& o, std::vector<gf_candidate>& out) {
  // candidate.cpp:140-171
  if (b == e) return;
  if (o.cluster_across_widths) std::sort(b, e, dm_group_order);
  else std::sort(b, e, width_dm_group_order);
  gf_peak* cluster = b;
  uint64_t prev_dm = b->dm_index, prev_w = b->width;
  for (gf_peak* p = b + 1; p != e; ++p) {
    const bool same_w = o.cluster_across_widths || p->width == prev_w;
    const bool same_dm = p->dm_index <= prev_dm || p->dm_index - prev_dm <= o.dm_cluster_radius;
    if (!same_w || !same_dm) {
      out.push_back(make_candidate(cluster, p));
      cluster = p;
    }
    prev_dm = p->dm_index;
    prev_w = p->width;
  }
  out.push_back(make_candidate(cluster, e));
}

bool better_candidate(const gf_candidate& l, const gf_candidate& r) {
  // candidate.cpp:48-62
  if (better_dm(l.best_peak, r.best_peak)) return true;
  if (better_dm(r.best_peak, l.best_peak)) return false;
  if (l.peak_count != r.peak_count) return l.peak_count > r.peak_count;
  if (l.frequency != r.frequency) return l.frequency < r.frequency;
  return l.dm_index < r.dm_index;
}

}  // namespace

// candidate.cpp:205-206: rank by is_better_candidate
void rank_candidates(std::vector<gf_candidate>& candidates) {
  std::sort(candidates.begin(), candidates.end(), better_candidate);
}

}  // namespace gf

using namespace gf;

extern "C" const char* gf_last_error(void) { return gf::last_error(); }

extern "C" const char* gf_status_string(int status) {
  switch (status) {
    case GF_OK: return "success";
    case GF_EINVAL: return "invalid argument";
    case GF_EOVERFLOW: return "overflow";
    case GF_ERUNTIME: return "runtime error";
    case GF_ENOMEM: return "out of memory";
    case GF_ECUDA: return "CUDA error";
    case GF_EDATA: return "data error reported by the device";
    case GF_EOVERFLOW_PEAKS: return "peak buffer overflow";
    default: return "unknown status";
  }
}

extern "C" const char* gf_build_info(void) {
  return "gaffa_b200: sm_100a; kernels: stage_kernel, dedisperse_bytes_kernel, subband_stage2_u32_kernel, "
         "scrunch_kernel, running_median_kernel, detrend_kernel, stats_kernel, normalise_kernel, "
         "prepare_kernel, ffa_small_kernel, ffa_cluster_kernel, ffa_level_kernel, fold_partial_kernel, "
         "fold_reduce_kernel, synth_kernel";
}

// cuda_device_count / cuda_runtime_version (src/gaffa/vector_add.cu:75-86):
// the devices visible to the runtime this library links, and its version
extern "C" int gf_cuda_device_count(int32_t* count) {
  return guarded([&] {
    check_arg(count != nullptr, "null argument");
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
      cudaGetLastError();  // clear the sticky-free error and report no devices
      n = 0;
    } else {
      cuda_check(e, "cudaGetDeviceCount");
    }
    *count = n;
  });
}

extern "C" int gf_cuda_runtime_version(int32_t* version) {
  return guarded([&] {
    check_arg(version != nullptr, "null argument");
    int v = 0;
    cuda_check(cudaRuntimeGetVersion(&v), "cudaRuntimeGetVersion");
    *version = v;
  });
}

extern "C" int gf_make_riptide_ffa_plan(uint64_t nsamples, double tsamp, const gf_plan_options* options,
                                        gf_ffa_task* tasks, uint64_t task_capacity, uint64_t* ntasks,
                                        uint64_t* widths, uint64_t width_capacity, uint64_t* nwidths) {
  return guarded([&] {
    check_arg(options && ntasks && nwidths, "null argument");
    std::vector<gf_ffa_task> t;
    std::vector<uint64_t> w;
    make_plan(nsamples, tsamp, *options, t, w);
    *ntasks = t.size();
    *nwidths = w.size();
    if (tasks && task_capacity) std::memcpy(tasks, t.data(), std::min<uint64_t>(task_capacity, t.size()) * sizeof(gf_ffa_task));
    if (widths && width_capacity) std::memcpy(widths, w.data(), std::min<uint64_t>(width_capacity, w.size()) * sizeof(uint64_t));
  });
}

extern "C" int gf_sort_peaks(gf_peak* peaks, uint64_t n) {
  return guarded([&] {
    check_arg(n == 0 || peaks, "null argument");
    std::sort(peaks, peaks + n, better_dm);
  });
}

extern "C" int gf_select_candidates(const gf_peak* peaks, uint64_t n, double tobs, const gf_candidate_options* o,
                                    gf_candidate* out, uint64_t capacity, uint64_t* ncand) {
  return guarded([&] {
    check_arg(o && ncand, "null argument");
    check_arg(tobs > 0.0 && std::isfinite(tobs), "Candidate selection observation_seconds must be finite and > 0");
    check_arg(o->frequency_cluster_radius >= 0.0 && std::isfinite(o->frequency_cluster_radius),
              "Candidate selection frequency_cluster_radius must be finite and >= 0");
    *ncand = 0;
    if (n == 0) return;
    check_arg(peaks != nullptr, "null argument");
    std::vector<gf_peak> sorted(peaks, peaks + n);
    for (const auto& p : sorted)
      check_arg(std::isfinite(p.dm) && std::isfinite(p.period) && std::isfinite(p.frequency) &&
                    std::isfinite(p.duty_cycle) && std::isfinite(p.snr),
                "Candidate selection peaks must contain finite scientific values");
    std::sort(sorted.begin(), sorted.end(), peak_order);
    const double radius = o->frequency_cluster_radius / tobs;
    std::vector<gf_candidate> cands;
    gf_peak* fb = sorted.data();
    double prev = fb->frequency;
    gf_peak* end = sorted.data() + sorted.size();
    for (gf_peak* p = fb + 1; p != end; ++p) {
      if (p->frequency - prev > radius) {
        append_dm_clusters(fb, p, *o, cands);
        fb = p;
      }
      prev = p->frequency;
    }
    append_dm_clusters(fb, end, *o, cands);
    std::sort(cands.begin(), cands.end(), better_candidate);
    if (o->max_candidates != 0 && cands.size() > o->max_candidates) cands.resize(o->max_candidates);
    *ncand = cands.size();
    if (out && capacity) std::memcpy(out, cands.data(), std::min<uint64_t>(capacity, cands.size()) * sizeof(gf_candidate));
  });
}

// ---------------------------------------------------------------------------
// Harmonic flagging (src/gaffa/harmonic.cpp:14-311)
// ---------------------------------------------------------------------------

namespace {

// Reduced ratios n/d (n <= max_harmonic, d <= denominator_max, n != d) by
// value, then numerator, then denominator; duplicates removed
// (harmonic.cpp:94-135).
std::vector<HarmonicRatio> harmonic_ratios(uint64_t max_harmonic, uint64_t denominator_max) {
  std::vector<HarmonicRatio> r;
  r.reserve(max_harmonic * denominator_max);
  for (uint64_t a = 1; a <= max_harmonic; ++a) {
    for (uint64_t b = 1; b <= denominator_max; ++b) {
      const uint64_t g = std::gcd(a, b);
      if (a / g == b / g) continue;
      r.push_back(HarmonicRatio{static_cast<int32_t>(a / g), static_cast<int32_t>(b / g),
                                static_cast<double>(a / g) / static_cast<double>(b / g)});
    }
  }
  std::sort(r.begin(), r.end(), [](const HarmonicRatio& x, const HarmonicRatio& y) {
    if (x.value != y.value) return x.value < y.value;
    if (x.num != y.num) return x.num < y.num;
    return x.den < y.den;
  });
  r.erase(std::unique(r.begin(), r.end(),
                      [](const HarmonicRatio& x, const HarmonicRatio& y) { return x.num == y.num && x.den == y.den; }),
          r.end());
  return r;
}

// harmonic.cpp:21-35
bool harmonic_rank(const gf_candidate& l, const gf_candidate& r) {
  if (l.snr != r.snr) return l.snr > r.snr;
  if (l.peak_count != r.peak_count) return l.peak_count > r.peak_count;
  if (l.frequency != r.frequency) return l.frequency < r.frequency;
  return l.dm_index < r.dm_index;
}

gf_harmonic_options default_harmonic_options() {
  gf_harmonic_options o{};
  o.max_harmonic = 16;
  o.denominator_max = 5;
  o.frequency_tolerance_bins = 1.5;
  o.phase_distance_max = 1.0;
  o.dm_distance_max = 3.0;
  o.use_snr_consistency = 0;
  o.snr_distance_max = 3.0;
  return o;
}

}  // namespace

namespace {

// |1/lo^2 - 1/hi^2| of the band (harmonic.cpp:170-179)
double harmonic_band(const gf_harmonic_context& ctx) {
  const double lo = std::min(ctx.frequency_low_mhz, ctx.frequency_high_mhz);
  const double hi = std::max(ctx.frequency_low_mhz, ctx.frequency_high_mhz);
  return std::abs(1.0 / (lo * lo) - 1.0 / (hi * hi));
}

// flag_harmonics_cpu (harmonic.cpp:245-292); device_id >= 0 marks the pairs
// on that device
int flag_harmonics(const gf_candidate* candidates, uint64_t n, const gf_harmonic_context* ctx,
                   const gf_harmonic_options* options, gf_candidate* sorted_out, gf_harmonic_relation* rel,
                   int device_id, void* stream);

}  // namespace

extern "C" int gf_flag_harmonics(const gf_candidate* candidates, uint64_t n, const gf_harmonic_context* ctx,
                                 const gf_harmonic_options* options, gf_candidate* sorted_out,
                                 gf_harmonic_relation* rel) {
  return flag_harmonics(candidates, n, ctx, options, sorted_out, rel, -1, nullptr);
}

extern "C" int gf_flag_harmonics_device(const gf_candidate* candidates, uint64_t n, const gf_harmonic_context* ctx,
                                        const gf_harmonic_options* options, gf_candidate* sorted_out,
                                        gf_harmonic_relation* rel, int32_t device_id, void* stream) {
  return flag_harmonics(candidates, n, ctx, options, sorted_out, rel, device_id < 0 ? 0 : device_id, stream);
}

namespace {

int flag_harmonics(const gf_candidate* candidates, uint64_t n, const gf_harmonic_context* ctx,
                   const gf_harmonic_options* options, gf_candidate* sorted_out, gf_harmonic_relation* rel,
                   int device_id, void* stream) {
  return guarded([&] {
    check_arg(ctx != nullptr, "null argument");
    const gf_harmonic_options o = options ? *options : default_harmonic_options();
    // harmonic.cpp:37-92
    check_arg(ctx->observation_seconds > 0.0 && std::isfinite(ctx->observation_seconds),
              "Harmonic context observation_seconds must be finite and > 0");
    check_arg(ctx->frequency_low_mhz > 0.0 && ctx->frequency_high_mhz > 0.0 && std::isfinite(ctx->frequency_low_mhz) &&
                  std::isfinite(ctx->frequency_high_mhz),
              "Harmonic context frequencies must be finite and > 0 MHz");
    check_arg(o.max_harmonic >= 2, "Harmonic max_harmonic must be >= 2");
    check_arg(o.denominator_max > 0, "Harmonic denominator_max must be > 0");
    check_arg(o.frequency_tolerance_bins >= 0.0 && std::isfinite(o.frequency_tolerance_bins),
              "Harmonic frequency_tolerance_bins must be finite and >= 0");
    check_arg(o.phase_distance_max >= 0.0 && std::isfinite(o.phase_distance_max),
              "Harmonic phase_distance_max must be finite and >= 0");
    check_arg(o.dm_distance_max >= 0.0 && std::isfinite(o.dm_distance_max),
              "Harmonic dm_distance_max must be finite and >= 0");
    check_arg(o.snr_distance_max >= 0.0 && std::isfinite(o.snr_distance_max),
              "Harmonic snr_distance_max must be finite and >= 0");
    if (n == 0) return;
    check_arg(candidates && sorted_out && rel, "null argument");
    for (uint64_t i = 0; i < n; ++i) {
      const gf_candidate& c = candidates[i];
      check_arg(std::isfinite(c.dm) && std::isfinite(c.period) && std::isfinite(c.frequency) &&
                    std::isfinite(c.duty_cycle) && std::isfinite(c.snr),
                "Harmonic candidates must contain finite scientific values");
      check_arg(c.frequency > 0.0 && c.period > 0.0 && c.duty_cycle > 0.0 && c.snr >= 0.0f,
                "Harmonic candidate frequency, period, duty_cycle, and snr are invalid");
    }
    std::vector<gf_candidate> s(candidates, candidates + n);
    std::sort(s.begin(), s.end(), harmonic_rank);
    std::vector<gf_harmonic_relation> rl(n);
    for (auto& r : rl) {
      r = gf_harmonic_relation{};
      r.parent_index = GF_NO_HARMONIC_PARENT;
      r.numerator = 1;
      r.denominator = 1;
    }
    const std::vector<HarmonicRatio> ratios = harmonic_ratios(o.max_harmonic, o.denominator_max);
    const double band = harmonic_band(*ctx);
    std::vector<HarmonicInput> in(n);
    for (uint64_t i = 0; i < n; ++i) in[i] = harmonic_input(s[i]);
    if (device_id >= 0) {
      // the pairwise marking on the device; the relations from the same test on the host
      std::vector<uint32_t> parent(n);
      flag_harmonics_on_device(in, ratios, ctx->observation_seconds, band, o, device_id, stream, parent);
      for (uint64_t ci = 0; ci < n; ++ci) {
        if (parent[ci] == UINT32_MAX) continue;
        const bool ok = harmonic_test(in[parent[ci]], in[ci], ratios.data(), static_cast<int>(ratios.size()),
                                      ctx->observation_seconds, band, o, parent[ci], &rl[ci]);
        if (!ok) raise(GF_ERUNTIME, "device harmonic flagging disagrees with the host test");
      }
    } else {
      // a candidate already flagged is neither a parent nor re-tested
      // (harmonic.cpp:271-289)
      for (uint64_t pi = 0; pi < n; ++pi) {
        if (rl[pi].is_harmonic) continue;
        for (uint64_t ci = pi + 1; ci < n; ++ci) {
          if (rl[ci].is_harmonic) continue;
          harmonic_test(in[pi], in[ci], ratios.data(), static_cast<int>(ratios.size()), ctx->observation_seconds,
                        band, o, pi, &rl[ci]);
        }
      }
    }
    std::memcpy(sorted_out, s.data(), n * sizeof(gf_candidate));
    std::memcpy(rel, rl.data(), n * sizeof(gf_harmonic_relation));
  });
}

}  // namespace

extern "C" int gf_remove_harmonics(const gf_candidate* sorted, const gf_harmonic_relation* rel, uint64_t n,
                                   uint64_t max_candidates, gf_candidate* out, uint64_t* nout) {
  return guarded([&] {
    check_arg(nout != nullptr, "null argument");
    *nout = 0;
    if (n == 0) return;
    check_arg(sorted && rel && out, "null argument");
    uint64_t k = 0;
    for (uint64_t i = 0; i < n; ++i) {
      if (rel[i].is_harmonic) continue;
      out[k++] = sorted[i];
      if (max_candidates != 0 && k >= max_candidates) break;
    }
    *nout = k;
  });
}
