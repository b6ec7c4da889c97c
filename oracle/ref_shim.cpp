// ref_shim.cpp -- C-ABI over the reference's own CPU implementation.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference C++ sources where they lie (src/gaffa/*.cpp of
// lintian233/gaffa) into oracle/_ref/libgaffa_ref.so.  The exported gfr_*
// functions have the same signatures as the gfo_* restatement in
// gaffa_oracle.h, so tests can run both on one input and compare bit for bit,
// and bench.py's reference arm can time the reference CPU path itself.
#include "gaffa_oracle.h"

#include "gaffa/candidate.h"
#include "gaffa/dedispersion.h"
#include "gaffa/dm_search.h"
#include "gaffa/ffa.h"
#include "gaffa/filterbank.h"
#include "gaffa/ffa_detection.h"
#include "gaffa/ffa_plan.h"
#include "gaffa/ffa_search.h"
#include "gaffa/folding.h"
#include "gaffa/harmonic.h"
#include "gaffa/preprocessing.h"
#include "gaffa/time_series.h"

#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>
#include <variant>
#include <vector>

namespace {

thread_local std::string g_error;

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return GFO_OK;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return GFO_EINVAL;
  } catch (const std::overflow_error& e) {
    g_error = e.what();
    return GFO_EOVERFLOW;
  } catch (const std::out_of_range& e) {
    g_error = e.what();
    return GFO_ERANGE;
  } catch (const std::bad_alloc& e) {
    g_error = e.what();
    return GFO_ENOMEM;
  } catch (const std::exception& e) {
    g_error = e.what();
    return GFO_ERUNTIME;
  }
}

gaffa::RiptideFfaPlanOptions plan_options(const gfo_plan_options* o) {
  return gaffa::RiptideFfaPlanOptions{
      .period_min = o->period_min,
      .period_max = o->period_max,
      .bins_min = o->bins_min,
      .bins_max = o->bins_max,
      .min_periods = o->min_periods,
      .duty_cycle_max = o->duty_cycle_max,
      .width_trial_spacing = o->width_trial_spacing,
      .max_tasks = o->max_tasks,
  };
}

gaffa::FfaSearchTask to_task(const gfo_ffa_task& t) {
  return gaffa::FfaSearchTask{
      .downsample_factor = t.downsample_factor,
      .effective_tsamp = t.effective_tsamp,
      .input_nsamples = t.input_nsamples,
      .prepared_nsamples = t.prepared_nsamples,
      .bins = t.bins,
      .rows = t.rows,
      .rows_eval = t.rows_eval,
      .period_begin = t.period_begin,
      .period_end = t.period_end,
  };
}

gfo_peak to_peak(const gaffa::FfaPeak& p, double dm, std::size_t dm_index) {
  gfo_peak out{};
  out.dm = dm;
  out.dm_index = dm_index;
  out.period = p.period;
  out.frequency = p.frequency;
  out.width = p.width;
  out.duty_cycle = p.duty_cycle;
  out.width_index = p.width_index;
  out.period_index = p.period_index;
  out.phase = p.phase;
  out.shift = p.shift;
  out.bins = p.bins;
  out.snr = p.snr;
  return out;
}

gaffa::DmPeak from_peak(const gfo_peak& p) {
  return gaffa::DmPeak{
      .dm = p.dm,
      .dm_index = p.dm_index,
      .peak = gaffa::FfaPeak{
          .period = p.period,
          .frequency = p.frequency,
          .width = p.width,
          .duty_cycle = p.duty_cycle,
          .width_index = p.width_index,
          .period_index = p.period_index,
          .phase = p.phase,
          .shift = p.shift,
          .bins = p.bins,
          .snr = p.snr,
      },
  };
}

template <typename T>
T* copy_out(const std::vector<T>& v) {
  T* p = static_cast<T*>(std::malloc(sizeof(T) * (v.empty() ? 1 : v.size())));
  if (!p) throw std::bad_alloc();
  if (!v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
  return p;
}

gaffa::MultiDmDedispersionPlan multi_plan(double dm_low, double dm_step,
                                          uint64_t ndm, double fref,
                                          double tsamp, uint64_t cb,
                                          uint64_t ce) {
  return gaffa::MultiDmDedispersionPlan{
      .dm_low = dm_low,
      .dm_step = dm_step,
      .ndm = ndm,
      .ref_frequency_mhz = fref,
      .tsamp = tsamp,
      .chan_begin = cb,
      .chan_end = ce,
  };
}

}  // namespace

extern "C" {

const char* gfr_last_error(void) { return g_error.c_str(); }
void gfr_free(void* p) { std::free(p); }

int gfr_dedisperse_multi_dm_u8(const uint8_t* in, uint64_t nsamples,
                               uint64_t nchans, const double* freq,
                               double dm_low, double dm_step, uint64_t ndm,
                               double fref, double tsamp, uint64_t cb,
                               uint64_t ce, uint32_t* out) {
  return guarded([&] {
    const gaffa::SampleShape shape{nsamples, 1, nchans};
    const auto view = gaffa::make_host_sample_view<std::uint8_t>(
        std::span<const std::uint8_t>(in, nsamples * nchans), shape);
    const auto r = gaffa::dedisperse_multi_dm_cpu(
        view, std::span<const double>(freq, nchans),
        multi_plan(dm_low, dm_step, ndm, fref, tsamp, cb, ce));
    std::memcpy(out, r.data.data(), r.data.size() * sizeof(uint32_t));
  });
}

int gfr_dedisperse_subband_u8(const uint8_t* in, uint64_t nsamples,
                              uint64_t nchans, const double* freq,
                              double dm_low, double dm_step, uint64_t ndm,
                              double fref, double tsamp, uint64_t cb,
                              uint64_t ce, uint64_t subband_channels,
                              uint64_t ndm_per_nominal, uint32_t* out) {
  return guarded([&] {
    const gaffa::SampleShape shape{nsamples, 1, nchans};
    const auto view = gaffa::make_host_sample_view<std::uint8_t>(
        std::span<const std::uint8_t>(in, nsamples * nchans), shape);
    const auto r = gaffa::dedisperse_subband_cpu(
        view, std::span<const double>(freq, nchans),
        multi_plan(dm_low, dm_step, ndm, fref, tsamp, cb, ce),
        gaffa::SubbandDedispersionOptions{
            .subband_channels = subband_channels,
            .ndm_per_nominal = ndm_per_nominal});
    std::memcpy(out, r.data.data(), r.data.size() * sizeof(uint32_t));
  });
}

int gfr_downsample_weighted_sum(const float* in, uint64_t n, double factor,
                                float* out) {
  return guarded([&] {
    const auto r =
        gaffa::downsample_weighted_sum_cpu(std::span<const float>(in, n), factor);
    std::memcpy(out, r.data(), r.size() * sizeof(float));
  });
}

int gfr_downsampled_variance(uint64_t n, double factor, double* out) {
  return guarded([&] { *out = gaffa::downsampled_variance(n, factor); });
}

int gfr_preprocess_riptide(float* data, uint64_t n, double tsamp,
                           const gfo_preprocess_options* o) {
  return guarded([&] {
    gaffa::RiptidePreprocessOptions opts;
    opts.running_median_width_seconds = o->window_seconds;
    opts.running_median_min_points = o->min_points;
    opts.normalise = o->normalise != 0;
    opts.normalise_options.reject_constant = o->reject_constant != 0;
    const auto plan = gaffa::make_riptide_preprocess_plan(tsamp, opts);
    gaffa::TimeSeries ts{std::vector<float>(data, data + n), tsamp};
    const auto r = gaffa::preprocess_time_series_cpu(ts, plan);
    std::memcpy(data, r.data.data(), n * sizeof(float));
  });
}

int gfr_make_riptide_ffa_plan(uint64_t nsamples, double tsamp,
                              const gfo_plan_options* o, gfo_ffa_task** tasks,
                              uint64_t* ntasks, uint64_t** widths,
                              uint64_t* nwidths) {
  return guarded([&] {
    const auto plan = gaffa::make_riptide_ffa_plan(nsamples, tsamp, plan_options(o));
    std::vector<gfo_ffa_task> t;
    for (const auto& x : plan.tasks) {
      t.push_back(gfo_ffa_task{x.downsample_factor, x.effective_tsamp,
                               x.input_nsamples, x.prepared_nsamples, x.bins,
                               x.rows, x.rows_eval, x.period_begin,
                               x.period_end});
    }
    std::vector<uint64_t> w(plan.width_trials.begin(), plan.width_trials.end());
    *tasks = copy_out(t);
    *ntasks = t.size();
    *widths = copy_out(w);
    *nwidths = w.size();
  });
}

int gfr_ffa_transform(const float* in, uint64_t rows, uint64_t bins,
                      float* out) {
  return guarded([&] {
    std::vector<float> scratch(rows * bins);
    gaffa::ffa_transform_block_cpu(std::span<const float>(in, rows * bins),
                                   gaffa::FfaTransformShape{rows, bins}, scratch,
                                   std::span<float>(out, rows * bins));
  });
}

int gfr_ffa_search(const float* series, uint64_t n, const gfo_ffa_task* tasks,
                   uint64_t ntasks, const uint64_t* widths, uint64_t nwidths,
                   float thr, uint64_t max_peaks, gfo_peak** peaks,
                   uint64_t* npeaks) {
  return guarded([&] {
    gaffa::FfaSearchPlan plan;
    for (uint64_t i = 0; i < ntasks; ++i) plan.tasks.push_back(to_task(tasks[i]));
    plan.width_trials.assign(widths, widths + nwidths);
    const auto r = gaffa::search_ffa_cpu(
        std::span<const float>(series, n), plan,
        gaffa::FfaSearchOptions{.snr_threshold = thr, .max_peaks = max_peaks});
    std::vector<gfo_peak> out;
    for (const auto& p : r.peaks) out.push_back(to_peak(p, 0.0, 0));
    *peaks = copy_out(out);
    *npeaks = out.size();
  });
}

// find_dm_peaks_cpu, or (with a width override) the same per-DM composition
// dm_time_series_cpu -> preprocess_time_series_cpu -> search_ffa_cpu that
// find_dm_peaks_cpu performs, with the plan's width trials replaced.
int gfr_find_dm_peaks_u32(const uint32_t* data, uint64_t ndm, uint64_t nsamples,
                          const double* dms, double tsamp,
                          const gfo_plan_options* po,
                          const gfo_preprocess_options* pre, float thr,
                          uint64_t max_peaks, const uint64_t* wo, uint64_t nwo,
                          gfo_peak** peaks, uint64_t* npeaks) {
  return guarded([&] {
    gaffa::DedispersedResult<std::uint32_t> input;
    input.data.assign(data, data + ndm * nsamples);
    input.shape = gaffa::DedispersedShape{ndm, nsamples};
    gaffa::PreprocessPlan pplan;
    if (pre) {
      gaffa::RiptidePreprocessOptions opts;
      opts.running_median_width_seconds = pre->window_seconds;
      opts.running_median_min_points = pre->min_points;
      opts.normalise = pre->normalise != 0;
      opts.normalise_options.reject_constant = pre->reject_constant != 0;
      pplan = gaffa::make_riptide_preprocess_plan(tsamp, opts);
    }
    std::vector<gfo_peak> out;
    if (!(wo && nwo)) {
      const auto r = gaffa::find_dm_peaks_cpu(
          input, std::span<const double>(dms, ndm), tsamp,
          gaffa::DmSearchOptions{.plan = plan_options(po),
                                 .preprocess = pplan,
                                 .snr_threshold = thr,
                                 .max_peaks = max_peaks});
      for (const auto& p : r.peaks) out.push_back(to_peak(p.peak, p.dm, p.dm_index));
    } else {
      gaffa::FfaSearchPlan plan =
          gaffa::make_riptide_ffa_plan(nsamples, tsamp, plan_options(po));
      plan.width_trials.assign(wo, wo + nwo);
      std::vector<std::vector<gfo_peak>> per_dm(ndm);
      std::exception_ptr error;
#pragma omp parallel for schedule(dynamic, 1)
      for (int64_t d = 0; d < static_cast<int64_t>(ndm); ++d) {
        try {
          gaffa::TimeSeries ts = gaffa::dm_time_series_cpu(input, d, tsamp);
          if (!pplan.steps.empty()) ts = gaffa::preprocess_time_series_cpu(ts, pplan);
          const auto r = gaffa::search_ffa_cpu(
              ts.data, plan,
              gaffa::FfaSearchOptions{.snr_threshold = thr, .max_peaks = max_peaks});
          for (const auto& p : r.peaks)
            per_dm[d].push_back(to_peak(p, dms[d], static_cast<std::size_t>(d)));
        } catch (...) {
#pragma omp critical(gfr_error)
          if (!error) error = std::current_exception();
        }
      }
      if (error) std::rethrow_exception(error);
      std::vector<gaffa::DmPeak> all;
      for (const auto& v : per_dm)
        for (const auto& p : v) all.push_back(from_peak(p));
      // dm_search.cpp:89-100 is_better_dm_peak ordering
      std::sort(all.begin(), all.end(), [](const gaffa::DmPeak& l, const gaffa::DmPeak& r) {
        if (gaffa::is_better_ffa_peak(l.peak, r.peak)) return true;
        if (gaffa::is_better_ffa_peak(r.peak, l.peak)) return false;
        if (l.dm_index != r.dm_index) return l.dm_index < r.dm_index;
        return l.dm < r.dm;
      });
      for (const auto& p : all) out.push_back(to_peak(p.peak, p.dm, p.dm_index));
    }
    *peaks = copy_out(out);
    *npeaks = out.size();
  });
}

int gfr_select_candidates(const gfo_peak* peaks, uint64_t n, double tobs,
                          const gfo_candidate_options* o,
                          gfo_candidate** candidates, uint64_t* ncandidates) {
  return guarded([&] {
    std::vector<gaffa::DmPeak> in;
    for (uint64_t i = 0; i < n; ++i) in.push_back(from_peak(peaks[i]));
    const auto r = gaffa::select_candidates_cpu(
        in, tobs,
        gaffa::CandidateSelectionOptions{
            .frequency_cluster_radius = o->frequency_cluster_radius,
            .dm_cluster_radius = o->dm_cluster_radius,
            .cluster_across_widths = o->cluster_across_widths != 0,
            .max_candidates = o->max_candidates});
    std::vector<gfo_candidate> out;
    for (const auto& c : r) {
      gfo_candidate x{};
      x.dm = c.dm;
      x.dm_index = c.dm_index;
      x.period = c.period;
      x.frequency = c.frequency;
      x.width = c.width;
      x.duty_cycle = c.duty_cycle;
      x.snr = c.snr;
      x.peak_count = c.peak_count;
      x.dm_index_min = c.dm_index_min;
      x.dm_index_max = c.dm_index_max;
      x.frequency_min = c.frequency_min;
      x.frequency_max = c.frequency_max;
      x.best_peak = to_peak(c.best_peak.peak, c.best_peak.dm, c.best_peak.dm_index);
      out.push_back(x);
    }
    *candidates = copy_out(out);
    *ncandidates = out.size();
  });
}

int gfr_fold_time_series_f32(const float* in, uint64_t n, double period,
                             double tsamp, uint64_t nbin, uint64_t start,
                             float* profile, double* exposure) {
  return guarded([&] {
    const auto r = gaffa::fold_time_series_cpu(
        std::span<const float>(in, n),
        gaffa::FoldOptions{.period = period, .tsamp = tsamp, .nbin = nbin,
                           .start_sample = start});
    std::memcpy(profile, r.profile.data(), nbin * sizeof(float));
    std::memcpy(exposure, r.exposure.data(), nbin * sizeof(double));
  });
}

int gfr_fold_time_series_u32(const uint32_t* in, uint64_t n, double period,
                             double tsamp, uint64_t nbin, uint64_t start,
                             float* profile, double* exposure) {
  return guarded([&] {
    const auto r = gaffa::fold_time_series_cpu(
        std::span<const std::uint32_t>(in, n),
        gaffa::FoldOptions{.period = period, .tsamp = tsamp, .nbin = nbin,
                           .start_sample = start});
    std::memcpy(profile, r.profile.data(), nbin * sizeof(float));
    std::memcpy(exposure, r.exposure.data(), nbin * sizeof(double));
  });
}


int gfr_flag_harmonics(const gfo_candidate* in, uint64_t n, const gfo_harmonic_context* ctx,
                       const gfo_harmonic_options* o, gfo_candidate* sorted,
                       gfo_harmonic_relation* rel) {
  return guarded([&] {
    std::vector<gaffa::Candidate> cands;
    for (uint64_t i = 0; i < n; ++i) {
      const gfo_candidate& c = in[i];
      gaffa::Candidate x{};
      x.dm = c.dm;
      x.dm_index = c.dm_index;
      x.period = c.period;
      x.frequency = c.frequency;
      x.width = c.width;
      x.duty_cycle = c.duty_cycle;
      x.snr = c.snr;
      x.peak_count = c.peak_count;
      x.dm_index_min = c.dm_index_min;
      x.dm_index_max = c.dm_index_max;
      x.frequency_min = c.frequency_min;
      x.frequency_max = c.frequency_max;
      x.best_peak = from_peak(c.best_peak);
      cands.push_back(x);
    }
    const auto r = gaffa::flag_harmonics_cpu(
        cands,
        gaffa::HarmonicContext{.observation_seconds = ctx->observation_seconds,
                               .frequency_low_mhz = ctx->frequency_low_mhz,
                               .frequency_high_mhz = ctx->frequency_high_mhz},
        gaffa::HarmonicOptions{.max_harmonic = o->max_harmonic,
                               .denominator_max = o->denominator_max,
                               .frequency_tolerance_bins = o->frequency_tolerance_bins,
                               .phase_distance_max = o->phase_distance_max,
                               .dm_distance_max = o->dm_distance_max,
                               .use_snr_consistency = o->use_snr_consistency != 0,
                               .snr_distance_max = o->snr_distance_max});
    for (size_t i = 0; i < r.size(); ++i) {
      const gaffa::Candidate& c = r[i].candidate;
      gfo_candidate& x = sorted[i];
      std::memset(&x, 0, sizeof x);
      x.dm = c.dm;
      x.dm_index = c.dm_index;
      x.period = c.period;
      x.frequency = c.frequency;
      x.width = c.width;
      x.duty_cycle = c.duty_cycle;
      x.snr = c.snr;
      x.peak_count = c.peak_count;
      x.dm_index_min = c.dm_index_min;
      x.dm_index_max = c.dm_index_max;
      x.frequency_min = c.frequency_min;
      x.frequency_max = c.frequency_max;
      x.best_peak = to_peak(c.best_peak.peak, c.best_peak.dm, c.best_peak.dm_index);
      const gaffa::HarmonicRelation& h = r[i].harmonic;
      gfo_harmonic_relation& y = rel[i];
      std::memset(&y, 0, sizeof y);
      y.is_harmonic = h.is_harmonic ? 1 : 0;
      y.parent_index = h.parent_index;
      y.numerator = h.numerator;
      y.denominator = h.denominator;
      y.frequency_error_bins = h.frequency_error_bins;
      y.phase_distance = h.phase_distance;
      y.dm_distance = h.dm_distance;
      y.expected_snr = h.expected_snr;
      y.snr_distance = h.snr_distance;
    }
  });
}

int gfr_remove_harmonics(const gfo_candidate* sorted, const gfo_harmonic_relation* rel, uint64_t n,
                         uint64_t max_candidates, gfo_candidate* out, uint64_t* nout) {
  return guarded([&] {
    // round-trip through the reference types: only is_harmonic and the
    // candidate order matter to remove_harmonics_cpu
    std::vector<gaffa::HarmonicCandidate> in(n);
    for (uint64_t i = 0; i < n; ++i) {
      in[i].candidate.frequency = static_cast<double>(i);  // index carrier
      in[i].harmonic.is_harmonic = rel[i].is_harmonic != 0;
    }
    const auto r = gaffa::remove_harmonics_cpu(in, max_candidates);
    for (size_t i = 0; i < r.size(); ++i) out[i] = sorted[static_cast<uint64_t>(r[i].frequency)];
    *nout = r.size();
  });
}

int gfr_dedisperse_spectrum_u8(const uint8_t* in, uint64_t nsamples, uint64_t nchans, const double* freq,
                               double dm, double ref, double tsamp, uint64_t cb, uint64_t ce, uint8_t* out,
                               uint64_t* nout) {
  return guarded([&] {
    const auto r = gaffa::dedisperse_spectrum_cpu(
        gaffa::HostSampleView<std::uint8_t>{std::span<const std::uint8_t>(in, nsamples * nchans),
                                            gaffa::SampleShape{nsamples, 1, nchans}},
        std::span<const double>(freq, nchans),
        gaffa::SingleDmDedispersionPlan{.dm = dm, .ref_frequency_mhz = ref, .tsamp = tsamp,
                                        .chan_begin = cb, .chan_end = ce});
    *nout = r.shape.nsamples;
    if (out) std::memcpy(out, r.data.data(), r.data.size());
  });
}

// read_filterbank (io/filterbank.cpp:335-348): header, frequencies and the
// samples' bytes (malloc'd, released with gfr_free).
int gfr_read_filterbank(const char* path, int preserve, gfo_filterbank_header* h, double* freq,
                        uint64_t capacity, void** samples, uint64_t* nbytes) {
  return guarded([&] {
    gaffa::FilterbankReadOptions o;
    if (preserve) o.channel_order = gaffa::ChannelOrderPolicy::PreserveFileOrder;
    const auto d = gaffa::read_filterbank(path, o);
    const auto& x = d.header;
    std::memset(h, 0, sizeof *h);
    h->header_size = x.header_size;
    h->nsamples = x.nsamples;
    h->telescope_id = x.telescope_id; h->machine_id = x.machine_id; h->data_type = x.data_type;
    h->barycentric = x.barycentric; h->pulsarcentric = x.pulsarcentric; h->ibeam = x.ibeam;
    h->nbeams = x.nbeams; h->npuls = x.npuls; h->nbins = x.nbins; h->nbits = x.nbits; h->nifs = x.nifs;
    h->nchans = x.nchans;
    h->az_start = x.az_start; h->za_start = x.za_start; h->src_raj = x.src_raj; h->src_dej = x.src_dej;
    h->tstart = x.tstart; h->tsamp = x.tsamp; h->fch1 = x.fch1; h->foff = x.foff; h->refdm = x.refdm;
    h->period = x.period;
    h->uses_frequency_table = x.uses_frequency_table ? 1 : 0;
    std::strncpy(h->rawdatafile, x.rawdatafile.c_str(), sizeof h->rawdatafile - 1);
    std::strncpy(h->source_name, x.source_name.c_str(), sizeof h->source_name - 1);
    for (uint64_t i = 0; i < capacity && i < x.frequency_table.size(); ++i) freq[i] = x.frequency_table[i];
    std::visit([&](const auto& v) {
      *nbytes = v.size() * sizeof(v[0]);
      *samples = std::malloc(*nbytes ? *nbytes : 1);
      if (*nbytes) std::memcpy(*samples, v.data(), *nbytes);
    }, d.samples);
  });
}

// fold_dedispersed_spectrum_view_cpu (folding.cpp:408-438) of a uint8
// [ns][nc] spectrum; outputs sized by the caller from nsubint (first call with
// cube == NULL returns it).
int gfr_fold_dedispersed_spectrum_u8(const uint8_t* in, uint64_t ns, uint64_t nc, double period, double tsamp,
                                     uint64_t nbin, double tsubint, uint64_t out_ch, uint64_t* nsubint,
                                     float* cube, double* exposure, float* profile, float* freq_phase,
                                     float* time_phase) {
  return guarded([&] {
    const auto r = gaffa::fold_dedispersed_spectrum_view_cpu(
        gaffa::HostSampleView<std::uint8_t>{std::span<const std::uint8_t>(in, ns * nc),
                                            gaffa::SampleShape{ns, 1, nc}},
        tsamp,
        gaffa::FoldDedispersedSpectrumOptions{.period = period, .nbin = nbin, .tsubint = tsubint,
                                              .output_channels = out_ch});
    *nsubint = r.nsubint;
    if (!cube) return;
    std::memcpy(cube, r.cube.data.data(), r.cube.data.size() * sizeof(float));
    std::memcpy(exposure, r.cube.exposure.data(), r.cube.exposure.size() * sizeof(double));
    std::memcpy(profile, r.profile.data(), r.profile.size() * sizeof(float));
    std::memcpy(freq_phase, r.freq_phase.data(), r.freq_phase.size() * sizeof(float));
    std::memcpy(time_phase, r.time_phase.data(), r.time_phase.size() * sizeof(float));
  });
}

}  // extern "C"
