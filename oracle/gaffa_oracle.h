/*
 * gaffa_oracle.h -- CPU restatement of gaffa's pulsar-search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product
 * in gaffa_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product never links or calls it.
 *
 * Every function restates the arithmetic of the reference C++ sources
 * (lintian233/gaffa, paths relative to that project) in plain C with the same
 * operation order, so results are bit-identical to the reference CPU path.
 * Parity of this restatement is pinned two ways (see tests/test_oracle_*.py):
 *   1. the reference's own golden vectors (tests/cpp/test_*.cpp), restated as
 *      fixtures in tests/golden/;
 *   2. fixtures produced by running the reference CPU sources compiled from
 *      their own files (oracle/Makefile -> oracle/_ref/), committed as .npz
 *      under tests/golden/ together with the script that generated them.
 *
 * Conventions: functions return 0 on success or a negative GFO_E* code and
 * record a message retrievable with gfo_last_error().  Buffers returned through
 * pointer-to-pointer arguments are malloc'd and released with gfo_free().
 */
#ifndef GAFFA_ORACLE_H
#define GAFFA_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  GFO_OK = 0,
  GFO_EINVAL = -1,   /* std::invalid_argument in the reference */
  GFO_EOVERFLOW = -2,/* std::overflow_error */
  GFO_ERUNTIME = -3, /* std::runtime_error (max_tasks / max_peaks guards) */
  GFO_ENOMEM = -4,
  GFO_ERANGE = -5    /* std::out_of_range */
};

typedef struct {
  double downsample_factor;
  double effective_tsamp;
  uint64_t input_nsamples;
  uint64_t prepared_nsamples;
  uint64_t bins;
  uint64_t rows;
  uint64_t rows_eval;
  double period_begin;
  double period_end;
} gfo_ffa_task; /* ffa_plan.h:8-32 FfaSearchTask */

typedef struct {
  double period_min;
  double period_max;
  uint64_t bins_min;
  uint64_t bins_max;
  uint64_t min_periods;
  double duty_cycle_max;
  double width_trial_spacing;
  uint64_t max_tasks;
} gfo_plan_options; /* ffa_plan.h:34-47 RiptideFfaPlanOptions */

typedef struct {
  double dm;
  uint64_t dm_index;
  double period;
  double frequency;
  uint64_t width;
  double duty_cycle;
  uint64_t width_index;
  uint64_t period_index;
  uint64_t phase;
  uint64_t shift;
  uint64_t bins;
  float snr;
  uint32_t reserved;
} gfo_peak; /* dm_search.h:16-20 DmPeak{dm, dm_index, FfaPeak ffa_peak.h:8-19} */

typedef struct {
  double dm;
  uint64_t dm_index;
  double period;
  double frequency;
  uint64_t width;
  double duty_cycle;
  float snr;
  uint32_t reserved;
  uint64_t peak_count;
  uint64_t dm_index_min;
  uint64_t dm_index_max;
  double frequency_min;
  double frequency_max;
  gfo_peak best_peak;
} gfo_candidate; /* candidate.h:11-28 Candidate */

typedef struct {
  double frequency_cluster_radius;
  uint64_t dm_cluster_radius;
  int32_t cluster_across_widths;
  int32_t reserved;
  uint64_t max_candidates;
} gfo_candidate_options; /* candidate.h:30-39 */

typedef struct {
  double window_seconds;   /* RiptidePreprocessOptions::running_median_width_seconds */
  uint64_t min_points;     /* running_median_min_points */
  int32_t normalise;       /* append a Normalise step */
  int32_t reject_constant; /* NormaliseOptions::reject_constant */
} gfo_preprocess_options; /* preprocessing.h:37-42 */

const char* gfo_last_error(void);
void gfo_free(void* p);

/* ---- dedispersion (internal/dedispersion_delay.h, dedispersion.cpp) ---- */
int32_t gfo_delay_bins(double dm, double frequency_mhz, double ref_frequency_mhz,
                       double tsamp);
int gfo_multi_dm_output_nsamples(const double* frequency_mhz, uint64_t nchans,
                                 uint64_t nsamples, double dm_low, double dm_step,
                                 uint64_t ndm, double ref_frequency_mhz,
                                 double tsamp, uint64_t chan_begin,
                                 uint64_t chan_end, uint64_t* nout);
/* in: [nsamples][nchans] time-major; out: [ndm][nout] (nout from the call above) */
int gfo_dedisperse_multi_dm_u8(const uint8_t* in, uint64_t nsamples, uint64_t nchans,
                               const double* frequency_mhz, double dm_low,
                               double dm_step, uint64_t ndm, double ref_frequency_mhz,
                               double tsamp, uint64_t chan_begin, uint64_t chan_end,
                               uint32_t* out);
int gfo_dedisperse_subband_u8(const uint8_t* in, uint64_t nsamples, uint64_t nchans,
                              const double* frequency_mhz, double dm_low,
                              double dm_step, uint64_t ndm, double ref_frequency_mhz,
                              double tsamp, uint64_t chan_begin, uint64_t chan_end,
                              uint64_t subband_channels, uint64_t ndm_per_nominal,
                              uint32_t* out);
/* 2-bit input: byte k of a time row holds channels 4k..4k+3, channel 4k+j in
 * bits [2j, 2j+1] (least-significant pair first).  nchans % 4 == 0. */
void gfo_unpack_2bit(const uint8_t* packed, uint64_t nsamples, uint64_t nchans,
                     uint8_t* out);

/* ---- time series (time_series.cpp) ---- */
int gfo_downsampled_size(uint64_t nsamples, double factor, uint64_t* out);
int gfo_downsampled_variance(uint64_t nsamples, double factor, double* out);
int gfo_downsample_weighted_sum(const float* in, uint64_t n, double factor,
                                float* out);
int gfo_normalise(const float* in, uint64_t n, int reject_constant, float* out);

/* ---- preprocessing (preprocessing.cpp) ---- */
int gfo_running_median_window(double window_seconds, double tsamp,
                              uint64_t* window_samples);
int gfo_detrend_running_median(const float* in, uint64_t n,
                               uint64_t window_samples, uint64_t min_points,
                               float* out);
/* make_riptide_preprocess_plan + preprocess_time_series_cpu, in place */
int gfo_preprocess_riptide(float* data, uint64_t n, double tsamp,
                           const gfo_preprocess_options* options);

/* ---- FFA plan / transform / detection / search ---- */
int gfo_make_riptide_ffa_plan(uint64_t nsamples, double tsamp,
                              const gfo_plan_options* options,
                              gfo_ffa_task** tasks, uint64_t* ntasks,
                              uint64_t** widths, uint64_t* nwidths);
int gfo_ffa_transform(const float* in, uint64_t rows, uint64_t bins, float* out);
int gfo_ffa_trial_periods(uint64_t rows, uint64_t bins, double tsamp,
                          double* periods);
float gfo_ffa_task_stdnoise(const gfo_ffa_task* task);
/* find_ffa_peaks_cpu over a materialised rows_eval x bins block */
int gfo_find_ffa_peaks(const float* transform, uint64_t rows, uint64_t bins,
                       const gfo_ffa_task* task, const uint64_t* widths,
                       uint64_t nwidths, float stdnoise, float snr_threshold,
                       uint64_t max_peaks, gfo_peak** peaks, uint64_t* npeaks);
/* search_ffa_cpu (peaks carry dm = 0, dm_index = 0) */
int gfo_ffa_search(const float* series, uint64_t n, const gfo_ffa_task* tasks,
                   uint64_t ntasks, const uint64_t* widths, uint64_t nwidths,
                   float snr_threshold, uint64_t max_peaks, gfo_peak** peaks,
                   uint64_t* npeaks);
/* find_dm_peaks_cpu over a uint32 dedispersed block [ndm][nsamples]; dms has
 * ndm entries; the FFA plan is built from plan_options on nsamples. */
int gfo_find_dm_peaks_u32(const uint32_t* data, uint64_t ndm, uint64_t nsamples,
                          const double* dms, double tsamp,
                          const gfo_plan_options* plan_options,
                          const gfo_preprocess_options* preprocess,
                          float snr_threshold, uint64_t max_peaks,
                          const uint64_t* width_override, uint64_t nwidth_override,
                          gfo_peak** peaks, uint64_t* npeaks);
int gfo_is_better_peak(const gfo_peak* lhs, const gfo_peak* rhs);
void gfo_sort_dm_peaks(gfo_peak* peaks, uint64_t n);

/* ---- candidates (candidate.cpp) ---- */
int gfo_select_candidates(const gfo_peak* peaks, uint64_t npeaks,
                          double observation_seconds,
                          const gfo_candidate_options* options,
                          gfo_candidate** candidates, uint64_t* ncandidates);

/* dedisperse_spectrum_cpu (dedispersion.cpp:249-289) for uint8 samples:
 * out[t][c] = in[t + d(c)][chan_begin + c], t < nout (computed first with
 * out == NULL). */
int gfo_dedisperse_spectrum_u8(const uint8_t* in, uint64_t nsamples, uint64_t nchans,
                               const double* freq, double dm, double ref_freq, double tsamp,
                               uint64_t chan_begin, uint64_t chan_end, uint8_t* out,
                               uint64_t* nout);

/* ---- filterbank header (reference checker only: io/filterbank.cpp) ---- */
typedef struct {
  int64_t header_size;
  int64_t nsamples;
  int32_t telescope_id, machine_id, data_type, barycentric, pulsarcentric;
  int32_t ibeam, nbeams, npuls, nbins, nbits, nifs, nchans;
  double az_start, za_start, src_raj, src_dej, tstart, tsamp, fch1, foff, refdm, period;
  int32_t uses_frequency_table;
  int32_t reversed;
  char rawdatafile[256];
  char source_name[256];
} gfo_filterbank_header; /* filterbank.h:33-65 FilterbankHeader */

/* ---- harmonics (harmonic.cpp) ---- */
typedef struct {
  double observation_seconds;
  double frequency_low_mhz;
  double frequency_high_mhz;
} gfo_harmonic_context; /* harmonic.h:16-20 HarmonicContext */

typedef struct {
  uint64_t max_harmonic;
  uint64_t denominator_max;
  double frequency_tolerance_bins;
  double phase_distance_max;
  double dm_distance_max;
  int32_t use_snr_consistency;
  int32_t reserved;
  double snr_distance_max;
} gfo_harmonic_options; /* harmonic.h:22-36 HarmonicOptions */

typedef struct {
  int32_t is_harmonic;
  int32_t reserved;
  uint64_t parent_index;
  int32_t numerator;
  int32_t denominator;
  double frequency_error_bins;
  double phase_distance;
  double dm_distance;
  double expected_snr;
  double snr_distance;
} gfo_harmonic_relation; /* harmonic.h:38-48 HarmonicRelation */

/* flag_harmonics_cpu (harmonic.cpp:245-292): candidates in harmonic ranking
 * order into sorted_out, their relations into relations_out. */
int gfo_flag_harmonics(const gfo_candidate* candidates, uint64_t n,
                       const gfo_harmonic_context* context,
                       const gfo_harmonic_options* options,
                       gfo_candidate* sorted_out, gfo_harmonic_relation* relations_out);
/* remove_harmonics_cpu (harmonic.cpp:294-309) */
int gfo_remove_harmonics(const gfo_candidate* sorted, const gfo_harmonic_relation* relations,
                         uint64_t n, uint64_t max_candidates, gfo_candidate* out,
                         uint64_t* nout);

/* ---- folding (folding.cpp) ---- */
int gfo_fold_time_series_f32(const float* in, uint64_t n, double period,
                             double tsamp, uint64_t nbin, uint64_t start_sample,
                             float* profile, double* exposure);
int gfo_fold_time_series_u32(const uint32_t* in, uint64_t n, double period,
                             double tsamp, uint64_t nbin, uint64_t start_sample,
                             float* profile, double* exposure);

/* ---- FP64 FFA search of one task (ffa64_oracle.c): the precision reference ---- */
int gfo64_downsample(const float* in, uint64_t n, double factor, double* out, uint64_t* nout);
int gfo64_ffa_transform(const double* in, uint64_t rows, uint64_t bins, double* out);
/* S/N and first best phase for every evaluated row and width, no threshold:
 * snr and phase are [rows_eval][nw]. */
int gfo64_ffa_task_snr(const float* series, uint64_t n, const gfo_ffa_task* task, const uint64_t* widths,
                       uint64_t nw, double* snr, uint64_t* phase);

/* ---- synthetic observations (synth_oracle.c; no reference counterpart) ---- */
typedef struct {
  double period, dm, duty_cycle, amplitude, phase;
} gfo_synth_pulsar;

typedef struct {
  uint64_t nchans, nsamples;
  double tsamp, f_low, f_high;
  int32_t nbits, npulsars;
  uint64_t seed;
  const gfo_synth_pulsar* pulsars;
  const uint8_t* narrowband_mask; /* nchans bytes, or NULL */
  double narrowband_hz, narrowband_amplitude;
  double impulse_hz, impulse_amplitude;
} gfo_synth_desc;

/* Rows [t_begin, t_end) of the gaffa_b200/synth.py observation, time-major:
 * nchans bytes per row (8-bit) or nchans/4 packed bytes (2-bit). */
int gfo_synth_generate(const gfo_synth_desc* d, uint64_t t_begin, uint64_t t_end, uint8_t* out);

#ifdef __cplusplus
}
#endif

#endif /* GAFFA_ORACLE_H */
