/*
 * gaffa_b200.h -- C ABI of the B200 (sm_100a) pulsar-search hot path.
 *
 * The library libgaffa_b200.so implements gaffa's search path -- brute-force
 * and subband dedispersion, running-median detrend + normalise, per-octave
 * downsampling, the FFA transform, boxcar S/N detection, candidate selection
 * and folding -- as hand-written CUDA kernels for sm_100a behind this plain C
 * interface: POD structs, int status codes, caller-owned device buffers and an
 * explicit cudaStream_t (passed as void*).  Nothing here throws, allocates
 * result memory for the caller, or synchronises implicitly unless stated.
 *
 * Each entry point names the reference interface it replaces
 * (lintian233/gaffa, path:line relative to that project).
 *
 * Status: 0 = success; negative values are error classes (GF_E*);
 * gf_last_error() returns the thread's last message.
 */
#ifndef GAFFA_B200_H
#define GAFFA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GF_OK 0
#define GF_EINVAL -1    /* std::invalid_argument */
#define GF_EOVERFLOW -2 /* std::overflow_error */
#define GF_ERUNTIME -3  /* std::runtime_error (guards, max_tasks) */
#define GF_ENOMEM -4    /* device or host allocation failed */
#define GF_ECUDA -5     /* CUDA runtime error (message has the CUDA string) */
#define GF_EDATA -6     /* deferred data error reported by a device status word */
#define GF_EOVERFLOW_PEAKS -7 /* peak buffer too small; count says how many */

/* Device status word bits (written by kernels with atomicOr). */
#define GF_STATUS_NONFINITE 1u
#define GF_STATUS_CONSTANT 2u
#define GF_STATUS_PEAK_OVERFLOW 4u
#define GF_STATUS_SCHEDULE 8u /* an FFA block schedule exceeded its tile (internal error) */
#define GF_STATUS_PIPELINE 16u /* a dedispersion copy stage did not complete within ~2 s (internal error) */

const char* gf_last_error(void);
const char* gf_status_string(int status);
/* Library build description (architecture, kernel list) for diagnostics. */
const char* gf_build_info(void);
/* Replace cuda_device_count / cuda_runtime_version (src/gaffa/vector_add.cu:75-86,
 * bound as gaffa._core.cuda_device_count / cuda_runtime_version): visible
 * devices (0 when there is no device or driver) and the CUDA runtime version
 * of this library (e.g. 12090). */
int gf_cuda_device_count(int32_t* count);
int gf_cuda_runtime_version(int32_t* version);

/* ------------------------------------------------------------------------ */
/* FFA plan (host)                                                           */
/* ------------------------------------------------------------------------ */

/* Same fields and meaning as FfaSearchTask, include/gaffa/ffa_plan.h:8-32. */
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
} gf_ffa_task;

/* RiptideFfaPlanOptions, include/gaffa/ffa_plan.h:34-47. */
typedef struct {
  double period_min;
  double period_max;
  uint64_t bins_min;
  uint64_t bins_max;
  uint64_t min_periods;
  double duty_cycle_max;
  double width_trial_spacing;
  uint64_t max_tasks;
} gf_plan_options;

/* Replaces make_riptide_ffa_plan, src/gaffa/ffa_plan.cpp:90-170.
 * Two-call pattern: pass capacities of 0 to learn ntasks / nwidths. */
int gf_make_riptide_ffa_plan(uint64_t nsamples, double tsamp,
                             const gf_plan_options* options, gf_ffa_task* tasks,
                             uint64_t task_capacity, uint64_t* ntasks,
                             uint64_t* widths, uint64_t width_capacity,
                             uint64_t* nwidths);

/* Replaces downsampled_size / downsampled_variance,
 * src/gaffa/time_series.cpp:118-138, and ffa_task_stdnoise,
 * src/gaffa/ffa_detection.cpp:256-264. */
int gf_downsampled_size(uint64_t nsamples, double factor, uint64_t* out);
int gf_downsampled_variance(uint64_t nsamples, double factor, double* out);
int gf_ffa_task_stdnoise(const gf_ffa_task* task, float* out);

/* ------------------------------------------------------------------------ */
/* Dedispersion                                                              */
/* ------------------------------------------------------------------------ */

#define GF_DEDISP_BRUTE 0
#define GF_DEDISP_SUBBAND 1

/* MultiDmDedispersionPlan (include/gaffa/dedispersion.h:24-32) plus
 * SubbandDedispersionOptions (:34-37), the sample type and the device. */
typedef struct {
  uint64_t nsamples;
  uint64_t nchans;
  const double* frequency_mhz; /* host pointer, nchans entries */
  double dm_low;
  double dm_step;
  uint64_t ndm;
  double ref_frequency_mhz;
  double tsamp;
  uint64_t chan_begin;
  uint64_t chan_end;
  int32_t nbits;      /* 8: uint8 [time][chan]; 2: packed, 4 channels per byte,
                         channel 4k+j in bits [2j, 2j+1] of byte k */
  int32_t algorithm;  /* GF_DEDISP_BRUTE or GF_DEDISP_SUBBAND */
  uint64_t subband_channels; /* subband only */
  uint64_t ndm_per_nominal;  /* subband only */
  int32_t device_id;
  int32_t launch_dms_per_cta; /* brute force launch shape, 0 = automatic: DMs per CTA (1, 2, 4, 8) */
  int32_t launch_chunk_rows;  /* 0 = automatic: channel rows staged per step (8, 16, 32, 64) */
  int32_t reserved;
} gf_dedisp_desc;

typedef struct {
  uint64_t nout;               /* valid output samples per DM */
  int32_t max_delay;           /* delay of the highest DM at the lowest channel */
  int32_t reserved;
  uint64_t input_bytes;        /* bytes of the time-major input */
  uint64_t staged_bytes;       /* bytes of the channel-major staging buffer */
  uint64_t staged_row_stride;  /* bytes between channel rows of the staging buffer */
  uint64_t workspace_bytes;    /* scratch for gf_dedisp_run (subband intermediate) */
  uint64_t metadata_bytes;     /* device tables owned by the program */
} gf_dedisp_info;

typedef struct gf_dedisp_program gf_dedisp_program;

/* Builds the delay tables of internal/dedispersion_delay.h:37-139 (FP64,
 * round half away from zero) and dedispersion.cpp:141-189 on the host, sorts
 * them into the per-warp gather records the kernels use and uploads them.
 * Replaces the delay kernels of src/gaffa/dedispersion_cuda.cu:190-267. */
int gf_dedisp_program_create(const gf_dedisp_desc* desc, gf_dedisp_program** out);
int gf_dedisp_program_destroy(gf_dedisp_program* program);
int gf_dedisp_program_info(const gf_dedisp_program* program, gf_dedisp_info* info);

/* Stage a device-resident time-major input ([nsamples][nchans] uint8, or the
 * packed 2-bit rows) into the channel-major uint8 layout the kernels read
 * (staged_bytes).  Counterpart of the H2D + layout step inside
 * dedisperse_*_cuda_device, dedispersion_cuda.cu:587-714. */
int gf_dedisp_stage(gf_dedisp_program* program, const void* dev_input,
                    void* dev_staged, void* stream);
/* Stage a host time-major input in chunks through pinned host memory. */
int gf_dedisp_stage_from_host(gf_dedisp_program* program, const void* host_input,
                              void* dev_staged, void* dev_bounce,
                              uint64_t bounce_bytes, void* stream);

/* Dedisperse DMs [dm_begin, dm_begin + dm_count) into dev_out
 * ([dm_count][out_stride] uint32, out_stride >= nout).  Bit-exact with
 * dedisperse_multi_dm_cpu (dedispersion.cpp:291-329) or
 * dedisperse_subband_cpu (:331-453).  Replaces multi_dm_kernel and
 * subband_stage1/2_kernel, dedispersion_cuda.cu:320-417.  Subband runs need
 * dm_begin / dm_count aligned to ndm_per_nominal (except at the end).
 * dev_staged and dev_workspace must be 16-byte aligned (the kernels copy
 * their rows with bulk copies); cudaMalloc'd buffers are. */
int gf_dedisp_run(gf_dedisp_program* program, const void* dev_staged,
                  uint64_t dm_begin, uint64_t dm_count, uint32_t* dev_out,
                  uint64_t out_stride, void* dev_workspace, void* stream);
/* Batched brute-force dedispersion: many (program, DM range) items, of
 * different observations, channel counts and lengths, in one launch.  The
 * reference launches multi_dm_kernel once per plan (dedispersion_cuda.cu:
 * 536-585); each item's output is identical to gf_dedisp_run of the same
 * range.  Pointers are fixed at creation, so gf_dedisp_batch_run can be
 * captured in a CUDA graph. */
typedef struct gf_dedisp_batch gf_dedisp_batch;
typedef struct {
  const gf_dedisp_program* program;   /* brute force */
  const void* dev_staged;             /* the program's staged filterbank */
  uint64_t dm_begin;                  /* multiple of 8 */
  uint64_t dm_count;
  uint32_t* dev_out;                  /* [dm_count][out_stride] */
  uint64_t out_stride;
} gf_dedisp_batch_item;
int gf_dedisp_batch_create(const gf_dedisp_batch_item* items, uint64_t nitems,
                           gf_dedisp_batch** out);
int gf_dedisp_batch_run(gf_dedisp_batch* batch, void* stream);
int gf_dedisp_batch_destroy(gf_dedisp_batch* batch);

/* Synchronises `stream` and reads (and clears) the program's device status
 * word: GF_ERUNTIME when a launch of gf_dedisp_run or gf_dedisp_batch_run gave
 * up waiting for one of its shared-memory copy stages (every wait is bounded;
 * such a launch writes no output).  Call after a group of runs, before their
 * output is used.  No reference counterpart: the reference's kernels have no
 * waits (dedispersion_cuda.cu:320-417). */
int gf_dedisp_check(gf_dedisp_program* program, void* stream);

/* Workspace bytes gf_dedisp_run needs for a batch of dm_count DMs (0 for
 * brute force; the subband intermediate otherwise).  Brute-force batches start
 * at multiples of 8 DMs, subband batches at multiples of ndm_per_nominal. */
int gf_dedisp_workspace_bytes(const gf_dedisp_program* program, uint64_t dm_count,
                              uint64_t* bytes);

/* Aligned single-DM spectrum.  Replaces dedisperse_spectrum_cpu /
 * dedisperse_spectrum_cuda (dedispersion.cpp:249-289,
 * dedispersion_cuda.cu:295-318): channels [chan_begin, chan_end) of a
 * time-major [nsamples][nchans] filterbank (elem_bytes 1 = uint8, 2 = uint16,
 * 4 = float), each shifted by its delay at dm:
 *   out[t][c] = in[t + d(c)][chan_begin + c],  t < nout,
 * nout = nsamples - d(dm, lowest selected frequency).  Writes *nout; with
 * dev_out == NULL only *nout is computed.  Runs on the current device. */
int gf_dedisperse_spectrum(const void* dev_in, int32_t elem_bytes, uint64_t nsamples,
                           uint64_t nchans, const double* frequency_mhz, double dm,
                           double ref_frequency_mhz, double tsamp, uint64_t chan_begin,
                           uint64_t chan_end, void* dev_out, uint64_t* nout, void* stream);

/* ------------------------------------------------------------------------ */
/* Filterbank ingest (SIGPROC)                                               */
/* ------------------------------------------------------------------------ */

#define GF_CHANNEL_ORDER_ASCENDING 0 /* ChannelOrderPolicy::FrequencyAscending */
#define GF_CHANNEL_ORDER_FILE 1      /* ChannelOrderPolicy::PreserveFileOrder */

/* FilterbankHeader, include/gaffa/filterbank.h:33-65, after
 * read_filterbank's metadata normalisation (src/gaffa/io/filterbank.cpp:105-118). */
typedef struct {
  int64_t header_size;
  int64_t nsamples;
  int32_t telescope_id, machine_id, data_type, barycentric, pulsarcentric;
  int32_t ibeam, nbeams, npuls, nbins, nbits, nifs, nchans;
  double az_start, za_start, src_raj, src_dej, tstart, tsamp, fch1, foff, refdm, period;
  int32_t uses_frequency_table;
  int32_t reversed; /* 1 when samples are delivered channel-reversed */
  char rawdatafile[256];
  char source_name[256];
} gf_filterbank_header;

/* The header part of read_filterbank (src/gaffa/io/filterbank.cpp:116-224,
 * 335-348): fields, and the frequency of each delivered channel (up to
 * capacity values; frequency_table may be NULL).  nbits 8, 16, 32 as the
 * reference; packed 1-, 2- and 4-bit rows are accepted in addition. */
int gf_filterbank_read_header(const char* path, int32_t channel_order,
                              gf_filterbank_header* header, double* frequency_table,
                              uint64_t capacity);
/* Rows [row_begin, row_begin + nrows) into host memory, channel order as
 * read_filterbank delivers it (src/gaffa/io/filterbank.cpp:243-333). */
int gf_filterbank_read_host(const char* path, int32_t channel_order, uint64_t row_begin,
                            uint64_t nrows, void* host_out);
/* The same rows straight into device memory: the file is read into the two
 * halves of a caller-owned pinned host buffer in turn, each half copied to the
 * device while the other fills, and the channel reversal runs on the GPU.
 * Returns once the last copy is issued; work is ordered on stream. */
int gf_filterbank_load(const char* path, int32_t channel_order, uint64_t row_begin,
                       uint64_t nrows, void* dev_out, void* host_bounce, uint64_t bounce_bytes,
                       void* stream);

/* ------------------------------------------------------------------------ */
/* Preprocessing: running-median detrend + normalise                         */
/* ------------------------------------------------------------------------ */

/* RiptidePreprocessOptions (include/gaffa/preprocessing.h:37-42) evaluated
 * for one tsamp, as make_riptide_preprocess_plan (preprocessing.cpp:190-210). */
typedef struct {
  double tsamp;
  double window_seconds;
  uint64_t min_points;
  int32_t normalise;
  int32_t reject_constant;
  uint64_t nsamples;   /* series length */
  uint64_t max_series; /* workspace is sized for this many series */
} gf_preprocess_desc;

typedef struct {
  uint64_t window_samples;
  uint64_t scrunch_factor;  /* 1 = exact running median */
  uint64_t low_nsamples;    /* scrunched length */
  uint64_t workspace_bytes;
} gf_preprocess_info;

int gf_preprocess_info_get(const gf_preprocess_desc* desc, gf_preprocess_info* info);

/* In place on [nseries][stride] 32-bit series (input_is_u32 = 1: uint32 sums
 * from gf_dedisp_run, converted exactly to float as dm_search.cpp:53-68; 0:
 * float).  On return the buffer holds float detrended values
 * (preprocessing.cpp:212-231) and dev_stats[2*s] / [2*s+1] hold the FP64 mean
 * and 1/stddev of time_series_stats_cpu (time_series.cpp:50-78); the
 * normalisation itself is applied by gf_normalise or fused into
 * gf_ffa_prepare.  Data errors set bits in *dev_status (deferred, as
 * preprocessing_cuda.cu:269-272,781-817).  Replaces
 * preprocess_time_series_batch_inplace_cuda, preprocessing_cuda.cu:819-864. */
int gf_preprocess_inplace(const gf_preprocess_desc* desc, void* dev_series,
                          int32_t input_is_u32, uint64_t nseries, uint64_t stride,
                          void* dev_workspace, double* dev_stats,
                          uint32_t* dev_status, void* stream);
/* Many gf_preprocess_inplace calls (series sets of different lengths,
 * windows and options) as one launch per stage: the per-set launches of
 * preprocess_time_series_batch_inplace_cuda (preprocessing_cuda.cu:819-864),
 * one per observation in the reference, fill the GPU together.  Each item's
 * results equal gf_preprocess_inplace with the same arguments.  Pointers are
 * fixed at creation, so gf_preprocess_batch_run can be captured in a CUDA
 * graph. */
typedef struct gf_preprocess_batch gf_preprocess_batch;
typedef struct {
  const gf_preprocess_desc* desc;   /* read at creation */
  void* dev_series;
  int32_t input_is_u32;
  int32_t reserved;
  uint64_t nseries;
  uint64_t stride;
  void* dev_workspace;
  double* dev_stats;
  uint32_t* dev_status;
} gf_preprocess_batch_item;
int gf_preprocess_batch_create(const gf_preprocess_batch_item* items, uint64_t nitems,
                               int32_t device_id, gf_preprocess_batch** out);
int gf_preprocess_batch_run(gf_preprocess_batch* batch, void* stream);
int gf_preprocess_batch_destroy(gf_preprocess_batch* batch);

/* x <- float((x - mean) * (1/stddev)) (time_series.cpp:98-103); zeroes
 * constant series when reject_constant == 0. */
int gf_normalise(float* dev_series, uint64_t nseries, uint64_t stride,
                 uint64_t nsamples, const double* dev_stats, void* stream);

/* ------------------------------------------------------------------------ */
/* FFA search                                                                */
/* ------------------------------------------------------------------------ */

typedef struct gf_ffa_program gf_ffa_program;

typedef struct {
  uint64_t ntasks;
  uint64_t noctaves;            /* distinct downsample factors (prepare groups) */
  uint64_t prepared_floats;     /* per series, all octaves */
  uint64_t scratch_bytes;       /* per gf_ffa_search call */
  uint64_t max_task_elements;   /* rows * bins of the largest task */
  uint64_t metadata_bytes;
  uint64_t nclasses;            /* kernel launches per gf_ffa_search */
} gf_ffa_info;

/* Compact device peak record (24 bytes); FfaCudaPeak of
 * src/gaffa/ffa_cuda_kernels.cuh:70-99 in spirit. */
typedef struct {
  uint32_t series;
  uint32_t task;
  uint32_t shift;
  uint16_t phase;
  uint16_t width_index;
  float snr;
  uint32_t reserved;
} gf_peak_record;

/* Host peak: DmPeak{dm, dm_index, FfaPeak} (dm_search.h:16-20,
 * ffa_peak.h:8-19); same layout as the oracle's gfo_peak. */
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
} gf_peak;

/* Replaces CudaFfaProgram + make_ffa_cuda_execution_plan,
 * src/gaffa/ffa_cuda_executor.cuh:44-80,144-210.  Uploads the task tables,
 * the boxcar trials (ffa_detection.cpp:60-80) and the per-octave prepare
 * tables; the program owns only metadata. */
int gf_ffa_program_create(const gf_ffa_task* tasks, uint64_t ntasks,
                          const uint64_t* widths, uint64_t nwidths,
                          uint64_t max_series, int32_t device_id,
                          gf_ffa_program** out);
int gf_ffa_program_destroy(gf_ffa_program* program);
int gf_ffa_program_info(const gf_ffa_program* program, gf_ffa_info* info);

/* Per-octave weighted-sum downsampling of every series
 * (downsample_weighted_sum_cpu, time_series.cpp:140-174, with the
 * ffa_executor.cpp:99-115 cache) into dev_prepared
 * ([nseries][prepared_floats]).  When dev_stats is given the normalisation
 * float((x - mean) * scale) is applied on the fly to each input sample.
 * Replaces prepare_ffa_input_cuda, ffa_cuda_executor.cuh:277-305, and
 * downsample_weighted_sum_float_kernel, time_series_cuda.cu:15-48. */
int gf_ffa_prepare(gf_ffa_program* program, const float* dev_series,
                   uint64_t nseries, uint64_t stride, const double* dev_stats,
                   float* dev_prepared, void* stream);

/* FFA transform of every task of every series followed by boxcar S/N
 * detection on the rows_eval final rows (ffa.cpp:127-251,
 * ffa_detection.cpp:126-372); peaks with S/N >= snr_threshold are appended
 * to dev_peaks.  dev_counters[0] receives the number of peaks found (which
 * may exceed capacity: then GF_STATUS_PEAK_OVERFLOW is set in
 * dev_counters[1] and the caller re-runs with a larger buffer).  Replaces
 * run_ffa_batch_cuda, ffa_cuda_executor.cuh:368-678, and the transform /
 * detection kernels of ffa_cuda_kernels.cuh:130-737.  dev_scratch must hold
 * scratch_bytes. */
int gf_ffa_search(gf_ffa_program* program, const float* dev_prepared,
                  uint64_t nseries, float snr_threshold, void* dev_scratch,
                  gf_peak_record* dev_peaks, uint64_t capacity,
                  uint64_t* dev_counters, void* stream);

/* Expands compact records into host peaks (make_ffa_peak,
 * ffa_detection.cpp:266-284); dm = dm_low + (series + series_offset) *
 * dm_step as cuda_dm_search_benchmark.cpp:255-258. */
int gf_ffa_expand_peaks(const gf_ffa_program* program,
                        const gf_peak_record* records, uint64_t n,
                        uint64_t series_offset, double dm_low, double dm_step,
                        gf_peak* out);

/* Batched FFA search: the plans of many observations (members) in one
 * program, so each launch class covers every member's (series, task) items
 * in one persistent launch.  The reference runs one CudaFfaProgram per
 * observation (ffa_cuda_executor.cuh:44-80, run_ffa_batch_cuda :672-678);
 * results are identical to searching each member with its own program.
 * Records name the global task (task_begin of its member + local index) and
 * the series within the member. */
typedef struct {
  const gf_ffa_task* tasks;
  uint64_t ntasks;
  const uint64_t* widths;
  uint64_t nwidths;
  uint64_t nseries;             /* series searched per gf_ffa_batch_search */
} gf_ffa_batch_member;

typedef struct {
  uint64_t nsamples;
  uint64_t nseries;
  uint64_t prepared_floats;     /* per series, all octaves */
  uint64_t task_begin;          /* first global task index of the member */
  uint64_t ntasks;
  uint64_t noctaves;
} gf_ffa_member_info;

int gf_ffa_batch_create(const gf_ffa_batch_member* members, uint64_t nmembers,
                        int32_t device_id, gf_ffa_program** out);
int gf_ffa_batch_member_info(const gf_ffa_program* program, uint64_t member,
                             gf_ffa_member_info* info);
/* dev_prepared: host array of nmembers device pointers, each
 * [nseries][prepared_floats] floats, 16-byte aligned.  Synchronous upload;
 * call before capturing launches into a CUDA graph. */
int gf_ffa_batch_bind(gf_ffa_program* program, const float* const* dev_prepared);
/* prepare_ffa_input_cuda of one member's nseries series into its bound buffer. */
int gf_ffa_batch_prepare(gf_ffa_program* program, uint64_t member,
                         const float* dev_series, uint64_t stride,
                         const double* dev_stats, void* stream);
/* The series gf_ffa_batch_prepare_all reads, for every member m:
 * dev_series[m] ([nseries][strides[m]] floats) and dev_stats[m] (the
 * member's gf_preprocess_inplace statistics; dev_stats or an entry may be
 * null: no normalisation).  Synchronous upload; call before capturing. */
int gf_ffa_batch_bind_series(gf_ffa_program* program, const float* const* dev_series,
                             const uint64_t* strides, const double* const* dev_stats);
/* gf_ffa_batch_prepare of every member in one launch. */
int gf_ffa_batch_prepare_all(gf_ffa_program* program, void* stream);
/* One launch per class over every member; no host synchronisation. */
int gf_ffa_batch_search(gf_ffa_program* program, float snr_threshold,
                        void* dev_scratch, gf_peak_record* dev_peaks,
                        uint64_t capacity, uint64_t* dev_counters, void* stream);
/* gf_ffa_expand_peaks with per-member series offsets and DM grids; member[i]
 * receives the record's member. */
int gf_ffa_batch_expand_peaks(const gf_ffa_program* program,
                              const gf_peak_record* records, uint64_t n,
                              const uint64_t* series_offset, const double* dm_low,
                              const double* dm_step, gf_peak* out, uint32_t* member);

/* One materialised FFA transform of [rows][bins] floats (ffa_transform_cpu /
 * ffa_transform_block_cuda, ffa.cpp:342-417, ffa_cuda.h:254-264).
 * dev_scratch needs rows * bins * 8 bytes. */
int gf_ffa_transform(const float* dev_input, uint64_t rows, uint64_t bins,
                     float* dev_output, void* dev_scratch, void* stream);

/* ------------------------------------------------------------------------ */
/* Host post-processing                                                      */
/* ------------------------------------------------------------------------ */

/* Sort by is_better_dm_peak (dm_search.cpp:89-100 over ffa_peak.cpp:16-45). */
int gf_sort_peaks(gf_peak* peaks, uint64_t n);

/* CandidateSelectionOptions, include/gaffa/candidate.h:30-39. */
typedef struct {
  double frequency_cluster_radius;
  uint64_t dm_cluster_radius;
  int32_t cluster_across_widths;
  int32_t reserved;
  uint64_t max_candidates;
} gf_candidate_options;

/* Candidate, include/gaffa/candidate.h:11-28 (same layout as gfo_candidate). */
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
  gf_peak best_peak;
} gf_candidate;

/* Replaces select_candidates_cpu, src/gaffa/candidate.cpp:175-212.
 * Two-call pattern on capacity. */
int gf_select_candidates(const gf_peak* peaks, uint64_t npeaks,
                         double observation_seconds,
                         const gf_candidate_options* options,
                         gf_candidate* out, uint64_t capacity,
                         uint64_t* ncandidates);

/* A run of compact device peak records from one gf_ffa_search call:
 * records [record_begin, record_begin + record_count) of the record array,
 * whose series s is DM trial series_offset + s. */
typedef struct {
  uint64_t record_begin;
  uint64_t record_count;
  uint64_t series_offset;
} gf_peak_segment;

/* select_candidates_cpu (src/gaffa/candidate.cpp:175-212) over compact
 * device records, for peak sets too large to expand and sort on the host:
 * the records are expanded on the device (make_ffa_peak,
 * ffa_detection.cpp:266-284; dm = dm_low + index * dm_step), ordered by
 * stable device radix sorts into the reference's peak and group orders,
 * split and reduced per cluster on the device; the candidates (best peak,
 * count, DM and frequency extent) are ranked on the host
 * (is_better_candidate, candidate.cpp:48-62) and written to out (two-call
 * pattern on capacity; synchronises the stream).  The result equals
 * gf_select_candidates on the expanded records.  program is the
 * single-plan FFA program that produced the records; dev_workspace needs
 * gf_select_candidates_device_workspace(total records) bytes. */
int gf_select_candidates_device_workspace(uint64_t npeaks, uint64_t* bytes);
int gf_select_candidates_device(const gf_ffa_program* program,
                                const gf_peak_record* dev_records,
                                const gf_peak_segment* segments, uint64_t nsegments,
                                double dm_low, double dm_step,
                                double observation_seconds,
                                const gf_candidate_options* options,
                                void* dev_workspace, uint64_t workspace_bytes,
                                gf_candidate* out, uint64_t capacity,
                                uint64_t* ncandidates, void* stream);

/* HarmonicContext, include/gaffa/harmonic.h:16-20. */
typedef struct {
  double observation_seconds;
  double frequency_low_mhz;
  double frequency_high_mhz;
} gf_harmonic_context;

/* HarmonicOptions, include/gaffa/harmonic.h:22-36 (defaults: 16, 5, 1.5,
 * 1.0, 3.0, 0, 3.0). */
typedef struct {
  uint64_t max_harmonic;
  uint64_t denominator_max;
  double frequency_tolerance_bins;
  double phase_distance_max;
  double dm_distance_max;
  int32_t use_snr_consistency;
  int32_t reserved;
  double snr_distance_max;
} gf_harmonic_options;

#define GF_NO_HARMONIC_PARENT UINT64_MAX

/* HarmonicRelation, include/gaffa/harmonic.h:38-48. */
typedef struct {
  int32_t is_harmonic;
  int32_t reserved;
  uint64_t parent_index; /* GF_NO_HARMONIC_PARENT when not a harmonic */
  int32_t numerator;
  int32_t denominator;
  double frequency_error_bins;
  double phase_distance;
  double dm_distance;
  double expected_snr;
  double snr_distance;
} gf_harmonic_relation;

/* Replaces flag_harmonics_cpu, src/gaffa/harmonic.cpp:245-292.  Writes the n
 * candidates in harmonic ranking order (S/N desc, peak_count desc, frequency
 * asc, dm_index asc) to sorted_out and their relations to relations_out
 * (parent_index refers to that order).  options may be NULL (defaults). */
int gf_flag_harmonics(const gf_candidate* candidates, uint64_t n,
                      const gf_harmonic_context* context,
                      const gf_harmonic_options* options,
                      gf_candidate* sorted_out,
                      gf_harmonic_relation* relations_out);
/* The same flagging with the pairwise tests on a device: for lists of 10^4+
 * candidates (the n^2 / 2 tests of harmonic.cpp:271-289 take minutes on a
 * CPU at 10^5).  The decisions use the same FP64 expressions with explicit
 * rounding, so outputs equal gf_flag_harmonics; host in, host out,
 * synchronous on `stream`. */
int gf_flag_harmonics_device(const gf_candidate* candidates, uint64_t n,
                             const gf_harmonic_context* context,
                             const gf_harmonic_options* options,
                             gf_candidate* sorted_out,
                             gf_harmonic_relation* relations_out,
                             int32_t device_id, void* stream);

/* Replaces remove_harmonics_cpu, src/gaffa/harmonic.cpp:294-309: the
 * non-harmonic candidates in order, at most max_candidates (0 = all). */
int gf_remove_harmonics(const gf_candidate* sorted, const gf_harmonic_relation* relations,
                        uint64_t n, uint64_t max_candidates, gf_candidate* out,
                        uint64_t* nout);

/* Spectrum folding.  Replaces fold_spectrum_cpu (src/gaffa/folding.cpp:
 * 300-420): a device time-major spectrum [nsamples][nchans] (elem_bytes 1, 2
 * or 4: uint8, uint16, float) folded at `period` into
 * cube[nsubint][nout][nbin] (float, sums / exposure) and
 * exposure[nsubint][nbin] (double), nsubint = ceil(nsamples / subint_samples),
 * nout = output_channels (0: nchans; adjacent input channels are averaged).
 * nbin <= 256.  dev_status receives GF_STATUS_NONFINITE for non-finite float
 * input.  FP64 sums in a different order from the reference: the cube agrees
 * to FP64 rounding. */
int gf_fold_spectrum(const void* dev_in, int32_t elem_bytes, uint64_t nsamples, uint64_t nchans,
                     double period, double tsamp, uint64_t nbin, uint64_t subint_samples,
                     uint64_t start_sample, uint64_t output_channels, float* dev_cube,
                     double* dev_exposure, uint32_t* dev_status, void* stream);
/* Replaces project_folded_cube (src/gaffa/folding.cpp:237-296): profile
 * [nbin], freq_phase [nchans][nbin] and time_phase [nsubint][nbin] of a
 * folded cube, in the reference's summation order. */
int gf_project_folded_cube(const float* dev_cube, const double* dev_exposure, uint64_t nsubint,
                           uint64_t nchans, uint64_t nbin, float* dev_profile, float* dev_freq_phase,
                           float* dev_time_phase, void* stream);

/* ------------------------------------------------------------------------ */
/* Learned DM/period proposal (no counterpart in the reference)              */
/* ------------------------------------------------------------------------ */
/* A small 1-D convolutional network that scores coarse DM trials per period
 * octave, so full-resolution search can run on the best-scoring DM windows
 * only; the exhaustive search stays the fallback.  Tensors are [batch]
 * [channels][length], activations and weights bf16 (uint16 storage),
 * accumulation and gradients fp32. */

/* y = act(bias + conv(x, w)), w [cout][cin][ksize], zero padding ksize/2,
 * relu 0/1.  cin <= 64, ksize odd <= 9. */
int gf_prop_conv_forward(const void* x, const void* w, const float* bias, void* y, int32_t batch,
                         int32_t cin, int32_t cout, int32_t length, int32_t ksize, int32_t relu,
                         void* stream);
/* Backward of a ReLU conv layer: dy (fp32, overwritten by dy * (y_act > 0)
 * when y_act != NULL) -> dw, db accumulated (+=), dx written when non-NULL. */
int gf_prop_conv_backward(const float* dy, const void* y_act, const void* x, const void* w, float* dx,
                          float* dw, float* db, int32_t batch, int32_t cin, int32_t cout, int32_t length,
                          int32_t ksize, void* stream);
/* Head (1x1 conv channels -> 1), per-octave log-mean-exp pooling over
 * length/octaves bins (<= 64), and with labels the positive-weighted binary
 * cross-entropy (added to *loss) and its gradients (dy written, dwh, dbh
 * accumulated). */
int gf_prop_head(const void* y, const float* wh, const float* bh, int32_t batch, int32_t channels,
                 int32_t length, int32_t octaves, const float* labels, float pos_weight,
                 float* logits, float* loss, float* dy, float* dwh, float* dbh, void* stream);
/* One Adam step on fp32 master weights (grad scaled by grad_scale); refreshes
 * the bf16 copy when param_bf16 != NULL. */
int gf_prop_adam(float* param, const float* grad, float* m, float* v, void* param_bf16, uint64_t n,
                 float lr, float beta1, float beta2, float eps, int32_t step, float grad_scale,
                 void* stream);
/* Harmonic-summed spectral features: power [nseries][nfreq] (white noise
 * mean 1 per bin, bin k at k*df Hz) -> feat bf16 [nseries][nbins] over the
 * log frequency bin edges[0..nbins]. */
int gf_prop_features(const float* power, uint64_t nseries, uint64_t nfreq, double df,
                     const float* edges, int32_t nbins, void* feat, void* stream);
/* out[r][t] = sum of `factor` consecutive uint32 samples of in[r] (float). */
int gf_prop_downsample(const uint32_t* in, uint64_t in_stride, uint64_t nrows, int32_t factor,
                       uint64_t nout, float* out, uint64_t out_stride, void* stream);

/* ------------------------------------------------------------------------ */
/* Folding                                                                   */
/* ------------------------------------------------------------------------ */

/* Replaces fold_time_series_cpu (src/gaffa/folding.cpp:452-502), which has no
 * CUDA path in the reference: FP64 fractional phase-overlap accumulation into
 * nbin bins; profile = sums / exposure.  Device input, device outputs
 * (dev_profile: nbin floats, dev_exposure: nbin doubles).  dev_workspace
 * needs gf_fold_workspace_bytes(n, nbin); the uint32 at byte offset
 * gf_fold_workspace_bytes(n, nbin) - 16 receives GF_STATUS_NONFINITE when a
 * float input sample is not finite (the reference rejects such input). */
uint64_t gf_fold_workspace_bytes(uint64_t n, uint64_t nbin);
int gf_fold_time_series(const void* dev_input, int32_t input_is_u32, uint64_t n,
                        double period, double tsamp, uint64_t nbin,
                        uint64_t start_sample, float* dev_profile,
                        double* dev_exposure, void* dev_workspace, void* stream);

/* Fold without allocating device memory.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc at fold time -- a process whose
 * device memory is all owned by another allocator's pool, or a
 * latency-critical loop that cannot afford cudaMalloc's implicit device
 * synchronisation.  Same arithmetic as gf_fold_time_series, but the per-block
 * partial sums live in a fixed scratch array compiled into the library (held
 * by every GPU that loads it until exit), so the work is capped:
 * ceil(n / 16384) * 2 * nbin doubles must fit in gf_fold_noalloc_max_bytes()
 * bytes (4 MiB; e.g. nbin = 64 allows about 67 million samples); larger
 * requests fail with GF_EINVAL.  dev_status (caller-owned, uint32) receives
 * GF_STATUS_NONFINITE for non-finite float input.  The first call on a
 * device resolves the array's device address for that device (call it once
 * before any stream capture).  That address is kept for the life of the
 * process: after a cudaDeviceReset the library's module is reloaded and the
 * kept address is stale, so do not use this entry point after a reset.  All
 * calls share the array: calls that overlap on the GPU race on it and must be
 * serialised by the caller. */
uint64_t gf_fold_noalloc_max_bytes(void);
int gf_fold_time_series_noalloc(const void* dev_input, int32_t input_is_u32,
                                uint64_t n, double period, double tsamp,
                                uint64_t nbin, uint64_t start_sample,
                                float* dev_profile, double* dev_exposure,
                                uint32_t* dev_status, void* stream);

/* ------------------------------------------------------------------------ */
/* Synthetic observations (no reference counterpart)                         */
/* ------------------------------------------------------------------------ */

typedef struct {
  double period, dm, duty_cycle, amplitude, phase;
} gf_synth_pulsar;

typedef struct {
  uint64_t nchans;
  uint64_t nsamples;
  double tsamp;
  double f_low;
  double f_high;
  int32_t nbits;  /* 8 or 2 (2: packed output, nchans % 4 == 0) */
  int32_t npulsars;
  uint64_t seed;
  const gf_synth_pulsar* pulsars; /* host pointer */
  double narrowband_fraction, narrowband_hz, narrowband_amplitude;
  double impulse_hz, impulse_amplitude;
  const uint8_t* narrowband_mask; /* host pointer, nchans entries or NULL */
} gf_synth_desc;

/* Generates time rows [t_begin, t_end) of the seeded observation defined in
 * gaffa_b200/synth.py (same noise stream, bit for bit) into dev_out
 * ([t_end - t_begin][row bytes]). */
int gf_synth_generate(const gf_synth_desc* desc, uint64_t t_begin, uint64_t t_end,
                      uint8_t* dev_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GAFFA_B200_H */
