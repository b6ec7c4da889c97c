// gaffa's C++ CUDA API (include/gaffa/*.h) over the C ABI of gaffa_b200.h.
//
// Every function here is defined by its qualified name, so this file only
// compiles against headers that declare exactly these signatures: the ones
// under include/gaffa/ and, as tests/test_cxx_api.py checks, the reference's
// own include/gaffa/dedispersion_cuda.h, ffa_cuda.h and ffa_plan.h.
//
// Error behaviour follows the reference: invalid input throws
// std::invalid_argument (or std::overflow_error), CUDA failures throw
// std::runtime_error("<operation>: <message>") (dedispersion_cuda.cu:53-58).
// Device buffers are RAII CudaDeviceBuffer objects, freed on their own device
// (cuda_memory.cu:50-80).  Work runs on the legacy default stream (or the
// program's stream for the FFA) and every host-visible result is complete
// when a function returns.
#include "gaffa/dedispersion_cuda.h"
#include "gaffa/ffa_cuda.h"
#include "gaffa/ffa_peak.h"
#include "gaffa/ffa_plan.h"
#include "gaffa_b200.h"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

[[noreturn]] void throw_status(int status, const char* operation) {
  const std::string message = gf_last_error();
  switch (status) {
    case GF_EINVAL:
      throw std::invalid_argument(message);
    case GF_EOVERFLOW:
      throw std::overflow_error(message);
    default:
      throw std::runtime_error(std::string(operation) + ": " + message);
  }
}

void check(int status, const char* operation) {
  if (status != GF_OK) throw_status(status, operation);
}

void check_cuda(cudaError_t status, const char* operation) {
  if (status != cudaSuccess) throw std::runtime_error(std::string(operation) + ": " + cudaGetErrorString(status));
}

// Makes `device` current for the scope and restores the caller's device.
class DeviceScope {
 public:
  explicit DeviceScope(int device) {
    if (device < 0) throw std::invalid_argument("CUDA device_id must be non-negative");
    check_cuda(cudaGetDevice(&previous_), "cudaGetDevice");
    if (previous_ != device) {
      check_cuda(cudaSetDevice(device), "cudaSetDevice");
      restore_ = true;
    }
  }
  ~DeviceScope() {
    if (restore_) static_cast<void>(cudaSetDevice(previous_));
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;

 private:
  int previous_ = 0;
  bool restore_ = false;
};

template <typename T>
void validate_samples(gaffa::HostSampleView<T> samples, std::span<const double> frequency_mhz) {
  if (samples.shape.nsamples == 0) throw std::invalid_argument("dedispersion requires at least one sample");
  if (samples.shape.nifs != 1) throw std::invalid_argument("dedispersion requires nifs == 1");
  if (samples.shape.nchans == 0) throw std::invalid_argument("dedispersion requires at least one channel");
  if (samples.data.size() != gaffa::sample_element_count(samples.shape))
    throw std::invalid_argument("sample view data size does not match shape");
  if (frequency_mhz.size() != samples.shape.nchans)
    throw std::invalid_argument("frequency table length must match nchans");
}

[[noreturn]] void unsupported_sample_type() {
  throw std::invalid_argument(
      "gaffa_b200 dedisperses uint8 samples; uint16 and float samples are taken by "
      "dedisperse_spectrum_cuda only");
}

struct DedispProgram {
  gf_dedisp_program* handle = nullptr;
  ~DedispProgram() {
    if (handle) gf_dedisp_program_destroy(handle);
  }
};

// Direct-sum (GF_DEDISP_BRUTE) or subband dedispersion of uint8 samples into a
// dense [ndm][nout] device result.
gaffa::CudaDedispersedResult<std::uint32_t> dedisperse_u8(gaffa::HostSampleView<std::uint8_t> samples,
                                                          std::span<const double> frequency_mhz, double dm_low,
                                                          double dm_step, std::size_t ndm, double ref_frequency_mhz,
                                                          double tsamp, std::size_t chan_begin, std::size_t chan_end,
                                                          int algorithm, std::size_t subband_channels,
                                                          std::size_t ndm_per_nominal, int device) {
  validate_samples(samples, frequency_mhz);
  if (ndm == 0) throw std::invalid_argument("dedispersion requires at least one DM trial");
  DeviceScope scope(device);
  gf_dedisp_desc d{};
  d.nsamples = samples.shape.nsamples;
  d.nchans = samples.shape.nchans;
  d.frequency_mhz = frequency_mhz.data();
  d.dm_low = dm_low;
  d.dm_step = ndm == 1 && dm_step == 0.0 ? 1.0 : dm_step;  // one trial has no spacing
  d.ndm = ndm;
  d.ref_frequency_mhz = ref_frequency_mhz;
  d.tsamp = tsamp;
  d.chan_begin = chan_begin;
  d.chan_end = chan_end;
  d.nbits = 8;
  d.algorithm = algorithm;
  d.subband_channels = subband_channels;
  d.ndm_per_nominal = ndm_per_nominal;
  d.device_id = device;
  DedispProgram program;
  check(gf_dedisp_program_create(&d, &program.handle), "dedisperse_cuda");
  gf_dedisp_info info{};
  check(gf_dedisp_program_info(program.handle, &info), "dedisperse_cuda");
  gaffa::CudaDeviceBuffer<std::uint8_t> input(info.input_bytes);
  check_cuda(cudaMemcpy(input.data(), samples.data_ptr(), info.input_bytes, cudaMemcpyHostToDevice),
             "cudaMemcpy host-to-device dedispersion input");
  gaffa::CudaDeviceBuffer<std::uint8_t> staged(info.staged_bytes);
  check(gf_dedisp_stage(program.handle, input.data(), staged.data(), nullptr), "dedisperse_cuda");
  gaffa::CudaDedispersedResult<std::uint32_t> result;
  result.shape = gaffa::DedispersedShape{ndm, info.nout};
  result.data = gaffa::CudaDeviceBuffer<std::uint32_t>(gaffa::dedispersed_element_count(result.shape));
  result.device_id = device;
  gaffa::CudaDeviceBuffer<std::uint8_t> workspace;
  if (algorithm == GF_DEDISP_SUBBAND) {
    uint64_t bytes = 0;
    check(gf_dedisp_workspace_bytes(program.handle, ndm, &bytes), "dedisperse_subband_cuda");
    workspace = gaffa::CudaDeviceBuffer<std::uint8_t>(bytes);
  }
  check(gf_dedisp_run(program.handle, staged.data(), 0, ndm, result.data.data(), info.nout, workspace.data(),
                      nullptr),
        "dedisperse_cuda");
  check(gf_dedisp_check(program.handle, nullptr), "dedisperse_cuda");  // synchronises
  return result;
}

template <typename T>
gaffa::CudaDedispersedSpectrum<T> spectrum_device(gaffa::HostSampleView<T> samples,
                                                  std::span<const double> frequency_mhz,
                                                  const gaffa::SingleDmDedispersionPlan& plan, int device) {
  validate_samples(samples, frequency_mhz);
  DeviceScope scope(device);
  const std::size_t ns = samples.shape.nsamples, nc = samples.shape.nchans;
  uint64_t nout = 0;
  check(gf_dedisperse_spectrum(nullptr, sizeof(T), ns, nc, frequency_mhz.data(), plan.dm, plan.ref_frequency_mhz,
                               plan.tsamp, plan.chan_begin, plan.chan_end, nullptr, &nout, nullptr),
        "dedisperse_spectrum_cuda");
  gaffa::CudaDeviceBuffer<T> input(ns * nc);
  check_cuda(cudaMemcpy(input.data(), samples.data_ptr(), input.bytes(), cudaMemcpyHostToDevice),
             "cudaMemcpy host-to-device spectrum input");
  gaffa::CudaDedispersedSpectrum<T> result;
  const std::size_t width = plan.chan_end - plan.chan_begin;
  result.shape = gaffa::SampleShape{nout, 1, width};
  result.data = gaffa::CudaDeviceBuffer<T>(nout * width);
  check(gf_dedisperse_spectrum(input.data(), sizeof(T), ns, nc, frequency_mhz.data(), plan.dm,
                               plan.ref_frequency_mhz, plan.tsamp, plan.chan_begin, plan.chan_end, result.data.data(),
                               &nout, nullptr),
        "dedisperse_spectrum_cuda");
  check_cuda(cudaStreamSynchronize(nullptr), "dedisperse_spectrum_cuda");
  result.dm = plan.dm;
  result.tsamp = plan.tsamp;
  result.chan_begin = plan.chan_begin;
  result.chan_end = plan.chan_end;
  result.device_id = device;
  return result;
}

template <typename T>
gaffa::DedispersedResult<T> result_to_host(const gaffa::CudaDedispersedResult<T>& result) {
  gaffa::DedispersedResult<T> out;
  out.shape = result.shape;
  out.data.resize(gaffa::dedispersed_element_count(result.shape));
  if (!out.data.empty()) {
    DeviceScope scope(result.device_id);
    check_cuda(cudaMemcpy(out.data.data(), result.data.data(), out.data.size() * sizeof(T), cudaMemcpyDeviceToHost),
               "cudaMemcpy device-to-host dedispersed result");
  }
  return out;
}

template <typename T>
gaffa::DedispersedSpectrum<T> spectrum_to_host(const gaffa::CudaDedispersedSpectrum<T>& result) {
  gaffa::DedispersedSpectrum<T> out;
  out.shape = result.shape;
  out.dm = result.dm;
  out.tsamp = result.tsamp;
  out.chan_begin = result.chan_begin;
  out.chan_end = result.chan_end;
  out.data.resize(result.data.size());
  if (!out.data.empty()) {
    DeviceScope scope(result.device_id);
    check_cuda(cudaMemcpy(out.data.data(), result.data.data(), out.data.size() * sizeof(T), cudaMemcpyDeviceToHost),
               "cudaMemcpy device-to-host dedispersed spectrum");
  }
  return out;
}

}  // namespace

// ---------------------------------------------------------------------------
// RAII device memory (cuda_memory.h)
// ---------------------------------------------------------------------------

gaffa::CudaDeviceMemory::CudaDeviceMemory(std::size_t bytes) {
  if (bytes == 0) return;
  check_cuda(cudaGetDevice(&device_id_), "cudaGetDevice");
  check_cuda(cudaMalloc(&data_, bytes), "cudaMalloc");
  bytes_ = bytes;
}

gaffa::CudaDeviceMemory::CudaDeviceMemory(CudaDeviceMemory&& other) noexcept
    : data_(other.data_), bytes_(other.bytes_), device_id_(other.device_id_) {
  other.data_ = nullptr;
  other.bytes_ = 0;
  other.device_id_ = -1;
}

gaffa::CudaDeviceMemory& gaffa::CudaDeviceMemory::operator=(CudaDeviceMemory&& other) noexcept {
  if (this != &other) {
    release_noexcept();
    data_ = other.data_;
    bytes_ = other.bytes_;
    device_id_ = other.device_id_;
    other.data_ = nullptr;
    other.bytes_ = 0;
    other.device_id_ = -1;
  }
  return *this;
}

gaffa::CudaDeviceMemory::~CudaDeviceMemory() { release_noexcept(); }

void gaffa::CudaDeviceMemory::reset() {
  if (data_ == nullptr) return;
  DeviceScope scope(device_id_);
  check_cuda(cudaFree(data_), "cudaFree");
  data_ = nullptr;
  bytes_ = 0;
  device_id_ = -1;
}

void* gaffa::CudaDeviceMemory::data() noexcept { return data_; }
const void* gaffa::CudaDeviceMemory::data() const noexcept { return data_; }
std::size_t gaffa::CudaDeviceMemory::bytes() const noexcept { return bytes_; }
int gaffa::CudaDeviceMemory::device_id() const noexcept { return device_id_; }

void gaffa::CudaDeviceMemory::release_noexcept() noexcept {
  if (data_ == nullptr) return;
  int previous = -1;
  if (cudaGetDevice(&previous) != cudaSuccess) return;
  const bool switched = previous != device_id_;
  if (switched && cudaSetDevice(device_id_) != cudaSuccess) return;
  if (cudaFree(data_) == cudaSuccess) {
    data_ = nullptr;
    bytes_ = 0;
    device_id_ = -1;
  }
  if (switched) static_cast<void>(cudaSetDevice(previous));
}

// ---------------------------------------------------------------------------
// Dedispersion (dedispersion_cuda.h)
// ---------------------------------------------------------------------------

gaffa::CudaDedispersedResult<std::uint32_t> gaffa::dedisperse_multi_dm_cuda_device(
    HostSampleView<std::uint8_t> samples, std::span<const double> frequency_mhz, const MultiDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options) {
  return dedisperse_u8(samples, frequency_mhz, plan.dm_low, plan.dm_step, plan.ndm, plan.ref_frequency_mhz,
                       plan.tsamp, plan.chan_begin, plan.chan_end, GF_DEDISP_BRUTE, 32, 32, options.device_id);
}

gaffa::CudaDedispersedResult<std::uint32_t> gaffa::dedisperse_multi_dm_cuda_device(
    HostSampleView<std::uint16_t>, std::span<const double>, const MultiDmDedispersionPlan&,
    const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::CudaDedispersedResult<float> gaffa::dedisperse_multi_dm_cuda_device(HostSampleView<float>,
                                                                           std::span<const double>,
                                                                           const MultiDmDedispersionPlan&,
                                                                           const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::CudaDedispersedResult<std::uint32_t> gaffa::dedisperse_single_dm_cuda_device(
    HostSampleView<std::uint8_t> samples, std::span<const double> frequency_mhz, const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options) {
  return dedisperse_u8(samples, frequency_mhz, plan.dm, 0.0, 1, plan.ref_frequency_mhz, plan.tsamp, plan.chan_begin,
                       plan.chan_end, GF_DEDISP_BRUTE, 32, 32, options.device_id);
}

gaffa::CudaDedispersedResult<std::uint32_t> gaffa::dedisperse_single_dm_cuda_device(
    HostSampleView<std::uint16_t>, std::span<const double>, const SingleDmDedispersionPlan&,
    const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::CudaDedispersedResult<float> gaffa::dedisperse_single_dm_cuda_device(HostSampleView<float>,
                                                                            std::span<const double>,
                                                                            const SingleDmDedispersionPlan&,
                                                                            const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::CudaDedispersedResult<std::uint32_t> gaffa::dedisperse_subband_cuda_device(
    HostSampleView<std::uint8_t> samples, std::span<const double> frequency_mhz, const MultiDmDedispersionPlan& plan,
    const SubbandDedispersionOptions& subband_options, const CudaDedispersionOptions& cuda_options) {
  return dedisperse_u8(samples, frequency_mhz, plan.dm_low, plan.dm_step, plan.ndm, plan.ref_frequency_mhz,
                       plan.tsamp, plan.chan_begin, plan.chan_end, GF_DEDISP_SUBBAND,
                       subband_options.subband_channels, subband_options.ndm_per_nominal, cuda_options.device_id);
}

gaffa::CudaDedispersedResult<std::uint32_t> gaffa::dedisperse_subband_cuda_device(
    HostSampleView<std::uint16_t>, std::span<const double>, const MultiDmDedispersionPlan&,
    const SubbandDedispersionOptions&, const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::CudaDedispersedResult<float> gaffa::dedisperse_subband_cuda_device(HostSampleView<float>,
                                                                          std::span<const double>,
                                                                          const MultiDmDedispersionPlan&,
                                                                          const SubbandDedispersionOptions&,
                                                                          const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::CudaDedispersedSpectrum<std::uint8_t> gaffa::dedisperse_spectrum_cuda_device(
    HostSampleView<std::uint8_t> samples, std::span<const double> frequency_mhz, const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options) {
  return spectrum_device(samples, frequency_mhz, plan, options.device_id);
}

gaffa::CudaDedispersedSpectrum<std::uint16_t> gaffa::dedisperse_spectrum_cuda_device(
    HostSampleView<std::uint16_t> samples, std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan, const CudaDedispersionOptions& options) {
  return spectrum_device(samples, frequency_mhz, plan, options.device_id);
}

gaffa::CudaDedispersedSpectrum<float> gaffa::dedisperse_spectrum_cuda_device(HostSampleView<float> samples,
                                                                            std::span<const double> frequency_mhz,
                                                                            const SingleDmDedispersionPlan& plan,
                                                                            const CudaDedispersionOptions& options) {
  return spectrum_device(samples, frequency_mhz, plan, options.device_id);
}

gaffa::DedispersedResult<std::uint32_t> gaffa::copy_to_host(const CudaDedispersedResult<std::uint32_t>& result) {
  return result_to_host(result);
}

gaffa::DedispersedResult<float> gaffa::copy_to_host(const CudaDedispersedResult<float>& result) {
  return result_to_host(result);
}

gaffa::DedispersedSpectrum<std::uint8_t> gaffa::copy_to_host(const CudaDedispersedSpectrum<std::uint8_t>& result) {
  return spectrum_to_host(result);
}

gaffa::DedispersedSpectrum<std::uint16_t> gaffa::copy_to_host(const CudaDedispersedSpectrum<std::uint16_t>& result) {
  return spectrum_to_host(result);
}

gaffa::DedispersedSpectrum<float> gaffa::copy_to_host(const CudaDedispersedSpectrum<float>& result) {
  return spectrum_to_host(result);
}

gaffa::DedispersedSpectrum<std::uint8_t> gaffa::dedisperse_spectrum_cuda(HostSampleView<std::uint8_t> samples,
                                                                         std::span<const double> frequency_mhz,
                                                                         const SingleDmDedispersionPlan& plan,
                                                                         const CudaDedispersionOptions& options) {
  return copy_to_host(dedisperse_spectrum_cuda_device(samples, frequency_mhz, plan, options));
}

gaffa::DedispersedSpectrum<std::uint16_t> gaffa::dedisperse_spectrum_cuda(HostSampleView<std::uint16_t> samples,
                                                                          std::span<const double> frequency_mhz,
                                                                          const SingleDmDedispersionPlan& plan,
                                                                          const CudaDedispersionOptions& options) {
  return copy_to_host(dedisperse_spectrum_cuda_device(samples, frequency_mhz, plan, options));
}

gaffa::DedispersedSpectrum<float> gaffa::dedisperse_spectrum_cuda(HostSampleView<float> samples,
                                                                  std::span<const double> frequency_mhz,
                                                                  const SingleDmDedispersionPlan& plan,
                                                                  const CudaDedispersionOptions& options) {
  return copy_to_host(dedisperse_spectrum_cuda_device(samples, frequency_mhz, plan, options));
}

gaffa::DedispersedResult<std::uint32_t> gaffa::dedisperse_single_dm_cuda(HostSampleView<std::uint8_t> samples,
                                                                         std::span<const double> frequency_mhz,
                                                                         const SingleDmDedispersionPlan& plan,
                                                                         const CudaDedispersionOptions& options) {
  return copy_to_host(dedisperse_single_dm_cuda_device(samples, frequency_mhz, plan, options));
}

gaffa::DedispersedResult<std::uint32_t> gaffa::dedisperse_single_dm_cuda(HostSampleView<std::uint16_t>,
                                                                         std::span<const double>,
                                                                         const SingleDmDedispersionPlan&,
                                                                         const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::DedispersedResult<float> gaffa::dedisperse_single_dm_cuda(HostSampleView<float>, std::span<const double>,
                                                                 const SingleDmDedispersionPlan&,
                                                                 const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::DedispersedResult<std::uint32_t> gaffa::dedisperse_multi_dm_cuda(HostSampleView<std::uint8_t> samples,
                                                                        std::span<const double> frequency_mhz,
                                                                        const MultiDmDedispersionPlan& plan,
                                                                        const CudaDedispersionOptions& options) {
  return copy_to_host(dedisperse_multi_dm_cuda_device(samples, frequency_mhz, plan, options));
}

gaffa::DedispersedResult<std::uint32_t> gaffa::dedisperse_multi_dm_cuda(HostSampleView<std::uint16_t>,
                                                                        std::span<const double>,
                                                                        const MultiDmDedispersionPlan&,
                                                                        const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::DedispersedResult<float> gaffa::dedisperse_multi_dm_cuda(HostSampleView<float>, std::span<const double>,
                                                                const MultiDmDedispersionPlan&,
                                                                const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::DedispersedResult<std::uint32_t> gaffa::dedisperse_subband_cuda(
    HostSampleView<std::uint8_t> samples, std::span<const double> frequency_mhz, const MultiDmDedispersionPlan& plan,
    const SubbandDedispersionOptions& subband_options, const CudaDedispersionOptions& cuda_options) {
  return copy_to_host(dedisperse_subband_cuda_device(samples, frequency_mhz, plan, subband_options, cuda_options));
}

gaffa::DedispersedResult<std::uint32_t> gaffa::dedisperse_subband_cuda(HostSampleView<std::uint16_t>,
                                                                       std::span<const double>,
                                                                       const MultiDmDedispersionPlan&,
                                                                       const SubbandDedispersionOptions&,
                                                                       const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

gaffa::DedispersedResult<float> gaffa::dedisperse_subband_cuda(HostSampleView<float>, std::span<const double>,
                                                               const MultiDmDedispersionPlan&,
                                                               const SubbandDedispersionOptions&,
                                                               const CudaDedispersionOptions&) {
  unsupported_sample_type();
}

// ---------------------------------------------------------------------------
// FFA plan and peaks (ffa_plan.h, ffa_peak.h)
// ---------------------------------------------------------------------------

gaffa::FfaSearchPlan gaffa::make_riptide_ffa_plan(std::size_t nsamples, double tsamp,
                                                  const RiptideFfaPlanOptions& options) {
  gf_plan_options o{options.period_min, options.period_max,    options.bins_min,          options.bins_max,
                    options.min_periods, options.duty_cycle_max, options.width_trial_spacing, options.max_tasks};
  uint64_t ntasks = 0, nwidths = 0;
  check(gf_make_riptide_ffa_plan(nsamples, tsamp, &o, nullptr, 0, &ntasks, nullptr, 0, &nwidths),
        "make_riptide_ffa_plan");
  std::vector<gf_ffa_task> tasks(ntasks);
  std::vector<uint64_t> widths(nwidths);
  check(gf_make_riptide_ffa_plan(nsamples, tsamp, &o, tasks.data(), ntasks, &ntasks, widths.data(), nwidths,
                                 &nwidths),
        "make_riptide_ffa_plan");
  FfaSearchPlan plan;
  for (const gf_ffa_task& t : tasks)
    plan.tasks.push_back(FfaSearchTask{t.downsample_factor, t.effective_tsamp, t.input_nsamples, t.prepared_nsamples,
                                       t.bins, t.rows, t.rows_eval, t.period_begin, t.period_end});
  plan.width_trials.assign(widths.begin(), widths.end());
  return plan;
}

bool gaffa::is_better_ffa_peak(const FfaPeak& lhs, const FfaPeak& rhs) {
  const bool lf = std::isfinite(lhs.snr) && std::isfinite(lhs.period) && std::isfinite(lhs.frequency);
  const bool rf = std::isfinite(rhs.snr) && std::isfinite(rhs.period) && std::isfinite(rhs.frequency);
  if (lf != rf) return lf;
  if (lhs.snr != rhs.snr) return lhs.snr > rhs.snr;
  if (lhs.period != rhs.period) return lhs.period < rhs.period;
  if (lhs.frequency != rhs.frequency) return lhs.frequency < rhs.frequency;
  if (lhs.width != rhs.width) return lhs.width < rhs.width;
  if (lhs.phase != rhs.phase) return lhs.phase < rhs.phase;
  if (lhs.shift != rhs.shift) return lhs.shift < rhs.shift;
  return lhs.bins < rhs.bins;
}

void gaffa::sort_ffa_peaks(std::vector<FfaPeak>& peaks) { std::sort(peaks.begin(), peaks.end(), is_better_ffa_peak); }

// ---------------------------------------------------------------------------
// CUDA FFA program (ffa_cuda.h)
// ---------------------------------------------------------------------------

struct gaffa::CudaFfaProgramImpl {
  gf_ffa_program* program = nullptr;
  int device = 0;
  std::size_t tile = 0;
  std::size_t nsamples = 0;
  gf_ffa_info info{};
  CudaFfaExecutionOptions execution{};
  CudaFfaWorkspaceShape shape{};
  CudaDeviceBuffer<float> prepared;
  CudaDeviceBuffer<std::uint8_t> scratch;
  CudaDeviceBuffer<gf_peak_record> peaks;
  CudaDeviceBuffer<std::uint64_t> counters;

  ~CudaFfaProgramImpl() {
    if (program) gf_ffa_program_destroy(program);
  }
};

gaffa::CudaFfaProgram::CudaFfaProgram(const FfaSearchPlan& plan, const CudaFfaProgramOptions& program_options,
                                      const CudaFfaExecutionOptions& execution_options) {
  if (plan.tasks.empty()) throw std::invalid_argument("FFA program plan must contain at least one task");
  if (plan.width_trials.empty()) throw std::invalid_argument("FFA search plan width_trials must not be empty");
  if (execution_options.series_tile_size == 0) throw std::invalid_argument("series_tile_size must be positive");
  auto impl = std::make_unique<CudaFfaProgramImpl>();
  impl->device = program_options.device_id;
  impl->tile = execution_options.series_tile_size;
  impl->execution = execution_options;
  impl->nsamples = plan.tasks.front().input_nsamples;
  DeviceScope scope(impl->device);
  std::vector<gf_ffa_task> tasks;
  for (const FfaSearchTask& t : plan.tasks)
    tasks.push_back(gf_ffa_task{t.downsample_factor, t.effective_tsamp, t.input_nsamples, t.prepared_nsamples, t.bins,
                                t.rows, t.rows_eval, t.period_begin, t.period_end});
  std::vector<uint64_t> widths(plan.width_trials.begin(), plan.width_trials.end());
  check(gf_ffa_program_create(tasks.data(), tasks.size(), widths.data(), widths.size(), impl->tile, impl->device,
                              &impl->program),
        "CudaFfaProgram");
  check(gf_ffa_program_info(impl->program, &impl->info), "CudaFfaProgram");
  impl->prepared = CudaDeviceBuffer<float>(impl->tile * impl->info.prepared_floats);
  impl->scratch = CudaDeviceBuffer<std::uint8_t>(std::max<std::size_t>(16, impl->info.scratch_bytes));
  impl->peaks = CudaDeviceBuffer<gf_peak_record>(
      std::max<std::size_t>(1024, execution_options.initial_peak_buffer_bytes / sizeof(gf_peak_record)));
  impl->counters = CudaDeviceBuffer<std::uint64_t>(2);
  CudaFfaWorkspaceShape& s = impl->shape;
  s.series_tile_size = impl->tile;
  s.max_prepared_nsamples = impl->info.prepared_floats;
  s.max_task_elements = impl->info.max_task_elements;
  s.prepared_bytes = impl->prepared.bytes();
  s.scratch_bytes = impl->scratch.bytes();
  s.detection_compact_bytes = impl->peaks.bytes() + impl->counters.bytes();
  s.total_bytes = s.prepared_bytes + s.scratch_bytes + s.detection_compact_bytes;
  if (execution_options.workspace_bytes_limit != 0 && s.total_bytes > execution_options.workspace_bytes_limit)
    throw std::invalid_argument("CUDA FFA workspace exceeds workspace_bytes_limit");
  impl_ = std::move(impl);
}

gaffa::CudaFfaProgram::~CudaFfaProgram() = default;
gaffa::CudaFfaProgram::CudaFfaProgram(CudaFfaProgram&&) noexcept = default;
gaffa::CudaFfaProgram& gaffa::CudaFfaProgram::operator=(CudaFfaProgram&&) noexcept = default;

bool gaffa::CudaFfaProgram::empty() const noexcept { return impl_ == nullptr; }

int gaffa::CudaFfaProgram::device_id() const {
  if (!impl_) throw std::logic_error("CUDA FFA program is empty");
  return impl_->device;
}

std::size_t gaffa::CudaFfaProgram::tile_capacity() const {
  if (!impl_) throw std::logic_error("CUDA FFA program is empty");
  return impl_->tile;
}

const gaffa::CudaFfaWorkspaceShape& gaffa::CudaFfaProgram::workspace_shape() const {
  if (!impl_) throw std::logic_error("CUDA FFA program is empty");
  return impl_->shape;
}

std::size_t gaffa::CudaFfaProgram::device_metadata_bytes() const {
  if (!impl_) throw std::logic_error("CUDA FFA program is empty");
  return impl_->info.metadata_bytes;
}

gaffa::FfaBatchSearchResult gaffa::run_ffa_batch_cuda(CudaFfaProgram& program, CudaTimeSeriesBatchView batch,
                                                      const FfaSearchOptions& options) {
  if (program.empty()) throw std::invalid_argument("CUDA FFA program must not be empty");
  CudaFfaProgramImpl& p = *program.impl_;
  if (!std::isfinite(options.snr_threshold)) throw std::invalid_argument("FFA search S/N threshold must be finite");
  if (batch.data == nullptr || batch.nseries == 0) throw std::invalid_argument("CUDA FFA batch must not be empty");
  if (batch.nseries > p.tile) throw std::invalid_argument("CUDA FFA batch exceeds the program's tile capacity");
  if (batch.nsamples != p.nsamples)
    throw std::invalid_argument("FFA executor task input_nsamples must match time series size");
  if (batch.device_id != p.device) throw std::invalid_argument("CUDA FFA batch device_id must match the program");
  DeviceScope scope(p.device);
  cudaStream_t stream = p.execution.stream;
  check(gf_ffa_prepare(p.program, batch.data, batch.nseries, batch.nsamples, nullptr, p.prepared.data(), stream),
        "run_ffa_batch_cuda");
  std::uint64_t counts[2] = {0, 0};
  for (;;) {
    check(gf_ffa_search(p.program, p.prepared.data(), batch.nseries, options.snr_threshold, p.scratch.data(),
                        p.peaks.data(), p.peaks.size(), p.counters.data(), stream),
          "run_ffa_batch_cuda");
    check_cuda(cudaMemcpyAsync(counts, p.counters.data(), sizeof counts, cudaMemcpyDeviceToHost, stream),
               "cudaMemcpyAsync FFA peak count");
    check_cuda(cudaStreamSynchronize(stream), "run_ffa_batch_cuda");
    if (counts[1] & GF_STATUS_SCHEDULE) throw std::runtime_error("run_ffa_batch_cuda: FFA schedule exceeded its tile");
    if (counts[0] <= p.peaks.size()) break;
    // the reference grows its peak buffer and re-runs (ffa_cuda_executor.cuh:395-404)
    const std::size_t grown = counts[0] + counts[0] / 4 + 1024;
    if (grown * sizeof(gf_peak_record) > p.execution.max_peak_buffer_bytes)
      throw std::runtime_error("run_ffa_batch_cuda: peak count exceeds max_peak_buffer_bytes");
    p.peaks = CudaDeviceBuffer<gf_peak_record>(grown);
  }
  const std::size_t n = counts[0];
  std::vector<gf_peak_record> records(n);
  if (n)
    check_cuda(cudaMemcpy(records.data(), p.peaks.data(), n * sizeof(gf_peak_record), cudaMemcpyDeviceToHost),
               "cudaMemcpy device-to-host FFA peaks");
  if (options.max_peaks != 0) {
    std::vector<std::size_t> per_series(batch.nseries, 0);
    for (const gf_peak_record& r : records)
      if (++per_series[r.series] > options.max_peaks)
        throw std::runtime_error("FFA detection peak count exceeded max_peaks safety guard");
  }
  std::vector<gf_peak> expanded(n);
  if (n) check(gf_ffa_expand_peaks(p.program, records.data(), n, 0, 0.0, 1.0, expanded.data()), "run_ffa_batch_cuda");
  FfaBatchSearchResult result;
  result.peaks.reserve(n);
  for (const gf_peak& e : expanded)
    result.peaks.push_back(FfaBatchPeak{
        e.dm_index, FfaPeak{e.period, e.frequency, e.width, e.duty_cycle, e.width_index, e.period_index, e.phase,
                            e.shift, e.bins, e.snr}});
  std::sort(result.peaks.begin(), result.peaks.end(), [](const FfaBatchPeak& l, const FfaBatchPeak& r) {
    if (l.series_index != r.series_index) return l.series_index < r.series_index;
    return is_better_ffa_peak(l.peak, r.peak);
  });
  return result;
}

gaffa::FfaSearchResult gaffa::search_ffa_cuda(CudaFfaProgram& program, CudaSpan<const float> time_series,
                                              const FfaSearchOptions& options) {
  if (time_series.data == nullptr || time_series.count == 0)
    throw std::invalid_argument("FFA time_series must not be empty");
  FfaBatchSearchResult batch = run_ffa_batch_cuda(
      program, CudaTimeSeriesBatchView{time_series.data, 1, time_series.count, time_series.device_id}, options);
  FfaSearchResult result;
  result.peaks.reserve(batch.peaks.size());
  for (const FfaBatchPeak& p : batch.peaks) result.peaks.push_back(p.peak);
  return result;
}

gaffa::FfaSearchResult gaffa::search_ffa_cuda(CudaSpan<const float> time_series, const FfaSearchPlan& plan,
                                              const FfaSearchOptions& options,
                                              const CudaFfaProgramOptions& program_options,
                                              const CudaFfaExecutionOptions& execution_options) {
  CudaFfaExecutionOptions one = execution_options;
  one.series_tile_size = 1;
  CudaFfaProgram program(plan, program_options, one);
  return search_ffa_cuda(program, time_series, options);
}
