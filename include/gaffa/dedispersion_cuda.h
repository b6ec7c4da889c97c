// gaffa C++ API on the B200 path: CUDA dedispersion (the reference's
// include/gaffa/dedispersion_cuda.h:10-306, same types, overloads and
// defaults).  Implemented in gaffa_b200/csrc/cxx_api.cpp over the C ABI of
// gaffa_b200.h (libgaffa_b200.so).  Host-returning functions copy the result
// back; *_device functions return device-resident results that own their
// memory.  Failures throw std::invalid_argument / std::overflow_error for
// invalid input and std::runtime_error("<operation>: <message>") for CUDA
// errors, as the reference does.
//
// Sample types: the direct-sum (multi-DM, single-DM) and subband paths take
// uint8 samples, the sample type of the search path; their uint16 and float
// overloads exist for source compatibility and throw std::invalid_argument.
// The aligned spectrum takes all three types.
#pragma once

#include "gaffa/cuda_memory.h"
#include "gaffa/dedispersion.h"

#include <cstddef>
#include <cstdint>
#include <span>

namespace gaffa {

struct CudaDedispersionOptions {
  int device_id = 0;
  std::size_t threads_per_block = 256;
  std::size_t time_tile_samples = 81920;
};

template <typename T>
struct CudaDedispersedView {
  T* data = nullptr;
  DedispersedShape shape{};
  int device_id = 0;

  CudaSpan<T> as_span() const noexcept { return CudaSpan<T>{data, size(), device_id}; }
  std::size_t size() const noexcept { return shape.ndm * shape.nsamples; }
  std::size_t bytes() const noexcept { return as_span().bytes(); }
};

template <typename T>
struct CudaDedispersedResult {
  CudaDeviceBuffer<T> data;
  DedispersedShape shape{};
  int device_id = 0;

  CudaDedispersedView<T> view() noexcept { return CudaDedispersedView<T>{data.data(), shape, device_id}; }
  CudaDedispersedView<const T> view() const noexcept {
    return CudaDedispersedView<const T>{data.data(), shape, device_id};
  }
  std::size_t size() const noexcept { return data.size(); }
  std::size_t bytes() const noexcept { return data.bytes(); }
};

template <typename T>
struct CudaDedispersedSpectrumView {
  T* data = nullptr;
  SampleShape shape{};
  int device_id = 0;

  CudaSpan<T> as_span() const noexcept { return CudaSpan<T>{data, size(), device_id}; }
  std::size_t size() const noexcept { return shape.nsamples * shape.nchans; }
  std::size_t bytes() const noexcept { return as_span().bytes(); }
};

template <typename T>
struct CudaDedispersedSpectrum {
  CudaDeviceBuffer<T> data;
  SampleShape shape{};
  double dm = 0.0;
  double tsamp = 0.0;
  std::size_t chan_begin = 0;
  std::size_t chan_end = 0;
  int device_id = 0;

  CudaDedispersedSpectrumView<T> view() noexcept {
    return CudaDedispersedSpectrumView<T>{data.data(), shape, device_id};
  }
  CudaDedispersedSpectrumView<const T> view() const noexcept {
    return CudaDedispersedSpectrumView<const T>{data.data(), shape, device_id};
  }
  std::size_t size() const noexcept { return data.size(); }
  std::size_t bytes() const noexcept { return data.bytes(); }
};

DedispersedSpectrum<std::uint8_t> dedisperse_spectrum_cuda(
    HostSampleView<std::uint8_t> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedSpectrum<std::uint16_t> dedisperse_spectrum_cuda(
    HostSampleView<std::uint16_t> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedSpectrum<float> dedisperse_spectrum_cuda(
    HostSampleView<float> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedResult<std::uint32_t> dedisperse_single_dm_cuda(
    HostSampleView<std::uint8_t> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedResult<std::uint32_t> dedisperse_single_dm_cuda(
    HostSampleView<std::uint16_t> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedResult<float> dedisperse_single_dm_cuda(
    HostSampleView<float> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedResult<std::uint32_t> dedisperse_multi_dm_cuda(
    HostSampleView<std::uint8_t> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedResult<std::uint32_t> dedisperse_multi_dm_cuda(
    HostSampleView<std::uint16_t> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedResult<float> dedisperse_multi_dm_cuda(
    HostSampleView<float> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

DedispersedResult<std::uint32_t> dedisperse_subband_cuda(
    HostSampleView<std::uint8_t> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const SubbandDedispersionOptions& subband_options = {},
    const CudaDedispersionOptions& cuda_options = {});

DedispersedResult<std::uint32_t> dedisperse_subband_cuda(
    HostSampleView<std::uint16_t> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const SubbandDedispersionOptions& subband_options = {},
    const CudaDedispersionOptions& cuda_options = {});

DedispersedResult<float> dedisperse_subband_cuda(
    HostSampleView<float> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const SubbandDedispersionOptions& subband_options = {},
    const CudaDedispersionOptions& cuda_options = {});

CudaDedispersedResult<std::uint32_t> dedisperse_single_dm_cuda_device(
    HostSampleView<std::uint8_t> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedResult<std::uint32_t> dedisperse_single_dm_cuda_device(
    HostSampleView<std::uint16_t> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedResult<float> dedisperse_single_dm_cuda_device(
    HostSampleView<float> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedSpectrum<std::uint8_t> dedisperse_spectrum_cuda_device(
    HostSampleView<std::uint8_t> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedSpectrum<std::uint16_t> dedisperse_spectrum_cuda_device(
    HostSampleView<std::uint16_t> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedSpectrum<float> dedisperse_spectrum_cuda_device(
    HostSampleView<float> samples,
    std::span<const double> frequency_mhz,
    const SingleDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedResult<std::uint32_t> dedisperse_multi_dm_cuda_device(
    HostSampleView<std::uint8_t> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedResult<std::uint32_t> dedisperse_multi_dm_cuda_device(
    HostSampleView<std::uint16_t> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedResult<float> dedisperse_multi_dm_cuda_device(
    HostSampleView<float> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const CudaDedispersionOptions& options = {});

CudaDedispersedResult<std::uint32_t> dedisperse_subband_cuda_device(
    HostSampleView<std::uint8_t> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const SubbandDedispersionOptions& subband_options = {},
    const CudaDedispersionOptions& cuda_options = {});

CudaDedispersedResult<std::uint32_t> dedisperse_subband_cuda_device(
    HostSampleView<std::uint16_t> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const SubbandDedispersionOptions& subband_options = {},
    const CudaDedispersionOptions& cuda_options = {});

CudaDedispersedResult<float> dedisperse_subband_cuda_device(
    HostSampleView<float> samples,
    std::span<const double> frequency_mhz,
    const MultiDmDedispersionPlan& plan,
    const SubbandDedispersionOptions& subband_options = {},
    const CudaDedispersionOptions& cuda_options = {});

DedispersedResult<std::uint32_t> copy_to_host(const CudaDedispersedResult<std::uint32_t>& result);

DedispersedResult<float> copy_to_host(const CudaDedispersedResult<float>& result);

DedispersedSpectrum<std::uint8_t> copy_to_host(const CudaDedispersedSpectrum<std::uint8_t>& result);

DedispersedSpectrum<std::uint16_t> copy_to_host(const CudaDedispersedSpectrum<std::uint16_t>& result);

DedispersedSpectrum<float> copy_to_host(const CudaDedispersedSpectrum<float>& result);

}  // namespace gaffa
