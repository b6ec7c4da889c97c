// gaffa C++ API on the B200 path: device time-series batch views
// (the reference's include/gaffa/time_series_cuda.h:10-40).
#pragma once

#include "gaffa/cuda_memory.h"
#include "gaffa/launch_cuda.h"

#include <cstddef>
#include <cstdint>

namespace gaffa {

// Dense [series][sample] float batch in device memory.
struct CudaTimeSeriesBatchView {
  const float* data = nullptr;
  std::size_t nseries = 0;
  std::size_t nsamples = 0;
  int device_id = 0;

  [[nodiscard]] std::size_t size() const noexcept { return nseries * nsamples; }
};

struct MutableCudaTimeSeriesBatchView {
  float* data = nullptr;
  std::size_t nseries = 0;
  std::size_t nsamples = 0;
  int device_id = 0;

  [[nodiscard]] std::size_t size() const noexcept { return nseries * nsamples; }
  [[nodiscard]] CudaTimeSeriesBatchView as_const() const noexcept {
    return CudaTimeSeriesBatchView{data, nseries, nsamples, device_id};
  }
};

}  // namespace gaffa
