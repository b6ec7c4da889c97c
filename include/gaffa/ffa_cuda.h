// gaffa C++ API on the B200 path: the CUDA FFA program and batch search
// (the reference's include/gaffa/ffa_cuda.h:20-279: CudaFfaProgramOptions,
// CudaFfaExecutionOptions, FfaBatchPeak, FfaBatchSearchResult,
// CudaFfaProgram, run_ffa_batch_cuda and both search_ffa_cuda overloads,
// same signatures and defaults).  The program owns the plan's device tables
// and a reusable workspace for series_tile_size series; it is move-only, not
// thread-safe, and runs one batch at a time.  Implemented in
// gaffa_b200/csrc/cxx_api.cpp over gf_ffa_* of gaffa_b200.h.
#pragma once

#include "gaffa/cuda_memory.h"
#include "gaffa/ffa.h"
#include "gaffa/ffa_search.h"
#include "gaffa/launch_cuda.h"
#include "gaffa/time_series_cuda.h"

#include <cstddef>
#include <memory>
#include <span>
#include <vector>

namespace gaffa {

namespace detail {
class CudaFfaTileRunner;
}

struct CudaFfaProgramOptions {
  int device_id = 0;
};

struct CudaFfaExecutionOptions {
  std::size_t series_tile_size = 16;
  std::size_t threads_per_block = 256;
  std::size_t workspace_bytes_limit = 0;
  std::size_t initial_peak_buffer_bytes = 64ULL * 1024ULL * 1024ULL;
  std::size_t max_peak_buffer_bytes = 1024ULL * 1024ULL * 1024ULL;
  cudaStream_t stream = nullptr;

  [[nodiscard]] CudaLaunchOptions async_launch_options(int device_id) const noexcept {
    return CudaLaunchOptions{device_id, threads_per_block, stream, false};
  }
};

struct FfaBatchPeak {
  std::size_t series_index = 0;
  FfaPeak peak{};
};

struct FfaBatchSearchResult {
  std::vector<FfaBatchPeak> peaks;
};

struct CudaFfaWorkspaceShape {
  std::size_t series_tile_size = 0;
  std::size_t max_prepared_nsamples = 0;
  std::size_t max_task_elements = 0;
  std::size_t max_detection_slots_per_series = 0;
  std::size_t prepared_bytes = 0;
  std::size_t scratch_bytes = 0;
  std::size_t output_bytes = 0;
  std::size_t detection_compact_bytes = 0;
  std::size_t total_bytes = 0;
};

struct CudaFfaProgramImpl;

class CudaFfaProgram {
 public:
  explicit CudaFfaProgram(const FfaSearchPlan& plan, const CudaFfaProgramOptions& program_options = {},
                          const CudaFfaExecutionOptions& execution_options = {});
  ~CudaFfaProgram();

  CudaFfaProgram(CudaFfaProgram&&) noexcept;
  CudaFfaProgram& operator=(CudaFfaProgram&&) noexcept;
  CudaFfaProgram(const CudaFfaProgram&) = delete;
  CudaFfaProgram& operator=(const CudaFfaProgram&) = delete;

  [[nodiscard]] bool empty() const noexcept;
  [[nodiscard]] int device_id() const;
  [[nodiscard]] std::size_t tile_capacity() const;
  [[nodiscard]] const CudaFfaWorkspaceShape& workspace_shape() const;
  [[nodiscard]] std::size_t device_metadata_bytes() const;

 private:
  friend class detail::CudaFfaTileRunner;
  friend FfaBatchSearchResult run_ffa_batch_cuda(CudaFfaProgram& program, CudaTimeSeriesBatchView batch,
                                                 const FfaSearchOptions& options);

  std::unique_ptr<CudaFfaProgramImpl> impl_;
};

// Searches one preprocessed dense [series][sample] tile (at most
// program.tile_capacity() series).  series_index is local to the tile; peaks
// are ordered by series, then is_better_ffa_peak.
FfaBatchSearchResult run_ffa_batch_cuda(CudaFfaProgram& program, CudaTimeSeriesBatchView batch,
                                        const FfaSearchOptions& options = {});

// One device series with a reusable program; peaks in is_better_ffa_peak order.
FfaSearchResult search_ffa_cuda(CudaFfaProgram& program, CudaSpan<const float> time_series,
                                const FfaSearchOptions& options = {});

// One-shot convenience form (builds a program for the plan).
FfaSearchResult search_ffa_cuda(CudaSpan<const float> time_series, const FfaSearchPlan& plan,
                                const FfaSearchOptions& options = {},
                                const CudaFfaProgramOptions& program_options = {},
                                const CudaFfaExecutionOptions& execution_options = {});

}  // namespace gaffa
