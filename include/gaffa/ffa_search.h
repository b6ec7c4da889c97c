// gaffa C++ API on the B200 path: FFA search options and results
// (the reference's include/gaffa/ffa_search.h; search_ffa_cpu is not part of
// this library, which has no CPU path -- use search_ffa_cuda, ffa_cuda.h).
#pragma once

#include "gaffa/ffa_peak.h"
#include "gaffa/ffa_plan.h"

#include <cstddef>
#include <span>
#include <vector>

namespace gaffa {

struct FfaSearchOptions {
  float snr_threshold = 6.0F;
  std::size_t max_peaks = 0;  // per series; 0 = unbounded, else exceeding it throws
};

struct FfaSearchResult {
  std::vector<FfaPeak> peaks;
};

}  // namespace gaffa
