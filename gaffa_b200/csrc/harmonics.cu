// Harmonic flagging of large candidate lists on the device.
//
// flag_harmonics_cpu (harmonic.cpp:245-292) ranks the candidates, then for
// every candidate that is not itself a harmonic tests every later candidate
// that is not yet a harmonic; a child takes the relation of the first such
// parent.  That is n^2 / 2 pairwise tests: with strong RFI the wide-range
// workload yields ~2.8e5 candidates, minutes on one core.
//
// Equivalently, child c is a harmonic of the smallest p < c that is not a
// harmonic itself and passes the test with c.  The status of p depends only
// on candidates before p, so the list is swept in chunks of kChunk in ranking
// order:
//   outer_kernel  every child of the chunk against every parent before the
//                 chunk (final statuses), in parallel over children and
//                 parent tiles; the smallest matching parent wins (atomicMin);
//   inner_kernel  one CTA walks the chunk's own candidates as parents in
//                 order (a barrier per parent), for the children still
//                 unmatched.
// The test is harmonic_math.cuh's, shared with the host loop, with explicitly
// rounded FP64 operations, so every decision equals the host's; the host
// recomputes the relation fields of each matched pair with the same code.
#include "common.cuh"
#include "harmonic_math.cuh"

#include <algorithm>
#include <vector>

namespace gf {
namespace {

constexpr int kChunk = 512;          // candidates per sweep step (inner CTA size)
constexpr int kOuterThreads = 256;   // children per outer CTA
constexpr int kParentTile = 2048;    // parents per outer CTA
constexpr int kMaxRatios = 128;
constexpr uint32_t kNone = 0xffffffffu;

struct HarmonicParams {
  double observation_seconds, band;
  gf_harmonic_options options;
  int nratios;
};

__device__ __forceinline__ void load_ratios(const HarmonicRatio* g, int n, HarmonicRatio* s) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = g[i];
}

// Children [c0, c1) against parents [p0, min(p0 + kParentTile, c0)); match[c]
// takes the smallest matching parent that is not a harmonic.
__global__ void __launch_bounds__(kOuterThreads) outer_kernel(const HarmonicInput* __restrict__ cand,
                                                              uint32_t* match, uint32_t c0, uint32_t c1,
                                                              const HarmonicRatio* __restrict__ ratios,
                                                              HarmonicParams hp) {
  __shared__ HarmonicRatio sr[kMaxRatios];
  __shared__ HarmonicInput sp[kOuterThreads];
  __shared__ uint32_t sok[kOuterThreads];
  load_ratios(ratios, hp.nratios, sr);
  const uint32_t c = c0 + blockIdx.x * kOuterThreads + threadIdx.x;
  const bool valid = c < c1;
  const uint32_t p0 = blockIdx.y * kParentTile;
  const uint32_t p1 = min(p0 + static_cast<uint32_t>(kParentTile), c0);
  HarmonicInput mine{};
  uint32_t best = kNone;
  if (valid) {
    mine = cand[c];
    best = match[c];  // another tile may already hold a smaller parent
  }
  bool done = !valid || best < p0;
  for (uint32_t t0 = p0; t0 < p1; t0 += kOuterThreads) {
    __syncthreads();
    const uint32_t p = t0 + threadIdx.x;
    if (p < p1) {
      sp[threadIdx.x] = cand[p];
      sok[threadIdx.x] = match[p] == kNone ? 1u : 0u;  // harmonics are no parents
    }
    __syncthreads();
    if (__syncthreads_and(done ? 1 : 0)) break;
    if (done) continue;
    const uint32_t cnt = min(static_cast<uint32_t>(kOuterThreads), p1 - t0);
    for (uint32_t j = 0; j < cnt; ++j) {
      if (t0 + j >= best) {
        done = true;
        break;
      }
      if (sok[j] && harmonic_test(sp[j], mine, sr, hp.nratios, hp.observation_seconds, hp.band, hp.options, 0,
                                  nullptr)) {
        best = t0 + j;
        done = true;
        break;
      }
    }
  }
  if (valid && best != kNone) atomicMin(&match[c], best);
}

// The chunk's own candidates as parents, in ranking order; blockDim = kChunk.
__global__ void __launch_bounds__(kChunk) inner_kernel(const HarmonicInput* __restrict__ cand, uint32_t* match,
                                                       uint32_t c0, uint32_t c1,
                                                       const HarmonicRatio* __restrict__ ratios, HarmonicParams hp) {
  __shared__ HarmonicRatio sr[kMaxRatios];
  __shared__ HarmonicInput sc[kChunk];
  __shared__ uint32_t sm[kChunk];
  load_ratios(ratios, hp.nratios, sr);
  const uint32_t t = threadIdx.x;
  const uint32_t c = c0 + t;
  const bool valid = c < c1;
  if (valid) {
    sc[t] = cand[c];
    sm[t] = match[c];
  }
  __syncthreads();
  const uint32_t n = c1 - c0;
  for (uint32_t j = 0; j + 1 < n; ++j) {
    // sm[j] is final: only candidates before j could set it
    if (valid && t > j && sm[j] == kNone && sm[t] == kNone &&
        harmonic_test(sc[j], sc[t], sr, hp.nratios, hp.observation_seconds, hp.band, hp.options, 0, nullptr))
      sm[t] = c0 + j;
    __syncthreads();
  }
  if (valid) match[c] = sm[t];
}

}  // namespace

void flag_harmonics_on_device(const std::vector<HarmonicInput>& candidates, const std::vector<HarmonicRatio>& ratios,
                              double observation_seconds, double band, const gf_harmonic_options& options,
                              int device, void* stream, std::vector<uint32_t>& parent) {
  const uint64_t n = candidates.size();
  check_arg(n < kNone, "too many candidates for device harmonic flagging");
  check_arg(ratios.size() <= static_cast<size_t>(kMaxRatios), "too many harmonic ratios for device flagging");
  parent.assign(n, kNone);
  if (n == 0) return;
  DeviceGuard dg(device);
  auto s = as_stream(stream);
  DeviceBlob cand_d, ratios_d, match_d;
  cand_d.upload(candidates.data(), n * sizeof(HarmonicInput), device);
  ratios_d.upload(ratios.data(), std::max<size_t>(1, ratios.size()) * sizeof(HarmonicRatio), device);
  match_d.upload(parent.data(), n * sizeof(uint32_t), device);  // all kNone
  HarmonicParams hp{observation_seconds, band, options, static_cast<int>(ratios.size())};
  uint32_t* match = match_d.as<uint32_t>();
  for (uint64_t c0 = 0; c0 < n; c0 += kChunk) {
    const uint64_t c1 = std::min<uint64_t>(n, c0 + kChunk);
    if (c0 > 0) {
      const dim3 grid(static_cast<unsigned>(ceil_div(c1 - c0, kOuterThreads)),
                      static_cast<unsigned>(ceil_div(c0, kParentTile)));
      outer_kernel<<<grid, kOuterThreads, 0, s>>>(cand_d.as<HarmonicInput>(), match, static_cast<uint32_t>(c0),
                                                  static_cast<uint32_t>(c1), ratios_d.as<HarmonicRatio>(), hp);
    }
    inner_kernel<<<1, kChunk, 0, s>>>(cand_d.as<HarmonicInput>(), match, static_cast<uint32_t>(c0),
                                      static_cast<uint32_t>(c1), ratios_d.as<HarmonicRatio>(), hp);
  }
  cuda_check(cudaGetLastError(), "harmonic flagging launch");
  cuda_check(cudaMemcpyAsync(parent.data(), match, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
             "harmonic flags");
  cuda_check(cudaStreamSynchronize(s), "harmonic flagging");
}

}  // namespace gf
