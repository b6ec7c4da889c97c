// Running-median detrend and normalisation for sm_100a.
//
// Reference arithmetic (src/gaffa/preprocessing.cpp, time_series.cpp):
//   window  = odd(round(window_seconds / tsamp))                :164-188
//   scrunch = max(1, floor(window / min_points))                :124-145
//   low[k]  = float(sum_{i<F} double(x[kF+i]) / F)              :78-92
//   median  = upper median of the edge-padded low-res window    :53-76
//   trend   = float((1-f)*low_med[j] + f*low_med[j+1])          :94-122
//   y       = x - trend                                         :212-231
//   mean, var from sequential FP64 sums of y and y*y            time_series.cpp:50-78
//   z       = float((y - mean) * (1/stddev))                    time_series.cpp:80-104
// Every FP64 step uses explicit _rn intrinsics so nvcc cannot contract a
// multiply-add into an FMA, and the FP64 sums run in the reference's
// sequential order (one thread per series), so outputs are bit-identical to
// the CPU path.
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace gf {
namespace {

constexpr int kMaxMedianWindow = 2047;
constexpr int kMedianWarps = 4;
constexpr int kStatsWarps = 4;

__device__ __forceinline__ float load_sample(const void* base, uint64_t i, bool u32) {
  if (u32) return static_cast<float>(static_cast<const uint32_t*>(base)[i]);
  return static_cast<const float*>(base)[i];
}
// for inputs no thread of the launch writes (scrunch and median inputs)
__device__ __forceinline__ float load_sample_ro(const void* base, uint64_t i, bool u32) {
  if (u32) return static_cast<float>(__ldg(static_cast<const uint32_t*>(base) + i));
  return __ldg(static_cast<const float*>(base) + i);
}

// One set of series of one length in a preprocessing launch: the arguments of
// gf_preprocess_inplace evaluated for every stage.
struct PrepItem {
  void* series;         // [nseries][stride] uint32 or float, detrended in place
  uint64_t stride, n;
  uint64_t factor, low_n, low_stride;
  float* low;           // scrunched series [nseries][low_stride] (factor > 1)
  float* lowmed;        // running median [nseries][low_stride]
  double* stats;        // [nseries][2]
  uint32_t* status;
  uint32_t nseries;
  int32_t w;            // median window (odd)
  int32_t u32;          // series holds uint32 sums
  int32_t normalise, reject_constant;
  int32_t reserved;
};

enum PrepStage { kScrunch = 0, kMedian, kDetrend, kStats, kStages };

// x blocks per series of the scrunch and detrend stages (1 for the others).
uint64_t stage_xblocks(const PrepItem& it, int stage) {
  switch (stage) {
    case kScrunch: return it.factor > 1 ? ceil_div(it.low_n, 128) : 0;
    case kDetrend: return ceil_div(it.n, 256);
    default: return 1;
  }
}

// CTAs of an item in each stage's batched launch.
uint64_t stage_ctas(const PrepItem& it, int stage) {
  switch (stage) {
    case kScrunch: return it.factor > 1 ? ceil_div(it.low_n, 128) * it.nseries : 0;
    case kMedian: return ceil_div(it.nseries, kMedianWarps);
    case kDetrend: return ceil_div(it.n, 256) * it.nseries;
    default: return ceil_div(it.nseries, kStatsWarps);
  }
}

// The items of a launch: a device table (batched) or one item by value.
struct PrepTable {
  const PrepItem* items;   // null: `one` is the launch's only item
  const uint64_t* begin;   // [kStages][nitems]: first CTA of each item in each stage
  int32_t nitems;
  PrepItem one;
};

// The item of this CTA and the CTA's index inside it.  A single-item launch
// (Batched = false) reads the kernel parameter directly; a batched one has
// thread 0 find the item (the last one starting at or before the CTA) and
// share a copy.  Launches stay below 2^31 CTAs, so CTA indices are 32-bit.
template <bool Batched>
__device__ __forceinline__ const PrepItem& cta_item(const PrepTable& t, int stage, PrepItem& shared_it,
                                                    uint32_t& shared_local, uint32_t& local) {
  if (!Batched) {
    local = blockIdx.x;
    return t.one;
  }
  if (threadIdx.x == 0) {
    const uint64_t b = blockIdx.x;
    const uint64_t* begin = t.begin + static_cast<uint64_t>(stage) * t.nitems;
    int lo = 0, hi = t.nitems;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (begin[mid] <= b) lo = mid; else hi = mid;
    }
    shared_it = t.items[lo];
    shared_local = static_cast<uint32_t>(b - begin[lo]);
  }
  __syncthreads();
  local = shared_local;
  return shared_it;
}

// low[s][k] = float(double sum of x[kF .. kF+F) / F); 128 outputs per CTA,
// staged 32 samples at a time so global loads stay coalesced.
template <bool U32>
__device__ __forceinline__ void scrunch_cta(const PrepItem& it, uint64_t s, uint64_t k0, float (*tile)[33]) {
  const uint64_t factor = it.factor, low_n = it.low_n;
  const char* row = static_cast<const char*>(it.series) + s * it.stride * 4;
  double acc = 0.0;
  for (uint64_t i0 = 0; i0 < factor; i0 += 32) {
    const int cols = static_cast<int>(umin64(32, factor - i0));
    __syncthreads();
    for (int e = threadIdx.x; e < 128 * 32; e += 128) {
      const int r = e >> 5, c = e & 31;
      const uint64_t k = k0 + r;
      float v = 0.0f;
      if (k < low_n && c < cols) v = load_sample_ro(row, k * factor + i0 + c, U32);
      tile[r][c] = v;
    }
    __syncthreads();
    const uint64_t k = k0 + threadIdx.x;
    if (k < low_n)
      for (int c = 0; c < cols; ++c) acc = __dadd_rn(acc, static_cast<double>(tile[threadIdx.x][c]));
  }
  const uint64_t k = k0 + threadIdx.x;
  if (k < low_n) it.low[s * it.low_stride + k] = static_cast<float>(__ddiv_rn(acc, static_cast<double>(factor)));
}

template <bool Batched>
__global__ void __launch_bounds__(128) scrunch_kernel(const __grid_constant__ PrepTable tab) {
  __shared__ PrepItem sit;
  __shared__ uint32_t sloc;
  uint32_t local;
  const PrepItem& it = cta_item<Batched>(tab, kScrunch, sit, sloc, local);
  uint64_t s, k0;
  if (Batched) {
    const uint32_t xblocks = static_cast<uint32_t>(ceil_div(it.low_n, 128));
    s = local / xblocks;
    k0 = static_cast<uint64_t>(local % xblocks) * 128;
  } else {
    s = blockIdx.y;
    k0 = static_cast<uint64_t>(blockIdx.x) * 128;
  }
  __shared__ float tile[128][33];
  if (it.u32)
    scrunch_cta<true>(it, s, k0, tile);
  else
    scrunch_cta<false>(it, s, k0, tile);
}

// Exact running median (window w odd) of an edge-padded series, one warp per
// series.  The warp keeps the window sorted in shared memory and slides it one
// sample at a time: locate one copy of the outgoing value, count the incoming
// value's rank, and rebuild each slot from its old neighbour (shift by -1, 0
// or +1).  The upper median of an odd window is its middle element, the same
// value std::nth_element selects.
// Input: the scrunched series (factor > 1) or the series itself.
template <bool Batched>
__global__ void __launch_bounds__(32 * kMedianWarps) running_median_kernel(const __grid_constant__ PrepTable tab) {
  __shared__ PrepItem sit;
  __shared__ uint32_t sloc;
  uint32_t local;
  const PrepItem& it = cta_item<Batched>(tab, kMedian, sit, sloc, local);
  extern __shared__ float med_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t s = static_cast<uint64_t>(local) * kMedianWarps + warp;
  if (s >= it.nseries) return;
  const bool scrunched = it.factor > 1;
  const void* in = scrunched ? static_cast<const void*>(it.low) : it.series;
  const uint64_t in_stride = scrunched ? it.low_stride : it.stride;
  const uint64_t n = scrunched ? it.low_n : it.n;
  const bool u32 = !scrunched && it.u32 != 0;
  const int w = it.w;
  const int cap = ((w + 31) / 32) * 32;
  float* A = med_smem + warp * 2 * cap;
  float* B = A + cap;
  const char* row = static_cast<const char*>(in) + s * in_stride * 4;
  float* orow = it.lowmed + s * it.low_stride;
  const int half = w / 2;
  auto padded = [&](int64_t j) -> float {
    int64_t i = j - half;
    i = i < 0 ? 0 : (i >= static_cast<int64_t>(n) ? static_cast<int64_t>(n) - 1 : i);
    return load_sample_ro(row, static_cast<uint64_t>(i), u32);
  };
  // initial window, sorted by an odd-even transposition sort over cap slots
  for (int j = lane; j < cap; j += 32) A[j] = j < w ? padded(j) : INFINITY;
  __syncwarp();
  for (int round = 0; round < cap; ++round) {
    for (int j = 2 * lane + (round & 1); j + 1 < cap; j += 64) {
      const float a = A[j], b = A[j + 1];
      if (b < a) { A[j] = b; A[j + 1] = a; }
    }
    __syncwarp();
  }
  const int slots = cap / 32;
  float pre_out = 0.0f, pre_in = 0.0f;
  for (uint64_t i = 0; i < n; ++i) {
    if (lane == 0) orow[i] = A[half];
    if (i + 1 == n) break;
    // every 32 steps each lane fetches one outgoing and one incoming value
    if ((i & 31) == 0) {
      pre_out = padded(static_cast<int64_t>(i) + lane);
      pre_in = padded(static_cast<int64_t>(i) + w + lane);
    }
    const float x_out = __shfl_sync(0xffffffffu, pre_out, static_cast<int>(i & 31));
    const float x_in = __shfl_sync(0xffffffffu, pre_in, static_cast<int>(i & 31));
    // position of the first copy of x_out, and rank of x_in
    int p = cap;
    int less = 0;
    for (int t = 0; t < slots; ++t) {
      const int j = lane + 32 * t;
      const float v = A[j];
      const unsigned eq = __ballot_sync(0xffffffffu, j < w && v == x_out);
      if (p == cap && eq) p = 32 * t + __ffs(eq) - 1;
      less += __popc(__ballot_sync(0xffffffffu, j < w && v < x_in));
    }
    if (x_out < x_in) less -= 1;  // the removed element no longer counts
    const int q = less;
    for (int t = 0; t < slots; ++t) {
      const int j = lane + 32 * t;
      if (j < w) {
        float v;
        if (j < q) v = A[j < p ? j : j + 1];
        else if (j == q) v = x_in;
        else v = A[(j - 1) < p ? j - 1 : j];
        B[j] = v;
      }
    }
    __syncwarp();
    float* tmp = A;
    A = B;
    B = tmp;
  }
}

// y = x - trend, written in place as float (buffer may hold uint32 input).
template <bool Batched>
__global__ void __launch_bounds__(256) detrend_kernel(const __grid_constant__ PrepTable tab) {
  __shared__ PrepItem sit;
  __shared__ uint32_t sloc;
  uint32_t local;
  const PrepItem& it = cta_item<Batched>(tab, kDetrend, sit, sloc, local);
  uint64_t s, i;
  if (Batched) {
    const uint32_t xblocks = static_cast<uint32_t>(ceil_div(it.n, 256));
    s = local / xblocks;
    i = static_cast<uint64_t>(local % xblocks) * 256 + threadIdx.x;
  } else {
    s = blockIdx.y;
    i = static_cast<uint64_t>(blockIdx.x) * 256 + threadIdx.x;
  }
  if (i >= it.n) return;
  const bool u32 = it.u32 != 0;
  char* row = static_cast<char*>(it.series) + s * it.stride * 4;
  const float* lm = it.lowmed + s * it.low_stride;
  const float x = load_sample(row, i, u32);
  if (!u32 && !isfinite(x)) atomicOr(it.status, GF_STATUS_NONFINITE);
  float trend;
  if (it.factor == 1) {
    trend = lm[i];
  } else {
    const uint64_t factor = it.factor, low_n = it.low_n;
    const double offset = 0.5 * static_cast<double>(factor - 1);
    const double pos = __ddiv_rn(__dsub_rn(static_cast<double>(i), offset), static_cast<double>(factor));
    if (pos <= 0.0) {
      trend = lm[0];
    } else {
      const uint64_t lower = static_cast<uint64_t>(floor(pos));
      if (lower >= low_n - 1) {
        trend = lm[low_n - 1];
      } else {
        const double frac = __dsub_rn(pos, static_cast<double>(lower));
        trend = static_cast<float>(__dadd_rn(__dmul_rn(__dsub_rn(1.0, frac), static_cast<double>(lm[lower])),
                                             __dmul_rn(frac, static_cast<double>(lm[lower + 1]))));
      }
    }
  }
  reinterpret_cast<float*>(row)[i] = __fsub_rn(x, trend);
}

// Sequential FP64 sums in the reference order, one warp per series: the
// lanes stream the series into shared memory with cp.async (two chunks in
// flight) while lane 0 runs the dependent chain sum += y; sq += y * y over the
// chunk already resident, so the chain never waits on global memory.
constexpr int kStatsChunk = 1024;  // floats per chunk

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::); }

template <bool Batched>
__global__ void __launch_bounds__(32 * kStatsWarps) stats_kernel(const __grid_constant__ PrepTable tab) {
  __shared__ PrepItem sit;
  __shared__ uint32_t sloc;
  uint32_t local;
  const PrepItem& it = cta_item<Batched>(tab, kStats, sit, sloc, local);
  __shared__ __align__(16) float buf[kStatsWarps][2][kStatsChunk];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t s = static_cast<uint64_t>(local) * kStatsWarps + warp;
  if (s >= it.nseries) return;
  const uint64_t n = it.n;
  const float* row = static_cast<const float*>(it.series) + s * it.stride;
  // vector staging needs 16-byte aligned rows; others take the scalar tail path
  const uint64_t nvec = (reinterpret_cast<uintptr_t>(row) & 15) == 0 ? n / 4 : 0;
  const uint64_t nchunks = (nvec * 4 + kStatsChunk - 1) / kStatsChunk;
  auto issue = [&](uint64_t c) {
    if (c < nchunks) {
      const uint64_t v0 = c * (kStatsChunk / 4);
      for (int v = lane; v < kStatsChunk / 4; v += 32)
        if (v0 + v < nvec) cp_async16(&buf[warp][c & 1][4 * v], row + 4 * (v0 + v));
    }
    cp_async_commit();
  };
  double sum = 0.0, sq = 0.0;
  issue(0);
  for (uint64_t c = 0; c < nchunks; ++c) {
    issue(c + 1);
    cp_async_wait_1();
    __syncwarp();
    if (lane == 0) {
      // four samples per vector load, the next vector loaded and the squares
      // formed ahead of the two dependent add chains (same order as one at a
      // time; len is a multiple of 4)
      const float4* b4 = reinterpret_cast<const float4*>(buf[warp][c & 1]);
      const uint32_t nv = static_cast<uint32_t>(umin64(kStatsChunk, nvec * 4 - c * kStatsChunk) / 4);
      float4 nxt = b4[0];
      for (uint32_t v = 0; v < nv; ++v) {
        const float4 cur = nxt;
        if (v + 1 < nv) nxt = b4[v + 1];
        const double a0 = cur.x, a1 = cur.y, a2 = cur.z, a3 = cur.w;
        const double q0 = __dmul_rn(a0, a0), q1 = __dmul_rn(a1, a1), q2 = __dmul_rn(a2, a2),
                     q3 = __dmul_rn(a3, a3);
        sum = __dadd_rn(sum, a0);
        sq = __dadd_rn(sq, q0);
        sum = __dadd_rn(sum, a1);
        sq = __dadd_rn(sq, q1);
        sum = __dadd_rn(sum, a2);
        sq = __dadd_rn(sq, q2);
        sum = __dadd_rn(sum, a3);
        sq = __dadd_rn(sq, q3);
      }
    }
    __syncwarp();
  }
  cp_async_wait_0();
  if (lane != 0) return;
  for (uint64_t i = nvec * 4; i < n; ++i) {
    const double a = row[i];
    sum = __dadd_rn(sum, a);
    sq = __dadd_rn(sq, __dmul_rn(a, a));
  }
  const double count = static_cast<double>(n);
  const double mean = __ddiv_rn(sum, count);
  double var = __dsub_rn(__ddiv_rn(sq, count), __dmul_rn(mean, mean));
  if (var < 0.0 && var > -1.0e-12) var = 0.0;
  double scale = 0.0;
  if (!(var >= 0.0) || !isfinite(var)) {
    atomicOr(it.status, GF_STATUS_NONFINITE);
  } else {
    const double sd = __dsqrt_rn(var);
    if (!(sd > 0.0) || !isfinite(sd)) {
      if (it.normalise && it.reject_constant) atomicOr(it.status, GF_STATUS_CONSTANT);
    } else {
      scale = __ddiv_rn(1.0, sd);
    }
  }
  it.stats[2 * s] = mean;
  it.stats[2 * s + 1] = scale;
}

__global__ void __launch_bounds__(256) normalise_kernel(float* series, uint64_t stride, uint64_t n,
                                                        const double* __restrict__ stats) {
  const int s = blockIdx.y;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double mean = stats[2 * s], scale = stats[2 * s + 1];
  float* row = series + s * stride;
  row[i] = scale == 0.0 ? 0.0f
                        : static_cast<float>(__dmul_rn(__dsub_rn(static_cast<double>(row[i]), mean), scale));
}

struct Geometry {
  uint64_t window = 0, factor = 1, low_n = 0, low_stride = 0;
};

Geometry geometry(const gf_preprocess_desc& d) {
  check_arg(d.nsamples > 0, "running median detrend input must not be empty");
  check_arg(d.window_seconds > 0.0 && std::isfinite(d.window_seconds),
            "running median window_seconds must be finite and > 0");
  check_arg(d.tsamp > 0.0 && std::isfinite(d.tsamp), "running median tsamp must be finite and > 0");
  Geometry g;
  const double r = std::round(d.window_seconds / d.tsamp);
  check_arg(std::isfinite(r) && r < 1.8e19, "running median window_samples is too large");
  g.window = static_cast<uint64_t>(std::max(1.0, r));
  if (g.window % 2 == 0) ++g.window;
  check_arg(d.min_points > 0 && d.min_points % 2 == 1, "running median detrend min_points must be odd and > 0");
  g.factor = std::max<uint64_t>(1, static_cast<uint64_t>(static_cast<double>(g.window) /
                                                       static_cast<double>(d.min_points)));
  if (g.factor == 1) {
    check_arg(g.window < d.nsamples, "running median detrend window_samples must be < input size");
    check_arg(g.window <= kMaxMedianWindow, "running median window exceeds the CUDA limit of 2047 samples");
    g.low_n = d.nsamples;
  } else {
    g.low_n = d.nsamples / g.factor;
    check_arg(g.low_n > d.min_points,
              "running median detrend low-resolution sample count must be > min_points");
    check_arg(d.min_points <= kMaxMedianWindow, "running median min_points exceeds the CUDA limit of 2047");
  }
  g.low_stride = round_up(g.low_n, 4);
  return g;
}

}  // namespace
}  // namespace gf

using namespace gf;

extern "C" int gf_preprocess_info_get(const gf_preprocess_desc* d, gf_preprocess_info* info) {
  return guarded([&] {
    check_arg(d && info, "null argument");
    const Geometry g = geometry(*d);
    info->window_samples = g.window;
    info->scrunch_factor = g.factor;
    info->low_nsamples = g.low_n;
    info->workspace_bytes = g.factor == 1 ? g.low_stride * 4 * d->max_series
                                          : 2 * g.low_stride * 4 * d->max_series;
  });
}

namespace {

// The launch item of gf_preprocess_inplace's arguments.
PrepItem make_item(const gf_preprocess_desc& d, void* dev_series, int32_t input_is_u32, uint64_t nseries,
                   uint64_t stride, void* dev_workspace, double* dev_stats, uint32_t* dev_status) {
  check_arg(dev_series && dev_workspace && dev_stats && dev_status, "null argument");
  check_arg(nseries > 0 && nseries <= d.max_series, "nseries must be in (0, max_series]");
  check_arg(nseries < (1ull << 31), "too many series per call");
  check_arg(stride >= d.nsamples, "stride must be >= nsamples");
  const Geometry g = geometry(d);
  PrepItem it{};
  it.series = dev_series;
  it.stride = stride;
  it.n = d.nsamples;
  it.factor = g.factor;
  it.low_n = g.low_n;
  it.low_stride = g.low_stride;
  it.low = static_cast<float*>(dev_workspace);
  it.lowmed = g.factor == 1 ? it.low : it.low + g.low_stride * nseries;
  it.stats = dev_stats;
  it.status = dev_status;
  it.nseries = static_cast<uint32_t>(nseries);
  it.w = static_cast<int32_t>(g.factor == 1 ? g.window : d.min_points);
  it.u32 = input_is_u32 ? 1 : 0;
  it.normalise = d.normalise;
  it.reject_constant = d.reject_constant;
  return it;
}

size_t median_smem(int w) {
  const int cap = ((w + 31) / 32) * 32;
  return static_cast<size_t>(kMedianWarps) * 2 * cap * sizeof(float);
}

// The four stages: a batched launch over a table whose stage grids are
// ctas[stage] CTAs; a single one with (x blocks, series) grids for scrunch
// and detrend (ctas[] then holds x blocks, and the series count is the item's).
template <bool Batched>
void launch_stages(const PrepTable& tab, const uint64_t (&ctas)[kStages], size_t med_smem, cudaStream_t s) {
  for (int st = 0; st < kStages; ++st)
    check_arg(ctas[st] < (1ull << 31), "preprocessing launch too large");
  const unsigned ny = Batched ? 1u : tab.one.nseries;
  cuda_check(cudaFuncSetAttribute(running_median_kernel<Batched>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(med_smem)),
             "cudaFuncSetAttribute(median)");
  if (ctas[kScrunch]) scrunch_kernel<Batched><<<dim3(static_cast<unsigned>(ctas[kScrunch]), ny), 128, 0, s>>>(tab);
  running_median_kernel<Batched><<<static_cast<unsigned>(ctas[kMedian]), 32 * kMedianWarps, med_smem, s>>>(tab);
  cuda_check(cudaGetLastError(), "running median launch");
  detrend_kernel<Batched><<<dim3(static_cast<unsigned>(ctas[kDetrend]), ny), 256, 0, s>>>(tab);
  cuda_check(cudaGetLastError(), "detrend launch");
  stats_kernel<Batched><<<static_cast<unsigned>(ctas[kStats]), 32 * kStatsWarps, 0, s>>>(tab);
  cuda_check(cudaGetLastError(), "stats launch");
}

}  // namespace

extern "C" int gf_preprocess_inplace(const gf_preprocess_desc* d, void* dev_series, int32_t input_is_u32,
                                     uint64_t nseries, uint64_t stride, void* dev_workspace,
                                     double* dev_stats, uint32_t* dev_status, void* stream) {
  return guarded([&] {
    check_arg(d != nullptr, "null argument");
    PrepTable tab{};
    tab.one = make_item(*d, dev_series, input_is_u32, nseries, stride, dev_workspace, dev_stats, dev_status);
    check_arg(nseries < 65536, "at most 65535 series per call");
    uint64_t ctas[kStages];
    for (int st = 0; st < kStages; ++st)
      ctas[st] = (st == kScrunch || st == kDetrend) ? stage_xblocks(tab.one, st) : stage_ctas(tab.one, st);
    launch_stages<false>(tab, ctas, median_smem(tab.one.w), as_stream(stream));
  });
}

// Many gf_preprocess_inplace calls (series of different lengths and options)
// as one launch per stage.
struct gf_preprocess_batch {
  int device = 0;
  int nitems = 0;
  uint64_t ctas[kStages] = {0, 0, 0, 0};
  size_t med_smem = 0;
  DeviceBlob items_d, begin_d;
};

extern "C" int gf_preprocess_batch_create(const gf_preprocess_batch_item* items, uint64_t nitems,
                                          int32_t device_id, gf_preprocess_batch** out) {
  return guarded([&] {
    check_arg(items && out, "null argument");
    *out = nullptr;
    check_arg(nitems > 0 && nitems < (1u << 20), "batched preprocessing takes 1 to 2^20 items");
    auto B = std::make_unique<gf_preprocess_batch>();
    B->device = device_id;
    B->nitems = static_cast<int>(nitems);
    std::vector<PrepItem> its;
    std::vector<uint64_t> begin(kStages * nitems);
    for (uint64_t i = 0; i < nitems; ++i) {
      const gf_preprocess_batch_item& x = items[i];
      check_arg(x.desc != nullptr, "null argument");
      its.push_back(make_item(*x.desc, x.dev_series, x.input_is_u32, x.nseries, x.stride, x.dev_workspace,
                              x.dev_stats, x.dev_status));
      B->med_smem = std::max(B->med_smem, median_smem(its.back().w));
      for (int st = 0; st < kStages; ++st) {
        begin[st * nitems + i] = B->ctas[st];
        B->ctas[st] += stage_ctas(its.back(), st);
      }
    }
    DeviceGuard dg(device_id);
    B->items_d.upload(its.data(), its.size() * sizeof(PrepItem), device_id);
    B->begin_d.upload(begin.data(), begin.size() * sizeof(uint64_t), device_id);
    *out = B.release();
  });
}

extern "C" int gf_preprocess_batch_run(gf_preprocess_batch* B, void* stream) {
  return guarded([&] {
    check_arg(B != nullptr, "null argument");
    DeviceGuard dg(B->device);
    PrepTable tab{};
    tab.items = B->items_d.as<PrepItem>();
    tab.begin = B->begin_d.as<uint64_t>();
    tab.nitems = B->nitems;
    launch_stages<true>(tab, B->ctas, B->med_smem, as_stream(stream));
  });
}

extern "C" int gf_preprocess_batch_destroy(gf_preprocess_batch* B) {
  return guarded([&] { delete B; });
}

extern "C" int gf_normalise(float* dev_series, uint64_t nseries, uint64_t stride, uint64_t nsamples,
                            const double* dev_stats, void* stream) {
  return guarded([&] {
    check_arg(dev_series && dev_stats, "null argument");
    check_arg(nseries > 0 && nseries < 65536 && stride >= nsamples, "invalid shape");
    dim3 g(static_cast<unsigned>(ceil_div(nsamples, 256)), static_cast<unsigned>(nseries));
    normalise_kernel<<<g, 256, 0, as_stream(stream)>>>(dev_series, stride, nsamples, dev_stats);
    cuda_check(cudaGetLastError(), "normalise launch");
  });
}
