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

namespace gf {
namespace {

constexpr int kMaxMedianWindow = 2047;

template <bool U32>
__device__ __forceinline__ float load_sample(const void* base, uint64_t i) {
  if (U32) return static_cast<float>(static_cast<const uint32_t*>(base)[i]);
  return static_cast<const float*>(base)[i];
}

// low[s][k] = float(double sum of x[kF .. kF+F) / F); 128 outputs per CTA,
// staged 32 samples at a time so global loads stay coalesced.
template <bool U32>
__global__ void __launch_bounds__(128) scrunch_kernel(const void* __restrict__ series, uint64_t stride,
                                                      uint64_t factor, uint64_t low_n,
                                                      float* __restrict__ low, uint64_t low_stride) {
  __shared__ float tile[128][33];
  const int s = blockIdx.y;
  const uint64_t k0 = static_cast<uint64_t>(blockIdx.x) * 128;
  const char* row = static_cast<const char*>(series) + s * stride * 4;
  double acc = 0.0;
  for (uint64_t i0 = 0; i0 < factor; i0 += 32) {
    const int cols = static_cast<int>(umin64(32, factor - i0));
    __syncthreads();
    for (int e = threadIdx.x; e < 128 * 32; e += 128) {
      const int r = e >> 5, c = e & 31;
      const uint64_t k = k0 + r;
      float v = 0.0f;
      if (k < low_n && c < cols) v = load_sample<U32>(row, k * factor + i0 + c);
      tile[r][c] = v;
    }
    __syncthreads();
    const uint64_t k = k0 + threadIdx.x;
    if (k < low_n)
      for (int c = 0; c < cols; ++c) acc = __dadd_rn(acc, static_cast<double>(tile[threadIdx.x][c]));
  }
  const uint64_t k = k0 + threadIdx.x;
  if (k < low_n) low[s * low_stride + k] = static_cast<float>(__ddiv_rn(acc, static_cast<double>(factor)));
}

// Exact running median (window w odd) of an edge-padded series, one warp per
// series.  The warp keeps the window sorted in shared memory and slides it one
// sample at a time: locate one copy of the outgoing value, count the incoming
// value's rank, and rebuild each slot from its old neighbour (shift by -1, 0
// or +1).  The upper median of an odd window is its middle element, the same
// value std::nth_element selects.
template <bool U32>
__global__ void __launch_bounds__(128) running_median_kernel(const void* __restrict__ in, uint64_t in_stride,
                                                             uint64_t n, int w, float* __restrict__ out,
                                                             uint64_t out_stride, int nseries) {
  extern __shared__ float med_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * (blockDim.x >> 5) + warp;
  if (s >= nseries) return;
  const int cap = ((w + 31) / 32) * 32;
  float* A = med_smem + warp * 2 * cap;
  float* B = A + cap;
  const char* row = static_cast<const char*>(in) + static_cast<uint64_t>(s) * in_stride * 4;
  float* orow = out + static_cast<uint64_t>(s) * out_stride;
  const int half = w / 2;
  auto padded = [&](int64_t j) -> float {
    int64_t i = j - half;
    i = i < 0 ? 0 : (i >= static_cast<int64_t>(n) ? static_cast<int64_t>(n) - 1 : i);
    return load_sample<U32>(row, static_cast<uint64_t>(i));
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
template <bool U32, bool Scrunched>
__global__ void __launch_bounds__(256) detrend_kernel(void* series, uint64_t stride, uint64_t n,
                                                      const float* __restrict__ lowmed, uint64_t low_stride,
                                                      uint64_t low_n, uint64_t factor, uint32_t* status) {
  const int s = blockIdx.y;
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  char* row = static_cast<char*>(series) + s * stride * 4;
  const float* lm = lowmed + s * low_stride;
  const float x = load_sample<U32>(row, i);
  if (!U32 && !isfinite(x)) atomicOr(status, GF_STATUS_NONFINITE);
  float trend;
  if (!Scrunched) {
    trend = lm[i];
  } else {
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
constexpr int kStatsWarps = 4;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::); }

__global__ void __launch_bounds__(32 * kStatsWarps) stats_kernel(const float* __restrict__ series, uint64_t stride,
                                                                 uint64_t n, int nseries, int normalise,
                                                                 int reject_constant, double* __restrict__ stats,
                                                                 uint32_t* status) {
  __shared__ __align__(16) float buf[kStatsWarps][2][kStatsChunk];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = blockIdx.x * kStatsWarps + warp;
  if (s >= nseries) return;
  const float* row = series + static_cast<uint64_t>(s) * stride;
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
      const float* b = buf[warp][c & 1];
      const uint64_t len = umin64(kStatsChunk, nvec * 4 - c * kStatsChunk);
      for (uint64_t i = 0; i < len; ++i) {
        const double a = b[i];
        sum = __dadd_rn(sum, a);
        sq = __dadd_rn(sq, __dmul_rn(a, a));
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
    atomicOr(status, GF_STATUS_NONFINITE);
  } else {
    const double sd = __dsqrt_rn(var);
    if (!(sd > 0.0) || !isfinite(sd)) {
      if (normalise && reject_constant) atomicOr(status, GF_STATUS_CONSTANT);
    } else {
      scale = __ddiv_rn(1.0, sd);
    }
  }
  stats[2 * s] = mean;
  stats[2 * s + 1] = scale;
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

extern "C" int gf_preprocess_inplace(const gf_preprocess_desc* d, void* dev_series, int32_t input_is_u32,
                                     uint64_t nseries, uint64_t stride, void* dev_workspace,
                                     double* dev_stats, uint32_t* dev_status, void* stream) {
  return guarded([&] {
    check_arg(d && dev_series && dev_workspace && dev_stats && dev_status, "null argument");
    check_arg(nseries > 0 && nseries <= d->max_series, "nseries must be in (0, max_series]");
    check_arg(nseries < 65536, "at most 65535 series per call");
    check_arg(stride >= d->nsamples, "stride must be >= nsamples");
    const Geometry g = geometry(*d);
    auto s = as_stream(stream);
    const uint64_t n = d->nsamples;
    float* low = static_cast<float*>(dev_workspace);
    float* lowmed = g.factor == 1 ? low : low + g.low_stride * nseries;
    const int w = static_cast<int>(g.factor == 1 ? g.window : d->min_points);
    const int cap = ((w + 31) / 32) * 32;
    const int warps = 4;
    const size_t med_smem = static_cast<size_t>(warps) * 2 * cap * sizeof(float);
    const unsigned med_grid = static_cast<unsigned>(ceil_div(nseries, warps));
    const unsigned rows = static_cast<unsigned>(nseries);
    cuda_check(cudaFuncSetAttribute(running_median_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(med_smem)), "cudaFuncSetAttribute(median)");
    cuda_check(cudaFuncSetAttribute(running_median_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(med_smem)), "cudaFuncSetAttribute(median)");
    if (g.factor > 1) {
      dim3 sg(static_cast<unsigned>(ceil_div(g.low_n, 128)), rows);
      if (input_is_u32)
        scrunch_kernel<true><<<sg, 128, 0, s>>>(dev_series, stride, g.factor, g.low_n, low, g.low_stride);
      else
        scrunch_kernel<false><<<sg, 128, 0, s>>>(dev_series, stride, g.factor, g.low_n, low, g.low_stride);
      running_median_kernel<false><<<med_grid, warps * 32, med_smem, s>>>(low, g.low_stride, g.low_n, w, lowmed,
                                                                          g.low_stride, static_cast<int>(nseries));
    } else {
      if (input_is_u32)
        running_median_kernel<true><<<med_grid, warps * 32, med_smem, s>>>(dev_series, stride, n, w, lowmed,
                                                                           g.low_stride, static_cast<int>(nseries));
      else
        running_median_kernel<false><<<med_grid, warps * 32, med_smem, s>>>(dev_series, stride, n, w, lowmed,
                                                                            g.low_stride, static_cast<int>(nseries));
    }
    cuda_check(cudaGetLastError(), "running median launch");
    dim3 dg(static_cast<unsigned>(ceil_div(n, 256)), rows);
    if (input_is_u32) {
      if (g.factor > 1)
        detrend_kernel<true, true><<<dg, 256, 0, s>>>(dev_series, stride, n, lowmed, g.low_stride, g.low_n, g.factor, dev_status);
      else
        detrend_kernel<true, false><<<dg, 256, 0, s>>>(dev_series, stride, n, lowmed, g.low_stride, g.low_n, g.factor, dev_status);
    } else {
      if (g.factor > 1)
        detrend_kernel<false, true><<<dg, 256, 0, s>>>(dev_series, stride, n, lowmed, g.low_stride, g.low_n, g.factor, dev_status);
      else
        detrend_kernel<false, false><<<dg, 256, 0, s>>>(dev_series, stride, n, lowmed, g.low_stride, g.low_n, g.factor, dev_status);
    }
    cuda_check(cudaGetLastError(), "detrend launch");
    stats_kernel<<<static_cast<unsigned>(ceil_div(nseries, kStatsWarps)), 32 * kStatsWarps, 0, s>>>(
        static_cast<const float*>(dev_series), stride, n, static_cast<int>(nseries), d->normalise,
        d->reject_constant, dev_stats, dev_status);
    cuda_check(cudaGetLastError(), "stats launch");
  });
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
