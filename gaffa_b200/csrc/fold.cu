// Folding of a dedispersed time series into phase bins on sm_100a.
//
// Reference: fold_time_series_cpu, src/gaffa/folding.cpp:452-502 with
// accumulate_interval :124-158.  Sample i covers the scaled phase interval
// [(start+i)*step, (start+i+1)*step), step = tsamp / period * nbin; each bin
// it overlaps receives value * overlap and overlap of exposure (FP64);
// profile = sums / exposure.  The reference has no CUDA path for this.
//
// Each thread folds a contiguous run of samples, carrying the current bin's
// partial sums in registers and flushing them to shared-memory FP64
// accumulators when the bin changes; CTA partials are reduced in a fixed
// order by a second kernel.  Like the reference's per-thread OpenMP
// histograms, the FP64 summation order differs from a serial loop, so
// results agree to FP64 rounding (the float profile to within an ulp).
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

namespace gf {
namespace {

constexpr int kThreads = 256;
constexpr int kSamplesPerThread = 64;
constexpr uint64_t kMaxBins = 8192;

template <bool U32>
__global__ void __launch_bounds__(kThreads) fold_partial_kernel(const void* __restrict__ in, uint64_t n,
                                                                double step, uint64_t start, uint64_t nbin,
                                                                double* __restrict__ partial,
                                                                uint32_t* status) {
  extern __shared__ double acc[];  // [2][nbin]
  double* sums = acc;
  double* expo = acc + nbin;
  for (uint64_t b = threadIdx.x; b < 2 * nbin; b += kThreads) acc[b] = 0.0;
  __syncthreads();
  const uint64_t i0 = (static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x) * kSamplesPerThread;
  const int64_t nb = static_cast<int64_t>(nbin);
  int64_t cur = -1;
  double cs = 0.0, ce = 0.0;
  for (uint64_t i = i0; i < n && i < i0 + kSamplesPerThread; ++i) {
    const double v = U32 ? static_cast<double>(static_cast<const uint32_t*>(in)[i])
                         : static_cast<double>(static_cast<const float*>(in)[i]);
    if (!U32 && !isfinite(v)) atomicOr(status, GF_STATUS_NONFINITE);
    const double lo = __dmul_rn(static_cast<double>(start + i), step);
    const double hi = __dadd_rn(lo, step);
    const int64_t first = static_cast<int64_t>(floor(lo));
    const int64_t last = static_cast<int64_t>(ceil(hi) - 1.0);
    for (int64_t bin = first; bin <= last; ++bin) {
      const double bl = static_cast<double>(bin), br = bl + 1.0;
      const double w = __dsub_rn(hi < br ? hi : br, lo > bl ? lo : bl);
      if (!(w > 0.0)) continue;
      int64_t m = bin % nb;
      if (m < 0) m += nb;
      if (m != cur) {
        if (cur >= 0) {
          atomicAdd(sums + cur, cs);
          atomicAdd(expo + cur, ce);
        }
        cur = m;
        cs = 0.0;
        ce = 0.0;
      }
      cs = __dadd_rn(cs, __dmul_rn(v, w));
      ce = __dadd_rn(ce, w);
    }
  }
  if (cur >= 0) {
    atomicAdd(sums + cur, cs);
    atomicAdd(expo + cur, ce);
  }
  __syncthreads();
  double* out = partial + static_cast<uint64_t>(blockIdx.x) * 2 * nbin;
  for (uint64_t b = threadIdx.x; b < 2 * nbin; b += kThreads) out[b] = acc[b];
}

__global__ void __launch_bounds__(kThreads) fold_reduce_kernel(const double* __restrict__ partial, int nblocks,
                                                               uint64_t nbin, float* __restrict__ profile,
                                                               double* __restrict__ exposure) {
  const uint64_t b = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (b >= nbin) return;
  double s = 0.0, e = 0.0;
  for (int k = 0; k < nblocks; ++k) {
    s = __dadd_rn(s, partial[static_cast<uint64_t>(k) * 2 * nbin + b]);
    e = __dadd_rn(e, partial[static_cast<uint64_t>(k) * 2 * nbin + nbin + b]);
  }
  exposure[b] = e;
  profile[b] = e > 0.0 ? static_cast<float>(__ddiv_rn(s, e)) : 0.0f;
}

uint64_t fold_blocks(uint64_t n) { return ceil_div(n, static_cast<uint64_t>(kThreads) * kSamplesPerThread); }

}  // namespace
}  // namespace gf

using namespace gf;

extern "C" uint64_t gf_fold_workspace_bytes(uint64_t n, uint64_t nbin) {
  return fold_blocks(n) * 2 * nbin * sizeof(double) + 16;
}

extern "C" int gf_fold_time_series(const void* dev_input, int32_t input_is_u32, uint64_t n, double period,
                                   double tsamp, uint64_t nbin, uint64_t start_sample, float* dev_profile,
                                   double* dev_exposure, void* dev_workspace, void* stream) {
  return guarded([&] {
    // folding.cpp:44-73 validation
    check_arg(std::isfinite(period) && period > 0.0, "fold period must be finite and positive");
    check_arg(std::isfinite(tsamp) && tsamp > 0.0, "fold tsamp must be finite and positive");
    check_arg(nbin > 0, "fold nbin must be positive");
    check_arg(nbin <= kMaxBins, "CUDA fold supports nbin <= 8192");
    check_arg(n > 0, "fold input must not be empty");
    check_arg(dev_input && dev_profile && dev_exposure && dev_workspace, "null argument");
    const double step = tsamp / period * static_cast<double>(nbin);
    const double hi = static_cast<double>(start_sample + n - 1) * step + step;
    check_arg(std::isfinite(hi) && std::ceil(hi) < 9.2e18, "fold phase bin index exceeds int64 range");
    auto s = as_stream(stream);
    const uint64_t blocks = fold_blocks(n);
    check_arg(blocks < (1ull << 31), "fold input too long");
    double* partial = static_cast<double*>(dev_workspace);
    uint32_t* status = reinterpret_cast<uint32_t*>(static_cast<char*>(dev_workspace) + blocks * 2 * nbin * 8);
    cuda_check(cudaMemsetAsync(status, 0, 4, s), "cudaMemsetAsync(fold status)");
    const size_t smem = 2 * nbin * sizeof(double);
    if (input_is_u32) {
      cuda_check(cudaFuncSetAttribute(fold_partial_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)), "cudaFuncSetAttribute(fold)");
      fold_partial_kernel<true><<<static_cast<unsigned>(blocks), kThreads, smem, s>>>(
          dev_input, n, step, start_sample, nbin, partial, status);
    } else {
      cuda_check(cudaFuncSetAttribute(fold_partial_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)), "cudaFuncSetAttribute(fold)");
      fold_partial_kernel<false><<<static_cast<unsigned>(blocks), kThreads, smem, s>>>(
          dev_input, n, step, start_sample, nbin, partial, status);
    }
    fold_reduce_kernel<<<static_cast<unsigned>(ceil_div(nbin, kThreads)), kThreads, 0, s>>>(
        partial, static_cast<int>(blocks), nbin, dev_profile, dev_exposure);
    cuda_check(cudaGetLastError(), "fold launch");
  });
}

// ---------------------------------------------------------------------------
// Fold without any device allocation.
//
// Some callers cannot allocate device memory when they fold: a process whose
// device memory has all been handed to another allocator's pool, or a
// latency-critical loop where cudaMalloc's implicit device synchronisation is
// not acceptable.  gf_fold_time_series_noalloc serves them with a fixed
// scratch area compiled into this library: a file-scope device array that
// every GPU which loads the library holds until the process exits.  Its size
// caps the work: fold_blocks(n) * 2 * nbin doubles must fit in
// kNoAllocScratchBytes (4 MiB: e.g. nbin = 64 up to ~67 million samples).
// All calls share the array and it keeps the last call's contents; the
// partial sums are fully rewritten by every call, so nothing needs clearing,
// but calls that overlap on the GPU (different streams, or different host
// threads) race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------

namespace {

constexpr uint64_t kNoAllocScratchBytes = 4ull << 20;
static __device__ __align__(256) unsigned char g_fold_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_fold_scratch_mutex;
void* g_fold_scratch_address[kMaxDevices] = {};

// Device address of g_fold_scratch on the current device, resolved once per
// device.  In host code the array's name is only a host-side stand-in, so
// the kernels must receive this address, never &g_fold_scratch.  The address
// is kept for the life of the process; a cudaDeviceReset reloads the module
// and makes it stale, so the entry point is not to be used after a reset.
void* fold_scratch_address() {
  int device = -1;
  cuda_check(cudaGetDevice(&device), "cudaGetDevice");
  check_arg(device >= 0 && device < kMaxDevices, "device ordinal out of range for the fixed fold scratch");
  std::lock_guard<std::mutex> lock(g_fold_scratch_mutex);
  if (g_fold_scratch_address[device] == nullptr) {
    void* ptr = nullptr;
    cuda_check(cudaGetSymbolAddress(&ptr, g_fold_scratch), "cudaGetSymbolAddress(fold scratch)");
    g_fold_scratch_address[device] = ptr;
  }
  return g_fold_scratch_address[device];
}

}  // namespace

extern "C" uint64_t gf_fold_noalloc_max_bytes(void) { return kNoAllocScratchBytes; }

extern "C" int gf_fold_time_series_noalloc(const void* dev_input, int32_t input_is_u32, uint64_t n, double period,
                                           double tsamp, uint64_t nbin, uint64_t start_sample, float* dev_profile,
                                           double* dev_exposure, uint32_t* dev_status, void* stream) {
  return guarded([&] {
    check_arg(n > 0, "fold input must not be empty");
    check_arg(nbin > 0, "fold nbin must be positive");
    check_arg(nbin <= kMaxBins, "CUDA fold supports nbin <= 8192");
    const uint64_t nblocks = fold_blocks(n);
    check_arg(nblocks < (1ull << 31), "fold input too long");
    // each block keeps 2 * nbin doubles; compared by division so nothing wraps
    if (nblocks > kNoAllocScratchBytes / (2 * nbin * sizeof(double))) {
      raise(GF_EINVAL, "fold without allocation: " + std::to_string(n) + " samples x " + std::to_string(nbin) +
                           " bins need " + std::to_string(nblocks) + " x " + std::to_string(2 * nbin * 8) +
                           " bytes of scratch, above the fixed " + std::to_string(kNoAllocScratchBytes) +
                           " bytes; use gf_fold_time_series");
    }
    // folding.cpp:44-73 validation, as gf_fold_time_series
    check_arg(std::isfinite(period) && period > 0.0, "fold period must be finite and positive");
    check_arg(std::isfinite(tsamp) && tsamp > 0.0, "fold tsamp must be finite and positive");
    check_arg(dev_input && dev_profile && dev_exposure && dev_status, "null argument");
    const double step = tsamp / period * static_cast<double>(nbin);
    const double hi = static_cast<double>(start_sample + n - 1) * step + step;
    check_arg(std::isfinite(hi) && std::ceil(hi) < 9.2e18, "fold phase bin index exceeds int64 range");
    auto s = as_stream(stream);
    const uint64_t blocks = nblocks;
    double* partial = static_cast<double*>(fold_scratch_address());
    // the status word must start at zero; the partial sums are overwritten
    cuda_check(cudaMemsetAsync(dev_status, 0, 4, s), "cudaMemsetAsync(fold status)");
    const size_t smem = 2 * nbin * sizeof(double);
    if (input_is_u32) {
      cuda_check(cudaFuncSetAttribute(fold_partial_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)), "cudaFuncSetAttribute(fold)");
      fold_partial_kernel<true><<<static_cast<unsigned>(blocks), kThreads, smem, s>>>(
          dev_input, n, step, start_sample, nbin, partial, dev_status);
    } else {
      cuda_check(cudaFuncSetAttribute(fold_partial_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)), "cudaFuncSetAttribute(fold)");
      fold_partial_kernel<false><<<static_cast<unsigned>(blocks), kThreads, smem, s>>>(
          dev_input, n, step, start_sample, nbin, partial, dev_status);
    }
    fold_reduce_kernel<<<static_cast<unsigned>(ceil_div(nbin, kThreads)), kThreads, 0, s>>>(
        partial, static_cast<int>(blocks), nbin, dev_profile, dev_exposure);
    cuda_check(cudaGetLastError(), "fold launch");
  });
}

// ---------------------------------------------------------------------------
// Spectrum folding: subint x channel x phase cubes (folding.cpp:237-438)
// ---------------------------------------------------------------------------
//
// fold_spectrum_cpu: sample t of subint s = t / subint_samples covers the
// scaled phase interval [(start+t)*step, (start+t+1)*step); every output
// channel's value (the mean of `factor` adjacent input channels) is added
// with the overlap weight to cube[s][c][phase], the weight to
// exposure[s][phase]; the cube is sums / exposure.  One CTA per (subint, 32
// output channels): a lane per channel, warps over the subint's samples,
// FP64 sums in shared memory.

namespace gf {
namespace {

constexpr uint64_t kSpecMaxBins = 256;

template <typename T>
__device__ __forceinline__ double spec_value(const T* row, uint64_t c, uint64_t factor) {
  double v = 0.0;
  for (uint64_t k = 0; k < factor; ++k) v += static_cast<double>(row[c * factor + k]);
  return factor == 1 ? v : v / static_cast<double>(factor);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) fold_spectrum_kernel(const T* __restrict__ in, uint64_t nsamples,
                                                                 uint64_t nchans, uint64_t nout, uint64_t factor,
                                                                 double step, uint64_t start, uint64_t nbin,
                                                                 uint64_t subint_samples, float* __restrict__ cube,
                                                                 double* __restrict__ exposure, uint32_t* status) {
  extern __shared__ double sacc[];  // sums [nbin][32], exposure [nbin]
  double* sums = sacc;
  double* expo = sacc + nbin * 32;
  const uint64_t s = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t c = static_cast<uint64_t>(blockIdx.y) * 32 + lane;
  const bool valid = c < nout;
  for (uint64_t i = threadIdx.x; i < nbin * 33; i += kThreads) sacc[i] = 0.0;
  __syncthreads();
  const uint64_t t0 = s * subint_samples;
  const uint64_t t1 = umin64(nsamples, t0 + subint_samples);
  const int64_t nb = static_cast<int64_t>(nbin);
  for (uint64_t t = t0 + warp; t < t1; t += kThreads / 32) {
    const T* row = in + t * nchans;
    double v = 0.0;
    if (valid) {
      v = spec_value(row, c, factor);
      if (!isfinite(v)) atomicOr(status, GF_STATUS_NONFINITE);
    }
    const double lo = __dmul_rn(static_cast<double>(start + t), step);
    const double hi = __dadd_rn(lo, step);
    const int64_t first = static_cast<int64_t>(floor(lo));
    const int64_t last = static_cast<int64_t>(ceil(hi) - 1.0);
    for (int64_t bin = first; bin <= last; ++bin) {
      const double bl = static_cast<double>(bin), br = bl + 1.0;
      const double w = __dsub_rn(hi < br ? hi : br, lo > bl ? lo : bl);
      if (!(w > 0.0)) continue;
      int64_t m = bin % nb;
      if (m < 0) m += nb;
      if (valid) atomicAdd(sums + m * 32 + lane, __dmul_rn(v, w));
      if (lane == 0) atomicAdd(expo + m, w);
    }
  }
  __syncthreads();
  if (valid) {
    float* out = cube + (s * nout + c) * nbin;
    for (uint64_t p = 0; p < nbin; ++p) {
      const double e = expo[p];
      out[p] = e > 0.0 ? static_cast<float>(sums[p * 32 + lane] / e) : 0.0f;
    }
  }
  if (blockIdx.y == 0)
    for (uint64_t p = threadIdx.x; p < nbin; p += kThreads) exposure[s * nbin + p] = expo[p];
}

// project_folded_cube (folding.cpp:237-296), the reference's summation order:
// time_phase[s][p] = mean over channels (FP64, channels ascending),
// freq_phase[c][p] and profile[p] exposure-weighted means (subints ascending,
// then channels).
__global__ void project_time_kernel(const float* __restrict__ cube, const double* __restrict__ exposure,
                                    uint64_t nsubint, uint64_t nchans, uint64_t nbin, float* __restrict__ time_phase) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= nsubint * nbin) return;
  const uint64_t s = i / nbin, p = i % nbin;
  if (!(exposure[i] > 0.0)) {
    time_phase[i] = 0.0f;
    return;
  }
  double acc = 0.0;
  for (uint64_t c = 0; c < nchans; ++c) acc += static_cast<double>(cube[(s * nchans + c) * nbin + p]);
  time_phase[i] = static_cast<float>(acc / static_cast<double>(nchans));
}

__global__ void project_freq_kernel(const float* __restrict__ cube, const double* __restrict__ exposure,
                                    uint64_t nsubint, uint64_t nchans, uint64_t nbin, float* __restrict__ freq_phase) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= nchans * nbin) return;
  const uint64_t c = i / nbin, p = i % nbin;
  double sum = 0.0, ex = 0.0;
  for (uint64_t s = 0; s < nsubint; ++s) {
    const double e = exposure[s * nbin + p];
    if (!(e > 0.0)) continue;
    sum += static_cast<double>(cube[(s * nchans + c) * nbin + p]) * e;
    ex += e;
  }
  freq_phase[i] = ex > 0.0 ? static_cast<float>(sum / ex) : 0.0f;
}

__global__ void project_profile_kernel(const float* __restrict__ cube, const double* __restrict__ exposure,
                                       uint64_t nsubint, uint64_t nchans, uint64_t nbin, float* __restrict__ profile) {
  const uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (p >= nbin) return;
  double sum = 0.0, ex = 0.0;
  for (uint64_t s = 0; s < nsubint; ++s) {
    const double e = exposure[s * nbin + p];
    if (!(e > 0.0)) continue;
    for (uint64_t c = 0; c < nchans; ++c) {
      sum += static_cast<double>(cube[(s * nchans + c) * nbin + p]) * e;
      ex += e;
    }
  }
  profile[p] = ex > 0.0 ? static_cast<float>(sum / ex) : 0.0f;
}

}  // namespace
}  // namespace gf

extern "C" int gf_fold_spectrum(const void* dev_in, int32_t elem_bytes, uint64_t nsamples, uint64_t nchans,
                                double period, double tsamp, uint64_t nbin, uint64_t subint_samples,
                                uint64_t start_sample, uint64_t output_channels, float* dev_cube,
                                double* dev_exposure, uint32_t* dev_status, void* stream) {
  return guarded([&] {
    check_arg(dev_in && dev_cube && dev_exposure && dev_status, "null argument");
    check_arg(elem_bytes == 1 || elem_bytes == 2 || elem_bytes == 4, "elem_bytes must be 1, 2 or 4");
    // folding.cpp:44-104 validate_fold_shape / validate_spectrum_input
    check_arg(std::isfinite(period) && period > 0.0, "fold period must be finite and positive");
    check_arg(std::isfinite(tsamp) && tsamp > 0.0, "fold tsamp must be finite and positive");
    check_arg(nbin > 0, "fold nbin must be positive");
    check_arg(nbin <= kSpecMaxBins, "fold spectrum CUDA path supports nbin <= 256");
    check_arg(nsamples > 0 && nchans > 0, "fold spectrum shape must be non-empty");
    check_arg(subint_samples > 0, "fold subint_samples must be positive");
    check_arg(output_channels <= nchans, "fold output_channels must be <= input channel count");
    check_arg(output_channels == 0 || nchans % output_channels == 0,
              "fold input channel count must be divisible by output_channels");
    const uint64_t nout = output_channels == 0 ? nchans : output_channels;
    const uint64_t factor = nchans / nout;
    const double step = tsamp / period * static_cast<double>(nbin);
    const double hi = static_cast<double>(start_sample + nsamples - 1) * step + step;
    check_arg(std::isfinite(hi), "fold phase interval is invalid");
    const uint64_t nsubint = ceil_div(nsamples, subint_samples);
    check_arg(nsubint < (1ull << 31) && ceil_div(nout, 32) < 65536, "fold spectrum too large");
    auto s = as_stream(stream);
    cuda_check(cudaMemsetAsync(dev_status, 0, sizeof(uint32_t), s), "cudaMemsetAsync(status)");
    const size_t smem = nbin * 33 * sizeof(double);
    dim3 grid(static_cast<unsigned>(nsubint), static_cast<unsigned>(ceil_div(nout, 32)));
    auto launch = [&](auto kernel, const auto* in) {
      cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                 "cudaFuncSetAttribute(fold_spectrum)");
      kernel<<<grid, kThreads, smem, s>>>(in, nsamples, nchans, nout, factor, step, start_sample, nbin,
                                          subint_samples, dev_cube, dev_exposure, dev_status);
    };
    if (elem_bytes == 1)
      launch(fold_spectrum_kernel<uint8_t>, static_cast<const uint8_t*>(dev_in));
    else if (elem_bytes == 2)
      launch(fold_spectrum_kernel<uint16_t>, static_cast<const uint16_t*>(dev_in));
    else
      launch(fold_spectrum_kernel<float>, static_cast<const float*>(dev_in));
    cuda_check(cudaGetLastError(), "fold_spectrum_kernel launch");
  });
}

extern "C" int gf_project_folded_cube(const float* dev_cube, const double* dev_exposure, uint64_t nsubint,
                                      uint64_t nchans, uint64_t nbin, float* dev_profile, float* dev_freq_phase,
                                      float* dev_time_phase, void* stream) {
  return guarded([&] {
    check_arg(dev_cube && dev_exposure && dev_profile && dev_freq_phase && dev_time_phase, "null argument");
    check_arg(nsubint > 0 && nchans > 0 && nbin > 0, "folded cube must be non-empty");
    auto s = as_stream(stream);
    project_time_kernel<<<static_cast<unsigned>(ceil_div(nsubint * nbin, 256)), 256, 0, s>>>(
        dev_cube, dev_exposure, nsubint, nchans, nbin, dev_time_phase);
    project_freq_kernel<<<static_cast<unsigned>(ceil_div(nchans * nbin, 256)), 256, 0, s>>>(
        dev_cube, dev_exposure, nsubint, nchans, nbin, dev_freq_phase);
    project_profile_kernel<<<static_cast<unsigned>(ceil_div(nbin, 64)), 64, 0, s>>>(dev_cube, dev_exposure, nsubint,
                                                                                     nchans, nbin, dev_profile);
    cuda_check(cudaGetLastError(), "project kernels launch");
  });
}
