// Shared helpers for the sm_100a kernels and the C ABI glue.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "gaffa_b200.h"

namespace gf {

// Thread-local last error message for gf_last_error().
void set_error(const char* fmt, ...);
const char* last_error();

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void raise(int code, const std::string& msg) { throw Error(code, msg); }

inline void check_arg(bool ok, const char* msg) {
  if (!ok) raise(GF_EINVAL, msg);
}

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    raise(e == cudaErrorMemoryAllocation ? GF_ENOMEM : GF_ECUDA,
          std::string(what) + ": " + cudaGetErrorString(e));
  }
}

// Runs f(); converts exceptions into status codes + a message (never throws
// across the C ABI).
template <typename F>
int guarded(F&& f) {
  try {
    f();
    return GF_OK;
  } catch (const Error& e) {
    set_error("%s", e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return GF_ENOMEM;
  } catch (const std::exception& e) {
    set_error("%s", e.what());
    return GF_ERUNTIME;
  }
}

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

__host__ __device__ inline uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__host__ __device__ inline uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

__host__ __device__ inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline uint64_t round_up(uint64_t a, uint64_t b) { return ceil_div(a, b) * b; }

// Sets the current device for the scope and restores the caller's device.
struct DeviceGuard {
  int previous = -1;
  explicit DeviceGuard(int device) {
    cuda_check(cudaGetDevice(&previous), "cudaGetDevice");
    if (previous != device) cuda_check(cudaSetDevice(device), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int now = -1;
    if (cudaGetDevice(&now) == cudaSuccess && now != previous && previous >= 0)
      cudaSetDevice(previous);
  }
};

// Owned device allocation for program metadata (freed on its device).
struct DeviceBlob {
  void* ptr = nullptr;
  size_t bytes = 0;
  int device = 0;
  DeviceBlob() = default;
  DeviceBlob(const DeviceBlob&) = delete;
  DeviceBlob& operator=(const DeviceBlob&) = delete;
  DeviceBlob(DeviceBlob&& o) noexcept : ptr(o.ptr), bytes(o.bytes), device(o.device) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  DeviceBlob& operator=(DeviceBlob&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      bytes = o.bytes;
      device = o.device;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DeviceBlob() { release(); }
  void release() {
    if (ptr) {
      int prev = -1;
      cudaGetDevice(&prev);
      if (prev != device) cudaSetDevice(device);
      cudaFree(ptr);
      if (prev != device && prev >= 0) cudaSetDevice(prev);
      ptr = nullptr;
      bytes = 0;
    }
  }
  void upload(const void* host, size_t n, int dev) {
    release();
    device = dev;
    bytes = n;
    if (n == 0) return;
    cuda_check(cudaMalloc(&ptr, n), "cudaMalloc(program metadata)");
    cuda_check(cudaMemcpy(ptr, host, n, cudaMemcpyHostToDevice), "cudaMemcpy(program metadata)");
  }
  template <typename T>
  T* as() const { return static_cast<T*>(ptr); }
};

// The cold-plasma delay in samples, internal/dedispersion_delay.h:37-50:
// round-half-away-from-zero of 4148.808 * dm * (f^-2 - fref^-2) / tsamp, in
// FP64 with the reference's operation order.
int32_t delay_bins(double dm, double f, double fref, double tsamp);

// One plan task's period arithmetic inputs (for device peak expansion).
struct PeakTaskInfo {
  double effective_tsamp;
  uint64_t bins, rows;
};
struct HarmonicRatio;
struct HarmonicInput;
// The pairwise marking of flag_harmonics_cpu (harmonic.cpp:271-289) on the
// device: parent[c] = the first non-harmonic candidate before c (in ranking
// order) of which c is a harmonic, or UINT32_MAX.
void flag_harmonics_on_device(const std::vector<HarmonicInput>& candidates, const std::vector<HarmonicRatio>& ratios,
                              double observation_seconds, double band, const gf_harmonic_options& options,
                              int device, void* stream, std::vector<uint32_t>& parent);

// The task table, width trials and device of a single-plan FFA program.
void ffa_program_peak_tables(const gf_ffa_program* program, std::vector<PeakTaskInfo>& tasks,
                             std::vector<uint64_t>& widths, int& device);

}  // namespace gf
