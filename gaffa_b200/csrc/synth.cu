// Seeded synthetic filterbanks on the GPU: the generator of
// gaffa_b200/synth.py (no reference counterpart).  Noise is an Irwin-Hall(12)
// deviate from a splitmix64 stream keyed by (seed, time, channel), so it is
// bit-identical to the numpy implementation; injected pulses and RFI are
// evaluated in FP64 and rounded to 1/4096 count.
#include "common.cuh"

#include <cmath>
#include <cstring>
#include <algorithm>
#include <vector>

namespace gf {
namespace {

struct SynthPulsarDev {
  double period, dm, sigma, amplitude, phase;
};

struct SynthParams {
  uint64_t nchans, seed;
  double tsamp, fref;
  const double* freq;
  const SynthPulsarDev* pulsars;
  int npulsars;
  int nbits;
  const uint8_t* nb_mask;  // may be null
  double nb_hz, nb_amp;
  int64_t impulse_period;  // 0 = none
  double impulse_amp;
  uint64_t t_begin;
  uint64_t row_bytes;
};

__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ int64_t noise_sum(uint64_t seed, uint64_t idx) {
  const uint64_t base = ((seed & 0xFFFFFull) << 44) ^ (idx * 3ull);
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const uint64_t h = splitmix(base + k);
    s += static_cast<int64_t>(h & 0xFFFFull) + static_cast<int64_t>((h >> 16) & 0xFFFFull) +
         static_cast<int64_t>((h >> 32) & 0xFFFFull) + static_cast<int64_t>(h >> 48);
  }
  return s;
}

__device__ __forceinline__ int64_t signal_units(const SynthParams& p, uint64_t t, uint64_t c) {
  const double tt = static_cast<double>(t) * p.tsamp;
  const double f = p.freq[c];
  double total = 0.0;
  for (int k = 0; k < p.npulsars; ++k) {
    const SynthPulsarDev ps = p.pulsars[k];
    const double delay = 4148.808 * ps.dm * (1.0 / (f * f) - 1.0 / (p.fref * p.fref));
    double ph = (tt - delay) / ps.period - ps.phase;
    ph = ph - floor(ph + 0.5);
    const double x = ph / ps.sigma;
    if (fabs(x) < 12.0) total = __dadd_rn(total, __dmul_rn(ps.amplitude, exp(__dmul_rn(-0.5, __dmul_rn(x, x)))));
  }
  if (p.nb_mask && p.nb_mask[c])
    total = __dadd_rn(total, __dmul_rn(p.nb_amp, sin(__dmul_rn(__dmul_rn(2.0 * 3.141592653589793, p.nb_hz), tt))));
  if (p.impulse_period > 0 && static_cast<int64_t>(t) % p.impulse_period == p.impulse_period / 2)
    total = __dadd_rn(total, p.impulse_amp);
  return static_cast<int64_t>(rint(total * 4096.0));
}

__global__ void __launch_bounds__(256) synth_kernel(SynthParams p, uint64_t nrows, uint8_t* out) {
  const uint64_t byte = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t r = blockIdx.y + static_cast<uint64_t>(blockIdx.z) * 65535ull;
  if (byte >= p.row_bytes || r >= nrows) return;
  const uint64_t t = p.t_begin + r;
  if (p.nbits == 8) {
    const uint64_t c = byte;
    const int64_t s = noise_sum(p.seed, t * p.nchans + c);
    const int64_t sig = p.npulsars || p.nb_mask || p.impulse_period ? signal_units(p, t, c) : 0;
    int64_t v = (32 * 4096 + s + sig + 2048) >> 12;
    v = v < 0 ? 0 : (v > 255 ? 255 : v);
    out[r * p.row_bytes + byte] = static_cast<uint8_t>(v);
  } else {
    uint32_t packed = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint64_t c = 4 * byte + j;
      const int64_t s = noise_sum(p.seed, t * p.nchans + c);
      const int64_t sig = p.npulsars || p.nb_mask || p.impulse_period ? signal_units(p, t, c) : 0;
      const int64_t zu = (s >> 4) - 24576 + (sig >> 4);
      const uint32_t lvl = (zu >= -2763) + (zu >= 0) + (zu >= 2763);
      packed |= lvl << (2 * j);
    }
    out[r * p.row_bytes + byte] = static_cast<uint8_t>(packed);
  }
}

}  // namespace
}  // namespace gf

using namespace gf;

extern "C" int gf_synth_generate(const gf_synth_desc* d, uint64_t t_begin, uint64_t t_end, uint8_t* dev_out,
                                 void* stream) {
  return guarded([&] {
    check_arg(d && dev_out, "null argument");
    check_arg(d->nbits == 8 || d->nbits == 2, "nbits must be 8 or 2");
    check_arg(d->nbits == 8 || d->nchans % 4 == 0, "2-bit output requires nchans % 4 == 0");
    check_arg(t_begin <= t_end && t_end <= d->nsamples, "time range out of bounds");
    check_arg(d->nchans > 0 && d->tsamp > 0.0, "invalid observation");
    if (t_end == t_begin) return;
    auto s = as_stream(stream);
    std::vector<double> freq(d->nchans);
    for (uint64_t c = 0; c < d->nchans; ++c)
      freq[c] = d->nchans == 1 ? d->f_high
                               : d->f_low + (d->f_high - d->f_low) * static_cast<double>(c) /
                                                static_cast<double>(d->nchans - 1);
    double fref = freq[0];
    for (double f : freq) fref = std::max(fref, f);
    std::vector<SynthPulsarDev> ps;
    for (int k = 0; k < d->npulsars; ++k) {
      const gf_synth_pulsar& q = d->pulsars[k];
      ps.push_back(SynthPulsarDev{q.period, q.dm, q.duty_cycle / 2.3548200450309493, q.amplitude, q.phase});
    }
    // small tables: staged through one temporary device allocation
    const size_t fb = freq.size() * sizeof(double);
    const size_t pb = ps.size() * sizeof(SynthPulsarDev);
    const size_t mb = d->narrowband_mask ? d->nchans : 0;
    DeviceBlob blob;
    std::vector<uint8_t> host(fb + pb + mb + 64);
    std::memcpy(host.data(), freq.data(), fb);
    if (pb) std::memcpy(host.data() + fb, ps.data(), pb);
    if (mb) std::memcpy(host.data() + fb + pb, d->narrowband_mask, mb);
    blob.upload(host.data(), host.size(), [] { int dev = 0; cudaGetDevice(&dev); return dev; }());
    SynthParams p{};
    p.nchans = d->nchans;
    p.seed = d->seed;
    p.tsamp = d->tsamp;
    p.fref = fref;
    p.freq = blob.as<double>();
    p.pulsars = reinterpret_cast<const SynthPulsarDev*>(blob.as<uint8_t>() + fb);
    p.npulsars = d->npulsars;
    p.nbits = d->nbits;
    p.nb_mask = mb ? blob.as<uint8_t>() + fb + pb : nullptr;
    p.nb_hz = d->narrowband_hz;
    p.nb_amp = d->narrowband_amplitude;
    p.impulse_period = d->impulse_hz > 0.0
                           ? std::max<int64_t>(1, static_cast<int64_t>(std::llround(1.0 / (d->impulse_hz * d->tsamp))))
                           : 0;
    p.impulse_amp = d->impulse_amplitude;
    p.t_begin = t_begin;
    p.row_bytes = d->nbits == 8 ? d->nchans : d->nchans / 4;
    const uint64_t nrows = t_end - t_begin;
    dim3 grid(static_cast<unsigned>(ceil_div(p.row_bytes, 256)), static_cast<unsigned>(std::min<uint64_t>(nrows, 65535)),
              static_cast<unsigned>(ceil_div(nrows, 65535)));
    synth_kernel<<<grid, 256, 0, s>>>(p, nrows, dev_out);
    cuda_check(cudaGetLastError(), "synth_kernel launch");
    // the tables must outlive the kernel
    cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize(synth)");
  });
}
