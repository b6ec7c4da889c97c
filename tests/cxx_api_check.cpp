// A C++ caller of gaffa's CUDA API (include/gaffa/*.h), written the way a
// program built against the reference's headers calls it: host sample
// views, plans, device results, copy_to_host, CudaFfaProgram,
// run_ffa_batch_cuda and both search_ffa_cuda overloads.  It generates a
// small seeded input, runs every call and writes inputs and outputs as raw
// little-endian arrays into the directory given as argv[1];
// tests/test_cxx_api.py compares them with the reference CPU path.
#include "gaffa/dedispersion_cuda.h"
#include "gaffa/ffa_cuda.h"
#include "gaffa/ffa_plan.h"

#include <cuda_runtime_api.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

std::string dir;

template <typename T>
void dump(const char* name, const std::vector<T>& v) {
  const std::string path = dir + "/" + name;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + path);
  if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
  std::fclose(f);
}

uint64_t lcg_state = 12345;
uint32_t lcg() {
  lcg_state = lcg_state * 6364136223846793005ull + 1442695040888963407ull;
  return static_cast<uint32_t>(lcg_state >> 33);
}

struct PeakRow {  // series, then the FfaPeak fields in declaration order
  uint64_t series;
  double period, frequency;
  uint64_t width;
  double duty_cycle;
  uint64_t width_index, period_index, phase, shift, bins;
  float snr;
  uint32_t pad;
};

PeakRow row(std::size_t series, const gaffa::FfaPeak& p) {
  return PeakRow{series, p.period, p.frequency, p.width, p.duty_cycle, p.width_index, p.period_index,
                 p.phase, p.shift, p.bins, p.snr, 0u};
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 2) {
    std::fprintf(stderr, "usage: cxx_api_check <output directory>\n");
    return 2;
  }
  dir = argv[1];
  try {
    // --- dedispersion: 64 channels, 3000 samples, ascending frequencies
    const std::size_t ns = 3000, nc = 64;
    std::vector<std::uint8_t> samples(ns * nc);
    for (auto& s : samples) s = static_cast<std::uint8_t>(96 + lcg() % 64);
    std::vector<double> freq(nc);
    for (std::size_t c = 0; c < nc; ++c) freq[c] = 1200.0 + 300.0 * static_cast<double>(c) / (nc - 1);
    dump("dd_input.u8", samples);
    dump("dd_freq.f64", freq);
    const gaffa::HostSampleView<std::uint8_t> view =
        gaffa::make_host_sample_view<std::uint8_t>(std::span<const std::uint8_t>(samples), {ns, 1, nc});

    gaffa::MultiDmDedispersionPlan multi{0.0, 2.0, 16, 1500.0, 1e-3, 0, nc};
    const auto m = gaffa::dedisperse_multi_dm_cuda(view, freq, multi);
    dump("dd_multi.u32", m.data);
    dump("dd_multi_shape.u64", std::vector<uint64_t>{m.shape.ndm, m.shape.nsamples});

    const auto dev = gaffa::dedisperse_multi_dm_cuda_device(view, freq, multi);
    const auto back = gaffa::copy_to_host(dev);
    dump("dd_multi_device.u32", back.data);

    const auto sb = gaffa::dedisperse_subband_cuda(view, freq, multi, gaffa::SubbandDedispersionOptions{16, 4});
    dump("dd_subband.u32", sb.data);

    gaffa::SingleDmDedispersionPlan single{10.0, 1500.0, 1e-3, 0, nc};
    const auto one = gaffa::dedisperse_single_dm_cuda(view, freq, single);
    dump("dd_single.u32", one.data);
    const auto spec = gaffa::dedisperse_spectrum_cuda(view, freq, single);
    dump("dd_spectrum.u8", spec.data);
    dump("dd_spectrum_shape.u64", std::vector<uint64_t>{spec.shape.nsamples, spec.shape.nifs, spec.shape.nchans});

    std::vector<uint64_t> errors;
    try {
      gaffa::MultiDmDedispersionPlan bad = multi;
      bad.ndm = 0;
      static_cast<void>(gaffa::dedisperse_multi_dm_cuda(view, freq, bad));
    } catch (const std::invalid_argument&) {
      errors.push_back(1);
    }
    try {
      std::vector<float> fs(ns * nc, 0.0f);
      static_cast<void>(gaffa::dedisperse_multi_dm_cuda(
          gaffa::make_host_sample_view<float>(std::span<const float>(fs), {ns, 1, nc}), freq, multi));
    } catch (const std::invalid_argument&) {
      errors.push_back(2);
    }

    // --- FFA: three series of 20000 samples with a weak pulse train
    const std::size_t n = 20000, nseries = 3;
    std::vector<float> series(nseries * n);
    for (std::size_t i = 0; i < series.size(); ++i) {
      // sum of four uniforms, centred: roughly unit-variance noise
      float v = 0.0f;
      for (int k = 0; k < 4; ++k) v += static_cast<float>(lcg() % 65536) / 65536.0f;
      series[i] = (v - 2.0f) * 1.7320508f;
      if ((i % n) % 331 == 7) series[i] += 2.5f;
    }
    dump("ffa_series.f32", series);
    const gaffa::FfaSearchPlan plan =
        gaffa::make_riptide_ffa_plan(n, 1e-3, gaffa::RiptideFfaPlanOptions{0.2, 1.0, 60, 80, 1, 0.2, 1.5, 1000000});
    std::vector<gaffa::FfaSearchTask> tasks(plan.tasks);
    dump("ffa_tasks.bin", tasks);
    dump("ffa_widths.u64", std::vector<uint64_t>(plan.width_trials.begin(), plan.width_trials.end()));

    gaffa::CudaDeviceBuffer<float> dseries(series.size());
    if (cudaMemcpy(dseries.data(), series.data(), dseries.bytes(), cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("cudaMemcpy");
    gaffa::CudaFfaExecutionOptions exec;
    exec.series_tile_size = 4;
    exec.initial_peak_buffer_bytes = 4096;  // small: forces the grow-and-rerun path
    gaffa::CudaFfaProgram program(plan, gaffa::CudaFfaProgramOptions{0}, exec);
    const auto batch = gaffa::run_ffa_batch_cuda(
        program, gaffa::CudaTimeSeriesBatchView{dseries.data(), nseries, n, 0}, gaffa::FfaSearchOptions{4.0f, 0});
    std::vector<PeakRow> rows;
    for (const auto& p : batch.peaks) rows.push_back(row(p.series_index, p.peak));
    dump("ffa_batch.bin", rows);

    const auto s1 = gaffa::search_ffa_cuda(program, gaffa::CudaSpan<const float>{dseries.data() + n, n, 0},
                                           gaffa::FfaSearchOptions{4.0f, 0});
    rows.clear();
    for (const auto& p : s1.peaks) rows.push_back(row(1, p));
    dump("ffa_search_program.bin", rows);
    const auto s2 = gaffa::search_ffa_cuda(gaffa::CudaSpan<const float>{dseries.data() + 2 * n, n, 0}, plan,
                                           gaffa::FfaSearchOptions{4.0f, 0});
    rows.clear();
    for (const auto& p : s2.peaks) rows.push_back(row(2, p));
    dump("ffa_search_oneshot.bin", rows);
    try {
      static_cast<void>(gaffa::search_ffa_cuda(program, gaffa::CudaSpan<const float>{dseries.data(), n, 0},
                                               gaffa::FfaSearchOptions{4.0f, 1}));
    } catch (const std::runtime_error&) {
      errors.push_back(3);
    }
    dump("errors.u64", errors);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cxx_api_check: %s\n", e.what());
    return 1;
  }
  std::printf("cxx_api_check ok\n");
  return 0;
}
