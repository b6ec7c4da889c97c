// SIGPROC filterbank ingest: header parsing, host reads, and device loads
// through pinned host memory with the channel reversal done on the GPU.
//
// Reference behaviour (lintian233/gaffa src/gaffa/io/filterbank.cpp):
//   read_header           :116-224  keyword stream (int length + bytes),
//                                   HEADER_START .. HEADER_END, FREQUENCY
//                                   blocks, nsamples from the file size
//   should_reverse_channels :86-95   ascending-frequency policy reverses a
//                                   descending band (foff < 0 or a
//                                   descending frequency table)
//   normalize_frequency_metadata :105-118
//   reverse_rows / read_samples :243-333 (each IF reversed independently)
// nbits 8, 16 and 32 follow the reference; packed 1-, 2- and 4-bit rows
// (channel k of a byte in bits [k*nbits, (k+1)*nbits)) are an addition: they
// load as packed rows and reverse field by field.
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace gf {
namespace {

struct FileCloser {
  FILE* f = nullptr;
  ~FileCloser() {
    if (f) std::fclose(f);
  }
};

void read_bytes(FILE* f, void* dst, size_t n, const char* what) {
  if (std::fread(dst, 1, n, f) != n) raise(GF_ERUNTIME, std::string("Failed to read filterbank field: ") + what);
}

std::string read_key(FILE* f) {
  int32_t len = 0;
  read_bytes(f, &len, sizeof len, "string length");
  if (len <= 0 || len > 4096) raise(GF_ERUNTIME, "Invalid filterbank string length");
  std::string s(static_cast<size_t>(len), '\0');
  if (std::fread(s.data(), 1, s.size(), f) != s.size()) raise(GF_ERUNTIME, "Failed to read filterbank string");
  return s;
}

uint64_t bits_row_bytes(int nbits, uint64_t nifs, uint64_t nchans) {
  if (nbits != 1 && nbits != 2 && nbits != 4 && nbits != 8 && nbits != 16 && nbits != 32)
    raise(GF_ERUNTIME, "Unsupported filterbank nbits");
  const uint64_t elems = nifs * nchans;
  if (nifs != 0 && elems / nifs != nchans) raise(GF_EOVERFLOW, "Filterbank size overflow: row elements");
  if (nbits < 8) {
    if ((nchans * static_cast<uint64_t>(nbits)) % 8 != 0)
      raise(GF_ERUNTIME, "packed filterbank rows must be whole bytes per IF");
    return elems * static_cast<uint64_t>(nbits) / 8;
  }
  return elems * static_cast<uint64_t>(nbits / 8);
}

struct Parsed {
  gf_filterbank_header h{};
  std::vector<double> freq;
  bool reverse = false;
  uint64_t row_bytes = 0;
};

void copy_string(char* dst, size_t cap, const std::string& s) {
  const size_t n = std::min(cap - 1, s.size());
  std::memcpy(dst, s.data(), n);
  dst[n] = '\0';
}

Parsed parse(const char* path, int32_t order) {
  check_arg(path != nullptr, "null argument");
  check_arg(order == GF_CHANNEL_ORDER_ASCENDING || order == GF_CHANNEL_ORDER_FILE, "unknown channel order");
  FileCloser fc;
  fc.f = std::fopen(path, "rb");
  if (!fc.f) raise(GF_ERUNTIME, std::string("Failed to open filterbank file: ") + path);
  FILE* f = fc.f;
  Parsed P;
  gf_filterbank_header& h = P.h;
  h.data_type = 1;
  h.nifs = 1;
  if (read_key(f) != "HEADER_START") raise(GF_ERUNTIME, "Non-standard filterbank file: missing HEADER_START");
  bool want_raw = false, want_source = false, in_freq = false;
  auto rd_i = [&](int32_t& v, const char* k) { read_bytes(f, &v, sizeof v, k); };
  auto rd_d = [&](double& v, const char* k) { read_bytes(f, &v, sizeof v, k); };
  while (true) {
    const std::string key = read_key(f);
    if (key == "HEADER_END") break;
    if (want_raw) {
      copy_string(h.rawdatafile, sizeof h.rawdatafile, key);
      want_raw = false;
    } else if (want_source) {
      copy_string(h.source_name, sizeof h.source_name, key);
      want_source = false;
    } else if (key == "rawdatafile") {
      want_raw = true;
    } else if (key == "source_name") {
      want_source = true;
    } else if (key == "FREQUENCY_START") {
      in_freq = true;
      h.uses_frequency_table = 1;
      P.freq.clear();
    } else if (key == "FREQUENCY_END") {
      in_freq = false;
      h.nchans = static_cast<int32_t>(P.freq.size());
    } else if (key == "fchannel") {
      if (!in_freq) raise(GF_ERUNTIME, "fchannel outside FREQUENCY block");
      double v = 0.0;
      rd_d(v, "fchannel");
      P.freq.push_back(v);
      h.fch1 = 0.0;
      h.foff = 0.0;
      h.uses_frequency_table = 1;
    } else if (key == "az_start") { rd_d(h.az_start, "az_start");
    } else if (key == "za_start") { rd_d(h.za_start, "za_start");
    } else if (key == "src_raj") { rd_d(h.src_raj, "src_raj");
    } else if (key == "src_dej") { rd_d(h.src_dej, "src_dej");
    } else if (key == "tstart") { rd_d(h.tstart, "tstart");
    } else if (key == "tsamp") { rd_d(h.tsamp, "tsamp");
    } else if (key == "period") { rd_d(h.period, "period");
    } else if (key == "fch1") { rd_d(h.fch1, "fch1");
    } else if (key == "foff") { rd_d(h.foff, "foff");
    } else if (key == "nchans") { rd_i(h.nchans, "nchans");
    } else if (key == "telescope_id") { rd_i(h.telescope_id, "telescope_id");
    } else if (key == "machine_id") { rd_i(h.machine_id, "machine_id");
    } else if (key == "data_type") { rd_i(h.data_type, "data_type");
    } else if (key == "ibeam") { rd_i(h.ibeam, "ibeam");
    } else if (key == "nbeams") { rd_i(h.nbeams, "nbeams");
    } else if (key == "nbits") { rd_i(h.nbits, "nbits");
    } else if (key == "barycentric") { rd_i(h.barycentric, "barycentric");
    } else if (key == "pulsarcentric") { rd_i(h.pulsarcentric, "pulsarcentric");
    } else if (key == "nbins") { rd_i(h.nbins, "nbins");
    } else if (key == "nsamples") { int32_t ignored = 0; rd_i(ignored, "nsamples");
    } else if (key == "nifs") { rd_i(h.nifs, "nifs");
    } else if (key == "npuls") { rd_i(h.npuls, "npuls");
    } else if (key == "refdm") { rd_d(h.refdm, "refdm");
    } else {
      raise(GF_ERUNTIME, "Unknown filterbank header field: " + key);
    }
  }
  const long pos = std::ftell(f);
  if (pos < 0) raise(GF_ERUNTIME, "Failed to determine filterbank header size");
  h.header_size = pos;
  if (h.nchans <= 0) raise(GF_ERUNTIME, "Invalid filterbank nchans");
  if (h.nifs <= 0) raise(GF_ERUNTIME, "Invalid filterbank nifs");
  if (std::fseek(f, 0, SEEK_END) != 0) raise(GF_ERUNTIME, "Failed to seek filterbank file");
  const long end = std::ftell(f);
  const int64_t data_bytes = static_cast<int64_t>(end) - h.header_size;
  if (data_bytes < 0) raise(GF_ERUNTIME, "Filterbank header is larger than file");
  P.row_bytes = bits_row_bytes(h.nbits, static_cast<uint64_t>(h.nifs), static_cast<uint64_t>(h.nchans));
  if (P.row_bytes == 0 || static_cast<uint64_t>(data_bytes) % P.row_bytes != 0)
    raise(GF_ERUNTIME, "Filterbank data size is not a whole number of rows");
  h.nsamples = data_bytes / static_cast<int64_t>(P.row_bytes);
  // frequencies of every channel in file order
  if (h.uses_frequency_table) {
    if (P.freq.size() != static_cast<size_t>(h.nchans)) raise(GF_ERUNTIME, "Frequency table length does not match nchans");
  } else {
    P.freq.resize(static_cast<size_t>(h.nchans));
    for (int32_t c = 0; c < h.nchans; ++c) P.freq[c] = h.fch1 + static_cast<double>(c) * h.foff;
  }
  if (order == GF_CHANNEL_ORDER_ASCENDING) {
    P.reverse = h.uses_frequency_table ? (P.freq.size() >= 2 && P.freq.front() > P.freq.back()) : h.foff < 0.0;
  }
  if (P.reverse) {
    std::reverse(P.freq.begin(), P.freq.end());
    if (!P.freq.empty()) h.fch1 = P.freq.front();
    if (!h.uses_frequency_table) h.foff = std::abs(h.foff);
  }
  h.reversed = P.reverse ? 1 : 0;
  return P;
}

// channel c of a packed byte row sits in bits [c*nbits, (c+1)*nbits) of byte
// c*nbits/8; reversing a whole-byte IF row reverses the bytes and the fields
// inside each byte
__host__ __device__ inline uint8_t reverse_fields(uint8_t b, int nbits) {
  if (nbits == 4) return static_cast<uint8_t>((b >> 4) | (b << 4));
  if (nbits == 2)
    return static_cast<uint8_t>(((b & 0x03u) << 6) | ((b & 0x0cu) << 2) | ((b & 0x30u) >> 2) | ((b & 0xc0u) >> 6));
  uint8_t r = 0;  // nbits == 1
  for (int i = 0; i < 8; ++i) r |= static_cast<uint8_t>(((b >> i) & 1u) << (7 - i));
  return r;
}

template <typename T>
void reverse_host(T* rows, uint64_t nrows, uint64_t nifs, uint64_t nelems) {
  for (uint64_t r = 0; r < nrows * nifs; ++r) std::reverse(rows + r * nelems, rows + (r + 1) * nelems);
}

void reverse_rows_host(uint8_t* data, uint64_t nrows, const Parsed& P) {
  const uint64_t nifs = static_cast<uint64_t>(P.h.nifs), nchans = static_cast<uint64_t>(P.h.nchans);
  switch (P.h.nbits) {
    case 8: reverse_host(data, nrows, nifs, nchans); break;
    case 16: reverse_host(reinterpret_cast<uint16_t*>(data), nrows, nifs, nchans); break;
    case 32: reverse_host(reinterpret_cast<float*>(data), nrows, nifs, nchans); break;
    default: {
      const uint64_t ifb = nchans * static_cast<uint64_t>(P.h.nbits) / 8;
      reverse_host(data, nrows, nifs, ifb);
      for (uint64_t i = 0; i < nrows * nifs * ifb; ++i) data[i] = reverse_fields(data[i], P.h.nbits);
    }
  }
}

// In-place channel reversal of rows*nifs IF rows of n elements: thread i swaps
// elements i and n-1-i of its row (the middle element of an odd row stays).
template <typename T>
__global__ void reverse_kernel(T* data, uint64_t nrowsif, uint64_t n) {
  const uint64_t half = (n + 1) / 2;
  const uint64_t total = nrowsif * half;
  for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < total;
       k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t r = k / half, i = k % half;
    T* row = data + r * n;
    const T a = row[i], b = row[n - 1 - i];
    row[i] = b;
    row[n - 1 - i] = a;
  }
}

__global__ void reverse_packed_kernel(uint8_t* data, uint64_t nrowsif, uint64_t n, int nbits) {
  const uint64_t half = (n + 1) / 2;
  const uint64_t total = nrowsif * half;
  for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < total;
       k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t r = k / half, i = k % half;
    uint8_t* row = data + r * n;
    const uint8_t a = row[i], b = row[n - 1 - i];
    row[i] = reverse_fields(b, nbits);
    row[n - 1 - i] = reverse_fields(a, nbits);
  }
}

void reverse_rows_device(void* data, uint64_t nrows, const Parsed& P, cudaStream_t s) {
  const uint64_t nifs = static_cast<uint64_t>(P.h.nifs), nchans = static_cast<uint64_t>(P.h.nchans);
  const uint64_t nrowsif = nrows * nifs;
  const unsigned grid = 148 * 8;
  switch (P.h.nbits) {
    case 8: reverse_kernel<uint8_t><<<grid, 256, 0, s>>>(static_cast<uint8_t*>(data), nrowsif, nchans); break;
    case 16: reverse_kernel<uint16_t><<<grid, 256, 0, s>>>(static_cast<uint16_t*>(data), nrowsif, nchans); break;
    case 32: reverse_kernel<float><<<grid, 256, 0, s>>>(static_cast<float*>(data), nrowsif, nchans); break;
    default:
      reverse_packed_kernel<<<grid, 256, 0, s>>>(static_cast<uint8_t*>(data), nrowsif,
                                                 nchans * static_cast<uint64_t>(P.h.nbits) / 8, P.h.nbits);
  }
  cuda_check(cudaGetLastError(), "filterbank reverse kernel launch");
}

void seek_rows(FILE* f, const Parsed& P, uint64_t row_begin) {
  const uint64_t off = static_cast<uint64_t>(P.h.header_size) + row_begin * P.row_bytes;
  if (fseeko(f, static_cast<off_t>(off), SEEK_SET) != 0) raise(GF_ERUNTIME, "Failed to seek filterbank file");
}

}  // namespace
}  // namespace gf

using namespace gf;

extern "C" int gf_filterbank_read_header(const char* path, int32_t channel_order, gf_filterbank_header* header,
                                         double* frequency_table, uint64_t capacity) {
  return guarded([&] {
    check_arg(header != nullptr, "null argument");
    const Parsed P = parse(path, channel_order);
    *header = P.h;
    if (frequency_table != nullptr)
      std::memcpy(frequency_table, P.freq.data(), std::min<uint64_t>(capacity, P.freq.size()) * sizeof(double));
  });
}

extern "C" int gf_filterbank_read_host(const char* path, int32_t channel_order, uint64_t row_begin, uint64_t nrows,
                                       void* host_out) {
  return guarded([&] {
    const Parsed P = parse(path, channel_order);
    check_arg(row_begin + nrows <= static_cast<uint64_t>(P.h.nsamples), "row range exceeds the file");
    if (nrows == 0) return;
    check_arg(host_out != nullptr, "null argument");
    FileCloser fc;
    fc.f = std::fopen(path, "rb");
    if (!fc.f) raise(GF_ERUNTIME, std::string("Failed to open filterbank file: ") + path);
    seek_rows(fc.f, P, row_begin);
    if (std::fread(host_out, 1, nrows * P.row_bytes, fc.f) != nrows * P.row_bytes)
      raise(GF_ERUNTIME, "Failed to read filterbank samples");
    if (P.reverse) reverse_rows_host(static_cast<uint8_t*>(host_out), nrows, P);
  });
}

extern "C" int gf_filterbank_load(const char* path, int32_t channel_order, uint64_t row_begin, uint64_t nrows,
                                  void* dev_out, void* host_bounce, uint64_t bounce_bytes, void* stream) {
  return guarded([&] {
    const Parsed P = parse(path, channel_order);
    check_arg(row_begin + nrows <= static_cast<uint64_t>(P.h.nsamples), "row range exceeds the file");
    if (nrows == 0) return;
    check_arg(dev_out && host_bounce, "null argument");
    // two halves of the pinned bounce buffer, whole rows each
    const uint64_t half_rows = (bounce_bytes / 2) / P.row_bytes;
    check_arg(half_rows > 0, "bounce buffer must hold two rows");
    auto s = as_stream(stream);
    FileCloser fc;
    fc.f = std::fopen(path, "rb");
    if (!fc.f) raise(GF_ERUNTIME, std::string("Failed to open filterbank file: ") + path);
    seek_rows(fc.f, P, row_begin);
    cudaEvent_t done[2];
    cuda_check(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming), "cudaEventCreate");
    struct Events {
      cudaEvent_t* e;
      ~Events() {
        cudaEventSynchronize(e[0]);
        cudaEventSynchronize(e[1]);
        cudaEventDestroy(e[0]);
        cudaEventDestroy(e[1]);
      }
    } guard{done};
    uint8_t* dst = static_cast<uint8_t*>(dev_out);
    bool used[2] = {false, false};
    // file reads of one half overlap the host-to-device copy of the other
    for (uint64_t r = 0, k = 0; r < nrows; r += half_rows, ++k) {
      const int b = static_cast<int>(k & 1);
      const uint64_t n = std::min(half_rows, nrows - r);
      uint8_t* buf = static_cast<uint8_t*>(host_bounce) + b * half_rows * P.row_bytes;
      if (used[b]) cuda_check(cudaEventSynchronize(done[b]), "cudaEventSynchronize(bounce)");
      if (std::fread(buf, 1, n * P.row_bytes, fc.f) != n * P.row_bytes)
        raise(GF_ERUNTIME, "Failed to read filterbank samples");
      cuda_check(cudaMemcpyAsync(dst + r * P.row_bytes, buf, n * P.row_bytes, cudaMemcpyHostToDevice, s),
                 "cudaMemcpyAsync(filterbank)");
      cuda_check(cudaEventRecord(done[b], s), "cudaEventRecord");
      used[b] = true;
    }
    if (P.reverse) reverse_rows_device(dev_out, nrows, P, s);
  });
}
