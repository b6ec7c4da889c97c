// Brute-force and subband incoherent dedispersion for sm_100a.
//
// Reference arithmetic: dedispersion.cpp:197-215 (direct_sum_at),
// :291-329 (dedisperse_multi_dm_cpu), :331-453 (dedisperse_subband_cpu) and
// internal/dedispersion_delay.h:37-139 (delay tables).  Sums are integer, so
// any summation order is bit-exact.
//
// Layout.  The time-major input ([time][chan] uint8, or packed 2-bit) is
// staged once into channel-major rows (one uint8 row per channel, row stride
// a multiple of 16 bytes); every DM block reuses it.
//
// Kernel.  One CTA = a block of DB DMs x a time tile; each warp owns one DM and
// 1008 consecutive output samples (252 output words of 4 samples).  The CTA
// streams channel chunks through a ring of 2-4 shared-memory stages: for each
// channel of a chunk one bulk copy (cp.async.bulk, completion counted in bytes
// on the stage's mbarrier) brings the window [t0 + base, t0 + base + RS)
// (base = delay of the block's first DM rounded down to 16), one more per DM
// its gather records, and one more the window bases of the chunk `stages`
// ahead.  Warps wait on the stage's barrier, sum, and release the stage with
// an acquire-release counter; the last warp to release it issues the copies
// of the chunk `stages` ahead into it, reading that chunk's window bases from
// the stage (so the refilling warp never waits on global memory).  No
// CTA-wide barrier runs per chunk, so warps drift apart by up to `stages`
// chunks.  DM blocks are the fastest grid index, so the CTAs resident at one
// time cover a few time tiles of every DM block of the launch and read each
// input window from L2.  A warp reads its DM's shifted window as aligned
// 32-bit words: the delay offset off = d - base splits into a word offset
// q = off >> 2 and a byte class s = off & 3.  The host sorts each warp's
// channels by class, so the class is static inside the loop: a word holds 4
// consecutive input bytes, which are split into even/odd byte pairs (LOP3 and
// PRMT) and accumulated in 16-bit lanes by IMAD; a class with an odd channel
// count ends with one single-channel step.  Per 256 channels the 16-bit lanes
// are flushed into 32-bit sums kept in shared memory after the ring,
// realigning class s by s bytes with one lane shuffle.  Lanes read
// consecutive words, so every LDS.32 is conflict-free.
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

namespace gf {

int32_t delay_bins(double dm, double f, double fref, double tsamp) {
  const double f2 = f * f;
  const double ref2 = fref * fref;
  const double delay = 4148.808 * dm * (1.0 / f2 - 1.0 / ref2);
  const double bins = std::round(delay / tsamp);
  if (bins < static_cast<double>(std::numeric_limits<int32_t>::min()) ||
      bins > static_cast<double>(std::numeric_limits<int32_t>::max()))
    raise(GF_EOVERFLOW, "dedispersion delay exceeds int32 range");
  return static_cast<int32_t>(bins);
}

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kWords = 8;                       // input words per lane
constexpr int kOutWords = 32 * kWords - 4;      // 252 output words per warp
constexpr int kWarpSamples = 4 * kOutWords;     // 1008 samples per warp
constexpr int kFlushChannels = 256;             // 16-bit lanes hold 256 x 255
constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxStages = 4;
// A stage whose copies have not landed after this many SM cycles (~2 s) is
// given up: the CTA sets GF_STATUS_PIPELINE in the program's status word
// (read by gf_dedisp_check) and returns.
constexpr long long kWaitCycles = 4000000000ll;

struct BytesParams {
  const uint8_t* in;         // group 0, row 0 of the launch
  uint64_t in_row_stride;    // bytes between channel rows
  uint64_t in_group_stride;  // bytes between groups
  uint64_t in_valid;         // valid samples per row (zero beyond)
  int rows_per_group;
  int total_rows;            // group g has min(rows_per_group, total_rows - g*rows_per_group) rows
  const int32_t* base;       // + g*base_group_stride + dm_block*base_block_stride
  uint64_t base_group_stride;
  uint64_t base_block_stride; // rows_per_group rounded up to 4 (16-byte aligned chunk rows)
  const uint32_t* records;   // + g*rec_group_stride + dm*rec_dm_stride + chunk*record_words
  uint64_t rec_group_stride;
  uint64_t rec_dm_stride;
  int nblocks;               // DM blocks per group in the launch (fastest grid index)
  uint32_t one;              // 1, opaque to the compiler: accumulation through IMAD
  int dm_count;              // DMs per group handled by the launch
  int dm_count_last;         // DMs of the launch's last group
  int ngroups;
  int dms_per_cta;
  int warps_per_dm;
  int chunk_rows;
  int nchunks;
  int row_bytes;
  int record_words;
  uint64_t cta_samples;
  void* out;                 // row (dm*out_dm_rows + g*out_group_rows)
  uint64_t out_row_stride;   // elements between output rows
  uint64_t out_dm_rows;
  uint64_t out_group_rows;
  uint64_t nout;             // valid output samples
  uint32_t grid_x;           // CTAs per group (grid x)
  int stages;                // shared-memory stages in the copy ring (2-4)
  uint32_t stage_bytes;      // windows, records and the window bases of the chunk `stages` ahead
  uint32_t base_bytes;       // chunk_rows * 4 rounded up to 16
  uint32_t* status;          // GF_STATUS_PIPELINE when a stage wait gives up
};

// Copy-ring state in static shared memory.
struct PipeShared {
  uint64_t full[kMaxStages];      // one phase per use of the stage: 32 arrivals + the copied bytes
  uint32_t released[kMaxStages];  // warps done with the stage's current chunk
  uint32_t failed;                // a wait of this CTA gave up
};

__device__ __forceinline__ uint32_t lo16(uint32_t v) { return v & 0xffffu; }
__device__ __forceinline__ uint32_t hi16(uint32_t v) { return v >> 16; }
// byte position b (0..3) of the 4-sample word, from the even/odd accumulators
__device__ __forceinline__ uint32_t pos_sum(uint32_t e, uint32_t o, int b) {
  return b == 0 ? lo16(e) : b == 1 ? lo16(o) : b == 2 ? hi16(e) : hi16(o);
}

// acc: the warp's 32-bit sums in shared memory, [m][position][lane].
template <int S>
__device__ __forceinline__ void flush_class(uint32_t (&e)[kWords], uint32_t (&o)[kWords], uint32_t* acc,
                                            int lane) {
#pragma unroll
  for (int m = 0; m < kWords; ++m) {
    if (S == 0) {
#pragma unroll
      for (int p = 0; p < 4; ++p) acc[(m * 4 + p) * 32 + lane] += pos_sum(e[m], o[m], p);
    } else {
      // class S word j contributes to output positions p = b - S of word j
      // (b >= S) and p = b - S + 4 of word j - 1 (b < S); so output word j
      // takes bytes b >= S of word j and bytes b < S of word j + 1.
      uint32_t ne = __shfl_down_sync(kFull, e[m], 1);
      uint32_t no = __shfl_down_sync(kFull, o[m], 1);
      const uint32_t we = __shfl_sync(kFull, m + 1 < kWords ? e[(m + 1) % kWords] : 0u, 0);
      const uint32_t wo = __shfl_sync(kFull, m + 1 < kWords ? o[(m + 1) % kWords] : 0u, 0);
      if (lane == 31) { ne = we; no = wo; }
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int b = p + S;
        acc[(m * 4 + p) * 32 + lane] += b < 4 ? pos_sum(e[m], o[m], b) : pos_sum(ne, no, b - 4);
      }
    }
    e[m] = 0u;
    o[m] = 0u;
  }
}

template <int S>
__device__ __forceinline__ void accumulate_class(const uint32_t* __restrict__ smem_words,
                                                 const uint32_t* __restrict__ rec, int& pos,
                                                 int npairs, int lane_word,
                                                 uint32_t (&e)[kWords], uint32_t (&o)[kWords], uint32_t one) {
  uint32_t next = npairs > 0 ? rec[pos] : 0u;  // the next pair's entry loads a pair ahead
  for (int i = 0; i < npairs; ++i) {
    const uint32_t entry = next;
    next = rec[pos + i + 1];
    const uint32_t* a = smem_words + (entry & 0xffffu) + lane_word;
    const uint32_t* b = smem_words + (entry >> 16) + lane_word;
#pragma unroll
    for (int m = 0; m < kWords; ++m) {
      const uint32_t w1 = a[32 * m];
      const uint32_t w2 = b[32 * m];
      e[m] = (w1 & 0x00ff00ffu) * one + e[m];
      e[m] = (w2 & 0x00ff00ffu) * one + e[m];
      o[m] = __byte_perm(w1, 0u, 0x4341) * one + o[m];
      o[m] = __byte_perm(w2, 0u, 0x4341) * one + o[m];
    }
  }
  pos += npairs;
}

// The last entry of a class with an odd channel count (low half of its word).
template <int S>
__device__ __forceinline__ void accumulate_single(const uint32_t* __restrict__ smem_words, uint32_t entry,
                                                  int lane_word, uint32_t (&e)[kWords], uint32_t (&o)[kWords],
                                                  uint32_t one) {
  const uint32_t* a = smem_words + (entry & 0xffffu) + lane_word;
#pragma unroll
  for (int m = 0; m < kWords; ++m) {
    const uint32_t w = a[32 * m];
    e[m] = (w & 0x00ff00ffu) * one + e[m];
    o[m] = __byte_perm(w, 0u, 0x4341) * one + o[m];
  }
}

// A class's entries: npairs = count / 2 pairs, then the odd one out.
template <int S>
__device__ __forceinline__ void accumulate_entries(const uint32_t* __restrict__ smem_words,
                                                   const uint32_t* __restrict__ rec, int& pos, uint32_t count,
                                                   int lane_word, uint32_t (&e)[kWords], uint32_t (&o)[kWords],
                                                   uint32_t one) {
  accumulate_class<S>(smem_words, rec, pos, static_cast<int>(count >> 1), lane_word, e, o, one);
  if (count & 1u) {
    accumulate_single<S>(smem_words, rec[pos], lane_word, e, o, one);
    ++pos;
  }
}

// -- copy ring primitives (PTX ISA 8.x: mbarrier, cp.async.bulk) -------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 state;\n\t"
      "mbarrier.arrive.release.cta.shared::cta.b64 state, [%0];\n}\n" ::"r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Global -> shared copy of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) completing on `bar`.  No multicast: the source is this GPU's memory.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ uint32_t release_stage(uint32_t* counter) {
  uint32_t old;
  asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;\n" : "=r"(old) : "r"(smem_u32(counter)) : "memory");
  return old;
}
// Waits for phase `parity` of `bar`; false when it gave up (this CTA's
// failure flag, another CTA's status bit, or kWaitCycles).
__device__ __forceinline__ bool wait_stage(uint64_t* bar, uint32_t parity, const PipeShared& ps,
                                        const uint32_t* status) {
  const long long start = clock64();
  for (uint32_t i = 0;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*reinterpret_cast<const volatile uint32_t*>(&ps.failed)) return false;
    if ((i & 255u) == 255u && (*reinterpret_cast<const volatile uint32_t*>(status) & GF_STATUS_PIPELINE))
      return false;
    if (clock64() - start > kWaitCycles) return false;
  }
}

// The calling warp stages chunk k of CTA (group, block, t0) into stage s:
// lane r copies channel rows r and r + 32 (bulk below the last 16-byte
// boundary of the valid samples, by hand with zeros past them), lanes
// d < dms_per_cta the records of DM d, and one lane the window bases of chunk
// k + stages (read by the warp that refills this stage).  The window bases of
// chunk k come from `bases` (shared memory; global for the first chunks).
// The stage's barrier completes after the 32 lane arrivals and the bytes
// that lane 0 announced.  Rows are taken one at a time to keep this path's
// registers few next to the summing loop's accumulators.
__device__ __forceinline__ uint32_t row_bulk_bytes(const BytesParams& p, uint64_t t_row) {
  const uint64_t bulk_end = p.in_valid & ~15ull;
  return t_row < bulk_end ? static_cast<uint32_t>(umin64(p.row_bytes, bulk_end - t_row)) : 0u;
}

__device__ __forceinline__ void issue_chunk(const BytesParams& p, PipeShared& ps, uint8_t* smem, int k, int s,
                                            int group, int block, uint64_t t0, int dm_limit, int group_rows,
                                            const int32_t* bases) {
  const int lane = threadIdx.x & 31;
  const int32_t* gbase = p.base + group * p.base_group_stride + static_cast<uint64_t>(block) * p.base_block_stride;
  const int row0 = k * p.chunk_rows;
  const int nrows = min(p.chunk_rows, group_rows - row0);
  const int dl = block * p.dms_per_cta + lane;
  const bool rec_copy = lane < p.dms_per_cta && dl < dm_limit;
  const bool base_copy = lane == 31 && k + p.stages < p.nchunks;
  uint32_t bytes = rec_copy ? static_cast<uint32_t>(p.record_words) * 4u : 0u;
  if (base_copy) bytes += p.base_bytes;
#pragma unroll 1
  for (int r = lane; r < nrows; r += 32) bytes += row_bulk_bytes(p, t0 + static_cast<uint64_t>(bases[r]));
  const uint32_t total = __reduce_add_sync(kFull, bytes);
  if (lane == 0) mbar_expect_tx(&ps.full[s], total);
  __syncwarp();
  fence_proxy_async_smem();  // earlier accesses of the stage before the copies' writes
  uint8_t* rows = smem + static_cast<uint32_t>(s) * p.stage_bytes;
  const uint32_t rows_bytes = static_cast<uint32_t>(p.chunk_rows) * p.row_bytes;
  const uint32_t rec_bytes = static_cast<uint32_t>(p.dms_per_cta * p.record_words) * 4u;
#pragma unroll 1
  for (int r = lane; r < nrows; r += 32) {
    const uint64_t t_row = t0 + static_cast<uint64_t>(bases[r]);
    const uint32_t nbulk = row_bulk_bytes(p, t_row);
    const uint8_t* src = p.in + group * p.in_group_stride + static_cast<uint64_t>(row0 + r) * p.in_row_stride;
    uint8_t* dst = rows + r * p.row_bytes;
    if (nbulk) bulk_copy(dst, src + t_row, nbulk, &ps.full[s]);
#pragma unroll 1
    for (uint32_t b = nbulk; b < static_cast<uint32_t>(p.row_bytes); b += 16) {
      const uint64_t t = t_row + b;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (t < p.in_valid) {
        uint8_t tmp[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) tmp[q] = (t + q < p.in_valid) ? src[t + q] : 0;
        memcpy(&v, tmp, 16);
      }
      *reinterpret_cast<uint4*>(dst + b) = v;
    }
  }
  if (rec_copy)
    bulk_copy(reinterpret_cast<uint32_t*>(rows + rows_bytes) + lane * p.record_words,
              p.records + group * p.rec_group_stride + dl * p.rec_dm_stride +
                  static_cast<uint64_t>(k) * p.record_words,
              static_cast<uint32_t>(p.record_words) * 4u, &ps.full[s]);
  // every lane has read `bases` (which may be this stage's base area) before
  // the copy of the next bases overwrites it
  __syncwarp();
  fence_proxy_async_smem();
  if (base_copy)
    bulk_copy(rows + rows_bytes + rec_bytes, gbase + static_cast<uint64_t>(k + p.stages) * p.chunk_rows,
              p.base_bytes, &ps.full[s]);
  mbar_arrive(&ps.full[s]);
}

// One CTA of a bytes launch: CTA bx of group `group` (grid x and z).
template <typename OutT>
__device__ __forceinline__ void bytes_cta(const BytesParams& p, unsigned bx, int group, uint8_t* smem,
                                          PipeShared& ps) {
  // DM block fastest: the CTAs resident at once share their input windows in L2
  const int block = static_cast<int>(bx % static_cast<unsigned>(p.nblocks));
  const uint64_t t0 = static_cast<uint64_t>(bx / static_cast<unsigned>(p.nblocks)) * p.cta_samples;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int dm_sub = warp / p.warps_per_dm;
  const int sub = warp % p.warps_per_dm;
  const int dm_local = block * p.dms_per_cta + dm_sub;
  const int dm_limit = group + 1 == p.ngroups ? p.dm_count_last : p.dm_count;
  const bool active = dm_sub < p.dms_per_cta && dm_local < dm_limit;

  const int group_rows = min(p.rows_per_group, p.total_rows - group * p.rows_per_group);
  // a stage: chunk_rows channel windows, then the chunk's records of every DM
  const uint32_t rows_bytes = static_cast<uint32_t>(p.chunk_rows) * p.row_bytes;

  if (threadIdx.x == 0) {
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(&ps.full[s], 32);
      ps.released[s] = 0;
    }
    // another CTA of the launch gave up: do nothing
    ps.failed = (*reinterpret_cast<const volatile uint32_t*>(p.status) & GF_STATUS_PIPELINE) ? 1u : 0u;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (ps.failed) return;

  // 16-bit lane sums per byte class in registers; 32-bit sums in shared
  // memory after the ring ([warp][m][position][lane], conflict-free)
  uint32_t e[4][kWords], o[4][kWords];
  uint32_t* acc = reinterpret_cast<uint32_t*>(smem + static_cast<uint32_t>(p.stages) * p.stage_bytes) +
                  warp * (kWords * 4 * 32);
#pragma unroll
  for (int m = 0; m < kWords; ++m) {
#pragma unroll
    for (int s = 0; s < 4; ++s) { e[s][m] = 0u; o[s][m] = 0u; }
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[(m * 4 + q) * 32 + lane] = 0u;
  }
  const int lane_word = sub * kOutWords + lane;
  const int chunks_per_flush = kFlushChannels / p.chunk_rows;

  if (warp == 0) {
    const int32_t* gbase =
        p.base + group * p.base_group_stride + static_cast<uint64_t>(block) * p.base_block_stride;
    for (int k = 0; k < min(p.stages, p.nchunks); ++k)
      issue_chunk(p, ps, smem, k, k, group, block, t0, dm_limit, group_rows, gbase + k * p.chunk_rows);
  }
  int s = 0;
  uint32_t parity = 0;
  bool ok = true;
  for (int k = 0; k < p.nchunks; ++k) {
    if (!wait_stage(&ps.full[s], parity, ps, p.status)) {
      ok = false;
      break;
    }
    if (active) {
      const uint8_t* rows = smem + static_cast<uint32_t>(s) * p.stage_bytes;
      const uint32_t* smem_words = reinterpret_cast<const uint32_t*>(rows);
      const uint32_t* rec = reinterpret_cast<const uint32_t*>(rows + rows_bytes) + dm_sub * p.record_words;
      const uint32_t counts = rec[0];
      int pos = 1;
      accumulate_entries<0>(smem_words, rec, pos, counts & 0xffu, lane_word, e[0], o[0], p.one);
      accumulate_entries<1>(smem_words, rec, pos, (counts >> 8) & 0xffu, lane_word, e[1], o[1], p.one);
      accumulate_entries<2>(smem_words, rec, pos, (counts >> 16) & 0xffu, lane_word, e[2], o[2], p.one);
      accumulate_entries<3>(smem_words, rec, pos, counts >> 24, lane_word, e[3], o[3], p.one);
      if ((k + 1) % chunks_per_flush == 0 || k + 1 == p.nchunks) {
        flush_class<0>(e[0], o[0], acc, lane);
        flush_class<1>(e[1], o[1], acc, lane);
        flush_class<2>(e[2], o[2], acc, lane);
        flush_class<3>(e[3], o[3], acc, lane);
      }
    }
    // release the stage; the last warp out refills it with chunk k + stages
    __syncwarp();
    uint32_t last = 0;
    if (lane == 0) {
      last = release_stage(&ps.released[s]) == static_cast<uint32_t>(kWarps - 1) ? 1u : 0u;
      if (last) ps.released[s] = 0;
    }
    last = __shfl_sync(kFull, last, 0);
    if (last && k + p.stages < p.nchunks) {
      const uint8_t* stage = smem + static_cast<uint32_t>(s) * p.stage_bytes;
      const int32_t* next_bases = reinterpret_cast<const int32_t*>(
          stage + static_cast<uint32_t>(p.chunk_rows) * p.row_bytes +
          static_cast<uint32_t>(p.dms_per_cta * p.record_words) * 4u);
      issue_chunk(p, ps, smem, k + p.stages, s, group, block, t0, dm_limit, group_rows, next_bases);
    }
    if (++s == p.stages) {
      s = 0;
      parity ^= 1u;
    }
  }
  if (!ok) {
    // give up: flag it, let the copies already issued to this stage land
    // (bounded), and write nothing
    if (lane == 0) {
      *reinterpret_cast<volatile uint32_t*>(&ps.failed) = 1u;
      atomicOr(p.status, GF_STATUS_PIPELINE);
    }
    const long long start = clock64();
    while (!mbar_try_wait(&ps.full[s], parity) && clock64() - start < kWaitCycles) {
    }
    return;
  }
  if (!active) return;
  OutT* out = static_cast<OutT*>(p.out) +
              (static_cast<uint64_t>(dm_local) * p.out_dm_rows +
               static_cast<uint64_t>(group) * p.out_group_rows) * p.out_row_stride;
#pragma unroll
  for (int m = 0; m < kWords; ++m) {
    const int j = lane + 32 * m;
    if (j >= kOutWords) continue;
    const uint64_t t = t0 + static_cast<uint64_t>(sub) * kWarpSamples + 4ull * j;
    if (t >= p.nout) continue;
    if (sizeof(OutT) == 4 && t + 4 <= p.nout && (p.out_row_stride & 3) == 0) {
      *reinterpret_cast<uint4*>(out + t) =
          make_uint4(acc[(m * 4) * 32 + lane], acc[(m * 4 + 1) * 32 + lane], acc[(m * 4 + 2) * 32 + lane],
                     acc[(m * 4 + 3) * 32 + lane]);
    } else if (sizeof(OutT) == 1 && t + 4 <= p.nout && (p.out_row_stride & 3) == 0) {
      *reinterpret_cast<uint32_t*>(out + t) =
          acc[(m * 4) * 32 + lane] | (acc[(m * 4 + 1) * 32 + lane] << 8) | (acc[(m * 4 + 2) * 32 + lane] << 16) |
          (acc[(m * 4 + 3) * 32 + lane] << 24);
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (t + q < p.nout) out[t + q] = static_cast<OutT>(acc[(m * 4 + q) * 32 + lane]);
    }
  }
}

template <typename OutT>
__global__ void __launch_bounds__(kThreads, 2) dedisperse_bytes_kernel(BytesParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ PipeShared ps;
  bytes_cta<OutT>(p, blockIdx.x, static_cast<int>(blockIdx.z), smem, ps);
}

// Many launches (programs, DM ranges, observations) as one grid: CTA b runs
// CTA b - block_begin[i] of launch i, the last launch starting at or before b.
__global__ void __launch_bounds__(kThreads, 2) dedisperse_bytes_batch_kernel(const BytesParams* __restrict__ items,
                                                                             const uint64_t* __restrict__ block_begin,
                                                                             int nitems) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ BytesParams sp;
  __shared__ uint32_t s_local;
  __shared__ PipeShared ps;
  if (threadIdx.x == 0) {
    const uint64_t b = blockIdx.x;
    int lo = 0, hi = nitems;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (block_begin[mid] <= b) lo = mid; else hi = mid;
    }
    sp = items[lo];
    s_local = static_cast<uint32_t>(b - block_begin[lo]);
  }
  __syncthreads();
  const uint32_t local = s_local;
  bytes_cta<uint32_t>(sp, local % sp.grid_x, static_cast<int>(local / sp.grid_x), smem, ps);
}

// Stage-2 sum over uint32 intermediate rows (subband with 8-bit input, where
// partial sums exceed a byte): out[dm][t] = sum_b inter[b][t + r(dm, b)].
__global__ void __launch_bounds__(256) subband_stage2_u32_kernel(
    const uint32_t* __restrict__ inter, uint64_t inter_row_stride, uint64_t inter_group_stride,
    uint64_t inter_valid, int nsb, const int32_t* __restrict__ resid, int ndm_group,
    uint32_t* __restrict__ out, uint64_t out_row_stride, uint64_t nout) {
  const int group = blockIdx.z;
  const int dm_local = blockIdx.y;
  if (dm_local >= ndm_group) return;
  const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nout) return;
  const uint32_t* base = inter + group * inter_group_stride;
  const int32_t* r = resid + (static_cast<uint64_t>(group) * ndm_group + dm_local) * nsb;
  uint32_t sum = 0;
  for (int b = 0; b < nsb; ++b) {
    const uint64_t st = t + static_cast<uint64_t>(r[b]);
    if (st < inter_valid) sum += __ldg(base + b * inter_row_stride + st);
  }
  out[(static_cast<uint64_t>(group) * ndm_group + dm_local) * out_row_stride + t] = sum;
}

// Aligned single-DM spectrum: out[t][c] = in[t + d(c)][chan_begin + c].  A
// warp per output time step, lanes over channels, so output rows are written
// coalesced; neighbouring channels read nearby input rows (the delay varies
// slowly across channels) and share L1/L2 lines.
template <typename T>
__global__ void __launch_bounds__(256) spectrum_kernel(const T* __restrict__ in, uint64_t nchans,
                                                       uint64_t chan_begin, uint32_t nc,
                                                       const int32_t* __restrict__ delay, uint64_t nout,
                                                       T* __restrict__ out) {
  const uint32_t c = blockIdx.y * 32 + (threadIdx.x & 31);
  if (c >= nc) return;
  const uint64_t d = static_cast<uint64_t>(delay[c]);
  const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * 64;
  for (uint32_t tt = threadIdx.x >> 5; tt < 64; tt += 8) {
    const uint64_t t = t0 + tt;
    if (t >= nout) break;
    out[t * nc + c] = in[(t + d) * nchans + chan_begin + c];
  }
}

// Time-major [nsamples][row_bytes] -> channel-major rows [chan][row_stride]
// for channels [chan_begin, chan_end); 8-bit copy or 2-bit unpack (channel
// 4k+j in bits [2j, 2j+1] of byte k).  64 samples x 64 channels per CTA.
template <int Bits>
__global__ void __launch_bounds__(256) stage_kernel(const uint8_t* __restrict__ in, uint64_t nsamples,
                                                    uint64_t in_row_bytes, int chan_begin, int nchan,
                                                    uint8_t* __restrict__ out, uint64_t out_stride,
                                                    uint64_t t_offset) {
  __shared__ uint8_t tile[64][64 + 4];
  const uint64_t tb = static_cast<uint64_t>(blockIdx.x) * 64;
  const int cb = blockIdx.y * 64;
  for (int i = threadIdx.x; i < 64 * 64; i += 256) {
    const int tt = i / 64, cc = i % 64;
    const uint64_t t = tb + tt;
    const int c = cb + cc;
    uint8_t v = 0;
    if (t < nsamples && c < nchan) {
      const int ch = chan_begin + c;
      if (Bits == 8) {
        v = in[t * in_row_bytes + ch];
      } else {
        v = (in[t * in_row_bytes + (ch >> 2)] >> (2 * (ch & 3))) & 3u;
      }
    }
    tile[tt][cc] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 64 * 64; i += 256) {
    const int cc = i / 64, tt = i % 64;
    const uint64_t t = tb + tt;
    const int c = cb + cc;
    if (t < nsamples && c < nchan) out[static_cast<uint64_t>(c) * out_stride + t_offset + t] = tile[tt][cc];
  }
}

// Class-sorted gather records: word 0 packs the four class counts (channels
// of byte class 0..3), then (chunk_rows + 4) / 2 words of u16 entry pairs
// (word offsets into the stage: row * row_bytes / 4 + delay offset / 4).
struct Records {
  std::vector<uint32_t> words;
  std::vector<int32_t> base;  // [group][block][base_stride]
  int base_stride = 0;
  int record_words = 0;
  int nchunks = 0;
  int max_off = 0;
};

// delays: [ngroups][ndm_group][rows_per_group] (rows beyond a ragged last
// group are ignored).  Builds base[group][block][row] (rows padded to a
// multiple of 4, so every chunk's bases start on 16 bytes) and the records.
Records build_records(const std::vector<int32_t>& delays, int ngroups, int ndm_group,
                      int rows_per_group, int total_rows, int dms_per_cta, int chunk_rows,
                      int row_bytes) {
  Records r;
  const int blocks = static_cast<int>(ceil_div(ndm_group, dms_per_cta));
  r.nchunks = static_cast<int>(ceil_div(rows_per_group, chunk_rows));
  r.record_words = static_cast<int>(round_up(1 + (chunk_rows + 4) / 2, 4));
  r.base_stride = static_cast<int>(round_up(rows_per_group, 4));
  // + 64 entries: the last chunk's 16-byte base copy may read past its block
  r.base.assign(static_cast<size_t>(ngroups) * blocks * r.base_stride + 64, 0);
  r.words.assign(static_cast<size_t>(ngroups) * ndm_group * r.nchunks * r.record_words, 0u);
  std::vector<uint16_t> cls[4];
  for (int g = 0; g < ngroups; ++g) {
    const int grows = std::min(rows_per_group, total_rows - g * rows_per_group);
    for (int b = 0; b < blocks; ++b) {
      const int d0 = b * dms_per_cta;
      for (int row = 0; row < grows; ++row) {
        const int32_t d = delays[(static_cast<size_t>(g) * ndm_group + d0) * rows_per_group + row];
        r.base[(static_cast<size_t>(g) * blocks + b) * r.base_stride + row] = d & ~15;
      }
    }
    for (int dm = 0; dm < ndm_group; ++dm) {
      const int b = dm / dms_per_cta;
      for (int k = 0; k < r.nchunks; ++k) {
        for (auto& c : cls) c.clear();
        const int row0 = k * chunk_rows;
        const int nrows = std::min(chunk_rows, grows - row0);
        for (int i = 0; i < nrows; ++i) {
          const int row = row0 + i;
          const int32_t d = delays[(static_cast<size_t>(g) * ndm_group + dm) * rows_per_group + row];
          const int32_t off = d - r.base[(static_cast<size_t>(g) * blocks + b) * r.base_stride + row];
          r.max_off = std::max(r.max_off, off);
          const int word = i * (row_bytes / 4) + (off >> 2);
          cls[off & 3].push_back(static_cast<uint16_t>(word));
        }
        uint32_t* rec = r.words.data() +
                        ((static_cast<size_t>(g) * ndm_group + dm) * r.nchunks + k) * r.record_words;
        uint32_t counts = 0;
        std::vector<uint16_t> flat;
        for (int s = 0; s < 4; ++s) {
          // the count is the class's channels; an odd class takes a whole
          // word for its last entry (high half unused), so classes start on words
          counts |= static_cast<uint32_t>(cls[s].size()) << (8 * s);
          if (cls[s].size() & 1) cls[s].push_back(0);
          flat.insert(flat.end(), cls[s].begin(), cls[s].end());
        }
        rec[0] = counts;
        for (size_t i = 0; i + 1 < flat.size(); i += 2)
          rec[1 + i / 2] = static_cast<uint32_t>(flat[i]) | (static_cast<uint32_t>(flat[i + 1]) << 16);
      }
    }
  }
  return r;
}

struct Launch {
  int dms_per_cta = kWarps;
  int warps_per_dm = 1;
  int chunk_rows = 64;
  int row_bytes = 0;
  int stages = 2;
  uint32_t stage_bytes = 0;
  size_t smem = 0;
};

// Picks the DM block size, channel chunk and ring depth so the stages fit in
// shared memory with two CTAs per SM when possible (228 KB per SM, 1 KB
// reserved per CTA, the ring state and batch table in static shared memory):
// the largest chunk with 4 stages, else 3, else 2.  dpc_fix / cr_fix (0 = any)
// pin the DM block or the chunk rows (launch shapes picked by an autotuner);
// every shape gives the same sums.
template <typename F>
Launch choose_launch(F&& max_off_for, int dpc_fix, int cr_fix) {
  const size_t acc = static_cast<size_t>(kWarps) * kWords * 4 * 32 * 4;  // 32-bit sums
  const size_t budget2 = 112 * 1024 - acc, budget1 = 224 * 1024 - acc;
  for (size_t budget : {budget2, budget1}) {
    for (int dpc : {8, 4, 2, 1}) {
      if (dpc_fix && dpc != dpc_fix) continue;
      const int wpd = kWarps / dpc;
      const int max_off = max_off_for(dpc);
      const int row_bytes = static_cast<int>(round_up(max_off + 4 * ((wpd - 1) * kOutWords + 32 * kWords), 16));
      for (int cr : {64, 32, 16, 8}) {
        if (cr_fix && cr != cr_fix) continue;
        const size_t rec = static_cast<size_t>(dpc) * round_up(1 + (cr + 4) / 2, 4) * 4;
        const size_t stage = static_cast<size_t>(cr) * row_bytes + rec + round_up(cr * 4, 16);
        if (static_cast<size_t>(cr) * row_bytes >= 65536 * 4) continue;  // u16 word offsets
        for (int st : {4, 3, 2}) {
          if (st * stage <= budget)
            return Launch{dpc, wpd, cr, row_bytes, st, static_cast<uint32_t>(stage), st * stage + acc};
        }
      }
    }
  }
  raise(GF_EINVAL, "dedispersion delay spread too large for a shared-memory tile");
}

int max_off_estimate(const std::vector<int32_t>& delays, int ngroups, int ndm_group,
                     int rows_per_group, int total_rows, int dpc) {
  int mo = 0;
  for (int g = 0; g < ngroups; ++g) {
    const int grows = std::min(rows_per_group, total_rows - g * rows_per_group);
    for (int dm = 0; dm < ndm_group; ++dm) {
      const int d0 = (dm / dpc) * dpc;
      for (int row = 0; row < grows; ++row) {
        const int32_t d = delays[(static_cast<size_t>(g) * ndm_group + dm) * rows_per_group + row];
        const int32_t b = delays[(static_cast<size_t>(g) * ndm_group + d0) * rows_per_group + row] & ~15;
        mo = std::max(mo, d - b);
      }
    }
  }
  return mo;
}

// One bytes-kernel configuration with its device tables: ngroups groups of
// ndm_group DMs over rows_per_group rows (ragged last group).
struct BytesStage {
  Launch launch;
  Records rec;
  DeviceBlob base_dev, rec_dev, status_dev;
  int ngroups = 0, ndm_group = 0, rows_per_group = 0, total_rows = 0, blocks = 0;

  void build(const std::vector<int32_t>& delays, int ng, int ndg, int rpg, int tr, int device, int dpc_fix = 0,
             int cr_fix = 0) {
    ngroups = ng;
    ndm_group = ndg;
    rows_per_group = rpg;
    total_rows = tr;
    launch = choose_launch([&](int dpc) { return max_off_estimate(delays, ng, ndg, rpg, tr, dpc); }, dpc_fix,
                           cr_fix);
    blocks = static_cast<int>(ceil_div(ndg, launch.dms_per_cta));
    rec = build_records(delays, ng, ndg, rpg, tr, launch.dms_per_cta, launch.chunk_rows, launch.row_bytes);
    base_dev.upload(rec.base.data(), rec.base.size() * sizeof(int32_t), device);
    rec_dev.upload(rec.words.data(), rec.words.size() * sizeof(uint32_t), device);
    const uint32_t zero = 0;
    status_dev.upload(&zero, sizeof zero, device);
  }

  // Reads and clears the status word (GF_STATUS_PIPELINE: a launch gave up).
  uint32_t take_status(cudaStream_t stream) const {
    if (!status_dev.ptr) return 0;
    uint32_t v = 0;
    cuda_check(cudaMemcpyAsync(&v, status_dev.ptr, sizeof v, cudaMemcpyDeviceToHost, stream), "dedispersion status");
    cuda_check(cudaStreamSynchronize(stream), "dedispersion status");
    if (v) cuda_check(cudaMemsetAsync(status_dev.ptr, 0, sizeof v, stream), "dedispersion status reset");
    return v;
  }

  uint64_t metadata_bytes() const { return base_dev.bytes + rec_dev.bytes; }

  // Launch for groups [g0, g0 + gcount) and, within each group, DMs
  // [dm_first, dm_first + dm_count) (dm_first a multiple of the DM block);
  // the last launched group handles dm_count_last DMs.  in / out point at the
  // launch's first group and first output row.
  BytesParams params(const uint8_t* in, uint64_t row_stride, uint64_t group_stride, uint64_t valid, int g0,
                     int gcount, int dm_first, int dm_count, int dm_count_last, void* out,
                     uint64_t out_row_stride, uint64_t out_dm_rows, uint64_t out_group_rows,
                     uint64_t nout) const {
    if (dm_first % launch.dms_per_cta != 0) raise(GF_EINVAL, "DM range not aligned to the DM block");
    // bulk copies: 16-byte aligned rows
    check_arg(reinterpret_cast<uintptr_t>(in) % 16 == 0 && row_stride % 16 == 0 && group_stride % 16 == 0,
              "dedispersion input must be 16-byte aligned");
    check_arg(valid <= row_stride, "dedispersion row stride below the valid samples");
    BytesParams p{};
    p.in = in;
    p.in_row_stride = row_stride;
    p.in_group_stride = group_stride;
    p.in_valid = valid;
    p.rows_per_group = rows_per_group;
    p.total_rows = total_rows - g0 * rows_per_group;
    p.base_block_stride = static_cast<uint64_t>(rec.base_stride);
    p.base_group_stride = static_cast<uint64_t>(blocks) * p.base_block_stride;
    p.base = base_dev.as<int32_t>() + g0 * p.base_group_stride +
             static_cast<uint64_t>(dm_first / launch.dms_per_cta) * p.base_block_stride;
    p.rec_dm_stride = static_cast<uint64_t>(rec.nchunks) * rec.record_words;
    p.rec_group_stride = static_cast<uint64_t>(ndm_group) * p.rec_dm_stride;
    p.records = rec_dev.as<uint32_t>() + g0 * p.rec_group_stride + dm_first * p.rec_dm_stride;
    p.dm_count = dm_count;
    p.dm_count_last = dm_count_last;
    p.ngroups = gcount;
    p.dms_per_cta = launch.dms_per_cta;
    p.warps_per_dm = launch.warps_per_dm;
    p.chunk_rows = launch.chunk_rows;
    p.nchunks = rec.nchunks;
    p.row_bytes = launch.row_bytes;
    p.record_words = rec.record_words;
    p.cta_samples = static_cast<uint64_t>(launch.warps_per_dm) * kWarpSamples;
    p.out = out;
    p.out_row_stride = out_row_stride;
    p.out_dm_rows = out_dm_rows;
    p.out_group_rows = out_group_rows;
    p.nout = nout;
    const int dmax = std::max(dm_count, dm_count_last);
    p.nblocks = static_cast<int>(ceil_div(dmax, launch.dms_per_cta));
    p.one = 1u;
    const uint64_t ctas = ceil_div(nout, p.cta_samples) * static_cast<uint64_t>(p.nblocks);
    if (ctas >= (1ull << 31)) raise(GF_EINVAL, "dedispersion launch too large");
    p.grid_x = static_cast<uint32_t>(ctas);
    p.stages = launch.stages;
    p.stage_bytes = launch.stage_bytes;
    p.base_bytes = static_cast<uint32_t>(round_up(launch.chunk_rows * 4, 16));
    p.status = status_dev.as<uint32_t>();
    return p;
  }

  template <typename OutT>
  void run(const uint8_t* in, uint64_t row_stride, uint64_t group_stride, uint64_t valid, int g0,
           int gcount, int dm_first, int dm_count, int dm_count_last, void* out,
           uint64_t out_row_stride, uint64_t out_dm_rows, uint64_t out_group_rows, uint64_t nout,
           cudaStream_t stream) const {
    const BytesParams p = params(in, row_stride, group_stride, valid, g0, gcount, dm_first, dm_count,
                                 dm_count_last, out, out_row_stride, out_dm_rows, out_group_rows, nout);
    dim3 grid(p.grid_x, 1u, static_cast<unsigned>(gcount));
    auto kernel = dedisperse_bytes_kernel<OutT>;
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(launch.smem)),
               "cudaFuncSetAttribute(dedisperse smem)");
    kernel<<<grid, kThreads, launch.smem, stream>>>(p);
    cuda_check(cudaGetLastError(), "dedisperse_bytes_kernel launch");
  }
};

}  // namespace
}  // namespace gf

using namespace gf;

struct gf_dedisp_program {
  gf_dedisp_desc desc{};
  std::vector<double> freq;
  uint64_t nc = 0;          // selected channels
  uint64_t nout = 0;
  int32_t max_delay = 0;
  uint64_t row_stride = 0;  // staged bytes per channel row
  // brute force
  BytesStage brute;
  // subband
  uint64_t nsb = 0, sbc = 0, nnom = 0, npn = 0;
  uint64_t inter_len = 0, inter_row_stride = 0;
  bool inter_u8 = false;
  BytesStage stage1, stage2;
  std::vector<int32_t> resid;
  DeviceBlob resid_dev;
};

namespace {

void validate_desc(const gf_dedisp_desc& d) {
  // dedispersion.cpp:49-139 validation order
  check_arg(d.nsamples > 0, "dedispersion requires at least one sample");
  check_arg(d.nchans > 0, "dedispersion requires at least one channel");
  check_arg(d.frequency_mhz != nullptr, "frequency table must not be null");
  for (uint64_t c = 0; c < d.nchans; ++c)
    check_arg(std::isfinite(d.frequency_mhz[c]) && d.frequency_mhz[c] > 0.0,
              "frequency values must be finite and positive");
  check_arg(std::isfinite(d.ref_frequency_mhz) && d.ref_frequency_mhz > 0.0,
            "reference frequency must be positive");
  check_arg(std::isfinite(d.tsamp) && d.tsamp > 0.0, "tsamp must be positive");
  check_arg(std::isfinite(d.dm_low) && d.dm_low >= 0.0, "dm_low must be finite and non-negative");
  check_arg(d.ndm > 0, "dedispersion requires at least one DM");
  check_arg(std::isfinite(d.dm_step) && d.dm_step > 0.0, "dm_step must be positive");
  check_arg(d.chan_begin < d.chan_end, "channel range must be non-empty");
  check_arg(d.chan_end <= d.nchans, "channel range exceeds sample channel count");
  for (uint64_t c = d.chan_begin; c < d.chan_end; ++c)
    check_arg(d.frequency_mhz[c] <= d.ref_frequency_mhz,
              "dedispersion requires selected frequencies <= reference frequency");
  check_arg(d.nbits == 8 || d.nbits == 2, "nbits must be 8 or 2");
  check_arg(d.nbits != 2 || d.nchans % 4 == 0, "2-bit input requires nchans % 4 == 0");
  check_arg(d.algorithm == GF_DEDISP_BRUTE || d.algorithm == GF_DEDISP_SUBBAND,
            "unknown dedispersion algorithm");
  if (d.algorithm == GF_DEDISP_SUBBAND) {
    check_arg(d.subband_channels > 0, "subband_channels must be positive");
    check_arg(d.ndm_per_nominal > 0, "ndm_per_nominal must be positive");
  }
  check_arg(d.chan_end - d.chan_begin < 65536, "at most 65535 channels per program");
  check_arg(d.launch_dms_per_cta == 0 || d.launch_dms_per_cta == 1 || d.launch_dms_per_cta == 2 ||
                d.launch_dms_per_cta == 4 || d.launch_dms_per_cta == 8,
            "launch_dms_per_cta must be 0, 1, 2, 4 or 8");
  check_arg(d.launch_chunk_rows == 0 || d.launch_chunk_rows == 8 || d.launch_chunk_rows == 16 ||
                d.launch_chunk_rows == 32 || d.launch_chunk_rows == 64,
            "launch_chunk_rows must be 0, 8, 16, 32 or 64");
  check_arg(d.ndm < (1ull << 31), "too many DM trials");
}

}  // namespace

extern "C" int gf_dedisp_program_create(const gf_dedisp_desc* desc, gf_dedisp_program** out) {
  return guarded([&] {
    check_arg(desc != nullptr && out != nullptr, "null argument");
    *out = nullptr;
    validate_desc(*desc);
    DeviceGuard dg(desc->device_id);
    auto prog = std::make_unique<gf_dedisp_program>();
    gf_dedisp_program& P = *prog;
    P.desc = *desc;
    P.freq.assign(desc->frequency_mhz, desc->frequency_mhz + desc->nchans);
    P.desc.frequency_mhz = P.freq.data();
    const auto& d = P.desc;
    P.nc = d.chan_end - d.chan_begin;
    // internal/dedispersion_delay.h:129-139 multi_dm_max_delay
    const double max_dm = d.dm_low + static_cast<double>(d.ndm - 1) * d.dm_step;
    double fmin = P.freq[d.chan_begin];
    for (uint64_t c = d.chan_begin; c < d.chan_end; ++c) fmin = std::min(fmin, P.freq[c]);
    P.max_delay = delay_bins(max_dm, fmin, d.ref_frequency_mhz, d.tsamp);
    check_arg(P.max_delay >= 0, "dedispersion requires non-negative delays");
    check_arg(static_cast<uint64_t>(P.max_delay) < d.nsamples, "dedispersion valid output range is empty");
    P.nout = d.nsamples - static_cast<uint64_t>(P.max_delay);
    P.row_stride = round_up(d.nsamples, 16);
    const int nc = static_cast<int>(P.nc);
    if (d.algorithm == GF_DEDISP_BRUTE) {
      std::vector<int32_t> delays(d.ndm * P.nc);
      for (uint64_t dm = 0; dm < d.ndm; ++dm) {
        const double v = d.dm_low + static_cast<double>(dm) * d.dm_step;
        for (uint64_t c = 0; c < P.nc; ++c)
          delays[dm * P.nc + c] = delay_bins(v, P.freq[d.chan_begin + c], d.ref_frequency_mhz, d.tsamp);
      }
      P.brute.build(delays, 1, static_cast<int>(d.ndm), nc, nc, d.device_id, d.launch_dms_per_cta,
                    d.launch_chunk_rows);
    } else {
      // dedispersion.cpp:360-388 subband geometry and tables
      P.sbc = d.subband_channels;
      P.npn = d.ndm_per_nominal;
      P.nsb = ceil_div(P.nc, P.sbc);
      P.nnom = ceil_div(d.ndm, P.npn);
      std::vector<double> sbf(P.nsb);
      for (uint64_t b = 0; b < P.nsb; ++b) {
        const uint64_t begin = d.chan_begin + b * P.sbc;
        const uint64_t end = std::min(begin + P.sbc, d.chan_end);
        sbf[b] = P.freq[(begin + end - 1) / 2];
      }
      // stage 1: groups = subbands, "DMs" = nominal DMs, rows = subband channels
      const int sbc = static_cast<int>(std::min<uint64_t>(P.sbc, P.nc));
      std::vector<int32_t> coarse(P.nsb * P.nnom * sbc, 0);
      for (uint64_t b = 0; b < P.nsb; ++b)
        for (uint64_t n = 0; n < P.nnom; ++n) {
          const double nominal = d.dm_low + static_cast<double>(n * P.npn) * d.dm_step;
          for (int i = 0; i < sbc; ++i) {
            const uint64_t c = b * P.sbc + i;
            if (c >= P.nc) break;
            coarse[(b * P.nnom + n) * sbc + i] =
                delay_bins(nominal, P.freq[d.chan_begin + c], d.ref_frequency_mhz, d.tsamp);
          }
        }
      P.stage1.build(coarse, static_cast<int>(P.nsb), static_cast<int>(P.nnom), sbc, nc, d.device_id);
      // stage 2: groups = nominal DMs, "DMs" = final DMs, rows = subbands
      P.resid.assign(P.nnom * P.npn * P.nsb, 0);
      for (uint64_t dm = 0; dm < d.ndm; ++dm) {
        const uint64_t n = dm / P.npn;
        const double nominal = d.dm_low + static_cast<double>(n * P.npn) * d.dm_step;
        const double fin = d.dm_low + static_cast<double>(dm) * d.dm_step;
        for (uint64_t b = 0; b < P.nsb; ++b)
          P.resid[dm * P.nsb + b] = delay_bins(fin - nominal, sbf[b], d.ref_frequency_mhz, d.tsamp);
      }
      // the last nominal group may be partial: pad with its last DM
      for (uint64_t dm = d.ndm; dm < P.nnom * P.npn; ++dm)
        for (uint64_t b = 0; b < P.nsb; ++b) P.resid[dm * P.nsb + b] = P.resid[(d.ndm - 1) * P.nsb + b];
      for (int32_t r : P.resid) check_arg(r >= 0, "dedispersion requires non-negative delays");
      P.inter_len = d.nsamples;
      P.inter_u8 = (d.nbits == 2 ? 3ull : 255ull) * P.sbc <= 255ull;
      if (P.inter_u8) {
        P.inter_row_stride = round_up(P.inter_len, 16);
        P.stage2.build(P.resid, static_cast<int>(P.nnom), static_cast<int>(P.npn),
                       static_cast<int>(P.nsb), static_cast<int>(P.nnom * P.nsb), d.device_id);
      } else {
        P.inter_row_stride = round_up(P.inter_len, 4);
        P.resid_dev.upload(P.resid.data(), P.resid.size() * sizeof(int32_t), d.device_id);
      }
    }
    *out = prog.release();
  });
}

extern "C" int gf_dedisp_program_destroy(gf_dedisp_program* program) {
  return guarded([&] { delete program; });
}

extern "C" int gf_dedisp_program_info(const gf_dedisp_program* P, gf_dedisp_info* info) {
  return guarded([&] {
    check_arg(P != nullptr && info != nullptr, "null argument");
    std::memset(info, 0, sizeof *info);
    info->nout = P->nout;
    info->max_delay = P->max_delay;
    const uint64_t row_bytes = P->desc.nbits == 8 ? P->desc.nchans : P->desc.nchans / 4;
    info->input_bytes = row_bytes * P->desc.nsamples;
    info->staged_row_stride = P->row_stride;
    info->staged_bytes = P->row_stride * P->nc;
    if (P->desc.algorithm == GF_DEDISP_SUBBAND) {
      const uint64_t elem = P->inter_u8 ? 1 : 4;
      info->workspace_bytes = P->nnom * P->nsb * P->inter_row_stride * elem;
    }
    info->metadata_bytes = P->brute.base_dev.bytes + P->brute.rec_dev.bytes + P->stage1.base_dev.bytes +
                           P->stage1.rec_dev.bytes + P->stage2.base_dev.bytes + P->stage2.rec_dev.bytes +
                           P->resid_dev.bytes;
  });
}

namespace {

void launch_stage(const gf_dedisp_program& P, const uint8_t* in, uint64_t nsamples, uint8_t* out,
                  uint64_t t_offset, cudaStream_t stream) {
  const auto& d = P.desc;
  const uint64_t row_bytes = d.nbits == 8 ? d.nchans : d.nchans / 4;
  dim3 grid(static_cast<unsigned>(ceil_div(nsamples, 64)), static_cast<unsigned>(ceil_div(P.nc, 64)));
  if (d.nbits == 8)
    stage_kernel<8><<<grid, 256, 0, stream>>>(in, nsamples, row_bytes, static_cast<int>(d.chan_begin),
                                              static_cast<int>(P.nc), out, P.row_stride, t_offset);
  else
    stage_kernel<2><<<grid, 256, 0, stream>>>(in, nsamples, row_bytes, static_cast<int>(d.chan_begin),
                                              static_cast<int>(P.nc), out, P.row_stride, t_offset);
  cuda_check(cudaGetLastError(), "stage_kernel launch");
}

}  // namespace

extern "C" int gf_dedisp_stage(gf_dedisp_program* P, const void* dev_input, void* dev_staged, void* stream) {
  return guarded([&] {
    check_arg(P && dev_input && dev_staged, "null argument");
    DeviceGuard dg(P->desc.device_id);
    launch_stage(*P, static_cast<const uint8_t*>(dev_input), P->desc.nsamples,
                 static_cast<uint8_t*>(dev_staged), 0, as_stream(stream));
  });
}

extern "C" int gf_dedisp_stage_from_host(gf_dedisp_program* P, const void* host_input, void* dev_staged,
                                         void* dev_bounce, uint64_t bounce_bytes, void* stream) {
  return guarded([&] {
    check_arg(P && host_input && dev_staged && dev_bounce, "null argument");
    DeviceGuard dg(P->desc.device_id);
    const uint64_t row_bytes = P->desc.nbits == 8 ? P->desc.nchans : P->desc.nchans / 4;
    const uint64_t rows_per = (bounce_bytes / 2) / row_bytes;
    check_arg(rows_per >= 64, "bounce buffer too small (needs 128 time rows)");
    const uint64_t chunk = (rows_per / 64) * 64;
    auto s = as_stream(stream);
    uint8_t* bounce[2] = {static_cast<uint8_t*>(dev_bounce),
                          static_cast<uint8_t*>(dev_bounce) + chunk * row_bytes};
    const auto* host = static_cast<const uint8_t*>(host_input);
    int k = 0;
    for (uint64_t t = 0; t < P->desc.nsamples; t += chunk, k ^= 1) {
      const uint64_t n = std::min(chunk, P->desc.nsamples - t);
      cuda_check(cudaMemcpyAsync(bounce[k], host + t * row_bytes, n * row_bytes, cudaMemcpyHostToDevice, s),
                 "cudaMemcpyAsync(stage)");
      launch_stage(*P, bounce[k], n, static_cast<uint8_t*>(dev_staged), t, s);
    }
  });
}

extern "C" int gf_dedisp_run(gf_dedisp_program* P, const void* dev_staged, uint64_t dm_begin,
                             uint64_t dm_count, uint32_t* dev_out, uint64_t out_stride,
                             void* dev_workspace, void* stream) {
  return guarded([&] {
    check_arg(P && dev_staged && dev_out, "null argument");
    const auto& d = P->desc;
    check_arg(dm_count > 0 && dm_begin < d.ndm && dm_begin + dm_count <= d.ndm, "DM range out of bounds");
    check_arg(out_stride >= P->nout, "out_stride must be >= nout");
    DeviceGuard dg(d.device_id);
    auto s = as_stream(stream);
    const auto* staged = static_cast<const uint8_t*>(dev_staged);
    if (d.algorithm == GF_DEDISP_BRUTE) {
      check_arg(dm_begin % 8 == 0, "dm_begin must be a multiple of 8");
      P->brute.run<uint32_t>(staged, P->row_stride, 0, d.nsamples, 0, 1, static_cast<int>(dm_begin),
                             static_cast<int>(dm_count), static_cast<int>(dm_count), dev_out, out_stride,
                             1, 0, P->nout, s);
      return;
    }
    check_arg(dev_workspace != nullptr, "subband dedispersion needs a workspace");
    check_arg(dm_begin % P->npn == 0, "subband dm_begin must be a multiple of ndm_per_nominal");
    check_arg(dm_count % P->npn == 0 || dm_begin + dm_count == d.ndm,
              "subband dm_count must be a multiple of ndm_per_nominal");
    const uint64_t n0 = dm_begin / P->npn;
    const uint64_t n1 = ceil_div(dm_begin + dm_count, P->npn);
    // stage 1: nominal DMs [nb, ne) (block aligned) for every subband;
    // workspace row (n - nb) * nsb + b
    const auto& s1 = P->stage1;
    const uint64_t dpc1 = s1.launch.dms_per_cta;
    const uint64_t nb = (n0 / dpc1) * dpc1;
    const uint64_t ne = std::min<uint64_t>(ceil_div(n1, dpc1) * dpc1, P->nnom);
    uint8_t* inter = static_cast<uint8_t*>(dev_workspace);
    const uint64_t elem = P->inter_u8 ? 1 : 4;
    if (P->inter_u8)
      s1.run<uint8_t>(staged, P->row_stride, P->sbc * P->row_stride, d.nsamples, 0,
                      static_cast<int>(P->nsb), static_cast<int>(nb), static_cast<int>(ne - nb),
                      static_cast<int>(ne - nb), inter, P->inter_row_stride, P->nsb, 1, P->inter_len, s);
    else
      s1.run<uint32_t>(staged, P->row_stride, P->sbc * P->row_stride, d.nsamples, 0,
                       static_cast<int>(P->nsb), static_cast<int>(nb), static_cast<int>(ne - nb),
                       static_cast<int>(ne - nb), inter, P->inter_row_stride, P->nsb, 1, P->inter_len, s);
    const uint8_t* inter_n0 = inter + (n0 - nb) * P->nsb * P->inter_row_stride * elem;
    const int last_cnt = static_cast<int>(std::min<uint64_t>(P->npn, d.ndm - (n1 - 1) * P->npn));
    if (P->inter_u8) {
      // stage 2: groups = nominal DMs [n0, n1), rows = subbands
      P->stage2.run<uint32_t>(inter_n0, P->inter_row_stride, P->nsb * P->inter_row_stride, P->inter_len,
                              static_cast<int>(n0), static_cast<int>(n1 - n0), 0, static_cast<int>(P->npn),
                              last_cnt, dev_out, out_stride, 1, P->npn, P->nout, s);
    } else {
      const auto* inter32 = reinterpret_cast<const uint32_t*>(inter_n0);
      for (uint64_t n = n0; n < n1; ++n) {
        const uint64_t first = n * P->npn;
        const uint64_t cnt = std::min(P->npn, d.ndm - first);
        dim3 g2(static_cast<unsigned>(ceil_div(P->nout, 256)), static_cast<unsigned>(cnt), 1);
        subband_stage2_u32_kernel<<<g2, 256, 0, s>>>(
            inter32 + (n - n0) * P->nsb * P->inter_row_stride, P->inter_row_stride, 0, P->inter_len,
            static_cast<int>(P->nsb), P->resid_dev.as<int32_t>() + first * P->nsb, static_cast<int>(cnt),
            dev_out + (first - dm_begin) * out_stride, out_stride, P->nout);
      }
      cuda_check(cudaGetLastError(), "subband stage 2 launch");
    }
  });
}

extern "C" int gf_dedisp_check(gf_dedisp_program* P, void* stream) {
  return guarded([&] {
    check_arg(P != nullptr, "null argument");
    DeviceGuard dg(P->desc.device_id);
    auto s = as_stream(stream);
    const uint32_t v = P->brute.take_status(s) | P->stage1.take_status(s) | P->stage2.take_status(s);
    if (v & GF_STATUS_PIPELINE)
      raise(GF_ERUNTIME, "dedispersion: a shared-memory copy stage did not complete (internal error)");
  });
}

extern "C" int gf_dedisp_workspace_bytes(const gf_dedisp_program* P, uint64_t dm_count, uint64_t* bytes) {
  return guarded([&] {
    check_arg(P && bytes, "null argument");
    *bytes = 0;
    if (P->desc.algorithm != GF_DEDISP_SUBBAND) return;
    const uint64_t dpc1 = P->stage1.launch.dms_per_cta;
    const uint64_t groups = std::min<uint64_t>(ceil_div(dm_count, P->npn) + 2 * dpc1, P->nnom + dpc1);
    *bytes = groups * P->nsb * P->inter_row_stride * (P->inter_u8 ? 1 : 4);
  });
}

// Batched brute-force dedispersion: the launches of many (program, DM range)
// items as one grid of dedisperse_bytes_batch_kernel.
struct gf_dedisp_batch {
  int device = 0;
  int nitems = 0;
  uint64_t blocks = 0;
  size_t smem = 0;
  DeviceBlob items_d, begin_d;
};

extern "C" int gf_dedisp_batch_create(const gf_dedisp_batch_item* items, uint64_t nitems, gf_dedisp_batch** out) {
  return guarded([&] {
    check_arg(items && out, "null argument");
    *out = nullptr;
    check_arg(nitems > 0 && nitems < (1u << 20), "batched dedispersion takes 1 to 2^20 items");
    auto B = std::make_unique<gf_dedisp_batch>();
    std::vector<BytesParams> params;
    std::vector<uint64_t> begin;
    for (uint64_t i = 0; i < nitems; ++i) {
      const gf_dedisp_batch_item& it = items[i];
      check_arg(it.program && it.dev_staged && it.dev_out, "null argument");
      const gf_dedisp_program* P = it.program;
      const auto& d = P->desc;
      check_arg(d.algorithm == GF_DEDISP_BRUTE, "batched dedispersion takes brute-force programs");
      check_arg(i == 0 || d.device_id == B->device, "batched dedispersion items must share one device");
      B->device = d.device_id;
      check_arg(it.dm_count > 0 && it.dm_begin < d.ndm && it.dm_begin + it.dm_count <= d.ndm,
                "DM range out of bounds");
      check_arg(it.dm_begin % 8 == 0, "dm_begin must be a multiple of 8");
      check_arg(it.out_stride >= P->nout, "out_stride must be >= nout");
      const BytesParams bp = P->brute.params(static_cast<const uint8_t*>(it.dev_staged), P->row_stride, 0,
                                             d.nsamples, 0, 1, static_cast<int>(it.dm_begin),
                                             static_cast<int>(it.dm_count), static_cast<int>(it.dm_count),
                                             it.dev_out, it.out_stride, 1, 0, P->nout);
      begin.push_back(B->blocks);
      B->blocks += bp.grid_x;
      B->smem = std::max(B->smem, P->brute.launch.smem);
      params.push_back(bp);
    }
    check_arg(B->blocks < (1ull << 31), "batched dedispersion launch too large");
    B->nitems = static_cast<int>(nitems);
    DeviceGuard dg(B->device);
    B->items_d.upload(params.data(), params.size() * sizeof(BytesParams), B->device);
    B->begin_d.upload(begin.data(), begin.size() * sizeof(uint64_t), B->device);
    *out = B.release();
  });
}

extern "C" int gf_dedisp_batch_run(gf_dedisp_batch* B, void* stream) {
  return guarded([&] {
    check_arg(B != nullptr, "null argument");
    DeviceGuard dg(B->device);
    cuda_check(cudaFuncSetAttribute(dedisperse_bytes_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(B->smem)),
               "cudaFuncSetAttribute(dedisperse batch smem)");
    dedisperse_bytes_batch_kernel<<<static_cast<unsigned>(B->blocks), kThreads, B->smem, as_stream(stream)>>>(
        B->items_d.as<BytesParams>(), B->begin_d.as<uint64_t>(), B->nitems);
    cuda_check(cudaGetLastError(), "dedisperse_bytes_batch_kernel launch");
  });
}

extern "C" int gf_dedisp_batch_destroy(gf_dedisp_batch* B) {
  return guarded([&] { delete B; });
}

extern "C" int gf_dedisperse_spectrum(const void* dev_in, int32_t elem_bytes, uint64_t nsamples, uint64_t nchans,
                                      const double* freq, double dm, double ref_frequency_mhz, double tsamp,
                                      uint64_t chan_begin, uint64_t chan_end, void* dev_out, uint64_t* nout,
                                      void* stream) {
  return guarded([&] {
    check_arg(freq != nullptr && nout != nullptr, "null argument");
    check_arg(elem_bytes == 1 || elem_bytes == 2 || elem_bytes == 4, "elem_bytes must be 1, 2 or 4");
    // dedispersion.cpp:99-110 validate_single_plan
    gf_dedisp_desc d{};
    d.nsamples = nsamples;
    d.nchans = nchans;
    d.frequency_mhz = freq;
    d.dm_low = dm;
    d.dm_step = 1.0;
    d.ndm = 1;
    d.ref_frequency_mhz = ref_frequency_mhz;
    d.tsamp = tsamp;
    d.chan_begin = chan_begin;
    d.chan_end = chan_end;
    d.nbits = 8;
    d.algorithm = GF_DEDISP_BRUTE;
    check_arg(std::isfinite(dm) && dm >= 0.0, "dm must be finite and non-negative");
    validate_desc(d);
    // internal/dedispersion_delay.h:52-62,121-128
    const uint64_t nc = chan_end - chan_begin;
    std::vector<int32_t> delays(nc);
    double fmin = freq[chan_begin];
    for (uint64_t c = chan_begin; c < chan_end; ++c) {
      delays[c - chan_begin] = delay_bins(dm, freq[c], ref_frequency_mhz, tsamp);
      fmin = std::min(fmin, freq[c]);
    }
    const int32_t max_delay = delay_bins(dm, fmin, ref_frequency_mhz, tsamp);
    check_arg(max_delay >= 0, "dedispersion requires non-negative delays");
    check_arg(static_cast<uint64_t>(max_delay) < nsamples, "dedispersion valid output range is empty");
    *nout = nsamples - static_cast<uint64_t>(max_delay);
    if (dev_out == nullptr) return;
    check_arg(dev_in != nullptr, "null argument");
    auto s = as_stream(stream);
    int32_t* dd = nullptr;
    cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&dd), nc * sizeof(int32_t), s), "cudaMallocAsync(delays)");
    cuda_check(cudaMemcpyAsync(dd, delays.data(), nc * sizeof(int32_t), cudaMemcpyHostToDevice, s),
               "cudaMemcpyAsync(delays)");
    const dim3 grid(static_cast<unsigned>(ceil_div(*nout, 64)), static_cast<unsigned>(ceil_div(nc, 32)));
    check_arg(ceil_div(*nout, 64) < (1ull << 31) && ceil_div(nc, 32) < 65536, "spectrum too large");
    if (elem_bytes == 1)
      spectrum_kernel<uint8_t><<<grid, 256, 0, s>>>(static_cast<const uint8_t*>(dev_in), nchans, chan_begin,
                                                    static_cast<uint32_t>(nc), dd, *nout,
                                                    static_cast<uint8_t*>(dev_out));
    else if (elem_bytes == 2)
      spectrum_kernel<uint16_t><<<grid, 256, 0, s>>>(static_cast<const uint16_t*>(dev_in), nchans, chan_begin,
                                                     static_cast<uint32_t>(nc), dd, *nout,
                                                     static_cast<uint16_t*>(dev_out));
    else
      spectrum_kernel<float><<<grid, 256, 0, s>>>(static_cast<const float*>(dev_in), nchans, chan_begin,
                                                  static_cast<uint32_t>(nc), dd, *nout,
                                                  static_cast<float*>(dev_out));
    cuda_check(cudaGetLastError(), "spectrum_kernel launch");
    cuda_check(cudaFreeAsync(dd, s), "cudaFreeAsync(delays)");
  });
}
