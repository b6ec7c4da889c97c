// FFA search for sm_100a: per-octave downsampling, the FFA transform and
// boxcar S/N detection.
//
// Reference arithmetic (lintian233/gaffa src/gaffa):
//   downsample_weighted_sum_cpu  time_series.cpp:140-174 (sequential float sum)
//   transform_recursive / merge  ffa.cpp:127-195 (head = rows/2, tail = rest;
//     out[s][j] = head[hs][j] + tail[ts][(j + s - ts) mod bins] with
//     hs = (size_t)(float((h-1)/(n-1)) * s + 0.5f), likewise ts)
//   emit_transform_rows          ffa.cpp:203-251 (rows_eval rows of the root)
//   fill_circular_prefix / scan  ffa_detection.cpp:126-170 (sequential prefix,
//     first phase of the maximum, S/N = ((h+b)*max - b*sum) * (1/stdnoise))
// Every float operation runs in the reference's order with _rn intrinsics, so
// transform rows, prefix sums and S/N values are bit-identical to the CPU.
//
// Execution.  The recursion tree is processed by depth: every node at depth d
// splits [a, a+n) into head [a, a+n/2) and tail [a+n/2, a+n); a node of one row
// is the input row itself.  A task whose rows fit a CTA's shared memory runs in
// one CTA (all levels on chip, root rows fed straight into detection).  Larger
// tasks run on a thread-block cluster: each CTA transforms subtrees of at most
// max_rows rows on chip and writes them to the cluster's global scratch; then
// column passes of up to three levels each climb to the root.  A column block
// computes a run of rows of one node from the rows three levels down that it
// depends on (the schedules are built on the host, once per program); blocks
// of a pass are split across the cluster's CTAs, and a hardware cluster
// barrier separates passes.  The root pass is fused with detection.  Kernels
// are instantiated per NB = ceil(bins / 32) so every row loop is unrolled.
#include "common.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

namespace cg = cooperative_groups;

namespace gf {
namespace {

// Search CTAs: tasks that fit one 512-thread CTA's tiles (110 KB, two CTAs
// per SM, more items in flight) run there; larger tasks run on one
// 1024-thread CTA per SM (222 KB: larger subtrees and column blocks, 2.5 %
// faster on the survey plan than two 512-thread CTAs).  512 threads for the
// prepare pass.
constexpr int kThreads = 1024;
constexpr int kSmallThreads = 512;
constexpr int kPrepareThreads = 512;
constexpr int kMaxBins = 512;
constexpr int kMaxWidths = 64;
// Largest thread-block cluster for one (series, task).  One CTA per item:
// on the survey plan at 16 and 256 series, clusters of up to 8 CTAs (sized
// by rows) ran 11-15 % slower than independent CTAs, which need no cluster
// barriers and keep every SM busy with its own item (16-CTA clusters were
// slower still).
constexpr int kClusterSize = 1;
constexpr int kPrepareChunk = 16384;

struct TaskDev {
  uint32_t bins, rows, rows_eval, octave;
  uint64_t prep_offset;   // floats from the series' prepared block
  float inv_stdnoise;
  uint32_t ntrials;
  uint32_t trial_offset;
  uint32_t split_depth;   // depth of the on-chip subtrees (0: whole task in one CTA)
  uint32_t max_width;
  uint32_t pass_begin;    // column passes (split_depth > 0)
  uint32_t npasses;
  uint32_t member;        // observation of a batched program (0 otherwise)
};

// Batched programs: one observation's prepared series, and a run of items
// (all series of one task of one observation) in a class's item order.
struct MemberDev {
  const float* prepared;
  uint64_t prep_stride;
};

struct UnitDev {
  uint64_t item_begin;
  uint32_t task;
  uint32_t member;
};

struct TrialDev {
  float height, baseline;
  uint32_t width, reserved;
};

struct OctaveDev {
  double factor;          // 1.0 = no downsampling
  uint64_t prepared;      // prepared samples
  uint64_t offset;        // floats from the series' prepared block
};

// ---------------------------------------------------------------------------
// prepare: all octaves in one pass over the series
// ---------------------------------------------------------------------------

// first output index k with floor(k * f) >= x (k * f evaluated as the
// reference does, (double)k * factor)
__device__ __forceinline__ uint64_t first_output_at(uint64_t x, double f) {
  uint64_t k = static_cast<uint64_t>(floor(__ddiv_rn(static_cast<double>(x), f)));
  while (k > 0 && floor(__dmul_rn(static_cast<double>(k - 1), f)) >= static_cast<double>(x)) --k;
  while (floor(__dmul_rn(static_cast<double>(k), f)) < static_cast<double>(x)) ++k;
  return k;
}

// One member's series in a prepare launch.
struct PrepareItem {
  const float* series;
  uint64_t stride, n;
  const double* stats;      // null: no normalisation
  const OctaveDev* octaves;
  int32_t noct;
  uint32_t nseries;
  uint64_t halo;
  float* prepared;
  uint64_t prep_stride;
};

// The items of a prepare launch: a device table (batched) or one by value.
struct PrepareTable {
  const PrepareItem* items;  // null: `one` only
  const uint64_t* begin;     // first CTA of each item
  int32_t nitems;
  PrepareItem one;
};

uint64_t prepare_ctas(const PrepareItem& it) { return ceil_div(it.n, kPrepareChunk) * it.nseries; }

template <bool Batched>
__global__ void __launch_bounds__(kPrepareThreads) prepare_kernel(const __grid_constant__ PrepareTable tab) {
  extern __shared__ float xs[];
  __shared__ uint64_t kb[32], cnt_prefix[33];
  __shared__ PrepareItem sit;
  __shared__ uint32_t sloc;
  // a single-item launch reads the parameter; a batched one shares thread 0's
  // lookup (the last item starting at or before the CTA)
  uint32_t local = blockIdx.x;
  if (Batched) {
    if (threadIdx.x == 0) {
      const uint64_t b = blockIdx.x;
      int lo = 0, hi = tab.nitems;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tab.begin[mid] <= b) lo = mid; else hi = mid;
      }
      sit = tab.items[lo];
      sloc = static_cast<uint32_t>(b - tab.begin[lo]);
    }
    __syncthreads();
    local = sloc;
  }
  const PrepareItem& it = Batched ? sit : tab.one;
  const uint64_t n = it.n, halo = it.halo;
  const OctaveDev* octaves = it.octaves;
  const int noct = it.noct;
  uint64_t s, c0;
  if (Batched) {
    const uint32_t xblocks = static_cast<uint32_t>(ceil_div(n, kPrepareChunk));
    s = local / xblocks;
    c0 = static_cast<uint64_t>(local % xblocks) * kPrepareChunk;
  } else {
    s = blockIdx.y;
    c0 = static_cast<uint64_t>(blockIdx.x) * kPrepareChunk;
  }
  const float* __restrict__ row = it.series + s * it.stride;
  // the series' mean and 1/stddev, loaded once (scale 0: a rejected series)
  const bool norm = it.stats != nullptr;
  const double mean = norm ? __ldg(it.stats + 2 * s) : 0.0;
  const double scale = norm ? __ldg(it.stats + 2 * s + 1) : 1.0;
  const uint64_t span = umin64(kPrepareChunk + halo, n - c0);
  for (uint64_t i = threadIdx.x; i < span; i += kPrepareThreads) {
    const float y = __ldg(row + c0 + i);
    xs[i] = !norm ? y : scale == 0.0 ? 0.0f : static_cast<float>(__dmul_rn(__dsub_rn(static_cast<double>(y), mean), scale));
  }
  if (threadIdx.x == 0) {
    cnt_prefix[0] = 0;
    for (int o = 0; o < noct; ++o) {
      const OctaveDev oc = octaves[o];
      uint64_t b, e;
      if (oc.factor == 1.0) {
        b = c0;
        e = umin64(c0 + kPrepareChunk, oc.prepared);
      } else {
        b = first_output_at(c0, oc.factor);
        e = umin64(first_output_at(c0 + kPrepareChunk, oc.factor), oc.prepared);
      }
      if (e < b) e = b;
      kb[o] = b;
      cnt_prefix[o + 1] = cnt_prefix[o] + (e - b);
    }
  }
  __syncthreads();
  const uint64_t total = cnt_prefix[noct];
  float* __restrict__ out_row = it.prepared + s * it.prep_stride;
  const double last_index = static_cast<double>(n - 1);
  for (uint64_t idx = threadIdx.x; idx < total; idx += kPrepareThreads) {
    int o = 0;
    while (cnt_prefix[o + 1] <= idx) ++o;
    const OctaveDev oc = octaves[o];
    const uint64_t k = kb[o] + (idx - cnt_prefix[o]);
    float sum;
    if (oc.factor == 1.0) {
      sum = xs[k - c0];
    } else {
      const double start = __dmul_rn(static_cast<double>(k), oc.factor);
      const double end = __dadd_rn(start, oc.factor);
      const uint64_t first = static_cast<uint64_t>(floor(start));
      const double fe = floor(end);
      const uint64_t last = static_cast<uint64_t>(fe < last_index ? fe : last_index);
      const float w0 = static_cast<float>(__dsub_rn(static_cast<double>(first + 1), start));
      const float w1 = static_cast<float>(__dsub_rn(end, static_cast<double>(last)));
      const float* x = xs + (first - c0);
      const uint64_t len = last - first;
      sum = __fmul_rn(w0, x[0]);
      for (uint64_t i = 1; i < len; ++i) sum = __fadd_rn(sum, x[i]);
      sum = __fadd_rn(sum, __fmul_rn(w1, x[len]));
    }
    out_row[oc.offset + k] = sum;
  }
}

// ---------------------------------------------------------------------------
// FFA tree evaluation
// ---------------------------------------------------------------------------
//
// A level of the tree is a list of rows, each produced by one MetaEntry:
//   MERGE  out = prev[a] + roll_left(prev[b], roll mod bins)   (ffa.cpp:110-171)
//   CARRY  out = prev[a]              (a one-row node carried up unchanged)
// Rows of a level live in one of two shared-memory buffers (pitch = bins|1);
// levels alternate buffers, so each level costs one __syncthreads.  Every
// loop over the bins of a row is unrolled for NB = ceil(bins / 32) (the
// kernels are instantiated per NB), so a merged element costs two shared
// loads, one add and one shared store.

enum : uint16_t { kMerge = 0, kCarry = 1 };

struct __align__(8) MetaEntry {
  uint16_t op, a, b, roll;
};

struct Node {
  uint32_t a, n, depth;
};

// The node at depth `depth` containing row r (stops at one-row nodes).
__device__ __forceinline__ Node node_of(uint32_t r, uint32_t n, uint32_t depth) {
  Node nd{0u, n, 0u};
  while (nd.depth < depth && nd.n > 1) {
    const uint32_t h = nd.n >> 1;
    if (r - nd.a < h) {
      nd.n = h;
    } else {
      nd.a += h;
      nd.n -= h;
    }
    ++nd.depth;
  }
  return nd;
}

// Node `index` (bits read MSB first, 0 = head) at depth `depth`.
__host__ __device__ __forceinline__ Node node_at(uint32_t index, uint32_t n, uint32_t depth) {
  Node nd{0u, n, depth};
  for (uint32_t b = depth; b-- > 0;) {
    const uint32_t h = nd.n >> 1;
    if ((index >> b) & 1u) {
      nd.a += h;
      nd.n -= h;
    } else {
      nd.n = h;
    }
  }
  return nd;
}

// ffa.cpp:153-171: hs = (size_t)(float((h-1)/(n-1)) * s + 0.5f), likewise ts
__device__ __forceinline__ float shift_scale(uint32_t part, uint32_t n) {
  return __fdiv_rn(static_cast<float>(part - 1), static_cast<float>(n - 1));
}
__device__ __forceinline__ uint32_t scaled_shift(float scale, uint32_t s) {
  return static_cast<uint32_t>(__fadd_rn(__fmul_rn(scale, static_cast<float>(s)), 0.5f));
}

__host__ __device__ __forceinline__ uint32_t tree_depth(uint32_t n) {
  uint32_t d = 0;
  while (n > 1) { n = (n + 1) >> 1; ++d; }
  return d;
}

// A column block of a pass (built on the host): rows [s0, s1) of one node X
// at depth dx, evaluated from the rows of depth dx + levels that they depend
// on.  Level k (0 = X) holds count[k] rows; the bottom level is loaded from
// the pass's source scratch as up to 8 runs of consecutive task rows.
struct ColBlock {
  uint32_t meta;          // first merge entry: levels-1, ..., 0 back to back
  uint32_t out_row;       // final pass: shift of the first root row; else task row of the first output row
  uint16_t count[4];      // rows at relative level 0 .. levels
  uint16_t run_off[8];    // bottom level: buffer row where each run starts
  uint16_t run_row[8];    // bottom level: task row where each run starts
  uint8_t levels, final_pass, nruns, reserved;
  uint32_t pad[3];
};
static_assert(sizeof(ColBlock) == 64, "ColBlock is 16 words");

struct PassDev {
  uint32_t block_begin, nblocks;
};

// Search-path device functions take the CTA size T (512 or 1024 threads).

// Dynamic shared memory of the search kernel: two ColBlock headers, the
// staged schedule, then two row buffers.
extern __shared__ __align__(16) float g_smem[];

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// One level: out row q (q < nrows) from `prev` by meta[q].  A warp per row,
// lane j handles bins j, j+32, ...; only the last iteration can be partial.
// The tail row is read at k = (j + roll) mod bins, computed branch-free as
// min(k, k - bins) in unsigned arithmetic (k < 2 bins).
template <int NB, int T>
__device__ __forceinline__ void merge_level(const MetaEntry* meta, uint32_t nrows, const float* prev, float* out,
                                            uint32_t pitch, uint32_t bins) {
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool last_ok = lane + 32u * (NB - 1) < bins;
  for (uint32_t q = warp; q < nrows; q += T / 32) {
    const MetaEntry m = meta[q];
    float* o = out + q * pitch + lane;
    const float* h = prev + m.a * pitch + lane;
    if (m.op == kMerge) {
      uint32_t r = m.roll;
      if (r >= bins) r %= bins;
      const uint32_t k0 = lane + r;       // < 2 bins
      const uint32_t k1 = k0 - bins;      // wraps when k0 < bins
      const float* t = prev + m.b * pitch;
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        if (i < NB - 1 || last_ok) {
          const uint32_t k = umin32(k0 + 32u * i, k1 + 32u * i);
          o[32 * i] = __fadd_rn(h[32 * i], t[k]);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < NB; ++i)
        if (i < NB - 1 || last_ok) o[32 * i] = h[32 * i];
    }
  }
}

// rows [0, n) of read-only global `src` (row length bins) into smem, async
template <int NB, int T>
__device__ __forceinline__ void load_rows_async(const float* src, uint32_t n, uint32_t bins, float* out,
                                                uint32_t pitch) {
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool last_ok = lane + 32u * (NB - 1) < bins;
  for (uint32_t q = warp; q < n; q += T / 32) {
    const float* g = src + static_cast<uint64_t>(q) * bins + lane;
    float* o = out + q * pitch + lane;
#pragma unroll
    for (int i = 0; i < NB; ++i)
      if (i < NB - 1 || last_ok) cp_async4(o + 32 * i, g + 32 * i);
  }
}

template <int NB, int T>
__device__ __forceinline__ void store_rows(const float* in, uint32_t pitch, uint32_t n, uint32_t bins, float* dst) {
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool last_ok = lane + 32u * (NB - 1) < bins;
  for (uint32_t q = warp; q < n; q += T / 32) {
    float* g = dst + static_cast<uint64_t>(q) * bins + lane;
    const float* s = in + q * pitch + lane;
#pragma unroll
    for (int i = 0; i < NB; ++i)
      if (i < NB - 1 || last_ok) __stcg(g + 32 * i, s[32 * i]);
  }
}

// ---------------------------------------------------------------------------
// detection
// ---------------------------------------------------------------------------

struct DetectArgs {
  const TrialDev* trials;
  uint32_t ntrials, max_width, bins;
  float inv_stdnoise, threshold;
  uint32_t series, task;
  gf_peak_record* peaks;
  uint64_t capacity;
  unsigned long long* counters;
};

// order-preserving map of finite floats to unsigned keys (for redux.sync)
__device__ __forceinline__ uint32_t float_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// rows[i] (pitch `pitch`) hold root rows shift0 + i, i < count.  Prefix sums
// are sequential per row (one thread per row, ffa_detection.cpp:126-139).
// Then a warp per row: lane j holds c[j + 32i] and, for every width, takes
// the maximum of c[ph + w] - c[ph] over its phases; redux.sync gives the
// row maximum, from which S/N follows (:141-170).  Only when S/N passes the
// threshold is the first phase attaining the maximum looked up (the
// reference's strict '>' scan keeps the first maximum), and a peak appended.
template <int NB, int T>
__device__ void detect_rows(const float* rows, uint32_t pitch, uint32_t count, uint32_t shift0, float* cp,
                            uint32_t cp_pitch, const DetectArgs& a) {
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bins = a.bins;
  if (threadIdx.x < count) {
    const float* prof = rows + threadIdx.x * pitch;
    float* c = cp + threadIdx.x * cp_pitch;
    float acc = 0.0f;
    c[0] = 0.0f;
    // loads of the next 8 samples overlap the current 8-add chain
    float cur[8], nxt[8];
    const uint32_t nfull = bins & ~7u;
#pragma unroll
    for (int j = 0; j < 8; ++j) cur[j] = (static_cast<uint32_t>(j) < nfull) ? prof[j] : 0.0f;
    for (uint32_t i = 0; i < nfull; i += 8) {
#pragma unroll
      for (int j = 0; j < 8; ++j) nxt[j] = (i + 8 + j < nfull) ? prof[i + 8 + j] : 0.0f;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        acc = __fadd_rn(acc, cur[j]);
        c[i + j + 1] = acc;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) cur[j] = nxt[j];
    }
    for (uint32_t i = nfull; i < bins; ++i) {
      acc = __fadd_rn(acc, prof[i]);
      c[i + 1] = acc;
    }
    for (uint32_t i = 0; i < a.max_width; ++i) {
      acc = __fadd_rn(acc, prof[i]);
      c[bins + i + 1] = acc;
    }
  }
  __syncthreads();
  const bool last_ok = lane + 32u * (NB - 1) < bins;
  for (uint32_t r = warp; r < count; r += T / 32) {
    const float* c = cp + r * cp_pitch + lane;
    float base[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) base[i] = (i < NB - 1 || last_ok) ? c[32 * i] : 0.0f;
    const float psum = cp[r * cp_pitch + bins];
    for (uint32_t k = 0; k < a.ntrials; ++k) {
      const TrialDev tr = a.trials[k];
      const float* cw = c + tr.width;
      float best = -INFINITY;
#pragma unroll
      for (int i = 0; i < NB; ++i)
        if (i < NB - 1 || last_ok) best = fmaxf(best, __fsub_rn(cw[32 * i], base[i]));
      // S/N is monotone in the boxcar sum, so the row passes the threshold
      // exactly when some lane's own maximum does
      const float lane_snr = __fmul_rn(
          __fsub_rn(__fmul_rn(__fadd_rn(tr.height, tr.baseline), best), __fmul_rn(tr.baseline, psum)),
          a.inv_stdnoise);
      if (__any_sync(0xffffffffu, lane_snr >= a.threshold)) {
        const float maxv = key_float(__reduce_max_sync(0xffffffffu, float_key(best)));
        const float snr = __fmul_rn(
            __fsub_rn(__fmul_rn(__fadd_rn(tr.height, tr.baseline), maxv), __fmul_rn(tr.baseline, psum)),
            a.inv_stdnoise);
        uint32_t first = 0xffffffffu;
#pragma unroll
        for (int i = NB - 1; i >= 0; --i)
          if ((i < NB - 1 || last_ok) && __fsub_rn(cw[32 * i], base[i]) == maxv) first = lane + 32u * i;
        const uint32_t ph = __reduce_min_sync(0xffffffffu, first);
        if (lane == 0) {
          const unsigned long long slot = atomicAdd(a.counters, 1ull);
          if (slot < a.capacity) {
            gf_peak_record rec;
            rec.series = a.series;
            rec.task = a.task;
            rec.shift = shift0 + r;
            rec.phase = static_cast<uint16_t>(ph);
            rec.width_index = static_cast<uint16_t>(k);
            rec.snr = snr;
            rec.reserved = 0u;
            a.peaks[slot] = rec;
          } else {
            atomicOr(reinterpret_cast<unsigned int*>(a.counters + 1), GF_STATUS_PEAK_OVERFLOW);
          }
        }
      }
    }
  }
  __syncthreads();
}

struct SearchParams {
  const float* prepared;
  uint64_t prep_stride;
  const TaskDev* tasks;
  const TrialDev* trials;
  const MetaEntry* sub_meta;    // subtree schedules by size
  const uint32_t* sub_offset;   // [max_rows + 1]
  const MetaEntry* col_meta;    // column-block merge entries
  const ColBlock* blocks;       // column blocks, pass by pass
  const PassDev* passes;
  const uint32_t* item_tasks;   // task indices of this launch's class
  uint32_t nitem_tasks;
  uint32_t nseries;
  const UnitDev* units;         // batched programs: item runs of this class (else null)
  const MemberDev* members;
  uint32_t nunits;
  uint64_t nitems;
  float threshold;
  gf_peak_record* peaks;
  uint64_t capacity;
  unsigned long long* counters;
  float* scratch;               // per cluster: 2 * scratch_elems floats
  uint64_t scratch_elems;
  uint32_t pitch;               // shared-memory row pitch (max bins | 1)
  uint32_t max_rows;            // rows per shared-memory buffer
  uint32_t front;               // floats before the first row buffer
};

__device__ __forceinline__ DetectArgs make_detect(const SearchParams& p, const TaskDev& t, uint32_t series,
                                                  uint32_t task) {
  DetectArgs da;
  da.trials = p.trials + t.trial_offset;
  da.ntrials = t.ntrials;
  da.max_width = t.max_width;
  da.bins = t.bins;
  da.inv_stdnoise = t.inv_stdnoise;
  da.threshold = p.threshold;
  da.series = series;
  da.task = task;
  da.peaks = p.peaks;
  da.capacity = p.capacity;
  da.counters = p.counters;
  return da;
}

// Evaluates a whole subtree of n <= max_rows rows (pointer `src` = its first
// input row) from its input rows up to relative level `stop` (0: the
// subtree root).  The subtree's schedule (depth x n entries, level depth-1
// first) is left in cmeta.  Returns the buffer holding level `stop`.
template <int NB, int T>
__device__ float* eval_subtree(const SearchParams& p, const float* src, uint32_t n, uint32_t bins, uint32_t stop,
                               float* buf0, float* buf1, MetaEntry* cmeta) {
  const uint32_t pitch = p.pitch;
  const uint32_t md = tree_depth(n);
  const MetaEntry* table = p.sub_meta + p.sub_offset[n];
  for (uint32_t e = threadIdx.x; e < md * n; e += T) cp_async8(cmeta + e, table + e);
  load_rows_async<NB, T>(src, n, bins, (md & 1) ? buf1 : buf0, pitch);
  cp_async_wait_all();
  __syncthreads();
  for (int l = static_cast<int>(md) - 1; l >= static_cast<int>(stop); --l) {
    merge_level<NB, T>(cmeta + (md - 1 - l) * n, n, ((l + 1) & 1) ? buf1 : buf0, (l & 1) ? buf1 : buf0, pitch, bins);
    __syncthreads();
  }
  return (stop & 1) ? buf1 : buf0;
}

// Column block `hb`: stages its merge entries, loads its bottom rows from
// `src` (scratch written by the cluster's CTAs in the previous phase),
// evaluates its levels.  The output rows (hb.count[0]) end in buf0.
template <int NB, int T>
__device__ void eval_block(const SearchParams& p, const ColBlock& hb, const float* src, uint32_t bins, float* buf0,
                           float* buf1, MetaEntry* cmeta) {
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t pitch = p.pitch;
  const uint32_t K = hb.levels;
  uint32_t nmeta = 0;
  for (uint32_t k = 0; k < K; ++k) nmeta += hb.count[k];
  const MetaEntry* gm = p.col_meta + hb.meta;  // 16-byte aligned, padded to an even count
  for (uint32_t e = 2 * threadIdx.x; e < nmeta; e += 2 * T) cp_async16(cmeta + e, gm + e);
  float* bottom = (K & 1) ? buf1 : buf0;
  const uint32_t nb = hb.count[K];
  const uint32_t nruns = hb.nruns;
  const bool last_ok = lane + 32u * (NB - 1) < bins;
  // Bottom rows: async copies, all in flight at once.  The rows were written
  // by other CTAs of the cluster before the cluster barrier, whose acquire
  // makes them visible to these (L1-allocating) reads.
  for (uint32_t q = warp; q < nb; q += T / 32) {
    uint32_t j = 0;  // run holding buffer row q (runs ascend in run_off)
#pragma unroll
    for (uint32_t r = 1; r < 8; ++r) j += (r < nruns && hb.run_off[r] <= q) ? 1u : 0u;
    const float* g = src + static_cast<uint64_t>(hb.run_row[j] + (q - hb.run_off[j])) * bins + lane;
    float* o = bottom + q * pitch + lane;
#pragma unroll
    for (int i = 0; i < NB; ++i)
      if (i < NB - 1 || last_ok) cp_async4(o + 32 * i, g + 32 * i);
  }
  cp_async_wait_all();
  __syncthreads();
  uint32_t off = 0;
  for (int k = static_cast<int>(K) - 1; k >= 0; --k) {
    merge_level<NB, T>(cmeta + off, hb.count[k], ((k + 1) & 1) ? buf1 : buf0, (k & 1) ? buf1 : buf0, pitch, bins);
    off += hb.count[k];
    __syncthreads();
  }
}

// 64-byte header, async (completes at the next cp_async_wait_all)
__device__ __forceinline__ void load_header(ColBlock* dst, const ColBlock* src) {
  if (threadIdx.x < 4)
    cp_async16(reinterpret_cast<uint4*>(dst) + threadIdx.x, reinterpret_cast<const uint4*>(src) + threadIdx.x);
}

// One (series, task) per cluster (cluster size 1, 2, 4 or 8); items are
// task-major so the series of one task run together.  NB = ceil(bins/32)
// of every task of the launch.
template <int NB, int T>
__global__ void __launch_bounds__(T, T <= 512 ? 2 : 1) ffa_search_kernel(SearchParams p) {
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t cs = cluster.num_blocks();
  const uint32_t rank = cluster.block_rank();
  const uint32_t cid = blockIdx.x / cs;
  const uint32_t nclusters = gridDim.x / cs;
  const uint32_t pitch = p.pitch;
  ColBlock* hdr = reinterpret_cast<ColBlock*>(g_smem);
  MetaEntry* cmeta = reinterpret_cast<MetaEntry*>(g_smem + 32);
  float* buf0 = g_smem + p.front;
  float* buf1 = buf0 + p.max_rows * pitch;
  float* q0 = p.scratch ? p.scratch + static_cast<uint64_t>(cid) * 2 * p.scratch_elems : nullptr;
  float* q1 = q0 ? q0 + p.scratch_elems : nullptr;
  const uint64_t nitems = p.units ? p.nitems : static_cast<uint64_t>(p.nseries) * p.nitem_tasks;
  for (uint64_t item = cid; item < nitems; item += nclusters) {
    uint32_t task, series;
    const float* base;
    uint64_t stride;
    if (p.units) {
      // last run starting at or before the item (runs in item order)
      uint32_t lo = 0, hi = p.nunits;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (p.units[mid].item_begin <= item) lo = mid; else hi = mid;
      }
      const UnitDev u = p.units[lo];
      task = u.task;
      series = static_cast<uint32_t>(item - u.item_begin);
      base = p.members[u.member].prepared;
      stride = p.members[u.member].prep_stride;
    } else {
      task = p.item_tasks[item / p.nseries];
      series = static_cast<uint32_t>(item % p.nseries);
      base = p.prepared;
      stride = p.prep_stride;
    }
    const TaskDev t = p.tasks[task];
    const float* input = base + series * stride + t.prep_offset;
    const uint32_t bins = t.bins;
    const DetectArgs da = make_detect(p, t, series, task);
    const uint32_t cp_pitch = (bins + t.max_width + 2) | 1u;
    const uint32_t dS = t.split_depth;
    if (dS == 0) {
      // whole task on chip: levels below the root, then root rows in batches
      if (t.rows == 1) {
        load_rows_async<NB, T>(input, 1, bins, buf0, pitch);
        cp_async_wait_all();
        __syncthreads();
        detect_rows<NB, T>(buf0, pitch, 1, 0, buf1, cp_pitch, da);
        __syncthreads();  // the width scans read buf1 until here; the next item loads into it
        continue;
      }
      float* lvl1 = eval_subtree<NB, T>(p, input, t.rows, bins, 1, buf0, buf1, cmeta);
      float* other = lvl1 == buf0 ? buf1 : buf0;
      const uint32_t md = tree_depth(t.rows);
      const MetaEntry* root = cmeta + (md - 1) * t.rows;
      const uint32_t batch = umin32(T, (p.max_rows * pitch) / (pitch + cp_pitch));
      for (uint32_t b0 = 0; b0 < t.rows_eval; b0 += batch) {
        const uint32_t cnt = umin32(batch, t.rows_eval - b0);
        merge_level<NB, T>(root + b0, cnt, lvl1, other, pitch, bins);
        __syncthreads();
        detect_rows<NB, T>(other, pitch, cnt, b0, other + batch * pitch, cp_pitch, da);
      }
      __syncthreads();  // the last width scans read `other` until here; the next item loads into it
      continue;
    }
    // 1. subtrees at depth dS, on chip, into scratch q0
    const uint32_t nsub = 1u << dS;
    for (uint32_t sub = rank; sub < nsub; sub += cs) {
      const Node nd = node_at(sub, t.rows, dS);
      const float* res = eval_subtree<NB, T>(p, input + static_cast<uint64_t>(nd.a) * bins, nd.n, bins, 0, buf0, buf1,
                                          cmeta);
      store_rows<NB, T>(res, pitch, nd.n, bins, q0 + static_cast<uint64_t>(nd.a) * bins);
      __syncthreads();
    }
    cluster.sync();
    // 2. column passes up to the root (the last one fused with detection)
    float* src = q0;
    float* dst = q1;
    for (uint32_t ps = 0; ps < t.npasses; ++ps) {
      const PassDev pd = p.passes[t.pass_begin + ps];
      const ColBlock* blocks = p.blocks + pd.block_begin;
      if (rank < pd.nblocks) load_header(&hdr[0], blocks + rank);
      cp_async_wait_all();
      __syncthreads();
      uint32_t it = 0;
      for (uint32_t u = rank; u < pd.nblocks; u += cs, ++it) {
        const ColBlock& hb = hdr[it & 1];
        if (u + cs < pd.nblocks) load_header(&hdr[(it + 1) & 1], blocks + u + cs);
        eval_block<NB, T>(p, hb, src, bins, buf0, buf1, cmeta);
        if (hb.final_pass) {
          detect_rows<NB, T>(buf0, pitch, hb.count[0], hb.out_row, buf1, cp_pitch, da);
          __syncthreads();  // the width scans read buf1 until here; the next block may load into it
        } else {
          store_rows<NB, T>(buf0, pitch, hb.count[0], bins, dst + static_cast<uint64_t>(hb.out_row) * bins);
          __syncthreads();
        }
      }
      cluster.sync();
      float* tmp = src;
      src = dst;
      dst = tmp;
    }
  }
}

// Materialised transform for tests and the block API: one depth per launch.
__global__ void __launch_bounds__(kThreads) ffa_level_kernel(const float* __restrict__ input, uint32_t rows,
                                                             uint32_t bins, uint32_t depth, const float* prev,
                                                             float* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t r = blockIdx.x * (kThreads / 32) + warp;
  if (r >= rows) return;
  const Node nd = node_of(r, rows, depth);
  if (nd.depth != depth || nd.n < 2) {
    // a one-row node carries its input row up to the next level
    for (uint32_t j = lane; j < bins; j += 32)
      out[static_cast<uint64_t>(r) * bins + j] = input[static_cast<uint64_t>(r) * bins + j];
    return;
  }
  const uint32_t h = nd.n >> 1, t = nd.n - h;
  const uint32_t s = r - nd.a;
  const uint32_t hs = scaled_shift(shift_scale(h, nd.n), s), ts = scaled_shift(shift_scale(t, nd.n), s);
  const float* head = (h == 1 ? input : prev) + static_cast<uint64_t>(nd.a + hs) * bins;
  const float* tail = (t == 1 ? input : prev) + static_cast<uint64_t>(nd.a + h + ts) * bins;
  const uint32_t roll = (s - ts) % bins;
  for (uint32_t j = lane; j < bins; j += 32) {
    uint32_t k = j + roll;
    if (k >= bins) k -= bins;
    out[static_cast<uint64_t>(r) * bins + j] = __fadd_rn(head[j], tail[k]);
  }
}

using SearchKernel = void (*)(SearchParams);

// ffa_search_kernel<NB, T> for NB = 1 .. 16 (bins <= 512), T = 512 or 1024
template <int T>
SearchKernel search_kernel_table(uint32_t nb) {
  static const SearchKernel table[16] = {
      ffa_search_kernel<1, T>,  ffa_search_kernel<2, T>,  ffa_search_kernel<3, T>,  ffa_search_kernel<4, T>,
      ffa_search_kernel<5, T>,  ffa_search_kernel<6, T>,  ffa_search_kernel<7, T>,  ffa_search_kernel<8, T>,
      ffa_search_kernel<9, T>,  ffa_search_kernel<10, T>, ffa_search_kernel<11, T>, ffa_search_kernel<12, T>,
      ffa_search_kernel<13, T>, ffa_search_kernel<14, T>, ffa_search_kernel<15, T>, ffa_search_kernel<16, T>};
  return table[nb - 1];
}

SearchKernel search_kernel_for(uint32_t nb, int threads) {
  return threads == kSmallThreads ? search_kernel_table<kSmallThreads>(nb) : search_kernel_table<kThreads>(nb);
}

}  // namespace
}  // namespace gf

using namespace gf;

// Shared-memory geometry of the launches of one NB = ceil(bins/32): row pitch,
// rows per buffer, column-block sizes and the dynamic shared memory.
struct FfaGeometry {
  uint32_t pitch = 0, max_rows = 0, block_rows = 0, final_rows = 0, levels = 0, front = 0;
  uint32_t cp_rows = 0;        // root rows whose prefix sums fit one row buffer
  size_t smem_bytes = 0;
};

struct FfaClass {
  int cluster = 1;             // CTAs cooperating on one (series, task)
  int threads = kThreads;      // CTA size (kSmallThreads or kThreads)
  uint32_t nb = 1;             // ceil(bins / 32) of every task of the class
  SearchKernel kernel = nullptr;
  std::vector<uint32_t> tasks; // largest first
  uint64_t max_elems = 0;      // rows * bins of the largest task (scratch per cluster)
  int nclusters = 0;           // resident clusters
  DeviceBlob tasks_d;
  std::vector<UnitDev> units;  // batched programs: one item run per task, in task order
  uint64_t nitems = 0;
  DeviceBlob units_d;
};

// One observation's plan inside a program; a single-plan program has one.
struct FfaMember {
  uint64_t nsamples = 0;
  uint64_t prep_stride = 0;    // prepared floats per series (all octaves)
  uint64_t halo = 0;
  uint64_t nseries = 0;        // series per search (batched programs)
  uint32_t task_begin = 0, ntasks = 0, max_width = 0;
  std::vector<uint64_t> widths;
  std::vector<OctaveDev> octaves;
  DeviceBlob octaves_d;
  const float* prepared = nullptr;  // bound prepared series (batched programs)
};

struct gf_ffa_program {
  int device = 0;
  bool batched = false;
  bool bound = false;
  std::vector<gf_ffa_task> tasks;        // every member's tasks, member by member
  std::vector<uint32_t> task_member;
  std::vector<FfaMember> members;
  std::vector<TaskDev> task_dev;
  std::vector<TrialDev> trial_dev;
  std::vector<MetaEntry> sub_meta;
  std::vector<uint32_t> sub_offset;
  std::vector<MetaEntry> col_meta;
  std::vector<ColBlock> blocks;
  std::vector<PassDev> passes;
  std::vector<FfaClass> classes;
  uint32_t max_bins = 0, max_width = 0;
  FfaGeometry geo[2][17];      // by CTA size (0: kSmallThreads, 1: kThreads) and NB (1..16)
  uint64_t max_series = 0;
  uint64_t scratch_floats = 0;
  DeviceBlob tasks_d, trials_d, sub_meta_d, sub_offset_d, col_meta_d, blocks_d, passes_d, members_d;
  // batched prepare of every member (gf_ffa_batch_bind_series)
  DeviceBlob prepare_items_d, prepare_begin_d;
  uint64_t prepare_ctas_total = 0, prepare_halo = 0;
};

namespace {

uint64_t downsampled_size_checked(uint64_t n, double f) {
  check_arg(n > 0, "time series must not be empty");
  check_arg(std::isfinite(f) && f > 1.0 && f <= static_cast<double>(n),
            "downsample factor must satisfy 1 < factor <= nsamples");
  return static_cast<uint64_t>(std::floor(static_cast<double>(n) / f));
}

double downsampled_variance_host(uint64_t n, double f) {
  // time_series.cpp:124-138
  const uint64_t m = downsampled_size_checked(n, f);
  const double whole = std::floor(f);
  const double frac = f - whole;
  const double span = static_cast<double>(m) * frac;
  if (span > 1.0) return f - 1.0 / 3.0;
  return std::pow(whole - 1.0, 2.0) + (2.0 / 3.0) * std::pow(span, 2.0) - span + 1.0;
}

float task_stdnoise(const gf_ffa_task& t) {
  // ffa_detection.cpp:256-264
  double var = 1.0;
  if (t.downsample_factor != 1.0) var = downsampled_variance_host(t.input_nsamples, t.downsample_factor);
  return static_cast<float>(std::sqrt(static_cast<double>(t.rows) * var));
}

void validate_task(const gf_ffa_task& t, uint64_t n) {
  // ffa_executor.cpp:196-245
  check_arg(t.input_nsamples == n, "FFA executor task input_nsamples must match time series size");
  check_arg(std::isfinite(t.downsample_factor) && t.downsample_factor >= 1.0,
            "FFA executor task downsample_factor must be finite and >= 1");
  check_arg(t.effective_tsamp > 0.0 && std::isfinite(t.effective_tsamp),
            "FFA executor task effective_tsamp must be finite and > 0");
  check_arg(t.bins > 1, "FFA executor task bins must be > 1");
  check_arg(t.rows > 0, "FFA executor task rows must be > 0");
  check_arg(t.rows_eval > 0 && t.rows_eval <= t.rows,
            "FFA executor task rows_eval must satisfy 0 < rows_eval <= rows");
  check_arg(t.prepared_nsamples > 0, "FFA executor task prepared_nsamples must be > 0");
  check_arg(t.rows * t.bins <= t.prepared_nsamples, "FFA executor task rows * bins must be <= prepared_nsamples");
  if (t.downsample_factor == 1.0) {
    check_arg(t.prepared_nsamples == n, "FFA executor no-downsample task prepared_nsamples must match input size");
  } else {
    check_arg(t.prepared_nsamples == downsampled_size_checked(n, t.downsample_factor),
              "FFA executor task prepared_nsamples must match downsampled_size");
  }
}

uint32_t host_tree_depth(uint64_t n) {
  uint32_t d = 0;
  while (n > 1) { n = (n + 1) / 2; ++d; }
  return d;
}

// Merge schedule of a subtree of n rows (ffa.cpp:127-195 recursion, by
// depth): for level l = depth-1 .. 0 and each row r, either MERGE(head row,
// tail row, roll) from level l+1 or CARRY(r) for rows of one-row nodes.
void build_subtree_schedule(uint32_t n, std::vector<MetaEntry>& out) {
  const uint32_t md = host_tree_depth(n);
  for (int l = static_cast<int>(md) - 1; l >= 0; --l) {
    for (uint32_t r = 0; r < n; ++r) {
      uint32_t a = 0, sz = n, depth = 0;
      while (depth < static_cast<uint32_t>(l) && sz > 1) {
        const uint32_t h = sz / 2;
        if (r - a < h) sz = h; else { a += h; sz -= h; }
        ++depth;
      }
      MetaEntry m{};
      if (depth != static_cast<uint32_t>(l) || sz < 2) {
        m.op = kCarry;
        m.a = static_cast<uint16_t>(r);
      } else {
        const uint32_t h = sz / 2, t = sz - h, s = r - a;
        const float hsc = static_cast<float>(h - 1) / static_cast<float>(sz - 1);
        const float tsc = static_cast<float>(t - 1) / static_cast<float>(sz - 1);
        const float hf = hsc * static_cast<float>(s);
        const float tf = tsc * static_cast<float>(s);
        const uint32_t hs = static_cast<uint32_t>(hf + 0.5f);
        const uint32_t ts = static_cast<uint32_t>(tf + 0.5f);
        m.op = kMerge;
        m.a = static_cast<uint16_t>(a + hs);
        m.b = static_cast<uint16_t>(a + h + ts);
        m.roll = static_cast<uint16_t>(s - ts);
      }
      out.push_back(m);
    }
  }
}

// Pass boundaries: depth cuts from split_depth down to 0, K levels per pass;
// the final pass takes the remainder (split_depth mod K, when non-zero).  A
// final pass of fewer levels has a shallower cone, so its blocks hold more
// root rows, and more threads share the sequential prefix sums of detection.
uint32_t cut_after(uint32_t d, uint32_t K) {
  return d > K ? d - K : 0;
}

// IEEE single arithmetic of ffa.cpp:153-171 (host code is built without
// contraction, so this matches the device's _rn intrinsics bit for bit)
float host_shift_scale(uint32_t part, uint32_t n) {
  return static_cast<float>(part - 1) / static_cast<float>(n - 1);
}
uint32_t host_scaled_shift(float scale, uint32_t s) {
  const float x = scale * static_cast<float>(s);
  return static_cast<uint32_t>(x + 0.5f);
}

struct ColumnNode {
  uint32_t a, n, u0, u1, off;  // task rows [a, a+n); rows [u0, u1) of it; buffer row of u0
};

// Column block: rows [s0, s1) of node X (task rows [xa, xa+xn)) from the rows
// K levels down.  Level k+1 holds, for every node of level k, the head- and
// tail-child rows its rows read (the index arithmetic of ffa.cpp), so each
// level stays within max_rows rows.
void build_column_block(uint32_t bins, uint32_t xa, uint32_t xn, uint32_t s0, uint32_t s1, uint32_t K,
                        uint32_t max_rows, bool final_pass, std::vector<MetaEntry>& meta,
                        std::vector<ColBlock>& blocks) {
  ColBlock b{};
  b.levels = static_cast<uint8_t>(K);
  b.final_pass = final_pass ? 1 : 0;
  b.out_row = final_pass ? s0 : xa + s0;
  b.count[0] = static_cast<uint16_t>(s1 - s0);
  std::vector<ColumnNode> nodes{ColumnNode{xa, xn, s0, s1, 0}};
  std::vector<std::vector<MetaEntry>> level(K);
  for (uint32_t k = 0; k < K; ++k) {
    std::vector<ColumnNode> children;
    uint32_t off = 0;
    for (const ColumnNode& nd : nodes) {
      check_arg(nd.n >= 2, "FFA column schedule reached a one-row node");
      const uint32_t h = nd.n / 2, t = nd.n - h;
      const float hsc = host_shift_scale(h, nd.n), tsc = host_shift_scale(t, nd.n);
      ColumnNode hc{nd.a, h, host_scaled_shift(hsc, nd.u0), host_scaled_shift(hsc, nd.u1 - 1) + 1, off};
      off += hc.u1 - hc.u0;
      ColumnNode tc{nd.a + h, t, host_scaled_shift(tsc, nd.u0), host_scaled_shift(tsc, nd.u1 - 1) + 1, off};
      off += tc.u1 - tc.u0;
      for (uint32_t u = nd.u0; u < nd.u1; ++u) {
        const uint32_t hs = host_scaled_shift(hsc, u), ts = host_scaled_shift(tsc, u);
        MetaEntry m{};
        m.op = kMerge;
        m.a = static_cast<uint16_t>(hc.off + hs - hc.u0);
        m.b = static_cast<uint16_t>(tc.off + ts - tc.u0);
        m.roll = static_cast<uint16_t>((u - ts) % bins);
        level[k].push_back(m);
      }
      children.push_back(hc);
      children.push_back(tc);
    }
    check_arg(off <= max_rows, "FFA column schedule exceeds the shared-memory tile");
    for (const MetaEntry& m : level[k])
      check_arg(m.a < off && m.b < off && m.roll < bins, "FFA column schedule entry out of range");
    b.count[k + 1] = static_cast<uint16_t>(off);
    nodes.swap(children);
  }
  check_arg(nodes.size() <= 8, "FFA column block has too many bottom runs");
  b.nruns = static_cast<uint8_t>(nodes.size());
  for (size_t j = 0; j < nodes.size(); ++j) {
    check_arg(nodes[j].u0 < nodes[j].u1 && nodes[j].u1 <= nodes[j].n, "FFA column run out of range");
    b.run_off[j] = static_cast<uint16_t>(nodes[j].off);
    b.run_row[j] = static_cast<uint16_t>(nodes[j].a + nodes[j].u0);
  }
  if (meta.size() & 1) meta.push_back(MetaEntry{});
  b.meta = static_cast<uint32_t>(meta.size());
  for (int k = static_cast<int>(K) - 1; k >= 0; --k) meta.insert(meta.end(), level[k].begin(), level[k].end());
  if (meta.size() & 1) meta.push_back(MetaEntry{});
  blocks.push_back(b);
}

// All column passes of a task split at depth dS (> 0).
void build_task_passes(gf_ffa_program& P, const FfaGeometry& g, TaskDev& d) {
  const uint32_t dS = d.split_depth, K = g.levels;
  d.pass_begin = static_cast<uint32_t>(P.passes.size());
  uint32_t depth = dS;
  while (true) {
    const uint32_t dn = cut_after(depth, K);
    const uint32_t levels = depth - dn;
    const bool final_pass = dn == 0;
    // final blocks: the rows whose cone of `levels` levels fits a row buffer
    // (R + 3 (2^levels - 1) at the bottom) and whose prefix sums fit the other
    const uint32_t R =
        final_pass ? std::min<uint32_t>(g.max_rows - 3 * ((1u << levels) - 1), g.cp_rows) : g.block_rows;
    const uint32_t nnodes = 1u << dn;
    const uint32_t maxn = (d.rows + nnodes - 1) >> dn;
    const uint32_t limit = final_pass ? d.rows_eval : maxn;
    const uint32_t bpn = (limit + R - 1) / R;
    PassDev pd{static_cast<uint32_t>(P.blocks.size()), 0u};
    for (uint32_t u = 0; u < nnodes * bpn; ++u) {
      const Node X = node_at(u / bpn, d.rows, dn);
      const uint32_t s0 = (u % bpn) * R;
      const uint32_t s1 = std::min<uint32_t>(s0 + R, final_pass ? d.rows_eval : X.n);
      if (s0 >= s1) continue;
      build_column_block(d.bins, X.a, X.n, s0, s1, levels, g.max_rows, final_pass, P.col_meta, P.blocks);
    }
    pd.nblocks = static_cast<uint32_t>(P.blocks.size()) - pd.block_begin;
    P.passes.push_back(pd);
    if (final_pass) break;
    depth = dn;
  }
  d.npasses = static_cast<uint32_t>(P.passes.size()) - d.pass_begin;
}

}  // namespace

extern "C" int gf_downsampled_size(uint64_t n, double factor, uint64_t* out) {
  return guarded([&] {
    check_arg(out != nullptr, "null argument");
    *out = downsampled_size_checked(n, factor);
  });
}

extern "C" int gf_downsampled_variance(uint64_t n, double factor, double* out) {
  return guarded([&] {
    check_arg(out != nullptr, "null argument");
    *out = downsampled_variance_host(n, factor);
  });
}

extern "C" int gf_ffa_task_stdnoise(const gf_ffa_task* t, float* out) {
  return guarded([&] {
    check_arg(t && out, "null argument");
    *out = task_stdnoise(*t);
  });
}

namespace {

struct MemberSpec {
  const gf_ffa_task* tasks;
  uint64_t ntasks;
  const uint64_t* widths;
  uint64_t nwidths;
  uint64_t nseries;
};

// Tables of every member's tasks: octaves, boxcar trials, on-chip geometry,
// column schedules and the launch classes.  Batched programs also get one
// item run per (task, member) so one launch per class covers every member.
std::unique_ptr<gf_ffa_program> build_program(const std::vector<MemberSpec>& specs, bool batched,
                                              uint64_t max_series, int device_id) {
  auto P = std::make_unique<gf_ffa_program>();
  P->device = device_id;
  P->batched = batched;
  P->max_series = max_series;
  std::vector<std::map<double, uint32_t>> octave_of(specs.size());
  for (size_t m = 0; m < specs.size(); ++m) {
    const MemberSpec& s = specs[m];
    check_arg(s.tasks && s.widths, "null argument");
    check_arg(s.ntasks > 0, "FFA executor plan must contain at least one task");
    check_arg(s.nwidths > 0, "FFA search plan width_trials must not be empty");
    check_arg(s.nwidths <= kMaxWidths, "at most 64 width trials");
    check_arg(P->tasks.size() + s.ntasks < (1ull << 31), "too many FFA tasks");
    FfaMember M;
    M.nsamples = s.tasks[0].input_nsamples;
    M.nseries = s.nseries;
    M.task_begin = static_cast<uint32_t>(P->tasks.size());
    M.ntasks = static_cast<uint32_t>(s.ntasks);
    M.widths.assign(s.widths, s.widths + s.nwidths);
    for (uint64_t i = 0; i < s.ntasks; ++i) validate_task(s.tasks[i], M.nsamples);
    // octaves = distinct prepare keys in plan order
    uint64_t off = 0;
    for (uint64_t i = 0; i < s.ntasks; ++i) {
      const gf_ffa_task& t = s.tasks[i];
      if (octave_of[m].count(t.downsample_factor)) continue;
      octave_of[m][t.downsample_factor] = static_cast<uint32_t>(M.octaves.size());
      M.octaves.push_back(OctaveDev{t.downsample_factor, t.prepared_nsamples, off});
      off = round_up(off + t.prepared_nsamples, 4);
      M.halo = std::max<uint64_t>(M.halo, static_cast<uint64_t>(std::ceil(t.downsample_factor)) + 2);
    }
    check_arg(M.octaves.size() <= 32, "at most 32 distinct downsample factors");
    M.prep_stride = round_up(off, 4);
    for (uint64_t i = 0; i < s.ntasks; ++i) {
      const gf_ffa_task& t = s.tasks[i];
      check_arg(t.bins <= kMaxBins, "FFA CUDA path supports bins <= 512");
      check_arg(t.rows < 65536, "FFA CUDA path supports at most 65535 rows per task");
      P->max_bins = std::max<uint32_t>(P->max_bins, static_cast<uint32_t>(t.bins));
    }
    for (uint64_t w : M.widths) M.max_width = std::max<uint32_t>(M.max_width, static_cast<uint32_t>(w));
    P->max_width = std::max(P->max_width, M.max_width);
    P->tasks.insert(P->tasks.end(), s.tasks, s.tasks + s.ntasks);
    P->task_member.insert(P->task_member.end(), s.ntasks, static_cast<uint32_t>(m));
    P->members.push_back(std::move(M));
  }
  // shared-memory geometry per CTA size and NB: two ColBlock headers, the
  // staged schedule, two row buffers of max_rows rows of the class's widest
  // rows; sized for two 512-thread CTAs or one 1024-thread CTA per SM (227 KB
  // per CTA at most, static state aside)
  uint32_t max_rows_all = 0;
  for (int gi = 0; gi < 2; ++gi)
  for (uint32_t nb = 1; nb <= 16; ++nb) {
    const size_t budget = gi == 0 ? 110 * 1024 : 222 * 1024;
    FfaGeometry& g = P->geo[gi][nb];
    const uint32_t cap = std::min<uint32_t>(32 * nb, P->max_bins);
    if (32 * (nb - 1) >= P->max_bins) break;
    g.pitch = cap | 1u;
    g.levels = 3;
    auto front_for = [&](uint32_t rows) {
      const uint64_t meta_cap = std::max<uint64_t>(static_cast<uint64_t>(tree_depth(rows)) * rows,
                                                   static_cast<uint64_t>(g.levels) * rows + 2);
      return static_cast<uint32_t>(round_up(std::max<uint64_t>(32 + 2 * meta_cap, cap), 4));
    };
    auto smem_for = [&](uint32_t rows) { return (front_for(rows) + 2ull * rows * g.pitch) * 4; };
    uint32_t rows = 8;
    while (rows < 65535 && smem_for(rows + 1) <= budget) ++rows;
    g.max_rows = rows;
    g.front = front_for(rows);
    // R + 3 (2^K - 1) rows at the bottom of a column
    while (g.levels > 1 && static_cast<int>(rows) - 3 * ((1 << g.levels) - 1) < 8) --g.levels;
    g.block_rows = rows - 3 * ((1u << g.levels) - 1);
    const uint32_t cp_pitch = (cap + P->max_width + 2) | 1u;
    g.cp_rows = (rows * g.pitch) / cp_pitch;
    g.final_rows = std::min<uint32_t>(g.block_rows, g.cp_rows);
    check_arg(g.final_rows >= 1 && g.block_rows >= 1, "FFA bins too large for the shared-memory tiles");
    g.smem_bytes = smem_for(rows);
    max_rows_all = std::max(max_rows_all, rows);
  }
  const uint32_t rows = max_rows_all;
  // subtree schedules for every size up to max_rows
  P->sub_offset.assign(rows + 1, 0u);
  for (uint32_t n = 1; n <= rows; ++n) {
    P->sub_offset[n] = static_cast<uint32_t>(P->sub_meta.size());
    build_subtree_schedule(n, P->sub_meta);
  }
  if (P->sub_meta.empty()) P->sub_meta.push_back(MetaEntry{});
  // tasks, trials, column schedules and classes
  std::map<std::tuple<int, uint32_t, int>, size_t> class_of;
  for (uint64_t i = 0; i < P->tasks.size(); ++i) {
    const auto& t = P->tasks[i];
    const uint32_t m = P->task_member[i];
    const FfaMember& M = P->members[m];
    for (uint64_t w : M.widths)
      check_arg(w > 0 && w < t.bins, "FFA detection width trials must satisfy 0 < width < bins");
    TaskDev d{};
    d.bins = static_cast<uint32_t>(t.bins);
    d.rows = static_cast<uint32_t>(t.rows);
    d.rows_eval = static_cast<uint32_t>(t.rows_eval);
    d.octave = octave_of[m][t.downsample_factor];
    d.prep_offset = M.octaves[d.octave].offset;
    d.inv_stdnoise = 1.0f / task_stdnoise(t);
    d.ntrials = static_cast<uint32_t>(M.widths.size());
    d.trial_offset = static_cast<uint32_t>(P->trial_dev.size());
    d.max_width = M.max_width;
    d.member = m;
    // ffa_detection.cpp:60-80 make_boxcar_trials (float arithmetic)
    const float bf = static_cast<float>(t.bins);
    for (uint64_t w : M.widths) {
      const float wf = static_cast<float>(w);
      const float h = std::sqrt((bf - wf) / (bf * wf));
      P->trial_dev.push_back(TrialDev{h, wf / (bf - wf) * h, static_cast<uint32_t>(w), 0u});
    }
    const uint32_t nbt = static_cast<uint32_t>(ceil_div(t.bins, 32));
    // on chip in a 512-thread CTA when it fits, else the 1024-thread tiles
    const int gi = t.rows <= P->geo[0][nbt].max_rows ? 0 : 1;
    const FfaGeometry& g = P->geo[gi][nbt];
    uint32_t ds = 0;
    while (ceil_div(t.rows, 1ull << ds) > g.max_rows) ++ds;
    check_arg(ds <= 15, "FFA task too deep");
    d.split_depth = ds;
    if (ds > 0) build_task_passes(*P, g, d);
    P->task_dev.push_back(d);
    // cluster sized by rows for split tasks; on-chip tasks use key 0
    int cluster = 1;
    if (ds > 0) {
      while (cluster < kClusterSize && static_cast<uint64_t>(cluster) * 512 < t.rows) cluster *= 2;
    }
    const uint32_t nb = static_cast<uint32_t>(ceil_div(t.bins, 32));
    const int threads = gi == 0 ? kSmallThreads : kThreads;
    const std::tuple<int, uint32_t, int> key{ds == 0 ? 0 : cluster, nb, threads};
    if (!class_of.count(key)) {
      class_of[key] = P->classes.size();
      P->classes.emplace_back();
      P->classes.back().cluster = cluster;
      P->classes.back().threads = threads;
      P->classes.back().nb = nb;
      P->classes.back().kernel = search_kernel_for(nb, threads);
    }
    FfaClass& c = P->classes[class_of[key]];
    c.tasks.push_back(static_cast<uint32_t>(i));
    if (ds > 0) c.max_elems = std::max<uint64_t>(c.max_elems, t.rows * t.bins);
  }
  // launch order: widest clusters (longest items) first
  std::stable_sort(P->classes.begin(), P->classes.end(), [](const FfaClass& x, const FfaClass& y) {
    return x.cluster != y.cluster ? x.cluster > y.cluster : x.nb > y.nb;
  });
  if (P->col_meta.empty()) P->col_meta.resize(2);
  if (P->blocks.empty()) P->blocks.resize(1);
  if (P->passes.empty()) P->passes.resize(1);
  for (auto& c : P->classes) {
    // largest tasks first so long items start early
    std::stable_sort(c.tasks.begin(), c.tasks.end(), [&](uint32_t x, uint32_t y) {
      return P->tasks[x].rows * P->tasks[x].bins > P->tasks[y].rows * P->tasks[y].bins;
    });
    if (batched) {
      for (uint32_t task : c.tasks) {
        const uint32_t m = P->task_member[task];
        c.units.push_back(UnitDev{c.nitems, task, m});
        c.nitems += P->members[m].nseries;
      }
      c.units_d.upload(c.units.data(), c.units.size() * sizeof(UnitDev), device_id);
    }
    const FfaGeometry& g = P->geo[c.threads == kSmallThreads ? 0 : 1][c.nb];
    cuda_check(cudaFuncSetAttribute(c.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(g.smem_bytes)),
               "cudaFuncSetAttribute(ffa_search_kernel)");
    cuda_check(cudaFuncSetAttribute(c.kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
               "cudaFuncSetAttribute(cluster size)");
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(c.cluster, 1, 1);
    cfg.blockDim = dim3(static_cast<unsigned>(c.threads), 1, 1);
    cfg.dynamicSmemBytes = g.smem_bytes;
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = c.cluster;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int n = 0;
    cuda_check(cudaOccupancyMaxActiveClusters(&n, c.kernel, &cfg), "cudaOccupancyMaxActiveClusters");
    check_arg(n > 0, "FFA kernel cannot be resident on this device");
    c.nclusters = n;
    // classes run one after another on the stream: they share the scratch
    P->scratch_floats = std::max<uint64_t>(P->scratch_floats, static_cast<uint64_t>(n) * 2 * c.max_elems);
    c.tasks_d.upload(c.tasks.data(), c.tasks.size() * sizeof(uint32_t), device_id);
  }
  P->tasks_d.upload(P->task_dev.data(), P->task_dev.size() * sizeof(TaskDev), device_id);
  P->trials_d.upload(P->trial_dev.data(), P->trial_dev.size() * sizeof(TrialDev), device_id);
  for (auto& M : P->members) M.octaves_d.upload(M.octaves.data(), M.octaves.size() * sizeof(OctaveDev), device_id);
  P->sub_meta_d.upload(P->sub_meta.data(), P->sub_meta.size() * sizeof(MetaEntry), device_id);
  P->sub_offset_d.upload(P->sub_offset.data(), P->sub_offset.size() * sizeof(uint32_t), device_id);
  P->col_meta_d.upload(P->col_meta.data(), P->col_meta.size() * sizeof(MetaEntry), device_id);
  P->blocks_d.upload(P->blocks.data(), P->blocks.size() * sizeof(ColBlock), device_id);
  P->passes_d.upload(P->passes.data(), P->passes.size() * sizeof(PassDev), device_id);
  return P;
}

PrepareItem prepare_item(const FfaMember& M, const float* dev_series, uint64_t nseries, uint64_t stride,
                         const double* dev_stats, float* dev_prepared) {
  check_arg(dev_series && dev_prepared, "null argument");
  check_arg(nseries > 0 && nseries < (1ull << 31), "nseries out of range");
  check_arg(stride >= M.nsamples, "stride must be >= nsamples");
  check_arg((kPrepareChunk + M.halo) * sizeof(float) <= 200 * 1024,
            "downsample factor too large for the prepare kernel");
  PrepareItem it{};
  it.series = dev_series;
  it.stride = stride;
  it.n = M.nsamples;
  it.stats = dev_stats;
  it.octaves = M.octaves_d.as<OctaveDev>();
  it.noct = static_cast<int32_t>(M.octaves.size());
  it.nseries = static_cast<uint32_t>(nseries);
  it.halo = M.halo;
  it.prepared = dev_prepared;
  it.prep_stride = M.prep_stride;
  return it;
}

// Batched: `ctas` CTAs over the table; single: (chunks, series) grid, ctas = chunks.
template <bool Batched>
void launch_prepare_table(const PrepareTable& tab, uint64_t ctas, uint64_t halo, cudaStream_t s) {
  const size_t smem = (kPrepareChunk + halo) * sizeof(float);
  check_arg(ctas < (1ull << 31), "prepare launch too large");
  cuda_check(cudaFuncSetAttribute(prepare_kernel<Batched>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)),
             "cudaFuncSetAttribute(prepare_kernel)");
  const dim3 grid(static_cast<unsigned>(ctas), Batched ? 1u : tab.one.nseries);
  prepare_kernel<Batched><<<grid, kPrepareThreads, smem, s>>>(tab);
  cuda_check(cudaGetLastError(), "prepare_kernel launch");
}

void launch_prepare(const gf_ffa_program* P, const FfaMember& M, const float* dev_series, uint64_t nseries,
                    uint64_t stride, const double* dev_stats, float* dev_prepared, cudaStream_t s) {
  DeviceGuard dg(P->device);
  PrepareTable tab{};
  tab.one = prepare_item(M, dev_series, nseries, stride, dev_stats, dev_prepared);
  check_arg(nseries < 65536, "nseries out of range");
  launch_prepare_table<false>(tab, ceil_div(M.nsamples, kPrepareChunk), M.halo, s);
}

// One launch per class; batched programs walk their item runs.
void launch_search(gf_ffa_program* P, const float* dev_prepared, uint64_t nseries, float snr_threshold,
                   void* dev_scratch, gf_peak_record* dev_peaks, uint64_t capacity, uint64_t* dev_counters,
                   cudaStream_t s) {
  check_arg(dev_counters, "null argument");
  check_arg(std::isfinite(snr_threshold), "FFA search S/N threshold must be finite");
  check_arg(capacity == 0 || dev_peaks != nullptr, "peak buffer must not be null");
  check_arg(P->scratch_floats == 0 || dev_scratch != nullptr, "FFA search needs scratch");
  DeviceGuard dg(P->device);
  cuda_check(cudaMemsetAsync(dev_counters, 0, 2 * sizeof(uint64_t), s), "cudaMemsetAsync(counters)");
  SearchParams sp{};
  sp.prepared = dev_prepared;
  sp.prep_stride = P->members[0].prep_stride;
  sp.tasks = P->tasks_d.as<TaskDev>();
  sp.trials = P->trials_d.as<TrialDev>();
  sp.sub_meta = P->sub_meta_d.as<MetaEntry>();
  sp.sub_offset = P->sub_offset_d.as<uint32_t>();
  sp.nseries = static_cast<uint32_t>(nseries);
  sp.members = P->batched ? P->members_d.as<MemberDev>() : nullptr;
  sp.threshold = snr_threshold;
  sp.peaks = dev_peaks;
  sp.capacity = capacity;
  sp.counters = reinterpret_cast<unsigned long long*>(dev_counters);
  sp.col_meta = P->col_meta_d.as<MetaEntry>();
  sp.blocks = P->blocks_d.as<ColBlock>();
  sp.passes = P->passes_d.as<PassDev>();
  sp.scratch = static_cast<float*>(dev_scratch);
  for (const FfaClass& c : P->classes) {
    sp.item_tasks = c.tasks_d.as<uint32_t>();
    sp.nitem_tasks = static_cast<uint32_t>(c.tasks.size());
    sp.units = P->batched ? c.units_d.as<UnitDev>() : nullptr;
    sp.nunits = static_cast<uint32_t>(c.units.size());
    sp.nitems = c.nitems;
    sp.scratch_elems = c.max_elems;
    const FfaGeometry& g = P->geo[c.threads == kSmallThreads ? 0 : 1][c.nb];
    sp.pitch = g.pitch;
    sp.max_rows = g.max_rows;
    sp.front = g.front;
    const uint64_t items = P->batched ? c.nitems : nseries * c.tasks.size();
    if (items == 0) continue;
    const unsigned nclusters = static_cast<unsigned>(std::min<uint64_t>(items, static_cast<uint64_t>(c.nclusters)));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(nclusters * c.cluster, 1, 1);
    cfg.blockDim = dim3(static_cast<unsigned>(c.threads), 1, 1);
    cfg.dynamicSmemBytes = g.smem_bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = c.cluster;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    cuda_check(cudaLaunchKernelEx(&cfg, c.kernel, sp), "ffa_search_kernel launch");
  }
}

// make_ffa_peak (ffa_detection.cpp:266-284) with trial_period
// (ffa_detection.cpp:115-124); dm = dm_low + (series_offset + series) * dm_step
void expand_record(const gf_ffa_program* P, const gf_peak_record& r, uint64_t series_offset, double dm_low,
                   double dm_step, gf_peak& p) {
  check_arg(r.task < P->tasks.size(), "corrupt peak record");
  const FfaMember& M = P->members[P->task_member[r.task]];
  check_arg(r.width_index < M.widths.size(), "corrupt peak record");
  const gf_ffa_task& t = P->tasks[r.task];
  double period;
  if (t.rows <= 1) {
    period = t.effective_tsamp * static_cast<double>(t.bins);
  } else {
    const double b = static_cast<double>(t.bins);
    period = t.effective_tsamp * b * b / (b - static_cast<double>(r.shift) / static_cast<double>(t.rows - 1));
  }
  const uint64_t series = series_offset + r.series;
  p.dm = dm_low + static_cast<double>(series) * dm_step;
  p.dm_index = series;
  p.period = period;
  p.frequency = 1.0 / period;
  p.width = M.widths[r.width_index];
  p.duty_cycle = static_cast<double>(p.width) / static_cast<double>(t.bins);
  p.width_index = r.width_index;
  p.period_index = r.shift;
  p.phase = r.phase;
  p.shift = r.shift;
  p.bins = t.bins;
  p.snr = r.snr;
  p.reserved = 0;
}

}  // namespace

namespace gf {
void ffa_program_peak_tables(const gf_ffa_program* P, std::vector<PeakTaskInfo>& tasks, std::vector<uint64_t>& widths,
                             int& device) {
  check_arg(P != nullptr, "null argument");
  check_arg(!P->batched && P->members.size() == 1, "device candidate selection takes a single-plan FFA program");
  tasks.clear();
  for (const gf_ffa_task& t : P->tasks) tasks.push_back(PeakTaskInfo{t.effective_tsamp, t.bins, t.rows});
  widths = P->members[0].widths;
  device = P->device;
}
}  // namespace gf

extern "C" int gf_ffa_program_create(const gf_ffa_task* tasks, uint64_t ntasks, const uint64_t* widths,
                                     uint64_t nwidths, uint64_t max_series, int32_t device_id,
                                     gf_ffa_program** out) {
  return guarded([&] {
    check_arg(out != nullptr, "null argument");
    *out = nullptr;
    check_arg(max_series > 0 && max_series < (1ull << 31), "max_series out of range");
    DeviceGuard dg(device_id);
    *out = build_program({MemberSpec{tasks, ntasks, widths, nwidths, max_series}}, false, max_series, device_id)
               .release();
  });
}

extern "C" int gf_ffa_batch_create(const gf_ffa_batch_member* members, uint64_t nmembers, int32_t device_id,
                                   gf_ffa_program** out) {
  return guarded([&] {
    check_arg(members && out, "null argument");
    *out = nullptr;
    check_arg(nmembers > 0 && nmembers < 65536, "batched FFA programs hold 1 to 65535 members");
    std::vector<MemberSpec> specs;
    uint64_t mx = 0;
    for (uint64_t m = 0; m < nmembers; ++m) {
      const gf_ffa_batch_member& b = members[m];
      check_arg(b.nseries > 0 && b.nseries < 65536, "member nseries out of range");
      specs.push_back(MemberSpec{b.tasks, b.ntasks, b.widths, b.nwidths, b.nseries});
      mx = std::max(mx, b.nseries);
    }
    DeviceGuard dg(device_id);
    *out = build_program(specs, true, mx, device_id).release();
  });
}

extern "C" int gf_ffa_program_destroy(gf_ffa_program* p) {
  return guarded([&] { delete p; });
}

extern "C" int gf_ffa_program_info(const gf_ffa_program* P, gf_ffa_info* info) {
  return guarded([&] {
    check_arg(P && info, "null argument");
    std::memset(info, 0, sizeof *info);
    info->ntasks = P->tasks.size();
    for (const auto& M : P->members) {
      info->noctaves = std::max<uint64_t>(info->noctaves, M.octaves.size());
      info->prepared_floats = std::max<uint64_t>(info->prepared_floats, M.prep_stride);
    }
    info->scratch_bytes = std::max<uint64_t>(16, P->scratch_floats * 4);
    uint64_t mx = 0;
    for (const auto& t : P->tasks) mx = std::max<uint64_t>(mx, t.rows * t.bins);
    info->max_task_elements = mx;
    info->metadata_bytes = P->tasks_d.bytes + P->trials_d.bytes + P->sub_meta_d.bytes + P->sub_offset_d.bytes +
                           P->col_meta_d.bytes + P->blocks_d.bytes + P->passes_d.bytes + P->members_d.bytes;
    for (const auto& M : P->members) info->metadata_bytes += M.octaves_d.bytes;
    for (const auto& c : P->classes) info->metadata_bytes += c.tasks_d.bytes + c.units_d.bytes;
    info->nclasses = P->classes.size();
  });
}

extern "C" int gf_ffa_batch_member_info(const gf_ffa_program* P, uint64_t member,
                                        gf_ffa_member_info* info) {
  return guarded([&] {
    check_arg(P && info, "null argument");
    check_arg(member < P->members.size(), "member out of range");
    const FfaMember& M = P->members[member];
    std::memset(info, 0, sizeof *info);
    info->nsamples = M.nsamples;
    info->nseries = M.nseries;
    info->prepared_floats = M.prep_stride;
    info->task_begin = M.task_begin;
    info->ntasks = M.ntasks;
    info->noctaves = M.octaves.size();
  });
}

extern "C" int gf_ffa_prepare(gf_ffa_program* P, const float* dev_series, uint64_t nseries, uint64_t stride,
                              const double* dev_stats, float* dev_prepared, void* stream) {
  return guarded([&] {
    check_arg(P != nullptr, "null argument");
    check_arg(!P->batched, "batched FFA programs prepare through gf_ffa_batch_prepare");
    launch_prepare(P, P->members[0], dev_series, nseries, stride, dev_stats, dev_prepared, as_stream(stream));
  });
}

extern "C" int gf_ffa_search(gf_ffa_program* P, const float* dev_prepared, uint64_t nseries, float snr_threshold,
                             void* dev_scratch, gf_peak_record* dev_peaks, uint64_t capacity,
                             uint64_t* dev_counters, void* stream) {
  return guarded([&] {
    check_arg(P && dev_prepared, "null argument");
    check_arg(!P->batched, "batched FFA programs search through gf_ffa_batch_search");
    check_arg(nseries > 0 && nseries <= P->max_series, "nseries must be in (0, max_series]");
    launch_search(P, dev_prepared, nseries, snr_threshold, dev_scratch, dev_peaks, capacity, dev_counters,
                  as_stream(stream));
  });
}

extern "C" int gf_ffa_batch_bind(gf_ffa_program* P, const float* const* dev_prepared) {
  return guarded([&] {
    check_arg(P && dev_prepared, "null argument");
    check_arg(P->batched, "gf_ffa_batch_bind needs a batched FFA program");
    DeviceGuard dg(P->device);
    std::vector<MemberDev> md(P->members.size());
    for (size_t m = 0; m < P->members.size(); ++m) {
      check_arg(dev_prepared[m] != nullptr, "null prepared buffer");
      check_arg((reinterpret_cast<uintptr_t>(dev_prepared[m]) & 15u) == 0,
                "prepared buffers must be 16-byte aligned");
      P->members[m].prepared = dev_prepared[m];
      md[m] = MemberDev{dev_prepared[m], P->members[m].prep_stride};
    }
    P->members_d.upload(md.data(), md.size() * sizeof(MemberDev), P->device);
    P->bound = true;
  });
}

extern "C" int gf_ffa_batch_prepare(gf_ffa_program* P, uint64_t member, const float* dev_series, uint64_t stride,
                                    const double* dev_stats, void* stream) {
  return guarded([&] {
    check_arg(P != nullptr, "null argument");
    check_arg(P->batched && P->bound, "gf_ffa_batch_prepare needs a bound batched FFA program");
    check_arg(member < P->members.size(), "member out of range");
    const FfaMember& M = P->members[member];
    launch_prepare(P, M, dev_series, M.nseries, stride, dev_stats, const_cast<float*>(M.prepared),
                   as_stream(stream));
  });
}

extern "C" int gf_ffa_batch_bind_series(gf_ffa_program* P, const float* const* dev_series, const uint64_t* strides,
                                        const double* const* dev_stats) {
  return guarded([&] {
    check_arg(P && dev_series && strides, "null argument");
    check_arg(P->batched && P->bound, "gf_ffa_batch_bind_series needs a bound batched FFA program");
    DeviceGuard dg(P->device);
    std::vector<PrepareItem> items;
    std::vector<uint64_t> begin;
    uint64_t total = 0, halo = 0;
    for (size_t m = 0; m < P->members.size(); ++m) {
      const FfaMember& M = P->members[m];
      items.push_back(prepare_item(M, dev_series[m], M.nseries, strides[m], dev_stats ? dev_stats[m] : nullptr,
                                   const_cast<float*>(M.prepared)));
      begin.push_back(total);
      total += prepare_ctas(items.back());
      halo = std::max(halo, M.halo);
    }
    P->prepare_items_d.upload(items.data(), items.size() * sizeof(PrepareItem), P->device);
    P->prepare_begin_d.upload(begin.data(), begin.size() * sizeof(uint64_t), P->device);
    P->prepare_ctas_total = total;
    P->prepare_halo = halo;
  });
}

extern "C" int gf_ffa_batch_prepare_all(gf_ffa_program* P, void* stream) {
  return guarded([&] {
    check_arg(P != nullptr, "null argument");
    check_arg(P->prepare_items_d.ptr != nullptr, "gf_ffa_batch_prepare_all needs gf_ffa_batch_bind_series");
    DeviceGuard dg(P->device);
    PrepareTable tab{};
    tab.items = P->prepare_items_d.as<PrepareItem>();
    tab.begin = P->prepare_begin_d.as<uint64_t>();
    tab.nitems = static_cast<int32_t>(P->members.size());
    launch_prepare_table<true>(tab, P->prepare_ctas_total, P->prepare_halo, as_stream(stream));
  });
}

extern "C" int gf_ffa_batch_search(gf_ffa_program* P, float snr_threshold, void* dev_scratch,
                                   gf_peak_record* dev_peaks, uint64_t capacity, uint64_t* dev_counters,
                                   void* stream) {
  return guarded([&] {
    check_arg(P != nullptr, "null argument");
    check_arg(P->batched && P->bound, "gf_ffa_batch_search needs a bound batched FFA program");
    launch_search(P, nullptr, 0, snr_threshold, dev_scratch, dev_peaks, capacity, dev_counters,
                  as_stream(stream));
  });
}

extern "C" int gf_ffa_expand_peaks(const gf_ffa_program* P, const gf_peak_record* records, uint64_t n,
                                   uint64_t series_offset, double dm_low, double dm_step, gf_peak* out) {
  return guarded([&] {
    check_arg(P && (n == 0 || (records && out)), "null argument");
    for (uint64_t i = 0; i < n; ++i) expand_record(P, records[i], series_offset, dm_low, dm_step, out[i]);
  });
}

extern "C" int gf_ffa_batch_expand_peaks(const gf_ffa_program* P, const gf_peak_record* records, uint64_t n,
                                         const uint64_t* series_offset, const double* dm_low,
                                         const double* dm_step, gf_peak* out, uint32_t* member) {
  return guarded([&] {
    check_arg(P && (n == 0 || (records && out && member && series_offset && dm_low && dm_step)),
              "null argument");
    for (uint64_t i = 0; i < n; ++i) {
      check_arg(records[i].task < P->tasks.size(), "corrupt peak record");
      const uint32_t m = P->task_member[records[i].task];
      check_arg(records[i].series < P->members[m].nseries, "corrupt peak record");
      expand_record(P, records[i], series_offset[m], dm_low[m], dm_step[m], out[i]);
      member[i] = m;
    }
  });
}

extern "C" int gf_ffa_transform(const float* dev_input, uint64_t rows, uint64_t bins, float* dev_output,
                                void* dev_scratch, void* stream) {
  return guarded([&] {
    check_arg(rows > 0, "FFA transform rows must be > 0");
    check_arg(bins > 1, "FFA transform bins must be > 1");
    check_arg(dev_input && dev_output && dev_scratch, "null argument");
    check_arg(rows < (1ull << 31) && bins < (1ull << 31), "FFA transform shape out of range");
    auto s = as_stream(stream);
    uint32_t depth = 0;
    for (uint64_t n = rows; n > 1; n = (n + 1) / 2) ++depth;
    float* q[2] = {static_cast<float*>(dev_scratch), static_cast<float*>(dev_scratch) + rows * bins};
    if (depth == 0) {
      cuda_check(cudaMemcpyAsync(dev_output, dev_input, rows * bins * 4, cudaMemcpyDeviceToDevice, s),
                 "cudaMemcpyAsync(transform)");
      return;
    }
    const unsigned grid = static_cast<unsigned>(ceil_div(rows, kThreads / 32));
    for (int d = static_cast<int>(depth) - 1; d >= 0; --d) {
      float* out = d == 0 ? dev_output : q[d & 1];
      const float* prev = q[(d + 1) & 1];
      ffa_level_kernel<<<grid, kThreads, 0, s>>>(dev_input, static_cast<uint32_t>(rows),
                                                 static_cast<uint32_t>(bins), static_cast<uint32_t>(d), prev, out);
    }
    cuda_check(cudaGetLastError(), "ffa_level_kernel launch");
  });
}
