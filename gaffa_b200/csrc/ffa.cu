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
// kLeafRows rows on chip and writes them to the cluster's global scratch,
// then the cluster steps up the tree one depth per cluster barrier (rows
// split across its CTAs, scratch kept hot in L2), and the root level is fused
// with detection.  No CTA ever waits on another except through the hardware
// cluster barrier.
#include "common.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

namespace cg = cooperative_groups;

namespace gf {
namespace {

constexpr int kThreads = 512;
constexpr int kLeafRows = 64;       // rows transformed on chip per subtree
constexpr int kMaxBins = 512;
constexpr int kMaxWidths = 64;
constexpr int kClusterSize = 8;
constexpr int kPrepareChunk = 16384;

struct TaskDev {
  uint32_t bins, rows, rows_eval, octave;
  uint64_t prep_offset;   // floats from the series' prepared block
  float inv_stdnoise;
  uint32_t ntrials;
  uint32_t trial_offset;
  uint32_t split_depth;   // depth of the on-chip subtrees (0: whole task in one CTA)
  uint32_t max_width;
  uint32_t reserved;
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

__device__ __forceinline__ float normalised(const float* row, uint64_t i, const double* stats) {
  const float y = row[i];
  if (stats == nullptr) return y;
  const double scale = stats[1];
  if (scale == 0.0) return 0.0f;
  return static_cast<float>(__dmul_rn(__dsub_rn(static_cast<double>(y), stats[0]), scale));
}

// first output index k with floor(k * f) >= x (k * f evaluated as the
// reference does, (double)k * factor)
__device__ __forceinline__ uint64_t first_output_at(uint64_t x, double f) {
  uint64_t k = static_cast<uint64_t>(floor(__ddiv_rn(static_cast<double>(x), f)));
  while (k > 0 && floor(__dmul_rn(static_cast<double>(k - 1), f)) >= static_cast<double>(x)) --k;
  while (floor(__dmul_rn(static_cast<double>(k), f)) < static_cast<double>(x)) ++k;
  return k;
}

__global__ void __launch_bounds__(kThreads) prepare_kernel(const float* __restrict__ series, uint64_t stride,
                                                           uint64_t n, const double* __restrict__ stats,
                                                           const OctaveDev* __restrict__ octaves, int noct,
                                                           uint64_t halo, float* __restrict__ prepared,
                                                           uint64_t prep_stride) {
  extern __shared__ float xs[];
  __shared__ uint64_t kb[32], cnt_prefix[33];
  const int s = blockIdx.y;
  const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kPrepareChunk;
  const float* row = series + s * stride;
  const double* st = stats ? stats + 2 * s : nullptr;
  const uint64_t span = umin64(kPrepareChunk + halo, n - c0);
  for (uint64_t i = threadIdx.x; i < span; i += kThreads) xs[i] = normalised(row, c0 + i, st);
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
  float* out_row = prepared + s * prep_stride;
  const double last_index = static_cast<double>(n - 1);
  for (uint64_t idx = threadIdx.x; idx < total; idx += kThreads) {
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
//   LOAD   out = global row a         (input rows or rows of a lower pass)
// Rows of a level live in one of two shared-memory buffers (pitch = bins|1);
// levels alternate buffers, so each level costs one __syncthreads.

enum : uint16_t { kMerge = 0, kCarry = 1, kLoad = 2 };

struct MetaEntry {
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
__device__ __forceinline__ Node node_at(uint32_t index, uint32_t n, uint32_t depth) {
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

template <bool GlobalCg>
__device__ __forceinline__ void eval_level(const MetaEntry* __restrict__ meta, uint32_t nrows,
                                           const float* __restrict__ prev, float* __restrict__ out,
                                           uint32_t pitch, const float* __restrict__ gsrc, uint32_t bins) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t q = warp; q < nrows; q += kThreads / 32) {
    const MetaEntry m = meta[q];
    float* o = out + q * pitch;
    if (m.op == kMerge) {
      const float* h = prev + m.a * pitch;
      const float* t = prev + m.b * pitch;
      const uint32_t r = m.roll < bins ? m.roll : m.roll % bins;
      for (uint32_t j = lane; j < bins; j += 32) {
        uint32_t k = j + r;
        if (k >= bins) k -= bins;
        o[j] = __fadd_rn(h[j], t[k]);
      }
    } else if (m.op == kCarry) {
      const float* h = prev + m.a * pitch;
      for (uint32_t j = lane; j < bins; j += 32) o[j] = h[j];
    } else {
      const float* g = gsrc + static_cast<uint64_t>(m.a) * bins;
      for (uint32_t j = lane; j < bins; j += 32) o[j] = GlobalCg ? __ldcg(g + j) : __ldg(g + j);
    }
  }
}

// rows [0, n) of `src` (global, pitch bins, row a0 first) into smem
template <bool GlobalCg>
__device__ __forceinline__ void load_rows(const float* src, uint32_t n, uint32_t bins, float* out, uint32_t pitch) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t q = warp; q < n; q += kThreads / 32)
    for (uint32_t j = lane; j < bins; j += 32)
      out[q * pitch + j] = GlobalCg ? __ldcg(src + static_cast<uint64_t>(q) * bins + j)
                                    : __ldg(src + static_cast<uint64_t>(q) * bins + j);
}

__device__ __forceinline__ void store_rows(const float* in, uint32_t pitch, uint32_t n, uint32_t bins, float* dst) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t q = warp; q < n; q += kThreads / 32)
    for (uint32_t j = lane; j < bins; j += 32) __stcg(dst + static_cast<uint64_t>(q) * bins + j, in[q * pitch + j]);
}

__device__ __forceinline__ uint32_t tree_depth(uint32_t n) {
  uint32_t d = 0;
  while (n > 1) { n = (n + 1) >> 1; ++d; }
  return d;
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

// rows[i] (pitch `pitch`) hold root rows shift0 + i, i < count.  Prefix sums
// are sequential per row (one thread per row, ffa_detection.cpp:126-139);
// each warp then scans one row for every width (first phase of the maximum,
// :141-170) and appends peaks with S/N >= threshold.
__device__ void detect_rows(const float* rows, uint32_t pitch, uint32_t count, uint32_t shift0, float* cp,
                            uint32_t cp_pitch, const DetectArgs& a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bins = a.bins;
  if (threadIdx.x < count) {
    const float* prof = rows + threadIdx.x * pitch;
    float* c = cp + threadIdx.x * cp_pitch;
    float acc = 0.0f;
    c[0] = 0.0f;
    for (uint32_t i = 0; i < bins; ++i) {
      acc = __fadd_rn(acc, prof[i]);
      c[i + 1] = acc;
    }
    for (uint32_t i = 0; i < a.max_width; ++i) {
      acc = __fadd_rn(acc, prof[i]);
      c[bins + i + 1] = acc;
    }
  }
  __syncthreads();
  for (uint32_t r = warp; r < count; r += kThreads / 32) {
    const float* c = cp + r * cp_pitch;
    const float psum = c[bins];
    for (uint32_t k = 0; k < a.ntrials; ++k) {
      const TrialDev tr = a.trials[k];
      float best = -INFINITY;
      uint32_t best_ph = 0xffffffffu;
      for (uint32_t ph = lane; ph < bins; ph += 32) {
        const float v = __fsub_rn(c[ph + tr.width], c[ph]);
        if (v > best) { best = v; best_ph = ph; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, best, off);
        const uint32_t op = __shfl_xor_sync(0xffffffffu, best_ph, off);
        if (ov > best || (ov == best && op < best_ph)) { best = ov; best_ph = op; }
      }
      if (lane == 0) {
        const float snr = __fmul_rn(
            __fsub_rn(__fmul_rn(__fadd_rn(tr.height, tr.baseline), best), __fmul_rn(tr.baseline, psum)),
            a.inv_stdnoise);
        if (snr >= a.threshold) {
          const unsigned long long slot = atomicAdd(a.counters, 1ull);
          if (slot < a.capacity) {
            gf_peak_record rec;
            rec.series = a.series;
            rec.task = a.task;
            rec.shift = shift0 + r;
            rec.phase = static_cast<uint16_t>(best_ph);
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
  const uint32_t* item_tasks;   // task indices of this launch's class
  uint32_t nitem_tasks;
  uint32_t nseries;
  float threshold;
  gf_peak_record* peaks;
  uint64_t capacity;
  unsigned long long* counters;
  float* scratch;               // per cluster: 2 * scratch_elems floats
  uint64_t scratch_elems;
  uint32_t pitch;               // shared-memory row pitch (max bins | 1)
  uint32_t max_rows;            // rows per shared-memory buffer
  uint32_t block_rows;          // R: output rows per column block
  uint32_t final_rows;          // R for the root pass (room for prefix sums)
  uint32_t levels;              // K: levels per column pass
  uint32_t* error;              // set when a schedule would overflow a buffer
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

// Evaluates a whole subtree of n <= max_rows rows starting at input row
// `a` (pointer `src` = row a), from its input rows up to relative level
// `stop` (0: the subtree root).  Returns the buffer holding level `stop`.
__device__ float* eval_subtree(const SearchParams& p, const float* src, uint32_t n, uint32_t bins, uint32_t stop,
                               float* buf0, float* buf1) {
  const uint32_t pitch = p.pitch;
  const uint32_t md = tree_depth(n);
  float* bufs[2] = {buf0, buf1};
  load_rows<false>(src, n, bins, bufs[md & 1], pitch);
  __syncthreads();
  const MetaEntry* table = p.sub_meta + p.sub_offset[n];
  for (int l = static_cast<int>(md) - 1; l >= static_cast<int>(stop); --l) {
    eval_level<false>(table + (md - 1 - l) * n, n, bufs[(l + 1) & 1], bufs[l & 1], pitch, nullptr, bins);
    __syncthreads();
  }
  return bufs[stop & 1];
}

// Column block: rows [s0, s1) of node X (task rows, depth dx) computed from
// the rows of depth dx + K held in global `src` (task row coordinates).
// Warp 0 builds the per-level row schedules top-down (only the rows the
// block needs, ffa.cpp index arithmetic); all warps then evaluate bottom-up.
// The result (s1 - s0 rows) is in buf0.
__device__ void eval_column(const SearchParams& p, Node X, uint32_t s0, uint32_t s1, uint32_t K, const float* src,
                            uint32_t bins, float* buf0, float* buf1, MetaEntry* cmeta, uint32_t* counts) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t max_rows = p.max_rows;
  if (warp == 0) {
    // per level: up to 2^k nodes (K <= 3 -> <= 8), one per lane
    uint32_t na = 0, nn = 0, nu0 = 0, nu1 = 0, noff = 0;  // this lane's node at the current level
    uint32_t count = 1;
    if (lane == 0) { na = X.a; nn = X.n; nu0 = s0; nu1 = s1; noff = 0; }
    uint32_t rows = s1 - s0;
    bool overflow = rows > max_rows;
    for (uint32_t k = 0; k < K; ++k) {
      // children of this lane's node
      uint32_t ha = 0, hn = 0, hu0 = 0, hu1 = 0, ta = 0, tn = 0, tu0 = 0, tu1 = 0;
      float hsc = 0.0f, tsc = 0.0f;
      if (lane < count) {
        const uint32_t h = nn >> 1, t = nn - h;
        hsc = shift_scale(h, nn);
        tsc = shift_scale(t, nn);
        ha = na; hn = h; hu0 = scaled_shift(hsc, nu0); hu1 = scaled_shift(hsc, nu1 - 1) + 1;
        ta = na + h; tn = t; tu0 = scaled_shift(tsc, nu0); tu1 = scaled_shift(tsc, nu1 - 1) + 1;
      }
      // offsets of the children rows at level k+1 (exclusive scan, head then tail)
      const uint32_t len = (hu1 - hu0) + (tu1 - tu0);
      uint32_t incl = len;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
      }
      const uint32_t hoff = incl - len, toff = hoff + (hu1 - hu0);
      const uint32_t next_rows = __shfl_sync(0xffffffffu, incl, 31);
      overflow |= next_rows > max_rows;
      if (lane == 0) counts[k + 1] = next_rows;
      // schedule of level k: rows of each node, lanes over rows
      MetaEntry* mk = cmeta + k * max_rows;
      for (uint32_t i = 0; i < count; ++i) {
        const uint32_t bu0 = __shfl_sync(0xffffffffu, nu0, i), bu1 = __shfl_sync(0xffffffffu, nu1, i);
        const uint32_t boff = __shfl_sync(0xffffffffu, noff, i);
        const float bh = __shfl_sync(0xffffffffu, hsc, i), bt = __shfl_sync(0xffffffffu, tsc, i);
        const uint32_t bho = __shfl_sync(0xffffffffu, hoff, i), bto = __shfl_sync(0xffffffffu, toff, i);
        const uint32_t bhu0 = __shfl_sync(0xffffffffu, hu0, i), btu0 = __shfl_sync(0xffffffffu, tu0, i);
        for (uint32_t u = bu0 + lane; u < bu1 && !overflow; u += 32) {
          const uint32_t hs = scaled_shift(bh, u), ts = scaled_shift(bt, u);
          MetaEntry m;
          m.op = kMerge;
          m.a = static_cast<uint16_t>(bho + hs - bhu0);
          m.b = static_cast<uint16_t>(bto + ts - btu0);
          m.roll = static_cast<uint16_t>(u - ts);
          mk[boff + u - bu0] = m;
        }
      }
      // children become the nodes of level k+1: lane l takes child l
      const uint32_t src_lane = lane >> 1;
      const bool is_tail = lane & 1;
      const uint32_t c_ha = __shfl_sync(0xffffffffu, ha, src_lane), c_ta = __shfl_sync(0xffffffffu, ta, src_lane);
      const uint32_t c_hn = __shfl_sync(0xffffffffu, hn, src_lane), c_tn = __shfl_sync(0xffffffffu, tn, src_lane);
      const uint32_t c_hu0 = __shfl_sync(0xffffffffu, hu0, src_lane), c_tu0 = __shfl_sync(0xffffffffu, tu0, src_lane);
      const uint32_t c_hu1 = __shfl_sync(0xffffffffu, hu1, src_lane), c_tu1 = __shfl_sync(0xffffffffu, tu1, src_lane);
      const uint32_t c_ho = __shfl_sync(0xffffffffu, hoff, src_lane), c_to = __shfl_sync(0xffffffffu, toff, src_lane);
      na = is_tail ? c_ta : c_ha;
      nn = is_tail ? c_tn : c_hn;
      nu0 = is_tail ? c_tu0 : c_hu0;
      nu1 = is_tail ? c_tu1 : c_hu1;
      noff = is_tail ? c_to : c_ho;
      count *= 2;
      rows = next_rows;
    }
    // bottom level K: rows loaded from src
    MetaEntry* mK = cmeta + K * max_rows;
    for (uint32_t i = 0; i < count; ++i) {
      const uint32_t ba = __shfl_sync(0xffffffffu, na, i);
      const uint32_t bu0 = __shfl_sync(0xffffffffu, nu0, i), bu1 = __shfl_sync(0xffffffffu, nu1, i);
      const uint32_t boff = __shfl_sync(0xffffffffu, noff, i);
      for (uint32_t u = bu0 + lane; u < bu1 && !overflow; u += 32) {
        MetaEntry m;
        m.op = kLoad;
        m.a = static_cast<uint16_t>(ba + u);
        m.b = 0;
        m.roll = 0;
        mK[boff + u - bu0] = m;
      }
    }
    if (lane == 0) {
      counts[0] = s1 - s0;
      if (overflow) {
        for (uint32_t k = 0; k <= K; ++k) counts[k] = 0u;
        atomicOr(p.error, GF_STATUS_SCHEDULE);
      }
    }
  }
  __syncthreads();
  float* bufs[2] = {buf0, buf1};
  // a failed schedule leaves counts at 0: nothing is evaluated
  eval_level<true>(cmeta + K * max_rows, counts[K], nullptr, bufs[K & 1], p.pitch, src, bins);
  __syncthreads();
  for (int k = static_cast<int>(K) - 1; k >= 0; --k) {
    eval_level<false>(cmeta + k * max_rows, counts[k], bufs[(k + 1) & 1], bufs[k & 1], p.pitch, nullptr, bins);
    __syncthreads();
  }
}

// Pass boundaries: depth cuts from split_depth down to 0, final pass K levels
// (or fewer), earlier passes K levels, the remainder at the bottom.
__device__ __forceinline__ uint32_t cut_after(uint32_t d, uint32_t dS, uint32_t K) {
  // next (shallower) cut below depth d in the chain dS -> ... -> 0
  const uint32_t r = dS % K;
  if (d == dS && r != 0) return dS - r;
  return d >= K ? d - K : 0;
}

// One (series, task) per cluster (cluster size 1, 2, 4 or 8).
__global__ void __launch_bounds__(kThreads, 2) ffa_task_kernel(SearchParams p) {
  extern __shared__ __align__(16) float sm[];
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t cs = cluster.num_blocks();
  const uint32_t rank = cluster.block_rank();
  const uint32_t cid = blockIdx.x / cs;
  const uint32_t nclusters = gridDim.x / cs;
  const uint32_t pitch = p.pitch;
  float* buf0 = sm;
  float* buf1 = sm + p.max_rows * pitch;
  MetaEntry* cmeta = reinterpret_cast<MetaEntry*>(buf1 + p.max_rows * pitch);
  uint32_t* counts = reinterpret_cast<uint32_t*>(cmeta + (p.levels + 1) * p.max_rows);
  float* q0 = p.scratch ? p.scratch + static_cast<uint64_t>(cid) * 2 * p.scratch_elems : nullptr;
  float* q1 = q0 ? q0 + p.scratch_elems : nullptr;
  const uint64_t nitems = static_cast<uint64_t>(p.nseries) * p.nitem_tasks;
  for (uint64_t item = cid; item < nitems; item += nclusters) {
    const uint32_t series = static_cast<uint32_t>(item / p.nitem_tasks);
    const uint32_t task = p.item_tasks[item % p.nitem_tasks];
    const TaskDev t = p.tasks[task];
    const float* input = p.prepared + series * p.prep_stride + t.prep_offset;
    const uint32_t bins = t.bins;
    const DetectArgs da = make_detect(p, t, series, task);
    const uint32_t cp_pitch = (bins + t.max_width + 2) | 1u;
    const uint32_t dS = t.split_depth;
    if (dS == 0) {
      // whole task on chip: levels below the root, then root rows in batches
      if (t.rows == 1) {
        load_rows<false>(input, 1, bins, buf0, pitch);
        __syncthreads();
        detect_rows(buf0, pitch, 1, 0, buf1, cp_pitch, da);
        continue;
      }
      float* lvl1 = eval_subtree(p, input, t.rows, bins, 1, buf0, buf1);
      float* other = lvl1 == buf0 ? buf1 : buf0;
      const uint32_t md = tree_depth(t.rows);
      const MetaEntry* root = p.sub_meta + p.sub_offset[t.rows] + (md - 1) * t.rows;
      const uint32_t batch = umin32(kThreads, (p.max_rows * pitch) / (pitch + cp_pitch));
      for (uint32_t b0 = 0; b0 < t.rows_eval; b0 += batch) {
        const uint32_t cnt = umin32(batch, t.rows_eval - b0);
        eval_level<false>(root + b0, cnt, lvl1, other, pitch, nullptr, bins);
        __syncthreads();
        detect_rows(other, pitch, cnt, b0, other + batch * pitch, cp_pitch, da);
      }
      continue;
    }
    // 1. subtrees at depth dS, on chip, into scratch q0
    const uint32_t nsub = 1u << dS;
    for (uint32_t sub = rank; sub < nsub; sub += cs) {
      const Node nd = node_at(sub, t.rows, dS);
      if (nd.n == 1) {
        load_rows<false>(input + static_cast<uint64_t>(nd.a) * bins, 1, bins, buf0, pitch);
        __syncthreads();
        store_rows(buf0, pitch, 1, bins, q0 + static_cast<uint64_t>(nd.a) * bins);
      } else {
        const float* res = eval_subtree(p, input + static_cast<uint64_t>(nd.a) * bins, nd.n, bins, 0, buf0, buf1);
        store_rows(res, pitch, nd.n, bins, q0 + static_cast<uint64_t>(nd.a) * bins);
      }
      __syncthreads();
    }
    cluster.sync();
    // 2. column passes up to the root
    float* src = q0;
    float* dst = q1;
    uint32_t d = dS;
    while (true) {
      const uint32_t dn = cut_after(d, dS, p.levels);
      const uint32_t K = d - dn;
      const bool final_pass = dn == 0;
      const uint32_t R = final_pass ? p.final_rows : p.block_rows;
      const uint32_t nnodes = 1u << dn;
      const uint32_t maxn = (t.rows + nnodes - 1) >> dn;
      const uint32_t limit = final_pass ? t.rows_eval : maxn;
      const uint32_t bpn = (limit + R - 1) / R;
      const uint32_t units = nnodes * bpn;
      for (uint32_t u = rank; u < units; u += cs) {
        const Node X = node_at(u / bpn, t.rows, dn);
        const uint32_t s0 = (u % bpn) * R;
        const uint32_t s1 = umin32(s0 + R, final_pass ? t.rows_eval : X.n);
        if (s0 >= s1) continue;
        eval_column(p, X, s0, s1, K, src, bins, buf0, buf1, cmeta, counts);
        if (final_pass) {
          detect_rows(buf0, pitch, counts[0], s0, buf1, cp_pitch, da);
        } else {
          store_rows(buf0, pitch, counts[0], bins, dst + static_cast<uint64_t>(X.a + s0) * bins);
          __syncthreads();
        }
      }
      cluster.sync();
      if (final_pass) break;
      float* tmp = src;
      src = dst;
      dst = tmp;
      d = dn;
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

}  // namespace
}  // namespace gf

using namespace gf;

struct FfaClass {
  int cluster = 1;             // CTAs cooperating on one (series, task)
  std::vector<uint32_t> tasks;
  uint64_t max_elems = 0;      // rows * bins of the largest task (scratch per cluster)
  int nclusters = 0;           // resident clusters
  uint64_t scratch_offset = 0; // floats into the program scratch
  DeviceBlob tasks_d;
};

struct gf_ffa_program {
  int device = 0;
  std::vector<gf_ffa_task> tasks;
  std::vector<uint64_t> widths;
  std::vector<TaskDev> task_dev;
  std::vector<TrialDev> trial_dev;
  std::vector<OctaveDev> octaves;
  std::vector<MetaEntry> sub_meta;
  std::vector<uint32_t> sub_offset;
  std::vector<FfaClass> classes;
  uint64_t nsamples = 0;
  uint64_t prep_stride = 0;
  uint32_t max_bins = 0, max_width = 0;
  uint32_t pitch = 0, max_rows = 0, block_rows = 0, final_rows = 0, levels = 0;
  uint64_t halo = 0;
  uint64_t max_series = 0;
  uint64_t scratch_floats = 0;
  size_t smem_bytes = 0;
  DeviceBlob tasks_d, trials_d, octaves_d, sub_meta_d, sub_offset_d;
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

extern "C" int gf_ffa_program_create(const gf_ffa_task* tasks, uint64_t ntasks, const uint64_t* widths,
                                     uint64_t nwidths, uint64_t max_series, int32_t device_id,
                                     gf_ffa_program** out) {
  return guarded([&] {
    check_arg(tasks && widths && out, "null argument");
    *out = nullptr;
    check_arg(ntasks > 0, "FFA executor plan must contain at least one task");
    check_arg(nwidths > 0, "FFA search plan width_trials must not be empty");
    check_arg(nwidths <= kMaxWidths, "at most 64 width trials");
    check_arg(max_series > 0 && max_series < (1ull << 31), "max_series out of range");
    DeviceGuard dg(device_id);
    auto P = std::make_unique<gf_ffa_program>();
    P->device = device_id;
    P->tasks.assign(tasks, tasks + ntasks);
    P->widths.assign(widths, widths + nwidths);
    P->max_series = max_series;
    P->nsamples = tasks[0].input_nsamples;
    for (const auto& t : P->tasks) validate_task(t, P->nsamples);
    // octaves = distinct prepare keys in plan order
    std::map<double, uint32_t> octave_of;
    uint64_t off = 0;
    for (const auto& t : P->tasks) {
      if (octave_of.count(t.downsample_factor)) continue;
      octave_of[t.downsample_factor] = static_cast<uint32_t>(P->octaves.size());
      OctaveDev o{t.downsample_factor, t.prepared_nsamples, off};
      P->octaves.push_back(o);
      off = round_up(off + t.prepared_nsamples, 4);
      P->halo = std::max<uint64_t>(P->halo, static_cast<uint64_t>(std::ceil(t.downsample_factor)) + 2);
    }
    check_arg(P->octaves.size() <= 32, "at most 32 distinct downsample factors");
    P->prep_stride = round_up(off, 4);
    for (const auto& t : P->tasks) {
      check_arg(t.bins <= kMaxBins, "FFA CUDA path supports bins <= 512");
      check_arg(t.rows < 65536, "FFA CUDA path supports at most 65535 rows per task");
      P->max_bins = std::max<uint32_t>(P->max_bins, static_cast<uint32_t>(t.bins));
    }
    for (uint64_t w : P->widths) P->max_width = std::max<uint32_t>(P->max_width, static_cast<uint32_t>(w));
    // shared-memory geometry: two row buffers of max_rows rows, the column
    // schedules, sized for two CTAs per SM where possible
    P->pitch = P->max_bins | 1u;
    P->levels = 3;
    const size_t budget = 110 * 1024;
    auto smem_for = [&](uint32_t rows, uint32_t K) {
      return 2ull * rows * P->pitch * 4 + (K + 1ull) * rows * sizeof(MetaEntry) + 64;
    };
    uint32_t rows = 8;
    while (smem_for(rows + 1, P->levels) <= budget) ++rows;
    P->max_rows = rows;
    // R + 3 (2^K - 1) rows at the bottom of a column
    while (P->levels > 1 && static_cast<int>(rows) - 3 * ((1 << P->levels) - 1) < 8) --P->levels;
    P->block_rows = rows - 3 * ((1u << P->levels) - 1);
    const uint32_t cp_pitch = (P->max_bins + P->max_width + 2) | 1u;
    P->final_rows = std::min<uint32_t>(P->block_rows, (rows * P->pitch) / cp_pitch);
    check_arg(P->final_rows >= 1 && P->block_rows >= 1, "FFA bins too large for the shared-memory tiles");
    P->smem_bytes = smem_for(rows, P->levels);
    // subtree schedules for every size up to max_rows
    P->sub_offset.assign(rows + 1, 0u);
    for (uint32_t n = 1; n <= rows; ++n) {
      P->sub_offset[n] = static_cast<uint32_t>(P->sub_meta.size());
      build_subtree_schedule(n, P->sub_meta);
    }
    if (P->sub_meta.empty()) P->sub_meta.push_back(MetaEntry{});
    // tasks, trials and classes
    std::map<int, size_t> class_of;
    for (uint64_t i = 0; i < ntasks; ++i) {
      const auto& t = P->tasks[i];
      for (uint64_t w : P->widths)
        check_arg(w > 0 && w < t.bins, "FFA detection width trials must satisfy 0 < width < bins");
      TaskDev d{};
      d.bins = static_cast<uint32_t>(t.bins);
      d.rows = static_cast<uint32_t>(t.rows);
      d.rows_eval = static_cast<uint32_t>(t.rows_eval);
      d.octave = octave_of[t.downsample_factor];
      d.prep_offset = P->octaves[d.octave].offset;
      d.inv_stdnoise = 1.0f / task_stdnoise(t);
      d.ntrials = static_cast<uint32_t>(nwidths);
      d.trial_offset = static_cast<uint32_t>(P->trial_dev.size());
      d.max_width = P->max_width;
      // ffa_detection.cpp:60-80 make_boxcar_trials (float arithmetic)
      const float bf = static_cast<float>(t.bins);
      for (uint64_t w : P->widths) {
        const float wf = static_cast<float>(w);
        const float h = std::sqrt((bf - wf) / (bf * wf));
        P->trial_dev.push_back(TrialDev{h, wf / (bf - wf) * h, static_cast<uint32_t>(w), 0u});
      }
      uint32_t ds = 0;
      while (ceil_div(t.rows, 1ull << ds) > rows) ++ds;
      check_arg(ds <= 15, "FFA task too deep");
      d.split_depth = ds;
      P->task_dev.push_back(d);
      int cluster = 1;
      if (ds > 0) {
        cluster = 0;  // medium and large tasks: scratch; cluster sized by rows
        const uint64_t per = 512;
        int c = 1;
        while (c < kClusterSize && static_cast<uint64_t>(c) * per < t.rows) c *= 2;
        cluster = c;
      }
      // class key: 0 = on-chip (no scratch), else the cluster size
      const int key = ds == 0 ? 0 : cluster;
      if (!class_of.count(key)) {
        class_of[key] = P->classes.size();
        P->classes.emplace_back();
        P->classes.back().cluster = ds == 0 ? 1 : cluster;
      }
      FfaClass& c = P->classes[class_of[key]];
      c.tasks.push_back(static_cast<uint32_t>(i));
      if (ds > 0) c.max_elems = std::max<uint64_t>(c.max_elems, t.rows * t.bins);
    }
    cuda_check(cudaFuncSetAttribute(ffa_task_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(P->smem_bytes)),
               "cudaFuncSetAttribute(ffa_task_kernel)");
    cuda_check(cudaFuncSetAttribute(ffa_task_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
               "cudaFuncSetAttribute(cluster size)");
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_id), "device attribute");
    for (auto& c : P->classes) {
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(c.cluster, 1, 1);
      cfg.blockDim = dim3(kThreads, 1, 1);
      cfg.dynamicSmemBytes = P->smem_bytes;
      cudaLaunchAttribute attr{};
      attr.id = cudaLaunchAttributeClusterDimension;
      attr.val.clusterDim.x = c.cluster;
      attr.val.clusterDim.y = 1;
      attr.val.clusterDim.z = 1;
      cfg.attrs = &attr;
      cfg.numAttrs = 1;
      int n = 0;
      cuda_check(cudaOccupancyMaxActiveClusters(&n, ffa_task_kernel, &cfg), "cudaOccupancyMaxActiveClusters");
      check_arg(n > 0, "FFA kernel cannot be resident on this device");
      c.nclusters = n;
      if (c.max_elems) {
        c.scratch_offset = P->scratch_floats;
        P->scratch_floats += static_cast<uint64_t>(n) * 2 * c.max_elems;
      }
      c.tasks_d.upload(c.tasks.data(), c.tasks.size() * sizeof(uint32_t), device_id);
    }
    P->tasks_d.upload(P->task_dev.data(), P->task_dev.size() * sizeof(TaskDev), device_id);
    P->trials_d.upload(P->trial_dev.data(), P->trial_dev.size() * sizeof(TrialDev), device_id);
    P->octaves_d.upload(P->octaves.data(), P->octaves.size() * sizeof(OctaveDev), device_id);
    P->sub_meta_d.upload(P->sub_meta.data(), P->sub_meta.size() * sizeof(MetaEntry), device_id);
    P->sub_offset_d.upload(P->sub_offset.data(), P->sub_offset.size() * sizeof(uint32_t), device_id);
    *out = P.release();
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
    info->noctaves = P->octaves.size();
    info->prepared_floats = P->prep_stride;
    info->scratch_bytes = std::max<uint64_t>(16, P->scratch_floats * 4);
    uint64_t mx = 0;
    for (const auto& t : P->tasks) mx = std::max<uint64_t>(mx, t.rows * t.bins);
    info->max_task_elements = mx;
    info->metadata_bytes = P->tasks_d.bytes + P->trials_d.bytes + P->octaves_d.bytes + P->sub_meta_d.bytes +
                           P->sub_offset_d.bytes;
    for (const auto& c : P->classes) info->metadata_bytes += c.tasks_d.bytes;
    info->nclasses = P->classes.size();
  });
}

extern "C" int gf_ffa_prepare(gf_ffa_program* P, const float* dev_series, uint64_t nseries, uint64_t stride,
                              const double* dev_stats, float* dev_prepared, void* stream) {
  return guarded([&] {
    check_arg(P && dev_series && dev_prepared, "null argument");
    check_arg(nseries > 0 && nseries < 65536, "nseries out of range");
    check_arg(stride >= P->nsamples, "stride must be >= nsamples");
    DeviceGuard dg(P->device);
    const size_t smem = (kPrepareChunk + P->halo) * sizeof(float);
    check_arg(smem <= 200 * 1024, "downsample factor too large for the prepare kernel");
    cuda_check(cudaFuncSetAttribute(prepare_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)),
               "cudaFuncSetAttribute(prepare_kernel)");
    dim3 grid(static_cast<unsigned>(ceil_div(P->nsamples, kPrepareChunk)), static_cast<unsigned>(nseries));
    prepare_kernel<<<grid, kThreads, smem, as_stream(stream)>>>(
        dev_series, stride, P->nsamples, dev_stats, P->octaves_d.as<OctaveDev>(),
        static_cast<int>(P->octaves.size()), P->halo, dev_prepared, P->prep_stride);
    cuda_check(cudaGetLastError(), "prepare_kernel launch");
  });
}

extern "C" int gf_ffa_search(gf_ffa_program* P, const float* dev_prepared, uint64_t nseries, float snr_threshold,
                             void* dev_scratch, gf_peak_record* dev_peaks, uint64_t capacity,
                             uint64_t* dev_counters, void* stream) {
  return guarded([&] {
    check_arg(P && dev_prepared && dev_counters, "null argument");
    check_arg(std::isfinite(snr_threshold), "FFA search S/N threshold must be finite");
    check_arg(nseries > 0 && nseries <= P->max_series, "nseries must be in (0, max_series]");
    check_arg(capacity == 0 || dev_peaks != nullptr, "peak buffer must not be null");
    check_arg(P->scratch_floats == 0 || dev_scratch != nullptr, "FFA search needs scratch");
    DeviceGuard dg(P->device);
    auto s = as_stream(stream);
    cuda_check(cudaMemsetAsync(dev_counters, 0, 2 * sizeof(uint64_t), s), "cudaMemsetAsync(counters)");
    SearchParams sp{};
    sp.prepared = dev_prepared;
    sp.prep_stride = P->prep_stride;
    sp.tasks = P->tasks_d.as<TaskDev>();
    sp.trials = P->trials_d.as<TrialDev>();
    sp.sub_meta = P->sub_meta_d.as<MetaEntry>();
    sp.sub_offset = P->sub_offset_d.as<uint32_t>();
    sp.nseries = static_cast<uint32_t>(nseries);
    sp.threshold = snr_threshold;
    sp.peaks = dev_peaks;
    sp.capacity = capacity;
    sp.counters = reinterpret_cast<unsigned long long*>(dev_counters);
    sp.pitch = P->pitch;
    sp.max_rows = P->max_rows;
    sp.block_rows = P->block_rows;
    sp.final_rows = P->final_rows;
    sp.levels = P->levels;
    sp.error = reinterpret_cast<uint32_t*>(dev_counters + 1);
    // largest tasks first so the long clusters start early
    for (auto it = P->classes.rbegin(); it != P->classes.rend(); ++it) {
      const FfaClass& c = *it;
      sp.item_tasks = c.tasks_d.as<uint32_t>();
      sp.nitem_tasks = static_cast<uint32_t>(c.tasks.size());
      sp.scratch = c.max_elems ? static_cast<float*>(dev_scratch) + c.scratch_offset : nullptr;
      sp.scratch_elems = c.max_elems;
      const uint64_t items = nseries * c.tasks.size();
      const unsigned nclusters = static_cast<unsigned>(std::min<uint64_t>(items, static_cast<uint64_t>(c.nclusters)));
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(nclusters * c.cluster, 1, 1);
      cfg.blockDim = dim3(kThreads, 1, 1);
      cfg.dynamicSmemBytes = P->smem_bytes;
      cfg.stream = s;
      cudaLaunchAttribute attr{};
      attr.id = cudaLaunchAttributeClusterDimension;
      attr.val.clusterDim.x = c.cluster;
      attr.val.clusterDim.y = 1;
      attr.val.clusterDim.z = 1;
      cfg.attrs = &attr;
      cfg.numAttrs = 1;
      cuda_check(cudaLaunchKernelEx(&cfg, ffa_task_kernel, sp), "ffa_task_kernel launch");
    }
  });
}

extern "C" int gf_ffa_expand_peaks(const gf_ffa_program* P, const gf_peak_record* records, uint64_t n,
                                   uint64_t series_offset, double dm_low, double dm_step, gf_peak* out) {
  return guarded([&] {
    check_arg(P && (n == 0 || (records && out)), "null argument");
    for (uint64_t i = 0; i < n; ++i) {
      const gf_peak_record& r = records[i];
      check_arg(r.task < P->tasks.size() && r.width_index < P->widths.size(), "corrupt peak record");
      const gf_ffa_task& t = P->tasks[r.task];
      // ffa_detection.cpp:115-124 trial_period, :266-284 make_ffa_peak
      double period;
      if (t.rows <= 1) {
        period = t.effective_tsamp * static_cast<double>(t.bins);
      } else {
        const double b = static_cast<double>(t.bins);
        period = t.effective_tsamp * b * b / (b - static_cast<double>(r.shift) / static_cast<double>(t.rows - 1));
      }
      gf_peak& p = out[i];
      const uint64_t series = series_offset + r.series;
      p.dm = dm_low + static_cast<double>(series) * dm_step;
      p.dm_index = series;
      p.period = period;
      p.frequency = 1.0 / period;
      p.width = P->widths[r.width_index];
      p.duty_cycle = static_cast<double>(p.width) / static_cast<double>(t.bins);
      p.width_index = r.width_index;
      p.period_index = r.shift;
      p.phase = r.phase;
      p.shift = r.shift;
      p.bins = t.bins;
      p.snr = r.snr;
      p.reserved = 0;
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
