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
  uint32_t leaf_depth;    // depth of the on-chip subtrees (0: whole task)
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
// FFA tree helpers
// ---------------------------------------------------------------------------

struct Node {
  uint32_t a, n, depth;
};

// The node at depth `depth` containing row r of an n-row tree, stopping early
// at one-row nodes (their depth is then < `depth`).
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

struct MergeIdx {
  uint32_t head_row, tail_row, roll;
  bool head_leaf, tail_leaf;
};

// ffa.cpp:153-171 merge_row index arithmetic for output row s of node (a, n)
__device__ __forceinline__ MergeIdx merge_index(uint32_t a, uint32_t n, uint32_t s, uint32_t bins) {
  const uint32_t h = n >> 1, t = n - h;
  const float nm1 = static_cast<float>(n - 1);
  const float hsc = __fdiv_rn(static_cast<float>(h - 1), nm1);
  const float tsc = __fdiv_rn(static_cast<float>(t - 1), nm1);
  const uint32_t hs = static_cast<uint32_t>(__fadd_rn(__fmul_rn(hsc, static_cast<float>(s)), 0.5f));
  const uint32_t ts = static_cast<uint32_t>(__fadd_rn(__fmul_rn(tsc, static_cast<float>(s)), 0.5f));
  MergeIdx m;
  m.head_row = a + hs;
  m.tail_row = a + h + ts;
  m.roll = (s - ts) % bins;
  m.head_leaf = h == 1;
  m.tail_leaf = t == 1;
  return m;
}

// out[j] = head[j] + tail[(j + roll) mod bins] for one row, by one warp
__device__ __forceinline__ void merge_row_warp(const float* __restrict__ head, const float* __restrict__ tail,
                                               uint32_t roll, uint32_t bins, float* __restrict__ out, int lane) {
  for (uint32_t j = lane; j < bins; j += 32) {
    uint32_t k = j + roll;
    if (k >= bins) k -= bins;
    out[j] = __fadd_rn(head[j], tail[k]);
  }
}

__device__ __forceinline__ void merge_row_warp_global(const float* head, const float* tail, uint32_t roll,
                                                      uint32_t bins, float* out, int lane) {
  for (uint32_t j = lane; j < bins; j += 32) {
    uint32_t k = j + roll;
    if (k >= bins) k -= bins;
    __stcg(out + j, __fadd_rn(__ldcg(head + j), __ldcg(tail + k)));
  }
}

// Transforms the subtree rooted at node (a0, n0) (depth d0 of an n-row tree)
// on chip, for depths from the deepest up to `stop_depth` inclusive.  Input
// rows come from `input` (global); node outputs of depth d live in
// buf[d & 1] at row index (row - a0).  Returns nothing; callers read
// buf[stop_depth & 1].
__device__ void transform_subtree(const float* __restrict__ input, uint32_t nrows, uint32_t bins, uint32_t a0,
                                  uint32_t n0, uint32_t d0, uint32_t stop_depth, float* buf0, float* buf1,
                                  uint32_t pitch) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // deepest depth with a split inside the subtree
  uint32_t max_d = d0;
  {
    uint32_t n = n0;
    while (n > 1) { n = (n + 1) >> 1; ++max_d; }
  }
  for (int d = static_cast<int>(max_d) - 1; d >= static_cast<int>(stop_depth); --d) {
    float* out = (d & 1) ? buf1 : buf0;
    const float* prev = (d & 1) ? buf0 : buf1;
    for (uint32_t r = warp; r < n0; r += kThreads / 32) {
      const Node nd = node_of(a0 + r, nrows, static_cast<uint32_t>(d));
      if (nd.depth != static_cast<uint32_t>(d) || nd.n < 2) continue;
      const MergeIdx m = merge_index(nd.a, nd.n, a0 + r - nd.a, bins);
      const float* head = m.head_leaf ? input + static_cast<uint64_t>(m.head_row) * bins
                                      : prev + (m.head_row - a0) * pitch;
      const float* tail = m.tail_leaf ? input + static_cast<uint64_t>(m.tail_row) * bins
                                      : prev + (m.tail_row - a0) * pitch;
      merge_row_warp(head, tail, m.roll, bins, out + r * pitch, lane);
    }
    __syncthreads();
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

// rows[i] (pitch `pitch`) hold root rows shift0 + i, i < count.  Prefix sums
// are sequential per row (one thread per row, ffa_detection.cpp:126-139);
// each warp then scans one row for every width.
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
  const uint32_t* item_tasks;   // task indices of this launch's class
  uint32_t nitem_tasks;
  uint32_t nseries;
  float threshold;
  gf_peak_record* peaks;
  uint64_t capacity;
  unsigned long long* counters;
  float* scratch;               // per cluster: 2 * scratch_elems floats
  uint64_t scratch_elems;
  uint32_t max_bins;
  uint32_t smem_pitch;          // pitch the shared buffers were sized with
};

__device__ __forceinline__ uint32_t pitch_of(uint32_t bins) { return bins | 1u; }

// Detect the root rows [r0, r1) of a task whose root children are in
// `child` (smem or global scratch, pitch cpitch) or are input rows.
// rowbuf points at `avail` free floats of shared memory; the batch size is the
// number of (row, prefix) pairs that fit.
template <bool GlobalChildren>
__device__ void root_detect(const float* input, const float* child, uint32_t cpitch, uint32_t nrows,
                            uint32_t r0, uint32_t r1, float* rowbuf, uint32_t avail, const DetectArgs& da) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bins = da.bins;
  const uint32_t pitch = pitch_of(bins);
  const uint32_t cp_pitch = (bins + da.max_width + 2) | 1u;
  const uint32_t batch = umin32(kThreads, avail / (pitch + cp_pitch));
  float* cp = rowbuf + batch * pitch;
  for (uint32_t b0 = r0; b0 < r1; b0 += batch) {
    const uint32_t cnt = umin32(batch, r1 - b0);
    for (uint32_t i = warp; i < cnt; i += kThreads / 32) {
      const uint32_t s = b0 + i;
      if (nrows == 1) {
        for (uint32_t j = lane; j < bins; j += 32) rowbuf[i * pitch + j] = input[j];
        continue;
      }
      const MergeIdx m = merge_index(0, nrows, s, bins);
      const float* head = m.head_leaf ? input + static_cast<uint64_t>(m.head_row) * bins
                                      : child + static_cast<uint64_t>(m.head_row) * cpitch;
      const float* tail = m.tail_leaf ? input + static_cast<uint64_t>(m.tail_row) * bins
                                      : child + static_cast<uint64_t>(m.tail_row) * cpitch;
      if (GlobalChildren) {
        for (uint32_t j = lane; j < bins; j += 32) {
          uint32_t k = j + m.roll;
          if (k >= bins) k -= bins;
          const float hv = m.head_leaf ? head[j] : __ldcg(head + j);
          const float tv = m.tail_leaf ? tail[k] : __ldcg(tail + k);
          rowbuf[i * pitch + j] = __fadd_rn(hv, tv);
        }
      } else {
        merge_row_warp(head, tail, m.roll, bins, rowbuf + i * pitch, lane);
      }
    }
    __syncthreads();
    detect_rows(rowbuf, pitch, cnt, b0, cp, cp_pitch, da);
  }
}

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

// One CTA per (series, task): the whole tree on chip.
__global__ void __launch_bounds__(kThreads) ffa_small_kernel(SearchParams p) {
  extern __shared__ float sm[];
  const uint64_t nitems = static_cast<uint64_t>(p.nseries) * p.nitem_tasks;
  for (uint64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
    const uint32_t series = static_cast<uint32_t>(item / p.nitem_tasks);
    const uint32_t task = p.item_tasks[item % p.nitem_tasks];
    const TaskDev t = p.tasks[task];
    const float* input = p.prepared + series * p.prep_stride + t.prep_offset;
    const uint32_t pitch = pitch_of(t.bins);
    float* buf0 = sm;
    float* buf1 = sm + kLeafRows * pitch;
    // everything below the root
    transform_subtree(input, t.rows, t.bins, 0, t.rows, 0, 1, buf0, buf1, pitch);
    // root children are in buf1 (depth 1); the root rows go to detection in
    // batches held in buf0, which depth 1 does not use.
    const DetectArgs da = make_detect(p, t, series, task);
    root_detect<false>(input, buf1, pitch, t.rows, 0, t.rows_eval, buf0, kLeafRows * pitch, da);
  }
}

// A cluster of kClusterSize CTAs per (series, task) for tasks larger than a
// CTA.  Scratch (global, per cluster) holds two full task buffers.
__global__ void __cluster_dims__(kClusterSize, 1, 1) __launch_bounds__(kThreads)
    ffa_cluster_kernel(SearchParams p) {
  extern __shared__ float sm[];
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t rank = cluster.block_rank();
  const uint32_t cid = blockIdx.x / kClusterSize;
  const uint32_t nclusters = gridDim.x / kClusterSize;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* q0 = p.scratch + static_cast<uint64_t>(cid) * 2 * p.scratch_elems;
  float* q1 = q0 + p.scratch_elems;
  const uint64_t nitems = static_cast<uint64_t>(p.nseries) * p.nitem_tasks;
  for (uint64_t item = cid; item < nitems; item += nclusters) {
    const uint32_t series = static_cast<uint32_t>(item / p.nitem_tasks);
    const uint32_t task = p.item_tasks[item % p.nitem_tasks];
    const TaskDev t = p.tasks[task];
    const float* input = p.prepared + series * p.prep_stride + t.prep_offset;
    const uint32_t bins = t.bins, pitch = pitch_of(bins);
    const uint32_t dl = t.leaf_depth;
    float* buf0 = sm;
    float* buf1 = sm + kLeafRows * pitch;
    // 1. subtrees at depth dl, on chip, written to scratch[dl & 1]
    const uint32_t nleaves = 1u << dl;
    float* qdl = (dl & 1) ? q1 : q0;
    for (uint32_t leaf = rank; leaf < nleaves; leaf += kClusterSize) {
      // locate leaf `leaf` (bits MSB first)
      uint32_t a = 0, n = t.rows;
      for (uint32_t b = dl; b-- > 0;) {
        const uint32_t h = n >> 1;
        if ((leaf >> b) & 1u) { a += h; n -= h; } else { n = h; }
      }
      if (n > 1) transform_subtree(input, t.rows, bins, a, n, dl, dl, buf0, buf1, pitch);
      const float* src = (n > 1) ? ((dl & 1) ? buf1 : buf0) : nullptr;
      for (uint32_t r = warp; r < n; r += kThreads / 32)
        for (uint32_t j = lane; j < bins; j += 32)
          __stcg(qdl + static_cast<uint64_t>(a + r) * bins + j,
                 src ? src[r * pitch + j] : input[static_cast<uint64_t>(a + r) * bins + j]);
      __syncthreads();
    }
    cluster.sync();
    // 2. depths dl-1 .. 1 through scratch, rows split across the cluster
    const uint32_t rows_per = (t.rows + kClusterSize - 1) / kClusterSize;
    const uint32_t r0 = rank * rows_per, r1 = min(t.rows, r0 + rows_per);
    for (int d = static_cast<int>(dl) - 1; d >= 1; --d) {
      float* out = (d & 1) ? q1 : q0;
      const float* prev = (d & 1) ? q0 : q1;
      for (uint32_t r = r0 + warp; r < r1; r += kThreads / 32) {
        const Node nd = node_of(r, t.rows, static_cast<uint32_t>(d));
        const MergeIdx m = merge_index(nd.a, nd.n, r - nd.a, bins);
        merge_row_warp_global(prev + static_cast<uint64_t>(m.head_row) * bins,
                              prev + static_cast<uint64_t>(m.tail_row) * bins, m.roll, bins,
                              out + static_cast<uint64_t>(r) * bins, lane);
      }
      cluster.sync();
    }
    // 3. root rows [0, rows_eval) split across the cluster, fused detection
    const DetectArgs da = make_detect(p, t, series, task);
    const uint32_t ev_per = (t.rows_eval + kClusterSize - 1) / kClusterSize;
    const uint32_t e0 = min(t.rows_eval, rank * ev_per), e1 = min(t.rows_eval, e0 + ev_per);
    root_detect<true>(input, q1, bins, t.rows, e0, e1, sm, 2 * kLeafRows * p.smem_pitch, da);
    // scratch is reused by the next item
    cluster.sync();
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
  const MergeIdx m = merge_index(nd.a, nd.n, r - nd.a, bins);
  const float* head = m.head_leaf ? input + static_cast<uint64_t>(m.head_row) * bins
                                  : prev + static_cast<uint64_t>(m.head_row) * bins;
  const float* tail = m.tail_leaf ? input + static_cast<uint64_t>(m.tail_row) * bins
                                  : prev + static_cast<uint64_t>(m.tail_row) * bins;
  merge_row_warp(head, tail, m.roll, bins, out + static_cast<uint64_t>(r) * bins, lane);
}

}  // namespace
}  // namespace gf

using namespace gf;

struct gf_ffa_program {
  int device = 0;
  std::vector<gf_ffa_task> tasks;
  std::vector<uint64_t> widths;
  std::vector<TaskDev> task_dev;
  std::vector<TrialDev> trial_dev;
  std::vector<OctaveDev> octaves;
  std::vector<uint32_t> small_tasks, big_tasks;
  uint64_t nsamples = 0;
  uint64_t prep_stride = 0;
  uint64_t max_big_elems = 0;
  uint32_t max_bins = 0, max_width = 0;
  uint64_t halo = 0;
  uint64_t max_series = 0;
  int big_clusters = 0;
  int small_ctas = 0;
  size_t smem_bytes = 0;
  DeviceBlob tasks_d, trials_d, octaves_d, small_d, big_d;
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
    for (uint64_t i = 0; i < ntasks; ++i) {
      const auto& t = P->tasks[i];
      check_arg(t.bins <= kMaxBins, "FFA CUDA path supports bins <= 512");
      check_arg(t.rows < (1ull << 31), "FFA rows out of range");
      uint64_t mw = 0;
      for (uint64_t w : P->widths) {
        check_arg(w > 0 && w < t.bins, "FFA detection width trials must satisfy 0 < width < bins");
        mw = std::max(mw, w);
      }
      TaskDev d{};
      d.bins = static_cast<uint32_t>(t.bins);
      d.rows = static_cast<uint32_t>(t.rows);
      d.rows_eval = static_cast<uint32_t>(t.rows_eval);
      d.octave = octave_of[t.downsample_factor];
      d.prep_offset = P->octaves[d.octave].offset;
      d.inv_stdnoise = 1.0f / task_stdnoise(t);
      d.ntrials = static_cast<uint32_t>(nwidths);
      d.trial_offset = static_cast<uint32_t>(P->trial_dev.size());
      d.max_width = static_cast<uint32_t>(mw);
      // ffa_detection.cpp:60-80 make_boxcar_trials (float arithmetic)
      const float bf = static_cast<float>(t.bins);
      for (uint64_t w : P->widths) {
        const float wf = static_cast<float>(w);
        const float h = std::sqrt((bf - wf) / (bf * wf));
        P->trial_dev.push_back(TrialDev{h, wf / (bf - wf) * h, static_cast<uint32_t>(w), 0u});
      }
      // leaf depth: smallest d with ceil(rows / 2^d) <= kLeafRows
      uint32_t dl = 0;
      while (ceil_div(t.rows, 1ull << dl) > static_cast<uint64_t>(kLeafRows)) ++dl;
      d.leaf_depth = dl;
      P->task_dev.push_back(d);
      P->max_bins = std::max<uint32_t>(P->max_bins, d.bins);
      P->max_width = std::max<uint32_t>(P->max_width, d.max_width);
      if (dl == 0) {
        P->small_tasks.push_back(static_cast<uint32_t>(i));
      } else {
        P->big_tasks.push_back(static_cast<uint32_t>(i));
        P->max_big_elems = std::max<uint64_t>(P->max_big_elems, t.rows * t.bins);
      }
    }
    // two kLeafRows-row transform buffers; detection batches reuse them
    const size_t pitch = P->max_bins | 1u;
    P->smem_bytes = 2ull * kLeafRows * pitch * sizeof(float);
    cuda_check(cudaFuncSetAttribute(ffa_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(P->smem_bytes)),
               "cudaFuncSetAttribute(ffa_small_kernel)");
    cuda_check(cudaFuncSetAttribute(ffa_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(P->smem_bytes)),
               "cudaFuncSetAttribute(ffa_cluster_kernel)");
    int sms = 0, per_sm = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_id), "device attribute");
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ffa_small_kernel, kThreads, P->smem_bytes),
               "occupancy(ffa_small_kernel)");
    P->small_ctas = std::max(1, sms * std::max(1, per_sm));
    if (!P->big_tasks.empty()) {
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(kClusterSize, 1, 1);
      cfg.blockDim = dim3(kThreads, 1, 1);
      cfg.dynamicSmemBytes = P->smem_bytes;
      cudaLaunchAttribute attr{};
      attr.id = cudaLaunchAttributeClusterDimension;
      attr.val.clusterDim.x = kClusterSize;
      attr.val.clusterDim.y = 1;
      attr.val.clusterDim.z = 1;
      cfg.attrs = &attr;
      cfg.numAttrs = 1;
      int nclusters = 0;
      cuda_check(cudaOccupancyMaxActiveClusters(&nclusters, ffa_cluster_kernel, &cfg),
                 "cudaOccupancyMaxActiveClusters");
      check_arg(nclusters > 0, "FFA cluster kernel cannot be resident on this device");
      P->big_clusters = nclusters;
    }
    std::vector<uint32_t> dummy{0u};
    P->tasks_d.upload(P->task_dev.data(), P->task_dev.size() * sizeof(TaskDev), device_id);
    P->trials_d.upload(P->trial_dev.data(), P->trial_dev.size() * sizeof(TrialDev), device_id);
    P->octaves_d.upload(P->octaves.data(), P->octaves.size() * sizeof(OctaveDev), device_id);
    const auto& sm_list = P->small_tasks.empty() ? dummy : P->small_tasks;
    const auto& bg_list = P->big_tasks.empty() ? dummy : P->big_tasks;
    P->small_d.upload(sm_list.data(), sm_list.size() * sizeof(uint32_t), device_id);
    P->big_d.upload(bg_list.data(), bg_list.size() * sizeof(uint32_t), device_id);
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
    info->scratch_bytes = static_cast<uint64_t>(std::max(1, P->big_clusters)) * 2 * std::max<uint64_t>(1, P->max_big_elems) * 4;
    uint64_t mx = 0;
    for (const auto& t : P->tasks) mx = std::max<uint64_t>(mx, t.rows * t.bins);
    info->max_task_elements = mx;
    info->metadata_bytes = P->tasks_d.bytes + P->trials_d.bytes + P->octaves_d.bytes + P->small_d.bytes + P->big_d.bytes;
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
    DeviceGuard dg(P->device);
    auto s = as_stream(stream);
    cuda_check(cudaMemsetAsync(dev_counters, 0, 2 * sizeof(uint64_t), s), "cudaMemsetAsync(counters)");
    SearchParams sp{};
    sp.prepared = dev_prepared;
    sp.prep_stride = P->prep_stride;
    sp.tasks = P->tasks_d.as<TaskDev>();
    sp.trials = P->trials_d.as<TrialDev>();
    sp.nseries = static_cast<uint32_t>(nseries);
    sp.threshold = snr_threshold;
    sp.peaks = dev_peaks;
    sp.capacity = capacity;
    sp.counters = reinterpret_cast<unsigned long long*>(dev_counters);
    sp.max_bins = P->max_bins;
    sp.smem_pitch = P->max_bins | 1u;
    if (!P->small_tasks.empty()) {
      sp.item_tasks = P->small_d.as<uint32_t>();
      sp.nitem_tasks = static_cast<uint32_t>(P->small_tasks.size());
      const uint64_t items = nseries * P->small_tasks.size();
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(items, static_cast<uint64_t>(P->small_ctas)));
      ffa_small_kernel<<<grid, kThreads, P->smem_bytes, s>>>(sp);
      cuda_check(cudaGetLastError(), "ffa_small_kernel launch");
    }
    if (!P->big_tasks.empty()) {
      check_arg(dev_scratch != nullptr, "FFA search needs scratch for large tasks");
      sp.item_tasks = P->big_d.as<uint32_t>();
      sp.nitem_tasks = static_cast<uint32_t>(P->big_tasks.size());
      sp.scratch = static_cast<float*>(dev_scratch);
      sp.scratch_elems = P->max_big_elems;
      const uint64_t items = nseries * P->big_tasks.size();
      const unsigned nclusters =
          static_cast<unsigned>(std::min<uint64_t>(items, static_cast<uint64_t>(P->big_clusters)));
      ffa_cluster_kernel<<<nclusters * kClusterSize, kThreads, P->smem_bytes, s>>>(sp);
      cuda_check(cudaGetLastError(), "ffa_cluster_kernel launch");
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
