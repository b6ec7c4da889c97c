// Candidate selection on the device for large raw-peak sets.
//
// select_candidates_cpu (candidate.cpp:175-212) sorts every raw peak by
// frequency (then width, DM index and is_better_dm_peak), splits the sorted
// list where consecutive frequencies differ by more than radius / T_obs,
// sorts each frequency group by DM index (then width, frequency), splits it
// where the DM index jumps by more than the DM radius (or, unless clustering
// across widths, where the width changes), and keeps the best peak of every
// cluster with the cluster's count and DM / frequency extent.  Workloads with
// strong RFI produce 10^8 raw peaks, whose expansion to 96-byte host records
// and host sort dominate the search.  Here the compact device records are
// expanded on the device (make_ffa_peak arithmetic, ffa_detection.cpp:266-284),
// ordered by stable radix sorts of 64-bit keys (least significant key first,
// so the result is the lexicographic order of the reference's comparators),
// split by device scans and reduced per cluster; only one record per cluster
// returns to the host, where the candidates are ranked (is_better_candidate)
// as on the CPU.
//
// Ties: the reference sorts each frequency group with std::sort, which leaves
// peaks that agree in (DM index, width, frequency) in an unspecified order.
// Here they keep the frequency-sorted order, one of the orders std::sort may
// give; cluster boundaries, counts, extents and best peaks do not depend on
// the order of such ties.
#include "common.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

namespace gf {
namespace {

constexpr int kThreads = 256;

struct TaskPeriod {
  double effective_tsamp;
  uint32_t bins, rows;
};

struct DevPeak {
  double frequency;
  double period;
  float snr;
  uint32_t dm_index;
  uint32_t shift;
  uint16_t phase;
  uint16_t width;
  uint16_t bins;
  uint16_t width_index;
  uint32_t reserved;
};
static_assert(sizeof(DevPeak) == 40, "DevPeak is 40 bytes");

// Per-cluster aggregate.  The best peak is carried as its rank in the
// is_better_dm_peak order (0 = best), so merging two aggregates is pure
// arithmetic: the reduction never reads memory through a carried value
// (a device reduction may apply its operator to the unloaded tail items of
// its last tile, whose fields are arbitrary).
struct ClusterAgg {
  uint32_t best_rank;
  uint32_t count;
  uint32_t dm_min, dm_max;
  double f_min, f_max;
};

// descending order-preserving key of a finite float (-0.0 counts as 0.0,
// as the reference's != comparison does)
__device__ __forceinline__ uint32_t snr_desc_key(float f) {
  const uint32_t u = __float_as_uint(f == 0.0f ? 0.0f : f);
  const uint32_t asc = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  return ~asc;
}


// make_ffa_peak with trial_period (ffa_detection.cpp:115-124,266-284), in the
// operation order of the host expansion.  status bit 1: a non-finite value
// (the reference rejects it in candidate selection); bit 2: a corrupt record;
// bit 4: a DM index or width beyond the sort keys' fields.
__global__ void expand_kernel(const gf_peak_record* __restrict__ rec, uint64_t n, uint64_t dm_offset,
                              const TaskPeriod* __restrict__ tasks, uint32_t ntasks,
                              const uint64_t* __restrict__ widths, uint32_t nwidths, DevPeak* __restrict__ out,
                              uint32_t* status) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i >= n) return;
  const gf_peak_record r = rec[i];
  DevPeak p{};
  if (r.task >= ntasks || r.width_index >= nwidths) {
    atomicOr(status, 2u);
    out[i] = p;
    return;
  }
  const TaskPeriod t = tasks[r.task];
  double period;
  if (t.rows <= 1) {
    period = __dmul_rn(t.effective_tsamp, static_cast<double>(t.bins));
  } else {
    const double b = static_cast<double>(t.bins);
    period = __ddiv_rn(__dmul_rn(__dmul_rn(t.effective_tsamp, b), b),
                       __dsub_rn(b, __ddiv_rn(static_cast<double>(r.shift), static_cast<double>(t.rows - 1))));
  }
  p.period = period;
  p.frequency = __ddiv_rn(1.0, period);
  p.snr = r.snr;
  p.dm_index = static_cast<uint32_t>(dm_offset + r.series);
  p.shift = r.shift;
  p.phase = r.phase;
  p.width = static_cast<uint16_t>(widths[r.width_index]);
  p.bins = static_cast<uint16_t>(t.bins);
  p.width_index = r.width_index;
  if (!isfinite(p.snr) || !isfinite(p.period) || !isfinite(p.frequency)) atomicOr(status, 1u);
  if (dm_offset + r.series >= (1ull << 22) || widths[r.width_index] >= 1024) atomicOr(status, 4u);
  out[i] = p;
}

__global__ void iota_kernel(uint32_t* idx, uint64_t n) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i < n) idx[i] = static_cast<uint32_t>(i);
}

// keys of the least-significant-first passes of peak_order
// (candidate.cpp:64-76 over is_better_dm_peak):
//   0: phase, shift, bins   1: period   2: width, DM index, S/N descending
//   3: frequency
__global__ void peak_order_key_kernel(const DevPeak* __restrict__ peaks, const uint32_t* __restrict__ idx,
                                      uint64_t n, int pass, uint64_t* __restrict__ keys) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i >= n) return;
  const DevPeak p = peaks[idx[i]];
  uint64_t k;
  switch (pass) {
    case 0:
      k = (static_cast<uint64_t>(p.phase) << 48) | (static_cast<uint64_t>(p.shift) << 16) | p.bins;
      break;
    case 1:
      k = static_cast<uint64_t>(__double_as_longlong(p.period));
      break;
    case 2:
      k = (static_cast<uint64_t>(p.width) << 54) | (static_cast<uint64_t>(p.dm_index) << 32) | snr_desc_key(p.snr);
      break;
    default:
      k = static_cast<uint64_t>(__double_as_longlong(p.frequency));
      break;
  }
  keys[i] = k;
}

// keys of the least-significant-first passes of is_better_dm_peak
// (dm_search.cpp:89-100 over ffa_peak.cpp:16-45; finite peaks, dm follows
// dm_index, equal periods give equal frequencies):
//   0: DM index   1: phase, shift, bins   2: width   3: period   4: S/N descending
__global__ void better_key_kernel(const DevPeak* __restrict__ peaks, const uint32_t* __restrict__ idx, uint64_t n,
                                  int pass, uint64_t* __restrict__ keys) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i >= n) return;
  const DevPeak p = peaks[idx[i]];
  uint64_t k;
  switch (pass) {
    case 0:
      k = p.dm_index;
      break;
    case 1:
      k = (static_cast<uint64_t>(p.phase) << 48) | (static_cast<uint64_t>(p.shift) << 16) | p.bins;
      break;
    case 2:
      k = p.width;
      break;
    case 3:
      k = static_cast<uint64_t>(__double_as_longlong(p.period));
      break;
    default:
      k = snr_desc_key(p.snr);
      break;
  }
  keys[i] = k;
}

// rank[order[r]] = r
__global__ void rank_kernel(const uint32_t* __restrict__ order, uint64_t n, uint32_t* __restrict__ rank) {
  const uint64_t r = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (r < n) rank[order[r]] = static_cast<uint32_t>(r);
}

// 1 where the sorted frequency steps by more than the radius (candidate.cpp:190-199)
__global__ void frequency_split_kernel(const DevPeak* __restrict__ peaks, const uint32_t* __restrict__ idx,
                                       uint64_t n, double radius_hz, uint32_t* __restrict__ flag) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i >= n) return;
  flag[i] = i > 0 && __dsub_rn(peaks[idx[i]].frequency, peaks[idx[i - 1]].frequency) > radius_hz ? 1u : 0u;
}

// dm_group_order (or width_then_dm_group_order) within frequency groups:
// group id in the high word, then DM index and width (candidate.cpp:78-94)
__global__ void group_key_kernel(const DevPeak* __restrict__ peaks, const uint32_t* __restrict__ idx,
                                 const uint32_t* __restrict__ group, uint64_t n, int across_widths,
                                 uint64_t* __restrict__ keys) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i >= n) return;
  const DevPeak p = peaks[idx[i]];
  const uint64_t g = static_cast<uint64_t>(group[i]) << 32;
  keys[i] = across_widths ? g | (static_cast<uint64_t>(p.dm_index) << 10) | p.width
                          : g | (static_cast<uint64_t>(p.width) << 22) | p.dm_index;
}

// cluster starts (append_dm_clusters, candidate.cpp:140-171) and the
// per-peak aggregate seeds
__global__ void cluster_split_kernel(const DevPeak* __restrict__ peaks, const uint32_t* __restrict__ idx,
                                     const uint32_t* __restrict__ rank, const uint64_t* __restrict__ keys,
                                     uint64_t n, int across_widths, uint64_t dm_radius,
                                     uint32_t* __restrict__ flag, ClusterAgg* __restrict__ seed) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i >= n) return;
  const DevPeak p = peaks[idx[i]];
  uint32_t f = 0u;
  if (i > 0) {
    const DevPeak q = peaks[idx[i - 1]];
    const bool new_group = (keys[i] >> 32) != (keys[i - 1] >> 32);
    const bool same_width = across_widths || p.width == q.width;
    const bool same_dm = p.dm_index <= q.dm_index || static_cast<uint64_t>(p.dm_index - q.dm_index) <= dm_radius;
    f = (new_group || !same_width || !same_dm) ? 1u : 0u;
  }
  flag[i] = f;
  seed[i] = ClusterAgg{rank[idx[i]], 1u, p.dm_index, p.dm_index, p.frequency, p.frequency};
}

struct MergeClusters {
  __device__ __forceinline__ ClusterAgg operator()(const ClusterAgg& a, const ClusterAgg& b) const {
    ClusterAgg c;
    c.best_rank = min(a.best_rank, b.best_rank);
    c.count = a.count + b.count;
    c.dm_min = min(a.dm_min, b.dm_min);
    c.dm_max = max(a.dm_max, b.dm_max);
    c.f_min = fmin(a.f_min, b.f_min);
    c.f_max = fmax(a.f_max, b.f_max);
    return c;
  }
};

__global__ void gather_best_kernel(const DevPeak* __restrict__ peaks, const uint32_t* __restrict__ order,
                                   const ClusterAgg* __restrict__ agg, const uint32_t* __restrict__ nclusters,
                                   uint64_t n, DevPeak* __restrict__ best) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
  if (i < *nclusters && agg[i].best_rank < n) best[i] = peaks[order[agg[i].best_rank]];
}

unsigned blocks_for(uint64_t n) { return static_cast<unsigned>(std::max<uint64_t>(1, ceil_div(n, kThreads))); }

struct Layout {
  size_t peaks, keys_a, keys_b, idx_a, idx_b, order_a, order_b, rank, u32_a, u32_b, seeds, aggs, best, counters,
      temp, temp_bytes, total;
};

// workspace carve-up for n peaks (256-byte aligned pieces)
Layout layout_for(uint64_t n, cudaStream_t s) {
  size_t temp = 0, t = 0;
  cub::DoubleBuffer<uint64_t> kb(nullptr, nullptr);
  cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
  cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, t, kb, vb, static_cast<int64_t>(n), 0, 64, s),
             "cub::DeviceRadixSort size");
  temp = std::max(temp, t);
  cuda_check(cub::DeviceScan::InclusiveSum(nullptr, t, static_cast<uint32_t*>(nullptr),
                                           static_cast<uint32_t*>(nullptr), static_cast<int64_t>(n), s),
             "cub::DeviceScan size");
  temp = std::max(temp, t);
  cuda_check(cub::DeviceReduce::ReduceByKey(nullptr, t, static_cast<uint32_t*>(nullptr),
                                            static_cast<uint32_t*>(nullptr), static_cast<ClusterAgg*>(nullptr),
                                            static_cast<ClusterAgg*>(nullptr), static_cast<uint32_t*>(nullptr),
                                            MergeClusters{}, static_cast<int64_t>(n), s),
             "cub::DeviceReduce size");
  temp = std::max(temp, t);
  Layout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = round_up(off + bytes, 256);
    return at;
  };
  L.peaks = take(n * sizeof(DevPeak));
  L.keys_a = take(n * 8);
  L.keys_b = take(n * 8);
  L.idx_a = take(n * 4);
  L.idx_b = take(n * 4);
  L.order_a = take(n * 4);
  L.order_b = take(n * 4);
  L.rank = take(n * 4);
  L.u32_a = take(n * 4);
  L.u32_b = take(n * 4);
  L.seeds = take(n * sizeof(ClusterAgg));
  L.aggs = take(n * sizeof(ClusterAgg));
  L.best = take(n * sizeof(DevPeak));
  L.counters = take(16);
  L.temp = take(temp);
  L.temp_bytes = temp;
  L.total = off;
  return L;
}

}  // namespace

// the sort of candidates by is_better_candidate (host.cpp)
void rank_candidates(std::vector<gf_candidate>& candidates);

}  // namespace gf

using namespace gf;

extern "C" int gf_select_candidates_device_workspace(uint64_t npeaks, uint64_t* bytes) {
  return guarded([&] {
    check_arg(bytes != nullptr, "null argument");
    check_arg(npeaks < (1ull << 31), "at most 2^31 - 1 peaks per candidate selection");
    *bytes = layout_for(std::max<uint64_t>(npeaks, 1), nullptr).total;
  });
}

extern "C" int gf_select_candidates_device(const gf_ffa_program* program, const gf_peak_record* dev_records,
                                           const gf_peak_segment* segments, uint64_t nsegments, double dm_low,
                                           double dm_step, double observation_seconds,
                                           const gf_candidate_options* o, void* dev_workspace,
                                           uint64_t workspace_bytes, gf_candidate* out, uint64_t capacity,
                                           uint64_t* ncandidates, void* stream) {
  return guarded([&] {
    check_arg(program && o && ncandidates && (nsegments == 0 || segments), "null argument");
    check_arg(observation_seconds > 0.0 && std::isfinite(observation_seconds),
              "Candidate selection observation_seconds must be finite and > 0");
    check_arg(o->frequency_cluster_radius >= 0.0 && std::isfinite(o->frequency_cluster_radius),
              "Candidate selection frequency_cluster_radius must be finite and >= 0");
    *ncandidates = 0;
    uint64_t n = 0;
    for (uint64_t k = 0; k < nsegments; ++k) n += segments[k].record_count;
    if (n == 0) return;
    check_arg(dev_records != nullptr && dev_workspace != nullptr, "null argument");
    check_arg(n < (1ull << 31), "at most 2^31 - 1 peaks per candidate selection");
    std::vector<PeakTaskInfo> tinfo;
    std::vector<uint64_t> widths;
    int device = 0;
    ffa_program_peak_tables(program, tinfo, widths, device);
    DeviceGuard dg(device);
    auto s = as_stream(stream);
    const Layout L = layout_for(n, s);
    check_arg(workspace_bytes >= L.total, "candidate workspace smaller than gf_select_candidates_device_workspace");
    char* ws = static_cast<char*>(dev_workspace);
    DevPeak* peaks = reinterpret_cast<DevPeak*>(ws + L.peaks);
    uint64_t* ka = reinterpret_cast<uint64_t*>(ws + L.keys_a);
    uint64_t* kb = reinterpret_cast<uint64_t*>(ws + L.keys_b);
    uint32_t* ia = reinterpret_cast<uint32_t*>(ws + L.idx_a);
    uint32_t* ib = reinterpret_cast<uint32_t*>(ws + L.idx_b);
    uint32_t* oa = reinterpret_cast<uint32_t*>(ws + L.order_a);
    uint32_t* ob = reinterpret_cast<uint32_t*>(ws + L.order_b);
    uint32_t* rank = reinterpret_cast<uint32_t*>(ws + L.rank);
    uint32_t* ua = reinterpret_cast<uint32_t*>(ws + L.u32_a);
    uint32_t* ub = reinterpret_cast<uint32_t*>(ws + L.u32_b);
    ClusterAgg* seeds = reinterpret_cast<ClusterAgg*>(ws + L.seeds);
    ClusterAgg* aggs = reinterpret_cast<ClusterAgg*>(ws + L.aggs);
    DevPeak* best = reinterpret_cast<DevPeak*>(ws + L.best);
    uint32_t* counters = reinterpret_cast<uint32_t*>(ws + L.counters);  // [0] status, [1] clusters
    void* temp = ws + L.temp;
    // the task table and widths: small, uploaded per call
    std::vector<TaskPeriod> tp(tinfo.size());
    for (size_t i = 0; i < tinfo.size(); ++i)
      tp[i] = TaskPeriod{tinfo[i].effective_tsamp, static_cast<uint32_t>(tinfo[i].bins),
                         static_cast<uint32_t>(tinfo[i].rows)};
    DeviceBlob tasks_d, widths_d;
    tasks_d.upload(tp.data(), tp.size() * sizeof(TaskPeriod), device);
    widths_d.upload(widths.data(), widths.size() * sizeof(uint64_t), device);
    cuda_check(cudaMemsetAsync(counters, 0, 16, s), "cudaMemsetAsync(candidate counters)");
    uint64_t at = 0;
    for (uint64_t k = 0; k < nsegments; ++k) {
      const gf_peak_segment& g = segments[k];
      if (g.record_count == 0) continue;
      expand_kernel<<<blocks_for(g.record_count), kThreads, 0, s>>>(
          dev_records + g.record_begin, g.record_count, g.series_offset, tasks_d.as<TaskPeriod>(),
          static_cast<uint32_t>(tp.size()), widths_d.as<uint64_t>(), static_cast<uint32_t>(widths.size()),
          peaks + at, counters);
      at += g.record_count;
    }
    cuda_check(cudaGetLastError(), "expand_kernel launch");
    const int64_t nn = static_cast<int64_t>(n);
    size_t temp_bytes = L.temp_bytes;
    cub::DoubleBuffer<uint64_t> keys(ka, kb);
    // rank of every peak in the is_better_dm_peak order: five stable passes
    iota_kernel<<<blocks_for(n), kThreads, 0, s>>>(oa, n);
    cub::DoubleBuffer<uint32_t> order(oa, ob);
    for (int pass = 0; pass < 5; ++pass) {
      better_key_kernel<<<blocks_for(n), kThreads, 0, s>>>(peaks, order.Current(), n, pass, keys.Current());
      cuda_check(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, order, nn, 0, 64, s), "best-peak sort");
    }
    rank_kernel<<<blocks_for(n), kThreads, 0, s>>>(order.Current(), n, rank);
    // peak_order: four stable passes, least significant key first
    iota_kernel<<<blocks_for(n), kThreads, 0, s>>>(ia, n);
    cub::DoubleBuffer<uint32_t> idx(ia, ib);
    for (int pass = 0; pass < 4; ++pass) {
      peak_order_key_kernel<<<blocks_for(n), kThreads, 0, s>>>(peaks, idx.Current(), n, pass, keys.Current());
      cuda_check(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, idx, nn, 0, 64, s), "peak sort");
    }
    // frequency groups
    frequency_split_kernel<<<blocks_for(n), kThreads, 0, s>>>(peaks, idx.Current(), n,
                                                               o->frequency_cluster_radius / observation_seconds, ua);
    cuda_check(cub::DeviceScan::InclusiveSum(temp, temp_bytes, ua, ub, nn, s), "group scan");
    // DM order within groups (stable: ties keep the frequency order)
    group_key_kernel<<<blocks_for(n), kThreads, 0, s>>>(peaks, idx.Current(), ub, n, o->cluster_across_widths,
                                                         keys.Current());
    cuda_check(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, idx, nn, 0, 64, s), "group sort");
    // clusters and their aggregates
    cluster_split_kernel<<<blocks_for(n), kThreads, 0, s>>>(peaks, idx.Current(), rank, keys.Current(), n,
                                                             o->cluster_across_widths, o->dm_cluster_radius, ua,
                                                             seeds);
    cuda_check(cub::DeviceScan::InclusiveSum(temp, temp_bytes, ua, ub, nn, s), "cluster scan");
    cuda_check(cub::DeviceReduce::ReduceByKey(temp, temp_bytes, ub, ua, seeds, aggs, counters + 1,
                                              MergeClusters{}, nn, s),
               "cluster reduce");
    gather_best_kernel<<<blocks_for(n), kThreads, 0, s>>>(peaks, order.Current(), aggs, counters + 1, n, best);
    cuda_check(cudaGetLastError(), "candidate kernels");
    uint32_t host_counters[2] = {0, 0};
    cuda_check(cudaMemcpyAsync(host_counters, counters, 8, cudaMemcpyDeviceToHost, s), "candidate counters");
    cuda_check(cudaStreamSynchronize(s), "candidate selection");
    if (host_counters[0] & 2u) raise(GF_EINVAL, "corrupt peak record");
    if (host_counters[0] & 4u) raise(GF_EINVAL, "device candidate selection takes DM indices below 2^22 and widths below 1024");
    if (host_counters[0] & 1u) raise(GF_EINVAL, "Candidate selection peaks must contain finite scientific values");
    const uint32_t nc = host_counters[1];
    std::vector<ClusterAgg> agg(nc);
    std::vector<DevPeak> bp(nc);
    cuda_check(cudaMemcpy(agg.data(), aggs, nc * sizeof(ClusterAgg), cudaMemcpyDeviceToHost), "cluster aggregates");
    cuda_check(cudaMemcpy(bp.data(), best, nc * sizeof(DevPeak), cudaMemcpyDeviceToHost), "cluster best peaks");
    std::vector<gf_candidate> cands(nc);
    for (uint32_t c = 0; c < nc; ++c) {
      const DevPeak& p = bp[c];
      gf_peak q{};
      q.dm = dm_low + static_cast<double>(p.dm_index) * dm_step;  // as cuda_dm_search_benchmark.cpp:255-258
      q.dm_index = p.dm_index;
      q.period = p.period;
      q.frequency = p.frequency;
      q.width = p.width;
      q.duty_cycle = static_cast<double>(p.width) / static_cast<double>(p.bins);
      q.width_index = p.width_index;
      q.period_index = p.shift;
      q.phase = p.phase;
      q.shift = p.shift;
      q.bins = p.bins;
      q.snr = p.snr;
      gf_candidate& k = cands[c];
      k.dm = q.dm;
      k.dm_index = q.dm_index;
      k.period = q.period;
      k.frequency = q.frequency;
      k.width = q.width;
      k.duty_cycle = q.duty_cycle;
      k.snr = q.snr;
      k.peak_count = agg[c].count;
      k.dm_index_min = agg[c].dm_min;
      k.dm_index_max = agg[c].dm_max;
      k.frequency_min = agg[c].f_min;
      k.frequency_max = agg[c].f_max;
      k.best_peak = q;
      if (!std::isfinite(k.duty_cycle) || !std::isfinite(k.dm))
        raise(GF_EINVAL, "Candidate selection peaks must contain finite scientific values");
    }
    rank_candidates(cands);
    if (o->max_candidates != 0 && cands.size() > o->max_candidates) cands.resize(o->max_candidates);
    *ncandidates = cands.size();
    if (out && capacity)
      std::copy(cands.begin(), cands.begin() + static_cast<ptrdiff_t>(std::min<uint64_t>(capacity, cands.size())),
                out);
  });
}
