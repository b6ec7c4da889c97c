// Learned DM/period proposal: coarse features and a small 1-D convolutional
// network with hand-written forward and backward kernels (bf16 activations and
// weights, fp32 accumulation, fp32 master weights updated by Adam).
//
// The network scores coarse DM trials.  Its input for one coarse DM is a
// [32 subbands][L] bf16 map: for each subband's coarse dedispersed series,
// the harmonic-summed power spectrum max-pooled into L log-spaced frequency
// bins (7 octaves x 64 bins).  Layers (zero-padded, stride 1):
//   conv 32->64 k9 ReLU, conv 64->64 k9 ReLU, conv 64->32 k9 ReLU,
//   conv 32->1 k1 (per-bin score s), then per octave o
//   logit[o] = log(mean_{bins of o} exp(s))    (a smooth maximum)
// trained with binary cross-entropy (positive weight pw) against labels
// derived from the exhaustive search's candidates.
//
// This component has no counterpart in the reference: the exhaustive search
// (every other file of this library) stays the fallback and the measure of
// its recall.
#include <cuda_bf16.h>

#include "common.cuh"

#include <cmath>

namespace gf {
namespace {

constexpr int kThreads = 256;
constexpr int kTileT = 64;    // output positions per block
constexpr int kTileC = 16;    // output channels per block
constexpr int kMaxCin = 64;
constexpr int kMaxK = 9;

__device__ __forceinline__ float load_f(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ float load_f(const float* p) { return *p; }
__device__ __forceinline__ void store_f(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ void store_f(float* p, float v) { *p = v; }

// y[b][co][t] = act(bias[co] + sum_{ci,k} W(co,ci,k) x[b][ci][t + k - K/2])
// where W(co,ci,k) = w[co][ci][k] (forward) or, for the data gradient of a
// forward layer with weights w[ci][co][*] (transposed = 1), w[ci][co][K-1-k].
template <typename TIn, typename TOut>
__global__ void __launch_bounds__(kThreads) conv_kernel(const TIn* __restrict__ x, const __nv_bfloat16* __restrict__ w,
                                                        const float* __restrict__ bias, TOut* __restrict__ y, int cin,
                                                        int cout, int L, int K, int transposed, int relu) {
  extern __shared__ float sm[];
  const int b = blockIdx.z;
  const int t0 = blockIdx.x * kTileT;
  const int c0 = blockIdx.y * kTileC;
  const int P = K / 2;
  const int W = kTileT + K - 1;
  float* xs = sm;                 // [cin][W]
  float* ws = sm + cin * W;       // [kTileC][cin][K]
  const TIn* xb = x + static_cast<size_t>(b) * cin * L;
  for (int i = threadIdx.x; i < cin * W; i += kThreads) {
    const int ci = i / W, j = i % W;
    const int t = t0 + j - P;
    xs[i] = (t >= 0 && t < L) ? load_f(xb + static_cast<size_t>(ci) * L + t) : 0.0f;
  }
  for (int i = threadIdx.x; i < kTileC * cin * K; i += kThreads) {
    const int c = i / (cin * K), r = i % (cin * K), ci = r / K, k = r % K;
    const int co = c0 + c;
    float v = 0.0f;
    if (co < cout)
      v = transposed ? __bfloat162float(w[(static_cast<size_t>(ci) * cout + co) * K + (K - 1 - k)])
                     : __bfloat162float(w[(static_cast<size_t>(co) * cin + ci) * K + k]);
    ws[i] = v;
  }
  __syncthreads();
  const int c = threadIdx.x / 16;        // output channel within the tile
  const int tg = (threadIdx.x % 16) * 4; // first of four output positions
  const int co = c0 + c;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  const float* wr = ws + c * cin * K;
  for (int ci = 0; ci < cin; ++ci) {
    const float* xr = xs + ci * W + tg;
    for (int k = 0; k < K; ++k) {
      const float wv = wr[ci * K + k];
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[j] = fmaf(wv, xr[j + k], acc[j]);
    }
  }
  if (co >= cout) return;
  const float bv = bias ? bias[co] : 0.0f;
  TOut* yr = y + (static_cast<size_t>(b) * cout + co) * L;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int t = t0 + tg + j;
    if (t < L) {
      float v = acc[j] + bv;
      if (relu) v = fmaxf(v, 0.0f);
      store_f(yr + t, v);
    }
  }
}

// dz = dy * (y > 0), in place on dy (fp32), y the bf16 post-ReLU output
__global__ void relu_grad_kernel(float* __restrict__ dy, const __nv_bfloat16* __restrict__ y, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    if (!(__bfloat162float(y[i]) > 0.0f)) dy[i] = 0.0f;
}

// dw[co][ci][k] += sum_{b,t} dz[b][co][t] x[b][ci][t + k - K/2]; db[co] += sum dz.
// One block per (co, 16 input channels); threads own (ci, k) pairs and stream
// the batch through shared memory tiles.
__global__ void __launch_bounds__(kThreads) conv_wgrad_kernel(const float* __restrict__ dz,
                                                              const __nv_bfloat16* __restrict__ x,
                                                              float* __restrict__ dw, float* __restrict__ db, int B,
                                                              int cin, int cout, int L, int K) {
  __shared__ float zs[kTileT];
  __shared__ float xs[16][kTileT + kMaxK - 1];
  const int co = blockIdx.x;
  const int ci0 = blockIdx.y * 16;
  const int P = K / 2;
  const int W = kTileT + K - 1;
  const int my_ci = threadIdx.x / K, my_k = threadIdx.x % K;
  const bool owner = threadIdx.x < 16 * K && ci0 + my_ci < cin;
  float acc = 0.0f, bacc = 0.0f;
  for (int b = 0; b < B; ++b) {
    for (int t0 = 0; t0 < L; t0 += kTileT) {
      __syncthreads();
      if (threadIdx.x < kTileT) {
        const int t = t0 + threadIdx.x;
        zs[threadIdx.x] = t < L ? dz[(static_cast<size_t>(b) * cout + co) * L + t] : 0.0f;
      }
      for (int i = threadIdx.x; i < 16 * W; i += kThreads) {
        const int c = i / W, j = i % W;
        const int t = t0 + j - P;
        const int ci = ci0 + c;
        xs[c][j] = (ci < cin && t >= 0 && t < L) ? __bfloat162float(x[(static_cast<size_t>(b) * cin + ci) * L + t])
                                                 : 0.0f;
      }
      __syncthreads();
      if (owner) {
        for (int j = 0; j < kTileT; ++j) acc = fmaf(zs[j], xs[my_ci][j + my_k], acc);
      }
      if (blockIdx.y == 0 && threadIdx.x == 0) {
        for (int j = 0; j < kTileT; ++j) bacc += zs[j];
      }
    }
  }
  if (owner) dw[(static_cast<size_t>(co) * cin + ci0 + my_ci) * K + my_k] += acc;
  if (blockIdx.y == 0 && threadIdx.x == 0 && db) db[co] += bacc;
}

// Head, octave pooling and loss (one block per sample b and octave o, 64 bins
// per octave, one thread per bin):
//   s[t] = bh + sum_c wh[c] y[b][c][t]
//   logit = log(mean_t exp(s[t]))
//   loss += pw*y*softplus(-logit) + (1-y)*softplus(logit)
// With grads != 0 also dlogit = sigmoid(logit)*(1-y+pw*y) - pw*y and
//   ds[t] = dlogit * softmax(s)[t], dy[b][c][t] = wh[c] ds[t],
//   dwh[c] += sum_t ds[t] y[b][c][t], dbh += sum_t ds[t].
__global__ void __launch_bounds__(64) head_kernel(const __nv_bfloat16* __restrict__ y, const float* __restrict__ wh,
                                                  const float* __restrict__ bh, int C, int L, int bins,
                                                  const float* __restrict__ labels, float pw, float* __restrict__ logits,
                                                  float* __restrict__ loss, float* __restrict__ dy,
                                                  float* __restrict__ dwh, float* __restrict__ dbh) {
  const int b = blockIdx.x, o = blockIdx.y, O = gridDim.y;
  const int t = o * bins + threadIdx.x;
  __shared__ float red[64];
  __shared__ float sh_logit, sh_dlogit;
  float s = -INFINITY;
  if (threadIdx.x < bins && t < L) {
    s = bh[0];
    for (int c = 0; c < C; ++c) s = fmaf(wh[c], __bfloat162float(y[(static_cast<size_t>(b) * C + c) * L + t]), s);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int off = 32; off > 0; off >>= 1) {
    if (threadIdx.x < off) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + off]);
    __syncthreads();
  }
  const float m = red[0];
  __syncthreads();
  const float e = (s == -INFINITY) ? 0.0f : expf(s - m);
  red[threadIdx.x] = e;
  __syncthreads();
  for (int off = 32; off > 0; off >>= 1) {
    if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  const float sum = red[0];
  if (threadIdx.x == 0) {
    const float z = m + logf(sum) - logf(static_cast<float>(bins));
    sh_logit = z;
    logits[static_cast<size_t>(b) * O + o] = z;
    if (labels) {
      const float lab = labels[static_cast<size_t>(b) * O + o];
      const float sp_neg = fmaxf(-z, 0.0f) + log1pf(expf(-fabsf(z)));   // softplus(-z)
      const float sp_pos = fmaxf(z, 0.0f) + log1pf(expf(-fabsf(z)));    // softplus(z)
      atomicAdd(loss, pw * lab * sp_neg + (1.0f - lab) * sp_pos);
      const float sig = 1.0f / (1.0f + expf(-z));
      sh_dlogit = sig * (1.0f - lab + pw * lab) - pw * lab;
    }
  }
  __syncthreads();
  if (dy == nullptr || labels == nullptr) return;
  const float ds = (threadIdx.x < bins && t < L) ? sh_dlogit * e / sum : 0.0f;
  __syncthreads();
  if (threadIdx.x < bins && t < L) {
    for (int c = 0; c < C; ++c) dy[(static_cast<size_t>(b) * C + c) * L + t] = wh[c] * ds;
  }
  // dwh[c] and dbh: block reductions over the 64 bins
  for (int c = 0; c <= C; ++c) {
    float v = 0.0f;
    if (threadIdx.x < bins && t < L)
      v = c < C ? ds * __bfloat162float(y[(static_cast<size_t>(b) * C + c) * L + t]) : ds;
    red[threadIdx.x] = v;
    __syncthreads();
    for (int off = 32; off > 0; off >>= 1) {
      if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
      __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(c < C ? &dwh[c] : dbh, red[0]);
    __syncthreads();
  }
}

// Adam on fp32 master weights; refreshes the bf16 copy the kernels read.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, __nv_bfloat16* __restrict__ pb, size_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2, float scale) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float gi = g[i] * scale;
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (pb) pb[i] = __float2bfloat16_rn(pi);
  }
}

// Features: for each series s, power p[s][0..nf) (normalised so white noise
// has mean 1 per bin), the harmonic sum H(k) = max over h in {1,2,4,8} of
// (sum_{m=1..h} p[m k] - h) / sqrt(h), then for every log bin j the maximum of
// H(k) over the Fourier bins k whose frequency k*df lies in [lo_j, hi_j) (the
// nearest bin when the range holds none), compressed as sign(H) log1p(|H|).
__global__ void __launch_bounds__(kThreads) features_kernel(const float* __restrict__ p, int nf, float df,
                                                            const float* __restrict__ edges, int L,
                                                            __nv_bfloat16* __restrict__ feat) {
  const int s = blockIdx.y;
  const int j = blockIdx.x * kThreads + threadIdx.x;
  if (j >= L) return;
  const float* ps = p + static_cast<size_t>(s) * nf;
  int k0 = static_cast<int>(ceilf(edges[j] / df));
  int k1 = static_cast<int>(ceilf(edges[j + 1] / df));
  if (k1 <= k0) {
    k0 = static_cast<int>(rintf(0.5f * (edges[j] + edges[j + 1]) / df));
    k1 = k0 + 1;
  }
  k0 = max(k0, 1);
  float best = -INFINITY;
  for (int k = k0; k < k1; ++k) {
    float acc = 0.0f;
    float h_best = -INFINITY;
    int h = 0;
    for (int hm = 1; hm <= 8; hm <<= 1) {
      for (; h < hm; ++h) {
        const long long kk = static_cast<long long>(k) * (h + 1);
        acc += kk < nf ? ps[kk] : 1.0f;
      }
      h_best = fmaxf(h_best, (acc - static_cast<float>(hm)) * rsqrtf(static_cast<float>(hm)));
    }
    best = fmaxf(best, h_best);
  }
  if (best == -INFINITY) best = 0.0f;
  const float v = copysignf(log1pf(fabsf(best)), best);
  feat[static_cast<size_t>(s) * L + j] = __float2bfloat16_rn(v);
}

// coarse[row][t] = sum_{i<f} in[row][t*f + i] (uint32 in, float out)
__global__ void downsample_kernel(const uint32_t* __restrict__ in, uint64_t in_stride, uint64_t nrows, int f,
                                  uint64_t nout, float* __restrict__ out, uint64_t out_stride) {
  const uint64_t total = nrows * nout;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t r = i / nout, t = i % nout;
    const uint32_t* src = in + r * in_stride + t * f;
    uint64_t acc = 0;
    for (int k = 0; k < f; ++k) acc += src[k];
    out[r * out_stride + t] = static_cast<float>(acc);
  }
}

unsigned grid_for(size_t n) { return static_cast<unsigned>(std::min<size_t>(ceil_div(n, 256), 148 * 16)); }

}  // namespace
}  // namespace gf

using namespace gf;

extern "C" int gf_prop_conv_forward(const void* x, const void* w, const float* bias, void* y, int32_t batch,
                                    int32_t cin, int32_t cout, int32_t length, int32_t ksize, int32_t relu,
                                    void* stream) {
  return guarded([&] {
    check_arg(x && w && y, "null argument");
    check_arg(batch > 0 && cin > 0 && cin <= kMaxCin && cout > 0 && length > 0, "conv shape out of range");
    check_arg(ksize > 0 && ksize <= kMaxK && (ksize & 1), "conv kernel size must be odd and <= 9");
    const size_t smem = (static_cast<size_t>(cin) * (kTileT + ksize - 1) + kTileC * cin * ksize) * sizeof(float);
    auto k = conv_kernel<__nv_bfloat16, __nv_bfloat16>;
    cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
               "cudaFuncSetAttribute(conv)");
    dim3 grid(static_cast<unsigned>(ceil_div(length, kTileT)), static_cast<unsigned>(ceil_div(cout, kTileC)),
              static_cast<unsigned>(batch));
    k<<<grid, kThreads, smem, as_stream(stream)>>>(static_cast<const __nv_bfloat16*>(x),
                                                   static_cast<const __nv_bfloat16*>(w), bias,
                                                   static_cast<__nv_bfloat16*>(y), cin, cout, length, ksize, 0, relu);
    cuda_check(cudaGetLastError(), "conv_kernel launch");
  });
}

extern "C" int gf_prop_conv_backward(const float* dy, const void* y_act, const void* x, const void* w, float* dx,
                                     float* dw, float* db, int32_t batch, int32_t cin, int32_t cout, int32_t length,
                                     int32_t ksize, void* stream) {
  return guarded([&] {
    check_arg(dy && x && w && dw, "null argument");
    check_arg(batch > 0 && cin > 0 && cin <= kMaxCin && cout > 0 && cout <= kMaxCin && length > 0,
              "conv shape out of range");
    check_arg(ksize > 0 && ksize <= kMaxK && (ksize & 1), "conv kernel size must be odd and <= 9");
    auto s = as_stream(stream);
    float* dz = const_cast<float*>(dy);
    const size_t n = static_cast<size_t>(batch) * cout * length;
    if (y_act) relu_grad_kernel<<<grid_for(n), 256, 0, s>>>(dz, static_cast<const __nv_bfloat16*>(y_act), n);
    dim3 wg(static_cast<unsigned>(cout), static_cast<unsigned>(ceil_div(cin, 16)));
    conv_wgrad_kernel<<<wg, kThreads, 0, s>>>(dz, static_cast<const __nv_bfloat16*>(x), dw, db, batch, cin, cout,
                                               length, ksize);
    if (dx) {
      const size_t smem = (static_cast<size_t>(cout) * (kTileT + ksize - 1) + kTileC * cout * ksize) * sizeof(float);
      auto k = conv_kernel<float, float>;
      cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                 "cudaFuncSetAttribute(conv)");
      dim3 grid(static_cast<unsigned>(ceil_div(length, kTileT)), static_cast<unsigned>(ceil_div(cin, kTileC)),
                static_cast<unsigned>(batch));
      k<<<grid, kThreads, smem, s>>>(dz, static_cast<const __nv_bfloat16*>(w), nullptr, dx, cout, cin, length, ksize,
                                     1, 0);
    }
    cuda_check(cudaGetLastError(), "conv backward launch");
  });
}

extern "C" int gf_prop_head(const void* y, const float* wh, const float* bh, int32_t batch, int32_t channels,
                            int32_t length, int32_t octaves, const float* labels, float pos_weight, float* logits,
                            float* loss, float* dy, float* dwh, float* dbh, void* stream) {
  return guarded([&] {
    check_arg(y && wh && bh && logits, "null argument");
    check_arg(octaves > 0 && length % octaves == 0 && length / octaves <= 64, "octave bins must be <= 64");
    check_arg(labels == nullptr || loss != nullptr, "loss needed with labels");
    check_arg(dy == nullptr || (labels && dwh && dbh), "gradients need labels, dwh and dbh");
    dim3 grid(static_cast<unsigned>(batch), static_cast<unsigned>(octaves));
    head_kernel<<<grid, 64, 0, as_stream(stream)>>>(static_cast<const __nv_bfloat16*>(y), wh, bh, channels, length,
                                                    length / octaves, labels, pos_weight, logits, loss, dy, dwh, dbh);
    cuda_check(cudaGetLastError(), "head_kernel launch");
  });
}

extern "C" int gf_prop_adam(float* param, const float* grad, float* m, float* v, void* param_bf16, uint64_t n,
                            float lr, float beta1, float beta2, float eps, int32_t step, float grad_scale,
                            void* stream) {
  return guarded([&] {
    check_arg(param && grad && m && v && step > 0, "invalid Adam arguments");
    const float c1 = 1.0f - std::pow(beta1, static_cast<float>(step));
    const float c2 = 1.0f - std::pow(beta2, static_cast<float>(step));
    adam_kernel<<<grid_for(n), 256, 0, as_stream(stream)>>>(param, grad, m, v,
                                                            static_cast<__nv_bfloat16*>(param_bf16), n, lr, beta1,
                                                            beta2, eps, c1, c2, grad_scale);
    cuda_check(cudaGetLastError(), "adam_kernel launch");
  });
}

extern "C" int gf_prop_features(const float* power, uint64_t nseries, uint64_t nfreq, double df, const float* edges,
                                int32_t nbins, void* feat, void* stream) {
  return guarded([&] {
    check_arg(power && edges && feat, "null argument");
    check_arg(nseries > 0 && nseries < 65536 && nfreq > 1 && nbins > 0 && df > 0.0, "feature shape out of range");
    dim3 grid(static_cast<unsigned>(ceil_div(nbins, kThreads)), static_cast<unsigned>(nseries));
    features_kernel<<<grid, kThreads, 0, as_stream(stream)>>>(power, static_cast<int>(nfreq), static_cast<float>(df),
                                                              edges, nbins, static_cast<__nv_bfloat16*>(feat));
    cuda_check(cudaGetLastError(), "features_kernel launch");
  });
}

extern "C" int gf_prop_downsample(const uint32_t* in, uint64_t in_stride, uint64_t nrows, int32_t factor,
                                  uint64_t nout, float* out, uint64_t out_stride, void* stream) {
  return guarded([&] {
    check_arg(in && out && factor > 0, "invalid downsample arguments");
    check_arg(nout * static_cast<uint64_t>(factor) <= in_stride, "downsample reads beyond the input row");
    downsample_kernel<<<grid_for(nrows * nout), 256, 0, as_stream(stream)>>>(in, in_stride, nrows, factor, nout, out,
                                                                             out_stride);
    cuda_check(cudaGetLastError(), "downsample_kernel launch");
  });
}
