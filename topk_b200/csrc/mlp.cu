// Learned k-th-score model: features from the partition statistics, and a small
// MLP (in -> 64 -> 64 -> 1, ReLU, FP32) trained and served by the kernels here.
//
// No reference counterpart: the reference's pruning only uses exact bounds
// (cpu/VTA.h:210-216, cpu/PTA.h:337-340).  The model predicts a query's k-th score
// so that a pruned scan can start from a high threshold; the scan's own count
// decides whether the prediction may be used (topk_abi.cpp), so exactness never
// depends on the model.
//
// Features of a query (F = 2d + 18 values), with S = sum_m |weights[attr[m]]|:
//   [0, d)        the weight on each attribute (summed over repeats) / S
//   [d, 2d)       ln(|that| ) for the queried attributes, 0 for the others
//   2d            log2(k) / 10
//   2d+1          qq / 16
//   2d+2..2d+9    the 1st, 2nd, 4th, ..., 128th largest partition bound / S, bound =
//                 sum_m w_m * (w_m >= 0 ? max : min) over the partition's values
//   2d+10..2d+17  the same ranks of the partition mean scores sum_m w_m * mean / S
// Target: u = qq * ln(gap / S) with gap = (largest bound - k-th score), at least
// 1e-9 S.  Near the top of a sum of qq attributes the number of objects within g of
// the largest bound grows about like g^qq, so an error e in u scales the objects
// above the predicted cut by about e^e whatever qq is.  Cut from a prediction u:
//   cut = largest bound - S * exp((u + margin) / qq).
//
// Parameters, one flat FP32 array: W1[64][F] b1[64] W2[64][64] b2[64] w3[64] b3.
// Training: kTrainCtas blocks, data-parallel over each batch, every step a gradient
// reduction and an Adam update split over the blocks (mlp_train_kernel); each epoch
// visits the samples in the order (a*i + c) mod N, gcd(a, N) = 1.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "batch_internal.h"
#include "block_select.cuh"
#include "device_common.cuh"

namespace topk {

uint32_t mlp_param_count(uint32_t F) { return kHid * F + kHid + kHid * kHid + kHid + kHid + 1; }

namespace {

__device__ __forceinline__ uint32_t param_count(uint32_t F) { return kHid * F + kHid + kHid * kHid + kHid + kHid + 1; }

constexpr int kMT = 256;        // threads of the training / gradient block
constexpr uint32_t kMB = 128;   // largest batch of one step

struct Net {
  float *W1, *b1, *W2, *b2, *w3, *b3;
};

__device__ __forceinline__ Net net_at(float *base, uint32_t F) {
  Net n;
  n.W1 = base;
  n.b1 = n.W1 + kHid * F;
  n.W2 = n.b1 + kHid;
  n.b2 = n.W2 + kHid * kHid;
  n.w3 = n.b2 + kHid;
  n.b3 = n.w3 + kHid;
  return n;
}

// Forward and backward of B samples of a batch of Bn (MSE loss over Bn); adds their
// share of the gradient into g (each element owned by one thread) and of the batch's
// mean squared error into *loss.
// X [B][F], y [B], H1/H2 [B][64], dy [B] in shared memory; ends with a barrier.
__device__ void batch_grad(const Net &p, const Net &g, const float *X, const float *y, uint32_t B, uint32_t F,
                           float *H1, float *H2, float *dy, float *loss, float Bn) {
  const int t = threadIdx.x;
  for (uint32_t e = t; e < B * kHid; e += kMT) {
    const uint32_t i = e / kHid, j = e % kHid;
    float s = p.b1[j];
    for (uint32_t f = 0; f < F; ++f) s = fmaf(p.W1[j * F + f], X[i * F + f], s);
    H1[e] = fmaxf(s, 0.0f);
  }
  __syncthreads();
  for (uint32_t e = t; e < B * kHid; e += kMT) {
    const uint32_t i = e / kHid, j = e % kHid;
    float s = p.b2[j];
    for (uint32_t l = 0; l < kHid; ++l) s = fmaf(p.W2[j * kHid + l], H1[i * kHid + l], s);
    H2[e] = fmaxf(s, 0.0f);
  }
  __syncthreads();
  for (uint32_t i = t; i < B; i += kMT) {
    float s = p.b3[0];
    for (uint32_t j = 0; j < kHid; ++j) s = fmaf(p.w3[j], H2[i * kHid + j], s);
    const float r = s - y[i];
    dy[i] = 2.0f * r / Bn;
    atomicAdd(loss, r * r / Bn);
  }
  __syncthreads();
  for (uint32_t j = t; j < kHid; j += kMT) {
    float s = 0.0f;
    for (uint32_t i = 0; i < B; ++i) s = fmaf(dy[i], H2[i * kHid + j], s);
    g.w3[j] += s;
  }
  if (t == 0) {
    float s = 0.0f;
    for (uint32_t i = 0; i < B; ++i) s += dy[i];
    g.b3[0] += s;
  }
  __syncthreads();
  for (uint32_t e = t; e < B * kHid; e += kMT) {  // D2 = dy * w3 where the unit was active
    const uint32_t i = e / kHid, j = e % kHid;
    H2[e] = H2[e] > 0.0f ? dy[i] * p.w3[j] : 0.0f;
  }
  __syncthreads();
  for (uint32_t e = t; e < kHid * kHid; e += kMT) {
    const uint32_t j = e / kHid, l = e % kHid;
    float s = 0.0f;
    for (uint32_t i = 0; i < B; ++i) s = fmaf(H2[i * kHid + j], H1[i * kHid + l], s);
    g.W2[e] += s;
  }
  for (uint32_t j = t; j < kHid; j += kMT) {
    float s = 0.0f;
    for (uint32_t i = 0; i < B; ++i) s += H2[i * kHid + j];
    g.b2[j] += s;
  }
  __syncthreads();
  constexpr uint32_t kPer = kMB * kHid / kMT;  // outputs of D1 per thread
  float d1[kPer];
#pragma unroll
  for (uint32_t r = 0; r < kPer; ++r) {
    const uint32_t e = t + r * kMT;
    d1[r] = 0.0f;
    if (e < B * kHid) {
      const uint32_t i = e / kHid, l = e % kHid;
      float s = 0.0f;
      for (uint32_t j = 0; j < kHid; ++j) s = fmaf(H2[i * kHid + j], p.W2[j * kHid + l], s);
      d1[r] = H1[e] > 0.0f ? s : 0.0f;
    }
  }
  __syncthreads();
#pragma unroll
  for (uint32_t r = 0; r < kPer; ++r) {
    const uint32_t e = t + r * kMT;
    if (e < B * kHid) H1[e] = d1[r];
  }
  __syncthreads();
  for (uint32_t e = t; e < kHid * F; e += kMT) {
    const uint32_t j = e / F, f = e % F;
    float s = 0.0f;
    for (uint32_t i = 0; i < B; ++i) s = fmaf(H1[i * kHid + j], X[i * F + f], s);
    g.W1[e] += s;
  }
  for (uint32_t j = t; j < kHid; j += kMT) {
    float s = 0.0f;
    for (uint32_t i = 0; i < B; ++i) s += H1[i * kHid + j];
    g.b1[j] += s;
  }
  __syncthreads();
}

// Shared layout of the single-block kernels: params | grad | X[kMB][F] | y | dy | H1 | H2 | loss
size_t mlp_smem(uint32_t F) {
  const size_t P = mlp_param_count(F);
  return (2 * P + (size_t)kMB * F + 2 * kMB + 2 * (size_t)kMB * kHid + 4) * sizeof(float);
}

struct MlpShared {
  float *params, *grad, *X, *y, *dy, *H1, *H2, *loss;
};

__device__ MlpShared mlp_shared(unsigned char *smem, uint32_t F) {
  const uint32_t P = param_count(F);
  MlpShared s;
  s.params = reinterpret_cast<float *>(smem);
  s.grad = s.params + P;
  s.X = s.grad + P;
  s.y = s.X + kMB * F;
  s.dy = s.y + kMB;
  s.H1 = s.dy + kMB;
  s.H2 = s.H1 + kMB * kHid;
  s.loss = s.H2 + kMB * kHid;
  return s;
}

// One batch: gradient and loss at the given parameters, no update.
__global__ void __launch_bounds__(kMT) mlp_grad_kernel(const float *__restrict__ params, const float *__restrict__ X,
                                                       const float *__restrict__ y, uint32_t B, uint32_t F,
                                                       float *__restrict__ grad, float *__restrict__ loss) {
  extern __shared__ __align__(16) unsigned char smem[];
  MlpShared s = mlp_shared(smem, F);
  const uint32_t P = param_count(F);
  for (uint32_t e = threadIdx.x; e < P; e += kMT) {
    s.params[e] = params[e];
    s.grad[e] = 0.0f;
  }
  for (uint32_t e = threadIdx.x; e < B * F; e += kMT) s.X[e] = X[e];
  for (uint32_t e = threadIdx.x; e < B; e += kMT) s.y[e] = y[e];
  if (threadIdx.x == 0) *s.loss = 0.0f;
  __syncthreads();
  batch_grad(net_at(s.params, F), net_at(s.grad, F), s.X, s.y, B, F, s.H1, s.H2, s.dy, s.loss, (float)B);
  for (uint32_t e = threadIdx.x; e < P; e += kMT) grad[e] = s.grad[e];
  if (threadIdx.x == 0) *loss = *s.loss;
}

// Grid barrier with a bounded wait (the training kernel is launched cooperatively, so
// every CTA is resident and the wait ends unless a CTA failed): returns false once a
// wait ran out or another CTA's did, after setting bar->err.
struct GridBar {
  unsigned int count, gen, err, pad;
};

__device__ bool grid_barrier(GridBar *bar, uint64_t limit) {
  __shared__ unsigned int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int g = ld_volatile_u32(&bar->gen);
    __threadfence();
    if (atomicAdd(&bar->count, 1u) == gridDim.x - 1u) {
      bar->count = 0u;  // everyone has arrived: reset for the next barrier, then release
      __threadfence();
      atomicExch(&bar->gen, g + 1u);
      ok_s = 1u;
    } else {
      uint64_t it = 0;
      while (ld_volatile_u32(&bar->gen) == g && !ld_volatile_u32(&bar->err) && it < limit) {
        __nanosleep(32);
        ++it;
      }
      ok_s = ld_volatile_u32(&bar->gen) != g ? 1u : 0u;
      if (!ok_s) atomicExch(&bar->err, 1u);
    }
    __threadfence();
    if (ld_volatile_u32(&bar->err)) ok_s = 0u;  // one decision for the whole block
  }
  __syncthreads();
  return ok_s != 0u;
}

// Training: epochs x floor(N / B) Adam steps, data-parallel over the grid.  In each
// step CTA c computes the gradient of its share of the batch (samples
// [c*B/G, (c+1)*B/G)) into gpart[c]; after a grid barrier CTA c sums the G partial
// gradients (in CTA order: deterministic) for its slice of the parameters and applies
// Adam to that slice in global memory; after a second barrier every CTA reloads the
// parameters.  mul/add: per-epoch visiting order (mul coprime with N).  m, v: Adam
// moments, epoch_loss: zeroed by the caller; epoch_loss[e] = mean batch loss of epoch e.
__global__ void __launch_bounds__(kMT) mlp_train_kernel(float *__restrict__ params, float *__restrict__ m,
                                                        float *__restrict__ v, const float *__restrict__ X,
                                                        const float *__restrict__ y, uint64_t N, uint32_t F,
                                                        uint32_t B, uint32_t epochs, const uint64_t *__restrict__ mul,
                                                        const uint64_t *__restrict__ add, float lr,
                                                        float *__restrict__ epoch_loss, float *__restrict__ gpart,
                                                        GridBar *bar, uint64_t wait_limit) {
  extern __shared__ __align__(16) unsigned char smem[];
  MlpShared s = mlp_shared(smem, F);
  const uint32_t P = param_count(F);
  const uint32_t G = gridDim.x, c = blockIdx.x;
  const uint32_t i0 = (uint32_t)((uint64_t)B * c / G), i1 = (uint32_t)((uint64_t)B * (c + 1) / G);
  const uint32_t nb = i1 - i0;
  const uint32_t e0 = (uint32_t)((uint64_t)P * c / G), e1 = (uint32_t)((uint64_t)P * (c + 1) / G);
  for (uint32_t e = threadIdx.x; e < P; e += kMT) s.params[e] = params[e];
  const Net pn = net_at(s.params, F), gn = net_at(s.grad, F);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float b1t = 1.0f, b2t = 1.0f;
  const uint64_t steps = N / B;
  float *mine = gpart + (size_t)c * P;
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    if (threadIdx.x == 0) *s.loss = 0.0f;
    for (uint64_t st = 0; st < steps; ++st) {
      __syncthreads();
      for (uint32_t e = threadIdx.x; e < P; e += kMT) s.grad[e] = 0.0f;
      for (uint32_t e = threadIdx.x; e < nb * F; e += kMT) {
        const uint32_t i = e / F, f = e % F;
        const uint64_t idx = (mul[ep] * (st * B + i0 + i) + add[ep]) % N;
        s.X[e] = X[idx * F + f];
        if (f == 0) s.y[i] = y[idx];
      }
      __syncthreads();
      batch_grad(pn, gn, s.X, s.y, nb, F, s.H1, s.H2, s.dy, s.loss, (float)B);
      for (uint32_t e = threadIdx.x; e < P; e += kMT) mine[e] = s.grad[e];
      if (!grid_barrier(bar, wait_limit)) return;
      b1t *= b1;
      b2t *= b2;
      const float c1 = 1.0f / (1.0f - b1t), c2 = 1.0f / (1.0f - b2t);
      for (uint32_t e = e0 + threadIdx.x; e < e1; e += kMT) {
        float gr = 0.0f;
        for (uint32_t j = 0; j < G; ++j) gr += __ldcg(gpart + (size_t)j * P + e);
        const float mm = b1 * m[e] + (1.0f - b1) * gr;
        const float vv = b2 * v[e] + (1.0f - b2) * gr * gr;
        m[e] = mm;
        v[e] = vv;
        params[e] = s.params[e] - lr * (mm * c1) / (sqrtf(vv * c2) + eps);
      }
      if (!grid_barrier(bar, wait_limit)) return;
      for (uint32_t e = threadIdx.x; e < P; e += kMT) s.params[e] = __ldcg(params + e);
    }
    __syncthreads();
    if (threadIdx.x == 0 && steps) atomicAdd(epoch_loss + ep, *s.loss / (float)steps);
  }
}

// Inference: one thread per sample, parameters in shared memory, the hidden
// activations in a per-thread shared slice.
__global__ void __launch_bounds__(128) mlp_predict_kernel(const float *__restrict__ params, const float *__restrict__ X,
                                                          uint64_t N, uint32_t F, float *__restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem[];
  float *sp = reinterpret_cast<float *>(smem);
  const uint32_t P = param_count(F);
  float *h = sp + P + threadIdx.x * (2 * kHid);
  for (uint32_t e = threadIdx.x; e < P; e += blockDim.x) sp[e] = params[e];
  __syncthreads();
  const Net p = net_at(sp, F);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
    const float *x = X + i * F;
    for (uint32_t j = 0; j < kHid; ++j) {
      float s = p.b1[j];
      for (uint32_t f = 0; f < F; ++f) s = fmaf(p.W1[j * F + f], x[f], s);
      h[j] = fmaxf(s, 0.0f);
    }
    for (uint32_t j = 0; j < kHid; ++j) {
      float s = p.b2[j];
      for (uint32_t l = 0; l < kHid; ++l) s = fmaf(p.W2[j * kHid + l], h[l], s);
      h[kHid + j] = fmaxf(s, 0.0f);
    }
    float s = p.b3[0];
    for (uint32_t j = 0; j < kHid; ++j) s = fmaf(p.w3[j], h[kHid + j], s);
    out[i] = s;
  }
}

// ---------------------------------------------------------------- features

// The K = min(P, 128) largest of each of two arrays a[0..P), b[0..P) in descending
// order into oa[0..K), ob[0..K): the K-th largest order key of each by a radix select
// (four 8-bit digit passes from the top, both arrays in the same passes, histogram
// updates aggregated per warp), the entries strictly above it (fewer than K) placed
// by their rank among themselves, the rest of the output the K-th value itself.
// Ranks 1, 2, 4, .. 128 are all the features need, so nothing else is sorted.
// hist: 512 words; buf / bkey: 2 * 128 entries; cnt: 2 words; sel: 4 words.
template <int NT>
__device__ void top_desc_two(const float *a, const float *b, uint32_t P, float *oa, float *ob, uint32_t *hist,
                             float *buf, uint32_t *bkey, uint32_t *cnt, uint32_t *sel) {
  const uint32_t t = threadIdx.x, lane = t & 31, K = min(P, 128u);
  uint32_t prefix[2] = {0u, 0u}, need[2] = {K, K};
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (uint32_t i = t; i < 512; i += NT) hist[i] = 0;
    __syncthreads();
    for (uint32_t base = 0; base < P; base += NT) {  // uniform trip count
      const uint32_t j = base + t;
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2) {
        uint32_t bin = 0xFFFFFFFFu;
        if (j < P) {
          const uint32_t key = f2key((s2 ? b : a)[j]);
          if (shift == 24 || (key >> (shift + 8)) == (prefix[s2] >> (shift + 8))) bin = (key >> shift) & 255u;
        }
        if (!__any_sync(0xFFFFFFFFu, bin != 0xFFFFFFFFu)) continue;  // warp-uniform
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, bin);
        if (bin != 0xFFFFFFFFu && lane == __ffs(peers) - 1)
          atomicAdd(&hist[256 * s2 + bin], (uint32_t)__popc(peers));
      }
    }
    __syncthreads();
    if (t < 64) {  // warp s2: lane l owns bins [255-8l-7, 255-8l] of array s2, high to low
      const uint32_t s2 = t >> 5;
      const int top = 255 - 8 * (int)lane;
      uint32_t local[8], sum = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        local[q] = hist[256 * s2 + top - q];
        sum += local[q];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      const uint32_t excl = incl - sum;
      if (excl < need[s2] && need[s2] <= incl) {
        uint32_t run = excl;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          if (run + local[q] >= need[s2]) {
            sel[2 * s2] = (uint32_t)(top - q);
            sel[2 * s2 + 1] = run;
            break;
          }
          run += local[q];
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int s2 = 0; s2 < 2; ++s2) {
      need[s2] -= sel[2 * s2 + 1];
      prefix[s2] |= sel[2 * s2] << shift;
    }
    __syncthreads();  // everyone has read the result before the next pass rewrites it
  }
  if (t < 2) cnt[t] = 0;
  __syncthreads();
  for (uint32_t j = t; j < P; j += NT) {
#pragma unroll
    for (int s2 = 0; s2 < 2; ++s2) {
      const float v = (s2 ? b : a)[j];
      const uint32_t key = f2key(v);
      if (key > prefix[s2]) {
        const uint32_t pos = atomicAdd(&cnt[s2], 1u);  // < K
        buf[128 * s2 + pos] = v;
        bkey[128 * s2 + pos] = key;
      }
    }
  }
  __syncthreads();
  for (uint32_t x = t; x < 2 * K; x += NT) {
    const uint32_t s2 = x / K, i = x % K, c = cnt[s2];
    float *out = s2 ? ob : oa;
    const uint32_t *bk = bkey + 128 * s2;
    if (i < c) {
      uint32_t rank = 0;
      for (uint32_t j = 0; j < c; ++j) rank += (bk[j] > bk[i] || (bk[j] == bk[i] && j < i)) ? 1u : 0u;
      out[rank] = buf[128 * s2 + i];
    } else {
      out[i] = key2f(prefix[s2]);
    }
  }
  __syncthreads();
}

// One block per query: the F features (and, with params, the model's prediction
// of k-th score / S, the MLP forward in the same block).  NT threads: 256 for
// batches (many blocks), 1024 for a single query (the selects are its critical path).
template <int NT>
__global__ void __launch_bounds__(NT) features_kernel(const float *__restrict__ pmin, const float *__restrict__ pmax,
                                                       const float *__restrict__ pmean, uint32_t P, uint32_t Ppad,
                                                       uint32_t d, const BatchQuery *__restrict__ qs,
                                                       float *__restrict__ X, const float *__restrict__ params,
                                                       float *__restrict__ pred, float margin,
                                                       uint32_t *__restrict__ seed, float *__restrict__ cut_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  float *bnd = reinterpret_cast<float *>(smem);
  float *mu = bnd + Ppad;
  float *feat = mu + Ppad;          // kMlpMaxIn
  float *h = feat + kMlpMaxIn;      // 2 * kHid
  __shared__ float S;
  __shared__ uint32_t hist[512], bkey[256], cnt[2], selw[4];
  __shared__ float tb[128], tm[128], buf[256];
  const BatchQuery &q = qs[blockIdx.x];
  const uint32_t F = feature_dim(d);
  if (threadIdx.x == 0) {
    float s = 0.0f;
    for (uint32_t m = 0; m < q.qq; ++m) s += fabsf(q.w[m]);
    S = s > 0.0f ? s : 1.0f;
  }
  for (uint32_t p = threadIdx.x; p < Ppad; p += blockDim.x) {
    float b = __int_as_float(0xFF800000), u = b;
    if (p < P) {
      b = 0.0f;
      u = 0.0f;
      // eight attributes' loads in flight before their sums (the statistics are
      // mostly out of L2 here: one DRAM round trip per attribute otherwise)
      for (uint32_t m0 = 0; m0 < q.qq; m0 += 8) {
        float xb[8], xm[8];
#pragma unroll
        for (uint32_t v = 0; v < 8; ++v) {
          xb[v] = xm[v] = 0.0f;
          if (m0 + v < q.qq) {
            const size_t o = (size_t)p * d + q.attr[m0 + v];
            xb[v] = q.w[m0 + v] >= 0.0f ? pmax[o] : pmin[o];
            xm[v] = pmean[o];
          }
        }
#pragma unroll
        for (uint32_t v = 0; v < 8; ++v)
          if (m0 + v < q.qq) {
            const float w = q.w[m0 + v];
            b += w * xb[v];
            u += w * xm[v];
          }
      }
    }
    bnd[p] = b;
    mu[p] = u;
  }
  for (uint32_t m = threadIdx.x; m < kMlpMaxIn; m += blockDim.x) feat[m] = 0.0f;
  __syncthreads();
  top_desc_two<NT>(bnd, mu, P, tb, tm, hist, buf, bkey, cnt, selw);
  if (threadIdx.x == 0) {
    const float inv = 1.0f / S;
    for (uint32_t m = 0; m < q.qq; ++m) feat[q.attr[m]] += q.w[m] * inv;
    for (uint32_t m = 0; m < d; ++m) feat[d + m] = feat[m] != 0.0f ? logf(fabsf(feat[m])) : 0.0f;
    feat[2 * d] = log2f((float)q.k) * 0.1f;
    feat[2 * d + 1] = (float)q.qq * (1.0f / 16.0f);
    for (uint32_t r = 0; r < 8; ++r) {
      const uint32_t at = min((1u << r), P) - 1u;
      feat[2 * d + 2 + r] = tb[at] * inv;
      feat[2 * d + 10 + r] = tm[at] * inv;
    }
  }
  __syncthreads();
  for (uint32_t f = threadIdx.x; f < F; f += blockDim.x) X[(size_t)blockIdx.x * F + f] = feat[f];
  if (!params) return;
  const Net p = net_at(const_cast<float *>(params), F);
  if (threadIdx.x < kHid) {
    const uint32_t j = threadIdx.x;
    float s = p.b1[j];
    for (uint32_t f = 0; f < F; ++f) s = fmaf(p.W1[j * F + f], feat[f], s);
    h[j] = fmaxf(s, 0.0f);
  }
  __syncthreads();
  if (threadIdx.x < kHid) {
    const uint32_t j = threadIdx.x;
    float s = p.b2[j];
    for (uint32_t l = 0; l < kHid; ++l) s = fmaf(p.W2[j * kHid + l], h[l], s);
    h[kHid + j] = fmaxf(s, 0.0f);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = p.b3[0];
    for (uint32_t j = 0; j < kHid; ++j) s = fmaf(p.w3[j], h[kHid + j], s);
    pred[blockIdx.x] = s;
    if (seed) {
      // a single pruned query: its seed key (0: none) and the cut itself, here rather
      // than in a launch of its own; S as the batched seed takes it (a NaN weight
      // gives a NaN cut: no seed)
      float Sw = 0.0f;
      for (uint32_t m = 0; m < q.qq; ++m) Sw += fabsf(q.w[m]);
      if (Sw == 0.0f) Sw = 1.0f;
      const float cut = learned_cut(s, feat[feature_bound_col(d)], Sw, (float)q.qq, margin);
      *seed = isfinite(cut) ? f2key(cut) : 0u;
      *cut_out = isfinite(cut) ? cut : __int_as_float(0x7FC00000);
    }
  }
}

// Each query's batched state starts at its learned cut (no start when the cut is
// not a finite number), nothing kept yet.  X: the features (row stride F, the
// largest bound / S at column bcol).
__global__ void learned_seed_kernel(const float *__restrict__ pred, const float *__restrict__ X, uint32_t F,
                                    uint32_t bcol, const BatchQuery *__restrict__ qs, float margin,
                                    BatchState *__restrict__ st, uint32_t nq) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nq) return;
  const BatchQuery &q = qs[j];
  float S = 0.0f;
  for (uint32_t m = 0; m < q.qq; ++m) S += fabsf(q.w[m]);
  if (S == 0.0f) S = 1.0f;
  const float cut = learned_cut(pred[j], X[(size_t)j * F + bcol], S, (float)q.qq, margin);
  BatchState s{};
  s.thr = isfinite(cut) ? f2key(cut) : 0u;  // a finite float's key is >= 0x007FFFFF
  s.seed = s.thr;
  st[j] = s;
}

}  // namespace

// ---------------------------------------------------------------- launchers
cudaError_t launch_learned_seed(const float *pred, const float *X, uint32_t d, const BatchQuery *qs, float margin,
                                BatchState *st, uint32_t nq, cudaStream_t s) {
  if (nq)
    learned_seed_kernel<<<(nq + 255) / 256, 256, 0, s>>>(pred, X, feature_dim(d), feature_bound_col(d), qs, margin, st,
                                                         nq);
  return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const float *params, const float *X, const float *y, uint32_t B, uint32_t F, float *grad,
                            float *loss, cudaStream_t s) {
  if (B == 0 || B > kMB || F == 0 || F > kMlpMaxIn) return cudaErrorInvalidValue;
  const size_t smem = mlp_smem(F);
  cudaError_t e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  mlp_grad_kernel<<<1, kMT, smem, s>>>(params, X, y, B, F, grad, loss);
  return cudaGetLastError();
}

size_t mlp_train_scratch_bytes(uint32_t F) { return (size_t)kTrainCtas * mlp_param_count(F) * 4 + sizeof(GridBar); }

cudaError_t launch_mlp_train(float *params, float *m, float *v, const float *X, const float *y, uint64_t N, uint32_t F,
                             uint32_t B, uint32_t epochs, const uint64_t *mul, const uint64_t *add, float lr,
                             float *epoch_loss, void *scratch, uint64_t wait_limit, cudaStream_t s) {
  if (B == 0 || B > kMB || F == 0 || F > kMlpMaxIn) return cudaErrorInvalidValue;
  const size_t smem = mlp_smem(F);
  cudaError_t e = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // the caller zeroed the scratch: partial gradients, then the barrier words
  float *gpart = static_cast<float *>(scratch);
  GridBar *bar = reinterpret_cast<GridBar *>(gpart + (size_t)kTrainCtas * mlp_param_count(F));
  const uint32_t G = std::min<uint32_t>(kTrainCtas, B);
  void *args[] = {&params, &m, &v, &X, &y, &N, &F, &B, &epochs, &mul, &add, &lr, &epoch_loss, &gpart, &bar, &wait_limit};
  e = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(mlp_train_kernel), dim3(G), dim3(kMT), args, smem, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

bool mlp_train_failed(const void *scratch, uint32_t F) {
  GridBar bar{};
  const float *gpart = static_cast<const float *>(scratch);
  if (cudaMemcpy(&bar, gpart + (size_t)kTrainCtas * mlp_param_count(F), sizeof(bar), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return true;
  return bar.err != 0u;
}

cudaError_t launch_mlp_predict(const float *params, const float *X, uint64_t N, uint32_t F, float *out, int num_sms,
                               cudaStream_t s) {
  if (F == 0 || F > kMlpMaxIn) return cudaErrorInvalidValue;
  const size_t smem = ((size_t)mlp_param_count(F) + 128 * 2 * kHid) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(mlp_predict_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const uint64_t blocks = std::min<uint64_t>((N + 127) / 128, (uint64_t)num_sms * 4);
  if (blocks) mlp_predict_kernel<<<(unsigned)blocks, 128, smem, s>>>(params, X, N, F, out);
  return cudaGetLastError();
}

cudaError_t launch_features(const float *pmin, const float *pmax, const float *pmean, uint32_t P, uint32_t d,
                            const BatchQuery *qs, uint32_t nq, float *X, const float *params, float *pred,
                            cudaStream_t s, float margin, uint32_t *seed, float *cut) {
  if (seed && (nq != 1 || !params || !cut)) return cudaErrorInvalidValue;
  if (feature_dim(d) > kMlpMaxIn || P == 0 || P > kMaxFeatureParts) return cudaErrorInvalidValue;
  uint32_t Ppad = 1;
  while (Ppad < P) Ppad <<= 1;
  const size_t smem = (2 * (size_t)Ppad + kMlpMaxIn + 2 * kHid) * sizeof(float);
  // the largest size, once per device (a driver call on every query otherwise)
  static std::atomic<uint64_t> opted{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(opted.load(std::memory_order_acquire) & bit)) {
    const int most = (int)((2 * (size_t)kMaxFeatureParts + kMlpMaxIn + 2 * kHid) * sizeof(float));
    e = cudaFuncSetAttribute(features_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(features_kernel<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
    if (e != cudaSuccess) return e;
    opted.fetch_or(bit, std::memory_order_release);
  }
  if (nq <= 4) {
    if (nq)
      features_kernel<1024><<<nq, 1024, smem, s>>>(pmin, pmax, pmean, P, Ppad, d, qs, X, params, pred, margin, seed,
                                                   cut);
  } else {
    features_kernel<256><<<nq, 256, smem, s>>>(pmin, pmax, pmean, P, Ppad, d, qs, X, params, pred, 0.0f, nullptr,
                                               nullptr);
  }
  return cudaGetLastError();
}

}  // namespace topk
