// Table kernels: seeded synthetic generation, normalize_transpose, and two small
// verification kernels (threshold counts, row gather).
//
// normalize_transpose (common/common.h:30-61) is reproduced bit-exactly:
//   * max starts at +0 and min at FLT_MAX (:36-37) and std::max / std::min replace
//     only on a strict comparison, so NaN never enters, max is +0 unless a positive
//     value exists, and a zero minimum keeps the sign of the FIRST zero in the
//     column.  Min and max are exact, so a parallel reduction on order-preserving
//     keys gives the same bits; the first-zero sign is tracked by index.
//   * v = (v - min) / (max - min) with IEEE round-to-nearest subtract and divide.
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "topk_internal.h"

namespace topk {

namespace {

// ---- seeded generator: same definition as the oracle's orc_generate ----
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t row) {
  return mix64(mix64(seed ^ (stream << 32) ^ (stream >> 32)) ^ row);
}
__device__ __forceinline__ uint32_t u24(uint64_t seed, uint64_t stream, uint64_t row) {
  return (uint32_t)(hash3(seed, stream, row) >> 40);
}

constexpr float kTwoM24 = 5.9604644775390625e-08f;
constexpr float kTwoM25 = 2.98023223876953125e-08f;
constexpr float kSigma = 0.05f;

__device__ __forceinline__ float normal01(uint64_t seed, uint64_t stream, uint64_t row) {
  int64_t acc = 0;
#pragma unroll
  for (int j = 0; j < 6; j++) {
    uint64_t h = hash3(seed, stream * 8 + (uint64_t)j, row);
    acc += (int64_t)(h >> 40);
    acc += (int64_t)((h >> 16) & 0xFFFFFFu);
  }
  int32_t z = (int32_t)(acc - 6 * (int64_t)16777216);
  return __fmul_rn(__int2float_rn(z), kTwoM24);
}

__device__ __forceinline__ float clamp01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

__global__ void generate_kernel(float *table, uint64_t ld, uint32_t d, uint64_t n, int dist, uint64_t seed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    int dd = dist;
    if (dd == 3) dd = (i % 3 == 0) ? 1 : ((i % 3 == 1) ? 0 : 2);
    if (dd == 1) {  // independent U[0,1)
      for (uint32_t m = 0; m < d; m++)
        table[(uint64_t)m * ld + i] = __fmul_rn(__uint2float_rn(u24(seed, 0x100u + m, i)), kTwoM24);
    } else if (dd == 0) {  // correlated: v ~ U[0,1) plus N(0, 0.05) per attribute, clipped
      const float v = __fmul_rn(__uint2float_rn(u24(seed, 0x200u, i)), kTwoM24);
      for (uint32_t m = 0; m < d; m++) {
        const float t = __fmul_rn(normal01(seed, 0x300u + m, i), kSigma);
        table[(uint64_t)m * ld + i] = clamp01(__fadd_rn(v, t));
      }
    } else {  // anticorrelated: Dirichlet spacings scaled to sum d/2, plus noise, clipped
      uint32_t s[64];
      const uint32_t cnt = d - 1;
      for (uint32_t j = 0; j < cnt; j++) s[j] = u24(seed, 0x400u + j, i);
      for (uint32_t a = 1; a < cnt; a++) {
        uint32_t v = s[a];
        uint32_t b = a;
        while (b > 0 && s[b - 1] > v) { s[b] = s[b - 1]; b--; }
        s[b] = v;
      }
      uint32_t prev = 0;
      for (uint32_t m = 0; m < d; m++) {
        const uint32_t cur = (m < cnt) ? s[m] : 16777216u;
        const uint32_t e = cur - prev;
        prev = cur;
        const float base = __fmul_rn(__int2float_rn((int32_t)(e * d)), kTwoM25);
        const float t = __fmul_rn(normal01(seed, 0x500u + m, i), kSigma);
        table[(uint64_t)m * ld + i] = clamp01(__fadd_rn(base, t));
      }
    }
  }
}

// ---- min / max ----
constexpr uint32_t kKeyPosZero = 0x80000000u;
constexpr uint32_t kKeyFltMax = 0xFF7FFFFFu;  // f2key(FLT_MAX)

__global__ void minmax_init_kernel(uint32_t *work, uint32_t d) {
  const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= d) return;
  uint32_t *w = work + (size_t)m * kMinmaxWords;
  w[0] = kKeyPosZero;  // max starts at +0
  w[1] = kKeyFltMax;   // min starts at FLT_MAX
  w[2] = w[3] = w[4] = w[5] = 0xFFFFFFFFu;
  w[6] = w[7] = 0;
}

__global__ void minmax_kernel(const float *table, uint64_t ld, uint64_t n, uint32_t *work) {
  const uint32_t m = blockIdx.y;
  const float *col = table + (uint64_t)m * ld;
  uint32_t kmax = kKeyPosZero, kmin = kKeyFltMax;
  uint64_t first_pz = ~0ull, first_nz = ~0ull;
  const uint64_t n4 = n / 4;
  const float4 *col4 = reinterpret_cast<const float4 *>(col);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  auto visit = [&](float v, uint64_t i) {
    if (v != v) return;
    if (v == 0.0f) {
      if (__float_as_uint(v) >> 31) first_nz = min(first_nz, i);
      else first_pz = min(first_pz, i);
      v = 0.0f;  // +0 for the key comparisons
    }
    const uint32_t kk = f2key(v);
    kmax = max(kmax, kk);
    kmin = min(kmin, kk);
  };
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n4; j += stride) {
    const float4 v = __ldcs(col4 + j);
    visit(v.x, 4 * j);
    visit(v.y, 4 * j + 1);
    visit(v.z, 4 * j + 2);
    visit(v.w, 4 * j + 3);
  }
  for (uint64_t i = 4 * n4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) visit(col[i], i);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    kmax = max(kmax, __shfl_xor_sync(0xFFFFFFFFu, kmax, o));
    kmin = min(kmin, __shfl_xor_sync(0xFFFFFFFFu, kmin, o));
  }
  uint32_t *w = work + (size_t)m * kMinmaxWords;
  if ((threadIdx.x & 31) == 0) {
    if (kmax != kKeyPosZero) atomicMax(&w[0], kmax);
    if (kmin != kKeyFltMax) atomicMin(&w[1], kmin);
  }
  unsigned long long *idx = reinterpret_cast<unsigned long long *>(w + 2);
  if (first_pz != ~0ull) atomicMin(&idx[0], (unsigned long long)first_pz);
  if (first_nz != ~0ull) atomicMin(&idx[1], (unsigned long long)first_nz);
}

__global__ void normalize_kernel(float *table, uint64_t ld, uint64_t n, const float *mins, const float *ranges) {
  const uint32_t m = blockIdx.y;
  float *col = table + (uint64_t)m * ld;
  const float mn = mins[m], mm = ranges[m];
  const uint64_t n4 = n / 4;
  float4 *col4 = reinterpret_cast<float4 *>(col);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n4; j += stride) {
    float4 v = col4[j];
    v.x = __fdiv_rn(__fsub_rn(v.x, mn), mm);
    v.y = __fdiv_rn(__fsub_rn(v.y, mn), mm);
    v.z = __fdiv_rn(__fsub_rn(v.z, mn), mm);
    v.w = __fdiv_rn(__fsub_rn(v.w, mn), mm);
    col4[j] = v;
  }
  for (uint64_t i = 4 * n4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    col[i] = __fdiv_rn(__fsub_rn(col[i], mn), mm);
}

struct CountParams {
  uint8_t attr[kMaxQ];
  float w[kMaxQ];
};

__global__ void count_kernel(const float *table, uint64_t ld, uint64_t r0, uint64_t r1, uint32_t qq,
                             const __grid_constant__ CountParams cp, float thr, unsigned long long *out2) {
  unsigned long long ge = 0, gt = 0;
  for (uint64_t i = r0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < r1; i += (uint64_t)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (uint32_t m = 0; m < qq; m++) s = __fadd_rn(s, __fmul_rn(table[(uint64_t)cp.attr[m] * ld + i], cp.w[m]));
    ge += (s >= thr);
    gt += (s > thr);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ge += __shfl_xor_sync(0xFFFFFFFFu, ge, o);
    gt += __shfl_xor_sync(0xFFFFFFFFu, gt, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out2[0], ge);
    atomicAdd(&out2[1], gt);
  }
}

__global__ void gather_kernel(const float *table, uint64_t ld, uint32_t d, const uint64_t *ids, uint64_t cnt,
                              float *out) {
  const uint64_t total = cnt * d;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = t / d, m = t % d;
    out[t] = table[m * ld + ids[j]];
  }
}

int grid_for(uint64_t work, int threads, int cap) {
  uint64_t g = (work + threads - 1) / threads;
  if (g > (uint64_t)cap) g = cap;
  return g < 1 ? 1 : (int)g;
}

}  // namespace

cudaError_t launch_generate(float *table, uint64_t ld, uint32_t d, uint64_t n, int dist, uint64_t seed,
                            cudaStream_t stream) {
  generate_kernel<<<grid_for(n, 256, 148 * 32), 256, 0, stream>>>(table, ld, d, n, dist, seed);
  return cudaGetLastError();
}

cudaError_t launch_minmax(const float *table, uint64_t ld, uint32_t d, uint64_t n, uint32_t *work,
                          cudaStream_t stream) {
  minmax_init_kernel<<<(d + 127) / 128, 128, 0, stream>>>(work, d);
  dim3 grid(grid_for((n + 3) / 4, 256, 148 * 8 / (d < 8 ? d : 8) + 1), d);
  minmax_kernel<<<grid, 256, 0, stream>>>(table, ld, n, work);
  return cudaGetLastError();
}

cudaError_t launch_normalize(float *table, uint64_t ld, uint32_t d, uint64_t n, const float *mins,
                             const float *ranges, cudaStream_t stream) {
  dim3 grid(grid_for((n + 3) / 4, 256, 148 * 8 / (d < 8 ? d : 8) + 1), d);
  normalize_kernel<<<grid, 256, 0, stream>>>(table, ld, n, mins, ranges);
  return cudaGetLastError();
}

cudaError_t launch_count(const float *table, uint64_t ld, uint64_t r0, uint64_t r1, uint32_t qq, const uint8_t *attr,
                         const float *w, float thr, unsigned long long *out2, cudaStream_t stream) {
  CountParams cp{};
  for (uint32_t m = 0; m < qq && m < kMaxQ; m++) { cp.attr[m] = attr[m]; cp.w[m] = w[m]; }
  cudaError_t e = cudaMemsetAsync(out2, 0, 2 * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return e;
  count_kernel<<<grid_for(r1 - r0, 256, 148 * 16), 256, 0, stream>>>(table, ld, r0, r1, qq, cp, thr, out2);
  return cudaGetLastError();
}

cudaError_t launch_gather(const float *table, uint64_t ld, uint32_t d, const uint64_t *ids, uint64_t cnt,
                          float *out, cudaStream_t stream) {
  gather_kernel<<<grid_for(cnt * d, 256, 1024), 256, 0, stream>>>(table, ld, d, ids, cnt, out);
  return cudaGetLastError();
}

}  // namespace topk
