// Skyline layers of SLA (cpu/SLA.h:102-139) on the device.
//
// The reference peels layers: while more than 100 rows remain, the skyline of the
// remaining rows (no other remaining row dominates them; p dominates q when p <= q in
// every attribute and p < q in one, on the values 1 - x, cpu/SLA.h:87-100) is the next
// layer, and the last <= 100 rows form one final layer.  Here the same layers come
// from depths: a row's depth is 1 + the largest depth of the rows that dominate it (0
// for the skyline).  Every dominator of a row has an FP32 coordinate sum no larger
// (one rounding per addition is monotone) and, at an equal sum, comes first in the
// lexicographic order of its values; so with the rows sorted that way (stable radix
// sorts, least significant key first) a row's dominators all come before it.  The
// sorted rows are cut into blocks of 256: a block's rows take the largest depth + 1 of
// their dominators in earlier blocks (accumulated by the panel kernels), then the block
// settles its own rows by relaxation (depths only grow; a pass changes nothing once
// every chain inside the block is resolved); then its panel kernel raises the
// candidate depth of every later row.  The stop rule is applied to the depths on the
// host: the first depth l with at most 100 rows at depth >= l takes all of them.
// O(n^2 d / 2) compares: meant for the table sizes the reference's SLA serves.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/topk_b200.h"
#include "device_common.cuh"
#include "topk_internal.h"

namespace topk {

namespace {

constexpr uint32_t kSkyBlock = 256;   // rows per block (= threads of the block kernels)
constexpr uint32_t kSkyMaxD = 32;
// Largest table the layer build accepts.  The build compares O(n^2 d / 2) pairs in
// n / 256 sequential settle + panel launch pairs: 2^22 rows are about 1.4e14 compares
// (seconds to minutes on one B200); 2^26 rows would be 256 times that.
constexpr uint64_t kSkyMaxRows = 1ull << 22;
constexpr uint64_t kSkyStopRows = 100;  // cpu/SLA.h:110

// key of column m of the sky values (m == d: the FP32 sum of all of them)
__global__ void sky_key_kernel(const float *__restrict__ table, uint64_t ld, uint32_t d, uint64_t n, uint32_t m,
                               uint32_t *__restrict__ keys, uint32_t *__restrict__ ids) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    float v;
    if (m < d) {
      v = __fsub_rn(1.0f, __ldg(table + (uint64_t)m * ld + i));
    } else {
      v = 0.0f;
      for (uint32_t j = 0; j < d; ++j) v = __fadd_rn(v, __fsub_rn(1.0f, __ldg(table + (uint64_t)j * ld + i)));
    }
    keys[i] = f2key(v);
    ids[i] = (uint32_t)i;
  }
}

// key of column m for the rows in the current order (the next stable pass)
__global__ void sky_key_perm_kernel(const float *__restrict__ table, uint64_t ld, uint32_t d, uint64_t n, uint32_t m,
                                    const uint32_t *__restrict__ order, uint32_t *__restrict__ keys) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = order[j];
    float v;
    if (m < d) {
      v = __fsub_rn(1.0f, __ldg(table + (uint64_t)m * ld + i));
    } else {
      v = 0.0f;
      for (uint32_t q = 0; q < d; ++q) v = __fadd_rn(v, __fsub_rn(1.0f, __ldg(table + (uint64_t)q * ld + i)));
    }
    keys[j] = f2key(v);
  }
}

// sky values of the rows in sorted order, column-major [d][n]
__global__ void sky_gather_kernel(const float *__restrict__ table, uint64_t ld, uint32_t d, uint64_t n,
                                  const uint32_t *__restrict__ order, float *__restrict__ xs) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = order[j];
    for (uint32_t m = 0; m < d; ++m) xs[(uint64_t)m * n + j] = __fsub_rn(1.0f, __ldg(table + (uint64_t)m * ld + i));
  }
}

__device__ __forceinline__ bool dominates(const float *__restrict__ p, uint32_t pstride, const float *q, uint32_t d) {
  bool strict = false;
  for (uint32_t m = 0; m < d; ++m) {
    const float a = p[m * pstride], b = q[m];
    if (!(a <= b)) return false;
    strict |= a < b;
  }
  return strict;
}

// Settle block a: rows [r0, r0 + len) start at their candidate depth and take
// 1 + the depth of every dominator inside the block until nothing changes.
__global__ void __launch_bounds__(kSkyBlock)
    sky_settle_kernel(const float *__restrict__ xs, uint64_t n, uint32_t d, uint64_t r0, uint32_t len,
                      const uint32_t *__restrict__ cand, uint32_t *__restrict__ depth) {
  __shared__ float sx[kSkyMaxD * kSkyBlock];  // [m][row]
  __shared__ uint32_t sd[kSkyBlock];
  const uint32_t t = threadIdx.x;
  const bool live = t < len;
  for (uint32_t m = 0; m < d; ++m) sx[m * kSkyBlock + t] = live ? xs[(uint64_t)m * n + r0 + t] : 0.0f;
  sd[t] = live ? cand[r0 + t] : 0u;
  float mine[kSkyMaxD];
#pragma unroll 1
  for (uint32_t m = 0; m < d; ++m) mine[m] = sx[m * kSkyBlock + t];
  __syncthreads();
  for (uint32_t pass = 0; pass <= kSkyBlock; ++pass) {  // each pass settles one more link of every chain
    uint32_t v = sd[t];
    if (live)
      for (uint32_t i = 0; i < t; ++i)
        if (sd[i] + 1u > v && dominates(sx + i, kSkyBlock, mine, d)) v = sd[i] + 1u;
    __syncthreads();
    const bool changed = v != sd[t];
    sd[t] = v;
    if (!__syncthreads_or(changed)) break;
  }
  if (live) depth[r0 + t] = sd[t];
}

// Panel of block a: every later row j takes 1 + the depth of its dominators in block a.
__global__ void __launch_bounds__(kSkyBlock)
    sky_panel_kernel(const float *__restrict__ xs, uint64_t n, uint32_t d, uint64_t r0, uint32_t len,
                     const uint32_t *__restrict__ depth, uint32_t *__restrict__ cand) {
  __shared__ float sx[kSkyMaxD * kSkyBlock];
  __shared__ uint32_t sd[kSkyBlock];
  const uint32_t t = threadIdx.x;
  for (uint32_t m = 0; m < d; ++m) sx[m * kSkyBlock + t] = t < len ? xs[(uint64_t)m * n + r0 + t] : 0.0f;
  sd[t] = t < len ? depth[r0 + t] : 0u;
  __syncthreads();
  const uint64_t first = r0 + len;
  for (uint64_t j = first + (uint64_t)blockIdx.x * blockDim.x + t; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    float mine[kSkyMaxD];
#pragma unroll 1
    for (uint32_t m = 0; m < d; ++m) mine[m] = xs[(uint64_t)m * n + j];
    uint32_t v = cand[j];
    for (uint32_t i = 0; i < len; ++i)
      if (sd[i] + 1u > v && dominates(sx + i, kSkyBlock, mine, d)) v = sd[i] + 1u;
    cand[j] = v;
  }
}

int grid_n(uint64_t work, int num_sms) {
  const uint64_t b = (work + 255) / 256;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)num_sms * 16));
}

}  // namespace

int skyline_layers_device(const float *table, uint64_t ld, uint32_t d, uint64_t n, int num_sms, uint32_t *layers,
                          uint64_t *num_layers, std::string *msg) {
  if (d == 0 || d > kSkyMaxD || n == 0 || n > kSkyMaxRows) {
    *msg = "skyline layers need 1 <= d <= 32 and 1 <= n <= 2^22 (the build compares O(n^2 d) pairs)";
    return TOPK_ERR_UNSUPPORTED;
  }
  cudaStream_t s = nullptr;
  uint32_t *kin = nullptr, *kout = nullptr, *oa = nullptr, *ob = nullptr, *cand = nullptr, *depth = nullptr;
  float *xs = nullptr;
  void *temp = nullptr;
  size_t tb = 0;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&kin, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&kout, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&oa, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&ob, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&cand, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&depth, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&xs, (size_t)d * n * sizeof(float));
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, oa, ob, (int)n, 0, 32, s);
  if (e == cudaSuccess) e = cudaMalloc(&temp, std::max<size_t>(tb, 16));
  const int g = grid_n(n, num_sms);
  // order: stable passes from the least significant key (the last value) to the sum
  if (e == cudaSuccess) {
    sky_key_kernel<<<g, 256, 0, s>>>(table, ld, d, n, d - 1, kin, oa);
    size_t t2 = tb;
    e = cub::DeviceRadixSort::SortPairs(temp, t2, kin, kout, oa, ob, (int)n, 0, 32, s);
    std::swap(oa, ob);
  }
  for (int m = (int)d - 2; e == cudaSuccess && m >= -1; --m) {
    const uint32_t key = m >= 0 ? (uint32_t)m : d;  // d: the sum, the most significant key
    sky_key_perm_kernel<<<g, 256, 0, s>>>(table, ld, d, n, key, oa, kin);
    size_t t2 = tb;
    e = cub::DeviceRadixSort::SortPairs(temp, t2, kin, kout, oa, ob, (int)n, 0, 32, s);
    std::swap(oa, ob);
  }
  if (e == cudaSuccess) {
    sky_gather_kernel<<<g, 256, 0, s>>>(table, ld, d, n, oa, xs);
    e = cudaMemsetAsync(cand, 0, n * sizeof(uint32_t), s);
  }
  const uint64_t nb = (n + kSkyBlock - 1) / kSkyBlock;
  for (uint64_t a = 0; a < nb && e == cudaSuccess; ++a) {
    const uint64_t r0 = a * kSkyBlock;
    const uint32_t len = (uint32_t)std::min<uint64_t>(kSkyBlock, n - r0);
    sky_settle_kernel<<<1, kSkyBlock, 0, s>>>(xs, n, d, r0, len, cand, depth);
    if (r0 + len < n) sky_panel_kernel<<<grid_n(n - r0 - len, num_sms), kSkyBlock, 0, s>>>(xs, n, d, r0, len,
                                                                                           depth, cand);
    if ((a & 255) == 255) e = cudaStreamSynchronize(s);  // keeps launch errors close to their cause
  }
  std::vector<uint32_t> dep(n), ord(n);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dep.data(), depth, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ord.data(), oa, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(kin);
  cudaFree(kout);
  cudaFree(oa);
  cudaFree(ob);
  cudaFree(cand);
  cudaFree(depth);
  cudaFree(xs);
  cudaFree(temp);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    *msg = std::string("skyline layers: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? TOPK_ERR_OOM : TOPK_ERR_CUDA;
  }
  // stop rule: the first depth l with at most 100 rows at depth >= l takes them all
  uint32_t dmax = 0;
  for (uint32_t v : dep) dmax = std::max(dmax, v);
  std::vector<uint64_t> beyond((size_t)dmax + 2, 0);
  for (uint32_t v : dep) beyond[v]++;
  for (int64_t l = (int64_t)dmax - 1; l >= 0; --l) beyond[(size_t)l] += beyond[(size_t)l + 1];
  uint32_t lstop = dmax + 1;
  for (uint32_t l = 0; l <= dmax; ++l)
    if (beyond[l] <= kSkyStopRows) {
      lstop = l;
      break;
    }
  uint32_t top = 0;
  for (uint64_t j = 0; j < n; ++j) {
    const uint32_t v = std::min(dep[j], lstop);
    layers[ord[j]] = v;
    top = std::max(top, v);
  }
  *num_layers = (uint64_t)top + 1;
  return TOPK_OK;
}

}  // namespace topk
