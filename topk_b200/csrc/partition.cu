// Partitioned copy of the table for pruned queries (device-built).
//
// The reference prunes with per-block upper bounds: VTA orders tuples and keeps,
// per block of 1024, the attribute values bounding every later tuple
// (cpu/VTA.h:74-158); PTA first splits the objects into partitions by the medians
// of their hyperspherical angles (cpu/PTA.h:88-267).  A query stops once its k-th
// score reaches the bound of what is left (cpu/VTA.h:210-216, cpu/PTA.h:337-340).
//
// Here the objects are reordered so that each partition of R = 2^r consecutive rows
// holds objects close in attribute space, and each partition keeps its per-attribute
// min, max and mean; a query then scans only the partitions whose bound
// sum_m w_m * (w_m >= 0 ? max : min) can still reach its threshold (topk_abi.cpp).
// The order is a counting sort by a 16-bit Morton code: each attribute quantised to
// b = 16 / d bits (at least 1; the first 16 attributes when d > 16) relative to the
// column's min and max, the bits interleaved most significant first.  The order only
// decides how much a bound prunes; the results never depend on it (the bounds are
// computed from the partitions as built, and ties go to the lower original id).
//
// Device layout: ptable column-major with the table's stride (partition p = rows
// [p*R, (p+1)*R)), row_ids[row] = original id, stats [P][d] each.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
#include "topk_internal.h"

namespace topk {

namespace {

constexpr uint32_t kBins = 1u << 16;

__global__ void morton_kernel(const float *__restrict__ table, uint64_t ld, uint32_t d, uint64_t n,
                              const float *__restrict__ lo, const float *__restrict__ scale, uint32_t bits,
                              uint16_t *__restrict__ keys) {
  const uint32_t dims = min(d, 16u);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t q[16];
    const uint32_t top = (1u << bits) - 1u;
    for (uint32_t m = 0; m < dims; ++m) {
      const float f = (__ldg(table + (uint64_t)m * ld + i) - lo[m]) * scale[m];  // scale = 2^bits / range
      q[m] = f >= 0.0f ? min((uint32_t)f, top) : 0u;  // NaN -> 0
    }
    uint32_t code = 0;
    for (int l = (int)bits - 1; l >= 0; --l)
      for (uint32_t m = 0; m < dims; ++m) code = (code << 1) | ((q[m] >> l) & 1u);
    keys[i] = (uint16_t)code;
  }
}

__global__ void hist_kernel(const uint16_t *__restrict__ keys, uint64_t n, uint32_t *__restrict__ hist) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(hist + keys[i], 1u);
}

// One block of 1024 threads: exclusive prefix sum of the 2^16 bin counts in place.
__global__ void __launch_bounds__(1024) bin_scan_kernel(uint32_t *__restrict__ hist) {
  __shared__ uint32_t part[1024];
  const uint32_t t = threadIdx.x;
  constexpr uint32_t per = kBins / 1024;
  uint32_t s = 0;
  for (uint32_t j = 0; j < per; ++j) s += hist[t * per + j];
  part[t] = s;
  __syncthreads();
  for (uint32_t o = 1; o < 1024; o <<= 1) {  // inclusive Hillis-Steele scan
    const uint32_t v = t >= o ? part[t - o] : 0u;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint32_t run = part[t] - s;
  for (uint32_t j = 0; j < per; ++j) {
    const uint32_t c = hist[t * per + j];
    hist[t * per + j] = run;
    run += c;
  }
}

__global__ void scatter_kernel(const uint16_t *__restrict__ keys, uint64_t n, uint32_t *__restrict__ cursor,
                               uint32_t *__restrict__ perm) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    perm[atomicAdd(cursor + keys[i], 1u)] = (uint32_t)i;
}

__global__ void gather_rows_kernel(const float *__restrict__ table, uint64_t ld, uint32_t d, uint64_t n,
                                   const uint32_t *__restrict__ perm, float *__restrict__ ptable) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t src = perm[i];
    for (uint32_t m = 0; m < d; ++m) ptable[(uint64_t)m * ld + i] = __ldg(table + (uint64_t)m * ld + src);
  }
}

// One block per partition: per-attribute min, max and mean of its rows.
__global__ void __launch_bounds__(256) part_stats_kernel(const float *__restrict__ ptable, uint64_t ld, uint32_t d,
                                                         uint64_t n, uint32_t rows_log2, float *__restrict__ mins,
                                                         float *__restrict__ maxs, float *__restrict__ means) {
  __shared__ float smn[8], smx[8];
  __shared__ double ssum[8];
  const uint64_t r0 = (uint64_t)blockIdx.x << rows_log2;
  const uint64_t r1 = min((uint64_t)n, r0 + (uint64_t)(1ull << rows_log2));
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t m = 0; m < d; ++m) {
    const float *col = ptable + (uint64_t)m * ld;
    float mn = __int_as_float(0x7F800000), mx = __int_as_float(0xFF800000);
    double sum = 0.0;
    for (uint64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const float x = col[r];
      mn = fminf(mn, x);
      mx = fmaxf(mx, x);
      sum += (double)x;
    }
    for (int o = 16; o > 0; o >>= 1) {
      mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
      mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
      sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
    }
    if (lane == 0) {
      smn[warp] = mn;
      smx[warp] = mx;
      ssum[warp] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (uint32_t w = 1; w < blockDim.x / 32; ++w) {
        mn = fminf(mn, smn[w]);
        mx = fmaxf(mx, smx[w]);
        sum += ssum[w];
      }
      const size_t o = (size_t)blockIdx.x * d + m;
      mins[o] = mn;
      maxs[o] = mx;
      means[o] = r1 > r0 ? (float)(sum / (double)(r1 - r0)) : 0.0f;
    }
    __syncthreads();
  }
}

int grid_for(uint64_t n, int num_sms) {
  const uint64_t b = (n + 255) / 256;
  return (int)(b < (uint64_t)num_sms * 16 ? (b ? b : 1) : (uint64_t)num_sms * 16);
}

}  // namespace

cudaError_t launch_partition_build(const float *table, uint64_t ld, uint32_t d, uint64_t n, const float *lo,
                                   const float *scale, uint32_t bits, uint16_t *keys, uint32_t *hist,
                                   uint32_t *perm, float *ptable, int num_sms, cudaStream_t s) {
  const int g = grid_for(n, num_sms);
  cudaError_t e = cudaMemsetAsync(hist, 0, kBins * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  morton_kernel<<<g, 256, 0, s>>>(table, ld, d, n, lo, scale, bits, keys);
  hist_kernel<<<g, 256, 0, s>>>(keys, n, hist);
  bin_scan_kernel<<<1, 1024, 0, s>>>(hist);
  scatter_kernel<<<g, 256, 0, s>>>(keys, n, hist, perm);
  gather_rows_kernel<<<g, 256, 0, s>>>(table, ld, d, n, perm, ptable);
  return cudaGetLastError();
}

cudaError_t launch_partition_stats(const float *ptable, uint64_t ld, uint32_t d, uint64_t n, uint32_t rows_log2,
                                   uint32_t num_parts, float *mins, float *maxs, float *means, cudaStream_t s) {
  part_stats_kernel<<<num_parts, 256, 0, s>>>(ptable, ld, d, n, rows_log2, mins, maxs, means);
  return cudaGetLastError();
}

}  // namespace topk
