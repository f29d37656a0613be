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
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "block_select.cuh"
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
  __shared__ float smn[8], smx[8], ssum[8];
  const uint64_t r0 = (uint64_t)blockIdx.x << rows_log2;
  const uint64_t r1 = min((uint64_t)n, r0 + (uint64_t)(1ull << rows_log2));
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t m = 0; m < d; ++m) {
    const float *col = ptable + (uint64_t)m * ld;
    float mn = __int_as_float(0x7F800000), mx = __int_as_float(0xFF800000);
    float sum = 0.0f;  // the mean is a model feature only: FP32 partial sums suffice
    for (uint64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const float x = col[r];
      mn = fminf(mn, x);
      mx = fmaxf(mx, x);
      sum += x;
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
      means[o] = r1 > r0 ? sum / (float)(r1 - r0) : 0.0f;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------- VTA and PTA orders
// VTA's index (cpu/VTA.h:121-135): each attribute's list sorted by value, descending;
// each tuple's minimum position over the lists; tuples sorted by that position.
// PTA's (cpu/PTA.h:88-167, 203-236): the tuples first split into partitions by the
// medians of their d-1 hyperspherical angles, then VTA's order inside each partition.
// VTA's threaded build (IMP 2) orders THREADS = 16 equal row ranges on their own.
// Here with stable device radix sorts, so ties go to the lower id (the reference's
// parallel sorts leave them unspecified).  The partition comes in as the high word of
// each list's 64-bit key (partition, then value descending); a partition's rows then
// hold one range of positions in every list, so the global minimum position orders
// the tuples by partition and, inside one, by the partition-local minimum position.
__global__ void col_keys_kernel(const float *__restrict__ col, uint64_t n, uint32_t *__restrict__ keys,
                                uint32_t *__restrict__ ids) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = f2key(__ldg(col + i));  // NaN -> 0: last in a descending list
    ids[i] = (uint32_t)i;
  }
}

// partition in the high word, value descending below it; part clamped to pmax
// (cpu/PTA.h:166)
__global__ void col_keys64_kernel(const float *__restrict__ col, uint64_t n, const uint32_t *__restrict__ part,
                                  uint32_t pmax, uint64_t *__restrict__ keys, uint32_t *__restrict__ ids) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = ((uint64_t)min(part[i], pmax) << 32) | (uint64_t)(~f2key(__ldg(col + i)));
    ids[i] = (uint32_t)i;
  }
}

// PTA's angle coordinate c of every row as a sort key (cpu/PTA.h:108-134):
// f_c = sqrt(sum_{j>c} (x_j - 1.1f)^2) / (x_c - 1.1f), every operation rounded on its
// own as in the reference's AVX path.  The reference keeps |atan(f_c)| * 180/pi, a
// monotone image of |f_c|, so |f_c| orders the rows the same way up to the ties its
// sort leaves unspecified.
__global__ void pta_angle_keys_kernel(const float *__restrict__ table, uint64_t ld, uint32_t d, uint64_t n,
                                      uint32_t c, uint32_t *__restrict__ keys, uint32_t *__restrict__ ids) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    float curr = __fsub_rn(__ldg(table + (uint64_t)(d - 1) * ld + i), 1.1f), s = 0.0f, nxt = 0.0f;
    for (uint32_t m = d - 1; m > c; --m) {
      nxt = __fsub_rn(__ldg(table + (uint64_t)(m - 1) * ld + i), 1.1f);
      s = __fadd_rn(s, __fmul_rn(curr, curr));
      curr = nxt;
    }
    keys[i] = f2key(fabsf(__fdiv_rn(__fsqrt_rn(s), nxt)));
    ids[i] = (uint32_t)i;
  }
}

// part[id] += mul * (rank / mod) over one angle's ascending list (cpu/PTA.h:152-163);
// rank < n <= 2 * mod + 1, so the quotient is 0, 1 or 2
__global__ void pta_part_add_kernel(const uint32_t *__restrict__ sorted_ids, uint64_t n, uint64_t mod, uint32_t mul,
                                    uint32_t *__restrict__ part) {
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t q = p >= 2 * mod ? 2u : (p >= mod ? 1u : 0u);
    if (q) part[sorted_ids[p]] += mul * q;  // each id once per list: no race
  }
}

// VTA's threaded build (IMP 2): rows in `slices` ranges of ceil(n / slices) rows, each
// ordered on its own (cpu/VTA.h:13,78-85)
__global__ void range_part_kernel(uint64_t n, uint64_t range_rows, uint32_t *__restrict__ part) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    part[i] = (uint32_t)(i / range_rows);
}

__global__ void iota_kernel(uint32_t *__restrict__ v, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}

__global__ void min_rank_kernel(const uint32_t *__restrict__ sorted_ids, uint64_t n, uint32_t *__restrict__ rank) {
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t id = sorted_ids[p];  // each id once per list: no race
    rank[id] = min(rank[id], (uint32_t)p);
  }
}

int grid_for(uint64_t n, int num_sms) {
  const uint64_t b = (n + 255) / 256;
  return (int)(b < (uint64_t)num_sms * 16 ? (b ? b : 1) : (uint64_t)num_sms * 16);
}

// ---------------------------------------------------------------- partition order of a query
// The bound of partition p for one query: the reference-order FP32 sum of
// w[attr[m]] * (w >= 0 ? max : min of column attr[m] in p).  IEEE multiplication and
// addition round monotonically, so no row of p scores above it (no slack needed, and
// a partition whose every queried value sits at its maximum scores exactly it).  The
// order key of the bound, or 0xFFFFFFFF (keep) when it is NaN.
// The extremes are read kBoundBatch attributes at a time, all loads of a batch issued
// before the first multiply: the statistics are usually out of L2 by the time a query
// reads them (the scans stream past it), and one DRAM round trip per attribute was the
// bound's whole cost.  The sum keeps the reference order.
constexpr uint32_t kBoundBatch = 8;
__device__ __forceinline__ uint32_t part_bound_key(const float *__restrict__ pmin, const float *__restrict__ pmax,
                                                   uint32_t d, uint32_t p, const PartQuery &q) {
  float sacc = 0.0f;
  for (uint32_t m0 = 0; m0 < q.qq; m0 += kBoundBatch) {
    float x[kBoundBatch];
#pragma unroll
    for (uint32_t u = 0; u < kBoundBatch; ++u) {
      const uint32_t m = m0 + u;
      x[u] = 0.0f;
      if (m < q.qq) {
        const size_t o = (size_t)p * d + q.attr[m];
        x[u] = q.w[m] >= 0.0f ? __ldg(pmax + o) : __ldg(pmin + o);
      }
    }
#pragma unroll
    for (uint32_t u = 0; u < kBoundBatch; ++u)
      if (m0 + u < q.qq) sacc = __fadd_rn(sacc, __fmul_rn(x[u], q.w[m0 + u]));
  }
  return sacc != sacc ? 0xFFFFFFFFu : f2key(sacc);
}

// One block: every partition's bound key, sorted descending (ties by the lower
// partition number) in shared memory by a bitonic network; plist[i] = partition of
// rank i, pkey[i] = its bound key.
constexpr uint32_t kOrderThreads = 1024;

// The partitions in bound order by a counting sort into kOrderThreads buckets over the
// range of the bound keys (bucket 0 = the highest keys); within a bucket in arrival
// order.  pkey[i] is the largest key of i's bucket: an upper bound of every score in
// each of its partitions, and non-increasing along the list (a bucket's keys all lie
// above the next bucket's), which is what the stop rule needs; the bucket width only
// costs pruning where bounds within (kmax - kmin) / 1024 of each other are split.  A
// NaN bound (key 0xFFFFFFFF) lands in bucket 0 and keeps its partition.
__global__ void __launch_bounds__(kOrderThreads) part_order_kernel(const float *__restrict__ pmin,
                                                                  const float *__restrict__ pmax, uint32_t P,
                                                                  uint32_t d, const PartQuery q,
                                                                  uint32_t *__restrict__ plist,
                                                                  uint32_t *__restrict__ pkey) {
  extern __shared__ uint32_t keys[];  // P bound keys
  __shared__ uint32_t cnt[kOrderThreads], bmax[kOrderThreads], wsum[32];
  __shared__ uint32_t kmin_s, kmax_s;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  cnt[t] = 0;
  bmax[t] = 0;
  if (t == 0) {
    kmin_s = 0xFFFFFFFFu;
    kmax_s = 0;
  }
  uint32_t lmin = 0xFFFFFFFFu, lmax = 0;
  for (uint32_t i = t; i < P; i += kOrderThreads) {
    const uint32_t k = part_bound_key(pmin, pmax, d, i, q);
    keys[i] = k;
    lmin = min(lmin, k);
    lmax = max(lmax, k);
  }
  lmin = __reduce_min_sync(0xFFFFFFFFu, lmin);
  lmax = __reduce_max_sync(0xFFFFFFFFu, lmax);
  __syncthreads();
  if (lane == 0) {
    atomicMin(&kmin_s, lmin);
    atomicMax(&kmax_s, lmax);
  }
  __syncthreads();
  const uint32_t kmax = kmax_s;
  const uint64_t span = (uint64_t)(kmax - kmin_s) + 1;
  auto bucket = [&](uint32_t k) { return (uint32_t)(((uint64_t)(kmax - k) * kOrderThreads) / span); };
  for (uint32_t i = t; i < P; i += kOrderThreads) {
    const uint32_t b = bucket(keys[i]);
    atomicAdd(&cnt[b], 1u);
    atomicMax(&bmax[b], keys[i]);
  }
  __syncthreads();
  // exclusive scan of the bucket counts, one bucket per thread
  const uint32_t c = cnt[t];
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = wsum[lane], wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= (uint32_t)o) wi += y;
    }
    wsum[lane] = wi - w;
  }
  __syncthreads();
  cnt[t] = wsum[warp] + incl - c;  // the bucket's first place
  __syncthreads();
  for (uint32_t i = t; i < P; i += kOrderThreads) {
    const uint32_t b = bucket(keys[i]);
    const uint32_t pos = atomicAdd(&cnt[b], 1u);
    plist[pos] = i;
    pkey[pos] = bmax[b];
  }
}

// Many partitions: the keys and partition numbers into arrays for a radix sort.
__global__ void part_keys_kernel(const float *__restrict__ pmin, const float *__restrict__ pmax, uint32_t P,
                                 uint32_t d, const PartQuery q, uint32_t *__restrict__ keys,
                                 uint32_t *__restrict__ ids) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
    keys[i] = part_bound_key(pmin, pmax, d, i, q);
    ids[i] = i;
  }
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

uint64_t index_order_work_words(uint64_t n, IndexOrder kind) { return (kind == IndexOrder::kVta ? 5 : 8) * n; }

cudaError_t launch_index_order(const float *table, uint64_t ld, uint32_t d, uint64_t n, IndexOrder kind,
                               uint32_t *perm, uint32_t *work, void *temp, size_t *temp_bytes, int num_sms,
                               cudaStream_t s, const uint32_t *groups, uint32_t group_bits) {
  const bool pta = kind == IndexOrder::kPta, grouped = kind != IndexOrder::kVta;
  if (n > 0x7FFFFFFFull || (pta && (n < 2 || d > 32))) return cudaErrorInvalidValue;
  if (kind == IndexOrder::kGroups && (!groups || group_bits > 31)) return cudaErrorInvalidValue;
  // work, VTA: keys in/out, ids in/out, min ranks (n words each); grouped orders:
  // 64-bit keys in/out (2n words each, the angle sorts use their first halves), ids
  // in/out, min ranks, groups
  uint32_t *kin = work, *kout = work + (grouped ? 2 * n : n);
  uint32_t *iin = work + (grouped ? 4 * n : 2 * n), *iout = iin + n, *rank = iout + n, *part = rank + n;
  uint64_t *kin64 = reinterpret_cast<uint64_t *>(kin), *kout64 = reinterpret_cast<uint64_t *>(kout);
  // groups < 2^gbits
  const uint32_t gbits = pta ? d - 1 : kind == IndexOrder::kGroups ? group_bits : (grouped ? 4 : 0);
  const int nn = (int)n;
  if (!temp) {  // size query
    size_t a = 0, b = 0, c = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(nullptr, a, kin, kout, iin, iout, nn, 0, 32, s);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, b, kin, kout, iin, iout, nn, 0, 32, s);
    if (e == cudaSuccess && grouped)
      e = cub::DeviceRadixSort::SortPairs(nullptr, c, kin64, kout64, iin, iout, nn, 0, 32 + (int)gbits, s);
    *temp_bytes = std::max(a, std::max(b, c));
    return e;
  }
  const int g = grid_for(n, num_sms);
  size_t tb = *temp_bytes;
  cudaError_t e = cudaMemsetAsync(rank, 0xFF, n * sizeof(uint32_t), s);
  if (pta) {
    if (e == cudaSuccess) e = cudaMemsetAsync(part, 0, n * sizeof(uint32_t), s);
    for (uint32_t c = 0; e == cudaSuccess && c + 1 < d; ++c) {  // median split per angle
      pta_angle_keys_kernel<<<g, 256, 0, s>>>(table, ld, d, n, c, kin, iin);
      e = cub::DeviceRadixSort::SortPairs(temp, tb, kin, kout, iin, iout, nn, 0, 32, s);
      if (e == cudaSuccess) pta_part_add_kernel<<<g, 256, 0, s>>>(iout, n, n / 2, 1u << c, part);
    }
  } else if (kind == IndexOrder::kGroups) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(part, groups, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
  } else if (grouped) {
    range_part_kernel<<<g, 256, 0, s>>>(n, (n - 1) / kVtaThreadRanges + 1, part);
  }
  for (uint32_t m = 0; e == cudaSuccess && m < d; ++m) {
    if (grouped) {
      col_keys64_kernel<<<g, 256, 0, s>>>(table + (uint64_t)m * ld, n, part, (1u << gbits) - 1u, kin64, iin);
      e = cub::DeviceRadixSort::SortPairs(temp, tb, kin64, kout64, iin, iout, nn, 0, 32 + (int)gbits, s);
    } else {
      col_keys_kernel<<<g, 256, 0, s>>>(table + (uint64_t)m * ld, n, kin, iin);
      e = cub::DeviceRadixSort::SortPairsDescending(temp, tb, kin, kout, iin, iout, nn, 0, 32, s);
    }
    if (e == cudaSuccess) min_rank_kernel<<<g, 256, 0, s>>>(iout, n, rank);
  }
  if (e != cudaSuccess) return e;
  // tuples by minimum position, ties by the lower id
  iota_kernel<<<g, 256, 0, s>>>(iin, n);
  e = cub::DeviceRadixSort::SortPairs(temp, tb, rank, kout, iin, perm, nn, 0, 32, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

namespace {

// ---- kd order: median splits along the attribute of widest spread ----
//
// The partitions are the leaves of a balanced binary tree over the rows: a node is a
// range of whole partitions [lo, hi) of the order; it splits into [lo, mid) and
// [mid, hi), mid = lo + ceil((hi - lo) / 2), by sorting its rows by the attribute
// whose values spread widest in it (largest max - min, FP32; the lower attribute on a
// tie), so the first half holds its lower values.  Level L sorts every node of level L
// at once: a stable radix sort of (node << 32 | order key of the value) with the row
// ids, which keeps each node's rows in its own range.  Node ids at level L follow the
// path from the root (left 0, right 1), so they increase along the rows.

__device__ __forceinline__ uint32_t kd_node_of(uint32_t part, uint32_t P, uint32_t level) {
  uint32_t lo = 0, hi = P, id = 0;
  for (uint32_t l = 0; l < level; ++l) {
    const uint32_t mid = lo + (hi - lo + 1) / 2;
    const uint32_t right = part >= mid ? 1u : 0u;
    id = 2 * id + right;
    if (right) lo = mid; else hi = mid;
  }
  return id;
}

// Per node and attribute: the largest and smallest order key of the node's values
// (NaN left out).  One block per chunk of 1024 positions (a chunk lies in one
// partition, so in one node); stats: [node][d] max keys, then [node][d] min keys.
__global__ void __launch_bounds__(256) kd_stats_kernel(const float *__restrict__ table, uint64_t ld, uint32_t d,
                                                       uint64_t n, const uint32_t *__restrict__ perm, uint32_t lg,
                                                       uint32_t P, uint32_t level, uint32_t nodes,
                                                       uint32_t *__restrict__ stats) {
  __shared__ uint32_t smax[32], smin[32];
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t chunks = (n + 1023) / 1024;
  for (uint64_t c = blockIdx.x; c < chunks; c += gridDim.x) {
    const uint64_t base = c * 1024;
    const uint32_t node = kd_node_of((uint32_t)(base >> lg), P, level);
    uint32_t id[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const uint64_t pos = base + threadIdx.x + 256u * v;
      id[v] = pos < n ? perm[pos] : 0xFFFFFFFFu;
    }
    for (uint32_t m0 = 0; m0 < d; m0 += 32) {
      const uint32_t dm = min(32u, d - m0);
      if (threadIdx.x < dm) {
        smax[threadIdx.x] = 0u;
        smin[threadIdx.x] = 0xFFFFFFFFu;
      }
      __syncthreads();
      for (uint32_t m = 0; m < dm; ++m) {
        uint32_t kmax = 0u, kmin = 0xFFFFFFFFu;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          if (id[v] == 0xFFFFFFFFu) continue;
          const float x = __ldg(table + (uint64_t)(m0 + m) * ld + id[v]);
          if (x != x) continue;
          const uint32_t k = f2key(x);
          kmax = max(kmax, k);
          kmin = min(kmin, k);
        }
        kmax = __reduce_max_sync(0xFFFFFFFFu, kmax);
        kmin = __reduce_min_sync(0xFFFFFFFFu, kmin);
        if (lane == 0) {
          atomicMax(&smax[m], kmax);
          atomicMin(&smin[m], kmin);
        }
      }
      __syncthreads();
      if (threadIdx.x < dm) {
        atomicMax(stats + (size_t)node * d + m0 + threadIdx.x, smax[threadIdx.x]);
        atomicMin(stats + (size_t)nodes * d + (size_t)node * d + m0 + threadIdx.x, smin[threadIdx.x]);
      }
      __syncthreads();
    }
  }
}

// Per node: the attribute of widest spread (0 for a node without values).
__global__ void kd_split_kernel(const uint32_t *__restrict__ stats, uint32_t d, uint32_t nodes,
                                uint32_t *__restrict__ attr) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nodes; j += gridDim.x * blockDim.x) {
    uint32_t best = 0;
    float bspread = 0.0f;
    for (uint32_t m = 0; m < d; ++m) {
      const uint32_t kmax = stats[(size_t)j * d + m], kmin = stats[(size_t)nodes * d + (size_t)j * d + m];
      float spread = 0.0f;
      if (kmax != 0u) {
        spread = __fsub_rn(key2f(kmax), key2f(kmin));
        if (spread != spread) spread = 0.0f;
      }
      if (m == 0 || spread > bspread) {
        bspread = spread;
        best = m;
      }
    }
    attr[j] = best;
  }
}

// Sort keys of level `level`: (node << 32 | order key of the row's value in the node's
// split attribute), with the row ids.
__global__ void kd_keys_kernel(const float *__restrict__ table, uint64_t ld, uint64_t n,
                               const uint32_t *__restrict__ perm, uint32_t lg, uint32_t P, uint32_t level,
                               const uint32_t *__restrict__ attr, unsigned long long *__restrict__ keys,
                               uint32_t *__restrict__ ids) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t node = kd_node_of((uint32_t)(i >> lg), P, level);
    const uint32_t id = perm[i];
    const float x = __ldg(table + (uint64_t)attr[node] * ld + id);
    keys[i] = ((unsigned long long)node << 32) | f2key(x);
    ids[i] = id;
  }
}

}  // namespace

uint32_t kd_levels(uint32_t P) {
  uint32_t L = 0;
  while ((1ull << L) < P) ++L;
  return L;
}

uint64_t kd_order_work_words(uint64_t n, uint32_t d, uint32_t P) {
  return 5 * n + 2 * (uint64_t)P * d + P;
}

cudaError_t launch_kd_order(const float *table, uint64_t ld, uint32_t d, uint64_t n, uint32_t part_log2,
                            uint32_t *perm, uint32_t *work, void *temp, size_t *temp_bytes, int num_sms,
                            cudaStream_t s) {
  if (n > 0x7FFFFFFFull || d == 0) return cudaErrorInvalidValue;
  const uint32_t P = (uint32_t)((n + (1ull << part_log2) - 1) >> part_log2);
  const uint32_t L = kd_levels(P);
  const int nn = (int)n;
  // work: keys in / out (2n words each), ids (n words), per-node stats, split attributes
  unsigned long long *kin = reinterpret_cast<unsigned long long *>(work);
  unsigned long long *kout = kin + n;
  uint32_t *ids = work + 4 * n;
  uint32_t *stats = work + 5 * n;
  uint32_t *attr = stats + 2 * (uint64_t)P * d;
  if (!temp) {  // size query
    return cub::DeviceRadixSort::SortPairs(nullptr, *temp_bytes, kin, kout, ids, perm, nn, 0, 64, s);
  }
  const int g = grid_for(n, num_sms);
  size_t tb = *temp_bytes;
  iota_kernel<<<g, 256, 0, s>>>(perm, n);
  cudaError_t e = cudaGetLastError();
  for (uint32_t level = 0; e == cudaSuccess && level < L; ++level) {
    const uint32_t nodes = 1u << level;
    e = cudaMemsetAsync(stats, 0, (size_t)nodes * d * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(stats + (size_t)nodes * d, 0xFF, (size_t)nodes * d * sizeof(uint32_t), s);
    if (e != cudaSuccess) break;
    const uint64_t chunks = (n + 1023) / 1024;
    const int gs = (int)std::min<uint64_t>(chunks, (uint64_t)num_sms * 8);
    kd_stats_kernel<<<gs, 256, 0, s>>>(table, ld, d, n, perm, part_log2, P, level, nodes, stats);
    kd_split_kernel<<<(nodes + 255) / 256, 256, 0, s>>>(stats, d, nodes, attr);
    kd_keys_kernel<<<g, 256, 0, s>>>(table, ld, n, perm, part_log2, P, level, attr, kin, ids);
    e = cudaGetLastError();
    // the sorted ids are the next order; node ids < 2^level sit above the 32 key bits
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(temp, tb, kin, kout, ids, perm, nn, 0, 32 + (int)level, s);
  }
  return e;
}

cudaError_t launch_gather_rows(const float *table, uint64_t ld, uint32_t d, uint64_t n, const uint32_t *perm,
                               float *ptable, int num_sms, cudaStream_t s) {
  gather_rows_kernel<<<grid_for(n, num_sms), 256, 0, s>>>(table, ld, d, n, perm, ptable);
  return cudaGetLastError();
}

cudaError_t launch_partition_stats(const float *ptable, uint64_t ld, uint32_t d, uint64_t n, uint32_t rows_log2,
                                   uint32_t num_parts, float *mins, float *maxs, float *means, cudaStream_t s) {
  part_stats_kernel<<<num_parts, 256, 0, s>>>(ptable, ld, d, n, rows_log2, mins, maxs, means);
  return cudaGetLastError();
}

size_t part_order_temp_bytes(uint32_t P) {
  if (P <= kPartOrderOneBlock) return 0;
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                            (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)P, 0, 32);
  return (tb + 255) / 256 * 256 + 2 * (size_t)P * sizeof(uint32_t);
}

cudaError_t launch_part_order(const float *pmin, const float *pmax, uint32_t P, uint32_t d, const PartQuery &q,
                              uint32_t *plist, uint32_t *pkey, void *temp, size_t temp_bytes, int num_sms,
                              cudaStream_t s) {
  if (P == 0) return cudaSuccess;
  if (P <= kPartOrderOneBlock) {
    const size_t smem = (size_t)P * 4;
    // the largest size once per device (a driver call on every query otherwise)
    static std::atomic<uint64_t> opted{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = 1ull << (dev & 63);
    if (!(opted.load(std::memory_order_acquire) & bit)) {
      e = cudaFuncSetAttribute(part_order_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(kPartOrderOneBlock * 4));
      if (e != cudaSuccess) return e;
      opted.fetch_or(bit, std::memory_order_release);
    }
    part_order_kernel<<<1, kOrderThreads, smem, s>>>(pmin, pmax, P, d, q, plist, pkey);
    return cudaGetLastError();
  }
  // keys_in | ids_in after the radix sort's own scratch
  if (temp_bytes < part_order_temp_bytes(P)) return cudaErrorInvalidValue;
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                            (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)P, 0, 32);
  uint32_t *kin = reinterpret_cast<uint32_t *>(static_cast<unsigned char *>(temp) + (tb + 255) / 256 * 256);
  uint32_t *iin = kin + P;
  part_keys_kernel<<<grid_for(P, num_sms), 256, 0, s>>>(pmin, pmax, P, d, q, kin, iin);
  // stable: equal keys keep ascending partition numbers
  cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(temp, tb, kin, pkey, iin, plist, (int)P, 0, 32, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace topk
