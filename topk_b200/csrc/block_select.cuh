// Block-wide exact selection on (key, id) candidate entries, shared by the fused
// single-query scan and the batched kernels.
//
// An entry is uint2{key, id}: key = order-preserving image of an FP32 score
// (NaN -> 0), id = object id.  Selection order = the 64-bit word key<<32 | ~id
// (higher score first, then lower id), so every entry is distinct and "the best k"
// is always exactly k entries.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"

namespace topk {

// Shared-memory state of one block's select (48 bytes, 8-byte aligned).
struct SelShared {
  uint32_t digit, above, eq;  // radix-select pass result
  uint32_t valid;             // entries with key >= min_key
  uint32_t wcount;            // compaction cursor
  uint32_t kept_min;          // min key among the kept entries
  uint32_t pad[2];
  unsigned long long mm[2];   // min / max composite of a select
};

struct SmemSrc {
  const uint2 *p;
  __device__ uint2 operator()(uint32_t j) const { return p[j]; }
};
struct KeySrc {  // bare keys (no ids), as a source of (key, 0) entries
  const uint32_t *p;
  __device__ uint2 operator()(uint32_t j) const { return make_uint2(p[j], 0u); }
};

// Block-wide radix select over `count` entries of `src` with key >= min_key: finds
// (prefix, mask) such that exactly `need` valid entries satisfy
// (composite & mask) >= prefix.  Requires need <= number of valid entries.
// Digits are taken from the highest bit where the valid entries differ (min/max of
// the composites first), 8 bits at a time; histogram updates are aggregated per
// warp with __match_any_sync, because candidates crowd into few bins.  `count`
// must be the same in every thread; `hist` holds 256 bins.
template <int NT, class Src>
__device__ void block_radix_select(const Src &src, uint32_t count, uint32_t min_key, uint32_t need,
                                   uint32_t *hist, SelShared *sh, uint64_t &prefix_out, uint64_t &mask_out) {
  static_assert(NT % 32 == 0 && NT >= 32, "whole warps");
  const int t = threadIdx.x;
  const int lane = t & 31;
  if (t == 0) {
    sh->mm[0] = ~0ull;
    sh->mm[1] = 0ull;
  }
  __syncthreads();
  {
    unsigned long long lo = ~0ull, hi = 0ull;
    for (uint32_t j = t; j < count; j += NT) {
      const uint2 e = src(j);
      if (e.x < min_key) continue;
      const unsigned long long c = composite(e.x, e.y);
      lo = c < lo ? c : lo;
      hi = c > hi ? c : hi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long a = __shfl_xor_sync(0xFFFFFFFFu, lo, o);
      const unsigned long long b = __shfl_xor_sync(0xFFFFFFFFu, hi, o);
      lo = a < lo ? a : lo;
      hi = b > hi ? b : hi;
    }
    if (lane == 0) {
      atomicMin(&sh->mm[0], lo);
      atomicMax(&sh->mm[1], hi);
    }
  }
  __syncthreads();
  const uint64_t cmin = sh->mm[0], cmax = sh->mm[1];
  const uint64_t diff = cmin ^ cmax;
  int hib = diff ? 63 - __clzll((long long)diff) : -1;  // highest differing bit
  uint64_t mask = hib >= 63 ? 0ull : (~0ull << (hib + 1));
  uint64_t prefix = cmin & mask;
  while (hib >= 0) {
    const int lob = hib >= 7 ? hib - 7 : 0;
    const uint32_t dmask = (1u << (hib - lob + 1)) - 1u;
    for (int b = t; b < 256; b += NT) hist[b] = 0;
    __syncthreads();
    for (uint32_t base = 0; base < count; base += NT) {  // uniform trip count
      const uint32_t j = base + t;
      uint32_t bin = 0xFFFFFFFFu;
      if (j < count) {
        const uint2 e = src(j);
        if (e.x >= min_key) {
          const uint64_t c = composite(e.x, e.y);
          if ((c & mask) == prefix) bin = (uint32_t)(c >> lob) & dmask;
        }
      }
      if (!__any_sync(0xFFFFFFFFu, bin != 0xFFFFFFFFu)) continue;  // warp-uniform: nothing to count
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, bin);
      if (bin != 0xFFFFFFFFu && lane == __ffs(peers) - 1) atomicAdd(&hist[bin], (uint32_t)__popc(peers));
    }
    __syncthreads();
    if (t < 32) {
      // lane l owns bins [255-8l-7, 255-8l], visited from high to low
      const int top = 255 - 8 * t;
      uint32_t local[8];
      uint32_t s = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        local[b] = hist[top - b];
        s += local[b];
      }
      uint32_t incl = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (t >= o) incl += v;
      }
      const uint32_t excl = incl - s;
      if (excl < need && need <= incl) {
        uint32_t run = excl;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          if (run + local[b] >= need) {
            sh->digit = (uint32_t)(top - b);
            sh->above = run;
            sh->eq = local[b];
            break;
          }
          run += local[b];
        }
      }
    }
    __syncthreads();
    const uint32_t digit = sh->digit, above = sh->above, eq = sh->eq;
    __syncthreads();  // everyone has read the result before the next pass rewrites it
    need -= above;
    prefix |= (uint64_t)digit << lob;
    mask |= (uint64_t)dmask << lob;
    if (eq == need) break;
    hib = lob - 1;
  }
  prefix_out = prefix;
  mask_out = mask;
}

// Keep the best k entries with key >= min_key of src[0..count), written to dst
// (out of place; dst must not overlap src).  Returns the number kept (the same in
// every thread); sh->kept_min gets their min key.
template <int NT>
__device__ uint32_t block_reduce(const uint2 *src, uint32_t count, uint2 *dst, uint32_t k, uint32_t min_key,
                                 uint32_t *hist, SelShared *sh) {
  const int t = threadIdx.x;
  uint32_t v = 0;
  for (uint32_t j = t; j < count; j += NT) v += (src[j].x >= min_key);
  v = warp_sum_u32(v);
  if (t == 0) {
    sh->valid = 0;
    sh->wcount = 0;
    sh->kept_min = 0xFFFFFFFFu;
  }
  __syncthreads();
  if ((t & 31) == 0) atomicAdd(&sh->valid, v);
  __syncthreads();
  const uint32_t valid = sh->valid;
  uint64_t prefix = 0, mask = 0;
  const bool select = valid > k;
  if (select) block_radix_select<NT>(SmemSrc{src}, count, min_key, k, hist, sh, prefix, mask);
  uint32_t kmin = 0xFFFFFFFFu;
  for (uint32_t base = 0; base < count; base += NT) {  // uniform trip count
    const uint32_t j = base + t;
    uint2 e = make_uint2(0u, 0u);
    bool keep = false;
    if (j < count) {
      e = src[j];
      keep = e.x >= min_key && (!select || (composite(e.x, e.y) & mask) >= prefix);
    }
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
    uint32_t pos = 0;
    if ((t & 31) == 0 && bal) pos = atomicAdd(&sh->wcount, (uint32_t)__popc(bal));
    pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
    if (keep) {
      dst[pos + __popc(bal & ((1u << (t & 31)) - 1u))] = e;
      kmin = min(kmin, e.x);
    }
  }
  kmin = warp_min_u32(kmin);
  if ((t & 31) == 0) atomicMin(&sh->kept_min, kmin);
  __syncthreads();
  const uint32_t kept = sh->wcount;
  __syncthreads();  // every thread has its copy before thread 0 may reset wcount
  return kept;
}

// The k-th largest key among the entries src(0..count) with key >= min_key (keys only:
// equal keys count once each, no ids): the key v with fewer than k entries above v and
// at least k at or above it; 0 when fewer than k entries qualify.  Four 8-bit digit
// passes from the top.  `count` must be the same in every thread; `hist` holds 256 bins.
// The source may live in global memory: each thread loads kKthBatch entries before it
// uses any, so a pass waits for one load latency per NT * kKthBatch entries.
constexpr int kKthBatch = 8;
template <int NT, class Src>
__device__ uint32_t block_kth_key(const Src &src, uint32_t count, uint32_t min_key, uint32_t k, uint32_t *hist,
                                  SelShared *sh) {
  const int t = threadIdx.x;
  const int lane = t & 31;
  uint32_t v = 0;
  for (uint32_t base = 0; base < count; base += NT * kKthBatch) {
    uint32_t key[kKthBatch];
#pragma unroll
    for (int u = 0; u < kKthBatch; ++u) {
      const uint32_t j = base + (uint32_t)u * NT + t;
      key[u] = j < count ? src(j).x : 0u;
    }
#pragma unroll
    for (int u = 0; u < kKthBatch; ++u) v += (base + (uint32_t)u * NT + t < count && key[u] >= min_key);
  }
  v = warp_sum_u32(v);
  if (t == 0) sh->valid = 0;
  __syncthreads();
  if (lane == 0) atomicAdd(&sh->valid, v);
  __syncthreads();
  if (sh->valid < k) return 0u;  // uniform
  uint32_t prefix = 0, need = k;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = t; b < 256; b += NT) hist[b] = 0;
    __syncthreads();
    for (uint32_t base = 0; base < count; base += NT * kKthBatch) {  // uniform trip count
      uint32_t key[kKthBatch];
#pragma unroll
      for (int u = 0; u < kKthBatch; ++u) {
        const uint32_t j = base + (uint32_t)u * NT + t;
        key[u] = j < count ? src(j).x : 0u;
      }
#pragma unroll
      for (int u = 0; u < kKthBatch; ++u) {
        if (base + (uint32_t)u * NT >= count) break;  // uniform: no entry of this slot in range
        uint32_t bin = 0xFFFFFFFFu;
        if (base + (uint32_t)u * NT + t < count && key[u] >= min_key &&
            (shift == 24 || (key[u] >> (shift + 8)) == (prefix >> (shift + 8))))
          bin = (key[u] >> shift) & 255u;
        if (!__any_sync(0xFFFFFFFFu, bin != 0xFFFFFFFFu)) continue;  // warp-uniform: nothing to count
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, bin);
        if (bin != 0xFFFFFFFFu && lane == __ffs(peers) - 1) atomicAdd(&hist[bin], (uint32_t)__popc(peers));
      }
    }
    __syncthreads();
    if (t < 32) {  // lane l owns bins [255-8l-7, 255-8l], visited from high to low
      const int top = 255 - 8 * t;
      uint32_t local[8], sum = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        local[b] = hist[top - b];
        sum += local[b];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (t >= o) incl += y;
      }
      const uint32_t excl = incl - sum;
      if (excl < need && need <= incl) {
        uint32_t run = excl;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          if (run + local[b] >= need) {
            sh->digit = (uint32_t)(top - b);
            sh->above = run;
            break;
          }
          run += local[b];
        }
      }
    }
    __syncthreads();
    need -= sh->above;
    prefix |= sh->digit << shift;
    __syncthreads();  // everyone has read the result before the next pass rewrites it
  }
  return prefix;
}

// Barrier after one stage of a bitonic network whose comparator i (thread i % NT, whole
// warps) exchanges elements lo = 2i - (i & (stride - 1)) and lo + stride.  Up to stride
// 32 the comparators of a warp touch only their own 64-element blocks, so the warp's
// own barrier orders the stage; larger strides need the block's.  The caller ends each
// size with a block barrier (the next size starts with its largest stride).
__device__ __forceinline__ void bitonic_stage_sync(uint32_t stride) {
  if (stride > 32) __syncthreads();
  else __syncwarp();
}

// Sort a[0..n) descending by composite (bitonic, padded to a power of two; the
// caller guarantees room for the padding).
template <int NT>
__device__ void block_sort_desc(uint2 *a, uint32_t n) {
  const int t = threadIdx.x;
  uint32_t P = 1;
  while (P < n) P <<= 1;
  for (uint32_t j = n + t; j < P; j += NT) a[j] = make_uint2(0u, 0xFFFFFFFFu);
  __syncthreads();
  for (uint32_t size = 2; size <= P; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = t; i < P / 2; i += NT) {
        const uint32_t lo = 2 * i - (i & (stride - 1));
        const uint32_t hi = lo + stride;
        const bool desc = (lo & size) == 0;
        const uint2 x = a[lo], y = a[hi];
        const uint64_t cx = composite(x.x, x.y), cy = composite(y.x, y.y);
        if (desc ? (cx < cy) : (cx > cy)) {
          a[lo] = y;
          a[hi] = x;
        }
      }
      bitonic_stage_sync(stride);
    }
    __syncthreads();
  }
}

// Lowest float whose key is >= thr, for thr > 0: keys 1..key(-inf) are the
// negative-NaN patterns no score maps to, so they all mean "any number".
__device__ __forceinline__ float thr_float(uint32_t thr) {
  return thr <= 0x007FFFFFu ? __int_as_float(0xFF800000) : key2f(thr);
}

}  // namespace topk
