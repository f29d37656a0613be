// Merge of per-shard top-k lists on the device: the last step of an object-sharded
// query.  The reference's threaded scan merges its per-thread heaps the same way
// (cpu/TPAc.h:335-346: every thread's k best pushed through one heap of k); here each
// shard is a GPU (or a row range), its list is exchanged with one collective, and one
// block keeps the best k of the union by an exact radix select on the (key, id) order
// (score descending, then the lower id), sorts them and writes them ascending.
//
// List layout (the exchange record of topk_b200/shard.py): list j starts at
// lists + j * 12 * stride: ids[stride] (u64), then scores[stride] (f32); its first
// counts[j] entries are valid, and base[j] is added to its ids (a shard table numbers
// its rows from 0; the merged ids are global).
#include <cstdint>
#include <cuda_runtime.h>

#include "block_select.cuh"
#include "device_common.cuh"
#include "topk_internal.h"

namespace topk {

namespace {

constexpr int kMT = 256;

struct MergeArgs {
  const unsigned char *lists;
  uint64_t stride;
  uint32_t nlists;
  uint32_t k;                      // min(k, total entries)
  uint32_t counts[kMaxMergeLists];
  uint32_t first[kMaxMergeLists + 1];  // prefix sums of counts
  uint32_t base[kMaxMergeLists];       // added to list j's ids (a shard's first global row)
  uint64_t *out_ids;
  float *out_scores;
  float *out_thr;
};

// Entry j of the union as (key, id).
struct ListSrc {
  const MergeArgs *a;
  __device__ uint2 operator()(uint32_t j) const {
    uint32_t l = 0;
    while (j >= a->first[l + 1]) ++l;
    const uint32_t i = j - a->first[l];
    const unsigned char *base = a->lists + (size_t)l * 12u * a->stride;
    const uint64_t id = reinterpret_cast<const uint64_t *>(base)[i];
    const float sc = reinterpret_cast<const float *>(base + 8u * a->stride)[i];
    return make_uint2(f2key(sc), (uint32_t)id + a->base[l]);
  }
};

__global__ void __launch_bounds__(kMT) merge_lists_kernel(const __grid_constant__ MergeArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  SelShared *sh = reinterpret_cast<SelShared *>(smem);
  uint32_t *hist = reinterpret_cast<uint32_t *>(smem + 64);
  uint2 *out = reinterpret_cast<uint2 *>(smem + 64 + 1024);
  const uint32_t total = a.first[a.nlists];
  const ListSrc src{&a};
  uint64_t prefix = 0, mask = 0;
  const bool select = total > a.k;
  if (select) block_radix_select<kMT>(src, total, 0u, a.k, hist, sh, prefix, mask);
  if (threadIdx.x == 0) sh->wcount = 0;
  __syncthreads();
  for (uint32_t base = 0; base < total; base += kMT) {  // uniform trip count
    const uint32_t j = base + threadIdx.x;
    uint2 e = make_uint2(0u, 0u);
    bool keep = false;
    if (j < total) {
      e = src(j);
      keep = !select || (composite(e.x, e.y) & mask) >= prefix;
    }
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
    uint32_t pos = 0;
    if ((threadIdx.x & 31) == 0 && bal) pos = atomicAdd(&sh->wcount, (uint32_t)__popc(bal));
    pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
    if (keep) out[pos + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u))] = e;
  }
  __syncthreads();
  const uint32_t n = a.k;  // exactly k kept (every composite is distinct)
  block_sort_desc<kMT>(out, n);
  for (uint32_t r = threadIdx.x; r < n; r += kMT) {
    const uint2 e = out[r];
    a.out_ids[n - 1 - r] = (uint64_t)e.y;  // ascending, like every result
    a.out_scores[n - 1 - r] = key2f(e.x);
  }
  if (threadIdx.x == 0 && a.out_thr) *a.out_thr = n ? key2f(out[n - 1].x) : 0.0f;
}

}  // namespace

cudaError_t launch_merge_lists(const unsigned char *lists, uint32_t nlists, uint64_t stride, const uint32_t *counts,
                               const uint32_t *base, uint32_t k, uint64_t *out_ids, float *out_scores, float *out_thr,
                               uint32_t *kept, cudaStream_t s) {
  if (nlists == 0 || nlists > kMaxMergeLists || k == 0 || k > kMaxK) return cudaErrorInvalidValue;
  MergeArgs a{};
  a.lists = lists;
  a.stride = stride;
  a.nlists = nlists;
  a.first[0] = 0;
  for (uint32_t j = 0; j < nlists; j++) {
    a.counts[j] = counts[j];
    a.first[j + 1] = a.first[j] + counts[j];
    a.base[j] = base ? base[j] : 0u;
  }
  a.k = k < a.first[nlists] ? k : a.first[nlists];
  *kept = a.k;
  if (a.k == 0) return cudaSuccess;
  a.out_ids = out_ids;
  a.out_scores = out_scores;
  a.out_thr = out_thr;
  uint32_t P = 1;
  while (P < a.k) P <<= 1;
  const size_t smem = 64 + 1024 + (size_t)P * 8;
  cudaError_t e = cudaFuncSetAttribute(merge_lists_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  merge_lists_kernel<<<1, kMT, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace topk
