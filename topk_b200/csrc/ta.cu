// The threshold algorithm over sorted attribute lists, on the device.
//
// The reference's TA (cpu/TA.h) sorts one list per attribute by value, descending
// (init, :40-58), then walks the queried lists in lock step: at depth i it scores every
// object it meets for the first time (random access to the table) and keeps the k best;
// the threshold is sum_m w_m * list_m[i], and it stops once the k-th score reaches it
// (:61-96).  Here the lists are built with stable device radix sorts (values
// descending, ties by the lower id) and kept as ids plus values, and a query walks them
// in blocks of growing depth (max(16384, 4k) entries per list, growing fourfold): one
// kernel takes every (list, depth) entry of the block, claims the object in a
// seen-bitmap (each object is scored once), scores it exactly in the reference order
// and appends it when it beats the current k-th; the appended keys and the running top
// k are radix-sorted and cut to k.  The bound of the unseen objects after depth i is
// the reference's threshold with each weight's sign respected (w < 0 takes the attribute's minimum), in the same FP32
// operations, so it bounds their scores exactly; the walk stops when the k-th score is
// strictly above it, so no unseen object can tie the k-th with a lower id.  Results are
// those of the full scan.
//
// The reference scores an object with the weight of the list it was found in for
// every attribute (cpu/TA.h:83: the inner loop reuses the outer `weight`), which gives
// wrong scores unless all weights are equal; this implementation uses each attribute's
// own weight.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/topk_b200.h"
#include "device_common.cuh"
#include "topk_internal.h"

namespace topk {

namespace {

struct TaQuery {
  uint32_t qq;
  uint8_t attr[kMaxQ];
  float w[kMaxQ];
};

__global__ void ta_keys_kernel(const float *__restrict__ col, uint64_t n, uint32_t *__restrict__ keys,
                               uint32_t *__restrict__ ids) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = f2key(__ldg(col + i));
    ids[i] = (uint32_t)i;
  }
}

__global__ void ta_values_kernel(const uint32_t *__restrict__ keys, uint64_t n, float *__restrict__ vals) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    vals[i] = key2f(keys[i]);
}

// Every entry (list m, depth i0 + j) of the block: first sight of the object claims it
// and scores it; it is appended when its key beats the current k-th key (0: fewer than
// k kept so far).
__global__ void __launch_bounds__(256)
    ta_score_kernel(const uint32_t *__restrict__ lists, uint64_t n, const float *__restrict__ table, uint64_t ld,
                    TaQuery q, uint64_t i0, uint64_t len, uint32_t *__restrict__ seen,
                    const unsigned long long *__restrict__ kth, unsigned long long *__restrict__ out,
                    uint32_t *__restrict__ count, uint32_t *__restrict__ scored) {
  const unsigned long long bar = *kth;
  const uint64_t total = len * q.qq;
  uint32_t mine = 0;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = (uint32_t)(e / len);
    const uint64_t pos = i0 + (e - (uint64_t)m * len);
    const uint32_t id = __ldg(lists + (uint64_t)q.attr[m] * n + pos);
    const uint32_t bit = 1u << (id & 31);
    if (atomicOr(seen + (id >> 5), bit) & bit) continue;  // met before
    ++mine;
    float s = 0.0f;
    for (uint32_t j = 0; j < q.qq; ++j)
      s = __fadd_rn(s, __fmul_rn(__ldg(table + (uint64_t)q.attr[j] * ld + id), q.w[j]));
    const unsigned long long key = composite(f2key(s), id);
    if (key > bar) out[atomicAdd(count, 1u)] = key;
  }
  mine = __reduce_add_sync(0xFFFFFFFFu, mine);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(scored, mine);
}

// The threshold after depth pos: sum_m w_m * (w_m >= 0 ? list_m[pos] : min_m), in the
// query's order with one rounding per operation (bounds every unseen object's score)
__global__ void ta_bound_kernel(const float *__restrict__ vals, uint64_t n, TaQuery q, uint64_t pos,
                                float *__restrict__ out) {
  float s = 0.0f;
  for (uint32_t j = 0; j < q.qq; ++j) {
    const float *list = vals + (uint64_t)q.attr[j] * n;
    const float x = q.w[j] >= 0.0f ? list[pos] : list[n - 1];
    s = __fadd_rn(s, __fmul_rn(x, q.w[j]));
  }
  *out = s;
}

int grid_of(uint64_t work, int num_sms) {
  const uint64_t b = (work + 255) / 256;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)num_sms * 16));
}

}  // namespace

// Sorted lists of the reference's TA: per attribute the ids by value descending (ties
// by the lower id) and the values in that order.  Both [d][n].
struct TaLists {
  uint64_t n = 0;
  uint32_t d = 0;
  uint32_t *ids = nullptr;
  float *vals = nullptr;
  // query scratch
  uint32_t *seen = nullptr;
  unsigned long long *buf[2] = {nullptr, nullptr};
  uint64_t cap = 0;
  void *temp = nullptr;
  size_t temp_bytes = 0;
  unsigned long long *kth = nullptr;
  uint32_t *counters = nullptr;  // [0] appended, [1] scored
  float *bound = nullptr;
  struct HostSlot {
    uint32_t count, scored;
    float bound;
    unsigned long long kth;
  } *host = nullptr;
  cudaStream_t s = nullptr;
  ~TaLists() {
    if (s) cudaStreamSynchronize(s);
    cudaFree(ids);
    cudaFree(vals);
    cudaFree(seen);
    cudaFree(buf[0]);
    cudaFree(buf[1]);
    cudaFree(temp);
    cudaFree(kth);
    cudaFree(counters);
    cudaFree(bound);
    cudaFreeHost(host);
    if (s) cudaStreamDestroy(s);
  }
};

void ta_lists_free(TaLists *L) { delete L; }

// Largest block of depth: its appended keys fit the scratch.
static uint64_t ta_block_cap(uint32_t qq) { return std::max<uint64_t>(1024, (1ull << 22) / std::max(1u, qq)); }

int ta_lists_build(TaLists **out, const float *table, uint64_t ld, uint32_t d, uint64_t n, int num_sms,
                   std::string *msg) {
  if (n > 0x7FFFFFFFull) {
    *msg = "sorted lists need n < 2^31";
    return TOPK_ERR_UNSUPPORTED;
  }
  TaLists *L = new TaLists();
  L->n = n;
  L->d = d;
  uint32_t *kin = nullptr, *kout = nullptr, *iin = nullptr;
  void *stemp = nullptr;
  size_t stb = 0;
  cudaError_t e = cudaStreamCreateWithFlags(&L->s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&L->ids, (size_t)d * n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&L->vals, (size_t)d * n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&kin, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&kout, n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&iin, n * sizeof(uint32_t));
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairsDescending(nullptr, stb, kin, kout, iin, L->ids, (int)n, 0, 32, L->s);
  if (e == cudaSuccess) e = cudaMalloc(&stemp, std::max<size_t>(stb, 16));
  const int g = grid_of(n, num_sms);
  for (uint32_t m = 0; m < d && e == cudaSuccess; ++m) {
    ta_keys_kernel<<<g, 256, 0, L->s>>>(table + (uint64_t)m * ld, n, kin, iin);
    size_t tb = stb;
    e = cub::DeviceRadixSort::SortPairsDescending(stemp, tb, kin, kout, iin, L->ids + (uint64_t)m * n, (int)n, 0, 32,
                                                  L->s);
    if (e == cudaSuccess) ta_values_kernel<<<g, 256, 0, L->s>>>(kout, n, L->vals + (uint64_t)m * n);
  }
  // query scratch: seen bitmap, two key buffers of k + one block's appends, sort scratch
  const uint64_t cap = kMaxK + (1ull << 22) + 64;
  if (e == cudaSuccess) e = cudaMalloc(&L->seen, ((n + 31) / 32) * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&L->buf[0], cap * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&L->buf[1], cap * sizeof(unsigned long long));
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortKeysDescending(nullptr, L->temp_bytes, L->buf[0], L->buf[1], (int)cap, 0, 64,
                                                  L->s);
  if (e == cudaSuccess) e = cudaMalloc(&L->temp, std::max<size_t>(L->temp_bytes, 16));
  if (e == cudaSuccess) e = cudaMalloc(&L->kth, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&L->counters, 2 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&L->bound, sizeof(float));
  if (e == cudaSuccess) e = cudaMallocHost(&L->host, sizeof(TaLists::HostSlot));
  if (e == cudaSuccess) e = cudaStreamSynchronize(L->s);
  cudaFree(kin);
  cudaFree(kout);
  cudaFree(iin);
  cudaFree(stemp);
  if (e != cudaSuccess) {
    *msg = std::string("building the sorted lists: ") + cudaGetErrorString(e);
    delete L;
    return e == cudaErrorMemoryAllocation ? TOPK_ERR_OOM : TOPK_ERR_CUDA;
  }
  L->cap = cap;
  *out = L;
  return TOPK_OK;
}

int ta_lists_read(const TaLists *L, uint32_t m, uint32_t *ids, float *vals, std::string *msg) {
  cudaError_t e = cudaSuccess;
  if (ids) e = cudaMemcpy(ids, L->ids + (uint64_t)m * L->n, L->n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && vals)
    e = cudaMemcpy(vals, L->vals + (uint64_t)m * L->n, L->n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    *msg = std::string("reading the lists: ") + cudaGetErrorString(e);
    return TOPK_ERR_CUDA;
  }
  return TOPK_OK;
}

int ta_query(TaLists *L, const float *table, uint64_t ld, uint64_t k, uint32_t qq, const float *weights,
             const uint8_t *attr, int num_sms, uint64_t *ids, float *scores, uint64_t *count, float *threshold,
             uint64_t *stats, std::string *msg) {
  const uint64_t n = L->n;
  const uint64_t kk = std::min<uint64_t>(k, n);
  TaQuery q{};
  q.qq = qq;
  for (uint32_t m = 0; m < qq; ++m) {
    q.attr[m] = attr[m];
    q.w[m] = weights[attr[m]];
  }
  cudaStream_t s = L->s;
  cudaError_t e = cudaMemsetAsync(L->seen, 0, ((n + 31) / 32) * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(L->kth, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(L->counters + 1, 0, sizeof(uint32_t), s);
  uint64_t kept = 0, depth = 0, iters = 0;
  int cur = 0;
  const uint64_t bmax = ta_block_cap(qq);
  uint64_t block = std::min<uint64_t>(bmax, std::max<uint64_t>(16384, 4 * kk));
  bool done = false;
  while (e == cudaSuccess && !done) {
    const uint64_t len = std::min<uint64_t>(block, n - depth);
    const uint32_t base = (uint32_t)kept;  // the running top k sits at the front of buf[cur]
    e = cudaMemcpyAsync(L->counters, &base, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) break;
    ta_score_kernel<<<grid_of(len * qq, num_sms), 256, 0, s>>>(L->ids, n, table, ld, q, depth, len, L->seen, L->kth,
                                                               L->buf[cur], L->counters, L->counters + 1);
    ta_bound_kernel<<<1, 1, 0, s>>>(L->vals, n, q, depth + len - 1, L->bound);
    e = cudaMemcpyAsync(&L->host->count, L->counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&L->host->bound, L->bound, sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) break;
    depth += len;
    ++iters;
    const uint64_t total = L->host->count;
    if (total > kept) {
      size_t tb = L->temp_bytes;
      e = cub::DeviceRadixSort::SortKeysDescending(L->temp, tb, L->buf[cur], L->buf[cur ^ 1], (int)total, 0, 64, s);
      if (e != cudaSuccess) break;
      cur ^= 1;
      kept = std::min<uint64_t>(kk, total);
      if (kept == kk) {  // the k-th key is the bar for later appends and the stop test
        e = cudaMemcpyAsync(L->kth, L->buf[cur] + kept - 1, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(&L->host->kth, L->kth, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) break;
      }
    }
    if (depth >= n) break;
    if (kept == kk) {
      // stop when the k-th score is strictly above every unseen object's bound
      const uint32_t kth_key = (uint32_t)(L->host->kth >> 32);
      const float b = L->host->bound;
      uint32_t bu;
      std::memcpy(&bu, &b, 4);
      const uint32_t bkey = (b != b) ? 0u : ((bu & 0x80000000u) ? ~bu : (bu | 0x80000000u));
      if (kth_key > bkey) done = true;
    }
    block = std::min<uint64_t>(bmax, block * 4);  // each block costs two host round trips
  }
  if (e != cudaSuccess) {
    *msg = std::string("TA query: ") + cudaGetErrorString(e);
    return TOPK_ERR_CUDA;
  }
  std::vector<unsigned long long> keys(kept);
  if (kept)
    e = cudaMemcpy(keys.data(), L->buf[cur], kept * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    *msg = std::string("TA query: ") + cudaGetErrorString(e);
    return TOPK_ERR_CUDA;
  }
  // ascending by score (the reference's heap drain): the descending keys reversed
  for (uint64_t j = 0; j < kept; ++j) {
    const unsigned long long key = keys[kept - 1 - j];
    const uint32_t kf = (uint32_t)(key >> 32);
    const uint32_t u = (kf & 0x80000000u) ? (kf & 0x7FFFFFFFu) : ~kf;
    float f;
    std::memcpy(&f, &u, 4);
    ids[j] = 0xFFFFFFFFull - (key & 0xFFFFFFFFull);
    scores[j] = f;
  }
  if (count) *count = kept;
  if (threshold) *threshold = kept ? scores[0] : 0.0f;
  if (stats) {
    stats[0] = depth;
    stats[1] = L->host->scored;
    stats[2] = iters;
  }
  return TOPK_OK;
}

}  // namespace topk
