// topk_query_noalloc: the fused scan + select without any allocation.
//
// Who needs it: callers that must not allocate GPU memory themselves or through
// this library.  Typical cases are host applications that own the whole device
// memory budget and hand every byte out through their own pool (a query engine
// running this as an operator, say), and latency-critical paths that cannot pay
// for cudaMalloc / cudaFree, which synchronise the whole device.  Such callers pass
// a table and output buffers they already own; the scratch the scan needs (its
// running threshold, arrival counters and merge-tree slots) lives in a fixed
// array compiled into this library.
//
// Limits and sharing:
//   * k <= kNoAllocMaxK (1024); the launch uses at most kNoAllocMaxGrid CTAs, and for
//     k above 256 fewer CTAs per SM than topk_query may use (the slots are fixed).
//   * The array takes kNoAllocScratchBytes (about 8.4 MB) of device memory on every
//     GPU that loads this library, for as long as the process lives.
//   * Every call on a device uses the same array.  Calls whose kernels overlap on
//     the GPU (different streams, or different host threads without ordering)
//     race on it and give wrong results; serialise them.
//   * The first call on each device does a one-time set-up on that device (it
//     looks up the array's device address and sets the kernels' shared-memory
//     limit); make that first call before capturing work on that device.
#include "../../include/topk_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "topk_internal.h"

using namespace topk;

namespace {

constexpr uint32_t kNoAllocMaxK = 1024;
// CTAs of one scan at most: 8 per SM of a B200 (148 SMs), as many as the scan's
// occupancy allows.  The merge-tree slots hold kNoAllocSlotEntries (key, id) entries
// in all; a scan with k entries per slot gets at most (entries / k - levels) / 2 CTAs
// (every CTA for k <= 256; about 3.4 per SM at k = 1024).
constexpr uint32_t kNoAllocMaxGrid = 8 * 148;
constexpr uint32_t kNoAllocSlotEntries = 1u << 20;  // 8 MiB
constexpr uint32_t kNoAllocMaxSlots = 2 * kNoAllocMaxGrid + kMaxLevels;
constexpr uint32_t kNoAllocMaxGroups = kNoAllocMaxGrid + kMaxLevels;
// published best keys before the merge: at most 8 * kPubMaxPerWarp per CTA
constexpr uint32_t kNoAllocPubEntries = 8 * kPubMaxPerWarp * kNoAllocMaxGrid;
// layout: ScanScratch | done[groups] | slot_count[slots] | pad | slots[entries] | pub[entries]
constexpr size_t kMetaBytes = sizeof(ScanScratch) + (size_t)kNoAllocMaxGroups * 4;
constexpr size_t kSlotsOff = (kMetaBytes + (size_t)kNoAllocMaxSlots * 4 + 255) / 256 * 256;
constexpr size_t kPubOff = kSlotsOff + (size_t)kNoAllocSlotEntries * sizeof(uint2);
constexpr size_t kNoAllocScratchBytes = kPubOff + (size_t)kNoAllocPubEntries * sizeof(uint2);

// The scratch.  In host code this name is only a stand-in for the symbol: its
// device address comes from cudaGetSymbolAddress below, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
// Per device: the SM count and shared-memory limit are written first, then the
// scratch address is published with a release store; a call that loads the address
// with acquire order and finds it set also sees the other two.
std::atomic<unsigned char *> g_scratch_ptr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};
size_t g_smem_optin[kMaxDevices] = {};

// Errors go to the same per-thread message that topk_last_error() returns.
int fail(int code, const char *fmt, ...) {
  char buf[384];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  set_last_error(buf);
  return code;
}

// One-time set-up for the current device: look up the scratch array's device
// address, read the SM count and shared-memory limit, set the scan kernels'
// shared-memory attribute.
int setup_current_device(int dev) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (g_scratch_ptr[dev].load(std::memory_order_acquire)) return TOPK_OK;
  void *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr) return fail(TOPK_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
  int v = 0;
  if ((e = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return fail(TOPK_ERR_CUDA, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
  g_num_sms[dev] = v;
  if ((e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
    return fail(TOPK_ERR_CUDA, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
  g_smem_optin[dev] = (size_t)v;
  if ((e = scan_set_attributes(g_smem_optin[dev])) != cudaSuccess)
    return fail(TOPK_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  g_scratch_ptr[dev].store(static_cast<unsigned char *>(ptr), std::memory_order_release);
  return TOPK_OK;
}

}  // namespace

extern "C" int topk_query_noalloc(const float *d_table, uint64_t n, uint64_t ld, uint32_t d, uint64_t k,
                                  uint32_t qq, const float *weights, const uint8_t *attr, uint64_t *d_ids,
                                  float *d_scores, float *d_threshold, void *stream) {
  set_last_error("");
  if (!d_table || !d_ids || !d_scores || !weights || !attr) return fail(TOPK_ERR_ARG, "null argument");
  if (n == 0 || d == 0 || d > TOPK_MAX_D) return fail(TOPK_ERR_ARG, "need n >= 1 and 1 <= d <= %u", TOPK_MAX_D);
  if (n >= 0xFFFFFFFFull) return fail(TOPK_ERR_UNSUPPORTED, "n must be < 2^32 - 1 (32-bit ids on the device)");
  if (ld < n || ld % 4 != 0) return fail(TOPK_ERR_ARG, "ld must be >= n and a multiple of 4");
  if (reinterpret_cast<uintptr_t>(d_table) % 16 != 0) return fail(TOPK_ERR_ARG, "d_table must be 16-byte aligned");
  if (k == 0) return fail(TOPK_ERR_ARG, "k must be >= 1");
  if (k > kNoAllocMaxK)
    return fail(TOPK_ERR_UNSUPPORTED, "k=%llu exceeds the %u that the fixed scratch of topk_query_noalloc holds",
                (unsigned long long)k, kNoAllocMaxK);
  if (qq == 0) return fail(TOPK_ERR_ARG, "qq must be >= 1");
  if (qq > kMaxQ) return fail(TOPK_ERR_UNSUPPORTED, "qq=%u exceeds TOPK_MAX_Q=%u", qq, kMaxQ);
  for (uint32_t m = 0; m < qq; m++)
    if (attr[m] >= d) return fail(TOPK_ERR_ARG, "attr[%u]=%u out of range (d=%u)", m, attr[m], d);

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(TOPK_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(TOPK_ERR_UNSUPPORTED, "device %d out of range", dev);
  unsigned char *blk = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!blk) {
    const int st = setup_current_device(dev);
    if (st != TOPK_OK) return st;
    blk = g_scratch_ptr[dev].load(std::memory_order_acquire);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the result holds min(k, n) objects, as topk_query's does
  const uint64_t kk = std::min<uint64_t>(k, n);

  ScanPlan pl = plan_scan(qq, (uint32_t)kk, n, g_num_sms[dev], g_smem_optin[dev]);
  if (pl.stages < 1) return fail(TOPK_ERR_UNSUPPORTED, "qq=%u, k=%llu do not fit in shared memory", qq, (unsigned long long)kk);
  ScanParams p{};
  p.table = d_table;
  p.ld = ld;
  p.row_begin = 0;
  p.row_end = n;
  p.tile_begin = 0;
  p.tile_end = (n + 3) & ~3ull;
  p.tile_step = pl.tile;
  const uint64_t tiles = (p.tile_end + pl.tile - 1) / pl.tile;
  p.num_tiles = (uint32_t)tiles;
  if ((uint64_t)pl.grid > tiles) pl.grid = (int)tiles;
  if ((uint32_t)pl.grid > kNoAllocMaxGrid) pl.grid = (int)kNoAllocMaxGrid;
  // the merge tree's slots (< (2 * grid + levels) * k entries) within the fixed array
  const uint64_t max_grid_k = (kNoAllocSlotEntries / kk - (uint64_t)kMaxLevels) / 2;
  if ((uint64_t)pl.grid > max_grid_k) pl.grid = (int)max_grid_k;
  p.qq = qq;
  p.k = (uint32_t)kk;
  p.cap = pl.cap;
  p.mcap = pl.mcap;
  uint32_t tree_slots = 0, tree_groups = 0;
  plan_merge_tree(p, (uint32_t)pl.grid, pl.fanin, &tree_slots, &tree_groups);
  if (tree_slots > kNoAllocMaxSlots || tree_groups > kNoAllocMaxGroups || p.nslots[p.levels] != 1 ||
      (uint64_t)tree_slots * kk > kNoAllocSlotEntries)
    return fail(TOPK_ERR_UNSUPPORTED, "merge tree of %d CTAs does not fit the fixed scratch", pl.grid);
  // No wait hook: with fault_mode 0 the scan has no device-side wait that can give
  // up (its only bounded wait is the fault-injection barrier of the handle-based
  // path), so a launch that succeeds always runs to the root and writes ids, scores
  // and the threshold; a failure shows as a CUDA error on the stream.
  p.wait_limit = 1ull << 26;
  p.fault_mode = 0;
  if (kk >= kPubMinK && (uint32_t)pl.grid >= kPubMinGrid) {
    p.pub = reinterpret_cast<uint2 *>(blk + kPubOff);
    p.pub_m = pub_keys_per_cta((uint32_t)kk, (uint32_t)pl.grid);
    p.pub_wait = kPubWaitPolls;
  }
  p.scratch = reinterpret_cast<ScanScratch *>(blk);
  p.done = reinterpret_cast<uint32_t *>(blk + sizeof(ScanScratch));
  p.slot_count = reinterpret_cast<uint32_t *>(blk + kMetaBytes);
  p.slots = reinterpret_cast<uint2 *>(blk + kSlotsOff);
  p.out_ids = d_ids;
  p.out_scores = d_scores;
  p.out_threshold = d_threshold;
  p.out_count = nullptr;
  p.out_stats = nullptr;
  for (uint32_t m = 0; m < qq; m++) {
    p.attr[m] = attr[m];
    p.w[m] = weights[attr[m]];
  }
  // The array keeps whatever the previous call left: zero the threshold and the
  // arrival counters (the scan expects them at zero when it starts).
  if ((e = cudaMemsetAsync(blk, 0, kMetaBytes, s)) != cudaSuccess)
    return fail(TOPK_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
  // Large k over a large table: the threshold pass over every kSampleStride-th tile
  // first, as topk_query runs it; its bound goes to a spare word of the array's header
  // (zeroed above) and seeds the scan.
  if (p.pub && kk >= sample_min_k(qq) && tiles >= kSampleMinTiles) {
    uint32_t *seed_word = &p.scratch->pad[0];
    ScanParams q = p;
    q.num_tiles = (uint32_t)((tiles + kSampleStride - 1) / kSampleStride);
    q.tile_step = (uint64_t)pl.tile * kSampleStride;
    q.kth_only = 1;
    q.out_kth_key = seed_word;
    q.out_ids = nullptr;
    q.out_scores = nullptr;
    q.out_threshold = nullptr;
    ScanPlan qp = pl;
    qp.grid = (int)std::min<uint64_t>((uint64_t)pl.grid, q.num_tiles);
    if ((uint32_t)qp.grid >= kPubMinGrid) {
      q.pub_m = pub_keys_per_cta((uint32_t)kk, (uint32_t)qp.grid);
      if ((e = launch_scan(qp, q, s)) != cudaSuccess)
        return fail(TOPK_ERR_CUDA, "threshold pass launch: %s", cudaGetErrorString(e));
      p.thr_seed_dev = seed_word;
    }
  }
  if ((e = launch_scan(pl, p, s)) != cudaSuccess)
    return fail(TOPK_ERR_CUDA, "scan launch: %s", cudaGetErrorString(e));
  return TOPK_OK;
}
