// Host runtime behind the C ABI (include/topk_b200.h).
//
// A handle owns the device copy of the table (column-major, stride ld = n rounded
// up to 64 rows so every column starts 256-byte aligned, which the bulk copies
// need) and a pool of query contexts.  A context is one stream, one device
// scratch block for the fused scan, one device result block and a pinned host
// mirror of it, so a synchronous query costs one kernel launch, one
// device-to-host copy and one stream synchronisation.  Concurrent callers (the
// reference's findTopKsimdMQ threads, validation/bench_cpu.h:204-212) each take
// their own context from the pool.
#include "../../include/topk_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "batch_internal.h"
#include "topk_internal.h"

using namespace topk;

namespace {

thread_local std::string g_last_error;
thread_local uint64_t g_last_cands = 0, g_last_reductions = 0;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  if (e == cudaErrorMemoryAllocation) return fail(TOPK_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
  return fail(TOPK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                    \
  do {                                              \
    cudaError_t _e = (call);                        \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

// Switch to the handle's device for the duration of a call.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Result block layout (device and pinned host mirror): header, ids[k], scores[k].
struct ResultHeader {
  uint32_t count;
  float threshold;
  uint32_t stats[3];  // candidates in the final select, block-selects, tiles scanned
  float cut;          // a pruned query's learned cut
  uint32_t pad[10];
};
constexpr size_t kHdr = sizeof(ResultHeader);  // 64 bytes
size_t result_bytes(uint32_t k) { return kHdr + (size_t)k * 8 + (size_t)k * 4; }
// The pinned result mirror also stages a pruned query's descriptor after the result.
constexpr size_t kStageBytes = 256;

struct Ctx {
  cudaStream_t stream = nullptr;
  // Device scratch of the fused scan, one allocation:
  //   ScanScratch | done[max_groups] | slot_count[max_slots] | pad | slots[max_slots * kMaxK]
  ScanScratch *scratch = nullptr;
  uint32_t *done = nullptr;
  uint32_t *slot_count = nullptr;
  uint2 *slots = nullptr;
  uint2 *pub = nullptr;  // published best keys before the merge (8 * kPubMaxPerWarp per CTA of the largest grid)
  uint32_t *d_seed_word = nullptr;  // a threshold pass's bound, read by the scan after it
  uint32_t max_slots = 0, max_groups = 0;
  size_t slot_entries = 0;  // capacity of `slots`
  size_t meta_bytes = 0;    // bytes that must be zero between queries (header + done)
  unsigned char *d_res = nullptr;  // device result block (kMaxK capacity)
  unsigned char *h_res = nullptr;  // pinned mirror
  // Result block of the synchronous queries in mapped pinned memory (h_out on the host,
  // d_out its device address): the scan's root writes ids, scores and the header
  // straight to the host, so no copy follows the scan.
  unsigned char *h_out = nullptr;
  unsigned char *d_out = nullptr;
  unsigned long long *d_count2 = nullptr;
  uint64_t *d_ids_scratch = nullptr;  // gather ids
  float *d_rows = nullptr;
  size_t rows_cap = 0;
  // pruned queries: partitions by bound and their bound keys, the radix sort's scratch
  // (many partitions only), the learned start's descriptor, features, prediction, seed
  uint32_t *d_plist = nullptr, *d_pkey = nullptr;
  size_t plist_cap = 0;
  void *d_ptemp = nullptr;
  size_t ptemp_bytes = 0;
  unsigned char *d_lq = nullptr;
  bool busy = false;
};

}  // namespace

void topk::set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

struct topk_table_s {
  int device = 0;
  uint64_t n = 0, ld = 0;
  uint32_t d = 0;
  float *table = nullptr;
  bool has_data = false;
  int num_sms = 148;
  size_t smem_optin = 0;
  uint64_t wait_limit = 1ull << 26;
  int fault_mode = 0;
  uint32_t max_ctas_per_sm = 0;  // 0 = as many as fit
  uint32_t *d_minmax = nullptr;
  float *d_norm = nullptr;  // mins[d], ranges[d]
  std::mutex mu;
  std::condition_variable cv;
  std::vector<Ctx *> ctxs;
  Ctx *primary = nullptr;
  // batched path: one batch at a time per handle, device buffers grow and are kept
  std::mutex batch_mu;
  int batch_method = TOPK_BATCH_AUTO;
  // batch tiles (topk_set_batch_tiles / topk_tune_batch): query tiles per filter CTA
  // (0: up to the kernel's 16) and rows of the exact bootstrap (= the first chunk)
  uint32_t batch_qt = 0, batch_boot = kBatchBootRows;
  struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
  };
  DevBuf b_q, b_st, b_best, b_cand, b_ids, b_scores, b_count, b_thr;
  // BF16 filter: split copy of the table (rebuilt when the table changed), the
  // per-column max |x| it was built from, the batch's query tiles and error word
  DevBuf xbf, xbf_absmax, b_abf, b_err, b_log, b_logh, b_sw, b_feat, b_pred;
  // compact active query tiles of the filter, slot -> query map and count; the plain
  // FP32 scorer's query order (by attribute count)
  DevBuf b_abf_act, b_amap, b_order;
  uint64_t data_version = 1, xbf_version = 0;
  std::vector<float> absmax, colmax, colmin;  // per column: max |x|, max, min (NaN left out)
  bool xbf_usable = false;
  // partitioned copy for pruned queries (topk_build_partitions): rows reordered,
  // original ids, per-partition [P][d] min / max / mean (device and host copies)
  float *ptable = nullptr;
  LoaderState *loader = nullptr;  // table-file pipeline buffers, made on the first load
  std::mutex loader_mu;           // one load / row-major transfer at a time uses them
  TaLists *ta = nullptr;          // sorted lists of the threshold algorithm
  uint64_t ta_version = 0;
  std::mutex ta_mu;               // TA queries share the lists' scratch
  uint32_t *pids = nullptr;
  float *pstats = nullptr;
  uint32_t part_log2 = 0, num_parts = 0;
  uint64_t part_version = 0;
  std::vector<float> pmin, pmax, pmean;
  // learned k-th-score model (topk_set_learned_model / topk_learned_fit): device
  // parameters, calibrated margin (in units of S = sum |w|), one query's buffers
  std::mutex learned_mu;
  float *mlp = nullptr;
  float mlp_margin = 0.0f;
  uint64_t mlp_part_version = 0;
  BatchQuery *lq_query = nullptr;
  float *lq_out = nullptr;  // features (kMlpMaxIn) then the prediction
  cudaEvent_t b_ev0 = nullptr, b_ev1 = nullptr;
  double last_batch_ms = 0, last_batch_err_ratio = 0;
  uint64_t last_batch_fallbacks = 0, last_batch_cands = 0, last_batch_learned_misses = 0;
  uint64_t last_batch_switched = 0;  // queries a hybrid batch moved from the filter to the FP32 scorer
  uint64_t last_batch_retired = 0;   // queries the filter retired (threshold above their score bound)
  double last_batch_filter_flops = 0;  // MMA flops the filter ran (three BF16 passes)
  // pinned host copies of a batch's results (grow-only): copied at full link speed,
  // no page faults on the critical path
  void *hb_res = nullptr;
  size_t hb_bytes = 0;
  // the device work of a batch, captured once per shape and replayed (a few shapes:
  // a learned batch's rerun of its misses is a second one)
  struct BatchGraph {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
    uint64_t used = 0;
  };
  BatchGraph b_graphs[4];
  uint64_t b_graph_tick = 0;
  // TOPK_BATCH_AUTO's memory: the table version on which the BF16 filter handed more
  // than three quarters of a batch's queries to the FP32 scorer (0: none)
  uint64_t auto_fp32_version = 0;
  int last_batch_method = 0;
};

namespace {

constexpr size_t kMaxContexts = 64;

int ctx_create(topk_table_t h, Ctx **out) {
  Ctx *c = new Ctx();
  auto bail = [&](cudaError_t e, const char *what) {
    if (c->stream) cudaStreamDestroy(c->stream);
    cudaFree(c->scratch);
    cudaFree(c->pub);
    cudaFree(c->d_seed_word);
    cudaFree(c->d_res);
    cudaFree(c->d_count2);
    if (c->h_res) cudaFreeHost(c->h_res);
    if (c->h_out) cudaFreeHost(c->h_out);
    delete c;
    return cuda_fail(e, what);
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
  // grid <= num_sms * 8 CTAs (256 threads each); with fan-in >= 2 each tree level has
  // at most half the slots of the one below, rounded up, so slots <= 2 * grid + levels
  // and groups <= grid + levels.  Slot entries (slots * k) have their own budget: the
  // planner keeps grid * k within it (large k means few CTAs per SM anyway).
  const uint32_t max_grid = (uint32_t)h->num_sms * 8u;
  c->max_slots = 2u * max_grid + (uint32_t)kMaxLevels;
  c->max_groups = max_grid + (uint32_t)kMaxLevels;
  c->slot_entries = (size_t)4 * (size_t)h->num_sms * kMaxK;
  c->meta_bytes = sizeof(ScanScratch) + (size_t)c->max_groups * 4;
  const size_t slots_off = (c->meta_bytes + (size_t)c->max_slots * 4 + 255) / 256 * 256;
  const size_t bytes = slots_off + c->slot_entries * sizeof(uint2);
  unsigned char *blk = nullptr;
  if ((e = cudaMalloc(&blk, bytes)) != cudaSuccess) return bail(e, "scan scratch");
  c->scratch = reinterpret_cast<ScanScratch *>(blk);
  c->done = reinterpret_cast<uint32_t *>(blk + sizeof(ScanScratch));
  c->slot_count = reinterpret_cast<uint32_t *>(blk + c->meta_bytes);
  c->slots = reinterpret_cast<uint2 *>(blk + slots_off);
  if ((e = cudaMemset(blk, 0, slots_off)) != cudaSuccess) return bail(e, "scratch memset");
  if ((e = cudaMalloc(&c->pub, (size_t)8 * kPubMaxPerWarp * max_grid * sizeof(uint2))) != cudaSuccess)
    return bail(e, "publish area");
  if ((e = cudaMalloc(&c->d_seed_word, 256)) != cudaSuccess) return bail(e, "seed word");
  if ((e = cudaMalloc(&c->d_res, result_bytes(kMaxK))) != cudaSuccess) return bail(e, "result block");
  if ((e = cudaMalloc(&c->d_count2, 2 * sizeof(unsigned long long))) != cudaSuccess) return bail(e, "count");
  if ((e = cudaHostAlloc(&c->h_res, result_bytes(kMaxK) + kStageBytes, cudaHostAllocDefault)) != cudaSuccess)
    return bail(e, "pinned result");
  if ((e = cudaHostAlloc(&c->h_out, result_bytes(kMaxK), cudaHostAllocMapped)) != cudaSuccess)
    return bail(e, "mapped result");
  if ((e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&c->d_out), c->h_out, 0)) != cudaSuccess)
    return bail(e, "mapped result address");
  *out = c;
  return TOPK_OK;
}

void ctx_free(Ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->stream) cudaStreamDestroy(c->stream);
  cudaFree(c->scratch);
  cudaFree(c->pub);
  cudaFree(c->d_seed_word);
  cudaFree(c->d_res);
  cudaFree(c->d_count2);
  cudaFree(c->d_ids_scratch);
  cudaFree(c->d_rows);
  cudaFree(c->d_plist);
  cudaFree(c->d_pkey);
  cudaFree(c->d_ptemp);
  cudaFree(c->d_lq);
  if (c->h_res) cudaFreeHost(c->h_res);
  if (c->h_out) cudaFreeHost(c->h_out);
  delete c;
}

// Take a free context (creating one up to kMaxContexts, else wait for one).
int ctx_acquire(topk_table_t h, Ctx **out) {
  std::unique_lock<std::mutex> lk(h->mu);
  for (;;) {
    for (Ctx *c : h->ctxs)
      if (!c->busy) { c->busy = true; *out = c; return TOPK_OK; }
    if (h->ctxs.size() < kMaxContexts) {
      Ctx *c = nullptr;
      int st = ctx_create(h, &c);
      if (st != TOPK_OK) return st;
      c->busy = true;
      h->ctxs.push_back(c);
      *out = c;
      return TOPK_OK;
    }
    h->cv.wait(lk);
  }
}

void ctx_release(topk_table_t h, Ctx *c) {
  {
    std::lock_guard<std::mutex> lk(h->mu);
    c->busy = false;
  }
  h->cv.notify_one();
}

struct CtxLease {
  topk_table_t h;
  Ctx *c = nullptr;
  int status;
  explicit CtxLease(topk_table_t hh) : h(hh) { status = ctx_acquire(h, &c); }
  ~CtxLease() { if (c) ctx_release(h, c); }
};

int check_query(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (!h->has_data) return fail(TOPK_ERR_STATE, "no table data: call topk_upload_colmajor or topk_generate first");
  if (k == 0) return fail(TOPK_ERR_ARG, "k must be >= 1");
  if (k > kMaxK) return fail(TOPK_ERR_UNSUPPORTED, "k=%llu exceeds TOPK_MAX_K=%u", (unsigned long long)k, kMaxK);
  if (qq == 0) return fail(TOPK_ERR_ARG, "qq must be >= 1");
  if (qq > kMaxQ) return fail(TOPK_ERR_UNSUPPORTED, "qq=%u exceeds TOPK_MAX_Q=%u", qq, kMaxQ);
  if (!weights || !attr) return fail(TOPK_ERR_ARG, "null weights or attr");
  for (uint32_t m = 0; m < qq; m++)
    if (attr[m] >= h->d) return fail(TOPK_ERR_ARG, "attr[%u]=%u out of range (d=%u)", m, attr[m], h->d);
  return TOPK_OK;
}

// A scan over a list of partitions of the partitioned copy, with a threshold seed.
struct PartScan {
  const uint32_t *d_list;  // partition numbers (device), by bound descending
  uint32_t count;
  uint32_t seed;           // objects need key >= seed (0: none)
  const uint32_t *d_key;   // bound key of each listed partition (null: no stop rule)
  const uint32_t *d_seed;  // a further seed in device memory (null: none)
  uint32_t *d_kth;         // receives the k-th key when k objects were found, else 0 (may be null)
  uint32_t max_ctas_per_sm;  // 0: as many as fit
  bool kth_only;           // threshold pass: only the bound from the published keys, into d_kth
};

// Enqueue one fused scan over rows [r0, r1) (or over the partitions of `ps`)
// writing into the given outputs.
int enqueue_scan(topk_table_t h, Ctx *c, cudaStream_t stream, uint64_t r0, uint64_t r1, uint64_t k, uint32_t qq,
                 const float *weights, const uint8_t *attr, uint64_t *d_ids, float *d_scores, float *d_thr,
                 uint32_t *d_count, uint32_t *d_stats = nullptr, const PartScan *ps = nullptr) {
  const uint64_t rows = ps ? ((uint64_t)ps->count << h->part_log2) : r1 - r0;
  ScanPlan pl = plan_scan(qq, (uint32_t)k, rows, h->num_sms, h->smem_optin, h->max_ctas_per_sm, ps != nullptr);
  if (pl.stages < 1) return fail(TOPK_ERR_UNSUPPORTED, "qq=%u, k=%llu do not fit in shared memory", qq, (unsigned long long)k);
  // keep the merge tree's slot entries (< (2 * grid + levels) * k) within the context budget
  const uint64_t max_grid_k = (c->slot_entries / k - (uint64_t)kMaxLevels) / 2;
  if ((uint64_t)pl.grid > max_grid_k) pl.grid = (int)max_grid_k;
  if ((uint64_t)pl.grid > c->max_groups - (uint64_t)kMaxLevels) pl.grid = (int)(c->max_groups - kMaxLevels);
  ScanParams p{};
  p.table = h->table;
  p.ld = h->ld;
  p.row_begin = r0;
  p.row_end = r1;
  p.tile_begin = r0 & ~3ull;
  p.tile_end = (r1 + 3) & ~3ull;
  p.tile_step = pl.tile;
  const uint64_t span = p.tile_end - p.tile_begin;
  uint64_t tiles = (span + pl.tile - 1) / pl.tile;
  if (ps) {  // tiles of the listed partitions of the reordered copy, original ids
    uint32_t tile_log2 = 0;
    while ((1u << tile_log2) < pl.tile) ++tile_log2;
    if ((1u << tile_log2) != pl.tile || h->part_log2 < tile_log2)
      return fail(TOPK_ERR_STATE, "partition rows 2^%u below the scan tile %u", h->part_log2, pl.tile);
    p.table = h->ptable;
    p.row_begin = 0;
    p.row_end = h->n;
    p.tile_begin = 0;
    p.tile_end = (h->n + 3) & ~3ull;
    p.part_list = ps->d_list;
    p.part_shift = h->part_log2 - tile_log2;
    p.part_rows_log2 = h->part_log2;
    p.row_ids = h->pids;
    p.thr_seed = ps->seed;
    p.part_key = ps->d_key;
    p.thr_seed_dev = ps->d_seed;
    p.out_kth_key = ps->d_kth;
    tiles = (uint64_t)ps->count << p.part_shift;
    if (tiles > 0xFFFFFFFFull) return fail(TOPK_ERR_UNSUPPORTED, "too many tiles");
  }
  p.num_tiles = (uint32_t)tiles;
  if (ps && ps->max_ctas_per_sm && (uint64_t)pl.grid > (uint64_t)h->num_sms * ps->max_ctas_per_sm)
    pl.grid = (int)((uint64_t)h->num_sms * ps->max_ctas_per_sm);
  if (ps && ps->d_key) {
    // With the stop rule, the first wave of CTAs scans its tiles before any threshold
    // exists; on a small copy keep that wave to about 1/32 of the tiles (one CTA per
    // SM at least), so most partitions are still decided by the rule.
    const uint64_t cap = std::max<uint64_t>((uint64_t)h->num_sms, tiles / 32);
    if ((uint64_t)pl.grid > cap) pl.grid = (int)cap;
  }
  if ((uint64_t)pl.grid > tiles) pl.grid = (int)tiles;
  p.qq = qq;
  p.k = (uint32_t)k;
  p.cap = pl.cap;
  p.mcap = pl.mcap;
  uint32_t tree_slots = 0, tree_groups = 0;
  plan_merge_tree(p, (uint32_t)pl.grid, pl.fanin, &tree_slots, &tree_groups);
  if (tree_slots > c->max_slots || tree_groups > c->max_groups || p.nslots[p.levels] != 1 ||
      (size_t)tree_slots * k > c->slot_entries)
    return fail(TOPK_ERR_UNSUPPORTED, "merge tree of %d CTAs does not fit the scratch", pl.grid);
  p.wait_limit = h->wait_limit;
  p.fault_mode = (uint32_t)h->fault_mode;
  if (k >= kPubMinK && (uint32_t)pl.grid >= kPubMinGrid) {
    p.pub = c->pub;
    p.pub_m = pub_keys_per_cta((uint32_t)k, (uint32_t)pl.grid);
    p.pub_wait = kPubWaitPolls;
  }
  p.scratch = c->scratch;
  p.slots = c->slots;
  p.slot_count = c->slot_count;
  p.done = c->done;
  p.out_ids = d_ids;
  p.out_scores = d_scores;
  p.out_threshold = d_thr;
  p.out_count = d_count;
  p.out_stats = d_stats;
  for (uint32_t m = 0; m < qq; m++) {
    p.attr[m] = attr[m];
    p.w[m] = weights[attr[m]];
  }
  if (ps && ps->kth_only) {
    // Every CTA publishes up to 4k / grid keys (at most 8 * kPubMaxPerWarp), so the
    // bound stays close to the k-th of the scanned rows even when their best objects
    // sit in few CTAs.  When the grid is too small for that (few tiles, large k) the
    // round runs the merge tree instead, whose root writes the exact k-th key of the
    // rows it scanned.
    const uint32_t m = pub_keys_per_cta(4 * (uint32_t)k, (uint32_t)pl.grid);
    if ((uint64_t)m * (uint64_t)pl.grid >= 4 * k) {
      p.pub = c->pub;
      p.pub_m = m;
      p.pub_wait = kPubWaitPolls;
      p.kth_only = 1;
    }
    p.out_kth_key = ps->d_kth;
    p.out_ids = nullptr;
    p.out_scores = nullptr;
    p.out_threshold = nullptr;
    p.out_count = nullptr;
    p.out_stats = nullptr;
  }
  // Large k over a large table in id order: a threshold pass over every
  // kSampleStride-th tile first (its own launch, same kernel, no merge), whose bound
  // seeds this scan, so its CTAs rarely need a select.
  if (!ps && p.pub && k >= sample_min_k(qq) && tiles >= kSampleMinTiles) {
    ScanParams q = p;
    q.num_tiles = (uint32_t)((tiles + kSampleStride - 1) / kSampleStride);
    q.tile_step = (uint64_t)pl.tile * kSampleStride;
    q.kth_only = 1;
    q.out_kth_key = c->d_seed_word;
    q.out_ids = nullptr;
    q.out_scores = nullptr;
    q.out_threshold = nullptr;
    q.out_count = nullptr;
    q.out_stats = nullptr;
    ScanPlan qp = pl;
    qp.grid = (int)std::min<uint64_t>((uint64_t)pl.grid, q.num_tiles);
    if ((uint32_t)qp.grid >= kPubMinGrid) {
      q.pub_m = pub_keys_per_cta((uint32_t)k, (uint32_t)qp.grid);
      CK(launch_scan(qp, q, stream));
      p.thr_seed_dev = c->d_seed_word;
    }
  }
  CK(launch_scan(pl, p, stream));
  return TOPK_OK;
}

// Synchronous query into host buffers through a leased context.
int run_query_sync(topk_table_t h, uint64_t r0, uint64_t r1, uint64_t k, uint32_t qq, const float *weights,
                   const uint8_t *attr, uint64_t *ids, float *scores, uint64_t *count, float *threshold) {
  int st = check_query(h, k, qq, weights, attr);
  if (st != TOPK_OK) return st;
  if (r1 > h->n || r0 > r1) return fail(TOPK_ERR_ARG, "row range [%llu, %llu) outside [0, %llu)",
                                        (unsigned long long)r0, (unsigned long long)r1, (unsigned long long)h->n);
  const uint64_t kk = std::min<uint64_t>(k, r1 - r0);
  if (kk == 0) {
    if (count) *count = 0;
    if (threshold) *threshold = 0.0f;
    return TOPK_OK;
  }
  if (!ids || !scores) return fail(TOPK_ERR_ARG, "null output buffer");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  CtxLease lease(h);
  if (lease.status != TOPK_OK) return lease.status;
  Ctx *c = lease.c;
  // the result goes straight to the mapped block (no copy after the scan)
  unsigned char *dr = c->d_out;
  ResultHeader *dh = reinterpret_cast<ResultHeader *>(dr);
  uint64_t *d_ids = reinterpret_cast<uint64_t *>(dr + kHdr);
  float *d_scores = reinterpret_cast<float *>(dr + kHdr + kk * 8);
  volatile ResultHeader *hh = reinterpret_cast<volatile ResultHeader *>(c->h_out);
  // a sentinel count tells a completed scan from one that left early
  hh->count = 0xFFFFFFFFu;
  st = enqueue_scan(h, c, c->stream, r0, r1, k, qq, weights, attr, d_ids, d_scores, &dh->threshold, &dh->count,
                    dh->stats);
  if (st != TOPK_OK) return st;
  CK(cudaStreamSynchronize(c->stream));
  if (hh->count != (uint32_t)kk) {
    ScanScratch s{};
    cudaMemcpy(&s, c->scratch, sizeof(s), cudaMemcpyDeviceToHost);
    cudaMemset(c->scratch, 0, c->meta_bytes);  // threshold, counters and group arrivals
    if (s.error & 1u)
      return fail(TOPK_ERR_TIMEOUT, "device wait gave up (limit %llu polls); diag %u block %u tile %u [%u %u]",
                  (unsigned long long)h->wait_limit, s.diag[0], s.diag[1], s.diag[2], s.diag[3], s.diag[4]);
    return fail(TOPK_ERR_CUDA, "scan did not complete (count %u, expected %llu, error 0x%x); diag %u block %u tile %u [%u %u]",
                (uint32_t)hh->count, (unsigned long long)kk, s.error, s.diag[0], s.diag[1], s.diag[2], s.diag[3],
                s.diag[4]);
  }
  std::memcpy(ids, c->h_out + kHdr, kk * 8);
  std::memcpy(scores, c->h_out + kHdr + kk * 8, kk * 4);
  if (count) *count = kk;
  if (threshold) *threshold = hh->threshold;
  g_last_cands = hh->stats[0];
  g_last_reductions = hh->stats[1];
  return TOPK_OK;
}

// ---------------------------------------------------------------- pruned queries
uint32_t host_f2key(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if (f != f) return 0u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

float host_key2f(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}


std::vector<BatchQuery> pack_queries(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs,
                                     const float *weights, uint64_t wstride, const uint8_t *attrs, uint64_t astride);

// CTAs per SM of a pruned scan and of its first round (measured on 2^27 x 8, kd order:
// 4 and 3 take 148 us a query against 153 for 3 and 4)
constexpr uint32_t kPrunedCtasPerSm = 4;
constexpr uint32_t kRound1CtasPerSm = 3;

// Exact top-k over the partitioned copy as one device pipeline on the context's
// stream; nothing is decided on the host between the launches.
//   1. A kernel orders the partitions by the query's bound (the reference-order FP32
//      sum over each partition's extremes: an exact upper bound of its scores).
//   2. Round 1 scans the first partitions of that order, about one wave of CTAs (and
//      enough rows for k), and leaves its k-th key t1 in device memory: the k-th score
//      of a subset, a lower bound of the true k-th.
//   3. Round 2 scans the partitions in the same order seeded with t1 (ties at t1 kept),
//      each CTA stopping at its first partition whose bound is below its running
//      threshold -- the reference's stop rule per block (cpu/VTA.h:210-216,
//      cpu/PTA.h:636-641); its merge tree gives the result.  (Round 1's partitions
//      come again; rescanning them is cheaper than merging two results.)
// With a seed (a predicted lower bound of the k-th score: `cut`, or the learned
// model's cut computed on the device) round 2 alone runs with it, and its result is
// accepted when it holds min(k, n) objects (then the true k-th score is at least the
// seed, so every object of the true top-k was scanned); otherwise the two rounds run
// without it.  stats: partitions scanned (tiles scanned / tiles per partition, over
// every scan), partitions, seed accepted (1/0), scans.
int run_pruned(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr, float cut,
               bool learned, uint64_t *ids, float *scores, uint64_t *count, float *threshold, uint64_t *stats,
               float *cut_out) {
  int st = check_query(h, k, qq, weights, attr);
  if (st != TOPK_OK) return st;
  if (!h->ptable || h->part_version != h->data_version)
    return fail(TOPK_ERR_STATE, "no partitions for the current table: call topk_build_partitions");
  const uint64_t kk = std::min<uint64_t>(k, h->n);
  if (!ids || !scores) return fail(TOPK_ERR_ARG, "null output buffer");
  if (learned && qq > kBatchMaxQ) return fail(TOPK_ERR_UNSUPPORTED, "the learned path supports qq <= %u", kBatchMaxQ);
  const float *mlp = nullptr;
  float margin = 0.0f;
  if (learned) {
    std::lock_guard<std::mutex> lk(h->learned_mu);
    if (!h->mlp || h->mlp_part_version != h->part_version || h->part_version != h->data_version)
      return fail(TOPK_ERR_STATE, "no learned model for the current partitions");
    mlp = h->mlp;
    margin = h->mlp_margin;
  }
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  CtxLease lease(h);
  if (lease.status != TOPK_OK) return lease.status;
  Ctx *c = lease.c;
  const uint32_t P = h->num_parts;
  cudaStream_t s = c->stream;
  if (c->plist_cap < P) {
    cudaFree(c->d_plist);
    cudaFree(c->d_pkey);
    cudaFree(c->d_ptemp);
    c->d_plist = c->d_pkey = nullptr;
    c->d_ptemp = nullptr;
    c->plist_cap = 0;
    c->ptemp_bytes = part_order_temp_bytes(P);
    CK(cudaMalloc(&c->d_plist, (size_t)P * 4));
    CK(cudaMalloc(&c->d_pkey, (size_t)P * 4));
    if (c->ptemp_bytes) CK(cudaMalloc(&c->d_ptemp, c->ptemp_bytes));
    c->plist_cap = P;
  }
  // device-side words (round 1's bound) in the device block; the result and the cut
  // the host reads go straight to the mapped block
  ResultHeader *dh = reinterpret_cast<ResultHeader *>(c->d_res);
  unsigned char *dro = c->d_out;
  ResultHeader *dho = reinterpret_cast<ResultHeader *>(dro);
  uint64_t *d_ids = reinterpret_cast<uint64_t *>(dro + kHdr);
  float *d_scores = reinterpret_cast<float *>(dro + kHdr + kk * 8);
  volatile ResultHeader *hh = reinterpret_cast<volatile ResultHeader *>(c->h_out);
  const uint32_t *d_seed = nullptr;
  if (learned) {
    // descriptor | features (kMlpMaxIn) | prediction | seed word
    const size_t qb = (sizeof(BatchQuery) + 15) / 16 * 16;
    if (!c->d_lq) CK(cudaMalloc(&c->d_lq, qb + (kMlpMaxIn + 2) * 4));
    const uint64_t k1 = k;
    const std::vector<BatchQuery> bq = pack_queries(h, 1, &k1, &qq, weights, 0, attr, 0);
    static_assert(sizeof(BatchQuery) <= kStageBytes, "descriptor staging");
    unsigned char *stage = c->h_res + result_bytes(kMaxK);  // pinned, after the result area
    std::memcpy(stage, &bq[0], sizeof(BatchQuery));
    BatchQuery *dq = reinterpret_cast<BatchQuery *>(c->d_lq);
    float *X = reinterpret_cast<float *>(c->d_lq + qb);
    uint32_t *seed = reinterpret_cast<uint32_t *>(X + kMlpMaxIn + 1);
    CK(cudaMemcpyAsync(dq, stage, sizeof(BatchQuery), cudaMemcpyHostToDevice, s));
    const size_t Pd = (size_t)P * h->d;
    CK(launch_features(h->pstats, h->pstats + Pd, h->pstats + 2 * Pd, P, h->d, dq, 1, X, mlp, X + kMlpMaxIn, s,
                       margin, seed, &dho->cut));
    d_seed = seed;
  }
  PartQuery pq{};
  pq.qq = qq;
  for (uint32_t m = 0; m < qq; m++) {
    pq.attr[m] = attr[m];
    pq.w[m] = weights[attr[m]];
  }
  CK(launch_part_order(h->pstats, h->pstats + (size_t)P * h->d, P, h->d, pq, c->d_plist, c->d_pkey, c->d_ptemp,
                       c->ptemp_bytes, h->num_sms, s));
  const uint32_t seed_host = std::isfinite(cut) ? host_f2key(cut) : 0u;
  const bool seeded = learned || seed_host != 0u;
  const uint64_t tiles_per_part = (1ull << h->part_log2) / 1024u;
  // round 1: about one wave of CTAs worth of the best partitions, and rows for k
  const uint64_t R = 1ull << h->part_log2;
  // A pruned scan reads a small part of the table: a few CTAs per SM keep enough loads
  // in flight for it, and fewer CTAs mean a shallower merge tree (kPrunedCtasPerSm).
  // Round 1 takes the best 1/32 of the partitions (and rows for k).
  const uint32_t m1 = (uint32_t)std::min<uint64_t>(P, std::max<uint64_t>((kk + R - 1) / R + 1, (P + 31) / 32));
  uint32_t *d_t1 = reinterpret_cast<uint32_t *>(&dh->pad[0]);  // round 1's k-th key
  uint64_t tiles = 0, scans = 0, accepted = 0;
  float cut_seen = cut;
  // the seeded attempt (if any), then the two rounds without a seed
  for (int attempt = seeded ? 0 : 1; attempt < 2; attempt++) {
    hh->count = 0xFFFFFFFFu;  // sentinel: a completed scan writes its count
    if (attempt == 0) {
      PartScan ps{c->d_plist, P, seed_host, c->d_pkey, d_seed, nullptr, kPrunedCtasPerSm, false};
      st = enqueue_scan(h, c, s, 0, h->n, k, qq, weights, attr, d_ids, d_scores, &dho->threshold, &dho->count,
                        dho->stats, &ps);
      scans += 1;
    } else {
      // round 1: a threshold pass (no merge, no result) over its partitions
      PartScan p1{c->d_plist, m1, 0u, nullptr, nullptr, d_t1, kRound1CtasPerSm, true};
      st = enqueue_scan(h, c, s, 0, h->n, k, qq, weights, attr, d_ids, d_scores, &dho->threshold, &dho->count,
                        nullptr, &p1);
      if (st != TOPK_OK) return st;
      PartScan p2{c->d_plist, P, 0u, c->d_pkey, d_t1, nullptr, kPrunedCtasPerSm, false};
      st = enqueue_scan(h, c, s, 0, h->n, k, qq, weights, attr, d_ids, d_scores, &dho->threshold, &dho->count,
                        dho->stats, &p2);
      scans += 2;
    }
    if (st != TOPK_OK) return st;
    CK(cudaStreamSynchronize(s));
    if (hh->count > kk) {
      ScanScratch sc{};
      cudaMemcpy(&sc, c->scratch, sizeof(sc), cudaMemcpyDeviceToHost);
      cudaMemset(c->scratch, 0, c->meta_bytes);
      if (sc.error & 1u) return fail(TOPK_ERR_TIMEOUT, "device wait gave up (limit %llu polls)", (unsigned long long)h->wait_limit);
      return fail(TOPK_ERR_CUDA, "partition scan did not complete (count %u, error 0x%x)", (uint32_t)hh->count,
                  sc.error);
    }
    if (learned && attempt == 0) cut_seen = hh->cut;
    tiles += hh->stats[2] + (attempt == 1 ? (uint64_t)m1 * tiles_per_part : 0u);
    if (attempt == 1) break;
    if (hh->count == kk) {
      accepted = 1;
      break;
    }
  }
  const uint32_t cnt = hh->count;
  std::memcpy(ids, c->h_out + kHdr, (size_t)cnt * 8);
  std::memcpy(scores, c->h_out + kHdr + kk * 8, (size_t)cnt * 4);
  if (count) *count = cnt;
  if (threshold) *threshold = hh->threshold;
  if (cut_out) *cut_out = cut_seen;
  if (stats) {
    stats[0] = (tiles + tiles_per_part - 1) / tiles_per_part;
    stats[1] = P;
    stats[2] = accepted;
    stats[3] = scans;
  }
  g_last_cands = hh->stats[0];
  g_last_reductions = hh->stats[1];
  return TOPK_OK;
}

// Grow a cached device buffer to at least `bytes`.
int ensure(topk_table_s::DevBuf &b, size_t bytes) {
  if (b.bytes >= bytes) return TOPK_OK;
  cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  CK(cudaMalloc(&b.p, bytes));
  b.bytes = bytes;
  return TOPK_OK;
}

void free_batch_buffers(topk_table_t h) {
  for (topk_table_s::DevBuf *b : {&h->b_q, &h->b_st, &h->b_best, &h->b_cand, &h->b_ids, &h->b_scores, &h->b_count,
                                  &h->b_thr, &h->xbf, &h->xbf_absmax, &h->b_abf, &h->b_err, &h->b_log,
                                  &h->b_logh, &h->b_sw, &h->b_feat, &h->b_pred, &h->b_abf_act, &h->b_amap,
                                  &h->b_order}) {
    cudaFree(b->p);
    b->p = nullptr;
    b->bytes = 0;
  }
  if (h->b_ev0) cudaEventDestroy(h->b_ev0);
  if (h->b_ev1) cudaEventDestroy(h->b_ev1);
  h->b_ev0 = h->b_ev1 = nullptr;
  if (h->hb_res) cudaFreeHost(h->hb_res);
  h->hb_res = nullptr;
  h->hb_bytes = 0;
  for (auto &g : h->b_graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = topk_table_s::BatchGraph{};
  }
}

// The device table is about to change: derived copies (the BF16 split) are stale.
void table_changed(topk_table_t h) {
  std::lock_guard<std::mutex> lk(h->batch_mu);
  ++h->data_version;
}

// Largest magnitude the BF16 filter accepts in the table and the weights: products
// and 48-term sums stay far from FP32 overflow, and bf16 rounding cannot overflow.
constexpr float kBf16MaxAbs = 1.152921504606846976e18f;  // 2^60

// Build (or reuse) the BF16 split of the table; caller holds batch_mu.  Sets
// h->xbf_usable: false for tables wider than 16 or holding non-finite or huge values.
int ensure_bf16_table(topk_table_t h, cudaStream_t s) {
  if (h->xbf_version == h->data_version) return TOPK_OK;
  h->xbf_usable = false;
  if (h->d > kBf16MaxD) {
    h->xbf_version = h->data_version;
    return TOPK_OK;
  }
  int st;
  if ((st = ensure(h->xbf, bf16_table_bytes(h->n))) != TOPK_OK) return st;
  if ((st = ensure(h->xbf_absmax, (size_t)h->d * 12)) != TOPK_OK) return st;
  CK(launch_bf16_pack(h->table, h->ld, h->d, h->n, static_cast<uint8_t *>(h->xbf.p),
                      static_cast<uint32_t *>(h->xbf_absmax.p), h->num_sms, s));
  std::vector<uint32_t> bits(3 * (size_t)h->d);
  CK(cudaMemcpyAsync(bits.data(), h->xbf_absmax.p, bits.size() * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  h->absmax.assign(h->d, 0.0f);
  h->colmax.assign(h->d, 0.0f);
  h->colmin.assign(h->d, 0.0f);
  bool usable = true;
  for (uint32_t m = 0; m < h->d; m++) {
    float f;
    std::memcpy(&f, &bits[m], 4);
    if (!(f <= kBf16MaxAbs)) usable = false;  // also NaN / inf
    h->absmax[m] = f;
    h->colmax[m] = host_key2f(bits[h->d + m]);      // NaN when the column holds no number
    h->colmin[m] = host_key2f(bits[2 * h->d + m]);
  }
  h->xbf_usable = usable;
  h->xbf_version = h->data_version;
  return TOPK_OK;
}

// Key of an upper bound of every reference-order FP32 score of query b over the table:
// the same sum, in the same order, over the column extremes (the max where the weight
// is >= 0, the min where it is negative).  IEEE multiplication and addition round
// monotonically, so no row's score exceeds it.  0xFFFFFFFF (no bound) when the sum is
// NaN (an all-NaN column, or inf times a zero weight).
uint32_t score_bound_key(const BatchQuery &b, const std::vector<float> &cmax, const std::vector<float> &cmin) {
  float s = 0.0f;
  for (uint32_t m = 0; m < b.qq; m++) {
    const float w = b.w[m];
    const float x = w >= 0.0f ? cmax[b.attr[m]] : cmin[b.attr[m]];
    const float prod = x * w;
    s = s + prod;
  }
  if (s != s) return 0xFFFFFFFFu;
  return host_f2key(s);
}

// Per-query bound of the BF16 filter, rounded up to a float:
// 2^-13 * sum_m |w_m| * absmax[attr_m] + 2^-100 * sum_m (|w_m| + absmax[attr_m]).
// Summed in FP32: each sum of at most 32 nonnegative terms is within 33 * 2^-24 of
// its exact value, so scaling by 1 + 2^-16 and rounding up keeps an upper bound.
float bf16_error_bound(const BatchQuery &b, const std::vector<float> &absmax) {
  float rel = 0.0f, tiny = 0.0f;
  for (uint32_t m = 0; m < b.qq; m++) {
    rel += std::fabs(b.w[m]) * absmax[b.attr[m]];
    tiny += std::fabs(b.w[m]) + absmax[b.attr[m]];
  }
  const float e = std::ldexp(rel, -13) * (1.0f + 0x1p-16f) + std::ldexp(tiny, -100) * (1.0f + 0x1p-16f);
  return std::nextafter(e, INFINITY);
}

// Chunks of a batch whose served query counts are recorded (a 2^32-row table needs 20).
constexpr uint32_t kMaxChunkLog = 64;

// Batched exact top-k on the handle's primary stream (caller holds batch_mu):
// bootstrap over the first rows, doubling chunks (score + reduce), finish.  Queries
// flagged for a candidate overflow are answered again by the single-query scan.
// With the learned start, each query's threshold begins at its predicted cut
// instead (no bootstrap); a query left with fewer than k objects at or above its
// cut is answered again by a batch without the learned start.
int run_batch(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs, const float *weights,
              uint64_t wstride, const uint8_t *attrs, uint64_t astride, uint64_t *ids, float *scores,
              uint64_t kstride, uint64_t *counts, float *thresholds, bool allow_learned = true,
              bool force_fp32 = false) {
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::vector<BatchQuery> q(nq);
  uint64_t best_total = 0, cand_total = 0;
  uint32_t kmax = 1, capmax = 1, qmax = 1;
  for (uint64_t j = 0; j < nq; j++) {
    BatchQuery &b = q[j];
    std::memset(&b, 0, sizeof(b));
    b.k = (uint32_t)std::min<uint64_t>(ks[j], h->n);
    b.qq = qqs[j];
    b.best_off = (uint32_t)best_total;
    best_total += b.k;
    b.cand_cap = 4 * b.k + 4096;
    b.cand_off = (uint32_t)cand_total;
    cand_total += b.cand_cap;
    for (uint32_t m = 0; m < b.qq; m++) {
      b.attr[m] = attrs[j * astride + m];
      b.w[m] = weights[j * wstride + b.attr[m]];
    }
    b.maxkey = 0xFFFFFFFFu;
    kmax = std::max(kmax, b.k);
    capmax = std::max(capmax, b.cand_cap);
    qmax = std::max(qmax, b.qq);
  }
  if (best_total > 0xFFFFFFFFull || cand_total > 0xFFFFFFFFull)
    return fail(TOPK_ERR_UNSUPPORTED, "batch too large: split it");
  int st;
  cudaStream_t s = h->primary->stream;
  // scorer: the BF16 tensor-core filter where the table and every weight allow it
  bool use_bf16 = false;
  if (!force_fp32 && (h->batch_method == TOPK_BATCH_AUTO || h->batch_method == TOPK_BATCH_BF16 ||
                      h->batch_method == TOPK_BATCH_LEARNED)) {
    if ((st = ensure_bf16_table(h, s)) != TOPK_OK) return st;
    use_bf16 = h->xbf_usable && nq <= 0xFFFFFFFFull;
    // AUTO: scores too dense around the thresholds for the filter on this table
    if (h->batch_method == TOPK_BATCH_AUTO && h->auto_fp32_version == h->data_version) use_bf16 = false;
    for (uint64_t j = 0; use_bf16 && j < nq; j++)
      for (uint32_t m = 0; m < q[j].qq; m++)
        if (!(std::fabs(q[j].w[m]) <= kBf16MaxAbs)) use_bf16 = false;
  }
  // learned start: a model fitted on the current partitions
  bool use_learned = false;
  if (allow_learned && (h->batch_method == TOPK_BATCH_AUTO || h->batch_method == TOPK_BATCH_LEARNED)) {
    std::lock_guard<std::mutex> lk(h->learned_mu);
    use_learned = h->mlp && h->mlp_part_version == h->part_version && h->part_version == h->data_version &&
                  feature_dim(h->d) <= kMlpMaxIn && h->num_parts <= kMaxFeatureParts && nq <= 0x7FFFFFFFull;
  }
  h->last_batch_method = use_learned ? TOPK_BATCH_LEARNED : use_bf16 ? TOPK_BATCH_BF16 : TOPK_BATCH_FP32;
  const uint32_t nqq_all = (uint32_t)nq;
  uint64_t log_ctas = 0;
  if (use_bf16) {
    std::vector<uint8_t> habf(bf16_query_bytes((uint32_t)nq), 0);
    for (uint64_t j = 0; j < nq; j++) {
      // a[m] = the sum of the weights on attribute m (repeated attributes add up; FP32,
      // within 2^-19 of the exact sum for <= 32 terms, well inside the filter's bound)
      float a[kBf16MaxD] = {0.0f};
      for (uint32_t m = 0; m < q[j].qq; m++) a[q[j].attr[m]] += q[j].w[m];
      bf16_pack_query(a, (uint32_t)j, habf.data());
      q[j].err = bf16_error_bound(q[j], h->absmax);
      q[j].maxkey = score_bound_key(q[j], h->colmax, h->colmin);
    }
    if ((st = ensure(h->b_abf, habf.size())) != TOPK_OK) return st;
    if ((st = ensure(h->b_abf_act, habf.size())) != TOPK_OK) return st;
    if ((st = ensure(h->b_amap, (nq + 1 + kMaxChunkLog) * sizeof(uint32_t))) != TOPK_OK) return st;
    if ((st = ensure(h->b_err, sizeof(uint32_t))) != TOPK_OK) return st;
    // survivor records: one log per filter CTA
    const FilterPlan fp = plan_bf16_filter(nqq_all, 0, h->n, h->num_sms, h->batch_qt);
    log_ctas = fp.grid;
    if ((st = ensure(h->b_log, log_ctas * kBf16LogCap * 8 * sizeof(uint4))) != TOPK_OK) return st;
    if ((st = ensure(h->b_logh, log_ctas * kBf16LogCap * sizeof(uint2))) != TOPK_OK) return st;
    CK(cudaMemcpyAsync(h->b_abf.p, habf.data(), habf.size(), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(h->b_err.p, 0, sizeof(uint32_t), s));
    CK(cudaStreamSynchronize(s));  // habf is pageable and goes out of scope
  }
  if ((st = ensure(h->b_q, nq * sizeof(BatchQuery))) != TOPK_OK) return st;
  if ((st = ensure(h->b_st, nq * sizeof(BatchState))) != TOPK_OK) return st;
  if ((st = ensure(h->b_best, best_total * sizeof(uint2))) != TOPK_OK) return st;
  if ((st = ensure(h->b_cand, cand_total * sizeof(uint2))) != TOPK_OK) return st;
  if ((st = ensure(h->b_ids, nq * kmax * sizeof(uint64_t))) != TOPK_OK) return st;
  if ((st = ensure(h->b_scores, nq * kmax * sizeof(float))) != TOPK_OK) return st;
  if ((st = ensure(h->b_count, nq * sizeof(uint32_t))) != TOPK_OK) return st;
  if ((st = ensure(h->b_thr, nq * sizeof(float))) != TOPK_OK) return st;
  if (!h->b_ev0) CK(cudaEventCreate(&h->b_ev0));
  if (!h->b_ev1) CK(cudaEventCreate(&h->b_ev1));
  // the plain FP32 scorer takes the queries ordered by attribute count, then by
  // attribute list: a warp's lanes then run the same number of steps and mostly read
  // the same rows of the staged tile at each step (shared-memory broadcast)
  uint32_t *dorder = nullptr;
  if (!use_bf16) {
    std::vector<uint32_t> order(nq);
    for (uint32_t j = 0; j < (uint32_t)nq; j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
      if (q[a].qq != q[b].qq) return q[a].qq < q[b].qq;
      return std::memcmp(q[a].attr, q[b].attr, q[a].qq) < 0;
    });
    if ((st = ensure(h->b_order, nq * sizeof(uint32_t))) != TOPK_OK) return st;
    dorder = static_cast<uint32_t *>(h->b_order.p);
    CK(cudaMemcpyAsync(dorder, order.data(), nq * 4, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));  // `order` is pageable and goes out of scope
  }
  BatchQuery *dq = static_cast<BatchQuery *>(h->b_q.p);
  BatchState *dst = static_cast<BatchState *>(h->b_st.p);
  uint2 *dbest = static_cast<uint2 *>(h->b_best.p);
  uint2 *dcand = static_cast<uint2 *>(h->b_cand.p);
  const uint32_t nqq = (uint32_t)nq;
  CK(cudaMemcpyAsync(dq, q.data(), nq * sizeof(BatchQuery), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(dst, 0, nq * sizeof(BatchState), s));
  if (use_learned) {
    if ((st = ensure(h->b_feat, nq * feature_dim(h->d) * sizeof(float))) != TOPK_OK) return st;
    if ((st = ensure(h->b_pred, nq * sizeof(float))) != TOPK_OK) return st;
  }
  const uint64_t boot = std::min<uint64_t>(h->n, h->batch_boot);
  const uint64_t r_start = use_learned ? 0 : boot;
  // Hybrid batch under the filter: a query for which the filter passes too much
  // (scores tied or dense at its threshold) moves to the exact FP32 scorer for the
  // rest of the batch.  The reduce lists it: sw[0] counts the moved queries (list A at
  // sw + 2), sw[1] those whose last chunk was discarded (list B at sw + 2 + nq), and
  // sw[2 + 2nq] is how far list B has been answered again, sw[3 + 2nq] the scorer's
  // work counter.  The scorer reads the counts on the device, so the host never waits
  // inside the batch.
  uint32_t *dsw = nullptr, *dredo = nullptr, *dwork = nullptr;
  if (use_bf16) {
    if ((st = ensure(h->b_sw, (4 + 2 * nq) * sizeof(uint32_t))) != TOPK_OK) return st;
    dsw = static_cast<uint32_t *>(h->b_sw.p);
    dredo = dsw + 2 + 2 * nq;
    dwork = dredo + 1;
    CK(cudaMemsetAsync(dsw, 0, 2 * sizeof(uint32_t), s));
    CK(cudaMemsetAsync(dredo, 0, sizeof(uint32_t), s));
  }
  uint32_t hsw[2] = {0, 0};
  uint32_t chunk = 0;  // chunk index while the launches are issued
  // the device work of the batch, from the first threshold to the results
  auto issue = [&]() -> int {
  chunk = 0;
  if (use_learned) {
    // features and the model in one kernel, then each query's threshold starts at
    // its cut (prediction - margin) * S; no bootstrap
    std::lock_guard<std::mutex> lk(h->learned_mu);
    const size_t P = h->num_parts, d = h->d;
    CK(launch_features(h->pstats, h->pstats + P * d, h->pstats + 2 * P * d, h->num_parts, h->d, dq, nqq,
                       static_cast<float *>(h->b_feat.p), h->mlp, static_cast<float *>(h->b_pred.p), s));
    CK(launch_learned_seed(static_cast<const float *>(h->b_pred.p), static_cast<const float *>(h->b_feat.p), h->d, dq,
                           h->mlp_margin, dst, nqq, s));
  } else {
    CK(launch_batch_bootstrap(h->table, h->ld, (uint32_t)boot, kmax, dq, nqq, dst, dbest, s));
  }
  uint64_t prev_r = r_start;
  // chunk boundaries stay multiples of 256 rows (the filter's object tiles)
  for (uint64_t r = r_start, size = h->batch_boot; r < h->n; size *= 2) {
    const uint64_t e = std::min<uint64_t>(h->n, r + size);
    if (use_bf16) {
      const FilterPlan fp = plan_bf16_filter(nqq, r, e, h->num_sms, h->batch_qt);
      if (fp.grid > log_ctas) return fail(TOPK_ERR_STATE, "filter grid %llu above its logs", (unsigned long long)fp.grid);
      // the queries still served by the filter, as compact tiles
      uint32_t *amap = static_cast<uint32_t *>(h->b_amap.p);
      // the chunk's active count also goes to its slot of the per-batch record
      uint32_t *logslot = chunk < kMaxChunkLog ? amap + nq + 1 + chunk : nullptr;
      ++chunk;
      CK(launch_batch_active(dq, dst, nqq, static_cast<const uint8_t *>(h->b_abf.p),
                             static_cast<uint8_t *>(h->b_abf_act.p), amap, amap + nq, logslot, s));
      CK(launch_bf16_filter(fp, static_cast<const uint8_t *>(h->xbf.p), static_cast<const uint8_t *>(h->b_abf_act.p),
                            amap, amap + nq, r, e, dq, dst, dcand, static_cast<uint4 *>(h->b_log.p),
                            static_cast<uint2 *>(h->b_logh.p), kBf16LogCap, h->wait_limit,
                            static_cast<uint32_t *>(h->b_err.p), s));
      // this chunk for every moved query; the previous one again for those that discarded it
      CK(launch_batch_score_fp32_list(h->table, h->ld, h->d, r, e, dq, dst, dcand, dsw + 2, dsw, nullptr, dwork, qmax,
                                      true, h->num_sms, s));
      CK(launch_batch_score_fp32_list(h->table, h->ld, h->d, prev_r, r, dq, dst, dcand, dsw + 2 + nq, dsw + 1,
                                      dredo, dwork, qmax, true, h->num_sms, s));
      CK(launch_copy_word(dredo, dsw + 1, s));
    } else {
      CK(launch_batch_score_fp32(h->table, h->ld, h->d, r, e, dq, nqq, dst, dcand, dorder, qmax, false, s));
    }
    CK(launch_batch_reduce(h->table, h->ld, dq, nqq, dst, dbest, dcand, kmax, capmax, use_bf16, dsw, s));
    prev_r = r;
    r = e;
  }
  if (use_bf16) {  // the last chunk again for the queries that discarded it (none: two empty launches)
    CK(launch_batch_score_fp32_list(h->table, h->ld, h->d, prev_r, h->n, dq, dst, dcand, dsw + 2 + nq, dsw + 1,
                                    dredo, dwork, qmax, true, h->num_sms, s));
    CK(launch_batch_reduce(h->table, h->ld, dq, nqq, dst, dbest, dcand, kmax, capmax, use_bf16, dsw, s));
  }
  // results compact (each query's at its best_off), so the download moves sum(k) entries
  CK(launch_batch_finish(dq, nqq, dst, dbest, kmax, static_cast<uint64_t *>(h->b_ids.p),
                         static_cast<float *>(h->b_scores.p), 0, static_cast<uint32_t *>(h->b_count.p),
                         static_cast<float *>(h->b_thr.p), s));
  return TOPK_OK;
  };
  // Captured into a CUDA graph once per shape and replayed: the key holds every
  // pointer and scalar the captured launches take (a buffer that grew or a new model
  // margin makes a new shape).  The graph reads the query descriptors and states that
  // the stream uploaded and cleared before it.
  std::vector<uint64_t> key = {nq, kmax, capmax, qmax, use_bf16, use_learned, h->n, h->d, h->ld, boot,
                               (uint64_t)h->num_sms, log_ctas, h->wait_limit, h->num_parts, h->batch_qt};
  const void *key_ptrs[] = {h->table, dq, dst, dbest, dcand, h->b_ids.p, h->b_scores.p, h->b_count.p,
                            h->b_thr.p, h->xbf.p, h->b_abf.p, h->b_log.p, h->b_logh.p, h->b_err.p, h->b_sw.p,
                            h->b_feat.p, h->b_pred.p, h->pstats, h->mlp, h->b_abf_act.p, h->b_amap.p, dorder};
  for (const void *ptr : key_ptrs) key.push_back((uint64_t)(uintptr_t)ptr);
  {
    uint32_t mb;
    std::memcpy(&mb, &h->mlp_margin, 4);
    key.push_back(use_learned ? mb : 0u);
  }
  topk_table_s::BatchGraph *gr = nullptr;
  for (auto &g : h->b_graphs)
    if (g.exec && g.key == key) gr = &g;
  if (!gr) {  // capture into the least recently used slot
    gr = &h->b_graphs[0];
    for (auto &g : h->b_graphs)
      if (g.used < gr->used) gr = &g;
    if (gr->exec) cudaGraphExecDestroy(gr->exec);
    *gr = topk_table_s::BatchGraph{};
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    const int ist = issue();
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ist != TOPK_OK) {
      if (graph) cudaGraphDestroy(graph);
      return ist;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&gr->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      gr->exec = nullptr;
      return cuda_fail(ie, "cudaGraphInstantiate");
    }
    gr->key = key;
  }
  gr->used = ++h->b_graph_tick;
  CK(cudaEventRecord(h->b_ev0, s));
  CK(cudaGraphLaunch(gr->exec, s));
  CK(cudaEventRecord(h->b_ev1, s));
  // results through the handle's pinned buffers (grown once), then into the caller's
  // arrays before anything below runs a nested batch that reuses them
  const size_t res_bytes = (size_t)best_total * 12;
  if (h->hb_bytes < res_bytes) {
    if (h->hb_res) cudaFreeHost(h->hb_res);
    h->hb_res = nullptr;
    h->hb_bytes = 0;
    if (cudaHostAlloc(&h->hb_res, res_bytes, cudaHostAllocDefault) != cudaSuccess)
      return fail(TOPK_ERR_OOM, "pinned result buffer of %zu bytes", res_bytes);
    h->hb_bytes = res_bytes;
  }
  uint64_t *hid = static_cast<uint64_t *>(h->hb_res);
  float *hsc = reinterpret_cast<float *>(hid + best_total);
  std::vector<float> hth(nq);
  std::vector<uint32_t> hcnt(nq);
  std::vector<BatchState> hst(nq);
  CK(cudaMemcpyAsync(hid, h->b_ids.p, best_total * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hsc, h->b_scores.p, best_total * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hcnt.data(), h->b_count.p, nq * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hth.data(), h->b_thr.p, nq * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hst.data(), dst, nq * sizeof(BatchState), cudaMemcpyDeviceToHost, s));
  uint32_t herr = 0;
  std::vector<uint32_t> hact(kMaxChunkLog, 0);
  if (use_bf16) CK(cudaMemcpyAsync(&herr, h->b_err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (use_bf16)
    CK(cudaMemcpyAsync(hact.data(), static_cast<uint32_t *>(h->b_amap.p) + nq + 1, kMaxChunkLog * 4,
                       cudaMemcpyDeviceToHost, s));
  if (use_bf16) CK(cudaMemcpyAsync(hsw, dsw, sizeof(hsw), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (herr) return fail(TOPK_ERR_TIMEOUT, "BF16 filter: a bounded device-side wait ran out");
  // MMA work of the filter: every served query tile (128 queries) against every object
  // tile of the chunk, three passes of 2 * 16 flops per (query, object)
  double filter_flops = 0;
  if (use_bf16) {
    uint32_t c = 0;  // the chunks as issued (the graph replays the same sequence)
    for (uint64_t r = r_start, size = h->batch_boot; r < h->n && c < kMaxChunkLog; size *= 2, ++c) {
      const uint64_t e = std::min<uint64_t>(h->n, r + size);
      filter_flops += (double)((hact[c] + 127) / 128 * 128) * (double)((e - r + 255) / 256 * 256) * 96.0;
      r = e;
    }
  }
  uint64_t switched_total = hsw[0], retired_total = 0;
  if (use_bf16)
    for (uint64_t j = 0; j < nq; j++)
      if (!(hst[j].flags & kFlagFp32) && hst[j].thr != 0u && hst[j].thr > q[j].maxkey) ++retired_total;
  for (uint64_t j = 0; j < nq; j++) {  // queries answered again below overwrite theirs
    const uint32_t c = std::min<uint32_t>(hcnt[j], (uint32_t)std::min<uint64_t>(kmax, kstride));
    std::memcpy(ids + j * kstride, hid + q[j].best_off, (size_t)c * 8);
    std::memcpy(scores + j * kstride, hsc + q[j].best_off, (size_t)c * 4);
  }
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->b_ev0, h->b_ev1));
  uint64_t cands = 0;
  double err_ratio = 0;
  for (uint64_t j = 0; j < nq; j++) {
    cands += hst[j].cands;
    float r;
    std::memcpy(&r, &hst[j].errmax, 4);
    err_ratio = std::max(err_ratio, (double)r);
  }
  // Queries answered again by a smaller batch, whose results replace this batch's:
  // a learned start that was too high (fewer than k objects reached the cut) runs
  // again without the learned start.  What overflows under the FP32 scorer is
  // answered by the single-query scan.
  double ms_total = ms;
  uint64_t cands_total = cands, misses_total = 0, scans = 0;
  double ratio_total = err_ratio;
  auto rerun = [&](const std::vector<uint64_t> &sub, bool learned, bool fp32) -> int {
    const uint64_t nm = sub.size();
    std::vector<uint64_t> mk(nm), mcnt(nm), mids(nm * kmax);
    std::vector<uint32_t> mqq(nm);
    std::vector<float> mw(nm * wstride), mth(nm), msc(nm * kmax);
    std::vector<uint8_t> ma(nm * astride);
    for (uint64_t i = 0; i < nm; i++) {
      const uint64_t j = sub[i];
      mk[i] = ks[j];
      mqq[i] = qqs[j];
      std::memcpy(&mw[i * wstride], weights + j * wstride, wstride * 4);
      std::memcpy(&ma[i * astride], attrs + j * astride, astride);
    }
    const int r = run_batch(h, nm, mk.data(), mqq.data(), mw.data(), wstride, ma.data(), astride, mids.data(),
                            msc.data(), kmax, mcnt.data(), mth.data(), learned, fp32);
    if (r != TOPK_OK) return r;
    for (uint64_t i = 0; i < nm; i++) {
      const uint64_t j = sub[i];
      hcnt[j] = (uint32_t)mcnt[i];
      hth[j] = mth[i];
      std::memcpy(ids + j * kstride, &mids[i * kmax], mcnt[i] * 8);
      std::memcpy(scores + j * kstride, &msc[i * kmax], mcnt[i] * 4);
      hst[j].flags = 0;
    }
    ms_total += h->last_batch_ms;
    cands_total += h->last_batch_cands;
    ratio_total = std::max(ratio_total, h->last_batch_err_ratio);
    misses_total += h->last_batch_learned_misses;
    scans += h->last_batch_fallbacks;
    switched_total += h->last_batch_switched;
    retired_total += h->last_batch_retired;
    filter_flops += h->last_batch_filter_flops;
    return TOPK_OK;
  };
  std::vector<uint64_t> sub;
  if (use_learned) {
    // too high a start (fewer than k objects reached it), or so low a one that even
    // the exact scorer's candidate region overflowed: again without it
    for (uint64_t j = 0; j < nq; j++)
      if ((hst[j].flags & kFlagOverflow) || hcnt[j] < q[j].k) sub.push_back(j);
    misses_total += sub.size();
    if (!sub.empty() && (st = rerun(sub, false, force_fp32)) != TOPK_OK) return st;
  }
  // AUTO remembers a table on which the filter handed most queries to the FP32 scorer
  if (use_bf16 && h->batch_method == TOPK_BATCH_AUTO && 4 * (uint64_t)hsw[0] > 3 * nq)
    h->auto_fp32_version = h->data_version;
  for (uint64_t j = 0; j < nq; j++) {
    if (hst[j].flags & 1u) {  // a candidate region overflowed under FP32: answer exactly with the scan
      ++scans;
      uint64_t c = 0;
      float th = 0;
      st = run_query_sync(h, 0, h->n, ks[j], qqs[j], weights + j * wstride, attrs + j * astride, ids + j * kstride,
                          scores + j * kstride, &c, &th);
      if (st != TOPK_OK) return st;
      if (counts) counts[j] = c;
      if (thresholds) thresholds[j] = th;
      continue;
    }
    if (counts) counts[j] = hcnt[j];
    if (thresholds) thresholds[j] = hth[j];
  }
  h->last_batch_ms = ms_total;
  h->last_batch_cands = cands_total;
  h->last_batch_err_ratio = ratio_total;
  h->last_batch_learned_misses = misses_total;
  h->last_batch_fallbacks = scans;
  h->last_batch_switched = switched_total;
  h->last_batch_retired = retired_total;
  h->last_batch_filter_flops = filter_flops;
  h->last_batch_method = use_learned ? TOPK_BATCH_LEARNED : use_bf16 ? TOPK_BATCH_BF16 : TOPK_BATCH_FP32;
  return TOPK_OK;
}

}  // namespace

extern "C" {

const char *topk_version(void) { return "topk_b200 0.1 (sm_100a)"; }

const char *topk_last_error(void) { return g_last_error.c_str(); }

const char *topk_status_name(int s) {
  switch (s) {
    case TOPK_OK: return "TOPK_OK";
    case TOPK_ERR_ARG: return "TOPK_ERR_ARG";
    case TOPK_ERR_CUDA: return "TOPK_ERR_CUDA";
    case TOPK_ERR_OOM: return "TOPK_ERR_OOM";
    case TOPK_ERR_TIMEOUT: return "TOPK_ERR_TIMEOUT";
    case TOPK_ERR_UNSUPPORTED: return "TOPK_ERR_UNSUPPORTED";
    case TOPK_ERR_STATE: return "TOPK_ERR_STATE";
    default: return "TOPK_ERR_UNKNOWN";
  }
}

int topk_create(uint64_t n, uint32_t d, int device, topk_table_t *out) {
  g_last_error.clear();
  if (!out) return fail(TOPK_ERR_ARG, "null output handle");
  *out = nullptr;
  if (n == 0 || d == 0) return fail(TOPK_ERR_ARG, "n and d must be >= 1");
  if (d > TOPK_MAX_D) return fail(TOPK_ERR_ARG, "d=%u exceeds %u", d, TOPK_MAX_D);
  if (n >= 0xFFFFFFFFull) return fail(TOPK_ERR_UNSUPPORTED, "n must be < 2^32 - 1 (32-bit ids on the device)");
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(TOPK_ERR_ARG, "device %d not present (%d devices)", device, ndev);
  DeviceGuard dg(device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  topk_table_t h = new topk_table_s();
  h->device = device;
  h->n = n;
  h->d = d;
  h->ld = (n + kLdAlign - 1) / kLdAlign * kLdAlign;
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  h->num_sms = v > 0 ? v : 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  h->smem_optin = v > 0 ? (size_t)v : 48 * 1024;
  cudaError_t e = scan_set_attributes(h->smem_optin);
  if (e == cudaSuccess) e = cudaMalloc(&h->table, h->ld * d * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(h->table, 0, h->ld * d * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&h->d_minmax, (size_t)d * kMinmaxWords * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&h->d_norm, (size_t)2 * d * sizeof(float));
  if (e != cudaSuccess) {
    cudaFree(h->table);
    cudaFree(h->d_minmax);
    cudaFree(h->d_norm);
    delete h;
    return cuda_fail(e, "topk_create");
  }
  int st = ctx_create(h, &h->primary);
  if (st != TOPK_OK) {
    cudaFree(h->table);
    cudaFree(h->d_minmax);
    cudaFree(h->d_norm);
    delete h;
    return st;
  }
  *out = h;
  return TOPK_OK;
}

int topk_destroy(topk_table_t h) {
  if (!h) return TOPK_OK;
  DeviceGuard dg(h->device);
  for (Ctx *c : h->ctxs) ctx_free(c);
  ctx_free(h->primary);
  free_batch_buffers(h);
  cudaFree(h->mlp);
  cudaFree(h->lq_query);
  cudaFree(h->lq_out);
  cudaFree(h->ptable);
  cudaFree(h->pids);
  cudaFree(h->pstats);
  cudaFree(h->table);
  loader_state_free(h->loader);
  ta_lists_free(h->ta);
  cudaFree(h->d_minmax);
  cudaFree(h->d_norm);
  delete h;
  return TOPK_OK;
}

int topk_shape(topk_table_t h, uint64_t *n, uint32_t *d, uint64_t *ld) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (n) *n = h->n;
  if (d) *d = h->d;
  if (ld) *ld = h->ld;
  return TOPK_OK;
}

int topk_set_wait_limit(topk_table_t h, uint64_t it) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  h->wait_limit = it ? it : (1ull << 26);
  return TOPK_OK;
}

int topk_upload_colmajor(topk_table_t h, const float *host, uint64_t ld_host) {
  if (!h || !host) return fail(TOPK_ERR_ARG, "null argument");
  if (ld_host < h->n) return fail(TOPK_ERR_ARG, "ld_host=%llu < n=%llu", (unsigned long long)ld_host, (unsigned long long)h->n);
  DeviceGuard dg(h->device);
  table_changed(h);
  CK(cudaMemcpy2D(h->table, h->ld * sizeof(float), host, ld_host * sizeof(float), h->n * sizeof(float), h->d,
                  cudaMemcpyHostToDevice));
  h->has_data = true;
  return TOPK_OK;
}

int topk_upload_rowmajor(topk_table_t h, const float *host, uint64_t row_stride) {
  g_last_error.clear();
  if (!h || !host) return fail(TOPK_ERR_ARG, "null argument");
  if (row_stride < h->d) return fail(TOPK_ERR_ARG, "row_stride=%llu < d=%u", (unsigned long long)row_stride, h->d);
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  table_changed(h);
  std::lock_guard<std::mutex> lk(h->loader_mu);
  if (!h->loader) h->loader = loader_state_new();
  std::string msg;
  const int rc = upload_rowmajor_device(h->loader, host, row_stride, h->table, h->ld, h->d, h->n, &msg);
  h->has_data = rc == TOPK_OK;
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_download_rowmajor(topk_table_t h, float *host, uint64_t row_stride) {
  g_last_error.clear();
  if (!h || !host) return fail(TOPK_ERR_ARG, "null argument");
  if (row_stride < h->d) return fail(TOPK_ERR_ARG, "row_stride=%llu < d=%u", (unsigned long long)row_stride, h->d);
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::lock_guard<std::mutex> lk(h->loader_mu);
  if (!h->loader) h->loader = loader_state_new();
  std::string msg;
  const int rc = download_rowmajor_device(h->loader, host, row_stride, h->table, h->ld, h->d, h->n, &msg);
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_skyline_layers(topk_table_t h, uint32_t *layers, uint64_t *num_layers) {
  g_last_error.clear();
  if (!h || !layers || !num_layers) return fail(TOPK_ERR_ARG, "null argument");
  if (!h->has_data) return fail(TOPK_ERR_STATE, "no table data");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::string msg;
  const int rc = skyline_layers_device(h->table, h->ld, h->d, h->n, h->num_sms, layers, num_layers, &msg);
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_build_lists(topk_table_t h) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (!h->has_data) return fail(TOPK_ERR_STATE, "no table data");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::lock_guard<std::mutex> lk(h->ta_mu);
  ta_lists_free(h->ta);
  h->ta = nullptr;
  std::string msg;
  const int rc = ta_lists_build(&h->ta, h->table, h->ld, h->d, h->n, h->num_sms, &msg);
  if (rc != TOPK_OK) return fail(rc, "%s", msg.c_str());
  h->ta_version = h->data_version;
  return TOPK_OK;
}

int topk_read_list(topk_table_t h, uint32_t m, uint32_t *ids, float *values) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (!h->ta || h->ta_version != h->data_version) return fail(TOPK_ERR_STATE, "no sorted lists of the current table");
  if (m >= h->d) return fail(TOPK_ERR_ARG, "attribute %u >= d", m);
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::lock_guard<std::mutex> lk(h->ta_mu);
  std::string msg;
  const int rc = ta_lists_read(h->ta, m, ids, values, &msg);
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_query_ta(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr, uint64_t *ids,
                  float *scores, uint64_t *count, float *threshold, uint64_t *stats) {
  g_last_error.clear();
  int st = check_query(h, k, qq, weights, attr);
  if (st != TOPK_OK) return st;
  if (!ids || !scores) return fail(TOPK_ERR_ARG, "null output buffer");
  if (!h->ta || h->ta_version != h->data_version)
    return fail(TOPK_ERR_STATE, "no sorted lists for the current table: call topk_build_lists");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::lock_guard<std::mutex> lk(h->ta_mu);
  std::string msg;
  const int rc = ta_query(h->ta, h->table, h->ld, k, qq, weights, attr, h->num_sms, ids, scores, count, threshold,
                          stats, &msg);
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_csv_shape(const char *path, uint64_t *n, uint64_t *d) {
  g_last_error.clear();
  if (!path || !n || !d) return fail(TOPK_ERR_ARG, "null argument");
  std::string msg;
  const int rc = csv_shape(path, n, d, &msg);
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_load_csv(topk_table_t h, const char *path, uint64_t chunk_bytes, uint64_t *stats) {
  g_last_error.clear();
  if (!h || !path) return fail(TOPK_ERR_ARG, "null argument");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  table_changed(h);
  std::string msg;
  std::lock_guard<std::mutex> lk(h->loader_mu);
  if (!h->loader) h->loader = loader_state_new();
  const int rc = load_csv_device(h->loader, path, h->table, h->ld, h->d, h->n, h->num_sms, chunk_bytes, stats, &msg);
  h->has_data = rc == TOPK_OK;  // a failed load leaves the table undefined
  return rc == TOPK_OK ? rc : fail(rc, "%s: %s", path, msg.c_str());
}

int topk_save_csv(topk_table_t h, const char *path) {
  g_last_error.clear();
  if (!h || !path) return fail(TOPK_ERR_ARG, "null argument");
  if (!h->has_data) return fail(TOPK_ERR_STATE, "no table data");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::string msg;
  const int rc = save_csv(path, h->table, h->ld, h->d, h->n, &msg);
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_binary_shape(const char *path, uint64_t *n, uint64_t *d) {
  g_last_error.clear();
  if (!path || !n || !d) return fail(TOPK_ERR_ARG, "null argument");
  std::string msg;
  const int rc = binary_shape(path, n, d, &msg);
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_load_binary(topk_table_t h, const char *path) {
  g_last_error.clear();
  if (!h || !path) return fail(TOPK_ERR_ARG, "null argument");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  table_changed(h);
  std::string msg;
  std::lock_guard<std::mutex> lk(h->loader_mu);
  if (!h->loader) h->loader = loader_state_new();
  const int rc = load_binary_device(h->loader, path, h->table, h->ld, h->d, h->n, &msg);
  h->has_data = rc == TOPK_OK;
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_save_binary(topk_table_t h, const char *path) {
  g_last_error.clear();
  if (!h || !path) return fail(TOPK_ERR_ARG, "null argument");
  if (!h->has_data) return fail(TOPK_ERR_STATE, "no table data");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::string msg;
  const int rc = save_binary(path, h->table, h->ld, h->d, h->n, &msg);
  return rc == TOPK_OK ? rc : fail(rc, "%s", msg.c_str());
}

int topk_download_colmajor(topk_table_t h, float *host, uint64_t ld_host) {
  if (!h || !host) return fail(TOPK_ERR_ARG, "null argument");
  if (ld_host < h->n) return fail(TOPK_ERR_ARG, "ld_host < n");
  DeviceGuard dg(h->device);
  CK(cudaMemcpy2D(host, ld_host * sizeof(float), h->table, h->ld * sizeof(float), h->n * sizeof(float), h->d,
                  cudaMemcpyDeviceToHost));
  return TOPK_OK;
}

int topk_generate(topk_table_t h, int dist, uint64_t seed) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (dist < 0 || dist > 3) return fail(TOPK_ERR_ARG, "dist must be 0..3");
  if (h->d > 64) return fail(TOPK_ERR_UNSUPPORTED, "generator supports d <= 64");
  DeviceGuard dg(h->device);
  table_changed(h);
  CK(launch_generate(h->table, h->ld, h->d, h->n, dist, seed, h->primary->stream));
  CK(cudaStreamSynchronize(h->primary->stream));
  h->has_data = true;
  return TOPK_OK;
}

int topk_normalize(topk_table_t h, float *mins, float *maxs) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (!h->has_data) return fail(TOPK_ERR_STATE, "no table data");
  DeviceGuard dg(h->device);
  cudaStream_t s = h->primary->stream;
  CK(launch_minmax(h->table, h->ld, h->d, h->n, h->d_minmax, s));
  std::vector<uint32_t> w((size_t)h->d * kMinmaxWords);
  CK(cudaMemcpyAsync(w.data(), h->d_minmax, w.size() * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::vector<float> host(2 * (size_t)h->d);
  for (uint32_t m = 0; m < h->d; m++) {
    const uint32_t *c = &w[(size_t)m * kMinmaxWords];
    auto k2f = [](uint32_t k) {
      uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
      float f;
      std::memcpy(&f, &u, 4);
      return f;
    };
    float mx = k2f(c[0]);
    float mn = k2f(c[1]);
    if (c[1] == 0x80000000u) {  // minimum is zero: sign of the first zero in the column
      uint64_t pz = (uint64_t)c[2] | ((uint64_t)c[3] << 32);
      uint64_t nz = (uint64_t)c[4] | ((uint64_t)c[5] << 32);
      mn = (nz < pz) ? -0.0f : 0.0f;
    }
    volatile float vmx = mx, vmn = mn;
    float range = vmx - vmn;  // _mm = _max - _min (common/common.h:50)
    host[m] = mn;
    host[h->d + m] = range;
    if (mins) mins[m] = mn;
    if (maxs) maxs[m] = mx;
  }
  CK(cudaMemcpyAsync(h->d_norm, host.data(), host.size() * 4, cudaMemcpyHostToDevice, s));
  table_changed(h);
  CK(launch_normalize(h->table, h->ld, h->d, h->n, h->d_norm, h->d_norm + h->d, s));
  CK(cudaStreamSynchronize(s));
  return TOPK_OK;
}

int topk_query(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr, uint64_t *ids,
               float *scores, uint64_t *count, float *threshold) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  return run_query_sync(h, 0, h->n, k, qq, weights, attr, ids, scores, count, threshold);
}

int topk_query_range(topk_table_t h, uint64_t r0, uint64_t r1, uint64_t k, uint32_t qq, const float *weights,
                     const uint8_t *attr, uint64_t *ids, float *scores, uint64_t *count, float *threshold) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  return run_query_sync(h, r0, r1, k, qq, weights, attr, ids, scores, count, threshold);
}

int topk_query_device(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr,
                      uint64_t *d_ids, float *d_scores, float *d_threshold, void *stream) {
  int st = check_query(h, k, qq, weights, attr);
  if (st != TOPK_OK) return st;
  if (!d_ids || !d_scores) return fail(TOPK_ERR_ARG, "null output buffer");
  DeviceGuard dg(h->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->primary->stream;
  return enqueue_scan(h, h->primary, s, 0, h->n, k, qq, weights, attr, d_ids, d_scores, d_threshold, nullptr);
}

int topk_query_range_device(topk_table_t h, uint64_t row_begin, uint64_t row_end, uint64_t k, uint32_t qq,
                            const float *weights, const uint8_t *attr, uint64_t *d_ids, float *d_scores,
                            float *d_threshold, void *stream) {
  int st = check_query(h, k, qq, weights, attr);
  if (st != TOPK_OK) return st;
  if (row_end > h->n || row_begin >= row_end)
    return fail(TOPK_ERR_ARG, "row range [%llu, %llu) empty or outside [0, %llu)", (unsigned long long)row_begin,
                (unsigned long long)row_end, (unsigned long long)h->n);
  if (!d_ids || !d_scores) return fail(TOPK_ERR_ARG, "null output buffer");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->primary->stream;
  return enqueue_scan(h, h->primary, s, row_begin, row_end, k, qq, weights, attr, d_ids, d_scores, d_threshold,
                      nullptr);
}

int topk_merge_lists(int device, const void *d_lists, uint32_t nlists, uint64_t stride, const uint64_t *counts,
                     const uint64_t *id_base, uint64_t k, uint64_t *d_ids, float *d_scores, float *d_threshold,
                     uint64_t *kept, void *stream) {
  g_last_error.clear();
  if (!d_lists || !counts || !d_ids || !d_scores || !kept) return fail(TOPK_ERR_ARG, "null argument");
  if (nlists == 0 || nlists > kMaxMergeLists)
    return fail(TOPK_ERR_UNSUPPORTED, "nlists=%u: 1 to %u lists", nlists, kMaxMergeLists);
  if (k == 0) return fail(TOPK_ERR_ARG, "k must be >= 1");
  if (k > kMaxK) return fail(TOPK_ERR_UNSUPPORTED, "k=%llu exceeds TOPK_MAX_K=%u", (unsigned long long)k, kMaxK);
  if (stride == 0 || stride > kMaxK) return fail(TOPK_ERR_ARG, "stride must be in [1, %u]", kMaxK);
  if (reinterpret_cast<uintptr_t>(d_lists) % 8 != 0) return fail(TOPK_ERR_ARG, "d_lists must be 8-byte aligned");
  uint32_t c32[kMaxMergeLists], b32[kMaxMergeLists];
  for (uint32_t j = 0; j < nlists; j++) {
    if (counts[j] > stride) return fail(TOPK_ERR_ARG, "counts[%u]=%llu above stride", j, (unsigned long long)counts[j]);
    if (id_base && id_base[j] >= 0xFFFFFFFFull) return fail(TOPK_ERR_UNSUPPORTED, "id_base[%u] must be < 2^32 - 1", j);
    c32[j] = (uint32_t)counts[j];
    b32[j] = id_base ? (uint32_t)id_base[j] : 0u;
  }
  DeviceGuard dg(device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  uint32_t kk = 0;
  CK(launch_merge_lists(static_cast<const unsigned char *>(d_lists), nlists, stride, c32, b32, (uint32_t)k, d_ids,
                        d_scores, d_threshold, &kk, static_cast<cudaStream_t>(stream)));
  *kept = kk;
  return TOPK_OK;
}

int topk_query_batch(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs, const float *weights,
                     uint64_t wstride, const uint8_t *attrs, uint64_t astride, uint64_t *ids, float *scores,
                     uint64_t kstride, uint64_t *counts, float *thresholds) {
  g_last_error.clear();
  if (!h || (nq && (!ks || !qqs || !weights || !attrs || !ids || !scores)))
    return fail(TOPK_ERR_ARG, "null argument");
  if (wstride < h->d) return fail(TOPK_ERR_ARG, "wstride < d");
  bool batchable = h->d <= kBatchMaxD && nq > 0 && nq < 0x7FFFFFFFull;
  for (uint64_t j = 0; j < nq; j++) {
    if (kstride < std::min<uint64_t>(ks[j], h->n)) return fail(TOPK_ERR_ARG, "kstride < k of query %llu", (unsigned long long)j);
    if (qqs[j] > astride) return fail(TOPK_ERR_ARG, "astride < qq of query %llu", (unsigned long long)j);
    int st = check_query(h, ks[j], qqs[j], weights + j * wstride, attrs + j * astride);
    if (st != TOPK_OK) return st;
    if (qqs[j] > kBatchMaxQ) batchable = false;
  }
  std::lock_guard<std::mutex> lk(h->batch_mu);
  if (h->batch_method != TOPK_BATCH_LOOP && batchable)
    return run_batch(h, nq, ks, qqs, weights, wstride, attrs, astride, ids, scores, kstride, counts, thresholds);
  h->last_batch_ms = 0;
  h->last_batch_fallbacks = 0;
  h->last_batch_switched = 0;
  h->last_batch_retired = 0;
  h->last_batch_filter_flops = 0;
  h->last_batch_cands = 0;
  h->last_batch_err_ratio = 0;
  h->last_batch_learned_misses = 0;
  h->last_batch_method = TOPK_BATCH_LOOP;
  for (uint64_t j = 0; j < nq; j++) {
    uint64_t c = 0;
    float th = 0;
    int st = run_query_sync(h, 0, h->n, ks[j], qqs[j], weights + j * wstride, attrs + j * astride, ids + j * kstride,
                            scores + j * kstride, &c, &th);
    if (st != TOPK_OK) return st;
    if (counts) counts[j] = c;
    if (thresholds) thresholds[j] = th;
  }
  return TOPK_OK;
}

int topk_set_batch_tiles(topk_table_t h, uint32_t qt_per_cta, uint32_t boot_rows) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (qt_per_cta > 16) return fail(TOPK_ERR_ARG, "qt_per_cta %u above 16", qt_per_cta);
  if (boot_rows < 256 || boot_rows > kBatchBootMax || boot_rows % 256)
    return fail(TOPK_ERR_ARG, "boot_rows %u: a multiple of 256 in [256, %u]", boot_rows, kBatchBootMax);
  std::lock_guard<std::mutex> lk(h->batch_mu);
  h->batch_qt = qt_per_cta;
  h->batch_boot = boot_rows;
  return TOPK_OK;
}

int topk_get_batch_tiles(topk_table_t h, uint32_t *qt_per_cta, uint32_t *boot_rows) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  std::lock_guard<std::mutex> lk(h->batch_mu);
  if (qt_per_cta) *qt_per_cta = h->batch_qt;
  if (boot_rows) *boot_rows = h->batch_boot;
  return TOPK_OK;
}

int topk_tune_batch(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs, const float *weights,
                    uint64_t wstride, const uint8_t *attrs, uint64_t astride, double *report) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (nq == 0 || !ks) return fail(TOPK_ERR_ARG, "empty query set");
  uint64_t kmax = 1;
  for (uint64_t j = 0; j < nq; j++) kmax = std::max<uint64_t>(kmax, std::min<uint64_t>(ks[j], h->n));
  std::vector<uint64_t> ids(nq * kmax), cnt(nq);
  std::vector<float> sc(nq * kmax), th(nq);
  const uint32_t qts[3] = {4, 8, 0}, boots[2] = {kBatchBootRows, kBatchBootMax};
  double best_ms = -1.0, default_ms = -1.0;
  uint32_t best_qt = 0, best_boot = kBatchBootRows, keep_qt, keep_boot;
  {
    std::lock_guard<std::mutex> lk(h->batch_mu);
    keep_qt = h->batch_qt;
    keep_boot = h->batch_boot;
  }
  auto set = [&](uint32_t qt, uint32_t b) {
    std::lock_guard<std::mutex> lk(h->batch_mu);
    h->batch_qt = qt;
    h->batch_boot = b;
  };
  for (uint32_t b : boots)
    for (uint32_t qt : qts) {
      set(qt, b);
      double ms = 0;
      for (int rep = 0; rep < 2; rep++) {  // the first run captures the batch's graph
        const int st = topk_query_batch(h, nq, ks, qqs, weights, wstride, attrs, astride, ids.data(), sc.data(), kmax,
                                        cnt.data(), th.data());
        if (st != TOPK_OK) {
          set(keep_qt, keep_boot);
          return st;
        }
        if ((topk_last_batch_stats(h, &ms, nullptr, nullptr)) != TOPK_OK) return TOPK_ERR_STATE;
      }
      if (qt == 0 && b == kBatchBootRows) default_ms = ms;
      if (best_ms < 0 || ms < best_ms) {
        best_ms = ms;
        best_qt = qt;
        best_boot = b;
      }
    }
  set(best_qt, best_boot);
  if (report) {
    report[0] = best_qt ? best_qt : 16;
    report[1] = best_boot;
    report[2] = best_ms;
    report[3] = default_ms;
  }
  return TOPK_OK;
}

int topk_set_batch_method(topk_table_t h, int method) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (method < TOPK_BATCH_AUTO || method > TOPK_BATCH_LEARNED)
    return fail(TOPK_ERR_UNSUPPORTED, "batch method %d not available", method);
  std::lock_guard<std::mutex> lk(h->batch_mu);
  h->batch_method = method;
  return TOPK_OK;
}

int topk_last_batch_stats(topk_table_t h, double *device_ms, uint64_t *fallbacks, uint64_t *candidates) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  std::lock_guard<std::mutex> lk(h->batch_mu);
  if (device_ms) *device_ms = h->last_batch_ms;
  if (fallbacks) *fallbacks = h->last_batch_fallbacks;
  if (candidates) *candidates = h->last_batch_cands;
  return TOPK_OK;
}

int topk_last_batch_info(topk_table_t h, int *method, double *max_err_ratio, uint64_t *learned_misses) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  std::lock_guard<std::mutex> lk(h->batch_mu);
  if (method) *method = h->last_batch_method;
  if (max_err_ratio) *max_err_ratio = h->last_batch_err_ratio;
  if (learned_misses) *learned_misses = h->last_batch_learned_misses;
  return TOPK_OK;
}

int topk_last_batch_filter_flops(topk_table_t h, double *flops) {
  if (!h || !flops) return fail(TOPK_ERR_ARG, "null argument");
  *flops = h->last_batch_filter_flops;
  return TOPK_OK;
}

int topk_last_batch_retired(topk_table_t h, uint64_t *retired) {
  if (!h || !retired) return fail(TOPK_ERR_ARG, "null argument");
  *retired = h->last_batch_retired;
  return TOPK_OK;
}

int topk_last_batch_switched(topk_table_t h, uint64_t *switched) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  std::lock_guard<std::mutex> lk(h->batch_mu);
  if (switched) *switched = h->last_batch_switched;
  return TOPK_OK;
}

int topk_build_partitions(topk_table_t h, uint32_t part_rows) {
  return topk_build_partitions_ordered(h, part_rows, TOPK_ORDER_MORTON);
}

int topk_partition_ids(topk_table_t h, uint32_t *ids) {
  g_last_error.clear();
  if (!h || !ids) return fail(TOPK_ERR_ARG, "null argument");
  if (!h->pids || h->part_version != h->data_version) return fail(TOPK_ERR_STATE, "no partitions of the current table");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  CK(cudaMemcpy(ids, h->pids, h->n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return TOPK_OK;
}

int topk_build_partitions_ordered(topk_table_t h, uint32_t part_rows, int order) {
  g_last_error.clear();
  if (order != TOPK_ORDER_MORTON && order != TOPK_ORDER_VTA && order != TOPK_ORDER_PTA &&
      order != TOPK_ORDER_VTA_THREADS && order != TOPK_ORDER_SLA && order != TOPK_ORDER_KD)
    return fail(TOPK_ERR_ARG, "unknown order %d", order);
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (!h->has_data) return fail(TOPK_ERR_STATE, "no table data");
  if (order != TOPK_ORDER_MORTON && h->n > 0x7FFFFFFFull)
    return fail(TOPK_ERR_UNSUPPORTED, "the VTA, PTA, SLA and kd orders need n < 2^31 rows");
  if (order == TOPK_ORDER_PTA && (h->n < 2 || h->d > 32))
    return fail(TOPK_ERR_UNSUPPORTED, "PTA order needs n >= 2 and d <= 32");
  if (order == TOPK_ORDER_SLA && h->d > 32) return fail(TOPK_ERR_UNSUPPORTED, "SLA order needs d <= 32");
  if (part_rows < 1024 || part_rows > (1u << 24) || (part_rows & (part_rows - 1)))
    return fail(TOPK_ERR_ARG, "part_rows must be a power of two in [1024, 2^24]");
  uint32_t lg = 0;
  while ((1u << lg) < part_rows) ++lg;
  const uint64_t P = (h->n + part_rows - 1) / part_rows;
  if (P > (1u << 22)) return fail(TOPK_ERR_UNSUPPORTED, "more than 2^22 partitions");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  cudaStream_t s = h->primary->stream;
  // SLA: the skyline layers first (they are the groups of the order)
  std::vector<uint32_t> sla_layers;
  uint32_t sla_bits = 0;
  if (order == TOPK_ORDER_SLA) {
    sla_layers.resize(h->n);
    uint64_t nl = 0;
    std::string msg;
    const int rc = skyline_layers_device(h->table, h->ld, h->d, h->n, h->num_sms, sla_layers.data(), &nl, &msg);
    if (rc != TOPK_OK) return fail(rc, "%s", msg.c_str());
    while (sla_bits < 31 && (1ull << sla_bits) < nl) ++sla_bits;
  }
  // column extremes: the Morton code quantises each attribute over [min, max]
  CK(launch_minmax(h->table, h->ld, h->d, h->n, h->d_minmax, s));
  std::vector<uint32_t> w((size_t)h->d * kMinmaxWords);
  CK(cudaMemcpyAsync(w.data(), h->d_minmax, w.size() * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  const uint32_t dims = std::min<uint32_t>(h->d, 16u);
  const uint32_t bits = std::max<uint32_t>(1u, 16u / dims);
  std::vector<float> lo_scale(2 * (size_t)h->d, 0.0f);
  for (uint32_t m = 0; m < h->d; m++) {
    auto k2f = [](uint32_t k) {
      uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
      float f;
      std::memcpy(&f, &u, 4);
      return f;
    };
    const float mx = k2f(w[(size_t)m * kMinmaxWords]), mn = k2f(w[(size_t)m * kMinmaxWords + 1]);
    const float range = mx - mn;  // only decides the order of the rows, never a result
    lo_scale[m] = std::isfinite(mn) ? mn : 0.0f;
    lo_scale[h->d + m] = (range > 0.0f && std::isfinite(range)) ? std::ldexp(1.0f, (int)bits) / range : 0.0f;
  }
  // release an older copy first (its memory may be needed)
  cudaFree(h->ptable);
  cudaFree(h->pids);
  cudaFree(h->pstats);
  h->ptable = nullptr;
  h->pids = nullptr;
  h->pstats = nullptr;
  h->num_parts = 0;
  uint16_t *keys = nullptr;
  uint32_t *hist = nullptr;
  float *dls = nullptr;
  auto cleanup = [&]() {
    cudaFree(keys);
    cudaFree(hist);
    cudaFree(dls);
  };
  cudaError_t e = cudaMalloc(&keys, h->n * sizeof(uint16_t));
  if (e == cudaSuccess) e = cudaMalloc(&hist, (1u << 16) * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&dls, lo_scale.size() * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&h->pids, h->n * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&h->ptable, h->ld * h->d * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&h->pstats, 3 * P * h->d * sizeof(float));
  if (e == cudaSuccess) e = cudaMemsetAsync(h->ptable, 0, h->ld * h->d * sizeof(float), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dls, lo_scale.data(), lo_scale.size() * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && order == TOPK_ORDER_MORTON)
    e = launch_partition_build(h->table, h->ld, h->d, h->n, dls, dls + h->d, bits, keys, hist, h->pids, h->ptable,
                               h->num_sms, s);
  if (e == cudaSuccess && order == TOPK_ORDER_KD) {
    uint32_t *work = nullptr;
    void *temp = nullptr;
    size_t temp_bytes = 0;
    e = launch_kd_order(h->table, h->ld, h->d, h->n, lg, h->pids, nullptr, nullptr, &temp_bytes, h->num_sms, s);
    if (e == cudaSuccess) e = cudaMalloc(&work, kd_order_work_words(h->n, h->d, (uint32_t)P) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&temp, std::max<size_t>(temp_bytes, 16));
    if (e == cudaSuccess)
      e = launch_kd_order(h->table, h->ld, h->d, h->n, lg, h->pids, work, temp, &temp_bytes, h->num_sms, s);
    if (e == cudaSuccess) e = launch_gather_rows(h->table, h->ld, h->d, h->n, h->pids, h->ptable, h->num_sms, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // before the scratch goes
    cudaFree(work);
    cudaFree(temp);
  }
  if (e == cudaSuccess && order != TOPK_ORDER_MORTON && order != TOPK_ORDER_KD) {
    const IndexOrder kind = order == TOPK_ORDER_PTA           ? IndexOrder::kPta
                            : order == TOPK_ORDER_VTA_THREADS ? IndexOrder::kVtaThreads
                            : order == TOPK_ORDER_SLA         ? IndexOrder::kGroups
                                                              : IndexOrder::kVta;
    uint32_t *work = nullptr, *groups = nullptr;
    void *temp = nullptr;
    size_t temp_bytes = 0;
    if (kind == IndexOrder::kGroups) {
      e = cudaMalloc(&groups, h->n * sizeof(uint32_t));
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(groups, sla_layers.data(), h->n * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess)
      e = launch_index_order(h->table, h->ld, h->d, h->n, kind, h->pids, nullptr, nullptr, &temp_bytes, h->num_sms, s,
                             groups, sla_bits);
    if (e == cudaSuccess) e = cudaMalloc(&work, index_order_work_words(h->n, kind) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&temp, std::max<size_t>(temp_bytes, 16));
    if (e == cudaSuccess)
      e = launch_index_order(h->table, h->ld, h->d, h->n, kind, h->pids, work, temp, &temp_bytes, h->num_sms, s,
                             groups, sla_bits);
    if (e == cudaSuccess) e = launch_gather_rows(h->table, h->ld, h->d, h->n, h->pids, h->ptable, h->num_sms, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // before the scratch goes
    cudaFree(work);
    cudaFree(temp);
    cudaFree(groups);
  }
  float *pmin = h->pstats, *pmax = h->pstats + P * h->d, *pmean = h->pstats + 2 * P * h->d;
  if (e == cudaSuccess) e = launch_partition_stats(h->ptable, h->ld, h->d, h->n, lg, (uint32_t)P, pmin, pmax, pmean, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cleanup();
  if (e != cudaSuccess) return cuda_fail(e, "topk_build_partitions");
  h->pmin.resize(P * h->d);
  h->pmax.resize(P * h->d);
  h->pmean.resize(P * h->d);
  CK(cudaMemcpy(h->pmin.data(), pmin, P * h->d * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h->pmax.data(), pmax, P * h->d * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h->pmean.data(), pmean, P * h->d * 4, cudaMemcpyDeviceToHost));
  h->part_log2 = lg;
  h->num_parts = (uint32_t)P;
  h->part_version = h->data_version;
  return TOPK_OK;
}

int topk_partition_info(topk_table_t h, uint32_t *num_parts, uint32_t *part_rows, float *mins, float *maxs,
                        float *means) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (!h->ptable || h->part_version != h->data_version)
    return fail(TOPK_ERR_STATE, "no partitions for the current table: call topk_build_partitions");
  const size_t cnt = (size_t)h->num_parts * h->d;
  if (num_parts) *num_parts = h->num_parts;
  if (part_rows) *part_rows = 1u << h->part_log2;
  if (mins) std::memcpy(mins, h->pmin.data(), cnt * 4);
  if (maxs) std::memcpy(maxs, h->pmax.data(), cnt * 4);
  if (means) std::memcpy(means, h->pmean.data(), cnt * 4);
  return TOPK_OK;
}

int topk_query_pruned(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr, float cut,
                      uint64_t *ids, float *scores, uint64_t *count, float *threshold, uint64_t *stats) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  return run_pruned(h, k, qq, weights, attr, cut, false, ids, scores, count, threshold, stats, nullptr);
}

}  // extern "C"

// ---------------------------------------------------------------- learned model
extern "C" uint64_t topk_mlp_param_count(uint32_t in_dim) { return mlp_param_count(in_dim); }

namespace {

// Device buffers of one standalone model call, freed on scope exit.
struct DevScope {
  std::vector<void *> ptrs;
  ~DevScope() {
    for (void *p : ptrs) cudaFree(p);
  }
  template <class T>
  cudaError_t alloc(T **p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes ? bytes : 4);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

int check_mlp_dims(uint32_t in_dim) {
  if (in_dim == 0 || in_dim > kMlpMaxIn) return fail(TOPK_ERR_ARG, "in_dim must be in [1, %u]", kMlpMaxIn);
  return TOPK_OK;
}

uint64_t splitmix(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t gcd64(uint64_t a, uint64_t b) {
  while (b) {
    const uint64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// Pack host queries into BatchQuery records (k clamped to n).
std::vector<BatchQuery> pack_queries(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs,
                                     const float *weights, uint64_t wstride, const uint8_t *attrs, uint64_t astride) {
  std::vector<BatchQuery> q(nq);
  for (uint64_t j = 0; j < nq; j++) {
    BatchQuery &b = q[j];
    std::memset(&b, 0, sizeof(b));
    b.k = (uint32_t)std::min<uint64_t>(ks[j], h->n);
    b.qq = qqs[j];
    for (uint32_t m = 0; m < b.qq; m++) {
      b.attr[m] = attrs[j * astride + m];
      b.w[m] = weights[j * wstride + b.attr[m]];
    }
  }
  return q;
}

float query_scale(const BatchQuery &b) {
  float s = 0.0f;
  for (uint32_t m = 0; m < b.qq; m++) s += std::fabs(b.w[m]);
  return s > 0.0f ? s : 1.0f;
}

// Training target of a query: qq * ln(gap / S), gap = largest bound - k-th score,
// at least 1e-9 S (the largest bound bounds every score, so gap >= 0 up to rounding).
float learned_target(float kth, float b1s, float S, uint32_t qq) {
  const float g = std::max(b1s - kth / S, 1e-9f);
  return (float)qq * std::log(g);
}

int check_features_ready(topk_table_t h) {
  if (!h->ptable || h->part_version != h->data_version)
    return fail(TOPK_ERR_STATE, "no partitions for the current table: call topk_build_partitions");
  if (feature_dim(h->d) > kMlpMaxIn)
    return fail(TOPK_ERR_UNSUPPORTED, "the learned model supports d <= %u", (kMlpMaxIn - 18) / 2);
  if (h->num_parts > kMaxFeatureParts)
    return fail(TOPK_ERR_UNSUPPORTED, "the features support at most %u partitions", kMaxFeatureParts);
  return TOPK_OK;
}

// Features of packed queries on the device: X (device, nq x feature_dim(d)).
int device_features(topk_table_t h, const BatchQuery *dq, uint32_t nq, float *dX, cudaStream_t s) {
  const size_t P = h->num_parts, d = h->d;
  CK(launch_features(h->pstats, h->pstats + P * d, h->pstats + 2 * P * d, h->num_parts, h->d, dq, nq, dX, nullptr,
                     nullptr, s));
  return TOPK_OK;
}

}  // namespace

extern "C" int topk_mlp_grad(int device, uint32_t in_dim, const float *params, const float *X, const float *y, uint32_t batch,
                  float *grad, float *loss) {
  g_last_error.clear();
  int st = check_mlp_dims(in_dim);
  if (st != TOPK_OK) return st;
  if (!params || !X || !y || !grad) return fail(TOPK_ERR_ARG, "null argument");
  if (batch == 0 || batch > 128) return fail(TOPK_ERR_ARG, "batch must be in [1, 128]");
  DeviceGuard dg(device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  const size_t P = mlp_param_count(in_dim);
  DevScope ds;
  float *dp, *dX, *dy, *dg2, *dl;
  CK(ds.alloc(&dp, P * 4));
  CK(ds.alloc(&dX, (size_t)batch * in_dim * 4));
  CK(ds.alloc(&dy, batch * 4));
  CK(ds.alloc(&dg2, P * 4));
  CK(ds.alloc(&dl, 4));
  CK(cudaMemcpy(dp, params, P * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dX, X, (size_t)batch * in_dim * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dy, y, batch * 4, cudaMemcpyHostToDevice));
  CK(launch_mlp_grad(dp, dX, dy, batch, in_dim, dg2, dl, 0));
  CK(cudaMemcpy(grad, dg2, P * 4, cudaMemcpyDeviceToHost));
  float l = 0;
  CK(cudaMemcpy(&l, dl, 4, cudaMemcpyDeviceToHost));
  if (loss) *loss = l;
  return TOPK_OK;
}

extern "C" int topk_mlp_predict(int device, uint32_t in_dim, const float *params, const float *X, uint64_t n, float *out) {
  g_last_error.clear();
  int st = check_mlp_dims(in_dim);
  if (st != TOPK_OK) return st;
  if (!params || (n && (!X || !out))) return fail(TOPK_ERR_ARG, "null argument");
  DeviceGuard dg(device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const size_t P = mlp_param_count(in_dim);
  DevScope ds;
  float *dp, *dX, *dout;
  CK(ds.alloc(&dp, P * 4));
  CK(ds.alloc(&dX, n * in_dim * 4));
  CK(ds.alloc(&dout, n * 4));
  CK(cudaMemcpy(dp, params, P * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dX, X, n * in_dim * 4, cudaMemcpyHostToDevice));
  CK(launch_mlp_predict(dp, dX, n, in_dim, dout, sms, 0));
  CK(cudaMemcpy(out, dout, n * 4, cudaMemcpyDeviceToHost));
  return TOPK_OK;
}

namespace {

// Adam training on the device; params (device) in/out, X/y device.
int device_train(uint32_t in_dim, float *dp, const float *dX, const float *dy, uint64_t n, uint32_t epochs,
                 uint32_t batch, float lr, uint64_t seed, float *epoch_loss) {
  const size_t P = mlp_param_count(in_dim);
  std::vector<uint64_t> mul(std::max<uint32_t>(epochs, 1)), add(mul.size());
  uint64_t x = seed;
  for (uint32_t e = 0; e < epochs; e++) {
    uint64_t a;
    do {
      a = (splitmix(x) % n) | 1u;
    } while (gcd64(a, n) != 1);
    mul[e] = a;
    add[e] = splitmix(x) % n;
  }
  DevScope ds;
  float *dm, *dv, *dl;
  uint64_t *dmul, *dadd;
  unsigned char *dscr;
  const size_t scr = mlp_train_scratch_bytes(in_dim);
  CK(ds.alloc(&dm, P * 4));
  CK(ds.alloc(&dv, P * 4));
  CK(ds.alloc(&dl, mul.size() * 4));
  CK(ds.alloc(&dmul, mul.size() * 8));
  CK(ds.alloc(&dadd, mul.size() * 8));
  CK(ds.alloc(&dscr, scr));
  CK(cudaMemset(dm, 0, P * 4));
  CK(cudaMemset(dv, 0, P * 4));
  CK(cudaMemset(dl, 0, mul.size() * 4));
  CK(cudaMemset(dscr, 0, scr));
  CK(cudaMemcpy(dmul, mul.data(), mul.size() * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dadd, add.data(), add.size() * 8, cudaMemcpyHostToDevice));
  // a barrier wait of 2^24 polls (~1 s) only runs out if a CTA failed
  CK(launch_mlp_train(dp, dm, dv, dX, dy, n, in_dim, batch, epochs, dmul, dadd, lr, dl, dscr, 1ull << 24, 0));
  CK(cudaDeviceSynchronize());
  if (mlp_train_failed(dscr, in_dim)) return fail(TOPK_ERR_TIMEOUT, "training: a grid barrier wait ran out");
  if (epoch_loss) CK(cudaMemcpy(epoch_loss, dl, (size_t)epochs * 4, cudaMemcpyDeviceToHost));
  return TOPK_OK;
}

}  // namespace

extern "C" int topk_mlp_train(int device, uint32_t in_dim, float *params, const float *X, const float *y, uint64_t n,
                   uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float *epoch_loss) {
  g_last_error.clear();
  int st = check_mlp_dims(in_dim);
  if (st != TOPK_OK) return st;
  if (!params || !X || !y) return fail(TOPK_ERR_ARG, "null argument");
  if (batch == 0 || batch > 128) return fail(TOPK_ERR_ARG, "batch must be in [1, 128]");
  if (n < batch || n >= (1ull << 31)) return fail(TOPK_ERR_ARG, "n must be in [batch, 2^31)");
  DeviceGuard dg(device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  const size_t P = mlp_param_count(in_dim);
  DevScope ds;
  float *dp, *dX, *dy;
  CK(ds.alloc(&dp, P * 4));
  CK(ds.alloc(&dX, n * in_dim * 4));
  CK(ds.alloc(&dy, n * 4));
  CK(cudaMemcpy(dp, params, P * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dX, X, n * in_dim * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dy, y, n * 4, cudaMemcpyHostToDevice));
  if ((st = device_train(in_dim, dp, dX, dy, n, epochs, batch, lr, seed, epoch_loss)) != TOPK_OK) return st;
  CK(cudaMemcpy(params, dp, P * 4, cudaMemcpyDeviceToHost));
  return TOPK_OK;
}

extern "C" int topk_query_features(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs, const float *weights,
                        uint64_t wstride, const uint8_t *attrs, uint64_t astride, float *X, float *scale) {
  g_last_error.clear();
  if (!h || (nq && (!ks || !qqs || !weights || !attrs || !X))) return fail(TOPK_ERR_ARG, "null argument");
  int st = check_features_ready(h);
  if (st != TOPK_OK) return st;
  if (nq >= (1ull << 31)) return fail(TOPK_ERR_ARG, "too many queries");
  for (uint64_t j = 0; j < nq; j++) {
    if ((st = check_query(h, ks[j], qqs[j], weights + j * wstride, attrs + j * astride)) != TOPK_OK) return st;
    if (qqs[j] > kBatchMaxQ) return fail(TOPK_ERR_UNSUPPORTED, "features support qq <= %u", kBatchMaxQ);
  }
  if (nq == 0) return TOPK_OK;
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  std::vector<BatchQuery> q = pack_queries(h, nq, ks, qqs, weights, wstride, attrs, astride);
  const uint32_t F = feature_dim(h->d);
  DevScope ds;
  BatchQuery *dq;
  float *dX;
  CK(ds.alloc(&dq, nq * sizeof(BatchQuery)));
  CK(ds.alloc(&dX, nq * F * 4));
  CK(cudaMemcpy(dq, q.data(), nq * sizeof(BatchQuery), cudaMemcpyHostToDevice));
  if ((st = device_features(h, dq, (uint32_t)nq, dX, 0)) != TOPK_OK) return st;
  CK(cudaMemcpy(X, dX, nq * F * 4, cudaMemcpyDeviceToHost));
  if (scale)
    for (uint64_t j = 0; j < nq; j++) scale[j] = query_scale(q[j]);
  return TOPK_OK;
}

extern "C" int topk_set_learned_model(topk_table_t h, const float *params, float margin) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  std::lock_guard<std::mutex> lk(h->learned_mu);
  DeviceGuard dg(h->device);
  if (!params) {
    cudaFree(h->mlp);
    h->mlp = nullptr;
    return TOPK_OK;
  }
  int st = check_features_ready(h);
  if (st != TOPK_OK) return st;
  if (!std::isfinite(margin)) return fail(TOPK_ERR_ARG, "margin must be finite");
  const size_t P = mlp_param_count(feature_dim(h->d));
  if (!h->mlp) CK(cudaMalloc(&h->mlp, P * 4));
  if (!h->lq_query) CK(cudaMalloc(&h->lq_query, sizeof(BatchQuery)));
  if (!h->lq_out) CK(cudaMalloc(&h->lq_out, (kMlpMaxIn + 1) * 4));
  CK(cudaMemcpy(h->mlp, params, P * 4, cudaMemcpyHostToDevice));
  h->mlp_margin = margin;
  h->mlp_part_version = h->part_version;
  return TOPK_OK;
}

extern "C" int topk_learned_fit(topk_table_t h, uint64_t n_train, uint64_t n_val, uint32_t kmin, uint32_t kmax, uint32_t qmin,
                     uint32_t qmax, uint32_t epochs, float miss_rate, uint64_t seed, double *report) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  int st = check_features_ready(h);
  if (st != TOPK_OK) return st;
  if (n_train < 128 || n_train + n_val >= (1ull << 31) || n_val == 0)
    return fail(TOPK_ERR_ARG, "need n_train >= 128 and n_val >= 1");
  if (kmin == 0 || kmin > kmax || kmax > kMaxK) return fail(TOPK_ERR_ARG, "need 1 <= kmin <= kmax <= %u", kMaxK);
  if (qmin == 0 || qmin > qmax || qmax > std::min<uint32_t>(h->d, kBatchMaxQ))
    return fail(TOPK_ERR_ARG, "need 1 <= qmin <= qmax <= min(d, %u)", kBatchMaxQ);
  if (!(miss_rate > 0.0f && miss_rate < 1.0f)) return fail(TOPK_ERR_ARG, "miss_rate must be in (0, 1)");
  DeviceGuard dg(h->device);
  if (!dg.ok) return fail(TOPK_ERR_CUDA, "cudaSetDevice(%d) failed", h->device);
  const uint32_t d = h->d, F = feature_dim(d);
  const uint64_t N = n_train + n_val;
  // random queries: qq uniform in [qmin, qmax] distinct attributes (ascending),
  // weights U(0,1] on the 2^-24 grid, k log-uniform in [kmin, kmax]
  std::vector<uint64_t> ks(N);
  std::vector<uint32_t> qqs(N);
  std::vector<float> W(N * d, 0.0f);
  std::vector<uint8_t> A(N * d, 0);
  uint64_t x = seed ^ 0x5EED0F7E11ull;
  for (uint64_t j = 0; j < N; j++) {
    const uint32_t q = qmin + (uint32_t)(splitmix(x) % (qmax - qmin + 1));
    std::vector<uint8_t> perm(d);
    for (uint32_t m = 0; m < d; m++) perm[m] = (uint8_t)m;
    for (uint32_t m = 0; m < q; m++) std::swap(perm[m], perm[m + splitmix(x) % (d - m)]);
    std::sort(perm.begin(), perm.begin() + q);
    for (uint32_t m = 0; m < q; m++) A[j * d + m] = perm[m];
    for (uint32_t m = 0; m < d; m++) W[j * d + m] = (float)((splitmix(x) >> 40) + 1) * 0x1p-24f;
    const double u = (double)(splitmix(x) >> 11) * 0x1p-53;
    const double lk = std::log((double)kmin) + u * (std::log((double)kmax + 1.0) - std::log((double)kmin));
    ks[j] = std::min<uint64_t>(kmax, std::max<uint64_t>(kmin, (uint64_t)std::exp(lk)));
    qqs[j] = q;
  }
  // exact labels: the k-th score of every query, by the batched exact path
  auto t0 = std::chrono::steady_clock::now();
  std::vector<float> kth(N);
  {
    std::lock_guard<std::mutex> lk(h->batch_mu);
    const uint64_t chunk = 4096;
    std::vector<uint64_t> ids(chunk * kmax), cnt(chunk);
    std::vector<float> sc(chunk * kmax);
    for (uint64_t j0 = 0; j0 < N; j0 += chunk) {
      const uint64_t c = std::min(chunk, N - j0);
      st = run_batch(h, c, &ks[j0], &qqs[j0], &W[j0 * d], d, &A[j0 * d], d, ids.data(), sc.data(), kmax, cnt.data(),
                     &kth[j0]);
      if (st != TOPK_OK) return st;
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  // features, then targets u = qq * ln(gap / S), gap = largest bound - k-th score
  std::vector<BatchQuery> q = pack_queries(h, N, ks.data(), qqs.data(), W.data(), d, A.data(), d);
  std::vector<float> y(N);
  const size_t P = mlp_param_count(F);
  DevScope ds;
  BatchQuery *dq;
  float *dX, *dy, *dp, *dpred;
  CK(ds.alloc(&dq, N * sizeof(BatchQuery)));
  CK(ds.alloc(&dX, N * F * 4));
  CK(ds.alloc(&dy, N * 4));
  CK(ds.alloc(&dp, P * 4));
  CK(ds.alloc(&dpred, n_val * 4));
  CK(cudaMemcpy(dq, q.data(), N * sizeof(BatchQuery), cudaMemcpyHostToDevice));
  if ((st = device_features(h, dq, (uint32_t)N, dX, 0)) != TOPK_OK) return st;
  {
    std::vector<float> b1s(N);
    CK(cudaMemcpy2D(b1s.data(), 4, dX + feature_bound_col(d), (size_t)F * 4, 4, N, cudaMemcpyDeviceToHost));
    for (uint64_t j = 0; j < N; j++) y[j] = learned_target(kth[j], b1s[j], query_scale(q[j]), q[j].qq);
    // Queries whose k-th score ties the largest partition bound (objects at the top
    // of every queried column, e.g. values clipped at 1) have no gap to predict: a
    // batch answers them from its bootstrap instead (their learned start overflows
    // and runs again without it).  Leave them out of training and calibration, so
    // that they do not widen the margin of every other query.
    std::vector<uint64_t> keep_tr, keep_val;
    for (uint64_t j = 0; j < N; j++) {
      const bool tie = !((double)b1s[j] - (double)kth[j] / (double)query_scale(q[j]) > 0x1p-20);
      if (!tie) (j < n_train ? keep_tr : keep_val).push_back(j);
    }
    if (keep_tr.size() >= 128 && !keep_val.empty() && keep_tr.size() + keep_val.size() < N) {
      std::vector<float> X(N * F), X2, y2;
      CK(cudaMemcpy(X.data(), dX, N * F * 4, cudaMemcpyDeviceToHost));
      for (const auto *v : {&keep_tr, &keep_val})
        for (uint64_t j : *v) {
          X2.insert(X2.end(), X.begin() + j * F, X.begin() + (j + 1) * F);
          y2.push_back(y[j]);
        }
      n_train = keep_tr.size();
      n_val = keep_val.size();
      CK(cudaMemcpy(dX, X2.data(), X2.size() * 4, cudaMemcpyHostToDevice));
      y.assign(y2.begin(), y2.end());
    }
  }
  CK(cudaMemcpy(dy, y.data(), y.size() * 4, cudaMemcpyHostToDevice));
  // initial parameters: uniform +-sqrt(6 / fan_in) weights, zero biases, b3 = mean target
  std::vector<float> params(P, 0.0f);
  {
    uint64_t r = seed * 0x2545F4914F6CDD1Dull + 1;
    auto uni = [&](double lim) { return (float)(((double)(splitmix(r) >> 11) * 0x1p-53 * 2.0 - 1.0) * lim); };
    size_t o = 0;
    for (uint32_t i = 0; i < kHid * F; i++) params[o++] = uni(std::sqrt(6.0 / F));
    o += kHid;
    for (uint32_t i = 0; i < kHid * kHid; i++) params[o++] = uni(std::sqrt(6.0 / kHid));
    o += kHid;
    for (uint32_t i = 0; i < kHid; i++) params[o++] = uni(std::sqrt(6.0 / kHid));
    double mean = 0;
    for (uint64_t j = 0; j < n_train; j++) mean += y[j];
    params[o] = (float)(mean / (double)n_train);
  }
  CK(cudaMemcpy(dp, params.data(), P * 4, cudaMemcpyHostToDevice));
  std::vector<float> eloss(std::max<uint32_t>(epochs, 1), 0.0f);
  if ((st = device_train(F, dp, dX, dy, n_train, epochs, 128, 1e-3f, seed, eloss.data())) != TOPK_OK) return st;
  auto t2 = std::chrono::steady_clock::now();
  // calibrate the margin on the held-out queries: the (1 - miss_rate) quantile of
  // target - prediction, so that the cut lies at or below the k-th score for that share
  int sms = h->num_sms;
  CK(launch_mlp_predict(dp, dX + n_train * F, n_val, F, dpred, sms, 0));
  std::vector<float> pred(n_val);
  CK(cudaMemcpy(pred.data(), dpred, n_val * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(params.data(), dp, P * 4, cudaMemcpyDeviceToHost));
  std::vector<double> res(n_val);
  double se = 0;
  for (uint64_t j = 0; j < n_val; j++) {
    res[j] = (double)y[n_train + j] - (double)pred[j];  // the cut is below the k-th score iff res <= margin
    se += res[j] * res[j];
  }
  std::vector<double> sorted = res;
  std::sort(sorted.begin(), sorted.end());
  const uint64_t qi = std::min<uint64_t>(n_val - 1, (uint64_t)std::ceil((1.0 - miss_rate) * (double)n_val));
  const float margin = (float)sorted[qi];
  uint64_t miss = 0;
  for (uint64_t j = 0; j < n_val; j++) miss += res[j] > margin;
  if ((st = topk_set_learned_model(h, params.data(), margin)) != TOPK_OK) return st;
  if (report) {
    report[0] = epochs ? eloss[epochs - 1] : 0.0;
    report[1] = std::sqrt(se / (double)n_val);
    report[2] = margin;
    report[3] = (double)miss / (double)n_val;
    report[4] = std::chrono::duration<double>(t1 - t0).count();
    report[5] = std::chrono::duration<double>(t2 - t1).count();
  }
  return TOPK_OK;
}

extern "C" int topk_get_learned_model(topk_table_t h, float *params, float *margin) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  std::lock_guard<std::mutex> lk(h->learned_mu);
  if (!h->mlp) return fail(TOPK_ERR_STATE, "no learned model");
  if (params) CK(cudaMemcpy(params, h->mlp, mlp_param_count(feature_dim(h->d)) * 4, cudaMemcpyDeviceToHost));
  if (margin) *margin = h->mlp_margin;
  return TOPK_OK;
}

extern "C" int topk_query_learned(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr,
                       uint64_t *ids, float *scores, uint64_t *count, float *threshold, uint64_t *stats,
                       float *cut_out) {
  g_last_error.clear();
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  return run_pruned(h, k, qq, weights, attr, NAN, true, ids, scores, count, threshold, stats, cut_out);
}

extern "C" {

int topk_gather_rows(topk_table_t h, const uint64_t *ids, uint64_t count, float *out) {
  if (!h || (count && (!ids || !out))) return fail(TOPK_ERR_ARG, "null argument");
  for (uint64_t j = 0; j < count; j++)
    if (ids[j] >= h->n) return fail(TOPK_ERR_ARG, "id %llu out of range", (unsigned long long)ids[j]);
  if (count == 0) return TOPK_OK;
  DeviceGuard dg(h->device);
  CtxLease lease(h);
  if (lease.status != TOPK_OK) return lease.status;
  Ctx *c = lease.c;
  const size_t need = (size_t)count * h->d;
  if (c->rows_cap < need) {
    cudaFree(c->d_rows);
    cudaFree(c->d_ids_scratch);
    c->d_rows = nullptr;
    c->d_ids_scratch = nullptr;
    c->rows_cap = 0;
    CK(cudaMalloc(&c->d_rows, need * sizeof(float)));
    CK(cudaMalloc(&c->d_ids_scratch, (size_t)count * sizeof(uint64_t) + need));  // ids fit: need >= count
    c->rows_cap = need;
  }
  CK(cudaMemcpyAsync(c->d_ids_scratch, ids, count * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
  CK(launch_gather(h->table, h->ld, h->d, c->d_ids_scratch, count, c->d_rows, c->stream));
  CK(cudaMemcpyAsync(out, c->d_rows, need * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TOPK_OK;
}

int topk_count_ge(topk_table_t h, uint64_t r0, uint64_t r1, uint32_t qq, const float *weights, const uint8_t *attr,
                  float thr, uint64_t *ge, uint64_t *gt) {
  int st = check_query(h, 1, qq, weights, attr);
  if (st != TOPK_OK) return st;
  if (r1 > h->n || r0 > r1) return fail(TOPK_ERR_ARG, "row range outside the table");
  DeviceGuard dg(h->device);
  CtxLease lease(h);
  if (lease.status != TOPK_OK) return lease.status;
  Ctx *c = lease.c;
  float w[kMaxQ];
  for (uint32_t m = 0; m < qq; m++) w[m] = weights[attr[m]];
  CK(launch_count(h->table, h->ld, r0, r1, qq, attr, w, thr, c->d_count2, c->stream));
  unsigned long long r[2];
  CK(cudaMemcpyAsync(r, c->d_count2, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (ge) *ge = r[0];
  if (gt) *gt = r[1];
  return TOPK_OK;
}

int topk_set_scan_tuning(topk_table_t h, uint32_t max_ctas_per_sm) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (max_ctas_per_sm > 8) return fail(TOPK_ERR_ARG, "max_ctas_per_sm must be 0..8");
  h->max_ctas_per_sm = max_ctas_per_sm;
  return TOPK_OK;
}

int topk_set_fault_injection(topk_table_t h, int mode) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (mode < 0 || mode > 1) return fail(TOPK_ERR_ARG, "mode must be 0 or 1");
  h->fault_mode = mode;
  return TOPK_OK;
}

int topk_last_stats(topk_table_t h, uint64_t *cands, uint64_t *reds) {
  if (!h) return fail(TOPK_ERR_ARG, "null handle");
  if (cands) *cands = g_last_cands;
  if (reds) *reds = g_last_reductions;
  return TOPK_OK;
}

}  // extern "C"
