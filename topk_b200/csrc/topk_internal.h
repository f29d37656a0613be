// Internal interface between the host runtime (topk_abi.cpp) and the kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <string>

namespace topk {

constexpr int kScanThreads = 256;     // threads per scan CTA
constexpr uint32_t kMaxQ = 64;        // attributes per query
constexpr uint32_t kMaxK = 4096;      // largest k of the fused path
constexpr uint32_t kLdAlign = 64;     // device column stride alignment (rows)
constexpr int kMaxLevels = 12;        // merge-tree levels (fan-in >= 2, <= 4096 CTAs)
constexpr int kScanSmemFixed = 1536;  // barriers, control block, radix histogram, weights

// Device-side per-context scratch of the fused scan.  Zero between queries:
// the kernel puts every counter back before it ends.
struct ScanScratch {
  uint32_t g_thr;           // running global threshold key (objects below it cannot win)
  uint32_t error;           // nonzero after a device wait gave up (bit 0: stage wait)
  uint32_t acc_reductions;  // CTA block-selects during this scan
  uint32_t last_cands;      // entries merged at the root of the last scan
  uint32_t last_reductions; // block-selects of the last scan
  // Diagnostics of a TOPK_BOUNDS_CHECK build: first failed check (code, block,
  // tile, two values); the access it guarded was skipped.
  uint32_t diag[5];
  uint32_t acc_tiles;       // tiles scanned during this scan (partition mode)
  uint32_t pub_arrived;     // CTAs that published their best keys (ScanParams::pub)
  uint32_t pub_ready;       // 1 once the bound from the published keys is in g_thr
  uint32_t pad[3];
};

// TOPK_BOUNDS_CHECK codes
enum : uint32_t {
  kDiagCopyShape = 1,   // bulk copy size/alignment/destination out of range
  kDiagCopySource = 2,  // bulk copy source outside the table
  kDiagPhase = 3,       // stage barrier re-armed before its previous phase completed
  kDiagAppend = 4,      // candidate append past capacity
  kDiagCompact = 5,     // compaction write past capacity
  kDiagWait = 6,        // a stage wait gave up
  kDiagOutput = 7,      // output index out of range
  kDiagMerge = 8,       // merge load past capacity
};

struct ScanParams {
  const float *table;   // column-major, stride ld
  uint64_t ld;
  uint64_t row_begin;   // rows [row_begin, row_end) are scanned
  uint64_t row_end;
  uint64_t tile_begin;  // row_begin rounded down to 4 (16-byte copies)
  uint64_t tile_end;    // row_end rounded up to 4 (<= ld)
  uint64_t tile_step;   // rows from one tile to the next (the tile size; a multiple for a sample)
  uint32_t num_tiles;
  uint32_t qq;
  uint32_t k;
  uint32_t cap;         // entries of the shared candidate buffer
  uint32_t mcap;        // shared entries: the buffer, then a select's output (<= k, padded
                        // to a power of two); the merge reuses all of them
  uint32_t fanin;       // merge-tree fan-in G
  uint32_t levels;      // merge-tree levels below the root (level l has nslots[l] slots)
  uint32_t nslots[kMaxLevels];
  uint32_t slot_off[kMaxLevels];  // first slot of level l in `slots` (slot = k entries)
  uint32_t done_off[kMaxLevels];  // first group counter of level l in `done`
  uint64_t wait_limit;  // polls per bounded wait
  uint32_t fault_mode;  // 1: wait on a barrier nothing completes (timeout test)
  ScanScratch *scratch;
  uint2 *slots;         // merge-tree slots, k entries each (key, id)
  // May be null.  Before the merge each CTA publishes the keys of its best pub_m
  // entries here (grid * pub_m entries) and the k-th largest of them raises the global
  // threshold; non-last CTAs wait at most pub_wait polls for it.
  uint2 *pub;
  uint32_t pub_m;
  uint32_t pub_wait;
  // Threshold pass (needs pub and out_kth_key): the published keys' k-th largest goes
  // to *out_kth_key (0 when fewer than k were published) and the scan ends there, no
  // merge and no result.  Run over a sample of the tiles (tile_step) it seeds the full
  // scan that follows: k real objects score at least that key.  It runs the kernel's
  // threshold-pass form: each thread keeps its best kPubMaxPerWarp (key, row) words in
  // registers (no candidate buffer, no select), so pub_m <= 8 * kPubMaxPerWarp.
  uint32_t kth_only;
  uint32_t *slot_count; // entries per slot
  uint32_t *done;       // per-group arrival counters (zero between queries)
  uint64_t *out_ids;    // min(k, rows) ids, ascending by score (null with out_scores: none written)
  float *out_scores;
  float *out_threshold; // may be null
  uint32_t *out_count;  // may be null
  uint32_t *out_kth_key; // may be null: the k-th entry's key when k entries were found, else 0
  uint32_t *out_stats;  // may be null: [0] entries merged at the root, [1] block-selects,
                        // [2] tiles scanned (partition mode)
  // Partition mode (part_list != null): tile t covers rows
  //   part_list[t >> part_shift] << part_rows_log2  +  (t & ((1 << part_shift) - 1)) * tile
  // instead of tile_begin + t * tile; rows stay within [row_begin, row_end).
  const uint32_t *part_list;
  // May be null.  part_key[i] = order key of an upper bound of every score in partition
  // part_list[i], non-increasing in i: a CTA stops at its first tile whose bound is
  // below its threshold (every later tile of that CTA is bounded lower still) -- the
  // reference's stop rule (cpu/VTA.h:210-216, cpu/PTA.h:636-641) per partition.
  const uint32_t *part_key;
  uint32_t part_shift;      // log2(tiles per partition)
  uint32_t part_rows_log2;  // log2(rows per partition)
  const uint32_t *row_ids;  // may be null: id of each row (a reordered table's original ids)
  uint32_t thr_seed;        // objects need key >= thr_seed from the start (0: none)
  const uint32_t *thr_seed_dev;  // may be null: a further seed read from device memory at start
  uint8_t attr[kMaxQ];
  float w[kMaxQ];       // weights[attr[m]], gathered on the host
  // Set by launch_scan: the first four queried columns (table + attr[m] * ld), the
  // rows from one tile of a CTA to its next in id order (grid * tile_step), and the
  // tiles [int_lo, int_lo + int_n) that lie wholly inside [row_begin, row_end).
  const float *colp[4];
  uint64_t grid_rows;
  uint32_t int_lo;
  uint32_t int_n;
};

// The published-keys bound before the merge (ScanParams::pub): used for k >= this and
// grids of at least kPubMinGrid CTAs; pub_keys_per_cta(k, grid) keys per CTA, so the
// array needs grid * 8 * kPubMaxPerWarp entries.  (From k = 128: at k = 64 the bound
// cost more than it saved, 0.447 against 0.439 ms at q = 2 on 2^28 rows.)
constexpr uint32_t kPubMinK = 128;
constexpr uint32_t kPubMinGrid = 16;
constexpr uint32_t kPubWaitPolls = 4096;  // ~64 ns each
// Keys published per CTA: a multiple of its 8 warps, at least ceil(k / grid) + 1, at
// most 8 * kPubMaxPerWarp.
constexpr uint32_t kPubMaxPerWarp = 4;
inline uint32_t pub_keys_per_cta(uint32_t k, uint32_t grid) {
  const uint32_t want = (k + grid - 1) / grid + 1;
  const uint32_t r = (want + 7) / 8;
  return 8 * (r < kPubMaxPerWarp ? r : kPubMaxPerWarp);
}
// A full-table scan with k >= sample_min_k(qq) first runs a threshold pass over every
// kSampleStride-th tile (kth_only), when the table has at least kSampleMinTiles tiles,
// and starts from its bound: few candidates ever reach the select.  The pass pays where
// the selects it saves are a large part of a short scan: from k = 128 at q <= 2, from
// k = 512 up to q = 8, never above (measured per q and k on 2^28 rows; at q = 16 it
// cost 1-3 %, at q = 2, k = 1024 it saved 60 %).
constexpr uint32_t kSampleMinK = 128;
inline uint32_t sample_min_k(uint32_t qq) { return qq <= 2 ? kSampleMinK : qq <= 8 ? 512u : 0xFFFFFFFFu; }
constexpr uint32_t kSampleStride = 64;
constexpr uint64_t kSampleMinTiles = 1u << 16;

struct ScanPlan {
  uint32_t tile;     // objects per tile
  uint32_t stages;   // 1 when the request fits in shared memory, else 0
  uint32_t cap;
  uint32_t mcap;
  uint32_t fanin;
  int ctas_per_sm;
  size_t smem;       // dynamic shared memory bytes
  int grid;
};

// Plan a launch for qq attributes and top-k over `rows` rows (max_ctas_per_sm 0 =
// as many as fit).  stages == 0 means the request does not fit.
ScanPlan plan_scan(uint32_t qq, uint32_t k, uint64_t rows, int num_sms, size_t smem_optin,
                   uint32_t max_ctas_per_sm = 0, bool part = false);
// Fill the merge-tree fields of p for `grid` CTAs; returns slots and group
// counters needed (entries = slots * k).
void plan_merge_tree(ScanParams &p, uint32_t grid, uint32_t fanin, uint32_t *total_slots, uint32_t *total_groups);
cudaError_t launch_scan(const ScanPlan &plan, const ScanParams &p, cudaStream_t stream);
cudaError_t scan_set_attributes(size_t smem_optin);

// Merge of per-shard top-k lists (merge.cu): list j at lists + j * 12 * stride holds
// ids[stride] (u64) then scores[stride] (f32), counts[j] of them valid, base[j] (may
// be null: 0) added to its ids; the best min(k, sum of counts) of the union (score
// descending, then lower id) are written ascending to out_ids / out_scores, the k-th
// score to out_thr (may be null).
constexpr uint32_t kMaxMergeLists = 64;
cudaError_t launch_merge_lists(const unsigned char *lists, uint32_t nlists, uint64_t stride, const uint32_t *counts,
                               const uint32_t *base, uint32_t k, uint64_t *out_ids, float *out_scores, float *out_thr,
                               uint32_t *kept, cudaStream_t s);

// Set the calling thread's message returned by topk_last_error().
void set_last_error(const char *msg);

// Table kernels.
cudaError_t launch_generate(float *table, uint64_t ld, uint32_t d, uint64_t n, int dist, uint64_t seed,
                            cudaStream_t stream);
// Per-column min/max with std::min/std::max semantics.
cudaError_t launch_minmax(const float *table, uint64_t ld, uint32_t d, uint64_t n, uint32_t *work,
                          cudaStream_t stream);
cudaError_t launch_normalize(float *table, uint64_t ld, uint32_t d, uint64_t n, const float *mins,
                             const float *ranges, cudaStream_t stream);
// work layout for launch_minmax (uint32 words): per column
//   [0] max key, [1] min key, [2..3] first +0 index, [4..5] first -0 index; 8 words per column.
constexpr int kMinmaxWords = 8;

// Plain reference-order count of objects in [r0, r1) with score >= thr and > thr.
cudaError_t launch_count(const float *table, uint64_t ld, uint64_t r0, uint64_t r1, uint32_t qq,
                         const uint8_t *attr, const float *w, float thr, unsigned long long *out2,
                         cudaStream_t stream);
// Gather full rows for a list of ids: out[j*d + m] = table[m*ld + ids[j]].
cudaError_t launch_gather(const float *table, uint64_t ld, uint32_t d, const uint64_t *ids, uint64_t cnt,
                          float *out, cudaStream_t stream);

// Partitioned copy (partition.cu): Morton-ordered counting sort of the rows into
// ptable (same stride), perm[row] = original id.  lo/scale: per attribute (device),
// scale = 2^bits / (max - min).  keys: n entries; hist: 2^16 entries.
cudaError_t launch_partition_build(const float *table, uint64_t ld, uint32_t d, uint64_t n, const float *lo,
                                   const float *scale, uint32_t bits, uint16_t *keys, uint32_t *hist,
                                   uint32_t *perm, float *ptable, int num_sms, cudaStream_t s);
// Index orders of the reference as a row permutation: VTA's (cpu/VTA.h:121-135), the
// same over kVtaThreadRanges equal row ranges as VTA's threaded build makes it (IMP 2,
// VPARTITIONS = THREADS, cpu/VTA.h:13,78-85), PTA's (cpu/PTA.h:88-167, 203-236).
// work holds index_order_work_words(n, kind) words; temp is the radix sorts' scratch
// (first call with temp == nullptr to size it).  n < 2^31; PTA also needs n >= 2 and
// d <= 32.
// kGroups: VTA's order inside caller-given groups (device array `groups`, each value
// < 2^group_bits, group_bits <= 31), groups by number: SLA's index with the skyline
// layer as the group (cpu/SLA.h:199-251).
enum class IndexOrder { kVta, kVtaThreads, kPta, kGroups };
constexpr uint32_t kVtaThreadRanges = 16;
uint64_t index_order_work_words(uint64_t n, IndexOrder kind);
cudaError_t launch_index_order(const float *table, uint64_t ld, uint32_t d, uint64_t n, IndexOrder kind,
                               uint32_t *perm, uint32_t *work, void *temp, size_t *temp_bytes, int num_sms,
                               cudaStream_t s, const uint32_t *groups = nullptr, uint32_t group_bits = 0);
// SLA's skyline layers (skyline.cu; cpu/SLA.h:102-139): the layer of every row, 0 = the
// first skyline, with the reference's stop rule (the last <= 100 rows form one layer).
// d <= 32, n < 2^31.  layers: n entries on the host.
int skyline_layers_device(const float *table, uint64_t ld, uint32_t d, uint64_t n, int num_sms, uint32_t *layers,
                          uint64_t *num_layers, std::string *msg);
cudaError_t launch_gather_rows(const float *table, uint64_t ld, uint32_t d, uint64_t n, const uint32_t *perm,
                               float *ptable, int num_sms, cudaStream_t s);
// kd order (partition.cu): the partitions of 2^part_log2 rows are the leaves of a
// balanced binary tree; each node is split at its middle partition boundary after its
// rows are sorted by the attribute of widest spread in it.  n < 2^31.  work:
// kd_order_work_words(n, d, P) words; temp: CUB storage (size query with temp null).
uint32_t kd_levels(uint32_t P);
uint64_t kd_order_work_words(uint64_t n, uint32_t d, uint32_t P);
cudaError_t launch_kd_order(const float *table, uint64_t ld, uint32_t d, uint64_t n, uint32_t part_log2,
                            uint32_t *perm, uint32_t *work, void *temp, size_t *temp_bytes, int num_sms,
                            cudaStream_t s);
// One query's attributes and gathered weights, for partition bounds.
struct PartQuery {
  uint32_t qq;
  uint8_t attr[kMaxQ];
  float w[kMaxQ];  // weights[attr[m]]
};
// Partitions in descending order of the query's bound (the reference-order FP32 sum
// over each partition's per-attribute max, or min for negative weights: an exact upper
// bound of its rows' scores): plist[i] = partition, pkey[i] = order key of an upper
// bound of its scores, non-increasing in i (0xFFFFFFFF for a NaN bound).  Up to
// kPartOrderOneBlock partitions one block orders them by a counting sort into 1024
// buckets over the range of the keys, pkey[i] = the largest key of i's bucket,
// partitions of one bucket in no set order; above, an exact radix sort (ties by the
// lower partition number) uses `temp` (part_order_temp_bytes(P) bytes).
constexpr uint32_t kPartOrderOneBlock = 16384;
size_t part_order_temp_bytes(uint32_t P);
cudaError_t launch_part_order(const float *pmin, const float *pmax, uint32_t P, uint32_t d, const PartQuery &q,
                              uint32_t *plist, uint32_t *pkey, void *temp, size_t temp_bytes, int num_sms,
                              cudaStream_t s);
// Per-partition min / max / mean of each attribute, [num_parts][d] each.
cudaError_t launch_partition_stats(const float *ptable, uint64_t ld, uint32_t d, uint64_t n, uint32_t rows_log2,
                                   uint32_t num_parts, float *mins, float *maxs, float *means, cudaStream_t s);

// Table files (loader.cu).  csv_shape: File<T>::count's n (newlines) and d (1 + commas
// of the first line).  load_csv_device: parses the first n rows of a comma-separated
// file into the column-major table on the device (FP32 correctly rounded, as fscanf's
// "%f"); stats (may be null): bytes consumed, rows found, host-converted values,
// chunks.  Both return a TOPK_* code and a message on failure.
int csv_shape(const char *path, uint64_t *n, uint64_t *d, std::string *msg);
struct LoaderState;  // the loader's pipeline buffers, kept between loads
LoaderState *loader_state_new();
void loader_state_free(LoaderState *L);
int load_csv_device(LoaderState *L, const char *path, float *table, uint64_t ld, uint32_t d, uint64_t n,
                    int num_sms, uint64_t chunk_bytes, uint64_t stats[4], std::string *msg);
int save_csv(const char *path, const float *table, uint64_t ld, uint32_t d, uint64_t n, std::string *msg);
// Binary column-major files: 64-byte header ("TOPKCOL1", version 1, element size 4, n,
// d), then d columns of n FP32 values.
int binary_shape(const char *path, uint64_t *n, uint64_t *d, std::string *msg);
int save_binary(const char *path, const float *table, uint64_t ld, uint32_t d, uint64_t n, std::string *msg);
int load_binary_device(LoaderState *L, const char *path, float *table, uint64_t ld, uint32_t d, uint64_t n,
                       std::string *msg);
// Row-major host tables (row i at host + i*row_stride) to and from the column-major
// device table, through the loader's buffers and a tiled transpose.
int upload_rowmajor_device(LoaderState *L, const float *host, uint64_t row_stride, float *table, uint64_t ld,
                           uint32_t d, uint64_t n, std::string *msg);
int download_rowmajor_device(LoaderState *L, float *host, uint64_t row_stride, const float *table, uint64_t ld,
                             uint32_t d, uint64_t n, std::string *msg);

// Threshold algorithm over sorted lists (ta.cu; cpu/TA.h).  ta_lists_build: per
// attribute the ids by value descending (ties by the lower id) and the sorted values,
// plus query scratch.  ta_query: exact top-k by walking the queried lists (results of
// the full scan); stats: depth walked, objects scored, blocks.  One query at a time
// per TaLists.
struct TaLists;
int ta_lists_build(TaLists **out, const float *table, uint64_t ld, uint32_t d, uint64_t n, int num_sms,
                   std::string *msg);
void ta_lists_free(TaLists *L);
int ta_lists_read(const TaLists *L, uint32_t m, uint32_t *ids, float *vals, std::string *msg);
int ta_query(TaLists *L, const float *table, uint64_t ld, uint64_t k, uint32_t qq, const float *weights,
             const uint8_t *attr, int num_sms, uint64_t *ids, float *scores, uint64_t *count, float *threshold,
             uint64_t *stats, std::string *msg);

}  // namespace topk
