// Internal interface of the batched multi-query path (batch.cu, bf16_filter.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace topk {

constexpr uint32_t kBatchMaxQ = 32;    // attributes per query on the batched path
constexpr uint32_t kBatchMaxD = 64;    // table width the FP32 scorer stages
constexpr uint32_t kBatchBootRows = 8192;  // rows of the exact bootstrap (default)
constexpr uint32_t kBatchBootMax = 16384;  // its shared-memory limit
constexpr uint32_t kBf16MaxD = 16;         // table width of the BF16 tensor-core filter (MMA K)
constexpr uint32_t kBf16LogCap = 32768;    // survivor records (32 values + header, 136 B) per filter CTA

// Per-query descriptor (device, read-only during a batch).
struct BatchQuery {
  uint32_t k, qq;
  uint32_t best_off;   // first entry of this query's best[] (k entries)
  uint32_t cand_off;   // first entry of this query's candidate region
  uint32_t cand_cap;   // entries of the candidate region
  float err;           // BF16 filter: bound on |filter score - exact score|
  float thr0;          // learned start: candidates below it are not kept (0: none)
  uint32_t maxkey;     // key of an upper bound of every score over the table (the
                       // reference-order FP32 sum over column extremes); 0xFFFFFFFF: none
  uint8_t attr[kBatchMaxQ];
  float w[kBatchMaxQ];  // weights[attr[m]]
};

// Per-query running state (device).
// BatchState::flags
constexpr uint32_t kFlagOverflow = 1u;  // candidates were lost (a region or a filter log overflowed)
constexpr uint32_t kFlagFp32 = 2u;      // hybrid batch: the query has moved to the exact FP32 scorer

struct BatchState {
  uint32_t thr;     // min key a later object needs (k-th key + 1 once best[] is full)
  uint32_t cnt;     // entries in best[]
  uint32_t ccount;  // candidates appended since the last reduce (may exceed the cap)
  uint32_t flags;   // kFlagOverflow | kFlagFp32
  uint32_t cands;   // candidates appended over the whole batch (saturating)
  uint32_t errmax;  // BF16 filter: max |filter score - exact score| / err, FP32 bits
  uint32_t seed;    // learned start: every kept entry needs key >= seed (0: none)
  uint32_t pad;
};

size_t batch_bootstrap_smem(uint32_t rows, uint32_t kmax);
cudaError_t launch_batch_bootstrap(const float *table, uint64_t ld, uint32_t rows, uint32_t kmax,
                                   const BatchQuery *qs, uint32_t nq, BatchState *st, uint2 *best, cudaStream_t s);
size_t batch_score_smem(uint32_t d);
// Exact FP32 scorer over rows [r0, r1) for queries qlist[0..nq) (qlist null: 0..nq-1);
// qmax = the largest attribute count among them.  retire: skip queries whose threshold
// is above BatchQuery::maxkey.
cudaError_t launch_batch_score_fp32(const float *table, uint64_t ld, uint32_t d, uint64_t r0, uint64_t r1,
                                    const BatchQuery *qs, uint32_t nq, BatchState *st, uint2 *cand,
                                    const uint32_t *qlist, uint32_t qmax, bool retire, cudaStream_t s);
// The same scorer over the queries qlist[*list_begin .. *list_end) (list_begin may be
// null: from 0), read from device memory when the kernel starts; a fixed grid of
// blocks takes the work items from the counter `work` (zeroed here, in stream order).
cudaError_t launch_batch_score_fp32_list(const float *table, uint64_t ld, uint32_t d, uint64_t r0, uint64_t r1,
                                         const BatchQuery *qs, BatchState *st, uint2 *cand, const uint32_t *qlist,
                                         const uint32_t *list_end, const uint32_t *list_begin, uint32_t *work,
                                         uint32_t qmax, bool retire, int num_sms, cudaStream_t s);
cudaError_t launch_copy_word(uint32_t *dst, const uint32_t *src, cudaStream_t s);  // *dst = *src, in stream order
size_t batch_reduce_smem(uint32_t kmax, uint32_t capmax);
cudaError_t launch_batch_reduce(const float *table, uint64_t ld, const BatchQuery *qs, uint32_t nq, BatchState *st,
                                uint2 *best, const uint2 *cand, uint32_t kmax, uint32_t capmax, bool rescore,
                                uint32_t *sw, cudaStream_t s);
// BF16 tensor-core filter (bf16_filter.cu).
uint64_t bf16_table_bytes(uint64_t n);
// Also the column extremes: ext[m] = largest |x| bits, ext[d + m] = largest order key,
// ext[2d + m] = smallest order key (NaN left out) of column m.
cudaError_t launch_bf16_pack(const float *table, uint64_t ld, uint32_t d, uint64_t n, uint8_t *xbf, uint32_t *ext,
                             int num_sms, cudaStream_t s);
size_t bf16_query_bytes(uint32_t nq);
// Host: write query j's 16-wide row a[] (hi and lo) into the tiled query buffer.
void bf16_pack_query(const float *a, uint32_t j, uint8_t *abf);
// One filter launch over rows [r0, r1): its object tiles, the most query tiles of 128
// one CTA takes (qt_cap) and the grid (the work split itself is made on the device
// from the active count, see launch_bf16_filter).
struct FilterPlan {
  uint64_t tile0, tile1;
  uint32_t qt_cap;
  uint64_t grid;
};
// nq: queries of the batch (the most that can be active); qt_cap 0: the kernel's maximum
FilterPlan plan_bf16_filter(uint32_t nq, uint64_t r0, uint64_t r1, int num_sms, uint32_t qt_cap = 0);
// r0 must be a multiple of 256.  The filter serves the *nact active queries in the
// compact tiles abf (slot -> query: amap); recv/rech hold grid * rec_cap records.
cudaError_t launch_bf16_filter(const FilterPlan &f, const uint8_t *xbf, const uint8_t *abf, const uint32_t *amap,
                               const uint32_t *nact, uint64_t r0, uint64_t r1, const BatchQuery *qs, BatchState *st,
                               uint2 *cand, uint4 *recv, uint2 *rech, uint32_t rec_cap, uint64_t wait_limit,
                               uint32_t *err, cudaStream_t s);
// Before each chunk: the queries the filter still serves (neither moved to the FP32
// scorer nor retired by BatchQuery::maxkey), their rows of abf copied into compact
// tiles abf_act (same size as abf), amap[slot] = query, *nact = count (and, when
// nact_log is not null, *nact_log = count: the chunk's entry of a per-batch record).
cudaError_t launch_batch_active(const BatchQuery *qs, const BatchState *st, uint32_t nq, const uint8_t *abf,
                                uint8_t *abf_act, uint32_t *amap, uint32_t *nact, uint32_t *nact_log,
                                cudaStream_t s);
// Learned k-th-score model (mlp.cu): in -> 64 -> 64 -> 1 ReLU MLP, features of
// feature_dim(d) values per query from the partition statistics ([P][d] each).
constexpr uint32_t kHid = 64;
constexpr uint32_t kMlpMaxIn = 64;
constexpr uint32_t kMaxFeatureParts = 16384;
__host__ __device__ constexpr uint32_t feature_dim(uint32_t d) { return 2 * d + 18; }
__host__ __device__ constexpr uint32_t feature_bound_col(uint32_t d) { return 2 * d + 2; }  // largest bound / S
uint32_t mlp_param_count(uint32_t F);
cudaError_t launch_mlp_grad(const float *params, const float *X, const float *y, uint32_t B, uint32_t F, float *grad,
                            float *loss, cudaStream_t s);
// Training on kTrainCtas CTAs (cooperative launch): scratch holds
// mlp_train_scratch_bytes(F) bytes, zeroed by the caller, and epoch_loss is zeroed too;
// every grid barrier waits at most wait_limit polls, after which the kernel stops and
// mlp_train_failed (after the stream is synchronised) reports it.
constexpr uint32_t kTrainCtas = 8;
size_t mlp_train_scratch_bytes(uint32_t F);
cudaError_t launch_mlp_train(float *params, float *m, float *v, const float *X, const float *y, uint64_t N, uint32_t F,
                             uint32_t B, uint32_t epochs, const uint64_t *mul, const uint64_t *add, float lr,
                             float *epoch_loss, void *scratch, uint64_t wait_limit, cudaStream_t s);
bool mlp_train_failed(const void *scratch, uint32_t F);
cudaError_t launch_mlp_predict(const float *params, const float *X, uint64_t N, uint32_t F, float *out, int num_sms,
                               cudaStream_t s);
// With seed (one query, params given): also *seed = key of its learned cut (0: none)
// and *cut = the cut (NaN when not finite), from the same launch.
cudaError_t launch_features(const float *pmin, const float *pmax, const float *pmean, uint32_t P, uint32_t d,
                            const BatchQuery *qs, uint32_t nq, float *X, const float *params, float *pred,
                            cudaStream_t s, float margin = 0.0f, uint32_t *seed = nullptr, float *cut = nullptr);
// The learned cut: largest bound - S * exp((u + margin) / qq), u the model's output
// (b1s: the largest partition bound / S, a feature).
__host__ __device__ inline float learned_cut(float u, float b1s, float S, float qq, float margin) {
  return (b1s - expf((u + margin) / qq)) * S;
}
// Start each query's state at its learned cut (pred: model outputs; X: features).
cudaError_t launch_learned_seed(const float *pred, const float *X, uint32_t d, const BatchQuery *qs, float margin,
                                BatchState *st, uint32_t nq, cudaStream_t s);
// Each query's result, ascending, at out + j * kstride, or at out + its best_off when
// kstride is 0 (compact: sum of k entries in all).
cudaError_t launch_batch_finish(const BatchQuery *qs, uint32_t nq, const BatchState *st, const uint2 *best,
                                uint32_t kmax, uint64_t *out_ids, float *out_scores, uint64_t kstride,
                                uint32_t *out_count, float *out_thr, cudaStream_t s);

}  // namespace topk
