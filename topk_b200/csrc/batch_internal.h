// Internal interface of the batched multi-query path (batch.cu, bf16_filter.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace topk {

constexpr uint32_t kBatchMaxQ = 32;    // attributes per query on the batched path
constexpr uint32_t kBatchGroup = 64;   // queries scored per staged table tile (FP32 scorer)
constexpr uint32_t kBatchMaxD = 64;    // table width the FP32 scorer stages
constexpr uint32_t kBatchBootRows = 8192;  // rows of the exact bootstrap

// Per-query descriptor (device, read-only during a batch).
struct BatchQuery {
  uint32_t k, qq;
  uint32_t best_off;   // first entry of this query's best[] (k entries)
  uint32_t cand_off;   // first entry of this query's candidate region
  uint32_t cand_cap;   // entries of the candidate region
  float err;           // tensor-core filter: bound on |approximate - exact score|
  float thr0;          // learned start: candidates below it are not kept (0: none)
  uint32_t pad;
  uint8_t attr[kBatchMaxQ];
  float w[kBatchMaxQ];  // weights[attr[m]]
};

// Per-query running state (device).
struct BatchState {
  uint32_t thr;     // min key a later object needs (k-th key + 1 once best[] is full)
  uint32_t cnt;     // entries in best[]
  uint32_t ccount;  // candidates appended since the last reduce (may exceed the cap)
  uint32_t flags;   // bit 0: a candidate region overflowed (exact fallback needed)
};

size_t batch_bootstrap_smem(uint32_t rows, uint32_t kmax);
cudaError_t launch_batch_bootstrap(const float *table, uint64_t ld, uint32_t rows, uint32_t kmax,
                                   const BatchQuery *qs, uint32_t nq, BatchState *st, uint2 *best, cudaStream_t s);
size_t batch_score_smem(uint32_t d);
cudaError_t launch_batch_score_fp32(const float *table, uint64_t ld, uint32_t d, uint64_t r0, uint64_t r1,
                                    const BatchQuery *qs, uint32_t nq, BatchState *st, uint2 *cand, cudaStream_t s);
size_t batch_reduce_smem(uint32_t kmax, uint32_t capmax);
cudaError_t launch_batch_reduce(const float *table, uint64_t ld, const BatchQuery *qs, uint32_t nq, BatchState *st,
                                uint2 *best, const uint2 *cand, uint32_t kmax, uint32_t capmax, bool rescore,
                                cudaStream_t s);
cudaError_t launch_batch_finish(const BatchQuery *qs, uint32_t nq, const BatchState *st, const uint2 *best,
                                uint32_t kmax, uint64_t *out_ids, float *out_scores, uint64_t kstride,
                                uint32_t *out_count, float *out_thr, cudaStream_t s);

}  // namespace topk
