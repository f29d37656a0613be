// Batched exact top-k: many independent queries over one resident table.
//
// Replaces the reference's multi-query loop (validation/bench_cpu.h:198-232 calling
// TPAc::findTopKsimdMQ, cpu/TPAc.h:210-254), which scans the whole table once per
// query; here every table tile read from HBM is scored for a whole group of queries.
// Arithmetic and tie rule per query are those of the single-query path.
//
// Schedule (host-driven, kernels below):
//   bootstrap   each query's exact top-k over the first S0 rows -> best[], and its
//               threshold thr = k-th key + 1 (later rows have larger ids, so an
//               object must beat the k-th strictly);
//   chunks      rows [S0, n) in chunks that double in size; per chunk a scorer
//               appends (key, id) of every object with key >= thr to the query's
//               candidate region, then a reduce merges best[] and the candidates
//               into the new top-k and raises thr.  Doubling keeps the expected
//               candidates per query per chunk near k*ln 2;
//   finish      sort each best[] and write the results ascending by score.
// A query whose candidate region overflows in some chunk (possible only on
// adversarial orders) is flagged; the host answers it with the single-query scan.
//
// Two scorers share this schedule: the plain FP32 one here (exact keys), and the
// BF16 tensor-core filter (bf16_filter.cu), whose candidates carry approximate
// keys that the reduce makes exact by rescoring them in the reference order.
#include <cstdint>
#include <cuda_runtime.h>

#include "batch_internal.h"
#include "block_select.cuh"
#include "device_common.cuh"

namespace topk {

namespace {

constexpr int kBT = 256;  // threads per block of the batched kernels

struct BatchShared {
  SelShared sel;
  uint32_t qq, k;
  uint32_t pad[2];
};

__device__ __forceinline__ float score_row(const float *table, uint64_t ld, uint64_t row, const uint8_t *attr,
                                           const float *w, uint32_t qq) {
  float s = 0.0f;
  for (uint32_t m = 0; m < qq; ++m) s = __fadd_rn(s, __fmul_rn(__ldg(table + (uint64_t)attr[m] * ld + row), w[m]));
  return s;
}

// ---------------------------------------------------------------- bootstrap
// One block per query: exact top-k of rows [0, rows).  Shared: entries[rows] and
// best[k] (dynamic), histogram, select state, the query's attr/weights.
__global__ void __launch_bounds__(kBT) batch_bootstrap_kernel(const float *__restrict__ table, uint64_t ld,
                                                              uint32_t rows, const BatchQuery *__restrict__ qs,
                                                              BatchState *__restrict__ st, uint2 *__restrict__ best) {
  extern __shared__ __align__(16) unsigned char smem[];
  BatchShared *sh = reinterpret_cast<BatchShared *>(smem);
  uint32_t *hist = reinterpret_cast<uint32_t *>(smem + 128);
  uint8_t *attr = smem + 1152;
  float *w = reinterpret_cast<float *>(smem + 1184);
  uint2 *ent = reinterpret_cast<uint2 *>(smem + 1408);
  const BatchQuery &q = qs[blockIdx.x];
  const int t = threadIdx.x;
  if (t < (int)kBatchMaxQ) {
    attr[t] = q.attr[t];
    w[t] = q.w[t];
  }
  if (t == 0) {
    sh->qq = q.qq;
    sh->k = q.k;
  }
  __syncthreads();
  const uint32_t qq = sh->qq, k = sh->k;
  uint2 *out = ent + rows;
  for (uint32_t i = t; i < rows; i += kBT) ent[i] = make_uint2(f2key(score_row(table, ld, i, attr, w, qq)), i);
  __syncthreads();
  const uint32_t kept = block_reduce<kBT>(ent, rows, out, k, 0u, hist, &sh->sel);
  uint2 *dst = best + q.best_off;
  for (uint32_t j = t; j < kept; j += kBT) dst[j] = out[j];
  if (t == 0) {
    BatchState s{};
    s.cnt = kept;
    s.thr = (kept == k) ? sh->sel.kept_min + 1u : 0u;
    st[blockIdx.x] = s;
  }
}

// ---------------------------------------------------------------- FP32 scorer
// Block (query group g, tile): rows [row0, row0 + OPT*256) of the chunk, all d
// columns staged in shared memory once, scored for the group's queries.  With a
// query list the groups are formed from qlist[0..nq) (the queries a hybrid batch has
// moved to this scorer), else from queries 0..nq-1.  With `list_end` the list is
// qlist[*list_begin .. *list_end) as the device holds it when the kernel starts (a
// hybrid batch's lists grow in its reduce, which the host does not wait for): the grid
// is then a fixed set of blocks taking (group, tile) items in order from the counter
// `work` (zero at launch; in order, so the groups reading one tile run together and
// find it in L2), and an empty list costs one read.
template <int OPT>
__global__ void __launch_bounds__(kBT) batch_score_fp32_kernel(const float *__restrict__ table, uint64_t ld,
                                                               uint32_t d, uint64_t r0, uint64_t r1,
                                                               const BatchQuery *__restrict__ qs, uint32_t nq,
                                                               BatchState *__restrict__ st,
                                                               uint2 *__restrict__ cand,
                                                               const uint32_t *__restrict__ qlist,
                                                               const uint32_t *__restrict__ list_end,
                                                               const uint32_t *__restrict__ list_begin,
                                                               uint32_t *__restrict__ work) {
  __shared__ uint32_t next_item;
  constexpr uint32_t TO = kBT * OPT;
  extern __shared__ __align__(16) unsigned char smem[];
  float *xs = reinterpret_cast<float *>(smem);                       // d x TO
  uint8_t *gattr = smem + (size_t)d * TO * 4;                        // kBatchGroup x kBatchMaxQ
  float *gw = reinterpret_cast<float *>(gattr + kBatchGroup * kBatchMaxQ);  // kBatchGroup x kBatchMaxQ
  uint32_t *gthr = reinterpret_cast<uint32_t *>(gw + kBatchGroup * kBatchMaxQ);
  uint32_t *gqq = gthr + kBatchGroup;
  uint32_t *gq = gqq + kBatchGroup;  // query of each group slot

  const int t = threadIdx.x;
  if (list_end) {
    const uint32_t b = list_begin ? *list_begin : 0u;
    nq = *list_end - b;
    qlist += b;
  }
  // item -> (query group, tile), groups fastest: the items of one tile run together
  // and its second and later reads come from L2
  const uint32_t ngroups = (nq + kBatchGroup - 1) / kBatchGroup;
  const uint64_t items = (uint64_t)ngroups * ((r1 - r0 + TO - 1) / TO);
  uint64_t item = blockIdx.x;  // without a list: one item per block
  if (list_end) {
    if (t == 0) next_item = atomicAdd(work, 1u);
    __syncthreads();
    item = next_item;
  }
  while (item < items) {
  const uint32_t q0 = (uint32_t)(item % ngroups) * kBatchGroup;
  const uint64_t tile = item / ngroups;
  const uint32_t nqg = min(kBatchGroup, nq - q0);
  const uint64_t base = r0 + tile * TO;
  const uint32_t valid = (uint32_t)min((uint64_t)TO, r1 - base);
  // stage the tile (rows beyond r1 read as 0 and are never appended)
  for (uint32_t m = 0; m < d; ++m) {
    const float *col = table + (uint64_t)m * ld + base;
    for (uint32_t i = t; i < TO; i += kBT) xs[m * TO + i] = i < valid ? __ldcs(col + i) : 0.0f;
  }
  for (uint32_t j = t; j < nqg; j += kBT) gq[j] = qlist ? qlist[q0 + j] : q0 + j;
  __syncthreads();
  for (uint32_t j = t; j < nqg * kBatchMaxQ; j += kBT) {
    const uint32_t qj = j / kBatchMaxQ, m = j % kBatchMaxQ;
    gattr[j] = qs[gq[qj]].attr[m];
    gw[j] = qs[gq[qj]].w[m];
  }
  for (uint32_t j = t; j < nqg; j += kBT) {
    gthr[j] = st[gq[j]].thr;
    gqq[j] = qs[gq[j]].qq;
  }
  __syncthreads();

  const int lane = t & 31;
  for (uint32_t j = 0; j < nqg; ++j) {
    const uint32_t qq = gqq[j];
    const uint8_t *a = gattr + j * kBatchMaxQ;
    const float *w = gw + j * kBatchMaxQ;
    float acc[OPT];
#pragma unroll
    for (int v = 0; v < OPT; ++v) acc[v] = 0.0f;
    for (uint32_t m = 0; m < qq; ++m) {
      const float *row = xs + (uint32_t)a[m] * TO + t * OPT;
      const float wm = w[m];
      if constexpr (OPT == 4) {
        const float4 x = *reinterpret_cast<const float4 *>(row);
        acc[0] = __fadd_rn(acc[0], __fmul_rn(x.x, wm));
        acc[1] = __fadd_rn(acc[1], __fmul_rn(x.y, wm));
        acc[2] = __fadd_rn(acc[2], __fmul_rn(x.z, wm));
        acc[3] = __fadd_rn(acc[3], __fmul_rn(x.w, wm));
      } else {
#pragma unroll
        for (int v = 0; v < OPT; ++v) acc[v] = __fadd_rn(acc[v], __fmul_rn(row[v], wm));
      }
    }
    const uint32_t thr = gthr[j];
    const bool take_all = thr == 0u;
    const float thr_f = thr_float(thr);
    unsigned pass = 0;
#pragma unroll
    for (int v = 0; v < OPT; ++v)
      pass |= (unsigned)((take_all || acc[v] >= thr_f) && (uint32_t)(t * OPT + v) < valid) << v;
    if (__ballot_sync(0xFFFFFFFFu, pass != 0u)) {  // warp-uniform
      const uint32_t np = __popc(pass);
      uint32_t incl = np;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      const uint32_t wtot = __shfl_sync(0xFFFFFFFFu, incl, 31);
      const BatchQuery &q = qs[gq[j]];
      uint32_t pos = 0;
      if (lane == 31) pos = atomicAdd(&st[gq[j]].ccount, wtot);
      pos = __shfl_sync(0xFFFFFFFFu, pos, 31) + incl - np;
#pragma unroll
      for (int v = 0; v < OPT; ++v)
        if (pass & (1u << v)) {
          if (pos < q.cand_cap) cand[q.cand_off + pos] = make_uint2(f2key(acc[v]), (uint32_t)(base + t * OPT + v));
          ++pos;
        }
    }
  }
  __syncthreads();  // the next item restages the shared tile
  if (!list_end) break;
  if (t == 0) next_item = atomicAdd(work, 1u);
  __syncthreads();
  item = next_item;
  }
}

__global__ void copy_word_kernel(uint32_t *dst, const uint32_t *src) { *dst = *src; }

// ---------------------------------------------------------------- reduce
// One block per query: merge best[] with the chunk's candidates into the new
// top-k.  Candidates of the BF16 filter carry approximate keys: with `rescore`
// each is first scored exactly in the reference order (and the filter's error,
// relative to its bound, recorded).
// Hybrid batches (`sw` non-null: sw[0], sw[1] counts, then two lists of nq
// queries) move a query from the filter to the exact FP32 scorer for the rest of
// the batch when the filter passes too much for it (scores tied or dense at its
// threshold): with more than 2k + 2048 candidates in a chunk the chunk is merged and
// the query is listed in the first list; when candidates were lost (its region or a
// filter log overflowed) the chunk is discarded and the query is listed in both, the
// second list naming the queries whose chunk the FP32 scorer answers again.
__global__ void __launch_bounds__(kBT) batch_reduce_kernel(const float *__restrict__ table, uint64_t ld,
                                                           const BatchQuery *__restrict__ qs,
                                                           BatchState *__restrict__ st, uint2 *__restrict__ best,
                                                           const uint2 *__restrict__ cand, int rescore,
                                                           uint32_t *__restrict__ sw, uint32_t nq) {
  extern __shared__ __align__(16) unsigned char smem[];
  BatchShared *sh = reinterpret_cast<BatchShared *>(smem);
  uint32_t *hist = reinterpret_cast<uint32_t *>(smem + 128);
  uint8_t *attr = smem + 1152;
  float *w = reinterpret_cast<float *>(smem + 1184);
  uint2 *ent = reinterpret_cast<uint2 *>(smem + 1408);
  const BatchQuery &q = qs[blockIdx.x];
  BatchState &s = st[blockIdx.x];
  const int t = threadIdx.x;
  if (t < (int)kBatchMaxQ) {
    attr[t] = q.attr[t];
    w[t] = q.w[t];
  }
  if (t == 0) {
    sh->qq = q.qq;
    sh->k = q.k;
    sh->pad[0] = 0u;  // largest |filter score - exact| / err of this chunk (FP32 bits)
  }
  __syncthreads();
  const uint32_t qq = sh->qq, k = sh->k;
  const uint32_t cnt = min(s.cnt, k);
  const uint32_t thr = s.thr;
  const uint32_t nc_raw = s.ccount;
  if (nc_raw == 0u && !(s.flags & kFlagOverflow)) return;  // nothing new: best[] and the state stand
  const bool filtered = rescore && !(s.flags & kFlagFp32);  // this chunk's candidates came from the filter
  if (sw && filtered && (nc_raw > q.cand_cap || (s.flags & kFlagOverflow))) {
    // block-uniform (every thread read the same state): discard the chunk
    __syncthreads();
    if (t == 0) {
      BatchState ns = s;
      ns.flags = (ns.flags | kFlagFp32) & ~kFlagOverflow;
      ns.cands = (ns.cands + nc_raw < ns.cands) ? 0xFFFFFFFFu : ns.cands + nc_raw;
      ns.ccount = 0;
      s = ns;
      sw[2 + atomicAdd(&sw[0], 1u)] = blockIdx.x;
      sw[2 + nq + atomicAdd(&sw[1], 1u)] = blockIdx.x;
    }
    return;
  }
  const uint32_t nc = min(nc_raw, q.cand_cap);
  const uint32_t total = cnt + nc;
  uint2 *out = ent + cnt + q.cand_cap;
  const uint2 *b = best + q.best_off;
  const uint2 *c = cand + q.cand_off;
  const float err = q.err;
  for (uint32_t j = t; j < cnt; j += kBT) ent[j] = b[j];
  for (uint32_t j = t; j < nc; j += kBT) {
    uint2 e = c[j];
    if (filtered) {
      const float exact = score_row(table, ld, e.y, attr, w, qq);
      const float ratio = fabsf(key2f(e.x) - exact) / err;
      if (ratio == ratio) atomicMax(&sh->pad[0], __float_as_uint(ratio));
      e.x = f2key(exact);
    }
    ent[cnt + j] = e;
  }
  __syncthreads();
  if (thr != 0u) {
    // new entries must reach thr: the k-th key + 1 once best[] is full, or a
    // predicted starting threshold (rescored filter candidates may not reach it)
    for (uint32_t j = cnt + t; j < total; j += kBT)
      if (ent[j].x < thr) ent[j] = make_uint2(0u, 0xFFFFFFFFu);  // below every real entry
    __syncthreads();
  }
  // Entries replaced above carry key 0 and one id, so they share one composite; the
  // select needs distinct composites at its k-th boundary.  Without a learned start
  // best[] is full whenever they exist and they stay below it; with one, the seed
  // (>= 1) as the minimum key leaves them out (and whatever lies below the start).
  const uint32_t kept = block_reduce<kBT>(ent, total, out, k, s.seed, hist, &sh->sel);
  uint2 *dst = best + q.best_off;
  for (uint32_t j = t; j < kept; j += kBT) dst[j] = out[j];
  if (t == 0) {
    BatchState ns = s;
    ns.cnt = kept;
    if (kept == k) ns.thr = max(thr, sh->sel.kept_min + 1u);
    if (nc_raw > q.cand_cap) ns.flags |= kFlagOverflow;
    if (sw && filtered && nc_raw > 2 * k + 2048) {  // tie-dense under the filter: exact scorer from now on
      ns.flags |= kFlagFp32;
      sw[2 + atomicAdd(&sw[0], 1u)] = blockIdx.x;
    }
    ns.cands = (ns.cands + nc_raw < ns.cands) ? 0xFFFFFFFFu : ns.cands + nc_raw;
    ns.errmax = max(ns.errmax, sh->pad[0]);
    ns.ccount = 0;
    s = ns;
  }
}

// ---------------------------------------------------------------- finish
// One block per query: sort best[] and write the result ascending by score.
__global__ void __launch_bounds__(kBT) batch_finish_kernel(const BatchQuery *__restrict__ qs,
                                                           const BatchState *__restrict__ st,
                                                           const uint2 *__restrict__ best, uint64_t *out_ids,
                                                           float *out_scores, uint64_t kstride, uint32_t *out_count,
                                                           float *out_thr) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint2 *a = reinterpret_cast<uint2 *>(smem);
  const BatchQuery &q = qs[blockIdx.x];
  const uint32_t cnt = min(st[blockIdx.x].cnt, q.k);
  const int t = threadIdx.x;
  for (uint32_t j = t; j < cnt; j += kBT) a[j] = best[q.best_off + j];
  __syncthreads();
  block_sort_desc<kBT>(a, cnt);
  uint64_t *ids = out_ids + (uint64_t)blockIdx.x * kstride;
  float *sc = out_scores + (uint64_t)blockIdx.x * kstride;
  for (uint32_t r = t; r < cnt; r += kBT) {
    const uint2 e = a[r];
    ids[cnt - 1 - r] = e.y;
    sc[cnt - 1 - r] = key2f(e.x);
  }
  if (t == 0) {
    out_count[blockIdx.x] = cnt;
    out_thr[blockIdx.x] = cnt ? key2f(a[cnt - 1].x) : 0.0f;
  }
}

constexpr size_t kQueryShared = 1408;  // select state, histogram, attr, weights

}  // namespace

// ---------------------------------------------------------------- launchers
size_t batch_bootstrap_smem(uint32_t rows, uint32_t kmax) { return kQueryShared + (size_t)(rows + kmax) * 8; }

cudaError_t launch_batch_bootstrap(const float *table, uint64_t ld, uint32_t rows, uint32_t kmax,
                                   const BatchQuery *qs, uint32_t nq, BatchState *st, uint2 *best, cudaStream_t s) {
  const size_t smem = batch_bootstrap_smem(rows, kmax);
  cudaError_t e = cudaFuncSetAttribute(batch_bootstrap_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  batch_bootstrap_kernel<<<nq, kBT, smem, s>>>(table, ld, rows, qs, st, best);
  return cudaGetLastError();
}

size_t batch_score_smem(uint32_t d) {
  const uint32_t to = (d <= 16 ? 4u : 1u) * kBT;
  return (size_t)d * to * 4 + kBatchGroup * kBatchMaxQ * 5 + kBatchGroup * 12;
}

cudaError_t launch_batch_score_fp32(const float *table, uint64_t ld, uint32_t d, uint64_t r0, uint64_t r1,
                                    const BatchQuery *qs, uint32_t nq, BatchState *st, uint2 *cand,
                                    const uint32_t *qlist, cudaStream_t s) {
  if (nq == 0 || r1 <= r0) return cudaSuccess;
  const size_t smem = batch_score_smem(d);
  const uint32_t opt = d <= 16 ? 4u : 1u;
  const uint64_t to = (uint64_t)opt * kBT;
  const uint64_t blocks = (uint64_t)((nq + kBatchGroup - 1) / kBatchGroup) * ((r1 - r0 + to - 1) / to);
  if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
  const dim3 grid((unsigned)blocks);
  cudaError_t e;
  if (opt == 4) {
    if ((e = cudaFuncSetAttribute(batch_score_fp32_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
        cudaSuccess)
      return e;
    batch_score_fp32_kernel<4><<<grid, kBT, smem, s>>>(table, ld, d, r0, r1, qs, nq, st, cand, qlist, nullptr, nullptr,
                                                        nullptr);
  } else {
    if ((e = cudaFuncSetAttribute(batch_score_fp32_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
        cudaSuccess)
      return e;
    batch_score_fp32_kernel<1><<<grid, kBT, smem, s>>>(table, ld, d, r0, r1, qs, nq, st, cand, qlist, nullptr, nullptr,
                                                        nullptr);
  }
  return cudaGetLastError();
}

cudaError_t launch_batch_score_fp32_list(const float *table, uint64_t ld, uint32_t d, uint64_t r0, uint64_t r1,
                                         const BatchQuery *qs, BatchState *st, uint2 *cand, const uint32_t *qlist,
                                         const uint32_t *list_end, const uint32_t *list_begin, uint32_t *work,
                                         int num_sms, cudaStream_t s) {
  if (r1 <= r0) return cudaSuccess;
  const size_t smem = batch_score_smem(d);
  const bool four = d <= 16;
  const void *fn = four ? reinterpret_cast<const void *>(batch_score_fp32_kernel<4>)
                        : reinterpret_cast<const void *>(batch_score_fp32_kernel<1>);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBT, smem)) != cudaSuccess) return e;
  const dim3 grid((unsigned)(std::max(1, per_sm) * std::max(1, num_sms)));
  if ((e = cudaMemsetAsync(work, 0, sizeof(uint32_t), s)) != cudaSuccess) return e;
  if (four)
    batch_score_fp32_kernel<4><<<grid, kBT, smem, s>>>(table, ld, d, r0, r1, qs, 0, st, cand, qlist, list_end, list_begin,
                                                        work);
  else
    batch_score_fp32_kernel<1><<<grid, kBT, smem, s>>>(table, ld, d, r0, r1, qs, 0, st, cand, qlist, list_end, list_begin,
                                                        work);
  return cudaGetLastError();
}

cudaError_t launch_copy_word(uint32_t *dst, const uint32_t *src, cudaStream_t s) {
  copy_word_kernel<<<1, 1, 0, s>>>(dst, src);
  return cudaGetLastError();
}

size_t batch_reduce_smem(uint32_t kmax, uint32_t capmax) { return kQueryShared + (size_t)(2 * kmax + capmax) * 8; }

cudaError_t launch_batch_reduce(const float *table, uint64_t ld, const BatchQuery *qs, uint32_t nq, BatchState *st,
                                uint2 *best, const uint2 *cand, uint32_t kmax, uint32_t capmax, bool rescore,
                                uint32_t *sw, cudaStream_t s) {
  const size_t smem = batch_reduce_smem(kmax, capmax);
  cudaError_t e = cudaFuncSetAttribute(batch_reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  batch_reduce_kernel<<<nq, kBT, smem, s>>>(table, ld, qs, st, best, cand, rescore ? 1 : 0, sw, nq);
  return cudaGetLastError();
}

cudaError_t launch_batch_finish(const BatchQuery *qs, uint32_t nq, const BatchState *st, const uint2 *best,
                                uint32_t kmax, uint64_t *out_ids, float *out_scores, uint64_t kstride,
                                uint32_t *out_count, float *out_thr, cudaStream_t s) {
  uint32_t P = 1;
  while (P < kmax) P <<= 1;
  const size_t smem = (size_t)P * 8;
  cudaError_t e = cudaFuncSetAttribute(batch_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  batch_finish_kernel<<<nq, kBT, smem, s>>>(qs, st, best, out_ids, out_scores, kstride, out_count, out_thr);
  return cudaGetLastError();
}

}  // namespace topk
