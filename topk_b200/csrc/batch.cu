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
#include <algorithm>
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

// A query's m-th weight and attribute (m < kBatchMaxQ; entries past qq are unused).
__device__ __forceinline__ float bq_w(const BatchQuery *qs, uint32_t q, int m) { return qs[q].w[m]; }
__device__ __forceinline__ uint32_t bq_attr(const BatchQuery *qs, uint32_t q, int m) { return qs[q].attr[m]; }

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
// One thread per query, one block per (group of 256 queries, tile of `to` rows).  The
// tile's d columns are staged once in shared memory (row stride to + 4 floats, so the
// 16-byte pieces of different attributes at one row fall in different banks), with
// one extra row of zeros; each thread then walks the tile 16 rows at a time and
// scores them for its own query in that query's attribute order (four 16-byte shared
// loads per attribute; weights and row offsets in registers).  A warp runs as many
// steps as its longest query; a shorter query's extra steps add 0 * 0 = +0, which
// leaves every sum as it is (no sum is ever -0: it starts at +0, and +0 + -0 = +0).
// Lanes of a warp read at most d distinct pieces per load -- few when the queries are
// ordered by attribute list, as the host orders them -- so one shared-memory wavefront
// serves up to 32 queries x 4 rows, and the kernel runs near the FP32 pipe's rate of
// one separately rounded multiply and add per product.  Groups are formed from
// qlist[0..nq), or from queries 0..nq-1.  With `list_end` the list is
// qlist[*list_begin .. *list_end) as the device holds it when the kernel starts (a
// hybrid batch's lists grow in its reduce, which the host does not wait for): the grid
// is then a fixed set of blocks taking (group, tile) items in order from the counter
// `work` (zero at launch), so the groups reading one tile run together and find it in
// L2, and an empty list costs one read.  With `retire` a query whose threshold is
// above its largest possible score (BatchQuery::maxkey) is skipped: no row can still
// enter its top-k.
constexpr uint32_t kScoreRows = 16;  // rows per step of a thread

template <int QM>
__global__ void __launch_bounds__(kBT) batch_score_fp32_kernel(const float *__restrict__ table, uint64_t ld,
                                                               uint32_t d, uint32_t to, uint64_t r0, uint64_t r1,
                                                               const BatchQuery *__restrict__ qs, uint32_t nq,
                                                               BatchState *__restrict__ st,
                                                               uint2 *__restrict__ cand,
                                                               const uint32_t *__restrict__ qlist,
                                                               const uint32_t *__restrict__ list_end,
                                                               const uint32_t *__restrict__ list_begin,
                                                               uint32_t *__restrict__ work, int retire) {
  __shared__ uint32_t next_item;
  extern __shared__ __align__(16) float xs[];  // d + 1 rows of `xstride` floats; row d is zero
  const uint32_t xstride = to + 4;
  const int t = threadIdx.x;
  for (uint32_t i = t; i < xstride; i += kBT) xs[d * xstride + i] = 0.0f;
  if (list_end) {
    const uint32_t b = list_begin ? *list_begin : 0u;
    nq = *list_end - b;
    qlist += b;
  }
  // item -> (query group, tile), groups fastest: the items of one tile run together
  // and its second and later reads come from L2
  const uint32_t ngroups = (nq + kBT - 1) / kBT;
  const uint64_t items = (uint64_t)ngroups * ((r1 - r0 + to - 1) / to);
  uint64_t item = blockIdx.x;  // without a list: one item per block
  if (list_end) {
    if (t == 0) next_item = atomicAdd(work, 1u);
    __syncthreads();
    item = next_item;
  }
  uint32_t group = 0xFFFFFFFFu;
  // this thread's query: weights and row offsets (attr * xstride) in registers;
  // steps past its attribute count read the zero row with weight 0
  float w[QM];
  uint32_t off[QM];
  uint32_t qq = 0, q = 0, ccap = 0, coff = 0;
  float thr_f = 0.0f;
  bool take_all = false;
  while (item < items) {
    const uint32_t g = (uint32_t)(item % ngroups);
    const uint64_t tile = item / ngroups;
    const uint64_t base = r0 + tile * to;
    const uint32_t valid = (uint32_t)min((uint64_t)to, r1 - base);
    // stage the tile (rows beyond r1 read as 0 and are never appended); 16-byte
    // loads where the columns allow them
    if ((ld & 3u) == 0 && (base & 3u) == 0) {
      const uint32_t v4 = (valid + 3) / 4, per = to / 4;
      for (uint32_t e = t; e < d * per; e += kBT) {
        const uint32_t m = e / per, i = e % per;
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i < v4) {
          if (4 * i + 4 <= valid) {
            x = __ldcs(reinterpret_cast<const float4 *>(table + (uint64_t)m * ld + base) + i);
          } else {
            const float *c = table + (uint64_t)m * ld + base + 4 * i;
            const uint32_t left = valid - 4 * i;
            x.x = __ldcs(c);
            if (left > 1) x.y = __ldcs(c + 1);
            if (left > 2) x.z = __ldcs(c + 2);
          }
        }
        *reinterpret_cast<float4 *>(xs + m * xstride + 4 * i) = x;
      }
    } else {
      for (uint32_t e = t; e < d * to; e += kBT) {
        const uint32_t m = e / to, i = e % to;
        xs[m * xstride + i] = i < valid ? __ldcs(table + (uint64_t)m * ld + base + i) : 0.0f;
      }
    }
    if (g != group) {
      group = g;
      const uint32_t slot = g * kBT + (uint32_t)t;
      qq = 0;
      if (slot < nq) {
        q = qlist ? qlist[slot] : slot;
        const BatchQuery &bq = qs[q];
        const uint32_t thr = st[q].thr;
        qq = bq.qq;
        if (retire && thr != 0u && thr > bq.maxkey) qq = 0;  // nothing left that can enter
        take_all = thr == 0u;
        thr_f = thr_float(thr);
        ccap = bq.cand_cap;
        coff = bq.cand_off;
      }
#pragma unroll
      for (int m = 0; m < QM; ++m) {
        w[m] = (uint32_t)m < qq ? bq_w(qs, q, m) : 0.0f;
        off[m] = ((uint32_t)m < qq ? (uint32_t)bq_attr(qs, q, m) : d) * xstride;
      }
    }
    __syncthreads();  // tile staged
    const uint32_t qmax = __reduce_max_sync(0xFFFFFFFFu, qq);  // warp-uniform step count
    if (qmax) {
      for (uint32_t o = 0; o < valid; o += kScoreRows) {
        float a[kScoreRows];
#pragma unroll
        for (int v = 0; v < (int)kScoreRows; ++v) a[v] = 0.0f;
#pragma unroll
        for (int m = 0; m < QM; ++m) {
          if ((uint32_t)m >= qmax) break;
          const float4 *row = reinterpret_cast<const float4 *>(xs + off[m] + o);
          const float wm = w[m];
#pragma unroll
          for (int c = 0; c < (int)kScoreRows / 4; ++c) {
            const float4 x = row[c];
            a[4 * c + 0] = __fadd_rn(a[4 * c + 0], __fmul_rn(x.x, wm));
            a[4 * c + 1] = __fadd_rn(a[4 * c + 1], __fmul_rn(x.y, wm));
            a[4 * c + 2] = __fadd_rn(a[4 * c + 2], __fmul_rn(x.z, wm));
            a[4 * c + 3] = __fadd_rn(a[4 * c + 3], __fmul_rn(x.w, wm));
          }
        }
        // the largest of the 16 against the threshold first (NaN never passes it)
        float mx = a[0];
#pragma unroll
        for (int v = 1; v < (int)kScoreRows; ++v) mx = fmaxf(mx, a[v]);
        if (qq && (take_all || mx >= thr_f)) {  // rare once a threshold is known
          unsigned pass = 0;
#pragma unroll
          for (int v = 0; v < (int)kScoreRows; ++v)
            pass |= (unsigned)((take_all || a[v] >= thr_f) && o + v < valid) << v;
          if (pass) {
            uint32_t pos = atomicAdd(&st[q].ccount, (uint32_t)__popc(pass));
#pragma unroll
            for (int v = 0; v < (int)kScoreRows; ++v)
              if (pass & (1u << v)) {
                if (pos < ccap) cand[coff + pos] = make_uint2(f2key(a[v]), (uint32_t)(base + o + v));
                ++pos;
              }
          }
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
  // kstride 0: compact, each query's entries at its best_off (sum of k entries in all)
  const uint64_t off = kstride ? (uint64_t)blockIdx.x * kstride : (uint64_t)q.best_off;
  uint64_t *ids = out_ids + off;
  float *sc = out_scores + off;
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

uint32_t batch_score_rows(uint32_t d) { return d <= 16 ? 1024u : d <= 32 ? 512u : 256u; }

size_t batch_score_smem(uint32_t d) { return (size_t)(d + 1) * (batch_score_rows(d) + 4) * 4; }

namespace {
using ScoreKernel = void (*)(const float *, uint64_t, uint32_t, uint32_t, uint64_t, uint64_t, const BatchQuery *, uint32_t,
                             BatchState *, uint2 *, const uint32_t *, const uint32_t *, const uint32_t *, uint32_t *, int);
ScoreKernel score_kernel(uint32_t qmax) {
  return qmax <= 16 ? batch_score_fp32_kernel<16> : batch_score_fp32_kernel<(int)kBatchMaxQ>;
}
}  // namespace

cudaError_t launch_batch_score_fp32(const float *table, uint64_t ld, uint32_t d, uint64_t r0, uint64_t r1,
                                    const BatchQuery *qs, uint32_t nq, BatchState *st, uint2 *cand,
                                    const uint32_t *qlist, uint32_t qmax, bool retire, cudaStream_t s) {
  if (nq == 0 || r1 <= r0) return cudaSuccess;
  const size_t smem = batch_score_smem(d);
  const uint64_t to = batch_score_rows(d);
  const uint64_t blocks = (uint64_t)((nq + kBT - 1) / kBT) * ((r1 - r0 + to - 1) / to);
  if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
  const ScoreKernel fn = score_kernel(qmax);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<(unsigned)blocks, kBT, smem, s>>>(table, ld, d, (uint32_t)to, r0, r1, qs, nq, st, cand, qlist, nullptr, nullptr,
                                         nullptr, retire ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_batch_score_fp32_list(const float *table, uint64_t ld, uint32_t d, uint64_t r0, uint64_t r1,
                                         const BatchQuery *qs, BatchState *st, uint2 *cand, const uint32_t *qlist,
                                         const uint32_t *list_end, const uint32_t *list_begin, uint32_t *work,
                                         uint32_t qmax, bool retire, int num_sms, cudaStream_t s) {
  if (r1 <= r0) return cudaSuccess;
  const size_t smem = batch_score_smem(d);
  const ScoreKernel fn = score_kernel(qmax);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBT, smem)) != cudaSuccess) return e;
  const dim3 grid((unsigned)(std::max(1, per_sm) * std::max(1, num_sms)));
  if ((e = cudaMemsetAsync(work, 0, sizeof(uint32_t), s)) != cudaSuccess) return e;
  fn<<<grid, kBT, smem, s>>>(table, ld, d, batch_score_rows(d), r0, r1, qs, 0, st, cand, qlist, list_end, list_begin,
                             work, retire ? 1 : 0);
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
