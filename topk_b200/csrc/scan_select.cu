// Fused single-query scan + exact top-k select (sm_100a).
//
// Replaces the TPAc full-table evaluation (cpu/TPAc.h:118-207 findTopKsimd,
// :257-358 findTopKthreads): the same per-object arithmetic
//     s = 0; for m in attr order: s = s + x[attr[m]] * w[attr[m]]   (RN mul, RN add)
// and the same result (the k best by score; ties here go to the lower id).
//
// Design, per persistent CTA (256 threads, one or more per SM):
//   * Only the qq queried columns are streamed.  For each tile of TILE objects the
//     elected thread issues one cp.async.bulk (TMA engine) copy per column into a
//     multi-stage shared-memory ring, completing on an mbarrier; the ring keeps
//     several tiles in flight per SM, which is what saturates HBM.
//   * Threads read their objects from shared memory with 128/64/32-bit loads and
//     score them; an object passes if its key >= the running threshold.  Passing
//     objects go to a shared candidate buffer (warp-aggregated append).
//   * When the buffer nears capacity the CTA selects its top-k by an 8-bit radix
//     select on the 64-bit (key, ~id) word, keeps those k, raises its local
//     threshold and publishes its k-th key with atomicMax to a global word that
//     every CTA folds into its own filter.  Any CTA's k-th best lower-bounds the
//     global k-th best, so nothing that can win is dropped.
//   * At the end each CTA appends its survivors to a global list; the last CTA to
//     finish selects the final top-k from it, sorts (bitonic) and writes the
//     result, then zeroes the scratch for the next query.
// Every mbarrier wait is bounded; a wait that runs out sets scratch->error and the
// CTA leaves uniformly.
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "topk_internal.h"

namespace topk {

namespace {

struct SmemCtl {
  uint32_t count;       // entries in cand[]
  uint32_t thr_local;   // min key that can still enter (k-th local key + 1)
  uint32_t thr_g;       // copy of the global threshold
  uint32_t kept_min;    // min key among kept entries (select result)
  uint32_t digit, above, eq, valid;
  uint32_t wcount;      // compaction write cursor
  uint32_t is_last;
  uint32_t reductions;
  uint32_t timed_out;
  uint32_t base;        // global append base
  uint32_t pad[3];
};

// shared layout: [0,64) stage barriers, [64,72) test barrier, [128,192) SmemCtl,
// then the radix histogram, the stage ring and the candidate buffer.
constexpr int kCtlBytes = 256;
constexpr int kHistBytes = 256 * 4;

// TOPK_BOUNDS_CHECK: record the first failed check in scratch->diag and tell the
// caller to skip the guarded access.  Compiled out of the product build.
#ifdef TOPK_BOUNDS_CHECK
__device__ __forceinline__ bool check(bool ok, ScanScratch *s, uint32_t code, uint32_t i, uint32_t a, uint32_t b) {
  if (!ok && atomicCAS(&s->diag[0], 0u, code) == 0u) {
    s->diag[1] = blockIdx.x;
    s->diag[2] = i;
    s->diag[3] = a;
    s->diag[4] = b;
  }
  return ok;
}
__device__ __forceinline__ bool mbar_test_parity(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
#define TOPK_CHECK(cond, code, i, a, b) check((cond), p.scratch, (code), (i), (a), (b))
#else
#define TOPK_CHECK(cond, code, i, a, b) true
#endif

// Source of candidate entries for the radix select: shared or global memory.
struct SmemSrc {
  const uint2 *p;
  __device__ uint2 operator()(uint32_t j) const { return p[j]; }
};
struct GlobalSrc {
  const uint2 *p;
  __device__ uint2 operator()(uint32_t j) const { return __ldcg(p + j); }
};

// Block-wide radix select over `count` entries of `src` that have key >= min_key:
// finds (prefix, mask) such that exactly `need` valid entries satisfy
// (composite & mask) >= prefix.  Requires need <= number of valid entries.
template <class Src>
__device__ void block_radix_select(const Src &src, uint32_t count, uint32_t min_key, uint32_t need,
                                   uint32_t *hist, SmemCtl *ctl, uint64_t &prefix_out,
                                   uint64_t &mask_out) {
  const int tid = threadIdx.x;
  uint64_t prefix = 0, mask = 0;
  for (int shift = 56; shift >= 0; shift -= 8) {
    hist[tid] = 0;  // kScanThreads == 256 bins
    __syncthreads();
    for (uint32_t j = tid; j < count; j += kScanThreads) {
      uint2 e = src(j);
      if (e.x < min_key) continue;
      uint64_t c = composite(e.x, e.y);
      if ((c & mask) == prefix) atomicAdd(&hist[(uint32_t)(c >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (tid < 32) {
      // lane l owns bins [255-8l-7, 255-8l], visited from high to low.
      const int hi = 255 - 8 * tid;
      uint32_t local[8];
      uint32_t s = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) { local[b] = hist[hi - b]; s += local[b]; }
      uint32_t incl = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (tid >= o) incl += v;
      }
      uint32_t excl = incl - s;
      if (excl < need && need <= incl) {
        uint32_t run = excl;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          if (run + local[b] >= need) {
            ctl->digit = (uint32_t)(hi - b);
            ctl->above = run;
            ctl->eq = local[b];
            break;
          }
          run += local[b];
        }
      }
    }
    __syncthreads();
    const uint32_t digit = ctl->digit, above = ctl->above, eq = ctl->eq;
    __syncthreads();  // everyone read ctl before it is rewritten next pass
    need -= above;
    prefix |= (uint64_t)digit << shift;
    mask |= (uint64_t)0xFFu << shift;
    if (eq == need) break;
  }
  prefix_out = prefix;
  mask_out = mask;
}

// Reduce the shared candidate buffer to its best k valid entries (in place).
// Valid = key >= min_key.  Updates ctl->count; returns true and sets
// ctl->kept_min when exactly k entries remain (the CTA then knows a k-th key).
template <int R>
__device__ bool block_reduce(uint2 *cand, uint32_t k, uint32_t min_key, uint32_t *hist, SmemCtl *ctl) {
  const int tid = threadIdx.x;
  const uint32_t count = ctl->count;
  // count valid entries
  uint32_t v = 0;
  for (uint32_t j = tid; j < count; j += kScanThreads) v += (cand[j].x >= min_key);
  v = warp_sum_u32(v);
  if (tid == 0) { ctl->valid = 0; ctl->wcount = 0; ctl->kept_min = 0xFFFFFFFFu; }
  __syncthreads();
  if ((tid & 31) == 0) atomicAdd(&ctl->valid, v);
  __syncthreads();
  const uint32_t valid = ctl->valid;
  uint64_t prefix = 0, mask = 0;
  const bool select = valid > k;
  if (select) block_radix_select(SmemSrc{cand}, count, min_key, k, hist, ctl, prefix, mask);
  // compaction: pull my entries into registers, then write the kept ones back
  uint2 mine[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    uint32_t j = tid + r * kScanThreads;
    mine[r] = (j < count) ? cand[j] : make_uint2(0u, 0xFFFFFFFFu);
  }
  __syncthreads();
  uint32_t kmin = 0xFFFFFFFFu;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    uint32_t j = tid + r * kScanThreads;
    bool keep = j < count && mine[r].x >= min_key &&
                (!select || (composite(mine[r].x, mine[r].y) & mask) >= prefix);
    unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
    uint32_t base = 0;
    if ((tid & 31) == 0 && bal) base = atomicAdd(&ctl->wcount, (uint32_t)__popc(bal));
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (keep) {
      cand[base + __popc(bal & ((1u << (tid & 31)) - 1u))] = mine[r];
      kmin = min(kmin, mine[r].x);
    }
  }
  kmin = warp_min_u32(kmin);
  if ((tid & 31) == 0) atomicMin(&ctl->kept_min, kmin);
  __syncthreads();
  if (tid == 0) ctl->count = ctl->wcount;
  __syncthreads();
  return ctl->count == k;
}

// Sort cand[0..n) descending by composite (bitonic, padded to a power of two).
__device__ void block_sort_desc(uint2 *cand, uint32_t n, uint32_t pcap) {
  const int tid = threadIdx.x;
  uint32_t P = 1;
  while (P < n) P <<= 1;
  (void)pcap;
  for (uint32_t j = n + tid; j < P; j += kScanThreads) cand[j] = make_uint2(0u, 0xFFFFFFFFu);
  __syncthreads();
  for (uint32_t size = 2; size <= P; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = tid; i < P / 2; i += kScanThreads) {
        uint32_t lo = 2 * i - (i & (stride - 1));
        uint32_t hi = lo + stride;
        bool desc = (lo & size) == 0;
        uint2 a = cand[lo], b = cand[hi];
        uint64_t ca = composite(a.x, a.y), cb = composite(b.x, b.y);
        if (desc ? (ca < cb) : (ca > cb)) { cand[lo] = b; cand[hi] = a; }
      }
      __syncthreads();
    }
  }
}

template <int VEC>
struct VecLoad;
template <>
struct VecLoad<1> {
  __device__ static void load(const float *p, float *x) { x[0] = p[0]; }
};
template <>
struct VecLoad<2> {
  __device__ static void load(const float *p, float *x) {
    float2 v = *reinterpret_cast<const float2 *>(p);
    x[0] = v.x; x[1] = v.y;
  }
};
template <>
struct VecLoad<4> {
  __device__ static void load(const float *p, float *x) {
    float4 v = *reinterpret_cast<const float4 *>(p);
    x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
  }
};

// R = max candidate entries per thread in block_reduce (cap / 256).
template <int VEC, int R>
__global__ void __launch_bounds__(kScanThreads, 1) scan_select_kernel(const __grid_constant__ ScanParams p) {
  constexpr uint32_t TILE = kScanThreads * VEC;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *never = reinterpret_cast<uint64_t *>(smem + 64);
  SmemCtl *ctl = reinterpret_cast<SmemCtl *>(smem + 128);
  uint32_t *hist = reinterpret_cast<uint32_t *>(smem + kCtlBytes);
  float *stage = reinterpret_cast<float *>(smem + kCtlBytes + kHistBytes);
  uint2 *cand = reinterpret_cast<uint2 *>(stage + (size_t)p.stages * p.qq * TILE);

  const int tid = threadIdx.x;
  const uint32_t qq = p.qq;
  const uint32_t S = p.stages;
  const uint32_t my_tiles =
      blockIdx.x < p.num_tiles ? (p.num_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

  if (tid == 0) {
    for (uint32_t s = 0; s < S; ++s) mbar_init(&full[s], 1);
    mbar_init(never, 1);
    fence_barrier_init();
    ctl->count = 0;
    ctl->thr_local = 0;
    ctl->thr_g = ld_volatile_u32(&p.scratch->g_thr);
    ctl->reductions = 0;
    ctl->timed_out = 0;
  }
  __syncthreads();

  auto issue = [&](uint32_t i) {
    const uint32_t s = i % S;
    const uint64_t t = blockIdx.x + (uint64_t)i * gridDim.x;
    const uint64_t base = p.tile_begin + t * TILE;
    const uint64_t left = p.tile_end - base;
    const uint32_t objs = left < TILE ? (uint32_t)left : TILE;
    const uint32_t bytes = objs * 4u;
#ifdef TOPK_BOUNDS_CHECK
    if (i >= S && !TOPK_CHECK(mbar_test_parity(&full[s], ((i - S) / S) & 1u), kDiagPhase, i, s, 0)) return;
#endif
    mbar_arrive_expect_tx(&full[s], bytes * qq);
    for (uint32_t m = 0; m < qq; ++m) {
      float *dst = stage + ((size_t)s * qq + m) * TILE;
      const float *src = p.table + (uint64_t)p.attr[m] * p.ld + base;
      if (!TOPK_CHECK(objs > 0 && (bytes & 15u) == 0 && ((uintptr_t)dst & 15u) == 0 &&
                          (const unsigned char *)dst + bytes <= (const unsigned char *)cand,
                      kDiagCopyShape, i, m, bytes))
        continue;
      if (!TOPK_CHECK(((uintptr_t)src & 15u) == 0 && base + objs <= p.ld && p.attr[m] < 255, kDiagCopySource, i,
                      m, (uint32_t)base))
        continue;
      bulk_g2s(dst, src, bytes, &full[s]);
    }
  };

  if (p.fault_mode == 1) {
    // Test hook: wait, before any copy is in flight, on a barrier that nothing
    // arrives on.  The bounded wait runs out and the scan reports a timeout.
    const bool ok = mbar_wait_bounded(never, 0, p.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(&p.scratch->error, 1u);
      return;
    }
  }

  if (tid == 0)
    for (uint32_t i = 0; i < S && i < my_tiles; ++i) issue(i);

  for (uint32_t i = 0; i < my_tiles; ++i) {
    const uint32_t s = i % S;
    const bool ok = mbar_wait_bounded(&full[s], (i / S) & 1u, p.wait_limit);
    const uint64_t t = blockIdx.x + (uint64_t)i * gridDim.x;
    const uint64_t row0 = p.tile_begin + t * TILE + (uint64_t)tid * VEC;
    const uint32_t thr = max(ctl->thr_local, *reinterpret_cast<volatile uint32_t *>(&ctl->thr_g));

    float acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = 0.0f;
    const float *col = stage + (size_t)s * qq * TILE + tid * VEC;
    for (uint32_t m = 0; m < qq; ++m) {
      float x[VEC];
      VecLoad<VEC>::load(col + (size_t)m * TILE, x);
      const float w = p.w[m];
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = __fadd_rn(acc[v], __fmul_rn(x[v], w));
    }
    // filter and append
    uint32_t keys[VEC];
    unsigned pass_mask = 0;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      keys[v] = f2key(acc[v]);
      const uint64_t row = row0 + v;
      if (row >= p.row_begin && row < p.row_end && keys[v] >= thr) pass_mask |= 1u << v;
    }
    uint32_t npass = __popc(pass_mask);
    uint32_t incl = npass;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if ((tid & 31) >= o) incl += y;
    }
    const uint32_t wtotal = __shfl_sync(0xFFFFFFFFu, incl, 31);
    // Buffer fill after this warp's append.  The warp that appends last in a tile
    // sees the tile's final count, so OR-voting "after > cap - TILE" at the barrier
    // below gives every thread the same reduce decision.  (Reading ctl->count after
    // the barrier would not: a fast warp may already be appending the next tile.)
    uint32_t after = 0;
    if (wtotal) {
      uint32_t base = 0;
      if ((tid & 31) == 31) base = atomicAdd(&ctl->count, wtotal);
      base = __shfl_sync(0xFFFFFFFFu, base, 31);
      after = base + wtotal;
      base += incl - npass;
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        if (pass_mask & (1u << v)) {
          if (TOPK_CHECK(base < p.cap, kDiagAppend, i, base, p.cap)) cand[base] = make_uint2(keys[v], (uint32_t)(row0 + v));
          ++base;
        }
    }
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        TOPK_CHECK(false, kDiagWait, i, s, (i / S) & 1u);
        atomicOr(&p.scratch->error, 1u);
        // let this CTA's own copies still in flight land (bounded) before leaving
        for (uint32_t j = i; j < i + S && j < my_tiles; ++j)
          mbar_wait_bounded(&full[j % S], (j / S) & 1u, p.wait_limit);
      }
      return;
    }
    if (tid == 0 && i + S < my_tiles) issue(i + S);
    if (__syncthreads_or(after > p.cap - TILE)) {
      if (tid == 0) ctl->thr_g = ld_volatile_u32(&p.scratch->g_thr);
      __syncthreads();
      const uint32_t min_key = max(ctl->thr_g, 0u);
      if (block_reduce<R>(cand, p.k, min_key, hist, ctl)) {
        if (tid == 0) {
          const uint32_t kth = ctl->kept_min;
          ctl->thr_local = kth + 1u;
          atomicMax(&p.scratch->g_thr, kth);
        }
      }
      if (tid == 0) ctl->reductions++;
      __syncthreads();
    } else if (tid == 0) {
      ctl->thr_g = ld_volatile_u32(&p.scratch->g_thr);
    }
  }

  // ---- end of scan: reduce to <= k, append survivors to the global list ----
  __syncthreads();
  if (tid == 0) ctl->thr_g = ld_volatile_u32(&p.scratch->g_thr);
  __syncthreads();
  if (ctl->count > p.k) {
    if (block_reduce<R>(cand, p.k, ctl->thr_g, hist, ctl)) {
      if (tid == 0) atomicMax(&p.scratch->g_thr, ctl->kept_min);
    }
    if (tid == 0) ctl->reductions++;
    __syncthreads();
  }
  if (tid == 0) {
    ctl->thr_g = ld_volatile_u32(&p.scratch->g_thr);
    ctl->wcount = 0;
  }
  __syncthreads();
  {
    const uint32_t g = ctl->thr_g;
    const uint32_t count = ctl->count;
    uint32_t v = 0;
    for (uint32_t j = tid; j < count; j += kScanThreads) v += cand[j].x >= g;
    v = warp_sum_u32(v);
    if ((tid & 31) == 0 && v) atomicAdd(&ctl->wcount, v);
    __syncthreads();
    if (tid == 0) {
      ctl->base = ctl->wcount ? atomicAdd(&p.scratch->cand_count, ctl->wcount) : 0u;
      ctl->wcount = 0;
      if (ctl->reductions) atomicAdd(&p.scratch->acc_reductions, ctl->reductions);
    }
    __syncthreads();
    const uint32_t base = ctl->base;
    for (uint32_t j = tid; j < count; j += kScanThreads) {
      const uint2 e = cand[j];
      if (e.x >= g) {
        const uint32_t slot = base + atomicAdd(&ctl->wcount, 1u);
        if (slot < p.gcand_cap) p.gcand[slot] = e;
        else atomicOr(&p.scratch->error, 2u);  // list sized too small (host bug)
      }
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) ctl->is_last = (atomicAdd(&p.scratch->done, 1u) == gridDim.x - 1) ? 1u : 0u;
  __syncthreads();
  if (!ctl->is_last) return;
  __threadfence();

  // ---- last CTA: final select over the global list ----
  if (tid == 0) {
    ctl->thr_g = ld_volatile_u32(&p.scratch->g_thr);
    ctl->base = min(ld_volatile_u32(&p.scratch->cand_count), p.gcand_cap);
    ctl->valid = 0;
    ctl->wcount = 0;
  }
  __syncthreads();
  const uint32_t g = ctl->thr_g;
  const uint32_t total = ctl->base;
  {
    uint32_t v = 0;
    for (uint32_t j = tid; j < total; j += kScanThreads) v += __ldcg(&p.gcand[j]).x >= g;
    v = warp_sum_u32(v);
    if ((tid & 31) == 0 && v) atomicAdd(&ctl->valid, v);
  }
  __syncthreads();
  const uint32_t valid = ctl->valid;
  const uint32_t kk = min(valid, p.k);
  uint64_t prefix = 0, mask = 0;
  const bool select = valid > kk;
  if (select) block_radix_select(GlobalSrc{p.gcand}, total, g, kk, hist, ctl, prefix, mask);
  __syncthreads();
  if (tid == 0) ctl->wcount = 0;
  __syncthreads();
  for (uint32_t j = tid; j < total; j += kScanThreads) {
    uint2 e = __ldcg(&p.gcand[j]);
    bool keep = e.x >= g && (!select || (composite(e.x, e.y) & mask) >= prefix);
    if (keep) {
      const uint32_t slot = atomicAdd(&ctl->wcount, 1u);
      if (slot < p.cap) cand[slot] = e;  // exactly kk <= k <= cap are kept
    }
  }
  __syncthreads();
  block_sort_desc(cand, kk, p.cap);
  for (uint32_t r = tid; r < kk; r += kScanThreads) {
    const uint2 e = cand[r];
    const uint32_t pos = kk - 1 - r;  // ascending output
    p.out_ids[pos] = (uint64_t)e.y;
    p.out_scores[pos] = key2f(e.x);
  }
  if (tid == 0) {
    if (p.out_threshold) *p.out_threshold = kk ? key2f(cand[kk - 1].x) : 0.0f;
    if (p.out_count) *p.out_count = kk;
    p.scratch->last_cands = total;
    p.scratch->last_reductions = ld_volatile_u32(&p.scratch->acc_reductions);
    if (p.out_stats) {
      p.out_stats[0] = total;
      p.out_stats[1] = p.scratch->last_reductions;
    }
    p.scratch->acc_reductions = 0;
    p.scratch->g_thr = 0;
    p.scratch->cand_count = 0;
    p.scratch->done = 0;
    __threadfence();
  }
}

template <int VEC, int R>
cudaError_t set_attr_one(size_t smem_optin) {
  return cudaFuncSetAttribute(scan_select_kernel<VEC, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_optin);
}

}  // namespace

cudaError_t scan_set_attributes(size_t smem_optin) {
  cudaError_t e;
#define TOPK_SET(V, R) \
  if ((e = set_attr_one<V, R>(smem_optin)) != cudaSuccess) return e;
  TOPK_SET(1, 8) TOPK_SET(1, 24) TOPK_SET(2, 8) TOPK_SET(2, 24) TOPK_SET(4, 16) TOPK_SET(4, 24)
#undef TOPK_SET
  return cudaSuccess;
}

ScanPlan plan_scan(uint32_t qq, uint32_t k, uint64_t rows, int num_sms, size_t smem_optin) {
  ScanPlan pl{};
  pl.vec = qq <= 8 ? 4 : (qq <= 16 ? 2 : 1);
  pl.tile = kScanThreads * pl.vec;
  uint32_t P = 1;
  while (P < k) P <<= 1;
  uint32_t cap = k + 2 * pl.tile;
  if (cap < P) cap = P;
  if (cap < 2048) cap = 2048;
  cap = (cap + kScanThreads - 1) / kScanThreads * kScanThreads;
  pl.cap = cap;
  const size_t fixed = kCtlBytes + kHistBytes + (size_t)cap * 8;
  const size_t stage_bytes = (size_t)qq * pl.tile * 4;
  size_t budget = smem_optin > fixed ? smem_optin - fixed : 0;
  uint32_t S = (uint32_t)(budget / stage_bytes);
  if (S > 8) S = 8;
  pl.stages = S;
  pl.smem = fixed + (size_t)S * stage_bytes;
  const uint64_t tiles = (rows + 3 + pl.tile) / pl.tile;
  uint64_t grid = (uint64_t)num_sms;
  if (grid > tiles) grid = tiles;
  if (grid < 1) grid = 1;
  pl.grid = (int)grid;
  return pl;
}

cudaError_t launch_scan(const ScanPlan &pl, const ScanParams &p, cudaStream_t stream) {
  const uint32_t R = (pl.cap + kScanThreads - 1) / kScanThreads;
  dim3 grid(pl.grid), block(kScanThreads);
  if (pl.vec == 1) {
    if (R <= 8) scan_select_kernel<1, 8><<<grid, block, pl.smem, stream>>>(p);
    else scan_select_kernel<1, 24><<<grid, block, pl.smem, stream>>>(p);
  } else if (pl.vec == 2) {
    if (R <= 8) scan_select_kernel<2, 8><<<grid, block, pl.smem, stream>>>(p);
    else scan_select_kernel<2, 24><<<grid, block, pl.smem, stream>>>(p);
  } else {
    if (R <= 16) scan_select_kernel<4, 16><<<grid, block, pl.smem, stream>>>(p);
    else scan_select_kernel<4, 24><<<grid, block, pl.smem, stream>>>(p);
  }
  return cudaGetLastError();
}

}  // namespace topk
