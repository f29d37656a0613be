// BF16 tensor-core filter of the batched path (tcgen05 + TMEM, sm_100a).
//
// For every (query, object) pair of a chunk the filter computes an approximate
// score on the 5th-generation tensor cores and keeps, per query, the objects whose
// approximate score can still reach the query's threshold.  batch_reduce_kernel
// (batch.cu) rescoring those candidates in the reference order (cpu/TPAc.h:135-150:
// s += x[attr[m]] * weights[attr[m]], FP32, no FMA) makes every kept key exact, so
// the results are bit-identical to the FP32 paths.
//
// Operands, both K-major without swizzle (core matrices of 8 rows x 16 bytes; the
// K-adjacent core matrix 128 B further on, the next 8 rows 256 B further on):
//   query  a 16-wide row a[m] = sum of weights[attr[j]] over the j with attr[j] = m,
//          split a = hi + lo (bf16 each, |a - hi - lo| <= 2^-16 |a|); tiles of 128
//          queries: hi 4 KB, then lo 4 KB                          (MMA A, M=128);
//   table  each object's 16 attributes split the same way; tiles of 256 objects:
//          hi 8 KB, then lo 8 KB                                    (MMA B, N=256).
// One (object tile, query tile) pair is three MMAs M=128 N=256 K=16 into FP32 TMEM
// (lane = query, column = object):
//   D = Ahi.Xhi + Ahi.Xlo + Alo.Xhi        (the lo.lo term lies inside the bound)
// Bound (host-computed per query, BatchQuery::err): |D - s_ref| <= E with
//   E = 2^-13 * sum_m |weights[attr[m]]| * max|column attr[m]|  (+ 2^-100 terms for
//   subnormal flushing).  Split and product errors give 3.1*2^-16, 48 FP32
//   accumulations 48*2^-22, the reference's own FP32 rounding 17*2^-24: about
//   2^-14 in all; the factor 2 covers the tensor core's accumulation rounding,
//   which is not specified (the largest error measured on rescored candidates is
//   below 2^-16 of the same sum).  An object with exact score >= the threshold
//   float t has D >= t - E, so the cut t - E (rounded down) loses none.
//
// Roles of the 576 threads of a CTA (one CTA per SM: TMEM is allocated whole):
//   warps 0-15 epilogue, two groups of eight: group g drains accumulator g (every
//              second pair); warp w reads TMEM lanes 32*(w%4).. (one query per
//              thread, its cut in a register) over half of the pair's 256 objects,
//              32 at a time: the largest value against the cut and a warp vote; for the
//              rare round trips with survivors each thread with a hit stores its 32
//              values as one record in the warp's own segment of the CTA's record
//              log in global memory (a count kept alike in every lane: no atomic and
//              no dependent work while the accumulator is held);
//   warp 16    producer: bulk-copies (cp.async.bulk, no tensor map, no multicast)
//              the CTA's query tiles once and object tiles into a 5-stage ring;
//   warp 17    allocates the 512 TMEM columns; lane 0 issues the MMAs into two
//              accumulators of 256 columns, one per epilogue group (at N=256 an MMA
//              takes longer to run than to issue, so one thread keeps the tensor
//              core busy).
// After the last tile the whole CTA expands its records into the queries' candidate
// regions: the values are compared with the cut again and the passing objects take
// their slots with one global atomic per record.  A record that finds its segment
// full flags its query for the exact single-query fallback.
// Every mbarrier wait is bounded; a wait that runs out sets the CTA's abort flag,
// every role leaves its loop, in-flight copies and MMAs are waited for (bounded),
// TMEM is freed and the error word is set (the host reports TOPK_ERR_TIMEOUT).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "batch_internal.h"
#include "block_select.cuh"
#include "device_common.cuh"

namespace topk {

namespace {

constexpr uint32_t kOTile = 256;         // objects per tile (MMA N, TMEM columns)
constexpr uint32_t kOTileBytes = 16384;  // hi + lo of one object tile
constexpr uint32_t kQTile = 128;         // queries per tile (MMA M, TMEM lanes)
constexpr uint32_t kQTileBytes = 8192;   // hi + lo of one query tile
constexpr uint32_t kStages = 5;
constexpr uint32_t kEpiWarps = 16;
constexpr uint32_t kProducerWarp = kEpiWarps, kMmaWarp = kEpiWarps + 1;
constexpr uint32_t kFThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kMaxQTPerCta = 16;
constexpr uint32_t kAcc = kTmemCols / kOTile;            // TMEM accumulators in flight
// Epilogue groups: group g drains the pairs seq = g mod kDrainGroups, so with two
// groups each accumulator has its own eight warps (4 round trips of 32 columns each).
// One group of all sixteen warps on every pair (2 round trips each) measured slower
// (C3 batch 34.1 against 31.7 ms): the drain is bound by its throughput, not by the
// latency of one warp's round trips.
constexpr uint32_t kDrainGroups = 2;
constexpr uint32_t kGroupWarps = kEpiWarps / kDrainGroups;  // epilogue warps draining one pair
constexpr uint32_t kWarpCols = kOTile * 4 / kGroupWarps;    // objects of one warp per pair
static_assert(kGroupWarps % 4 == 0 && kEpiWarps % kDrainGroups == 0, "whole TMEM lane quarters per group");
static_assert(kQTile == 128 && kWarpCols % 32 == 0, "a query per TMEM lane; whole 32-column round trips");
constexpr size_t kMinFilterSmem = 120 * 1024;  // more than half an SM: one CTA per SM

// Instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16 (bits
// 7-9 = 1, 10-12 = 1), both K-major, N>>3 at bits 17-22, M>>4 at bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((kOTile >> 3) << 17) | ((kQTile >> 4) << 24);

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B (K-adjacent
// core matrices), SBO 256 B (next 8 rows), version 1 (bit 46).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
         (1ull << 46);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

#define TOPK_R8(i) "=r"(v[i]), "=r"(v[i + 1]), "=r"(v[i + 2]), "=r"(v[i + 3]), "=r"(v[i + 4]), "=r"(v[i + 5]), \
                   "=r"(v[i + 6]), "=r"(v[i + 7])
// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t *v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : TOPK_R8(0), TOPK_R8(8), TOPK_R8(16), TOPK_R8(24)
      : "r"(taddr));
}
#undef TOPK_R8

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Largest of 32 FP32 values (three-input max, a tree of depth 4).  A NaN value is
// ignored, as a NaN also fails the compare it replaces.
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float max32(const uint32_t *v) {
  float m[11];
#pragma unroll
  for (int i = 0; i < 10; ++i)
    m[i] = max3f(__uint_as_float(v[3 * i]), __uint_as_float(v[3 * i + 1]), __uint_as_float(v[3 * i + 2]));
  m[10] = fmaxf(__uint_as_float(v[30]), __uint_as_float(v[31]));
  const float a = max3f(m[0], m[1], m[2]), b = max3f(m[3], m[4], m[5]), c = max3f(m[6], m[7], m[8]);
  return max3f(max3f(a, b, c), m[9], m[10]);
}

// Bounded wait that also gives up once another role of the CTA has aborted.
__device__ __forceinline__ bool fwait(uint64_t *bar, uint32_t parity, uint64_t limit, volatile uint32_t *abort_flag) {
  for (uint64_t it = 0; it < limit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 63u && *abort_flag) return false;
  }
  *abort_flag = 1u;
  return false;
}

struct FilterArgs {
  const uint8_t *xbf;  // object tiles (kOTileBytes each)
  const uint8_t *abf;  // query tiles (kQTileBytes each)
  const BatchQuery *qs;
  BatchState *st;
  uint2 *cand;
  uint4 *recv;         // per-CTA survivor records, rec_cap each: 32 FP32 values
                       // (8 x uint4) of one query over 32 consecutive objects
  uint2 *rech;         // and their headers: (first object, CTA-relative query)
  uint32_t rec_cap;
  const uint32_t *amap;  // compact query slot -> query (batch_active_kernel)
  const uint32_t *nact;  // active queries (slots 0..*nact-1), read when the kernel starts
  uint32_t qt_cap;       // query tiles of 128 per CTA at most
  uint64_t tile0, tile1;  // object tiles of the chunk
  uint64_t r1;            // rows >= r1 are never appended
  uint64_t wait_limit;
  uint32_t *err;
};

__global__ void __launch_bounds__(kFThreads, 1) bf16_filter_kernel(const FilterArgs p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  // Work split from the active query count: the chunk's active queries in tiles of
  // 128, the tiles in groups of at most qt_cap per CTA (balanced), each group's object
  // tiles split among cpg CTAs.  Every thread reads the same count, so the early
  // returns below are uniform over the block (no barrier or TMEM touched yet).
  const uint32_t nact = *p.nact;
  const uint32_t nqt_all = (nact + kQTile - 1) / kQTile;
  if (nqt_all == 0) return;
  const uint32_t ngroups = (nqt_all + p.qt_cap - 1) / p.qt_cap;
  const uint32_t QT = (nqt_all + ngroups - 1) / ngroups;
  const uint64_t ntiles = p.tile1 - p.tile0;
  const uint32_t cpg = (uint32_t)max((uint64_t)1, min(ntiles, (uint64_t)(gridDim.x / ngroups)));
  if (blockIdx.x >= ngroups * cpg) return;
  const uint32_t g = blockIdx.x % ngroups, c = blockIdx.x / ngroups;
  const uint32_t qt0 = g * QT;
  if (qt0 >= nqt_all) return;
  const uint32_t nqt = min(QT, nqt_all - qt0);
  const uint64_t per = (ntiles + cpg - 1) / cpg;
  const uint64_t tb = p.tile0 + (uint64_t)c * per;
  const uint64_t te = min(p.tile1, tb + per);
  if (tb >= te) return;

  // shared layout: query tiles | object ring | cut[QT*kQTile] | barriers and words
  unsigned char *sq = smem;
  unsigned char *so = smem + (size_t)p.qt_cap * kQTileBytes;
  float *scut = reinterpret_cast<float *>(so + (size_t)kStages * kOTileBytes);
  uint64_t *bars = reinterpret_cast<uint64_t *>(scut + p.qt_cap * kQTile);
  uint64_t *full = bars, *empty = bars + kStages, *accf = bars + 2 * kStages, *acce = accf + kAcc;
  uint64_t *qfull = acce + kAcc, *mdone = qfull + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mdone + 1);
  volatile uint32_t *abort_flag = tmem_slot + 1;
  uint32_t *wrec_n = tmem_slot + 2;  // records in each epilogue warp's segment
  const uint32_t seg_cap = p.rec_cap / kEpiWarps;
  uint4 *recv = p.recv + (size_t)blockIdx.x * p.rec_cap * 8u;
  uint2 *rech = p.rech + (size_t)blockIdx.x * p.rec_cap;
  const uint32_t q0 = qt0 * kQTile;  // first query slot of this CTA

  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t limit = p.wait_limit;
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < kStages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    for (uint32_t b = 0; b < kAcc; ++b) {
      mbar_init(accf + b, 1);
      mbar_init(acce + b, kGroupWarps);  // the epilogue warps that drain a pair
    }
    mbar_init(qfull, 1);
    mbar_init(mdone, 1);
    *abort_flag = 0u;
    for (uint32_t w = 0; w < kEpiWarps; ++w) wrec_n[w] = 0u;
    fence_barrier_init();
  }
  // per-slot cut: threshold float minus the bound, rounded down; +inf for slots past
  // the last active query, -inf while best[] is not full (every object is a candidate)
  for (uint32_t j = threadIdx.x; j < QT * kQTile; j += kFThreads) {
    const uint32_t sl = q0 + j;
    float cut = __int_as_float(0x7F800000);
    if (j < nqt * kQTile && sl < nact) {
      const uint32_t q = p.amap[sl];
      const BatchState sq_st = p.st[q];
      // the active list holds neither moved nor retired queries; a query moved to the
      // exact FP32 scorer since keeps +inf: nothing passes for it
      if (!(sq_st.flags & kFlagFp32))
        cut = sq_st.thr == 0u ? __int_as_float(0xFF800000) : __fsub_rd(thr_float(sq_st.thr), p.qs[q].err);
    }
    scut[j] = cut;
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kProducerWarp) {
    // ---------------------------------------------------------------- producer
    if (lane == 0) {
      mbar_arrive_expect_tx(qfull, nqt * kQTileBytes);
      for (uint32_t i = 0; i < nqt; ++i)
        bulk_g2s(sq + (size_t)i * kQTileBytes, p.abf + (size_t)(qt0 + i) * kQTileBytes, kQTileBytes, qfull);
      uint64_t it = 0;
      for (uint64_t t = tb; t < te; ++t, ++it) {
        const uint32_t s = (uint32_t)(it % kStages);
        if (it >= kStages && !fwait(empty + s, (uint32_t)((it / kStages - 1) & 1), limit, abort_flag)) break;
        mbar_arrive_expect_tx(full + s, kOTileBytes);
        bulk_g2s(so + (size_t)s * kOTileBytes, p.xbf + t * kOTileBytes, kOTileBytes, full + s);
      }
      // the CTA must not exit with copies in flight: wait for the last use of each stage
      const uint64_t first = it > kStages ? it - kStages : 0;
      for (uint64_t j = first; j < it; ++j)
        if (!mbar_wait_bounded(full + (j % kStages), (uint32_t)((j / kStages) & 1), limit)) *abort_flag = 1u;
      if (!mbar_wait_bounded(qfull, 0, limit)) *abort_flag = 1u;
    }
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      bool ok = fwait(qfull, 0, limit, abort_flag);
      uint64_t it = 0;
      uint32_t seq = 0;
      for (uint64_t t = tb; ok && t < te; ++t, ++it) {
        const uint32_t s = (uint32_t)(it % kStages);
        if (!fwait(full + s, (uint32_t)((it / kStages) & 1), limit, abort_flag)) break;
        tc_fence_after();
        const uint32_t os = smem_u32(so + (size_t)s * kOTileBytes);
        const uint64_t xhi = smem_desc(os), xlo = smem_desc(os + kOTileBytes / 2);
        for (uint32_t i = 0; i < nqt; ++i, ++seq) {
          const uint32_t buf = seq % kAcc;
          if (seq >= kAcc && !fwait(acce + buf, (seq / kAcc - 1) & 1u, limit, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t qsa = smem_u32(sq + (size_t)i * kQTileBytes);
          const uint64_t ahi = smem_desc(qsa), alo = smem_desc(qsa + kQTileBytes / 2);
          const uint32_t d = tmem + buf * kOTile;
          tc_mma(d, ahi, xhi, 0u);
          tc_mma(d, ahi, xlo, 1u);
          tc_mma(d, alo, xhi, 1u);
          tc_commit(accf + buf);
        }
        if (!ok) break;
        tc_commit(empty + s);  // the stage is free once these MMAs have read it
      }
      // TMEM is freed below: every issued MMA must have completed first
      tc_commit(mdone);
      if (!mbar_wait_bounded(mdone, 0, limit)) *abort_flag = 1u;
    }
  } else {
    // ---------------------------------------------------------------- epilogue
    // warps kGroupWarps*g.. drain the pairs seq = g mod kDrainGroups, pair seq in
    // accumulator seq mod kAcc.  Thread (warp w, lane l) owns TMEM lane 32*(w%4)+l, one
    // query of the pair's query tile, and reads kWarpCols of its objects in round trips
    // of 32 columns: one cut in a register, the largest value against it, a warp vote.
    const uint32_t quarter = warp & 3u, grp = warp / kGroupWarps, part = (warp % kGroupWarps) >> 2;
    const uint32_t tcol0 = tmem + ((quarter * 32u) << 16) + part * kWarpCols;
    // this warp's record segment and its fill, the same in every lane (no atomics)
    uint4 *wrecv = recv + (size_t)warp * seg_cap * 8u;
    uint2 *wrech = rech + (size_t)warp * seg_cap;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t wcnt = 0;
    const uint64_t npairs = (te - tb) * nqt;
    uint32_t qt = grp % nqt;       // query tile and
    uint64_t t = tb + grp / nqt;   // object tile of pair seq = t * nqt + qt
    for (uint64_t seq = grp; seq < npairs; seq += kDrainGroups) {
      const uint32_t buf = (uint32_t)(seq % kAcc), parity = (uint32_t)((seq / kAcc) & 1u);
      const uint32_t tcol = tcol0 + buf * kOTile;
      if (!__all_sync(0xFFFFFFFFu, fwait(accf + buf, parity, limit, abort_flag))) break;
      tc_fence_after();
      const uint32_t ql = qt * kQTile + quarter * 32u + lane;  // this thread's query, CTA-relative
      const float cut = scut[ql];
      const uint64_t obj0 = t * kOTile + part * kWarpCols;
#pragma unroll 1
      for (uint32_t rt = 0; rt < kWarpCols / 32u; ++rt) {
        uint32_t v[32];
        tmem_ld32(tcol + rt * 32u, v);
        tmem_wait_ld();
        if (rt + 1 == kWarpCols / 32u) {
          // the accumulator is free once its last columns are in registers
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(acce + buf);
        }
        // hot path: the largest of the 32 values against the thread's cut
        const float m = max32(v);
        const bool hit = m >= cut;
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, hit);
        if (b == 0u) continue;  // common case
        // cold path: each thread with a hit stores its 32 values as one record (eight
        // asynchronous 16-byte stores); which objects pass is worked out after the
        // pipeline, where no accumulator waits on it
        const uint32_t e = wcnt + __popc(b & lt_mask);
        wcnt += __popc(b);
        if (hit) {
          if (e < seg_cap) {
            uint4 *dst = wrecv + (size_t)e * 8u;
#pragma unroll
            for (int c = 0; c < 8; ++c) dst[c] = make_uint4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
            wrech[e] = make_uint2((uint32_t)(obj0 + rt * 32u), ql);
          } else {
            atomicOr(&p.st[p.amap[q0 + ql]].flags, kFlagOverflow);  // lost: the query moves to the exact scorer
          }
        }
      }
      qt += kDrainGroups;
      while (qt >= nqt) {
        qt -= nqt;
        ++t;
      }
    }
    if (lane == 0) wrec_n[warp] = min(wcnt, seg_cap);
  }

  // ---------------------------------------------------------------- teardown
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
  if (*abort_flag) {
    if (threadIdx.x == 0) atomicExch(p.err, 1u);
    return;
  }
  // the CTA's records into their queries' candidate regions: each thread takes a
  // record, compares its values with the query's cut again (the same cut, still in
  // shared memory) and reserves the passing objects' slots with one atomic
  for (uint32_t w = 0; w < kEpiWarps; ++w) {
    const uint32_t n = wrec_n[w];
    const uint4 *wv = recv + (size_t)w * seg_cap * 8u;
    const uint2 *wh = rech + (size_t)w * seg_cap;
    for (uint32_t e = threadIdx.x; e < n; e += kFThreads) {
      const uint2 h = wh[e];
      uint32_t v[32];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const uint4 x = wv[(size_t)e * 8u + c];
        v[4 * c] = x.x;
        v[4 * c + 1] = x.y;
        v[4 * c + 2] = x.z;
        v[4 * c + 3] = x.w;
      }
      const float cut = scut[h.y];
      uint32_t mask = 0;
#pragma unroll
      for (int j = 0; j < 32; ++j) mask |= (__uint_as_float(v[j]) >= cut ? 1u : 0u) << j;
      // objects past the table's last row (zero padding of the last tile) drop out
      const uint32_t nvalid = h.x >= p.r1 ? 0u : p.r1 - h.x >= 32u ? 32u : (uint32_t)(p.r1 - h.x);
      if (nvalid < 32u) mask &= (1u << nvalid) - 1u;
      if (!mask) continue;
      const uint32_t q = p.amap[q0 + h.y];
      uint32_t at = atomicAdd(&p.st[q].ccount, (uint32_t)__popc(mask));
      const BatchQuery &bq = p.qs[q];
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (mask & (1u << j)) {
          if (at < bq.cand_cap) p.cand[bq.cand_off + at] = make_uint2(f2key(__uint_as_float(v[j])), h.x + j);
          ++at;
        }
    }
  }
}

// ---------------------------------------------------------------- table split
// One thread per object (grid-stride): reads its 16 attributes (columns >= d and
// rows >= n are zero), writes hi and lo in the tiled core-matrix layout, and keeps
// per column the largest |x| bit pattern (NaN and inf show as >= 0x7F800000) and the
// largest and smallest order keys (NaN left out of both).
__global__ void __launch_bounds__(256) bf16_pack_kernel(const float *__restrict__ table, uint64_t ld, uint32_t d,
                                                        uint64_t n, uint64_t nobj, uint8_t *__restrict__ xbf,
                                                        uint32_t *__restrict__ ext) {
  uint32_t amax[16], kmax[16], kmin[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    amax[m] = 0u;
    kmax[m] = 0u;
    kmin[m] = 0xFFFFFFFFu;
  }
  for (uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nobj; o += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t hi[8], lo[8];
#pragma unroll
    for (int m = 0; m < 16; m += 2) {
      float x[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const bool in = (uint32_t)(m + e) < d && o < n;
        x[e] = in ? __ldg(table + (uint64_t)(m + e) * ld + o) : 0.0f;
        amax[m + e] = max(amax[m + e], __float_as_uint(x[e]) & 0x7FFFFFFFu);
        if (in && x[e] == x[e]) {
          const uint32_t k = f2key(x[e]);
          kmax[m + e] = max(kmax[m + e], k);
          kmin[m + e] = min(kmin[m + e], k);
        }
      }
      const __nv_bfloat16 h0 = __float2bfloat16_rn(x[0]), h1 = __float2bfloat16_rn(x[1]);
      const __nv_bfloat16 l0 = __float2bfloat16_rn(x[0] - __bfloat162float(h0));
      const __nv_bfloat16 l1 = __float2bfloat16_rn(x[1] - __bfloat162float(h1));
      hi[m / 2] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
      lo[m / 2] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    const uint64_t t = o / kOTile;
    const uint32_t r = (uint32_t)(o % kOTile);
    uint8_t *base = xbf + t * kOTileBytes + (r >> 3) * 256u + (r & 7u) * 16u;
    *reinterpret_cast<uint4 *>(base) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4 *>(base + 128) = make_uint4(hi[4], hi[5], hi[6], hi[7]);
    *reinterpret_cast<uint4 *>(base + kOTileBytes / 2) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    *reinterpret_cast<uint4 *>(base + kOTileBytes / 2 + 128) = make_uint4(lo[4], lo[5], lo[6], lo[7]);
  }
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    uint32_t a = amax[m], hk = kmax[m], lk = kmin[m];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a = max(a, __shfl_xor_sync(0xFFFFFFFFu, a, o));
      hk = max(hk, __shfl_xor_sync(0xFFFFFFFFu, hk, o));
      lk = min(lk, __shfl_xor_sync(0xFFFFFFFFu, lk, o));
    }
    if ((threadIdx.x & 31) == 0 && (uint32_t)m < d) {
      atomicMax(ext + m, a);
      atomicMax(ext + d + m, hk);
      atomicMin(ext + 2 * d + m, lk);
    }
  }
}

// ---------------------------------------------------------------- active queries
// One block, before each chunk's filter: lists the queries the filter still has to
// serve, in query order, as compact slots (amap[slot] = query, *nact = count), and
// copies each one's operand row (hi and lo, 64 bytes) from the batch's query tiles to
// its slot in the compact tiles.  A query is left out once it has moved to the exact
// FP32 scorer, or once its threshold is above the largest score any row can have
// (BatchQuery::maxkey: the reference-order FP32 sum over the column extremes, an
// exact upper bound because rounding is monotone) -- then no later row can enter its
// top-k.  This is the reference's stop rule (cpu/VTA.h:210-216, cpu/PTA.h:636-641:
// stop once the k-th score reaches the bound of what is left) with the whole table as
// the block.  The rows of the last tile past the count are zeroed.
constexpr uint32_t kActThreads = 1024;

__device__ __forceinline__ size_t qrow_off(uint32_t j) {  // query j's hi row in the tile layout
  return (size_t)(j / kQTile) * kQTileBytes + ((j % kQTile) >> 3) * 256u + (j & 7u) * 16u;
}

__global__ void __launch_bounds__(kActThreads) batch_active_kernel(const BatchQuery *__restrict__ qs,
                                                                 const BatchState *__restrict__ st, uint32_t nq,
                                                                 const uint8_t *__restrict__ abf,
                                                                 uint8_t *__restrict__ abf_act,
                                                                 uint32_t *__restrict__ amap,
                                                                 uint32_t *__restrict__ nact,
                                                                 uint32_t *__restrict__ nact_log) {
  __shared__ uint32_t wsum[kActThreads / 32];
  __shared__ uint32_t base;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  if (t == 0) base = 0;
  __syncthreads();
  for (uint32_t j0 = 0; j0 < nq; j0 += kActThreads) {
    const uint32_t j = j0 + t;
    bool act = false;
    if (j < nq) {
      const BatchState s = st[j];
      act = !(s.flags & kFlagFp32) && !(s.thr != 0u && s.thr > qs[j].maxkey);
    }
    const unsigned b = __ballot_sync(0xFFFFFFFFu, act);
    if (lane == 0) wsum[warp] = __popc(b);
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the 32 warp counts
      const uint32_t v = wsum[lane];
      uint32_t incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      wsum[lane] = incl - v;
    }
    __syncthreads();
    const uint32_t slot = base + wsum[warp] + __popc(b & ((1u << lane) - 1u));
    if (act) {
      amap[slot] = j;
      const uint4 *src = reinterpret_cast<const uint4 *>(abf + qrow_off(j));
      uint4 *dst = reinterpret_cast<uint4 *>(abf_act + qrow_off(slot));
      dst[0] = src[0];                      // hi, attributes 0-7
      dst[8] = src[8];                      // hi, attributes 8-15 (128 bytes on)
      dst[kQTileBytes / 32] = src[kQTileBytes / 32];          // lo
      dst[kQTileBytes / 32 + 8] = src[kQTileBytes / 32 + 8];
    }
    __syncthreads();
    if (t == kActThreads - 1) base = slot + (act ? 1u : 0u);
    __syncthreads();
  }
  const uint32_t total = base;
  for (uint32_t sl = total + t; sl < (total + kQTile - 1) / kQTile * kQTile; sl += kActThreads) {
    uint4 *dst = reinterpret_cast<uint4 *>(abf_act + qrow_off(sl));
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    dst[0] = z;
    dst[8] = z;
    dst[kQTileBytes / 32] = z;
    dst[kQTileBytes / 32 + 8] = z;
  }
  if (t == 0) {
    *nact = total;
    if (nact_log) *nact_log = total;
  }
}

}  // namespace

// ---------------------------------------------------------------- launchers
// query tiles | object ring | cuts | barriers and words
size_t filter_smem_bytes(uint32_t qt) {
  return (size_t)qt * (kQTileBytes + kQTile * 4) + (size_t)kStages * kOTileBytes + 512;
}

uint64_t bf16_table_bytes(uint64_t n) { return (n + kOTile - 1) / kOTile * kOTileBytes; }

cudaError_t launch_bf16_pack(const float *table, uint64_t ld, uint32_t d, uint64_t n, uint8_t *xbf, uint32_t *ext,
                             int num_sms, cudaStream_t s) {
  if (d > kBf16MaxD) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(ext, 0, 2 * d * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(ext + 2 * d, 0xFF, d * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  const uint64_t nobj = (n + kOTile - 1) / kOTile * kOTile;
  const uint64_t blocks = std::min<uint64_t>((nobj + 255) / 256, (uint64_t)num_sms * 8);
  bf16_pack_kernel<<<(unsigned)blocks, 256, 0, s>>>(table, ld, d, n, nobj, xbf, ext);
  return cudaGetLastError();
}

size_t bf16_query_bytes(uint32_t nq) { return (size_t)((nq + kQTile - 1) / kQTile) * kQTileBytes; }

void bf16_pack_query(const float *a, uint32_t j, uint8_t *abf) {
  auto f2bf = [](float f) -> uint16_t {  // round to nearest even (finite inputs)
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
  };
  auto bf2f = [](uint16_t b) -> float {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
  };
  const uint32_t tile = j / kQTile, r = j % kQTile;
  uint8_t *base = abf + (size_t)tile * kQTileBytes + (r >> 3) * 256u + (r & 7u) * 16u;
  for (uint32_t m = 0; m < kBf16MaxD; ++m) {
    const uint16_t h = f2bf(a[m]);
    const volatile float res = a[m] - bf2f(h);  // exact: hi is within a factor 2 of a[m]
    const uint16_t l = f2bf(res);
    const size_t off = (m >> 3) * 128u + (m & 7u) * 2u;
    __builtin_memcpy(base + off, &h, 2);
    __builtin_memcpy(base + kQTileBytes / 2 + off, &l, 2);
  }
}

FilterPlan plan_bf16_filter(uint32_t nq, uint64_t r0, uint64_t r1, int num_sms, uint32_t qt_cap) {
  FilterPlan f{};
  f.tile0 = r0 / kOTile;
  f.tile1 = (r1 + kOTile - 1) / kOTile;
  const uint32_t nqt = (nq + kQTile - 1) / kQTile;
  f.qt_cap = (qt_cap >= 1 && qt_cap < kMaxQTPerCta) ? qt_cap : kMaxQTPerCta;
  // enough CTAs for every group the active count can need, and at least one per SM
  const uint64_t groups = (nqt + f.qt_cap - 1) / f.qt_cap;
  f.grid = std::max<uint64_t>((uint64_t)std::max(1, num_sms), groups);
  return f;
}

cudaError_t launch_bf16_filter(const FilterPlan &f, const uint8_t *xbf, const uint8_t *abf, const uint32_t *amap,
                               const uint32_t *nact, uint64_t r0, uint64_t r1, const BatchQuery *qs, BatchState *st,
                               uint2 *cand, uint4 *recv, uint2 *rech, uint32_t rec_cap, uint64_t wait_limit,
                               uint32_t *err, cudaStream_t s) {
  if (r0 % kOTile || f.grid == 0 || f.grid > 0x7FFFFFFFull) return cudaErrorInvalidValue;
  FilterArgs p{};
  p.xbf = xbf;
  p.abf = abf;
  p.qs = qs;
  p.st = st;
  p.cand = cand;
  p.recv = recv;
  p.rech = rech;
  p.rec_cap = rec_cap;
  p.amap = amap;
  p.nact = nact;
  p.qt_cap = f.qt_cap;
  p.tile0 = f.tile0;
  p.tile1 = f.tile1;
  p.r1 = r1;
  p.wait_limit = wait_limit;
  p.err = err;
  const size_t smem = std::max(kMinFilterSmem, filter_smem_bytes(f.qt_cap));
  cudaError_t e = cudaFuncSetAttribute(bf16_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  bf16_filter_kernel<<<(unsigned)f.grid, kFThreads, smem, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_batch_active(const BatchQuery *qs, const BatchState *st, uint32_t nq, const uint8_t *abf,
                                uint8_t *abf_act, uint32_t *amap, uint32_t *nact, uint32_t *nact_log,
                                cudaStream_t s) {
  batch_active_kernel<<<1, kActThreads, 0, s>>>(qs, st, nq, abf, abf_act, amap, nact, nact_log);
  return cudaGetLastError();
}

}  // namespace topk
