// Fused single-query scan + exact top-k select (sm_100a).
//
// Replaces the TPAc full-table evaluation (cpu/TPAc.h:118-207 findTopKsimd,
// :257-358 findTopKthreads): the same per-object arithmetic
//     s = 0; for m in attr order: s = s + x[attr[m]] * w[attr[m]]   (RN mul, RN add)
// and the same result (the k best by score; ties here go to the lower id).
//
// Persistent CTAs of 256 threads, several per SM:
//   * Each tile is 1024 objects (4 per thread).  A thread issues one 128-bit
//     streaming load (ld.global.cs) per queried column for its 4 objects, all of
//     them before the first multiply, so each warp keeps q x 512 bytes in flight and
//     an SM with several CTAs keeps far more than the ~45 KB that HBM3e latency
//     needs.  Only the queried columns are read.  (A TMA bulk-copy ring with a
//     producer warp was measured on this GPU at 2.6-4.9 TB/s against 3.1-5.9 TB/s
//     for plain loads, so the scan uses plain loads.)  For q <= 4 a thread also keeps
//     the next tile's loads in flight while it scores, appends and synchronises on
//     the current one, and loads a partial tile's rows past its end from row 0 (in
//     bounds, masked out) instead of selecting zeros value by value (q = 2: 3.3 ->
//     3.6 TB/s; q = 4: 4.5 -> 5.5 TB/s, same-box A/B).
//   * An object passes if its score is >= the running threshold; passing objects
//     go to a shared candidate buffer (warp-aggregated append).  When the buffer
//     nears capacity (a barrier vote, so every thread decides alike) the CTA keeps
//     its top-k by an 8-bit radix select on the 64-bit (key, ~id) word, raises its
//     own threshold and publishes its k-th key with atomicMax to a global word that
//     every CTA folds into its filter.  Any CTA's k-th best lower-bounds the global
//     k-th best, so nothing that can win is dropped.
//   * End: a merge tree with fan-in G.  Each CTA writes its survivors to a slot; the
//     last CTA of each group of G slots (per-group arrival counter) merges them to k
//     entries in shared memory and moves up; the root sorts (bitonic) and writes the
//     result.  Counters are put back to zero for the next query.
#include <cstdint>
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "block_select.cuh"
#include "device_common.cuh"
#include "topk_internal.h"

namespace topk {

namespace {

struct SmemCtl {
  uint32_t count;      // entries in the current candidate buffer
  uint32_t thr_local;  // min key that can still enter (k-th CTA key + 1)
  uint32_t thr_g[2];   // CTA copy of the global threshold: tile i reads [i & 1], thread 0
                       // writes [(i + 1) & 1] before tile i's barrier, so with a vote
                       // barrier every tile (partition mode, whose stop rule needs it)
                       // every thread of a tile reads the same value; with a vote every
                       // two tiles a thread may read a slot before or after an update,
                       // both valid bounds
  uint32_t reductions;
  uint32_t is_last;
  uint32_t red_g;      // threshold snapshot shared by the block
  SelShared sel;       // state of the block-wide selects
};

// shared layout
constexpr int kOffCtl = 0;        // SmemCtl (80 B)
constexpr int kOffNever = 96;     // test barrier (u64)
constexpr int kOffHist = 128;     // 256-bin radix histogram
constexpr int kOffWsm = 1152;     // weights of the runtime-q path (kMaxQ floats)
constexpr int kOffScnt = 1408;    // entry counts of a merge group's slots (kMaxFanin words)
constexpr int kOffCand = kScanSmemFixed;
constexpr uint32_t kMaxFanin = 32;  // merge-tree fan-in at most (small k: two levels for 592 CTAs)
static_assert(kOffWsm + 4 * (int)kMaxQ <= kOffScnt && kOffScnt + 4 * (int)kMaxFanin <= kScanSmemFixed,
              "fixed shared block");
static_assert(sizeof(SmemCtl) <= kOffNever, "control block layout");
static_assert(kScanThreads == 256, "one histogram bin per thread");

constexpr int kVec = 4;                      // objects per thread per tile
constexpr uint32_t kTile = kScanThreads * kVec;

__device__ __forceinline__ void bsync() { __syncthreads(); }

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
#define TOPK_CHECK(cond, code, i, a, b) check((cond), p.scratch, (code), (i), (a), (b))
#else
#define TOPK_CHECK(cond, code, i, a, b) (true)
#endif

__device__ __forceinline__ float4 ld_stream(const float *p) { return __ldcs(reinterpret_cast<const float4 *>(p)); }

// Scores of this thread's 4 objects at rows [row0, row0+4) of one tile, reference
// order.  QQ > 0: compile-time attribute count, every load issued before the first
// multiply, weights as constant-bank operands.  QQ == 0: runtime count, weights
// from shared memory.  `guard`: partial tile, load only below tile_end.
template <int QQ>
__device__ __forceinline__ float4 score4(const ScanParams &p, const float *wsm, uint32_t qq, uint64_t row0,
                                         bool guard) {
  float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
  const bool inb = !guard || row0 < p.tile_end;  // tile_end <= ld, multiple of 4
  if constexpr (QQ > 0) {
    float4 x[QQ];
#pragma unroll
    for (int m = 0; m < QQ; ++m)
      x[m] = inb ? ld_stream(p.table + (uint64_t)p.attr[m] * p.ld + row0) : make_float4(0.f, 0.f, 0.f, 0.f);
    // every load is issued before the first multiply (the compiler may not sink them
    // below this point): QQ x 16 bytes in flight per thread
    asm volatile("" ::: "memory");
#pragma unroll
    for (int m = 0; m < QQ; ++m) {
      const float w = p.w[m];
      a0 = __fadd_rn(a0, __fmul_rn(x[m].x, w));
      a1 = __fadd_rn(a1, __fmul_rn(x[m].y, w));
      a2 = __fadd_rn(a2, __fmul_rn(x[m].z, w));
      a3 = __fadd_rn(a3, __fmul_rn(x[m].w, w));
    }
  } else {
    uint32_t m = 0;
    for (; m + 4 <= qq; m += 4) {  // four loads in flight at a time
      float4 x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        x[u] = inb ? ld_stream(p.table + (uint64_t)p.attr[m + u] * p.ld + row0) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float w = wsm[m + u];
        a0 = __fadd_rn(a0, __fmul_rn(x[u].x, w));
        a1 = __fadd_rn(a1, __fmul_rn(x[u].y, w));
        a2 = __fadd_rn(a2, __fmul_rn(x[u].z, w));
        a3 = __fadd_rn(a3, __fmul_rn(x[u].w, w));
      }
    }
    for (; m < qq; ++m) {
      const float4 x = inb ? ld_stream(p.table + (uint64_t)p.attr[m] * p.ld + row0) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float w = wsm[m];
      a0 = __fadd_rn(a0, __fmul_rn(x.x, w));
      a1 = __fadd_rn(a1, __fmul_rn(x.y, w));
      a2 = __fadd_rn(a2, __fmul_rn(x.z, w));
      a3 = __fadd_rn(a3, __fmul_rn(x.w, w));
    }
  }
  return make_float4(a0, a1, a2, a3);
}

// Loads of this thread's 4 objects at rows [row0, row0+4) in the QQ queried columns,
// and their scores in reference order.  `guard`: partial tile; a thread whose rows
// lie at or past tile_end loads row 0 instead (always in bounds) and its scores are
// meaningless — the caller's row-range mask drops them.  One select per tile, none
// per value, and the column pointers computed once by the caller.
template <int QQ>
__device__ __forceinline__ void load_cols(const ScanParams &p, const float *const *col, uint64_t row0, bool guard,
                                          float4 *x) {
  row0 = (!guard || row0 < p.tile_end) ? row0 : 0;
#pragma unroll
  for (int m = 0; m < QQ; ++m) x[m] = ld_stream(col[m] + row0);
}
template <int QQ>
__device__ __forceinline__ float4 score_cols(const ScanParams &p, const float4 *x) {
  float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
#pragma unroll
  for (int m = 0; m < QQ; ++m) {
    const float w = p.w[m];
    a0 = __fadd_rn(a0, __fmul_rn(x[m].x, w));
    a1 = __fadd_rn(a1, __fmul_rn(x[m].y, w));
    a2 = __fadd_rn(a2, __fmul_rn(x[m].z, w));
    a3 = __fadd_rn(a3, __fmul_rn(x[m].w, w));
  }
  return make_float4(a0, a1, a2, a3);
}

// Up to this many queried columns the scan keeps the next tile's loads in flight
// while it scores, appends and synchronises on the current one (few columns give a
// thread too few bytes in flight otherwise).
constexpr int kPrefetchQ = 4;

// Tiles between two select votes of the scan (see scan_select_kernel).
__host__ __device__ constexpr uint32_t scan_vote_tiles(int qq, bool part) {
  return (qq >= 1 && qq <= 2 && !part) ? 2u : 1u;
}

// CTAs per SM the register budget is sized for: few queried columns need little data
// in flight and gain from more CTAs (6: 42 registers); more columns need their loads
// in flight without spills (5: 51 registers up to 8 columns, 4: 64 above).
template <int QQ>
constexpr int scan_min_blocks() {
  return (QQ >= 1 && QQ <= 2) ? 6 : (QQ >= 3 && QQ <= 8) ? 5 : 4;
}

// QQ: compile-time attribute count (0 = runtime, any qq <= kMaxQ).  PART: partition
// mode (p.part_list set): tiles of listed partitions of a reordered copy.  KTH: a
// threshold pass (p.kth_only, p.pub set): no candidate buffer, no select and no merge;
// each thread keeps the best kPubMaxPerWarp (key, row) words of its own objects in
// registers, each warp publishes its best pub_m / 8 of them, and the last CTA writes
// the k-th largest published key.
template <int QQ, bool PART, bool KTH>
__global__ void __launch_bounds__(kScanThreads, scan_min_blocks<QQ>()) scan_select_kernel(const __grid_constant__ ScanParams p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  SmemCtl *ctl = reinterpret_cast<SmemCtl *>(smem + kOffCtl);
  uint64_t *never = reinterpret_cast<uint64_t *>(smem + kOffNever);
  uint32_t *hist = reinterpret_cast<uint32_t *>(smem + kOffHist);
  float *wsm = reinterpret_cast<float *>(smem + kOffWsm);
  uint32_t *scnt = reinterpret_cast<uint32_t *>(smem + kOffScnt);
  // the candidate buffer (cap entries), then the select's output (the rest of mcap);
  // the merge reuses both
  uint2 *cand0 = reinterpret_cast<uint2 *>(smem + kOffCand);
  uint2 *selb = cand0 + p.cap;
  uint2 *mbuf = cand0;

  const int t = threadIdx.x;
  const int lane = t & 31;
  const uint32_t qq = QQ > 0 ? (uint32_t)QQ : p.qq;
  const uint32_t cap = p.cap;
  const uint32_t my_tiles =
      blockIdx.x < p.num_tiles ? (p.num_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

  if (QQ == 0 && t < (int)kMaxQ && t < (int)qq) wsm[t] = p.w[t];
  if (t == 0) {
    mbar_init(never, 1);
    fence_barrier_init();
    ctl->count = 0;
    ctl->thr_local = 0;
    const uint32_t seed = max(p.thr_seed, p.thr_seed_dev ? *p.thr_seed_dev : 0u);
    if (seed) atomicMax(&p.scratch->g_thr, seed);  // every later read includes it
    // both slots hold a valid bound from the start: with two tiles per vote a thread
    // can read the second slot before thread 0's first copy into it
    ctl->thr_g[0] = ctl->thr_g[1] = max(ld_volatile_u32(&p.scratch->g_thr), seed);
    ctl->reductions = 0;
  }
  bsync();

  if (p.fault_mode == 1) {
    // Test hook: wait on a barrier that nothing arrives on.  The bounded wait runs
    // out and the scan reports a timeout; nothing else is in flight.
    const bool ok = mbar_wait_bounded(never, 0, p.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (t == 0) atomicOr(&p.scratch->error, 1u);
      return;
    }
  }

  uint32_t g_pending = 0;  // thread 0's in-flight copy of the global threshold
  // next-tile prefetch: the loads of tile i + 1 are in flight while tile i is scored
  constexpr int kPQ = (QQ >= 1 && QQ <= kPrefetchQ) ? QQ : 1;
  constexpr bool prefetch = QQ >= 1 && QQ <= kPrefetchQ;
  // queried columns of the prefetching forms: read from the parameter block (colp), no
  // registers held
  // partition mode: the partitions (and bounds) of tiles i and i + 1 are known at the
  // start of tile i, the one of tile i + 2 is loaded during it
  const uint32_t pmask = (1u << p.part_shift) - 1u;
  uint32_t part_cur = 0, key_cur = 0xFFFFFFFFu, part_nx = 0, key_nx = 0xFFFFFFFFu;
  auto part_of = [&](uint32_t j, uint32_t &part, uint32_t &key) {
    const uint64_t x = ((uint64_t)blockIdx.x + (uint64_t)j * gridDim.x) >> p.part_shift;
    part = __ldg(p.part_list + x);
    if (p.part_key) key = __ldg(p.part_key + x);
  };
  if (PART) {
    if (my_tiles > 0) part_of(0, part_cur, key_cur);
    if (my_tiles > 1) part_of(1, part_nx, key_nx);
  }
  auto tile_row = [&](uint32_t j, uint32_t part) -> uint64_t {  // first row of tile j of this CTA
    const uint64_t tix = blockIdx.x + (uint64_t)j * gridDim.x;
    if constexpr (PART) return ((uint64_t)part << p.part_rows_log2) + (tix & pmask) * kTile;
    return p.tile_begin + tix * p.tile_step;
  };
  auto load_rows = [&](uint64_t tl, float4 *dst) {  // the tile that starts at row tl
    const float *c[kPQ];
#pragma unroll
    for (int m = 0; m < kPQ; ++m) c[m] = p.colp[m];
    load_cols<kPQ>(p, c, tl + (uint64_t)t * kVec, !(tl >= p.row_begin && tl + kTile <= p.row_end), dst);
  };
  // id order with prefetch: first row and index of the tile whose loads went out last;
  // tile j lies wholly inside [row_begin, row_end) iff j - int_lo < int_n (unsigned)
  uint64_t next_row = p.tile_begin + (uint64_t)blockIdx.x * p.tile_step;
  uint32_t next_tix = blockIdx.x;
  auto load_next = [&](float4 *dst) {
    const uint64_t r = next_row + (uint64_t)t * kVec;
    const bool inner = next_tix - p.int_lo < p.int_n;
    load_cols<kPQ>(p, p.colp, r, !inner, dst);
  };
  float4 xn[kPQ];
  if (prefetch && my_tiles) {
    if constexpr (PART) load_rows(tile_row(0, part_cur), xn);
    else load_next(xn);
  }
  // tiles between two select votes: 2 for q <= 2 in id order (a thread's work per tile
  // is small there and the vote's barrier was the top stall), 1 elsewhere; the buffer
  // has room for that many tiles above its select mark (plan_scan)
  constexpr uint32_t kVoteTiles = scan_vote_tiles(QQ, PART);
  uint32_t after = 0;  // fill after this thread's warp last appended, since the last vote
  uint64_t kbest[KTH ? kPubMaxPerWarp : 1];  // KTH: this thread's best words, descending
#pragma unroll
  for (int b = 0; b < (KTH ? (int)kPubMaxPerWarp : 1); ++b) kbest[b] = 0ull;
  uint32_t i = 0;  // after the loop: the tiles this CTA scanned
  // q <= 2 in id order: two tiles per loop pass, so the prefetched registers swap roles
  // instead of being copied (q = 2 on 2^28 rows: 0.420 -> 0.406 ms)
  constexpr int kUnroll = kVoteTiles == 2 ? 2 : 1;
#pragma unroll(kUnroll)
  for (; i < my_tiles; ++i) {
    // every thread reads the same thresholds in tile i (see SmemCtl::thr_g); in id
    // order they are read after the scores, so they hold no register across the loads
    uint32_t thr = 0;
    if constexpr (PART && !KTH) {
      thr = max(ctl->thr_local, ctl->thr_g[i & 1u]);
      // nothing in this partition (nor in any later one of this CTA) can reach thr
      if (key_cur < thr) break;
    }
    const uint64_t tile0 = (prefetch && !PART) ? next_row : tile_row(i, part_cur);
    const uint64_t row0 = tile0 + (uint64_t)t * kVec;
    const bool interior = (prefetch && !PART) ? next_tix - p.int_lo < p.int_n
                                              : tile0 >= p.row_begin && tile0 + kTile <= p.row_end;  // uniform
    float4 s;
    if (prefetch) {
      float4 x[kPQ];
#pragma unroll
      for (int m = 0; m < kPQ; ++m) x[m] = xn[m];
      if (i + 1 < my_tiles) {
        if constexpr (PART) {
          load_rows(tile_row(i + 1, part_nx), xn);
        } else {
          next_row += p.grid_rows;
          next_tix += gridDim.x;
          load_next(xn);
        }
      }
      s = score_cols<kPQ>(p, x);
    } else {
      s = score4<QQ>(p, wsm, qq, row0, !interior);
    }
    if constexpr (PART) {
      part_cur = part_nx;
      key_cur = key_nx;
      if (i + 2 < my_tiles) part_of(i + 2, part_nx, key_nx);
    }

    if constexpr (KTH) {
      // a threshold pass: every object of the tile against this thread's best words
      const float sk[4] = {s.x, s.y, s.z, s.w};
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const bool ok = interior || (row0 + v >= p.row_begin && row0 + v < p.row_end);
        uint64_t c = ok ? composite(f2key(sk[v]), (uint32_t)(row0 + v)) : 0ull;
#pragma unroll
        for (int b = 0; b < (int)kPubMaxPerWarp; ++b)
          if (c > kbest[b]) {
            const uint64_t x = kbest[b];
            kbest[b] = c;
            c = x;
          }
      }
      continue;
    }
    if constexpr (!PART) thr = max(ctl->thr_local, ctl->thr_g[i & 1u]);
    // key(score) >= thr  <=>  thr == 0 (everything, NaN included) or score >= thr_float(thr)
    const bool take_all = thr == 0u;
    const float thr_f = thr_float(thr);
    const float sv[4] = {s.x, s.y, s.z, s.w};
    unsigned pass_mask = 0;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      bool pv = take_all || sv[v] >= thr_f;
      if (!interior) pv = pv && row0 + v >= p.row_begin && row0 + v < p.row_end;
      pass_mask |= (unsigned)pv << v;
    }
    // `after` = fill after this warp's append.  The warp that appends last before a
    // vote sees the final count, so OR-voting "after > cap - kVoteTiles * TILE" at the
    // barrier gives every thread the same reduce decision.  (Reading ctl->count after
    // a barrier would not: a fast warp may already be appending the next tile.)
    if (__ballot_sync(0xFFFFFFFFu, pass_mask != 0u)) {  // warp-uniform: some lane passed
      uint2 *cand = cand0;
      const uint32_t npass = __popc(pass_mask);
      uint32_t incl = npass;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      const uint32_t wtotal = __shfl_sync(0xFFFFFFFFu, incl, 31);
      uint32_t base = 0;
      if (lane == 31) base = atomicAdd(&ctl->count, wtotal);
      base = __shfl_sync(0xFFFFFFFFu, base, 31);
      after = base + wtotal;
      base += incl - npass;
#pragma unroll
      for (int v = 0; v < 4; ++v)
        if (pass_mask & (1u << v)) {
          if (TOPK_CHECK(base < cap, kDiagAppend, i, base, cap))
            cand[base] = make_uint2(f2key(sv[v]), p.row_ids ? __ldg(p.row_ids + row0 + v) : (uint32_t)(row0 + v));
          ++base;
        }
    }
    // thread 0 hands the CTA its copy of the global threshold (see SmemCtl::thr_g): it
    // loads the global word every 8 tiles and applies it 7 tiles later, so the L2 round
    // trip is never waited on.  The new value goes to the slot the next tile reads, and
    // on the tile after into the other slot too; between updates both slots agree.
    if (t == 0) {
      if ((i & 7u) == 7u) ctl->thr_g[(i + 1u) & 1u] = max(ctl->thr_g[i & 1u], g_pending);
      if ((i & 7u) == 0u) {
        ctl->thr_g[(i + 1u) & 1u] = ctl->thr_g[i & 1u];
        g_pending = ld_volatile_u32(&p.scratch->g_thr);
      }
    }
    // (uniform: every thread takes the same votes)
    if (kVoteTiles > 1 && (i % kVoteTiles) != kVoteTiles - 1 && i + 1 < my_tiles) continue;
    const bool full = __syncthreads_or(after > cap - kVoteTiles * kTile);
    after = 0;
    if (full) {
      if (t == 0) ctl->red_g = ld_volatile_u32(&p.scratch->g_thr);
      bsync();
      // the best k into the output area, then back to the front of the buffer
      const uint32_t kept = block_reduce<kScanThreads>(cand0, ctl->count, selb, p.k, ctl->red_g, hist, &ctl->sel);
      for (uint32_t j = t; j < kept; j += kScanThreads) cand0[j] = selb[j];
      if (t == 0) {
        ctl->count = kept;
        ctl->reductions++;
        if (kept == p.k) {  // the CTA knows a k-th key
          // Rows in id order: a later row has a larger id and loses a tie with the
          // k-th, so it must beat it strictly.  Rows carrying their own ids (a
          // reordered copy) may win the tie: the threshold stays inclusive.
          ctl->thr_local = ctl->sel.kept_min + (p.row_ids ? 0u : 1u);
          atomicMax(&p.scratch->g_thr, ctl->sel.kept_min);
        }
      }
      bsync();
    }
  }

  // ---- end of scan: reduce to <= k (a threshold pass publishes from its buffer as is) ----
  bsync();
  if (t == 0) ctl->red_g = ld_volatile_u32(&p.scratch->g_thr);
  bsync();
  if (!KTH && ctl->count > p.k && !p.kth_only) {
    const uint32_t kept = block_reduce<kScanThreads>(cand0, ctl->count, selb, p.k, ctl->red_g, hist, &ctl->sel);
    for (uint32_t j = t; j < kept; j += kScanThreads) cand0[j] = selb[j];
    if (t == 0) {
      ctl->count = kept;
      ctl->reductions++;
      if (kept == p.k) atomicMax(&p.scratch->g_thr, ctl->sel.kept_min);
    }
    bsync();
  }
  if (t == 0 && ctl->reductions) atomicAdd(&p.scratch->acc_reductions, ctl->reductions);
  if (PART && t == 0) atomicAdd(&p.scratch->acc_tiles, i);

  // ---- a tight bound before the merge (p.pub set: large k) ----
  // Each CTA's own k-th key is a weak bound of the global k-th (the best of one CTA's
  // share), so without more every CTA would pass ~k entries up the merge tree.  Each
  // CTA publishes the keys of its best M = pub_m entries; the last to arrive takes the
  // k-th largest of all published keys -- k real objects score at least that, so it is
  // a lower bound of the global k-th, close to it when the best objects are spread over
  // the CTAs -- and raises the global threshold to it; the others wait for that (a
  // bounded wait: if it runs out they go on with the threshold they have, which is
  // still exact, only slower) and the merge tree then carries about k entries in all.
  if (KTH || p.pub) {
    const uint2 *res0 = cand0;
    // Each warp publishes the best r = pub_m / 8 entries of its share of the buffer
    // (entries j = t, t + 256, ...): every thread keeps its own best r, then r rounds of
    // a warp maximum, each taken from the lane that holds it.  The CTA's pub_m keys are
    // the best of 8 disjoint shares -- keys of distinct real objects, which is all the
    // bound needs.  Unused places publish key 0.
    {
      constexpr int kR = kPubMaxPerWarp;
      const uint32_t r = p.pub_m / 8u;
      const uint32_t n = ctl->count;
      uint64_t best[kR];
#pragma unroll
      for (int i = 0; i < kR; ++i) best[i] = KTH ? kbest[i] : 0ull;
      for (uint32_t j = t; !KTH && j < n; j += kScanThreads) {
        const uint2 e = res0[j];
        uint64_t c = composite(e.x, e.y);
#pragma unroll
        for (int i = 0; i < kR; ++i)  // insertion into the descending list
          if (c > best[i]) {
            const uint64_t x = best[i];
            best[i] = c;
            c = x;
          }
      }
      uint2 *mine = p.pub + (size_t)blockIdx.x * p.pub_m + (size_t)(t >> 5) * r;
      for (uint32_t i = 0; i < r; ++i) {
        uint64_t m = best[0];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const uint64_t y = __shfl_xor_sync(0xFFFFFFFFu, m, o);
          m = y > m ? y : m;
        }
        if (m != 0ull && best[0] == m) {  // the one lane that holds it pops it
#pragma unroll
          for (int x = 0; x + 1 < kR; ++x) best[x] = best[x + 1];
          best[kR - 1] = 0ull;
        }
        // (key, place): distinct entries even for padding
        if (lane == 0) mine[i] = make_uint2((uint32_t)(m >> 32), blockIdx.x * p.pub_m + (t >> 5) * r + i);
      }
    }
    __threadfence();
    bsync();
    if (t == 0) ctl->is_last = atomicAdd(&p.scratch->pub_arrived, 1u) == gridDim.x - 1u ? 1u : 0u;
    bsync();
    if ((KTH || p.kth_only) && !ctl->is_last) return;  // a threshold pass: only the last CTA goes on
    if (ctl->is_last) {
      __threadfence();
      // the k-th largest published key; entries of key 0 are padding (or NaN scores,
      // the lowest anyway): left out.  The keys go to this CTA's free candidate space
      // first (independent loads, kStageBatch in flight per thread), so the select's
      // five passes read shared memory, not L2.
      const uint32_t np = gridDim.x * p.pub_m;
      // (a threshold pass has no candidates; a scan's <= k sit at the buffer's front)
      uint32_t *stage = reinterpret_cast<uint32_t *>(KTH ? cand0 : cand0 + p.k);
      const uint32_t stage_cap = KTH ? 2u * p.mcap : 2u * (p.mcap - p.k);
      uint32_t kth;
      if (np <= stage_cap) {
        constexpr int kStageBatch = 8;
        for (uint32_t base = 0; base < np; base += kScanThreads * kStageBatch) {
          uint32_t v[kStageBatch];
#pragma unroll
          for (int u = 0; u < kStageBatch; ++u) {
            const uint32_t j = base + (uint32_t)u * kScanThreads + t;
            v[u] = j < np ? __ldcg(&p.pub[j].x) : 0u;
          }
#pragma unroll
          for (int u = 0; u < kStageBatch; ++u) {
            const uint32_t j = base + (uint32_t)u * kScanThreads + t;
            if (j < np) stage[j] = v[u];
          }
        }
        bsync();
        kth = block_kth_key<kScanThreads>(KeySrc{stage}, np, 1u, p.k, hist, &ctl->sel);
      } else {
        kth = block_kth_key<kScanThreads>(SmemSrc{p.pub}, np, 1u, p.k, hist, &ctl->sel);
      }
      if (KTH || p.kth_only) {
        // the bound is the pass's result; every other CTA has left: put the counters back
        if (t == 0) {
          *p.out_kth_key = kth;
          p.scratch->g_thr = 0;
          p.scratch->acc_reductions = 0;
          p.scratch->acc_tiles = 0;
          p.scratch->pub_arrived = 0;
          p.scratch->pub_ready = 0;
          __threadfence();
        }
        return;
      }
      if (t == 0) {
        if (kth) atomicMax(&p.scratch->g_thr, kth);
        __threadfence();
        atomicExch(&p.scratch->pub_ready, 1u);
      }
    } else if (t == 0) {
      for (uint32_t it = 0; it < p.pub_wait && !ld_volatile_u32(&p.scratch->pub_ready); ++it) __nanosleep(64);
      __threadfence();  // the raised g_thr is read after the flag
    }
    bsync();
  }

  if constexpr (KTH) return;  // (the last CTA has returned above)

  // ---- merge tree ----
  const uint32_t k = p.k;
  uint2 *res = cand0;
  uint32_t res_n = ctl->count;
  uint32_t level = 0, slot = blockIdx.x, merged = res_n;
  uint32_t kpad = 1;  // k rounded up to a power of two: the kept entries and the sort's padding
  while (kpad < k) kpad <<= 1;
  uint2 *outb = mbuf + (p.mcap - kpad);
  while (p.nslots[level] > 1) {
    // publish my result into slot (level, slot), filtered by the current threshold
    if (t == 0) {
      ctl->red_g = ld_volatile_u32(&p.scratch->g_thr);
      ctl->sel.wcount = 0;
    }
    bsync();
    {
      const uint32_t g = ctl->red_g;
      uint2 *dst = p.slots + (size_t)(p.slot_off[level] + slot) * k;
      for (uint32_t j = t; j < res_n; j += kScanThreads) {
        const uint2 e = res[j];
        if (e.x >= g) dst[atomicAdd(&ctl->sel.wcount, 1u)] = e;  // <= res_n <= k entries
      }
    }
    __threadfence();  // each writer makes its slot entries visible device-wide
    bsync();
    const uint32_t grp = slot / p.fanin;
    const uint32_t first = grp * p.fanin;
    const uint32_t gsize = min(p.fanin, p.nslots[level] - first);
    if (t == 0) {
      p.slot_count[p.slot_off[level] + slot] = ctl->sel.wcount;
      __threadfence();
      const uint32_t arrived = atomicAdd(&p.done[p.done_off[level] + grp], 1u);
      ctl->is_last = (arrived == gsize - 1u) ? 1u : 0u;
      if (ctl->is_last) p.done[p.done_off[level] + grp] = 0u;  // every arrival is in: reset
    }
    bsync();
    if (!ctl->is_last) return;
    __threadfence();
    // the last arrival merges the group's slots: their counts first, then all their
    // entries as one flat index space, kMergeBatch loads per thread in flight at a
    // time, in chunks that fit the shared input area; the best k so far (in `outb`)
    // open each chunk after the first
    if (t == 0) ctl->red_g = ld_volatile_u32(&p.scratch->g_thr);
    if (t < (int)gsize) scnt[t] = __ldcg(&p.slot_count[p.slot_off[level] + first + t]);
    bsync();
    {
      const uint32_t g = ctl->red_g;
      const uint32_t in_cap = p.mcap - kpad;  // input area [0, in_cap), outb after it
      uint32_t total = 0;
      for (uint32_t si = 0; si < gsize; ++si) total += scnt[si];
      uint32_t kept = 0, done = 0;
      merged = 0;
      do {
        for (uint32_t j = t; j < kept; j += kScanThreads) mbuf[j] = outb[j];
        if (t == 0) ctl->sel.wcount = kept;
        bsync();
        const uint32_t n_load = min(total - done, in_cap - kept);
        constexpr int kMergeBatch = 2;
        for (uint32_t base = 0; base < n_load; base += kScanThreads * kMergeBatch) {
          uint2 e[kMergeBatch];
#pragma unroll
          for (int u = 0; u < kMergeBatch; ++u) {
            const uint32_t j = base + (uint32_t)u * kScanThreads + t;
            e[u] = make_uint2(0u, 0u);
            if (j < n_load) {
              uint32_t f = done + j, si = 0;
              while (f >= scnt[si]) f -= scnt[si++];  // done + j < total: ends inside a slot
              e[u] = __ldcg(p.slots + (size_t)(p.slot_off[level] + first + si) * k + f);
            }
          }
#pragma unroll
          for (int u = 0; u < kMergeBatch; ++u) {
            if (base + (uint32_t)u * kScanThreads + t < n_load && e[u].x >= g) {
              const uint32_t pos = atomicAdd(&ctl->sel.wcount, 1u);
              if (TOPK_CHECK(pos < in_cap, kDiagMerge, level, pos, in_cap)) mbuf[pos] = e[u];
            }
          }
        }
        bsync();
        const uint32_t loaded = min(ctl->sel.wcount, in_cap);
        bsync();  // every thread has `loaded` before block_reduce resets wcount
        merged += loaded - kept;
        kept = block_reduce<kScanThreads>(mbuf, loaded, outb, k, 0u, hist, &ctl->sel);
        done += n_load;
      } while (done < total);
      res_n = kept;
    }
    res = outb;
    level += 1;
    slot = grp;
  }

  // ---- root: sort and write the result (res has room for the padding) ----
  block_sort_desc<kScanThreads>(res, res_n);
  if (p.out_ids) {  // (a round that only wants the k-th key has no result arrays)
    for (uint32_t r = t; r < res_n; r += kScanThreads) {
      const uint2 e = res[r];
      const uint32_t pos = res_n - 1 - r;  // ascending output
      p.out_ids[pos] = (uint64_t)e.y;
      p.out_scores[pos] = key2f(e.x);
    }
  }
  if (t == 0) {
    if (p.out_threshold) *p.out_threshold = res_n ? key2f(res[res_n - 1].x) : 0.0f;
    if (p.out_count) *p.out_count = res_n;
    if (p.out_kth_key) *p.out_kth_key = res_n == k ? res[res_n - 1].x : 0u;
    const uint32_t reds = ld_volatile_u32(&p.scratch->acc_reductions);
    const uint32_t tiles = ld_volatile_u32(&p.scratch->acc_tiles);
    p.scratch->last_cands = merged;
    p.scratch->last_reductions = reds;
    if (p.out_stats) {
      p.out_stats[0] = merged;
      p.out_stats[1] = reds;
      p.out_stats[2] = tiles;
    }
    p.scratch->acc_reductions = 0;
    p.scratch->acc_tiles = 0;
    p.scratch->pub_arrived = 0;  // every CTA has left its wait: it published a slot above
    p.scratch->pub_ready = 0;
    p.scratch->g_thr = 0;
    __threadfence();
  }
}

using ScanKernel = void (*)(ScanParams);

// [kth][part][q] for q = 1..16; [..][0] is the runtime-q kernel used for q > 16
#define TOPK_SCAN_ROW(P, K)                                                                                   \
  {scan_select_kernel<0, P, K>,  scan_select_kernel<1, P, K>,  scan_select_kernel<2, P, K>,                   \
   scan_select_kernel<3, P, K>,  scan_select_kernel<4, P, K>,  scan_select_kernel<5, P, K>,                   \
   scan_select_kernel<6, P, K>,  scan_select_kernel<7, P, K>,  scan_select_kernel<8, P, K>,                   \
   scan_select_kernel<9, P, K>,  scan_select_kernel<10, P, K>, scan_select_kernel<11, P, K>,                  \
   scan_select_kernel<12, P, K>, scan_select_kernel<13, P, K>, scan_select_kernel<14, P, K>,                  \
   scan_select_kernel<15, P, K>, scan_select_kernel<16, P, K>}
const ScanKernel kKernels[2][2][17] = {{TOPK_SCAN_ROW(false, false), TOPK_SCAN_ROW(true, false)},
                                       {TOPK_SCAN_ROW(false, true), TOPK_SCAN_ROW(true, true)}};
#undef TOPK_SCAN_ROW

ScanKernel kernel_for(uint32_t qq, bool part, bool kth = false) {
  return kKernels[kth ? 1 : 0][part ? 1 : 0][qq <= 16 ? qq : 0];
}

}  // namespace

cudaError_t scan_set_attributes(size_t smem_optin) {
  for (const auto &mode : kKernels)
    for (const auto &row : mode)
      for (ScanKernel f : row) {
        const cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void *>(f),
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_optin);
        if (e != cudaSuccess) return e;
      }
  return cudaSuccess;
}

namespace {

// Shared memory of an SM that the unified L1 / shared memory can give (B200: 228 KB),
// the L1 the scan keeps (its 128-bit loads land in L1 while in flight: with less, the
// loads in flight per SM, and the bandwidth, shrink), and the per-CTA reserve.
constexpr size_t kSmemPerSm = 228 * 1024;
constexpr size_t kScanL1Keep = 60 * 1024;
constexpr size_t kSmemPerCtaReserve = 1024;

// The shared-memory carveout last set on each scan kernel, per device (the attribute
// is per function and device; setting it again costs a driver call).
std::mutex g_carveout_mu;
int g_carveout[64][2][2][17];

void set_carveout(const void *fn, bool part, uint32_t qq, int percent, bool kth = false) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lk(g_carveout_mu);
  int &cur = g_carveout[dev][kth ? 1 : 0][part ? 1 : 0][qq <= 16 ? qq : 0];
  if (cur == percent + 1) return;  // stored plus one: 0 means not set yet
  if (cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, percent) == cudaSuccess)
    cur = percent + 1;
  else
    (void)cudaGetLastError();
}

}  // namespace

namespace {

// Plans by (device, q, k, partition mode, CTA cap): the occupancy queries behind a plan
// are driver calls, a few microseconds each, on every query's critical path otherwise.
struct PlanEntry {
  ScanPlan pl;
  int carveout;
};
std::mutex g_plan_mu;
std::map<std::tuple<int, uint32_t, uint32_t, bool, uint32_t>, PlanEntry> g_plans;

}  // namespace

ScanPlan plan_scan(uint32_t qq, uint32_t k, uint64_t rows, int num_sms, size_t smem_optin, uint32_t max_ctas_per_sm,
                   bool part) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    dev = -1;
  }
  const auto key = std::make_tuple(dev, qq <= 16 ? qq : 0u, k, part, max_ctas_per_sm);
  const void *fn = reinterpret_cast<const void *>(kernel_for(qq, part));
  const void *fn_kth = reinterpret_cast<const void *>(kernel_for(qq, part, true));
  const uint64_t tiles = (rows + 3 + kTile) / kTile;
  auto finish = [&](ScanPlan pl) {
    uint64_t grid = (uint64_t)num_sms * (uint64_t)pl.ctas_per_sm;
    if (grid > tiles) grid = tiles;
    if (grid < 1) grid = 1;
    pl.grid = (int)grid;
    return pl;
  };
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    const auto it = g_plans.find(key);
    if (it != g_plans.end()) {
      const PlanEntry pe = it->second;
      // the carveout is per function: another plan may have changed it since
      set_carveout(fn, part, qq, pe.carveout);
      set_carveout(fn_kth, part, qq, pe.carveout, true);
      return finish(pe.pl);
    }
  }
  ScanPlan pl{};
  pl.tile = kTile;
  uint32_t P = 1;
  while (P < k) P <<= 1;
  // after a select the buffer holds <= k entries; kVoteTiles tiles add <= that many times
  // kTile, and a select runs once the fill exceeds cap - kVoteTiles * kTile
  // (plus half a tile of slack when every tile votes; with two tiles per vote the
  // rounding below leaves some, and more would cost q <= 2 a CTA per SM)
  const uint32_t vote_tiles = scan_vote_tiles(qq <= 16 ? (int)qq : 0, part);
  uint32_t cap = k + vote_tiles * kTile + (vote_tiles == 1 ? kTile / 2 : 0u);
  if (cap < P) cap = P;
  if (cap < 2048) cap = 2048;
  cap = (cap + kScanThreads - 1) / kScanThreads * kScanThreads;
  pl.cap = cap;
  // the select writes <= k entries (padded to P for the sort) after the buffer; the
  // merge reuses both, its input in chunks of up to cap entries, so the fan-in is not
  // bound by it: G = what two buffers of cap would hold, 4 to kMaxFanin
  uint32_t mcap = cap + P;
  uint32_t G = (2 * cap - P) / k;
  if (G > kMaxFanin) G = kMaxFanin;
  if (G < 4) G = 4;
  pl.fanin = G;
  pl.mcap = mcap;
  pl.smem = kScanSmemFixed + (size_t)mcap * 8;
  pl.stages = pl.smem <= smem_optin ? 1u : 0u;
  // CTAs per SM: as many as registers and threads allow, and as the shared memory
  // allows with kScanL1Keep left as L1 (or the caller's number); the carveout is set to
  // just fit them, so the rest of the unified memory stays L1
  set_carveout(fn, part, qq, 100);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kScanThreads, pl.smem) != cudaSuccess || occ < 1) {
    (void)cudaGetLastError();
    occ = 1;
  }
  const size_t per_cta = pl.smem + kSmemPerCtaReserve;
  const int by_l1 = (int)std::max<size_t>(1, (kSmemPerSm - kScanL1Keep) / per_cta);
  if (max_ctas_per_sm >= 1) occ = std::min<int>(occ, (int)max_ctas_per_sm);
  else occ = std::min(occ, by_l1);
  // the smallest shared-memory size of the SM (KB) that holds them, as a percentage
  static const size_t kSizesKb[] = {0, 8, 16, 32, 64, 100, 132, 164, 196, 228};
  size_t want = per_cta * (size_t)occ, size_kb = 228;
  for (size_t kb : kSizesKb)
    if (kb * 1024 >= want) {
      size_kb = kb;
      break;
    }
  const int carveout = (int)((size_kb * 100 + 227) / 228);
  set_carveout(fn, part, qq, carveout);
  // the threshold-pass form of the kernel runs with the same plan
  set_carveout(fn_kth, part, qq, carveout, true);
  int fit = 0;  // what the driver reports with that preference
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fn, kScanThreads, pl.smem) == cudaSuccess && fit >= 1)
    occ = std::min(occ, fit);
  else
    (void)cudaGetLastError();
  pl.ctas_per_sm = occ;
  if (dev >= 0) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plans[key] = PlanEntry{pl, carveout};
  }
  return finish(pl);
}

void plan_merge_tree(ScanParams &p, uint32_t grid, uint32_t fanin, uint32_t *total_slots, uint32_t *total_groups) {
  uint32_t l = 0, soff = 0, doff = 0;
  p.nslots[0] = grid;
  while (p.nslots[l] > 1 && l + 1 < (uint32_t)kMaxLevels) {
    const uint32_t groups = (p.nslots[l] + fanin - 1) / fanin;
    p.slot_off[l] = soff;
    p.done_off[l] = doff;
    soff += p.nslots[l];
    doff += groups;
    p.nslots[l + 1] = groups;
    ++l;
  }
  p.slot_off[l] = soff;
  p.done_off[l] = doff;
  p.levels = l;
  p.fanin = fanin;
  *total_slots = soff;
  *total_groups = doff;
}

cudaError_t launch_scan(const ScanPlan &pl, const ScanParams &p, cudaStream_t stream) {
  if (pl.stages < 1) return cudaErrorInvalidValue;
  // a threshold pass needs the published-keys area
  if (p.kth_only && (!p.pub || !p.out_kth_key || p.pub_m == 0 || p.pub_m > 8 * kPubMaxPerWarp))
    return cudaErrorInvalidValue;
  ScanParams q = p;
  for (uint32_t m = 0; m < 4; ++m) q.colp[m] = m < p.qq ? p.table + (uint64_t)p.attr[m] * p.ld : p.table;
  q.grid_rows = (uint64_t)pl.grid * p.tile_step;
  // id order: tiles [int_lo, int_lo + int_n) lie wholly inside [row_begin, row_end)
  q.int_lo = p.tile_begin < p.row_begin ? 1u : 0u;
  uint64_t hi = 0;
  if (p.row_end >= p.tile_begin + kTile) hi = (p.row_end - p.tile_begin - kTile) / p.tile_step + 1;
  if (hi > p.num_tiles) hi = p.num_tiles;
  q.int_n = hi > q.int_lo ? (uint32_t)(hi - q.int_lo) : 0u;
  kernel_for(p.qq, p.part_list != nullptr, p.kth_only != 0)<<<pl.grid, kScanThreads, pl.smem, stream>>>(q);
  return cudaGetLastError();
}

}  // namespace topk
