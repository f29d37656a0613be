/*
 * C-ABI shim around the reference's own TPAc class (TEST INFRASTRUCTURE ONLY).
 *
 * Compiled by oracle/build_ref.py from the reference sources where they lie
 * (cpu/TPAc.h, cpu/AA.h, common/common.h, time/Time.h) into oracle/_ref/.
 * Nothing from the reference is copied here: this file only instantiates
 * TPAc<float,uint64_t> and forwards to its public methods, so tests can
 *   - pin the C restatement (topk_oracle.c) against the real code, and
 *   - time TPAc::findTopKthreads / findTopKsimdMQ as the CPU baseline.
 *
 * Flags are strict (-O3 -ffp-contract=off, no -ffast-math): with them the
 * reference's scalar, SIMD and threaded paths agree bit-for-bit.
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <queue>
#include <sstream>
#include <vector>

#include <omp.h>

/* Compile-time knobs the reference headers read (Makefile:16-54). */
#ifndef MQTHREADS
#define MQTHREADS 256
#endif
#ifndef STATS_EFF
#define STATS_EFF false
#endif
#ifndef IMP
#define IMP 2
#endif
#ifndef LD
#define LD 1
#endif
#ifndef WORKLOAD
#define WORKLOAD 1024
#endif
#ifndef NUM_DIMS
#define NUM_DIMS 16
#endif

#include "time/Time.h"
#include "cpu/TPAc.h"
#include "cpu/TPAr.h"
#include "cpu/TA.h"

namespace {

/* The reference prints one line per query; silence it while forwarding. */
struct Quiet {
  std::streambuf *old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

using RefTPAc = TPAc<float, uint64_t>;
using RefTPAr = TPAr<float, uint64_t>;

template <class A>
uint64_t run_query(A *t, int impl, uint64_t k, uint8_t qq, float *weights, uint8_t *attr, uint64_t *ids,
                   float *scores, uint64_t cap, float *thres, double *ms) {
  Quiet q;
  t->reset_clocks();
  double t0 = omp_get_wtime();
  if (impl == 0) t->findTopKscalar(k, qq, weights, attr);
  else if (impl == 1) t->findTopKsimd(k, qq, weights, attr);
  else t->findTopKthreads(k, qq, weights, attr);
  double t1 = omp_get_wtime();
  std::vector<tuple_<float, uint64_t>> res = t->get_res();
  uint64_t c = res.size() < cap ? res.size() : cap;
  for (uint64_t j = 0; j < c; j++) { ids[j] = res[j].tid; scores[j] = res[j].score; }
  if (thres) *thres = t->get_thres();
  if (ms) *ms = (t1 - t0) * 1e3;
  return res.size();
}

template <class A>
int load_table(A *t, const float *src, uint64_t n, uint64_t d) {
  size_t bytes = sizeof(float) * n * d;
  float *buf = static_cast<float *>(aligned_alloc(64, (bytes + 63) / 64 * 64));
  if (!buf) return 1;
  std::memcpy(buf, src, bytes);
  float *&cd = t->get_cdata();
  if (cd) std::free(cd);
  cd = buf;
  return 0;
}

}  // namespace

extern "C" {

void *ref_tpac_create(uint64_t n, uint64_t d) { return new RefTPAc(n, d); }

void ref_tpac_destroy(void *h) { delete static_cast<RefTPAc *>(h); }

/* Copies a column-major n x d table into an aligned buffer that AA owns and
 * frees with free() (cpu/AA.h:147-150). */
int ref_tpac_load(void *h, const float *colmajor, uint64_t n, uint64_t d) {
  RefTPAc *t = static_cast<RefTPAc *>(h);
  size_t bytes = sizeof(float) * n * d;
  size_t alloc = (bytes + 63) / 64 * 64;
  float *buf = static_cast<float *>(aligned_alloc(64, alloc));
  if (!buf) return 1;
  std::memcpy(buf, colmajor, bytes);
  float *&cd = t->get_cdata();
  if (cd) std::free(cd);
  cd = buf;
  return 0;
}

void ref_tpac_init(void *h) {
  Quiet q;
  static_cast<RefTPAc *>(h)->init();
}

void ref_tpac_get_data(void *h, float *out, uint64_t n, uint64_t d) {
  std::memcpy(out, static_cast<RefTPAc *>(h)->get_cdata(), sizeof(float) * n * d);
}

/* impl: 0 findTopKscalar, 1 findTopKsimd, 2 findTopKthreads.
 * Writes res in the reference's own order (ascending heap drain).
 * Returns the number of tuples; *thres = get_thres(); *ms = query-body time. */
uint64_t ref_tpac_query(void *h, int impl, uint64_t k, uint8_t qq, float *weights, uint8_t *attr,
                        uint64_t *ids, float *scores, uint64_t cap, float *thres, double *ms) {
  RefTPAc *t = static_cast<RefTPAc *>(h);
  Quiet q;
  t->reset_clocks();
  double t0 = omp_get_wtime();
  if (impl == 0) t->findTopKscalar(k, qq, weights, attr);
  else if (impl == 1) t->findTopKsimd(k, qq, weights, attr);
  else t->findTopKthreads(k, qq, weights, attr);
  double t1 = omp_get_wtime();
  std::vector<tuple_<float, uint64_t>> res = t->get_res();
  uint64_t c = res.size() < cap ? res.size() : cap;
  for (uint64_t j = 0; j < c; j++) { ids[j] = res[j].tid; scores[j] = res[j].score; }
  if (thres) *thres = t->get_thres();
  if (ms) *ms = (t1 - t0) * 1e3;
  return res.size();
}

/* Multi-query loop as in validation/bench_cpu.h:198-213: `threads` OpenMP threads
 * each call findTopKsimdMQ on their share of the queries. Timing only (that path
 * keeps no result, cpu/TPAc.h:210-254). attrs is nq x stride. Returns wall ms. */
double ref_tpac_mq(void *h, uint64_t nq, const uint64_t *ks, const uint8_t *qqs, float *weights,
                   uint8_t *attrs, uint64_t stride, int threads) {
  RefTPAc *t = static_cast<RefTPAc *>(h);
  if (threads > MQTHREADS) threads = MQTHREADS;
  Quiet q;
  omp_set_num_threads(threads);
  double t0 = omp_get_wtime();
#pragma omp parallel
  {
    uint32_t tid = omp_get_thread_num();
    for (uint64_t j = tid; j < nq; j += (uint64_t)threads)
      t->findTopKsimdMQ(ks[j], qqs[j], weights + j * stride, attrs + j * stride, tid);
  }
  double t1 = omp_get_wtime();
  return (t1 - t0) * 1e3;
}

/* normalize_transpose (common/common.h:30-61) on a caller buffer. */
void ref_normalize_transpose(float *data, uint64_t n, uint64_t d) {
  normalize_transpose<float, uint64_t>(data, n, d);
}

int ref_threads_constant(void) { return THREADS; }

/* TA<float,uint64_t> (cpu/TA.h): sorted lists over a row-major table (load as for
 * TPAr); query = findTopK.  Returns the result count; ids/scores in res order. */
void *ref_ta_create(uint64_t n, uint64_t d) { return new TA<float, uint64_t>(n, d); }
void ref_ta_destroy(void *h) { delete static_cast<TA<float, uint64_t> *>(h); }
int ref_ta_load(void *h, const float *rows, uint64_t n, uint64_t d) {
  return load_table(static_cast<TA<float, uint64_t> *>(h), rows, n, d);
}
void ref_ta_init(void *h) {
  Quiet q;
  static_cast<TA<float, uint64_t> *>(h)->init();
}
uint64_t ref_ta_query(void *h, uint64_t k, uint8_t qq, float *weights, uint8_t *attr, uint64_t *ids, float *scores,
                      uint64_t cap, float *thres, double *ms) {
  TA<float, uint64_t> *t = static_cast<TA<float, uint64_t> *>(h);
  Quiet q;
  t->reset_clocks();
  double t0 = omp_get_wtime();
  t->findTopK(k, qq, weights, attr);
  double t1 = omp_get_wtime();
  std::vector<tuple_<float, uint64_t>> res = t->get_res();
  uint64_t c = res.size() < cap ? res.size() : cap;
  for (uint64_t j = 0; j < c; j++) { ids[j] = res[j].tid; scores[j] = res[j].score; }
  if (thres) *thres = t->get_thres();
  if (ms) *ms = (t1 - t0) * 1e3;
  return res.size();
}

/* TPAr<float,uint64_t> (cpu/TPAr.h): the row-major variant.  load copies an n x d
 * row-major table (object i at src + i*d); init normalises it (common/common.h:63-92);
 * impl as ref_tpac_query.  Its query loops take 8 (scalar, simd) or 16 (threads,
 * per thread share) objects per step with no tail: n must be a multiple of 16*THREADS
 * for all three to stay inside the table. */
void *ref_tpar_create(uint64_t n, uint64_t d) { return new RefTPAr(n, d); }
void ref_tpar_destroy(void *h) { delete static_cast<RefTPAr *>(h); }
int ref_tpar_load(void *h, const float *rows, uint64_t n, uint64_t d) {
  return load_table(static_cast<RefTPAr *>(h), rows, n, d);
}
void ref_tpar_init(void *h) {
  Quiet q;
  static_cast<RefTPAr *>(h)->init();
}
void ref_tpar_get_data(void *h, float *out, uint64_t n, uint64_t d) {
  std::memcpy(out, static_cast<RefTPAr *>(h)->get_cdata(), sizeof(float) * n * d);
}
uint64_t ref_tpar_query(void *h, int impl, uint64_t k, uint8_t qq, float *weights, uint8_t *attr, uint64_t *ids,
                        float *scores, uint64_t cap, float *thres, double *ms) {
  return run_query(static_cast<RefTPAr *>(h), impl, k, qq, weights, attr, ids, scores, cap, thres, ms);
}

}  // extern "C"
