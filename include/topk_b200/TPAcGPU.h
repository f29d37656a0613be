// TPAcGPU<T,Z>: drop-in replacement for the reference's TPAc<T,Z> (cpu/TPAc.h:6-25)
// that runs on a B200 through the C ABI in topk_b200.h.
//
// It derives from the reference's own AA<T,Z> (cpu/AA.h:63-122), so the harness
// code that drives TPAc (validation/bench_cpu.h:155-237) works unchanged after
// replacing the type:
//
//     TPAcGPU<float,uint64_t> tpac(f.rows(), f.items());   // was TPAc<float,uint64_t>
//     f.gen(tpac.get_cdata(), DISTR);  tpac.init();  tpac.findTopKsimd(k, q, weights, attr);
//
// Build: put the reference tree's root (for "cpu/AA.h") and this repository's
// include/ directory on the include path, define the reference's compile-time knobs
// as its Makefile does (MQTHREADS, STATS_EFF, IMP, LD, WORKLOAD), and link
// topk_b200/_lib/libtopk_b200.so.
//
// Behaviour, method by method:
//   init()              uploads cdata to the GPU and runs normalize_transpose there
//                       (common/common.h:30-61, bit-exact); the normalised table is
//                       copied back into cdata so the object's state matches the
//                       reference's after init().
//   findTopKscalar / findTopKsimd / findTopKthreads
//                       one exact GPU query each; res = k tuples ascending by score,
//                       threshold = k-th score, tt_processing accumulates the query
//                       time, and the same progress line is printed.  All three use
//                       attr[m] for column m (the reference's scalar path uses
//                       attr[0]+m, cpu/TPAc.h:53-81, which agrees for contiguous
//                       ascending attribute sets).
//   findTopKsimdMQ      safe to call from many threads at once on one object (the
//                       multi-query harness does, validation/bench_cpu.h:204-212);
//                       like the reference it keeps no result, only time per thread.
// Ties at the k-th score go to the lower id.  Only weights[attr[m]] are read.
// Errors print the status and message and exit(1), as the reference does.
#ifndef TOPK_B200_TPACGPU_H
#define TOPK_B200_TPACGPU_H

#include <cstdint>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <type_traits>
#include <vector>

#include "cpu/AA.h"
#include "topk_b200.h"

template <class T, class Z>
class TPAcGPU : public AA<T, Z> {
  static_assert(std::is_same<T, float>::value, "TPAcGPU computes in FP32 like the reference TPAc<float,...>");
  static_assert(std::is_integral<Z>::value && sizeof(Z) >= 4, "object ids must be an integer type of >= 32 bits");

 public:
  TPAcGPU(uint64_t n, uint64_t d, int device = 0) : AA<T, Z>(n, d) {
    this->algo = "TPAcGPU";
    check(topk_create(n, (uint32_t)d, device, &h_));
  }
  ~TPAcGPU() { topk_destroy(h_); }
  TPAcGPU(const TPAcGPU &) = delete;
  TPAcGPU &operator=(const TPAcGPU &) = delete;

  void init() {
    if (this->cdata == NULL) die(TOPK_ERR_STATE, "init() before the table was loaded into get_cdata()");
    check(topk_upload_colmajor(h_, this->cdata, this->n));
    check(topk_normalize(h_, NULL, NULL));
    check(topk_download_colmajor(h_, this->cdata, this->n));
    this->t.start();
    this->tt_init = this->t.lap();
  }

  void findTopKscalar(uint64_t k, uint8_t qq, T *weights, uint8_t *attr) { query(k, qq, weights, attr, "scalar"); }
  void findTopKsimd(uint64_t k, uint8_t qq, T *weights, uint8_t *attr) { query(k, qq, weights, attr, "simd"); }
  void findTopKthreads(uint64_t k, uint8_t qq, T *weights, uint8_t *attr) { query(k, qq, weights, attr, "threads"); }

  void findTopKsimdMQ(uint64_t k, uint8_t qq, T *weights, uint8_t *attr, uint32_t tid) {
    Time<msecs> t;
    const uint64_t c = k < this->n ? k : this->n;
    std::vector<uint64_t> ids(c);
    std::vector<float> scores(c);
    t.start();
    check(topk_query(h_, k, qq, weights, attr, ids.data(), scores.data(), NULL, NULL));
    this->tt_array[tid] += t.lap();
  }

  topk_table_t handle() const { return h_; }

 private:
  topk_table_t h_ = nullptr;

 protected:
  [[noreturn]] static void die(int st, const char *msg) {
    std::cout << "topk_b200: " << topk_status_name(st) << ": " << msg << std::endl;
    exit(1);
  }
  static void check(int st) {
    if (st != TOPK_OK) die(st, topk_last_error());
  }

 private:
  void query(uint64_t k, uint8_t qq, T *weights, uint8_t *attr, const char *how) {
    std::cout << this->algo << " find top-" << k << " " << how << " (" << (int)qq << "D) ...";
    if (this->res.size() > 0) this->res.clear();
    const uint64_t c = k < this->n ? k : this->n;
    std::vector<uint64_t> ids(c);
    std::vector<float> scores(c);
    uint64_t count = 0;
    float threshold = 0;
    this->t.start();
    check(topk_query(h_, k, qq, weights, attr, ids.data(), scores.data(), &count, &threshold));
    this->tt_processing += this->t.lap();
    if (STATS_EFF) this->tuple_count = this->n;
    for (uint64_t j = 0; j < count; j++) this->res.push_back(tuple_<T, Z>((Z)ids[j], scores[j]));
    std::cout << std::fixed << std::setprecision(4);
    std::cout << " threshold=[" << threshold << "] (" << this->res.size() << ")" << std::endl;
    this->threshold = threshold;
  }
};

#endif  // TOPK_B200_TPACGPU_H
