// Drop-in check for the threshold algorithm: the reference's TA<float,uint64_t>
// (cpu/TA.h, on the CPU) and TAGPU<float,uint64_t> (include/topk_b200/TAGPU.h, on the
// GPU) load the same row-major table through get_cdata(), run init(), and answer the
// harness's queries (k doubling, last-q attribute sets) with equal weights (the
// reference's scores are right only then, cpu/TA.h:83); results must agree: same k-th
// score, same score multiset, same ids above it.
// Built by tests/dropin/build_demo.py; run by tests/test_gpu_dropin.py.  Usage:
//     ta_dropin_demo <n> <d> <seed>
#define MQTHREADS 64
#define STATS_EFF false
#define IMP 1
#define LD 1
#define WORKLOAD 1024
#define NUM_DIMS 16

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <queue>
#include <sstream>
#include <vector>

#include "time/Time.h"
#include "cpu/TA.h"
#include "topk_b200/TAGPU.h"

// Deterministic U[0,1) table (xorshift64*), row-major.
static void fill(float *data, uint64_t n, uint64_t d, uint64_t seed) {
  uint64_t x = seed * 0x9E3779B97F4A7C15ull + 7;
  for (uint64_t i = 0; i < n * d; i++) {
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    data[i] = (float)((x * 0x2545F4914F6CDD1Dull) >> 40) * (1.0f / 16777216.0f);
  }
}

template <class A, class B>
static bool agree(A &ref, B &gpu) {
  std::vector<tuple_<float, uint64_t>> a = ref.get_res(), b = gpu.get_res();
  bool ok = a.size() == b.size() && ref.get_thres() == gpu.get_thres();
  std::vector<float> sa, sb;
  std::vector<uint64_t> ia, ib;
  for (auto &e : a) {
    sa.push_back(e.score);
    if (e.score > ref.get_thres()) ia.push_back(e.tid);
  }
  for (auto &e : b) {
    sb.push_back(e.score);
    if (e.score > gpu.get_thres()) ib.push_back(e.tid);
  }
  std::sort(sa.begin(), sa.end());
  std::sort(sb.begin(), sb.end());
  std::sort(ia.begin(), ia.end());
  std::sort(ib.begin(), ib.end());
  return ok && sa == sb && ia == ib;
}

int main(int argc, char **argv) {
  const uint64_t n = argc > 1 ? strtoull(argv[1], nullptr, 10) : (1u << 20);
  const uint64_t d = argc > 2 ? strtoull(argv[2], nullptr, 10) : 8;
  const uint64_t seed = argc > 3 ? strtoull(argv[3], nullptr, 10) : 1;
  TA<float, uint64_t> ref(n, d);
  TAGPU<float, uint64_t> gpu(n, d);
  ref.get_cdata() = static_cast<float *>(aligned_alloc(64, sizeof(float) * n * d));
  gpu.get_cdata() = static_cast<float *>(aligned_alloc(64, sizeof(float) * n * d));
  fill(ref.get_cdata(), n, d, seed);
  std::memcpy(gpu.get_cdata(), ref.get_cdata(), sizeof(float) * n * d);

  std::ostringstream sink;
  std::streambuf *old = std::cout.rdbuf(sink.rdbuf());
  ref.init();
  gpu.init();
  std::cout.rdbuf(old);
  if (std::memcmp(ref.get_cdata(), gpu.get_cdata(), sizeof(float) * n * d) != 0) {
    std::printf("normalize MISMATCH\n");
    return 1;
  }
  std::printf("normalize ok\n");

  std::vector<float> weights(d, 0.5f);  // equal weights: the reference scores them right
  int bad = 0;
  for (uint64_t k = 16; k <= 1024; k *= 4) {
    for (uint64_t q = 2; q <= d; q += 2) {
      std::vector<uint8_t> attr(q);
      for (uint64_t m = 0; m < q; m++) attr[m] = (uint8_t)(d - q + m);
      old = std::cout.rdbuf(sink.rdbuf());
      ref.findTopK(k, (uint8_t)q, weights.data(), attr.data());
      gpu.findTopK(k, (uint8_t)q, weights.data(), attr.data());
      std::cout.rdbuf(old);
      const bool ok = agree(ref, gpu);
      std::printf("k=%llu q=%llu threshold=%.9g %s\n", (unsigned long long)k, (unsigned long long)q,
                  (double)gpu.get_thres(), ok ? "ok" : "MISMATCH");
      bad += ok ? 0 : 1;
    }
  }
  std::printf("%s\n", bad ? "FAIL" : "PASS");
  return bad ? 1 : 0;
}
