// Drop-in check for the row-major variant: the reference's TPAr<float,uint64_t>
// (cpu/TPAr.h, on the CPU) and TPArGPU<float,uint64_t> (include/topk_b200/TPArGPU.h,
// on the GPU) load the same row-major table through get_cdata(), run init(), and
// answer the harness's queries (k doubling, last-q attribute sets, all three of the
// reference's query entries); results must agree: same k-th score, same score
// multiset, same ids above it (the reference's vector entries' ids mapped back, see
// agree()).  The reference's loops need n to be a multiple of 256.
// Built by tests/dropin/build_demo.py; run by tests/test_gpu_dropin.py.  Usage:
//     tpar_dropin_demo <n> <d> <seed>
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
#include "cpu/TPAr.h"
#include "topk_b200/TPArGPU.h"

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

// mirror: the reference's findTopKsimd/findTopKthreads push lane j of each group of 8
// with id base + j while it holds object base + 7 - j (_mm256_set_ps fills lanes from
// the highest down, cpu/TPAr.h:140-158); their ids are mapped back before comparing.
template <class A, class B>
static bool agree(A &ref, B &gpu, bool mirror) {
  std::vector<tuple_<float, uint64_t>> a = ref.get_res(), b = gpu.get_res();
  if (mirror)
    for (auto &e : a) e.tid = (e.tid / 8) * 8 + 7 - e.tid % 8;
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
  if (n % 256) {
    std::printf("n must be a multiple of 256 for the reference TPAr\n");
    return 2;
  }
  TPAr<float, uint64_t> ref(n, d);
  TPArGPU<float, uint64_t> gpu(n, d);
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

  std::vector<float> weights(d);
  for (uint64_t m = 0; m < d; m++) weights[m] = 0.1f * (float)(m + 1);
  int bad = 0;
  for (uint64_t k = 16; k <= 1024; k *= 4) {
    for (uint64_t q = 2; q <= d; q += 2) {
      std::vector<uint8_t> attr(q);
      for (uint64_t m = 0; m < q; m++) attr[m] = (uint8_t)(d - q + m);
      for (int impl = 0; impl < 3; impl++) {
        old = std::cout.rdbuf(sink.rdbuf());
        if (impl == 0) ref.findTopKscalar(k, (uint8_t)q, weights.data(), attr.data());
        if (impl == 1) ref.findTopKsimd(k, (uint8_t)q, weights.data(), attr.data());
        if (impl == 2) ref.findTopKthreads(k, (uint8_t)q, weights.data(), attr.data());
        gpu.findTopKsimd(k, (uint8_t)q, weights.data(), attr.data());
        std::cout.rdbuf(old);
        const bool ok = agree(ref, gpu, impl != 0);
        std::printf("k=%llu q=%llu impl=%d threshold=%.9g %s\n", (unsigned long long)k, (unsigned long long)q, impl,
                    (double)gpu.get_thres(), ok ? "ok" : "MISMATCH");
        bad += ok ? 0 : 1;
      }
    }
  }
  std::printf("%s\n", bad ? "FAIL" : "PASS");
  return bad ? 1 : 0;
}
