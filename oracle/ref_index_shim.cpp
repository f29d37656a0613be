/*
 * C-ABI shim around the reference's VTA and PTA index builds (TEST INFRASTRUCTURE ONLY).
 *
 * Compiled by oracle/build.py from the reference sources where they lie (cpu/VTA.h,
 * cpu/PTA.h, cpu/AA.h, common/common.h, time/Time.h) into oracle/_ref/, once per
 * NUM_DIMS (the reference fixes the attribute count at compile time, Makefile:60) and
 * per IMP (IMP 2, the shipped default, makes VTA split the rows into THREADS equal
 * ranges, cpu/VTA.h:13).  Nothing from the reference is copied here: this file runs
 * VTA<float,uint64_t>::init / PTA<float,uint64_t>::init on a caller table and reads the
 * index they built, so tests can pin the numpy restatement of the orders against the
 * real code and the benchmark can time the reference's own index build.
 *
 * The index (parts, blocks) is private in the reference classes; `private` is defined
 * to `public` around their headers only, after every library header is in.
 */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <map>
#include <queue>
#include <sstream>
#include <vector>

#include <immintrin.h>
#include <omp.h>
#include <parallel/algorithm>

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
#error "NUM_DIMS must be given"
#endif

#include "time/Time.h"
#include "cpu/AA.h"
#define private public
#include "cpu/PTA.h"
#include "cpu/VTA.h"
#undef private

namespace {

/* tt_init is protected in AA: read it from a derived class. */
struct VtaRef : VTA<float, uint64_t> {
  using VTA<float, uint64_t>::VTA;
  double init_ms() const { return this->tt_init; }
};
struct PtaRef : PTA<float, uint64_t> {
  using PTA<float, uint64_t>::PTA;
  double init_ms() const { return this->tt_init; }
};

struct Quiet {
  std::streambuf *old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

template <class A>
bool load(A &a, const float *colmajor, uint64_t n, uint64_t d) {
  const size_t bytes = sizeof(float) * n * d;
  float *buf = static_cast<float *>(aligned_alloc(64, (bytes + 63) / 64 * 64));
  if (!buf) return false;
  std::memcpy(buf, colmajor, bytes);
  a.get_cdata() = buf;
  return true;
}

/* Rows of every block of every partition in index order, out[r * d + m]. */
template <class Part, size_t NP, size_t BS>
uint64_t read_rows(Part (&parts)[NP], uint64_t d, uint64_t cap, float *out) {
  uint64_t r = 0;
  for (size_t i = 0; i < NP; i++) {
    if (parts[i].size == 0) continue;
    uint64_t left = parts[i].size;
    for (uint64_t b = 0; b < parts[i].block_num && left > 0; b++) {
      const uint64_t t = parts[i].blocks[b].tuple_num;
      for (uint64_t j = 0; j < t && r < cap; j++, r++)
        for (uint64_t m = 0; m < d; m++) out[r * d + m] = parts[i].blocks[b].tuples[m * BS + j];
      left -= t < left ? t : left;
    }
    std::free(parts[i].blocks);
    parts[i].blocks = nullptr;
  }
  return r;
}

}  // namespace

extern "C" {

/* VTA<float,uint64_t>::init (normalisation included) on a copy of the raw column-major
 * table; writes up to n rows in index order.  Returns the rows written; *init_ms is the
 * reference's own init timer (tt_init, index build after normalisation). */
uint64_t ref_vta_rows(const float *colmajor, uint64_t n, uint64_t d, float *out_rows, double *init_ms) {
  if (d > NUM_DIMS) return 0;
  VtaRef v(n, d);
  if (!load(v, colmajor, n, d)) return 0;
  {
    Quiet q;
    v.init();
  }
  if (init_ms) *init_ms = v.init_ms();
  return read_rows<vta_partition<float, uint64_t>, VPARTITIONS, VBLOCK_SIZE>(v.parts, d, n, out_rows);
}

/* PTA<float,uint64_t>::init likewise (polar partitions, then VTA's order in each). */
uint64_t ref_pta_rows(const float *colmajor, uint64_t n, uint64_t d, float *out_rows, double *init_ms) {
  if (d != NUM_DIMS) return 0;
  PtaRef p(n, d);
  if (!load(p, colmajor, n, d)) return 0;
  {
    Quiet q;
    p.init();
  }
  if (init_ms) *init_ms = p.init_ms();
  return read_rows<pta_partition<float, uint64_t>, PPARTITIONS, PBLOCK_SIZE>(p.parts, d, n, out_rows);
}

int ref_index_num_dims(void) { return NUM_DIMS; }
int ref_index_vta_partitions(void) { return (int)VPARTITIONS; }

}  // extern "C"
