/*
 * C-ABI shim around the reference's SLA layer build (TEST INFRASTRUCTURE ONLY).
 *
 * Compiled by oracle/build.py from cpu/SLA.h and the skyline library it vendors
 * (skyline/hybrid, skyline/common, skyline/util), where they lie, into
 * oracle/_ref/libref_sla_d{D}.so, one library per NUM_DIMS (the reference and its
 * skyline library fix the attribute count at compile time).  Nothing from the
 * reference is copied here: this file runs SLA<float,uint64_t>::init on a caller table
 * and reads the skyline layers and the index it built (cpu/SLA.h:102-139, 199-251), so
 * tests can pin a restatement of the layer peeling and the index order against the
 * real code.
 *
 * The layers are private in SLA; `private` is defined to `public` around its header
 * only, after every library header is in.
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
#include <unordered_map>
#include <unordered_set>
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
#include "skyline/hybrid/hybrid.h"
#include "cpu/VTA.h"  // SLA's queries use VTA's VBLOCK_SIZE (cpu/SLA.h:308); the reference includes both
#define private public
#include "cpu/SLA.h"
#undef private

namespace {
struct Quiet {
  std::streambuf *old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};
}  // namespace

extern "C" {

/* SLA<float,uint64_t>::init on a copy of the raw column-major n x d table (d must be
 * NUM_DIMS); writes each row's layer number (0 = the first skyline) into layer_of and
 * returns the number of layers (0 on failure). */
uint64_t ref_sla_layers(const float *colmajor, uint64_t n, uint64_t d, uint32_t *layer_of) {
  if (d != NUM_DIMS) return 0;
  SLA<float, uint64_t> s(n, d);
  const size_t bytes = sizeof(float) * n * d;
  float *buf = static_cast<float *>(aligned_alloc(64, (bytes + 63) / 64 * 64));
  if (!buf) return 0;
  std::memcpy(buf, colmajor, bytes);
  s.get_cdata() = buf;
  {
    Quiet q;
    s.init();
  }
  for (uint64_t l = 0; l < s.layers.size(); ++l)
    for (uint64_t id : s.layers[l]) layer_of[id] = (uint32_t)l;
  return s.layers.size();
}

/* The same build's rows in index order (layer by layer, block by block: the layer's
 * rows in VTA's order, cpu/SLA.h:199-251), out[r * d + m]; returns the rows written. */
uint64_t ref_sla_rows(const float *colmajor, uint64_t n, uint64_t d, float *out_rows) {
  if (d != NUM_DIMS) return 0;
  SLA<float, uint64_t> s(n, d);
  const size_t bytes = sizeof(float) * n * d;
  float *buf = static_cast<float *>(aligned_alloc(64, (bytes + 63) / 64 * 64));
  if (!buf) return 0;
  std::memcpy(buf, colmajor, bytes);
  s.get_cdata() = buf;
  {
    Quiet q;
    s.init();
  }
  uint64_t r = 0;
  for (uint64_t i = 0; i < s.layer_num; ++i)
    for (uint64_t b = 0; b < s.parts[i].block_num; ++b)
      for (uint64_t j = 0; j < s.parts[i].blocks[b].tuple_num && r < n; ++j, ++r)
        for (uint64_t m = 0; m < d; ++m) out_rows[r * d + m] = s.parts[i].blocks[b].tuples[m * SBLOCK_SIZE + j];
  return r;
}

int ref_sla_num_dims(void) { return NUM_DIMS; }

}  // extern "C"
