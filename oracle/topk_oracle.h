/*
 * CPU oracle for exact top-k linear aggregation (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C restatement of the reference's TPAc path, used by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py as the checker.
 * The product (topk_b200/) never links, imports or calls it.
 *
 * Reference behaviour restated here (paths relative to the TopK project):
 *   - normalize_transpose      common/common.h:30-61
 *   - TPAc score arithmetic    cpu/TPAc.h:129-147 (mul then add, no FMA, attr order)
 *   - bounded min-heap result  cpu/TPAc.h:151-206, MaxCMP cpu/AA.h:53-58
 *   - result/threshold shape   cpu/AA.h:29-35, 71-73
 *
 * The seeded synthetic-table generators are this project's own definition
 * (the reference seeds its generator with time(NULL), randdataset.c:330) and
 * are mirrored bit-for-bit by the device generator in topk_b200/csrc.
 */
#ifndef TOPK_ORACLE_H
#define TOPK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Distribution codes follow the reference's File::gen numbering
 * (input/File.h:345-352): 0 correlated, 1 independent, 2 anticorrelated.
 * 3 = mixed (object i uses independent/correlated/anticorrelated by i % 3). */
enum { ORC_CORRELATED = 0, ORC_INDEPENDENT = 1, ORC_ANTICORRELATED = 2, ORC_MIXED = 3 };

/* Fill rows [row0, row0+rows) of a column-major table with stride ld. */
void orc_generate(float *data, uint64_t ld, uint32_t d, uint64_t row0, uint64_t rows,
                  int dist, uint64_t seed);

/* Fill `count` query weights U(0,1] from (seed, stream). */
void orc_gen_weights(float *w, uint32_t count, uint64_t seed, uint64_t stream);

/* normalize_transpose (common/common.h:30-61) on a column-major table with
 * stride ld; writes the per-column min/max it used when mins/maxs != NULL. */
void orc_normalize(float *data, uint64_t n, uint64_t ld, uint32_t d, float *mins, float *maxs);

/* Exact FP32 score of object i in the reference order (cpu/TPAc.h:132-142). */
float orc_score(const float *data, uint64_t ld, uint64_t i, uint32_t qq, const float *weights,
                const uint8_t *attr);

/* Exact top-k over rows [row0, row1): results ascending by (score, -id), i.e. the
 * reverse of the selection order (score desc, id asc). Returns the count
 * (min(k, rows)); *threshold = k-th best score. NaN scores rank lowest. */
uint64_t orc_topk(const float *data, uint64_t ld, uint64_t row0, uint64_t row1, uint32_t qq,
                  const float *weights, const uint8_t *attr, uint64_t k, uint64_t *ids,
                  float *scores, float *threshold);

/* Same selection with FP64 scores (error reporting only). */
uint64_t orc_topk_f64(const float *data, uint64_t ld, uint64_t row0, uint64_t row1, uint32_t qq,
                      const float *weights, const uint8_t *attr, uint64_t k, uint64_t *ids,
                      double *scores);

/* FP64 score of object i, same attribute order. */
double orc_score_f64(const float *data, uint64_t ld, uint64_t i, uint32_t qq,
                     const float *weights, const uint8_t *attr);

/* Order-preserving u32 key of a float (NaN -> 0). */
uint32_t orc_key(float s);

#ifdef __cplusplus
}
#endif
#endif
