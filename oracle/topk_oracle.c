/*
 * CPU oracle for exact top-k linear aggregation (TEST INFRASTRUCTURE ONLY).
 * See topk_oracle.h for what is restated from the reference and where.
 *
 * Build strictly: -O2 -ffp-contract=off, never -ffast-math, so that every
 * multiply and add rounds once, as in the reference's AVX2 path
 * (cpu/TPAc.h:139-142 uses _mm256_mul_ps then _mm256_add_ps).
 */
#include "topk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------
 * Seeded counter-based generator (this project's definition).
 * splitmix64 finaliser (Steele, Lea, Flood 2014) applied to (seed, stream, row).
 * ------------------------------------------------------------------------- */
static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t row) {
  return mix64(mix64(seed ^ (stream << 32) ^ (stream >> 32)) ^ row);
}

/* 24-bit uniform integer in [0, 2^24). */
static inline uint32_t u24(uint64_t seed, uint64_t stream, uint64_t row) {
  return (uint32_t)(hash3(seed, stream, row) >> 40);
}

static const float TWO_M24 = 5.9604644775390625e-08f; /* 2^-24 */
static const float TWO_M25 = 2.98023223876953125e-08f; /* 2^-25 */
static const float NOISE_SIGMA = 0.05f;

/* Irwin-Hall N(0,1) approximation: sum of 12 U[0,1) minus 6 (the construction of
 * the reference's random_normal, randdataset.c:249-253), done in integers so it is
 * exact; six hashes give the twelve 24-bit draws. */
static inline float normal01(uint64_t seed, uint64_t stream, uint64_t row) {
  int64_t acc = 0;
  for (int j = 0; j < 6; j++) {
    uint64_t h = hash3(seed, stream * 8 + (uint64_t)j, row);
    acc += (int64_t)(h >> 40);
    acc += (int64_t)((h >> 16) & 0xFFFFFFu);
  }
  int32_t z = (int32_t)(acc - 6 * (int64_t)16777216);
  return (float)z * TWO_M24;
}

static inline float clamp01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

/* Stream ids, kept apart per distribution so the mixed table reuses them. */
#define ST_INDEP(m) (0x100u + (m))
#define ST_CORR_BASE 0x200u
#define ST_CORR_NOISE(m) (0x300u + (m))
#define ST_ANTI_SPLIT(j) (0x400u + (j))
#define ST_ANTI_NOISE(m) (0x500u + (m))

static void gen_row(float *out, uint32_t d, uint64_t i, int dist, uint64_t seed) {
  if (dist == ORC_MIXED) dist = (int)(i % 3 == 0 ? ORC_INDEPENDENT : (i % 3 == 1 ? ORC_CORRELATED : ORC_ANTICORRELATED));
  if (dist == ORC_INDEPENDENT) {
    for (uint32_t m = 0; m < d; m++) out[m] = (float)u24(seed, ST_INDEP(m), i) * TWO_M24;
  } else if (dist == ORC_CORRELATED) {
    float v = (float)u24(seed, ST_CORR_BASE, i) * TWO_M24;
    for (uint32_t m = 0; m < d; m++) {
      float t = normal01(seed, ST_CORR_NOISE(m), i) * NOISE_SIGMA;
      out[m] = clamp01(v + t);
    }
  } else { /* anticorrelated: Dirichlet(1..1) spacings scaled to sum d/2, plus noise */
    uint32_t s[64];
    uint32_t cnt = d - 1;
    for (uint32_t j = 0; j < cnt; j++) s[j] = u24(seed, ST_ANTI_SPLIT(j), i);
    for (uint32_t a = 1; a < cnt; a++) { /* insertion sort, ascending */
      uint32_t v = s[a];
      uint32_t b = a;
      while (b > 0 && s[b - 1] > v) { s[b] = s[b - 1]; b--; }
      s[b] = v;
    }
    uint32_t prev = 0;
    for (uint32_t m = 0; m < d; m++) {
      uint32_t cur = (m < cnt) ? s[m] : 16777216u;
      uint32_t e = cur - prev;
      prev = cur;
      float base = (float)(int32_t)(e * d) * TWO_M25; /* (d/2) * e / 2^24 */
      float t = normal01(seed, ST_ANTI_NOISE(m), i) * NOISE_SIGMA;
      out[m] = clamp01(base + t);
    }
  }
}

void orc_generate(float *data, uint64_t ld, uint32_t d, uint64_t row0, uint64_t rows, int dist,
                  uint64_t seed) {
#pragma omp parallel for schedule(static)
  for (uint64_t r = 0; r < rows; r++) {
    float tmp[64];
    uint64_t i = row0 + r;
    gen_row(tmp, d, i, dist, seed);
    for (uint32_t m = 0; m < d; m++) data[(uint64_t)m * ld + i] = tmp[m];
  }
}

void orc_gen_weights(float *w, uint32_t count, uint64_t seed, uint64_t stream) {
  for (uint32_t j = 0; j < count; j++) w[j] = (float)(u24(seed, 0x10000u + stream, j) + 1u) * TWO_M24;
}

/* ---------------------------------------------------------------------------
 * normalize_transpose, common/common.h:30-61: per column, max starts at 0 (:36)
 * and min at FLT_MAX (:37), std::max/std::min comparisons (NaN is skipped), then
 * v = (v - min) / (max - min) with one IEEE division (:53-55).
 * ------------------------------------------------------------------------- */
void orc_normalize(float *data, uint64_t n, uint64_t ld, uint32_t d, float *mins, float *maxs) {
  for (uint32_t m = 0; m < d; m++) {
    float mx = 0.0f, mn = 3.40282346638528859812e+38f;
    float *col = data + (uint64_t)m * ld;
    for (uint64_t i = 0; i < n; i++) {
      float v = col[i];
      mx = (mx < v) ? v : mx; /* std::max(a,b) = (a<b)?b:a */
      mn = (v < mn) ? v : mn; /* std::min(a,b) = (b<a)?b:a */
    }
    float mm = mx - mn;
    for (uint64_t i = 0; i < n; i++) col[i] = (col[i] - mn) / mm;
    if (mins) mins[m] = mn;
    if (maxs) maxs[m] = mx;
  }
}

/* ---------------------------------------------------------------------------
 * Scoring, cpu/TPAc.h:130-142: s = 0; for m in attr order: s = s + x*w (two roundings).
 * ------------------------------------------------------------------------- */
float orc_score(const float *data, uint64_t ld, uint64_t i, uint32_t qq, const float *weights,
                const uint8_t *attr) {
  float s = 0.0f;
  for (uint32_t m = 0; m < qq; m++) {
    float p = data[(uint64_t)attr[m] * ld + i] * weights[attr[m]];
    s = s + p;
  }
  return s;
}

double orc_score_f64(const float *data, uint64_t ld, uint64_t i, uint32_t qq,
                     const float *weights, const uint8_t *attr) {
  double s = 0.0;
  for (uint32_t m = 0; m < qq; m++)
    s += (double)data[(uint64_t)attr[m] * ld + i] * (double)weights[attr[m]];
  return s;
}

uint32_t orc_key(float s) {
  uint32_t u;
  memcpy(&u, &s, 4);
  if (s != s) return 0u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

/* ---------------------------------------------------------------------------
 * Bounded selection.  The reference keeps a min-heap of at least k tuples and
 * replaces the top when a strictly larger score arrives (cpu/TPAc.h:168-185),
 * so the set is the top-k by score; equal scores at the boundary depend on heap
 * order there.  The oracle fixes them deterministically: rank by (score desc,
 * id asc), i.e. ties go to the lower id.
 * ------------------------------------------------------------------------- */
typedef struct { uint64_t key; uint64_t id; } ent_t; /* key: higher is better */

static inline int worse(const ent_t *a, const ent_t *b) { /* a ranks below b */
  return a->key < b->key || (a->key == b->key && a->id > b->id);
}

static void sift_down(ent_t *h, uint64_t len, uint64_t i) {
  for (;;) {
    uint64_t l = 2 * i + 1, r = l + 1, w = i;
    if (l < len && worse(&h[l], &h[w])) w = l;
    if (r < len && worse(&h[r], &h[w])) w = r;
    if (w == i) return;
    ent_t t = h[i]; h[i] = h[w]; h[w] = t;
    i = w;
  }
}

static void sift_up(ent_t *h, uint64_t i) {
  while (i > 0) {
    uint64_t p = (i - 1) / 2;
    if (!worse(&h[i], &h[p])) return;
    ent_t t = h[i]; h[i] = h[p]; h[p] = t;
    i = p;
  }
}

/* Keeps the best k entries in a heap whose root is the worst kept entry. */
typedef struct { ent_t *h; uint64_t len, cap; } sel_t;

static inline void sel_push(sel_t *s, uint64_t key, uint64_t id) {
  ent_t e = {key, id};
  if (s->len < s->cap) { s->h[s->len] = e; sift_up(s->h, s->len); s->len++; }
  else if (s->cap > 0 && worse(&s->h[0], &e)) { s->h[0] = e; sift_down(s->h, s->len, 0); }
}

/* Pops worst-first, which is ascending by (score, -id). */
static uint64_t sel_drain(sel_t *s, ent_t *out) {
  uint64_t c = s->len;
  for (uint64_t j = 0; j < c; j++) {
    out[j] = s->h[0];
    s->h[0] = s->h[s->len - 1];
    s->len--;
    sift_down(s->h, s->len, 0);
  }
  return c;
}

uint64_t orc_topk(const float *data, uint64_t ld, uint64_t row0, uint64_t row1, uint32_t qq,
                  const float *weights, const uint8_t *attr, uint64_t k, uint64_t *ids,
                  float *scores, float *threshold) {
  uint64_t rows = row1 > row0 ? row1 - row0 : 0;
  uint64_t cap = k < rows ? k : rows;
  sel_t s = {(ent_t *)malloc(sizeof(ent_t) * (cap ? cap : 1)), 0, cap};
  for (uint64_t i = row0; i < row1; i++) sel_push(&s, orc_key(orc_score(data, ld, i, qq, weights, attr)), i);
  ent_t *out = (ent_t *)malloc(sizeof(ent_t) * (cap ? cap : 1));
  uint64_t c = sel_drain(&s, out);
  for (uint64_t j = 0; j < c; j++) {
    ids[j] = out[j].id;
    scores[j] = orc_score(data, ld, out[j].id, qq, weights, attr);
  }
  if (threshold) *threshold = c ? scores[0] : 0.0f;
  free(out);
  free(s.h);
  return c;
}

static uint64_t key64(double s) {
  uint64_t u;
  memcpy(&u, &s, 8);
  if (s != s) return 0u;
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

uint64_t orc_topk_f64(const float *data, uint64_t ld, uint64_t row0, uint64_t row1, uint32_t qq,
                      const float *weights, const uint8_t *attr, uint64_t k, uint64_t *ids,
                      double *scores) {
  uint64_t rows = row1 > row0 ? row1 - row0 : 0;
  uint64_t cap = k < rows ? k : rows;
  sel_t s = {(ent_t *)malloc(sizeof(ent_t) * (cap ? cap : 1)), 0, cap};
  for (uint64_t i = row0; i < row1; i++) sel_push(&s, key64(orc_score_f64(data, ld, i, qq, weights, attr)), i);
  ent_t *out = (ent_t *)malloc(sizeof(ent_t) * (cap ? cap : 1));
  uint64_t c = sel_drain(&s, out);
  for (uint64_t j = 0; j < c; j++) {
    ids[j] = out[j].id;
    scores[j] = orc_score_f64(data, ld, out[j].id, qq, weights, attr);
  }
  free(out);
  free(s.h);
  return c;
}
