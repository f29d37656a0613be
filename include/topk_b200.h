/*
 * topk_b200 - C ABI of the B200 (sm_100a) exact top-k linear-aggregation engine.
 *
 * One handle holds one n x d FP32 table, column-major, resident in HBM (the
 * device copy of AA::cdata).  Queries return the k object ids with the largest
 * weighted sums over a subset of attributes, bit-exact with the reference's
 * strict-FP32 TPAc path.  Everything in these signatures is plain C: pointers,
 * sizes and int status codes.
 *
 * Reference interfaces replaced (paths inside the TopK project):
 *   AA<T,Z>::AA(n,d), get_cdata()            cpu/AA.h:66, :77      -> topk_create, topk_upload_colmajor
 *   TPAc::init() -> normalize_transpose       cpu/TPAc.h:28-32,
 *                                             common/common.h:30-61 -> topk_normalize
 *   File<T>::gen(data, type)                  input/File.h:335-354  -> topk_generate
 *   TPAr<T,Z> (row-major cdata), normalize    cpu/TPAr.h:6-33,
 *                                             common/common.h:63-92 -> topk_upload_rowmajor,
 *                                                                      topk_download_rowmajor
 *   TA<T,Z>::init, findTopK                   cpu/TA.h:40-96        -> topk_build_lists, topk_query_ta
 *   SLA<T,Z>::build_layers, create_lists      cpu/SLA.h:102-251     -> topk_skyline_layers,
 *                                                                      topk_build_partitions_ordered(SLA)
 *   File<T>::count, load (transpose), store   input/File.h:108-132,
 *                                             233-330, 405-431      -> topk_csv_shape, topk_load_csv,
 *                                                                      topk_save_csv
 *   TPAc::findTopKscalar/simd/threads         cpu/TPAc.h:35,118,257 -> topk_query
 *   TPAc::findTopKsimdMQ + MQ loop            cpu/TPAc.h:210-254,
 *                                             validation/bench_cpu.h:198-232 -> topk_query_batch
 *   AA::get_res(), get_thres()                cpu/AA.h:71,73        -> ids/scores/threshold outputs
 *   AA::~AA()                                 cpu/AA.h:147-150      -> topk_destroy
 *
 * Semantics (same meaning as the reference's arguments):
 *   weights  - indexed by ATTRIBUTE ID, length >= d (cpu/TPAc.h:135 weights[attr[m]]).
 *   attr     - qq attribute ids; the score is s = 0; for m in 0..qq-1:
 *              s = s + x[attr[m]] * weights[attr[m]]  (one rounding per op, no FMA).
 *   result   - min(k, rows) tuples ASCENDING by score, like the reference's min-heap
 *              drain (cpu/TPAc.h:198-203); threshold = the k-th best score
 *              (cpu/TPAc.h:199).  Ties are ranked by lower id first, so among equal
 *              scores the ascending output lists the higher id first.
 *   NaN scores rank below every number.
 *
 * Errors: every call returns TOPK_OK or a TOPK_ERR_* code; topk_last_error()
 * gives a message for the calling thread.  (The reference prints and exit(1)s;
 * the C++ drop-in wrapper keeps that behaviour on top of these codes.)
 *
 * Threading: topk_query and topk_query_batch are safe to call concurrently on one
 * handle (each call takes its own scratch context and stream from a pool), which
 * is what the reference's findTopKsimdMQ callers do (validation/bench_cpu.h:204-212).
 * topk_query_device uses the handle's primary context: callers serialise it.
 */
#ifndef TOPK_B200_H
#define TOPK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TOPK_OK 0
#define TOPK_ERR_ARG 1         /* bad argument (k == 0, qq == 0, attr >= d, null pointer, ...) */
#define TOPK_ERR_CUDA 2        /* a CUDA runtime call failed */
#define TOPK_ERR_OOM 3         /* device or pinned allocation failed */
#define TOPK_ERR_TIMEOUT 4     /* a bounded device-side wait gave up */
#define TOPK_ERR_UNSUPPORTED 5 /* valid request outside this build's limits (e.g. k > TOPK_MAX_K) */
#define TOPK_ERR_STATE 6       /* call out of order (e.g. query before any table data) */

#define TOPK_MAX_K 4096u   /* largest k of the fused scan + select path */
#define TOPK_MAX_Q 64u     /* largest qq per query */
#define TOPK_MAX_D 255u    /* attr ids are uint8_t in the reference (cpu/TPAc.h:19) */

/* Distribution codes of topk_generate, numbered like File<T>::gen
 * (input/File.h:345-352); 3 mixes them by object id modulo 3. */
#define TOPK_DIST_CORRELATED 0
#define TOPK_DIST_INDEPENDENT 1
#define TOPK_DIST_ANTICORRELATED 2
#define TOPK_DIST_MIXED 3

typedef struct topk_table_s *topk_table_t;

/* Create a handle for an n x d table on CUDA device `device` and allocate its
 * device copy (column stride rounded up to 64 rows).  Replaces AA(n,d). */
int topk_create(uint64_t n, uint32_t d, int device, topk_table_t *out);

/* Free the device table and every scratch context.  Replaces ~AA(). */
int topk_destroy(topk_table_t h);

/* Copy a host column-major table (column m at host + m*ld_host, ld_host >= n)
 * into the device copy.  Replaces filling get_cdata(). */
int topk_upload_colmajor(topk_table_t h, const float *host, uint64_t ld_host);

/* Fill the device table with this engine's seeded synthetic distribution
 * (bit-identical to the oracle's generator).  Replaces File<T>::gen. */
int topk_generate(topk_table_t h, int dist, uint64_t seed);

/* normalize_transpose on the device copy: per-attribute min/max, then
 * v = (v - min) / (max - min), IEEE division.  Replaces TPAc::init().
 * mins/maxs (length d, may be NULL) receive the values used. */
int topk_normalize(topk_table_t h, float *mins, float *maxs);

/* Copy the device table back (column-major, host stride ld_host >= n). */
int topk_download_colmajor(topk_table_t h, float *host, uint64_t ld_host);

/* The threshold algorithm (cpu/TA.h).  topk_build_lists: TA::init's sorted lists
 * (:40-58), one per attribute, ids by value descending (ties by the lower id) with the
 * values in that order, built on the device (radix sorts, n < 2^31; 8*d*n bytes plus
 * ~70 MB of query scratch); rebuild after the table changes.  topk_read_list: list m's
 * ids and values (n each, either may be NULL).  topk_query_ta: TA::findTopK (:61-96)
 * on the device, exact: the queried lists are walked in blocks of growing depth,
 * every object met is scored once in the query's order, and the walk stops when the
 * k-th score is strictly above the threshold of the unseen objects (sum of
 * w * list value at the depth reached; the attribute's minimum for w < 0), so the
 * result equals topk_query's, ties to the lower id.  The reference scores every
 * attribute of an object with the weight of the list it was found in (cpu/TA.h:83),
 * which is wrong unless all weights are equal; here each attribute has its own weight.
 * stats (3 entries, may be NULL): depth walked, objects scored, blocks.  TA queries on
 * one handle run one at a time. */
int topk_build_lists(topk_table_t h);
int topk_read_list(topk_table_t h, uint32_t m, uint32_t *ids, float *values);
int topk_query_ta(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr, uint64_t *ids,
                  float *scores, uint64_t *count, float *threshold, uint64_t *stats);

/* Row-major host tables (row i at host + i*row_stride floats, row_stride >= d), the
 * layout of the reference's TPAr (cpu/TPAr.h: cdata[i*d + m]).  The rows are copied in
 * blocks and transposed on the device into the column-major table, so every query
 * entry serves them; TPAr's normalize (common/common.h:63-92) is the same arithmetic
 * per attribute as topk_normalize.  Replace filling TPAr's get_cdata() and reading it
 * back. */
int topk_upload_rowmajor(topk_table_t h, const float *host, uint64_t row_stride);
int topk_download_rowmajor(topk_table_t h, float *host, uint64_t row_stride);

/* Table files.  Replace File<T> (input/File.h).
 *
 * topk_csv_shape: the shape File<T>::count reads from a comma-separated file
 * (input/File.h:108-132): d = 1 + the commas of the first line, n = the number of
 * '\n' (a last line without one is not counted, as there).
 *
 * topk_load_csv: the first n rows of a comma-separated file into the table,
 * column-major, as File<T>::load with transpose (input/File.h:233-265, 306-330), each
 * value rounded to FP32 as fscanf's "%f" does (correctly rounded).  The text is parsed
 * on the device: the file streams through pinned buffers (chunk_bytes each, 0 = 16 MiB;
 * a line must fit in one) and each chunk is split into rows and parsed there; values
 * outside the device parser's exact range (more than 19 significant digits, exponents
 * beyond +-22 after scaling, inf, nan, hex; at most 2^20 per load) are converted on the
 * host with strtof.  Fields are separated by ',' with optional blanks, one object per
 * line, blank lines skipped.  Rows with fewer or more than d fields, fields that are not
 * numbers, or fewer than n rows return TOPK_ERR_ARG naming the row, and leave the table
 * without data.  stats (4 entries, may be NULL): bytes parsed, rows found, values
 * converted on the host, chunks.  The handle keeps the pipeline's buffers (two pinned
 * and two device chunk buffers with their row arrays) for later loads; loads and
 * row-major transfers on one handle take turns on them.
 *
 * topk_save_csv: the table as File<T>::store writes it (input/File.h:405-431): one
 * line per object, "%f" fields separated by ','.
 *
 * Binary column-major files (topk_save_binary / topk_load_binary / topk_binary_shape):
 * a 64-byte header ("TOPKCOL1", uint32 version 1, uint32 element size 4, uint64 n,
 * uint64 d, 32 reserved bytes), then the d columns of n FP32 values; loads stream
 * through pinned buffers.  The file's n and d must equal the table's. */
int topk_csv_shape(const char *path, uint64_t *n, uint64_t *d);
int topk_load_csv(topk_table_t h, const char *path, uint64_t chunk_bytes, uint64_t *stats);
int topk_save_csv(topk_table_t h, const char *path);
int topk_binary_shape(const char *path, uint64_t *n, uint64_t *d);
int topk_load_binary(topk_table_t h, const char *path);
int topk_save_binary(topk_table_t h, const char *path);

/* Exact top-k over all n objects with host inputs and host outputs (synchronous).
 * ids/scores must hold min(k, n) entries; count/threshold may be NULL.
 * Replaces findTopKscalar / findTopKsimd / findTopKthreads + get_res/get_thres. */
int topk_query(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr,
               uint64_t *ids, float *scores, uint64_t *count, float *threshold);

/* Same over rows [row_begin, row_end) only (one shard of the objects).
 * Ids stay global.  No reference counterpart: it is the per-shard step of an
 * object-sharded query. */
int topk_query_range(topk_table_t h, uint64_t row_begin, uint64_t row_end, uint64_t k, uint32_t qq,
                     const float *weights, const uint8_t *attr, uint64_t *ids, float *scores,
                     uint64_t *count, float *threshold);

/* Asynchronous form with DEVICE outputs on a caller stream (cudaStream_t passed
 * as void*; NULL = the handle's own stream).  d_ids/d_scores hold min(k, n)
 * entries; d_threshold (may be NULL) receives the k-th score.  Uses the handle's
 * primary scratch: calls on one handle must not overlap.  Same results as
 * topk_query. */
int topk_query_device(topk_table_t h, uint64_t k, uint32_t qq, const float *weights,
                      const uint8_t *attr, uint64_t *d_ids, float *d_scores, float *d_threshold,
                      void *stream);

/* topk_query_device over rows [row_begin, row_end) only (one shard of the objects):
 * d_ids/d_scores receive min(k, row_end - row_begin) entries with global ids.  No
 * reference counterpart: the device-side per-shard step of an object-sharded query
 * (topk_b200/shard.py), whose lists topk_merge_lists combines. */
int topk_query_range_device(topk_table_t h, uint64_t row_begin, uint64_t row_end, uint64_t k, uint32_t qq,
                            const float *weights, const uint8_t *attr, uint64_t *d_ids, float *d_scores,
                            float *d_threshold, void *stream);

/* Merge per-shard top-k lists on the device (one block, exact): list j starts at
 * d_lists + j * 12 * stride bytes and holds ids[stride] (uint64) then scores[stride]
 * (float); its first counts[j] entries are valid, and id_base[j] (host array, may be
 * NULL for all zero) is added to its ids -- a shard table numbers its rows from 0.
 * The best min(k, sum of counts) of the union -- score descending, ties to the lower
 * global id, the engine's order -- go to d_ids / d_scores ascending like every result,
 * the k-th score to d_threshold (may be NULL), their number to *kept.  Enqueued on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) on CUDA device
 * `device`.  nlists <= 64, k and stride <= TOPK_MAX_K, global ids < 2^32 - 1.
 * Replaces the merge of the per-thread heaps in TPAc::findTopKthreads
 * (cpu/TPAc.h:335-346) for shards held by different GPUs (the lists arrive by one
 * all_gather). */
int topk_merge_lists(int device, const void *d_lists, uint32_t nlists, uint64_t stride, const uint64_t *counts,
                     const uint64_t *id_base, uint64_t k, uint64_t *d_ids, float *d_scores, float *d_threshold,
                     uint64_t *kept, void *stream);

/* The same exact top-k as topk_query_device, for callers that must not allocate GPU
 * memory: no handle, no cudaMalloc/cudaFree, nothing from an allocating library.
 * It serves host applications that own the whole device memory budget and hand it
 * out through their own pool, and latency-critical paths that cannot pay for
 * cudaMalloc/cudaFree (both synchronise the device).  No counterpart in the
 * reference.  The caller passes a column-major table it owns (d_table, 16-byte
 * aligned, column m at d_table + m*ld, ld >= n and a multiple of 4, n < 2^32 - 1),
 * the query (host weights indexed by attribute id, host attr), and device outputs
 * for min(k, n) ids / scores (d_threshold may be NULL); work is enqueued on
 * `stream` (a cudaStream_t, NULL = the legacy default stream).  The scan's scratch
 * is a fixed array compiled into the library (about 8.4 MB on each GPU that loads
 * it, held until the process exits): k is limited to 1024 (TOPK_ERR_UNSUPPORTED
 * above), and calls whose work overlaps on the GPU share that array and race, so
 * serialise them.  The first call on each device performs a one-time set-up on
 * that device; make it before capturing work on that device.  The scan behind this
 * entry has no device-side wait that can give up, so a call that returns TOPK_OK
 * has enqueued work that always writes all its outputs; a kernel failure shows as a
 * CUDA error on `stream`.  Errors: the usual status codes, message from
 * topk_last_error(). */
int topk_query_noalloc(const float *d_table, uint64_t n, uint64_t ld, uint32_t d, uint64_t k, uint32_t qq,
                       const float *weights, const uint8_t *attr, uint64_t *d_ids, float *d_scores,
                       float *d_threshold, void *stream);

/* A batch of independent queries with host inputs/outputs (synchronous).
 * Query j uses ks[j], qqs[j], weights + j*wstride (indexed by attribute id),
 * attrs + j*astride.  Outputs: ids/scores + j*kstride (kstride >= max k),
 * counts[j], thresholds[j] (either may be NULL).  Replaces the multi-query
 * findTopKsimdMQ loop, and unlike it keeps every result. */
int topk_query_batch(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs,
                     const float *weights, uint64_t wstride, const uint8_t *attrs, uint64_t astride,
                     uint64_t *ids, float *scores, uint64_t kstride, uint64_t *counts,
                     float *thresholds);

/* Build a partitioned copy of the current table for pruned queries: the rows
 * reordered (Morton order of the attribute values) into partitions of part_rows
 * consecutive rows (a power of two in [1024, 2^24]), each with its per-attribute
 * min, max and mean, computed on the device.  Replaces the index build of
 * VTA::init / PTA::init (cpu/VTA.h:74-158, cpu/PTA.h:88-267).  Needs about
 * 4*(d+1)*n more bytes of device memory; rebuild after the table changes. */
int topk_build_partitions(topk_table_t h, uint32_t part_rows);

/* Orders of the partitioned copy. */
#define TOPK_ORDER_MORTON 0 /* Morton code of the attribute values (topk_build_partitions) */
#define TOPK_ORDER_VTA 1    /* VTA's order (cpu/VTA.h:121-135): each attribute's list sorted
                             * by value descending, each row's minimum position over the
                             * lists, rows by that position.  With part_rows = 1024 the
                             * partitions are VTA's blocks; their per-attribute max bounds
                             * every row of the block, at most the reference's tarray of
                             * the block before. */
#define TOPK_ORDER_PTA 2    /* PTA's order (cpu/PTA.h:88-167, 203-236): rows split into
                             * 2^(d-1) groups by the medians of their d-1 hyperspherical
                             * angles, each group in VTA's order, groups by number.
                             * Partitions are part_rows consecutive rows of that order, so
                             * one may span two groups (the reference starts a block at
                             * each group).  Needs n >= 2 and d <= 32. */
#define TOPK_ORDER_VTA_THREADS 3 /* VTA's order as its threaded build makes it (IMP 2, the
                                  * reference's default): 16 ranges of ceil(n/16) rows,
                                  * each in VTA's order on its own (cpu/VTA.h:13,78-85). */
#define TOPK_ORDER_SLA 4    /* SLA's order (cpu/SLA.h:102-139, 199-251): rows grouped by
                             * skyline layer (the skyline of 1 - x, peeled while more than
                             * 100 rows remain; see topk_skyline_layers), each layer in
                             * VTA's order, layers by number.  Needs d <= 32 and
                             * n <= TOPK_SKYLINE_MAX_ROWS; the layer build compares
                             * O(n^2 d) pairs. */
#define TOPK_ORDER_KD 5     /* No reference counterpart: the partitions are the leaves of a
                             * balanced binary tree over the rows; each node (a range of
                             * whole partitions) is split at its middle partition boundary
                             * after its rows are sorted, stably, by the attribute whose
                             * values spread widest in it (FP32 max - min, the lower
                             * attribute on a tie).  Boxes shrink in the attributes that
                             * vary most, so partition bounds are tighter than in the
                             * Morton order.  n < 2^31; about 20*n + 8*P*d bytes of scratch
                             * while it runs. */
/* In the VTA and PTA orders ties go to the lower row id (the reference's sorts are not
 * stable and leave them unspecified: rows sharing a minimum position, equal values);
 * PTA's angles order as their tangents, which are compared. */

/* topk_build_partitions with a choice of order.  The VTA and PTA orders sort on the
 * device (radix sorts, n < 2^31) and need about 20*n (VTA) or 32*n (VTA_THREADS, PTA)
 * bytes of scratch while they run. */
int topk_build_partitions_ordered(topk_table_t h, uint32_t part_rows, int order);

/* SLA's skyline layers (cpu/SLA.h:102-139), built on the device: layers[i] = the layer
 * of row i (0 = the skyline of the values 1 - x: no other row is <= in every attribute
 * and < in one); each next layer is the skyline of the rows left, and once at most 100
 * rows are left they form the last layer, as in the reference.  num_layers = the
 * count.  d <= 32 and n <= TOPK_SKYLINE_MAX_ROWS (2^22): the build compares
 * O(n^2 d) pairs, so larger tables return TOPK_ERR_UNSUPPORTED. */
#define TOPK_SKYLINE_MAX_ROWS (1ull << 22)
int topk_skyline_layers(topk_table_t h, uint32_t *layers, uint64_t *num_layers);

/* The partitioned copy's row ids (n entries): row i of the copy is row ids[i] of the
 * table. */
int topk_partition_ids(topk_table_t h, uint32_t *ids);

/* The partitions: count, rows each, and (arrays of num_parts*d, row p*d + m for
 * partition p, attribute m; any may be NULL) per-attribute min, max and mean. */
int topk_partition_info(topk_table_t h, uint32_t *num_parts, uint32_t *part_rows, float *mins, float *maxs,
                        float *means);

/* Exact top-k like topk_query, scanning only the partitions whose bound
 * sum_m weights[attr[m]] * (weight >= 0 ? max : min) can reach the threshold
 * (the stop rule of VTA/PTA::findTopK*, cpu/VTA.h:210-216, cpu/PTA.h:337-340).
 * cut: a predicted lower bound of the k-th score (e.g. from the learned model),
 * or NaN for none.  With a cut, one scan of the partitions reaching it; the
 * answer is accepted only if at least min(k, n) objects score >= cut, else the
 * plain two-round pruned method runs.  Results identical to topk_query.
 * stats (may be NULL): [0] partitions scanned, [1] partitions, [2] 1 if the cut
 * was accepted, [3] scans launched. */
int topk_query_pruned(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr, float cut,
                      uint64_t *ids, float *scores, uint64_t *count, float *threshold, uint64_t *stats);

/* ---- Learned k-th-score model (no reference counterpart) ------------------------
 * An MLP in_dim -> 64 -> 64 -> 1 (ReLU, FP32) predicting u = qq * ln(gap / S) of a
 * query, gap = (largest partition bound) - (k-th score), S = sum_m
 * |weights[attr[m]]|, from in_dim = 2d + 18 features: the query's weight per
 * attribute / S, ln of those (0 where not queried), log2(k) / 10, qq / 16, the 1st,
 * 2nd, 4th .. 128th largest partition bound / S and the same ranks of the partition
 * mean scores / S (needs d <= 23).  The cut of a prediction
 * is largest bound - S * exp((u + margin) / qq).  Parameters are one FP32 array:
 * W1[64][in_dim] b1[64] W2[64][64] b2[64] w3[64] b3.  Training and inference run
 * in this library's own kernels.  The cut is only a starting threshold: the
 * pruned and batched queries accept it when enough objects reach it, so results
 * never depend on the model. */
#define TOPK_MLP_HIDDEN 64u
#define TOPK_MLP_MAX_IN 64u

/* Number of parameters of the model for in_dim inputs. */
uint64_t topk_mlp_param_count(uint32_t in_dim);

/* Mean squared error over one batch (<= 128 samples, X row-major batch x in_dim)
 * and its gradient with respect to every parameter, computed on CUDA device
 * `device`; no update.  For checking the training kernels against a reference. */
int topk_mlp_grad(int device, uint32_t in_dim, const float *params, const float *X, const float *y, uint32_t batch,
                  float *grad, float *loss);

/* Predictions for n samples. */
int topk_mlp_predict(int device, uint32_t in_dim, const float *params, const float *X, uint64_t n, float *out);

/* Train in place with Adam (lr, batch <= 128) for `epochs` passes over n samples
 * in a seeded order; epoch_loss (may be NULL) receives each epoch's mean loss. */
int topk_mlp_train(int device, uint32_t in_dim, float *params, const float *X, const float *y, uint64_t n,
                   uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float *epoch_loss);

/* Features of nq queries (layout of topk_query_batch's arguments) from the current
 * partitions: X receives nq rows of 2d + 18 values; scale (may be NULL) receives S. */
int topk_query_features(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs, const float *weights,
                        uint64_t wstride, const uint8_t *attrs, uint64_t astride, float *X, float *scale);

/* Install (params != NULL) or remove the handle's model and its margin (in units
 * of u, see above). */
int topk_set_learned_model(topk_table_t h, const float *params, float margin);

/* Copy the handle's model out (params may be NULL). */
int topk_get_learned_model(topk_table_t h, float *params, float *margin);

/* Fit the handle's model: n_train + n_val random queries (attribute subsets of
 * size U{qmin..qmax}, weights U(0,1], k log-uniform in [kmin, kmax], seeded),
 * labelled with their exact k-th scores by topk_query_batch, features on the
 * device, `epochs` of Adam on the device, then the margin = the (1 - miss_rate)
 * quantile of (target - prediction) over the n_val held-out queries.
 * report (may be NULL, 6 values): last epoch's loss, held-out RMSE, margin,
 * held-out miss rate at that margin, labelling seconds, training seconds. */
int topk_learned_fit(topk_table_t h, uint64_t n_train, uint64_t n_val, uint32_t kmin, uint32_t kmax, uint32_t qmin,
                     uint32_t qmax, uint32_t epochs, float miss_rate, uint64_t seed, double *report);

/* Exact top-k through the model: features and the MLP forward in one kernel give
 * the cut, then topk_query_pruned(cut).  Same results as
 * topk_query; stats as topk_query_pruned; cut_out (may be NULL) receives the cut. */
int topk_query_learned(topk_table_t h, uint64_t k, uint32_t qq, const float *weights, const uint8_t *attr,
                       uint64_t *ids, float *scores, uint64_t *count, float *threshold, uint64_t *stats,
                       float *cut_out);

/* Verification entry (no reference counterpart): copy the full rows of `count`
 * objects to host memory, out[j*d + m] = attribute m of object ids[j]. */
int topk_gather_rows(topk_table_t h, const uint64_t *ids, uint64_t count, float *out);

/* Verification entry (no reference counterpart): with a plain kernel independent
 * of the fused scan, count objects in rows [row_begin, row_end) whose
 * reference-order score is >= thr and > thr.  For a correct top-k over all rows,
 * count_gt < k <= count_ge at thr = the k-th score. */
int topk_count_ge(topk_table_t h, uint64_t row_begin, uint64_t row_end, uint32_t qq, const float *weights,
                  const uint8_t *attr, float thr, uint64_t *count_ge, uint64_t *count_gt);

/* Tuning entry (no reference counterpart): the most CTAs of the fused scan per SM
 * (0 = as many as fit, up to 8).  Results do not depend on it. */
int topk_set_scan_tuning(topk_table_t h, uint32_t max_ctas_per_sm);

/* Test entry (no reference counterpart): mode 1 makes the next fused scans wait,
 * before any copy is issued, on a barrier that nothing completes, so the bounded
 * wait runs out and the call returns TOPK_ERR_TIMEOUT; 0 turns it off.  Host-side
 * fault injection: no GPU fault, the context stays usable. */
int topk_set_fault_injection(topk_table_t h, int mode);

/* Methods of topk_query_batch (no reference counterpart; results are identical). */
#define TOPK_BATCH_AUTO 0  /* TOPK_BATCH_LEARNED with a fitted model, else TOPK_BATCH_BF16
                            * where it applies, else TOPK_BATCH_FP32.  Once a BF16 batch
                            * hands more than three quarters of its queries to the FP32
                            * scorer (scores too dense around the thresholds, e.g.
                            * anticorrelated data), later AUTO batches on the same table
                            * use the FP32 scorer from the start */
#define TOPK_BATCH_LOOP 1  /* one fused single-query scan per query */
#define TOPK_BATCH_FP32 2  /* batched plain FP32: each table tile scored for 64 queries */
#define TOPK_BATCH_BF16 3  /* BF16 tensor-core filter (tcgen05) with a per-query error
                            * bound; candidates rescored exactly in FP32.  Applies to
                            * d <= 16 with finite table values and weights of magnitude
                            * <= 2^60; other batches run TOPK_BATCH_FP32.  Hybrid: a
                            * query for which the filter passes too much (tied or dense
                            * scores at its threshold: more than 2k + 2048 candidates in
                            * a chunk, or lost ones) moves to the exact FP32 scorer for
                            * the rest of the batch, inside the same call */
#define TOPK_BATCH_LEARNED 4 /* TOPK_BATCH_BF16 (or FP32) whose per-query threshold starts
                              * at the learned cut (prediction - margin) * S instead of a
                              * bootstrap over the first rows; a query left with fewer
                              * than k objects at or above its cut runs again without it.
                              * Needs a model on the current partitions
                              * (topk_learned_fit / topk_set_learned_model); without one
                              * it runs as TOPK_BATCH_BF16 */

/* Choose the method of topk_query_batch on this handle. */
int topk_set_batch_method(topk_table_t h, int method);

/* Tiles of the batched path (no reference counterpart; results never depend on
 * them): query tiles of 128 per BF16-filter CTA (1..16, 0 = up to 16) and rows of the
 * exact bootstrap, which is also the first chunk (a multiple of 256 in [256, 16384];
 * default 8192). */
int topk_set_batch_tiles(topk_table_t h, uint32_t qt_per_cta, uint32_t boot_rows);
int topk_get_batch_tiles(topk_table_t h, uint32_t *qt_per_cta, uint32_t *boot_rows);

/* Autotuner of the batched path: runs the caller's queries (arguments as in
 * topk_query_batch, with the handle's current method) under query tiles per CTA of
 * 4, 8 and 16 and bootstraps of 8192 and 16384 rows, each twice, keeps the fastest
 * device time in the handle and reports {query tiles, bootstrap rows, best ms, ms of
 * the default 16 / 8192}.  Twelve batches: call it once per workload shape. */
int topk_tune_batch(topk_table_t h, uint64_t nq, const uint64_t *ks, const uint32_t *qqs, const float *weights,
                    uint64_t wstride, const uint8_t *attrs, uint64_t astride, double *report);

/* Statistics of the handle's last topk_query_batch: device time of the batched
 * kernels (CUDA events; 0 for the loop method), queries answered again by the
 * single-query scan after a candidate overflow, candidates appended by the
 * scorer over all chunks. */
int topk_last_batch_stats(topk_table_t h, double *device_ms, uint64_t *fallbacks, uint64_t *candidates);

/* More about the last topk_query_batch: the method that ran (TOPK_BATCH_*), for the
 * BF16 filter the largest |filter score - exact score| / bound seen over the
 * rescored candidates (must stay below 1; 0 for the other methods), and the
 * queries whose learned start was too high (answered again without it). */
int topk_last_batch_info(topk_table_t h, int *method, double *max_err_ratio, uint64_t *learned_misses);

/* How many queries of the last topk_query_batch the hybrid BF16 batch moved to the
 * exact FP32 scorer (0 for the other methods). */
int topk_last_batch_switched(topk_table_t h, uint64_t *switched);

/* How many queries of the last topk_query_batch the BF16 filter retired before the
 * table's end: their k-th score had reached the largest score any object can have
 * (the reference-order sum over the column extremes), so no later object could enter
 * their top-k and the filter stopped serving them -- the reference's stop rule
 * (cpu/VTA.h:210-216, cpu/PTA.h:636-641) with the whole table as the block.  0 for the
 * other methods. */
int topk_last_batch_retired(topk_table_t h, uint64_t *retired);

/* The tensor-core work the last topk_query_batch ran under the BF16 filter: for every
 * chunk, its served query tiles (128 queries each) times its object tiles (256 rows),
 * three BF16 MMA passes of 2 * 16 flops per (query, object).  0 for the other methods.
 * No reference counterpart (a measurement of this engine). */
int topk_last_batch_filter_flops(topk_table_t h, double *flops);

/* Device-side scan statistics of the last topk_query* on this thread:
 * candidates kept by the fused select and the number of block reductions. */
int topk_last_stats(topk_table_t h, uint64_t *candidates, uint64_t *reductions);

/* Bound (in polling iterations) on every device-side wait; 0 restores the default.
 * A wait that runs out makes the call return TOPK_ERR_TIMEOUT. */
int topk_set_wait_limit(topk_table_t h, uint64_t iterations);

/* Table shape and device stride. */
int topk_shape(topk_table_t h, uint64_t *n, uint32_t *d, uint64_t *ld);

/* Message for the last error on the calling thread ("" if none). */
const char *topk_last_error(void);

/* Name of a status code. */
const char *topk_status_name(int status);

/* Library version string. */
const char *topk_version(void);

#ifdef __cplusplus
}
#endif
#endif /* TOPK_B200_H */
