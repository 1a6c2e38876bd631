/*
 * lgbm_b200 — a B200 (sm_100a) tree-learning path for lightgbm-rust.
 *
 * C ABI of the drop-in. Each entry point replaces one call the Rust host
 * (crates/lgbm-core) makes on its CPU path; the comment above each names
 * the reference interface (path relative to the lightgbm-rust project):
 *
 *   SerialTreeLearner::new            crates/lgbm-core/src/learner/mod.rs:220
 *   SerialTreeLearner::set_bagging_data                       learner/mod.rs:545
 *   ColSampler::reset_by_tree (mask)  crates/lgbm-core/src/learner/col_sampler.rs:88
 *   SerialTreeLearner::train          learner/mod.rs:572
 *   SerialTreeLearner::add_leaf_outputs                       learner/mod.rs:537
 *   SerialTreeLearner::partition      learner/mod.rs:312
 *   RowObjective::gradients           crates/lgbm-core/src/objective/mod.rs:52
 *   Gbdt::train_one_iter (device-resident loop)     crates/lgbm-core/src/boosting.rs:957
 *   Gbdt::predict_matrix_early_stop   crates/lgbm-core/src/predict.rs:231
 *
 * Conventions:
 *   - every call returns an int status: LGBM_B200_OK or an LGBM_B200_ERR_*
 *     code whose kind matches the reference's LgbmError variants
 *     (crates/lgbm-core/src/error.rs:5-18); lgbm_b200_last_error() gives the
 *     message of the last failure on the calling thread;
 *   - device buffers are owned by the handle; host buffers passed in are
 *     only read (or written) during the call;
 *   - one CUDA stream per handle; a handle is not thread-safe;
 *   - every device-side wait is bounded and reports LGBM_B200_ERR_TIMEOUT;
 *   - `location` arguments say whether a pointer is host memory
 *     (LGBM_B200_HOST) or device memory of the handle's GPU (LGBM_B200_DEVICE).
 */
#ifndef LGBM_B200_H_
#define LGBM_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LGBM_B200_OK 0
#define LGBM_B200_ERR_INVALID_PARAMETER 1
#define LGBM_B200_ERR_INVALID_DATA 2
#define LGBM_B200_ERR_MODEL_FORMAT 3
#define LGBM_B200_ERR_UNSUPPORTED 4
#define LGBM_B200_ERR_INTERNAL 5
#define LGBM_B200_ERR_CUDA 6
#define LGBM_B200_ERR_TIMEOUT 7

#define LGBM_B200_HOST 0
#define LGBM_B200_DEVICE 1

/* Histogram accumulation forms. */
#define LGBM_B200_HIST_F64 0   /* FP64 sums of f32 gradients (the reference's form) */
#define LGBM_B200_HIST_F32C 1  /* FP32 two-float compensated partials, merged in FP64 */
#define LGBM_B200_HIST_QUANT 2 /* int8 quantized gradients, int16/int32 integer histograms */

#define LGBM_B200_OBJ_BINARY 0
#define LGBM_B200_OBJ_REGRESSION 1 /* L2 */
#define LGBM_B200_OBJ_MULTICLASS 2 /* softmax */
#define LGBM_B200_OBJ_LAMBDARANK 3

const char* lgbm_b200_last_error(void);
/* Library version string. */
const char* lgbm_b200_version(void);

/* ------------------------------------------------------------------------
 * Binned dataset (host). Stands in for the Rust host's Dataset
 * (crates/lgbm-core/src/dataset.rs:355 Dataset::from_dense with the bin
 * mappers of binning.rs): it produces the u8 feature-group bin matrix the
 * learner uploads once. Only dense single-feature groups are supported.
 * ------------------------------------------------------------------------ */
typedef struct LgbmB200Dataset LgbmB200Dataset;

typedef struct {
  int32_t max_bin, min_data_in_bin, min_data_in_leaf, bin_construct_sample_cnt, data_random_seed;
  int32_t use_missing, zero_as_missing, feature_pre_filter;
  const int32_t* categorical; /* column indices of categorical features */
  int32_t num_categorical;
} LgbmB200BinParams;

typedef struct {
  int64_t num_data;
  int32_t num_features;       /* used (non-trivial) features, the learner's inner features */
  int32_t num_total_features; /* columns of the input matrix */
  const uint8_t* bins;        /* row-major [num_data x num_features] stored group values */
  const int32_t* num_bin;
  const int32_t* missing_type; /* 0 none, 1 zero, 2 NaN */
  const int32_t* default_bin;
  const int32_t* most_freq_bin;
  const int32_t* bin_type; /* 0 numerical, 1 categorical */
  const int32_t* real_index;
  const double* upper_bounds; /* numerical bin upper bounds, feature f at [ub_offsets[f], ub_offsets[f+1]) */
  const int64_t* ub_offsets;
  const int32_t* bin_to_cat; /* categorical bin -> category, feature f at [cat_offsets[f], cat_offsets[f+1]) */
  const int64_t* cat_offsets;
} LgbmB200DatasetView;

/* Dataset::from_dense (dataset.rs:355): X is row-major f32 [n x ncol]. */
int lgbm_b200_dataset_create(const float* X, int64_t n, int32_t ncol, const LgbmB200BinParams* params,
                             LgbmB200Dataset** out);
/* Dataset::from_dense_with_reference (dataset.rs:446): bins with `ref`'s mappers. */
int lgbm_b200_dataset_create_valid(const float* X, int64_t n, int32_t ncol, const LgbmB200Dataset* ref,
                                   LgbmB200Dataset** out);
/* The same two builds with the rows binned on CUDA device `device`
 * (value_to_bin, binning.rs:637-667, and the group push,
 * feature_group.rs:144-154, as a kernel over every row and used feature).
 * The bin mappers are still found on the host from the row sample, and the
 * resulting dataset is identical, byte for byte, to the host build's. Fails
 * with LGBM_B200_ERR_UNSUPPORTED when a categorical feature holds a category
 * value of 2^22 or more (the device keeps a dense table per feature). */
int lgbm_b200_dataset_create_device(const float* X, int64_t n, int32_t ncol, const LgbmB200BinParams* params,
                                    int32_t device, LgbmB200Dataset** out);
int lgbm_b200_dataset_create_valid_device(const float* X, int64_t n, int32_t ncol, const LgbmB200Dataset* ref,
                                          int32_t device, LgbmB200Dataset** out);
/* The view points into the dataset; valid until lgbm_b200_dataset_free. */
int lgbm_b200_dataset_view(LgbmB200Dataset* ds, LgbmB200DatasetView* out);
/* Dataset::feature_infos (dataset.rs:770-776) as the model text's
 * feature_infos line holds it: one entry per input column, space-separated
 * ("[min:max]" for a numerical feature, its categories joined by ':' for a
 * categorical one, "none" for an unused column). *out stays valid until
 * lgbm_b200_dataset_free. */
int lgbm_b200_dataset_feature_infos(LgbmB200Dataset* ds, const char** out);
void lgbm_b200_dataset_free(LgbmB200Dataset* ds);

/* ------------------------------------------------------------------------
 * Evaluation metrics on the device (Metric::eval, metric.rs:520-770), so
 * that validation scores kept on the device need not be copied back every
 * iteration. Unweighted labels. AUC (metric.rs:701-731) is exact and equals
 * the reference's value bit for bit; the loss metrics are FP64 means whose
 * summation order differs from the reference's sequential loop.
 * ------------------------------------------------------------------------ */
enum {
  LGBM_B200_METRIC_AUC = 0,
  LGBM_B200_METRIC_BINARY_LOGLOSS = 1, /* on 1 / (1 + exp(-sigmoid * score)) (binary.rs:164-166) */
  LGBM_B200_METRIC_BINARY_ERROR = 2,
  LGBM_B200_METRIC_L2 = 3,
  LGBM_B200_METRIC_RMSE = 4,
  LGBM_B200_METRIC_MULTI_LOGLOSS = 5,  /* on the softmax of class-major scores [num_class x n] */
  LGBM_B200_METRIC_MULTI_ERROR = 6
};

typedef struct {
  int32_t metric;            /* LGBM_B200_METRIC_* */
  int32_t num_class;         /* multiclass metrics */
  double sigmoid;            /* binary metrics: the objective's sigmoid */
  int32_t multi_error_top_k; /* multi_error: a row counts as an error when more than top_k classes score >= its label's */
} LgbmB200MetricConfig;

/* The metric of `score` against `label` (n rows; multiclass scores are
 * class-major, n x num_class values) into *out. location: LGBM_B200_HOST
 * or LGBM_B200_DEVICE for both buffers. */
int lgbm_b200_metric_eval(const LgbmB200MetricConfig* cfg, const float* label, const double* score, int64_t n,
                          int32_t location, int32_t device, double* out);
/* NDCG@eval_at[j] (metric.rs:546-598, dcg.rs; no query weights) into
 * out[j]: per query the stable descending order of the scores and the best
 * DCG from the label counts, the mean over queries. query_boundaries is host
 * memory ([num_queries + 1], from 0); labels are integers in [0, 30]. */
int lgbm_b200_metric_ndcg(const float* label, const double* score, const int32_t* query_boundaries,
                          int32_t num_queries, const int32_t* eval_at, int32_t num_eval_at, int32_t location,
                          int32_t device, double* out);

/* ------------------------------------------------------------------------
 * Tree learner.
 * ------------------------------------------------------------------------ */
typedef struct LgbmB200Learner LgbmB200Learner;

typedef struct {
  int32_t num_leaves, max_depth, min_data_in_leaf;
  double min_sum_hessian_in_leaf, lambda_l1, lambda_l2, max_delta_step, path_smooth, min_gain_to_split;
  int32_t max_cat_to_onehot, max_cat_threshold;
  double cat_l2, cat_smooth;
  int32_t min_data_per_group;
  double monotone_penalty;
  int32_t hist_precision; /* LGBM_B200_HIST_* */
  /* quantized gradients (learner/quant.rs) */
  int32_t num_grad_quant_bins, stochastic_rounding, quant_train_renew_leaf, seed;
  int32_t quant_num_threads; /* the reference's num_threads: shapes its stochastic-rounding tables */
  int32_t is_constant_hessian;
  /* trees grown together in lockstep (multiclass: num_class; otherwise 1) */
  int32_t num_tree_slots;
  int32_t device;
  /* launch shape knobs; 0 picks the built-in defaults */
  int32_t hist_rows_per_block, hist_block_threads, use_cuda_graph;
  /* 1: grow each tree in one persistent cooperative launch (grid barriers
   * between the split phases); 0: one launch per kernel per split step */
  int32_t persistent_grow;
} LgbmB200LearnerConfig;

typedef struct {
  int32_t num_bin, missing_type, default_bin, most_freq_bin, bin_type, monotone_type, real_index;
  double penalty; /* feature_contri */
} LgbmB200FeatureMeta;

/* One trained tree in the reference's Tree layout (crates/lgbm-core/src/tree.rs:120-160).
 * Pointers are owned by the learner and stay valid until its next train call. */
typedef struct {
  int32_t num_leaves;
  const int32_t* split_feature_inner;
  const int32_t* split_feature;
  const float* split_gain;
  const uint32_t* threshold_in_bin;
  const double* threshold;
  const int8_t* decision_type;
  const int32_t* left_child;
  const int32_t* right_child;
  const int32_t* leaf_parent;
  const double* leaf_value; /* before shrinkage */
  const double* leaf_weight;
  const int32_t* leaf_count;
  const int32_t* leaf_depth;
  const double* internal_value;
  const double* internal_weight;
  const int32_t* internal_count;
  int32_t num_cat;
  const int32_t* cat_boundaries;       /* num_cat + 1 */
  const uint32_t* cat_threshold;       /* category bitsets */
  const int32_t* cat_boundaries_inner; /* num_cat + 1 */
  const uint32_t* cat_threshold_inner; /* bin bitsets */
  /* the FP64 gain of each split before split_gain rounds it to f32 (the
   * reference keeps only the f32; for parity checks). May be NULL in views a
   * caller passes in. */
  const double* split_gain_f64;
} LgbmB200TreeView;

/* SerialTreeLearner::new (learner/mod.rs:220): uploads the bin matrix
 * (row-major u8 [num_data x num_features]) once. upper_bounds/bin_to_cat
 * (laid out as in LgbmB200DatasetView) give the real-valued thresholds and
 * category bitsets of the returned trees; either may be NULL. */
int lgbm_b200_learner_create(const LgbmB200LearnerConfig* cfg, const uint8_t* bins, int64_t num_data,
                             int32_t num_features, const LgbmB200FeatureMeta* metas, const double* upper_bounds,
                             const int64_t* ub_offsets, const int32_t* bin_to_cat, const int64_t* cat_offsets,
                             LgbmB200Learner** out);
void lgbm_b200_learner_destroy(LgbmB200Learner* h);

/* set_bagging_data(used, subset=false) (learner/mod.rs:545): `used` holds
 * the in-bag rows in ascending order; NULL trains on every row. */
int lgbm_b200_learner_set_bagging(LgbmB200Learner* h, const uint32_t* used, int64_t num_used, int32_t location);

/* The by-tree feature mask of ColSampler::reset_by_tree (col_sampler.rs:88)
 * for tree slot `slot`; NULL uses every feature. */
int lgbm_b200_learner_set_feature_mask(LgbmB200Learner* h, int32_t slot, const uint8_t* is_used);

/* train(grad, hess, is_first_tree) (learner/mod.rs:572) for every tree
 * slot: grad/hess are class-major [num_tree_slots x num_data]. `out`
 * receives num_tree_slots views. is_first_tree is accepted as the reference
 * takes it; there it only keeps linear-tree leaves constant, and linear
 * trees are not on this path. */
int lgbm_b200_learner_train(LgbmB200Learner* h, const float* grad, const float* hess, int32_t is_first_tree,
                            int32_t location, LgbmB200TreeView* out);

/* add_leaf_outputs(leaf_values, score) (learner/mod.rs:537) for slot
 * `slot`: score[row] += leaf_values[leaf of row] over the in-bag rows. */
int lgbm_b200_learner_add_leaf_outputs(LgbmB200Learner* h, int32_t slot, const double* leaf_values,
                                       int32_t num_leaves, double* score, int32_t location);

/* partition() (learner/mod.rs:312): the rows of each leaf of the last tree
 * of `slot`. leaf_begin/leaf_count: [num_leaves]; indices: [num_used]. Each
 * leaf's rows are in ascending order, as the reference's stable partition
 * keeps them (partition.rs:107-174). */
int lgbm_b200_learner_get_partition(LgbmB200Learner* h, int32_t slot, int32_t* leaf_begin, int32_t* leaf_count,
                                    uint32_t* indices);

/* ------------------------------------------------------------------------
 * Data-parallel growth: the rows are sharded over ranks (one learner per
 * rank and GPU, each created on its own rows, all with the same bin
 * mappers); the trees are the ones a single learner grows on all rows. The
 * reference's learner is serial and has no counterpart; this follows the
 * data-parallel scheme of its upstream (LightGBM's data-parallel tree
 * learner: a histogram all-reduce per split). Per tree the ranks reduce:
 * the quantization maxima (max), the root sums, each split step's smaller-
 * leaf histogram, the rows each step sends left, and the leaf renewal sums
 * (sums). The learner calls `fn` for each reduction, on a device buffer of
 * its own device, after synchronising its stream; fn must reduce the buffer
 * in place over every rank (same call order on every rank) and return 0
 * once the result is in the buffer. One tree slot only (not multiclass); no
 * bagging; growth runs step by step (no CUDA graph).
 * ------------------------------------------------------------------------ */
enum { LGBM_B200_DT_INT64 = 0, LGBM_B200_DT_FLOAT64 = 1, LGBM_B200_DT_INT32 = 2 };
enum { LGBM_B200_OP_SUM = 0, LGBM_B200_OP_MAX = 1 };
typedef int32_t (*LgbmB200AllReduceFn)(void* device_buf, int64_t count, int32_t dtype, int32_t op, void* user);
/* row_offset: this rank's first row in the global row order; global_num_data:
 * every rank's rows. Call once, after lgbm_b200_learner_create. */
int lgbm_b200_learner_set_data_parallel(LgbmB200Learner* h, int64_t row_offset, int64_t global_num_data,
                                        LgbmB200AllReduceFn fn, void* user);

/* Launch shape of the per-split-step kernels (the default launch strategy;
 * the persistent one has none). No field changes a result: the shapes differ
 * only in speed. No counterpart in the reference, whose CPU learner has a
 * thread count instead. */
typedef struct {
  int32_t partition_ctas;      /* CTAs of the row partition per tree slot, in [1, 65535] */
  int32_t hist_ctas;           /* histogram CTAs per tree slot and feature tile, in [1, 65535];
                                  rounded up to a multiple of the histogram cluster size */
  int32_t hist_rows_per_block; /* least rows a histogram CTA takes, in [32, 1 << 24] */
} LgbmB200LaunchShape;

int lgbm_b200_learner_get_launch_shape(LgbmB200Learner* h, LgbmB200LaunchShape* out);
int lgbm_b200_learner_set_launch_shape(LgbmB200Learner* h, const LgbmB200LaunchShape* shape);

/* The autotuner's measurement: regrows the trees of the last train call
 * (the same gradients and quantization offsets, so the same trees) under each
 * candidate shape, `reps` timed times after one untimed replay, writes each
 * candidate's median device ms per tree to ms_per_tree[i], and keeps the
 * fastest (its index in *chosen). The random streams of later train calls
 * are untouched. Requires a train call before it; not with persistent_grow. */
int lgbm_b200_learner_autotune(LgbmB200Learner* h, const LgbmB200LaunchShape* candidates, int32_t num_candidates,
                               int32_t reps, int32_t* chosen, double* ms_per_tree);

/* Per-kernel timing: when enabled, every split step of the next train calls
 * is bracketed by CUDA events on the learner's stream (no extra syncs). */
int lgbm_b200_learner_set_timing(LgbmB200Learner* h, int32_t enabled);
/* Timing marks: record event `mark` (0..15) on the learner's stream; the
 * elapsed device time between two recorded marks, in ms. */
int lgbm_b200_learner_record(LgbmB200Learner* h, int32_t mark);
int lgbm_b200_learner_elapsed(LgbmB200Learner* h, int32_t a, int32_t b, double* ms);
/* Device time of the last train call summed per kernel family, ms:
 * [histogram, scan, partition, other]; rows histogrammed; kernels launched. */
int lgbm_b200_learner_last_timing(LgbmB200Learner* h, double* ms, int64_t* hist_rows, int32_t* launches);
/* With timing on (lgbm_b200_learner_set_timing), the device time of the
 * histogram, scan and partition launches of every split step of the last
 * train call: ms[3 * step + {0, 1, 2}] for step < min(*steps, capacity).
 * Histogram step s builds the smaller child of split s - 1 (step 0: the
 * root). A diagnostic with no counterpart in the reference. */
int lgbm_b200_learner_step_times(LgbmB200Learner* h, float* ms, int32_t capacity, int32_t* steps);
/* Rows of the last train call: histogrammed by the histogram kernel, and
 * moved by the partition. For the bench's bandwidth figures; no
 * counterpart in the reference. */
int lgbm_b200_learner_last_rows(LgbmB200Learner* h, int64_t* hist_rows, int64_t* partition_rows);

/* Diagnostics for the parity tests. lgbm_b200_learner_histogram runs the
 * learner's histogram kernel over `rows` (NULL: every row) of slot `slot`'s
 * gradients from the last train call (quantized form: its packed values) and
 * writes the histogram in the learner's layout: per inner feature its
 * num_bin - offset stored bins, FP64 [g, h] pairs (F64 / F32C forms) or packed
 * (g << 32) + h int64 sums (quantized form). lgbm_b200_learner_quantized
 * returns the last packed quantized gradients and [grad_scale, hess_scale]
 * (learner/quant.rs:411-448). These replace no reference call. */
int lgbm_b200_learner_histogram(LgbmB200Learner* h, int32_t slot, const uint32_t* rows, int64_t num_rows,
                                void* out);
int lgbm_b200_learner_quantized(LgbmB200Learner* h, int32_t slot, int64_t* packed, double* scales);

/* ------------------------------------------------------------------------
 * Objective gradients: RowObjective::gradients (objective/mod.rs:52) for
 * binary (binary.rs:101), L2 (regression.rs:209), softmax (multiclass.rs:126)
 * and lambdarank (rank.rs:192). scores/grad/hess are class-major. Lambdarank
 * takes query_boundaries in host memory ([num_queries + 1], from 0 to
 * num_data; at most 10000 rows per query) and builds the objective's tables
 * (rank.rs:119-176) on each call; other objectives ignore them.
 * ------------------------------------------------------------------------ */
typedef struct {
  int32_t objective; /* LGBM_B200_OBJ_* */
  int32_t num_class;
  double sigmoid;
  int32_t lambdarank_truncation_level, lambdarank_norm;
} LgbmB200ObjectiveConfig;

int lgbm_b200_gradients(const LgbmB200ObjectiveConfig* cfg, const float* label, const double* scores,
                        int64_t num_data, const int32_t* query_boundaries, int32_t num_queries, float* grad,
                        float* hess, int32_t location, int32_t device);

/* An objective bound to its labels once (RowObjective::init,
 * objective/mod.rs:50): the labels (and the lambdarank tables) stay on the
 * device, and each RowObjective::gradients call (objective/mod.rs:52) moves
 * only the scores in and the gradients out. label and query_boundaries are
 * host memory. */
typedef struct LgbmB200Objective LgbmB200Objective;
int lgbm_b200_objective_create(const LgbmB200ObjectiveConfig* cfg, const float* label, int64_t num_data,
                               const int32_t* query_boundaries, int32_t num_queries, int32_t device,
                               LgbmB200Objective** out);
/* scores [k x num_data] in, grad / hess [k x num_data] out, all at `location`. */
int lgbm_b200_objective_gradients(LgbmB200Objective* obj, const double* scores, float* grad, float* hess,
                                  int32_t location);
void lgbm_b200_objective_free(LgbmB200Objective* obj);

/* ------------------------------------------------------------------------
 * Device-resident boosting: Gbdt::train_one_iter (boosting.rs:957) with the
 * gradients, bagging draw (sample_strategy.rs:280-320), tree learner and
 * score updates (boosting.rs:1381-1408) on the GPU. The host gets each
 * iteration's trees back.
 * ------------------------------------------------------------------------ */
typedef struct LgbmB200Booster LgbmB200Booster;

typedef struct {
  LgbmB200ObjectiveConfig objective;
  double learning_rate;
  int32_t boost_from_average;
  double bagging_fraction;
  int32_t bagging_freq, bagging_seed;
  double feature_fraction;
  int32_t feature_fraction_seed;
} LgbmB200BoostConfig;

/* `learner` stays owned by the caller and must outlive the booster. label: host
 * [num_data]; query_boundaries: host [num_queries + 1] for lambdarank (NULL
 * otherwise); valid_bins: optional held-out bin matrix [num_valid x
 * num_features] scored every iteration like the reference's valid sets. */
int lgbm_b200_booster_create(LgbmB200Learner* learner, const LgbmB200BoostConfig* cfg, const float* label,
                             const int32_t* query_boundaries, int32_t num_queries, const uint8_t* valid_bins,
                             int64_t num_valid, LgbmB200Booster** out);
void lgbm_b200_booster_destroy(LgbmB200Booster* b);
/* One iteration; *stop is set when no tree could split. `out` receives the
 * iteration's num_tree_slots trees (after shrinkage and bias, as stored). */
int lgbm_b200_booster_train_iter(LgbmB200Booster* b, int32_t* stop, LgbmB200TreeView* out);
/* Scores (class-major): which = 0 training, 1 validation. */
int lgbm_b200_booster_scores(LgbmB200Booster* b, int32_t which, double* out, int32_t location);
/* Start-of-training score per class added by boost_from_average. */
int lgbm_b200_booster_init_scores(LgbmB200Booster* b, double* out);

/* ------------------------------------------------------------------------
 * Batched prediction: Gbdt::predict_matrix_early_stop (predict.rs:231) with
 * PredictKind::Raw on row-major f32 features. The forest is uploaded once.
 * ------------------------------------------------------------------------ */
typedef struct LgbmB200Forest LgbmB200Forest;

/* Trees in model order; a tree with num_leaves == 1 contributes leaf_value[0]. */
int lgbm_b200_forest_create(const LgbmB200TreeView* trees, int32_t num_trees, int32_t num_tree_per_iteration,
                            int32_t device, LgbmB200Forest** out);
void lgbm_b200_forest_destroy(LgbmB200Forest* f);
/* out: row-major [nrow x num_tree_per_iteration] raw scores. */
int lgbm_b200_predict(LgbmB200Forest* f, const float* X, int64_t nrow, int32_t ncol, double* out,
                      int32_t location);

/* lgbm_b200_predict with HOST buffers (X and out in host memory) that
 * allocates no device memory; it has no counterpart in the reference. It is
 * for callers that cannot allocate while they predict: a serving process
 * whose free device memory is held by another allocator, or a
 * latency-bound thread that must not wait on allocation or on the
 * synchronisation that freeing memory can bring. Rows and scores go
 * through one 16 MiB array in device memory compiled into the library, in
 * chunks of rows; a row needing more than 16 MiB - 256 bytes of staging
 * (4 x ncol + 8 x num_tree_per_iteration) is rejected with
 * LGBM_B200_ERR_INVALID_PARAMETER. The array is shared by every call on a
 * device: calls that overlap in time on one device race on it and must be
 * serialised by the caller. The first call on a device resolves the array's
 * address (cudaGetSymbolAddress); make it before capturing any stream on
 * that device. The calling thread's current device is left as it was.
 * Results equal lgbm_b200_predict's. */
int lgbm_b200_predict_noalloc(LgbmB200Forest* f, const float* X, int64_t nrow, int32_t ncol, double* out);

#ifdef __cplusplus
}
#endif

#endif /* LGBM_B200_H_ */
