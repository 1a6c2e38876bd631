// C ABI of the CPU oracle, loaded by the tests with ctypes.
// TEST INFRASTRUCTURE ONLY: nothing in the product links or loads this.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleBooster OracleBooster;

// Training parameters (names follow lightgbm-rust's config.rs).
typedef struct {
  int32_t objective;  // 0 binary, 1 regression (L2), 2 multiclass (softmax), 3 lambdarank
  int32_t num_class;
  double sigmoid;
  int32_t num_iterations;
  double learning_rate;
  int32_t boost_from_average;
  int32_t num_leaves, max_depth, min_data_in_leaf;
  double min_sum_hessian_in_leaf, lambda_l1, lambda_l2, max_delta_step, path_smooth, min_gain_to_split;
  int32_t max_cat_to_onehot, max_cat_threshold;
  double cat_l2, cat_smooth;
  int32_t min_data_per_group;
  double bagging_fraction;
  int32_t bagging_freq, bagging_seed;
  double feature_fraction;
  int32_t feature_fraction_seed;
  int32_t use_quantized_grad, num_grad_quant_bins, stochastic_rounding, quant_train_renew_leaf, seed, num_threads;
  double monotone_penalty;
  int32_t lambdarank_truncation_level, lambdarank_norm;
} OracleParams;

// A binned dataset: row-major u8 group values plus per-inner-feature metadata.
typedef struct {
  int64_t num_data;
  int32_t num_features;
  const uint8_t* bins;
  const int32_t* num_bin;
  const int32_t* missing_type;
  const int32_t* default_bin;
  const int32_t* most_freq_bin;
  const int32_t* bin_type;
  const int32_t* real_index;
  const int8_t* monotone;        // per inner feature, NULL: no monotone constraints
  const double* upper_bounds;    // numerical thresholds, by ub_offsets
  const int64_t* ub_offsets;
  const int32_t* bin_to_cat;     // categorical bin -> category, by cat_offsets
  const int64_t* cat_offsets;
} OracleData;

typedef struct {
  int32_t num_leaves;
  const int32_t* split_feature;
  const int32_t* split_feature_inner;
  const float* split_gain;
  const uint32_t* threshold_in_bin;
  const double* threshold;
  const int8_t* decision_type;
  const int32_t* left_child;
  const int32_t* right_child;
  const double* leaf_value;
  const double* leaf_weight;
  const int32_t* leaf_count;
  const double* internal_value;
  const double* internal_weight;
  const int32_t* internal_count;
  const int32_t* leaf_depth;
  int32_t num_cat;
  const int32_t* cat_boundaries;
  const uint32_t* cat_threshold;
  int32_t num_cat_threshold;
  double shrinkage;
} OracleTreeView;

typedef struct {
  int32_t num_bin, missing_type, default_bin, most_freq_bin, bin_type, monotone_type;
  int32_t offset;  /* stored-bin offset of the view (1 when bin 0 is not stored) */
  double penalty;
  int32_t use_constraint;
  double constraint_min, constraint_max;
} OracleFeature;

typedef struct {
  int32_t splittable;
  uint32_t threshold;
  double gain, left_output, right_output;
  int32_t left_count, right_count;
  double left_sum_gradient, left_sum_hessian, right_sum_gradient, right_sum_hessian;
  int32_t default_left;
  int32_t num_cat;
  uint32_t cat_threshold[256];
  int64_t left_sum_gh, right_sum_gh;
} OracleSplit;

// Bin parameters of a dataset build (config.rs names).
typedef struct {
  int32_t max_bin, min_data_in_bin, min_data_in_leaf, bin_construct_sample_cnt, data_random_seed;
  int32_t use_missing, zero_as_missing, feature_pre_filter;
  const int32_t* categorical;  // column indices of categorical features
  int32_t num_categorical;
} OracleBinParams;

typedef struct OracleDataset OracleDataset;

const char* oracle_last_error(void);
// Dataset::from_dense (dataset.rs:355) and from_dense_with_reference (:446):
// the oracle's own bin finding and stored group values (binning.cpp).
int oracle_dataset_create(const float* X, int64_t n, int32_t ncol, const OracleBinParams* p, OracleDataset** out);
int oracle_dataset_create_valid(const float* X, int64_t n, int32_t ncol, const OracleDataset* ref,
                                OracleDataset** out);
// The binned matrix and per-feature metadata (valid until the dataset is freed).
int oracle_dataset_view(OracleDataset* d, OracleData* out, int32_t* num_total_features);
// Dataset::feature_infos (dataset.rs:770), space-separated.
const char* oracle_dataset_feature_infos(OracleDataset* d);
void oracle_dataset_free(OracleDataset* d);
int oracle_train(const OracleParams* p, const OracleData* train, const float* label, const int32_t* query_boundaries,
                 int32_t num_queries, const OracleData* valid, OracleBooster** out);
int oracle_train_tree(const OracleParams* p, const OracleData* train, const float* grad, const float* hess,
                      const uint32_t* bag, int64_t n_bag, int32_t num_trees, const uint8_t* bytree,
                      OracleBooster** out);
int oracle_booster_update(OracleBooster* h, int32_t* stop);
int oracle_booster_partition(OracleBooster* h, int32_t* leaf_begin, int32_t* leaf_count, uint32_t* indices);
void oracle_booster_free(OracleBooster* h);
int32_t oracle_booster_num_trees(OracleBooster* h);
int oracle_booster_tree(OracleBooster* h, int32_t i, OracleTreeView* out);
int oracle_booster_trace(OracleBooster* h, int32_t i, int32_t* n, int32_t* leaf, int32_t* feature,
                         uint32_t* threshold, double* gain);
int oracle_booster_scores(OracleBooster* h, int valid, double* out);
// Gbdt::save_model_to_string (io.rs:13-85) up to the feature importances:
// the header, every tree (tree.rs:718-773) and the split counts. The text
// stays valid until the booster is freed or the next call.
int oracle_model_to_string(OracleBooster* h, int32_t num_total_features, const char* feature_infos,
                           const int8_t* monotone, int32_t num_monotone, const char** out);
int oracle_predict_raw(OracleBooster* h, const float* X, int64_t nrow, int32_t ncol, double* out);
double oracle_auc(const float* label, const double* score, int64_t n);
int oracle_ndcg(const float* label, const double* score, const int32_t* bnd, int32_t nq, const int32_t* ks,
                int32_t nk, double* out);
int oracle_gradients(int32_t objective, int32_t num_class, double sigmoid, const float* label, const double* scores,
                     int64_t n, const int32_t* bnd, int32_t nq, int32_t truncation, int32_t norm, float* g, float* h);
int oracle_hist(const OracleData* d, const uint32_t* rows, int64_t nrows, const float* g, const float* h,
                const int64_t* packed, double* out_f64, int64_t* out_int);
int oracle_fix_hist(int32_t num_bin, int32_t offset, int32_t most_freq_bin, double sum_g, double sum_h,
                    double* hist);
int32_t oracle_better_than(double gain_a, int32_t feature_a, double gain_b, int32_t feature_b);
int oracle_find_best_threshold(const OracleFeature* f, const OracleParams* p, const double* hist,
                               const int64_t* ihist, double sum_g, double sum_h, int64_t int_sum, double gscale,
                               double hscale, int32_t num_data, double parent_output, OracleSplit* out);
int oracle_discretize(int32_t bins, int32_t seed, int32_t const_hess, int32_t stochastic, int64_t n,
                      int32_t num_threads, int32_t num_calls, const float* g, const float* h, int64_t* packed,
                      double* scales);
int oracle_mt19937(uint32_t seed, int32_t n, uint32_t* out);
int oracle_lcg_sample(int32_t seed, int32_t n, int32_t k, int32_t* out, int32_t* out_len);
int oracle_block_info(int64_t threads, int64_t cnt, int64_t min_cnt, int64_t* out);
int8_t oracle_to_i8(double x);

#ifdef __cplusplus
}
#endif
