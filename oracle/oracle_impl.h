// Internal declarations shared by the oracle's translation units.
// TEST INFRASTRUCTURE ONLY (see oracle.h).
#pragma once
#include "oracle.h"

#include <array>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>

namespace oracle {

// Error state of the C ABI: an entry point body runs inside ORACLE_TRY, which
// returns 0, or -1 with the exception's message kept for oracle_last_error().
void set_last_error(const std::string& msg);
#define ORACLE_TRY(...)                       \
  try {                                       \
    __VA_ARGS__;                              \
    return 0;                                 \
  } catch (const std::exception& e) {         \
    ::oracle::set_last_error(e.what());       \
    return -1;                                \
  }

// split.cpp
double threshold_l1(double s, double l1);
double leaf_output_t(double g, double h, const SplitParams& p, bool use_l1, bool use_max, bool use_smooth,
                     int32_t num_data, double parent_output);
double leaf_output(double g, double h, const SplitParams& p, int32_t num_data, double parent_output);
double refit_leaf_output(double g, double h, const SplitParams& p, bool smooth, int32_t n, double parent);
double root_output(double g, double h, const SplitParams& p, int32_t num_data);
bool find_best_threshold(const double* hist, const FeatureMeta& meta, const SplitParams& p, double sum_gradient,
                         double sum_hessian, int32_t num_data, double parent_output, const BasicConstraint* mc,
                         SplitInfo& out);
bool find_best_threshold_int(const int64_t* hist, const FeatureMeta& meta, const SplitParams& p, int64_t sum,
                             double grad_scale, double hess_scale, int32_t num_data, double parent_output,
                             const BasicConstraint* mc, SplitInfo& out);
void fix_hist(const FeatureMeta& m, double sum_g, double sum_h, double* hist);
void fix_hist_int(const FeatureMeta& m, int64_t int_sum, int64_t* hist);

// rng.cpp — random.rs (upstream LCG) and mt19937.rs (libstdc++ mt19937).
struct Random {
  uint32_t x;
  explicit Random(int32_t seed) : x((uint32_t)seed) {}
  int32_t rand_int16() { x = x * 214013u + 2531011u; return (int32_t)((x >> 16) & 0x7FFF); }
  int32_t rand_int32() { x = x * 214013u + 2531011u; return (int32_t)(x & 0x7FFFFFFF); }
  int32_t next_short(int32_t lo, int32_t hi) { return rand_int16() % (hi - lo) + lo; }
  int32_t next_int(int32_t lo, int32_t hi) { return rand_int32() % (hi - lo) + lo; }
  float next_float() { return (float)rand_int16() / 32768.0f; }
  std::vector<int32_t> sample(int32_t n, int32_t k);
};
struct Mt19937 {
  uint32_t state[624];
  int idx;
  explicit Mt19937(uint32_t seed);
  void twist();
  uint32_t next_u32();
  double canonical();
  double uniform01() { return canonical() * (1.0 - 0.0) + 0.0; }
  int32_t uniform_int(int32_t a, int32_t b);
};
// multi_val_bin.rs:337-345 Threading::BlockInfo
void block_info(size_t num_threads, size_t cnt, size_t min_cnt_per_block, size_t* nblock, size_t* block_size);

// quant.rs: GradientDiscretizer.
struct GradientDiscretizer {
  int32_t num_grad_quant_bins;
  bool is_constant_hessian, stochastic_rounding;
  std::vector<double> gradient_random_values, hessian_random_values;
  Mt19937 start_eng;
  int32_t start_max;
  std::vector<std::array<int8_t, 2>> raw;  // [hess, grad]
  std::vector<int64_t> packed;
  double grad_scale = 0, hess_scale = 0;
  GradientDiscretizer(int32_t bins, int32_t seed, bool const_hess, bool stochastic, size_t num_data, size_t num_threads);
  void discretize(const float* grad, const float* hess, size_t n_all, const uint32_t* rows, size_t n_rows);
  void root_sums(const uint32_t* rows, size_t n, double* sg, double* sh, int64_t* si) const;
};
int8_t to_i8(double x);

// tree.cpp — tree.rs Tree::split / split_categorical / shrink / add_bias.
struct SplitArgs {
  int32_t leaf, feature_inner, feature_real;
  uint32_t threshold_bin;
  double threshold, left_value, right_value;
  int32_t left_count, right_count;
  double left_weight, right_weight;
  float gain;
  int32_t missing_type;
  bool default_left;
};
int32_t tree_split(Tree& t, const SplitArgs& a);
int32_t tree_split_categorical(Tree& t, const SplitArgs& a, const std::vector<uint32_t>& bits_inner,
                               const std::vector<uint32_t>& bits);
void tree_set_leaf_output(Tree& t, int32_t leaf, double v);
void tree_shrink(Tree& t, double rate);
void tree_add_bias(Tree& t, double v);
void tree_as_constant(Tree& t, double v, int32_t count);
double maybe_round_to_zero(double v);
std::vector<uint32_t> construct_bitset(const std::vector<int32_t>& vals);
bool find_in_bitset(const uint32_t* bits, size_t n, int32_t pos);
int32_t tree_leaf_binned(const Tree& t, const BinnedData& d, int64_t row);

// learner.cpp — learner/mod.rs SerialTreeLearner.
struct LearnerConfig {
  SplitParams params;
  int32_t num_leaves, max_depth;
  double monotone_penalty;
  bool use_monotone;       // monotone_constraints non-empty, basic method
  bool quantized;
  int32_t num_grad_quant_bins;
  bool stochastic_rounding, quant_renew;
  int32_t seed;
  int32_t num_threads;     // only shapes the quantization random tables
  bool is_constant_hessian;
};

struct TreeTraceEntry {
  int32_t leaf, feature;
  uint32_t threshold;
  double gain;
};

class SerialTreeLearner {
 public:
  SerialTreeLearner(const BinnedData* data, const LearnerConfig& cfg);
  void set_bagging_data(const uint32_t* used, size_t n_used);
  void set_bytree_mask(const std::vector<bool>& used) { bytree_ = used; }
  Tree train(const float* grad, const float* hess);
  void add_leaf_outputs(const std::vector<double>& leaf_values, double* score) const;
  const std::vector<uint32_t>& indices() const { return indices_; }
  size_t leaf_begin(int l) const { return leaf_begin_[l]; }
  size_t leaf_count(int l) const { return leaf_count_[l]; }
  std::vector<TreeTraceEntry> trace;
  const GradientDiscretizer* quant() const { return quant_.get(); }

  // Histogram layout: feature f's view starts at view_start_[f] stored bins.
  std::vector<size_t> view_start_;
  size_t total_bins_ = 0;
  void build_hist(const uint32_t* rows, size_t n, const float* grad, const float* hess, double* out) const;
  void build_hist_block(const uint32_t* rows, size_t k0, size_t k1, const float* grad, const float* hess,
                        double* out) const;
  void build_hist_int(const uint32_t* rows, size_t n, const int64_t* packed, int64_t* out) const;
  size_t partition_split(int32_t leaf, int32_t inner, const std::vector<bool>& lut, int32_t right_leaf);

 private:
  struct LeafSplits {
    int32_t leaf = -1, num_data = 0;
    double sum_gradients = 0, sum_hessians = 0;
    int64_t int_sum = 0;
    double weight = 0;
  };
  const BinnedData* d_;
  LearnerConfig cfg_;
  std::vector<bool> bytree_;
  std::vector<uint32_t> indices_;
  std::vector<size_t> leaf_begin_, leaf_count_;
  int32_t part_num_leaves_ = 1;
  bool bagging_ = false;
  std::vector<uint32_t> used_;
  std::vector<std::vector<double>> hist_;
  std::vector<std::vector<int64_t>> ihist_;
  std::vector<std::vector<bool>> splittable_;
  std::vector<SplitInfo> best_split_per_leaf_;
  std::vector<BasicConstraint> constraints_;
  LeafSplits smaller_, larger_;
  std::unique_ptr<GradientDiscretizer> quant_;

  bool before_find_best_split(const Tree& tree, int32_t left, int32_t right);
  void find_best_splits(const Tree& tree, const float* grad, const float* hess, int32_t left, int32_t right);
  std::pair<int32_t, int32_t> split(Tree& tree, int32_t best_leaf);
  int32_t best_leaf() const;
};

}  // namespace oracle
