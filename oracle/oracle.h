// CPU oracle: a single-threaded C++ restatement of lightgbm-rust's serial
// tree learner and the boosting loop around it. TEST INFRASTRUCTURE ONLY —
// it is the checker for the CUDA path, never part of the product.
//
// Every function cites the reference file:line it restates (paths are
// relative to the lightgbm-rust project root, crates/lgbm-core/src/...).
// Summation order equals the reference at num_threads=1, force_row_wise:
// rows in ascending partition order, per-bin sequential FP64 sums.
//
// Parity pins: the reference's own in-source known-answer tests (histogram
// fix, split KATs, quantization packing, block_info, MT19937 sequence, LCG,
// learner step tests), ported in tests/test_oracle_kat.py.
#pragma once
#include <cstdint>
#include <cmath>
#include <vector>
#include <limits>

namespace oracle {

// consts.rs:8-20 — upstream declares these as float literals.
constexpr double kEpsilon = (double)1e-15f;
constexpr double kZeroThreshold = (double)1e-35f;
constexpr double kMinScore = -std::numeric_limits<double>::infinity();

enum MissingType { kMissingNone = 0, kMissingZero = 1, kMissingNaN = 2 };
enum BinType { kNumerical = 0, kCategorical = 1 };

// learner/split.rs:17-29 (FeatureMeta) plus the real column index.
struct FeatureMeta {
  int32_t num_bin;
  int32_t missing_type;
  int32_t offset;          // 1 when most_freq_bin == 0 (bin 0 not stored)
  uint32_t default_bin;
  uint32_t most_freq_bin;
  int32_t bin_type;
  int32_t monotone_type;
  double penalty;          // feature_contri
  int32_t real_index;
};

// learner/split.rs:33-46
struct SplitParams {
  double lambda_l1, lambda_l2, max_delta_step, path_smooth;
  int32_t min_data_in_leaf;
  double min_sum_hessian_in_leaf, min_gain_to_split;
  int32_t max_cat_to_onehot, max_cat_threshold;
  double cat_l2, cat_smooth;
  int32_t min_data_per_group;
};

// learner/constraints.rs BasicConstraint (min, max) with C++ clamp semantics.
struct BasicConstraint {
  double min = -std::numeric_limits<double>::max();
  double max = std::numeric_limits<double>::max();
  double clamp(double v) const { return v < min ? min : (v > max ? max : v); }
};

// learner/split.rs:61-104
struct SplitInfo {
  int32_t feature = -1;       // real index
  int32_t feature_inner = -1;
  uint32_t threshold = 0;
  std::vector<uint32_t> cat_threshold;
  double left_output = 0, right_output = 0;
  double gain = kMinScore;
  int32_t left_count = 0, right_count = 0;
  double left_sum_gradient = 0, left_sum_hessian = 0;
  double right_sum_gradient = 0, right_sum_hessian = 0;
  bool default_left = true;
  int32_t monotone_type = 0;
  int64_t left_sum_gh = 0, right_sum_gh = 0;
  void reset() { feature = -1; gain = kMinScore; }
  // split.rs:114-121
  bool better_than(const SplitInfo& o) const {
    if (gain != o.gain) return gain > o.gain;
    int32_t a = feature == -1 ? INT32_MAX : feature;
    int32_t b = o.feature == -1 ? INT32_MAX : o.feature;
    return a < b;
  }
};

// tree.rs:120-160 (fields used by the learner, predict and model text).
struct Tree {
  int32_t num_leaves = 1;
  std::vector<int32_t> split_feature_inner, split_feature;
  std::vector<float> split_gain;
  std::vector<uint32_t> threshold_in_bin;
  std::vector<double> threshold;
  std::vector<int8_t> decision_type;
  std::vector<int32_t> left_child, right_child;
  std::vector<int32_t> leaf_parent{-1};
  std::vector<double> leaf_value{0.0}, leaf_weight{0.0};
  std::vector<int32_t> leaf_count{0}, leaf_depth{0};
  std::vector<double> internal_value, internal_weight;
  std::vector<int32_t> internal_count;
  double shrinkage = 1.0;
  int32_t num_cat = 0;
  std::vector<int32_t> cat_boundaries{0}, cat_boundaries_inner{0};
  std::vector<uint32_t> cat_threshold, cat_threshold_inner;
};

// Binned feature data as the learner sees it: row-major u8 values of the
// single-feature groups (0 = most frequent bin, else bin - (mfb==0) + 1,
// feature_group.rs:144-154), plus per-feature metadata and, for raw-value
// thresholds, each feature's bin upper bounds / bin categories.
struct BinnedData {
  int64_t num_data = 0;
  int32_t num_features = 0;
  const uint8_t* bins = nullptr;           // [num_data * num_features]
  std::vector<FeatureMeta> metas;
  std::vector<std::vector<double>> upper_bounds;  // numerical: bin_upper_bound
  std::vector<std::vector<int32_t>> bin_to_cat;   // categorical: bin_2_categorical
};

}  // namespace oracle
