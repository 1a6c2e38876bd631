// Host-side internals of liblgbm_b200 (no CUDA types).
#pragma once
#include <cmath>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/lgbm_b200.h"

namespace lgbm_b200 {

struct Status {
  int code = LGBM_B200_OK;
  std::string msg;
  Status() = default;
  Status(int c, std::string m) : code(c), msg(std::move(m)) {}
  bool ok() const { return code == LGBM_B200_OK; }
};

void set_last_error(const std::string& msg);

// crates/lgbm-core/src/binning.rs:49-66 BinMapper (fields the learner reads).
struct BinMapper {
  int32_t num_bin = 1;
  int32_t missing_type = 0;
  std::vector<double> bin_upper_bound{INFINITY};
  bool is_trivial = true;
  double sparse_rate = 1.0;
  int32_t bin_type = 0;
  double min_val = 0, max_val = 0;
  uint32_t default_bin = 0, most_freq_bin = 0;
  std::vector<int32_t> bin_2_categorical;
  std::map<int32_t, uint32_t> categorical_2_bin;
};

uint32_t value_to_bin(const BinMapper& m, double value);

struct Dataset {
  int64_t num_data = 0;
  int32_t num_total_features = 0;
  std::vector<int32_t> used;  // real column of each inner feature
  std::vector<BinMapper> mappers;
  std::vector<uint8_t> bins;  // row-major [num_data x used.size()]
  // flattened view storage
  std::vector<int32_t> num_bin, missing_type, default_bin, most_freq_bin, bin_type, real_index, bin_to_cat;
  std::vector<double> upper_bounds;
  std::vector<int64_t> ub_offsets, cat_offsets;
  std::string feature_infos;  // built on request
  void fill_view(LgbmB200DatasetView* v);
  // Dataset::feature_infos (dataset.rs:770-776), space-separated
  const std::string& infos();
};

// device < 0: the rows are binned on the host; else on that CUDA device
// (the bin mappers come from the host's row sample either way)
Status build_dataset(const float* X, int64_t n, int32_t ncol, const LgbmB200BinParams& p, Dataset& d,
                     int device = -1);
Status build_valid_dataset(const float* X, int64_t n, int32_t ncol, const Dataset& ref, Dataset& d,
                           int device = -1);
// The rows of X binned with d's mappers on `device` into d.bins (binning_kernels.cu).
Status push_bins_device(Dataset& d, const float* X, int64_t n, int32_t ncol, int device);

}  // namespace lgbm_b200
