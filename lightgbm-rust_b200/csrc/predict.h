// Flat forest layout for batched prediction on the device.
#pragma once
#include "device_common.cuh"

namespace lgbm_b200 {

struct DForest {
  int32_t num_trees, ntpi;
  const int32_t* node_off;    // [num_trees] first node of each tree
  const int32_t* leaf_off;    // [num_trees] first leaf value of each tree
  const int32_t* num_leaves;  // [num_trees]
  const int32_t* feature;     // real column of each node
  const double* threshold;
  const int8_t* dtype;        // decision_type
  const int32_t* left;
  const int32_t* right;
  const int32_t* cat_idx;     // categorical nodes: index into cat_bnd
  const int32_t* cat_bnd;     // bitset word ranges
  const uint32_t* cat_words;  // category bitsets
  const double* leaf_value;
};

void launch_predict(const DForest& f, const float* X, int64_t nrow, int32_t ncol, double* out, cudaStream_t s);

// Device, stream, flat layout and trees per iteration of a forest made by
// lgbm_b200_forest_create.
void forest_parts(const LgbmB200Forest* F, int* device, cudaStream_t* stream, const DForest** f, int32_t* ntpi);

}  // namespace lgbm_b200
