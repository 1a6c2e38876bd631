// Flat forest layout for batched prediction on the device.
#pragma once
#include "device_common.cuh"

namespace lgbm_b200 {

// One internal node in 16 bytes: a tree walk step is one vector load.
// Categorical nodes keep the index of their category bitset (into cat_bnd)
// in the threshold's bits.
struct __align__(16) DNode {
  double threshold;
  int32_t feat_dt;  // real feature column (low 24 bits) | decision_type << 24
  int16_t left, right;  // child node, or ~leaf
};

// The same for trees with more than 32,768 leaves.
struct __align__(8) DNodeWide {
  double threshold;
  int32_t feat_dt;
  int32_t pad;
  int32_t left, right;
};

constexpr int32_t kNodeFeatureBits = 24;

struct DForest {
  int32_t num_trees, ntpi;
  bool wide;              // nodes are DNodeWide
  const int4* tree;       // [num_trees] (first node, first leaf value, num_leaves, 0)
  const void* nodes;      // DNode or DNodeWide, trees concatenated
  const int32_t* cat_bnd; // bitset word ranges
  const uint32_t* cat_words;  // category bitsets
  const double* leaf_value;
};

// Raw scores out[r * ntpi + k] of rows X[r * ncol ...] (device pointers).
// Allocates nothing.
cudaError_t launch_predict(const DForest& f, const float* X, int64_t nrow, int32_t ncol, double* out, cudaStream_t s);

// Device, stream, flat layout and trees per iteration of a forest made by
// lgbm_b200_forest_create.
void forest_parts(const LgbmB200Forest* F, int* device, cudaStream_t* stream, const DForest** f, int32_t* ntpi);

}  // namespace lgbm_b200
