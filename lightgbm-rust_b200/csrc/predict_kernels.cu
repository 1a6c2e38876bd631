// Batched raw-score prediction: Gbdt::predict_matrix_early_stop with
// PredictKind::Raw (crates/lgbm-core/src/predict.rs:43-138, :231-339).
// One thread per row walks every tree in model order with the decisions of
// FlatTree::step / step_any and sums per class in that order, so the FP64
// sums equal the reference's.
#include "predict.h"

namespace lgbm_b200 {

__device__ __forceinline__ bool find_in_bitset(const uint32_t* bits, int32_t n, int32_t pos) {  // tree.rs:46-52
  int32_t i1 = pos / 32;
  if (i1 >= n) return false;
  return ((bits[i1] >> (pos % 32)) & 1u) == 1u;
}

template <int kMaxClass>
__global__ void __launch_bounds__(128) k_predict(DForest f, const float* X, int64_t nrow, int32_t ncol, double* out) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrow) return;
  const float* row = X + r * ncol;
  double acc[kMaxClass];
#pragma unroll
  for (int k = 0; k < kMaxClass; ++k) acc[k] = 0.0;
  const int ntpi = f.ntpi;
  for (int32_t t = 0; t < f.num_trees; ++t) {
    const int32_t nb = f.node_off[t];
    const int32_t lb = f.leaf_off[t];
    int32_t node = 0;
    if (f.num_leaves[t] > 1) {
      while (node >= 0) {
        const int32_t nd = nb + node;
        const int32_t feat = f.feature[nd];
        // the row is converted to f64 and |v| <= kZeroThreshold dropped (predict.rs:265-275);
        // features past the row read 0.0
        double v = feat < ncol ? (double)row[feat] : 0.0;
        if (!isnan(v) && fabs(v) <= kZeroThreshold) v = 0.0;
        const int8_t dt = f.dtype[nd];
        bool left;
        if (dt & 1) {  // FlatTree::step_any (predict.rs:77-90)
          const int32_t ci = f.cat_idx[nd];
          const int32_t b0 = f.cat_bnd[ci], b1 = f.cat_bnd[ci + 1];
          left = !isnan(v) && (int32_t)v >= 0 && find_in_bitset(f.cat_words + b0, b1 - b0, (int32_t)v);
        } else {  // FlatTree::step (predict.rs:95-111)
          const int mt = (dt >> 2) & 3;
          const bool nan = isnan(v);
          const bool nan_split = mt == 2;
          if (nan && !nan_split) v = 0.0;
          const bool zero = v >= -kZeroThreshold && v <= kZeroThreshold;
          const bool is_default = (mt == 1 && zero) || (nan_split && nan);
          left = is_default ? (dt & 2) != 0 : v <= f.threshold[nd];
        }
        node = left ? f.left[nd] : f.right[nd];
      }
      node = ~node;
    }
    const int k = t % ntpi;
#pragma unroll
    for (int c = 0; c < kMaxClass; ++c)
      if (c == k) acc[c] += f.leaf_value[lb + node];
  }
  for (int k = 0; k < ntpi; ++k) out[r * ntpi + k] = acc[k];
}

void launch_predict(const DForest& f, const float* X, int64_t nrow, int32_t ncol, double* out, cudaStream_t s) {
  int64_t blocks = (nrow + 127) / 128;
  if (f.ntpi <= 1) k_predict<1><<<(unsigned)blocks, 128, 0, s>>>(f, X, nrow, ncol, out);
  else if (f.ntpi <= 4) k_predict<4><<<(unsigned)blocks, 128, 0, s>>>(f, X, nrow, ncol, out);
  else if (f.ntpi <= 16) k_predict<16><<<(unsigned)blocks, 128, 0, s>>>(f, X, nrow, ncol, out);
  else k_predict<64><<<(unsigned)blocks, 128, 0, s>>>(f, X, nrow, ncol, out);
}

}  // namespace lgbm_b200
