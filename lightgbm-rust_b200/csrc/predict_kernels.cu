// Batched raw-score prediction: Gbdt::predict_matrix_early_stop with
// PredictKind::Raw (crates/lgbm-core/src/predict.rs:43-138, :231-339).
//
// A CTA of 128 threads takes 128 consecutive rows. When a row fits (up to
// kStageMaxCols features) the CTA first copies its rows, which are one
// contiguous block of X, into shared memory with coalesced (16-byte where
// aligned) loads, so a tree walk reads its row from shared memory instead of
// gathering 4 bytes from a 32-byte sector per node visit. The reference walks
// 16-row blocks level by level (predict.rs:43-138); here each thread walks
// its own row and a warp advances 32 rows together.
//
// Each thread sums, per class k, the leaf values of trees k, k + ntpi, ... in
// model order, which is the reference's summation order for that class
// (predict.rs:231-339), so the FP64 sums are the reference's. Any number of
// classes works: no per-class array is kept.
#include <mutex>

#include "predict.h"

namespace lgbm_b200 {

constexpr int kPredictThreads = 128;
constexpr int kStageMaxCols = 223;  // 128 rows x 224 floats = 112 KiB of shared memory
constexpr int kMaxPredictDevices = 64;

__device__ __forceinline__ bool find_in_bitset(const uint32_t* bits, int32_t n, int32_t pos) {  // tree.rs:46-52
  int32_t i1 = pos / 32;
  if (i1 >= n) return false;
  return ((bits[i1] >> (pos % 32)) & 1u) == 1u;
}

// The row is converted to f64 and |v| <= kZeroThreshold dropped
// (predict.rs:265-275).
__device__ __forceinline__ float drop_tiny(float x) {
  const double v = (double)x;
  return (!isnan(v) && fabs(v) <= kZeroThreshold) ? 0.0f : x;
}

__device__ __forceinline__ void load_node(const DNode* nodes, int32_t i, double& thr, int32_t& fd, int32_t& l,
                                          int32_t& r) {
  const DNode n = nodes[i];
  thr = n.threshold;
  fd = n.feat_dt;
  l = n.left;
  r = n.right;
}

__device__ __forceinline__ void load_node(const DNodeWide* nodes, int32_t i, double& thr, int32_t& fd, int32_t& l,
                                          int32_t& r) {
  const DNodeWide n = nodes[i];
  thr = n.threshold;
  fd = n.feat_dt;
  l = n.left;
  r = n.right;
}

// One decision: FlatTree::step (numerical, predict.rs:95-111) or step_any
// (categorical, :77-90). v is the row's value, already free of tiny values.
__device__ __forceinline__ bool goes_left(const DForest& f, double thr, int8_t dt, double v) {
  if (dt & 1) {
    const int32_t ci = (int32_t)__double_as_longlong(thr);
    const int32_t b0 = f.cat_bnd[ci], b1 = f.cat_bnd[ci + 1];
    return !isnan(v) && (int32_t)v >= 0 && find_in_bitset(f.cat_words + b0, b1 - b0, (int32_t)v);
  }
  const int mt = (dt >> 2) & 3;
  const bool nan = isnan(v);
  const bool nan_split = mt == 2;
  if (nan && !nan_split) v = 0.0;
  const bool zero = v >= -kZeroThreshold && v <= kZeroThreshold;
  const bool is_default = (mt == 1 && zero) || (nan_split && nan);
  return is_default ? (dt & 2) != 0 : v <= thr;
}

template <class Node, bool kStage>
__global__ void __launch_bounds__(kPredictThreads) k_predict(DForest f, const float* X, int64_t nrow, int32_t ncol,
                                                             int32_t ncolp, double* out) {
  extern __shared__ float srows[];
  const int64_t r0 = (int64_t)blockIdx.x * kPredictThreads;
  const int64_t r = r0 + threadIdx.x;
  const float* row;
  if constexpr (kStage) {
    const int nr = (int)(nrow - r0 < kPredictThreads ? nrow - r0 : (int64_t)kPredictThreads);
    const float* src = X + r0 * ncol;
    const int32_t total = nr * ncol;
    if ((ncol & 3) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
      const float4* s4 = reinterpret_cast<const float4*>(src);
      for (int32_t i = threadIdx.x; i < (total >> 2); i += kPredictThreads) {
        const float4 v = __ldg(s4 + i);
        const int32_t e = i << 2;
        const int32_t rr = e / ncol, cc = e - rr * ncol;  // the 4 values lie in one row
        float* d = srows + rr * ncolp + cc;
        d[0] = drop_tiny(v.x);
        d[1] = drop_tiny(v.y);
        d[2] = drop_tiny(v.z);
        d[3] = drop_tiny(v.w);
      }
    } else {
      for (int32_t i = threadIdx.x; i < total; i += kPredictThreads) {
        const int32_t rr = i / ncol, cc = i - rr * ncol;
        srows[rr * ncolp + cc] = drop_tiny(__ldg(src + i));
      }
    }
    __syncthreads();
    row = srows + threadIdx.x * ncolp;
  } else {
    row = X + r * ncol;
  }
  if (r >= nrow) return;
  const Node* nodes = static_cast<const Node*>(f.nodes);
  const int ntpi = f.ntpi;
  for (int k = 0; k < ntpi; ++k) {
    double acc = 0.0;
    for (int32_t t = k; t < f.num_trees; t += ntpi) {
      const int4 tt = f.tree[t];  // first node, first leaf, num_leaves
      int32_t node = 0;
      if (tt.z > 1) {
        while (node >= 0) {
          double thr;
          int32_t fd, l, rc;
          load_node(nodes, tt.x + node, thr, fd, l, rc);
          const int32_t feat = fd & ((1 << kNodeFeatureBits) - 1);
          // features past the row read 0.0
          double v = 0.0;
          if (feat < ncol) {
            if constexpr (kStage) {
              v = (double)row[feat];
            } else {
              v = (double)drop_tiny(row[feat]);
            }
          }
          node = goes_left(f, thr, (int8_t)(fd >> kNodeFeatureBits), v) ? l : rc;
        }
        node = ~node;
      }
      acc += f.leaf_value[tt.y + node];
    }
    out[r * ntpi + k] = acc;
  }
}

static std::once_flag g_predict_attr_once[kMaxPredictDevices];
static cudaError_t g_predict_attr_err[kMaxPredictDevices];

// Opt the staged kernels in to more than 48 KiB of dynamic shared memory,
// once per device (the setting belongs to the device's context).
static cudaError_t predict_attributes() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxPredictDevices) return cudaErrorInvalidDevice;
  std::call_once(g_predict_attr_once[dev], [dev] {
    const int bytes = kPredictThreads * (kStageMaxCols + 1) * (int)sizeof(float);
    cudaError_t x = cudaFuncSetAttribute(k_predict<DNode, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (x == cudaSuccess)
      x = cudaFuncSetAttribute(k_predict<DNodeWide, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    g_predict_attr_err[dev] = x;
  });
  return g_predict_attr_err[dev];
}

cudaError_t launch_predict(const DForest& f, const float* X, int64_t nrow, int32_t ncol, double* out, cudaStream_t s) {
  if (nrow <= 0) return cudaSuccess;
  const int64_t blocks = (nrow + kPredictThreads - 1) / kPredictThreads;
  if (blocks > 0x7fffffff) return cudaErrorInvalidValue;
  if (ncol <= kStageMaxCols) {
    cudaError_t e = predict_attributes();
    if (e != cudaSuccess) return e;
    const int32_t ncolp = ncol | 1;  // odd row stride in shared memory
    const size_t smem = sizeof(float) * (size_t)kPredictThreads * ncolp;
    if (f.wide)
      k_predict<DNodeWide, true><<<(unsigned)blocks, kPredictThreads, smem, s>>>(f, X, nrow, ncol, ncolp, out);
    else
      k_predict<DNode, true><<<(unsigned)blocks, kPredictThreads, smem, s>>>(f, X, nrow, ncol, ncolp, out);
  } else if (f.wide) {
    k_predict<DNodeWide, false><<<(unsigned)blocks, kPredictThreads, 0, s>>>(f, X, nrow, ncol, ncol, out);
  } else {
    k_predict<DNode, false><<<(unsigned)blocks, kPredictThreads, 0, s>>>(f, X, nrow, ncol, ncol, out);
  }
  return cudaGetLastError();
}

}  // namespace lgbm_b200
