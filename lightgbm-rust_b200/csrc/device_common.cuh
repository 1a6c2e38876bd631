// Device-side structures and the split arithmetic shared by the learner's
// kernels. All FP64 expressions keep the reference's operation order and
// the library is compiled with --fmad=false, so a gain computed here from a
// histogram equals the CPU reference's gain for the same histogram bit for
// bit (crates/lgbm-core/src/learner/split.rs:124-231).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/lgbm_b200.h"

namespace lgbm_b200 {

constexpr double kEpsilon = (double)1e-15f;        // consts.rs:8
constexpr double kZeroThreshold = (double)1e-35f;  // consts.rs:15
constexpr int kMaxBins = 256;                      // stored values per single-feature group (u8)
constexpr int kCatWords = kMaxBins / 32;           // bitset words over bins
constexpr int kSpinLimit = 1 << 24;                // bound of every device-side wait

enum : int32_t { kStatusOk = 0, kStatusTimeout = 1, kStatusEmptyChild = 2, kStatusOverflow = 3 };

struct DFeature {
  int32_t num_bin, offset, default_bin, most_freq_bin, missing_type, bin_type, monotone_type, real_index;
  double penalty;
  int32_t view_start;  // first stored bin of this feature in a leaf histogram
  int32_t view_len;    // num_bin - offset
};

// learner/split.rs:33-46 plus the tree-level knobs the kernels read.
struct DParams {
  double lambda_l1, lambda_l2, max_delta_step, path_smooth;
  int32_t min_data_in_leaf;
  double min_sum_hessian_in_leaf, min_gain_to_split;
  int32_t max_cat_to_onehot, max_cat_threshold;
  double cat_l2, cat_smooth;
  int32_t min_data_per_group;
  int32_t num_leaves, max_depth;
  double monotone_penalty;
  int32_t use_monotone;
};

// learner/split.rs:61-81 SplitInfo; categorical bins sent left as a bitset.
struct DSplit {
  int32_t feature;  // real index, -1 none
  int32_t inner;
  uint32_t threshold;
  int32_t left_count, right_count;
  int32_t default_left;
  int32_t monotone_type;
  int32_t num_cat;  // categorical split: number of bins sent left (0: numerical)
  double left_output, right_output, gain;
  double left_sum_gradient, left_sum_hessian, right_sum_gradient, right_sum_hessian;
  int64_t left_sum_gh, right_sum_gh;
  uint32_t cat_bits[kCatWords];
};

struct DLeafSplits {  // learner/mod.rs:63-71
  int32_t leaf, num_data;
  double sum_gradients, sum_hessians;
  int64_t int_sum;
  double weight;
};

// Control block of one tree being grown (one per tree slot).
struct DSlotState {
  int32_t num_leaves_cur;  // tree.num_leaves
  int32_t done;
  int32_t status;
  int32_t need_find;       // before_find_best_split of (left_leaf, right_leaf)
  int32_t left_leaf, right_leaf;
  int32_t scan_done;       // CTAs of a scan + partition launch whose scans are stored
  int32_t part_ticket;     // next row tile of the running partition
  int32_t part_done;       // partition CTAs finished
  int32_t part_left;       // rows sent left (posted by the last tile)
  uint32_t part_epoch;
  int32_t num_used;        // in-bag rows
  int32_t num_cat;         // categorical splits so far
  int32_t use_indices_root;
  double grad_scale, hess_scale;  // quantized gradients
  DLeafSplits smaller, larger;
  int32_t s_begin, s_side, s_buf;  // the smaller leaf's range start, index buffer and histogram buffer
  int32_t s_count;                 // the smaller leaf's rows in this learner's range (data-parallel: this
                                   // rank's; smaller.num_data counts every rank's)
  int32_t l_buf;                   // the larger leaf's histogram buffer
  // A split step whose end (finish_step) runs beside the next histogram
  // launch's row CTAs: the partition posts the split leaf's rows and the
  // decision here. The histogram's row CTAs derive the smaller child's range
  // from them and the left count, and read nothing the step's end writes.
  int32_t pending;                 // 1: the posted step has not been finished
  int32_t pd_bl, pd_begin, pd_cnt, pd_side, pd_depth;  // the split leaf, its rows, its children's depth
  int32_t pd_need, pd_S, pd_G, pd_Lft, pd_R;            // the step's head
  int32_t pd_bf[2];                // the new leaves' best candidates (inner feature, -1 none)
  double pd_bg[2];                 // and their penalized gains
  int64_t hist_rows;       // rows histogrammed in this tree (statistics)
  int64_t part_rows;       // rows partitioned in this tree (statistics)
};

// One node / leaf record of the tree grown on the device (tree.rs:120-160).
struct DTree {
  int32_t* split_feature_inner;
  int32_t* split_feature;
  float* split_gain;
  uint32_t* threshold_in_bin;
  int8_t* decision_type;
  int32_t* left_child;
  int32_t* right_child;
  int32_t* leaf_parent;
  double* leaf_value;
  double* leaf_weight;
  int32_t* leaf_count;
  int32_t* leaf_depth;
  double* internal_value;
  double* internal_weight;
  int32_t* internal_count;
  uint32_t* cat_bits;  // [node][kCatWords] bins sent left by categorical nodes
  double* node_gain;   // unrounded gain of each split (diagnostics)
};

// Device pointers of one tree slot.
struct DSlot {
  DSlotState* st;
  uint32_t* idx[2];        // ping-pong row index buffers [num_data]
  int32_t* leaf_begin;
  int32_t* leaf_count;     // this rank's rows of each leaf (the row ranges)
  int32_t* leaf_gcount;    // every rank's rows of each leaf: the counts (leaf_count itself unless data-parallel)
  int32_t* leaf_side;      // which idx buffer holds the leaf's rows
  int32_t* buf_of;         // histogram buffer of each leaf
  DSplit* best;            // best_split_per_leaf [num_leaves]
  double* bgain;           // best[l].gain and best[l].feature, compact for the best-leaf argmax
  int32_t* bfeat;
  uint8_t* splittable;     // [num_leaves][num_features]
  double* cmin;            // basic monotone constraint per leaf
  double* cmax;
  void* hist;              // [num_leaves][total_bins] cells
  DSplit* feat_res;        // scan results [2][num_features]
  uint8_t* lut_cand;       // goes-left flag per stored value of each scan result [2][num_features][kMaxBins]
  uint8_t* leaf_lut;       // the same for each leaf's best split [num_leaves][kMaxBins]
  uint8_t* feat_ok;        // [2][num_features]
  unsigned long long* tile_status;  // partition look-back [max_tiles]
  const float2* gh;        // this slot's interleaved (gradient, hessian) [num_data]
  int32_t* packed;         // quantized gradients per row: (g << 16) + h
  uint8_t* bytree;         // by-tree feature mask [num_features]
  double* root_partials;   // [2 x kRootBlocks] (g, h) partial sums
  long long* root_ipartials;
  int32_t* root_counter;
  DTree tree;
  // data-parallel growth: the split decision the partition leaves for the
  // finishing launch, and this rank's rows sent left
  unsigned char* dp_dec;
  int32_t* dp_left;
};

constexpr int kRootBlocks = 296;
constexpr int kDpDecBytes = 2048;  // a split decision kept between a data-parallel partition and its finish
constexpr int kMaxSlots = 16;  // tree slots grown together (slot structs travel as kernel parameters)

struct DCtx {
  const uint8_t* bins;  // row-major, row stride `stride` bytes
  const uint8_t* colbins;  // column-major copy [num_features x num_data]
  int64_t num_data;
  int32_t stride;
  int32_t num_features;
  int32_t total_bins;
  int32_t hist_mode;   // LGBM_B200_HIST_*
  int32_t bagging;     // 1 when the in-bag rows are a strict subset
  const DFeature* feats;
  DParams p;
  DSlot slots[kMaxSlots];  // by value: read from the constant bank
  int32_t num_slots;
  int32_t rows_per_block;  // histogram rows per CTA (minimum)
  int32_t dp;              // 1: rows sharded over ranks; the step's end waits for the global left count
  int32_t defer;           // 1: a partition posts its step's end for the next histogram launch to run
  int32_t hist_direct;     // 1: the quantized one-group histogram runs the direct loop (asynchronous
                           // copies per warp, no tile barriers)
  int32_t q_in_row;        // 1: each row's packed gradient also fills its bin row's padding bytes 28..31
                           // (one tree slot, one feature tile of at most 28 features)
};

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while its predecessor in the stream still runs.
// pdl_wait blocks until the predecessor has finished and its writes are
// visible (a no-op for an ordinary launch); pdl_trigger lets the next kernel
// of the stream start launching.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---- split arithmetic (learner/split.rs:124-231) -------------------------------------
__device__ __forceinline__ double dsign(double x) { return (double)((x > 0.0) - (x < 0.0)); }
__device__ __forceinline__ double threshold_l1(double s, double l1) {
  double reg = fmax(fabs(s) - l1, 0.0);
  return dsign(s) * reg;
}
__device__ __forceinline__ bool use_l1(const DParams& p) { return p.lambda_l1 > 0.0; }
__device__ __forceinline__ bool use_max_output(const DParams& p) { return p.max_delta_step > 0.0; }
__device__ __forceinline__ bool use_smoothing(const DParams& p) { return p.path_smooth > kEpsilon; }

__device__ __forceinline__ double leaf_output_t(double g, double h, const DParams& p, bool l1, bool mx, bool sm,
                                                int32_t num_data, double parent_output) {
  double ret = l1 ? -threshold_l1(g, p.lambda_l1) / (h + p.lambda_l2) : -g / (h + p.lambda_l2);
  if (mx && p.max_delta_step > 0.0 && fabs(ret) > p.max_delta_step) ret = dsign(ret) * p.max_delta_step;
  if (sm) {
    double n = (double)num_data;
    ret = ret * (n / p.path_smooth) / (n / p.path_smooth + 1.0) + parent_output / (n / p.path_smooth + 1.0);
  }
  return ret;
}
__device__ __forceinline__ double leaf_output(double g, double h, const DParams& p, int32_t n, double po) {
  return leaf_output_t(g, h, p, use_l1(p), use_max_output(p), use_smoothing(p), n, po);
}
__device__ __forceinline__ double root_output(double g, double h, const DParams& p, int32_t n) {
  return leaf_output_t(g, h, p, true, true, false, n, 0.0);
}
__device__ __forceinline__ double refit_leaf_output(double g, double h, const DParams& p, int32_t n) {
  return leaf_output_t(g, h, p, true, true, false, n, 0.0);
}
__device__ __forceinline__ double leaf_gain_given_output(double g, double h, const DParams& p, double out) {
  double sg = use_l1(p) ? threshold_l1(g, p.lambda_l1) : g;
  return -(2.0 * sg * out + (h + p.lambda_l2) * out * out);
}
__device__ __forceinline__ double leaf_gain(double g, double h, const DParams& p, int32_t n, double po) {
  if (!use_max_output(p) && !use_smoothing(p)) {
    if (use_l1(p)) {
      double sg = threshold_l1(g, p.lambda_l1);
      return (sg * sg) / (h + p.lambda_l2);
    }
    return (g * g) / (h + p.lambda_l2);
  }
  double out = leaf_output(g, h, p, n, po);
  return leaf_gain_given_output(g, h, p, out);
}
__device__ __forceinline__ double clampc(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }
// split.rs:205-226; `mc` enables the basic monotone constraint [cmin, cmax].
__device__ __forceinline__ double split_gain(double lg, double lh, double rg, double rh, const DParams& p, int32_t lc,
                                             int32_t rc, double po, bool mc, double cmin, double cmax, int32_t mono) {
  if (!mc) return leaf_gain(lg, lh, p, lc, po) + leaf_gain(rg, rh, p, rc, po);
  double left = clampc(leaf_output(lg, lh, p, lc, po), cmin, cmax);
  double right = clampc(leaf_output(rg, rh, p, rc, po), cmin, cmax);
  if ((mono > 0 && left > right) || (mono < 0 && left < right)) return 0.0;
  return leaf_gain_given_output(lg, lh, p, left) + leaf_gain_given_output(rg, rh, p, right);
}

// The scan's hot code: with no L1, max_delta_step, path smoothing or
// monotone bounds every formula above reduces to its plain form, evaluated
// inline with the same operations; otherwise the full formula is called out
// of line, which keeps the threshold scan's instruction footprint small.
__device__ __forceinline__ bool plain_split(const DParams& p, bool mc) {
  return !mc && !use_l1(p) && !use_max_output(p) && !use_smoothing(p);
}
static __device__ __noinline__ double split_gain_full(double lg, double lh, double rg, double rh, const DParams& p,
                                                      int32_t lc, int32_t rc, double po, bool mc, double cmin,
                                                      double cmax, int32_t mono) {
  return split_gain(lg, lh, rg, rh, p, lc, rc, po, mc, cmin, cmax, mono);
}
static __device__ __noinline__ double leaf_output_full(double g, double h, const DParams& p, int32_t n, double po) {
  return leaf_output(g, h, p, n, po);
}
static __device__ __noinline__ double leaf_gain_full(double g, double h, const DParams& p, int32_t n, double po) {
  return leaf_gain(g, h, p, n, po);
}
__device__ __forceinline__ double split_gain_hot(bool plain, double lg, double lh, double rg, double rh,
                                                 const DParams& p, int32_t lc, int32_t rc, double po, bool mc,
                                                 double cmin, double cmax, int32_t mono) {
  if (plain) return (lg * lg) / (lh + p.lambda_l2) + (rg * rg) / (rh + p.lambda_l2);
  return split_gain_full(lg, lh, rg, rh, p, lc, rc, po, mc, cmin, cmax, mono);
}
__device__ __forceinline__ double leaf_output_hot(bool plain, double g, double h, const DParams& p, int32_t n,
                                                  double po) {
  if (plain) return -g / (h + p.lambda_l2);
  return leaf_output_full(g, h, p, n, po);
}
__device__ __forceinline__ double leaf_gain_hot(bool plain, double g, double h, const DParams& p, int32_t n,
                                                double po) {
  if (plain) return (g * g) / (h + p.lambda_l2);
  return leaf_gain_full(g, h, p, n, po);
}

__device__ __forceinline__ int32_t round_int(double x) { return (int32_t)(x + (double)0.5f); }

// split.rs:114-121 SplitInfo::better_than
__device__ __forceinline__ bool better_than(double ga, int32_t fa, double gb, int32_t fb) {
  if (ga != gb) return ga > gb;
  int32_t a = fa == -1 ? INT32_MAX : fa;
  int32_t b = fb == -1 ? INT32_MAX : fb;
  return a < b;
}

__device__ __forceinline__ double maybe_round_to_zero(double v) {  // tree.rs:27-29
  return (v >= -kZeroThreshold && v <= kZeroThreshold) ? 0.0 : v;
}

// FeatureBins::decode (feature_group.rs:206-208) for a single-feature group.
__device__ __forceinline__ uint32_t decode_bin(uint32_t raw, const DFeature& f) {
  return raw == 0 ? (uint32_t)f.most_freq_bin : raw - 1u + (uint32_t)(f.most_freq_bin == 0);
}

// Quantized packed sums: gradient in the high 32 bits, hessian in the low 32.
__device__ __forceinline__ int32_t int_grad(int64_t x) { return (int32_t)(x >> 32); }
__device__ __forceinline__ uint32_t int_hess(int64_t x) { return (uint32_t)x; }

}  // namespace lgbm_b200
