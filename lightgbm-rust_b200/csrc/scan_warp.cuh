// Building blocks of the parallel numerical threshold scan (split.rs:676-891
// and :995-1190) that reproduces the reference's sequential loop exactly.
//
// The FP64 cumulative sums must be formed in the reference's order (one add
// per visited bin, in scan order), so they are computed as a carry chain:
// each lane of a warp owns 8 consecutive stored bins, and the lane holding
// the first bins in scan order adds its bins to the carry and passes it on
// with a shuffle. Every other quantity (count estimates, break / skip rules,
// gains, the argmax) is evaluated in parallel. Packed integer sums are exact
// in any order, so the quantized form uses a plain warp prefix scan.
#pragma once
#include "device_common.cuh"

namespace lgbm_b200 {

constexpr int kPer = kMaxBins / 32;  // bins per lane


// Sequential fold over the visited bins in scan order (ascending when !desc),
// carrying (a, b, c) lane to lane: visit(j, a, b, c) updates the carry with
// owned bin j and records the running values. Lanes [klo, khi] own bins.
template <class Visit>
__device__ __forceinline__ void carry_chain(bool desc, int klo, int khi, double& a, double& b, int32_t& c,
                                            Visit visit) {
  const int lane = threadIdx.x & 31;
  if (desc) {
    for (int k = khi; k >= klo; --k) {
      if (lane == k) {
#pragma unroll
        for (int j = kPer - 1; j >= 0; --j) visit(j, a, b, c);
      }
      a = __shfl_sync(0xffffffffu, a, k);
      b = __shfl_sync(0xffffffffu, b, k);
      c = __shfl_sync(0xffffffffu, c, k);
    }
  } else {
    for (int k = klo; k <= khi; ++k) {
      if (lane == k) {
#pragma unroll
        for (int j = 0; j < kPer; ++j) visit(j, a, b, c);
      }
      a = __shfl_sync(0xffffffffu, a, k);
      b = __shfl_sync(0xffffffffu, b, k);
      c = __shfl_sync(0xffffffffu, c, k);
    }
  }
}

struct ScanBest {
  double gain;  // best gain (not yet minus min_gain_shift); -inf: none
  int32_t t;    // winning t, or INT32_MIN
  bool splittable;
  double acc_g, acc_h;  // cumulative (accumulated side) values at the winner (FP form)
  int32_t acc_c;
  int64_t acc_q;  // cumulative packed sum at the winner (quantized form)
};

// Warp reduction with the scan's rules: larger gain wins; at equal gain the
// candidate met first in scan order (reverse: larger t; forward: smaller t).
__device__ __forceinline__ void warp_pick(bool desc, double& gain, int32_t& t) {
  for (int o = 16; o > 0; o >>= 1) {
    double og = __shfl_xor_sync(0xffffffffu, gain, o);
    int32_t ot = __shfl_xor_sync(0xffffffffu, t, o);
    bool take = og > gain || (og == gain && ot != INT32_MIN && (t == INT32_MIN || (desc ? ot > t : ot < t)));
    if (take) {
      gain = og;
      t = ot;
    }
  }
}

// The update of `out` after one direction (split.rs:864-889 / :1167-1188), by
// one warp: lane 0 forms the left child's sums and output, lane 1 the right
// child's (the same expressions, so the same values), and lane 0 writes.
template <bool kInt>
__device__ void apply_direction(const ScanBest& r, const DFeature& m, const DParams& p, double sum_g, double sum_h,
                                int64_t int_sum, double gs, double hs, int32_t num_data, double parent_output, bool mc,
                                double cmin, double cmax, double min_gain_shift, double cnt_factor, bool reverse,
                                DSplit& out) {
  const int lane = threadIdx.x & 31;
  // a basic constraint with min > max never accepts a threshold (split.rs:765-771)
  if (r.t == INT32_MIN || (mc && cmin > cmax)) return;
  const double cur = out.gain;
  __syncwarp();
  if (!(r.splittable && r.gain > cur + min_gain_shift)) return;
  const bool right = (lane & 1) != 0;
  double g, h, o;
  int32_t cnt;
  int64_t q = 0;
  if (kInt) {
    const int64_t left = reverse ? (int64_t)((uint64_t)int_sum - (uint64_t)r.acc_q) : r.acc_q;
    q = right ? (int64_t)((uint64_t)int_sum - (uint64_t)left) : left;
    g = (double)int_grad(q) * gs;
    h = (double)int_hess(q) * hs;
    cnt = round_int((double)int_hess(q) * cnt_factor);
    o = leaf_output_hot(plain_split(p, mc), g, h, p, cnt, parent_output);
  } else {
    double slg, slh;
    int32_t left_count;
    if (reverse) {
      slg = sum_g - r.acc_g;
      slh = sum_h - r.acc_h;
      left_count = num_data - r.acc_c;
    } else {
      slg = r.acc_g;
      slh = r.acc_h;
      left_count = r.acc_c;
    }
    g = right ? sum_g - slg : slg;
    h = right ? sum_h - slh : slh;
    cnt = right ? num_data - left_count : left_count;
    o = leaf_output_hot(plain_split(p, mc), g, h, p, cnt, parent_output);
    h = right ? sum_h - slh - kEpsilon : slh - kEpsilon;  // the stored hessian sums
  }
  if (mc) o = clampc(o, cmin, cmax);
  const double rg = __shfl_sync(0xffffffffu, g, 1), rh = __shfl_sync(0xffffffffu, h, 1);
  const double ro = __shfl_sync(0xffffffffu, o, 1);
  const int32_t rc = __shfl_sync(0xffffffffu, cnt, 1);
  const int64_t rq = __shfl_sync(0xffffffffu, q, 1);
  if (lane == 0) {
    const int offset = m.offset;
    out.threshold = (uint32_t)(reverse ? r.t - 1 + offset : r.t + offset);
    out.left_output = o;
    out.right_output = ro;
    out.left_count = cnt;
    out.right_count = rc;
    out.left_sum_gradient = g;
    out.left_sum_hessian = h;
    out.right_sum_gradient = rg;
    out.right_sum_hessian = rh;
    if (kInt) {
      out.left_sum_gh = q;
      out.right_sum_gh = rq;
    }
    out.gain = r.gain - min_gain_shift;
    out.default_left = reverse ? 1 : 0;
  }
  __syncwarp();
}

}  // namespace lgbm_b200
