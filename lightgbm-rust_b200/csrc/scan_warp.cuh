// Warp-parallel numerical threshold scan (split.rs:676-891 and :995-1190)
// that reproduces the reference's sequential loop exactly.
//
// Each lane owns 8 consecutive stored bins of the feature view. The FP64
// cumulative sums must be formed in the reference's order (one add per
// visited bin, in scan order), so they are computed as a carry chain: the
// lane holding the first bins in scan order adds its bins to the carry and
// passes it on with a shuffle. Every other quantity (count estimates,
// break / skip rules, gains, the argmax) is evaluated in parallel. Packed
// integer sums are exact in any order, so the quantized form uses a plain
// warp prefix scan.
#pragma once
#include "device_common.cuh"

namespace lgbm_b200 {

constexpr int kPer = kMaxBins / 32;  // bins per lane

struct LaneBins {
  double g[kPer], h[kPer];
  int64_t q[kPer];
};

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

// One direction of FindBestThresholdSequentially. `v` holds this lane's bins
// (the view is [0, len) stored bins); cnt_est[j] the reference's count
// estimate of owned bin j. Returns the best candidate of the direction.
template <bool kInt>
__device__ ScanBest scan_direction(const LaneBins& v, const int32_t (&cnt_est)[kPer], const DFeature& m,
                                   const DParams& p, double sum_g, double sum_h, int64_t int_sum, double gs, double hs,
                                   int32_t num_data, double parent_output, bool mc, double cmin, double cmax,
                                   double min_gain_shift, double cnt_factor, bool reverse, bool skip_default,
                                   bool na_as_missing) {
  const int lane = threadIdx.x & 31;
  const int offset = m.offset;
  const int len = m.view_len;
  const int klo = 0, khi = len > 0 ? (len - 1) / kPer : -1;
  int32_t t_lo, t_hi;
  if (reverse) {
    t_hi = m.num_bin - 1 - offset - (int32_t)na_as_missing;
    t_lo = 1 - offset;
  } else {
    t_lo = 0;
    t_hi = m.num_bin - 2 - offset;
  }
  const int32_t skip_t = skip_default ? m.default_bin - offset : INT32_MIN;
  double cg[kPer], ch[kPer];
  int32_t cc[kPer];
  int64_t cq[kPer];
  bool vis[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    int t = lane * kPer + j;
    vis[j] = t >= t_lo && t <= t_hi && t != skip_t && t < len;
    cg[j] = ch[j] = 0.0;
    cc[j] = 0;
    cq[j] = 0;
  }
  // extra candidate t = -1 (forward with NaN missing and no stored bin 0)
  const bool first_extra = !reverse && na_as_missing && offset == 1;
  double eg = 0.0, eh = 0.0;
  int32_t ec = 0;
  int64_t eq = 0;
  if (!kInt) {
    double a = 0.0, b = kEpsilon;
    int32_t c = 0;
    if (first_extra) {  // split.rs:787-800: start from the leaf sums minus every bin, ascending
      a = sum_g;
      b = sum_h - kEpsilon;
      c = num_data;
      const int32_t nstored = m.num_bin - offset;
      carry_chain(false, klo, khi, a, b, c, [&](int j, double& x, double& y, int32_t& z) {
        int t = lane * kPer + j;
        if (t < nstored) {
          x -= v.g[j];
          y -= v.h[j];
          z -= cnt_est[j];
        }
      });
      eg = a;
      eh = b;
      ec = c;
    }
    carry_chain(reverse, klo, khi, a, b, c, [&](int j, double& x, double& y, int32_t& z) {
      if (vis[j]) {
        x += v.g[j];
        y += v.h[j];
        z += cnt_est[j];
        cg[j] = x;
        ch[j] = y;
        cc[j] = z;
      }
    });
  } else {
    // exact packed sums: local sequential part plus a warp scan of lane totals in scan order
    int64_t loc = 0;
    if (reverse) {
#pragma unroll
      for (int j = kPer - 1; j >= 0; --j)
        if (vis[j]) {
          loc = (int64_t)((uint64_t)loc + (uint64_t)v.q[j]);
          cq[j] = loc;
        }
    } else {
#pragma unroll
      for (int j = 0; j < kPer; ++j)
        if (vis[j]) {
          loc = (int64_t)((uint64_t)loc + (uint64_t)v.q[j]);
          cq[j] = loc;
        }
    }
    // inclusive scan of lane totals (reverse: from lane 31 down)
    int64_t incl = loc;
    for (int o = 1; o < 32; o <<= 1) {
      int64_t other = reverse ? __shfl_down_sync(0xffffffffu, incl, o) : __shfl_up_sync(0xffffffffu, incl, o);
      bool ok = reverse ? lane + o < 32 : lane >= o;
      if (ok) incl = (int64_t)((uint64_t)incl + (uint64_t)other);
    }
    int64_t excl = (int64_t)((uint64_t)incl - (uint64_t)loc);
    int64_t base = 0;
    if (first_extra) {
      int64_t all = 0;
#pragma unroll
      for (int j = 0; j < kPer; ++j)
        if (lane * kPer + j < m.num_bin - offset) all = (int64_t)((uint64_t)all + (uint64_t)v.q[j]);
      for (int o = 16; o > 0; o >>= 1) all = (int64_t)((uint64_t)all + (uint64_t)__shfl_xor_sync(0xffffffffu, all, o));
      base = (int64_t)((uint64_t)int_sum - (uint64_t)all);
      eq = base;
    }
#pragma unroll
    for (int j = 0; j < kPer; ++j)
      if (vis[j]) {
        cq[j] = (int64_t)((uint64_t)base + (uint64_t)excl + (uint64_t)cq[j]);
        cc[j] = round_int((double)int_hess(cq[j]) * cnt_factor);
      }
    if (first_extra) ec = round_int((double)int_hess(eq) * cnt_factor);
  }
  const int32_t min_data = p.min_data_in_leaf;
  const double min_hess = p.min_sum_hessian_in_leaf;
  // accumulated side's hessian / count and the rest side's, for candidate j
  auto sides = [&](double acc_h, int32_t acc_c, int64_t acc_q, double& ha, double& hr) {
    if (kInt) {
      ha = (double)int_hess(acc_q) * hs;
      hr = (double)int_hess((int64_t)((uint64_t)int_sum - (uint64_t)acc_q)) * hs;
    } else {
      ha = acc_h;
      hr = sum_h - acc_h;
    }
  };
  // pass 1: the first break in scan order
  int32_t brk = reverse ? INT32_MIN : INT32_MAX;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    if (!vis[j]) continue;
    int t = lane * kPer + j;
    double ha, hr;
    sides(ch[j], cc[j], cq[j], ha, hr);
    bool skip1 = cc[j] < min_data || ha < min_hess;
    if (!skip1 && (num_data - cc[j] < min_data || hr < min_hess)) brk = reverse ? max(brk, t) : min(brk, t);
  }
  if (first_extra && lane == 0) {
    double ha, hr;
    sides(eh, ec, eq, ha, hr);
    bool skip1 = ec < min_data || ha < min_hess;
    if (!skip1 && (num_data - ec < min_data || hr < min_hess)) brk = -1;
  }
  for (int o = 16; o > 0; o >>= 1) {
    int32_t ob = __shfl_xor_sync(0xffffffffu, brk, o);
    brk = reverse ? max(brk, ob) : min(brk, ob);
  }
  // pass 2: gains of the candidates before the break
  double best_gain = -INFINITY;
  int32_t best_t = INT32_MIN;
  bool splittable = false;
  auto eval = [&](int t, double ag, double ah, int32_t ac, int64_t aq) {
    double ha, hr;
    sides(ah, ac, aq, ha, hr);
    if (ac < min_data || ha < min_hess) return;
    double ga, gr;
    if (kInt) {
      int64_t rest = (int64_t)((uint64_t)int_sum - (uint64_t)aq);
      ga = (double)int_grad(aq) * gs;
      gr = (double)int_grad(rest) * gs;
      ha += kEpsilon;
      hr += kEpsilon;
    } else {
      ga = ag;
      gr = sum_g - ag;
    }
    int32_t rc = num_data - ac;
    double gain = reverse ? split_gain(gr, hr, ga, ha, p, rc, ac, parent_output, mc, cmin, cmax, m.monotone_type)
                          : split_gain(ga, ha, gr, hr, p, ac, rc, parent_output, mc, cmin, cmax, m.monotone_type);
    if (gain <= min_gain_shift) return;
    splittable = true;
    if (gain > best_gain || (gain == best_gain && best_t != INT32_MIN && (reverse ? t > best_t : t < best_t))) {
      best_gain = gain;
      best_t = t;
    }
  };
  if (first_extra && lane == 0 && brk > -1) eval(-1, eg, eh, ec, eq);
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    if (!vis[j]) continue;
    int t = lane * kPer + j;
    if (reverse ? t <= brk : t >= brk) continue;
    eval(t, cg[j], ch[j], cc[j], cq[j]);
  }
  ScanBest r;
  r.splittable = __any_sync(0xffffffffu, splittable);
  warp_pick(reverse, best_gain, best_t);
  r.gain = best_gain;
  r.t = best_t;
  // cumulative values of the winner, from its owner lane
  int owner = best_t == INT32_MIN ? 0 : (best_t < 0 ? 0 : best_t / kPer);
  int jj = best_t < 0 ? 0 : best_t % kPer;
  double wg = 0.0, wh = 0.0;
  int32_t wc = 0;
  int64_t wq = 0;
#pragma unroll
  for (int j = 0; j < kPer; ++j)
    if (j == jj) {
      wg = cg[j];
      wh = ch[j];
      wc = cc[j];
      wq = cq[j];
    }
  if (best_t == -1) {
    wg = eg;
    wh = eh;
    wc = ec;
    wq = eq;
  }
  r.acc_g = __shfl_sync(0xffffffffu, wg, owner);
  r.acc_h = __shfl_sync(0xffffffffu, wh, owner);
  r.acc_c = __shfl_sync(0xffffffffu, wc, owner);
  r.acc_q = __shfl_sync(0xffffffffu, wq, owner);
  return r;
}

// The update of `out` after one direction (split.rs:864-889 / :1167-1188), lane 0.
template <bool kInt>
__device__ void apply_direction(const ScanBest& r, const DFeature& m, const DParams& p, double sum_g, double sum_h,
                                int64_t int_sum, double gs, double hs, int32_t num_data, double parent_output, bool mc,
                                double cmin, double cmax, double min_gain_shift, double cnt_factor, bool reverse,
                                DSplit& out) {
  // a basic constraint with min > max never accepts a threshold (split.rs:765-771)
  if (r.t == INT32_MIN || (mc && cmin > cmax)) return;
  if (!(r.splittable && r.gain > out.gain + min_gain_shift)) return;
  const int offset = m.offset;
  out.threshold = (uint32_t)(reverse ? r.t - 1 + offset : r.t + offset);
  if (kInt) {
    int64_t left = reverse ? (int64_t)((uint64_t)int_sum - (uint64_t)r.acc_q) : r.acc_q;
    int64_t right = (int64_t)((uint64_t)int_sum - (uint64_t)left);
    double lg = (double)int_grad(left) * gs, lh = (double)int_hess(left) * hs;
    double rg = (double)int_grad(right) * gs, rh = (double)int_hess(right) * hs;
    int32_t lcnt = round_int((double)int_hess(left) * cnt_factor);
    int32_t rcnt = round_int((double)int_hess(right) * cnt_factor);
    double lo = leaf_output(lg, lh, p, lcnt, parent_output);
    double ro = leaf_output(rg, rh, p, rcnt, parent_output);
    out.left_output = mc ? clampc(lo, cmin, cmax) : lo;
    out.right_output = mc ? clampc(ro, cmin, cmax) : ro;
    out.left_count = lcnt;
    out.right_count = rcnt;
    out.left_sum_gradient = lg;
    out.left_sum_hessian = lh;
    out.right_sum_gradient = rg;
    out.right_sum_hessian = rh;
    out.left_sum_gh = left;
    out.right_sum_gh = right;
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
    double lo = leaf_output(slg, slh, p, left_count, parent_output);
    double ro = leaf_output(sum_g - slg, sum_h - slh, p, num_data - left_count, parent_output);
    out.left_output = mc ? clampc(lo, cmin, cmax) : lo;
    out.right_output = mc ? clampc(ro, cmin, cmax) : ro;
    out.left_count = left_count;
    out.left_sum_gradient = slg;
    out.left_sum_hessian = slh - kEpsilon;
    out.right_count = num_data - left_count;
    out.right_sum_gradient = sum_g - slg;
    out.right_sum_hessian = sum_h - slh - kEpsilon;
  }
  out.gain = r.gain - min_gain_shift;
  out.default_left = reverse ? 1 : 0;
}

}  // namespace lgbm_b200
