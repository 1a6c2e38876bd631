// Oracle: threshold search on one feature histogram — a restatement of
// crates/lgbm-core/src/learner/split.rs (FP64 and quantized scans) and
// histogram.rs (fix / subtract). Test infrastructure only.
#include "oracle_impl.h"

#include <algorithm>

namespace oracle {

static inline double sign(double x) { return (double)((x > 0.0) - (x < 0.0)); }  // split.rs:124-127

double threshold_l1(double s, double l1) {  // split.rs:129-133
  double reg = std::max(std::fabs(s) - l1, 0.0);
  return sign(s) * reg;
}

// split.rs:137-161 CalculateSplittedLeafOutput<USE_L1, USE_MAX_OUTPUT, USE_SMOOTHING>
double leaf_output_t(double g, double h, const SplitParams& p, bool use_l1, bool use_max, bool use_smooth,
                     int32_t num_data, double parent_output) {
  double ret = use_l1 ? -threshold_l1(g, p.lambda_l1) / (h + p.lambda_l2) : -g / (h + p.lambda_l2);
  if (use_max && p.max_delta_step > 0.0 && std::fabs(ret) > p.max_delta_step) ret = sign(ret) * p.max_delta_step;
  if (use_smooth) {
    double n = (double)num_data;
    ret = ret * (n / p.path_smooth) / (n / p.path_smooth + 1.0) + parent_output / (n / p.path_smooth + 1.0);
  }
  return ret;
}

static inline bool use_l1(const SplitParams& p) { return p.lambda_l1 > 0.0; }
static inline bool use_max_output(const SplitParams& p) { return p.max_delta_step > 0.0; }
static inline bool use_smoothing(const SplitParams& p) { return p.path_smooth > kEpsilon; }

double leaf_output(double g, double h, const SplitParams& p, int32_t num_data, double parent_output) {  // :165
  return leaf_output_t(g, h, p, use_l1(p), use_max_output(p), use_smoothing(p), num_data, parent_output);
}
double refit_leaf_output(double g, double h, const SplitParams& p, bool smooth, int32_t n, double parent) {  // :172
  return leaf_output_t(g, h, p, true, true, smooth, n, parent);
}
double root_output(double g, double h, const SplitParams& p, int32_t num_data) {  // :178
  return leaf_output_t(g, h, p, true, true, false, num_data, 0.0);
}

static inline double leaf_gain_given_output(double g, double h, const SplitParams& p, double output) {  // :183
  double sg = use_l1(p) ? threshold_l1(g, p.lambda_l1) : g;
  return -(2.0 * sg * output + (h + p.lambda_l2) * output * output);
}

static double leaf_gain(double g, double h, const SplitParams& p, int32_t num_data, double parent_output) {  // :189
  if (!use_max_output(p) && !use_smoothing(p)) {
    if (use_l1(p)) {
      double sg = threshold_l1(g, p.lambda_l1);
      return (sg * sg) / (h + p.lambda_l2);
    }
    return (g * g) / (h + p.lambda_l2);
  }
  double out = leaf_output(g, h, p, num_data, parent_output);
  return leaf_gain_given_output(g, h, p, out);
}

// split.rs:205-226; `mc` is the leaf's basic constraint when monotone
// constraints are configured (upstream USE_MC).
static double split_gain(double lg, double lh, double rg, double rh, const SplitParams& p, int32_t lc, int32_t rc,
                         double parent_output, const BasicConstraint* mc, int32_t monotone_type) {
  if (!mc) return leaf_gain(lg, lh, p, lc, parent_output) + leaf_gain(rg, rh, p, rc, parent_output);
  double left = mc->clamp(leaf_output(lg, lh, p, lc, parent_output));
  double right = mc->clamp(leaf_output(rg, rh, p, rc, parent_output));
  if ((monotone_type > 0 && left > right) || (monotone_type < 0 && left < right)) return 0.0;
  return leaf_gain_given_output(lg, lh, p, left) + leaf_gain_given_output(rg, rh, p, right);
}

static inline int32_t round_int(double x) { return (int32_t)(x + (double)0.5f); }  // split.rs:229-231

// split.rs:676-891 FindBestThresholdSequentially (no extra-trees draw).
static bool scan(const double* hist, const FeatureMeta& meta, const SplitParams& p, double sum_gradient,
                 double sum_hessian, int32_t num_data, double min_gain_shift, double parent_output, bool reverse,
                 bool skip_default_bin, bool na_as_missing, const BasicConstraint* mc, SplitInfo& out) {
  const int32_t offset = meta.offset;
  auto g = [&](int32_t t) { return hist[2 * t]; };
  auto h = [&](int32_t t) { return hist[2 * t + 1]; };
  bool is_splittable = false;
  double best_sum_left_gradient = NAN, best_sum_left_hessian = NAN;
  double best_gain = kMinScore;
  int32_t best_left_count = 0;
  uint32_t best_threshold = (uint32_t)meta.num_bin;
  double cnt_factor = (double)num_data / sum_hessian;
  int32_t min_data = p.min_data_in_leaf;
  double min_hess = p.min_sum_hessian_in_leaf;
  BasicConstraint best_left_c, best_right_c;
  int32_t mono = meta.monotone_type;

  if (reverse) {
    double sum_right_gradient = 0.0, sum_right_hessian = kEpsilon;
    int32_t right_count = 0;
    int32_t t = meta.num_bin - 1 - offset - (int32_t)na_as_missing;
    int32_t t_end = 1 - offset;
    for (; t >= t_end; --t) {
      if (skip_default_bin && (t + offset) == (int32_t)meta.default_bin) continue;
      double gr = g(t), hs = h(t);
      int32_t cnt = round_int(hs * cnt_factor);
      sum_right_gradient += gr;
      sum_right_hessian += hs;
      right_count += cnt;
      if (right_count < min_data || sum_right_hessian < min_hess) continue;
      int32_t left_count = num_data - right_count;
      if (left_count < min_data) break;
      double sum_left_hessian = sum_hessian - sum_right_hessian;
      if (sum_left_hessian < min_hess) break;
      double sum_left_gradient = sum_gradient - sum_right_gradient;
      double current_gain = split_gain(sum_left_gradient, sum_left_hessian, sum_right_gradient, sum_right_hessian, p,
                                       left_count, right_count, parent_output, mc, mono);
      if (current_gain <= min_gain_shift) continue;
      is_splittable = true;
      if (current_gain > best_gain) {
        if (mc) {
          best_right_c = *mc;
          best_left_c = *mc;
          if (best_right_c.min > best_right_c.max || best_left_c.min > best_left_c.max) continue;
        }
        best_left_count = left_count;
        best_sum_left_gradient = sum_left_gradient;
        best_sum_left_hessian = sum_left_hessian;
        best_threshold = (uint32_t)(t - 1 + offset);
        best_gain = current_gain;
      }
    }
  } else {
    double sum_left_gradient = 0.0, sum_left_hessian = kEpsilon;
    int32_t left_count = 0;
    int32_t t = 0;
    int32_t t_end = meta.num_bin - 2 - offset;
    if (na_as_missing && offset == 1) {
      sum_left_gradient = sum_gradient;
      sum_left_hessian = sum_hessian - kEpsilon;
      left_count = num_data;
      for (int32_t i = 0; i < meta.num_bin - offset; ++i) {
        double gr = g(i), hs = h(i);
        int32_t cnt = round_int(hs * cnt_factor);
        sum_left_gradient -= gr;
        sum_left_hessian -= hs;
        left_count -= cnt;
      }
      t = -1;
    }
    for (; t <= t_end; ++t) {
      if (skip_default_bin && (t + offset) == (int32_t)meta.default_bin) continue;
      if (t >= 0) {
        sum_left_gradient += g(t);
        sum_left_hessian += h(t);
        left_count += round_int(h(t) * cnt_factor);
      }
      if (left_count < min_data || sum_left_hessian < min_hess) continue;
      int32_t right_count = num_data - left_count;
      if (right_count < min_data) break;
      double sum_right_hessian = sum_hessian - sum_left_hessian;
      if (sum_right_hessian < min_hess) break;
      double sum_right_gradient = sum_gradient - sum_left_gradient;
      double current_gain = split_gain(sum_left_gradient, sum_left_hessian, sum_right_gradient, sum_right_hessian, p,
                                       left_count, right_count, parent_output, mc, mono);
      if (current_gain <= min_gain_shift) continue;
      is_splittable = true;
      if (current_gain > best_gain) {
        if (mc) {
          best_right_c = *mc;
          best_left_c = *mc;
          if (best_right_c.min > best_right_c.max || best_left_c.min > best_left_c.max) continue;
        }
        best_left_count = left_count;
        best_sum_left_gradient = sum_left_gradient;
        best_sum_left_hessian = sum_left_hessian;
        best_threshold = (uint32_t)(t + offset);
        best_gain = current_gain;
      }
    }
  }

  if (is_splittable && best_gain > out.gain + min_gain_shift) {
    auto clamp = [&](double v, const BasicConstraint& c) { return mc ? c.clamp(v) : v; };
    out.threshold = best_threshold;
    out.left_output =
        clamp(leaf_output(best_sum_left_gradient, best_sum_left_hessian, p, best_left_count, parent_output), best_left_c);
    out.left_count = best_left_count;
    out.left_sum_gradient = best_sum_left_gradient;
    out.left_sum_hessian = best_sum_left_hessian - kEpsilon;
    out.right_output = clamp(leaf_output(sum_gradient - best_sum_left_gradient, sum_hessian - best_sum_left_hessian, p,
                                         num_data - best_left_count, parent_output),
                             best_right_c);
    out.right_count = num_data - best_left_count;
    out.right_sum_gradient = sum_gradient - best_sum_left_gradient;
    out.right_sum_hessian = sum_hessian - best_sum_left_hessian - kEpsilon;
    out.gain = best_gain - min_gain_shift;
    out.default_left = reverse;
  }
  return is_splittable;
}

// split.rs:402-441 (BeforeNumerical + direction scans).
static bool numerical(const double* hist, const FeatureMeta& meta, const SplitParams& p, double sum_gradient,
                      double sum_hessian, int32_t num_data, double parent_output, const BasicConstraint* mc,
                      SplitInfo& out) {
  out.monotone_type = meta.monotone_type;
  double min_gain_shift = leaf_gain(sum_gradient, sum_hessian, p, num_data, parent_output) + p.min_gain_to_split;
  bool splittable = false;
  auto run = [&](bool reverse, bool skip_default, bool na_as_missing) {
    splittable |= scan(hist, meta, p, sum_gradient, sum_hessian, num_data, min_gain_shift, parent_output, reverse,
                       skip_default, na_as_missing, mc, out);
  };
  if (meta.num_bin > 2 && meta.missing_type != kMissingNone) {
    if (meta.missing_type == kMissingZero) {
      run(true, true, false);
      run(false, true, false);
    } else {
      run(true, false, true);
      run(false, false, true);
    }
  } else {
    run(true, false, false);
    if (meta.missing_type == kMissingNaN) out.default_left = false;
  }
  return splittable;
}

// split.rs:448-670 FindBestThresholdCategoricalInner (no extra trees).
static bool categorical(const double* hist, const FeatureMeta& meta, const SplitParams& p, double sum_gradient,
                        double sum_hessian, int32_t num_data, double parent_output, const BasicConstraint* mc,
                        SplitInfo& out) {
  auto g = [&](int32_t t) { return hist[2 * t]; };
  auto h = [&](int32_t t) { return hist[2 * t + 1]; };
  bool is_splittable = false;
  out.default_left = false;
  double best_gain = kMinScore;
  int32_t best_left_count = 0;
  double best_sum_left_gradient = 0.0, best_sum_left_hessian = 0.0;
  double gain_shift = use_smoothing(p) ? leaf_gain_given_output(sum_gradient, sum_hessian, p, parent_output)
                                       : leaf_gain(sum_gradient, sum_hessian, p, num_data, 0.0);
  double min_gain_shift = gain_shift + p.min_gain_to_split;
  int32_t offset = meta.offset;
  int32_t bin_start = 1 - offset, bin_end = meta.num_bin - offset;
  int32_t used_bin = -1;
  std::vector<int32_t> sorted_idx;
  SplitParams pc = p;
  bool use_onehot = meta.num_bin <= p.max_cat_to_onehot;
  int32_t best_threshold = -1, best_dir = 1;
  double cnt_factor = (double)num_data / sum_hessian;
  if (use_onehot) {
    for (int32_t t = bin_start; t < bin_end; ++t) {
      double grad = g(t), hess = h(t);
      int32_t cnt = round_int(hess * cnt_factor);
      if (cnt < p.min_data_in_leaf || hess < p.min_sum_hessian_in_leaf) continue;
      int32_t other_count = num_data - cnt;
      if (other_count < p.min_data_in_leaf) continue;
      double sum_other_hessian = sum_hessian - hess - kEpsilon;
      if (sum_other_hessian < p.min_sum_hessian_in_leaf) continue;
      double sum_other_gradient = sum_gradient - grad;
      double current_gain = split_gain(sum_other_gradient, sum_other_hessian, grad, hess + kEpsilon, pc, other_count,
                                       cnt, parent_output, mc, 0);
      if (current_gain <= min_gain_shift) continue;
      is_splittable = true;
      if (current_gain > best_gain) {
        best_threshold = t;
        best_sum_left_gradient = grad;
        best_sum_left_hessian = hess + kEpsilon;
        best_left_count = cnt;
        best_gain = current_gain;
      }
    }
  } else {
    for (int32_t i = bin_start; i < bin_end; ++i)
      if ((double)round_int(h(i) * cnt_factor) >= p.cat_smooth) sorted_idx.push_back(i);
    used_bin = (int32_t)sorted_idx.size();
    pc.lambda_l2 += p.cat_l2;
    auto ctr = [&](int32_t i) { return g(i) / (h(i) + p.cat_smooth); };
    std::stable_sort(sorted_idx.begin(), sorted_idx.end(), [&](int32_t a, int32_t b) { return ctr(a) < ctr(b); });
    int32_t max_num_cat = std::min(p.max_cat_threshold, (used_bin + 1) / 2);
    is_splittable = false;
    const int32_t dirs[2] = {1, -1};
    const int32_t starts[2] = {0, used_bin - 1};
    for (int d = 0; d < 2; ++d) {
      int32_t dir = dirs[d], start_pos = starts[d];
      int32_t cnt_cur_group = 0;
      double sum_left_gradient = 0.0, sum_left_hessian = kEpsilon;
      int32_t left_count = 0;
      for (int32_t i = 0; i < used_bin && i < max_num_cat; ++i) {
        int32_t t = sorted_idx[start_pos];
        start_pos += dir;
        double grad = g(t), hess = h(t);
        int32_t cnt = round_int(hess * cnt_factor);
        sum_left_gradient += grad;
        sum_left_hessian += hess;
        left_count += cnt;
        cnt_cur_group += cnt;
        if (left_count < p.min_data_in_leaf || sum_left_hessian < p.min_sum_hessian_in_leaf) continue;
        int32_t right_count = num_data - left_count;
        if (right_count < p.min_data_in_leaf || right_count < p.min_data_per_group) break;
        double sum_right_hessian = sum_hessian - sum_left_hessian;
        if (sum_right_hessian < p.min_sum_hessian_in_leaf) break;
        if (cnt_cur_group < p.min_data_per_group) continue;
        cnt_cur_group = 0;
        double sum_right_gradient = sum_gradient - sum_left_gradient;
        double current_gain = split_gain(sum_left_gradient, sum_left_hessian, sum_right_gradient, sum_right_hessian, pc,
                                         left_count, right_count, parent_output, mc, 0);
        if (current_gain <= min_gain_shift) continue;
        is_splittable = true;
        if (current_gain > best_gain) {
          best_left_count = left_count;
          best_sum_left_gradient = sum_left_gradient;
          best_sum_left_hessian = sum_left_hessian;
          best_threshold = i;
          best_gain = current_gain;
          best_dir = dir;
        }
      }
    }
  }
  if (is_splittable) {
    auto clamp = [&](double v) { return mc ? mc->clamp(v) : v; };
    out.left_output = clamp(leaf_output(best_sum_left_gradient, best_sum_left_hessian, pc, best_left_count, parent_output));
    out.left_count = best_left_count;
    out.left_sum_gradient = best_sum_left_gradient;
    out.left_sum_hessian = best_sum_left_hessian - kEpsilon;
    out.right_output = clamp(leaf_output(sum_gradient - best_sum_left_gradient, sum_hessian - best_sum_left_hessian, pc,
                                         num_data - best_left_count, parent_output));
    out.monotone_type = 0;
    out.right_count = num_data - best_left_count;
    out.right_sum_gradient = sum_gradient - best_sum_left_gradient;
    out.right_sum_hessian = sum_hessian - best_sum_left_hessian - kEpsilon;
    out.gain = best_gain - min_gain_shift;
    out.cat_threshold.clear();
    if (use_onehot) {
      out.cat_threshold.push_back((uint32_t)(best_threshold + offset));
    } else if (best_dir == 1) {
      for (int32_t i = 0; i <= best_threshold; ++i) out.cat_threshold.push_back((uint32_t)(sorted_idx[i] + offset));
    } else {
      for (int32_t i = 0; i <= best_threshold; ++i)
        out.cat_threshold.push_back((uint32_t)(sorted_idx[used_bin - 1 - i] + offset));
    }
  }
  return is_splittable;
}

// split.rs:246-271 find_best_threshold.
bool find_best_threshold(const double* hist, const FeatureMeta& meta, const SplitParams& p, double sum_gradient,
                         double sum_hessian, int32_t num_data, double parent_output, const BasicConstraint* mc,
                         SplitInfo& out) {
  out.default_left = true;
  out.gain = kMinScore;
  double sh = sum_hessian + 2.0 * kEpsilon;
  bool ok = meta.bin_type == kCategorical
                ? categorical(hist, meta, p, sum_gradient, sh, num_data, parent_output, mc, out)
                : numerical(hist, meta, p, sum_gradient, sh, num_data, parent_output, mc, out);
  out.gain *= meta.penalty;
  return ok;
}

// ---- quantized (split.rs:893-1400) ------------------------------------------------
static inline int32_t int_grad(int64_t x) { return (int32_t)(x >> 32); }
static inline uint32_t int_hess(int64_t x) { return (uint32_t)x; }
static inline int64_t wadd(int64_t a, int64_t b) { return (int64_t)((uint64_t)a + (uint64_t)b); }
static inline int64_t wsub(int64_t a, int64_t b) { return (int64_t)((uint64_t)a - (uint64_t)b); }

struct IntSums {
  int64_t sum;
  double gs, hs;
  double gradient() const { return (double)int_grad(sum) * gs; }
  double hessian() const { return (double)int_hess(sum) * hs; }
  double cnt_factor(int32_t n) const { return (double)n / (double)int_hess(sum); }
};

// split.rs:995-1190 FindBestThresholdSequentiallyInt.
static bool scan_int(const int64_t* hist, const FeatureMeta& meta, const SplitParams& p, IntSums sums, int32_t num_data,
                     double min_gain_shift, double parent_output, bool reverse, bool skip_default_bin,
                     bool na_as_missing, const BasicConstraint* mc, SplitInfo& out) {
  int32_t offset = meta.offset;
  double gs = sums.gs, hs = sums.hs;
  int64_t local_sum = sums.sum;
  int64_t best_sum_left = 0;
  double best_gain = kMinScore;
  uint32_t best_threshold = (uint32_t)meta.num_bin;
  double cnt_factor = sums.cnt_factor(num_data);
  int32_t min_data = p.min_data_in_leaf;
  double min_hess = p.min_sum_hessian_in_leaf;
  BasicConstraint best_left_c, best_right_c;
  int32_t mono = meta.monotone_type;
  bool is_splittable = false;
  if (reverse) {
    int64_t sum_right = 0;
    int32_t t = meta.num_bin - 1 - offset - (int32_t)na_as_missing;
    int32_t t_end = 1 - offset;
    for (; t >= t_end; --t) {
      if (skip_default_bin && (t + offset) == (int32_t)meta.default_bin) continue;
      sum_right = wadd(sum_right, hist[t]);
      int32_t right_count = round_int((double)int_hess(sum_right) * cnt_factor);
      double sum_right_hessian = (double)int_hess(sum_right) * hs;
      if (right_count < min_data || sum_right_hessian < min_hess) continue;
      int32_t left_count = num_data - right_count;
      if (left_count < min_data) break;
      int64_t sum_left = wsub(local_sum, sum_right);
      double sum_left_hessian = (double)int_hess(sum_left) * hs;
      if (sum_left_hessian < min_hess) break;
      double sum_right_gradient = (double)int_grad(sum_right) * gs;
      double sum_left_gradient = (double)int_grad(sum_left) * gs;
      double current_gain = split_gain(sum_left_gradient, sum_left_hessian + kEpsilon, sum_right_gradient,
                                       sum_right_hessian + kEpsilon, p, left_count, right_count, parent_output, mc, mono);
      if (current_gain <= min_gain_shift) continue;
      is_splittable = true;
      if (current_gain > best_gain) {
        if (mc) {
          best_right_c = *mc;
          best_left_c = *mc;
          if (best_right_c.min > best_right_c.max || best_left_c.min > best_left_c.max) continue;
        }
        best_sum_left = sum_left;
        best_threshold = (uint32_t)(t - 1 + offset);
        best_gain = current_gain;
      }
    }
  } else {
    int64_t sum_left = 0;
    int32_t t = 0;
    int32_t t_end = meta.num_bin - 2 - offset;
    if (na_as_missing && offset == 1) {
      sum_left = local_sum;
      for (int32_t i = 0; i < meta.num_bin - offset; ++i) sum_left = wsub(sum_left, hist[i]);
      t = -1;
    }
    for (; t <= t_end; ++t) {
      if (skip_default_bin && (t + offset) == (int32_t)meta.default_bin) continue;
      if (t >= 0) sum_left = wadd(sum_left, hist[t]);
      int32_t left_count = round_int((double)int_hess(sum_left) * cnt_factor);
      double sum_left_hessian = (double)int_hess(sum_left) * hs;
      if (left_count < min_data || sum_left_hessian < min_hess) continue;
      int32_t right_count = num_data - left_count;
      if (right_count < min_data) break;
      int64_t sum_right = wsub(local_sum, sum_left);
      double sum_right_hessian = (double)int_hess(sum_right) * hs;
      if (sum_right_hessian < min_hess) break;
      double sum_right_gradient = (double)int_grad(sum_right) * gs;
      double sum_left_gradient = (double)int_grad(sum_left) * gs;
      double current_gain = split_gain(sum_left_gradient, sum_left_hessian + kEpsilon, sum_right_gradient,
                                       sum_right_hessian + kEpsilon, p, left_count, right_count, parent_output, mc, mono);
      if (current_gain <= min_gain_shift) continue;
      is_splittable = true;
      if (current_gain > best_gain) {
        if (mc) {
          best_right_c = *mc;
          best_left_c = *mc;
          if (best_right_c.min > best_right_c.max || best_left_c.min > best_left_c.max) continue;
        }
        best_sum_left = sum_left;
        best_threshold = (uint32_t)(t + offset);
        best_gain = current_gain;
      }
    }
  }
  if (is_splittable && best_gain > out.gain + min_gain_shift) {
    auto clamp = [&](double v, const BasicConstraint& c) { return mc ? c.clamp(v) : v; };
    int64_t left = best_sum_left;
    int64_t right = wsub(sums.sum, left);
    double left_g = (double)int_grad(left) * gs, left_h = (double)int_hess(left) * hs;
    double right_g = (double)int_grad(right) * gs, right_h = (double)int_hess(right) * hs;
    int32_t left_count = round_int((double)int_hess(left) * cnt_factor);
    int32_t right_count = round_int((double)int_hess(right) * cnt_factor);
    out.threshold = best_threshold;
    out.left_output = clamp(leaf_output(left_g, left_h, p, left_count, parent_output), best_left_c);
    out.left_count = left_count;
    out.left_sum_gradient = left_g;
    out.left_sum_hessian = left_h;
    out.left_sum_gh = left;
    out.right_output = clamp(leaf_output(right_g, right_h, p, right_count, parent_output), best_right_c);
    out.right_count = right_count;
    out.right_sum_gradient = right_g;
    out.right_sum_hessian = right_h;
    out.right_sum_gh = right;
    out.gain = best_gain - min_gain_shift;
    out.default_left = reverse;
  }
  return is_splittable;
}

// split.rs:954-990
static bool numerical_int(const int64_t* hist, const FeatureMeta& meta, const SplitParams& p, IntSums sums,
                          int32_t num_data, double parent_output, const BasicConstraint* mc, SplitInfo& out) {
  out.monotone_type = meta.monotone_type;
  double min_gain_shift = leaf_gain(sums.gradient(), sums.hessian(), p, num_data, parent_output) + p.min_gain_to_split;
  bool splittable = false;
  auto run = [&](bool reverse, bool skip_default, bool na_as_missing) {
    splittable |= scan_int(hist, meta, p, sums, num_data, min_gain_shift, parent_output, reverse, skip_default,
                           na_as_missing, mc, out);
  };
  if (meta.num_bin > 2 && meta.missing_type != kMissingNone) {
    if (meta.missing_type == kMissingZero) {
      run(true, true, false);
      run(false, true, false);
    } else {
      run(true, false, true);
      run(false, false, true);
    }
  } else {
    run(true, false, false);
    if (meta.missing_type == kMissingNaN) out.default_left = false;
  }
  return splittable;
}

// split.rs:1194-1400 FindBestThresholdCategoricalIntInner.
static bool categorical_int(const int64_t* hist, const FeatureMeta& meta, const SplitParams& p, IntSums sums,
                            int32_t num_data, double parent_output, const BasicConstraint* mc, SplitInfo& out) {
  double gs = sums.gs, hs = sums.hs;
  bool is_splittable = false;
  out.default_left = false;
  double best_gain = kMinScore;
  int64_t best_sum_left = 0;
  int64_t local_sum = sums.sum;
  double sum_gradient = sums.gradient(), sum_hessian = sums.hessian();
  double gain_shift = use_smoothing(p) ? leaf_gain_given_output(sum_gradient, sum_hessian, p, parent_output)
                                       : leaf_gain(sum_gradient, sum_hessian, p, num_data, 0.0);
  double min_gain_shift = gain_shift + p.min_gain_to_split;
  int32_t offset = meta.offset;
  int32_t bin_start = 1 - offset, bin_end = meta.num_bin - offset;
  int32_t used_bin = -1;
  std::vector<int32_t> sorted_idx;
  SplitParams pc = p;
  bool use_onehot = meta.num_bin <= p.max_cat_to_onehot;
  int32_t best_threshold = -1, best_dir = 1;
  double cnt_factor = sums.cnt_factor(num_data);
  if (use_onehot) {
    for (int32_t t = bin_start; t < bin_end; ++t) {
      int64_t gh = hist[t];
      int32_t cnt = round_int((double)int_hess(gh) * cnt_factor);
      double hess = (double)int_hess(gh) * hs;
      if (cnt < p.min_data_in_leaf || hess < p.min_sum_hessian_in_leaf) continue;
      int32_t other_count = num_data - cnt;
      if (other_count < p.min_data_in_leaf) continue;
      int64_t sum_other = wsub(local_sum, gh);
      double sum_other_hessian = (double)int_hess(sum_other) * hs;
      if (sum_other_hessian < p.min_sum_hessian_in_leaf) continue;
      double grad = (double)int_grad(gh) * gs;
      double sum_other_gradient = (double)int_grad(sum_other) * gs;
      double current_gain =
          split_gain(sum_other_gradient, sum_other_hessian, grad, hess, pc, other_count, cnt, parent_output, mc, 0);
      if (current_gain <= min_gain_shift) continue;
      is_splittable = true;
      if (current_gain > best_gain) {
        best_threshold = t;
        best_sum_left = gh;
        best_gain = current_gain;
      }
    }
  } else {
    for (int32_t i = bin_start; i < bin_end; ++i)
      if ((double)round_int((double)int_hess(hist[i]) * cnt_factor) >= p.cat_smooth) sorted_idx.push_back(i);
    used_bin = (int32_t)sorted_idx.size();
    pc.lambda_l2 += p.cat_l2;
    auto ctr = [&](int32_t i) {
      int64_t gh = hist[i];
      return ((double)int_grad(gh) * gs) / ((double)int_hess(gh) * hs + p.cat_smooth);
    };
    std::stable_sort(sorted_idx.begin(), sorted_idx.end(), [&](int32_t a, int32_t b) { return ctr(a) < ctr(b); });
    int32_t max_num_cat = std::min(p.max_cat_threshold, (used_bin + 1) / 2);
    const int32_t dirs[2] = {1, -1};
    const int32_t starts[2] = {0, used_bin - 1};
    for (int d = 0; d < 2; ++d) {
      int32_t dir = dirs[d], start_pos = starts[d];
      int32_t cnt_cur_group = 0;
      int64_t sum_left = 0;
      int32_t left_count = 0;
      for (int32_t i = 0; i < used_bin && i < max_num_cat; ++i) {
        int32_t t = sorted_idx[start_pos];
        start_pos += dir;
        int64_t gh = hist[t];
        int32_t cnt = round_int((double)int_hess(gh) * cnt_factor);
        sum_left = wadd(sum_left, gh);
        left_count += cnt;
        cnt_cur_group += cnt;
        double sum_left_hessian = (double)int_hess(sum_left) * hs;
        if (left_count < p.min_data_in_leaf || sum_left_hessian < p.min_sum_hessian_in_leaf) continue;
        int32_t right_count = num_data - left_count;
        if (right_count < p.min_data_in_leaf || right_count < p.min_data_per_group) break;
        int64_t sum_right = wsub(local_sum, sum_left);
        double sum_right_hessian = (double)int_hess(sum_right) * hs;
        if (sum_right_hessian < p.min_sum_hessian_in_leaf) break;
        if (cnt_cur_group < p.min_data_per_group) continue;
        cnt_cur_group = 0;
        double sum_left_gradient = (double)int_grad(sum_left) * gs;
        double sum_right_gradient = (double)int_grad(sum_right) * gs;
        double current_gain = split_gain(sum_left_gradient, sum_left_hessian, sum_right_gradient, sum_right_hessian, pc,
                                         left_count, right_count, parent_output, mc, 0);
        if (current_gain <= min_gain_shift) continue;
        is_splittable = true;
        if (current_gain > best_gain) {
          best_sum_left = sum_left;
          best_threshold = i;
          best_gain = current_gain;
          best_dir = dir;
        }
      }
    }
  }
  if (is_splittable) {
    auto clamp = [&](double v) { return mc ? mc->clamp(v) : v; };
    int64_t left = best_sum_left;
    int64_t right = wsub(local_sum, left);
    double left_g = (double)int_grad(left) * gs, left_h = (double)int_hess(left) * hs;
    double right_g = (double)int_grad(right) * gs, right_h = (double)int_hess(right) * hs;
    int32_t left_count = round_int((double)int_hess(left) * cnt_factor);
    int32_t right_count = round_int((double)int_hess(right) * cnt_factor);
    out.left_output = clamp(leaf_output(left_g, left_h, pc, left_count, parent_output));
    out.left_count = left_count;
    out.left_sum_gradient = left_g;
    out.left_sum_hessian = left_h;
    out.right_output = clamp(leaf_output(right_g, right_h, pc, right_count, parent_output));
    out.right_count = right_count;
    out.right_sum_gradient = right_g;
    out.right_sum_hessian = right_h;
    out.gain = best_gain - min_gain_shift;
    out.left_sum_gh = left;
    out.right_sum_gh = right;
    out.cat_threshold.clear();
    if (use_onehot) {
      out.cat_threshold.push_back((uint32_t)(best_threshold + offset));
    } else if (best_dir == 1) {
      for (int32_t i = 0; i <= best_threshold; ++i) out.cat_threshold.push_back((uint32_t)(sorted_idx[i] + offset));
    } else {
      for (int32_t i = 0; i <= best_threshold; ++i)
        out.cat_threshold.push_back((uint32_t)(sorted_idx[used_bin - 1 - i] + offset));
    }
    out.monotone_type = 0;
  }
  return is_splittable;
}

// split.rs:930-950
bool find_best_threshold_int(const int64_t* hist, const FeatureMeta& meta, const SplitParams& p, int64_t sum,
                             double grad_scale, double hess_scale, int32_t num_data, double parent_output,
                             const BasicConstraint* mc, SplitInfo& out) {
  out.default_left = true;
  out.gain = kMinScore;
  IntSums s{sum, grad_scale, hess_scale};
  bool ok = meta.bin_type == kCategorical ? categorical_int(hist, meta, p, s, num_data, parent_output, mc, out)
                                          : numerical_int(hist, meta, p, s, num_data, parent_output, mc, out);
  out.gain *= meta.penalty;
  return ok;
}

// histogram.rs:42-56 FixHistogram on one feature view.
void fix_hist(const FeatureMeta& m, double sum_g, double sum_h, double* hist) {
  uint32_t mfb = m.most_freq_bin;
  if (mfb > 0) {
    double g = sum_g, h = sum_h;
    for (int32_t i = 0; i < m.num_bin; ++i) {
      if ((uint32_t)i != mfb) {
        g -= hist[2 * i];
        h -= hist[2 * i + 1];
      }
    }
    hist[2 * mfb] = g;
    hist[2 * mfb + 1] = h;
  }
}

// histogram.rs:67-78 FixHistogramInt.
void fix_hist_int(const FeatureMeta& m, int64_t int_sum, int64_t* hist) {
  uint32_t mfb = m.most_freq_bin;
  if (mfb > 0) {
    int64_t s = int_sum;
    for (int32_t i = 0; i < m.num_bin; ++i)
      if ((uint32_t)i != mfb) s = wsub(s, hist[i]);
    hist[mfb] = s;
  }
}

}  // namespace oracle
