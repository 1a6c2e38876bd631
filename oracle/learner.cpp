// Oracle: the serial leaf-wise tree learner — a restatement of
// crates/lgbm-core/src/learner/mod.rs (train, find_best_splits, split),
// learner/partition.rs (stable DataPartition) and the row-wise histogram
// build of multi_val_bin.rs at one thread. Test infrastructure only.
//
// Scope: dense single-feature groups (u8 values), row-wise layout, no
// forced splits / CEGB / linear trees / extra trees / interaction
// constraints; bagging without subset; basic monotone constraints.
#include <omp.h>

#include <algorithm>
#include <memory>
#include <stdexcept>

#include "oracle_impl.h"

namespace oracle {

static double monotone_split_gain_penalty(int32_t depth, double penalization) {  // constraints.rs:852-861
  double d = (double)depth;
  if (penalization >= d + 1.0) return kEpsilon;
  if (penalization <= 1.0) return 1.0 - penalization / std::pow(2.0, d) + kEpsilon;
  return 1.0 - std::pow(2.0, penalization - 1.0 - d) + kEpsilon;
}

SerialTreeLearner::SerialTreeLearner(const BinnedData* data, const LearnerConfig& cfg) : d_(data), cfg_(cfg) {
  cfg_.num_leaves = std::max(cfg.num_leaves, 2);
  int32_t nf = d_->num_features;
  view_start_.resize(nf);
  size_t pos = 0;
  for (int32_t f = 0; f < nf; ++f) {
    view_start_[f] = pos;
    pos += (size_t)(d_->metas[f].num_bin - d_->metas[f].offset);
  }
  total_bins_ = pos;
  bytree_.assign(nf, true);
  indices_.resize((size_t)d_->num_data);
  leaf_begin_.assign(cfg_.num_leaves, 0);
  leaf_count_.assign(cfg_.num_leaves, 0);
  hist_.resize(cfg_.num_leaves);
  ihist_.resize(cfg_.num_leaves);
  splittable_.assign(cfg_.num_leaves, std::vector<bool>(nf, true));
  best_split_per_leaf_.resize(cfg_.num_leaves);
  constraints_.resize(cfg_.num_leaves);
  if (cfg_.quantized)
    quant_ = std::make_unique<GradientDiscretizer>(cfg_.num_grad_quant_bins, cfg_.seed, cfg_.is_constant_hessian,
                                                   cfg_.stochastic_rounding, (size_t)d_->num_data,
                                                   (size_t)std::max(cfg_.num_threads, 1));
}

void SerialTreeLearner::set_bagging_data(const uint32_t* used, size_t n_used) {  // learner/mod.rs:545-568
  if (used) {
    bagging_ = true;
    used_.assign(used, used + n_used);
  } else {
    bagging_ = false;
    used_.clear();
  }
}

// multi_val_bin.rs:644-648 (per row, per column: out[bin] += [g, h]);
// `rows == nullptr` walks every row.
void SerialTreeLearner::build_hist_block(const uint32_t* rows, size_t k0, size_t k1, const float* grad,
                                         const float* hess, double* out) const {
  int32_t nf = d_->num_features;
  for (size_t k = k0; k < k1; ++k) {
    size_t r = rows ? rows[k] : k;
    double g = (double)grad[r], h = (double)hess[r];
    const uint8_t* row = d_->bins + r * (size_t)nf;
    for (int32_t f = 0; f < nf; ++f) {
      uint32_t raw = row[f];
      if (raw == 0) continue;  // most frequent bin: group slot 0, outside every feature view
      size_t t = view_start_[f] + raw - 1;
      out[2 * t] += g;
      out[2 * t + 1] += h;
    }
  }
}

// multi_val_bin.rs:556-611 construct: rows split into Threading::BlockInfo
// blocks (min block size from multi_val_bin.rs:348-351), each summed in row
// order, blocks added in block order (HistMerge) — equal to the reference
// at the same thread count.
void SerialTreeLearner::build_hist(const uint32_t* rows, size_t n, const float* grad, const float* hess,
                                   double* out) const {
  std::fill(out, out + 2 * total_bins_, 0.0);
  size_t threads = (size_t)std::max(cfg_.num_threads, 1);
  size_t nblock = 1, bsize = n;
  if (threads > 1) {
    size_t mv_bins = total_bins_ + (size_t)d_->num_features;  // + each group's slot 0
    int32_t mbs = (int32_t)((double)(0.3f * (float)mv_bins) / ((double)d_->num_features + kZeroThreshold));
    size_t min_block = (size_t)std::min(std::max(mbs + 1, 32), 1024);
    block_info(threads, n, min_block, &nblock, &bsize);
  }
  if (nblock == 1) {
    build_hist_block(rows, 0, n, grad, hess, out);
    return;
  }
  std::vector<std::vector<double>> bufs(nblock - 1, std::vector<double>(2 * total_bins_, 0.0));
#pragma omp parallel for schedule(static, 1) num_threads((int)threads)
  for (long b = 0; b < (long)nblock; ++b) {
    size_t s = std::min((size_t)b * bsize, n), e = std::min(s + bsize, n);
    build_hist_block(rows, s, e, grad, hess, b == 0 ? out : bufs[(size_t)b - 1].data());
  }
  for (auto& src : bufs)
    for (size_t i = 0; i < 2 * total_bins_; ++i) out[i] += src[i];
}

// multi_val_bin.rs:763-791 construct_int (wrapping packed sums).
void SerialTreeLearner::build_hist_int(const uint32_t* rows, size_t n, const int64_t* packed, int64_t* out) const {
  std::fill(out, out + total_bins_, 0);
  int32_t nf = d_->num_features;
  int threads = std::max(cfg_.num_threads, 1);
  if (threads > 1 && n > 4096) {  // integer sums: any block split gives the same result
    std::vector<std::vector<int64_t>> bufs((size_t)threads, std::vector<int64_t>(total_bins_, 0));
#pragma omp parallel num_threads(threads)
    {
      int t = omp_get_thread_num();
      size_t s = n * (size_t)t / (size_t)threads, e = n * (size_t)(t + 1) / (size_t)threads;
      int64_t* o = bufs[(size_t)t].data();
      for (size_t k = s; k < e; ++k) {
        size_t r = rows ? rows[k] : k;
        uint64_t v = (uint64_t)packed[r];
        const uint8_t* row = d_->bins + r * (size_t)nf;
        for (int32_t f = 0; f < nf; ++f) {
          uint32_t raw = row[f];
          if (raw == 0) continue;
          size_t ti = view_start_[f] + raw - 1;
          o[ti] = (int64_t)((uint64_t)o[ti] + v);
        }
      }
    }
    for (auto& b : bufs)
      for (size_t i = 0; i < total_bins_; ++i) out[i] = (int64_t)((uint64_t)out[i] + (uint64_t)b[i]);
    return;
  }
  for (size_t k = 0; k < n; ++k) {
    size_t r = rows ? rows[k] : k;
    uint64_t v = (uint64_t)packed[r];
    const uint8_t* row = d_->bins + r * (size_t)nf;
    for (int32_t f = 0; f < nf; ++f) {
      uint32_t raw = row[f];
      if (raw == 0) continue;
      size_t t = view_start_[f] + raw - 1;
      out[t] = (int64_t)((uint64_t)out[t] + v);
    }
  }
}

// partition.rs:235-262 (sequential branch): stable split by lut[bin(row)].
size_t SerialTreeLearner::partition_split(int32_t leaf, int32_t inner, const std::vector<bool>& lut,
                                          int32_t right_leaf) {
  size_t begin = leaf_begin_[leaf], cnt = leaf_count_[leaf];
  const FeatureMeta& m = d_->metas[inner];
  std::vector<uint32_t> left, right;
  left.reserve(cnt);
  right.reserve(cnt);
  int32_t nf = d_->num_features;
  for (size_t k = begin; k < begin + cnt; ++k) {
    uint32_t r = indices_[k];
    uint32_t raw = d_->bins[(size_t)r * nf + inner];
    uint32_t b = raw == 0 ? m.most_freq_bin : raw - 1 + (uint32_t)(m.most_freq_bin == 0);
    if (lut[b]) left.push_back(r);
    else right.push_back(r);
  }
  std::copy(left.begin(), left.end(), indices_.begin() + begin);
  std::copy(right.begin(), right.end(), indices_.begin() + begin + left.size());
  leaf_count_[leaf] = left.size();
  leaf_begin_[right_leaf] = begin + left.size();
  leaf_count_[right_leaf] = cnt - left.size();
  part_num_leaves_ += 1;
  return left.size();
}

// partition.rs:306-319
void SerialTreeLearner::add_leaf_outputs(const std::vector<double>& leaf_values, double* score) const {
  int32_t leaves = std::min<int32_t>(part_num_leaves_, (int32_t)leaf_values.size());
  for (int32_t l = 0; l < leaves; ++l)
    for (size_t k = leaf_begin_[l]; k < leaf_begin_[l] + leaf_count_[l]; ++k) score[indices_[k]] += leaf_values[l];
}

int32_t SerialTreeLearner::best_leaf() const {  // learner/mod.rs:698-706
  int32_t best = 0;
  for (size_t i = 1; i < best_split_per_leaf_.size(); ++i)
    if (best_split_per_leaf_[i].better_than(best_split_per_leaf_[best])) best = (int32_t)i;
  return best;
}

bool SerialTreeLearner::before_find_best_split(const Tree& tree, int32_t left, int32_t right) {  // :712-731
  if (cfg_.max_depth > 0 && tree.leaf_depth[left] >= cfg_.max_depth) {
    best_split_per_leaf_[left].gain = kMinScore;
    if (right >= 0) best_split_per_leaf_[right].gain = kMinScore;
    return false;
  }
  int32_t nl = left >= 0 ? (int32_t)leaf_count_[left] : 0;
  int32_t nr = right >= 0 ? (int32_t)leaf_count_[right] : 0;
  int32_t min2 = cfg_.params.min_data_in_leaf * 2;
  if (nr < min2 && nl < min2) {
    best_split_per_leaf_[left].gain = kMinScore;
    if (right >= 0) best_split_per_leaf_[right].gain = kMinScore;
    return false;
  }
  return true;
}

// learner/mod.rs:816-1103 find_best_splits (row-wise, no forced features).
void SerialTreeLearner::find_best_splits(const Tree& tree, const float* grad, const float* hess, int32_t left,
                                         int32_t right) {
  int32_t nf = d_->num_features;
  const SplitParams& p = cfg_.params;
  bool have_parent = right >= 0;
  // HistogramPool::Move: the parent's buffer (slot `left`) goes to the larger
  // leaf, the right slot's buffer to the smaller one.
  std::vector<double> parent_buf, s_buf;
  std::vector<int64_t> parent_ibuf, s_ibuf;
  std::vector<bool> parent_spl, s_spl_init;
  if (have_parent) {
    parent_buf = std::move(hist_[left]);
    parent_ibuf = std::move(ihist_[left]);
    parent_spl = splittable_[left];
    s_buf = std::move(hist_[right]);
    s_ibuf = std::move(ihist_[right]);
    s_spl_init = splittable_[right];
  } else {
    s_buf = std::move(hist_[0]);
    s_ibuf = std::move(ihist_[0]);
    s_spl_init = splittable_[0];
  }
  if (cfg_.quantized) s_ibuf.resize(total_bins_, 0);
  else s_buf.resize(2 * total_bins_, 0.0);
  std::vector<bool> is_used(nf);
  for (int32_t f = 0; f < nf; ++f) is_used[f] = have_parent ? (parent_spl[f] && bytree_[f]) : (bool)bytree_[f];
  for (int32_t f = 0; f < nf; ++f)
    if (bytree_[f] && !is_used[f]) s_spl_init[f] = false;
  std::vector<bool> l_spl = have_parent ? parent_spl : std::vector<bool>();

  int32_t sm_leaf = smaller_.leaf;
  bool use_indices = right >= 0 || leaf_count_[sm_leaf] != (size_t)d_->num_data;
  const uint32_t* rows = use_indices ? indices_.data() + leaf_begin_[sm_leaf] : nullptr;
  size_t nrows = use_indices ? leaf_count_[sm_leaf] : (size_t)d_->num_data;
  if (cfg_.quantized) build_hist_int(rows, nrows, quant_->packed.data(), s_ibuf.data());
  else build_hist(rows, nrows, grad, hess, s_buf.data());

  auto parent_output = [&](const LeafSplits& ls) {  // learner/mod.rs:1303-1309
    return tree.num_leaves == 1 ? root_output(ls.sum_gradients, ls.sum_hessians, p, ls.num_data) : ls.weight;
  };
  double s_parent_out = parent_output(smaller_);
  double l_parent_out = larger_.leaf >= 0 ? parent_output(larger_) : 0.0;
  auto penalty = [&](int32_t leaf) {
    return leaf >= 0 ? monotone_split_gain_penalty(tree.leaf_depth[leaf], cfg_.monotone_penalty) : 0.0;
  };
  double s_pen = penalty(smaller_.leaf), l_pen = penalty(larger_.leaf);
  const BasicConstraint* s_mc = cfg_.use_monotone ? &constraints_[smaller_.leaf] : nullptr;
  const BasicConstraint* l_mc = (cfg_.use_monotone && larger_.leaf >= 0) ? &constraints_[larger_.leaf] : nullptr;
  double gscale = quant_ ? quant_->grad_scale : 0.0, hscale = quant_ ? quant_->hess_scale : 0.0;

  SplitInfo s_best, l_best;
  std::vector<bool> s_spl = s_spl_init;
  // per-feature searches are independent (learner/mod.rs:954-1057); the
  // reduction below walks the features in order
  std::vector<SplitInfo> s_res(nf), l_res(nf);
  std::vector<char> s_okv(nf, 0), l_okv(nf, 0);
#pragma omp parallel for schedule(dynamic) num_threads(std::max(cfg_.num_threads, 1))
  for (int32_t f = 0; f < nf; ++f) {
    if (!is_used[f]) continue;
    const FeatureMeta& meta = d_->metas[f];
    SplitInfo& s_split = s_res[f];
    SplitInfo& l_split = l_res[f];
    bool s_ok, l_ok = false;
    if (cfg_.quantized) {
      int64_t* hist = s_ibuf.data() + view_start_[f];
      fix_hist_int(meta, smaller_.int_sum, hist);
      s_ok = find_best_threshold_int(hist, meta, p, smaller_.int_sum, gscale, hscale, smaller_.num_data, s_parent_out,
                                     s_mc, s_split);
      if (larger_.leaf >= 0) {
        int64_t* lh = parent_ibuf.data() + view_start_[f];
        for (int32_t t = 0; t < meta.num_bin - meta.offset; ++t) lh[t] = (int64_t)((uint64_t)lh[t] - (uint64_t)hist[t]);
        l_ok = find_best_threshold_int(lh, meta, p, larger_.int_sum, gscale, hscale, larger_.num_data, l_parent_out,
                                       l_mc, l_split);
      }
    } else {
      double* hist = s_buf.data() + 2 * view_start_[f];
      fix_hist(meta, smaller_.sum_gradients, smaller_.sum_hessians, hist);
      s_ok = find_best_threshold(hist, meta, p, smaller_.sum_gradients, smaller_.sum_hessians, smaller_.num_data,
                                 s_parent_out, s_mc, s_split);
      if (larger_.leaf >= 0) {
        double* lh = parent_buf.data() + 2 * view_start_[f];
        for (int32_t t = 0; t < 2 * (meta.num_bin - meta.offset); ++t) lh[t] -= hist[t];
        l_ok = find_best_threshold(lh, meta, p, larger_.sum_gradients, larger_.sum_hessians, larger_.num_data,
                                   l_parent_out, l_mc, l_split);
      }
    }
    s_split.feature = meta.real_index;
    s_split.feature_inner = f;
    l_split.feature = meta.real_index;
    l_split.feature_inner = f;
    s_okv[f] = s_ok;
    l_okv[f] = l_ok;
  }
  for (int32_t f = 0; f < nf; ++f) {
    if (!is_used[f]) continue;
    SplitInfo& s_split = s_res[f];
    SplitInfo& l_split = l_res[f];
    // finish_split (learner/mod.rs:1283-1300): the monotone depth penalty.
    if (s_split.monotone_type != 0) s_split.gain *= s_pen;
    if (s_split.better_than(s_best)) s_best = s_split;
    s_spl[f] = s_okv[f] != 0;
    if (larger_.leaf >= 0) {
      if (l_split.monotone_type != 0) l_split.gain *= l_pen;
      if (l_split.better_than(l_best)) l_best = l_split;
      l_spl[f] = l_okv[f] != 0;
    }
  }
  best_split_per_leaf_[sm_leaf] = s_best;
  hist_[sm_leaf] = std::move(s_buf);
  ihist_[sm_leaf] = std::move(s_ibuf);
  splittable_[sm_leaf] = s_spl;
  if (larger_.leaf >= 0) {
    int32_t lg = larger_.leaf;
    best_split_per_leaf_[lg] = l_best;
    hist_[lg] = std::move(parent_buf);
    ihist_[lg] = std::move(parent_ibuf);
    splittable_[lg] = l_spl;
  }
}

// learner/mod.rs:1313-1317 / :1323-1329
static bool goes_left(uint32_t b, const FeatureMeta& m, uint32_t threshold, bool default_left) {
  bool is_missing = (m.missing_type == kMissingZero && b == m.default_bin) ||
                    (m.missing_type == kMissingNaN && b == (uint32_t)(m.num_bin - 1));
  return is_missing ? default_left : b <= threshold;
}
static bool goes_left_categorical(uint32_t b, const FeatureMeta& m, const std::vector<uint32_t>& bits) {
  if (b == m.most_freq_bin)
    return m.most_freq_bin > 0 && find_in_bitset(bits.data(), bits.size(), (int32_t)m.most_freq_bin);
  return find_in_bitset(bits.data(), bits.size(), (int32_t)b);
}

// learner/mod.rs:1105-1225 split.
std::pair<int32_t, int32_t> SerialTreeLearner::split(Tree& tree, int32_t best_leaf) {
  SplitInfo info = best_split_per_leaf_[best_leaf];
  int32_t inner = info.feature_inner;
  const FeatureMeta& meta = d_->metas[inner];
  int32_t next_leaf = tree.num_leaves;
  uint32_t num_bin = (uint32_t)std::max(meta.num_bin, 1);
  bool numerical = meta.bin_type == kNumerical;
  std::vector<bool> lut(num_bin);
  std::vector<uint32_t> bits_inner, bits;
  if (numerical) {
    for (uint32_t b = 0; b < num_bin; ++b) lut[b] = goes_left(b, meta, info.threshold, info.default_left);
  } else {
    std::vector<int32_t> ci, cv;
    for (uint32_t c : info.cat_threshold) {
      ci.push_back((int32_t)c);
      cv.push_back(d_->bin_to_cat[inner][c]);
    }
    bits_inner = construct_bitset(ci);
    bits = construct_bitset(cv);
    for (uint32_t b = 0; b < num_bin; ++b) lut[b] = goes_left_categorical(b, meta, bits_inner);
  }
  partition_split(best_leaf, inner, lut, next_leaf);
  info.left_count = (int32_t)leaf_count_[best_leaf];
  info.right_count = (int32_t)leaf_count_[next_leaf];
  SplitArgs a;
  a.leaf = best_leaf;
  a.feature_inner = inner;
  a.feature_real = info.feature;
  a.threshold_bin = info.threshold;
  a.threshold = numerical ? d_->upper_bounds[inner][info.threshold] : 0.0;
  a.left_value = info.left_output;
  a.right_value = info.right_output;
  a.left_count = info.left_count;
  a.right_count = info.right_count;
  a.left_weight = info.left_sum_hessian;
  a.right_weight = info.right_sum_hessian;
  a.gain = (float)(info.gain + cfg_.params.min_gain_to_split);
  a.missing_type = meta.missing_type;
  a.default_left = info.default_left;
  int32_t right = numerical ? tree_split(tree, a) : tree_split_categorical(tree, a, bits_inner, bits);
  trace.push_back({best_leaf, info.feature, info.threshold, info.gain});
  LeafSplits ls{best_leaf, info.left_count, info.left_sum_gradient, info.left_sum_hessian, info.left_sum_gh,
                info.left_output};
  LeafSplits rs{right, info.right_count, info.right_sum_gradient, info.right_sum_hessian, info.right_sum_gh,
                info.right_output};
  if (info.left_count < info.right_count) {
    if (info.left_count <= 0) throw std::runtime_error("Check failed: (best_split_info.left_count) > (0)");
    smaller_ = ls;
    larger_ = rs;
  } else {
    if (info.right_count <= 0) throw std::runtime_error("Check failed: (best_split_info.right_count) > (0)");
    smaller_ = rs;
    larger_ = ls;
  }
  if (cfg_.use_monotone) {  // constraints.rs:467-480 (basic method)
    constraints_[right] = constraints_[best_leaf];
    if (numerical) {
      double mid = (info.left_output + info.right_output) / 2.0;
      auto upd_min = [](BasicConstraint& c, double v) { c.min = v < c.min ? c.min : v; };
      auto upd_max = [](BasicConstraint& c, double v) { c.max = c.max < v ? c.max : v; };
      if (info.monotone_type < 0) {
        upd_min(constraints_[best_leaf], mid);
        upd_max(constraints_[right], mid);
      } else if (info.monotone_type > 0) {
        upd_max(constraints_[best_leaf], mid);
        upd_min(constraints_[right], mid);
      }
    }
  }
  return {best_leaf, right};
}

// learner/mod.rs:572-695 train (no forced splits, no linear trees).
Tree SerialTreeLearner::train(const float* grad, const float* hess) {
  size_t n = (size_t)d_->num_data;
  if (cfg_.quantized) quant_->discretize(grad, hess, n, nullptr, 0);
  // DataPartition::init (partition.rs:202-218)
  std::fill(leaf_begin_.begin(), leaf_begin_.end(), 0);
  std::fill(leaf_count_.begin(), leaf_count_.end(), 0);
  if (bagging_) {
    std::copy(used_.begin(), used_.end(), indices_.begin());
    leaf_count_[0] = used_.size();
  } else {
    for (size_t i = 0; i < n; ++i) indices_[i] = (uint32_t)i;
    leaf_count_[0] = n;
  }
  part_num_leaves_ = 1;
  for (auto& c : constraints_) c = BasicConstraint();
  for (auto& s : best_split_per_leaf_) s.reset();
  trace.clear();
  size_t root_cnt = leaf_count_[0];
  double sg = 0.0, sh = 0.0;
  int64_t int_sum = 0;
  if (cfg_.quantized) {
    if (root_cnt == n) {
      quant_->root_sums(indices_.data(), root_cnt, &sg, &sh, &int_sum);
    } else {  // quant.rs:467-477 bag_root_sums: f32 scales, packed sum by position
      float gs = (float)quant_->grad_scale, hs = (float)quant_->hess_scale;
      uint64_t si = 0;
      for (size_t i = 0; i < root_cnt; ++i) {
        auto& r = quant_->raw[indices_[i]];
        sg += (double)((float)r[1] * gs);
        sh += (double)((float)r[0] * hs);
        si += (uint64_t)quant_->packed[i];
      }
      int_sum = (int64_t)si;
    }
  } else if (root_cnt == n) {
    for (size_t i = 0; i < n; ++i) {
      sg += (double)grad[i];
      sh += (double)hess[i];
    }
  } else {
    for (size_t k = 0; k < root_cnt; ++k) {
      sg += (double)grad[indices_[k]];
      sh += (double)hess[indices_[k]];
    }
  }
  smaller_ = LeafSplits{0, (int32_t)root_cnt, sg, sh, int_sum, 0.0};
  larger_ = LeafSplits{};
  Tree tree;
  tree_set_leaf_output(tree, 0, root_output(sg, sh, cfg_.params, (int32_t)root_cnt));
  int32_t left = 0, right = -1;
  for (int32_t it = 0; it < cfg_.num_leaves - 1; ++it) {
    if (before_find_best_split(tree, left, right)) find_best_splits(tree, grad, hess, left, right);
    int32_t bl = best_leaf();
    double gain = best_split_per_leaf_[bl].gain;
    if (!(gain > 0.0)) break;
    auto lr = split(tree, bl);
    left = lr.first;
    right = lr.second;
  }
  if (cfg_.quantized && cfg_.quant_renew) {  // learner/mod.rs:736-747
    for (int32_t leaf = 0; leaf < tree.num_leaves; ++leaf) {
      double a = 0.0, b = 0.0;
      for (size_t k = leaf_begin_[leaf]; k < leaf_begin_[leaf] + leaf_count_[leaf]; ++k) {
        a += (double)grad[indices_[k]];
        b += (double)hess[indices_[k]];
      }
      tree_set_leaf_output(tree, leaf, refit_leaf_output(a, b, cfg_.params, false, (int32_t)leaf_count_[leaf], 0.0));
    }
  }
  return tree;
}

}  // namespace oracle
