// Oracle: objectives (objective/{binary,regression,multiclass,rank}.rs,
// dcg.rs), the boosting loop (boosting.rs train_one_iter / update_score),
// bagging (sample_strategy.rs), the by-tree column sampler
// (learner/col_sampler.rs), raw-value prediction (predict.rs) and metrics
// (metric.rs), plus the C ABI the tests load with ctypes.
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>

#include "oracle_abi.h"
#include "oracle_impl.h"

namespace oracle {

// ---- objectives ----------------------------------------------------------------------
// objective/binary.rs:101-127 (no weights, is_unbalance off, scale_pos_weight 1).
static void grad_binary(const float* label, const double* s, size_t n, double sigmoid, float* g, float* h) {
  for (size_t i = 0; i < n; ++i) {
    double lab = label[i] > 0.0f ? 1.0 : -1.0;
    double response = -lab * sigmoid / ((double)1.0f + std::exp(lab * sigmoid * s[i]));
    double ar = std::fabs(response);
    g[i] = (float)(response * 1.0);
    h[i] = (float)(ar * (sigmoid - ar) * 1.0);
  }
}
// objective/binary.rs:129-154
static double boost_binary(const float* label, size_t n, double sigmoid) {
  double suml = 0.0;
  for (size_t i = 0; i < n; ++i) suml += (double)(int32_t)(label[i] > 0.0f);
  double pavg = suml / (double)n;
  pavg = std::min(pavg, 1.0 - kEpsilon);
  pavg = std::max(pavg, kEpsilon);
  return std::log(pavg / ((double)1.0f - pavg)) / sigmoid;
}
// objective/regression.rs:223 (L2, no weights)
static void grad_l2(const float* label, const double* s, size_t n, float* g, float* h) {
  for (size_t i = 0; i < n; ++i) {
    g[i] = (float)(s[i] - (double)label[i]);
    h[i] = 1.0f;
  }
}
static double boost_l2(const float* label, size_t n) {  // regression.rs:123-139
  double suml = 0.0;
  for (size_t i = 0; i < n; ++i) suml += (double)label[i];
  return suml / (double)n;
}
// objective/multiclass.rs:16-30
static void softmax(const double* in, double* out, int k) {
  double wmax = in[0];
  for (int c = 1; c < k; ++c) wmax = in[c] < wmax ? wmax : in[c];
  double wsum = 0.0;
  for (int c = 0; c < k; ++c) {
    out[c] = std::exp(in[c] - wmax);
    wsum += out[c];
  }
  for (int c = 0; c < k; ++c) out[c] /= wsum;
}
// objective/multiclass.rs:126-154
static void grad_softmax(const float* label, const double* s, size_t n, int k, float* g, float* h) {
  double factor = (double)k / (double)((float)k - 1.0f);
  std::vector<double> raw(k), rec(k);
  for (size_t i = 0; i < n; ++i) {
    for (int c = 0; c < k; ++c) raw[c] = s[(size_t)c * n + i];
    softmax(raw.data(), rec.data(), k);
    int32_t li = (int32_t)label[i];
    for (int c = 0; c < k; ++c) {
      double p = rec[c];
      double gg = li == c ? p - (double)1.0f : p;
      double hh = factor * p * ((double)1.0f - p);
      g[(size_t)c * n + i] = (float)gg;
      h[(size_t)c * n + i] = (float)hh;
    }
  }
}

// dcg.rs:27-34, 44-48, 66-84
struct Dcg {
  std::vector<double> label_gain, discount;
  Dcg() {
    label_gain.push_back(0.0);
    for (int i = 1; i < 31; ++i) label_gain.push_back((double)((1 << i) - 1));
    for (int i = 0; i < 10000; ++i) discount.push_back(1.0 / std::log2(2.0 + (double)i));
  }
  double max_dcg_at_k(size_t k, const float* label, size_t n) const {
    std::vector<int32_t> cnt(label_gain.size(), 0);
    for (size_t i = 0; i < n; ++i) cnt[(int32_t)label[i]] += 1;
    int32_t top = (int32_t)label_gain.size() - 1;
    double ret = 0.0;
    for (size_t j = 0; j < std::min(k, n); ++j) {
      while (top > 0 && cnt[top] <= 0) top -= 1;
      if (top < 0) break;
      ret += discount[j] * label_gain[top];
      cnt[top] -= 1;
    }
    return ret;
  }
};
// dcg.rs:167-179 (stable sort, descending score)
static std::vector<size_t> sort_by_score_desc(const double* score, size_t n) {
  std::vector<size_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return score[a] > score[b]; });
  return idx;
}

// objective/rank.rs:119-262 LambdarankNDCG (no weights / positions).
struct Lambdarank {
  double sigmoid;
  bool norm;
  int32_t truncation_level;
  Dcg dcg;
  std::vector<double> inverse_max_dcgs, sigmoid_table;
  double min_in = -50.0, max_in = 50.0, idx_factor = 0.0;
  static constexpr size_t kBins = 1024 * 1024;
  Lambdarank(double sig, bool nrm, int32_t trunc, const float* label, const int32_t* bnd, size_t nq)
      : sigmoid(sig), norm(nrm), truncation_level(trunc) {
    size_t k = (size_t)std::max(trunc, 0);
    for (size_t q = 0; q < nq; ++q) {
      double v = dcg.max_dcg_at_k(k, label + bnd[q], (size_t)(bnd[q + 1] - bnd[q]));
      inverse_max_dcgs.push_back(v > 0.0 ? 1.0 / v : v);
    }
    min_in = min_in / sigmoid / 2.0;  // rank.rs:162-176
    max_in = -min_in;
    idx_factor = (double)kBins / (max_in - min_in);
    sigmoid_table.resize(kBins);
    for (size_t i = 0; i < kBins; ++i) {
      double score = (double)i / idx_factor + min_in;
      sigmoid_table[i] = 1.0 / (1.0 + std::exp(score * sigmoid));
    }
  }
  double get_sigmoid(double score) const {
    if (score <= min_in) return sigmoid_table[0];
    if (score >= max_in) return sigmoid_table[kBins - 1];
    return sigmoid_table[(size_t)((score - min_in) * idx_factor)];
  }
  void one_query(size_t q, const float* label, const double* score, size_t cnt, float* lambdas, float* hessians) const {
    double inverse_max_dcg = inverse_max_dcgs[q];
    std::fill(lambdas, lambdas + cnt, 0.0f);
    std::fill(hessians, hessians + cnt, 0.0f);
    if (cnt == 0) return;
    auto sorted = sort_by_score_desc(score, cnt);
    double best_score = score[sorted[0]];
    size_t worst_idx = cnt - 1;
    if (worst_idx > 0 && score[sorted[worst_idx]] == kMinScore) worst_idx -= 1;
    double worst_score = score[sorted[worst_idx]];
    double sum_lambdas = 0.0;
    for (size_t i = 0; i + 1 < cnt && (int64_t)i < (int64_t)truncation_level; ++i) {
      if (score[sorted[i]] == kMinScore) continue;
      for (size_t j = i + 1; j < cnt; ++j) {
        if (score[sorted[j]] == kMinScore) continue;
        if (label[sorted[i]] == label[sorted[j]]) continue;
        size_t high_rank = i, low_rank = j;
        if (!(label[sorted[i]] > label[sorted[j]])) {
          high_rank = j;
          low_rank = i;
        }
        size_t high = sorted[high_rank], low = sorted[low_rank];
        double high_score = score[high], low_score = score[low];
        double high_label_gain = dcg.label_gain[(int32_t)label[high]];
        double low_label_gain = dcg.label_gain[(int32_t)label[low]];
        double high_discount = dcg.discount[high_rank], low_discount = dcg.discount[low_rank];
        double delta_score = high_score - low_score;
        double dcg_gap = high_label_gain - low_label_gain;
        double paired_discount = std::fabs(high_discount - low_discount);
        double delta_pair_ndcg = dcg_gap * paired_discount * inverse_max_dcg;
        if (norm && best_score != worst_score) delta_pair_ndcg /= (double)0.01f + std::fabs(delta_score);
        double p_lambda = get_sigmoid(delta_score);
        double p_hessian = p_lambda * (1.0 - p_lambda);
        p_lambda *= -sigmoid * delta_pair_ndcg;
        p_hessian *= sigmoid * sigmoid * delta_pair_ndcg;
        lambdas[low] -= (float)p_lambda;
        hessians[low] += (float)p_hessian;
        lambdas[high] += (float)p_lambda;
        hessians[high] += (float)p_hessian;
        sum_lambdas -= 2.0 * p_lambda;
      }
    }
    if (norm && sum_lambdas > 0.0) {
      double norm_factor = std::log2(1.0 + sum_lambdas) / sum_lambdas;
      for (size_t i = 0; i < cnt; ++i) {
        lambdas[i] = (float)((double)lambdas[i] * norm_factor);
        hessians[i] = (float)((double)hessians[i] * norm_factor);
      }
    }
  }
};

// ---- metrics ---------------------------------------------------------------------------
// metric.rs:701-731 AUC (no weights).
double auc(const float* label, const double* score, size_t n) {
  auto idx = sort_by_score_desc(score, n);
  double cur_pos = 0, sum_pos = 0, accum = 0, cur_neg = 0;
  double threshold = score[idx[0]];
  for (size_t i : idx) {
    float lbl = label[i];
    double s = score[i];
    if (s != threshold) {
      threshold = s;
      accum += cur_neg * (cur_pos * 0.5 + sum_pos);
      sum_pos += cur_pos;
      cur_neg = 0;
      cur_pos = 0;
    }
    cur_neg += (double)(int32_t)(lbl <= 0.0f);
    cur_pos += (double)(int32_t)(lbl > 0.0f);
  }
  accum += cur_neg * (cur_pos * 0.5 + sum_pos);
  sum_pos += cur_pos;
  double sw = (double)n;
  return (sum_pos > 0.0 && sum_pos != sw) ? accum / (sum_pos * (sw - sum_pos)) : 1.0;
}

// ---- boosting loop -------------------------------------------------------------------
struct Booster {
  OracleParams p;
  BinnedData data;
  BinnedData valid;
  std::vector<float> label, valid_label;
  std::vector<int32_t> bnd;
  int ntpi = 1;
  std::vector<double> scores, valid_scores;
  std::vector<float> grad, hess;
  std::vector<Tree> models;
  std::vector<bool> class_need_train;
  std::unique_ptr<SerialTreeLearner> learner;
  std::unique_ptr<Lambdarank> rank;
  // bagging (sample_strategy.rs:280-320)
  std::vector<Random> rands;
  std::vector<uint32_t> bag_indices;
  size_t bag_cnt = 0;
  bool need_re_bagging = true;
  // column sampler (col_sampler.rs)
  Random col_rand{0};
  int32_t used_cnt_bytree = 0;
  int iter = 0;
  std::vector<std::vector<TreeTraceEntry>> traces;
  std::string model_text;
};

static void add_const(std::vector<double>& s, int k, size_t n, double v) {
  for (size_t i = 0; i < n; ++i) s[(size_t)k * n + i] += v;
}

static void gradients(Booster& b) {
  size_t n = (size_t)b.data.num_data;
  switch (b.p.objective) {
    case 0: grad_binary(b.label.data(), b.scores.data(), n, b.p.sigmoid, b.grad.data(), b.hess.data()); break;
    case 1: grad_l2(b.label.data(), b.scores.data(), n, b.grad.data(), b.hess.data()); break;
    case 2: grad_softmax(b.label.data(), b.scores.data(), n, b.ntpi, b.grad.data(), b.hess.data()); break;
    case 3:
      for (size_t q = 0; q + 1 < b.bnd.size(); ++q) {
        size_t s = (size_t)b.bnd[q], c = (size_t)(b.bnd[q + 1] - b.bnd[q]);
        b.rank->one_query(q, b.label.data() + s, b.scores.data() + s, c, b.grad.data() + s, b.hess.data() + s);
      }
      break;
  }
}

static double boost_from_score(Booster& b, int k) {
  size_t n = (size_t)b.data.num_data;
  switch (b.p.objective) {
    case 0: return boost_binary(b.label.data(), n, b.p.sigmoid);
    case 1: return boost_l2(b.label.data(), n);
    case 2: {
      double c = 0.0;
      for (size_t i = 0; i < n; ++i) c += (int32_t)b.label[i] == k ? 1.0 : 0.0;
      return std::log(std::max(kEpsilon, c / (double)n));
    }
    default: return 0.0;
  }
}

// col_sampler.rs:27-31 get_cnt and :88-96 reset_by_tree.
static std::vector<bool> reset_by_tree(Booster& b) {
  int32_t nf = b.data.num_features;
  std::vector<bool> used(nf, true);
  if (b.p.feature_fraction < 1.0) {
    std::fill(used.begin(), used.end(), false);
    for (int32_t i : b.col_rand.sample(nf, b.used_cnt_bytree)) used[i] = true;
  }
  return used;
}

static void tree_to_scores(const Tree& t, const BinnedData& d, std::vector<double>& s, size_t off,
                           const uint32_t* rows, size_t nrows) {
  if (rows) {
    for (size_t k = 0; k < nrows; ++k) s[off + rows[k]] += t.leaf_value[tree_leaf_binned(t, d, rows[k])];
  } else {
    for (int64_t i = 0; i < d.num_data; ++i) s[off + (size_t)i] += t.leaf_value[tree_leaf_binned(t, d, i)];
  }
}

// boosting.rs:957-1130 train_one_iter; returns true when training stops.
static bool train_one_iter(Booster& b) {
  size_t n = (size_t)b.data.num_data;
  int ntpi = b.ntpi;
  std::vector<double> init_scores(ntpi, 0.0);
  for (int k = 0; k < ntpi; ++k) {  // boosting.rs:480-509 boost_from_average
    if (b.models.empty() && b.p.boost_from_average) {
      double init = boost_from_score(b, k);
      if (std::fabs(init) > kEpsilon) {
        add_const(b.scores, k, n, init);
        if (b.valid.num_data) add_const(b.valid_scores, k, (size_t)b.valid.num_data, init);
        init_scores[k] = init;
      }
    }
  }
  gradients(b);
  bool bagging = b.p.bagging_fraction < 1.0 && b.p.bagging_freq > 0;
  if (bagging && ((b.bag_cnt < n && b.iter % b.p.bagging_freq == 0) || b.need_re_bagging)) {
    b.need_re_bagging = false;
    size_t left = 0, right = n;
    for (size_t i = 0; i < n; ++i) {
      double r = (double)b.rands[i / 1024].next_float();
      if (r < b.p.bagging_fraction) b.bag_indices[left++] = (uint32_t)i;
      else b.bag_indices[--right] = (uint32_t)i;
    }
    b.bag_cnt = left;
    b.learner->set_bagging_data(b.bag_indices.data(), b.bag_cnt);
  }
  bool should_continue = false;
  for (int k = 0; k < ntpi; ++k) {
    size_t off = (size_t)k * n;
    Tree tree;
    bool need_train = b.class_need_train[k] && b.data.num_features > 0;
    if (need_train) {
      b.learner->set_bytree_mask(reset_by_tree(b));
      tree = b.learner->train(b.grad.data() + off, b.hess.data() + off);
      b.traces.push_back(b.learner->trace);
    }
    if (tree.num_leaves > 1) {
      should_continue = true;
      tree_shrink(tree, b.p.learning_rate);
      // boosting.rs:1381-1408 update_score
      b.learner->add_leaf_outputs(tree.leaf_value, b.scores.data() + off);
      if (bagging) tree_to_scores(tree, b.data, b.scores, off, b.bag_indices.data() + b.bag_cnt, n - b.bag_cnt);
      if (b.valid.num_data) tree_to_scores(tree, b.valid, b.valid_scores, (size_t)k * b.valid.num_data, nullptr, 0);
      if (std::fabs(init_scores[k]) > kEpsilon) tree_add_bias(tree, init_scores[k]);
    } else if ((int)b.models.size() < ntpi) {
      tree_as_constant(tree, init_scores[k], (int32_t)n);
    } else {
      tree_as_constant(tree, 0.0, (int32_t)n);
    }
    b.models.push_back(tree);
  }
  if (!should_continue) {
    if ((int)b.models.size() > ntpi)
      for (int k = 0; k < ntpi; ++k) b.models.pop_back();
    return true;
  }
  b.iter += 1;
  return false;
}

static BinnedData make_binned(const OracleData& d) {
  BinnedData b;
  b.num_data = d.num_data;
  b.num_features = d.num_features;
  b.bins = d.bins;
  for (int32_t f = 0; f < d.num_features; ++f) {
    FeatureMeta m;
    m.num_bin = d.num_bin[f];
    m.missing_type = d.missing_type[f];
    m.most_freq_bin = (uint32_t)d.most_freq_bin[f];
    m.default_bin = (uint32_t)d.default_bin[f];
    m.offset = m.most_freq_bin == 0 ? 1 : 0;
    m.bin_type = d.bin_type[f];
    m.monotone_type = d.monotone ? d.monotone[f] : 0;
    m.penalty = 1.0;
    m.real_index = d.real_index[f];
    b.metas.push_back(m);
    if (d.upper_bounds) b.upper_bounds.emplace_back(d.upper_bounds + d.ub_offsets[f], d.upper_bounds + d.ub_offsets[f + 1]);
    else b.upper_bounds.emplace_back();
    if (d.bin_to_cat) b.bin_to_cat.emplace_back(d.bin_to_cat + d.cat_offsets[f], d.bin_to_cat + d.cat_offsets[f + 1]);
    else b.bin_to_cat.emplace_back();
  }
  return b;
}

static SplitParams split_params(const OracleParams& p) {
  SplitParams s;
  s.lambda_l1 = p.lambda_l1;
  s.lambda_l2 = p.lambda_l2;
  s.max_delta_step = p.max_delta_step;
  s.path_smooth = p.path_smooth;
  s.min_data_in_leaf = p.min_data_in_leaf;
  s.min_sum_hessian_in_leaf = p.min_sum_hessian_in_leaf;
  s.min_gain_to_split = p.min_gain_to_split;
  s.max_cat_to_onehot = p.max_cat_to_onehot;
  s.max_cat_threshold = p.max_cat_threshold;
  s.cat_l2 = p.cat_l2;
  s.cat_smooth = p.cat_smooth;
  s.min_data_per_group = p.min_data_per_group;
  return s;
}

}  // namespace oracle

using namespace oracle;

static thread_local std::string g_last_error;
void oracle::set_last_error(const std::string& msg) { g_last_error = msg; }

extern "C" {

const char* oracle_last_error() { return g_last_error.c_str(); }

int oracle_train(const OracleParams* p, const OracleData* train, const float* label, const int32_t* query_boundaries,
                 int32_t num_queries, const OracleData* valid, OracleBooster** out) {
  ORACLE_TRY({
    auto b = std::make_unique<Booster>();
    b->p = *p;
    b->data = make_binned(*train);
    size_t n = (size_t)train->num_data;
    b->label.assign(label, label + n);
    b->ntpi = p->objective == 2 ? p->num_class : 1;
    if (valid && valid->num_data > 0) {
      b->valid = make_binned(*valid);
      b->valid_scores.assign((size_t)valid->num_data * b->ntpi, 0.0);
    }
    b->scores.assign(n * b->ntpi, 0.0);
    b->grad.assign(n * b->ntpi, 0.0f);
    b->hess.assign(n * b->ntpi, 0.0f);
    b->class_need_train.assign(b->ntpi, true);
    if (p->objective == 2) {
      for (int k = 0; k < b->ntpi; ++k) {
        double c = 0.0;
        for (size_t i = 0; i < n; ++i) c += (int32_t)label[i] == k ? 1.0 : 0.0;
        double pr = std::fabs(c / (double)n);
        b->class_need_train[k] = !(pr <= kEpsilon || pr >= 1.0 - kEpsilon);
      }
    }
    if (p->objective == 3) {
      b->bnd.assign(query_boundaries, query_boundaries + num_queries + 1);
      b->rank = std::make_unique<Lambdarank>(p->sigmoid, p->lambdarank_norm != 0, p->lambdarank_truncation_level,
                                             label, query_boundaries, (size_t)num_queries);
    }
    LearnerConfig lc;
    lc.params = split_params(*p);
    lc.num_leaves = p->num_leaves;
    lc.max_depth = p->max_depth;
    lc.monotone_penalty = p->monotone_penalty;
    lc.use_monotone = train->monotone != nullptr;
    lc.quantized = p->use_quantized_grad != 0;
    lc.num_grad_quant_bins = p->num_grad_quant_bins;
    lc.stochastic_rounding = p->stochastic_rounding != 0;
    lc.quant_renew = p->quant_train_renew_leaf != 0;
    lc.seed = p->seed;
    lc.num_threads = p->num_threads;
    lc.is_constant_hessian = p->objective == 1;  // L2 without weights
    b->learner = std::make_unique<SerialTreeLearner>(&b->data, lc);
    if (p->bagging_fraction < 1.0 && p->bagging_freq > 0) {
      for (size_t i = 0; i < (n + 1023) / 1024; ++i) b->rands.emplace_back(p->bagging_seed + (int32_t)i);
      b->bag_indices.assign(n, 0);
      b->bag_cnt = n;
    }
    b->col_rand = Random(p->feature_fraction_seed);
    int32_t total = train->num_features;
    b->used_cnt_bytree = p->feature_fraction < 1.0
                             ? std::max(std::min(1, total), (int32_t)((double)total * p->feature_fraction + (double)0.5f))
                             : total;
    for (int32_t it = 0; it < p->num_iterations; ++it)
      if (train_one_iter(*b)) break;
    *out = reinterpret_cast<OracleBooster*>(b.release());
  })
}

// One more boosting iteration of a booster made by oracle_train (which may
// have run 0 iterations): Gbdt::train_one_iter (boosting.rs:957). *stop is 1
// when the iteration found no split (training has finished).
int oracle_booster_update(OracleBooster* h, int32_t* stop) {
  ORACLE_TRY({
    Booster* b = reinterpret_cast<Booster*>(h);
    const bool finished = train_one_iter(*b);
    if (stop) *stop = finished ? 1 : 0;
  })
}

// SerialTreeLearner::train on given gradients (class-major, `num_trees`
// trees in sequence on one learner) — the learner-level parity entry.
// `bytree` (optional, [num_trees x num_features]) is each tree's by-tree mask.
int oracle_train_tree(const OracleParams* p, const OracleData* train, const float* grad, const float* hess,
                      const uint32_t* bag, int64_t n_bag, int32_t num_trees, const uint8_t* bytree,
                      OracleBooster** out) {
  ORACLE_TRY({
    auto b = std::make_unique<Booster>();
    b->p = *p;
    b->data = make_binned(*train);
    size_t n = (size_t)train->num_data;
    LearnerConfig lc;
    lc.params = split_params(*p);
    lc.num_leaves = p->num_leaves;
    lc.max_depth = p->max_depth;
    lc.monotone_penalty = p->monotone_penalty;
    lc.use_monotone = train->monotone != nullptr;
    lc.quantized = p->use_quantized_grad != 0;
    lc.num_grad_quant_bins = p->num_grad_quant_bins;
    lc.stochastic_rounding = p->stochastic_rounding != 0;
    lc.quant_renew = p->quant_train_renew_leaf != 0;
    lc.seed = p->seed;
    lc.num_threads = p->num_threads;
    lc.is_constant_hessian = p->objective == 1;
    b->learner = std::make_unique<SerialTreeLearner>(&b->data, lc);
    if (bag) b->learner->set_bagging_data(bag, (size_t)n_bag);
    b->ntpi = 1;
    for (int32_t k = 0; k < num_trees; ++k) {
      if (bytree) {
        std::vector<bool> m((size_t)train->num_features);
        for (int32_t f = 0; f < train->num_features; ++f) m[f] = bytree[(size_t)k * train->num_features + f] != 0;
        b->learner->set_bytree_mask(m);
      }
      b->models.push_back(b->learner->train(grad + (size_t)k * n, hess + (size_t)k * n));
      b->traces.push_back(b->learner->trace);
    }
    *out = reinterpret_cast<OracleBooster*>(b.release());
  })
}

// partition() of the last trained tree: per-leaf begin/count and the rows.
int oracle_booster_partition(OracleBooster* h, int32_t* leaf_begin, int32_t* leaf_count, uint32_t* indices) {
  auto* b = reinterpret_cast<Booster*>(h);
  const Tree& t = b->models.back();
  for (int32_t l = 0; l < t.num_leaves; ++l) {
    leaf_begin[l] = (int32_t)b->learner->leaf_begin(l);
    leaf_count[l] = (int32_t)b->learner->leaf_count(l);
  }
  const auto& idx = b->learner->indices();
  std::copy(idx.begin(), idx.end(), indices);
  return 0;
}

void oracle_booster_free(OracleBooster* h) { delete reinterpret_cast<Booster*>(h); }

int32_t oracle_booster_num_trees(OracleBooster* h) { return (int32_t)reinterpret_cast<Booster*>(h)->models.size(); }

int oracle_booster_tree(OracleBooster* h, int32_t i, OracleTreeView* out) {
  auto* b = reinterpret_cast<Booster*>(h);
  if (i < 0 || (size_t)i >= b->models.size()) return -1;
  const Tree& t = b->models[(size_t)i];
  out->num_leaves = t.num_leaves;
  out->split_feature = t.split_feature.data();
  out->split_feature_inner = t.split_feature_inner.data();
  out->split_gain = t.split_gain.data();
  out->threshold_in_bin = t.threshold_in_bin.data();
  out->threshold = t.threshold.data();
  out->decision_type = t.decision_type.data();
  out->left_child = t.left_child.data();
  out->right_child = t.right_child.data();
  out->leaf_value = t.leaf_value.data();
  out->leaf_weight = t.leaf_weight.data();
  out->leaf_count = t.leaf_count.data();
  out->internal_value = t.internal_value.data();
  out->internal_weight = t.internal_weight.data();
  out->internal_count = t.internal_count.data();
  out->leaf_depth = t.leaf_depth.data();
  out->num_cat = t.num_cat;
  out->cat_boundaries = t.cat_boundaries.data();
  out->cat_threshold = t.cat_threshold.data();
  out->num_cat_threshold = (int32_t)t.cat_threshold.size();
  out->shrinkage = t.shrinkage;
  return 0;
}

int oracle_booster_trace(OracleBooster* h, int32_t i, int32_t* n, int32_t* leaf, int32_t* feature,
                         uint32_t* threshold, double* gain) {
  auto* b = reinterpret_cast<Booster*>(h);
  if (i < 0 || (size_t)i >= b->traces.size()) return -1;
  const auto& tr = b->traces[(size_t)i];
  if (!leaf) {
    *n = (int32_t)tr.size();
    return 0;
  }
  for (size_t k = 0; k < tr.size() && (int32_t)k < *n; ++k) {
    leaf[k] = tr[k].leaf;
    feature[k] = tr[k].feature;
    threshold[k] = tr[k].threshold;
    gain[k] = tr[k].gain;
  }
  return 0;
}

int oracle_booster_scores(OracleBooster* h, int valid, double* out) {
  auto* b = reinterpret_cast<Booster*>(h);
  const auto& s = valid ? b->valid_scores : b->scores;
  std::memcpy(out, s.data(), s.size() * sizeof(double));
  return 0;
}

// predict.rs:95-111 FlatTree::step semantics on raw f32 values (rows
// converted to f64 and |v| <= kZeroThreshold dropped, predict.rs:265-275).
int oracle_predict_raw(OracleBooster* h, const float* X, int64_t nrow, int32_t ncol, double* out) {
  auto* b = reinterpret_cast<Booster*>(h);
  int ntpi = b->ntpi;
  std::vector<double> row((size_t)ncol + 1);
  for (int64_t r = 0; r < nrow; ++r) {
    for (int32_t c = 0; c < ncol; ++c) {
      double v = (double)X[r * ncol + c];
      if (!std::isnan(v) && std::fabs(v) <= kZeroThreshold) v = 0.0;
      row[c] = v;
    }
    row[ncol] = 0.0;
    for (int k = 0; k < ntpi; ++k) out[r * ntpi + k] = 0.0;
    for (size_t m = 0; m < b->models.size(); ++m) {
      const Tree& t = b->models[m];
      int k = (int)(m % (size_t)ntpi);
      int32_t node = 0;
      if (t.num_leaves > 1) {
        while (node >= 0) {
          int32_t f = std::min(t.split_feature[node], ncol);
          double v = row[f];
          int8_t dt = t.decision_type[node];
          if (dt & 1) {  // categorical (predict.rs:77-90)
            int32_t c = (int32_t)t.threshold[node];
            bool left = !std::isnan(v) && (int32_t)v >= 0 &&
                        find_in_bitset(t.cat_threshold.data() + t.cat_boundaries[c],
                                       (size_t)(t.cat_boundaries[c + 1] - t.cat_boundaries[c]), (int32_t)v);
            node = left ? t.left_child[node] : t.right_child[node];
            continue;
          }
          int32_t mt = (dt >> 2) & 3;
          bool nan = std::isnan(v);
          bool nan_split = mt == kMissingNaN;
          if (nan && !nan_split) v = 0.0;
          bool zero = v >= -kZeroThreshold && v <= kZeroThreshold;
          bool is_default = (mt == kMissingZero && zero) || (nan_split && nan);
          bool left = is_default ? (dt & 2) != 0 : v <= t.threshold[node];
          node = left ? t.left_child[node] : t.right_child[node];
        }
        node = ~node;
      }
      out[r * ntpi + k] += t.leaf_value[node];
    }
  }
  return 0;
}

double oracle_auc(const float* label, const double* score, int64_t n) { return auc(label, score, (size_t)n); }

// metric.rs:546-598 NDCG@k for each of `ks` (no query weights).
int oracle_ndcg(const float* label, const double* score, const int32_t* bnd, int32_t nq, const int32_t* ks,
                int32_t nk, double* out) {
  Dcg dcg;
  std::vector<double> acc((size_t)nk, 0.0);
  for (int32_t q = 0; q < nq; ++q) {
    size_t s = (size_t)bnd[q], cnt = (size_t)(bnd[q + 1] - bnd[q]);
    std::vector<double> inv((size_t)nk);
    for (int32_t j = 0; j < nk; ++j) {
      double v = dcg.max_dcg_at_k((size_t)ks[j], label + s, cnt);
      inv[j] = v > 0.0 ? 1.0 / v : -1.0;
    }
    if (inv[0] <= 0.0) {
      for (auto& a : acc) a += 1.0;
      continue;
    }
    auto sorted = sort_by_score_desc(score + s, cnt);
    double cur = 0.0;
    size_t left = 0;
    for (int32_t j = 0; j < nk; ++j) {
      size_t k = std::min((size_t)ks[j], cnt);
      for (size_t r = left; r < k; ++r) cur += dcg.label_gain[(int32_t)label[s + sorted[r]]] * dcg.discount[r];
      acc[j] += cur * inv[j];
      left = k;
    }
  }
  for (int32_t j = 0; j < nk; ++j) out[j] = acc[j] / (double)nq;
  return 0;
}

int oracle_gradients(int32_t objective, int32_t num_class, double sigmoid, const float* label, const double* scores,
                     int64_t n, const int32_t* bnd, int32_t nq, int32_t truncation, int32_t norm, float* g, float* h) {
  ORACLE_TRY({
    switch (objective) {
      case 0: grad_binary(label, scores, (size_t)n, sigmoid, g, h); break;
      case 1: grad_l2(label, scores, (size_t)n, g, h); break;
      case 2: grad_softmax(label, scores, (size_t)n, num_class, g, h); break;
      case 3: {
        Lambdarank lr(sigmoid, norm != 0, truncation, label, bnd, (size_t)nq);
        for (int32_t q = 0; q < nq; ++q)
          lr.one_query((size_t)q, label + bnd[q], scores + bnd[q], (size_t)(bnd[q + 1] - bnd[q]), g + bnd[q], h + bnd[q]);
        break;
      }
      default: throw std::runtime_error("unknown objective");
    }
  })
}

// FP64 / packed-int histogram of a row subset, in the learner's layout.
int oracle_hist(const OracleData* d, const uint32_t* rows, int64_t nrows, const float* g, const float* h,
                const int64_t* packed, double* out_f64, int64_t* out_int) {
  ORACLE_TRY({
    BinnedData b = make_binned(*d);
    LearnerConfig lc{};
    lc.num_leaves = 2;
    SerialTreeLearner l(&b, lc);
    size_t n = rows ? (size_t)nrows : (size_t)d->num_data;
    if (out_f64) l.build_hist(rows, n, g, h, out_f64);
    if (out_int) l.build_hist_int(rows, n, packed, out_int);
  })
}

// histogram.rs:42-56 fix on one feature view: num_bin bins, the view
// starting at bin `offset`, hist holding 2 * (num_bin - offset) values.
int oracle_fix_hist(int32_t num_bin, int32_t offset, int32_t most_freq_bin, double sum_g, double sum_h,
                    double* hist) {
  ORACLE_TRY({
    FeatureMeta m{};
    m.num_bin = num_bin;
    m.offset = offset;
    m.most_freq_bin = (uint32_t)most_freq_bin;
    if (offset == 0) fix_hist(m, sum_g, sum_h, hist);  // an offset view has no stored most-frequent bin to fix
  })
}

// split.rs:114-121 SplitInfo::better_than of (gain_a, feature_a) against
// (gain_b, feature_b); feature -1 is "no split".
int32_t oracle_better_than(double gain_a, int32_t feature_a, double gain_b, int32_t feature_b) {
  SplitInfo a, b;
  a.gain = gain_a;
  a.feature = feature_a;
  b.gain = gain_b;
  b.feature = feature_b;
  return a.better_than(b) ? 1 : 0;
}

int oracle_find_best_threshold(const OracleFeature* f, const OracleParams* p, const double* hist,
                               const int64_t* ihist, double sum_g, double sum_h, int64_t int_sum, double gscale,
                               double hscale, int32_t num_data, double parent_output, OracleSplit* out) {
  ORACLE_TRY({
    FeatureMeta m;
    m.num_bin = f->num_bin;
    m.missing_type = f->missing_type;
    m.default_bin = (uint32_t)f->default_bin;
    m.most_freq_bin = (uint32_t)f->most_freq_bin;
    m.offset = f->offset;
    m.bin_type = f->bin_type;
    m.monotone_type = f->monotone_type;
    m.penalty = f->penalty;
    m.real_index = 0;
    SplitParams sp = split_params(*p);
    SplitInfo s;
    BasicConstraint c{f->constraint_min, f->constraint_max};
    const BasicConstraint* mc = f->use_constraint ? &c : nullptr;
    bool ok = ihist ? find_best_threshold_int(ihist, m, sp, int_sum, gscale, hscale, num_data, parent_output, mc, s)
                    : find_best_threshold(hist, m, sp, sum_g, sum_h, num_data, parent_output, mc, s);
    out->splittable = ok;
    out->threshold = s.threshold;
    out->gain = s.gain;
    out->left_output = s.left_output;
    out->right_output = s.right_output;
    out->left_count = s.left_count;
    out->right_count = s.right_count;
    out->left_sum_gradient = s.left_sum_gradient;
    out->left_sum_hessian = s.left_sum_hessian;
    out->right_sum_gradient = s.right_sum_gradient;
    out->right_sum_hessian = s.right_sum_hessian;
    out->default_left = s.default_left;
    out->num_cat = (int32_t)s.cat_threshold.size();
    for (size_t i = 0; i < s.cat_threshold.size() && i < 256; ++i) out->cat_threshold[i] = s.cat_threshold[i];
    out->left_sum_gh = s.left_sum_gh;
    out->right_sum_gh = s.right_sum_gh;
  })
}

int oracle_discretize(int32_t bins, int32_t seed, int32_t const_hess, int32_t stochastic, int64_t n,
                      int32_t num_threads, int32_t num_calls, const float* g, const float* h, int64_t* packed,
                      double* scales) {
  ORACLE_TRY({
    GradientDiscretizer q(bins, seed, const_hess != 0, stochastic != 0, (size_t)n, (size_t)num_threads);
    for (int32_t c = 0; c < num_calls; ++c) q.discretize(g, h, (size_t)n, nullptr, 0);
    std::memcpy(packed, q.packed.data(), (size_t)n * sizeof(int64_t));
    scales[0] = q.grad_scale;
    scales[1] = q.hess_scale;
  })
}

int oracle_mt19937(uint32_t seed, int32_t n, uint32_t* out) {
  Mt19937 m(seed);
  for (int32_t i = 0; i < n; ++i) out[i] = m.next_u32();
  return 0;
}

int oracle_lcg_sample(int32_t seed, int32_t n, int32_t k, int32_t* out, int32_t* out_len) {
  Random r(seed);
  auto v = r.sample(n, k);
  for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
  *out_len = (int32_t)v.size();
  return 0;
}

int oracle_block_info(int64_t threads, int64_t cnt, int64_t min_cnt, int64_t* out) {
  size_t a, b;
  block_info((size_t)threads, (size_t)cnt, (size_t)min_cnt, &a, &b);
  out[0] = (int64_t)a;
  out[1] = (int64_t)b;
  return 0;
}

int8_t oracle_to_i8(double x) { return to_i8(x); }


}  // extern "C"

// ---- model text: io.rs:13-85 (save_model_to_string), tree.rs:718-773
// (Tree::to_model_string) and fmt.rs (%g / %.17g) ---------------------------
// The text stops after the feature importances: the "parameters:" block is
// the Config's own text (config.rs:1169-1187), which is not on this path.
static std::string fmt_g(double v, int prec) {  // fmt.rs fmt_g: C printf("%.{prec}g")
  if (std::isnan(v)) return std::signbit(v) ? "-nan" : "nan";
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.*g", prec, v);
  return buf;
}

template <class T, class F>
static std::string join_arr(const T* a, size_t n, F f) {
  std::string s;
  for (size_t i = 0; i < n; ++i) {
    if (i) s += ' ';
    s += f(a[i]);
  }
  return s;
}

static std::string tree_text(const Tree& t) {  // tree.rs:718-773 (is_linear false)
  const size_t n = (size_t)t.num_leaves, ni = n - 1;
  auto i2s = [](auto x) { return std::to_string((long long)x); };
  auto g6 = [](double x) { return fmt_g(x, 6); };
  auto g17 = [](double x) { return fmt_g(x, 17); };
  std::string s;
  s += "num_leaves=" + std::to_string(n) + "\n";
  s += "num_cat=" + std::to_string(t.num_cat) + "\n";
  s += "split_feature=" + join_arr(t.split_feature.data(), ni, i2s) + "\n";
  s += "split_gain=" + join_arr(t.split_gain.data(), ni, [&](float x) { return g6((double)x); }) + "\n";
  s += "threshold=" + join_arr(t.threshold.data(), ni, g17) + "\n";
  s += "decision_type=" + join_arr(t.decision_type.data(), ni, i2s) + "\n";
  s += "left_child=" + join_arr(t.left_child.data(), ni, i2s) + "\n";
  s += "right_child=" + join_arr(t.right_child.data(), ni, i2s) + "\n";
  s += "leaf_value=" + join_arr(t.leaf_value.data(), n, g17) + "\n";
  s += "leaf_weight=" + join_arr(t.leaf_weight.data(), std::min(n, t.leaf_weight.size()), g17) + "\n";
  s += "leaf_count=" + join_arr(t.leaf_count.data(), n, i2s) + "\n";
  s += "internal_value=" + join_arr(t.internal_value.data(), ni, g6) + "\n";
  s += "internal_weight=" + join_arr(t.internal_weight.data(), ni, g6) + "\n";
  s += "internal_count=" + join_arr(t.internal_count.data(), ni, i2s) + "\n";
  if (t.num_cat > 0) {
    s += "cat_boundaries=" + join_arr(t.cat_boundaries.data(), (size_t)t.num_cat + 1, i2s) + "\n";
    s += "cat_threshold=" + join_arr(t.cat_threshold.data(), t.cat_threshold.size(), i2s) + "\n";
  }
  s += "is_linear=0\n";
  s += "shrinkage=" + g6(t.shrinkage) + "\n";
  s += "\n";
  return s;
}

extern "C" {

int oracle_model_to_string(OracleBooster* h, int32_t num_total_features, const char* feature_infos,
                           const int8_t* monotone, int32_t num_monotone, const char** out) {
  ORACLE_TRY({
    Booster* b = reinterpret_cast<Booster*>(h);
    const OracleParams& p = b->p;
    std::string obj;  // the objectives' to_model_string
    if (p.objective == 0) obj = "binary sigmoid:" + fmt_g(p.sigmoid, 6);  // binary.rs:168-170
    else if (p.objective == 1) obj = "regression";                       // regression.rs:346-348
    else if (p.objective == 2) obj = "multiclass num_class:" + std::to_string(p.num_class);  // multiclass.rs:169
    else obj = "lambdarank";                                              // rank.rs:338-340
    std::string s = "tree\nversion=v4\n";
    s += "num_class=" + std::to_string(p.objective == 2 ? p.num_class : 1) + "\n";
    s += "num_tree_per_iteration=" + std::to_string(b->ntpi) + "\n";
    s += "label_index=0\n";
    s += "max_feature_idx=" + std::to_string(num_total_features - 1) + "\n";
    s += "objective=" + obj + "\n";
    std::string names;
    for (int32_t c = 0; c < num_total_features; ++c) names += (c ? " Column_" : "Column_") + std::to_string(c);
    s += "feature_names=" + names + "\n";
    if (monotone && num_monotone > 0)
      s += "monotone_constraints=" + join_arr(monotone, (size_t)num_monotone, [](int8_t x) {
             return std::to_string((int)x);
           }) + "\n";
    s += std::string("feature_infos=") + (feature_infos ? feature_infos : "") + "\n";
    std::vector<std::string> trees;
    for (size_t i = 0; i < b->models.size(); ++i)
      trees.push_back("Tree=" + std::to_string(i) + "\n" + tree_text(b->models[i]) + "\n");
    std::string sizes;
    for (size_t i = 0; i < trees.size(); ++i) sizes += (i ? " " : "") + std::to_string(trees[i].size());
    s += "tree_sizes=" + sizes + "\n\n";
    for (const std::string& t : trees) s += t;
    s += "end of trees\n";
    // boosting.rs:1337-1360 split counts, importance_type 0; sorted by count,
    // descending, stable
    std::vector<long long> imp((size_t)num_total_features, 0);
    for (const Tree& t : b->models)
      for (int32_t k = 0; k + 1 < t.num_leaves; ++k)
        if (t.split_gain[(size_t)k] > 0.0f) imp[(size_t)t.split_feature[(size_t)k]] += 1;
    std::vector<int32_t> order;
    for (int32_t c = 0; c < num_total_features; ++c)
      if (imp[(size_t)c] > 0) order.push_back(c);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t c) { return imp[(size_t)a] > imp[(size_t)c]; });
    s += "\nfeature_importances:\n";
    for (int32_t c : order) s += "Column_" + std::to_string(c) + "=" + std::to_string(imp[(size_t)c]) + "\n";
    b->model_text = s;
    *out = b->model_text.c_str();
  });
}

}  // extern "C"
