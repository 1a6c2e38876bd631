// Oracle: RNGs (random.rs, mt19937.rs), gradient discretizer (learner/quant.rs)
// and tree bookkeeping (tree.rs). Test infrastructure only.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <set>

#include "oracle_impl.h"

namespace oracle {

// random.rs:45-70 Random::sample
std::vector<int32_t> Random::sample(int32_t n, int32_t k) {
  std::vector<int32_t> ret;
  if (k > n || k <= 0) return ret;
  if (k == n) {
    for (int32_t i = 0; i < n; ++i) ret.push_back(i);
  } else if (k > 1 && (double)k > ((double)n / std::log2((double)k))) {
    for (int32_t i = 0; i < n; ++i) {
      double prob = (double)((size_t)k - ret.size()) / (double)(n - i);
      if ((double)next_float() < prob) ret.push_back(i);
    }
  } else {
    std::set<int32_t> s;
    for (int32_t r = n - k; r < n; ++r) {
      int32_t v = next_int(0, r + 1);
      if (!s.insert(v).second) s.insert(r);
    }
    ret.assign(s.begin(), s.end());
  }
  return ret;
}

// mt19937.rs:128-193
Mt19937::Mt19937(uint32_t seed) {
  state[0] = seed;
  for (int i = 1; i < 624; ++i) {
    uint32_t prev = state[i - 1];
    state[i] = 1812433253u * (prev ^ (prev >> 30)) + (uint32_t)i;
  }
  idx = 624;
}
void Mt19937::twist() {
  for (int k = 0; k < 624; ++k) {
    uint32_t y = (state[k] & 0x80000000u) | (state[(k + 1) % 624] & 0x7fffffffu);
    uint32_t mag = (y & 1u) ? 0x9908b0dfu : 0u;
    state[k] = state[(k + 397) % 624] ^ (y >> 1) ^ mag;
  }
  idx = 0;
}
uint32_t Mt19937::next_u32() {
  if (idx >= 624) twist();
  uint32_t z = state[idx++];
  z ^= z >> 11;
  z ^= (z << 7) & 0x9d2c5680u;
  z ^= (z << 15) & 0xefc60000u;
  z ^= z >> 18;
  return z;
}
double Mt19937::canonical() {
  const double R = 4294967296.0;
  double sum = (double)next_u32();
  sum += (double)next_u32() * R;
  double ret = sum / (R * R);
  if (ret >= 1.0) {
    uint64_t bits = 0x3FEFFFFFFFFFFFFFull;
    std::memcpy(&ret, &bits, 8);
  }
  return ret;
}
int32_t Mt19937::uniform_int(int32_t a, int32_t b) {
  uint32_t range = (uint32_t)((int64_t)b - (int64_t)a + 1);
  uint64_t product = (uint64_t)next_u32() * (uint64_t)range;
  uint32_t low = (uint32_t)product;
  if (low < range) {
    uint32_t threshold = (uint32_t)(-range) % range;
    while (low < threshold) {
      product = (uint64_t)next_u32() * (uint64_t)range;
      low = (uint32_t)product;
    }
  }
  return (int32_t)((int64_t)(product >> 32) + (int64_t)a);
}

// multi_val_bin.rs:337-345
void block_info(size_t num_threads, size_t cnt, size_t min_cnt_per_block, size_t* nblock, size_t* block_size) {
  size_t nb = std::max<size_t>(1, std::min(num_threads, (cnt + min_cnt_per_block - 1) / min_cnt_per_block));
  if (nb > 1) {
    size_t size = (cnt + nb - 1) / nb;
    *nblock = nb;
    *block_size = (size + 31) / 32 * 32;
  } else {
    *nblock = 1;
    *block_size = cnt;
  }
}

// quant.rs:355-359 static_cast<int8_t>(double) as x86-64 compiles it.
int8_t to_i8(double x) {
  int32_t t = (std::isnan(x) || !(x >= -2147483648.0 && x < 2147483648.0)) ? INT32_MIN : (int32_t)x;
  return (int8_t)t;
}

// quant.rs:364-398
GradientDiscretizer::GradientDiscretizer(int32_t bins, int32_t seed, bool const_hess, bool stochastic,
                                         size_t num_data, size_t num_threads)
    : num_grad_quant_bins(bins), is_constant_hessian(const_hess), stochastic_rounding(stochastic),
      gradient_random_values(num_data, 0.0), hessian_random_values(num_data, 0.0), start_eng((uint32_t)seed),
      start_max((int32_t)num_data), raw(num_data, {0, 0}), packed(num_data, 0) {
  size_t nblock, bsize;
  block_info(num_threads, num_data, 512, &nblock, &bsize);
  for (size_t b = 0; b < nblock; ++b) {
    size_t start = b * bsize, end = std::min(start + bsize, num_data);
    Mt19937 ge((uint32_t)(seed + (int32_t)b));
    Mt19937 he((uint32_t)(seed + (int32_t)b + (int32_t)num_threads));
    for (size_t i = start; i < end; ++i) {
      gradient_random_values[i] = ge.uniform01();
      hessian_random_values[i] = he.uniform01();
    }
  }
}

// quant.rs:411-448 DiscretizeGradients; rows == nullptr means every row.
void GradientDiscretizer::discretize(const float* grad, const float* hess, size_t n_all, const uint32_t* rows,
                                     size_t n_rows) {
  size_t n = rows ? n_rows : n_all;
  if (n == 0) return;
  auto row = [&](size_t i) { return rows ? (size_t)rows[i] : i; };
  double max_g = std::fabs((double)grad[row(0)]), max_h = std::fabs((double)hess[row(0)]);
  for (size_t i = 0; i < n; ++i) {
    double g = std::fabs((double)grad[row(i)]), h = std::fabs((double)hess[row(i)]);
    if (g > max_g) max_g = g;
    if (h > max_h) max_h = h;
  }
  grad_scale = max_g / (double)(num_grad_quant_bins / 2);
  hess_scale = is_constant_hessian ? max_h : max_h / (double)num_grad_quant_bins;
  double inv_g = 1.0 / grad_scale, inv_h = 1.0 / hess_scale;
  size_t start = (size_t)start_eng.uniform_int(0, start_max);
  for (size_t i = 0; i < n; ++i) {
    size_t r = row(i);
    double g = (double)grad[r];
    double rg = 0.5, rh = 0.5;
    if (stochastic_rounding) {
      size_t pos = (i + start) % n;
      rg = gradient_random_values[pos];
      rh = hessian_random_values[pos];
    }
    int8_t gq = g >= 0.0 ? to_i8(g * inv_g + rg) : to_i8(g * inv_g - rg);
    int8_t hq = is_constant_hessian ? (int8_t)1 : to_i8((double)hess[r] * inv_h + rh);
    raw[r] = {hq, gq};
    packed[r] = (int64_t)((uint64_t)((int64_t)gq) << 32) | (int64_t)(uint8_t)hq;
  }
}

// quant.rs:452-461 (all rows) — the bag variant (quant.rs:467-477) is
// applied by the learner.
void GradientDiscretizer::root_sums(const uint32_t* rows, size_t n, double* sg, double* sh, int64_t* si) const {
  double a = 0, b = 0;
  uint64_t s = 0;
  for (size_t k = 0; k < n; ++k) {
    auto& r = raw[rows[k]];
    a += (double)r[1] * grad_scale;
    b += (double)r[0] * hess_scale;
    s += (uint64_t)packed[rows[k]];
  }
  *sg = a;
  *sh = b;
  *si = (int64_t)s;
}

// ---- tree.rs ---------------------------------------------------------------------
double maybe_round_to_zero(double v) { return (v >= -kZeroThreshold && v <= kZeroThreshold) ? 0.0 : v; }

std::vector<uint32_t> construct_bitset(const std::vector<int32_t>& vals) {  // tree.rs:32-42
  std::vector<uint32_t> ret;
  for (int32_t v : vals) {
    size_t i1 = (size_t)(v / 32);
    int32_t i2 = v % 32;
    if (ret.size() < i1 + 1) ret.resize(i1 + 1, 0);
    ret[i1] |= 1u << i2;
  }
  return ret;
}
bool find_in_bitset(const uint32_t* bits, size_t n, int32_t pos) {  // tree.rs:46-52
  size_t i1 = (size_t)(pos / 32);
  if (i1 >= n) return false;
  return ((bits[i1] >> (pos % 32)) & 1u) == 1u;
}

// tree.rs:254-297 Tree::split
int32_t tree_split(Tree& t, const SplitArgs& a) {
  int32_t leaf = a.leaf;
  int32_t new_node = t.num_leaves - 1;
  int32_t new_leaf = t.num_leaves;
  int32_t parent = t.leaf_parent[leaf];
  if (parent >= 0) {
    if (t.left_child[parent] == ~leaf) t.left_child[parent] = new_node;
    else t.right_child[parent] = new_node;
  }
  t.split_feature_inner.push_back(a.feature_inner);
  t.split_feature.push_back(a.feature_real);
  t.split_gain.push_back(a.gain);
  t.left_child.push_back(~leaf);
  t.right_child.push_back(~new_leaf);
  t.leaf_parent[leaf] = new_node;
  t.leaf_parent.push_back(new_node);
  t.internal_weight.push_back(a.left_weight + a.right_weight);
  t.internal_value.push_back(t.leaf_value[leaf]);
  t.internal_count.push_back(a.left_count + a.right_count);
  t.leaf_value[leaf] = std::isnan(a.left_value) ? 0.0 : a.left_value;
  t.leaf_weight[leaf] = a.left_weight;
  t.leaf_count[leaf] = a.left_count;
  t.leaf_value.push_back(std::isnan(a.right_value) ? 0.0 : a.right_value);
  t.leaf_weight.push_back(a.right_weight);
  t.leaf_count.push_back(a.right_count);
  int32_t d = t.leaf_depth[leaf] + 1;
  t.leaf_depth[leaf] = d;
  t.leaf_depth.push_back(d);
  int8_t dt = 0;
  if (a.default_left) dt |= 2;
  dt = (int8_t)((dt & 3) | (a.missing_type << 2));
  t.decision_type.push_back(dt);
  t.threshold_in_bin.push_back(a.threshold_bin);
  t.threshold.push_back(a.threshold);
  t.num_leaves += 1;
  return new_leaf;
}

// tree.rs:240-251 Tree::split_categorical
int32_t tree_split_categorical(Tree& t, const SplitArgs& a, const std::vector<uint32_t>& bits_inner,
                               const std::vector<uint32_t>& bits) {
  SplitArgs b = a;
  b.threshold_bin = (uint32_t)t.num_cat;
  b.threshold = (double)t.num_cat;
  b.default_left = false;
  int32_t right = tree_split(t, b);
  t.decision_type.back() |= 1;
  t.num_cat += 1;
  t.cat_boundaries.push_back(t.cat_boundaries.back() + (int32_t)bits.size());
  t.cat_threshold.insert(t.cat_threshold.end(), bits.begin(), bits.end());
  t.cat_boundaries_inner.push_back(t.cat_boundaries_inner.back() + (int32_t)bits_inner.size());
  t.cat_threshold_inner.insert(t.cat_threshold_inner.end(), bits_inner.begin(), bits_inner.end());
  return right;
}

void tree_set_leaf_output(Tree& t, int32_t leaf, double v) { t.leaf_value[leaf] = maybe_round_to_zero(v); }

void tree_shrink(Tree& t, double rate) {  // tree.rs:303-319
  for (int32_t i = 0; i < t.num_leaves - 1; ++i) {
    t.leaf_value[i] = maybe_round_to_zero(t.leaf_value[i] * rate);
    t.internal_value[i] = maybe_round_to_zero(t.internal_value[i] * rate);
  }
  int32_t last = t.num_leaves - 1;
  t.leaf_value[last] = maybe_round_to_zero(t.leaf_value[last] * rate);
  t.shrinkage *= rate;
}

void tree_add_bias(Tree& t, double v) {  // tree.rs:321-335
  for (int32_t i = 0; i < t.num_leaves - 1; ++i) {
    t.leaf_value[i] = maybe_round_to_zero(t.leaf_value[i] + v);
    t.internal_value[i] = maybe_round_to_zero(t.internal_value[i] + v);
  }
  int32_t last = t.num_leaves - 1;
  t.leaf_value[last] = maybe_round_to_zero(t.leaf_value[last] + v);
  t.shrinkage = 1.0;
}

void tree_as_constant(Tree& t, double v, int32_t count) {
  Tree c;
  c.leaf_value[0] = v;
  c.leaf_count[0] = count;
  t = c;
}

// tree.rs:588-633 leaf of a row of a binned dataset (single-feature groups).
int32_t tree_leaf_binned(const Tree& t, const BinnedData& d, int64_t row) {
  if (t.num_leaves <= 1) return 0;
  int32_t node = 0;
  while (node >= 0) {
    int32_t inner = t.split_feature_inner[node];
    const FeatureMeta& m = d.metas[inner];
    uint32_t raw = d.bins[row * d.num_features + inner];
    uint32_t b = raw == 0 ? m.most_freq_bin : raw - 1 + (uint32_t)(m.most_freq_bin == 0);
    if (t.decision_type[node] & 1) {
      int32_t c = (int32_t)t.threshold_in_bin[node];
      const uint32_t* bits = t.cat_threshold_inner.data() + t.cat_boundaries_inner[c];
      size_t nb = (size_t)(t.cat_boundaries_inner[c + 1] - t.cat_boundaries_inner[c]);
      node = find_in_bitset(bits, nb, (int32_t)b) ? t.left_child[node] : t.right_child[node];
      continue;
    }
    int32_t mt = (t.decision_type[node] >> 2) & 3;
    bool is_default = (mt == kMissingZero && b == m.default_bin) || (mt == kMissingNaN && b == (uint32_t)(m.num_bin - 1));
    if (is_default) node = (t.decision_type[node] & 2) ? t.left_child[node] : t.right_child[node];
    else node = b <= t.threshold_in_bin[node] ? t.left_child[node] : t.right_child[node];
  }
  return ~node;
}

}  // namespace oracle
