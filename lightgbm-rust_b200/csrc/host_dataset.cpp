// Host-side dataset construction: the part of lightgbm-rust's Dataset that
// produces the u8 feature-group bin matrix the GPU learner uploads once.
// This stands in for the Rust host's own binning (which stays on the host);
// it restates, bit-exactly:
//   crates/lgbm-core/src/binning.rs   GreedyFindBin, FindBinWithZeroAsOneBin,
//                                     BinMapper::find_bin / finish / value_to_bin
//   crates/lgbm-core/src/dataset.rs   :394-399 row sampling, :860-918 bin params
//   crates/lgbm-core/src/random.rs    the LCG and Random::sample
//   crates/lgbm-core/src/feature_group.rs :144-154 the stored group value
// Only dense single-feature groups are produced: a dataset whose features
// exclusive feature bundling could merge (feature_groups.rs) is rejected
// with LGBM_B200_ERR_UNSUPPORTED.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <set>
#include <string>
#include <vector>

#include "lgbm_b200_internal.h"

namespace lgbm_b200 {

namespace {

constexpr double kZeroThreshold = (double)1e-35f;
constexpr double kSparseThreshold = 0.7;

struct Lcg {  // random.rs:9-70
  uint32_t x;
  explicit Lcg(int32_t seed) : x((uint32_t)seed) {}
  int32_t rand_int16() { x = x * 214013u + 2531011u; return (int32_t)((x >> 16) & 0x7FFF); }
  int32_t rand_int32() { x = x * 214013u + 2531011u; return (int32_t)(x & 0x7FFFFFFF); }
  int32_t next_int(int32_t lo, int32_t hi) { return rand_int32() % (hi - lo) + lo; }
  float next_float() { return (float)rand_int16() / 32768.0f; }
  std::vector<int32_t> sample(int32_t n, int32_t k) {
    std::vector<int32_t> ret;
    if (k > n || k <= 0) return ret;
    if (k == n) {
      ret.resize(n);
      std::iota(ret.begin(), ret.end(), 0);
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
};

inline double next_up(double a) { return std::nextafter(a, INFINITY); }
inline bool check_double_equal_ordered(double a, double b) { return b <= next_up(a); }

// binning.rs:98-118
bool need_filter(const std::vector<int32_t>& cnt_in_bin, int32_t total_cnt, int32_t filter_cnt, int32_t bin_type) {
  if (bin_type == 0) {
    int32_t sum_left = 0;
    for (size_t i = 0; i + 1 < cnt_in_bin.size(); ++i) {
      sum_left += cnt_in_bin[i];
      if (sum_left >= filter_cnt && total_cnt - sum_left >= filter_cnt) return false;
    }
  } else {
    if (cnt_in_bin.size() > 2) return false;
    for (size_t i = 0; i + 1 < cnt_in_bin.size(); ++i) {
      int32_t sum_left = cnt_in_bin[i];
      if (sum_left >= filter_cnt && total_cnt - sum_left >= filter_cnt) return false;
    }
  }
  return true;
}

// binning.rs:121-212
std::vector<double> greedy_find_bin(const double* dv, const int32_t* counts, int32_t ndv, int32_t max_bin,
                                    size_t total_cnt, int32_t min_data_in_bin) {
  std::vector<double> ub;
  if (ndv == 0) return {INFINITY};
  if (ndv <= max_bin) {
    int32_t cur = 0;
    for (int32_t i = 0; i < ndv - 1; ++i) {
      cur += counts[i];
      if (cur >= min_data_in_bin) {
        double val = next_up((dv[i] + dv[i + 1]) / 2.0);
        if (ub.empty() || !check_double_equal_ordered(ub.back(), val)) {
          ub.push_back(val);
          cur = 0;
        }
      }
    }
    ub.push_back(INFINITY);
  } else {
    if (min_data_in_bin > 0) {
      max_bin = std::min(max_bin, (int32_t)(total_cnt / (size_t)min_data_in_bin));
      max_bin = std::max(max_bin, 1);
    }
    double mean_bin_size = (double)total_cnt / (double)max_bin;
    int32_t rest_bin_cnt = max_bin;
    int32_t rest_sample_cnt = (int32_t)total_cnt;
    size_t n = (size_t)ndv;
    std::vector<char> big(n, 0);
    for (size_t i = 0; i < n; ++i) {
      if ((double)counts[i] >= mean_bin_size) {
        big[i] = 1;
        rest_bin_cnt -= 1;
        rest_sample_cnt -= counts[i];
      }
    }
    mean_bin_size = (double)rest_sample_cnt / (double)rest_bin_cnt;
    std::vector<double> upper(max_bin, INFINITY), lower(max_bin, INFINITY);
    int32_t bin_cnt = 0;
    lower[0] = dv[0];
    int32_t cur = 0;
    for (size_t i = 0; i + 1 < n; ++i) {
      if (!big[i]) rest_sample_cnt -= counts[i];
      cur += counts[i];
      double half = std::max(mean_bin_size * (double)0.5f, 1.0);
      if (big[i] || (double)cur >= mean_bin_size || (big[i + 1] && (double)cur >= half)) {
        upper[bin_cnt] = dv[i];
        bin_cnt += 1;
        lower[bin_cnt] = dv[i + 1];
        if (bin_cnt >= max_bin - 1) break;
        cur = 0;
        if (!big[i]) {
          rest_bin_cnt -= 1;
          mean_bin_size = (double)rest_sample_cnt / (double)rest_bin_cnt;
        }
      }
    }
    bin_cnt += 1;
    for (int32_t i = 0; i < bin_cnt - 1; ++i) {
      double val = next_up((upper[i] + lower[i + 1]) / 2.0);
      if (ub.empty() || !check_double_equal_ordered(ub.back(), val)) ub.push_back(val);
    }
    ub.push_back(INFINITY);
  }
  return ub;
}

// binning.rs:215-279
std::vector<double> find_bin_with_zero_as_one_bin(const std::vector<double>& dv, const std::vector<int32_t>& counts,
                                                  int32_t max_bin, size_t total_sample_cnt, int32_t min_data_in_bin) {
  size_t n = dv.size();
  std::vector<double> ub;
  int32_t left_cnt_data = 0, cnt_zero = 0, right_cnt_data = 0;
  for (size_t i = 0; i < n; ++i) {
    if (dv[i] <= -kZeroThreshold) left_cnt_data += counts[i];
    else if (dv[i] > kZeroThreshold) right_cnt_data += counts[i];
    else cnt_zero += counts[i];
  }
  size_t left_cnt = n;
  for (size_t i = 0; i < n; ++i)
    if (dv[i] > -kZeroThreshold) {
      left_cnt = i;
      break;
    }
  if (left_cnt > 0 && max_bin > 1) {
    double denom = (double)(total_sample_cnt - (size_t)cnt_zero);
    int32_t left_max_bin = (int32_t)((double)left_cnt_data / denom * (double)(max_bin - 1));
    left_max_bin = std::max(left_max_bin, 1);
    ub = greedy_find_bin(dv.data(), counts.data(), (int32_t)left_cnt, left_max_bin, (size_t)left_cnt_data,
                         min_data_in_bin);
    if (!ub.empty()) ub.back() = -kZeroThreshold;
  }
  size_t right_start = n;
  for (size_t i = left_cnt; i < n; ++i)
    if (dv[i] > kZeroThreshold) {
      right_start = i;
      break;
    }
  int32_t right_max_bin = max_bin - 1 - (int32_t)ub.size();
  if (right_start < n && right_max_bin > 0) {
    auto rb = greedy_find_bin(dv.data() + right_start, counts.data() + right_start, (int32_t)(n - right_start),
                              right_max_bin, (size_t)right_cnt_data, min_data_in_bin);
    ub.push_back(kZeroThreshold);
    ub.insert(ub.end(), rb.begin(), rb.end());
  } else {
    ub.push_back(INFINITY);
  }
  return ub;
}

struct BinParams {
  int32_t max_bin, min_data_in_bin, min_split_data;
  bool pre_filter, use_missing, zero_as_missing;
};

// binning.rs:605-633 BinMapper::finish
void finish(BinMapper& m, const std::vector<int32_t>& cnt_in_bin, size_t total, const BinParams& p) {
  m.is_trivial = m.num_bin <= 1;
  if (!m.is_trivial && p.pre_filter && need_filter(cnt_in_bin, (int32_t)total, p.min_split_data, m.bin_type))
    m.is_trivial = true;
  if (!m.is_trivial) {
    m.default_bin = value_to_bin(m, 0.0);
    size_t arg_max = 0;
    for (size_t i = 1; i < cnt_in_bin.size(); ++i)
      if (cnt_in_bin[i] > cnt_in_bin[arg_max]) arg_max = i;
    m.most_freq_bin = (uint32_t)arg_max;
    double max_sparse_rate = (double)cnt_in_bin[arg_max] / (double)total;
    if (m.most_freq_bin != m.default_bin && max_sparse_rate < kSparseThreshold) m.most_freq_bin = m.default_bin;
    m.sparse_rate = (double)cnt_in_bin[m.most_freq_bin] / (double)total;
  } else {
    m.sparse_rate = 1.0;
  }
}

// binning.rs:387-603 BinMapper::find_bin (no forced bounds).
BinMapper find_bin(const std::vector<double>& values, size_t total_sample_cnt, int32_t bin_type, const BinParams& p) {
  int32_t num_in = (int32_t)values.size();
  std::vector<double> vals;
  vals.reserve(values.size());
  for (double v : values)
    if (!std::isnan(v)) vals.push_back(v);
  int32_t non_na = (int32_t)vals.size();
  int32_t na_cnt = 0;
  int32_t missing_type;
  if (!p.use_missing) missing_type = 0;
  else if (p.zero_as_missing) missing_type = 1;
  else if (non_na == num_in) missing_type = 0;
  else {
    na_cnt = num_in - non_na;
    missing_type = 2;
  }
  int32_t nsv = non_na;
  int32_t zero_cnt = (int32_t)((int64_t)total_sample_cnt - nsv - na_cnt);
  std::stable_sort(vals.begin(), vals.end());
  std::vector<double> dv;
  std::vector<int32_t> counts;
  if (nsv == 0 || (vals[0] > 0.0 && zero_cnt > 0)) {
    dv.push_back(0.0);
    counts.push_back(zero_cnt);
  }
  if (nsv > 0) {
    dv.push_back(vals[0]);
    counts.push_back(1);
  }
  for (int32_t i = 1; i < nsv; ++i) {
    if (!check_double_equal_ordered(vals[i - 1], vals[i])) {
      if (vals[i - 1] < 0.0 && vals[i] > 0.0) {
        dv.push_back(0.0);
        counts.push_back(zero_cnt);
      }
      dv.push_back(vals[i]);
      counts.push_back(1);
    } else {
      dv.back() = vals[i];
      counts.back() += 1;
    }
  }
  if (nsv > 0 && vals[nsv - 1] < 0.0 && zero_cnt > 0) {
    dv.push_back(0.0);
    counts.push_back(zero_cnt);
  }
  BinMapper m;
  m.min_val = dv[0];
  m.max_val = dv.back();
  m.bin_type = bin_type;
  if (bin_type == 1) {  // binning.rs:521-603 categorical
    m.missing_type = missing_type;
    std::vector<int32_t> dvi, ci;
    for (size_t i = 0; i < dv.size(); ++i) {
      int32_t val = (int32_t)dv[i];
      if (val < 0) na_cnt += counts[i];
      else if (dvi.empty() || dvi.back() != val) {
        dvi.push_back(val);
        ci.push_back(counts[i]);
      } else {
        ci.back() += counts[i];
      }
    }
    std::vector<int32_t> cnt_in_bin;
    int32_t rest_cnt = (int32_t)((int64_t)total_sample_cnt - na_cnt);
    m.num_bin = 1;
    m.bin_upper_bound = {INFINITY};
    if (rest_cnt > 0) {
      std::vector<std::pair<int32_t, int32_t>> pairs;
      for (size_t i = 0; i < dvi.size(); ++i) pairs.push_back({ci[i], dvi[i]});
      std::stable_sort(pairs.begin(), pairs.end(), [](auto& a, auto& b) { return a.first > b.first; });
      int32_t cut_cnt = (int32_t)((double)((float)(total_sample_cnt - (size_t)na_cnt) * 0.99f) + (double)0.5f);
      int32_t distinct_cnt = (int32_t)pairs.size() + (na_cnt > 0 ? 1 : 0);
      int32_t max_bin = std::min(distinct_cnt, p.max_bin);
      m.bin_2_categorical.push_back(-1);
      m.categorical_2_bin[-1] = 0;
      cnt_in_bin.push_back(0);
      int32_t used_cnt = 0;
      size_t cur = 0;
      while (cur < pairs.size() && (used_cnt < cut_cnt || m.num_bin < max_bin)) {
        if (pairs[cur].first < p.min_data_in_bin && cur > 1) break;
        m.bin_2_categorical.push_back(pairs[cur].second);
        m.categorical_2_bin[pairs[cur].second] = (uint32_t)m.num_bin;
        used_cnt += pairs[cur].first;
        cnt_in_bin.push_back(pairs[cur].first);
        m.num_bin += 1;
        cur += 1;
      }
      m.missing_type = (cur == pairs.size() && na_cnt == 0) ? 0 : 2;
      cnt_in_bin[0] = (int32_t)((int64_t)total_sample_cnt - used_cnt);
    }
    finish(m, cnt_in_bin, total_sample_cnt, p);
    return m;
  }
  std::vector<double> ub;
  if (missing_type == 1) {
    ub = find_bin_with_zero_as_one_bin(dv, counts, p.max_bin, total_sample_cnt, p.min_data_in_bin);
    if (ub.size() == 2) missing_type = 0;
  } else if (missing_type == 0) {
    ub = find_bin_with_zero_as_one_bin(dv, counts, p.max_bin, total_sample_cnt, p.min_data_in_bin);
  } else {
    ub = find_bin_with_zero_as_one_bin(dv, counts, p.max_bin - 1, total_sample_cnt - (size_t)na_cnt, p.min_data_in_bin);
    ub.push_back(NAN);
  }
  m.num_bin = (int32_t)ub.size();
  m.missing_type = missing_type;
  std::vector<int32_t> cnt_in_bin((size_t)m.num_bin, 0);
  size_t i_bin = 0;
  for (size_t i = 0; i < dv.size(); ++i) {
    while (dv[i] > ub[i_bin] && (int32_t)i_bin < m.num_bin - 1) i_bin += 1;
    cnt_in_bin[i_bin] += counts[i];
  }
  if (missing_type == 2) cnt_in_bin[(size_t)m.num_bin - 1] = na_cnt;
  m.bin_upper_bound = std::move(ub);
  finish(m, cnt_in_bin, total_sample_cnt, p);
  return m;
}

}  // namespace

// binning.rs:637-667 BinMapper::value_to_bin
uint32_t value_to_bin(const BinMapper& m, double value) {
  if (m.bin_type == 1) {
    if (std::isnan(value)) return 0;
    int32_t v = (int32_t)value;
    if (v < 0) return 0;
    auto it = m.categorical_2_bin.find(v);
    return it == m.categorical_2_bin.end() ? 0 : it->second;
  }
  if (std::isnan(value)) {
    if (m.missing_type == 2) return (uint32_t)(m.num_bin - 1);
    value = 0.0;
  }
  int32_t l = 0, r = m.num_bin - 1;
  if (m.missing_type == 2) r -= 1;
  while (l < r) {
    int32_t mid = (r + l - 1) / 2;
    if (value <= m.bin_upper_bound[(size_t)mid]) r = mid;
    else l = mid + 1;
  }
  return (uint32_t)l;
}

// feature_group.rs:144-154 for a single-feature group: 0 for the most
// frequent bin, else bin - (mfb == 0) + 1.
static inline uint8_t group_value(const BinMapper& m, uint32_t bin) {
  if (bin == m.most_freq_bin) return 0;
  return (uint8_t)(bin - (m.most_freq_bin == 0 ? 1u : 0u) + 1u);
}

static void push_bins(Dataset& d, const float* X, int64_t n, int32_t ncol) {
  int32_t nf = (int32_t)d.used.size();
  d.bins.assign((size_t)n * (size_t)nf, 0);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; ++r) {
    uint8_t* out = d.bins.data() + (size_t)r * nf;
    const float* row = X + (size_t)r * ncol;
    for (int32_t f = 0; f < nf; ++f) {
      const BinMapper& m = d.mappers[(size_t)f];
      out[f] = group_value(m, value_to_bin(m, (double)row[d.used[(size_t)f]]));
    }
  }
}

Status build_dataset(const float* X, int64_t n, int32_t ncol, const LgbmB200BinParams& p, Dataset& d, int device) {
  if (n <= 0 || ncol <= 0) return Status(LGBM_B200_ERR_INVALID_DATA, "empty matrix");
  if (n > INT32_MAX) return Status(LGBM_B200_ERR_INVALID_DATA, "more than 2^31-1 rows");
  std::vector<char> is_cat((size_t)ncol, 0);
  for (int32_t i = 0; i < p.num_categorical; ++i)
    if (p.categorical[i] >= 0 && p.categorical[i] < ncol) is_cat[(size_t)p.categorical[i]] = 1;
  // dataset.rs:394-396 row sample
  int32_t sample_cnt = (int32_t)std::min<int64_t>(n, std::max(p.bin_construct_sample_cnt, 0));
  Lcg rnd(p.data_random_seed);
  std::vector<int32_t> sample = rnd.sample((int32_t)n, sample_cnt);
  size_t total = sample.size();
  BinParams bp;
  bp.max_bin = p.max_bin;
  bp.min_data_in_bin = p.min_data_in_bin;
  bp.min_split_data = (int32_t)((double)p.min_data_in_leaf * (double)total / (double)n);
  bp.pre_filter = p.feature_pre_filter != 0;
  bp.use_missing = p.use_missing != 0;
  bp.zero_as_missing = p.zero_as_missing != 0;
  std::vector<BinMapper> all((size_t)ncol);
  std::vector<size_t> nonzero((size_t)ncol, 0);
  std::vector<std::vector<double>> cols((size_t)ncol);
#pragma omp parallel for schedule(dynamic)
  for (int32_t c = 0; c < ncol; ++c) {
    std::vector<double>& vals = cols[(size_t)c];
    for (int32_t r : sample) {  // matrix.rs:198-214 sample_columns
      double v = (double)X[(size_t)r * ncol + c];
      if (std::fabs(v) > kZeroThreshold || std::isnan(v)) vals.push_back(v);
    }
    nonzero[(size_t)c] = vals.size();
    all[(size_t)c] = find_bin(vals, total, is_cat[(size_t)c] ? 1 : 0, bp);
  }
  d.num_data = n;
  d.num_total_features = ncol;
  d.used.clear();
  d.mappers.clear();
  for (int32_t c = 0; c < ncol; ++c) {
    if (all[(size_t)c].is_trivial) continue;
    d.used.push_back(c);
    d.mappers.push_back(all[(size_t)c]);
  }
  // Exclusive feature bundling (feature_groups.rs:66-156) keeps every
  // feature in its own dense group when no two features fit together in
  // the sample and every feature is dense enough (>= 40% of the sample away
  // from its most frequent bin).
  size_t max_conflict = total / 10000;
  std::vector<size_t> nz;
  for (size_t k = 0; k < d.used.size(); ++k) {
    const BinMapper& m = d.mappers[k];
    size_t c = nonzero[(size_t)d.used[k]];
    if (m.default_bin != m.most_freq_bin) {  // feature_groups.rs:21-42 FixSampleIndices
      c = 0;
      std::vector<double>& vals = cols[(size_t)d.used[k]];
      size_t zeros = total - vals.size();
      if (m.default_bin != m.most_freq_bin) c += zeros;  // zeros sit in the default bin
      for (double v : vals)
        if (value_to_bin(m, v) != m.most_freq_bin) c += 1;
    }
    nz.push_back(c);
    if ((double)c / (double)total < 0.4)
      return Status(LGBM_B200_ERR_UNSUPPORTED, "feature " + std::to_string(d.used[k]) +
                                                   " is sparse (it would join a multi-value feature group)");
    if (m.bin_type == 0 ? m.num_bin > 255 + (m.most_freq_bin == 0 ? 1 : 0) : m.num_bin > 255)
      return Status(LGBM_B200_ERR_UNSUPPORTED, "more than 256 stored bins in feature " + std::to_string(d.used[k]));
  }
  if (nz.size() >= 2) {
    std::vector<size_t> s = nz;
    std::sort(s.begin(), s.end());
    if (s[0] + s[1] <= total + max_conflict)
      return Status(LGBM_B200_ERR_UNSUPPORTED, "features could be bundled (exclusive feature bundling)");
  }
  if (device >= 0) return push_bins_device(d, X, n, ncol, device);
  push_bins(d, X, n, ncol);
  return Status();
}

Status build_valid_dataset(const float* X, int64_t n, int32_t ncol, const Dataset& ref, Dataset& d, int device) {
  if (ncol != ref.num_total_features)
    return Status(LGBM_B200_ERR_INVALID_DATA, "validation data has a different number of columns");
  d.num_data = n;
  d.num_total_features = ncol;
  d.used = ref.used;
  d.mappers = ref.mappers;
  if (device >= 0) return push_bins_device(d, X, n, ncol, device);
  push_bins(d, X, n, ncol);
  return Status();
}

// dataset.rs:770-776 with BinMapper::bin_info_string (binning.rs:680-686):
// "[min:max]" (%.17g, the reference's fmt_g17) for a numerical feature, the
// category of every bin joined by ':' for a categorical one, "none" for a
// column left out as trivial.
const std::string& Dataset::infos() {
  if (!feature_infos.empty() || num_total_features == 0) return feature_infos;
  std::vector<int32_t> inner((size_t)num_total_features, -1);
  for (size_t k = 0; k < used.size(); ++k) inner[(size_t)used[k]] = (int32_t)k;
  std::string s;
  char buf[64];
  for (int32_t c = 0; c < num_total_features; ++c) {
    if (c) s += ' ';
    if (inner[(size_t)c] < 0) {
      s += "none";
      continue;
    }
    const BinMapper& m = mappers[(size_t)inner[(size_t)c]];
    if (m.bin_type == 1) {
      for (size_t i = 0; i < m.bin_2_categorical.size(); ++i) {
        if (i) s += ':';
        s += std::to_string(m.bin_2_categorical[i]);
      }
    } else {
      std::snprintf(buf, sizeof(buf), "[%.17g:", m.min_val);
      s += buf;
      std::snprintf(buf, sizeof(buf), "%.17g]", m.max_val);
      s += buf;
    }
  }
  feature_infos = s;
  return feature_infos;
}

void Dataset::fill_view(LgbmB200DatasetView* v) {
  size_t nf = used.size();
  num_bin.resize(nf);
  missing_type.resize(nf);
  default_bin.resize(nf);
  most_freq_bin.resize(nf);
  bin_type.resize(nf);
  real_index.resize(nf);
  ub_offsets.assign(nf + 1, 0);
  cat_offsets.assign(nf + 1, 0);
  upper_bounds.clear();
  bin_to_cat.clear();
  for (size_t f = 0; f < nf; ++f) {
    const BinMapper& m = mappers[f];
    num_bin[f] = m.num_bin;
    missing_type[f] = m.missing_type;
    default_bin[f] = (int32_t)m.default_bin;
    most_freq_bin[f] = (int32_t)m.most_freq_bin;
    bin_type[f] = m.bin_type;
    real_index[f] = used[f];
    if (m.bin_type == 0) upper_bounds.insert(upper_bounds.end(), m.bin_upper_bound.begin(), m.bin_upper_bound.end());
    else bin_to_cat.insert(bin_to_cat.end(), m.bin_2_categorical.begin(), m.bin_2_categorical.end());
    ub_offsets[f + 1] = (int64_t)upper_bounds.size();
    cat_offsets[f + 1] = (int64_t)bin_to_cat.size();
  }
  v->num_data = num_data;
  v->num_features = (int32_t)nf;
  v->num_total_features = num_total_features;
  v->bins = bins.data();
  v->num_bin = num_bin.data();
  v->missing_type = missing_type.data();
  v->default_bin = default_bin.data();
  v->most_freq_bin = most_freq_bin.data();
  v->bin_type = bin_type.data();
  v->real_index = real_index.data();
  v->upper_bounds = upper_bounds.data();
  v->ub_offsets = ub_offsets.data();
  v->bin_to_cat = bin_to_cat.data();
  v->cat_offsets = cat_offsets.data();
}

}  // namespace lgbm_b200
