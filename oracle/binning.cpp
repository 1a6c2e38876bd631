// The oracle's own dataset construction: bin finding and the stored group
// values of a dense matrix, restated from the reference (single-threaded).
// TEST INFRASTRUCTURE ONLY (see oracle.h): it lets the oracle and the CPU
// baseline bin a matrix without the product library, and it is the checker
// the product's host binning is compared against.
//
//   crates/lgbm-core/src/binning.rs:98-118    need_filter
//   crates/lgbm-core/src/binning.rs:121-212   greedy_find_bin
//   crates/lgbm-core/src/binning.rs:214-275   find_bin_with_zero_as_one_bin
//   crates/lgbm-core/src/binning.rs:401-515   BinMapper::find_bin_logged
//   crates/lgbm-core/src/binning.rs:517-592   finish_categorical
//   crates/lgbm-core/src/binning.rs:596-622   finish
//   crates/lgbm-core/src/binning.rs:625-658   value_to_bin
//   crates/lgbm-core/src/binning.rs:680-686   bin_info_string
//   crates/lgbm-core/src/dataset.rs:394-399   row sample (Random::sample)
//   crates/lgbm-core/src/matrix.rs:198-214    sampled column values
//   crates/lgbm-core/src/dataset.rs:860-918   per-column bin parameters
//   crates/lgbm-core/src/dataset.rs:770-776   feature_infos
//   crates/lgbm-core/src/feature_group.rs:144-154  the stored value of a bin
//
// Forced bins, max_bin_by_feature and exclusive feature bundling are not
// restated: the workloads here use none of them, and a matrix whose features
// the reference would bundle is refused by the same rule the product applies
// (feature_groups.rs:66-156: every feature dense and no two fitting together).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>

#include "oracle_abi.h"
#include "oracle_impl.h"

namespace oracle {

namespace {

constexpr double kSparseThreshold = 0.7;  // consts.rs

double next_up(double a) { return std::nextafter(a, std::numeric_limits<double>::infinity()); }

struct BinParams {  // binning.rs:39-47
  int32_t max_bin, min_data_in_bin, min_split_data;
  bool pre_filter, use_missing, zero_as_missing;
};

struct Mapper {  // binning.rs:49-66
  int32_t num_bin = 1;
  int32_t missing_type = kMissingNone;
  std::vector<double> upper;  // bin_upper_bound
  bool is_trivial = true;
  int32_t bin_type = kNumerical;
  double min_val = 0.0, max_val = 0.0;
  uint32_t default_bin = 0, most_freq_bin = 0;
  std::vector<int32_t> bin_2_cat;
  std::map<int32_t, uint32_t> cat_2_bin;

  // binning.rs:625-658
  uint32_t value_to_bin(double value) const {
    if (bin_type == kCategorical) {
      if (std::isnan(value)) return 0;
      const int32_t v = (int32_t)value;
      if (v < 0) return 0;
      auto it = cat_2_bin.find(v);
      return it == cat_2_bin.end() ? 0u : it->second;
    }
    if (std::isnan(value)) {
      if (missing_type == kMissingNaN) return (uint32_t)(num_bin - 1);
      value = 0.0;
    }
    int32_t lo = 0, hi = num_bin - 1;
    if (missing_type == kMissingNaN) hi -= 1;
    while (lo < hi) {
      const int32_t mid = (hi + lo - 1) / 2;
      if (value <= upper[(size_t)mid]) hi = mid;
      else lo = mid + 1;
    }
    return (uint32_t)lo;
  }
};

// binning.rs:98-118
bool need_filter(const std::vector<int32_t>& cnt, int32_t total, int32_t filter_cnt, int32_t bin_type) {
  if (bin_type == kNumerical) {
    int32_t left = 0;
    for (size_t i = 0; i + 1 < cnt.size(); ++i) {
      left += cnt[i];
      if (left >= filter_cnt && total - left >= filter_cnt) return false;
    }
    return true;
  }
  if (cnt.size() > 2) return false;
  for (size_t i = 0; i + 1 < cnt.size(); ++i)
    if (cnt[i] >= filter_cnt && total - cnt[i] >= filter_cnt) return false;
  return true;
}

// Appends `val` unless it lies within one ulp above the last bound
// (the repeated check of binning.rs:137-146, :200-208).
void push_bound(std::vector<double>& b, double val) {
  if (b.empty() || !(val <= next_up(b.back()))) b.push_back(val);
}

// binning.rs:121-212
std::vector<double> greedy_find_bin(const double* dv, const int32_t* cnt, size_t ndv, int32_t max_bin, size_t total,
                                    int32_t min_data_in_bin) {
  std::vector<double> out;
  if (ndv == 0) return {std::numeric_limits<double>::infinity()};
  if ((int64_t)ndv <= max_bin) {
    int32_t cur = 0;
    for (size_t i = 0; i + 1 < ndv; ++i) {
      cur += cnt[i];
      if (cur >= min_data_in_bin) {
        const double val = next_up((dv[i] + dv[i + 1]) / 2.0);
        const size_t before = out.size();
        push_bound(out, val);
        if (out.size() != before) cur = 0;
      }
    }
    out.push_back(std::numeric_limits<double>::infinity());
    return out;
  }
  if (min_data_in_bin > 0) {
    max_bin = std::min(max_bin, (int32_t)(total / (size_t)min_data_in_bin));
    max_bin = std::max(max_bin, 1);
  }
  double mean = (double)total / (double)max_bin;
  int32_t rest_bins = max_bin;
  int32_t rest_cnt = (int32_t)total;
  std::vector<char> big(ndv, 0);
  for (size_t i = 0; i < ndv; ++i) {
    if ((double)cnt[i] >= mean) {
      big[i] = 1;
      rest_bins -= 1;
      rest_cnt -= cnt[i];
    }
  }
  mean = (double)rest_cnt / (double)rest_bins;
  std::vector<double> ub((size_t)max_bin, std::numeric_limits<double>::infinity());
  std::vector<double> lb((size_t)max_bin, std::numeric_limits<double>::infinity());
  int32_t nb = 0;
  lb[0] = dv[0];
  int32_t cur = 0;
  for (size_t i = 0; i + 1 < ndv; ++i) {
    if (!big[i]) rest_cnt -= cnt[i];
    cur += cnt[i];
    const double half = std::max(mean * (double)0.5f, 1.0);
    if (big[i] || (double)cur >= mean || (big[i + 1] && (double)cur >= half)) {
      ub[(size_t)nb] = dv[i];
      ++nb;
      lb[(size_t)nb] = dv[i + 1];
      if (nb >= max_bin - 1) break;
      cur = 0;
      if (!big[i]) {
        rest_bins -= 1;
        mean = (double)rest_cnt / (double)rest_bins;
      }
    }
  }
  ++nb;
  for (int32_t i = 0; i + 1 < nb; ++i) push_bound(out, next_up((ub[(size_t)i] + lb[(size_t)i + 1]) / 2.0));
  out.push_back(std::numeric_limits<double>::infinity());
  return out;
}

// binning.rs:214-275
std::vector<double> zero_as_one_bin(const std::vector<double>& dv, const std::vector<int32_t>& cnt, int32_t max_bin,
                                    size_t total, int32_t min_data_in_bin) {
  const size_t n = dv.size();
  std::vector<double> out;
  int32_t left_data = 0, zeros = 0, right_data = 0;
  for (size_t i = 0; i < n; ++i) {
    if (dv[i] <= -kZeroThreshold) left_data += cnt[i];
    else if (dv[i] > kZeroThreshold) right_data += cnt[i];
    else zeros += cnt[i];
  }
  size_t left_cnt = n;
  for (size_t i = 0; i < n; ++i)
    if (dv[i] > -kZeroThreshold) {
      left_cnt = i;
      break;
    }
  if (left_cnt > 0 && max_bin > 1) {
    // total - zeros as an unsigned difference, as the reference computes it
    const double denom = (double)(size_t)(total - (size_t)zeros);
    int32_t left_max = (int32_t)((double)left_data / denom * (double)(max_bin - 1));
    left_max = std::max(left_max, 1);
    out = greedy_find_bin(dv.data(), cnt.data(), left_cnt, left_max, (size_t)left_data, min_data_in_bin);
    if (!out.empty()) out.back() = -kZeroThreshold;
  }
  size_t right_start = n;
  for (size_t i = left_cnt; i < n; ++i)
    if (dv[i] > kZeroThreshold) {
      right_start = i;
      break;
    }
  const int32_t right_max = max_bin - 1 - (int32_t)out.size();
  if (right_start < n && right_max > 0) {
    std::vector<double> r = greedy_find_bin(dv.data() + right_start, cnt.data() + right_start, n - right_start,
                                            right_max, (size_t)right_data, min_data_in_bin);
    out.push_back(kZeroThreshold);
    out.insert(out.end(), r.begin(), r.end());
  } else {
    out.push_back(std::numeric_limits<double>::infinity());
  }
  return out;
}

// binning.rs:596-622
void finish(Mapper& m, const std::vector<int32_t>& cnt_in_bin, size_t total, const BinParams& p) {
  m.is_trivial = m.num_bin <= 1;
  if (!m.is_trivial && p.pre_filter && need_filter(cnt_in_bin, (int32_t)total, p.min_split_data, m.bin_type))
    m.is_trivial = true;
  if (m.is_trivial) return;
  m.default_bin = m.value_to_bin(0.0);
  size_t arg_max = 0;
  for (size_t i = 1; i < cnt_in_bin.size(); ++i)
    if (cnt_in_bin[i] > cnt_in_bin[arg_max]) arg_max = i;
  m.most_freq_bin = (uint32_t)arg_max;
  const double rate = (double)cnt_in_bin[arg_max] / (double)total;
  if (m.most_freq_bin != m.default_bin && rate < kSparseThreshold) m.most_freq_bin = m.default_bin;
}

// binning.rs:517-592
void finish_categorical(Mapper& m, const std::vector<double>& dv, const std::vector<int32_t>& cnt, int32_t na_cnt,
                        size_t total, const BinParams& p) {
  std::vector<int32_t> vals, counts;
  for (size_t i = 0; i < dv.size(); ++i) {
    const int32_t v = (int32_t)dv[i];
    if (v < 0) {
      na_cnt += cnt[i];
    } else if (vals.empty() || vals.back() != v) {
      vals.push_back(v);
      counts.push_back(cnt[i]);
    } else {
      counts.back() += cnt[i];
    }
  }
  std::vector<int32_t> cnt_in_bin;
  const int32_t rest = (int32_t)((int64_t)total - (int64_t)na_cnt);
  if (rest > 0) {
    // stable by count, descending (Common::SortForPair with is_reverse)
    std::vector<size_t> order(vals.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return counts[a] > counts[b]; });
    // RoundInt((total - na_cnt) * 0.99f) with a float product
    const int32_t cut = (int32_t)((double)((float)(size_t)(total - (size_t)na_cnt) * 0.99f) + (double)0.5f);
    int32_t distinct = (int32_t)vals.size() + (na_cnt > 0 ? 1 : 0);
    const int32_t max_bin = std::min(distinct, p.max_bin);
    m.bin_2_cat.push_back(-1);
    m.cat_2_bin[-1] = 0;
    cnt_in_bin.push_back(0);
    m.num_bin = 1;
    int32_t used = 0;
    size_t k = 0;
    while (k < order.size() && (used < cut || m.num_bin < max_bin)) {
      const size_t j = order[k];
      if (counts[j] < p.min_data_in_bin && k > 1) break;
      m.bin_2_cat.push_back(vals[j]);
      m.cat_2_bin[vals[j]] = (uint32_t)m.num_bin;
      used += counts[j];
      cnt_in_bin.push_back(counts[j]);
      m.num_bin += 1;
      ++k;
    }
    m.missing_type = (k == order.size() && na_cnt == 0) ? kMissingNone : kMissingNaN;
    cnt_in_bin[0] = (int32_t)((int64_t)total - (int64_t)used);
  }
  finish(m, cnt_in_bin, total, p);
}

// binning.rs:401-515 (no forced bounds)
Mapper find_bin(std::vector<double> vals_in, size_t total, int32_t bin_type, const BinParams& p) {
  const int32_t n_in = (int32_t)vals_in.size();
  std::vector<double> vals;
  for (double v : vals_in)
    if (!std::isnan(v)) vals.push_back(v);
  const int32_t non_na = (int32_t)vals.size();
  int32_t na_cnt = 0;
  int32_t missing;
  if (!p.use_missing) missing = kMissingNone;
  else if (p.zero_as_missing) missing = kMissingZero;
  else if (non_na == n_in) missing = kMissingNone;
  else {
    na_cnt = n_in - non_na;
    missing = kMissingNaN;
  }
  const int32_t zero_cnt = (int32_t)((int64_t)total - (int64_t)non_na - (int64_t)na_cnt);
  std::stable_sort(vals.begin(), vals.end());
  std::vector<double> dv;
  std::vector<int32_t> cnt;
  if (non_na == 0 || (vals[0] > 0.0 && zero_cnt > 0)) {
    dv.push_back(0.0);
    cnt.push_back(zero_cnt);
  }
  if (non_na > 0) {
    dv.push_back(vals[0]);
    cnt.push_back(1);
  }
  for (int32_t i = 1; i < non_na; ++i) {
    if (!(vals[(size_t)i] <= next_up(vals[(size_t)i - 1]))) {
      if (vals[(size_t)i - 1] < 0.0 && vals[(size_t)i] > 0.0) {
        dv.push_back(0.0);
        cnt.push_back(zero_cnt);
      }
      dv.push_back(vals[(size_t)i]);
      cnt.push_back(1);
    } else {
      dv.back() = vals[(size_t)i];
      cnt.back() += 1;
    }
  }
  if (non_na > 0 && vals[(size_t)non_na - 1] < 0.0 && zero_cnt > 0) {
    dv.push_back(0.0);
    cnt.push_back(zero_cnt);
  }
  Mapper m;
  m.min_val = dv.front();
  m.max_val = dv.back();
  m.missing_type = missing;
  if (bin_type == kCategorical) {
    m.bin_type = kCategorical;
    m.upper = {std::numeric_limits<double>::infinity()};
    finish_categorical(m, dv, cnt, na_cnt, total, p);
    return m;
  }
  std::vector<double> b;
  if (missing == kMissingZero) {
    b = zero_as_one_bin(dv, cnt, p.max_bin, total, p.min_data_in_bin);
    if (b.size() == 2) m.missing_type = kMissingNone;
  } else if (missing == kMissingNone) {
    b = zero_as_one_bin(dv, cnt, p.max_bin, total, p.min_data_in_bin);
  } else {
    b = zero_as_one_bin(dv, cnt, p.max_bin - 1, total - (size_t)na_cnt, p.min_data_in_bin);
    b.push_back(std::numeric_limits<double>::quiet_NaN());
  }
  m.num_bin = (int32_t)b.size();
  m.upper = b;
  std::vector<int32_t> cnt_in_bin((size_t)m.num_bin, 0);
  size_t ib = 0;
  for (size_t i = 0; i < dv.size(); ++i) {
    while (dv[i] > m.upper[ib] && (int32_t)ib < m.num_bin - 1) ++ib;  // a NaN bound compares false
    cnt_in_bin[ib] += cnt[i];
  }
  if (m.missing_type == kMissingNaN) cnt_in_bin[(size_t)m.num_bin - 1] = na_cnt;
  finish(m, cnt_in_bin, total, p);
  return m;
}

// %.17g, as the reference's fmt_g17 (fmt.rs) prints a double
std::string g17(double v) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.17g", v);
  return buf;
}

}  // namespace

struct Dataset {
  int64_t num_data = 0;
  int32_t num_total = 0;
  std::vector<Mapper> all;     // every column
  std::vector<int32_t> used;   // non-trivial columns, in column order
  std::vector<uint8_t> bins;   // row-major [num_data x used.size()] stored group values
  // the OracleData view
  std::vector<int32_t> num_bin, missing_type, default_bin, most_freq_bin, bin_type, real_index;
  std::vector<double> upper_bounds;
  std::vector<int64_t> ub_offsets, cat_offsets;
  std::vector<int32_t> bin_to_cat;
  std::string infos;

  void push_rows(const float* X) {
    const size_t nf = used.size();
    bins.assign((size_t)num_data * nf, 0);
    for (int64_t r = 0; r < num_data; ++r) {
      for (size_t f = 0; f < nf; ++f) {
        const Mapper& m = all[(size_t)used[f]];
        const uint32_t b = m.value_to_bin((double)X[(size_t)r * (size_t)num_total + (size_t)used[f]]);
        // feature_group.rs:144-154, one feature per group: the most frequent
        // bin is not pushed (stored 0); bin b is stored as b - (mfb == 0) + 1
        bins[(size_t)r * nf + f] = b == m.most_freq_bin ? 0 : (uint8_t)(b - (m.most_freq_bin == 0 ? 1u : 0u) + 1u);
      }
    }
  }

  void make_view() {
    num_bin.clear();
    missing_type.clear();
    default_bin.clear();
    most_freq_bin.clear();
    bin_type.clear();
    real_index.clear();
    upper_bounds.clear();
    bin_to_cat.clear();
    ub_offsets.assign(1, 0);
    cat_offsets.assign(1, 0);
    for (int32_t c : used) {
      const Mapper& m = all[(size_t)c];
      num_bin.push_back(m.num_bin);
      missing_type.push_back(m.missing_type);
      default_bin.push_back((int32_t)m.default_bin);
      most_freq_bin.push_back((int32_t)m.most_freq_bin);
      bin_type.push_back(m.bin_type);
      real_index.push_back(c);
      if (m.bin_type == kNumerical) upper_bounds.insert(upper_bounds.end(), m.upper.begin(), m.upper.end());
      else bin_to_cat.insert(bin_to_cat.end(), m.bin_2_cat.begin(), m.bin_2_cat.end());
      ub_offsets.push_back((int64_t)upper_bounds.size());
      cat_offsets.push_back((int64_t)bin_to_cat.size());
    }
    // dataset.rs:770-776 feature_infos, with bin_info_string (binning.rs:680-686)
    infos.clear();
    for (int32_t c = 0; c < num_total; ++c) {
      const Mapper& m = all[(size_t)c];
      if (c) infos += ' ';
      if (m.is_trivial) {
        infos += "none";
      } else if (m.bin_type == kCategorical) {
        for (size_t i = 0; i < m.bin_2_cat.size(); ++i) {
          if (i) infos += ':';
          infos += std::to_string(m.bin_2_cat[i]);
        }
      } else {
        infos += "[" + g17(m.min_val) + ":" + g17(m.max_val) + "]";
      }
    }
  }
};

}  // namespace oracle

using namespace oracle;

struct OracleDataset : oracle::Dataset {};

extern "C" {

int oracle_dataset_create(const float* X, int64_t n, int32_t ncol, const OracleBinParams* bp, OracleDataset** out) {
  ORACLE_TRY({
    if (!X || !bp || !out || n <= 0 || ncol <= 0 || n > INT32_MAX) throw std::runtime_error("bad argument");
    auto d = std::make_unique<OracleDataset>();
    d->num_data = n;
    d->num_total = ncol;
    std::vector<char> is_cat((size_t)ncol, 0);
    for (int32_t i = 0; i < bp->num_categorical; ++i)
      if (bp->categorical[i] >= 0 && bp->categorical[i] < ncol) is_cat[(size_t)bp->categorical[i]] = 1;
    // dataset.rs:394-396: sample_cnt = min(n, max(bin_construct_sample_cnt, 0)) rows by Random::sample
    const int32_t k = (int32_t)std::min<int64_t>(n, std::max(bp->bin_construct_sample_cnt, 0));
    Random rnd(bp->data_random_seed);
    const std::vector<int32_t> sample = rnd.sample((int32_t)n, k);
    const size_t total = sample.size();
    BinParams p;
    p.max_bin = bp->max_bin;
    p.min_data_in_bin = bp->min_data_in_bin;
    p.min_split_data = (int32_t)((double)bp->min_data_in_leaf * (double)total / (double)n);  // dataset.rs:871
    p.pre_filter = bp->feature_pre_filter != 0;
    p.use_missing = bp->use_missing != 0;
    p.zero_as_missing = bp->zero_as_missing != 0;
    std::vector<std::vector<double>> cols((size_t)ncol);
    for (int32_t c = 0; c < ncol; ++c) {
      std::vector<double>& v = cols[(size_t)c];
      for (int32_t r : sample) {  // matrix.rs:198-214: keep |v| > kZeroThreshold or NaN
        const double x = (double)X[(size_t)r * (size_t)ncol + (size_t)c];
        if (std::fabs(x) > kZeroThreshold || std::isnan(x)) v.push_back(x);
      }
      d->all.push_back(find_bin(v, total, is_cat[(size_t)c] ? kCategorical : kNumerical, p));
    }
    for (int32_t c = 0; c < ncol; ++c)
      if (!d->all[(size_t)c].is_trivial) d->used.push_back(c);
    // exclusive feature bundling would leave every feature in its own dense
    // group: each is dense (>= 40% of the sample off its most frequent bin)
    // and no two fit together within the allowed conflicts
    // (feature_groups.rs:21-42, :66-156)
    std::vector<size_t> nz;
    for (int32_t c : d->used) {
      const Mapper& m = d->all[(size_t)c];
      size_t cnt = cols[(size_t)c].size();
      if (m.default_bin != m.most_freq_bin) {
        cnt = total - cols[(size_t)c].size();
        for (double v : cols[(size_t)c])
          if (m.value_to_bin(v) != m.most_freq_bin) cnt += 1;
      }
      if ((double)cnt / (double)total < 0.4) throw std::runtime_error("sparse feature: would form a multi-value group");
      nz.push_back(cnt);
    }
    if (nz.size() >= 2) {
      std::sort(nz.begin(), nz.end());
      if (nz[0] + nz[1] <= total + total / 10000) throw std::runtime_error("features would be bundled");
    }
    d->push_rows(X);
    d->make_view();
    *out = d.release();
  });
}

int oracle_dataset_create_valid(const float* X, int64_t n, int32_t ncol, const OracleDataset* ref,
                                OracleDataset** out) {
  ORACLE_TRY({
    if (!X || !ref || !out || n <= 0 || ncol != ref->num_total) throw std::runtime_error("bad argument");
    auto d = std::make_unique<OracleDataset>();
    d->num_data = n;
    d->num_total = ncol;
    d->all = ref->all;
    d->used = ref->used;
    d->push_rows(X);
    d->make_view();
    *out = d.release();
  });
}

int oracle_dataset_view(OracleDataset* d, OracleData* v, int32_t* num_total_features) {
  ORACLE_TRY({
    v->num_data = d->num_data;
    v->num_features = (int32_t)d->used.size();
    v->bins = d->bins.data();
    v->num_bin = d->num_bin.data();
    v->missing_type = d->missing_type.data();
    v->default_bin = d->default_bin.data();
    v->most_freq_bin = d->most_freq_bin.data();
    v->bin_type = d->bin_type.data();
    v->real_index = d->real_index.data();
    v->monotone = nullptr;
    v->upper_bounds = d->upper_bounds.data();
    v->ub_offsets = d->ub_offsets.data();
    v->bin_to_cat = d->bin_to_cat.data();
    v->cat_offsets = d->cat_offsets.data();
    if (num_total_features) *num_total_features = d->num_total;
  });
}

const char* oracle_dataset_feature_infos(OracleDataset* d) { return d ? d->infos.c_str() : ""; }

void oracle_dataset_free(OracleDataset* d) { delete d; }

}  // extern "C"
