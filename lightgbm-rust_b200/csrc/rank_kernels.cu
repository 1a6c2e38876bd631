// LambdarankNDCG gradients (crates/lgbm-core/src/objective/rank.rs:119-262,
// RankingBase::gradients :63-111) on the device.
//
// Two launches per call:
//   k_rank_sort    one CTA per query (grid-stride): the stable descending
//                  order of the query's scores (dcg.rs:167-179) by rank
//                  counting in shared memory, with the scores and labels
//                  written out in that order
//   k_lambdarank   one warp per query. The reference's pair loop (outer
//                  position i below the truncation level, inner j > i) adds
//                  to the row at position p first the pairs (i, p) for
//                  i < p in order of i, then, when p itself is an outer
//                  position, the pairs (p, j) in order of j. Lane l takes
//                  the positions l, l + 32, ... and adds exactly those pairs
//                  in that order in registers, so every f32 lambda and
//                  hessian is formed as on the CPU. The FP64 sum of the
//                  lambdas (for the normalisation) is one sequential chain
//                  in the loop's order: the lanes compute 32 consecutive
//                  pair values at a time and lane 0 subtracts them in order
//                  (a skipped pair adds +0.0, which changes no sum).
// The tables the reference builds in its constructor (label gains,
// discounts, inverse max DCG per query, the 2^20-entry sigmoid table) are
// built on the host by the same arithmetic and uploaded once.
#include "rank.h"

namespace lgbm_b200 {

constexpr double kMinScoreD = -INFINITY;  // consts.rs kMinScore
constexpr int kRankSortThreads = 128;
constexpr int kRankSmemScores = 2048;  // queries up to this size sort from shared memory

// Strict total order of the sort: larger score first, equal scores by
// position (a stable sort); a NaN score orders after every number.
__device__ __forceinline__ bool precedes(double sj, int j, double si, int i) {
  const bool nj = isnan(sj), ni = isnan(si);
  if (nj != ni) return ni;  // the number precedes the NaN
  if (!nj && sj != si) return sj > si;
  return j < i;
}

__global__ void __launch_bounds__(kRankSortThreads) k_rank_sort(DRank r, const double* score, const float* label) {
  __shared__ double s[kRankSmemScores];
  for (int32_t q = blockIdx.x; q < r.nq; q += gridDim.x) {
    const int32_t b0 = r.bnd[q], cnt = r.bnd[q + 1] - b0;
    const double* sc = score + b0;
    const bool in_smem = cnt <= kRankSmemScores;
    __syncthreads();
    if (in_smem)
      for (int i = threadIdx.x; i < cnt; i += blockDim.x) s[i] = sc[i];
    __syncthreads();
    const double* src = in_smem ? s : sc;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const double si = src[i];
      int32_t rank = 0;
      for (int j = 0; j < cnt; ++j) rank += precedes(src[j], j, si, i) ? 1 : 0;
      r.sorted[b0 + rank] = (uint32_t)i;
      r.sorted_score[b0 + rank] = si;
      r.sorted_label[b0 + rank] = label[b0 + i];
    }
  }
}

__device__ __forceinline__ double rank_sigmoid(const DRank& r, double score) {  // rank.rs:178-186
  if (score <= r.min_in) return r.sigmoid_table[0];
  if (score >= r.max_in) return r.sigmoid_table[kRankSigmoidBins - 1];
  return r.sigmoid_table[(size_t)((score - r.min_in) * r.idx_factor)];
}

// One query's sorted scores and labels and the values its pairs share.
struct QueryView {
  const double* ssc;
  const float* slb;
  double inverse_max_dcg;
  bool scale_by_score;  // norm and best_score != worst_score (rank.rs:231-233)
};

__device__ __forceinline__ QueryView query_view(const DRank& r, int32_t q, int32_t b0, int32_t cnt) {
  QueryView v;
  v.ssc = r.sorted_score + b0;
  v.slb = r.sorted_label + b0;
  v.inverse_max_dcg = r.inv_max_dcg[q];
  const double best_score = v.ssc[0];
  int32_t worst_idx = cnt - 1;
  if (worst_idx > 0 && v.ssc[worst_idx] == kMinScoreD) worst_idx -= 1;
  v.scale_by_score = r.norm && best_score != v.ssc[worst_idx];
  return v;
}

// The pair of sorted positions a < b (labels la != lb, neither score the
// minimum): its lambda and hessian by the reference's FP64 operations
// (rank.rs:217-252), and whether a is the higher-labelled of the two. Both
// rows of a pair evaluate the same operations, so they get the same values.
__device__ __forceinline__ void pair_value(const DRank& r, const QueryView& v, int32_t a, int32_t b, float la,
                                           float lb, double& p_lambda, double& p_hessian, bool& a_high) {
  a_high = la > lb;
  const int32_t high_rank = a_high ? a : b, low_rank = a_high ? b : a;
  const double high_score = v.ssc[high_rank], low_score = v.ssc[low_rank];
  const double high_label_gain = r.label_gain[(int32_t)(a_high ? la : lb)];
  const double low_label_gain = r.label_gain[(int32_t)(a_high ? lb : la)];
  const double high_discount = r.discount[high_rank], low_discount = r.discount[low_rank];
  const double delta_score = high_score - low_score;
  const double dcg_gap = high_label_gain - low_label_gain;
  const double paired_discount = fabs(high_discount - low_discount);
  double delta_pair_ndcg = dcg_gap * paired_discount * v.inverse_max_dcg;
  if (v.scale_by_score) delta_pair_ndcg /= (double)0.01f + fabs(delta_score);
  double pl = rank_sigmoid(r, delta_score);
  double ph = pl * (1.0 - pl);
  pl *= -r.sigmoid * delta_pair_ndcg;
  ph *= r.sigmoid * r.sigmoid * delta_pair_ndcg;
  p_lambda = pl;
  p_hessian = ph;
}

constexpr int kRankWarps = 8;  // queries per CTA (one warp each)

// LambdarankNDCG::one_query (rank.rs:192-262) for every query, one warp
// each. Writes g/h (class-major float arrays) and/or the interleaved pairs.
__global__ void __launch_bounds__(kRankWarps * 32) k_lambdarank(DRank r, float* g, float* h, float2* gh) {
  __shared__ __align__(16) double chain[kRankWarps][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int32_t T = r.truncation_level;
  for (int64_t q = (int64_t)blockIdx.x * kRankWarps + wib; q < r.nq; q += (int64_t)gridDim.x * kRankWarps) {
    const int32_t b0 = r.bnd[q], cnt = r.bnd[q + 1] - b0;
    if (cnt == 0) continue;
    const QueryView v = query_view(r, (int32_t)q, b0, cnt);
    // every row's lambda and hessian, the pairs added in the reference's order
    for (int32_t p = lane; p < cnt; p += 32) {
      float acc_l = 0.0f, acc_h = 0.0f;
      const double sp = v.ssc[p];
      const float lp = v.slb[p];
      if (sp != kMinScoreD) {
        // as the inner position: the outer positions i < p (all i + 1 < cnt)
        const int32_t imax = min(p, T);
        for (int32_t i = 0; i < imax; ++i) {
          if (v.ssc[i] == kMinScoreD) continue;
          const float li = v.slb[i];
          if (li == lp) continue;
          double pl, ph;
          bool i_high;
          pair_value(r, v, i, p, li, lp, pl, ph, i_high);
          acc_l += i_high ? -(float)pl : (float)pl;  // the lower-labelled row takes -lambda
          acc_h += (float)ph;
        }
        // as the outer position
        if (p < T && p + 1 < cnt) {
          for (int32_t j = p + 1; j < cnt; ++j) {
            if (v.ssc[j] == kMinScoreD) continue;
            const float lj = v.slb[j];
            if (lj == lp) continue;
            double pl, ph;
            bool p_high;
            pair_value(r, v, p, j, lp, lj, pl, ph, p_high);
            acc_l += p_high ? (float)pl : -(float)pl;
            acc_h += (float)ph;
          }
        }
      }
      const uint32_t row = r.sorted[b0 + p];
      if (g) {
        g[b0 + row] = acc_l;
        h[b0 + row] = acc_h;
      } else {
        gh[b0 + row] = make_float2(acc_l, acc_h);
      }
    }
    if (!r.norm) continue;
    // sum_lambdas -= 2 p_lambda over the pairs in the loop's order (lane 0's chain)
    double sum_lambdas = 0.0;
    for (int32_t i = 0; i + 1 < cnt && i < T; ++i) {
      if (v.ssc[i] == kMinScoreD) continue;  // uniform over the warp
      const float li = v.slb[i];
      for (int32_t jb = i + 1; jb < cnt; jb += 32) {
        const int32_t j = jb + lane;
        double val = 0.0;
        if (j < cnt && v.ssc[j] != kMinScoreD && v.slb[j] != li) {
          double pl, ph;
          bool i_high;
          pair_value(r, v, i, j, li, v.slb[j], pl, ph, i_high);
          val = 2.0 * pl;
        }
        chain[wib][lane] = val;
        __syncwarp();
        if (lane == 0) {
          // all 32 in order: the slots past the query hold +0.0, which
          // changes no sum; unrolled, the loads go in pairs
#pragma unroll
          for (int32_t k = 0; k < 32; k += 2) {
            const double2 two = *reinterpret_cast<const double2*>(&chain[wib][k]);
            sum_lambdas -= two.x;
            sum_lambdas -= two.y;
          }
        }
        __syncwarp();
      }
    }
    sum_lambdas = __shfl_sync(0xffffffffu, sum_lambdas, 0);
    if (sum_lambdas > 0.0) {  // every lane's rows are written (the warp's stores are ordered by __syncwarp)
      __syncwarp();
      const double norm_factor = log2(1.0 + sum_lambdas) / sum_lambdas;
      for (int32_t x = lane; x < cnt; x += 32) {
        if (g) {
          g[b0 + x] = (float)((double)g[b0 + x] * norm_factor);
          h[b0 + x] = (float)((double)h[b0 + x] * norm_factor);
        } else {
          gh[b0 + x].x = (float)((double)gh[b0 + x].x * norm_factor);
          gh[b0 + x].y = (float)((double)gh[b0 + x].y * norm_factor);
        }
      }
    }
  }
}

// NDCG@k of every query (metric.rs:546-598, no query weights), one thread
// per query, with the additions in the reference's order: out[q * nk + j]
// (1.0 for every k when the query's best DCG at ks[0] is 0). `r.sorted`
// holds the stable descending order of the query's scores (k_rank_sort).
__global__ void __launch_bounds__(128) k_ndcg(DRank r, const float* label, const int32_t* ks, int32_t nk,
                                              double* out) {
  for (int32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < r.nq; q += gridDim.x * blockDim.x) {
    const int32_t b0 = r.bnd[q], cnt = r.bnd[q + 1] - b0;
    const float* lb = label + b0;
    const uint32_t* sorted = r.sorted + b0;
    double* o = out + (size_t)q * nk;
    // dcg.rs max_dcg_at_k for each k, from the label counts
    bool first_ok = true;
    for (int32_t j = 0; j < nk; ++j) {
      int32_t counts[31];
      for (int v = 0; v < 31; ++v) counts[v] = 0;
      for (int32_t i = 0; i < cnt; ++i) counts[(int32_t)lb[i]] += 1;
      int32_t top = 30;
      double v = 0.0;
      const int32_t kk = min(ks[j], cnt);
      for (int32_t i = 0; i < kk; ++i) {
        while (top > 0 && counts[top] <= 0) top -= 1;
        v += r.discount[i] * r.label_gain[top];
        counts[top] -= 1;
      }
      o[j] = v > 0.0 ? 1.0 / v : -1.0;  // the inverse for now
      if (j == 0) first_ok = o[0] > 0.0;
    }
    if (!first_ok) {
      for (int32_t j = 0; j < nk; ++j) o[j] = 1.0;
      continue;
    }
    double cur = 0.0;
    int32_t left = 0;
    for (int32_t j = 0; j < nk; ++j) {
      const int32_t kk = min(ks[j], cnt);
      for (int32_t i = left; i < kk; ++i) cur += r.label_gain[(int32_t)lb[sorted[i]]] * r.discount[i];
      o[j] = cur * o[j];
      left = kk;
    }
  }
}

Status launch_ndcg(const DRank& r, const float* label, const double* score, const int32_t* ks, int32_t nk,
                   double* out, int sms, cudaStream_t s) {
  if (r.nq == 0) return Status();
  const int sort_grid = (int)std::min<int64_t>(r.nq, (int64_t)sms * 16);
  k_rank_sort<<<sort_grid, kRankSortThreads, 0, s>>>(r, score, label);
  CU_LAUNCH();
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((r.nq + 127) / 128, (int64_t)sms * 16));
  k_ndcg<<<grid, 128, 0, s>>>(r, label, ks, nk, out);
  CU_LAUNCH();
  return Status();
}

Status RankTables::build(const float* label_h, const int32_t* bnd_h, int32_t nq_, double sigmoid, int32_t trunc,
                         bool norm) {
  nq = nq_;
  const int64_t n = bnd_h[nq];
  for (int32_t q = 0; q < nq; ++q)
    if (bnd_h[q + 1] < bnd_h[q]) return Status(LGBM_B200_ERR_INVALID_DATA, "query boundaries must not decrease");
  // dcg.rs: label gains 2^i - 1 and discounts 1 / log2(2 + i)
  std::vector<double> label_gain, discount;
  label_gain.push_back(0.0);
  for (int i = 1; i < 31; ++i) label_gain.push_back((double)((1 << i) - 1));
  for (int i = 0; i < kRankMaxQuery; ++i) discount.push_back(1.0 / std::log2(2.0 + (double)i));
  for (int64_t i = 0; i < n; ++i) {
    const float l = label_h[i];
    if (!(l >= 0.0f) || (int32_t)l >= (int32_t)label_gain.size())
      return Status(LGBM_B200_ERR_INVALID_DATA, "lambdarank labels must be integers in [0, 30]");
  }
  // inverse max DCG at the truncation level per query (rank.rs:140-156)
  std::vector<double> inv((size_t)nq);
  const size_t k = (size_t)std::max(trunc, 0);
  for (int32_t q = 0; q < nq; ++q) {
    const size_t cnt_q = (size_t)(bnd_h[q + 1] - bnd_h[q]);
    if (cnt_q > (size_t)kRankMaxQuery)
      return Status(LGBM_B200_ERR_UNSUPPORTED, "a query holds more than 10000 rows");
    std::vector<int32_t> cnt(label_gain.size(), 0);
    for (size_t i = 0; i < cnt_q; ++i) cnt[(int32_t)label_h[bnd_h[q] + i]] += 1;
    int32_t top = (int32_t)label_gain.size() - 1;
    double v = 0.0;
    for (size_t j = 0; j < std::min(k, cnt_q); ++j) {
      while (top > 0 && cnt[top] <= 0) top -= 1;
      if (top < 0) break;
      v += discount[j] * label_gain[top];
      cnt[top] -= 1;
    }
    inv[(size_t)q] = v > 0.0 ? 1.0 / v : v;
  }
  // the sigmoid table (rank.rs:162-176)
  double min_in = -50.0 / sigmoid / 2.0;
  double max_in = -min_in;
  double idx_factor = (double)kRankSigmoidBins / (max_in - min_in);
  std::vector<double> table((size_t)kRankSigmoidBins);
  for (size_t i = 0; i < (size_t)kRankSigmoidBins; ++i) {
    double score = (double)i / idx_factor + min_in;
    table[i] = 1.0 / (1.0 + std::exp(score * sigmoid));
  }
  arena.free_all();
  Status s;
  int32_t* bnd_d;
  double *inv_d, *table_d, *gain_d, *disc_d;
  uint32_t* sorted_d;
  double* sorted_score_d;
  float* sorted_label_d;
  const size_t n1 = (size_t)std::max<int64_t>(1, n);
  if (!(s = arena.alloc_n(&bnd_d, (size_t)nq + 1)).ok() || !(s = arena.alloc_n(&inv_d, std::max<size_t>(1, nq))).ok() ||
      !(s = arena.alloc_n(&table_d, table.size())).ok() || !(s = arena.alloc_n(&gain_d, label_gain.size())).ok() ||
      !(s = arena.alloc_n(&disc_d, discount.size())).ok() || !(s = arena.alloc_n(&sorted_d, n1)).ok() ||
      !(s = arena.alloc_n(&sorted_score_d, n1)).ok() || !(s = arena.alloc_n(&sorted_label_d, n1)).ok())
    return s;
  CU(cudaMemcpy(bnd_d, bnd_h, sizeof(int32_t) * ((size_t)nq + 1), cudaMemcpyHostToDevice));
  if (nq > 0) CU(cudaMemcpy(inv_d, inv.data(), sizeof(double) * nq, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(table_d, table.data(), sizeof(double) * table.size(), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(gain_d, label_gain.data(), sizeof(double) * label_gain.size(), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(disc_d, discount.data(), sizeof(double) * discount.size(), cudaMemcpyHostToDevice));
  d.bnd = bnd_d;
  d.nq = nq;
  d.inv_max_dcg = inv_d;
  d.sigmoid_table = table_d;
  d.label_gain = gain_d;
  d.discount = disc_d;
  d.sorted = sorted_d;
  d.sorted_score = sorted_score_d;
  d.sorted_label = sorted_label_d;
  d.sigmoid = sigmoid;
  d.min_in = min_in;
  d.max_in = max_in;
  d.idx_factor = idx_factor;
  d.truncation_level = trunc;
  d.norm = norm ? 1 : 0;
  return Status();
}

Status launch_lambdarank(const DRank& r, const float* label, const double* score, float* g, float* h, float2* gh,
                         int sms, cudaStream_t s) {
  if (r.nq == 0) return Status();
  const int sort_grid = (int)std::min<int64_t>(r.nq, (int64_t)sms * 16);
  k_rank_sort<<<sort_grid, kRankSortThreads, 0, s>>>(r, score, label);
  CU_LAUNCH();
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((r.nq + kRankWarps - 1) / kRankWarps, (int64_t)sms * 32));
  k_lambdarank<<<grid, kRankWarps * 32, 0, s>>>(r, g, h, gh);
  CU_LAUNCH();
  return Status();
}

}  // namespace lgbm_b200
