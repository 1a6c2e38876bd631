// Lambdarank gradients on the device (objective/rank.rs:119-262): the
// tables the objective builds once, and the launch.
#pragma once
#include "learner_impl.h"

namespace lgbm_b200 {

constexpr int kRankSigmoidBins = 1024 * 1024;  // rank.rs sigmoid table size
constexpr int kRankMaxQuery = 10000;           // rows per query (size of the discount table)

// Device view of the objective's tables.
struct DRank {
  const int32_t* bnd;          // query boundaries [nq + 1]
  int32_t nq;
  const double* inv_max_dcg;   // [nq]
  const double* sigmoid_table; // [kRankSigmoidBins]
  const double* label_gain;    // [31]
  const double* discount;      // [kRankMaxQuery]
  uint32_t* sorted;            // [n] per query: positions in descending score order
  double* sorted_score;        // [n] the query's scores in that order
  float* sorted_label;         // [n] the query's labels in that order
  double sigmoid, min_in, max_in, idx_factor;
  int32_t truncation_level;
  int32_t norm;
};

// Host owner of the tables (built from the labels and query boundaries once).
struct RankTables {
  DeviceArena arena;
  DRank d{};
  int32_t nq = 0;
  Status build(const float* label_h, const int32_t* bnd_h, int32_t nq, double sigmoid, int32_t trunc, bool norm);
  ~RankTables() { arena.free_all(); }
};

Status launch_lambdarank(const DRank& r, const float* label, const double* score, float* g, float* h, float2* gh,
                         int sms, cudaStream_t s);
// NDCG@ks[j] of every query into out[q * nk + j] (device buffers).
Status launch_ndcg(const DRank& r, const float* label, const double* score, const int32_t* ks, int32_t nk,
                   double* out, int sms, cudaStream_t s);

}  // namespace lgbm_b200
