// Device-resident boosting (Gbdt::train_one_iter, crates/lgbm-core/src/boosting.rs:957-1130),
// the stand-alone objective gradients (RowObjective::gradients) and the
// batched predictor (predict.rs:231), behind the C ABI of include/lgbm_b200.h.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "learner_impl.h"
#include "rank.h"

using namespace lgbm_b200;

namespace lgbm_b200 {

// objective/*.rs boost_from_score for the supported objectives (first iteration only).
static double boost_from_score(const LgbmB200ObjectiveConfig& o, const std::vector<float>& label, int k) {
  const size_t n = label.size();
  if (o.objective == LGBM_B200_OBJ_BINARY) {  // binary.rs:129-154
    double suml = 0.0;
    for (size_t i = 0; i < n; ++i) suml += (double)(int32_t)(label[i] > 0.0f);
    double pavg = suml / (double)n;
    pavg = std::min(pavg, 1.0 - kEpsilon);
    pavg = std::max(pavg, kEpsilon);
    return std::log(pavg / ((double)1.0f - pavg)) / o.sigmoid;
  }
  if (o.objective == LGBM_B200_OBJ_REGRESSION) {  // regression.rs:123-139
    double suml = 0.0;
    for (size_t i = 0; i < n; ++i) suml += (double)label[i];
    return suml / (double)n;
  }
  if (o.objective == LGBM_B200_OBJ_MULTICLASS) {  // multiclass.rs:97-124, :156-158
    double c = 0.0;
    for (size_t i = 0; i < n; ++i) c += (int32_t)label[i] == k ? 1.0 : 0.0;
    return std::log(std::max(kEpsilon, c / (double)n));
  }
  return 0.0;
}

static Status launch_gradients(const LgbmB200ObjectiveConfig& o, const float* label, const double* score, int64_t n,
                               float2* gh, float* g, float* h, int sms, cudaStream_t s, const DRank* rank = nullptr) {
  int blocks = std::max(1, (int)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  switch (o.objective) {
    case LGBM_B200_OBJ_LAMBDARANK:
      if (!rank) return Status(LGBM_B200_ERR_INVALID_PARAMETER, "lambdarank needs query boundaries");
      return launch_lambdarank(*rank, label, score, g, h, gh, sms, s);
    case LGBM_B200_OBJ_BINARY: k_grad_binary<<<blocks, 256, 0, s>>>(label, score, n, o.sigmoid, gh, g, h); break;
    case LGBM_B200_OBJ_REGRESSION: k_grad_l2<<<blocks, 256, 0, s>>>(label, score, n, gh, g, h); break;
    case LGBM_B200_OBJ_MULTICLASS:
      k_grad_softmax<<<blocks, 256, 0, s>>>(label, score, n, o.num_class, gh, n, g, h);
      break;
    default: return Status(LGBM_B200_ERR_UNSUPPORTED, "objective not supported by the device gradients");
  }
  CU_LAUNCH();
  return Status();
}

// Tree::shrink / add_bias / as_constant on the host copy (tree.rs:303-348).
static void shrink(HostTree& t, double rate) {
  for (int i = 0; i < t.num_leaves - 1; ++i) {
    t.leaf_value[i] = maybe_round_to_zero_h(t.leaf_value[i] * rate);
    t.internal_value[i] = maybe_round_to_zero_h(t.internal_value[i] * rate);
  }
  int last = t.num_leaves - 1;
  t.leaf_value[last] = maybe_round_to_zero_h(t.leaf_value[last] * rate);
}
static void add_bias(HostTree& t, double v) {
  for (int i = 0; i < t.num_leaves - 1; ++i) {
    t.leaf_value[i] = maybe_round_to_zero_h(t.leaf_value[i] + v);
    t.internal_value[i] = maybe_round_to_zero_h(t.internal_value[i] + v);
  }
  int last = t.num_leaves - 1;
  t.leaf_value[last] = maybe_round_to_zero_h(t.leaf_value[last] + v);
}
static void as_constant(HostTree& t, double v, int32_t count) {
  HostTree c;
  c.num_leaves = 1;
  c.leaf_parent = {-1};
  c.leaf_value = {v};
  c.leaf_weight = {0.0};
  c.leaf_count = {count};
  c.leaf_depth = {0};
  c.cat_boundaries = {0};
  c.cat_boundaries_inner = {0};
  t = c;
}

}  // namespace lgbm_b200

struct LgbmB200Booster {
  LgbmB200Learner* L = nullptr;
  LgbmB200BoostConfig cfg{};
  int K = 1;
  int64_t n = 0, nv = 0;
  std::vector<float> label_h;
  float* label_d = nullptr;
  double* score = nullptr;        // [K x n]
  double* valid_score = nullptr;  // [K x nv]
  uint8_t* valid_bins = nullptr;
  int32_t valid_stride = 0;
  DeviceArena arena;
  std::vector<double> init_scores;
  std::vector<bool> class_need_train;
  int iter = 0;
  bool first = true;
  // bagging (sample_strategy.rs)
  bool bagging = false;
  uint32_t* rng = nullptr;
  uint8_t* in_bag = nullptr;
  uint32_t* bag = nullptr;
  uint32_t* oob = nullptr;
  int32_t* counts = nullptr;
  int32_t* block_in = nullptr;    // in-bag rows per 1024-row block
  int32_t* block_base = nullptr;  // in-bag rows of the blocks before each
  int32_t bag_cnt = 0, oob_cnt = 0;
  bool need_re_bagging = true;
  // column sampler (col_sampler.rs)
  std::unique_ptr<Lcg> col_rand;
  int32_t used_cnt_bytree = 0;
  std::vector<HostTree> out_trees;
  double* lv_dev = nullptr;  // [K x L] shrunk leaf values
  std::unique_ptr<RankTables> rank;  // lambdarank objective tables
  // by-tree feature masks: the last one sent per class, and pinned staging
  // (a mask is sent without a synchronisation, and only when it changes)
  std::vector<std::vector<uint8_t>> sent_mask;
  uint8_t* mask_h = nullptr;
  // one captured graph per iteration (gradients, quantization, the tree, the
  // score updates), recaptured when the learner's launch settings change
  bool iter_graph = true;
  cudaGraphExec_t iter_exec = nullptr;
  int iter_key = -1;
  ~LgbmB200Booster() {
    if (iter_exec) cudaGraphExecDestroy(iter_exec);
    arena.free_all();
    if (mask_h) cudaFreeHost(mask_h);
  }
};

namespace lgbm_b200 {

static Status booster_create(LgbmB200Booster* b, LgbmB200Learner* L, const LgbmB200BoostConfig* cfg,
                             const float* label, const int32_t* query_boundaries, int32_t num_queries,
                             const uint8_t* valid_bins, int64_t nv) {
  b->L = L;
  b->cfg = *cfg;
  b->K = L->K;
  b->n = L->n;
  b->nv = nv;
  CU(cudaSetDevice(L->device));
  const LgbmB200ObjectiveConfig& o = cfg->objective;
  int want_k = o.objective == LGBM_B200_OBJ_MULTICLASS ? o.num_class : 1;
  if (want_k != b->K)
    return Status(LGBM_B200_ERR_INVALID_PARAMETER, "learner num_tree_slots must equal the objective's tree count");
  const int64_t n = b->n;
  if (o.objective == LGBM_B200_OBJ_LAMBDARANK) {  // rank.rs:119-176: tables built once
    if (!query_boundaries || num_queries <= 0 || query_boundaries[0] != 0 || query_boundaries[num_queries] != n)
      return Status(LGBM_B200_ERR_INVALID_DATA, "lambdarank needs query boundaries covering every row");
    b->rank = std::make_unique<RankTables>();
    Status rs = b->rank->build(label, query_boundaries, num_queries, o.sigmoid, o.lambdarank_truncation_level,
                               o.lambdarank_norm != 0);
    if (!rs.ok()) return rs;
  }
  b->label_h.assign(label, label + n);
  DeviceArena& A = b->arena;
  Status s;
  if (!(s = A.alloc_n(&b->label_d, (size_t)n)).ok()) return s;
  CU(cudaMemcpy(b->label_d, label, sizeof(float) * n, cudaMemcpyHostToDevice));
  if (!(s = A.alloc_n(&b->score, (size_t)b->K * n)).ok()) return s;
  CU(cudaMemset(b->score, 0, sizeof(double) * b->K * n));
  if (nv > 0) {
    b->valid_stride = L->stride;
    if (!(s = A.alloc_n(&b->valid_bins, (size_t)nv * b->valid_stride)).ok()) return s;
    std::vector<uint8_t> padded((size_t)nv * b->valid_stride, 0);
    for (int64_t r = 0; r < nv; ++r)
      std::memcpy(&padded[(size_t)r * b->valid_stride], valid_bins + (size_t)r * L->nf, (size_t)L->nf);
    CU(cudaMemcpy(b->valid_bins, padded.data(), padded.size(), cudaMemcpyHostToDevice));
    if (!(s = A.alloc_n(&b->valid_score, (size_t)b->K * nv)).ok()) return s;
    CU(cudaMemset(b->valid_score, 0, sizeof(double) * b->K * nv));
  }
  if (!(s = A.alloc_n(&b->lv_dev, (size_t)b->K * L->L)).ok()) return s;
  b->init_scores.assign(b->K, 0.0);
  b->class_need_train.assign(b->K, true);
  if (o.objective == LGBM_B200_OBJ_MULTICLASS) {
    for (int k = 0; k < b->K; ++k) {
      double c = 0.0;
      for (int64_t i = 0; i < n; ++i) c += (int32_t)label[i] == k ? 1.0 : 0.0;
      double p = std::fabs(c / (double)n);
      b->class_need_train[k] = !(p <= kEpsilon || p >= 1.0 - kEpsilon);
      if (!b->class_need_train[k])
        return Status(LGBM_B200_ERR_UNSUPPORTED, "a class without rows (or with every row) in the device booster");
    }
  }
  b->bagging = cfg->bagging_fraction < 1.0 && cfg->bagging_freq > 0;
  if (b->bagging) {
    int64_t nb = (n + 1023) / 1024;
    std::vector<uint32_t> seeds((size_t)nb);
    for (int64_t i = 0; i < nb; ++i) seeds[(size_t)i] = (uint32_t)(cfg->bagging_seed + (int32_t)i);
    if (!(s = A.alloc_n(&b->rng, (size_t)nb)).ok()) return s;
    CU(cudaMemcpy(b->rng, seeds.data(), sizeof(uint32_t) * nb, cudaMemcpyHostToDevice));
    if (!(s = A.alloc_n(&b->in_bag, (size_t)n)).ok()) return s;
    if (!(s = A.alloc_n(&b->bag, (size_t)n)).ok()) return s;
    if (!(s = A.alloc_n(&b->oob, (size_t)n)).ok()) return s;
    if (!(s = A.alloc_n(&b->counts, 2)).ok()) return s;
    if (!(s = A.alloc_n(&b->block_in, (size_t)nb)).ok()) return s;
    if (!(s = A.alloc_n(&b->block_base, (size_t)nb)).ok()) return s;
    b->bag_cnt = (int32_t)n;
  }
  // LGBM_B200_ITER_GRAPH=0: every iteration runs launch by launch (each tree
  // still replays its own graph)
  if (const char* e = std::getenv("LGBM_B200_ITER_GRAPH")) b->iter_graph = std::atoi(e) != 0;
  b->col_rand = std::make_unique<Lcg>(cfg->feature_fraction_seed);
  int32_t total = L->nf;
  b->used_cnt_bytree = cfg->feature_fraction < 1.0
                           ? std::max(std::min(1, total), (int32_t)((double)total * cfg->feature_fraction + (double)0.5f))
                           : total;
  b->out_trees.resize(b->K);
  return Status();
}

// The shrunk leaf values of each slot's new tree (tree.rs shrinkage:
// round_to_zero(value * rate)), 0 for a tree of one leaf (no update).
// Grid (1, 1, slots).
__global__ void k_shrink_leaves(const __grid_constant__ DCtx c, double rate, double* lv, int32_t L) {
  const DSlot& s = c.slots[blockIdx.z];
  const int32_t nl = s.st->num_leaves_cur;
  for (int32_t l = threadIdx.x; l < L; l += blockDim.x)
    lv[(size_t)blockIdx.z * L + l] = (nl > 1 && l < nl) ? maybe_round_to_zero(s.tree.leaf_value[l] * rate) : 0.0;
}

// Score updates (boosting.rs:1381-1408) with the leaf values shrunk on the
// device, enqueued before the trees are read back.
static Status enqueue_score_updates(LgbmB200Booster* b) {
  LgbmB200Learner* L = b->L;
  cudaStream_t s = L->stream;
  const int K = b->K;
  const int64_t n = b->n;
  const int sms = L->num_sms;
  DCtx c = L->ctx;
  k_shrink_leaves<<<dim3(1, 1, K), 256, 0, s>>>(c, b->cfg.learning_rate, b->lv_dev, L->L);
  CU_LAUNCH();
  k_add_leaf_outputs<<<dim3(sms * 4, 1, K), 256, 16 * (size_t)L->L, s>>>(c, b->lv_dev, L->L, b->score, n);
  CU_LAUNCH();
  if (b->bagging && b->oob_cnt > 0) {
    k_add_tree_binned<<<dim3(std::max(1, (int)std::min<int64_t>((b->oob_cnt + 255) / 256, sms * 8)), 1, K), 256, 0,
                        s>>>(c, c.bins, c.stride, b->oob, b->oob_cnt, b->lv_dev, L->L, b->score, n);
    CU_LAUNCH();
  }
  if (b->nv > 0) {
    k_add_tree_binned<<<dim3(std::max(1, (int)std::min<int64_t>((b->nv + 255) / 256, sms * 8)), 1, K), 256, 0, s>>>(
        c, b->valid_bins, b->valid_stride, nullptr, b->nv, b->lv_dev, L->L, b->valid_score, b->nv);
    CU_LAUNCH();
  }
  return Status();
}

// One iteration's device work after the masks and the quantization offsets
// are staged: gradients, quantization, the tree's launches and the score
// updates. No launch carries a value that changes between iterations, so the
// sequence is captured once and replayed.
static Status enqueue_iteration(LgbmB200Booster* b) {
  LgbmB200Learner* L = b->L;
  Status st = launch_gradients(b->cfg.objective, b->label_d, b->score, b->n, L->gh_all, nullptr, nullptr, L->num_sms,
                               L->stream, b->rank ? &b->rank->d : nullptr);
  if (!st.ok()) return st;
  if (L->cfg.hist_precision == LGBM_B200_HIST_QUANT && !(st = enqueue_quant(L)).ok()) return st;
  if (!(st = enqueue_tree(L)).ok()) return st;
  return enqueue_score_updates(b);
}

static Status booster_iter(LgbmB200Booster* b, int32_t* stop) {
  LgbmB200Learner* L = b->L;
  CU(cudaSetDevice(L->device));
  cudaStream_t s = L->stream;
  const int K = b->K;
  const int64_t n = b->n;
  const int sms = L->num_sms;
  const int blocks = std::max(1, (int)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  std::vector<double> init(K, 0.0);
  if (b->first && b->cfg.boost_from_average) {  // boosting.rs:480-509
    for (int k = 0; k < K; ++k) {
      double v = boost_from_score(b->cfg.objective, b->label_h, k);
      if (std::fabs(v) > kEpsilon) {
        k_add_const<<<blocks, 256, 0, s>>>(b->score + (size_t)k * n, n, v);
        CU_LAUNCH();
        if (b->nv > 0) {
          k_add_const<<<blocks, 256, 0, s>>>(b->valid_score + (size_t)k * b->nv, b->nv, v);
          CU_LAUNCH();
        }
        init[k] = v;
      }
    }
    b->init_scores = init;
  }
  // the first iteration (boost from average, constant trees) and bagged ones
  // (the bag size is read back mid-iteration) run launch by launch; the others
  // replay one captured graph
  const bool graphed = b->iter_graph && !b->first && !b->bagging && L->cfg.use_cuda_graph &&
                       !L->cfg.persistent_grow && !L->timing;
  Status st;
  if (!graphed) {
    st = launch_gradients(b->cfg.objective, b->label_d, b->score, n, L->gh_all, nullptr, nullptr, sms, s,
                          b->rank ? &b->rank->d : nullptr);
    if (!st.ok()) return st;
  }
  // bagging (sample_strategy.rs:280-320)
  if (b->bagging && ((b->bag_cnt < n && b->iter % b->cfg.bagging_freq == 0) || b->need_re_bagging)) {
    b->need_re_bagging = false;
    int64_t nb = (n + 1023) / 1024;
    k_bagging<<<(unsigned)((nb + 127) / 128), 128, 0, s>>>(b->rng, n, b->cfg.bagging_fraction, b->in_bag,
                                                           b->block_in);
    CU_LAUNCH();
    k_bag_scan<<<1, 1024, 0, s>>>(b->block_in, (int32_t)nb, n, b->block_base, b->counts);
    CU_LAUNCH();
    k_bag_scatter<<<(unsigned)nb, 1024, 0, s>>>(b->in_bag, n, b->block_base, b->bag, b->oob);
    CU_LAUNCH();
    int32_t cnt[2];
    CU(cudaMemcpyAsync(cnt, b->counts, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    b->bag_cnt = cnt[0];
    b->oob_cnt = cnt[1];
    int rc = lgbm_b200_learner_set_bagging(L, b->bag, b->bag_cnt, LGBM_B200_DEVICE);
    if (rc != LGBM_B200_OK) return Status(rc, lgbm_b200_last_error());
  }
  // by-tree column samples, one per class tree (col_sampler.rs:88-96); the
  // staging is pinned and rewritten only after the iteration's final
  // synchronisation, so no copy waits
  if (!b->mask_h) CU(cudaHostAlloc(reinterpret_cast<void**>(&b->mask_h), (size_t)K * L->nf, cudaHostAllocDefault));
  b->sent_mask.resize((size_t)K);
  for (int k = 0; k < K; ++k) {
    std::vector<uint8_t> used((size_t)L->nf, 1);
    if (b->cfg.feature_fraction < 1.0) {
      std::fill(used.begin(), used.end(), 0);
      for (int32_t i : b->col_rand->sample(L->nf, b->used_cnt_bytree)) used[(size_t)i] = 1;
    }
    if (used != b->sent_mask[(size_t)k]) {
      uint8_t* h = b->mask_h + (size_t)k * L->nf;
      std::copy(used.begin(), used.end(), h);
      CU(cudaMemcpyAsync(L->slots_h[k].bytree, h, used.size(), cudaMemcpyHostToDevice, s));
      b->sent_mask[(size_t)k] = used;
    }
  }
  if (graphed) {
    // the offsets are drawn on the host and staged; the graph's copy reads them
    if (L->cfg.hist_precision == LGBM_B200_HIST_QUANT) draw_quant_starts(L, false);
    if (b->iter_exec == nullptr || b->iter_key != L->config_epoch) {
      if (b->iter_exec) {
        cudaGraphExecDestroy(b->iter_exec);
        b->iter_exec = nullptr;
      }
      cudaGraph_t g = nullptr;
      CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      st = enqueue_iteration(b);
      cudaError_t e = cudaStreamEndCapture(s, &g);
      if (!st.ok()) {
        if (g) cudaGraphDestroy(g);
        return st;
      }
      if (e != cudaSuccess) return Status(LGBM_B200_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&b->iter_exec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return Status(LGBM_B200_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
      b->iter_key = L->config_epoch;
    }
    CU(cudaGraphLaunch(b->iter_exec, s));
    L->trained = true;
    L->last_ms[0] = L->last_ms[1] = L->last_ms[2] = L->last_ms[3] = 0;
  } else {
    if (!(st = train_enqueue(L, nullptr, nullptr, LGBM_B200_DEVICE)).ok()) return st;
    if (!(st = enqueue_score_updates(b)).ok()) return st;
  }
  if (!(st = train_collect(L)).ok()) return st;  // synchronises
  bool should_continue = false;
  for (int k = 0; k < K; ++k) {
    HostTree& t = b->out_trees[k];
    t = L->trees[k];
    if (t.num_leaves > 1) {
      should_continue = true;
      shrink(t, b->cfg.learning_rate);
    }
  }
  for (int k = 0; k < K; ++k) {
    HostTree& t = b->out_trees[k];
    if (t.num_leaves > 1) {
      if (std::fabs(b->init_scores[k]) > kEpsilon && b->first) add_bias(t, b->init_scores[k]);
    } else if (b->first) {
      as_constant(t, b->init_scores[k], (int32_t)n);
    } else {
      as_constant(t, 0.0, (int32_t)n);
    }
  }
  b->first = false;
  *stop = should_continue ? 0 : 1;
  if (should_continue) b->iter += 1;
  return Status();
}

// ---- stand-alone gradients with a cached per-device workspace -----------------------------
struct GradWorkspace {
  std::mutex mu;
  int device = -1;
  cudaStream_t stream = nullptr;
  ChunkStreams chunks;  // row chunks of the elementwise objectives
  DeviceArena arena;
  size_t cap = 0;       // values (rows x classes) of score, g and h
  size_t cap_rows = 0;  // rows of label
  float* label = nullptr;
  double* score = nullptr;
  float* g = nullptr;
  float* h = nullptr;
};
static GradWorkspace g_ws;

}  // namespace lgbm_b200

// ---- an objective bound to its labels (RowObjective::init, objective/mod.rs:50) -------------
struct LgbmB200Objective {
  LgbmB200ObjectiveConfig cfg{};
  int device = 0;
  int64_t n = 0;
  int k = 1;
  lgbm_b200::DeviceArena arena;
  float* label = nullptr;  // on the device for the objective's lifetime
  double* score = nullptr;  // staging of host scores [k x n]
  float* g = nullptr;
  float* h = nullptr;
  std::unique_ptr<lgbm_b200::RankTables> rank;
  cudaStream_t stream = nullptr;
  ChunkStreams chunks;
  ~LgbmB200Objective() {
    chunks.release();
    arena.free_all();
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" {

int lgbm_b200_gradients(const LgbmB200ObjectiveConfig* cfg, const float* label, const double* scores,
                        int64_t num_data, const int32_t* query_boundaries, int32_t num_queries, float* grad,
                        float* hess, int32_t location, int32_t device) {
  if (!cfg || !label || !scores || !grad || !hess || num_data <= 0)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  if (cudaSetDevice(device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  const int k = cfg->objective == LGBM_B200_OBJ_MULTICLASS ? cfg->num_class : 1;
  const size_t n = (size_t)num_data, nk = n * (size_t)k;
  // lambdarank: the objective's tables from the labels and host query boundaries
  std::unique_ptr<RankTables> rank;
  if (cfg->objective == LGBM_B200_OBJ_LAMBDARANK) {
    if (!query_boundaries || num_queries <= 0 || query_boundaries[0] != 0 ||
        query_boundaries[num_queries] != num_data)
      return fail(Status(LGBM_B200_ERR_INVALID_DATA, "lambdarank needs query boundaries covering every row"));
    std::vector<float> lh;
    const float* lp = label;
    if (location == LGBM_B200_DEVICE) {
      lh.resize(n);
      if (cudaMemcpy(lh.data(), label, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(Status(LGBM_B200_ERR_CUDA, "label copy"));
      lp = lh.data();
    }
    rank = std::make_unique<RankTables>();
    Status rs = rank->build(lp, query_boundaries, num_queries, cfg->sigmoid, cfg->lambdarank_truncation_level,
                            cfg->lambdarank_norm != 0);
    if (!rs.ok()) return fail(rs);
  }
  const DRank* rk = rank ? &rank->d : nullptr;
  if (location == LGBM_B200_DEVICE) {
    Status s = launch_gradients(*cfg, label, scores, num_data, nullptr, grad, hess, current_device_sms(), 0, rk);
    if (!s.ok()) return fail(s);
    cudaError_t e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
    return LGBM_B200_OK;
  }
  std::lock_guard<std::mutex> lock(g_ws.mu);
  GradWorkspace& w = g_ws;
  if (w.device != device) {
    w.arena.free_all();
    w.cap = 0;
    w.cap_rows = 0;
    if (w.stream) cudaStreamDestroy(w.stream);
    w.chunks.release();
    if (cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess || !w.chunks.init())
      return fail(Status(LGBM_B200_ERR_CUDA, "stream"));
    w.device = device;
  }
  // both capacities are checked: a call with more rows but fewer values than
  // an earlier multiclass one needs a larger label buffer
  if (w.cap < nk || w.cap_rows < n) {
    w.arena.free_all();
    const size_t rows = std::max(n, w.cap_rows), vals = std::max(nk, w.cap);
    Status s;
    if (!(s = w.arena.alloc_n(&w.label, rows)).ok() || !(s = w.arena.alloc_n(&w.score, vals)).ok() ||
        !(s = w.arena.alloc_n(&w.g, vals)).ok() || !(s = w.arena.alloc_n(&w.h, vals)).ok()) {
      w.cap = 0;
      w.cap_rows = 0;
      return fail(s);
    }
    w.cap = vals;
    w.cap_rows = rows;
  }
  cudaStream_t s = w.stream;
  if (k == 1 && (cfg->objective == LGBM_B200_OBJ_BINARY || cfg->objective == LGBM_B200_OBJ_REGRESSION)) {
    // one value per row: chunks of rows, each chunk's copies in, kernel and
    // copies out on one of three streams, so that copies in and out of
    // different chunks overlap
    cudaError_t e = cudaSuccess;
    const char* where = "";
    for (int64_t r0 = 0, c = 0; r0 < num_data && e == cudaSuccess; r0 += ChunkStreams::kRows, ++c) {
      const int64_t m = std::min<int64_t>(ChunkStreams::kRows, num_data - r0);
      cudaStream_t cs = w.chunks.s[c % ChunkStreams::kN];
      where = "labels in";
      e = cudaMemcpyAsync(w.label + r0, label + r0, sizeof(float) * m, cudaMemcpyHostToDevice, cs);
      if (e == cudaSuccess) {
        where = "scores in";
        e = cudaMemcpyAsync(w.score + r0, scores + r0, sizeof(double) * m, cudaMemcpyHostToDevice, cs);
      }
      if (e == cudaSuccess) {
        Status st = launch_gradients(*cfg, w.label + r0, w.score + r0, m, nullptr, w.g + r0, w.h + r0, current_device_sms(), cs, rk);
        if (!st.ok()) {
          w.chunks.sync();
          return fail(st);
        }
        where = "gradient launch";
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) {
        where = "gradients out";
        e = cudaMemcpyAsync(grad + r0, w.g + r0, sizeof(float) * m, cudaMemcpyDeviceToHost, cs);
      }
      if (e == cudaSuccess) e = cudaMemcpyAsync(hess + r0, w.h + r0, sizeof(float) * m, cudaMemcpyDeviceToHost, cs);
    }
    cudaError_t e2 = w.chunks.sync();
    if (e == cudaSuccess && e2 != cudaSuccess) {
      e = e2;
      where = "chunk sync";
    }
    if (e != cudaSuccess)
      return fail(Status(LGBM_B200_ERR_CUDA, std::string("gradients (") + where + "): " + cudaGetErrorString(e)));
    return LGBM_B200_OK;
  }
  cudaMemcpyAsync(w.label, label, sizeof(float) * n, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(w.score, scores, sizeof(double) * nk, cudaMemcpyHostToDevice, s);
  Status st = launch_gradients(*cfg, w.label, w.score, num_data, nullptr, w.g, w.h, current_device_sms(), s, rk);
  if (!st.ok()) return fail(st);
  cudaMemcpyAsync(grad, w.g, sizeof(float) * nk, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hess, w.h, sizeof(float) * nk, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  return LGBM_B200_OK;
}

int lgbm_b200_objective_create(const LgbmB200ObjectiveConfig* cfg, const float* label, int64_t num_data,
                               const int32_t* query_boundaries, int32_t num_queries, int32_t device,
                               LgbmB200Objective** out) {
  if (!cfg || !label || !out || num_data <= 0) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  if (cudaSetDevice(device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  auto o = std::make_unique<LgbmB200Objective>();
  o->cfg = *cfg;
  o->device = device;
  o->n = num_data;
  o->k = cfg->objective == LGBM_B200_OBJ_MULTICLASS ? std::max(1, cfg->num_class) : 1;
  if (cfg->objective == LGBM_B200_OBJ_LAMBDARANK) {
    if (!query_boundaries || num_queries <= 0 || query_boundaries[0] != 0 ||
        query_boundaries[num_queries] != num_data)
      return fail(Status(LGBM_B200_ERR_INVALID_DATA, "lambdarank needs query boundaries covering every row"));
    o->rank = std::make_unique<RankTables>();
    Status rs = o->rank->build(label, query_boundaries, num_queries, cfg->sigmoid, cfg->lambdarank_truncation_level,
                               cfg->lambdarank_norm != 0);
    if (!rs.ok()) return fail(rs);
  }
  const size_t n = (size_t)num_data, nk = n * (size_t)o->k;
  Status st;
  if (!(st = o->arena.alloc_n(&o->label, n)).ok() || !(st = o->arena.alloc_n(&o->score, nk)).ok() ||
      !(st = o->arena.alloc_n(&o->g, nk)).ok() || !(st = o->arena.alloc_n(&o->h, nk)).ok())
    return fail(st);
  if (cudaStreamCreateWithFlags(&o->stream, cudaStreamNonBlocking) != cudaSuccess || !o->chunks.init())
    return fail(Status(LGBM_B200_ERR_CUDA, "stream"));
  if (cudaMemcpy(o->label, label, sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(Status(LGBM_B200_ERR_CUDA, "label copy"));
  *out = o.release();
  return LGBM_B200_OK;
}

int lgbm_b200_objective_gradients(LgbmB200Objective* o, const double* scores, float* grad, float* hess,
                                  int32_t location) {
  if (!o || !scores || !grad || !hess) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  if (cudaSetDevice(o->device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  const DRank* rk = o->rank ? &o->rank->d : nullptr;
  const int64_t n = o->n;
  const size_t nk = (size_t)n * (size_t)o->k;
  cudaError_t e = cudaSuccess;
  if (location == LGBM_B200_DEVICE) {
    Status st = launch_gradients(o->cfg, o->label, scores, n, nullptr, grad, hess, current_device_sms(), o->stream, rk);
    if (!st.ok()) return fail(st);
    e = cudaStreamSynchronize(o->stream);
  } else if (o->k == 1 && (o->cfg.objective == LGBM_B200_OBJ_BINARY || o->cfg.objective == LGBM_B200_OBJ_REGRESSION)) {
    // one value per row: scores in and g/h out stream in chunks over three
    // streams, so that copies in and out of different chunks overlap
    for (int64_t r0 = 0, c = 0; r0 < n && e == cudaSuccess; r0 += ChunkStreams::kRows, ++c) {
      const int64_t m = std::min<int64_t>(ChunkStreams::kRows, n - r0);
      cudaStream_t cs = o->chunks.s[c % ChunkStreams::kN];
      e = cudaMemcpyAsync(o->score + r0, scores + r0, sizeof(double) * m, cudaMemcpyHostToDevice, cs);
      if (e == cudaSuccess) {
        Status st = launch_gradients(o->cfg, o->label + r0, o->score + r0, m, nullptr, o->g + r0, o->h + r0, current_device_sms(), cs, rk);
        if (!st.ok()) {
          o->chunks.sync();
          return fail(st);
        }
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaMemcpyAsync(grad + r0, o->g + r0, sizeof(float) * m, cudaMemcpyDeviceToHost, cs);
      if (e == cudaSuccess) e = cudaMemcpyAsync(hess + r0, o->h + r0, sizeof(float) * m, cudaMemcpyDeviceToHost, cs);
    }
    cudaError_t e2 = o->chunks.sync();
    if (e == cudaSuccess) e = e2;
  } else {
    cudaStream_t s = o->stream;
    e = cudaMemcpyAsync(o->score, scores, sizeof(double) * nk, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
      Status st = launch_gradients(o->cfg, o->label, o->score, n, nullptr, o->g, o->h, current_device_sms(), s, rk);
      if (!st.ok()) return fail(st);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(grad, o->g, sizeof(float) * nk, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hess, o->h, sizeof(float) * nk, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  return LGBM_B200_OK;
}

void lgbm_b200_objective_free(LgbmB200Objective* o) {
  if (o) {
    cudaSetDevice(o->device);
    delete o;
    teardown_done("lgbm_b200_objective_free");
  }
}

int lgbm_b200_booster_create(LgbmB200Learner* learner, const LgbmB200BoostConfig* cfg, const float* label,
                             const int32_t* query_boundaries, int32_t num_queries, const uint8_t* valid_bins,
                             int64_t num_valid, LgbmB200Booster** out) {
  if (!learner || !cfg || !label || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  if (learner->dp)  // its init score and metrics would need reductions over the ranks too
    return fail(Status(LGBM_B200_ERR_UNSUPPORTED, "the device booster does not drive a data-parallel learner"));
  auto b = std::make_unique<LgbmB200Booster>();
  Status s = booster_create(b.get(), learner, cfg, label, query_boundaries, num_queries, valid_bins,
                            valid_bins ? num_valid : 0);
  if (!s.ok()) return fail(s);
  *out = b.release();
  return LGBM_B200_OK;
}

void lgbm_b200_booster_destroy(LgbmB200Booster* b) {
  if (b) {
    cudaSetDevice(b->L->device);
    delete b;
    teardown_done("lgbm_b200_booster_destroy");
  }
}

int lgbm_b200_booster_train_iter(LgbmB200Booster* b, int32_t* stop, LgbmB200TreeView* out) {
  if (!b || !stop) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  Status s = booster_iter(b, stop);
  if (!s.ok()) return fail(s);
  if (out)
    for (int k = 0; k < b->K; ++k) b->out_trees[k].view(&out[k]);
  return LGBM_B200_OK;
}

int lgbm_b200_booster_scores(LgbmB200Booster* b, int32_t which, double* out, int32_t location) {
  if (!b || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  cudaSetDevice(b->L->device);
  const double* src = which == 0 ? b->score : b->valid_score;
  size_t cnt = (size_t)b->K * (which == 0 ? b->n : b->nv);
  if (!src || cnt == 0) return LGBM_B200_OK;
  cudaError_t e = cudaMemcpyAsync(out, src, sizeof(double) * cnt,
                                  location == LGBM_B200_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                  b->L->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->L->stream);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  return LGBM_B200_OK;
}

int lgbm_b200_booster_init_scores(LgbmB200Booster* b, double* out) {
  if (!b || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  for (int k = 0; k < b->K; ++k) out[k] = b->init_scores[k];
  return LGBM_B200_OK;
}

}  // extern "C"

// ---- forest / batched prediction ---------------------------------------------------------------
struct LgbmB200Forest {
  int device = 0;
  cudaStream_t stream = nullptr;
  DeviceArena arena;
  DForest f{};
  int32_t ntpi = 1;
  // staging of host rows and scores, grown on demand and kept: a pool
  // allocation per call would be unmapped and mapped again around every
  // synchronisation
  void* stage = nullptr;
  size_t stage_bytes = 0;
  // pinned staging of two row chunks and their scores (host rows), and the
  // event marking when each chunk's buffers are free again
  void* pin = nullptr;
  size_t pin_bytes = 0;
  cudaEvent_t chunk_done[2] = {nullptr, nullptr};
  ~LgbmB200Forest() {
    arena.free_all();
    if (stage) cudaFree(stage);
    if (pin) cudaFreeHost(pin);
    for (auto e : chunk_done)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace lgbm_b200 {
static Status forest_create(LgbmB200Forest* F, const LgbmB200TreeView* trees, int32_t nt, int32_t ntpi,
                            int32_t device) {
  F->device = device;
  F->ntpi = std::max(1, ntpi);
  bool wide = false;
  for (int32_t t = 0; t < nt; ++t) {
    const LgbmB200TreeView& v = trees[t];
    if (v.num_leaves < 1) return Status(LGBM_B200_ERR_INVALID_PARAMETER, "forest_create: a tree has no leaves");
    if (v.num_leaves > 32768) wide = true;
    for (int32_t nd = 0; nd < v.num_leaves - 1; ++nd)
      if (v.split_feature[nd] < 0 || v.split_feature[nd] >= (1 << kNodeFeatureBits))
        return Status(LGBM_B200_ERR_UNSUPPORTED, "forest_create: split feature index outside [0, 2^24)");
  }
  CU(cudaSetDevice(device));
  CU(cudaStreamCreateWithFlags(&F->stream, cudaStreamNonBlocking));
  std::vector<int4> tree;
  std::vector<DNode> nodes;
  std::vector<DNodeWide> wnodes;
  std::vector<int32_t> cat_bnd{0};
  std::vector<double> leaf_value;
  std::vector<uint32_t> cat_words;
  int32_t node_count = 0;
  for (int32_t t = 0; t < nt; ++t) {
    const LgbmB200TreeView& v = trees[t];
    tree.push_back(make_int4(node_count, (int32_t)leaf_value.size(), v.num_leaves, 0));
    int32_t cat_base = (int32_t)cat_bnd.size() - 1;
    for (int32_t c = 0; c < v.num_cat; ++c) {
      int32_t b0 = v.cat_boundaries[c], b1 = v.cat_boundaries[c + 1];
      for (int32_t w = b0; w < b1; ++w) cat_words.push_back(v.cat_threshold[w]);
      cat_bnd.push_back((int32_t)cat_words.size());
    }
    for (int32_t nd = 0; nd < v.num_leaves - 1; ++nd) {
      double thr = v.threshold[nd];
      if (v.decision_type[nd] & 1) {  // categorical: the bitset's index in the threshold's bits
        const int64_t ci = cat_base + (int64_t)v.threshold[nd];
        std::memcpy(&thr, &ci, sizeof(thr));
      }
      const int32_t fd = v.split_feature[nd] | ((int32_t)(uint8_t)v.decision_type[nd] << kNodeFeatureBits);
      if (wide) {
        DNodeWide n{thr, fd, 0, v.left_child[nd], v.right_child[nd]};
        wnodes.push_back(n);
      } else {
        DNode n{thr, fd, (int16_t)v.left_child[nd], (int16_t)v.right_child[nd]};
        nodes.push_back(n);
      }
      ++node_count;
    }
    for (int32_t l = 0; l < v.num_leaves; ++l) leaf_value.push_back(v.leaf_value[l]);
  }
  DeviceArena& A = F->arena;
  auto up = [&](auto& vec, auto** dst) -> Status {
    Status s = A.alloc_n(dst, std::max<size_t>(vec.size(), 1));
    if (!s.ok()) return s;
    if (!vec.empty()) CU(cudaMemcpy(*dst, vec.data(), sizeof(vec[0]) * vec.size(), cudaMemcpyHostToDevice));
    return Status();
  };
  DForest& f = F->f;
  f.num_trees = nt;
  f.ntpi = F->ntpi;
  f.wide = wide;
  Status s;
  int4* tt;
  DNode* dn = nullptr;
  DNodeWide* dw = nullptr;
  int32_t* cb;
  double* lv;
  uint32_t* cw;
  if (!(s = up(tree, &tt)).ok() || !(s = up(cat_bnd, &cb)).ok() || !(s = up(leaf_value, &lv)).ok() ||
      !(s = up(cat_words, &cw)).ok())
    return s;
  if (!(s = wide ? up(wnodes, &dw) : up(nodes, &dn)).ok()) return s;
  f.tree = tt;
  f.nodes = wide ? static_cast<const void*>(dw) : static_cast<const void*>(dn);
  f.cat_bnd = cb;
  f.leaf_value = lv;
  f.cat_words = cw;
  return Status();
}
}  // namespace lgbm_b200

extern "C" {

int lgbm_b200_forest_create(const LgbmB200TreeView* trees, int32_t num_trees, int32_t num_tree_per_iteration,
                            int32_t device, LgbmB200Forest** out) {
  if (!trees || num_trees < 0 || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  auto F = std::make_unique<LgbmB200Forest>();
  Status s = forest_create(F.get(), trees, num_trees, num_tree_per_iteration, device);
  if (!s.ok()) return fail(s);
  *out = F.release();
  return LGBM_B200_OK;
}

void lgbm_b200_forest_destroy(LgbmB200Forest* f) {
  if (f) {
    cudaSetDevice(f->device);
    delete f;
    teardown_done("lgbm_b200_forest_destroy");
  }
}

namespace {

// dst[0, bytes) = src[0, bytes), split over the host's OpenMP threads in 4 MB pieces.
void parallel_copy(void* dst, const void* src, size_t bytes) {
  constexpr size_t kPiece = (size_t)4 << 20;
  const int64_t pieces = (int64_t)((bytes + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < pieces; ++i) {
    const size_t o = (size_t)i * kPiece;
    std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, std::min(kPiece, bytes - o));
  }
}

cudaError_t grow_device(void** p, size_t* have, size_t need) {
  if (*have >= need) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc(p, need);
  if (e == cudaSuccess) *have = need;
  return e;
}

cudaError_t grow_pinned(void** p, size_t* have, size_t need) {
  if (*have >= need) return cudaSuccess;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *have = 0;
  cudaError_t e = cudaHostAlloc(p, need, cudaHostAllocDefault);
  if (e == cudaSuccess) *have = need;
  return e;
}

// Prediction of host rows: they stream through the device in chunks of
// about 256 MB. The host's threads copy chunk c into one of two pinned
// buffers while the copy engine moves chunk c - 1 and the kernel predicts
// it; each chunk's scores come back through pinned memory and are copied out
// two chunks later, when that buffer is needed again. (One copy from
// pageable memory goes through the driver's own staging, a single thread's
// memcpy wide.)
cudaError_t predict_host(LgbmB200Forest* F, const float* X, int64_t nrow, int32_t ncol, double* out) {
  cudaStream_t s = F->stream;
  const int64_t row_bytes = (int64_t)sizeof(float) * ncol;
  int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(nrow, ((int64_t)256 << 20) / row_bytes));
  // LGBM_B200_PREDICT_CHUNK_ROWS: a smaller chunk (tests of the chunk pipeline)
  if (const char* v = std::getenv("LGBM_B200_PREDICT_CHUNK_ROWS"))
    chunk = std::max<int64_t>(1, std::min<int64_t>(chunk, std::atoll(v)));
  const size_t xb = ((size_t)(chunk * row_bytes) + 255) / 256 * 256;
  const size_t ob = (sizeof(double) * (size_t)chunk * F->ntpi + 255) / 256 * 256;
  cudaError_t e = grow_device(&F->stage, &F->stage_bytes, 2 * (xb + ob));
  if (e == cudaSuccess) e = grow_pinned(&F->pin, &F->pin_bytes, 2 * (xb + ob));
  for (int b = 0; b < 2 && e == cudaSuccess; ++b)
    if (!F->chunk_done[b]) e = cudaEventCreateWithFlags(&F->chunk_done[b], cudaEventDisableTiming);
  if (e != cudaSuccess) return e;
  char* dbase = static_cast<char*>(F->stage);
  char* hbase = static_cast<char*>(F->pin);
  const int64_t nchunks = (nrow + chunk - 1) / chunk;
  // scores of chunk c (in pinned buffer c % 2) to the caller's array
  auto copy_out = [&](int64_t c) {
    const int64_t r0 = c * chunk, m = std::min(chunk, nrow - r0);
    parallel_copy(out + (size_t)r0 * F->ntpi, hbase + (c & 1) * (xb + ob) + xb, sizeof(double) * (size_t)m * F->ntpi);
  };
  for (int64_t c = 0; c < nchunks && e == cudaSuccess; ++c) {
    const int b = (int)(c & 1);
    const int64_t r0 = c * chunk, m = std::min(chunk, nrow - r0);
    float* hx = reinterpret_cast<float*>(hbase + b * (xb + ob));
    double* ho = reinterpret_cast<double*>(hbase + b * (xb + ob) + xb);
    float* dx = reinterpret_cast<float*>(dbase + b * (xb + ob));
    double* dout = reinterpret_cast<double*>(dbase + b * (xb + ob) + xb);
    if (c >= 2) {  // buffer b last served chunk c - 2: its copies have run, its scores go out
      if ((e = cudaEventSynchronize(F->chunk_done[b])) != cudaSuccess) break;
      copy_out(c - 2);
    }
    parallel_copy(hx, X + (size_t)r0 * ncol, (size_t)(m * row_bytes));
    e = cudaMemcpyAsync(dx, hx, (size_t)(m * row_bytes), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
      e = launch_predict(F->f, dx, m, ncol, dout, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(ho, dout, sizeof(double) * (size_t)m * F->ntpi, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(F->chunk_done[b], s);
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) return e;
  for (int64_t c = std::max<int64_t>(0, nchunks - 2); c < nchunks; ++c) copy_out(c);
  return cudaSuccess;
}

}  // namespace

int lgbm_b200_predict(LgbmB200Forest* F, const float* X, int64_t nrow, int32_t ncol, double* out,
                      int32_t location) {
  if (!F || !X || !out || nrow < 0 || ncol <= 0) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  if (nrow == 0) return LGBM_B200_OK;
  cudaSetDevice(F->device);
  cudaError_t e;
  if (location == LGBM_B200_HOST) {
    e = predict_host(F, X, nrow, ncol, out);
  } else {
    e = launch_predict(F->f, X, nrow, ncol, out, F->stream);
    cudaError_t e2 = cudaStreamSynchronize(F->stream);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  return LGBM_B200_OK;
}

}  // extern "C"

namespace lgbm_b200 {
void forest_parts(const LgbmB200Forest* F, int* device, cudaStream_t* stream, const DForest** f, int32_t* ntpi) {
  *device = F->device;
  *stream = F->stream;
  *f = &F->f;
  *ntpi = F->ntpi;
}
}  // namespace lgbm_b200
