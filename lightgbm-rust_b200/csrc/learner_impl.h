// Host-side internals of the learner handle shared by the CUDA translation
// units (learner.cu, booster.cu).
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "kernels.h"
#include "lgbm_b200_internal.h"
#include "predict.h"

namespace lgbm_b200 {


#define CU(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return Status(LGBM_B200_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

#define CU_LAUNCH()                                                                              \
  do {                                                                                           \
    cudaError_t e_ = cudaGetLastError();                                                         \
    if (e_ != cudaSuccess) return Status(LGBM_B200_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
  } while (0)

inline int fail(const Status& s) {
  set_last_error(s.msg);
  return s.code;
}

// The end of a void teardown entry point (destroy / free): it cannot report
// a CUDA error, so it consumes any its calls left as the thread's last
// error; otherwise the next, unrelated call that checks cudaGetLastError
// would return it. LGBM_B200_DEBUG_TEARDOWN=1 prints what was consumed.
inline void teardown_done(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess && std::getenv("LGBM_B200_DEBUG_TEARDOWN"))
    std::fprintf(stderr, "lgbm_b200: %s left %s\n", what, cudaGetErrorString(e));
}

// ------------------------------------------------------------------------------------------
// host RNGs used by the learner (learner/quant.rs random tables; col_sampler.rs)
// ------------------------------------------------------------------------------------------
struct Mt19937 {  // crates/lgbm-core/src/mt19937.rs (libstdc++ mt19937)
  uint32_t state[624];
  int idx;
  explicit Mt19937(uint32_t seed) {
    state[0] = seed;
    for (int i = 1; i < 624; ++i) state[i] = 1812433253u * (state[i - 1] ^ (state[i - 1] >> 30)) + (uint32_t)i;
    idx = 624;
  }
  uint32_t next_u32() {
    if (idx >= 624) {
      for (int k = 0; k < 624; ++k) {
        uint32_t y = (state[k] & 0x80000000u) | (state[(k + 1) % 624] & 0x7fffffffu);
        state[k] = state[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
      }
      idx = 0;
    }
    uint32_t z = state[idx++];
    z ^= z >> 11;
    z ^= (z << 7) & 0x9d2c5680u;
    z ^= (z << 15) & 0xefc60000u;
    z ^= z >> 18;
    return z;
  }
  double uniform01() {
    const double R = 4294967296.0;
    double sum = (double)next_u32();
    sum += (double)next_u32() * R;
    double ret = sum / (R * R);
    if (ret >= 1.0) {
      uint64_t bits = 0x3FEFFFFFFFFFFFFFull;
      std::memcpy(&ret, &bits, 8);
    }
    return ret * (1.0 - 0.0) + 0.0;
  }
  int32_t uniform_int(int32_t a, int32_t b) {
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
};

struct Lcg {  // crates/lgbm-core/src/random.rs
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
      for (int32_t i = 0; i < n; ++i) ret.push_back(i);
    } else if (k > 1 && (double)k > ((double)n / std::log2((double)k))) {
      for (int32_t i = 0; i < n; ++i) {
        double prob = (double)((size_t)k - ret.size()) / (double)(n - i);
        if ((double)next_float() < prob) ret.push_back(i);
      }
    } else {
      std::vector<char> seen((size_t)n, 0);
      for (int32_t r = n - k; r < n; ++r) {
        int32_t v = next_int(0, r + 1);
        if (seen[(size_t)v]) seen[(size_t)r] = 1;
        else seen[(size_t)v] = 1;
      }
      for (int32_t i = 0; i < n; ++i)
        if (seen[(size_t)i]) ret.push_back(i);
    }
    return ret;
  }
};

// ------------------------------------------------------------------------------------------
// device memory
// ------------------------------------------------------------------------------------------
struct DeviceArena {
  std::vector<void*> ptrs;
  size_t bytes = 0;
  Status alloc(void** p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(p, n);
    if (e != cudaSuccess)
      return Status(LGBM_B200_ERR_CUDA, "cudaMalloc(" + std::to_string(n) + "): " + cudaGetErrorString(e));
    ptrs.push_back(*p);
    bytes += n;
    return Status();
  }
  template <class T>
  Status alloc_n(T** p, size_t n) {
    return alloc(reinterpret_cast<void**>(p), n * sizeof(T));
  }
  void free_all() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

struct HostTree {  // the reference's Tree arrays for one trained tree
  int32_t num_leaves = 1;
  std::vector<int32_t> split_feature_inner, split_feature, left_child, right_child, leaf_parent, leaf_count,
      leaf_depth, internal_count, cat_boundaries, cat_boundaries_inner;
  std::vector<float> split_gain;
  std::vector<uint32_t> threshold_in_bin, cat_threshold, cat_threshold_inner, cat_bits;
  std::vector<double> threshold, leaf_value, leaf_weight, internal_value, internal_weight, node_gain;
  std::vector<int8_t> decision_type;
  int32_t num_cat = 0;
  void view(LgbmB200TreeView* v) const {
    v->num_leaves = num_leaves;
    v->split_feature_inner = split_feature_inner.data();
    v->split_feature = split_feature.data();
    v->split_gain = split_gain.data();
    v->threshold_in_bin = threshold_in_bin.data();
    v->threshold = threshold.data();
    v->decision_type = decision_type.data();
    v->left_child = left_child.data();
    v->right_child = right_child.data();
    v->leaf_parent = leaf_parent.data();
    v->leaf_value = leaf_value.data();
    v->leaf_weight = leaf_weight.data();
    v->leaf_count = leaf_count.data();
    v->leaf_depth = leaf_depth.data();
    v->internal_value = internal_value.data();
    v->internal_weight = internal_weight.data();
    v->internal_count = internal_count.data();
    v->num_cat = num_cat;
    v->cat_boundaries = cat_boundaries.data();
    v->cat_threshold = cat_threshold.data();
    v->cat_boundaries_inner = cat_boundaries_inner.data();
    v->cat_threshold_inner = cat_threshold_inner.data();
    v->split_gain_f64 = node_gain.data();
  }
};

}  // namespace lgbm_b200

using namespace lgbm_b200;

// Multiprocessors of the current device (queried once per device).
inline int current_device_sms() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int v = 0;
    cached[dev] = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0 ? v : 148;
  }
  return cached[dev];
}

// Streams over which a call with host buffers pipelines its row chunks: the
// copy in, the kernel and the copy out of successive chunks overlap (the two
// copy directions run on separate copy engines).
struct ChunkStreams {
  static constexpr int kN = 3;
  static constexpr int64_t kRows = 1 << 20;  // rows per chunk
  cudaStream_t s[kN] = {};
  cudaEvent_t ready = nullptr;  // recorded on the caller's stream: the chunks start after it
  bool init() {
    if (ready) return true;
    for (int i = 0; i < kN; ++i)
      if (cudaStreamCreateWithFlags(&s[i], cudaStreamNonBlocking) != cudaSuccess) return false;
    return cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) == cudaSuccess;
  }
  cudaError_t sync() {
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < kN; ++i) {
      cudaError_t ei = s[i] ? cudaStreamSynchronize(s[i]) : cudaSuccess;
      if (e == cudaSuccess) e = ei;
    }
    return e;
  }
  void release() {
    for (int i = 0; i < kN; ++i)
      if (s[i]) cudaStreamDestroy(s[i]);
    if (ready) cudaEventDestroy(ready);
    for (int i = 0; i < kN; ++i) s[i] = nullptr;
    ready = nullptr;
  }
};

struct LgbmB200Learner {
  LgbmB200LearnerConfig cfg{};
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  DeviceArena arena;
  int64_t n = 0;
  int32_t nf = 0, stride = 0, total_bins = 0, K = 1, L = 2;
  std::vector<DFeature> feats;
  std::vector<std::vector<double>> upper_bounds;
  std::vector<std::vector<int32_t>> bin_to_cat;
  DCtx ctx{};
  DTileTable tiles{};
  int ntiles = 1;
  int hist_ng = 1;  // 32-feature groups per histogram tile
  int use_pdl = 0;  // kernel edges chained by programmatic dependent launch (bits: histogram, scan, partition)
  int grow_grid = 0;       // CTAs of the persistent grow launch
  size_t grow_smem = 0;
  GrowSync* grow_sync = nullptr;
  long long* phase_ns = nullptr;  // persistent growth: device ns per phase
  size_t hist_smem = 0, scan_smem = 0;
  int hist_grid = 148, part_grid = 592, root_grid = kRootBlocks;
  int32_t sub_rows = 8192;
  std::vector<DSlot> slots_h;
  float2* gh_all = nullptr;  // [K x n] interleaved gradients of every slot
  // quantization
  double* grv = nullptr;
  double* hrv = nullptr;
  std::unique_ptr<Mt19937> start_eng;
  int64_t* start_dev = nullptr;  // [K] each slot's offset into the rounding tables, read by k_quant_apply
  int64_t* start_h = nullptr;    // [K] pinned staging of those offsets
  unsigned long long* maxbits = nullptr;
  int32_t* quant_counter = nullptr;
  // bagging
  uint32_t* bag = nullptr;
  int32_t* n_used_dev = nullptr;  // in-bag row count read by k_tree_init
  int32_t n_used = 0;
  bool bagging = false;
  // leaf renewal scratch: [K][leaf_sum_warps + L][2] segment sums, [K][L + 1] leaf ranks
  double* leaf_sums = nullptr;
  int32_t* leaf_rank = nullptr;
  double* leaf_values_dev = nullptr;  // [K][L] for add_leaf_outputs
  double* score_scratch = nullptr;  // host gradients staged for train (2 x num_data floats)
  double* score_stage = nullptr;    // host scores staged for add_leaf_outputs (num_data doubles)
  int32_t* leaf_of_row = nullptr;   // leaf of each in-bag row (-1 out of bag), for add_leaf_outputs from host
  ChunkStreams chunks;              // add_leaf_outputs from host buffers
  // readback
  std::vector<DSlotState> st_h;
  // Every slot's state and tree arrays in one device block (rb_slot bytes
  // per slot, at the offsets in rb), so that one copy into the pinned mirror
  // reads a whole tree set back.
  struct ReadbackLayout {
    size_t st, sfi, sf, sg, tib, dt, lc, rc, lp, lv, lw, lcnt, ld, iv, iw, ic, cb, ng;
  } rb{};
  unsigned char* rb_dev = nullptr;
  unsigned char* rb_host = nullptr;
  size_t rb_slot = 0;
  std::vector<HostTree> trees;
  std::vector<int32_t> tmp_i32;
  // timing
  bool timing = false;
  std::vector<cudaEvent_t> ev;
  cudaEvent_t marks[16] = {};  // caller-placed timing marks on the learner's stream
  double last_ms[4] = {0, 0, 0, 0};
  std::vector<float> last_step_ms;  // timing on: (histogram, scan, partition) ms of every split step
  // data-parallel growth (lgbm_b200_learner_set_data_parallel)
  bool dp = false;
  int64_t dp_offset = 0, dp_global_n = 0;
  LgbmB200AllReduceFn dp_fn = nullptr;
  void* dp_user = nullptr;
  double* dp_f64 = nullptr;     // [2 * L + 4] root / renewal sums
  long long* dp_i64 = nullptr;  // [4]
  int64_t last_hist_rows = 0;
  int64_t last_part_rows = 0;
  bool scan_wide = false;  // the register-capped scan variant (many CTAs per step)
  // the quantized scan by one warp per (feature, side): the item of each
  // warp of each CTA (feature * 2 + side, -1 none; at most one categorical
  // item per CTA) and the CTAs per slot
  bool scan_warp = false;
  int32_t* scan_items = nullptr;
  int scan_warp_grid = 0;
  bool scan_part = false;  // scans and partition of a step in one cooperative launch
  int scan_part_grid = 0;
  int scan_part_max = 0;  // CTAs of that launch resident at once, shared by the slots
  // the last train call: whether one ran, and each slot's quantization offset
  bool trained = false;
  std::vector<int64_t> last_start;
  // bumped whenever a host-side setting that enqueue_tree's launches carry
  // changes (launch shape, bagging): graphs captured before it are stale
  int config_epoch = 0;
  int32_t last_launches = 0;
  // captured tree growth
  cudaGraphExec_t graph_exec = nullptr;
  int graph_key = -1;
  ~LgbmB200Learner() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    for (auto e : ev) cudaEventDestroy(e);
    for (auto e : marks)
      if (e) cudaEventDestroy(e);
    arena.free_all();
    chunks.release();
    if (start_h) cudaFreeHost(start_h);
    if (rb_host) cudaFreeHost(rb_host);
    if (stream) cudaStreamDestroy(stream);
  }
};


namespace lgbm_b200 {
// Warps of the leaf renewal's sum kernel (4 CTAs of 8 warps per SM); its
// partial sums are laid out by warp.
inline int32_t leaf_sum_warps(const LgbmB200Learner* h) { return h->num_sms * 4 * 8; }
// One tree per slot from the given gradients (class-major [K x n]); NULL
// gradients reuse the slots' interleaved buffers filled by the caller.
Status train(LgbmB200Learner* h, const float* grad, const float* hess, int32_t location);
// train in two halves: enqueue the tree's work; read the trees back (synchronises)
Status train_enqueue(LgbmB200Learner* h, const float* grad, const float* hess, int32_t location);
Status train_collect(LgbmB200Learner* h);
// the pieces of train_enqueue a captured booster iteration uses: the host
// draw of the quantization offsets, then (capturable) their copy and the
// quantization, and the launches of one tree
void draw_quant_starts(LgbmB200Learner* h, bool replay);
Status enqueue_quant(LgbmB200Learner* h);
// the stochastic-rounding tables of `rows` rows (learner/quant.rs:364-398)
Status quant_tables(LgbmB200Learner* h, int64_t rows);
// data-parallel growth: one in-place reduction over the ranks of a device buffer
Status dp_allreduce(LgbmB200Learner* h, void* buf, int64_t count, int32_t dtype, int32_t op);
Status enqueue_tree(LgbmB200Learner* h);
Status get_launch_shape(const LgbmB200Learner* h, LgbmB200LaunchShape* out);
Status set_launch_shape(LgbmB200Learner* h, const LgbmB200LaunchShape& in);
Status autotune(LgbmB200Learner* h, const LgbmB200LaunchShape* cand, int32_t num, int32_t reps, int32_t* chosen,
                double* ms);
Status histogram_of_rows(LgbmB200Learner* h, int slot, const uint32_t* rows, int64_t nrows, void* out);
}  // namespace lgbm_b200

namespace lgbm_b200 {
inline double maybe_round_to_zero_h(double v) {  // tree.rs:22-29
  return (v >= -(double)1e-35f && v <= (double)1e-35f) ? 0.0 : v;
}
}  // namespace lgbm_b200
