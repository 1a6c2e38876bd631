// Evaluation metrics on the device (Metric::eval, metric.rs:520-770):
// AUC, binary logloss and error, L2 and RMSE, multiclass logloss and error,
// over labels and scores already in device memory (a booster's validation
// scores need not come back to the host every iteration).
//
// AUC (metric.rs:701-731) without weights accumulates only counts and sums
// of count x (count / 2 + count): every partial sum is a multiple of 1/2
// below 2^52, exact in FP64, so the order of the additions does not matter
// and the device result equals the reference's bit for bit. The scores are
// sorted in descending order with their classes (a bitonic network written
// here), positives are counted by prefix, and one thread per group of tied
// scores adds that group's share.
//
// The losses are FP64 sums of per-row terms; their order differs from the
// reference's sequential loop (within a few ulps of the mean).
#include <algorithm>
#include <mutex>
#include <vector>

#include "learner_impl.h"
#include "rank.h"

namespace lgbm_b200 {

constexpr double kMetricEpsilon = (double)1e-15f;  // consts.rs K_EPSILON
constexpr int kSortBlock = 1024;                   // elements sorted in shared memory by one CTA

// Monotone map of a double onto uint64 (larger score, larger key).
__device__ __forceinline__ uint64_t score_key(double s) {
  if (s == 0.0) s = 0.0;  // -0 and +0 are one score, as the reference compares them
  const uint64_t b = (uint64_t)__double_as_longlong(s);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

// The per-row terms of the loss metrics.
struct LossArgs {
  int32_t metric, num_class, top_k;
  double sigmoid, neg_log_eps;
};

__device__ double row_loss(const LossArgs& a, const float* label, const double* score, int64_t n, int64_t i) {
  const float l = label[i];
  switch (a.metric) {
    case LGBM_B200_METRIC_BINARY_LOGLOSS:
    case LGBM_B200_METRIC_BINARY_ERROR: {
      const double prob = 1.0 / (1.0 + exp(-a.sigmoid * score[i]));  // binary.rs:164-166
      if (a.metric == LGBM_B200_METRIC_BINARY_ERROR) return prob <= 0.5 ? (l > 0.0f ? 1.0 : 0.0) : (l <= 0.0f ? 1.0 : 0.0);
      if (l <= 0.0f) return 1.0 - prob > kMetricEpsilon ? -log(1.0 - prob) : a.neg_log_eps;
      return prob > kMetricEpsilon ? -log(prob) : a.neg_log_eps;
    }
    case LGBM_B200_METRIC_L2:
    case LGBM_B200_METRIC_RMSE: {
      const double d = score[i] - (double)l;
      return d * d;
    }
    default: {  // multiclass: softmax over the class-major scores (multiclass.rs:165)
      const int k = a.num_class;
      const int lk = (int)l;
      double wmax = score[i];
      for (int c = 1; c < k; ++c) wmax = fmax(wmax, score[(int64_t)c * n + i]);
      double wsum = 0.0;
      for (int c = 0; c < k; ++c) wsum += exp(score[(int64_t)c * n + i] - wmax);
      const double pl = exp(score[(int64_t)lk * n + i] - wmax) / wsum;
      if (a.metric == LGBM_B200_METRIC_MULTI_LOGLOSS) return pl > kMetricEpsilon ? -log(pl) : a.neg_log_eps;
      int larger = 0;  // metric.rs:252-265
      for (int c = 0; c < k; ++c) {
        const double pc = exp(score[(int64_t)c * n + i] - wmax) / wsum;
        if (pc >= pl && ++larger > a.top_k) return 1.0;
      }
      return 0.0;
    }
  }
}

// Per-CTA partial sums of the loss terms (added on the host in CTA order).
__global__ void __launch_bounds__(256) k_metric_sum(LossArgs a, const float* label, const double* score, int64_t n,
                                                    double* partial) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += row_loss(a, label, score, n, i);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double ws[8];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
    partial[blockIdx.x] = t;
  }
}

// AUC: keys and classes of m = 2^p slots: 0 negative (label <= 0), 1
// positive (label > 0), 2 padding, 3 a NaN label (neither, as in the
// reference's loop).
__global__ void k_auc_keys(const float* label, const double* score, int64_t n, int64_t m, uint64_t* key,
                           uint8_t* cls) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < n) {
      key[i] = score_key(score[i]);
      const float l = label[i];
      cls[i] = l > 0.0f ? 1 : (l <= 0.0f ? 0 : 3);
    } else {
      key[i] = 0;  // below every score: sorts last
      cls[i] = 2;
    }
  }
}

// One compare-exchange step (k, j) of the bitonic network, descending overall.
__global__ void k_bitonic_global(uint64_t* key, uint8_t* cls, int64_t m, int64_t k, int64_t j) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t l = i ^ j;
    if (l <= i) continue;
    const bool desc = (i & k) == 0;
    const uint64_t a = key[i], b = key[l];
    if (desc ? a < b : a > b) {
      key[i] = b;
      key[l] = a;
      const uint8_t t = cls[i];
      cls[i] = cls[l];
      cls[l] = t;
    }
  }
}

// The steps j = min(k, kSortBlock) / 2 ... 1 of stage k inside blocks of
// kSortBlock slots (k <= kSortBlock: whole stages; larger k: its tail).
__global__ void __launch_bounds__(kSortBlock / 2) k_bitonic_shared(uint64_t* key, uint8_t* cls, int64_t k_from,
                                                                   int64_t k_to) {
  __shared__ uint64_t sk[kSortBlock];
  __shared__ uint8_t sc[kSortBlock];
  const int64_t base = (int64_t)blockIdx.x * kSortBlock;
  for (int t = threadIdx.x; t < kSortBlock; t += blockDim.x) {
    sk[t] = key[base + t];
    sc[t] = cls[base + t];
  }
  __syncthreads();
  for (int64_t k = k_from; k <= k_to; k <<= 1) {
    for (int64_t j = min(k, (int64_t)kSortBlock) >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < kSortBlock; t += blockDim.x) {
        const int l = t ^ (int)j;
        if (l > t) {
          const bool desc = ((base + t) & k) == 0;
          const uint64_t a = sk[t], b = sk[l];
          if (desc ? a < b : a > b) {
            sk[t] = b;
            sk[l] = a;
            const uint8_t c = sc[t];
            sc[t] = sc[l];
            sc[l] = c;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < kSortBlock; t += blockDim.x) {
    key[base + t] = sk[t];
    cls[base + t] = sc[t];
  }
}

// Positives in each block of kSortBlock sorted slots.
__global__ void __launch_bounds__(256) k_auc_block_pos(const uint8_t* cls, int64_t nb, int32_t* block_pos) {
  for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
    int32_t c = 0;
    for (int t = threadIdx.x; t < kSortBlock; t += blockDim.x) c += cls[b * kSortBlock + t] == 1 ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int32_t ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      int32_t s = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += ws[w];
      block_pos[b] = s;
    }
    __syncthreads();
  }
}

// Every group of tied scores adds neg_g * (pos_g / 2 + positives before it)
// (metric.rs:713-723), computed by the thread at the group's first slot;
// `before` holds the positives before each block of slots.
__global__ void __launch_bounds__(kSortBlock) k_auc_groups(const uint64_t* key, const uint8_t* cls, int64_t n,
                                                           const int64_t* before, double* accum) {
  __shared__ int32_t ws[kSortBlock / 32];
  const int64_t i = (int64_t)blockIdx.x * kSortBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // positives before slot i inside its block: a block-wide exclusive scan
  const int32_t p = (i < n && cls[i] == 1) ? 1 : 0;
  int32_t incl = p;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) ws[warp] = incl;
  __syncthreads();
  int32_t wbase = 0;
  for (int w = 0; w < warp; ++w) wbase += ws[w];
  const int64_t pos_before = before[blockIdx.x] + wbase + incl - p;
  if (i >= n) return;
  const uint64_t k0 = key[i];
  if (i > 0 && key[i - 1] == k0) return;  // not the first of its group
  double pos_g = 0.0, neg_g = 0.0;
  for (int64_t j = i; j < n && key[j] == k0; ++j) {
    if (cls[j] == 1) pos_g += 1.0;
    else if (cls[j] == 0) neg_g += 1.0;
  }
  if (neg_g > 0.0) atomicAdd(accum, neg_g * (pos_g * 0.5 + (double)pos_before));
}

namespace {

// Device memory of metric_eval, one set per device: allocated on first use
// and reallocated only when a call needs more (never shrunk), so a call
// allocates and frees nothing (cudaFree synchronises the whole device).
// Calls on one device are serialised by the mutex. The buffers live until
// the process ends.
enum WsSlot { kWsKey, kWsCls, kWsBlockPos, kWsBefore, kWsAcc, kWsPartial, kWsLabel, kWsScore, kWsSlots };
constexpr int kMaxMetricDevices = 64;

struct MetricWorkspace {
  std::mutex mu;
  void* buf[kWsSlots] = {};
  size_t cap[kWsSlots] = {};
  cudaError_t get(WsSlot slot, size_t bytes, void** p) {
    bytes = std::max<size_t>(bytes, 256);
    if (cap[slot] < bytes) {
      if (buf[slot]) {
        cudaError_t e = cudaFree(buf[slot]);
        buf[slot] = nullptr;
        cap[slot] = 0;
        if (e != cudaSuccess) return e;
      }
      cudaError_t e = cudaMalloc(&buf[slot], bytes);
      if (e != cudaSuccess) {
        buf[slot] = nullptr;
        return e;
      }
      cap[slot] = bytes;
    }
    *p = buf[slot];
    return cudaSuccess;
  }
};

MetricWorkspace& metric_workspace(int device) {
  static MetricWorkspace ws[kMaxMetricDevices];
  return ws[device];
}

Status metric_device(MetricWorkspace& ws, const LgbmB200MetricConfig& cfg, const float* label, const double* score,
                     int64_t n, cudaStream_t s, double* out) {
  auto dalloc = [&](WsSlot slot, void** p, size_t bytes) { return ws.get(slot, bytes, p); };
  cudaError_t e = cudaSuccess;
  if (cfg.metric == LGBM_B200_METRIC_AUC) {
    int64_t m = kSortBlock;
    while (m < n) m <<= 1;
    const int64_t nb = m / kSortBlock;
    uint64_t* key = nullptr;
    uint8_t* cls = nullptr;
    int32_t* block_pos = nullptr;
    int64_t* before = nullptr;
    double* acc = nullptr;
    if ((e = dalloc(kWsKey, (void**)&key, sizeof(uint64_t) * m)) != cudaSuccess ||
        (e = dalloc(kWsCls, (void**)&cls, (size_t)m)) != cudaSuccess ||
        (e = dalloc(kWsBlockPos, (void**)&block_pos, sizeof(int32_t) * nb)) != cudaSuccess ||
        (e = dalloc(kWsBefore, (void**)&before, sizeof(int64_t) * nb)) != cudaSuccess ||
        (e = dalloc(kWsAcc, (void**)&acc, sizeof(double))) != cudaSuccess)
      return Status(LGBM_B200_ERR_CUDA, std::string("metric: ") + cudaGetErrorString(e));
    const int grid = (int)std::min<int64_t>((m + 255) / 256, current_device_sms() * 16);
    k_auc_keys<<<grid, 256, 0, s>>>(label, score, n, m, key, cls);
    // bitonic sort: stages up to kSortBlock in shared memory, then each larger
    // stage's steps of span >= kSortBlock in global memory and its tail in shared
    k_bitonic_shared<<<(unsigned)nb, kSortBlock / 2, 0, s>>>(key, cls, 2, kSortBlock);
    for (int64_t k = 2 * (int64_t)kSortBlock; k <= m; k <<= 1) {
      for (int64_t j = k >> 1; j >= kSortBlock; j >>= 1) k_bitonic_global<<<grid, 256, 0, s>>>(key, cls, m, k, j);
      k_bitonic_shared<<<(unsigned)nb, kSortBlock / 2, 0, s>>>(key, cls, k, k);
    }
    k_auc_block_pos<<<(unsigned)std::min<int64_t>(nb, current_device_sms() * 8), 256, 0, s>>>(cls, nb, block_pos);
    std::vector<int32_t> bp((size_t)nb);
    std::vector<int64_t> bf((size_t)nb);
    e = cudaMemcpyAsync(bp.data(), block_pos, sizeof(int32_t) * nb, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    int64_t sum_pos = 0;
    for (int64_t b = 0; b < nb; ++b) {
      bf[(size_t)b] = sum_pos;
      sum_pos += bp[(size_t)b];
    }
    double accum = 0.0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(before, bf.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(double), s);
    if (e == cudaSuccess) {
      k_auc_groups<<<(unsigned)nb, kSortBlock, 0, s>>>(key, cls, n, before, acc);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&accum, acc, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return Status(LGBM_B200_ERR_CUDA, std::string("metric: ") + cudaGetErrorString(e));
    const double sp = (double)sum_pos, sw = (double)n;
    *out = (sp > 0.0 && sp != sw) ? accum / (sp * (sw - sp)) : 1.0;  // metric.rs:724-730
    return Status();
  }
  LossArgs a;
  a.metric = cfg.metric;
  a.num_class = std::max(1, cfg.num_class);
  a.top_k = cfg.multi_error_top_k;
  a.sigmoid = cfg.sigmoid;
  a.neg_log_eps = -(double)std::log(1e-15f);  // consts.rs neg_log_epsilon: the f32 log, promoted
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, current_device_sms() * 8));
  double* partial = nullptr;
  if ((e = dalloc(kWsPartial, (void**)&partial, sizeof(double) * grid)) != cudaSuccess)
    return Status(LGBM_B200_ERR_CUDA, std::string("metric: ") + cudaGetErrorString(e));
  k_metric_sum<<<grid, 256, 0, s>>>(a, label, score, n, partial);
  std::vector<double> ph((size_t)grid);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(ph.data(), partial, sizeof(double) * grid, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return Status(LGBM_B200_ERR_CUDA, std::string("metric: ") + cudaGetErrorString(e));
  double sum = 0.0;
  for (double v : ph) sum += v;
  const double mean = sum / (double)n;  // unweighted: sum_weights = n
  *out = cfg.metric == LGBM_B200_METRIC_RMSE ? std::sqrt(mean) : mean;
  return Status();
}

}  // namespace

}  // namespace lgbm_b200

using namespace lgbm_b200;

extern "C" int lgbm_b200_metric_eval(const LgbmB200MetricConfig* cfg, const float* label, const double* score,
                                     int64_t n, int32_t location, int32_t device, double* out) {
  if (!cfg || !label || !score || !out || n <= 0 || n > ((int64_t)1 << 31))
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "metric: bad argument"));
  if (cfg->metric < LGBM_B200_METRIC_AUC || cfg->metric > LGBM_B200_METRIC_MULTI_ERROR)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "metric: unknown metric"));
  const bool multi = cfg->metric == LGBM_B200_METRIC_MULTI_LOGLOSS || cfg->metric == LGBM_B200_METRIC_MULTI_ERROR;
  if (multi && cfg->num_class < 2) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "metric: num_class < 2"));
  if (device < 0 || device >= kMaxMetricDevices) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "metric: device"));
  if (cudaSetDevice(device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  const int64_t ns = n * (multi ? cfg->num_class : 1);
  MetricWorkspace& ws = metric_workspace(device);
  std::lock_guard<std::mutex> lock(ws.mu);
  // the legacy default stream: device inputs written by work on it are ordered before the metric
  if (location == LGBM_B200_DEVICE) {
    Status st = metric_device(ws, *cfg, label, score, n, 0, out);
    return st.ok() ? LGBM_B200_OK : fail(st);
  }
  float* ld = nullptr;
  double* sd = nullptr;
  if (ws.get(kWsLabel, sizeof(float) * n, (void**)&ld) != cudaSuccess ||
      ws.get(kWsScore, sizeof(double) * ns, (void**)&sd) != cudaSuccess)
    return fail(Status(LGBM_B200_ERR_CUDA, "metric: cudaMalloc"));
  Status st;
  if (cudaMemcpy(ld, label, sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(sd, score, sizeof(double) * ns, cudaMemcpyHostToDevice) != cudaSuccess)
    st = Status(LGBM_B200_ERR_CUDA, "metric: copy");
  else
    st = metric_device(ws, *cfg, ld, sd, n, 0, out);
  return st.ok() ? LGBM_B200_OK : fail(st);
}

extern "C" int lgbm_b200_metric_ndcg(const float* label, const double* score, const int32_t* query_boundaries,
                                     int32_t num_queries, const int32_t* eval_at, int32_t num_eval_at,
                                     int32_t location, int32_t device, double* out) {
  if (!label || !score || !query_boundaries || num_queries <= 0 || !eval_at || num_eval_at <= 0 || !out ||
      query_boundaries[0] != 0)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "ndcg: bad argument"));
  for (int32_t j = 0; j < num_eval_at; ++j)
    if (eval_at[j] <= 0) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "ndcg: eval_at must be positive"));
  if (cudaSetDevice(device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  const int64_t n = query_boundaries[num_queries];
  // the label gains, discounts and query checks of the ranking objective's tables
  std::vector<float> lh;
  const float* lp = label;
  if (location == LGBM_B200_DEVICE) {
    lh.resize((size_t)n);
    if (cudaMemcpy(lh.data(), label, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(Status(LGBM_B200_ERR_CUDA, "ndcg: label copy"));
    lp = lh.data();
  }
  RankTables rt;
  Status st = rt.build(lp, query_boundaries, num_queries, 1.0, 1, false);
  if (!st.ok()) return fail(st);
  float* ld = nullptr;
  double* sd = nullptr;
  int32_t* kd = nullptr;
  double* od = nullptr;
  const size_t nq = (size_t)num_queries, nk = (size_t)num_eval_at;
  cudaError_t e = cudaSuccess;
  if (location != LGBM_B200_DEVICE) {
    if ((e = cudaMalloc(&ld, sizeof(float) * n)) == cudaSuccess) e = cudaMalloc(&sd, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMemcpy(ld, label, sizeof(float) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(sd, score, sizeof(double) * n, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc(&kd, sizeof(int32_t) * nk);
  if (e == cudaSuccess) e = cudaMalloc(&od, sizeof(double) * nq * nk);
  if (e == cudaSuccess) e = cudaMemcpy(kd, eval_at, sizeof(int32_t) * nk, cudaMemcpyHostToDevice);
  std::vector<double> per(nq * nk);
  if (e == cudaSuccess) {
    const float* lbl = location == LGBM_B200_DEVICE ? label : ld;
    const double* sc = location == LGBM_B200_DEVICE ? score : sd;
    st = launch_ndcg(rt.d, lbl, sc, kd, num_eval_at, od, current_device_sms(), 0);
    if (st.ok()) e = cudaMemcpy(per.data(), od, sizeof(double) * nq * nk, cudaMemcpyDeviceToHost);
  }
  if (ld) cudaFree(ld);
  if (sd) cudaFree(sd);
  if (kd) cudaFree(kd);
  if (od) cudaFree(od);
  if (!st.ok()) return fail(st);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, std::string("ndcg: ") + cudaGetErrorString(e)));
  // the mean over queries, added in query order
  for (size_t j = 0; j < nk; ++j) {
    double acc = 0.0;
    for (size_t q = 0; q < nq; ++q) acc += per[q * nk + j];
    out[j] = acc / (double)num_queries;
  }
  return LGBM_B200_OK;
}
