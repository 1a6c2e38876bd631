// Binning of the rows on the device: BinMapper::value_to_bin
// (binning.rs:637-667) and the single-feature group push
// (feature_group.rs:144-154) for every row and used feature, with the bin
// mappers found on the host from the row sample (dataset.rs:394-396).
//
// The kernel restates the host's value_to_bin exactly (the same double
// comparisons and the same binary-search steps), so the matrix it writes is
// bit-identical to the host's. Categorical maps become dense tables indexed
// by category value (unseen values and negative ones give bin 0, as the map
// lookup does).
//
// Rows stream through the device in chunks over three streams: one chunk's
// f32 rows go in while another's bins come out (separate copy engines) and a
// third is binned.
#include <algorithm>

#include "learner_impl.h"

namespace lgbm_b200 {

// One used feature's mapper in device form.
struct DBinMeta {
  int32_t col;        // column of the input matrix
  int32_t bin_type;   // 0 numerical, 1 categorical
  int32_t missing_type;
  int32_t num_bin;
  int32_t mfb;        // most frequent bin
  int32_t ub_off;     // numerical: upper bounds at [ub_off, ub_off + num_bin)
  int32_t cat_off;    // categorical: bins of values [0, cat_size) at [cat_off, cat_off + cat_size)
  int32_t cat_size;
};

constexpr int32_t kMaxCategoryValue = 1 << 22;  // dense category tables stop here

__device__ __forceinline__ uint32_t device_value_to_bin(const DBinMeta& m, const double* ub, const int32_t* cat,
                                                        double value) {
  if (m.bin_type == 1) {
    if (isnan(value)) return 0;
    const int32_t v = (int32_t)value;  // toward zero; out-of-range values land on a bound, which no table holds
    if (v < 0 || v >= m.cat_size) return 0;
    return (uint32_t)cat[m.cat_off + v];
  }
  if (isnan(value)) {
    if (m.missing_type == 2) return (uint32_t)(m.num_bin - 1);
    value = 0.0;
  }
  int32_t l = 0, r = m.num_bin - 1;
  if (m.missing_type == 2) r -= 1;
  const double* u = ub + m.ub_off;
  while (l < r) {
    const int32_t mid = (r + l - 1) / 2;
    if (value <= __ldg(u + mid)) r = mid;
    else l = mid + 1;
  }
  return (uint32_t)l;
}

// bins[r][f] for rows [0, n) of a chunk: thread (r, f) reads X[r][col(f)]
// (neighbouring threads read neighbouring columns of a row) and writes one
// byte (neighbouring threads write neighbouring bytes).
__global__ void __launch_bounds__(256) k_bin_rows(const float* X, int64_t n, int32_t ncol, int32_t nf,
                                                  const DBinMeta* metas, const double* ub, const int32_t* cat,
                                                  uint8_t* bins) {
  const int64_t total = n * (int64_t)nf;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / nf;
    const int32_t f = (int32_t)(i - r * nf);
    const DBinMeta m = metas[f];
    const uint32_t bin = device_value_to_bin(m, ub, cat, (double)X[r * ncol + m.col]);
    // feature_group.rs:144-154: 0 for the most frequent bin, else bin - (mfb == 0) + 1
    bins[i] = bin == (uint32_t)m.mfb ? (uint8_t)0 : (uint8_t)(bin - (m.mfb == 0 ? 1u : 0u) + 1u);
  }
}

#define BIN_CU(x)                                                                       \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess) {                                                            \
      st = Status(LGBM_B200_ERR_CUDA, std::string("device binning: ") + cudaGetErrorString(e_)); \
      goto done;                                                                        \
    }                                                                                   \
  } while (0)

Status push_bins_device(Dataset& d, const float* X, int64_t n, int32_t ncol, int device) {
  const int32_t nf = (int32_t)d.used.size();
  d.bins.assign((size_t)n * (size_t)nf, 0);
  if (n == 0 || nf == 0) return Status();
  // device form of the mappers
  std::vector<DBinMeta> metas((size_t)nf);
  std::vector<double> ub;
  std::vector<int32_t> cat;
  for (int32_t f = 0; f < nf; ++f) {
    const BinMapper& m = d.mappers[(size_t)f];
    DBinMeta& dm = metas[(size_t)f];
    dm.col = d.used[(size_t)f];
    dm.bin_type = m.bin_type;
    dm.missing_type = m.missing_type;
    dm.num_bin = m.num_bin;
    dm.mfb = (int32_t)m.most_freq_bin;
    dm.ub_off = (int32_t)ub.size();
    dm.cat_off = (int32_t)cat.size();
    dm.cat_size = 0;
    if (m.bin_type == 0) {
      ub.insert(ub.end(), m.bin_upper_bound.begin(), m.bin_upper_bound.end());
    } else {
      int32_t top = -1;
      for (const auto& kv : m.categorical_2_bin) top = std::max(top, kv.first);
      if (top >= kMaxCategoryValue)
        return Status(LGBM_B200_ERR_UNSUPPORTED, "device binning: a category value above 2^22 (bin on the host)");
      dm.cat_size = top + 1;
      cat.resize(cat.size() + (size_t)dm.cat_size, 0);
      for (const auto& kv : m.categorical_2_bin)
        if (kv.first >= 0) cat[(size_t)dm.cat_off + (size_t)kv.first] = (int32_t)kv.second;
    }
  }
  if (ub.empty()) ub.push_back(0.0);
  if (cat.empty()) cat.push_back(0);

  Status st;
  int prev = 0;
  cudaGetDevice(&prev);
  ChunkStreams cs;
  DBinMeta* metas_d = nullptr;
  double* ub_d = nullptr;
  int32_t* cat_d = nullptr;
  float* x_d[ChunkStreams::kN] = {};
  uint8_t* b_d[ChunkStreams::kN] = {};
  // rows per chunk: about 64 MB of f32 rows
  const int64_t chunk = std::max<int64_t>(1024, std::min<int64_t>(ChunkStreams::kRows, ((int64_t)64 << 20) / (4 * (int64_t)ncol)));
  const int64_t rows_per_buf = std::min(chunk, n);
  if (cudaSetDevice(device) != cudaSuccess) return Status(LGBM_B200_ERR_CUDA, "device binning: cudaSetDevice");
  if (!cs.init()) {
    st = Status(LGBM_B200_ERR_CUDA, "device binning: streams");
    goto done;
  }
  BIN_CU(cudaMalloc(&metas_d, sizeof(DBinMeta) * (size_t)nf));
  BIN_CU(cudaMalloc(&ub_d, sizeof(double) * ub.size()));
  BIN_CU(cudaMalloc(&cat_d, sizeof(int32_t) * cat.size()));
  BIN_CU(cudaMemcpy(metas_d, metas.data(), sizeof(DBinMeta) * (size_t)nf, cudaMemcpyHostToDevice));
  BIN_CU(cudaMemcpy(ub_d, ub.data(), sizeof(double) * ub.size(), cudaMemcpyHostToDevice));
  BIN_CU(cudaMemcpy(cat_d, cat.data(), sizeof(int32_t) * cat.size(), cudaMemcpyHostToDevice));
  for (int i = 0; i < ChunkStreams::kN; ++i) {
    BIN_CU(cudaMalloc(&x_d[i], sizeof(float) * (size_t)rows_per_buf * (size_t)ncol));
    BIN_CU(cudaMalloc(&b_d[i], (size_t)rows_per_buf * (size_t)nf));
  }
  for (int64_t r0 = 0, k = 0; r0 < n; r0 += chunk, ++k) {
    const int64_t m = std::min(chunk, n - r0);
    const int i = (int)(k % ChunkStreams::kN);
    cudaStream_t s = cs.s[i];
    // a buffer is reused by the chunk three later, on the same stream: in order
    BIN_CU(cudaMemcpyAsync(x_d[i], X + r0 * ncol, sizeof(float) * (size_t)m * (size_t)ncol, cudaMemcpyHostToDevice, s));
    const int64_t items = m * (int64_t)nf;
    const int blocks = (int)std::min<int64_t>((items + 255) / 256, current_device_sms() * 16);
    k_bin_rows<<<blocks, 256, 0, s>>>(x_d[i], m, ncol, nf, metas_d, ub_d, cat_d, b_d[i]);
    BIN_CU(cudaGetLastError());
    BIN_CU(cudaMemcpyAsync(d.bins.data() + (size_t)r0 * (size_t)nf, b_d[i], (size_t)m * (size_t)nf,
                           cudaMemcpyDeviceToHost, s));
  }
  BIN_CU(cs.sync());
done:
  cs.sync();
  for (int i = 0; i < ChunkStreams::kN; ++i) {
    if (x_d[i]) cudaFree(x_d[i]);
    if (b_d[i]) cudaFree(b_d[i]);
  }
  if (metas_d) cudaFree(metas_d);
  if (ub_d) cudaFree(ub_d);
  if (cat_d) cudaFree(cat_d);
  cs.release();
  cudaSetDevice(prev);
  return st;
}

}  // namespace lgbm_b200
