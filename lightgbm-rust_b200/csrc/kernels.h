// Kernel declarations and launch-shape constants shared by the kernel
// translation units and the host driver.
#pragma once
#include <utility>

#include "device_common.cuh"

namespace lgbm_b200 {

constexpr int kHistThreads = 512;
constexpr int kHistTileRows = kHistThreads;  // rows staged per histogram tile: one per thread
constexpr int kHistAsyncStages = 4;  // stages of each warp's copy ring (asynchronously staged histogram rows)
constexpr int kPartThreads = 256;             // threads of a partition CTA
#ifndef LGBM_B200_PART_TILE_ROWS
#define LGBM_B200_PART_TILE_ROWS 1024
#endif
constexpr int kPartTileRows = LGBM_B200_PART_TILE_ROWS;  // rows per partition tile (one look-back word each)
#ifndef LGBM_B200_HIST_CLUSTER
#define LGBM_B200_HIST_CLUSTER 8
#endif
constexpr int kHistCluster = LGBM_B200_HIST_CLUSTER;  // CTAs per quantized histogram cluster (one reduction each)
// CTAs per histogram cluster of a form: the float forms' CTAs fill an SM each and flush alone
__host__ __device__ constexpr int hist_cluster(int mode) { return mode == 2 ? kHistCluster : 1; }
constexpr int kMaxTiles = 64;
constexpr int kMaxLaneGroups = 4;  // 32-feature groups per histogram tile (int32 cells)

// Feature tiles of a histogram launch (blockIdx.y): tile k covers features
// [f0[k], f0[k+1]) whose stored bins are [bin0[k], bin0[k+1]).
struct DTileTable {
  int32_t f0[kMaxTiles + 1];
  int32_t bin0[kMaxTiles + 1];
};

constexpr int kScanThreads = 256;  // one thread per stored bin of a feature view

struct ScanSmem {
  double g[kMaxBins], h[kMaxBins];        // this leaf's feature view
  double cg[kMaxBins], ch[kMaxBins];      // cumulative sums in scan order
  int32_t cc[kMaxBins];                   // cumulative count estimates
  double cg2[kMaxBins], ch2[kMaxBins];    // the forward direction's, formed beside the reverse one's
  int32_t cc2[kMaxBins];
  int32_t ce[kMaxBins];                   // count estimate of each bin
  int64_t ig[kMaxBins];                   // quantized view
  int64_t cq[kMaxBins];                   // quantized cumulative sums in scan order
  int32_t tpos[kMaxBins];                 // categorical: bins with enough data
  int32_t sorted[kMaxBins];               // categorical order
  double key[kMaxBins];
  double eg, eh;                          // the extra candidate t = -1
  int32_t ec, brk, ok;
  int64_t eq;
  int64_t wq[32], wa[32];                 // per-warp totals of the quantized cumulative scan
  double wgain[32];                       // per-warp best candidates (up to 32 warps)
  int32_t wt[32];
  DSplit out;                             // the result, stored to global memory once
};

__global__ void k_tree_init(const __grid_constant__ DCtx c, const uint32_t* bag, const int32_t* n_used);
template <int kMode, int kNG>
__global__ void k_hist(const __grid_constant__ DCtx c, DTileTable tt, int32_t sub_rows, int32_t lead);
// dynamic shared memory, kernel and launch of the histogram for a form and groups per tile
size_t hist_smem_bytes(int mode, int ng);
const void* hist_kernel(int mode, int ng);
// finish: one more cluster whose first CTA runs the previous split step's end,
// which the partition posted (DCtx::defer)
cudaError_t launch_hist(int mode, int ng, dim3 grid, size_t smem, cudaStream_t st, const DCtx& c, const DTileTable& tt,
                        int32_t sub_rows, bool pdl, bool finish);

// A kernel launch, optionally with programmatic stream serialisation (the
// kernel may start launching while its predecessor in the stream runs; it
// calls pdl_wait before reading anything the predecessor writes).
template <typename... Params, typename... Args>
inline cudaError_t launch_ex(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                             Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
constexpr int kScanWideBlocks = 4;  // scan CTAs per SM when a step's scans span several waves
template <bool kInt, int kMinBlocks>
__global__ void k_scan(const __grid_constant__ DCtx c);
// The threshold scans and the partition of one step in one cooperative
// launch (the CTAs wait for each other's scans; co-residency is required).
template <bool kInt>
__global__ void k_scan_partition(const __grid_constant__ DCtx c);

// A cooperative launch (every CTA of the grid resident at once), capturable
// in a CUDA graph.
template <typename... Params, typename... Args>
inline cudaError_t launch_coop(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                               Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Persistent tree growth (one cooperative launch per tree).
constexpr int kGrowThreads = 512;
struct GrowSync {
  unsigned int count;  // CTAs arrived at the current barrier
  unsigned int gen;    // barrier generation
  int status;          // kStatusTimeout when a wait gave up
  int pad;
};
const void* grow_kernel(int mode, int ng);
size_t grow_smem_bytes(int mode, int ng);
cudaError_t launch_grow(int mode, int ng, int grid, size_t smem, cudaStream_t st, const DCtx& c, const DTileTable& tt,
                        int32_t sub_rows, int32_t ntiles, GrowSync* gs, int32_t num_steps, long long* phase_ns);
__global__ void k_partition(const __grid_constant__ DCtx c);
// the quantized threshold scan by one warp per (feature, side) item;
// grid (CTAs, 1, slots), kScanThreads threads
template <int kMinBlocks>
__global__ void k_scan_warp(const __grid_constant__ DCtx c, const int32_t* items);
// the last split step's end, when the partitions post theirs (DCtx::defer);
// grid (1, 1, slots), kPartThreads threads
__global__ void k_finish(const __grid_constant__ DCtx c);
__global__ void k_transpose_bins(const uint8_t* bins, int64_t n, int32_t stride, int32_t nf, uint8_t* colbins);
__global__ void k_leaf_sums(const __grid_constant__ DCtx c, double* partial, int32_t* rank);
__global__ void k_leaf_renew(const __grid_constant__ DCtx c, const double* partial, const int32_t* rank,
                             int32_t nwarps, double* totals);
__global__ void k_dp_leaf_apply(const __grid_constant__ DCtx c, const double* totals);
__global__ void k_dp_finish(const __grid_constant__ DCtx c);
__global__ void k_dp_root_pack(const __grid_constant__ DCtx c, double* f, long long* q);
__global__ void k_dp_root_apply(const __grid_constant__ DCtx c, const double* f, const long long* q);
__global__ void k_add_leaf_outputs(const __grid_constant__ DCtx c, const double* leaf_values, int32_t lv_stride, double* score,
                                   int64_t score_stride);
__global__ void k_leaf_of_row(const __grid_constant__ DCtx c, int32_t* leaf_of_row);
__global__ void k_add_by_row(const int32_t* leaf_of_row, const double* leaf_values, double* score, int64_t n);
__global__ void k_add_tree_binned(const __grid_constant__ DCtx c, const uint8_t* bins, int32_t stride, const uint32_t* rows, int64_t n,
                                  const double* leaf_values, int32_t lv_stride, double* score, int64_t score_stride);

// objective_kernels.cu
__global__ void k_grad_binary(const float* label, const double* score, int64_t n, double sigmoid, float2* gh_out,
                              float* g, float* h);
__global__ void k_grad_l2(const float* label, const double* score, int64_t n, float2* gh_out, float* g, float* h);
__global__ void k_grad_softmax(const float* label, const double* score, int64_t n, int32_t k, float2* gh_out,
                               int64_t gh_stride, float* g, float* h);
__global__ void k_interleave(const float* g, const float* h, int64_t n, float2* gh);
__global__ void k_quant_absmax(const float2* gh, int64_t n, unsigned long long* maxbits, int32_t* counter,
                               DSlotState* st, int32_t bins, int32_t const_hess, int32_t num_blocks, int32_t derive);
__global__ void k_quant_scales(unsigned long long* maxbits, DSlotState* st, int32_t bins, int32_t const_hess);
__global__ void k_quant_apply(const float2* gh, int64_t n, const double* grv, const double* hrv,
                              const int64_t* start_dev, const DSlotState* st, int32_t const_hess, int32_t stochastic,
                              int32_t* packed, int64_t row_offset, int64_t table_n, uint8_t* row_q,
                              int32_t row_stride);
__global__ void k_bagging(uint32_t* rng_state, int64_t n, double fraction, uint8_t* in_bag, int32_t* block_in);
__global__ void k_bag_scan(const int32_t* block_in, int32_t nb, int64_t n, int32_t* block_base, int32_t* counts);
__global__ void k_bag_scatter(const uint8_t* in_bag, int64_t n, const int32_t* block_base, uint32_t* bag,
                              uint32_t* oob);
__global__ void k_add_const(double* score, int64_t n, double v);

}  // namespace lgbm_b200
