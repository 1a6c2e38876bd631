// Host driver of the B200 tree learner and the C ABI of include/lgbm_b200.h.
//
// A learner handle owns the uploaded bin matrix and, per tree slot, every
// device buffer the grow loop touches. One train call enqueues the whole
// tree (init, then num_leaves-1 steps of histogram / scan / partition) on
// the handle's stream without reading anything back until the tree is done
// (optionally replayed from a captured CUDA graph), then copies the tree
// arrays back and rebuilds the reference's Tree layout on the host.
#include <cstdlib>
#include <algorithm>
#include <functional>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "learner_impl.h"

namespace lgbm_b200 {
static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace lgbm_b200

namespace lgbm_b200 {

static Status setup_learner(LgbmB200Learner* h, const LgbmB200LearnerConfig* cfg, const uint8_t* bins, int64_t n,
                            int32_t nf, const LgbmB200FeatureMeta* metas) {
  h->cfg = *cfg;
  if (n <= 0 || n > INT32_MAX) return Status(LGBM_B200_ERR_INVALID_DATA, "num_data must be in [1, 2^31-1]");
  if (nf <= 0) return Status(LGBM_B200_ERR_INVALID_DATA, "no features");
  if (cfg->num_leaves > 8192)
    return Status(LGBM_B200_ERR_UNSUPPORTED, "num_leaves above 8192 on the device learner");
  h->device = cfg->device;
  CU(cudaSetDevice(h->device));
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, h->device));
  h->num_sms = prop.multiProcessorCount;
  CU(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  h->n = n;
  h->nf = nf;
  h->K = std::max(1, cfg->num_tree_slots);
  if (h->K > kMaxSlots) return Status(LGBM_B200_ERR_UNSUPPORTED, "more than 16 trees grown together");
  h->L = std::max(2, cfg->num_leaves);
  h->stride = (nf + 31) / 32 * 32;
  // features and histogram layout
  int32_t pos = 0;
  h->feats.resize(nf);
  for (int32_t f = 0; f < nf; ++f) {
    const LgbmB200FeatureMeta& m = metas[f];
    DFeature& d = h->feats[f];
    d.num_bin = m.num_bin;
    d.most_freq_bin = m.most_freq_bin;
    d.offset = m.most_freq_bin == 0 ? 1 : 0;
    d.default_bin = m.default_bin;
    d.missing_type = m.missing_type;
    d.bin_type = m.bin_type;
    d.monotone_type = m.monotone_type;
    d.real_index = m.real_index;
    d.penalty = m.penalty;
    d.view_start = pos;
    d.view_len = m.num_bin - d.offset;
    if (d.view_len + 1 > kMaxBins || d.view_len < 0)
      return Status(LGBM_B200_ERR_UNSUPPORTED, "feature " + std::to_string(f) + " stores more than 256 bins");
    if (d.monotone_type != 0 && d.bin_type == 1)
      return Status(LGBM_B200_ERR_INVALID_PARAMETER,
                    "The output cannot be monotone with respect to categorical features");
    pos += d.view_len;
  }
  h->total_bins = pos;
  bool use_monotone = false;
  for (auto& f : h->feats) use_monotone |= f.monotone_type != 0;
  // feature tiles: groups of 32 features (lane l of a warp owns feature
  // f0 + 32g + l); int32 cells allow up to kMaxLaneGroups groups per tile,
  // FP64 / FP32-pair cells (16 bytes) one group
  const int mode = cfg->hist_precision;
  if (mode < 0 || mode > 2) return Status(LGBM_B200_ERR_INVALID_PARAMETER, "hist_precision");
  const size_t cell = mode == LGBM_B200_HIST_QUANT ? 4 : 16;
  // One group per tile by default: a one-group CTA takes 52 KB of shared
  // memory (two resident per SM, the register limit) where a four-group one
  // takes 196 KB (one per SM, its warps stalled at the tile barriers). More
  // tiles re-read each row's index and gradient once per tile, which costs
  // less: multiclass K=10 x 200 features 51.0 -> 35.4 ms per iteration,
  // lambdarank x 136 features 53.8 -> 38.1 (three groups: 38.4 / 36.5).
  // LGBM_B200_HIST_GROUPS (1..kMaxLaneGroups) sets the quantized form's groups
  // per tile.
  int groups_per_tile = 1;
  if (const char* e = std::getenv("LGBM_B200_HIST_GROUPS"))
    if (mode == LGBM_B200_HIST_QUANT) groups_per_tile = std::max(1, std::min(kMaxLaneGroups, std::atoi(e)));
  {
    const int ngroups = (nf + 31) / 32;
    h->ntiles = (ngroups + groups_per_tile - 1) / groups_per_tile;
    if (h->ntiles > kMaxTiles) return Status(LGBM_B200_ERR_UNSUPPORTED, "too many histogram feature tiles");
    for (int t = 0; t <= h->ntiles; ++t) {
      int f = std::min(nf, t * groups_per_tile * 32);
      h->tiles.f0[t] = f;
      h->tiles.bin0[t] = f < nf ? h->feats[f].view_start : h->total_bins;
    }
    h->hist_ng = std::min(ngroups, groups_per_tile);
    h->hist_smem = hist_smem_bytes(mode, h->hist_ng);
  }
  if (mode == LGBM_B200_HIST_QUANT) {
    int32_t half = std::max(1, cfg->num_grad_quant_bins / 2);
    int64_t lim = std::min<int64_t>(32767 / half, 65535 / std::max(1, cfg->num_grad_quant_bins));
    // a cell packs (g << 16) + h: per-row |g| <= bins / 2 and h <= bins keep
    // both 16-bit halves exact over `lim` rows
    h->sub_rows = (int32_t)lim;
    if (cfg->num_grad_quant_bins < 2 || cfg->num_grad_quant_bins > 64)
      return Status(LGBM_B200_ERR_UNSUPPORTED, "num_grad_quant_bins must be in [2, 64]");
  }
  // kernel attributes and grid sizes
  const void* hk = hist_kernel(mode, h->hist_ng);
  CU(cudaFuncSetAttribute(hk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->hist_smem));
  // clusters above 8 CTAs are a non-portable size the kernel must opt into
  if (hist_cluster(mode) > 8) CU(cudaFuncSetAttribute(hk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  h->scan_smem = sizeof(ScanSmem);
  // the per-position leaf kernels hold a 16-byte table entry per leaf
  CU(cudaFuncSetAttribute(k_leaf_sums, cudaFuncAttributeMaxDynamicSharedMemorySize, 16 * h->L));
  CU(cudaFuncSetAttribute(k_add_leaf_outputs, cudaFuncAttributeMaxDynamicSharedMemorySize, 16 * h->L));
  CU(cudaFuncSetAttribute(k_leaf_of_row, cudaFuncAttributeMaxDynamicSharedMemorySize, 16 * h->L));
  CU(cudaFuncSetAttribute(k_scan<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->scan_smem));
  CU(cudaFuncSetAttribute(k_scan<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->scan_smem));
  CU(cudaFuncSetAttribute(k_scan<false, kScanWideBlocks>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)h->scan_smem));
  CU(cudaFuncSetAttribute(k_scan<true, kScanWideBlocks>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)h->scan_smem));
  // a step's scans are (feature, side, slot) CTAs: beyond two CTAs per SM they
  // run in waves, and the register-capped variant keeps more of them resident
  // (LGBM_B200_SCAN_WIDE=0/1 forces either)
  h->scan_wide = (int64_t)nf * 2 * std::max(1, cfg->num_tree_slots) > 2 * (int64_t)h->num_sms;
  if (const char* e = std::getenv("LGBM_B200_SCAN_WIDE")) h->scan_wide = std::atoi(e) != 0;
  {
    // the histogram runs in clusters (of hist_cluster(mode) CTAs): as many
    // clusters as fit on the device at once, shared among the feature tiles
    cudaLaunchConfig_t lc = {};
    const int cl = hist_cluster(mode);
    lc.gridDim = dim3(cl * 64, 1, 1);
    lc.blockDim = dim3(kHistThreads, 1, 1);
    lc.dynamicSmemBytes = h->hist_smem;
    int clusters = 0;
    CU(cudaOccupancyMaxActiveClusters(&clusters, hk, &lc));
    if (clusters < 1) return Status(LGBM_B200_ERR_CUDA, "histogram cluster does not fit on the device");
    h->hist_grid = std::max(1, clusters / std::max(1, h->ntiles)) * cl;
  }
  h->part_grid = h->num_sms * 3;  // 3 CTAs per SM measured best with 1024-row tiles (2 and 2.5 per SM are slower)
  // LGBM_B200_PART_GRID sets the partition's CTA count (launch-shape sweeps)
  if (const char* e = std::getenv("LGBM_B200_PART_GRID")) h->part_grid = std::max(1, std::atoi(e));
  // LGBM_B200_SCANPART=1: the threshold scans and the partition of a step run
  // as one cooperative launch (one kernel boundary less per split); the
  // grid is what stays resident at once, shared by the tree slots
  h->scan_part = false;
  if (const char* e = std::getenv("LGBM_B200_SCANPART"))
    h->scan_part = std::atoi(e) != 0 && !cfg->persistent_grow;
  if (h->scan_part) {
    const void* k = mode == LGBM_B200_HIST_QUANT ? (const void*)k_scan_partition<true> : (const void*)k_scan_partition<false>;
    int per_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kPartThreads, h->scan_smem));
    const int K = std::max(1, cfg->num_tree_slots);
    h->scan_part_max = per_sm * h->num_sms / K;
    h->scan_part_grid = std::min(h->part_grid, h->scan_part_max);
    if (h->scan_part_grid < 1) return Status(LGBM_B200_ERR_UNSUPPORTED, "scan + partition launch does not fit");
  }
  // programmatic dependent launch per kernel edge, a bit mask: 1 the
  // histogram (after the partition), 2 the scan (after the histogram), 4 the
  // partition (after the scan)
  if (const char* e = std::getenv("LGBM_B200_PDL")) h->use_pdl = std::atoi(e) & 7;
  if (cfg->persistent_grow) {
    // one resident CTA group per slot: the cooperative launch holds every CTA
    const void* gk = grow_kernel(mode, h->hist_ng);
    h->grow_smem = grow_smem_bytes(mode, h->hist_ng);
    CU(cudaFuncSetAttribute(gk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->grow_smem));
    int per_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gk, kGrowThreads, h->grow_smem));
    const int k = std::max(1, cfg->num_tree_slots);
    h->grow_grid = per_sm * h->num_sms / k * k;
    if (h->grow_grid < k) return Status(LGBM_B200_ERR_UNSUPPORTED, "persistent growth does not fit on the device");
  }
  int32_t rpb = cfg->hist_rows_per_block > 0 ? cfg->hist_rows_per_block : 512;

  // device buffers
  DeviceArena& A = h->arena;
  uint8_t* bins_d;
  Status s = A.alloc_n(&bins_d, (size_t)n * h->stride);
  if (!s.ok()) return s;
  {
    // host copy with the padded row stride, uploaded once
    std::vector<uint8_t> padded((size_t)n * h->stride, 0);
    for (int64_t r = 0; r < n; ++r) std::memcpy(&padded[(size_t)r * h->stride], bins + (size_t)r * nf, (size_t)nf);
    CU(cudaMemcpy(bins_d, padded.data(), padded.size(), cudaMemcpyHostToDevice));
  }
  uint8_t* colbins_d;
  if (!(s = A.alloc_n(&colbins_d, (size_t)n * nf)).ok()) return s;
  k_transpose_bins<<<h->num_sms * 8, 256>>>(bins_d, n, h->stride, nf, colbins_d);
  CU(cudaGetLastError());
  CU(cudaDeviceSynchronize());
  DFeature* feats_d;
  if (!(s = A.alloc_n(&feats_d, (size_t)nf)).ok()) return s;
  CU(cudaMemcpy(feats_d, h->feats.data(), sizeof(DFeature) * nf, cudaMemcpyHostToDevice));
  const int K = h->K, L = h->L;
  // The quantized scan by one warp per (feature, side) item, for steps whose
  // block scans would run in waves (many features or tree slots): there the
  // scan is bound by throughput, and eight items share a CTA without block
  // barriers (multiclass K=10 x 200 features: 29.6 -> 25.1 ms per iteration).
  // With few items each item's latency counts, and the block scan's 256
  // threads per item are faster (binary x 28 features: 7.39 against 8.54 ms;
  // lambdarank x 136: 29.9 against 31.1). Each CTA takes up to `per` items,
  // at most one of them categorical (the CTA's scratch holds its sort).
  // LGBM_B200_SCAN_WARP=0/1 forces either; LGBM_B200_SCAN_PER=<1..8> sets the
  // items per CTA.
  h->scan_warp = mode == LGBM_B200_HIST_QUANT && h->scan_wide;
  if (const char* e = std::getenv("LGBM_B200_SCAN_WARP"))
    h->scan_warp = mode == LGBM_B200_HIST_QUANT && std::atoi(e) != 0;
  if (h->scan_warp) {
    constexpr int kWarps = kScanThreads / 32;
    std::vector<int32_t> numer, cats;
    for (int f = 0; f < nf; ++f)
      for (int side = 0; side < 2; ++side) (h->feats[f].bin_type == 1 ? cats : numer).push_back(f * 2 + side);
    const int64_t items = (int64_t)numer.size() + (int64_t)cats.size();
    int per = (int)std::min<int64_t>(kWarps, std::max<int64_t>(1, (items * K + h->num_sms - 1) / h->num_sms));
    if (const char* e = std::getenv("LGBM_B200_SCAN_PER")) per = std::max(1, std::min(kWarps, std::atoi(e)));
    const int64_t ctas = std::max<int64_t>((items + per - 1) / per, (int64_t)cats.size());
    std::vector<int32_t> table((size_t)ctas * kWarps, -1);
    size_t next = 0;
    for (int64_t b = 0; b < ctas; ++b) {
      int used = 0;
      if ((size_t)b < cats.size()) table[(size_t)b * kWarps + used++] = cats[(size_t)b];
      while (used < per && next < numer.size()) table[(size_t)b * kWarps + used++] = numer[next++];
    }
    if (!(s = A.alloc_n(&h->scan_items, table.size())).ok()) return s;
    CU(cudaMemcpy(h->scan_items, table.data(), sizeof(int32_t) * table.size(), cudaMemcpyHostToDevice));
    h->scan_warp_grid = (int)ctas;
  }
  const size_t cells = (size_t)h->total_bins * (mode == LGBM_B200_HIST_QUANT ? 1 : 2);
  const size_t max_tiles = ((size_t)n + kPartTileRows - 1) / kPartTileRows + 1;
  {
    // the readback block: each slot's state, then its tree arrays, each
    // piece on a 256-byte boundary
    size_t off = 0;
    auto take = [&](size_t bytes) {
      const size_t o = off;
      off += (bytes + 255) / 256 * 256;
      return o;
    };
    auto& rb = h->rb;
    const size_t Ls = (size_t)L;
    rb.st = take(sizeof(DSlotState));
    rb.sfi = take(4 * Ls);
    rb.sf = take(4 * Ls);
    rb.sg = take(4 * Ls);
    rb.tib = take(4 * Ls);
    rb.dt = take(Ls);
    rb.lc = take(4 * Ls);
    rb.rc = take(4 * Ls);
    rb.lp = take(4 * Ls);
    rb.lv = take(8 * Ls);
    rb.lw = take(8 * Ls);
    rb.lcnt = take(4 * Ls);
    rb.ld = take(4 * Ls);
    rb.iv = take(8 * Ls);
    rb.iw = take(8 * Ls);
    rb.ic = take(4 * Ls);
    rb.cb = take(4 * Ls * kCatWords);
    rb.ng = take(8 * Ls);
    h->rb_slot = off;
    if (!(s = A.alloc(reinterpret_cast<void**>(&h->rb_dev), off * (size_t)K)).ok()) return s;
    CU(cudaHostAlloc(reinterpret_cast<void**>(&h->rb_host), off * (size_t)K, cudaHostAllocDefault));
  }
  h->slots_h.resize(K);
  for (int k = 0; k < K; ++k) {
    DSlot& d = h->slots_h[k];
    std::memset(&d, 0, sizeof(d));
#define ALLOC(ptr, count)                                  \
  if (!(s = A.alloc_n(&(ptr), (size_t)(count))).ok()) return s;
    unsigned char* rbk = h->rb_dev + (size_t)k * h->rb_slot;
    d.st = reinterpret_cast<DSlotState*>(rbk + h->rb.st);
    ALLOC(d.idx[0], n);
    ALLOC(d.idx[1], n);
    ALLOC(d.leaf_begin, L);
    ALLOC(d.leaf_count, L);
    d.leaf_gcount = d.leaf_count;  // one learner holds every row: its counts are its ranges
    ALLOC(d.leaf_side, L);
    ALLOC(d.buf_of, L);
    ALLOC(d.best, L);
    ALLOC(d.bgain, L);
    ALLOC(d.bfeat, L);
    ALLOC(d.splittable, (size_t)L * nf);
    ALLOC(d.cmin, L);
    ALLOC(d.cmax, L);
    {
      double* hp;
      ALLOC(hp, cells * L);
      d.hist = hp;
    }
    ALLOC(d.feat_res, 2 * (size_t)nf);
    ALLOC(d.lut_cand, 2 * (size_t)nf * kMaxBins);
    ALLOC(d.leaf_lut, (size_t)L * kMaxBins);
    ALLOC(d.feat_ok, 4 * (size_t)nf);
    ALLOC(d.tile_status, max_tiles);
    d.gh = nullptr;  // set below from the contiguous [K x n] buffer
    if (mode == LGBM_B200_HIST_QUANT) ALLOC(d.packed, n);
    ALLOC(d.bytree, nf);
    ALLOC(d.root_partials, 2 * kRootBlocks);
    ALLOC(d.root_ipartials, kRootBlocks);
    ALLOC(d.root_counter, 1);
    DTree& t = d.tree;
    const auto& rb = h->rb;
    t.split_feature_inner = reinterpret_cast<int32_t*>(rbk + rb.sfi);
    t.split_feature = reinterpret_cast<int32_t*>(rbk + rb.sf);
    t.split_gain = reinterpret_cast<float*>(rbk + rb.sg);
    t.threshold_in_bin = reinterpret_cast<uint32_t*>(rbk + rb.tib);
    t.decision_type = reinterpret_cast<int8_t*>(rbk + rb.dt);
    t.left_child = reinterpret_cast<int32_t*>(rbk + rb.lc);
    t.right_child = reinterpret_cast<int32_t*>(rbk + rb.rc);
    t.leaf_parent = reinterpret_cast<int32_t*>(rbk + rb.lp);
    t.leaf_value = reinterpret_cast<double*>(rbk + rb.lv);
    t.leaf_weight = reinterpret_cast<double*>(rbk + rb.lw);
    t.leaf_count = reinterpret_cast<int32_t*>(rbk + rb.lcnt);
    t.leaf_depth = reinterpret_cast<int32_t*>(rbk + rb.ld);
    t.internal_value = reinterpret_cast<double*>(rbk + rb.iv);
    t.internal_weight = reinterpret_cast<double*>(rbk + rb.iw);
    t.internal_count = reinterpret_cast<int32_t*>(rbk + rb.ic);
    t.cat_bits = reinterpret_cast<uint32_t*>(rbk + rb.cb);
    t.node_gain = reinterpret_cast<double*>(rbk + rb.ng);
    CU(cudaMemset(d.st, 0, sizeof(DSlotState)));
    CU(cudaMemset(d.tile_status, 0, max_tiles * sizeof(unsigned long long)));
    CU(cudaMemset(d.root_counter, 0, sizeof(int32_t)));
    CU(cudaMemset(d.bytree, 1, nf));
  }
  if (!(s = A.alloc_n(&h->gh_all, (size_t)K * n)).ok()) return s;
  for (int k = 0; k < K; ++k) h->slots_h[k].gh = h->gh_all + (size_t)k * n;
  if (!(s = A.alloc_n(&h->bag, (size_t)n)).ok()) return s;
  if (!(s = A.alloc_n(&h->n_used_dev, 1)).ok()) return s;
  {
    int32_t nn = (int32_t)n;
    CU(cudaMemcpy(h->n_used_dev, &nn, sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  // leaf renewal: a sum pair per (warp share, leaf) segment and each leaf's rank
  if (!(s = A.alloc_n(&h->leaf_sums, (size_t)K * (leaf_sum_warps(h) + L) * 2)).ok()) return s;
  if (!(s = A.alloc_n(&h->leaf_rank, (size_t)K * (L + 1))).ok()) return s;
  if (!(s = A.alloc_n(&h->leaf_values_dev, (size_t)K * L)).ok()) return s;
  if (cfg->persistent_grow) {
    if (!(s = A.alloc_n(&h->grow_sync, 1)).ok()) return s;
    if (!(s = A.alloc_n(&h->phase_ns, 4)).ok()) return s;
    CU(cudaMemset(h->grow_sync, 0, sizeof(GrowSync)));
    CU(cudaMemset(h->phase_ns, 0, 4 * sizeof(long long)));
  }
  if (mode == LGBM_B200_HIST_QUANT) {
    if (!(s = A.alloc_n(&h->maxbits, 2)).ok()) return s;
    if (!(s = A.alloc_n(&h->quant_counter, 1)).ok()) return s;
    CU(cudaMemset(h->maxbits, 0, 2 * sizeof(unsigned long long)));
    CU(cudaMemset(h->quant_counter, 0, sizeof(int32_t)));
    if (cfg->stochastic_rounding && !(s = quant_tables(h, n)).ok()) return s;
    h->start_eng = std::make_unique<Mt19937>((uint32_t)cfg->seed);
    if (!(s = A.alloc_n(&h->start_dev, (size_t)K)).ok()) return s;
    CU(cudaHostAlloc(reinterpret_cast<void**>(&h->start_h), sizeof(int64_t) * K, cudaHostAllocDefault));
  }
  // context
  DCtx& c = h->ctx;
  c.bins = bins_d;
  c.colbins = colbins_d;
  c.num_data = n;
  c.stride = h->stride;
  c.num_features = nf;
  c.total_bins = h->total_bins;
  c.hist_mode = mode;
  c.bagging = 0;
  // each partition posts its step's end for the next histogram launch (one
  // leading CTA) to run beside the row CTAs, off the step's critical path
  c.defer = 1;
  // LGBM_B200_DEFER=0: the partition's last CTA ends the step itself (A/B)
  if (const char* e = std::getenv("LGBM_B200_DEFER")) c.defer = std::atoi(e) != 0;
  // LGBM_B200_HIST_DIRECT=0: the quantized one-group histogram runs the
  // tile loop with block barriers instead of the direct loop (A/B)
  c.hist_direct = 1;
  if (const char* e = std::getenv("LGBM_B200_HIST_DIRECT")) c.hist_direct = std::atoi(e) != 0;
  // One slot and a single 32-byte row of at most 28 features: the packed
  // gradient of a row rides in its row's padding, so the direct histogram
  // loop reads one sector per row instead of two. LGBM_B200_Q_IN_ROW=0 keeps
  // it in its own array only (A/B).
  c.q_in_row = (mode == LGBM_B200_HIST_QUANT && K == 1 && h->ntiles == 1 && nf <= 28 && c.hist_direct) ? 1 : 0;
  if (const char* e = std::getenv("LGBM_B200_Q_IN_ROW"))
    if (std::atoi(e) == 0) c.q_in_row = 0;
  c.feats = feats_d;
  DParams& p = c.p;
  p.lambda_l1 = cfg->lambda_l1;
  p.lambda_l2 = cfg->lambda_l2;
  p.max_delta_step = cfg->max_delta_step;
  p.path_smooth = cfg->path_smooth;
  p.min_data_in_leaf = cfg->min_data_in_leaf;
  p.min_sum_hessian_in_leaf = cfg->min_sum_hessian_in_leaf;
  p.min_gain_to_split = cfg->min_gain_to_split;
  p.max_cat_to_onehot = cfg->max_cat_to_onehot;
  p.max_cat_threshold = cfg->max_cat_threshold;
  p.cat_l2 = cfg->cat_l2;
  p.cat_smooth = cfg->cat_smooth;
  p.min_data_per_group = cfg->min_data_per_group;
  p.num_leaves = L;
  p.max_depth = cfg->max_depth;
  p.monotone_penalty = cfg->monotone_penalty;
  p.use_monotone = use_monotone ? 1 : 0;
  for (int k = 0; k < K; ++k) c.slots[k] = h->slots_h[k];
  c.num_slots = K;
  c.rows_per_block = rpb;
  h->n_used = (int32_t)n;
  h->st_h.resize(K);
  h->trees.resize(K);
  h->timing = false;
  for (int i = 0; i < 4 * (h->L - 1); ++i) {
    cudaEvent_t e;
    CU(cudaEventCreate(&e));
    h->ev.push_back(e);
  }
  for (int i = 0; i < 16; ++i) CU(cudaEventCreate(&h->marks[i]));
  return Status();
}

// learner/quant.rs:364-398: the stochastic-rounding tables of `rows` rows,
// drawn per block by MT19937 (the block layout follows the reference's thread
// count), uploaded to new device arrays.
Status quant_tables(LgbmB200Learner* h, int64_t rows) {
  const LgbmB200LearnerConfig* cfg = &h->cfg;
  const size_t n = (size_t)rows;
  size_t nt = (size_t)std::max(1, cfg->quant_num_threads);
  size_t nb = std::max<size_t>(1, std::min(nt, (n + 511) / 512));
  size_t bs = n;
  if (nb > 1) bs = ((n + nb - 1) / nb + 31) / 32 * 32;
  std::vector<double> g(n), hh(n);
  for (size_t b = 0; b < nb; ++b) {
    size_t st = b * bs, en = std::min(n, st + bs);
    Mt19937 ge((uint32_t)(cfg->seed + (int32_t)b));
    Mt19937 he((uint32_t)(cfg->seed + (int32_t)b + (int32_t)nt));
    for (size_t i = st; i < en; ++i) {
      g[i] = ge.uniform01();
      hh[i] = he.uniform01();
    }
  }
  Status s;
  if (!(s = h->arena.alloc_n(&h->grv, n)).ok()) return s;
  if (!(s = h->arena.alloc_n(&h->hrv, n)).ok()) return s;
  CU(cudaMemcpy(h->grv, g.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(h->hrv, hh.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  return Status();
}

// Enqueue one whole tree (every slot) on the stream: init, the split steps
// and leaf renewal. Nothing here reads device memory back.
Status enqueue_tree(LgbmB200Learner* h) {
  const DCtx& c = h->ctx;
  const int K = h->K, L = h->L;
  const int mode = h->cfg.hist_precision;
  cudaStream_t s = h->stream;
  dim3 init_grid(h->root_grid, 1, K);
  k_tree_init<<<init_grid, 256, 0, s>>>(c, h->bagging ? h->bag : nullptr, h->n_used_dev);
  CU_LAUNCH();
  dim3 hist_grid(h->hist_grid, h->ntiles, K);
  dim3 scan_grid(h->nf, 2, K);
  dim3 part_grid(h->part_grid, 1, K);
  if (h->cfg.persistent_grow) {
    CU(cudaMemsetAsync(h->grow_sync, 0, sizeof(GrowSync), s));
    if (h->timing) CU(cudaMemsetAsync(h->phase_ns, 0, 4 * sizeof(long long), s));
    CU(launch_grow(mode, h->hist_ng, h->grow_grid, h->grow_smem, s, c, h->tiles, h->sub_rows, h->ntiles,
                   h->grow_sync, L - 1, h->timing ? h->phase_ns : nullptr));
  }
  for (int step = 0; step < (h->cfg.persistent_grow ? 0 : L - 1); ++step) {
    cudaEvent_t* ev = h->timing ? &h->ev[(size_t)4 * step] : nullptr;
    if (ev) CU(cudaEventRecordWithFlags(ev[0], s, cudaEventRecordExternal));
    // the three launches of a step chain by programmatic dependent launch
    // (not when events are recorded between them)
    const int pdl_edges = h->timing ? 0 : h->use_pdl;
    const bool pdl = (pdl_edges & 1) != 0, pdl_scan = (pdl_edges & 2) != 0, pdl_part = (pdl_edges & 4) != 0;
    CU(launch_hist(mode, h->hist_ng, hist_grid, h->hist_smem, s, c, h->tiles, h->sub_rows, pdl && step > 0,
                   c.defer && step > 0));
    if (ev) CU(cudaEventRecordWithFlags(ev[1], s, cudaEventRecordExternal));
    if (h->scan_part) {  // scans and partition in one launch: the scan interval records as empty
      if (ev) CU(cudaEventRecordWithFlags(ev[2], s, cudaEventRecordExternal));
      const dim3 g(h->scan_part_grid, 1, K);
      if (mode == LGBM_B200_HIST_QUANT) CU(launch_coop(k_scan_partition<true>, g, dim3(kPartThreads), h->scan_smem, s, c));
      else CU(launch_coop(k_scan_partition<false>, g, dim3(kPartThreads), h->scan_smem, s, c));
      if (ev) CU(cudaEventRecordWithFlags(ev[3], s, cudaEventRecordExternal));
      continue;
    }
    if (mode == LGBM_B200_HIST_QUANT && h->scan_warp) {
      const dim3 g(h->scan_warp_grid, 1, K);
      if (h->scan_wide)
        CU(launch_ex(k_scan_warp<kScanWideBlocks>, g, dim3(kScanThreads), 0, s, pdl_scan, c,
                     (const int32_t*)h->scan_items));
      else CU(launch_ex(k_scan_warp<2>, g, dim3(kScanThreads), 0, s, pdl_scan, c, (const int32_t*)h->scan_items));
    } else if (mode == LGBM_B200_HIST_QUANT) {
      if (h->scan_wide)
        CU(launch_ex(k_scan<true, kScanWideBlocks>, scan_grid, dim3(kScanThreads), h->scan_smem, s, pdl_scan, c));
      else CU(launch_ex(k_scan<true, 1>, scan_grid, dim3(kScanThreads), h->scan_smem, s, pdl_scan, c));
    } else if (h->scan_wide) {
      CU(launch_ex(k_scan<false, kScanWideBlocks>, scan_grid, dim3(kScanThreads), h->scan_smem, s, pdl_scan, c));
    } else {
      CU(launch_ex(k_scan<false, 1>, scan_grid, dim3(kScanThreads), h->scan_smem, s, pdl_scan, c));
    }
    if (ev) CU(cudaEventRecordWithFlags(ev[2], s, cudaEventRecordExternal));
    CU(launch_ex(k_partition, part_grid, dim3(256), 0, s, pdl_part, c));
    if (ev) CU(cudaEventRecordWithFlags(ev[3], s, cudaEventRecordExternal));
  }
  // the last split step's end (the earlier ones ran beside the histograms)
  const bool tail = c.defer && !h->cfg.persistent_grow && L > 1;
  if (tail) {
    k_finish<<<dim3(1, 1, K), kPartThreads, 0, s>>>(c);
    CU_LAUNCH();
  }
  if (mode == LGBM_B200_HIST_QUANT && h->cfg.quant_train_renew_leaf) {
    k_leaf_sums<<<dim3(leaf_sum_warps(h) / 8, 1, K), 256, 16 * (size_t)L, s>>>(c, h->leaf_sums, h->leaf_rank);
    CU_LAUNCH();
    k_leaf_renew<<<dim3(1, 1, K), 256, 0, s>>>(c, h->leaf_sums, h->leaf_rank, leaf_sum_warps(h), nullptr);
    CU_LAUNCH();
  }
  h->last_launches = 1 + (h->cfg.persistent_grow ? 1 : (h->scan_part ? 2 * (L - 1)
                                                                                   : 3 * (L - 1))) +
                     (tail ? 1 : 0) + ((mode == LGBM_B200_HIST_QUANT && h->cfg.quant_train_renew_leaf) ? 2 : 0);
  return Status();
}

// Data-parallel growth: one reduction over the ranks, in place on a device
// buffer, once this learner's stream has run up to here.
Status dp_allreduce(LgbmB200Learner* h, void* buf, int64_t count, int32_t dtype, int32_t op) {
  CU(cudaStreamSynchronize(h->stream));
  const int32_t rc = h->dp_fn(buf, count, dtype, op, h->dp_user);
  if (rc != 0) return Status(LGBM_B200_ERR_INTERNAL, "data-parallel all-reduce failed with " + std::to_string(rc));
  return Status();
}

static Status launch_scan(LgbmB200Learner* h, bool pdl) {
  const DCtx& c = h->ctx;
  const dim3 g(h->nf, 2, h->K);
  cudaStream_t s = h->stream;
  if (h->cfg.hist_precision == LGBM_B200_HIST_QUANT && h->scan_warp) {
    const dim3 gw(h->scan_warp_grid, 1, h->K);
    if (h->scan_wide)
      CU(launch_ex(k_scan_warp<kScanWideBlocks>, gw, dim3(kScanThreads), 0, s, pdl, c, (const int32_t*)h->scan_items));
    else CU(launch_ex(k_scan_warp<2>, gw, dim3(kScanThreads), 0, s, pdl, c, (const int32_t*)h->scan_items));
  } else if (h->cfg.hist_precision == LGBM_B200_HIST_QUANT) {
    if (h->scan_wide) CU(launch_ex(k_scan<true, kScanWideBlocks>, g, dim3(kScanThreads), h->scan_smem, s, pdl, c));
    else CU(launch_ex(k_scan<true, 1>, g, dim3(kScanThreads), h->scan_smem, s, pdl, c));
  } else if (h->scan_wide) {
    CU(launch_ex(k_scan<false, kScanWideBlocks>, g, dim3(kScanThreads), h->scan_smem, s, pdl, c));
  } else {
    CU(launch_ex(k_scan<false, 1>, g, dim3(kScanThreads), h->scan_smem, s, pdl, c));
  }
  return Status();
}

// One tree grown data-parallel (one slot): the launches of enqueue_tree, with
// the reductions over ranks between them. The host reads the slot state
// after every step, which is what keeps every rank's calls in step: the
// decisions come from the reduced histograms, so they are the same on every
// rank.
static Status run_tree_dp(LgbmB200Learner* h) {
  const DCtx& c = h->ctx;
  const int L = h->L;
  const int mode = h->cfg.hist_precision;
  cudaStream_t s = h->stream;
  const DSlot& d = h->slots_h[0];
  Status st;
  k_tree_init<<<dim3(h->root_grid, 1, 1), 256, 0, s>>>(c, nullptr, h->n_used_dev);
  CU_LAUNCH();
  k_dp_root_pack<<<1, 1, 0, s>>>(c, h->dp_f64, h->dp_i64);
  CU_LAUNCH();
  if (!(st = dp_allreduce(h, h->dp_f64, 2, LGBM_B200_DT_FLOAT64, LGBM_B200_OP_SUM)).ok()) return st;
  if (!(st = dp_allreduce(h, h->dp_i64, 2, LGBM_B200_DT_INT64, LGBM_B200_OP_SUM)).ok()) return st;
  k_dp_root_apply<<<1, 1, 0, s>>>(c, h->dp_f64, h->dp_i64);
  CU_LAUNCH();
  const size_t cells = (size_t)h->total_bins * (mode == LGBM_B200_HIST_QUANT ? 1 : 2);
  const dim3 hist_grid(h->hist_grid, h->ntiles, 1);
  for (int step = 0; step < L - 1; ++step) {
    DSlotState ss;
    CU(cudaMemcpyAsync(&ss, d.st, sizeof(ss), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (ss.done) break;
    CU(launch_hist(mode, h->hist_ng, hist_grid, h->hist_smem, s, c, h->tiles, h->sub_rows, false, false));
    if (ss.need_find) {  // the smaller leaf's histogram, summed over the ranks
      void* buf = static_cast<char*>(d.hist) + (size_t)ss.s_buf * cells * 8;
      const int32_t dt = mode == LGBM_B200_HIST_QUANT ? LGBM_B200_DT_INT64 : LGBM_B200_DT_FLOAT64;
      if (!(st = dp_allreduce(h, buf, (int64_t)cells, dt, LGBM_B200_OP_SUM)).ok()) return st;
    }
    if (!(st = launch_scan(h, false)).ok()) return st;
    CU(launch_ex(k_partition, dim3(h->part_grid, 1, 1), dim3(kPartThreads), 0, s, false, c));
    CU(cudaMemcpyAsync(&ss, d.st, sizeof(ss), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (ss.done) break;  // no leaf had a positive gain: the tree is finished
    if (!(st = dp_allreduce(h, d.dp_left, 1, LGBM_B200_DT_INT32, LGBM_B200_OP_SUM)).ok()) return st;
    k_dp_finish<<<1, kPartThreads, 0, s>>>(c);
    CU_LAUNCH();
  }
  if (mode == LGBM_B200_HIST_QUANT && h->cfg.quant_train_renew_leaf) {
    k_leaf_sums<<<dim3(leaf_sum_warps(h) / 8, 1, 1), 256, 16 * (size_t)L, s>>>(c, h->leaf_sums, h->leaf_rank);
    CU_LAUNCH();
    k_leaf_renew<<<1, 256, 0, s>>>(c, h->leaf_sums, h->leaf_rank, leaf_sum_warps(h), h->dp_f64);
    CU_LAUNCH();
    if (!(st = dp_allreduce(h, h->dp_f64, 2 * (int64_t)L, LGBM_B200_DT_FLOAT64, LGBM_B200_OP_SUM)).ok()) return st;
    k_dp_leaf_apply<<<1, 256, 0, s>>>(c, h->dp_f64);
    CU_LAUNCH();
  }
  h->last_launches = 0;
  return Status();
}

static Status run_tree(LgbmB200Learner* h) {
  if (h->dp) return run_tree_dp(h);
  cudaStream_t s = h->stream;
  // a cooperative launch is enqueued directly rather than captured
  const bool graph = h->cfg.use_cuda_graph != 0 && !h->cfg.persistent_grow;
  const int key = (h->bagging ? 1 : 0) + 2 * h->ctx.bagging + 4 * (h->timing ? 1 : 0);
  if (!graph) return enqueue_tree(h);
  if (h->graph_exec == nullptr || h->graph_key != key) {
    if (h->graph_exec) {
      cudaGraphExecDestroy(h->graph_exec);
      h->graph_exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    Status st = enqueue_tree(h);
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (!st.ok()) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return Status(LGBM_B200_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    CU(cudaGraphInstantiate(&h->graph_exec, g, 0));
    cudaGraphDestroy(g);
    h->graph_key = key;
  }
  CU(cudaGraphLaunch(h->graph_exec, s));
  return Status();
}

// Rebuilds one slot's tree as the reference's arrays, from the readback
// block's pinned mirror.
static Status read_tree(LgbmB200Learner* h, int k) {
  const DSlotState& st = h->st_h[k];
  HostTree& t = h->trees[k];
  const int nl = std::max(1, st.num_leaves_cur);
  const int nn = nl - 1;
  t.num_leaves = nl;
  // the slot's tree arrays from the pinned mirror of the readback block
  // (train_collect copied every slot's in one transfer)
  const unsigned char* base = h->rb_host + (size_t)k * h->rb_slot;
  const auto& rb = h->rb;
  auto get = [&](auto& vec, size_t offset, int count) {
    vec.resize((size_t)std::max(count, 0));
    if (count > 0) std::memcpy(vec.data(), base + offset, sizeof(vec[0]) * (size_t)count);
  };
  get(t.split_feature_inner, rb.sfi, nn);
  get(t.split_feature, rb.sf, nn);
  get(t.split_gain, rb.sg, nn);
  get(t.threshold_in_bin, rb.tib, nn);
  get(t.decision_type, rb.dt, nn);
  get(t.left_child, rb.lc, nn);
  get(t.right_child, rb.rc, nn);
  get(t.leaf_parent, rb.lp, nl);
  get(t.leaf_value, rb.lv, nl);
  get(t.leaf_weight, rb.lw, nl);
  get(t.leaf_count, rb.lcnt, nl);
  get(t.leaf_depth, rb.ld, nl);
  get(t.internal_value, rb.iv, nn);
  get(t.internal_weight, rb.iw, nn);
  get(t.internal_count, rb.ic, nn);
  get(t.cat_bits, rb.cb, nn * kCatWords);
  get(t.node_gain, rb.ng, nn);
  // real-valued thresholds and category bitsets (learner/mod.rs:1132-1165)
  t.threshold.assign((size_t)nn, 0.0);
  t.num_cat = 0;
  t.cat_boundaries.assign(1, 0);
  t.cat_boundaries_inner.assign(1, 0);
  t.cat_threshold.clear();
  t.cat_threshold_inner.clear();
  for (int node = 0; node < nn; ++node) {
    int inner = t.split_feature_inner[node];
    if (t.decision_type[node] & 1) {
      std::vector<uint32_t> bi, bc;
      for (int b = 0; b < kMaxBins; ++b) {
        if ((t.cat_bits[(size_t)node * kCatWords + b / 32] >> (b % 32)) & 1u) {
          size_t w = (size_t)(b / 32);
          if (bi.size() < w + 1) bi.resize(w + 1, 0);
          bi[w] |= 1u << (b % 32);
          int32_t cat = (inner < (int)h->bin_to_cat.size() && b < (int)h->bin_to_cat[inner].size())
                            ? h->bin_to_cat[inner][b]
                            : b;
          if (cat >= 0) {
            size_t wc = (size_t)(cat / 32);
            if (bc.size() < wc + 1) bc.resize(wc + 1, 0);
            bc[wc] |= 1u << (cat % 32);
          }
        }
      }
      t.threshold[node] = (double)t.threshold_in_bin[node];
      t.cat_boundaries.push_back(t.cat_boundaries.back() + (int32_t)bc.size());
      t.cat_threshold.insert(t.cat_threshold.end(), bc.begin(), bc.end());
      t.cat_boundaries_inner.push_back(t.cat_boundaries_inner.back() + (int32_t)bi.size());
      t.cat_threshold_inner.insert(t.cat_threshold_inner.end(), bi.begin(), bi.end());
      t.num_cat += 1;
    } else {
      uint32_t tb = t.threshold_in_bin[node];
      t.threshold[node] = (inner < (int)h->upper_bounds.size() && tb < h->upper_bounds[inner].size())
                              ? h->upper_bounds[inner][tb]
                              : (double)tb;
    }
  }
  return Status();
}

Status train(LgbmB200Learner* h, const float* grad, const float* hess, int32_t location) {
  Status st = train_enqueue(h, grad, hess, location);
  return st.ok() ? train_collect(h) : st;
}

// The quantization offsets of the next tree, one per slot in slot order:
// drawn from the tree-start engine (learner/quant.rs:114), or the last
// tree's again (`replay`). They go to pinned staging, which is written only
// after the stream's last synchronisation (every train and booster iteration
// ends with one), and which the copy in enqueue_quant reads when it runs.
void draw_quant_starts(LgbmB200Learner* h, bool replay) {
  const int K = h->K;
  if (h->last_start.size() < (size_t)K) h->last_start.resize((size_t)K, 0);
  for (int k = 0; k < K; ++k) {
    const int64_t rows = h->dp ? h->dp_global_n : h->n;  // the tables cover every rank's rows
    const int64_t start = replay ? h->last_start[k] : h->start_eng->uniform_int(0, (int32_t)rows);
    h->last_start[k] = start;
    h->start_h[k] = start;
  }
}

// The quantization of every slot's gradients (learner/quant.rs:92-158),
// enqueued: the offsets staged by draw_quant_starts, then each slot's max-abs
// and packing. Nothing here depends on host values that change per tree, so
// it can be captured once and replayed.
Status enqueue_quant(LgbmB200Learner* h) {
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  const int64_t offset = h->dp ? h->dp_offset : 0, table_n = h->dp ? h->dp_global_n : n;
  CU(cudaMemcpyAsync(h->start_dev, h->start_h, sizeof(int64_t) * h->K, cudaMemcpyHostToDevice, s));
  for (int k = 0; k < h->K; ++k) {
    int blocks = h->num_sms * 4;
    k_quant_absmax<<<blocks, 256, 0, s>>>(h->slots_h[k].gh, n, h->maxbits, h->quant_counter, h->slots_h[k].st,
                                          h->cfg.num_grad_quant_bins, h->cfg.is_constant_hessian, blocks,
                                          h->dp ? 0 : 1);
    CU_LAUNCH();
    if (h->dp) {  // the scales from the maxima over every rank
      Status st = dp_allreduce(h, h->maxbits, 2, LGBM_B200_DT_INT64, LGBM_B200_OP_MAX);
      if (!st.ok()) return st;
      k_quant_scales<<<1, 1, 0, s>>>(h->maxbits, h->slots_h[k].st, h->cfg.num_grad_quant_bins,
                                     h->cfg.is_constant_hessian);
      CU_LAUNCH();
    }
    k_quant_apply<<<blocks, 256, 0, s>>>(h->slots_h[k].gh, n, h->grv, h->hrv, h->start_dev + k, h->slots_h[k].st,
                                         h->cfg.is_constant_hessian, h->cfg.stochastic_rounding && h->grv,
                                         h->slots_h[k].packed, offset, table_n,
                                         h->ctx.q_in_row ? const_cast<uint8_t*>(h->ctx.bins) + 28 : nullptr,
                                         h->stride);
    CU_LAUNCH();
  }
  return Status();
}

// The gradients and their quantization for one tree, enqueued on the
// learner's stream. `replay` quantizes with the last call's offsets instead
// of drawing new ones (the autotuner's replays of the same tree).
static Status prepare_tree(LgbmB200Learner* h, const float* grad, const float* hess, int32_t location, bool replay) {
  const int K = h->K;
  const int64_t n = h->n;
  cudaStream_t s = h->stream;
  // gradients into the interleaved per-slot buffers
  if (grad) {
    if (location == LGBM_B200_HOST) {
      if (!h->score_scratch) {
        Status st = h->arena.alloc(reinterpret_cast<void**>(&h->score_scratch), sizeof(float) * 2 * n);
        if (!st.ok()) return st;
      }
      float* tmp = reinterpret_cast<float*>(h->score_scratch);
      for (int k = 0; k < K; ++k) {
        CU(cudaMemcpyAsync(tmp, grad + (size_t)k * n, sizeof(float) * n, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(tmp + n, hess + (size_t)k * n, sizeof(float) * n, cudaMemcpyHostToDevice, s));
        k_interleave<<<h->num_sms * 4, 256, 0, s>>>(tmp, tmp + n, n, const_cast<float2*>(h->slots_h[k].gh));
        CU_LAUNCH();
      }
    } else {
      for (int k = 0; k < K; ++k) {
        k_interleave<<<h->num_sms * 4, 256, 0, s>>>(grad + (size_t)k * n, hess + (size_t)k * n, n,
                                                    const_cast<float2*>(h->slots_h[k].gh));
        CU_LAUNCH();
      }
    }
  }
  if (h->cfg.hist_precision == LGBM_B200_HIST_QUANT) {
    draw_quant_starts(h, replay);
    return enqueue_quant(h);
  }
  return Status();
}

// Everything of one tree up to its growth, enqueued on the learner's stream.
Status train_enqueue(LgbmB200Learner* h, const float* grad, const float* hess, int32_t location) {
  CU(cudaSetDevice(h->device));
  Status st = prepare_tree(h, grad, hess, location, false);
  if (!st.ok()) return st;
  h->trained = true;
  h->last_ms[0] = h->last_ms[1] = h->last_ms[2] = h->last_ms[3] = 0;
  return run_tree(h);
}

// The trees of the last train_enqueue, read back once the stream has run
// (with every status check).
Status train_collect(LgbmB200Learner* h) {
  CU(cudaSetDevice(h->device));
  const int K = h->K;
  cudaStream_t s = h->stream;
  Status st;
  // every slot's state and tree arrays in one transfer
  CU(cudaMemcpyAsync(h->rb_host, h->rb_dev, h->rb_slot * (size_t)K, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  for (int k = 0; k < K; ++k)
    std::memcpy(&h->st_h[k], h->rb_host + (size_t)k * h->rb_slot + h->rb.st, sizeof(DSlotState));
  if (h->cfg.persistent_grow) {
    GrowSync gsh;
    long long ph[4] = {0, 0, 0, 0};
    CU(cudaMemcpyAsync(&gsh, h->grow_sync, sizeof(gsh), cudaMemcpyDeviceToHost, s));
    if (h->timing) CU(cudaMemcpyAsync(ph, h->phase_ns, sizeof(ph), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (gsh.status != 0) return Status(LGBM_B200_ERR_TIMEOUT, "device-side wait timed out (grid barrier)");
    // phase times seen by the first CTA: histogram, scan, partition, bookkeeping
    for (int i = 0; i < 4; ++i) h->last_ms[i] = (double)ph[i] / 1e6;
  } else if (h->timing) {  // per-kernel-family device time of this tree
    h->last_step_ms.assign((size_t)3 * (h->L - 1), 0.0f);
    for (int step = 0; step < h->L - 1; ++step) {
      cudaEvent_t* ev = &h->ev[(size_t)4 * step];
      float a, b, d;
      CU(cudaEventElapsedTime(&a, ev[0], ev[1]));
      CU(cudaEventElapsedTime(&b, ev[1], ev[2]));
      CU(cudaEventElapsedTime(&d, ev[2], ev[3]));
      h->last_ms[0] += a;
      h->last_ms[1] += b;
      h->last_ms[2] += d;
      h->last_step_ms[(size_t)3 * step] = a;
      h->last_step_ms[(size_t)3 * step + 1] = b;
      h->last_step_ms[(size_t)3 * step + 2] = d;
    }
  }
  h->last_hist_rows = 0;
  h->last_part_rows = 0;
  for (int k = 0; k < K; ++k) {
    const DSlotState& ss = h->st_h[k];
    h->last_hist_rows += ss.hist_rows;
    h->last_part_rows += ss.part_rows;
    if (ss.status == kStatusTimeout) return Status(LGBM_B200_ERR_TIMEOUT, "device-side wait timed out (partition)");
    if (ss.status == kStatusEmptyChild)
      return Status(LGBM_B200_ERR_INVALID_PARAMETER, "Check failed: (best_split_info.left_count) > (0)");
    if (!(st = read_tree(h, k)).ok()) return st;
  }
  return Status();
}

Status get_launch_shape(const LgbmB200Learner* h, LgbmB200LaunchShape* out) {
  out->partition_ctas = h->part_grid;
  out->hist_ctas = h->hist_grid;
  out->hist_rows_per_block = h->ctx.rows_per_block;
  return Status();
}

static Status check_launch_shape(const LgbmB200LaunchShape& in) {
  if (in.partition_ctas < 1 || in.partition_ctas > 65535 || in.hist_ctas < 1 || in.hist_ctas > 65535 ||
      in.hist_rows_per_block < 32 || in.hist_rows_per_block > (1 << 24))
    return Status(LGBM_B200_ERR_INVALID_PARAMETER, "launch shape out of range");
  return Status();
}

// No kernel sizes a buffer or a wait by these grids: the partition's tiles
// are claimed by ticket and its last CTA is found by an exit counter, the
// histogram CTAs split the leaf's rows among themselves. The cooperative
// scan + partition launch stays within what is resident at once.
Status set_launch_shape(LgbmB200Learner* h, const LgbmB200LaunchShape& in) {
  Status st = check_launch_shape(in);
  if (!st.ok()) return st;
  const int cl = hist_cluster(h->cfg.hist_precision);
  h->part_grid = in.partition_ctas;
  h->hist_grid = (in.hist_ctas + cl - 1) / cl * cl;
  h->ctx.rows_per_block = in.hist_rows_per_block;
  if (h->scan_part) h->scan_part_grid = std::max(1, std::min(h->part_grid, h->scan_part_max));
  h->config_epoch += 1;
  if (h->graph_exec) {  // the captured launches carry the old grids
    CU(cudaGraphExecDestroy(h->graph_exec));
    h->graph_exec = nullptr;
  }
  return Status();
}

Status autotune(LgbmB200Learner* h, const LgbmB200LaunchShape* cand, int32_t num, int32_t reps, int32_t* chosen,
                double* ms) {
  if (h->cfg.persistent_grow)
    return Status(LGBM_B200_ERR_UNSUPPORTED, "the persistent launch has no per-step launch shape");
  if (!h->trained) return Status(LGBM_B200_ERR_INVALID_PARAMETER, "autotune replays the last train call: train first");
  if (num < 1 || reps < 1 || reps > 1000) return Status(LGBM_B200_ERR_INVALID_PARAMETER, "candidates or reps");
  for (int32_t i = 0; i < num; ++i) {
    Status st = check_launch_shape(cand[i]);
    if (!st.ok()) return st;
  }
  CU(cudaSetDevice(h->device));
  cudaStream_t s = h->stream;
  // events and the per-step timing flag are restored on every exit
  struct Guard {
    LgbmB200Learner* h;
    bool timing;
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~Guard() {
      for (auto x : e)
        if (x) cudaEventDestroy(x);
      h->timing = timing;
    }
  } g{h, h->timing};
  h->timing = false;
  CU(cudaEventCreate(&g.e[0]));
  CU(cudaEventCreate(&g.e[1]));
  Status st = prepare_tree(h, nullptr, nullptr, LGBM_B200_DEVICE, true);
  if (!st.ok()) return st;
  std::vector<DSlotState> ss((size_t)h->K);
  std::vector<float> t((size_t)reps);
  int32_t best = -1;
  for (int32_t i = 0; i < num; ++i) {
    if (!(st = set_launch_shape(h, cand[i])).ok()) return st;
    if (!(st = run_tree(h)).ok()) return st;  // captures the graph
    for (int32_t r = 0; r < reps; ++r) {
      CU(cudaEventRecord(g.e[0], s));
      if (!(st = run_tree(h)).ok()) return st;
      CU(cudaEventRecord(g.e[1], s));
      CU(cudaEventSynchronize(g.e[1]));
      CU(cudaEventElapsedTime(&t[(size_t)r], g.e[0], g.e[1]));
    }
    for (int k = 0; k < h->K; ++k)
      CU(cudaMemcpyAsync(&ss[(size_t)k], h->slots_h[k].st, sizeof(DSlotState), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    for (const DSlotState& x : ss)
      if (x.status == kStatusTimeout) return Status(LGBM_B200_ERR_TIMEOUT, "device-side wait timed out (partition)");
    std::sort(t.begin(), t.end());
    ms[i] = (double)t[(size_t)reps / 2];
    if (best < 0 || ms[i] < ms[best]) best = i;
  }
  *chosen = best;
  return set_launch_shape(h, cand[best]);
}

// The learner's histogram kernel over an arbitrary row subset of the
// slot's current gradients (quantized: its current packed values), for the
// parity tests. Rows (host, in the given order) stand in for leaf 0.
Status histogram_of_rows(LgbmB200Learner* h, int slot, const uint32_t* rows, int64_t nrows, void* out) {
  CU(cudaSetDevice(h->device));
  cudaStream_t s = h->stream;
  const DSlot& d = h->slots_h[slot];
  const int64_t cnt = rows ? nrows : h->n;
  std::vector<uint32_t> r((size_t)cnt);
  for (int64_t i = 0; i < cnt; ++i) r[(size_t)i] = rows ? rows[i] : (uint32_t)i;
  CU(cudaMemcpyAsync(d.idx[0], r.data(), sizeof(uint32_t) * cnt, cudaMemcpyHostToDevice, s));
  int32_t zero = 0, c32 = (int32_t)cnt;
  CU(cudaMemcpyAsync(d.leaf_begin, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(d.leaf_count, &c32, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(d.leaf_side, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(d.buf_of, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  DSlotState ss;
  CU(cudaMemcpyAsync(&ss, d.st, sizeof(ss), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  ss.done = 0;
  ss.need_find = 1;
  ss.smaller.leaf = 0;
  ss.smaller.num_data = (int32_t)cnt;
  ss.s_count = (int32_t)cnt;
  ss.s_begin = 0;
  ss.s_side = 0;
  ss.s_buf = 0;
  ss.pending = 0;
  CU(cudaMemcpyAsync(d.st, &ss, sizeof(ss), cudaMemcpyHostToDevice, s));
  const int mode = h->cfg.hist_precision;
  const size_t cells = (size_t)h->total_bins * (mode == LGBM_B200_HIST_QUANT ? 1 : 2);
  CU(cudaMemsetAsync(d.hist, 0, cells * 8, s));
  // one slot only: a context whose slot array starts at `slot`
  DCtx c = h->ctx;
  c.slots[0] = h->ctx.slots[slot];
  dim3 grid(h->hist_grid, h->ntiles, 1);
  CU(launch_hist(mode, h->hist_ng, grid, h->hist_smem, s, c, h->tiles, h->sub_rows, false, false));
  CU_LAUNCH();
  CU(cudaMemcpyAsync(out, d.hist, cells * 8, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  return Status();
}

}  // namespace lgbm_b200

// ==========================================================================================
// C ABI
// ==========================================================================================
extern "C" {

const char* lgbm_b200_last_error(void) { return g_last_error.c_str(); }
const char* lgbm_b200_version(void) { return "lgbm_b200 0.1 (sm_100a)"; }

int lgbm_b200_dataset_create(const float* X, int64_t n, int32_t ncol, const LgbmB200BinParams* params,
                             LgbmB200Dataset** out) {
  if (!X || !params || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  auto d = std::make_unique<Dataset>();
  Status s = build_dataset(X, n, ncol, *params, *d);
  if (!s.ok()) return fail(s);
  *out = reinterpret_cast<LgbmB200Dataset*>(d.release());
  return LGBM_B200_OK;
}

int lgbm_b200_dataset_create_valid(const float* X, int64_t n, int32_t ncol, const LgbmB200Dataset* ref,
                                   LgbmB200Dataset** out) {
  if (!X || !ref || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  auto d = std::make_unique<Dataset>();
  Status s = build_valid_dataset(X, n, ncol, *reinterpret_cast<const Dataset*>(ref), *d);
  if (!s.ok()) return fail(s);
  *out = reinterpret_cast<LgbmB200Dataset*>(d.release());
  return LGBM_B200_OK;
}

int lgbm_b200_dataset_view(LgbmB200Dataset* ds, LgbmB200DatasetView* out) {
  if (!ds || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  reinterpret_cast<Dataset*>(ds)->fill_view(out);
  return LGBM_B200_OK;
}

int lgbm_b200_dataset_feature_infos(LgbmB200Dataset* ds, const char** out) {
  if (!ds || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  *out = reinterpret_cast<Dataset*>(ds)->infos().c_str();
  return LGBM_B200_OK;
}

int lgbm_b200_dataset_create_device(const float* X, int64_t n, int32_t ncol, const LgbmB200BinParams* params,
                                    int32_t device, LgbmB200Dataset** out) {
  if (!X || !params || !out || device < 0) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  auto d = std::make_unique<Dataset>();
  Status s = build_dataset(X, n, ncol, *params, *d, device);
  if (!s.ok()) return fail(s);
  *out = reinterpret_cast<LgbmB200Dataset*>(d.release());
  return LGBM_B200_OK;
}

int lgbm_b200_dataset_create_valid_device(const float* X, int64_t n, int32_t ncol, const LgbmB200Dataset* ref,
                                          int32_t device, LgbmB200Dataset** out) {
  if (!X || !ref || !out || device < 0) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  auto d = std::make_unique<Dataset>();
  Status s = build_valid_dataset(X, n, ncol, *reinterpret_cast<const Dataset*>(ref), *d, device);
  if (!s.ok()) return fail(s);
  *out = reinterpret_cast<LgbmB200Dataset*>(d.release());
  return LGBM_B200_OK;
}

void lgbm_b200_dataset_free(LgbmB200Dataset* ds) {
  delete reinterpret_cast<Dataset*>(ds);
  teardown_done("lgbm_b200_dataset_free");
}

int lgbm_b200_learner_create(const LgbmB200LearnerConfig* cfg, const uint8_t* bins, int64_t num_data,
                             int32_t num_features, const LgbmB200FeatureMeta* metas, const double* upper_bounds,
                             const int64_t* ub_offsets, const int32_t* bin_to_cat, const int64_t* cat_offsets,
                             LgbmB200Learner** out) {
  if (!cfg || !bins || !metas || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  auto h = std::make_unique<LgbmB200Learner>();
  Status s = setup_learner(h.get(), cfg, bins, num_data, num_features, metas);
  if (!s.ok()) return fail(s);
  h->upper_bounds.resize(num_features);
  h->bin_to_cat.resize(num_features);
  for (int32_t f = 0; f < num_features; ++f) {
    if (upper_bounds && ub_offsets)
      h->upper_bounds[f].assign(upper_bounds + ub_offsets[f], upper_bounds + ub_offsets[f + 1]);
    if (bin_to_cat && cat_offsets) h->bin_to_cat[f].assign(bin_to_cat + cat_offsets[f], bin_to_cat + cat_offsets[f + 1]);
  }
  *out = h.release();
  return LGBM_B200_OK;
}

void lgbm_b200_learner_destroy(LgbmB200Learner* h) {
  if (h) {
    cudaSetDevice(h->device);
    delete h;
    teardown_done("lgbm_b200_learner_destroy");
  }
}

int lgbm_b200_learner_set_bagging(LgbmB200Learner* h, const uint32_t* used, int64_t num_used, int32_t location) {
  if (!h) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null handle"));
  if (cudaSetDevice(h->device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  if (!used) {
    h->bagging = false;
    h->n_used = (int32_t)h->n;
    h->ctx.bagging = 0;
    int32_t nn = (int32_t)h->n;
    cudaError_t e0 = cudaMemcpyAsync(h->n_used_dev, &nn, sizeof(int32_t), cudaMemcpyHostToDevice, h->stream);
    if (e0 == cudaSuccess) e0 = cudaStreamSynchronize(h->stream);
    if (e0 != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e0)));
    h->config_epoch += 1;
    return LGBM_B200_OK;
  }
  if (num_used < 0 || num_used > h->n) return fail(Status(LGBM_B200_ERR_INVALID_DATA, "bag size"));
  cudaError_t e = cudaMemcpyAsync(h->bag, used, sizeof(uint32_t) * (size_t)num_used,
                                  location == LGBM_B200_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                  h->stream);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  int32_t nu = (int32_t)num_used;
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->n_used_dev, &nu, sizeof(int32_t), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  h->bagging = true;
  h->n_used = (int32_t)num_used;
  h->ctx.bagging = num_used < h->n ? 1 : 0;
  h->config_epoch += 1;
  return LGBM_B200_OK;
}

int lgbm_b200_learner_set_feature_mask(LgbmB200Learner* h, int32_t slot, const uint8_t* is_used) {
  if (!h || slot < 0 || slot >= h->K) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "slot"));
  cudaSetDevice(h->device);
  std::vector<uint8_t> m((size_t)h->nf, 1);
  if (is_used)
    for (int32_t f = 0; f < h->nf; ++f) m[f] = is_used[f] ? 1 : 0;
  cudaError_t e = cudaMemcpyAsync(h->slots_h[slot].bytree, m.data(), (size_t)h->nf, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  return LGBM_B200_OK;
}

int lgbm_b200_learner_train(LgbmB200Learner* h, const float* grad, const float* hess, int32_t is_first_tree,
                            int32_t location, LgbmB200TreeView* out) {
  if (!h || !grad || !hess) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  // is_first_tree only keeps the leaves of linear trees constant
  // (learner/mod.rs:571-572, :685); linear trees are not on this path
  (void)is_first_tree;
  Status s = lgbm_b200::train(h, grad, hess, location);
  if (!s.ok()) return fail(s);
  if (out)
    for (int k = 0; k < h->K; ++k) h->trees[k].view(&out[k]);
  return LGBM_B200_OK;
}

int lgbm_b200_learner_add_leaf_outputs(LgbmB200Learner* h, int32_t slot, const double* leaf_values,
                                       int32_t num_leaves, double* score, int32_t location) {
  if (!h || !leaf_values || !score || slot < 0 || slot >= h->K)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  cudaSetDevice(h->device);
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  const int L = h->L;
  std::vector<double> lv((size_t)L, 0.0);
  for (int l = 0; l < std::min(num_leaves, L); ++l) lv[l] = leaf_values[l];
  double* lvd = h->leaf_values_dev + (size_t)slot * L;
  cudaError_t e = cudaMemcpyAsync(lvd, lv.data(), sizeof(double) * L, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  // launch only over this slot: grid.z = 1 with a context whose slots start at `slot`
  DCtx c = h->ctx;
  c.slots[0] = h->ctx.slots[slot];
  if (location == LGBM_B200_HOST) {
    // Host scores: the leaf of every row is found first (in row order), then
    // the scores go through the device in chunks of rows, each chunk's copy
    // in, update and copy out on one of three streams, so that copies in and
    // out of different chunks overlap. The buffers are kept for the learner's
    // lifetime (a pool allocation per call would be mapped again each time).
    Status st;
    if (!h->score_stage) st = h->arena.alloc_n(&h->score_stage, (size_t)n);
    if (st.ok() && !h->leaf_of_row) st = h->arena.alloc_n(&h->leaf_of_row, (size_t)n);
    if (!st.ok()) return fail(st);
    if (!h->chunks.init()) return fail(Status(LGBM_B200_ERR_CUDA, "chunk streams"));
    e = cudaMemsetAsync(h->leaf_of_row, 0xFF, sizeof(int32_t) * n, s);  // -1: out of the bag
    if (e == cudaSuccess) {
      k_leaf_of_row<<<h->num_sms * 4, 256, 16 * (size_t)L, s>>>(c, h->leaf_of_row);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(h->chunks.ready, s);
    for (int64_t r0 = 0, k = 0; r0 < n && e == cudaSuccess; r0 += ChunkStreams::kRows, ++k) {
      const int64_t m = std::min<int64_t>(ChunkStreams::kRows, n - r0);
      cudaStream_t cs = h->chunks.s[k % ChunkStreams::kN];
      e = cudaStreamWaitEvent(cs, h->chunks.ready, 0);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->score_stage + r0, score + r0, sizeof(double) * m, cudaMemcpyHostToDevice, cs);
      if (e == cudaSuccess) {
        const int blocks = (int)std::min<int64_t>((m + 255) / 256, (int64_t)h->num_sms * 8);
        k_add_by_row<<<blocks, 256, 0, cs>>>(h->leaf_of_row + r0, lvd, h->score_stage + r0, m);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(score + r0, h->score_stage + r0, sizeof(double) * m, cudaMemcpyDeviceToHost, cs);
    }
    cudaError_t e2 = h->chunks.sync();
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
    return LGBM_B200_OK;
  }
  k_add_leaf_outputs<<<dim3(h->num_sms * 4, 1, 1), 256, 16 * (size_t)L, s>>>(c, lvd, 0, score, 0);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  return LGBM_B200_OK;
}

int lgbm_b200_learner_get_partition(LgbmB200Learner* h, int32_t slot, int32_t* leaf_begin, int32_t* leaf_count,
                                    uint32_t* indices) {
  if (!h || slot < 0 || slot >= h->K) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "slot"));
  cudaSetDevice(h->device);
  const DSlot& d = h->slots_h[slot];
  const int nl = std::max(1, h->st_h[slot].num_leaves_cur);
  std::vector<int32_t> side((size_t)nl), beg((size_t)nl), cnt((size_t)nl);
  cudaStream_t s = h->stream;
  cudaMemcpyAsync(beg.data(), d.leaf_begin, sizeof(int32_t) * nl, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(cnt.data(), d.leaf_count, sizeof(int32_t) * nl, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(side.data(), d.leaf_side, sizeof(int32_t) * nl, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "readback"));
  for (int l = 0; l < nl; ++l) {
    if (leaf_begin) leaf_begin[l] = beg[l];
    if (leaf_count) leaf_count[l] = cnt[l];
    if (indices && cnt[l] > 0)
      cudaMemcpyAsync(indices + beg[l], d.idx[side[l]] + beg[l], sizeof(uint32_t) * cnt[l], cudaMemcpyDeviceToHost, s);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "readback"));
  // The device keeps a split's left rows in their order and writes its right
  // rows reversed, so each leaf's rows are in ascending or descending order.
  // partition() hands them out ascending, as the reference's stable
  // partition does (partition.rs:107-174).
  if (indices) {
    for (int l = 0; l < nl; ++l) {
      if (cnt[l] < 2) continue;
      uint32_t* a = indices + beg[l];
      uint32_t* e = a + cnt[l];
      if (std::is_sorted(a, e)) continue;
      if (std::is_sorted(a, e, std::greater<uint32_t>())) std::reverse(a, e);
      else std::sort(a, e);
    }
  }
  return LGBM_B200_OK;
}

int lgbm_b200_learner_last_timing(LgbmB200Learner* h, double* ms, int64_t* hist_rows, int32_t* launches) {
  if (!h) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null handle"));
  if (ms)
    for (int i = 0; i < 4; ++i) ms[i] = h->last_ms[i];
  if (hist_rows) *hist_rows = h->last_hist_rows;
  if (launches) *launches = h->last_launches;
  return LGBM_B200_OK;
}

int lgbm_b200_learner_set_data_parallel(LgbmB200Learner* h, int64_t row_offset, int64_t global_num_data,
                                        LgbmB200AllReduceFn fn, void* user) {
  if (!h || !fn) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "set_data_parallel: null argument"));
  if (h->dp) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "set_data_parallel: already set"));
  if (h->K != 1)
    return fail(Status(LGBM_B200_ERR_UNSUPPORTED, "data-parallel growth takes one tree slot (no multiclass)"));
  if (h->bagging) return fail(Status(LGBM_B200_ERR_UNSUPPORTED, "data-parallel growth does not take bagging"));
  if (row_offset < 0 || global_num_data < row_offset + h->n || global_num_data > INT32_MAX)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "set_data_parallel: rows outside [0, global_num_data)"));
  if (cudaSetDevice(h->device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  DeviceArena& A = h->arena;
  DSlot& d = h->slots_h[0];
  Status s;
  const int L = h->L;
  if (!(s = A.alloc_n(&d.leaf_gcount, (size_t)L)).ok() || !(s = A.alloc_n(&d.dp_left, 2)).ok() ||
      !(s = A.alloc_n(&h->dp_f64, (size_t)(2 * L + 4))).ok() || !(s = A.alloc_n(&h->dp_i64, 4)).ok())
    return fail(s);
  if (!(s = A.alloc(reinterpret_cast<void**>(&d.dp_dec), kDpDecBytes)).ok()) return fail(s);
  if (h->cfg.hist_precision == LGBM_B200_HIST_QUANT && h->cfg.stochastic_rounding &&
      !(s = quant_tables(h, global_num_data)).ok())
    return fail(s);
  h->ctx.slots[0] = d;
  h->ctx.dp = 1;
  h->ctx.defer = 0;  // the step's end waits for the left count summed over the ranks
  h->scan_part = false;
  h->cfg.persistent_grow = 0;
  h->cfg.use_cuda_graph = 0;
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
  }
  h->dp = true;
  h->dp_offset = row_offset;
  h->dp_global_n = global_num_data;
  h->dp_fn = fn;
  h->dp_user = user;
  return LGBM_B200_OK;
}

int lgbm_b200_learner_step_times(LgbmB200Learner* h, float* ms, int32_t capacity, int32_t* steps) {
  if (!h || !steps) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  const int32_t n = (int32_t)(h->last_step_ms.size() / 3);
  *steps = n;
  if (ms)
    for (int32_t i = 0; i < std::min(n, capacity) * 3; ++i) ms[i] = h->last_step_ms[(size_t)i];
  return LGBM_B200_OK;
}

int lgbm_b200_learner_last_rows(LgbmB200Learner* h, int64_t* hist_rows, int64_t* partition_rows) {
  if (!h) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null handle"));
  if (hist_rows) *hist_rows = h->last_hist_rows;
  if (partition_rows) *partition_rows = h->last_part_rows;
  return LGBM_B200_OK;
}

int lgbm_b200_learner_histogram(LgbmB200Learner* h, int32_t slot, const uint32_t* rows, int64_t num_rows,
                                void* out) {
  if (!h || slot < 0 || slot >= h->K || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  Status st = lgbm_b200::histogram_of_rows(h, slot, rows, num_rows, out);
  if (!st.ok()) return fail(st);
  return LGBM_B200_OK;
}

int lgbm_b200_learner_quantized(LgbmB200Learner* h, int32_t slot, int64_t* packed, double* scales) {
  if (!h || slot < 0 || slot >= h->K) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "bad argument"));
  if (h->cfg.hist_precision != LGBM_B200_HIST_QUANT)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "the learner does not quantize gradients"));
  cudaSetDevice(h->device);
  std::vector<int32_t> v((size_t)h->n);
  DSlotState ss;
  cudaMemcpyAsync(v.data(), h->slots_h[slot].packed, sizeof(int32_t) * h->n, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(&ss, h->slots_h[slot].st, sizeof(ss), cudaMemcpyDeviceToHost, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "readback"));
  for (int64_t i = 0; i < h->n; ++i) {
    int64_t hq = (int64_t)(v[i] & 0xFFFF);
    int64_t gq = (int64_t)((v[i] - (int32_t)hq) >> 16);
    if (packed) packed[i] = (int64_t)((uint64_t)(gq << 32) + (uint64_t)hq);
  }
  if (scales) {
    scales[0] = ss.grad_scale;
    scales[1] = ss.hess_scale;
  }
  return LGBM_B200_OK;
}

int lgbm_b200_learner_record(LgbmB200Learner* h, int32_t mark) {
  if (!h || mark < 0 || mark >= 16) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "mark"));
  cudaSetDevice(h->device);
  cudaError_t e = cudaEventRecord(h->marks[mark], h->stream);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  return LGBM_B200_OK;
}

int lgbm_b200_learner_elapsed(LgbmB200Learner* h, int32_t a, int32_t b, double* ms) {
  if (!h || a < 0 || a >= 16 || b < 0 || b >= 16 || !ms) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "mark"));
  cudaSetDevice(h->device);
  float t = 0.f;
  cudaError_t e = cudaEventSynchronize(h->marks[b]);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, h->marks[a], h->marks[b]);
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  *ms = t;
  return LGBM_B200_OK;
}

int lgbm_b200_learner_get_launch_shape(LgbmB200Learner* h, LgbmB200LaunchShape* out) {
  if (!h || !out) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  Status st = lgbm_b200::get_launch_shape(h, out);
  return st.ok() ? LGBM_B200_OK : fail(st);
}

int lgbm_b200_learner_set_launch_shape(LgbmB200Learner* h, const LgbmB200LaunchShape* shape) {
  if (!h || !shape) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  if (cudaSetDevice(h->device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  Status st = lgbm_b200::set_launch_shape(h, *shape);
  return st.ok() ? LGBM_B200_OK : fail(st);
}

int lgbm_b200_learner_autotune(LgbmB200Learner* h, const LgbmB200LaunchShape* candidates, int32_t num_candidates,
                               int32_t reps, int32_t* chosen, double* ms_per_tree) {
  if (!h || !candidates || !chosen || !ms_per_tree)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null argument"));
  Status st = lgbm_b200::autotune(h, candidates, num_candidates, reps, chosen, ms_per_tree);
  return st.ok() ? LGBM_B200_OK : fail(st);
}

int lgbm_b200_learner_set_timing(LgbmB200Learner* h, int32_t enabled) {
  if (!h) return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "null handle"));
  h->timing = enabled != 0;
  return LGBM_B200_OK;
}

}  // extern "C"
