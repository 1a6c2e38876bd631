// The tree learner's sm_100a kernels. One tree (or one tree per class slot,
// grown in lockstep) is grown entirely on the device: every kernel reads
// the current leaf, counts and split from the slot's control block, so the
// per-split launches need no host round trip and can be captured in a CUDA
// graph.
//
// Per split step (learner/mod.rs:653-666):
//   k_hist       histogram of the smaller leaf      (multi_val_bin.rs:556-703)
//   k_scan       fix / subtract / threshold scan per feature, then in the
//                last CTA: best split per leaf, best leaf, Tree::split
//                bookkeeping and the partition LUT  (learner/mod.rs:816-1225,
//                split.rs, histogram.rs:42-85, tree.rs:254-297)
//   k_partition  stable-by-leaf row split with decoupled look-back, then the
//                smaller/larger choice and before_find_best_split
//                (partition.rs:107-174, learner/mod.rs:1200-1208, :712-731)
#include <cooperative_groups.h>

#include <type_traits>

#include "device_common.cuh"
#include "kernels.h"
#include "scan_warp.cuh"

namespace lgbm_b200 {

// =====================================================================================
// tree init: DataPartition::init, root sums and the root LeafSplits
// (learner/mod.rs:572-648, partition.rs:202-218)
// =====================================================================================
__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ bool before_find_best_split(const DCtx& c, const DSlot& s, int32_t left, int32_t right) {
  const DParams& p = c.p;
  if (p.max_depth > 0 && s.tree.leaf_depth[left] >= p.max_depth) {
    s.best[left].gain = -INFINITY;
    s.bgain[left] = -INFINITY;
    if (right >= 0) {
      s.best[right].gain = -INFINITY;
      s.bgain[right] = -INFINITY;
    }
    return false;
  }
  int32_t nl = left >= 0 ? s.leaf_gcount[left] : 0;
  int32_t nr = right >= 0 ? s.leaf_gcount[right] : 0;
  int32_t min2 = p.min_data_in_leaf * 2;
  if (nr < min2 && nl < min2) {
    s.best[left].gain = -INFINITY;
    s.bgain[left] = -INFINITY;
    if (right >= 0) {
      s.best[right].gain = -INFINITY;
      s.bgain[right] = -INFINITY;
    }
    return false;
  }
  return true;
}

// Grid (kRootBlocks, 1, slots), 256 threads.
__global__ void __launch_bounds__(256) k_tree_init(const __grid_constant__ DCtx c, const uint32_t* bag, const int32_t* n_used) {
  const DSlot& s = c.slots[blockIdx.z];
  const int64_t n = *n_used;
  const int tid = threadIdx.x;
  // positions -> rows (identity, or the in-bag rows)
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + tid; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s.idx[0][i] = bag ? bag[i] : (uint32_t)i;
  // zero the root's histogram buffer (pool buffer 0)
  size_t cells = (size_t)c.total_bins * (c.hist_mode == LGBM_B200_HIST_QUANT ? 1 : 2);
  double* h0 = reinterpret_cast<double*>(s.hist);  // cells are 8 bytes in every form
  for (size_t i = (size_t)blockIdx.x * blockDim.x + tid; i < cells; i += (size_t)gridDim.x * blockDim.x) h0[i] = 0.0;

  // deterministic partial sums over this block's contiguous chunk (a
  // multiple of 8 rows, so that the in-order loops below load 16-byte
  // aligned groups)
  const int64_t chunk = ((n + gridDim.x - 1) / gridDim.x + 7) & ~(int64_t)7;
  const int64_t b0 = min(n, (int64_t)blockIdx.x * chunk), b1 = min(n, b0 + chunk);
  double sg = 0.0, sh = 0.0;
  long long si = 0;
  if (c.hist_mode == LGBM_B200_HIST_QUANT && !bag) {
    // rows in order: eight packed values per thread and iteration
    const double gsc = s.st->grad_scale, hsc = s.st->hess_scale;
    for (int64_t i = b0 + 8 * (int64_t)tid; i < b1; i += 8 * (int64_t)blockDim.x) {
      int32_t w[8];
      if (i + 8 <= b1) {
        const int4 a = *reinterpret_cast<const int4*>(s.packed + i);
        const int4 b = *reinterpret_cast<const int4*>(s.packed + i + 4);
        w[0] = a.x, w[1] = a.y, w[2] = a.z, w[3] = a.w, w[4] = b.x, w[5] = b.y, w[6] = b.z, w[7] = b.w;
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) w[j] = i + j < b1 ? s.packed[i + j] : 0;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int64_t gq = (int64_t)(w[j] >> 16), hq = (int64_t)(w[j] & 0xFFFF);
        si += (long long)((uint64_t)(gq << 32) + (uint64_t)hq);
        sg += (double)(w[j] >> 16) * gsc;
        sh += (double)(w[j] & 0xFFFF) * hsc;
      }
    }
  } else if (c.hist_mode == LGBM_B200_HIST_QUANT) {
    for (int64_t i = b0 + tid; i < b1; i += blockDim.x) {
      // quant.rs:452-477: the bag variant sums packed values by position
      int64_t r = (c.bagging) ? i : (int64_t)(bag ? bag[i] : (uint32_t)i);
      int32_t v = s.packed[r];
      int64_t gq = (int64_t)(v >> 16), hq = (int64_t)(v & 0xFFFF);
      si += (long long)((uint64_t)(gq << 32) + (uint64_t)hq);
      int32_t w = s.packed[bag ? bag[i] : (uint32_t)i];
      if (c.bagging) {  // f32 scales (quant.rs:467-477)
        sg += (double)((float)(w >> 16) * (float)s.st->grad_scale);
        sh += (double)((float)(w & 0xFFFF) * (float)s.st->hess_scale);
      } else {
        sg += (double)(w >> 16) * s.st->grad_scale;
        sh += (double)(w & 0xFFFF) * s.st->hess_scale;
      }
    }
  } else if (!bag && (reinterpret_cast<uintptr_t>(s.gh) & 15) == 0) {
    // rows in order: four (g, h) pairs per thread and iteration (a slot's
    // pairs start 16-byte aligned unless the row count is odd)
    for (int64_t i = b0 + 4 * (int64_t)tid; i < b1; i += 4 * (int64_t)blockDim.x) {
      float2 v[4];
      if (i + 4 <= b1) {
        const float4 a = *reinterpret_cast<const float4*>(s.gh + i);
        const float4 b = *reinterpret_cast<const float4*>(s.gh + i + 2);
        v[0] = make_float2(a.x, a.y), v[1] = make_float2(a.z, a.w), v[2] = make_float2(b.x, b.y),
        v[3] = make_float2(b.z, b.w);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = i + j < b1 ? s.gh[i + j] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        sg += (double)v[j].x;
        sh += (double)v[j].y;
      }
    }
  } else {
    for (int64_t i = b0 + tid; i < b1; i += blockDim.x) {
      float2 v = s.gh[bag ? bag[i] : (uint32_t)i];
      sg += (double)v.x;
      sh += (double)v.y;
    }
  }
  __shared__ double red_g[8], red_h[8];
  __shared__ long long red_i[8];
  sg = warp_sum_d(sg);
  sh = warp_sum_d(sh);
  si = warp_sum_ll(si);
  if ((tid & 31) == 0) {
    red_g[tid >> 5] = sg;
    red_h[tid >> 5] = sh;
    red_i[tid >> 5] = si;
  }
  __syncthreads();
  __shared__ bool last;
  if (tid == 0) {
    double a = 0, b = 0;
    long long d = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += red_g[w];
      b += red_h[w];
      d += red_i[w];
    }
    s.root_partials[blockIdx.x] = a;
    s.root_partials[kRootBlocks + blockIdx.x] = b;
    s.root_ipartials[blockIdx.x] = d;
    __threadfence();
    last = atomicAdd(s.root_counter, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const DParams& p = c.p;
  DSlotState* st = s.st;
  // per-leaf state
  for (int l = tid; l < p.num_leaves; l += blockDim.x) {
    s.best[l].feature = -1;
    s.best[l].inner = -1;
    s.best[l].gain = -INFINITY;
    s.bgain[l] = -INFINITY;
    s.bfeat[l] = -1;
    s.cmin[l] = -1.7976931348623157e308;
    s.cmax[l] = 1.7976931348623157e308;
    s.buf_of[l] = l;
    s.leaf_begin[l] = 0;
    s.leaf_count[l] = 0;
    s.leaf_gcount[l] = 0;
    s.leaf_side[l] = 0;
  }
  for (int f = tid; f < c.num_features; f += blockDim.x) s.splittable[f] = 1;
  __syncthreads();
  if (tid != 0) return;
  *s.root_counter = 0;
  double a = 0, b = 0;
  long long d = 0;
  for (int k = 0; k < (int)gridDim.x; ++k) {
    a += s.root_partials[k];
    b += s.root_partials[kRootBlocks + k];
    d += s.root_ipartials[k];
  }
  s.leaf_count[0] = (int32_t)n;
  s.leaf_gcount[0] = (int32_t)n;  // data-parallel: the global count replaces it after the root sums' reduction
  st->num_used = (int32_t)n;
  st->num_leaves_cur = 1;
  st->done = 0;
  st->status = kStatusOk;
  st->num_cat = 0;
  st->scan_done = 0;
  st->part_ticket = 0;
  st->part_done = 0;
  st->pending = 0;
  st->hist_rows = 0;
  st->part_rows = 0;
  st->smaller.leaf = 0;
  st->smaller.num_data = (int32_t)n;
  st->s_begin = 0;
  st->s_count = (int32_t)n;
  st->s_side = 0;
  st->s_buf = 0;
  st->l_buf = -1;
  st->smaller.sum_gradients = a;
  st->smaller.sum_hessians = b;
  st->smaller.int_sum = (int64_t)d;
  st->larger.leaf = -1;
  st->larger.num_data = 0;
  st->left_leaf = 0;
  st->right_leaf = -1;
  const DTree& t = s.tree;
  t.leaf_parent[0] = -1;
  t.leaf_value[0] = maybe_round_to_zero(root_output(a, b, p, (int32_t)n));
  t.leaf_weight[0] = 0.0;
  t.leaf_count[0] = 0;
  t.leaf_depth[0] = 0;
  st->need_find = before_find_best_split(c, s, 0, -1) ? 1 : 0;
}

// =====================================================================================
// histogram of the smaller leaf (multi_val_bin.rs:556-703, :710-791)
// =====================================================================================
struct LeafRows {
  const uint32_t* idx;  // position -> row
  int64_t begin, count;
  int32_t buf;          // the leaf's histogram buffer
};

// Rows [r0, r1) of the smaller leaf for this CTA. CTAs are used in whole
// clusters of kCl so that every CTA of a used cluster takes part in
// the cluster's reduction (its row range may be empty); returns false for
// CTAs of unused clusters and when no histogram is needed.
template <int kCl>
__device__ __forceinline__ bool hist_setup(const DCtx& c, const DSlot& s, int rank, int count, LeafRows& lr,
                                           int64_t& r0, int64_t& r1) {
  DSlotState* st = s.st;
  // every field read at once
  const int32_t done = st->done, need = st->need_find, count_s = st->s_count, begin_s = st->s_begin,
                side_s = st->s_side, buf_s = st->s_buf;
  const int32_t pending = st->pending, pbegin = st->pd_begin, pcnt = st->pd_cnt, pside = st->pd_side,
                pdepth = st->pd_depth, pR = st->pd_R, status = st->status, left = st->part_left;
  if (pending) {
    // The previous step's end runs beside this launch: the smaller child's
    // range and before_find_best_split as partition_finalize derives them.
    // (A step end that records a status sets done; either value read here
    // leads to the same skip.)
    if (done || status != kStatusOk) return false;
    const int32_t nl = pcnt > 0 ? left : 0, nr = pcnt - nl;
    const bool left_smaller = nl < nr;
    const int32_t sc = left_smaller ? nl : nr;
    if (sc <= 0) return false;
    if (c.p.max_depth > 0 && pdepth >= c.p.max_depth) return false;
    if (nr < c.p.min_data_in_leaf * 2 && nl < c.p.min_data_in_leaf * 2) return false;
    lr.buf = pR;
    lr.count = sc;
    lr.begin = left_smaller ? pbegin : pbegin + nl;
    lr.idx = pside == 0 ? s.idx[1] : s.idx[0];
  } else {
    if (done || !need) return false;
    lr.buf = buf_s;
    lr.count = count_s;
    lr.begin = begin_s;
    lr.idx = side_s == 0 ? s.idx[0] : s.idx[1];
  }
  int64_t per = c.rows_per_block;
  int64_t active = min((int64_t)count, (lr.count + per - 1) / per);
  active = (active + kCl - 1) / kCl * kCl;
  if ((int64_t)rank >= active) return false;
  int64_t chunk = (lr.count + active - 1) / active;
  r0 = min(lr.count, (int64_t)rank * chunk);
  r1 = min(lr.count, r0 + chunk);
  return true;
}

// Feature tile of a histogram launch: features [f0, f1), stored bins [bin0, bin0 + nbins).
__device__ __forceinline__ void tile_of(const DTileTable& tt, int tile, int& f0, int& f1, int& bin0, int& nbins) {
  f0 = tt.f0[tile];
  f1 = tt.f0[tile + 1];
  bin0 = tt.bin0[tile];
  nbins = tt.bin0[tile + 1] - bin0;
}

// Histogram of the smaller leaf's rows over one feature tile of kNG groups of
// 32 features. The CTA walks its rows in tiles of kHistTileRows (one row per
// thread): a thread loads its row index, its gradient pair and the row's
// 32 x kNG bin bytes (16-byte vector loads of the row-major matrix) into
// registers one tile ahead, so the gathers of the next tile are in flight
// while the current tile is accumulated. A tile is staged in shared memory
// and accumulated in a bin-major layout: feature f0 + 32g + lane keeps its
// cell of stored value `raw` at cells[g][raw][lane], so in every warp-wide
// atomic the 32 lanes touch 32 different banks. Stored value 0 (the most
// frequent bin) and the zero padding of short rows land in cells[g][0],
// which no feature view contains.
//   kMode 0: FP64 g / h cells (the reference's sums, reordered by atomics)
//   kMode 1: FP32 (hi, lo) pairs per value, the rounding error of every
//            add kept in lo (TwoSum), merged in FP64 when flushed
//   kMode 2: int32 cells holding (g << 16) + h of quantized gradients,
//            flushed at least every `sub_rows` rows into packed int64 sums
// The quantized form runs in clusters of kHistCluster CTAs: at the end every
// CTA reduces one slice of the cells over the cluster's shared memories
// (distributed shared memory) and adds it to the leaf histogram, so a
// cluster issues one global atomic per cell instead of one per CTA. The
// float forms (one 148 KB CTA per SM) flush each CTA's own cells.
template <int kMode, int kNG, int kCl>
__device__ void hist_body(const DCtx& c, const DSlot& s, const DTileTable& tt, int tile, const LeafRows& lr,
                          int64_t r0, int64_t r1, int32_t sub_rows, unsigned char* smem_raw) {
  namespace cg = cooperative_groups;
  int f0, f1, bin0, nbins;
  tile_of(tt, tile, f0, f1, bin0, nbins);
  (void)nbins;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = kHistThreads / 32;
  constexpr int kRowsPerWarp = kHistTileRows / kWarps;
  static_assert(kRowsPerWarp == 32, "one staged row per lane of a warp");
  static_assert(kNG >= 1 && kNG <= 4, "the row loop dispatches 1 to 4 lane groups");
  constexpr int kCellBytes = kMode == 2 ? 4 : 16;
  constexpr int kGroupCells = kMaxBins * 32;
  constexpr int kRowBytes = 32 * kNG;
  const int ngroups = (f1 - f0 + 31) >> 5;  // <= kNG
  unsigned char* cells = smem_raw;
  uint4* sbins = reinterpret_cast<uint4*>(smem_raw + (size_t)kNG * kGroupCells * kCellBytes);
  int32_t* sq = reinterpret_cast<int32_t*>(sbins + kHistTileRows * 2 * kNG);
  float2* sgh = reinterpret_cast<float2*>(sq);
  __shared__ int32_t s_vlen[32 * kNG], s_vstart[32 * kNG];
  static_assert(32 * kNG <= kHistThreads, "one feature view per thread");
  // the views are stored to shared memory after the first gathers are issued
  int32_t my_vlen = 0, my_vstart = 0;
  if (threadIdx.x < 32 * kNG) {
    const int f = f0 + (int)threadIdx.x;
    if (((int)threadIdx.x >> 5) < ngroups && f < f1) {
      my_vlen = c.feats[f].view_len;
      my_vstart = c.feats[f].view_start;
    }
  }
  {
    uint4* z = reinterpret_cast<uint4*>(cells);
    const int n16 = ngroups * kGroupCells * kCellBytes / 16;
    for (int i = threadIdx.x; i < n16; i += kHistThreads) z[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  const uint32_t* idx = lr.idx + lr.begin;
  const size_t stride = (size_t)c.stride;
  double* outf = reinterpret_cast<double*>(s.hist) + (size_t)lr.buf * c.total_bins * 2;
  unsigned long long* outi = reinterpret_cast<unsigned long long*>(s.hist) + (size_t)lr.buf * c.total_bins;
  // Adds cell i (over groups) of the CTAs `src` to the leaf histogram; cells
  // outside the features' views are skipped.
  auto emit = [&](int i, auto read_cell) {
    const int g = i / kGroupCells, k = i % kGroupCells;
    const int raw = k >> 5, fl = (g << 5) | (k & 31);
    if (raw == 0 || raw > s_vlen[fl]) return;
    const size_t dst = (size_t)s_vstart[fl] + raw - 1;
    if constexpr (kMode == 2) {
      int64_t gq, hq;
      read_cell(i, gq, hq);
      if (gq != 0 || hq != 0) atomicAdd(outi + dst, (unsigned long long)((uint64_t)(gq << 32) + (uint64_t)hq));
    } else {
      double gv, hv;
      read_cell(i, gv, hv);
      if (gv != 0.0 || hv != 0.0) {
        atomicAdd(outf + 2 * dst, gv);
        atomicAdd(outf + 2 * dst + 1, hv);
      }
    }
  };
  // the (g, h) of cell i in the shared memory `base` of one CTA
  auto cell_of = [&](const unsigned char* base, int i, auto& gv, auto& hv) {
    if constexpr (kMode == 2) {
      const int32_t cell = reinterpret_cast<const int32_t*>(base)[i];
      const int64_t h = (int64_t)(cell & 0xFFFF);
      gv = (int64_t)((cell - (int32_t)h) >> 16);
      hv = h;
    } else if constexpr (kMode == 0) {
      const int g = i / kGroupCells, k = i % kGroupCells;
      const double* d = reinterpret_cast<const double*>(base + (size_t)g * kGroupCells * 16);
      gv = d[k];
      hv = d[kGroupCells + k];
    } else {
      const int g = i / kGroupCells, k = i % kGroupCells;
      const float* fl = reinterpret_cast<const float*>(base + (size_t)g * kGroupCells * 16);
      gv = (double)fl[k] + (double)fl[kGroupCells + k];
      hv = (double)fl[2 * kGroupCells + k] + (double)fl[3 * kGroupCells + k];
    }
  };
  bool direct = false;
  if constexpr (kMode == 2 && kNG == 1) {
    direct = c.hist_direct != 0;
    if (direct) {
      // Direct row loop (quantized, one lane group), without tile barriers.
      // A warp adds its rows four at a time: lane l takes word a = l & 7
      // (features f0 + 4a .. f0 + 4a + 3) of row j = l >> 3 and in pass k
      // (0..3) adds byte b = (k + j) & 3 of it, feature 4a + b, whose cell
      // raw * 32 + 4a + b lies in bank 4a + b: the 32 lanes of every
      // warp-wide atomic touch 32 different banks.
      if (threadIdx.x < 32) {
        s_vlen[threadIdx.x] = my_vlen;
        s_vstart[threadIdx.x] = my_vstart;
      }
      const int j = lane >> 3, a = lane & 7;
      int32_t* icells = reinterpret_cast<int32_t*>(cells);
      // positions in the leaf fit 31 bits
      const int32_t R0 = (int32_t)r0, R1 = (int32_t)r1;
      // pass k: the shared address of the cell of stored value 0 of this
      // lane's feature (value v adds v * 128 bytes); the word is rotated by
      // j bytes once, so that pass k takes its byte k
      uint32_t cb[4];
      const uint32_t cells_s = (uint32_t)__cvta_generic_to_shared(icells);
#pragma unroll
      for (int k = 0; k < 4; ++k) cb[k] = cells_s + 4u * (4u * (uint32_t)a + (uint32_t)((k + j) & 3));
      const uint32_t rot = 8u * (uint32_t)j;
      // The rows are staged by asynchronous copies: each warp keeps a private
      // ring of kS stages of 16 rows (their 32-byte bin segments, and their
      // gradients when these do not ride in the rows) in shared memory and
      // copies kS - 1 batches ahead of the one it adds, so the bytes in flight
      // take no registers. kQ: the packed gradient is the row's word 7.
      auto rows_async = [&](auto q_in_row) {
        constexpr bool kQ = decltype(q_in_row)::value;
        constexpr int kS = kHistAsyncStages;
        constexpr int kRowsB = 16;                  // rows per warp and batch
        constexpr int32_t kStep = kWarps * kRowsB;  // rows per CTA and batch
        constexpr uint32_t kStageBytes = kRowsB * 32 + kRowsB * 4;
        const uint32_t ring = (uint32_t)__cvta_generic_to_shared(smem_raw + (size_t)kGroupCells * 4) +
                              (uint32_t)warp * kS * kStageBytes;
        const unsigned char* rowsrc = c.bins + f0 + 16 * (lane & 1);  // lane l copies half (l & 1) of row l >> 1
        for (int32_t seg0 = R0; seg0 < R1;) {
          const int32_t seg1 = seg0 + min(R1 - seg0, sub_rows);
          const int32_t b0 = seg0 + warp * kRowsB;
          auto load_rid = [&](int32_t bt) {
            const int32_t pos = bt + (lane >> 1);
            return pos < seg1 ? __ldcg(idx + pos) : 0u;
          };
          auto issue = [&](int32_t bt, int stage, uint32_t rid) {
            const uint32_t st_addr = ring + (uint32_t)stage * kStageBytes;
            if (bt + (lane >> 1) < seg1) {
              const unsigned char* src = rowsrc + (size_t)rid * stride;
              asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(st_addr + 16u * (uint32_t)lane), "l"(src)
                           : "memory");
            }
            if constexpr (!kQ) {
              const uint32_t ridq = __shfl_sync(0xffffffffu, rid, (lane * 2) & 31);  // row `lane`'s index
              if (lane < kRowsB && bt + lane < seg1)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(st_addr + kRowsB * 32 + 4u * (uint32_t)lane),
                             "l"(s.packed + ridq)
                             : "memory");
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
          };
          // batches 0 .. kS - 2 in flight, the indices of batch kS - 1 loaded
          {
            uint32_t r[kS - 1];
#pragma unroll
            for (int t = 0; t < kS - 1; ++t) r[t] = load_rid(b0 + t * kStep);
#pragma unroll
            for (int t = 0; t < kS - 1; ++t) issue(b0 + t * kStep, t, r[t]);
          }
          uint32_t rid_next = load_rid(b0 + (kS - 1) * kStep);
          // every cell is zeroed (above, or by the last flush) before the first add
          if (seg0 == R0) __syncthreads();
          int stage = 0;
          for (int32_t bt = b0; bt < seg1; bt += kStep) {
            issue(bt + (kS - 1) * kStep, stage == 0 ? kS - 1 : stage - 1, rid_next);
            rid_next = load_rid(bt + kS * kStep);
            asm volatile("cp.async.wait_group %0;" ::"n"(kS - 1) : "memory");
            __syncwarp();
            const uint32_t st_addr = ring + (uint32_t)stage * kStageBytes;
            uint32_t w[4];
            int32_t q[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int rr = 4 * u + j;
              const bool live = bt + rr < seg1;
              uint32_t x, y;
              asm volatile("ld.shared.u32 %0, [%1];" : "=r"(x) : "r"(st_addr + 32u * rr + 4u * a) : "memory");
              if constexpr (kQ) {
                asm volatile("ld.shared.u32 %0, [%1];" : "=r"(y) : "r"(st_addr + 32u * rr + 28u) : "memory");
              } else {
                asm volatile("ld.shared.u32 %0, [%1];" : "=r"(y) : "r"(st_addr + kRowsB * 32 + 4u * rr) : "memory");
              }
              w[u] = __funnelshift_r(x, x, rot);  // byte k is the row's byte (k + j) & 3
              q[u] = live ? (int32_t)y : 0;       // a dead row adds 0 wherever its stale word points
            }
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const uint32_t addr = cb[k] + (__byte_perm(w[u], 0u, 0x4440u | k) << 7);
                asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(addr), "r"(q[u]) : "memory");
              }
            __syncwarp();  // the stage is refilled by the next batch's copies
            stage = stage == kS - 1 ? 0 : stage + 1;
          }
          asm volatile("cp.async.wait_all;" ::: "memory");
          seg0 = seg1;
          if (seg0 < R1) {
            __syncthreads();
            for (int i = threadIdx.x; i < kGroupCells; i += kHistThreads) {
              emit(i, [&](int ii, int64_t& gv, int64_t& hv) { cell_of(cells, ii, gv, hv); });
              icells[i] = 0;
            }
            __syncthreads();
          }
        }
      };
      if (c.q_in_row) rows_async(std::true_type{});
      else rows_async(std::false_type{});
    }
  }
  if (!direct) {
    // registers of the next tile: this thread's row of it
    uint32_t nrow = 0;
    int32_t nq = 0;
    float2 ngh = make_float2(0.f, 0.f);
    uint4 nb[2 * kNG];
    // row indices run one tile ahead of the gathers that use them
    auto load_idx = [&](int64_t pos) { return pos < r1 ? __ldcg(idx + pos) : 0u; };  // written by the partition
    uint32_t idx_ahead = 0;
    auto fetch = [&](int64_t pos, uint32_t row) {
      const bool live = pos < r1;
      nrow = row;
      if (kMode == 2) nq = live ? __ldg(s.packed + nrow) : 0;
      else ngh = live ? s.gh[nrow] : make_float2(0.f, 0.f);
      const uint4* src = reinterpret_cast<const uint4*>(c.bins + (size_t)nrow * stride + f0);
#pragma unroll
      for (int k = 0; k < 2 * kNG; ++k)
        nb[k] = (live && (k >> 1) < ngroups) ? __ldg(src + k) : make_uint4(0u, 0u, 0u, 0u);
    };
    {
      const uint32_t first = load_idx(r0 + threadIdx.x);
      idx_ahead = load_idx(r0 + kHistTileRows + threadIdx.x);
      fetch(r0 + threadIdx.x, first);
    }
    if (threadIdx.x < 32 * kNG) {
      s_vlen[threadIdx.x] = my_vlen;
      s_vstart[threadIdx.x] = my_vstart;
    }
    int32_t since_flush = 0;
    __syncthreads();
    for (int64_t t0 = r0; t0 < r1; t0 += kHistTileRows) {
      const int tile_rows = (int)min((int64_t)kHistTileRows, r1 - t0);
      // stage this tile (the previous tile's accumulation has finished); rows
      // past the range stage as zeros and add nothing
#pragma unroll
      for (int k = 0; k < 2 * kNG; ++k) sbins[threadIdx.x * 2 * kNG + k] = nb[k];
      if (kMode == 2) sq[threadIdx.x] = nq;
      else sgh[threadIdx.x] = ngh;
      __syncthreads();
      // the next tile's gathers run while this one is accumulated
      if (t0 + kHistTileRows < r1) {
        fetch(t0 + kHistTileRows + threadIdx.x, idx_ahead);
        idx_ahead = load_idx(t0 + 2 * kHistTileRows + threadIdx.x);
      }
      const int rw0 = warp * kRowsPerWarp;
      if (rw0 < tile_rows) {
        // this warp's 32 staged rows; lane l adds feature f0 + 32 g + l of
        // each row. The gradients of two or four rows arrive in one broadcast
        // load.
        const unsigned char* rowp = reinterpret_cast<const unsigned char*>(sbins) + rw0 * kRowBytes + lane;
        auto rows = [&](auto groups) {
          constexpr int kG = decltype(groups)::value;
          // rows per batch: every byte of a batch is loaded before its first
          // atomic (the compiler cannot move loads past shared atomics that may
          // alias them), so a batch waits for one shared-load latency
          constexpr int kB = kG == 1 ? 8 : 4;
#pragma unroll
          for (int jb = 0; jb < kRowsPerWarp / kB; ++jb) {
            int raw[kB][kG];
#pragma unroll
            for (int u = 0; u < kB; ++u)
#pragma unroll
              for (int g = 0; g < kG; ++g) raw[u][g] = (int)rowp[(kB * jb + u) * kRowBytes + 32 * g];
            if constexpr (kMode == 2) {
              int32_t qs[kB];
#pragma unroll
              for (int v = 0; v < kB / 4; ++v) {
                const int4 q4 = reinterpret_cast<const int4*>(sq + rw0 + kB * jb)[v];
                qs[4 * v] = q4.x;
                qs[4 * v + 1] = q4.y;
                qs[4 * v + 2] = q4.z;
                qs[4 * v + 3] = q4.w;
              }
#pragma unroll
              for (int u = 0; u < kB; ++u)
#pragma unroll
                for (int g = 0; g < kG; ++g)
                  atomicAdd(reinterpret_cast<int32_t*>(cells) + g * kGroupCells + raw[u][g] * 32 + lane, qs[u]);
            } else {
              float gs[kB], hs[kB];
#pragma unroll
              for (int v = 0; v < kB / 2; ++v) {
                const float4 t = reinterpret_cast<const float4*>(sgh + rw0 + kB * jb)[v];
                gs[2 * v] = t.x;
                hs[2 * v] = t.y;
                gs[2 * v + 1] = t.z;
                hs[2 * v + 1] = t.w;
              }
#pragma unroll
              for (int u = 0; u < kB; ++u)
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                  // float cells take a compare-and-swap loop per add: skip value 0
                  if (raw[u][g] == 0) continue;
                  const int k = raw[u][g] * 32 + lane;
                  const float gv = gs[u], hv = hs[u];
                  if constexpr (kMode == 0) {
                    double* d = reinterpret_cast<double*>(cells + (size_t)g * kGroupCells * 16);
                    atomicAdd(d + k, (double)gv);
                    atomicAdd(d + kGroupCells + k, (double)hv);
                  } else {
                    float* fl = reinterpret_cast<float*>(cells + (size_t)g * kGroupCells * 16);
                    float og = atomicAdd(fl + k, gv);
                    float sg = __fadd_rn(og, gv);
                    float bg = __fsub_rn(sg, og);
                    atomicAdd(fl + kGroupCells + k, __fadd_rn(__fsub_rn(og, __fsub_rn(sg, bg)), __fsub_rn(gv, bg)));
                    float oh = atomicAdd(fl + 2 * kGroupCells + k, hv);
                    float s2 = __fadd_rn(oh, hv);
                    float bh = __fsub_rn(s2, oh);
                    atomicAdd(fl + 3 * kGroupCells + k, __fadd_rn(__fsub_rn(oh, __fsub_rn(s2, bh)), __fsub_rn(hv, bh)));
                  }
                }
            }
          }
        };
        // the group count is a compile-time constant inside the row loop
        if (ngroups == kNG) {
          rows(std::integral_constant<int, kNG>{});
        } else {
          if constexpr (kNG > 1) {
            if (ngroups == 1) rows(std::integral_constant<int, 1>{});
            else if constexpr (kNG > 2) {
              if (ngroups == 2) rows(std::integral_constant<int, 2>{});
              else if constexpr (kNG > 3) {
                if (ngroups == 3) rows(std::integral_constant<int, 3>{});
              }
            }
          }
        }
      }
      since_flush += tile_rows;
      __syncthreads();
      // int32 cells hold at most sub_rows rows before their 16-bit halves could
      // wrap: this CTA adds its own cells to the histogram and clears them
      if constexpr (kMode == 2) {
        if (t0 + kHistTileRows < r1 && since_flush + kHistTileRows > sub_rows) {
          const int total = ngroups * kGroupCells;
          for (int i = threadIdx.x; i < total; i += kHistThreads) {
            emit(i, [&](int ii, int64_t& gv, int64_t& hv) { cell_of(cells, ii, gv, hv); });
            reinterpret_cast<int32_t*>(cells)[i] = 0;
          }
          since_flush = 0;
          __syncthreads();
        }
      }
    }
  }
  // cluster reduction: CTA rank r adds slice r of the cells, summed over the
  // cluster's CTAs in rank order (a cluster of one adds its own cells)
  if constexpr (kCl > 1) cg::this_cluster().sync();
  else __syncthreads();
  if constexpr (kCl > 1 && kMode == 2) {
    // the slice's sums are read from the cluster's shared memories first;
    // once they are in registers this CTA arrives at the final barrier (its
    // reads of the peers are complete: every value has been consumed), then
    // issues its global atomics while the peers arrive
    constexpr int kSlice = (kNG * kGroupCells + kCl - 1) / kCl;
    constexpr int kPerThread = (kSlice + kHistThreads - 1) / kHistThreads;
    const int total = ngroups * kGroupCells;
    const int per = (total + kCl - 1) / kCl;
    const int crank = (int)cg::this_cluster().block_rank();
    const int lo = crank * per, hi = min(total, lo + per);
    int64_t sg[kPerThread], sh[kPerThread];
#pragma unroll
    for (int j = 0; j < kPerThread; ++j) {
      const int i = lo + (int)threadIdx.x + j * kHistThreads;
      sg[j] = 0;
      sh[j] = 0;
      if (i < hi) {
#pragma unroll
        for (int r = 0; r < kCl; ++r) {
          int64_t a, b;
          cell_of(cg::this_cluster().map_shared_rank(cells, r), i, a, b);
          sg[j] += a;
          sh[j] += b;
        }
      }
    }
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < kPerThread; ++j) {
      const int i = lo + (int)threadIdx.x + j * kHistThreads;
      if (i < hi) emit(i, [&](int, int64_t& gv, int64_t& hv) {
          gv = sg[j];
          hv = sh[j];
        });
    }
    // no CTA leaves (or reuses its cells) while another may still read them
    asm volatile("barrier.cluster.wait.aligned;" ::: "memory");
    return;
  }
  {
    const int total = ngroups * kGroupCells;
    const int per = (total + kCl - 1) / kCl;
    int crank = 0;
    if constexpr (kCl > 1) crank = (int)cg::this_cluster().block_rank();
    const int lo = crank * per, hi = min(total, lo + per);
    for (int i = lo + (int)threadIdx.x; i < hi; i += kHistThreads) {
      if constexpr (kMode == 2) {
        emit(i, [&](int ii, int64_t& gv, int64_t& hv) {
          gv = 0;
          hv = 0;
#pragma unroll
          for (int r = 0; r < kCl; ++r) {
            int64_t a, b;
            if constexpr (kCl > 1) cell_of(cg::this_cluster().map_shared_rank(cells, r), ii, a, b);
            else cell_of(cells, ii, a, b);
            gv += a;
            hv += b;
          }
        });
      } else {
        emit(i, [&](int ii, double& gv, double& hv) {
          gv = 0.0;
          hv = 0.0;
#pragma unroll
          for (int r = 0; r < kCl; ++r) {
            double a, b;
            if constexpr (kCl > 1) cell_of(cg::this_cluster().map_shared_rank(cells, r), ii, a, b);
            else cell_of(cells, ii, a, b);
            gv += a;
            hv += b;
          }
        });
      }
    }
  }
  // no CTA leaves (or reuses its cells) while another may still read them:
  // the peers consumed what they read before arriving, so the arrive needs
  // no release ordering (this CTA's global atomics need not be waited for)
  if constexpr (kCl > 1) {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n\tbarrier.cluster.wait.aligned;" ::: "memory");
  } else {
    __syncthreads();
  }
}

__device__ void deferred_finish(const DCtx& c, const DSlot& s, void* dec_smem);

// Grid (lead + row CTAs, feature tiles, slots). With lead > 0 (one cluster)
// the first CTA of each slot runs the previous split step's end, which its
// partition posted, while the row CTAs build the histogram.
template <int kMode, int kNG>
__global__ void __cluster_dims__(hist_cluster(kMode), 1, 1) __launch_bounds__(kHistThreads, 2)
    k_hist(const __grid_constant__ DCtx c, DTileTable tt, int32_t sub_rows, int32_t lead) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_wait();
  pdl_trigger();
  const DSlot& s = c.slots[blockIdx.z];
  if ((int)blockIdx.x < lead) {
    if (blockIdx.x == 0 && blockIdx.y == 0) deferred_finish(c, s, smem_raw);
    return;
  }
  const int rank = (int)blockIdx.x - lead;
  LeafRows lr;
  int64_t r0, r1;
  if (!hist_setup<hist_cluster(kMode)>(c, s, rank, (int)gridDim.x - lead, lr, r0, r1)) return;
  if (rank == 0 && blockIdx.y == 0 && threadIdx.x == 0) s.st->hist_rows += lr.count;
  hist_body<kMode, kNG, hist_cluster(kMode)>(c, s, tt, blockIdx.y, lr, r0, r1, sub_rows, smem_raw);
}

#define LGBM_B200_HIST_INST(M, G) \
  template __global__ void k_hist<M, G>(const __grid_constant__ DCtx, DTileTable, int32_t, int32_t);
LGBM_B200_HIST_INST(0, 1)
LGBM_B200_HIST_INST(1, 1)
LGBM_B200_HIST_INST(2, 1)
LGBM_B200_HIST_INST(2, 2)
LGBM_B200_HIST_INST(2, 3)
LGBM_B200_HIST_INST(2, 4)
#undef LGBM_B200_HIST_INST

size_t hist_smem_bytes(int mode, int ng) {
  const size_t cell = mode == 2 ? 4 : 16;
  const size_t staged = (size_t)ng * kMaxBins * 32 * cell + (size_t)kHistTileRows * 32 * ng + (size_t)kHistTileRows * 8;
  if (mode == 2 && ng == 1) {  // or the cells and every warp's ring of asynchronous copies
    const size_t ring = (size_t)(kHistThreads / 32) * kHistAsyncStages * (16 * 32 + 16 * 4);
    return std::max(staged, (size_t)kMaxBins * 32 * 4 + ring);
  }
  return staged;
}

const void* hist_kernel(int mode, int ng) {
  if (mode == 0) return reinterpret_cast<const void*>(&k_hist<0, 1>);
  if (mode == 1) return reinterpret_cast<const void*>(&k_hist<1, 1>);
  switch (ng) {
    case 1: return reinterpret_cast<const void*>(&k_hist<2, 1>);
    case 2: return reinterpret_cast<const void*>(&k_hist<2, 2>);
    case 3: return reinterpret_cast<const void*>(&k_hist<2, 3>);
    default: return reinterpret_cast<const void*>(&k_hist<2, 4>);
  }
}

cudaError_t launch_hist(int mode, int ng, dim3 grid, size_t smem, cudaStream_t st, const DCtx& c, const DTileTable& tt,
                        int32_t sub_rows, bool pdl, bool finish) {
  // the step-end CTA leads as one whole cluster, so the row CTAs' clusters keep their alignment
  const int32_t lead = finish ? hist_cluster(mode) : 0;
  grid.x += (unsigned)lead;
  if (mode == 0) return launch_ex(k_hist<0, 1>, grid, dim3(kHistThreads), smem, st, pdl, c, tt, sub_rows, lead);
  if (mode == 1) return launch_ex(k_hist<1, 1>, grid, dim3(kHistThreads), smem, st, pdl, c, tt, sub_rows, lead);
  if (ng == 1) return launch_ex(k_hist<2, 1>, grid, dim3(kHistThreads), smem, st, pdl, c, tt, sub_rows, lead);
  if (ng == 2) return launch_ex(k_hist<2, 2>, grid, dim3(kHistThreads), smem, st, pdl, c, tt, sub_rows, lead);
  if (ng == 3) return launch_ex(k_hist<2, 3>, grid, dim3(kHistThreads), smem, st, pdl, c, tt, sub_rows, lead);
  return launch_ex(k_hist<2, 4>, grid, dim3(kHistThreads), smem, st, pdl, c, tt, sub_rows, lead);
}

// =====================================================================================
// split scan (split.rs:246-891 and :930-1400) — one CTA of two warps per
// (feature, slot): warp 0 the smaller leaf, warp 1 the larger leaf.
// =====================================================================================


struct LeafCtx {
  double sum_g, sum_h;  // sum_h includes 2*kEpsilon (FP forms)
  int64_t int_sum;
  double gs, hs;
  int32_t num_data;
  double parent_output;
  bool mc;
  double cmin, cmax;
};

// Warp-wide argmax with the scan's tie rule: larger gain, then smaller position.
__device__ __forceinline__ void warp_best(double& gain, int32_t& pos) {
  for (int o = 16; o > 0; o >>= 1) {
    double og = __shfl_xor_sync(0xffffffffu, gain, o);
    int32_t op = __shfl_xor_sync(0xffffffffu, pos, o);
    if (og > gain || (og == gain && op < pos)) {
      gain = og;
      pos = op;
    }
  }
}
__device__ __forceinline__ int32_t warp_min_i(int32_t v) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// split.rs:448-670 / :1194-1400 categorical threshold search, in lane 0
// (the candidate lists are at most a few dozen bins; the stable sort is a
// rank sort done by the whole warp).
template <bool kInt>
__device__ __noinline__ bool scan_categorical(ScanSmem& sm, const DFeature& m, const DParams& p, const LeafCtx& lc, DSplit& out) {
  const int lane = threadIdx.x & 31;
  const int offset = m.offset;
  const int bin_start = 1 - offset, bin_end = m.num_bin - offset;
  const bool use_onehot = m.num_bin <= p.max_cat_to_onehot;
  const double gs = lc.gs, hs = lc.hs;
  double sum_gradient = kInt ? (double)int_grad(lc.int_sum) * gs : lc.sum_g;
  double sum_hessian = kInt ? (double)int_hess(lc.int_sum) * hs : lc.sum_h;
  const double cnt_factor = kInt ? (double)lc.num_data / (double)int_hess(lc.int_sum) : (double)lc.num_data / lc.sum_h;
  auto G = [&](int t) { return kInt ? (double)int_grad(sm.ig[t]) * gs : sm.g[t]; };
  auto H = [&](int t) { return kInt ? (double)int_hess(sm.ig[t]) * hs : sm.h[t]; };
  auto CNT = [&](int t) {
    return kInt ? round_int((double)int_hess(sm.ig[t]) * cnt_factor) : round_int(sm.h[t] * cnt_factor);
  };
  int32_t used_bin = 0;
  if (!use_onehot) {
    // bins with enough data, then a stable sort by sum_grad / (sum_hess + cat_smooth)
    if (lane == 0) {
      for (int i = bin_start; i < bin_end; ++i)
        if ((double)CNT(i) >= p.cat_smooth) sm.tpos[used_bin++] = i;
    }
    used_bin = __shfl_sync(0xffffffffu, used_bin, 0);
    __syncwarp();
    for (int k = lane; k < used_bin; k += 32) {
      int i = sm.tpos[k];
      sm.key[k] = G(i) / (H(i) + p.cat_smooth);
    }
    __syncwarp();
    for (int k = lane; k < used_bin; k += 32) {
      double kk = sm.key[k];
      int rank = 0;
      for (int j = 0; j < used_bin; ++j) {
        double kj = sm.key[j];
        if (kj < kk || (j < k && !(kk < kj) && !(kj < kk))) ++rank;
      }
      sm.sorted[rank] = sm.tpos[k];
    }
    __syncwarp();
  }
  bool is_splittable = false;
  if (lane == 0) {
    out.default_left = 0;
    double gain_shift = use_smoothing(p) ? leaf_gain_given_output(sum_gradient, sum_hessian, p, lc.parent_output)
                                         : leaf_gain(sum_gradient, sum_hessian, p, lc.num_data, 0.0);
    double min_gain_shift = gain_shift + p.min_gain_to_split;
    DParams pc = p;
    double best_gain = -INFINITY;
    int32_t best_left_count = 0, best_threshold = -1, best_dir = 1;
    double best_slg = 0.0, best_slh = 0.0;
    int64_t best_left_int = 0;
    if (use_onehot) {
      for (int t = bin_start; t < bin_end; ++t) {
        int32_t cnt = CNT(t);
        double grad = G(t), hess = H(t);
        if (cnt < p.min_data_in_leaf || hess < p.min_sum_hessian_in_leaf) continue;
        int32_t other_count = lc.num_data - cnt;
        if (other_count < p.min_data_in_leaf) continue;
        double soh, sog;
        if (kInt) {
          int64_t other = (int64_t)((uint64_t)lc.int_sum - (uint64_t)sm.ig[t]);
          soh = (double)int_hess(other) * hs;
          if (soh < p.min_sum_hessian_in_leaf) continue;
          sog = (double)int_grad(other) * gs;
        } else {
          soh = sum_hessian - hess - kEpsilon;
          if (soh < p.min_sum_hessian_in_leaf) continue;
          sog = sum_gradient - grad;
        }
        double gain = split_gain(sog, soh, grad, kInt ? hess : hess + kEpsilon, pc, other_count, cnt, lc.parent_output,
                                 lc.mc, lc.cmin, lc.cmax, 0);
        if (gain <= min_gain_shift) continue;
        is_splittable = true;
        if (gain > best_gain) {
          best_threshold = t;
          best_slg = grad;
          best_slh = kInt ? hess : hess + kEpsilon;
          best_left_count = cnt;
          best_left_int = kInt ? sm.ig[t] : 0;
          best_gain = gain;
        }
      }
    } else {
      pc.lambda_l2 += p.cat_l2;
      int32_t max_num_cat = min(p.max_cat_threshold, (used_bin + 1) / 2);
      for (int d = 0; d < 2; ++d) {
        int32_t dir = d == 0 ? 1 : -1;
        int32_t start_pos = d == 0 ? 0 : used_bin - 1;
        int32_t cnt_cur_group = 0, left_count = 0;
        double slg = 0.0, slh = kEpsilon;
        int64_t sl_int = 0;
        for (int32_t i = 0; i < used_bin && i < max_num_cat; ++i) {
          int t = sm.sorted[start_pos];
          start_pos += dir;
          int32_t cnt = CNT(t);
          double srh, srg, slh_eff;
          if (kInt) {
            sl_int = (int64_t)((uint64_t)sl_int + (uint64_t)sm.ig[t]);
            left_count += cnt;
            cnt_cur_group += cnt;
            slh_eff = (double)int_hess(sl_int) * hs;
            if (left_count < p.min_data_in_leaf || slh_eff < p.min_sum_hessian_in_leaf) continue;
            int32_t right_count = lc.num_data - left_count;
            if (right_count < p.min_data_in_leaf || right_count < p.min_data_per_group) break;
            int64_t sr_int = (int64_t)((uint64_t)lc.int_sum - (uint64_t)sl_int);
            srh = (double)int_hess(sr_int) * hs;
            if (srh < p.min_sum_hessian_in_leaf) break;
            if (cnt_cur_group < p.min_data_per_group) continue;
            cnt_cur_group = 0;
            double slg_i = (double)int_grad(sl_int) * gs;
            srg = (double)int_grad(sr_int) * gs;
            double gain = split_gain(slg_i, slh_eff, srg, srh, pc, left_count, right_count, lc.parent_output, lc.mc,
                                     lc.cmin, lc.cmax, 0);
            if (gain <= min_gain_shift) continue;
            is_splittable = true;
            if (gain > best_gain) {
              best_left_int = sl_int;
              best_threshold = i;
              best_gain = gain;
              best_dir = dir;
            }
          } else {
            slg += G(t);
            slh += H(t);
            left_count += cnt;
            cnt_cur_group += cnt;
            if (left_count < p.min_data_in_leaf || slh < p.min_sum_hessian_in_leaf) continue;
            int32_t right_count = lc.num_data - left_count;
            if (right_count < p.min_data_in_leaf || right_count < p.min_data_per_group) break;
            srh = sum_hessian - slh;
            if (srh < p.min_sum_hessian_in_leaf) break;
            if (cnt_cur_group < p.min_data_per_group) continue;
            cnt_cur_group = 0;
            srg = sum_gradient - slg;
            double gain = split_gain(slg, slh, srg, srh, pc, left_count, right_count, lc.parent_output, lc.mc, lc.cmin,
                                     lc.cmax, 0);
            if (gain <= min_gain_shift) continue;
            is_splittable = true;
            if (gain > best_gain) {
              best_left_count = left_count;
              best_slg = slg;
              best_slh = slh;
              best_threshold = i;
              best_gain = gain;
              best_dir = dir;
            }
          }
        }
      }
    }
    if (is_splittable) {
      if (kInt) {
        int64_t left = best_left_int;
        int64_t right = (int64_t)((uint64_t)lc.int_sum - (uint64_t)left);
        double lg = (double)int_grad(left) * gs, lh = (double)int_hess(left) * hs;
        double rg = (double)int_grad(right) * gs, rh = (double)int_hess(right) * hs;
        int32_t lcnt = round_int((double)int_hess(left) * cnt_factor);
        int32_t rcnt = round_int((double)int_hess(right) * cnt_factor);
        double lo = leaf_output(lg, lh, pc, lcnt, lc.parent_output);
        double ro = leaf_output(rg, rh, pc, rcnt, lc.parent_output);
        out.left_output = lc.mc ? clampc(lo, lc.cmin, lc.cmax) : lo;
        out.right_output = lc.mc ? clampc(ro, lc.cmin, lc.cmax) : ro;
        out.left_count = lcnt;
        out.right_count = rcnt;
        out.left_sum_gradient = lg;
        out.left_sum_hessian = lh;
        out.right_sum_gradient = rg;
        out.right_sum_hessian = rh;
        out.left_sum_gh = left;
        out.right_sum_gh = right;
      } else {
        double lo = leaf_output(best_slg, best_slh, pc, best_left_count, lc.parent_output);
        double ro = leaf_output(sum_gradient - best_slg, sum_hessian - best_slh, pc, lc.num_data - best_left_count,
                                lc.parent_output);
        out.left_output = lc.mc ? clampc(lo, lc.cmin, lc.cmax) : lo;
        out.right_output = lc.mc ? clampc(ro, lc.cmin, lc.cmax) : ro;
        out.left_count = best_left_count;
        out.left_sum_gradient = best_slg;
        out.left_sum_hessian = best_slh - kEpsilon;
        out.right_count = lc.num_data - best_left_count;
        out.right_sum_gradient = sum_gradient - best_slg;
        out.right_sum_hessian = sum_hessian - best_slh - kEpsilon;
      }
      out.monotone_type = 0;
      out.gain = best_gain - min_gain_shift;
      for (int w = 0; w < kCatWords; ++w) out.cat_bits[w] = 0;
      int32_t ncat = 0;
      if (use_onehot) {
        uint32_t b = (uint32_t)(best_threshold + offset);
        out.cat_bits[b >> 5] |= 1u << (b & 31);
        ncat = 1;
      } else {
        for (int32_t i = 0; i <= best_threshold; ++i) {
          uint32_t b = (uint32_t)((best_dir == 1 ? sm.sorted[i] : sm.sorted[used_bin - 1 - i]) + offset);
          out.cat_bits[b >> 5] |= 1u << (b & 31);
          ++ncat;
        }
      }
      out.num_cat = ncat;
    }
  }
  is_splittable = __shfl_sync(0xffffffffu, (int)is_splittable, 0) != 0;
  __syncwarp();
  return is_splittable;
}

// The FP64 cumulative sums of one scan direction in the reference's order
// (split.rs:676-891): a lane carry chain by one warp, one add per visited
// bin in scan order, into chain set `set` of `sm` (0: cg/ch/cc, 1:
// cg2/ch2/cc2); the forward direction's extra candidate (NaN missing, no
// stored bin 0) into eg/eh/ec.
__device__ void fp64_direction_chain(ScanSmem& sm, const DFeature& m, const LeafCtx& lc, bool reverse,
                                     bool skip_default, bool na_as_missing, int set) {
  const int lane = threadIdx.x & 31;
  const int offset = m.offset;
  const int len = m.view_len;
  int32_t t_lo, t_hi;
  if (reverse) {
    t_hi = m.num_bin - 1 - offset - (int32_t)na_as_missing;
    t_lo = 1 - offset;
  } else {
    t_lo = 0;
    t_hi = m.num_bin - 2 - offset;
  }
  const int32_t skip_t = skip_default ? m.default_bin - offset : INT32_MIN;
  auto visited = [&](int t) { return t >= t_lo && t <= t_hi && t != skip_t && t < len; };
  const bool first_extra = !reverse && na_as_missing && offset == 1;
  const int32_t nstored = m.num_bin - offset;
  const int khi = len > 0 ? (len - 1) / kPer : -1;
  double* cg = set ? sm.cg2 : sm.cg;
  double* ch = set ? sm.ch2 : sm.ch;
  int32_t* cc = set ? sm.cc2 : sm.cc;
  // this lane's bins in registers first, so that no shared load sits on the
  // chain's critical path
  double gv[kPer], hv[kPer];
  int32_t cv[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int t = lane * kPer + j;
    gv[j] = t < len ? sm.g[t] : 0.0;
    hv[j] = t < len ? sm.h[t] : 0.0;
    cv[j] = t < len ? sm.ce[t] : 0;
  }
  double a = 0.0, b = kEpsilon;
  int32_t c = 0;
  if (first_extra) {  // split.rs:787-800: the leaf sums minus every stored bin, ascending
    a = lc.sum_g;
    b = lc.sum_h - kEpsilon;
    c = lc.num_data;
    carry_chain(false, 0, khi, a, b, c, [&](int j, double& x, double& y, int32_t& z) {
      int t = lane * kPer + j;
      if (t < nstored && t < len) {
        x -= gv[j];
        y -= hv[j];
        z -= cv[j];
      }
    });
    if (lane == 0) {
      sm.eg = a;
      sm.eh = b;
      sm.ec = c;
    }
  }
  carry_chain(reverse, 0, khi, a, b, c, [&](int j, double& x, double& y, int32_t& z) {
    int t = lane * kPer + j;
    if (visited(t)) {
      x += gv[j];
      y += hv[j];
      z += cv[j];
      cg[t] = x;
      ch[t] = y;
      cc[t] = z;
    }
  });
}

// One direction of FindBestThresholdSequentially (split.rs:676-891 and
// :995-1190) over the view in `sm`, by the whole CTA. Warp 0 forms the
// cumulative sums in the reference's order (FP64: a lane carry chain, one
// add per visited bin in scan order; packed integers: any order is exact);
// then thread t evaluates candidate t and the CTA reduces the first break
// and the best gain with the sequential loop's rules. Thread 0 applies the
// winner to `out`. Returns whether any candidate was splittable.
template <bool kInt>
__device__ bool scan_direction_block(ScanSmem& sm, const DFeature& m, const DParams& p, const LeafCtx& lc,
                                     double min_gain_shift, double cnt_factor, bool reverse, bool skip_default,
                                     bool na_as_missing, DSplit& out, int chain = -1) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int offset = m.offset;
  const int len = m.view_len;
  int32_t t_lo, t_hi;
  if (reverse) {
    t_hi = m.num_bin - 1 - offset - (int32_t)na_as_missing;
    t_lo = 1 - offset;
  } else {
    t_lo = 0;
    t_hi = m.num_bin - 2 - offset;
  }
  const int32_t skip_t = skip_default ? m.default_bin - offset : INT32_MIN;
  auto visited = [&](int t) { return t >= t_lo && t <= t_hi && t != skip_t && t < len; };
  // extra candidate t = -1 (forward with NaN missing and no stored bin 0)
  const bool first_extra = !reverse && na_as_missing && offset == 1;
  const int32_t nstored = m.num_bin - offset;
  if (!kInt) {
    const bool own = chain < 0;  // form the chain here (warp 0), or use the one formed before
    if (own && warp == 0) fp64_direction_chain(sm, m, lc, reverse, skip_default, na_as_missing, 0);
    if (tid == 0) sm.brk = reverse ? INT32_MIN : INT32_MAX;
  } else {
    // exact packed sums (any order): thread u holds scan position u, a block
    // scan over the threads in scan order gives every cumulative sum
    const int t = reverse ? len - 1 - tid : tid;
    const bool vis = tid < len && visited(t);
    const uint64_t v = vis ? (uint64_t)sm.ig[t] : 0ull;
    const uint64_t a = (first_extra && tid < len && t < nstored) ? (uint64_t)sm.ig[t] : 0ull;  // every stored bin
    uint64_t incl = v, asum = a;
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t other = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += other;
      asum += __shfl_xor_sync(0xffffffffu, asum, o);
    }
    if (lane == 31) sm.wq[warp] = (int64_t)incl;
    if (lane == 0) sm.wa[warp] = (int64_t)asum;
    if (tid == 0) sm.brk = reverse ? INT32_MIN : INT32_MAX;
    __syncthreads();
    uint64_t pre = 0, all = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      if (w < warp) pre += (uint64_t)sm.wq[w];
      all += (uint64_t)sm.wa[w];
    }
    const uint64_t base = first_extra ? (uint64_t)lc.int_sum - all : 0ull;
    if (first_extra && tid == 0) {  // split.rs:1097-1103: the leaf sum minus every stored bin
      sm.eq = (int64_t)base;
      sm.ec = round_int((double)int_hess((int64_t)base) * cnt_factor);
    }
    if (vis) {
      const int64_t cq = (int64_t)(base + pre + incl);
      sm.cq[t] = cq;
      sm.cc[t] = round_int((double)int_hess(cq) * cnt_factor);
    }
  }
  __syncthreads();
  const int32_t min_data = p.min_data_in_leaf;
  const double min_hess = p.min_sum_hessian_in_leaf;
  const bool plain = plain_split(p, lc.mc);
  // accumulated side's values of candidate t (t = -1: the extra candidate)
  auto acc = [&](int t, double& ag, double& ah, int32_t& ac, int64_t& aq) {
    if (t < 0) {
      ag = sm.eg;
      ah = sm.eh;
      ac = sm.ec;
      aq = sm.eq;
    } else {
      ag = kInt ? 0.0 : (chain == 1 ? sm.cg2[t] : sm.cg[t]);
      ah = kInt ? 0.0 : (chain == 1 ? sm.ch2[t] : sm.ch[t]);
      ac = (!kInt && chain == 1) ? sm.cc2[t] : sm.cc[t];
      aq = kInt ? sm.cq[t] : 0;
    }
  };
  auto sides = [&](double ah, int64_t aq, double& ha, double& hr) {
    if (kInt) {
      ha = (double)int_hess(aq) * lc.hs;
      hr = (double)int_hess((int64_t)((uint64_t)lc.int_sum - (uint64_t)aq)) * lc.hs;
    } else {
      ha = ah;
      hr = lc.sum_h - ah;
    }
  };
  // thread 0 also owns the extra candidate
  const int ncand = (tid == 0 && first_extra) ? 2 : 1;
  // pass 1: the first break in scan order
  {
    int32_t brk = reverse ? INT32_MIN : INT32_MAX;
#pragma unroll 1
    for (int k = 0; k < ncand; ++k) {
      const int t = k == 0 ? tid : -1;
      if (t >= 0 && !visited(t)) continue;
      double ag, ah, ha, hr;
      int32_t ac;
      int64_t aq;
      acc(t, ag, ah, ac, aq);
      sides(ah, aq, ha, hr);
      bool skip1 = ac < min_data || ha < min_hess;
      if (!skip1 && (lc.num_data - ac < min_data || hr < min_hess)) brk = reverse ? max(brk, t) : min(brk, t);
    }
    for (int o = 16; o > 0; o >>= 1) {
      int32_t ob = __shfl_xor_sync(0xffffffffu, brk, o);
      brk = reverse ? max(brk, ob) : min(brk, ob);
    }
    if (lane == 0 && brk != (reverse ? INT32_MIN : INT32_MAX)) {
      if (reverse) atomicMax(&sm.brk, brk);
      else atomicMin(&sm.brk, brk);
    }
  }
  __syncthreads();
  const int32_t brk = sm.brk;
  // pass 2: gains of the candidates before the break
  double best_gain = -INFINITY;
  int32_t best_t = INT32_MIN;
  bool splittable = false;
#pragma unroll 1
  for (int k = 0; k < ncand; ++k) {
    const int t = k == 0 ? tid : -1;
    if (t >= 0 && !visited(t)) continue;
    if (t >= 0 ? (reverse ? t <= brk : t >= brk) : !(brk > -1)) continue;
    double ag, ah, ha, hr;
    int32_t ac;
    int64_t aq;
    acc(t, ag, ah, ac, aq);
    sides(ah, aq, ha, hr);
    if (ac < min_data || ha < min_hess) continue;
    double ga, gr;
    if (kInt) {
      int64_t rest = (int64_t)((uint64_t)lc.int_sum - (uint64_t)aq);
      ga = (double)int_grad(aq) * lc.gs;
      gr = (double)int_grad(rest) * lc.gs;
      ha += kEpsilon;
      hr += kEpsilon;
    } else {
      ga = ag;
      gr = lc.sum_g - ag;
    }
    int32_t rc = lc.num_data - ac;
    // the left child is the rest when scanning in reverse
    const double g1 = reverse ? gr : ga, h1 = reverse ? hr : ha, g2 = reverse ? ga : gr, h2 = reverse ? ha : hr;
    const int32_t c1 = reverse ? rc : ac, c2 = reverse ? ac : rc;
    double gain = split_gain_hot(plain, g1, h1, g2, h2, p, c1, c2, lc.parent_output, lc.mc, lc.cmin, lc.cmax,
                                 m.monotone_type);
    if (gain <= min_gain_shift) continue;
    splittable = true;
    if (gain > best_gain || (gain == best_gain && best_t != INT32_MIN && (reverse ? t > best_t : t < best_t))) {
      best_gain = gain;
      best_t = t;
    }
  }
  warp_pick(reverse, best_gain, best_t);
  if (lane == 0) {
    sm.wgain[warp] = best_gain;
    sm.wt[warp] = best_t;
  }
  const bool any = __syncthreads_or(splittable) != 0;
  if (warp == 0) {
    // the warps' winners reduced with the same rule (candidates are distinct t)
    double bg = -INFINITY;
    int32_t bt = INT32_MIN;
    if (lane < (int)(blockDim.x >> 5)) {
      bg = sm.wgain[lane];
      bt = sm.wt[lane];
    }
    warp_pick(reverse, bg, bt);
    ScanBest r;
    r.splittable = any;
    r.gain = bg;
    r.t = bt;
    r.acc_g = r.acc_h = 0.0;
    r.acc_c = 0;
    r.acc_q = 0;
    if (bt != INT32_MIN) {
      double ag, ah;
      int32_t ac;
      int64_t aq;
      acc(bt, ag, ah, ac, aq);
      r.acc_g = ag;
      r.acc_h = ah;
      r.acc_c = ac;
      r.acc_q = aq;
    }
    apply_direction<kInt>(r, m, p, lc.sum_g, lc.sum_h, lc.int_sum, lc.gs, lc.hs, lc.num_data, lc.parent_output,
                          lc.mc, lc.cmin, lc.cmax, min_gain_shift, cnt_factor, reverse, out);
  }
  __syncthreads();
  return any;
}

// find_best_threshold (split.rs:246-271, :930-950) for one leaf and feature,
// by the whole CTA; the view is in `sm` (g/h, or ig for the quantized form).
template <bool kInt>
__device__ bool find_best_threshold_block(ScanSmem& sm, const DFeature& m, const DParams& p, LeafCtx lc, DSplit& out) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    out.default_left = 1;
    out.gain = -INFINITY;
    out.num_cat = 0;
    out.monotone_type = 0;
  }
  if (!kInt) lc.sum_h = lc.sum_h + 2.0 * kEpsilon;
  bool ok;
  if (m.bin_type == 1) {
    __syncthreads();
    if (tid < 32) {
      bool r = scan_categorical<kInt>(sm, m, p, lc, out);
      if (tid == 0) sm.ok = r ? 1 : 0;
    }
    __syncthreads();
    ok = sm.ok != 0;
  } else {
    if (tid == 0) out.monotone_type = m.monotone_type;
    double sg = kInt ? (double)int_grad(lc.int_sum) * lc.gs : lc.sum_g;
    double sh = kInt ? (double)int_hess(lc.int_sum) * lc.hs : lc.sum_h;
    double min_gain_shift = leaf_gain_hot(plain_split(p, lc.mc), sg, sh, p, lc.num_data, lc.parent_output) +
                            p.min_gain_to_split;
    double cnt_factor =
        kInt ? (double)lc.num_data / (double)int_hess(lc.int_sum) : (double)lc.num_data / lc.sum_h;
    if (!kInt && tid < m.view_len) sm.ce[tid] = round_int(sm.h[tid] * cnt_factor);
    __syncthreads();
    // split.rs:426-439: the directions scanned and their missing-value rules
    const bool two = m.num_bin > 2 && m.missing_type != 0;
    const bool skip_default = two && m.missing_type == 1;
    const bool na_missing = two && m.missing_type == 2;
    ok = false;
    if (!kInt && two) {
      // both directions' chains at once (warp 0 reverse, warp 1 forward): they
      // read the same view and write separate sums; each direction's scan
      // then reads its own (the barrier at its start orders them)
      const int warp = tid >> 5;
      if (warp < 2) fp64_direction_chain(sm, m, lc, warp == 0, skip_default, na_missing, warp);
      ok |= scan_direction_block<kInt>(sm, m, p, lc, min_gain_shift, cnt_factor, true, skip_default, na_missing, out,
                                        0);
      ok |= scan_direction_block<kInt>(sm, m, p, lc, min_gain_shift, cnt_factor, false, skip_default, na_missing, out,
                                        1);
    } else {
#pragma unroll 1
      for (int d = 0; d < (two ? 2 : 1); ++d)
        ok |= scan_direction_block<kInt>(sm, m, p, lc, min_gain_shift, cnt_factor, d == 0, skip_default, na_missing,
                                          out);
    }
    if (!two && tid == 0 && m.missing_type == 2) out.default_left = 0;
  }
  if (tid == 0) out.gain *= m.penalty;
  __syncthreads();
  return ok;
}

__device__ double monotone_split_gain_penalty(int32_t depth, double penalization) {  // constraints.rs:852-861
  double d = (double)depth;
  if (penalization >= d + 1.0) return kEpsilon;
  if (penalization <= 1.0) return 1.0 - penalization / pow(2.0, d) + kEpsilon;
  return 1.0 - pow(2.0, penalization - 1.0 - d) + kEpsilon;
}

__device__ __forceinline__ bool split_better(const DSplit& a, const DSplit& b) {
  return better_than(a.gain, a.feature, b.gain, b.feature);
}

// Partition LUT over stored group values (learner/mod.rs:1313-1329): one
// goes-left flag per value a row of the split feature can hold; thread t
// of the CTA writes value t.
__device__ void build_partition_lut(const DFeature& m, const DSplit& info, uint8_t* lut, int32_t first,
                                    int32_t step) {
  const bool numerical = m.bin_type == 0;
  const bool default_left = numerical ? info.default_left != 0 : false;
  const int32_t ntb = m.view_len + 1;
  for (int32_t raw = first; raw < kMaxBins; raw += step) {
    uint8_t left = 0;
    if (raw < ntb) {
      uint32_t b = decode_bin((uint32_t)raw, m);
      if (numerical) {
        bool miss = (m.missing_type == 1 && b == (uint32_t)m.default_bin) ||
                    (m.missing_type == 2 && b == (uint32_t)(m.num_bin - 1));
        left = miss ? (uint8_t)default_left : (uint8_t)(b <= info.threshold);
      } else {
        auto bit = [&](uint32_t v) { return (info.cat_bits[v >> 5] >> (v & 31)) & 1u; };
        if (b == (uint32_t)m.most_freq_bin) left = (uint8_t)(m.most_freq_bin > 0 && bit(b));
        else left = (uint8_t)bit(b);
      }
    }
    lut[raw] = left;
  }
}

// What apply_split reads (loaded early, so that the loads overlap other work).
struct ApplyIn {
  DSplit info;
  DFeature m;
  int32_t parent, parent_left, depth, num_cat;
  double old_value, cmin0, cmax0;
};

__device__ __forceinline__ ApplyIn apply_load(const DCtx& c, const DSlot& s, const DSplit& src, int32_t bl) {
  ApplyIn a;
  a.info = src;
  a.parent = s.tree.leaf_parent[bl];
  a.old_value = s.tree.leaf_value[bl];
  a.depth = s.tree.leaf_depth[bl] + 1;
  a.num_cat = s.st->num_cat;
  a.cmin0 = c.p.use_monotone ? s.cmin[bl] : 0.0;
  a.cmax0 = c.p.use_monotone ? s.cmax[bl] : 0.0;
  a.m = c.feats[a.info.inner];
  a.parent_left = a.parent >= 0 ? s.tree.left_child[a.parent] : 0;
  return a;
}

// The selected split applied to the tree (tree.rs:240-297); one thread.
__device__ void apply_split(const DCtx& c, const DSlot& s, int32_t bl, int32_t R, const ApplyIn& a) {
  DSlotState* st = s.st;
  const DParams& p = c.p;
  const DTree& t = s.tree;
  const DSplit& info = a.info;
  const DFeature& m = a.m;
  const int32_t parent = a.parent, parent_left = a.parent_left, d = a.depth, num_cat = a.num_cat;
  const double old_value = a.old_value, cmin0 = a.cmin0, cmax0 = a.cmax0;
  const int32_t node = R - 1;
  const bool numerical = m.bin_type == 0;
  if (parent >= 0) {
    if (parent_left == ~bl) t.left_child[parent] = node;
    else t.right_child[parent] = node;
  }
  t.split_feature_inner[node] = info.inner;
  t.split_feature[node] = info.feature;
  t.split_gain[node] = (float)(info.gain + p.min_gain_to_split);
  t.node_gain[node] = info.gain;
  t.left_child[node] = ~bl;
  t.right_child[node] = ~R;
  t.leaf_parent[bl] = node;
  t.leaf_parent[R] = node;
  t.internal_weight[node] = info.left_sum_hessian + info.right_sum_hessian;
  t.internal_value[node] = old_value;
  t.leaf_value[bl] = isnan(info.left_output) ? 0.0 : info.left_output;
  t.leaf_weight[bl] = info.left_sum_hessian;
  t.leaf_value[R] = isnan(info.right_output) ? 0.0 : info.right_output;
  t.leaf_weight[R] = info.right_sum_hessian;
  t.leaf_depth[bl] = d;
  t.leaf_depth[R] = d;
  int8_t dt = 0;
  const bool default_left = numerical ? info.default_left != 0 : false;
  if (default_left) dt |= 2;
  dt = (int8_t)((dt & 3) | (m.missing_type << 2));
  if (!numerical) dt |= 1;
  t.decision_type[node] = dt;
  t.threshold_in_bin[node] = numerical ? info.threshold : (uint32_t)num_cat;
  for (int w = 0; w < kCatWords; ++w) t.cat_bits[node * kCatWords + w] = numerical ? 0u : info.cat_bits[w];
  if (!numerical) st->num_cat = num_cat + 1;
  // basic monotone constraints (constraints.rs:467-480)
  if (p.use_monotone) {
    double lmin = cmin0, lmax = cmax0, rmin = cmin0, rmax = cmax0;
    if (numerical) {
      double mid = (info.left_output + info.right_output) / 2.0;
      if (info.monotone_type < 0) {
        lmin = mid < lmin ? lmin : mid;
        rmax = rmax < mid ? rmax : mid;
      } else if (info.monotone_type > 0) {
        lmax = lmax < mid ? lmax : mid;
        rmin = mid < rmin ? rmin : mid;
      }
    }
    s.cmin[bl] = lmin;
    s.cmax[bl] = lmax;
    s.cmin[R] = rmin;
    s.cmax[R] = rmax;
  }
  st->num_leaves_cur = R + 1;
}

// Threshold scan of feature f for one leaf side (0: smaller, 1: larger) of
// slot s, by the whole CTA (at least kScanThreads threads): the leaf's view
// is fixed (histogram.rs:42-56), the larger leaf's is formed as parent -
// smaller (histogram.rs:59-63) and stored, and the best threshold is written
// to feat_res / feat_ok.
template <bool kInt>
__device__ void scan_item(const DCtx& c, const DSlot& s, int f, int side, ScanSmem& sm) {
  DSlotState* st = s.st;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const DFeature m = c.feats[f];
  const DParams& p = c.p;
  const int32_t nf = c.num_features;
  // The loads run in two waves so that their latencies overlap: the slot
  // state, then everything that depends on it (the feature's flags, both
  // histogram views, the leaf's output bounds).
  const int32_t larger_leaf = st->larger.leaf, L = st->left_leaf, s_buf = st->s_buf, l_buf = st->l_buf;
  const bool need = st->need_find != 0 && st->done == 0;
  const int32_t nl_cur = st->num_leaves_cur;
  const DLeafSplits sl = st->smaller;
  const DLeafSplits ls = side == 0 ? sl : st->larger;
  const double gsc = st->grad_scale, hsc = st->hess_scale;
  const bool have_larger = larger_leaf >= 0;
  // the buffers and the leaf are valid whenever this side has a leaf to search
  const bool live = need && (side == 0 || have_larger);
  const int len = m.view_len;
  const size_t sbase = (size_t)s_buf * c.total_bins + m.view_start;
  const size_t lbase = (size_t)l_buf * c.total_bins + m.view_start;
  const bool in_view = live && tid < len;
  const bool sub = side == 1 && in_view;
  // histogram cells are written by other CTAs' atomics: loaded through L2
  int64_t sq = 0, pq = 0;
  double sgv = 0.0, shv = 0.0, pgv = 0.0, phv = 0.0;
  if (kInt) {
    const long long* hs = reinterpret_cast<const long long*>(s.hist);
    if (in_view) sq = (int64_t)__ldcg(hs + sbase + tid);
    if (sub) pq = (int64_t)__ldcg(hs + lbase + tid);
  } else {
    const double* hs = reinterpret_cast<const double*>(s.hist);
    if (in_view) {
      sgv = __ldcg(hs + 2 * (sbase + tid));
      shv = __ldcg(hs + 2 * (sbase + tid) + 1);
    }
    if (sub) {
      pgv = __ldcg(hs + 2 * (lbase + tid));
      phv = __ldcg(hs + 2 * (lbase + tid) + 1);
    }
  }
  const uint8_t in_tree = s.bytree[f];
  const uint8_t split_ok = have_larger ? s.splittable[L * nf + f] : (uint8_t)1;
  const double cmin = live ? s.cmin[ls.leaf] : 0.0, cmax = live ? s.cmax[ls.leaf] : 0.0;
  if (!(live && in_tree && split_ok)) return;
  {
    // the smaller leaf's view with its most frequent bin fixed (histogram.rs:42-56)
    if (kInt) {
      if (in_view) sm.ig[tid] = sq;
    } else {
      if (in_view) {
        sm.g[tid] = sgv;
        sm.h[tid] = shv;
      }
    }
    __syncthreads();
    if (m.most_freq_bin > 0 && warp == 0) {
      if (kInt) {  // exact: any summation order
        int64_t part = 0;
        for (int i = lane; i < m.num_bin; i += 32)
          if (i != m.most_freq_bin) part = (int64_t)((uint64_t)part + (uint64_t)sm.ig[i]);
        for (int o = 16; o > 0; o >>= 1)
          part = (int64_t)((uint64_t)part + (uint64_t)__shfl_xor_sync(0xffffffffu, part, o));
        int64_t fixed = (int64_t)((uint64_t)sl.int_sum - (uint64_t)part);
        __syncwarp();
        if (lane == 0) {
          sm.ig[m.most_freq_bin] = fixed;
          if (side == 0) reinterpret_cast<int64_t*>(s.hist)[sbase + m.most_freq_bin] = fixed;
        }
      } else {  // sequential subtraction in bin order, as a lane carry chain
        double g8[kPer], h8[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
          int t = lane * kPer + j;
          g8[j] = t < len ? sm.g[t] : 0.0;
          h8[j] = t < len ? sm.h[t] : 0.0;
        }
        double g = sl.sum_gradients, h = sl.sum_hessians;
        int32_t unused = 0;
        carry_chain(false, 0, (m.num_bin - 1) / kPer, g, h, unused, [&](int j, double& x, double& y, int32_t&) {
          int t = lane * kPer + j;
          if (t < m.num_bin && t != m.most_freq_bin) {
            x -= g8[j];
            y -= h8[j];
          }
        });
        __syncwarp();
        if (lane == 0) {
          sm.g[m.most_freq_bin] = g;
          sm.h[m.most_freq_bin] = h;
          if (side == 0) {
            double* w = reinterpret_cast<double*>(s.hist) + 2 * (sbase + m.most_freq_bin);
            w[0] = g;
            w[1] = h;
          }
        }
      }
    }
    __syncthreads();
    if (side == 1) {  // larger = parent - smaller, in the parent's buffer (histogram.rs:59-63)
      if (in_view) {
        if (kInt) {
          int64_t* lh = reinterpret_cast<int64_t*>(s.hist) + lbase;
          int64_t v = (int64_t)((uint64_t)pq - (uint64_t)sm.ig[tid]);
          sm.ig[tid] = v;
          lh[tid] = v;
        } else {
          double* lh = reinterpret_cast<double*>(s.hist) + 2 * lbase;
          double g = pgv - sm.g[tid], h = phv - sm.h[tid];
          sm.g[tid] = g;
          sm.h[tid] = h;
          lh[2 * tid] = g;
          lh[2 * tid + 1] = h;
        }
      }
      __syncthreads();
    }
    LeafCtx lc;
    lc.sum_g = ls.sum_gradients;
    lc.sum_h = ls.sum_hessians;
    lc.int_sum = ls.int_sum;
    lc.gs = gsc;
    lc.hs = hsc;
    lc.num_data = ls.num_data;
    // learner/mod.rs:1303-1309 parent output
    lc.parent_output = nl_cur == 1 ? root_output(ls.sum_gradients, ls.sum_hessians, p, ls.num_data) : ls.weight;
    lc.mc = p.use_monotone != 0;
    lc.cmin = cmin;
    lc.cmax = cmax;
    // the result is built in shared memory and stored once
    DSplit& out = sm.out;
    bool ok = find_best_threshold_block<kInt>(sm, m, p, lc, out);
    if (tid == 0) {
      out.feature = m.real_index;
      out.inner = f;
      s.feat_ok[side * nf + f] = ok ? 1 : 0;
    }
    __syncthreads();
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&out);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&s.feat_res[side * nf + f]);
    for (int i = tid; i < (int)(sizeof(DSplit) / 4); i += blockDim.x) dst[i] = src[i];
    // the partition's goes-left table for this candidate, ready if it wins
    if (ok) build_partition_lut(m, out, s.lut_cand + ((size_t)side * nf + f) * kMaxBins, tid, (int32_t)blockDim.x);
  }
}

// =====================================================================================
// Quantized threshold scan, one warp per (feature, side): the same search as
// scan_item / find_best_threshold_block / scan_direction_block for packed
// integer sums, with lane l holding stored bins 8l .. 8l + 7 in registers.
// Integer cumulative sums are exact in any order, and every per-candidate
// value comes from the same expressions, so the results are the block
// version's bit for bit; candidates reduce with the same tie rules. No block
// barrier is involved, so a CTA runs eight items side by side.
// =====================================================================================

// One direction of the quantized scan by one warp. vw[32 j + lane] is stored
// bin 8 * lane + j of the leaf's view (the most frequent bin fixed, the
// larger leaf's view already formed), in this warp's shared memory.
__device__ __noinline__ bool scan_direction_warp(const int64_t* vw, const DFeature& m, const DParams& p, const LeafCtx& lc,
                                    double min_gain_shift, double cnt_factor, bool reverse, bool skip_default,
                                    bool na_as_missing, DSplit& out) {
  const int lane = threadIdx.x & 31;
  const int offset = m.offset;
  const int len = m.view_len;
  int32_t t_lo, t_hi;
  if (reverse) {
    t_hi = m.num_bin - 1 - offset - (int32_t)na_as_missing;
    t_lo = 1 - offset;
  } else {
    t_lo = 0;
    t_hi = m.num_bin - 2 - offset;
  }
  const int32_t skip_t = skip_default ? m.default_bin - offset : INT32_MIN;
  auto visited = [&](int t) { return t >= t_lo && t <= t_hi && t != skip_t && t < len; };
  const bool first_extra = !reverse && na_as_missing && offset == 1;
  const int32_t nstored = m.num_bin - offset;
  // cumulative sums in scan order: ascending, the visited bins up to t;
  // reverse, the visited bins from t up (the total minus those below t)
  uint64_t pre = 0, all = 0;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int t = lane * kPer + j;
    const uint64_t x = (uint64_t)vw[32 * j + lane];
    if (visited(t)) pre += x;
    if (first_extra && t < len && t < nstored) all += x;
  }
  uint64_t incl = pre;  // inclusive over lanes of this lane's visited sum
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t other = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += other;
    all += __shfl_xor_sync(0xffffffffu, all, o);
  }
  const uint64_t total = __shfl_sync(0xffffffffu, incl, 31);
  const uint64_t base = first_extra ? (uint64_t)lc.int_sum - all : 0ull;
  const uint64_t run0 = incl - pre;  // visited bins below this lane's first
  // visits this lane's visited candidates with their cumulative packed sum
  // and count estimate, recomputed on each walk (no per-bin arrays live)
  auto walk = [&](auto fn) {
    uint64_t run = run0;
#pragma unroll 1
    for (int j = 0; j < kPer; ++j) {
      const int t = lane * kPer + j;
      const bool vis = visited(t);
      const uint64_t below = run;  // visited bins below t
      if (vis) {
        run += (uint64_t)vw[32 * j + lane];
        const int64_t q = (int64_t)(reverse ? total - below : base + run);
        fn(t, round_int((double)int_hess(q) * cnt_factor), q);
      }
    }
  };
  // the extra candidate t = -1 (lane 0)
  const int64_t eq = (int64_t)base;
  const int32_t ec = round_int((double)int_hess(eq) * cnt_factor);
  const int32_t min_data = p.min_data_in_leaf;
  const double min_hess = p.min_sum_hessian_in_leaf;
  const bool plain = plain_split(p, lc.mc);
  const bool extra = lane == 0 && first_extra;
  auto hsides = [&](int64_t aq, double& ha, double& hr) {
    ha = (double)int_hess(aq) * lc.hs;
    hr = (double)int_hess((int64_t)((uint64_t)lc.int_sum - (uint64_t)aq)) * lc.hs;
  };
  // pass 1: the first break in scan order
  int32_t brk = reverse ? INT32_MIN : INT32_MAX;
  auto break_at = [&](int t, int32_t ac, int64_t aq) {
    double ha, hr;
    hsides(aq, ha, hr);
    const bool skip1 = ac < min_data || ha < min_hess;
    if (!skip1 && (lc.num_data - ac < min_data || hr < min_hess)) brk = reverse ? max(brk, t) : min(brk, t);
  };
  walk(break_at);
  if (extra) break_at(-1, ec, eq);
  for (int o = 16; o > 0; o >>= 1) {
    const int32_t ob = __shfl_xor_sync(0xffffffffu, brk, o);
    brk = reverse ? max(brk, ob) : min(brk, ob);
  }
  // pass 2: gains of the candidates before the break
  double best_gain = -INFINITY;
  int32_t best_t = INT32_MIN;
  bool splittable = false;
  int64_t wq = 0;  // this lane's best candidate's cumulative values
  int32_t wc = 0;
  auto consider = [&](int t, int32_t ac, int64_t aq) {
    if (t >= 0 ? (reverse ? t <= brk : t >= brk) : !(brk > -1)) return;
    double ha, hr;
    hsides(aq, ha, hr);
    if (ac < min_data || ha < min_hess) return;
    const int64_t rest = (int64_t)((uint64_t)lc.int_sum - (uint64_t)aq);
    const double ga = (double)int_grad(aq) * lc.gs, gr = (double)int_grad(rest) * lc.gs;
    ha += kEpsilon;
    hr += kEpsilon;
    const int32_t rc = lc.num_data - ac;
    // the left child is the rest when scanning in reverse
    const double g1 = reverse ? gr : ga, h1 = reverse ? hr : ha, g2 = reverse ? ga : gr, h2 = reverse ? ha : hr;
    const int32_t c1 = reverse ? rc : ac, c2 = reverse ? ac : rc;
    const double gain = split_gain_hot(plain, g1, h1, g2, h2, p, c1, c2, lc.parent_output, lc.mc, lc.cmin, lc.cmax,
                                       m.monotone_type);
    if (gain <= min_gain_shift) return;
    splittable = true;
    if (gain > best_gain || (gain == best_gain && best_t != INT32_MIN && (reverse ? t > best_t : t < best_t))) {
      best_gain = gain;
      best_t = t;
      wq = aq;
      wc = ac;
    }
  };
  walk(consider);
  if (extra) consider(-1, ec, eq);
  warp_pick(reverse, best_gain, best_t);
  const bool any = __any_sync(0xffffffffu, splittable);
  ScanBest r;
  r.splittable = any;
  r.gain = best_gain;
  r.t = best_t;
  r.acc_g = r.acc_h = 0.0;
  // the winner's cumulative values, from the lane whose best it was (the
  // extra candidate t = -1 is lane 0's)
  const int src = best_t >= 0 ? best_t / kPer : 0;
  wq = (int64_t)__shfl_sync(0xffffffffu, (unsigned long long)wq, src);
  wc = __shfl_sync(0xffffffffu, wc, src);
  r.acc_q = best_t == INT32_MIN ? 0 : wq;
  r.acc_c = best_t == INT32_MIN ? 0 : wc;
  apply_direction<true>(r, m, p, lc.sum_g, lc.sum_h, lc.int_sum, lc.gs, lc.hs, lc.num_data, lc.parent_output, lc.mc,
                        lc.cmin, lc.cmax, min_gain_shift, cnt_factor, reverse, out);
  __syncwarp();
  return any;
}

// find_best_threshold (split.rs:246-271, :930-950) of the quantized form for
// one leaf and feature, by one warp; cat: the CTA's scratch, for a
// categorical feature (its view is copied there first).
__device__ bool find_best_threshold_warp(const int64_t* vw, ScanSmem* cat, const DFeature& m,
                                         const DParams& p, const LeafCtx& lc, DSplit& out) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    out.default_left = 1;
    out.gain = -INFINITY;
    out.num_cat = 0;
    out.monotone_type = 0;
  }
  __syncwarp();
  bool ok = false;
  if (m.bin_type == 1) {
#pragma unroll
    for (int j = 0; j < kPer; ++j) cat->ig[lane * kPer + j] = vw[32 * j + lane];
    __syncwarp();
    ok = scan_categorical<true>(*cat, m, p, lc, out);
  } else {
    if (lane == 0) out.monotone_type = m.monotone_type;
    const double sg = (double)int_grad(lc.int_sum) * lc.gs;
    const double sh = (double)int_hess(lc.int_sum) * lc.hs;
    const double min_gain_shift =
        leaf_gain_hot(plain_split(p, lc.mc), sg, sh, p, lc.num_data, lc.parent_output) + p.min_gain_to_split;
    const double cnt_factor = (double)lc.num_data / (double)int_hess(lc.int_sum);
    // split.rs:426-439: the directions scanned and their missing-value rules
    const bool two = m.num_bin > 2 && m.missing_type != 0;
    const bool skip_default = two && m.missing_type == 1;
    const bool na_missing = two && m.missing_type == 2;
#pragma unroll 1
    for (int d = 0; d < (two ? 2 : 1); ++d)
      ok |= scan_direction_warp(vw, m, p, lc, min_gain_shift, cnt_factor, d == 0, skip_default, na_missing, out);
    if (!two && lane == 0 && m.missing_type == 2) out.default_left = 0;
  }
  __syncwarp();
  if (lane == 0) out.gain *= m.penalty;
  __syncwarp();
  return ok;
}

// scan_item for the quantized form by one warp: feature f, side (0 smaller,
// 1 larger) of slot s. vw: this warp's view in shared memory ([kPer][32]);
// out: its result in shared memory.
__device__ void scan_item_warp(const DCtx& c, const DSlot& s, int f, int side, ScanSmem* cat, int64_t* vw,
                               DSplit& out) {
  DSlotState* st = s.st;
  const int lane = threadIdx.x & 31;
  const DFeature m = c.feats[f];
  const DParams& p = c.p;
  const int32_t nf = c.num_features;
  // two waves of loads, as in the block version: the slot state, then what
  // depends on it
  const int32_t larger_leaf = st->larger.leaf, L = st->left_leaf, s_buf = st->s_buf, l_buf = st->l_buf;
  const bool need = st->need_find != 0 && st->done == 0;
  const int32_t nl_cur = st->num_leaves_cur;
  const DLeafSplits sl = st->smaller;
  const DLeafSplits ls = side == 0 ? sl : st->larger;
  const double gsc = st->grad_scale, hsc = st->hess_scale;
  const bool have_larger = larger_leaf >= 0;
  const bool live = need && (side == 0 || have_larger);
  const int len = m.view_len;
  const size_t sbase = (size_t)s_buf * c.total_bins + m.view_start;
  const size_t lbase = (size_t)l_buf * c.total_bins + m.view_start;
  const long long* hsrc = reinterpret_cast<const long long*>(s.hist);
  int64_t v[kPer], pv[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int i = lane * kPer + j;
    // histogram cells are written by other CTAs' atomics: loaded through L2
    v[j] = (live && i < len) ? (int64_t)__ldcg(hsrc + sbase + i) : 0;
    pv[j] = (live && side == 1 && i < len) ? (int64_t)__ldcg(hsrc + lbase + i) : 0;
  }
  const uint8_t in_tree = s.bytree[f];
  const uint8_t split_ok = have_larger ? s.splittable[L * nf + f] : (uint8_t)1;
  const double cmin = live ? s.cmin[ls.leaf] : 0.0, cmax = live ? s.cmax[ls.leaf] : 0.0;
  if (!(live && in_tree && split_ok)) return;
  int64_t* hdst = reinterpret_cast<int64_t*>(s.hist);
  // the smaller leaf's view with its most frequent bin fixed (histogram.rs:42-56; exact in any order)
  if (m.most_freq_bin > 0) {
    uint64_t part = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = lane * kPer + j;
      if (i < m.num_bin && i != m.most_freq_bin) part += (uint64_t)v[j];
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    const int64_t fixed = (int64_t)((uint64_t)sl.int_sum - part);
#pragma unroll
    for (int j = 0; j < kPer; ++j)
      if (lane * kPer + j == m.most_freq_bin) {
        v[j] = fixed;
        if (side == 0) hdst[sbase + m.most_freq_bin] = fixed;
      }
  }
  if (side == 1) {  // larger = parent - smaller, in the parent's buffer (histogram.rs:59-63)
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = lane * kPer + j;
      if (i < len) {
        v[j] = (int64_t)((uint64_t)pv[j] - (uint64_t)v[j]);
        hdst[lbase + i] = v[j];
      }
    }
  }
  LeafCtx lc;
  lc.sum_g = ls.sum_gradients;
  lc.sum_h = ls.sum_hessians;
  lc.int_sum = ls.int_sum;
  lc.gs = gsc;
  lc.hs = hsc;
  lc.num_data = ls.num_data;
  // learner/mod.rs:1303-1309 parent output
  lc.parent_output = nl_cur == 1 ? root_output(ls.sum_gradients, ls.sum_hessians, p, ls.num_data) : ls.weight;
  lc.mc = p.use_monotone != 0;
  lc.cmin = cmin;
  lc.cmax = cmax;
#pragma unroll
  for (int j = 0; j < kPer; ++j) vw[32 * j + lane] = v[j];
  __syncwarp();
  const bool ok = find_best_threshold_warp(vw, cat, m, p, lc, out);
  if (lane == 0) {
    out.feature = m.real_index;
    out.inner = f;
    s.feat_ok[side * nf + f] = ok ? 1 : 0;
  }
  __syncwarp();
  const uint32_t* src = reinterpret_cast<const uint32_t*>(&out);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&s.feat_res[side * nf + f]);
  for (int i = lane; i < (int)(sizeof(DSplit) / 4); i += 32) dst[i] = src[i];
  // the partition's goes-left table for this candidate, ready if it wins
  if (ok) build_partition_lut(m, out, s.lut_cand + ((size_t)side * nf + f) * kMaxBins, lane, 32);
}

// Grid (CTAs, 1, slots), kScanThreads threads: warp w of CTA b scans item
// items[8b + w] (feature * 2 + side, or -1 for none) of slot z. The host
// gives each CTA at most one categorical item, which uses the CTA's scratch.
template <int kMinBlocks>
__global__ void __launch_bounds__(kScanThreads, kMinBlocks) k_scan_warp(const __grid_constant__ DCtx c,
                                                                        const int32_t* items) {
  __shared__ ScanSmem cat;
  __shared__ DSplit outs[kScanThreads / 32];
  __shared__ int64_t views[kScanThreads / 32][kPer * 32];
  pdl_wait();
  pdl_trigger();
  const DSlot& s = c.slots[blockIdx.z];
  DSlotState* st = s.st;
  const int warp = threadIdx.x >> 5;
  // the partition that follows claims its row tiles from this counter
  if (blockIdx.x == 0 && threadIdx.x == 0 && !st->done) {
    st->part_ticket = 0;
    st->part_done = 0;
  }
  const int32_t it = items[blockIdx.x * (kScanThreads / 32) + warp];
  if (it < 0) return;
  scan_item_warp(c, s, it >> 1, it & 1, &cat, views[warp], outs[warp]);
}
template __global__ void k_scan_warp<2>(const __grid_constant__ DCtx, const int32_t*);
template __global__ void k_scan_warp<kScanWideBlocks>(const __grid_constant__ DCtx, const int32_t*);

// kMinBlocks: CTAs the compiler keeps resident per SM (registers capped to
// fit). 1 for a step of few features, where each CTA's latency is what counts;
// kScanWideBlocks when a step's (feature, side, slot) CTAs span several waves
// (many features or tree slots), where residency counts more than the few
// registers that then spill.
template <bool kInt, int kMinBlocks>
__global__ void __launch_bounds__(kScanThreads, kMinBlocks) k_scan(const __grid_constant__ DCtx c) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_wait();
  pdl_trigger();
  const DSlot& s = c.slots[blockIdx.z];
  DSlotState* st = s.st;
  // the partition that follows claims its row tiles from this counter
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && !st->done) {
    st->part_ticket = 0;
    st->part_done = 0;
  }
  scan_item<kInt>(c, s, blockIdx.x, blockIdx.y, *reinterpret_cast<ScanSmem*>(smem_raw));
}
template __global__ void k_scan<false, 1>(const __grid_constant__ DCtx);
template __global__ void k_scan<true, 1>(const __grid_constant__ DCtx);
template __global__ void k_scan<false, kScanWideBlocks>(const __grid_constant__ DCtx);
template __global__ void k_scan<true, kScanWideBlocks>(const __grid_constant__ DCtx);

// =====================================================================================
// partition (partition.rs:107-174): out-of-place split of the leaf's rows into
// the other index buffer; left rows keep their order, right rows are written
// from the end (reversed). Tiles are claimed in order and chained with a
// decoupled look-back on the running left count.
// =====================================================================================
constexpr unsigned long long kFlagAgg = 1ull << 62, kFlagInc = 2ull << 62;
constexpr uint32_t kEpochMask = 0x7FFFFFFFu;
constexpr unsigned long long kValueMask = (1ull << 31) - 1;

// status word: flag (2 bits) | epoch (31 bits) | left count (31 bits)
__device__ __forceinline__ unsigned long long pack_status(uint32_t epoch, unsigned long long flag, uint64_t v) {
  return flag | ((unsigned long long)(epoch & kEpochMask) << 31) | (v & kValueMask);
}

// What partition_finalize reads, loaded before apply_split runs so that the
// two sets of loads overlap.
struct FinalizeIn {
  int32_t begin, cnt, gcnt, side, buf_L, depth, status;
  DLeafSplits ls0, rs0;
};

__device__ __forceinline__ FinalizeIn finalize_inputs(const DSlot& s, int32_t L, int32_t R, const DSplit& info) {
  FinalizeIn f;
  f.begin = s.leaf_begin[L];
  f.cnt = s.leaf_count[L];
  f.gcnt = s.leaf_gcount[L];
  f.side = s.leaf_side[L];
  f.buf_L = s.buf_of[L];
  f.depth = s.tree.leaf_depth[L] + 1;  // both children's depth after the split
  f.status = s.st->status;
  f.ls0 = DLeafSplits{L, 0, info.left_sum_gradient, info.left_sum_hessian, info.left_sum_gh, info.left_output};
  f.rs0 = DLeafSplits{R, 0, info.right_sum_gradient, info.right_sum_hessian, info.right_sum_gh, info.right_output};
  return f;
}

// gleft: every rank's rows sent left (data-parallel growth), or -1: this
// rank's total_left is the whole count.
__device__ void partition_finalize(const DCtx& c, const DSlot& s, int32_t L, int32_t R, int32_t total_left,
                                   const FinalizeIn& fin, int32_t gleft = -1) {
  DSlotState* st = s.st;
  const DParams& p = c.p;
  const int32_t begin = fin.begin, cnt = fin.cnt, side = fin.side, buf_L = fin.buf_L, depth = fin.depth;
  const DLeafSplits ls0 = fin.ls0, rs0 = fin.rs0;
  const int32_t status = fin.status;
  const int32_t nl = total_left, nr = cnt - total_left;  // this rank's rows: the ranges
  const int32_t gl = gleft >= 0 ? gleft : nl, gr = gleft >= 0 ? fin.gcnt - gleft : nr;  // the counts
  s.leaf_count[L] = nl;
  s.leaf_begin[R] = begin + nl;
  s.leaf_count[R] = nr;
  s.leaf_gcount[L] = gl;
  s.leaf_gcount[R] = gr;
  s.leaf_side[L] = 1 - side;
  s.leaf_side[R] = 1 - side;
  const DTree& t = s.tree;
  const int32_t node = R - 1;
  t.leaf_count[L] = gl;
  t.leaf_count[R] = gr;
  t.internal_count[node] = gl + gr;
  DLeafSplits ls = ls0, rs = rs0;
  ls.num_data = gl;
  rs.num_data = gr;
  int32_t new_status = status;
  const bool left_smaller = gl < gr;  // learner/mod.rs:1200-1208
  if ((left_smaller ? gl : gr) <= 0 && status == kStatusOk) new_status = kStatusEmptyChild;
  st->smaller = left_smaller ? ls : rs;
  st->larger = left_smaller ? rs : ls;
  if (new_status != kStatusOk) {
    st->status = new_status;
    st->done = 1;
    return;
  }
  // HistogramPool::Move: the parent's buffer goes to the larger leaf, the
  // fresh buffer R (zeroed by this kernel) to the smaller one.
  if (!left_smaller) {
    s.buf_of[R] = R;
  } else {
    s.buf_of[R] = buf_L;
    s.buf_of[L] = R;
  }
  // the next step's histogram and scan read these instead of the leaf arrays
  st->s_begin = left_smaller ? begin : begin + nl;
  st->s_count = left_smaller ? nl : nr;
  st->s_side = 1 - side;
  st->s_buf = R;
  st->l_buf = buf_L;
  st->left_leaf = L;
  st->right_leaf = R;
  // before_find_best_split (learner/mod.rs:712-731) on the values just written
  bool need = true;
  if (p.max_depth > 0 && depth >= p.max_depth) need = false;
  else if (gr < p.min_data_in_leaf * 2 && gl < p.min_data_in_leaf * 2) need = false;
  if (!need) {
    s.best[L].gain = -INFINITY;
    s.bgain[L] = -INFINITY;
    s.best[R].gain = -INFINITY;
    s.bgain[R] = -INFINITY;
  }
  st->need_find = need ? 1 : 0;
}

// The slot-state fields a partition CTA reads first, loaded together.
struct StepHead {
  int32_t done, need, S, G, Lft, R;
  uint32_t epoch;
};

__device__ __forceinline__ StepHead load_step_head(const DSlotState* st) {
  StepHead h;
  h.done = st->done;
  h.need = st->need_find;
  h.S = st->smaller.leaf;
  h.G = st->larger.leaf;
  h.Lft = st->left_leaf;
  h.R = st->num_leaves_cur;
  h.epoch = st->part_epoch;
  return h;
}

// Decision state a partition CTA derives from the scan results.
struct SplitDecision {
  double side_bg[2];     // best (penalized) gain of the smaller / larger new leaf
  int32_t side_feat[2];  // its real feature, -1 none
  int32_t side_bf[2];    // its inner feature, -1 none
  double wbg[32];
  int32_t wfeat[32], wleaf[32];
  int32_t bl;            // the leaf to split, -1: the tree is finished
};
static_assert(sizeof(SplitDecision) <= kDpDecBytes, "the data-parallel decision buffer is too small");


// Best split of a new leaf over its features and its per-feature splittable
// flags (learner/mod.rs:842-849, :1066-1086); one warp.
__device__ void new_leaf_best(const DCtx& c, const DSlot& s, int side, int32_t leaf, bool have_larger, int32_t Lft,
                              double& bg, int32_t& bfeat, int32_t& bf) {
  const int lane = threadIdx.x & 31;
  const DParams& p = c.p;
  const int32_t nf = c.num_features;
  double pen = p.use_monotone ? monotone_split_gain_penalty(s.tree.leaf_depth[leaf], p.monotone_penalty) : 1.0;
  bg = -INFINITY;
  bfeat = -1;
  bf = -1;
  for (int ff = lane; ff < nf; ff += 32) {
    // every input read at once (none of these loads depends on another)
    const uint8_t in_tree = s.bytree[ff];
    const uint8_t split_ok = have_larger ? s.splittable[Lft * nf + ff] : (uint8_t)1;
    const DSplit& r = s.feat_res[side * nf + ff];
    double g = r.gain;
    const int32_t fe = r.feature;
    const int32_t mono = r.monotone_type;
    if (!(in_tree && split_ok)) continue;
    if (mono != 0) g *= pen;
    if (better_than(g, fe, bg, bfeat)) {
      bg = g;
      bfeat = fe;
      bf = ff;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    double og = __shfl_xor_sync(0xffffffffu, bg, o);
    int32_t ofe = __shfl_xor_sync(0xffffffffu, bfeat, o);
    int32_t off = __shfl_xor_sync(0xffffffffu, bf, o);
    if (better_than(og, ofe, bg, bfeat)) {
      bg = og;
      bfeat = ofe;
      bf = off;
    }
  }
}

// Leaf argmax rule of best_leaf (learner/mod.rs:698-706): larger gain, then
// smaller feature, then smaller leaf.
__device__ __forceinline__ bool leaf_takes(double og, int32_t ofe, int32_t ol, double bg, int32_t bfeat, int32_t bl) {
  if (ol == INT32_MAX) return false;
  if (bl == INT32_MAX) return true;
  if (better_than(og, ofe, bg, bfeat)) return true;
  return !better_than(bg, bfeat, og, ofe) && ol < bl;
}

// Split decision of this step, computed by every partition CTA: the best
// split of the two new leaves (warps 0, 1), the best of the other leaves
// (warps 2..), then the best leaf (thread 0).
__device__ void decide_split(const DCtx& c, const DSlot& s, const StepHead& h, SplitDecision& d) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool need = h.need != 0;
  const int32_t S = h.S, G = h.G, Lft = h.Lft;
  const bool have_larger = G >= 0;
  const int32_t NL = c.p.num_leaves;
  if (warp < 2) {
    double bg = -INFINITY;
    int32_t bfeat = -1, bf = -1;
    if (need && (warp == 0 || have_larger)) new_leaf_best(c, s, warp, warp == 0 ? S : G, have_larger, Lft, bg, bfeat, bf);
    if (lane == 0) {
      d.side_bg[warp] = bf >= 0 ? bg : -INFINITY;
      d.side_feat[warp] = bf >= 0 ? bfeat : -1;
      d.side_bf[warp] = bf;
    }
  } else {
    double bg = -INFINITY;
    int32_t bfeat = -1, bl = INT32_MAX;
    for (int32_t l = tid - 64; l < NL; l += (int32_t)blockDim.x - 64) {
      if (need && (l == S || l == G)) continue;
      double g = s.bgain[l];
      int32_t fe = s.bfeat[l];
      if (leaf_takes(g, fe, l, bg, bfeat, bl)) {
        bg = g;
        bfeat = fe;
        bl = l;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double og = __shfl_xor_sync(0xffffffffu, bg, o);
      int32_t ofe = __shfl_xor_sync(0xffffffffu, bfeat, o);
      int32_t ol = __shfl_xor_sync(0xffffffffu, bl, o);
      if (leaf_takes(og, ofe, ol, bg, bfeat, bl)) {
        bg = og;
        bfeat = ofe;
        bl = ol;
      }
    }
    if (lane == 0) {
      d.wbg[warp] = bg;
      d.wfeat[warp] = bfeat;
      d.wleaf[warp] = bl;
    }
  }
  __syncthreads();
  if (tid == 0) {
    double bg = -INFINITY;
    int32_t bfeat = -1, bl = INT32_MAX;
    auto offer = [&](double g, int32_t fe, int32_t l) {
      if (leaf_takes(g, fe, l, bg, bfeat, bl)) {
        bg = g;
        bfeat = fe;
        bl = l;
      }
    };
    for (int w = 2; w < (int)(blockDim.x >> 5); ++w) offer(d.wbg[w], d.wfeat[w], d.wleaf[w]);
    if (need) {
      offer(d.side_bg[0], d.side_feat[0], S);
      if (have_larger) offer(d.side_bg[1], d.side_feat[1], G);
    }
    d.bl = (bl != INT32_MAX && bg > 0.0) ? bl : -1;
  }
  __syncthreads();
}

// End of a split step, by the last CTA of the launch to finish: the new
// leaves' best splits and splittable flags are stored, the split is applied
// to the tree (tree.rs:240-297) and the children's ranges, smaller / larger
// choice and before_find_best_split are recorded. Every other CTA of the
// launch has exited, so none of them reads the state changed here.
__device__ void finish_step(const DCtx& c, const DSlot& s, const StepHead& h, const SplitDecision& d, int32_t bl,
                            int32_t R, int32_t cnt, int32_t gleft = -1) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  DSlotState* st = s.st;
  const int32_t nf = c.num_features;
  const bool need = h.need != 0;
  const int32_t S = h.S, G = h.G, Lft = h.Lft;
  const bool have_larger = G >= 0;
  // the split's record, where the decision found it (not modified below)
  const DSplit& src = (need && bl == S)   ? s.feat_res[d.side_bf[0]]
                      : (need && bl == G) ? s.feat_res[nf + d.side_bf[1]]
                                          : s.best[bl];
  // Every warp starts at once: the stored records of the new leaves (warps 2
  // and 3) and their splittable flags (warps 4 and up) are nothing the tree
  // update (thread 0) or the leaf bookkeeping (thread 32) reads, and the
  // split's record is read from the scan results when it is a new leaf's.
  ApplyIn ain;
  FinalizeIn fin;
  int32_t total_left = 0;
  if (tid == 0) {
    ain = apply_load(c, s, src, bl);
    // the persisted record carries the penalized gain
    if (need && bl == S) ain.info.gain = d.side_bg[0];
    else if (need && bl == G) ain.info.gain = d.side_bg[1];
  } else if (tid == 32) {
    fin = finalize_inputs(s, bl, R, src);
    total_left = cnt > 0 ? *reinterpret_cast<volatile int32_t*>(&st->part_left) : 0;
  }
  if (need) {
    // one thread per feature: its flag is read before it is overwritten (the
    // smaller leaf can be the left leaf whose flags are read)
    for (int ff = tid - 128; tid >= 128 && ff < nf; ff += (int)blockDim.x - 128) {
      bool u = s.bytree[ff] && (!have_larger || s.splittable[Lft * nf + ff]);
      uint8_t ns = u ? s.feat_ok[ff] : 0;
      uint8_t ng = u ? s.feat_ok[nf + ff] : 0;
      s.splittable[S * nf + ff] = ns;
      if (have_larger) s.splittable[G * nf + ff] = ng;
    }
    const int side = warp - 2;
    if ((side == 0 || (side == 1 && have_larger))) {
      const int32_t leaf = side == 0 ? S : G;
      const int32_t bf = d.side_bf[side];
      DSplit& dst = s.best[leaf];
      if (bf >= 0) {
        const uint32_t* from = reinterpret_cast<const uint32_t*>(&s.feat_res[side * nf + bf]);
        uint32_t* w = reinterpret_cast<uint32_t*>(&dst);
        for (int i = lane; i < (int)(sizeof(DSplit) / 4); i += 32) w[i] = from[i];
        if (lane < kMaxBins / 16)
          reinterpret_cast<uint4*>(s.leaf_lut + (size_t)leaf * kMaxBins)[lane] =
              reinterpret_cast<const uint4*>(s.lut_cand + ((size_t)side * nf + bf) * kMaxBins)[lane];
        __syncwarp();
        if (lane == 0) {
          dst.gain = d.side_bg[side];
          s.bgain[leaf] = d.side_bg[side];
          s.bfeat[leaf] = dst.feature;
        }
      } else if (lane == 0) {
        dst.feature = -1;
        dst.inner = -1;
        dst.gain = -INFINITY;
        s.bgain[leaf] = -INFINITY;
        s.bfeat[leaf] = -1;
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    apply_split(c, s, bl, R, ain);
  } else if (tid == 32) {
    partition_finalize(c, s, bl, R, total_left, fin, gleft);
    st->part_epoch += 1;
    // every CTA of the launch has passed its last use of the step counters
    st->part_ticket = 0;
    st->part_done = 0;
    st->scan_done = 0;
  }
}

// Shared state of a partition CTA.
struct PartShared {
  alignas(16) uint8_t lut[kMaxBins];
  int32_t warp_tot[32];
  int32_t tile, prefix;
  bool last;
  SplitDecision dec;
};


// The leaf a step splits: its rows and the feature its split tests.
struct SplitLeaf {
  int32_t L, begin, cnt, side, inner;
  int32_t depth;  // the children's depth (CTA 0 of a deferring launch only)
};

// Step prologue of a partition CTA: the split decision and, when a leaf is
// split, its goes-left LUT in ps.lut (built by the scan for each candidate
// and kept per leaf when the candidates are stored). L < 0: the tree is
// finished.
__device__ SplitLeaf partition_prologue(const DCtx& c, const DSlot& s, const StepHead& h, PartShared& ps) {
  decide_split(c, s, h, ps.dec);
  SplitLeaf sl;
  sl.L = ps.dec.bl;
  if (sl.L < 0) return sl;
  const int32_t L = sl.L, nf = c.num_features;
  const bool from_s = h.need && L == h.S, from_g = h.need && L == h.G;
  const int32_t cand = from_s ? ps.dec.side_bf[0] : from_g ? nf + ps.dec.side_bf[1] : -1;
  // every load of the leaf's facts and its table at once
  const DSplit& info = cand >= 0 ? s.feat_res[cand] : s.best[L];
  const uint8_t* lut = cand >= 0 ? s.lut_cand + (size_t)cand * kMaxBins : s.leaf_lut + (size_t)L * kMaxBins;
  sl.begin = s.leaf_begin[L];
  sl.cnt = s.leaf_count[L];
  sl.side = s.leaf_side[L];
  sl.inner = info.inner;
  sl.depth = (c.defer && blockIdx.x == 0) ? s.tree.leaf_depth[L] + 1 : 0;
  if (threadIdx.x < kMaxBins / 16)
    reinterpret_cast<uint4*>(ps.lut)[threadIdx.x] = reinterpret_cast<const uint4*>(lut)[threadIdx.x];
  return sl;
}

// One partition tile after its goes-left flags are known: a block scan of
// the per-thread left counts, the decoupled look-back for the tile's prefix,
// then the scatter (left rows ascending from the range start, right rows
// descending from its end). The CTA of the last tile posts the left count.
template <int kItems>
__device__ void tile_scatter(const DSlot& s, PartShared& ps, int32_t tile, int32_t ntiles, uint32_t epoch, int32_t t0,
                             int32_t cnt, const uint32_t (&rows)[kItems], uint32_t flags, int32_t nleft,
                             uint32_t* out) {
  DSlotState* st = s.st;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // block exclusive scan of per-thread left counts
    int32_t incl = nleft;
    for (int o = 1; o < 32; o <<= 1) {
      int32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) ps.warp_tot[warp] = incl;
    __syncthreads();
    int32_t wbase = 0, tile_left = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      if (w < warp) wbase += ps.warp_tot[w];
      tile_left += ps.warp_tot[w];
    }
    const int32_t excl = wbase + incl - nleft;
    // decoupled look-back on the left count: warp 0 reads 32 predecessors at a
    // time and sums back to the nearest one whose inclusive prefix is posted
    if (warp == 0) {
      unsigned long long* stat = s.tile_status;
      if (tile == 0) {
        if (lane == 0) {
          atomicExch(&stat[0], pack_status(epoch, kFlagInc, (uint64_t)tile_left));
          ps.prefix = 0;
        }
      } else {
        if (lane == 0) atomicExch(&stat[tile], pack_status(epoch, kFlagAgg, (uint64_t)tile_left));
        int64_t acc = 0;
        int32_t base = tile - 1;
        int spins = 0;
        while (true) {
          const int32_t pred = base - lane;
          bool valid = true, inc = true;
          uint64_t val = 0;
          if (pred >= 0) {
            unsigned long long v = *reinterpret_cast<volatile unsigned long long*>(&stat[pred]);
            uint32_t ve = (uint32_t)((v >> 31) & kEpochMask);
            unsigned long long flag = v & (3ull << 62);
            valid = ve == (epoch & kEpochMask) && flag != 0;
            inc = flag == kFlagInc;
            val = v & kValueMask;
          }
          const unsigned inc_mask = __ballot_sync(0xffffffffu, valid && inc);
          const unsigned bad_mask = __ballot_sync(0xffffffffu, !valid);
          const int first_inc = inc_mask ? __ffs(inc_mask) - 1 : 32;
          const unsigned need = first_inc >= 31 ? 0xffffffffu : ((2u << first_inc) - 1u);
          if (bad_mask & need) {
            if (++spins > kSpinLimit) {  // give up: the prefix 0 keeps every write in the leaf's range;
              if (lane == 0) st->status = kStatusTimeout;  // the step's end then finishes the tree
              acc = 0;
              break;
            }
            __nanosleep(32);
            continue;
          }
          int64_t part = lane <= first_inc ? (int64_t)val : 0;
          for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
          acc += part;
          if (first_inc < 32) break;
          base -= 32;
        }
        if (lane == 0) {
          atomicExch(&stat[tile], pack_status(epoch, kFlagInc, (uint64_t)(acc + tile_left)));
          ps.prefix = (int32_t)acc;
        }
      }
    }
    __syncthreads();
    const int32_t prefix = ps.prefix;
    // scatter: left rows ascending from begin, right rows descending from the end
    int32_t lrank = prefix + excl;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
      int32_t pos = t0 + tid * kItems + k;
      if (pos < cnt) {
        if (flags & (1u << k)) {
          out[lrank++] = rows[k];
        } else {
          int32_t rrank = pos - lrank;  // rights before this row
          out[cnt - 1 - rrank] = rows[k];
        }
      }
    }
    if (tile == ntiles - 1 && tid == 0) st->part_left = prefix + tile_left;
}

// Row tiles of the split leaf L claimed in order by the CTAs (kItems rows
// per thread, blockDim.x * kItems == kPartTileRows), each chained to its
// predecessors by a decoupled look-back on the left count. The CTA that
// partitions the last tile posts the left count in st->part_left.
// With `claimed` the CTA's first ticket is already in ps.tile; the next one
// is claimed while a tile runs and used after it.
template <int kItems>
__device__ void partition_rows(const DCtx& c, const DSlot& s, PartShared& ps, const SplitLeaf& sl, uint32_t epoch,
                               bool claimed) {
  static_assert(kItems <= 32, "one goes-left bit per item");
  DSlotState* st = s.st;
  const int tid = threadIdx.x;
  const int32_t begin = sl.begin, cnt = sl.cnt, side = sl.side, inner = sl.inner;
  if (cnt == 0) return;
  const uint32_t* in = s.idx[side] + begin;
  uint32_t* out = s.idx[1 - side] + begin;
  const int32_t ntiles = (cnt + kPartTileRows - 1) / kPartTileRows;
  const uint8_t* col = c.colbins + (size_t)inner * (size_t)c.num_data;
  const uint8_t* lut = ps.lut;
  int32_t next = -1;  // thread 0: the ticket after the current tile (the counter is contended: used a tile later)
  while (true) {
    __syncthreads();
    if (tid == 0 && !claimed) ps.tile = next >= 0 ? next : atomicAdd(&st->part_ticket, 1);
    claimed = false;
    __syncthreads();
    const int32_t tile = ps.tile;
    if (tile >= ntiles) break;
    if (tid == 0) next = atomicAdd(&st->part_ticket, 1);
    const int32_t t0 = tile * kPartTileRows;
    uint32_t rows[kItems];
    uint32_t flags = 0;
    int32_t nleft = 0;
    // every row index first, then every byte of the split feature: each
    // group of loads is in flight together
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
      const int32_t pos = t0 + tid * kItems + k;
      rows[k] = pos < cnt ? __ldcg(in + pos) : 0u;
    }
    uint32_t raws[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
      const int32_t pos = t0 + tid * kItems + k;
      raws[k] = pos < cnt ? (uint32_t)col[rows[k]] : 0u;
    }
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
      const int32_t pos = t0 + tid * kItems + k;
      if (pos < cnt && lut[raws[k]]) {
        flags |= 1u << k;
        ++nleft;
      }
    }
    tile_scatter<kItems>(s, ps, tile, ntiles, epoch, t0, cnt, rows, flags, nleft, out);
  }
}

// Zeroes histogram buffer R (the next smaller leaf's), spread over `count`
// CTAs of which this is `rank`.
__device__ __forceinline__ void zero_hist_buffer(const DCtx& c, const DSlot& s, int32_t R, int rank, int count) {
  size_t cells = (size_t)c.total_bins * (c.hist_mode == LGBM_B200_HIST_QUANT ? 1 : 2);
  double* h = reinterpret_cast<double*>(s.hist) + (size_t)R * cells;
  for (size_t i = (size_t)rank * blockDim.x + threadIdx.x; i < cells; i += (size_t)count * blockDim.x) h[i] = 0.0;
}

// The partition of a step after the step fields are loaded and the first
// ticket is claimed (in ps.tile).
__device__ __forceinline__ void partition_body(const DCtx& c, const DSlot& s, PartShared& ps, const StepHead& h) {
  DSlotState* st = s.st;
  const int tid = threadIdx.x;
  const int32_t R = h.R;
  const SplitLeaf sl = partition_prologue(c, s, h, ps);
  const int32_t L = sl.L;
  if (L < 0) {
    if (blockIdx.x == 0 && tid == 0) {
      st->done = 1;
      st->pending = 0;
    }
    return;
  }
  if (c.defer && blockIdx.x == 0 && tid == 0) {
    // the step's end is left to the next histogram launch: post what it and
    // the histogram's row CTAs need (the left count follows from the tiles)
    st->pd_bl = L;
    st->pd_begin = sl.begin;
    st->pd_cnt = sl.cnt;
    st->pd_side = sl.side;
    st->pd_depth = sl.depth;
    st->pd_need = h.need;
    st->pd_S = h.S;
    st->pd_G = h.G;
    st->pd_Lft = h.Lft;
    st->pd_R = R;
    for (int k = 0; k < 2; ++k) {
      st->pd_bf[k] = ps.dec.side_bf[k];
      st->pd_bg[k] = ps.dec.side_bg[k];
    }
    st->pending = 1;
  }
  zero_hist_buffer(c, s, R, blockIdx.x, gridDim.x);
  if (blockIdx.x == 0 && tid == 0) st->part_rows += sl.cnt;
  partition_rows<kPartTileRows / kPartThreads>(c, s, ps, sl, h.epoch, true);
  if (c.defer) return;
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    ps.last = atomicAdd(&st->part_done, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (ps.last) {
    __threadfence();
    if (c.dp) {
      // data-parallel: the step ends in k_dp_finish once the left rows of every
      // rank are summed; the decision and this rank's left rows wait for it
      const uint32_t* from = reinterpret_cast<const uint32_t*>(&ps.dec);
      uint32_t* to = reinterpret_cast<uint32_t*>(s.dp_dec);
      for (int i = tid; i < (int)(sizeof(SplitDecision) / 4); i += blockDim.x) to[i] = from[i];
      if (tid == 0) s.dp_left[0] = sl.cnt > 0 ? *reinterpret_cast<volatile int32_t*>(&st->part_left) : 0;
    } else {
      finish_step(c, s, h, ps.dec, L, R, sl.cnt);
    }
  }
}

// Data-parallel growth: the end of a split step (finish_step) after the
// partition, with dp_left[0] holding the rows every rank sent left. Grid
// (1, 1, slots), kPartThreads threads.
__global__ void __launch_bounds__(kPartThreads) k_dp_finish(const __grid_constant__ DCtx c) {
  const DSlot& s = c.slots[blockIdx.z];
  __shared__ SplitDecision dec;
  const StepHead h = load_step_head(s.st);
  if (h.done) return;
  const uint32_t* from = reinterpret_cast<const uint32_t*>(s.dp_dec);
  uint32_t* to = reinterpret_cast<uint32_t*>(&dec);
  for (int i = threadIdx.x; i < (int)(sizeof(SplitDecision) / 4); i += blockDim.x) to[i] = from[i];
  __syncthreads();
  const int32_t L = dec.bl;
  if (L < 0) return;
  finish_step(c, s, h, dec, L, h.R, s.leaf_count[L], s.dp_left[0]);
}

// Data-parallel growth: the root's sums of this rank out (sum_g, sum_h as
// f64; the packed integer sum and the row count as i64), and back in once
// summed over the ranks, with what k_tree_init derived from them. Grid (1, 1, slots).
__global__ void k_dp_root_pack(const __grid_constant__ DCtx c, double* f, long long* q) {
  const DSlotState* st = c.slots[blockIdx.z].st;
  f[2 * blockIdx.z] = st->smaller.sum_gradients;
  f[2 * blockIdx.z + 1] = st->smaller.sum_hessians;
  q[2 * blockIdx.z] = (long long)st->smaller.int_sum;
  q[2 * blockIdx.z + 1] = (long long)st->smaller.num_data;
}

__global__ void k_dp_root_apply(const __grid_constant__ DCtx c, const double* f, const long long* q) {
  const DSlot& s = c.slots[blockIdx.z];
  DSlotState* st = s.st;
  const double a = f[2 * blockIdx.z], b = f[2 * blockIdx.z + 1];
  const int32_t n = (int32_t)q[2 * blockIdx.z + 1];
  st->smaller.sum_gradients = a;
  st->smaller.sum_hessians = b;
  st->smaller.int_sum = (int64_t)q[2 * blockIdx.z];
  st->smaller.num_data = n;
  s.leaf_gcount[0] = n;
  s.tree.leaf_value[0] = maybe_round_to_zero(root_output(a, b, c.p, n));
  st->need_find = before_find_best_split(c, s, 0, -1) ? 1 : 0;
}

// Grid (G, 1, slots), kPartThreads threads. Every CTA first derives the
// step's split decision and the goes-left LUT, then claims row tiles; the
// last CTA to exit ends the step.
__global__ void __launch_bounds__(kPartThreads) k_partition(const __grid_constant__ DCtx c) {
  pdl_wait();
  pdl_trigger();
  const DSlot& s = c.slots[blockIdx.z];
  __shared__ PartShared ps;
  // the step's fields and this CTA's first row tile, in one round trip (a
  // finished tree's launch claims tickets nobody uses; the counter is reset
  // before every partition of a live tree)
  const StepHead h = load_step_head(s.st);
  if (threadIdx.x == 0) ps.tile = atomicAdd(&s.st->part_ticket, 1);
  if (h.done) {
    // a step end that finished the tree ran beside the last histogram launch
    if (blockIdx.x == 0 && threadIdx.x == 0) s.st->pending = 0;
    return;
  }
  partition_body(c, s, ps, h);
}

// The end of a split step that a partition posted (finish_step with the
// posted head and decision), by one whole CTA of at least kPartThreads
// threads; dec_smem holds a SplitDecision. Nothing else of the launch reads
// what it writes.
__device__ void deferred_finish(const DCtx& c, const DSlot& s, void* dec_smem) {
  DSlotState* st = s.st;
  SplitDecision& d = *static_cast<SplitDecision*>(dec_smem);
  // every field read at once (the same addresses in every thread)
  const int32_t pending = st->pending, bl = st->pd_bl, cnt = st->pd_cnt;
  StepHead h;
  h.done = 0;
  h.need = st->pd_need;
  h.S = st->pd_S;
  h.G = st->pd_G;
  h.Lft = st->pd_Lft;
  h.R = st->pd_R;
  h.epoch = 0;
  if (threadIdx.x < 2) {
    d.side_bf[threadIdx.x] = st->pd_bf[threadIdx.x];
    d.side_bg[threadIdx.x] = st->pd_bg[threadIdx.x];
  }
  if (threadIdx.x == 0) d.bl = bl;
  __syncthreads();
  if (!pending) return;
  finish_step(c, s, h, d, bl, h.R, cnt);
}

__global__ void __launch_bounds__(kPartThreads) k_finish(const __grid_constant__ DCtx c) {
  __shared__ SplitDecision dec;
  const DSlot& s = c.slots[blockIdx.z];
  deferred_finish(c, s, &dec);
  __syncthreads();
  if (threadIdx.x == 0) s.st->pending = 0;
}

// Threshold scans, then the partition, of one step (one cooperative launch):
// CTA b scans items b, b + grid, ... ((feature, side) pairs), publishes them
// on the slot's scan counter and waits until every CTA of the slot has done
// so. The wait is bounded: past kSpinLimit polls the CTA records
// kStatusTimeout (the host reports it) and carries on.
template <bool kInt>
__global__ void __launch_bounds__(kPartThreads) k_scan_partition(const __grid_constant__ DCtx c) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const DSlot& s = c.slots[blockIdx.z];
  DSlotState* st = s.st;
  __shared__ PartShared ps;
  const StepHead h = load_step_head(st);
  if (threadIdx.x == 0) ps.tile = atomicAdd(&st->part_ticket, 1);
  if (h.done) {  // no CTA of this launch sets done before every CTA has passed the wait below
    if (blockIdx.x == 0 && threadIdx.x == 0) st->pending = 0;
    return;
  }
  const int nitems = 2 * c.num_features;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    scan_item<kInt>(c, s, it >> 1, it & 1, *reinterpret_cast<ScanSmem*>(smem_raw));
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&st->scan_done, 1);
    int spins = 0;
    while (*reinterpret_cast<volatile int32_t*>(&st->scan_done) < (int)gridDim.x) {
      if (++spins > kSpinLimit) {
        st->status = kStatusTimeout;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
  partition_body(c, s, ps, h);
}
template __global__ void k_scan_partition<false>(const __grid_constant__ DCtx);
template __global__ void k_scan_partition<true>(const __grid_constant__ DCtx);


// Column-major copy of the bin matrix (the partition reads one feature of the
// rows of a leaf, which are ascending, so neighbouring rows share sectors).
__global__ void __launch_bounds__(256) k_transpose_bins(const uint8_t* bins, int64_t n, int32_t stride, int32_t nf,
                                                        uint8_t* colbins) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    for (int32_t f = 0; f < nf; ++f) colbins[(size_t)f * n + r] = bins[(size_t)r * stride + f];
}

// =====================================================================================
// leaf renewal from FP64 gradient sums (learner/mod.rs:736-747) and the
// score updates (partition.rs:306-319; tree.rs:605-711 binned routing)
// =====================================================================================
// Grid (G, num_leaves, slots): block (x, leaf) sums a chunk of the leaf's rows.
// Leaf of each row position: every CTA builds a table of the tree's
// non-empty leaves in position order (a leaf is a contiguous range of the
// partition) in shared memory, then walks positions grid-stride and finds
// each position's leaf by binary search. Work is spread evenly over the
// rows whatever the leaf sizes. Dynamic shared memory: 16 bytes per leaf.
struct LeafTable {
  int32_t* begin;  // sorted range starts
  int32_t* leaf;
  int32_t* side;
  int32_t n;       // non-empty leaves
  int32_t total;   // positions covered
};

__device__ LeafTable build_leaf_table(const DSlot& s, int32_t nl, int32_t* smem) {
  int32_t* beg = smem;
  int32_t* cnt = smem + nl;
  LeafTable t;
  t.begin = smem + 2 * nl;
  t.leaf = smem + 3 * nl;
  t.side = cnt;  // reused after ranking: side of the leaf at each rank
  __shared__ int32_t s_n, s_total;
  for (int32_t l = threadIdx.x; l < nl; l += blockDim.x) {
    beg[l] = s.leaf_begin[l];
    cnt[l] = s.leaf_count[l];
  }
  if (threadIdx.x == 0) {
    s_n = 0;
    s_total = 0;
  }
  __syncthreads();
  for (int32_t l = threadIdx.x; l < nl; l += blockDim.x) {
    if (cnt[l] <= 0) continue;
    const int32_t b = beg[l];
    int32_t r = 0;  // non-empty leaves start at distinct positions
    for (int32_t m = 0; m < nl; ++m) r += (cnt[m] > 0 && beg[m] < b) ? 1 : 0;
    t.begin[r] = b;
    t.leaf[r] = l;
    atomicAdd(&s_n, 1);
    atomicMax(&s_total, b + cnt[l]);
  }
  __syncthreads();
  for (int32_t r = threadIdx.x; r < s_n; r += blockDim.x) t.side[r] = s.leaf_side[t.leaf[r]];
  __syncthreads();
  t.n = s_n;
  t.total = s_total;
  return t;
}

__device__ __forceinline__ int32_t leaf_rank_of(const LeafTable& t, int32_t p) {
  int32_t lo = 0, hi = t.n - 1;
  while (lo < hi) {
    const int32_t mid = (lo + hi + 1) >> 1;
    if (t.begin[mid] <= p) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Each warp takes a contiguous share of the positions [0, t.total), in steps
// of 32 (lane = offset), and follows the leaf boundaries as it goes: its
// first leaf is found once by binary search, later ones by stepping the
// rank. visit(q, rank, same) is called for every position q of the share;
// same is true when q lies in the warp's current leaf, which the warp
// leaves through end_leaf(rank) (warp-uniform) before moving on.
template <class Visit, class EndLeaf>
__device__ __forceinline__ void walk_leaf_positions(const LeafTable& t, Visit visit, EndLeaf end_leaf) {
  const int lane = threadIdx.x & 31;
  const int32_t nwarps = (int32_t)(gridDim.x * (blockDim.x >> 5));
  const int32_t gw = (int32_t)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
  const int32_t per = ((t.total + nwarps - 1) / nwarps + 31) & ~31;
  const int32_t p0 = min(t.total, gw * per), p1 = min(t.total, p0 + per);
  if (p0 >= p1 || t.n == 0) return;
  int32_t r = leaf_rank_of(t, p0);
  int32_t end = r + 1 < t.n ? t.begin[r + 1] : t.total;  // first position past leaf r
  for (int32_t p = p0; p < p1; p += 32) {
    const int32_t q = p + lane;
    if (p + 32 <= end && p + 32 <= p1) {  // the whole step lies in leaf r
      visit(q, r, true);
      continue;
    }
    if (q < p1) {
      int32_t rq = r;
      while (rq + 1 < t.n && t.begin[rq + 1] <= q) ++rq;
      visit(q, rq, rq == r);
    }
    if (p + 32 < p1) {  // leaf r ended inside this step; the share goes on
      end_leaf(r);
      while (r + 1 < t.n && t.begin[r + 1] <= p + 32) ++r;
      end = r + 1 < t.n ? t.begin[r + 1] : t.total;
    }
  }
  end_leaf(r);
}

// FP64 (g, h) sums of each leaf's rows for the leaf renewal
// (learner/mod.rs:736-747), in a fixed order so that a tree's leaf values
// are the same on every run. Grid (G, 1, slots), 256 threads. Warp w takes
// the positions [w * per, (w + 1) * per) (per = the positions over the
// warps, rounded up to 32) and visits the leaves its share meets in
// position order. For each it sums the share's part of the leaf lane-wise
// (position q to lane q mod 32, in order) and across lanes by a fixed
// butterfly, and stores the pair at segment w + rank, where rank is the
// leaf's place in position order. Along the positions both w and rank only
// grow and one of them grows at every new segment, so no two segments share
// an index. Block 0 also records each leaf's rank and the share size for
// k_leaf_renew, which adds a leaf's segments in warp order.
// partial: [slots][G * 8 + num_leaves][2]; rank: [slots][num_leaves + 1].
__global__ void __launch_bounds__(256) k_leaf_sums(const __grid_constant__ DCtx c, double* partial, int32_t* rank) {
  extern __shared__ int32_t lt_smem[];
  const DSlot& s = c.slots[blockIdx.z];
  const int32_t nl = s.st->num_leaves_cur;
  const LeafTable t = build_leaf_table(s, nl, lt_smem);
  const int lane = threadIdx.x & 31;
  const int32_t nwarps = (int32_t)(gridDim.x * (blockDim.x >> 5));
  const int32_t gw = (int32_t)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
  const int32_t per = ((t.total + nwarps - 1) / nwarps + 31) & ~31;
  int32_t* rk = rank + (size_t)blockIdx.z * (c.p.num_leaves + 1);
  if (blockIdx.x == 0) {
    for (int32_t r = threadIdx.x; r < t.n; r += blockDim.x) rk[t.leaf[r]] = r;
    if (threadIdx.x == 0) rk[c.p.num_leaves] = per;
  }
  const int32_t p0 = min(t.total, gw * per), p1 = min(t.total, p0 + per);
  if (p0 >= p1 || t.n == 0) return;
  double* base = partial + (size_t)blockIdx.z * (nwarps + c.p.num_leaves) * 2;
  int32_t r = leaf_rank_of(t, p0);
  for (int32_t q0 = p0; q0 < p1; ++r) {
    const int32_t end = min(p1, r + 1 < t.n ? t.begin[r + 1] : t.total);
    const uint32_t* idx = s.idx[t.side[r]];
    double g = 0.0, h = 0.0;
    for (int32_t q = q0 + lane; q < end; q += 32) {
      const float2 v = s.gh[idx[q]];
      g += (double)v.x;
      h += (double)v.y;
    }
    g = warp_sum_d(g);
    h = warp_sum_d(h);
    if (lane == 0) {
      base[2 * (gw + r)] = g;
      base[2 * (gw + r) + 1] = h;
    }
    q0 = end;
  }
}

// Leaf outputs from the segment sums of k_leaf_sums (grid (1, 1, slots)):
// a leaf at rank r covering positions [b, e) adds segments w + r for
// w = b / per ... (e - 1) / per, in that order.
__global__ void k_leaf_renew(const __grid_constant__ DCtx c, const double* partial, const int32_t* rank,
                             int32_t nwarps, double* totals) {
  const DSlot& s = c.slots[blockIdx.z];
  DSlotState* st = s.st;
  const int32_t* rk = rank + (size_t)blockIdx.z * (c.p.num_leaves + 1);
  const int32_t per = rk[c.p.num_leaves];
  const double* base = partial + (size_t)blockIdx.z * (nwarps + c.p.num_leaves) * 2;
  for (int32_t leaf = threadIdx.x; leaf < st->num_leaves_cur; leaf += blockDim.x) {
    const int32_t cnt = s.leaf_count[leaf];
    double g = 0.0, h = 0.0;
    if (cnt > 0) {
      const int32_t b = s.leaf_begin[leaf], r = rk[leaf];
      for (int32_t w = b / per; w <= (b + cnt - 1) / per; ++w) {
        g += base[2 * (w + r)];
        h += base[2 * (w + r) + 1];
      }
    }
    if (totals) {  // data-parallel: this rank's sums, refit after the reduction over ranks
      totals[((size_t)blockIdx.z * c.p.num_leaves + leaf) * 2] = g;
      totals[((size_t)blockIdx.z * c.p.num_leaves + leaf) * 2 + 1] = h;
    } else {
      s.tree.leaf_value[leaf] = maybe_round_to_zero(refit_leaf_output(g, h, c.p, s.leaf_gcount[leaf]));
    }
  }
}

// Data-parallel growth: leaf outputs from the per-leaf sums over every rank.
__global__ void k_dp_leaf_apply(const __grid_constant__ DCtx c, const double* totals) {
  const DSlot& s = c.slots[blockIdx.z];
  for (int32_t leaf = threadIdx.x; leaf < s.st->num_leaves_cur; leaf += blockDim.x) {
    const double* o = totals + ((size_t)blockIdx.z * c.p.num_leaves + leaf) * 2;
    s.tree.leaf_value[leaf] = maybe_round_to_zero(refit_leaf_output(o[0], o[1], c.p, s.leaf_gcount[leaf]));
  }
}

// score[row] += leaf_values[leaf of row] over the in-bag rows
// (partition.rs:178-191). Grid (G, 1, slots), 256 threads.
__global__ void __launch_bounds__(256) k_add_leaf_outputs(const __grid_constant__ DCtx c, const double* leaf_values, int32_t lv_stride,
                                                          double* score, int64_t score_stride) {
  extern __shared__ int32_t lt_smem[];
  const DSlot& s = c.slots[blockIdx.z];
  const int32_t nl = s.st->num_leaves_cur;
  const LeafTable t = build_leaf_table(s, nl, lt_smem);
  const double* lv = leaf_values + (size_t)blockIdx.z * lv_stride;
  double* sc = score + (size_t)blockIdx.z * score_stride;
  walk_leaf_positions(
      t, [&](int32_t q, int32_t rank, bool) { sc[s.idx[t.side[rank]][q]] += lv[t.leaf[rank]]; }, [](int32_t) {});
}

// The leaf of every in-bag row, in row order, for the score update from host
// buffers (rows out of the bag keep -1). Grid (G, 1, 1), 256 threads, the
// slot in c.slots[0].
__global__ void __launch_bounds__(256) k_leaf_of_row(const __grid_constant__ DCtx c, int32_t* leaf_of_row) {
  extern __shared__ int32_t lt_smem[];
  const DSlot& s = c.slots[0];
  const LeafTable t = build_leaf_table(s, s.st->num_leaves_cur, lt_smem);
  walk_leaf_positions(
      t, [&](int32_t q, int32_t rank, bool) { leaf_of_row[s.idx[t.side[rank]][q]] = t.leaf[rank]; },
      [](int32_t) {});
}

// score[r] += leaf_values[leaf_of_row[r]] for rows [0, n) of a chunk
// (partition.rs:178-191 in row order).
__global__ void __launch_bounds__(256) k_add_by_row(const int32_t* leaf_of_row, const double* leaf_values,
                                                    double* score, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t l = leaf_of_row[i];
    if (l >= 0) score[i] += leaf_values[l];
  }
}

// Binned tree walk (tree.rs:588-633) for rows `rows` (or 0..n): score += leaf value.
__global__ void __launch_bounds__(256) k_add_tree_binned(const __grid_constant__ DCtx c, const uint8_t* bins, int32_t stride,
                                                         const uint32_t* rows, int64_t n, const double* leaf_values,
                                                         int32_t lv_stride, double* score, int64_t score_stride) {
  const DSlot& s = c.slots[blockIdx.z];
  const DTree& t = s.tree;
  int32_t nl = s.st->num_leaves_cur;
  const double* lv = leaf_values + (size_t)blockIdx.z * lv_stride;
  double* sc = score + (size_t)blockIdx.z * score_stride;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = rows ? (int64_t)rows[i] : i;
    int32_t node = 0;
    if (nl > 1) {
      while (node >= 0) {
        int32_t inner = t.split_feature_inner[node];
        const DFeature& m = c.feats[inner];
        uint32_t b = decode_bin(bins[(size_t)r * stride + inner], m);
        int8_t dt = t.decision_type[node];
        if (dt & 1) {
          const uint32_t* bits = t.cat_bits + node * kCatWords;
          bool left = b < (uint32_t)kMaxBins && ((bits[b >> 5] >> (b & 31)) & 1u);
          node = left ? t.left_child[node] : t.right_child[node];
          continue;
        }
        int32_t mt = (dt >> 2) & 3;
        bool is_default = (mt == 1 && b == (uint32_t)m.default_bin) || (mt == 2 && b == (uint32_t)(m.num_bin - 1));
        bool left = is_default ? (dt & 2) != 0 : b <= t.threshold_in_bin[node];
        node = left ? t.left_child[node] : t.right_child[node];
      }
      node = ~node;
    }
    sc[r] += lv[node];
  }
}

// =====================================================================================
// Persistent tree growth: one cooperative launch grows the whole tree (every
// slot). Per split step the CTAs run the phases of the per-step kernels,
// separated by grid barriers:
//   H  histogram of each slot's smaller leaf (the slot's CTA group shares the rows)
//   S  threshold scans, items (slot, feature, leaf side) over all CTAs
//   P  split decision, LUT and row partition (each slot's CTA group)
//   F  the step's bookkeeping by the first CTA of each group
// The cooperative launch keeps every CTA resident, so a barrier never waits
// on a CTA that has not started; every wait is still bounded and reports a
// timeout instead of hanging.
// =====================================================================================

// Grid barrier over `nblocks` CTAs (sense reversal on a generation counter).
// Returns false when a wait timed out here or anywhere in the grid.
__device__ bool grid_barrier(GrowSync* gs, unsigned int nblocks) {
  __shared__ int s_ok;
  __threadfence();  // this thread's writes before the barrier are visible to the grid
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = &gs->gen;
    const unsigned int g = *vgen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&gs->count, 1u) == nblocks - 1u) {
      gs->count = 0;  // no CTA touches the count before the generation moves
      __threadfence();
      atomicAdd(&gs->gen, 1u);
    } else {
      int spins = 0;
      while (*vgen == g) {
        if (++spins > kSpinLimit) {
          atomicExch(&gs->status, kStatusTimeout);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (*reinterpret_cast<volatile int*>(&gs->status) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  __threadfence();  // later reads observe the other CTAs' writes
  return s_ok != 0;
}

__device__ __forceinline__ int64_t global_ns() {
  int64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <int kMode, int kNG>
__global__ void __launch_bounds__(kGrowThreads, 1)
    k_grow(const __grid_constant__ DCtx c, DTileTable tt, int32_t sub_rows, int32_t ntiles, GrowSync* gs,
           int32_t num_steps, long long* phase_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PartShared ps;
  __shared__ int s_any;
  constexpr bool kInt = kMode == 2;
  const unsigned int G = gridDim.x;
  const int K = c.num_slots;
  const int per = (int)G / K;  // CTAs per slot group (the host makes G a multiple of K)
  const int slot = (int)blockIdx.x / per;
  const int rank = (int)blockIdx.x - slot * per;
  const DSlot& s = c.slots[slot];
  DSlotState* st = s.st;
  const int tid = threadIdx.x;
  const int32_t nf = c.num_features;
  const bool timer = blockIdx.x == 0 && tid == 0 && phase_ns != nullptr;
  int64_t t_prev = timer ? global_ns() : 0;
  auto mark = [&](int phase) {
    if (timer) {
      const int64_t t = global_ns();
      phase_ns[phase] += t - t_prev;
      t_prev = t;
    }
  };
  for (int step = 0; step < num_steps; ++step) {
    // every CTA reads the same flags after a barrier: the loop ends together
    if (tid == 0) {
      int any = 0;
      for (int k = 0; k < K; ++k) any |= *reinterpret_cast<volatile int32_t*>(&c.slots[k].st->done) == 0;
      s_any = any;
    }
    __syncthreads();
    if (!s_any) break;
    // H: histogram of the slot's smaller leaf
    {
      LeafRows lr;
      int64_t r0, r1;
      if (hist_setup<1>(c, s, rank, per, lr, r0, r1)) {
        if (rank == 0 && tid == 0) st->hist_rows += lr.count;
        for (int t = 0; t < ntiles; ++t) hist_body<kMode, kNG, 1>(c, s, tt, t, lr, r0, r1, sub_rows, smem_raw);
      }
    }
    if (!grid_barrier(gs, G)) return;
    mark(0);
    // S: threshold scans
    {
      ScanSmem& sm = *reinterpret_cast<ScanSmem*>(smem_raw);
      const int nitems = K * nf * 2;
      for (int it = blockIdx.x; it < nitems; it += (int)G) {
        const int k = it / (2 * nf), rem = it - k * 2 * nf;
        const DSlot& sk = c.slots[k];
        if (*reinterpret_cast<volatile int32_t*>(&sk.st->done)) continue;
        scan_item<kInt>(c, sk, rem >> 1, rem & 1, sm);
        __syncthreads();
      }
      if (blockIdx.x == 0 && tid < K) c.slots[tid].st->part_ticket = 0;
    }
    if (!grid_barrier(gs, G)) return;
    mark(1);
    // P: the split decision and the row partition of the slot
    SplitLeaf sl;
    sl.L = -1;
    int32_t R = 0;
    StepHead h = {};
    if (!*reinterpret_cast<volatile int32_t*>(&st->done)) {
      h = load_step_head(st);
      R = h.R;
      sl = partition_prologue(c, s, h, ps);
      if (sl.L < 0) {
        if (rank == 0 && tid == 0) st->done = 1;
      } else {
        zero_hist_buffer(c, s, R, rank, per);
        partition_rows<kPartTileRows / kGrowThreads>(c, s, ps, sl, h.epoch, false);
      }
    }
    if (!grid_barrier(gs, G)) return;
    mark(2);
    // F: bookkeeping of the step
    if (sl.L >= 0 && rank == 0)
      finish_step(c, s, h, ps.dec, sl.L, R, sl.cnt);
    if (!grid_barrier(gs, G)) return;
    mark(3);
  }
}

#define LGBM_B200_GROW_INST(M, G)                                                                            \
  template __global__ void k_grow<M, G>(const __grid_constant__ DCtx, DTileTable, int32_t, int32_t, GrowSync*, \
                                        int32_t, long long*);
LGBM_B200_GROW_INST(0, 1)
LGBM_B200_GROW_INST(1, 1)
LGBM_B200_GROW_INST(2, 1)
LGBM_B200_GROW_INST(2, 2)
LGBM_B200_GROW_INST(2, 3)
LGBM_B200_GROW_INST(2, 4)
#undef LGBM_B200_GROW_INST

const void* grow_kernel(int mode, int ng) {
  if (mode == 0) return reinterpret_cast<const void*>(&k_grow<0, 1>);
  if (mode == 1) return reinterpret_cast<const void*>(&k_grow<1, 1>);
  switch (ng) {
    case 1: return reinterpret_cast<const void*>(&k_grow<2, 1>);
    case 2: return reinterpret_cast<const void*>(&k_grow<2, 2>);
    case 3: return reinterpret_cast<const void*>(&k_grow<2, 3>);
    default: return reinterpret_cast<const void*>(&k_grow<2, 4>);
  }
}

size_t grow_smem_bytes(int mode, int ng) { return std::max(hist_smem_bytes(mode, ng), sizeof(ScanSmem)); }

cudaError_t launch_grow(int mode, int ng, int grid, size_t smem, cudaStream_t st, const DCtx& c, const DTileTable& tt,
                        int32_t sub_rows, int32_t ntiles, GrowSync* gs, int32_t num_steps, long long* phase_ns) {
  void* args[] = {const_cast<DCtx*>(&c), const_cast<DTileTable*>(&tt), &sub_rows, &ntiles, &gs, &num_steps, &phase_ns};
  return cudaLaunchCooperativeKernel(grow_kernel(mode, ng), dim3(grid), dim3(kGrowThreads), args, smem, st);
}

}  // namespace lgbm_b200
