// Objective gradients, quantized gradients and bagging on the device.
//   k_grad_binary   objective/binary.rs:101-127
//   k_grad_l2       objective/regression.rs:209-224 (L2, no weights)
//   k_grad_softmax  objective/multiclass.rs:16-30, :126-154
//   k_quant_*       learner/quant.rs:411-448 (DiscretizeGradients)
//   k_bagging       sample_strategy.rs:280-320 (one LCG per 1024-row block)
// Each kernel can write the learner's interleaved (g, h) buffer directly.
#include "kernels.h"

namespace lgbm_b200 {

__global__ void __launch_bounds__(256) k_grad_binary(const float* label, const double* score, int64_t n,
                                                     double sigmoid, float2* gh_out, float* g, float* h) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double lab = label[i] > 0.0f ? 1.0 : -1.0;
    double response = -lab * sigmoid / ((double)1.0f + exp(lab * sigmoid * score[i]));
    double ar = fabs(response);
    float gv = (float)(response * 1.0);
    float hv = (float)(ar * (sigmoid - ar) * 1.0);
    if (gh_out) gh_out[i] = make_float2(gv, hv);
    if (g) {
      g[i] = gv;
      h[i] = hv;
    }
  }
}

__global__ void __launch_bounds__(256) k_grad_l2(const float* label, const double* score, int64_t n, float2* gh_out,
                                                 float* g, float* h) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float gv = (float)(score[i] - (double)label[i]);
    if (gh_out) gh_out[i] = make_float2(gv, 1.0f);
    if (g) {
      g[i] = gv;
      h[i] = 1.0f;
    }
  }
}

// One row per thread; scores / outputs are class-major [k x n].
__global__ void __launch_bounds__(256) k_grad_softmax(const float* label, const double* score, int64_t n, int32_t k,
                                                      float2* gh_out, int64_t gh_stride, float* g, float* h) {
  const double factor = (double)k / (double)((float)k - 1.0f);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double wmax = score[i];
    for (int c = 1; c < k; ++c) {
      double v = score[(int64_t)c * n + i];
      wmax = v < wmax ? wmax : v;
    }
    double wsum = 0.0;
    for (int c = 0; c < k; ++c) wsum += exp(score[(int64_t)c * n + i] - wmax);
    int32_t li = (int32_t)label[i];
    for (int c = 0; c < k; ++c) {
      double p = exp(score[(int64_t)c * n + i] - wmax) / wsum;
      double gg = li == c ? p - (double)1.0f : p;
      double hh = factor * p * ((double)1.0f - p);
      if (gh_out) gh_out[(int64_t)c * gh_stride + i] = make_float2((float)gg, (float)hh);
      if (g) {
        g[(int64_t)c * n + i] = (float)gg;
        h[(int64_t)c * n + i] = (float)hh;
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_interleave(const float* g, const float* h, int64_t n, float2* gh) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    gh[i] = make_float2(g[i], h[i]);
}

// max |g| and |h| (order-independent, exact); the last block derives the
// scales exactly as quant.rs:429-430 does.
// derive 0 (data-parallel): the last block leaves the maxima in maxbits for
// the reduction over ranks; k_quant_scales derives the scales after it.
__global__ void __launch_bounds__(256) k_quant_absmax(const float2* gh, int64_t n, unsigned long long* maxbits,
                                                      int32_t* counter, DSlotState* st, int32_t bins,
                                                      int32_t const_hess, int32_t num_blocks, int32_t derive) {
  double mg = 0.0, mh = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float2 v = gh[i];
    mg = fmax(mg, fabs((double)v.x));
    mh = fmax(mh, fabs((double)v.y));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mg = fmax(mg, __shfl_xor_sync(0xffffffffu, mg, o));
    mh = fmax(mh, __shfl_xor_sync(0xffffffffu, mh, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&maxbits[0], (unsigned long long)__double_as_longlong(mg));
    atomicMax(&maxbits[1], (unsigned long long)__double_as_longlong(mh));
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1) == num_blocks - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  if (!derive) {
    *counter = 0;
    return;
  }
  double max_g = __longlong_as_double((long long)atomicAdd(&maxbits[0], 0ull));
  double max_h = __longlong_as_double((long long)atomicAdd(&maxbits[1], 0ull));
  st->grad_scale = max_g / (double)(bins / 2);
  st->hess_scale = const_hess ? max_h : max_h / (double)bins;
  maxbits[0] = 0;
  maxbits[1] = 0;
  *counter = 0;
}

// The scales from maxima taken over every rank, as the last
// block of k_quant_absmax derives them (quant.rs:429-430). One thread.
__global__ void k_quant_scales(unsigned long long* maxbits, DSlotState* st, int32_t bins, int32_t const_hess) {
  const double max_g = __longlong_as_double((long long)maxbits[0]);
  const double max_h = __longlong_as_double((long long)maxbits[1]);
  st->grad_scale = max_g / (double)(bins / 2);
  st->hess_scale = const_hess ? max_h : max_h / (double)bins;
  maxbits[0] = 0;
  maxbits[1] = 0;
}

// quant.rs:355-359 static_cast<int8_t>(double) as x86-64 compiles it.
__device__ __forceinline__ int32_t to_i8(double x) {
  int32_t t = (isnan(x) || !(x >= -2147483648.0 && x < 2147483648.0)) ? INT32_MIN : (int32_t)x;
  return (int32_t)(int8_t)t;
}

// quant.rs:434-447; packed[i] = (g << 16) + (h as u8). The tree's start
// offset into the rounding tables is read from device memory, so a captured
// launch takes each tree's new offset.
__global__ void __launch_bounds__(256) k_quant_apply(const float2* gh, int64_t n, const double* grv,
                                                     const double* hrv, const int64_t* start_dev,
                                                     const DSlotState* st, int32_t const_hess, int32_t stochastic,
                                                     int32_t* packed, int64_t row_offset, int64_t table_n,
                                                     uint8_t* row_q, int32_t row_stride) {
  const int64_t start = *start_dev;
  const double inv_g = 1.0 / st->grad_scale;
  const double inv_h = 1.0 / st->hess_scale;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float2 v = gh[i];
    double g = (double)v.x;
    double rg = 0.5, rh = 0.5;
    if (stochastic) {
      // (global row + start) mod the table length, with both below it
      // (data-parallel: row_offset is this rank's first global row)
      int64_t pos = row_offset + i + start;
      if (pos >= table_n) pos -= table_n;
      rg = grv[pos];
      rh = hrv[pos];
    }
    int32_t gq = g >= 0.0 ? to_i8(g * inv_g + rg) : to_i8(g * inv_g - rg);
    int32_t hq = const_hess ? 1 : to_i8((double)v.y * inv_h + rh);
    const int32_t pq = gq * 65536 + (int32_t)(uint8_t)hq;
    packed[i] = pq;
    // the copy in the row's padding, read with the row's bins
    if (row_q) *reinterpret_cast<int32_t*>(row_q + i * row_stride) = pq;
  }
}

// sample_strategy.rs:280-320: rows of block b draw from the LCG `state[b]`
// (Random(bagging_seed + b)) in row order; r < fraction keeps the row.
// One thread per 1024-row block; block_in[b] receives the block's in-bag count.
__global__ void k_bagging(uint32_t* rng_state, int64_t n, double fraction, uint8_t* in_bag, int32_t* block_in) {
  int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t r0 = b * 1024;
  if (r0 >= n) return;
  int64_t r1 = min(n, r0 + 1024);
  uint32_t x = rng_state[b];
  int32_t cnt = 0;
  for (int64_t r = r0; r < r1; ++r) {
    x = x * 214013u + 2531011u;
    float f = (float)((x >> 16) & 0x7FFF) / 32768.0f;
    const bool keep = (double)f < fraction;
    in_bag[r] = keep ? 1 : 0;
    cnt += keep ? 1 : 0;
  }
  rng_state[b] = x;
  block_in[b] = cnt;
}

// Exclusive prefix of the blocks' in-bag counts (one CTA of 1024 threads,
// each over a contiguous run of blocks); counts[0] / counts[1] receive the
// in-bag and out-of-bag totals.
__global__ void __launch_bounds__(1024) k_bag_scan(const int32_t* block_in, int32_t nb, int64_t n, int32_t* block_base,
                                                   int32_t* counts) {
  __shared__ int32_t warp_sum[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int32_t per = (nb + (int32_t)blockDim.x - 1) / (int32_t)blockDim.x;
  const int32_t b0 = min(nb, tid * per), b1 = min(nb, b0 + per);
  int32_t local = 0;
  for (int32_t b = b0; b < b1; ++b) local += block_in[b];
  int32_t incl = local;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  int32_t base = 0, total = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    if (w < warp) base += warp_sum[w];
    total += warp_sum[w];
  }
  int32_t run = base + incl - local;
  for (int32_t b = b0; b < b1; ++b) {
    block_base[b] = run;
    run += block_in[b];
  }
  if (tid == 0) {
    counts[0] = total;
    counts[1] = (int32_t)(n - total);
  }
}

// Ascending in-bag rows and the out-of-bag rows: CTA b places the rows of
// 1024-row block b after the block_base[b] in-bag (b * 1024 - block_base[b]
// out-of-bag) rows of the blocks before it.
__global__ void __launch_bounds__(1024) k_bag_scatter(const uint8_t* in_bag, int64_t n, const int32_t* block_base,
                                                      uint32_t* bag, uint32_t* oob) {
  __shared__ int32_t warp_in[32], warp_out[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t r = (int64_t)blockIdx.x * 1024 + tid;
  const bool valid = r < n;
  const bool in = valid && in_bag[r];
  const unsigned bi = __ballot_sync(0xffffffffu, in);
  const unsigned bo = __ballot_sync(0xffffffffu, valid && !in);
  if (lane == 0) {
    warp_in[warp] = __popc(bi);
    warp_out[warp] = __popc(bo);
  }
  __syncthreads();
  int32_t pi = 0, po = 0;
  for (int w = 0; w < warp; ++w) {
    pi += warp_in[w];
    po += warp_out[w];
  }
  const int32_t base_in = block_base[blockIdx.x];
  const int32_t base_out = (int32_t)((int64_t)blockIdx.x * 1024 - base_in);
  const unsigned below = (1u << lane) - 1u;
  if (in) bag[base_in + pi + __popc(bi & below)] = (uint32_t)r;
  else if (valid) oob[base_out + po + __popc(bo & below)] = (uint32_t)r;
}

__global__ void __launch_bounds__(256) k_add_const(double* score, int64_t n, double v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    score[i] += v;
}

}  // namespace lgbm_b200
