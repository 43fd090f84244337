// Front-to-back alpha compositing, forward and backward (reference src/rasterize.rs).
//
// One 256-thread block per 16x16 tile, one pixel per thread. Warps own 8x4 pixel
// sub-blocks so that an entry whose pixel rectangle misses a sub-block is skipped by the
// whole warp with one uniform branch. The tile's sorted entries are staged through shared
// memory in chunks of 256 (each thread gathers one entry's 48-byte record). Every
// per-pixel decision (sigma range, alpha >= 1/255, the 0.99 clamp, T < 1e-4) is taken on
// values computed exactly as the reference computes them: unfused arithmetic and a
// correctly rounded exp.
#include "common.cuh"
#include "kernels.cuh"

namespace splat {

constexpr int kRasterThreads = 256;
constexpr int kChunk = 256;

struct PixelGeom {
  uint32_t px_i, py_j;   // absolute pixel
  uint32_t bx0, by0;     // warp sub-block origin
  bool inside;
};

__device__ __forceinline__ PixelGeom pixel_geom(uint32_t tile, uint32_t tiles_x, uint32_t width, uint32_t height) {
  const uint32_t tx = tile % tiles_x, ty = tile / tiles_x;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  PixelGeom p;
  p.bx0 = tx * kTile + (warp & 1u) * 8u;
  p.by0 = ty * kTile + (warp >> 1) * 4u;
  p.px_i = p.bx0 + (lane & 7u);
  p.py_j = p.by0 + (lane >> 3);
  p.inside = p.px_i < width && p.py_j < height;
  return p;
}

// Entry rectangle against the warp's 8x4 sub-block (warp-uniform).
__device__ __forceinline__ bool rect_hits_block(uint32_t rx, uint32_t ry, const PixelGeom& p) {
  const uint32_t x0 = rx & 0xffffu, x1 = rx >> 16, y0 = ry & 0xffffu, y1 = ry >> 16;
  return !(x1 <= p.bx0 || x0 >= p.bx0 + 8u || y1 <= p.by0 || y0 >= p.by0 + 4u);
}

__device__ __forceinline__ bool pixel_in_rect(uint32_t rx, uint32_t ry, const PixelGeom& p) {
  const uint32_t x0 = rx & 0xffffu, x1 = rx >> 16, y0 = ry & 0xffffu, y1 = ry >> 16;
  return p.px_i >= x0 && p.px_i < x1 && p.py_j >= y0 && p.py_j < y1;
}

// evaluate (rasterize.rs:231-244). Returns false when skipped.
__device__ __forceinline__ bool evaluate(float px, float py, float mx, float my, float A, float B, float C,
                                         float opacity, float sigma_max, float* gauss_out, float* alpha_out) {
  const float dx = px - mx;
  const float dy = py - my;
  const float sigma = 0.5f * (A * dx * dx + C * dy * dy) + B * dx * dy;
  if (sigma < 0.0f || sigma > sigma_max) return false;
  const float gauss = crm::expf_cr(-sigma);
  const float og = opacity * gauss;
  if (og < SPLAT_ALPHA_MIN) return false;
  *gauss_out = gauss;
  *alpha_out = fminf(og, SPLAT_ALPHA_MAX);
  return true;
}

// evaluate for the backward pass. The decisions must be the forward's, which were taken on
// the correctly rounded exp; the value may carry a few ulps. A fast exp (MUFU ex2) decides
// whenever the product opacity * gauss lies outside a relative band of kExpBand around the
// two thresholds (1/255 and 0.99); inside the band the correctly rounded exp is evaluated
// and decides. kExpBand bounds the fast exp's relative error on the argument range
// [-ln(255), 0] with a wide margin (the bound is checked on the device by
// splat_diag_fast_exp_error). *unclamped is the reference's `opacity * gauss < 0.99`.
constexpr float kExpBand = 3e-5f;

__device__ __forceinline__ bool evaluate_bwd(float px, float py, float mx, float my, float A, float B, float C,
                                             float opacity, float sigma_max, float* gauss_out, float* alpha_out,
                                             bool* unclamped) {
  const float dx = px - mx;
  const float dy = py - my;
  const float sigma = 0.5f * (A * dx * dx + C * dy * dy) + B * dx * dy;
  if (sigma < 0.0f || sigma > sigma_max) return false;
  float gauss = __expf(-sigma);
  float og = opacity * gauss;
  const bool near_min = og < SPLAT_ALPHA_MIN * (1.0f + kExpBand) && og > SPLAT_ALPHA_MIN * (1.0f - kExpBand);
  const bool near_max = og < SPLAT_ALPHA_MAX * (1.0f + kExpBand) && og > SPLAT_ALPHA_MAX * (1.0f - kExpBand);
  if (near_min || near_max) {
    gauss = crm::expf_cr(-sigma);
    og = opacity * gauss;
  }
  if (og < SPLAT_ALPHA_MIN) return false;
  *gauss_out = gauss;
  *alpha_out = fminf(og, SPLAT_ALPHA_MAX);
  *unclamped = og < SPLAT_ALPHA_MAX;
  return true;
}

// Largest relative error of the fast exp against the correctly rounded one over every
// float in [lo, hi] (a diagnostic of the bound kExpBand relies on).
__global__ void diag_fast_exp_kernel(uint32_t lo_bits, uint32_t count, int negative, unsigned int* max_rel_bits) {
  float worst = 0.0f;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const uint32_t b = lo_bits + k;
    const float x = negative ? -__uint_as_float(b) : __uint_as_float(b);
    const float e = crm::expf_cr(x);
    const float f = __expf(x);
    if (e > 0.0f) worst = fmaxf(worst, fabsf(f - e) / e);
  }
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if ((threadIdx.x & 31) == 0) atomicMax(max_rel_bits, __float_as_uint(worst));
}

Status launch_diag_fast_exp(Ctx* c, float magnitude_lo, float magnitude_hi, int negative, float* out_host) {
  unsigned int* d = nullptr;
  SPLAT_TRY(arena_reserve(c, 4, (void**)&d));
  SPLAT_CUDA(cudaMemsetAsync(d, 0, 4, c->stream));
  const uint32_t lo = fbits(magnitude_lo), hi = fbits(magnitude_hi);
  diag_fast_exp_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(lo, hi - lo + 1, negative, d);
  c->launches.count++;
  SPLAT_LAUNCHED("diag_fast_exp_kernel");
  unsigned int h = 0;
  SPLAT_CUDA(cudaMemcpyAsync(&h, d, 4, cudaMemcpyDeviceToHost, c->stream));
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  *out_host = bitsf(h);
  return Status::ok();
}

// forward_tile (rasterize.rs:249-302) for one tile per block.
__global__ void __launch_bounds__(kRasterThreads) raster_fwd_kernel(
    const float4* __restrict__ rec, const uint32_t* __restrict__ gauss, const uint2* __restrict__ ranges,
    uint32_t width, uint32_t height, uint32_t tiles_x, float bg0, float bg1, float bg2, float* __restrict__ image,
    float* __restrict__ final_t, uint32_t* __restrict__ n_contrib, unsigned long long* __restrict__ pairs) {
  __shared__ float4 s0[kChunk], s1[kChunk], s2[kChunk];
  const PixelGeom pg = pixel_geom(blockIdx.x, tiles_x, width, height);
  const float px = (float)pg.px_i + 0.5f, py = (float)pg.py_j + 0.5f;
  const uint2 range = ranges[blockIdx.x];
  float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
  uint32_t ncon = 0;
  bool done = !pg.inside;
  unsigned long long npairs = 0;
  for (uint32_t base = range.x; base < range.y; base += kChunk) {
    if (__syncthreads_count(!done) == 0) break;
    const uint32_t idx = base + threadIdx.x;
    if (idx < range.y) {
      const uint32_t g = gauss[idx];
      s0[threadIdx.x] = rec[4 * (size_t)g];
      s1[threadIdx.x] = rec[4 * (size_t)g + 1];
      s2[threadIdx.x] = rec[4 * (size_t)g + 2];
    }
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kChunk, range.y - base);
    for (uint32_t k = 0; k < cnt; k++) {
      if (__all_sync(0xffffffffu, done)) break;
      const float4 e2 = s2[k];
      const uint32_t rx = fbits(e2.z), ry = fbits(e2.w);
      if (!rect_hits_block(rx, ry, pg)) continue;
      if (done || !pixel_in_rect(rx, ry, pg)) continue;
      npairs++;
      const float4 e0 = s0[k], e1 = s1[k];
      float gval, alpha;
      if (!evaluate(px, py, e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, &gval, &alpha)) continue;
      const float test_t = T * (1.0f - alpha);
      if (test_t < SPLAT_T_MIN) {
        done = true;
        continue;
      }
      const float at = alpha * T;
      cr += at * e1.w;
      cg += at * e2.x;
      cb += at * e2.y;
      T = test_t;
      ncon = base - range.x + k + 1;
    }
    __syncthreads();
  }
  if (pg.inside) {
    const size_t pix = (size_t)pg.py_j * width + pg.px_i;
    image[3 * pix] = cr + T * bg0;
    image[3 * pix + 1] = cg + T * bg1;
    image[3 * pix + 2] = cb + T * bg2;
    final_t[pix] = T;
    n_contrib[pix] = ncon;
  }
  if (pairs) {
    for (int o = 16; o > 0; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    if ((threadIdx.x & 31) == 0 && npairs) atomicAdd(pairs, npairs);
  }
}

// backward_tile (rasterize.rs:354-455) for one tile per block. Per-pixel contributions to
// an entry's 11 gradient slots are summed across the warp with shuffles, across the
// block's warps in shared memory, and across tiles with one vector atomic per plane.
constexpr int kSlots = 12;  // 11 used, padded for float4 flushes

__global__ void __launch_bounds__(kRasterThreads) raster_bwd_kernel(
    const float4* __restrict__ rec, const uint32_t* __restrict__ gauss, const uint2* __restrict__ ranges,
    uint32_t width, uint32_t height, uint32_t tiles_x, float bg0, float bg1, float bg2,
    const float* __restrict__ final_t, const uint32_t* __restrict__ n_contrib, const float* __restrict__ dimage,
    float4* __restrict__ pgrad, int64_t cap, unsigned long long* __restrict__ pairs) {
  __shared__ float4 s0[kChunk], s1[kChunk], s2[kChunk];
  __shared__ uint32_t sg[kChunk];
  __shared__ float acc[kChunk * kSlots];
  __shared__ uint32_t s_max_last;
  const PixelGeom pg = pixel_geom(blockIdx.x, tiles_x, width, height);
  const float px = (float)pg.px_i + 0.5f, py = (float)pg.py_j + 0.5f;
  const uint2 range = ranges[blockIdx.x];
  const int lane = threadIdx.x & 31;

  uint32_t last = 0;
  float T = 1.0f, t_fin = 1.0f, d0 = 0.0f, d1 = 0.0f, d2 = 0.0f, bg_dot = 0.0f;
  const uint32_t list_len = range.y - range.x;
  if (pg.inside) {
    const size_t pix = (size_t)pg.py_j * width + pg.px_i;
    last = min(n_contrib[pix], list_len);  // n_contrib never exceeds its tile's list
    T = final_t[pix];
    t_fin = T;
    d0 = dimage[3 * pix];
    d1 = dimage[3 * pix + 1];
    d2 = dimage[3 * pix + 2];
    bg_dot = bg0 * d0 + bg1 * d1 + bg2 * d2;
  }
  if (threadIdx.x == 0) s_max_last = 0;
  for (int i = threadIdx.x; i < kChunk * kSlots; i += kRasterThreads) acc[i] = 0.0f;
  __syncthreads();
  {
    const uint32_t m = __reduce_max_sync(0xffffffffu, last);
    if (lane == 0) atomicMax(&s_max_last, m);
  }
  __syncthreads();
  const uint32_t max_last = s_max_last;
  float acc_r = 0.0f, acc_g = 0.0f, acc_b = 0.0f;  // accum (rasterize.rs:347)
  float last_alpha = 0.0f, lc_r = 0.0f, lc_g = 0.0f, lc_b = 0.0f;
  unsigned long long npairs = 0;

  for (uint32_t cend = max_last; cend > 0;) {
    const uint32_t cstart = cend > (uint32_t)kChunk ? cend - kChunk : 0u;
    const uint32_t cnt = cend - cstart;
    if (threadIdx.x < cnt) {
      const uint32_t g = gauss[range.x + cstart + threadIdx.x];
      sg[threadIdx.x] = g;
      s0[threadIdx.x] = rec[4 * (size_t)g];
      s1[threadIdx.x] = rec[4 * (size_t)g + 1];
      s2[threadIdx.x] = rec[4 * (size_t)g + 2];
    }
    __syncthreads();
    for (int kk = (int)cnt - 1; kk >= 0; kk--) {
      const uint32_t k = cstart + (uint32_t)kk;
      const float4 e2 = s2[kk];
      const uint32_t rx = fbits(e2.z), ry = fbits(e2.w);
      if (!rect_hits_block(rx, ry, pg)) continue;
      float c[11];
#pragma unroll
      for (int s = 0; s < 11; s++) c[s] = 0.0f;
      bool active = false;
      if (k < last && pixel_in_rect(rx, ry, pg)) {
        npairs++;
        const float4 e0 = s0[kk], e1 = s1[kk];
        float gval, alpha;
        bool unclamped;
        if (evaluate_bwd(px, py, e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, &gval, &alpha, &unclamped)) {
          active = true;
          // Values only from here on: the arithmetic is fused and the divisions are
          // reciprocals; every decision was taken above exactly as in the forward pass.
          const float col_r = e1.w, col_g = e2.x, col_b = e2.y;
          const float inv = __frcp_rn(1.0f - alpha);
          T = T * inv;
          const float t = T;
          const float keep = 1.0f - last_alpha;
          acc_r = __fmaf_rn(last_alpha, lc_r, keep * acc_r);
          acc_g = __fmaf_rn(last_alpha, lc_g, keep * acc_g);
          acc_b = __fmaf_rn(last_alpha, lc_b, keep * acc_b);
          float dalpha = (col_r - acc_r) * d0;
          dalpha = __fmaf_rn(col_g - acc_g, d1, dalpha);
          dalpha = __fmaf_rn(col_b - acc_b, d2, dalpha);
          const float at = alpha * t;
          c[6] = at * d0;
          c[7] = at * d1;
          c[8] = at * d2;
          lc_r = col_r;
          lc_g = col_g;
          lc_b = col_b;
          last_alpha = alpha;
          dalpha = __fmaf_rn(dalpha, t, -t_fin * inv * bg_dot);
          if (unclamped) {
            const float opacity = e1.y;
            c[5] = gval * dalpha;
            const float dsigma = -(opacity * dalpha) * gval;
            const float dx = px - e0.x;
            const float dy = py - e0.y;
            const float ddx = dsigma * __fmaf_rn(e0.z, dx, e0.w * dy);
            const float ddy = dsigma * __fmaf_rn(e0.w, dx, e1.x * dy);
            c[0] = -ddx;
            c[1] = -ddy;
            const float hs = 0.5f * dsigma;
            c[2] = hs * dx * dx;
            c[3] = dsigma * dx * dy;
            c[4] = hs * dy * dy;
            c[9] = fabsf(ddx);
            c[10] = fabsf(ddy);
          }
        }
      }
      if (__any_sync(0xffffffffu, active)) {
#pragma unroll
        for (int s = 0; s < 11; s++) {
          float v = c[s];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          c[s] = v;
        }
        if (lane == 0) {
#pragma unroll
          for (int s = 0; s < 11; s++) atomicAdd(&acc[kk * kSlots + s], c[s]);
        }
      }
    }
    __syncthreads();
    if (threadIdx.x < cnt) {
      float* a = &acc[threadIdx.x * kSlots];
      const size_t g = sg[threadIdx.x];
      const float4 v0 = make_float4(a[0], a[1], a[2], a[3]);
      const float4 v1 = make_float4(a[4], a[5], a[6], a[7]);
      const float4 v2 = make_float4(a[8], a[9], a[10], 0.0f);
      if (v0.x != 0.0f || v0.y != 0.0f || v0.z != 0.0f || v0.w != 0.0f) atomicAdd(&pgrad[g], v0);
      if (v1.x != 0.0f || v1.y != 0.0f || v1.z != 0.0f || v1.w != 0.0f) atomicAdd(&pgrad[cap + g], v1);
      if (v2.x != 0.0f || v2.y != 0.0f || v2.z != 0.0f) atomicAdd(&pgrad[2 * cap + g], v2);
#pragma unroll
      for (int s = 0; s < kSlots; s++) a[s] = 0.0f;
    }
    __syncthreads();
    cend = cstart;
  }
  if (pairs) {
    for (int o = 16; o > 0; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    if (lane == 0 && npairs) atomicAdd(pairs, npairs);
  }
}

Status launch_raster_fwd(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges, uint32_t width,
                         uint32_t height, const float bg[3], float* image, float* final_t, uint32_t* n_contrib,
                         uint64_t* pairs) {
  const uint32_t tiles_x = (width + kTile - 1) / kTile, tiles_y = (height + kTile - 1) / kTile;
  if (tiles_x * tiles_y == 0) return Status::ok();
  raster_fwd_kernel<<<tiles_x * tiles_y, kRasterThreads, 0, c->stream>>>(
      reinterpret_cast<const float4*>(proj), gauss, reinterpret_cast<const uint2*>(ranges), width, height, tiles_x,
      bg[0], bg[1], bg[2], image, final_t, n_contrib, reinterpret_cast<unsigned long long*>(pairs));
  c->launches.count++;
  SPLAT_LAUNCHED("raster_fwd_kernel");
  return Status::ok();
}

Status launch_raster_bwd(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges, uint32_t width,
                         uint32_t height, const float bg[3], const float* final_t, const uint32_t* n_contrib,
                         const float* dimage, float* pgrad, int64_t cap, uint64_t* pairs) {
  const uint32_t tiles_x = (width + kTile - 1) / kTile, tiles_y = (height + kTile - 1) / kTile;
  if (tiles_x * tiles_y == 0) return Status::ok();
  raster_bwd_kernel<<<tiles_x * tiles_y, kRasterThreads, 0, c->stream>>>(
      reinterpret_cast<const float4*>(proj), gauss, reinterpret_cast<const uint2*>(ranges), width, height, tiles_x,
      bg[0], bg[1], bg[2], final_t, n_contrib, dimage, reinterpret_cast<float4*>(pgrad), cap,
      reinterpret_cast<unsigned long long*>(pairs));
  c->launches.count++;
  SPLAT_LAUNCHED("raster_bwd_kernel");
  return Status::ok();
}

}  // namespace splat
