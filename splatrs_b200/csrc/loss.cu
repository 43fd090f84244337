// Photometric loss (1 - lambda) L1 + lambda (1 - SSIM) with its gradient (reference
// src/loss.rs:14-190), as two tiled kernels.
//
//   ssim_fwd: per 32x32 output tile and channel, the 11-tap separable zero-padded blur of
//     x, y, x^2, y^2 and xy from a shared-memory tile with a 5-pixel halo; per-pixel SSIM
//     and its partial derivatives w.r.t. mu_x, E[x^2], E[xy] (written to scratch); block
//     sums of SSIM, |x - y| and the clamped squared error for PSNR (loss.rs:175-190).
//   ssim_bwd: the same blur of the three partial maps (the blur is self-adjoint,
//     loss.rs:124-127) and the gradient of the whole loss w.r.t. the prediction.
// The target can be the view's 8-bit pixels, converted exactly as View::to_real does
// (reference src/dataset.rs:23-25), or floats. Blur sums run over the window in the
// reference's order and skip out-of-image taps, so the blurred maps, the partial maps and
// the gradient are bit-identical to the reference's; only the three scalar sums depend on
// summation order (accumulated in double here). Blurs of two maps run together as f32x2
// pairs (pair.cuh: each half rounded as the scalar operation), so a tap of (x, y) or of
// (x^2, y^2) is one paired multiply and one paired add.
#include "common.cuh"
#include "kernels.cuh"
#include "pair.cuh"

namespace splat {

constexpr int kLT = 32;            // output tile edge
constexpr int kHalo = 5;           // SSIM_WINDOW / 2
constexpr int kLE = kLT + 2 * kHalo;
constexpr int kLossThreads = 256;
constexpr int kRB = 2;             // consecutive outputs per thread in each blur pass
static_assert(kLT % kRB == 0, "blocks of kRB outputs tile the output rows and columns");

struct LossKernel {
  float w[11];
};

__device__ __forceinline__ float load_target(const void* target, int target_u8, size_t idx) {
  if (target_u8) return (float)static_cast<const uint8_t*>(target)[idx] / 255.0f;
  return static_cast<const float*>(target)[idx];
}

// Sums: [0] SSIM, [1] |x - y|, [2] squared clamped error (PSNR).
__global__ void __launch_bounds__(kLossThreads) ssim_fwd_kernel(const float* __restrict__ pred,
                                                                const void* __restrict__ target_arg, int target_u8,
                                                                uint32_t width, uint32_t height, LossKernel K,
                                                                float* __restrict__ dmaps, double* __restrict__ sums,
                                                                const StepParams* __restrict__ sp,
                                                                const BatchTable* __restrict__ bt) {
  const void* target = sp ? sp->target : target_arg;
  int bxi = blockIdx.x, byi = blockIdx.y;
  if (bt) {  // a batch: flat block index -> view, block within the view, buffer offsets
    if (blockIdx.x >= bt->loss_start[bt->views]) return;
    const int v = batch_view_of(bt->loss_start, bt->views, blockIdx.x);
    const uint32_t local = blockIdx.x - bt->loss_start[v];
    bxi = local % bt->loss_blocks_x[v];
    byi = local / bt->loss_blocks_x[v];
    width = bt->cam[v].width;
    height = bt->cam[v].height;
    pred += 3 * bt->pix_start[v];
    target = bt->target[v];
    dmaps += 9 * bt->pix_start[v];
    sums += 3 * v;
  }
  __shared__ float2 xy_tile[kLE][kLE];             // (prediction, target)
  __shared__ float2 h01[kLE][kLT], h23[kLE][kLT];  // horizontal blurs of (x, y) and (x^2, y^2)
  __shared__ float h4[kLE][kLT];                   // and of x y
  __shared__ double red[3][kLossThreads / 32];
  const int ox0 = bxi * kLT, oy0 = byi * kLT;
  const int tid = threadIdx.x;
  const float c1 = 0.01f * 0.01f, c2 = 0.03f * 0.03f;
  f2 wp[11];
#pragma unroll
  for (int k = 0; k < 11; k++) wp[k] = f2_splat(K.w[k]);
  double s_ssim = 0.0, s_l1 = 0.0, s_se = 0.0;
  for (int ch = 0; ch < 3; ch++) {
    for (int i = tid; i < kLE * kLE; i += kLossThreads) {
      const int r = i / kLE, c = i % kLE;
      const int gy = oy0 - kHalo + r, gx = ox0 - kHalo + c;
      float vx = 0.0f, vy = 0.0f;
      if (gx >= 0 && gx < (int)width && gy >= 0 && gy < (int)height) {
        const size_t idx = ((size_t)gy * width + gx) * 3 + ch;
        vx = pred[idx];
        vy = load_target(target, target_u8, idx);
      }
      xy_tile[r][c] = make_float2(vx, vy);
    }
    __syncthreads();
    // Horizontal pass (loss.rs:42-56) for every halo row: a thread takes kRB consecutive
    // output columns of a row and streams their kRB + 10 inputs once, each tap added in
    // window order. Taps outside the image read the tile's zero padding and add +0.0,
    // which leaves every sum as the reference's (it skips them).
    for (int item = tid; item < kLE * (kLT / kRB); item += kLossThreads) {
      const int r = item / (kLT / kRB), c0 = (item % (kLT / kRB)) * kRB;
      f2 a01[kRB], a23[kRB];
      float a4[kRB];
#pragma unroll
      for (int o = 0; o < kRB; o++) {
        a01[o] = a23[o] = f2_splat(0.0f);
        a4[o] = 0.0f;
      }
#pragma unroll
      for (int q = 0; q < kRB + 10; q++) {
        const float2 t = xy_tile[r][c0 + q];
        const f2 v = f2_make(t.x, t.y), sq = f2_mul(v, v);
        const float xy = t.x * t.y;
#pragma unroll
        for (int o = 0; o < kRB; o++) {
          const int k = q - o;
          if (k < 0 || k > 10) continue;
          a01[o] = f2_add(a01[o], f2_mul(wp[k], v));
          a23[o] = f2_add(a23[o], f2_mul(wp[k], sq));
          a4[o] += K.w[k] * xy;
        }
      }
#pragma unroll
      for (int o = 0; o < kRB; o++) {
        float lo, hi;
        f2_split(a01[o], lo, hi);
        h01[r][c0 + o] = make_float2(lo, hi);
        f2_split(a23[o], lo, hi);
        h23[r][c0 + o] = make_float2(lo, hi);
        h4[r][c0 + o] = a4[o];
      }
    }
    __syncthreads();
    // Vertical pass (loss.rs:58-70) and per-pixel SSIM (loss.rs:101-119): a thread takes kRB
    // consecutive rows of a column, streamed the same way.
    for (int item = tid; item < kLT * (kLT / kRB); item += kLossThreads) {
      const int c = item % kLT, r0 = (item / kLT) * kRB;
      f2 m01[kRB], e23[kRB];
      float exy_[kRB];
#pragma unroll
      for (int o = 0; o < kRB; o++) {
        m01[o] = e23[o] = f2_splat(0.0f);
        exy_[o] = 0.0f;
      }
#pragma unroll
      for (int q = 0; q < kRB + 10; q++) {
        const float2 t01 = h01[r0 + q][c], t23 = h23[r0 + q][c];
        const float t4 = h4[r0 + q][c];
        const f2 v01 = f2_make(t01.x, t01.y), v23 = f2_make(t23.x, t23.y);
#pragma unroll
        for (int o = 0; o < kRB; o++) {
          const int k = q - o;
          if (k < 0 || k > 10) continue;
          m01[o] = f2_add(m01[o], f2_mul(wp[k], v01));
          e23[o] = f2_add(e23[o], f2_mul(wp[k], v23));
          exy_[o] += K.w[k] * t4;
        }
      }
#pragma unroll
      for (int o = 0; o < kRB; o++) {
        const int r = r0 + o;
        const int gy = oy0 + r, gx = ox0 + c;
        if (gx >= (int)width || gy >= (int)height) continue;
        float mx, my, exx, eyy;
        f2_split(m01[o], mx, my);
        f2_split(e23[o], exx, eyy);
        const float exy = exy_[o];
        const float sx2 = exx - mx * mx;
        const float sy2 = eyy - my * my;
        const float sxy = exy - mx * my;
        const float n1 = 2.0f * mx * my + c1;
        const float n2 = 2.0f * sxy + c2;
        const float d1 = mx * mx + my * my + c1;
        const float d2 = sx2 + sy2 + c2;
        const float num = n1 * n2;
        const float den = d1 * d2;
        const float sv = num / den;
        const float dn_dmx = 2.0f * my * n2 - 2.0f * my * n1;
        const float dd_dmx = 2.0f * mx * d2 - 2.0f * mx * d1;
        // The partial maps are planar (map, channel, pixel), so that the backward's per-channel
        // tile loads are contiguous.
        const size_t pix = (size_t)gy * width + gx, npix = (size_t)width * height;
        dmaps[(size_t)ch * npix + pix] = (dn_dmx * den - num * dd_dmx) / (den * den);
        dmaps[(size_t)(3 + ch) * npix + pix] = -num * d1 / (den * den);
        dmaps[(size_t)(6 + ch) * npix + pix] = 2.0f * n1 / den;
        const float2 xy = xy_tile[r + kHalo][c + kHalo];
        const float x = xy.x, y = xy.y;
        s_ssim += (double)sv;
        s_l1 += (double)fabsf(x - y);
        const double e = (double)fminf(fmaxf(x, 0.0f), 1.0f) - (double)fminf(fmaxf(y, 0.0f), 1.0f);
        s_se += e * e;
      }
    }
    __syncthreads();
  }
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s_ssim += __shfl_xor_sync(0xffffffffu, s_ssim, o);
    s_l1 += __shfl_xor_sync(0xffffffffu, s_l1, o);
    s_se += __shfl_xor_sync(0xffffffffu, s_se, o);
  }
  if (lane == 0) {
    red[0][warp] = s_ssim;
    red[1][warp] = s_l1;
    red[2][warp] = s_se;
  }
  __syncthreads();
  if (tid < 3) {
    double t = 0.0;
    for (int w = 0; w < kLossThreads / 32; w++) t += red[tid][w];
    atomicAdd(&sums[tid], t);
  }
}

// Gradient of the loss w.r.t. the prediction (loss.rs:124-133, :155-169).
__global__ void __launch_bounds__(kLossThreads) ssim_bwd_kernel(const float* __restrict__ pred,
                                                                const void* __restrict__ target_arg, int target_u8,
                                                                uint32_t width, uint32_t height, LossKernel K,
                                                                const float* __restrict__ dmaps, float lambda,
                                                                float* __restrict__ grad,
                                                                const StepParams* __restrict__ sp,
                                                                const BatchTable* __restrict__ bt) {
  const void* target = sp ? sp->target : target_arg;
  int bxi = blockIdx.x, byi = blockIdx.y;
  float scale = 1.0f;  // a batch averages the views' gradients
  if (bt) {
    if (blockIdx.x >= bt->loss_start[bt->views]) return;
    const int v = batch_view_of(bt->loss_start, bt->views, blockIdx.x);
    const uint32_t local = blockIdx.x - bt->loss_start[v];
    bxi = local % bt->loss_blocks_x[v];
    byi = local / bt->loss_blocks_x[v];
    width = bt->cam[v].width;
    height = bt->cam[v].height;
    pred += 3 * bt->pix_start[v];
    target = bt->target[v];
    dmaps += 9 * bt->pix_start[v];
    grad += 3 * bt->pix_start[v];
    scale = bt->inv_views;
  }
  __shared__ float2 sm01[kLE][kLE];  // partial maps w.r.t. mu_x and E[x^2]
  __shared__ float sm2[kLE][kLE];    // and w.r.t. E[xy]
  __shared__ float2 h01[kLE][kLT];
  __shared__ float h2[kLE][kLT];
  const int ox0 = bxi * kLT, oy0 = byi * kLT;
  const int tid = threadIdx.x;
  const size_t npix3 = (size_t)width * height * 3;
  const float inv_n = 1.0f / (float)npix3;
  const float w1 = (1.0f - lambda) * inv_n;
  f2 wp[11];
#pragma unroll
  for (int k = 0; k < 11; k++) wp[k] = f2_splat(K.w[k]);
  for (int ch = 0; ch < 3; ch++) {
    for (int i = tid; i < kLE * kLE; i += kLossThreads) {
      const int r = i / kLE, c = i % kLE;
      const int gy = oy0 - kHalo + r, gx = ox0 - kHalo + c;
      float a = 0.0f, b = 0.0f, e = 0.0f;
      if (gx >= 0 && gx < (int)width && gy >= 0 && gy < (int)height) {
        const size_t pix = (size_t)gy * width + gx, npix = (size_t)width * height;
        a = dmaps[(size_t)ch * npix + pix];
        b = dmaps[(size_t)(3 + ch) * npix + pix];
        e = dmaps[(size_t)(6 + ch) * npix + pix];
      }
      sm01[r][c] = make_float2(a, b);
      sm2[r][c] = e;
    }
    __syncthreads();
    // The blur of the three partial maps (loss.rs:124-127), blocked and streamed as in
    // ssim_fwd_kernel; zero-padded taps add +0.0 (the sums start at +0.0 and never become
    // -0.0).
    for (int item = tid; item < kLE * (kLT / kRB); item += kLossThreads) {
      const int r = item / (kLT / kRB), c0 = (item % (kLT / kRB)) * kRB;
      f2 a01[kRB];
      float a2[kRB];
#pragma unroll
      for (int o = 0; o < kRB; o++) {
        a01[o] = f2_splat(0.0f);
        a2[o] = 0.0f;
      }
#pragma unroll
      for (int q = 0; q < kRB + 10; q++) {
        const float2 t = sm01[r][c0 + q];
        const f2 v = f2_make(t.x, t.y);
        const float e = sm2[r][c0 + q];
#pragma unroll
        for (int o = 0; o < kRB; o++) {
          const int k = q - o;
          if (k < 0 || k > 10) continue;
          a01[o] = f2_add(a01[o], f2_mul(wp[k], v));
          a2[o] += K.w[k] * e;
        }
      }
#pragma unroll
      for (int o = 0; o < kRB; o++) {
        float lo, hi;
        f2_split(a01[o], lo, hi);
        h01[r][c0 + o] = make_float2(lo, hi);
        h2[r][c0 + o] = a2[o];
      }
    }
    __syncthreads();
    for (int item = tid; item < kLT * (kLT / kRB); item += kLossThreads) {
      const int c = item % kLT, r0 = (item / kLT) * kRB;
      f2 b01[kRB];
      float b2[kRB];
#pragma unroll
      for (int o = 0; o < kRB; o++) {
        b01[o] = f2_splat(0.0f);
        b2[o] = 0.0f;
      }
#pragma unroll
      for (int q = 0; q < kRB + 10; q++) {
        const float2 t = h01[r0 + q][c];
        const f2 v = f2_make(t.x, t.y);
        const float e = h2[r0 + q][c];
#pragma unroll
        for (int o = 0; o < kRB; o++) {
          const int k = q - o;
          if (k < 0 || k > 10) continue;
          b01[o] = f2_add(b01[o], f2_mul(wp[k], v));
          b2[o] += K.w[k] * e;
        }
      }
#pragma unroll
      for (int o = 0; o < kRB; o++) {
        const int gy = oy0 + r0 + o, gx = ox0 + c;
        if (gx >= (int)width || gy >= (int)height) continue;
        float bmu, bexx;
        f2_split(b01[o], bmu, bexx);
        const float bexy = b2[o];
        const size_t idx = ((size_t)gy * width + gx) * 3 + ch;
        const float x = pred[idx];
        const float y = load_target(target, target_u8, idx);
        const float dssim = (bmu + 2.0f * x * bexx + y * bexy) * inv_n;
        const float d = x - y;
        const float sign = d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f);
        grad[idx] = (w1 * sign - lambda * dssim) * scale;
      }
    }
    __syncthreads();
  }
}

// loss = (1 - lambda) * l1 + lambda * (1 - ssim) (loss.rs:147-154) and PSNR (loss.rs:175-190).
__global__ void loss_finalize_kernel(const double* __restrict__ sums, uint64_t n, float lambda, float* __restrict__ out,
                                     const BatchTable* __restrict__ bt) {
  if (bt) {  // one thread per view: its own sums, pixel count and outputs
    const int v = threadIdx.x;
    if (v >= bt->views) return;
    sums += 3 * v;
    out += 3 * v;
    n = 3 * (bt->pix_start[v + 1] - bt->pix_start[v]);
  } else if (threadIdx.x > 0) {
    return;
  }
  const float inv_n = 1.0f / (float)n;
  const float l1 = (float)sums[1] * inv_n;
  const float ssim = (float)(sums[0] / (double)n);
  out[0] = (1.0f - lambda) * l1 + lambda * (1.0f - ssim);
  out[1] = ssim;
  const double mse = sums[2] / (double)(n > 0 ? n : 1);
  out[2] = mse <= 0.0 ? INFINITY : (float)(-10.0 * log10(mse));
}

LossKernel make_loss_kernel() {
  // gaussian_kernel (loss.rs:14-27), in f32 with the host libm, as the reference does.
  LossKernel k;
  const float sigma = 1.5f;
  float sum = 0.0f;
  for (int i = 0; i < 11; i++) {
    const float x = (float)i - 5.0f;
    k.w[i] = expf(-(x * x) / (2.0f * sigma * sigma));
    sum += k.w[i];
  }
  for (int i = 0; i < 11; i++) k.w[i] /= sum;
  return k;
}

Status launch_loss(Ctx* c, const float* pred, const void* target, int target_u8, uint32_t width, uint32_t height,
                   float lambda, float* grad, float* out3, const StepParams* sp, const BatchTable* bt,
                   uint32_t blocks_cap, uint64_t pix_cap) {
  const size_t npix3 = bt ? (size_t)pix_cap * 3 : (size_t)width * height * 3;
  const int nsums = bt ? kMaxViews : 1;
  float* dmaps = nullptr;
  double* sums = nullptr;
  SPLAT_TRY(arena_reserve(c, npix3 * 3 * 4, (void**)&dmaps));
  SPLAT_TRY(arena_reserve(c, 3 * 8 * nsums, (void**)&sums));
  SPLAT_TRY(launch_fill_u32(c, sums, 3 * 2 * nsums, 0u));
  const LossKernel K = make_loss_kernel();
  const dim3 grid = bt ? dim3(blocks_cap) : dim3(ceil_div(width, kLT), ceil_div(height, kLT));
  ssim_fwd_kernel<<<grid, kLossThreads, 0, c->stream>>>(pred, target, target_u8, width, height, K, dmaps, sums, sp,
                                                         bt);
  ssim_bwd_kernel<<<grid, kLossThreads, 0, c->stream>>>(pred, target, target_u8, width, height, K, dmaps, lambda,
                                                         grad, sp, bt);
  loss_finalize_kernel<<<1, bt ? kMaxViews : 1, 0, c->stream>>>(sums, npix3, lambda, out3, bt);
  c->launches.count += 3;
  SPLAT_LAUNCHED("loss kernels");
  return Status::ok();
}

}  // namespace splat
