// EWA projection with spherical-harmonics colour, forward and backward, one thread per
// Gaussian (reference src/project.rs). Parameters are read as 128-bit loads from the
// float4 planes (a warp reads 512 contiguous bytes per plane); only the SH planes the
// active degree needs are touched.
#include "common.cuh"
#include "kernels.cuh"
#include "adam.cuh"

#include <cuda_bf16.h>

namespace splat {

// Real SH basis constants (reference src/sh.rs:16-33), f64 literals rounded to f32.
#define SH_C0 ((float)0.28209479177387814)
#define SH_C1 ((float)0.4886025119029199)
#define SH_C2_0 ((float)1.0925484305920792)
#define SH_C2_1 ((float)-1.0925484305920792)
#define SH_C2_2 ((float)0.31539156525252005)
#define SH_C2_3 ((float)-1.0925484305920792)
#define SH_C2_4 ((float)0.5462742152960396)
#define SH_C3_0 ((float)-0.5900435899266435)
#define SH_C3_1 ((float)2.890611442640554)
#define SH_C3_2 ((float)-0.4570457994644658)
#define SH_C3_3 ((float)0.3731763325901154)
#define SH_C3_4 ((float)-0.4570457994644658)
#define SH_C3_5 ((float)1.445305721320277)
#define SH_C3_6 ((float)-0.5900435899266435)

__device__ __forceinline__ float sigmoid_f(float x) { return 1.0f / (1.0f + crm::expf_cr(-x)); }

// sh.rs:47-75
template <int DEG>
__device__ __forceinline__ void sh_basis(float x, float y, float z, float b[16]) {
  b[0] = SH_C0;
  if (DEG >= 1) {
    b[1] = -SH_C1 * y;
    b[2] = SH_C1 * z;
    b[3] = -SH_C1 * x;
  }
  if (DEG >= 2) {
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xy = x * y, yz = y * z, xz = x * z;
    b[4] = SH_C2_0 * xy;
    b[5] = SH_C2_1 * yz;
    b[6] = SH_C2_2 * (2.0f * zz - xx - yy);
    b[7] = SH_C2_3 * xz;
    b[8] = SH_C2_4 * (xx - yy);
    if (DEG >= 3) {
      b[9] = SH_C3_0 * y * (3.0f * xx - yy);
      b[10] = SH_C3_1 * xy * z;
      b[11] = SH_C3_2 * y * (4.0f * zz - xx - yy);
      b[12] = SH_C3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
      b[13] = SH_C3_4 * x * (4.0f * zz - xx - yy);
      b[14] = SH_C3_5 * z * (xx - yy);
      b[15] = SH_C3_6 * x * (xx - 3.0f * yy);
    }
  }
}

// sh.rs:80-130 (gradient of every basis function with respect to the direction).
template <int DEG>
__device__ __forceinline__ void sh_basis_grad(float x, float y, float z, float gx[16], float gy[16], float gz[16]) {
#pragma unroll
  for (int k = 0; k < 16; k++) gx[k] = gy[k] = gz[k] = 0.0f;
  if (DEG >= 1) {
    gy[1] = -SH_C1;
    gz[2] = SH_C1;
    gx[3] = -SH_C1;
  }
  if (DEG >= 2) {
    const float xx = x * x, yy = y * y, zz = z * z;
    gx[4] = SH_C2_0 * y;
    gy[4] = SH_C2_0 * x;
    gy[5] = SH_C2_1 * z;
    gz[5] = SH_C2_1 * y;
    gx[6] = -2.0f * SH_C2_2 * x;
    gy[6] = -2.0f * SH_C2_2 * y;
    gz[6] = 4.0f * SH_C2_2 * z;
    gx[7] = SH_C2_3 * z;
    gz[7] = SH_C2_3 * x;
    gx[8] = 2.0f * SH_C2_4 * x;
    gy[8] = -2.0f * SH_C2_4 * y;
    if (DEG >= 3) {
      gx[9] = SH_C3_0 * 6.0f * x * y;
      gy[9] = SH_C3_0 * (3.0f * xx - 3.0f * yy);
      gx[10] = SH_C3_1 * y * z;
      gy[10] = SH_C3_1 * x * z;
      gz[10] = SH_C3_1 * x * y;
      gx[11] = SH_C3_2 * (-2.0f * x * y);
      gy[11] = SH_C3_2 * (4.0f * zz - xx - 3.0f * yy);
      gz[11] = SH_C3_2 * 8.0f * y * z;
      gx[12] = SH_C3_3 * (-6.0f * x * z);
      gy[12] = SH_C3_3 * (-6.0f * y * z);
      gz[12] = SH_C3_3 * (6.0f * zz - 3.0f * xx - 3.0f * yy);
      gx[13] = SH_C3_4 * (4.0f * zz - 3.0f * xx - yy);
      gy[13] = SH_C3_4 * (-2.0f * x * y);
      gz[13] = SH_C3_4 * 8.0f * x * z;
      gx[14] = SH_C3_5 * 2.0f * x * z;
      gy[14] = -SH_C3_5 * 2.0f * y * z;
      gz[14] = SH_C3_5 * (xx - yy);
      gx[15] = SH_C3_6 * (3.0f * xx - 3.0f * yy);
      gy[15] = SH_C3_6 * (-6.0f * x * y);
    }
  }
}

// One Gaussian's parameters in registers.
struct GParams {
  float mean[3];
  float log_scale[3];
  float quat[4];
  float opacity;
  float sh[48];  // sh[3*k + c]
};

// BF16 render copy: planes 1..14 (quaternion, log-scales, SH) as 4 x bf16 per Gaussian,
// plane q at bf[(q - 1) * cap + i]; plane 0 (mean, opacity) stays in the f32 planes.
__device__ __forceinline__ float4 unpack_bf16x4(uint2 u) {
  return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u), __uint_as_float(u.y << 16),
                     __uint_as_float(u.y & 0xffff0000u));
}

__device__ __forceinline__ uint2 pack_bf16x4(float4 v) {
  const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(v.x));
  const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(v.y));
  const uint32_t c = __bfloat16_as_ushort(__float2bfloat16_rn(v.z));
  const uint32_t d = __bfloat16_as_ushort(__float2bfloat16_rn(v.w));
  return make_uint2(a | (b << 16), c | (d << 16));
}

template <bool BF16>
__device__ __forceinline__ float4 load_plane(const float4* __restrict__ planes, const uint2* __restrict__ bf,
                                             int64_t cap, int q, int64_t i) {
  if (BF16 && q > 0) return unpack_bf16x4(bf[(int64_t)(q - 1) * cap + i]);
  return planes[(int64_t)q * cap + i];
}

template <int DEG, bool BF16 = false>
__device__ __forceinline__ void load_params(const float4* __restrict__ planes, int64_t cap, int64_t i, GParams& g,
                                            const uint2* __restrict__ bf = nullptr) {
  const float4 p0 = planes[i];
  const float4 p1 = load_plane<BF16>(planes, bf, cap, 1, i);
  const float4 p2 = load_plane<BF16>(planes, bf, cap, 2, i);
  g.mean[0] = p0.x;
  g.mean[1] = p0.y;
  g.mean[2] = p0.z;
  g.opacity = p0.w;
  g.quat[0] = p1.x;
  g.quat[1] = p1.y;
  g.quat[2] = p1.z;
  g.quat[3] = p1.w;
  g.log_scale[0] = p2.x;
  g.log_scale[1] = p2.y;
  g.log_scale[2] = p2.z;
  constexpr int NC = (DEG + 1) * (DEG + 1);
  constexpr int NQ = (3 * NC + 3) / 4;
#pragma unroll
  for (int q = 0; q < 12; q++) {
    if (q < NQ) {
      const float4 s = load_plane<BF16>(planes, bf, cap, 3 + q, i);
      g.sh[4 * q] = s.x;
      g.sh[4 * q + 1] = s.y;
      g.sh[4 * q + 2] = s.z;
      g.sh[4 * q + 3] = s.w;
    } else {
      g.sh[4 * q] = g.sh[4 * q + 1] = g.sh[4 * q + 2] = g.sh[4 * q + 3] = 0.0f;
    }
  }
}

// Everything project.rs::core computes (project.rs:96-125).
struct CoreOut {
  float t[3];
  float txc, tyc;
  bool clamped_x, clamped_y;
  float s[3];
  float q[4];
  float rq[3][3];
  float m[3][3];
  float sigma[3][3];
  float tmat[2][3];
  float a0, b0, c0, det0, a, b, c, det;
  float conic[3];
  float comp;
  float mean2d[2];
  float radius;
  float o_raw;
  float dir[3];
  float dist;
  float basis[16];
  float color_raw[3];
};

__device__ __forceinline__ float clamp_flag(float v, float lo, float hi, bool* flag) {
  if (v < lo) {
    *flag = true;
    return lo;
  }
  if (v > hi) {
    *flag = true;
    return hi;
  }
  *flag = false;
  return v;
}

// project.rs:137-269, operation for operation. Returns false when culled.
template <int DEG>
__device__ __forceinline__ bool core(const GParams& g, const splat_camera& cam, const splat_proj_opts& opts,
                                     CoreOut& k) {
  const float* R = cam.rot;
  // t = W p + c (camera.rs:36, math.rs:233)
  float t[3];
#pragma unroll
  for (int r = 0; r < 3; r++) t[r] = (R[3 * r] * g.mean[0] + R[3 * r + 1] * g.mean[1] + R[3 * r + 2] * g.mean[2]) + cam.trans[r];
  if (t[2] != t[2] || t[2] <= opts.near_plane) return false;
  float s[3];
#pragma unroll
  for (int j = 0; j < 3; j++) s[j] = crm::expf_cr(g.log_scale[j]);
  // Quat::normalized (math.rs:353-365) and to_mat (math.rs:368-389)
  float qn = sqrtf(g.quat[0] * g.quat[0] + g.quat[1] * g.quat[1] + g.quat[2] * g.quat[2] + g.quat[3] * g.quat[3]);
  float w, x, y, z;
  if (qn > 0.0f) {
    w = g.quat[0] / qn;
    x = g.quat[1] / qn;
    y = g.quat[2] / qn;
    z = g.quat[3] / qn;
  } else {
    w = 1.0f;
    x = y = z = 0.0f;
  }
  float rq[3][3];
  rq[0][0] = 1.0f - 2.0f * (y * y + z * z);
  rq[0][1] = 2.0f * (x * y - w * z);
  rq[0][2] = 2.0f * (x * z + w * y);
  rq[1][0] = 2.0f * (x * y + w * z);
  rq[1][1] = 1.0f - 2.0f * (x * x + z * z);
  rq[1][2] = 2.0f * (y * z - w * x);
  rq[2][0] = 2.0f * (x * z - w * y);
  rq[2][1] = 2.0f * (y * z + w * x);
  rq[2][2] = 1.0f - 2.0f * (x * x + y * y);
  float m[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    m[i][0] = rq[i][0] * s[0];
    m[i][1] = rq[i][1] * s[1];
    m[i][2] = rq[i][2] * s[2];
  }
  // Sigma = M M^T (math.rs:238-250: s starts at 0 and accumulates k = 0, 1, 2)
  float sigma[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float acc = 0.0f;
#pragma unroll
      for (int kk = 0; kk < 3; kk++) acc += m[i][kk] * m[j][kk];
      sigma[i][j] = acc;
    }

  const float W = (float)cam.width, H = (float)cam.height;
  const float tan_x = 0.5f * W / cam.fx;
  const float tan_y = 0.5f * H / cam.fy;
  const float lim_x_pos = (W - cam.cx) / cam.fx + 0.3f * tan_x;
  const float lim_x_neg = cam.cx / cam.fx + 0.3f * tan_x;
  const float lim_y_pos = (H - cam.cy) / cam.fy + 0.3f * tan_y;
  const float lim_y_neg = cam.cy / cam.fy + 0.3f * tan_y;
  const float rz = 1.0f / t[2];
  const float rx = t[0] * rz;
  const float ry = t[1] * rz;
  bool cxf, cyf;
  const float rxc = clamp_flag(rx, -lim_x_neg, lim_x_pos, &cxf);
  const float ryc = clamp_flag(ry, -lim_y_neg, lim_y_pos, &cyf);
  const float txc = rxc * t[2];
  const float tyc = ryc * t[2];
  const float rz2 = rz * rz;
  const float j[2][3] = {{cam.fx * rz, 0.0f, -cam.fx * txc * rz2}, {0.0f, cam.fy * rz, -cam.fy * tyc * rz2}};
  float tmat[2][3];
#pragma unroll
  for (int r = 0; r < 2; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float acc = 0.0f;
#pragma unroll
      for (int kk = 0; kk < 3; kk++) acc += j[r][kk] * R[3 * kk + c];
      tmat[r][c] = acc;
    }
  float ts[2][3];
#pragma unroll
  for (int r = 0; r < 2; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float acc = 0.0f;
#pragma unroll
      for (int kk = 0; kk < 3; kk++) acc += tmat[r][kk] * sigma[kk][c];
      ts[r][c] = acc;
    }
  float a0 = 0.0f, b0 = 0.0f, c0 = 0.0f;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    a0 += ts[0][c] * tmat[0][c];
    b0 += ts[0][c] * tmat[1][c];
    c0 += ts[1][c] * tmat[1][c];
  }
  float det0 = a0 * c0 - b0 * b0;
  float a = a0 + opts.eps2d;
  float b = b0;
  float c = c0 + opts.eps2d;
  float det = a * c - b * b;
  // The trigger is tested on the f32 determinant, whose own error near a ratio of 1e-6
  // reaches ~10%; at 1e-4 it is below 0.1%, so every covariance under 1e-6 * trace^2 is
  // caught. Ordinary Gaussians never reach it (it needs a projected axis ratio near 100).
  if (opts.fp64_conic && (a + c) * (a + c) * 1e-4f > det) {
    // Ill-conditioned in f32 (a needle-like Gaussian: the 2x2 covariance is nearly rank
    // one and its determinant cancels). Rebuild it in f64 from the f32 M and T, whose
    // products are exact in f64: Sigma = M M^T, then T Sigma T^T, determinant and inverse.
    double sd[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++)
        sd[i][jj] = (double)m[i][0] * m[jj][0] + (double)m[i][1] * m[jj][1] + (double)m[i][2] * m[jj][2];
    double tsd[2][3];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
      for (int cc = 0; cc < 3; cc++)
        tsd[r][cc] = (double)tmat[r][0] * sd[0][cc] + (double)tmat[r][1] * sd[1][cc] + (double)tmat[r][2] * sd[2][cc];
    double a0d = 0.0, b0d = 0.0, c0d = 0.0;
#pragma unroll
    for (int cc = 0; cc < 3; cc++) {
      a0d += tsd[0][cc] * tmat[0][cc];
      b0d += tsd[0][cc] * tmat[1][cc];
      c0d += tsd[1][cc] * tmat[1][cc];
    }
    const double ad = a0d + opts.eps2d, cd = c0d + opts.eps2d;
    const double dd = ad * cd - b0d * b0d;
    if (dd != dd || dd <= 0.0) return false;
    a0 = (float)a0d;
    b0 = (float)b0d;
    c0 = (float)c0d;
    det0 = (float)(a0d * c0d - b0d * b0d);
    a = (float)ad;
    b = (float)b0d;
    c = (float)cd;
    det = (float)dd;
    k.conic[0] = (float)(cd / dd);
    k.conic[1] = (float)(-b0d / dd);
    k.conic[2] = (float)(ad / dd);
  } else {
    if (det != det || det <= 0.0f) return false;
    const float inv_det0 = 1.0f / det;
    k.conic[0] = c * inv_det0;
    k.conic[1] = -b * inv_det0;
    k.conic[2] = a * inv_det0;
  }
  const float inv_det = 1.0f / det;
  float comp;
  if (opts.antialias)
    comp = det0 > 0.0f ? sqrtf(det0 * inv_det) : 0.0f;
  else
    comp = 1.0f;
  const float mid = 0.5f * (a + c);
  const float lambda1 = mid + sqrtf(fmaxf(mid * mid - det, 0.1f));
  k.radius = ceilf(3.0f * sqrtf(lambda1));
  k.mean2d[0] = cam.fx * rx + cam.cx;
  k.mean2d[1] = cam.fy * ry + cam.cy;
  k.o_raw = sigmoid_f(g.opacity);

  // View direction from the camera centre -(R^T t) (camera.rs:41).
  float ctr[3];
#pragma unroll
  for (int col = 0; col < 3; col++) ctr[col] = -((R[col] * cam.trans[0] + R[3 + col] * cam.trans[1]) + R[6 + col] * cam.trans[2]);
  const float d0 = g.mean[0] - ctr[0], d1 = g.mean[1] - ctr[1], d2 = g.mean[2] - ctr[2];
  const float dist = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
  const float inv = 1.0f / dist;
  k.dir[0] = d0 * inv;
  k.dir[1] = d1 * inv;
  k.dir[2] = d2 * inv;
#pragma unroll
  for (int i = 0; i < 16; i++) k.basis[i] = 0.0f;
  sh_basis<DEG>(k.dir[0], k.dir[1], k.dir[2], k.basis);
  constexpr int NC = (DEG + 1) * (DEG + 1);
  k.color_raw[0] = k.color_raw[1] = k.color_raw[2] = 0.5f;
#pragma unroll
  for (int kk = 0; kk < NC; kk++)
#pragma unroll
    for (int ch = 0; ch < 3; ch++) k.color_raw[ch] += k.basis[kk] * g.sh[3 * kk + ch];

#pragma unroll
  for (int i = 0; i < 3; i++) {
    k.t[i] = t[i];
    k.s[i] = s[i];
  }
  k.q[0] = w;
  k.q[1] = x;
  k.q[2] = y;
  k.q[3] = z;
  k.txc = txc;
  k.tyc = tyc;
  k.clamped_x = cxf;
  k.clamped_y = cyf;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int jj = 0; jj < 3; jj++) {
      k.rq[i][jj] = rq[i][jj];
      k.m[i][jj] = m[i][jj];
      k.sigma[i][jj] = sigma[i][jj];
    }
#pragma unroll
  for (int r = 0; r < 2; r++)
#pragma unroll
    for (int cc = 0; cc < 3; cc++) k.tmat[r][cc] = tmat[r][cc];
  k.a0 = a0;
  k.b0 = b0;
  k.c0 = c0;
  k.det0 = det0;
  k.a = a;
  k.b = b;
  k.c = c;
  k.det = det;
  k.comp = comp;
  k.dist = dist;
  return true;
}

__device__ __forceinline__ uint32_t clamp_tile(float v, uint32_t n) {
  if (v <= 0.0f) return 0u;
  if (v >= (float)n) return n;
  return (uint32_t)v;
}

// Absolute pixel bound of a per-entry rectangle, clamped to [0, n]; NaN maps to 0. The
// reference clips per tile (rasterize.rs:158-164); clipping the absolute bound to the image
// first selects the same pixels of every tile.
__device__ __forceinline__ uint32_t abs_bound(float v, uint32_t n) {
  if (v != v || v <= 0.0f) return 0u;
  if (v >= (float)n) return n;
  return (uint32_t)v;
}

// Finish a projection record from the reference Proj fields. The compositing quantities
// sigma_max and the ellipse bounding box follow TileGauss::new (rasterize.rs:149-182).
__device__ __forceinline__ void write_record(float4* __restrict__ rec, uint32_t* __restrict__ num_tiles, int64_t i,
                                             const float mean2d[2], const float conic[3], float depth, uint32_t radius,
                                             float opacity, const float color[3], uint32_t tx0, uint32_t ty0,
                                             uint32_t tx1, uint32_t ty1, uint32_t width, uint32_t height,
                                             uint32_t* depth_range, uint32_t tile_w, uint32_t tile_h) {
  const float sigma_max = crm::logf_cr(opacity / SPLAT_ALPHA_MIN);
  const float A = conic[0], B = conic[1], Cc = conic[2];
  const float det = A * Cc - B * B;
  uint32_t x0 = 0, x1 = 0, y0 = 0, y1 = 0;
  if (sigma_max > 0.0f && det > 0.0f) {
    const float half_x = sqrtf(2.0f * sigma_max * Cc / det) + 1e-3f;
    const float half_y = sqrtf(2.0f * sigma_max * A / det) + 1e-3f;
    x0 = abs_bound(ceilf(mean2d[0] - half_x - 0.5f), width);
    x1 = abs_bound(floorf(mean2d[0] + half_x - 0.5f) + 1.0f, width);
    y0 = abs_bound(ceilf(mean2d[1] - half_y - 0.5f), height);
    y1 = abs_bound(floorf(mean2d[1] + half_y - 0.5f) + 1.0f, height);
  }
  if (tile_w != kTile || tile_h != kTile) {
    // Another tile shape: the pixels the entry may touch are its alpha box within its
    // 16-pixel tile rectangle (what the reference's tile lists and per-pixel test allow
    // together), and its tiles are the ones that box overlaps, so every pixel composites
    // the same entries in the same order as with 16x16 tiles.
    const uint32_t ex0 = max(x0, tx0 * kTile), ex1 = min(x1, tx1 * kTile);
    const uint32_t ey0 = max(y0, ty0 * kTile), ey1 = min(y1, ty1 * kTile);
    if (ex0 < ex1 && ey0 < ey1) {
      x0 = ex0;
      x1 = ex1;
      y0 = ey0;
      y1 = ey1;
      tx0 = ex0 / tile_w;
      tx1 = (ex1 + tile_w - 1) / tile_w;
      ty0 = ey0 / tile_h;
      ty1 = (ey1 + tile_h - 1) / tile_h;
    } else {
      x0 = x1 = y0 = y1 = 0;
      tx0 = tx1 = ty0 = ty1 = 0;
    }
  }
  rec[4 * i + 0] = make_float4(mean2d[0], mean2d[1], A, B);
  rec[4 * i + 1] = make_float4(Cc, opacity, sigma_max, color[0]);
  rec[4 * i + 2] = make_float4(color[1], color[2], bitsf(x0 | (x1 << 16)), bitsf(y0 | (y1 << 16)));
  rec[4 * i + 3] = make_float4(depth, bitsf(radius), bitsf(tx0 | (ty0 << 16)), bitsf(tx1 | (ty1 << 16)));
  num_tiles[i] = (tx1 - tx0) * (ty1 - ty0);
  (void)depth_range;
}

__device__ __forceinline__ void write_culled(float4* __restrict__ rec, uint32_t* __restrict__ num_tiles, int64_t i) {
  const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  rec[4 * i + 0] = z;
  rec[4 * i + 1] = z;
  rec[4 * i + 2] = z;
  rec[4 * i + 3] = z;
  num_tiles[i] = 0;
}

// Warp-aggregated min/max of the visible depth bits.
__device__ __forceinline__ void depth_range_update(uint32_t* depth_range, bool visible, float depth) {
  const uint32_t bits = fbits(depth);
  const uint32_t mn = __reduce_min_sync(0xffffffffu, visible ? bits : 0xffffffffu);
  const uint32_t mx = __reduce_max_sync(0xffffffffu, visible ? bits : 0u);
  if ((threadIdx.x & 31) == 0 && __any_sync(1u, true)) {
    if (mn != 0xffffffffu) atomicMin(&depth_range[0], mn);
    if (mx != 0u) atomicMax(&depth_range[1], mx);
  }
}

// project_one (project.rs:277-317) for every Gaussian.
template <int DEG, bool BF16>
__global__ void __launch_bounds__(256) project_fwd_kernel(const float4* __restrict__ planes, int64_t n, int64_t cap,
                                                          splat_camera cam_arg, splat_proj_opts opts,
                                                          float4* __restrict__ rec, uint32_t* __restrict__ num_tiles,
                                                          uint32_t* __restrict__ depth_range,
                                                          const StepParams* __restrict__ sp,
                                                          const uint2* __restrict__ bf,
                                                          const BatchTable* __restrict__ bt, uint32_t tile_w,
                                                          uint32_t tile_h) {
  // A batch launch has one grid row per view; its records follow view-major.
  const int view = bt ? (int)blockIdx.y : 0;
  if (bt && view >= bt->views) return;
  const splat_camera cam = bt ? bt->cam[view] : (sp ? sp->cam : cam_arg);
  if (bt) {
    rec += 4 * (size_t)view * n;
    num_tiles += (size_t)view * n;
  }
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool visible = false;
  float depth = 0.0f;
  if (i < n) {
    GParams g;
    load_params<DEG, BF16>(planes, cap, i, g, bf);
    CoreOut k;
    bool ok = core<DEG>(g, cam, opts, k);
    if (ok) {
      const uint32_t tiles_x = (cam.width + kTile - 1) / kTile, tiles_y = (cam.height + kTile - 1) / kTile;
      const float r = k.radius;
      if (!(r != r || r <= 0.0f)) {
        const float tile = (float)kTile;
        const uint32_t tx0 = clamp_tile(floorf((k.mean2d[0] - r) / tile), tiles_x);
        const uint32_t tx1 = clamp_tile(ceilf((k.mean2d[0] + r) / tile), tiles_x);
        const uint32_t ty0 = clamp_tile(floorf((k.mean2d[1] - r) / tile), tiles_y);
        const uint32_t ty1 = clamp_tile(ceilf((k.mean2d[1] + r) / tile), tiles_y);
        if (tx0 < tx1 && ty0 < ty1) {
          float color[3];
#pragma unroll
          for (int ch = 0; ch < 3; ch++) color[ch] = fmaxf(k.color_raw[ch], 0.0f);
          const float opacity = k.o_raw * k.comp;
          write_record(rec, num_tiles, i, k.mean2d, k.conic, k.t[2], sat_u32(r), opacity, color, tx0, ty0, tx1, ty1,
                       cam.width, cam.height, depth_range, tile_w, tile_h);
          visible = true;
          depth = k.t[2];
        }
      }
    }
    if (!visible) write_culled(rec, num_tiles, i);
  }
  depth_range_update(depth_range, visible, depth);
}

// Records from reference-layout Proj values.
__global__ void proj_from_reference_kernel(const float* __restrict__ p15, int64_t n, uint32_t width, uint32_t height,
                                           float4* __restrict__ rec, uint32_t* __restrict__ num_tiles,
                                           uint32_t* __restrict__ depth_range, uint32_t tile_w, uint32_t tile_h) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool visible = false;
  float depth = 0.0f;
  if (i < n) {
    const float* p = p15 + 15 * i;
    const uint32_t radius = (uint32_t)p[6];
    // A tile rectangle outside the grid is clamped to it (the reference panics there,
    // src/rasterize.rs:65-69), so no entry can name a tile that does not exist.
    const uint32_t tiles_x = (width + kTile - 1) / kTile, tiles_y = (height + kTile - 1) / kTile;
    const uint32_t tx0 = (uint32_t)p[11], ty0 = (uint32_t)p[12];
    const uint32_t tx1 = min((uint32_t)p[13], tiles_x), ty1 = min((uint32_t)p[14], tiles_y);
    if (radius > 0 && tx0 < tx1 && ty0 < ty1) {
      const float mean2d[2] = {p[0], p[1]};
      const float conic[3] = {p[2], p[3], p[4]};
      const float color[3] = {p[8], p[9], p[10]};
      write_record(rec, num_tiles, i, mean2d, conic, p[5], radius, p[7], color, tx0, ty0, tx1, ty1, width, height,
                   depth_range, tile_w, tile_h);
      visible = true;
      depth = p[5];
    } else {
      write_culled(rec, num_tiles, i);
    }
  }
  depth_range_update(depth_range, visible, depth);
}

__global__ void proj_to_reference_kernel(const float4* __restrict__ rec, int64_t n, float* __restrict__ p15) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 r0 = rec[4 * i], r1 = rec[4 * i + 1], r2 = rec[4 * i + 2], r3 = rec[4 * i + 3];
  float* p = p15 + 15 * i;
  const uint32_t radius = fbits(r3.y);
  const uint32_t tmin = fbits(r3.z), tmax = fbits(r3.w);
  p[0] = r0.x;
  p[1] = r0.y;
  p[2] = r0.z;
  p[3] = r0.w;
  p[4] = r1.x;
  p[5] = r3.x;
  p[6] = (float)radius;
  p[7] = r1.y;
  p[8] = r1.w;
  p[9] = r2.x;
  p[10] = r2.y;
  p[11] = (float)(tmin & 0xffffu);
  p[12] = (float)(tmin >> 16);
  p[13] = (float)(tmax & 0xffffu);
  p[14] = (float)(tmax >> 16);
}

// project_backward_one (project.rs:335-474) for parameters g seen by camera cam, given the
// screen-space gradient (g0, g1, g2 as in the ProjGrad planes): the 59 parameter gradients,
// zero when the Gaussian is culled.
struct ParamGrad {
  float mean[3], op, q[4], ls[3], sh[48];
};

template <int DEG>
__device__ __forceinline__ void proj_grad_one(const GParams& g, const splat_camera& cam, const splat_proj_opts& opts,
                                              const float4 g0, const float4 g1, const float4 g2, ParamGrad& out) {
  const float dp_mean2d[2] = {g0.x, g0.y};
  const float dp_conic[3] = {g0.z, g0.w, g1.x};
  const float dp_opacity = g1.y;
  const float dp_color[3] = {g1.z, g1.w, g2.x};
  float* o_mean = out.mean;
  float* o_ls = out.ls;
  float* o_q = out.q;
  float* o_sh = out.sh;
  float& o_op = out.op;
#pragma unroll
  for (int q = 0; q < 3; q++) o_mean[q] = o_ls[q] = 0.0f;
#pragma unroll
  for (int q = 0; q < 4; q++) o_q[q] = 0.0f;
  o_op = 0.0f;
#pragma unroll
  for (int q = 0; q < 48; q++) o_sh[q] = 0.0f;
  CoreOut k;
  if (core<DEG>(g, cam, opts, k)) {
    constexpr int NC = (DEG + 1) * (DEG + 1);
    float bgx[16], bgy[16], bgz[16];
    sh_basis_grad<DEG>(k.dir[0], k.dir[1], k.dir[2], bgx, bgy, bgz);
    float ddir[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int ch = 0; ch < 3; ch++) {
      if (k.color_raw[ch] > 0.0f) {
        const float dc = dp_color[ch];
#pragma unroll
        for (int kk = 0; kk < NC; kk++) {
          o_sh[3 * kk + ch] = dc * k.basis[kk];
          const float wgt = dc * g.sh[3 * kk + ch];
          ddir[0] += bgx[kk] * wgt;
          ddir[1] += bgy[kk] * wgt;
          ddir[2] += bgz[kk] * wgt;
        }
      }
    }
    const float dd = k.dir[0] * ddir[0] + k.dir[1] * ddir[1] + k.dir[2] * ddir[2];
    const float idist = 1.0f / k.dist;
    float dmean_color[3];
#pragma unroll
    for (int a = 0; a < 3; a++) dmean_color[a] = (ddir[a] - k.dir[a] * dd) * idist;

    const float do_raw = dp_opacity * k.comp;
    const float dcomp = dp_opacity * k.o_raw;
    o_op = do_raw * k.o_raw * (1.0f - k.o_raw);

    const float a = k.a, b = k.b, c = k.c, det = k.det;
    const float da_ = dp_conic[0], db_ = dp_conic[1], dc_ = dp_conic[2];
    const float inv_det2 = 1.0f / (det * det);
    float da = (-c * c * da_ + b * c * db_ - b * b * dc_) * inv_det2;
    float db = (2.0f * b * c * da_ - (a * c + b * b) * db_ + 2.0f * a * b * dc_) * inv_det2;
    float dcv = (-b * b * da_ + a * b * db_ - a * a * dc_) * inv_det2;
    if (opts.antialias && k.det0 > 0.0f) {
      const float ddet0 = dcomp * 0.5f * k.comp / k.det0;
      const float ddet = -dcomp * 0.5f * k.comp / det;
      da += ddet0 * k.c0 + ddet * c;
      dcv += ddet0 * k.a0 + ddet * a;
      db += ddet0 * (-2.0f * k.b0) + ddet * (-2.0f * b);
    }
    const float gm[2][2] = {{da, 0.5f * db}, {0.5f * db, dcv}};
    float gt[2][3];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
      for (int col = 0; col < 3; col++) gt[r][col] = gm[r][0] * k.tmat[0][col] + gm[r][1] * k.tmat[1][col];
    float dsigma[3][3];
#pragma unroll
    for (int ii = 0; ii < 3; ii++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++) dsigma[ii][jj] = k.tmat[0][ii] * gt[0][jj] + k.tmat[1][ii] * gt[1][jj];
    float dt[2][3];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
      for (int col = 0; col < 3; col++) {
        float acc = 0.0f;
#pragma unroll
        for (int kk = 0; kk < 3; kk++) acc += gt[r][kk] * k.sigma[kk][col];
        dt[r][col] = 2.0f * acc;
      }
    const float* R = cam.rot;
    float dj[2][3];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
      for (int col = 0; col < 3; col++) {
        float acc = 0.0f;
#pragma unroll
        for (int kk = 0; kk < 3; kk++) acc += dt[r][kk] * R[3 * col + kk];
        dj[r][col] = acc;
      }
    const float fx = cam.fx, fy = cam.fy;
    const float rz = 1.0f / k.t[2];
    const float rz2 = rz * rz;
    const float rz3 = rz2 * rz;
    const float dtxc = dj[0][2] * (-fx * rz2);
    const float dtyc = dj[1][2] * (-fy * rz2);
    float dtx = 0.0f, dty = 0.0f;
    float dtz = dj[0][0] * (-fx * rz2) + dj[1][1] * (-fy * rz2) + dj[0][2] * (2.0f * fx * k.txc * rz3) +
                dj[1][2] * (2.0f * fy * k.tyc * rz3);
    if (k.clamped_x)
      dtz += dtxc * k.txc * rz;
    else
      dtx += dtxc;
    if (k.clamped_y)
      dtz += dtyc * k.tyc * rz;
    else
      dty += dtyc;
    dtx += dp_mean2d[0] * fx * rz;
    dtz += dp_mean2d[0] * (-fx * k.t[0] * rz2);
    dty += dp_mean2d[1] * fy * rz;
    dtz += dp_mean2d[1] * (-fy * k.t[1] * rz2);
    // dmean = R^T (dtx, dty, dtz) + dmean_color (math.rs:233 on the transpose)
#pragma unroll
    for (int col = 0; col < 3; col++) o_mean[col] = (R[col] * dtx + R[3 + col] * dty + R[6 + col] * dtz) + dmean_color[col];

    // dM = 2 dSigma M (math.rs:238, :275)
    float dm[3][3];
#pragma unroll
    for (int ii = 0; ii < 3; ii++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++) {
        float acc = 0.0f;
#pragma unroll
        for (int kk = 0; kk < 3; kk++) acc += dsigma[ii][kk] * k.m[kk][jj];
        dm[ii][jj] = acc * 2.0f;
      }
    float ds[3] = {0.0f, 0.0f, 0.0f};
    float dr[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int col = 0; col < 3; col++) {
        ds[col] += dm[r][col] * k.rq[r][col];
        dr[r][col] = dm[r][col] * k.s[col];
      }
#pragma unroll
    for (int ii = 0; ii < 3; ii++) o_ls[ii] = ds[ii] * k.s[ii];
    // quat_to_mat_backward (math.rs:395-431) as Frobenius products with dR.
    const float w = k.q[0], x = k.q[1], y = k.q[2], z = k.q[3];
    const float Mw[9] = {0.0f, -2.0f * z, 2.0f * y, 2.0f * z, 0.0f, -2.0f * x, -2.0f * y, 2.0f * x, 0.0f};
    const float Mx[9] = {0.0f, 2.0f * y, 2.0f * z, 2.0f * y, -4.0f * x, -2.0f * w, 2.0f * z, 2.0f * w, -4.0f * x};
    const float My[9] = {-4.0f * y, 2.0f * x, 2.0f * w, 2.0f * x, 0.0f, 2.0f * z, -2.0f * w, 2.0f * z, -4.0f * y};
    const float Mz[9] = {-4.0f * z, -2.0f * w, 2.0f * x, 2.0f * w, -4.0f * z, 2.0f * y, 2.0f * x, 2.0f * y, 0.0f};
    float dq[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int e = 0; e < 9; e++) {
      const float d = dr[e / 3][e % 3];
      dq[0] += d * Mw[e];
      dq[1] += d * Mx[e];
      dq[2] += d * My[e];
      dq[3] += d * Mz[e];
    }
    // normalize_backward (math.rs:434-446)
    const float nrm = sqrtf(g.quat[0] * g.quat[0] + g.quat[1] * g.quat[1] + g.quat[2] * g.quat[2] + g.quat[3] * g.quat[3]);
    if (nrm > 0.0f) {
      const float u[4] = {g.quat[0] / nrm, g.quat[1] / nrm, g.quat[2] / nrm, g.quat[3] / nrm};
      const float dot = u[0] * dq[0] + u[1] * dq[1] + u[2] * dq[2] + u[3] * dq[3];
#pragma unroll
      for (int ii = 0; ii < 4; ii++) o_q[ii] = (dq[ii] - u[ii] * dot) / nrm;
    }
  }
}

// project_backward_one (project.rs:335-474), plus DensifyStats::accumulate
// (densify.rs:36-60) when `stats` is given. With ADAM the 59 gradients never leave the
// registers: Adam::step (adam.rs:77-161) updates the parameters in place and the moments m
// and v, over every plane (zero gradients still decay the moments, adam.rs:56-60).
// Four blocks of 128 per SM: the 59 gradients and the streamed parameters and moments
// would take 190-242 registers (8 warps per SM, too few to hide the memory latency of an
// HBM-bound kernel); capped at 128 the kernel spills a few hundred bytes to L1 and runs
// 22-23% faster (measured at 1M Gaussians: 0.606 -> 0.475 ms with Adam, 0.149 -> 0.115 ms
// without).
template <int DEG, bool ADAM, bool BF16>
__global__ void __launch_bounds__(128, 4) project_bwd_kernel(const float4* __restrict__ planes, int64_t n, int64_t cap,
                                                          splat_camera cam_arg, splat_proj_opts opts,
                                                          const float4* __restrict__ rec,
                                                          const float4* __restrict__ pgrad,
                                                          float4* __restrict__ out, float* __restrict__ stat_accum,
                                                          uint32_t* __restrict__ stat_denom,
                                                          uint32_t* __restrict__ stat_maxr, int absgrad,
                                                          float4* __restrict__ adam_m, float4* __restrict__ adam_v,
                                                          AdamArgs adam_arg, const uint32_t* __restrict__ skip,
                                                          const StepParams* __restrict__ sp, uint2* bf,
                                                          float* __restrict__ stat_maxg) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (ADAM && skip && *skip) return;
  const splat_camera cam = sp ? sp->cam : cam_arg;
  const AdamArgs adam = (ADAM && sp) ? sp->adam : adam_arg;
  const float4 g0 = pgrad[i], g1 = pgrad[cap + i], g2 = pgrad[2 * cap + i];

  if (stat_accum != nullptr) {
    const uint32_t radius = fbits(rec[4 * i + 3].y);
    if (radius > 0) {
      const float sx = (float)cam.width * 0.5f;
      const float sy = (float)cam.height * 0.5f;
      const float gx = (absgrad ? g2.y : g0.x) * sx;
      const float gy = (absgrad ? g2.z : g0.y) * sy;
      const float gn = sqrtf(gx * gx + gy * gy);
      stat_accum[i] += gn;
      stat_denom[i] += 1u;
      stat_maxr[i] = max(stat_maxr[i], radius);
      if (stat_maxg) {
        stat_maxg[i] = fmaxf(stat_maxg[i], gn);
        stat_maxg[cap + i] += g2.w;  // contribution: the view's blending weight sum (alpha T)
      }
    }
  }

  GParams g;
  load_params<DEG, BF16>(planes, cap, i, g, bf);
  ParamGrad pgr;
  proj_grad_one<DEG>(g, cam, opts, g0, g1, g2, pgr);
  const float* o_mean = pgr.mean;
  const float* o_q = pgr.q;
  const float* o_ls = pgr.ls;
  const float* o_sh = pgr.sh;
  const float o_op = pgr.op;
  if (!ADAM) {
    out[i] = make_float4(o_mean[0], o_mean[1], o_mean[2], o_op);
    out[cap + i] = make_float4(o_q[0], o_q[1], o_q[2], o_q[3]);
    out[2 * cap + i] = make_float4(o_ls[0], o_ls[1], o_ls[2], 0.0f);
#pragma unroll
    for (int q = 0; q < 12; q++) out[(3 + q) * cap + i] = make_float4(o_sh[4 * q], o_sh[4 * q + 1], o_sh[4 * q + 2], o_sh[4 * q + 3]);
  } else {
    // The parameters are read above only through `planes`; each element is read before
    // this thread writes it and no other thread touches Gaussian i.
    float4* pw = const_cast<float4*>(planes);
#pragma unroll
    for (int q = 0; q < kPlanes; q++) {
      float4 g;
      if (q == 0)
        g = make_float4(o_mean[0], o_mean[1], o_mean[2], o_op);
      else if (q == 1)
        g = make_float4(o_q[0], o_q[1], o_q[2], o_q[3]);
      else if (q == 2)
        g = make_float4(o_ls[0], o_ls[1], o_ls[2], 0.0f);
      else
        g = make_float4(o_sh[4 * (q - 3)], o_sh[4 * (q - 3) + 1], o_sh[4 * (q - 3) + 2], o_sh[4 * (q - 3) + 3]);
      const int64_t o = (int64_t)q * cap + i;
      float4 p = pw[o], m = adam_m[o], v = adam_v[o];
      adam_plane(adam, q, p, g, m, v);
      pw[o] = p;
      adam_m[o] = m;
      adam_v[o] = v;
      // The render copy follows the f32 master (round to nearest even).
      if (BF16 && q > 0) bf[(int64_t)(q - 1) * cap + i] = pack_bf16x4(p);
    }
  }
}

// Reference Gaussian records <-> planes, 128 Gaussians per block through shared memory so
// that both the plane side (128-bit loads/stores) and the record side (contiguous 59-float
// rows) are coalesced.
constexpr int kConvG = 128;

// Position of record field f (0..58) in the 60-float plane order (mean xyz, opacity, quat,
// log-scale xyz, pad, sh...).
__device__ __forceinline__ int plane_slot_of_field(int f) {
  if (f < 3) return f;          // mean
  if (f < 6) return 8 + f - 3;  // log_scale
  if (f < 10) return 4 + f - 6; // quat
  if (f == 10) return 3;        // opacity
  return 12 + f - 11;           // sh
}

__global__ void __launch_bounds__(kConvG) aos_to_planes_kernel(const float* __restrict__ aos, int64_t n,
                                                               float4* __restrict__ planes, int64_t cap) {
  __shared__ float tile[kConvG][61];
  const int64_t base = (int64_t)blockIdx.x * kConvG;
  const int cnt = (int)min((int64_t)kConvG, n - base);
  const float* src = aos + base * 59;
  for (int L = threadIdx.x; L < cnt * 59; L += kConvG) {
    const int g = L / 59, f = L - g * 59;
    tile[g][plane_slot_of_field(f)] = src[L];
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < cnt) {
    tile[t][11] = 0.0f;  // pad lane of the log-scale plane
#pragma unroll
    for (int q = 0; q < kPlanes; q++)
      planes[q * cap + base + t] = make_float4(tile[t][4 * q], tile[t][4 * q + 1], tile[t][4 * q + 2], tile[t][4 * q + 3]);
  }
}

__global__ void __launch_bounds__(kConvG) planes_to_aos_kernel(const float4* __restrict__ planes, int64_t n, int64_t cap,
                                                               float* __restrict__ aos) {
  __shared__ float tile[kConvG][61];
  const int64_t base = (int64_t)blockIdx.x * kConvG;
  const int cnt = (int)min((int64_t)kConvG, n - base);
  const int t = threadIdx.x;
  if (t < cnt) {
#pragma unroll
    for (int q = 0; q < kPlanes; q++) {
      const float4 v = planes[q * cap + base + t];
      tile[t][4 * q] = v.x;
      tile[t][4 * q + 1] = v.y;
      tile[t][4 * q + 2] = v.z;
      tile[t][4 * q + 3] = v.w;
    }
  }
  __syncthreads();
  float* dst = aos + base * 59;
  for (int L = threadIdx.x; L < cnt * 59; L += kConvG) {
    const int g = L / 59, f = L - g * 59;
    dst[L] = tile[g][plane_slot_of_field(f)];
  }
}

// ---------------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------------
Status launch_project_fwd(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                          const splat_proj_opts& opts, float* proj, uint32_t* num_tiles, uint32_t* depth_range,
                          const StepParams* sp, const void* bf16, const BatchTable* bt) {
  SPLAT_TRY(launch_fill_u32(c, depth_range, 1, 0xffffffffu));
  SPLAT_TRY(launch_fill_u32(c, depth_range + 1, 1, 0u));
  if (n == 0) return Status::ok();
  const int bs = 256;
  const uint32_t grid = ceil_div(n, bs);
  const float4* p = reinterpret_cast<const float4*>(planes);
  float4* r = reinterpret_cast<float4*>(proj);
  const uint2* bf = static_cast<const uint2*>(bf16);
#define SPLAT_PFWD(D, B) \
  project_fwd_kernel<D, B><<<dim3(grid, bt ? kMaxViews : 1), bs, 0, c->stream>>>(p, n, cap, cam, opts, r, num_tiles, \
                                                                                 depth_range, sp, bf, bt, \
                                                                                 c->raster.tile_w, c->raster.tile_h)
  if (bf) {
    switch (opts.sh_degree) {
      case 0: SPLAT_PFWD(0, true); break;
      case 1: SPLAT_PFWD(1, true); break;
      case 2: SPLAT_PFWD(2, true); break;
      default: SPLAT_PFWD(3, true); break;
    }
  } else {
    switch (opts.sh_degree) {
      case 0: SPLAT_PFWD(0, false); break;
      case 1: SPLAT_PFWD(1, false); break;
      case 2: SPLAT_PFWD(2, false); break;
      default: SPLAT_PFWD(3, false); break;
    }
  }
#undef SPLAT_PFWD
  c->launches.count++;
  SPLAT_LAUNCHED("project_fwd_kernel");
  return Status::ok();
}

Status launch_proj_from_reference(Ctx* c, const float* p15, int64_t n, uint32_t width, uint32_t height, float* proj,
                                  uint32_t* num_tiles, uint32_t* depth_range) {
  SPLAT_TRY(launch_fill_u32(c, depth_range, 1, 0xffffffffu));
  SPLAT_TRY(launch_fill_u32(c, depth_range + 1, 1, 0u));
  if (n == 0) return Status::ok();
  proj_from_reference_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(p15, n, width, height,
                                                                       reinterpret_cast<float4*>(proj), num_tiles,
                                                                       depth_range, c->raster.tile_w,
                                                                       c->raster.tile_h);
  c->launches.count++;
  SPLAT_LAUNCHED("proj_from_reference_kernel");
  return Status::ok();
}

Status launch_proj_to_reference(Ctx* c, const float* proj, int64_t n, float* p15) {
  if (n == 0) return Status::ok();
  proj_to_reference_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(reinterpret_cast<const float4*>(proj), n, p15);
  c->launches.count++;
  SPLAT_LAUNCHED("proj_to_reference_kernel");
  return Status::ok();
}

template <bool ADAM, bool BF16>
static Status project_bwd_launch(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                                 const splat_proj_opts& opts, const float* proj, const float* pgrad, float* out,
                                 void* stats, int absgrad, float* m, float* v, const AdamArgs& adam,
                                 const uint32_t* skip, const StepParams* sp, uint2* bf, bool with_maxg) {
  if (n == 0) return Status::ok();
  const int bs = 128;
  const uint32_t grid = ceil_div(n, bs);
  const float4* p = reinterpret_cast<const float4*>(planes);
  const float4* r = reinterpret_cast<const float4*>(proj);
  const float4* pg = reinterpret_cast<const float4*>(pgrad);
  float4* o = reinterpret_cast<float4*>(out);
  float4* am = reinterpret_cast<float4*>(m);
  float4* av = reinterpret_cast<float4*>(v);
  float* sa = nullptr;
  uint32_t *sd = nullptr, *sm = nullptr;
  float* smg = nullptr;
  if (stats) {
    sa = reinterpret_cast<float*>(stats);
    sd = reinterpret_cast<uint32_t*>(sa + cap);
    sm = sd + cap;
    if (with_maxg) smg = reinterpret_cast<float*>(sm + cap);
  }
#define SPLAT_PBWD(D) \
  project_bwd_kernel<D, ADAM, BF16><<<grid, bs, 0, c->stream>>>(p, n, cap, cam, opts, r, pg, o, sa, sd, sm, absgrad, am, av, adam, skip, sp, bf, smg)
  switch (opts.sh_degree) {
    case 0: SPLAT_PBWD(0); break;
    case 1: SPLAT_PBWD(1); break;
    case 2: SPLAT_PBWD(2); break;
    default: SPLAT_PBWD(3); break;
  }
#undef SPLAT_PBWD
  c->launches.count++;
  SPLAT_LAUNCHED("project_bwd_kernel");
  return Status::ok();
}

Status launch_project_bwd(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                          const splat_proj_opts& opts, const float* proj, const float* pgrad, float* out,
                          void* stats, int absgrad) {
  return project_bwd_launch<false, false>(c, planes, n, cap, cam, opts, proj, pgrad, out, stats, absgrad, nullptr,
                                          nullptr, AdamArgs(), nullptr, nullptr, nullptr, false);
}

Status launch_project_bwd_adam(Ctx* c, float* planes, float* m, float* v, int64_t n, int64_t cap,
                               const splat_camera& cam, const splat_proj_opts& opts, const float* proj,
                               const float* pgrad, void* stats, int absgrad, uint64_t step, const splat_lr& lr,
                               const uint32_t* skip, const StepParams* sp, void* bf16, bool stats_maxg) {
  if (bf16)
    return project_bwd_launch<true, true>(c, planes, n, cap, cam, opts, proj, pgrad, nullptr, stats, absgrad, m, v,
                                          make_adam_args(step, lr), skip, sp, static_cast<uint2*>(bf16), stats_maxg);
  return project_bwd_launch<true, false>(c, planes, n, cap, cam, opts, proj, pgrad, nullptr, stats, absgrad, m, v,
                                         make_adam_args(step, lr), skip, sp, nullptr, stats_maxg);
}

// A batch's projection backward fused with one Adam step: for every view that sees the
// Gaussian (radius > 0) the view's 59 gradients (project_backward_one with that view's
// camera and screen-space gradient, already scaled by 1/views through dL/dpixel) are added,
// in view order, into a per-thread column of shared memory together with the view's
// densification statistics; Adam then updates the parameters once with the sum.
constexpr int kBatchBwdThreads = 128;

template <int DEG, bool BF16>
__global__ void __launch_bounds__(kBatchBwdThreads) project_bwd_batch_adam_kernel(
    float4* planes, int64_t n, int64_t cap, splat_proj_opts opts, const float4* __restrict__ rec,
    const float4* __restrict__ pgrad, int64_t pcap, float* __restrict__ stat_accum, uint32_t* __restrict__ stat_denom,
    uint32_t* __restrict__ stat_maxr, int absgrad, float4* __restrict__ adam_m, float4* __restrict__ adam_v,
    const uint32_t* __restrict__ skip, const BatchTable* __restrict__ bt, uint2* bf, float* __restrict__ stat_maxg) {
  __shared__ float acc[kPlanes * 4][kBatchBwdThreads];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (skip && *skip) return;
  const int tid = threadIdx.x;
#pragma unroll
  for (int f = 0; f < kPlanes * 4; f++) acc[f][tid] = 0.0f;
  GParams g;
  load_params<DEG, BF16>(planes, cap, i, g, bf);
  const int views = bt->views;
  for (int v = 0; v < views; v++) {
    const int64_t r = (int64_t)v * n + i;
    const uint32_t radius = fbits(rec[4 * r + 3].y);
    if (radius == 0) continue;  // not drawn in this view: zero gradient, no statistics
    const float4 g0 = pgrad[r], g1 = pgrad[pcap + r], g2 = pgrad[2 * pcap + r];
    const splat_camera cam = bt->cam[v];
    if (stat_accum != nullptr) {  // DensifyStats::accumulate per view (densify.rs:36-60)
      // The view's own gradient: dL/dpixel carried the batch's 1/views averaging.
      const float sx = (float)cam.width * 0.5f * (float)views;
      const float sy = (float)cam.height * 0.5f * (float)views;
      const float gx = (absgrad ? g2.y : g0.x) * sx;
      const float gy = (absgrad ? g2.z : g0.y) * sy;
      const float gn = sqrtf(gx * gx + gy * gy);
      stat_accum[i] += gn;
      stat_denom[i] += 1u;
      stat_maxr[i] = max(stat_maxr[i], radius);
      if (stat_maxg) {
        stat_maxg[i] = fmaxf(stat_maxg[i], gn);
        stat_maxg[cap + i] += g2.w;  // contribution: the view's blending weight sum (alpha T)
      }
    }
    ParamGrad pgr;
    proj_grad_one<DEG>(g, cam, opts, g0, g1, g2, pgr);
#pragma unroll
    for (int q = 0; q < 3; q++) acc[q][tid] += pgr.mean[q];
    acc[3][tid] += pgr.op;
#pragma unroll
    for (int q = 0; q < 4; q++) acc[4 + q][tid] += pgr.q[q];
#pragma unroll
    for (int q = 0; q < 3; q++) acc[8 + q][tid] += pgr.ls[q];
#pragma unroll
    for (int q = 0; q < 48; q++) acc[12 + q][tid] += pgr.sh[q];
  }
  const AdamArgs adam = bt->adam;
#pragma unroll
  for (int q = 0; q < kPlanes; q++) {
    const float4 gq = make_float4(acc[4 * q][tid], acc[4 * q + 1][tid], acc[4 * q + 2][tid], acc[4 * q + 3][tid]);
    const int64_t o = (int64_t)q * cap + i;
    float4 p = planes[o], m = adam_m[o], v = adam_v[o];
    adam_plane(adam, q, p, gq, m, v);
    planes[o] = p;
    adam_m[o] = m;
    adam_v[o] = v;
    if (BF16 && q > 0) bf[(int64_t)(q - 1) * cap + i] = pack_bf16x4(p);
  }
}

Status launch_project_bwd_batch_adam(Ctx* c, float* planes, float* m, float* v, int64_t n, int64_t cap,
                                     const splat_proj_opts& opts, const float* proj, const float* pgrad, int64_t pcap,
                                     void* stats, int absgrad, const uint32_t* skip, const BatchTable* bt,
                                     void* bf16, bool stats_maxg) {
  if (n == 0) return Status::ok();
  const uint32_t grid = ceil_div(n, kBatchBwdThreads);
  float4* p = reinterpret_cast<float4*>(planes);
  const float4* r = reinterpret_cast<const float4*>(proj);
  const float4* pg = reinterpret_cast<const float4*>(pgrad);
  float* sa = nullptr;
  uint32_t *sd = nullptr, *sm = nullptr;
  float* smg = nullptr;
  if (stats) {
    sa = reinterpret_cast<float*>(stats);
    sd = reinterpret_cast<uint32_t*>(sa + cap);
    sm = sd + cap;
    if (stats_maxg) smg = reinterpret_cast<float*>(sm + cap);
  }
  float4* am = reinterpret_cast<float4*>(m);
  float4* av = reinterpret_cast<float4*>(v);
  uint2* bf = static_cast<uint2*>(bf16);
#define SPLAT_PBB(D, B)                                                                                          \
  project_bwd_batch_adam_kernel<D, B><<<grid, kBatchBwdThreads, 0, c->stream>>>(p, n, cap, opts, r, pg, pcap, sa, sd, \
                                                                                 sm, absgrad, am, av, skip, bt, bf, smg)
  if (bf) {
    switch (opts.sh_degree) {
      case 0: SPLAT_PBB(0, true); break;
      case 1: SPLAT_PBB(1, true); break;
      case 2: SPLAT_PBB(2, true); break;
      default: SPLAT_PBB(3, true); break;
    }
  } else {
    switch (opts.sh_degree) {
      case 0: SPLAT_PBB(0, false); break;
      case 1: SPLAT_PBB(1, false); break;
      case 2: SPLAT_PBB(2, false); break;
      default: SPLAT_PBB(3, false); break;
    }
  }
#undef SPLAT_PBB
  c->launches.count++;
  SPLAT_LAUNCHED("project_bwd_batch_adam_kernel");
  return Status::ok();
}

__global__ void planes_to_bf16_kernel(const float4* __restrict__ planes, int64_t n, int64_t cap,
                                      uint2* __restrict__ bf) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)(kPlanes - 1) * n) return;
  const int q = 1 + (int)(t / n);
  const int64_t i = t - (int64_t)(q - 1) * n;
  bf[(int64_t)(q - 1) * cap + i] = pack_bf16x4(planes[(int64_t)q * cap + i]);
}

Status launch_planes_to_bf16(Ctx* c, const float* planes, int64_t n, int64_t cap, void* bf16) {
  if (n == 0) return Status::ok();
  planes_to_bf16_kernel<<<ceil_div((uint64_t)(kPlanes - 1) * n, 256), 256, 0, c->stream>>>(
      reinterpret_cast<const float4*>(planes), n, cap, static_cast<uint2*>(bf16));
  c->launches.count++;
  SPLAT_LAUNCHED("planes_to_bf16_kernel");
  return Status::ok();
}

Status launch_params_from_aos(Ctx* c, const float* aos, int64_t n, float* planes, int64_t cap) {
  if (n == 0) return Status::ok();
  aos_to_planes_kernel<<<ceil_div(n, kConvG), kConvG, 0, c->stream>>>(aos, n, reinterpret_cast<float4*>(planes), cap);
  c->launches.count++;
  SPLAT_LAUNCHED("aos_to_planes_kernel");
  return Status::ok();
}

Status launch_params_to_aos(Ctx* c, const float* planes, int64_t n, int64_t cap, float* aos) {
  if (n == 0) return Status::ok();
  planes_to_aos_kernel<<<ceil_div(n, kConvG), kConvG, 0, c->stream>>>(reinterpret_cast<const float4*>(planes), n, cap,
                                                                      aos);
  c->launches.count++;
  SPLAT_LAUNCHED("planes_to_aos_kernel");
  return Status::ok();
}

}  // namespace splat
