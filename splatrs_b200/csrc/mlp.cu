// The learned-densification network (no reference counterpart; it proposes, per Gaussian,
// one of {keep, clone/split, prune} beside the threshold rule of src/densify.rs:125-221):
// 16 features -> 64 SiLU -> 64 SiLU -> 3 logits -> softmax, BF16 operands on the tensor
// cores (mma.sync m16n8k16) with FP32 accumulation.
//
// Parameters are one FP32 vector (the optimiser's master copy): W1 [16][64], b1 [64],
// W2 [64][64], b2 [64], W3 [64][3], b3 [3] with W[in][out]. Each block rounds them to BF16
// into shared memory in the layouts the B operands want. A warp takes 16 Gaussians: the
// accumulator fragment of one layer is, repacked to BF16, the A fragment of the next, so
// the forward never leaves registers; the backward's transposed products (weight
// gradients) read the warp's activations back from shared memory. Rounding points match
// the oracle's bf16 mode: inputs, weights, hidden activations, and in the backward the
// logit gradient and hidden-layer gradients before each product; biases and their
// gradients stay FP32.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.cuh"

namespace splat {

namespace {
constexpr int kIn = 16, kHid = 64, kOut = 3;
constexpr int kW1 = 0, kB1 = kW1 + kIn * kHid, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid, kW3 = kB2 + kHid,
              kB3 = kW3 + kHid * kOut, kParams = kB3 + kOut;
constexpr int kWarps = 4, kThreads = 32 * kWarps, kRows = 16 * kWarps;

typedef __nv_bfloat16 bf;

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
  const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
  return a | (b << 16);
}
__device__ __forceinline__ uint32_t pack2h(bf lo, bf hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
__device__ __forceinline__ uint32_t ld2(const bf* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D = A (16x16, row) * B (16x8, col) + C, bf16 x bf16 -> f32.
__device__ __forceinline__ void mma16816(float d[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Shared memory: BF16 weights in operand layouts, FP32 biases, per-warp staging, FP32
// gradient accumulators (training only).
struct MlpSmem {
  bf w1t[kHid][kIn];    // layer 1 B: [n = out][k = in]
  bf w2t[kHid][kHid];   // layer 2 B: [out][in]
  bf w3t[8][kHid];      // layer 3 B: [out, padded to 8][in]
  bf w2[kHid][kHid];    // dh1 = dz2 W2^T, B: [n = in][k = out]
  bf w3[kHid][16];      // dh2 = dz3 W3^T, B: [n = in][k = out, padded to 16]
  float b1[kHid], b2[kHid], b3[8];
  bf x[kWarps][16][kIn];
  bf h1[kWarps][16][kHid];
  bf h2[kWarps][16][kHid];
  bf dz1[kWarps][16][kHid];
  bf dz2[kWarps][16][kHid];
  bf dz3[kWarps][16][8];
};

__device__ void load_weights(MlpSmem& s, const float* __restrict__ th) {
  for (int i = threadIdx.x; i < kIn * kHid; i += kThreads) {
    const int in = i / kHid, out = i % kHid;
    s.w1t[out][in] = __float2bfloat16_rn(th[kW1 + i]);
  }
  for (int i = threadIdx.x; i < kHid * kHid; i += kThreads) {
    const int in = i / kHid, out = i % kHid;
    const bf v = __float2bfloat16_rn(th[kW2 + i]);
    s.w2t[out][in] = v;
    s.w2[in][out] = v;
  }
  for (int i = threadIdx.x; i < 8 * kHid; i += kThreads) {
    const int out = i / kHid, in = i % kHid;
    s.w3t[out][in] = out < kOut ? __float2bfloat16_rn(th[kW3 + in * kOut + out]) : __float2bfloat16_rn(0.0f);
  }
  for (int i = threadIdx.x; i < kHid * 16; i += kThreads) {
    const int in = i / 16, out = i % 16;
    s.w3[in][out] = out < kOut ? __float2bfloat16_rn(th[kW3 + in * kOut + out]) : __float2bfloat16_rn(0.0f);
  }
  for (int i = threadIdx.x; i < kHid; i += kThreads) {
    s.b1[i] = th[kB1 + i];
    s.b2[i] = th[kB2 + i];
  }
  if (threadIdx.x < 8) s.b3[threadIdx.x] = threadIdx.x < kOut ? th[kB3 + threadIdx.x] : 0.0f;
}

// The forward of one warp's 16 rows. Outputs the pre-activations z1, z2 (accumulator
// layout, 8 column tiles of 8) and the logits z3 (one tile), and stages x, h1, h2 in
// shared memory for the backward.
__device__ __forceinline__ void mlp_forward_warp(MlpSmem& s, const float* __restrict__ x, int64_t row0, int64_t n,
                                                 float z1[8][4], float z2[8][4], float z3[4]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int64_t ra = row0 + g, rb = row0 + g + 8;
  float xa[4], xb[4];
#pragma unroll
  for (int q = 0; q < 2; q++)
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int col = 2 * t + 8 * q + e;
      xa[2 * q + e] = ra < n ? x[ra * kIn + col] : 0.0f;
      xb[2 * q + e] = rb < n ? x[rb * kIn + col] : 0.0f;
    }
  const uint32_t a0 = pack2(xa[0], xa[1]), a1 = pack2(xb[0], xb[1]), a2 = pack2(xa[2], xa[3]), a3 = pack2(xb[2], xb[3]);
  *reinterpret_cast<uint32_t*>(&s.x[warp][g][2 * t]) = a0;
  *reinterpret_cast<uint32_t*>(&s.x[warp][g + 8][2 * t]) = a1;
  *reinterpret_cast<uint32_t*>(&s.x[warp][g][2 * t + 8]) = a2;
  *reinterpret_cast<uint32_t*>(&s.x[warp][g + 8][2 * t + 8]) = a3;
  // Layer 1: 8 column tiles, one k-step.
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    mma16816(d, a0, a1, a2, a3, ld2(&s.w1t[8 * j + g][2 * t]), ld2(&s.w1t[8 * j + g][2 * t + 8]));
    const float c0 = s.b1[8 * j + 2 * t], c1 = s.b1[8 * j + 2 * t + 1];
    z1[j][0] = d[0] + c0;
    z1[j][1] = d[1] + c1;
    z1[j][2] = d[2] + c0;
    z1[j][3] = d[3] + c1;
  }
  // h1 = silu(z1) as BF16: A fragments of layer 2 and staged rows.
  uint32_t h[8][2];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    h[j][0] = pack2(silu(z1[j][0]), silu(z1[j][1]));
    h[j][1] = pack2(silu(z1[j][2]), silu(z1[j][3]));
    *reinterpret_cast<uint32_t*>(&s.h1[warp][g][8 * j + 2 * t]) = h[j][0];
    *reinterpret_cast<uint32_t*>(&s.h1[warp][g + 8][8 * j + 2 * t]) = h[j][1];
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kk = 0; kk < 4; kk++)
      mma16816(d, h[2 * kk][0], h[2 * kk][1], h[2 * kk + 1][0], h[2 * kk + 1][1],
               ld2(&s.w2t[8 * j + g][16 * kk + 2 * t]), ld2(&s.w2t[8 * j + g][16 * kk + 8 + 2 * t]));
    const float c0 = s.b2[8 * j + 2 * t], c1 = s.b2[8 * j + 2 * t + 1];
    z2[j][0] = d[0] + c0;
    z2[j][1] = d[1] + c1;
    z2[j][2] = d[2] + c0;
    z2[j][3] = d[3] + c1;
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    h[j][0] = pack2(silu(z2[j][0]), silu(z2[j][1]));
    h[j][1] = pack2(silu(z2[j][2]), silu(z2[j][3]));
    *reinterpret_cast<uint32_t*>(&s.h2[warp][g][8 * j + 2 * t]) = h[j][0];
    *reinterpret_cast<uint32_t*>(&s.h2[warp][g + 8][8 * j + 2 * t]) = h[j][1];
  }
  float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int kk = 0; kk < 4; kk++)
    mma16816(d, h[2 * kk][0], h[2 * kk][1], h[2 * kk + 1][0], h[2 * kk + 1][1], ld2(&s.w3t[g][16 * kk + 2 * t]),
             ld2(&s.w3t[g][16 * kk + 8 + 2 * t]));
  z3[0] = d[0] + s.b3[2 * t];
  z3[1] = d[1] + s.b3[2 * t + 1];
  z3[2] = d[2] + s.b3[2 * t];
  z3[3] = d[3] + s.b3[2 * t + 1];
}

// Softmax of the three logits of rows g and g + 8, gathered from lanes t = 0 (columns 0,
// 1) and t = 1 (column 2) of the quad.
__device__ __forceinline__ void softmax_rows(const float z3[4], float pa[3], float pb[3]) {
  const int lane = threadIdx.x & 31, q0 = lane & ~3;
  const float a0 = __shfl_sync(0xffffffffu, z3[0], q0), a1 = __shfl_sync(0xffffffffu, z3[1], q0);
  const float a2 = __shfl_sync(0xffffffffu, z3[0], q0 + 1);
  const float b0 = __shfl_sync(0xffffffffu, z3[2], q0), b1 = __shfl_sync(0xffffffffu, z3[3], q0);
  const float b2 = __shfl_sync(0xffffffffu, z3[2], q0 + 1);
  const float ma = fmaxf(a0, fmaxf(a1, a2)), mb = fmaxf(b0, fmaxf(b1, b2));
  const float ea0 = __expf(a0 - ma), ea1 = __expf(a1 - ma), ea2 = __expf(a2 - ma);
  const float eb0 = __expf(b0 - mb), eb1 = __expf(b1 - mb), eb2 = __expf(b2 - mb);
  const float sa = 1.0f / (ea0 + ea1 + ea2), sb = 1.0f / (eb0 + eb1 + eb2);
  pa[0] = ea0 * sa;
  pa[1] = ea1 * sa;
  pa[2] = ea2 * sa;
  pb[0] = eb0 * sb;
  pb[1] = eb1 * sb;
  pb[2] = eb2 * sb;
}

__global__ void __launch_bounds__(kThreads) mlp_forward_kernel(const float* __restrict__ x, int64_t n,
                                                                const float* __restrict__ theta,
                                                                float* __restrict__ prob) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(smem_raw);
  load_weights(s, theta);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int64_t row0 = (int64_t)blockIdx.x * kRows + 16 * warp;
  float z1[8][4], z2[8][4], z3[4];
  mlp_forward_warp(s, x, row0, n, z1, z2, z3);
  float pa[3], pb[3];
  softmax_rows(z3, pa, pb);
  if (t == 0) {
    if (row0 + g < n)
#pragma unroll
      for (int c = 0; c < 3; c++) prob[(row0 + g) * 3 + c] = pa[c];
    if (row0 + g + 8 < n)
#pragma unroll
      for (int c = 0; c < 3; c++) prob[(row0 + g + 8) * 3 + c] = pb[c];
  }
}

// Sum over the 16 rows of a column pair held in accumulator layout (rows g and g + 8 in
// this lane): reduce over g; lanes with g == 0 hold the column sums.
__device__ __forceinline__ void col_sums(float c0, float c1, float c2, float c3, float& s0, float& s1) {
  s0 = c0 + c2;
  s1 = c1 + c3;
#pragma unroll
  for (int o = 4; o < 32; o <<= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
}

// Gradient of  sum_s w_s * -log p_s[y_s] * scale  (scale = 1 / sum of weights) added into
// grad (FP32, parameter layout).
__global__ void __launch_bounds__(kThreads) mlp_grad_kernel(const float* __restrict__ x, const int32_t* __restrict__ y,
                                                             const float* __restrict__ w, int64_t n, float scale,
                                                             const float* __restrict__ theta,
                                                             float* __restrict__ grad) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(smem_raw);
  float* sg = reinterpret_cast<float*>(smem_raw + sizeof(MlpSmem));  // kParams accumulators
  load_weights(s, theta);
  for (int i = threadIdx.x; i < kParams; i += kThreads) sg[i] = 0.0f;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int64_t row0 = (int64_t)blockIdx.x * kRows + 16 * warp;
  const int64_t ra = row0 + g, rb = row0 + g + 8;
  float z1[8][4], z2[8][4], z3[4];
  mlp_forward_warp(s, x, row0, n, z1, z2, z3);
  float pa[3], pb[3];
  softmax_rows(z3, pa, pb);
  // dz3 = (p - onehot(y)) * w * scale for this lane's columns 2t, 2t + 1 (only 0..2 exist).
  const int ya = ra < n ? y[ra] : -1, yb = rb < n ? y[rb] : -1;
  const float wa = ra < n ? w[ra] * scale : 0.0f, wb = rb < n ? w[rb] * scale : 0.0f;
  float dz3[4];
#pragma unroll
  for (int e = 0; e < 2; e++) {
    const int col = 2 * t + e;
    dz3[e] = col < kOut ? (pa[col < kOut ? col : 0] - (ya == col ? 1.0f : 0.0f)) * wa : 0.0f;
    dz3[2 + e] = col < kOut ? (pb[col < kOut ? col : 0] - (yb == col ? 1.0f : 0.0f)) * wb : 0.0f;
  }
  const uint32_t d3a = pack2(dz3[0], dz3[1]), d3b = pack2(dz3[2], dz3[3]);
  *reinterpret_cast<uint32_t*>(&s.dz3[warp][g][2 * t]) = d3a;
  *reinterpret_cast<uint32_t*>(&s.dz3[warp][g + 8][2 * t]) = d3b;
  {
    float s0, s1;
    col_sums(dz3[0], dz3[1], dz3[2], dz3[3], s0, s1);
    if (g == 0) {
      if (2 * t < kOut) atomicAdd(&sg[kB3 + 2 * t], s0);
      if (2 * t + 1 < kOut) atomicAdd(&sg[kB3 + 2 * t + 1], s1);
    }
  }
  __syncwarp();
  // dW3[in][out] = h2^T dz3: four row tiles of 16 inputs, K = the 16 rows of the warp.
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const bf(*H)[kHid] = s.h2[warp];
    const bf(*D)[8] = s.dz3[warp];
    const uint32_t a0 = pack2h(H[2 * t][16 * i + g], H[2 * t + 1][16 * i + g]);
    const uint32_t a1 = pack2h(H[2 * t][16 * i + g + 8], H[2 * t + 1][16 * i + g + 8]);
    const uint32_t a2 = pack2h(H[2 * t + 8][16 * i + g], H[2 * t + 9][16 * i + g]);
    const uint32_t a3 = pack2h(H[2 * t + 8][16 * i + g + 8], H[2 * t + 9][16 * i + g + 8]);
    const uint32_t b0 = pack2h(D[2 * t][g], D[2 * t + 1][g]), b1 = pack2h(D[2 * t + 8][g], D[2 * t + 9][g]);
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    mma16816(d, a0, a1, a2, a3, b0, b1);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int out = 2 * t + e;
      if (out < kOut) {
        atomicAdd(&sg[kW3 + (16 * i + g) * kOut + out], d[e]);
        atomicAdd(&sg[kW3 + (16 * i + g + 8) * kOut + out], d[2 + e]);
      }
    }
  }
  // dh2 = dz3 W3^T (K = outputs padded to 16), then dz2 = dh2 * silu'(z2).
  float dz2[8][4];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    mma16816(d, d3a, d3b, 0u, 0u, ld2(&s.w3[8 * j + g][2 * t]), ld2(&s.w3[8 * j + g][2 * t + 8]));
#pragma unroll
    for (int e = 0; e < 4; e++) dz2[j][e] = d[e] * silu_grad(z2[j][e]);
  }
  uint32_t p2[8][2];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    p2[j][0] = pack2(dz2[j][0], dz2[j][1]);
    p2[j][1] = pack2(dz2[j][2], dz2[j][3]);
    *reinterpret_cast<uint32_t*>(&s.dz2[warp][g][8 * j + 2 * t]) = p2[j][0];
    *reinterpret_cast<uint32_t*>(&s.dz2[warp][g + 8][8 * j + 2 * t]) = p2[j][1];
    float s0, s1;
    col_sums(dz2[j][0], dz2[j][1], dz2[j][2], dz2[j][3], s0, s1);
    if (g == 0) {
      atomicAdd(&sg[kB2 + 8 * j + 2 * t], s0);
      atomicAdd(&sg[kB2 + 8 * j + 2 * t + 1], s1);
    }
  }
  __syncwarp();
  // dW2[in][out] = h1^T dz2.
#pragma unroll 1
  for (int i = 0; i < 4; i++) {
    const bf(*H)[kHid] = s.h1[warp];
    const bf(*D)[kHid] = s.dz2[warp];
    const uint32_t a0 = pack2h(H[2 * t][16 * i + g], H[2 * t + 1][16 * i + g]);
    const uint32_t a1 = pack2h(H[2 * t][16 * i + g + 8], H[2 * t + 1][16 * i + g + 8]);
    const uint32_t a2 = pack2h(H[2 * t + 8][16 * i + g], H[2 * t + 9][16 * i + g]);
    const uint32_t a3 = pack2h(H[2 * t + 8][16 * i + g + 8], H[2 * t + 9][16 * i + g + 8]);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint32_t b0 = pack2h(D[2 * t][8 * j + g], D[2 * t + 1][8 * j + g]);
      const uint32_t b1 = pack2h(D[2 * t + 8][8 * j + g], D[2 * t + 9][8 * j + g]);
      float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      mma16816(d, a0, a1, a2, a3, b0, b1);
      atomicAdd(&sg[kW2 + (16 * i + g) * kHid + 8 * j + 2 * t], d[0]);
      atomicAdd(&sg[kW2 + (16 * i + g) * kHid + 8 * j + 2 * t + 1], d[1]);
      atomicAdd(&sg[kW2 + (16 * i + g + 8) * kHid + 8 * j + 2 * t], d[2]);
      atomicAdd(&sg[kW2 + (16 * i + g + 8) * kHid + 8 * j + 2 * t + 1], d[3]);
    }
  }
  // dh1 = dz2 W2^T, then dz1 = dh1 * silu'(z1).
  float dz1[8][4];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kk = 0; kk < 4; kk++)
      mma16816(d, p2[2 * kk][0], p2[2 * kk][1], p2[2 * kk + 1][0], p2[2 * kk + 1][1],
               ld2(&s.w2[8 * j + g][16 * kk + 2 * t]), ld2(&s.w2[8 * j + g][16 * kk + 8 + 2 * t]));
#pragma unroll
    for (int e = 0; e < 4; e++) dz1[j][e] = d[e] * silu_grad(z1[j][e]);
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    *reinterpret_cast<uint32_t*>(&s.dz1[warp][g][8 * j + 2 * t]) = pack2(dz1[j][0], dz1[j][1]);
    *reinterpret_cast<uint32_t*>(&s.dz1[warp][g + 8][8 * j + 2 * t]) = pack2(dz1[j][2], dz1[j][3]);
    float s0, s1;
    col_sums(dz1[j][0], dz1[j][1], dz1[j][2], dz1[j][3], s0, s1);
    if (g == 0) {
      atomicAdd(&sg[kB1 + 8 * j + 2 * t], s0);
      atomicAdd(&sg[kB1 + 8 * j + 2 * t + 1], s1);
    }
  }
  __syncwarp();
  // dW1[in][out] = x^T dz1 (one row tile: the 16 inputs).
  {
    const bf(*X)[kIn] = s.x[warp];
    const bf(*D)[kHid] = s.dz1[warp];
    const uint32_t a0 = pack2h(X[2 * t][g], X[2 * t + 1][g]);
    const uint32_t a1 = pack2h(X[2 * t][g + 8], X[2 * t + 1][g + 8]);
    const uint32_t a2 = pack2h(X[2 * t + 8][g], X[2 * t + 9][g]);
    const uint32_t a3 = pack2h(X[2 * t + 8][g + 8], X[2 * t + 9][g + 8]);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint32_t b0 = pack2h(D[2 * t][8 * j + g], D[2 * t + 1][8 * j + g]);
      const uint32_t b1 = pack2h(D[2 * t + 8][8 * j + g], D[2 * t + 9][8 * j + g]);
      float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      mma16816(d, a0, a1, a2, a3, b0, b1);
      atomicAdd(&sg[kW1 + g * kHid + 8 * j + 2 * t], d[0]);
      atomicAdd(&sg[kW1 + g * kHid + 8 * j + 2 * t + 1], d[1]);
      atomicAdd(&sg[kW1 + (g + 8) * kHid + 8 * j + 2 * t], d[2]);
      atomicAdd(&sg[kW1 + (g + 8) * kHid + 8 * j + 2 * t + 1], d[3]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kParams; i += kThreads)
    if (sg[i] != 0.0f) atomicAdd(&grad[i], sg[i]);
}

__global__ void mlp_adam_kernel(float* __restrict__ theta, const float* __restrict__ grad, float* __restrict__ m,
                                float* __restrict__ v, float lr, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  const float gi = grad[i];
  m[i] = 0.9f * m[i] + 0.1f * gi;
  v[i] = 0.999f * v[i] + 0.001f * gi * gi;
  theta[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + 1e-8f);
}
}  // namespace

int mlp_num_params() { return kParams; }

Status launch_mlp_forward(Ctx* c, const float* x, int64_t n, const float* theta, float* prob) {
  if (n == 0) return Status::ok();
  const size_t smem = sizeof(MlpSmem);
  SPLAT_CUDA(cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  mlp_forward_kernel<<<ceil_div(n, kRows), kThreads, smem, c->stream>>>(x, n, theta, prob);
  c->launches.count++;
  SPLAT_LAUNCHED("mlp_forward_kernel");
  return Status::ok();
}

Status launch_mlp_grad(Ctx* c, const float* x, const int32_t* y, const float* w, int64_t n, float scale,
                       const float* theta, float* grad) {
  if (n == 0) return Status::ok();
  const size_t smem = sizeof(MlpSmem) + (size_t)kParams * 4;
  SPLAT_CUDA(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  mlp_grad_kernel<<<ceil_div(n, kRows), kThreads, smem, c->stream>>>(x, y, w, n, scale, theta, grad);
  c->launches.count++;
  SPLAT_LAUNCHED("mlp_grad_kernel");
  return Status::ok();
}

Status launch_mlp_adam(Ctx* c, float* theta, const float* grad, float* m, float* v, uint64_t step, float lr) {
  const float c1 = 1.0f - powf(0.9f, (float)step), c2 = 1.0f - powf(0.999f, (float)step);
  mlp_adam_kernel<<<ceil_div((uint64_t)kParams, 256), 256, 0, c->stream>>>(theta, grad, m, v, lr, c1, c2);
  c->launches.count++;
  SPLAT_LAUNCHED("mlp_adam_kernel");
  return Status::ok();
}

}  // namespace splat
