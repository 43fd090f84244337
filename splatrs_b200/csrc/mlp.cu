// The learned-densification network (no reference counterpart; it proposes, per Gaussian,
// one of {keep, clone/split, prune} beside the threshold rule of src/densify.rs:125-221):
// 16 features -> 64 SiLU -> 64 SiLU -> 3 logits -> softmax, BF16 operands on the tensor
// cores with FP32 accumulation, in two generations: mma.sync m16n8k16 kernels (forward and
// gradient, register fragments, below) and tcgen05 kernels (forward and gradient,
// accumulators in tensor memory, further down), which the trainer runs; both give the same
// results up to summation order.
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

#include <atomic>

#include "common.cuh"
#include "kernels.cuh"

namespace splat {

namespace {
constexpr int kIn = 16, kHid = 64, kOut = 3;
constexpr int kW1 = 0, kB1 = kW1 + kIn * kHid, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid, kW3 = kB2 + kHid,
              kB3 = kW3 + kHid * kOut, kParams = kB3 + kOut;
constexpr int kWarps = 4, kThreads = 32 * kWarps, kRows = 16 * kWarps;

typedef __nv_bfloat16 bf;

// Two values rounded to BF16 (nearest even) in one conversion: lo in the low half.
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
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

// The logistic function as 0.5 (1 + tanh(z / 2)) with the hardware tanh approximation (one
// special-function instruction where exp and a reciprocal take two; the epilogues are
// bound by that unit). Its error, about 2^-11 relative, sits below the BF16 rounding of the
// activations that follows.
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigmoid(float z) { return 0.5f + 0.5f * tanh_fast(0.5f * z); }
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = sigmoid(z);
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
// ---------------------------------------------------------------------------------------
// The forward on the 5th-generation tensor cores (tcgen05): CTAs of 4 warps over tiles of
// 128 Gaussians (M = 128, TMEM lane = row), operands in shared memory in the canonical
// K-major, no-swizzle layout (8-row x 16-byte core matrices; K-adjacent cores 128 bytes
// apart, row groups SBO apart), accumulators in 64 TMEM columns that each layer reuses once
// the previous epilogue has read them. One thread issues each layer's MMAs and
// commits them to an mbarrier; every thread waits on it (bounded: a timeout sets *err and
// skips to the end, which waits once more, also bounded, for the MMAs in flight and always
// frees the TMEM), reads its row with tcgen05.ld, applies bias and SiLU and writes the next
// layer's A operand back to shared memory.
// ---------------------------------------------------------------------------------------
constexpr int kTcRows = 128;
constexpr uint32_t kTmemCols = 64;

struct TcSmem {
  alignas(1024) unsigned char ax[kTcRows * kIn * 2];    // A layer 1: [128][16]
  alignas(1024) unsigned char ah[kTcRows * kHid * 2];   // A layers 2-3: [128][64]
  alignas(1024) unsigned char bw1[kHid * kIn * 2];      // B layer 1: [64 out][16 in]
  alignas(1024) unsigned char bw2[kHid * kHid * 2];     // B layer 2: [64 out][64 in]
  alignas(1024) unsigned char bw3[16 * kHid * 2];       // B layer 3: [16 out (3 used)][64 in]
  float b1[kHid], b2[kHid], b3[16];
  alignas(8) uint64_t mbar;
  uint32_t tmem_base;
};

// Byte offset of element (row, k) of a K-major operand with `kdim` columns.
__device__ __forceinline__ uint32_t core_off(int row, int k, int kdim) {
  return (uint32_t)((row >> 3) * (kdim / 8) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t sbo) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((128u >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // LBO 128 B, version 1, no swizzle
}

// kind::f16 instruction descriptor: BF16 A and B, F32 accumulator, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(a) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint32_t limit = 1u << 22) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  for (uint32_t it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive accumulator columns of this thread's row.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Hidden layer epilogue: this thread's row of the accumulator at column col0, plus bias,
// SiLU, rounded to BF16 into the A operand of the next layer.
__device__ __forceinline__ void hidden_epilogue(TcSmem& s, uint32_t tmem_row, uint32_t col0, const float* bias,
                                                int row) {
#pragma unroll
  for (int c = 0; c < kHid; c += 16) {
    float v[16];
    tmem_ld16(tmem_row + col0 + c, v);
#pragma unroll
    for (int h = 0; h < 16; h += 8) {  // one 16-byte core-matrix row per store
      uint32_t w[4];
#pragma unroll
      for (int i = 0; i < 4; i++)
        w[i] = pack2(silu(v[h + 2 * i] + bias[c + h + 2 * i]), silu(v[h + 2 * i + 1] + bias[c + h + 2 * i + 1]));
      *reinterpret_cast<uint4*>(s.ah + core_off(row, c + h, kHid)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// A 128-row tile of feature rows (512 float4, contiguous) into registers, coalesced:
// thread t holds float4s t, t + 128, t + 256 and t + 384 of the tile.
__device__ __forceinline__ void load_tile(const float* __restrict__ x, int64_t tile, int64_t n, float4 r[4]) {
  const float4* x4 = reinterpret_cast<const float4*>(x);
  const int64_t base = tile * kTcRows * (kIn / 4), lim = n * (kIn / 4);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int64_t i = base + threadIdx.x + kTcRows * q;
    r[q] = i < lim ? __ldcs(x4 + i) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// Persistent: a CTA lays the weights out once and loops over 128-row tiles with stride
// gridDim.x, loading the next tile's rows into registers while this tile's MMAs run.
__global__ void __launch_bounds__(kTcRows) mlp_forward_tc_kernel(const float* __restrict__ x, int64_t n,
                                                                  const float* __restrict__ th,
                                                                  float* __restrict__ prob,
                                                                  volatile uint32_t* __restrict__ err) {
  extern __shared__ unsigned char tc_raw[];
  TcSmem& s = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  if (tid == 0) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(&s.mbar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(&s.tmem_base);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // Weights, rounded to BF16, in the K-major operand layouts.
  for (int i = tid; i < kIn * kHid; i += kTcRows) {
    const int in = i / kHid, out = i % kHid;
    *reinterpret_cast<bf*>(s.bw1 + core_off(out, in, kIn)) = __float2bfloat16_rn(th[kW1 + i]);
  }
  for (int i = tid; i < kHid * kHid; i += kTcRows) {
    const int in = i / kHid, out = i % kHid;
    *reinterpret_cast<bf*>(s.bw2 + core_off(out, in, kHid)) = __float2bfloat16_rn(th[kW2 + i]);
  }
  for (int i = tid; i < 16 * kHid; i += kTcRows) {
    const int out = i / kHid, in = i % kHid;
    const float w = out < kOut ? th[kW3 + in * kOut + out] : 0.0f;
    *reinterpret_cast<bf*>(s.bw3 + core_off(out, in, kHid)) = __float2bfloat16_rn(w);
  }
  if (tid < kHid) {
    s.b1[tid] = th[kB1 + tid];
    s.b2[tid] = th[kB2 + tid];
  }
  if (tid < 16) s.b3[tid] = tid < kOut ? th[kB3 + tid] : 0.0f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem_base;
  const uint32_t tmem_row = tmem + ((uint32_t)(32 * warp) << 16);
  bool ok = true;
  uint32_t phase = 0;
  float4 xr[4];
  int64_t tile = blockIdx.x;
  if (tile < tiles) load_tile(x, tile, n, xr);
  for (; tile < tiles; tile += gridDim.x) {
    const int64_t row_g = tile * kTcRows + tid;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int f = tid + kTcRows * q;  // row f / 4, columns 4 (f % 4) .. + 3
      *reinterpret_cast<uint2*>(s.ax + core_off(f >> 2, (f & 3) * 4, kIn)) =
          make_uint2(pack2(xr[q].x, xr[q].y), pack2(xr[q].z, xr[q].w));
    }
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Layer 1: [128 x 16] x [16 x 64] into columns 0-63.
    if (tid == 0) {
      tc_mma(tmem, smem_desc(s.ax, 256), smem_desc(s.bw1, 256), idesc_bf16(kHid), 0u);
      tc_commit(&s.mbar);
    }
    if (tile + gridDim.x < tiles) load_tile(x, tile + gridDim.x, n, xr);
    ok = !__syncthreads_or(!mbar_wait(&s.mbar, phase));  // the block agrees
    if (!ok) break;
    phase ^= 1u;
    tc_fence_after();
    hidden_epilogue(s, tmem_row, 0, s.b1, tid);
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Layer 2: [128 x 64] x [64 x 64] into columns 0-63, four K-steps of 16.
    if (tid == 0) {
#pragma unroll
      for (int k = 0; k < 4; k++)
        tc_mma(tmem, smem_desc(s.ah + 256 * k, 1024), smem_desc(s.bw2 + 256 * k, 1024), idesc_bf16(kHid),
               k > 0 ? 1u : 0u);
      tc_commit(&s.mbar);
    }
    ok = !__syncthreads_or(!mbar_wait(&s.mbar, phase));
    if (!ok) break;
    phase ^= 1u;
    tc_fence_after();
    hidden_epilogue(s, tmem_row, 0, s.b2, tid);
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Layer 3: [128 x 64] x [64 x 16] into columns 0-15.
    if (tid == 0) {
#pragma unroll
      for (int k = 0; k < 4; k++)
        tc_mma(tmem, smem_desc(s.ah + 256 * k, 1024), smem_desc(s.bw3 + 256 * k, 1024), idesc_bf16(16),
               k > 0 ? 1u : 0u);
      tc_commit(&s.mbar);
    }
    ok = !__syncthreads_or(!mbar_wait(&s.mbar, phase));
    if (!ok) break;
    phase ^= 1u;
    tc_fence_after();
    float v[16];
    tmem_ld16(tmem_row, v);
    const float z0 = v[0] + s.b3[0], z1 = v[1] + s.b3[1], z2 = v[2] + s.b3[2];
    const float m = fmaxf(z0, fmaxf(z1, z2));
    const float e0 = __expf(z0 - m), e1 = __expf(z1 - m), e2 = __expf(z2 - m);
    const float inv = 1.0f / (e0 + e1 + e2);
    if (row_g < n) {
      prob[row_g * 3] = e0 * inv;
      prob[row_g * 3 + 1] = e1 * inv;
      prob[row_g * 3 + 2] = e2 * inv;
    }
  }
  if (!ok) {
    mbar_wait(&s.mbar, phase);  // the timed-out MMAs, before their TMEM is freed
    if (tid == 0) *err = 1u;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}
// ---------------------------------------------------------------------------------------
// The gradient on tcgen05: the forward of a 128-row tile as above with its layer outputs
// z1, z2, z3 kept in tensor memory, then
//   dh2 = dz3 W3^T and dh1 = dz2 W2^T     (M = the tile's rows, K-major operands), and
//   [dW2^T ; dW1^T] = [dz2 | dz1]^T [h1 | x]   and   dW3^T = [. | dz3 | .]^T h2,
// the weight gradients as two M = 128 products over the tile's rows (K), which read the
// same shared-memory buffers as MN-major operands: a buffer laid out K-major for one
// product is, core matrix for core matrix, the MN-major operand of the transposed one.
// dW2^T and dW1^T are the diagonal blocks of one 128 x 80 product; dW3^T is rows 64-66 of a
// 128 x 64 one whose A is the dz buffer while dz3 sits in its columns 64-79. Both
// accumulate in tensor memory over all of the CTA's tiles and reach global memory once.
// Bias gradients (unrounded dz) go through shared memory. Rounding points are those of the
// mma.sync kernel and the oracle's bf16 mode.
// ---------------------------------------------------------------------------------------
constexpr uint32_t kGradTmemCols = 512;
constexpr uint32_t kZ1 = 0, kZ2 = 64, kZ3 = 128, kDH = 160, kAcc3 = 224, kAccW = 288;
constexpr int kXH = 80;   // columns of the [h1 | x] buffer
constexpr int kDZ = 128;  // columns of the [dz2 | dz1] buffer (dz3 in 64-79 before dz1)

struct TcGradSmem {
  alignas(1024) unsigned char xh[kTcRows * kXH * 2];
  alignas(1024) unsigned char h2[kTcRows * kHid * 2];
  alignas(1024) unsigned char dz[kTcRows * kDZ * 2];
  alignas(1024) unsigned char w1t[kHid * kIn * 2];   // B of layer 1: [out][in], K = in
  alignas(1024) unsigned char w2t[kHid * kHid * 2];  // B of layer 2: [out][in]
  alignas(1024) unsigned char w3t[16 * kHid * 2];    // B of layer 3: [out (16)][in]
  alignas(1024) unsigned char w2n[kHid * kHid * 2];  // B of dh1 = dz2 W2^T: [in][out], K = out
  alignas(1024) unsigned char w3n[kHid * 16 * 2];    // B of dh2 = dz3 W3^T: [in][out (16)]
  float b1[kHid], b2[kHid], b3[16];
  float gb[kHid + kHid + 16];  // bias gradients: b1, b2, b3
  float f[kTcRows][kHid + 1];  // a tile's unrounded dz2 or dz1, for the column sums of the bias gradients
  alignas(8) uint64_t mbar;
  uint32_t tmem_base;
};

__host__ __device__ constexpr uint32_t idesc_bf16_major(uint32_t n, uint32_t a_mn, uint32_t b_mn) {
  return idesc_bf16(n) | (a_mn << 15) | (b_mn << 16);
}

__device__ __forceinline__ uint64_t smem_desc_lbo(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Reads 64 accumulator columns from col0 of this thread's row, adds the bias and writes
// SiLU of the sum, rounded to BF16, to columns 0..63 of a K-major buffer of kdim columns.
__device__ __forceinline__ void silu_to(unsigned char* buf, int kdim, uint32_t tmem_row, uint32_t col0,
                                        const float* bias, int row) {
#pragma unroll
  for (int c = 0; c < kHid; c += 16) {
    float v[16];
    tmem_ld16(tmem_row + col0 + c, v);
#pragma unroll
    for (int h = 0; h < 16; h += 8) {
      uint32_t w[4];
#pragma unroll
      for (int i = 0; i < 4; i++)
        w[i] = pack2(silu(v[h + 2 * i] + bias[c + h + 2 * i]), silu(v[h + 2 * i + 1] + bias[c + h + 2 * i + 1]));
      *reinterpret_cast<uint4*>(buf + core_off(row, c + h, kdim)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// dz = dh * SiLU'(z + bias) for 64 columns (dh at dh_col, z at z_col of this thread's row),
// rounded to BF16 into columns col_out.. of the dz buffer; the unrounded dz into row `row`
// of the staging tile f (a row past the batch has dz = 0: its weight is 0).
__device__ __forceinline__ void dz_to(TcGradSmem& s, uint32_t tmem_row, uint32_t dh_col, uint32_t z_col,
                                      const float* bias, int col_out, int row) {
#pragma unroll
  for (int c = 0; c < kHid; c += 16) {
    float d[16], z[16];
    tmem_ld16(tmem_row + dh_col + c, d);
    tmem_ld16(tmem_row + z_col + c, z);
#pragma unroll
    for (int i = 0; i < 16; i++) d[i] *= silu_grad(z[i] + bias[c + i]);
#pragma unroll
    for (int h = 0; h < 16; h += 8) {
      uint32_t w[4];
#pragma unroll
      for (int i = 0; i < 4; i++) w[i] = pack2(d[h + 2 * i], d[h + 2 * i + 1]);
      *reinterpret_cast<uint4*>(s.dz + core_off(row, col_out + c + h, kDZ)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
#pragma unroll
    for (int i = 0; i < 16; i++) s.f[row][c + i] = d[i];
  }
}

// This thread's share of the staging tile's column sums: column tid % 64 over half of the
// rows (conflict-free: the tile's rows are 65 floats apart).
__device__ __forceinline__ float column_half_sum(const TcGradSmem& s, int tid) {
  const int col = tid & (kHid - 1), r0 = (tid >> 6) * (kTcRows / 2);
  float acc = 0.0f;
#pragma unroll 8
  for (int r = 0; r < kTcRows / 2; r++) acc += s.f[r0 + r][col];
  return acc;
}

__global__ void __launch_bounds__(kTcRows) mlp_grad_tc_kernel(const float* __restrict__ x,
                                                               const int32_t* __restrict__ y,
                                                               const float* __restrict__ wgt, int64_t n, float scale,
                                                               const float* __restrict__ th, float* __restrict__ grad,
                                                               volatile uint32_t* __restrict__ err) {
  extern __shared__ unsigned char tc_raw[];
  TcGradSmem& s = *reinterpret_cast<TcGradSmem*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  if (tid == 0) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(&s.mbar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(&s.tmem_base);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(kGradTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  for (int i = tid; i < kIn * kHid; i += kTcRows) {
    const int in = i / kHid, out = i % kHid;
    *reinterpret_cast<bf*>(s.w1t + core_off(out, in, kIn)) = __float2bfloat16_rn(th[kW1 + i]);
  }
  for (int i = tid; i < kHid * kHid; i += kTcRows) {
    const int in = i / kHid, out = i % kHid;
    const bf v = __float2bfloat16_rn(th[kW2 + i]);
    *reinterpret_cast<bf*>(s.w2t + core_off(out, in, kHid)) = v;
    *reinterpret_cast<bf*>(s.w2n + core_off(in, out, kHid)) = v;
  }
  for (int i = tid; i < 16 * kHid; i += kTcRows) {
    const int out = i / kHid, in = i % kHid;
    const bf v = __float2bfloat16_rn(out < kOut ? th[kW3 + in * kOut + out] : 0.0f);
    *reinterpret_cast<bf*>(s.w3t + core_off(out, in, kHid)) = v;
    *reinterpret_cast<bf*>(s.w3n + core_off(in, out, 16)) = v;
  }
  if (tid < kHid) {
    s.b1[tid] = th[kB1 + tid];
    s.b2[tid] = th[kB2 + tid];
  }
  if (tid < 16) s.b3[tid] = tid < kOut ? th[kB3 + tid] : 0.0f;
  for (int i = tid; i < kHid + kHid + 16; i += kTcRows) s.gb[i] = 0.0f;
  for (int i = tid; i < kTcRows * kDZ / 8; i += kTcRows) reinterpret_cast<uint4*>(s.dz)[i] = make_uint4(0, 0, 0, 0);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem_base;
  const uint32_t tmem_row = tmem + ((uint32_t)(32 * warp) << 16);
  bool ok = true, first = true;
  uint32_t phase = 0;
  float gacc1 = 0.0f, gacc2 = 0.0f;  // this thread's share of the b1 and b2 gradients
  float4 xr[4];
  int64_t tile = blockIdx.x;
  if (tile < tiles) load_tile(x, tile, n, xr);
  // One wait for the MMAs committed by thread 0; the whole block agrees on the outcome.
#define SPLAT_TC_WAIT()                                          \
  do {                                                           \
    ok = !__syncthreads_or(!mbar_wait(&s.mbar, phase));          \
    if (!ok) goto done;                                          \
    phase ^= 1u;                                                 \
    tc_fence_after();                                            \
  } while (0)
#define SPLAT_TC_HANDOFF()  \
  do {                      \
    async_proxy_fence();    \
    tc_fence_before();      \
    __syncthreads();        \
    tc_fence_after();       \
  } while (0)
  for (; tile < tiles; tile += gridDim.x) {
    const int64_t row_g = tile * kTcRows + tid;
    const bool live = row_g < n;
    const int yl = live ? y[row_g] : -1;
    const float wl = live ? wgt[row_g] * scale : 0.0f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int f = tid + kTcRows * q;
      *reinterpret_cast<uint2*>(s.xh + core_off(f >> 2, kHid + (f & 3) * 4, kXH)) =
          make_uint2(pack2(xr[q].x, xr[q].y), pack2(xr[q].z, xr[q].w));
    }
    SPLAT_TC_HANDOFF();
    if (tid == 0) {  // z1 = x W1
      tc_mma(tmem + kZ1, smem_desc_lbo(s.xh + 8 * 128, 128, kXH / 8 * 128), smem_desc(s.w1t, 256), idesc_bf16(kHid),
             0u);
      tc_commit(&s.mbar);
    }
    if (tile + gridDim.x < tiles) load_tile(x, tile + gridDim.x, n, xr);
    SPLAT_TC_WAIT();
    silu_to(s.xh, kXH, tmem_row, kZ1, s.b1, tid);  // h1 into columns 0-63
    SPLAT_TC_HANDOFF();
    if (tid == 0) {  // z2 = h1 W2
#pragma unroll
      for (int k = 0; k < 4; k++)
        tc_mma(tmem + kZ2, smem_desc_lbo(s.xh + 256 * k, 128, kXH / 8 * 128), smem_desc(s.w2t + 256 * k, 1024),
               idesc_bf16(kHid), k > 0 ? 1u : 0u);
      tc_commit(&s.mbar);
    }
    SPLAT_TC_WAIT();
    silu_to(s.h2, kHid, tmem_row, kZ2, s.b2, tid);
    SPLAT_TC_HANDOFF();
    if (tid == 0) {  // z3 = h2 W3
#pragma unroll
      for (int k = 0; k < 4; k++)
        tc_mma(tmem + kZ3, smem_desc(s.h2 + 256 * k, 1024), smem_desc(s.w3t + 256 * k, 1024), idesc_bf16(16),
               k > 0 ? 1u : 0u);
      tc_commit(&s.mbar);
    }
    SPLAT_TC_WAIT();
    {  // softmax and dz3 = (p - onehot(y)) w scale, into dz columns 64-79
      float v[16];
      tmem_ld16(tmem_row + kZ3, v);
      const float z0 = v[0] + s.b3[0], z1 = v[1] + s.b3[1], z2 = v[2] + s.b3[2];
      const float m = fmaxf(z0, fmaxf(z1, z2));
      const float e0 = __expf(z0 - m), e1 = __expf(z1 - m), e2 = __expf(z2 - m);
      const float inv = 1.0f / (e0 + e1 + e2);
      const float d0 = (e0 * inv - (yl == 0 ? 1.0f : 0.0f)) * wl;
      const float d1 = (e1 * inv - (yl == 1 ? 1.0f : 0.0f)) * wl;
      const float d2 = (e2 * inv - (yl == 2 ? 1.0f : 0.0f)) * wl;
      *reinterpret_cast<uint4*>(s.dz + core_off(tid, kHid, kDZ)) = make_uint4(pack2(d0, d1), pack2(d2, 0.0f), 0u, 0u);
      *reinterpret_cast<uint4*>(s.dz + core_off(tid, kHid + 8, kDZ)) = make_uint4(0u, 0u, 0u, 0u);
      float r0 = d0, r1 = d1, r2 = d2;  // b3 gradient: the warp's sums, one atomic each
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        r0 += __shfl_xor_sync(0xffffffffu, r0, o);
        r1 += __shfl_xor_sync(0xffffffffu, r1, o);
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
      }
      if ((tid & 31) == 0) {
        atomicAdd(&s.gb[2 * kHid], r0);
        atomicAdd(&s.gb[2 * kHid + 1], r1);
        atomicAdd(&s.gb[2 * kHid + 2], r2);
      }
    }
    SPLAT_TC_HANDOFF();
    if (tid == 0) {
      // dh2 = dz3 W3^T (K = 16 outputs, 3 used)
      tc_mma(tmem + kDH, smem_desc_lbo(s.dz + 8 * 128, 128, kDZ / 8 * 128), smem_desc(s.w3n, 256), idesc_bf16(kHid),
             0u);
      // dW3^T += (dz columns)^T h2 over the tile's rows: A MN-major (M = 128 columns), B MN-major (N = 64)
#pragma unroll
      for (int k = 0; k < kTcRows / 16; k++)
        tc_mma(tmem + kAcc3, smem_desc_lbo(s.dz + 2 * k * (kDZ / 8 * 128), kDZ / 8 * 128, 128),
               smem_desc_lbo(s.h2 + 2 * k * 1024, 1024, 128), idesc_bf16_major(kHid, 1u, 1u),
               (first && k == 0) ? 0u : 1u);
      tc_commit(&s.mbar);
    }
    SPLAT_TC_WAIT();
    dz_to(s, tmem_row, kDH, kZ2, s.b2, 0, tid);  // dz2 into columns 0-63
    SPLAT_TC_HANDOFF();
    if (tid == 0) {  // dh1 = dz2 W2^T
#pragma unroll
      for (int k = 0; k < 4; k++)
        tc_mma(tmem + kDH, smem_desc_lbo(s.dz + 256 * k, 128, kDZ / 8 * 128), smem_desc(s.w2n + 256 * k, 1024),
               idesc_bf16(kHid), k > 0 ? 1u : 0u);
      tc_commit(&s.mbar);
    }
    gacc2 += column_half_sum(s, tid);  // while the MMAs run
    SPLAT_TC_WAIT();
    dz_to(s, tmem_row, kDH, kZ1, s.b1, kHid, tid);  // dz1 into columns 64-127
    SPLAT_TC_HANDOFF();
    if (tid == 0) {  // [dW2^T ; dW1^T] += [dz2 | dz1]^T [h1 | x]
#pragma unroll
      for (int k = 0; k < kTcRows / 16; k++)
        tc_mma(tmem + kAccW, smem_desc_lbo(s.dz + 2 * k * (kDZ / 8 * 128), kDZ / 8 * 128, 128),
               smem_desc_lbo(s.xh + 2 * k * (kXH / 8 * 128), kXH / 8 * 128, 128), idesc_bf16_major(kXH, 1u, 1u),
               (first && k == 0) ? 0u : 1u);
      tc_commit(&s.mbar);
    }
    gacc1 += column_half_sum(s, tid);
    SPLAT_TC_WAIT();  // the buffers are free for the next tile
    first = false;
  }
  if (!first) {  // this CTA's accumulated weight gradients, once
    if (warp == 2) {  // dW3^T rows 64-66: lanes 0-2
#pragma unroll
      for (int c = 0; c < kHid; c += 16) {
        float v[16];
        tmem_ld16(tmem_row + kAcc3 + c, v);
        const int out = tid - 2 * 32;
        if (out < kOut)
#pragma unroll
          for (int i = 0; i < 16; i++) atomicAdd(&grad[kW3 + (c + i) * kOut + out], v[i]);
      }
    }
    if (warp < 2) {  // dW2^T rows 0-63, columns 0-63
#pragma unroll
      for (int c = 0; c < kHid; c += 16) {
        float v[16];
        tmem_ld16(tmem_row + kAccW + c, v);
#pragma unroll
        for (int i = 0; i < 16; i++) atomicAdd(&grad[kW2 + (c + i) * kHid + tid], v[i]);
      }
    } else {  // dW1^T rows 64-127, columns 64-79
      float v[16];
      tmem_ld16(tmem_row + kAccW + kHid, v);
#pragma unroll
      for (int i = 0; i < 16; i++) atomicAdd(&grad[kW1 + i * kHid + (tid - kHid)], v[i]);
    }
    atomicAdd(&s.gb[tid & (kHid - 1)], gacc1);
    atomicAdd(&s.gb[kHid + (tid & (kHid - 1))], gacc2);
    __syncthreads();
    for (int i = tid; i < kHid; i += kTcRows) {
      atomicAdd(&grad[kB1 + i], s.gb[i]);
      atomicAdd(&grad[kB2 + i], s.gb[kHid + i]);
    }
    if (tid < kOut) atomicAdd(&grad[kB3 + tid], s.gb[2 * kHid + tid]);
  }
done:
  if (!ok) {
    mbar_wait(&s.mbar, phase);  // the timed-out MMAs, before their TMEM is freed
    if (tid == 0) *err = 1u;
  }
#undef SPLAT_TC_WAIT
#undef SPLAT_TC_HANDOFF
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kGradTmemCols) : "memory");
  }
}
}  // namespace

int mlp_num_params() { return kParams; }

Status launch_mlp_forward_tc(Ctx* c, const float* x, int64_t n, const float* theta, float* prob, uint32_t* err) {
  if (n == 0) return Status::ok();
  const size_t smem = sizeof(TcSmem) + 1024;
  SPLAT_CUDA(cudaFuncSetAttribute(mlp_forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, sms = 0, smem_sm = 0, smem_rsv = 0;
  SPLAT_CUDA(cudaGetDevice(&dev));
  SPLAT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  SPLAT_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  SPLAT_CUDA(cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
  // As many CTAs as fit at once: shared memory, and 512 / 64 tensor-memory columns.
  const int per_sm = std::max(1, std::min<int>(smem_sm / (int)(smem + smem_rsv), 512 / (int)kTmemCols));
  const int64_t grid = std::min<int64_t>(ceil_div(n, kTcRows), (int64_t)per_sm * sms);
  mlp_forward_tc_kernel<<<(unsigned)grid, kTcRows, smem, c->stream>>>(x, n, theta, prob, err);
  c->launches.count++;
  SPLAT_LAUNCHED("mlp_forward_tc_kernel");
  return Status::ok();
}

Status mlp_forward_tc_checked(Ctx* c, const float* x, int64_t n, const float* theta, float* prob) {
  volatile uint32_t* h = reinterpret_cast<volatile uint32_t*>(c->host_small) + kTcErrWord;
  *h = 0u;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  SPLAT_TRY(launch_mlp_forward_tc(c, x, n, theta, prob, reinterpret_cast<uint32_t*>(c->host_small_dev) + kTcErrWord));
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  if (*h != 0u) return Status::make(SPLAT_ERR_TIMEOUT, "mlp_forward_tc: a wait for the tensor cores timed out");
  return Status::ok();
}

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

Status launch_mlp_grad_tc(Ctx* c, const float* x, const int32_t* y, const float* w, int64_t n, float scale,
                          const float* theta, float* grad, uint32_t* err) {
  if (n == 0) return Status::ok();
  const size_t smem = sizeof(TcGradSmem) + 1024;
  SPLAT_CUDA(cudaFuncSetAttribute(mlp_grad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, sms = 0;
  SPLAT_CUDA(cudaGetDevice(&dev));
  SPLAT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // One CTA per SM: each holds all 512 tensor-memory columns.
  const int64_t grid = std::min<int64_t>(ceil_div(n, kTcRows), (int64_t)sms);
  mlp_grad_tc_kernel<<<(unsigned)grid, kTcRows, smem, c->stream>>>(x, y, w, n, scale, theta, grad, err);
  c->launches.count++;
  SPLAT_LAUNCHED("mlp_grad_tc_kernel");
  return Status::ok();
}

// Diagnostic of the bounded wait and of the error word the tensor-core kernels report in:
// one block waits, with `limit` tries, on an mbarrier that nothing arrives on (arrive == 0),
// or that one thread has completed first (arrive != 0). When the wait runs out the block
// reports it exactly as the tensor-core kernels do, completes the phase itself and
// invalidates the barrier before it exits.
__global__ void diag_mbar_wait_kernel(uint32_t limit, int arrive, uint32_t* err) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (arrive && threadIdx.x == 0)
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(a) : "memory");
  const bool ok = !__syncthreads_or(!mbar_wait(&bar, 0u, limit));
  if (threadIdx.x == 0) {
    if (!ok) {
      *err = 1u;
      asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(a) : "memory");
    }
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(a) : "memory");
  }
}

Status diag_mbar_wait(Ctx* c, uint32_t limit, int arrive) {
  SPLAT_TRY(mlp_tc_error_clear(c));
  diag_mbar_wait_kernel<<<1, 32, 0, c->stream>>>(limit, arrive, mlp_tc_error_word(c));
  c->launches.count++;
  SPLAT_LAUNCHED("diag_mbar_wait_kernel");
  SPLAT_CUDA(cudaGetLastError());
  return mlp_tc_error_check(c);
}

Status mlp_tc_error_clear(Ctx* c) {
  volatile uint32_t* h = reinterpret_cast<volatile uint32_t*>(c->host_small) + kTcErrWord;
  *h = 0u;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  return Status::ok();
}

uint32_t* mlp_tc_error_word(Ctx* c) { return reinterpret_cast<uint32_t*>(c->host_small_dev) + kTcErrWord; }

Status mlp_tc_error_check(Ctx* c) {
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  volatile uint32_t* h = reinterpret_cast<volatile uint32_t*>(c->host_small) + kTcErrWord;
  if (*h != 0u) return Status::make(SPLAT_ERR_TIMEOUT, "tcgen05 network kernel: a wait for the tensor cores timed out");
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
