// Adam::step (reference src/adam.rs:44-161) on one float4 of a parameter plane, shared by
// the stand-alone optimiser kernel and the projection backward that applies it in place.
#pragma once
#include "common.cuh"

namespace splat {

struct AdamArgs {
  float lr[4][4];  // per lane of planes 0..3; planes >= 4 use sh_rest
  float sh_rest;
  float b1, b2, c1, c2, eps;
};

// adam.rs:44-61, in the reference's operation order (compiled without contraction).
__device__ __forceinline__ void adam_update(float& p, float g, float& m, float& v, float lr, float b1, float b2,
                                            float c1, float c2, float eps) {
  m = b1 * m + (1.0f - b1) * g;
  v = b2 * v + (1.0f - b2) * g * g;
  const float m_hat = m / c1;
  const float v_hat = v / c2;
  p -= lr * m_hat / (sqrtf(v_hat) + eps);
}

// One float4 of plane `plane` with the learning rate of each lane's parameter group.
__device__ __forceinline__ void adam_plane(const AdamArgs& a, int plane, float4& p, const float4& g, float4& m,
                                           float4& v) {
  float lr0, lr1, lr2, lr3;
  if (plane < 4) {
    lr0 = a.lr[plane][0];
    lr1 = a.lr[plane][1];
    lr2 = a.lr[plane][2];
    lr3 = a.lr[plane][3];
  } else {
    lr0 = lr1 = lr2 = lr3 = a.sh_rest;
  }
  adam_update(p.x, g.x, m.x, v.x, lr0, a.b1, a.b2, a.c1, a.c2, a.eps);
  adam_update(p.y, g.y, m.y, v.y, lr1, a.b1, a.b2, a.c1, a.c2, a.eps);
  adam_update(p.z, g.z, m.z, v.z, lr2, a.b1, a.b2, a.c1, a.c2, a.eps);
  adam_update(p.w, g.w, m.w, v.w, lr3, a.b1, a.b2, a.c1, a.c2, a.eps);
}

// Bias corrections for step `step` (after the increment) and the per-lane rates.
AdamArgs make_adam_args(uint64_t step, const splat_lr& lr);

}  // namespace splat
