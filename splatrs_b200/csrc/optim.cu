// Optimiser and density control on the parameter planes:
//   adam_kernel        Adam::step (reference src/adam.rs:44-161), one float4 per thread;
//   densify_mark       the clone / split / prune decisions of densify_and_prune
//                      (src/densify.rs:125-221) and their counts;
//   densify_scatter    the compaction that writes survivors, clones and split children in
//                      the reference's order (originals, clones, children) with their Adam
//                      state (kept for survivors, zero for new Gaussians, adam.rs:164-173);
//   reset_opacity      reset_opacity (src/densify.rs:224-230).
// All arithmetic keeps the reference's operation order (compiled without contraction), so
// the updated parameters are bit-identical to the reference's given the same inputs.
#include "common.cuh"
#include "kernels.cuh"
#include "adam.cuh"

namespace splat {

__global__ void __launch_bounds__(256) adam_kernel(float4* __restrict__ p, const float4* __restrict__ g,
                                                   float4* __restrict__ m, float4* __restrict__ v, int64_t n,
                                                   int64_t cap, AdamArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)kPlanes * n;
  if (t >= total) return;
  const int plane = (int)(t / n);
  const int64_t i = t - (int64_t)plane * n;
  const int64_t o = (int64_t)plane * cap + i;
  float4 pp = p[o], gg = g[o], mm = m[o], vv = v[o];
  adam_plane(a, plane, pp, gg, mm, vv);
  p[o] = pp;
  m[o] = mm;
  v[o] = vv;
}

// Right-to-left binary exponentiation, as Rust's powi lowers to.
static float powi_f(float a, int b) {
  const bool recip = b < 0;
  float r = 1.0f;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0f / r : r;
}

AdamArgs make_adam_args(uint64_t step, const splat_lr& lr) {
  AdamArgs a;
  a.b1 = 0.9f;
  a.b2 = 0.999f;
  a.eps = 1e-15f;
  a.c1 = 1.0f - powi_f(a.b1, (int)step);
  a.c2 = 1.0f - powi_f(a.b2, (int)step);
  // Plane 0: mean x y z, opacity; plane 1: quat; plane 2: log-scale x y z, pad;
  // plane 3: sh[0][0..3] (DC) and sh[1][0] (rest).
  const float L[4][4] = {{lr.mean, lr.mean, lr.mean, lr.opacity},
                         {lr.quat, lr.quat, lr.quat, lr.quat},
                         {lr.log_scale, lr.log_scale, lr.log_scale, lr.log_scale},
                         {lr.sh_dc, lr.sh_dc, lr.sh_dc, lr.sh_rest}};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) a.lr[i][j] = L[i][j];
  a.sh_rest = lr.sh_rest;
  return a;
}

Status launch_adam(Ctx* c, float* params, const float* grads, float* m, float* v, int64_t n, int64_t cap,
                   uint64_t step, const splat_lr& lr) {
  if (n == 0) return Status::ok();
  const AdamArgs a = make_adam_args(step, lr);
  const int64_t total = (int64_t)kPlanes * n;
  adam_kernel<<<ceil_div(total, 256), 256, 0, c->stream>>>(reinterpret_cast<float4*>(params),
                                                           reinterpret_cast<const float4*>(grads),
                                                           reinterpret_cast<float4*>(m), reinterpret_cast<float4*>(v),
                                                           n, cap, a);
  c->launches.count++;
  SPLAT_LAUNCHED("adam_kernel");
  return Status::ok();
}

// ---------------------------------------------------------------------------------------
// Densification
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ float max_scale_of(float ls0, float ls1, float ls2) {
  // Gaussian::scales().max_elem() (model.rs:37-39, math.rs:149)
  return fmaxf(fmaxf(crm::expf_cr(ls0), crm::expf_cr(ls1)), crm::expf_cr(ls2));
}

__device__ __forceinline__ float alpha_of(float logit) { return 1.0f / (1.0f + crm::expf_cr(-logit)); }

// Flags per original Gaussian: bit 0 keep original, bit 1 clone exists, bit 2 clone kept,
// bit 3 split, bits 4.. keep child j (4 + j). Counts: [0] kept originals, [1] clones,
// [2] kept clones, [3] splits, [4] kept children, [5] pruned.
__global__ void densify_mark_kernel(const float4* __restrict__ p, int64_t n, int64_t cap,
                                    const float* __restrict__ accum, const uint32_t* __restrict__ denom,
                                    const uint32_t* __restrict__ maxr, DensifyArgs a, uint32_t* __restrict__ flags,
                                    uint32_t* __restrict__ keep_orig, uint32_t* __restrict__ keep_clone,
                                    uint32_t* __restrict__ split_flag, uint32_t* __restrict__ keep_child,
                                    unsigned long long* __restrict__ counts) {
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i0 < n;
  const int64_t i = valid ? i0 : 0;
  const float4 p0 = p[i], p2 = p[2 * cap + i];
  const float g = denom[i] > 0 ? accum[i] / (float)denom[i] : 0.0f;  // densify.rs:135-143
  const float ms = max_scale_of(p2.x, p2.y, p2.z);
  bool hot = a.grow && g >= a.grad_threshold;
  const float alpha = alpha_of(p0.w);
  float p_prune = 0.0f;
  if (a.policy && valid) {
    const float pk = a.policy[3 * i], pc = a.policy[3 * i + 1];
    p_prune = a.policy[3 * i + 2];
    if (hot && pk > pc && pk >= 0.6f) hot = false;  // the network vetoes this densification
  }
  const bool clone = hot && ms <= a.size_limit;
  const bool split = hot && ms > a.size_limit;
  // Prune rules (densify.rs:203-215) for the original, its clone and its children.
  bool prune_o = alpha < a.min_opacity;
  bool prune_c = prune_o;
  if (a.prune_big_world) {
    prune_o |= ms > a.big_world_limit;
    prune_c = prune_o;
  }
  if (a.max_screen_size >= 0) prune_o |= (int64_t)maxr[i] > a.max_screen_size;
  if (a.policy && p_prune >= a.prune_conf) prune_o = true;
  if (a.action && valid) a.action[i] = (prune_o && !split) ? 2u : ((clone || split) ? 1u : 0u);
  uint32_t f = 0, kc = 0;
  const bool ko = !split && !prune_o;
  if (ko) f |= 1u;
  if (clone) {
    f |= 2u;
    if (!prune_c) f |= 4u;
  }
  if (split) {
    f |= 8u;
    // A child's scale is the parent's shrunk by exp(-shrink) on every axis.
    bool prune_k = alpha < a.min_opacity;
    if (a.prune_big_world) prune_k |= max_scale_of(p2.x - a.shrink, p2.y - a.shrink, p2.z - a.shrink) > a.big_world_limit;
    if (!prune_k) {
      for (int j = 0; j < a.children; j++) f |= 1u << (4 + j);
      kc = (uint32_t)a.children;
    }
  }
  uint32_t pruned = 0;
  if (!split && prune_o) pruned++;
  if (clone && prune_c) pruned++;
  if (split && kc == 0) pruned += (uint32_t)a.children;
  if (valid) {
    flags[i] = f;
    keep_orig[i] = ko ? 1u : 0u;
    keep_clone[i] = (f & 4u) ? 1u : 0u;
    split_flag[i] = split ? 1u : 0u;
    keep_child[i] = kc;
  }
  // Warp-aggregated counts.
  const uint32_t v[6] = {valid && ko ? 1u : 0u, valid && clone ? 1u : 0u, valid && (f & 4u) ? 1u : 0u,
                         valid && split ? 1u : 0u, valid ? kc : 0u, valid ? pruned : 0u};
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const uint32_t s = __reduce_add_sync(0xffffffffu, v[q]);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&counts[q], (unsigned long long)s);
  }
}

// Copies survivors and writes clones and children into the new arrays. Offsets are the
// exclusive scans of keep_orig, keep_clone, split_flag and keep_child.
__global__ void densify_scatter_kernel(const float4* __restrict__ p, const float4* __restrict__ m,
                                       const float4* __restrict__ v, int64_t n, int64_t cap,
                                       const uint32_t* __restrict__ flags, const uint32_t* __restrict__ off_orig,
                                       const uint32_t* __restrict__ off_clone, const uint32_t* __restrict__ off_split,
                                       const uint32_t* __restrict__ off_child, uint32_t n_orig, uint32_t n_clone,
                                       const double* __restrict__ normals, DensifyArgs a, float4* __restrict__ po,
                                       float4* __restrict__ mo, float4* __restrict__ vo, int64_t cap_out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t f = flags[i];
  if (f & 1u) {
    const int64_t d = off_orig[i];
    for (int q = 0; q < kPlanes; q++) {
      po[q * cap_out + d] = p[q * cap + i];
      mo[q * cap_out + d] = m[q * cap + i];
      vo[q * cap_out + d] = v[q * cap + i];
    }
    if (a.origin_out) a.origin_out[d] = (uint32_t)i;
    if (a.birth_out) a.birth_out[d] = a.birth_in ? a.birth_in[i] : 0u;
  }
  const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (f & 4u) {
    const int64_t d = (int64_t)n_orig + off_clone[i];
    for (int q = 0; q < kPlanes; q++) {
      po[q * cap_out + d] = p[q * cap + i];
      mo[q * cap_out + d] = z;
      vo[q * cap_out + d] = z;
    }
    if (a.origin_out) a.origin_out[d] = (uint32_t)i;
    if (a.birth_out) a.birth_out[d] = a.birth_now;
  }
  if ((f & 8u) && (f >> 4)) {
    const float4 p0 = p[i], p1 = p[cap + i], p2 = p[2 * cap + i];
    const float s0 = crm::expf_cr(p2.x), s1 = crm::expf_cr(p2.y), s2 = crm::expf_cr(p2.z);
    // Rotation of the normalised quaternion (math.rs:353-389).
    const float qn = sqrtf(p1.x * p1.x + p1.y * p1.y + p1.z * p1.z + p1.w * p1.w);
    float w, x, y, zq;
    if (qn > 0.0f) {
      w = p1.x / qn;
      x = p1.y / qn;
      y = p1.z / qn;
      zq = p1.w / qn;
    } else {
      w = 1.0f;
      x = y = zq = 0.0f;
    }
    float R[3][3];
    R[0][0] = 1.0f - 2.0f * (y * y + zq * zq);
    R[0][1] = 2.0f * (x * y - w * zq);
    R[0][2] = 2.0f * (x * zq + w * y);
    R[1][0] = 2.0f * (x * y + w * zq);
    R[1][1] = 1.0f - 2.0f * (x * x + zq * zq);
    R[1][2] = 2.0f * (y * zq - w * x);
    R[2][0] = 2.0f * (x * zq - w * y);
    R[2][1] = 2.0f * (y * zq + w * x);
    R[2][2] = 1.0f - 2.0f * (x * x + y * y);
    const int64_t split_rank = off_split[i];
    int64_t d = (int64_t)n_orig + n_clone + off_child[i];
    for (int j = 0; j < a.children; j++) {
      const double* nr = normals + (split_rank * a.children + j) * 3;
      const float l0 = (float)nr[0] * s0, l1 = (float)nr[1] * s1, l2 = (float)nr[2] * s2;
      float mean[3];
      const float pm[3] = {p0.x, p0.y, p0.z};
      for (int r = 0; r < 3; r++) mean[r] = pm[r] + (R[r][0] * l0 + R[r][1] * l1 + R[r][2] * l2);
      po[d] = make_float4(mean[0], mean[1], mean[2], p0.w);
      po[cap_out + d] = p1;
      po[2 * cap_out + d] = make_float4(p2.x - a.shrink, p2.y - a.shrink, p2.z - a.shrink, p2.w);
      for (int q = 3; q < kPlanes; q++) po[q * cap_out + d] = p[q * cap + i];
      for (int q = 0; q < kPlanes; q++) {
        mo[q * cap_out + d] = z;
        vo[q * cap_out + d] = z;
      }
      if (a.origin_out) a.origin_out[d] = (uint32_t)i;
      if (a.birth_out) a.birth_out[d] = a.birth_now;
      d++;
    }
  }
}

// reset_opacity (densify.rs:224-230): opacity = min(opacity, limit); opacity moments zeroed.
__global__ void reset_opacity_kernel(float4* __restrict__ p, float4* __restrict__ m, float4* __restrict__ v, int64_t n,
                                     float limit) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 a = p[i];
  a.w = fminf(a.w, limit);
  p[i] = a;
  float4 b = m[i];
  b.w = 0.0f;
  m[i] = b;
  float4 c = v[i];
  c.w = 0.0f;
  v[i] = c;
}

Status launch_reset_opacity(Ctx* c, float* params, float* m, float* v, int64_t n, float limit) {
  if (n == 0) return Status::ok();
  reset_opacity_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(reinterpret_cast<float4*>(params),
                                                                 reinterpret_cast<float4*>(m),
                                                                 reinterpret_cast<float4*>(v), n, limit);
  c->launches.count++;
  SPLAT_LAUNCHED("reset_opacity_kernel");
  return Status::ok();
}

Status densify_plan(Ctx* c, const float* params, int64_t n, int64_t cap, const float* accum, const uint32_t* denom,
                    const uint32_t* maxr, const DensifyParams& dp, DensifyPlan* plan) {
  DensifyArgs a;
  a.grad_threshold = dp.cfg.grad_threshold;
  a.size_limit = dp.cfg.percent_dense * dp.extent;
  a.min_opacity = dp.cfg.min_opacity;
  a.big_world_limit = dp.cfg.max_world_size_frac * dp.extent;
  a.prune_big_world = dp.cfg.prune_big_world;
  a.max_screen_size = dp.cfg.max_screen_size;
  a.children = dp.cfg.split_children;
  a.shrink = dp.shrink;
  a.grow = dp.grow ? 1 : 0;
  a.policy = dp.policy;
  a.prune_conf = dp.prune_conf;
  a.action = dp.action;
  a.origin_out = dp.origin_out;
  a.birth_in = dp.birth_in;
  a.birth_out = dp.birth_out;
  a.birth_now = dp.birth_now;
  uint32_t *flags, *ko, *kcl, *sp, *kch, *oo, *oc, *os, *ok;
  unsigned long long* counts;
  uint64_t* tot;
  const size_t nb = (size_t)std::max<int64_t>(n, 1) * 4;
  for (uint32_t** q : {&flags, &ko, &kcl, &sp, &kch, &oo, &oc, &os, &ok}) SPLAT_TRY(arena_reserve(c, nb + 4, (void**)q));
  SPLAT_TRY(arena_reserve(c, 8 * 8, (void**)&counts));
  SPLAT_TRY(arena_reserve(c, 8 * 4, (void**)&tot));
  SPLAT_CUDA(cudaMemsetAsync(counts, 0, 8 * 8, c->stream));
  if (n > 0) {
    densify_mark_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(reinterpret_cast<const float4*>(params), n, cap,
                                                                 accum, denom, maxr, a, flags, ko, kcl, sp, kch,
                                                                 counts);
    c->launches.count++;
    SPLAT_LAUNCHED("densify_mark_kernel");
    SPLAT_TRY(launch_scan_u32(c, ko, n, oo, 0, tot));
    SPLAT_TRY(launch_scan_u32(c, kcl, n, oc, 0, tot + 1));
    SPLAT_TRY(launch_scan_u32(c, sp, n, os, 0, tot + 2));
    SPLAT_TRY(launch_scan_u32(c, kch, n, ok, 0, tot + 3));
  }
  unsigned long long* h = reinterpret_cast<unsigned long long*>(c->host_small);
  SPLAT_CUDA(cudaMemcpyAsync(h, counts, 6 * 8, cudaMemcpyDeviceToHost, c->stream));
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  plan->kept_orig = h[0];
  plan->cloned = h[1];
  plan->kept_clones = h[2];
  plan->split = h[3];
  plan->kept_children = h[4];
  plan->pruned = h[5];
  plan->flags = flags;
  plan->off_orig = oo;
  plan->off_clone = oc;
  plan->off_split = os;
  plan->off_child = ok;
  plan->args = a;
  return Status::ok();
}

Status densify_apply(Ctx* c, const float* params, const float* m, const float* v, int64_t n, int64_t cap,
                     const DensifyPlan& plan, const double* normals_dev, float* po, float* mo, float* vo,
                     int64_t cap_out) {
  if (n == 0) return Status::ok();
  densify_scatter_kernel<<<ceil_div(n, 128), 128, 0, c->stream>>>(
      reinterpret_cast<const float4*>(params), reinterpret_cast<const float4*>(m), reinterpret_cast<const float4*>(v), n,
      cap, plan.flags, plan.off_orig, plan.off_clone, plan.off_split, plan.off_child, (uint32_t)plan.kept_orig,
      (uint32_t)plan.kept_clones, normals_dev, plan.args, reinterpret_cast<float4*>(po), reinterpret_cast<float4*>(mo),
      reinterpret_cast<float4*>(vo), cap_out);
  c->launches.count++;
  SPLAT_LAUNCHED("densify_scatter_kernel");
  return Status::ok();
}

}  // namespace splat
