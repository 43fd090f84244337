// Learned densification around the reference's threshold rule (src/densify.rs:125-221),
// which this code never replaces: it computes what the network sees and what it learns.
//
//   densify_features: 16 features per Gaussian at a densification: mean and max
//     view-space gradient, visibility count, log-scales, opacity, largest screen radius,
//     SH-DC energy, age, size against the rule's clone/split limit, contribution (blending
//     weight per visible view over the window), and four statistics of its neighbourhood
//     (a hashed grid of cells two rule-limits wide: count, mean opacity, mean gradient,
//     mean log-size).
//   outcome counts / hindsight labels: every Gaussian carries the index of the record it
//     descends from at the previous densification. At the next one, a record whose
//     clone/split left fewer than two useful descendants (opacity >= tau and, when tau_c
//     is set, a window contribution >= tau_c) is relabelled keep (the edit was wasted), a
//     kept record with no descendant left, or whose descendants contributed less than
//     tau_c in all, is relabelled prune, and a pruned one stays prune.
#include "common.cuh"
#include "kernels.cuh"

namespace splat {

namespace {
constexpr int kF = 16;

__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + __expf(-x)); }

__device__ __forceinline__ uint32_t cell_hash(float3 m, float inv_cell, uint32_t mask) {
  const int ix = __float2int_rd(m.x * inv_cell), iy = __float2int_rd(m.y * inv_cell), iz = __float2int_rd(m.z * inv_cell);
  return ((uint32_t)ix * 73856093u ^ (uint32_t)iy * 19349663u ^ (uint32_t)iz * 83492791u) & mask;
}

// Grid cell per entry: count, sum opacity, sum gradient, sum log max-scale.
__global__ void grid_accumulate_kernel(const float4* __restrict__ p, int64_t n, int64_t cap,
                                       const float* __restrict__ accum, const uint32_t* __restrict__ denom,
                                       float inv_cell, uint32_t mask, uint32_t* __restrict__ cnt,
                                       float* __restrict__ sop, float* __restrict__ sgr, float* __restrict__ sls) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p0 = p[i], p2 = p[2 * cap + i];
  const uint32_t h = cell_hash(make_float3(p0.x, p0.y, p0.z), inv_cell, mask);
  const float gr = denom[i] > 0 ? accum[i] / (float)denom[i] : 0.0f;
  atomicAdd(&cnt[h], 1u);
  atomicAdd(&sop[h], sigmoidf_(p0.w));
  atomicAdd(&sgr[h], gr);
  atomicAdd(&sls[h], fmaxf(p2.x, fmaxf(p2.y, p2.z)));
}

__global__ void features_kernel(const float4* __restrict__ p, int64_t n, int64_t cap,
                                const float* __restrict__ accum, const uint32_t* __restrict__ denom,
                                const uint32_t* __restrict__ maxr, const float* __restrict__ maxg,
                                const float* __restrict__ contrib, const uint32_t* __restrict__ birth, uint32_t now,
                                float size_limit, float inv_cell, uint32_t mask, const uint32_t* __restrict__ cnt,
                                const float* __restrict__ sop, const float* __restrict__ sgr,
                                const float* __restrict__ sls, float* __restrict__ x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p0 = p[i], p2 = p[2 * cap + i], p3 = p[3 * cap + i];
  const float gr = denom[i] > 0 ? accum[i] / (float)denom[i] : 0.0f;
  const float ms = fmaxf(p2.x, fmaxf(p2.y, p2.z));
  const uint32_t h = cell_hash(make_float3(p0.x, p0.y, p0.z), inv_cell, mask);
  const float c = (float)max(cnt[h], 1u);
  float f[kF];
  f[0] = gr * 1e3f;
  f[1] = (maxg ? maxg[i] : gr) * 1e3f;
  f[2] = log1pf((float)denom[i]);
  f[3] = p2.x + 4.0f;
  f[4] = p2.y + 4.0f;
  f[5] = p2.z + 4.0f;
  f[6] = sigmoidf_(p0.w);
  f[7] = log1pf((float)maxr[i]);
  f[8] = p3.x * p3.x + p3.y * p3.y + p3.z * p3.z;  // SH DC (sh[0][0..3])
  f[9] = birth ? (float)(now - min(birth[i], now)) * 1e-3f : 0.0f;
  f[10] = ms - logf(size_limit);  // log of max scale over the clone/split limit
  f[11] = logf(c);
  f[12] = sop[h] / c;
  f[13] = sgr[h] / c * 1e3f;
  f[14] = sls[h] / c + 4.0f;
  f[15] = contrib ? log1pf(contrib[i] / (float)max(denom[i], 1u)) : 0.0f;
#pragma unroll
  for (int k = 0; k < kF; k++) x[i * kF + k] = f[k];
}

__global__ void outcome_counts_kernel(const float4* __restrict__ p, int64_t n, const uint32_t* __restrict__ origin,
                                      int64_t n_prev, float tau_logit, const float* __restrict__ contrib, float tau_c,
                                      uint32_t* __restrict__ alive, uint32_t* __restrict__ useful,
                                      float* __restrict__ csum) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = origin[i];
  if ((int64_t)r >= n_prev) return;
  const float cb = contrib ? contrib[i] : 0.0f;
  atomicAdd(&alive[r], 1u);
  atomicAdd(&csum[r], cb);
  if (p[i].w >= tau_logit && !(tau_c > 0.0f && cb < tau_c)) atomicAdd(&useful[r], 1u);
}

__global__ void hindsight_labels_kernel(const uint32_t* __restrict__ action, const uint32_t* __restrict__ alive,
                                        const uint32_t* __restrict__ useful, const float* __restrict__ csum,
                                        float tau_c, int64_t n_prev, int32_t* __restrict__ y,
                                        unsigned long long* __restrict__ counts) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_prev) return;
  const uint32_t a = action[r];
  int32_t lab;
  if (a == 1u)
    lab = useful[r] >= 2u ? 1 : 0;
  else if (a == 0u)
    lab = (alive[r] == 0u || (tau_c > 0.0f && csum[r] < tau_c)) ? 2 : 0;
  else
    lab = 2;
  y[r] = lab;
  atomicAdd(&counts[lab], 1ull);
}

// Held-out accuracy before training on a densification's labels: [0] the network's
// argmax equals the label, [1] the rule's action equals it, [2] records.
__global__ void label_accuracy_kernel(const float* __restrict__ prob, const uint32_t* __restrict__ action,
                                      const int32_t* __restrict__ y, int64_t n_prev,
                                      unsigned long long* __restrict__ acc) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = r < n_prev;
  uint32_t net = 0, rule = 0;
  if (valid) {
    const float p0 = prob[3 * r], p1 = prob[3 * r + 1], p2 = prob[3 * r + 2];
    const int32_t am = (p1 > p0 && p1 >= p2) ? 1 : ((p2 > p0 && p2 > p1) ? 2 : 0);
    net = am == y[r] ? 1u : 0u;
    rule = (int32_t)action[r] == y[r] ? 1u : 0u;
  }
  const uint32_t a = __reduce_add_sync(0xffffffffu, net), b = __reduce_add_sync(0xffffffffu, rule),
                 c = __reduce_add_sync(0xffffffffu, valid ? 1u : 0u);
  if ((threadIdx.x & 31) == 0) {
    if (a) atomicAdd(&acc[0], (unsigned long long)a);
    if (b) atomicAdd(&acc[1], (unsigned long long)b);
    if (c) atomicAdd(&acc[2], (unsigned long long)c);
  }
}

// Every `stride`-th record (from `first`) into a compact training set with class weights.
__global__ void gather_training_kernel(const float* __restrict__ x, const int32_t* __restrict__ y, int64_t n_prev,
                                       int64_t first, int64_t stride, float w0, float w1, float w2,
                                       float* __restrict__ xo, int32_t* __restrict__ yo, float* __restrict__ wo,
                                       int64_t m) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int64_t r = first + k * stride;
  if (r >= n_prev) {  // never reached with m from the caller; left harmless
    wo[k] = 0.0f;
    yo[k] = 0;
    for (int f = 0; f < kF; f++) xo[k * kF + f] = 0.0f;
    return;
  }
  for (int f = 0; f < kF; f++) xo[k * kF + f] = x[r * kF + f];
  const int32_t lab = y[r];
  yo[k] = lab;
  wo[k] = lab == 0 ? w0 : (lab == 1 ? w1 : w2);
}
}  // namespace

size_t densify_features_scratch_bytes(int64_t n) {
  uint32_t t = 1024;
  while ((int64_t)t < 2 * n && t < (1u << 24)) t <<= 1;
  return (size_t)t * 4 * 4;
}

Status launch_densify_features(Ctx* c, const float* params, int64_t n, int64_t cap, const float* accum,
                               const uint32_t* denom, const uint32_t* maxr, const float* maxg, const float* contrib,
                               const uint32_t* birth, uint32_t now, float size_limit, void* scratch, float* x_out) {
  if (n == 0) return Status::ok();
  uint32_t t = 1024;
  while ((int64_t)t < 2 * n && t < (1u << 24)) t <<= 1;
  uint32_t* cnt = static_cast<uint32_t*>(scratch);
  float* sop = reinterpret_cast<float*>(cnt + t);
  float* sgr = sop + t;
  float* sls = sgr + t;
  SPLAT_TRY(launch_fill_u32(c, scratch, (size_t)t * 4, 0u));
  const float inv_cell = 1.0f / (2.0f * size_limit);
  const float4* p = reinterpret_cast<const float4*>(params);
  grid_accumulate_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(p, n, cap, accum, denom, inv_cell, t - 1, cnt, sop,
                                                                   sgr, sls);
  features_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(p, n, cap, accum, denom, maxr, maxg, contrib, birth, now,
                                                            size_limit, inv_cell, t - 1, cnt, sop, sgr, sls, x_out);
  c->launches.count += 2;
  SPLAT_LAUNCHED("densify features");
  return Status::ok();
}

Status launch_hindsight_labels(Ctx* c, const float* params, int64_t n, const uint32_t* origin, int64_t n_prev,
                               const uint32_t* action, float tau, const float* contrib, float tau_c,
                               uint32_t* alive, uint32_t* useful, float* csum, int32_t* y,
                               unsigned long long* counts) {
  SPLAT_TRY(launch_fill_u32(c, alive, (size_t)n_prev, 0u));
  SPLAT_TRY(launch_fill_u32(c, useful, (size_t)n_prev, 0u));
  SPLAT_TRY(launch_fill_u32(c, csum, (size_t)n_prev, 0u));
  SPLAT_TRY(launch_fill_u32(c, counts, 6, 0u));
  const float tau_logit = logf(tau / (1.0f - tau));
  if (n > 0)
    outcome_counts_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(reinterpret_cast<const float4*>(params), n, origin,
                                                                    n_prev, tau_logit, contrib, tau_c, alive, useful,
                                                                    csum);
  if (n_prev > 0)
    hindsight_labels_kernel<<<ceil_div(n_prev, 256), 256, 0, c->stream>>>(action, alive, useful, csum, tau_c, n_prev,
                                                                           y, counts);
  c->launches.count += 2;
  SPLAT_LAUNCHED("hindsight labels");
  return Status::ok();
}

Status launch_label_accuracy(Ctx* c, const float* prob, const uint32_t* action, const int32_t* y, int64_t n_prev,
                             unsigned long long* acc) {
  if (n_prev == 0) return Status::ok();
  label_accuracy_kernel<<<ceil_div(n_prev, 256), 256, 0, c->stream>>>(prob, action, y, n_prev, acc);
  c->launches.count++;
  SPLAT_LAUNCHED("label_accuracy_kernel");
  return Status::ok();
}

Status launch_gather_training(Ctx* c, const float* x, const int32_t* y, int64_t n_prev, int64_t first, int64_t stride,
                              const float w[3], float* xo, int32_t* yo, float* wo, int64_t m) {
  if (m == 0) return Status::ok();
  gather_training_kernel<<<ceil_div(m, 256), 256, 0, c->stream>>>(x, y, n_prev, first, stride, w[0], w[1], w[2], xo,
                                                                  yo, wo, m);
  c->launches.count++;
  SPLAT_LAUNCHED("gather_training_kernel");
  return Status::ok();
}

}  // namespace splat
