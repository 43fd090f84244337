// Model::from_points (reference src/model.rs:77-104) on the device: every point's mean
// squared distance to its three nearest other points (mean_nn_dist2, model.rs:128-186),
// then the initial Gaussian (scale from that distance, identity rotation, opacity 0.1,
// colour in the DC coefficient).
//
// The search is exact and brute force: one thread per query point sweeps all points,
// staged through shared memory in tiles, keeping the three smallest squared distances. The
// reference's kd-tree (kiddo 5.3.3) returns the same neighbours; coincident points count as
// zero-distance neighbours there as here. Distances are computed in double from the f32
// coordinates with the reference's operation order (dx*dx + dy*dy + dz*dz), and the three
// are summed in ascending order, so the result equals the reference's to the bit.
#include "common.cuh"
#include "kernels.cuh"
#include "renderer.cuh"

namespace splat {

constexpr int kKnnThreads = 256;

__global__ void __launch_bounds__(kKnnThreads) knn3_kernel(const float* __restrict__ pts, int64_t n,
                                                           double* __restrict__ out) {
  __shared__ float sp[kKnnThreads * 3];
  const int64_t i = (int64_t)blockIdx.x * kKnnThreads + threadIdx.x;
  const bool valid = i < n;
  const double qx = valid ? (double)pts[3 * i] : 0.0, qy = valid ? (double)pts[3 * i + 1] : 0.0,
               qz = valid ? (double)pts[3 * i + 2] : 0.0;
  double b0 = INFINITY, b1 = INFINITY, b2 = INFINITY;
  int found = 0;
  for (int64_t base = 0; base < n; base += kKnnThreads) {
    const int64_t j = base + threadIdx.x;
    if (j < n) {
      sp[3 * threadIdx.x] = pts[3 * j];
      sp[3 * threadIdx.x + 1] = pts[3 * j + 1];
      sp[3 * threadIdx.x + 2] = pts[3 * j + 2];
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)kKnnThreads, n - base);
    if (valid) {
      for (int k = 0; k < cnt; k++) {
        if (base + k == i) continue;
        const double dx = qx - (double)sp[3 * k];
        const double dy = qy - (double)sp[3 * k + 1];
        const double dz = qz - (double)sp[3 * k + 2];
        const double d = dx * dx + dy * dy + dz * dz;
        if (d < b2) {
          if (d < b1) {
            b2 = b1;
            if (d < b0) {
              b1 = b0;
              b0 = d;
            } else {
              b1 = d;
            }
          } else {
            b2 = d;
          }
        }
        found = found < 3 ? found + 1 : 3;
      }
    }
    __syncthreads();
  }
  if (valid) {
    double sum = 0.0;
    if (found > 0) sum += b0;
    if (found > 1) sum += b1;
    if (found > 2) sum += b2;
    out[i] = found > 0 ? sum / (double)found : 0.0;
  }
}

// The initial record of each point (model.rs:80-97) written into the parameter planes.
__global__ void init_gaussians_kernel(const float* __restrict__ pts, const uint8_t* __restrict__ rgb,
                                      const double* __restrict__ d2, int64_t n, float opacity_logit, float sh_c0,
                                      float4* __restrict__ planes, int64_t cap) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float d = fmaxf((float)d2[i], 1e-7f);
  const float log_s = crm::logf_cr(sqrtf(d));
  float dc[3];
#pragma unroll
  for (int c = 0; c < 3; c++) dc[c] = ((float)rgb[3 * i + c] / 255.0f - 0.5f) / sh_c0;  // rgb_to_sh (sh.rs:41)
  planes[i] = make_float4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], opacity_logit);
  planes[cap + i] = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
  planes[2 * cap + i] = make_float4(log_s, log_s, log_s, 0.0f);
  planes[3 * cap + i] = make_float4(dc[0], dc[1], dc[2], 0.0f);
  const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int q = 4; q < kPlanes; q++) planes[q * cap + i] = z;
}

}  // namespace splat

using namespace splat;

extern "C" {

// mean_nn_dist2 (reference src/model.rs:128-186): points (n x 3 float, device) -> out (n
// doubles, device).
SPLAT_API int splat_mean_nn_dist2(splat_ctx* ctx, const float* points_dev, int64_t n, double* out_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  Ctx* c = splat_ctx_impl(ctx);
  if (n < 0 || (n && (!points_dev || !out_dev))) {
    c->last_error = "splat_mean_nn_dist2: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  if (n == 0) return SPLAT_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != c->device) cudaSetDevice(c->device);
  knn3_kernel<<<ceil_div(n, kKnnThreads), kKnnThreads, 0, c->stream>>>(points_dev, n, out_dev);
  c->launches.count++;
  const Status s = cuda_status(cudaGetLastError(), "knn3_kernel");
  if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
  if (!s.good()) {
    c->last_error = s.msg;
    return s.code;
  }
  return SPLAT_OK;
}

// Model::from_points (reference src/model.rs:77-104): n points (x y z float) and colours
// (r g b uint8) on the host -> n Gaussians in parameter planes of capacity cap on the
// device. Synchronises.
SPLAT_API int splat_init_from_points(splat_ctx* ctx, const float* points_host, const uint8_t* rgb_host, int64_t n,
                                     float* planes_dev, int64_t cap) {
  if (!ctx) return SPLAT_ERR_INVALID;
  Ctx* c = splat_ctx_impl(ctx);
  if (n < 0 || cap < n || (n && (!points_host || !rgb_host || !planes_dev))) {
    c->last_error = "splat_init_from_points: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  if (n == 0) return SPLAT_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != c->device) cudaSetDevice(c->device);
  arena_reset(c);
  float* pts = nullptr;
  uint8_t* col = nullptr;
  double* d2 = nullptr;
  Status s = arena_reserve(c, (size_t)n * 12, (void**)&pts);
  if (s.good()) s = arena_reserve(c, (size_t)n * 3, (void**)&col);
  if (s.good()) s = arena_reserve(c, (size_t)n * 8, (void**)&d2);
  if (s.good()) s = cuda_status(cudaMemcpyAsync(pts, points_host, (size_t)n * 12, cudaMemcpyHostToDevice, c->stream),
                                "upload points");
  if (s.good()) s = cuda_status(cudaMemcpyAsync(col, rgb_host, (size_t)n * 3, cudaMemcpyHostToDevice, c->stream),
                                "upload colours");
  if (s.good()) {
    knn3_kernel<<<ceil_div(n, kKnnThreads), kKnnThreads, 0, c->stream>>>(pts, n, d2);
    c->launches.count++;
    s = cuda_status(cudaGetLastError(), "knn3_kernel");
  }
  if (s.good()) {
    const float x = 0.1f;
    const float logit = logf(x / (1.0f - x));  // inverse_sigmoid(0.1) (math.rs:454)
    init_gaussians_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(pts, col, d2, n, logit,
                                                                   (float)0.28209479177387814,
                                                                   reinterpret_cast<float4*>(planes_dev), cap);
    c->launches.count++;
    s = cuda_status(cudaGetLastError(), "init_gaussians_kernel");
  }
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
  if (!s.good()) {
    c->last_error = s.msg;
    return s.code;
  }
  return SPLAT_OK;
}

}  // extern "C"
