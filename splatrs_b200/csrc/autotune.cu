// Autotuning of the compositing configuration (not in the reference): tile shape
// {8x8, 16x16, 16x32} x shared-memory chunk depth {32, 64, 128, 256} x the backward's
// pixels per thread {1, 2}, timed on the caller's own workload with CUDA events and kept on
// the context.
#include <cmath>
#include <functional>

#include "common.cuh"
#include "kernels.cuh"
#include "renderer.cuh"

namespace splat {

const RasterConfig kRasterCandidateList[kRasterCandidates] = {
    {16, 16, 256, 1}, {16, 16, 128, 1}, {16, 16, 64, 1}, {16, 16, 32, 1}, {8, 8, 256, 1},  {8, 8, 128, 1},
    {8, 8, 64, 1},    {8, 8, 32, 1},    {16, 32, 256, 1}, {16, 32, 128, 1}, {16, 32, 64, 1}, {16, 32, 32, 1},
    {16, 16, 256, 2}, {16, 16, 128, 2}, {16, 16, 64, 2}, {16, 16, 32, 2}, {8, 8, 256, 2},  {8, 8, 128, 2},
    {8, 8, 64, 2},    {8, 8, 32, 2},    {16, 32, 256, 2}, {16, 32, 128, 2}, {16, 32, 64, 2}, {16, 32, 32, 2}};

Status tune_raster(Ctx* c, const std::function<Status(bool)>& pass, int reps, float ms[kRasterCandidates]) {
  cudaEvent_t ev[2] = {nullptr, nullptr};
  Status s = cuda_status(cudaEventCreate(&ev[0]), "cudaEventCreate");
  if (s.good()) s = cuda_status(cudaEventCreate(&ev[1]), "cudaEventCreate");
  const RasterConfig start = c->raster;
  RasterConfig best = start;
  float best_ms = INFINITY;
  for (int k = 0; k < kRasterCandidates; k++) ms[k] = NAN;
  for (int k = 0; s.good() && k < kRasterCandidates; k++) {
    c->raster = kRasterCandidateList[k];
    s = pass(true);
    if (s.good()) s = cuda_status(cudaEventRecord(ev[0], c->stream), "cudaEventRecord");
    for (int r = 0; s.good() && r < reps; r++) s = pass(false);
    if (s.good()) s = cuda_status(cudaEventRecord(ev[1], c->stream), "cudaEventRecord");
    if (s.good()) s = cuda_status(cudaEventSynchronize(ev[1]), "cudaEventSynchronize");
    float t = 0.0f;
    if (s.good()) s = cuda_status(cudaEventElapsedTime(&t, ev[0], ev[1]), "cudaEventElapsedTime");
    if (!s.good()) break;
    ms[k] = t / (float)reps;
    if (ms[k] < best_ms) {
      best_ms = ms[k];
      best = c->raster;
    }
  }
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
  c->raster = s.good() ? best : start;
  return s;
}

Status tune_render(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                   const splat_proj_opts& opts, const float bg[3], const float* dimage, int reps,
                   float ms[kRasterCandidates]) {
  ViewBuffers v;
  DevBuf pgrad;
  v.e_cap = std::max<int64_t>(8 * std::max<int64_t>(n, 1), 1 << 16);
  // One view: projection, device-driven binning, forward and backward compositing. The
  // untimed pass waits for the result and redoes the view with more room for tile entries
  // until its binning fits.
  auto pass = [&](bool warm) -> Status {
    arena_reset(c);
    if (warm) SPLAT_TRY(pgrad.ensure((size_t)std::max<int64_t>(cap, 1) * 48));
    for (;;) {
      SPLAT_TRY(render_view_dev(c, planes, n, cap, cam, opts, bg, v));
      SPLAT_TRY(launch_fill_u32(c, pgrad.ptr, (size_t)std::max<int64_t>(cap, 1) * 12, 0u));
      SPLAT_TRY(launch_raster_bwd(c, v.proj.as<float>(), v.gauss.as<uint32_t>(), v.tile_range.as<uint32_t>(),
                                  cam.width, cam.height, bg, v.final_t.as<float>(), v.n_contrib.as<uint32_t>(), dimage,
                                  pgrad.as<float>(), cap, nullptr));
      if (!warm) return Status::ok();
      uint32_t w[4];
      SPLAT_CUDA(cudaMemcpyAsync(w, v.counters.ptr, 16, cudaMemcpyDeviceToHost, c->stream));
      SPLAT_CUDA(cudaStreamSynchronize(c->stream));
      if (w[2] == 0) return Status::ok();
      if (w[2] & 2u) return Status::make(SPLAT_ERR_TIMEOUT, "radix sort: a tile's look-back wait ran out");
      const uint64_t entries = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
      v.e_cap = std::max<int64_t>(2 * v.e_cap, (int64_t)(entries + entries / 4 + 4096));
      if (v.e_cap >= 0xffffffffLL) return Status::make(SPLAT_ERR_CAPACITY, "too many tile entries for 32-bit offsets");
      SPLAT_TRY(launch_fill_u32(c, v.overflow_flag(), 1, 0u));
      arena_reset(c);
    }
  };
  const Status s = tune_raster(c, pass, reps, ms);
  cudaStreamSynchronize(c->stream);
  v.release();
  pgrad.release();
  return s;
}

}  // namespace splat
