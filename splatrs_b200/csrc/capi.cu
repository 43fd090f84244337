// The C ABI (include/splat_gpu.h): argument checks, context and scratch management, and
// dispatch to the stage launchers. No entry point aborts; failures return a status and
// leave a message on the context.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "renderer.cuh"

namespace splat {

Status arena_reserve(Ctx* c, size_t bytes, void** out) {
  Arena& a = c->arena;
  bytes = (bytes + 255) & ~(size_t)255;
  if (bytes == 0) bytes = 256;
  if (a.chunks.empty() || a.used + bytes > a.chunks.back().size) {
    size_t want = std::max(bytes, a.chunks.empty() ? (size_t)(64u << 20) : a.chunks.back().size * 2);
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return Status::make(SPLAT_ERR_CUDA, std::string("scratch allocation of ") + std::to_string(want) +
                                              " bytes failed: " + cudaGetErrorString(e));
    }
    a.chunks.push_back(ArenaChunk{p, want});
    a.used = 0;
    a.generation++;
  }
  *out = static_cast<char*>(a.chunks.back().ptr) + a.used;
  a.used += bytes;
  return Status::ok();
}

void arena_reset(Ctx* c) {
  Arena& a = c->arena;
  if (a.chunks.size() > 1) {
    size_t total = 0;
    for (auto& ch : a.chunks) total += ch.size;
    cudaStreamSynchronize(c->stream);
    for (auto& ch : a.chunks) cudaFree(ch.ptr);
    a.chunks.clear();
    a.generation++;
    void* p = nullptr;
    if (cudaMalloc(&p, total) == cudaSuccess)
      a.chunks.push_back(ArenaChunk{p, total});
    else
      cudaGetLastError();
  }
  a.used = 0;
}

void arena_free(Ctx* c) {
  for (auto& ch : c->arena.chunks) cudaFree(ch.ptr);
  c->arena.chunks.clear();
  c->arena.used = 0;
  c->arena.generation++;
}

}  // namespace splat

using namespace splat;

struct splat_ctx {
  Ctx c;
};

namespace splat {
Ctx* splat_ctx_impl(splat_ctx* ctx) { return &ctx->c; }
}  // namespace splat

namespace {
int fail(splat_ctx* ctx, const Status& s) {
  if (ctx) ctx->c.last_error = s.msg;
  return s.code;
}
int invalid(splat_ctx* ctx, const char* msg) { return fail(ctx, Status::make(SPLAT_ERR_INVALID, msg)); }

// Every entry point runs on the context's device with a fresh scratch arena.
struct Enter {
  splat_ctx* ctx;
  int prev = -1;
  explicit Enter(splat_ctx* x) : ctx(x) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != x->c.device) cudaSetDevice(x->c.device);
    arena_reset(&x->c);
  }
  ~Enter() {
    if (prev >= 0 && prev != ctx->c.device) cudaSetDevice(prev);
  }
};

int finish(splat_ctx* ctx, const Status& s) { return s.good() ? SPLAT_OK : fail(ctx, s); }

bool cam_ok(const splat_camera* cam) {
  return cam && cam->width > 0 && cam->height > 0 && cam->width <= 65535 && cam->height <= 65535;
}
bool opts_ok(const splat_proj_opts* o) { return o && o->sh_degree >= 0 && o->sh_degree <= 3; }
}  // namespace

extern "C" {

SPLAT_API int splat_version(void) { return 1; }

SPLAT_API int32_t splat_struct_sizes(uint64_t* out) {
  const uint64_t sizes[] = {sizeof(splat_camera),         sizeof(splat_proj_opts),      sizeof(splat_lr),
                            sizeof(splat_densify_config), sizeof(splat_train_config),   sizeof(splat_densify_report),
                            sizeof(splat_step_info)};
  const int32_t k = (int32_t)(sizeof(sizes) / sizeof(sizes[0]));
  if (out)
    for (int32_t i = 0; i < k; i++) out[i] = sizes[i];
  return k;
}

SPLAT_API const char* splat_status_string(int status) {
  switch (status) {
    case SPLAT_OK: return "ok";
    case SPLAT_ERR_INVALID: return "invalid argument";
    case SPLAT_ERR_CAPACITY: return "capacity exceeded";
    case SPLAT_ERR_CUDA: return "CUDA error";
    case SPLAT_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

SPLAT_API int splat_ctx_create(int device, void* stream, splat_ctx** out) {
  if (!out) return SPLAT_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return SPLAT_ERR_CUDA;
  }
  splat_ctx* ctx = new (std::nothrow) splat_ctx();
  if (!ctx) return SPLAT_ERR_INVALID;
  ctx->c.device = device;
  ctx->c.stream = reinterpret_cast<cudaStream_t>(stream);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaDeviceGetAttribute(&ctx->c.sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaHostAlloc(&ctx->c.host_small, 4096, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(&ctx->c.host_small_dev, ctx->c.host_small, 0) != cudaSuccess) {
    if (ctx->c.host_small) cudaFreeHost(ctx->c.host_small);
    cudaGetLastError();
    cudaSetDevice(prev);
    delete ctx;
    return SPLAT_ERR_CUDA;
  }
  std::memset(ctx->c.host_small, 0, 4096);
  cudaSetDevice(prev);
  *out = ctx;
  return SPLAT_OK;
}

SPLAT_API int splat_ctx_destroy(splat_ctx* ctx) {
  if (!ctx) return SPLAT_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->c.device);
  cudaStreamSynchronize(ctx->c.stream);
  arena_free(&ctx->c);
  if (ctx->c.host_small) cudaFreeHost(ctx->c.host_small);
  cudaSetDevice(prev);
  delete ctx;
  return SPLAT_OK;
}

SPLAT_API int splat_ctx_set_stream(splat_ctx* ctx, void* stream) {
  if (!ctx) return SPLAT_ERR_INVALID;
  ctx->c.stream = reinterpret_cast<cudaStream_t>(stream);
  return SPLAT_OK;
}

SPLAT_API int splat_ctx_synchronize(splat_ctx* ctx) {
  if (!ctx) return SPLAT_ERR_INVALID;
  Enter e(ctx);
  Status s = cuda_status(cudaStreamSynchronize(ctx->c.stream), "cudaStreamSynchronize");
  if (s.good()) s = take_sort_error(&ctx->c);
  return finish(ctx, s);
}

SPLAT_API const char* splat_last_error(const splat_ctx* ctx) { return ctx ? ctx->c.last_error.c_str() : "no context"; }

SPLAT_API uint64_t splat_ctx_launch_count(const splat_ctx* ctx) { return ctx ? ctx->c.launches.count : 0; }

SPLAT_API int splat_diag_pair_exact(splat_ctx* ctx, uint32_t n, uint32_t* mismatches2) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!mismatches2) return invalid(ctx, "splat_diag_pair_exact: null output");
  Enter e(ctx);
  return finish(ctx, launch_diag_pair_exact(&ctx->c, n, mismatches2));
}

SPLAT_API int splat_diag_fast_exp_error(splat_ctx* ctx, float lo, float hi, int32_t negative, float* max_rel_error) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!max_rel_error || !(lo >= 0.0f) || !(hi >= lo) || !(hi < 1e30f)) return invalid(ctx, "splat_diag_fast_exp_error: bad range");
  Enter e(ctx);
  return finish(ctx, launch_diag_fast_exp(&ctx->c, lo, hi, negative, max_rel_error));
}

SPLAT_API int splat_diag_peak(splat_ctx* ctx, int32_t unit, double* ops_per_s, float* ms) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if ((unit != 0 && unit != 1) || !ops_per_s || !ms) return invalid(ctx, "splat_diag_peak: unit must be 0 or 1");
  Enter e(ctx);
  return finish(ctx, launch_diag_peak(&ctx->c, unit, ops_per_s, ms));
}

SPLAT_API int splat_ctx_scratch_info(const splat_ctx* ctx, uint64_t* out2) {
  if (!ctx || !out2) return SPLAT_ERR_INVALID;
  uint64_t bytes = 0;
  for (const auto& ch : ctx->c.arena.chunks) bytes += ch.size;
  out2[0] = bytes;
  out2[1] = ctx->c.arena.generation;
  return SPLAT_OK;
}

SPLAT_API int splat_diag_mbarrier_wait(splat_ctx* ctx, uint32_t limit, int32_t arrive) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (limit == 0 || limit > (1u << 22)) return invalid(ctx, "splat_diag_mbarrier_wait: limit must be in 1..4194304");
  Enter e(ctx);
  return finish(ctx, diag_mbar_wait(&ctx->c, limit, arrive));
}

SPLAT_API int splat_zero(splat_ctx* ctx, void* dev, size_t bytes) {
  if (!ctx || (!dev && bytes)) return invalid(ctx, "splat_zero: null pointer");
  Enter e(ctx);
  return finish(ctx, cuda_status(cudaMemsetAsync(dev, 0, bytes, ctx->c.stream), "cudaMemsetAsync"));
}

SPLAT_API int splat_params_from_aos(splat_ctx* ctx, const float* aos59_dev, int64_t n, float* planes_dev, int64_t cap) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || cap < n || (n && (!aos59_dev || !planes_dev))) return invalid(ctx, "splat_params_from_aos: bad sizes");
  Enter e(ctx);
  return finish(ctx, launch_params_from_aos(&ctx->c, aos59_dev, n, planes_dev, cap));
}

SPLAT_API int splat_params_to_aos(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap, float* aos59_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || cap < n || (n && (!aos59_dev || !planes_dev))) return invalid(ctx, "splat_params_to_aos: bad sizes");
  Enter e(ctx);
  return finish(ctx, launch_params_to_aos(&ctx->c, planes_dev, n, cap, aos59_dev));
}

SPLAT_API int splat_project_fwd(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap,
                                const splat_camera* cam, const splat_proj_opts* opts, float* proj_dev,
                                uint32_t* num_tiles_dev, uint32_t* depth_range_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!cam_ok(cam)) return invalid(ctx, "splat_project_fwd: camera size must be in 1..65535");
  if (!opts_ok(opts)) return invalid(ctx, "splat_project_fwd: sh_degree must be in 0..3");
  if (n < 0 || cap < n || !depth_range_dev || (n && (!planes_dev || !proj_dev || !num_tiles_dev)))
    return invalid(ctx, "splat_project_fwd: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_project_fwd(&ctx->c, planes_dev, n, cap, *cam, *opts, proj_dev, num_tiles_dev,
                                        depth_range_dev));
}

SPLAT_API int splat_params_to_bf16(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap, void* bf16_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || cap < n || (n && (!planes_dev || !bf16_dev))) return invalid(ctx, "splat_params_to_bf16: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_planes_to_bf16(&ctx->c, planes_dev, n, cap, bf16_dev));
}

SPLAT_API int splat_project_fwd_bf16(splat_ctx* ctx, const float* planes_dev, const void* bf16_dev, int64_t n,
                                     int64_t cap, const splat_camera* cam, const splat_proj_opts* opts,
                                     float* proj_dev, uint32_t* num_tiles_dev, uint32_t* depth_range_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!cam_ok(cam)) return invalid(ctx, "splat_project_fwd_bf16: camera size must be in 1..65535");
  if (!opts_ok(opts)) return invalid(ctx, "splat_project_fwd_bf16: sh_degree must be in 0..3");
  if (n < 0 || cap < n || !depth_range_dev || (n && (!planes_dev || !bf16_dev || !proj_dev || !num_tiles_dev)))
    return invalid(ctx, "splat_project_fwd_bf16: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_project_fwd(&ctx->c, planes_dev, n, cap, *cam, *opts, proj_dev, num_tiles_dev,
                                        depth_range_dev, nullptr, bf16_dev));
}

SPLAT_API int splat_proj_from_reference(splat_ctx* ctx, const float* proj15_dev, int64_t n, uint32_t width,
                                        uint32_t height, float* proj_dev, uint32_t* num_tiles_dev,
                                        uint32_t* depth_range_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (width == 0 || height == 0 || width > 65535 || height > 65535)
    return invalid(ctx, "splat_proj_from_reference: image size must be in 1..65535");
  if (n < 0 || !depth_range_dev || (n && (!proj15_dev || !proj_dev || !num_tiles_dev)))
    return invalid(ctx, "splat_proj_from_reference: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_proj_from_reference(&ctx->c, proj15_dev, n, width, height, proj_dev, num_tiles_dev,
                                                depth_range_dev));
}

SPLAT_API int splat_proj_to_reference(splat_ctx* ctx, const float* proj_dev, int64_t n, float* proj15_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || (n && (!proj_dev || !proj15_dev))) return invalid(ctx, "splat_proj_to_reference: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_proj_to_reference(&ctx->c, proj_dev, n, proj15_dev));
}

SPLAT_API int splat_bin_count(splat_ctx* ctx, const uint32_t* num_tiles_dev, int64_t n, uint32_t* entry_offset_dev,
                              int64_t* num_entries) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || !entry_offset_dev || !num_entries || (n && !num_tiles_dev))
    return invalid(ctx, "splat_bin_count: bad buffers");
  Enter e(ctx);
  uint64_t* total = nullptr;
  Status s = arena_reserve(&ctx->c, 8, (void**)&total);
  if (s.good()) s = launch_scan_u32(&ctx->c, num_tiles_dev, n, entry_offset_dev, 1, total);
  uint64_t* h = reinterpret_cast<uint64_t*>(ctx->c.host_small);
  if (s.good()) s = cuda_status(cudaMemcpyAsync(h, total, 8, cudaMemcpyDeviceToHost, ctx->c.stream), "read entry count");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(ctx->c.stream), "cudaStreamSynchronize");
  if (s.good()) s = take_sort_error(&ctx->c);
  if (!s.good()) return fail(ctx, s);
  if (h[0] >= 0xffffffffull) return fail(ctx, Status::make(SPLAT_ERR_CAPACITY, "too many tile entries for 32-bit offsets"));
  *num_entries = (int64_t)h[0];
  return SPLAT_OK;
}

SPLAT_API int splat_bin_sort(splat_ctx* ctx, const float* proj_dev, const uint32_t* entry_offset_dev, int64_t n,
                             int64_t num_entries, const uint32_t* depth_range_dev, uint32_t width, uint32_t height,
                             uint32_t* gauss_dev, uint64_t* keys_dev, uint32_t* tile_range_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (width == 0 || height == 0 || width > 65535 || height > 65535)
    return invalid(ctx, "splat_bin_sort: image size must be in 1..65535");
  if (n < 0 || num_entries < 0 || !tile_range_dev || !depth_range_dev ||
      (num_entries && (!proj_dev || !entry_offset_dev || !gauss_dev)))
    return invalid(ctx, "splat_bin_sort: bad buffers");
  Enter e(ctx);
  uint32_t* h = reinterpret_cast<uint32_t*>(ctx->c.host_small);
  Status s = cuda_status(cudaMemcpyAsync(h, depth_range_dev, 8, cudaMemcpyDeviceToHost, ctx->c.stream), "read depth range");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(ctx->c.stream), "cudaStreamSynchronize");
  if (s.good()) s = take_sort_error(&ctx->c);  // of an earlier sort on this context
  if (!s.good()) return fail(ctx, s);
  const uint32_t dmin = h[0], dmax = h[1];
  if (num_entries > 0 && dmin > dmax) return invalid(ctx, "splat_bin_sort: depth range is empty but entries exist");
  return finish(ctx, launch_bin_sort(&ctx->c, proj_dev, entry_offset_dev, n, num_entries, depth_range_dev, dmin,
                                     num_entries > 0 ? dmax : dmin, width, height, gauss_dev, keys_dev,
                                     tile_range_dev));
}

SPLAT_API int32_t splat_raster_candidates(uint32_t* out) {
  if (out)
    for (int k = 0; k < kRasterCandidates; k++) {
      out[4 * k] = kRasterCandidateList[k].tile_w;
      out[4 * k + 1] = kRasterCandidateList[k].tile_h;
      out[4 * k + 2] = kRasterCandidateList[k].chunk;
      out[4 * k + 3] = kRasterCandidateList[k].ppl;
    }
  return kRasterCandidates;
}

SPLAT_API int splat_set_raster_config(splat_ctx* ctx, uint32_t tile_w, uint32_t tile_h, uint32_t chunk,
                                      uint32_t pixels_per_thread) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!RasterConfig::supported(tile_w, tile_h, chunk, pixels_per_thread))
    return invalid(ctx, "splat_set_raster_config: tiles 8x8, 16x16 or 16x32, chunk depth 32, 64, 128 or 256 and 1 "
                        "or 2 pixels per thread");
  ctx->c.raster.tile_w = tile_w;
  ctx->c.raster.tile_h = tile_h;
  ctx->c.raster.chunk = chunk;
  ctx->c.raster.ppl = pixels_per_thread;
  return SPLAT_OK;
}

SPLAT_API int splat_get_raster_config(splat_ctx* ctx, uint32_t* out4) {
  if (!ctx || !out4) return SPLAT_ERR_INVALID;
  out4[0] = ctx->c.raster.tile_w;
  out4[1] = ctx->c.raster.tile_h;
  out4[2] = ctx->c.raster.chunk;
  out4[3] = ctx->c.raster.ppl;
  return SPLAT_OK;
}

SPLAT_API int splat_autotune_render(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap,
                                    const splat_camera* cam, const splat_proj_opts* opts, const float* background,
                                    const float* dimage_dev, int32_t reps, float* ms_out, uint32_t* picked) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!cam_ok(cam) || !opts_ok(opts) || !background || !dimage_dev || reps < 1 || n < 0 || cap < n ||
      (n && !planes_dev))
    return invalid(ctx, "splat_autotune_render: bad arguments");
  Enter e(ctx);
  float ms[kRasterCandidates];
  const Status s = tune_render(&ctx->c, planes_dev, n, cap, *cam, *opts, background, dimage_dev, reps, ms);
  if (!s.good()) return fail(ctx, s);
  if (ms_out)
    for (int k = 0; k < kRasterCandidates; k++) ms_out[k] = ms[k];
  if (picked) splat_get_raster_config(ctx, picked);
  return SPLAT_OK;
}

SPLAT_API int32_t splat_mlp_num_params(void) { return mlp_num_params(); }

SPLAT_API int splat_mlp_forward(splat_ctx* ctx, const float* x_dev, int64_t n, const float* theta_dev, float* prob_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || !theta_dev || (n && (!x_dev || !prob_dev))) return invalid(ctx, "splat_mlp_forward: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_mlp_forward(&ctx->c, x_dev, n, theta_dev, prob_dev));
}

SPLAT_API int splat_mlp_forward_tc(splat_ctx* ctx, const float* x_dev, int64_t n, const float* theta_dev,
                                  float* prob_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || !theta_dev || (n && (!x_dev || !prob_dev))) return invalid(ctx, "splat_mlp_forward_tc: bad buffers");
  if (reinterpret_cast<uintptr_t>(x_dev) % 16) return invalid(ctx, "splat_mlp_forward_tc: x_dev not 16-byte aligned");
  Enter e(ctx);
  return finish(ctx, mlp_forward_tc_checked(&ctx->c, x_dev, n, theta_dev, prob_dev));
}

SPLAT_API int splat_mlp_grad(splat_ctx* ctx, const float* x_dev, const int32_t* y_dev, const float* w_dev, int64_t n,
                             float scale, const float* theta_dev, float* grad_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || !theta_dev || !grad_dev || (n && (!x_dev || !y_dev || !w_dev)))
    return invalid(ctx, "splat_mlp_grad: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_mlp_grad(&ctx->c, x_dev, y_dev, w_dev, n, scale, theta_dev, grad_dev));
}

SPLAT_API int splat_mlp_grad_tc(splat_ctx* ctx, const float* x_dev, const int32_t* y_dev, const float* w_dev,
                               int64_t n, float scale, const float* theta_dev, float* grad_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || !theta_dev || !grad_dev || (n && (!x_dev || !y_dev || !w_dev)))
    return invalid(ctx, "splat_mlp_grad_tc: bad buffers");
  if (reinterpret_cast<uintptr_t>(x_dev) % 16) return invalid(ctx, "splat_mlp_grad_tc: x_dev not 16-byte aligned");
  Enter e(ctx);
  Status s = mlp_tc_error_clear(&ctx->c);
  if (s.good()) s = launch_mlp_grad_tc(&ctx->c, x_dev, y_dev, w_dev, n, scale, theta_dev, grad_dev,
                                       mlp_tc_error_word(&ctx->c));
  if (s.good()) s = mlp_tc_error_check(&ctx->c);
  return finish(ctx, s);
}

SPLAT_API int splat_mlp_adam(splat_ctx* ctx, float* theta_dev, const float* grad_dev, float* m_dev, float* v_dev,
                             uint64_t step, float lr) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!theta_dev || !grad_dev || !m_dev || !v_dev || step == 0) return invalid(ctx, "splat_mlp_adam: bad arguments");
  Enter e(ctx);
  return finish(ctx, launch_mlp_adam(&ctx->c, theta_dev, grad_dev, m_dev, v_dev, step, lr));
}

SPLAT_API int splat_bin_count_device(splat_ctx* ctx, const uint32_t* num_tiles_dev, int64_t n,
                                     uint32_t* entry_offset_dev, uint64_t* num_entries_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || !entry_offset_dev || !num_entries_dev || (n && !num_tiles_dev))
    return invalid(ctx, "splat_bin_count_device: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_scan_u32(&ctx->c, num_tiles_dev, n, entry_offset_dev, 1, num_entries_dev));
}

SPLAT_API size_t splat_bin_sort_device_scratch_bytes(int64_t capacity) {
  return capacity < 0 ? 0 : dev_sort_scratch_bytes(capacity);
}

SPLAT_API int splat_bin_sort_device(splat_ctx* ctx, const float* proj_dev, const uint32_t* entry_offset_dev, int64_t n,
                                    const uint64_t* num_entries_dev, int64_t capacity,
                                    const uint32_t* depth_range_dev, uint32_t width, uint32_t height,
                                    void* scratch_dev, uint32_t* gauss_dev, uint32_t* tile_range_dev,
                                    uint32_t* overflow_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (width == 0 || height == 0 || width > 65535 || height > 65535)
    return invalid(ctx, "splat_bin_sort_device: image size must be in 1..65535");
  if (n < 0 || capacity < 0 || capacity >= 0xffffffffLL || !num_entries_dev || !depth_range_dev || !scratch_dev ||
      !gauss_dev || !tile_range_dev || !overflow_dev || (n && (!proj_dev || !entry_offset_dev)))
    return invalid(ctx, "splat_bin_sort_device: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_bin_sort_dev(&ctx->c, proj_dev, entry_offset_dev, n, num_entries_dev, capacity,
                                         depth_range_dev, width, height, scratch_dev, gauss_dev, tile_range_dev,
                                         overflow_dev));
}

SPLAT_API int splat_rasterize_fwd(splat_ctx* ctx, const float* proj_dev, const uint32_t* gauss_dev,
                                  const uint32_t* tile_range_dev, uint32_t width, uint32_t height,
                                  const float background[3], float* image_dev, float* final_t_dev,
                                  uint32_t* n_contrib_dev, uint64_t* pairs_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (width == 0 || height == 0 || width > 65535 || height > 65535)
    return invalid(ctx, "splat_rasterize_fwd: image size must be in 1..65535");
  if (!background || !tile_range_dev || !image_dev || !final_t_dev || !n_contrib_dev)
    return invalid(ctx, "splat_rasterize_fwd: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_raster_fwd(&ctx->c, proj_dev, gauss_dev, tile_range_dev, width, height, background,
                                       image_dev, final_t_dev, n_contrib_dev, pairs_dev));
}

SPLAT_API int splat_rasterize_bwd(splat_ctx* ctx, const float* proj_dev, const uint32_t* gauss_dev,
                                  const uint32_t* tile_range_dev, uint32_t width, uint32_t height,
                                  const float background[3], const float* final_t_dev,
                                  const uint32_t* n_contrib_dev, const float* dimage_dev, float* pgrad_dev,
                                  int64_t cap, uint64_t* pairs_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (width == 0 || height == 0 || width > 65535 || height > 65535)
    return invalid(ctx, "splat_rasterize_bwd: image size must be in 1..65535");
  if (!background || !tile_range_dev || !final_t_dev || !n_contrib_dev || !dimage_dev || !pgrad_dev || cap < 0)
    return invalid(ctx, "splat_rasterize_bwd: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_raster_bwd(&ctx->c, proj_dev, gauss_dev, tile_range_dev, width, height, background,
                                       final_t_dev, n_contrib_dev, dimage_dev, pgrad_dev, cap, pairs_dev));
}

SPLAT_API int splat_rasterize_bwd_deterministic(splat_ctx* ctx, const float* proj_dev, const uint32_t* gauss_dev,
                                                const uint32_t* tile_range_dev, const uint32_t* entry_offset_dev,
                                                int64_t n, int64_t num_entries, uint32_t width, uint32_t height,
                                                const float background[3], const float* final_t_dev,
                                                const uint32_t* n_contrib_dev, const float* dimage_dev,
                                                float* pgrad_dev, int64_t cap) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (width == 0 || height == 0 || width > 65535 || height > 65535)
    return invalid(ctx, "splat_rasterize_bwd_deterministic: image size must be in 1..65535");
  if (n < 0 || cap < n || num_entries < 0 || !background || !tile_range_dev || !final_t_dev || !n_contrib_dev ||
      !dimage_dev || (n && (!entry_offset_dev || !pgrad_dev || !proj_dev)) || (num_entries && !gauss_dev))
    return invalid(ctx, "splat_rasterize_bwd_deterministic: bad buffers");
  Enter e(ctx);
  float* eslot = nullptr;
  Status s = arena_reserve(&ctx->c, (size_t)std::max<int64_t>(num_entries, 1) * 48, (void**)&eslot);
  if (s.good())
    s = launch_raster_bwd_det(&ctx->c, proj_dev, gauss_dev, tile_range_dev, entry_offset_dev, n, num_entries, width,
                              height, background, final_t_dev, n_contrib_dev, dimage_dev, eslot, pgrad_dev, cap);
  return finish(ctx, s);
}

SPLAT_API int splat_project_bwd(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap,
                                const splat_camera* cam, const splat_proj_opts* opts, const float* proj_dev,
                                const float* pgrad_dev, float* grad_planes_dev, void* stats_dev, int32_t absgrad) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!cam_ok(cam)) return invalid(ctx, "splat_project_bwd: camera size must be in 1..65535");
  if (!opts_ok(opts)) return invalid(ctx, "splat_project_bwd: sh_degree must be in 0..3");
  if (n < 0 || cap < n || (n && (!planes_dev || !proj_dev || !pgrad_dev || !grad_planes_dev)))
    return invalid(ctx, "splat_project_bwd: bad buffers");
  Enter e(ctx);
  return finish(ctx, launch_project_bwd(&ctx->c, planes_dev, n, cap, *cam, *opts, proj_dev, pgrad_dev,
                                        grad_planes_dev, stats_dev, absgrad));
}

SPLAT_API int splat_project_bwd_adam(splat_ctx* ctx, float* planes_dev, float* m_dev, float* v_dev, int64_t n,
                                     int64_t cap, const splat_camera* cam, const splat_proj_opts* opts,
                                     const float* proj_dev, const float* pgrad_dev, void* stats_dev, int32_t absgrad,
                                     uint64_t step, const splat_lr* lr, void* bf16_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!cam_ok(cam)) return invalid(ctx, "splat_project_bwd_adam: camera size must be in 1..65535");
  if (!opts_ok(opts)) return invalid(ctx, "splat_project_bwd_adam: sh_degree must be in 0..3");
  if (!lr || step == 0 || n < 0 || cap < n || (n && (!planes_dev || !m_dev || !v_dev || !proj_dev || !pgrad_dev)))
    return invalid(ctx, "splat_project_bwd_adam: bad arguments");
  Enter e(ctx);
  return finish(ctx, launch_project_bwd_adam(&ctx->c, planes_dev, m_dev, v_dev, n, cap, *cam, *opts, proj_dev,
                                             pgrad_dev, stats_dev, absgrad, step, *lr, nullptr, nullptr, bf16_dev));
}

}  // extern "C"

namespace {
struct SplitMix64State {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {  // Box-Muller with u1 kept away from zero (densify.rs:116-121)
    const double u1 = std::max(uniform(), 1e-12);
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.14159265358979323846 * u2);
  }
};
}  // namespace

extern "C" {

SPLAT_API int splat_loss_fwd_bwd(splat_ctx* ctx, const float* pred_dev, const void* target_dev, int32_t target_is_u8,
                                 uint32_t width, uint32_t height, float lambda_dssim, float* grad_dev,
                                 float* out3_dev) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!pred_dev || !target_dev || !grad_dev || !out3_dev || width == 0 || height == 0)
    return invalid(ctx, "splat_loss_fwd_bwd: bad arguments");
  Enter e(ctx);
  return finish(ctx, launch_loss(&ctx->c, pred_dev, target_dev, target_is_u8 ? 1 : 0, width, height, lambda_dssim,
                                 grad_dev, out3_dev));
}

SPLAT_API int splat_adam_step(splat_ctx* ctx, float* planes_dev, const float* grad_planes_dev, float* m_dev,
                              float* v_dev, int64_t n, int64_t cap, uint64_t step, const splat_lr* lr) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!lr || n < 0 || cap < n || step == 0 || (n && (!planes_dev || !grad_planes_dev || !m_dev || !v_dev)))
    return invalid(ctx, "splat_adam_step: bad arguments");
  Enter e(ctx);
  return finish(ctx, launch_adam(&ctx->c, planes_dev, grad_planes_dev, m_dev, v_dev, n, cap, step, *lr));
}

SPLAT_API int splat_densify(splat_ctx* ctx, const float* planes_dev, const float* m_dev, const float* v_dev, int64_t n,
                            int64_t cap, const void* stats_dev, const splat_densify_config* cfg, float extent,
                            uint64_t* rng_state, float* planes_out_dev, float* m_out_dev, float* v_out_dev,
                            int64_t cap_out, splat_densify_report* report) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (!cfg || !rng_state || !report || n < 0 || cap < n || cfg->split_children < 1 || cfg->split_children > 16 ||
      (n && (!planes_dev || !m_dev || !v_dev || !stats_dev || !planes_out_dev || !m_out_dev || !v_out_dev)))
    return invalid(ctx, "splat_densify: bad arguments");
  Enter e(ctx);
  Ctx* c = &ctx->c;
  DensifyParams dp;
  dp.cfg = *cfg;
  dp.extent = extent;
  dp.shrink = logf(0.8f * (float)cfg->split_children);
  const float* accum = static_cast<const float*>(stats_dev);
  const uint32_t* denom = reinterpret_cast<const uint32_t*>(accum + cap);
  const uint32_t* maxr = denom + cap;
  DensifyPlan plan;
  Status s = densify_plan(c, planes_dev, n, cap, accum, denom, maxr, dp, &plan);
  if (!s.good()) return fail(ctx, s);
  report->cloned = plan.cloned;
  report->split = plan.split;
  report->pruned = plan.pruned;
  report->new_count = plan.new_count();
  if ((int64_t)plan.new_count() > cap_out)
    return fail(ctx, Status::make(SPLAT_ERR_CAPACITY, "splat_densify: output capacity too small"));
  SplitMix64State rng{*rng_state};
  const size_t nn = (size_t)plan.split * cfg->split_children * 3;
  std::vector<double> normals(nn);
  for (size_t q = 0; q < nn; q++) normals[q] = rng.normal();
  double* nd = nullptr;
  s = arena_reserve(c, std::max<size_t>(nn, 1) * 8, (void**)&nd);
  if (s.good() && nn) s = cuda_status(cudaMemcpyAsync(nd, normals.data(), nn * 8, cudaMemcpyHostToDevice, c->stream),
                                      "upload normals");
  if (s.good()) s = densify_apply(c, planes_dev, m_dev, v_dev, n, cap, plan, nd, planes_out_dev, m_out_dev, v_out_dev,
                                  cap_out);
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  if (!s.good()) return fail(ctx, s);
  *rng_state = rng.s;
  return SPLAT_OK;
}

SPLAT_API int splat_reset_opacity(splat_ctx* ctx, float* planes_dev, float* m_dev, float* v_dev, int64_t n,
                                  float max_alpha) {
  if (!ctx) return SPLAT_ERR_INVALID;
  if (n < 0 || (n && (!planes_dev || !m_dev || !v_dev))) return invalid(ctx, "splat_reset_opacity: bad arguments");
  Enter e(ctx);
  const float limit = logf(max_alpha / (1.0f - max_alpha));  // inverse_sigmoid (math.rs:454)
  return finish(ctx, launch_reset_opacity(&ctx->c, planes_dev, m_dev, v_dev, n, limit));
}

}  // extern "C"
