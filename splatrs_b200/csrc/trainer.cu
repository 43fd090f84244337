// splat_trainer: the training loop of the reference (src/train.rs:161-306) with every
// stage on the device. The model, its Adam moments, the densification statistics and the
// training views (8-bit pixels) stay resident in device memory; one call runs one
// iteration. The host keeps only the schedule and the seeded generator: the view order
// (an epoch-shuffled order consumed from the back, train.rs:203-207) and the split offsets
// (drawn per split parent, per child, x then y then z, densify.rs:161-191) come from
// SplitMix64 (Steele, Lea & Flood 2014) with Box-Muller normals, in the same sequence as
// the CPU oracle's trainer, so both see the same views and the same splits.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "renderer.cuh"

namespace splat {

namespace {
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed = 0) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {
    const double u1 = std::max(uniform(), 1e-12);
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.14159265358979323846 * u2);
  }
  uint32_t index(uint32_t n) { return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32); }
};

struct View {
  splat_camera cam;
  DevBuf rgb;  // H*W*3 uint8
};

// The model and its optimiser state, in parameter-plane layout with capacity `cap`.
struct ModelBufs {
  DevBuf params, m, v;
  int64_t cap = 0;
  Status ensure(int64_t want) {
    SPLAT_TRY(params.ensure((size_t)want * kPlanes * 16));
    SPLAT_TRY(m.ensure((size_t)want * kPlanes * 16));
    SPLAT_TRY(v.ensure((size_t)want * kPlanes * 16));
    cap = (int64_t)(params.bytes / (kPlanes * 16));
    return Status::ok();
  }
  void release() {
    params.release();
    m.release();
    v.release();
    cap = 0;
  }
};
}  // namespace

}  // namespace splat

using namespace splat;

struct splat_trainer {
  splat_ctx* ctx = nullptr;
  Ctx* c = nullptr;
  splat_train_config cfg{};
  float extent = 1.0f;
  int64_t n = 0;
  int sh_degree = 0;
  ModelBufs cur, next;
  DevBuf pgrad, stats, pred_grad, loss_out, normals, init;
  int64_t stats_cap = 0;
  ViewBuffers vb;
  std::vector<View*> views;
  SplitMix64 rng;
  std::vector<uint32_t> order;
  uint32_t iteration = 0;
  uint64_t adam_step = 0;
  float* loss_host = nullptr;  // pinned
};

namespace {
int tfail(splat_trainer* t, const Status& s) {
  t->c->last_error = s.msg;
  return s.code;
}
struct TEnter {
  splat_trainer* t;
  int prev = -1;
  explicit TEnter(splat_trainer* x) : t(x) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != x->c->device) cudaSetDevice(x->c->device);
    arena_reset(x->c);
  }
  ~TEnter() {
    if (prev >= 0 && prev != t->c->device) cudaSetDevice(prev);
  }
};

// train.rs:132-137 (host f32 with the platform libm, as the reference).
float position_lr(const splat_train_config& c, uint32_t iteration, float extent) {
  float t = (float)iteration / (float)std::max<uint32_t>(c.position_lr_max_steps, 1u);
  t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
  const float init = c.position_lr_init * extent;
  const float fin = c.position_lr_final * extent;
  return expf(logf(init) * (1.0f - t) + logf(fin) * t);
}

// The statistics are three arrays of `cap` words (grad_accum, denom, max_radii) laid out
// with the model's capacity, as splat_project_bwd expects. They are zero after every
// densification (densify.rs:219), the only time the capacity changes, so a new layout
// starts from zeros.
Status ensure_stats(splat_trainer* t, int64_t cap) {
  if (t->stats_cap == cap) return Status::ok();
  SPLAT_CUDA(cudaStreamSynchronize(t->c->stream));
  SPLAT_TRY(t->stats.ensure((size_t)cap * 12));
  t->stats_cap = cap;
  SPLAT_TRY(launch_fill_u32(t->c, t->stats.ptr, t->stats.bytes / 4, 0u));
  return Status::ok();
}

Status reset_stats(splat_trainer* t) {
  return launch_fill_u32(t->c, t->stats.ptr, t->stats.bytes / 4, 0u);
}

Status step(splat_trainer* t, splat_step_info* info) {
  Ctx* c = t->c;
  const splat_train_config& cfg = t->cfg;
  t->iteration += 1;
  const uint32_t it = t->iteration;
  if (cfg.sh_degree_interval > 0 && it % cfg.sh_degree_interval == 0 && t->sh_degree < cfg.sh_degree) t->sh_degree++;
  if (t->order.empty()) {
    const uint32_t nv = (uint32_t)t->views.size();
    t->order.resize(nv);
    for (uint32_t i = 0; i < nv; i++) t->order[i] = i;
    for (uint32_t i = nv; i-- > 1;) std::swap(t->order[i], t->order[t->rng.index(i + 1)]);
  }
  const uint32_t vi = t->order.back();
  t->order.pop_back();
  View& view = *t->views[vi];
  const splat_camera& cam = view.cam;
  const float bgv = cfg.white_background ? 1.0f : 0.0f;
  const float bg[3] = {bgv, bgv, bgv};
  splat_proj_opts opts;
  opts.near_plane = cfg.near_plane;
  opts.eps2d = 0.3f;
  opts.antialias = cfg.antialias;
  opts.sh_degree = t->sh_degree;
  const int64_t n = t->n, cap = t->cur.cap;

  // Forward (train.rs:212-223).
  int64_t entries = 0;
  SPLAT_TRY(render_view(c, t->cur.params.as<float>(), n, cap, cam, opts, bg, t->vb, &entries));
  const size_t npix = (size_t)cam.width * cam.height;
  SPLAT_TRY(t->pred_grad.ensure(npix * 12));
  SPLAT_TRY(t->loss_out.ensure(16));
  SPLAT_TRY(launch_loss(c, t->vb.image.as<float>(), view.rgb.ptr, 1, cam.width, cam.height, cfg.lambda_dssim,
                        t->pred_grad.as<float>(), t->loss_out.as<float>()));
  SPLAT_CUDA(cudaMemcpyAsync(t->loss_host, t->loss_out.ptr, 12, cudaMemcpyDeviceToHost, c->stream));

  // Backward (train.rs:226-235).
  SPLAT_TRY(t->pgrad.ensure((size_t)cap * 48));
  SPLAT_TRY(launch_fill_u32(c, t->pgrad.ptr, (size_t)cap * 12, 0u));
  SPLAT_TRY(launch_raster_bwd(c, t->vb.proj.as<float>(), t->vb.gauss.as<uint32_t>(), t->vb.tile_range.as<uint32_t>(),
                              cam.width, cam.height, bg, t->vb.final_t.as<float>(), t->vb.n_contrib.as<uint32_t>(),
                              t->pred_grad.as<float>(), t->pgrad.as<float>(), cap, nullptr));
  const bool densify_window = cfg.densify && it < cfg.densify_until_iter;
  SPLAT_TRY(ensure_stats(t, cap));
  // Optimiser step (train.rs:238-246), fused into the projection backward: the 59
  // gradients per Gaussian go from registers straight into Adam.
  splat_lr lr;
  lr.mean = position_lr(cfg, it, t->extent);
  lr.log_scale = cfg.scaling_lr;
  lr.quat = cfg.rotation_lr;
  lr.opacity = cfg.opacity_lr;
  lr.sh_dc = cfg.feature_lr;
  lr.sh_rest = cfg.feature_lr / 20.0f;
  t->adam_step += 1;
  SPLAT_TRY(launch_project_bwd_adam(c, t->cur.params.as<float>(), t->cur.m.as<float>(), t->cur.v.as<float>(), n, cap,
                                    cam, opts, t->vb.proj.as<float>(), t->pgrad.as<float>(),
                                    densify_window ? t->stats.ptr : nullptr, cfg.absgrad, t->adam_step, lr));

  // Density control (train.rs:249-272).
  info->densified = 0;
  info->reset = 0;
  info->cloned = info->split = info->pruned = 0;
  if (densify_window) {
    if (it > cfg.densify_from_iter && it % cfg.densification_interval == 0) {
      DensifyParams dp;
      dp.cfg.grad_threshold = cfg.densify_grad_threshold;
      dp.cfg.percent_dense = cfg.percent_dense;
      dp.cfg.min_opacity = cfg.min_opacity;
      dp.cfg.prune_big_world = cfg.opacity_reset_interval > 0 && it > cfg.opacity_reset_interval;
      dp.cfg.max_world_size_frac = 0.1f;
      dp.cfg.max_screen_size = cfg.max_screen_size;
      dp.cfg.split_children = 2;
      dp.extent = t->extent;
      dp.shrink = logf(0.8f * (float)dp.cfg.split_children);
      float* accum = t->stats.as<float>();
      uint32_t* denom = reinterpret_cast<uint32_t*>(accum + t->stats_cap);
      uint32_t* maxr = denom + t->stats_cap;
      DensifyPlan plan;
      SPLAT_TRY(densify_plan(c, t->cur.params.as<float>(), n, cap, accum, denom, maxr, dp, &plan));
      if (cfg.max_gaussians > 0 && plan.new_count() > cfg.max_gaussians) {
        // Growth would pass the configured limit: this densification only prunes.
        dp.grow = false;
        SPLAT_TRY(densify_plan(c, t->cur.params.as<float>(), n, cap, accum, denom, maxr, dp, &plan));
      }
      const size_t nn = (size_t)plan.split * dp.cfg.split_children * 3;
      std::vector<double> normals(nn);
      for (size_t q = 0; q < nn; q++) normals[q] = t->rng.normal();
      SPLAT_TRY(t->normals.ensure(std::max<size_t>(nn, 1) * 8));
      if (nn)
        SPLAT_CUDA(cudaMemcpyAsync(t->normals.ptr, normals.data(), nn * 8, cudaMemcpyHostToDevice, c->stream));
      const int64_t new_n = (int64_t)plan.new_count();
      const int64_t want = std::max<int64_t>(new_n, 1);
      if (t->next.cap < want) SPLAT_TRY(t->next.ensure(std::max<int64_t>(want, cap)));
      SPLAT_TRY(densify_apply(c, t->cur.params.as<float>(), t->cur.m.as<float>(), t->cur.v.as<float>(), n, cap, plan,
                              t->normals.as<double>(), t->next.params.as<float>(), t->next.m.as<float>(),
                              t->next.v.as<float>(), t->next.cap));
      // The normals buffer is read by the scatter; keep the host vector alive until done.
      SPLAT_CUDA(cudaStreamSynchronize(c->stream));
      std::swap(t->cur, t->next);
      t->n = new_n;
      SPLAT_TRY(ensure_stats(t, t->cur.cap));
      SPLAT_TRY(reset_stats(t));
      info->densified = 1;
      info->cloned = plan.cloned;
      info->split = plan.split;
      info->pruned = plan.pruned;
    }
    const bool reset = cfg.opacity_reset_interval > 0 &&
                       (it % cfg.opacity_reset_interval == 0 || (cfg.white_background && it == cfg.densify_from_iter));
    if (reset) {
      const float x = 0.01f;
      const float limit = logf(x / (1.0f - x));  // inverse_sigmoid (math.rs:454)
      SPLAT_TRY(launch_reset_opacity(c, t->cur.params.as<float>(), t->cur.m.as<float>(), t->cur.v.as<float>(), t->n,
                                     limit));
      info->reset = 1;
    }
  }
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  info->loss = t->loss_host[0];
  info->psnr = t->loss_host[2];
  info->view = vi;
  info->num_gaussians = (uint64_t)t->n;
  info->entries = (uint64_t)entries;
  return Status::ok();
}
}  // namespace

extern "C" {

SPLAT_API int splat_trainer_create(splat_ctx* ctx, const splat_train_config* cfg, float extent, splat_trainer** out) {
  if (!ctx || !cfg || !out) return SPLAT_ERR_INVALID;
  *out = nullptr;
  if (cfg->iterations == 0) {
    splat_ctx_impl(ctx)->last_error = "iterations must be at least 1";  // train.rs:172-176
    return SPLAT_ERR_INVALID;
  }
  if (cfg->sh_degree < 0 || cfg->sh_degree > 3) {
    splat_ctx_impl(ctx)->last_error = "sh_degree exceeds the maximum of 3";  // train.rs:177-183
    return SPLAT_ERR_INVALID;
  }
  splat_trainer* t = new (std::nothrow) splat_trainer();
  if (!t) return SPLAT_ERR_INVALID;
  t->ctx = ctx;
  t->c = splat_ctx_impl(ctx);
  t->cfg = *cfg;
  t->extent = extent;
  if (cudaMallocHost(&t->loss_host, 64) != cudaSuccess) {
    cudaGetLastError();
    delete t;
    return SPLAT_ERR_CUDA;
  }
  *out = t;
  return SPLAT_OK;
}

SPLAT_API int splat_trainer_destroy(splat_trainer* t) {
  if (!t) return SPLAT_OK;
  {
    TEnter e(t);
    cudaStreamSynchronize(t->c->stream);
    t->cur.release();
    t->next.release();
    for (DevBuf* b : {&t->pgrad, &t->stats, &t->pred_grad, &t->loss_out, &t->normals, &t->init}) b->release();
    t->vb.release();
    for (View* v : t->views) {
      v->rgb.release();
      delete v;
    }
    t->views.clear();
    if (t->loss_host) cudaFreeHost(t->loss_host);
  }
  delete t;
  return SPLAT_OK;
}

SPLAT_API int splat_trainer_set_model(splat_trainer* t, const float* aos59_host, int64_t n) {
  if (!t) return SPLAT_ERR_INVALID;
  if (n < 0 || (n && !aos59_host)) {
    t->c->last_error = "splat_trainer_set_model: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  TEnter e(t);
  Ctx* c = t->c;
  const int64_t cap = std::max<int64_t>(n, 1);
  Status s = t->cur.ensure(cap);
  if (s.good()) s = t->init.ensure((size_t)cap * 59 * 4);
  if (s.good() && n)
    s = cuda_status(cudaMemcpyAsync(t->init.ptr, aos59_host, (size_t)n * 59 * 4, cudaMemcpyHostToDevice, c->stream),
                    "upload model");
  if (s.good()) s = cuda_status(cudaMemsetAsync(t->cur.params.ptr, 0, t->cur.params.bytes, c->stream), "zero params");
  if (s.good()) s = launch_params_from_aos(c, t->init.as<float>(), n, t->cur.params.as<float>(), t->cur.cap);
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  if (!s.good()) return tfail(t, s);
  t->init.release();
  t->n = n;
  return SPLAT_OK;
}

SPLAT_API int splat_trainer_add_view(splat_trainer* t, const splat_camera* cam, const uint8_t* rgb_host) {
  if (!t) return SPLAT_ERR_INVALID;
  if (!cam || !rgb_host || cam->width == 0 || cam->height == 0 || cam->width > 65535 || cam->height > 65535) {
    t->c->last_error = "splat_trainer_add_view: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  TEnter e(t);
  View* v = new (std::nothrow) View();
  if (!v) return SPLAT_ERR_INVALID;
  v->cam = *cam;
  const size_t bytes = (size_t)cam->width * cam->height * 3;
  Status s = v->rgb.ensure(bytes);
  if (s.good()) s = cuda_status(cudaMemcpy(v->rgb.ptr, rgb_host, bytes, cudaMemcpyHostToDevice), "upload view");
  if (!s.good()) {
    v->rgb.release();
    delete v;
    return tfail(t, s);
  }
  t->views.push_back(v);
  return SPLAT_OK;
}

// train.rs:184-189: fresh generator, optimiser state and statistics; SH degree 0.
SPLAT_API int splat_trainer_start(splat_trainer* t) {
  if (!t) return SPLAT_ERR_INVALID;
  if (t->views.empty()) {
    t->c->last_error = "no training views";  // train.rs:169-171
    return SPLAT_ERR_INVALID;
  }
  TEnter e(t);
  Ctx* c = t->c;
  t->rng = SplitMix64(t->cfg.seed);
  t->order.clear();
  t->iteration = 0;
  t->adam_step = 0;
  t->sh_degree = 0;
  Status s = ensure_stats(t, t->cur.cap);
  if (s.good()) s = reset_stats(t);
  if (s.good()) s = cuda_status(cudaMemsetAsync(t->cur.m.ptr, 0, t->cur.m.bytes, c->stream), "zero m");
  if (s.good()) s = cuda_status(cudaMemsetAsync(t->cur.v.ptr, 0, t->cur.v.bytes, c->stream), "zero v");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return s.good() ? SPLAT_OK : tfail(t, s);
}

SPLAT_API int splat_trainer_step(splat_trainer* t, splat_step_info* info) {
  if (!t || !info) return SPLAT_ERR_INVALID;
  if (t->views.empty()) {
    t->c->last_error = "no training views";
    return SPLAT_ERR_INVALID;
  }
  TEnter e(t);
  Status s = step(t, info);
  return s.good() ? SPLAT_OK : tfail(t, s);
}

SPLAT_API int64_t splat_trainer_count(const splat_trainer* t) { return t ? t->n : -1; }
SPLAT_API int32_t splat_trainer_sh_degree(const splat_trainer* t) { return t ? t->sh_degree : -1; }
SPLAT_API uint32_t splat_trainer_iteration(const splat_trainer* t) { return t ? t->iteration : 0; }

SPLAT_API int splat_trainer_get_model(splat_trainer* t, float* aos59_host) {
  if (!t || (!aos59_host && t->n)) return SPLAT_ERR_INVALID;
  TEnter e(t);
  Ctx* c = t->c;
  DevBuf tmp;
  Status s = tmp.ensure((size_t)std::max<int64_t>(t->n, 1) * 59 * 4);
  if (s.good()) s = launch_params_to_aos(c, t->cur.params.as<float>(), t->n, t->cur.cap, tmp.as<float>());
  if (s.good() && t->n)
    s = cuda_status(cudaMemcpyAsync(aos59_host, tmp.ptr, (size_t)t->n * 59 * 4, cudaMemcpyDeviceToHost, c->stream),
                    "download model");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  tmp.release();
  return s.good() ? SPLAT_OK : tfail(t, s);
}

// render::render of the current model at the trainer's active SH degree and background.
SPLAT_API int splat_trainer_render(splat_trainer* t, const splat_camera* cam, float* image_host) {
  if (!t || !cam || !image_host || cam->width == 0 || cam->height == 0 || cam->width > 65535 || cam->height > 65535)
    return SPLAT_ERR_INVALID;
  TEnter e(t);
  Ctx* c = t->c;
  const float bgv = t->cfg.white_background ? 1.0f : 0.0f;
  const float bg[3] = {bgv, bgv, bgv};
  splat_proj_opts opts;
  opts.near_plane = t->cfg.near_plane;
  opts.eps2d = 0.3f;
  opts.antialias = t->cfg.antialias;
  opts.sh_degree = t->sh_degree;
  Status s = render_view(c, t->cur.params.as<float>(), t->n, t->cur.cap, *cam, opts, bg, t->vb, nullptr);
  if (s.good())
    s = cuda_status(cudaMemcpyAsync(image_host, t->vb.image.ptr, (size_t)cam->width * cam->height * 12,
                                    cudaMemcpyDeviceToHost, c->stream),
                    "download image");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return s.good() ? SPLAT_OK : tfail(t, s);
}

}  // extern "C"
