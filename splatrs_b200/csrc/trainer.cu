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
  // Coarse copy for the first cfg.coarse_until iterations (not in the reference): the view
  // box-filtered by cfg.coarse_factor, with the camera scaled to match.
  splat_camera coarse_cam;
  DevBuf coarse_rgb;
};

// Box filter of an 8-bit RGB image by an integer factor f (output pixel (x, y) averages the
// f x f input pixels from (f x, f y), rounded to nearest; rows and columns past the last
// whole block are dropped).
__global__ void box_downscale_u8_kernel(const uint8_t* __restrict__ in, uint32_t w, uint32_t h, uint32_t f,
                                        uint8_t* __restrict__ out, uint32_t w2, uint32_t h2) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)w2 * h2 * 3) return;
  const uint32_t ch = (uint32_t)(i % 3), px = (uint32_t)((i / 3) % w2), py = (uint32_t)(i / 3 / w2);
  uint32_t sum = 0;
  for (uint32_t dy = 0; dy < f; dy++)
    for (uint32_t dx = 0; dx < f; dx++) sum += in[((size_t)(f * py + dy) * w + f * px + dx) * 3 + ch];
  out[i] = (uint8_t)((sum + f * f / 2) / (f * f));
}

// The camera of a view downscaled by f: pixel centres (i + 0.5) / f of the original.
splat_camera scaled_camera(const splat_camera& c, uint32_t f) {
  splat_camera s = c;
  s.width = c.width / f;
  s.height = c.height / f;
  s.fx = c.fx / (float)f;
  s.fy = c.fy / (float)f;
  s.cx = c.cx / (float)f;
  s.cy = c.cy / (float)f;
  return s;
}

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
  DevBuf bf16;  // BF16 render copy of planes 1..14 when cfg.bf16_storage
  int64_t stats_cap = 0;
  ViewBuffers vb;
  std::vector<View*> views;
  SplitMix64 rng;
  std::vector<uint32_t> order;
  uint32_t iteration = 0;
  uint64_t adam_step = 0;
  // Mapped pinned read-back slots, one per iteration in flight: loss, ssim, psnr (f32),
  // entry count (u64), overflow flag; written by a kernel at the end of an iteration.
  uint32_t* slots_host = nullptr;
  void* slots_dev = nullptr;
  cudaEvent_t slot_done[2] = {nullptr, nullptr};
  // Per-iteration arguments: one mapped host slot per iteration in flight, loaded into
  // params_dev by the iteration's first kernel.
  StepParams* params_host = nullptr;
  void* params_host_dev = nullptr;
  DevBuf params_dev;
  // The iteration captured as a CUDA graph, one per read-back slot, and the state it was
  // captured for (sizes, SH degree, buffer addresses); a change of state re-captures.
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  std::vector<uint64_t> gkey;
  int g_uses = 0;           // uncaptured iterations run with the current key
  uint64_t g_launches = 0;  // kernels in one captured iteration
  bool graphs = true;       // false after a failed capture: plain launches from then on
  bool last_replayed = false;
  // Batches (cfg.batch_views > 1): one mapped table per slot, its device copy, and the
  // capacities that size every batch launch (the largest view times the batch).
  int batch = 1;
  BatchTable* batch_host = nullptr;
  void* batch_host_dev = nullptr;
  DevBuf batch_dev;
  uint32_t tiles_cap = 0, loss_cap = 0;
  uint64_t pix_cap = 0;
  // Autotuning (cfg.autotune): Gaussian count at the last tuning, how many tunings ran,
  // and the last one's milliseconds per render pass of every candidate configuration.
  int64_t tuned_n = 0;
  uint32_t tunes = 0;
  float tune_ms[kRasterCandidates] = {};
  // Learned densification: birth iteration and (learning) origin of every Gaussian, the
  // previous densification's records (features, rule action), the network and its Adam
  // state, and what learning did.
  DevBuf birth, birth_next, origin, origin_next, feat, feat_scratch, policy;
  DevBuf rec_x, rec_action, alive, useful, rec_csum, labels, label_counts, train_x, train_y, train_w;
  DevBuf mlp_theta, mlp_m, mlp_v, mlp_grad;
  DevBuf eval_out;  // splat_trainer_evaluate: loss, SSIM, PSNR per view
  DevBuf eslot;     // cfg.deterministic: 12 gradient slots per tile entry (emission order)
  int64_t rec_n = 0;
  bool rec_valid = false;
  bool mlp_ready = false;
  uint64_t mlp_steps = 0, learn_events = 0, learn_records = 0, label_hist[3] = {0, 0, 0};
  uint64_t held_out[3] = {0, 0, 0};  // network correct, rule correct, records (before training on them)
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

// train.rs:132-137 in host f32 with the correctly rounded exp and log the kernels use (the
// platform's expf/logf misround some inputs; one of the 2,000 rates of a 2,000-iteration
// run differs by an ulp).
float position_lr(const splat_train_config& c, uint32_t iteration, float extent) {
  float t = (float)iteration / (float)std::max<uint32_t>(c.position_lr_max_steps, 1u);
  t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
  const float init = c.position_lr_init * extent;
  const float fin = c.position_lr_final * extent;
  return crm::expf_cr(crm::logf_cr(init) * (1.0f - t) + crm::logf_cr(fin) * t);
}

// The statistics are three arrays of `cap` words (grad_accum, denom, max_radii) laid out
// with the model's capacity, as splat_project_bwd expects. They are zero after every
// densification (densify.rs:219), the only time the capacity changes, so a new layout
// starts from zeros.
Status ensure_stats(splat_trainer* t, int64_t cap) {
  if (t->stats_cap == cap) return Status::ok();
  SPLAT_CUDA(cudaStreamSynchronize(t->c->stream));
  SPLAT_TRY(t->stats.ensure((size_t)cap * 20));  // accum, denom, max radius, max gradient, contribution
  t->stats_cap = cap;
  SPLAT_TRY(launch_fill_u32(t->c, t->stats.ptr, t->stats.bytes / 4, 0u));
  return Status::ok();
}

// The BF16 render copy follows the f32 parameters after anything but an optimiser step
// (which rewrites it itself).
Status refresh_bf16(splat_trainer* t) {
  if (!t->cfg.bf16_storage) return Status::ok();
  SPLAT_TRY(t->bf16.ensure((size_t)std::max<int64_t>(t->cur.cap, 1) * (kPlanes - 1) * 8));
  return launch_planes_to_bf16(t->c, t->cur.params.as<float>(), t->n, t->cur.cap, t->bf16.ptr);
}

const void* bf16_copy(const splat_trainer* t) { return t->cfg.bf16_storage ? t->bf16.ptr : nullptr; }

Status reset_stats(splat_trainer* t) {
  return launch_fill_u32(t->c, t->stats.ptr, t->stats.bytes / 4, 0u);
}

// Words per read-back slot: 3 per view (loss, ssim, psnr) and the binning counters.
constexpr int kSlotWords = 32;

// The host side of one iteration (train.rs:196-247): its number, view(s), SH degree,
// learning rates, Adam step and what density control runs after it.
struct IterPlan {
  uint32_t views[kMaxViews] = {};
  int nviews = 1;
  uint32_t it = 0, view = 0;
  int sh_degree = 0;
  splat_lr lr{};
  uint64_t adam_step = 0;
  bool densify_window = false, densify_now = false, reset_now = false;
  bool coarse = false;  // the iteration trains on the views' coarse copies
};

// The camera and target of view v for iteration p (its coarse copy while p.coarse).
const splat_camera& plan_cam(const IterPlan& p, const View& v) { return p.coarse ? v.coarse_cam : v.cam; }
const void* plan_rgb(const IterPlan& p, const View& v) { return p.coarse ? v.coarse_rgb.ptr : v.rgb.ptr; }

IterPlan schedule(splat_trainer* t) {
  const splat_train_config& cfg = t->cfg;
  IterPlan p;
  t->iteration += 1;
  p.it = t->iteration;
  if (cfg.sh_degree_interval > 0 && p.it % cfg.sh_degree_interval == 0 && t->sh_degree < cfg.sh_degree) t->sh_degree++;
  p.sh_degree = t->sh_degree;
  if (t->order.empty()) {
    const uint32_t nv = (uint32_t)t->views.size();
    t->order.resize(nv);
    for (uint32_t i = 0; i < nv; i++) t->order[i] = i;
    for (uint32_t i = nv; i-- > 1;) std::swap(t->order[i], t->order[t->rng.index(i + 1)]);
  }
  p.nviews = t->batch;
  for (int b = 0; b < p.nviews; b++) {
    if (t->order.empty()) {  // a new epoch inside the batch
      const uint32_t nv = (uint32_t)t->views.size();
      t->order.resize(nv);
      for (uint32_t i = 0; i < nv; i++) t->order[i] = i;
      for (uint32_t i = nv; i-- > 1;) std::swap(t->order[i], t->order[t->rng.index(i + 1)]);
    }
    p.views[b] = t->order.back();
    t->order.pop_back();
  }
  p.view = p.views[p.nviews - 1];
  p.lr.mean = position_lr(cfg, p.it, t->extent);
  p.lr.log_scale = cfg.scaling_lr;
  p.lr.quat = cfg.rotation_lr;
  p.lr.opacity = cfg.opacity_lr;
  p.lr.sh_dc = cfg.feature_lr;
  p.lr.sh_rest = cfg.feature_lr / 20.0f;
  t->adam_step += 1;
  p.adam_step = t->adam_step;
  p.densify_window = cfg.densify && p.it < cfg.densify_until_iter;
  p.densify_now = p.densify_window && p.it > cfg.densify_from_iter && p.it % cfg.densification_interval == 0;
  p.reset_now = p.densify_window && cfg.opacity_reset_interval > 0 &&
                (p.it % cfg.opacity_reset_interval == 0 || (cfg.white_background && p.it == cfg.densify_from_iter));
  p.coarse = cfg.coarse_until > 0 && p.it <= cfg.coarse_until;
  return p;
}

std::vector<uint64_t> graph_key(splat_trainer* t, const IterPlan& p) {
  const splat_camera& cam = plan_cam(p, *t->views[p.view]);
  // A batch's launches are sized by the capacities, not by its views' sizes.
  const uint64_t w = t->batch > 1 ? 0 : cam.width, h = t->batch > 1 ? 0 : cam.height;
  std::vector<uint64_t> k = {(uint64_t)t->n, (uint64_t)t->cur.cap, (uint64_t)t->vb.e_cap, (uint64_t)p.sh_degree,
                             (uint64_t)p.densify_window, w, h, t->c->arena.generation, (uint64_t)t->stats_cap,
                             (uint64_t)t->batch, t->tiles_cap, t->pix_cap, t->c->raster.tile_w,
                             t->c->raster.tile_h, t->c->raster.chunk, t->c->raster.ppl};
  for (const DevBuf* b : {&t->cur.params, &t->cur.m, &t->cur.v, &t->bf16, &t->stats, &t->pgrad, &t->eslot, &t->pred_grad, &t->loss_out,
                          &t->params_dev, &t->batch_dev, &t->vb.proj, &t->vb.num_tiles, &t->vb.entry_offset, &t->vb.depth_range,
                          &t->vb.tile_range, &t->vb.gauss, &t->vb.image, &t->vb.final_t, &t->vb.n_contrib,
                          &t->vb.sort_scratch, &t->vb.scan_partial, &t->vb.counters})
    k.push_back((uint64_t)(uintptr_t)b->ptr);
  return k;
}

void drop_graphs(splat_trainer* t) {
  for (cudaGraphExec_t& e : t->exec)
    if (e) {
      cudaGraphExecDestroy(e);
      e = nullptr;
    }
}

// The kernels of one iteration (train.rs:212-246): forward with device-driven binning,
// loss, backward, and the projection backward fused with Adam, which does nothing if the
// binning overflowed; then the read-back kernel for slot `slot`. The camera, Adam step and
// target view come from params_dev (loaded first from the slot's host parameters), so a
// captured copy replays for any view of the same size.
Status body(splat_trainer* t, const IterPlan& p, int slot, bool probe = false) {
  Ctx* c = t->c;
  const splat_train_config& cfg = t->cfg;
  View& view = *t->views[p.view];
  const splat_camera& cam = plan_cam(p, view);
  const float bgv = cfg.white_background ? 1.0f : 0.0f;
  const float bg[3] = {bgv, bgv, bgv};
  splat_proj_opts opts;
  opts.near_plane = cfg.near_plane;
  opts.eps2d = 0.3f;
  opts.antialias = cfg.antialias;
  opts.sh_degree = p.sh_degree;
  opts.fp64_conic = cfg.fp64_conic;
  const int64_t n = t->n, cap = t->cur.cap;
  const StepParams* sp = t->params_dev.as<StepParams>();
  SPLAT_TRY(launch_load_words(c, static_cast<const char*>(t->params_host_dev) + slot * sizeof(StepParams),
                              t->params_dev.ptr, (int)(sizeof(StepParams) / 4)));
  SPLAT_TRY(render_view_dev(c, t->cur.params.as<float>(), n, cap, cam, opts, bg, t->vb, sp, bf16_copy(t)));
  const size_t npix = (size_t)cam.width * cam.height;
  SPLAT_TRY(t->pred_grad.ensure(npix * 12));
  SPLAT_TRY(t->loss_out.ensure(16));
  SPLAT_TRY(launch_loss(c, t->vb.image.as<float>(), plan_rgb(p, view), 1, cam.width, cam.height, cfg.lambda_dssim,
                        t->pred_grad.as<float>(), t->loss_out.as<float>(), sp));
  SPLAT_TRY(t->pgrad.ensure((size_t)cap * 48));
  if (cfg.deterministic) {
    // The reference's reduction (per-entry slots, ordered per-Gaussian sums); writes pgrad.
    SPLAT_TRY(t->eslot.ensure((size_t)std::max<int64_t>(t->vb.e_cap, 1) * 48));
    SPLAT_TRY(launch_raster_bwd_det(c, t->vb.proj.as<float>(), t->vb.gauss.as<uint32_t>(),
                                    t->vb.tile_range.as<uint32_t>(), t->vb.entry_offset.as<uint32_t>(), n, t->vb.e_cap,
                                    cam.width, cam.height, bg, t->vb.final_t.as<float>(),
                                    t->vb.n_contrib.as<uint32_t>(), t->pred_grad.as<float>(), t->eslot.as<float>(),
                                    t->pgrad.as<float>(), cap));
  } else {
    SPLAT_TRY(launch_fill_u32(c, t->pgrad.ptr, (size_t)cap * 12, 0u));
    SPLAT_TRY(launch_raster_bwd(c, t->vb.proj.as<float>(), t->vb.gauss.as<uint32_t>(),
                                t->vb.tile_range.as<uint32_t>(), cam.width, cam.height, bg, t->vb.final_t.as<float>(),
                                t->vb.n_contrib.as<uint32_t>(), t->pred_grad.as<float>(), t->pgrad.as<float>(), cap,
                                nullptr));
  }
  // Optimiser step (train.rs:238-246), fused into the projection backward: the 59
  // gradients per Gaussian go from registers straight into Adam. A probe (autotuning)
  // leaves the model as it is.
  if (!probe)
    SPLAT_TRY(launch_project_bwd_adam(c, t->cur.params.as<float>(), t->cur.m.as<float>(), t->cur.v.as<float>(), n, cap,
                                    cam, opts, t->vb.proj.as<float>(), t->pgrad.as<float>(),
                                    p.densify_window ? t->stats.ptr : nullptr, cfg.absgrad, p.adam_step, p.lr,
                                    t->vb.overflow_flag(), sp, const_cast<void*>(bf16_copy(t)), true));
  SPLAT_TRY(launch_publish_u32_to(c, t->loss_out.as<uint32_t>(), 3, t->vb.counters.as<uint32_t>(), 3,
                                  static_cast<uint32_t*>(t->slots_dev) + kSlotWords * slot));
  return Status::ok();
}

// One batch: every stage one launch over all the batch's views, sized for the capacities
// and driven by the batch table loaded first from the slot's host copy.
Status body_batch(splat_trainer* t, const IterPlan& p, int slot, bool probe = false) {
  Ctx* c = t->c;
  const splat_train_config& cfg = t->cfg;
  const float bgv = cfg.white_background ? 1.0f : 0.0f;
  const float bg[3] = {bgv, bgv, bgv};
  splat_proj_opts opts;
  opts.near_plane = cfg.near_plane;
  opts.eps2d = 0.3f;
  opts.antialias = cfg.antialias;
  opts.sh_degree = p.sh_degree;
  opts.fp64_conic = cfg.fp64_conic;
  const int64_t n = t->n, cap = t->cur.cap, records = (int64_t)t->batch * n, pcap = (int64_t)t->batch * cap;
  const splat_camera& cam0 = plan_cam(p, *t->views[p.views[0]]);  // launch arguments only; the table rules
  const BatchTable* bt = t->batch_dev.as<BatchTable>();
  ViewBuffers& v = t->vb;
  SPLAT_TRY(launch_load_words(c, static_cast<const char*>(t->batch_host_dev) + slot * sizeof(BatchTable),
                              t->batch_dev.ptr, (int)(sizeof(BatchTable) / 4)));
  SPLAT_TRY(v.ensure_batch(records, t->pix_cap, t->tiles_cap));
  const int64_t e_cap = std::max<int64_t>(v.e_cap, 1);
  SPLAT_TRY(v.gauss.ensure((size_t)e_cap * 4));
  SPLAT_TRY(v.sort_scratch.ensure(dev_sort_scratch_bytes(e_cap)));
  SPLAT_TRY(v.scan_partial.ensure(((size_t)std::max<int64_t>(records, 1) / kScanValuesPerBlock + 2) * 8));
  if (v.counters.bytes == 0) {
    SPLAT_TRY(v.counters.ensure(64));
    SPLAT_TRY(launch_fill_u32(c, v.counters.ptr, 16, 0u));
  }
  float* proj = v.proj.as<float>();
  uint32_t* dr = v.depth_range.as<uint32_t>();
  SPLAT_TRY(launch_project_fwd(c, t->cur.params.as<float>(), n, cap, cam0, opts, proj, v.num_tiles.as<uint32_t>(), dr,
                               nullptr, bf16_copy(t), bt));
  SPLAT_TRY(launch_scan_u32_into(c, v.num_tiles.as<uint32_t>(), records, v.entry_offset.as<uint32_t>(), 1,
                                 v.scan_partial.as<uint64_t>(), v.entry_count()));
  SPLAT_TRY(launch_bin_sort_dev(c, proj, v.entry_offset.as<uint32_t>(), records, v.entry_count(), e_cap, dr, cam0.width,
                                cam0.height, v.sort_scratch.ptr, v.gauss.as<uint32_t>(), v.tile_range.as<uint32_t>(),
                                v.overflow_flag(), bt, n, t->tiles_cap));
  SPLAT_TRY(launch_raster_fwd(c, proj, v.gauss.as<uint32_t>(), v.tile_range.as<uint32_t>(), cam0.width, cam0.height, bg,
                              v.image.as<float>(), v.final_t.as<float>(), v.n_contrib.as<uint32_t>(), nullptr, bt,
                              t->tiles_cap));
  SPLAT_TRY(t->pred_grad.ensure(t->pix_cap * 12));
  SPLAT_TRY(t->loss_out.ensure(3 * kMaxViews * 4));
  SPLAT_TRY(launch_loss(c, v.image.as<float>(), nullptr, 1, cam0.width, cam0.height, cfg.lambda_dssim,
                        t->pred_grad.as<float>(), t->loss_out.as<float>(), nullptr, bt, t->loss_cap, t->pix_cap));
  SPLAT_TRY(t->pgrad.ensure((size_t)pcap * 48));
  SPLAT_TRY(launch_fill_u32(c, t->pgrad.ptr, (size_t)pcap * 12, 0u));
  SPLAT_TRY(launch_raster_bwd(c, proj, v.gauss.as<uint32_t>(), v.tile_range.as<uint32_t>(), cam0.width, cam0.height, bg,
                              v.final_t.as<float>(), v.n_contrib.as<uint32_t>(), t->pred_grad.as<float>(),
                              t->pgrad.as<float>(), pcap, nullptr, bt, t->tiles_cap));
  if (!probe)
    SPLAT_TRY(launch_project_bwd_batch_adam(c, t->cur.params.as<float>(), t->cur.m.as<float>(), t->cur.v.as<float>(), n,
                                          cap, opts, proj, t->pgrad.as<float>(), pcap,
                                          p.densify_window ? t->stats.ptr : nullptr, cfg.absgrad, v.overflow_flag(),
                                          bt, const_cast<void*>(bf16_copy(t)), true));
  SPLAT_TRY(launch_publish_u32_to(c, t->loss_out.as<uint32_t>(), 3 * t->batch, v.counters.as<uint32_t>(), 3,
                                  static_cast<uint32_t*>(t->slots_dev) + kSlotWords * slot));
  return Status::ok();
}

// The batch table of plan p: views, their cameras, targets, tile/pixel/SSIM-block offsets.
void fill_batch_table(splat_trainer* t, const IterPlan& p, BatchTable& b) {
  std::memset(&b, 0, sizeof(b));
  b.views = p.nviews;
  b.inv_views = 1.0f / (float)p.nviews;
  b.adam = make_adam_args(p.adam_step, p.lr);
  for (int k = 0; k < p.nviews; k++) {
    const View& v = *t->views[p.views[k]];
    const splat_camera& vc = plan_cam(p, v);
    const uint32_t tx = t->c->raster.tiles_x(vc.width), ty = t->c->raster.tiles_y(vc.height);
    const uint32_t lx = (vc.width + 31) / 32, ly = (vc.height + 31) / 32;
    b.cam[k] = vc;
    b.target[k] = plan_rgb(p, v);
    b.tiles_x[k] = tx;
    b.tile_start[k + 1] = b.tile_start[k] + tx * ty;
    b.loss_blocks_x[k] = lx;
    b.loss_start[k + 1] = b.loss_start[k] + lx * ly;
    b.pix_start[k + 1] = b.pix_start[k] + (uint64_t)vc.width * vc.height;
  }
}

// The slot's host parameters of iteration p: the batch table, or the step parameters.
Status prepare(splat_trainer* t, const IterPlan& p, int slot) {
  if (t->batch > 1) {
    fill_batch_table(t, p, t->batch_host[slot]);
    SPLAT_TRY(t->batch_dev.ensure(sizeof(BatchTable)));
  } else {
    View& view = *t->views[p.view];
    StepParams& hp = t->params_host[slot];
    hp.cam = plan_cam(p, view);
    hp.adam = make_adam_args(p.adam_step, p.lr);
    hp.target = plan_rgb(p, view);
  }
  return t->params_dev.ensure(sizeof(StepParams));
}

// Batch capacities under the context's compositing configuration: the largest view's
// tiles, SSIM blocks and pixels, times the batch.
void size_batch_caps(splat_trainer* t) {
  if (t->batch <= 1) return;
  uint32_t most_tiles = 0, most_loss = 0;
  uint64_t most_pix = 0;
  for (const View* v : t->views) {
    const uint32_t w = v->cam.width, h = v->cam.height;
    most_tiles = std::max(most_tiles, t->c->raster.tiles(w, h));
    most_loss = std::max(most_loss, ((w + 31) / 32) * ((h + 31) / 32));
    most_pix = std::max<uint64_t>(most_pix, (uint64_t)w * h);
  }
  t->tiles_cap = most_tiles * t->batch;
  t->loss_cap = most_loss * t->batch;
  t->pix_cap = most_pix * t->batch;
}

// Captures body() for `slot` into a graph; on any failure graphs are switched off and the
// trainer keeps launching kernels one by one.
void capture(splat_trainer* t, const IterPlan& p, int slot) {
  Ctx* c = t->c;
  if (cudaStreamBeginCapture(t->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    t->graphs = false;
    return;
  }
  cudaStream_t orig = c->stream;
  c->stream = t->cap_stream;
  const uint64_t l0 = c->launches.count;
  const Status s = t->batch > 1 ? body_batch(t, p, slot) : body(t, p, slot);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(t->cap_stream, &g);
  c->stream = orig;
  const uint64_t nl = c->launches.count - l0;
  c->launches.count = l0;
  if (!s.good() || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    t->graphs = false;
    return;
  }
  const cudaError_t ei = cudaGraphInstantiate(&t->exec[slot], g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    t->exec[slot] = nullptr;
    cudaGetLastError();
    t->graphs = false;
    drop_graphs(t);
    return;
  }
  t->g_launches = nl;
}

// Queues one iteration without any host wait and records slot `slot`'s event: the captured
// graph when one matches the current state, else the kernels one by one (the first
// iteration after a change of state, which also sizes every buffer before a capture).
Status enqueue(splat_trainer* t, const IterPlan& p, int slot) {
  Ctx* c = t->c;
  // Scratch of the previous iteration is free for reuse: all of it is consumed on this
  // stream before anything queued now runs.
  arena_reset(c);
  SPLAT_TRY(prepare(t, p, slot));
  if (t->graphs) {
    const std::vector<uint64_t> key = graph_key(t, p);
    if (key != t->gkey) {
      drop_graphs(t);
      t->g_uses = 0;
    } else if (!t->exec[slot] && t->g_uses > 0) {
      capture(t, p, slot);
    }
    if (t->graphs && t->exec[slot]) {
      t->last_replayed = true;
      SPLAT_CUDA(cudaGraphLaunch(t->exec[slot], c->stream));
      c->launches.count += t->g_launches;
      SPLAT_CUDA(cudaEventRecord(t->slot_done[slot], c->stream));
      return Status::ok();
    }
  }
  t->last_replayed = false;
  SPLAT_TRY(t->batch > 1 ? body_batch(t, p, slot) : body(t, p, slot));
  SPLAT_CUDA(cudaEventRecord(t->slot_done[slot], c->stream));
  if (t->graphs) {
    t->gkey = graph_key(t, p);  // the state after this iteration's allocations
    t->g_uses++;
  }
  return Status::ok();
}

struct SlotResult {
  float loss, psnr;
  uint64_t entries;
  bool overflow;  // the binning overflowed its capacity (bit 1) or its sort failed (bit 2)
  bool timeout;   // the sort's look-back wait ran out (bit 2): an error, not a capacity matter
};

SlotResult read_slot(splat_trainer* t, int slot) {
  const volatile uint32_t* w = t->slots_host + kSlotWords * slot;
  const int nv = t->batch;
  SlotResult r;
  double loss = 0.0, psnr = 0.0;
  for (int v = 0; v < nv; v++) {  // the mean over the batch's views
    float l, q;
    uint32_t b0 = w[3 * v], b2 = w[3 * v + 2];
    std::memcpy(&l, &b0, 4);
    std::memcpy(&q, &b2, 4);
    loss += l;
    psnr += q;
  }
  r.loss = (float)(loss / nv);
  r.psnr = (float)(psnr / nv);
  r.entries = (uint64_t)w[3 * nv] | ((uint64_t)w[3 * nv + 1] << 32);
  r.overflow = w[3 * nv + 2] != 0;
  r.timeout = (w[3 * nv + 2] & 2u) != 0;
  return r;
}

// After an overflow: room for the view that overflowed with a margin, the flag cleared. A
// failed sort is an error instead.
Status grow_entries(splat_trainer* t, const SlotResult& r) {
  if (r.timeout) return Status::make(SPLAT_ERR_TIMEOUT, "radix sort: a tile's look-back wait ran out");
  const uint64_t entries = r.entries;
  t->vb.e_cap = std::max<int64_t>(t->vb.e_cap * 2, (int64_t)(entries + entries / 4 + 4096));
  if (t->vb.e_cap >= 0xffffffffLL) return Status::make(SPLAT_ERR_CAPACITY, "too many tile entries for 32-bit offsets");
  return launch_fill_u32(t->c, t->vb.overflow_flag(), 1, 0u);
}

// The densification network's parameters on the device (Xavier-uniform from the seed
// unless set by splat_trainer_set_mlp) and its Adam state.
Status ensure_mlp(splat_trainer* t) {
  const size_t np = (size_t)mlp_num_params();
  if (t->mlp_theta.bytes >= np * 4 && t->mlp_ready) return Status::ok();
  for (DevBuf* b : {&t->mlp_theta, &t->mlp_m, &t->mlp_v, &t->mlp_grad}) SPLAT_TRY(b->ensure(np * 4));
  if (!t->mlp_ready) {
    std::vector<float> th(np, 0.0f);
    SplitMix64 r(t->cfg.seed ^ 0x6d6c7064656e7369ull);
    const int dims[3][2] = {{16, 64}, {64, 64}, {64, 3}};
    size_t o = 0;
    for (auto& d : dims) {
      const double lim = std::sqrt(6.0 / (d[0] + d[1]));
      for (int k = 0; k < d[0] * d[1]; k++) th[o++] = (float)((2.0 * r.uniform() - 1.0) * lim);
      o += d[1];  // bias
    }
    SPLAT_CUDA(cudaMemcpyAsync(t->mlp_theta.ptr, th.data(), np * 4, cudaMemcpyHostToDevice, t->c->stream));
    SPLAT_CUDA(cudaStreamSynchronize(t->c->stream));
    t->mlp_ready = true;
  }
  SPLAT_TRY(launch_fill_u32(t->c, t->mlp_m.ptr, np, 0u));
  SPLAT_TRY(launch_fill_u32(t->c, t->mlp_v.ptr, np, 0u));
  return Status::ok();
}

// Opacity a descendant needs at the next densification for its edit to count as useful.
constexpr float kUsefulOpacity = 0.02f;

// Labels the previous densification's records from what became of their descendants and
// trains the network on a strided, class-weighted subset (40 Adam steps).
Status learn_from_previous(splat_trainer* t) {
  Ctx* c = t->c;
  const int64_t rn = t->rec_n;
  for (DevBuf* b : {&t->alive, &t->useful, &t->rec_csum, &t->labels}) SPLAT_TRY(b->ensure((size_t)rn * 4));
  SPLAT_TRY(t->label_counts.ensure(64));
  // The window's contribution of every current Gaussian: the fifth statistics array.
  const float* contrib = t->stats.as<float>() + 4 * t->stats_cap;
  SPLAT_TRY(launch_hindsight_labels(c, t->cur.params.as<float>(), t->n, t->origin.as<uint32_t>(), rn,
                                    t->rec_action.as<uint32_t>(), kUsefulOpacity, contrib,
                                    t->cfg.learn_contribution, t->alive.as<uint32_t>(), t->useful.as<uint32_t>(),
                                    t->rec_csum.as<float>(), t->labels.as<int32_t>(),
                                    t->label_counts.as<unsigned long long>()));
  unsigned long long cnt[3];
  SPLAT_CUDA(cudaMemcpyAsync(cnt, t->label_counts.ptr, 24, cudaMemcpyDeviceToHost, c->stream));
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  const double total = (double)(cnt[0] + cnt[1] + cnt[2]);
  if (total == 0.0) return Status::ok();
  // Held-out accuracy: the network predicts these labels before it trains on them.
  SPLAT_TRY(t->policy.ensure((size_t)rn * 12));
  SPLAT_TRY(mlp_forward_tc_checked(c, t->rec_x.as<float>(), rn, t->mlp_theta.as<float>(), t->policy.as<float>()));
  unsigned long long* acc = t->label_counts.as<unsigned long long>() + 3;
  SPLAT_TRY(launch_fill_u32(c, acc, 6, 0u));
  SPLAT_TRY(launch_label_accuracy(c, t->policy.as<float>(), t->rec_action.as<uint32_t>(), t->labels.as<int32_t>(), rn,
                                  acc));
  unsigned long long ha[3];
  SPLAT_CUDA(cudaMemcpyAsync(ha, acc, 24, cudaMemcpyDeviceToHost, c->stream));
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 3; k++) t->held_out[k] += ha[k];
  const int64_t cap_m = 65536;
  const int64_t stride = std::max<int64_t>(1, (rn + cap_m - 1) / cap_m);
  const int64_t first = (int64_t)(t->learn_events % (uint64_t)stride);
  const int64_t m = (rn - first + stride - 1) / stride;
  float w[3];
  // Balanced classes: each outcome weighs as much in total.
  for (int k = 0; k < 3; k++) w[k] = cnt[k] ? (float)(total / (3.0 * (double)cnt[k])) : 0.0f;
  SPLAT_TRY(t->train_x.ensure((size_t)m * 64));
  SPLAT_TRY(t->train_y.ensure((size_t)m * 4));
  SPLAT_TRY(t->train_w.ensure((size_t)m * 4));
  SPLAT_TRY(launch_gather_training(c, t->rec_x.as<float>(), t->labels.as<int32_t>(), rn, first, stride, w,
                                   t->train_x.as<float>(), t->train_y.as<int32_t>(), t->train_w.as<float>(), m));
  const size_t np = (size_t)mlp_num_params();
  // 40 Adam steps, the gradients on tcgen05; one check of its timeout word at the end.
  SPLAT_TRY(mlp_tc_error_clear(c));
  for (int k = 0; k < 40; k++) {
    SPLAT_TRY(launch_fill_u32(c, t->mlp_grad.ptr, np, 0u));
    SPLAT_TRY(launch_mlp_grad_tc(c, t->train_x.as<float>(), t->train_y.as<int32_t>(), t->train_w.as<float>(), m,
                                 1.0f / (float)m, t->mlp_theta.as<float>(), t->mlp_grad.as<float>(),
                                 mlp_tc_error_word(c)));
    SPLAT_TRY(launch_mlp_adam(c, t->mlp_theta.as<float>(), t->mlp_grad.as<float>(), t->mlp_m.as<float>(),
                              t->mlp_v.as<float>(), ++t->mlp_steps, 1e-3f));
  }
  SPLAT_TRY(mlp_tc_error_check(c));
  t->learn_events++;
  t->learn_records += (uint64_t)m;
  for (int k = 0; k < 3; k++) t->label_hist[k] += cnt[k];
  return Status::ok();
}

// Density control after iteration p (train.rs:249-272); synchronises.
Status density_control(splat_trainer* t, const IterPlan& p, splat_step_info* info) {
  Ctx* c = t->c;
  const splat_train_config& cfg = t->cfg;
  const int64_t n = t->n, cap = t->cur.cap;
  if (p.densify_now) {
    DensifyParams dp;
    dp.cfg.grad_threshold = cfg.densify_grad_threshold;
    dp.cfg.percent_dense = cfg.percent_dense;
    dp.cfg.min_opacity = cfg.min_opacity;
    dp.cfg.prune_big_world = cfg.opacity_reset_interval > 0 && p.it > cfg.opacity_reset_interval;
    dp.cfg.max_world_size_frac = 0.1f;
    dp.cfg.max_screen_size = cfg.max_screen_size;
    dp.cfg.split_children = 2;
    dp.extent = t->extent;
    dp.shrink = crm::logf_cr(0.8f * (float)dp.cfg.split_children);
    float* accum = t->stats.as<float>();
    uint32_t* denom = reinterpret_cast<uint32_t*>(accum + t->stats_cap);
    uint32_t* maxr = denom + t->stats_cap;
    float* maxg = reinterpret_cast<float*>(maxr + t->stats_cap);
    const float* contrib = maxg + t->stats_cap;
    // Learned densification: features of every Gaussian; learning labels the previous
    // records and trains; applying turns the network's probabilities into a policy.
    const bool learn = cfg.learned_densify == 1, apply = cfg.learned_densify == 2;
    SPLAT_TRY(t->birth.ensure((size_t)std::max<int64_t>(cap, 1) * 4));
    if (learn || apply) {
      SPLAT_TRY(ensure_mlp(t));
      SPLAT_TRY(t->feat.ensure((size_t)std::max<int64_t>(n, 1) * 64));
      SPLAT_TRY(t->feat_scratch.ensure(densify_features_scratch_bytes(n)));
      SPLAT_TRY(launch_densify_features(c, t->cur.params.as<float>(), n, cap, accum, denom, maxr, maxg, contrib,
                                        t->birth.as<uint32_t>(), p.it, cfg.percent_dense * t->extent,
                                        t->feat_scratch.ptr, t->feat.as<float>()));
    }
    if (learn && t->rec_valid && t->rec_n > 0) SPLAT_TRY(learn_from_previous(t));
    if (apply) {
      SPLAT_TRY(t->policy.ensure((size_t)std::max<int64_t>(n, 1) * 12));
      SPLAT_TRY(mlp_forward_tc_checked(c, t->feat.as<float>(), n, t->mlp_theta.as<float>(), t->policy.as<float>()));
      dp.policy = t->policy.as<float>();
      if (cfg.learn_prune_confidence > 0.0f) dp.prune_conf = cfg.learn_prune_confidence;
    }
    if (learn) {
      SPLAT_TRY(t->rec_action.ensure((size_t)std::max<int64_t>(n, 1) * 4));
      dp.action = t->rec_action.as<uint32_t>();
    }
    dp.birth_in = t->birth.as<uint32_t>();
    dp.birth_now = p.it;
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
    if (nn) SPLAT_CUDA(cudaMemcpyAsync(t->normals.ptr, normals.data(), nn * 8, cudaMemcpyHostToDevice, c->stream));
    const int64_t new_n = (int64_t)plan.new_count();
    const int64_t want = std::max<int64_t>(new_n, 1);
    if (t->next.cap < want) SPLAT_TRY(t->next.ensure(std::max<int64_t>(want, cap)));
    SPLAT_TRY(t->birth_next.ensure((size_t)t->next.cap * 4));
    plan.args.birth_out = t->birth_next.as<uint32_t>();
    if (learn) {
      SPLAT_TRY(t->origin_next.ensure((size_t)t->next.cap * 4));
      plan.args.origin_out = t->origin_next.as<uint32_t>();
    }
    SPLAT_TRY(densify_apply(c, t->cur.params.as<float>(), t->cur.m.as<float>(), t->cur.v.as<float>(), n, cap, plan,
                            t->normals.as<double>(), t->next.params.as<float>(), t->next.m.as<float>(),
                            t->next.v.as<float>(), t->next.cap));
    // The normals buffer is read by the scatter; keep the host vector alive until done.
    SPLAT_CUDA(cudaStreamSynchronize(c->stream));
    std::swap(t->cur, t->next);
    std::swap(t->birth, t->birth_next);
    if (learn) {  // this densification's records, to be labelled at the next one
      std::swap(t->origin, t->origin_next);
      std::swap(t->rec_x, t->feat);
      t->rec_n = n;
      t->rec_valid = true;
    }
    t->n = new_n;
    SPLAT_TRY(ensure_stats(t, t->cur.cap));
    SPLAT_TRY(reset_stats(t));
    SPLAT_TRY(refresh_bf16(t));
    info->densified = 1;
    info->cloned = plan.cloned;
    info->split = plan.split;
    info->pruned = plan.pruned;
  }
  if (p.reset_now) {
    const float x = 0.01f;
    const float limit = crm::logf_cr(x / (1.0f - x));  // inverse_sigmoid (math.rs:454)
    SPLAT_TRY(launch_reset_opacity(c, t->cur.params.as<float>(), t->cur.m.as<float>(), t->cur.v.as<float>(), t->n,
                                   limit));
    info->reset = 1;
    t->rec_valid = false;  // opacities restart: the outcome of the last records is unreadable
  }
  return Status::ok();
}

void fill_info(splat_trainer* t, const IterPlan& p, const SlotResult& r, splat_step_info* info) {
  info->loss = r.loss;
  info->psnr = r.psnr;
  info->view = p.view;
  info->num_gaussians = (uint64_t)t->n;
  info->entries = r.entries;
  info->replayed = t->last_replayed ? 1u : 0u;
}

Status initial_capacity(splat_trainer* t) {
  if (t->vb.e_cap == 0)
    t->vb.e_cap = t->cfg.entry_capacity > 0 ? (int64_t)std::min<uint64_t>(t->cfg.entry_capacity, 0xfffffffeull)
                                            : std::max<int64_t>(8 * t->batch * std::max<int64_t>(t->n, 1), 1 << 16);
  return ensure_stats(t, t->cur.cap);
}

// Autotuning is due before the first iteration and whenever the Gaussian count has doubled
// or halved since the last tuning (a tuning costs about a hundred probe passes, so a growing
// model is retuned a handful of times, not at every densification).
bool tune_due(const splat_trainer* t) {
  if (!t->cfg.autotune) return false;
  if (t->tunes == 0) return true;
  return t->n >= 2 * t->tuned_n || 2 * t->n <= t->tuned_n;
}

// Times iteration p's render stages (a probe: everything but the optimiser step, so the
// model is left as it is) under every compositing configuration and keeps the fastest.
// Needs no iteration in flight; uses slot 0.
Status autotune(splat_trainer* t, const IterPlan& p) {
  Ctx* c = t->c;
  auto pass = [&](bool warm) -> Status {
    arena_reset(c);
    if (warm) {
      size_batch_caps(t);
      SPLAT_TRY(prepare(t, p, 0));
    }
    for (;;) {
      SPLAT_TRY(t->batch > 1 ? body_batch(t, p, 0, true) : body(t, p, 0, true));
      if (!warm) return Status::ok();
      SPLAT_CUDA(cudaStreamSynchronize(c->stream));
      const SlotResult r = read_slot(t, 0);
      if (!r.overflow) return Status::ok();
      SPLAT_TRY(grow_entries(t, r));
      arena_reset(c);
    }
  };
  const Status s = tune_raster(c, pass, 3, t->tune_ms);
  size_batch_caps(t);
  SPLAT_TRY(s);
  t->tuned_n = t->n;
  t->tunes++;
  return Status::ok();
}

// Runs iteration p to completion, redoing it with more room if its binning overflowed.
Status run_one(splat_trainer* t, const IterPlan& p, int slot, SlotResult* out) {
  for (;;) {
    SPLAT_TRY(enqueue(t, p, slot));
    SPLAT_CUDA(cudaEventSynchronize(t->slot_done[slot]));
    *out = read_slot(t, slot);
    if (!out->overflow) return Status::ok();
    SPLAT_TRY(grow_entries(t, *out));
  }
}

Status step(splat_trainer* t, splat_step_info* info) {
  SPLAT_TRY(initial_capacity(t));
  const IterPlan p = schedule(t);
  info->densified = 0;
  info->reset = 0;
  info->cloned = info->split = info->pruned = 0;
  SlotResult r;
  if (tune_due(t)) SPLAT_TRY(autotune(t, p));
  SPLAT_TRY(run_one(t, p, 0, &r));
  SPLAT_TRY(density_control(t, p, info));
  if (p.densify_now || p.reset_now) SPLAT_CUDA(cudaStreamSynchronize(t->c->stream));
  fill_info(t, p, r, info);
  return Status::ok();
}

// `count` iterations with the host one iteration ahead of the device: iteration i+1 is
// queued before iteration i's read-back is checked. Iterations followed by density
// control run to completion first. An overflow at iteration i also voids i+1 (the flag is
// sticky, so i+1's update was skipped too): both are redone, in order, with more room.
Status run(splat_trainer* t, uint32_t count, splat_step_info* info) {
  SPLAT_TRY(initial_capacity(t));
  info->densified = 0;
  info->reset = 0;
  info->cloned = info->split = info->pruned = 0;
  IterPlan pending;
  bool has_pending = false;
  int pending_slot = 0;
  SlotResult r{};
  IterPlan last{};
  for (uint32_t k = 0; k < count; k++) {
    const IterPlan p = schedule(t);
    const int slot = has_pending ? 1 - pending_slot : 0;
    if (!has_pending && tune_due(t)) SPLAT_TRY(autotune(t, p));
    SPLAT_TRY(enqueue(t, p, slot));
    if (has_pending) {
      SPLAT_CUDA(cudaEventSynchronize(t->slot_done[pending_slot]));
      const SlotResult pr = read_slot(t, pending_slot);
      if (pr.overflow) {
        SPLAT_CUDA(cudaEventSynchronize(t->slot_done[slot]));
        SPLAT_TRY(grow_entries(t, pr));
        SlotResult tmp;
        SPLAT_TRY(run_one(t, pending, pending_slot, &tmp));
        SPLAT_TRY(run_one(t, p, slot, &tmp));
      }
      has_pending = false;
    }
    if (p.densify_now || p.reset_now || k + 1 == count) {
      SPLAT_CUDA(cudaEventSynchronize(t->slot_done[slot]));
      r = read_slot(t, slot);
      if (r.overflow) {
        SPLAT_TRY(grow_entries(t, r));
        SPLAT_TRY(run_one(t, p, slot, &r));
      }
      SPLAT_TRY(density_control(t, p, info));
      last = p;
    } else {
      pending = p;
      pending_slot = slot;
      has_pending = true;
    }
  }
  SPLAT_CUDA(cudaStreamSynchronize(t->c->stream));
  fill_info(t, last, r, info);
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
  if (cfg->batch_views > (uint32_t)kMaxViews) {
    splat_ctx_impl(ctx)->last_error = "batch_views exceeds the maximum of 8";
    return SPLAT_ERR_INVALID;
  }
  if (cfg->coarse_until > 0 && cfg->coarse_factor != 2 && cfg->coarse_factor != 4) {
    splat_ctx_impl(ctx)->last_error = "coarse_factor must be 2 or 4";
    return SPLAT_ERR_INVALID;
  }
  if (cfg->deterministic && (cfg->batch_views > 1 || cfg->autotune || cfg->bf16_storage || cfg->fp64_conic ||
                             cfg->learned_densify || cfg->coarse_until ||
                             !splat_ctx_impl(ctx)->raster.reference_tiles())) {
    splat_ctx_impl(ctx)->last_error =
        "deterministic needs one view per iteration, the 16x16 tiles and no autotune, BF16 copy, f64 conics, "
        "learned densification or coarse views";
    return SPLAT_ERR_INVALID;
  }
  splat_trainer* t = new (std::nothrow) splat_trainer();
  if (!t) return SPLAT_ERR_INVALID;
  t->ctx = ctx;
  t->c = splat_ctx_impl(ctx);
  t->cfg = *cfg;
  t->extent = extent;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(t->c->device);
  bool ok = cudaHostAlloc((void**)&t->slots_host, 2 * kSlotWords * 4, cudaHostAllocMapped) == cudaSuccess;
  ok = ok && cudaHostGetDevicePointer(&t->slots_dev, t->slots_host, 0) == cudaSuccess;
  for (cudaEvent_t& ev : t->slot_done) ok = ok && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
  cudaSetDevice(prev);
  if (!ok) {
    cudaGetLastError();
    for (cudaEvent_t ev : t->slot_done)
      if (ev) cudaEventDestroy(ev);
    if (t->slots_host) cudaFreeHost(t->slots_host);
    delete t;
    return SPLAT_ERR_CUDA;
  }
  std::memset(t->slots_host, 0, 2 * kSlotWords * 4);
  cudaSetDevice(t->c->device);
  ok = cudaHostAlloc((void**)&t->params_host, 2 * sizeof(StepParams), cudaHostAllocMapped) == cudaSuccess;
  ok = ok && cudaHostGetDevicePointer(&t->params_host_dev, t->params_host, 0) == cudaSuccess;
  ok = ok && cudaHostAlloc((void**)&t->batch_host, 2 * sizeof(BatchTable), cudaHostAllocMapped) == cudaSuccess;
  ok = ok && cudaHostGetDevicePointer(&t->batch_host_dev, t->batch_host, 0) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&t->cap_stream, cudaStreamNonBlocking) == cudaSuccess;
  cudaSetDevice(prev);
  if (!ok) {
    cudaGetLastError();
    t->c->last_error = "splat_trainer_create: host or stream allocation failed";
    splat_trainer_destroy(t);
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
    for (DevBuf* b : {&t->pgrad, &t->stats, &t->pred_grad, &t->loss_out, &t->normals, &t->init, &t->bf16, &t->eslot})
      b->release();
    for (DevBuf* b : {&t->birth, &t->birth_next, &t->origin, &t->origin_next, &t->feat, &t->feat_scratch, &t->policy,
                      &t->rec_x, &t->rec_action, &t->alive, &t->useful, &t->rec_csum, &t->labels, &t->label_counts,
                      &t->train_x, &t->eval_out,
                      &t->train_y, &t->train_w, &t->mlp_theta, &t->mlp_m, &t->mlp_v, &t->mlp_grad})
      b->release();
    t->vb.release();
    for (View* v : t->views) {
      v->rgb.release();
      v->coarse_rgb.release();
      delete v;
    }
    t->views.clear();
    drop_graphs(t);
    t->params_dev.release();
    for (cudaEvent_t ev : t->slot_done)
      if (ev) cudaEventDestroy(ev);
    if (t->slots_host) cudaFreeHost(t->slots_host);
    if (t->params_host) cudaFreeHost(t->params_host);
    if (t->batch_host) cudaFreeHost(t->batch_host);
    t->batch_dev.release();
    if (t->cap_stream) cudaStreamDestroy(t->cap_stream);
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
  t->batch = t->cfg.batch_views > 1 ? (int)t->cfg.batch_views : 1;
  size_batch_caps(t);
  t->tuned_n = 0;
  t->tunes = 0;
  t->iteration = 0;
  t->adam_step = 0;
  t->sh_degree = 0;
  Status s = ensure_stats(t, t->cur.cap);
  if (s.good()) s = reset_stats(t);
  if (s.good()) s = cuda_status(cudaMemsetAsync(t->cur.m.ptr, 0, t->cur.m.bytes, c->stream), "zero m");
  if (s.good()) s = cuda_status(cudaMemsetAsync(t->cur.v.ptr, 0, t->cur.v.bytes, c->stream), "zero v");
  if (s.good()) s = refresh_bf16(t);
  if (s.good()) s = t->birth.ensure((size_t)std::max<int64_t>(t->cur.cap, 1) * 4);
  if (s.good()) s = launch_fill_u32(c, t->birth.ptr, t->birth.bytes / 4, 0u);
  t->rec_n = 0;
  t->rec_valid = false;
  // Coarse copies of the views for the first coarse_until iterations.
  if (t->cfg.coarse_until > 0) {
    const uint32_t f = t->cfg.coarse_factor;
    for (View* v : t->views) {
      if (!s.good()) break;
      v->coarse_cam = scaled_camera(v->cam, f);
      if (v->coarse_cam.width == 0 || v->coarse_cam.height == 0) {
        s = Status::make(SPLAT_ERR_INVALID, "a view is smaller than coarse_factor");
        break;
      }
      const uint64_t outs = (uint64_t)v->coarse_cam.width * v->coarse_cam.height * 3;
      s = v->coarse_rgb.ensure(outs);
      if (s.good()) {
        box_downscale_u8_kernel<<<ceil_div(outs, 256), 256, 0, c->stream>>>(
            static_cast<const uint8_t*>(v->rgb.ptr), v->cam.width, v->cam.height, f,
            static_cast<uint8_t*>(v->coarse_rgb.ptr), v->coarse_cam.width, v->coarse_cam.height);
        c->launches.count++;
        s = cuda_status(cudaGetLastError(), "box_downscale_u8_kernel");
      }
    }
  }
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

SPLAT_API int splat_trainer_run(splat_trainer* t, uint32_t iterations, splat_step_info* info) {
  if (!t || !info) return SPLAT_ERR_INVALID;
  if (t->views.empty()) {
    t->c->last_error = "no training views";
    return SPLAT_ERR_INVALID;
  }
  if (iterations == 0) return SPLAT_OK;
  TEnter e(t);
  Status s = run(t, iterations, info);
  return s.good() ? SPLAT_OK : tfail(t, s);
}

SPLAT_API int64_t splat_trainer_count(const splat_trainer* t) { return t ? t->n : -1; }

SPLAT_API int splat_trainer_get_mlp(splat_trainer* t, float* theta_host) {
  if (!t || !theta_host) return SPLAT_ERR_INVALID;
  TEnter e(t);
  Status s = ensure_mlp(t);
  if (s.good())
    s = cuda_status(cudaMemcpyAsync(theta_host, t->mlp_theta.ptr, (size_t)mlp_num_params() * 4, cudaMemcpyDeviceToHost,
                                    t->c->stream),
                    "download network");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(t->c->stream), "cudaStreamSynchronize");
  return s.good() ? SPLAT_OK : tfail(t, s);
}

SPLAT_API int splat_trainer_set_mlp(splat_trainer* t, const float* theta_host) {
  if (!t || !theta_host) return SPLAT_ERR_INVALID;
  TEnter e(t);
  t->mlp_ready = true;  // the caller's parameters replace the initialisation
  Status s = ensure_mlp(t);
  if (s.good())
    s = cuda_status(cudaMemcpyAsync(t->mlp_theta.ptr, theta_host, (size_t)mlp_num_params() * 4, cudaMemcpyHostToDevice,
                                    t->c->stream),
                    "upload network");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(t->c->stream), "cudaStreamSynchronize");
  return s.good() ? SPLAT_OK : tfail(t, s);
}

SPLAT_API int splat_trainer_mlp_stats(const splat_trainer* t, uint64_t out[9]) {
  if (!t || !out) return SPLAT_ERR_INVALID;
  out[6] = t->held_out[0];
  out[7] = t->held_out[1];
  out[8] = t->held_out[2];
  out[0] = t->learn_events;
  out[1] = t->learn_records;
  out[2] = t->label_hist[0];
  out[3] = t->label_hist[1];
  out[4] = t->label_hist[2];
  out[5] = t->mlp_steps;
  return SPLAT_OK;
}
SPLAT_API int splat_trainer_tuning(const splat_trainer* t, float* ms_out, uint32_t* picked, uint32_t* tunes) {
  if (!t) return SPLAT_ERR_INVALID;
  if (ms_out)
    for (int k = 0; k < kRasterCandidates; k++) ms_out[k] = t->tune_ms[k];
  if (picked) {
    picked[0] = t->c->raster.tile_w;
    picked[1] = t->c->raster.tile_h;
    picked[2] = t->c->raster.chunk;
    picked[3] = t->c->raster.ppl;
  }
  if (tunes) *tunes = t->tunes;
  return SPLAT_OK;
}
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

// Adam's first and second moments (Adam::m, Adam::v, reference src/adam.rs:28-41) in the
// 59-float record layout, like splat_trainer_get_model.
SPLAT_API int splat_trainer_get_moments(splat_trainer* t, float* m_aos59_host, float* v_aos59_host) {
  if (!t || (t->n && (!m_aos59_host || !v_aos59_host))) return SPLAT_ERR_INVALID;
  TEnter e(t);
  Ctx* c = t->c;
  DevBuf tmp;
  Status s = tmp.ensure((size_t)std::max<int64_t>(t->n, 1) * 59 * 4);
  for (int k = 0; k < 2 && s.good(); k++) {
    s = launch_params_to_aos(c, (k ? t->cur.v : t->cur.m).as<float>(), t->n, t->cur.cap, tmp.as<float>());
    if (s.good() && t->n)
      s = cuda_status(cudaMemcpyAsync(k ? v_aos59_host : m_aos59_host, tmp.ptr, (size_t)t->n * 59 * 4,
                                      cudaMemcpyDeviceToHost, c->stream),
                      "download moments");
    if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  }
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
  opts.fp64_conic = t->cfg.fp64_conic;
  Status s = render_view(c, t->cur.params.as<float>(), t->n, t->cur.cap, *cam, opts, bg, t->vb, nullptr, bf16_copy(t));
  if (s.good())
    s = cuda_status(cudaMemcpyAsync(image_host, t->vb.image.ptr, (size_t)cam->width * cam->height * 12,
                                    cudaMemcpyDeviceToHost, c->stream),
                    "download image");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return s.good() ? SPLAT_OK : tfail(t, s);
}

// evaluate (train.rs:309-321) on the device: every training view rendered with the current
// model at the trainer's SH degree and background, and scored by the loss kernel (loss,
// SSIM and PSNR per view, PSNR as loss.rs:175-190). All views are queued without a host
// wait (device-driven binning); if any view's binning overflowed, all are redone with more
// room.
SPLAT_API int splat_trainer_evaluate(splat_trainer* t, float* per_view3_host, double* mean_psnr) {
  if (!t || !mean_psnr) return SPLAT_ERR_INVALID;
  *mean_psnr = NAN;
  const size_t nv = t->views.size();
  if (nv == 0) return SPLAT_OK;  // the reference returns NaN for no views
  TEnter e(t);
  Ctx* c = t->c;
  const float bgv = t->cfg.white_background ? 1.0f : 0.0f;
  const float bg[3] = {bgv, bgv, bgv};
  splat_proj_opts opts;
  opts.near_plane = t->cfg.near_plane;
  opts.eps2d = 0.3f;
  opts.antialias = t->cfg.antialias;
  opts.sh_degree = t->sh_degree;
  opts.fp64_conic = t->cfg.fp64_conic;
  Status s = initial_capacity(t);
  size_t most_pix = 0;
  for (const View* v : t->views) most_pix = std::max(most_pix, (size_t)v->cam.width * v->cam.height);
  if (s.good()) s = t->pred_grad.ensure(most_pix * 12);
  if (s.good()) s = t->eval_out.ensure(nv * 12);
  for (int attempt = 0; s.good(); attempt++) {
    for (size_t k = 0; k < nv && s.good(); k++) {
      const View& v = *t->views[k];
      arena_reset(c);  // the previous view's scratch is consumed on this stream first
      s = render_view_dev(c, t->cur.params.as<float>(), t->n, t->cur.cap, v.cam, opts, bg, t->vb, nullptr,
                          bf16_copy(t));
      if (s.good())
        s = launch_loss(c, t->vb.image.as<float>(), v.rgb.ptr, 1, v.cam.width, v.cam.height, t->cfg.lambda_dssim,
                        t->pred_grad.as<float>(), t->eval_out.as<float>() + 3 * k);
    }
    uint32_t w[4] = {0, 0, 0, 0};
    if (s.good()) s = cuda_status(cudaMemcpyAsync(w, t->vb.counters.ptr, 16, cudaMemcpyDeviceToHost, c->stream),
                                  "read binning counters");
    if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    if (!s.good() || w[2] == 0) break;
    SlotResult gr{};
    gr.entries = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
    gr.overflow = true;
    gr.timeout = (w[2] & 2u) != 0;
    s = grow_entries(t, gr);
  }
  std::vector<float> res(nv * 3);
  if (s.good())
    s = cuda_status(cudaMemcpy(res.data(), t->eval_out.ptr, nv * 12, cudaMemcpyDeviceToHost), "read evaluation");
  if (!s.good()) return tfail(t, s);
  double tot = 0.0;
  for (size_t k = 0; k < nv; k++) tot += res[3 * k + 2];
  *mean_psnr = tot / (double)nv;
  if (per_view3_host) std::memcpy(per_view3_host, res.data(), nv * 12);
  return SPLAT_OK;
}

}  // extern "C"
