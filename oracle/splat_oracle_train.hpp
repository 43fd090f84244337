// Oracle training loop: restatement of the reference's src/train.rs:20-321. TEST
// INFRASTRUCTURE ONLY (see splat_oracle.hpp).
//
// One deliberate difference: the view order and split samples come from the documented
// SplitMix64 generator (splat_oracle.hpp) instead of ChaCha8 (train.rs:184, :205;
// densify.rs:116). The CUDA trainer's host code draws from the same generator in the same
// sequence, so both trainers see identical view orders and split offsets.
#pragma once
#include "splat_oracle.hpp"

namespace ora {

template <class Real> struct TrainConfig {  // train.rs:20-109 (defaults at :77-109)
  uint32_t iterations = 30000;
  Real position_lr_init = ORA_L(0.00016);
  Real position_lr_final = ORA_L(0.0000016);
  uint32_t position_lr_max_steps = 30000;
  Real feature_lr = ORA_L(0.0025);
  Real opacity_lr = ORA_L(0.025);
  Real scaling_lr = ORA_L(0.005);
  Real rotation_lr = ORA_L(0.001);
  Real lambda_dssim = ORA_L(0.2);
  bool densify = true;
  uint32_t densify_from_iter = 500;
  uint32_t densify_until_iter = 15000;
  uint32_t densification_interval = 100;
  uint32_t opacity_reset_interval = 3000;
  Real densify_grad_threshold = ORA_L(0.0002);
  Real percent_dense = ORA_L(0.01);
  Real min_opacity = ORA_L(0.005);
  int64_t max_screen_size = -1;
  bool absgrad = false;
  bool antialias = false;
  bool white_background = false;
  int sh_degree = 3;
  uint32_t sh_degree_interval = 1000;
  Real near_ = ORA_L(0.2);
  uint64_t seed = 0;

  void background(Real bg[3]) const {  // train.rs:113-119
    for (int i = 0; i < 3; i++) bg[i] = white_background ? (Real)1 : (Real)0;
  }
  ProjOpts<Real> proj_opts(int degree) const {  // train.rs:122-129
    ProjOpts<Real> o;
    o.near_ = near_;
    o.eps2d = ORA_L(0.3);
    o.antialias = antialias;
    o.sh_degree = degree;
    return o;
  }
  Real position_lr(uint32_t iteration, Real extent) const {  // train.rs:132-137
    Real t = rclamp((Real)iteration / (Real)std::max<uint32_t>(position_lr_max_steps, 1), (Real)0, (Real)1);
    Real init = position_lr_init * extent;
    Real fin = position_lr_final * extent;
    return rexp(rln(init) * ((Real)1 - t) + rln(fin) * t);
  }
};

template <class Real> struct View {  // dataset.rs:14-26
  Camera<Real> camera;
  std::vector<uint8_t> rgb;
  std::vector<Real> to_real() const {
    std::vector<Real> out(rgb.size());
    for (size_t i = 0; i < rgb.size(); i++) out[i] = (Real)rgb[i] / (Real)255;
    return out;
  }
};

struct StepInfo {
  double loss = 0;
  double psnr = 0;
  uint32_t view = 0;
  uint64_t num_gaussians = 0;
  uint64_t cloned = 0, split = 0, pruned = 0;
  int densified = 0;
  int reset = 0;
  uint64_t entries = 0;
};

// The body of train.rs:196-272, one iteration per call.
template <class Real> struct Trainer {
  std::vector<Gaussian<Real>> model;
  int sh_degree = 0;
  std::vector<View<Real>> views;
  Real extent = 1;
  TrainConfig<Real> cfg;
  Adam<Real> adam;
  DensifyStats<Real> stats;
  SplitMix64 rng{0};
  std::vector<uint32_t> order;
  uint32_t iteration = 0;
  std::vector<Real> last_image;

  void start() {  // train.rs:169-189
    rng = SplitMix64(cfg.seed);
    adam = Adam<Real>(model.size());
    stats = DensifyStats<Real>(model.size());
    sh_degree = 0;
    iteration = 0;
    order.clear();
  }

  // Fisher-Yates over 0..n, consumed from the back (train.rs:203-207).
  void refill_order() {
    const uint32_t n = (uint32_t)views.size();
    order.resize(n);
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    for (uint32_t i = n; i-- > 1;) std::swap(order[i], order[rng.index(i + 1)]);
  }

  StepInfo step() {
    StepInfo info;
    iteration += 1;
    const uint32_t it = iteration;
    if (cfg.sh_degree_interval > 0 && it % cfg.sh_degree_interval == 0 && sh_degree < cfg.sh_degree) sh_degree += 1;
    if (order.empty()) refill_order();
    uint32_t vi = order.back();
    order.pop_back();
    info.view = vi;
    const View<Real>& view = views[vi];
    const Camera<Real>& cam = view.camera;
    const uint32_t w = cam.width, h = cam.height;
    Real bg[3];
    cfg.background(bg);

    // Forward (train.rs:212-223).
    ProjOpts<Real> opts = cfg.proj_opts(sh_degree);
    const size_t n = model.size();
    std::vector<Proj<Real>> projs(n);
    project_all(model.data(), (int64_t)n, cam, opts, projs.data());
    Binning binning;
    bin(projs.data(), (int64_t)n, w, h, binning);
    info.entries = binning.sorted.size();
    RasterSettings<Real> st{w, h, {bg[0], bg[1], bg[2]}};
    RasterOutput<Real> out;
    rasterize_forward(projs.data(), binning, st, out);
    std::vector<Real> gt = view.to_real();
    std::vector<Real> dimage(gt.size());
    Real loss = photometric_loss(out.image.data(), gt.data(), w, h, cfg.lambda_dssim, dimage.data());
    info.loss = loss;

    // Backward (train.rs:226-235).
    std::vector<ProjGrad<Real>> pgrads(n);
    std::vector<Real> abs_grads(2 * n);
    rasterize_backward(projs.data(), (int64_t)n, binning, st, out, dimage.data(), pgrads.data(), abs_grads.data());
    std::vector<Gaussian<Real>> grads(n);
    project_backward_all(model.data(), (int64_t)n, cam, opts, pgrads.data(), grads.data());
    if (cfg.densify && it < cfg.densify_until_iter)
      stats.accumulate(projs.data(), pgrads.data(), cfg.absgrad ? abs_grads.data() : nullptr, n, w, h);

    // Optimiser step (train.rs:238-246).
    LearningRates<Real> lrs{cfg.position_lr(it, extent), cfg.scaling_lr, cfg.rotation_lr,
                            cfg.opacity_lr,              cfg.feature_lr, cfg.feature_lr / (Real)20};
    adam.do_step(model.data(), grads.data(), n, lrs);

    // Density control (train.rs:249-272).
    if (cfg.densify && it < cfg.densify_until_iter) {
      if (it > cfg.densify_from_iter && it % cfg.densification_interval == 0) {
        DensifyConfig<Real> dc;
        dc.grad_threshold = cfg.densify_grad_threshold;
        dc.percent_dense = cfg.percent_dense;
        dc.min_opacity = cfg.min_opacity;
        dc.prune_big_world = cfg.opacity_reset_interval > 0 && it > cfg.opacity_reset_interval;
        dc.max_screen_size = cfg.max_screen_size;
        DensifyReport r = densify_and_prune(model, adam, stats, dc, extent, [&]() { return rng.normal(); });
        info.densified = 1;
        info.cloned = r.cloned;
        info.split = r.split;
        info.pruned = r.pruned;
      }
      bool reset = cfg.opacity_reset_interval > 0 &&
                   (it % cfg.opacity_reset_interval == 0 || (cfg.white_background && it == cfg.densify_from_iter));
      if (reset) {
        reset_opacity(model, adam, ORA_L(0.01));
        info.reset = 1;
      }
    }
    info.psnr = (double)psnr(out.image.data(), gt.data(), gt.size());
    info.num_gaussians = model.size();
    last_image.swap(out.image);
    return info;
  }

  // train.rs:309-321
  Real evaluate(const std::vector<View<Real>>& eval_views) const {
    if (eval_views.empty()) return std::numeric_limits<Real>::quiet_NaN();
    ProjOpts<Real> opts = cfg.proj_opts(sh_degree);
    Real bg[3];
    cfg.background(bg);
    Real total = 0;
    for (const auto& v : eval_views) {
      std::vector<Real> img = render(v.camera, opts, bg);
      std::vector<Real> gt = v.to_real();
      total += psnr(img.data(), gt.data(), gt.size());
    }
    return total / (Real)eval_views.size();
  }

  // render.rs:14-23
  std::vector<Real> render(const Camera<Real>& cam, const ProjOpts<Real>& opts, const Real bg[3]) const {
    const size_t n = model.size();
    std::vector<Proj<Real>> projs(n);
    project_all(model.data(), (int64_t)n, cam, opts, projs.data());
    Binning binning;
    bin(projs.data(), (int64_t)n, cam.width, cam.height, binning);
    RasterSettings<Real> st{cam.width, cam.height, {bg[0], bg[1], bg[2]}};
    RasterOutput<Real> out;
    rasterize_forward(projs.data(), binning, st, out);
    return out.image;
  }
};

}  // namespace ora
