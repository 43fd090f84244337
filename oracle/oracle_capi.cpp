// C ABI over the CPU oracle, for the test suite and the CPU-baseline leg of the benchmark
// (loaded with ctypes). TEST INFRASTRUCTURE ONLY; the product never links it.
//
// Layouts (all row-major, Real = float for *_f and double for *_d):
//   Gaussian record: 59 Reals = mean[3] log_scale[3] quat[4] opacity sh[16][3]
//                    (reference src/model.rs:16-28).
//   Camera:          18 Reals = width height fx fy cx cy rot[9] trans[3]
//                    (reference src/camera.rs:13-32).
//   Proj record:     15 Reals = mean2d[2] conic[3] depth radius opacity color[3]
//                    tile_min[2] tile_max[2]; the integer fields are stored as exact Reals
//                    (reference src/project.rs:47-64).
//   ProjGrad:        9 Reals = mean2d[2] conic[3] opacity color[3] (src/project.rs:84-93).
#include <condition_variable>
#include <cstdio>
#include <mutex>
#include <unordered_map>

#include "splat_oracle_train.hpp"

namespace ora {

bool Math::cr = false;

// ---------------------------------------------------------------------------------------
// Thread pool
// ---------------------------------------------------------------------------------------
namespace {
thread_local bool t_in_parallel = false;
void t_in_parallel_mark() { t_in_parallel = true; }

struct Pool {
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  const std::function<void(int64_t, int64_t)>* job = nullptr;
  int64_t n = 0, grain = 1;
  std::atomic<int64_t> next{0};
  int active = 0;
  uint64_t generation = 0;
  bool stop = false;
  int size = 1;

  void start(int threads) {
    size = std::max(1, threads);
    for (int i = 0; i < size - 1; i++) workers.emplace_back([this] { loop(); });
  }
  void shutdown() {
    {
      std::lock_guard<std::mutex> g(mu);
      stop = true;
    }
    cv.notify_all();
    for (auto& t : workers) t.join();
    workers.clear();
    stop = false;
  }
  void run_chunks() {
    for (;;) {
      int64_t lo = next.fetch_add(grain);
      if (lo >= n) break;
      (*job)(lo, std::min(n, lo + grain));
    }
  }
  void loop() {
    t_in_parallel_mark();
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || generation != seen; });
        if (stop) return;
        seen = generation;
        active++;
      }
      run_chunks();
      {
        std::lock_guard<std::mutex> g(mu);
        active--;
      }
      done_cv.notify_all();
    }
  }
};

Pool* g_pool = nullptr;
std::mutex g_pool_mu;

Pool& pool() {
  if (!g_pool) {
    g_pool = new Pool();
    unsigned hc = std::thread::hardware_concurrency();
    const char* env = std::getenv("SPLAT_ORACLE_THREADS");
    int n = env ? std::atoi(env) : (int)(hc ? hc : 1);
    g_pool->start(n);
  }
  return *g_pool;
}
}  // namespace

int num_threads() { return pool().size; }

void set_num_threads(int n) {
  std::lock_guard<std::mutex> g(g_pool_mu);
  Pool& p = pool();
  p.shutdown();
  p.start(n);
}

void parallel_for(int64_t n, int64_t grain, const std::function<void(int64_t, int64_t)>& f) {
  if (n <= 0) return;
  grain = std::max<int64_t>(1, grain);
  if (t_in_parallel || n <= grain) {
    f(0, n);
    return;
  }
  std::lock_guard<std::mutex> g(g_pool_mu);
  Pool& p = pool();
  if (p.size == 1) {
    f(0, n);
    return;
  }
  {
    std::lock_guard<std::mutex> lk(p.mu);
    p.job = &f;
    p.n = n;
    p.grain = grain;
    p.next = 0;
    p.generation++;
  }
  p.cv.notify_all();
  t_in_parallel = true;
  p.run_chunks();
  t_in_parallel = false;
  std::unique_lock<std::mutex> lk(p.mu);
  p.done_cv.wait(lk, [&] { return p.active == 0 && p.next.load() >= p.n; });
  p.job = nullptr;
}

void parallel_sort_pairs(std::vector<std::pair<uint64_t, uint32_t>>& v) {
  const int64_t n = (int64_t)v.size();
  int parts = 1;
  while (parts < num_threads()) parts *= 2;
  if (n < 65536 || parts == 1) {
    std::sort(v.begin(), v.end());
    return;
  }
  std::vector<int64_t> bounds(parts + 1);
  for (int i = 0; i <= parts; i++) bounds[i] = n * i / parts;
  parallel_for(parts, 1, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; i++) std::sort(v.begin() + bounds[i], v.begin() + bounds[i + 1]);
  });
  std::vector<std::pair<uint64_t, uint32_t>> tmp(n);
  auto* src = &v;
  auto* dst = &tmp;
  for (int width = 1; width < parts; width *= 2) {
    int merges = parts / (2 * width);
    parallel_for(merges, 1, [&](int64_t lo, int64_t hi) {
      for (int64_t m = lo; m < hi; m++) {
        int64_t a = bounds[2 * width * m], b = bounds[2 * width * m + width], c = bounds[2 * width * (m + 1)];
        std::merge(src->begin() + a, src->begin() + b, src->begin() + b, src->begin() + c, dst->begin() + a);
      }
    });
    std::swap(src, dst);
  }
  if (src != &v) v.swap(tmp);
}

// Exact mean squared distance to the three nearest other points (reference
// src/model.rs:128-186), found with a uniform grid instead of a kd-tree. Coincident points
// count as zero-distance neighbours, as in the reference.
void mean_nn_dist2(const float* pts, int64_t n, double* out) {
  if (n < 2) {
    for (int64_t i = 0; i < n; i++) out[i] = 0;
    return;
  }
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      lo[k] = std::min(lo[k], (double)pts[3 * i + k]);
      hi[k] = std::max(hi[k], (double)pts[3 * i + k]);
    }
  double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-30});
  int64_t dim[3];
  double cell = std::max(ext / std::max(1.0, std::cbrt((double)n / 2.0)), ext / 1000.0);
  for (int k = 0; k < 3; k++) dim[k] = std::max<int64_t>(1, std::min<int64_t>(1024, (int64_t)((hi[k] - lo[k]) / cell) + 1));
  auto cell_of = [&](int64_t i, int k) {
    int64_t c = (int64_t)(((double)pts[3 * i + k] - lo[k]) / cell);
    return std::min(std::max<int64_t>(c, 0), dim[k] - 1);
  };
  const int64_t ncell = dim[0] * dim[1] * dim[2];
  std::vector<int64_t> start(ncell + 1, 0), items(n);
  std::vector<int64_t> cid(n);
  for (int64_t i = 0; i < n; i++) {
    cid[i] = (cell_of(i, 2) * dim[1] + cell_of(i, 1)) * dim[0] + cell_of(i, 0);
    start[cid[i] + 1]++;
  }
  for (int64_t c = 0; c < ncell; c++) start[c + 1] += start[c];
  {
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t i = 0; i < n; i++) items[fill[cid[i]]++] = i;
  }
  parallel_for(n, 1024, [&](int64_t a, int64_t b) {
    for (int64_t i = a; i < b; i++) {
      double best[3] = {1e300, 1e300, 1e300};
      int found = 0;
      int64_t c[3] = {cell_of(i, 0), cell_of(i, 1), cell_of(i, 2)};
      int64_t maxr = std::max({dim[0], dim[1], dim[2]});
      for (int64_t r = 0; r <= maxr; r++) {
        if (found >= 3) {
          double reach = (double)(r - 1) * cell;
          if (reach > 0 && reach * reach > best[2]) break;
        }
        for (int64_t z = c[2] - r; z <= c[2] + r; z++) {
          if (z < 0 || z >= dim[2]) continue;
          for (int64_t y = c[1] - r; y <= c[1] + r; y++) {
            if (y < 0 || y >= dim[1]) continue;
            for (int64_t x = c[0] - r; x <= c[0] + r; x++) {
              if (x < 0 || x >= dim[0]) continue;
              if (std::max({std::llabs(x - c[0]), std::llabs(y - c[1]), std::llabs(z - c[2])}) != r) continue;
              int64_t cc = (z * dim[1] + y) * dim[0] + x;
              for (int64_t q = start[cc]; q < start[cc + 1]; q++) {
                int64_t j = items[q];
                if (j == i) continue;
                double dx = (double)pts[3 * i] - (double)pts[3 * j];
                double dy = (double)pts[3 * i + 1] - (double)pts[3 * j + 1];
                double dz = (double)pts[3 * i + 2] - (double)pts[3 * j + 2];
                double d = dx * dx + dy * dy + dz * dz;
                if (found < 3 || d < best[2]) {
                  int p = std::min(found, 2);
                  best[p] = d;
                  for (int s = p; s > 0 && best[s] < best[s - 1]; s--) std::swap(best[s], best[s - 1]);
                  found = std::min(found + 1, 3);
                }
              }
            }
          }
        }
      }
      double sum = 0;
      for (int s = 0; s < found; s++) sum += best[s];
      out[i] = found > 0 ? sum / (double)found : 0.0;
    }
  });
}

}  // namespace ora

using namespace ora;


namespace {
template <class R> Camera<R> cam_from(const R* c) {
  Camera<R> cam;
  cam.width = (uint32_t)c[0];
  cam.height = (uint32_t)c[1];
  cam.fx = c[2];
  cam.fy = c[3];
  cam.cx = c[4];
  cam.cy = c[5];
  for (int i = 0; i < 9; i++) cam.rot.m[i / 3][i % 3] = c[6 + i];
  cam.trans = V3<R>(c[15], c[16], c[17]);
  return cam;
}
template <class R> void cam_to(const Camera<R>& cam, R* c) {
  c[0] = (R)cam.width;
  c[1] = (R)cam.height;
  c[2] = cam.fx;
  c[3] = cam.fy;
  c[4] = cam.cx;
  c[5] = cam.cy;
  for (int i = 0; i < 9; i++) c[6 + i] = cam.rot.m[i / 3][i % 3];
  c[15] = cam.trans.x;
  c[16] = cam.trans.y;
  c[17] = cam.trans.z;
}
template <class R> ProjOpts<R> opts_from(R near_, R eps2d, int aa, int deg) {
  ProjOpts<R> o;
  o.near_ = near_;
  o.eps2d = eps2d;
  o.antialias = aa != 0;
  o.sh_degree = deg;
  return o;
}
template <class R> void proj_to(const Proj<R>& p, R* o) {
  o[0] = p.mean2d[0];
  o[1] = p.mean2d[1];
  o[2] = p.conic[0];
  o[3] = p.conic[1];
  o[4] = p.conic[2];
  o[5] = p.depth;
  o[6] = (R)p.radius;
  o[7] = p.opacity;
  o[8] = p.color[0];
  o[9] = p.color[1];
  o[10] = p.color[2];
  o[11] = (R)p.tile_min[0];
  o[12] = (R)p.tile_min[1];
  o[13] = (R)p.tile_max[0];
  o[14] = (R)p.tile_max[1];
}
template <class R> Proj<R> proj_from(const R* o) {
  Proj<R> p;
  p.mean2d[0] = o[0];
  p.mean2d[1] = o[1];
  p.conic[0] = o[2];
  p.conic[1] = o[3];
  p.conic[2] = o[4];
  p.depth = o[5];
  p.radius = (uint32_t)o[6];
  p.opacity = o[7];
  p.color[0] = o[8];
  p.color[1] = o[9];
  p.color[2] = o[10];
  p.tile_min[0] = (uint32_t)o[11];
  p.tile_min[1] = (uint32_t)o[12];
  p.tile_max[0] = (uint32_t)o[13];
  p.tile_max[1] = (uint32_t)o[14];
  return p;
}
template <class R> std::vector<Proj<R>> projs_from(const R* p15, int64_t n) {
  std::vector<Proj<R>> v(n);
  for (int64_t i = 0; i < n; i++) v[i] = proj_from(p15 + 15 * i);
  return v;
}

template <class R> void do_project_all(const R* params, int64_t n, const R* cam18, R near_, R eps2d, int aa, int deg,
                                       R* out15) {
  Camera<R> cam = cam_from(cam18);
  ProjOpts<R> o = opts_from(near_, eps2d, aa, deg);
  std::vector<Proj<R>> projs(n);
  project_all(reinterpret_cast<const Gaussian<R>*>(params), n, cam, o, projs.data());
  for (int64_t i = 0; i < n; i++) proj_to(projs[i], out15 + 15 * i);
}

template <class R> void do_project_backward_all(const R* params, int64_t n, const R* cam18, R near_, R eps2d, int aa,
                                                int deg, const R* grads9, R* out59) {
  Camera<R> cam = cam_from(cam18);
  ProjOpts<R> o = opts_from(near_, eps2d, aa, deg);
  std::vector<ProjGrad<R>> g(n);
  for (int64_t i = 0; i < n; i++) {
    const R* s = grads9 + 9 * i;
    g[i].mean2d[0] = s[0];
    g[i].mean2d[1] = s[1];
    g[i].conic[0] = s[2];
    g[i].conic[1] = s[3];
    g[i].conic[2] = s[4];
    g[i].opacity = s[5];
    g[i].color[0] = s[6];
    g[i].color[1] = s[7];
    g[i].color[2] = s[8];
  }
  project_backward_all(reinterpret_cast<const Gaussian<R>*>(params), n, cam, o, g.data(),
                       reinterpret_cast<Gaussian<R>*>(out59));
}

template <class R> Binning* do_bin(const R* p15, int64_t n, uint32_t w, uint32_t h) {
  std::vector<Proj<R>> projs = projs_from(p15, n);
  Binning* b = new Binning();
  if (!bin(projs.data(), n, w, h, *b)) {
    delete b;
    return nullptr;
  }
  return b;
}

// Pairs that passed the alpha threshold in the last forward and backward call (read by
// ora_last_passed_pairs; calls are not expected to overlap).
static std::atomic<uint64_t> g_last_passed[2];

template <class R> void do_raster_fwd(const R* p15, int64_t n, const Binning* b, uint32_t w, uint32_t h, const R* bg,
                                      R* image, R* final_t, uint32_t* n_contrib, uint64_t* pairs) {
  std::vector<Proj<R>> projs = projs_from(p15, n);
  RasterSettings<R> st{w, h, {bg[0], bg[1], bg[2]}};
  RasterOutput<R> out;
  RasterCounters cnt;
  rasterize_forward(projs.data(), *b, st, out, &cnt);
  std::memcpy(image, out.image.data(), out.image.size() * sizeof(R));
  std::memcpy(final_t, out.final_t.data(), out.final_t.size() * sizeof(R));
  std::memcpy(n_contrib, out.n_contrib.data(), out.n_contrib.size() * sizeof(uint32_t));
  if (pairs) *pairs = cnt.pairs_fwd.load();
  g_last_passed[0] = cnt.passed_fwd.load();
}

template <class R> void do_raster_bwd(const R* p15, int64_t n, const Binning* b, uint32_t w, uint32_t h, const R* bg,
                                      const R* final_t, const uint32_t* n_contrib, const R* dimage, R* grads9,
                                      R* abs2, uint64_t* pairs) {
  std::vector<Proj<R>> projs = projs_from(p15, n);
  RasterSettings<R> st{w, h, {bg[0], bg[1], bg[2]}};
  RasterOutput<R> out;
  size_t npix = (size_t)w * h;
  out.final_t.assign(final_t, final_t + npix);
  out.n_contrib.assign(n_contrib, n_contrib + npix);
  std::vector<ProjGrad<R>> g(n);
  RasterCounters cnt;
  rasterize_backward(projs.data(), n, *b, st, out, dimage, g.data(), abs2, &cnt);
  for (int64_t i = 0; i < n; i++) {
    R* d = grads9 + 9 * i;
    d[0] = g[i].mean2d[0];
    d[1] = g[i].mean2d[1];
    d[2] = g[i].conic[0];
    d[3] = g[i].conic[1];
    d[4] = g[i].conic[2];
    d[5] = g[i].opacity;
    d[6] = g[i].color[0];
    d[7] = g[i].color[1];
    d[8] = g[i].color[2];
  }
  if (pairs) *pairs = cnt.pairs_bwd.load();
  g_last_passed[1] = cnt.passed_bwd.load();
}

template <class R> int64_t do_densify(const R* params, const R* m, const R* v, int64_t n0, const R* grad_accum,
                                      const uint32_t* denom, const uint32_t* max_radii, R grad_threshold,
                                      R percent_dense, R min_opacity, int prune_big_world, R max_world_size_frac,
                                      int64_t max_screen_size, int split_children, R extent, const double* normals,
                                      int64_t n_normals, R* out_params, R* out_m, R* out_v, int64_t* report) {
  std::vector<Gaussian<R>> model(reinterpret_cast<const Gaussian<R>*>(params),
                                 reinterpret_cast<const Gaussian<R>*>(params) + n0);
  Adam<R> adam(0);
  adam.m.assign(reinterpret_cast<const Gaussian<R>*>(m), reinterpret_cast<const Gaussian<R>*>(m) + n0);
  adam.v.assign(reinterpret_cast<const Gaussian<R>*>(v), reinterpret_cast<const Gaussian<R>*>(v) + n0);
  DensifyStats<R> stats(n0);
  for (int64_t i = 0; i < n0; i++) {
    stats.grad_accum[i] = grad_accum[i];
    stats.denom[i] = denom[i];
    stats.max_radii[i] = max_radii[i];
  }
  DensifyConfig<R> cfg;
  cfg.grad_threshold = grad_threshold;
  cfg.percent_dense = percent_dense;
  cfg.min_opacity = min_opacity;
  cfg.prune_big_world = prune_big_world != 0;
  cfg.max_world_size_frac = max_world_size_frac;
  cfg.max_screen_size = max_screen_size;
  cfg.split_children = split_children;
  int64_t used = 0;
  bool overrun = false;
  DensifyReport r = densify_and_prune(model, adam, stats, cfg, extent, [&]() -> double {
    if (used >= n_normals) {
      overrun = true;
      return 0.0;
    }
    return normals[used++];
  });
  if (overrun) return -1;
  std::memcpy(out_params, model.data(), model.size() * sizeof(Gaussian<R>));
  std::memcpy(out_m, adam.m.data(), model.size() * sizeof(Gaussian<R>));
  std::memcpy(out_v, adam.v.data(), model.size() * sizeof(Gaussian<R>));
  report[0] = (int64_t)r.cloned;
  report[1] = (int64_t)r.split;
  report[2] = (int64_t)r.pruned;
  report[3] = used;
  return (int64_t)model.size();
}
}  // namespace

#define ORA_API extern "C" __attribute__((visibility("default")))

ORA_API int ora_threads(void) { return num_threads(); }
ORA_API void ora_last_passed_pairs(uint64_t* out2) {
  out2[0] = g_last_passed[0].load();
  out2[1] = g_last_passed[1].load();
}
ORA_API void ora_set_threads(int n) { set_num_threads(n); }
ORA_API void ora_set_cr_math(int on) { Math::cr = on != 0; }
ORA_API float ora_expf(float x) { return rexp(x); }
ORA_API float ora_logf(float x) { return rln(x); }
ORA_API float ora_expf_cr(float x) { return crm::expf_cr(x); }
ORA_API float ora_logf_cr(float x) { return crm::logf_cr(x); }

#define ORA_BOTH(R, S)                                                                                             \
  ORA_API void ora_project_all_##S(const R* params, int64_t n, const R* cam18, R near_, R eps2d, int aa, int deg,   \
                                   R* out15) {                                                                     \
    do_project_all<R>(params, n, cam18, near_, eps2d, aa, deg, out15);                                             \
  }                                                                                                                \
  ORA_API void ora_project_backward_all_##S(const R* params, int64_t n, const R* cam18, R near_, R eps2d, int aa,   \
                                            int deg, const R* grads9, R* out59) {                                  \
    do_project_backward_all<R>(params, n, cam18, near_, eps2d, aa, deg, grads9, out59);                            \
  }                                                                                                                \
  ORA_API void* ora_bin_##S(const R* p15, int64_t n, uint32_t w, uint32_t h) { return do_bin<R>(p15, n, w, h); }   \
  ORA_API void ora_rasterize_forward_##S(const R* p15, int64_t n, const void* b, uint32_t w, uint32_t h,            \
                                         const R* bg, R* image, R* final_t, uint32_t* n_contrib, uint64_t* pairs) { \
    do_raster_fwd<R>(p15, n, (const Binning*)b, w, h, bg, image, final_t, n_contrib, pairs);                       \
  }                                                                                                                \
  ORA_API void ora_rasterize_backward_##S(const R* p15, int64_t n, const void* b, uint32_t w, uint32_t h,           \
                                          const R* bg, const R* final_t, const uint32_t* n_contrib,                \
                                          const R* dimage, R* grads9, R* abs2, uint64_t* pairs) {                  \
    do_raster_bwd<R>(p15, n, (const Binning*)b, w, h, bg, final_t, n_contrib, dimage, grads9, abs2, pairs);        \
  }                                                                                                                \
  ORA_API void ora_naive_render_##S(const R* p15, int64_t n, uint32_t w, uint32_t h, const R* bg, R* image) {      \
    std::vector<Proj<R>> projs = projs_from(p15, n);                                                               \
    naive_render(projs.data(), n, w, h, bg, image);                                                                \
  }                                                                                                                \
  ORA_API R ora_photometric_loss_##S(const R* pred, const R* target, int64_t w, int64_t h, R lambda, R* grad) {     \
    return photometric_loss<R>(pred, target, (size_t)w, (size_t)h, lambda, grad);                                  \
  }                                                                                                                \
  ORA_API R ora_ssim_with_grad_##S(const R* x, const R* y, int64_t w, int64_t h, R* grad) {                         \
    return ssim_with_grad<R>(x, y, (size_t)w, (size_t)h, grad);                                                    \
  }                                                                                                                \
  ORA_API void ora_blur_##S(const R* src, int64_t w, int64_t h, int64_t ch, R* dst) {                              \
    R k[SSIM_WINDOW];                                                                                              \
    gaussian_kernel(k);                                                                                            \
    blur<R>(src, (size_t)w, (size_t)h, (size_t)ch, k, dst);                                                        \
  }                                                                                                                \
  ORA_API R ora_psnr_##S(const R* pred, const R* target, int64_t n) { return psnr<R>(pred, target, (size_t)n); }    \
  ORA_API uint64_t ora_adam_step_##S(R* params, const R* grads, R* m, R* v, int64_t n, uint64_t step,               \
                                     const R* lr6) {                                                               \
    Adam<R> adam(0);                                                                                               \
    adam.m.assign((Gaussian<R>*)m, (Gaussian<R>*)m + n);                                                           \
    adam.v.assign((Gaussian<R>*)v, (Gaussian<R>*)v + n);                                                           \
    adam.step = step;                                                                                              \
    LearningRates<R> lr{lr6[0], lr6[1], lr6[2], lr6[3], lr6[4], lr6[5]};                                           \
    adam.do_step((Gaussian<R>*)params, (const Gaussian<R>*)grads, (size_t)n, lr);                                  \
    std::memcpy(m, adam.m.data(), n * sizeof(Gaussian<R>));                                                        \
    std::memcpy(v, adam.v.data(), n * sizeof(Gaussian<R>));                                                        \
    return adam.step;                                                                                              \
  }                                                                                                                \
  ORA_API void ora_densify_accumulate_##S(const R* p15, const R* grads9, const R* abs2, int64_t n, uint32_t w,      \
                                          uint32_t h, R* grad_accum, uint32_t* denom, uint32_t* max_radii) {       \
    DensifyStats<R> st(n);                                                                                         \
    std::memcpy(st.grad_accum.data(), grad_accum, n * sizeof(R));                                                  \
    std::memcpy(st.denom.data(), denom, n * 4);                                                                    \
    std::memcpy(st.max_radii.data(), max_radii, n * 4);                                                            \
    std::vector<Proj<R>> projs = projs_from(p15, n);                                                               \
    std::vector<ProjGrad<R>> g(n);                                                                                 \
    for (int64_t i = 0; i < n; i++) {                                                                              \
      g[i].mean2d[0] = grads9[9 * i];                                                                              \
      g[i].mean2d[1] = grads9[9 * i + 1];                                                                          \
    }                                                                                                              \
    st.accumulate(projs.data(), g.data(), abs2, (size_t)n, w, h);                                                  \
    std::memcpy(grad_accum, st.grad_accum.data(), n * sizeof(R));                                                  \
    std::memcpy(denom, st.denom.data(), n * 4);                                                                    \
    std::memcpy(max_radii, st.max_radii.data(), n * 4);                                                            \
  }                                                                                                                \
  ORA_API int64_t ora_densify_##S(const R* params, const R* m, const R* v, int64_t n0, const R* grad_accum,         \
                                  const uint32_t* denom, const uint32_t* max_radii, R grad_threshold,              \
                                  R percent_dense, R min_opacity, int prune_big_world, R max_world_size_frac,      \
                                  int64_t max_screen_size, int split_children, R extent, const double* normals,    \
                                  int64_t n_normals, R* out_params, R* out_m, R* out_v, int64_t* report) {         \
    return do_densify<R>(params, m, v, n0, grad_accum, denom, max_radii, grad_threshold, percent_dense,            \
                         min_opacity, prune_big_world, max_world_size_frac, max_screen_size, split_children,       \
                         extent, normals, n_normals, out_params, out_m, out_v, report);                            \
  }                                                                                                                \
  ORA_API void ora_reset_opacity_##S(R* params, R* m, R* v, int64_t n, R max_alpha) {                              \
    std::vector<Gaussian<R>> model((Gaussian<R>*)params, (Gaussian<R>*)params + n);                                \
    Adam<R> adam(0);                                                                                               \
    adam.m.assign((Gaussian<R>*)m, (Gaussian<R>*)m + n);                                                           \
    adam.v.assign((Gaussian<R>*)v, (Gaussian<R>*)v + n);                                                           \
    reset_opacity(model, adam, max_alpha);                                                                         \
    std::memcpy(params, model.data(), n * sizeof(Gaussian<R>));                                                   \
    std::memcpy(m, adam.m.data(), n * sizeof(Gaussian<R>));                                                        \
    std::memcpy(v, adam.v.data(), n * sizeof(Gaussian<R>));                                                        \
  }                                                                                                                \
  ORA_API void ora_from_points_##S(const float* pts, const uint8_t* rgb, int64_t n, R* out59) {                    \
    std::vector<Gaussian<R>> model;                                                                                \
    from_points<R>(pts, rgb, n, model);                                                                            \
    std::memcpy(out59, model.data(), n * sizeof(Gaussian<R>));                                                     \
  }                                                                                                                \
  ORA_API void ora_look_at_##S(uint32_t w, uint32_t h, R fx, R fy, const R* eye, const R* target, const R* up,     \
                               R* cam18) {                                                                         \
    Camera<R> c = Camera<R>::look_at(w, h, fx, fy, V3<R>(eye[0], eye[1], eye[2]),                                  \
                                     V3<R>(target[0], target[1], target[2]), V3<R>(up[0], up[1], up[2]));          \
    cam_to(c, cam18);                                                                                              \
  }                                                                                                                \
  ORA_API R ora_scene_extent_##S(const R* cams18, int64_t n) {                                                     \
    std::vector<Camera<R>> cams(n);                                                                                \
    for (int64_t i = 0; i < n; i++) cams[i] = cam_from(cams18 + 18 * i);                                           \
    return scene_extent(cams);                                                                                     \
  }                                                                                                                \
  ORA_API void ora_sh_basis_##S(int deg, const R* dir, R* out16) {                                                 \
    sh_basis<R>(deg, V3<R>(dir[0], dir[1], dir[2]), out16);                                                        \
  }                                                                                                                \
  ORA_API void ora_sh_basis_grad_##S(int deg, const R* dir, R* out48) {                                            \
    V3<R> g[MAX_COEFFS];                                                                                           \
    sh_basis_grad<R>(deg, V3<R>(dir[0], dir[1], dir[2]), g);                                                       \
    for (int k = 0; k < MAX_COEFFS; k++) {                                                                         \
      out48[3 * k] = g[k].x;                                                                                       \
      out48[3 * k + 1] = g[k].y;                                                                                   \
      out48[3 * k + 2] = g[k].z;                                                                                   \
    }                                                                                                              \
  }                                                                                                                \
  ORA_API void ora_quat_to_mat_##S(const R* q, R* out9) {                                                          \
    M3<R> m = Quat<R>{q[0], q[1], q[2], q[3]}.normalized().to_mat();                                               \
    for (int i = 0; i < 9; i++) out9[i] = m.m[i / 3][i % 3];                                                       \
  }                                                                                                                \
  ORA_API R ora_sigmoid_##S(R x) { return sigmoid(x); }                                                            \
  ORA_API R ora_inverse_sigmoid_##S(R x) { return inverse_sigmoid(x); }

ORA_BOTH(float, f)
ORA_BOTH(double, d)

ORA_API void ora_binning_free(void* b) { delete (Binning*)b; }
ORA_API int64_t ora_binning_num_entries(const void* b) { return (int64_t)((const Binning*)b)->sorted.size(); }
// keys/entries: sorted (key, entry) pairs; entry_gaussian indexed by entry;
// entry_offset (n+1); tile_range (2 per tile).
ORA_API void ora_binning_get(const void* bp, uint64_t* keys, uint32_t* entries, uint32_t* entry_gaussian,
                             uint32_t* entry_offset, uint32_t* tile_range) {
  const Binning* b = (const Binning*)bp;
  for (size_t i = 0; i < b->sorted.size(); i++) {
    if (keys) keys[i] = b->sorted[i].first;
    if (entries) entries[i] = b->sorted[i].second;
  }
  if (entry_gaussian) std::memcpy(entry_gaussian, b->entry_gaussian.data(), b->entry_gaussian.size() * 4);
  if (entry_offset) std::memcpy(entry_offset, b->entry_offset.data(), b->entry_offset.size() * 4);
  if (tile_range)
    for (size_t t = 0; t < b->tile_range.size(); t++) {
      tile_range[2 * t] = b->tile_range[t].first;
      tile_range[2 * t + 1] = b->tile_range[t].second;
    }
}

ORA_API void ora_mean_nn_dist2(const float* pts, int64_t n, double* out) { mean_nn_dist2(pts, n, out); }

ORA_API uint64_t ora_splitmix_next(uint64_t* state) {
  SplitMix64 r(*state);
  uint64_t v = r.next();
  *state = r.s;
  return v;
}
ORA_API double ora_splitmix_normal(uint64_t* state) {
  SplitMix64 r(*state);
  double v = r.normal();
  *state = r.s;
  return v;
}
// `count` successive normals of the generator (the same values ora_splitmix_normal returns
// one by one).
ORA_API void ora_splitmix_normals(uint64_t* state, int64_t count, double* out) {
  SplitMix64 r(*state);
  for (int64_t i = 0; i < count; i++) out[i] = r.normal();
  *state = r.s;
}

// ---------------------------------------------------------------------------------------
// Trainer (float only). The config is passed field by field through an array of doubles
// in the order of ora_train_config_fields() so that the Python side stays declarative.
// ---------------------------------------------------------------------------------------
static const char* kTrainFields =
    "iterations,position_lr_init,position_lr_final,position_lr_max_steps,feature_lr,opacity_lr,scaling_lr,"
    "rotation_lr,lambda_dssim,densify,densify_from_iter,densify_until_iter,densification_interval,"
    "opacity_reset_interval,densify_grad_threshold,percent_dense,min_opacity,max_screen_size,absgrad,antialias,"
    "white_background,sh_degree,sh_degree_interval,near,seed";

ORA_API const char* ora_train_config_fields(void) { return kTrainFields; }

ORA_API void* ora_trainer_new(const float* init59, int64_t n, float extent, const double* cfgv) {
  auto* t = new Trainer<float>();
  t->model.assign((const Gaussian<float>*)init59, (const Gaussian<float>*)init59 + n);
  t->extent = extent;
  TrainConfig<float>& c = t->cfg;
  int i = 0;
  c.iterations = (uint32_t)cfgv[i++];
  c.position_lr_init = (float)cfgv[i++];
  c.position_lr_final = (float)cfgv[i++];
  c.position_lr_max_steps = (uint32_t)cfgv[i++];
  c.feature_lr = (float)cfgv[i++];
  c.opacity_lr = (float)cfgv[i++];
  c.scaling_lr = (float)cfgv[i++];
  c.rotation_lr = (float)cfgv[i++];
  c.lambda_dssim = (float)cfgv[i++];
  c.densify = cfgv[i++] != 0;
  c.densify_from_iter = (uint32_t)cfgv[i++];
  c.densify_until_iter = (uint32_t)cfgv[i++];
  c.densification_interval = (uint32_t)cfgv[i++];
  c.opacity_reset_interval = (uint32_t)cfgv[i++];
  c.densify_grad_threshold = (float)cfgv[i++];
  c.percent_dense = (float)cfgv[i++];
  c.min_opacity = (float)cfgv[i++];
  c.max_screen_size = (int64_t)cfgv[i++];
  c.absgrad = cfgv[i++] != 0;
  c.antialias = cfgv[i++] != 0;
  c.white_background = cfgv[i++] != 0;
  c.sh_degree = (int)cfgv[i++];
  c.sh_degree_interval = (uint32_t)cfgv[i++];
  c.near_ = (float)cfgv[i++];
  c.seed = (uint64_t)cfgv[i++];
  return t;
}
ORA_API void ora_trainer_add_view(void* tp, const float* cam18, const uint8_t* rgb) {
  auto* t = (Trainer<float>*)tp;
  View<float> v;
  v.camera = cam_from(cam18);
  v.rgb.assign(rgb, rgb + (size_t)v.camera.width * v.camera.height * 3);
  t->views.push_back(std::move(v));
}
ORA_API void ora_trainer_start(void* tp) { ((Trainer<float>*)tp)->start(); }
// info: loss, psnr, view, num_gaussians, cloned, split, pruned, densified, reset, entries
ORA_API void ora_trainer_step(void* tp, double* info10) {
  StepInfo s = ((Trainer<float>*)tp)->step();
  double v[10] = {s.loss, s.psnr, (double)s.view, (double)s.num_gaussians, (double)s.cloned, (double)s.split,
                  (double)s.pruned, (double)s.densified, (double)s.reset, (double)s.entries};
  std::memcpy(info10, v, sizeof(v));
}
ORA_API int64_t ora_trainer_count(const void* tp) { return (int64_t)((const Trainer<float>*)tp)->model.size(); }
ORA_API int ora_trainer_sh_degree(const void* tp) { return ((const Trainer<float>*)tp)->sh_degree; }
ORA_API void ora_trainer_get_model(const void* tp, float* out59) {
  const auto* t = (const Trainer<float>*)tp;
  std::memcpy(out59, t->model.data(), t->model.size() * sizeof(Gaussian<float>));
}
ORA_API void ora_trainer_render(const void* tp, const float* cam18, float* image) {
  const auto* t = (const Trainer<float>*)tp;
  float bg[3];
  t->cfg.background(bg);
  std::vector<float> img = t->render(cam_from(cam18), t->cfg.proj_opts(t->sh_degree), bg);
  std::memcpy(image, img.data(), img.size() * sizeof(float));
}
ORA_API void ora_trainer_free(void* tp) { delete (Trainer<float>*)tp; }
