// Host-side launchers of the device stages; each returns a Status and launches on the
// context stream.
#pragma once
#include <functional>
#include "common.cuh"
#include "adam.cuh"

namespace splat {

// Per-iteration arguments read from device memory, so that a captured training step
// (a CUDA graph) replays with a new view, camera and Adam step. Kernels given a non-NULL
// StepParams* use its fields in place of the corresponding by-value arguments.
struct StepParams {
  splat_camera cam;
  AdamArgs adam;
  const void* target;  // the view's 8-bit pixels
};

// A batch of views rendered and back-propagated together, one launch per stage. Records
// are view-major (record r = v * n + i for Gaussian i), tiles are numbered across the
// batch (view v owns global tiles [tile_start[v], tile_start[v + 1])), images are
// concatenated (view v's pixels start at pix_start[v]) and SSIM blocks likewise. Kernels
// launched for a capacity exit in blocks past the batch's totals, so one captured graph
// serves any mix of view sizes.
constexpr int kMaxViews = 8;
struct BatchTable {
  splat_camera cam[kMaxViews];
  const void* target[kMaxViews];
  uint32_t tiles_x[kMaxViews];
  uint32_t tile_start[kMaxViews + 1];
  uint32_t loss_blocks_x[kMaxViews];
  uint32_t loss_start[kMaxViews + 1];
  uint64_t pix_start[kMaxViews + 1];
  AdamArgs adam;
  int32_t views;
  float inv_views;
};

__device__ __forceinline__ int batch_view_of(const uint32_t* start, int views, uint32_t b) {
  int v = 0;
  while (v + 1 < views && b >= start[v + 1]) v++;
  return v;
}

Status launch_params_from_aos(Ctx* c, const float* aos, int64_t n, float* planes, int64_t cap);
Status launch_params_to_aos(Ctx* c, const float* planes, int64_t n, int64_t cap, float* aos);

Status launch_project_fwd(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                          const splat_proj_opts& opts, float* proj, uint32_t* num_tiles, uint32_t* depth_range,
                          const StepParams* sp = nullptr, const void* bf16 = nullptr,
                          const BatchTable* bt = nullptr);
Status launch_proj_from_reference(Ctx* c, const float* p15, int64_t n, uint32_t width, uint32_t height, float* proj,
                                  uint32_t* num_tiles, uint32_t* depth_range);
Status launch_proj_to_reference(Ctx* c, const float* proj, int64_t n, float* p15);
Status launch_project_bwd(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                          const splat_proj_opts& opts, const float* proj, const float* pgrad, float* out,
                          void* stats, int absgrad);

// project_backward_all fused with Adam::step: parameters updated in place.
// A nonzero *skip (may be NULL) makes the kernel return without touching anything (a view
// whose binning overflowed).
Status launch_project_bwd_adam(Ctx* c, float* planes, float* m, float* v, int64_t n, int64_t cap,
                               const splat_camera& cam, const splat_proj_opts& opts, const float* proj,
                               const float* pgrad, void* stats, int absgrad, uint64_t step, const splat_lr& lr,
                               const uint32_t* skip = nullptr, const StepParams* sp = nullptr,
                               void* bf16 = nullptr, bool stats_maxg = false);
// With stats_maxg the statistics are the trainer's five arrays of cap entries: accum,
// denom, max radius, max gradient and contribution (each view adds the entry's blending
// weight sum(alpha T) from plane 2's w of the screen-space gradient).

// A batch's projection backward (records view-major, screen-space gradient planes with
// stride pcap) summed over the views that see each Gaussian, then one Adam step with the
// batch's AdamArgs (bt->adam); densification statistics accumulate per view.
Status launch_project_bwd_batch_adam(Ctx* c, float* planes, float* m, float* v, int64_t n, int64_t cap,
                                     const splat_proj_opts& opts, const float* proj, const float* pgrad, int64_t pcap,
                                     void* stats, int absgrad, const uint32_t* skip, const BatchTable* bt,
                                     void* bf16, bool stats_maxg = false);

// The BF16 render copy of parameter planes 1..14 (quaternion, log-scales, SH; 4 x bf16 per
// Gaussian and plane, plane q at (q - 1) * cap, rounded to nearest even). With a copy,
// launch_project_fwd reads those planes from it, and launch_project_bwd_adam computes the
// gradient at the copy's values, updates the f32 master and rewrites the copy.
Status launch_planes_to_bf16(Ctx* c, const float* planes, int64_t n, int64_t cap, void* bf16);

Status launch_scan_u32(Ctx* c, const uint32_t* in, int64_t n, uint32_t* out, int write_total, uint64_t* total_dev);

// Binning without a host read-back: the entry count (*E_dev, from the entry-offset scan)
// and the depth range stay on the device; `scratch` holds dev_sort_scratch_bytes(E_cap)
// bytes. Counts above E_cap set *overflow and leave the view's results invalid.
size_t dev_sort_scratch_bytes(int64_t E_cap);
Status launch_bin_sort_dev(Ctx* c, const float* proj, const uint32_t* entry_offset, int64_t n, const uint64_t* E_dev,
                           int64_t E_cap, const uint32_t* depth_range_dev, uint32_t width, uint32_t height,
                           void* scratch, uint32_t* gauss_out, uint32_t* ranges, uint32_t* overflow,
                           const BatchTable* bt = nullptr, int64_t n_view = 1, uint32_t tiles_cap = 0);

// The learned-densification network (mlp.cu): 16 -> 64 -> 64 -> 3, FP32 parameter vector.
int mlp_num_params();
Status launch_mlp_forward(Ctx* c, const float* x, int64_t n, const float* theta, float* prob);
// The same on tcgen05 (TMEM accumulators). `err` is a word the device can store to (the
// context's mapped host page): set to 1 if a wait for the tensor cores timed out.
Status launch_mlp_forward_tc(Ctx* c, const float* x, int64_t n, const float* theta, float* prob, uint32_t* err);
// Word of the context's mapped host page (c->host_small) that the tcgen05 kernels report
// timeouts in.
constexpr int kTcErrWord = 1000;
// Word of the context's mapped host memory where a radix sort records a look-back wait that
// ran out (bit 2); read and cleared by take_sort_error at the context's next synchronising
// entry point.
constexpr int kSortErrWord = 1001;
constexpr size_t kAsyncErrorWordOffset = (size_t)kSortErrWord * 4;
Status take_sort_error(Ctx* c);
// Runs the tcgen05 forward with the error word cleared, synchronises and turns a reported
// timeout into an error status.
Status mlp_forward_tc_checked(Ctx* c, const float* x, int64_t n, const float* theta, float* prob);
// The gradient of launch_mlp_grad on tcgen05 (tensor-memory accumulators; one CTA per SM),
// added to grad. `err` as for launch_mlp_forward_tc.
Status launch_mlp_grad_tc(Ctx* c, const float* x, const int32_t* y, const float* w, int64_t n, float scale,
                          const float* theta, float* grad, uint32_t* err);
// The error word of the tcgen05 network kernels: cleared on the host before a run of
// launches, checked (after a synchronisation) once they are done.
Status mlp_tc_error_clear(Ctx* c);
uint32_t* mlp_tc_error_word(Ctx* c);
Status mlp_tc_error_check(Ctx* c);
// Runs one bounded mbarrier wait of `limit` tries that times out unless `arrive`, through
// the error word; SPLAT_ERR_TIMEOUT when it ran out. Synchronises.
Status diag_mbar_wait(Ctx* c, uint32_t limit, int arrive);
Status launch_mlp_grad(Ctx* c, const float* x, const int32_t* y, const float* w, int64_t n, float scale,
                       const float* theta, float* grad);
Status launch_mlp_adam(Ctx* c, float* theta, const float* grad, float* m, float* v, uint64_t step, float lr);

// Learned densification (densify_learn.cu): features of every Gaussian (n x 16) from its
// parameters, densification statistics (accum, denom, max radius, max gradient,
// contribution) and birth iteration; hindsight labels of the previous densification's
// records from the origin of every current Gaussian (a descendant is useful when its
// opacity is at least tau and, with tau_c > 0, its contribution over the window at least
// tau_c; a kept record whose descendants contributed less than tau_c in all is
// relabelled prune); a strided, class-weighted training subset.
size_t densify_features_scratch_bytes(int64_t n);
Status launch_densify_features(Ctx* c, const float* params, int64_t n, int64_t cap, const float* accum,
                               const uint32_t* denom, const uint32_t* maxr, const float* maxg, const float* contrib,
                               const uint32_t* birth, uint32_t now, float size_limit, void* scratch, float* x_out);
Status launch_hindsight_labels(Ctx* c, const float* params, int64_t n, const uint32_t* origin, int64_t n_prev,
                               const uint32_t* action, float tau, const float* contrib, float tau_c,
                               uint32_t* alive, uint32_t* useful, float* csum, int32_t* y,
                               unsigned long long* counts);
Status launch_label_accuracy(Ctx* c, const float* prob, const uint32_t* action, const int32_t* y, int64_t n_prev,
                             unsigned long long* acc);
Status launch_gather_training(Ctx* c, const float* x, const int32_t* y, int64_t n_prev, int64_t first, int64_t stride,
                              const float w[3], float* xo, int32_t* yo, float* wo, int64_t m);

// Fills `words` 32-bit words at `dst` with `value` by a kernel on the context stream (in
// place of cudaMemsetAsync, so the compute stream holds kernels only).
Status launch_fill_u32(Ctx* c, void* dst, size_t words, uint32_t value);

// Copies na words from a and then nb words from b (device memory, na + nb <= 32) into the
// context's mapped host buffer (c->host_small) with a one-warp kernel; the host reads them
// after synchronising the stream.
Status launch_publish_u32(Ctx* c, const uint32_t* a, int na, const uint32_t* b, int nb);
// The same into another mapped host buffer (its device alias `out_dev`).
Status launch_publish_u32_to(Ctx* c, const uint32_t* a, int na, const uint32_t* b, int nb, void* out_dev);
Status launch_scan_u32_into(Ctx* c, const uint32_t* in, int64_t n, uint32_t* out, int write_total,
                            uint64_t* partial, uint64_t* total);
constexpr int kScanValuesPerBlock = 4096;
Status launch_bin_sort(Ctx* c, const float* proj, const uint32_t* entry_offset, int64_t n, int64_t E,
                       const uint32_t* depth_range_dev, uint32_t depth_min, uint32_t depth_max, uint32_t width,
                       uint32_t height, uint32_t* gauss_out, uint64_t* keys_out, uint32_t* ranges);

// The supported compositing configurations (tile shapes x chunk depths x backward pixels
// per thread).
constexpr int kRasterCandidates = 24;
extern const RasterConfig kRasterCandidateList[kRasterCandidates];
// Times pass() under every candidate configuration: pass(true) once, untimed (it may
// synchronise, size buffers and redo work), then pass(false) `reps` times between two
// events on c->stream. Leaves c->raster at the fastest (at its old value on failure) and
// writes each candidate's mean milliseconds per pass to ms[].
Status tune_raster(Ctx* c, const std::function<Status(bool)>& pass, int reps, float ms[kRasterCandidates]);
// tune_raster over one view's projection, binning and forward + backward compositing
// (dimage: dL/dimage of the view); allocates and frees its own buffers.
Status tune_render(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                   const splat_proj_opts& opts, const float bg[3], const float* dimage, int reps,
                   float ms[kRasterCandidates]);

Status launch_raster_fwd(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges, uint32_t width,
                         uint32_t height, const float bg[3], float* image, float* final_t, uint32_t* n_contrib,
                         uint64_t* pairs, const BatchTable* bt = nullptr, uint32_t tiles_cap = 0);
Status launch_raster_bwd(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges, uint32_t width,
                         uint32_t height, const float bg[3], const float* final_t, const uint32_t* n_contrib,
                         const float* dimage, float* pgrad, int64_t cap, uint64_t* pairs,
                         const BatchTable* bt = nullptr, uint32_t tiles_cap = 0);
// The deterministic backward (16x16 tiles only): per-entry slot sums in the reference's
// pixel order into eslot (12 floats per entry, e_cap entries, indexed by emission order),
// then per-Gaussian sums in entry order written into pgrad (3 planes, stride cap).
Status launch_raster_bwd_det(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges,
                             const uint32_t* entry_offset, int64_t n, int64_t e_cap, uint32_t width, uint32_t height,
                             const float bg[3], const float* final_t, const uint32_t* n_contrib, const float* dimage,
                             float* eslot, float* pgrad, int64_t cap);

Status launch_diag_fast_exp(Ctx* c, float magnitude_lo, float magnitude_hi, int negative, float* out_host);
Status launch_diag_pair_exact(Ctx* c, uint32_t n, uint32_t* out_host);
// Throughput of one unit (0: FP32 FMA, in FLOP/s; 1: MUFU ex2, in operations/s), peaks.cu.
Status launch_diag_peak(Ctx* c, int unit, double* ops_per_s, float* ms_out);

Status launch_loss(Ctx* c, const float* pred, const void* target, int target_u8, uint32_t width, uint32_t height,
                   float lambda, float* grad, float* out3, const StepParams* sp = nullptr,
                   const BatchTable* bt = nullptr, uint32_t blocks_cap = 0, uint64_t pix_cap = 0);

// Copies `words` 32-bit words (a StepParams) from mapped host memory to device memory with
// one warp.
Status launch_load_words(Ctx* c, const void* src_mapped_dev, void* dst, int words);

Status launch_adam(Ctx* c, float* params, const float* grads, float* m, float* v, int64_t n, int64_t cap,
                   uint64_t step, const splat_lr& lr);
Status launch_reset_opacity(Ctx* c, float* params, float* m, float* v, int64_t n, float limit);

struct DensifyArgs {
  float grad_threshold, size_limit, min_opacity, big_world_limit, shrink;
  int prune_big_world;
  int64_t max_screen_size;
  int children;
  int grow;  // 0: clone and split nothing (prune only)
  // Learned densification (none of it in the reference; all optional):
  const float* policy;    // per Gaussian {keep, clone/split, prune} probabilities (n x 3):
                          // a densification is vetoed when keep is the likelier of the two
                          // and at least 0.6; a prune probability >= prune_conf prunes
  float prune_conf;
  uint32_t* action;       // out: the rule's action per Gaussian (0 keep, 1 clone/split, 2 prune)
  uint32_t* origin_out;   // out: for every new Gaussian, the index it came from
  const uint32_t* birth_in;
  uint32_t* birth_out;    // survivors keep their birth iteration, new Gaussians get birth_now
  uint32_t birth_now;
};
struct DensifyParams {
  splat_densify_config cfg;
  float extent;
  float shrink;  // ln(0.8 * children), densify.rs:169
  bool grow = true;
  const float* policy = nullptr;
  float prune_conf = 0.9f;
  uint32_t* action = nullptr;
  uint32_t* origin_out = nullptr;
  const uint32_t* birth_in = nullptr;
  uint32_t* birth_out = nullptr;
  uint32_t birth_now = 0;
};
// Decisions of one densification step; the arrays live in the context arena until the
// next entry point.
struct DensifyPlan {
  uint64_t kept_orig = 0, cloned = 0, kept_clones = 0, split = 0, kept_children = 0, pruned = 0;
  uint32_t *flags = nullptr, *off_orig = nullptr, *off_clone = nullptr, *off_split = nullptr, *off_child = nullptr;
  DensifyArgs args;
  uint64_t new_count() const { return kept_orig + kept_clones + kept_children; }
};
// Marks, scans and reads the counts back (synchronises).
Status densify_plan(Ctx* c, const float* params, int64_t n, int64_t cap, const float* accum, const uint32_t* denom,
                    const uint32_t* maxr, const DensifyParams& dp, DensifyPlan* plan);
// Writes the new parameters and Adam state (out of place). `normals_dev` holds
// 3 * children samples per split parent, in the reference's draw order.
Status densify_apply(Ctx* c, const float* params, const float* m, const float* v, int64_t n, int64_t cap,
                     const DensifyPlan& plan, const double* normals_dev, float* po, float* mo, float* vo,
                     int64_t cap_out);

}  // namespace splat
