/*
 * splat_gpu.h: the C ABI of the B200 (sm_100a) render-and-train path for 3D Gaussian
 * splatting.
 *
 * The reference implementation (harryprayiv/splatrs) is a pure-Rust CPU crate with no FFI
 * today (`#![forbid(unsafe_code)]`, src/lib.rs:13). These entry points are what its
 * functions would bind to, one per reference function, named in each comment. Plain C
 * types only: pointers, sizes, POD structs. No C++ or torch types cross this boundary.
 *
 * Conventions
 *  - Every entry point returns an int status (SPLAT_OK on success) and never aborts. The
 *    message of the last failure on a context is available from splat_last_error().
 *  - Pointers whose name ends in `_dev` are device pointers (cudaMalloc'd or any device
 *    allocation on the context's device); `_host` pointers are host memory (pinned or
 *    pageable). The stage functions are asynchronous on the context's stream unless their
 *    comment says they synchronise (they do only to read a count back, as the reference's
 *    `Vec` sizes require).
 *  - A context is used from one host thread at a time. Separate contexts may run
 *    concurrently on separate streams. Renderers and trainers borrow their context and
 *    must be destroyed before it.
 *
 * Device layouts
 *  - Parameter planes (`planes_dev`): SPLAT_PLANES planes of float4, plane p at
 *    planes_dev + 4*p*cap floats, element i of plane p holds:
 *        plane 0: mean.x mean.y mean.z opacity(logit)
 *        plane 1: quat w x y z (unnormalised)
 *        plane 2: log_scale x y z, 0
 *        plane 3+q (q = 0..11): sh coefficients j = 4q..4q+3 where j = 3*k + channel
 *    Gradients and Adam moments use the same layout. Each warp-wide load of a plane is one
 *    contiguous 512-byte transaction.
 *  - Reference Gaussian record (`aos59`): 59 floats = mean[3] log_scale[3] quat[4]
 *    opacity sh[16][3] (reference src/model.rs:16-28), the layout the .ply codec and a
 *    Rust `&[Gaussian]` hand over.
 *  - Projection record (`proj_dev`): 16 floats per Gaussian (see SPLAT_PROJ_FLOATS),
 *    produced by splat_project_fwd or splat_proj_from_reference and consumed by the
 *    binning, compositing and projection-backward stages.
 *  - Reference projection record (`proj15`): 15 floats = mean2d[2] conic[3] depth radius
 *    opacity color[3] tile_min[2] tile_max[2] with the integers stored as exact floats
 *    (reference src/project.rs:47-64).
 *  - Screen-space gradients (`pgrad_dev`): 3 planes of float4 with stride cap:
 *        (d mean2d.x, d mean2d.y, d conic.A, d conic.B), (d conic.C, d opacity, d r, d g),
 *        (d b, |d mean2d.x| sum, |d mean2d.y| sum, 0)
 *    i.e. ProjGrad plus the AbsGS accumulators (reference src/project.rs:84-93,
 *    src/rasterize.rs:339-341).
 *  - Images are row-major H x W x 3 float (reference src/rasterize.rs:43-50).
 */
#ifndef SPLAT_GPU_H
#define SPLAT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPLAT_API __attribute__((visibility("default")))

/* Status codes. */
#define SPLAT_OK 0
#define SPLAT_ERR_INVALID 1   /* bad argument; the reference panics or returns Error::Invalid */
#define SPLAT_ERR_CAPACITY 2  /* a fixed-capacity buffer is too small; retry with a larger one */
#define SPLAT_ERR_CUDA 3      /* a CUDA runtime call failed */
#define SPLAT_ERR_TIMEOUT 4   /* a bounded device wait ran out */

#define SPLAT_PLANES 15
#define SPLAT_PROJ_FLOATS 16
#define SPLAT_TILE 16

/* Pinhole camera with COLMAP conventions (reference src/camera.rs:13-32). */
typedef struct splat_camera {
  uint32_t width, height;
  float fx, fy, cx, cy;
  float rot[9];   /* world-to-camera rotation, row major */
  float trans[3]; /* world-to-camera translation */
} splat_camera;

/* Projection options (reference src/project.rs:22-43). */
typedef struct splat_proj_opts {
  float near_plane; /* 0.2 */
  float eps2d;      /* 0.3 */
  int32_t antialias;
  int32_t sh_degree;
  /* Not in the reference (0 reproduces it): when the f32 determinant of the projected 2x2
   * covariance is ill-conditioned, rebuild that covariance, its determinant and inverse in
   * f64. The test is det < 1e-4 * trace^2 on the f32 values, so that every covariance with
   * det < 1e-6 * trace^2 is caught although the f32 determinant tested is itself off by up
   * to ~10% near that ratio. */
  int32_t fp64_conic;
} splat_proj_opts;

/* Per-group learning rates (reference src/adam.rs:11-24). */
typedef struct splat_lr {
  float mean, log_scale, quat, opacity, sh_dc, sh_rest;
} splat_lr;

/* Densification thresholds (reference src/densify.rs:69-103). */
typedef struct splat_densify_config {
  float grad_threshold;      /* 0.0002 */
  float percent_dense;       /* 0.01 */
  float min_opacity;         /* 0.005 */
  int32_t prune_big_world;   /* 0 */
  float max_world_size_frac; /* 0.1 */
  int64_t max_screen_size;   /* < 0 means None */
  int32_t split_children;    /* 2 */
} splat_densify_config;

/* Training hyperparameters (reference src/train.rs:20-109). */
typedef struct splat_train_config {
  uint32_t iterations;
  float position_lr_init, position_lr_final;
  uint32_t position_lr_max_steps;
  float feature_lr, opacity_lr, scaling_lr, rotation_lr, lambda_dssim;
  int32_t densify;
  uint32_t densify_from_iter, densify_until_iter, densification_interval, opacity_reset_interval;
  float densify_grad_threshold, percent_dense, min_opacity;
  int64_t max_screen_size; /* < 0 means None */
  int32_t absgrad, antialias, white_background, sh_degree;
  uint32_t sh_degree_interval;
  float near_plane;
  uint64_t seed;
  /* Not in the reference: 0 = no limit. When a densification would leave more Gaussians
   * than this, that densification clones and splits nothing and only prunes. */
  uint64_t max_gaussians;
  /* Not in the reference: tile entries the binning buffers hold at first (0 = automatic).
   * An iteration whose view needs more is redone with larger buffers. */
  uint64_t entry_capacity;
  /* Not in the reference: render from a BF16 copy of quaternion, log-scales and SH (the
   * f32 parameters stay the optimiser's master copy), and re-solve ill-conditioned 2x2
   * conics in f64 (splat_proj_opts.fp64_conic). */
  int32_t bf16_storage;
  int32_t fp64_conic;
  /* Not in the reference: views per iteration (0 or 1: one, as the reference; at most 8).
   * A batch renders and back-propagates its views (of any sizes) in one launch per stage
   * and takes one Adam step on the mean of their gradients. */
  uint32_t batch_views;
  /* Not in the reference: learned densification. 0 off; 1 learn: densify by the rule and
   * train the trainer's network online on hindsight-labelled outcomes of its edits; 2
   * apply: the network's {keep, clone/split, prune} probabilities veto a densification
   * when keep is the likelier of the two and at least 0.6, and prune with probability
   * >= 0.9, the rule deciding everything else (with an all-zero network this is exactly
   * the rule). */
  int32_t learned_densify;
  /* Not in the reference: 1 times the iteration's render stages (no optimiser step) under
   * every compositing configuration (splat_raster_candidates) before the first iteration
   * and again whenever the Gaussian count has doubled or halved since, and
   * keeps the fastest on the context; 0 uses the context's configuration as it is. */
  int32_t autotune;
  /* Not in the reference; learned densification only. learn_contribution > 0: hindsight
   * labels also weigh contribution, each Gaussian's blending weight sum(alpha T) over the
   * pixels of every view between two densifications (pixel units): a kept Gaussian whose
   * descendants contributed less is labelled prune, and a clone/split descendant counts as
   * useful only from that contribution on. 0: labels from opacity alone.
   * learn_prune_confidence > 0: the prune probability at which applying prunes (default
   * 0.9). */
  float learn_contribution;
  float learn_prune_confidence;
  /* Not in the reference's config, but its arithmetic: 1 takes every iteration's compositing
   * backward through splat_rasterize_bwd_deterministic's reduction (the reference's per-entry
   * slots and ordered per-Gaussian sums), so the whole run equals the reference's CPU
   * trainer (with correctly rounded exp/log) bit for bit; 0 (default) sums with float
   * atomics, whose order is unspecified. Needs one view per iteration, 16x16 tiles, no
   * autotuning, no BF16 copy and no f64 conics. */
  int32_t deterministic;
  /* Not in the reference: coarse-to-fine training. Iterations 1..coarse_until train on
   * every view box-filtered by coarse_factor (2 or 4; the camera's size, focal lengths and
   * principal point divided by it, rows and columns past the last whole block dropped), the
   * rest on the views as given. 0 (default) is off. Evaluation always uses the views as
   * given. Not with `deterministic`. */
  uint32_t coarse_until;
  uint32_t coarse_factor;
} splat_train_config;

typedef struct splat_ctx splat_ctx;

/* ----------------------------------------------------------------------------------------
 * Context: device, stream, scratch arena, error message. No counterpart in the reference,
 * whose functions run on the caller's thread and the global rayon pool and panic on
 * violated invariants (e.g. src/rasterize.rs:65-74, :466-469); here every entry point
 * returns a status and leaves the message in the context.
 * -------------------------------------------------------------------------------------- */
/* `stream` is a cudaStream_t (NULL for the legacy default stream). */
SPLAT_API int splat_ctx_create(int device, void* stream, splat_ctx** out);
SPLAT_API int splat_ctx_destroy(splat_ctx* ctx);
SPLAT_API int splat_ctx_set_stream(splat_ctx* ctx, void* stream);
SPLAT_API int splat_ctx_synchronize(splat_ctx* ctx);
SPLAT_API const char* splat_last_error(const splat_ctx* ctx);
SPLAT_API const char* splat_status_string(int status);
SPLAT_API int splat_version(void);
/* sizeof of the public structs, for bindings to check their layouts against: splat_camera,
 * splat_proj_opts, splat_lr, splat_densify_config, splat_train_config,
 * splat_densify_report, splat_step_info (7 values written to out; returns 7). */
SPLAT_API int32_t splat_struct_sizes(uint64_t* out);
/* Kernels launched through this context since creation (all stage entry points count). */
SPLAT_API uint64_t splat_ctx_launch_count(const splat_ctx* ctx);
/* The context's scratch arena: out2[0] = bytes it holds on the device, out2[1] = a counter
 * that changes whenever it allocates or frees (no counterpart in the reference; lets a
 * caller check that an entry point allocated nothing). */
SPLAT_API int splat_ctx_scratch_info(const splat_ctx* ctx, uint64_t* out2);

/* ----------------------------------------------------------------------------------------
 * Parameter layout conversion: the reference's Gaussian records (59 floats in field order,
 * reference src/model.rs:16-28; the caller's &[Gaussian]) to and from the device
 * parameter planes.
 * -------------------------------------------------------------------------------------- */
SPLAT_API int splat_params_from_aos(splat_ctx* ctx, const float* aos59_dev, int64_t n, float* planes_dev,
                                    int64_t cap);
SPLAT_API int splat_params_to_aos(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap,
                                  float* aos59_dev);

/* ----------------------------------------------------------------------------------------
 * Projection: project_all (reference src/project.rs:320-330, project_one :277-317,
 * core :137-269). Writes n projection records and n per-Gaussian tile counts
 * (Proj::num_tiles, :73-79). `depth_range_dev` (2 x uint32) receives the min and max
 * float bits of the visible depths; it is reset by this call.
 * -------------------------------------------------------------------------------------- */
SPLAT_API int splat_project_fwd(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap,
                                const splat_camera* cam, const splat_proj_opts* opts, float* proj_dev,
                                uint32_t* num_tiles_dev, uint32_t* depth_range_dev);

/* BF16 storage (not in the reference). splat_params_to_bf16 writes the BF16 render copy of
 * parameter planes 1..14 (quaternion, log-scales, SH: 4 x bf16 per Gaussian and plane,
 * plane q at offset (q - 1) * cap, 8 * 14 * cap bytes, rounded to nearest even); means and
 * opacity stay in f32 plane 0. splat_project_fwd_bf16 is splat_project_fwd reading those
 * planes from the copy (112 bytes per Gaussian instead of 224): its records equal
 * splat_project_fwd's on planes rounded to bf16. */
SPLAT_API int splat_params_to_bf16(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap, void* bf16_dev);
SPLAT_API int splat_project_fwd_bf16(splat_ctx* ctx, const float* planes_dev, const void* bf16_dev, int64_t n,
                                     int64_t cap, const splat_camera* cam, const splat_proj_opts* opts,
                                     float* proj_dev, uint32_t* num_tiles_dev, uint32_t* depth_range_dev);

/* Build projection records from reference-layout Proj records (proj15, device), e.g. to
 * bin and composite projections made elsewhere. Also writes tile counts and depth range. */
SPLAT_API int splat_proj_from_reference(splat_ctx* ctx, const float* proj15_dev, int64_t n, uint32_t width,
                                        uint32_t height, float* proj_dev, uint32_t* num_tiles_dev,
                                        uint32_t* depth_range_dev);

/* Reference-layout Proj records (proj15, device) from projection records. */
SPLAT_API int splat_proj_to_reference(splat_ctx* ctx, const float* proj_dev, int64_t n, float* proj15_dev);

/* ----------------------------------------------------------------------------------------
 * Binning: bin (reference src/rasterize.rs:60-128), in two calls.
 * splat_bin_count: exclusive scan of the tile counts into entry_offset_dev (n + 1 values,
 * Binning::entry_offset) and the number of entries. Synchronises to return the count and
 * the depth range used by splat_bin_sort.
 * splat_bin_sort: emits one (tile | depth) key per (Gaussian, tile) in Gaussian order,
 * radix-sorts them stably (ties keep entry order, as the reference's (key, entry) sort
 * does) and writes, for every sorted entry, its Gaussian index (gauss_dev), its 64-bit
 * reference key (keys_dev, optional: may be NULL) and the [start, end) range of every
 * tile (tile_range_dev, 2 x uint32 per tile, Binning::tile_range).
 * -------------------------------------------------------------------------------------- */
SPLAT_API int splat_bin_count(splat_ctx* ctx, const uint32_t* num_tiles_dev, int64_t n,
                              uint32_t* entry_offset_dev, int64_t* num_entries);
/* splat_bin_count for callers that cannot let this library allocate device memory: hosts
 * that plan all device memory themselves (a fixed per-frame budget, or their own allocator
 * owning the device) and cannot afford the synchronisation cudaMalloc/cudaFree may cause.
 * It has no counterpart in the reference. Same inputs, outputs and result as
 * splat_bin_count, but its scratch is a fixed 32 KiB array in device memory held by every
 * GPU that loads the library, so n may be at most 16,777,216 (larger n returns
 * SPLAT_ERR_CAPACITY). The first call on each device looks the array's address up; make
 * it before any stream capture; the address is cached for the process and does not
 * survive cudaDeviceReset. All calls share the array: calls that overlap on the GPU race.
 * Allocates nothing; synchronises to return the count. */
SPLAT_API int splat_bin_count_noalloc(splat_ctx* ctx, const uint32_t* num_tiles_dev, int64_t n,
                                      uint32_t* entry_offset_dev, int64_t* num_entries);
SPLAT_API int splat_bin_sort(splat_ctx* ctx, const float* proj_dev, const uint32_t* entry_offset_dev, int64_t n,
                             int64_t num_entries, const uint32_t* depth_range_dev, uint32_t width, uint32_t height,
                             uint32_t* gauss_dev, uint64_t* keys_dev, uint32_t* tile_range_dev);

/* The same binning with no host read-back, for callers that queue whole steps ahead (or
 * capture them in a CUDA graph): splat_bin_count_device writes the entry count to device
 * memory (*num_entries_dev, uint64) instead of returning it, and splat_bin_sort_device
 * reads it there. Buffers are sized for `capacity` entries: gauss_dev holds capacity
 * values and scratch_dev splat_bin_sort_device_scratch_bytes(capacity) bytes. When the
 * count exceeds capacity the call sorts only the first `capacity` entries and sets
 * *overflow_dev to 1 (it is never cleared here): the view must then be redone with larger
 * buffers. Otherwise gauss_dev and tile_range_dev equal splat_bin_sort's. */
SPLAT_API int splat_bin_count_device(splat_ctx* ctx, const uint32_t* num_tiles_dev, int64_t n,
                                     uint32_t* entry_offset_dev, uint64_t* num_entries_dev);
SPLAT_API size_t splat_bin_sort_device_scratch_bytes(int64_t capacity);
SPLAT_API int splat_bin_sort_device(splat_ctx* ctx, const float* proj_dev, const uint32_t* entry_offset_dev, int64_t n,
                                    const uint64_t* num_entries_dev, int64_t capacity,
                                    const uint32_t* depth_range_dev, uint32_t width, uint32_t height,
                                    void* scratch_dev, uint32_t* gauss_dev, uint32_t* tile_range_dev,
                                    uint32_t* overflow_dev);

/* ----------------------------------------------------------------------------------------
 * Compositing forward: rasterize_forward (reference src/rasterize.rs:305-337,
 * forward_tile :249-302). Writes image (H*W*3), final transmittance (H*W) and n_contrib
 * (H*W). `pairs_dev` (optional, 1 x uint64, accumulated) counts evaluated (entry, pixel)
 * pairs.
 * -------------------------------------------------------------------------------------- */
SPLAT_API int splat_rasterize_fwd(splat_ctx* ctx, const float* proj_dev, const uint32_t* gauss_dev,
                                  const uint32_t* tile_range_dev, uint32_t width, uint32_t height,
                                  const float background[3], float* image_dev, float* final_t_dev,
                                  uint32_t* n_contrib_dev, uint64_t* pairs_dev);

/* Compositing backward: rasterize_backward (reference src/rasterize.rs:459-505,
 * backward_tile :354-455). Accumulates into pgrad_dev (3 planes, stride cap), which the
 * caller zeroes (splat_zero) before the first view whose gradients it wants. */
SPLAT_API int splat_rasterize_bwd(splat_ctx* ctx, const float* proj_dev, const uint32_t* gauss_dev,
                                  const uint32_t* tile_range_dev, uint32_t width, uint32_t height,
                                  const float background[3], const float* final_t_dev,
                                  const uint32_t* n_contrib_dev, const float* dimage_dev, float* pgrad_dev,
                                  int64_t cap, uint64_t* pairs_dev);

/* The compositing backward with the reference's own reduction, bit for bit
 * (src/rasterize.rs:341-505): every entry's 11 gradient slots (and the blending weight) are
 * summed over its pixel rectangle in row-major order, in the reference's unfused f32
 * arithmetic with the correctly rounded exp, stored per entry in emission order
 * (rasterize.rs:449-454), then summed per Gaussian over its contiguous entries in order
 * (:480-503). WRITES pgrad_dev (3 planes, stride cap), it does not accumulate. Needs the
 * reference's 16x16 tiles (splat_set_raster_config) and entry_offset_dev / num_entries from
 * splat_bin_count. Slower than splat_rasterize_bwd, whose float atomics sum in an
 * unspecified order; for bit-exact comparison with the reference's CPU path. */
SPLAT_API int splat_rasterize_bwd_deterministic(splat_ctx* ctx, const float* proj_dev, const uint32_t* gauss_dev,
                                                const uint32_t* tile_range_dev, const uint32_t* entry_offset_dev,
                                                int64_t n, int64_t num_entries, uint32_t width, uint32_t height,
                                                const float background[3], const float* final_t_dev,
                                                const uint32_t* n_contrib_dev, const float* dimage_dev,
                                                float* pgrad_dev, int64_t cap);

/* ----------------------------------------------------------------------------------------
 * Projection backward: project_backward_all (reference src/project.rs:477-493,
 * project_backward_one :335-474). Writes the 59 parameter gradients into grad_planes_dev
 * (parameter-plane layout). If `stats_dev` is not NULL it also performs
 * DensifyStats::accumulate (reference src/densify.rs:36-60) for this view: stats_dev holds
 * grad_accum (float, cap), denom (uint32, cap) and max_radii (uint32, cap), in that order;
 * `absgrad` selects the AbsGS accumulators.
 * -------------------------------------------------------------------------------------- */
SPLAT_API int splat_project_bwd(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap,
                                const splat_camera* cam, const splat_proj_opts* opts, const float* proj_dev,
                                const float* pgrad_dev, float* grad_planes_dev, void* stats_dev, int32_t absgrad);

/* Diagnostic: the largest relative error of the fast exp used for the backward pass's
 * screening against the correctly rounded exp, over every float x with |x| in [lo, hi]
 * (negative != 0 selects -|x|). Synchronises. */
SPLAT_API int splat_diag_fast_exp_error(splat_ctx* ctx, float lo, float hi, int32_t negative, float* max_rel_error);

/* Diagnostic: the paired (f32x2) arithmetic of the compositing backward and the SSIM loss
 * against scalar arithmetic with one rounding per operation, on n seeded inputs:
 * mismatches2[0] counts sigma values (rasterize.rs:236) that differ, mismatches2[1] blur
 * accumulation steps (loss.rs:42-70). Both must be 0. Synchronises. */
SPLAT_API int splat_diag_pair_exact(splat_ctx* ctx, uint32_t n, uint32_t* mismatches2);

/* Diagnostic of the bounded waits of the tensor-core kernels: one block waits on an
 * mbarrier with `limit` tries (1..4194304; the kernels use 4194304), through the same wait
 * and error word as those kernels. With arrive == 0 nothing arrives: the wait runs out and
 * the call returns SPLAT_ERR_TIMEOUT. With arrive != 0 the phase completes first and it
 * returns SPLAT_OK. The context stays usable either way. Synchronises. */
SPLAT_API int splat_diag_mbarrier_wait(splat_ctx* ctx, uint32_t limit, int32_t arrive);

/* Diagnostic: throughput of the units that bound the compositing kernels, measured on the
 * context's device (no counterpart in the reference). unit 0: FP32 fused multiply-adds,
 * *ops_per_s in FLOP/s (2 per FMA); unit 1: special-function unit ex2 (the fast exp),
 * operations/s. One timed launch of about 2 ms (*ms) after an untimed one, CUDA events on
 * the context's stream, at the current SM clock. Synchronises. */
SPLAT_API int splat_diag_peak(splat_ctx* ctx, int32_t unit, double* ops_per_s, float* ms);

/* project_backward_all fused with Adam::step (reference src/project.rs:477-493,
 * src/adam.rs:77-161): the parameter gradients stay in registers and update planes_dev in
 * place together with the moments m_dev and v_dev (parameter-plane layout, capacity cap);
 * `step` is the Adam step count after the increment. Optional densification statistics as
 * in splat_project_bwd. Results equal splat_project_bwd followed by splat_adam_step. With a
 * BF16 render copy (bf16_dev, see splat_params_to_bf16; may be NULL) the gradient is taken
 * at the copy's values and the copy is rewritten from the updated f32 planes. */
SPLAT_API int splat_project_bwd_adam(splat_ctx* ctx, float* planes_dev, float* m_dev, float* v_dev, int64_t n,
                                     int64_t cap, const splat_camera* cam, const splat_proj_opts* opts,
                                     const float* proj_dev, const float* pgrad_dev, void* stats_dev, int32_t absgrad,
                                     uint64_t step, const splat_lr* lr, void* bf16_dev);

/* ----------------------------------------------------------------------------------------
 * The learned-densification network (no counterpart in the reference): per Gaussian, 16
 * features -> 64 SiLU -> 64 SiLU -> 3 logits -> softmax over {keep, clone/split, prune},
 * BF16 operands on the tensor cores with FP32 accumulation. Its parameters are one FP32
 * vector of splat_mlp_num_params() values: W1 [16][64], b1 [64], W2 [64][64], b2 [64],
 * W3 [64][3], b3 [3] (W[in][out]).
 *   splat_mlp_forward: probabilities (n x 3) of n feature rows (n x 16).
 *   splat_mlp_forward_tc: the same on the 5th-generation tensor cores (tcgen05 MMAs,
 *     accumulators in tensor memory, persistent blocks of 128-row tiles); x_dev 16-byte
 *     aligned; same rounding points, sums in another order. Synchronises; a timed-out wait
 *     for the tensor cores returns SPLAT_ERR_TIMEOUT.
 *   splat_mlp_grad: adds to grad_dev the gradient of the weighted mean cross-entropy
 *     sum_s w_s * -log p_s[y_s] / sum_s w_s (labels y in 0..2; scale = 1 / sum_s w_s).
 *   splat_mlp_grad_tc: the same on tcgen05 (tensor-memory accumulators for the layer
 *     outputs and the weight gradients, which are summed over each CTA's tiles; x_dev
 *     16-byte aligned). Synchronises; SPLAT_ERR_TIMEOUT if a tensor-core wait ran out.
 *   splat_mlp_adam: one Adam step (beta 0.9 / 0.999, eps 1e-8) on the FP32 parameters.
 * -------------------------------------------------------------------------------------- */
SPLAT_API int32_t splat_mlp_num_params(void);
SPLAT_API int splat_mlp_forward(splat_ctx* ctx, const float* x_dev, int64_t n, const float* theta_dev, float* prob_dev);
SPLAT_API int splat_mlp_forward_tc(splat_ctx* ctx, const float* x_dev, int64_t n, const float* theta_dev,
                                  float* prob_dev);
SPLAT_API int splat_mlp_grad(splat_ctx* ctx, const float* x_dev, const int32_t* y_dev, const float* w_dev, int64_t n,
                             float scale, const float* theta_dev, float* grad_dev);
SPLAT_API int splat_mlp_grad_tc(splat_ctx* ctx, const float* x_dev, const int32_t* y_dev, const float* w_dev,
                               int64_t n, float scale, const float* theta_dev, float* grad_dev);
SPLAT_API int splat_mlp_adam(splat_ctx* ctx, float* theta_dev, const float* grad_dev, float* m_dev, float* v_dev,
                             uint64_t step, float lr);

/* ----------------------------------------------------------------------------------------
 * Compositing configuration (not in the reference): tile shape, shared-memory chunk depth
 * and the backward's pixels per thread, held by the context and used by every later launch
 * (projection, binning and compositing must run under the same one). 16x16 tiles are the
 * reference's and give its tile lists; 8x8 and 16x32 give other lists but identical
 * images, final transmittances and, up to summation order, gradients (each entry's pixel
 * rectangle is first narrowed to its 16-pixel tile rectangle). Chunk depth: entries
 * staged in shared memory per round, 32, 64, 128 or 256 (with 16-pixel-wide tiles it sets
 * the backward's; their forward always stages 256). Pixels per thread of the
 * backward: 1 or 2 (a warp then covers 8x8 pixels). Default 16x16, 256, 2.
 *   splat_raster_candidates: writes the supported (tile_w, tile_h, chunk,
 *     pixels_per_thread) quadruples to out (4 values each; out may be NULL) and returns
 *     how many (24).
 *   splat_set_raster_config: SPLAT_ERR_INVALID for an unsupported quadruple.
 *   splat_autotune_render: times projection + binning + forward + backward compositing of
 *     one view (dimage_dev: dL/dimage, H*W*3) under every candidate, `reps` timed passes
 *     each after an untimed one, sets the fastest on the context and writes the mean
 *     milliseconds per pass of every candidate to ms_out (one per candidate) and the pick
 *     to picked (4).
 *     Synchronises; changes no caller buffer.
 * -------------------------------------------------------------------------------------- */
SPLAT_API int32_t splat_raster_candidates(uint32_t* out);
SPLAT_API int splat_set_raster_config(splat_ctx* ctx, uint32_t tile_w, uint32_t tile_h, uint32_t chunk,
                                      uint32_t pixels_per_thread);
SPLAT_API int splat_get_raster_config(splat_ctx* ctx, uint32_t* out4);
SPLAT_API int splat_autotune_render(splat_ctx* ctx, const float* planes_dev, int64_t n, int64_t cap,
                                    const splat_camera* cam, const splat_proj_opts* opts, const float* background,
                                    const float* dimage_dev, int32_t reps, float* ms_out, uint32_t* picked);

/* Fill `bytes` bytes of device memory with zeros on the context stream (no reference
 * counterpart: host vectors there are zeroed on allocation). */
SPLAT_API int splat_zero(splat_ctx* ctx, void* dev, size_t bytes);

/* ----------------------------------------------------------------------------------------
 * Renderer: a model resident in device memory, driven with HOST buffers. All calls but
 * splat_renderer_submit_backward synchronise before returning.
 *   splat_renderer_set_model: upload n reference Gaussian records (aos59, host) and the
 *     model's active SH degree (Model::sh_degree, reference src/model.rs:54-61).
 *   splat_renderer_render: render::render (reference src/render.rs:14-23) into a host
 *     H*W*3 image (the model's SH degree overrides opts->sh_degree, as project_all does,
 *     src/project.rs:321-324).
 *   splat_renderer_render_backward: the differentiable chain of examples/profile.rs:34-52:
 *     project_all -> bin -> rasterize_forward (image to image_host if not NULL) ->
 *     rasterize_backward with dimage_host (H*W*3) -> project_backward_all, writing the
 *     parameter gradients as n reference records (grads_aos59_host, may be NULL).
 * -------------------------------------------------------------------------------------- */
typedef struct splat_renderer splat_renderer;
SPLAT_API int splat_renderer_create(splat_ctx* ctx, splat_renderer** out);
SPLAT_API int splat_renderer_destroy(splat_renderer* r);
SPLAT_API int splat_renderer_set_model(splat_renderer* r, const float* aos59_host, int64_t n, int32_t sh_degree);
SPLAT_API int splat_renderer_render(splat_renderer* r, const splat_camera* cam, const splat_proj_opts* opts,
                                    const float background[3], float* image_host);
SPLAT_API int splat_renderer_render_backward(splat_renderer* r, const splat_camera* cam, const splat_proj_opts* opts,
                                             const float background[3], const float* dimage_host, float* image_host,
                                             float* grads_aos59_host);
/* splat_renderer_render_backward split in two so that consecutive views overlap: submit
 * queues the step and returns a ticket once its work is queued (it waits on the host only for
 * the forward pass's entry count and, when two steps are already in flight, for the older of
 * them); splat_renderer_wait(ticket) returns when that step's image and gradients are in the
 * host buffers. Up to two steps are in flight, so step k+1 computes while step k's gradients
 * cross PCIe. The three host buffers belong to the step until its wait returns (pinned host
 * memory lets the copies run asynchronously). splat_renderer_render_backward is submit
 * followed by wait. Waiting on a step that is already complete returns SPLAT_OK at once. */
SPLAT_API int splat_renderer_submit_backward(splat_renderer* r, const splat_camera* cam, const splat_proj_opts* opts,
                                             const float background[3], const float* dimage_host, float* image_host,
                                             float* grads_aos59_host, uint64_t* ticket);
SPLAT_API int splat_renderer_wait(splat_renderer* r, uint64_t ticket);
/* Tile entries of the last rendered view (Binning::sorted.len()). */
SPLAT_API int64_t splat_renderer_last_entries(const splat_renderer* r);

/* ----------------------------------------------------------------------------------------
 * Loss: photometric_loss (reference src/loss.rs:137-171, ssim_with_grad :75-134) with the
 * prediction pred_dev (H*W*3 float) against target_dev, either 8-bit pixels converted as
 * View::to_real does (target_is_u8 = 1, reference src/dataset.rs:23-25) or floats. Writes
 * d loss / d pred to grad_dev and (loss, mean SSIM, PSNR) to out3_dev (3 floats; PSNR as
 * in loss.rs:175-190).
 * -------------------------------------------------------------------------------------- */
SPLAT_API int splat_loss_fwd_bwd(splat_ctx* ctx, const float* pred_dev, const void* target_dev, int32_t target_is_u8,
                                 uint32_t width, uint32_t height, float lambda_dssim, float* grad_dev,
                                 float* out3_dev);

/* Adam::step (reference src/adam.rs:77-161) on parameter planes: params, first and second
 * moments updated in place from the gradient planes. `step` is the step count after the
 * increment (1 for the first step); beta1 0.9, beta2 0.999, eps 1e-15. */
SPLAT_API int splat_adam_step(splat_ctx* ctx, float* planes_dev, const float* grad_planes_dev, float* m_dev,
                              float* v_dev, int64_t n, int64_t cap, uint64_t step, const splat_lr* lr);

/* What one densification step did (reference src/densify.rs:107-114) and the new count. */
typedef struct splat_densify_report {
  uint64_t cloned, split, pruned, new_count;
} splat_densify_report;

/* densify_and_prune (reference src/densify.rs:125-221): clone, split and prune n Gaussians
 * (params, Adam moments, statistics as written by splat_project_bwd) into the output
 * planes (capacity cap_out), in the reference's order: surviving originals, surviving
 * clones, surviving split children. Split offsets are drawn from the SplitMix64 generator
 * whose state is *rng_state (advanced in place), per split parent, per child, x then y
 * then z, with Box-Muller normals. If the survivors exceed cap_out the call returns
 * SPLAT_ERR_CAPACITY with report->new_count set, writes nothing and leaves *rng_state
 * unchanged. Synchronises once to read the counts. */
SPLAT_API int splat_densify(splat_ctx* ctx, const float* planes_dev, const float* m_dev, const float* v_dev, int64_t n,
                            int64_t cap, const void* stats_dev, const splat_densify_config* cfg, float extent,
                            uint64_t* rng_state, float* planes_out_dev, float* m_out_dev, float* v_out_dev,
                            int64_t cap_out, splat_densify_report* report);

/* reset_opacity (reference src/densify.rs:224-230): opacity logits clamped to
 * inverse_sigmoid(max_alpha) and the opacity moments zeroed. */
SPLAT_API int splat_reset_opacity(splat_ctx* ctx, float* planes_dev, float* m_dev, float* v_dev, int64_t n,
                                  float max_alpha);

/* ----------------------------------------------------------------------------------------
 * Initialisation from a sparse point cloud: Model::from_points (reference
 * src/model.rs:77-104) with mean_nn_dist2 (:128-186), an exact brute-force 3-NN search.
 *   splat_mean_nn_dist2: points (n x 3 float, device) -> mean squared distance to the three
 *     nearest other points (n doubles, device); coincident points count as neighbours.
 *   splat_init_from_points: points (n x 3 float) and colours (n x 3 uint8) on the host ->
 *     n Gaussians in parameter planes (capacity cap) on the device. Synchronises.
 * -------------------------------------------------------------------------------------- */
SPLAT_API int splat_mean_nn_dist2(splat_ctx* ctx, const float* points_dev, int64_t n, double* out_dev);
SPLAT_API int splat_init_from_points(splat_ctx* ctx, const float* points_host, const uint8_t* rgb_host, int64_t n,
                                     float* planes_dev, int64_t cap);

/* ----------------------------------------------------------------------------------------
 * PLY codec: the standard 3DGS binary little-endian float32 layout (reference
 * src/ply.rs:19-181) straight into / out of parameter planes on the device.
 *   splat_ply_read_header: vertex count and SH degree (from the f_rest count) of a file.
 *   splat_ply_read: read (ply.rs:73-181) into planes of capacity cap (SPLAT_ERR_CAPACITY if
 *     the file holds more Gaussians); property order is taken from the header; format
 *     errors return SPLAT_ERR_INVALID with the reference's messages.
 *   splat_ply_write: write (ply.rs:19-69) n Gaussians with coefficients up to sh_degree.
 * -------------------------------------------------------------------------------------- */
SPLAT_API int splat_ply_read_header(splat_ctx* ctx, const char* path, int64_t* count, int32_t* sh_degree);
SPLAT_API int splat_ply_read(splat_ctx* ctx, const char* path, float* planes_dev, int64_t cap, int64_t* count,
                             int32_t* sh_degree);
SPLAT_API int splat_ply_write(splat_ctx* ctx, const char* path, const float* planes_dev, int64_t n, int64_t cap,
                              int32_t sh_degree);

/* ----------------------------------------------------------------------------------------
 * Trainer: train::train (reference src/train.rs:161-306) one iteration per call, with the
 * model, Adam state, statistics and the training views (8-bit pixels) resident in device
 * memory. The view order and split offsets come from a SplitMix64 generator seeded with
 * cfg->seed (the reference uses ChaCha8; the schedule is otherwise the reference's).
 * -------------------------------------------------------------------------------------- */
typedef struct splat_trainer splat_trainer;

/* Progress of one iteration (reference src/train.rs:142-157, DensifyReport). */
typedef struct splat_step_info {
  double loss;
  double psnr; /* of this iteration's render against its view */
  uint32_t view;
  int32_t densified;
  int32_t reset;
  uint64_t num_gaussians;
  uint64_t cloned, split, pruned;
  uint64_t entries;
  uint32_t replayed; /* not in the reference: 1 when the iteration ran as a replayed CUDA graph */
} splat_step_info;

/* Fails with SPLAT_ERR_INVALID for zero iterations or sh_degree > 3 (train.rs:169-183). */
SPLAT_API int splat_trainer_create(splat_ctx* ctx, const splat_train_config* cfg, float extent, splat_trainer** out);
SPLAT_API int splat_trainer_destroy(splat_trainer* t);
/* Initial model as n reference records (e.g. from Model::from_points). */
SPLAT_API int splat_trainer_set_model(splat_trainer* t, const float* aos59_host, int64_t n);
/* One training view: camera and H*W*3 8-bit pixels (View, reference src/dataset.rs:14-26). */
SPLAT_API int splat_trainer_add_view(splat_trainer* t, const splat_camera* cam, const uint8_t* rgb_host);
/* Reset generator, optimiser state and statistics; SH degree 0 (train.rs:184-189). */
SPLAT_API int splat_trainer_start(splat_trainer* t);
/* `iterations` iterations of splat_trainer_step in one call, queued one iteration ahead of
 * the device (no host wait inside an iteration); `info` describes the last one, with the
 * densification fields of the last iteration that densified. */
SPLAT_API int splat_trainer_run(splat_trainer* t, uint32_t iterations, splat_step_info* info);
SPLAT_API int splat_trainer_step(splat_trainer* t, splat_step_info* info);
SPLAT_API int64_t splat_trainer_count(const splat_trainer* t);
/* The trainer's densification network (splat_mlp_num_params() floats, layout as
 * splat_mlp_forward), and what learning did so far: out[0] densifications learned from,
 * out[1] records trained on, out[2..4] hindsight labels keep / clone-split / prune, out[5]
 * Adam steps of the network, out[6..8] held-out accuracy (each densification's labels
 * predicted before training on them): records the network got right, records the rule's
 * own action got right, records. */
SPLAT_API int splat_trainer_get_mlp(splat_trainer* t, float* theta_host);
SPLAT_API int splat_trainer_set_mlp(splat_trainer* t, const float* theta_host);
SPLAT_API int splat_trainer_mlp_stats(const splat_trainer* t, uint64_t out[9]);
/* Autotuning (splat_train_config.autotune): the last tuning's milliseconds per render pass
 * of every candidate (ms_out, one per candidate, in splat_raster_candidates order; 0 before any), the
 * configuration in use (picked, 4) and how many tunings ran. Any pointer may be NULL. */
SPLAT_API int splat_trainer_tuning(const splat_trainer* t, float* ms_out, uint32_t* picked, uint32_t* tunes);
SPLAT_API int32_t splat_trainer_sh_degree(const splat_trainer* t);
SPLAT_API uint32_t splat_trainer_iteration(const splat_trainer* t);
SPLAT_API int splat_trainer_get_model(splat_trainer* t, float* aos59_host);
/* The optimiser's state: Adam's first and second moments (reference Adam::m / Adam::v,
 * src/adam.rs:28-41), one 59-float record per Gaussian in the model's order. */
SPLAT_API int splat_trainer_get_moments(splat_trainer* t, float* m_aos59_host, float* v_aos59_host);
/* render::render of the current model at the active SH degree and the config's background. */
SPLAT_API int splat_trainer_render(splat_trainer* t, const splat_camera* cam, float* image_host);
/* evaluate (train.rs:309-321) on the device: renders every training view with the current
 * model (trainer's SH degree and background) and scores it with the loss kernel. Writes
 * the mean PSNR (loss.rs:175-190; NaN without views) to *mean_psnr and, when per_view3_host
 * is not NULL, {loss, SSIM, PSNR} of every view (3 floats per view, in the order the views
 * were added). One host wait for all views. */
SPLAT_API int splat_trainer_evaluate(splat_trainer* t, float* per_view3_host, double* mean_psnr);

#ifdef __cplusplus
}
#endif

#endif /* SPLAT_GPU_H */
