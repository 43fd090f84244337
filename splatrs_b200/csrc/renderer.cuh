// Device buffers of the render path, shared by the renderer and the trainer.
#pragma once
#include "common.cuh"
#include "kernels.cuh"

struct splat_ctx;

namespace splat {

// The Ctx inside a public splat_ctx handle (defined in capi.cu).
Ctx* splat_ctx_impl(splat_ctx* ctx);

// A grow-only device allocation.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  Status ensure(size_t want);
  void release();
  template <typename T> T* as() const { return reinterpret_cast<T*>(ptr); }
};

// Per-view buffers: projection records, binning and forward outputs.
struct ViewBuffers {
  DevBuf proj, num_tiles, entry_offset, depth_range, tile_range, gauss, image, final_t, n_contrib, dimage, pairs;
  // Device-driven binning (render_view_dev): sort scratch for e_cap entries, scan partials,
  // and counters = {uint64 entry count, uint32 overflow flag (sticky), pad}.
  DevBuf sort_scratch, scan_partial, counters;
  int64_t e_cap = 0;
  Status ensure(int64_t n, uint32_t width, uint32_t height);
  // A batch: `records` projection records, `pixels` pixels and `tiles` tiles in all.
  Status ensure_batch(int64_t records, uint64_t pixels, uint32_t tiles);
  void release();
  uint64_t* entry_count() const { return counters.as<uint64_t>(); }
  uint32_t* overflow_flag() const { return counters.as<uint32_t>() + 2; }
};

// Projection, binning and forward compositing of one view. Synchronises once to read the
// number of tile entries back.
Status render_view(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                   const splat_proj_opts& opts, const float bg[3], ViewBuffers& v, int64_t* entries_out,
                   const void* bf16 = nullptr);

// The same without any host wait: binning reads the entry count on the device and sorts at
// most e_cap entries (v.e_cap, set by the caller; buffers grow to it here). If the view
// has more, *v.overflow_flag() becomes 1 and the view's outputs are invalid.
Status render_view_dev(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                       const splat_proj_opts& opts, const float bg[3], ViewBuffers& v,
                       const StepParams* sp = nullptr, const void* bf16 = nullptr);

}  // namespace splat
