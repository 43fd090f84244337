// Device buffers of the render path, shared by the renderer and the trainer.
#pragma once
#include "common.cuh"

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
  Status ensure(int64_t n, uint32_t width, uint32_t height);
  void release();
};

// Projection, binning and forward compositing of one view. Synchronises once to read the
// number of tile entries back.
Status render_view(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                   const splat_proj_opts& opts, const float bg[3], ViewBuffers& v, int64_t* entries_out);

}  // namespace splat
