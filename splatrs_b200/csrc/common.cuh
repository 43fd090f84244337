// Shared definitions for the sm_100a kernels and their host launchers.
//
// Every translation unit is compiled with --fmad=false: a*b+c is two roundings, as in the
// reference's Rust, so decisions taken on float values (the alpha and transmittance
// thresholds, tile rectangles, radii) come out exactly as the reference computes them.
// Kernels that only accumulate gradients opt in to fused multiply-adds explicitly.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/splat_gpu.h"
#include "crmath.h"

namespace splat {

constexpr int kPlanes = SPLAT_PLANES;
constexpr int kProjFloats = SPLAT_PROJ_FLOATS;
constexpr uint32_t kTile = SPLAT_TILE;

// Error carried from a launcher to the C ABI.
struct Status {
  int code = SPLAT_OK;
  std::string msg;
  static Status ok() { return Status(); }
  static Status make(int c, std::string m) {
    Status s;
    s.code = c;
    s.msg = std::move(m);
    return s;
  }
  bool good() const { return code == SPLAT_OK; }
};

inline Status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return Status::ok();
  return Status::make(SPLAT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define SPLAT_TRY(expr)            \
  do {                             \
    ::splat::Status _s = (expr);   \
    if (!_s.good()) return _s;     \
  } while (0)

#define SPLAT_CUDA(expr) SPLAT_TRY(::splat::cuda_status((expr), #expr))
#define SPLAT_LAUNCHED(what) SPLAT_TRY(::splat::cuda_status(cudaGetLastError(), what))

// Scratch memory handed out by the context: a list of device chunks. Reserving never
// moves memory already handed out; chunks are merged at the next reset.
struct ArenaChunk {
  void* ptr;
  size_t size;
};
struct Arena {
  std::vector<ArenaChunk> chunks;
  size_t used = 0;       // bytes used in the last chunk
  uint64_t generation = 0;  // changes whenever chunks are allocated or freed
};

// Launch bookkeeping shared by all launchers.
struct LaunchCounter {
  uint64_t count = 0;
};

// Compositing configuration: tile shape in pixels, shared-memory chunk depth (entries
// staged per round) and the backward's pixels per thread. 16x16 is the reference's tile and binning; 8x8 and 16x32 composite the
// same entries per pixel in the same order (the projection narrows each entry's pixel
// rectangle to its 16-pixel tile rectangle first), so images match the 16x16 path.
struct RasterConfig {
  uint32_t tile_w = kTile, tile_h = kTile, chunk = 256;
  uint32_t ppl = 2;  // pixels per thread of the compositing backward (1 or 2)
  bool operator==(const RasterConfig& o) const {
    return tile_w == o.tile_w && tile_h == o.tile_h && chunk == o.chunk && ppl == o.ppl;
  }
  bool operator!=(const RasterConfig& o) const { return !(*this == o); }
  bool reference_tiles() const { return tile_w == kTile && tile_h == kTile; }
  uint32_t tiles_x(uint32_t width) const { return (width + tile_w - 1) / tile_w; }
  uint32_t tiles_y(uint32_t height) const { return (height + tile_h - 1) / tile_h; }
  uint32_t tiles(uint32_t width, uint32_t height) const { return tiles_x(width) * tiles_y(height); }
  // Tile shapes {8x8, 16x16, 16x32} x chunk depths {32, 64, 128, 256} x backward pixels
  // per thread {1, 2}.
  static bool supported(uint32_t w, uint32_t h, uint32_t chunk, uint32_t ppl) {
    const bool shape = (w == 8 && h == 8) || (w == 16 && h == 16) || (w == 16 && h == 32);
    return shape && (chunk == 32 || chunk == 64 || chunk == 128 || chunk == 256) && (ppl == 1 || ppl == 2);
  }
};
// Most tiles any supported shape gives an image (8x8): sizes per-tile buffers for all.
inline uint32_t max_tiles(uint32_t width, uint32_t height) { return ((width + 7) / 8) * ((height + 7) / 8); }

struct Ctx {
  int device = 0;
  RasterConfig raster;
  cudaStream_t stream = nullptr;
  Arena arena;
  LaunchCounter launches;
  std::string last_error;
  int sm_count = 148;
  // Mapped pinned host memory for small read-backs: kernels store into it through
  // host_small_dev, so a read-back never queues on a copy engine behind large transfers.
  void* host_small = nullptr;
  void* host_small_dev = nullptr;
};

// Reserve `bytes` of scratch (256-byte aligned) from the context arena. The arena is
// reset at the start of every public entry point; reserving more than is available
// reallocates it (after synchronising the stream, so no kernel still uses the old one).
Status arena_reserve(Ctx* c, size_t bytes, void** out);
void arena_reset(Ctx* c);
void arena_free(Ctx* c);

inline uint32_t ceil_div(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Float <-> bits.
__host__ __device__ __forceinline__ uint32_t fbits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t b;
  __builtin_memcpy(&b, &f, 4);
  return b;
#endif
}
__host__ __device__ __forceinline__ float bitsf(uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(b);
#else
  float f;
  __builtin_memcpy(&f, &b, 4);
  return f;
#endif
}

// Rust's saturating `as u32` for floats (NaN and negatives to 0).
__host__ __device__ __forceinline__ uint32_t sat_u32(float v) {
  if (!(v > 0.0f)) return 0u;
  if (v >= 4294967295.0f) return 0xffffffffu;
  return (uint32_t)v;
}

// Compositing constants (reference src/rasterize.rs:53-57).
#define SPLAT_ALPHA_MIN (1.0f / 255.0f)
#define SPLAT_ALPHA_MAX 0.99f
#define SPLAT_T_MIN 1e-4f

}  // namespace splat
