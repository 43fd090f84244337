// Front-to-back alpha compositing, forward and backward (reference src/rasterize.rs).
//
// One block per tile (16x16 by default; 8x8 and 16x32 too), one pixel per thread. Warps own
// 8x4 pixel sub-blocks so that an entry whose pixel rectangle misses a sub-block is skipped
// by the whole warp with one uniform branch. The tile's sorted entries are staged through
// shared memory in chunks of CH entries (32-256; each entry's 48-byte record gathered by one
// thread). Tile shape and chunk depth are template parameters, chosen at run time from the
// context's configuration (the autotuner's pick). Every
// per-pixel decision (sigma range, alpha >= 1/255, the 0.99 clamp, T < 1e-4) is taken on
// values computed exactly as the reference computes them: unfused arithmetic and a
// correctly rounded exp.
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"
#include "pair.cuh"

namespace splat {

// Geometry of a TW x TH tile: TW * TH threads, warps over 8x4 sub-blocks row by row. An
// entry's pixel rectangle within the tile is a column mask and a row mask packed in one
// word (rows from bit kRowShift), 32 bits while the rows fit in 16, else 64.
template <int TW, int TH>
struct TileGeo {
  static constexpr int kThreads = TW * TH;
  static constexpr int kWarps = kThreads / 32;
  static constexpr int kWarpsX = TW / 8;
  static constexpr int kRowShift = TH > 16 ? 32 : 16;
  typedef typename std::conditional<(TH > 16), unsigned long long, uint32_t>::type Mask;
  typedef typename std::conditional<(kWarps > 8), uint16_t, uint8_t>::type WarpMask;
  static_assert(TW % 8 == 0 && TH % 4 == 0 && TW <= 16 && TH <= 32, "tile shape");
};

struct PixelGeom {
  uint32_t px_i, py_j;   // absolute pixel
  uint32_t bx0, by0;     // warp sub-block origin
  bool inside;
};

template <int TW, int TH>
__device__ __forceinline__ PixelGeom pixel_geom(uint32_t tile, uint32_t tiles_x, uint32_t width, uint32_t height) {
  constexpr int WX = TileGeo<TW, TH>::kWarpsX;
  const uint32_t tx = tile % tiles_x, ty = tile / tiles_x;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  PixelGeom p;
  p.bx0 = tx * TW + (warp % WX) * 8u;
  p.by0 = ty * TH + (warp / WX) * 4u;
  p.px_i = p.bx0 + (lane & 7u);
  p.py_j = p.by0 + (lane >> 3);
  p.inside = p.px_i < width && p.py_j < height;
  return p;
}


__constant__ double kExp2Tab64[64] = CRM_EXP2_TAB64;

// evaluate (rasterize.rs:231-244). Returns false when skipped. `tab` is the table of
// crm::expf_cr_neg in shared memory.
__device__ __forceinline__ bool evaluate(float px, float py, float mx, float my, float A, float B, float C,
                                         float opacity, float sigma_max, const double* tab, float* gauss_out,
                                         float* alpha_out) {
  const float dx = px - mx;
  const float dy = py - my;
  const float sigma = 0.5f * (A * dx * dx + C * dy * dy) + B * dx * dy;
  if (sigma < 0.0f || sigma > sigma_max) return false;
  const float gauss = crm::expf_cr_neg(-sigma, tab);
  const float og = opacity * gauss;
  if (og < SPLAT_ALPHA_MIN) return false;
  *gauss_out = gauss;
  *alpha_out = fminf(og, SPLAT_ALPHA_MAX);
  return true;
}

// evaluate (rasterize.rs:231-244) with the general correctly rounded exp: same values and
// decisions as evaluate() (the narrow-range table form equals it on the whole argument range).
__device__ __forceinline__ bool evaluate_ref(float px, float py, float mx, float my, float A, float B, float C,
                                             float opacity, float sigma_max, float* gauss_out, float* alpha_out) {
  const float dx = px - mx;
  const float dy = py - my;
  const float sigma = 0.5f * (A * dx * dx + C * dy * dy) + B * dx * dy;
  if (sigma < 0.0f || sigma > sigma_max) return false;
  const float gauss = crm::expf_cr(-sigma);
  const float og = opacity * gauss;
  if (og < SPLAT_ALPHA_MIN) return false;
  *gauss_out = gauss;
  *alpha_out = fminf(og, SPLAT_ALPHA_MAX);
  return true;
}

// evaluate for the backward pass. The decisions must be the forward's, which were taken on
// the correctly rounded exp; the value may carry a few ulps. A fast exp (MUFU ex2) decides
// whenever the product opacity * gauss lies outside a relative band of kExpBand around the
// two thresholds (1/255 and 0.99); inside the band the correctly rounded exp is evaluated
// and decides. kExpBand bounds the fast exp's relative error on the argument range
// [-ln(255), 0] with a wide margin (the bound is checked on the device by
// splat_diag_fast_exp_error). *unclamped is the reference's `opacity * gauss < 0.99`.
constexpr float kExpBand = 3e-5f;

// exp(x) through the special-function unit: 2^(x log2 e), the product rounded to nearest,
// then ex2.approx (flush-to-zero). Relative error of the product's rounding is 2^-24 of an
// exponent below 9 in magnitude on the range used, and ex2.approx's own is about 2^-22;
// splat_diag_fast_exp_error measures the sum on every float of the range.
constexpr float kLog2e = 1.44269504088896341f;

__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float fast_exp(float x) { return ex2_approx(__fmul_rn(x, kLog2e)); }

// sigma = 0.5 (A dx dx + C dy dy) + B dx dy for a pair of pixels, operation for operation as
// the reference (rasterize.rs:236), one rounding per operation (f2_mul is never contracted).
// Also returns A dx, C dy and B dx for the gradients. A zero product may carry the other
// sign than the scalar one; no decision on sigma depends on the sign of a zero.
__device__ __forceinline__ f2 paired_sigma(f2 A, f2 B, f2 C, f2 dx, f2 dy, f2* adx, f2* cdy, f2* bdx) {
  *adx = f2_mul(A, dx);
  *cdy = f2_mul(C, dy);
  *bdx = f2_mul(B, dx);
  return f2_add(f2_mul(f2_splat(0.5f), f2_add(f2_mul(*adx, dx), f2_mul(*cdy, dy))), f2_mul(*bdx, dy));
}

__device__ __forceinline__ bool evaluate_bwd(float px, float py, float mx, float my, float A, float B, float C,
                                             float opacity, float sigma_max, float* gauss_out, float* alpha_out,
                                             bool* unclamped) {
  const float dx = px - mx;
  const float dy = py - my;
  const float sigma = 0.5f * (A * dx * dx + C * dy * dy) + B * dx * dy;
  if (sigma < 0.0f || sigma > sigma_max) return false;
  float gauss = fast_exp(-sigma);
  float og = opacity * gauss;
  const bool near_min = fabsf(og - SPLAT_ALPHA_MIN) < SPLAT_ALPHA_MIN * kExpBand;
  const bool near_max = fabsf(og - SPLAT_ALPHA_MAX) < SPLAT_ALPHA_MAX * kExpBand;
  if (near_min || near_max) {
    gauss = crm::expf_cr(-sigma);
    og = opacity * gauss;
  }
  if (og < SPLAT_ALPHA_MIN) return false;
  *gauss_out = gauss;
  *alpha_out = fminf(og, SPLAT_ALPHA_MAX);
  *unclamped = og < SPLAT_ALPHA_MAX;
  return true;
}

// Largest relative error of the fast exp against the correctly rounded one over every
// float in [lo, hi] (a diagnostic of the bound kExpBand relies on).
__global__ void diag_fast_exp_kernel(uint32_t lo_bits, uint32_t count, int negative, unsigned int* max_rel_bits) {
  float worst = 0.0f;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const uint32_t b = lo_bits + k;
    const float x = negative ? -__uint_as_float(b) : __uint_as_float(b);
    const float e = crm::expf_cr(x);
    const float f = fast_exp(x);
    if (e > 0.0f) worst = fmaxf(worst, fabsf(f - e) / e);
  }
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if ((threadIdx.x & 31) == 0) atomicMax(max_rel_bits, __float_as_uint(worst));
}

Status launch_diag_fast_exp(Ctx* c, float magnitude_lo, float magnitude_hi, int negative, float* out_host) {
  unsigned int* d = nullptr;
  SPLAT_TRY(arena_reserve(c, 4, (void**)&d));
  SPLAT_CUDA(cudaMemsetAsync(d, 0, 4, c->stream));
  const uint32_t lo = fbits(magnitude_lo), hi = fbits(magnitude_hi);
  diag_fast_exp_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(lo, hi - lo + 1, negative, d);
  c->launches.count++;
  SPLAT_LAUNCHED("diag_fast_exp_kernel");
  unsigned int h = 0;
  SPLAT_CUDA(cudaMemcpyAsync(&h, d, 4, cudaMemcpyDeviceToHost, c->stream));
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  *out_host = bitsf(h);
  return Status::ok();
}

// Paired arithmetic against scalar unfused arithmetic on seeded inputs: [0] counts pixels
// whose paired_sigma differs from the scalar sigma of rasterize.rs:236, [1] blur steps
// acc + w x (the SSIM loss's accumulation) that differ. Both must be zero.
__device__ __forceinline__ float diag_uniform(uint32_t i, uint32_t salt, float lo, float hi) {
  uint32_t h = i * 0x9e3779b9u ^ salt;
  h ^= h >> 16;
  h *= 0x7feb352du;
  h ^= h >> 15;
  h *= 0x846ca68bu;
  h ^= h >> 16;
  return lo + (hi - lo) * (float)(h >> 8) * (1.0f / 16777216.0f);
}

__global__ void diag_pair_exact_kernel(uint32_t n, unsigned int* __restrict__ mism) {
  unsigned int bad_sigma = 0, bad_blur = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float A = diag_uniform(i, 1u, 0.0f, 3.4f), B = diag_uniform(i, 2u, -1.7f, 1.7f);
    const float C = diag_uniform(i, 3u, 0.0f, 3.4f), dx = diag_uniform(i, 4u, -48.0f, 48.0f);
    const float dy0 = diag_uniform(i, 5u, -48.0f, 48.0f), dy1 = diag_uniform(i, 6u, -48.0f, 48.0f);
    f2 adx, cdy, bdx;
    float p0, p1;
    f2_split(paired_sigma(f2_splat(A), f2_splat(B), f2_splat(C), f2_splat(dx), f2_make(dy0, dy1), &adx, &cdy, &bdx),
             p0, p1);
    const float dys[2] = {dy0, dy1}, ps[2] = {p0, p1};
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const float dy = dys[q];
      const float s = __fadd_rn(__fmul_rn(0.5f, __fadd_rn(__fmul_rn(__fmul_rn(A, dx), dx), __fmul_rn(__fmul_rn(C, dy), dy))),
                                __fmul_rn(__fmul_rn(B, dx), dy));
      bad_sigma += !(ps[q] == s);
    }
    const float w = diag_uniform(i, 7u, 0.0f, 0.3f), acc0 = diag_uniform(i, 8u, -2.0f, 2.0f);
    const float acc1 = diag_uniform(i, 9u, 0.0f, 1.5f), x0 = diag_uniform(i, 10u, -0.2f, 1.2f);
    const float x1 = diag_uniform(i, 11u, 0.0f, 1.0f);
    float b0, b1;
    f2_split(f2_add(f2_make(acc0, acc1), f2_mul(f2_splat(w), f2_make(x0, x1))), b0, b1);
    bad_blur += !(b0 == __fadd_rn(acc0, __fmul_rn(w, x0))) + !(b1 == __fadd_rn(acc1, __fmul_rn(w, x1)));
  }
  for (int o = 16; o > 0; o >>= 1) {
    bad_sigma += __shfl_xor_sync(0xffffffffu, bad_sigma, o);
    bad_blur += __shfl_xor_sync(0xffffffffu, bad_blur, o);
  }
  if ((threadIdx.x & 31) == 0 && (bad_sigma | bad_blur)) {
    atomicAdd(&mism[0], bad_sigma);
    atomicAdd(&mism[1], bad_blur);
  }
}

Status launch_diag_pair_exact(Ctx* c, uint32_t n, uint32_t* out_host) {
  unsigned int* d = nullptr;
  SPLAT_TRY(arena_reserve(c, 8, (void**)&d));
  SPLAT_CUDA(cudaMemsetAsync(d, 0, 8, c->stream));
  diag_pair_exact_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(n, d);
  c->launches.count++;
  SPLAT_LAUNCHED("diag_pair_exact_kernel");
  SPLAT_CUDA(cudaMemcpyAsync(out_host, d, 8, cudaMemcpyDeviceToHost, c->stream));
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  return Status::ok();
}

// The entry's pixel rectangle within the TW x TH tile whose top-left pixel is (ox, oy) as a
// mask of the columns (low bits) and a mask of the rows (from bit kRowShift) it covers.
template <int TW, int TH>
__device__ __forceinline__ typename TileGeo<TW, TH>::Mask tile_rect_masks(uint32_t rx, uint32_t ry, uint32_t ox,
                                                                           uint32_t oy) {
  typedef typename TileGeo<TW, TH>::Mask Mask;
  const int x0 = (int)(rx & 0xffffu) - (int)ox, x1 = (int)(rx >> 16) - (int)ox;
  const int y0 = (int)(ry & 0xffffu) - (int)oy, y1 = (int)(ry >> 16) - (int)oy;
  const uint32_t cx0 = (uint32_t)min(max(x0, 0), TW), cx1 = (uint32_t)min(max(x1, 0), TW);
  const uint32_t cy0 = (uint32_t)min(max(y0, 0), TH), cy1 = (uint32_t)min(max(y1, 0), TH);
  const uint32_t cols = cx1 > cx0 ? ((0xffffffffu >> (32u - (cx1 - cx0))) << cx0) : 0u;
  const uint32_t rows = cy1 > cy0 ? ((0xffffffffu >> (32u - (cy1 - cy0))) << cy0) : 0u;
  return (Mask)cols | ((Mask)rows << TileGeo<TW, TH>::kRowShift);
}

// Bit w of the result is set when the pixel rectangle (x0|x1<<16, y0|y1<<16, absolute
// pixels) overlaps warp w's 8 x SBH sub-block of the tile whose top-left pixel is (ox, oy)
// (warps row by row, TW / 8 across).
template <int TW, int TH, int SBH = 4>
__device__ __forceinline__ uint32_t subblock_mask(uint32_t rx, uint32_t ry, uint32_t ox, uint32_t oy) {
  constexpr int WX = TileGeo<TW, TH>::kWarpsX;
  const uint32_t x0 = rx & 0xffffu, x1 = rx >> 16, y0 = ry & 0xffffu, y1 = ry >> 16;
  bool col[WX];
#pragma unroll
  for (int qx = 0; qx < WX; qx++) col[qx] = x0 < ox + 8u * qx + 8u && x1 > ox + 8u * qx;
  uint32_t m = 0;
#pragma unroll
  for (uint32_t qy = 0; qy < (uint32_t)(TH / SBH); qy++) {
    const bool row = y0 < oy + (uint32_t)SBH * qy + (uint32_t)SBH && y1 > oy + (uint32_t)SBH * qy;
#pragma unroll
    for (int qx = 0; qx < WX; qx++)
      if (row && col[qx]) m |= 1u << (qy * WX + qx);
  }
  return m;
}

// 32x32 bit-matrix transpose across a warp: lane j holds row j on entry; on return lane L
// holds column L (bit j of the result = bit L of lane j's input). Five exchange stages,
// each swapping the off-diagonal blocks of size s.
__device__ __forceinline__ uint32_t warp_transpose_bits(uint32_t x) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t masks[5] = {0x0000ffffu, 0x00ff00ffu, 0x0f0f0f0fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int i = 0; i < 5; i++) {
    const uint32_t sh = 16u >> i, m = masks[i];
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, sh);
    x = (lane & sh) ? ((x & ~m) | ((y & ~m) >> sh)) : ((x & m) | ((y & m) << sh));
  }
  return x;
}

// Compacts, in order, the chunk-local indices k < cnt whose mask has this warp's bit (and,
// when `limit` is finite, k < limit) into list[]; returns how many.
template <typename WM>
__device__ __forceinline__ uint32_t build_warp_list(const WM* __restrict__ smask, uint32_t cnt, uint32_t limit,
                                                    uint8_t* __restrict__ list) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t n = 0;
  for (uint32_t b = 0; b < cnt; b += 32) {
    const uint32_t k = b + lane;
    const bool hit = k < cnt && k < limit && ((smask[k] >> warp) & 1u);
    const uint32_t bal = __ballot_sync(0xffffffffu, hit);
    if (hit) list[n + __popc(bal & lt)] = (uint8_t)k;
    n += __popc(bal);
  }
  __syncwarp();
  return n;
}

// forward_tile (rasterize.rs:249-302) for one tile per block. Each warp walks, 32 at a
// time, the chunk's entries whose pixel rectangle touches its 8x4 sub-block; a lane takes
// only the entries whose rectangle covers its own pixel (the rectangle test of the
// reference), found from the batch's coverage masks transposed across the warp, so the
// warp runs as many rounds as its busiest lane rather than one round per entry. Each lane
// still composites its entries in list (depth) order. kCount adds the evaluated-pair counter
// (untimed diagnostics only).
template <int TW, int TH, int CH, bool kCount>
__global__ void __launch_bounds__(TW * TH, 1536 / (TW * TH)) raster_fwd_kernel(
    const float4* __restrict__ rec, const uint32_t* __restrict__ gauss, const uint2* __restrict__ ranges,
    uint32_t width, uint32_t height, uint32_t tiles_x, float bg0, float bg1, float bg2, float* __restrict__ image,
    float* __restrict__ final_t, uint32_t* __restrict__ n_contrib, unsigned long long* __restrict__ pairs,
    const BatchTable* __restrict__ bt) {
  typedef TileGeo<TW, TH> Geo;
  constexpr int NT = Geo::kThreads;
  if (bt && blockIdx.x >= bt->tile_start[bt->views]) return;  // past the batch's tiles
  __shared__ float4 s0[CH], s1[CH];
  __shared__ float2 s2[CH];
  __shared__ typename Geo::Mask srect[CH];
  __shared__ typename Geo::WarpMask smask[CH];
  __shared__ uint8_t slist[Geo::kWarps][CH];
  __shared__ double stab[crm::kExpNegEntries];
  for (int i = threadIdx.x; i < crm::kExpNegEntries; i += NT) stab[i] = crm::exp2_neg_entry(i, kExp2Tab64);
  // In a batch the block is a global tile: find its view, local tile and image offset.
  uint32_t tile = blockIdx.x;
  size_t pix0 = 0;
  if (bt) {
    const int v = batch_view_of(bt->tile_start, bt->views, blockIdx.x);
    tile = blockIdx.x - bt->tile_start[v];
    width = bt->cam[v].width;
    height = bt->cam[v].height;
    tiles_x = bt->tiles_x[v];
    pix0 = bt->pix_start[v];
  }
  const PixelGeom pg = pixel_geom<TW, TH>(tile, tiles_x, width, height);
  const uint32_t ox = (tile % tiles_x) * TW, oy = (tile / tiles_x) * TH;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Sub-block origin in the tile; its rows' bits in the rectangle masks.
  const uint32_t sbx = (warp % Geo::kWarpsX) * 8u, sby = (warp / Geo::kWarpsX) * 4u + Geo::kRowShift;
  const float px = (float)pg.px_i + 0.5f, py = (float)pg.py_j + 0.5f;
  const uint2 range = ranges[blockIdx.x];
  uint8_t* list = slist[warp];
  float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
  uint32_t ncon = 0;
  bool done = !pg.inside;
  unsigned long long npairs = 0;
  for (uint32_t base = range.x; base < range.y; base += CH) {
    if (__syncthreads_count(!done) == 0) break;
#pragma unroll
    for (uint32_t e = threadIdx.x; e < (uint32_t)CH; e += NT) {
      const uint32_t idx = base + e;
      uint32_t m = 0;
      if (idx < range.y) {
        const uint32_t g = gauss[idx];
        s0[e] = rec[4 * (size_t)g];
        s1[e] = rec[4 * (size_t)g + 1];
        const float4 e2 = rec[4 * (size_t)g + 2];
        s2[e] = make_float2(e2.x, e2.y);
        srect[e] = tile_rect_masks<TW, TH>(fbits(e2.z), fbits(e2.w), ox, oy);
        m = subblock_mask<TW, TH>(fbits(e2.z), fbits(e2.w), ox, oy);
      }
      smask[e] = (typename Geo::WarpMask)m;
    }
    __syncthreads();
    const uint32_t cnt = min((uint32_t)CH, range.y - base);
    const uint32_t nl = build_warp_list(smask, cnt, 0xffffffffu, list);
    for (uint32_t b0 = 0; b0 < nl; b0 += 32) {
      if (__all_sync(0xffffffffu, done)) break;
      // Lane j loads entry j of the batch and expands its rectangle to a 32-bit mask of the
      // sub-block's pixels (bit 8 * row + column); the transpose gives each lane the mask of
      // the batch entries that cover its pixel.
      const uint32_t j = b0 + lane;
      uint32_t kl = 0, cov = 0;
      if (j < nl) {
        kl = list[j];
        const typename Geo::Mask rm = srect[kl];
        const uint32_t c8 = (uint32_t)(rm >> sbx) & 0xffu;
        const uint32_t r4 = (uint32_t)(rm >> sby) & 0xfu;
        cov = c8 * ((r4 & 1u) | ((r4 & 2u) << 7) | ((r4 & 4u) << 14) | ((r4 & 8u) << 21));
      }
      uint32_t mine = warp_transpose_bits(cov);
      if (done) mine = 0;
      while (__any_sync(0xffffffffu, mine != 0u)) {
        const uint32_t k = __shfl_sync(0xffffffffu, kl, (__ffs(mine) - 1) & 31);
        if (mine == 0u) continue;
        mine &= mine - 1u;
        if (kCount) npairs++;
        const float4 e0 = s0[k], e1 = s1[k];
        const float2 e2 = s2[k];
        float gval, alpha;
        if (!evaluate(px, py, e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, stab, &gval, &alpha)) continue;
        const float test_t = T * (1.0f - alpha);
        if (test_t < SPLAT_T_MIN) {
          done = true;
          mine = 0;
          continue;
        }
        const float at = alpha * T;
        cr += at * e1.w;
        cg += at * e2.x;
        cb += at * e2.y;
        T = test_t;
        ncon = base - range.x + k + 1;
      }
    }
    __syncthreads();
  }
  if (pg.inside) {
    const size_t pix = pix0 + (size_t)pg.py_j * width + pg.px_i;
    image[3 * pix] = cr + T * bg0;
    image[3 * pix + 1] = cg + T * bg1;
    image[3 * pix + 2] = cb + T * bg2;
    final_t[pix] = T;
    n_contrib[pix] = ncon;
  }
  if (kCount) {
    for (int o = 16; o > 0; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    if (lane == 0 && npairs) atomicAdd(pairs, npairs);
  }
}

// backward_tile (rasterize.rs:354-455) for one tile per block. Per-pixel contributions to
// an entry's 11 gradient slots are summed across the warp by a transposing butterfly
// (13 shuffles leave each slot's warp total in a pair of lanes), across the block's warps
// with one shared-memory atomic instruction per warp, and across tiles with three float4
// vector atomics per entry.
// Slots per entry: ProjGrad (9), the AbsGS accumulators (2) and the entry's blending weight
// sum(alpha * T) over the tile's pixels (the trainer's contribution statistic).
constexpr int kSlots = 12;

// v[0..11] per lane in; out, the warp total of slot 6*b4 + 3*b3 + 2*b2 + b1 (b_i = bit i of
// the lane) when 2*b2 + b1 < 3, in both lanes of a pair. Each exchange stage keeps the half
// of the values selected by the lane's bit and adds the partner's copy of that half:
// 6 + 3 + 2 + 1 + 1 = 13 shuffles for 12 slots.
__device__ __forceinline__ float warp_transpose_reduce12(const float v[12]) {
  const uint32_t lane = threadIdx.x & 31;
  const bool b4 = lane & 16u, b3 = lane & 8u, b2 = lane & 4u, b1 = lane & 2u;
  float w[6], x[4], y[2];
#pragma unroll
  for (int i = 0; i < 6; i++) {
    const float send = b4 ? v[i] : v[i + 6];
    const float keep = b4 ? v[i + 6] : v[i];
    w[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const float send = b3 ? w[i] : w[i + 3];
    const float keep = b3 ? w[i + 3] : w[i];
    x[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  x[3] = 0.0f;
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const float send = b2 ? x[i] : x[i + 2];
    const float keep = b2 ? x[i + 2] : x[i];
    y[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  const float send = b1 ? y[0] : y[1];
  const float keep = b1 ? y[1] : y[0];
  float z = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  return z;
}

// 1 / x for x in [0.01, 1] by the special-function unit alone (relative error within a few
// ulps; values only, never a decision). Over a pixel's reverse walk the recovered
// transmittance then carries at most about one ulp per entry walked, far inside the
// gradients' 1e-3 bar.
__device__ __forceinline__ float rcp_fast(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// PPL pixels per thread in scalar arithmetic: a warp owns an 8 x (4 PPL) sub-block, lane L
// the pixels (L % 8, L / 8 + 4 q) of it for q < PPL. It is launched with one pixel per
// thread (64 registers, 32 warps per SM); two pixels per thread run as pairs in
// raster_bwd_x2_kernel below, which replaced this kernel's PPL = 2 form (1.24-1.27 ms
// against 0.91 ms on the render benchmark).
template <int TW, int TH, int CH, int PPL>
__global__ void __launch_bounds__(TW * TH / PPL, (PPL == 1 ? 1024 : 768) / (TW * TH / PPL)) raster_bwd_kernel(
    const float4* __restrict__ rec, const uint32_t* __restrict__ gauss, const uint2* __restrict__ ranges,
    uint32_t width, uint32_t height, uint32_t tiles_x, float bg0, float bg1, float bg2,
    const float* __restrict__ final_t, const uint32_t* __restrict__ n_contrib, const float* __restrict__ dimage,
    float4* __restrict__ pgrad, int64_t cap, unsigned long long* __restrict__ pairs,
    const BatchTable* __restrict__ bt) {
  typedef TileGeo<TW, TH> Geo;
  constexpr int NT = TW * TH / PPL, NW = NT / 32, WX = TW / 8, SBH = 4 * PPL;
  typedef typename std::conditional<(NW > 8), uint16_t, uint8_t>::type WarpMask;
  if (bt && blockIdx.x >= bt->tile_start[bt->views]) return;  // past the batch's tiles
  __shared__ float4 s0[CH], s1[CH];
  __shared__ float2 s2[CH];
  __shared__ typename Geo::Mask srect[CH];
  __shared__ uint32_t sg[CH];
  __shared__ float acc[CH * kSlots];
  __shared__ WarpMask smask[CH];
  __shared__ uint8_t slist[NW][CH];
  __shared__ uint32_t s_max_last;
  // In a batch the block is a global tile: find its view, local tile and image offset.
  uint32_t tile = blockIdx.x;
  size_t pix0 = 0;
  if (bt) {
    const int v = batch_view_of(bt->tile_start, bt->views, blockIdx.x);
    tile = blockIdx.x - bt->tile_start[v];
    width = bt->cam[v].width;
    height = bt->cam[v].height;
    tiles_x = bt->tiles_x[v];
    pix0 = bt->pix_start[v];
  }
  const uint32_t ox = (tile % tiles_x) * TW, oy = (tile / tiles_x) * TH;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lx = (warp % WX) * 8u + (lane & 7u);        // column in the tile
  const uint32_t ly0 = (warp / WX) * (uint32_t)SBH + (lane >> 3);  // row of pixel 0 in the tile
  const float px = (float)(ox + lx) + 0.5f;
  const uint2 range = ranges[blockIdx.x];
  uint8_t* list = slist[warp];
  const uint32_t list_len = range.y - range.x;

  // Per pixel: contributor count, transmittance, dL/dpixel and the running sums of the
  // reverse walk (rasterize.rs:347-455).
  uint32_t last[PPL];
  // nbg = -T_final (bg . dL/dpixel): the background's share of dL/dalpha is nbg / (1 - alpha).
  float T[PPL], nbg[PPL], d0[PPL], d1[PPL], d2[PPL], py[PPL];
  float acc_r[PPL], acc_g[PPL], acc_b[PPL], last_alpha[PPL], lc_r[PPL], lc_g[PPL], lc_b[PPL];
  uint32_t lane_last = 0;
#pragma unroll
  for (int q = 0; q < PPL; q++) {
    const uint32_t y = oy + ly0 + 4u * q, x = ox + lx;
    py[q] = (float)y + 0.5f;
    last[q] = 0;
    T[q] = 1.0f;
    d0[q] = d1[q] = d2[q] = nbg[q] = 0.0f;
    if (x < width && y < height) {
      const size_t pix = pix0 + (size_t)y * width + x;
      last[q] = min(n_contrib[pix], list_len);  // n_contrib never exceeds its tile's list
      T[q] = final_t[pix];
      d0[q] = dimage[3 * pix];
      d1[q] = dimage[3 * pix + 1];
      d2[q] = dimage[3 * pix + 2];
      nbg[q] = -T[q] * (bg0 * d0[q] + bg1 * d1[q] + bg2 * d2[q]);
    }
    acc_r[q] = acc_g[q] = acc_b[q] = 0.0f;  // accum (rasterize.rs:347)
    last_alpha[q] = lc_r[q] = lc_g[q] = lc_b[q] = 0.0f;
    lane_last = max(lane_last, last[q]);
  }
  if (threadIdx.x == 0) s_max_last = 0;
  for (int i = threadIdx.x; i < CH * kSlots; i += NT) acc[i] = 0.0f;
  __syncthreads();
  const uint32_t warp_max_last = __reduce_max_sync(0xffffffffu, lane_last);
  if (lane == 0) atomicMax(&s_max_last, warp_max_last);
  __syncthreads();
  const uint32_t max_last = s_max_last;
  uint32_t npairs = 0;

  for (uint32_t cend = max_last; cend > 0;) {
    const uint32_t cstart = cend > (uint32_t)CH ? cend - CH : 0u;
    const uint32_t cnt = cend - cstart;
#pragma unroll
    for (uint32_t e = threadIdx.x; e < (uint32_t)CH; e += NT) {
      uint32_t m = 0;
      if (e < cnt) {
        const uint32_t g = gauss[range.x + cstart + e];
        sg[e] = g;
        s0[e] = rec[4 * (size_t)g];
        s1[e] = rec[4 * (size_t)g + 1];
        const float4 e2 = rec[4 * (size_t)g + 2];
        s2[e] = make_float2(e2.x, e2.y);
        srect[e] = tile_rect_masks<TW, TH>(fbits(e2.z), fbits(e2.w), ox, oy);
        m = subblock_mask<TW, TH, SBH>(fbits(e2.z), fbits(e2.w), ox, oy);
      }
      smask[e] = (WarpMask)m;
    }
    __syncthreads();
    // Entries at or past every lane's n_contrib contribute nothing to this warp.
    const uint32_t limit = warp_max_last > cstart ? warp_max_last - cstart : 0u;
    const uint32_t nl = build_warp_list(smask, cnt, limit, list);
    for (int i = (int)nl - 1; i >= 0; i--) {
      const uint32_t kk = list[i];
      const uint32_t k = cstart + kk;
      const typename Geo::Mask rm = srect[kk];
      float c[kSlots];
#pragma unroll
      for (int q = 0; q < kSlots; q++) c[q] = 0.0f;
      bool active = false;
      const bool col_in = (uint32_t)(rm >> lx) & 1u;
#pragma unroll
      for (int q = 0; q < PPL; q++) {
        if (!(col_in && k < last[q] && ((uint32_t)(rm >> (ly0 + 4u * q + Geo::kRowShift)) & 1u))) continue;
        const float2 e2 = s2[kk];
        npairs++;
        const float4 e0 = s0[kk], e1 = s1[kk];
        float gval, alpha;
        bool unclamped;
        if (!evaluate_bwd(px, py[q], e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, &gval, &alpha, &unclamped)) continue;
        active = true;
        // Values only from here on: the arithmetic is fused and the divisions are
        // reciprocals; every decision was taken above exactly as in the forward pass.
        const float col_r = e1.w, col_g = e2.x, col_b = e2.y;
        const float inv = rcp_fast(1.0f - alpha);
        T[q] = T[q] * inv;
        const float t = T[q];
        const float keep = 1.0f - last_alpha[q];
        acc_r[q] = __fmaf_rn(last_alpha[q], lc_r[q], keep * acc_r[q]);
        acc_g[q] = __fmaf_rn(last_alpha[q], lc_g[q], keep * acc_g[q]);
        acc_b[q] = __fmaf_rn(last_alpha[q], lc_b[q], keep * acc_b[q]);
        float dalpha = (col_r - acc_r[q]) * d0[q];
        dalpha = __fmaf_rn(col_g - acc_g[q], d1[q], dalpha);
        dalpha = __fmaf_rn(col_b - acc_b[q], d2[q], dalpha);
        const float at = alpha * t;
        c[6] = __fmaf_rn(at, d0[q], c[6]);
        c[7] = __fmaf_rn(at, d1[q], c[7]);
        c[8] = __fmaf_rn(at, d2[q], c[8]);
        c[11] += at;
        lc_r[q] = col_r;
        lc_g[q] = col_g;
        lc_b[q] = col_b;
        last_alpha[q] = alpha;
        dalpha = __fmaf_rn(dalpha, t, nbg[q] * inv);
        if (unclamped) {
          const float opacity = e1.y;
          c[5] = __fmaf_rn(gval, dalpha, c[5]);
          const float dsigma = -(opacity * dalpha) * gval;
          const float dx = px - e0.x;
          const float dy = py[q] - e0.y;
          const float ddx = dsigma * __fmaf_rn(e0.z, dx, e0.w * dy);
          const float ddy = dsigma * __fmaf_rn(e0.w, dx, e1.x * dy);
          c[0] -= ddx;
          c[1] -= ddy;
          const float hs = 0.5f * dsigma;
          c[2] = __fmaf_rn(hs * dx, dx, c[2]);
          c[3] = __fmaf_rn(dsigma * dx, dy, c[3]);
          c[4] = __fmaf_rn(hs * dy, dy, c[4]);
          c[9] += fabsf(ddx);
          c[10] += fabsf(ddy);
        }
      }
      if (__any_sync(0xffffffffu, active)) {
        const float tot = warp_transpose_reduce12(c);
        const uint32_t local = (lane >> 1) & 3u;
        const uint32_t slot = 6u * ((lane >> 4) & 1u) + 3u * ((lane >> 3) & 1u) + local;
        if (!(lane & 1u) && local < 3u) atomicAdd(&acc[kk * kSlots + slot], tot);
      }
    }
    __syncthreads();
#pragma unroll
    for (uint32_t e = threadIdx.x; e < (uint32_t)CH; e += NT) {
      if (e >= cnt) break;
      float* a = &acc[e * kSlots];
      const size_t g = sg[e];
      const float4 v0 = make_float4(a[0], a[1], a[2], a[3]);
      const float4 v1 = make_float4(a[4], a[5], a[6], a[7]);
      const float4 v2 = make_float4(a[8], a[9], a[10], a[11]);
      if (v0.x != 0.0f || v0.y != 0.0f || v0.z != 0.0f || v0.w != 0.0f) atomicAdd(&pgrad[g], v0);
      if (v1.x != 0.0f || v1.y != 0.0f || v1.z != 0.0f || v1.w != 0.0f) atomicAdd(&pgrad[cap + g], v1);
      if (v2.x != 0.0f || v2.y != 0.0f || v2.z != 0.0f || v2.w != 0.0f) atomicAdd(&pgrad[2 * cap + g], v2);
#pragma unroll
      for (int q = 0; q < kSlots; q++) a[q] = 0.0f;
    }
    __syncthreads();
    cend = cstart;
  }
  if (pairs) {
    unsigned long long np = npairs;
    for (int o = 16; o > 0; o >>= 1) np += __shfl_xor_sync(0xffffffffu, np, o);
    if (lane == 0 && np) atomicAdd(pairs, np);
  }
}

// Backward decisions without the exp. The reference skips a pixel when sigma < 0, sigma >
// sigma_max or fl(opacity * exp(-sigma)) < 1/255 (rasterize.rs:231-244), with sigma_max =
// ln(opacity * 255) (both correctly rounded). fl(opacity * exp(-sigma)) does not increase
// with sigma, and for sigma <= sigma_max - kSigmaEdge it is at least
// (1/255) e^(kSigmaEdge - 7.2e-7) (1 - 2^-23) > 1/255 (the roundings of the quotient, the
// logarithm, the difference, the exp and the product, with ln(255 opacity) <= ln 255), so
// such a pixel passes the alpha test whatever the exp's value: the decision needs sigma
// only. Pixels within kSigmaEdge of sigma_max take the correctly rounded exp. Likewise
// fl(opacity * exp(-sigma)) <= opacity, so an entry with opacity < 0.99 never clamps.
constexpr float kSigmaEdge = 1e-4f;

// The backward with two pixels per thread computed as pairs. Lane L owns the pixels
// (L % 8, L / 8) and (L % 8, L / 8 + 4) of its warp's 8x8 sub-block; every per-pixel value of
// backward_tile (rasterize.rs:394-454) is a pair, computed with the paired instructions of
// pair.cuh, and an entry's record is staged in shared memory with each scalar duplicated
// into both halves so that it is an operand as it stands. Decisions are taken on the
// halves: sigma (bit-identical to the scalar sigma) against the entry's range, as above.
// A pixel the entry does not reach (outside the rectangle, at or past n_contrib, skipped by
// a decision) runs the arithmetic with sigma = +inf, so gauss = alpha = 0: its
// transmittance is multiplied by rcp(1) = 1 exactly, its colour accumulator by 0 + 1, and
// all its contributions are exactly zero; both pixels of a pair always run together and
// still leave the scalar kernel's state and sums. The colour accumulator is advanced right
// after its use (accum + alpha (c - accum)) instead of on the pixel's next entry, which
// needs the same operands and so leaves neither last_alpha nor last_color to carry. A
// lane's two contributions to each slot are added before the warp reduction. kCount adds
// the evaluated-pair counter (untimed diagnostics only).
template <int TW, int TH, int CH, bool kCount>
__global__ void __launch_bounds__(TW * TH / 2, 768 / (TW * TH / 2)) raster_bwd_x2_kernel(
    const float4* __restrict__ rec, const uint32_t* __restrict__ gauss, const uint2* __restrict__ ranges,
    uint32_t width, uint32_t height, uint32_t tiles_x, float bg0, float bg1, float bg2,
    const float* __restrict__ final_t, const uint32_t* __restrict__ n_contrib, const float* __restrict__ dimage,
    float4* __restrict__ pgrad, int64_t cap, unsigned long long* __restrict__ pairs,
    const BatchTable* __restrict__ bt) {
  typedef TileGeo<TW, TH> Geo;
  typedef typename Geo::Mask Mask;
  constexpr int NT = TW * TH / 2, NW = NT / 32, WX = TW / 8, SBH = 8;
  typedef typename std::conditional<(NW > 8), uint16_t, uint8_t>::type WarpMask;
  if (bt && blockIdx.x >= bt->tile_start[bt->views]) return;  // past the batch's tiles
  // Per entry, duplicated: (mx, mx, my, my), (A, A, B, B), (C, C, opacity, opacity),
  // (r, r, g, g), (b, b); and (sigma_max, sigma_max - kSigmaEdge).
  __shared__ float4 sxy[CH], sab[CH], sco[CH], srg[CH];
  __shared__ float2 sb[CH], ssig[CH];
  __shared__ Mask srect[CH];
  __shared__ uint32_t sg[CH];
  __shared__ float acc[CH * kSlots];
  __shared__ WarpMask smask[CH];
  __shared__ uint8_t slist[NW][CH];
  __shared__ uint32_t s_max_last;
  uint32_t tile = blockIdx.x;
  size_t pix0 = 0;
  if (bt) {
    const int v = batch_view_of(bt->tile_start, bt->views, blockIdx.x);
    tile = blockIdx.x - bt->tile_start[v];
    width = bt->cam[v].width;
    height = bt->cam[v].height;
    tiles_x = bt->tiles_x[v];
    pix0 = bt->pix_start[v];
  }
  const uint32_t ox = (tile % tiles_x) * TW, oy = (tile / tiles_x) * TH;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lx = (warp % WX) * 8u + (lane & 7u);
  const uint32_t ly0 = (warp / WX) * (uint32_t)SBH + (lane >> 3);
  // A pixel is in an entry's rectangle when both its column and its row bit are set.
  const Mask bits0 = ((Mask)1 << lx) | ((Mask)1 << (ly0 + Geo::kRowShift));
  const Mask bits1 = ((Mask)1 << lx) | ((Mask)1 << (ly0 + 4u + Geo::kRowShift));
  const uint2 range = ranges[blockIdx.x];
  uint8_t* list = slist[warp];
  const uint32_t list_len = range.y - range.x;

  // Per pixel pair: pixel centres, contributor counts, transmittance, dL/dpixel, the
  // background's share of dL/dalpha (times 1 - alpha) and the colour accumulator.
  const float pxf = (float)(ox + lx) + 0.5f;
  const f2 px = f2_splat(pxf);
  const f2 py = f2_make((float)(oy + ly0) + 0.5f, (float)(oy + ly0 + 4u) + 0.5f);
  uint32_t last[2];
  float Tq[2], nbgq[2], d0q[2], d1q[2], d2q[2];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const uint32_t y = oy + ly0 + 4u * q, x = ox + lx;
    last[q] = 0;
    Tq[q] = 1.0f;
    d0q[q] = d1q[q] = d2q[q] = nbgq[q] = 0.0f;
    if (x < width && y < height) {
      const size_t pix = pix0 + (size_t)y * width + x;
      last[q] = min(n_contrib[pix], list_len);
      Tq[q] = final_t[pix];
      d0q[q] = dimage[3 * pix];
      d1q[q] = dimage[3 * pix + 1];
      d2q[q] = dimage[3 * pix + 2];
      nbgq[q] = -Tq[q] * (bg0 * d0q[q] + bg1 * d1q[q] + bg2 * d2q[q]);
    }
  }
  f2 T = f2_make(Tq[0], Tq[1]);
  const f2 nbg = f2_make(nbgq[0], nbgq[1]);
  const f2 d0 = f2_make(d0q[0], d0q[1]), d1 = f2_make(d1q[0], d1q[1]), d2 = f2_make(d2q[0], d2q[1]);
  f2 acc_r = f2_splat(0.0f), acc_g = acc_r, acc_b = acc_r;
  const f2 half = f2_splat(0.5f), one = f2_splat(1.0f), nlog2e = f2_splat(-kLog2e);
  const uint32_t lane_last = max(last[0], last[1]);

  if (threadIdx.x == 0) s_max_last = 0;
  for (int i = threadIdx.x; i < CH * kSlots; i += NT) acc[i] = 0.0f;
  __syncthreads();
  const uint32_t warp_max_last = __reduce_max_sync(0xffffffffu, lane_last);
  if (lane == 0) atomicMax(&s_max_last, warp_max_last);
  __syncthreads();
  const uint32_t max_last = s_max_last;
  uint32_t npairs = 0;

  for (uint32_t cend = max_last; cend > 0;) {
    const uint32_t cstart = cend > (uint32_t)CH ? cend - CH : 0u;
    const uint32_t cnt = cend - cstart;
#pragma unroll
    for (uint32_t e = threadIdx.x; e < (uint32_t)CH; e += NT) {
      uint32_t m = 0;
      if (e < cnt) {
        const uint32_t g = gauss[range.x + cstart + e];
        sg[e] = g;
        const float4 r0 = rec[4 * (size_t)g], r1 = rec[4 * (size_t)g + 1], r2 = rec[4 * (size_t)g + 2];
        sxy[e] = make_float4(r0.x, r0.x, r0.y, r0.y);
        sab[e] = make_float4(r0.z, r0.z, r0.w, r0.w);
        sco[e] = make_float4(r1.x, r1.x, r1.y, r1.y);
        srg[e] = make_float4(r1.w, r1.w, r2.x, r2.x);
        sb[e] = make_float2(r2.y, r2.y);
        ssig[e] = make_float2(r1.z, r1.z - kSigmaEdge);
        srect[e] = tile_rect_masks<TW, TH>(fbits(r2.z), fbits(r2.w), ox, oy);
        m = subblock_mask<TW, TH, SBH>(fbits(r2.z), fbits(r2.w), ox, oy);
      }
      smask[e] = (WarpMask)m;
    }
    __syncthreads();
    const uint32_t limit = warp_max_last > cstart ? warp_max_last - cstart : 0u;
    const uint32_t nl = build_warp_list(smask, cnt, limit, list);
    for (int i = (int)nl - 1; i >= 0; i--) {
      const uint32_t kk = list[i];
      const uint32_t k = cstart + kk;
      const Mask rm = srect[kk];
      const bool cov0 = (rm & bits0) == bits0 && k < last[0];
      const bool cov1 = (rm & bits1) == bits1 && k < last[1];
      if (kCount) npairs += (uint32_t)cov0 + (uint32_t)cov1;
      const float4 exy = sxy[kk], eab = sab[kk], eco = sco[kk], erg = srg[kk];
      const float2 eb = sb[kk], esig = ssig[kk];
      const f2 mx = f2_make(exy.x, exy.y), my = f2_make(exy.z, exy.w);
      const f2 A = f2_make(eab.x, eab.y), B = f2_make(eab.z, eab.w);
      const f2 Cc = f2_make(eco.x, eco.y), op = f2_make(eco.z, eco.w);
      const f2 dx = f2_sub(px, mx), dy = f2_sub(py, my);
      f2 adx, cdy, bdx;
      const f2 sigma = paired_sigma(A, B, Cc, dx, dy, &adx, &cdy, &bdx);
      float s0, s1;
      f2_split(sigma, s0, s1);
      // The reference's range test (false for NaN, as there), then the alpha test by sigma.
      const bool in0 = cov0 && !(s0 < 0.0f) && !(s0 > esig.x);
      const bool in1 = cov1 && !(s1 < 0.0f) && !(s1 > esig.x);
      bool v0 = in0 && s0 <= esig.y, v1 = in1 && s1 <= esig.y;
      const bool edge0 = in0 && !v0, edge1 = in1 && !v1;
      if (__any_sync(0xffffffffu, edge0 || edge1)) {  // rare: the correctly rounded exp decides
        if (edge0) v0 = !(eco.z * crm::expf_cr(-s0) < SPLAT_ALPHA_MIN);
        if (edge1) v1 = !(eco.w * crm::expf_cr(-s1) < SPLAT_ALPHA_MIN);
      }
      // No pixel of the warp takes the entry: every update below would be an identity.
      if (!__any_sync(0xffffffffu, v0 || v1)) continue;
      const float inf = __int_as_float(0x7f800000);
      float g0, g1;
      f2_split(f2_mul(f2_make(v0 ? s0 : inf, v1 ? s1 : inf), nlog2e), g0, g1);
      f2 gv = f2_make(ex2_approx(g0), ex2_approx(g1));  // gauss (fast exp), 0 where skipped
      f2 alpha = f2_mul(op, gv);
      if (!(eco.z < SPLAT_ALPHA_MAX)) {
        // Opacity >= 0.99 (uniform over the warp): alpha clamps at 0.99 and the gradients
        // through sigma and opacity vanish there (rasterize.rs:414-432). Products within a
        // relative band of the clamp are decided with the correctly rounded exp.
        float a0, a1, q0, q1;
        f2_split(alpha, a0, a1);
        f2_split(gv, q0, q1);
        if (fabsf(a0 - SPLAT_ALPHA_MAX) < SPLAT_ALPHA_MAX * kExpBand) {
          q0 = crm::expf_cr(-s0);
          a0 = eco.z * q0;
        }
        if (fabsf(a1 - SPLAT_ALPHA_MAX) < SPLAT_ALPHA_MAX * kExpBand) {
          q1 = crm::expf_cr(-s1);
          a1 = eco.w * q1;
        }
        gv = f2_make(a0 < SPLAT_ALPHA_MAX ? q0 : 0.0f, a1 < SPLAT_ALPHA_MAX ? q1 : 0.0f);
        alpha = f2_make(fminf(a0, SPLAT_ALPHA_MAX), fminf(a1, SPLAT_ALPHA_MAX));
      }
      // Values only from here on (fused, reciprocal for division).
      float o0, o1;
      f2_split(f2_sub(one, alpha), o0, o1);
      const f2 inv = f2_make(rcp_fast(o0), rcp_fast(o1));
      T = f2_mul(T, inv);
      const f2 dr = f2_sub(f2_make(erg.x, erg.y), acc_r);
      const f2 dg = f2_sub(f2_make(erg.z, erg.w), acc_g);
      const f2 db = f2_sub(f2_make(eb.x, eb.y), acc_b);
      f2 dalpha = f2_fma(db, d2, f2_fma(dg, d1, f2_mul(dr, d0)));
      const f2 at = f2_mul(alpha, T);
      acc_r = f2_fma(alpha, dr, acc_r);
      acc_g = f2_fma(alpha, dg, acc_g);
      acc_b = f2_fma(alpha, db, acc_b);
      dalpha = f2_fma(dalpha, T, f2_mul(nbg, inv));
      const f2 c5 = f2_mul(gv, dalpha);
      // nds = opacity dalpha gauss = -dsigma; the signs are applied in the lane sums below.
      const f2 nds = f2_mul(f2_mul(op, dalpha), gv);
      const f2 ndx = f2_mul(nds, f2_fma(B, dy, adx));  // -ddx = -dsigma (A dx + B dy)
      const f2 ndy = f2_mul(nds, f2_add(bdx, cdy));    // -ddy = -dsigma (B dx + C dy)
      const f2 hs = f2_mul(half, nds);
      const f2 c2 = f2_mul(f2_mul(hs, dx), dx);
      const f2 c3 = f2_mul(f2_mul(nds, dx), dy);
      const f2 c4 = f2_mul(f2_mul(hs, dy), dy);
      const f2 c6 = f2_mul(at, d0), c7 = f2_mul(at, d1), c8 = f2_mul(at, d2);
      float c[kSlots], lo, hi;
      f2_split(ndx, lo, hi);
      c[0] = lo + hi;
      c[9] = fabsf(lo) + fabsf(hi);
      f2_split(ndy, lo, hi);
      c[1] = lo + hi;
      c[10] = fabsf(lo) + fabsf(hi);
      f2_split(c2, lo, hi);
      c[2] = -lo - hi;
      f2_split(c3, lo, hi);
      c[3] = -lo - hi;
      f2_split(c4, lo, hi);
      c[4] = -lo - hi;
      f2_split(c5, lo, hi);
      c[5] = lo + hi;
      f2_split(c6, lo, hi);
      c[6] = lo + hi;
      f2_split(c7, lo, hi);
      c[7] = lo + hi;
      f2_split(c8, lo, hi);
      c[8] = lo + hi;
      f2_split(at, lo, hi);
      c[11] = lo + hi;
      const float tot = warp_transpose_reduce12(c);
      const uint32_t local = (lane >> 1) & 3u;
      const uint32_t slot = 6u * ((lane >> 4) & 1u) + 3u * ((lane >> 3) & 1u) + local;
      if (!(lane & 1u) && local < 3u) atomicAdd(&acc[kk * kSlots + slot], tot);
    }
    __syncthreads();
#pragma unroll
    for (uint32_t e = threadIdx.x; e < (uint32_t)CH; e += NT) {
      if (e >= cnt) break;
      float* a = &acc[e * kSlots];
      const size_t g = sg[e];
      const float4 v0 = make_float4(a[0], a[1], a[2], a[3]);
      const float4 v1 = make_float4(a[4], a[5], a[6], a[7]);
      const float4 v2 = make_float4(a[8], a[9], a[10], a[11]);
      if (v0.x != 0.0f || v0.y != 0.0f || v0.z != 0.0f || v0.w != 0.0f) atomicAdd(&pgrad[g], v0);
      if (v1.x != 0.0f || v1.y != 0.0f || v1.z != 0.0f || v1.w != 0.0f) atomicAdd(&pgrad[cap + g], v1);
      if (v2.x != 0.0f || v2.y != 0.0f || v2.z != 0.0f || v2.w != 0.0f) atomicAdd(&pgrad[2 * cap + g], v2);
#pragma unroll
      for (int q = 0; q < kSlots; q++) a[q] = 0.0f;
    }
    __syncthreads();
    cend = cstart;
  }
  if (kCount) {
    unsigned long long np = npairs;
    for (int o = 16; o > 0; o >>= 1) np += __shfl_xor_sync(0xffffffffu, np, o);
    if (lane == 0 && np) atomicAdd(pairs, np);
  }
}

// ---------------------------------------------------------------------------------------
// Deterministic backward (16x16 tiles): the reference's own reduction, bit for bit.
//
// backward_tile (rasterize.rs:394-454) sums each entry's 11 slots over the pixels of its
// rectangle in row-major order, in unfused f32 arithmetic, and stores them per entry;
// rasterize_backward (:480-503) then sums every Gaussian's entries in entry order. Here a
// block walks its tile's list in reverse like the atomic kernel, but every pixel writes its
// per-entry contribution to shared memory (kDetGroup entries at a time) and one thread per
// (entry, slot) adds the contributions of the rectangle's pixels in row-major order; the
// per-entry sums go to a slot array indexed by the entry's emission index (Gaussian-major,
// rasterize.rs:76-97), which entry_slots_reduce_kernel sums per Gaussian. Pixels that do not
// contribute add +0.0, which leaves a sum unchanged (a sum that starts at +0.0 is never -0.0),
// so the totals equal the reference's, which skips them. The arithmetic per pixel is the
// reference's operation for operation: the correctly rounded exp of the forward, true
// divisions, no contraction (the file is compiled with --fmad=false), and dalpha built from
// 0.0 as the reference builds it.
// ---------------------------------------------------------------------------------------
constexpr int kDetGroup = 8;
constexpr int kDetChunk = 64;
constexpr size_t kDetSmemBytes = (size_t)kDetGroup * kSlots * 256 * sizeof(float);

// Emission index of the entry of Gaussian g in tile (tx, ty): its entries are emitted row by
// row over its tile rectangle (rasterize.rs:87-96).
__device__ __forceinline__ uint32_t entry_index(const float4* __restrict__ rec,
                                                const uint32_t* __restrict__ entry_offset, uint32_t g, uint32_t tx,
                                                uint32_t ty) {
  const float4 r3 = rec[4 * (size_t)g + 3];
  const uint32_t tmin = fbits(r3.z), tmax = fbits(r3.w);
  const uint32_t tx0 = tmin & 0xffffu, ty0 = tmin >> 16, w = (tmax & 0xffffu) - tx0;
  return entry_offset[g] + (ty - ty0) * w + (tx - tx0);
}

__global__ void __launch_bounds__(256) raster_bwd_det_kernel(
    const float4* __restrict__ rec, const uint32_t* __restrict__ gauss, const uint2* __restrict__ ranges,
    const uint32_t* __restrict__ entry_offset, int64_t e_cap, uint32_t width, uint32_t height, uint32_t tiles_x,
    float bg0, float bg1, float bg2, const float* __restrict__ final_t, const uint32_t* __restrict__ n_contrib,
    const float* __restrict__ dimage, float* __restrict__ eslot) {
  extern __shared__ float cbuf[];  // [kDetGroup][kSlots][256], pixel index row-major in the tile
  __shared__ float4 s0[kDetChunk], s1[kDetChunk];
  __shared__ float2 s2[kDetChunk];
  __shared__ uint32_t srect[kDetChunk];
  __shared__ uint32_t sent[kDetChunk];
  __shared__ uint32_t s_max_last;
  const uint32_t tile = blockIdx.x;
  const uint32_t tx = tile % tiles_x, ty = tile / tiles_x;
  const uint32_t ox = tx * 16u, oy = ty * 16u;
  const uint32_t lx = threadIdx.x & 15u, ly = threadIdx.x >> 4;
  const uint32_t x = ox + lx, y = oy + ly;
  const bool inside = x < width && y < height;
  const float px = (float)x + 0.5f, py = (float)y + 0.5f;
  const uint2 range = ranges[tile];
  const uint32_t list_len = range.y - range.x;
  // Clipped extent of the tile (tile_geom, rasterize.rs:203-215).
  const uint32_t gw = min(width - ox, 16u), gh = min(height - oy, 16u);

  uint32_t last = 0;
  float T = 1.0f, t_fin = 1.0f, d0 = 0.0f, d1 = 0.0f, d2 = 0.0f, bg_dot = 0.0f;
  if (inside) {
    const size_t pix = (size_t)y * width + x;
    last = min(n_contrib[pix], list_len);
    T = final_t[pix];
    t_fin = T;
    d0 = dimage[3 * pix];
    d1 = dimage[3 * pix + 1];
    d2 = dimage[3 * pix + 2];
    bg_dot = bg0 * d0 + bg1 * d1 + bg2 * d2;
  }
  float acc_r = 0.0f, acc_g = 0.0f, acc_b = 0.0f, last_alpha = 0.0f, lc_r = 0.0f, lc_g = 0.0f, lc_b = 0.0f;
  if (threadIdx.x == 0) s_max_last = 0;
  __syncthreads();
  const uint32_t wmax = __reduce_max_sync(0xffffffffu, last);
  if ((threadIdx.x & 31u) == 0) atomicMax(&s_max_last, wmax);
  __syncthreads();
  const uint32_t max_last = s_max_last;
  // Entries no pixel reaches keep zero slots.
  for (uint32_t k = max_last + threadIdx.x; k < list_len; k += 256) {
    const uint32_t e = entry_index(rec, entry_offset, gauss[range.x + k], tx, ty);
    if (e < e_cap) {
#pragma unroll
      for (int q = 0; q < kSlots; q++) eslot[(size_t)e * kSlots + q] = 0.0f;
    }
  }

  for (uint32_t cend = max_last; cend > 0;) {
    const uint32_t cstart = cend > (uint32_t)kDetChunk ? cend - kDetChunk : 0u;
    const uint32_t cnt = cend - cstart;
    for (uint32_t e = threadIdx.x; e < cnt; e += 256) {
      const uint32_t g = gauss[range.x + cstart + e];
      s0[e] = rec[4 * (size_t)g];
      s1[e] = rec[4 * (size_t)g + 1];
      const float4 e2 = rec[4 * (size_t)g + 2];
      s2[e] = make_float2(e2.x, e2.y);
      srect[e] = tile_rect_masks<16, 16>(fbits(e2.z), fbits(e2.w), ox, oy);
      sent[e] = entry_index(rec, entry_offset, g, tx, ty);
    }
    __syncthreads();
    for (uint32_t gend = cnt; gend > 0;) {
      const uint32_t gstart = gend > (uint32_t)kDetGroup ? gend - kDetGroup : 0u;
      // Each pixel's contributions to the group's entries, in reverse depth order.
      for (uint32_t kk = gend; kk-- > gstart;) {
        const uint32_t j = gend - 1u - kk;
        const uint32_t rm = srect[kk];
        if (!inside || !((rm >> lx) & 1u) || !((rm >> (16u + ly)) & 1u)) continue;  // outside the rectangle
        float c[kSlots];
#pragma unroll
        for (int q = 0; q < kSlots; q++) c[q] = 0.0f;
        const uint32_t k = cstart + kk;
        const float4 e0 = s0[kk], e1 = s1[kk];
        const float2 e2 = s2[kk];
        float gval, alpha;
        if (k < last && evaluate_ref(px, py, e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, &gval, &alpha)) {
          const float col_r = e1.w, col_g = e2.x, col_b = e2.y;
          T = T / (1.0f - alpha);
          const float t = T;
          float dalpha = 0.0f;
          acc_r = last_alpha * lc_r + (1.0f - last_alpha) * acc_r;
          dalpha += (col_r - acc_r) * d0;
          c[6] = alpha * t * d0;
          acc_g = last_alpha * lc_g + (1.0f - last_alpha) * acc_g;
          dalpha += (col_g - acc_g) * d1;
          c[7] = alpha * t * d1;
          acc_b = last_alpha * lc_b + (1.0f - last_alpha) * acc_b;
          dalpha += (col_b - acc_b) * d2;
          c[8] = alpha * t * d2;
          dalpha *= t;
          lc_r = col_r;
          lc_g = col_g;
          lc_b = col_b;
          last_alpha = alpha;
          dalpha += -t_fin / (1.0f - alpha) * bg_dot;
          c[11] = alpha * t;
          const float opacity = e1.y;
          if (opacity * gval < SPLAT_ALPHA_MAX) {
            c[5] = gval * dalpha;
            const float dgauss = opacity * dalpha;
            const float dsigma = -dgauss * gval;
            const float dx = px - e0.x;
            const float dy = py - e0.y;
            const float ddx = dsigma * (e0.z * dx + e0.w * dy);
            const float ddy = dsigma * (e0.w * dx + e1.x * dy);
            c[0] = -ddx;
            c[1] = -ddy;
            c[2] = dsigma * 0.5f * dx * dx;
            c[3] = dsigma * dx * dy;
            c[4] = dsigma * 0.5f * dy * dy;
            c[9] = fabsf(ddx);
            c[10] = fabsf(ddy);
          }
        }
#pragma unroll
        for (int q = 0; q < kSlots; q++) cbuf[((size_t)j * kSlots + q) * 256 + threadIdx.x] = c[q];
      }
      __syncthreads();
      // One thread per (entry, slot): the rectangle's pixels in row-major order.
      if (threadIdx.x < (gend - gstart) * (uint32_t)kSlots) {
        const uint32_t j = threadIdx.x / kSlots, q = threadIdx.x % kSlots;
        const uint32_t kk = gend - 1u - j;
        const uint32_t rm = srect[kk];
        const uint32_t cols = rm & 0xffffu, rows = rm >> 16;
        float a = 0.0f;
        if (cols && rows) {
          const uint32_t x0 = __ffs(cols) - 1u, x1 = min(32u - __clz(cols), gw);
          const uint32_t y0 = __ffs(rows) - 1u, y1 = min(32u - __clz(rows), gh);
          const float* b = cbuf + ((size_t)j * kSlots + q) * 256;
          for (uint32_t yy = y0; yy < y1; yy++)
            for (uint32_t xx = x0; xx < x1; xx++) a += b[yy * 16u + xx];
        }
        const uint32_t e = sent[kk];
        if (e < e_cap) eslot[(size_t)e * kSlots + q] = a;
      }
      __syncthreads();
      gend = gstart;
    }
    cend = cstart;
  }
}

// The per-Gaussian sum of rasterize_backward (rasterize.rs:480-503): entries in emission
// order from 0.0, into the screen-space gradient planes (written, not accumulated).
__global__ void __launch_bounds__(256) entry_slots_reduce_kernel(const uint32_t* __restrict__ entry_offset,
                                                                 int64_t n, const float4* __restrict__ eslot,
                                                                 int64_t e_cap, float4* __restrict__ pgrad,
                                                                 int64_t cap) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const int64_t s = entry_offset[g], e = min((int64_t)entry_offset[g + 1], e_cap);
  float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), b = a, c = a;
  for (int64_t i = s; i < e; i++) {
    const float4 u = eslot[3 * i], v = eslot[3 * i + 1], w = eslot[3 * i + 2];
    a.x += u.x; a.y += u.y; a.z += u.z; a.w += u.w;
    b.x += v.x; b.y += v.y; b.z += v.z; b.w += v.w;
    c.x += w.x; c.y += w.y; c.z += w.z; c.w += w.w;
  }
  pgrad[g] = a;
  pgrad[cap + g] = b;
  pgrad[2 * cap + g] = c;
}

Status launch_raster_bwd_det(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges,
                             const uint32_t* entry_offset, int64_t n, int64_t e_cap, uint32_t width, uint32_t height,
                             const float bg[3], const float* final_t, const uint32_t* n_contrib, const float* dimage,
                             float* eslot, float* pgrad, int64_t cap) {
  if (!c->raster.reference_tiles())
    return Status::make(SPLAT_ERR_INVALID, "the deterministic backward needs the reference's 16x16 tiles");
  static bool attr_set[64] = {};
  if (c->device >= 0 && c->device < 64 && !attr_set[c->device]) {
    SPLAT_CUDA(cudaFuncSetAttribute(raster_bwd_det_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kDetSmemBytes));
    attr_set[c->device] = true;
  }
  const uint32_t tiles_x = c->raster.tiles_x(width);
  const uint32_t blocks = c->raster.tiles(width, height);
  if (blocks > 0 && e_cap > 0) {
    raster_bwd_det_kernel<<<blocks, 256, kDetSmemBytes, c->stream>>>(
        reinterpret_cast<const float4*>(proj), gauss, reinterpret_cast<const uint2*>(ranges), entry_offset, e_cap,
        width, height, tiles_x, bg[0], bg[1], bg[2], final_t, n_contrib, dimage, eslot);
    c->launches.count++;
    SPLAT_LAUNCHED("raster_bwd_det_kernel");
  }
  if (n > 0) {
    entry_slots_reduce_kernel<<<ceil_div(n, 256), 256, 0, c->stream>>>(
        entry_offset, n, reinterpret_cast<const float4*>(eslot), e_cap, reinterpret_cast<float4*>(pgrad), cap);
    c->launches.count++;
    SPLAT_LAUNCHED("entry_slots_reduce_kernel");
  }
  return Status::ok();
}

// Expands CALL(TW, TH, CH) for the configuration rc; an unsupported one is an error.
#define SPLAT_RASTER_DISPATCH(rc, CALL)                                                       \
  do {                                                                                         \
    const uint32_t w_ = (rc).tile_w, h_ = (rc).tile_h, c_ = (rc).chunk;                        \
    if (w_ == 16 && h_ == 16 && c_ == 256) CALL(16, 16, 256);                                  \
    else if (w_ == 16 && h_ == 16 && c_ == 128) CALL(16, 16, 128);                             \
    else if (w_ == 16 && h_ == 16 && c_ == 64) CALL(16, 16, 64);                               \
    else if (w_ == 16 && h_ == 16 && c_ == 32) CALL(16, 16, 32);                               \
    else if (w_ == 8 && h_ == 8 && c_ == 256) CALL(8, 8, 256);                                 \
    else if (w_ == 8 && h_ == 8 && c_ == 128) CALL(8, 8, 128);                                 \
    else if (w_ == 8 && h_ == 8 && c_ == 64) CALL(8, 8, 64);                                   \
    else if (w_ == 8 && h_ == 8 && c_ == 32) CALL(8, 8, 32);                                   \
    else if (w_ == 16 && h_ == 32 && c_ == 256) CALL(16, 32, 256);                             \
    else if (w_ == 16 && h_ == 32 && c_ == 128) CALL(16, 32, 128);                             \
    else if (w_ == 16 && h_ == 32 && c_ == 64) CALL(16, 32, 64);                               \
    else if (w_ == 16 && h_ == 32 && c_ == 32) CALL(16, 32, 32);                               \
    else return Status::make(SPLAT_ERR_INVALID, "unsupported raster configuration");           \
  } while (0)

constexpr int kFwdChunk = 256;

Status launch_raster_fwd(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges, uint32_t width,
                         uint32_t height, const float bg[3], float* image, float* final_t, uint32_t* n_contrib,
                         uint64_t* pairs, const BatchTable* bt, uint32_t tiles_cap) {
  const RasterConfig& rc = c->raster;
  const uint32_t tiles_x = rc.tiles_x(width);
  const uint32_t blocks = bt ? tiles_cap : rc.tiles(width, height);
  if (blocks == 0) return Status::ok();
// With the 16-column tiles the forward stages chunks of kFwdChunk entries whatever the
// configuration's chunk depth (which then sets the backward's): fewer chunks mean fewer block
// barriers, and 256 was the faster forward on both shapes (16x16: 0.553 ms against 0.570
// with 128; 16x32: 0.585 against 0.616). 8x8 tiles (two warps) keep the configured depth.
#define SPLAT_FWD(TW, TH, CH, K)                                                                                  \
  raster_fwd_kernel<TW, TH, CH, K><<<blocks, TW * TH, 0, c->stream>>>(                                           \
      reinterpret_cast<const float4*>(proj), gauss, reinterpret_cast<const uint2*>(ranges), width, height, tiles_x, \
      bg[0], bg[1], bg[2], image, final_t, n_contrib, reinterpret_cast<unsigned long long*>(pairs), bt)
#define SPLAT_FWD8(TW, TH, CH) \
  if (pairs) SPLAT_FWD(TW, TH, CH, true); else SPLAT_FWD(TW, TH, CH, false)
  const bool count = pairs != nullptr;
  if (rc.tile_w == 16 && rc.tile_h == 16) {
    if (count) SPLAT_FWD(16, 16, kFwdChunk, true); else SPLAT_FWD(16, 16, kFwdChunk, false);
  } else if (rc.tile_w == 16 && rc.tile_h == 32) {
    if (count) SPLAT_FWD(16, 32, kFwdChunk, true); else SPLAT_FWD(16, 32, kFwdChunk, false);
  } else if (rc.tile_w == 8 && rc.tile_h == 8 && rc.chunk == 256) {
    SPLAT_FWD8(8, 8, 256);
  } else if (rc.tile_w == 8 && rc.tile_h == 8 && rc.chunk == 128) {
    SPLAT_FWD8(8, 8, 128);
  } else if (rc.tile_w == 8 && rc.tile_h == 8 && rc.chunk == 64) {
    SPLAT_FWD8(8, 8, 64);
  } else if (rc.tile_w == 8 && rc.tile_h == 8 && rc.chunk == 32) {
    SPLAT_FWD8(8, 8, 32);
  } else {
    return Status::make(SPLAT_ERR_INVALID, "unsupported raster configuration");
  }
#undef SPLAT_FWD8
#undef SPLAT_FWD
  c->launches.count++;
  SPLAT_LAUNCHED("raster_fwd_kernel");
  return Status::ok();
}

Status launch_raster_bwd(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges, uint32_t width,
                         uint32_t height, const float bg[3], const float* final_t, const uint32_t* n_contrib,
                         const float* dimage, float* pgrad, int64_t cap, uint64_t* pairs, const BatchTable* bt,
                         uint32_t tiles_cap) {
  const RasterConfig& rc = c->raster;
  const uint32_t tiles_x = rc.tiles_x(width);
  const uint32_t blocks = bt ? tiles_cap : rc.tiles(width, height);
  if (blocks == 0) return Status::ok();
#define SPLAT_BWD(TW, TH, CH, P)                                                                                  \
  raster_bwd_kernel<TW, TH, CH, P><<<blocks, TW * TH / P, 0, c->stream>>>(                                       \
      reinterpret_cast<const float4*>(proj), gauss, reinterpret_cast<const uint2*>(ranges), width, height, tiles_x, \
      bg[0], bg[1], bg[2], final_t, n_contrib, dimage, reinterpret_cast<float4*>(pgrad), cap,                     \
      reinterpret_cast<unsigned long long*>(pairs), bt)
#define SPLAT_BWD1(TW, TH, CH) SPLAT_BWD(TW, TH, CH, 1)
#define SPLAT_BWD2X(TW, TH, CH, K)                                                                                \
  raster_bwd_x2_kernel<TW, TH, CH, K><<<blocks, TW * TH / 2, 0, c->stream>>>(                                    \
      reinterpret_cast<const float4*>(proj), gauss, reinterpret_cast<const uint2*>(ranges), width, height, tiles_x, \
      bg[0], bg[1], bg[2], final_t, n_contrib, dimage, reinterpret_cast<float4*>(pgrad), cap,                     \
      reinterpret_cast<unsigned long long*>(pairs), bt)
#define SPLAT_BWD2(TW, TH, CH) SPLAT_BWD2X(TW, TH, CH, false)
#define SPLAT_BWD2C(TW, TH, CH) SPLAT_BWD2X(TW, TH, CH, true)
  if (rc.ppl == 2 && pairs)
    SPLAT_RASTER_DISPATCH(rc, SPLAT_BWD2C);
  else if (rc.ppl == 2)
    SPLAT_RASTER_DISPATCH(rc, SPLAT_BWD2);
  else
    SPLAT_RASTER_DISPATCH(rc, SPLAT_BWD1);
#undef SPLAT_BWD2C
#undef SPLAT_BWD2
#undef SPLAT_BWD2X
#undef SPLAT_BWD1
#undef SPLAT_BWD
  c->launches.count++;
  SPLAT_LAUNCHED("raster_bwd_kernel");
  return Status::ok();
}

}  // namespace splat
