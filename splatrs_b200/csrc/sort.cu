// Binning (reference src/rasterize.rs:60-128) on the device:
//   scan of per-Gaussian tile counts -> entry offsets (Binning::entry_offset),
//   warp-cooperative emission of one (tile | depth) key per entry in Gaussian order,
//   stable LSD radix sort of the keys carrying the Gaussian index,
//   per-tile [start, end) ranges.
//
// Keys are compacted before sorting: the reference key is (tile << 32) | depth_bits with
// depth_bits the f32 bits of a positive depth. Subtracting the smallest visible depth bits
// and packing the tile above the remaining significant bits keeps the order of every pair
// of keys, so the sort runs over ceil((tile bits + depth bits) / 8) passes instead of 8.
// The sort is stable, and entries enter it in entry order, which reproduces the
// reference's tie-break on the entry index.
#include <atomic>

#include "common.cuh"
#include "kernels.cuh"

namespace splat {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096 values per block

// ---------------------------------------------------------------------------------------
// Exclusive scan of uint32 counts into uint32 offsets (with the total written at [n]).
// Three kernels: per-block sums, a single-block scan of the sums, per-block scan + add.
// Totals are carried in 64 bits; a total that does not fit in 32 bits raises a flag.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t block_sum_u64(uint64_t v, uint64_t* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  uint64_t t = 0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

// Block-wide exclusive scan of one uint64 per thread; returns the exclusive prefix, and
// the block total through *total.
__device__ __forceinline__ uint64_t block_exclusive_u64(uint64_t v, uint64_t* sh, uint64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint64_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) sh[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint64_t w = lane < nw ? sh[lane] : 0;
    uint64_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) sh[lane] = wi - w;
    if (lane == nw - 1) sh[32] = wi;
  }
  __syncthreads();
  uint64_t r = sh[warp] + incl - v;
  *total = sh[32];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t* __restrict__ in, int64_t n,
                                                                   uint64_t* __restrict__ partial) {
  __shared__ uint64_t sh[33];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  uint64_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const int64_t idx = base + (int64_t)j * kScanThreads + threadIdx.x;
    if (idx < n) s += in[idx];
  }
  s = block_sum_u64(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Single block: exclusive scan of `m` partials in place; total to *total.
__global__ void __launch_bounds__(1024) scan_partials_kernel(uint64_t* __restrict__ partial, int64_t m,
                                                             uint64_t* __restrict__ total) {
  __shared__ uint64_t sh[33];
  uint64_t carry = 0;
  for (int64_t base = 0; base < m; base += blockDim.x) {
    const int64_t idx = base + threadIdx.x;
    const uint64_t v = idx < m ? partial[idx] : 0;
    uint64_t tot;
    const uint64_t ex = block_exclusive_u64(v, sh, &tot);
    if (idx < m) partial[idx] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

// Writes out[i] = exclusive prefix (uint32) for i < n, and out[n] = total when `write_total`.
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const uint32_t* __restrict__ in, int64_t n,
                                                                  const uint64_t* __restrict__ partial,
                                                                  const uint64_t* __restrict__ total,
                                                                  uint32_t* __restrict__ out, int write_total) {
  __shared__ uint64_t sh[33];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint64_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const int64_t idx = base + j;
    v[j] = idx < n ? in[idx] : 0u;
    s += v[j];
  }
  uint64_t tot;
  uint64_t run = partial[blockIdx.x] + block_exclusive_u64(s, sh, &tot);
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    const int64_t idx = base + j;
    if (idx < n) out[idx] = (uint32_t)run;
    run += v[j];
  }
  if (write_total && blockIdx.x == 0 && threadIdx.x == 0) out[n] = (uint32_t)*total;
}

__global__ void fill_u32_kernel(uint32_t* __restrict__ dst, size_t words, uint32_t value, int vector) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t quads = vector ? words / 4 : 0;
  uint4* d4 = reinterpret_cast<uint4*>(dst);
  const uint4 v4 = make_uint4(value, value, value, value);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < quads; i += stride) d4[i] = v4;
  for (size_t i = quads * 4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) dst[i] = value;
}

// Zeroes up to three regions of 32-bit words in one launch.
__global__ void zero3_u32_kernel(uint32_t* __restrict__ a, size_t na, uint32_t* __restrict__ b, size_t nb,
                                 uint32_t* __restrict__ c3, size_t nc) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < na + nb + nc; i += stride) {
    if (i < na)
      a[i] = 0u;
    else if (i < na + nb)
      b[i - na] = 0u;
    else
      c3[i - na - nb] = 0u;
  }
}

Status launch_zero3_u32(Ctx* c, void* a, size_t na, void* b, size_t nb, void* c3, size_t nc) {
  const size_t words = na + nb + nc;
  if (words == 0) return Status::ok();
  const uint32_t grid = (uint32_t)std::min<size_t>((words + 255) / 256, (size_t)c->sm_count * 8);
  zero3_u32_kernel<<<grid, 256, 0, c->stream>>>(static_cast<uint32_t*>(a), na, static_cast<uint32_t*>(b), nb,
                                                static_cast<uint32_t*>(c3), nc);
  c->launches.count++;
  SPLAT_LAUNCHED("zero3_u32_kernel");
  return Status::ok();
}

Status launch_fill_u32(Ctx* c, void* dst, size_t words, uint32_t value) {
  if (words == 0) return Status::ok();
  const int vector = (reinterpret_cast<uintptr_t>(dst) & 15u) == 0;
  const size_t items = vector ? (words + 3) / 4 : words;
  const uint32_t grid = (uint32_t)std::min<size_t>((items + 255) / 256, (size_t)c->sm_count * 8);
  fill_u32_kernel<<<grid, 256, 0, c->stream>>>(reinterpret_cast<uint32_t*>(dst), words, value, vector);
  c->launches.count++;
  SPLAT_LAUNCHED("fill_u32_kernel");
  return Status::ok();
}

__global__ void publish_u32_kernel(const uint32_t* __restrict__ a, int na, const uint32_t* __restrict__ b, int nb,
                                   volatile uint32_t* out) {
  const int lane = threadIdx.x;
  if (lane < na) out[lane] = a[lane];
  if (lane < nb) out[na + lane] = b[lane];
  __threadfence_system();
}

__global__ void load_words_kernel(const volatile uint32_t* src, uint32_t* __restrict__ dst, int words) {
  for (int i = threadIdx.x; i < words; i += 32) dst[i] = src[i];
}

Status launch_load_words(Ctx* c, const void* src_mapped_dev, void* dst, int words) {
  load_words_kernel<<<1, 32, 0, c->stream>>>(static_cast<const volatile uint32_t*>(src_mapped_dev),
                                             static_cast<uint32_t*>(dst), words);
  c->launches.count++;
  SPLAT_LAUNCHED("load_words_kernel");
  return Status::ok();
}

Status launch_publish_u32(Ctx* c, const uint32_t* a, int na, const uint32_t* b, int nb) {
  return launch_publish_u32_to(c, a, na, b, nb, c->host_small_dev);
}

Status launch_publish_u32_to(Ctx* c, const uint32_t* a, int na, const uint32_t* b, int nb, void* out_dev) {
  if (na < 0 || nb < 0 || na + nb > 32) return Status::make(SPLAT_ERR_INVALID, "publish: at most 32 words");
  publish_u32_kernel<<<1, 32, 0, c->stream>>>(a, na, b, nb, reinterpret_cast<volatile uint32_t*>(out_dev));
  c->launches.count++;
  SPLAT_LAUNCHED("publish_u32_kernel");
  return Status::ok();
}

Status take_sort_error(Ctx* c) {
  volatile uint32_t* w = reinterpret_cast<volatile uint32_t*>(c->host_small) + kSortErrWord;
  if (*w == 0) return Status::ok();
  *w = 0;
  return Status::make(SPLAT_ERR_TIMEOUT, "radix sort: a tile's look-back wait ran out; that sort's output is invalid");
}

Status launch_scan_u32(Ctx* c, const uint32_t* in, int64_t n, uint32_t* out, int write_total, uint64_t* total_dev) {
  const uint32_t blocks = ceil_div((uint64_t)std::max<int64_t>(n, 1), kScanTile);
  uint64_t* partial = nullptr;
  SPLAT_TRY(arena_reserve(c, (size_t)blocks * 8, (void**)&partial));
  scan_reduce_kernel<<<blocks, kScanThreads, 0, c->stream>>>(in, n, partial);
  scan_partials_kernel<<<1, 1024, 0, c->stream>>>(partial, blocks, total_dev);
  scan_apply_kernel<<<blocks, kScanThreads, 0, c->stream>>>(in, n, partial, total_dev, out, write_total);
  c->launches.count += 3;
  SPLAT_LAUNCHED("scan kernels");
  return Status::ok();
}

// ---------------------------------------------------------------------------------------
// Key emission (rasterize.rs:76-104): the entries of Gaussian g occupy
// [entry_offset[g], entry_offset[g+1]) and enumerate its tile rectangle row by row.
// Each warp takes 32 consecutive Gaussians and writes their entries contiguously.
// ---------------------------------------------------------------------------------------
template <typename K>
__device__ __forceinline__ void emit_keys_body(const float4* __restrict__ rec, const uint32_t* __restrict__ entry_offset,
                                               int64_t n, uint32_t tiles_x, const uint32_t* __restrict__ depth_range,
                                               int dbits, int64_t limit, K* __restrict__ keys,
                                               uint32_t* __restrict__ vals, const BatchTable* bt = nullptr,
                                               int64_t n_view = 1) {
  const int lane = threadIdx.x & 31;
  const int64_t warp_id = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t g = warp_id * 32 + lane;
  const int64_t first = warp_id * 32;
  if (first >= n) return;
  uint32_t cnt = 0, tx0 = 0, ty0 = 0, w = 1, dkey = 0, toff = 0, txs = tiles_x;
  if (g < n) {
    if (bt) {  // batch: the record's view sets its tile grid and first global tile
      const int v = (int)(g / n_view);
      toff = bt->tile_start[v];
      txs = bt->tiles_x[v];
    }
    const uint32_t o0 = entry_offset[g], o1 = entry_offset[g + 1];
    cnt = o1 - o0;
    if (cnt) {
      const float4 r3 = rec[4 * g + 3];
      const uint32_t tmin = fbits(r3.z), tmax = fbits(r3.w);
      tx0 = tmin & 0xffffu;
      ty0 = tmin >> 16;
      w = (tmax & 0xffffu) - tx0;
      dkey = fbits(r3.x) - depth_range[0];
    }
  }
  const uint32_t start = entry_offset[first];
  // Inclusive warp scan of the counts.
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  for (uint32_t j0 = 0; j0 < total; j0 += 32) {
    const uint32_t j = j0 + lane;
    // Owner lane: first lane whose inclusive count exceeds j (binary search over lanes).
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const uint32_t v = __shfl_sync(0xffffffffu, incl, lo + step - 1);
      if (v <= j) lo += step;
    }
    const uint32_t o_incl = __shfl_sync(0xffffffffu, incl, lo);
    const uint32_t o_cnt = __shfl_sync(0xffffffffu, cnt, lo);
    const uint32_t o_tx0 = __shfl_sync(0xffffffffu, tx0, lo);
    const uint32_t o_ty0 = __shfl_sync(0xffffffffu, ty0, lo);
    const uint32_t o_w = __shfl_sync(0xffffffffu, w, lo);
    const uint32_t o_dkey = __shfl_sync(0xffffffffu, dkey, lo);
    const uint32_t o_toff = __shfl_sync(0xffffffffu, toff, lo);
    const uint32_t o_txs = __shfl_sync(0xffffffffu, txs, lo);
    if (j < total && (int64_t)start + j < limit) {
      const uint32_t local = j - (o_incl - o_cnt);
      const uint32_t ty = o_ty0 + local / o_w;
      const uint32_t tx = o_tx0 + local % o_w;
      const uint64_t tile = (uint64_t)o_toff + (uint64_t)ty * o_txs + tx;
      keys[start + j] = (K)((tile << dbits) | (uint64_t)o_dkey);
      vals[start + j] = (uint32_t)(first + lo);
    }
  }
}

template <typename K>
__global__ void __launch_bounds__(256) emit_keys_kernel(const float4* __restrict__ rec,
                                                        const uint32_t* __restrict__ entry_offset, int64_t n,
                                                        uint32_t tiles_x, const uint32_t* __restrict__ depth_range,
                                                        int dbits, K* __restrict__ keys, uint32_t* __restrict__ vals) {
  emit_keys_body<K>(rec, entry_offset, n, tiles_x, depth_range, dbits, INT64_MAX, keys, vals);
}

// ---------------------------------------------------------------------------------------
// Stable LSD radix sort, 8-bit digits, one kernel per pass (onesweep).
// One histogram kernel counts every pass's digits in a single read of the keys. Each pass
// kernel then takes tiles of 4096 keys in ticket order (an atomic counter, so a tile only
// ever waits for tiles whose blocks already run): 8 warps each rank 512 consecutive keys in
// 16 rounds of 32 (position order) with match-any peer groups and per-warp digit counters;
// a per-digit prefix over the warps gives block-local stable ranks. The tile's global
// offset per digit is the digit's start (a prefix over the pass's histogram) plus the
// counts of that digit in all earlier tiles, found by decoupled look-back: every tile
// publishes its count per digit as soon as it has it (AGGREGATE), then its inclusive
// prefix (PREFIX); a tile walks back over its predecessors' words, adding aggregates until
// it meets a prefix. Every wait on a predecessor is bounded: past kLookbackSpins polls the
// tile sets the error bit 2 in *err, sets the abort word so no other tile waits any longer,
// and writes nothing (callers treat the sort as failed).
// ---------------------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
// A pass block ranks ROUNDS rounds of 256 keys: 16 (4,096-key tiles) for large sorts, 4
// (1,024-key tiles) when there are at most kSmallSortKeys keys, so that a small sort still
// spreads over many SMs.
constexpr int kSortRounds = 16;
constexpr int kSortRoundsSmall = 4;
constexpr int64_t kSmallSortKeys = 1 << 20;
inline int sort_rounds_for(int64_t keys) { return keys <= kSmallSortKeys ? kSortRoundsSmall : kSortRounds; }
constexpr int kMaxPasses = 8;
constexpr uint64_t kLbAggregate = 1ull << 62, kLbPrefix = 2ull << 62, kLbCount = (1ull << 62) - 1ull;
constexpr uint32_t kLookbackSpins = 1u << 22;
constexpr int kLbWindow = 16;

// Control words of one sort (zeroed before it): the digit histogram of every pass, one
// ticket counter per pass, the abort word, and per pass one look-back word per tile and digit.
struct SortCtl {
  uint32_t* hist;     // [kMaxPasses][256]
  uint32_t* ticket;   // [kMaxPasses]
  uint32_t* abort;    // [1]
  uint64_t* status;   // [kMaxPasses][tiles][256]
};
inline size_t sort_ctl_bytes(uint64_t tiles) {
  return (size_t)kMaxPasses * 256 * 4 + kMaxPasses * 4 + 8 + (size_t)kMaxPasses * tiles * 256 * 8 + 64;
}
inline SortCtl carve_sort_ctl(void* base, uint64_t tiles) {
  SortCtl ctl;
  char* b = static_cast<char*>(base);
  ctl.status = reinterpret_cast<uint64_t*>(b);
  b += (size_t)kMaxPasses * tiles * 256 * 8;
  ctl.hist = reinterpret_cast<uint32_t*>(b);
  b += (size_t)kMaxPasses * 256 * 4;
  ctl.ticket = reinterpret_cast<uint32_t*>(b);
  b += kMaxPasses * 4;
  ctl.abort = reinterpret_cast<uint32_t*>(b);
  return ctl;
}

// Digit histograms of `passes` passes over keys[0, n): per-block counters in shared memory
// (native integer atomics), added to the global ones once per block.
template <typename K>
__device__ __forceinline__ void hist_body(const K* __restrict__ keys, int64_t n, int passes,
                                          uint32_t* __restrict__ hist, uint32_t (*cnt)[256]) {
  for (int i = threadIdx.x; i < kMaxPasses * 256; i += blockDim.x) cnt[i >> 8][i & 255] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const K k = keys[i];
    for (int p = 0; p < passes; p++) atomicAdd(&cnt[p][(uint32_t)(k >> (8 * p)) & 0xffu], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
    const uint32_t v = cnt[i >> 8][i & 255];
    if (v) atomicAdd(&hist[i], v);
  }
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const K* __restrict__ keys, int64_t n, int passes,
                                                                  uint32_t* __restrict__ hist) {
  __shared__ uint32_t cnt[kMaxPasses][256];
  hist_body<K>(keys, n, passes, hist, cnt);
}

// Dynamic shared memory of a pass: the tile's keys and values reordered by digit, the
// per-warp digit counters, the digits' block starts and output offsets, scan scratch.
template <typename K, int ROUNDS> constexpr size_t onesweep_smem() {
  return (size_t)kSortThreads * ROUNDS * (sizeof(K) + 4) + (size_t)kSortWarps * 256 * 4 + 2 * 256 * 4 + 64;
}

// Exclusive prefix over the 256 digits of v (thread d holds digit d's value); `wsum` holds
// kSortWarps words. Returns thread d's prefix.
__device__ __forceinline__ uint32_t digit_exclusive(uint32_t v, uint32_t* wsum) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  __syncthreads();
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  uint32_t wprefix = 0;
  for (int w = 0; w < warp; w++) wprefix += wsum[w];
  return wprefix + incl - v;
}

// One pass over keys_in[0, n) (digit at `shift`): `hist` is this pass's 256 global counts,
// `status` its look-back words, `ticket` its tile counter.
template <typename K, int ROUNDS>
__device__ __forceinline__ void onesweep_body(const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                              int64_t n, int shift, const uint32_t* __restrict__ hist,
                                              uint64_t* __restrict__ status, uint32_t* __restrict__ ticket,
                                              uint32_t* __restrict__ abort_word, uint32_t* __restrict__ err,
                                              K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                              unsigned char* dsm) {
  constexpr int TILE = kSortThreads * ROUNDS;
  K* sk = reinterpret_cast<K*>(dsm);
  uint32_t* sv = reinterpret_cast<uint32_t*>(sk + TILE);
  uint32_t(*wcnt)[256] = reinterpret_cast<uint32_t(*)[256]>(sv + TILE);
  uint32_t* dstart = reinterpret_cast<uint32_t*>(wcnt) + kSortWarps * 256;
  uint32_t* doff = dstart + 256;
  uint32_t* wsum = doff + 256;  // kSortWarps words, then the tile number and the failure word
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t tiles = (n + TILE - 1) / TILE;
  if (threadIdx.x == 0) {
    wsum[kSortWarps] = atomicAdd(ticket, 1u);
    wsum[kSortWarps + 1] = 0;
  }
  for (int d = lane; d < 256; d += 32) wcnt[warp][d] = 0;
  __syncthreads();
  const uint32_t tile = wsum[kSortWarps];
  if ((int64_t)tile >= tiles) return;
  const int64_t bbase = (int64_t)tile * TILE;
  const int64_t wbase = bbase + (int64_t)warp * (32 * ROUNDS);
  K k[ROUNDS];
  uint32_t v[ROUNDS];
  uint32_t rank[ROUNDS];
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    const int64_t idx = wbase + r * 32 + lane;
    const bool valid = idx < n;
    k[r] = valid ? keys_in[idx] : (K)0;
    v[r] = valid ? vals_in[idx] : 0u;
    const uint32_t d = valid ? ((uint32_t)(k[r] >> shift) & 0xffu) : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t before = valid ? wcnt[warp][d] : 0u;
    rank[r] = before + __popc(peers & lt);
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // Per digit (thread d): exclusive prefix over the warps and the tile's count.
  const int d = threadIdx.x;
  uint32_t total = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) {
    const uint32_t c = wcnt[w][d];
    wcnt[w][d] = total;
    total += c;
  }
  // Publish the tile's count of digit d at once; tile 0's is already its prefix.
  volatile uint64_t* my_word = status + (size_t)tile * 256 + d;
  *my_word = (tile == 0 ? kLbPrefix : kLbAggregate) | (uint64_t)total;
  // Look back over the earlier tiles, kLbWindow words at a time (independent loads), nearest
  // first: add aggregates until a prefix; a word not yet published is polled alone (bounded).
  uint64_t excl = 0;
  bool failed = false;
  int64_t t = (int64_t)tile - 1;
  while (t >= 0) {
    uint64_t w[kLbWindow];
#pragma unroll
    for (int i = 0; i < kLbWindow; i++)
      w[i] = t - i >= 0 ? *(const volatile uint64_t*)(status + (size_t)(t - i) * 256 + d) : kLbPrefix;
    int i = 0;
    bool done = false;
#pragma unroll
    for (int q = 0; q < kLbWindow; q++) {
      if (done || i < q) continue;  // stopped at a prefix or an unpublished word before q
      const uint64_t sq = w[q];
      if ((sq >> 62) == 0) continue;
      excl += sq & kLbCount;
      i = q + 1;
      if ((sq >> 62) == 2) done = true;
    }
    if (done) break;
    t -= i;
    if (i == kLbWindow) continue;
    // Word t is not published yet: wait for it.
    const volatile uint64_t* wp = status + (size_t)t * 256 + d;
    uint32_t spins = 0;
    while ((*wp >> 62) == 0) {
      if (++spins >= kLookbackSpins || *(volatile uint32_t*)abort_word) {
        failed = true;
        break;
      }
      __nanosleep(32);
    }
    if (failed) break;
  }
  if (failed) {
    atomicOr(abort_word, 1u);
    // A plain store: err may be mapped host memory. Racing writers all set the same bit.
    volatile uint32_t* e = err;
    *e = *e | 2u;
    wsum[kSortWarps + 1] = 1;
  } else if (tile > 0) {
    *my_word = kLbPrefix | (excl + total);
  }
  // Block starts of the digits and the pass's global digit starts.
  const uint32_t start = digit_exclusive(total, wsum);
  dstart[d] = start;
  const uint32_t gstart = digit_exclusive(hist[d], wsum);
  doff[d] = gstart + (uint32_t)excl - start;  // output index = doff[digit] + block-sorted index
  __syncthreads();
  if (wsum[kSortWarps + 1]) return;
  // Reorder the tile's keys by digit in shared memory (stable).
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    const int64_t idx = wbase + r * 32 + lane;
    if (idx < n) {
      const uint32_t dg = (uint32_t)(k[r] >> shift) & 0xffu;
      const uint32_t pos = dstart[dg] + wcnt[warp][dg] + rank[r];
      sk[pos] = k[r];
      sv[pos] = v[r];
    }
  }
  __syncthreads();
  // Write out runs of equal digits contiguously.
  const int64_t nb = n - bbase < TILE ? n - bbase : TILE;
  for (int i = threadIdx.x; i < nb; i += kSortThreads) {
    const K key = sk[i];
    const uint32_t dg = (uint32_t)(key >> shift) & 0xffu;
    const uint32_t pos = doff[dg] + (uint32_t)i;
    if (pos < (uint64_t)n) {
      keys_out[pos] = key;
      vals_out[pos] = sv[i];
    }
  }
}

template <typename K, int ROUNDS>
__global__ void __launch_bounds__(kSortThreads) radix_onesweep_kernel(const K* __restrict__ keys_in,
                                                                      const uint32_t* __restrict__ vals_in, int64_t n,
                                                                      int pass, SortCtl ctl, uint32_t* __restrict__ err,
                                                                      K* __restrict__ keys_out,
                                                                      uint32_t* __restrict__ vals_out) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const uint64_t tiles = (uint64_t)((n + kSortThreads * ROUNDS - 1) / (kSortThreads * ROUNDS));
  onesweep_body<K, ROUNDS>(keys_in, vals_in, n, 8 * pass, ctl.hist + 256 * pass, ctl.status + (size_t)pass * tiles * 256,
                   ctl.ticket + pass, ctl.abort, err, keys_out, vals_out, dsm);
}

// Tile ranges (rasterize.rs:108-119) and, optionally, the reference 64-bit keys.
template <typename K>
__global__ void tile_ranges_kernel(const K* __restrict__ keys, int64_t n, int dbits,
                                   const uint32_t* __restrict__ depth_range, uint32_t* __restrict__ ranges,
                                   uint64_t* __restrict__ ref_keys) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = (uint64_t)keys[i];
  const uint64_t tile = k >> dbits;
  if (i == 0 || ((uint64_t)keys[i - 1] >> dbits) != tile) ranges[2 * tile] = (uint32_t)i;
  if (i == n - 1 || ((uint64_t)keys[i + 1] >> dbits) != tile) ranges[2 * tile + 1] = (uint32_t)(i + 1);
  if (ref_keys) {
    const uint64_t mask = dbits >= 64 ? ~0ull : ((1ull << dbits) - 1ull);
    const uint32_t depth_bits = (uint32_t)(k & mask) + depth_range[0];
    ref_keys[i] = (tile << 32) | depth_bits;
  }
}

// One pass of the sort over E keys with tiles of ROUNDS rounds (the kernel's shared memory
// attribute set on first use).
template <typename K, int ROUNDS>
static Status launch_onesweep(Ctx* c, const K* kin, const uint32_t* vin, int64_t E, int pass, const SortCtl& ctl,
                              uint32_t* err, K* kout, uint32_t* vout) {
  static std::atomic<uint64_t> attr_done{0};
  if (c->device >= 64 || !(attr_done.load() & (1ull << c->device))) {
    SPLAT_CUDA(cudaFuncSetAttribute(radix_onesweep_kernel<K, ROUNDS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)onesweep_smem<K, ROUNDS>()));
    if (c->device < 64) attr_done.fetch_or(1ull << c->device);
  }
  const uint64_t tiles = ceil_div(E, (uint64_t)kSortThreads * ROUNDS);
  radix_onesweep_kernel<K, ROUNDS><<<(uint32_t)tiles, kSortThreads, onesweep_smem<K, ROUNDS>(), c->stream>>>(
      kin, vin, E, pass, ctl, err, kout, vout);
  c->launches.count++;
  SPLAT_LAUNCHED("radix_onesweep_kernel");
  return Status::ok();
}

template <typename K>
static Status sort_and_range(Ctx* c, const float* proj, const uint32_t* entry_offset, int64_t n, int64_t E,
                             const uint32_t* depth_range, int dbits, int total_bits, uint32_t tiles_x,
                             uint32_t num_tiles, uint32_t* gauss_out, uint64_t* keys_out, uint32_t* ranges) {
  const int passes = std::max(1, (total_bits + 7) / 8);
  const int rounds = sort_rounds_for(E);
  K *ka = nullptr, *kb = nullptr;
  uint32_t* vb = nullptr;
  SPLAT_TRY(arena_reserve(c, (size_t)E * sizeof(K), (void**)&ka));
  SPLAT_TRY(arena_reserve(c, (size_t)E * sizeof(K), (void**)&kb));
  SPLAT_TRY(arena_reserve(c, (size_t)E * 4, (void**)&vb));
  const uint64_t tiles = ceil_div(E, (uint64_t)kSortThreads * rounds);
  void* ctl_base = nullptr;
  SPLAT_TRY(arena_reserve(c, sort_ctl_bytes(tiles), &ctl_base));
  const SortCtl ctl = carve_sort_ctl(ctl_base, tiles);
  SPLAT_TRY(launch_fill_u32(c, ctl_base, sort_ctl_bytes(tiles) / 4, 0u));
  // Ping-pong so that the last pass writes the caller's buffer.
  uint32_t* va = (passes % 2 == 0) ? gauss_out : vb;
  uint32_t* vo = (passes % 2 == 0) ? vb : gauss_out;
  const uint32_t warps = ceil_div(n, 32);
  emit_keys_kernel<K><<<ceil_div((uint64_t)warps * 32, 256), 256, 0, c->stream>>>(
      reinterpret_cast<const float4*>(proj), entry_offset, n, tiles_x, depth_range, dbits, ka, va);
  c->launches.count++;
  SPLAT_LAUNCHED("emit_keys_kernel");
  radix_hist_kernel<K><<<std::min<uint64_t>(tiles, (uint64_t)c->sm_count * 4), kSortThreads, 0, c->stream>>>(
      ka, E, passes, ctl.hist);
  c->launches.count++;
  SPLAT_LAUNCHED("radix_hist_kernel");
  uint32_t* err = reinterpret_cast<uint32_t*>(static_cast<char*>(c->host_small_dev) + kAsyncErrorWordOffset);
  K* kin = ka;
  K* kout = kb;
  uint32_t* vin = va;
  uint32_t* vout = vo;
  for (int p = 0; p < passes; p++) {
    if (rounds == kSortRoundsSmall)
      SPLAT_TRY((launch_onesweep<K, kSortRoundsSmall>(c, kin, vin, E, p, ctl, err, kout, vout)));
    else
      SPLAT_TRY((launch_onesweep<K, kSortRounds>(c, kin, vin, E, p, ctl, err, kout, vout)));
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  SPLAT_TRY(launch_fill_u32(c, ranges, (size_t)num_tiles * 2, 0u));
  tile_ranges_kernel<K><<<ceil_div(E, 256), 256, 0, c->stream>>>(kin, E, dbits, depth_range, ranges, keys_out);
  c->launches.count++;
  SPLAT_LAUNCHED("tile_ranges_kernel");
  return Status::ok();
}

Status launch_bin_sort(Ctx* c, const float* proj, const uint32_t* entry_offset, int64_t n, int64_t E,
                       const uint32_t* depth_range_dev, uint32_t depth_min, uint32_t depth_max, uint32_t width,
                       uint32_t height, uint32_t* gauss_out, uint64_t* keys_out, uint32_t* ranges) {
  const uint32_t tiles_x = c->raster.tiles_x(width), tiles_y = c->raster.tiles_y(height);
  const uint32_t num_tiles = tiles_x * tiles_y;
  if (E == 0) {
    SPLAT_TRY(launch_fill_u32(c, ranges, (size_t)num_tiles * 2, 0u));
    return Status::ok();
  }
  const uint32_t span = depth_max - depth_min;
  const int dbits = span == 0 ? 0 : 32 - __builtin_clz(span);
  const int tbits = num_tiles <= 1 ? 0 : 32 - __builtin_clz(num_tiles - 1);
  const int total = dbits + tbits;
  if (total <= 32)
    return sort_and_range<uint32_t>(c, proj, entry_offset, n, E, depth_range_dev, dbits, total, tiles_x, num_tiles,
                                    gauss_out, keys_out, ranges);
  return sort_and_range<uint64_t>(c, proj, entry_offset, n, E, depth_range_dev, dbits, total, tiles_x, num_tiles,
                                  gauss_out, keys_out, ranges);
}

// ---------------------------------------------------------------------------------------
// Device-driven binning: the entry count and the depth range stay in device memory, so the
// host never waits for them. Grids and buffers are sized for a capacity E_cap; every
// kernel reads the count (clamped to E_cap) and the key width from device memory, skips
// passes the keys do not need, and the last needed pass writes the caller's buffer. An
// entry count above E_cap sets *overflow (sticky) and sorts only the first E_cap entries;
// the caller must discard that view's results. Keys are the compacted keys of
// launch_bin_sort held in 64 bits, and the passes are the same, so the output equals it.
// ---------------------------------------------------------------------------------------
struct DevSortPlan {
  int64_t E;
  int dbits;
  int passes;
};

__device__ __forceinline__ DevSortPlan dev_sort_plan(const uint64_t* __restrict__ E_dev, int64_t E_cap,
                                                     const uint32_t* __restrict__ dr, int tbits) {
  DevSortPlan p;
  const uint64_t e = *E_dev;
  p.E = e < (uint64_t)E_cap ? (int64_t)e : E_cap;
  const uint32_t span = p.E > 0 ? dr[1] - dr[0] : 0u;
  p.dbits = span == 0 ? 0 : 32 - __clz(span);
  const int total = p.dbits + tbits;
  p.passes = total == 0 ? 1 : (total + 7) / 8;
  return p;
}

__global__ void __launch_bounds__(256) emit_keys_dev_kernel(const float4* __restrict__ rec,
                                                            const uint32_t* __restrict__ entry_offset, int64_t n,
                                                            uint32_t tiles_x, const uint32_t* __restrict__ depth_range,
                                                            const uint64_t* __restrict__ E_dev, int64_t E_cap, int tbits,
                                                            uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                                            uint32_t* __restrict__ overflow,
                                                            const BatchTable* __restrict__ bt, int64_t n_view) {
  const DevSortPlan p = dev_sort_plan(E_dev, E_cap, depth_range, tbits);
  if (blockIdx.x == 0 && threadIdx.x == 0 && *E_dev > (uint64_t)E_cap) atomicOr(overflow, 1u);
  emit_keys_body<uint64_t>(rec, entry_offset, n, tiles_x, depth_range, p.dbits, E_cap, keys, vals, bt, n_view);
}

__global__ void __launch_bounds__(kSortThreads) radix_hist_dev_kernel(const uint64_t* __restrict__ keys,
                                                                      const uint64_t* __restrict__ E_dev,
                                                                      int64_t E_cap, const uint32_t* __restrict__ dr,
                                                                      int tbits, uint32_t* __restrict__ hist) {
  __shared__ uint32_t cnt[kMaxPasses][256];
  const DevSortPlan p = dev_sort_plan(E_dev, E_cap, dr, tbits);
  hist_body<uint64_t>(keys, p.E, p.passes, hist, cnt);
}

template <int ROUNDS>
__global__ void __launch_bounds__(kSortThreads) radix_onesweep_dev_kernel(
    uint64_t* __restrict__ ka, uint64_t* __restrict__ kb, uint32_t* __restrict__ va, uint32_t* __restrict__ vb,
    const uint64_t* __restrict__ E_dev, int64_t E_cap, const uint32_t* __restrict__ dr, int tbits, int pass,
    SortCtl ctl, uint64_t tiles_cap, uint32_t* __restrict__ err, uint32_t* __restrict__ vals_final) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const DevSortPlan p = dev_sort_plan(E_dev, E_cap, dr, tbits);
  if (pass >= p.passes) return;
  const bool odd = pass & 1;
  uint32_t* vout = pass == p.passes - 1 ? vals_final : (odd ? va : vb);
  onesweep_body<uint64_t, ROUNDS>(odd ? kb : ka, odd ? vb : va, p.E, 8 * pass, ctl.hist + 256 * pass,
                          ctl.status + (size_t)pass * tiles_cap * 256, ctl.ticket + pass, ctl.abort, err,
                          odd ? ka : kb, vout, dsm);
}

__global__ void tile_ranges_dev_kernel(const uint64_t* __restrict__ ka, const uint64_t* __restrict__ kb,
                                       const uint64_t* __restrict__ E_dev, int64_t E_cap,
                                       const uint32_t* __restrict__ dr, int tbits, uint32_t* __restrict__ ranges) {
  const DevSortPlan p = dev_sort_plan(E_dev, E_cap, dr, tbits);
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.E) return;
  const uint64_t* keys = ((p.passes - 1) & 1) ? ka : kb;  // written by the last pass
  const uint64_t tile = keys[i] >> p.dbits;
  if (i == 0 || (keys[i - 1] >> p.dbits) != tile) ranges[2 * tile] = (uint32_t)i;
  if (i == p.E - 1 || (keys[i + 1] >> p.dbits) != tile) ranges[2 * tile + 1] = (uint32_t)(i + 1);
}

size_t dev_sort_scratch_bytes(int64_t E_cap) {
  const uint64_t cap = (uint64_t)std::max<int64_t>(E_cap, 1);
  const uint64_t tiles = ceil_div(cap, (uint64_t)kSortThreads * sort_rounds_for((int64_t)cap));
  return 2 * cap * 8 + 2 * cap * 4 + sort_ctl_bytes(tiles) + 6 * 256;  // 5 pieces, 256-aligned
}

template <int ROUNDS>
static Status launch_onesweep_dev(Ctx* c, uint64_t* ka, uint64_t* kb, uint32_t* va, uint32_t* vb,
                                  const uint64_t* E_dev, int64_t E_cap, const uint32_t* dr, int tbits, int pass,
                                  const SortCtl& ctl, uint64_t tiles, uint32_t* overflow, uint32_t* gauss_out) {
  static std::atomic<uint64_t> attr_done{0};
  if (c->device >= 64 || !(attr_done.load() & (1ull << c->device))) {
    SPLAT_CUDA(cudaFuncSetAttribute(radix_onesweep_dev_kernel<ROUNDS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)onesweep_smem<uint64_t, ROUNDS>()));
    if (c->device < 64) attr_done.fetch_or(1ull << c->device);
  }
  radix_onesweep_dev_kernel<ROUNDS><<<(uint32_t)tiles, kSortThreads, onesweep_smem<uint64_t, ROUNDS>(), c->stream>>>(
      ka, kb, va, vb, E_dev, E_cap, dr, tbits, pass, ctl, tiles, overflow, gauss_out);
  c->launches.count++;
  SPLAT_LAUNCHED("radix_onesweep_dev_kernel");
  return Status::ok();
}

Status launch_bin_sort_dev(Ctx* c, const float* proj, const uint32_t* entry_offset, int64_t n, const uint64_t* E_dev,
                           int64_t E_cap, const uint32_t* depth_range_dev, uint32_t width, uint32_t height,
                           void* scratch, uint32_t* gauss_out, uint32_t* ranges, uint32_t* overflow,
                           const BatchTable* bt, int64_t n_view, uint32_t tiles_cap) {
  const uint32_t tiles_x = c->raster.tiles_x(width), tiles_y = c->raster.tiles_y(height);
  const uint32_t num_tiles = bt ? tiles_cap : tiles_x * tiles_y;
  const int tbits = num_tiles <= 1 ? 0 : 32 - __builtin_clz(num_tiles - 1);
  const int max_passes = (tbits + 32 + 7) / 8;
  const uint64_t cap = (uint64_t)std::max<int64_t>(E_cap, 1);
  const int rounds = sort_rounds_for((int64_t)cap);
  const uint64_t tiles = ceil_div(cap, (uint64_t)kSortThreads * rounds);
  // Carve the scratch (256-byte aligned pieces).
  auto carve = [&](size_t bytes) {
    void* p = scratch;
    scratch = static_cast<char*>(scratch) + ((bytes + 255) & ~(size_t)255);
    return p;
  };
  uint64_t* ka = static_cast<uint64_t*>(carve(cap * 8));
  uint64_t* kb = static_cast<uint64_t*>(carve(cap * 8));
  uint32_t* va = static_cast<uint32_t*>(carve(cap * 4));
  uint32_t* vb = static_cast<uint32_t*>(carve(cap * 4));
  void* ctl_base = carve(sort_ctl_bytes(tiles));
  const SortCtl ctl = carve_sort_ctl(ctl_base, tiles);
  // One launch clears the tile ranges, the look-back words of the passes these keys can need,
  // and the histograms, tickets and abort word.
  SPLAT_TRY(launch_zero3_u32(c, ranges, (size_t)num_tiles * 2, ctl.status, (size_t)max_passes * tiles * 256 * 2,
                             ctl.hist, (size_t)(kMaxPasses * 256 + kMaxPasses + 2)));
  if (n > 0) {
    const uint32_t warps = ceil_div(n, 32);
    emit_keys_dev_kernel<<<ceil_div((uint64_t)warps * 32, 256), 256, 0, c->stream>>>(
        reinterpret_cast<const float4*>(proj), entry_offset, n, tiles_x, depth_range_dev, E_dev, E_cap, tbits, ka, va,
        overflow, bt, std::max<int64_t>(n_view, 1));
    c->launches.count++;
    SPLAT_LAUNCHED("emit_keys_dev_kernel");
  }
  radix_hist_dev_kernel<<<(uint32_t)std::min<uint64_t>(tiles, (uint64_t)c->sm_count * 4), kSortThreads, 0,
                          c->stream>>>(ka, E_dev, E_cap, depth_range_dev, tbits, ctl.hist);
  c->launches.count++;
  SPLAT_LAUNCHED("radix_hist_dev_kernel");
  for (int pass = 0; pass < max_passes; pass++) {
    if (rounds == kSortRoundsSmall)
      SPLAT_TRY(launch_onesweep_dev<kSortRoundsSmall>(c, ka, kb, va, vb, E_dev, E_cap, depth_range_dev, tbits, pass,
                                                      ctl, tiles, overflow, gauss_out));
    else
      SPLAT_TRY(launch_onesweep_dev<kSortRounds>(c, ka, kb, va, vb, E_dev, E_cap, depth_range_dev, tbits, pass, ctl,
                                                 tiles, overflow, gauss_out));
  }
  tile_ranges_dev_kernel<<<ceil_div(cap, 256), 256, 0, c->stream>>>(ka, kb, E_dev, E_cap, depth_range_dev, tbits,
                                                                     ranges);
  c->launches.count++;
  SPLAT_LAUNCHED("tile_ranges_dev_kernel");
  return Status::ok();
}

}  // namespace splat

namespace splat {

// The scan of launch_scan_u32 with caller-provided scratch: `partial` holds one uint64 per
// 4096 input values and `total` one uint64. Allocates nothing.
Status launch_scan_u32_into(Ctx* c, const uint32_t* in, int64_t n, uint32_t* out, int write_total,
                            uint64_t* partial, uint64_t* total) {
  const uint32_t blocks = ceil_div((uint64_t)std::max<int64_t>(n, 1), kScanTile);
  scan_reduce_kernel<<<blocks, kScanThreads, 0, c->stream>>>(in, n, partial);
  scan_partials_kernel<<<1, 1024, 0, c->stream>>>(partial, blocks, total);
  scan_apply_kernel<<<blocks, kScanThreads, 0, c->stream>>>(in, n, partial, total, out, write_total);
  c->launches.count += 3;
  SPLAT_LAUNCHED("scan kernels");
  return Status::ok();
}

}  // namespace splat
