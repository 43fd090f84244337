// splat_bin_count_noalloc: the entry-offset scan of splat_bin_count for callers that cannot
// let this library allocate device memory.
//
// Who cannot allocate, and why: an application that plans its whole device memory up front
// and hands every buffer to this library itself, for instance a renderer with a fixed
// per-frame memory budget or a host whose own allocator owns the device (a second
// allocator's cudaMalloc would fail once the budget is taken, or fragment it). Such a
// caller also cannot accept the device-wide synchronisation that cudaMalloc/cudaFree may
// imply in the middle of a frame. splat_bin_count takes its scratch from the context's
// arena, which may grow with cudaMalloc; this variant takes it from a fixed array in device
// memory instead and calls no allocating routine.
//
// The scratch is a file-scope __device__ array of kNoAllocScratchWords 64-bit words
// (32 KiB + 8 bytes): one partial sum per 4096 tile counts plus the total, so at most
// kNoAllocMaxGaussians (16,777,216) counts per call. Every GPU that loads the library holds
// it until the process exits. Host code cannot use the array's name as a device address,
// so the first call on each device resolves the address with cudaGetSymbolAddress (with
// that device current) and caches it; make that first call before any stream capture. The
// cached address belongs to the device's primary context: after cudaDeviceReset (which
// destroys that context) it is stale, so do not call this entry point again in a process
// that has reset the device.
// All calls share the array and it keeps the last call's contents; each call overwrites
// every word it reads, so nothing has to start at zero. Calls whose kernels overlap on the
// GPU (different streams, or different host threads) race on the array.
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"
#include "renderer.cuh"

namespace splat {

constexpr int64_t kNoAllocMaxGaussians = 16777216;
constexpr int64_t kNoAllocScratchWords = kNoAllocMaxGaussians / kScanValuesPerBlock + 1;

static __device__ __align__(256) uint64_t g_noalloc_scan_scratch[kNoAllocScratchWords];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
uint64_t* g_addr[kMaxDevices] = {};

// Device address of the scratch on the current device (resolved once per device).
Status scratch_address(int device, uint64_t** out) {
  if (device < 0 || device >= kMaxDevices) return Status::make(SPLAT_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> g(g_addr_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return Status::make(SPLAT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    g_addr[device] = static_cast<uint64_t*>(p);
  }
  *out = g_addr[device];
  return Status::ok();
}
}  // namespace

}  // namespace splat

using namespace splat;

extern "C" SPLAT_API int splat_bin_count_noalloc(splat_ctx* ctx, const uint32_t* num_tiles_dev, int64_t n,
                                                 uint32_t* entry_offset_dev, int64_t* num_entries) {
  if (!ctx) return SPLAT_ERR_INVALID;
  Ctx* c = splat_ctx_impl(ctx);
  if (n < 0 || !entry_offset_dev || !num_entries || (n && !num_tiles_dev)) {
    c->last_error = "splat_bin_count_noalloc: bad buffers";
    return SPLAT_ERR_INVALID;
  }
  if (n > kNoAllocMaxGaussians) {
    c->last_error = "splat_bin_count_noalloc: n exceeds the fixed scratch limit of 16777216 Gaussians";
    return SPLAT_ERR_CAPACITY;
  }
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) {
    cudaGetLastError();
    prev = -1;
  }
  if (prev != c->device) {
    const cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) {
      // Resolving (and caching) the scratch address now would do it on the wrong device.
      cudaGetLastError();
      c->last_error = std::string("splat_bin_count_noalloc: cudaSetDevice: ") + cudaGetErrorString(e);
      return SPLAT_ERR_CUDA;
    }
  }
  uint64_t* scratch = nullptr;
  Status s = scratch_address(c->device, &scratch);
  if (s.good()) s = launch_scan_u32_into(c, num_tiles_dev, n, entry_offset_dev, 1, scratch,
                                        scratch + (kNoAllocScratchWords - 1));
  uint64_t* h = reinterpret_cast<uint64_t*>(c->host_small);
  if (s.good())
    s = cuda_status(cudaMemcpyAsync(h, scratch + (kNoAllocScratchWords - 1), 8, cudaMemcpyDeviceToHost, c->stream),
                    "read entry count");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
  if (!s.good()) {
    c->last_error = s.msg;
    return s.code;
  }
  if (h[0] >= 0xffffffffull) {
    c->last_error = "too many tile entries for 32-bit offsets";
    return SPLAT_ERR_CAPACITY;
  }
  *num_entries = (int64_t)h[0];
  return SPLAT_OK;
}
