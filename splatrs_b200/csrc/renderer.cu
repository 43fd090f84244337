// splat_renderer: a model resident in device memory plus the per-view buffers of the
// render path, driven with host buffers. It is the drop-in for render::render
// (reference src/render.rs:14-23) and for the differentiable chain of
// examples/profile.rs:34-52 (project_all -> bin -> rasterize_forward -> rasterize_backward
// -> project_backward_all).
#include <algorithm>
#include <cstring>
#include <new>

#include "common.cuh"
#include "kernels.cuh"
#include "renderer.cuh"

namespace splat {

Status DevBuf::ensure(size_t want) {
  if (want <= bytes) return Status::ok();
  const size_t grow = std::max(want, bytes + bytes / 2);
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
  cudaError_t e = cudaMalloc(&ptr, grow);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return Status::make(SPLAT_ERR_CUDA, std::string("device allocation of ") + std::to_string(grow) +
                                            " bytes failed: " + cudaGetErrorString(e));
  }
  bytes = grow;
  return Status::ok();
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

Status ViewBuffers::ensure(int64_t n, uint32_t width, uint32_t height) {
  const size_t npix = (size_t)width * height;
  const uint32_t tiles = max_tiles(width, height);  // room for every tile shape
  SPLAT_TRY(proj.ensure((size_t)std::max<int64_t>(n, 1) * kProjFloats * 4));
  SPLAT_TRY(num_tiles.ensure((size_t)std::max<int64_t>(n, 1) * 4));
  SPLAT_TRY(entry_offset.ensure((size_t)(n + 1) * 4));
  SPLAT_TRY(depth_range.ensure(8));
  SPLAT_TRY(tile_range.ensure((size_t)tiles * 8));
  SPLAT_TRY(image.ensure(npix * 12));
  SPLAT_TRY(final_t.ensure(npix * 4));
  SPLAT_TRY(n_contrib.ensure(npix * 4));
  SPLAT_TRY(dimage.ensure(npix * 12));
  SPLAT_TRY(pairs.ensure(16));
  return Status::ok();
}

Status ViewBuffers::ensure_batch(int64_t records, uint64_t pixels, uint32_t tiles) {
  SPLAT_TRY(proj.ensure((size_t)std::max<int64_t>(records, 1) * kProjFloats * 4));
  SPLAT_TRY(num_tiles.ensure((size_t)std::max<int64_t>(records, 1) * 4));
  SPLAT_TRY(entry_offset.ensure((size_t)(records + 1) * 4));
  SPLAT_TRY(depth_range.ensure(8));
  SPLAT_TRY(tile_range.ensure((size_t)tiles * 8));
  SPLAT_TRY(image.ensure(pixels * 12));
  SPLAT_TRY(final_t.ensure(pixels * 4));
  SPLAT_TRY(n_contrib.ensure(pixels * 4));
  SPLAT_TRY(pairs.ensure(16));
  return Status::ok();
}

void ViewBuffers::release() {
  for (DevBuf* b : {&proj, &num_tiles, &entry_offset, &depth_range, &tile_range, &gauss, &image, &final_t, &n_contrib,
                    &dimage, &pairs, &sort_scratch, &scan_partial, &counters})
    b->release();
}

Status render_view_dev(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                       const splat_proj_opts& opts, const float bg[3], ViewBuffers& v, const StepParams* sp,
                       const void* bf16) {
  SPLAT_TRY(v.ensure(n, cam.width, cam.height));
  const int64_t e_cap = std::max<int64_t>(v.e_cap, 1);
  SPLAT_TRY(v.gauss.ensure((size_t)e_cap * 4));
  SPLAT_TRY(v.sort_scratch.ensure(dev_sort_scratch_bytes(e_cap)));
  SPLAT_TRY(v.scan_partial.ensure(((size_t)std::max<int64_t>(n, 1) / kScanValuesPerBlock + 2) * 8));
  if (v.counters.bytes == 0) {
    SPLAT_TRY(v.counters.ensure(64));
    SPLAT_TRY(launch_fill_u32(c, v.counters.ptr, 16, 0u));
  }
  float* proj = v.proj.as<float>();
  uint32_t* nt = v.num_tiles.as<uint32_t>();
  uint32_t* dr = v.depth_range.as<uint32_t>();
  SPLAT_TRY(launch_project_fwd(c, planes, n, cap, cam, opts, proj, nt, dr, sp, bf16));
  SPLAT_TRY(launch_scan_u32_into(c, nt, n, v.entry_offset.as<uint32_t>(), 1, v.scan_partial.as<uint64_t>(),
                                 v.entry_count()));
  SPLAT_TRY(launch_bin_sort_dev(c, proj, v.entry_offset.as<uint32_t>(), n, v.entry_count(), e_cap, dr, cam.width,
                                cam.height, v.sort_scratch.ptr, v.gauss.as<uint32_t>(), v.tile_range.as<uint32_t>(),
                                v.overflow_flag()));
  return launch_raster_fwd(c, proj, v.gauss.as<uint32_t>(), v.tile_range.as<uint32_t>(), cam.width, cam.height, bg,
                           v.image.as<float>(), v.final_t.as<float>(), v.n_contrib.as<uint32_t>(), nullptr);
}

// Projection, binning and forward compositing of one view into `v`.
Status render_view(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                   const splat_proj_opts& opts, const float bg[3], ViewBuffers& v, int64_t* entries_out,
                   const void* bf16) {
  SPLAT_TRY(v.ensure(n, cam.width, cam.height));
  float* proj = v.proj.as<float>();
  uint32_t* nt = v.num_tiles.as<uint32_t>();
  uint32_t* dr = v.depth_range.as<uint32_t>();
  SPLAT_TRY(launch_project_fwd(c, planes, n, cap, cam, opts, proj, nt, dr, nullptr, bf16));
  uint64_t* total = nullptr;
  SPLAT_TRY(arena_reserve(c, 8, (void**)&total));
  SPLAT_TRY(launch_scan_u32(c, nt, n, v.entry_offset.as<uint32_t>(), 1, total));
  // One read-back per view: the entry count and the depth range size the sort. A kernel
  // stores them into mapped host memory, so the read does not wait behind transfers queued
  // on a copy engine (a renderer step's downloads overlap the next step).
  SPLAT_TRY(launch_publish_u32(c, reinterpret_cast<const uint32_t*>(total), 2, dr, 2));
  SPLAT_CUDA(cudaStreamSynchronize(c->stream));
  SPLAT_TRY(take_sort_error(c));
  const volatile uint64_t* h = reinterpret_cast<const volatile uint64_t*>(c->host_small);
  const uint64_t E = h[0];
  if (E >= 0xffffffffull) return Status::make(SPLAT_ERR_CAPACITY, "too many tile entries for 32-bit offsets");
  const uint64_t drw = h[1];
  const uint32_t drh[2] = {(uint32_t)drw, (uint32_t)(drw >> 32)};
  SPLAT_TRY(v.gauss.ensure((size_t)std::max<uint64_t>(E, 1) * 4));
  SPLAT_TRY(launch_bin_sort(c, proj, v.entry_offset.as<uint32_t>(), n, (int64_t)E, dr, drh[0],
                            E > 0 ? drh[1] : drh[0], cam.width, cam.height, v.gauss.as<uint32_t>(), nullptr,
                            v.tile_range.as<uint32_t>()));
  SPLAT_TRY(launch_raster_fwd(c, proj, v.gauss.as<uint32_t>(), v.tile_range.as<uint32_t>(), cam.width, cam.height, bg,
                              v.image.as<float>(), v.final_t.as<float>(), v.n_contrib.as<uint32_t>(), nullptr));
  if (entries_out) *entries_out = (int64_t)E;
  return Status::ok();
}

}  // namespace splat

using namespace splat;

// Chunks of the gradient download: the projection backward and the record conversion of
// chunk i+1 run while chunk i crosses PCIe on the download stream.
constexpr int kDownloadChunks = 8;
// Steps in flight. Each slot owns its view buffers, gradient buffers and events, so step k+1
// computes while step k's gradients cross PCIe; uploads and downloads use separate streams
// (separate copy engines).
constexpr int kSlots = 2;

struct RSlot {
  ViewBuffers v;
  DevBuf pgrad, grad_planes, grad_aos;
  cudaEvent_t ev_up = nullptr, ev_img = nullptr, ev_fin = nullptr, ev_done = nullptr;
  cudaEvent_t ev_chunk[kDownloadChunks] = {};
  uint64_t ticket = 0;  // step occupying the slot; 0 when idle
  int64_t entries = 0;
};

struct splat_renderer {
  splat_ctx* ctx;
  Ctx* c;
  int64_t n = 0, cap = 0;
  int32_t sh_degree = 3;
  DevBuf planes, aos;
  RSlot slots[kSlots];
  uint64_t next_ticket = 1;
  int64_t last_entries = 0;
  cudaStream_t up = nullptr, down = nullptr;  // host->device and device->host transfers
};

namespace {
int rfail(splat_renderer* r, const Status& s) {
  r->c->last_error = s.msg;
  return s.code;
}
struct REnter {
  splat_renderer* r;
  int prev = -1;
  explicit REnter(splat_renderer* x) : r(x) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != x->c->device) cudaSetDevice(x->c->device);
    arena_reset(x->c);
  }
  ~REnter() {
    if (prev >= 0 && prev != r->c->device) cudaSetDevice(prev);
  }
};
bool cam_ok(const splat_camera* cam) {
  return cam && cam->width > 0 && cam->height > 0 && cam->width <= 65535 && cam->height <= 65535;
}

// Blocks until the slot's step has finished (its downloads included) and frees the slot.
Status retire(splat_renderer* r, RSlot& sl) {
  if (!sl.ticket) return Status::ok();
  sl.ticket = 0;
  return cuda_status(cudaEventSynchronize(sl.ev_done), "waiting for a submitted step");
}

Status retire_all(splat_renderer* r) {
  Status s = Status::ok();
  for (RSlot& sl : r->slots) {
    const Status t = retire(r, sl);
    if (s.good()) s = t;
  }
  return s;
}

// Queues one differentiable render into slot `sl`: dL/dimage up, forward, backward,
// projection backward, image and gradient records down. Returns after the queueing (the
// forward's entry-count read-back is the one host wait inside).
Status submit_backward(splat_renderer* r, RSlot& sl, const splat_camera& cam, const splat_proj_opts& o,
                       const float bg[3], const float* dimage_host, float* image_host, float* grads_host) {
  Ctx* c = r->c;
  const size_t npix = (size_t)cam.width * cam.height;
  SPLAT_TRY(sl.v.ensure(r->n, cam.width, cam.height));
  SPLAT_TRY(sl.pgrad.ensure((size_t)r->cap * 3 * 16));
  SPLAT_TRY(sl.grad_planes.ensure((size_t)r->cap * kPlanes * 16));
  if (grads_host) SPLAT_TRY(sl.grad_aos.ensure((size_t)r->cap * 59 * 4));
  // dL/dimage crosses PCIe while the forward pass runs.
  SPLAT_CUDA(cudaMemcpyAsync(sl.v.dimage.ptr, dimage_host, npix * 12, cudaMemcpyHostToDevice, r->up));
  SPLAT_CUDA(cudaEventRecord(sl.ev_up, r->up));
  SPLAT_TRY(render_view(c, r->planes.as<float>(), r->n, r->cap, cam, o, bg, sl.v, &sl.entries));
  // The image crosses PCIe while the backward pass runs.
  if (image_host) {
    SPLAT_CUDA(cudaEventRecord(sl.ev_img, c->stream));
    SPLAT_CUDA(cudaStreamWaitEvent(r->down, sl.ev_img, 0));
    SPLAT_CUDA(cudaMemcpyAsync(image_host, sl.v.image.ptr, npix * 12, cudaMemcpyDeviceToHost, r->down));
  }
  SPLAT_CUDA(cudaStreamWaitEvent(c->stream, sl.ev_up, 0));
  SPLAT_TRY(launch_fill_u32(c, sl.pgrad.ptr, (size_t)r->cap * 12, 0u));
  SPLAT_TRY(launch_raster_bwd(c, sl.v.proj.as<float>(), sl.v.gauss.as<uint32_t>(), sl.v.tile_range.as<uint32_t>(),
                              cam.width, cam.height, bg, sl.v.final_t.as<float>(), sl.v.n_contrib.as<uint32_t>(),
                              sl.v.dimage.as<float>(), sl.pgrad.as<float>(), r->cap, nullptr));
  // Projection backward, record conversion and download in chunks of Gaussians.
  const int64_t chunk = ((r->n + kDownloadChunks - 1) / kDownloadChunks + 127) / 128 * 128;
  for (int k = 0; k < kDownloadChunks; k++) {
    const int64_t i0 = (int64_t)k * chunk;
    if (i0 >= r->n) break;
    const int64_t cnt = std::min(chunk, r->n - i0);
    SPLAT_TRY(launch_project_bwd(c, r->planes.as<float>() + 4 * i0, cnt, r->cap, cam, o,
                                 sl.v.proj.as<float>() + 16 * i0, sl.pgrad.as<float>() + 4 * i0,
                                 sl.grad_planes.as<float>() + 4 * i0, nullptr, 0));
    if (grads_host) {
      SPLAT_TRY(launch_params_to_aos(c, sl.grad_planes.as<float>() + 4 * i0, cnt, r->cap,
                                     sl.grad_aos.as<float>() + 59 * i0));
      SPLAT_CUDA(cudaEventRecord(sl.ev_chunk[k], c->stream));
      SPLAT_CUDA(cudaStreamWaitEvent(r->down, sl.ev_chunk[k], 0));
      SPLAT_CUDA(cudaMemcpyAsync(grads_host + 59 * i0, sl.grad_aos.as<float>() + 59 * i0, (size_t)cnt * 59 * 4,
                                 cudaMemcpyDeviceToHost, r->down));
    }
  }
  SPLAT_CUDA(cudaEventRecord(sl.ev_fin, c->stream));
  SPLAT_CUDA(cudaStreamWaitEvent(r->down, sl.ev_fin, 0));
  SPLAT_CUDA(cudaEventRecord(sl.ev_done, r->down));
  r->last_entries = sl.entries;
  return Status::ok();
}
}  // namespace

extern "C" {

SPLAT_API int splat_renderer_create(splat_ctx* ctx, splat_renderer** out) {
  if (!ctx || !out) return SPLAT_ERR_INVALID;
  splat_renderer* r = new (std::nothrow) splat_renderer();
  if (!r) return SPLAT_ERR_INVALID;
  r->ctx = ctx;
  r->c = splat_ctx_impl(ctx);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(r->c->device);
  bool ok = cudaStreamCreateWithFlags(&r->up, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&r->down, cudaStreamNonBlocking) == cudaSuccess;
  for (RSlot& sl : r->slots) {
    for (cudaEvent_t* ev : {&sl.ev_up, &sl.ev_img, &sl.ev_fin, &sl.ev_done})
      ok = ok && cudaEventCreateWithFlags(ev, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < kDownloadChunks && ok; i++)
      ok = cudaEventCreateWithFlags(&sl.ev_chunk[i], cudaEventDisableTiming) == cudaSuccess;
  }
  cudaSetDevice(prev);
  if (!ok) {
    cudaGetLastError();
    r->c->last_error = "splat_renderer_create: stream or event creation failed";
    splat_renderer_destroy(r);
    return SPLAT_ERR_CUDA;
  }
  *out = r;
  return SPLAT_OK;
}

SPLAT_API int splat_renderer_destroy(splat_renderer* r) {
  if (!r) return SPLAT_OK;
  {
    REnter e(r);
    cudaStreamSynchronize(r->c->stream);
    if (r->up) cudaStreamSynchronize(r->up);
    if (r->down) cudaStreamSynchronize(r->down);
    for (DevBuf* b : {&r->planes, &r->aos}) b->release();
    for (RSlot& sl : r->slots) {
      sl.v.release();
      for (DevBuf* b : {&sl.pgrad, &sl.grad_planes, &sl.grad_aos}) b->release();
      for (cudaEvent_t ev : sl.ev_chunk)
        if (ev) cudaEventDestroy(ev);
      for (cudaEvent_t ev : {sl.ev_up, sl.ev_img, sl.ev_fin, sl.ev_done})
        if (ev) cudaEventDestroy(ev);
    }
    if (r->up) cudaStreamDestroy(r->up);
    if (r->down) cudaStreamDestroy(r->down);
  }
  delete r;
  return SPLAT_OK;
}

SPLAT_API int splat_renderer_set_model(splat_renderer* r, const float* aos59_host, int64_t n, int32_t sh_degree) {
  if (!r) return SPLAT_ERR_INVALID;
  if (n < 0 || (n && !aos59_host) || sh_degree < 0 || sh_degree > 3) {
    r->c->last_error = "splat_renderer_set_model: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  REnter e(r);
  Ctx* c = r->c;
  const int64_t cap = std::max<int64_t>(n, 1);
  Status s = retire_all(r);  // in-flight steps read the current model
  if (s.good()) s = r->planes.ensure((size_t)cap * kPlanes * 16);
  if (s.good()) s = r->aos.ensure((size_t)cap * 59 * 4);
  if (s.good() && n) s = cuda_status(cudaMemcpyAsync(r->aos.ptr, aos59_host, (size_t)n * 59 * 4, cudaMemcpyHostToDevice,
                                                     c->stream), "upload model");
  if (s.good()) s = launch_params_from_aos(c, r->aos.as<float>(), n, r->planes.as<float>(), cap);
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  if (!s.good()) return rfail(r, s);
  r->n = n;
  r->cap = cap;
  r->sh_degree = sh_degree;
  return SPLAT_OK;
}

SPLAT_API int splat_renderer_render(splat_renderer* r, const splat_camera* cam, const splat_proj_opts* opts,
                                    const float background[3], float* image_host) {
  if (!r) return SPLAT_ERR_INVALID;
  if (!cam_ok(cam) || !opts || !background) {
    r->c->last_error = "splat_renderer_render: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  REnter e(r);
  Ctx* c = r->c;
  splat_proj_opts o = *opts;
  o.sh_degree = r->sh_degree;  // project_all uses the model's active degree (project.rs:321-324)
  Status s = retire_all(r);
  RSlot& sl = r->slots[0];
  if (s.good()) s = render_view(c, r->planes.as<float>(), r->n, r->cap, *cam, o, background, sl.v, &sl.entries);
  if (s.good()) r->last_entries = sl.entries;
  const size_t npix = (size_t)cam->width * cam->height;
  if (s.good() && image_host)
    s = cuda_status(cudaMemcpyAsync(image_host, sl.v.image.ptr, npix * 12, cudaMemcpyDeviceToHost, c->stream),
                    "download image");
  if (s.good()) s = cuda_status(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return s.good() ? SPLAT_OK : rfail(r, s);
}

SPLAT_API int splat_renderer_submit_backward(splat_renderer* r, const splat_camera* cam, const splat_proj_opts* opts,
                                             const float background[3], const float* dimage_host, float* image_host,
                                             float* grads_aos59_host, uint64_t* ticket) {
  if (!r) return SPLAT_ERR_INVALID;
  if (!cam_ok(cam) || !opts || !background || !dimage_host || !ticket) {
    r->c->last_error = "splat_renderer_submit_backward: bad arguments";
    return SPLAT_ERR_INVALID;
  }
  *ticket = 0;
  REnter e(r);
  splat_proj_opts o = *opts;
  o.sh_degree = r->sh_degree;
  // The slot of the oldest step in flight (the next in round-robin order) is reused.
  RSlot& sl = r->slots[r->next_ticket % kSlots];
  Status s = retire(r, sl);
  if (s.good()) s = submit_backward(r, sl, *cam, o, background, dimage_host, image_host, grads_aos59_host);
  if (!s.good()) {
    // Leave nothing in flight behind an error.
    cudaStreamSynchronize(r->c->stream);
    cudaStreamSynchronize(r->up);
    cudaStreamSynchronize(r->down);
    cudaGetLastError();
    return rfail(r, s);
  }
  sl.ticket = r->next_ticket++;
  *ticket = sl.ticket;
  return SPLAT_OK;
}

SPLAT_API int splat_renderer_wait(splat_renderer* r, uint64_t ticket) {
  if (!r) return SPLAT_ERR_INVALID;
  if (ticket == 0 || ticket >= r->next_ticket) {
    r->c->last_error = "splat_renderer_wait: no such submitted step";
    return SPLAT_ERR_INVALID;
  }
  REnter e(r);
  for (RSlot& sl : r->slots)
    if (sl.ticket == ticket) {
      const Status s = retire(r, sl);
      return s.good() ? SPLAT_OK : rfail(r, s);
    }
  return SPLAT_OK;  // already retired
}

SPLAT_API int splat_renderer_render_backward(splat_renderer* r, const splat_camera* cam, const splat_proj_opts* opts,
                                             const float background[3], const float* dimage_host, float* image_host,
                                             float* grads_aos59_host) {
  uint64_t t = 0;
  const int st = splat_renderer_submit_backward(r, cam, opts, background, dimage_host, image_host, grads_aos59_host, &t);
  if (st != SPLAT_OK) return st;
  return splat_renderer_wait(r, t);
}

SPLAT_API int64_t splat_renderer_last_entries(const splat_renderer* r) { return r ? r->last_entries : -1; }

}  // extern "C"
