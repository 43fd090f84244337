// Host-side launchers of the device stages; each returns a Status and launches on the
// context stream.
#pragma once
#include "common.cuh"

namespace splat {

Status launch_params_from_aos(Ctx* c, const float* aos, int64_t n, float* planes, int64_t cap);
Status launch_params_to_aos(Ctx* c, const float* planes, int64_t n, int64_t cap, float* aos);

Status launch_project_fwd(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                          const splat_proj_opts& opts, float* proj, uint32_t* num_tiles, uint32_t* depth_range);
Status launch_proj_from_reference(Ctx* c, const float* p15, int64_t n, uint32_t width, uint32_t height, float* proj,
                                  uint32_t* num_tiles, uint32_t* depth_range);
Status launch_proj_to_reference(Ctx* c, const float* proj, int64_t n, float* p15);
Status launch_project_bwd(Ctx* c, const float* planes, int64_t n, int64_t cap, const splat_camera& cam,
                          const splat_proj_opts& opts, const float* proj, const float* pgrad, float* out,
                          void* stats, int absgrad);

Status launch_scan_u32(Ctx* c, const uint32_t* in, int64_t n, uint32_t* out, int write_total, uint64_t* total_dev);
Status launch_bin_sort(Ctx* c, const float* proj, const uint32_t* entry_offset, int64_t n, int64_t E,
                       const uint32_t* depth_range_dev, uint32_t depth_min, uint32_t depth_max, uint32_t width,
                       uint32_t height, uint32_t* gauss_out, uint64_t* keys_out, uint32_t* ranges);

Status launch_raster_fwd(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges, uint32_t width,
                         uint32_t height, const float bg[3], float* image, float* final_t, uint32_t* n_contrib,
                         uint64_t* pairs);
Status launch_raster_bwd(Ctx* c, const float* proj, const uint32_t* gauss, const uint32_t* ranges, uint32_t width,
                         uint32_t height, const float bg[3], const float* final_t, const uint32_t* n_contrib,
                         const float* dimage, float* pgrad, int64_t cap, uint64_t* pairs);

}  // namespace splat
