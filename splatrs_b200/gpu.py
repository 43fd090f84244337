"""Python mirror of the reference's hot-path API over the C ABI, on device tensors.

Function names and argument meaning follow the reference (harryprayiv/splatrs, src/):
``project_all`` (src/project.rs:320), ``bin`` (src/rasterize.rs:60), ``rasterize_forward``
(:305), ``rasterize_backward`` (:459), ``project_backward_all`` (src/project.rs:477). Device
memory comes from torch tensors (plumbing only); every computation runs in the sm_100a
kernels of libsplatrs_b200.so. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass

import torch

from . import _lib as L
from ._lib import Camera, DensifyConfig, DensifyReport, LearningRates, ProjOpts, StepInfo, TrainConfig, check

PLANES = L.PLANES
PROJ_FLOATS = L.PROJ_FLOATS


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Context:
    """A splat_ctx: device, stream and scratch arena."""

    def __init__(self, device: int = 0, stream=None):
        self.device = device
        self.lib = L.lib()
        h = C.c_void_p()
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream(device).cuda_stream
        st = self.lib.splat_ctx_create(device, C.c_void_p(s), C.byref(h))
        if st != L.SPLAT_OK:
            raise L.SplatError(st, "splat_ctx_create failed")
        self.h = h
        self._dependents = weakref.WeakSet()

    def _adopt(self, obj):
        """Renderers and trainers must be destroyed before their context."""
        self._dependents.add(obj)

    def set_stream(self, stream):
        check(self.lib.splat_ctx_set_stream(self.h, C.c_void_p(stream.cuda_stream)), self.h)

    def synchronize(self):
        check(self.lib.splat_ctx_synchronize(self.h), self.h)

    @property
    def launches(self) -> int:
        return int(self.lib.splat_ctx_launch_count(self.h))

    @property
    def scratch_info(self) -> tuple:
        """(bytes the scratch arena holds on the device, its allocation counter)."""
        out = (C.c_uint64 * 2)()
        check(self.lib.splat_ctx_scratch_info(self.h, out), self.h)
        return int(out[0]), int(out[1])

    def peak(self, unit: str) -> dict:
        """Measured throughput of 'fp32' (FMA, FLOP/s) or 'mufu' (ex2, operations/s) on this
        context's device (splat_diag_peak)."""
        ops, ms = C.c_double(), C.c_float()
        check(self.lib.splat_diag_peak(self.h, {"fp32": 0, "mufu": 1}[unit], C.byref(ops), C.byref(ms)), self.h)
        return {"ops_per_s": float(ops.value), "ms": float(ms.value)}

    @staticmethod
    def raster_candidates() -> list:
        """The supported compositing configurations (tile_w, tile_h, chunk depth, backward
        pixels per thread)."""
        lib = L.lib()
        out = (C.c_uint32 * (4 * int(lib.splat_raster_candidates(None))))()
        k = int(lib.splat_raster_candidates(out))
        return [tuple(int(v) for v in out[4 * i:4 * i + 4]) for i in range(k)]

    @property
    def raster_config(self) -> tuple:
        """(tile_w, tile_h, chunk depth, backward pixels per thread) that projection,
        binning and compositing use."""
        out = (C.c_uint32 * 4)()
        check(self.lib.splat_get_raster_config(self.h, out), self.h)
        return tuple(int(v) for v in out)

    @raster_config.setter
    def raster_config(self, cfg):
        cfg = tuple(int(v) for v in cfg)
        if len(cfg) == 3:
            cfg = cfg + (1,)
        check(self.lib.splat_set_raster_config(self.h, *cfg), self.h)

    def autotune_render(self, planes, n, cap, cam, opts, background, dimage, reps: int = 3) -> dict:
        """Times one view's render + backward under every configuration and keeps the
        fastest; returns {config: ms per pass} and the pick."""
        ms = (C.c_float * int(self.lib.splat_raster_candidates(None)))()
        picked = (C.c_uint32 * 4)()
        bgp, _keep = _bg(background)
        check(self.lib.splat_autotune_render(self.h, _ptr(planes), n, cap, C.byref(cam), C.byref(opts), bgp,
                                             _ptr(dimage), reps, ms, picked), self.h)
        cands = Context.raster_candidates()
        return {"ms": {c: float(ms[i]) for i, c in enumerate(cands)}, "picked": tuple(int(v) for v in picked)}

    def zero(self, t: torch.Tensor):
        check(self.lib.splat_zero(self.h, _ptr(t), t.numel() * t.element_size()), self.h)

    def close(self):
        if getattr(self, "h", None):
            for d in list(getattr(self, "_dependents", ())):
                d.close()
            self.lib.splat_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def empty_planes(cap: int, device="cuda") -> torch.Tensor:
    return torch.zeros(PLANES * cap * 4, dtype=torch.float32, device=device)


def params_to_planes(ctx: Context, aos59: torch.Tensor, cap: int | None = None) -> torch.Tensor:
    """Reference Gaussian records (n, 59) on the device -> parameter planes."""
    aos59 = aos59.contiguous().to(torch.float32)
    n = aos59.shape[0]
    cap = n if cap is None else cap
    planes = empty_planes(cap, aos59.device)
    check(ctx.lib.splat_params_from_aos(ctx.h, _ptr(aos59), n, _ptr(planes), cap), ctx.h)
    return planes


def planes_to_params(ctx: Context, planes: torch.Tensor, n: int, cap: int) -> torch.Tensor:
    out = torch.empty((n, 59), dtype=torch.float32, device=planes.device)
    check(ctx.lib.splat_params_to_aos(ctx.h, _ptr(planes), n, cap, _ptr(out)), ctx.h)
    return out


@dataclass
class Projection:
    """Projection records for one camera (the device form of Vec<Proj>)."""
    rec: torch.Tensor          # (n, 16) float32
    num_tiles: torch.Tensor    # (n,) int32 (uint32 values)
    depth_range: torch.Tensor  # (2,) int32 (uint32 bits)
    n: int
    width: int
    height: int

    def to_reference(self, ctx: Context) -> torch.Tensor:
        """Reference-layout Proj records (n, 15)."""
        out = torch.empty((self.n, 15), dtype=torch.float32, device=self.rec.device)
        check(ctx.lib.splat_proj_to_reference(ctx.h, _ptr(self.rec), self.n, _ptr(out)), ctx.h)
        return out


def project_all(ctx: Context, planes: torch.Tensor, n: int, cap: int, cam: Camera, opts: ProjOpts) -> Projection:
    """project_all (src/project.rs:320-330)."""
    dev = planes.device
    rec = torch.empty((n, PROJ_FLOATS), dtype=torch.float32, device=dev)
    nt = torch.empty(n, dtype=torch.int32, device=dev)
    dr = torch.empty(2, dtype=torch.int32, device=dev)
    check(ctx.lib.splat_project_fwd(ctx.h, _ptr(planes), n, cap, C.byref(cam), C.byref(opts), _ptr(rec), _ptr(nt),
                                    _ptr(dr)), ctx.h)
    return Projection(rec, nt, dr, n, cam.width, cam.height)


def proj_from_reference(ctx: Context, proj15: torch.Tensor, width: int, height: int) -> Projection:
    """Projection records from reference-layout Proj records (n, 15) on the device."""
    proj15 = proj15.contiguous().to(torch.float32)
    n = proj15.shape[0]
    dev = proj15.device
    rec = torch.empty((n, PROJ_FLOATS), dtype=torch.float32, device=dev)
    nt = torch.empty(n, dtype=torch.int32, device=dev)
    dr = torch.empty(2, dtype=torch.int32, device=dev)
    check(ctx.lib.splat_proj_from_reference(ctx.h, _ptr(proj15), n, width, height, _ptr(rec), _ptr(nt), _ptr(dr)),
          ctx.h)
    return Projection(rec, nt, dr, n, width, height)


@dataclass
class Binning:
    """Binning (src/rasterize.rs:26-39) on the device: sorted Gaussian indices per entry."""
    entry_offset: torch.Tensor  # (n + 1,)
    gauss: torch.Tensor         # (E,) Gaussian index of each sorted entry
    keys: torch.Tensor | None   # (E,) int64 (uint64 reference keys) if requested
    tile_range: torch.Tensor    # (tiles, 2)
    num_entries: int
    tiles_x: int
    tiles_y: int


def bin(ctx: Context, proj: Projection, want_keys: bool = False) -> Binning:
    """bin (src/rasterize.rs:60-128)."""
    dev = proj.rec.device
    off = torch.empty(proj.n + 1, dtype=torch.int32, device=dev)
    e = C.c_int64()
    check(ctx.lib.splat_bin_count(ctx.h, _ptr(proj.num_tiles), proj.n, _ptr(off), C.byref(e)), ctx.h)
    E = int(e.value)
    tw, th = ctx.raster_config[:2]
    tx = (proj.width + tw - 1) // tw
    ty = (proj.height + th - 1) // th
    gauss = torch.empty(max(E, 1), dtype=torch.int32, device=dev)
    keys = torch.empty(max(E, 1), dtype=torch.int64, device=dev) if want_keys else None
    tr = torch.empty((tx * ty, 2), dtype=torch.int32, device=dev)
    check(ctx.lib.splat_bin_sort(ctx.h, _ptr(proj.rec), _ptr(off), proj.n, E, _ptr(proj.depth_range), proj.width,
                                 proj.height, _ptr(gauss), _ptr(keys), _ptr(tr)), ctx.h)
    return Binning(off, gauss[:E], keys[:E] if keys is not None else None, tr, E, tx, ty)


def bin_device(ctx: Context, proj: Projection, capacity: int, scratch: torch.Tensor | None = None):
    """bin without a host read-back (splat_bin_count_device + splat_bin_sort_device).
    Returns (gauss (capacity,), tile ranges, entry count (device uint64), overflow flag
    (device), scratch); results are valid only when the flag is 0."""
    dev = proj.rec.device
    off = torch.empty(proj.n + 1, dtype=torch.int32, device=dev)
    e_dev = torch.zeros(1, dtype=torch.int64, device=dev)
    check(ctx.lib.splat_bin_count_device(ctx.h, _ptr(proj.num_tiles), proj.n, _ptr(off), _ptr(e_dev)), ctx.h)
    tw, th = ctx.raster_config[:2]
    tx = (proj.width + tw - 1) // tw
    ty = (proj.height + th - 1) // th
    need = int(ctx.lib.splat_bin_sort_device_scratch_bytes(capacity))
    if scratch is None or scratch.numel() < need:
        scratch = torch.empty(need, dtype=torch.uint8, device=dev)
    gauss = torch.empty(max(capacity, 1), dtype=torch.int32, device=dev)
    tr = torch.empty((tx * ty, 2), dtype=torch.int32, device=dev)
    flag = torch.zeros(1, dtype=torch.int32, device=dev)
    check(ctx.lib.splat_bin_sort_device(ctx.h, _ptr(proj.rec), _ptr(off), proj.n, _ptr(e_dev), capacity,
                                        _ptr(proj.depth_range), proj.width, proj.height, _ptr(scratch), _ptr(gauss),
                                        _ptr(tr), _ptr(flag)), ctx.h)
    return gauss, tr, e_dev, flag, scratch


def _bg(background):
    arr = (C.c_float * 3)(*[float(x) for x in background])
    return C.cast(arr, C.POINTER(C.c_float)), arr


@dataclass
class RasterOutput:
    """RasterOutput (src/rasterize.rs:43-50) on the device."""
    image: torch.Tensor    # (H*W*3,)
    final_t: torch.Tensor  # (H*W,)
    n_contrib: torch.Tensor  # (H*W,) int32
    pairs: torch.Tensor    # (1,) int64, evaluated (entry, pixel) pairs


def rasterize_forward(ctx: Context, proj: Projection, b: Binning, background, count_pairs: bool = True,
                      out: RasterOutput | None = None) -> RasterOutput:
    """rasterize_forward (src/rasterize.rs:305-337). `out` reuses buffers of a previous call."""
    dev = proj.rec.device
    npix = proj.width * proj.height
    if out is not None:
        image, ft, nc = out.image, out.final_t, out.n_contrib
    else:
        image = torch.empty(npix * 3, dtype=torch.float32, device=dev)
        ft = torch.empty(npix, dtype=torch.float32, device=dev)
        nc = torch.empty(npix, dtype=torch.int32, device=dev)
    pairs = torch.zeros(1, dtype=torch.int64, device=dev) if count_pairs else None
    bgp, keep = _bg(background)
    check(ctx.lib.splat_rasterize_fwd(ctx.h, _ptr(proj.rec), _ptr(b.gauss), _ptr(b.tile_range), proj.width,
                                      proj.height, bgp, _ptr(image), _ptr(ft), _ptr(nc), _ptr(pairs)), ctx.h)
    return RasterOutput(image, ft, nc, pairs)


def rasterize_backward(ctx: Context, proj: Projection, b: Binning, background, out: RasterOutput,
                       dimage: torch.Tensor, pgrad: torch.Tensor | None = None, cap: int | None = None,
                       pairs: torch.Tensor | None = None) -> torch.Tensor:
    """rasterize_backward (src/rasterize.rs:459-505). Returns the screen-space gradient
    planes (3, cap, 4): ProjGrad plus the AbsGS accumulators."""
    dev = proj.rec.device
    cap = proj.n if cap is None else cap
    if pgrad is None:
        pgrad = torch.zeros((3, cap, 4), dtype=torch.float32, device=dev)
    bgp, keep = _bg(background)
    check(ctx.lib.splat_rasterize_bwd(ctx.h, _ptr(proj.rec), _ptr(b.gauss), _ptr(b.tile_range), proj.width,
                                      proj.height, bgp, _ptr(out.final_t), _ptr(out.n_contrib),
                                      _ptr(dimage.contiguous()), _ptr(pgrad), cap, _ptr(pairs)), ctx.h)
    return pgrad


def rasterize_backward_deterministic(ctx: Context, proj: Projection, b: Binning, background, out: RasterOutput,
                                     dimage: torch.Tensor, pgrad: torch.Tensor | None = None,
                                     cap: int | None = None) -> torch.Tensor:
    """rasterize_backward (src/rasterize.rs:459-505) with the reference's own reduction
    (per-entry slots in pixel order, ordered per-Gaussian sums): the screen-space gradient
    planes (3, cap, 4), written (not accumulated), bit for bit the reference's."""
    dev = proj.rec.device
    cap = proj.n if cap is None else cap
    if pgrad is None:
        pgrad = torch.empty((3, cap, 4), dtype=torch.float32, device=dev)
    bgp, keep = _bg(background)
    check(ctx.lib.splat_rasterize_bwd_deterministic(
        ctx.h, _ptr(proj.rec), _ptr(b.gauss), _ptr(b.tile_range), _ptr(b.entry_offset), proj.n, b.num_entries,
        proj.width, proj.height, bgp, _ptr(out.final_t), _ptr(out.n_contrib), _ptr(dimage.contiguous()),
        _ptr(pgrad), cap), ctx.h)
    return pgrad


def pgrad_to_reference(pgrad: torch.Tensor, n: int):
    """Screen-space gradient planes -> (ProjGrad (n, 9), abs (n, 2)) in the reference layout."""
    g0, g1, g2 = pgrad[0, :n], pgrad[1, :n], pgrad[2, :n]
    grads = torch.stack([g0[:, 0], g0[:, 1], g0[:, 2], g0[:, 3], g1[:, 0], g1[:, 1], g1[:, 2], g1[:, 3], g2[:, 0]], 1)
    absg = g2[:, 1:3]
    return grads, absg


def pgrad_from_reference(grads9: torch.Tensor, abs2: torch.Tensor | None = None, cap: int | None = None):
    n = grads9.shape[0]
    cap = n if cap is None else cap
    p = torch.zeros((3, cap, 4), dtype=torch.float32, device=grads9.device)
    p[0, :n] = grads9[:, 0:4]
    p[1, :n] = grads9[:, 4:8]
    p[2, :n, 0] = grads9[:, 8]
    if abs2 is not None:
        p[2, :n, 1:3] = abs2
    return p


def project_backward_all(ctx: Context, planes: torch.Tensor, n: int, cap: int, cam: Camera, opts: ProjOpts,
                         proj: Projection, pgrad: torch.Tensor, stats: torch.Tensor | None = None,
                         absgrad: bool = False) -> torch.Tensor:
    """project_backward_all (src/project.rs:477-493); returns gradient planes.

    With ``stats`` (3 * cap 32-bit words: grad_accum f32, denom u32, max_radii u32) it also
    performs DensifyStats::accumulate (src/densify.rs:36-60)."""
    out = torch.empty(PLANES * cap * 4, dtype=torch.float32, device=planes.device)
    check(ctx.lib.splat_project_bwd(ctx.h, _ptr(planes), n, cap, C.byref(cam), C.byref(opts), _ptr(proj.rec),
                                    _ptr(pgrad), _ptr(out), _ptr(stats), int(bool(absgrad))), ctx.h)
    return out


class Renderer:
    """splat_renderer: a device-resident model driven with host (numpy) buffers.

    ``render`` is render::render (src/render.rs:14-23); ``render_backward`` runs the chain
    of examples/profile.rs:34-52 and returns the parameter gradients as reference records."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        check(self.lib.splat_renderer_create(ctx.h, C.byref(h)), ctx.h)
        self.h = h
        self.n = 0
        ctx._adopt(self)

    def set_model(self, aos59, sh_degree: int):
        import numpy as np
        a = np.ascontiguousarray(aos59, np.float32).reshape(-1, 59)
        self.n = a.shape[0]
        check(self.lib.splat_renderer_set_model(self.h, a.ctypes.data_as(C.c_void_p), self.n, sh_degree), self.ctx.h)

    def render(self, cam: Camera, opts: ProjOpts, background, image_out=None):
        import numpy as np
        if image_out is None:
            image_out = np.empty(cam.width * cam.height * 3, np.float32)
        bgp, keep = _bg(background)
        check(self.lib.splat_renderer_render(self.h, C.byref(cam), C.byref(opts), bgp,
                                             image_out.ctypes.data_as(C.c_void_p)), self.ctx.h)
        return image_out

    def render_backward(self, cam: Camera, opts: ProjOpts, background, dimage, image_out=None, grads_out=None,
                        want_image=True, want_grads=True):
        import numpy as np
        if want_image and image_out is None:
            image_out = np.empty(cam.width * cam.height * 3, np.float32)
        if want_grads and grads_out is None:
            grads_out = np.empty((self.n, 59), np.float32)
        d = np.ascontiguousarray(dimage, np.float32)
        bgp, keep = _bg(background)
        check(self.lib.splat_renderer_render_backward(
            self.h, C.byref(cam), C.byref(opts), bgp, d.ctypes.data_as(C.c_void_p),
            image_out.ctypes.data_as(C.c_void_p) if want_image else None,
            grads_out.ctypes.data_as(C.c_void_p) if want_grads else None), self.ctx.h)
        return image_out, grads_out

    def submit_backward(self, cam: Camera, opts: ProjOpts, background, dimage, image_out, grads_out) -> int:
        """Queues render_backward into caller-owned host buffers (numpy or pinned torch CPU
        tensors, None to skip an output) and returns a ticket for ``wait``. The buffers
        belong to the step until its wait returns."""
        def ptr(a):
            if a is None:
                return None
            return C.c_void_p(a.data_ptr()) if hasattr(a, "data_ptr") else a.ctypes.data_as(C.c_void_p)
        bgp, keep = _bg(background)
        t = C.c_uint64()
        check(self.lib.splat_renderer_submit_backward(self.h, C.byref(cam), C.byref(opts), bgp, ptr(dimage),
                                                      ptr(image_out), ptr(grads_out), C.byref(t)), self.ctx.h)
        return int(t.value)

    def wait(self, ticket: int):
        check(self.lib.splat_renderer_wait(self.h, ticket), self.ctx.h)

    @property
    def last_entries(self) -> int:
        return int(self.lib.splat_renderer_last_entries(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.splat_renderer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def photometric_loss(ctx: Context, pred: torch.Tensor, target: torch.Tensor, width: int, height: int,
                     lambda_dssim: float):
    """photometric_loss (src/loss.rs:137-171): returns (loss, mean ssim, psnr) as a device
    tensor of 3 floats and the gradient w.r.t. pred. `target` may be uint8 (converted as
    View::to_real, src/dataset.rs:23-25) or float32."""
    pred = pred.contiguous()
    target = target.contiguous()
    is_u8 = target.dtype == torch.uint8
    grad = torch.empty_like(pred)
    out = torch.empty(3, dtype=torch.float32, device=pred.device)
    check(ctx.lib.splat_loss_fwd_bwd(ctx.h, _ptr(pred), _ptr(target), int(is_u8), width, height, float(lambda_dssim),
                                     _ptr(grad), _ptr(out)), ctx.h)
    return out, grad


def adam_step(ctx: Context, planes, grads, m, v, n: int, cap: int, step: int, lr: LearningRates):
    """Adam::step (src/adam.rs:77-161) in place; `step` is the count after the increment."""
    check(ctx.lib.splat_adam_step(ctx.h, _ptr(planes), _ptr(grads), _ptr(m), _ptr(v), n, cap, step, C.byref(lr)),
          ctx.h)


def params_to_bf16(ctx: Context, planes, n: int, cap: int) -> torch.Tensor:
    """BF16 render copy of parameter planes 1..14 (splat_params_to_bf16)."""
    out = torch.empty((PLANES - 1) * cap * 4, dtype=torch.bfloat16, device=planes.device)
    check(ctx.lib.splat_params_to_bf16(ctx.h, _ptr(planes), n, cap, _ptr(out)), ctx.h)
    return out


def project_all_bf16(ctx: Context, planes, bf16, n: int, cap: int, cam: Camera, opts: ProjOpts) -> Projection:
    """project_all reading quaternion, log-scales and SH from the BF16 copy."""
    dev = planes.device
    rec = torch.empty((n, PROJ_FLOATS), dtype=torch.float32, device=dev)
    nt = torch.empty(n, dtype=torch.int32, device=dev)
    dr = torch.empty(2, dtype=torch.int32, device=dev)
    check(ctx.lib.splat_project_fwd_bf16(ctx.h, _ptr(planes), _ptr(bf16), n, cap, C.byref(cam), C.byref(opts),
                                         _ptr(rec), _ptr(nt), _ptr(dr)), ctx.h)
    return Projection(rec, nt, dr, n, cam.width, cam.height)


def project_backward_adam(ctx: Context, planes, m, v, n: int, cap: int, cam: Camera, opts: ProjOpts,
                          proj: Projection, pgrad, step: int, lr: LearningRates, stats=None, absgrad=False,
                          bf16=None):
    """project_backward_all (src/project.rs:477-493) fused with Adam::step
    (src/adam.rs:77-161): planes, m and v updated in place; `step` is the count after the
    increment."""
    check(ctx.lib.splat_project_bwd_adam(ctx.h, _ptr(planes), _ptr(m), _ptr(v), n, cap, C.byref(cam), C.byref(opts),
                                         _ptr(proj.rec), _ptr(pgrad), _ptr(stats), int(bool(absgrad)), step,
                                         C.byref(lr), _ptr(bf16)), ctx.h)


def densify_and_prune(ctx: Context, planes, m, v, n: int, cap: int, stats, cfg: DensifyConfig, extent: float,
                      rng_state: int, cap_out: int | None = None):
    """densify_and_prune (src/densify.rs:125-221). Returns (planes, m, v, report, rng_state)."""
    cap_out = cap_out if cap_out is not None else max(1, n * (2 + cfg.split_children))
    po = torch.zeros(PLANES * cap_out * 4, dtype=torch.float32, device=planes.device)
    mo = torch.zeros_like(po)
    vo = torch.zeros_like(po)
    st = C.c_uint64(rng_state)
    rep = DensifyReport()
    check(ctx.lib.splat_densify(ctx.h, _ptr(planes), _ptr(m), _ptr(v), n, cap, _ptr(stats), C.byref(cfg),
                                float(extent), C.byref(st), _ptr(po), _ptr(mo), _ptr(vo), cap_out, C.byref(rep)), ctx.h)
    return po, mo, vo, rep, int(st.value), cap_out


def reset_opacity(ctx: Context, planes, m, v, n: int, max_alpha: float = 0.01):
    """reset_opacity (src/densify.rs:224-230) in place."""
    check(ctx.lib.splat_reset_opacity(ctx.h, _ptr(planes), _ptr(m), _ptr(v), n, float(max_alpha)), ctx.h)


class Trainer:
    """train::train (src/train.rs:161-306) on the device, one iteration per step()."""

    def __init__(self, ctx: Context, init_params, extent: float, views, **cfg):
        import numpy as np
        self.ctx = ctx
        self.lib = ctx.lib
        self.cfg = TrainConfig.make(**cfg)
        h = C.c_void_p()
        check(self.lib.splat_trainer_create(ctx.h, C.byref(self.cfg), float(extent), C.byref(h)), ctx.h)
        self.h = h
        ctx._adopt(self)
        p = np.ascontiguousarray(init_params, np.float32).reshape(-1, 59)
        check(self.lib.splat_trainer_set_model(self.h, p.ctypes.data_as(C.c_void_p), p.shape[0]), ctx.h)
        self._nviews = 0
        for cam, rgb in views:
            c = cam if isinstance(cam, Camera) else Camera.from_record(cam)
            r = np.ascontiguousarray(rgb, np.uint8)
            check(self.lib.splat_trainer_add_view(self.h, C.byref(c), r.ctypes.data_as(C.c_void_p)), ctx.h)
            self._nviews += 1
        check(self.lib.splat_trainer_start(self.h), ctx.h)

    def step(self) -> dict:
        info = StepInfo()
        check(self.lib.splat_trainer_step(self.h, C.byref(info)), self.ctx.h)
        return info.as_dict()

    def get_mlp(self):
        """The trainer's densification network parameters (numpy float32)."""
        import numpy as np
        out = np.zeros(int(self.lib.splat_mlp_num_params()), np.float32)
        check(self.lib.splat_trainer_get_mlp(self.h, out.ctypes.data_as(C.c_void_p)), self.ctx.h)
        return out

    def set_mlp(self, theta):
        import numpy as np
        a = np.ascontiguousarray(theta, np.float32)
        check(self.lib.splat_trainer_set_mlp(self.h, a.ctypes.data_as(C.c_void_p)), self.ctx.h)

    def mlp_stats(self) -> dict:
        out = (C.c_uint64 * 9)()
        check(self.lib.splat_trainer_mlp_stats(self.h, out), self.ctx.h)
        keys = ("events", "records", "label_keep", "label_densify", "label_prune", "adam_steps", "heldout_net",
                "heldout_rule", "heldout_records")
        return dict(zip(keys, [int(v) for v in out]))

    def evaluate(self) -> dict:
        """evaluate (src/train.rs:309-321) on the device over the training views: mean PSNR,
        and loss, SSIM and PSNR per view."""
        import numpy as np
        nv = self._nviews
        per = np.zeros((max(nv, 1), 3), np.float32)
        mean = C.c_double()
        check(self.lib.splat_trainer_evaluate(self.h, per.ctypes.data_as(C.c_void_p), C.byref(mean)), self.ctx.h)
        per = per[:nv]
        return {"psnr": float(mean.value), "ssim": float(per[:, 1].mean()) if nv else float("nan"),
                "per_view": per}

    def tuning(self) -> dict:
        """The autotuner's last timings (ms per render pass per configuration), the
        configuration in use and how many tunings ran."""
        ms = (C.c_float * int(self.lib.splat_raster_candidates(None)))()
        picked = (C.c_uint32 * 4)()
        tunes = C.c_uint32()
        check(self.lib.splat_trainer_tuning(self.h, ms, picked, C.byref(tunes)), self.ctx.h)
        cands = Context.raster_candidates()
        return {"ms": {c: float(ms[i]) for i, c in enumerate(cands)}, "picked": tuple(int(v) for v in picked),
                "tunes": int(tunes.value)}

    def run(self, iterations: int) -> dict:
        """``iterations`` steps in one call, queued ahead of the device; info of the last."""
        info = StepInfo()
        check(self.lib.splat_trainer_run(self.h, iterations, C.byref(info)), self.ctx.h)
        return info.as_dict()

    @property
    def count(self) -> int:
        return int(self.lib.splat_trainer_count(self.h))

    @property
    def sh_degree(self) -> int:
        return int(self.lib.splat_trainer_sh_degree(self.h))

    def model(self):
        import numpy as np
        out = np.empty((self.count, 59), np.float32)
        check(self.lib.splat_trainer_get_model(self.h, out.ctypes.data_as(C.c_void_p)), self.ctx.h)
        return out

    def moments(self):
        """Adam's first and second moments, (count, 59) each (numpy float32)."""
        import numpy as np
        m = np.empty((self.count, 59), np.float32)
        v = np.empty((self.count, 59), np.float32)
        check(self.lib.splat_trainer_get_moments(self.h, m.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p)),
              self.ctx.h)
        return m, v

    def render(self, cam):
        import numpy as np
        c = cam if isinstance(cam, Camera) else Camera.from_record(cam)
        out = np.empty(c.width * c.height * 3, np.float32)
        check(self.lib.splat_trainer_render(self.h, C.byref(c), out.ctypes.data_as(C.c_void_p)), self.ctx.h)
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.splat_trainer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ply_read(ctx: Context, path: str, cap: int | None = None):
    """ply::read (src/ply.rs:73-181) into parameter planes: returns (planes, n, sh_degree)."""
    n = C.c_int64()
    d = C.c_int32()
    check(ctx.lib.splat_ply_read_header(ctx.h, path.encode(), C.byref(n), C.byref(d)), ctx.h)
    cap = max(1, n.value if cap is None else cap)
    planes = empty_planes(cap, torch.device("cuda", ctx.device))
    check(ctx.lib.splat_ply_read(ctx.h, path.encode(), _ptr(planes), cap, C.byref(n), C.byref(d)), ctx.h)
    return planes, int(n.value), int(d.value), cap


def ply_write(ctx: Context, path: str, planes: torch.Tensor, n: int, cap: int, sh_degree: int):
    """ply::write (src/ply.rs:19-69) from parameter planes."""
    check(ctx.lib.splat_ply_write(ctx.h, path.encode(), _ptr(planes), n, cap, sh_degree), ctx.h)


def mean_nn_dist2(ctx: Context, points: torch.Tensor) -> torch.Tensor:
    """mean_nn_dist2 (src/model.rs:128-186) on device points (n, 3) float32."""
    pts = points.contiguous().to(torch.float32)
    out = torch.empty(pts.shape[0], dtype=torch.float64, device=pts.device)
    check(ctx.lib.splat_mean_nn_dist2(ctx.h, _ptr(pts), pts.shape[0], _ptr(out)), ctx.h)
    return out


def init_from_points(ctx: Context, points, rgb, cap: int | None = None) -> torch.Tensor:
    """Model::from_points (src/model.rs:77-104): host points (n, 3) float32 and colours
    (n, 3) uint8 -> parameter planes of capacity cap."""
    import numpy as np
    p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    c = np.ascontiguousarray(rgb, np.uint8).reshape(-1, 3)
    n = p.shape[0]
    cap = max(1, n if cap is None else cap)
    planes = empty_planes(cap, torch.device("cuda", ctx.device))
    check(ctx.lib.splat_init_from_points(ctx.h, p.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p), n,
                                         _ptr(planes), cap), ctx.h)
    return planes


def diag_mbarrier_wait(ctx: Context, limit: int, arrive: bool) -> None:
    """splat_diag_mbarrier_wait: one bounded mbarrier wait of `limit` tries through the
    tensor-core kernels' wait and error word; raises SplatError with SPLAT_ERR_TIMEOUT when
    it ran out (nothing arrived)."""
    check(ctx.lib.splat_diag_mbarrier_wait(ctx.h, int(limit), int(bool(arrive))), ctx.h)


def mlp_forward(ctx: Context, x: torch.Tensor, theta: torch.Tensor, tcgen05: bool = False) -> torch.Tensor:
    """Learned-densification network: probabilities (n, 3) of feature rows (n, 16); with
    `tcgen05` on the 5th-generation tensor cores (accumulators in tensor memory)."""
    x = x.contiguous().float()
    prob = torch.empty((x.shape[0], 3), dtype=torch.float32, device=x.device)
    fn = ctx.lib.splat_mlp_forward_tc if tcgen05 else ctx.lib.splat_mlp_forward
    check(fn(ctx.h, _ptr(x), x.shape[0], _ptr(theta), _ptr(prob)), ctx.h)
    return prob


def mlp_grad(ctx: Context, x, y, w, theta, grad=None, tcgen05: bool = False):
    """Gradient of the weighted mean cross-entropy (added into `grad` when given); with
    `tcgen05` on the 5th-generation tensor cores."""
    x = x.contiguous().float()
    y = y.contiguous().to(torch.int32)
    w = w.contiguous().float()
    if grad is None:
        grad = torch.zeros(int(ctx.lib.splat_mlp_num_params()), dtype=torch.float32, device=x.device)
    scale = 1.0 / float(w.sum().item())
    fn = ctx.lib.splat_mlp_grad_tc if tcgen05 else ctx.lib.splat_mlp_grad
    check(fn(ctx.h, _ptr(x), _ptr(y), _ptr(w), x.shape[0], scale, _ptr(theta), _ptr(grad)), ctx.h)
    return grad
