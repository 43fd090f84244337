"""ctypes bindings for the CPU oracle (``oracle/_build/liboracle.so``).

TEST INFRASTRUCTURE ONLY: the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use this module as the checker. The product package never imports it.

Each function mirrors one function of the reference implementation (harryprayiv/splatrs,
``src/``) and names it; array layouts are documented in ``oracle_capi.cpp``. ``dtype``
selects the f32 build (the reference's default) or the f64 build (its ``--features f64``
gradient-check oracle).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

NUM_PARAMS = 59
PROJ_FIELDS = 15
CAM_FIELDS = 18


SOURCES = ("oracle_capi.cpp", "splat_oracle.hpp", "splat_oracle_train.hpp", "Makefile",
           os.path.join("..", "splatrs_b200", "csrc", "crmath.h"))


def stale() -> bool:
    """The library is missing or older than one of its sources."""
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t for f in SOURCES)


def build(force: bool = False, if_stale: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off): always with `force`,
    when out of date with `if_stale`, else only when the library is missing."""
    if force or not os.path.exists(LIB_PATH) or (if_stale and stale()):
        subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []), check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _declare(L):
    vp, i64, u32, u64, ci, cd, cf = C.c_void_p, C.c_int64, C.c_uint32, C.c_uint64, C.c_int, C.c_double, C.c_float
    for s, R in (("f", cf), ("d", cd)):
        f = getattr(L, f"ora_project_all_{s}"); f.argtypes = [vp, i64, vp, R, R, ci, ci, vp]; f.restype = None
        f = getattr(L, f"ora_project_backward_all_{s}"); f.argtypes = [vp, i64, vp, R, R, ci, ci, vp, vp]; f.restype = None
        f = getattr(L, f"ora_bin_{s}"); f.argtypes = [vp, i64, u32, u32]; f.restype = vp
        f = getattr(L, f"ora_rasterize_forward_{s}"); f.argtypes = [vp, i64, vp, u32, u32, vp, vp, vp, vp, vp]; f.restype = None
        f = getattr(L, f"ora_rasterize_backward_{s}"); f.argtypes = [vp, i64, vp, u32, u32, vp, vp, vp, vp, vp, vp, vp]; f.restype = None
        f = getattr(L, f"ora_naive_render_{s}"); f.argtypes = [vp, i64, u32, u32, vp, vp]; f.restype = None
        f = getattr(L, f"ora_photometric_loss_{s}"); f.argtypes = [vp, vp, i64, i64, R, vp]; f.restype = R
        f = getattr(L, f"ora_ssim_with_grad_{s}"); f.argtypes = [vp, vp, i64, i64, vp]; f.restype = R
        f = getattr(L, f"ora_blur_{s}"); f.argtypes = [vp, i64, i64, i64, vp]; f.restype = None
        f = getattr(L, f"ora_psnr_{s}"); f.argtypes = [vp, vp, i64]; f.restype = R
        f = getattr(L, f"ora_adam_step_{s}"); f.argtypes = [vp, vp, vp, vp, i64, u64, vp]; f.restype = u64
        f = getattr(L, f"ora_densify_accumulate_{s}"); f.argtypes = [vp, vp, vp, i64, u32, u32, vp, vp, vp]; f.restype = None
        f = getattr(L, f"ora_densify_{s}")
        f.argtypes = [vp, vp, vp, i64, vp, vp, vp, R, R, R, ci, R, i64, ci, R, vp, i64, vp, vp, vp, vp]
        f.restype = i64
        f = getattr(L, f"ora_reset_opacity_{s}"); f.argtypes = [vp, vp, vp, i64, R]; f.restype = None
        f = getattr(L, f"ora_from_points_{s}"); f.argtypes = [vp, vp, i64, vp]; f.restype = None
        f = getattr(L, f"ora_look_at_{s}"); f.argtypes = [u32, u32, R, R, vp, vp, vp, vp]; f.restype = None
        f = getattr(L, f"ora_scene_extent_{s}"); f.argtypes = [vp, i64]; f.restype = R
        f = getattr(L, f"ora_sh_basis_{s}"); f.argtypes = [ci, vp, vp]; f.restype = None
        f = getattr(L, f"ora_sh_basis_grad_{s}"); f.argtypes = [ci, vp, vp]; f.restype = None
        f = getattr(L, f"ora_quat_to_mat_{s}"); f.argtypes = [vp, vp]; f.restype = None
        f = getattr(L, f"ora_sigmoid_{s}"); f.argtypes = [R]; f.restype = R
        f = getattr(L, f"ora_inverse_sigmoid_{s}"); f.argtypes = [R]; f.restype = R
    L.ora_threads.restype = ci
    L.ora_last_passed_pairs.argtypes = [vp]
    L.ora_last_passed_pairs.restype = None
    L.ora_set_threads.argtypes = [ci]
    L.ora_set_cr_math.argtypes = [ci]
    for nm in ("ora_expf", "ora_logf", "ora_expf_cr", "ora_logf_cr"):
        getattr(L, nm).argtypes = [cf]
        getattr(L, nm).restype = cf
    L.ora_binning_free.argtypes = [vp]
    L.ora_binning_num_entries.argtypes = [vp]; L.ora_binning_num_entries.restype = i64
    L.ora_binning_get.argtypes = [vp, vp, vp, vp, vp, vp]
    L.ora_mean_nn_dist2.argtypes = [vp, i64, vp]
    L.ora_splitmix_next.argtypes = [vp]; L.ora_splitmix_next.restype = u64
    L.ora_splitmix_normal.argtypes = [vp]; L.ora_splitmix_normal.restype = cd
    L.ora_splitmix_normals.argtypes = [vp, i64, vp]; L.ora_splitmix_normals.restype = None
    L.ora_train_config_fields.restype = C.c_char_p
    L.ora_trainer_new.argtypes = [vp, i64, cf, vp]; L.ora_trainer_new.restype = vp
    L.ora_trainer_add_view.argtypes = [vp, vp, vp]
    L.ora_trainer_start.argtypes = [vp]
    L.ora_trainer_step.argtypes = [vp, vp]
    L.ora_trainer_count.argtypes = [vp]; L.ora_trainer_count.restype = i64
    L.ora_trainer_sh_degree.argtypes = [vp]; L.ora_trainer_sh_degree.restype = ci
    L.ora_trainer_get_model.argtypes = [vp, vp]
    L.ora_trainer_render.argtypes = [vp, vp, vp]
    L.ora_trainer_free.argtypes = [vp]


def _sfx(dtype):
    dtype = np.dtype(dtype)
    if dtype == np.float32:
        return "f", np.float32
    if dtype == np.float64:
        return "d", np.float64
    raise TypeError(dtype)


def _arr(a, dt, shape_tail=None):
    a = np.ascontiguousarray(a, dtype=dt)
    if shape_tail is not None:
        a = a.reshape(-1, shape_tail)
    return a


def set_threads(n: int) -> None:
    lib().ora_set_threads(int(n))


def threads() -> int:
    return lib().ora_threads()


def set_cr_math(on: bool) -> None:
    """Use the correctly rounded exp/log (as the CUDA kernels do) instead of the host libm."""
    lib().ora_set_cr_math(1 if on else 0)


# --- camera.rs -------------------------------------------------------------------------
def look_at(width, height, fx, fy, eye, target, up, dtype=np.float32):
    """Camera::look_at (src/camera.rs:66-93); returns the 18-value camera record."""
    s, dt = _sfx(dtype)
    out = np.zeros(CAM_FIELDS, dt)
    getattr(lib(), f"ora_look_at_{s}")(width, height, fx, fy, _p(_arr(eye, dt)), _p(_arr(target, dt)),
                                       _p(_arr(up, dt)), _p(out))
    return out


def scene_extent(cams, dtype=np.float32):
    """scene_extent (src/camera.rs:99-118)."""
    s, dt = _sfx(dtype)
    c = _arr(cams, dt, CAM_FIELDS)
    return float(getattr(lib(), f"ora_scene_extent_{s}")(_p(c), c.shape[0]))


# --- sh.rs, math.rs --------------------------------------------------------------------
def sh_basis(degree, d, dtype=np.float64):
    s, dt = _sfx(dtype)
    out = np.zeros(16, dt)
    getattr(lib(), f"ora_sh_basis_{s}")(degree, _p(_arr(d, dt)), _p(out))
    return out


def sh_basis_grad(degree, d, dtype=np.float64):
    s, dt = _sfx(dtype)
    out = np.zeros(48, dt)
    getattr(lib(), f"ora_sh_basis_grad_{s}")(degree, _p(_arr(d, dt)), _p(out))
    return out.reshape(16, 3)


def quat_to_mat(q, dtype=np.float64):
    s, dt = _sfx(dtype)
    out = np.zeros(9, dt)
    getattr(lib(), f"ora_quat_to_mat_{s}")(_p(_arr(q, dt)), _p(out))
    return out.reshape(3, 3)


def sigmoid(x, dtype=np.float32):
    s, _ = _sfx(dtype)
    return getattr(lib(), f"ora_sigmoid_{s}")(x)


def inverse_sigmoid(x, dtype=np.float32):
    s, _ = _sfx(dtype)
    return getattr(lib(), f"ora_inverse_sigmoid_{s}")(x)


# --- project.rs ------------------------------------------------------------------------
def project_all(params, cam, near=0.2, eps2d=0.3, antialias=False, sh_degree=3, dtype=np.float32):
    """project_all (src/project.rs:320-330); returns (n, 15) Proj records."""
    s, dt = _sfx(dtype)
    p = _arr(params, dt, NUM_PARAMS)
    out = np.zeros((p.shape[0], PROJ_FIELDS), dt)
    getattr(lib(), f"ora_project_all_{s}")(_p(p), p.shape[0], _p(_arr(cam, dt)), near, eps2d,
                                           int(antialias), int(sh_degree), _p(out))
    return out


def project_backward_all(params, cam, grads9, near=0.2, eps2d=0.3, antialias=False, sh_degree=3,
                         dtype=np.float32):
    """project_backward_all (src/project.rs:477-493); returns (n, 59) gradient records."""
    s, dt = _sfx(dtype)
    p = _arr(params, dt, NUM_PARAMS)
    g = _arr(grads9, dt, 9)
    out = np.zeros_like(p)
    getattr(lib(), f"ora_project_backward_all_{s}")(_p(p), p.shape[0], _p(_arr(cam, dt)), near, eps2d,
                                                    int(antialias), int(sh_degree), _p(g), _p(out))
    return out


# --- rasterize.rs ----------------------------------------------------------------------
class Binning:
    """Binning (src/rasterize.rs:26-39) held in oracle memory."""

    def __init__(self, handle, n_gauss, width, height):
        self.h = handle
        self.n_gauss = n_gauss
        self.width, self.height = width, height
        self.tiles_x = (width + 15) // 16
        self.tiles_y = (height + 15) // 16
        self.num_entries = lib().ora_binning_num_entries(handle)

    def arrays(self):
        e = self.num_entries
        keys = np.zeros(e, np.uint64)
        entries = np.zeros(e, np.uint32)
        eg = np.zeros(e, np.uint32)
        off = np.zeros(self.n_gauss + 1, np.uint32)
        tr = np.zeros((self.tiles_x * self.tiles_y, 2), np.uint32)
        lib().ora_binning_get(self.h, _p(keys), _p(entries), _p(eg), _p(off), _p(tr))
        return dict(keys=keys, entries=entries, entry_gaussian=eg, entry_offset=off, tile_range=tr)

    def __del__(self):
        try:
            if self.h:
                lib().ora_binning_free(self.h)
        except Exception:
            pass


def bin(projs, width, height, dtype=np.float32):
    """bin (src/rasterize.rs:60-128)."""
    s, dt = _sfx(dtype)
    p = _arr(projs, dt, PROJ_FIELDS)
    h = getattr(lib(), f"ora_bin_{s}")(_p(p), p.shape[0], width, height)
    if not h:
        raise ValueError("projection tile rectangle exceeds the tile grid")
    return Binning(h, p.shape[0], width, height)


def rasterize_forward(projs, binning, width, height, background, dtype=np.float32):
    """rasterize_forward (src/rasterize.rs:305-337); returns (image, final_t, n_contrib, pairs)."""
    s, dt = _sfx(dtype)
    p = _arr(projs, dt, PROJ_FIELDS)
    img = np.zeros(width * height * 3, dt)
    ft = np.zeros(width * height, dt)
    nc = np.zeros(width * height, np.uint32)
    pairs = np.zeros(1, np.uint64)
    getattr(lib(), f"ora_rasterize_forward_{s}")(_p(p), p.shape[0], binning.h, width, height,
                                                 _p(_arr(background, dt)), _p(img), _p(ft), _p(nc), _p(pairs))
    return img, ft, nc, int(pairs[0])


def rasterize_backward(projs, binning, width, height, background, final_t, n_contrib, dimage, dtype=np.float32):
    """rasterize_backward (src/rasterize.rs:459-505); returns (grads (n,9), abs (n,2), pairs)."""
    s, dt = _sfx(dtype)
    p = _arr(projs, dt, PROJ_FIELDS)
    n = p.shape[0]
    g = np.zeros((n, 9), dt)
    a = np.zeros((n, 2), dt)
    pairs = np.zeros(1, np.uint64)
    getattr(lib(), f"ora_rasterize_backward_{s}")(
        _p(p), n, binning.h, width, height, _p(_arr(background, dt)), _p(_arr(final_t, dt)),
        _p(np.ascontiguousarray(n_contrib, np.uint32)), _p(_arr(dimage, dt)), _p(g), _p(a), _p(pairs))
    return g, a, int(pairs[0])


def splitmix_normals(state, count):
    """`count` normals of the shared SplitMix64 generator; `state` (np.uint64 array of
    one) advances as by `count` single draws."""
    out = np.zeros(count, np.float64)
    lib().ora_splitmix_normals(_p(state), count, _p(out))
    return out


def last_passed_pairs():
    """(forward, backward) pairs that passed the alpha threshold in the last
    rasterize_forward / rasterize_backward call: the unit of the reference's published
    per-core cost (README.md:153)."""
    out = np.zeros(2, np.uint64)
    lib().ora_last_passed_pairs(_p(out))
    return int(out[0]), int(out[1])


def naive_render(projs, width, height, background, dtype=np.float32):
    """The per-pixel compositor of tests/pipeline.rs:134-186."""
    s, dt = _sfx(dtype)
    p = _arr(projs, dt, PROJ_FIELDS)
    img = np.zeros(width * height * 3, dt)
    getattr(lib(), f"ora_naive_render_{s}")(_p(p), p.shape[0], width, height, _p(_arr(background, dt)), _p(img))
    return img


# --- loss.rs ---------------------------------------------------------------------------
def photometric_loss(pred, target, width, height, lam, dtype=np.float32):
    """photometric_loss (src/loss.rs:137-171); returns (loss, grad)."""
    s, dt = _sfx(dtype)
    x = _arr(pred, dt).ravel()
    y = _arr(target, dt).ravel()
    g = np.zeros_like(x)
    loss = getattr(lib(), f"ora_photometric_loss_{s}")(_p(x), _p(y), width, height, lam, _p(g))
    return float(loss), g


def ssim_with_grad(x, y, width, height, dtype=np.float32):
    """ssim_with_grad (src/loss.rs:75-134); returns (mean ssim, grad)."""
    s, dt = _sfx(dtype)
    x = _arr(x, dt).ravel()
    y = _arr(y, dt).ravel()
    g = np.zeros_like(x)
    v = getattr(lib(), f"ora_ssim_with_grad_{s}")(_p(x), _p(y), width, height, _p(g))
    return float(v), g


def blur(src, width, height, channels, dtype=np.float32):
    s, dt = _sfx(dtype)
    x = _arr(src, dt).ravel()
    out = np.zeros_like(x)
    getattr(lib(), f"ora_blur_{s}")(_p(x), width, height, channels, _p(out))
    return out


def psnr(pred, target, dtype=np.float32):
    s, dt = _sfx(dtype)
    x = _arr(pred, dt).ravel()
    y = _arr(target, dt).ravel()
    return float(getattr(lib(), f"ora_psnr_{s}")(_p(x), _p(y), x.size))


# --- adam.rs, densify.rs ---------------------------------------------------------------
def adam_step(params, grads, m, v, step, lr6, dtype=np.float32):
    """Adam::step (src/adam.rs:77-161), in place on params/m/v; returns the new step count."""
    s, dt = _sfx(dtype)
    for a in (params, grads, m, v):
        assert a.dtype == dt and a.flags.c_contiguous
    lr = np.ascontiguousarray(lr6, dt)
    return int(getattr(lib(), f"ora_adam_step_{s}")(_p(params), _p(grads), _p(m), _p(v),
                                                    params.shape[0], step, _p(lr)))


def densify_accumulate(projs, grads9, abs2, width, height, grad_accum, denom, max_radii, dtype=np.float32):
    """DensifyStats::accumulate (src/densify.rs:36-60), in place."""
    s, dt = _sfx(dtype)
    p = _arr(projs, dt, PROJ_FIELDS)
    getattr(lib(), f"ora_densify_accumulate_{s}")(_p(p), _p(_arr(grads9, dt, 9)),
                                                  _p(_arr(abs2, dt, 2)) if abs2 is not None else None,
                                                  p.shape[0], width, height, _p(grad_accum), _p(denom), _p(max_radii))


def densify_and_prune(params, m, v, grad_accum, denom, max_radii, extent, normals, grad_threshold=0.0002,
                      percent_dense=0.01, min_opacity=0.005, prune_big_world=False, max_world_size_frac=0.1,
                      max_screen_size=None, split_children=2, dtype=np.float32):
    """densify_and_prune (src/densify.rs:125-221) with pre-drawn normal samples.

    Returns (params, m, v, report) with report = (cloned, split, pruned, normals used)."""
    s, dt = _sfx(dtype)
    p = _arr(params, dt, NUM_PARAMS)
    n0 = p.shape[0]
    cap = n0 * (2 + split_children) + 1
    op = np.zeros((cap, NUM_PARAMS), dt)
    om = np.zeros_like(op)
    ov = np.zeros_like(op)
    rep = np.zeros(4, np.int64)
    nrm = np.ascontiguousarray(normals, np.float64)
    n = getattr(lib(), f"ora_densify_{s}")(
        _p(p), _p(_arr(m, dt, NUM_PARAMS)), _p(_arr(v, dt, NUM_PARAMS)), n0, _p(_arr(grad_accum, dt)),
        _p(np.ascontiguousarray(denom, np.uint32)), _p(np.ascontiguousarray(max_radii, np.uint32)),
        grad_threshold, percent_dense, min_opacity, int(prune_big_world), max_world_size_frac,
        -1 if max_screen_size is None else int(max_screen_size), split_children, extent, _p(nrm), nrm.size,
        _p(op), _p(om), _p(ov), _p(rep))
    if n < 0:
        raise ValueError("not enough normal samples")
    return op[:n].copy(), om[:n].copy(), ov[:n].copy(), tuple(int(x) for x in rep)


def reset_opacity(params, m, v, max_alpha=0.01, dtype=np.float32):
    """reset_opacity (src/densify.rs:224-230), in place."""
    s, dt = _sfx(dtype)
    getattr(lib(), f"ora_reset_opacity_{s}")(_p(params), _p(m), _p(v), params.shape[0], max_alpha)


# --- model.rs --------------------------------------------------------------------------
def mean_nn_dist2(points):
    pts = _arr(points, np.float32, 3)
    out = np.zeros(pts.shape[0], np.float64)
    lib().ora_mean_nn_dist2(_p(pts), pts.shape[0], _p(out))
    return out


def from_points(points, rgb, dtype=np.float32):
    """Model::from_points (src/model.rs:77-104)."""
    s, dt = _sfx(dtype)
    pts = _arr(points, np.float32, 3)
    col = np.ascontiguousarray(rgb, np.uint8).reshape(-1, 3)
    out = np.zeros((pts.shape[0], NUM_PARAMS), dt)
    getattr(lib(), f"ora_from_points_{s}")(_p(pts), _p(col), pts.shape[0], _p(out))
    return out


# --- train.rs --------------------------------------------------------------------------
TRAIN_DEFAULTS = dict(
    iterations=30000, position_lr_init=0.00016, position_lr_final=0.0000016, position_lr_max_steps=30000,
    feature_lr=0.0025, opacity_lr=0.025, scaling_lr=0.005, rotation_lr=0.001, lambda_dssim=0.2, densify=1,
    densify_from_iter=500, densify_until_iter=15000, densification_interval=100, opacity_reset_interval=3000,
    densify_grad_threshold=0.0002, percent_dense=0.01, min_opacity=0.005, max_screen_size=-1, absgrad=0,
    antialias=0, white_background=0, sh_degree=3, sh_degree_interval=1000, near=0.2, seed=0)


def train_config_vector(**overrides):
    fields = lib().ora_train_config_fields().decode().split(",")
    cfg = dict(TRAIN_DEFAULTS)
    for k, v in overrides.items():
        if k not in cfg:
            raise KeyError(k)
        cfg[k] = -1 if (k == "max_screen_size" and v is None) else v
    return np.array([float(cfg[f]) for f in fields], np.float64)


STEP_FIELDS = ("loss", "psnr", "view", "num_gaussians", "cloned", "split", "pruned", "densified", "reset", "entries")


class Trainer:
    """train::train (src/train.rs:161-306) one iteration at a time, f32."""

    def __init__(self, init_params, extent, views, **cfg):
        p = _arr(init_params, np.float32, NUM_PARAMS)
        self.cfgv = train_config_vector(**cfg)
        self.h = lib().ora_trainer_new(_p(p), p.shape[0], extent, _p(self.cfgv))
        for cam, rgb in views:
            lib().ora_trainer_add_view(self.h, _p(_arr(cam, np.float32)), _p(np.ascontiguousarray(rgb, np.uint8)))
        lib().ora_trainer_start(self.h)

    def step(self):
        info = np.zeros(10, np.float64)
        lib().ora_trainer_step(self.h, _p(info))
        return dict(zip(STEP_FIELDS, info.tolist()))

    @property
    def count(self):
        return lib().ora_trainer_count(self.h)

    @property
    def sh_degree(self):
        return lib().ora_trainer_sh_degree(self.h)

    def model(self):
        out = np.zeros((self.count, NUM_PARAMS), np.float32)
        lib().ora_trainer_get_model(self.h, _p(out))
        return out

    def render(self, cam):
        cam = _arr(cam, np.float32)
        out = np.zeros(int(cam[0]) * int(cam[1]) * 3, np.float32)
        lib().ora_trainer_render(self.h, _p(cam), _p(out))
        return out

    def __del__(self):
        try:
            if self.h:
                lib().ora_trainer_free(self.h)
        except Exception:
            pass
