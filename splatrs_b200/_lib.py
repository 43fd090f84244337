"""ctypes binding of libsplatrs_b200.so, the C ABI declared in include/splat_gpu.h.

The library is built in-tree (splatrs_b200/build.py). There is no fallback: if the
library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsplatrs_b200.so")

SPLAT_OK = 0
SPLAT_ERR_INVALID = 1
SPLAT_ERR_CAPACITY = 2
SPLAT_ERR_CUDA = 3
SPLAT_ERR_TIMEOUT = 4
PLANES = 15
PROJ_FLOATS = 16


class SplatError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class Camera(C.Structure):
    """splat_camera (reference src/camera.rs:13-32)."""
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("fx", C.c_float), ("fy", C.c_float),
                ("cx", C.c_float), ("cy", C.c_float), ("rot", C.c_float * 9), ("trans", C.c_float * 3)]

    @classmethod
    def from_record(cls, rec):
        """From the 18-value record width, height, fx, fy, cx, cy, rot[9], trans[3]."""
        r = [float(x) for x in rec]
        c = cls()
        c.width, c.height = int(r[0]), int(r[1])
        c.fx, c.fy, c.cx, c.cy = r[2], r[3], r[4], r[5]
        for i in range(9):
            c.rot[i] = r[6 + i]
        for i in range(3):
            c.trans[i] = r[15 + i]
        return c


class ProjOpts(C.Structure):
    """splat_proj_opts (reference src/project.rs:22-43)."""
    _fields_ = [("near_plane", C.c_float), ("eps2d", C.c_float), ("antialias", C.c_int32), ("sh_degree", C.c_int32),
                ("fp64_conic", C.c_int32)]

    @classmethod
    def make(cls, near=0.2, eps2d=0.3, antialias=False, sh_degree=3, fp64_conic=False):
        return cls(near, eps2d, int(bool(antialias)), int(sh_degree), int(bool(fp64_conic)))


class LearningRates(C.Structure):
    """splat_lr (reference src/adam.rs:11-24)."""
    _fields_ = [(n, C.c_float) for n in ("mean", "log_scale", "quat", "opacity", "sh_dc", "sh_rest")]


class DensifyConfig(C.Structure):
    """splat_densify_config (reference src/densify.rs:69-103)."""
    _fields_ = [("grad_threshold", C.c_float), ("percent_dense", C.c_float), ("min_opacity", C.c_float),
                ("prune_big_world", C.c_int32), ("max_world_size_frac", C.c_float), ("max_screen_size", C.c_int64),
                ("split_children", C.c_int32)]

    @classmethod
    def make(cls, grad_threshold=0.0002, percent_dense=0.01, min_opacity=0.005, prune_big_world=False,
             max_world_size_frac=0.1, max_screen_size=None, split_children=2):
        return cls(grad_threshold, percent_dense, min_opacity, int(bool(prune_big_world)), max_world_size_frac,
                   -1 if max_screen_size is None else int(max_screen_size), int(split_children))


class TrainConfig(C.Structure):
    """splat_train_config (reference src/train.rs:20-109)."""
    _fields_ = [("iterations", C.c_uint32), ("position_lr_init", C.c_float), ("position_lr_final", C.c_float),
                ("position_lr_max_steps", C.c_uint32), ("feature_lr", C.c_float), ("opacity_lr", C.c_float),
                ("scaling_lr", C.c_float), ("rotation_lr", C.c_float), ("lambda_dssim", C.c_float),
                ("densify", C.c_int32), ("densify_from_iter", C.c_uint32), ("densify_until_iter", C.c_uint32),
                ("densification_interval", C.c_uint32), ("opacity_reset_interval", C.c_uint32),
                ("densify_grad_threshold", C.c_float), ("percent_dense", C.c_float), ("min_opacity", C.c_float),
                ("max_screen_size", C.c_int64), ("absgrad", C.c_int32), ("antialias", C.c_int32),
                ("white_background", C.c_int32), ("sh_degree", C.c_int32), ("sh_degree_interval", C.c_uint32),
                ("near_plane", C.c_float), ("seed", C.c_uint64), ("max_gaussians", C.c_uint64),
                ("entry_capacity", C.c_uint64), ("bf16_storage", C.c_int32), ("fp64_conic", C.c_int32),
                ("batch_views", C.c_uint32), ("learned_densify", C.c_int32), ("autotune", C.c_int32),
                ("learn_contribution", C.c_float), ("learn_prune_confidence", C.c_float), ("deterministic", C.c_int32),
                ("coarse_until", C.c_uint32), ("coarse_factor", C.c_uint32)]

    DEFAULTS = dict(iterations=30000, position_lr_init=0.00016, position_lr_final=0.0000016,
                    position_lr_max_steps=30000, feature_lr=0.0025, opacity_lr=0.025, scaling_lr=0.005,
                    rotation_lr=0.001, lambda_dssim=0.2, densify=1, densify_from_iter=500, densify_until_iter=15000,
                    densification_interval=100, opacity_reset_interval=3000, densify_grad_threshold=0.0002,
                    percent_dense=0.01, min_opacity=0.005, max_screen_size=-1, absgrad=0, antialias=0,
                    white_background=0, sh_degree=3, sh_degree_interval=1000, near_plane=0.2, seed=0,
                    max_gaussians=0, entry_capacity=0, bf16_storage=0, fp64_conic=0,
                    batch_views=0, learned_densify=0, autotune=0, learn_contribution=0.0,
                    learn_prune_confidence=0.0, deterministic=0, coarse_until=0, coarse_factor=2)

    @classmethod
    def make(cls, **kw):
        d = dict(cls.DEFAULTS)
        if "near" in kw:
            kw["near_plane"] = kw.pop("near")
        for k, v in kw.items():
            if k not in d:
                raise KeyError(k)
            d[k] = -1 if (k == "max_screen_size" and v is None) else v
        c = cls()
        for k, v in d.items():
            setattr(c, k, int(v) if isinstance(getattr(c, k), int) else float(v))
        return c


class DensifyReport(C.Structure):
    """splat_densify_report (reference src/densify.rs:107-114, plus the new count)."""
    _fields_ = [("cloned", C.c_uint64), ("split", C.c_uint64), ("pruned", C.c_uint64), ("new_count", C.c_uint64)]


class StepInfo(C.Structure):
    """splat_step_info (reference src/train.rs:142-157)."""
    _fields_ = [("loss", C.c_double), ("psnr", C.c_double), ("view", C.c_uint32), ("densified", C.c_int32),
                ("reset", C.c_int32), ("num_gaussians", C.c_uint64), ("cloned", C.c_uint64), ("split", C.c_uint64),
                ("pruned", C.c_uint64), ("entries", C.c_uint64), ("replayed", C.c_uint32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def _declare(L):
    vp, i64, u32, i32, sz = C.c_void_p, C.c_int64, C.c_uint32, C.c_int32, C.c_size_t
    P = C.POINTER
    sig = {
        "splat_version": ([], C.c_int),
        "splat_status_string": ([C.c_int], C.c_char_p),
        "splat_ctx_create": ([C.c_int, vp, P(vp)], C.c_int),
        "splat_ctx_destroy": ([vp], C.c_int),
        "splat_ctx_set_stream": ([vp, vp], C.c_int),
        "splat_ctx_synchronize": ([vp], C.c_int),
        "splat_last_error": ([vp], C.c_char_p),
        "splat_ctx_launch_count": ([vp], C.c_uint64),
        "splat_zero": ([vp, vp, sz], C.c_int),
        "splat_diag_fast_exp_error": ([vp, C.c_float, C.c_float, i32, P(C.c_float)], C.c_int),
        "splat_diag_pair_exact": ([vp, C.c_uint32, P(C.c_uint32)], C.c_int),
        "splat_diag_mbarrier_wait": ([vp, u32, i32], C.c_int),
        "splat_diag_peak": ([vp, i32, P(C.c_double), P(C.c_float)], C.c_int),
        "splat_ctx_scratch_info": ([vp, P(C.c_uint64)], C.c_int),
        "splat_params_from_aos": ([vp, vp, i64, vp, i64], C.c_int),
        "splat_params_to_aos": ([vp, vp, i64, i64, vp], C.c_int),
        "splat_project_fwd": ([vp, vp, i64, i64, P(Camera), P(ProjOpts), vp, vp, vp], C.c_int),
        "splat_proj_from_reference": ([vp, vp, i64, u32, u32, vp, vp, vp], C.c_int),
        "splat_proj_to_reference": ([vp, vp, i64, vp], C.c_int),
        "splat_bin_count": ([vp, vp, i64, vp, P(i64)], C.c_int),
        "splat_bin_count_noalloc": ([vp, vp, i64, vp, P(i64)], C.c_int),
        "splat_bin_sort": ([vp, vp, vp, i64, i64, vp, u32, u32, vp, vp, vp], C.c_int),
        "splat_bin_count_device": ([vp, vp, i64, vp, vp], C.c_int),
        "splat_struct_sizes": ([P(C.c_uint64)], i32),
        "splat_mlp_num_params": ([], i32),
        "splat_mlp_forward": ([vp, vp, i64, vp, vp], C.c_int),
        "splat_mlp_forward_tc": ([vp, vp, i64, vp, vp], C.c_int),
        "splat_mlp_grad": ([vp, vp, vp, vp, i64, C.c_float, vp, vp], C.c_int),
        "splat_mlp_grad_tc": ([vp, vp, vp, vp, i64, C.c_float, vp, vp], C.c_int),
        "splat_mlp_adam": ([vp, vp, vp, vp, vp, C.c_uint64, C.c_float], C.c_int),
        "splat_raster_candidates": ([P(C.c_uint32)], i32),
        "splat_set_raster_config": ([vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32], C.c_int),
        "splat_get_raster_config": ([vp, P(C.c_uint32)], C.c_int),
        "splat_autotune_render": ([vp, vp, i64, i64, vp, vp, P(C.c_float), vp, i32, P(C.c_float), P(C.c_uint32)],
                                  C.c_int),
        "splat_bin_sort_device_scratch_bytes": ([i64], sz),
        "splat_bin_sort_device": ([vp, vp, vp, i64, vp, i64, vp, u32, u32, vp, vp, vp, vp], C.c_int),
        "splat_rasterize_fwd": ([vp, vp, vp, vp, u32, u32, P(C.c_float), vp, vp, vp, vp], C.c_int),
        "splat_rasterize_bwd": ([vp, vp, vp, vp, u32, u32, P(C.c_float), vp, vp, vp, vp, i64, vp], C.c_int),
        "splat_rasterize_bwd_deterministic": ([vp, vp, vp, vp, vp, i64, i64, u32, u32, P(C.c_float), vp, vp, vp, vp,
                                               i64], C.c_int),
        "splat_project_bwd": ([vp, vp, i64, i64, P(Camera), P(ProjOpts), vp, vp, vp, vp, i32], C.c_int),
    }
    sig.update({
        "splat_renderer_create": ([vp, P(vp)], C.c_int),
        "splat_renderer_destroy": ([vp], C.c_int),
        "splat_renderer_set_model": ([vp, vp, i64, i32], C.c_int),
        "splat_renderer_render": ([vp, P(Camera), P(ProjOpts), P(C.c_float), vp], C.c_int),
        "splat_renderer_render_backward": ([vp, P(Camera), P(ProjOpts), P(C.c_float), vp, vp, vp], C.c_int),
        "splat_renderer_submit_backward": ([vp, P(Camera), P(ProjOpts), P(C.c_float), vp, vp, vp, P(C.c_uint64)],
                                           C.c_int),
        "splat_renderer_wait": ([vp, C.c_uint64], C.c_int),
        "splat_renderer_last_entries": ([vp], i64),
    })
    sig.update({
        "splat_loss_fwd_bwd": ([vp, vp, vp, i32, u32, u32, C.c_float, vp, vp], C.c_int),
        "splat_adam_step": ([vp, vp, vp, vp, vp, i64, i64, C.c_uint64, P(LearningRates)], C.c_int),
        "splat_project_bwd_adam": ([vp, vp, vp, vp, i64, i64, P(Camera), P(ProjOpts), vp, vp, vp, i32, C.c_uint64,
                                    P(LearningRates), vp], C.c_int),
        "splat_params_to_bf16": ([vp, vp, i64, i64, vp], C.c_int),
        "splat_project_fwd_bf16": ([vp, vp, vp, i64, i64, P(Camera), P(ProjOpts), vp, vp, vp], C.c_int),
        "splat_densify": ([vp, vp, vp, vp, i64, i64, vp, P(DensifyConfig), C.c_float, P(C.c_uint64), vp, vp, vp, i64,
                           P(DensifyReport)], C.c_int),
        "splat_reset_opacity": ([vp, vp, vp, vp, i64, C.c_float], C.c_int),
        "splat_mean_nn_dist2": ([vp, vp, i64, vp], C.c_int),
        "splat_init_from_points": ([vp, vp, vp, i64, vp, i64], C.c_int),
        "splat_ply_read_header": ([vp, C.c_char_p, P(i64), P(i32)], C.c_int),
        "splat_ply_read": ([vp, C.c_char_p, vp, i64, P(i64), P(i32)], C.c_int),
        "splat_ply_write": ([vp, C.c_char_p, vp, i64, i64, i32], C.c_int),
        "splat_trainer_create": ([vp, P(TrainConfig), C.c_float, P(vp)], C.c_int),
        "splat_trainer_destroy": ([vp], C.c_int),
        "splat_trainer_set_model": ([vp, vp, i64], C.c_int),
        "splat_trainer_add_view": ([vp, P(Camera), vp], C.c_int),
        "splat_trainer_start": ([vp], C.c_int),
        "splat_trainer_step": ([vp, P(StepInfo)], C.c_int),
        "splat_trainer_run": ([vp, u32, P(StepInfo)], C.c_int),
        "splat_trainer_get_mlp": ([vp, vp], C.c_int),
        "splat_trainer_set_mlp": ([vp, vp], C.c_int),
        "splat_trainer_mlp_stats": ([vp, P(C.c_uint64)], C.c_int),
        "splat_trainer_tuning": ([vp, P(C.c_float), P(C.c_uint32), P(C.c_uint32)], C.c_int),
        "splat_trainer_evaluate": ([vp, vp, P(C.c_double)], C.c_int),
        "splat_trainer_count": ([vp], i64),
        "splat_trainer_sh_degree": ([vp], i32),
        "splat_trainer_iteration": ([vp], u32),
        "splat_trainer_get_model": ([vp, vp], C.c_int),
        "splat_trainer_get_moments": ([vp, vp, vp], C.c_int),
        "splat_trainer_render": ([vp, P(Camera), vp], C.c_int),
    })
    optional = {}
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    for name, (args, res) in optional.items():
        if hasattr(L, name):
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res


def exported_symbols():
    """Names this binding expects the library to export."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "splat_gpu.h")
    with open(hdr) as f:
        return sorted(set(re.findall(r"SPLAT_API\s+[\w\s\*]+?\b(splat_\w+)\s*\(", f.read())))


def lib():
    """Load the in-tree library; raises if it is missing (there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m splatrs_b200.build` "
                               "(or __graft_entry__.build()); the CUDA path has no fallback")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def check(status: int, ctx=None):
    if status != SPLAT_OK:
        msg = lib().splat_last_error(ctx).decode() if ctx else lib().splat_status_string(status).decode()
        raise SplatError(status, msg)
