"""Scene and parameter fixtures mirroring the reference's test helpers
(tests/common/mod.rs and tests/common/scene.rs), drawn from numpy generators instead of
ChaCha8: the distributions and shapes are the reference's, the exact draws are not."""
from __future__ import annotations

import math

import numpy as np

from oracle import oracle as O

NUM_PARAMS = 59
SH_C0 = 0.28209479177387814

# tests/common/mod.rs:16-34
TOL = {
    np.float32: dict(H=1e-2, RTOL=5e-2, ATOL=1e-3),
    np.float64: dict(H=1e-6, RTOL=1e-5, ATOL=1e-8),
}


def check(what, analytic, numeric, scale, dtype):
    """tests/common/mod.rs:37-43."""
    t = TOL[dtype]
    tol = t["ATOL"] * scale + t["RTOL"] * max(abs(analytic), abs(numeric))
    assert abs(analytic - numeric) <= tol, (
        f"{what}: analytic {analytic:.9e} vs finite difference {numeric:.9e} (tol {tol:.3e})")


def central(x, h, f):
    """tests/common/mod.rs:46-48."""
    return (f(x + h) - f(x - h)) / (2.0 * h)


def rnd(rng, lo, hi):
    return lo + (hi - lo) * rng.random()


def random_gaussian(rng):
    """tests/common/mod.rs:61-92: a Gaussian near the origin with clearly positive colours."""
    g = np.zeros(NUM_PARAMS)
    sh = np.zeros((16, 3))
    for k in range(16):
        for c in range(3):
            sh[k, c] = rnd(rng, 0.2, 1.5) if k == 0 else rnd(rng, -0.15, 0.15)
    g[0:3] = [rnd(rng, -0.6, 0.6), rnd(rng, -0.4, 0.4), rnd(rng, -0.5, 0.5)]
    g[3:6] = [rnd(rng, -2.5, -1.2) for _ in range(3)]
    g[6:10] = [rnd(rng, 0.5, 1.5), rnd(rng, -0.7, 0.7), rnd(rng, -0.7, 0.7), rnd(rng, -0.7, 0.7)]
    g[10] = rnd(rng, -1.0, 2.0)
    g[11:] = sh.ravel()
    return g


def test_camera(width, height, dtype=np.float32):
    """tests/common/mod.rs:95-106."""
    return O.look_at(width, height, width * 0.9, width * 0.9, [0.3, -0.2, -3.0], [0, 0, 0], [0, -1, 0], dtype)


def param_name(i):
    """tests/common/mod.rs:142-152."""
    if i < 3:
        return f"mean[{i}]"
    if i < 6:
        return f"log_scale[{i - 3}]"
    if i < 10:
        return f"quat[{i - 6}]"
    if i == 10:
        return "opacity"
    j = i - 11
    return f"sh[{j // 3}][{j % 3}]"


def ring_cameras(n, width, height, radius, dtype=np.float32):
    """tests/common/scene.rs:32-53."""
    cams = []
    for i in range(n):
        a = i / n * math.tau
        eye = [radius * math.cos(a), -0.6 + 0.3 * math.sin(3.0 * a), radius * math.sin(a)]
        cams.append(O.look_at(width, height, width * 1.1, width * 1.1, eye, [0, 0, 0], [0, -1, 0], dtype))
    return np.stack(cams)


def ground_truth(rng, n):
    """tests/common/scene.rs:56-94: random blobs, SH degree 1."""
    out = np.zeros((n, NUM_PARAMS))
    for i in range(n):
        sh = np.zeros((16, 3))
        for c in range(3):
            sh[0, c] = (rnd(rng, 0.1, 0.9) - 0.5) / SH_C0
        for k in range(1, 4):
            for c in range(3):
                sh[k, c] = rnd(rng, -0.2, 0.2)
        out[i, 0:3] = [rnd(rng, -0.7, 0.7), rnd(rng, -0.5, 0.5), rnd(rng, -0.7, 0.7)]
        out[i, 3:6] = [rnd(rng, -2.6, -1.6) for _ in range(3)]
        out[i, 6:10] = [rnd(rng, 0.5, 1.0), rnd(rng, -0.5, 0.5), rnd(rng, -0.5, 0.5), rnd(rng, -0.5, 0.5)]
        out[i, 10] = rnd(rng, 0.5, 3.0)
        out[i, 11:] = sh.ravel()
    return out.astype(np.float32)


def to_rgb8(image):
    """render.rs:26-31."""
    return np.round(np.clip(image, 0.0, 1.0) * 255.0).astype(np.uint8)


def render(params, cam, sh_degree, background, antialias=False, dtype=np.float32):
    """render::render (src/render.rs:14-23) on the oracle."""
    w, h = int(cam[0]), int(cam[1])
    projs = O.project_all(params, cam, antialias=antialias, sh_degree=sh_degree, dtype=dtype)
    b = O.bin(projs, w, h, dtype=dtype)
    img, _, _, _ = O.rasterize_forward(projs, b, w, h, background, dtype=dtype)
    return img


def render_views(gt, cams, sh_degree, background):
    """tests/common/scene.rs:96-108."""
    return [(cam, to_rgb8(render(gt, cam, sh_degree, background))) for cam in cams]


def init_points(gt, rng):
    """tests/common/scene.rs:111-128."""
    pts = gt[:, 0:3].astype(np.float64) + np.array([[rnd(rng, -0.03, 0.03) for _ in range(3)] for _ in gt])
    rgb = np.round(np.clip(gt[:, 11:14] * SH_C0 + 0.5, 0.0, 1.0) * 255.0).astype(np.uint8)
    return pts.astype(np.float32), rgb


def evaluate(params, views, sh_degree, background, antialias=False):
    """train::evaluate (src/train.rs:309-321) on the oracle."""
    total = 0.0
    for cam, rgb in views:
        img = render(params, cam, sh_degree, background, antialias)
        total += O.psnr(img, rgb.astype(np.float32).ravel() / np.float32(255.0))
    return total / len(views)


def write_ply_reference_layout(path, params, degree):
    """A .ply written as ply::write does (src/ply.rs:19-69), in plain Python: binary
    little-endian float32 rows x y z nx ny nz f_dc_0..2 f_rest_* (channel-major) opacity
    scale_0..2 rot_0..3."""
    K = (degree + 1) ** 2
    n_rest = 3 * (K - 1)
    names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
    names += [f"f_rest_{i}" for i in range(n_rest)] + ["opacity", "scale_0", "scale_1", "scale_2"]
    names += ["rot_0", "rot_1", "rot_2", "rot_3"]
    header = "ply\nformat binary_little_endian 1.0\n" + f"element vertex {len(params)}\n"
    header += "".join(f"property float {nm}\n" for nm in names) + "end_header\n"
    rows = np.zeros((len(params), len(names)), np.float32)
    p = np.asarray(params, np.float32)
    sh = p[:, 11:].reshape(-1, 16, 3)
    rows[:, 0:3] = p[:, 0:3]
    rows[:, 6:9] = sh[:, 0, :]
    for c in range(3):
        for k in range(1, K):
            rows[:, 9 + c * (K - 1) + (k - 1)] = sh[:, k, c]
    rows[:, 9 + n_rest] = p[:, 10]
    rows[:, 10 + n_rest:13 + n_rest] = p[:, 3:6]
    rows[:, 13 + n_rest:17 + n_rest] = p[:, 6:10]
    with open(path, "wb") as f:
        f.write(header.encode())
        f.write(rows.astype("<f4").tobytes())
