"""Seeded synthetic scenes with the shapes and value distributions of the benchmark
configurations. No public dataset is involved: every scene is drawn from numpy generators
with fixed seeds, and the same arrays feed the CUDA path and the CPU oracle.

Parameter records use the reference layout (59 floats per Gaussian: mean[3] log_scale[3]
quat[4] opacity sh[16][3], reference src/model.rs:16-28); cameras are 18-value records
(width, height, fx, fy, cx, cy, rot[9] row major, trans[3]) built like Camera::look_at
(reference src/camera.rs:66-93).
"""
from __future__ import annotations

import math

import numpy as np

SH_C0 = 0.28209479177387814


def look_at(width, height, fx, fy, eye, target, up=(0.0, -1.0, 0.0)):
    """Camera::look_at (src/camera.rs:66-93): +z forward, x right, y down."""
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    rot = np.stack([right, down, fwd]).astype(np.float32)
    trans = -(rot.astype(np.float64) @ eye)
    rec = np.zeros(18, np.float32)
    rec[0:6] = [width, height, fx, fy, width / 2.0, height / 2.0]
    rec[6:15] = rot.ravel()
    rec[15:18] = trans
    return rec


def random_gaussians(rng, n, mean_lo, mean_hi, log_scale_mu, log_scale_sigma, opacity_sigma, dc_mu=0.5,
                     dc_sigma=0.2, rest_sigma=0.05):
    """Gaussians with means uniform in a box, normal log-scales and opacity logits,
    quaternions normalise(N(0,1)^4), SH degree 3 with normal DC and higher bands."""
    g = np.zeros((n, 59), np.float32)
    g[:, 0:3] = rng.uniform(mean_lo, mean_hi, (n, 3))
    g[:, 3:6] = rng.normal(log_scale_mu, log_scale_sigma, (n, 3))
    q = rng.normal(0.0, 1.0, (n, 4))
    g[:, 6:10] = q / np.linalg.norm(q, axis=1, keepdims=True)
    g[:, 10] = rng.normal(0.0, opacity_sigma, n)
    sh = rng.normal(0.0, rest_sigma, (n, 16, 3))
    sh[:, 0, :] = rng.normal(dc_mu, dc_sigma, (n, 3))
    g[:, 11:] = sh.reshape(n, 48)
    return g


def fibonacci_sphere(n, radius):
    """n points spread over a sphere (golden-angle spiral), none at the poles."""
    pts = []
    ga = math.pi * (3.0 - math.sqrt(5.0))
    for i in range(n):
        y = 1.0 - 2.0 * (i + 0.5) / n
        r = math.sqrt(max(0.0, 1.0 - y * y))
        th = ga * i
        pts.append((radius * r * math.cos(th), radius * y, radius * r * math.sin(th)))
    return np.array(pts)


def blob_scene(seed_gt=0, seed_init=1, n_gt=10000, n_cams=16, size=256, f=300.0, n_init=5000):
    """Plain method on a small scene: 10k ground-truth Gaussians in [-1,1]^3, log-scales
    N(-4,0.3), opacity logits N(0,1), SH degree 3 (DC N(0.5,0.2), rest N(0,0.05)); 16
    cameras on a radius-4 sphere looking at the origin at 256x256, f=300, c=128; 5k
    initial points = ground-truth means + N(0,0.02)."""
    rng = np.random.default_rng(seed_gt)
    gt = random_gaussians(rng, n_gt, -1.0, 1.0, -4.0, 0.3, 1.0)
    cams = np.stack([look_at(size, size, f, f, eye, (0, 0, 0)) for eye in fibonacci_sphere(n_cams, 4.0)])
    rng1 = np.random.default_rng(seed_init)
    pick = rng1.choice(n_gt, size=n_init, replace=False)
    pts = (gt[pick, 0:3] + rng1.normal(0.0, 0.02, (n_init, 3))).astype(np.float32)
    rgb = np.round(np.clip(gt[pick, 11:14] * SH_C0 + 0.5, 0.0, 1.0) * 255.0).astype(np.uint8)
    return dict(gt=gt, cams=cams, init_points=pts, init_rgb=rgb, sh_degree=3, background=(0.0, 0.0, 0.0))


def render_benchmark_scene(seed=0, n=1_000_000, width=1920, height=1080, f=1500.0, distance=12.0):
    """Render-only kernel benchmark: 1M Gaussians with means uniform in a 10x10x10 box
    centred at the origin, camera at distance 12 looking at the centre, f=1500, 1920x1080,
    log-scales N(-4.5,0.5), opacity logits N(0,1.5), SH degree 3 as in blob_scene, and an
    upstream dL/dpixel drawn N(0,1) per channel."""
    rng = np.random.default_rng(seed)
    g = random_gaussians(rng, n, -5.0, 5.0, -4.5, 0.5, 1.5)
    cam = look_at(width, height, f, f, (0.0, 0.0, -distance), (0.0, 0.0, 0.0))
    dimage = rng.normal(0.0, 1.0, width * height * 3).astype(np.float32)
    return dict(params=g, cam=cam, dimage=dimage, sh_degree=3, background=(0.0, 0.0, 0.0))


def hemisphere_cameras(n, radius, width, height, f):
    """n cameras spread over the upper hemisphere (-y is up) by a golden-angle spiral,
    looking at the origin; none sits exactly at the pole."""
    ga = math.pi * (3.0 - math.sqrt(5.0))
    cams = []
    for i in range(n):
        y = -(i + 0.5) / n
        r = math.sqrt(max(0.0, 1.0 - y * y))
        th = ga * i
        eye = (radius * r * math.cos(th), radius * y, radius * r * math.sin(th))
        cams.append(look_at(width, height, f, f, eye, (0.0, 0.0, 0.0)))
    return np.stack(cams)


def shell_scene(seed_gt=0, seed_init=1, n_gt=500_000, n_shells=40, n_cams=200, width=1297, height=840, f=1150.0,
            n_init=100_000, cube=6.0):
    """Clustered multi-view scene: n_gt Gaussians on n_shells shells inside a cube of side
    `cube` centred at the origin, half of them spheres and half planar discs, radius
    U(0.2, 2), each point jittered N(0, 0.01) per axis; points split over the shells in
    proportion to their area. Log-scales N(-4.5, 0.3), opacity logits N(0, 1), SH degree 3
    as in blob_scene. n_cams cameras on a radius-8 hemisphere at width x height, f = 1150.
    n_init initial points = ground-truth means + N(0, 0.02), colours from the ground-truth
    DC band."""
    rng = np.random.default_rng(seed_gt)
    radius = rng.uniform(0.2, 2.0, n_shells)
    planar = rng.uniform(0.0, 1.0, n_shells) < 0.5
    half = cube / 2.0
    centre = np.stack([rng.uniform(-half + r, half - r, 3) for r in radius])
    normal = rng.normal(0.0, 1.0, (n_shells, 3))
    normal /= np.linalg.norm(normal, axis=1, keepdims=True)
    area = np.where(planar, math.pi * radius ** 2, 4.0 * math.pi * radius ** 2)
    counts = np.floor(area / area.sum() * n_gt).astype(np.int64)
    counts[: n_gt - counts.sum()] += 1
    pts = []
    for s in range(n_shells):
        k = int(counts[s])
        if planar[s]:
            a = np.cross(normal[s], [1.0, 0.0, 0.0] if abs(normal[s][0]) < 0.9 else [0.0, 1.0, 0.0])
            a /= np.linalg.norm(a)
            b = np.cross(normal[s], a)
            rr = radius[s] * np.sqrt(rng.uniform(0.0, 1.0, k))
            th = rng.uniform(0.0, 2.0 * math.pi, k)
            p = centre[s] + (rr * np.cos(th))[:, None] * a + (rr * np.sin(th))[:, None] * b
        else:
            u = rng.normal(0.0, 1.0, (k, 3))
            p = centre[s] + radius[s] * u / np.linalg.norm(u, axis=1, keepdims=True)
        pts.append(p + rng.normal(0.0, 0.01, (k, 3)))
    gt = random_gaussians(rng, n_gt, 0.0, 0.0, -4.5, 0.3, 1.0)
    gt[:, 0:3] = np.concatenate(pts)
    cams = hemisphere_cameras(n_cams, 8.0, width, height, f)
    rng1 = np.random.default_rng(seed_init)
    pick = rng1.choice(n_gt, size=n_init, replace=False)
    ip = (gt[pick, 0:3] + rng1.normal(0.0, 0.02, (n_init, 3))).astype(np.float32)
    rgb = np.round(np.clip(gt[pick, 11:14] * SH_C0 + 0.5, 0.0, 1.0) * 255.0).astype(np.uint8)
    return dict(gt=gt, cams=cams, init_points=ip, init_rgb=rgb, sh_degree=3, background=(0.0, 0.0, 0.0))


MIXED_VIEW_SIZES = ((640, 480), (1024, 768), (1297, 840), (1600, 1200))


def shell_scene_mixed_sizes(seed_sizes=7, **kw):
    """shell_scene with every camera at a resolution drawn uniformly from MIXED_VIEW_SIZES
    (seeded), its focal length scaled with the width (f = 1150 at 1297 pixels)."""
    s = shell_scene(**kw)
    rng = np.random.default_rng(seed_sizes)
    pick = rng.integers(0, len(MIXED_VIEW_SIZES), len(s["cams"]))
    cams = []
    for cam, k in zip(s["cams"], pick):
        w, h = MIXED_VIEW_SIZES[k]
        c = cam.copy()
        f = 1150.0 * w / 1297.0
        c[0:6] = [w, h, f, f, w / 2.0, h / 2.0]
        cams.append(c)
    s["cams"] = np.stack(cams)
    return s


def scene_extent(cams):
    """scene_extent (src/camera.rs:99-118): 1.1 x the largest distance from a camera centre
    to the mean centre."""
    cams = np.asarray(cams, np.float64).reshape(-1, 18)
    centers = np.stack([-(c[6:15].reshape(3, 3).T @ c[15:18]) for c in cams])
    mean = centers.mean(0)
    ext = float(np.max(np.linalg.norm(centers - mean, axis=1))) * 1.1
    return ext if ext > 0 else 1.0


def to_rgb8(image):
    """render::to_rgb8 (src/render.rs:26-31)."""
    return np.round(np.clip(image, 0.0, 1.0) * 255.0).astype(np.uint8)


def psnr(pred, target_u8):
    """psnr (src/loss.rs:175-190) against an 8-bit view converted as View::to_real."""
    t = np.asarray(target_u8, np.float32) / np.float32(255.0)
    d = np.clip(np.asarray(pred, np.float32), 0, 1).astype(np.float64) - np.clip(t, 0, 1).astype(np.float64)
    mse = float((d * d).mean())
    return float("inf") if mse <= 0 else -10.0 * np.log10(mse)
