"""The seeded synthetic scenes that stand in for the benchmark workloads: shapes, sizes and
value distributions as documented in splatrs_b200/scenes.py (statistics checked at sizes
that keep the suite fast). CPU only."""
import math

import numpy as np

from splatrs_b200 import scenes as S


def cam_centre(c):
    c = np.asarray(c, np.float64)
    return -(c[6:15].reshape(3, 3).T @ c[15:18])


def test_look_at_is_a_rotation_facing_the_target():
    """Camera::look_at (reference src/camera.rs:66-93): orthonormal rotation; the target
    lies on the camera's +z axis at the eye's distance."""
    c = S.look_at(320, 240, 300.0, 300.0, (1.0, -2.0, -5.0), (0.2, 0.1, 0.3))
    r = c[6:15].reshape(3, 3).astype(np.float64)
    assert np.allclose(r @ r.T, np.eye(3), atol=1e-6)
    assert np.allclose(cam_centre(c), [1.0, -2.0, -5.0], atol=1e-5)
    t = r @ np.array([0.2, 0.1, 0.3]) + c[15:18]
    assert abs(t[0]) < 1e-5 and abs(t[1]) < 1e-5
    assert abs(t[2] - np.linalg.norm(np.array([0.2, 0.1, 0.3]) - [1.0, -2.0, -5.0])) < 1e-5
    assert list(c[0:6]) == [320, 240, 300.0, 300.0, 160.0, 120.0]


def test_render_benchmark_scene_distributions():
    """1M Gaussians at full size; checked on 200k: means uniform in the 10 m cube,
    log-scales N(-4.5, 0.5), opacity logits N(0, 1.5), unit quaternions, SH DC N(0.5, 0.2),
    dL/dpix N(0, 1) over the 1920x1080 image, camera 12 m from the centre at f = 1500."""
    s = S.render_benchmark_scene(n=200_000)
    g = s["params"]
    assert g.shape == (200_000, 59) and g.dtype == np.float32
    assert g[:, 0:3].min() >= -5.0 and g[:, 0:3].max() <= 5.0
    assert abs(g[:, 0:3].mean()) < 0.05 and abs(g[:, 0:3].std() - 10.0 / math.sqrt(12.0)) < 0.02
    ls = g[:, 3:6]
    assert abs(ls.mean() + 4.5) < 0.01 and abs(ls.std() - 0.5) < 0.01
    assert abs(g[:, 10].mean()) < 0.02 and abs(g[:, 10].std() - 1.5) < 0.02
    assert np.allclose(np.linalg.norm(g[:, 6:10], axis=1), 1.0, atol=1e-5)
    dc = g[:, 11:14]
    assert abs(dc.mean() - 0.5) < 0.01 and abs(dc.std() - 0.2) < 0.01
    assert abs(g[:, 14:].std() - 0.05) < 0.002
    d = s["dimage"]
    assert d.shape == (1920 * 1080 * 3,) and abs(d.mean()) < 0.01 and abs(d.std() - 1.0) < 0.01
    c = s["cam"]
    assert list(c[0:4]) == [1920, 1080, 1500.0, 1500.0]
    assert abs(np.linalg.norm(cam_centre(c)) - 12.0) < 1e-4
    assert s["sh_degree"] == 3


def test_blob_scene_layout():
    """10k ground-truth Gaussians in [-1, 1]^3 with log-scales N(-4, 0.3); 16 cameras at
    256x256, f = 300, 4 from the origin; 5k initial points near ground-truth means, with
    colours from their DC band."""
    s = S.blob_scene()
    gt = s["gt"]
    assert gt.shape == (10_000, 59)
    assert gt[:, 0:3].min() >= -1.0 and gt[:, 0:3].max() <= 1.0
    assert abs(gt[:, 3:6].mean() + 4.0) < 0.02 and abs(gt[:, 3:6].std() - 0.3) < 0.02
    assert s["cams"].shape == (16, 18)
    for c in s["cams"]:
        assert list(c[0:6]) == [256, 256, 300.0, 300.0, 128.0, 128.0]
        assert abs(np.linalg.norm(cam_centre(c)) - 4.0) < 1e-4
    p, rgb = s["init_points"], s["init_rgb"]
    assert p.shape == (5_000, 3) and rgb.shape == (5_000, 3) and rgb.dtype == np.uint8
    d = np.sqrt(((p[:, None, :] - gt[None, :, 0:3]) ** 2).sum(-1)).min(1)
    assert np.median(d) < 0.05


def test_shell_scene_layout():
    """Ground-truth points on shells inside the 6 m cube (plus the 0.01 jitter), log-scales
    N(-4.5, 0.3), opacity logits N(0, 1); cameras on the upper hemisphere (-y up) of radius 8
    at 1297x840, f = 1150; initial points drawn from the ground truth."""
    s = S.shell_scene(n_gt=20_000, n_cams=12, n_init=2_000)
    gt = s["gt"]
    assert gt.shape == (20_000, 59)
    assert np.abs(gt[:, 0:3]).max() < 3.0 + 0.06
    assert abs(gt[:, 3:6].mean() + 4.5) < 0.02 and abs(gt[:, 3:6].std() - 0.3) < 0.02
    assert abs(gt[:, 10].std() - 1.0) < 0.03
    assert s["cams"].shape == (12, 18)
    for c in s["cams"]:
        assert list(c[0:4]) == [1297, 840, 1150.0, 1150.0]
        e = cam_centre(c)
        assert abs(np.linalg.norm(e) - 8.0) < 1e-4 and e[1] < 0.0
    assert s["init_points"].shape == (2_000, 3) and s["init_rgb"].shape == (2_000, 3)


def test_mixed_view_sizes():
    """Every camera at one of the four sizes, focal length scaled with the width; all four
    sizes occur; the scene is otherwise the shell scene's."""
    s = S.shell_scene_mixed_sizes(n_gt=5_000, n_cams=40, n_init=500)
    base = S.shell_scene(n_gt=5_000, n_cams=40, n_init=500)
    seen = set()
    for c, b in zip(s["cams"], base["cams"]):
        w, h = int(c[0]), int(c[1])
        assert (w, h) in S.MIXED_VIEW_SIZES
        seen.add((w, h))
        assert abs(c[2] - 1150.0 * w / 1297.0) < 1e-3 and c[4] == w / 2.0 and c[5] == h / 2.0
        assert np.array_equal(c[6:18], b[6:18])
    assert seen == set(S.MIXED_VIEW_SIZES)
    assert np.array_equal(s["gt"], base["gt"])
