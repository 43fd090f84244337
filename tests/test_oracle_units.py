"""The reference's unit tests with exact answers, replayed against the CPU oracle.

Each test names the reference test it replays. These pin the oracle before it is used to
check the CUDA kernels."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests import fixtures as F


def test_rotation_is_orthonormal():
    """src/math.rs:403-425."""
    for dt in (np.float32, np.float64):
        r = O.quat_to_mat([0.3, -0.5, 0.7, 0.2], dt).astype(np.float64)
        assert np.abs(r.T @ r - np.eye(3)).max() < 1e-5
        assert np.linalg.norm(np.cross(r[:, 0], r[:, 1]) - r[:, 2]) < 1e-5


def test_sigmoid_roundtrip():
    """src/math.rs:427-433."""
    for v in (0.01, 0.1, 0.5, 0.9, 0.99):
        assert abs(O.sigmoid(O.inverse_sigmoid(v)) - v) < 1e-5


def test_look_at_projects_target_to_principal_point():
    """src/camera.rs:124-139."""
    cam = O.look_at(64, 48, 50.0, 50.0, [1.0, 2.0, -5.0], [0, 0, 0], [0, -1, 0]).astype(np.float64)
    rot = cam[6:15].reshape(3, 3)
    t = cam[15:18]
    p = rot @ np.zeros(3) + t
    assert abs(p[0]) < 1e-5 and abs(p[1]) < 1e-5 and p[2] > 0
    c = -(rot.T @ t)
    assert np.linalg.norm(c - np.array([1.0, 2.0, -5.0])) < 1e-4


def test_identical_images_have_unit_ssim():
    """src/loss.rs:196-207."""
    w, h = 20, 14
    img = np.array([((i * 7919) % 255) / 255.0 for i in range(w * h * 3)], np.float32)
    s, g = O.ssim_with_grad(img, img, w, h)
    assert abs(s - 1.0) < 1e-4
    assert np.abs(g).max() < 1e-3


def _g(mean, log_scale, opacity):
    g = np.zeros(59, np.float32)
    g[0:3] = mean
    g[3:6] = log_scale
    g[6] = 1.0
    g[10] = opacity
    return g


def test_clone_split_prune_bookkeeping():
    """src/densify.rs:247-288: small+high grad clones, large+high grad splits,
    transparent prunes, ordinary stays; survivors keep the reference's order."""
    model = np.stack([
        _g(0.0, math.log(0.001), 2.0),
        _g(1.0, math.log(0.5), 2.0),
        _g(2.0, math.log(0.001), -10.0),
        _g(3.0, math.log(0.001), 2.0),
    ])
    m = np.zeros_like(model)
    v = np.zeros_like(model)
    normals = np.random.default_rng(1).standard_normal(64)
    p, m2, v2, rep = O.densify_and_prune(model, m, v, np.array([1.0, 1.0, 0.0, 0.0], np.float32),
                                         np.ones(4, np.uint32), np.zeros(4, np.uint32), 10.0, normals)
    assert rep[:3] == (1, 1, 1)
    assert rep[3] == 6  # one split parent, two children, three samples each
    assert p.shape[0] == 5 and m2.shape[0] == 5 and v2.shape[0] == 5
    assert (p[0, 0:3] == 0.0).all()
    assert (p[1, 0:3] == 3.0).all()
    assert (p[2, 0:3] == 0.0).all()
    expect = np.float32(math.log(0.5)) - np.float32(math.log(1.6))
    for child in p[3:5]:
        assert abs(child[3] - expect) < 1e-5


def test_retain_mask_keeps_order():
    """src/model.rs:248-253 (retain_by_mask), through the prune path of densify."""
    model = np.stack([_g(float(i), math.log(0.001), 2.0 if i % 2 == 0 else -10.0) for i in range(5)])
    z = np.zeros_like(model)
    p, _, _, rep = O.densify_and_prune(model, z, z, np.zeros(5, np.float32), np.zeros(5, np.uint32),
                                       np.zeros(5, np.uint32), 10.0, np.zeros(0))
    assert rep[:3] == (0, 0, 2)
    assert p[:, 0].tolist() == [0.0, 2.0, 4.0]


def test_nn_distances_match_brute_force():
    """src/model.rs:192-226."""
    rng = np.random.default_rng(12345)
    pts = rng.random((200, 3)).astype(np.float32)
    got = O.mean_nn_dist2(pts)
    p64 = pts.astype(np.float64)
    for i in range(len(pts)):
        d = ((p64 - p64[i]) ** 2).sum(1)
        d = np.sort(np.delete(d, i))
        want = (d[0] + d[1] + d[2]) / 3.0
        assert abs(got[i] - want) < 1e-5 * max(want, 1e-6)


def test_nn_distances_handle_many_coincident_points():
    """src/model.rs:228-246."""
    pts = np.zeros((42, 3), np.float32)
    pts[40] = [1, 0, 0]
    pts[41] = [0, 2, 0]
    got = O.mean_nn_dist2(pts)
    assert (got[:40] == 0.0).all()
    assert abs(got[40] - 1.0) < 1e-12
    assert abs(got[41] - 4.0) < 1e-12
    got = O.mean_nn_dist2(np.array([[0, 0, 0], [0, 0, 3]], np.float32))
    assert abs(got[0] - 9.0) < 1e-12 and abs(got[1] - 9.0) < 1e-12


def test_from_points_initialisation():
    """src/model.rs:77-104: scale from the 3-NN distance, identity rotation, opacity 0.1, DC colour."""
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 2, 0], [0, 0, 3]], np.float32)
    rgb = np.array([[255, 0, 128]] * 4, np.uint8)
    g = O.from_points(pts, rgb)
    d2 = O.mean_nn_dist2(pts)
    for i in range(4):
        ls = np.float32(math.log(math.sqrt(np.float32(d2[i]))))
        assert abs(g[i, 3] - ls) < 1e-6 and g[i, 3] == g[i, 4] == g[i, 5]
        assert g[i, 6:10].tolist() == [1, 0, 0, 0]
        assert abs(O.sigmoid(float(g[i, 10])) - 0.1) < 1e-6
        assert abs(g[i, 11] * F.SH_C0 + 0.5 - 1.0) < 1e-6


def test_crmath_matches_exact_values():
    """The correctly rounded exp/log that the CUDA kernels use, against 60-digit decimal
    arithmetic on a spread of inputs (the exhaustive sweep over every float is too slow
    for the unit suite)."""
    from decimal import Decimal, getcontext
    getcontext().prec = 60
    L = O.lib()
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.uniform(-103, 88, 3000), rng.uniform(-6, 0, 3000),
                         rng.uniform(-1e-3, 1e-3, 1000)]).astype(np.float32)
    for x in xs:
        got = np.float32(L.ora_expf_cr(float(x)))
        exact = Decimal(float(x)).exp()
        cands = [got, np.nextafter(got, np.float32(np.inf)), np.nextafter(got, np.float32(-np.inf))]
        best = min(cands, key=lambda c: abs(Decimal(float(c)) - exact))
        assert best == got, f"exp({x!r})"
    ys = np.concatenate([rng.uniform(1e-6, 300, 3000), rng.uniform(0.5, 2, 2000)]).astype(np.float32)
    for y in ys:
        got = np.float32(L.ora_logf_cr(float(y)))
        exact = Decimal(float(y)).ln()
        cands = [got, np.nextafter(got, np.float32(np.inf)), np.nextafter(got, np.float32(-np.inf))]
        best = min(cands, key=lambda c: abs(Decimal(float(c)) - exact))
        assert best == got, f"log({y!r})"


def test_psnr_clamps_and_handles_identity():
    """src/loss.rs:175-190."""
    a = np.array([0.5, 1.5, -0.2], np.float32)
    assert O.psnr(a, a) == float("inf")
    b = np.array([0.5, 1.0, 0.0], np.float32)
    assert O.psnr(a, b) == float("inf")
    c = np.array([0.4, 1.0, 0.0], np.float32)
    mse = (np.float64(np.float32(0.5)) - np.float64(np.float32(0.4))) ** 2 / 3
    assert abs(O.psnr(a, c) - (-10 * math.log10(mse))) < 1e-4


def test_splitmix_bulk_equals_single_draws():
    """The bulk generator used by the densification parity tests draws the same normals,
    and leaves the same state, as single draws."""
    s1 = np.array([1234], np.uint64)
    one = np.array([O.lib().ora_splitmix_normal(s1.ctypes.data) for _ in range(1000)])
    s2 = np.array([1234], np.uint64)
    bulk = O.splitmix_normals(s2, 1000)
    assert np.array_equal(one, bulk) and s1[0] == s2[0]
