"""Finite-difference gradient checks of the CPU oracle: a replay of the reference's
tests/gradcheck.rs (f32 and f64) and tests/gradcheck_f64.rs (f64 only), with numpy draws
in place of ChaCha8. They pin the hand-derived backward passes that the CUDA kernels are
then compared against."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import fixtures as F

DTYPES = [np.float32, np.float64]


@pytest.mark.parametrize("dt", DTYPES)
def test_sh_basis_gradient(dt):
    """tests/gradcheck.rs:21-47."""
    rng = np.random.default_rng(7)
    H = F.TOL[dt]["H"]
    for _ in range(20):
        d = rng.uniform(-1, 1, 3)
        d = d / np.linalg.norm(d)
        g = O.sh_basis_grad(3, d, dt)
        for axis in range(3):
            for k in range(16):
                def f(e):
                    p = d.copy()
                    p[axis] += e
                    return float(O.sh_basis(3, p, dt)[k])
                F.check(f"basis[{k}] d/d{axis}", float(g[k, axis]), F.central(0.0, H, f), 1.0, dt)


def _proj_loss(p, w):
    """tests/gradcheck.rs:50-60: a random linear functional of the screen quantities."""
    return float(w[0] * p[0] + w[1] * p[1] + w[2] * p[2] + w[3] * p[3] + w[4] * p[4]
                 + w[6] * p[8] + w[7] * p[9] + w[8] * p[10] + w[5] * p[7])


def _random_weights(rng):
    return np.array([F.rnd(rng, -1, 1) for _ in range(9)])


def _check_projection(cam, g, opts, rng, label, dt):
    """tests/gradcheck.rs:79-105."""
    H = F.TOL[dt]["H"]
    base = O.project_all(g[None], cam, dtype=dt, **opts)[0]
    assert base[6] > 0, f"{label}: test Gaussian must be visible"
    w = _random_weights(rng)
    analytic = O.project_backward_all(g[None], cam, w[None], dtype=dt, **opts)[0]
    scale = 1.0 + abs(float(base[2])) + abs(float(base[4]))
    for i in range(59):
        def f(e):
            gg = g.astype(dt).copy()
            gg[i] += e
            p = O.project_all(gg[None], cam, dtype=dt, **opts)[0]
            assert p[6] > 0, f"{label}: perturbed Gaussian left the view"
            return _proj_loss(p.astype(np.float64), w)
        F.check(f"{label} {F.param_name(i)}", float(analytic[i]), F.central(0.0, H, f), scale, dt)


@pytest.mark.parametrize("dt", DTYPES)
def test_projection_gradient_plain(dt):
    """tests/gradcheck.rs:107-120."""
    rng = np.random.default_rng(11)
    cam = F.test_camera(96, 64, dt)
    for n in range(12):
        g = F.random_gaussian(rng)
        _check_projection(cam, g, dict(antialias=False, sh_degree=3), rng, f"plain #{n}", dt)


@pytest.mark.parametrize("dt", DTYPES)
def test_projection_gradient_antialiased(dt):
    """tests/gradcheck.rs:122-135."""
    rng = np.random.default_rng(12)
    cam = F.test_camera(96, 64, dt)
    for n in range(12):
        g = F.random_gaussian(rng)
        _check_projection(cam, g, dict(antialias=True, sh_degree=3), rng, f"antialiased #{n}", dt)


@pytest.mark.parametrize("dt", DTYPES)
def test_projection_gradient_lower_degrees(dt):
    """tests/gradcheck.rs:137-150."""
    rng = np.random.default_rng(13)
    cam = F.test_camera(96, 64, dt)
    for degree in range(3):
        g = F.random_gaussian(rng)
        _check_projection(cam, g, dict(antialias=False, sh_degree=degree), rng, f"degree {degree}", dt)


@pytest.mark.parametrize("dt", DTYPES)
def test_projection_gradient_with_jacobian_clamping(dt):
    """tests/gradcheck.rs:152-181: a large Gaussian past the clamp limit."""
    rng = np.random.default_rng(14)
    cam = O.look_at(64, 48, 60.0, 60.0, [0, 0, -2.0], [0, 0, 0], [0, -1, 0], dt)
    g = F.random_gaussian(rng)
    g[0:3] = [3.2, 0.1, 0.0]
    g[3:6] = [0.4, 0.4, 0.4]
    rot = cam[6:15].astype(np.float64).reshape(3, 3)
    t = rot @ g[0:3] + cam[15:18]
    lim = (cam[0] - cam[4]) / cam[2] + 0.3 * 0.5 * cam[0] / cam[2]
    assert t[0] / t[2] > lim, "test setup: Gaussian must be past the clamp limit"
    _check_projection(cam, g, dict(antialias=True, sh_degree=2), rng, "clamped", dt)


# ---------------------------------------------------------------------------------------
# tests/gradcheck_f64.rs (double precision only)
# ---------------------------------------------------------------------------------------
H_CONIC = 1e-6
D = np.float64


def random_projs(rng, width, height, n):
    """tests/gradcheck_f64.rs:28-55: screen-space Gaussians covering the image."""
    tx, ty = (width + 15) // 16, (height + 15) // 16
    out = np.zeros((n, 15))
    for i in range(n):
        l00 = F.rnd(rng, 1.5, 4.0)
        l10 = F.rnd(rng, -2.0, 2.0)
        l11 = F.rnd(rng, 1.5, 4.0)
        a, b, c = l00 * l00, l00 * l10, l10 * l10 + l11 * l11
        det = a * c - b * b
        out[i, 0:2] = [F.rnd(rng, 4.0, width - 4.0), F.rnd(rng, 4.0, height - 4.0)]
        out[i, 2:5] = [c / det, -b / det, a / det]
        out[i, 5] = 1.0 + i * 0.37
        out[i, 6] = 1000
        out[i, 7] = F.rnd(rng, 0.3, 0.9)
        out[i, 8:11] = [F.rnd(rng, 0, 1) for _ in range(3)]
        out[i, 11:15] = [0, 0, tx, ty]
    return out


def _raster_loss(projs, w, h, bg, weights):
    b = O.bin(projs, w, h, D)
    img, _, _, _ = O.rasterize_forward(projs, b, w, h, bg, D)
    return float(img @ weights)


def test_rasterizer_gradient():
    """tests/gradcheck_f64.rs:63-104, including the AbsGS bound."""
    rng = np.random.default_rng(21)
    w, h = 40, 28
    bg = np.array([0.2, 0.5, 0.8])
    projs = random_projs(rng, w, h, 9)
    weights = rng.uniform(-1, 1, w * h * 3)
    b = O.bin(projs, w, h, D)
    img, ft, nc, _ = O.rasterize_forward(projs, b, w, h, bg, D)
    grads, absg, _ = O.rasterize_backward(projs, b, w, h, bg, ft, nc, weights, D)
    col = {0: 0, 1: 1, 2: 2, 3: 3, 4: 4, 5: 7, 6: 8, 7: 9, 8: 10}
    for i in range(projs.shape[0]):
        for field in range(9):
            hh = H_CONIC if 2 <= field <= 4 else F.TOL[D]["H"]
            def f(e):
                p = projs.copy()
                p[i, col[field]] += e
                return _raster_loss(p, w, h, bg, weights)
            F.check(f"gaussian {i} field {field}", float(grads[i, field]), F.central(0.0, hh, f), 1.0, D)
        assert absg[i, 0] + 1e-9 >= abs(grads[i, 0])
        assert absg[i, 1] + 1e-9 >= abs(grads[i, 1])


def test_ssim_gradient():
    """tests/gradcheck_f64.rs:106-122."""
    rng = np.random.default_rng(31)
    w, h = 18, 13
    x = rng.uniform(0, 1, w * h * 3)
    y = rng.uniform(0, 1, w * h * 3)
    _, grad = O.ssim_with_grad(x, y, w, h, D)
    for _ in range(40):
        i = int(rng.integers(0, x.size))
        def f(e):
            xp = x.copy()
            xp[i] += e
            return O.ssim_with_grad(xp, y, w, h, D)[0]
        F.check(f"ssim d/dx[{i}]", float(grad[i]), F.central(0.0, F.TOL[D]["H"], f), 1.0, D)


def test_photometric_loss_gradient():
    """tests/gradcheck_f64.rs:124-140."""
    rng = np.random.default_rng(32)
    w, h = 16, 12
    x = rng.uniform(0, 1, w * h * 3)
    y = rng.uniform(0, 1, w * h * 3)
    _, grad = O.photometric_loss(x, y, w, h, 0.2, D)
    for _ in range(40):
        i = int(rng.integers(0, x.size))
        def f(e):
            xp = x.copy()
            xp[i] += e
            return O.photometric_loss(xp, y, w, h, 0.2, D)[0]
        F.check(f"loss d/dx[{i}]", float(grad[i]), F.central(0.0, F.TOL[D]["H"], f), 1.0, D)


def test_end_to_end_gradient():
    """tests/gradcheck_f64.rs:146-216: parameters -> projection -> rasterization -> loss."""
    rng = np.random.default_rng(41)
    cam = F.test_camera(48, 32, D)
    w, h = 48, 32
    gs = []
    for _ in range(6):
        g = F.random_gaussian(rng)
        g[3:6] = [F.rnd(rng, -1.6, -0.9) for _ in range(3)]
        gs.append(g)
    model = np.stack(gs)
    target = rng.uniform(0, 1, w * h * 3)
    opts = dict(antialias=True, sh_degree=3)
    bg = np.array([0.1, 0.1, 0.1])

    def loss_of(m):
        projs = O.project_all(m, cam, dtype=D, **opts)
        b = O.bin(projs, w, h, D)
        img, _, _, _ = O.rasterize_forward(projs, b, w, h, bg, D)
        return O.photometric_loss(img, target, w, h, 1.0, D)[0]

    projs = O.project_all(model, cam, dtype=D, **opts)
    assert (projs[:, 6] > 0).all()
    b = O.bin(projs, w, h, D)
    img, ft, nc, _ = O.rasterize_forward(projs, b, w, h, bg, D)
    _, dimage = O.photometric_loss(img, target, w, h, 1.0, D)
    pg, _, _ = O.rasterize_backward(projs, b, w, h, bg, ft, nc, dimage, D)
    grads = O.project_backward_all(model, cam, pg, dtype=D, **opts)
    hh = 1e-5
    for gi in range(model.shape[0]):
        for i in range(59):
            def f(e):
                m = model.copy()
                m[gi, i] += e
                return loss_of(m)
            F.check(f"gaussian {gi} {F.param_name(i)}", float(grads[gi, i]), F.central(0.0, hh, f), 1.0, D)
