"""The compositing backward's decision procedure, emulated on the host over a projected scene
and compared with the reference's rule, with the correctly rounded exp of the oracle.

The reference takes a pixel for an entry when !(sigma < 0), !(sigma > sigma_max) and
!(fl(opacity * exp(-sigma)) < 1/255), and clamps alpha when opacity * exp(-sigma) >= 0.99
(src/rasterize.rs:231-244, :414-432). The paired backward decides the first from sigma alone
when sigma <= fl(sigma_max - 1e-4), evaluates the correctly rounded exp only between that
threshold and sigma_max, and treats an entry with opacity < 0.99 as never clamped. Here both
procedures run over every (Gaussian, pixel) pair of the Gaussians' tile rectangles in a
320x240 scene, in float32 with the reference's operation order; their decisions must agree
pair for pair."""
import numpy as np

from oracle import oracle as O
from splatrs_b200 import scenes

ALPHA_MIN = np.float32(1.0) / np.float32(255.0)
ALPHA_MAX = np.float32(0.99)
EDGE = np.float32(1e-4)


def test_sigma_threshold_decisions_equal_the_reference_rule():
    rng = np.random.default_rng(11)
    w, h = 320, 240
    g = scenes.random_gaussians(rng, 2000, -1.0, 1.0, -3.5, 0.5, 1.2)
    g[::9, 10] = 5.0  # opacities near 1, so that clamping occurs
    cam = scenes.look_at(w, h, 0.9 * w, 0.9 * w, (0.4, -0.3, -3.2), (0, 0, 0))
    O.set_cr_math(True)
    try:
        p = O.project_all(g, cam, sh_degree=1)
    finally:
        O.set_cr_math(False)
    lib = O.lib()
    cr_exp = np.vectorize(lambda x: lib.ora_expf_cr(float(x)), otypes=[np.float32])
    vis = p[:, 6].view(np.uint32) > 0 if p.dtype == np.float32 else p[:, 6] > 0
    taken = edge_pairs = clamped = 0
    for k in np.nonzero(vis)[0]:
        mx, my, A, B, C = (np.float32(v) for v in p[k, :5])
        op = np.float32(p[k, 7])
        tx0, ty0, tx1, ty1 = (int(v) for v in p[k, 11:15])
        xs = np.arange(tx0 * 16, min(tx1 * 16, w), dtype=np.float32) + np.float32(0.5)
        ys = np.arange(ty0 * 16, min(ty1 * 16, h), dtype=np.float32) + np.float32(0.5)
        px, py = np.meshgrid(xs, ys)
        dx, dy = px - mx, py - my
        sigma = np.float32(0.5) * (A * dx * dx + C * dy * dy) + B * dx * dy
        smax = np.float32(lib.ora_logf_cr(float(op / ALPHA_MIN)))
        smaxd = np.float32(smax - EDGE)
        inr = ~(sigma < 0) & ~(sigma > smax)
        s_in = sigma[inr]
        og = op * cr_exp(-s_in)  # float32 product of the correctly rounded exp
        ref = ~(og < ALPHA_MIN)
        fast = s_in <= smaxd
        dev = fast | (~fast & ~(og < ALPHA_MIN))
        assert (dev == ref).all(), (k, int((dev != ref).sum()))
        # An entry below 0.99 never clamps.
        if op < ALPHA_MAX:
            assert (og[ref] < ALPHA_MAX).all()
        else:
            clamped += int((og[ref] >= ALPHA_MAX).sum())
        taken += int(ref.sum())
        edge_pairs += int((~fast).sum())
    assert taken > 100_000
    print(f"\n{taken} taken pairs; {edge_pairs} in-range pairs within 1e-4 of sigma_max took the "
          f"correctly rounded exp; {clamped} clamped")
