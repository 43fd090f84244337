"""The bound behind the compositing backward's alpha decisions, checked on the host.

The reference skips a pixel when fl(opacity * exp(-sigma)) < 1/255 (src/rasterize.rs:231-244);
the projection stores sigma_max = ln(opacity / (1/255)) (quotient and logarithm correctly
rounded, as TileGauss::new computes it, rasterize.rs:149-182). The device backward takes the
alpha test from sigma alone when sigma <= fl(sigma_max - 1e-4): the product is then at least
(1/255) e^(1e-4 - 7.2e-7) (1 - 2^-23) whatever the exp's rounding. fl(opacity * exp(-sigma))
does not increase with sigma, so the largest such sigma decides: this test evaluates
opacity * exp(-fl(sigma_max - 1e-4)) in double precision, whose error is far below the
margin, for 4M opacities spread over (1/255, 1] and the edge values, and requires it to
clear 1/255 by more than the float roundings that follow (so the float product clears it
too). No GPU: the check is of the inequality, which the kernel relies on as stated."""
import numpy as np

ALPHA_MIN = np.float32(1.0) / np.float32(255.0)
SIGMA_EDGE = np.float32(1e-4)


def sigma_max_of(opacity):
    """sigma_max as the projection computes it: the float quotient, then the logarithm
    rounded to float (double precision's logarithm rounds to the same float except in
    cases within 2^-29 of a midpoint, which the 1e-4 margin absorbs)."""
    q = (opacity / ALPHA_MIN).astype(np.float32)
    return np.log(q.astype(np.float64)).astype(np.float32)


def test_sigma_threshold_implies_alpha_test():
    rng = np.random.default_rng(7)
    op = rng.uniform(float(ALPHA_MIN), 1.0, 4_000_000).astype(np.float32)
    edges = np.array([np.nextafter(ALPHA_MIN, np.float32(2)), ALPHA_MIN * np.float32(1.0001), np.float32(0.5),
                      np.float32(0.98999), np.float32(0.99), np.float32(0.999), np.float32(1.0)], np.float32)
    op = np.concatenate([op, edges])
    smax = sigma_max_of(op)
    smaxd = (smax - SIGMA_EDGE).astype(np.float32)  # as staged by the kernel, in float
    live = smaxd >= 0  # below that no pixel passes sigma >= 0 and sigma <= smaxd together
    og = op.astype(np.float64)[live] * np.exp(-smaxd.astype(np.float64)[live])
    # The float exp and the float product each round by at most 2^-24 relative.
    margin = og / float(ALPHA_MIN) - 1.0
    assert margin.min() > 2.0 ** -22, margin.min()
    # The margin is the 1e-4 of the threshold up to the roundings of sigma_max.
    assert margin.min() > 9e-5 and margin.max() < 1.2e-4, (margin.min(), margin.max())


def test_opacity_below_clamp_never_clamps():
    """fl(opacity * g) <= opacity for g <= 1 (rounding is monotone), so an entry with
    opacity < 0.99 never reaches the 0.99 clamp; the backward skips that test for it."""
    rng = np.random.default_rng(8)
    op = rng.uniform(0.0, 0.99, 1_000_000).astype(np.float32)
    op = op[op < np.float32(0.99)]
    g = rng.uniform(0.0, 1.0, op.shape[0]).astype(np.float32)
    g[:10] = np.float32(1.0)
    assert ((op * g).astype(np.float32) < np.float32(0.99)).all()
