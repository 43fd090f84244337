"""The learned-densification network's tensor-core kernels against the CPU oracle
(oracle/mlp.py): probabilities and parameter gradients in the oracle's bf16 mode (same
rounding points, so differences come from accumulation order and the hardware tanh in
SiLU), each also reported against the float64 oracle; the tcgen05 forward against both
the oracle and the mma.sync forward; Adam; and a learning sanity check."""
import numpy as np
import pytest
import torch

from oracle import mlp as M
from splatrs_b200 import gpu as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def _case(seed, n):
    rng = np.random.default_rng(seed)
    theta = M.init_params(seed)
    theta[M.NUM_PARAMS - 3:] = rng.normal(0, 0.3, 3)
    x = rng.normal(0, 1, (n, M.IN))
    y = rng.integers(0, M.OUT, n)
    w = rng.uniform(0.2, 2.0, n)
    return theta, x, y, w


def _t(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


@pytest.mark.parametrize("n", [1, 37, 1000, 4099])
def test_mlp_forward_matches_oracle(ctx, n):
    theta, x, _, _ = _case(10 + n, n)
    got = G.mlp_forward(ctx, _t(x), _t(theta)).cpu().numpy()
    want, _ = M.forward(theta, x, bf16_like=True)
    assert np.abs(got - want).max() < 5e-3
    p64, _ = M.forward(theta, x)
    print(f"\nn={n}: probabilities max-abs vs bf16 oracle {np.abs(got - want).max():.2e}, "
          f"vs f64 oracle {np.abs(got - p64).max():.2e}")


@pytest.mark.parametrize("n", [1, 127, 128, 129, 4099, 100_000])
def test_mlp_forward_tcgen05_matches_oracle(ctx, n):
    """The tcgen05 forward (accumulators in tensor memory) against the bf16 oracle and the
    mma.sync forward: same rounding points, sums in another order, so a hidden activation
    may round to the neighbouring BF16 value; probabilities agree to well under 5e-3."""
    theta, x, _, _ = _case(50 + n, n)
    tx, tth = _t(x), _t(theta)
    got = G.mlp_forward(ctx, tx, tth, tcgen05=True).cpu().numpy()
    ref = G.mlp_forward(ctx, tx, tth).cpu().numpy()
    m = min(n, 4099)
    want, _ = M.forward(theta, x[:m], bf16_like=True)
    assert np.isfinite(got).all()
    assert np.abs(got[:m] - want).max() < 5e-3
    assert np.abs(got - ref).max() < 5e-3
    assert np.abs(got.sum(1) - 1.0).max() < 1e-5
    print(f"\nn={n}: tcgen05 max-abs vs bf16 oracle {np.abs(got[:m] - want).max():.2e}, "
          f"vs mma.sync {np.abs(got - ref).max():.2e}, equal rows {np.mean(np.all(got == ref, 1)):.3f}")


def test_bounded_wait_times_out_and_context_stays_usable(ctx):
    """The tensor-core kernels' bounded mbarrier wait, run out on purpose (nothing arrives;
    4096 tries): SPLAT_ERR_TIMEOUT through the kernels' error word. The same wait with the
    phase completed first succeeds, and the context keeps working: the tcgen05 forward still
    matches the oracle afterwards."""
    from splatrs_b200._lib import SplatError
    G.diag_mbarrier_wait(ctx, 4096, True)
    with pytest.raises(SplatError) as e:
        G.diag_mbarrier_wait(ctx, 4096, False)
    assert e.value.status == 4
    G.diag_mbarrier_wait(ctx, 4096, True)
    theta, x, _, _ = _case(90, 300)
    got = G.mlp_forward(ctx, _t(x), _t(theta), tcgen05=True).cpu().numpy()
    want, _ = M.forward(theta, x, bf16_like=True)
    assert np.abs(got - want).max() < 5e-3


def test_mlp_forward_tcgen05_empty_and_repeated(ctx):
    theta, x, _, _ = _case(70, 300)
    empty = G.mlp_forward(ctx, _t(x[:0]), _t(theta), tcgen05=True)
    assert empty.shape == (0, 3)
    a = G.mlp_forward(ctx, _t(x), _t(theta), tcgen05=True).cpu().numpy()
    b = G.mlp_forward(ctx, _t(x), _t(theta), tcgen05=True).cpu().numpy()
    assert np.array_equal(a, b)


@pytest.mark.parametrize("n", [64, 1000])
def test_mlp_gradient_matches_oracle(ctx, n):
    theta, x, y, w = _case(20 + n, n)
    got = G.mlp_grad(ctx, _t(x), _t(y, torch.int32), _t(w), _t(theta)).cpu().numpy().astype(np.float64)
    want = M.backward(theta, x, y, w, bf16_like=True)
    g64 = M.backward(theta, x, y, w)
    o = 0
    for name, shape in M.SIZES:
        k = int(np.prod(shape))
        a, b, c = got[o:o + k], want[o:o + k], g64[o:o + k]
        rel = np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)
        print(f"\n{name}: rel. error vs bf16 oracle {rel:.2e}, vs f64 oracle "
              f"{np.abs(a - c).max() / max(np.abs(c).max(), 1e-30):.2e}")
        assert rel < 2e-2, name
        o += k


@pytest.mark.parametrize("n", [1, 100, 128, 129, 1000, 40_000])
def test_mlp_gradient_tcgen05_matches_oracle(ctx, n):
    """The tcgen05 gradient (layer outputs and weight gradients in tensor memory, the
    weight gradients as stacked M = 128 products over the rows) against the bf16 oracle and
    the mma.sync kernel: same rounding points, sums in another order."""
    theta, x, y, w = _case(80 + n % 97, n)
    tx, ty, tw, tth = _t(x), _t(y, torch.int32), _t(w), _t(theta)
    got = G.mlp_grad(ctx, tx, ty, tw, tth, tcgen05=True).cpu().numpy().astype(np.float64)
    ref = G.mlp_grad(ctx, tx, ty, tw, tth).cpu().numpy().astype(np.float64)
    m = min(n, 4000)
    want = M.backward(theta, x[:m], y[:m], w[:m], bf16_like=True) if n <= 4000 else None
    o = 0
    for name, shape in M.SIZES:
        k = int(np.prod(shape))
        a, r = got[o:o + k], ref[o:o + k]
        assert np.isfinite(a).all(), name
        scale = max(np.abs(r).max(), 1e-30)
        rel_ref = np.abs(a - r).max() / scale
        msg = f"{name}: rel. vs mma.sync {rel_ref:.2e}"
        assert rel_ref < 2e-2, msg
        if want is not None:
            b = want[o:o + k]
            rel = np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)
            msg += f", vs bf16 oracle {rel:.2e}"
            assert rel < 2e-2, msg
        print("\n" + msg)
        o += k


def test_mlp_adam_matches_oracle(ctx):
    rng = np.random.default_rng(30)
    theta = rng.normal(0, 1, M.NUM_PARAMS).astype(np.float32)
    t = _t(theta)
    m, v = torch.zeros_like(t), torch.zeros_like(t)
    mo, vo = np.zeros(M.NUM_PARAMS, np.float32), np.zeros(M.NUM_PARAMS, np.float32)
    for step in (1, 2, 3):
        g = rng.normal(0, 1e-2, M.NUM_PARAMS).astype(np.float32)
        G.check(ctx.lib.splat_mlp_adam(ctx.h, G._ptr(t), G._ptr(_t(g)), G._ptr(m), G._ptr(v), step, 1e-3), ctx.h)
        theta = M.adam(theta, g, mo, vo, step, 1e-3)
    assert np.abs(t.cpu().numpy() - theta).max() < 1e-6


def test_mlp_learns_a_separable_rule(ctx):
    """Trained on the device (grad + Adam) it learns a three-way rule of the features."""
    rng = np.random.default_rng(40)
    x = rng.normal(0, 1, (4000, M.IN))
    y = np.where(x[:, 0] > 0.5, 1, np.where(x[:, 1] < -0.5, 2, 0))
    theta = _t(M.init_params(1))
    m, v = torch.zeros_like(theta), torch.zeros_like(theta)
    xt, yt, wt = _t(x), _t(y, torch.int32), _t(np.ones(len(y)))
    for step in range(1, 301):
        g = G.mlp_grad(ctx, xt, yt, wt, theta)
        G.check(ctx.lib.splat_mlp_adam(ctx.h, G._ptr(theta), G._ptr(g), G._ptr(m), G._ptr(v), step, 3e-3), ctx.h)
    acc = (G.mlp_forward(ctx, xt, theta).argmax(1).cpu().numpy() == y).mean()
    print(f"\naccuracy after 300 steps: {acc:.3f}")
    assert acc > 0.95
