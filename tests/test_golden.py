"""The oracle against the committed golden fixtures (tests/golden/, made by
tests/golden/make_golden.py): a drift check of the checker itself, so that a change of
compiler, flags or oracle code that moves any result fails here before any GPU comparison is
trusted. CPU only."""
import numpy as np
import pytest

from oracle import mlp as M
from oracle import oracle as O
from tests.golden import make_golden as MG

RENDER_INPUTS = ("params", "cam", "background", "dimage", "antialias", "sh_degree")


def load(path):
    with np.load(path) as d:
        return {k: d[k] for k in d.files}


@pytest.fixture(scope="module")
def render_golden():
    return load(MG.RENDER_FILE)


def same_bits(a, b):
    a, b = np.atleast_1d(np.asarray(a)), np.atleast_1d(np.asarray(b))
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("threads", [1, 4])
def test_oracle_reproduces_render_golden(render_golden, threads):
    """Correctly rounded exp/log (the kernels' mode): every output of projection, binning,
    compositing forward and backward and projection backward bit-identical to the fixture,
    whatever the oracle's thread count."""
    inp = {k: render_golden[k] for k in RENDER_INPUTS}
    old = O.threads()
    O.set_threads(threads)
    O.set_cr_math(True)
    try:
        out = MG.render_outputs(inp)
    finally:
        O.set_cr_math(False)
        O.set_threads(old)
    bad = [k for k in out if not same_bits(out[k], render_golden[k])]
    assert not bad, f"oracle drifted from the golden vectors in {bad}"


def test_libm_oracle_near_render_golden(render_golden):
    """The faithful mode (host libm, as the reference's f32 build) differs from the fixture
    only where glibc's expf/logf misround: same tile lists and contributor counts, image and
    gradients within a few float32 ulps."""
    inp = {k: render_golden[k] for k in RENDER_INPUTS}
    out = MG.render_outputs(inp)
    for k in ("proj", "tile_range", "gauss", "n_contrib", "pairs", "bwd_pairs"):
        assert same_bits(out[k], render_golden[k]), k
    img_err = np.abs(out["image"] - render_golden["image"]).max()
    g = render_golden["param_grads"]
    g_err = (np.abs(out["param_grads"] - g).max(0) / np.maximum(np.abs(g).max(0), 1e-30)).max()
    print(f"\nlibm oracle vs golden: image max-abs {img_err:.2e}, parameter gradients rel. {g_err:.2e}")
    assert img_err <= 1e-6 and g_err <= 1e-5


def test_render_golden_covers_edge_cases(render_golden):
    """The fixture holds what the reference's tests exercise: a ragged view, culled
    Gaussians with zero gradients, multi-tile Gaussians, and depth ties (exact duplicates)
    ordered by entry index inside every tile."""
    d = render_golden
    w, h = int(d["cam"][0]), int(d["cam"][1])
    assert w % 16 and h % 16 and d["tile_range"].shape[0] == ((w + 15) // 16) * ((h + 15) // 16)
    culled = d["proj"][:, 6] == 0
    assert culled.sum() >= 10 and not d["param_grads"][culled].any() and not d["screen_grads"][culled].any()
    tiles_per = np.bincount(d["gauss"], minlength=d["params"].shape[0])
    assert tiles_per.max() >= 6
    ties = 0
    for s, e in d["tile_range"]:
        lst = d["gauss"][s:e].tolist()
        for j in range(100, 110):
            if j in lst and j + 100 in lst:
                ties += 1
                assert lst.index(j) < lst.index(j + 100)
    assert ties >= 10
    assert (d["n_contrib"] > 0).mean() > 0.5 and int(d["pairs"]) > 0 and int(d["bwd_pairs"]) > 0


def test_passed_pair_counters(render_golden):
    """The counters behind the CPU baseline's ns per pair per core: pairs passing the alpha
    threshold are a subset of the evaluated ones; the backward walks only entries before a
    pixel's last contributor, so it never passes more than the forward."""
    inp = {k: render_golden[k] for k in RENDER_INPUTS}
    MG.render_outputs(inp)
    fwd, bwd = O.last_passed_pairs()
    assert 0 < bwd <= fwd <= int(render_golden["pairs"])
    assert bwd <= int(render_golden["bwd_pairs"])


def test_oracle_reproduces_mlp_golden():
    """The network oracle (bf16 mode) on the fixture's rows: probabilities and gradient as
    stored, to float64 rounding (numpy's exp may differ by an ulp between CPUs)."""
    d = load(MG.MLP_FILE)
    probs, _ = M.forward(d["theta"], d["x"], bf16_like=True)
    grad = M.backward(d["theta"], d["x"], d["y"], d["w"], bf16_like=True)
    assert np.allclose(probs, d["probs"], rtol=1e-12, atol=1e-15)
    assert np.allclose(grad, d["grad"], rtol=1e-10, atol=1e-15)
    assert d["theta"].shape == (M.NUM_PARAMS,) and d["x"].shape == (256, M.IN)
