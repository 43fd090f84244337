"""The CUDA path through the C ABI against the committed golden fixtures (tests/golden/):
the same bars as the stage-by-stage parity tests, on inputs and answers that are fixed in
the repository instead of recomputed by the oracle at test time.

Bars: projection records, tile lists, images, final transmittance, contributor counts and
the projection backward's 59 gradients bit-identical (the fixture was computed with the
correctly rounded exp/log the kernels use); screen-space and end-to-end parameter gradients
within 1e-3 of each quantity's scale; the network's probabilities within 5e-3 and its
gradient within 2e-2 relative (bf16 operands, sums in another order)."""
import numpy as np
import pytest
import torch

from oracle import mlp as M
from splatrs_b200 import gpu as G
from splatrs_b200._lib import Camera, ProjOpts
from tests.golden import make_golden as MG

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def gold():
    with np.load(MG.RENDER_FILE) as d:
        return {k: d[k] for k in d.files}


def dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def grad_rel_error(got, want):
    scale = np.maximum(np.abs(want).max(0), 1e-30)
    return np.abs(got - want).max(0) / scale


def setup(gold):
    g, cam = gold["params"], gold["cam"]
    opts = dict(antialias=bool(gold["antialias"]), sh_degree=int(gold["sh_degree"]))
    return g, cam, opts, int(cam[0]), int(cam[1]), gold["background"]


def test_projection_equals_golden(ctx, gold):
    g, cam, opts, _, _, _ = setup(gold)
    planes = G.params_to_planes(ctx, dev(g))
    proj = G.project_all(ctx, planes, g.shape[0], g.shape[0], Camera.from_record(cam), ProjOpts.make(**opts))
    got = proj.to_reference(ctx).cpu().numpy()
    mism = (bits(got) != bits(gold["proj"])).any(1)
    assert mism.sum() == 0, f"{mism.sum()} projections differ, first {np.nonzero(mism)[0][:5]}"


def test_binning_and_forward_equal_golden(ctx, gold):
    """Fed the fixture's projections: tile lists (with the duplicates' depth ties), image,
    final transmittance, contributor counts and evaluated pairs identical."""
    _, _, _, w, h, bg = setup(gold)
    proj = G.proj_from_reference(ctx, dev(gold["proj"]), w, h)
    b = G.bin(ctx, proj)
    assert b.num_entries == gold["gauss"].size
    assert (b.gauss.cpu().numpy().view(np.uint32) == gold["gauss"]).all()
    assert (b.tile_range.cpu().numpy().view(np.uint32) == gold["tile_range"]).all()
    out = G.rasterize_forward(ctx, proj, b, bg)
    assert (bits(out.image.cpu().numpy()) == bits(gold["image"])).all()
    assert (bits(out.final_t.cpu().numpy()) == bits(gold["final_t"])).all()
    assert (out.n_contrib.cpu().numpy().view(np.uint32) == gold["n_contrib"]).all()
    assert int(out.pairs.item()) == int(gold["pairs"])


def test_backward_matches_golden(ctx, gold):
    """Compositing backward fed the fixture's projections and dL/dpix: ProjGrad and the
    AbsGS accumulators within 1e-3 of each quantity's scale; culled Gaussians get none."""
    g, _, _, w, h, bg = setup(gold)
    proj = G.proj_from_reference(ctx, dev(gold["proj"]), w, h)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    pairs = torch.zeros(1, dtype=torch.int64, device="cuda")
    pg = G.rasterize_backward(ctx, proj, b, bg, out, dev(gold["dimage"]), pairs=pairs)
    gg, ga = G.pgrad_to_reference(pg, g.shape[0])
    gg, ga = gg.cpu().numpy(), ga.cpu().numpy()
    assert int(pairs.item()) == int(gold["bwd_pairs"])
    err = grad_rel_error(gg, gold["screen_grads"])
    assert err.max() < 1e-3, err
    assert grad_rel_error(ga, gold["screen_abs"]).max() < 1e-3
    culled = gold["proj"][:, 6] == 0
    assert not gg[culled].any()


def test_project_backward_equals_golden(ctx, gold):
    """Projection backward fed the fixture's screen-space gradients: the 59 parameter
    gradients bit-identical."""
    g, cam, opts, _, _, _ = setup(gold)
    n = g.shape[0]
    planes = G.params_to_planes(ctx, dev(g))
    proj = G.project_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(**opts))
    pg = G.pgrad_from_reference(dev(gold["screen_grads"]))
    gp = G.project_backward_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(**opts), proj, pg)
    got = G.planes_to_params(ctx, gp, n, n).cpu().numpy()
    mism = (bits(got) != bits(gold["param_grads"])).any(1)
    assert mism.sum() == 0, f"{mism.sum()} gradient records differ, first {np.nonzero(mism)[0][:5]}"


def test_end_to_end_chain_matches_golden(ctx, gold):
    """Parameters -> ... -> parameter gradients, all on the GPU: image identical, gradients
    within 1e-3 of each parameter's scale."""
    g, cam, opts, _, _, bg = setup(gold)
    n = g.shape[0]
    planes = G.params_to_planes(ctx, dev(g))
    proj = G.project_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(**opts))
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    pg = G.rasterize_backward(ctx, proj, b, bg, out, dev(gold["dimage"]))
    gp = G.project_backward_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(**opts), proj, pg)
    got = G.planes_to_params(ctx, gp, n, n).cpu().numpy()
    assert (bits(out.image.cpu().numpy()) == bits(gold["image"])).all()
    want = gold["param_grads"]
    active = np.abs(want).max(0) > 0
    err = grad_rel_error(got, want)
    assert err[active].max() < 1e-3, err


@pytest.mark.parametrize("tcgen05", [False, True])
def test_mlp_matches_golden(ctx, tcgen05):
    with np.load(MG.MLP_FILE) as d:
        d = {k: d[k] for k in d.files}
    tth = dev(d["theta"])
    probs = G.mlp_forward(ctx, dev(d["x"]), tth, tcgen05=tcgen05).cpu().numpy()
    assert np.abs(probs - d["probs"]).max() < 5e-3
    grad = G.mlp_grad(ctx, dev(d["x"]), dev(d["y"], torch.int32), dev(d["w"]), tth,
                      tcgen05=tcgen05).cpu().numpy().astype(np.float64)
    o = 0
    for name, shape in M.SIZES:
        k = int(np.prod(shape))
        a, b = grad[o:o + k], d["grad"][o:o + k]
        rel = np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)
        assert rel < 2e-2, f"{name}: {rel:.2e}"
        o += k
