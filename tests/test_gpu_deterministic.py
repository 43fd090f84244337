"""The deterministic compositing backward and the deterministic trainer against the
correctly rounded oracle, bit for bit, through the C ABI.

The reference's backward (src/rasterize.rs:341-505) stores every entry's gradient slots,
each summed over the entry's pixel rectangle in row-major order, and then sums every
Gaussian's entries in entry order: a fixed order. The default CUDA backward sums with float
atomics (unspecified order), which the 1e-3 bar covers; splat_rasterize_bwd_deterministic and
the trainer's `deterministic` mode reproduce the reference's order, so their results must be
bit-identical to the oracle's (run with the correctly rounded exp/log the kernels use). Over a
whole training run that makes the GPU trainer the oracle trainer, step for step.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from splatrs_b200 import gpu as G
from splatrs_b200 import scenes
from splatrs_b200._lib import Camera, ProjOpts, SplatError
from tests.golden import make_golden as MG

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


@pytest.fixture
def cr_math():
    O.set_cr_math(True)
    yield
    O.set_cr_math(False)


def dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def det_backward(ctx, p, w, h, bg, dimage):
    """The deterministic backward fed the oracle's projections; also the oracle's answer."""
    ob = O.bin(p, w, h)
    img, ft, nc, _ = O.rasterize_forward(p, ob, w, h, bg)
    og, oa, _ = O.rasterize_backward(p, ob, w, h, bg, ft, nc, dimage)
    proj = G.proj_from_reference(ctx, dev(p), w, h)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    pg = G.rasterize_backward_deterministic(ctx, proj, b, bg, out, dev(dimage))
    gg, ga = G.pgrad_to_reference(pg, p.shape[0])
    return gg.cpu().numpy(), ga.cpu().numpy(), og, oa, ob.num_entries


def test_deterministic_backward_equals_golden(ctx):
    """The golden fixture (ragged 72x56 view, depth ties, culled and near-threshold
    Gaussians): ProjGrad and the AbsGS sums bit-identical to the fixture's."""
    with np.load(MG.RENDER_FILE) as d:
        gold = {k: d[k] for k in d.files}
    cam = gold["cam"]
    w, h = int(cam[0]), int(cam[1])
    proj = G.proj_from_reference(ctx, dev(gold["proj"]), w, h)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, gold["background"])
    pg = G.rasterize_backward_deterministic(ctx, proj, b, gold["background"], out, dev(gold["dimage"]))
    gg, ga = G.pgrad_to_reference(pg, gold["proj"].shape[0])
    assert (bits(gg.cpu().numpy()) == bits(gold["screen_grads"])).all()
    assert (bits(ga.cpu().numpy()) == bits(gold["screen_abs"])).all()


@pytest.mark.parametrize("seed,n,size,bgv", [(21, 4000, (320, 240), 0.0), (22, 20000, (1000, 700), 0.3),
                                             (23, 2500, (77, 53), 1.0)])
def test_deterministic_backward_bit_exact(ctx, cr_math, seed, n, size, bgv):
    """Random scenes (ragged edge tiles, a non-black background): bit-identical ProjGrad
    and AbsGS sums; the atomic backward differs from them only in the last bits."""
    rng = np.random.default_rng(seed)
    g = scenes.random_gaussians(rng, n, -1.0, 1.0, -3.5, 0.5, 1.2)
    cam = scenes.look_at(size[0], size[1], 0.9 * size[0], 0.9 * size[0], (0.4, -0.3, -3.2), (0, 0, 0))
    p = O.project_all(g, cam, sh_degree=3)
    bg = np.full(3, bgv, np.float32)
    dimage = rng.normal(0, 1, size[0] * size[1] * 3).astype(np.float32)
    gg, ga, og, oa, entries = det_backward(ctx, p, size[0], size[1], bg, dimage)
    assert entries > n
    mism = (bits(gg) != bits(og)).any(1) | (bits(ga) != bits(oa)).any(1)
    assert mism.sum() == 0, f"{mism.sum()} of {n} Gaussians differ, first {np.nonzero(mism)[0][:5]}"


def test_deterministic_backward_render_benchmark_workload(ctx, cr_math):
    """The render benchmark's full workload (1M Gaussians, 1920x1080, dL/dpix ~ N(0,1),
    3.06M entries): bit-identical screen-space gradients for every Gaussian."""
    s = scenes.render_benchmark_scene(n=1_000_000)
    p = O.project_all(s["params"], s["cam"], sh_degree=3)
    gg, ga, og, oa, entries = det_backward(ctx, p, 1920, 1080, np.zeros(3, np.float32), s["dimage"])
    mism = (bits(gg) != bits(og)).any(1) | (bits(ga) != bits(oa)).any(1)
    assert mism.sum() == 0, f"{mism.sum()} Gaussians differ, first {np.nonzero(mism)[0][:5]}"
    print(f"\n1M / 1080p deterministic backward: {entries} entries, all 1,000,000 ProjGrad records bit-identical")


def test_deterministic_backward_needs_reference_tiles(ctx):
    """Another tile shape is refused with SPLAT_ERR_INVALID (the reference's slot sums are
    per 16x16 tile)."""
    rng = np.random.default_rng(3)
    g = scenes.random_gaussians(rng, 500, -1.0, 1.0, -3.5, 0.5, 1.2)
    cam = scenes.look_at(64, 48, 60.0, 60.0, (0.4, -0.3, -3.2), (0, 0, 0))
    old = ctx.raster_config
    ctx.raster_config = (8, 8, 64, 1)
    try:
        planes = G.params_to_planes(ctx, dev(g))
        proj = G.project_all(ctx, planes, 500, 500, Camera.from_record(cam), ProjOpts.make())
        b = G.bin(ctx, proj)
        out = G.rasterize_forward(ctx, proj, b, (0, 0, 0))
        with pytest.raises(SplatError) as e:
            G.rasterize_backward_deterministic(ctx, proj, b, (0, 0, 0), out, torch.zeros(64 * 48 * 3, device="cuda"))
        assert e.value.status == 1
    finally:
        ctx.raster_config = old


# The small blob scene's training configuration: 10k ground-truth Gaussians, 16 views at
# 256x256, 5k initial points, 2,000 iterations, densification every 100 from 500 to 1,500
# (threshold 2e-4), lambda 0.2, SH degree 3 with the reference's ramp.
BLOB_TRAIN = dict(iterations=2000, densify=1, densify_from_iter=500, densify_until_iter=1500,
                  densification_interval=100, densify_grad_threshold=0.0002, lambda_dssim=0.2, sh_degree=3,
                  position_lr_max_steps=2000, seed=0)


def blob_inputs(ctx):
    """Targets rendered by the device renderer (u8) and the device's point-cloud
    initialisation: one set of inputs fed to both trainers."""
    s = scenes.blob_scene()
    r = G.Renderer(ctx)
    r.set_model(s["gt"], 3)
    views = [(cam, scenes.to_rgb8(r.render(Camera.from_record(cam), ProjOpts.make(sh_degree=3), (0, 0, 0))))
             for cam in s["cams"]]
    r.close()
    ip = G.init_from_points(ctx, s["init_points"], s["init_rgb"])
    n0 = len(s["init_points"])
    init = G.planes_to_params(ctx, ip, n0, n0).cpu().numpy()
    return init, views, scenes.scene_extent(s["cams"])


def test_deterministic_trainer_equals_oracle_trainer_on_blob_scene(ctx, cr_math):
    """The full small-scene training run (2,000 iterations, 5k -> ~34k Gaussians through
    ten densifications) in deterministic mode against the oracle trainer: every step's view,
    entry count, Gaussian count and clone/split/prune counts equal, the loss within 1e-4
    relative, and the model bit-identical at checkpoints and at the end. The loss is only
    reported: the reference sums its 196,608 per-pixel terms in f32 in rayon's chunks (the
    oracle in fixed chunks), the device in f64, and no gradient depends on that sum."""
    init, views, extent = blob_inputs(ctx)
    t = G.Trainer(ctx, init, extent, views, deterministic=1, **BLOB_TRAIN)
    ot = O.Trainer(init, extent, views, **BLOB_TRAIN)
    checkpoints = {1, 2, 10, 100, 499, 501, 700, 1000, 1501, 2000}
    worst_loss = 0.0
    for it in range(1, BLOB_TRAIN["iterations"] + 1):
        a, b = t.step(), ot.step()
        assert a["view"] == b["view"], it
        assert a["entries"] == b["entries"], it
        assert a["num_gaussians"] == b["num_gaussians"], it
        assert (a["cloned"], a["split"], a["pruned"]) == (b["cloned"], b["split"], b["pruned"]), it
        rel = abs(a["loss"] - b["loss"]) / max(abs(b["loss"]), 1e-30)
        worst_loss = max(worst_loss, rel)
        assert rel < 1e-4, (it, a["loss"], b["loss"])
        if it in checkpoints:
            gm, om = t.model(), ot.model()
            mism = (bits(gm) != bits(om)).any(1)
            assert mism.sum() == 0, f"iteration {it}: {mism.sum()} of {len(om)} Gaussians differ"
    print(f"\nblob scene, 2,000 iterations deterministic: {t.count} Gaussians, model bit-identical to the oracle "
          f"trainer's; loss within {worst_loss:.1e} relative")
    t.close()


def test_deterministic_trainer_refuses_unsupported_settings(ctx):
    """Batches, autotuning, the BF16 copy, f64 conics and learned densification change the
    arithmetic or the order of the sums: the trainer refuses them in deterministic mode."""
    init = np.zeros((1, 59), np.float32)
    for extra in (dict(batch_views=2), dict(autotune=1), dict(bf16_storage=1), dict(fp64_conic=1),
                  dict(learned_densify=1)):
        with pytest.raises(SplatError) as e:
            G.Trainer(ctx, init, 1.0, [], deterministic=1, iterations=10, **extra)
        assert e.value.status == 1
