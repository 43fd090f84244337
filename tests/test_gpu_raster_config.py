"""Compositing configurations (tile shape x shared-memory chunk depth x the backward's pixels
per thread) and the autotuner.

Every configuration composites the same entries per pixel in the same depth order (the
projection narrows each entry's pixel rectangle to its 16-pixel tile rectangle before
binning it into 8x8 or 16x32 tiles), so with the correctly rounded math the image, final
transmittance and evaluated-pair count equal the oracle's (reference 16x16) bit for bit
under every configuration; contributor counts are positions in a tile's list and match
only for 16x16 tiles. Gradients meet the 1e-3 bar against the oracle. The autotuner times
all candidates on the caller's workload and keeps one; the trainer under any configuration
takes the same steps up to the summation order of gradients."""
import functools

import numpy as np
import pytest
import torch

from oracle import oracle as O
from splatrs_b200 import gpu as G
from splatrs_b200 import scenes
from splatrs_b200._lib import Camera, ProjOpts, SplatError
from tests import fixtures as F

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16, 256), (16, 16, 128), (16, 16, 64), (16, 16, 32), (8, 8, 256), (8, 8, 128), (8, 8, 64),
          (8, 8, 32), (16, 32, 256), (16, 32, 128), (16, 32, 64), (16, 32, 32)]
CANDS = [s + (1,) for s in SHAPES] + [s + (2,) for s in SHAPES]
DEFAULT = (16, 16, 256, 2)
SIZE = (640, 480)


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


@functools.lru_cache(maxsize=None)
def oracle_case(seed=41, n=20000):
    """A 640x480 scene with wide, opaque and faint Gaussians (so alpha boxes reach past
    the 3-sigma tile rectangles), its oracle projections, forward and backward."""
    O.set_cr_math(True)
    try:
        rng = np.random.default_rng(seed)
        g = scenes.random_gaussians(rng, n, -1.0, 1.0, -3.5, 0.5, 1.2)
        g[::10, 3:6] = [-0.7, -0.9, -0.8]
        g[::7, 10] = -5.0
        g[::5, 10] = 4.0
        cam = scenes.look_at(SIZE[0], SIZE[1], 0.9 * SIZE[0], 0.9 * SIZE[0], (0.4, -0.3, -3.2), (0, 0, 0))
        p = O.project_all(g, cam, antialias=True, sh_degree=3)
        bg = np.array((0.3, 0.6, 0.1), np.float32)
        ob = O.bin(p, *SIZE)
        img, ft, nc, pairs = O.rasterize_forward(p, ob, SIZE[0], SIZE[1], bg)
        dimage = rng.normal(0, 1, SIZE[0] * SIZE[1] * 3).astype(np.float32)
        og, oa, opairs = O.rasterize_backward(p, ob, SIZE[0], SIZE[1], bg, ft, nc, dimage)
    finally:
        O.set_cr_math(False)
    return g, cam, p, bg, img, ft, nc, pairs, dimage, og, oa, opairs


@pytest.fixture
def config(ctx):
    def use(cfg):
        ctx.raster_config = cfg
    yield use
    ctx.raster_config = DEFAULT


def test_candidates_and_invalid_configs(ctx):
    assert G.Context.raster_candidates() == CANDS
    assert ctx.raster_config == DEFAULT
    for bad in [(16, 16, 16, 1), (16, 16, 512, 1), (32, 32, 256, 1), (8, 16, 64, 1), (0, 0, 0, 1), (16, 16, 256, 3),
                (16, 16, 256, 0)]:
        with pytest.raises(SplatError):
            ctx.raster_config = bad
    assert ctx.raster_config == DEFAULT


@pytest.mark.parametrize("cfg", CANDS)
def test_forward_bit_identical_to_oracle_under_every_config(ctx, cr_math, config, cfg):
    g, cam, p, bg, img, ft, nc, pairs, *_ = oracle_case()
    config(cfg)
    proj = G.proj_from_reference(ctx, dev(p), *SIZE)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    assert (bits(out.image.cpu().numpy()) == bits(img)).all()
    assert (bits(out.final_t.cpu().numpy()) == bits(ft)).all()
    assert int(out.pairs.item()) == pairs
    if cfg[:2] == (16, 16):
        assert (out.n_contrib.cpu().numpy().view(np.uint32) == nc).all()
    print(f"\n{cfg}: {b.num_entries} tile entries, {b.tiles_x}x{b.tiles_y} tiles")


@pytest.mark.parametrize("cfg", CANDS)
def test_backward_matches_oracle_under_every_config(ctx, cr_math, config, cfg):
    g, cam, p, bg, img, ft, nc, pairs, dimage, og, oa, opairs = oracle_case()
    config(cfg)
    proj = G.proj_from_reference(ctx, dev(p), *SIZE)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    pg = G.rasterize_backward(ctx, proj, b, bg, out, dev(dimage), pairs=cnt)
    gg, ga = G.pgrad_to_reference(pg, p.shape[0])
    gg, ga = gg.cpu().numpy(), ga.cpu().numpy()
    scale = np.maximum(np.abs(og).max(0), 1e-30)
    err = (np.abs(gg - og).max(0) / scale).max()
    assert int(cnt.item()) == opairs
    assert err < 1e-3, err
    assert (np.abs(ga - oa).max(0) / np.maximum(np.abs(oa).max(0), 1e-30)).max() < 1e-3
    print(f"\n{cfg}: screen-space gradients max rel. error vs oracle {err:.2e}")


@pytest.mark.parametrize("cfg", [(8, 8, 64, 1), (16, 32, 128, 2)])
def test_device_projection_path_identical_across_configs(ctx, config, cfg):
    """The full device chain (projection, device-driven counts, binning, compositing) gives
    the same image under another tile shape as under 16x16."""
    g, cam, *_ = oracle_case()
    bg = [0.0, 0.0, 0.0]
    cam_c, opts = Camera.from_record(cam), ProjOpts.make(sh_degree=3)
    planes = G.params_to_planes(ctx, dev(g))
    n = g.shape[0]

    def render():
        proj = G.project_all(ctx, planes, n, n, cam_c, opts)
        b = G.bin(ctx, proj)
        return G.rasterize_forward(ctx, proj, b, bg).image.cpu().numpy(), b.num_entries

    ref, e16 = render()
    config(cfg)
    got, e = render()
    assert (bits(got) == bits(ref)).all()
    print(f"\n{cfg}: {e} entries vs {e16} with 16x16 tiles")


def test_autotune_render_times_every_candidate(ctx, config):
    s = scenes.render_benchmark_scene(n=100_000, width=1280, height=720, f=1000.0)
    n = s["params"].shape[0]
    planes = G.params_to_planes(ctx, dev(s["params"]))
    cam, opts = Camera.from_record(s["cam"]), ProjOpts.make(sh_degree=3)
    dimage = dev(s["dimage"][: 1280 * 720 * 3])
    proj = G.project_all(ctx, planes, n, n, cam, opts)
    b = G.bin(ctx, proj)
    ref = G.rasterize_forward(ctx, proj, b, [0.0, 0.0, 0.0]).image.cpu().numpy()
    res = ctx.autotune_render(planes, n, n, cam, opts, [0.0, 0.0, 0.0], dimage, reps=2)
    try:
        assert sorted(res["ms"]) == sorted(CANDS)
        assert all(np.isfinite(v) and v > 0 for v in res["ms"].values())
        assert res["picked"] in CANDS and ctx.raster_config == res["picked"]
        assert res["ms"][res["picked"]] == min(res["ms"].values())
        proj = G.project_all(ctx, planes, n, n, cam, opts)
        b = G.bin(ctx, proj)
        got = G.rasterize_forward(ctx, proj, b, [0.0, 0.0, 0.0]).image.cpu().numpy()
        assert (bits(got) == bits(ref)).all()
        print("\n" + ", ".join(f"{k}: {v:.3f} ms" for k, v in res["ms"].items()) + f"; picked {res['picked']}")
    finally:
        ctx.raster_config = DEFAULT


def _views(seed, sizes):
    rng = np.random.default_rng(seed)
    gt = F.ground_truth(rng, 60)
    cams = [F.ring_cameras(len(sizes), w, h, 2.6)[k] for k, (w, h) in enumerate(sizes)]
    views = F.render_views(gt, cams, 1, [0.0, 0.0, 0.0])
    pts, rgb = F.init_points(gt, rng)
    return views, O.scene_extent(np.stack(cams)), O.from_points(pts, rgb)


@pytest.mark.parametrize("batch", [1, 3])
def test_trainer_same_first_step_under_every_tile_shape(ctx, config, batch):
    """One iteration from the same model under each tile shape: the rendered images are
    identical, so the losses agree to the rounding of the SSIM sums, and the Adam step (a
    sign step at step 1) moves the parameters alike; only gradients that are zero up to
    rounding noise (whose sign follows the summation order) may step the other way."""
    views, extent, init = _views(310, [(64, 48), (80, 60), (50, 70)])
    cfg = dict(iterations=10, densify=0, sh_degree=1, sh_degree_interval=1000, position_lr_max_steps=10, seed=2,
               batch_views=batch)
    results = []
    for shape in [(16, 16, 256, 1), (8, 8, 64, 2), (16, 32, 128, 1), (16, 16, 128, 2)]:
        config(shape)
        t = G.Trainer(ctx, init, extent, views, **cfg)
        info = t.step()
        results.append((info["loss"], t.model()))
        t.close()
    l0, m0 = results[0]
    for loss, m in results[1:]:
        assert abs(loss - l0) <= 1e-6 * l0
        close = np.abs(m - m0) <= 1e-6 * (1.0 + np.abs(m0))
        print(f"\nbatch {batch}: {close.mean():.4f} of parameters equal after the step")
        assert close.mean() > 0.95
        assert np.abs(m - m0).max() < 0.05


def _psnr(t, views):
    tot = 0.0
    for cam, rgb in views:
        tot += O.psnr(t.render(cam), rgb.astype(np.float32) / np.float32(255.0))
    return tot / len(views)


def test_trainer_autotune_trains_like_fixed_config(ctx, config):
    """autotune = 1 tunes once before the first iteration (the count never moves without
    densification) and trains to the quality of the untuned trainer: the probes leave the
    model untouched, and configurations differ only in gradient summation order."""
    views, extent, init = _views(311, [(96, 72)] * 6)
    cfg = dict(iterations=300, densify=0, sh_degree=1, sh_degree_interval=100, position_lr_max_steps=300, seed=4,
               batch_views=2)
    plain = G.Trainer(ctx, init, extent, views, **cfg)
    plain.run(300)
    tuned = G.Trainer(ctx, init, extent, views, autotune=1, **cfg)
    tuned.run(300)
    info = tuned.tuning()
    assert info["tunes"] == 1
    assert info["picked"] in CANDS and ctx.raster_config == info["picked"]
    assert all(v > 0 for v in info["ms"].values())
    p0, p1 = _psnr(plain, views), _psnr(tuned, views)
    print(f"\nplain {p0:.3f} dB; tuned {p1:.3f} dB, picked {info['picked']}")
    assert abs(p1 - p0) < 0.1
    plain.close()
    tuned.close()


def test_trainer_autotune_retunes_as_the_count_grows(ctx, config):
    """With densification the count doubles past the last tuning's, which triggers new
    tunings; training still converges."""
    views, extent, init = _views(312, [(96, 72)] * 6)
    cfg = dict(iterations=400, densify=1, densify_from_iter=50, densify_until_iter=300, densification_interval=50,
               opacity_reset_interval=0, sh_degree=1, sh_degree_interval=100, position_lr_max_steps=400, seed=4,
               batch_views=2, autotune=1)
    t = G.Trainer(ctx, init, extent, views, **cfg)
    n0 = t.count
    t.run(400)
    info = t.tuning()
    p = _psnr(t, views)
    print(f"\n{n0} -> {t.count} Gaussians, {info['tunes']} tunings, picked {info['picked']}, {p:.2f} dB")
    assert t.count > 2 * n0 and info["tunes"] >= 2
    assert p > 25.0
    t.close()


def test_blend_weight_statistic_sums_to_coverage(ctx, config):
    """The backward's fourth value of gradient plane 2 is each Gaussian's blending weight
    sum(alpha T) over the view's pixels. Per pixel those weights telescope to 1 - T_final,
    so over the image they sum to sum(1 - final T); they are non-negative, zero for unseen
    Gaussians, and the same under every tile shape up to summation order."""
    g, cam, p, bg, img, ft, nc, pairs, dimage, *_ = oracle_case()
    per = {}
    for cfg in [(16, 16, 256, 1), (8, 8, 64, 1), (16, 32, 128, 2), (16, 16, 256, 2)]:
        config(cfg)
        proj = G.proj_from_reference(ctx, dev(p), *SIZE)
        b = G.bin(ctx, proj)
        out = G.rasterize_forward(ctx, proj, b, bg)
        pg = G.rasterize_backward(ctx, proj, b, bg, out, dev(dimage))
        w = pg[2, :, 3].double().cpu().numpy()
        cover = float((1.0 - out.final_t.double()).sum().item())
        assert (w >= 0).all()
        assert (w[p[:, 6] == 0] == 0).all()
        assert abs(w.sum() - cover) <= 1e-4 * cover, (w.sum(), cover)
        per[cfg] = w
    ref = per[(16, 16, 256, 1)]
    for cfg, w in per.items():
        assert np.abs(w - ref).max() <= 1e-5 * ref.max(), cfg


@pytest.mark.parametrize("cfg", [(8, 8, 32, 2), (16, 32, 64, 1), (16, 16, 128, 2)])
def test_ragged_image_sizes_under_other_configs(ctx, cr_math, config, cfg):
    """Image sizes that are no multiple of any tile edge (97x61, 1024x36): forward
    bit-identical to the oracle, backward within the bar."""
    for seed, n, size in [(51, 1500, (97, 61)), (52, 2500, (1024, 36))]:
        rng = np.random.default_rng(seed)
        g = scenes.random_gaussians(rng, n, -1.0, 1.0, -3.5, 0.5, 1.2)
        cam = scenes.look_at(size[0], size[1], 0.9 * size[0], 0.9 * size[0], (0.4, -0.3, -3.2), (0, 0, 0))
        p = O.project_all(g, cam, antialias=True, sh_degree=3)
        bg = np.array((0.3, 0.6, 0.1), np.float32)
        ob = O.bin(p, *size)
        img, ft, nc, pairs = O.rasterize_forward(p, ob, size[0], size[1], bg)
        dimage = rng.normal(0, 1, size[0] * size[1] * 3).astype(np.float32)
        og, _, _ = O.rasterize_backward(p, ob, size[0], size[1], bg, ft, nc, dimage)
        config(cfg)
        proj = G.proj_from_reference(ctx, dev(p), *size)
        b = G.bin(ctx, proj)
        out = G.rasterize_forward(ctx, proj, b, bg)
        assert (bits(out.image.cpu().numpy()) == bits(img)).all()
        assert (bits(out.final_t.cpu().numpy()) == bits(ft)).all()
        pg = G.rasterize_backward(ctx, proj, b, bg, out, dev(dimage))
        gg, _ = G.pgrad_to_reference(pg, n)
        err = (np.abs(gg.cpu().numpy() - og).max(0) / np.maximum(np.abs(og).max(0), 1e-30)).max()
        assert err < 1e-3, (size, err)
        config(DEFAULT)


@pytest.mark.parametrize("cfg", [(16, 16, 256, 1), (8, 8, 64, 2), (16, 32, 256, 2)])
def test_empty_and_fully_culled_under_every_shape(ctx, config, cfg):
    """No Gaussian at all, and every Gaussian behind the camera: the image is the
    background, final T is 1, contributor counts and gradients are zero."""
    config(cfg)
    bgv = [0.2, 0.3, 0.4]
    cam_rec = scenes.look_at(80, 60, 70.0, 70.0, (0.0, 0.0, -3.0), (0, 0, 0))
    cam, opts = Camera.from_record(cam_rec), ProjOpts.make(sh_degree=3)
    rng = np.random.default_rng(60)
    behind = scenes.random_gaussians(rng, 64, -1.0, 1.0, -3.5, 0.5, 1.0)
    behind[:, 2] = -50.0
    for g in (behind[:0], behind):
        n = g.shape[0]
        planes = G.params_to_planes(ctx, dev(g), max(n, 1))
        proj = G.project_all(ctx, planes, n, max(n, 1), cam, opts)
        b = G.bin(ctx, proj)
        out = G.rasterize_forward(ctx, proj, b, bgv)
        assert b.num_entries == 0
        assert np.allclose(out.image.cpu().numpy().reshape(-1, 3), bgv)
        assert (out.final_t.cpu().numpy() == 1.0).all() and (out.n_contrib.cpu().numpy() == 0).all()
        pg = G.rasterize_backward(ctx, proj, b, bgv, out, torch.ones(80 * 60 * 3, device="cuda"), cap=max(n, 1))
        assert (pg.cpu().numpy() == 0).all()
