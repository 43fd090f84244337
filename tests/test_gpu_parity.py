"""Parity of the sm_100a kernels with the CPU oracle, stage by stage, through the C ABI.

Bars: tile lists and sort order bit-exact when fed the same projections;
images within 1e-4 max-abs; per-parameter gradients within 1e-3 relative error; every
result also reports its error against the FP64 oracle.

The oracle runs in two modes. With the host libm (its default) it reproduces the
reference's f32 results; the GPU differs from it only where glibc's expf/logf are not
correctly rounded (1 ulp on ~0.1% of inputs), so decisions and images agree to rounding.
With the correctly rounded exp/log that the kernels use, the oracle and the GPU evaluate
the same operations in the same order, so projections, images, transmittance and
contributor counts must be bit-identical.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from splatrs_b200 import gpu as G
from splatrs_b200 import scenes
from splatrs_b200._lib import Camera, LearningRates, ProjOpts
from tests import fixtures as F

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


def small_scene(seed=3, n=3000, size=(320, 240)):
    rng = np.random.default_rng(seed)
    g = scenes.random_gaussians(rng, n, -1.0, 1.0, -3.5, 0.5, 1.2)
    cam = scenes.look_at(size[0], size[1], 0.9 * size[0], 0.9 * size[0], (0.4, -0.3, -3.2), (0, 0, 0))
    return g, cam


def gpu_project(ctx, g, cam, **opts):
    planes = G.params_to_planes(ctx, dev(g))
    proj = G.project_all(ctx, planes, g.shape[0], g.shape[0], Camera.from_record(cam), ProjOpts.make(**opts))
    return planes, proj


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


CASES = [dict(antialias=False, sh_degree=3), dict(antialias=True, sh_degree=3), dict(antialias=False, sh_degree=0),
         dict(antialias=True, sh_degree=1), dict(antialias=False, sh_degree=2)]


@pytest.mark.parametrize("opts", CASES)
def test_projection_bit_exact_with_cr_math(ctx, cr_math, opts):
    """project_all: every field bit-identical to the oracle with correctly rounded exp/log."""
    g, cam = small_scene()
    _, proj = gpu_project(ctx, g, cam, **opts)
    got = proj.to_reference(ctx).cpu().numpy()
    want = O.project_all(g, cam, **opts)
    assert (want[:, 6] > 0).sum() > 1000
    mism = (bits(got) != bits(want)).any(1)
    assert mism.sum() == 0, f"{mism.sum()} projections differ, first {np.nonzero(mism)[0][:5]}"


@pytest.mark.parametrize("opts", CASES[:2])
def test_projection_matches_libm_oracle(ctx, opts):
    """project_all against the faithful oracle: integers exact, floats to a few ulps."""
    g, cam = small_scene(seed=4)
    _, proj = gpu_project(ctx, g, cam, **opts)
    got = proj.to_reference(ctx).cpu().numpy()
    want = O.project_all(g, cam, **opts)
    ints = [6, 11, 12, 13, 14]
    assert (got[:, ints] == want[:, ints]).all()
    fl = [0, 1, 2, 3, 4, 5, 7, 8, 9, 10]
    rel = np.abs(got[:, fl] - want[:, fl]) / np.maximum(np.abs(want[:, fl]), 1e-6)
    assert rel.max() < 1e-5, rel.max()


def per_tile_lists(gauss, tile_range):
    return [gauss[s:e].tolist() for s, e in tile_range]


def oracle_tile_lists(b):
    a = b.arrays()
    eg = a["entry_gaussian"][a["entries"]]
    return per_tile_lists(eg, a["tile_range"]), a


@pytest.mark.parametrize("seed,size", [(5, (320, 240)), (6, (97, 61)), (7, (1024, 64))])
def test_binning_bit_exact_from_oracle_projections(ctx, seed, size):
    """bin: fed the oracle's projections, per-tile lists, order and keys are identical."""
    g, cam = small_scene(seed=seed, n=4000, size=size)
    want_p = O.project_all(g, cam, sh_degree=3)
    # Force depth ties inside tiles to exercise the entry-index tie break.
    want_p[::7, 5] = want_p[3, 5]
    proj = G.proj_from_reference(ctx, dev(want_p), size[0], size[1])
    b = G.bin(ctx, proj, want_keys=True)
    ob = O.bin(want_p, size[0], size[1])
    ol, oa = oracle_tile_lists(ob)
    assert b.num_entries == ob.num_entries
    gl = per_tile_lists(b.gauss.cpu().numpy(), b.tile_range.cpu().numpy().astype(np.int64))
    assert gl == ol
    assert (b.keys.cpu().numpy().view(np.uint64) == oa["keys"]).all()
    assert (b.entry_offset.cpu().numpy().view(np.uint32) == oa["entry_offset"]).all()
    assert (b.tile_range.cpu().numpy().view(np.uint32) == oa["tile_range"]).all()


def test_binning_large_single_view(ctx):
    """bin on a 1M-Gaussian full-HD view (the render benchmark's scene): identical lists."""
    s = scenes.render_benchmark_scene(n=1_000_000)
    want_p = O.project_all(s["params"], s["cam"], sh_degree=3)
    proj = G.proj_from_reference(ctx, dev(want_p), 1920, 1080)
    b = G.bin(ctx, proj)
    ob = O.bin(want_p, 1920, 1080)
    a = ob.arrays()
    assert b.num_entries == ob.num_entries
    assert (b.gauss.cpu().numpy().view(np.uint32) == a["entry_gaussian"][a["entries"]]).all()
    assert (b.tile_range.cpu().numpy().view(np.uint32) == a["tile_range"]).all()


def test_render_benchmark_workload_matches_oracle(ctx, cr_math):
    """The render benchmark's workload at full size (1M Gaussians, 1920x1080, SH degree 3,
    dL/dpix ~ N(0,1)), stage by stage against the correctly rounded oracle: projections
    bit-identical; fed the oracle's projections, image, final T, contributor counts and
    evaluated pairs bit-identical, screen-space gradients within 1e-3 of each quantity's
    scale; fed the oracle's screen-space gradients, the 59 parameter gradients
    bit-identical."""
    s = scenes.render_benchmark_scene(n=1_000_000)
    g, cam, dimage = s["params"], s["cam"], s["dimage"]
    w, h, n = 1920, 1080, g.shape[0]
    bg = np.zeros(3, np.float32)
    p = O.project_all(g, cam, sh_degree=3)
    planes, gproj = gpu_project(ctx, g, cam, sh_degree=3)
    mism = (bits(gproj.to_reference(ctx).cpu().numpy()) != bits(p)).any(1)
    assert mism.sum() == 0, f"{mism.sum()} projections differ, first {np.nonzero(mism)[0][:5]}"
    ob = O.bin(p, w, h)
    img, ft, nc, pairs = O.rasterize_forward(p, ob, w, h, bg)
    og, oa, bpairs = O.rasterize_backward(p, ob, w, h, bg, ft, nc, dimage)
    proj = G.proj_from_reference(ctx, dev(p), w, h)
    b = G.bin(ctx, proj)
    assert b.num_entries == ob.num_entries
    out = G.rasterize_forward(ctx, proj, b, bg)
    assert (bits(out.image.cpu().numpy()) == bits(img)).all()
    assert (bits(out.final_t.cpu().numpy()) == bits(ft)).all()
    assert (out.n_contrib.cpu().numpy().view(np.uint32) == nc).all()
    assert int(out.pairs.item()) == pairs
    tp = torch.zeros(1, dtype=torch.int64, device="cuda")
    pg = G.rasterize_backward(ctx, proj, b, bg, out, dev(dimage), pairs=tp)
    gg, ga = G.pgrad_to_reference(pg, n)
    gg, ga = gg.cpu().numpy(), ga.cpu().numpy()
    assert int(tp.item()) == bpairs
    err = grad_rel_error(gg, og)
    assert err.max() < 1e-3, err
    assert grad_rel_error(ga, oa).max() < 1e-3
    gp = G.project_backward_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(sh_degree=3), gproj,
                                G.pgrad_from_reference(dev(og)))
    got = G.planes_to_params(ctx, gp, n, n).cpu().numpy()
    want = O.project_backward_all(g, cam, og, sh_degree=3)
    mism = (bits(got) != bits(want)).any(1)
    assert mism.sum() == 0, f"{mism.sum()} gradient records differ, first {np.nonzero(mism)[0][:5]}"
    print(f"\n1M / 1080p: {ob.num_entries} entries, {pairs} forward and {bpairs} backward pairs, "
          f"screen-space gradient error {err.max():.2e} of scale")


@pytest.mark.parametrize("seed,size", [(8, (320, 240)), (9, (1024, 64)), (10, (1920, 1080))])
def test_device_driven_binning_equals_host_driven(ctx, seed, size):
    """splat_bin_count_device + splat_bin_sort_device (no host read-back, capacity-sized
    buffers): per-tile lists and ranges identical to splat_bin_sort; a second, smaller
    view through the same scratch too; a capacity below the count raises the overflow
    flag instead of writing past the buffers."""
    g, cam = small_scene(seed=seed, n=20000, size=size)
    _, proj = gpu_project(ctx, g, cam, sh_degree=3)
    want = G.bin(ctx, proj)
    E = want.num_entries
    gauss, tr, e_dev, flag, scratch = G.bin_device(ctx, proj, E + 4097)
    assert int(e_dev.item()) == E and int(flag.item()) == 0
    assert torch.equal(tr, want.tile_range)
    assert torch.equal(gauss[:E], want.gauss)
    g2, cam2 = small_scene(seed=seed + 100, n=3000, size=(size[0] // 2 + 1, size[1] // 2 + 1))
    _, proj2 = gpu_project(ctx, g2, cam2, sh_degree=1)
    want2 = G.bin(ctx, proj2)
    gauss2, tr2, e2, flag2, _ = G.bin_device(ctx, proj2, E + 4097, scratch)
    assert int(flag2.item()) == 0 and torch.equal(tr2, want2.tile_range)
    assert torch.equal(gauss2[:want2.num_entries], want2.gauss)
    _, _, _, flag3, _ = G.bin_device(ctx, proj, E // 2)
    assert int(flag3.item()) == 1


def test_binning_empty_and_offscreen(ctx):
    """No visible Gaussian: zero entries, every tile range empty."""
    g, cam = small_scene(n=50)
    g[:, 2] = -50.0  # all behind the camera
    _, proj = gpu_project(ctx, g, cam)
    b = G.bin(ctx, proj)
    assert b.num_entries == 0
    assert (b.tile_range.cpu().numpy() == 0).all()
    out = G.rasterize_forward(ctx, proj, b, [0.2, 0.3, 0.4])
    img = out.image.cpu().numpy().reshape(-1, 3)
    assert np.allclose(img, [0.2, 0.3, 0.4]) and (out.n_contrib.cpu().numpy() == 0).all()


def raster_case(seed, n, size, antialias=True, bg=(0.3, 0.6, 0.1)):
    g, cam = small_scene(seed=seed, n=n, size=size)
    g[::10, 3:6] = [-0.7, -0.9, -0.8]
    g[::7, 10] = -5.0
    p = O.project_all(g, cam, antialias=antialias, sh_degree=3)
    return g, cam, p, np.array(bg, np.float32)


@pytest.mark.parametrize("seed,n,size", [(11, 3000, (320, 240)), (12, 400, (70, 50)), (13, 20000, (640, 480))])
def test_rasterize_forward_bit_exact_with_cr_math(ctx, cr_math, seed, n, size):
    """rasterize_forward fed the oracle's projections: image, final T and n_contrib identical."""
    g, cam, p, bg = raster_case(seed, n, size)
    proj = G.proj_from_reference(ctx, dev(p), *size)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    ob = O.bin(p, *size)
    img, ft, nc, pairs = O.rasterize_forward(p, ob, size[0], size[1], bg)
    assert (bits(out.image.cpu().numpy()) == bits(img)).all()
    assert (bits(out.final_t.cpu().numpy()) == bits(ft)).all()
    assert (out.n_contrib.cpu().numpy().view(np.uint32) == nc).all()
    assert int(out.pairs.item()) == pairs


@pytest.mark.parametrize("seed,n,size", [(21, 3000, (320, 240)), (22, 20000, (640, 480))])
def test_rasterize_forward_matches_libm_oracle(ctx, seed, n, size):
    """rasterize_forward against the faithful oracle: max-abs < 1e-4."""
    g, cam, p, bg = raster_case(seed, n, size)
    proj = G.proj_from_reference(ctx, dev(p), *size)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    ob = O.bin(p, *size)
    img, ft, nc, _ = O.rasterize_forward(p, ob, size[0], size[1], bg)
    err = np.abs(out.image.cpu().numpy() - img).max()
    assert err < 1e-4, err
    # FP64 oracle error of both, for the record.
    ob64 = O.bin(p.astype(np.float64), *size, dtype=np.float64)
    img64, _, _, _ = O.rasterize_forward(p.astype(np.float64), ob64, size[0], size[1], bg.astype(np.float64),
                                         dtype=np.float64)
    print(f"\nimage max-abs vs f32 oracle {err:.3e}; vs f64 oracle: gpu "
          f"{np.abs(out.image.cpu().numpy() - img64).max():.3e}, f32 oracle {np.abs(img - img64).max():.3e}")


def grad_rel_error(got, want):
    """Per-column error relative to the column's scale: max_i |got - want| / max_i |want|."""
    scale = np.maximum(np.abs(want).max(0), 1e-30)
    return (np.abs(got - want).max(0) / scale)


@pytest.mark.parametrize("seed,n,size", [(31, 3000, (320, 240)), (32, 20000, (640, 480))])
def test_rasterize_backward_matches_oracle(ctx, cr_math, seed, n, size):
    """rasterize_backward fed the oracle's forward state: screen-space gradients per Gaussian
    within 1e-3 of each quantity's scale; AbsGS accumulators bound the signed sums."""
    g, cam, p, bg = raster_case(seed, n, size)
    rng = np.random.default_rng(seed)
    dimage = rng.normal(0, 1, size[0] * size[1] * 3).astype(np.float32)
    ob = O.bin(p, *size)
    img, ft, nc, _ = O.rasterize_forward(p, ob, size[0], size[1], bg)
    og, oa, opairs = O.rasterize_backward(p, ob, size[0], size[1], bg, ft, nc, dimage)
    proj = G.proj_from_reference(ctx, dev(p), *size)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    pairs = torch.zeros(1, dtype=torch.int64, device="cuda")
    pg = G.rasterize_backward(ctx, proj, b, bg, out, dev(dimage), pairs=pairs)
    gg, ga = G.pgrad_to_reference(pg, p.shape[0])
    gg, ga = gg.cpu().numpy(), ga.cpu().numpy()
    assert int(pairs.item()) == opairs
    err = grad_rel_error(gg, og)
    assert err.max() < 1e-3, err
    assert grad_rel_error(ga, oa).max() < 1e-3
    assert (ga + 1e-5 >= np.abs(gg[:, 0:2])).all()
    p64 = p.astype(np.float64)
    ob64 = O.bin(p64, *size, dtype=np.float64)
    _, ft64, nc64, _ = O.rasterize_forward(p64, ob64, size[0], size[1], bg.astype(np.float64), dtype=np.float64)
    og64, _, _ = O.rasterize_backward(p64, ob64, size[0], size[1], bg.astype(np.float64), ft64, nc64,
                                      dimage.astype(np.float64), dtype=np.float64)
    print(f"\nscreen grads vs f64 oracle: gpu {grad_rel_error(gg, og64).max():.3e}, "
          f"f32 oracle {grad_rel_error(og, og64).max():.3e}")


@pytest.mark.parametrize("opts", CASES)
def test_project_backward_matches_oracle(ctx, cr_math, opts):
    """project_backward_all fed the same screen-space gradients: 59 parameter gradients
    bit-identical to the oracle (same operations, same order)."""
    g, cam = small_scene(seed=41)
    rng = np.random.default_rng(41)
    w = rng.uniform(-1, 1, (g.shape[0], 9)).astype(np.float32)
    planes, proj = gpu_project(ctx, g, cam, **opts)
    pg = G.pgrad_from_reference(dev(w))
    gp = G.project_backward_all(ctx, planes, g.shape[0], g.shape[0], Camera.from_record(cam),
                                ProjOpts.make(**opts), proj, pg)
    got = G.planes_to_params(ctx, gp, g.shape[0], g.shape[0]).cpu().numpy()
    want = O.project_backward_all(g, cam, w, **opts)
    mism = (bits(got) != bits(want)).any(1)
    assert mism.sum() == 0, f"{mism.sum()} gradient records differ, first {np.nonzero(mism)[0][:5]}"


def test_project_backward_densify_stats(ctx):
    """DensifyStats::accumulate fused into the projection backward (signed and AbsGS)."""
    g, cam = small_scene(seed=42, n=2000)
    rng = np.random.default_rng(42)
    w = rng.uniform(-1, 1, (g.shape[0], 9)).astype(np.float32)
    a2 = np.abs(rng.uniform(-1, 1, (g.shape[0], 2))).astype(np.float32)
    planes, proj = gpu_project(ctx, g, cam)
    pg = G.pgrad_from_reference(dev(w), dev(a2))
    p = proj.to_reference(ctx).cpu().numpy()
    for absgrad in (False, True):
        n = g.shape[0]
        stats = torch.zeros(3 * n, dtype=torch.int32, device="cuda")
        G.project_backward_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(), proj, pg, stats, absgrad)
        G.project_backward_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(), proj, pg, stats, absgrad)
        s = stats.cpu().numpy()
        acc, den, mr = s[:n].view(np.float32), s[n:2 * n].view(np.uint32), s[2 * n:].view(np.uint32)
        oacc = np.zeros(n, np.float32)
        oden = np.zeros(n, np.uint32)
        omr = np.zeros(n, np.uint32)
        for _ in range(2):
            O.densify_accumulate(p, w, a2 if absgrad else None, int(cam[0]), int(cam[1]), oacc, oden, omr)
        assert (bits(acc) == bits(oacc)).all() and (den == oden).all() and (mr == omr).all()


@pytest.mark.parametrize("sh_degree", [0, 3])
def test_project_backward_adam_equals_separate_steps(ctx, sh_degree):
    """splat_project_bwd_adam over three steps equals splat_project_bwd followed by
    splat_adam_step bit for bit: parameters, both moments and the densification stats."""
    g, cam = small_scene(seed=43, n=3000)
    n = g.shape[0]
    rng = np.random.default_rng(43)
    opts = ProjOpts.make(sh_degree=sh_degree)
    lr = LearningRates(0.00016 * 3.3, 0.005, 0.001, 0.025, 0.0025, 0.0025 / 20)
    fused = G.params_to_planes(ctx, dev(g), n)
    sep = fused.clone()
    fm, fv = torch.zeros_like(fused), torch.zeros_like(fused)
    sm, sv = torch.zeros_like(fused), torch.zeros_like(fused)
    fst = torch.zeros(3 * n, dtype=torch.int32, device="cuda")
    sst = torch.zeros_like(fst)
    for step in (1, 2, 3):
        w = rng.uniform(-1, 1, (n, 9)).astype(np.float32)
        a2 = np.abs(rng.uniform(-1, 1, (n, 2))).astype(np.float32)
        pg = G.pgrad_from_reference(dev(w), dev(a2))
        proj = G.project_all(ctx, sep, n, n, Camera.from_record(cam), opts)
        gp = G.project_backward_all(ctx, sep, n, n, Camera.from_record(cam), opts, proj, pg, sst, True)
        G.adam_step(ctx, sep, gp, sm, sv, n, n, step, lr)
        proj = G.project_all(ctx, fused, n, n, Camera.from_record(cam), opts)
        G.project_backward_adam(ctx, fused, fm, fv, n, n, Camera.from_record(cam), opts, proj, pg, step, lr, fst, True)
        assert torch.equal(fused, sep) and torch.equal(fm, sm) and torch.equal(fv, sv)
        assert torch.equal(fst, sst)
    assert not torch.equal(fused, G.params_to_planes(ctx, dev(g), n))


def test_end_to_end_chain_matches_oracle(ctx):
    """Parameters -> projection -> binning -> compositing -> backward -> parameter
    gradients, all on the GPU, against the same chain on the f32 oracle and the f64 oracle."""
    rng = np.random.default_rng(51)
    g = scenes.random_gaussians(rng, 6000, -1.0, 1.0, -3.8, 0.4, 1.0)
    cam = scenes.look_at(256, 256, 300.0, 300.0, (0.0, 0.5, -4.0), (0, 0, 0))
    bg = np.array([0.1, 0.1, 0.1], np.float32)
    dimage = rng.normal(0, 1, 256 * 256 * 3).astype(np.float32)
    opts = dict(antialias=True, sh_degree=3)
    planes, proj = gpu_project(ctx, g, cam, **opts)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    pg = G.rasterize_backward(ctx, proj, b, bg, out, dev(dimage))
    gp = G.project_backward_all(ctx, planes, g.shape[0], g.shape[0], Camera.from_record(cam), ProjOpts.make(**opts),
                                proj, pg)
    got = G.planes_to_params(ctx, gp, g.shape[0], g.shape[0]).cpu().numpy()

    def chain(dt):
        pp = O.project_all(g.astype(dt), cam.astype(dt), dtype=dt, **opts)
        ob = O.bin(pp, 256, 256, dtype=dt)
        img, ft, nc, _ = O.rasterize_forward(pp, ob, 256, 256, bg.astype(dt), dtype=dt)
        og, _, _ = O.rasterize_backward(pp, ob, 256, 256, bg.astype(dt), ft, nc, dimage.astype(dt), dtype=dt)
        return img, O.project_backward_all(g.astype(dt), cam.astype(dt), og, dtype=dt, **opts)

    img32, want32 = chain(np.float32)
    img64, want64 = chain(np.float64)
    assert np.abs(out.image.cpu().numpy() - img32).max() < 1e-4
    err = grad_rel_error(got, want32)
    active = np.abs(want32).max(0) > 0
    assert err[active].max() < 1e-3, err
    print(f"\nparameter grads vs f64 oracle: gpu {grad_rel_error(got, want64)[active].max():.3e}, "
          f"f32 oracle {grad_rel_error(want32, want64)[active].max():.3e}; image vs f64 oracle: gpu "
          f"{np.abs(out.image.cpu().numpy() - img64).max():.3e}")


def test_invalid_arguments_return_status(ctx):
    """Hot-path invariant violations return SPLAT_ERR_INVALID instead of aborting
    (the reference panics: src/rasterize.rs:65-74, :466-469)."""
    from splatrs_b200._lib import SplatError
    g, cam = small_scene(n=10)
    bad = cam.copy()
    bad[0] = 70000
    planes = G.params_to_planes(ctx, dev(g))
    with pytest.raises(SplatError) as e:
        G.project_all(ctx, planes, 10, 10, Camera.from_record(bad), ProjOpts.make())
    assert e.value.status == 1
    with pytest.raises(SplatError):
        G.project_all(ctx, planes, 10, 10, Camera.from_record(cam), ProjOpts.make(sh_degree=4))


def test_fast_exp_bound_behind_backward_screening(ctx):
    """The backward pass decides with a fast exp outside a relative band of 3e-5 around its
    thresholds; its error over every float of the argument range [-(ln 255 + 0.5), 0] must
    stay far inside that band."""
    import ctypes as C
    out = C.c_float()
    G.check(ctx.lib.splat_diag_fast_exp_error(ctx.h, 0.0, 6.05, 1, C.byref(out)), ctx.h)
    print(f"\nfast exp max relative error on [-6.05, 0]: {out.value:.3e}")
    assert 0.0 < out.value < 3e-6


def test_paired_arithmetic_keeps_one_rounding_per_operation(ctx):
    """The compositing backward computes sigma, and the SSIM loss its blur sums, on f32x2
    pairs; the code generator would fuse a paired multiply into a following add. Over 4M
    seeded inputs the paired sigma and blur steps equal the scalar unfused values."""
    import ctypes as C
    out = (C.c_uint32 * 2)()
    G.check(ctx.lib.splat_diag_pair_exact(ctx.h, 1 << 22, out), ctx.h)
    assert (out[0], out[1]) == (0, 0), (out[0], out[1])


def _bf16_round_params(g):
    """Reference records with quaternion, log-scales and SH rounded to bf16 (nearest even),
    the values the BF16 render copy holds; means and opacity stay f32."""
    r = g.copy()
    cols = list(range(3, 10)) + list(range(11, 59))
    r[:, cols] = torch.from_numpy(g[:, cols]).to(torch.bfloat16).to(torch.float32).numpy()
    return r


@pytest.mark.parametrize("sh_degree", [0, 3])
def test_bf16_projection_equals_f32_on_rounded_params(ctx, sh_degree):
    """splat_project_fwd_bf16 reads quaternion, log-scales and SH from the BF16 copy: its
    records are bit-identical to splat_project_fwd on parameters rounded to bf16."""
    g, cam = small_scene(seed=61)
    n = g.shape[0]
    opts = ProjOpts.make(sh_degree=sh_degree, antialias=True)
    planes = G.params_to_planes(ctx, dev(g), n)
    bf = G.params_to_bf16(ctx, planes, n, n)
    got = G.project_all_bf16(ctx, planes, bf, n, n, Camera.from_record(cam), opts)
    want = G.project_all(ctx, G.params_to_planes(ctx, dev(_bf16_round_params(g)), n), n, n, Camera.from_record(cam),
                         opts)
    assert torch.equal(got.rec, want.rec) and torch.equal(got.num_tiles, want.num_tiles)
    assert torch.equal(got.depth_range, want.depth_range)
    p64 = O.project_all(g.astype(np.float64), cam.astype(np.float64), antialias=True, sh_degree=sh_degree,
                        dtype=np.float64)
    vis = p64[:, 6] > 0
    rel = np.abs(got.to_reference(ctx).cpu().numpy()[vis, 7:11] - p64[vis, 7:11]).max()
    print(f"\nbf16 storage: opacity/colour max-abs vs the f64 oracle of the f32 parameters {rel:.2e}")


def test_bf16_fused_adam_equals_separate_steps(ctx):
    """splat_project_bwd_adam with a BF16 copy: the gradient is taken at the copy's values
    and Adam updates the f32 master, bit-identical to splat_project_bwd on the rounded
    parameters followed by splat_adam_step on the master; the copy is rewritten as the
    rounding of the updated master."""
    g, cam = small_scene(seed=62, n=2000)
    n = g.shape[0]
    rng = np.random.default_rng(62)
    opts = ProjOpts.make(sh_degree=3)
    lr = LearningRates(0.00016 * 3.3, 0.005, 0.001, 0.025, 0.0025, 0.0025 / 20)
    master = G.params_to_planes(ctx, dev(g), n)
    bf = G.params_to_bf16(ctx, master, n, n)
    sep = master.clone()
    fm, fv = torch.zeros_like(master), torch.zeros_like(master)
    sm, sv = torch.zeros_like(master), torch.zeros_like(master)
    for step in (1, 2):
        pg = G.pgrad_from_reference(dev(rng.uniform(-1, 1, (n, 9)).astype(np.float32)))
        rounded = G.params_to_planes(ctx, dev(_bf16_round_params(G.planes_to_params(ctx, sep, n, n).cpu().numpy())), n)
        proj = G.project_all(ctx, rounded, n, n, Camera.from_record(cam), opts)
        gp = G.project_backward_all(ctx, rounded, n, n, Camera.from_record(cam), opts, proj, pg)
        G.adam_step(ctx, sep, gp, sm, sv, n, n, step, lr)
        projb = G.project_all_bf16(ctx, master, bf, n, n, Camera.from_record(cam), opts)
        assert torch.equal(projb.rec, proj.rec)
        G.project_backward_adam(ctx, master, fm, fv, n, n, Camera.from_record(cam), opts, projb, pg, step, lr, bf16=bf)
        assert torch.equal(master, sep) and torch.equal(fm, sm) and torch.equal(fv, sv)
        assert torch.equal(bf, G.params_to_bf16(ctx, sep, n, n))


def _needles(seed, n=3000):
    """Long thin Gaussians (one axis e^2, two e^-6) close to the camera: their projected
    2x2 covariances are nearly rank one."""
    rng = np.random.default_rng(seed)
    g = scenes.random_gaussians(rng, n, -0.6, 0.6, -6.0, 0.0, 1.0)
    g[:, 3] = 2.0
    cam = scenes.look_at(640, 480, 500.0, 500.0, (0.0, 0.0, -3.0), (0, 0, 0))
    return g, cam


def test_fp64_conic_resolves_ill_conditioned_covariances(ctx):
    """fp64_conic: for needle-like Gaussians whose f32 2x2 determinant is ill-conditioned
    the conic matches the f64 oracle far better than the f32 path; ordinary scenes never
    take the f64 path (records identical with and without it)."""
    g, cam = _needles(63)
    n = g.shape[0]
    planes = G.params_to_planes(ctx, dev(g), n)
    off = G.project_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(sh_degree=0))
    on = G.project_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make(sh_degree=0, fp64_conic=True))
    p64 = O.project_all(g.astype(np.float64), cam.astype(np.float64), sh_degree=0, dtype=np.float64)
    ro, rn = off.to_reference(ctx).cpu().numpy(), on.to_reference(ctx).cpu().numpy()
    vis = (p64[:, 6] > 0) & (ro[:, 6] > 0) & (rn[:, 6] > 0)
    A, B, Cc = p64[vis, 2], p64[vis, 3], p64[vis, 4]
    det = 1.0 / (A * Cc - B * B)
    trace = (A + Cc) * det
    ill = det < 1e-6 * trace * trace
    assert ill.sum() > 50, ill.sum()
    scale = np.abs(p64[vis][:, 2:5]).max(1, keepdims=True)
    e_off = (np.abs(ro[vis][:, 2:5] - p64[vis][:, 2:5]) / scale).max(1)
    e_on = (np.abs(rn[vis][:, 2:5] - p64[vis][:, 2:5]) / scale).max(1)
    print(f"\nill-conditioned: {ill.sum()} of {vis.sum()}; conic rel. error vs f64 oracle: "
          f"f32 median {np.median(e_off[ill]):.2e} max {e_off[ill].max():.2e}, "
          f"f64 re-solve median {np.median(e_on[ill]):.2e} max {e_on[ill].max():.2e}")
    assert e_on[ill].max() < 1e-4
    assert np.median(e_off[ill]) > 10 * np.median(e_on[ill])
    g2, cam2 = small_scene(seed=64)
    p2 = G.params_to_planes(ctx, dev(g2), g2.shape[0])
    a = G.project_all(ctx, p2, g2.shape[0], g2.shape[0], Camera.from_record(cam2), ProjOpts.make())
    b = G.project_all(ctx, p2, g2.shape[0], g2.shape[0], Camera.from_record(cam2), ProjOpts.make(fp64_conic=True))
    assert torch.equal(a.rec, b.rec)
