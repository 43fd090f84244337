"""Initialisation from a point cloud on the device (reference src/model.rs:77-186) and the
host-buffer renderer against the stage functions."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from splatrs_b200 import gpu as G
from splatrs_b200 import scenes
from splatrs_b200._lib import Camera, ProjOpts

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


def test_nn_distances_match_brute_force(ctx):
    """src/model.rs:192-226 on the device, and bit-identical to the oracle."""
    rng = np.random.default_rng(12345)
    pts = rng.random((2000, 3)).astype(np.float32)
    got = G.mean_nn_dist2(ctx, torch.from_numpy(pts).cuda()).cpu().numpy()
    assert np.array_equal(got, O.mean_nn_dist2(pts))
    p64 = pts.astype(np.float64)
    for i in range(0, 2000, 97):
        d = np.sort(np.delete(((p64 - p64[i]) ** 2).sum(1), i))
        want = (d[0] + d[1] + d[2]) / 3.0
        assert abs(got[i] - want) < 1e-12 * max(want, 1e-6)


def test_nn_distances_handle_coincident_points(ctx):
    """src/model.rs:228-246 on the device."""
    pts = np.zeros((42, 3), np.float32)
    pts[40] = [1, 0, 0]
    pts[41] = [0, 2, 0]
    got = G.mean_nn_dist2(ctx, torch.from_numpy(pts).cuda()).cpu().numpy()
    assert (got[:40] == 0.0).all() and got[40] == 1.0 and got[41] == 4.0
    two = np.array([[0, 0, 0], [0, 0, 3]], np.float32)
    got = G.mean_nn_dist2(ctx, torch.from_numpy(two).cuda()).cpu().numpy()
    assert got[0] == 9.0 and got[1] == 9.0


def test_init_from_points_bit_exact(ctx, cr_math):
    """Model::from_points: every record bit-identical to the oracle's."""
    rng = np.random.default_rng(3)
    pts = rng.normal(0, 1, (5000, 3)).astype(np.float32)
    rgb = rng.integers(0, 256, (5000, 3)).astype(np.uint8)
    planes = G.init_from_points(ctx, pts, rgb)
    got = G.planes_to_params(ctx, planes, 5000, 5000).cpu().numpy()
    want = O.from_points(pts, rgb)
    assert np.array_equal(got, want)


def test_renderer_host_api_matches_stage_api(ctx):
    """splat_renderer_render_backward (host buffers, pipelined copies) returns the image of
    the stage functions bit for bit and the same parameter gradients."""
    rng = np.random.default_rng(8)
    g = scenes.random_gaussians(rng, 30000, -1.0, 1.0, -3.6, 0.5, 1.0)
    camr = scenes.look_at(800, 600, 700.0, 700.0, (0.3, -0.4, -3.3), (0, 0, 0))
    cam = Camera.from_record(camr)
    opts = ProjOpts.make(sh_degree=2)
    bg = (0.2, 0.1, 0.0)
    dimage = rng.normal(0, 1, 800 * 600 * 3).astype(np.float32)
    r = G.Renderer(ctx)
    r.set_model(g, 2)
    image, grads = r.render_backward(cam, opts, bg, dimage)
    assert np.array_equal(r.render(cam, opts, bg), image)
    planes = G.params_to_planes(ctx, torch.from_numpy(g).cuda())
    proj = G.project_all(ctx, planes, g.shape[0], g.shape[0], cam, opts)
    b = G.bin(ctx, proj)
    out = G.rasterize_forward(ctx, proj, b, bg)
    pg = G.rasterize_backward(ctx, proj, b, bg, out, torch.from_numpy(dimage).cuda())
    gp = G.project_backward_all(ctx, planes, g.shape[0], g.shape[0], cam, opts, proj, pg)
    want = G.planes_to_params(ctx, gp, g.shape[0], g.shape[0]).cpu().numpy()
    assert np.array_equal(out.image.cpu().numpy(), image)
    scale = np.maximum(np.abs(want).max(0), 1e-30)
    assert (np.abs(grads - want).max(0) / scale).max() < 1e-5
    assert r.last_entries == b.num_entries
    r.close()
