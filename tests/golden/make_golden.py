"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

The reference (a Rust crate) ships no golden vectors and cannot be built in this
environment, so these vectors are the oracle's answers on fixed inputs. The oracle itself is
pinned by replaying the reference's own tests (tests/test_oracle_*.py: its finite-difference
gradient checks, tiled == naive compositing, the training tests and its exact-answer unit
tests). The fixtures freeze those answers: tests/test_golden.py checks that the oracle still
reproduces them bit for bit, and tests/test_gpu_golden.py checks the CUDA path against them.

render_chain_72x56.npz — one view of the whole render path, computed with the correctly
rounded exp/log that the kernels use (the oracle's `set_cr_math(True)` mode):
  inputs   params (n, 59) f32 (reference record order), cam (18,) f32, background (3,) f32,
           dimage (H*W*3,) f32, antialias / sh_degree scalars;
  outputs  proj (n, 15) (project_all), tile_range (tiles, 2) u32 and gauss (entries,) u32
           (bin, entries in sorted order), image / final_t / n_contrib / pairs
           (rasterize_forward), screen_grads (n, 9) / screen_abs (n, 2) / bwd_pairs
           (rasterize_backward), param_grads (n, 59) (project_backward_all of screen_grads).
  The scene holds the cases the reference's tests exercise: a ragged 72x56 view (4.5 x 3.5
  tiles), large Gaussians spanning many tiles, faint ones near the 1/255 alpha cut-off,
  Gaussians behind the camera (culled, zero gradients), and exact duplicates, whose equal
  depths make the sort fall back to the entry-index tie break.

mlp_bf16_256.npz — the learned-densification network (no reference counterpart) on 256
feature rows: theta (5443,) f32, x (256, 16) f32, y (256,) i32, w (256,) f32; outputs
probs (256, 3) and grad (5443,) in the oracle's bf16 mode, both float64.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import mlp as M  # noqa: E402
from oracle import oracle as O  # noqa: E402
from splatrs_b200 import scenes  # noqa: E402

RENDER_FILE = os.path.join(HERE, "render_chain_72x56.npz")
MLP_FILE = os.path.join(HERE, "mlp_bf16_256.npz")
WIDTH, HEIGHT = 72, 56


def render_inputs():
    rng = np.random.default_rng(2024)
    g = scenes.random_gaussians(rng, 300, -1.0, 1.0, -3.3, 0.5, 1.2)
    g[::10, 3:6] = [-0.8, -1.0, -0.9]   # large: many tiles each
    g[5::17, 10] = -4.8                 # faint: alpha near the 1/255 cut-off
    g[3::23, 2] = -50.0                 # behind the camera: culled
    g[200:210] = g[100:110]             # exact duplicates: depth ties
    cam = scenes.look_at(WIDTH, HEIGHT, 0.9 * WIDTH, 0.9 * WIDTH, (0.4, -0.3, -3.2), (0, 0, 0))
    bg = np.array([0.3, 0.6, 0.1], np.float32)
    dimage = rng.normal(0.0, 1.0, WIDTH * HEIGHT * 3).astype(np.float32)
    return dict(params=g, cam=cam, background=bg, dimage=dimage, antialias=np.int32(1), sh_degree=np.int32(3))


def render_outputs(inp):
    """The oracle's render path on `inp` (in whatever exp/log mode is set)."""
    g, cam, bg, dimage = inp["params"], inp["cam"], inp["background"], inp["dimage"]
    opts = dict(antialias=bool(inp["antialias"]), sh_degree=int(inp["sh_degree"]))
    p = O.project_all(g, cam, **opts)
    ob = O.bin(p, WIDTH, HEIGHT)
    a = ob.arrays()
    img, ft, nc, pairs = O.rasterize_forward(p, ob, WIDTH, HEIGHT, bg)
    sg, sa, bpairs = O.rasterize_backward(p, ob, WIDTH, HEIGHT, bg, ft, nc, dimage)
    pgr = O.project_backward_all(g, cam, sg, **opts)
    return dict(proj=p, tile_range=a["tile_range"], gauss=a["entry_gaussian"][a["entries"]], image=img, final_t=ft,
                n_contrib=nc, pairs=np.uint64(pairs), screen_grads=sg, screen_abs=sa, bwd_pairs=np.uint64(bpairs),
                param_grads=pgr)


def mlp_inputs():
    rng = np.random.default_rng(77)
    theta = M.init_params(77).astype(np.float32)
    theta[M.NUM_PARAMS - 3:] = rng.normal(0.0, 0.3, 3)
    x = rng.normal(0.0, 1.0, (256, M.IN)).astype(np.float32)
    y = rng.integers(0, M.OUT, 256).astype(np.int32)
    w = rng.uniform(0.2, 2.0, 256).astype(np.float32)
    return dict(theta=theta, x=x, y=y, w=w)


def mlp_outputs(inp):
    probs, _ = M.forward(inp["theta"], inp["x"], bf16_like=True)
    grad = M.backward(inp["theta"], inp["x"], inp["y"], inp["w"], bf16_like=True)
    return dict(probs=probs, grad=grad)


def main():
    O.set_cr_math(True)
    try:
        inp = render_inputs()
        out = render_outputs(inp)
    finally:
        O.set_cr_math(False)
    np.savez_compressed(RENDER_FILE, **inp, **out)
    vis = int((out["proj"][:, 6] > 0).sum())
    print(f"{RENDER_FILE}: {inp['params'].shape[0]} Gaussians, {vis} visible, {out['gauss'].size} entries, "
          f"{int(out['pairs'])} pairs")
    mi = mlp_inputs()
    np.savez_compressed(MLP_FILE, **mi, **mlp_outputs(mi))
    print(MLP_FILE)


if __name__ == "__main__":
    main()
