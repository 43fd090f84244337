"""splat_bin_count_noalloc against splat_bin_count, through the C ABI.

The no-allocation entry point exists for callers that plan all device memory themselves
(a fixed per-frame budget, or their own allocator owning the device) and so cannot let the
library call cudaMalloc; it takes its scratch from a fixed array in device memory. This
file is collected last so that a failure here comes after every other test has run; it
also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from splatrs_b200 import _lib
from splatrs_b200 import gpu as G
from splatrs_b200 import scenes
from splatrs_b200._lib import Camera, ProjOpts

pytestmark = pytest.mark.gpu


def _tile_counts(ctx, seed, n):
    rng = np.random.default_rng(seed)
    g = scenes.random_gaussians(rng, n, -1.0, 1.0, -3.5, 0.6, 1.0)
    cam = scenes.look_at(640, 480, 560.0, 560.0, (0.2, -0.1, -3.0), (0, 0, 0))
    planes = G.params_to_planes(ctx, torch.from_numpy(g).cuda())
    proj = G.project_all(ctx, planes, n, n, Camera.from_record(cam), ProjOpts.make())
    return proj.num_tiles


def _count(ctx, fn, num_tiles):
    n = num_tiles.numel()
    off = torch.full((n + 1,), -7, dtype=torch.int32, device="cuda")
    e = C.c_int64(-1)
    st = fn(ctx.h, C.c_void_p(num_tiles.data_ptr()), n, C.c_void_p(off.data_ptr()), C.byref(e))
    _lib.check(st, ctx.h)
    return off.cpu().numpy(), int(e.value)


def test_bin_count_noalloc_matches_bin_count_on_two_calls():
    """Two calls in a row with different inputs: offsets and counts equal the allocating
    entry point's exactly (integer results)."""
    ctx = G.Context(0)
    L = ctx.lib
    for seed, n in ((1, 50_000), (2, 123_457)):
        nt = _tile_counts(ctx, seed, n)
        want_off, want_e = _count(ctx, L.splat_bin_count, nt)
        got_off, got_e = _count(ctx, L.splat_bin_count_noalloc, nt)
        assert want_e > n // 2
        assert got_e == want_e
        assert np.array_equal(got_off, want_off)
    ctx.close()


def test_bin_count_noalloc_allocates_nothing_at_its_largest_size():
    """n = 16,777,216, the largest size the fixed scratch accepts (its 4,096 partial sums
    and the total fill the array to its last word), on a fresh context: the result equals
    the allocating entry point's, and neither the context's scratch arena nor the device's
    free memory changes around the call."""
    n = 16_777_216
    torch.manual_seed(5)
    nt = torch.randint(0, 4, (n,), dtype=torch.int32, device="cuda")
    off = torch.full((n + 1,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx = G.Context(0)
    L = ctx.lib
    # A first call resolves the scratch address once (no allocation either way).
    e = C.c_int64(-1)
    _lib.check(L.splat_bin_count_noalloc(ctx.h, C.c_void_p(nt.data_ptr()), 16, C.c_void_p(off.data_ptr()),
                                         C.byref(e)), ctx.h)
    torch.cuda.synchronize()
    arena0 = ctx.scratch_info
    free0 = torch.cuda.mem_get_info()[0]
    _lib.check(L.splat_bin_count_noalloc(ctx.h, C.c_void_p(nt.data_ptr()), n, C.c_void_p(off.data_ptr()),
                                         C.byref(e)), ctx.h)
    torch.cuda.synchronize()
    assert ctx.scratch_info == arena0 == (0, 0)
    assert torch.cuda.mem_get_info()[0] == free0
    got_off, got_e = off.cpu().numpy().copy(), int(e.value)
    want_off, want_e = _count(ctx, L.splat_bin_count, nt)
    assert got_e == want_e == int(nt.sum().item())
    assert np.array_equal(got_off, want_off)
    ctx.close()


def test_bin_count_noalloc_rejects_sizes_beyond_its_scratch():
    """More counts than the fixed scratch covers: SPLAT_ERR_CAPACITY before any device work."""
    ctx = G.Context(0)
    nt = torch.zeros(16, dtype=torch.int32, device="cuda")
    off = torch.zeros(17, dtype=torch.int32, device="cuda")
    e = C.c_int64(-1)
    st = ctx.lib.splat_bin_count_noalloc(ctx.h, C.c_void_p(nt.data_ptr()), 16_777_217, C.c_void_p(off.data_ptr()),
                                         C.byref(e))
    assert st == _lib.SPLAT_ERR_CAPACITY
    assert b"16777216" in ctx.lib.splat_last_error(ctx.h)
    ctx.close()
