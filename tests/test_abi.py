"""The C-ABI library loads on a machine without a GPU and exports every entry point the
header declares (no compute calls here)."""
import ctypes as C
import os
import re

from splatrs_b200 import _lib


def declared():
    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "splat_gpu.h")
    with open(hdr) as f:
        src = f.read()
    return sorted(set(re.findall(r"SPLAT_API\s+[\w\s\*]+?\b(splat_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    names = declared()
    assert len(names) >= 20
    L = _lib.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_version():
    L = _lib.lib()
    assert L.splat_version() >= 1
    assert L.splat_status_string(0) == b"ok"
    assert L.splat_status_string(2) == b"capacity exceeded"


def test_context_creation_fails_cleanly_without_device():
    import torch
    if torch.cuda.is_available():
        return
    L = _lib.lib()
    h = C.c_void_p()
    st = L.splat_ctx_create(0, None, C.byref(h))
    assert st == _lib.SPLAT_ERR_CUDA and not h.value


def test_struct_layouts_match_the_library():
    """The ctypes mirrors of the public structs have the sizes the library was compiled
    with (a field added on one side only shows here)."""
    L = _lib.lib()
    out = (C.c_uint64 * 16)()
    k = L.splat_struct_sizes(out)
    mirrors = [_lib.Camera, _lib.ProjOpts, _lib.LearningRates, _lib.DensifyConfig, _lib.TrainConfig,
               _lib.DensifyReport, _lib.StepInfo]
    assert k == len(mirrors)
    for i, m in enumerate(mirrors):
        assert C.sizeof(m) == out[i], (m.__name__, C.sizeof(m), out[i])


def test_every_status_has_its_string():
    L = _lib.lib()
    want = {0: b"ok", 1: b"invalid argument", 2: b"capacity exceeded", 3: b"CUDA error", 4: b"device wait timed out"}
    for code, text in want.items():
        assert L.splat_status_string(code) == text
    assert L.splat_status_string(99) == b"unknown status"


def test_raster_candidates_are_the_supported_configurations():
    """splat_raster_candidates needs no device: the 24 compositing configurations (tile
    8x8, 16x16 or 16x32; chunk depth 32-256; 1 or 2 backward pixels per thread), each once,
    the reference's 16x16 tile with the deepest chunk first; NULL asks only for the count."""
    from splatrs_b200.gpu import Context
    L = _lib.lib()
    assert L.splat_raster_candidates(None) == 24
    cands = Context.raster_candidates()
    want = {(w, h, ch, p) for (w, h) in ((8, 8), (16, 16), (16, 32)) for ch in (32, 64, 128, 256) for p in (1, 2)}
    assert len(cands) == 24 and set(cands) == want
    assert cands[0] == (16, 16, 256, 1)


def test_train_config_rejects_unknown_fields():
    """TrainConfig.make (the ctypes mirror of splat_train_config) fills the defaults, takes
    `near` for near_plane and refuses a field the library does not have."""
    import pytest
    c = _lib.TrainConfig.make(iterations=123, near=0.5, autotune=1)
    assert c.iterations == 123 and abs(c.near_plane - 0.5) < 1e-7 and c.autotune == 1
    assert c.densify_from_iter == 500 and c.densify_until_iter == 15000 and c.sh_degree == 3
    with pytest.raises(KeyError):
        _lib.TrainConfig.make(iterationz=1)
