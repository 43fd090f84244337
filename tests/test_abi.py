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
