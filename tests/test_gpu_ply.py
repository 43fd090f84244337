"""PLY codec (reference src/ply.rs) straight into and out of device parameter planes."""
import os

import numpy as np
import pytest
import torch

from splatrs_b200 import gpu as G
from splatrs_b200._lib import SplatError
from tests import fixtures as F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def _model(n, seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 1, (n, 59)).astype(np.float32)


def test_roundtrip_like_reference(ctx, tmp_path):
    """src/ply.rs:192-237: write then read returns every scalar (here: bit-exactly)."""
    g = np.zeros((5, 59), np.float32)
    for i in range(5):
        f = float(i)
        g[i, 0:3] = [f, f + 0.5, f - 0.5]
        g[i, 3:6] = [-f, -f - 1.0, -f - 2.0]
        g[i, 6:10] = [1.0, 0.1 * f, 0.2 * f, 0.3 * f]
        g[i, 10] = f * 0.3
        for k in range(16):
            for c in range(3):
                g[i, 11 + 3 * k + c] = f + k * 0.1 + c * 0.01
    planes = G.params_to_planes(ctx, torch.from_numpy(g).cuda())
    path = str(tmp_path / "m.ply")
    G.ply_write(ctx, path, planes, 5, 5, 3)
    back, n, d, cap = G.ply_read(ctx, path)
    assert (n, d) == (5, 3)
    assert np.array_equal(G.planes_to_params(ctx, back, n, cap).cpu().numpy(), g)


@pytest.mark.parametrize("degree", [0, 1, 2, 3])
def test_reads_reference_layout_and_writes_it_back(ctx, tmp_path, degree):
    """A file in the reference's layout (written here in plain Python) reads into the same
    records, coefficients above the file's degree reading as zero; writing reproduces the
    file byte for byte."""
    g = _model(1000, degree)
    K = (degree + 1) ** 2
    want = g.copy()
    want[:, 11 + 3 * K:] = 0.0
    path = str(tmp_path / f"ref{degree}.ply")
    F.write_ply_reference_layout(path, g, degree)
    planes, n, d, cap = G.ply_read(ctx, path)
    assert (n, d) == (1000, degree)
    assert np.array_equal(G.planes_to_params(ctx, planes, n, cap).cpu().numpy(), want)
    out = str(tmp_path / f"out{degree}.ply")
    G.ply_write(ctx, out, planes, n, cap, degree)
    with open(path, "rb") as a, open(out, "rb") as b:
        assert a.read() == b.read()


def test_property_order_from_header(ctx, tmp_path):
    """Properties in another order (as other tools write them) load by name."""
    g = _model(50, 7)
    names = ["rot_0", "rot_1", "rot_2", "rot_3", "x", "y", "z", "opacity", "scale_0", "scale_1", "scale_2",
             "f_dc_0", "f_dc_1", "f_dc_2"]
    cols = {"x": g[:, 0], "y": g[:, 1], "z": g[:, 2], "scale_0": g[:, 3], "scale_1": g[:, 4], "scale_2": g[:, 5],
            "rot_0": g[:, 6], "rot_1": g[:, 7], "rot_2": g[:, 8], "rot_3": g[:, 9], "opacity": g[:, 10],
            "f_dc_0": g[:, 11], "f_dc_1": g[:, 12], "f_dc_2": g[:, 13]}
    rows = np.stack([cols[nm] for nm in names], 1).astype("<f4")
    path = str(tmp_path / "reordered.ply")
    with open(path, "wb") as f:
        f.write(("ply\nformat binary_little_endian 1.0\nelement vertex 50\n" +
                 "".join(f"property float {nm}\n" for nm in names) + "end_header\n").encode())
        f.write(rows.tobytes())
    planes, n, d, cap = G.ply_read(ctx, path)
    got = G.planes_to_params(ctx, planes, n, cap).cpu().numpy()
    assert d == 0 and np.array_equal(got[:, :14], g[:, :14]) and (got[:, 14:] == 0).all()


@pytest.mark.parametrize("text,msg", [
    (b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n", b"only binary_little_endian"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\n", b"missing end_header"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty double x\nend_header\n", b"only float"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 3\nproperty float x\nend_header\n\0\0\0\0",
     b"shorter than the header"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 0\nproperty float x\nend_header\n", b"missing property y"),
])
def test_format_errors_are_reported(ctx, tmp_path, text, msg):
    """Malformed files fail with SPLAT_ERR_INVALID and the reference's messages."""
    path = str(tmp_path / "bad.ply")
    with open(path, "wb") as f:
        f.write(text)
    with pytest.raises(SplatError) as e:
        G.ply_read(ctx, path)
    assert e.value.status == 1 and msg.decode() in str(e.value)
