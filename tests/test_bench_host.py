"""The bench line's host arithmetic: per-stage rooflines (the bound is the unit whose
measured peak needs the longest for the stage's algorithmic work) and the workload config
both arms report. No GPU."""
import bench


def test_stage_rooflines_pick_the_slowest_unit():
    # The render benchmark's counts with round peaks: 6,500 GB/s, 72.5 TFLOP/s, 4,650 Gop/s.
    ms = {"project_fwd": 0.084, "bin": 0.322, "raster_fwd": 0.542, "raster_bwd": 0.913, "project_bwd": 0.133}
    out = bench.stage_rooflines(ms, 1_000_000, 3_064_031, 109_027_430, 107_974_552, 1920 * 1080, 6500.0, 72.5, 4650.0)
    assert set(out) == set(ms)
    for k, v in out.items():
        assert v["bound"] == max(v["unit_ms"], key=v["unit_ms"].get)
        assert abs(v["frac"] - v["roofline_ms"] / ms[k]) < 1e-3
        assert 0.0 < v["frac"] < 1.0
    # Projection and binning have bytes only; the compositing stages also FLOP and SFU work.
    assert set(out["project_fwd"]["unit_ms"]) == {"hbm"}
    assert set(out["raster_bwd"]["unit_ms"]) == {"hbm", "fp32", "mufu"}
    # 50 FLOP per backward pair: 5.40 GFLOP at 72.5 TFLOP/s is 0.0745 ms, longer than the
    # 200.8 MB at 6.5 TB/s (0.0309 ms) and the 216M exp + reciprocal at 4,650 Gop/s (0.0464 ms).
    assert out["raster_bwd"]["bound"] == "fp32"
    assert abs(out["raster_bwd"]["roofline_ms"] - 0.0745) < 1e-3
    assert out["project_bwd"]["bytes"] == (236 + 36 + 236) * 1_000_000


def test_workload_config_is_the_same_in_both_arms():
    a, b = bench.workload_config(1_000_000, 1), bench.workload_config(1_000_000, 1)
    assert a == b
    assert a["gaussians"] == 1_000_000 and (a["width"], a["height"]) == (1920, 1080)
    assert bench.workload_config(1_000_000, 4)["parallelism"] == "replicas x4"
