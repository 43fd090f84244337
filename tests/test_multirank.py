"""The N > 1 host logic of bench.py (replicas, max over ranks, the reference arm under
torchrun) on two gloo ranks on CPU."""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
from datetime import timedelta
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
import bench
rank, world, local = bench.dist_info()
assert world == 2
v = bench.max_over_ranks(10.0 + 5.0 * rank, world)
assert v == 15.0, v
w = bench.max_over_ranks(3.0 - rank, world)
assert w == 3.0, w
dist.barrier()
dist.destroy_process_group()
print("rank", rank, "ok")
"""


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_max_over_ranks_with_two_gloo_ranks():
    port = free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        out, _ = p.communicate(timeout=120)
        outs.append(out)
        assert p.returncode == 0, out
    assert all("ok" in o for o in outs)


def test_reference_arm_under_two_ranks():
    """`bench.py --impl reference` launched as two ranks: rank 0 alone times the CPU path
    and prints one JSON line with impl "reference" and its e2e object; rank 1 prints
    nothing and both exit 0."""
    import json
    port = free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                                       "--gpus", "2", "--steps", "1", "--warmup", "1", "--n", "20000"], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=300)
        assert p.returncode == 0, err[-2000:]
        outs.append([ln for ln in out.splitlines() if ln.startswith("{")])
    assert len(outs[0]) == 1 and not outs[1]
    line = json.loads(outs[0][0])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["n_gpus"] == 2 and line["higher_is_better"] is True and "workload" in line["config"]
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["unit"] == line["unit"] and cb["cores"] >= 1 and cb["sample"]
    assert set(cb["stages_ms"]) == {"project", "bin", "raster_fwd", "raster_bwd", "project_bwd"}
    assert cb["passed_pairs"]["forward"] >= cb["passed_pairs"]["backward"] > 0
    assert cb["ns_per_pair_core"]["forward"] > 0 and cb["ns_per_pair_core"]["backward"] > 0
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["d2h_bytes_per_step"] == 0
