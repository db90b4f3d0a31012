"""CPU: the multi-rank plumbing of bench.py (replicas, no data-path
collective) with world size 2 over gloo: every rank takes the same
collective steps, the reported device time is the slowest rank's, and the
whole-job rate counts every rank's zones."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, %r)
import bench
world, rank, local = bench.dist_setup(backend="gloo")
ms = 10.0 + 5.0 * rank                      # rank 1 is the slower one
bench.barrier(world)
tmax = bench.reduce_max(ms, world, local)
zones, steps = 1000, 4
value = zones * steps * world / (tmax / 1e3)
with open(os.path.join(sys.argv[1], "rank%%d.json" %% rank), "w") as f:
    json.dump({"rank": rank, "world": world, "tmax": tmax, "value": value}, f)
import torch.distributed as dist
dist.barrier()
dist.destroy_process_group()
""" % ROOT


def test_two_gloo_ranks_report_the_slowest_rank(tmp_path):
    w = tmp_path / "worker.py"
    w.write_text(WORKER)
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", "--master-port=%d" % port, str(w), str(tmp_path)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=240, env=env)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-3000:])
    import json
    lines = [json.load(open(tmp_path / ("rank%d.json" % k))) for k in range(2)]
    assert len(lines) == 2
    for d in lines:
        assert d["world"] == 2
        assert d["tmax"] == 15.0
        assert abs(d["value"] - 1000 * 4 * 2 / 0.015) < 1e-6
