"""bench.py's multi-rank plumbing with two gloo ranks on the CPU (one process
per rank under torch.distributed.run, rendezvous on 127.0.0.1): the barrier,
the max over ranks of the timed region, and the reference arm, which rank 0
alone runs and prints. Each rank sends its stdout to a file of its own, so the
ranks' lines cannot interleave on one pipe."""
import json
import os
import socket
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
rank, world, local = bench.env_rank()
sys.stdout = open(os.path.join({outdir!r}, f"rank{{rank}}.out"), "w")
dist = bench.dist_init(world, False)
bench.dist_barrier(dist, False)
# each rank's timed region differs; every rank must see the largest
m = bench.dist_max(dist, 1.5 * (rank + 1), False)
# the reference arm with its CPU sampler stubbed: rank 0 alone runs and prints
bench.run_cpu = lambda steps, warm, n: {{"value": 0.5, "cores": 1, "kind": "port",
                                        "sample": "stub", "cell_updates_per_s": 1.0}}
class Args:
    steps, warmup, n, gpus, direct_steps = 2, 3, 16, world, 0
bench.reference_arm(Args, rank, world)
bench.dist_barrier(dist, False)
print(json.dumps({{"rank": rank, "world": world, "max": m}}), flush=True)
sys.stdout.close()
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks():
    with tempfile.TemporaryDirectory() as d:
        script = os.path.join(d, "rank.py")
        with open(script, "w") as f:
            f.write(RANK_SCRIPT.format(root=ROOT, outdir=d))
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
               "--master-addr", "127.0.0.1", "--master-port", str(free_port()), script]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=240)
        assert r.returncode == 0, r.stderr[-3000:]
        lines = []
        for rank in (0, 1):
            with open(os.path.join(d, f"rank{rank}.out")) as f:
                lines += [json.loads(x) for x in f.read().splitlines() if x.startswith("{")]
    ranks = [x for x in lines if "rank" in x]
    refs = [x for x in lines if x.get("impl") == "reference"]
    assert sorted(x["rank"] for x in ranks) == [0, 1]
    assert all(x["world"] == 2 and x["max"] == 3.0 for x in ranks)
    assert len(refs) == 1 and refs[0]["value"] == 0.5 and refs[0]["n_gpus"] == 2
