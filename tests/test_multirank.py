"""The N > 1 host path of bench.py on CPU ranks (gloo, world size 2): the
max / sum reductions of the timings, the gather of per-request latencies
and the partition of the serving stream across ranks."""
import json
import os
import socket
import subprocess
import sys
import tempfile

from conftest import ROOT

RANK_SCRIPT = r'''
import json, os, sys
sys.path.insert(0, {root!r})
import bench
ws, rank, local = bench.dist_setup()
out = {{
    "ws": ws, "rank": rank,
    "max": bench.allreduce_max(float(rank + 1) * 1.5, ws),
    "sum": bench.allreduce_sum(float(rank + 1), ws),
    "gather": bench.gather([rank, rank * 10], ws),
    "shard": bench.serving_shard(7, ws, rank),
}}
bench.barrier(ws)
json.dump(out, open(os.path.join({tmp!r}, "rank%d.json" % rank), "w"))
import torch.distributed as dist
dist.destroy_process_group()
'''


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_reduce_gather_and_shard():
    with tempfile.TemporaryDirectory() as tmp:
        script = os.path.join(tmp, "rank.py")
        open(script, "w").write(RANK_SCRIPT.format(root=ROOT, tmp=tmp))
        env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
               "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), script]
        r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        outs = [json.load(open(os.path.join(tmp, f"rank{k}.json"))) for k in range(2)]
    for o in outs:
        assert o["ws"] == 2
        assert o["max"] == 3.0 and o["sum"] == 3.0
        assert o["gather"] == [[0, 0], [1, 10]]
    shards = [o["shard"] for o in sorted(outs, key=lambda o: o["rank"])]
    assert shards == [[0, 2, 4, 6], [1, 3, 5]]
    assert sorted(shards[0] + shards[1]) == list(range(7))
