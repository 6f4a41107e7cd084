"""Multi-rank host logic of bench.py on CPU: two `gloo` ranks (world size 2), each building its own
shard of the batched workload, timing with a barrier and a max-over-ranks reduction; no data-path
collective.  Runs as spawned child processes on 127.0.0.1."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import bench
from mumblebee_b200.ipm import Context

class A: pass
ws, rank, local, pg = bench.dist_setup(A())
probs, sizes = bench.make_problems(6, 0, rank, Context.host())
again, sizes2 = bench.make_problems(6, 0, rank, Context.host())
bench.barrier(pg, local)
mx = bench.allreduce_max(pg, 10.0 + rank, local)
print(json.dumps({"rank": rank, "ws": ws, "sizes": [int(s) for s in sizes], "same": list(sizes) == list(sizes2),
                  "max": mx, "n": [p.info()["n"] for p in probs]}), flush=True)
pg.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_instances_and_reduce_max():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(r),
                   LOCAL_RANK=str(r), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=300)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    outs.sort(key=lambda d: d["rank"])
    assert [d["ws"] for d in outs] == [2, 2]
    assert all(d["same"] for d in outs)                  # each rank's shard is deterministic
    assert outs[0]["sizes"] != outs[1]["sizes"]          # and the ranks solve different instances
    assert all(d["max"] == 11.0 for d in outs)           # device time = max over ranks
    for d in outs:                                       # problem n = n_assets + nfac + (1 + n_assets + nfac)
        assert d["n"] == [2 * s + 21 for s in d["sizes"]]
