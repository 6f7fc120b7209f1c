"""CPU test of bench.py's multi-process plumbing (one process per GPU on a
B200 node): two gloo ranks, each with its own value; the max over ranks is
what every rank gets, as the timings and the Res64 verdicts use it."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys, json
sys.path.insert(0, %r)
import bench
world, rank, local = bench.dist_init("gloo")
t = bench.allreduce_max(10.0 * (rank + 1), world)
ok = bench.allreduce_max(0.0 if rank == 0 else 1.0, world)
bench.barrier(world)
print(json.dumps({"rank": rank, "world": world, "max": t, "any_failed": ok}))
import torch.distributed as dist
dist.destroy_process_group()
""" % ROOT


def test_two_rank_max_over_ranks_with_gloo(tmp_path):
    script = tmp_path / "child.py"
    script.write_text(CHILD)
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT="29613")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    assert all(p.returncode == 0 for p in procs), [o[1][-500:] for o in outs]
    import json
    res = [json.loads(o[0].strip().split("\n")[-1]) for o in outs]
    assert sorted(r["rank"] for r in res) == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 20.0 and r["any_failed"] == 1.0 for r in res)
