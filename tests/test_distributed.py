"""Replica plumbing of bench.py on CPU: two gloo ranks, barrier and max-over-ranks timing.

The path has no exchange step (molecules are independent), so multi-GPU runs are replicas;
this covers the host-side logic a 2-rank run uses, without a GPU.
"""
import os
import subprocess
import sys
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

WORKER = textwrap.dedent("""
    import os, sys, json
    sys.path.insert(0, {root!r})
    import bench
    world, rank, local, pg = bench.dist_setup("gloo")
    bench.barrier(pg)
    t = bench.max_over_ranks(pg, 10.0 + rank)
    # each replica evaluates the full workload: value = world * points / max time
    v = world * 128 ** 3 / (t / 1000.0)
    print(json.dumps({{"rank": rank, "world": world, "t": t, "value": v}}))
    pg.destroy_process_group()
""")


def test_two_rank_replicas_gloo(tmp_path):
    w = tmp_path / "worker.py"
    w.write_text(WORKER.format(root=str(ROOT)))
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT="29513")
    procs = []
    for r in range(2):
        e = dict(env, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2")
        procs.append(subprocess.Popen([sys.executable, str(w)], env=e, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    assert all(p.returncode == 0 for p in procs), [o[1][-2000:] for o in outs]
    import json
    res = [json.loads(o[0].strip().splitlines()[-1]) for o in outs]
    assert all(r["t"] == 11.0 for r in res)            # max over ranks
    assert all(r["world"] == 2 for r in res)
    assert abs(res[0]["value"] - 2 * 128 ** 3 / 0.011) < 1e-3
