"""The N > 1 path of bench.py on CPU with world size 2: replicas timed with
a barrier on both sides and the maximum over ranks (gloo standing in for
NCCL), the whole-job value from the slowest rank, and the reference arm
under torch.distributed.run (rank 0 alone runs and prints one line)."""
import datetime
import json
import os
import socket
import subprocess
import sys
import time

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica_rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from batsrus_b200 import configs
    from oracle import Oracle
    g, s, st, _ = configs.orszag_tang_3d(nRoot=2)
    o = Oracle(g, s, n_thread=1)
    o.set_state(st)
    o.exchange_messages()
    o.advance(1)
    local = {}

    def timed():
        t0 = time.perf_counter()
        o.advance(2)
        if rank == 1:
            time.sleep(0.3)  # the slower replica
        local["ms"] = 1e3 * (time.perf_counter() - t0)
        return local["ms"]
    value, ms = bench.replica_rate(timed, g.nCell * 2, world)
    with open(os.path.join(out_dir, "r%d.json" % rank), "w") as f:
        json.dump({"value": value, "ms": ms, "local_ms": local["ms"], "cells": g.nCell}, f)
    dist.destroy_process_group()


def test_replicas_are_timed_by_the_slowest_rank(tmp_path):
    mp.spawn(_replica_rank, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    r = [json.load(open(os.path.join(str(tmp_path), "r%d.json" % k))) for k in range(2)]
    assert r[0]["ms"] == r[1]["ms"] == max(r[0]["local_ms"], r[1]["local_ms"])
    assert r[1]["local_ms"] >= 300
    for q in r:
        assert abs(q["value"] - 2 * q["cells"] * 2 / (q["ms"] * 1e-3)) <= 1e-9 * q["value"]


def test_reference_arm_prints_one_line_from_rank_zero():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
