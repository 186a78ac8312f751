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
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--nroot", "8"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["cells"] == 64 ** 3 and d["config"]["blocks"] == 512


def _gloo_send_recv(peer, out, shape):
    """one pairwise halo exchange over gloo (nonblocking send and receive);
    empty directions are skipped on both sides"""
    import numpy as np
    import torch
    import torch.distributed as dist
    reqs = []
    if out.shape[0]:
        reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(out)), dst=peer))
    got = torch.empty(shape, dtype=torch.float64)
    if shape[0]:
        reqs.append(dist.irecv(got, src=peer))
    for r in reqs:
        r.wait()
    return got.numpy()


def _sharded_rank(rank, world, port, out_dir, case):
    """One rank of the partitioned oracle: the owned blocks plus halo copies
    of the remote blocks they read, the halos refreshed by point-to-point
    exchange before every stage, the time step a MIN over the ranks."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import numpy as np
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from batsrus_b200 import shard
    from oracle import Oracle
    g, s, st, nStep = _sharded_case(case)
    rank_of = shard.partition(g, world)
    dom = shard.RankDomain(g, rank_of, rank)
    o = Oracle(dom.grid, s, n_thread=1)
    o.set_owned(dom.owned)
    o.set_state(st[dom.glob])
    isl = dom.grid.interior_slices()
    for _ in range(nStep):
        dt = torch.tensor([o.local_dtmin()], dtype=torch.float64)
        dist.all_reduce(dt, op=dist.ReduceOp.MIN)
        o.begin_step(float(dt.item()))
        for stage in range(1, s.nStage + 1):
            S = o.get_state()
            inner = S[isl]
            dom.exchange(inner, _gloo_send_recv)
            S[isl] = inner
            o.set_state(S)
            o.exchange_messages()
            o.stage(stage)
        o.end_step()
    S = o.get_state()[isl][:dom.nOwned]
    np.save(os.path.join(out_dir, "r%d.npy" % rank), S)
    np.save(os.path.join(out_dir, "g%d.npy" % rank), dom.glob[:dom.nOwned])
    with open(os.path.join(out_dir, "t%d.json" % rank), "w") as f:
        json.dump(list(o.time()), f)
    dist.barrier()
    dist.destroy_process_group()


def _sharded_case(case):
    from batsrus_b200 import configs, initial
    if case == "amr":
        g, s, _, _ = configs.amr_blast(nRoot=2, maxLevel=2, precision="fp64", with_state=False)
        st = initial.perturbed_ot(g, seed=3, amplitude=5e-2, kmax=4)
        return g, s, st, 3
    g, s, st, _ = configs.uniform_3d_case(2, "Linde", "mc3", 1.2, state="ot")
    return g, s, st, 3


def _check_sharded(tmp_path, case, world):
    import numpy as np
    from oracle import Oracle
    mp.spawn(_sharded_rank, args=(world, free_port(), str(tmp_path), case), nprocs=world, join=True)
    g, s, st, nStep = _sharded_case(case)
    o = Oracle(g, s)
    o.set_state(st)
    o.exchange_messages()
    o.advance(nStep)
    ref = o.get_state()[g.interior_slices()]
    seen = np.zeros(g.nBlock, dtype=bool)
    for r in range(world):
        S = np.load(os.path.join(str(tmp_path), "r%d.npy" % r))
        glob = np.load(os.path.join(str(tmp_path), "g%d.npy" % r))
        assert len(glob) > 0 and not seen[glob].any()
        seen[glob] = True
        assert np.array_equal(S, ref[glob]), (r, np.abs(S - ref[glob]).max())
        assert json.load(open(os.path.join(str(tmp_path), "t%d.json" % r))) == list(o.time())
    assert seen.all()


def test_sharded_orszag_tang_matches_one_domain_bit_for_bit(tmp_path):
    """A periodic 16^3 Orszag-Tang grid (8 blocks) split into two Morton
    ranges over two gloo ranks: three steps of the partitioned oracle give
    the single-domain state and time bit for bit."""
    _check_sharded(tmp_path, "ot", 2)


def test_sharded_amr_with_resolution_changes_matches_one_domain(tmp_path):
    """A two-level periodic grid (120 blocks) on three ranks, TVD faces at
    the resolution changes: halo copies of coarser and finer neighbours
    supply the ghost fill and the flux correction; bit for bit."""
    _check_sharded(tmp_path, "amr", 3)


def test_partition_and_halo_lists():
    """Morton ranges of equal block counts (or weights); every block a rank
    reads is owned or a halo copy; the send list of one rank is the receive
    list of its peer, block for block."""
    import numpy as np
    from batsrus_b200 import configs, restart, shard
    g = configs.amr_blast(nRoot=2, maxLevel=2, with_state=False)[0]
    for n in (1, 2, 3, 5):
        r = shard.partition(g, n)
        counts = np.bincount(r, minlength=n)
        assert counts.max() - counts.min() <= 1
        pos = restart.morton_order(g) - 1
        assert (np.diff(r[np.argsort(pos)]) >= 0).all()  # contiguous along the curve
    w = 1.0 + g.iLevelCoord[:, 0]
    r = shard.partition(g, 3, weights=w)
    load = np.bincount(r, weights=w, minlength=3)
    assert load.max() - load.min() <= 2 * w.max()
    rank_of = shard.partition(g, 3)
    rd = shard.reads(g)
    doms = [shard.RankDomain(g, rank_of, q) for q in range(3)]
    for q, d in enumerate(doms):
        have = set(int(b) for b in d.glob)
        for b in d.glob[:d.nOwned]:
            assert rank_of[b] == q and set(int(x) for x in rd[b]) <= have
        for p, idx in d.send.items():
            assert np.array_equal(d.glob[idx], doms[p].glob[doms[p].recv[q]])
