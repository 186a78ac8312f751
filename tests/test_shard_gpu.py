"""One rank of a partitioned grid on the GPU, through the C ABI (bx_init
with nOwned, bx_halo_pack / bx_halo_unpack, bx_get_dtmin / bx_set_dtmin,
bx_end_step), with the other ranks run by the partitioned oracle in the
same process and the halo interiors moved through host memory before every
stage.  Every rank's owned blocks must match the single-domain oracle:
within 1e-12 per step in FP64, within the FP32-bulk bound (relative L1
1e-6) in FP32-bulk, where stage 2 exchanges the FP32 intermediate state.
One GPU is enough: no kernel waits on another rank."""
import numpy as np
import pytest
import torch

from batsrus_b200 import configs, initial, shard
from batsrus_b200.explicit import ExplicitSolver
from oracle import Oracle

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    ax = tuple(range(a.ndim - 1))
    scale = np.abs(b).max(axis=ax)
    scale[1:4] = np.sqrt((b[..., 1:4] ** 2).sum(-1)).max()
    scale[4:7] = np.sqrt((b[..., 4:7] ** 2).sum(-1)).max()
    return (np.abs(a - b).max(axis=ax) / np.maximum(scale, 1e-300)).max()


def case(name, precision):
    if name == "amr":
        g, s, _, _ = configs.amr_blast(nRoot=2, maxLevel=2, precision=precision, with_state=False)
        return g, s, initial.perturbed_ot(g, seed=3, amplitude=5e-2, kmax=4)
    g, s, st, _ = configs.uniform_3d_case(2, "Linde", "mc3", 1.2, precision=precision, state="ot")
    return g, s, st


def run_hybrid(name, nRank, nStep, precision):
    g, s, st = case(name, precision)
    _, s64, _ = case(name, "fp64")
    rank_of = shard.partition(g, nRank)
    doms = [shard.RankDomain(g, rank_of, r) for r in range(nRank)]
    d0 = doms[0]
    x = ExplicitSolver(d0.grid, s, nOwned=d0.nOwned)
    x.set_state(st[d0.glob])
    ora = {}
    for r in range(1, nRank):
        o = Oracle(doms[r].grid, s64)
        o.set_owned(doms[r].owned)
        o.set_state(st[doms[r].glob])
        ora[r] = o
    isl = g.interior_slices()
    nc = (g.nK, g.nJ, g.nI)

    def to_gpu_layout(inner, dtype):  # (n, k, j, i, v) -> (n, v, k, j, i)
        return torch.from_numpy(np.ascontiguousarray(np.moveaxis(inner, -1, 1)).astype(dtype)).cuda()

    for _ in range(nStep):
        dt = min([x.get_dtmin()] + [o.local_dtmin() for o in ora.values()])
        x.set_dtmin(dt)
        x.set_global_timestep()
        for o in ora.values():
            o.begin_step(dt)
        for stage in range(1, s.nStage + 1):
            dtype = np.float32 if x.halo_bytes(stage) == 4 * 8 * g.nI * g.nJ * g.nK else np.float64
            S = {r: o.get_state() for r, o in ora.items()}
            for r in ora:
                dr = doms[r]
                if r in d0.send:  # GPU rank 0 -> oracle rank r
                    n = len(d0.send[r])
                    buf = torch.empty((n, 8) + nc, dtype=torch.float32 if dtype == np.float32 else torch.float64,
                                      device="cuda")
                    x.halo_pack(stage, d0.send[r], buf.data_ptr())
                    got = np.moveaxis(buf.cpu().numpy().astype(np.float64), 1, -1)
                    inner = S[r][isl]
                    inner[dr.recv[0]] = got
                    S[r][isl] = inner
                if 0 in dr.send:  # oracle rank r -> GPU rank 0
                    buf = to_gpu_layout(S[r][isl][dr.send[0]], dtype)
                    x.halo_unpack(stage, d0.recv[r], buf.data_ptr())
            for r in ora:  # between oracle ranks
                for p in ora:
                    if p != r and p in doms[r].send:
                        inner = S[p][isl]
                        inner[doms[p].recv[r]] = S[r][isl][doms[r].send[p]]
                        S[p][isl] = inner
            for r, o in ora.items():
                o.set_state(S[r])
                o.exchange_messages()
            torch.cuda.synchronize()
            x.set_stage(stage)
            x.update_state_fast()
            for o in ora.values():
                o.stage(stage)
        x.end_step()
        for o in ora.values():
            o.end_step()
    out = {0: x.get_state()[isl][:d0.nOwned]}
    t0 = x.time()
    x.close()
    for r, o in ora.items():
        out[r] = o.get_state()[isl][:doms[r].nOwned]
    ref = Oracle(g, s64)
    ref.set_state(st)
    ref.exchange_messages()
    ref.advance(nStep)
    R = ref.get_state()[isl]
    return {r: (out[r], R[doms[r].glob[:doms[r].nOwned]]) for r in out}, t0, ref.time()


@pytest.mark.parametrize("name,nRank", [("ot", 2), ("amr", 3)])
def test_gpu_rank_matches_single_domain_fp64(name, nRank):
    """Orszag-Tang 16^3 on two ranks, the two-level grid with TVD resolution
    changes on three: the GPU rank and the oracle ranks within 1e-12 of the
    single-domain oracle after three steps, the time within 1e-12."""
    res, tg, to = run_hybrid(name, nRank, 3, "fp64")
    for r, (a, b) in res.items():
        assert rel_err(a, b) < 1e-12, (r, rel_err(a, b))
    assert tg[2] == to[2] and abs(tg[0] - to[0]) <= 1e-12 * to[0]


def test_gpu_rank_fp32_bulk_exchanges_the_fp32_stage():
    """FP32-bulk on the GPU rank: stage 2 exchanges the FP32 intermediate
    state (bx_halo_bytes 4 bytes per value); the result stays within the
    mode's relative L1 bound of the FP64 single-domain oracle."""
    res, _, _ = run_hybrid("amr", 2, 3, "fp32")
    a, b = res[0]
    l1 = np.abs(a - b).sum() / np.abs(b).sum()
    assert l1 < 1e-6, l1


def test_rank_api_rejects_misuse():
    """nOwned beyond the block list, writing an owned block as a halo copy,
    and the parts not built for a partitioned grid return errors."""
    from batsrus_b200 import capi
    g, s, st = case("ot", "fp64")
    rank_of = shard.partition(g, 2)
    d = shard.RankDomain(g, rank_of, 0)
    with pytest.raises(capi.BxError):
        ExplicitSolver(d.grid, s, nOwned=d.grid.nBlock + 1)
    x = ExplicitSolver(d.grid, s, nOwned=d.nOwned)
    buf = torch.zeros(8 * 512, dtype=torch.float64, device="cuda")
    with pytest.raises(capi.BxError):
        x.halo_unpack(1, [0], buf.data_ptr())
    x.halo_unpack(1, [d.nOwned], buf.data_ptr())  # a halo copy
    with pytest.raises(capi.BxError):
        x.calc_face_value(d.nOwned + 1)
    x.close()


def _gpu_rank_process(rank, world, port, out_dir, name, precision):
    import datetime
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    g, s, st = case(name, precision)
    r = shard.GpuRank(g, s, world, rank, device=0)
    r.set_state(st)
    r.advance(3)
    np.save(os.path.join(out_dir, "s%d.npy" % rank), r.get_owned_state()[g.interior_slices()])
    np.save(os.path.join(out_dir, "g%d.npy" % rank), r.dom.glob[:r.dom.nOwned])
    r.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("ot", 2), ("amr", 2)])
def test_gpu_ranks_in_two_processes(tmp_path, name, world):
    """shard.GpuRank in two processes (gloo through host memory, both
    contexts on GPU 0; each exchange completes on the host before the next
    launch): the owned blocks of both ranks match the single-domain oracle
    within 1e-12 after three steps."""
    import os
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    mp.spawn(_gpu_rank_process, args=(world, port, str(tmp_path), name, "fp64"), nprocs=world, join=True)
    g, s, st = case(name, "fp64")
    ref = Oracle(g, s)
    ref.set_state(st)
    ref.exchange_messages()
    ref.advance(3)
    R = ref.get_state()[g.interior_slices()]
    seen = np.zeros(g.nBlock, dtype=bool)
    for q in range(world):
        S = np.load(os.path.join(str(tmp_path), "s%d.npy" % q))
        glob = np.load(os.path.join(str(tmp_path), "g%d.npy" % q))
        seen[glob] = True
        assert rel_err(S, R[glob]) < 1e-12, q
    assert seen.all()
