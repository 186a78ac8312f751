"""Partition of a block-adaptive grid over ranks (one GPU per rank) and the
ghost bookkeeping of each rank.

BATS-R-US distributes the blocks over MPI ranks and passes ghost cells with
BATL's message_pass_cell / message_pass_face (call sites
src/ModMessagePass.f90:147-226, src/ModAdvanceExplicit.f90:127); the time
step is an MPI_allreduce MIN (src/ModTimeStepControl.f90:392).  Here:

* ``partition``: contiguous ranges of the space-filling (Morton) order of
  the blocks, iMortonNode_A of the restart files, balanced by block count
  (each block costs the same with one global time step) or by given
  per-block weights.
* ``reads``: the blocks whose interior the stage of a block reads.  The
  stencil of a face reaches two cells across the block side: the
  same-level neighbour's interior; at a resolution change the coarser
  neighbour (injection into two ghost layers) or the four finer neighbours
  (their cells next to the face for the restriction, and their faces'
  fluxes for the flux correction, which depend on their first cell layers
  and, through their own ghost cells, on this block).
* ``RankDomain``: the local block list of one rank, its owned blocks
  first (in Morton order), then copies of the remote blocks they read
  ("halo blocks", also in Morton order), with the lists of blocks to send
  to and receive from every other rank.  Every rank derives every list from
  the global tree, so no list is exchanged.  Before each stage the owners
  send the interiors of the blocks in the peers' lists and the peers
  overwrite their halo copies; then each rank runs the stage over its owned
  blocks only, and a MIN over the ranks gives the next time step.

A halo block is a full copy of the remote block's interior; the stage reads
only the layers it needs from it.  No kernel reads another GPU's memory:
the copies live in the receiving rank's own state array.
"""
import numpy as np

from .grid import BlockGrid
from .restart import morton_order


def partition(grid, nRank, weights=None):
    """rank of every block: the blocks in Morton order cut into nRank
    contiguous ranges of (nearly) equal weight (default: one per block)"""
    if nRank < 1:
        raise ValueError("nRank=%d" % nRank)
    order = morton_order(grid) - 1  # position of block b along the curve
    blocks = np.argsort(order, kind="stable")  # blocks along the curve
    w = np.ones(grid.nBlock) if weights is None else np.asarray(weights, dtype=np.float64)
    if w.shape != (grid.nBlock,) or (w <= 0).any():
        raise ValueError("one positive weight per block")
    cum = np.cumsum(w[blocks])
    total = cum[-1]
    rank = np.empty(grid.nBlock, dtype=np.int32)
    # block at position p goes to the rank whose share its weight centre falls in
    centre = cum - 0.5 * w[blocks]
    rank[blocks] = np.minimum((centre * nRank / total).astype(np.int64), nRank - 1)
    return rank


def reads(grid):
    """list of arrays: reads(grid)[b] = the blocks (other than b) whose
    interior the stage of block b reads"""
    dil, jb = grid.neighbors()
    out = []
    for b in range(grid.nBlock):
        s = set()
        for side in range(6):
            if dil[b, side] == 0 or dil[b, side] == 1:
                s.add(int(jb[b, side, 0]))
            elif dil[b, side] == -1:
                s.update(int(q) for q in jb[b, side] if q >= 0)
        s.discard(b)
        out.append(np.array(sorted(s), dtype=np.int64))
    return out


class RankDomain:
    """The block list of rank r: owned blocks, then halo copies.

    Attributes: ``glob`` (local -> global block index), ``nOwned``,
    ``grid`` (the local BlockGrid), ``owned`` (0/1 per local block),
    ``send[p]`` / ``recv[p]`` (local block indices whose interiors go to /
    come from rank p, in the order both sides use)."""

    def __init__(self, grid, rank_of, r, read_lists=None):
        rank_of = np.asarray(rank_of)
        nRank = int(rank_of.max()) + 1
        pos = morton_order(grid) - 1
        rd = reads(grid) if read_lists is None else read_lists

        def halo_of(q):
            mine = np.nonzero(rank_of == q)[0]
            need = set()
            for b in mine:
                need.update(int(x) for x in rd[b] if rank_of[x] != q)
            return sorted(mine, key=lambda b: pos[b]), sorted(need, key=lambda b: pos[b])

        owned, halo = halo_of(r)
        self.rank, self.nRank = r, nRank
        self.glob = np.array(owned + halo, dtype=np.int64)
        self.nOwned = len(owned)
        self.owned = np.zeros(len(self.glob), dtype=np.int32)
        self.owned[:self.nOwned] = 1
        local = {int(g): i for i, g in enumerate(self.glob)}
        self.grid = BlockGrid(grid.nDim, grid.nI, grid.nJ, grid.nK, grid.nRoot, grid.xyzMin, grid.xyzMax,
                              grid.typeBc, np.ascontiguousarray(grid.iLevelCoord[self.glob]))
        self.recv, self.send = {}, {}
        for p in range(nRank):
            if p == r:
                continue
            got = [local[b] for b in halo if rank_of[b] == p]
            if got:
                self.recv[p] = np.array(got, dtype=np.int64)
            _, halo_p = halo_of(p)
            give = [local[b] for b in halo_p if rank_of[b] == r]
            if give:
                self.send[p] = np.array(give, dtype=np.int64)

    def exchange(self, interiors, send_recv):
        """Refresh the halo copies: interiors is an array with the local
        blocks first (block index on axis 0); send_recv(peer, send_array,
        recv_shape) performs one pairwise exchange and returns the received
        array.  Pairs are visited in rank order so that blocking
        implementations do not deadlock."""
        for p in range(self.nRank):
            if p == self.rank or (p not in self.send and p not in self.recv):
                continue
            out = interiors[self.send[p]] if p in self.send else interiors[:0]
            n = len(self.recv.get(p, ()))
            got = send_recv(p, np.ascontiguousarray(out), (n,) + interiors.shape[1:])
            if n:
                interiors[self.recv[p]] = got


class GpuRank:
    """One rank of the partitioned explicit update on its GPU: an
    ExplicitSolver over the rank's block list (owned blocks, then halo
    copies) and, before every stage, the pairwise exchange of halo interiors
    through torch.distributed; the time step is an all_reduce MIN.  With
    the NCCL backend the buffers stay on the GPU; with gloo they go through
    host memory.  Every exchange completes on the host before the next
    stage is launched, so no kernel waits on another rank.

    The sequence per step is the one of the C ABI (include/bx200.h, "one
    rank of a partitioned grid"): bx_get_dtmin -> MIN -> bx_set_dtmin ->
    bx_set_global_timestep -> (exchange, bx_set_stage, bx_update_state_fast)
    per stage -> bx_end_step."""

    def __init__(self, grid, scheme, nRank, rank, device=0, weights=None):
        from .explicit import ExplicitSolver
        self.dom = RankDomain(grid, partition(grid, nRank, weights), rank)
        self.device = device
        self.x = ExplicitSolver(self.dom.grid, scheme, device=device, nOwned=self.dom.nOwned)
        self.nStage = scheme.nStage

    def set_state(self, State_VGB):
        """the global State_VGB (all blocks, reference layout): this rank's
        owned blocks and halo copies are taken from it"""
        self.x.set_state(np.ascontiguousarray(State_VGB[self.dom.glob]))

    def get_owned_state(self):
        """State_VGB of the owned blocks (their global indices: dom.glob[:nOwned])"""
        return self.x.get_state()[:self.dom.nOwned]

    def time(self):
        return self.x.time()

    def close(self):
        self.x.close()

    def _exchange(self, iStage):
        import torch
        import torch.distributed as dist
        nb = self.x.halo_bytes(iStage)
        dtype = torch.float32 if nb == 4 * 8 * self.x.grid.nI * self.x.grid.nJ * self.x.grid.nK else torch.float64
        per = nb // (4 if dtype == torch.float32 else 8)
        dev = torch.device("cuda", self.device)
        onGpu = dist.get_backend() == "nccl"
        d = self.dom
        for p in range(d.nRank):
            if p == d.rank or (p not in d.send and p not in d.recv):
                continue
            reqs = []
            if p in d.send:
                out = torch.empty(len(d.send[p]) * per, dtype=dtype, device=dev)
                self.x.halo_pack(iStage, d.send[p], out.data_ptr())
                reqs.append(dist.isend(out if onGpu else out.cpu(), dst=p))
            got = None
            if p in d.recv:
                got = torch.empty(len(d.recv[p]) * per, dtype=dtype, device=dev if onGpu else "cpu")
                reqs.append(dist.irecv(got, src=p))
            for r in reqs:
                r.wait()
            if got is not None:
                g = got if onGpu else got.to(dev)
                torch.cuda.current_stream(dev).synchronize()
                self.x.halo_unpack(iStage, d.recv[p], g.data_ptr())

    def advance(self, nStep=1, TimeSimulationLimit=-1.0):
        import torch
        import torch.distributed as dist
        multi = dist.is_available() and dist.is_initialized() and self.dom.nRank > 1
        for _ in range(nStep):
            if multi:
                onGpu = dist.get_backend() == "nccl"
                dt = torch.tensor([self.x.get_dtmin()], dtype=torch.float64,
                                  device=torch.device("cuda", self.device) if onGpu else "cpu")
                dist.all_reduce(dt, op=dist.ReduceOp.MIN)
                self.x.set_dtmin(float(dt.item()))
            self.x.set_global_timestep(TimeSimulationLimit)
            for s in range(1, self.nStage + 1):
                if multi:
                    self._exchange(s)
                self.x.set_stage(s)
                self.x.update_state_fast()
            self.x.end_step(TimeSimulationLimit)
