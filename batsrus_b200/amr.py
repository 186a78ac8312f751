"""Dynamic AMR on the host: the refinement decisions of BATL's
``set_amr_criteria`` / ``regrid_batl`` (srcBATL, absent from the reference
tree) restated from their documented behaviour, and the remap table with
which ``bx_regrid`` moves the state onto the new grid.

Documented behaviour followed here (PARAM.XML:6658-6910, ``#AMRLEVELS``,
``#AMR``, ``#DOAMR``, ``#AMRCRITERIA``; Doc/Tex/grid.tex:50-110):

* Refinement splits a block into 2^nDim children, and coarsening merges
  2^nDim siblings into their parent.
* A block is refined if ANY criterion exceeds its RefineLimit, and its level
  is below MaxBlockLevel.
* A block is coarsened if ALL criteria are below their CoarsenLimit, its level
  is above MinBlockLevel and below MaxBlockLevel, all its siblings are leaves
  that may be coarsened as well, and no block next to their parent is finer
  than the siblings.  The check is made on the tree after the refinements, so
  a block refined in this pass keeps its neighbours.
* Neighbouring blocks (across faces, edges and corners) differ by at most one
  level: a refinement splits coarser neighbours until this holds, as
  ``BlockGrid.adaptive`` builds its trees.
* The number of blocks does not exceed MaxTotalBlocks.  Refinements are taken
  in decreasing order of the largest criterion-to-RefineLimit ratio, each
  with the splits of its neighbours, and the first one that would pass the
  limit ends the refinements.

The criteria themselves are computed on the GPU (``bx_amr_criteria``): the
maximum over a block's cells of ``gradt``, ``gradlogrho``, ``gradlogp``,
``gradp``, ``pjumpratio`` or ``-divu`` (src/ModAMR.f90:388-723), in normalised units
(the reference multiplies some by No2Io_V, which is 1 for normalised I/O
units).
"""
from dataclasses import dataclass, field

import numpy as np

from .grid import BlockGrid, morton_key

REMAP_INTS = 10
COPY, PROLONG, RESTRICT = 0, 1, 2


@dataclass
class AmrCriterion:
    """One #AMRCRITERIA entry: TypeRefine, CoarsenLimit, RefineLimit."""
    name: str
    coarsenLimit: float
    refineLimit: float


@dataclass
class AmrParams:
    """#DOAMR / #AMR (DnRefine, MaxTotalBlocks), #AMRCRITERIA, #AMRLEVELS."""
    dnRefine: int = -1
    criteria: list = field(default_factory=list)
    minBlockLevel: int = 0
    maxBlockLevel: int = 99
    maxTotalBlocks: int = 99999


def read_amr_params(info):
    """AmrParams from the commands that ``param.apply_commands`` left in its
    info dictionary (the last occurrence of each command wins)."""
    p = AmrParams()
    if "#DOAMR" in info:
        v = info["#DOAMR"][-1]
        p.dnRefine = int(v[1]) if bool(v[0]) else -1
    if "#AMR" in info:
        v = info["#AMR"][-1]
        p.dnRefine = int(v[0])
        if p.dnRefine > 0 and len(v) > 4 and bool(v[1]):
            p.maxTotalBlocks = int(v[4])
    if "#AMRCRITERIA" in info:
        v = info["#AMRCRITERIA"][-1]
        n = int(v[0])
        p.criteria = [AmrCriterion(str(v[1 + 3 * q]).lower(), float(v[2 + 3 * q]), float(v[3 + 3 * q]))
                      for q in range(n)]
    if "#AMRLEVELS" in info:
        v = info["#AMRLEVELS"][-1]
        p.minBlockLevel, p.maxBlockLevel = int(v[0]), int(v[1])
    return p


class _Tree:
    """The leaves of a block tree, with the neighbour searches of the regrid."""

    def __init__(self, grid):
        self.nDim = grid.nDim
        self.nb0 = [grid.nRoot[d] if d < grid.nDim else 1 for d in range(3)]
        self.per = [grid.typeBc[2 * d] == "periodic" for d in range(3)]
        self.leaves = {tuple(int(v) for v in c) for c in grid.iLevelCoord}
        self.kids = [(a, b, c) for c in range(2 if self.nDim > 2 else 1)
                     for b in range(2 if self.nDim > 1 else 1) for a in range(2)]
        rng = (-1, 0, 1)
        self.offs = [(a, b, c) for c in (rng if self.nDim > 2 else (0,))
                     for b in (rng if self.nDim > 1 else (0,)) for a in rng if (a, b, c) != (0, 0, 0)]

    def wrap(self, lv, c):
        """level-lv block index c wrapped at periodic sides, or None outside"""
        c = list(c)
        for d in range(3):
            n = self.nb0[d] << lv if d < self.nDim else 1
            if c[d] < 0 or c[d] >= n:
                if d >= self.nDim or not self.per[d]:
                    return None
                c[d] %= n
        return c

    def leaf_at(self, lv, c):
        """the leaf at level lv or coarser covering position c (wrapped);
        None outside the domain or where finer leaves cover it"""
        c = self.wrap(lv, c)
        if c is None:
            return None
        for l2 in range(lv, -1, -1):
            s = lv - l2
            key = (l2, c[0] >> s, c[1] >> s, c[2] >> s)
            if key in self.leaves:
                return key
        return None

    def children(self, key):
        lv, i, j, k = key
        return [(lv + 1, 2 * i + a, 2 * j + b, 2 * k + c) for a, b, c in self.kids]

    def split(self, key, journal):
        """split key, then split coarser neighbours until the levels of all
        neighbouring leaves differ by at most one"""
        work = [key]
        while work:
            q = work.pop()
            if q not in self.leaves:
                continue
            self.leaves.remove(q)
            ch = self.children(q)
            self.leaves.update(ch)
            journal.append(q)
            for c in ch:
                for a, b, e in self.offs:
                    nk = self.leaf_at(c[0], (c[1] + a, c[2] + b, c[3] + e))
                    if nk is not None and nk[0] < c[0] - 1:
                        work.append(nk)

    def unsplit(self, journal):
        for q in reversed(journal):
            for c in self.children(q):
                self.leaves.discard(c)
            self.leaves.add(q)

    def finer_next_to(self, parent):
        """is any leaf next to the region of ``parent`` finer than its
        children?"""
        lv = parent[0] + 1
        inside = set(self.children(parent))
        for c in inside:
            for a, b, e in self.offs:
                pos = (c[1] + a, c[2] + b, c[3] + e)
                w = self.wrap(lv, pos)
                if w is None or (lv, *w) in inside:
                    continue
                if self.leaf_at(lv, pos) is None:  # inside the domain, covered by finer leaves
                    return True
        return False


def order_leaves(leaves):
    """Blocks along the Morton curve of the finest level (BlockGrid.adaptive)."""
    mx = max(k[0] for k in leaves)

    def key(c):
        s = mx - c[0]
        return (morton_key(c[1] << s, c[2] << s, c[3] << s), c[0])
    return sorted(leaves, key=key)


def regrid(grid, crit, params):
    """New grid and remap table from the per-block criteria ``crit``
    (nBlock x nCrit, as ``bx_amr_criteria`` returns them).  Returns
    (new_grid, remap, changed); ``remap`` is the iRemap_IB array of
    bx_regrid (1-based blocks)."""
    crit = np.asarray(crit, dtype=np.float64).reshape(grid.nBlock, -1)
    cr = params.criteria
    if crit.shape[1] != len(cr):
        raise ValueError("%d criteria values per block, %d criteria" % (crit.shape[1], len(cr)))
    keys = [tuple(int(v) for v in c) for c in grid.iLevelCoord]
    lev = grid.iLevelCoord[:, 0]
    refL = np.array([c.refineLimit for c in cr])
    coaL = np.array([c.coarsenLimit for c in cr])
    want_ref = (crit > refL).any(axis=1) & (lev < params.maxBlockLevel)
    want_coa = (crit < coaL).all(axis=1) & (lev > params.minBlockLevel) & (lev < params.maxBlockLevel) & ~want_ref
    tree = _Tree(grid)
    # refinements, largest criterion ratio first, within MaxTotalBlocks
    ratio = (crit / np.where(refL != 0, refL, 1.0)).max(axis=1)
    for b in sorted(np.flatnonzero(want_ref), key=lambda b: (-ratio[b], b)):
        if keys[b] not in tree.leaves:
            continue  # already split as a neighbour of an earlier refinement
        journal = []
        tree.split(keys[b], journal)
        if len(tree.leaves) > params.maxTotalBlocks:
            tree.unsplit(journal)
            break
    # coarsening of whole sibling groups
    groups = {}
    for b in np.flatnonzero(want_coa):
        k = keys[b]
        if k in tree.leaves:
            groups.setdefault((k[0] - 1, k[1] >> 1, k[2] >> 1, k[3] >> 1), []).append(k)
    nKid = len(tree.kids)
    merge = [p for p, ch in sorted(groups.items())
             if len(ch) == nKid and all(c in tree.leaves for c in tree.children(p)) and not tree.finer_next_to(p)]
    for p in merge:
        for c in tree.children(p):
            tree.leaves.discard(c)
        tree.leaves.add(p)
    coords = order_leaves(tree.leaves)
    new = BlockGrid(grid.nDim, grid.nI, grid.nJ, grid.nK, grid.nRoot, grid.xyzMin, grid.xyzMax, grid.typeBc,
                    np.array(coords, dtype=np.int32))
    changed = len(coords) != len(keys) or any(a != b for a, b in zip(coords, keys))
    return new, remap_table(grid, new), changed


def plan_native(grid, crit, params):
    """the same decisions made by the library (bx_amr_plan, host code, no
    device needed): (new_grid, remap, changed)"""
    import ctypes
    from . import capi
    L = capi.load()
    crit = np.ascontiguousarray(crit, dtype=np.float64).reshape(grid.nBlock, -1)
    gd = capi.grid_desc(grid)
    cp = capi.amr_params(params)
    ip = ctypes.POINTER(ctypes.c_int)
    nMax = max(8 * grid.nBlock, 64)
    lc = np.empty((nMax, 4), dtype=np.int32)
    R = np.empty((nMax, REMAP_INTS), dtype=np.int32)
    n, ch = ctypes.c_int(), ctypes.c_int()
    capi.check(L.bx_amr_plan(ctypes.byref(gd), ctypes.byref(cp), capi.dptr(crit), nMax, ctypes.byref(n),
                             lc.ctypes.data_as(ip), R.ctypes.data_as(ip), ctypes.byref(ch)))
    new = BlockGrid(grid.nDim, grid.nI, grid.nJ, grid.nK, grid.nRoot, grid.xyzMin, grid.xyzMax, grid.typeBc,
                    lc[:n.value].copy())
    return new, R[:n.value].copy(), bool(ch.value)


def remap_table(old, new):
    """iRemap_IB of bx_regrid: per new block the operation and the old
    blocks (1-based) it is made from."""
    index = {tuple(int(v) for v in c): b for b, c in enumerate(old.iLevelCoord)}
    R = np.zeros((new.nBlock, REMAP_INTS), dtype=np.int32)
    for b, c in enumerate(new.iLevelCoord.tolist()):
        key = tuple(c)
        lv, i, j, k = key
        if key in index:
            R[b, 0], R[b, 1] = COPY, index[key] + 1
            continue
        parent = (lv - 1, i >> 1, j >> 1, k >> 1)
        if lv > 0 and parent in index:
            R[b, 0], R[b, 1] = PROLONG, index[parent] + 1
            R[b, 2] = (i & 1) + 2 * (j & 1) + 4 * (k & 1)
            continue
        R[b, 0] = RESTRICT
        for o in range(8):
            ch = (lv + 1, 2 * i + (o & 1), 2 * j + ((o >> 1) & 1), 2 * k + (o >> 2))
            if ch not in index:
                raise ValueError("new block %s: neither kept, refined once nor coarsened once" % (key,))
            R[b, 1 + o] = index[ch] + 1
    return R


def is_balanced(grid):
    """do all neighbouring leaves (faces, edges, corners) differ by at most
    one level?"""
    t = _Tree(grid)
    for key in t.leaves:
        for a, b, e in t.offs:
            nk = t.leaf_at(key[0], (key[1] + a, key[2] + b, key[3] + e))
            if nk is not None and nk[0] < key[0] - 1:
                return False
    return True
