"""Block grid description (host side).

Mirrors the part of BATL (srcBATL, absent from the reference tree) that the
hot path needs: a list of nI x nJ x nK blocks, each identified by its
refinement level and integer block index at that level, on a Cartesian
domain with float or periodic outer boundaries.  Ghost layers are nG = 2 as
in the reference's -ng=2 builds.

The Fortran state layout State_VGB(nVar, MinI:MaxI, MinJ:MaxJ, MinK:MaxK,
nBlock) (src/ModAdvance.f90:296) maps to the C-order numpy shape
``(nBlock, nKg, nJg, nIg, nVar)``.
"""
from dataclasses import dataclass, field

import numpy as np

NVAR = 8
NG = 2


def morton_key(ix, iy, iz):
    """Interleave the bits of three block indices (z-order curve)."""
    key = 0
    for bit in range(21):
        key |= ((ix >> bit) & 1) << (3 * bit)
        key |= ((iy >> bit) & 1) << (3 * bit + 1)
        key |= ((iz >> bit) & 1) << (3 * bit + 2)
    return key


@dataclass
class BlockGrid:
    nDim: int
    nI: int
    nJ: int
    nK: int
    nRoot: tuple
    xyzMin: tuple
    xyzMax: tuple
    typeBc: tuple  # 6 sides: 'float' | 'periodic'
    iLevelCoord: np.ndarray = field(default=None)  # (nBlock, 4): level, ix, iy, iz

    @classmethod
    def uniform(cls, nDim, nCellBlock, nRoot, xyzMin, xyzMax, typeBc, level=0,
                order="x"):
        """All blocks at one level.  ``order`` 'x' numbers the blocks with x
        fastest (BATL root-block order); 'morton' uses the z-order curve."""
        nI, nJ, nK = nCellBlock
        nb = [nRoot[d] << level if d < nDim else 1 for d in range(3)]
        coords = [(level, i, j, k) for k in range(nb[2]) for j in range(nb[1])
                  for i in range(nb[0])]
        if order == "morton":
            coords.sort(key=lambda c: morton_key(c[1], c[2], c[3]))
        return cls(nDim, nI, nJ, nK, tuple(nRoot), tuple(map(float, xyzMin)),
                   tuple(map(float, xyzMax)), tuple(typeBc),
                   np.array(coords, dtype=np.int32))

    # -- sizes ---------------------------------------------------------------
    @property
    def nBlock(self):
        return len(self.iLevelCoord)

    @property
    def nCellBlock(self):
        return self.nI * self.nJ * self.nK

    @property
    def nCell(self):
        return self.nBlock * self.nCellBlock

    @property
    def ghost_extent(self):
        nIg = self.nI + 2 * NG
        nJg = self.nJ + 2 * NG if self.nDim > 1 else 1
        nKg = self.nK + 2 * NG if self.nDim > 2 else 1
        return nIg, nJg, nKg

    def state_shape_fortran(self):
        nIg, nJg, nKg = self.ghost_extent
        return (self.nBlock, nKg, nJg, nIg, NVAR)

    def interior_slices(self):
        """Index of the physical cells in the (nBlock,nKg,nJg,nIg,nVar) array."""
        gi = NG
        gj = NG if self.nDim > 1 else 0
        gk = NG if self.nDim > 2 else 0
        return (slice(None), slice(gk, gk + self.nK), slice(gj, gj + self.nJ),
                slice(gi, gi + self.nI), slice(None))

    # -- geometry ------------------------------------------------------------
    def block_geometry(self):
        """Block corner (nBlock,3) and cell size (nBlock,3); ignored
        dimensions span the whole domain as in BATL."""
        lev = self.iLevelCoord[:, 0]
        corner = np.zeros((self.nBlock, 3))
        size = np.zeros((self.nBlock, 3))
        ncell = (self.nI, self.nJ, self.nK)
        for d in range(3):
            ext = self.xyzMax[d] - self.xyzMin[d]
            if d < self.nDim:
                bsize = ext / (self.nRoot[d] * (2.0 ** lev))
                corner[:, d] = self.xyzMin[d] + self.iLevelCoord[:, 1 + d] * bsize
                size[:, d] = bsize / ncell[d]
            else:
                corner[:, d] = self.xyzMin[d]
                size[:, d] = ext
        return corner, size

    def cell_centers(self, with_ghost=True):
        """Cell-centre coordinates, shape (nBlock, nKg, nJg, nIg, 3)
        (Xyz_DGB = corner + (i - 1/2) * CellSize)."""
        corner, size = self.block_geometry()
        nIg, nJg, nKg = self.ghost_extent
        gi = NG
        gj = NG if self.nDim > 1 else 0
        gk = NG if self.nDim > 2 else 0
        i = np.arange(nIg) - gi + 0.5
        j = np.arange(nJg) - gj + 0.5
        k = np.arange(nKg) - gk + 0.5
        xyz = np.empty((self.nBlock, nKg, nJg, nIg, 3))
        xyz[..., 0] = corner[:, None, None, None, 0] + i[None, None, None, :] * size[:, None, None, None, 0]
        xyz[..., 1] = corner[:, None, None, None, 1] + j[None, None, :, None] * size[:, None, None, None, 1]
        xyz[..., 2] = corner[:, None, None, None, 2] + k[None, :, None, None] * size[:, None, None, None, 2]
        if self.nDim < 2:
            xyz[..., 1] = 0.5 * (self.xyzMin[1] + self.xyzMax[1])
        if self.nDim < 3:
            xyz[..., 2] = 0.5 * (self.xyzMin[2] + self.xyzMax[2])
        if not with_ghost:
            xyz = xyz[self.interior_slices()[:4]]
        return xyz

    # -- static block-adaptive grids -------------------------------------------
    @classmethod
    def adaptive(cls, nDim, nCellBlock, nRoot, xyzMin, xyzMax, typeBc, maxLevel, refine):
        """A static refined grid: starting from the root blocks, every block
        of level L < maxLevel for which ``refine(level, ix, iy, iz)`` is true
        is split into 2^nDim children; then blocks are split until
        neighbouring blocks (across faces, edges and corners) differ by at
        most one level, as BATL keeps its tree.  Blocks are numbered along
        the Morton curve of the finest level (the order of BATL's
        space-filling curve over the tree)."""
        nb0 = [nRoot[d] if d < nDim else 1 for d in range(3)]
        leaves = {(0, i, j, k) for k in range(nb0[2]) for j in range(nb0[1]) for i in range(nb0[0])}
        per = [typeBc[2 * d] == "periodic" for d in range(3)]
        kids = [(a, b, c) for c in range(2 if nDim > 2 else 1) for b in range(2 if nDim > 1 else 1) for a in range(2)]

        def split(key):
            leaves.discard(key)
            lv, i, j, k = key
            for a, b, c in kids:
                leaves.add((lv + 1, 2 * i + a, 2 * j + b, 2 * k + c))

        def leaf_at(lv, c):
            """leaf covering the level-lv block index c (wrapped), or None"""
            n = [nb0[d] << lv if d < nDim else 1 for d in range(3)]
            c = list(c)
            for d in range(3):
                if c[d] < 0 or c[d] >= n[d]:
                    if d >= nDim or not per[d]:
                        return None
                    c[d] %= n[d]
            for l2 in range(lv, -1, -1):
                s = lv - l2
                key = (l2, c[0] >> s, c[1] >> s, c[2] >> s) if nDim == 3 else \
                    (l2, c[0] >> s, (c[1] >> s) if nDim > 1 else 0, 0)
                if key in leaves:
                    return key
            return None

        offs = [(a, b, c) for c in ((-1, 0, 1) if nDim > 2 else (0,)) for b in ((-1, 0, 1) if nDim > 1 else (0,))
                for a in (-1, 0, 1) if (a, b, c) != (0, 0, 0)]
        for lv in range(maxLevel):
            for key in sorted(k for k in leaves if k[0] == lv):
                if refine(*key):
                    split(key)
            changed = True
            while changed:
                changed = False
                for key in sorted(leaves):
                    if key not in leaves:
                        continue
                    l0, i, j, k = key
                    for a, b, c in offs:
                        nk = leaf_at(l0, (i + a, j + b, k + c))
                        if nk is not None and nk[0] < l0 - 1:
                            split(nk)
                            changed = True
        mx = max(k[0] for k in leaves)

        def order_key(key):
            s = mx - key[0]
            return (morton_key(key[1] << s, key[2] << s, key[3] << s), key[0])

        coords = sorted(leaves, key=order_key)
        return cls(nDim, nCellBlock[0], nCellBlock[1], nCellBlock[2], tuple(nRoot), tuple(map(float, xyzMin)),
                   tuple(map(float, xyzMax)), tuple(typeBc), np.array(coords, dtype=np.int32))

    def neighbors(self):
        """DiLevel_EB and jBlock_IEB of ModParallel (0-based block indices):
        for each block and side (x-, x+, y-, y+, z-, z+) the level
        difference to the neighbour (0 same level, +1 coarser, -1 finer,
        -100 (BATL Unset_) at a float boundary or an ignored dimension) and the
        neighbour blocks: one for 0 and +1; for -1 the 2^(nDim-1) finer
        blocks touching the face, ordered by their two transverse indices
        (first transverse direction fastest)."""
        index = {tuple(int(v) for v in c): b for b, c in enumerate(self.iLevelCoord)}
        nb0 = [self.nRoot[d] if d < self.nDim else 1 for d in range(3)]
        per = [self.typeBc[2 * d] == "periodic" for d in range(3)]
        dil = np.zeros((self.nBlock, 6), dtype=np.int32)
        jb = -np.ones((self.nBlock, 6, 4), dtype=np.int32)
        for b, (lv, i, j, k) in enumerate(self.iLevelCoord.tolist()):
            for d in range(3):
                for side in range(2):
                    s = 2 * d + side
                    if d >= self.nDim:
                        dil[b, s] = -100
                        continue
                    c = [i, j, k]
                    c[d] += 1 if side else -1
                    n = nb0[d] << lv
                    if c[d] < 0 or c[d] >= n:
                        if not per[d]:
                            dil[b, s] = -100
                            continue
                        c[d] %= n
                    if (lv, *c) in index:
                        dil[b, s] = 0
                        jb[b, s, 0] = index[(lv, *c)]
                    elif lv > 0 and (lv - 1, c[0] >> 1, c[1] >> 1, c[2] >> 1) in index:
                        dil[b, s] = 1
                        jb[b, s, 0] = index[(lv - 1, c[0] >> 1, c[1] >> 1, c[2] >> 1)]
                    else:
                        dil[b, s] = -1
                        t = [e for e in range(3) if e != d and e < self.nDim]
                        m = 0
                        for q1 in range(2 if len(t) > 1 else 1):
                            for q0 in range(2 if len(t) > 0 else 1):
                                f = [2 * c[0], 2 * c[1] if self.nDim > 1 else 0, 2 * c[2] if self.nDim > 2 else 0]
                                f[d] += 0 if side else 1  # the child layer touching the face
                                if len(t) > 0:
                                    f[t[0]] += q0
                                if len(t) > 1:
                                    f[t[1]] += q1
                                key = (lv + 1, *f)
                                if key not in index:
                                    raise ValueError("block %d side %d: unbalanced tree" % (b, s))
                                jb[b, s, m] = index[key]
                                m += 1
        return dil, jb
