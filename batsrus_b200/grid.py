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
