"""CPU restatement of the dynamic-AMR arithmetic, for the tests only (test
infrastructure, like the rest of this directory; nothing in batsrus_b200/
imports it).

* ``criteria``: amr_criteria (src/ModAMR.f90:388-723) for gradt,
  gradlogrho, gradlogp, gradp (calc_gradient3 on Cartesian blocks,
  src/ModCellGradient.f90:345-380), pjumpratio (src/ModAMR.f90:483-495) and
  -divu / -divudx (src/ModAMR.f90:476-497 with calc_divergence,
  src/ModCellGradient.f90:72-83; the reference scales by the cell diagonal
  only for a name 'divudx' that its case selector never passes),
  from a State_VGB whose ghost cells the oracle's exchange_messages filled.
  The operations and their order are those of the GPU kernel, so the values
  agree bit for bit except where log10 differs in the last place.
* ``remap_state``: the state on the new grid after a regrid: kept blocks
  copied, refined blocks by injection from the parent cell covering each new
  cell, coarsened blocks as the mean of the 2x2x2 child cells summed in the
  order (z, y, x) with x fastest, then times 1/8.  The refinement and
  coarsening operators of BATL (absent from the reference tree) are
  restated from Doc/Tex/grid.tex:50-66 ("standard multigrid-type restriction
  and prolongation"), with the first-order prolongation of #PROLONGATION
  (PARAM.XML:7929-7953).  Parity unpinned: no reference output covers it.
"""
import numpy as np

NG = 2


def block_geometry(grid):
    """cell sizes, volume and CellFace = CellVolume / CellSize per block, in
    the operation order of the C ABI's BlockGeom"""
    nc = (grid.nI, grid.nJ, grid.nK)
    lev = grid.iLevelCoord[:, 0]
    cs = np.empty((grid.nBlock, 3))
    for d in range(3):
        ext = grid.xyzMax[d] - grid.xyzMin[d]
        cs[:, d] = ext / (float(grid.nRoot[d]) * (2.0 ** lev)) / nc[d]
    vol = cs[:, 0] * cs[:, 1] * cs[:, 2]
    area = vol[:, None] / cs
    return cs, vol, area


def criteria(State_VGB, grid, names):
    """Crit_IB (nBlock, len(names)) from a ghost-filled State_VGB of shape
    (nBlock, nKg, nJg, nIg, 8)"""
    S = np.asarray(State_VGB, dtype=np.float64)
    rho, p = S[..., 0], S[..., 7]
    cs, vol, area = block_geometry(grid)
    vInvHalf = 0.5 / vol
    g = NG
    inner = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))

    def shifted(f, d, s):
        """f at the neighbour s (-1 or +1) along dimension d (0 = x, the last axis)"""
        sl = [slice(None), slice(g, -g), slice(g, -g), slice(g, -g)]
        ax = 3 - d
        sl[ax] = slice(g + s, -g + s if -g + s != 0 else None)
        return f[tuple(sl)]

    out = np.empty((grid.nBlock, len(names)))
    # (edge and corner ghost cells, which no criterion reads, may be zero)
    with np.errstate(divide="ignore", invalid="ignore"):
        _criteria(out, names, rho, p, area, vInvHalf, shifted, inner, grid, S, 0.5 / cs)
    return out


def _criteria(out, names, rho, p, area, vInvHalf, shifted, inner, grid, S, invHalf):
    for q, name in enumerate(names):
        name = name.lower()
        if name in ("-divu", "-divudx"):
            div = None
            for d in range(3):
                u = S[..., 1 + d] / rho
                t = invHalf[:, d][:, None, None, None] * (shifted(u, d, 1) - shifted(u, d, -1))
                div = t if div is None else div + t
            out[:, q] = (-div).reshape(grid.nBlock, -1).max(axis=1)
            continue
        if name == "pjumpratio":
            val = np.zeros(p[inner].shape)
            for d in range(3):
                pm, p0, pp = shifted(p, d, -1), p[inner], shifted(p, d, 1)
                mx = np.maximum(np.maximum(pm, p0), pp)
                mn = np.minimum(np.minimum(pm, p0), pp)
                val = np.maximum(val, mx / mn)
            out[:, q] = val.reshape(grid.nBlock, -1).max(axis=1)
            continue
        if name == "gradt":
            f = p / rho
        elif name == "gradlogrho":
            f = np.log10(rho)
        elif name == "gradlogp":
            f = np.log10(p)
        elif name == "gradp":
            f = p
        else:
            raise ValueError(name)
        g2 = None
        for d in range(3):
            a = area[:, d][:, None, None, None]
            gd = (a * (shifted(f, d, 1) - shifted(f, d, -1))) * vInvHalf[:, None, None, None]
            g2 = gd * gd if g2 is None else g2 + gd * gd
        out[:, q] = np.sqrt(g2.reshape(grid.nBlock, -1).max(axis=1))


def remap_state(State_VGB, remap, new_grid):
    """State_VGB on the new grid (ghost cells zero) from the old one and the
    iRemap_IB table of bx_regrid (1-based blocks)"""
    S = np.asarray(State_VGB, dtype=np.float64)
    g = NG
    A = S[:, g:-g, g:-g, g:-g, :]  # (nBlock, N, N, N, 8) as [k, j, i]
    N = A.shape[1]
    h = N // 2
    out = np.zeros(new_grid.state_shape_fortran())
    B = out[:, g:-g, g:-g, g:-g, :]
    R = np.asarray(remap)
    for b in range(new_grid.nBlock):
        op = R[b, 0]
        if op == 0:
            B[b] = A[R[b, 1] - 1]
        elif op == 1:
            o = R[b, 2]
            ox, oy, oz = o & 1, (o >> 1) & 1, o >> 2
            sub = A[R[b, 1] - 1][oz * h:(oz + 1) * h, oy * h:(oy + 1) * h, ox * h:(ox + 1) * h]
            B[b] = sub.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)
        else:
            for o in range(8):
                ox, oy, oz = o & 1, (o >> 1) & 1, o >> 2
                C = A[R[b, 1 + o] - 1]
                s = 0.0
                for kk in range(2):
                    for jj in range(2):
                        for ii in range(2):
                            s = s + C[kk::2, jj::2, ii::2]
                B[b][oz * h:(oz + 1) * h, oy * h:(oy + 1) * h, ox * h:(ox + 1) * h] = s * 0.125
    return out
