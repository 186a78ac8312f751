"""Restart files of BATS-R-US (src/ModRestartFile.f90) for the GPU solver.

A restart directory holds:

* ``restart.H``: the header of ``write_restart_header``
  (src/ModRestartFile.f90:367-618), PARAM.in commands that a later session
  reads: ``#COMPONENT``, ``#PRECISION``, ``#EQUATION``, ``#RESTARTVARIABLES``,
  ``#CHECKGRIDSIZE``, ``#NEWRESTART``, ``#RESTARTINFILE``, ``#NSTEP``,
  ``#TIMESIMULATION``, ``#GRID``, ``#COORDSYSTEM``, ``#NORMALIZATION``.
* the block data, in one of the reference's two layouts:

  * ``one`` (``write_direct_restart_file``, :1040-1107): ``data.rst``, a
    direct-access file of one record per block.  A record is DtMax_B,
    CellSize_DB(3), Coord111_DB(3) and State_VGB(1:nVar,1:nI,1:nJ,1:nK)
    (variable fastest), all real(8) without record markers.  Block b sits
    at record iMortonNode_A(b).
  * ``block`` (``write_restart_file``, :795-833): ``blkNNNNN.rst`` per
    block, numbered by iMortonNode_A with at least 5 digits.  Each file has
    three Fortran sequential unformatted records, each with 4-byte length
    markers: (DtMax_B, tSimulation), (CellSize_DB, Coord111_DB), and the
    state variable by variable: (State_VGB(iVar,1:nI,1:nJ,1:nK), iVar=1,nVar).

  When the last step was implicit BDF2 (nStepPrev == nStep), the header has
  ``#NPREVIOUS`` (nStepPrev, DtPrev, :457-461) and each block also carries
  the previous step's state ImplOld_VCB: in ``one`` appended to the record
  variable by variable (State8_CV, :1084-1091, read at :1002-1010), in
  ``block`` as a fourth record (:828-829, read at :732-736).

* ``octree_blocks.txt``: the block tree.  BATL writes ``octree.rst`` with
  ``write_tree_file`` (srcBATL, absent from the reference tree), whose
  layout cannot be restated.  This file is a plain text list instead: the
  outer boundaries, then one line per block with its level and indices.  A
  BATS-R-US run restarting from this directory needs its own
  ``octree.rst``.  The block data files match the reference's layouts.

iMortonNode_A is BATL's space-filling order of the tree's leaves.  It is
restated here as the root blocks in Fortran order (x fastest), and within
each root block the z-order (x fastest, then y, then z) of its leaves.
"""
import os
import struct

import numpy as np

from .grid import NG, NVAR, BlockGrid, morton_key

NAME_HEADER = "restart.H"
NAME_DATA = "data.rst"
NAME_TREE = "octree_blocks.txt"
VAR_NAMES = "Rho Mx My Mz Bx By Bz P"


def morton_order(grid):
    """iMortonNode_A: the 1-based record index of every block"""
    lv = grid.iLevelCoord[:, 0]
    mx = int(lv.max())
    keys = []
    for b, (l, i, j, k) in enumerate(grid.iLevelCoord.tolist()):
        s = mx - l
        r = (i >> l, j >> l, k >> l)  # root block
        iRoot = r[0] + grid.nRoot[0] * (r[1] + grid.nRoot[1] * r[2])
        loc = ((i - (r[0] << l)) << s, (j - (r[1] << l)) << s, (k - (r[2] << l)) << s)
        keys.append((iRoot, morton_key(*loc), b))
    order = np.empty(grid.nBlock, dtype=np.int64)
    for rank, (_, _, b) in enumerate(sorted(keys)):
        order[b] = rank + 1
    return order


def block_geometry(grid):
    """CellSize_DB (nBlock, 3) and Coord111_DB, the centre of cell (1,1,1)"""
    nc = (grid.nI, grid.nJ, grid.nK)
    lev = grid.iLevelCoord[:, 0]
    cs = np.empty((grid.nBlock, 3))
    c111 = np.empty((grid.nBlock, 3))
    for d in range(3):
        ext = grid.xyzMax[d] - grid.xyzMin[d]
        if d < grid.nDim:
            bsize = ext / (float(grid.nRoot[d]) * (2.0 ** lev))
            cs[:, d] = bsize / nc[d]
            c111[:, d] = grid.xyzMin[d] + grid.iLevelCoord[:, 1 + d] * bsize + 0.5 * cs[:, d]
        else:
            cs[:, d] = ext
            c111[:, d] = 0.5 * (grid.xyzMin[d] + grid.xyzMax[d])
    return cs, c111


def _header(grid, tSimulation, nStep, typeRestart, dtPrev=None):
    tab = "\t\t"
    L = []

    def cmd(name, *vals):
        L.append(name)
        for v, n in vals:
            if isinstance(v, float):
                L.append("%22.15E%s%s" % (v, tab, n))
            elif isinstance(v, bool):
                L.append("%s%s%s" % ("T" if v else "F", tab + "\t", n))
            elif isinstance(v, int):
                L.append("%8d%s%s" % (v, tab, n))
            else:
                L.append("%s%s%s" % (v, tab + "\t", n))
        L.append("")
    cmd("#COMPONENT", ("GM", "NameComp"))
    cmd("#PRECISION", (8, "nByteReal"))
    cmd("#EQUATION", ("MHD", "NameEquation"), (NVAR, "nVar"))
    cmd("#RESTARTVARIABLES", (VAR_NAMES, "NameRestartVar"))
    cmd("#CHECKGRIDSIZE", (grid.nI, "nI"), (grid.nJ, "nJ"), (grid.nK, "nK"), (grid.nBlock, "MinBlockAll"))
    cmd("#NEWRESTART", (False, "DoRestartBFace"))
    cmd("#RESTARTINFILE", (typeRestart, "StringRestartInFile"))
    cmd("#NSTEP", (int(nStep), "nStep"))
    if dtPrev is not None:
        cmd("#NPREVIOUS", (int(nStep), "nPrev"), (float(dtPrev), "DtPrev"))
    cmd("#TIMESIMULATION", (float(tSimulation), "tSimulation"))
    cmd("#GRID", (int(grid.nRoot[0]), "nRootBlock1"), (int(grid.nRoot[1]), "nRootBlock2"),
        (int(grid.nRoot[2]), "nRootBlock3"),
        (float(grid.xyzMin[0]), "xMin"), (float(grid.xyzMax[0]), "xMax"),
        (float(grid.xyzMin[1]), "yMin"), (float(grid.xyzMax[1]), "yMax"),
        (float(grid.xyzMin[2]), "zMin"), (float(grid.xyzMax[2]), "zMax"))
    cmd("#COORDSYSTEM", ("GSM", "TypeCoordSystem"))
    cmd("#NORMALIZATION", ("NONE", "TypeNormalization"))
    return "\n".join(L) + "\n"


def write_restart_arrays(dirname, grid, State_VGB, tSimulation, nStep, DtMax_B, typeRestart="one",
                         ImplOld=None, DtPrev=None):
    """Write a restart directory from host arrays (State_VGB in the
    reference layout, shape grid.state_shape_fortran()).  ImplOld (nBlock,
    nK, nJ, nI, nVar) and DtPrev, given together, are the previous BDF2 step
    (#NPREVIOUS with nStepPrev = nStep)."""
    if (ImplOld is None) != (DtPrev is None):
        raise ValueError("ImplOld and DtPrev go together")
    if typeRestart not in ("one", "block"):
        raise ValueError("TypeRestartOutFile %r: 'one' and 'block' are written" % typeRestart)
    os.makedirs(dirname, exist_ok=True)
    S = np.asarray(State_VGB, dtype=np.float64)
    inner = S[grid.interior_slices()]  # (nBlock, nK, nJ, nI, nVar)
    cs, c111 = block_geometry(grid)
    order = morton_order(grid)
    dtB = np.asarray(DtMax_B, dtype=np.float64)
    with open(os.path.join(dirname, NAME_HEADER), "w") as f:
        f.write(_header(grid, tSimulation, nStep, typeRestart, DtPrev))
    with open(os.path.join(dirname, NAME_TREE), "w") as f:
        f.write("%d %d %d %d\n" % (grid.nDim, grid.nI, grid.nJ, grid.nK))
        f.write(" ".join(grid.typeBc) + "\n")
        f.write("%d\n" % grid.nBlock)
        for c in grid.iLevelCoord.tolist():
            f.write("%d %d %d %d\n" % tuple(c))
    nCellVar = NVAR * grid.nI * grid.nJ * grid.nK
    prev = None
    if ImplOld is not None:
        prev = np.asarray(ImplOld, dtype=np.float64).reshape(grid.nBlock, grid.nK, grid.nJ, grid.nI, NVAR)
    nExtra = 0 if prev is None else nCellVar
    if typeRestart == "one":
        rec = np.empty((grid.nBlock, 7 + nCellVar + nExtra))
        for b in range(grid.nBlock):
            r = order[b] - 1
            rec[r, 0] = dtB[b]
            rec[r, 1:4] = cs[b]
            rec[r, 4:7] = c111[b]
            # (nVar, nI, nJ, nK) with the variable fastest = [k][j][i][v] in C order
            rec[r, 7:7 + nCellVar] = inner[b].reshape(-1)
            if prev is not None:  # State8_CV: the variable slowest
                rec[r, 7 + nCellVar:] = np.moveaxis(prev[b], -1, 0).reshape(-1)
        rec.tofile(os.path.join(dirname, NAME_DATA))
        return
    for b in range(grid.nBlock):
        nd = max(5, int(1 + np.log10(float(order[b]))))
        name = os.path.join(dirname, "blk%0*d.rst" % (nd, order[b]))
        with open(name, "wb") as f:
            payloads = [np.array([dtB[b], tSimulation]), np.concatenate([cs[b], c111[b]]),
                        np.ascontiguousarray(np.moveaxis(inner[b], -1, 0)).reshape(-1)]
            if prev is not None:
                payloads.append(np.ascontiguousarray(np.moveaxis(prev[b], -1, 0)).reshape(-1))
            for payload in payloads:
                raw = payload.astype("<f8").tobytes()
                f.write(struct.pack("<i", len(raw)) + raw + struct.pack("<i", len(raw)))


def read_header(dirname):
    """the commands of restart.H: {name: [values]}"""
    out, cur = {}, None
    with open(os.path.join(dirname, NAME_HEADER)) as f:
        for line in f:
            s = line.strip()
            if not s:
                cur = None
                continue
            if s.startswith("#"):
                cur = s.split()[0]
                out[cur] = []
            elif cur is not None:
                out[cur].append(s.split("\t")[0].strip())
    return out


def read_restart(dirname):
    """(grid, State_VGB, tSimulation, nStep, DtMax_B) of a restart directory"""
    return _read(dirname)[:5]


def read_restart_previous(dirname):
    """(DtPrev, ImplOld (nBlock, nK, nJ, nI, nVar)) of a restart written
    after a BDF2 step (#NPREVIOUS), else None"""
    return _read(dirname)[5]


def _read(dirname):
    h = read_header(dirname)
    if int(h["#PRECISION"][0]) != 8 or int(h["#EQUATION"][1]) != NVAR:
        raise ValueError("restart with nByteReal %s and nVar %s: 8 and %d are read" %
                         (h["#PRECISION"][0], h["#EQUATION"][1], NVAR))
    nI, nJ, nK, nBlock = (int(v) for v in h["#CHECKGRIDSIZE"])
    g = [float(v) for v in h["#GRID"][3:9]]
    nRoot = tuple(int(v) for v in h["#GRID"][:3])
    with open(os.path.join(dirname, NAME_TREE)) as f:
        nDim = int(f.readline().split()[0])
        typeBc = tuple(f.readline().split())
        n = int(f.readline())
        lc = np.array([[int(v) for v in f.readline().split()] for _ in range(n)], dtype=np.int32)
    if n != nBlock:
        raise ValueError("%d blocks in the tree file, %d in restart.H" % (n, nBlock))
    grid = BlockGrid(nDim, nI, nJ, nK, nRoot, (g[0], g[2], g[4]), (g[1], g[3], g[5]), typeBc, lc)
    tSimulation = float(h["#TIMESIMULATION"][0])
    nStep = int(h["#NSTEP"][0])
    typeRestart = h["#RESTARTINFILE"][0]
    order = morton_order(grid)
    nCellVar = NVAR * nI * nJ * nK
    hasPrev = "#NPREVIOUS" in h and int(h["#NPREVIOUS"][0]) == nStep
    nExtra = nCellVar if hasPrev else 0
    prev = np.empty((nBlock, nK, nJ, nI, NVAR)) if hasPrev else None
    S = np.zeros(grid.state_shape_fortran())
    inner = np.empty((nBlock, nK, nJ, nI, NVAR))
    dtB = np.empty(nBlock)
    if typeRestart == "one":
        rec = np.fromfile(os.path.join(dirname, NAME_DATA), dtype="<f8")
        nRec = 7 + nCellVar + nExtra
        if rec.size != nBlock * nRec:
            raise ValueError("data.rst holds %d reals, %d expected" % (rec.size, nBlock * nRec))
        rec = rec.reshape(nBlock, nRec)
        for b in range(nBlock):
            r = rec[order[b] - 1]
            dtB[b] = r[0]
            inner[b] = r[7:7 + nCellVar].reshape(nK, nJ, nI, NVAR)
            if hasPrev:
                prev[b] = np.moveaxis(r[7 + nCellVar:].reshape(NVAR, nK, nJ, nI), 0, -1)
    elif typeRestart == "block":
        for b in range(nBlock):
            nd = max(5, int(1 + np.log10(float(order[b]))))
            with open(os.path.join(dirname, "blk%0*d.rst" % (nd, order[b])), "rb") as f:
                recs = []
                for _ in range(4 if hasPrev else 3):
                    m = struct.unpack("<i", f.read(4))[0]
                    recs.append(np.frombuffer(f.read(m), dtype="<f8"))
                    if struct.unpack("<i", f.read(4))[0] != m:
                        raise ValueError("record markers of block file %d differ" % order[b])
            dtB[b] = recs[0][0]
            inner[b] = np.moveaxis(recs[2].reshape(NVAR, nK, nJ, nI), 0, -1)
            if hasPrev:
                prev[b] = np.moveaxis(recs[3].reshape(NVAR, nK, nJ, nI), 0, -1)
    else:
        raise ValueError("TypeRestartInFile %r: 'one' and 'block' are read" % typeRestart)
    S[grid.interior_slices()] = inner
    prevOut = (float(h["#NPREVIOUS"][1]), prev) if hasPrev else None
    return grid, S, tSimulation, nStep, dtB, prevOut


def write_restart(dirname, solver, typeRestart="one"):
    """write_restart_files for an ExplicitSolver: its state, time, step and
    DtMax_B"""
    t, _, n = solver.time()
    write_restart_arrays(dirname, solver.grid, solver.get_state(), t, n, solver.block_dt(), typeRestart)


def restart_solver(dirname, scheme, device=0):
    """a new ExplicitSolver from a restart directory (read_restart_files):
    the grid, the state, the time and step, and DtMax_B for the next step"""
    from .explicit import ExplicitSolver
    grid, S, t, n, dtB = read_restart(dirname)
    x = ExplicitSolver(grid, scheme, device=device)
    x.set_state(S)
    x.set_time(t, n)
    if n > 0:
        x.set_block_dt(dtB)
    return x
