"""Restart files (batsrus_b200.restart, src/ModRestartFile.f90): the 'one'
direct-access and 'block' sequential layouts round-trip grid, state, time,
step and DtMax_B; records sit at the space-filling order of the tree;
record contents and Fortran record markers are as the reference writes
them.  CPU only."""
import os
import struct

import numpy as np
import pytest

from batsrus_b200 import configs, restart
from batsrus_b200.grid import BlockGrid


def case():
    g = configs.amr_blast(nRoot=2, maxLevel=2, with_state=False)[0]
    rng = np.random.default_rng(5)
    S = np.zeros(g.state_shape_fortran())
    S[g.interior_slices()] = rng.normal(size=S[g.interior_slices()].shape)
    return g, S, 0.125, 17, rng.uniform(1e-3, 2e-3, size=g.nBlock)


@pytest.mark.parametrize("kind", ["one", "block"])
def test_round_trip(tmp_path, kind):
    g, S, t, n, dtB = case()
    restart.write_restart_arrays(str(tmp_path), g, S, t, n, dtB, kind)
    g2, S2, t2, n2, dtB2 = restart.read_restart(str(tmp_path))
    assert np.array_equal(g2.iLevelCoord, g.iLevelCoord) and g2.typeBc == g.typeBc and g2.nRoot == g.nRoot
    assert g2.xyzMin == g.xyzMin and g2.xyzMax == g.xyzMax
    assert np.array_equal(S2[g.interior_slices()], S[g.interior_slices()])
    assert (t2, n2) == (t, n) and np.array_equal(dtB2, dtB)
    h = restart.read_header(str(tmp_path))
    assert h["#RESTARTINFILE"] == [kind] and h["#CHECKGRIDSIZE"] == ["8", "8", "8", str(g.nBlock)]


def test_one_file_records(tmp_path):
    g, S, t, n, dtB = case()
    restart.write_restart_arrays(str(tmp_path), g, S, t, n, dtB, "one")
    raw = np.fromfile(os.path.join(str(tmp_path), "data.rst"), dtype="<f8")
    nRec = 7 + 8 * 512
    assert raw.size == g.nBlock * nRec  # direct access: no record markers
    order = restart.morton_order(g)
    cs, c111 = restart.block_geometry(g)
    for b in (0, g.nBlock // 2, g.nBlock - 1):
        r = raw[(order[b] - 1) * nRec:order[b] * nRec]
        assert r[0] == dtB[b] and np.array_equal(r[1:4], cs[b]) and np.array_equal(r[4:7], c111[b])
        inner = S[g.interior_slices()][b]  # [k][j][i][v]
        # State_VGB(iVar, i, j, k): variable fastest, then i, j, k
        i, j, k, v = 3, 1, 6, 4
        assert r[7 + v + 8 * (i + 8 * (j + 8 * k))] == inner[k, j, i, v]


def test_block_files_have_fortran_records(tmp_path):
    g, S, t, n, dtB = case()
    restart.write_restart_arrays(str(tmp_path), g, S, t, n, dtB, "block")
    files = sorted(f for f in os.listdir(str(tmp_path)) if f.startswith("blk"))
    assert len(files) == g.nBlock and files[0] == "blk00001.rst"
    order = restart.morton_order(g)
    b = 7
    with open(os.path.join(str(tmp_path), "blk%05d.rst" % order[b]), "rb") as f:
        data = f.read()
    sizes = [16, 48, 8 * 512 * 8]
    pos = 0
    recs = []
    for m in sizes:
        assert struct.unpack("<i", data[pos:pos + 4])[0] == m
        recs.append(np.frombuffer(data[pos + 4:pos + 4 + m], dtype="<f8"))
        assert struct.unpack("<i", data[pos + 4 + m:pos + 8 + m])[0] == m
        pos += m + 8
    assert pos == len(data)
    assert recs[0][0] == dtB[b] and recs[0][1] == t
    # (State_VGB(iVar,1:nI,1:nJ,1:nK), iVar=1,nVar): variable by variable
    inner = S[g.interior_slices()][b]
    assert recs[2][3 * 512 + 2 + 8 * (5 + 8 * 1)] == inner[1, 5, 2, 3]


def test_morton_order_is_root_major_z_order():
    g = BlockGrid.uniform(3, (8, 8, 8), (2, 1, 1), (0, 0, 0), (2, 1, 1), ("float",) * 6, level=1)
    order = restart.morton_order(g)
    assert sorted(order) == list(range(1, g.nBlock + 1))
    lc = g.iLevelCoord
    # every block of root 0 (ix < 2) comes before those of root 1
    assert order[lc[:, 1] < 2].max() < order[lc[:, 1] >= 2].min()
    # inside a root: x fastest, then y, then z
    first = {tuple(c[1:]): o for c, o in zip(lc.tolist(), order) if c[1] < 2}
    assert [first[(0, 0, 0)], first[(1, 0, 0)], first[(0, 1, 0)], first[(1, 1, 0)], first[(0, 0, 1)]] == [1, 2, 3, 4, 5]


@pytest.mark.parametrize("kind", ["one", "block"])
def test_bdf2_previous_state_round_trip(tmp_path, kind):
    """A restart after a BDF2 step (nStepPrev == nStep) carries #NPREVIOUS and
    ImplOld_VCB per block (src/ModRestartFile.f90:457-461, 828-829,
    1084-1091); the state and the previous state both come back."""
    g, S, t, n, dtB = case()
    prev = np.random.default_rng(9).normal(size=(g.nBlock, 8, 8, 8, 8))
    restart.write_restart_arrays(str(tmp_path), g, S, t, n, dtB, kind, ImplOld=prev, DtPrev=3.5e-3)
    g2, S2, t2, n2, dtB2 = restart.read_restart(str(tmp_path))
    assert np.array_equal(S2[g.interior_slices()], S[g.interior_slices()]) and (t2, n2) == (t, n)
    assert np.array_equal(dtB2, dtB)
    dtPrev, prev2 = restart.read_restart_previous(str(tmp_path))
    assert dtPrev == 3.5e-3 and np.array_equal(prev2, prev)
    h = restart.read_header(str(tmp_path))
    assert h["#NPREVIOUS"][0] == str(n)
    if kind == "one":
        raw = np.fromfile(os.path.join(str(tmp_path), "data.rst"), dtype="<f8")
        nRec = 7 + 2 * 8 * 512
        assert raw.size == g.nBlock * nRec
        order = restart.morton_order(g)
        b = 3
        r = raw[(order[b] - 1) * nRec:order[b] * nRec]
        # State8_CV(i, j, k, iVar): the variable slowest
        i, j, k, v = 2, 5, 1, 6
        assert r[7 + 8 * 512 + i + 8 * (j + 8 * (k + 8 * v))] == prev[b, k, j, i, v]
    assert restart.read_restart_previous(str(tmp_path)) is not None


def test_no_previous_state_without_bdf2(tmp_path):
    g, S, t, n, dtB = case()
    restart.write_restart_arrays(str(tmp_path), g, S, t, n, dtB, "one")
    assert restart.read_restart_previous(str(tmp_path)) is None
