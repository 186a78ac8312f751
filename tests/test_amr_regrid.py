"""Host side of the dynamic AMR (batsrus_b200.amr, the BATL regrid rules
restated from PARAM.XML's #AMR / #AMRCRITERIA / #AMRLEVELS): refinement with
the splits that keep neighbouring levels within one, coarsening of whole
sibling groups only, the level and block-count limits, the remap table of
bx_regrid, the PARAM.in commands, and the conservation of the oracle's
restated remap (injection and 2x2x2 means).  CPU only."""
import numpy as np
import pytest

from batsrus_b200 import amr, configs
from batsrus_b200.grid import BlockGrid
from batsrus_b200.param import apply_commands, read_param, Scheme
from amr_ref import block_geometry, remap_state


def uniform(n=2, level=0, bc="periodic"):
    return BlockGrid.uniform(3, (8, 8, 8), (n,) * 3, (-0.5,) * 3, (0.5,) * 3, (bc,) * 6, level=level, order="morton")


def params(coarsen=0.2, refine=1.0, **kw):
    return amr.AmrParams(dnRefine=1, criteria=[amr.AmrCriterion("gradlogp", coarsen, refine)], **kw)


def crit_for(grid, refine_keys=(), coarsen_all=False, value=0.5):
    c = np.full((grid.nBlock, 1), 0.0 if coarsen_all else value)
    keys = [tuple(int(v) for v in k) for k in grid.iLevelCoord]
    for b, k in enumerate(keys):
        if k in refine_keys:
            c[b, 0] = 10.0
    return c


def keyset(grid):
    return {tuple(int(v) for v in k) for k in grid.iLevelCoord}


def test_refine_one_block_of_a_uniform_grid():
    g = uniform(2)
    new, R, changed = amr.regrid(g, crit_for(g, {(0, 0, 0, 0)}), params())
    assert changed and new.nBlock == g.nBlock + 7
    assert amr.is_balanced(new)
    ops = R[:, 0]
    assert (ops == amr.PROLONG).sum() == 8 and (ops == amr.COPY).sum() == 7
    kids = R[ops == amr.PROLONG]
    assert set(kids[:, 1]) == {1 + [tuple(k) for k in g.iLevelCoord.tolist()].index((0, 0, 0, 0))}
    assert sorted(kids[:, 2]) == list(range(8))


def test_refinement_splits_coarser_neighbours():
    g = uniform(2)
    g1, _, _ = amr.regrid(g, crit_for(g, {(0, 0, 0, 0)}), params())
    # refine a level-1 child at the corner of the refined region: the level-0
    # blocks across its faces, edges and corners (periodic) must split too
    new, R, _ = amr.regrid(g1, crit_for(g1, {(1, 0, 0, 0)}), params())
    assert amr.is_balanced(new)
    levels = np.bincount(new.iLevelCoord[:, 0])
    assert levels[2] == 8 and new.nBlock > g1.nBlock + 7
    # every new block is kept, refined once or coarsened once
    assert set(np.unique(R[:, 0])) <= {amr.COPY, amr.PROLONG}


def test_no_criterion_fired_keeps_the_grid():
    g = configs.amr_blast(nRoot=2, maxLevel=2, with_state=False)[0]
    new, R, changed = amr.regrid(g, crit_for(g), params())
    assert not changed and np.array_equal(new.iLevelCoord, g.iLevelCoord)
    assert (R[:, 0] == amr.COPY).all() and np.array_equal(R[:, 1], np.arange(1, g.nBlock + 1))


def test_coarsening_merges_whole_sibling_groups_away_from_finer_blocks():
    g = configs.amr_blast(nRoot=2, maxLevel=2, with_state=False)[0]
    new, R, changed = amr.regrid(g, crit_for(g, coarsen_all=True), params())
    assert changed and new.nBlock < g.nBlock and amr.is_balanced(new)
    old = keyset(g)
    for b in np.flatnonzero(R[:, 0] == amr.RESTRICT):
        lv, i, j, k = new.iLevelCoord[b]
        for o in range(8):
            assert (lv + 1, 2 * i + (o & 1), 2 * j + ((o >> 1) & 1), 2 * k + (o >> 2)) in old
    # the finest level cannot coarsen where a level-2 block touches level-1
    # siblings, so one pass coarsens by at most one level everywhere
    assert new.iLevelCoord[:, 0].max() >= g.iLevelCoord[:, 0].max() - 1


def test_refine_then_coarsen_restores_a_uniform_grid():
    g = uniform(2)
    up, _, _ = amr.regrid(g, np.full((g.nBlock, 1), 10.0), params())
    assert up.nBlock == 8 * g.nBlock and (up.iLevelCoord[:, 0] == 1).all()
    down, R, _ = amr.regrid(up, crit_for(up, coarsen_all=True), params())
    assert keyset(down) == keyset(g) and (R[:, 0] == amr.RESTRICT).all()


def test_level_limits():
    g = uniform(2, level=1)
    p = params(minBlockLevel=1, maxBlockLevel=2)
    down, _, changed = amr.regrid(g, crit_for(g, coarsen_all=True), p)
    assert not changed  # MinBlockLevel = 1: no coarsening below level 1
    up, _, _ = amr.regrid(g, np.full((g.nBlock, 1), 10.0), p)
    assert (up.iLevelCoord[:, 0] == 2).all()
    again, _, changed = amr.regrid(up, np.full((up.nBlock, 1), 10.0), p)
    assert not changed  # MaxBlockLevel = 2: level-2 blocks neither refine nor coarsen
    again, _, changed = amr.regrid(up, crit_for(up, coarsen_all=True), p)
    assert not changed


def test_max_total_blocks():
    g = uniform(2)
    c = np.arange(g.nBlock, dtype=float)[:, None] + 2.0  # every block asks, largest last
    new, _, _ = amr.regrid(g, c, params(maxTotalBlocks=g.nBlock + 2 * 7))
    assert new.nBlock <= g.nBlock + 14 and amr.is_balanced(new)
    # the two largest criteria were refined
    lv1 = {(int(k[1]) >> 1, int(k[2]) >> 1, int(k[3]) >> 1) for k in new.iLevelCoord if k[0] == 1}
    keys = [tuple(int(v) for v in k[1:]) for k in g.iLevelCoord]
    assert lv1 >= {keys[-1]} and len(lv1) >= 1


@pytest.mark.parametrize("seed", range(6))
def test_random_regrids_stay_balanced_and_remap_covers_every_cell(seed):
    rng = np.random.default_rng(seed)
    g = configs.amr_blast(nRoot=2, maxLevel=2, with_state=False)[0]
    for _ in range(3):
        c = rng.uniform(0.0, 2.0, size=(g.nBlock, 1))
        new, R, _ = amr.regrid(g, c, params(coarsen=0.5, refine=1.5, maxBlockLevel=4))
        assert amr.is_balanced(new)
        # volume: kept + refined + coarsened blocks tile the old domain
        _, vold, _ = block_geometry(g)
        _, vnew, _ = block_geometry(new)
        assert np.isclose(vold.sum() * 512, vnew.sum() * 512)
        old_keys = [tuple(int(v) for v in k) for k in g.iLevelCoord]
        used = np.zeros(g.nBlock, int)
        for b in range(new.nBlock):
            if R[b, 0] == amr.COPY:
                used[R[b, 1] - 1] += 8
            elif R[b, 0] == amr.PROLONG:
                used[R[b, 1] - 1] += 1
            else:
                used[R[b, 1:9] - 1] += 8
        assert (used == 8).all()  # every old block's volume goes exactly once
        g = new


def test_oracle_remap_conserves_mass_and_is_exact_for_copies():
    g = configs.amr_blast(nRoot=2, maxLevel=2, with_state=False)[0]
    from batsrus_b200 import initial
    st = initial.blast(g)
    # refine the coarsest blocks, coarsen everything else
    lev = g.iLevelCoord[:, :1]
    c = np.where(lev == lev.min(), 10.0, 0.0)
    new, R, _ = amr.regrid(g, c, params(maxBlockLevel=4))
    assert (R[:, 0] == amr.PROLONG).any() and (R[:, 0] == amr.RESTRICT).any()
    s2 = remap_state(st, R, new)
    isl = g.interior_slices()
    _, vo, _ = block_geometry(g)
    _, vn, _ = block_geometry(new)
    m0 = (st[isl][..., 0].reshape(g.nBlock, -1).sum(1) * vo).sum()
    m1 = (s2[new.interior_slices()][..., 0].reshape(new.nBlock, -1).sum(1) * vn).sum()
    assert abs(m1 - m0) <= 1e-13 * m0
    for b in np.flatnonzero(R[:, 0] == amr.COPY):
        assert np.array_equal(s2[new.interior_slices()][b], st[isl][R[b, 1] - 1])


def test_param_commands():
    text = """
#DOAMR
T			DoAmr
4			DnAmr
-1.0			DtAmr
T			IsStrictAmr

#AMRCRITERIA
2			nRefineCrit
gradlogP		TypeRefine
0.3			CoarsenLimit
1.2			RefineLimit
pjumpratio		TypeRefine
1.1			CoarsenLimit
1.6			RefineLimit

#AMRLEVELS
0			MinBlockLevel
3			MaxBlockLevel
"""
    info = apply_commands(read_param(text)[0], Scheme())
    p = amr.read_amr_params(info)
    assert p.dnRefine == 4 and p.minBlockLevel == 0 and p.maxBlockLevel == 3
    assert [(c.name, c.coarsenLimit, c.refineLimit) for c in p.criteria] == [
        ("gradlogp", 0.3, 1.2), ("pjumpratio", 1.1, 1.6)]


def crit_patterns(g, rng):
    """criteria that refine, coarsen, both, or hit the block limit"""
    lev = g.iLevelCoord[:, :1]
    yield rng.uniform(0.0, 2.0, size=(g.nBlock, 1)), params(coarsen=0.5, refine=1.5, maxBlockLevel=4)
    yield np.zeros((g.nBlock, 1)), params()
    yield np.where(lev == lev.min(), 10.0, 0.0), params(maxBlockLevel=4)
    yield np.where(lev == lev.max(), 0.0, 0.5), params(maxBlockLevel=4)
    yield rng.uniform(0.0, 20.0, size=(g.nBlock, 1)), params(maxTotalBlocks=g.nBlock + 40, maxBlockLevel=5)
    yield rng.uniform(0.0, 2.0, size=(g.nBlock, 1)), params(coarsen=0.9, refine=1.8, minBlockLevel=1, maxBlockLevel=3)


@pytest.mark.parametrize("nRoot,maxLevel", [(2, 2), (4, 2), (3, 3)])
def test_native_plan_matches_restatement(nRoot, maxLevel):
    """bx_amr_plan (the library's C++ tree code, host only) makes the same
    decisions as the Python restatement: same blocks in the same order, same
    remap table"""
    g = configs.amr_blast(nRoot=nRoot, maxLevel=maxLevel, with_state=False)[0]
    rng = np.random.default_rng(nRoot + 10 * maxLevel)
    seen = set()
    for c, p in crit_patterns(g, rng):
        a = amr.regrid(g, c, p)
        b = amr.plan_native(g, c, p)
        assert np.array_equal(a[0].iLevelCoord, b[0].iLevelCoord) and np.array_equal(a[1], b[1]) and a[2] == b[2]
        seen.update(np.unique(a[1][:, 0]).tolist())
        # a second pass from the new grid
        c2 = rng.uniform(0.0, 2.0, size=(a[0].nBlock, 1))
        p2 = params(coarsen=0.7, refine=1.7, maxBlockLevel=maxLevel + 2)
        a2, b2 = amr.regrid(a[0], c2, p2), amr.plan_native(a[0], c2, p2)
        assert np.array_equal(a2[0].iLevelCoord, b2[0].iLevelCoord) and np.array_equal(a2[1], b2[1])
    assert seen == {amr.COPY, amr.PROLONG, amr.RESTRICT}


@pytest.mark.parametrize("order", ["morton", "x"])
def test_native_plan_without_requests_keeps_or_reorders_the_grid(order):
    """No block asks to refine or coarsen: on a grid in the planner's own
    order (levels-mixed Morton of the finest level) bx_amr_plan returns the
    grid unchanged with copies in place, without rebuilding the tree; on a
    grid in another order it reorders, as the Python restatement does."""
    g = configs.amr_blast(nRoot=3, maxLevel=2, with_state=False)[0]
    p = params(coarsen=0.2, refine=1.0)
    g = amr.plan_native(g, np.full((g.nBlock, 1), 0.5), p)[0]  # the planner's order
    if order == "x":
        perm = np.random.default_rng(3).permutation(g.nBlock)
        g = BlockGrid(g.nDim, g.nI, g.nJ, g.nK, g.nRoot, g.xyzMin, g.xyzMax, g.typeBc, g.iLevelCoord[perm].copy())
    c = np.full((g.nBlock, 1), 0.5)  # between the coarsen and refine limits
    a, b = amr.regrid(g, c, p), amr.plan_native(g, c, p)
    assert np.array_equal(a[0].iLevelCoord, b[0].iLevelCoord) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    if order == "morton":
        assert not b[2] and np.array_equal(b[0].iLevelCoord, g.iLevelCoord)
        assert (b[1][:, 0] == amr.COPY).all() and np.array_equal(b[1][:, 1], np.arange(1, g.nBlock + 1))
    else:
        assert b[2]


def test_minus_divu_criterion_is_exact_for_a_linear_velocity():
    """'-divu' (src/ModAMR.f90:476-497) of the CPU restatement: the central
    differences of calc_divergence are exact for a linear velocity field, so
    every block of a two-level grid gets -div u = -(a + b + c), with the
    ghost cells holding the same field; a uniform flow gives 0."""
    from amr_ref import criteria
    g = configs.amr_blast(nRoot=2, maxLevel=1, with_state=False)[0]
    xyz = g.cell_centers(with_ghost=True)
    S = np.zeros(xyz.shape[:-1] + (8,))
    S[..., 0] = 2.0
    S[..., 7] = 1.0
    coef = (0.5, -1.5, 2.0)
    for d in range(3):
        S[..., 1 + d] = S[..., 0] * coef[d] * xyz[..., d]
    c = criteria(S, g, ["-divu", "-divudx"])
    assert np.allclose(c, -sum(coef), rtol=0, atol=1e-12)
    S[..., 1:4] = 0.3
    assert np.abs(criteria(S, g, ["-divu"])).max() == 0.0
