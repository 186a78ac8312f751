"""GPU parity of the block-adaptive explicit update against the oracle on a
static two- or three-level blast grid: the neighbour bookkeeping
(DiLevel_EB / jBlock_IEB) bit-exact, FP64 states within 1e-12 per step
for each flux (resolution-change ghost cells by injection / restriction,
first-order faces next to coarser blocks, flux correction on the coarse
side), conservation of mass and momentum through the flux correction, and
the FP32-bulk mode within 1e-6 relative L1 of the FP64 oracle."""
import numpy as np
import pytest

from batsrus_b200 import configs
from batsrus_b200.explicit import ExplicitSolver
from batsrus_b200.grid import BlockGrid
from batsrus_b200.param import Scheme
from batsrus_b200 import initial, capi
from oracle import Oracle

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    ax = tuple(range(a.ndim - 1))
    scale = np.abs(b).max(axis=ax)
    scale[1:4] = np.sqrt((b[..., 1:4] ** 2).sum(-1)).max()
    scale[4:7] = np.sqrt((b[..., 4:7] ** 2).sum(-1)).max()
    scale = np.maximum(scale, 1e-300)
    return (np.abs(a - b).max(axis=ax) / scale).max()


def grid(nRoot=2, maxLevel=2):
    return configs.amr_blast(nRoot=nRoot, maxLevel=maxLevel, with_state=False)[0]


def scheme(flux, limiter="mc", precision="fp64", tvd=True):
    return Scheme(nOrder=2, nStage=2, typeFlux=flux, typeLimiter=limiter, limiterBeta=1.5, cfl=0.8,
                  gamma=5.0 / 3.0, useDivbSource=True, useHalfStep=True, precision=precision,
                  useTvdResChange=tvd)


def test_neighbor_tables_bit_exact():
    import ctypes
    g = grid(4, 2)
    dil, jb = g.neighbors()
    assert (dil == 1).any() and (dil == -1).any()
    x = ExplicitSolver(g, scheme("Linde"))
    L = capi.load()
    d = np.zeros(6 * g.nBlock, dtype=np.int32)
    j = np.zeros(24 * g.nBlock, dtype=np.int32)
    capi.check(L.bx_get_neighbors(d.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  j.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
    x.close()
    assert np.array_equal(d.reshape(-1, 6), dil)
    assert np.array_equal(j.reshape(-1, 6, 4), jb + 1)


@pytest.mark.parametrize("tvd", [True, False], ids=["tvd_reschange", "first_order_reschange"])
@pytest.mark.parametrize("flux,limiter", [("Rusanov", "mc"), ("Linde", "mc3"), ("HLLD", "mc"), ("Roe", "mc3")])
def test_amr_fp64_steps_match_oracle(flux, limiter, tvd):
    """#RESOLUTIONCHANGE T (the reference's default: tvd_reschange faces, two
    coarse ghost layers, correct_monotone_restrict) and F (first-order faces)
    on a perturbed Orszag-Tang state, which varies across the resolution
    changes from the first step."""
    g = grid(2, 2)
    s = scheme(flux, limiter, tvd=tvd)
    st = initial.perturbed_ot(g, seed=3, amplitude=5e-2, kmax=4)
    o = Oracle(g, s)
    o.set_state(st)
    o.exchange_messages()
    x = ExplicitSolver(g, s)
    x.set_state(st)
    isl = g.interior_slices()
    for step in range(4):
        o.advance(1)
        x.advance(1)
        e = rel_err(x.get_state()[isl], o.get_state()[isl])
        assert e < 1e-12, (flux, step, e)
    to, _, no = o.time()
    tg, _, ng = x.time()
    assert ng == no and abs(tg - to) <= 1e-12 * to
    x.close()


@pytest.mark.parametrize("tvd", [True, False], ids=["tvd_reschange", "first_order_reschange"])
def test_amr_conserves_mass_and_momentum(tvd):
    import dataclasses
    g = grid(2, 2)
    # the Powell source would change the momentum of a state with div B /= 0
    s = dataclasses.replace(scheme("HLLD", tvd=tvd), useDivbSource=False)
    st = initial.perturbed_ot(g, seed=3, amplitude=5e-2, kmax=4)
    x = ExplicitSolver(g, s)
    x.set_state(st)
    isl = g.interior_slices()
    vol = g.block_geometry()[1].prod(1)

    def totals(u):
        u = u[isl]
        return np.array([(u[..., v].sum(axis=(1, 2, 3)) * vol).sum() for v in range(4)])

    m0 = totals(st)
    x.advance(6)
    m1 = totals(x.get_state())
    x.close()
    assert abs(m1[0] - m0[0]) <= 1e-13 * m0[0]
    assert np.abs(m1[1:] - m0[1:]).max() <= 1e-13 * m0[0]


def test_amr_fp32_bulk_l1():
    g = grid(2, 2)
    s64, s32 = scheme("HLLD"), scheme("HLLD", precision="fp32")
    st = initial.blast(g)
    o = Oracle(g, s64)
    o.set_state(st)
    o.exchange_messages()
    x = ExplicitSolver(g, s32)
    x.set_state(st)
    for _ in range(4):
        o.advance(1)
    x.advance(4)
    isl = g.interior_slices()
    a, b = x.get_state()[isl], o.get_state()[isl]
    l1 = np.abs(a - b).sum() / np.abs(b).sum()
    x.close()
    assert l1 < 1e-6, l1


def test_amr_beta_limiter_reschange_matches_oracle():
    """#RESOLUTIONCHANGE with BetaLimiterResChange 1.1 below the MC limiter's
    1.5: the two cells next to every resolution change and every outer
    (float) boundary take the softer limiter (src/ModFaceValue.f90:1979-2014),
    on top of the TVD faces."""
    import dataclasses
    g = configs.amr_blast(nRoot=2, maxLevel=2, with_state=False)[0]
    g = BlockGrid(g.nDim, g.nI, g.nJ, g.nK, g.nRoot, g.xyzMin, g.xyzMax, ("float",) * 6, g.iLevelCoord)
    s = dataclasses.replace(scheme("Linde", "mc"), betaLimiterResChange=1.1, nFaceLimiterResChange=2)
    st = initial.perturbed_ot(g, seed=4, amplitude=5e-2, kmax=4)
    o = Oracle(g, s)
    o.set_state(st)
    o.exchange_messages()
    x = ExplicitSolver(g, s)
    x.set_state(st)
    isl = g.interior_slices()
    for step in range(3):
        o.advance(1)
        x.advance(1)
        assert rel_err(x.get_state()[isl], o.get_state()[isl]) < 1e-12, step
    # the softer limiter changes the result
    o2 = Oracle(g, scheme("Linde", "mc"))
    o2.set_state(st)
    o2.exchange_messages()
    o2.advance(3)
    assert rel_err(o2.get_state()[isl], o.get_state()[isl]) > 1e-8
    x.close()
