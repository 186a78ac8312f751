"""The hot-path workloads: grid, scheme and initial state of each.

* ``shocktube_1d_golden`` -- the reference's own GPU test
  ``test_shocktube_1d`` (Makefile.test:293-323): 16 blocks of 64 cells on
  [-128,128], MhdHyp with Hyp = 0 and no hyperbolic cleaning (identical to
  ideal MHD), gamma 2, first-order Rusanov, 1 stage, Dt fixed at 0.05,
  512 steps to t = 25.6, float boundaries.
* ``brio_wu_1d`` -- 256 cells as 32 blocks of 8 on [-0.5,0.5], gamma 2,
  Rusanov, MC limiter beta 1.5, 2-stage, CFL 0.8, to t = 0.1, float
  boundaries, no Powell source (nDim = 1).
* ``orszag_tang_3d`` -- periodic unit cube, (8 nRoot)^3 cells in 8^3 blocks
  (nRoot = 32 gives 256^3 = 32768 blocks), Linde HLL flux, Koren (mc3)
  limiter with beta 1.2 (the PARAM.XML default for mc3), CFL 0.8,
  gamma 5/3, Powell source on.
* ``jfnk_ot`` -- the implicit workload: periodic unit cube of (8 nRoot)^3
  cells (nRoot = 16 gives 128^3 = 4096 blocks), Orszag-Tang plus a seeded
  Gaussian random-phase perturbation (amplitude 1e-2, |k| <= 8), the
  explicit scheme of ``orszag_tang_3d`` for the high-order residual, and
  BDF2 with CflImpl 20, GMRES(30) to 1e-3 relative.
* ``amr_blast`` -- the block-adaptive workload: [-0.5,0.5]^3 (periodic),
  root blocks of 8^3 cells refined up to maxLevel where |grad p|/p > 0.5 on
  the initial blast state (rho = 1, p = 10 inside r < 0.1 and 0.1 outside,
  B = (1,1,0)/sqrt 2), levels balanced 2:1; HLLD flux, MC limiter (beta
  1.5), CFL 0.8, 2-stage, Powell source, flux correction at resolution
  changes.
"""
import math

from . import initial
from .grid import BlockGrid
from .param import Scheme


def shocktube_1d_golden():
    g = BlockGrid.uniform(1, (64, 1, 1), (16, 1, 1), (-128.0, -0.125, -0.125),
                          (128.0, 0.125, 0.125), ("float",) * 6)
    s = Scheme(nOrder=1, nStage=1, typeFlux="Rusanov", typeLimiter="no", cfl=1.0, gamma=2.0,
               useDivbSource=False, useDtFixed=True, dtFixed=0.05, useHalfStep=True)
    st = initial.shocktube(g, [1, 0, 0, 0, 0.75, 1, 0, 1], [0.125, 0, 0, 0, 0.75, -1, 0, 0.1])
    return g, s, st, {"nStep": 512, "tSimulationMax": 25.6}


def fast_wave_golden():
    """Param/SHOCKTUBE/PARAM.in.fast_wave (Makefile.test:439-459) on its
    root grid: 5 x 5 x 20 blocks of 10^3 cells, [-45.255, 45.255]^2 x
    [-181.02, 181.02], periodic; the uniform state rho = 1, u = (0, 0,
    0.005), B = (0, 0.04, 0), p = 4.5e-4 with the fast-wave perturbations
    (lambda = 32) rotated by 45 degrees (ShockSlope = 1); fixed time step 0.5
    (Cfl = 1 with a fixed step), the pressure equation (#NONCONSERVATIVE),
    Powell source; three sessions: Rusanov first order to t = 25, Rusanov
    second order mc3 (beta 1.2) to t = 50, Linde mc3 to t = 75.  The
    reference run also refines the two root blocks that touch the box
    [-1, 1]^3; this grid has no refinement, so a comparison excludes the
    refined patch and its surroundings."""
    g = BlockGrid.uniform(3, (10, 10, 10), (5, 5, 20), (-45.255, -45.255, -181.02),
                          (45.255, 45.255, 181.02), ("periodic",) * 6)
    base = dict(cfl=1.0, gamma=5.0 / 3.0, useDivbSource=True, useDtFixed=True, dtFixed=0.5,
                useHalfStep=True, useNonConservative=True)
    sessions = [
        (Scheme(nOrder=1, nStage=1, typeFlux="Rusanov", typeLimiter="no", **base), 25.0),
        (Scheme(nOrder=2, nStage=2, typeFlux="Rusanov", typeLimiter="mc3", limiterBeta=1.2, **base), 50.0),
        (Scheme(nOrder=2, nStage=2, typeFlux="Linde", typeLimiter="mc3", limiterBeta=1.2, **base), 75.0),
    ]
    waves = [("Rho", 1000.0, 0.1, 32.0, -1.0, -1.0, 0.0),
             ("Ux", 1000.0, 0.005, 32.0, -1.0, -1.0, 0.0),
             ("Uz", 1000.0, 0.0001, -1.0, -1.0, 32.0, 0.0),
             ("Bx", 1000.0, 0.0004, 32.0, -1.0, -1.0, 0.0),
             ("By", 1000.0, 0.004, 32.0, -1.0, -1.0, 0.0),
             ("p", 10000.0, 7.5e-5, 32.0, -1.0, -1.0, 0.0)]
    st = initial.uniform_waves(g, [1.0, 0.0, 0.0, 0.005, 0.0, 0.04, 0.0, 4.5e-4], waves, shock_slope=1.0)
    return g, sessions, st


def brio_wu_1d(nBlock=32):
    g = BlockGrid.uniform(1, (8, 1, 1), (nBlock, 1, 1), (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5),
                          ("float",) * 6)
    s = Scheme(nOrder=2, nStage=2, typeFlux="Rusanov", typeLimiter="mc", limiterBeta=1.5, cfl=0.8,
               gamma=2.0, useDivbSource=False, useHalfStep=True)
    st = initial.shocktube(g, [1, 0, 0, 0, 0.75, 1, 0, 1], [0.125, 0, 0, 0, 0.75, -1, 0, 0.1])
    return g, s, st, {"tSimulationMax": 0.1}


def orszag_tang_3d(nRoot=32, precision="fp64", flux="Linde", limiter="mc3", beta=1.2,
                   nCellBlock=(8, 8, 8), order="x", with_state=True):
    g = BlockGrid.uniform(3, nCellBlock, (nRoot,) * 3, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0),
                          ("periodic",) * 6, order=order)
    s = Scheme(nOrder=2, nStage=2, typeFlux=flux, typeLimiter=limiter, limiterBeta=beta, cfl=0.8,
               gamma=5.0 / 3.0, useDivbSource=True, useHalfStep=True, precision=precision)
    st = initial.orszag_tang_3d(g) if with_state else None
    return g, s, st, {"nStep": 20}


def uniform_3d_case(nRoot, flux, limiter="mc3", beta=1.2, precision="fp64", nCellBlock=(8, 8, 8),
                    state="ot", bc="periodic"):
    """Small 3D parity case with any flux/limiter."""
    g = BlockGrid.uniform(3, nCellBlock, tuple(nRoot) if hasattr(nRoot, "__len__") else (nRoot,) * 3,
                          (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (bc,) * 6)
    s = Scheme(nOrder=2, nStage=2, typeFlux=flux, typeLimiter=limiter, limiterBeta=beta, cfl=0.8,
               gamma=5.0 / 3.0, useDivbSource=True, useHalfStep=True, precision=precision)
    if state == "ot":
        st = initial.orszag_tang_3d(g)
    elif state == "blast":
        g = BlockGrid.uniform(3, nCellBlock, tuple(nRoot) if hasattr(nRoot, "__len__") else (nRoot,) * 3,
                              (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5), (bc,) * 6)
        st = initial.blast(g)
    else:
        st = initial.perturbed_ot(g, seed=7, amplitude=0.05, kmax=2)
    return g, s, st, {}


def jfnk_ot(nRoot=16, precond="BILU", seed=2024, with_state=True, precondPrecision="bf16"):
    """The implicit workload: perturbed Orszag-Tang on (8 nRoot)^3 cells,
    BDF2 at CFL 20, GMRES(30) to 1e-3; BILU factors stored in BF16 unless
    precondPrecision says otherwise."""
    from .implicit_params import ImplicitParams
    g = BlockGrid.uniform(3, (8, 8, 8), (nRoot,) * 3, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), ("periodic",) * 6)
    s = Scheme(nOrder=2, nStage=2, typeFlux="Linde", typeLimiter="mc3", limiterBeta=1.2, cfl=0.8,
               gamma=5.0 / 3.0, useDivbSource=True, useHalfStep=True)
    p = ImplicitParams(cflImpl=20.0, useBdf2=True, nKrylovVector=30, maxMatvec=100, errorMax=1e-3,
                       typePrecond=precond, precondPrecision=precondPrecision)
    st = initial.perturbed_ot(g, seed=seed, amplitude=1e-2, kmax=8) if with_state else None
    return g, s, p, st


def _blast_refine(nRoot, pin=10.0, pout=0.1, r0=0.1, crit=0.5):
    """refine(level, ix, iy, iz): |grad p|/p > crit somewhere in the block,
    with the gradient by central differences of the initial pressure on the
    block's own cells (one cell of the block's resolution across)."""
    import numpy as np

    def refine(lv, i, j, k):
        n = nRoot << lv
        bs = 1.0 / n
        h = bs / 8
        x = -0.5 + (np.array([i, j, k])[:, None] * bs) + (np.arange(-1, 9)[None, :] + 0.5) * h
        X, Y, Z = np.meshgrid(x[0], x[1], x[2], indexing="ij")
        p = np.where(X * X + Y * Y + Z * Z < r0 * r0, pin, pout)
        gx = (p[2:, 1:-1, 1:-1] - p[:-2, 1:-1, 1:-1]) / (2 * h)
        gy = (p[1:-1, 2:, 1:-1] - p[1:-1, :-2, 1:-1]) / (2 * h)
        gz = (p[1:-1, 1:-1, 2:] - p[1:-1, 1:-1, :-2]) / (2 * h)
        g = np.sqrt(gx * gx + gy * gy + gz * gz) / p[1:-1, 1:-1, 1:-1]
        return bool((g > crit).any())

    return refine


def amr_blast(nRoot=8, maxLevel=3, precision="fp32", flux="HLLD", limiter="mc", beta=1.5, with_state=True):
    g = BlockGrid.adaptive(3, (8, 8, 8), (nRoot,) * 3, (-0.5,) * 3, (0.5,) * 3, ("periodic",) * 6, maxLevel,
                           _blast_refine(nRoot))
    s = Scheme(nOrder=2, nStage=2, typeFlux=flux, typeLimiter=limiter, limiterBeta=beta, cfl=0.8,
               gamma=5.0 / 3.0, useDivbSource=True, useHalfStep=True, precision=precision)
    st = initial.blast(g) if with_state else None
    return g, s, st, {"nStep": 50}


CELLS_PER_STEP_BYTES = {"fp64": 320, "fp32": 256}
