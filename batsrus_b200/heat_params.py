"""Parameters and workload of the semi-implicit field-aligned heat conduction
(#SEMIIMPLICIT parcond, #SEMIKRYLOV, #SEMIPRECOND of
src/ModSemiImplicit.f90:51-108; the heat conduction coefficients of
src/ModHeatConduction.f90).

The workload: a uniform periodic-free unit cube [-0.5, 0.5]^3 of
(8 nRoot)^3 cells in 8^3 blocks (nRoot = 32 gives 256^3) with float outer
boundaries; Te = 1 + exp(sigma g), one plus a log-normal perturbation with
sigma = 0.3 made from a seeded unit-variance Gaussian random-phase field g
(|k| <= 8); B from a
dipole at the origin along z; cells with r < 0.2 are not used (their
temperature is held); HeatCoef = HeatCondPar Te^2.5 along the field and
(1 - FractionFieldAligned) of it across, so kappa_par / kappa_perp = 1e6.
"""
import math
from dataclasses import dataclass

import numpy as np


@dataclass
class HeatParams:
    heatCondPar: float = 1.0          # HeatCondPar (Spitzer coefficient, normalised)
    fieldAligned: float = 1.0 - 1e-6  # FractionFieldAligned: kappa_perp / kappa_par = 1e-6
    cv: float = 1.5                   # DconsDsemi = n / (gamma_e - 1), n = 1
    dt: float = 1e-4                  # semi-implicit time step (about 100x the explicit limit)
    semiImplCoeff: float = 1.0        # SemiImplCoeff (backward Euler)
    nKrylovVector: int = 30           # #SEMIKRYLOV
    maxMatvec: int = 1000
    errorMax: float = 1e-6
    typePrecond: str = "BILU"         # BILU | NONE | LEARNED (#SEMIPRECOND)
    precondPrecision: str = "fp64"    # BILU sweeps: fp64 | fp32 (FP32 coefficients and arithmetic)
    operatorPrecision: str = "fp64"   # face tensor of the Krylov matvec: fp64 | fp32 (FP64 arithmetic)


def heat_dipole(nRoot=32, seed=2024, sigma=0.3, rExcl=0.2):
    """Global fields of the workload, x fastest: Te (n^3), unit field b
    (n^3 x 3), used mask (n^3), cell size; n = 8 nRoot."""
    from . import initial
    from .grid import BlockGrid
    n = 8 * nRoot
    g = BlockGrid.uniform(3, (8, 8, 8), (nRoot,) * 3, (-0.5,) * 3, (0.5,) * 3, ("float",) * 6)
    rng = np.random.default_rng(seed)
    kmax = 8
    ks = [(kx, ky, kz) for kx in range(-kmax, kmax + 1) for ky in range(-kmax, kmax + 1)
          for kz in range(0, kmax + 1) if 0 < kx * kx + ky * ky + kz * kz <= kmax * kmax]
    amp = rng.normal(size=len(ks)) + 1j * rng.normal(size=len(ks))
    # the random field on the global mesh through the block-grid routine
    xyz = g.cell_centers(with_ghost=False)
    f = initial._random_phase_field(g, xyz, ks, amp)
    f /= max(f.std(), 1e-300)
    Te_blocks = 1.0 + np.exp(sigma * f)
    x = (np.arange(n) + 0.5) / n - 0.5
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z)
    rs = np.maximum(r, 1e-12)
    # dipole m = z: B = (3 (m.rhat) rhat - m) / r^3, direction only
    mr = Z / rs
    B = np.stack([3 * mr * X / rs, 3 * mr * Y / rs, 3 * mr * Z / rs - 1.0], axis=-1)
    b = B / np.maximum(np.sqrt((B * B).sum(-1, keepdims=True)), 1e-300)
    used = (r >= rExcl).astype(np.uint8)
    Te = blocks_to_global(Te_blocks, nRoot)
    return g, Te.ravel(), b.reshape(-1, 3), used.ravel(), 1.0 / n


def blocks_to_global(a, nRoot):
    """(nBlock, 8, 8, 8[, ...]) in x-fastest block order -> (n, n, n[, ...])
    indexed [k][j][i]"""
    n = 8 * nRoot
    rest = a.shape[4:]
    a = a.reshape((nRoot, nRoot, nRoot, 8, 8, 8) + rest)  # bz, by, bx, k, j, i
    a = np.moveaxis(a, (0, 1, 2, 3, 4, 5), (0, 2, 4, 1, 3, 5))
    return a.reshape((n, n, n) + rest)


def global_to_blocks(a, nRoot):
    """inverse of blocks_to_global: (n, n, n[, ...]) -> (nBlock, 8, 8, 8[, ...])"""
    rest = a.shape[3:]
    a = a.reshape((nRoot, 8, nRoot, 8, nRoot, 8) + rest)  # bz, k, by, j, bx, i
    a = np.moveaxis(a, (0, 2, 4, 1, 3, 5), (0, 1, 2, 3, 4, 5))
    return a.reshape((nRoot ** 3, 8, 8, 8) + rest)
