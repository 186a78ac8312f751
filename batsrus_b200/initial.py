"""Initial states (host side), following src/ModSetInitialCondition.f90.

``set_initial_condition`` (:153-330) fills every cell of a block, ghost cells
included, with the primitive state and then converts velocity to momentum
(RhoU = Rho*U).  The states used by the hot-path configurations:

* ``shocktube``  -- #SHOCKTUBE left/right states split at ShockPosition with
  ShockSlope = 0 (:231-262);
* ``uniform``    -- #UNIFORMSTATE (:74);
* ``orszag_tang_3d`` -- Orszag-Tang vortex extended in z;
* ``blast``      -- MHD blast wave (pressure jump inside r < r0);
* ``perturbed_ot`` -- Orszag-Tang plus a seeded Gaussian random-phase
  perturbation for the implicit configuration.

All functions return the Fortran-layout array ``(nBlock, nKg, nJg, nIg, 8)``
with conservative momentum and primitive pressure (the reference stores p,
not energy, in State_VGB).
"""
import math

import numpy as np

from .grid import NVAR

PRIM_NAMES = ("rho", "ux", "uy", "uz", "bx", "by", "bz", "p")


def _from_primitive(prim):
    st = prim.copy()
    st[..., 1:4] = prim[..., 0:1] * prim[..., 1:4]
    return st


def shocktube(grid, left, right, shock_position=0.0):
    """#SHOCKTUBE: ``left``/``right`` are 8 primitive values."""
    xyz = grid.cell_centers()
    prim = np.empty(grid.state_shape_fortran())
    isleft = (xyz[..., 0] - shock_position) < 0.0
    prim[...] = np.asarray(right, dtype=np.float64)
    prim[isleft] = np.asarray(left, dtype=np.float64)
    return _from_primitive(prim)


def uniform(grid, state):
    prim = np.empty(grid.state_shape_fortran())
    prim[...] = np.asarray(state, dtype=np.float64)
    return _from_primitive(prim)


def orszag_tang_3d(grid):
    """rho = 25/(36 pi), p = 5/(12 pi), u = (-sin 2pi y, sin 2pi x,
    0.01 sin 2pi z), B = (-sin 2pi y, sin 4pi x, 0)/sqrt(4 pi)."""
    xyz = grid.cell_centers()
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    twopi = 2.0 * math.pi
    prim = np.empty(grid.state_shape_fortran())
    prim[..., 0] = 25.0 / (36.0 * math.pi)
    prim[..., 1] = -np.sin(twopi * y)
    prim[..., 2] = np.sin(twopi * x)
    prim[..., 3] = 0.01 * np.sin(twopi * z)
    b0 = 1.0 / math.sqrt(4.0 * math.pi)
    prim[..., 4] = -b0 * np.sin(twopi * y)
    prim[..., 5] = b0 * np.sin(2.0 * twopi * x)
    prim[..., 6] = 0.0
    prim[..., 7] = 5.0 / (12.0 * math.pi)
    return _from_primitive(prim)


def blast(grid, p_in=10.0, p_out=0.1, r0=0.1, rho=1.0, b=(1 / math.sqrt(2), 1 / math.sqrt(2), 0.0)):
    xyz = grid.cell_centers()
    r = np.sqrt((xyz ** 2).sum(-1))
    prim = np.empty(grid.state_shape_fortran())
    prim[..., 0] = rho
    prim[..., 1:4] = 0.0
    prim[..., 4:7] = np.asarray(b)
    prim[..., 7] = np.where(r < r0, p_in, p_out)
    return _from_primitive(prim)


def _random_phase_field(grid, xyz, ks, amp):
    """sum_k Re(a_k exp(2 pi i k.x)) at the cell centres xyz (ghosts included).

    On a single-level grid whose domain has unit length in every direction
    (so that the field is periodic over it) the sum is one inverse FFT of
    the uniform N^3 mesh, with the half-cell shift of the cell centres in the
    amplitudes; each cell (ghost cells by their periodic image) then reads
    its mesh value.  Otherwise the modes are summed directly."""
    lev = grid.iLevelCoord[:, 0]
    ext = [grid.xyzMax[d] - grid.xyzMin[d] for d in range(3)]
    if grid.nDim == 3 and np.all(lev == lev[0]) and all(abs(e - 1.0) < 1e-14 for e in ext):
        n = [grid.nRoot[d] * (1 << int(lev[0])) * (grid.nI, grid.nJ, grid.nK)[d] for d in range(3)]
        spec = np.zeros(n, dtype=complex)
        for (kx, ky, kz), a in zip(ks, amp):
            x0 = [grid.xyzMin[d] + 0.5 / n[d] for d in range(3)]
            shift = np.exp(2j * math.pi * (kx * x0[0] + ky * x0[1] + kz * x0[2]))
            spec[kx % n[0], ky % n[1], kz % n[2]] += a * shift
        mesh = (np.fft.ifftn(spec) * (n[0] * n[1] * n[2])).real
        idx = [np.floor((xyz[..., d] - grid.xyzMin[d]) * n[d]).astype(np.int64) % n[d] for d in range(3)]
        return mesh[idx[0], idx[1], idx[2]]
    field = np.zeros(xyz.shape[:-1])
    for (kx, ky, kz), a in zip(ks, amp):
        ph = 2 * math.pi * (kx * xyz[..., 0] + ky * xyz[..., 1] + kz * xyz[..., 2])
        field += (a * np.exp(1j * ph)).real
    return field


def perturbed_ot(grid, seed=2024, amplitude=1e-2, kmax=8):
    """Orszag-Tang plus a Gaussian random-phase perturbation of every
    primitive variable: sum over integer wave vectors 0 < |k| <= kmax of
    complex amplitudes drawn from numpy ``default_rng(seed)``, normalised to
    unit variance and scaled by ``amplitude`` (relative for rho and p)."""
    st = orszag_tang_3d(grid)
    prim = st.copy()
    prim[..., 1:4] = st[..., 1:4] / st[..., 0:1]
    xyz = grid.cell_centers()
    rng = np.random.default_rng(seed)
    ks = [(kx, ky, kz) for kx in range(-kmax, kmax + 1) for ky in range(-kmax, kmax + 1)
          for kz in range(0, kmax + 1) if 0 < kx * kx + ky * ky + kz * kz <= kmax * kmax]
    for v in range(NVAR):
        amp = rng.normal(size=len(ks)) + 1j * rng.normal(size=len(ks))
        field = _random_phase_field(grid, xyz, ks, amp)
        field /= max(field.std(), 1e-300)
        if v in (0, 7):
            prim[..., v] *= 1.0 + amplitude * field
        else:
            prim[..., v] += amplitude * field
    return _from_primitive(prim)
