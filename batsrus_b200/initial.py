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


# primitive variable order of the wave tables below
_PRIM = {"rho": 0, "ux": 1, "uy": 2, "uz": 3, "bx": 4, "by": 5, "bz": 6, "p": 7}


def uniform_waves(grid, state, waves, shock_slope=0.0):
    """#UNIFORMSTATE + #WAVE perturbations with #SHOCKPOSITION's slope
    (set_initial_condition, apply_wave and rotate_wave of
    src/ModSetInitialCondition.f90:195-528).

    ``state`` is the primitive uniform state; each wave is (name, width,
    amplitude, lambda_x, lambda_y, lambda_z, phase in degrees), a negative
    wavelength meaning no variation along that axis.  With a nonzero slope
    the vector variables of the uniform state, the wave amplitudes of the
    vector pairs (x, y) and all wave vectors are rotated by atan(slope) in
    the x-y plane; a vector pair with a wave on one component only copies
    that wave's width, wave vector, phase and power to the other component
    first (copy_wave)."""
    nV = 8
    width = np.zeros(nV)
    ampl = np.zeros(nV)
    kx = np.zeros(nV)
    ky = np.zeros(nV)
    kz = np.zeros(nV)
    phase = np.zeros(nV)
    for name, w, a, lx, ly, lz, ph in waves:
        v = _PRIM[name.lower()]
        width[v], ampl[v], phase[v] = w, a, ph * math.pi / 180.0
        kx[v] = max(0.0, 2.0 * math.pi / lx)
        ky[v] = max(0.0, 2.0 * math.pi / ly)
        kz[v] = max(0.0, 2.0 * math.pi / lz)
    prim0 = np.array(state, dtype=np.float64)
    if shock_slope != 0.0:
        c = 1.0 / math.sqrt(1.0 + shock_slope ** 2)
        s = shock_slope * c
        for vx in (1, 4):  # (Ux, Uy) and (Bx, By)
            vy = vx + 1
            for src, dst in ((vx, vy), (vy, vx)):
                if width[src] > 0.0 and width[dst] == 0.0:
                    width[dst], kx[dst], ky[dst], kz[dst], phase[dst] = \
                        width[src], kx[src], ky[src], kz[src], phase[src]
            x, y = ampl[vx], ampl[vy]
            ampl[vx], ampl[vy] = c * x - s * y, s * x + c * y
            x, y = prim0[vx], prim0[vy]
            prim0[vx], prim0[vy] = c * x - s * y, s * x + c * y
        x, y = kx.copy(), ky.copy()
        kx, ky = c * x - s * y, s * x + c * y
    xyz = grid.cell_centers()
    X, Y, Z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    prim = np.empty(grid.state_shape_fortran())
    prim[...] = prim0
    for v in range(nV):
        if ampl[v] == 0.0:
            continue
        inside = np.ones(X.shape, dtype=bool)
        if width[v] > 0.0:
            if kx[v] > 0.0:
                inside = np.abs(X + shock_slope * Y) <= width[v]
            elif ky[v] > 0.0:
                inside = np.abs(Y) <= width[v]
            elif kz[v] > 0.0:
                inside = np.abs(Z) <= width[v]
        wave = ampl[v] * np.cos(phase[v] + kx[v] * X + ky[v] * Y + kz[v] * Z)
        prim[..., v] = np.where(inside, prim[..., v] + wave, prim[..., v])
    return _from_primitive(prim)
