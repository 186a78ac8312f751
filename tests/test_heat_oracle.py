"""The CPU oracle of the semi-implicit field-aligned heat conduction
(ModSemiImplicit parcond, ModHeatConduction) against an independent
vectorised numpy restatement, exact properties of the operator, and the
Krylov tolerance of its solve (test infrastructure check, no GPU).

The reference has no unit-level golden vector for this solve (its only
golden touching it, Param/CORONA/TestOutput/heatcond_2d_ref.out, needs the
MhdPe equation set and the full SWMF driver), so the oracle is pinned by
restatement and by properties: the isotropic limit is the 7-point
Laplacian, a field along x gives 1D diffusion along x, constants are in the
null space of the flux divergence, and the block ILU(0) solve equals
(D+U)^-1 D (L+D)^-1 on the in-block 7-point matrix."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from batsrus_b200.heat_params import HeatParams, heat_dipole
from oracle import HeatOracle


def pad(a):
    return np.pad(a, [(1, 1)] * 3 + [(0, 0)] * (a.ndim - 3), mode="edge")


def window(Ap, n, d, lr, off):
    """Slab of the padded array for the faces of dimension d: left (lr=0) or
    right (lr=1) cell, shifted by off (x, y, z) in the transverse dims;
    array axes are (z, y, x)."""
    sl = []
    for ax in range(3):
        g = 2 - ax
        if g == d:
            sl.append(slice(lr, lr + n + 1))
        else:
            sl.append(slice(1 + off[g], 1 + off[g] + n))
    return Ap[tuple(sl)]


def bb(b, f, d1, d2):
    return f * b[..., d1] * b[..., d2] + (1.0 - f) * (1.0 if d1 == d2 else 0.0)


def residual_np(S, HC, b3, f, dx):
    """Res = -sum_d (F+ - F-)/V, F = -Area HeatCoef BbF . FaceGrad
    (get_heat_conduction_rhs, src/ModHeatConduction.f90:1434-1545, with the
    face gradient of src/ModFaceGradient.f90 on a uniform grid)."""
    n = S.shape[0]
    V, area = dx ** 3, dx * dx
    Sp, Hp, Bp = pad(S), pad(HC), pad(b3)
    Res = np.zeros_like(S)
    z = (0, 0, 0)
    for d in range(3):
        SL, SR = window(Sp, n, d, 0, z), window(Sp, n, d, 1, z)
        g = [None] * 3
        g[d] = (1.0 / dx) * (SR - SL)
        for e in range(3):
            if e == d:
                continue
            o = [0, 0, 0]
            o[e] = 1
            om = [0, 0, 0]
            om[e] = -1
            sm = window(Sp, n, d, 0, om) + window(Sp, n, d, 1, om)
            s0 = SL + SR
            spp = window(Sp, n, d, 0, o) + window(Sp, n, d, 1, o)
            g[e] = (-0.25 / dx) * sm + 0.0 * s0 + (0.25 / dx) * spp
        HL, HR = window(Hp, n, d, 0, z), window(Hp, n, d, 1, z)
        BL, BR = window(Bp, n, d, 0, z), window(Bp, n, d, 1, z)
        F = 0.0
        for q in range(3):
            F = F + area * (0.5 * (HR + HL)) * (0.5 * (bb(BR, f, d, q) + bb(BL, f, d, q))) * g[q]
        F = -F
        ax = 2 - d
        up = [slice(None)] * 3
        dn = [slice(None)] * 3
        up[ax] = slice(1, None)
        dn[ax] = slice(None, -1)
        Res = Res - (F[tuple(up)] - F[tuple(dn)]) / V
    return Res


def case(nRoot=2, seed=7, **kw):
    g, Te, b, used, dx = heat_dipole(nRoot=nRoot, seed=seed)
    n = 8 * nRoot
    p = HeatParams(**kw)
    return n, dx, Te, b, used, p


def test_rhs_and_matvec_match_numpy_restatement():
    n, dx, Te, b, used, p = case()
    o = HeatOracle(n, dx, Te, b, used, p)
    T3, b3 = Te.reshape(n, n, n), b.reshape(n, n, n, 3)
    HC = p.heatCondPar * T3 ** 2.5
    Res = residual_np(T3, HC, b3, p.fieldAligned, dx)
    V = dx ** 3
    ref = np.where(used.reshape(n, n, n) == 1, V * Res, 0.0).ravel()
    got = o.rhs()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    x = np.random.default_rng(1).normal(size=n ** 3)
    u = used.reshape(n, n, n) == 1
    S = np.where(u, x.reshape(n, n, n), 0.0)
    Rx = residual_np(S, HC, b3, p.fieldAligned, dx)
    yref = np.where(u, V * (S * p.cv / p.dt - p.semiImplCoeff * Rx), V * (x.reshape(n, n, n) * p.cv / p.dt)).ravel()
    y = o.matvec(x)
    assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()
    o.close()


def test_periodic_boundaries_commute_with_a_cyclic_shift():
    """Periodic in all three dimensions, every cell used: the right-hand side
    of the cyclically shifted temperature and field is the shifted
    right-hand side (the boundary faces couple the opposite sides), and the
    fluxes through the periodic faces cancel: the sum of V Res is zero to
    rounding.  With float boundaries the shift changes the result."""
    n, dx, Te, b, used, p = case()
    used = np.ones_like(used)
    T3, b3 = Te.reshape(n, n, n), b.reshape(n, n, n, 3)
    sh = (3, 5, 7)
    roll = lambda a: np.roll(a, sh, axis=(0, 1, 2))
    per = (True, True, True)
    o = HeatOracle(n, dx, Te, b, used, p, periodic=per)
    o2 = HeatOracle(n, dx, roll(T3).ravel(), roll(b3).reshape(-1, 3), used, p, periodic=per)
    r1, r2 = o.rhs().reshape(n, n, n), o2.rhs().reshape(n, n, n)
    assert np.abs(roll(r1) - r2).max() <= 1e-12 * np.abs(r1).max()
    assert abs(r1.sum()) <= 1e-10 * np.abs(r1).sum()
    o.close()
    o2.close()
    f = HeatOracle(n, dx, Te, b, used, p)
    f2 = HeatOracle(n, dx, roll(T3).ravel(), roll(b3).reshape(-1, 3), used, p)
    assert np.abs(roll(f.rhs().reshape(n, n, n)) - f2.rhs().reshape(n, n, n)).max() > 1e-6 * np.abs(r1).max()
    f.close()
    f2.close()


def test_isotropic_limit_is_the_7_point_laplacian():
    n = 16
    dx = 1.0 / n
    Te = np.ones(n ** 3)
    b = np.tile([0.6, 0.0, 0.8], (n ** 3, 1))
    used = np.ones(n ** 3, dtype=np.uint8)
    p = HeatParams(fieldAligned=0.0)
    o = HeatOracle(n, dx, Te, b, used, p)
    x = np.random.default_rng(2).normal(size=(n, n, n))
    xp = pad(x)
    lap = (xp[2:, 1:-1, 1:-1] + xp[:-2, 1:-1, 1:-1] + xp[1:-1, 2:, 1:-1] + xp[1:-1, :-2, 1:-1] +
           xp[1:-1, 1:-1, 2:] + xp[1:-1, 1:-1, :-2] - 6 * x) / dx ** 2
    V = dx ** 3
    yref = V * (x * p.cv / p.dt - lap)
    y = o.matvec(x.ravel()).reshape(n, n, n)
    assert np.abs(y - yref).max() <= 1e-10 * np.abs(yref).max()
    assert np.abs(o.rhs()).max() == 0.0  # constant Te: no flux divergence
    o.close()


def test_field_along_x_is_1d_diffusion():
    n = 16
    dx = 1.0 / n
    Te = np.ones(n ** 3)
    b = np.tile([1.0, 0.0, 0.0], (n ** 3, 1))
    used = np.ones(n ** 3, dtype=np.uint8)
    p = HeatParams(fieldAligned=1.0)
    o = HeatOracle(n, dx, Te, b, used, p)
    x = np.random.default_rng(3).normal(size=(n, n, n))
    xp = pad(x)
    lapx = (xp[1:-1, 1:-1, 2:] + xp[1:-1, 1:-1, :-2] - 2 * x) / dx ** 2
    V = dx ** 3
    yref = V * (x * p.cv / p.dt - lapx)
    y = o.matvec(x.ravel()).reshape(n, n, n)
    assert np.abs(y - yref).max() <= 1e-10 * np.abs(yref).max()
    o.close()


def jacobian_blocks(n, dx, Te, b, used, p):
    """The in-block 7-point matrix of the preconditioner (add_jacobian_heat_cond,
    src/ModHeatConduction.f90:1547-1638), couplings across 8^3 block faces
    and to unused cells dropped, as a scipy matrix in x-fastest order."""
    T3, b3 = Te.reshape(n, n, n), b.reshape(n, n, n, 3)
    u = used.reshape(n, n, n) == 1
    HC = p.heatCondPar * T3 ** 2.5
    V, area = dx ** 3, dx * dx
    Hp, Bp = pad(HC), pad(b3)
    idx = np.arange(n ** 3).reshape(n, n, n)
    rows, cols, vals = [], [], []
    diag = np.full((n, n, n), V * p.cv / p.dt)
    sumJ = np.zeros((n, n, n))
    Coeff = -p.semiImplCoeff * V
    for d in range(3):
        ax = 2 - d
        z = (0, 0, 0)
        # face values of the n+1 faces, then left/right of every cell
        hf = area * (0.5 * (window(Hp, n, d, 0, z) + window(Hp, n, d, 1, z))) * \
            (0.5 * (bb(window(Bp, n, d, 0, z), p.fieldAligned, d, d) + bb(window(Bp, n, d, 1, z), p.fieldAligned, d, d)))
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(None, -1)
        hi[ax] = slice(1, None)
        DL = (1.0 / dx) / V * hf[tuple(lo)]
        DR = (1.0 / dx) / V * hf[tuple(hi)]
        sumJ = sumJ - (DL + DR)
        for side, D in ((-1, DL), (1, DR)):
            nb = np.roll(idx, -side, axis=ax)
            pos = np.indices((n, n, n))[ax]
            inb = ((pos + side) >= 0) & ((pos + side) < n) & ((pos + side) // 8 == pos // 8)
            nbu = np.roll(u, -side, axis=ax)
            m = u & inb & nbu
            rows.append(idx[m])
            cols.append(nb[m])
            vals.append(Coeff * D[m])
    diag = np.where(u, Coeff * sumJ + V * p.cv / p.dt, V * p.cv / p.dt)
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(diag.ravel())
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n ** 3, n ** 3))


def block_perm(n):
    """permutation from x-fastest global order to block order (cells of a
    block contiguous, x fastest inside), the natural ILU order"""
    nR = n // 8
    idx = np.arange(n ** 3).reshape(nR, 8, nR, 8, nR, 8)  # bz k by j bx i
    return idx.transpose(0, 2, 4, 1, 3, 5).ravel()


def test_bilu_solve_matches_triangular_factors():
    n, dx, Te, b, used, p = case(nRoot=2, seed=11)
    o = HeatOracle(n, dx, Te, b, used, p)
    A = jacobian_blocks(n, dx, Te, b, used, p)
    P = block_perm(n)
    Ab = A[P][:, P].tocsr()
    N = n ** 3
    # ILU(0) diagonal by the natural-order recurrence over lower neighbours
    L = sp.tril(Ab, -1).tocsr()
    U = sp.triu(Ab, 1).tocsc()
    d = Ab.diagonal().copy()
    for q in range(N):
        lo, hi = L.indptr[q], L.indptr[q + 1]
        for kk, a in zip(L.indices[lo:hi], L.data[lo:hi]):
            d[q] -= a * Ab[kk, q] / d[kk]
    D = sp.diags(d)
    r = np.random.default_rng(5).normal(size=N)
    y = spl.spsolve_triangular((L + D).tocsr(), r[P], lower=True)
    zb = spl.spsolve_triangular((D + U).tocsr(), D @ y, lower=False)
    zref = np.empty(N)
    zref[P] = zb
    z = o.precond(r)
    assert np.abs(z - zref).max() <= 1e-11 * np.abs(zref).max()
    o.close()


@pytest.mark.parametrize("prec", ["NONE", "BILU"])
def test_solve_reaches_tolerance(prec):
    n, dx, Te, b, used, p = case(nRoot=2, seed=3, typePrecond=prec)
    o = HeatOracle(n, dx, Te, b, used, p)
    bvec = o.rhs()
    r, x, nm, err = o.solve()
    assert r == 0 and err <= p.errorMax and nm > 0
    # the true preconditioned residual of the returned x on a fresh copy
    o2 = HeatOracle(n, dx, Te, b, used, p)
    res = o2.precond(bvec - o2.matvec(x))
    rel = np.linalg.norm(res) / np.linalg.norm(o2.precond(bvec))
    assert rel <= 1.5 * p.errorMax, rel
    te = o.te()
    u = used == 1
    assert np.array_equal(te[~u], Te[~u])
    assert np.abs(te[u] - (Te[u] + x[u])).max() <= 1e-15 * Te.max()
    o.close()
    o2.close()


def test_bilu_needs_fewer_matvecs_than_none():
    res = {}
    for prec in ("NONE", "BILU"):
        n, dx, Te, b, used, p = case(nRoot=2, seed=3, typePrecond=prec)
        o = HeatOracle(n, dx, Te, b, used, p)
        res[prec] = o.solve()[2]
        o.close()
    assert res["BILU"] < res["NONE"], res
