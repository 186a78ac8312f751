"""GPU parity of the implicit JFNK step against the CPU oracle through the C
ABI: the normalised Krylov system (Rhs, Norm_V), the matrix-free product,
the BILU preconditioner, and whole implicit steps (Krylov iteration count
and state).

Tolerances: Rhs, Norm_V and the matrix-free product are FP64 evaluations of
the same formulas (1e-10 relative; the finite-difference product divides a
residual difference by eps = 1e-6/rms(x), which amplifies rounding by 1e6).
The preconditioner is compared at 1e-10.  A whole step solves the linear
system to the Krylov tolerance 1e-3; with one Gram-Schmidt step per pass
(krylov_gs_steps = 1, the oracle's modified Gram-Schmidt) the GPU and
oracle iterates differ only by the summation order of the FP64 inner
products, so the step results (state and the time, whose next step is taken
from the new state) agree to 1e-8 relative and the matrix-vector counts
agree within one.  The default two steps per pass rounds the Krylov
coefficients differently; it is compared with one step per pass to 1e-6,
far inside the Krylov tolerance.
"""
import numpy as np
import pytest

from batsrus_b200 import capi, configs
from batsrus_b200.explicit import ExplicitSolver
from batsrus_b200.implicit import ImplicitSolver
from batsrus_b200.implicit_params import ImplicitParams
from oracle import Oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def pair(prec="BILU", nRoot=2, state="pert", bdf2=True, precondPrecision="fp64"):
    g, s, st, _ = configs.uniform_3d_case(nRoot, "Linde", "mc3", 1.2, state=state)
    p = ImplicitParams(typePrecond=prec, useBdf2=bdf2, precondPrecision=precondPrecision)
    o = Oracle(g, s)
    o.set_state(st)
    o.exchange_messages()
    o.set_implicit(p)
    x = ExplicitSolver(g, s)
    x.set_state(st)
    im = ImplicitSolver(x, p)
    return g, o, x, im


@pytest.fixture
def one_step_gram_schmidt():
    capi.tune_set("krylov_gs_steps", 1)
    yield
    capi.tune_reset()


@pytest.mark.parametrize("prec", ["BILU", "NONE"])
def test_gpu_jfnk_steps_match_oracle(prec, one_step_gram_schmidt):
    g, o, x, im = pair(prec)
    isl = g.interior_slices()
    for step in range(4):
        stats = im.advance_part_impl()
        r, nm, err = o.advance_implicit()
        assert r == 0 and stats["iError"] == 0
        assert abs(stats["nMatvec"] - nm) <= 1, (step, stats["nMatvec"], nm)
        # the next time step is taken from the new state, which agrees with
        # the oracle's to the Krylov-iterate level, so the time does too
        to, dto, no = o.time()
        tg, _, ng = x.time()
        assert ng == no and abs(tg - to) <= 1e-8 * max(to, 1.0), (step, tg, to)
        assert rel(x.get_state()[isl], o.get_state()[isl]) < 1e-8, step


def test_gpu_jfnk_system_matches_oracle():
    g, o, x, im = pair("BILU")
    im.advance_part_impl()
    o.advance_implicit()
    im.advance_part_impl()
    o.advance_implicit()
    rg, ng = im.rhs()
    ro, no = o.impl_rhs()
    assert rel(ng, no) < 1e-12
    assert rel(rg, ro) < 1e-10
    rng = np.random.default_rng(3)
    v = rng.normal(size=rg.size)
    assert rel(im.matvec(v), o.impl_matvec(v)) < 1e-8
    assert rel(im.precond(v), o.impl_precond(v)) < 1e-10
    # the Krylov solution satisfies the tolerance on the oracle's operator
    xs = im.x()
    res = o.impl_matvec(xs) - ro
    assert np.linalg.norm(res) <= 1.2e-3 * np.linalg.norm(ro)


def test_gpu_jfnk_fp32_factors(one_step_gram_schmidt):
    """BILU factors in FP32: the FP64 Jacobian stored in FP32, factorised in
    FP32 (D^-1 and the premultiplied D^-1 A of the backward sweep), the
    sweeps in FP64 arithmetic.
    The apply agrees with the oracle's FP64 BILU to 1e-6 relative: FP32
    rounding (6e-8) of the blocks and of the factorisation, grown by the
    condition of the 8x8 pivots.  A preconditioner only steers the flexible
    GMRES: every step's matrix-vector count stays within two of the
    oracle's, its Krylov solution satisfies the tolerance 1e-3 on the
    oracle's operator, and the states agree to 1e-6 relative, far inside
    the Krylov tolerance of the update."""
    g, o, x, im = pair("BILU", precondPrecision="fp32")
    isl = g.interior_slices()
    for step in range(4):
        stats = im.advance_part_impl()
        r, nm, err = o.advance_implicit()
        assert r == 0 and stats["iError"] == 0
        assert abs(stats["nMatvec"] - nm) <= 2, (step, stats["nMatvec"], nm)
        assert rel(x.get_state()[isl], o.get_state()[isl]) < 1e-6, step
    rg, _ = im.rhs()
    ro, _ = o.impl_rhs()
    v = np.random.default_rng(3).normal(size=rg.size)
    assert rel(im.precond(v), o.impl_precond(v)) < 1e-6
    res = o.impl_matvec(im.x()) - ro
    assert np.linalg.norm(res) <= 1.2e-3 * np.linalg.norm(ro)
    x.close()


def test_gpu_jfnk_bf16_factors(one_step_gram_schmidt):
    """BILU factors stored in BF16 (FP64 Jacobian, FP32 factorisation, FP64
    sweeps): the apply within 2e-2 of the oracle's FP64 BILU (BF16 keeps 8
    significant bits, 2e-3 per entry, grown by the condition of the 8x8
    pivots; 5.5e-3 measured here).  Such a preconditioner changes the path
    of FGMRES, not the system it solves: the first implicit step's Krylov
    solution meets the tolerance 1e-3 on the oracle's operator (the states
    are identical before it), every step converges with the
    matrix-vector count within two of the oracle's, and the states stay
    within 5e-3 of the oracle's (steps solved to 1e-3 by different Krylov
    iterates; 8e-4 measured)."""
    g, o, x, im = pair("BILU", precondPrecision="bf16")
    isl = g.interior_slices()
    for step in range(4):
        stats = im.advance_part_impl()
        r, nm, err = o.advance_implicit()
        assert r == 0 and stats["iError"] == 0 and stats["Error"] <= 1e-3
        assert abs(stats["nMatvec"] - nm) <= 2, (step, stats["nMatvec"], nm)
        if step == 1:
            res = o.impl_matvec(im.x()) - o.impl_rhs()[0]
            assert np.linalg.norm(res) <= 1.2e-3 * np.linalg.norm(o.impl_rhs()[0])
        assert rel(x.get_state()[isl], o.get_state()[isl]) < 5e-3, step
    rg, _ = im.rhs()
    v = np.random.default_rng(3).normal(size=rg.size)
    assert rel(im.precond(v), o.impl_precond(v)) < 2e-2
    x.close()


def test_gpu_jfnk_first_step_only_sets_the_time_step():
    g, o, x, im = pair("BILU")
    st0 = x.get_state()
    stats = im.advance_part_impl()
    assert stats["Dt"] == 0.0 and stats["nMatvec"] == 0
    isl = g.interior_slices()
    assert rel(x.get_state()[isl], st0[isl]) < 1e-14


@pytest.mark.parametrize("prec,steps_per_pass", [("BILU", 2), ("NONE", 2), ("BILU", 3), ("NONE", 4)])
def test_multi_step_gram_schmidt_steps_agree_with_one_step(prec, steps_per_pass):
    """krylov_gs_steps = 2..4 against 1: the same implicit steps to 1e-6
    relative and the matrix-vector counts within one per step"""
    out = {}
    for steps in (1, steps_per_pass):
        capi.tune_set("krylov_gs_steps", steps)
        g, o, x, im = pair(prec)
        stats = [im.advance_part_impl() for _ in range(4)]
        out[steps] = ([q["nMatvec"] for q in stats], x.get_state()[g.interior_slices()])
        x.close()
    capi.tune_reset()
    (n1, s1), (n2, s2) = out[1], out[steps_per_pass]
    assert all(abs(a - b) <= 1 for a, b in zip(n1, n2)), (n1, n2)
    assert rel(s2, s1) < 1e-6
