"""The autotuner (bx_autotune, bx_tune_set): every candidate launch shape of
a knob computes the same result (bit for bit where neither a reduction order
nor a separate instantiation of a kernel is involved, to rounding
otherwise), and bx_autotune picks a candidate of every knob whose context is
ready, times it, and keeps knobs that the caller set."""
import numpy as np
import pytest

from batsrus_b200 import capi, configs
from batsrus_b200.explicit import ExplicitSolver
from batsrus_b200.heat import HeatSolver
from batsrus_b200.heat_params import HeatParams, global_to_blocks, heat_dipole
from batsrus_b200.implicit import ImplicitSolver
from batsrus_b200.param import Scheme

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def fresh_knobs():
    capi.tune_reset()
    yield
    capi.tune_reset()


def test_stage_grid_candidates_bit_identical():
    # 512 blocks of 4^3: several persistent CTAs fit on an SM, and the grid
    # (148 x candidate CTAs, at most 512) differs between the candidates
    g, s, st, _ = configs.uniform_3d_case(8, "Linde", "mc3", 1.2, nCellBlock=(4, 4, 4), state="blast")
    out = {}
    for v in capi.tune_info()["stage_ctas_per_sm"]["candidates"]:
        capi.tune_set("stage_ctas_per_sm", v)
        x = ExplicitSolver(g, s)
        x.set_state(st)
        x.advance(3)
        out[v] = x.get_state()
        x.close()
    ref = out[1]
    for v, a in out.items():
        assert np.array_equal(a, ref), v


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_stage_variants_agree(prec):
    """The three 8^3 stage kernels (one face phase; one direction at a time
    with one or two faces per thread) on a blast state with HLLD and Linde
    and the Koren limiter, on a static AMR grid with resolution changes, and
    in the implicit residual mode: the same state to rounding."""
    out = {}
    cases = []
    for flux in ("Linde", "HLLD"):
        cases.append((flux,) + configs.uniform_3d_case(2, flux, "mc3", 1.2, precision=prec, state="blast")[:3])
    g, s, st, _ = configs.amr_blast(nRoot=2, maxLevel=2, precision=prec)
    cases.append(("amr",) + (g, s, st))
    for name, g, s, st in cases:
        for f in capi.tune_info()["stage_variant"]["candidates"]:
            capi.tune_set("stage_variant", f)
            x = ExplicitSolver(g, s)
            x.set_state(st)
            x.advance(3)
            out[(name, f)] = (x.get_state(), x.time())
            x.close()
        # the instantiations may contract multiply-adds differently, so the
        # variants agree to rounding
        for f in (0, 2, 3):
            a, b = out[(name, f)][0], out[(name, 1)][0]
            rel = np.abs(a - b).max() / np.abs(b).max()
            assert rel <= (1e-13 if prec == "fp64" else 1e-5), (name, f, rel)
            assert abs(out[(name, f)][1][0] - out[(name, 1)][1][0]) <= 1e-12 * abs(out[(name, 1)][1][0])
    capi.tune_set("stage_variant", 0)


def heat_case(nRoot=2, prec="BILU"):
    """solver, heat solver and the block-layout fields (Te, bhat, used)"""
    g, Te, b, used, dx = heat_dipole(nRoot=nRoot, seed=9)
    n = 8 * nRoot
    tb = lambda a: global_to_blocks(a.reshape((n, n, n) + a.shape[1:]), nRoot)
    fields = (tb(Te), tb(b), tb(used))
    x = ExplicitSolver(g, Scheme())
    h = HeatSolver(x, HeatParams(typePrecond=prec), *fields)
    return x, h, fields


def test_heat_ilu_warps_bit_identical():
    x, h, _ = heat_case(nRoot=4)  # 512 blocks: 16 groups of 32
    r = np.random.default_rng(3).normal(size=h.shape)
    out = {}
    for w in capi.tune_info()["heat_ilu_warps"]["candidates"]:
        capi.tune_set("heat_ilu_warps", w)
        out[w] = h.precond(r)
    for w, z in out.items():
        assert np.array_equal(z, out[1]), w
    x.close()


def test_bilu_threads_bit_identical():
    g, s, p, st = configs.jfnk_ot(nRoot=2, precond="BILU")
    x = ExplicitSolver(g, s)
    x.set_state(st)
    im = ImplicitSolver(x, p)
    im.advance_part_impl()  # sets the time step
    im.advance_part_impl()  # builds the Jacobian and its BILU
    r = np.random.default_rng(4).normal(size=g.nCell * 8)
    out = {}
    for v in capi.tune_info()["bilu_threads"]["candidates"]:
        capi.tune_set("bilu_threads", v)
        out[v] = im.precond(r)
    for v, z in out.items():
        assert np.array_equal(z, out[0]), v
    x.close()


def test_krylov_grid_and_unroll_agree_to_rounding():
    x, h, (Te0, b, used) = heat_case(nRoot=3)
    res = {}
    for c, u in ((2, 1), (8, 4)):
        capi.tune_set("krylov_ctas_per_sm", c)
        capi.tune_set("krylov_unroll", u)
        h2 = HeatSolver(x, HeatParams(), Te0, b, used)
        s = h2.advance_semi_impl()
        res[(c, u)] = (s["nMatvec"], h2.te())
    (n1, t1), (n2, t2) = res.values()
    assert abs(n1 - n2) <= 1
    dT = np.abs(t1 - Te0).max()
    assert np.abs(t1 - t2).max() <= 1e-9 * dT
    x.close()


def test_autotune_picks_candidates_and_keeps_caller_choice():
    x, h, _ = heat_case(nRoot=4)
    capi.tune_set("krylov_unroll", 1)
    knobs = x.autotune()
    for name in ("stage_ctas_per_sm", "stage_variant", "krylov_ctas_per_sm", "heat_ilu_warps"):
        k = knobs[name]
        assert k["tuned"] == 1 and k["value"] in k["candidates"], (name, k)
        assert all(m > 0 for m in k["ms"]), (name, k)
        assert k["ms"][k["candidates"].index(k["value"])] == min(k["ms"]), (name, k)
    assert knobs["krylov_unroll"]["tuned"] == 2 and knobs["krylov_unroll"]["value"] == 1
    assert knobs["bilu_threads"]["tuned"] == 0  # no implicit context
    s = h.advance_semi_impl()  # the tuned shapes run
    assert s["iError"] == 0
    x.close()


def test_multi_step_gram_schmidt_agrees_with_one_step():
    """krylov_gs_steps = 2, 3, 4 (Gram-Schmidt steps per pass over w) give
    the same heat solve as one step per pass, to rounding"""
    x, h, (Te0, b, used) = heat_case(nRoot=3)
    res = {}
    for steps in (1, 2, 3, 4):
        capi.tune_set("krylov_gs_steps", steps)
        h2 = HeatSolver(x, HeatParams(), Te0, b, used)
        s = h2.advance_semi_impl()
        res[steps] = (s["nMatvec"], h2.te(), s["Error"])
    n1, t1, e1 = res[1]
    dT = np.abs(t1 - Te0).max()
    for steps in (2, 3, 4):
        n2, t2, e2 = res[steps]
        assert abs(n1 - n2) <= 1 and e2 <= 1e-6, steps
        assert np.abs(t1 - t2).max() <= 1e-9 * dT, steps
    x.close()
