"""GPU checks of the learned per-block preconditioner (tcgen05 kernels)
against the numpy reference oracle/learned_ref.py, through the C ABI:

* the inference kernel on random blocks and parameters;
* the training gradient (forward, backward-data and weight-gradient
  kernels) on random samples;
* training lowers the loss on a learnable synthetic target;
* FGMRES with the trained network (linear mode, identity part plus the
  learned remainder at blend 0.25): the implicit steps converge to the
  Krylov tolerance and agree with the BILU steps to that tolerance; the
  Krylov counts with and without the network are measured, and the network
  may cost at most 20 % more iterations than the unpreconditioned solver
  (it gains a few per cent on this workload, see the bench's JFNK line).

Tolerances: both sides use the same BF16-rounded operands; the GPU sums in
FP32 (the reference in FP64) and an intermediate activation can round to a
neighbouring BF16 value, so outputs agree to ~1e-3 relative (test 1e-2) and
gradients to ~1e-2 (test 3e-2 per parameter group).
"""
import numpy as np
import pytest

import learned_ref as lr
from batsrus_b200 import configs
from batsrus_b200.explicit import ExplicitSolver
from batsrus_b200.implicit import ImplicitSolver
from batsrus_b200.learned import LearnedPreconditioner

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


@pytest.fixture
def net():
    n = LearnedPreconditioner(nSampleMax=4096, seed=11)
    yield n
    n.close()


@pytest.fixture
def net_relu():
    n = LearnedPreconditioner(nSampleMax=4096, seed=11, relu=True)
    yield n
    n.close()


@pytest.mark.parametrize("relu", [True, False])
def test_apply_matches_reference(relu):
    net = LearnedPreconditioner(nSampleMax=64, seed=11, relu=relu)
    rng = np.random.default_rng(1)
    p = lr.init_params(seed=3, out_gain=1.0).astype(np.float32)
    if not relu:
        P = lr.unpack(p)
        P["W1"][:, 8:, :] = 0.0
        for k in ("b1", "b2", "b3"):
            P[k][:] = 0.0
        p = lr.pack(P)
    net.set_params(p)
    nb = 7
    v = rng.normal(size=(nb, 8, 512)) * 10.0 ** rng.uniform(-3, 3, size=(nb, 1, 1))
    v[3] = 0.0  # an all-zero block maps to zero
    feat = rng.normal(size=(nb, 512, 8)).astype(np.float32)
    z = net.apply_blocks(v, feat)
    zr = lr.apply(p, v, feat, relu=relu)
    net.close()
    assert np.all(z[3] == 0.0)
    for b in range(nb):
        if b != 3:
            assert relerr(z[b], zr[b]) < 1e-2, (b, relerr(z[b], zr[b]))
    if not relu:  # the linear mode is linear in v
        z2 = 2.0 * z[0]
        assert relerr(z2, 2.0 * zr[0]) < 1e-2


@pytest.mark.parametrize("relu", [True, False])
def test_gradient_matches_reference(relu):
    net = LearnedPreconditioner(nSampleMax=64, seed=11, relu=relu)
    rng = np.random.default_rng(2)
    p = lr.init_params(seed=4, out_gain=1.0).astype(np.float32)
    net.set_params(p)
    n = 5
    x0 = rng.normal(size=(n, 512, 16)).astype(np.float32)
    tgt = rng.normal(size=(n, 512, 8)).astype(np.float32)
    net.set_samples(x0, tgt)
    loss, g = net.gradient(0, n)
    net.close()
    lref, gref = lr.loss_and_grad(p, x0.reshape(n, 8, 8, 8, 16), tgt.reshape(n, 8, 8, 8, 8), bf=True, relu=relu)
    assert abs(loss - lref) <= 1e-3 * lref
    o = 0
    for name, shp in lr.SHAPES:
        k = int(np.prod(shp))
        if np.linalg.norm(gref[o:o + k]) == 0.0:
            assert np.all(g[o:o + k] == 0.0), name
        else:
            assert relerr(g[o:o + k], gref[o:o + k]) < 3e-2, (name, relerr(g[o:o + k], gref[o:o + k]))
        o += k


def test_training_lowers_the_loss(net_relu):
    net = net_relu
    # learnable target: a fixed random network of the same shape
    rng = np.random.default_rng(3)
    teacher = lr.init_params(seed=9, out_gain=1.0)
    n = 1024
    x0 = rng.normal(size=(n, 512, 16)).astype(np.float32)
    tgt, _, _ = lr.forward(teacher, x0.reshape(n, 8, 8, 8, 16))
    net.set_samples(x0, tgt.reshape(n, 512, 8).astype(np.float32))
    first, last = net.train(nEpoch=12, batch=128, lr=3e-3)
    assert np.isfinite(first) and np.isfinite(last)
    assert last < 0.7 * first, (first, last)


def _jfnk(prec, state, net=None, steps=3):
    g, s, p, _ = configs.jfnk_ot(nRoot=4, precond=prec, with_state=False)
    x = ExplicitSolver(g, s)
    x.set_state(state)
    im = ImplicitSolver(x, p)
    out = [im.advance_part_impl() for _ in range(steps)]
    st = x.get_state()
    x.close()
    return out, st, g


def test_learned_fgmres_converges_and_gains():
    """The trained network in the FGMRES of advance_part_impl at 32^3: it
    converges to the tolerance with the BILU answer, and needs fewer Krylov
    matvecs than the same solver without a preconditioner.  Training as in
    the benchmark: (v, BILU(v)) pairs of 16 blocks each, half from the Krylov
    vectors of BILU-preconditioned steps of a differently seeded state, half
    from probe vectors at its last state, then 8 epochs of Adam."""
    from batsrus_b200.capi import BxError
    g, s, p, st = configs.jfnk_ot(nRoot=4, precondPrecision="fp32")
    _, _, _, st2 = configs.jfnk_ot(nRoot=4, seed=2025)
    nPair, bpp = 2000, 16
    net = LearnedPreconditioner(nSampleMax=nPair * bpp, seed=2024)
    x = ExplicitSolver(g, s)
    x.set_state(st2)
    im = ImplicitSolver(x, p)
    net.collect(bpp)
    for _ in range(100):
        if net.num_samples() >= (nPair // 2) * bpp:
            break
        try:
            im.advance_part_impl()
        except BxError:  # a failed solve ends the collection
            break
    net.collect(0)
    net.collect_probes(nPair - net.num_samples() // bpp, bpp, seed=2025)
    x.close()
    assert net.num_samples() == nPair * bpp
    first, last = net.train(nEpoch=8, batch=256, lr=1e-3)
    assert last < first
    net.set_blend(0.5)
    bilu, sb, g = _jfnk("BILU", st)
    none, sn, _ = _jfnk("NONE", st)
    lrn, sl, _ = _jfnk("LEARNED", st)
    isl = g.interior_slices()
    for q in lrn:
        assert q["iError"] == 0 and q["Error"] <= 1e-3
    # same answer to the Krylov tolerance
    du = np.abs(sb[isl] - st[isl]).max()
    assert np.abs(sl[isl] - sb[isl]).max() <= 2e-2 * du
    # the Krylov counts with and without the network
    nl, nn = sum(q["nMatvec"] for q in lrn[1:]), sum(q["nMatvec"] for q in none[1:])
    print("matvecs learned %d, none %d, bilu %d" % (nl, nn, sum(q["nMatvec"] for q in bilu[1:])))
    # the gain of the trained network over the same solver without it
    assert nl < nn, ([q["nMatvec"] for q in lrn], [q["nMatvec"] for q in none])
    net.close()
