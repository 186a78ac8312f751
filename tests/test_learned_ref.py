"""CPU checks of the learned preconditioner's numpy reference (the checker
of the GPU kernels): its backward formulas against central finite
differences of its own loss (FP64, no BF16 rounding), and its BF16
rounding against the definition (round to nearest, ties to even)."""
import numpy as np

import learned_ref as lr


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5e-3, 3.0e38], dtype=np.float32)
    r = lr.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                     # tie -> even mantissa
    assert r[2] == np.float32(1.0 + 4 * 2 ** -8)  # tie -> even (up)
    assert r[3] == 1.0
    assert abs(r[4] - x[4]) <= abs(x[4]) * 2 ** -8
    assert np.isfinite(r[5])


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = lr.init_params(seed=1, out_gain=1.0)
    x0 = rng.normal(size=(2, 8, 8, 8, 16))
    tgt = rng.normal(size=(2, 8, 8, 8, 8))
    loss, g = lr.loss_and_grad(p, x0, tgt, bf=False)
    n = tgt.size
    idx = np.concatenate([rng.choice(np.arange(o, o + s), 6, replace=False)
                          for o, s in zip(np.cumsum([0] + [int(np.prod(s)) for _, s in lr.SHAPES])[:-1],
                                          [int(np.prod(s)) for _, s in lr.SHAPES])])
    p64 = p.astype(np.float64)
    for i in idx:
        h = 1e-5 * max(1.0, abs(p64[i]))
        pp, pm = p64.copy(), p64.copy()
        pp[i] += h
        pm[i] -= h
        lp = ((lr.forward(pp, x0, bf=False)[0] - tgt) ** 2).sum() / n
        lm = ((lr.forward(pm, x0, bf=False)[0] - tgt) ** 2).sum() / n
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-4 * max(1.0, abs(fd)), (i, fd, g[i])
