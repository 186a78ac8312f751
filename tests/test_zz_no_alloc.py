"""bx_impl_norm_noalloc (no device allocation, static scratch) against the
Norm_V of the implicit step (bx_impl_get_rhs), called twice in a row on a
device copy of the step's starting state in the reference's Impl_VGB order.
Named to run after the other tests; it also passes alone."""
import ctypes

import numpy as np
import pytest

from batsrus_b200 import capi, configs
from batsrus_b200.explicit import ExplicitSolver
from batsrus_b200.implicit import ImplicitSolver
from batsrus_b200.implicit_params import ImplicitParams

pytestmark = pytest.mark.gpu


def impl_vgb(state, grid, gamma):
    """Implicit variables (energy instead of pressure) of the physical cells,
    Impl_VGB order: [block][k][j][i][var]."""
    u = state[grid.interior_slices()].copy()
    rho = u[..., 0]
    ke = 0.5 * (u[..., 1] ** 2 + u[..., 2] ** 2 + u[..., 3] ** 2) / rho
    me = 0.5 * (u[..., 4] ** 2 + u[..., 5] ** 2 + u[..., 6] ** 2)
    u[..., 7] = u[..., 7] / (gamma - 1.0) + ke + me
    return np.ascontiguousarray(u)


def test_norm_noalloc_matches_the_implicit_step():
    import torch

    g, s, st, _ = configs.uniform_3d_case(2, "Linde", "mc3", 1.2, state="pert")
    x = ExplicitSolver(g, s)
    x.set_state(st)
    im = ImplicitSolver(x, ImplicitParams(typePrecond="BILU"))
    im.advance_part_impl()            # Dt = 0 step
    u0 = x.get_state()                # the next step starts from this state
    im.advance_part_impl()
    _, norm_ref = im.rhs()
    x.close()

    dev = torch.from_numpy(impl_vgb(u0, g, s.gamma)).cuda()
    L = capi.load()
    out = []
    for _ in range(2):
        n = np.empty(8)
        capi.check(L.bx_impl_norm_noalloc(ctypes.c_void_p(dev.data_ptr()), g.nCellBlock, g.nBlock, None,
                                          capi.dptr(n)))
        out.append(n)
    for n in out:
        assert np.abs(n - norm_ref).max() <= 1e-12 * np.abs(norm_ref).max(), (n, norm_ref)

    # beyond the static scratch: a clear argument error, nothing launched
    n = np.empty(8)
    r = L.bx_impl_norm_noalloc(ctypes.c_void_p(dev.data_ptr()), g.nCellBlock, capi.NOALLOC_MAX_BLOCK + 1, None,
                               capi.dptr(n))
    assert r == 1 and b"BX_NOALLOC_MAX_BLOCK" in L.bx_last_error()
