"""Host-side mirror of the reference's semi-implicit heat conduction
(TypeSemiImplicit = 'parcond', src/ModSemiImplicit.f90).

``HeatSolver`` works on the grid of an
:class:`~batsrus_b200.explicit.ExplicitSolver` (all blocks of 8^3 at one
level, float or periodic boundaries):

* ``advance_semi_impl()`` -- one solve of advance_semi_impl (:240): the
  right-hand side, the block ILU(0) preconditioner, left-preconditioned
  GMRES with semi_impl_matvec (:578), then Te += x on used cells; raises
  :class:`~batsrus_b200.capi.BxError` (BX_ERR_KRYLOV) when MaxMatvec is
  reached first, as the reference stops on iError /= 0;
* ``rhs()``, ``matvec(x)``, ``precond(r)`` -- the linear system of the next
  solve; ``te()`` -- the temperature.

Vectors are (nBlock, nK, nJ, nI) arrays in the grid's block order (the
Fortran (nI, nJ, nK, nBlock) layout); bhat has a trailing axis of 3.
"""
import ctypes

import numpy as np

from . import capi
from .capi import check, dptr
from .heat_params import HeatParams  # noqa: F401  (re-export)


class HeatSolver:
    def __init__(self, explicit_solver, params, Te, bhat, used):
        g = explicit_solver.grid
        self.L = capi.load()
        self.params = params
        self.shape = (g.nBlock, g.nK, g.nJ, g.nI)
        Te = np.ascontiguousarray(Te, dtype=np.float64).reshape(self.shape)
        bhat = np.ascontiguousarray(bhat, dtype=np.float64).reshape(self.shape + (3,))
        used = np.ascontiguousarray(used, dtype=np.uint8).reshape(self.shape)
        self._p = capi.heat_params(params)
        check(self.L.bx_heat_init(ctypes.byref(self._p), dptr(Te), dptr(bhat),
                                  used.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))))

    def advance_semi_impl(self):
        s = capi.KrylovStats()
        check(self.L.bx_advance_semi_impl(ctypes.byref(s)))
        return {"nMatvec": s.nMatvec, "iError": s.iError, "Error": s.Error, "Dt": s.Dt, "msStep": s.msStep}

    def _out(self):
        return np.empty(self.shape)

    def te(self):
        t = self._out()
        check(self.L.bx_heat_get_te(dptr(t)))
        return t

    def rhs(self):
        b = self._out()
        check(self.L.bx_heat_get_rhs(dptr(b)))
        return b

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.shape)
        y = self._out()
        check(self.L.bx_heat_matvec(dptr(x), dptr(y)))
        return y

    def precond(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(self.shape)
        z = self._out()
        check(self.L.bx_heat_precond(dptr(r), dptr(z)))
        return z
