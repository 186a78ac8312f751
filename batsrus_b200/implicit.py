"""Host-side mirror of the reference's implicit step interface.

``ImplicitSolver`` adds the full implicit JFNK step to an
:class:`~batsrus_b200.explicit.ExplicitSolver` (the same grid and state):

* ``advance_part_impl(TimeSimulationLimit)`` -- one BATS_advance step with
  advance_part_impl (src/ModPartImplicit.f90:322);
* ``rhs()``, ``matvec(x)``, ``precond(r)``, ``x()`` -- the normalised Krylov
  system of the last step in the reference's Rhs_I order (variable fastest,
  then cells, then blocks): impl_newton_init (:816), impl_matvec_free
  (:1144), the preconditioner, and the Krylov solution.
"""
import ctypes

import numpy as np

from . import capi
from .capi import check, dptr
from .implicit_params import ImplicitParams  # noqa: F401  (re-export)


class ImplicitSolver:
    def __init__(self, explicit_solver, params):
        self.x_ = explicit_solver
        self.L = capi.load()
        self.params = params
        self._p = capi.implicit_params(params)
        check(self.L.bx_implicit_init(ctypes.byref(self._p)))
        self.n = explicit_solver.grid.nCell * 8

    def advance_part_impl(self, TimeSimulationLimit=-1.0):
        s = capi.KrylovStats()
        check(self.L.bx_advance_part_impl(TimeSimulationLimit, ctypes.byref(s)))
        return {"nMatvec": s.nMatvec, "iError": s.iError, "Error": s.Error, "Dt": s.Dt,
                "msStep": s.msStep, "msPrecondSetup": s.msPrecondSetup}

    def rhs(self):
        r, nrm = np.empty(self.n), np.empty(8)
        check(self.L.bx_impl_get_rhs(dptr(r), dptr(nrm)))
        return r, nrm

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        check(self.L.bx_impl_matvec(dptr(x), dptr(y)))
        return y

    def precond(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        check(self.L.bx_impl_precond(dptr(r), dptr(z)))
        return z

    def x(self):
        out = np.empty(self.n)
        check(self.L.bx_impl_get_x(dptr(out)))
        return out
