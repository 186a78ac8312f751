"""ctypes wrapper of the CPU parity oracle (oracle/bx_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  The oracle
restates the BATS-R-US "orig" explicit path (src/ModFaceValue.f90,
src/ModFaceFlux.f90, src/ModCalcSource.f90, src/ModUpdateState.f90,
src/ModTimeStepControl.f90, src/ModAdvanceExplicit.f90).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")

FLUX = {"rusanov": 0, "linde": 1, "hlld": 2, "roe": 3}
LIMITER = {"minmod": 0, "mc": 1, "mc3": 2, "koren": 2, "no": 0}
BC = {"float": 0, "periodic": 1}


class OraConfig(ctypes.Structure):
    _fields_ = [
        ("nDim", ctypes.c_int),
        ("nI", ctypes.c_int), ("nJ", ctypes.c_int), ("nK", ctypes.c_int),
        ("nRoot", ctypes.c_int * 3),
        ("xyzMin", ctypes.c_double * 3), ("xyzMax", ctypes.c_double * 3),
        ("typeBc", ctypes.c_int * 6),
        ("nOrder", ctypes.c_int), ("nStage", ctypes.c_int),
        ("typeFlux", ctypes.c_int), ("typeLimiter", ctypes.c_int),
        ("limiterBeta", ctypes.c_double),
        ("cfl", ctypes.c_double), ("gamma", ctypes.c_double),
        ("useDivbSource", ctypes.c_int),
        ("useDtFixed", ctypes.c_int), ("dtFixed", ctypes.c_double),
        ("useHalfStep", ctypes.c_int),
        ("nThread", ctypes.c_int),
        ("useNonConservative", ctypes.c_int),
        ("rhoMin", ctypes.c_double), ("pMin", ctypes.c_double), ("tMin", ctypes.c_double),
        ("massIon", ctypes.c_double),
        ("useTvdResChange", ctypes.c_int), ("betaLimiterResChange", ctypes.c_double),
        ("nFaceLimiterResChange", ctypes.c_int),
    ]


def build():
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(_HERE, f) for f in ("bx_oracle.cpp", "bx_oracle.h")]
        if not os.path.exists(_LIB) or any(os.path.getmtime(f) > os.path.getmtime(_LIB) for f in srcs):
            build()
        L = ctypes.CDLL(_LIB)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.ora_new.restype = vp
        L.ora_new.argtypes = [ctypes.POINTER(OraConfig), ctypes.c_int, ip]
        L.ora_free.argtypes = [vp]
        L.ora_state_size.restype = ctypes.c_long
        L.ora_state_size.argtypes = [vp]
        for name in ("ora_set_state", "ora_get_state", "ora_get_source"):
            getattr(L, name).argtypes = [vp, dp]
        L.ora_exchange_messages.argtypes = [vp]
        L.ora_advance.restype = ctypes.c_int
        L.ora_advance.argtypes = [vp, ctypes.c_double]
        L.ora_advance_n.restype = ctypes.c_int
        L.ora_advance_n.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        L.ora_get_time.argtypes = [vp, dp, dp, ip]
        L.ora_set_time.argtypes = [vp, ctypes.c_double, ctypes.c_int]
        for name in ("ora_calc_face_value", "ora_calc_face_flux", "ora_calc_source",
                     "ora_calc_timestep"):
            getattr(L, name).argtypes = [vp, ctypes.c_int]
        L.ora_get_face_values.argtypes = [vp, ctypes.c_int, dp, dp]
        L.ora_get_face_flux.argtypes = [vp, ctypes.c_int, dp]
        L.ora_get_dtmax.argtypes = [vp, dp, dp]
        L.ora_set_owned.argtypes = [vp, ip]
        L.ora_local_dtmin.restype = ctypes.c_double
        L.ora_local_dtmin.argtypes = [vp]
        L.ora_begin_step.argtypes = [vp, ctypes.c_double, ctypes.c_double]
        L.ora_stage.restype = ctypes.c_int
        L.ora_stage.argtypes = [vp, ctypes.c_int]
        L.ora_end_step.argtypes = [vp, ctypes.c_double]
        L.ora_recompute_timestep.restype = ctypes.c_int
        L.ora_recompute_timestep.argtypes = [vp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """One oracle grid.  ``scheme`` and ``grid`` use the same keys as
    :class:`batsrus_b200.session.Scheme` / :class:`batsrus_b200.grid.BlockGrid`."""

    NVAR = 8

    def __init__(self, grid, scheme, n_thread=0):
        c = OraConfig()
        c.nDim = grid.nDim
        c.nI, c.nJ, c.nK = grid.nI, grid.nJ, grid.nK
        for d in range(3):
            c.nRoot[d] = grid.nRoot[d]
            c.xyzMin[d] = grid.xyzMin[d]
            c.xyzMax[d] = grid.xyzMax[d]
        for s in range(6):
            c.typeBc[s] = BC[grid.typeBc[s]]
        c.nOrder = scheme.nOrder
        c.nStage = scheme.nStage
        c.typeFlux = FLUX[scheme.typeFlux.lower()]
        c.typeLimiter = LIMITER[scheme.typeLimiter.lower()]
        c.limiterBeta = scheme.limiterBeta
        c.cfl = scheme.cfl
        c.gamma = scheme.gamma
        c.useDivbSource = int(scheme.useDivbSource)
        c.useDtFixed = int(scheme.useDtFixed)
        c.dtFixed = scheme.dtFixed
        c.useHalfStep = int(scheme.useHalfStep)
        c.nThread = n_thread
        c.useNonConservative = int(getattr(scheme, "useNonConservative", False))
        c.rhoMin = getattr(scheme, "rhoMin", -1.0)
        c.pMin = getattr(scheme, "pMin", -1.0)
        c.tMin = getattr(scheme, "tMin", -1.0)
        c.massIon = getattr(scheme, "massIon", 1.0)
        c.useTvdResChange = int(getattr(scheme, "useTvdResChange", True))
        c.betaLimiterResChange = getattr(scheme, "betaLimiterResChange", 2.0)
        c.nFaceLimiterResChange = getattr(scheme, "nFaceLimiterResChange", 2)
        self.cfg = c
        self.grid = grid
        lc = np.ascontiguousarray(grid.iLevelCoord, dtype=np.int32)
        self.h = lib().ora_new(ctypes.byref(c), grid.nBlock,
                               lc.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        self.shape = grid.state_shape_fortran()  # (nBlock, nKg, nJg, nIg, nVar)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ora_free(self.h)
            self.h = None

    def set_state(self, State_VGB):
        a = np.ascontiguousarray(State_VGB, dtype=np.float64)
        assert a.size == lib().ora_state_size(self.h)
        lib().ora_set_state(self.h, _dp(a))

    def get_state(self):
        a = np.empty(self.shape, dtype=np.float64)
        lib().ora_get_state(self.h, _dp(a))
        return a

    def exchange_messages(self):
        lib().ora_exchange_messages(self.h)

    def advance(self, n=1, t_limit=-1.0):
        err = lib().ora_advance_n(self.h, n, t_limit)
        if err:
            raise RuntimeError("oracle advance failed (HLLD negative density ratio)")

    # one rank of a partitioned grid (batsrus_b200.shard)
    def set_owned(self, owned):
        a = np.ascontiguousarray(owned, dtype=np.int32)
        lib().ora_set_owned(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))

    def local_dtmin(self):
        return lib().ora_local_dtmin(self.h)

    def begin_step(self, dt_min_global, t_limit=-1.0):
        lib().ora_begin_step(self.h, dt_min_global, t_limit)

    def stage(self, i_stage):
        if lib().ora_stage(self.h, i_stage):
            raise RuntimeError("oracle stage failed (HLLD negative density ratio)")

    def end_step(self, t_limit=-1.0):
        lib().ora_end_step(self.h, t_limit)

    def recompute_timestep(self):
        """cell time steps of the current state, no update (after a regrid)"""
        if lib().ora_recompute_timestep(self.h):
            raise RuntimeError("oracle time step failed (HLLD negative density ratio)")

    def time(self):
        t, dt, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        lib().ora_get_time(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(n))
        return t.value, dt.value, n.value

    def set_time(self, t, n_step):
        lib().ora_set_time(self.h, t, n_step)

    # per-block orig routines (iBlock 1-based)
    def calc_face_value(self, iBlock):
        lib().ora_calc_face_value(self.h, iBlock)

    def calc_face_flux(self, iBlock):
        lib().ora_calc_face_flux(self.h, iBlock)

    def calc_source(self, iBlock):
        lib().ora_calc_source(self.h, iBlock)

    def face_values(self, iDim):
        g = self.grid
        n = [g.nI, g.nJ, g.nK]
        n[iDim] += 1
        L = np.empty((n[2], n[1], n[0], self.NVAR))
        R = np.empty_like(L)
        lib().ora_get_face_values(self.h, iDim, _dp(L), _dp(R))
        return L, R

    def face_flux(self, iDim):
        g = self.grid
        n = [g.nI, g.nJ, g.nK]
        n[iDim] += 1
        F = np.empty((n[2], n[1], n[0], 11))
        lib().ora_get_face_flux(self.h, iDim, _dp(F))
        return F

    def source(self):
        g = self.grid
        S = np.empty((g.nK, g.nJ, g.nI, self.NVAR + 1))
        lib().ora_get_source(self.h, _dp(S))
        return S


class OraImplConfig(ctypes.Structure):
    _fields_ = [
        ("cflImpl", ctypes.c_double), ("implCoeff0", ctypes.c_double), ("useBdf2", ctypes.c_int),
        ("nOrderImpl", ctypes.c_int), ("typeFluxImpl", ctypes.c_int), ("jacobianEps", ctypes.c_double),
        ("nKrylovVector", ctypes.c_int), ("maxMatvec", ctypes.c_int), ("errorMax", ctypes.c_double),
        ("typePrecond", ctypes.c_int),
    ]


PRECOND = {"none": 0, "bilu": 1}


def _impl_lib():
    L = lib()
    if not hasattr(L, "_impl_ready"):
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.ora_set_implicit.argtypes = [vp, ctypes.POINTER(OraImplConfig)]
        L.ora_advance_implicit.restype = ctypes.c_int
        L.ora_advance_implicit.argtypes = [vp, ctypes.c_double, ip, dp]
        L.ora_impl_get_rhs.argtypes = [vp, dp, dp]
        L.ora_impl_matvec.argtypes = [vp, dp, dp]
        L.ora_impl_precond.argtypes = [vp, dp, dp]
        L.ora_impl_get_x.argtypes = [vp, dp]
        L._impl_ready = True
    return L


def implicit_config(impl):
    """``impl`` uses the keys of batsrus_b200.implicit.ImplicitParams"""
    c = OraImplConfig()
    c.cflImpl = impl.cflImpl
    c.implCoeff0 = impl.implCoeff0
    c.useBdf2 = int(impl.useBdf2)
    c.nOrderImpl = impl.nOrderImpl
    c.typeFluxImpl = -1 if impl.typeFluxImpl in (None, "default") else FLUX[impl.typeFluxImpl.lower()]
    c.jacobianEps = impl.jacobianEps
    c.nKrylovVector = impl.nKrylovVector
    c.maxMatvec = impl.maxMatvec
    c.errorMax = impl.errorMax
    c.typePrecond = PRECOND[impl.typePrecond.lower()] if impl.typePrecond.lower() in PRECOND else 1
    return c


def _oracle_set_implicit(self, impl):
    self._icfg = implicit_config(impl)
    _impl_lib().ora_set_implicit(self.h, ctypes.byref(self._icfg))
    self.nvec = self.grid.nCell * self.NVAR


def _oracle_advance_implicit(self, t_limit=-1.0):
    n, e = ctypes.c_int(), ctypes.c_double()
    r = _impl_lib().ora_advance_implicit(self.h, t_limit, ctypes.byref(n), ctypes.byref(e))
    return r, n.value, e.value


def _oracle_impl_rhs(self):
    rhs, norm = np.empty(self.nvec), np.empty(8)
    _impl_lib().ora_impl_get_rhs(self.h, _dp(rhs), _dp(norm))
    return rhs, norm


def _oracle_impl_matvec(self, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    _impl_lib().ora_impl_matvec(self.h, _dp(x), _dp(y))
    return y


def _oracle_impl_precond(self, r):
    r = np.ascontiguousarray(r, dtype=np.float64)
    z = np.empty_like(r)
    _impl_lib().ora_impl_precond(self.h, _dp(r), _dp(z))
    return z


def _oracle_impl_x(self):
    x = np.empty(self.nvec)
    _impl_lib().ora_impl_get_x(self.h, _dp(x))
    return x


Oracle.set_implicit = _oracle_set_implicit
Oracle.advance_implicit = _oracle_advance_implicit
Oracle.impl_rhs = _oracle_impl_rhs
Oracle.impl_matvec = _oracle_impl_matvec
Oracle.impl_precond = _oracle_impl_precond
Oracle.impl_x = _oracle_impl_x


class HeatConfig(ctypes.Structure):
    _fields_ = [("heatCondPar", ctypes.c_double), ("fieldAligned", ctypes.c_double), ("cv", ctypes.c_double),
                ("dt", ctypes.c_double), ("semiImplCoeff", ctypes.c_double), ("nKrylovVector", ctypes.c_int),
                ("maxMatvec", ctypes.c_int), ("errorMax", ctypes.c_double), ("typePrecond", ctypes.c_int),
                ("periodic", ctypes.c_int * 3)]


class HeatOracle:
    """Semi-implicit heat conduction restated on the CPU (global arrays,
    x fastest; blocks of 8^3 for the block ILU)."""

    def __init__(self, n, dx, Te, bhat, used, params, periodic=(False, False, False)):
        L = lib()
        for name, res in (("ora_heat_new", ctypes.c_void_p), ("ora_heat_solve", ctypes.c_int)):
            getattr(L, name).restype = res
        L.ora_heat_new.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(HeatConfig)]
        for name in ("ora_heat_free", "ora_heat_rhs", "ora_heat_matvec", "ora_heat_precond", "ora_heat_solve",
                     "ora_heat_get_te"):
            getattr(L, name).argtypes = None
        c = HeatConfig(params.heatCondPar, params.fieldAligned, params.cv, params.dt, params.semiImplCoeff,
                       params.nKrylovVector, params.maxMatvec, params.errorMax,
                       {"none": 0, "bilu": 1}[params.typePrecond.lower()],
                       (ctypes.c_int * 3)(*[int(bool(q)) for q in periodic]))
        self.N = n ** 3
        self._keep = [np.ascontiguousarray(Te, dtype=np.float64), np.ascontiguousarray(bhat, dtype=np.float64),
                      np.ascontiguousarray(used, dtype=np.uint8)]
        nc = (ctypes.c_int * 3)(n, n, n)
        d3 = (ctypes.c_double * 3)(dx, dx, dx)
        self.h = ctypes.c_void_p(L.ora_heat_new(nc, 8, d3, self._keep[0].ctypes.data, self._keep[1].ctypes.data,
                                                self._keep[2].ctypes.data, ctypes.byref(c)))
        self.L = L

    def close(self):
        self.L.ora_heat_free(self.h)

    def _vec(self):
        return np.zeros(self.N)

    def rhs(self):
        b = self._vec()
        self.L.ora_heat_rhs(self.h, b.ctypes.data_as(ctypes.c_void_p))
        return b

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = self._vec()
        self.L.ora_heat_matvec(self.h, x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p))
        return y

    def precond(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = self._vec()
        self.L.ora_heat_precond(self.h, r.ctypes.data_as(ctypes.c_void_p), z.ctypes.data_as(ctypes.c_void_p))
        return z

    def solve(self):
        x = self._vec()
        nm, err = ctypes.c_int(0), ctypes.c_double(0)
        r = self.L.ora_heat_solve(self.h, x.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nm), ctypes.byref(err))
        return r, x, nm.value, err.value

    def te(self):
        t = self._vec()
        self.L.ora_heat_get_te(self.h, t.ctypes.data_as(ctypes.c_void_p))
        return t
