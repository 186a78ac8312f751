"""ctypes binding of libbx200.so (include/bx200.h).

The library is the product: it owns the device state and launches the
sm_100a kernels.  Importing this module fails loudly when the library has
not been built (``python -m batsrus_b200.build`` or
``__graft_entry__.build()``); there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libbx200.so")

BX_OK = 0
STATUS = {0: "BX_OK", 1: "BX_ERR_ARG", 2: "BX_ERR_CUDA", 3: "BX_ERR_STATE", 4: "BX_ERR_NONPHYSICAL",
          5: "BX_ERR_HLLD", 6: "BX_ERR_KRYLOV", 7: "BX_ERR_TIMEOUT", 8: "BX_ERR_NOMEM"}
FLUX = {"rusanov": 0, "linde": 1, "hlld": 2, "roe": 3}
LIMITER = {"minmod": 0, "mc": 1, "mc3": 2, "koren": 2, "no": 0}
BC = {"float": 0, "periodic": 1}
PRECISION = {"fp64": 0, "fp32": 1, "fp32-bulk": 1}
PRECOND_PRECISION = {"fp64": 0, "fp32": 1, "bf16": 2}  # BILU factor storage of the implicit step

# every entry point declared in include/bx200.h
EXPORTS = (
    "bx_init", "bx_set_scheme", "bx_finalize", "bx_last_error", "bx_get_neighbors", "bx_upload_state",
    "bx_download_state", "bx_set_time", "bx_get_time", "bx_calc_face_value", "bx_calc_face_flux",
    "bx_calc_source", "bx_update_state", "bx_calc_timestep", "bx_get_face_values",
    "bx_get_face_flux", "bx_get_source", "bx_set_stage", "bx_update_state_fast",
    "bx_exchange_messages", "bx_set_global_timestep", "bx_advance_explicit", "bx_advance",
    "bx_set_graph_steps", "bx_synchronize", "bx_timing_enable", "bx_timing_get", "bx_timing_reset",
    "bx_region_begin", "bx_region_end",
    "bx_implicit_init", "bx_advance_part_impl", "bx_impl_get_rhs", "bx_impl_matvec",
    "bx_impl_precond", "bx_impl_get_x",
    "bx_learned_init", "bx_learned_set_activation", "bx_learned_set_blend", "bx_learned_finalize", "bx_learned_nparam", "bx_learned_set_params",
    "bx_learned_get_params", "bx_learned_collect", "bx_learned_collect_probes", "bx_learned_num_samples", "bx_learned_set_samples",
    "bx_learned_gradient", "bx_learned_train", "bx_learned_apply_blocks",
    "bx_impl_norm_noalloc",
    "bx_heat_init", "bx_advance_semi_impl", "bx_heat_get_te", "bx_heat_get_rhs", "bx_heat_matvec",
    "bx_heat_precond",
    "bx_autotune", "bx_tune_info", "bx_tune_set", "bx_tune_reset",
    "bx_amr_criteria", "bx_regrid", "bx_amr_plan", "bx_do_amr", "bx_get_grid",
    "bx_get_block_dt", "bx_set_block_dt",
    "bx_halo_bytes", "bx_halo_pack", "bx_halo_unpack", "bx_get_dtmin", "bx_set_dtmin", "bx_end_step",
)
# #AMRCRITERIA TypeRefine -> BX_AMR_*
AMR_CRIT = {"gradt": 1, "gradlogrho": 2, "gradlogp": 3, "gradp": 4, "pjumpratio": 5, "-divu": 6, "-divudx": 6}
PRECOND = {"none": 0, "bilu": 1, "learned": 2}
NOALLOC_MAX_BLOCK = 32768  # BX_NOALLOC_MAX_BLOCK


class ImplicitParamsC(ctypes.Structure):
    _fields_ = [
        ("CflImpl", ctypes.c_double), ("ImplCoeff", ctypes.c_double), ("UseBdf2", ctypes.c_int),
        ("nOrderImpl", ctypes.c_int), ("TypeFluxImpl", ctypes.c_int), ("JacobianEps", ctypes.c_double),
        ("nKrylovVector", ctypes.c_int), ("MaxMatvec", ctypes.c_int), ("ErrorMax", ctypes.c_double),
        ("TypePrecond", ctypes.c_int), ("PrecondPrecision", ctypes.c_int),
    ]


class KrylovStats(ctypes.Structure):
    _fields_ = [
        ("nMatvec", ctypes.c_int), ("iError", ctypes.c_int), ("Error", ctypes.c_double),
        ("Dt", ctypes.c_double), ("msStep", ctypes.c_double), ("msPrecondSetup", ctypes.c_double),
    ]


class AmrParamsC(ctypes.Structure):
    _fields_ = [
        ("nCrit", ctypes.c_int), ("iTypeCrit", ctypes.c_int * 3), ("CoarsenLimit", ctypes.c_double * 3),
        ("RefineLimit", ctypes.c_double * 3), ("MinBlockLevel", ctypes.c_int), ("MaxBlockLevel", ctypes.c_int),
        ("MaxTotalBlocks", ctypes.c_int),
    ]


def amr_params(p):
    """bx_amr_params from batsrus_b200.amr.AmrParams"""
    c = AmrParamsC()
    if not 1 <= len(p.criteria) <= 3:
        raise ValueError("1 to 3 AMR criteria, got %d" % len(p.criteria))
    c.nCrit = len(p.criteria)
    for q, cr in enumerate(p.criteria):
        try:
            c.iTypeCrit[q] = AMR_CRIT[cr.name.lower()]
        except KeyError:
            raise ValueError("AMR criterion %s is not built (built: %s)" % (cr.name, ", ".join(AMR_CRIT)))
        c.CoarsenLimit[q] = cr.coarsenLimit
        c.RefineLimit[q] = cr.refineLimit
    c.MinBlockLevel, c.MaxBlockLevel, c.MaxTotalBlocks = p.minBlockLevel, p.maxBlockLevel, p.maxTotalBlocks
    return c


class HeatParamsC(ctypes.Structure):
    _fields_ = [
        ("HeatCondPar", ctypes.c_double), ("FractionFieldAligned", ctypes.c_double), ("Cv", ctypes.c_double),
        ("Dt", ctypes.c_double), ("SemiImplCoeff", ctypes.c_double), ("nKrylovVector", ctypes.c_int),
        ("MaxMatvec", ctypes.c_int), ("ErrorMax", ctypes.c_double), ("TypePrecond", ctypes.c_int),
        ("PrecondPrecision", ctypes.c_int), ("OperatorPrecision", ctypes.c_int),
    ]


def heat_params(p):
    return HeatParamsC(p.heatCondPar, p.fieldAligned, p.cv, p.dt, p.semiImplCoeff, p.nKrylovVector,
                       p.maxMatvec, p.errorMax, PRECOND[p.typePrecond.lower()],
                       PRECISION[p.precondPrecision.lower()], PRECISION[p.operatorPrecision.lower()])


def implicit_params(p):
    c = ImplicitParamsC()
    c.CflImpl = p.cflImpl
    c.ImplCoeff = p.implCoeff0
    c.UseBdf2 = int(p.useBdf2)
    c.nOrderImpl = p.nOrderImpl
    c.TypeFluxImpl = -1 if p.typeFluxImpl in (None, "default") else FLUX[p.typeFluxImpl.lower()]
    c.JacobianEps = p.jacobianEps
    c.nKrylovVector = p.nKrylovVector
    c.MaxMatvec = p.maxMatvec
    c.ErrorMax = p.errorMax
    c.TypePrecond = PRECOND[p.typePrecond.lower()]
    c.PrecondPrecision = PRECOND_PRECISION[p.precondPrecision.lower()]
    return c


class BxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS.get(code, code), msg))
        self.code = code


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("nDim", ctypes.c_int), ("nI", ctypes.c_int), ("nJ", ctypes.c_int), ("nK", ctypes.c_int),
        ("nRootBlock", ctypes.c_int * 3),
        ("CoordMin", ctypes.c_double * 3), ("CoordMax", ctypes.c_double * 3),
        ("TypeBc", ctypes.c_int * 6),
        ("nBlock", ctypes.c_int),
        ("iLevelCoord_IB", ctypes.POINTER(ctypes.c_int)),
        ("iDevice", ctypes.c_int),
        ("nOwned", ctypes.c_int),
    ]


class SchemeParams(ctypes.Structure):
    _fields_ = [
        ("nOrder", ctypes.c_int), ("nStage", ctypes.c_int),
        ("TypeFlux", ctypes.c_int), ("TypeLimiter", ctypes.c_int),
        ("LimiterBeta", ctypes.c_double), ("Cfl", ctypes.c_double), ("Gamma", ctypes.c_double),
        ("UseDivbSource", ctypes.c_int), ("UseHalfStep", ctypes.c_int),
        ("UseDtFixed", ctypes.c_int), ("DtFixed", ctypes.c_double),
        ("Precision", ctypes.c_int),
        ("RhoMin", ctypes.c_double), ("pMin", ctypes.c_double), ("TMin", ctypes.c_double),
        ("MassIon", ctypes.c_double),
        ("UseTvdResChange", ctypes.c_int), ("BetaLimiterResChange", ctypes.c_double),
        ("nFaceLimiterResChange", ctypes.c_int),
    ]


_lib = None


def load():
    """Load libbx200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libbx200.so not found at %s: build it with __graft_entry__.build() "
                          "(the hot path has no CPU fallback)" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    i, d, p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    fp = ctypes.POINTER(ctypes.c_float)
    sig = {
        "bx_init": [ctypes.POINTER(GridDesc), ctypes.POINTER(SchemeParams)],
        "bx_set_scheme": [ctypes.POINTER(SchemeParams)],
        "bx_finalize": [], "bx_get_neighbors": [ip, ip],
        "bx_upload_state": [dp, i], "bx_download_state": [dp, i],
        "bx_set_time": [d, i], "bx_get_time": [dp, dp, ip],
        "bx_calc_face_value": [i, i, i], "bx_calc_face_flux": [i, i],
        "bx_calc_source": [i], "bx_update_state": [i], "bx_calc_timestep": [i],
        "bx_get_face_values": [i, dp, dp], "bx_get_face_flux": [i, dp], "bx_get_source": [dp],
        "bx_set_stage": [i], "bx_update_state_fast": [], "bx_exchange_messages": [i],
        "bx_set_global_timestep": [d, dp], "bx_advance_explicit": [i], "bx_advance": [i, d],
        "bx_halo_bytes": [i, ip], "bx_halo_pack": [i, ip, i, p], "bx_halo_unpack": [i, ip, i, p],
        "bx_get_dtmin": [dp], "bx_set_dtmin": [d], "bx_end_step": [d],
        "bx_set_graph_steps": [i], "bx_synchronize": [], "bx_timing_enable": [i], "bx_timing_get": [dp, ip, ip],
        "bx_timing_reset": [], "bx_region_begin": [], "bx_region_end": [dp],
        "bx_implicit_init": [ctypes.POINTER(ImplicitParamsC)],
        "bx_advance_part_impl": [d, ctypes.POINTER(KrylovStats)],
        "bx_impl_get_rhs": [dp, dp], "bx_impl_matvec": [dp, dp], "bx_impl_precond": [dp, dp],
        "bx_impl_get_x": [dp],
        "bx_learned_init": [ctypes.c_longlong, ctypes.c_ulonglong], "bx_learned_finalize": [],
        "bx_learned_set_activation": [i], "bx_learned_set_blend": [d],
        "bx_learned_nparam": [ip], "bx_learned_set_params": [fp, i], "bx_learned_get_params": [fp, i],
        "bx_learned_collect": [i], "bx_learned_collect_probes": [i, i, ctypes.c_ulonglong], "bx_learned_num_samples": [ctypes.POINTER(ctypes.c_longlong)],
        "bx_learned_set_samples": [fp, fp, ctypes.c_longlong],
        "bx_learned_gradient": [ctypes.c_longlong, i, fp, dp],
        "bx_learned_train": [i, i, d, dp, dp],
        "bx_learned_apply_blocks": [dp, fp, i, dp],
        "bx_impl_norm_noalloc": [p, i, i, p, dp],
        "bx_heat_init": [ctypes.POINTER(HeatParamsC), dp, dp, ctypes.POINTER(ctypes.c_ubyte)],
        "bx_advance_semi_impl": [ctypes.POINTER(KrylovStats)],
        "bx_autotune": [], "bx_tune_set": [ctypes.c_char_p, i], "bx_tune_reset": [],
        "bx_tune_info": [i, ctypes.c_char_p, i, ip, ip, ip, ip, fp],
        "bx_heat_get_te": [dp], "bx_heat_get_rhs": [dp], "bx_heat_matvec": [dp, dp], "bx_heat_precond": [dp, dp],
        "bx_amr_criteria": [i, ip, dp], "bx_regrid": [ctypes.POINTER(GridDesc), ip],
        "bx_amr_plan": [ctypes.POINTER(GridDesc), ctypes.POINTER(AmrParamsC), dp, i, ip, ip, ip, ip],
        "bx_do_amr": [ctypes.POINTER(AmrParamsC), ip, ip], "bx_get_grid": [ip],
        "bx_get_block_dt": [dp], "bx_set_block_dt": [dp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L.bx_last_error.argtypes = []
    L.bx_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def check(code):
    if code != BX_OK:
        raise BxError(code, load().bx_last_error().decode())
    return code


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def grid_desc(grid, device=0, nOwned=0):
    g = GridDesc()
    g.nDim = grid.nDim
    g.nI, g.nJ, g.nK = grid.nI, grid.nJ, grid.nK
    for d in range(3):
        g.nRootBlock[d] = grid.nRoot[d]
        g.CoordMin[d] = grid.xyzMin[d]
        g.CoordMax[d] = grid.xyzMax[d]
    for s in range(6):
        g.TypeBc[s] = BC[grid.typeBc[s]]
    g.nBlock = grid.nBlock
    lc = np.ascontiguousarray(grid.iLevelCoord, dtype=np.int32)
    g.iLevelCoord_IB = lc.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    g._keep = lc  # keep the array alive while the struct is used
    g.iDevice = device
    g.nOwned = nOwned
    return g


def scheme_params(s):
    if getattr(s, "useNonConservative", False):
        raise ValueError("#NONCONSERVATIVE (the pressure equation) is not on the GPU path: "
                         "bx_update_state_fast solves for the energy")
    p = SchemeParams()
    p.nOrder = s.nOrder
    p.nStage = s.nStage
    p.TypeFlux = FLUX[s.typeFlux.lower()]
    p.TypeLimiter = LIMITER[s.typeLimiter.lower()]
    p.LimiterBeta = s.limiterBeta
    p.Cfl = s.cfl
    p.Gamma = s.gamma
    p.UseDivbSource = int(s.useDivbSource)
    p.UseHalfStep = int(s.useHalfStep)
    p.UseDtFixed = int(s.useDtFixed)
    p.DtFixed = s.dtFixed
    p.Precision = PRECISION[s.precision.lower()]
    p.RhoMin = getattr(s, "rhoMin", -1.0)
    p.pMin = getattr(s, "pMin", -1.0)
    p.TMin = getattr(s, "tMin", -1.0)
    p.MassIon = getattr(s, "massIon", 1.0)
    p.UseTvdResChange = int(getattr(s, "useTvdResChange", True))
    p.BetaLimiterResChange = getattr(s, "betaLimiterResChange", 2.0)
    p.nFaceLimiterResChange = getattr(s, "nFaceLimiterResChange", 2)
    return p


def tune_info():
    """The autotuner's knobs: {name: {"value", "tuned", "candidates", "ms"}}."""
    L = load()
    out = {}
    i = 0
    while True:
        name = ctypes.create_string_buffer(64)
        v, t, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        cand = (ctypes.c_int * 8)()
        ms = (ctypes.c_float * 8)()
        if L.bx_tune_info(i, name, 64, ctypes.byref(v), ctypes.byref(t), ctypes.byref(n), cand, ms) != BX_OK:
            break
        out[name.value.decode()] = {"value": v.value, "tuned": t.value, "candidates": list(cand[:n.value]),
                                    "ms": [round(float(x), 4) for x in ms[:n.value]]}
        i += 1
    return out


def tune_set(name, value):
    check(load().bx_tune_set(name.encode(), int(value)))


def tune_reset():
    check(load().bx_tune_reset())


def autotune():
    check(load().bx_autotune())
    return tune_info()
