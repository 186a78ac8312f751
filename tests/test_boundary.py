"""C-ABI boundary checks that need no GPU: the library loads, exports every
entry point include/bx200.h declares, the ctypes structures match the header,
and argument errors come back as status codes (no CUDA call is made)."""
import ctypes
import os
import re

import pytest

from batsrus_b200 import capi, configs
from batsrus_b200.param import Scheme, apply_commands, read_param

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "bx200.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"BX_API\s+(?:const\s+char\s*\*|int)\s*(bx_\w+)\s*\(", txt)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(capi.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = capi.load()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_structs_match_header_field_order():
    txt = open(HEADER).read()
    for cname, pystruct in (("bx_grid_desc", capi.GridDesc), ("bx_scheme_params", capi.SchemeParams),
                            ("bx_implicit_params", capi.ImplicitParamsC), ("bx_krylov_stats", capi.KrylovStats),
                            ("bx_heat_params", capi.HeatParamsC), ("bx_amr_params", capi.AmrParamsC)):
        body = re.search(r"typedef struct \{([^{}]*)\}\s*%s;" % cname, txt).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        names = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            for part in decl.split(","):
                m = re.search(r"\*?\s*(\w+)\s*(\[\d+\])?\s*$", part.strip())
                names.append(m.group(1))
        assert names == [f[0] for f in pystruct._fields_], cname


def test_argument_errors_without_gpu():
    L = capi.load()
    # calls before bx_init are refused
    assert L.bx_advance(1, -1.0) == 3
    assert b"bx_init" in L.bx_last_error()
    assert L.bx_autotune() == 3
    # the autotuner's table needs no device
    knobs = capi.tune_info()
    assert set(knobs) == {"stage_ctas_per_sm", "krylov_ctas_per_sm", "krylov_unroll", "heat_ilu_warps",
                          "bilu_threads", "stage_variant", "krylov_gs_steps"}
    assert all(k["value"] in k["candidates"] and k["tuned"] == 0 for k in knobs.values())
    assert L.bx_tune_set(b"krylov_unroll", 3) == 1 and L.bx_tune_set(b"no_such_knob", 1) == 1
    capi.tune_set("krylov_unroll", 4)
    assert capi.tune_info()["krylov_unroll"] == dict(knobs["krylov_unroll"], value=4, tuned=2)
    capi.tune_reset()
    assert capi.tune_info() == knobs
    # dynamic AMR entry points need a grid
    assert L.bx_do_amr(None, None, None) == 3 and L.bx_get_grid(None) == 3
    # unsupported block size is rejected before any device call
    g, s, _, _ = configs.brio_wu_1d()
    gd = capi.grid_desc(g)
    gd.nI = 7
    assert L.bx_init(ctypes.byref(gd), ctypes.byref(capi.scheme_params(s))) == 1
    assert b"not supported" in L.bx_last_error()
    # FP32-bulk needs 3D blocks
    gd = capi.grid_desc(g)
    s.precision = "fp32"
    assert L.bx_init(ctypes.byref(gd), ctypes.byref(capi.scheme_params(s))) == 1


def test_param_reader_scheme_commands():
    text = """
#GAMMA
2.0			Gamma

#TIMESTEPPING
1			nStage
0.8			CflExpl

#FIXEDTIMESTEP
T			UseDtFixed
0.05			DtFixedDim

#SCHEME
1			nOrder
Rusanov			TypeFlux

#STOP
-1			MaxIteration
25.6			tSimulationMax

#RUN

#SCHEME
2			nOrder
Linde			TypeFlux
mc3			TypeLimiter
1.2			LimiterBeta

#END
"""
    sessions = read_param(text)
    assert len(sessions) == 2
    s = Scheme()
    info = apply_commands(sessions[0], s)
    assert (s.nOrder, s.nStage, s.typeFlux, s.gamma) == (1, 1, "Rusanov", 2.0)
    assert s.useDtFixed and s.dtFixed == 0.05 and s.cfl == 1.0
    assert info["tSimulationMax"] == 25.6
    apply_commands(sessions[1], s)
    assert (s.nOrder, s.nStage, s.typeFlux, s.typeLimiter, s.limiterBeta) == (2, 2, "Linde", "mc3", 1.2)
    assert s.useHalfStep
