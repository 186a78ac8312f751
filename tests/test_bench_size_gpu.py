"""GPU parity at the sizes the benchmark times, through the C ABI.

* The headline workload: 3D Orszag-Tang at 256^3 (32768 blocks of 8^3),
  Linde HLL + Koren (mc3, beta 1.2), CFL 0.8, 2-stage half step, Powell
  source, FP64: the first (Dt = 0) step and two full steps, each within
  1e-12 of the oracle (normwise per variable, vector components against
  their vector's largest magnitude), the time step within 1e-14.
* The block-adaptive blast at the benchmark's size: levels 0-3 on 19^3 root
  blocks (20,544 blocks, 10.5 M cells), HLLD + MC (beta 1.5), FP64:
  DiLevel_EB / jBlock_IEB bit-exact against the host tree, then three steps
  within 1e-12 of the oracle.

The comparison runs block range by block range so that the 256^3 arrays
(3.6 GB each with ghost cells) need no full-size temporaries.
"""
import ctypes

import numpy as np
import pytest

from batsrus_b200 import capi, configs
from batsrus_b200.explicit import ExplicitSolver
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def chunked_rel_err(a, b, isl, chunk=2048):
    """max over variables of max|a - b| / scale, over the interior cells;
    a, b: (nBlock, nKg, nJg, nIg, 8) with ghosts, isl the interior slices"""
    nB = a.shape[0]
    dmax = np.zeros(8)
    smax = np.zeros(8)
    vmax = np.zeros(2)
    for b0 in range(0, nB, chunk):
        sl = (slice(b0, min(nB, b0 + chunk)),) + tuple(isl[1:])
        A, B = a[sl], b[sl]
        dmax = np.maximum(dmax, np.abs(A - B).max(axis=(0, 1, 2, 3)))
        smax = np.maximum(smax, np.abs(B).max(axis=(0, 1, 2, 3)))
        vmax = np.maximum(vmax, [np.sqrt((B[..., 1:4] ** 2).sum(-1)).max(),
                                 np.sqrt((B[..., 4:7] ** 2).sum(-1)).max()])
    scale = smax.copy()
    scale[1:4] = vmax[0]
    scale[4:7] = vmax[1]
    return (dmax / np.maximum(scale, 1e-300)).max()


def test_orszag_tang_256cubed_linde_koren_fp64_matches_oracle():
    g, s, st, _ = configs.orszag_tang_3d(nRoot=32, precision="fp64", flux="Linde")
    assert g.nBlock == 32768 and (s.typeFlux, s.typeLimiter, s.limiterBeta) == ("Linde", "mc3", 1.2)
    o = Oracle(g, s)
    o.set_state(st)
    o.exchange_messages()
    x = ExplicitSolver(g, s)
    x.set_state(st)
    del st
    isl = g.interior_slices()
    for step in range(3):  # the Dt = 0 step, then two full steps
        x.advance(1)
        o.advance(1)
        tg, dtg, ng = x.time()
        to, dto, no = o.time()
        assert ng == no and abs(dtg - dto) <= 1e-14 * max(abs(dto), 1e-300), (step, dtg, dto)
        e = chunked_rel_err(x.get_state(), o.get_state(), isl)
        assert e < TOL_FP64, (step, e)
    x.close()


def test_amr_blast_bench_size_fp64_matches_oracle():
    g, s, st, _ = configs.amr_blast(nRoot=19, maxLevel=3, precision="fp64")
    lev = np.bincount(g.iLevelCoord[:, 0])
    assert g.nBlock == 20544 and len(lev) == 4 and (s.typeFlux, s.typeLimiter) == ("HLLD", "mc")
    x = ExplicitSolver(g, s)
    # the neighbour bookkeeping of the whole grid, bit for bit
    dil, jb = g.neighbors()
    L = capi.load()
    d = np.zeros(6 * g.nBlock, dtype=np.int32)
    j = np.zeros(24 * g.nBlock, dtype=np.int32)
    capi.check(L.bx_get_neighbors(d.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  j.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
    assert np.array_equal(d.reshape(-1, 6), dil)
    assert np.array_equal(j.reshape(-1, 6, 4), jb + 1)
    o = Oracle(g, s)
    o.set_state(st)
    o.exchange_messages()
    x.set_state(st)
    del st
    isl = g.interior_slices()
    for step in range(4):  # the Dt = 0 step, then three full steps
        x.advance(1)
        o.advance(1)
        tg, dtg, ng = x.time()
        to, dto, no = o.time()
        assert ng == no and abs(dtg - dto) <= 1e-13 * max(abs(dto), 1e-300), (step, dtg, dto)
        e = chunked_rel_err(x.get_state(), o.get_state(), isl)
        assert e < TOL_FP64, (step, e)
    x.close()
