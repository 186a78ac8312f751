"""Host-side mirror of the reference's explicit-update interface.

``ExplicitSolver`` exposes the entry points a BATS-R-US driver calls on the
explicit path, with the reference's names and argument meaning, on top of
the C ABI of libbx200 (include/bx200.h):

* set-up: ``init_mod_advance`` (src/ModAdvance.f90:296) -> ``__init__``;
* per block (orig path, src/ModAdvanceExplicit.f90:140-226):
  ``calc_face_value(iBlock, DoResChangeOnly, DoMonotoneRestrict)``,
  ``calc_face_flux(DoResChangeOnly, iBlock)``, ``calc_source(iBlock)``,
  ``calc_timestep(iBlock)``, ``update_state(iBlock)``;
* batched: ``update_state_fast()`` (src/ModUpdateStateFast.f90:190),
  ``exchange_messages()`` (src/ModMessagePass.f90:27),
  ``set_global_timestep(TimeSimulationLimit)``
  (src/ModTimeStepControl.f90:306), ``advance_explicit()``
  (src/ModAdvanceExplicit.f90:18), ``advance(nStep, TimeSimulationLimit)``
  (nStep calls of BATS_advance, src/ModBatsrusMethods.f90:493).

Errors come back as :class:`batsrus_b200.capi.BxError` instead of the
reference's ``stop_mpi`` abort.  One solver is active per process (the
library keeps one context, like the Fortran module globals).
"""
import ctypes

import numpy as np

from . import capi
from .capi import check, dptr


class ExplicitSolver:
    def __init__(self, grid, scheme, device=0, nOwned=0):
        """nOwned > 0: one rank of a partitioned grid whose first nOwned
        blocks it updates (batsrus_b200.shard.RankDomain); the other blocks
        are copies of remote neighbours."""
        self.L = capi.load()
        self.grid = grid
        self.scheme = scheme
        self.nOwned = nOwned if nOwned > 0 else grid.nBlock
        self._gd = capi.grid_desc(grid, device, nOwned)
        self._sp = capi.scheme_params(scheme)
        check(self.L.bx_init(ctypes.byref(self._gd), ctypes.byref(self._sp)))

    def set_scheme(self, scheme):
        """#SCHEME / #TIMESTEPPING of a new session."""
        self.scheme = scheme
        self._sp = capi.scheme_params(scheme)
        check(self.L.bx_set_scheme(ctypes.byref(self._sp)))

    def close(self):
        self.L.bx_finalize()

    # -- state ---------------------------------------------------------------
    def set_state(self, State_VGB):
        a = np.ascontiguousarray(State_VGB, dtype=np.float64)
        assert a.shape == self.grid.state_shape_fortran(), a.shape
        check(self.L.bx_upload_state(dptr(a), self.grid.nBlock))

    def get_state(self, out=None):
        a = out if out is not None else np.empty(self.grid.state_shape_fortran())
        check(self.L.bx_download_state(dptr(a), self.grid.nBlock))
        return a

    def set_time(self, tSimulation, nStep):
        check(self.L.bx_set_time(tSimulation, nStep))

    def time(self):
        t, dt, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        check(self.L.bx_get_time(ctypes.byref(t), ctypes.byref(dt), ctypes.byref(n)))
        return t.value, dt.value, n.value

    def block_dt(self):
        """DtMax_B of every block from the last step (bx_get_block_dt)"""
        out = np.empty(self.grid.nBlock)
        check(self.L.bx_get_block_dt(dptr(out)))
        return out

    def set_block_dt(self, DtMax_B):
        """DtMax_B from a restart: the next step's time step (bx_set_block_dt)"""
        a = np.ascontiguousarray(DtMax_B, dtype=np.float64)
        assert a.shape == (self.grid.nBlock,), a.shape
        check(self.L.bx_set_block_dt(dptr(a)))

    # -- per-block orig path ------------------------------------------------
    def calc_face_value(self, iBlock, DoResChangeOnly=False, DoMonotoneRestrict=True):
        check(self.L.bx_calc_face_value(iBlock, int(DoResChangeOnly), int(DoMonotoneRestrict)))

    def calc_face_flux(self, DoResChangeOnly, iBlock):
        check(self.L.bx_calc_face_flux(int(DoResChangeOnly), iBlock))

    def calc_source(self, iBlock):
        check(self.L.bx_calc_source(iBlock))

    def calc_timestep(self, iBlock):
        check(self.L.bx_calc_timestep(iBlock))

    def update_state(self, iBlock):
        check(self.L.bx_update_state(iBlock))

    def _nface(self, iDim):
        n = [self.grid.nI, self.grid.nJ, self.grid.nK]
        n[iDim] += 1
        return n

    def face_values(self, iDim):
        n = self._nface(iDim)
        L = np.empty((n[2], n[1], n[0], 8))
        R = np.empty_like(L)
        check(self.L.bx_get_face_values(iDim, dptr(L), dptr(R)))
        return L, R

    def face_flux(self, iDim):
        n = self._nface(iDim)
        F = np.empty((n[2], n[1], n[0], 9))
        check(self.L.bx_get_face_flux(iDim, dptr(F)))
        return F

    def source(self):
        g = self.grid
        S = np.empty((g.nK, g.nJ, g.nI, 9))
        check(self.L.bx_get_source(dptr(S)))
        return S

    # -- batched path --------------------------------------------------------
    def set_stage(self, iStage):
        check(self.L.bx_set_stage(iStage))

    def update_state_fast(self):
        check(self.L.bx_update_state_fast())

    def exchange_messages(self, DoResChangeOnly=False):
        check(self.L.bx_exchange_messages(int(DoResChangeOnly)))

    def set_global_timestep(self, TimeSimulationLimit=-1.0):
        dt = ctypes.c_double()
        check(self.L.bx_set_global_timestep(TimeSimulationLimit, ctypes.byref(dt)))
        return dt.value

    # -- one rank of a partitioned grid ------------------------------------
    def halo_bytes(self, iStage):
        n = ctypes.c_int()
        check(self.L.bx_halo_bytes(iStage, ctypes.byref(n)))
        return n.value

    def halo_pack(self, iStage, blocks, buf_ptr):
        """the interiors of blocks (0-based local indices) that stage iStage
        reads, into the device buffer at buf_ptr"""
        b = np.ascontiguousarray(np.asarray(blocks) + 1, dtype=np.int32)
        check(self.L.bx_halo_pack(iStage, b.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(b),
                                  ctypes.c_void_p(buf_ptr)))

    def halo_unpack(self, iStage, blocks, buf_ptr):
        b = np.ascontiguousarray(np.asarray(blocks) + 1, dtype=np.int32)
        check(self.L.bx_halo_unpack(iStage, b.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(b),
                                    ctypes.c_void_p(buf_ptr)))

    def get_dtmin(self):
        v = ctypes.c_double()
        check(self.L.bx_get_dtmin(ctypes.byref(v)))
        return v.value

    def set_dtmin(self, v):
        check(self.L.bx_set_dtmin(float(v)))

    def end_step(self, TimeSimulationLimit=-1.0):
        check(self.L.bx_end_step(TimeSimulationLimit))

    def advance_explicit(self, DoCalcTimestep=True):
        check(self.L.bx_advance_explicit(int(DoCalcTimestep)))

    def advance(self, nStep=1, TimeSimulationLimit=-1.0):
        check(self.L.bx_advance(nStep, TimeSimulationLimit))

    def set_graph_steps(self, n):
        """time steps captured in one CUDA graph by advance()"""
        check(self.L.bx_set_graph_steps(int(n)))

    def synchronize(self):
        check(self.L.bx_synchronize())

    # -- dynamic AMR (src/ModAMR.f90) ----------------------------------------
    def amr_criteria(self, names):
        """amr_criteria (src/ModAMR.f90:388-723) on the GPU: Crit_IB as an
        (nBlock, len(names)) array, names from #AMRCRITERIA."""
        n = len(names)
        try:
            codes = (ctypes.c_int * n)(*[capi.AMR_CRIT[str(t).lower()] for t in names])
        except KeyError as e:
            raise ValueError("AMR criterion %s is not built (built: %s)" % (e, ", ".join(capi.AMR_CRIT)))
        out = np.empty((self.grid.nBlock, n))
        check(self.L.bx_amr_criteria(n, codes, dptr(out)))
        return out

    def regrid(self, grid, remap):
        """bx_regrid: replace the grid and move the state onto it."""
        gd = capi.grid_desc(grid, self._gd.iDevice)
        R = np.ascontiguousarray(remap, dtype=np.int32)
        assert R.shape == (grid.nBlock, 10), R.shape
        check(self.L.bx_regrid(ctypes.byref(gd), R.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.grid, self._gd = grid, gd

    def do_amr(self, params):
        """prepare_amr + do_amr (src/ModAMR.f90:171-386) in one library call
        (bx_do_amr): criteria on the GPU, the new tree in the library's host
        code, the state moved on the GPU.  Returns True if the grid changed."""
        from .grid import BlockGrid
        cp = capi.amr_params(params)
        n, ch = ctypes.c_int(), ctypes.c_int()
        check(self.L.bx_do_amr(ctypes.byref(cp), ctypes.byref(n), ctypes.byref(ch)))
        if ch.value:
            lc = np.empty((n.value, 4), dtype=np.int32)
            check(self.L.bx_get_grid(lc.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
            g = self.grid
            self.grid = BlockGrid(g.nDim, g.nI, g.nJ, g.nK, g.nRoot, g.xyzMin, g.xyzMax, g.typeBc, lc)
            self._gd = capi.grid_desc(self.grid, self._gd.iDevice)
        return bool(ch.value)

    def advance_amr(self, nStep, params, TimeSimulationLimit=-1.0):
        """nStep steps of BATS_advance with do_amr after every step whose
        number is a multiple of DnRefine (src/ModBatsrusMethods.f90:493-760).
        Returns the number of regrids that changed the grid."""
        if params.dnRefine <= 0:
            self.advance(nStep, TimeSimulationLimit)
            return 0
        nRegrid = 0
        done = 0
        while done < nStep:
            n0 = self.time()[2]
            k = min(nStep - done, params.dnRefine - n0 % params.dnRefine)
            self.advance(k, TimeSimulationLimit)
            done += k
            if self.time()[2] % params.dnRefine == 0:
                nRegrid += self.do_amr(params)
        return nRegrid

    # -- measurement -----------------------------------------------------------
    def autotune(self):
        """bx_autotune: time the candidate launch shapes of every kernel whose
        context is ready and keep the fastest; returns the knob table."""
        return capi.autotune()

    def timing(self, on):
        check(self.L.bx_timing_enable(int(on)))

    def timing_reset(self):
        check(self.L.bx_timing_reset())

    def region_begin(self):
        check(self.L.bx_region_begin())

    def region_end(self):
        ms = ctypes.c_double()
        check(self.L.bx_region_end(ctypes.byref(ms)))
        return ms.value

    def timing_get(self):
        ms, n, ntot = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        check(self.L.bx_timing_get(ctypes.byref(ms), ctypes.byref(n), ctypes.byref(ntot)))
        return ms.value, n.value, ntot.value
