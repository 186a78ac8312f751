! bx200_interface.f90 -- ISO_C_BINDING interface of libbx200 (bx200.h).
!
! A BATS-R-US build adds this module and calls the bx_* functions from
! ModAdvanceExplicit / ModBatsrusMethods in place of the explicit update.
! Logical flags cross as integers (0/1); iBlock is the Fortran block index;
! State_VGB is passed as is (real(8), nVar fastest, ghost cells included).
! Every function returns an integer status (0 = success); the message of a
! failure is returned by bx_last_error.
!
! This file is not compiled in the repository's own build or tests (no
! Fortran compiler is installed where they run).
module bx200_interface

  use, intrinsic :: iso_c_binding, only: c_int, c_double, c_ptr, c_char, c_signed_char

  implicit none

  integer(c_int), parameter:: BX_FLUX_RUSANOV = 0, BX_FLUX_LINDE = 1, &
       BX_FLUX_HLLD = 2, BX_FLUX_ROE = 3
  integer(c_int), parameter:: BX_LIM_MINMOD = 0, BX_LIM_MC = 1, BX_LIM_MC3 = 2
  integer(c_int), parameter:: BX_BC_FLOAT = 0, BX_BC_PERIODIC = 1
  integer(c_int), parameter:: BX_FP64 = 0, BX_FP32_BULK = 1, BX_BF16_FACTORS = 2

  type, bind(C):: bx_grid_desc
     integer(c_int):: nDim, nI, nJ, nK
     integer(c_int):: nRootBlock(3)
     real(c_double):: CoordMin(3), CoordMax(3)
     integer(c_int):: TypeBc(6)
     integer(c_int):: nBlock
     type(c_ptr)   :: iLevelCoord_IB   ! c_loc of integer(c_int) (4,nBlock)
     integer(c_int):: iDevice
     integer(c_int):: nOwned           ! 0: all blocks are this rank's
  end type bx_grid_desc

  integer(c_int), parameter:: BX_PRECOND_NONE = 0, BX_PRECOND_BILU = 1, &
       BX_PRECOND_LEARNED = 2

  type, bind(C):: bx_implicit_params
     real(c_double):: CflImpl, ImplCoeff
     integer(c_int):: UseBdf2, nOrderImpl, TypeFluxImpl
     real(c_double):: JacobianEps
     integer(c_int):: nKrylovVector, MaxMatvec
     real(c_double):: ErrorMax
     integer(c_int):: TypePrecond, PrecondPrecision
  end type bx_implicit_params

  type, bind(C):: bx_krylov_stats
     integer(c_int):: nMatvec, iError
     real(c_double):: Error, Dt, msStep, msPrecondSetup
  end type bx_krylov_stats

  integer(c_int), parameter:: BX_AMR_GRADT = 1, BX_AMR_GRADLOGRHO = 2, &
       BX_AMR_GRADLOGP = 3, BX_AMR_GRADP = 4, BX_AMR_PJUMPRATIO = 5

  ! #AMRCRITERIA, #AMRLEVELS, #AMR MaxTotalBlocks
  type, bind(C):: bx_amr_params
     integer(c_int):: nCrit
     integer(c_int):: iTypeCrit(3)
     real(c_double):: CoarsenLimit(3), RefineLimit(3)
     integer(c_int):: MinBlockLevel, MaxBlockLevel, MaxTotalBlocks
  end type bx_amr_params

  type, bind(C):: bx_heat_params
     real(c_double):: HeatCondPar, FractionFieldAligned, Cv, Dt, SemiImplCoeff
     integer(c_int):: nKrylovVector, MaxMatvec
     real(c_double):: ErrorMax
     integer(c_int):: TypePrecond, PrecondPrecision, OperatorPrecision
  end type bx_heat_params

  type, bind(C):: bx_scheme_params
     integer(c_int):: nOrder, nStage, TypeFlux, TypeLimiter
     real(c_double):: LimiterBeta, Cfl, Gamma
     integer(c_int):: UseDivbSource, UseHalfStep, UseDtFixed
     real(c_double):: DtFixed
     integer(c_int):: Precision
     real(c_double):: RhoMin, pMin, TMin, MassIon
     integer(c_int):: UseTvdResChange
     real(c_double):: BetaLimiterResChange
     integer(c_int):: nFaceLimiterResChange
  end type bx_scheme_params

  interface
     integer(c_int) function bx_init(Grid, Scheme) bind(C, name='bx_init')
       import:: c_int, bx_grid_desc, bx_scheme_params
       type(bx_grid_desc), intent(in):: Grid
       type(bx_scheme_params), intent(in):: Scheme
     end function bx_init

     integer(c_int) function bx_set_scheme(Scheme) bind(C, name='bx_set_scheme')
       import:: c_int, bx_scheme_params
       type(bx_scheme_params), intent(in):: Scheme
     end function bx_set_scheme

     integer(c_int) function bx_finalize() bind(C, name='bx_finalize')
       import:: c_int
     end function bx_finalize

     type(c_ptr) function bx_last_error() bind(C, name='bx_last_error')
       import:: c_ptr
     end function bx_last_error

     integer(c_int) function bx_upload_state(State_VGB, nBlock) &
          bind(C, name='bx_upload_state')
       import:: c_int, c_double
       real(c_double), intent(in):: State_VGB(*)
       integer(c_int), value:: nBlock
     end function bx_upload_state

     integer(c_int) function bx_download_state(State_VGB, nBlock) &
          bind(C, name='bx_download_state')
       import:: c_int, c_double
       real(c_double), intent(out):: State_VGB(*)
       integer(c_int), value:: nBlock
     end function bx_download_state

     integer(c_int) function bx_calc_face_value(iBlock, DoResChangeOnly, &
          DoMonotoneRestrict) bind(C, name='bx_calc_face_value')
       import:: c_int
       integer(c_int), value:: iBlock, DoResChangeOnly, DoMonotoneRestrict
     end function bx_calc_face_value

     integer(c_int) function bx_calc_face_flux(DoResChangeOnly, iBlock) &
          bind(C, name='bx_calc_face_flux')
       import:: c_int
       integer(c_int), value:: DoResChangeOnly, iBlock
     end function bx_calc_face_flux

     integer(c_int) function bx_calc_source(iBlock) &
          bind(C, name='bx_calc_source')
       import:: c_int
       integer(c_int), value:: iBlock
     end function bx_calc_source

     integer(c_int) function bx_update_state(iBlock) &
          bind(C, name='bx_update_state')
       import:: c_int
       integer(c_int), value:: iBlock
     end function bx_update_state

     integer(c_int) function bx_calc_timestep(iBlock) &
          bind(C, name='bx_calc_timestep')
       import:: c_int
       integer(c_int), value:: iBlock
     end function bx_calc_timestep

     integer(c_int) function bx_set_stage(iStage) bind(C, name='bx_set_stage')
       import:: c_int
       integer(c_int), value:: iStage
     end function bx_set_stage

     integer(c_int) function bx_update_state_fast() &
          bind(C, name='bx_update_state_fast')
       import:: c_int
     end function bx_update_state_fast

     integer(c_int) function bx_exchange_messages(DoResChangeOnly) &
          bind(C, name='bx_exchange_messages')
       import:: c_int
       integer(c_int), value:: DoResChangeOnly
     end function bx_exchange_messages

     integer(c_int) function bx_set_global_timestep(TimeSimulationLimit, Dt) &
          bind(C, name='bx_set_global_timestep')
       import:: c_int, c_double
       real(c_double), value:: TimeSimulationLimit
       real(c_double), intent(out):: Dt
     end function bx_set_global_timestep
     integer(c_int) function bx_halo_bytes(iStage, BytesPerBlock) bind(C, name='bx_halo_bytes')
       import:: c_int
       integer(c_int), value:: iStage
       integer(c_int), intent(out):: BytesPerBlock
     end function bx_halo_bytes
     integer(c_int) function bx_halo_pack(iStage, iBlock_I, nBlock, Buf_dev) bind(C, name='bx_halo_pack')
       import:: c_int, c_ptr
       integer(c_int), value:: iStage, nBlock
       integer(c_int), intent(in):: iBlock_I(*)
       type(c_ptr), value:: Buf_dev
     end function bx_halo_pack
     integer(c_int) function bx_halo_unpack(iStage, iBlock_I, nBlock, Buf_dev) bind(C, name='bx_halo_unpack')
       import:: c_int, c_ptr
       integer(c_int), value:: iStage, nBlock
       integer(c_int), intent(in):: iBlock_I(*)
       type(c_ptr), value:: Buf_dev
     end function bx_halo_unpack
     integer(c_int) function bx_get_dtmin(DtMin) bind(C, name='bx_get_dtmin')
       import:: c_int, c_double
       real(c_double), intent(out):: DtMin
     end function bx_get_dtmin
     integer(c_int) function bx_set_dtmin(DtMin) bind(C, name='bx_set_dtmin')
       import:: c_int, c_double
       real(c_double), value:: DtMin
     end function bx_set_dtmin
     integer(c_int) function bx_end_step(tLimit) bind(C, name='bx_end_step')
       import:: c_int, c_double
       real(c_double), value:: tLimit
     end function bx_end_step

     integer(c_int) function bx_advance_explicit(DoCalcTimestep) &
          bind(C, name='bx_advance_explicit')
       import:: c_int
       integer(c_int), value:: DoCalcTimestep
     end function bx_advance_explicit

     integer(c_int) function bx_advance(nStep, TimeSimulationLimit) &
          bind(C, name='bx_advance')
       import:: c_int, c_double
       integer(c_int), value:: nStep
       real(c_double), value:: TimeSimulationLimit
     end function bx_advance

     integer(c_int) function bx_get_time(tSimulation, Dt, nStep) &
          bind(C, name='bx_get_time')
       import:: c_int, c_double
       real(c_double), intent(out):: tSimulation, Dt
       integer(c_int), intent(out):: nStep
     end function bx_get_time

     integer(c_int) function bx_set_time(tSimulation, nStep) &
          bind(C, name='bx_set_time')
       import:: c_int, c_double
       real(c_double), value:: tSimulation
       integer(c_int), value:: nStep
     end function bx_set_time
  end interface

  interface
     integer(c_int) function bx_get_neighbors(DiLevel_EB, jBlock_IEB) &
          bind(C, name='bx_get_neighbors')
       import:: c_int
       integer(c_int), intent(out):: DiLevel_EB(*), jBlock_IEB(*)
     end function bx_get_neighbors

     integer(c_int) function bx_set_graph_steps(nStepPerGraph) &
          bind(C, name='bx_set_graph_steps')
       import:: c_int
       integer(c_int), value:: nStepPerGraph
     end function bx_set_graph_steps

     integer(c_int) function bx_implicit_init(Params) &
          bind(C, name='bx_implicit_init')
       import:: c_int, bx_implicit_params
       type(bx_implicit_params), intent(in):: Params
     end function bx_implicit_init

     integer(c_int) function bx_advance_part_impl(TimeSimulationLimit, Stats) &
          bind(C, name='bx_advance_part_impl')
       import:: c_int, c_double, bx_krylov_stats
       real(c_double), value:: TimeSimulationLimit
       type(bx_krylov_stats), intent(out):: Stats
     end function bx_advance_part_impl

     ! DtMax_B for write_restart_file / from read_restart_file
     ! (src/ModRestartFile.f90:682-833)
     integer(c_int) function bx_get_block_dt(DtMax_B) bind(C, name='bx_get_block_dt')
       import:: c_int, c_double
       real(c_double), intent(out):: DtMax_B(*)
     end function bx_get_block_dt
     integer(c_int) function bx_set_block_dt(DtMax_B) bind(C, name='bx_set_block_dt')
       import:: c_int, c_double
       real(c_double), intent(in):: DtMax_B(*)
     end function bx_set_block_dt

     ! prepare_amr + do_amr (src/ModAMR.f90:171-386): criteria, new tree,
     ! state moved onto it; the new block list comes from bx_get_grid
     integer(c_int) function bx_do_amr(Params, nBlockNew, IsChanged) bind(C, name='bx_do_amr')
       import:: c_int, bx_amr_params
       type(bx_amr_params), intent(in):: Params
       integer(c_int), intent(out):: nBlockNew, IsChanged
     end function bx_do_amr
     integer(c_int) function bx_get_grid(iLevelCoord_IB) bind(C, name='bx_get_grid')
       import:: c_int
       integer(c_int), intent(out):: iLevelCoord_IB(*)
     end function bx_get_grid
     ! amr_criteria (src/ModAMR.f90:388-723): Crit_IB(nCrit, nBlock)
     integer(c_int) function bx_amr_criteria(nCrit, iTypeCrit_I, Crit_IB) bind(C, name='bx_amr_criteria')
       import:: c_int, c_double
       integer(c_int), value:: nCrit
       integer(c_int), intent(in):: iTypeCrit_I(*)
       real(c_double), intent(out):: Crit_IB(*)
     end function bx_amr_criteria
     ! regrid_batl with a caller-made tree: iRemap_IB(10, nBlockNew)
     integer(c_int) function bx_regrid(Grid, iRemap_IB) bind(C, name='bx_regrid')
       import:: c_int, bx_grid_desc
       type(bx_grid_desc), intent(in):: Grid
       integer(c_int), intent(in):: iRemap_IB(*)
     end function bx_regrid

     ! advance_semi_impl (src/ModSemiImplicit.f90:240), TypeSemiImplicit = parcond
     integer(c_int) function bx_heat_init(Params, Te, Bhat, Used) bind(C, name='bx_heat_init')
       import:: c_int, c_double, c_signed_char, bx_heat_params
       type(bx_heat_params), intent(in):: Params
       real(c_double), intent(in):: Te(*), Bhat(*)
       integer(c_signed_char), intent(in):: Used(*)
     end function bx_heat_init
     integer(c_int) function bx_advance_semi_impl(Stats) bind(C, name='bx_advance_semi_impl')
       import:: c_int, bx_krylov_stats
       type(bx_krylov_stats), intent(out):: Stats
     end function bx_advance_semi_impl
     integer(c_int) function bx_heat_get_te(Te) bind(C, name='bx_heat_get_te')
       import:: c_int, c_double
       real(c_double), intent(out):: Te(*)
     end function bx_heat_get_te
  end interface

end module bx200_interface
