!ISO_C_BINDING interface to the B200 GAMERA step library (include/gamgpu.h).
!
!A Fortran gamApp_T keeps its Model_T/Grid_T/State_T and Hatch. After Hatch it calls gam_gpu_create
!with the arrays Hatch produced; stepGamera becomes gam_gpu_step and gamAdvanceModel gam_gpu_advance,
!and the host arrays are refreshed only at IO/restart points with gam_gpu_sync_to_host.
!Array arguments are the Fortran arrays themselves (contiguous, column-major, ghosts included).
!The derived types below are field-for-field the C structs of include/gamgpu.h (same order, same C
!types), so bind(C) gives them the C layout.
module gamgpu_mod
    use, intrinsic :: iso_c_binding
    implicit none

    integer(c_int), parameter :: GAM_OK = 0, GAM_ERR_NAN = 1, GAM_ERR_DT_COLLAPSE = 2, GAM_ERR_CUDA = 3, &
                                 GAM_ERR_TIMEOUT = 4, GAM_ERR_UNSUPPORTED = 5, GAM_ERR_ARG = 6
    integer(c_int), parameter :: GAM_FP64 = 0, GAM_FP32FLUX = 1
    integer(c_int), parameter :: GAM_BC_PERIODIC = 0, GAM_BC_ZEROGRAD = 1, GAM_BC_LFMPOLE = 2, GAM_BC_LFMBW = 3, &
                                 GAM_BC_HALO = 4, GAM_BC_ION = 5, GAM_BC_WIND = 6
    integer(c_int), parameter :: GAM_NMSPH = 23
    integer(c_int), parameter :: GAM_RING_PLM = 0, GAM_RING_PPM = 1, GAM_RING_PCM = 2
    integer(c_int), parameter :: GAM_RM_8CENT = 0, GAM_RM_7UP = 1
    integer(c_int), parameter :: GAM_HALO_STATE = 1, GAM_HALO_OSTATE = 2, GAM_HALO_BXYZ = 4
    integer(c_int), parameter :: GAM_SYNC_STATE = 1, GAM_SYNC_OSTATE = 2
    integer(c_int), parameter :: GAM_SLICE_FAT = 1

    !Model_T fields the step reads (src/base/types/gamtypes.F90:71-146); C: gam_model_c
    type, bind(C) :: gam_model_c
        integer(c_int) :: Nip, Njp, Nkp, nG
        real(c_double) :: gamma, CFL, pdmb, Vd0, cHogH, cHogM, Ca, dFloor, pFloor, limDT0
        real(c_double) :: t, tFin, dt, dt0
        integer(c_int) :: ts
        integer(c_int) :: doMHD, doBoris, do25D, doLFMLim, rmeth, fixedTimestep
        integer(c_int) :: doBackground, doGrav, doResistive, doRing, doMultiF, doAB3, nSpc, hasHooks
        integer(c_int) :: bc(6)
        ! ring averaging about the LFM axis (Model%Ring as InitRings set it, ringutils.F90:37-226)
        integer(c_int) :: ringNumR
        integer(c_int) :: ringNch(32)
        integer(c_int) :: ringRecon
        integer(c_int) :: ringDoS, ringDoE
        ! the LFM blast wave's predictor fix, the gas of its GAM_BC_LFMBW shells, its dt domain (ICs/lfmbw.F90)
        integer(c_int) :: predFixLFM
        real(c_double) :: bwD0, bwP0
        integer(c_int) :: dtActive
    end type gam_model_c

    !Grid_T metric arrays (gamtypes.F90:163-245) as C addresses; C: gam_grid_c
    type, bind(C) :: gam_grid_c
        type(c_ptr) :: xyzcc, xfc, di, dj, dk, volume, face, edge, Tf, Te, Teb
        ! background field (Grid%fcB0, edgB0, B0, bFlux0, dpB0); c_null_ptr unless Model%doBackground
        type(c_ptr) :: fcB0 = c_null_ptr, edgB0 = c_null_ptr, B0 = c_null_ptr, bFlux0 = c_null_ptr, dpB0 = c_null_ptr
        type(c_ptr) :: xyz = c_null_ptr   ! Grid%xyz, for the slice output
    end type gam_grid_c

    !C: gam_status_c
    type, bind(C) :: gam_status_c
        real(c_double) :: t, dt, dt0, time, otime
        integer(c_int) :: ts
        integer(c_int) :: status
        integer(c_int) :: nanCells
        integer(c_int) :: precision
        integer(c_long_long) :: kernelLaunches
    end type gam_status_c

    interface
        integer(c_int) function gam_gpu_create(h, m, g, gas, magflux, bxyz, ogas, omagflux, obxyz, time, otime) &
                bind(C, name="gam_gpu_create")
            import :: c_int, c_ptr, c_double, gam_model_c, gam_grid_c
            type(c_ptr), intent(out) :: h
            type(gam_model_c), intent(in) :: m
            type(gam_grid_c), intent(in) :: g
            real(c_double), intent(in) :: gas(*), magflux(*), bxyz(*), ogas(*), omagflux(*), obxyz(*)
            real(c_double), value :: time, otime
        end function gam_gpu_create

        integer(c_int) function gam_gpu_create_from_corners(h, m, xyz, ic) bind(C, name="gam_gpu_create_from_corners")
            import :: c_int, c_ptr, c_double, gam_model_c
            type(c_ptr), intent(out) :: h
            type(gam_model_c), intent(in) :: m
            real(c_double), intent(in) :: xyz(*)
            integer(c_int), value :: ic
        end function gam_gpu_create_from_corners

        integer(c_int) function gam_gpu_create_from_corners_ic(h, m, xyz, ic, icPar, nPar) &
                bind(C, name="gam_gpu_create_from_corners_ic")
            import :: c_int, c_ptr, c_double, gam_model_c
            type(c_ptr), intent(out) :: h
            type(gam_model_c), intent(in) :: m
            real(c_double), intent(in) :: xyz(*), icPar(*)
            integer(c_int), value :: ic, nPar
        end function gam_gpu_create_from_corners_ic

        integer(c_int) function gam_gpu_create_from_corners_b0(h, m, xyz, ic, b0Kind, b0Par) &
                bind(C, name="gam_gpu_create_from_corners_b0")
            import :: c_int, c_ptr, c_double, gam_model_c
            type(c_ptr), intent(out) :: h
            type(gam_model_c), intent(in) :: m
            real(c_double), intent(in) :: xyz(*), b0Par(4)
            integer(c_int), value :: ic, b0Kind
        end function gam_gpu_create_from_corners_b0

        integer(c_int) function gam_gpu_step(h, dt, ts, t) bind(C, name="gam_gpu_step")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: dt, t
            integer(c_int), intent(out) :: ts
        end function gam_gpu_step

        integer(c_int) function gam_gpu_advance(h, dtAdv) bind(C, name="gam_gpu_advance")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), value :: dtAdv
        end function gam_gpu_advance

        integer(c_int) function gam_gpu_run_steps(h, n) bind(C, name="gam_gpu_run_steps")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: n
        end function gam_gpu_run_steps

        integer(c_int) function gam_gpu_run_steps_timed(h, n, ms) bind(C, name="gam_gpu_run_steps_timed")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: n
            real(c_double), intent(out) :: ms
        end function gam_gpu_run_steps_timed

        integer(c_int) function gam_gpu_sync_to_host(h, what, gas, magflux, bxyz, ogas, omagflux) &
                bind(C, name="gam_gpu_sync_to_host")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: what
            real(c_double), intent(inout) :: gas(*), magflux(*), bxyz(*), ogas(*), omagflux(*)
        end function gam_gpu_sync_to_host

        integer(c_int) function gam_gpu_sync_to_device(h, what, gas, magflux, bxyz, ogas, omagflux, obxyz, &
                                                       time, otime) bind(C, name="gam_gpu_sync_to_device")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: what
            real(c_double), intent(in) :: gas(*), magflux(*), bxyz(*), ogas(*), omagflux(*), obxyz(*)
            real(c_double), value :: time, otime
        end function gam_gpu_sync_to_device

        integer(c_int) function gam_gpu_get_status(h, s) bind(C, name="gam_gpu_get_status")
            import :: c_int, c_ptr, gam_status_c
            type(c_ptr), value :: h
            type(gam_status_c), intent(out) :: s
        end function gam_gpu_get_status

        integer(c_int) function gam_gpu_set_scalars(h, t, dt, dt0, ts, time, otime) bind(C, name="gam_gpu_set_scalars")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), value :: t, dt, dt0, time, otime
            integer(c_int), value :: ts
        end function gam_gpu_set_scalars

        integer(c_int) function gam_gpu_set_precision(h, mode) bind(C, name="gam_gpu_set_precision")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: mode
        end function gam_gpu_set_precision

        integer(c_int) function gam_gpu_set_tile(h, what, val) bind(C, name="gam_gpu_set_tile")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: what, val
        end function gam_gpu_set_tile

        ! the magnetosphere's hooks and gravity (voltron/ICs/earthcmi.F90 initUser) for a problem created from
        ! Hatch's arrays; par = the GAM_NMSPH code-unit values (include/gamgpu.h, GAM_IC_MAGSPHERE)
        integer(c_int) function gam_gpu_set_magnetosphere(h, par, n) bind(C, name="gam_gpu_set_magnetosphere")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: par(*)
            integer(c_int), value :: n
        end function gam_gpu_set_magnetosphere

        integer(c_int) function gam_gpu_divb(h, tot) bind(C, name="gam_gpu_divb")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: tot
        end function gam_gpu_divb

        ! DivB without a handle or any allocation; magflux/bflux0/tot are device addresses (bflux0 may be
        ! c_null_ptr). For hosts whose device arrays belong to another runtime.
        integer(c_int) function gam_divb_noalloc(magflux, bflux0, Nip, Njp, Nkp, nG, tot) &
                bind(C, name="gam_divb_noalloc")
            import :: c_int, c_ptr
            type(c_ptr), value :: magflux, bflux0, tot
            integer(c_int), value :: Nip, Njp, Nkp, nG
        end function gam_divb_noalloc

        ! any Solver/Grid array by its reference name ("StateHf"/"hgas", "Efld", "dGasH", ...) into out(1:n)
        integer(c_int) function gam_gpu_fetch(h, name, out, n) bind(C, name="gam_gpu_fetch")
            import :: c_int, c_ptr, c_double, c_char, c_long_long
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: name(*)
            real(c_double), intent(out) :: out(*)
            integer(c_long_long), value :: n
        end function gam_gpu_fetch

        ! the variables writeSlc writes (src/gamera/gioH5.F90:255-602), computed on the device
        integer(c_long_long) function gam_gpu_slice_count(h, flags) bind(C, name="gam_gpu_slice_count")
            import :: c_int, c_ptr, c_long_long
            type(c_ptr), value :: h
            integer(c_int), value :: flags
        end function gam_gpu_slice_count

        integer(c_int) function gam_gpu_slice_begin(h, flags, out, n) bind(C, name="gam_gpu_slice_begin")
            import :: c_int, c_ptr, c_double, c_long_long
            type(c_ptr), value :: h
            integer(c_int), value :: flags
            real(c_double), intent(out) :: out(*)   ! pinned or pageable; filled by gam_gpu_slice_wait
            integer(c_long_long), value :: n
        end function gam_gpu_slice_begin

        integer(c_int) function gam_gpu_slice_wait(h) bind(C, name="gam_gpu_slice_wait")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function gam_gpu_slice_wait

        integer(c_int) function gam_gpu_slice(h, flags, out, n) bind(C, name="gam_gpu_slice")
            import :: c_int, c_ptr, c_double, c_long_long
            type(c_ptr), value :: h
            integer(c_int), value :: flags
            real(c_double), intent(out) :: out(*)
            integer(c_long_long), value :: n
        end function gam_gpu_slice

        subroutine gam_gpu_destroy(h) bind(C, name="gam_gpu_destroy")
            import :: c_ptr
            type(c_ptr), value :: h
        end subroutine gam_gpu_destroy

        ! k-decomposed runs, one rank per GPU (stepGamera_mpi, src/gamera/mpi/gamapp_mpi.F90:665-692).
        ! dtWords and the halo buffers are device addresses.
        integer(c_int) function gam_gpu_step_local(h, dtWords) bind(C, name="gam_gpu_step_local")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, dtWords
        end function gam_gpu_step_local

        integer(c_int) function gam_gpu_step_bcs(h, dtWords) bind(C, name="gam_gpu_step_bcs")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, dtWords
        end function gam_gpu_step_bcs

        integer(c_int) function gam_gpu_step_ghosts(h) bind(C, name="gam_gpu_step_ghosts")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function gam_gpu_step_ghosts

        integer(c_int) function gam_gpu_calcdt_local(h, dtWords) bind(C, name="gam_gpu_calcdt_local")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, dtWords
        end function gam_gpu_calcdt_local

        integer(c_int) function gam_gpu_calcdt_finish(h, dtWords) bind(C, name="gam_gpu_calcdt_finish")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, dtWords
        end function gam_gpu_calcdt_finish

        integer(c_int) function gam_gpu_halo_bytes(h, side, what, sendBytes, recvBytes) &
                bind(C, name="gam_gpu_halo_bytes")
            import :: c_int, c_ptr, c_long_long
            type(c_ptr), value :: h
            integer(c_int), value :: side, what
            integer(c_long_long), intent(out) :: sendBytes, recvBytes
        end function gam_gpu_halo_bytes

        integer(c_int) function gam_gpu_halo_pack(h, side, what, dst) bind(C, name="gam_gpu_halo_pack")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, dst
            integer(c_int), value :: side, what
        end function gam_gpu_halo_pack

        integer(c_int) function gam_gpu_halo_unpack(h, side, what, src) bind(C, name="gam_gpu_halo_unpack")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, src
            integer(c_int), value :: side, what
        end function gam_gpu_halo_unpack

        integer(c_int) function gam_gpu_stream(h, stream) bind(C, name="gam_gpu_stream")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            type(c_ptr), intent(out) :: stream
        end function gam_gpu_stream
    end interface

contains

    !Fill the C mirror of Model_T. The dummy arguments carry the reference's names (Model_T fields,
    !gamtypes.F90:71-146; pdmb of recon.F90:28; dFloor/pFloor of gdefs.F90:12), so a gamApp_T caller
    !passes its own values, e.g. doLFMLim=Model%doLFMLim and
    !rmeth=merge(GAM_RM_7UP, GAM_RM_8CENT, associated(GetLRs, Up7LRs)) for the sim/rmeth choice of
    !initModel (init.F90:450-462). hasHooks is 1 when any user hook other than the LFM blast wave's
    !PredFix is associated. Rings and the LFM blast wave's fields are set with gamgpu_set_ring and
    !gamgpu_set_lfmbw.
    function gamgpu_model(Nip, Njp, Nkp, nG, gamma, CFL, pdmb, Vd0, doHogs, cHogH, cHogM, Ca, dFloor, pFloor, &
                          limDT0, t, tFin, dt, dt0, ts, doMHD, doBoris, do25D, doLFMLim, rmeth, fixedTimestep, &
                          doBackground, doGrav, doResistive, doRing, doMultiF, doAB3, nSpc, hasHooks, bcs) result(m)
        integer, intent(in) :: Nip, Njp, Nkp, nG, ts, rmeth, nSpc, bcs(6)
        real(c_double), intent(in) :: gamma, CFL, pdmb, Vd0, cHogH, cHogM, Ca, dFloor, pFloor, limDT0
        real(c_double), intent(in) :: t, tFin, dt, dt0
        logical, intent(in) :: doHogs, doMHD, doBoris, do25D, doLFMLim, fixedTimestep
        logical, intent(in) :: doBackground, doGrav, doResistive, doRing, doMultiF, doAB3, hasHooks
        type(gam_model_c) :: m
        m%Nip = Nip; m%Njp = Njp; m%Nkp = Nkp; m%nG = nG
        m%gamma = gamma; m%CFL = CFL; m%pdmb = pdmb; m%Vd0 = Vd0
        ! doHogs = F is the HOGS terms with zero coefficients (stress.F90)
        m%cHogH = merge(cHogH, 0.0_c_double, doHogs); m%cHogM = merge(cHogM, 0.0_c_double, doHogs)
        m%Ca = Ca; m%dFloor = dFloor; m%pFloor = pFloor; m%limDT0 = limDT0
        m%t = t; m%tFin = tFin; m%dt = dt; m%dt0 = dt0; m%ts = ts
        m%doMHD = merge(1, 0, doMHD); m%doBoris = merge(1, 0, doBoris); m%do25D = merge(1, 0, do25D)
        m%doLFMLim = merge(1, 0, doLFMLim); m%rmeth = rmeth; m%fixedTimestep = merge(1, 0, fixedTimestep)
        m%doBackground = merge(1, 0, doBackground); m%doGrav = merge(1, 0, doGrav)
        m%doResistive = merge(1, 0, doResistive); m%doRing = merge(1, 0, doRing)
        m%doMultiF = merge(1, 0, doMultiF); m%doAB3 = merge(1, 0, doAB3)
        m%nSpc = nSpc; m%hasHooks = merge(1, 0, hasHooks)
        m%bc = bcs
        m%ringNumR = 0; m%ringNch = 0; m%ringRecon = GAM_RING_PPM; m%ringDoS = 0; m%ringDoE = 0
        m%predFixLFM = 0; m%bwD0 = 1.0_c_double; m%bwP0 = 0.1_c_double; m%dtActive = 0
    end function gamgpu_model

    !Ring averaging about the LFM axis: Model%Ring%NumR, Nch(1:NumR) and the ring/rngrec choice
    !(GAM_RING_*), with Ring%doS/doE (both true on an untiled grid)
    subroutine gamgpu_set_ring(m, NumR, Nch, recon, doS, doE)
        type(gam_model_c), intent(inout) :: m
        integer, intent(in) :: NumR, Nch(:), recon
        logical, intent(in) :: doS, doE
        m%ringNumR = NumR
        m%ringNch = 0
        m%ringNch(1:NumR) = Nch(1:NumR)
        m%ringRecon = recon
        m%ringDoS = merge(1, 0, doS); m%ringDoE = merge(1, 0, doE)
    end subroutine gamgpu_set_ring

    !The LFM blast wave (src/gamera/ICs/lfmbw.F90): its predictor fix, the D0/P0 of its fixed shells
    !and its timestep domain over the active cells
    subroutine gamgpu_set_lfmbw(m, D0, P0)
        type(gam_model_c), intent(inout) :: m
        real(c_double), intent(in) :: D0, P0
        m%predFixLFM = 1; m%bwD0 = D0; m%bwP0 = P0; m%dtActive = 1
    end subroutine gamgpu_set_lfmbw

end module gamgpu_mod
