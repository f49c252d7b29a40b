!ISO_C_BINDING interface to the B200 GAMERA step library (include/gamgpu.h).
!
!A Fortran gamApp_T keeps its Model_T/Grid_T/State_T and Hatch. After Hatch it calls gamgpu_create
!with the arrays Hatch produced; stepGamera becomes gamgpu_step (see stepGamera_gpu below) and the
!host arrays are refreshed only at IO/restart points with gam_gpu_sync_to_host.
!Array arguments are the Fortran arrays themselves (contiguous, column-major, ghosts included).
module gamgpu_mod
    use, intrinsic :: iso_c_binding
    implicit none

    integer(c_int), parameter :: GAM_OK = 0, GAM_ERR_NAN = 1, GAM_ERR_DT_COLLAPSE = 2, GAM_ERR_CUDA = 3, &
                                 GAM_ERR_TIMEOUT = 4, GAM_ERR_UNSUPPORTED = 5, GAM_ERR_ARG = 6
    integer(c_int), parameter :: GAM_FP64 = 0, GAM_FP32FLUX = 1
    integer(c_int), parameter :: GAM_BC_PERIODIC = 0, GAM_BC_ZEROGRAD = 1, GAM_BC_LFMPOLE = 2, GAM_BC_LFMBW = 3, &
                                 GAM_BC_HALO = 4
    integer(c_int), parameter :: GAM_HALO_STATE = 1, GAM_HALO_OSTATE = 2, GAM_HALO_BXYZ = 4
    integer(c_int), parameter :: GAM_SYNC_STATE = 1, GAM_SYNC_OSTATE = 2

    type, bind(C) :: gam_model_c
        integer(c_int) :: Nip, Njp, Nkp, nG
        real(c_double) :: gamma, CFL, pdmb, Vd0, cHogH, cHogM, Ca, dFloor, pFloor, limDT0
        real(c_double) :: t, tFin, dt, dt0
        integer(c_int) :: ts
        integer(c_int) :: doMHD, doBoris, do25D, doLFMLim, rmeth, fixedTimestep
        integer(c_int) :: doBackground, doGrav, doResistive, doRing, doMultiF, doAB3, nSpc, hasHooks
        integer(c_int) :: bc(6)
    end type gam_model_c

    type, bind(C) :: gam_grid_c
        type(c_ptr) :: xyzcc, xfc, di, dj, dk, volume, face, edge, Tf, Te, Teb
        ! background field (Grid%fcB0, edgB0, B0, bFlux0, dpB0); c_null_ptr unless Model%doBackground
        type(c_ptr) :: fcB0 = c_null_ptr, edgB0 = c_null_ptr, B0 = c_null_ptr, bFlux0 = c_null_ptr, dpB0 = c_null_ptr
        type(c_ptr) :: xyz = c_null_ptr   ! Grid%xyz, for the slice output
    end type gam_grid_c

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

        integer(c_int) function gam_gpu_sync_to_host(h, what, gas, magflux, bxyz, ogas, omagflux) &
                bind(C, name="gam_gpu_sync_to_host")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: what
            real(c_double), intent(inout) :: gas(*), magflux(*), bxyz(*), ogas(*), omagflux(*)
        end function gam_gpu_sync_to_host

        integer(c_int) function gam_gpu_set_precision(h, mode) bind(C, name="gam_gpu_set_precision")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: mode
        end function gam_gpu_set_precision

        integer(c_int) function gam_gpu_divb(h, tot) bind(C, name="gam_gpu_divb")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: tot
        end function gam_gpu_divb

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

    !Fill the C mirror of Model_T from the reference's Model_T fields (gamtypes.F90:71-146).
    !(Kept as plain arguments so this module does not depend on gamtypes; a gamApp_T caller passes
    ! Model%gamma, Model%CFL, ... and the BC kinds it allocated.)
    function gamgpu_model(Nip, Njp, Nkp, gamma, CFL, pdmb, Vd0, cHogH, cHogM, Ca, t, tFin, dt, dt0, ts, &
                          doMHD, doBoris, do25D, bcs) result(m)
        integer, intent(in) :: Nip, Njp, Nkp, ts, bcs(6)
        real(c_double), intent(in) :: gamma, CFL, pdmb, Vd0, cHogH, cHogM, Ca, t, tFin, dt, dt0
        logical, intent(in) :: doMHD, doBoris, do25D
        type(gam_model_c) :: m
        m%Nip = Nip; m%Njp = Njp; m%Nkp = Nkp; m%nG = 4
        m%gamma = gamma; m%CFL = CFL; m%pdmb = pdmb; m%Vd0 = Vd0; m%cHogH = cHogH; m%cHogM = cHogM
        m%Ca = Ca; m%dFloor = 1.0d-12; m%pFloor = 1.0d-12; m%limDT0 = 1.0d-3
        m%t = t; m%tFin = tFin; m%dt = dt; m%dt0 = dt0; m%ts = ts
        m%doMHD = merge(1, 0, doMHD); m%doBoris = merge(1, 0, doBoris); m%do25D = merge(1, 0, do25D)
        m%doLFMLim = 1; m%rmeth = 0; m%fixedTimestep = 0
        m%doBackground = 0; m%doGrav = 0; m%doResistive = 0; m%doRing = 0; m%doMultiF = 0; m%doAB3 = 0
        m%nSpc = 0; m%hasHooks = 0
        m%bc = bcs
    end function gamgpu_model

end module gamgpu_mod
