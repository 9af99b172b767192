    ! GPU_TimeStep.f90 -- B200 TimeStep for QGN_Module.
    !
    ! Drop-in for the scheme include of TimeStep: replace
    !     include "ARK43_QGLeith.f90"
    ! at QGN_Module.f90:306 by
    !     include "GPU_TimeStep.f90"
    ! and link libqgn_b200.so.  The scheme is chosen with QGN_SCHEME below (the values of
    ! include/qgn_gpu.h: 0 ARK43_QGLeith, 1 ARK43, 2 BSRK3, 3 RK4, 4 AB3); the physical
    ! constants come from parameters.f90 and the module state (H, S, uBar, qyBar, Modes,
    ! EVals) built by Initialize, by host association.  TimeStep's own
    ! `call DeAlias(q_hat)` (QGN_Module.f90:307) still follows this include.
    !
    ! The device context is created on the first call and kept for the whole run (the
    ! counterpart of the `save` variables of the scheme include files).
    integer(c_int), parameter :: QGN_SCHEME = 0_c_int
    integer(c_int), parameter :: QGN_PRECISION = 0_c_int   ! 0 FP64, 1 mixed
    type, bind(C) :: qgn_params_t
        integer(c_int) :: nx, ny, nz, is_explicit
        real(c_double) :: Lx, Ly, Htot, f0, beta, A2, A8, r0, C_d, TOL, dt_max
        integer(c_int) :: max_rejects, reserved
    end type qgn_params_t
    interface
        integer(c_int) function qgn_create(p, H_, S_, uBar_, qyBar_, Modes_, EVals_, scheme, precision, ctx) &
                bind(C, name="qgn_create")
            import :: c_int, c_double, c_ptr, qgn_params_t
            type(qgn_params_t), intent(in) :: p
            real(c_double), intent(in) :: H_(*), S_(*), uBar_(*), qyBar_(*), Modes_(*), EVals_(*)
            integer(c_int), value :: scheme, precision
            type(c_ptr), intent(out) :: ctx
        end function qgn_create
        integer(c_int) function qgn_step(ctx, q, t_, dt_) bind(C, name="qgn_step")
            import :: c_int, c_double, c_double_complex, c_ptr
            type(c_ptr), value :: ctx
            complex(c_double_complex), intent(inout) :: q(*)
            real(c_double), intent(inout) :: t_, dt_
        end function qgn_step
        type(c_ptr) function qgn_last_error(ctx) bind(C, name="qgn_last_error")
            import :: c_ptr
            type(c_ptr), value :: ctx
        end function qgn_last_error
    end interface
    type(c_ptr), save :: qgn_ctx = c_null_ptr
    type(qgn_params_t) :: qgn_p
    integer(c_int) :: qgn_status

    if (.not. c_associated(qgn_ctx)) then
        qgn_p = qgn_params_t(nx, ny, nz, merge(1_c_int, 0_c_int, is_explicit), Lx, Ly, Htot, f0, beta, &
                             A2, A8, r0, C_d, TOL, dt_max, 0_c_int, 0_c_int)
        qgn_status = qgn_create(qgn_p, H, S, uBar, qyBar, Modes, EVals, QGN_SCHEME, QGN_PRECISION, qgn_ctx)
        if (qgn_status /= 0_c_int) then
            print *, 'qgn_create failed with status ', qgn_status
            error stop
        end if
    end if
    qgn_status = qgn_step(qgn_ctx, q_hat, t, dt)
    if (qgn_status /= 0_c_int) then
        print *, 'qgn_step failed with status ', qgn_status
        error stop
    end if
