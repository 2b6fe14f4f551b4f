! rp_gpu_mod.f90 -- ISO_C_BINDING interface of the B200 particle step.
!
! The Fortran driver of ROMSPath (ROMSPath.f90) uses this module to call the
! C ABI of include/romspath_gpu.h: one bind(C) interface per entry point and
! one bind(C) derived type per C struct, field for field.  The call that
! replaces update_particles is rp_step (ROMSPath.f90:529, from
! run_Internal_Timestep); rp_upload_frame follows each updateHydro
! (ROMSPath.f90:307-309, 492); rp_create / rp_locate_particles sit in
! ini_ROMSPath (ROMSPath.f90:182-461).
!
! Conventions of the bindings:
!  * rp_ctx* is type(c_ptr), value; rp_ctx** (rp_create's output) is a
!    type(c_ptr) passed by reference.
!  * Required arrays are assumed-size arrays of the matching C kind; an
!    argument the C side allows to be NULL is type(c_ptr), value (pass
!    c_null_ptr, or c_loc(x) of a target array).
!  * uint32_t / uint64_t arguments are integer(c_int32_t) / (c_int64_t):
!    the same bits.
module rp_gpu_mod
  use iso_c_binding
  implicit none

  integer, parameter :: RP_MAXNGRID = 5
  integer(c_int), parameter :: RP_OK = 0, RP_ERR_ARG = -1, RP_ERR_CUDA = -2, RP_ERR_STATE = -3
  integer(c_int), parameter :: RP_ERR_NOMEM = -4, RP_ERR_UNSUPPORTED = -5, RP_ERR_NOEXT = -6
  integer(c_int32_t), parameter :: RP_FIELD_F64 = 0, RP_FIELD_F32 = 1
  integer(c_int32_t), parameter :: RP_FIELD_MIXED = 2, RP_FIELD_MIXED_I16 = 3
  integer(c_int32_t), parameter :: RP_FLAG_OOB = 1, RP_FLAG_NODE = 2, RP_FLAG_WBOT = 4
  integer(c_int32_t), parameter :: RP_FLAG_WTOP = 8, RP_FLAG_SPLINE = 16
  integer(c_int32_t), parameter :: RP_DIAG_SALTTEMP = 1, RP_DIAG_SALTTEMP_MEAN = 2, RP_DIAG_BOTTOM = 4
  integer(c_int64_t), parameter :: RP_NOALLOC_MAX_PARTICLES = 1048576_c_int64_t

  type, bind(C) :: rp_params
    integer(c_int32_t) :: numpar, idt, dt, scheme, nsb, vturb_on, hturb_on
    integer(c_int32_t) :: open_ocean_boundary, behavior, stokes, field_dtype, spline_max_iter
    real(c_double) :: vertdist
    real(c_double) :: serr, smth, sub, deltat, aksback
    real(c_double) :: constant_hturb(RP_MAXNGRID)
    integer(c_int64_t) :: seed
    integer(c_int32_t) :: device
    integer(c_int32_t) :: reserved(7)
  end type rp_params

  type, bind(C) :: rp_grid
    integer(c_int32_t) :: xi_rho, eta_rho
    integer(c_int32_t) :: n_rho
    integer(c_int32_t) :: vtransform
    real(c_double) :: hc
    type(c_ptr) :: h, pm, pn
    type(c_ptr) :: mask_rho
    type(c_ptr) :: mask_u
    type(c_ptr) :: mask_v
    type(c_ptr) :: s_rho, cs_r
    type(c_ptr) :: s_w, cs_w
    type(c_ptr) :: scl, off
  end type rp_grid

  type, bind(C) :: rp_frame
    integer(c_int32_t) :: f32
    type(c_ptr) :: zeta, u, v, w, aks
    type(c_ptr) :: su, sv
    type(c_ptr) :: salt, temp, bustr, bvstr
    type(c_ptr) :: wetdry_rho, wetdry_u, wetdry_v
    type(c_ptr) :: turbaccel, turbvort, waveaccelu, waveaccelv
  end type rp_frame

  type, bind(C) :: rp_behavior
    integer(c_int32_t) :: behavior, process_va, process_wa, va_flag
    real(c_double) :: swimfast
    real(c_double) :: initsize
    real(c_double) :: vort_cr, vort_sat, b0pv, b1pv, b0wv, b1w
    real(c_double) :: acc_cr, acc_sat, b0pa, b1pa, b0wa
  end type rp_behavior

  type, bind(C) :: rp_device_state
    integer(c_int64_t) :: n
    type(c_ptr) :: x, y, z, age, dob, status, wd, zeta, bath
    type(c_ptr) :: gid
    type(c_ptr) :: isin
    type(c_ptr) :: pid, flags
    type(c_ptr) :: stream
  end type rp_device_state

  type, bind(C) :: rp_adj_step
    real(c_double) :: ex(3)
    real(c_double) :: ix(3)
    integer(c_int32_t) :: ets
    integer(c_int32_t) :: frame_b, frame_c, frame_f
    integer(c_int64_t) :: step_index
  end type rp_adj_step

  interface

    ! ---- context, frames, particles (ini_ROMSPath, updateHydro, par columns)

    integer(c_int) function rp_create(params, ngrid, grids, out) bind(C, name="rp_create")
      import :: c_int, c_int32_t, c_ptr, rp_params, rp_grid
      type(rp_params), intent(in) :: params
      integer(c_int32_t), value :: ngrid
      type(rp_grid), intent(in) :: grids(*)
      type(c_ptr), intent(out) :: out
    end function rp_create

    integer(c_int) function rp_upload_frame(ctx, ng, slot, zeta, u, v, w, aks, su, sv) &
        bind(C, name="rp_upload_frame")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ng, slot
      real(c_double), intent(in) :: zeta(*), u(*), v(*), w(*), aks(*)
      type(c_ptr), value :: su, sv
    end function rp_upload_frame

    integer(c_int) function rp_upload_frame_f32(ctx, ng, slot, zeta, u, v, w, aks, su, sv) &
        bind(C, name="rp_upload_frame_f32")
      import :: c_int, c_int32_t, c_ptr, c_float
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ng, slot
      real(c_float), intent(in) :: zeta(*), u(*), v(*), w(*), aks(*)
      type(c_ptr), value :: su, sv
    end function rp_upload_frame_f32

    integer(c_int) function rp_upload_frame_ext(ctx, ng, slot, zeta, u, v, w, aks, su, sv, &
        salt, temp, bustr, bvstr) bind(C, name="rp_upload_frame_ext")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ng, slot
      real(c_double), intent(in) :: zeta(*), u(*), v(*), w(*), aks(*)
      type(c_ptr), value :: su, sv, salt, temp, bustr, bvstr
    end function rp_upload_frame_ext

    integer(c_int) function rp_upload_frame_ext_f32(ctx, ng, slot, zeta, u, v, w, aks, su, sv, &
        salt, temp, bustr, bvstr) bind(C, name="rp_upload_frame_ext_f32")
      import :: c_int, c_int32_t, c_ptr, c_float
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ng, slot
      real(c_float), intent(in) :: zeta(*), u(*), v(*), w(*), aks(*)
      type(c_ptr), value :: su, sv, salt, temp, bustr, bvstr
    end function rp_upload_frame_ext_f32

    integer(c_int) function rp_upload_frame_desc(ctx, ng, slot, frame) bind(C, name="rp_upload_frame_desc")
      import :: c_int, c_int32_t, c_ptr, rp_frame
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ng, slot
      type(rp_frame), intent(in) :: frame
    end function rp_upload_frame_desc

    integer(c_int) function rp_set_particles(ctx, n, x, y, z, dob, age, status, gid, isin) &
        bind(C, name="rp_set_particles")
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: n
      real(c_double), intent(in) :: x(*), y(*), z(*), dob(*), age(*), status(*), gid(*)
      integer(c_int32_t), intent(in) :: isin(*)
    end function rp_set_particles

    integer(c_int) function rp_locate_particles(ctx, n, ipos, jpos, z, dob, t_b) &
        bind(C, name="rp_locate_particles")
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: n
      real(c_double), intent(in) :: ipos(*), jpos(*), z(*), dob(*)
      integer(c_int32_t), value :: t_b
    end function rp_locate_particles

    integer(c_int) function rp_set_grid_angle(ctx, ng, angle, spherical) bind(C, name="rp_set_grid_angle")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ng
      type(c_ptr), value :: angle
      integer(c_int32_t), value :: spherical
    end function rp_set_grid_angle

    integer(c_int) function rp_locate_lonlat(ctx, n, lon, lat, z, dob, t_b, ipos_out, jpos_out) &
        bind(C, name="rp_locate_lonlat")
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: n
      real(c_double), intent(in) :: lon(*), lat(*), z(*), dob(*)
      integer(c_int32_t), value :: t_b
      type(c_ptr), value :: ipos_out, jpos_out
    end function rp_locate_lonlat

    integer(c_int) function rp_nest_maps(ngrid, xi_rho, eta_rho, lon_rho, lat_rho, refine, scl, off) &
        bind(C, name="rp_nest_maps")
      import :: c_int, c_int32_t, c_ptr, c_double
      integer(c_int32_t), value :: ngrid
      integer(c_int32_t), intent(in) :: xi_rho(*), eta_rho(*)
      type(c_ptr), intent(in) :: lon_rho(*), lat_rho(*)
      real(c_double), intent(in) :: refine(*)
      real(c_double), intent(out) :: scl(*), off(*)
    end function rp_nest_maps

    ! ---- the step (update_particles, ROMSPath.f90:608-1008)

    integer(c_int) function rp_step(ctx, ex, ix, ets, t_b, t_c, t_f) bind(C, name="rp_step")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: ex(3), ix(3)
      integer(c_int32_t), value :: ets, t_b, t_c, t_f
    end function rp_step

    integer(c_int) function rp_step_n(ctx, nsteps, ex, ix, ets, t_b, t_c, t_f) bind(C, name="rp_step_n")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nsteps
      real(c_double), intent(in) :: ex(*), ix(*)
      integer(c_int32_t), intent(in) :: ets(*), t_b(*), t_c(*), t_f(*)
    end function rp_step_n

    integer(c_int) function rp_get_particles(ctx, n, x, y, z, age, status, gid, isin, wd, zeta, bath, flags) &
        bind(C, name="rp_get_particles")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: n
      type(c_ptr), value :: x, y, z, age, status, gid, isin, wd, zeta, bath, flags
    end function rp_get_particles

    ! ---- behave, diagnostics, output records (ROMSPath.f90:800-804, 935-986, 1012-1072)

    integer(c_int) function rp_set_behavior(ctx, b) bind(C, name="rp_set_behavior")
      import :: c_int, c_ptr, rp_behavior
      type(c_ptr), value :: ctx
      type(rp_behavior), intent(in) :: b
    end function rp_set_behavior

    integer(c_int) function rp_get_behavior(ctx, n, acc, vort, behavew, ssf) bind(C, name="rp_get_behavior")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: n
      type(c_ptr), value :: acc, vort, behavew, ssf
    end function rp_get_behavior

    integer(c_int) function rp_get_diagnostics(ctx, n, salt, temp, mean_salt, mean_temp, hob, bustr, bvstr) &
        bind(C, name="rp_get_diagnostics")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: n
      type(c_ptr), value :: salt, temp, mean_salt, mean_temp, hob, bustr, bvstr
    end function rp_get_diagnostics

    integer(c_int) function rp_reset_diagnostics(ctx) bind(C, name="rp_reset_diagnostics")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function rp_reset_diagnostics

    integer(c_int) function rp_set_grid_lonlat(ctx, ng, lon_rho, lat_rho) bind(C, name="rp_set_grid_lonlat")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ng
      real(c_double), intent(in) :: lon_rho(*), lat_rho(*)
    end function rp_set_grid_lonlat

    integer(c_int) function rp_output_record(ctx, n, mi, lon, lat, zp, age, status, gid, salt, temp, hob, &
        bustr, bvstr) bind(C, name="rp_output_record")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: n
      integer(c_int32_t), value :: mi
      type(c_ptr), value :: lon, lat, zp, age, status, gid, salt, temp, hob, bustr, bvstr
    end function rp_output_record

    integer(c_int) function rp_output_record_async(ctx, n, mi, lon, lat, zp, age, status, gid, salt, temp, &
        hob, bustr, bvstr) bind(C, name="rp_output_record_async")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: n
      integer(c_int32_t), value :: mi
      type(c_ptr), value :: lon, lat, zp, age, status, gid, salt, temp, hob, bustr, bvstr
    end function rp_output_record_async

    integer(c_int) function rp_output_wait(ctx) bind(C, name="rp_output_wait")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function rp_output_wait

    ! ---- noise, ids, synchronisation, errors

    integer(c_int) function rp_set_id_base(ctx, base) bind(C, name="rp_set_id_base")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: base
    end function rp_set_id_base

    integer(c_int) function rp_set_step_index(ctx, step_index) bind(C, name="rp_set_step_index")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: step_index
    end function rp_set_step_index

    integer(c_int) function rp_set_noise_hook(ctx, noise, nsteps) bind(C, name="rp_set_noise_hook")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr), value :: noise
      integer(c_int64_t), value :: nsteps
    end function rp_set_noise_hook

    integer(c_int) function rp_synchronize(ctx) bind(C, name="rp_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function rp_synchronize

    integer(c_int) function rp_last_error(ctx, buf, len) bind(C, name="rp_last_error")
      import :: c_int, c_int32_t, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_int32_t), value :: len
    end function rp_last_error

    integer(c_int) function rp_destroy(ctx) bind(C, name="rp_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function rp_destroy

    ! ---- device-resident particles (no reference counterpart)

    integer(c_int) function rp_device_state_get(ctx, out) bind(C, name="rp_device_state_get")
      import :: c_int, c_ptr, rp_device_state
      type(c_ptr), value :: ctx
      type(rp_device_state), intent(out) :: out
    end function rp_device_state_get

    integer(c_int) function rp_step_noalloc(ctx, state, ex, ix, ets, t_b, t_c, t_f) &
        bind(C, name="rp_step_noalloc")
      import :: c_int, c_int32_t, c_ptr, c_double, rp_device_state
      type(c_ptr), value :: ctx
      type(rp_device_state), intent(in) :: state
      real(c_double), intent(in) :: ex(3), ix(3)
      integer(c_int32_t), value :: ets, t_b, t_c, t_f
    end function rp_step_noalloc

    ! ---- adjoint pair (no reference counterpart)

    integer(c_int) function rp_adj_frames(ctx, nframes) bind(C, name="rp_adj_frames")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nframes
    end function rp_adj_frames

    integer(c_int) function rp_adj_set_frame(ctx, ng, frame, zeta, u, v, w, aks, su, sv) &
        bind(C, name="rp_adj_set_frame")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ng, frame
      real(c_double), intent(in) :: zeta(*), u(*), v(*), w(*), aks(*)
      type(c_ptr), value :: su, sv
    end function rp_adj_set_frame

    integer(c_int) function rp_forward(ctx, nsteps, steps, kappa, checkpoint_every) bind(C, name="rp_forward")
      import :: c_int, c_int32_t, c_ptr, c_double, rp_adj_step
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nsteps
      type(rp_adj_step), intent(in) :: steps(*)
      real(c_double), value :: kappa
      integer(c_int32_t), value :: checkpoint_every
    end function rp_forward

    integer(c_int) function rp_backward(ctx, dl_dx, dl_dy, dl_dz, dl_dx0, dl_dy0, dl_dz0, dl_dkappa) &
        bind(C, name="rp_backward")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: dl_dx(*), dl_dy(*), dl_dz(*)
      real(c_double), intent(out) :: dl_dx0(*), dl_dy0(*), dl_dz0(*)
      real(c_double), intent(out) :: dl_dkappa
    end function rp_backward

    integer(c_int) function rp_tangent(ctx, kappa, jac) bind(C, name="rp_tangent")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: kappa
      real(c_double), intent(out) :: jac(*)
    end function rp_tangent

    integer(c_int) function rp_adj_replay(ctx, x0, y0, z0, kappa, xf, yf, zf) bind(C, name="rp_adj_replay")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      type(c_ptr), value :: x0, y0, z0
      real(c_double), value :: kappa
      real(c_double), intent(out) :: xf(*), yf(*), zf(*)
    end function rp_adj_replay

    ! ---- launch settings, timing, counters (no reference counterpart)

    integer(c_int) function rp_set_launch(ctx, resort, blocks_per_sm) bind(C, name="rp_set_launch")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: resort, blocks_per_sm
    end function rp_set_launch

    integer(c_int) function rp_set_kernel_form(ctx, form) bind(C, name="rp_set_kernel_form")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: form
    end function rp_set_kernel_form

    integer(c_int) function rp_last_step_stats(ctx, ms, kernels) bind(C, name="rp_last_step_stats")
      import :: c_int, c_int32_t, c_ptr, c_float
      type(c_ptr), value :: ctx
      real(c_float), intent(out) :: ms
      integer(c_int32_t), intent(out) :: kernels
    end function rp_last_step_stats

    integer(c_int) function rp_count_spline_passes(ctx, on) bind(C, name="rp_count_spline_passes")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: on
    end function rp_count_spline_passes

    integer(c_int) function rp_spline_pass_counts(ctx, fits, passes) bind(C, name="rp_spline_pass_counts")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int64_t), intent(out) :: fits, passes
    end function rp_spline_pass_counts

    integer(c_int) function rp_kernel_launches(ctx, count) bind(C, name="rp_kernel_launches")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int64_t), intent(out) :: count
    end function rp_kernel_launches

    type(c_ptr) function rp_version() bind(C, name="rp_version")
      import :: c_ptr
    end function rp_version

  end interface
end module rp_gpu_mod
