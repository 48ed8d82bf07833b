!> ISO_C_BINDING interface to libnuvort_gpu.so (include/nuvort_gpu.h) for the NuVort Fortran
!> host.  type(qvort) (src/cdata.f90:19-29) is not interoperable, so the wrappers below pack
!> f(:) into plain arrays for nv_upload and unpack them after nv_download; every status other
!> than NV_OK ends the run through the host's fatal_error, as the replaced routines do.
!>
!> Not compiled in this repository's environment (there is no Fortran compiler here); the
!> same C ABI is exercised by the Python binding and the tests.
module nuvort_gpu
  use iso_c_binding
  implicit none

  integer(c_int32_t), parameter :: NV_OK = 0
  integer(c_int32_t), parameter :: NV_VEL_LIA = 0, NV_VEL_BS = 1, NV_VEL_TREE = 2
  integer(c_int32_t), parameter :: NV_BC_PERIODIC = 0, NV_BC_OPEN = 1, NV_BC_SOLID = 2
  integer(c_int32_t), parameter :: NV_NF_ZERO = 0, NV_NF_XFLOW = 1, NV_NF_UNIFORM = 2
  integer(c_int32_t), parameter :: NV_NF_SHEAR_XFLOW = 3, NV_NF_CHANNEL = 4, NV_NF_YCHANNEL = 5
  integer(c_int32_t), parameter :: NV_NF_NOISEY_XFLOW = 6, NV_NF_LAIZET_DNS = 7, NV_NF_TURB_DNS = 8
  integer(c_int32_t), parameter :: NV_PREC_FP64 = 0, NV_PREC_MIXED = 1

  type, bind(c) :: nv_params
    integer(c_int32_t) :: nsteps, shots, recon_shots, velocity
    integer(c_int32_t) :: boundary(3)
    integer(c_int32_t) :: normal_velocity, tree_extra_correction, nan_test
    integer(c_int32_t) :: overide_timestep_check, precision
    real(c_double) :: dt, delta, quant_circ, corea
    real(c_double) :: box_size(3)
    real(c_double) :: tree_theta, norm_vel_xflow
    real(c_double) :: norm_vel_vec(3), alpha(2), super_velocity(3)
    real(c_double) :: normal_fluid_cutoff, t_zero_normal_fluid
    real(c_double) :: norm_shear_omega
  end type

  integer(c_int32_t), parameter :: NV_EV_INSERT = 1, NV_EV_RECON = 2, NV_EV_REMOVE = 3
  integer(c_int32_t), parameter :: NV_EV_LOOPKILL = 4, NV_EV_WALL = 5, NV_EV_CLEAR = 6

  type, bind(c) :: nv_host_state
    integer(c_int32_t) :: pcount
    type(c_ptr) :: x, u, u1, u2, ghosti, ghostb
    type(c_ptr) :: infront, behind, closest, closestd
    type(c_ptr) :: wpinned, pinnedi, pinnedb  ! solid walls: wpinned(3,pcount), logicals as 0/1
  end type

  type, bind(c) :: nv_counters
    integer(c_int32_t) :: pcount, live, recon_count, remove_count, insert_count, loop_kills
    integer(c_int64_t) :: tree_eval, tree_tests
    integer(c_int32_t) :: itime, n_events
    real(c_double) :: t
    integer(c_int64_t) :: event_hash  ! unsigned on the C side; compare bit patterns only
    integer(c_int32_t) :: wall_recon_count, reserved
  end type

  !> one data/ts.log row (print_info) and the values behind it
  type, bind(c) :: nv_ts_row
    integer(c_int32_t) :: itime, live, recon_count, wall_recon_count, remove_count, reserved
    integer(c_int64_t) :: tree_eval
    real(c_double) :: t, delta, avg_sep, total_length, maxu, maxdu, mean_u_sup, mean_u_mf
    real(c_double) :: kappa_bar, kappa_min, kappa_max
  end type

  interface
    integer(c_int) function nv_params_default(p) bind(c, name='nv_params_default')
      import :: c_int, nv_params
      type(nv_params), intent(out) :: p
    end function
    integer(c_int) function nv_read_run_file(path, p) bind(c, name='nv_read_run_file')
      import :: c_int, c_char, nv_params
      character(kind=c_char), dimension(*), intent(in) :: path
      type(nv_params), intent(inout) :: p
    end function
    integer(c_int) function nv_create(params, nsys, capacity, device, h) bind(c, name='nv_create')
      import :: c_int, c_int32_t, c_ptr, nv_params
      type(nv_params), dimension(*), intent(in) :: params
      integer(c_int32_t), value :: nsys, device
      integer(c_int32_t), dimension(*), intent(in) :: capacity
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function nv_destroy(h) bind(c, name='nv_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_upload(h, sys, st) bind(c, name='nv_upload')
      import :: c_int, c_int32_t, c_ptr, nv_host_state
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys
      type(nv_host_state), intent(in) :: st
    end function
    integer(c_int) function nv_download(h, sys, st, cap) bind(c, name='nv_download')
      import :: c_int, c_int32_t, c_ptr, nv_host_state
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys, cap
      type(nv_host_state), intent(inout) :: st
    end function
    integer(c_int) function nv_set_clock(h, sys, t, itime) bind(c, name='nv_set_clock')
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys, itime
      real(c_double), value :: t
    end function
    integer(c_int) function nv_counters_get(h, sys, c) bind(c, name='nv_counters_get')
      import :: c_int, c_int32_t, c_ptr, nv_counters
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys
      type(nv_counters), intent(out) :: c
    end function
    integer(c_int) function nv_step(h, nsteps) bind(c, name='nv_step')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: nsteps
    end function
    ! one call per procedure of src/run.f90:26-64
    integer(c_int) function nv_ghostp(h) bind(c, name='nv_ghostp')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_construct_tree(h) bind(c, name='nv_construct_tree')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_pmotion(h) bind(c, name='nv_pmotion')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_pinsert(h) bind(c, name='nv_pinsert')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_pclose(h) bind(c, name='nv_pclose')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_precon(h) bind(c, name='nv_precon')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_wall_recon(h) bind(c, name='nv_wall_recon')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_premove(h) bind(c, name='nv_premove')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_enforce_boundary(h) bind(c, name='nv_enforce_boundary')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_empty_tree(h) bind(c, name='nv_empty_tree')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_end_step(h) bind(c, name='nv_end_step')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_calculate_diagnostics(h) bind(c, name='nv_calculate_diagnostics')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_ts_row_get(h, sys, row) bind(c, name='nv_ts_row_get')
      import :: c_int, c_int32_t, c_ptr, nv_ts_row
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys
      type(nv_ts_row), intent(out) :: row
    end function
    integer(c_int) function nv_format_ts_row(row, shots, buf, cap) bind(c, name='nv_format_ts_row')
      import :: c_int, c_int32_t, c_char, nv_ts_row
      type(nv_ts_row), intent(in) :: row
      integer(c_int32_t), value :: shots, cap
      character(kind=c_char), dimension(*), intent(out) :: buf
    end function
    integer(c_int) function nv_write_snapshot(h, sys, path) bind(c, name='nv_write_snapshot')
      import :: c_int, c_int32_t, c_ptr, c_char
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function nv_write_dump(h, sys, path) bind(c, name='nv_write_dump')
      import :: c_int, c_int32_t, c_ptr, c_char
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function nv_restore_dump(h, sys, path) bind(c, name='nv_restore_dump')
      import :: c_int, c_int32_t, c_ptr, c_char
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function nv_set_normal_fluid_noise(h, sys, noise, n) bind(c, name='nv_set_normal_fluid_noise')
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys, n
      real(c_double), dimension(*), intent(in) :: noise
    end function
    integer(c_int) function nv_set_normal_fluid_grid(h, sys, u, nx, ny, nz, yp) &
        bind(c, name='nv_set_normal_fluid_grid')
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys, nx, ny, nz
      real(c_double), dimension(*), intent(in) :: u, yp
    end function
    !> event margins of the topology tests (smallest relative distance from each threshold)
    integer(c_int) function nv_set_event_margins(h, on) bind(c, name='nv_set_event_margins')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: on
    end function
    integer(c_int) function nv_event_margins_get(h, sys, out) bind(c, name='nv_event_margins_get')
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys
      real(c_double), intent(out) :: out(4)
    end function
    !> every listed system at once (st(i) describes system sys(i), 0-based)
    integer(c_int) function nv_upload_many(h, count, sys, st) bind(c, name='nv_upload_many')
      import :: c_int, c_int32_t, c_ptr, nv_host_state
      type(c_ptr), value :: h
      integer(c_int32_t), value :: count
      integer(c_int32_t), intent(in) :: sys(*)
      type(nv_host_state), intent(in) :: st(*)
    end function
    integer(c_int) function nv_download_many(h, count, sys, st, cap) bind(c, name='nv_download_many')
      import :: c_int, c_int32_t, c_ptr, nv_host_state
      type(c_ptr), value :: h
      integer(c_int32_t), value :: count
      integer(c_int32_t), intent(in) :: sys(*), cap(*)
      type(nv_host_state), intent(inout) :: st(*)
    end function
    !> every system at once, host arrays packed system after system (pcounts(nsys))
    integer(c_int) function nv_upload_packed(h, all, pcounts) bind(c, name='nv_upload_packed')
      import :: c_int, c_int32_t, c_ptr, nv_host_state
      type(c_ptr), value :: h
      type(nv_host_state), intent(in) :: all
      integer(c_int32_t), intent(in) :: pcounts(*)
    end function
    integer(c_int) function nv_download_packed(h, all, cap_rows, pcounts) bind(c, name='nv_download_packed')
      import :: c_int, c_int32_t, c_int64_t, c_ptr, nv_host_state
      type(c_ptr), value :: h
      type(nv_host_state), intent(inout) :: all
      integer(c_int64_t), value :: cap_rows
      integer(c_int32_t), intent(out) :: pcounts(*)
    end function
    !> page-lock (cudaHostRegister) a host range, e.g. f(:)'s packed arrays
    integer(c_int) function nv_host_register(p, bytes) bind(c, name='nv_host_register')
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: p
      integer(c_size_t), value :: bytes
    end function
    integer(c_int) function nv_host_unregister(p) bind(c, name='nv_host_unregister')
      import :: c_int, c_ptr
      type(c_ptr), value :: p
    end function
    !> one tangle over several GPUs: the step's two halves, the walk range of this rank and the
    !> exchange of velocities by walk position (device buffers, e.g. for an MPI/NCCL all-gather)
    integer(c_int) function nv_step_velocity(h) bind(c, name='nv_step_velocity')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_step_finish(h) bind(c, name='nv_step_finish')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function nv_set_walk_range(h, sys, lo, hi) bind(c, name='nv_set_walk_range')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sys, lo, hi
    end function
    integer(c_int) function nv_velocity_pack(h, sys, lo, count, d_buf) bind(c, name='nv_velocity_pack')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h, d_buf
      integer(c_int32_t), value :: sys, lo, count
    end function
    integer(c_int) function nv_velocity_unpack(h, sys, lo, count, d_buf) bind(c, name='nv_velocity_unpack')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h, d_buf
      integer(c_int32_t), value :: sys, lo, count
    end function
    type(c_ptr) function nv_last_error() bind(c, name='nv_last_error')
      import :: c_ptr
    end function
  end interface

  !> device handle of the run (one system)
  type(c_ptr), save :: nv_h = c_null_ptr

contains

  !> run.in values of the host (module cdata) -> nv_params
  subroutine nv_params_from_cdata(p)
    use cdata
    type(nv_params), intent(out) :: p
    integer :: k, rc
    rc = nv_params_default(p)
    p%nsteps = nsteps ; p%shots = shots ; p%recon_shots = recon_shots
    select case (velocity)
      case ('LIA') ; p%velocity = NV_VEL_LIA
      case ('BS') ; p%velocity = NV_VEL_BS
      case ('Tree') ; p%velocity = NV_VEL_TREE
    end select
    do k = 1, 3
      p%boundary(k) = NV_BC_PERIODIC
    end do
    if (boundary_x == 'open') p%boundary(1) = NV_BC_OPEN
    if (boundary_y == 'open') p%boundary(2) = NV_BC_OPEN
    if (boundary_z == 'open') p%boundary(3) = NV_BC_OPEN
    if (boundary_x == 'solid') p%boundary(1) = NV_BC_SOLID
    if (boundary_y == 'solid') p%boundary(2) = NV_BC_SOLID
    if (boundary_z == 'solid') p%boundary(3) = NV_BC_SOLID
    select case (trim(normal_velocity))
      case ('xflow') ; p%normal_velocity = NV_NF_XFLOW
      case ('shear_xflow') ; p%normal_velocity = NV_NF_SHEAR_XFLOW
      case ('channel') ; p%normal_velocity = NV_NF_CHANNEL
      case ('ychannel') ; p%normal_velocity = NV_NF_YCHANNEL
      case ('noisey_xflow') ; p%normal_velocity = NV_NF_NOISEY_XFLOW
      case ('laizetDNS') ; p%normal_velocity = NV_NF_LAIZET_DNS
      case ('turbDNS') ; p%normal_velocity = NV_NF_TURB_DNS
      case default ; p%normal_velocity = NV_NF_ZERO
    end select
    p%tree_extra_correction = merge(1, 0, tree_extra_correction)
    p%nan_test = merge(1, 0, NAN_test)
    p%overide_timestep_check = merge(1, 0, overide_timestep_check)
    p%dt = dt ; p%delta = delta ; p%quant_circ = quant_circ ; p%corea = corea
    p%box_size = box_size ; p%tree_theta = tree_theta ; p%norm_vel_xflow = norm_vel_xflow
    p%alpha = alpha ; p%super_velocity = super_velocity
    p%normal_fluid_cutoff = normal_fluid_cutoff ; p%t_zero_normal_fluid = t_zero_normal_fluid
    p%norm_shear_omega = norm_shear_omega
  end subroutine

  subroutine nv_check(rc, where)
    use cdata, only: fatal_error
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    character(len=256) :: text
    integer :: k
    if (rc == NV_OK) return
    call c_f_pointer(nv_last_error(), msg, [256])
    text = ' '
    do k = 1, 256
      if (msg(k) == c_null_char) exit
      text(k:k) = msg(k)
    end do
    call fatal_error(where, trim(text))
  end subroutine

  !> f(:), pcount, t, itime -> device (replaces the host copy of the state)
  subroutine nv_push_state(cap)
    use cdata
    integer, intent(in) :: cap
    type(nv_params) :: p(1)
    integer(c_int32_t) :: caps(1)
    real(c_double), allocatable, target :: x(:,:), u(:,:), u1(:,:), u2(:,:)
    integer(c_int32_t), allocatable, target :: inf(:), beh(:), wp(:,:), pi(:), pb(:)
    type(nv_host_state) :: st
    integer :: i
    if (.not. c_associated(nv_h)) then
      call nv_params_from_cdata(p(1))
      caps(1) = cap
      call nv_check(nv_create(p, 1_c_int32_t, caps, 0_c_int32_t, nv_h), 'nuvort_gpu:nv_create')
    end if
    allocate(x(3,pcount), u(3,pcount), u1(3,pcount), u2(3,pcount), inf(pcount), beh(pcount))
    allocate(wp(3,pcount), pi(pcount), pb(pcount))
    do i = 1, pcount
      x(:,i) = f(i)%x ; u(:,i) = f(i)%u ; u1(:,i) = f(i)%u1 ; u2(:,i) = f(i)%u2
      inf(i) = f(i)%infront ; beh(i) = f(i)%behind
      wp(:,i) = f(i)%wpinned
      pi(i) = merge(1, 0, f(i)%pinnedi) ; pb(i) = merge(1, 0, f(i)%pinnedb)
    end do
    st%pcount = pcount
    st%x = c_loc(x) ; st%u = c_loc(u) ; st%u1 = c_loc(u1) ; st%u2 = c_loc(u2)
    st%ghosti = c_null_ptr ; st%ghostb = c_null_ptr
    st%infront = c_loc(inf) ; st%behind = c_loc(beh)
    st%closest = c_null_ptr ; st%closestd = c_null_ptr
    if (n_mirror > 0) then
      st%wpinned = c_loc(wp) ; st%pinnedi = c_loc(pi) ; st%pinnedb = c_loc(pb)
    else
      st%wpinned = c_null_ptr ; st%pinnedi = c_null_ptr ; st%pinnedb = c_null_ptr
    end if
    call nv_check(nv_upload(nv_h, 0_c_int32_t, st), 'nuvort_gpu:nv_upload')
    call nv_check(nv_set_clock(nv_h, 0_c_int32_t, t, int(itime, c_int32_t)), 'nuvort_gpu:nv_set_clock')
  end subroutine

  !> device -> f(:), pcount (f is grown when pinsert appended slots on the device)
  subroutine nv_pull_state(cap)
    use cdata
    integer, intent(in) :: cap
    real(c_double), allocatable, target :: x(:,:), u(:,:), u1(:,:), u2(:,:)
    integer(c_int32_t), allocatable, target :: inf(:), beh(:), wp(:,:), pi(:), pb(:)
    type(qvort), allocatable :: tmp(:)
    type(nv_host_state) :: st
    type(nv_counters) :: c
    integer :: i
    allocate(x(3,cap), u(3,cap), u1(3,cap), u2(3,cap), inf(cap), beh(cap))
    allocate(wp(3,cap), pi(cap), pb(cap))
    st%x = c_loc(x) ; st%u = c_loc(u) ; st%u1 = c_loc(u1) ; st%u2 = c_loc(u2)
    st%ghosti = c_null_ptr ; st%ghostb = c_null_ptr
    st%infront = c_loc(inf) ; st%behind = c_loc(beh)
    st%closest = c_null_ptr ; st%closestd = c_null_ptr
    st%wpinned = c_loc(wp) ; st%pinnedi = c_loc(pi) ; st%pinnedb = c_loc(pb)
    call nv_check(nv_download(nv_h, 0_c_int32_t, st, int(cap, c_int32_t)), 'nuvort_gpu:nv_download')
    if (st%pcount > size(f)) then
      allocate(tmp(st%pcount)) ; tmp(:)%infront = 0
      tmp(1:size(f)) = f
      call move_alloc(from=tmp, to=f)
    end if
    pcount = st%pcount
    do i = 1, pcount
      f(i)%x = x(:,i) ; f(i)%u = u(:,i) ; f(i)%u1 = u1(:,i) ; f(i)%u2 = u2(:,i)
      f(i)%infront = inf(i) ; f(i)%behind = beh(i)
      f(i)%wpinned = wp(:,i) ; f(i)%pinnedi = pi(i) /= 0 ; f(i)%pinnedb = pb(i) /= 0
    end do
    call nv_check(nv_counters_get(nv_h, 0_c_int32_t, c), 'nuvort_gpu:nv_counters_get')
    recon_count = c%recon_count ; remove_count = c%remove_count ; t = c%t
    wall_recon_count = c%wall_recon_count
  end subroutine

end module
