! Fortran 2018 interface to libhydft_gpu.so (include/hydft_gpu.h).
!
! With this module HyDFT's driver and tests can run the solver step on a
! B200: `model_gpu_t` holds the C handle and offers the calls of model_t
! (src/model/model.f90:29-49) -- init, advance, rhs, compute_dt -- plus
! state transfer.  Every C call returns a status; on failure the wrapper
! calls the reference's `fatal` with hydft_gpu_last_error(), so the
! observable behaviour (message + error stop 1) is the reference's.
!
! Build: gfortran -c hydft_gpu_mod.f90 (after the reference's modules for
! hydft_kinds and hydft_params), link with -L<lib> -lhydft_gpu -lstdc++.
module hydft_gpu_mod
  use, intrinsic :: iso_c_binding
  use hydft_kinds, only: rp, fatal
  use hydft_params, only: params_t
  implicit none
  private
  public :: model_gpu_t, hydft_params_c, to_c_params

  ! hydft_params (C struct, include/hydft_gpu.h); field order and sizes match
  type, bind(C) :: hydft_params_c
    integer(c_int) :: nx, ny, nz
    real(c_double) :: lx, ly, lz
    integer(c_int) :: dealias
    character(kind=c_char) :: kind(16)
    real(c_double) :: gamma, kappa, rs, theta, mass
    character(kind=c_char) :: terms(64)
    real(c_double) :: tfk_gamma
    character(kind=c_char) :: closure(16)
    character(kind=c_char) :: transport(16)
    real(c_double) :: eta, xi, tau
    character(kind=c_char) :: tau_model(16)
    real(c_double) :: adiabatic_index
    character(kind=c_char) :: structure(16)
    character(kind=c_char) :: structure_file(256)
    character(kind=c_char) :: structure_kind(4)
    integer(c_int) :: hnc_nr, hnc_maxiter
    real(c_double) :: hnc_rmax, hnc_tol, hnc_mix
    real(c_double) :: dt, cfl, tend
    integer(c_int) :: nsteps_max, iout, iprobe, idiag
    character(kind=c_char) :: ic(16)
    real(c_double) :: ic_amplitude
    integer(c_int) :: ic_mode(3)
    real(c_double) :: ic_width
    integer(c_int) :: ic_seed
    character(kind=c_char) :: vext(16)
    real(c_double) :: vext_amplitude
    integer(c_int) :: vext_mode(3)
    real(c_double) :: vext_omega, vext_width, vext_ramp
    integer(c_int) :: probe_mode(3)
    character(kind=c_char) :: prefix(256)
    character(kind=c_char) :: gpu_precision(8)
  end type hydft_params_c

  interface
    integer(c_int) function hydft_params_default(p) bind(C, name='hydft_params_default')
      import :: hydft_params_c, c_int
      type(hydft_params_c), intent(inout) :: p
    end function
    integer(c_int) function hydft_params_finalize(p) bind(C, name='hydft_params_finalize')
      import :: hydft_params_c, c_int
      type(hydft_params_c), intent(inout) :: p
    end function
    integer(c_int) function hydft_gpu_create(p, st, device, h) bind(C, name='hydft_gpu_create')
      import :: hydft_params_c, c_int, c_ptr
      type(hydft_params_c), intent(in) :: p
      type(c_ptr), value :: st
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: h
    end function
    subroutine hydft_gpu_destroy(h) bind(C, name='hydft_gpu_destroy')
      import :: c_ptr
      type(c_ptr), value :: h
    end subroutine
    type(c_ptr) function hydft_gpu_last_error(h) bind(C, name='hydft_gpu_last_error')
      import :: c_ptr
      type(c_ptr), value :: h
    end function
    type(c_ptr) function hydft_gpu_create_error() bind(C, name='hydft_gpu_create_error')
      import :: c_ptr
    end function
    integer(c_int) function hydft_gpu_set_state(h, n, mom, pi) bind(C, name='hydft_gpu_set_state')
      import :: c_ptr, c_int
      type(c_ptr), value :: h, n, mom, pi
    end function
    integer(c_int) function hydft_gpu_get_state(h, n, mom, pi) bind(C, name='hydft_gpu_get_state')
      import :: c_ptr, c_int
      type(c_ptr), value :: h, n, mom, pi
    end function
    integer(c_int) function hydft_gpu_advance(h, nsteps) bind(C, name='hydft_gpu_advance')
      import :: c_ptr, c_int
      type(c_ptr), value :: h
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function hydft_gpu_rhs(h, t, dn, dmom, dpi) bind(C, name='hydft_gpu_rhs')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h
      real(c_double), value :: t
      type(c_ptr), value :: dn, dmom, dpi
    end function
    integer(c_int) function hydft_gpu_compute_dt(h, dt) bind(C, name='hydft_gpu_compute_dt')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: dt
    end function
    integer(c_int) function hydft_gpu_get_scalar(h, name, v) bind(C, name='hydft_gpu_get_scalar')
      import :: c_ptr, c_int, c_double, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: name(*)
      real(c_double), intent(out) :: v
    end function
    integer(c_int) function hydft_gpu_get_time(h, t, dt, step) bind(C, name='hydft_gpu_get_time')
      import :: c_ptr, c_int, c_double, c_int64_t
      type(c_ptr), value :: h
      real(c_double), intent(out) :: t, dt
      integer(c_int64_t), intent(out) :: step
    end function
    integer(c_int) function hydft_gpu_budgets(h, mass, mom, ekin, fe, nmin, nmax) bind(C, name='hydft_gpu_budgets')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: mass, mom(3), ekin, fe, nmin, nmax
    end function
    integer(c_int) function hydft_gpu_mode(h, field, mx, my, mz, re, im) bind(C, name='hydft_gpu_mode')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: field, mx, my, mz
      real(c_double), intent(out) :: re, im
    end function
    integer(c_int) function hydft_gpu_write_fields(h, prefix) bind(C, name='hydft_gpu_write_fields')
      import :: c_ptr, c_int, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: prefix(*)
    end function
    integer(c_int) function hydft_gpu_read_fields(h, path) bind(C, name='hydft_gpu_read_fields')
      import :: c_ptr, c_int, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: path(*)
    end function
    integer(c_int) function hydft_gpu_run(h) bind(C, name='hydft_gpu_run')
      import :: c_ptr, c_int
      type(c_ptr), value :: h
    end function
  end interface

  !> model_t on the GPU: the state lives on the device and is copied to the
  !> host arrays n, mom, pi by sync_to_host (the reference's tests read
  !> m%sp%n etc. directly; call sync_to_host first).
  type :: model_gpu_t
    type(c_ptr) :: h = c_null_ptr
    integer :: nx = 0, ny = 0, nz = 0
    logical :: has_pi = .false.
    real(rp) :: t = 0.0_rp, dt = 0.0_rp
    integer :: step = 0
    real(rp), allocatable :: n(:,:,:), mom(:,:,:,:), pi(:,:,:,:)
  contains
    procedure :: init => gpu_init
    procedure :: advance => gpu_advance
    procedure :: rhs => gpu_rhs
    procedure :: compute_dt => gpu_compute_dt
    procedure :: sync_to_host => gpu_sync_to_host
    procedure :: sync_to_device => gpu_sync_to_device
    procedure :: budgets => gpu_budgets
    procedure :: write_fields => gpu_write_fields
    procedure :: read_fields => gpu_read_fields
    procedure :: run => gpu_run
    procedure :: destroy => gpu_destroy
  end type model_gpu_t

contains

  subroutine put(dst, s)
    character(kind=c_char), intent(out) :: dst(:)
    character(len=*), intent(in) :: s
    integer :: i
    dst = c_null_char
    do i = 1, min(len_trim(s), size(dst) - 1)
      dst(i) = s(i:i)
    end do
  end subroutine put

  !> params_t -> hydft_params (same names and meanings)
  function to_c_params(p, precision) result(c)
    type(params_t), intent(in) :: p
    character(len=*), intent(in), optional :: precision
    type(hydft_params_c) :: c
    integer(c_int) :: rc
    rc = hydft_params_default(c)
    c%nx = p%nx; c%ny = p%ny; c%nz = p%nz
    c%lx = p%lx; c%ly = p%ly; c%lz = p%lz
    c%dealias = merge(1, 0, p%dealias)
    call put(c%kind, p%kind)
    c%gamma = p%gamma; c%kappa = p%kappa; c%rs = p%rs; c%theta = p%theta; c%mass = p%mass
    call put(c%terms, p%terms)
    c%tfk_gamma = p%tfk_gamma
    call put(c%closure, p%closure)
    call put(c%transport, p%transport)
    c%eta = p%eta; c%xi = p%xi; c%tau = p%tau
    call put(c%tau_model, p%tau_model)
    c%adiabatic_index = p%adiabatic_index
    call put(c%structure, p%structure)
    call put(c%structure_file, p%structure_file)
    call put(c%structure_kind, p%structure_kind)
    c%hnc_nr = p%hnc_nr; c%hnc_maxiter = p%hnc_maxiter
    c%hnc_rmax = p%hnc_rmax; c%hnc_tol = p%hnc_tol; c%hnc_mix = p%hnc_mix
    c%dt = p%dt; c%cfl = p%cfl; c%tend = p%tend
    call put(c%vext, p%vext)
    c%vext_amplitude = p%vext_amplitude; c%vext_mode = p%vext_mode
    c%vext_omega = p%vext_omega; c%vext_width = p%vext_width; c%vext_ramp = p%vext_ramp
    c%nsteps_max = p%nsteps_max; c%iout = p%iout; c%iprobe = p%iprobe; c%idiag = p%idiag
    c%probe_mode = p%probe_mode
    call put(c%prefix, p%prefix)
    if (present(precision)) call put(c%gpu_precision, precision)
    rc = hydft_params_finalize(c)
  end function to_c_params

  subroutine check(m, rc)
    class(model_gpu_t), intent(in) :: m
    integer(c_int), intent(in) :: rc
    character(len=512) :: msg
    if (rc == 0) return
    call c_string(hydft_gpu_last_error(m%h), msg)
    call fatal(trim(msg))
  end subroutine check

  subroutine c_string(p, s)
    type(c_ptr), intent(in) :: p
    character(len=*), intent(out) :: s
    character(kind=c_char), pointer :: a(:)
    integer :: i
    s = ''
    if (.not. c_associated(p)) return
    call c_f_pointer(p, a, [len(s)])
    do i = 1, len(s)
      if (a(i) == c_null_char) exit
      s(i:i) = a(i)
    end do
  end subroutine c_string

  !> model_t%init (model.f90:56-74) on device `device`
  subroutine gpu_init(m, p, precision, device)
    class(model_gpu_t), intent(inout) :: m
    type(params_t), intent(in) :: p
    character(len=*), intent(in), optional :: precision
    integer, intent(in), optional :: device
    type(hydft_params_c), target :: c
    integer(c_int) :: rc, dev
    real(c_double) :: ev
    character(len=512) :: msg
    c = to_c_params(p, precision)
    dev = 0
    if (present(device)) dev = device
    rc = hydft_gpu_create(c, c_null_ptr, dev, m%h)
    if (rc /= 0) then
      call c_string(hydft_gpu_create_error(), msg)
      call fatal(trim(msg))
    end if
    m%nx = p%nx; m%ny = p%ny; m%nz = p%nz
    ! Pi is a state variable only for the Maxwell closure with tau > 0 (stress.f90:47-49)
    call check(m, hydft_gpu_get_scalar(m%h, 'evolve'//c_null_char, ev))
    m%has_pi = ev > 0.5_c_double
    allocate(m%n(m%nx, m%ny, m%nz), m%mom(m%nx, m%ny, m%nz, 3))
    if (m%has_pi) allocate(m%pi(m%nx, m%ny, m%nz, 6))
    call m%sync_to_host()
  end subroutine gpu_init

  subroutine gpu_sync_to_host(m)
    class(model_gpu_t), intent(inout), target :: m
    integer(c_int64_t) :: st
    type(c_ptr) :: ppi
    ppi = c_null_ptr
    if (allocated(m%pi)) ppi = c_loc(m%pi)
    call check(m, hydft_gpu_get_state(m%h, c_loc(m%n), c_loc(m%mom), ppi))
    call check(m, hydft_gpu_get_time(m%h, m%t, m%dt, st))
    m%step = int(st)
  end subroutine gpu_sync_to_host

  subroutine gpu_sync_to_device(m)
    class(model_gpu_t), intent(inout), target :: m
    type(c_ptr) :: ppi
    ppi = c_null_ptr
    if (allocated(m%pi)) ppi = c_loc(m%pi)
    call check(m, hydft_gpu_set_state(m%h, c_loc(m%n), c_loc(m%mom), ppi))
  end subroutine gpu_sync_to_device

  !> model_t%advance (model.f90:186-227), nsteps times
  subroutine gpu_advance(m, nsteps)
    class(model_gpu_t), intent(inout) :: m
    integer, intent(in), optional :: nsteps
    integer(c_int) :: k
    integer(c_int64_t) :: st
    k = 1
    if (present(nsteps)) k = nsteps
    call check(m, hydft_gpu_advance(m%h, k))
    call check(m, hydft_gpu_get_time(m%h, m%t, m%dt, st))
    m%step = int(st)
  end subroutine gpu_advance

  !> model_t%rhs (model.f90:85-146)
  subroutine gpu_rhs(m, t, dn, dmom, dpi)
    class(model_gpu_t), intent(inout) :: m
    real(rp), intent(in) :: t
    real(rp), intent(out), target :: dn(:,:,:), dmom(:,:,:,:), dpi(:,:,:,:)
    call check(m, hydft_gpu_rhs(m%h, t, c_loc(dn), c_loc(dmom), c_loc(dpi)))
  end subroutine gpu_rhs

  !> model_t%compute_dt (model.f90:150-183)
  subroutine gpu_compute_dt(m)
    class(model_gpu_t), intent(inout) :: m
    real(c_double) :: dt
    call check(m, hydft_gpu_compute_dt(m%h, dt))
    m%dt = dt
  end subroutine gpu_compute_dt

  !> diag_t%budgets (diagnostics.f90:41-60) of the device state
  subroutine gpu_budgets(m, mass, mom, ekin, fe)
    class(model_gpu_t), intent(inout) :: m
    real(rp), intent(out) :: mass, mom(3), ekin, fe
    real(c_double) :: nmin, nmax
    call check(m, hydft_gpu_budgets(m%h, mass, mom, ekin, fe, nmin, nmax))
  end subroutine gpu_budgets

  !> write_fields (io.f90:19-35)
  subroutine gpu_write_fields(m, prefix)
    class(model_gpu_t), intent(inout) :: m
    character(len=*), intent(in) :: prefix
    call check(m, hydft_gpu_write_fields(m%h, trim(prefix)//c_null_char))
  end subroutine gpu_write_fields

  !> resume from a field file written by write_fields
  subroutine gpu_read_fields(m, path)
    class(model_gpu_t), intent(inout) :: m
    character(len=*), intent(in) :: path
    integer(c_int64_t) :: st
    call check(m, hydft_gpu_read_fields(m%h, trim(path)//c_null_char))
    call check(m, hydft_gpu_get_time(m%h, m%t, m%dt, st))
    m%step = int(st)
  end subroutine gpu_read_fields

  !> hydft_run's loop (hydft.f90:30-60) on the device, with its output files
  subroutine gpu_run(m)
    class(model_gpu_t), intent(inout) :: m
    integer(c_int64_t) :: st
    call check(m, hydft_gpu_run(m%h))
    call check(m, hydft_gpu_get_time(m%h, m%t, m%dt, st))
    m%step = int(st)
  end subroutine gpu_run

  subroutine gpu_destroy(m)
    class(model_gpu_t), intent(inout) :: m
    if (c_associated(m%h)) call hydft_gpu_destroy(m%h)
    m%h = c_null_ptr
  end subroutine gpu_destroy

end module hydft_gpu_mod
