!=====================================================================
!  em2g_shim.f90 -- em2's move / curnt / fields subroutines on the GPU.
!
!  em2 (fanyumeng666/maccpic, pic/) calls, every step (pic/main.f90:154-169):
!      call move; call curnt; [call output]; it = it + 1; call fields
!  on the module `global` (pic/global.f90:31-45).  This file provides the
!  three subroutines with the same names and no arguments, so that em2
!  links it in place of move.o, curnt.o and fields.o (pic/Makefile:7) with
!  main.f90, output.f90, cont.f90 and the modules unchanged.  The state
!  lives on the GPU in one libem2g context (include/em2g.h); it is copied
!  into `global` only where em2 reads it on the host: before `output`
!  (the predicate of pic/main.f90:158-159) and, for the energies, after
!  `fields` at isav steps.  One MPI rank only (nproc = 1): em2's
!  allreduces are then identities.
!
!  Build (where gfortran exists):
!      mpif90 -O3 -c em2g_shim.f90
!      mpif90 -o em2 input.o global.o main.o init.o output.o creator.o \
!             cont.o smear.o setrho.o setv.o smooth.o em2g_shim.o dran2.o \
!             -L<repo>/maccpic_b200 -lem2g -lcudart
!=====================================================================
module em2g_c
  use iso_c_binding
  implicit none
  ! struct em2g_params of include/em2g.h, member for member
  type, bind(c) :: em2g_params
    integer(c_int32_t) :: struct_size
    integer(c_int32_t) :: nx, ny, nsp, isav, precision
    real(c_double)     :: dx, dy, dt, c
    real(c_double)     :: qm(4), q(4), dn(4), am(4), tx(4), ty(4)
    integer(c_int64_t) :: np_max(4)
    integer(c_int32_t) :: cg_maxits, energy_mode
    real(c_double)     :: cg_eps, qme, wpe
    integer(c_int32_t) :: device, sort_interval, smooth_current, poisson, staging_mib
    integer(c_int32_t) :: reserved(13)
  end type em2g_params

  interface
    integer(c_int) function em2g_params_init(p) bind(c)
      import
      type(em2g_params) :: p
    end function
    integer(c_int) function em2g_create(p, ctx) bind(c)
      import
      type(em2g_params) :: p
      type(c_ptr) :: ctx
    end function
    integer(c_int) function em2g_destroy(ctx) bind(c)
      import
      type(c_ptr), value :: ctx
    end function
    type(c_ptr) function em2g_last_error() bind(c)
      import
    end function
    integer(c_int) function em2g_set_field(ctx, id, a) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: id
      real(c_double) :: a(*)
    end function
    integer(c_int) function em2g_get_field(ctx, id, a) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: id
      real(c_double) :: a(*)
    end function
    integer(c_int) function em2g_set_particles(ctx, isp, n, x, y, vx, vy, vz, g) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: isp
      integer(c_int64_t), value :: n
      real(c_double) :: x(*), y(*), vx(*), vy(*), vz(*), g(*)
    end function
    integer(c_int) function em2g_get_particles(ctx, isp, n, x, y, vx, vy, vz, g) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: isp
      integer(c_int64_t) :: n
      real(c_double) :: x(*), y(*), vx(*), vy(*), vz(*), g(*)
    end function
    integer(c_int) function em2g_set_step(ctx, it) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: it
    end function
    integer(c_int) function em2g_move_curnt(ctx, ake) bind(c)
      import
      type(c_ptr), value :: ctx
      real(c_double) :: ake(*)
    end function
    integer(c_int) function em2g_fields(ctx, it, e6, n) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: it
      real(c_double) :: e6(6)
      integer(c_int) :: n
    end function
    integer(c_int) function em2g_smooth2(ctx, id) bind(c)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: id
    end function
  end interface

  type(c_ptr), save :: ctx = c_null_ptr

contains

  ! a nonzero status ends the run with the library's message (em2 itself
  ! has no error returns: it prints and carries on, or stops)
  subroutine em2g_check(rc, what)
    integer(c_int), intent(in) :: rc
    character(*), intent(in) :: what
    character(kind=c_char), pointer :: msg(:)
    integer :: k
    if (rc == 0) return
    call c_f_pointer(em2g_last_error(), msg, [512])
    k = 0
    do while (k < 512)
      if (msg(k + 1) == c_null_char) exit
      k = k + 1
    end do
    write(*,*) 'em2g: ', what, ' failed: ', msg(1:k)
    error stop 1
  end subroutine em2g_check

end module em2g_c

! Creates the context from `global` and uploads fields and particles, on
! the first call of move, curnt or fields (after init or cont filled them).
subroutine em2g_ensure
  use global
  use em2g_c
  implicit none
  type(em2g_params) :: p
  real(8), dimension(nsp) :: dn_, q_, qm_
  real(8), dimension(0:nx2,0:ny2) :: f
  integer :: isp, k
  if (c_associated(ctx)) return
  call com_den(dn_, q_, qm_)                   ! pic/input.f90:61-69
  call em2g_check(em2g_params_init(p), 'em2g_params_init')
  p%nx = nx;  p%ny = ny;  p%nsp = nsp;  p%isav = isav
  p%dx = dx;  p%dy = dy;  p%dt = dt;  p%c = c
  p%qme = qme;  p%wpe = wpe
  p%qm(1:nsp) = qm_;  p%q(1:nsp) = q_;  p%dn(1:nsp) = dn_
  p%am(1:nsp) = am;  p%tx(1:nsp) = tx;  p%ty(1:nsp) = ty   ! pic/init.f90:116-125
  p%np_max(1:nsp) = np
  call em2g_check(em2g_create(p, ctx), 'em2g_create')
  call em2g_check(em2g_set_step(ctx, it), 'em2g_set_step')
  do k = 0, 12                                 ! enum em2g_field order
    select case (k)
    case (0);  f = ex
    case (1);  f = ey
    case (2);  f = ez
    case (3);  f = bx
    case (4);  f = by
    case (5);  f = bz
    case (6);  f = rho
    case (7);  f = jxm
    case (8);  f = jxp
    case (9);  f = jym
    case (10); f = jyp
    case (11); f = jzm
    case (12); f = jzp
    end select
    call em2g_check(em2g_set_field(ctx, k, f), 'em2g_set_field')
  end do
  do isp = 1, nsp
    call em2g_check(em2g_set_particles(ctx, isp - 1, np(isp), x(:,isp), y(:,isp), &
                    vx(:,isp), vy(:,isp), vz(:,isp), gamma(:,isp)), 'em2g_set_particles')
  end do
end subroutine em2g_ensure

! Copies the GPU state into `global`: every field array and every particle.
subroutine em2g_download
  use global
  use em2g_c
  implicit none
  integer :: isp
  integer(c_int64_t) :: n
  call em2g_check(em2g_get_field(ctx, 0, ex), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 1, ey), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 2, ez), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 3, bx), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 4, by), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 5, bz), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 6, rho), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 7, jxm), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 8, jxp), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 9, jym), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 10, jyp), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 11, jzm), 'em2g_get_field')
  call em2g_check(em2g_get_field(ctx, 12, jzp), 'em2g_get_field')
  do isp = 1, nsp
    call em2g_check(em2g_get_particles(ctx, isp - 1, n, x(:,isp), y(:,isp), vx(:,isp), &
                    vy(:,isp), vz(:,isp), gamma(:,isp)), 'em2g_get_particles')
  end do
end subroutine em2g_download

! replaces pic/move.f90: the push runs fused with curnt's deposit (nothing
! reads the velocities between the two calls, pic/main.f90:154-155)
subroutine move
  implicit none
  call em2g_ensure
end subroutine move

! replaces pic/curnt.f90: gather, Boris push, move and deposit of every
! species in one fused kernel each; ake as after pic/move.f90:208-214
subroutine curnt
  use global
  use em2g_c
  implicit none
  call em2g_ensure
  call em2g_check(em2g_move_curnt(ctx, ake), 'em2g_move_curnt')
  ! output reads E, B, rho, J and the particles on the host
  if ((mod(it,isav) == 0) .or. (it == 1) .or. (mod(it,iphs) == 0) .or. (it == nt)) then
    call em2g_download
  end if
end subroutine curnt

! replaces pic/fields.f90: fold, Yee, filters, Poisson/cgm, energies
subroutine fields
  use global
  use em2g_c
  implicit none
  real(c_double) :: e6(6)
  integer(c_int) :: n
  call em2g_ensure
  call em2g_check(em2g_fields(ctx, it, e6, n), 'em2g_fields')
  if (mod(it,isav) == 0) then
    exe = e6(1);  eye = e6(2);  eze = e6(3)
    bxe = e6(4);  bye = e6(5);  bze = e6(6)
  end if
end subroutine fields
