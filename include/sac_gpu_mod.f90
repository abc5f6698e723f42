! sac_gpu_mod.f90 -- Fortran 2003 (ISO_C_BINDING) interface of libsacgpu.so,
! the mirror of include/sac_gpu.h for the reference's Fortran host (program vac,
! src/vac.t of drewleonard42/SAC).  The derived types are bind(C): their
! components follow sac_gpu.h's structs field by field, in the same order, so the
! companion C compiler lays them out identically (tests/test_fortran_binding.py
! checks every component offset against offsetof).  Every function returns a
! sac_status (0 = SAC_OK); the host maps a non-zero status to die().
module sacgpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: SAC_OK = 0, SAC_ERR_ARG = 1, SAC_ERR_STATE = 2, SAC_ERR_CUDA = 3, &
       SAC_ERR_NOMEM = 4, SAC_ERR_UNSUPPORTED = 5, SAC_ERR_NONFINITE = 6, SAC_ERR_TIMEOUT = 7, &
       SAC_ERR_NODEVICE = 8
  integer(c_int), parameter :: SAC_PREC_FP64 = 0, SAC_PREC_FP32 = 1
  integer(c_int), parameter :: SAC_USR_NONE = 0, SAC_USR_VISCOSITY = 1, SAC_USR_SLOG = 2, &
       SAC_USR_GRAVVISC = 3, SAC_USR_STRAT = 4, SAC_USR_TUBE = 5
  integer(c_int), parameter :: SAC_LENTYPE = 10, SAC_NHIB = 10, SAC_NWMAX = 13

  ! the context program vac's host shim (sac_b200/fortran/vacgpu.t) drives
  type(c_ptr), save :: vac_ctx = c_null_ptr

  type, bind(C) :: sac_params
     real(c_double) :: gamma
     real(c_double) :: eta
     real(c_double) :: grav(3)
     real(c_double) :: nu
     real(c_double) :: courantpar
     real(c_double) :: dtpar
     real(c_double) :: dtdiffpar
     integer(c_int) :: dtcantgrow
     character(kind=c_char) :: typeadvance(11)
     character(kind=c_char) :: typepred(11)
     integer(c_int) :: sourceunsplit
     integer(c_int) :: divbfix
     integer(c_int) :: user
     real(c_double) :: userpar(16)
     integer(c_int) :: alias_nu_grav3
     integer(c_int) :: precision
     integer(c_int) :: device
     integer(c_int) :: smallfix
     real(c_double) :: smallp
     real(c_double) :: smallrho
     real(c_double) :: vacuumrho
     integer(c_int) :: compactres
  end type sac_params

  type, bind(C) :: sac_diag_out
     real(c_double) :: wmean(13)
     real(c_double) :: divb_l2
     real(c_double) :: divb_linf
     real(c_double) :: maxviscoef
     real(c_double) :: ctot(3)
     integer(c_int) :: nonfinite
     integer(c_int) :: nerror_toosmallp
     integer(c_int) :: toosmallp_it
     real(c_double) :: toosmallp_min
  end type sac_diag_out

  interface
     subroutine sac_default_params(p) bind(C, name='sac_default_params')
       import :: sac_params
       type(sac_params) :: p
     end subroutine sac_default_params

     integer(c_int) function sac_create(p, ctx) bind(C, name='sac_create')
       import :: c_int, c_ptr, sac_params
       type(sac_params), intent(in) :: p
       type(c_ptr) :: ctx
     end function sac_create

     integer(c_int) function sac_set_grid(ctx, ndim, ndir, ixGhi, ixM, x, fullgridini) &
          bind(C, name='sac_set_grid')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: ndim, ndir
       integer(c_int), intent(in) :: ixGhi(3), ixM(6)
       real(c_double), intent(in) :: x(*)
       integer(c_int), value :: fullgridini
     end function sac_set_grid

     ! ixB(ndim,nB,2): ixBmin(:,1:nB) then ixBmax(:,1:nB), idimB(nB), upperB(nB) 0/1
     ! and ipairB(nB) (0: automatic).  After boundsetup these hold the default
     ! regions too; the library recognises them (C callers may pass NULL instead)
     integer(c_int) function sac_set_boundaries(ctx, nB, typeB, ixB, idimB, upperB, ipairB) &
          bind(C, name='sac_set_boundaries')
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: ctx
       integer(c_int), value :: nB
       character(kind=c_char), intent(in) :: typeB(*)
       integer(c_int), intent(in) :: ixB(*), idimB(*), upperB(*), ipairB(*)
     end function sac_set_boundaries

     integer(c_int) function sac_upload(ctx, w) bind(C, name='sac_upload')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: w(*)
     end function sac_upload

     integer(c_int) function sac_download(ctx, w) bind(C, name='sac_download')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double) :: w(*)
     end function sac_download

     integer(c_int) function sac_getboundary(ctx, t) bind(C, name='sac_getboundary')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), value :: t
     end function sac_getboundary

     integer(c_int) function sac_getdt(ctx, dt, it) bind(C, name='sac_getdt')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double) :: dt
       integer(c_int), value :: it
     end function sac_getdt

     integer(c_int) function sac_getdt_static(ctx, dt, it) bind(C, name='sac_getdt_static')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double) :: dt
       integer(c_int), value :: it
     end function sac_getdt_static

     integer(c_int) function sac_advect(ctx, method, iws, idimmin, idimmax, dt, t, it) &
          bind(C, name='sac_advect')
       import :: c_int, c_ptr, c_double, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char), intent(in) :: method(*)
       integer(c_int), intent(in) :: iws(*)
       integer(c_int), value :: idimmin, idimmax
       real(c_double), value :: dt, t
       integer(c_int), value :: it
     end function sac_advect

     integer(c_int) function sac_diag(ctx, d) bind(C, name='sac_diag')
       import :: c_int, c_ptr, sac_diag_out
       type(c_ptr), value :: ctx
       type(sac_diag_out) :: d
     end function sac_diag

     integer(c_int) function sac_synchronize(ctx) bind(C, name='sac_synchronize')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function sac_synchronize

     type(c_ptr) function sac_last_error(ctx) bind(C, name='sac_last_error')
       import :: c_ptr
       type(c_ptr), value :: ctx
     end function sac_last_error

     subroutine sac_destroy(ctx) bind(C, name='sac_destroy')
       import :: c_ptr
       type(c_ptr), value :: ctx
     end subroutine sac_destroy

     integer(c_size_t) function c_strlen(s) bind(C, name='strlen')
       import :: c_size_t, c_ptr
       type(c_ptr), value :: s
     end function c_strlen
  end interface

contains

  ! the NUL-terminated text of sac_last_error as a Fortran string (for die())
  function sac_error_text(ctx) result(msg)
    type(c_ptr), intent(in) :: ctx
    character(len=:), allocatable :: msg
    character(kind=c_char), pointer :: p(:)
    type(c_ptr) :: s
    integer :: n, i
    s = sac_last_error(ctx)
    n = int(c_strlen(s))
    call c_f_pointer(s, p, [n])
    allocate(character(len=n) :: msg)
    do i = 1, n
       msg(i:i) = p(i)
    end do
  end function sac_error_text

  ! a Fortran string into a NUL-terminated CHARACTER*11 component
  subroutine sac_set_name(dst, src)
    character(kind=c_char), intent(out) :: dst(11)
    character(len=*), intent(in) :: src
    integer :: i, n
    dst = c_null_char
    n = min(len_trim(src), 10)
    do i = 1, n
       dst(i) = src(i:i)
    end do
  end subroutine sac_set_name
end module sacgpu
