! cadmas_gpu.f90 -- ISO_C_BINDING interface to libcadmas_gpu.so for the
! CADMAS-SURF/3D time loop (Fortran 2003).
!
! The derived types are interoperable with the structs of cadmas_gpu.h
! (same member order and kinds).  cadmas_params%damp(m,jd) is DAMP(m,jd)
! of /VF_APHYSR/: the C array damp[4][4] stored row-major is the same
! memory as the Fortran array damp(4,4) stored column-major.
!
! Use from the time loop (vf_a1main.f):
!   after the set-up block (VF_CINIT done, before the loop at :919)
!     CALL CADMAS_DEFAULT_PARAMS(PRM)      ! then copy the COMMON values
!     IERR = CADMAS_CREATE(DIMS, PRM, HGPU)
!     IERR = CADMAS_UPLOAD_STATIC(HGPU, STAT)
!   in place of CALL VF_V1CAL(...) (:1058-1066)
!     IERR = VF_V1CAL_GPU(HGPU, TNOW, DTNOW, NNOW, UU, VV, WW, PP, FF,
!    &                    NF, INDC, BCU, BCV, BCW, BCP, BCF)
!   in place of CALL VF_F1CAL(...) (:1104-1115)
!     IERR = VF_F1CAL_GPU(HGPU, TNOW, DTNOW, NNOW, UU, VV, WW, PP, FF,
!    &                    NF, INDC, BCU, BCV, BCW, BCP, BCF)
!   and IERR /= CADMAS_OK goes to VF_A2ERR with CADMAS_STRERROR's text.
module cadmas_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: CADMAS_OK = 0, CADMAS_EINVAL = 1, CADMAS_ECUDA = 2, &
       CADMAS_ENOTCONV = 3, CADMAS_EDIVERGE = 4, CADMAS_EPIVOT = 5, CADMAS_EPG = 6, &
       CADMAS_ECAP = 7, CADMAS_ENOMEM = 8, CADMAS_EUNSUPPORTED = 9, CADMAS_ENOSTATIC = 10, &
       CADMAS_ETIMEOUT = 11, CADMAS_ESCRATCH = 12, CADMAS_EIO = 13

  type, bind(C) :: cadmas_dims
     integer(c_int) :: numi, numj, numk, numb
  end type cadmas_dims

  type, bind(C) :: cadmas_params
     real(c_double) :: rho0, grz0, vvmax, cgpara, cgepsa, cgepsr, cgdiv
     real(c_double) :: flower, fupper, plower, scmvp, wvlvl, wbub
     real(c_double) :: glxmin, glxmax, glymin, glymax
     real(c_double) :: damp(4, 4)
     integer(c_int) :: idamp(4)
     integer(c_int) :: icgtyp, icgmax, ibsuw0
     integer(c_int) :: precond_ti, precond_tj
     integer(c_int) :: diag_relres
     integer(c_int) :: solver
     integer(c_int) :: warm_start
     integer(c_int) :: precond_split
     integer(c_int) :: idrop
     integer(c_int) :: iscmff
     integer(c_int) :: leqk, pad0
     real(c_double) :: anu0, scmk, akmink, akmine, akinik, akinie
     real(c_double) :: akcmu, aksgk, aksge, akc1, akc2, akc3
     real(c_double) :: akk0, aka0                ! log law (IB 6, 8)
     real(c_double) :: mixed_eps_inner           ! floor of the FP32 inner tolerance (solver 1)
     real(c_double) :: wait_limit_s              ! device-side wait limit, seconds
     integer(c_int) :: sweep_occupancy, dot_passes  ! MILU sweep blocks per SM (0 = default); FP32 sums in the sweeps (0)
  end type cadmas_params

  ! c_loc() of the static arrays (XX(6,NUMI) ... INDB(4,NUMB))
  type, bind(C) :: cadmas_static
     type(c_ptr) :: xx, yy, zz
     type(c_ptr) :: ggv, ggx, ggy, ggz
     type(c_ptr) :: glv, glx, gly, glz
     type(c_ptr) :: cd0, anu
     type(c_ptr) :: indx, indy, indz, indb
     type(c_ptr) :: indbk, indbe, bck, bce   ! k-epsilon (LEQK /= 0)
     type(c_ptr) :: bcvi                     ! roughness of rough walls
  end type cadmas_static

  type, bind(C) :: cadmas_stats
     real(c_double) :: fsum, fcut, cgbnrm, cgxnrm, divnorm, true_relres
     integer(c_int) :: icgitr, nums, last_status, fallbacks
  end type cadmas_stats

  interface
     subroutine cadmas_default_params(p) bind(C, name='cadmas_default_params')
       import :: cadmas_params
       type(cadmas_params), intent(out) :: p
     end subroutine cadmas_default_params

     integer(c_int) function cadmas_create(d, p, h) bind(C, name='cadmas_create')
       import :: c_int, c_ptr, cadmas_dims, cadmas_params
       type(cadmas_dims), intent(in) :: d
       type(cadmas_params), intent(in) :: p
       type(c_ptr), intent(out) :: h
     end function cadmas_create

     integer(c_int) function cadmas_destroy(h) bind(C, name='cadmas_destroy')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function cadmas_destroy

     integer(c_int) function cadmas_upload_static(h, s) bind(C, name='cadmas_upload_static')
       import :: c_int, c_ptr, cadmas_static
       type(c_ptr), value :: h
       type(cadmas_static), intent(in) :: s
     end function cadmas_upload_static

     integer(c_int) function cadmas_get_stats(h, st) bind(C, name='cadmas_get_stats')
       import :: c_int, c_ptr, cadmas_stats
       type(c_ptr), value :: h
       type(cadmas_stats), intent(out) :: st
     end function cadmas_get_stats

     integer(c_int) function vf_v1cal_gpu(h, tnow, dtnow, nnow, uu, vv, ww, pp, ff, nf, indc, &
          bcu, bcv, bcw, bcp, bcf) bind(C, name='vf_v1cal_gpu_')
       import :: c_int, c_double, c_ptr
       type(c_ptr), intent(in) :: h
       real(c_double), intent(in) :: tnow, dtnow
       integer(c_int), intent(in) :: nnow
       real(c_double), intent(inout) :: uu(*), vv(*), ww(*), pp(*), ff(*)
       integer(c_int), intent(inout) :: nf(*), indc(*)
       real(c_double), intent(inout) :: bcu(*), bcv(*), bcw(*), bcp(*), bcf(*)
     end function vf_v1cal_gpu

     integer(c_int) function vf_f1cal_gpu(h, tnow, dtnow, nnow, uu, vv, ww, pp, ff, nf, indc, &
          bcu, bcv, bcw, bcp, bcf) bind(C, name='vf_f1cal_gpu_')
       import :: c_int, c_double, c_ptr
       type(c_ptr), intent(in) :: h
       real(c_double), intent(in) :: tnow, dtnow
       integer(c_int), intent(in) :: nnow
       real(c_double), intent(inout) :: uu(*), vv(*), ww(*), pp(*), ff(*)
       integer(c_int), intent(inout) :: nf(*), indc(*)
       real(c_double), intent(inout) :: bcu(*), bcv(*), bcw(*), bcp(*), bcf(*)
     end function vf_f1cal_gpu

     ! Both calls in one, advancing TNOW/NNOW by DTNOW itself.
     integer(c_int) function vf_step_gpu(h, dtnow, uu, vv, ww, pp, ff, nf, indc, &
          bcu, bcv, bcw, bcp, bcf, tnow, nnow) bind(C, name='vf_step_gpu_')
       import :: c_int, c_double, c_ptr
       type(c_ptr), intent(in) :: h
       real(c_double), intent(in) :: dtnow
       real(c_double), intent(inout) :: uu(*), vv(*), ww(*), pp(*), ff(*)
       integer(c_int), intent(inout) :: nf(*), indc(*)
       real(c_double), intent(inout) :: bcu(*), bcv(*), bcw(*), bcp(*), bcf(*)
       real(c_double), intent(inout) :: tnow
       integer(c_int), intent(inout) :: nnow
     end function vf_step_gpu

     ! Restart file of the reference (vf_or1ini.f / vf_or1trn.f / vf_ir1inp.f);
     ! path is a NUL-terminated name (TRIM(NAME)//C_NULL_CHAR).
     integer(c_int) function cadmas_restart_create(h, path) bind(C, name='cadmas_restart_create')
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
     end function cadmas_restart_create

     integer(c_int) function cadmas_restart_append(h, path) bind(C, name='cadmas_restart_append')
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
     end function cadmas_restart_append

     integer(c_int) function cadmas_restart_load(h, path, nnow) bind(C, name='cadmas_restart_load')
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
       integer(c_int), value :: nnow
     end function cadmas_restart_load

     type(c_ptr) function cadmas_strerror(status) bind(C, name='cadmas_strerror')
       import :: c_int, c_ptr
       integer(c_int), value :: status
     end function cadmas_strerror
  end interface
end module cadmas_gpu
