! pcom_gpu.f90 -- ISO_C_BINDING interface module for include/pcom_gpu.h.
!
! A PCOM build that keeps main.f90 adds this module, creates a handle after
! inistat (main.f90:122) and replaces the per-step call block of
! main.f90:205-223 (and den_prho at main.f90:179,200) with pcom_gpu_step.
! The derived types are bind(c) mirrors of the C structs, member for member
! and in the same order; arrays are passed as c_loc() of the module-global
! arrays of mod_arrays, which are already in Fortran order over the padded
! ni x nj domain.  type_mat arrays (g?j%dx, prho) are passed as they are:
! their memory is the AoS pair layout the C side expects.
module mod_pcom_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: PCOM_OK = 0, PCOM_ERR_ARG = 1, PCOM_ERR_CUDA = 2, &
                               PCOM_ERR_STATE = 3, PCOM_ERR_NUMERIC = 4, PCOM_ERR_TIMEOUT = 5
  integer(c_int32_t), parameter :: PCOM_PREC_FP64 = 0, PCOM_PREC_MIXED = 1, PCOM_LIT_R8 = 16

  ! sizes and time steps (mod_param.f90:40-81)
  type, bind(c) :: pcom_dims
    integer(c_int32_t) :: glo_ni, glo_nj, nk
    integer(c_int32_t) :: ni, nj
    integer(c_int32_t) :: dtbt, dtbc
    integer(c_int32_t) :: flags
    integer(c_int32_t) :: rst
    integer(c_int32_t) :: reserved(3)
  end type pcom_dims

  ! static grid data (main.f90:105-122)
  type, bind(c) :: pcom_static
    type(c_ptr) :: rh(4), tn(4), dx(4)
    type(c_ptr) :: z1, pr1, dz1, dpr1
    type(c_ptr) :: z2, pr2, dz2, dpr2
    type(c_ptr) :: msk_t, lev_t, msk_u, lev_u
    type(c_ptr) :: phih_t, prh_t, phih_u, prh_u
    type(c_ptr) :: cv1, cv2, cor
    type(c_ptr) :: km, kh
    type(c_ptr) :: graphihx, graphihy
  end type pcom_static

  ! prognostic and carried state (mod_arrays.f90:80-116); c_null_ptr skips a field
  type, bind(c) :: pcom_state
    type(c_ptr) :: tc, sc, tp, sp
    type(c_ptr) :: uc, vc, up, vp
    type(c_ptr) :: auc, aup, aupp, avc, avp, avpp
    type(c_ptr) :: ubc, vbc, ubp, vbp
    type(c_ptr) :: chc, chp, mch, mch2
    type(c_ptr) :: am
    type(c_ptr) :: prho
    type(c_ptr) :: alpha, adp
    type(c_ptr) :: wm
  end type pcom_state

  ! daily surface forcing after int_bnd (mod_int.f90:649-691)
  type, bind(c) :: pcom_forcing
    type(c_ptr) :: taux, tauy, t, s, pa, fw
  end type pcom_forcing

  ! time-mean accumulators and their record counters (mod_type.f90:155-205)
  type, bind(c) :: pcom_accum
    type(c_ptr) :: act, acs, acr, acu, acv, acw
    type(c_ptr) :: acch, acssh
    integer(c_int32_t) :: n_ts, n_uv, n_w, n_ch, n_ssh
  end type pcom_accum

  interface
    integer(c_int) function pcom_gpu_create(d, h) bind(c)
      import; type(pcom_dims), intent(in) :: d; type(c_ptr) :: h
    end function
    integer(c_int) function pcom_gpu_destroy(h) bind(c)
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function pcom_gpu_upload_static(h, s) bind(c)
      import; type(c_ptr), value :: h; type(pcom_static), intent(in) :: s
    end function
    integer(c_int) function pcom_gpu_set_state(h, s) bind(c)
      import; type(c_ptr), value :: h; type(pcom_state), intent(in) :: s
    end function
    integer(c_int) function pcom_gpu_get_state(h, s) bind(c)
      import; type(c_ptr), value :: h; type(pcom_state) :: s
    end function
    integer(c_int) function pcom_gpu_set_forcing(h, f) bind(c)
      import; type(c_ptr), value :: h; type(pcom_forcing), intent(in) :: f
    end function
    integer(c_int) function pcom_gpu_set_forcing_async(h, f) bind(c)
      import; type(c_ptr), value :: h; type(pcom_forcing), intent(in) :: f
    end function
    integer(c_int) function pcom_gpu_get_state_async(h, s) bind(c)
      import; type(c_ptr), value :: h; type(pcom_state) :: s
    end function
    integer(c_int) function pcom_gpu_get_accum(h, a) bind(c)
      import; type(c_ptr), value :: h; type(pcom_accum) :: a
    end function
    integer(c_int) function pcom_gpu_reset_accum(h) bind(c)
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function pcom_gpu_den_prho(h) bind(c)
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function pcom_gpu_step(h, i) bind(c)
      import; type(c_ptr), value :: h; integer(c_int64_t), value :: i
    end function
    integer(c_int) function pcom_gpu_step_async(h, i) bind(c)
      import; type(c_ptr), value :: h; integer(c_int64_t), value :: i
    end function
    integer(c_int) function pcom_gpu_phase(h, p, i) bind(c)
      import; type(c_ptr), value :: h; integer(c_int32_t), value :: p; integer(c_int64_t), value :: i
    end function
    integer(c_int) function pcom_gpu_sync(h) bind(c)
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function pcom_gpu_check_finite(h) bind(c)
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function pcom_gpu_get_field(h, name, host, n) bind(c)
      import; type(c_ptr), value :: h; character(kind=c_char) :: name(*)
      real(c_double) :: host(*); integer(c_int64_t), value :: n
    end function
    integer(c_int) function pcom_gpu_last_error(buf, n) bind(c)
      import; character(kind=c_char) :: buf(*); integer(c_int32_t), value :: n
    end function
  end interface
end module mod_pcom_gpu
