! Generated by include/make_fortran_module.py from include/fourphonon_b200.h: do not edit.
! ISO_C_BINDING interfaces of the B200 scattering-rate path.  Each function replaces the
! Fortran subroutine named in the header's comment above its prototype and takes that
! subroutine's arguments, in the same order, plus the context and the fp4_globals record.
module fp4_b200
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: FP4_OK = 0
  integer(c_int), parameter :: FP4_E_ARG = -1
  integer(c_int), parameter :: FP4_E_CUDA = -2
  integer(c_int), parameter :: FP4_E_CAPACITY = -3
  integer(c_int), parameter :: FP4_E_TIMEOUT = -4
  integer(c_int), parameter :: FP4_E_STATE = -5
  integer(c_int), parameter :: FP4_PREC_FP64 = 0
  integer(c_int), parameter :: FP4_PREC_MIXED = 1
  integer(c_int), parameter :: FP4_PREC_MIXED_SIMT = 2

  ! The reference's module globals (Src/config.f90:9-47), fields in the header's order.
  type, bind(c) :: fp4_globals
     integer(c_int32_t) :: ngrid(3)
     integer(c_int32_t) :: nbands
     real(c_double)     :: rlattvec(3,3)
     real(c_double)     :: T
     real(c_double)     :: scalebroad
     real(c_double)     :: omega_max
     integer(c_int32_t) :: onlyharmonic
     integer(c_int32_t) :: nelements
     integer(c_int32_t) :: natoms
     type(c_ptr)        :: masses
     type(c_ptr)        :: types
  end type fp4_globals

  interface
     integer(c_int) function fp4_create(ctx, device) bind(c, name="fp4_create")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), intent(out) :: ctx
       integer(c_int), value :: device
     end function fp4_create

     integer(c_int) function fp4_destroy(ctx) bind(c, name="fp4_destroy")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
     end function fp4_destroy

     type(c_ptr) function fp4_last_error(ctx) bind(c, name="fp4_last_error")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
     end function fp4_last_error

     integer(c_int) function fp4_set_precision(ctx, precision) bind(c, name="fp4_set_precision")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       integer(c_int), value :: precision
     end function fp4_set_precision

     integer(c_int) function fp4_np_driver(ctx, g, energy, velocity, nlist, list, ijk, n_plus, &
          pspace_plus, n_minus, pspace_minus) bind(c, name="fp4_np_driver")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), intent(inout) :: n_plus(*)
       real(c_double), intent(inout) :: pspace_plus(*)
       integer(c_int32_t), intent(inout) :: n_minus(*)
       real(c_double), intent(inout) :: pspace_minus(*)
     end function fp4_np_driver

     integer(c_int) function fp4_np_driver_4ph(ctx, g, energy, velocity, nlist, list, ijk, &
          n_plusplus, pspace_plusplus, n_plusminus, pspace_plusminus, n_minusminus, &
          pspace_minusminus) bind(c, name="fp4_np_driver_4ph")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int64_t), intent(inout) :: n_plusplus(*)
       real(c_double), intent(inout) :: pspace_plusplus(*)
       integer(c_int64_t), intent(inout) :: n_plusminus(*)
       real(c_double), intent(inout) :: pspace_plusminus(*)
       integer(c_int64_t), intent(inout) :: n_minusminus(*)
       real(c_double), intent(inout) :: pspace_minusminus(*)
     end function fp4_np_driver_4ph

     integer(c_int) function fp4_ind_only_driver(ctx, g, energy, velocity, nlist, list, ijk, &
          n_plus, n_minus, ind2_plus, ind3_plus, ind2_minus, ind3_minus) &
          bind(c, name="fp4_ind_only_driver")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), intent(in) :: n_plus(*)
       integer(c_int32_t), intent(in) :: n_minus(*)
       integer(c_int32_t), intent(inout) :: ind2_plus(*)
       integer(c_int32_t), intent(inout) :: ind3_plus(*)
       integer(c_int32_t), intent(inout) :: ind2_minus(*)
       integer(c_int32_t), intent(inout) :: ind3_minus(*)
     end function fp4_ind_only_driver

     integer(c_int) function fp4_ind_only_driver_4ph(ctx, g, energy, velocity, nlist, list, ijk, &
          n_plusplus, n_plusminus, n_minusminus, ind2_pp, ind3_pp, ind4_pp, ind2_pm, ind3_pm, &
          ind4_pm, ind2_mm, ind3_mm, ind4_mm) bind(c, name="fp4_ind_only_driver_4ph")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int64_t), intent(in) :: n_plusplus(*)
       integer(c_int64_t), intent(in) :: n_plusminus(*)
       integer(c_int64_t), intent(in) :: n_minusminus(*)
       integer(c_int64_t), intent(inout) :: ind2_pp(*)
       integer(c_int64_t), intent(inout) :: ind3_pp(*)
       integer(c_int64_t), intent(inout) :: ind4_pp(*)
       integer(c_int64_t), intent(inout) :: ind2_pm(*)
       integer(c_int64_t), intent(inout) :: ind3_pm(*)
       integer(c_int64_t), intent(inout) :: ind4_pm(*)
       integer(c_int64_t), intent(inout) :: ind2_mm(*)
       integer(c_int64_t), intent(inout) :: ind3_mm(*)
       integer(c_int64_t), intent(inout) :: ind4_mm(*)
     end function fp4_ind_only_driver_4ph

     integer(c_int) function fp4_rta_driver(ctx, g, energy, velocity, eigenvect, nlist, list, ijk, &
          ntri, phi, r_j, r_k, index_i, index_j, index_k, rate, rate_plus, rate_minus, wp3_plus, &
          wp3_minus) bind(c, name="fp4_rta_driver")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), value :: ntri
       real(c_double), intent(in) :: phi(*)
       real(c_double), intent(in) :: r_j(*)
       real(c_double), intent(in) :: r_k(*)
       integer(c_int32_t), intent(in) :: index_i(*)
       integer(c_int32_t), intent(in) :: index_j(*)
       integer(c_int32_t), intent(in) :: index_k(*)
       real(c_double), intent(inout) :: rate(*)
       real(c_double), intent(inout) :: rate_plus(*)
       real(c_double), intent(inout) :: rate_minus(*)
       real(c_double), intent(inout) :: wp3_plus(*)
       real(c_double), intent(inout) :: wp3_minus(*)
     end function fp4_rta_driver

     integer(c_int) function fp4_rta_driver_4ph(ctx, g, energy, velocity, eigenvect, nlist, list, &
          ijk, ntri, psi, r_j, r_k, r_l, index_i, index_j, index_k, index_l, rate_4ph, &
          rate_plusplus, rate_plusminus, rate_minusminus, wp4_plusplus, wp4_plusminus, &
          wp4_minusminus) bind(c, name="fp4_rta_driver_4ph")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), value :: ntri
       real(c_double), intent(in) :: psi(*)
       real(c_double), intent(in) :: r_j(*)
       real(c_double), intent(in) :: r_k(*)
       real(c_double), intent(in) :: r_l(*)
       integer(c_int32_t), intent(in) :: index_i(*)
       integer(c_int32_t), intent(in) :: index_j(*)
       integer(c_int32_t), intent(in) :: index_k(*)
       integer(c_int32_t), intent(in) :: index_l(*)
       real(c_double), intent(inout) :: rate_4ph(*)
       real(c_double), intent(inout) :: rate_plusplus(*)
       real(c_double), intent(inout) :: rate_plusminus(*)
       real(c_double), intent(inout) :: rate_minusminus(*)
       real(c_double), intent(inout) :: wp4_plusplus(*)
       real(c_double), intent(inout) :: wp4_plusminus(*)
       real(c_double), intent(inout) :: wp4_minusminus(*)
     end function fp4_rta_driver_4ph

     integer(c_int) function fp4_rta_driver_4ph_multi_t(ctx, g, nT, temperatures, energy, velocity, &
          eigenvect, nlist, list, ijk, ntri, psi, r_j, r_k, r_l, index_i, index_j, index_k, &
          index_l, rate_plusplus, rate_plusminus, rate_minusminus, wp4_plusplus, wp4_plusminus, &
          wp4_minusminus) bind(c, name="fp4_rta_driver_4ph_multi_t")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       integer(c_int32_t), value :: nT
       real(c_double), intent(in) :: temperatures(*)
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), value :: ntri
       real(c_double), intent(in) :: psi(*)
       real(c_double), intent(in) :: r_j(*)
       real(c_double), intent(in) :: r_k(*)
       real(c_double), intent(in) :: r_l(*)
       integer(c_int32_t), intent(in) :: index_i(*)
       integer(c_int32_t), intent(in) :: index_j(*)
       integer(c_int32_t), intent(in) :: index_k(*)
       integer(c_int32_t), intent(in) :: index_l(*)
       real(c_double), intent(inout) :: rate_plusplus(*)
       real(c_double), intent(inout) :: rate_plusminus(*)
       real(c_double), intent(inout) :: rate_minusminus(*)
       real(c_double), intent(inout) :: wp4_plusplus(*)
       real(c_double), intent(inout) :: wp4_plusminus(*)
       real(c_double), intent(inout) :: wp4_minusminus(*)
     end function fp4_rta_driver_4ph_multi_t

     integer(c_int) function fp4_ind_driver(ctx, g, energy, velocity, eigenvect, nlist, list, ijk, &
          n_plus, n_minus, ntri, phi, r_j, r_k, index_i, index_j, index_k, ind2_plus, ind3_plus, &
          gamma_plus, ind2_minus, ind3_minus, gamma_minus, rate, rate_plus, rate_minus, wp3_plus, &
          wp3_minus) bind(c, name="fp4_ind_driver")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), intent(in) :: n_plus(*)
       integer(c_int32_t), intent(in) :: n_minus(*)
       integer(c_int32_t), value :: ntri
       real(c_double), intent(in) :: phi(*)
       real(c_double), intent(in) :: r_j(*)
       real(c_double), intent(in) :: r_k(*)
       integer(c_int32_t), intent(in) :: index_i(*)
       integer(c_int32_t), intent(in) :: index_j(*)
       integer(c_int32_t), intent(in) :: index_k(*)
       integer(c_int32_t), intent(inout) :: ind2_plus(*)
       integer(c_int32_t), intent(inout) :: ind3_plus(*)
       real(c_double), intent(inout) :: gamma_plus(*)
       integer(c_int32_t), intent(inout) :: ind2_minus(*)
       integer(c_int32_t), intent(inout) :: ind3_minus(*)
       real(c_double), intent(inout) :: gamma_minus(*)
       real(c_double), intent(inout) :: rate(*)
       real(c_double), intent(inout) :: rate_plus(*)
       real(c_double), intent(inout) :: rate_minus(*)
       real(c_double), intent(inout) :: wp3_plus(*)
       real(c_double), intent(inout) :: wp3_minus(*)
     end function fp4_ind_driver

     integer(c_int) function fp4_ind_driver_4ph(ctx, g, energy, velocity, eigenvect, nlist, list, &
          ijk, n_plusplus, n_plusminus, n_minusminus, ntri, psi, r_j, r_k, r_l, index_i, index_j, &
          index_k, index_l, ind2_pp, ind3_pp, ind4_pp, gamma_pp, ind2_pm, ind3_pm, ind4_pm, &
          gamma_pm, ind2_mm, ind3_mm, ind4_mm, gamma_mm, rate_4ph, rate_plusplus, rate_plusminus, &
          rate_minusminus, wp4_plusplus, wp4_plusminus, wp4_minusminus) &
          bind(c, name="fp4_ind_driver_4ph")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int64_t), intent(in) :: n_plusplus(*)
       integer(c_int64_t), intent(in) :: n_plusminus(*)
       integer(c_int64_t), intent(in) :: n_minusminus(*)
       integer(c_int32_t), value :: ntri
       real(c_double), intent(in) :: psi(*)
       real(c_double), intent(in) :: r_j(*)
       real(c_double), intent(in) :: r_k(*)
       real(c_double), intent(in) :: r_l(*)
       integer(c_int32_t), intent(in) :: index_i(*)
       integer(c_int32_t), intent(in) :: index_j(*)
       integer(c_int32_t), intent(in) :: index_k(*)
       integer(c_int32_t), intent(in) :: index_l(*)
       integer(c_int64_t), intent(inout) :: ind2_pp(*)
       integer(c_int64_t), intent(inout) :: ind3_pp(*)
       integer(c_int64_t), intent(inout) :: ind4_pp(*)
       real(c_double), intent(inout) :: gamma_pp(*)
       integer(c_int64_t), intent(inout) :: ind2_pm(*)
       integer(c_int64_t), intent(inout) :: ind3_pm(*)
       integer(c_int64_t), intent(inout) :: ind4_pm(*)
       real(c_double), intent(inout) :: gamma_pm(*)
       integer(c_int64_t), intent(inout) :: ind2_mm(*)
       integer(c_int64_t), intent(inout) :: ind3_mm(*)
       integer(c_int64_t), intent(inout) :: ind4_mm(*)
       real(c_double), intent(inout) :: gamma_mm(*)
       real(c_double), intent(inout) :: rate_4ph(*)
       real(c_double), intent(inout) :: rate_plusplus(*)
       real(c_double), intent(inout) :: rate_plusminus(*)
       real(c_double), intent(inout) :: rate_minusminus(*)
       real(c_double), intent(inout) :: wp4_plusplus(*)
       real(c_double), intent(inout) :: wp4_plusminus(*)
       real(c_double), intent(inout) :: wp4_minusminus(*)
     end function fp4_ind_driver_4ph

     integer(c_int) function fp4_iteration0(ctx, g, nlist, nequi, allequilist, nsymm_rot, omega, &
          velocity, tau_zero, f_n) bind(c, name="fp4_iteration0")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: nequi(*)
       integer(c_int32_t), intent(in) :: allequilist(*)
       integer(c_int32_t), value :: nsymm_rot
       real(c_double), intent(in) :: omega(*)
       real(c_double), intent(in) :: velocity(*)
       real(c_double), intent(in) :: tau_zero(*)
       real(c_double), intent(inout) :: f_n(*)
     end function fp4_iteration0

     integer(c_int) function fp4_iteration(ctx, g, nlist, nequi, allequilist, typeofsymmetry, &
          nsymm_rot, id_equi, symmetrizers, n_plus, n_minus, ntotal_plus, ntotal_minus, ind2_plus, &
          ind3_plus, ind2_minus, ind3_minus, omega, velocity, gamma_plus, gamma_minus, tau_zero, f_n) &
          bind(c, name="fp4_iteration")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: nequi(*)
       integer(c_int32_t), intent(in) :: allequilist(*)
       integer(c_int32_t), intent(in) :: typeofsymmetry(*)
       integer(c_int32_t), value :: nsymm_rot
       integer(c_int32_t), intent(in) :: id_equi(*)
       real(c_double), intent(in) :: symmetrizers(*)
       integer(c_int32_t), intent(in) :: n_plus(*)
       integer(c_int32_t), intent(in) :: n_minus(*)
       integer(c_int32_t), value :: ntotal_plus
       integer(c_int32_t), value :: ntotal_minus
       integer(c_int32_t), intent(in) :: ind2_plus(*)
       integer(c_int32_t), intent(in) :: ind3_plus(*)
       integer(c_int32_t), intent(in) :: ind2_minus(*)
       integer(c_int32_t), intent(in) :: ind3_minus(*)
       real(c_double), intent(in) :: omega(*)
       real(c_double), intent(in) :: velocity(*)
       real(c_double), intent(in) :: gamma_plus(*)
       real(c_double), intent(in) :: gamma_minus(*)
       real(c_double), intent(in) :: tau_zero(*)
       real(c_double), intent(inout) :: f_n(*)
     end function fp4_iteration

     integer(c_int) function fp4_iteration_jacobi(ctx, g, nlist, nequi, allequi, typeofsym, &
          nsymm_rot, id_equi, symmetrizers, n_plus, n_minus, ntotal_plus, ntotal_minus, ind2_plus, &
          ind3_plus, ind2_minus, ind3_minus, energy, velocity, gamma_plus, gamma_minus, tau_zero, &
          f_n) bind(c, name="fp4_iteration_jacobi")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: nequi(*)
       integer(c_int32_t), intent(in) :: allequi(*)
       integer(c_int32_t), intent(in) :: typeofsym(*)
       integer(c_int32_t), value :: nsymm_rot
       integer(c_int32_t), intent(in) :: id_equi(*)
       real(c_double), intent(in) :: symmetrizers(*)
       integer(c_int32_t), intent(in) :: n_plus(*)
       integer(c_int32_t), intent(in) :: n_minus(*)
       integer(c_int32_t), value :: ntotal_plus
       integer(c_int32_t), value :: ntotal_minus
       integer(c_int32_t), intent(in) :: ind2_plus(*)
       integer(c_int32_t), intent(in) :: ind3_plus(*)
       integer(c_int32_t), intent(in) :: ind2_minus(*)
       integer(c_int32_t), intent(in) :: ind3_minus(*)
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       real(c_double), intent(in) :: gamma_plus(*)
       real(c_double), intent(in) :: gamma_minus(*)
       real(c_double), intent(in) :: tau_zero(*)
       real(c_double), intent(inout) :: f_n(*)
     end function fp4_iteration_jacobi

     integer(c_int) function fp4_iteration_4ph(ctx, g, nlist, nequi, allequilist, typeofsymmetry, &
          nsymm_rot, id_equi, symmetrizers, n_plus, n_minus, ntotal_plus, ntotal_minus, n_plusplus, &
          n_plusminus, n_minusminus, ntotal_plusplus, ntotal_plusminus, ntotal_minusminus, &
          ind2_plus, ind3_plus, ind2_minus, ind3_minus, ind2_pp, ind3_pp, ind4_pp, ind2_pm, &
          ind3_pm, ind4_pm, ind2_mm, ind3_mm, ind4_mm, omega, velocity, gamma_plus, gamma_minus, &
          gamma_pp, gamma_pm, gamma_mm, tau_zero, f_n) bind(c, name="fp4_iteration_4ph")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: nequi(*)
       integer(c_int32_t), intent(in) :: allequilist(*)
       integer(c_int32_t), intent(in) :: typeofsymmetry(*)
       integer(c_int32_t), value :: nsymm_rot
       integer(c_int32_t), intent(in) :: id_equi(*)
       real(c_double), intent(in) :: symmetrizers(*)
       integer(c_int32_t), intent(in) :: n_plus(*)
       integer(c_int32_t), intent(in) :: n_minus(*)
       integer(c_int32_t), value :: ntotal_plus
       integer(c_int32_t), value :: ntotal_minus
       integer(c_int64_t), intent(in) :: n_plusplus(*)
       integer(c_int64_t), intent(in) :: n_plusminus(*)
       integer(c_int64_t), intent(in) :: n_minusminus(*)
       integer(c_int64_t), value :: ntotal_plusplus
       integer(c_int64_t), value :: ntotal_plusminus
       integer(c_int64_t), value :: ntotal_minusminus
       integer(c_int32_t), intent(in) :: ind2_plus(*)
       integer(c_int32_t), intent(in) :: ind3_plus(*)
       integer(c_int32_t), intent(in) :: ind2_minus(*)
       integer(c_int32_t), intent(in) :: ind3_minus(*)
       integer(c_int64_t), intent(in) :: ind2_pp(*)
       integer(c_int64_t), intent(in) :: ind3_pp(*)
       integer(c_int64_t), intent(in) :: ind4_pp(*)
       integer(c_int64_t), intent(in) :: ind2_pm(*)
       integer(c_int64_t), intent(in) :: ind3_pm(*)
       integer(c_int64_t), intent(in) :: ind4_pm(*)
       integer(c_int64_t), intent(in) :: ind2_mm(*)
       integer(c_int64_t), intent(in) :: ind3_mm(*)
       integer(c_int64_t), intent(in) :: ind4_mm(*)
       real(c_double), intent(in) :: omega(*)
       real(c_double), intent(in) :: velocity(*)
       real(c_double), intent(in) :: gamma_plus(*)
       real(c_double), intent(in) :: gamma_minus(*)
       real(c_double), intent(in) :: gamma_pp(*)
       real(c_double), intent(in) :: gamma_pm(*)
       real(c_double), intent(in) :: gamma_mm(*)
       real(c_double), intent(in) :: tau_zero(*)
       real(c_double), intent(inout) :: f_n(*)
     end function fp4_iteration_4ph

     integer(c_int) function fp4_symmetrize_fn(ctx, g, symmetrizers, f_n) &
          bind(c, name="fp4_symmetrize_fn")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: symmetrizers(*)
       real(c_double), intent(inout) :: f_n(*)
     end function fp4_symmetrize_fn

     integer(c_int) function fp4_tconduct(ctx, g, V, omega, velocity, f_n, thconductivity, &
          thconductivitymode) bind(c, name="fp4_tconduct")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), value :: V
       real(c_double), intent(in) :: omega(*)
       real(c_double), intent(in) :: velocity(*)
       real(c_double), intent(in) :: f_n(*)
       real(c_double), intent(inout) :: thconductivity(*)
       real(c_double), intent(inout) :: thconductivitymode(*)
     end function fp4_tconduct

     integer(c_int) function fp4_last_stats(ctx, n_processes, n_contracted, call_ms, kernel_ms, &
          launches) bind(c, name="fp4_last_stats")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(out) :: n_processes
       integer(c_int64_t), intent(out) :: n_contracted
       real(c_double), intent(out) :: call_ms
       real(c_double), intent(out) :: kernel_ms
       integer(c_int64_t), intent(out) :: launches
     end function fp4_last_stats

     integer(c_int) function fp4_np_driver_sample(ctx, g, energy, velocity, nlist, list, ijk, &
          nsamples, seed, n_plus, pspace_plus, n_minus, pspace_minus) &
          bind(c, name="fp4_np_driver_sample")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int64_t), value :: nsamples
       integer(c_int64_t), value :: seed
       integer(c_int32_t), intent(inout) :: n_plus(*)
       real(c_double), intent(inout) :: pspace_plus(*)
       integer(c_int32_t), intent(inout) :: n_minus(*)
       real(c_double), intent(inout) :: pspace_minus(*)
     end function fp4_np_driver_sample

     integer(c_int) function fp4_rta_driver_sample(ctx, g, energy, velocity, eigenvect, nlist, &
          list, ijk, ntri, phi, r_j, r_k, index_i, index_j, index_k, nsamples, seed, rate, &
          rate_plus, rate_minus, wp3_plus, wp3_minus) bind(c, name="fp4_rta_driver_sample")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), value :: ntri
       real(c_double), intent(in) :: phi(*)
       real(c_double), intent(in) :: r_j(*)
       real(c_double), intent(in) :: r_k(*)
       integer(c_int32_t), intent(in) :: index_i(*)
       integer(c_int32_t), intent(in) :: index_j(*)
       integer(c_int32_t), intent(in) :: index_k(*)
       integer(c_int64_t), value :: nsamples
       integer(c_int64_t), value :: seed
       real(c_double), intent(inout) :: rate(*)
       real(c_double), intent(inout) :: rate_plus(*)
       real(c_double), intent(inout) :: rate_minus(*)
       real(c_double), intent(inout) :: wp3_plus(*)
       real(c_double), intent(inout) :: wp3_minus(*)
     end function fp4_rta_driver_sample

     integer(c_int) function fp4_np_driver_4ph_sample(ctx, g, energy, velocity, nlist, list, ijk, &
          nsamples, seed, n_plusplus, pspace_plusplus, n_plusminus, pspace_plusminus, n_minusminus, &
          pspace_minusminus) bind(c, name="fp4_np_driver_4ph_sample")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int64_t), value :: nsamples
       integer(c_int64_t), value :: seed
       integer(c_int64_t), intent(inout) :: n_plusplus(*)
       real(c_double), intent(inout) :: pspace_plusplus(*)
       integer(c_int64_t), intent(inout) :: n_plusminus(*)
       real(c_double), intent(inout) :: pspace_plusminus(*)
       integer(c_int64_t), intent(inout) :: n_minusminus(*)
       real(c_double), intent(inout) :: pspace_minusminus(*)
     end function fp4_np_driver_4ph_sample

     integer(c_int) function fp4_rta_driver_4ph_sample(ctx, g, energy, velocity, eigenvect, nlist, &
          list, ijk, ntri, psi, r_j, r_k, r_l, index_i, index_j, index_k, index_l, nsamples, seed, &
          rate_4ph, rate_plusplus, rate_plusminus, rate_minusminus, wp4_plusplus, wp4_plusminus, &
          wp4_minusminus) bind(c, name="fp4_rta_driver_4ph_sample")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), value :: ntri
       real(c_double), intent(in) :: psi(*)
       real(c_double), intent(in) :: r_j(*)
       real(c_double), intent(in) :: r_k(*)
       real(c_double), intent(in) :: r_l(*)
       integer(c_int32_t), intent(in) :: index_i(*)
       integer(c_int32_t), intent(in) :: index_j(*)
       integer(c_int32_t), intent(in) :: index_k(*)
       integer(c_int32_t), intent(in) :: index_l(*)
       integer(c_int64_t), value :: nsamples
       integer(c_int64_t), value :: seed
       real(c_double), intent(inout) :: rate_4ph(*)
       real(c_double), intent(inout) :: rate_plusplus(*)
       real(c_double), intent(inout) :: rate_plusminus(*)
       real(c_double), intent(inout) :: rate_minusminus(*)
       real(c_double), intent(inout) :: wp4_plusplus(*)
       real(c_double), intent(inout) :: wp4_plusminus(*)
       real(c_double), intent(inout) :: wp4_minusminus(*)
     end function fp4_rta_driver_4ph_sample

     integer(c_int) function fp4_rta_driver_4ph_sample_multi_t(ctx, g, nT, temperatures, energy, &
          velocity, eigenvect, nlist, list, ijk, ntri, psi, r_j, r_k, r_l, index_i, index_j, &
          index_k, index_l, nsamples, seed, rate_plusplus, rate_plusminus, rate_minusminus, &
          wp4_plusplus, wp4_plusminus, wp4_minusminus) &
          bind(c, name="fp4_rta_driver_4ph_sample_multi_t")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       integer(c_int32_t), value :: nT
       real(c_double), intent(in) :: temperatures(*)
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), value :: ntri
       real(c_double), intent(in) :: psi(*)
       real(c_double), intent(in) :: r_j(*)
       real(c_double), intent(in) :: r_k(*)
       real(c_double), intent(in) :: r_l(*)
       integer(c_int32_t), intent(in) :: index_i(*)
       integer(c_int32_t), intent(in) :: index_j(*)
       integer(c_int32_t), intent(in) :: index_k(*)
       integer(c_int32_t), intent(in) :: index_l(*)
       integer(c_int64_t), value :: nsamples
       integer(c_int64_t), value :: seed
       real(c_double), intent(inout) :: rate_plusplus(*)
       real(c_double), intent(inout) :: rate_plusminus(*)
       real(c_double), intent(inout) :: rate_minusminus(*)
       real(c_double), intent(inout) :: wp4_plusplus(*)
       real(c_double), intent(inout) :: wp4_plusminus(*)
       real(c_double), intent(inout) :: wp4_minusminus(*)
     end function fp4_rta_driver_4ph_sample_multi_t

     integer(c_int) function fp4_cumulative_tconduct(ctx, g, V, omega, velocity, f_n, nticks, &
          ticks, results) bind(c, name="fp4_cumulative_tconduct")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), value :: V
       real(c_double), intent(in) :: omega(*)
       real(c_double), intent(in) :: velocity(*)
       real(c_double), intent(in) :: f_n(*)
       integer(c_int32_t), value :: nticks
       real(c_double), intent(inout) :: ticks(*)
       real(c_double), intent(inout) :: results(*)
     end function fp4_cumulative_tconduct

     integer(c_int) function fp4_cumulative_tconduct_omega(ctx, g, V, omega, velocity, f_n, nticks, &
          ticks, results) bind(c, name="fp4_cumulative_tconduct_omega")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), value :: V
       real(c_double), intent(in) :: omega(*)
       real(c_double), intent(in) :: velocity(*)
       real(c_double), intent(in) :: f_n(*)
       integer(c_int32_t), value :: nticks
       real(c_double), intent(inout) :: ticks(*)
       real(c_double), intent(inout) :: results(*)
     end function fp4_cumulative_tconduct_omega

     integer(c_int) function fp4_eigen_dm(ctx, g, lattvec, cartesian, scell, fc, nonanalytic, &
          epsilon, born, V, symmetrizers, omega, velocity, eigenvect) bind(c, name="fp4_eigen_dm")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: lattvec(*)
       real(c_double), intent(in) :: cartesian(*)
       integer(c_int32_t), intent(in) :: scell(3)
       real(c_double), intent(in) :: fc(*)
       integer(c_int32_t), value :: nonanalytic
       real(c_double), intent(in) :: epsilon(*)
       real(c_double), intent(in) :: born(*)
       real(c_double), value :: V
       real(c_double), intent(in) :: symmetrizers(*)
       real(c_double), intent(inout) :: omega(*)
       real(c_double), intent(inout) :: velocity(*)
       complex(c_double_complex), intent(inout) :: eigenvect(*)
     end function fp4_eigen_dm

     integer(c_int) function fp4_np_driver_4ph_noalloc(g, energy, velocity, nlist, list, &
          n_plusplus, pspace_plusplus, n_plusminus, pspace_plusminus, n_minusminus, &
          pspace_minusminus, stream) bind(c, name="fp4_np_driver_4ph_noalloc")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(fp4_globals), intent(in) :: g
       type(c_ptr), value :: energy
       type(c_ptr), value :: velocity
       integer(c_int32_t), value :: nlist
       type(c_ptr), value :: list
       type(c_ptr), value :: n_plusplus
       type(c_ptr), value :: pspace_plusplus
       type(c_ptr), value :: n_plusminus
       type(c_ptr), value :: pspace_plusminus
       type(c_ptr), value :: n_minusminus
       type(c_ptr), value :: pspace_minusminus
       type(c_ptr), value :: stream
     end function fp4_np_driver_4ph_noalloc

     integer(c_int) function fp4_rta4_partials(ctx, ll, ii0, ii1, t, rate_pp, rate_pm, rate_mm, &
          wp_pp, wp_pm, wp_mm) bind(c, name="fp4_rta4_partials")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: ll
       integer(c_int32_t), value :: ii0
       integer(c_int32_t), value :: ii1
       integer(c_int32_t), value :: t
       real(c_double), intent(inout) :: rate_pp(*)
       real(c_double), intent(inout) :: rate_pm(*)
       real(c_double), intent(inout) :: rate_mm(*)
       real(c_double), intent(inout) :: wp_pp(*)
       real(c_double), intent(inout) :: wp_pm(*)
       real(c_double), intent(inout) :: wp_mm(*)
     end function fp4_rta4_partials

     integer(c_int) function fp4_tc_selftest(K, N, A, B, D) bind(c, name="fp4_tc_selftest")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       integer(c_int32_t), value :: K
       integer(c_int32_t), value :: N
       integer(c_int16_t), intent(in) :: A(*)
       integer(c_int16_t), intent(in) :: B(*)
       real(c_float), intent(inout) :: D(*)
     end function fp4_tc_selftest

     integer(c_int) function fp4_last_counters(ctx, counters) bind(c, name="fp4_last_counters")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(inout) :: counters(8)
     end function fp4_last_counters

     integer(c_int) function fp4_last_phase_cycles(ctx, cycles) &
          bind(c, name="fp4_last_phase_cycles")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(inout) :: cycles(8)
     end function fp4_last_phase_cycles

     integer(c_int) function fp4_set_stream(ctx, stream) bind(c, name="fp4_set_stream")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       type(c_ptr), value :: stream
     end function fp4_set_stream

     integer(c_int) function fp4_set_upload_cache(ctx, enable) bind(c, name="fp4_set_upload_cache")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: ctx
       integer(c_int), value :: enable
     end function fp4_set_upload_cache

     integer(c_int) function fp4_server_create(srv, device, precision, max_slots, max_bands, &
          hbm_budget_bytes) bind(c, name="fp4_server_create")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), intent(out) :: srv
       integer(c_int), value :: device
       integer(c_int), value :: precision
       integer(c_int32_t), value :: max_slots
       integer(c_int32_t), value :: max_bands
       integer(c_int64_t), value :: hbm_budget_bytes
     end function fp4_server_create

     integer(c_int) function fp4_server_destroy(srv) bind(c, name="fp4_server_destroy")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: srv
     end function fp4_server_destroy

     type(c_ptr) function fp4_server_last_error(srv) bind(c, name="fp4_server_last_error")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: srv
     end function fp4_server_last_error

     integer(c_int64_t) function fp4_server_footprint(nbands, nlist, ngrid, ntri3, ntri4, nsymm_rot) &
          bind(c, name="fp4_server_footprint")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       integer(c_int32_t), value :: nbands
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: ngrid(3)
       integer(c_int32_t), value :: ntri3
       integer(c_int32_t), value :: ntri4
       integer(c_int32_t), value :: nsymm_rot
     end function fp4_server_footprint

     integer(c_int) function fp4_server_admit(srv, g, energy, velocity, eigenvect, nlist, list, &
          ijk, ntri3, phi, r_j3, r_k3, index_i3, index_j3, index_k3, ntri4, psi, r_j4, r_k4, r_l4, &
          index_i4, index_j4, index_k4, index_l4, nsymm_rot, nequi, allequilist, crotations, &
          volume, slot) bind(c, name="fp4_server_admit")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: srv
       type(fp4_globals), intent(in) :: g
       real(c_double), intent(in) :: energy(*)
       real(c_double), intent(in) :: velocity(*)
       complex(c_double_complex), intent(in) :: eigenvect(*)
       integer(c_int32_t), value :: nlist
       integer(c_int32_t), intent(in) :: list(*)
       integer(c_int32_t), intent(in) :: ijk(*)
       integer(c_int32_t), value :: ntri3
       real(c_double), intent(in) :: phi(*)
       real(c_double), intent(in) :: r_j3(*)
       real(c_double), intent(in) :: r_k3(*)
       integer(c_int32_t), intent(in) :: index_i3(*)
       integer(c_int32_t), intent(in) :: index_j3(*)
       integer(c_int32_t), intent(in) :: index_k3(*)
       integer(c_int32_t), value :: ntri4
       real(c_double), intent(in) :: psi(*)
       real(c_double), intent(in) :: r_j4(*)
       real(c_double), intent(in) :: r_k4(*)
       real(c_double), intent(in) :: r_l4(*)
       integer(c_int32_t), intent(in) :: index_i4(*)
       integer(c_int32_t), intent(in) :: index_j4(*)
       integer(c_int32_t), intent(in) :: index_k4(*)
       integer(c_int32_t), intent(in) :: index_l4(*)
       integer(c_int32_t), value :: nsymm_rot
       integer(c_int32_t), intent(in) :: nequi(*)
       integer(c_int32_t), intent(in) :: allequilist(*)
       real(c_double), intent(in) :: crotations(*)
       real(c_double), value :: volume
       integer(c_int32_t), intent(out) :: slot
     end function fp4_server_admit

     integer(c_int) function fp4_server_tick(srv, max_items, finished, nfinished) &
          bind(c, name="fp4_server_tick")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: srv
       integer(c_int64_t), value :: max_items
       integer(c_int32_t), intent(inout) :: finished(*)
       integer(c_int32_t), intent(out) :: nfinished
     end function fp4_server_tick

     integer(c_int) function fp4_server_collect(srv, slot, rate3_plus, rate3_minus, rate4_pp, &
          rate4_pm, rate4_mm, kappa_branch, kappa, n_processes) bind(c, name="fp4_server_collect")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: srv
       integer(c_int32_t), value :: slot
       real(c_double), intent(inout) :: rate3_plus(*)
       real(c_double), intent(inout) :: rate3_minus(*)
       real(c_double), intent(inout) :: rate4_pp(*)
       real(c_double), intent(inout) :: rate4_pm(*)
       real(c_double), intent(inout) :: rate4_mm(*)
       real(c_double), intent(inout) :: kappa_branch(*)
       real(c_double), intent(inout) :: kappa(*)
       integer(c_int64_t), intent(out) :: n_processes
     end function fp4_server_collect

     integer(c_int) function fp4_server_status(srv, running, done, bytes_in_use, last_tick_ms, ticks) &
          bind(c, name="fp4_server_status")
       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &
            c_double_complex, fp4_globals
       type(c_ptr), value :: srv
       integer(c_int32_t), intent(out) :: running
       integer(c_int32_t), intent(out) :: done
       integer(c_int64_t), intent(out) :: bytes_in_use
       real(c_double), intent(out) :: last_tick_ms
       integer(c_int64_t), intent(out) :: ticks
     end function fp4_server_status
  end interface
end module fp4_b200
