! pf3d_bind.f90 -- ISO_C_BINDING interface of libpf3d (include/pf3d.h) for
! the reference's Fortran time loop (ileaof/phase-field-project-3D,
! source/principal.f90:93-226).  A maintainer adds this file to the
! reference's source/ and replaces the bodies of the hot subroutines
! (temperatura, equacao_campo_fase, concentracao_soluto, auxiliar,
! diagnosticos) with calls through it.  The derived types mirror the C
! structs field by field, in the same order and with the same C types.
! No Fortran compiler exists in the build image: this file is not compiled
! here; the same entry points are exercised through ctypes.
module pf3d_bind
  use iso_c_binding
  implicit none
  integer(c_int), parameter :: PF_FP64 = 64, PF_FP32 = 32
  integer(c_int), parameter :: PF_PHASE_OLD = 0, PF_PHASE_NEW = 1, PF_CONC_OLD = 2, &
                               PF_CONC_NEW = 3, PF_TOLD = 4, PF_TNEW = 5, PF_DPP = 6
  type, bind(C) :: pf_grid
     integer(c_int) :: nx, ny, nz
     real(c_double) :: dx, dy, dz
  end type
  type, bind(C) :: pf_params            ! field order of include/pf3d.h
     real(c_double) :: Tm, T0, delta_H, M0, Cp_s, D, AAA, DELTA_EPSLON, D_sol, D_liq
     real(c_float)  :: Ke
     real(c_double) :: Me, Vm, R, C0, Thin_Interface
     real(c_float)  :: Sigma, Beta, ajuste
     real(c_double) :: TP, taxa_resfr
     integer(c_int) :: n_varreduras, h_quintico, ruido_tipo, bc
     real(c_double) :: stoptime
     integer(c_int) :: WriteFileD_timeCounter
  end type
  type(c_ptr), save :: pf_ctx = c_null_ptr
  interface
     integer(c_int) function pf_create(g, p, prec, ctx) bind(C, name="pf_create")
       import; type(pf_grid), intent(in) :: g; type(pf_params), intent(in) :: p
       integer(c_int), value :: prec; type(c_ptr), intent(out) :: ctx
     end function
     integer(c_int) function pf_upload(ctx, f, host) bind(C, name="pf_upload")
       import; type(c_ptr), value :: ctx; integer(c_int), value :: f; type(c_ptr), value :: host
     end function
     integer(c_int) function pf_download(ctx, f, host) bind(C, name="pf_download")
       import; type(c_ptr), value :: ctx; integer(c_int), value :: f; type(c_ptr), value :: host
     end function
     integer(c_int) function pf_temperatura(ctx, TP) bind(C, name="pf_temperatura")
       import; type(c_ptr), value :: ctx; real(c_double), value :: TP
     end function
     integer(c_int) function pf_equacao_campo_fase(ctx, it, TP, M0, Cs_eq, Cl_eq) &
          bind(C, name="pf_equacao_campo_fase")
       import; type(c_ptr), value :: ctx; integer(c_int), value :: it
       real(c_double), value :: TP, M0; real(c_double), intent(out) :: Cs_eq, Cl_eq
     end function
     integer(c_int) function pf_copy_phase_new_to_old(ctx) bind(C, name="pf_copy_phase_new_to_old")
       import; type(c_ptr), value :: ctx
     end function
     integer(c_int) function pf_concentracao_soluto(ctx) bind(C, name="pf_concentracao_soluto")
       import; type(c_ptr), value :: ctx
     end function
     integer(c_int) function pf_auxiliar(ctx, TP, Cs_eq, Cl_eq, M0) bind(C, name="pf_auxiliar")
       import; type(c_ptr), value :: ctx; real(c_double), value :: TP, Cs_eq, Cl_eq
       real(c_double), intent(out) :: M0
     end function
     integer(c_int) function pf_diagnosticos(ctx, out) bind(C, name="pf_diagnosticos")
       import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: out(5)
     end function
     integer(c_int) function pf_swap(ctx) bind(C, name="pf_swap")
       import; type(c_ptr), value :: ctx
     end function
     integer(c_int) function pf_probe(ctx, f, i, j, k, v) bind(C, name="pf_probe")
       import; type(c_ptr), value :: ctx; integer(c_int), value :: f, i, j, k
       real(c_double), intent(out) :: v
     end function
  end interface
contains
  subroutine pf_check(rc)
    integer(c_int), intent(in) :: rc
    if (rc /= 0) error stop 'pf3d call failed (see pf_last_error)'
  end subroutine
end module pf3d_bind
