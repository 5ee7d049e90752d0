! mdff_engine.f90 -- iso_c_binding interface to the B200 force engine
! (include/mdff_engine.h) for the Fortran host code.
!
! The derived type mdff_params_t is interoperable with struct mdff_params.
! C stores the per-type tables row-major as [i][j] (and [p][i][j]); a Fortran
! array with the same memory therefore has its indices reversed: the C entry
! for the reference's (it,jt) is params%epslj(jt,it), and for (ip,it,jt) it is
! params%ldip_damping(jt,it,ip).  mdff_fill_params in engforce_shim.f90 does
! that transposition from the reference's module variables.
!
! No Fortran compiler exists on the machine this file was written on; it
! follows the Fortran 2003 interoperability rules and the header field for
! field, and the ctypes mirror (mdff_b200/abi.py) of the same layout is checked
! against the compiled library's sizeof by the tests.
module mdff_engine
  use iso_c_binding
  implicit none

  integer, parameter :: MDFF_NTYPE_MAX = 16

  integer(c_int), parameter :: MDFF_OK = 0, MDFF_E_ARG = -1, MDFF_E_CUDA = -2, MDFF_E_NOCONV = -3, &
                               MDFF_E_LISTOVF = -4, MDFF_E_NONFINITE = -5, MDFF_E_STATE = -6, &
                               MDFF_E_UNSUPPORTED = -7, MDFF_E_NOMEM = -8
  integer(c_int), parameter :: MDFF_TRUNC_NONE = 0, MDFF_TRUNC_LINEAR = 1, MDFF_TRUNC_QUADRATIC = 2
  integer(c_int), parameter :: MDFF_POLA_SCF = 0, MDFF_POLA_PCG = 1
  integer(c_int), parameter :: MDFF_EXT_POLY = 0, MDFF_EXT_ASPC = 1
  integer(c_int), parameter :: MDFF_NVE_VV = 0, MDFF_NVT_NHCN = 1, MDFF_NPT_NHCNP = 2, MDFF_NVT_NHC2 = 3
  integer(c_int), parameter :: MDFF_PREC_FP64 = 0, MDFF_PREC_MIXED = 1

  type, bind(C) :: mdff_params_t
    integer(c_int) :: ntype
    integer(c_int) :: lnmlj, lbmhft, lbmhftd, lmorse, lcoulomb, lvnlist, lreduced, lsurf
    real(c_double) :: cutshortrange, cutlongrange, skindiff
    real(c_double) :: mass(MDFF_NTYPE_MAX)
    real(c_double) :: qch(MDFF_NTYPE_MAX)
    real(c_double) :: dip(3, MDFF_NTYPE_MAX)                 ! C dip[it][c]
    real(c_double) :: poldip_iso(MDFF_NTYPE_MAX)
    integer(c_int) :: ldip_polar(MDFF_NTYPE_MAX)
    integer(c_int) :: symmetric_pot
    integer(c_int) :: trunc
    real(c_double) :: epslj(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: sigmalj(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: plj(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: qlj(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: epsmor(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: sigmamor(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: rhomor(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: Abmhftd(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: Bbmhftd(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: Cbmhftd(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: Dbmhftd(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: BDbmhftd(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    integer(c_int) :: ldip_damping(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: dip_pol_damp_b(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: dip_pol_damp_c(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    integer(c_int) :: dip_pol_damp_k(MDFF_NTYPE_MAX, MDFF_NTYPE_MAX, MDFF_NTYPE_MAX)
    real(c_double) :: alphaES
    integer(c_int) :: kES(3)
    integer(c_int) :: lautoES
    real(c_double) :: epsw
    integer(c_int) :: doefield, doefg
    real(c_double) :: conv_tol_ind
    integer(c_int) :: min_scf_pol_iter, max_scf_pol_iter
    integer(c_int) :: algo_moment_from_pola
    integer(c_int) :: extrapolate_order
    integer(c_int) :: algo_ext_dipole
    integer(c_int) :: integrator
    real(c_double) :: dt
    real(c_double) :: temp
    integer(c_int) :: nhc_n, nhc_yosh_order, nhc_mults
    real(c_double) :: timesca_thermo
    integer(c_int) :: precision
    integer(c_int) :: efg_period
    integer(c_int) :: nlist_capacity
    integer(c_int) :: device
    integer(c_int) :: erfc_ref
    integer(c_int) :: nhc_literal
    real(c_double) :: mixed_ksplit
    integer(c_int) :: kspace_reuse
    real(c_double) :: mixed_keps
    integer(c_int) :: autotune
    integer(c_int) :: kspace_tc
    real(c_double) :: press
    real(c_double) :: timesca_baro
    real(c_double) :: fp64_keps
  end type mdff_params_t

  type, bind(C) :: mdff_energies_t
    real(c_double) :: u_lj, u_bmhft, u_morse
    real(c_double) :: u_coul
    real(c_double) :: u_dir, u_rec, u_self, u_surf, u_pol
    real(c_double) :: vir_lj, vir_bmhft, vir_morse
    real(c_double) :: pvirial_coul
    real(c_double) :: utail, ptail
    integer(c_int) :: scf_iter
    real(c_double) :: scf_rmsd
  end type mdff_energies_t

  type, bind(C) :: mdff_thermo_t
    integer(c_int) :: step
    real(c_double) :: e_kin, temp_r
    real(c_double) :: u_tot, e_tot, h_tot
    real(c_double) :: u_lj, u_bmhft, u_morse, u_coul, u_pol
    real(c_double) :: e_nvt
    real(c_double) :: pressure_tot
    real(c_double) :: pvirial_tot
    integer(c_int) :: nlist_rebuilt
    integer(c_int) :: scf_iter
    real(c_double) :: scf_rmsd
    real(c_double) :: volume
  end type mdff_thermo_t

  type, bind(C) :: mdff_opt_result_t
    real(c_double) :: u_initial, u_final, phigrad
    integer(c_int) :: iterations, nforce, status, info
  end type mdff_opt_result_t

  ! efgtag's distribution settings (src/efg.f90:171-190)
  type, bind(C) :: mdff_efg_dist_params_t
    real(c_double) :: vzzmin, resvzz, reseta, umin, resu, smax
  end type mdff_efg_dist_params_t

  ! frame header of the on-disk formats: natm, simu_cell%A (column-major),
  ! system, atypei, natmi (the config module's values)
  type, bind(C) :: mdff_frame_header_t
    integer(c_int) :: natm, ntype
    real(c_double) :: a(9)
    character(kind=c_char) :: system(60)
    character(kind=c_char) :: atypei(3, MDFF_NTYPE_MAX)
    integer(c_int) :: natmi(MDFF_NTYPE_MAX)
  end type mdff_frame_header_t

  ! rmctag (src/rmc.f90:36-50) and the chain's report
  type, bind(C) :: mdff_rmc_params_t
    real(c_double) :: max_displacement, resolution_gr, cut_rmc
    real(c_double) :: temp_rmc(6)
    integer(c_long_long) :: acceptance_max, max_trials
  end type mdff_rmc_params_t
  type, bind(C) :: mdff_rmc_result_t
    integer(c_long_long) :: kall, kacc, uniforms_used
    real(c_double) :: chisq(6)
    integer(c_int) :: status, pad
  end type mdff_rmc_result_t
  ! rmctag's EFG terms (src/rmc.f90:40-60)
  type, bind(C) :: mdff_rmc_efg_params_t
    integer(c_int) :: lrmc_u, lrmc_vzz, lrmc_eta, efg_start
    real(c_double) :: resolution_u_efg, u_efg_min, resolution_vzz_efg, vzz_efg_min, resolution_eta_efg
    integer(c_int) :: lrmc_var, pad_
  end type mdff_rmc_efg_params_t

  integer(c_int), parameter :: MDFF_FILE_TRAJFF = 0, MDFF_FILE_CONTFF = 1, MDFF_FILE_EFGALL = 2, &
                               MDFF_FILE_DIPFF = 3, MDFF_FILE_EFALL = 4, MDFF_DATA_V = 1, MDFF_DATA_F = 2

  interface
    subroutine mdff_params_default(p) bind(C, name="mdff_params_default")
      import :: mdff_params_t
      type(mdff_params_t), intent(out) :: p
    end subroutine

    integer(c_int) function mdff_create(p, ctx) bind(C, name="mdff_create")
      import :: c_int, c_ptr, mdff_params_t
      type(mdff_params_t), intent(in) :: p
      type(c_ptr), intent(out) :: ctx
    end function

    subroutine mdff_destroy(ctx) bind(C, name="mdff_destroy")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end subroutine

    type(c_ptr) function mdff_last_error(ctx) bind(C, name="mdff_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function

    integer(c_int) function mdff_set_system(ctx, natm, itype, rx, ry, rz, A) bind(C, name="mdff_set_system")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: natm
      integer(c_int), intent(in) :: itype(*)
      real(c_double), intent(in) :: rx(*), ry(*), rz(*), A(9)
    end function

    integer(c_int) function mdff_set_positions(ctx, rx, ry, rz) bind(C, name="mdff_set_positions")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: rx(*), ry(*), rz(*)
    end function

    integer(c_int) function mdff_get_positions(ctx, rx, ry, rz) bind(C, name="mdff_get_positions")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: rx(*), ry(*), rz(*)
    end function

    integer(c_int) function mdff_engforce(ctx, fx, fy, fz, e, tau_nonb, tau_coul, ef, efg, mu) &
        bind(C, name="mdff_engforce")
      import :: c_int, c_double, c_ptr, mdff_energies_t
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: fx(*), fy(*), fz(*)
      type(mdff_energies_t), intent(out) :: e
      real(c_double), intent(out) :: tau_nonb(9), tau_coul(9)
      real(c_double), intent(out) :: ef(*), efg(*), mu(*)
    end function

    integer(c_int) function mdff_opt_sastry(ctx, itmax, res) bind(C, name="mdff_opt_sastry")
      import :: c_int, c_ptr, mdff_opt_result_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: itmax
      type(mdff_opt_result_t), intent(out) :: res
    end function

    ! optalgo = 'm1qn3' of opt_main: niter = nsim = 6000, epsg = epsrel_m1qn3
    integer(c_int) function mdff_opt_m1qn3(ctx, niter, nsim, epsg, res) bind(C, name="mdff_opt_m1qn3")
      import :: c_int, c_double, c_ptr, mdff_opt_result_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: niter, nsim
      real(c_double), value :: epsg
      type(mdff_opt_result_t), intent(out) :: res
    end function

    ! optalgo = 'lbfgs' of opt_main: eps = epsrel_lbfgs
    integer(c_int) function mdff_opt_lbfgs(ctx, itmax, eps, res) bind(C, name="mdff_opt_lbfgs")
      import :: c_int, c_double, c_ptr, mdff_opt_result_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: itmax
      real(c_double), value :: eps
      type(mdff_opt_result_t), intent(out) :: res
    end function

    ! efg_stat on the device over nconf configurations: efg6 = c_loc(efg(1,1,1))
    ! of efg(natm,6,nconf), or c_null_ptr with nconf = 1 for the context's own
    ! tensors; nmr(natm,4,nconf), u(natm,5,nconf), s(natm,nconf)
    integer(c_int) function mdff_efg_nmr(ctx, nconf, efg6, nmr, u, s) bind(C, name="mdff_efg_nmr")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, efg6
      integer(c_int), value :: nconf
      real(c_double), intent(out) :: nmr(*), u(*), s(*)
    end function

    ! stats(8,0:ntype,nconf), mu(5,0:ntype), m2u(5,5,0:ntype), dibvzz(0:PANvzz,0:ntype),
    ! dibeta(0:PANeta,0:ntype), dibu(0:PANU,0:ntype,6), dibs(0:PANS,0:ntype)
    integer(c_int) function mdff_efg_dist(ctx, nconf, efg6, dp, stats, mu, m2u, dibvzz, dibeta, dibu, dibs) &
        bind(C, name="mdff_efg_dist")
      import :: c_int, c_ptr, c_double, mdff_efg_dist_params_t
      type(c_ptr), value :: ctx, efg6
      integer(c_int), value :: nconf
      type(mdff_efg_dist_params_t), intent(in) :: dp
      real(c_double), intent(out) :: stats(*), mu(*), m2u(*)
      integer(c_int), intent(out) :: dibvzz(*), dibeta(*), dibu(*), dibs(*)
    end function

    integer(c_int) function mdff_nlist_build(ctx) bind(C, name="mdff_nlist_build")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    integer(c_int) function mdff_nlist_get(ctx, which, point, list, cap, nlist) bind(C, name="mdff_nlist_get")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: which, cap
      integer(c_int), intent(out) :: point(*), list(*)
      integer(c_int), intent(out) :: nlist
    end function

    integer(c_int) function mdff_md_start(ctx, vx, vy, vz, t0) bind(C, name="mdff_md_start")
      import :: c_int, c_double, c_ptr, mdff_thermo_t
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: vx(*), vy(*), vz(*)
      type(mdff_thermo_t), intent(out) :: t0
    end function

    integer(c_int) function mdff_step(ctx, nsteps, rx, ry, rz, vx, vy, vz, fx, fy, fz, thermo) &
        bind(C, name="mdff_step")
      import :: c_int, c_double, c_ptr, mdff_thermo_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
      real(c_double), intent(inout) :: rx(*), ry(*), rz(*), vx(*), vy(*), vz(*)
      real(c_double), intent(out) :: fx(*), fy(*), fz(*)
      type(mdff_thermo_t), intent(out) :: thermo(*)
    end function
    ! a new cell (column-major) for the same atoms: lattice, tail corrections, k tables
    integer(c_int) function mdff_set_cell(ctx, a) bind(C, name="mdff_set_cell")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: a(9)
    end function

    ! g(r) as rmc_gr forms it: grr(0:nbins-1, 0:npairs); grr may be c_null_ptr to get nbins
    integer(c_int) function mdff_gr(ctx, cut, res, grr, nbins) bind(C, name="mdff_gr")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, grr
      real(c_double), value :: cut, res
      integer(c_int), intent(out) :: nbins
    end function

    ! rmc_main on the g(r) chi^2; uniforms = c_loc of the host's stream or c_null_ptr (engine stream from seed)
    integer(c_int) function mdff_rmc(ctx, rp, grr_exp, uniforms, nuni, seed, grr_out, res) bind(C, name="mdff_rmc")
      import :: c_int, c_ptr, c_double, c_long_long, mdff_rmc_params_t, mdff_rmc_result_t
      type(c_ptr), value :: ctx, uniforms, grr_out
      type(mdff_rmc_params_t), intent(in) :: rp
      real(c_double), intent(in) :: grr_exp(*)
      integer(c_long_long), value :: nuni, seed
      type(mdff_rmc_result_t), intent(out) :: res
    end function

    ! rmc_main with its EFG terms: dibU_exp(6, 0:ntype, 0:PANU), dibvzz_exp(0:ntype, 0:PANvzz),
    ! dibeta_exp(0:ntype, 0:PANeta) as rmc_main allocates them (c_null_ptr for an inactive term)
    integer(c_int) function mdff_rmc_efg(ctx, rp, ep, grr_exp, dibU_exp, dibvzz_exp, dibeta_exp, uniforms, nuni, &
                                         seed, grr_out, dibU_out, dibvzz_out, dibeta_out, res) &
        bind(C, name="mdff_rmc_efg")
      import :: c_int, c_ptr, c_double, c_long_long, mdff_rmc_params_t, mdff_rmc_efg_params_t, mdff_rmc_result_t
      type(c_ptr), value :: ctx, dibU_exp, dibvzz_exp, dibeta_exp, uniforms, grr_out, dibU_out, dibvzz_out, dibeta_out
      type(mdff_rmc_params_t), intent(in) :: rp
      type(mdff_rmc_efg_params_t), intent(in) :: ep
      real(c_double), intent(in) :: grr_exp(*)
      integer(c_long_long), value :: nuni, seed
      type(mdff_rmc_result_t), intent(out) :: res
    end function

    ! streaming writer: frames of the context's state, written in the background
    integer(c_int) function mdff_writer_open(ctx, path, file, iformat, data, h, nslot, w) &
        bind(C, name="mdff_writer_open")
      import :: c_int, c_ptr, c_char, mdff_frame_header_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)     ! NUL terminated
      integer(c_int), value :: file, iformat, data, nslot
      type(mdff_frame_header_t), intent(in) :: h
      type(c_ptr), intent(out) :: w
    end function

    integer(c_int) function mdff_writer_frame(w) bind(C, name="mdff_writer_frame")
      import :: c_int, c_ptr
      type(c_ptr), value :: w
    end function

    integer(c_int) function mdff_writer_close(w) bind(C, name="mdff_writer_close")
      import :: c_int, c_ptr
      type(c_ptr), value :: w
    end function

    ! whole-state checkpoint into / from a caller's buffer (buf = c_null_ptr to query len)
    integer(c_int) function mdff_checkpoint_save(ctx, buf, cap, len) bind(C, name="mdff_checkpoint_save")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx, buf
      integer(c_size_t), value :: cap
      integer(c_size_t), intent(out) :: len
    end function

    integer(c_int) function mdff_checkpoint_load(ctx, buf, len) bind(C, name="mdff_checkpoint_load")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx, buf
      integer(c_size_t), value :: len
    end function
  end interface

contains

  ! Message of the last error as a Fortran string.
  function mdff_error_string(ctx) result(msg)
    type(c_ptr), intent(in) :: ctx
    character(len=256) :: msg
    character(kind=c_char), pointer :: p(:)
    integer :: k
    msg = ' '
    call c_f_pointer(mdff_last_error(ctx), p, [256])
    do k = 1, 256
      if (p(k) == c_null_char) exit
      msg(k:k) = p(k)
    enddo
  end function mdff_error_string

end module mdff_engine
