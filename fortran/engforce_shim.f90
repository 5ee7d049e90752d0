! engforce_shim.f90 -- drop-in body for the reference's engforce_driver
! (src/field.f90:1111-1166) and md_run's integrator call
! (src/runmd.f90:268-277) on top of the B200 engine.
!
! Build: compile mdff_engine.f90 and this file with the reference's modules
! and link libmdff_engine.so.  The reference's own
! engforce_driver is renamed (or its body replaced by CALL engforce_b200);
! every other caller keeps calling engforce_driver.
!
! State crossing the boundary on each call: positions in (rx,ry,rz); forces,
! stresses, energies, field, field gradient and total dipoles out.  The
! engine context persists between calls (device buffers, Verlet lists,
! dipole history for the extrapolation).
module engforce_b200_mod
  use iso_c_binding
  use mdff_engine
  implicit none
  type(c_ptr), save :: b200_ctx = c_null_ptr
  logical, save :: b200_ready = .false.
contains

  ! Fill mdff_params_t from the reference's module variables (&controltag,
  ! &fieldtag, &mdtag), transposing the per-type tables to the C layout.
  subroutine mdff_fill_params(prm)
    use control, only : lnmlj, lbmhft, lbmhftd, lmorse, lcoulomb, lvnlist, lreduced, lsurf, &
                        cutshortrange, cutlongrange, skindiff
    use field, only : mass, qch, dip, poldip_iso, ldip_polar, symmetric_pot, trunc, epslj, sigmalj, plj, qlj, &
                      epsmor, sigmamor, rhomor, Abmhftd, Bbmhftd, Cbmhftd, Dbmhftd, BDbmhftd, ldip_damping, &
                      dip_pol_damp_b, dip_pol_damp_c, dip_pol_damp_k, alphaES, kES, lautoES, epsw, doefield, &
                      doefg, conv_tol_ind, min_scf_pol_iter, max_scf_pol_iter, extrapolate_order, &
                      algo_ext_dipole, algo_moment_from_pola
    use config, only : ntype
    use md, only : integrator, dt, temp, nhc_n, nhc_yosh_order, nhc_mults, timesca_thermo, press, timesca_baro
    use constants, only : time_unit, boltz_unit, press_unit
    type(mdff_params_t), intent(out) :: prm
    integer :: it, jt, ip
    call mdff_params_default(prm)
    prm%ntype = ntype
    prm%lnmlj = merge(1, 0, lnmlj); prm%lbmhft = merge(1, 0, lbmhft); prm%lbmhftd = merge(1, 0, lbmhftd)
    prm%lmorse = merge(1, 0, lmorse); prm%lcoulomb = merge(1, 0, lcoulomb); prm%lvnlist = merge(1, 0, lvnlist)
    prm%lreduced = merge(1, 0, lreduced); prm%lsurf = merge(1, 0, lsurf)
    prm%cutshortrange = cutshortrange; prm%cutlongrange = cutlongrange; prm%skindiff = skindiff
    prm%symmetric_pot = merge(1, 0, symmetric_pot)
    prm%trunc = trunc
    do it = 1, ntype
      prm%mass(it) = mass(it)
      prm%qch(it) = qch(it)
      prm%dip(:, it) = dip(it, :)
      prm%poldip_iso(it) = poldip_iso(it)
      prm%ldip_polar(it) = merge(1, 0, ldip_polar(it))
      do jt = 1, ntype
        prm%epslj(jt, it) = epslj(it, jt);       prm%sigmalj(jt, it) = sigmalj(it, jt)
        prm%plj(jt, it) = plj(it, jt);           prm%qlj(jt, it) = qlj(it, jt)
        prm%epsmor(jt, it) = epsmor(it, jt);     prm%sigmamor(jt, it) = sigmamor(it, jt)
        prm%rhomor(jt, it) = rhomor(it, jt)
        prm%Abmhftd(jt, it) = Abmhftd(it, jt);   prm%Bbmhftd(jt, it) = Bbmhftd(it, jt)
        prm%Cbmhftd(jt, it) = Cbmhftd(it, jt);   prm%Dbmhftd(jt, it) = Dbmhftd(it, jt)
        prm%BDbmhftd(jt, it) = BDbmhftd(it, jt)
        do ip = 1, ntype
          prm%ldip_damping(jt, it, ip) = merge(1, 0, ldip_damping(ip, it, jt))
          prm%dip_pol_damp_b(jt, it, ip) = dip_pol_damp_b(ip, it, jt)
          prm%dip_pol_damp_c(jt, it, ip) = dip_pol_damp_c(ip, it, jt)
          prm%dip_pol_damp_k(jt, it, ip) = dip_pol_damp_k(ip, it, jt)
        enddo
      enddo
    enddo
    prm%alphaES = alphaES
    prm%kES = kES
    prm%lautoES = merge(1, 0, lautoES)
    prm%epsw = epsw
    prm%doefield = merge(1, 0, doefield)
    prm%doefg = merge(1, 0, doefg)
    prm%conv_tol_ind = conv_tol_ind
    prm%min_scf_pol_iter = min_scf_pol_iter
    prm%max_scf_pol_iter = max_scf_pol_iter
    prm%extrapolate_order = extrapolate_order
    prm%algo_ext_dipole = merge(MDFF_EXT_ASPC, MDFF_EXT_POLY, algo_ext_dipole == 'aspc')
    prm%algo_moment_from_pola = merge(MDFF_POLA_PCG, MDFF_POLA_SCF, algo_moment_from_pola == 'cng')
    prm%integrator = MDFF_NVE_VV
    if (integrator == 'nvt-nhcn') prm%integrator = MDFF_NVT_NHCN
    if (integrator == 'nvt-nhc2') prm%integrator = MDFF_NVT_NHC2
    if (integrator == 'npt-nhcnp') prm%integrator = MDFF_NPT_NHCNP
    ! md_init has already converted dt, temp and timesca_thermo to internal
    ! units (src/md.f90:314-324); the engine takes control-file units
    prm%dt = dt / time_unit
    prm%temp = temp / boltz_unit
    prm%timesca_thermo = timesca_thermo / time_unit
    prm%press = press / press_unit
    prm%timesca_baro = timesca_baro / time_unit
    prm%nhc_n = nhc_n; prm%nhc_yosh_order = nhc_yosh_order; prm%nhc_mults = nhc_mults
  end subroutine mdff_fill_params

  ! Replacement body of engforce_driver.
  subroutine engforce_b200
    use config, only : natm, itype, rx, ry, rz, fx, fy, fz, simu_cell, tau_nonb, tau_coul
    use thermodynamic, only : u_lj, u_bmhft, u_morse, u_coul, u_pol, vir_lj, vir_bmhft, vir_morse, pvirial_coul
    use field, only : ef_t, efg_t, mu_t
    use constants, only : coul_unit
    type(mdff_params_t) :: prm
    type(mdff_energies_t) :: e
    real(c_double) :: A(9), tn(9), tc(9)
    real(c_double), allocatable :: ef(:), efg(:), mu(:)
    integer(c_int) :: rc
    integer :: c
    if (.not. b200_ready) then
      call mdff_fill_params(prm)
      rc = mdff_create(prm, b200_ctx)
      if (rc /= MDFF_OK) stop 'mdff_create failed'
      A = reshape(simu_cell%A, [9])
      rc = mdff_set_system(b200_ctx, int(natm, c_int), itype, rx, ry, rz, A)
      if (rc /= MDFF_OK) stop 'mdff_set_system failed'
      b200_ready = .true.
    else
      rc = mdff_set_positions(b200_ctx, rx, ry, rz)
    endif
    allocate (ef(3 * natm), efg(6 * natm), mu(3 * natm))
    rc = mdff_engforce(b200_ctx, fx, fy, fz, e, tn, tc, ef, efg, mu)
    if (rc /= MDFF_OK) then
      write (*, '(a)') trim(mdff_error_string(b200_ctx))
      stop 'mdff_engforce failed'
    endif
    tau_nonb = reshape(tn, [3, 3])
    tau_coul = reshape(tc, [3, 3])
    u_lj = e%u_lj; u_bmhft = e%u_bmhft; u_morse = e%u_morse; u_coul = e%u_coul
    u_pol = e%u_pol / coul_unit
    vir_lj = e%vir_lj; vir_bmhft = e%vir_bmhft; vir_morse = e%vir_morse
    pvirial_coul = e%pvirial_coul
    do c = 1, 3
      ef_t(:, c) = ef((c - 1) * natm + 1 : c * natm)
      mu_t(:, c) = mu((c - 1) * natm + 1 : c * natm)
    enddo
    ! efg components xx yy zz xy xz yz (the ones the reference reduces, field.f90:2619-2624)
    efg_t(:, 1, 1) = efg(1:natm);              efg_t(:, 2, 2) = efg(natm + 1:2 * natm)
    efg_t(:, 3, 3) = efg(2 * natm + 1:3 * natm); efg_t(:, 1, 2) = efg(3 * natm + 1:4 * natm)
    efg_t(:, 1, 3) = efg(4 * natm + 1:5 * natm); efg_t(:, 2, 3) = efg(5 * natm + 1:6 * natm)
    deallocate (ef, efg, mu)
  end subroutine engforce_b200

end module engforce_b200_mod
