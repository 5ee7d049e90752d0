"""ctypes mirror of include/mdff_engine.h.

The structures below must match the C declarations field for field; a CPU
test compares ``ctypes.sizeof`` and the defaults against the compiled
library.  Field meanings follow the reference's namelist tags
(src/control.f90:128-160, src/field.f90:450-500, src/md.f90:109-132).
"""
import ctypes as C
import numpy as np

NTYPE_MAX = 16
TT_MAX_ORDER = 8

OK = 0
E_ARG = -1
E_CUDA = -2
E_NOCONV = -3
E_LISTOVF = -4
E_NONFINITE = -5
E_STATE = -6
E_UNSUPPORTED = -7
E_NOMEM = -8

TRUNC_NONE, TRUNC_LINEAR, TRUNC_QUADRATIC = 0, 1, 2
POLA_SCF, POLA_PCG = 0, 1
EXT_POLY, EXT_ASPC = 0, 1
NVE_VV, NVT_NHCN, NPT_NHCNP, NVT_NHC2 = 0, 1, 2, 3
PREC_FP64, PREC_MIXED = 0, 1

_T = NTYPE_MAX
_D1 = C.c_double * _T
_D2 = (C.c_double * _T) * _T
_I1 = C.c_int * _T
_D3 = ((C.c_double * _T) * _T) * _T
_I3 = ((C.c_int * _T) * _T) * _T


class Params(C.Structure):
    _fields_ = [
        ("ntype", C.c_int),
        ("lnmlj", C.c_int), ("lbmhft", C.c_int), ("lbmhftd", C.c_int), ("lmorse", C.c_int),
        ("lcoulomb", C.c_int), ("lvnlist", C.c_int), ("lreduced", C.c_int), ("lsurf", C.c_int),
        ("cutshortrange", C.c_double), ("cutlongrange", C.c_double), ("skindiff", C.c_double),
        ("mass", _D1), ("qch", _D1), ("dip", (C.c_double * 3) * _T), ("poldip_iso", _D1),
        ("ldip_polar", _I1), ("symmetric_pot", C.c_int), ("trunc", C.c_int),
        ("epslj", _D2), ("sigmalj", _D2), ("plj", _D2), ("qlj", _D2),
        ("epsmor", _D2), ("sigmamor", _D2), ("rhomor", _D2),
        ("Abmhftd", _D2), ("Bbmhftd", _D2), ("Cbmhftd", _D2), ("Dbmhftd", _D2), ("BDbmhftd", _D2),
        ("ldip_damping", _I3), ("dip_pol_damp_b", _D3), ("dip_pol_damp_c", _D3), ("dip_pol_damp_k", _I3),
        ("alphaES", C.c_double), ("kES", C.c_int * 3), ("lautoES", C.c_int), ("epsw", C.c_double),
        ("doefield", C.c_int), ("doefg", C.c_int),
        ("conv_tol_ind", C.c_double), ("min_scf_pol_iter", C.c_int), ("max_scf_pol_iter", C.c_int),
        ("algo_moment_from_pola", C.c_int), ("extrapolate_order", C.c_int), ("algo_ext_dipole", C.c_int),
        ("integrator", C.c_int), ("dt", C.c_double), ("temp", C.c_double),
        ("nhc_n", C.c_int), ("nhc_yosh_order", C.c_int), ("nhc_mults", C.c_int),
        ("timesca_thermo", C.c_double),
        ("precision", C.c_int), ("efg_period", C.c_int), ("nlist_capacity", C.c_int), ("device", C.c_int),
        ("erfc_ref", C.c_int), ("nhc_literal", C.c_int), ("mixed_ksplit", C.c_double),
        ("kspace_reuse", C.c_int), ("mixed_keps", C.c_double), ("autotune", C.c_int),
        ("kspace_tc", C.c_int),
        ("press", C.c_double), ("timesca_baro", C.c_double),
        ("fp64_keps", C.c_double),
    ]


class Energies(C.Structure):
    _fields_ = [
        ("u_lj", C.c_double), ("u_bmhft", C.c_double), ("u_morse", C.c_double),
        ("u_coul", C.c_double),
        ("u_dir", C.c_double), ("u_rec", C.c_double), ("u_self", C.c_double), ("u_surf", C.c_double),
        ("u_pol", C.c_double),
        ("vir_lj", C.c_double), ("vir_bmhft", C.c_double), ("vir_morse", C.c_double),
        ("pvirial_coul", C.c_double),
        ("utail", C.c_double), ("ptail", C.c_double),
        ("scf_iter", C.c_int), ("scf_rmsd", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Thermo(C.Structure):
    _fields_ = [
        ("step", C.c_int),
        ("e_kin", C.c_double), ("temp_r", C.c_double),
        ("u_tot", C.c_double), ("e_tot", C.c_double), ("h_tot", C.c_double),
        ("u_lj", C.c_double), ("u_bmhft", C.c_double), ("u_morse", C.c_double),
        ("u_coul", C.c_double), ("u_pol", C.c_double),
        ("e_nvt", C.c_double), ("pressure_tot", C.c_double), ("pvirial_tot", C.c_double),
        ("nlist_rebuilt", C.c_int), ("scf_iter", C.c_int), ("scf_rmsd", C.c_double),
        ("volume", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# epsrel_lbfgs and epsrel_m1qn3 default to 1.0e-5 (src/opt.f90:139-140), a
# default-real literal: its double value is that of the single-precision 1e-5
EPSREL_OPT = float(np.float32(1.0e-5))


class OptResult(C.Structure):
    """mdff_opt_result: one structure optimisation (opt_main's report)."""
    _fields_ = [("u_initial", C.c_double), ("u_final", C.c_double), ("phigrad", C.c_double),
                ("iterations", C.c_int), ("nforce", C.c_int), ("status", C.c_int), ("info", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


FILE_TRAJFF, FILE_CONTFF, FILE_EFGALL, FILE_DIPFF, FILE_EFALL = 0, 1, 2, 3, 4
DATA_V, DATA_F = 1, 2
TRAJ_DATA = {"rnn": 0, "rvn": DATA_V, "rnf": DATA_F, "rvf": DATA_V | DATA_F}


class FrameHeader(C.Structure):
    """mdff_frame_header: natm, system, simu_cell%A (column-major), ntype,
    atypei, natmi of one frame."""
    _fields_ = [("natm", C.c_int), ("ntype", C.c_int), ("A", C.c_double * 9), ("system", C.c_char * 60),
                ("atypei", (C.c_char * 3) * NTYPE_MAX), ("natmi", C.c_int * NTYPE_MAX)]


class RmcParams(C.Structure):
    """mdff_rmc_params: rmctag's max_displacement, resolution_gr, cut_rmc,
    temp_rmc (five components and the total), acceptance_max, and a bound on
    the trial moves."""
    _fields_ = [("max_displacement", C.c_double), ("resolution_gr", C.c_double), ("cut_rmc", C.c_double),
                ("temp_rmc", C.c_double * 6), ("acceptance_max", C.c_longlong), ("max_trials", C.c_longlong)]


class RmcEfgParams(C.Structure):
    """mdff_rmc_efg_params: rmctag's EFG terms (lrmc_u, lrmc_vzz, lrmc_eta),
    efg_start and the bins of rmc_efg, and the distance-variance term
    (lrmc_var)."""
    _fields_ = [("lrmc_u", C.c_int), ("lrmc_vzz", C.c_int), ("lrmc_eta", C.c_int), ("efg_start", C.c_int),
                ("resolution_u_efg", C.c_double), ("u_efg_min", C.c_double),
                ("resolution_vzz_efg", C.c_double), ("vzz_efg_min", C.c_double),
                ("resolution_eta_efg", C.c_double), ("lrmc_var", C.c_int), ("pad_", C.c_int)]

    def shapes(self, ntype):
        """Array shapes of the U, Vzz and eta distributions: the reference's
        Fortran layouts dibU(6, 0:ntype, 0:PANU), dib(0:ntype, 0:PAN) read in C
        order, so index [bin, mp, ui - 1] and [bin, mp]."""
        panu = int(2.0 * abs(self.u_efg_min) / self.resolution_u_efg)
        panv = int(2.0 * abs(self.vzz_efg_min) / self.resolution_vzz_efg)
        pane = int(1.0 / self.resolution_eta_efg)
        return (panu + 1, ntype + 1, 6), (panv + 1, ntype + 1), (pane + 1, ntype + 1)


class RmcResult(C.Structure):
    _fields_ = [("kall", C.c_longlong), ("kacc", C.c_longlong), ("uniforms_used", C.c_longlong),
                ("chisq", C.c_double * 6), ("status", C.c_int), ("pad", C.c_int)]

    def as_dict(self):
        return {"kall": self.kall, "kacc": self.kacc, "uniforms_used": self.uniforms_used,
                "chisq": list(self.chisq), "status": self.status}


class EfgDistParams(C.Structure):
    """mdff_efg_dist_params: efg_stat's distribution settings (efgtag:
    vzzmin, resvzz, reseta, umin, resu, smax; src/efg.f90:171-190)."""
    _fields_ = [("vzzmin", C.c_double), ("resvzz", C.c_double), ("reseta", C.c_double),
                ("umin", C.c_double), ("resu", C.c_double), ("smax", C.c_double)]

    def bins(self):
        """(PANvzz, PANeta, PANU, PANS) as efg_check_tag sets them (src/efg.f90:233-236);
        zeros where a resolution is not positive (the engine rejects those)."""
        if not (self.resvzz > 0 and self.reseta > 0 and self.resu > 0):
            return (0, 0, 0, 0)
        return (int((2.0 * abs(self.vzzmin)) / self.resvzz), int(1.0 / self.reseta),
                int((2.0 * abs(self.umin)) / self.resu), int(self.smax / self.resu))


class ParamGrad(C.Structure):
    """mdff_param_grad: derivative of a loss with respect to the force-field
    tables, unordered pairs in the upper-triangle slot [a][b], a <= b."""
    _fields_ = [
        ("Abmhftd", _D2), ("Bbmhftd", _D2), ("Cbmhftd", _D2), ("Dbmhftd", _D2), ("BDbmhftd", _D2),
        ("epsmor", _D2), ("sigmamor", _D2), ("rhomor", _D2),
        ("poldip_iso", _D1),
        ("dip_pol_damp_b", _D3), ("dip_pol_damp_c", _D3),
    ]

    def array(self, name):
        import numpy as np
        return np.ctypeslib.as_array(getattr(self, name)).copy()


def default_params():
    """Reference defaults: control_default_tag (src/control.f90:199-243),
    field_default_tag (src/field.f90:192-273), md_default_tag
    (src/md.f90:178-205).  Mirrors mdff_params_default() in the library."""
    p = Params()
    p.ntype = 1
    p.lvnlist = 1
    p.skindiff = 0.15
    p.symmetric_pot = 1
    p.trunc = TRUNC_NONE
    for i in range(_T):
        p.mass[i] = 1.0
        for j in range(_T):
            p.qlj[i][j] = 12.0
            p.plj[i][j] = 6.0
    p.alphaES = 1.0
    p.kES[0] = p.kES[1] = p.kES[2] = 10
    p.epsw = 1e-6
    p.conv_tol_ind = 1e-6
    p.min_scf_pol_iter = 3
    p.max_scf_pol_iter = 100
    p.extrapolate_order = 0
    p.algo_ext_dipole = EXT_POLY
    p.algo_moment_from_pola = POLA_SCF
    p.integrator = NVE_VV
    p.temp = 1.0
    p.nhc_n = 4
    p.nhc_yosh_order = 3
    p.nhc_mults = 2
    p.timesca_thermo = 1.0
    p.precision = PREC_FP64
    p.efg_period = 0
    p.nlist_capacity = 0
    p.device = 0
    p.mixed_ksplit = 2.5
    p.mixed_keps = 1e-7
    p.kspace_tc = 2
    p.press = 0.0
    p.timesca_baro = 1.0
    return p
