// mdff_oracle.cpp -- CPU FP64 restatement of MDFF's force-and-integration path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// engine in mdff_b200/csrc.  Only the tests, the smoke check and the CPU
// baseline leg of bench.py load it; the engine never links, calls or falls
// back to it.
//
// Every routine follows one reference routine (jamruam/mdff, Fortran 90) and
// cites it by file:line.  Arithmetic is FP64 evaluated left to right with no
// FMA contraction (built with -ffp-contract=off), which is the operation order
// the reference source spells out; the Verlet-list inclusion test therefore
// reproduces the reference's decisions bit for bit.
//
// Deliberate deviations from the reference (each a defect of the reference or
// an undefined behaviour there):
//   D1  T4/T5 multipole tensors are not built: alpha9/d9 are never assigned
//       (src/field.f90:2098,2225) and no output reads T4/T5 without
//       quadrupoles, which this path does not support.
//   D2  BMH without damping (lbmhft): fdiff6/fdiff8 are uninitialised in the
//       reference (src/field.f90:2975); here they are 0.
//   D3  Morse: erh2/u2 are uninitialised and the force lacks 1/r
//       (src/field.f90:3058,3124,3132); here the force is the analytic
//       derivative of the reference energy expression (:3119-3122).
//   D4  LJ, BMH(FTD) and Morse each zero the forces (src/field.f90:1220-1222,
//       2904-2906, 3088-3090); here their forces are summed.
//   D10 xs/ys/zs (last-build positions for vnlistcheck) are never set by the
//       initial vnlist_pbc (src/mdff.f90:192); here every build records them.
//   D11 Positions are not round-tripped in place through kardir/dirkar on
//       every force call (src/field.f90:1237,1341 and similar).
//   D13 chain_nhcn (src/integration.f90:617-649) uses G(2..M-1) before
//       computing them on the first downward pass of every call (they are 0,
//       then stale), so for chains longer than 2 the extended energy is not
//       conserved.  Here the inner chain forces are refreshed first (the
//       Martyna-Tuckerman-Klein order); identical to the reference for M = 2.
//       nhc_literal = 1 restores the reference's order.
//   D14-D17 constant pressure (nhcnp, src/integration.f90:715-1160): the
//       k mesh and tail corrections follow the cell (the reference keeps
//       those of the start-up cell); the barostat momentum gets both half
//       kicks (the reference's trotter orders -1/+1 give one); chain forces
//       G = p^2/Q - kT and Gb_1 = ve^2/W - kT (the reference halves them);
//       kinetic pressure (1 + 3/Nf) 2K/3V (the reference uses K).  With
//       these the reference's e_npt + e_tot is conserved.
//   D18 rmc_main (src/rmc.f90:470-640) converts every position to direct
//       coordinates and back at each trial move (the round trip changes the
//       last bits of all atoms every move); here the chain keeps direct
//       coordinates and converts once at each end.
//   D20 eval_chisq_rmc sums the squared g(r) differences left to right;
//       here by a fixed tree (1024 strided partial sums, then halving trees),
//       the order of the device's parallel sum (last-bit differences only).
//   D19 the reference's Metropolis loop reads temp_rmc(6) past its
//       5-element array (src/rmc.f90:44,531); here the total's temperature
//       is a parameter.
//   D23 nhc2's thermostat energy (src/integration.f90:243-250) writes
//       vxi^2 / (2 Q), the momentum form of nhcn, although chain_nhc2's vxi
//       are velocities; here Q vxi^2 / 2 (the conserved quantity of the
//       Frenkel-Smit chain).  nhc_literal = 1 restores the reference's form.
//   D12 errfc: the reference's fitted erfc (src/functions.f90:28-39, a
//       published Chebyshev fit, relative error ~1.2e-7) is selectable with
//       orc_set_erfc_mode(sys, 0); mode 1 (default) uses libm erfc.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/mdff_engine.h"

namespace {

constexpr double PI = 3.14159265358979323846264338327950;   // constants.f90:62
constexpr double TPI = 2.0 * PI;
const double PIROOT = std::sqrt(PI);

constexpr int NT = MDFF_NTYPE_MAX;

struct Units { double press, boltz, time, coul; };

// celltype (src/lattice.f90:33-45): A[i][j] = A(i+1,j+1), column j = basis vector j.
struct Cell {
    double A[3][3];
    double B[3][3];
    double omega, WA, WB, WC;
    double anorm[3];
};

// lattice (src/lattice.f90:60-175): reciprocal basis scaled by 1/omega, volume,
// perpendicular widths and norms.
void lattice(Cell& c) {
    auto expro = [&](int out, int a, int b) {   // EXPRO(H,U1,U2), tools.f90:743-753
        c.B[0][out] = c.A[1][a] * c.A[2][b] - c.A[2][a] * c.A[1][b];
        c.B[1][out] = c.A[2][a] * c.A[0][b] - c.A[0][a] * c.A[2][b];
        c.B[2][out] = c.A[0][a] * c.A[1][b] - c.A[1][a] * c.A[0][b];
    };
    expro(0, 1, 2);
    expro(1, 2, 0);
    expro(2, 0, 1);
    double omega = c.B[0][0] * c.A[0][0] + c.B[1][0] * c.A[1][0] + c.B[2][0] * c.A[2][0];
    c.omega = omega;
    c.WA = omega / std::sqrt(c.B[0][0] * c.B[0][0] + c.B[1][0] * c.B[1][0] + c.B[2][0] * c.B[2][0]);
    c.WB = omega / std::sqrt(c.B[0][1] * c.B[0][1] + c.B[1][1] * c.B[1][1] + c.B[2][1] * c.B[2][1]);
    c.WC = omega / std::sqrt(c.B[0][2] * c.B[0][2] + c.B[1][2] * c.B[1][2] + c.B[2][2] * c.B[2][2]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c.B[i][j] = c.B[i][j] / omega;
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += c.A[k][i] * c.A[k][i];
        c.anorm[i] = std::sqrt(s);
    }
}

// kardir (src/lattice.f90:183-222): Cartesian -> direct, V_j = X*B(1,j)+Y*B(2,j)+Z*B(3,j).
inline void kardir1(const Cell& c, double x, double y, double z, double& s1, double& s2, double& s3) {
    s1 = x * c.B[0][0] + y * c.B[1][0] + z * c.B[2][0];
    s2 = x * c.B[0][1] + y * c.B[1][1] + z * c.B[2][1];
    s3 = x * c.B[0][2] + y * c.B[1][2] + z * c.B[2][2];
}
// dirkar (src/lattice.f90:229-262): direct -> Cartesian, V_i = X*A(i,1)+Y*A(i,2)+Z*A(i,3).
inline void dirkar1(const Cell& c, double x, double y, double z, double& r1, double& r2, double& r3) {
    r1 = x * c.A[0][0] + y * c.A[0][1] + z * c.A[0][2];
    r2 = x * c.A[1][0] + y * c.A[1][1] + z * c.A[1][2];
    r3 = x * c.A[2][0] + y * c.A[2][1] + z * c.A[2][2];
}
// Fortran NINT rounds half away from zero.
inline double nint(double x) { return std::round(x); }

// Minimum-image pair vector from direct coordinates, in the order of
// vnlist_pbc (src/tools.f90:323-332) and every pair routine.
inline double pairvec(const Cell& c, double si1, double si2, double si3,
                      double sj1, double sj2, double sj3, double& rx, double& ry, double& rz) {
    double dx = si1 - sj1, dy = si2 - sj2, dz = si3 - sj3;
    double sx = dx - nint(dx), sy = dy - nint(dy), sz = dz - nint(dz);
    rx = sx * c.A[0][0] + sy * c.A[0][1] + sz * c.A[0][2];
    ry = sx * c.A[1][0] + sy * c.A[1][1] + sz * c.A[1][2];
    rz = sx * c.A[2][0] + sy * c.A[2][1] + sz * c.A[2][2];
    return rx * rx + ry * ry + rz * rz;
}

// errfc (src/functions.f90:28-39): the reference's fitted complementary error
// function (Numerical Recipes' Chebyshev fit).
double errfc_ref(double x) {
    double z = std::fabs(x);
    double t = 1.0 / (1.0 + 0.5 * z);
    double r = t * std::exp(-z * z - 1.26551223 + t * (1.00002368 + t * (.37409196 +
               t * (.09678418 + t * (-.18628806 + t * (.27886807 + t * (-1.13520398 +
               t * (1.48851587 + t * (-.82215223 + t * .17087277)))))))));
    if (x < 0.0) r = 2.0 - r;
    return r;
}

// get_TT_damp (src/tt_damp.f90:13-29)
double E_TT[MDFF_TT_MAX_ORDER + 1];
struct TTInit { TTInit() { E_TT[0] = 1.0; for (int k = 1; k <= MDFF_TT_MAX_ORDER; ++k) E_TT[k] = E_TT[k - 1] / double(k); } } tt_init_;

// TT_damping_functions (src/field.f90:3775-3805)
inline void tt_damp(double b, double c, double r, int order, double& f, double& fd) {
    double br = b * r;
    double expbdr = std::exp(-br) * c;
    f = E_TT[order];
    for (int k = order - 1; k >= 1; --k) f = f * br + E_TT[k];
    f = f * br + E_TT[0];
    f = 1.0 - f * expbdr;
    fd = E_TT[order] * std::pow(br, order) * expbdr * b;
}

struct KMesh {   // kmesh (src/kspace.f90:37-53)
    int nk = 0;
    std::vector<double> kx, ky, kz, kk, Ak, kcoe;
};

// Verlet list in the reference layout (config.f90:64-72), 0-based internally.
struct VList {
    double cut = 0.0;
    std::vector<int> point;   // natm+1
    std::vector<int> list;
};

}  // namespace

struct orc_sys {
    mdff_params p;
    Units u;
    Cell cell;
    int natm = 0;
    int ntype = 0;
    int m1_indica = 0;   // mlis3's SAVEd indica (src/m1qn3.f90:1040-1041), zero in a fresh process
    std::vector<int> itype;          // 0-based
    std::vector<double> rx, ry, rz, vx, vy, vz, fx, fy, fz;
    std::vector<double> massia, qia, poldia, invpoldia;
    std::vector<double> dipx, dipy, dipz;   // static dipoles
    std::vector<int> natmi;
    // nonbonded constants (initialize_param_non_bonded, field.f90:914-1101)
    double rcutsq[NT][NT], sigsq[NT][NT], epsp[NT][NT], fc[NT][NT], uc[NT][NT], uc1[NT][NT], uc2[NT][NT];
    double fm[NT][NT], rs[NT][NT];
    double utail = 0.0, ptail = 0.0;
    double cutlongrange = 0.0;
    double alphaES = 0.0;
    int kES[3] = {0, 0, 0};
    KMesh km;
    VList vdw, coul;
    std::vector<double> xs, ys, zs;
    bool have_list = false;
    // induced dipoles: history dipia_ind_t(extrapolate_order+1, natm, 3) (field.f90:1612)
    std::vector<double> dip_hist;    // [(order+1)][natm][3]
    double u_pol = 0.0;              // thermodynamic u_pol (module variable)
    int itime = 0;
    // MD state (md.f90:60-62)
    std::vector<double> xi, vxi;
    double dt = 0.0, temp = 0.0, timesca = 0.0;
    // constant pressure (md.f90:60-62): barostat chain, log-volume and momentum
    std::vector<double> xib, vxib;
    double xe = 0.0, ve = 0.0, xe0 = 0.0, e_npt = 0.0;
    double scale = 1.0, scale_build = 1.0;   // linear cell scale now / at the last list build
    double omega0 = 0.0, utail0 = 0.0, ptail0 = 0.0;
    int erfc_mode = 1;
    // outputs of the last engforce
    mdff_energies en;
    double tau_nonb[3][3], tau_coul[3][3];
    std::vector<double> ef, efg, mu;  // ef [3][N], efg [3][3][N], mu [3][N]
    double e_kin = 0.0, temp_r = 0.0, e_nvt = 0.0;
    int step_rebuilt = 0;
    std::string err;
};

namespace {

inline double& EFG(orc_sys* s, std::vector<double>& a, int i, int j, int ia) { return a[(size_t)(i * 3 + j) * s->natm + ia]; }

double erfc_sel(const orc_sys* s, double x) { return s->erfc_mode == 0 ? errfc_ref(x) : std::erfc(x); }

void set_units(orc_sys* s) {
    if (s->p.lreduced) { s->u = {1.0, 1.0, 1.0, 1.0}; return; }   // reduced_units, constants.f90:135-146
    s->u.press = 0.00624150964712042;                               // constants.f90:85-89
    s->u.boltz = 8.61734229648141e-05;
    s->u.time = 98.2269514139276;
    s->u.coul = 14.3996441494161;
}

// field_check_tag symmetrisation (src/field.f90:316-339)
void symmetrise(mdff_params& p) {
    if (!p.symmetric_pot) return;
    int n = p.ntype;
    for (int it = 0; it < n; ++it)
        for (int jt = 0; jt < n; ++jt) {
            p.epslj[jt][it] = p.epslj[it][jt];
            p.sigmalj[jt][it] = p.sigmalj[it][jt];
            p.plj[jt][it] = p.plj[it][jt];
            p.qlj[jt][it] = p.qlj[it][jt];
            p.Abmhftd[jt][it] = p.Abmhftd[it][jt];
            p.Bbmhftd[jt][it] = p.Bbmhftd[it][jt];
            p.Cbmhftd[jt][it] = p.Cbmhftd[it][jt];
            p.Dbmhftd[jt][it] = p.Dbmhftd[it][jt];
            p.BDbmhftd[jt][it] = p.BDbmhftd[it][jt];
            for (int it2 = 0; it2 < n; ++it2) {
                p.ldip_damping[it2][jt][it] = p.ldip_damping[it2][it][jt];
                p.dip_pol_damp_b[it2][jt][it] = p.dip_pol_damp_b[it2][it][jt];
                p.dip_pol_damp_c[it2][jt][it] = p.dip_pol_damp_c[it2][it][jt];
                p.dip_pol_damp_k[it2][jt][it] = p.dip_pol_damp_k[it2][it][jt];
            }
        }
}

// ewald_param (src/field.f90:860-908): clamp of cutlongrange and optional
// DL_POLY-style automatic alpha / kmax.
void ewald_param(orc_sys* s) {
    const Cell& c = s->cell;
    double rcut = 0.5 * std::min(c.WA, std::min(c.WB, c.WC));
    s->cutlongrange = std::min(s->p.cutlongrange, rcut);
    double eps = std::min(std::fabs(s->p.epsw), 0.5);
    double tol = std::sqrt(std::fabs(std::log(eps * s->cutlongrange)));
    double alpha = std::sqrt(std::fabs(std::log(eps * s->cutlongrange * tol))) / rcut;
    double tol1 = std::sqrt(-std::log(eps * s->cutlongrange * (2.0 * tol * alpha) * (2.0 * tol * alpha)));
    s->alphaES = s->p.alphaES;
    for (int i = 0; i < 3; ++i) s->kES[i] = s->p.kES[i];
    if (s->p.lautoES) {
        s->alphaES = alpha;
        for (int i = 0; i < 3; ++i) s->kES[i] = (int)nint(0.25 + c.anorm[i] * alpha * tol1 / PI);
    }
}

// initialize_param_non_bonded (src/field.f90:914-1101)
void init_nonbonded(orc_sys* s) {
    const mdff_params& p = s->p;
    double one16 = 1.0 / 6.0;
    double two16 = std::pow(2.0, one16);
    s->utail = 0.0; s->ptail = 0.0;
    for (int it = 0; it < s->ntype; ++it)
        for (int jt = 0; jt < s->ntype; ++jt) {
            double pp = p.plj[it][jt], qq = p.qlj[it][jt];
            double pp3 = pp - 3.0, qq3 = qq - 3.0;
            double rcut = p.cutshortrange;
            s->rcutsq[it][jt] = rcut * rcut;
            double rcut3 = rcut * s->rcutsq[it][jt];
            double ppqq = pp * qq;
            s->epsp[it][jt] = p.epslj[it][jt] / (qq - pp);
            s->sigsq[it][jt] = two16 * two16 * p.sigmalj[it][jt] * p.sigmalj[it][jt];
            double sr2 = s->sigsq[it][jt] / s->rcutsq[it][jt];
            double sr = std::sqrt(sr2);
            double srp = std::pow(sr, pp), srq = std::pow(sr, qq);
            double ep = s->epsp[it][jt];
            s->uc[it][jt] = ep * (pp * srq - qq * srp);
            s->uc1[it][jt] = ep * ppqq / (2.0 * s->rcutsq[it][jt]) * (srq - srp);
            s->uc2[it][jt] = 0.5 * ep * ((2.0 * pp + ppqq) * srq - (2.0 * qq + ppqq) * srp);
            s->fc[it][jt] = ppqq * ep / s->sigsq[it][jt];
            s->fm[it][jt] = -2.0 * p.epsmor[it][jt] * p.rhomor[it][jt] * std::exp(p.rhomor[it][jt] * p.sigmamor[it][jt]);
            s->rs[it][jt] = std::exp(p.rhomor[it][jt] * p.sigmamor[it][jt]);
            double ut = ep * (pp * srq / qq3 - qq * srp / pp3);
            double pt = ppqq * ep * (srq / qq3 - srp / pp3);
            ut = ut * rcut3 * TPI;
            pt = pt * rcut3 * TPI;
            if (s->natmi[it] != 0 && s->natmi[jt] != 0) {
                s->utail = s->utail + ut * s->natmi[it] * s->natmi[jt] / s->cell.omega;
                s->ptail = s->ptail + pt * s->natmi[it] * s->natmi[jt] / s->cell.omega;
            }
        }
    s->ptail = s->ptail / s->u.press / s->cell.omega / 3.0;
}

// kpoint_sum_init + reorder_kpt (src/kspace.f90:142-207, 287-345)
void kpoint_sum_init(orc_sys* s) {
    KMesh& km = s->km;
    const Cell& c = s->cell;
    double alpha2 = s->alphaES * s->alphaES;
    km = KMesh();
    std::vector<double> kx, ky, kz, kk, Ak, kcoe;
    for (int nx = 0; nx <= s->kES[0]; ++nx) {
        int nymin = (nx == 0) ? 0 : -s->kES[1];
        for (int ny = nymin; ny <= s->kES[1]; ++ny) {
            int nzmin = (nx == 0 && ny == 0) ? 1 : -s->kES[2];
            for (int nz = nzmin; nz <= s->kES[2]; ++nz) {
                double x = TPI * (double(nx) * c.B[0][0] + double(ny) * c.B[0][1] + double(nz) * c.B[0][2]);
                double y = TPI * (double(nx) * c.B[1][0] + double(ny) * c.B[1][1] + double(nz) * c.B[1][2]);
                double z = TPI * (double(nx) * c.B[2][0] + double(ny) * c.B[2][1] + double(nz) * c.B[2][2]);
                double k2 = x * x + y * y + z * z;
                kx.push_back(x); ky.push_back(y); kz.push_back(z); kk.push_back(k2);
                Ak.push_back(std::exp(-k2 * 0.25 / alpha2) / k2);
                kcoe.push_back(2.0 * (1.0 / k2 + 1.0 / alpha2 / 4.0));
            }
        }
    }
    int nk = (int)kx.size();
    std::vector<int> idx(nk);
    for (int i = 0; i < nk; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return kk[a] < kk[b]; });   // merge_sort: stable
    km.nk = nk;
    km.kx.resize(nk); km.ky.resize(nk); km.kz.resize(nk); km.kk.resize(nk); km.Ak.resize(nk); km.kcoe.resize(nk);
    for (int i = 0; i < nk; ++i) {
        int l = idx[i];
        km.kx[i] = kx[l]; km.ky[i] = ky[l]; km.kz[i] = kz[l]; km.kk[i] = kk[l]; km.Ak[i] = Ak[l]; km.kcoe[i] = kcoe[l];
    }
}

void direct_coords(const orc_sys* s, std::vector<double>& sx, std::vector<double>& sy, std::vector<double>& sz) {
    sx.resize(s->natm); sy.resize(s->natm); sz.resize(s->natm);
    for (int i = 0; i < s->natm; ++i) kardir1(s->cell, s->rx[i], s->ry[i], s->rz[i], sx[i], sy[i], sz[i]);
}

// vnlist_pbc (src/tools.f90:274-370): both lists in one all-pairs pass, half
// lists with the parity ownership rule, ascending ja per atom.
void vnlist_pbc(orc_sys* s) {
    int n = s->natm;
    std::vector<double> sx, sy, sz;
    direct_coords(s, sx, sy, sz);
    double rv = s->vdw.cut + s->p.skindiff;  double rskinsq_vdw = rv * rv;
    double rc = s->coul.cut + s->p.skindiff; double rskinsq_coul = rc * rc;
    std::vector<std::vector<int>> lv(n), lc(n);
#pragma omp parallel for schedule(dynamic, 16)
    for (int ia = 0; ia < n; ++ia) {
        for (int ja = 0; ja < n; ++ja) {
            int I = ia + 1, J = ja + 1;   // 1-based parity rule
            if ((I > J && ((I + J) % 2 == 0)) || (I < J && ((I + J) % 2 != 0))) {
                double rxij, ryij, rzij;
                double rijsq = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], rxij, ryij, rzij);
                if (rijsq <= rskinsq_vdw) lv[ia].push_back(ja);
                if (rijsq <= rskinsq_coul) lc[ia].push_back(ja);
            }
        }
    }
    auto pack = [&](VList& L, std::vector<std::vector<int>>& l) {
        L.point.assign(n + 1, 0);
        L.list.clear();
        for (int ia = 0; ia < n; ++ia) {
            L.point[ia] = (int)L.list.size();
            L.list.insert(L.list.end(), l[ia].begin(), l[ia].end());
        }
        L.point[n] = (int)L.list.size();
    };
    pack(s->vdw, lv);
    pack(s->coul, lc);
    s->xs = sx; s->ys = sy; s->zs = sz;   // D10
    s->have_list = true;
    s->scale_build = s->scale;
}

// vnlistcheck (src/tools.f90:446-535): largest + second largest displacement
// since the last build against skindiff.
bool vnlistcheck(orc_sys* s) {
    double dmax = 0.0, dmax2 = 0.0;
    for (int ia = 0; ia < s->natm; ++ia) {
        double s1, s2, s3;
        kardir1(s->cell, s->rx[ia], s->ry[ia], s->rz[ia], s1, s2, s3);
        double rxsi, rysi, rzsi;
        double d2 = pairvec(s->cell, s1, s2, s3, s->xs[ia], s->ys[ia], s->zs[ia], rxsi, rysi, rzsi);
        double drnei = std::sqrt(d2);
        if (drnei > dmax) { dmax2 = dmax; dmax = drnei; }
        else if (drnei > dmax2) dmax2 = drnei;
    }
    // a shrinking cell (constant pressure) brings pairs beyond the list radius
    // closer by the same factor: that margin comes off the allowance
    const double shrink = std::max(0.0, 1.0 - s->scale / s->scale_build);
    const double rl = std::max(s->vdw.cut, s->coul.cut) + s->p.skindiff;
    if (dmax + dmax2 > s->p.skindiff - shrink * rl) { vnlist_pbc(s); return true; }
    return false;
}

// Pair iteration over a half list (lvnlist) or all ja > ia, as the pair
// routines do (e.g. src/field.f90:1241-1263).
template <class F>
void for_pairs(orc_sys* s, const VList& L, const std::vector<double>& sx, const std::vector<double>& sy,
               const std::vector<double>& sz, F&& f) {
    int n = s->natm;
    if (s->p.lvnlist) {
        for (int ia = 0; ia < n; ++ia)
            for (int j1 = L.point[ia]; j1 < L.point[ia + 1]; ++j1) {
                int ja = L.list[j1];
                if (ja == ia) continue;
                f(ia, ja);
            }
    } else {
        for (int ia = 0; ia < n; ++ia)
            for (int ja = ia + 1; ja < n; ++ja) f(ia, ja);
    }
}

// engforce_nmlj_pbc (src/field.f90:1181-1345)
void engforce_nmlj(orc_sys* s, const std::vector<double>& sx, const std::vector<double>& sy, const std::vector<double>& sz) {
    const mdff_params& p = s->p;
    double u = 0.0, vir = 0.0;
    double tau[3][3] = {{0}};
    for_pairs(s, s->vdw, sx, sy, sz, [&](int ia, int ja) {
        double rxij, ryij, rzij;
        double rijsq = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], rxij, ryij, rzij);
        int p1 = s->itype[ia], p2 = s->itype[ja];
        if (rijsq < s->rcutsq[p1][p2]) {
            double sr2 = s->sigsq[p1][p2] / rijsq;
            double srp = std::pow(sr2, p.plj[p1][p2] * 0.5);
            double srq = std::pow(sr2, p.qlj[p1][p2] * 0.5);
            if (p.trunc == 0) u = u + s->epsp[p1][p2] * (p.plj[p1][p2] * srq - p.qlj[p1][p2] * srp);
            if (p.trunc == 1) u = u + s->epsp[p1][p2] * (p.plj[p1][p2] * srq - p.qlj[p1][p2] * srp) - s->uc[p1][p2];
            if (p.trunc == 2) u = u + s->epsp[p1][p2] * (p.plj[p1][p2] * srq - p.qlj[p1][p2] * srp) + s->uc1[p1][p2] * rijsq - s->uc2[p1][p2];
            double wij = s->fc[p1][p2] * (srq - srp) * sr2;
            double f[3] = {wij * rxij, wij * ryij, wij * rzij};
            double r[3] = {rxij, ryij, rzij};
            vir = vir + wij * rijsq;
            s->fx[ia] += f[0]; s->fy[ia] += f[1]; s->fz[ia] += f[2];
            s->fx[ja] -= f[0]; s->fy[ja] -= f[1]; s->fz[ja] -= f[2];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) tau[a][b] = tau[a][b] + (r[a] * f[b] + r[b] * f[a]) * 0.5;
        }
    });
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) s->tau_nonb[a][b] += tau[a][b] / s->cell.omega / s->u.press;
    s->en.u_lj = u;
    s->en.vir_lj = vir / 3.0;
}

// engforce_bmhftd_pbc (src/field.f90:2876-3026)
void engforce_bmhftd(orc_sys* s, const std::vector<double>& sx, const std::vector<double>& sy, const std::vector<double>& sz) {
    const mdff_params& p = s->p;
    double u = 0.0, vir = 0.0;
    double tau[3][3] = {{0}};
    for_pairs(s, s->vdw, sx, sy, sz, [&](int ia, int ja) {
        double rxij, ryij, rzij;
        double rijsq = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], rxij, ryij, rzij);
        int p1 = s->itype[ia], p2 = s->itype[ja];
        if (p.Abmhftd[p1][p2] == 0.0) return;
        if (rijsq < s->rcutsq[p1][p2]) {
            double ir2 = 1.0 / rijsq;
            double d = std::sqrt(rijsq);
            double erh = p.Abmhftd[p1][p2] * std::exp(-p.Bbmhftd[p1][p2] * d);
            double ir6 = ir2 * ir2 * ir2;
            double ir8 = ir6 * ir2;
            ir6 = ir6 * p.Cbmhftd[p1][p2];
            ir8 = ir8 * p.Dbmhftd[p1][p2];
            double ir6d, ir8d, fdiff6 = 0.0, fdiff8 = 0.0;   // D2
            if (p.lbmhftd) {
                double f6, f8;
                tt_damp(p.BDbmhftd[p1][p2], 1.0, d, 6, f6, fdiff6);
                tt_damp(p.BDbmhftd[p1][p2], 1.0, d, 8, f8, fdiff8);
                ir6d = ir6 * f6;
                ir8d = ir8 * f8;
            } else {
                ir6d = ir6;
                ir8d = ir8;
            }
            double ir7 = 6.0 * ir6d / d;
            double ir9 = 8.0 * ir8d / d;
            u = u + erh - ir6d - ir8d;
            double wij = p.Bbmhftd[p1][p2] * erh - ir7 - ir9 + ir6 * fdiff6 + ir8 * fdiff8;
            wij = wij / d;
            double f[3] = {wij * rxij, wij * ryij, wij * rzij};
            double r[3] = {rxij, ryij, rzij};
            vir = vir + (rxij * f[0] + ryij * f[1] + rzij * f[2]);
            s->fx[ia] += f[0]; s->fy[ia] += f[1]; s->fz[ia] += f[2];
            s->fx[ja] -= f[0]; s->fy[ja] -= f[1]; s->fz[ja] -= f[2];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) tau[a][b] = tau[a][b] + (r[a] * f[b] + r[b] * f[a]);
        }
    });
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) s->tau_nonb[a][b] += tau[a][b] / s->cell.omega / s->u.press * 0.5;
    s->en.u_bmhft = u;
    s->en.vir_bmhft = vir / 3.0;
}

// engforce_morse_pbc (src/field.f90:3039-3185) with the analytic force (D3).
void engforce_morse(orc_sys* s, const std::vector<double>& sx, const std::vector<double>& sy, const std::vector<double>& sz) {
    const mdff_params& p = s->p;
    double u = 0.0, vir = 0.0;
    double tau[3][3] = {{0}};
    for_pairs(s, s->vdw, sx, sy, sz, [&](int ia, int ja) {
        double rxij, ryij, rzij;
        double rijsq = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], rxij, ryij, rzij);
        int p1 = s->itype[ja], p2 = s->itype[ia];
        if (rijsq < s->rcutsq[p1][p2]) {
            double d = std::sqrt(rijsq);
            double erh = std::exp(-d * p.rhomor[p1][p2]);
            double e = erh * s->rs[p1][p2];
            double expon = e - 1.0;
            expon = expon * expon - 1.0;
            u = u + p.epsmor[p1][p2] * expon;
            // -dU/dr / r with U = eps*((e-1)^2-1), e = exp(-rho (r - sigma))
            double wij = 2.0 * p.epsmor[p1][p2] * p.rhomor[p1][p2] * e * (e - 1.0) / d;
            vir = vir + wij * rijsq;
            double f[3] = {wij * rxij, wij * ryij, wij * rzij};
            double r[3] = {rxij, ryij, rzij};
            s->fx[ia] += f[0]; s->fy[ia] += f[1]; s->fz[ia] += f[2];
            s->fx[ja] -= f[0]; s->fy[ja] -= f[1]; s->fz[ja] -= f[2];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) tau[a][b] = tau[a][b] + r[a] * f[b];
        }
    });
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) s->tau_nonb[a][b] += tau[a][b] / s->cell.omega / s->u.press;
    s->en.u_morse = u;
    s->en.vir_morse = vir / 3.0;
}

struct ESOut {
    double u_dir = 0, u_rec = 0, u_self = 0, u_surf = 0;
    std::vector<double> ef;      // [3][N]
    std::vector<double> efg;     // [3][3][N]
    std::vector<double> f;       // [3][N]
    double tau[3][3] = {{0}};
};

// multipole_ES_dir (src/field.f90:2057-2643), charges and dipoles.
void multipole_ES_dir(orc_sys* s, const std::vector<double>& q, const std::vector<double>& mu, const bool task[6],
                      bool damp_ind, bool do_efield, bool do_efg, bool do_forces, bool do_stress,
                      double& u_dir, std::vector<double>& ef, std::vector<double>& efg, std::vector<double>& f,
                      double tau[3][3]) {
    const mdff_params& p = s->p;
    int n = s->natm;
    std::vector<double> sx, sy, sz;
    direct_coords(s, sx, sy, sz);
    bool charge_charge = task[0], charge_dipole = task[1], dipole_dipole = task[2];
    double cutsq = s->coul.cut * s->coul.cut;
    double aES = s->alphaES;
    double alpha2 = aES * aES, alpha3 = alpha2 * aES, alpha5 = alpha3 * alpha2;
    auto MU = [&](int c, int i) { return mu[(size_t)c * n + i]; };
    auto EF = [&](int c, int i) -> double& { return ef[(size_t)c * n + i]; };
    auto G = [&](int a, int b, int i) -> double& { return efg[(size_t)(a * 3 + b) * n + i]; };
    auto FF = [&](int c, int i) -> double& { return f[(size_t)c * n + i]; };
    for_pairs(s, s->coul, sx, sy, sz, [&](int ia, int ja) {
        int ita = s->itype[ia], jta = s->itype[ja];
        double qi = q[ia], qj = q[ja];
        double mui[3] = {MU(0, ia), MU(1, ia), MU(2, ia)};
        double muj[3] = {MU(0, ja), MU(1, ja), MU(2, ja)};
        bool dip_i = mui[0] != 0.0 || mui[1] != 0.0 || mui[2] != 0.0;
        bool dip_j = muj[0] != 0.0 || muj[1] != 0.0 || muj[2] != 0.0;
        double qij = qi * qj;
        double rij[3];
        double d2 = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], rij[0], rij[1], rij[2]);
        if (d2 > cutsq) return;
        double d = std::sqrt(d2);
        double d3 = d2 * d, d5 = d3 * d2;
        double dm1 = 1.0 / d, dm3 = dm1 / d2, dm5 = dm3 / d2, dm7 = dm5 / d2;
        bool ldamp = p.ldip_damping[ita][ita][jta] || p.ldip_damping[jta][ita][jta];
        if (!damp_ind) ldamp = false;
        double fdamp = 1.0, fdamp2 = 1.0, fdampdiff = 0.0, fdampdiff2 = 0.0;
        if (ldamp) {
            tt_damp(p.dip_pol_damp_b[ita][ita][jta], p.dip_pol_damp_c[ita][ita][jta], d, p.dip_pol_damp_k[ita][ita][jta], fdamp, fdampdiff);
            tt_damp(p.dip_pol_damp_b[jta][ita][jta], p.dip_pol_damp_c[jta][ita][jta], d, p.dip_pol_damp_k[jta][ita][jta], fdamp2, fdampdiff2);
        }
        double expon = std::exp(-alpha2 * d2) / PIROOT;
        double F0 = erfc_sel(s, aES * d);
        double F1 = F0 + 2.0 * aES * d * expon;
        double F2 = F1 + 4.0 * alpha3 * d3 * expon / 3.0;
        double F3 = F2 + 8.0 * alpha5 * d5 * expon / 15.0;
        double F1d = -fdamp + 1.0;
        double F2d = F1d + (d / 3.0) * fdampdiff;
        double F1d2 = -fdamp2 + 1.0;
        double F2d2 = F1d2 + (d / 3.0) * fdampdiff2;
        double T0 = dm1 * F0;
        double T1[3], T1d[3] = {0, 0, 0}, T1d2[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a) T1[a] = -rij[a] * dm3;
        if (ldamp)
            for (int a = 0; a < 3; ++a) { T1d[a] = T1[a] * F1d; T1d2[a] = T1[a] * F1d2; }
        for (int a = 0; a < 3; ++a) T1[a] = T1[a] * F1;
        double T2[3][3], T2d[3][3] = {{0}}, T2d2[3][3] = {{0}};
        double F2_dm5 = 3.0 * F2 * dm5, F2d_dm5 = 3.0 * F2d * dm5, F2d2_dm5 = 3.0 * F2d2 * dm5;
        double F1_dm3 = F1 * dm3, F1d_dm3 = F1d * dm3, F1d2_dm3 = F1d2 * dm3;
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
                T2[j][k] = rij[j] * rij[k] * F2_dm5;
                if (j == k) T2[j][j] = T2[j][j] - F1_dm3;
                if (ldamp) {
                    T2d[j][k] = rij[j] * rij[k] * F2d_dm5;
                    T2d2[j][k] = rij[j] * rij[k] * F2d2_dm5;
                    if (j == k) { T2d[j][j] = T2d[j][j] - F1d_dm3; T2d2[j][j] = T2d2[j][j] - F1d2_dm3; }
                }
            }
        double F3_dm7 = F3 * dm7 * 15.0;
        double T3[3][3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    T3[i][j][k] = -rij[i] * rij[j] * rij[k] * F3_dm7;
                    if (i == j) T3[i][j][k] = T3[i][j][k] + rij[k] * F2_dm5;
                    if (i == k) T3[i][j][k] = T3[i][j][k] + rij[j] * F2_dm5;
                    if (j == k) T3[i][j][k] = T3[i][j][k] + rij[i] * F2_dm5;
                }
        double fij[3];
        if (charge_charge) {   // field.f90:2363-2403
            u_dir = u_dir + qij * T0;
            if (do_efield) {
                for (int a = 0; a < 3; ++a) { EF(a, ia) = EF(a, ia) - qj * T1[a]; EF(a, ja) = EF(a, ja) + qi * T1[a]; }
                if (ldamp)
                    for (int a = 0; a < 3; ++a) { EF(a, ia) = EF(a, ia) + qj * T1d[a]; EF(a, ja) = EF(a, ja) - qi * T1d2[a]; }
            }
            if (do_efg)
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) { G(a, b, ia) = G(a, b, ia) - qj * T2[a][b]; G(a, b, ja) = G(a, b, ja) - qi * T2[a][b]; }
            for (int a = 0; a < 3; ++a) fij[a] = qij * T1[a];
            if (do_forces)
                for (int a = 0; a < 3; ++a) { FF(a, ia) = FF(a, ia) - fij[a]; FF(a, ja) = FF(a, ja) + fij[a]; }
            if (do_stress)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) tau[j][k] = tau[j][k] - (rij[j] * fij[k] + rij[k] * fij[j]);
        }
        if (dipole_dipole && (dip_i || dip_j)) {   // field.f90:2407-2456
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) u_dir = u_dir - mui[j] * T2[j][k] * muj[k];
            if (do_efield)
                for (int k = 0; k < 3; ++k)
                    for (int a = 0; a < 3; ++a) { EF(a, ia) = EF(a, ia) + T2[a][k] * muj[k]; EF(a, ja) = EF(a, ja) + T2[a][k] * mui[k]; }
            if (do_efg)
                for (int k = 0; k < 3; ++k)
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) {
                            G(a, b, ia) = G(a, b, ia) + T3[a][b][k] * muj[k];
                            G(a, b, ja) = G(a, b, ja) - T3[a][b][k] * mui[k];
                        }
            fij[0] = fij[1] = fij[2] = 0.0;
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k)
                    for (int a = 0; a < 3; ++a) fij[a] = fij[a] + mui[j] * T3[j][a][k] * muj[k];
            if (do_forces)
                for (int a = 0; a < 3; ++a) { FF(a, ia) = FF(a, ia) + fij[a]; FF(a, ja) = FF(a, ja) - fij[a]; }
            if (do_stress)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) tau[j][k] = tau[j][k] + (rij[j] * fij[k] + rij[k] * fij[j]);
        }
        if (charge_dipole && (dip_i || dip_j)) {   // field.f90:2462-2534
            for (int k = 0; k < 3; ++k) {
                u_dir = u_dir - qi * T1[k] * muj[k];
                u_dir = u_dir + qj * T1[k] * mui[k];
                if (ldamp) {
                    u_dir = u_dir + qi * T1d2[k] * muj[k];
                    u_dir = u_dir - qj * T1d[k] * mui[k];
                }
            }
            fij[0] = fij[1] = fij[2] = 0.0;
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    fij[k] = fij[k] + qi * T2[k][j] * muj[j];
                    fij[k] = fij[k] - qj * T2[k][j] * mui[j];
                }
            if (do_forces)
                for (int a = 0; a < 3; ++a) { FF(a, ia) = FF(a, ia) + fij[a]; FF(a, ja) = FF(a, ja) - fij[a]; }
            if (do_stress)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) tau[j][k] = tau[j][k] + (rij[j] * fij[k] + rij[k] * fij[j]);
            if (ldamp) {
                fij[0] = fij[1] = fij[2] = 0.0;
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        fij[k] = fij[k] + qj * T2d[k][j] * mui[j];
                        fij[k] = fij[k] - qi * T2d2[k][j] * muj[j];
                    }
                if (do_forces)
                    for (int a = 0; a < 3; ++a) { FF(a, ia) = FF(a, ia) + fij[a]; FF(a, ja) = FF(a, ja) - fij[a]; }
                if (do_stress)
                    for (int j = 0; j < 3; ++j)
                        for (int k = 0; k < 3; ++k) tau[j][k] = tau[j][k] + (rij[j] * fij[k] + rij[k] * fij[j]);
            }
        }
    });
    if (do_stress)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) tau[a][b] = tau[a][b] / s->cell.omega * 0.5;
}

// multipole_ES_rec (src/field.f90:2646-2873), charges and dipoles; k-vectors
// in parallel with per-thread partial sums combined in thread order.
void multipole_ES_rec(orc_sys* s, const std::vector<double>& q, const std::vector<double>& mu, const bool task[6],
                      bool do_efield, bool do_efg, bool do_forces, bool do_stress,
                      double& u_rec, std::vector<double>& ef, std::vector<double>& efg, std::vector<double>& f,
                      double tau[3][3]) {
    int n = s->natm;
    const KMesh& km = s->km;
    double tpi_V = TPI / s->cell.omega;
    double fpi_V = tpi_V * 2.0;
    bool ldip = task[1] || task[2];
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    std::vector<std::vector<double>> tef(nth), tefg(nth), tf(nth);
    std::vector<double> tu(nth, 0.0), ttau(nth * 9, 0.0);
#pragma omp parallel
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        std::vector<double>& lef = tef[t];
        std::vector<double>& lefg = tefg[t];
        std::vector<double>& lf = tf[t];
        if (do_efield) lef.assign((size_t)3 * n, 0.0);
        if (do_efg) lefg.assign((size_t)9 * n, 0.0);
        if (do_forces) lf.assign((size_t)3 * n, 0.0);
        std::vector<double> ckr(n), skr(n);
        double lu = 0.0;
        double* lt = &ttau[(size_t)t * 9];
#pragma omp for schedule(static)
        for (int ik = 0; ik < km.nk; ++ik) {
            if (km.kk[ik] == 0.0) continue;
            double kx = km.kx[ik], ky = km.ky[ik], kz = km.kz[ik], Ak = km.Ak[ik], kcoe = km.kcoe[ik];
            double rhonk_R = 0.0, rhonk_I = 0.0;
            for (int ia = 0; ia < n; ++ia) {
                double qi = q[ia];
                double k_dot_r = (kx * s->rx[ia] + ky * s->ry[ia] + kz * s->rz[ia]);
                ckr[ia] = std::cos(k_dot_r);
                skr[ia] = std::sin(k_dot_r);
                rhonk_R = rhonk_R + qi * ckr[ia];
                rhonk_I = rhonk_I + qi * skr[ia];
                if (!ldip) continue;
                double k_dot_mu = (mu[ia] * kx + mu[(size_t)n + ia] * ky + mu[(size_t)2 * n + ia] * kz);
                rhonk_R = rhonk_R - k_dot_mu * skr[ia];
                rhonk_I = rhonk_I + k_dot_mu * ckr[ia];
            }
            double str = (rhonk_R * rhonk_R + rhonk_I * rhonk_I) * Ak;
            lu = lu + str;
            for (int ia = 0; ia < n; ++ia) {
                double fxij = 0, fyij = 0, fzij = 0;
                if (do_efield || do_forces) {
                    double recarg = Ak * (rhonk_I * ckr[ia] - rhonk_R * skr[ia]);
                    fxij = kx * recarg; fyij = ky * recarg; fzij = kz * recarg;
                }
                if (do_efield) {
                    lef[ia] = lef[ia] - fxij;
                    lef[(size_t)n + ia] = lef[(size_t)n + ia] - fyij;
                    lef[(size_t)2 * n + ia] = lef[(size_t)2 * n + ia] - fzij;
                }
                if (do_efg) {
                    double recarg2 = Ak * (rhonk_R * ckr[ia] + rhonk_I * skr[ia]);
                    lefg[(size_t)0 * n + ia] += kx * kx * recarg2;   // (1,1)
                    lefg[(size_t)4 * n + ia] += ky * ky * recarg2;   // (2,2)
                    lefg[(size_t)8 * n + ia] += kz * kz * recarg2;   // (3,3)
                    lefg[(size_t)1 * n + ia] += kx * ky * recarg2;   // (1,2)
                    lefg[(size_t)2 * n + ia] += kx * kz * recarg2;   // (1,3)
                    lefg[(size_t)5 * n + ia] += ky * kz * recarg2;   // (2,3)
                }
                if (do_forces) {
                    double qi = q[ia];
                    lf[ia] = lf[ia] - qi * fxij;
                    lf[(size_t)n + ia] = lf[(size_t)n + ia] - qi * fyij;
                    lf[(size_t)2 * n + ia] = lf[(size_t)2 * n + ia] - qi * fzij;
                    if (!ldip) continue;
                    double recarg2 = Ak * (rhonk_R * ckr[ia] + rhonk_I * skr[ia]);
                    double k_dot_mu = (mu[ia] * kx + mu[(size_t)n + ia] * ky + mu[(size_t)2 * n + ia] * kz) * recarg2;
                    lf[ia] = lf[ia] + kx * k_dot_mu;
                    lf[(size_t)n + ia] = lf[(size_t)n + ia] + ky * k_dot_mu;
                    lf[(size_t)2 * n + ia] = lf[(size_t)2 * n + ia] + kz * k_dot_mu;
                }
            }
            if (do_stress) {
                double kk3[3] = {kx, ky, kz};
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        lt[a * 3 + b] += ((a == b ? 1.0 : 0.0) - kcoe * kk3[a] * kk3[b]) * str;
            }
        }
        tu[t] = lu;
    }
    double usum = 0.0;
    for (int t = 0; t < nth; ++t) {
        usum += tu[t];
        if (do_efield) for (size_t i = 0; i < (size_t)3 * n; ++i) ef[i] += 2.0 * fpi_V * tef[t][i];
        if (do_efg) for (size_t i = 0; i < (size_t)9 * n; ++i) efg[i] += 2.0 * fpi_V * tefg[t][i];
        if (do_forces) for (size_t i = 0; i < (size_t)3 * n; ++i) f[i] += 2.0 * fpi_V * tf[t][i];
        if (do_stress) for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) tau[a][b] += 2.0 * ttau[(size_t)t * 9 + a * 3 + b] * tpi_V / s->cell.omega;
    }
    u_rec = usum * 2.0 * tpi_V;
}

// multipole_ES (src/field.f90:1817-2054): direct + reciprocal + self
// (+ surface), totals and units.  Forces are added to s->fx/fy/fz.
void multipole_ES(orc_sys* s, std::vector<double>& ef_out, std::vector<double>& efg_out,
                  const std::vector<double>& q, const std::vector<double>& mu, const bool task[6],
                  bool damp_ind, bool do_efield, bool do_efg, bool do_forces, bool do_stress, double& u_coul_out) {
    int n = s->natm;
    std::vector<double> ef_dir(3 * (size_t)n, 0.0), efg_dir(9 * (size_t)n, 0.0), f_dir(3 * (size_t)n, 0.0);
    std::vector<double> ef_rec(3 * (size_t)n, 0.0), efg_rec(9 * (size_t)n, 0.0), f_rec(3 * (size_t)n, 0.0);
    double tau_dir[3][3] = {{0}}, tau_rec[3][3] = {{0}};
    double mutot[3] = {0, 0, 0}, musq = 0.0, qtot[3] = {0, 0, 0}, qsq = 0.0;
    for (int ia = 0; ia < n; ++ia) {
        double m0 = mu[ia], m1 = mu[(size_t)n + ia], m2 = mu[(size_t)2 * n + ia];
        mutot[0] += m0; mutot[1] += m1; mutot[2] += m2;
        musq = musq + (m0 * m0 + m1 * m1 + m2 * m2);
        qtot[0] += q[ia] * s->rx[ia]; qtot[1] += q[ia] * s->ry[ia]; qtot[2] += q[ia] * s->rz[ia];
        qsq = qsq + q[ia] * q[ia];
    }
    double qmu_sum[3] = {qtot[0] + mutot[0], qtot[1] + mutot[1], qtot[2] + mutot[2]};
    double tpi_V = TPI / s->cell.omega, tpi_3V = tpi_V / 3.0, fpi_3V = tpi_3V * 2.0;
    double alpha2 = s->alphaES * s->alphaES;
    double selfa = s->alphaES / PIROOT;
    double selfa2 = 2.0 * selfa * alpha2 / 3.0;
    double u_dir = 0.0, u_rec = 0.0;
    multipole_ES_dir(s, q, mu, task, damp_ind, do_efield, do_efg, do_forces, do_stress, u_dir, ef_dir, efg_dir, f_dir, tau_dir);
    multipole_ES_rec(s, q, mu, task, do_efield, do_efg, do_forces, do_stress, u_rec, ef_rec, efg_rec, f_rec, tau_rec);
    double u_surf = (qtot[0] * qtot[0] + qtot[1] * qtot[1] + qtot[2] * qtot[2]) +
                    2.0 * (qtot[0] * mutot[0] + qtot[1] * mutot[1] + qtot[2] * mutot[2]) +
                    (mutot[0] * mutot[0] + mutot[1] * mutot[1] + mutot[2] * mutot[2]);
    u_surf = u_surf * tpi_3V;
    double u_self = -selfa * qsq - selfa2 * musq;
    double cu = s->u.coul;
    bool lsurf = s->p.lsurf != 0;
    double u = u_dir + u_rec + u_self + s->u_pol;
    if (lsurf) u += u_surf;
    u_coul_out = u * cu;
    ef_out.assign(3 * (size_t)n, 0.0);
    efg_out.assign(9 * (size_t)n, 0.0);
    for (int c = 0; c < 3; ++c)
        for (int ia = 0; ia < n; ++ia) {
            size_t k = (size_t)c * n + ia;
            double v = ef_dir[k] + ef_rec[k] + 2.0 * selfa2 * mu[k];
            if (lsurf) v += qmu_sum[c];
            ef_out[k] = v;
            double fv = f_rec[k] + f_dir[k];
            if (lsurf) fv += -q[ia] * qmu_sum[c] * fpi_3V;
            double* fa = c == 0 ? s->fx.data() : c == 1 ? s->fy.data() : s->fz.data();
            fa[ia] = fa[ia] + fv * cu;
        }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int ia = 0; ia < n; ++ia) {
                size_t k = (size_t)(a * 3 + b) * n + ia;
                double v = efg_dir[k] + efg_rec[k] + (a == b ? -2.0 * selfa2 * q[ia] : 0.0);
                efg_out[k] = v * cu;
            }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) s->tau_coul[a][b] = (tau_dir[a][b] + tau_rec[a][b]) * cu / s->u.press;
    s->en.u_dir = u_dir * cu;
    s->en.u_rec = u_rec * cu;
    s->en.u_self = u_self * cu;
    s->en.u_surf = lsurf ? u_surf * cu : 0.0;
    s->en.pvirial_coul = 1.0 / 3.0 * (s->tau_coul[0][0] + s->tau_coul[1][1] + s->tau_coul[2][2]) * s->u.press;
}

bool any_polar(const orc_sys* s) {
    for (int it = 0; it < s->ntype; ++it) if (s->p.ldip_polar[it]) return true;
    return false;
}

// induced_moment (src/field.f90:1716-1803), isotropic polarisabilities.
void induced_moment(orc_sys* s, const std::vector<double>& E, std::vector<double>& mu_ind, double& u_pol) {
    int n = s->natm;
    mu_ind.assign(3 * (size_t)n, 0.0);
    for (int ia = 0; ia < n; ++ia) {
        if (!s->p.ldip_polar[s->itype[ia]]) continue;
        for (int a = 0; a < 3; ++a) mu_ind[(size_t)a * n + ia] = s->poldia[ia] * E[(size_t)a * n + ia];
    }
    double up = 0.0;
    for (int ia = 0; ia < n; ++ia) {
        if (!s->p.ldip_polar[s->itype[ia]]) continue;
        for (int a = 0; a < 3; ++a) up = up + mu_ind[(size_t)a * n + ia] * s->invpoldia[ia] * mu_ind[(size_t)a * n + ia];
    }
    u_pol = up * 0.5;
}

// polint (src/field.f90:3995-4042): Neville interpolation evaluated at x = 1.
double polint(const int* xa, const double* ya, int n, double& dy) {
    double c[16], d[16];
    int ns = 1;
    double dif = std::fabs(1.0 - xa[0]);
    for (int i = 1; i <= n; ++i) {
        double dift = std::fabs(1.0 - xa[i - 1]);
        if (dift < dif) { ns = i; dif = dift; }
        c[i - 1] = ya[i - 1]; d[i - 1] = ya[i - 1];
    }
    double y = ya[ns - 1];
    ns = ns - 1;
    for (int m = 1; m <= n - 1; ++m) {
        for (int i = 1; i <= n - m; ++i) {
            double ho = double(xa[i - 1] - 1), hp = double(xa[i] - 1);
            double w = c[i] - d[i - 1];
            double den = ho - hp;
            den = w / den;
            d[i - 1] = hp * den;
            c[i - 1] = ho * den;
        }
        if (2 * ns < n - m) dy = c[ns];
        else { dy = d[ns - 1]; ns = ns - 1; }
        y = y + dy;
    }
    return y;
}

inline double& HIST(orc_sys* s, int t, int c, int ia) { return s->dip_hist[((size_t)t * 3 + c) * s->natm + ia]; }

// extrapolate_dipole_poly (src/field.f90:3807-3920)
void extrapolate_poly(orc_sys* s, std::vector<double>& mu_ind) {
    int n = s->natm, ord = s->p.extrapolate_order, itime = s->itime;
    mu_ind.assign(3 * (size_t)n, 0.0);
    auto shift = [&]() { for (int ie = ord; ie >= 1; --ie) for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) HIST(s, ie, c, ia) = HIST(s, ie - 1, c, ia); };
    if (ord == 0)
        for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) mu_ind[(size_t)c * n + ia] = HIST(s, 0, c, ia);
    if (ord == 1 && itime > ord) {
        for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) mu_ind[(size_t)c * n + ia] = 2.0 * HIST(s, 0, c, ia) - HIST(s, 1, c, ia);
        for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) HIST(s, 1, c, ia) = HIST(s, 0, c, ia);
    } else if (ord == 1 && itime <= ord) {
        for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) { mu_ind[(size_t)c * n + ia] = HIST(s, 0, c, ia); HIST(s, 1, c, ia) = HIST(s, 0, c, ia); }
    }
    if (ord >= 2 && itime > ord) {
        int xa[16];
        for (int t = 1; t <= ord + 1; ++t) xa[t - 1] = 1 - t;
        double ya[16], err;
        for (int ia = 0; ia < n; ++ia)
            for (int c = 0; c < 3; ++c) {
                for (int t = 0; t <= ord; ++t) ya[t] = HIST(s, t, c, ia);
                mu_ind[(size_t)c * n + ia] = polint(xa, ya, ord + 1, err);
            }
        shift();
    } else if (ord >= 2 && itime <= ord) {
        if (itime <= 1)
            for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) mu_ind[(size_t)c * n + ia] = HIST(s, 0, c, ia);
        if (itime == 2)
            for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) mu_ind[(size_t)c * n + ia] = 2.0 * HIST(s, 0, c, ia) - HIST(s, 1, c, ia);
        if (itime > 2) {
            int xa[16];
            for (int t = 1; t <= itime + 1; ++t) xa[t - 1] = 1 - t;
            double ya[16], err;
            for (int ia = 0; ia < n; ++ia)
                for (int c = 0; c < 3; ++c) {
                    for (int t = 0; t <= itime; ++t) ya[t] = HIST(s, t, c, ia);
                    mu_ind[(size_t)c * n + ia] = polint(xa, ya, itime + 1, err);
                }
        }
        shift();
    }
}

// ASPC coefficients (src/field.f90:3931-3968), Kolafa's always-stable predictor-corrector.
void aspc_coeffs(int ord, double B[6], double& w) {
    for (int i = 0; i < 6; ++i) B[i] = 0.0;
    switch (ord) {
        case 0: B[0] = 1.0; w = 0.0; break;
        case 1: B[0] = 2.0; B[1] = -1.0; w = 2.0 / 3.0; break;
        case 2: B[0] = 2.5; B[1] = -2.0; B[2] = 0.5; w = 0.6; break;
        case 3: B[0] = 2.8; B[1] = -2.8; B[2] = 1.2; B[3] = -0.2; w = 4.0 / 7.0; break;
        case 4: B[0] = 3.0; B[1] = -24.0 / 7.0; B[2] = 27.0 / 14.0; B[3] = -4.0 / 7.0; B[4] = 1.0 / 14.0; w = 5.0 / 9.0; break;
        default: B[0] = 22.0 / 7.0; B[1] = -55.0 / 14.0; B[2] = 55.0 / 21.0; B[3] = -22.0 / 21.0; B[4] = 5.0 / 21.0; B[5] = -1.0 / 42.0; w = 6.0 / 11.0; break;
    }
}

int aspc_order(const orc_sys* s) {
    int ord = s->p.extrapolate_order, itime = s->itime;
    if (itime >= ord + 1) return ord;
    if (itime == 1 || itime == 0) return 0;
    return itime - 1;
}

// SCF rmsd (src/field.f90:3378-3400)
double scf_rmsd(orc_sys* s, const std::vector<double>& mu_ind, const std::vector<double>& E) {
    int n = s->natm;
    double r = 0.0;
    int npol = 0;
    for (int ia = 0; ia < n; ++ia) {
        if (!s->p.ldip_polar[s->itype[ia]]) continue;
        npol++;
        for (int a = 0; a < 3; ++a) {
            if (s->poldia[ia] == 0.0) continue;
            double t = mu_ind[(size_t)a * n + ia] / s->poldia[ia] - E[(size_t)a * n + ia];
            r = r + t * t;
        }
    }
    return std::sqrt(r / double(npol));
}

// Induced field operator: E_ind(mu) = multipole_ES with the induced dipoles
// only, dipole-dipole task, no damping (src/field.f90:3354-3357).
void induced_field(orc_sys* s, const std::vector<double>& mu_ind, std::vector<double>& E_ind) {
    int n = s->natm;
    std::vector<double> zq(n, 0.0), efg;
    bool task_ind[6] = {false, false, true, false, false, false};
    std::vector<double> fx = s->fx, fy = s->fy, fz = s->fz;
    double tn[3][3]; std::memcpy(tn, s->tau_coul, sizeof tn);
    double uc;
    multipole_ES(s, E_ind, efg, zq, mu_ind, task_ind, false, true, false, false, false, uc);
    s->fx = fx; s->fy = fy; s->fz = fz;
    std::memcpy(s->tau_coul, tn, sizeof tn);
}

// moment_from_pola_scf (src/field.f90:3200-3458); with MDFF_POLA_PCG the same
// linear system (1/alpha - T) mu = E_stat is solved by Jacobi-preconditioned CG.
void moment_from_pola(orc_sys* s, std::vector<double>& mu_ind) {
    int n = s->natm;
    const mdff_params& p = s->p;
    mu_ind.assign(3 * (size_t)n, 0.0);
    if (!any_polar(s)) return;
    // static field from charges (and static dipoles), damped
    std::vector<double> Estat, efg;
    bool task_static[6] = {true, false, false, false, false, false};
    bool ldip = false;
    for (int it = 0; it < s->ntype; ++it) for (int c = 0; c < 3; ++c) if (p.dip[it][c] != 0.0) ldip = true;
    if (ldip) { task_static[1] = true; task_static[2] = true; }
    std::vector<double> dipia(3 * (size_t)n);
    for (int ia = 0; ia < n; ++ia) { dipia[ia] = s->dipx[ia]; dipia[(size_t)n + ia] = s->dipy[ia]; dipia[(size_t)2 * n + ia] = s->dipz[ia]; }
    {
        std::vector<double> fx = s->fx, fy = s->fy, fz = s->fz;
        double uc;
        multipole_ES(s, Estat, efg, s->qia, dipia, task_static, true, true, false, false, false, uc);
        s->fx = fx; s->fy = fy; s->fz = fz;
    }
    std::vector<double> E = Estat, Eind(3 * (size_t)n, 0.0);
    int iscf = 0;
    double rmsd = 1e300;
    if (p.algo_moment_from_pola == MDFF_POLA_SCF) {
        std::vector<double> mu_p_save;
        while (((iscf < p.max_scf_pol_iter) && (rmsd > p.conv_tol_ind)) || (iscf < p.min_scf_pol_iter)) {
            iscf++;
            if (iscf != 1) {
                induced_moment(s, E, mu_ind, s->u_pol);
            } else {
                if (p.algo_ext_dipole == MDFF_EXT_POLY) extrapolate_poly(s, mu_ind);
                else {
                    int eo = aspc_order(s);
                    double B[6], w;
                    aspc_coeffs(eo, B, w);
                    mu_ind.assign(3 * (size_t)n, 0.0);
                    for (int k = 0; k <= eo; ++k)
                        for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) mu_ind[(size_t)c * n + ia] += B[k] * HIST(s, k, c, ia);
                    for (int k = eo; k >= 1; --k)
                        for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) HIST(s, k, c, ia) = HIST(s, k - 1, c, ia);
                }
            }
            induced_field(s, mu_ind, Eind);
            for (size_t k = 0; k < E.size(); ++k) E[k] = Estat[k] + Eind[k];
            if (iscf == 1 && p.algo_ext_dipole == MDFF_EXT_ASPC) {   // corrector (field.f90:3987-3991)
                int eo = aspc_order(s);
                double B[6], w;
                aspc_coeffs(eo, B, w);
                mu_p_save = mu_ind;
                induced_moment(s, E, mu_ind, s->u_pol);
                for (size_t k = 0; k < mu_ind.size(); ++k) mu_ind[k] = w * mu_ind[k] + (1.0 - w) * mu_p_save[k];
            }
            rmsd = scf_rmsd(s, mu_ind, E);
        }
    } else {
        // PCG on the polarisable atoms.  A mu = (1/alpha) mu - E_ind(mu), b = E_stat.
        std::vector<double> x;
        if (p.algo_ext_dipole == MDFF_EXT_POLY) extrapolate_poly(s, x);
        else {
            int eo = aspc_order(s);
            double B[6], w;
            aspc_coeffs(eo, B, w);
            x.assign(3 * (size_t)n, 0.0);
            for (int k = 0; k <= eo; ++k)
                for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) x[(size_t)c * n + ia] += B[k] * HIST(s, k, c, ia);
            for (int k = eo; k >= 1; --k)
                for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) HIST(s, k, c, ia) = HIST(s, k - 1, c, ia);
        }
        std::vector<char> pol(n, 0);
        int npol = 0;
        for (int ia = 0; ia < n; ++ia) if (p.ldip_polar[s->itype[ia]] && s->poldia[ia] != 0.0) { pol[ia] = 1; npol++; }
        for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) if (!pol[ia]) x[(size_t)c * n + ia] = 0.0;
        auto apply = [&](const std::vector<double>& v, std::vector<double>& out) {
            induced_field(s, v, Eind);
            out.assign(3 * (size_t)n, 0.0);
            for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia)
                if (pol[ia]) out[(size_t)c * n + ia] = v[(size_t)c * n + ia] * s->invpoldia[ia] - Eind[(size_t)c * n + ia];
        };
        std::vector<double> r(3 * (size_t)n), z(3 * (size_t)n), d(3 * (size_t)n), Ad;
        apply(x, Ad);
        for (size_t k = 0; k < r.size(); ++k) r[k] = pol[k % n] ? Estat[k] - Ad[k] : 0.0;
        // Jacobi preconditioner: diagonal of A = 1/alpha - (self-field coefficient)
        double selfc = 2.0 * (2.0 * s->alphaES / PIROOT * s->alphaES * s->alphaES / 3.0);
        auto prec = [&](const std::vector<double>& in, std::vector<double>& out) {
            for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) {
                size_t k = (size_t)c * n + ia;
                out[k] = pol[ia] ? in[k] / (s->invpoldia[ia] - selfc) : 0.0;
            }
        };
        auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) { double t = 0; for (size_t k = 0; k < a.size(); ++k) t += a[k] * b[k]; return t; };
        prec(r, z);
        d = z;
        double rz = dot(r, z);
        rmsd = std::sqrt(dot(r, r) / double(npol));
        while ((iscf < p.max_scf_pol_iter && rmsd > p.conv_tol_ind) || iscf < 1) {
            iscf++;
            apply(d, Ad);
            double alpha = rz / dot(d, Ad);
            for (size_t k = 0; k < x.size(); ++k) { x[k] += alpha * d[k]; r[k] -= alpha * Ad[k]; }
            rmsd = std::sqrt(dot(r, r) / double(npol));
            prec(r, z);
            double rz2 = dot(r, z);
            double beta = rz2 / rz;
            rz = rz2;
            for (size_t k = 0; k < d.size(); ++k) d[k] = z[k] + beta * d[k];
        }
        mu_ind = x;
        // u_pol from the final iterate (induced_moment form)
        double up = 0.0;
        for (int ia = 0; ia < n; ++ia) if (pol[ia]) for (int c = 0; c < 3; ++c) up += mu_ind[(size_t)c * n + ia] * s->invpoldia[ia] * mu_ind[(size_t)c * n + ia];
        s->u_pol = 0.5 * up;
    }
    for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia) HIST(s, 0, c, ia) = mu_ind[(size_t)c * n + ia];
    s->en.scf_iter = iscf;
    s->en.scf_rmsd = rmsd;
}

// engforce_driver (src/field.f90:1111-1166) with D4 (forces summed).
void engforce(orc_sys* s) {
    int n = s->natm;
    std::fill(s->fx.begin(), s->fx.end(), 0.0);
    std::fill(s->fy.begin(), s->fy.end(), 0.0);
    std::fill(s->fz.begin(), s->fz.end(), 0.0);
    std::memset(s->tau_nonb, 0, sizeof s->tau_nonb);
    std::memset(s->tau_coul, 0, sizeof s->tau_coul);
    mdff_energies e0;
    std::memset(&e0, 0, sizeof e0);
    s->en = e0;
    s->en.utail = s->utail;
    s->en.ptail = s->ptail;
    std::vector<double> sx, sy, sz;
    direct_coords(s, sx, sy, sz);
    if (s->p.lnmlj) engforce_nmlj(s, sx, sy, sz);
    if (s->p.lbmhftd || s->p.lbmhft) engforce_bmhftd(s, sx, sy, sz);
    if (s->p.lmorse) engforce_morse(s, sx, sy, sz);
    if (s->p.lcoulomb) {
        std::vector<double> mu_ind;
        moment_from_pola(s, mu_ind);   // get_moments (field.f90:3686-3765)
        s->mu.assign(3 * (size_t)n, 0.0);
        for (int ia = 0; ia < n; ++ia) {
            s->mu[ia] = s->dipx[ia] + mu_ind[ia];
            s->mu[(size_t)n + ia] = s->dipy[ia] + mu_ind[(size_t)n + ia];
            s->mu[(size_t)2 * n + ia] = s->dipz[ia] + mu_ind[(size_t)2 * n + ia];
        }
        bool task[6] = {false, false, false, false, false, false};
        bool lqch = false, ldipt = false;
        for (int it = 0; it < s->ntype; ++it) {
            if (s->p.qch[it] != 0.0) lqch = true;
            for (int c = 0; c < 3; ++c) if (s->p.dip[it][c] != 0.0) ldipt = true;
            if (s->p.ldip_polar[it]) ldipt = true;
        }
        if (lqch) task[0] = true;
        if (ldipt) { if (lqch) task[1] = true; task[2] = true; }
        double uc;
        multipole_ES(s, s->ef, s->efg, s->qia, s->mu, task, true, s->p.doefield != 0, s->p.doefg != 0, true, true, uc);
        s->en.u_coul = uc;
        s->en.u_pol = s->u_pol * s->u.coul;
    }
}

// calc_temp (src/kinetic.f90:531-560)
void calc_temp(orc_sys* s, double& T, double& ekin) {
    double L = 3.0 * double(s->natm);
    ekin = 0.0;
    for (int ia = 0; ia < s->natm; ++ia)
        ekin = ekin + (s->vx[ia] * s->vx[ia] + s->vy[ia] * s->vy[ia] + s->vz[ia] * s->vz[ia]) * s->massia[ia];
    ekin = ekin * 0.5;
    T = 2.0 * ekin / s->u.boltz;
    T = T / L;
}

// chain_nhcn (src/integration.f90:564-713), trotter_order = -1 branch.
void chain_nhcn(orc_sys* s, double& kin, const std::vector<double>& Q, double L) {
    const mdff_params& p = s->p;
    int nhc = p.nhc_n;
    double yw[9] = {0};
    switch (p.nhc_yosh_order) {
        case 1: yw[0] = 1.0; break;
        case 3: yw[0] = 1.0 / (2.0 - std::pow(2.0, 1.0 / 3.0)); yw[1] = 1.0 - 2.0 * yw[0]; yw[2] = yw[0]; break;
        case 5: yw[0] = 1.0 / (4.0 - std::pow(4.0, 1.0 / 3.0)); yw[1] = yw[0]; yw[2] = yw[0]; yw[3] = yw[0]; yw[4] = 1.0 - 4.0 * yw[0]; break;
        case 7:
            yw[0] = .78451361047756; yw[1] = .235573213359357; yw[2] = -1.17767998417887;
            yw[3] = 1.0 - 2.0 * (yw[0] + yw[1] + yw[2]); yw[4] = yw[2]; yw[5] = yw[1]; yw[6] = yw[0]; break;
        default:
            yw[0] = 0.192; yw[1] = 0.554910818409783619692725006662999; yw[2] = 0.124659619941888644216504240951585;
            yw[3] = -0.843182063596933505315033808282941; yw[4] = 1.0 - 2.0 * (yw[0] + yw[1] + yw[2] + yw[3]);
            yw[5] = yw[3]; yw[6] = yw[2]; yw[7] = yw[1]; yw[8] = yw[0]; break;
    }
    std::vector<double> G(nhc, 0.0);
    std::vector<double>& vxi = s->vxi;
    std::vector<double>& xi = s->xi;
    double temp = s->temp;
    double sc = 1.0;
    G[0] = 2.0 * kin - L * temp;
    for (int k = 0; k < p.nhc_mults; ++k) {
        for (int j = 0; j < p.nhc_yosh_order; ++j) {
            double dts = yw[j] * s->dt / double(p.nhc_mults);
            double dts2 = dts * 0.5, dts4 = dts2 * 0.5, dts8 = dts4 * 0.5;
            G[nhc - 1] = (vxi[nhc - 2] * vxi[nhc - 2] / Q[nhc - 2] - temp);
            if (!p.nhc_literal)   // D13: refresh the inner chain forces before the downward pass
                for (int inh = 1; inh < nhc - 1; ++inh) G[inh] = vxi[inh - 1] * vxi[inh - 1] / Q[inh - 1] - temp;
            vxi[nhc - 1] = vxi[nhc - 1] + G[nhc - 1] * dts4;
            for (int inh = nhc - 2; inh >= 0; --inh) {
                vxi[inh] = vxi[inh] * std::exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                vxi[inh] = vxi[inh] + G[inh] * dts4;
                vxi[inh] = vxi[inh] * std::exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
            }
            sc = sc * std::exp(-vxi[0] * dts2 / Q[0]);
            for (int inh = 0; inh < nhc; ++inh) xi[inh] = xi[inh] + vxi[inh] * dts2 / Q[inh];
            G[0] = 2.0 * kin * sc * sc - L * temp;
            for (int inh = 0; inh < nhc - 1; ++inh) {
                vxi[inh] = vxi[inh] * std::exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                vxi[inh] = vxi[inh] + G[inh] * dts4;
                vxi[inh] = vxi[inh] * std::exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                G[inh + 1] = (vxi[inh] * vxi[inh] / Q[inh] - temp);
            }
            vxi[nhc - 1] = vxi[nhc - 1] + G[nhc - 1] * dts4;
        }
    }
    kin = 0.0;
    for (int ia = 0; ia < s->natm; ++ia) {
        s->vx[ia] = sc * s->vx[ia];
        s->vy[ia] = sc * s->vy[ia];
        s->vz[ia] = sc * s->vz[ia];
        kin = kin + (s->vx[ia] * s->vx[ia] + s->vy[ia] * s->vy[ia] + s->vz[ia] * s->vz[ia]) * s->massia[ia];
    }
    kin = kin * 0.5;
}

// prop_velocity_verlet (src/integration.f90:131-194)
void prop_velocity_verlet(orc_sys* s) {
    int n = s->natm;
    std::vector<double> fsx = s->fx, fsy = s->fy, fsz = s->fz;
    double dt = s->dt, dtsq2 = dt * dt * 0.5, dt2 = dt * 0.5;
    for (int ia = 0; ia < n; ++ia) {
        s->rx[ia] = s->rx[ia] + s->vx[ia] * dt + (s->fx[ia] * dtsq2) / s->massia[ia];
        s->ry[ia] = s->ry[ia] + s->vy[ia] * dt + (s->fy[ia] * dtsq2) / s->massia[ia];
        s->rz[ia] = s->rz[ia] + s->vz[ia] * dt + (s->fz[ia] * dtsq2) / s->massia[ia];
    }
    engforce(s);
    for (int ia = 0; ia < n; ++ia) {
        s->vx[ia] = s->vx[ia] + (fsx[ia] + s->fx[ia]) * dt2 / s->massia[ia];
        s->vy[ia] = s->vy[ia] + (fsy[ia] + s->fy[ia]) * dt2 / s->massia[ia];
        s->vz[ia] = s->vz[ia] + (fsz[ia] + s->fz[ia]) * dt2 / s->massia[ia];
    }
    calc_temp(s, s->temp_r, s->e_kin);
}

// prop_pos_vel_verlet (src/integration.f90:333-385)
void prop_pos_vel_verlet(orc_sys* s, double& kin) {
    int n = s->natm;
    double dt = s->dt, dt2 = dt * 0.5;
    for (int ia = 0; ia < n; ++ia) {
        s->vx[ia] = s->vx[ia] + s->fx[ia] * dt2 / s->massia[ia];
        s->vy[ia] = s->vy[ia] + s->fy[ia] * dt2 / s->massia[ia];
        s->vz[ia] = s->vz[ia] + s->fz[ia] * dt2 / s->massia[ia];
        s->rx[ia] = s->rx[ia] + s->vx[ia] * dt;
        s->ry[ia] = s->ry[ia] + s->vy[ia] * dt;
        s->rz[ia] = s->rz[ia] + s->vz[ia] * dt;
    }
    engforce(s);
    kin = 0.0;
    for (int ia = 0; ia < n; ++ia) {
        s->vx[ia] = s->vx[ia] + s->fx[ia] * dt2 / s->massia[ia];
        s->vy[ia] = s->vy[ia] + s->fy[ia] * dt2 / s->massia[ia];
        s->vz[ia] = s->vz[ia] + s->fz[ia] * dt2 / s->massia[ia];
        kin = kin + (s->vx[ia] * s->vx[ia] + s->vy[ia] * s->vy[ia] + s->vz[ia] * s->vz[ia]) * s->massia[ia];
    }
    kin = kin * 0.5;
}

// nhcn (src/integration.f90:476-558)
void nhcn(orc_sys* s) {
    const mdff_params& p = s->p;
    double L = 3.0 * double(s->natm);
    std::vector<double> Q(p.nhc_n, s->timesca * s->timesca * s->temp);
    Q[0] = Q[0] * L;
    double tempi, kin;
    calc_temp(s, tempi, kin);
    chain_nhcn(s, kin, Q, L);
    prop_pos_vel_verlet(s, kin);
    chain_nhcn(s, kin, Q, L);
    calc_temp(s, s->temp_r, s->e_kin);
    double nvt1 = L * s->temp * s->xi[0];
    double nvt2 = s->vxi[0] * s->vxi[0] * 0.5 / Q[0];
    double nvt3 = 0.0, nvt4 = 0.0;
    for (int inhc = 1; inhc < p.nhc_n; ++inhc) {
        nvt3 = nvt3 + s->vxi[inhc] * s->vxi[inhc] * 0.5 / Q[inhc];
        nvt4 = nvt4 + s->temp * s->xi[inhc];
    }
    s->e_nvt = nvt1 + nvt2 + nvt3 + nvt4;
}

// chain_nhc2 (src/integration.f90:265-324): Frenkel and Smit's two-thermostat
// chain; vxi are thermostat velocities; kin is updated to s^2 kin inside and
// the velocities are scaled by s at the end.
void chain_nhc2(orc_sys* s, double& kin, const double Q[2], double L) {
    std::vector<double>& vxi = s->vxi;
    std::vector<double>& xi = s->xi;
    const double temp = s->temp;
    double sc = 1.0;
    const double dt2 = s->dt * 0.5, dt4 = dt2 * 0.5, dt8 = dt4 * 0.5;
    double G1 = (2.0 * kin - L * temp) / Q[0];
    double G2 = (Q[0] * vxi[0] * vxi[0] - temp) / Q[1];
    vxi[1] = vxi[1] + G2 * dt4;
    vxi[0] = vxi[0] * std::exp(-vxi[1] * dt8);
    vxi[0] = vxi[0] + G1 * dt4;
    vxi[0] = vxi[0] * std::exp(-vxi[1] * dt8);
    sc = sc * std::exp(-vxi[0] * dt2);
    kin = sc * sc * kin;
    xi[0] = xi[0] + vxi[0] * dt2;
    xi[1] = xi[1] + vxi[1] * dt2;
    G1 = (2.0 * kin - L * temp) / Q[0];
    vxi[0] = vxi[0] * std::exp(-vxi[1] * dt8);
    vxi[0] = vxi[0] + G1 * dt4;
    vxi[0] = vxi[0] * std::exp(-vxi[1] * dt8);
    G2 = (Q[0] * vxi[0] * vxi[0] - temp) / Q[1];
    vxi[1] = vxi[1] + G2 * dt4;
    for (int ia = 0; ia < s->natm; ++ia) {
        s->vx[ia] = sc * s->vx[ia];
        s->vy[ia] = sc * s->vy[ia];
        s->vz[ia] = sc * s->vz[ia];
    }
}

// nhc2 (src/integration.f90:205-254): L = 3 (natm - 1), Q(1) = tau^2 T L,
// Q(2) = tau^2 T.  The thermostat energy uses Q vxi^2 / 2, the kinetic
// energy of the velocities vxi (D23: the reference writes vxi^2 / (2 Q), the
// momentum form of nhcn, which is not conserved here); nhc_literal = 1
// restores the reference's expression.
void nhc2(orc_sys* s) {
    const double L = 3.0 * (double(s->natm) - 1.0);
    const double Q[2] = {s->timesca * s->timesca * s->temp * L, s->timesca * s->timesca * s->temp};
    double tempi, kin;
    calc_temp(s, tempi, kin);
    chain_nhc2(s, kin, Q, L);
    prop_pos_vel_verlet(s, kin);
    chain_nhc2(s, kin, Q, L);
    calc_temp(s, s->temp_r, s->e_kin);
    const bool lit = s->p.nhc_literal != 0;
    double e = L * s->temp * s->xi[0];
    e = e + (lit ? s->vxi[0] * s->vxi[0] * 0.5 / Q[0] : Q[0] * s->vxi[0] * s->vxi[0] * 0.5);
    e = e + (lit ? s->vxi[1] * s->vxi[1] * 0.5 / Q[1] : Q[1] * s->vxi[1] * s->vxi[1] * 0.5);
    e = e + s->temp * s->xi[1];
    s->e_nvt = e;
}

// A new cell for the same atoms (D14): lattice, tail corrections and k mesh.
void set_cell(orc_sys* s, const double A[3][3]) {
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) s->cell.A[i][j] = A[i][j];
    lattice(s->cell);
    const double r = s->omega0 / s->cell.omega;
    s->utail = s->utail0 * r;
    s->ptail = s->ptail0 * r * r;
    if (s->p.lcoulomb) kpoint_sum_init(s);
}

// chain_nhcnp (src/integration.f90:724-964), one half: first = barostat chain
// then particle chain (trotter order -1), else particle then barostat (+1);
// D13 and D16 as in the header.  Velocities scaled by s, ve by sb; kin
// recomputed from the scaled velocities.
void chain_nhcnp(orc_sys* s, double& kin, const std::vector<double>& Q, const std::vector<double>& Qb, double W,
                 double L, bool first) {
    const mdff_params& p = s->p;
    const int nhc = p.nhc_n;
    double yw[9] = {0};
    switch (p.nhc_yosh_order) {
        case 1: yw[0] = 1.0; break;
        case 3: yw[0] = 1.0 / (2.0 - std::pow(2.0, 1.0 / 3.0)); yw[1] = 1.0 - 2.0 * yw[0]; yw[2] = yw[0]; break;
        case 5: yw[0] = 1.0 / (4.0 - std::pow(4.0, 1.0 / 3.0)); yw[1] = yw[0]; yw[2] = yw[0]; yw[3] = yw[0]; yw[4] = 1.0 - 4.0 * yw[0]; break;
        case 7:
            yw[0] = .78451361047756; yw[1] = .235573213359357; yw[2] = -1.17767998417887;
            yw[3] = 1.0 - 2.0 * (yw[0] + yw[1] + yw[2]); yw[4] = yw[2]; yw[5] = yw[1]; yw[6] = yw[0]; break;
        default:
            yw[0] = 0.192; yw[1] = 0.554910818409783619692725006662999; yw[2] = 0.124659619941888644216504240951585;
            yw[3] = -0.843182063596933505315033808282941; yw[4] = 1.0 - 2.0 * (yw[0] + yw[1] + yw[2] + yw[3]);
            yw[5] = yw[3]; yw[6] = yw[2]; yw[7] = yw[1]; yw[8] = yw[0]; break;
    }
    const double temp = s->temp;
    std::vector<double> G(nhc, 0.0), Gb(nhc, 0.0);
    double sc = 1.0, sb = 1.0;
    G[0] = 2.0 * kin - L * temp;
    Gb[0] = s->ve * s->ve / W - temp;
    // one Trotter piece of a chain (src/integration.f90:830-877)
    auto piece = [&](std::vector<double>& v, std::vector<double>& x, const std::vector<double>& q,
                     std::vector<double>& g, double& f, bool baro, double dts) {
        double dts2 = dts * 0.5, dts4 = dts2 * 0.5, dts8 = dts4 * 0.5;
        g[nhc - 1] = v[nhc - 2] * v[nhc - 2] / q[nhc - 2] - temp;
        if (!p.nhc_literal)
            for (int inh = 1; inh < nhc - 1; ++inh) g[inh] = v[inh - 1] * v[inh - 1] / q[inh - 1] - temp;
        v[nhc - 1] = v[nhc - 1] + g[nhc - 1] * dts4;
        for (int inh = nhc - 2; inh >= 0; --inh) {
            v[inh] = v[inh] * std::exp(-v[inh + 1] * dts8 / q[inh + 1]);
            v[inh] = v[inh] + g[inh] * dts4;
            v[inh] = v[inh] * std::exp(-v[inh + 1] * dts8 / q[inh + 1]);
        }
        f = f * std::exp(-v[0] * dts2 / q[0]);
        for (int inh = 0; inh < nhc; ++inh) x[inh] = x[inh] + v[inh] * dts2 / q[inh];
        g[0] = baro ? s->ve * s->ve * f * f / W - temp : 2.0 * kin * f * f - L * temp;
        for (int inh = 0; inh < nhc - 1; ++inh) {
            v[inh] = v[inh] * std::exp(-v[inh + 1] * dts8 / q[inh + 1]);
            v[inh] = v[inh] + g[inh] * dts4;
            v[inh] = v[inh] * std::exp(-v[inh + 1] * dts8 / q[inh + 1]);
            g[inh + 1] = v[inh] * v[inh] / q[inh] - temp;
        }
        v[nhc - 1] = v[nhc - 1] + g[nhc - 1] * dts4;
    };
    for (int k = 0; k < p.nhc_mults; ++k)
        for (int j = 0; j < p.nhc_yosh_order; ++j) {
            double dts = yw[j] * s->dt / double(p.nhc_mults);
            if (first) {
                piece(s->vxib, s->xib, Qb, Gb, sb, true, dts);
                piece(s->vxi, s->xi, Q, G, sc, false, dts);
            } else {
                piece(s->vxi, s->xi, Q, G, sc, false, dts);
                piece(s->vxib, s->xib, Qb, Gb, sb, true, dts);
            }
        }
    kin = 0.0;
    for (int ia = 0; ia < s->natm; ++ia) {
        s->vx[ia] = sc * s->vx[ia];
        s->vy[ia] = sc * s->vy[ia];
        s->vz[ia] = sc * s->vz[ia];
        kin = kin + (s->vx[ia] * s->vx[ia] + s->vy[ia] * s->vy[ia] + s->vz[ia] * s->vz[ia]) * s->massia[ia];
    }
    kin = kin * 0.5;
    s->ve = s->ve * sb;
}

// nhcnp (src/integration.f90:966-1042) with prop_pos_vel_verlet_npt
// (:1049-1160); D15, D17: ve += Ge dt/2 after the first chain half and before
// the second, Ge = 3V ((1 + 3/L) 2K / 3V + pvirial - press).
void nhcnp(orc_sys* s) {
    const mdff_params& p = s->p;
    const double L = 3.0 * double(s->natm);
    std::vector<double> Q(p.nhc_n, s->timesca * s->timesca * s->temp), Qb(p.nhc_n);
    Q[0] = Q[0] * L;
    const double tb = p.timesca_baro * s->u.time;
    for (int k = 0; k < p.nhc_n; ++k) Qb[k] = tb * tb * s->temp;
    Qb[0] = Qb[0] * 9.0;
    const double W = (L + 1.0) * tb * tb * s->temp;
    const double press = p.press * s->u.press;
    const double odnf = 1.0 + 3.0 / L, dt = s->dt, dt2 = dt * 0.5, dt4 = dt2 * 0.5;
    auto pvirial = [&]() { return (s->en.vir_lj + s->en.vir_morse + s->en.vir_bmhft) / s->cell.omega + s->en.pvirial_coul; };
    auto kick_ve = [&](double kin) {
        double P_kin = odnf * 2.0 * kin / (3.0 * s->cell.omega);
        double Ge = 3.0 * s->cell.omega * (P_kin + pvirial() - press);
        s->ve = s->ve + Ge * dt2;
    };
    auto poly = [](double arg) {
        const double e2 = 1.0 / 6.0, e4 = e2 / 20.0, e6 = e4 / 42.0, e8 = e6 / 72.0;
        double a2 = arg * arg;
        return (((e8 * a2 + e6) * a2 + e4) * a2 + e2) * a2 + 1.0;
    };
    double tempi, kin;
    calc_temp(s, tempi, kin);
    chain_nhcnp(s, kin, Q, Qb, W, L, true);
    kick_ve(kin);
    double arg = odnf * s->ve * dt4 / W;
    double aa = std::exp(-arg), AA2 = aa * aa, BB = aa * dt2 * poly(arg);
    for (int ia = 0; ia < s->natm; ++ia) {
        s->vx[ia] = s->vx[ia] * AA2 + s->fx[ia] * BB / s->massia[ia];
        s->vy[ia] = s->vy[ia] * AA2 + s->fy[ia] * BB / s->massia[ia];
        s->vz[ia] = s->vz[ia] * AA2 + s->fz[ia] * BB / s->massia[ia];
    }
    s->xe = s->xe + s->ve * dt / W;
    const double g = std::exp(s->xe - s->xe0);
    double A[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = s->cell.A[i][j] * g;
    s->xe0 = s->xe;
    s->scale = s->scale * g;
    set_cell(s, A);
    arg = s->ve * dt2 / W;
    aa = std::exp(arg);
    AA2 = aa * aa;
    BB = aa * poly(arg) * dt;
    for (int ia = 0; ia < s->natm; ++ia) {
        s->rx[ia] = s->rx[ia] * AA2 + s->vx[ia] * BB;
        s->ry[ia] = s->ry[ia] * AA2 + s->vy[ia] * BB;
        s->rz[ia] = s->rz[ia] * AA2 + s->vz[ia] * BB;
    }
    engforce(s);
    arg = odnf * s->ve * dt4 / W;
    aa = std::exp(-arg);
    AA2 = aa * aa;
    BB = aa * poly(arg) * dt2;
    kin = 0.0;
    for (int ia = 0; ia < s->natm; ++ia) {
        s->vx[ia] = s->vx[ia] * AA2 + s->fx[ia] * BB / s->massia[ia];
        s->vy[ia] = s->vy[ia] * AA2 + s->fy[ia] * BB / s->massia[ia];
        s->vz[ia] = s->vz[ia] * AA2 + s->fz[ia] * BB / s->massia[ia];
        kin = kin + (s->vx[ia] * s->vx[ia] + s->vy[ia] * s->vy[ia] + s->vz[ia] * s->vz[ia]) * s->massia[ia];
    }
    kin = kin * 0.5;
    kick_ve(kin);
    chain_nhcnp(s, kin, Q, Qb, W, L, false);
    calc_temp(s, s->temp_r, s->e_kin);
    double e = press * s->cell.omega + s->ve * s->ve * 0.5 / W + L * s->temp * s->xi[0] + s->temp * s->xib[0] +
               s->vxi[0] * s->vxi[0] * 0.5 / Q[0] + s->vxib[0] * s->vxib[0] * 0.5 / Qb[0];
    for (int k = 1; k < p.nhc_n; ++k)
        e = e + s->vxi[k] * s->vxi[k] * 0.5 / Q[k] + s->vxib[k] * s->vxib[k] * 0.5 / Qb[k] + s->temp * s->xi[k] +
            s->temp * s->xib[k];
    s->e_npt = e;
}

// calc_thermo (src/thermo.f90:116-207), non-reduced output path.
void calc_thermo(orc_sys* s, mdff_thermo* t, int step) {
    double omega = s->cell.omega;
    double nr = s->p.lreduced ? double(s->natm) : 1.0;
    t->step = step;
    t->e_kin = s->e_kin / nr;
    t->temp_r = s->temp_r;
    t->u_lj = s->en.u_lj / nr; t->u_bmhft = s->en.u_bmhft / nr; t->u_morse = s->en.u_morse / nr;
    t->u_coul = s->en.u_coul / nr; t->u_pol = s->en.u_pol / nr;
    t->u_tot = t->u_lj + t->u_coul + t->u_morse + t->u_bmhft;
    t->e_tot = t->u_tot + t->e_kin;
    t->e_nvt = (s->p.integrator == MDFF_NPT_NHCNP ? s->e_npt : s->e_nvt) / nr;
    t->h_tot = (s->p.integrator == MDFF_NVE_VV) ? t->e_tot : t->e_tot + t->e_nvt;   // thermo.f90:184-199
    t->volume = omega;
    double pv = (s->en.vir_lj + s->en.vir_morse + s->en.vir_bmhft) / omega / nr + s->en.pvirial_coul / nr;
    t->pvirial_tot = pv / s->u.press;
    t->pressure_tot = (pv + s->temp_r * s->u.boltz / omega) / s->u.press;
    t->nlist_rebuilt = s->step_rebuilt;
    t->scf_iter = s->en.scf_iter;
    t->scf_rmsd = s->en.scf_rmsd;
}

void copy_out(orc_sys* s, double* fx, double* fy, double* fz, mdff_energies* e, double* tn, double* tc,
              double* ef, double* efg, double* mu) {
    int n = s->natm;
    if (fx) std::memcpy(fx, s->fx.data(), sizeof(double) * n);
    if (fy) std::memcpy(fy, s->fy.data(), sizeof(double) * n);
    if (fz) std::memcpy(fz, s->fz.data(), sizeof(double) * n);
    if (e) *e = s->en;
    if (tn) for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) tn[b * 3 + a] = s->tau_nonb[a][b];
    if (tc) for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) tc[b * 3 + a] = s->tau_coul[a][b];
    if (ef) { if (s->ef.size() == 3 * (size_t)n) std::memcpy(ef, s->ef.data(), sizeof(double) * 3 * n); else std::memset(ef, 0, sizeof(double) * 3 * n); }
    if (efg) {
        static const int comp[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
        for (int c = 0; c < 6; ++c)
            for (int ia = 0; ia < n; ++ia)
                efg[(size_t)c * n + ia] = s->efg.size() == 9 * (size_t)n ? s->efg[(size_t)(comp[c][0] * 3 + comp[c][1]) * n + ia] : 0.0;
    }
    if (mu) { if (s->mu.size() == 3 * (size_t)n) std::memcpy(mu, s->mu.data(), sizeof(double) * 3 * n); else std::memset(mu, 0, sizeof(double) * 3 * n); }
}


// ---------------------------------------------------------------------------
// Force-matching loss and its gradient with respect to the force-field
// parameters.  The reference has no derivatives: this is the FP64 checker of
// the engine's adjoint kernels, written from the engine's own force
// expressions (the ones restated above) by hand differentiation.
//
// Loss of one configuration:  L = cF sum_i |F_i - F*_i|^2 + cS sum_ab (tau_ab - tau*_ab)^2
// with F the total force (eV/A) and tau = tau_nonb + tau_coul (GPa).
// With R_i = dL/dF_i and S = dL/dtau held fixed, dL/dtheta is the derivative
// of J = sum_i R_i.F_i + S:tau.  J depends on theta directly and through the
// induced dipoles mu, which solve A mu = b with A = 1/alpha - T (T the
// undamped dipole field operator, symmetric) and b the damped static field.
// The adjoint lambda = A^{-1} dJ/dmu gives
//   dL/dtheta = dJ/dtheta|_mu + lambda.(db/dtheta - dA/dtheta mu).
// ---------------------------------------------------------------------------

// Tang-Toennies pieces and their parameter derivatives:
// g = 1 - f = c e^{-x} sum_{m<=k} x^m/m!,  gd = f' = c b e^{-x} x^k/k!,  x = b r.
struct TTDeriv { double g, gd, dg_db, dg_dc, dgd_db, dgd_dc; };
TTDeriv tt_deriv(double b, double c, double r, int k) {
    double x = b * r, e = std::exp(-x);
    double sum = E_TT[k];
    for (int m = k - 1; m >= 0; --m) sum = sum * x + E_TT[m];
    double tk = E_TT[k] * std::pow(x, k);
    TTDeriv t;
    t.g = c * e * sum;
    t.gd = c * b * e * tk;
    t.dg_dc = e * sum;
    t.dg_db = -c * r * e * tk;
    t.dgd_dc = b * e * tk;
    t.dgd_db = c * e * tk * (1.0 + k - x);
    return t;
}

// Upper-triangle slot of an unordered type pair.
inline void upper(int& a, int& b) { if (a > b) std::swap(a, b); }

// Jacobi-preconditioned CG on the polarisable atoms: (1/alpha - T) x = rhs.
int adjoint_solve(orc_sys* s, const std::vector<double>& rhs, std::vector<double>& x, const std::vector<char>& pol,
                  int npol) {
    int n = s->natm;
    const mdff_params& p = s->p;
    std::vector<double> Eind(3 * (size_t)n, 0.0);
    auto apply = [&](const std::vector<double>& v, std::vector<double>& out) {
        induced_field(s, v, Eind);
        out.assign(3 * (size_t)n, 0.0);
        for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia)
            if (pol[ia]) out[(size_t)c * n + ia] = v[(size_t)c * n + ia] * s->invpoldia[ia] - Eind[(size_t)c * n + ia];
    };
    auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) { double t = 0; for (size_t k = 0; k < a.size(); ++k) t += a[k] * b[k]; return t; };
    x.assign(3 * (size_t)n, 0.0);
    for (int c = 0; c < 3; ++c) for (int ia = 0; ia < n; ++ia)
        if (pol[ia]) x[(size_t)c * n + ia] = s->poldia[ia] * rhs[(size_t)c * n + ia];
    std::vector<double> r(3 * (size_t)n), z(3 * (size_t)n), d, Ad;
    apply(x, Ad);
    for (size_t k = 0; k < r.size(); ++k) r[k] = pol[k % n] ? rhs[k] - Ad[k] : 0.0;
    for (size_t k = 0; k < r.size(); ++k) z[k] = s->poldia[k % n] * r[k];
    d = z;
    double rz = dot(r, z);
    double rmsd = std::sqrt(dot(r, r) / double(npol));
    int it = 0;
    while (it < p.max_scf_pol_iter && rmsd > p.conv_tol_ind) {
        it++;
        apply(d, Ad);
        double a = rz / dot(d, Ad);
        for (size_t k = 0; k < x.size(); ++k) { x[k] += a * d[k]; r[k] -= a * Ad[k]; }
        for (size_t k = 0; k < r.size(); ++k) z[k] = s->poldia[k % n] * r[k];
        double rz2 = dot(r, z);
        rmsd = std::sqrt(dot(r, r) / double(npol));
        double beta = rz2 / rz;
        rz = rz2;
        for (size_t k = 0; k < d.size(); ++k) d[k] = z[k] + beta * d[k];
    }
    return it;
}

int loss_grad(orc_sys* s, const double* fxt, const double* fyt, const double* fzt, const double* taut, double cF,
              double cS, double* loss, mdff_param_grad* g, int* iters) {
    const int n = s->natm;
    const mdff_params& p = s->p;
    // a fresh solve: no predictor history
    std::fill(s->dip_hist.begin(), s->dip_hist.end(), 0.0);
    s->itime = 0;
    engforce(s);
    iters[0] = s->en.scf_iter;
    iters[1] = 0;
    std::vector<double> R(3 * (size_t)n);
    double L = 0.0;
    const double* ft[3] = {fxt, fyt, fzt};
    const std::vector<double>* fv[3] = {&s->fx, &s->fy, &s->fz};
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < n; ++i) {
            double dlt = (*fv[c])[i] - ft[c][i];
            L += cF * dlt * dlt;
            R[(size_t)c * n + i] = 2.0 * cF * dlt;
        }
    double S[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double dlt = s->tau_nonb[a][b] + s->tau_coul[a][b] - taut[3 * b + a];
            L += cS * dlt * dlt;
            S[a][b] = 2.0 * cS * dlt;
        }
    *loss += L;
    const double so = 1.0 / (s->cell.omega * s->u.press);   // stress per unit pair virial
    std::vector<double> sx, sy, sz;
    direct_coords(s, sx, sy, sz);
    auto RR = [&](int c, int i) { return R[(size_t)c * n + i]; };
    auto Sr = [&](const double r[3], double out[3]) {
        for (int a = 0; a < 3; ++a) out[a] = S[a][0] * r[0] + S[a][1] * r[1] + S[a][2] * r[2];
    };
    // --- short-range pairs: dJ/dtheta = sum_pairs dw/dtheta [(R_i - R_j).r + r.S.r/(omega press)]
    if (p.lbmhft || p.lbmhftd || p.lmorse) {
        for_pairs(s, s->vdw, sx, sy, sz, [&](int ia, int ja) {
            double r[3];
            double rsq = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], r[0], r[1], r[2]);
            double srv[3];
            Sr(r, srv);
            double geo = 0.0;
            for (int c = 0; c < 3; ++c) geo += (RR(c, ia) - RR(c, ja)) * r[c] + so * r[c] * srv[c];
            int t1 = s->itype[ia], t2 = s->itype[ja];
            if ((p.lbmhft || p.lbmhftd) && p.Abmhftd[t1][t2] != 0.0 && rsq < s->rcutsq[t1][t2]) {
                double d = std::sqrt(rsq);
                double A = p.Abmhftd[t1][t2], B = p.Bbmhftd[t1][t2], C = p.Cbmhftd[t1][t2], D = p.Dbmhftd[t1][t2];
                double e1 = std::exp(-B * d), erh = A * e1;
                double d6 = 1.0 / (rsq * rsq * rsq), d8 = d6 / rsq;
                double f6 = 1.0, f8 = 1.0, fd6 = 0.0, fd8 = 0.0, df6 = 0.0, df8 = 0.0, dfd6 = 0.0, dfd8 = 0.0;
                if (p.lbmhftd) {
                    double bd = p.BDbmhftd[t1][t2];
                    TTDeriv a6 = tt_deriv(bd, 1.0, d, 6), a8 = tt_deriv(bd, 1.0, d, 8);
                    f6 = 1.0 - a6.g; fd6 = a6.gd; df6 = -a6.dg_db; dfd6 = a6.dgd_db;
                    f8 = 1.0 - a8.g; fd8 = a8.gd; df8 = -a8.dg_db; dfd8 = a8.dgd_db;
                }
                int a = t1, b = t2;
                upper(a, b);
                g->Abmhftd[a][b] += geo * B * e1 / d;
                g->Bbmhftd[a][b] += geo * erh * (1.0 - B * d) / d;
                g->Cbmhftd[a][b] += geo * (-6.0 * f6 * d6 / d + fd6 * d6) / d;
                g->Dbmhftd[a][b] += geo * (-8.0 * f8 * d8 / d + fd8 * d8) / d;
                if (p.lbmhftd)
                    g->BDbmhftd[a][b] += geo * (-6.0 * C * d6 / d * df6 - 8.0 * D * d8 / d * df8 + C * d6 * dfd6 + D * d8 * dfd8) / d;
            }
            int m1 = s->itype[ja], m2 = s->itype[ia];
            if (p.lmorse && rsq < s->rcutsq[m1][m2]) {
                double d = std::sqrt(rsq);
                double eps = p.epsmor[m1][m2], rho = p.rhomor[m1][m2], sig = p.sigmamor[m1][m2];
                double e = std::exp(-d * rho) * s->rs[m1][m2];
                int a = m1, b = m2;
                upper(a, b);
                g->epsmor[a][b] += geo * 2.0 * rho * e * (e - 1.0) / d;
                g->rhomor[a][b] += geo * 2.0 * eps / d * (e * (e - 1.0) + rho * (sig - d) * e * (2.0 * e - 1.0));
                g->sigmamor[a][b] += geo * 2.0 * eps * rho / d * rho * e * (2.0 * e - 1.0);
            }
        });
    }
    if (!p.lcoulomb || !any_polar(s)) return 0;
    // --- electrostatics: h = dJ/dmu (real + reciprocal space), damping terms of dJ/dtheta
    const double cu = s->u.coul;
    std::vector<char> pol(n, 0);
    int npol = 0;
    for (int ia = 0; ia < n; ++ia) if (p.ldip_polar[s->itype[ia]] && s->poldia[ia] != 0.0) { pol[ia] = 1; npol++; }
    const std::vector<double>& mu = s->mu;
    const std::vector<double>& q = s->qia;
    std::vector<double> h(3 * (size_t)n, 0.0);
    const double aES = s->alphaES, a2 = aES * aES, a3 = a2 * aES, a5 = a3 * a2;
    const double cutsq = s->coul.cut * s->coul.cut;
    auto MU = [&](int c, int i) { return mu[(size_t)c * n + i]; };
    struct PairGeo { double r[3], d, A1, B2, C3; };
    auto geom = [&](int ia, int ja, PairGeo& G) -> bool {
        double d2 = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], G.r[0], G.r[1], G.r[2]);
        if (d2 > cutsq) return false;
        double d = std::sqrt(d2);
        double expon = std::exp(-a2 * d2) / PIROOT;
        double F0 = erfc_sel(s, aES * d);
        double F1 = F0 + 2.0 * aES * d * expon;
        double F2 = F1 + 4.0 * a3 * d2 * d * expon / 3.0;
        double F3 = F2 + 8.0 * a5 * d2 * d2 * d * expon / 15.0;
        G.d = d;
        G.A1 = F1 / (d2 * d);
        G.B2 = 3.0 * F2 / (d2 * d2 * d);
        G.C3 = 15.0 * F3 / (d2 * d2 * d2 * d);
        return true;
    };
    for_pairs(s, s->coul, sx, sy, sz, [&](int ia, int ja) {
        PairGeo G;
        if (!geom(ia, ja, G)) return;
        const double* r = G.r;
        int ti = s->itype[ia], tj = s->itype[ja];
        double qi = q[ia], qj = q[ja];
        double mi[3] = {MU(0, ia), MU(1, ia), MU(2, ia)}, mj[3] = {MU(0, ja), MU(1, ja), MU(2, ja)};
        double srv[3], W[3];
        Sr(r, srv);
        for (int c = 0; c < 3; ++c) W[c] = cu * (RR(c, ia) - RR(c, ja)) + cu * so * srv[c];
        double wr = W[0] * r[0] + W[1] * r[1] + W[2] * r[2];
        double rmi = r[0] * mi[0] + r[1] * mi[1] + r[2] * mi[2], rmj = r[0] * mj[0] + r[1] * mj[1] + r[2] * mj[2];
        double Wmi = W[0] * mi[0] + W[1] * mi[1] + W[2] * mi[2], Wmj = W[0] * mj[0] + W[1] * mj[1] + W[2] * mj[2];
        double hi[3], hj[3];
        for (int c = 0; c < 3; ++c) {
            // dipole-dipole
            hi[c] = wr * (-r[c] * rmj * G.C3 + mj[c] * G.B2) + W[c] * rmj * G.B2 + Wmj * r[c] * G.B2;
            hj[c] = wr * (-r[c] * rmi * G.C3 + mi[c] * G.B2) + Wmi * r[c] * G.B2 + W[c] * rmi * G.B2;
            // charge-dipole
            hi[c] += -wr * qj * r[c] * G.B2 + qj * W[c] * G.A1;
            hj[c] += wr * qi * r[c] * G.B2 - qi * W[c] * G.A1;
        }
        bool ldamp = p.ldip_damping[ti][ti][tj] || p.ldip_damping[tj][ti][tj];
        if (ldamp) {
            double d = G.d, d3 = d * d * d, d5 = d3 * d * d;
            TTDeriv Ti = tt_deriv(p.dip_pol_damp_b[ti][ti][tj], p.dip_pol_damp_c[ti][ti][tj], d, p.dip_pol_damp_k[ti][ti][tj]);
            TTDeriv Tj = tt_deriv(p.dip_pol_damp_b[tj][ti][tj], p.dip_pol_damp_c[tj][ti][tj], d, p.dip_pol_damp_k[tj][ti][tj]);
            double Ai = Ti.g / d3, Bi = 3.0 * (Ti.g + d / 3.0 * Ti.gd) / d5;
            double Aj = Tj.g / d3, Bj = 3.0 * (Tj.g + d / 3.0 * Tj.gd) / d5;
            for (int c = 0; c < 3; ++c) {
                hi[c] += qj * (wr * r[c] * Bi - W[c] * Ai);
                hj[c] += -qi * (wr * r[c] * Bj - W[c] * Aj);
            }
            // dJ/d(b,c) at fixed mu: the damped charge-dipole force
            double dAi_b = Ti.dg_db / d3, dBi_b = (3.0 * Ti.dg_db + d * Ti.dgd_db) / d5;
            double dAi_c = Ti.dg_dc / d3, dBi_c = (3.0 * Ti.dg_dc + d * Ti.dgd_dc) / d5;
            double dAj_b = Tj.dg_db / d3, dBj_b = (3.0 * Tj.dg_db + d * Tj.dgd_db) / d5;
            double dAj_c = Tj.dg_dc / d3, dBj_c = (3.0 * Tj.dg_dc + d * Tj.dgd_dc) / d5;
            int a = ti, b = tj;
            upper(a, b);
            g->dip_pol_damp_b[ti][a][b] += qj * (wr * rmi * dBi_b - Wmi * dAi_b);
            g->dip_pol_damp_c[ti][a][b] += qj * (wr * rmi * dBi_c - Wmi * dAi_c);
            g->dip_pol_damp_b[tj][a][b] += -qi * (wr * rmj * dBj_b - Wmj * dAj_b);
            g->dip_pol_damp_c[tj][a][b] += -qi * (wr * rmj * dBj_c - Wmj * dAj_c);
        }
        for (int c = 0; c < 3; ++c) { h[(size_t)c * n + ia] += hi[c]; h[(size_t)c * n + ja] += hj[c]; }
    });
    // reciprocal space: forces F = -fpi_V grad sum_k A_k |rho_k|^2 (half mesh), stress
    // (2 tpi_V / omega) sum_k (delta - kcoe k k) A_k |rho_k|^2.
    {
        const KMesh& km = s->km;
        double tpi_V = TPI / s->cell.omega, fpi_V = 2.0 * tpi_V;
        double cs = cu / s->u.press * 2.0 * tpi_V / s->cell.omega;
        double trS = S[0][0] + S[1][1] + S[2][2];
        int nth = 1;
#ifdef _OPENMP
        nth = omp_get_max_threads();
#endif
        std::vector<std::vector<double>> th(nth, std::vector<double>(3 * (size_t)n, 0.0));
#pragma omp parallel
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            std::vector<double>& lh = th[t];
            std::vector<double> ck(n), sk(n);
#pragma omp for schedule(static)
            for (int ik = 0; ik < km.nk; ++ik) {
                if (km.kk[ik] == 0.0) continue;
                double k[3] = {km.kx[ik], km.ky[ik], km.kz[ik]}, Ak = km.Ak[ik];
                double rhoR = 0, rhoI = 0, sgR = 0, sgI = 0;
                for (int ia = 0; ia < n; ++ia) {
                    double kr = k[0] * s->rx[ia] + k[1] * s->ry[ia] + k[2] * s->rz[ia];
                    ck[ia] = std::cos(kr);
                    sk[ia] = std::sin(kr);
                    double m = k[0] * MU(0, ia) + k[1] * MU(1, ia) + k[2] * MU(2, ia);
                    double kR = k[0] * RR(0, ia) + k[1] * RR(1, ia) + k[2] * RR(2, ia);
                    double aR = q[ia] * ck[ia] - m * sk[ia], aI = q[ia] * sk[ia] + m * ck[ia];
                    rhoR += aR; rhoI += aI;
                    sgR += kR * aR; sgI += kR * aI;
                }
                double kSk = 0.0;
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) kSk += k[a] * S[a][b] * k[b];
                double sk_ = trS - km.kcoe[ik] * kSk;
                for (int ja = 0; ja < n; ++ja) {
                    double kR = k[0] * RR(0, ja) + k[1] * RR(1, ja) + k[2] * RR(2, ja);
                    double v = 2.0 * cu * fpi_V * Ak * (kR * (rhoR * ck[ja] + rhoI * sk[ja]) - (sgR * ck[ja] + sgI * sk[ja]))
                             - 2.0 * cs * sk_ * Ak * (rhoR * sk[ja] - rhoI * ck[ja]);
                    for (int c = 0; c < 3; ++c) lh[(size_t)c * n + ja] += k[c] * v;
                }
            }
        }
        for (int t = 0; t < nth; ++t) for (size_t k = 0; k < h.size(); ++k) h[k] += th[t][k];
    }
    for (size_t k = 0; k < h.size(); ++k) if (!pol[k % n]) h[k] = 0.0;
    std::vector<double> lam;
    iters[1] = adjoint_solve(s, h, lam, pol, npol);
    // polarisabilities: dA/dalpha_t = -1/alpha_t^2 on type-t atoms
    for (int ia = 0; ia < n; ++ia) {
        if (!pol[ia]) continue;
        double lm = 0.0;
        for (int c = 0; c < 3; ++c) lm += lam[(size_t)c * n + ia] * (MU(c, ia) - (c == 0 ? s->dipx[ia] : c == 1 ? s->dipy[ia] : s->dipz[ia]));
        g->poldip_iso[s->itype[ia]] += lm * s->invpoldia[ia] * s->invpoldia[ia];
    }
    // damping in the static field b: E_i += qj (F1 - g_i) r/d^3, E_j -= qi (F1 - g_j) r/d^3
    for_pairs(s, s->coul, sx, sy, sz, [&](int ia, int ja) {
        int ti = s->itype[ia], tj = s->itype[ja];
        if (!(p.ldip_damping[ti][ti][tj] || p.ldip_damping[tj][ti][tj])) return;
        PairGeo G;
        if (!geom(ia, ja, G)) return;
        double d = G.d, d3 = d * d * d;
        double li = 0.0, lj = 0.0;
        for (int c = 0; c < 3; ++c) { li += lam[(size_t)c * n + ia] * G.r[c]; lj += lam[(size_t)c * n + ja] * G.r[c]; }
        TTDeriv Ti = tt_deriv(p.dip_pol_damp_b[ti][ti][tj], p.dip_pol_damp_c[ti][ti][tj], d, p.dip_pol_damp_k[ti][ti][tj]);
        TTDeriv Tj = tt_deriv(p.dip_pol_damp_b[tj][ti][tj], p.dip_pol_damp_c[tj][ti][tj], d, p.dip_pol_damp_k[tj][ti][tj]);
        int a = ti, b = tj;
        upper(a, b);
        g->dip_pol_damp_b[ti][a][b] += -q[ja] * li / d3 * Ti.dg_db;
        g->dip_pol_damp_c[ti][a][b] += -q[ja] * li / d3 * Ti.dg_dc;
        g->dip_pol_damp_b[tj][a][b] += q[ia] * lj / d3 * Tj.dg_db;
        g->dip_pol_damp_c[tj][a][b] += q[ia] * lj / d3 * Tj.dg_dc;
    });
    return 0;
}

}  // namespace


// ---- structure optimisation ------------------------------------------------
// sastry (src/opt.f90:452-849): conjugate gradients on U(r) with the search
// direction normalised to unit length, each line minimised by cubic
// interpolation of U along it (eforce1d, :864-933, evaluates U and dU/dx at
// r + x xi).  Stated as the reference runs it: trial evaluations leave their
// forces in fx (the next direction uses the forces of the last accepted
// trial point), u_tot is reassigned only where the reference assigns it, and
// the energy test uses ftol = tiny(1.0_dp).
static double opt_utot(const orc_sys* s) { return s->en.u_lj + s->en.u_coul + s->en.u_morse + s->en.u_bmhft; }

static void opt_eforce1d(orc_sys* s, double x, double& pot, double& f1d, const std::vector<double>& xix,
                         const std::vector<double>& xiy, const std::vector<double>& xiz, int& neng) {
    const int n = s->natm;
    std::vector<double> tx = s->rx, ty = s->ry, tz = s->rz;
    for (int ia = 0; ia < n; ++ia) {
        s->rx[ia] = tx[ia] + x * xix[ia];
        s->ry[ia] = ty[ia] + x * xiy[ia];
        s->rz[ia] = tz[ia] + x * xiz[ia];
    }
    engforce(s);
    pot = opt_utot(s);
    neng = neng + 1;
    s->rx = tx; s->ry = ty; s->rz = tz;
    f1d = 0.0;
    for (int ia = 0; ia < n; ++ia) f1d = f1d + s->fx[ia] * xix[ia] + s->fy[ia] * xiy[ia] + s->fz[ia] * xiz[ia];
    f1d = -f1d;
}

// The reference halves a trial step without bound while U stays above ukeep
// (labels 524, 525); after OPT_MAX_HALVINGS halvings the step is x0 to the
// last bit, and the minimisation ends at x0 with status 3 (as the engine).
constexpr int OPT_MAX_HALVINGS = 64;

static int opt_sastry(orc_sys* s, int itmax, mdff_opt_result* R) {
    const int n = s->natm;
    std::vector<double> gx(n), gy(n), gz(n), hx(n), hy(n), hz(n), xix(n), xiy(n), xiz(n);
    const double ftol = 2.2250738585072014e-308, epsilon = 1.0e-14;   // tiny(1.0_dp)
    int neng = 0;
    engforce(s);
    neng = neng + 1;
    double u_tot = opt_utot(s);
    R->u_initial = u_tot;
    R->status = 1;
    auto steepest = [&]() {
        double umag = 0.0;
        for (int ja = 0; ja < n; ++ja) {
            xix[ja] = -s->fx[ja]; xiy[ja] = -s->fy[ja]; xiz[ja] = -s->fz[ja];
            gx[ja] = -xix[ja]; gy[ja] = -xiy[ja]; gz[ja] = -xiz[ja];
            hx[ja] = gx[ja]; hy[ja] = gy[ja]; hz[ja] = gz[ja];
            xix[ja] = hx[ja]; xiy[ja] = hy[ja]; xiz[ja] = hz[ja];
            umag = umag + xix[ja] * xix[ja] + xiy[ja] * xiy[ja] + xiz[ja] * xiz[ja];
        }
        umag = std::sqrt(umag);
        for (int ja = 0; ja < n; ++ja) { xix[ja] = xix[ja] / umag; xiy[ja] = xiy[ja] / umag; xiz[ja] = xiz[ja] / umag; }
    };
    auto fdotxi = [&]() {
        double f = 0.0;
        for (int ia = 0; ia < n; ++ia) f = f + s->fx[ia] * xix[ia] + s->fy[ia] * xiy[ia] + s->fz[ia] * xiz[ia];
        return -f;
    };
    auto sumf2 = [&]() {
        double g = 0.0;
        for (int ia = 0; ia < n; ++ia) g = g + s->fx[ia] * s->fx[ia] + s->fy[ia] * s->fy[ia] + s->fz[ia] * s->fz[ia];
        return g;
    };
    auto move = [&](double x) {
        for (int ia = 0; ia < n; ++ia) {
            s->rx[ia] = s->rx[ia] + x * xix[ia];
            s->ry[ia] = s->ry[ia] + x * xiy[ia];
            s->rz[ia] = s->rz[ia] + x * xiz[ia];
        }
    };
    steepest();
    double ds = 0.2, dutol = 1.0e-12, phigrad = 0.0, Eis = u_tot, xsol = 0.0;
    int its;
    for (its = 1; its <= itmax; ++its) {
        phigrad = sumf2();
        R->iterations = its;
        double ukeep = u_tot, x0 = 0.0, u0 = u_tot, f1_dp = fdotxi();
        if (f1_dp >= 0.0) {   // reset to the steepest-descent direction
            steepest();
            ukeep = u_tot; x0 = 0.0; u0 = u_tot; f1_dp = fdotxi();
        }
        double x1 = ds, u1, f1d1, u2 = 0.0, f1ds = 0.0;
        auto stalled = [&]() {
            move(x0);
            R->u_final = u0; R->phigrad = phigrad; R->nforce = neng; R->status = 3;
            return 0;
        };
        opt_eforce1d(s, x1, u1, f1d1, xix, xiy, xiz, neng);
        int nstep = 0;
        double uprev = std::min(u1, u0);
        for (;;) {   // label 777
            nstep = nstep + 1;
            double dx = x1 - x0, dx2 = dx * dx, dx3 = dx * dx2;
            (void)dx3;
            if (nstep > 100) {
                if (std::min(u0, u1) > ukeep) {
                    Eis = u0;
                    R->u_final = Eis; R->phigrad = phigrad; R->nforce = neng; R->status = 3;
                    return 0;
                }
                if (u0 < u1) {
                    opt_eforce1d(s, x0, u0, f1_dp, xix, xiy, xiz, neng);
                    xsol = x0; u_tot = u0; f1ds = f1_dp;
                } else {
                    xsol = x1; u_tot = u1; f1ds = f1d1;
                }
                move(xsol);
                break;
            }
            if (f1_dp * f1d1 < 0.0) {
                const double uppcub = (2.0 / dx2) * (3.0 * (u1 - u0) - (f1d1 + 2.0 * f1_dp) * dx);
                const double u3pcub = (-12.0 / dx3) * ((u1 - u0) - (f1d1 + f1_dp) * (dx / 2.0));
                double x1sol = -uppcub + std::sqrt(uppcub * uppcub - 2.0 * u3pcub * f1_dp);
                x1sol = x1sol / u3pcub;
                double x2sol = -uppcub - std::sqrt(uppcub * uppcub - 2.0 * u3pcub * f1_dp);
                x2sol = x2sol / u3pcub;
                const double curv1 = uppcub + u3pcub * x1sol, curv2 = uppcub + u3pcub * x2sol;
                if (curv1 > 0.0) xsol = x1sol + x0;
                if (curv2 > 0.0) xsol = x2sol + x0;
                for (int nh = 0;; ++nh) {   // label 524: keep u2 below ukeep
                    opt_eforce1d(s, xsol, u2, f1ds, xix, xiy, xiz, neng);
                    if (u2 > ukeep) {
                        if (nh == OPT_MAX_HALVINGS) return stalled();
                        xsol = x0 + (xsol - x0) / 2.0;
                        continue;
                    }
                    break;
                }
                if (std::fabs((uprev - u2) / u2) < dutol) {
                    move(xsol);
                    u_tot = u2; ds = xsol;
                    if (xsol <= 1.0e-8) ds = 1.0e-8;
                    break;
                }
                if (f1_dp * f1ds <= 0.0) { x1 = xsol; u1 = u2; f1d1 = f1ds; }
                else { x0 = xsol; u0 = u2; f1_dp = f1ds; }
                uprev = std::min(u0, u1);
            } else {
                const double u2pdis = (f1d1 - f1_dp) / (x1 - x0), adx = std::fabs(x1 - x0);
                if (u2pdis > 0.0) {
                    xsol = x0 - f1_dp / u2pdis;
                    if (std::fabs(xsol - x0) > 3.0 * adx) xsol = x0 + 3.0 * adx;
                } else {
                    xsol = x0 + 1.50 * adx;
                }
                for (int nh = 0;; ++nh) {   // label 525
                    opt_eforce1d(s, xsol, u2, f1ds, xix, xiy, xiz, neng);
                    if (u2 > ukeep) {
                        if (nh == OPT_MAX_HALVINGS) return stalled();
                        xsol = x0 + (xsol - x0) / 2.0;
                        continue;
                    }
                    break;
                }
                if (std::fabs((uprev - u2) / u2) < dutol) {
                    move(xsol);
                    u_tot = u2; ds = xsol;
                    if (xsol <= 1.0e-8) ds = 1.0e-8;
                    break;
                }
                if (u1 < u0) { x0 = x1; u0 = u1; f1_dp = f1d1; }
                x1 = xsol; u1 = u2; f1d1 = f1ds;
                uprev = std::min(u0, u1);
            }
        }
        // label 676
        const double DD1 = 2.0 * std::fabs(ukeep - u_tot);
        const double DD2 = ftol * (std::fabs(ukeep) + std::fabs(u_tot) + epsilon);
        if (DD1 <= DD2) {
            engforce(s);
            neng = neng + 1;
            Eis = u_tot;
            phigrad = sumf2();
            R->u_final = Eis; R->phigrad = phigrad; R->nforce = neng; R->status = 0;
            return 0;
        } else if (std::fabs(1.0 - u_tot / ukeep) < dutol) {
            dutol = std::fabs(1.0 - u_tot / ukeep);
        }
        double gg = 0.0, dgg = 0.0;
        for (int ja = 0; ja < n; ++ja) {
            xix[ja] = -s->fx[ja]; xiy[ja] = -s->fy[ja]; xiz[ja] = -s->fz[ja];
            gg = gg + gx[ja] * gx[ja] + gy[ja] * gy[ja] + gz[ja] * gz[ja];
            dgg = dgg + (xix[ja] + gx[ja]) * xix[ja] + (xiy[ja] + gy[ja]) * xiy[ja] + (xiz[ja] + gz[ja]) * xiz[ja];
        }
        if (gg == 0.0) {
            R->u_final = u_tot; R->phigrad = phigrad; R->nforce = neng; R->status = 2;
            return 0;
        }
        const double gam = dgg / gg;
        double umag = 0.0;
        for (int ja = 0; ja < n; ++ja) {
            gx[ja] = -xix[ja]; gy[ja] = -xiy[ja]; gz[ja] = -xiz[ja];
            hx[ja] = gx[ja] + gam * hx[ja]; hy[ja] = gy[ja] + gam * hy[ja]; hz[ja] = gz[ja] + gam * hz[ja];
            xix[ja] = hx[ja]; xiy[ja] = hy[ja]; xiz[ja] = hz[ja];
            umag = umag + xix[ja] * xix[ja] + xiy[ja] * xiy[ja] + xiz[ja] * xiz[ja];
        }
        umag = std::sqrt(umag);
        for (int ja = 0; ja < n; ++ja) { xix[ja] = xix[ja] / umag; xiy[ja] = xiy[ja] / umag; xiz[ja] = xiz[ja] / umag; }
    }
    R->u_final = u_tot; R->phigrad = phigrad; R->nforce = neng; R->status = 1;
    R->iterations = itmax;
    return 0;
}

extern "C" {

orc_sys* orc_create(const mdff_params* p, int natm, const int* itype, const double* rx, const double* ry,
                    const double* rz, const double A[9]) {
    orc_sys* s = new orc_sys();
    s->p = *p;
    if (s->p.integrator == MDFF_NVT_NHC2) s->p.nhc_n = 2;   // extended_coordinates_alloc (src/md.f90:335-340)
    symmetrise(s->p);
    set_units(s);
    s->natm = natm;
    s->ntype = p->ntype;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) s->cell.A[i][j] = A[3 * j + i];
    lattice(s->cell);
    s->itype.resize(natm);
    s->natmi.assign(NT, 0);
    for (int i = 0; i < natm; ++i) { s->itype[i] = itype[i] - 1; s->natmi[itype[i] - 1]++; }
    // read_pos.f90:148-150: kardir, periodicbc, dirkar
    s->rx.resize(natm); s->ry.resize(natm); s->rz.resize(natm);
    for (int i = 0; i < natm; ++i) {
        double a, b, c;
        kardir1(s->cell, rx[i], ry[i], rz[i], a, b, c);
        a = a - nint(a); b = b - nint(b); c = c - nint(c);
        dirkar1(s->cell, a, b, c, s->rx[i], s->ry[i], s->rz[i]);
    }
    s->vx.assign(natm, 0.0); s->vy.assign(natm, 0.0); s->vz.assign(natm, 0.0);
    s->fx.assign(natm, 0.0); s->fy.assign(natm, 0.0); s->fz.assign(natm, 0.0);
    // typeinfo_init (read_pos.f90:162-219)
    s->massia.resize(natm); s->qia.resize(natm); s->poldia.resize(natm); s->invpoldia.resize(natm);
    s->dipx.resize(natm); s->dipy.resize(natm); s->dipz.resize(natm);
    for (int i = 0; i < natm; ++i) {
        int t = s->itype[i];
        s->massia[i] = s->p.mass[t];
        s->qia[i] = s->p.qch[t];
        s->poldia[i] = s->p.ldip_polar[t] ? s->p.poldip_iso[t] : 0.0;
        s->invpoldia[i] = s->poldia[i] != 0.0 ? 1.0 / s->poldia[i] : 0.0;
        s->dipx[i] = s->p.dip[t][0]; s->dipy[i] = s->p.dip[t][1]; s->dipz[i] = s->p.dip[t][2];
    }
    if (s->p.lcoulomb) ewald_param(s);
    else s->cutlongrange = s->p.cutlongrange;
    init_nonbonded(s);
    if (s->p.lcoulomb) kpoint_sum_init(s);
    s->vdw.cut = s->p.cutshortrange;
    s->coul.cut = s->cutlongrange;
    s->dip_hist.assign((size_t)(s->p.extrapolate_order + 1) * 3 * natm, 0.0);
    s->dt = s->p.dt * s->u.time;
    s->temp = s->p.temp * s->u.boltz;
    s->timesca = s->p.timesca_thermo * s->u.time;
    s->xi.assign(std::max(2, s->p.nhc_n), 0.0);
    s->vxi.assign(std::max(2, s->p.nhc_n), 0.0);
    s->xib.assign(std::max(2, s->p.nhc_n), 0.0);
    s->vxib.assign(std::max(2, s->p.nhc_n), 0.0);
    s->omega0 = s->cell.omega;
    s->utail0 = s->utail;
    s->ptail0 = s->ptail;
    if (s->p.lvnlist) vnlist_pbc(s);
    return s;
}

void orc_destroy(orc_sys* s) { delete s; }

void orc_set_erfc_mode(orc_sys* s, int mode) { s->erfc_mode = mode; }

void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

double orc_errfc(double x) { return errfc_ref(x); }

void orc_tt_damp(double b, double c, double r, int order, double* f, double* fd) { tt_damp(b, c, r, order, *f, *fd); }

void orc_lattice(const double A[9], double B[9], double* omega, double W[3], double anorm[3]) {
    Cell c;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) c.A[i][j] = A[3 * j + i];
    lattice(c);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) B[3 * j + i] = c.B[i][j];
    *omega = c.omega;
    W[0] = c.WA; W[1] = c.WB; W[2] = c.WC;
    for (int i = 0; i < 3; ++i) anorm[i] = c.anorm[i];
}

// Ewald set-up actually used: alpha, kmax, nk, clamped cutlongrange.
void orc_ewald_info(orc_sys* s, double* alpha, int kmax[3], int* nk, double* cutlong) {
    *alpha = s->alphaES;
    for (int i = 0; i < 3; ++i) kmax[i] = s->kES[i];
    *nk = s->km.nk;
    *cutlong = s->cutlongrange;
}

int orc_set_positions(orc_sys* s, const double* rx, const double* ry, const double* rz) {
    std::memcpy(s->rx.data(), rx, sizeof(double) * s->natm);
    std::memcpy(s->ry.data(), ry, sizeof(double) * s->natm);
    std::memcpy(s->rz.data(), rz, sizeof(double) * s->natm);
    return 0;
}

int orc_get_positions(orc_sys* s, double* rx, double* ry, double* rz) {
    std::memcpy(rx, s->rx.data(), sizeof(double) * s->natm);
    std::memcpy(ry, s->ry.data(), sizeof(double) * s->natm);
    std::memcpy(rz, s->rz.data(), sizeof(double) * s->natm);
    return 0;
}

int orc_nlist_build(orc_sys* s) { vnlist_pbc(s); return 0; }

int orc_nlist_get(orc_sys* s, int which, int* point, int* list, int cap, int* nlist) {
    const VList& L = which == 0 ? s->vdw : s->coul;
    if (!s->have_list) return MDFF_E_STATE;
    *nlist = (int)L.list.size();
    if ((int)L.list.size() > cap) return MDFF_E_LISTOVF;
    for (int i = 0; i <= s->natm; ++i) point[i] = L.point[i] + 1;
    for (size_t k = 0; k < L.list.size(); ++k) list[k] = L.list[k] + 1;
    return 0;
}

// Force-matching loss of this configuration and its parameter gradient,
// ADDED to *loss and *g (see loss_grad).  iters[0], iters[1]: iterations of
// the forward and adjoint solves.
int orc_loss_grad(orc_sys* s, const double* fxt, const double* fyt, const double* fzt, const double taut[9],
                  double cF, double cS, double* loss, mdff_param_grad* g, int iters[2]) {
    return loss_grad(s, fxt, fyt, fzt, taut, cF, cS, loss, g, iters);
}

// ---- L-BFGS ------------------------------------------------------------------
// lbfgs_driver (src/opt.f90:972-1194) calling LBFGS (src/lbfgs.f90:243-456)
// by reverse communication, as the reference runs it: X = (rx, ry, rz),
// G = -(fx, fy, fz) packed component-major, F = u_tot, m = 5, DIAGCO false,
// EPS = epsrel_lbfgs, XTOL = tiny(1.0_dp); the line search MCSRCH
// (:655-957, FTOL 1e-4, MAXFEV 100 as LBFGS sets them; GTOL 0.9, STPMIN
// 1e-20, STPMAX 1e20 from BLOCK DATA LB2, :536-540) with MCSTEP (:960-1186).
// The work vector W keeps the reference's layout: W(1..N) gradient and
// direction scratch, then rho (M), alpha (M), the M search steps and the M
// gradient differences; the SAVEd locals live in LbRC.  Dot products are
// DDOT's left-to-right sums.
struct LbRC {
    int iter = 0, nfun = 0, point = 0, ispt = 0, iypt = 0, info = 0, bound = 0, npt = 0, cp = 0, nfev = 0,
        maxfev = 0;
    double gnorm = 0, stp1 = 0, ftol = 0, stp = 0, ys = 0, yy = 0, xnorm = 0;
    bool finish = false;
    // MCSRCH's SAVEd state
    int infoc = 0;
    bool brackt = false, stage1 = false;
    double dginit = 0, dgtest = 0, dgx = 0, dgy = 0, finit = 0, fx = 0, fy = 0, stx = 0, sty = 0, stmin = 0,
           stmax = 0, width = 0, width1 = 0;
};

static double lb_ddot(int n, const double* a, const double* b) {
    double t = 0.0;
    for (int i = 0; i < n; ++i) t = t + a[i] * b[i];
    return t;
}

static void lb_mcstep(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy, double& stp,
                      double fp, double dp, bool& brackt, double stpmin, double stpmax, int& info) {
    info = 0;
    if ((brackt && (stp <= std::min(stx, sty) || stp >= std::max(stx, sty))) || dx * (stp - stx) >= 0.0 ||
        stpmax < stpmin)
        return;
    const double sgnd = dp * (dx / std::fabs(dx));
    double stpf, stpc, stpq, theta, sc, gamma, p, q, r;
    bool bound;
    auto smax3 = [](double a, double b, double c) { return std::max(std::max(a, b), c); };
    if (fp > fx) {   // a higher function value: the minimum is bracketed
        info = 1;
        bound = true;
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
        sc = smax3(std::fabs(theta), std::fabs(dx), std::fabs(dp));
        gamma = sc * std::sqrt((theta / sc) * (theta / sc) - (dx / sc) * (dp / sc));
        if (stp < stx) gamma = -gamma;
        p = (gamma - dx) + theta;
        q = ((gamma - dx) + gamma) + dp;
        r = p / q;
        stpc = stx + r * (stp - stx);
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2) * (stp - stx);
        stpf = std::fabs(stpc - stx) < std::fabs(stpq - stx) ? stpc : stpc + (stpq - stpc) / 2;
        brackt = true;
    } else if (sgnd < 0.0) {   // lower value, derivatives of opposite sign
        info = 2;
        bound = false;
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
        sc = smax3(std::fabs(theta), std::fabs(dx), std::fabs(dp));
        gamma = sc * std::sqrt((theta / sc) * (theta / sc) - (dx / sc) * (dp / sc));
        if (stp > stx) gamma = -gamma;
        p = (gamma - dp) + theta;
        q = ((gamma - dp) + gamma) + dx;
        r = p / q;
        stpc = stp + r * (stx - stp);
        stpq = stp + (dp / (dp - dx)) * (stx - stp);
        stpf = std::fabs(stpc - stp) > std::fabs(stpq - stp) ? stpc : stpq;
        brackt = true;
    } else if (std::fabs(dp) < std::fabs(dx)) {   // same sign, derivative magnitude decreases
        info = 3;
        bound = true;
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
        sc = smax3(std::fabs(theta), std::fabs(dx), std::fabs(dp));
        gamma = sc * std::sqrt(std::max(0.0, (theta / sc) * (theta / sc) - (dx / sc) * (dp / sc)));
        if (stp > stx) gamma = -gamma;
        p = (gamma - dp) + theta;
        q = (gamma + (dx - dp)) + gamma;
        r = p / q;
        if (r < 0.0 && gamma != 0.0) stpc = stp + r * (stx - stp);
        else if (stp > stx) stpc = stpmax;
        else stpc = stpmin;
        stpq = stp + (dp / (dp - dx)) * (stx - stp);
        if (brackt) stpf = std::fabs(stp - stpc) < std::fabs(stp - stpq) ? stpc : stpq;
        else stpf = std::fabs(stp - stpc) > std::fabs(stp - stpq) ? stpc : stpq;
    } else {   // same sign, derivative magnitude does not decrease
        info = 4;
        bound = false;
        if (brackt) {
            theta = 3 * (fp - fy) / (sty - stp) + dy + dp;
            sc = smax3(std::fabs(theta), std::fabs(dy), std::fabs(dp));
            gamma = sc * std::sqrt((theta / sc) * (theta / sc) - (dy / sc) * (dp / sc));
            if (stp > sty) gamma = -gamma;
            p = (gamma - dp) + theta;
            q = ((gamma - dp) + gamma) + dy;
            r = p / q;
            stpc = stp + r * (sty - stp);
            stpf = stpc;
        } else {
            stpf = stp > stx ? stpmax : stpmin;
        }
    }
    if (fp > fx) {
        sty = stp; fy = fp; dy = dp;
    } else {
        if (sgnd < 0.0) { sty = stx; fy = fx; dy = dx; }
        stx = stp; fx = fp; dx = dp;
    }
    stpf = std::min(stpmax, stpf);
    stpf = std::max(stpmin, stpf);
    stp = stpf;
    if (brackt && bound) {   // 0.66: a default-real constant in the reference
        if (sty > stx) stp = std::min(stx + (double)0.66f * (sty - stx), stp);
        else stp = std::max(stx + (double)0.66f * (sty - stx), stp);
    }
}

// MCSRCH by reverse communication: info = -1 on return asks for F and G at X
static void lb_mcsrch(LbRC& c, int n, double* x, double f, const double* g, const double* sdir, double& stp,
                      double ftol, double xtol, int maxfev, int& info, int& nfev, double* wa) {
    const double gtol = 0.9, stpmin = 1.0e-20, stpmax = 1.0e20, p5 = 0.5, p66 = 0.66, xtrapf = 4.0;
    if (info != -1) {
        c.infoc = 1;
        if (n <= 0 || stp <= 0.0 || ftol < 0.0 || gtol < 0.0 || xtol < 0.0 || stpmin < 0.0 || stpmax < stpmin ||
            maxfev <= 0)
            return;
        c.dginit = 0.0;
        for (int j = 0; j < n; ++j) c.dginit = c.dginit + g[j] * sdir[j];
        if (c.dginit >= 0.0) return;   // not a descent direction
        c.brackt = false;
        c.stage1 = true;
        nfev = 0;
        c.finit = f;
        c.dgtest = ftol * c.dginit;
        c.width = stpmax - stpmin;
        c.width1 = c.width / p5;
        for (int j = 0; j < n; ++j) wa[j] = x[j];
        c.stx = 0.0; c.fx = c.finit; c.dgx = c.dginit;
        c.sty = 0.0; c.fy = c.finit; c.dgy = c.dginit;
    } else {
        info = 0;
        nfev = nfev + 1;
        double dg = 0.0;
        for (int j = 0; j < n; ++j) dg = dg + g[j] * sdir[j];
        const double ftest1 = c.finit + stp * c.dgtest;
        if ((c.brackt && (stp <= c.stmin || stp >= c.stmax)) || c.infoc == 0) info = 6;
        if (stp == stpmax && f <= ftest1 && dg <= c.dgtest) info = 5;
        if (stp == stpmin && (f > ftest1 || dg >= c.dgtest)) info = 4;
        if (nfev >= maxfev) info = 3;
        if (c.brackt && c.stmax - c.stmin <= xtol * c.stmax) info = 2;
        if (f <= ftest1 && std::fabs(dg) <= gtol * (-c.dginit)) info = 1;
        if (info != 0) return;
        if (c.stage1 && f <= ftest1 && dg >= std::min(ftol, gtol) * c.dginit) c.stage1 = false;
        if (c.stage1 && f <= c.fx && f > ftest1) {   // the modified function
            double fm = f - stp * c.dgtest, fxm = c.fx - c.stx * c.dgtest, fym = c.fy - c.sty * c.dgtest;
            double dgm = dg - c.dgtest, dgxm = c.dgx - c.dgtest, dgym = c.dgy - c.dgtest;
            lb_mcstep(c.stx, fxm, dgxm, c.sty, fym, dgym, stp, fm, dgm, c.brackt, c.stmin, c.stmax, c.infoc);
            c.fx = fxm + c.stx * c.dgtest;
            c.fy = fym + c.sty * c.dgtest;
            c.dgx = dgxm + c.dgtest;
            c.dgy = dgym + c.dgtest;
        } else {
            lb_mcstep(c.stx, c.fx, c.dgx, c.sty, c.fy, c.dgy, stp, f, dg, c.brackt, c.stmin, c.stmax, c.infoc);
        }
        if (c.brackt) {
            if (std::fabs(c.sty - c.stx) >= p66 * c.width1) stp = c.stx + p5 * (c.sty - c.stx);
            c.width1 = c.width;
            c.width = std::fabs(c.sty - c.stx);
        }
    }
    // label 30: the next trial step
    if (c.brackt) {
        c.stmin = std::min(c.stx, c.sty);
        c.stmax = std::max(c.stx, c.sty);
    } else {
        c.stmin = c.stx;
        c.stmax = stp + xtrapf * (stp - c.stx);
    }
    stp = std::max(stp, stpmin);
    stp = std::min(stp, stpmax);
    if ((c.brackt && (stp <= c.stmin || stp >= c.stmax)) || nfev >= maxfev - 1 || c.infoc == 0 ||
        (c.brackt && c.stmax - c.stmin <= xtol * c.stmax))
        stp = c.stx;
    for (int j = 0; j < n; ++j) x[j] = wa[j] + stp * sdir[j];
    info = -1;
}

// LBFGS (DIAGCO false): iflag 0 starts, 1 re-enters after an evaluation;
// on return 1 asks for F and G at X, 0 converged, -1 line search failed
static void lb_lbfgs(LbRC& c, int n, int m, double* x, double f, double* g, double* diag, double eps, double xtol,
                     double* w, int& iflag) {
    // 1-based W(k) of the reference is w[k - 1]
    bool search = false;
    if (iflag == 1) {
        search = true;   // label 172
    } else {
        c.iter = 0;
        c.nfun = 1;
        c.point = 0;
        c.finish = false;
        for (int i = 0; i < n; ++i) diag[i] = 1.0;
        c.ispt = n + 2 * m;
        c.iypt = c.ispt + n * m;
        for (int i = 0; i < n; ++i) w[c.ispt + i] = -g[i] * diag[i];
        c.gnorm = std::sqrt(lb_ddot(n, g, g));
        c.stp1 = 1.0 / c.gnorm;
        c.ftol = 1.0e-4;
        c.maxfev = 100;
    }
    for (;;) {
        if (!search) {   // label 80
            c.iter = c.iter + 1;
            c.info = 0;
            c.bound = c.iter - 1;
            if (c.iter != 1) {
                if (c.iter > m) c.bound = m;
                c.ys = lb_ddot(n, &w[c.iypt + c.npt], &w[c.ispt + c.npt]);
                c.yy = lb_ddot(n, &w[c.iypt + c.npt], &w[c.iypt + c.npt]);
                for (int i = 0; i < n; ++i) diag[i] = c.ys / c.yy;
                c.cp = c.point;
                if (c.point == 0) c.cp = m;
                w[n + c.cp - 1] = 1.0 / c.ys;
                for (int i = 0; i < n; ++i) w[i] = -g[i];
                c.cp = c.point;
                for (int i = 0; i < c.bound; ++i) {
                    c.cp = c.cp - 1;
                    if (c.cp == -1) c.cp = m - 1;
                    const double sq = lb_ddot(n, &w[c.ispt + c.cp * n], w);
                    const int inmc = n + m + c.cp;
                    const int iycn = c.iypt + c.cp * n;
                    w[inmc] = w[n + c.cp] * sq;
                    const double a = -w[inmc];
                    for (int j = 0; j < n; ++j) w[j] = w[j] + a * w[iycn + j];
                }
                for (int i = 0; i < n; ++i) w[i] = diag[i] * w[i];
                for (int i = 0; i < c.bound; ++i) {
                    const double yr = lb_ddot(n, &w[c.iypt + c.cp * n], w);
                    double beta = w[n + c.cp] * yr;
                    const int inmc = n + m + c.cp;
                    beta = w[inmc] - beta;
                    const int iscn = c.ispt + c.cp * n;
                    for (int j = 0; j < n; ++j) w[j] = w[j] + beta * w[iscn + j];
                    c.cp = c.cp + 1;
                    if (c.cp == m) c.cp = 0;
                }
                for (int i = 0; i < n; ++i) w[c.ispt + c.point * n + i] = w[i];
            }
            // label 165
            c.nfev = 0;
            c.stp = 1.0;
            if (c.iter == 1) c.stp = c.stp1;
            for (int i = 0; i < n; ++i) w[i] = g[i];
        }
        search = false;
        // label 172
        lb_mcsrch(c, n, x, f, g, &w[c.ispt + c.point * n], c.stp, c.ftol, xtol, c.maxfev, c.info, c.nfev, diag);
        if (c.info == -1) {
            iflag = 1;
            return;
        }
        if (c.info != 1) {
            iflag = -1;
            return;
        }
        c.nfun = c.nfun + c.nfev;
        c.npt = c.point * n;
        for (int i = 0; i < n; ++i) {
            w[c.ispt + c.npt + i] = c.stp * w[c.ispt + c.npt + i];
            w[c.iypt + c.npt + i] = g[i] - w[i];
        }
        c.point = c.point + 1;
        if (c.point == m) c.point = 0;
        c.gnorm = std::sqrt(lb_ddot(n, g, g));
        c.xnorm = std::sqrt(lb_ddot(n, x, x));
        c.xnorm = std::max(1.0, c.xnorm);
        if (c.gnorm / c.xnorm <= eps) c.finish = true;
        if (c.finish) {
            iflag = 0;
            return;
        }
    }
}

static int opt_lbfgs(orc_sys* s, int itmax, double eps, mdff_opt_result* R) {
    const int natm = s->natm, n = 3 * natm, m = 5;
    std::vector<double> X(n), G(n), DIAG(n), W((size_t)n * (2 * m + 1) + 2 * m);
    const double xtol = 2.2250738585072014e-308;   // tiny(1.0_dp)
    LbRC c;
    int iflag = 0, icall = 0;
    double phigrad = 0.0;
    for (int ia = 0; ia < natm; ++ia) {
        X[ia] = s->rx[ia];
        X[natm + ia] = s->ry[ia];
        X[2 * natm + ia] = s->rz[ia];
    }
    R->status = 1;
    for (int its = 1; its <= itmax; ++its) {
        engforce(s);
        for (int ia = 0; ia < natm; ++ia) {
            G[ia] = -s->fx[ia];
            G[natm + ia] = -s->fy[ia];
            G[2 * natm + ia] = -s->fz[ia];
        }
        const double F = opt_utot(s);
        if (icall == 0) R->u_initial = F;
        icall = icall + 1;
        lb_lbfgs(c, n, m, X.data(), F, G.data(), DIAG.data(), eps, xtol, W.data(), iflag);
        R->u_final = F;
        R->iterations = c.iter;
        R->nforce = icall;
        if (iflag <= 0) {
            R->phigrad = phigrad;
            R->status = iflag == 0 ? 0 : 3;
            R->info = iflag == 0 ? 0 : c.info;
            return 0;
        }
        phigrad = 0.0;
        for (int ia = 0; ia < natm; ++ia)
            phigrad = phigrad + G[ia] * G[ia] + G[natm + ia] * G[natm + ia] + G[2 * natm + ia] * G[2 * natm + ia];
        R->phigrad = phigrad;
        if (its == itmax) break;   // the positions stay those of the last evaluation
        for (int ia = 0; ia < natm; ++ia) {
            s->rx[ia] = X[ia];
            s->ry[ia] = X[natm + ia];
            s->rz[ia] = X[2 * natm + ia];
        }
    }
    return 0;
}

// ---- M1QN3 -------------------------------------------------------------------
// m1qn3_driver (src/opt.f90:1203-1330) over M1QN3 3.3 (src/m1qn3.f90:90-1382)
// by reverse communication, labels as goto: m1qn3 (argument checks, mupdts,
// the split of dz), m1qn3a (:371-837), dd (:839-923), mlis3 (:999-1316),
// ecube (:1318-1382), in the driver's configuration (DIS mode, cold start,
// ndz = 4n + 5(2n+1), euclid, identity ctonb/ctcab, normtype 'dfn',
// dxmin = tiny(1.0_dp), df1 = 1, impres 0).  The SAVEd locals live in M1RC;
// mlis3's indica, never reset by the reference, lives in the system
// (zero for a fresh one, as a static variable in a fresh process).
struct M1RC {
    int reentry = 0, m = 0;
    int id = 0, igg = 0, idiag = 0, iaux = 0, ialpha = 0, iybar = 0, isbar = 0;   // 0-based offsets into dz
    // m1qn3a
    bool sscale = false, cold = true, warm = false, skip_update = false;
    int itmax = 0, moderl = 0, isim = 0, jcour = 0;
    double d1 = 0, t = 0, tmin = 0, tmax = 0, gnorm = 0, gnorms = 0, eps1 = 0, ff = 0, precos = 0, ys = 0, den = 0,
           ps = 0, hp0 = 0;
    // mlis3
    int indicd = 0;
    double tesf = 0, tesd = 0, tg = 0, fg = 0, fpg = 0, td = 0, ta = 0, fa = 0, fpa = 0, fn = 0, fp = 0, ffn = 0,
           fd = 0, fpd = 0, barmin = 0, barmul = 0, barmax = 0, barr = 0, gauche = 0, droite = 0, taa = 0;
};

static double m1o_prosca(int n, const double* x, const double* y) {   // euclid
    double ps = 0.0;
    for (int i = 0; i < n; ++i) ps = ps + x[i] * y[i];
    return ps;
}

static void m1o_ecube(double& t, double f, double fp, double ta, double fa, double fpa, double tlower,
                      double tupper) {
    double z1, b, discri, sign, den, anum;
    z1 = fp + fpa - 3.0 * (fa - f) / (ta - t);
    b = z1 + fp;
    if (std::fabs(z1) <= 1.0) {
        discri = z1 * z1 - fp * fpa;
    } else {
        discri = fp / z1;
        discri = discri * fpa;
        discri = z1 - discri;
        if (z1 >= 0.0 && discri >= 0.0) {
            discri = std::sqrt(z1) * std::sqrt(discri);
            goto L120;
        }
        if (z1 <= 0.0 && discri <= 0.0) {
            discri = std::sqrt(-z1) * std::sqrt(-discri);
            goto L120;
        }
        discri = -1.0;
    }
    if (discri < 0.0) {
        if (fp < 0.0) t = tupper;
        if (fp >= 0.0) t = tlower;
        goto L900;
    }
    discri = std::sqrt(discri);
L120:
    if (t - ta < 0.0) discri = -discri;
    sign = (t - ta) / std::fabs(t - ta);
    if (b * sign > 0.0) {
        t = t + fp * (ta - t) / (b + discri);
    } else {
        den = z1 + b + fpa;
        anum = b - discri;
        if (std::fabs((t - ta) * anum) < (tupper - tlower) * std::fabs(den)) t = t + anum * (ta - t) / den;
        else t = tupper;
    }
L900:
    t = std::max(t, tlower);
    t = std::min(t, tupper);
}

static void m1o_mlis3(M1RC& c, int n, double* x, double& f, double fpn, double& t, double& tmin, double tmax,
                      const double* d, const double* g, double amd, double amf, int& logic, int& nap, int napmax,
                      double* xn, int& reentry, int& indic, int& indica) {
    if (reentry == 2) goto L9999;
    if (n > 0 && fpn < 0.0 && t > 0.0 && tmax > 0.0 && amf > 0.0 && amd > amf && amd < 1.0) goto L5;
    logic = 6;
    goto L999;
L5:
    c.tesf = amf * fpn;
    c.tesd = amd * fpn;
    c.barmin = 0.01;
    c.barmul = 5.0;
    c.barmax = 0.3;
    c.barr = c.barmin;
    c.td = 0.0;
    c.tg = 0.0;
    c.fn = f;
    c.fg = c.fn;
    c.fpg = fpn;
    c.ta = 0.0;
    c.fa = c.fn;
    c.fpa = fpn;
    if (t < tmin) {
        t = tmin;
        if (t > tmax) tmin = tmax;
    }
    while (c.fn + t * fpn >= c.fn + 0.9 * t * fpn) t = 2.0 * t;
    logic = 0;
    if (t > tmax) {
        t = tmax;
        logic = 1;
    }
    for (int i = 0; i < n; ++i) {
        xn[i] = x[i];
        x[i] = xn[i] + t * d[i];
    }
L100:
    nap = nap + 1;
    if (nap > napmax) {
        logic = 4;
        c.fn = c.fg;
        for (int i = 0; i < n; ++i) xn[i] = xn[i] + c.tg * d[i];
        goto L999;
    }
    indic = 4;
    reentry = 2;
    return;
L9999:
    if (indic == 0) {
        logic = 5;
        c.fn = f;
        for (int i = 0; i < n; ++i) xn[i] = x[i];
        goto L999;
    }
    if (indic < 0) {
        c.td = t;
        c.indicd = indic;
        logic = 0;
        t = c.tg + 0.1 * (c.td - c.tg);
        goto L905;
    }
    c.fp = m1o_prosca(n, d, g);
    c.ffn = f - c.fn;   // first Wolfe test
    if (c.ffn > t * c.tesf) {
        c.td = t;
        c.fd = f;
        c.fpd = c.fp;
        c.indicd = indic;
        logic = 0;
        goto L500;
    }
    if (c.fp > c.tesd) {   // second Wolfe test
        logic = 0;
        goto L320;
    }
    if (logic == 0) goto L350;
L320:
    c.fn = f;
    for (int i = 0; i < n; ++i) xn[i] = x[i];
    goto L999;
L350:
    c.tg = t;
    c.fg = f;
    c.fpg = c.fp;
    if (c.td != 0.0) goto L500;
    c.taa = t;   // extrapolation
    c.gauche = (1.0 + c.barmin) * t;
    c.droite = 10.0 * t;
    m1o_ecube(t, f, c.fp, c.ta, c.fa, c.fpa, c.gauche, c.droite);
    c.ta = c.taa;
    if (t < tmax) goto L900;
    logic = 1;
    t = tmax;
    goto L900;
L500:   // interpolation
    if (indica <= 0) {
        c.ta = t;
        t = 0.9 * c.tg + 0.1 * c.td;
        goto L900;
    }
    {
        const double test = c.barr * (c.td - c.tg);
        c.gauche = c.tg + test;
        c.droite = c.td - test;
    }
    c.taa = t;
    m1o_ecube(t, f, c.fp, c.ta, c.fa, c.fpa, c.gauche, c.droite);
    c.ta = c.taa;
    if (t > c.gauche && t < c.droite) c.barr = std::max(c.barmin, c.barr / c.barmul);
    else c.barr = std::min(c.barmul * c.barr, c.barmax);
L900:
    c.fa = f;
    c.fpa = c.fp;
L905:
    indica = indic;
    if (c.td == 0.0) goto L950;
    if (c.td - c.tg < tmin) goto L920;
    for (int i = 0; i < n; ++i) {
        const double z = xn[i] + t * d[i];
        if (z != xn[i] && z != x[i]) goto L950;
    }
L920:
    logic = 6;
    if (c.indicd < 0) logic = c.indicd;
    if (c.tg == 0.0) goto L999;
    c.fn = c.fg;
    for (int i = 0; i < n; ++i) xn[i] = xn[i] + c.tg * d[i];
    goto L999;
L950:
    for (int i = 0; i < n; ++i) x[i] = xn[i] + t * d[i];
    goto L100;
L999:
    reentry = 0;
}

// dd with jmin, jmax 1-based and the pairs ybar(., j), sbar(., j) column j - 1
static void m1o_dd(int n, int nm, double* depl, double* aux, int jmin, int jmax, const double* diag, double* alpha,
                   const double* ybar, const double* sbar) {
    int jfin = jmax;
    if (jfin < jmin) jfin = jmax + nm;
    for (int j = jfin; j >= jmin; --j) {
        int jp = j;
        if (jp > nm) jp = jp - nm;
        const double r = m1o_prosca(n, depl, &sbar[(size_t)(jp - 1) * n]);
        alpha[jp - 1] = r;
        for (int i = 0; i < n; ++i) depl[i] = depl[i] - r * ybar[(size_t)(jp - 1) * n + i];
    }
    for (int i = 0; i < n; ++i) aux[i] = depl[i];
    for (int i = 0; i < n; ++i) aux[i] = aux[i] * diag[i];
    for (int i = 0; i < n; ++i) depl[i] = aux[i];
    for (int j = jmin; j <= jfin; ++j) {
        int jp = j;
        if (jp > nm) jp = jp - nm;
        const double ps = m1o_prosca(n, depl, &ybar[(size_t)(jp - 1) * n]);
        const double r = alpha[jp - 1] - ps;
        for (int i = 0; i < n; ++i) depl[i] = depl[i] + r * sbar[(size_t)(jp - 1) * n + i];
    }
}

static void m1o_m1qn3a(M1RC& c, int n, double* x, double& f, double* g, double dxmin, double df1, double& epsg,
                       int& omode, int& niter, int& nsim, int m, int& jmin, int& jmax, double* d, double* gg,
                       double* diag, double* aux, double* alpha, double* ybar, double* sbar, int& reverse,
                       int& reentry, int& indic, int& indica) {
    const double rm1 = 0.0001, rm2 = 0.99, rmin = 1.0e-20;
    if (reentry == 2) goto L9999;
    c.sscale = false;   // imode(1) = 0
    c.warm = false;     // imode(2) = 0
    c.cold = !c.warm;
    c.skip_update = false;
    c.itmax = niter;
    niter = 0;
    c.isim = 1;
    c.eps1 = 1.0;
    c.ps = m1o_prosca(n, g, g);
    c.gnorm = std::sqrt(c.ps);
    c.gnorms = c.gnorm;   // 'dfn'
    if (c.gnorms < rmin) {
        omode = 2;
        goto L1000;
    }
    if (c.cold) {
        jmin = 1;
        jmax = 0;
    }
    c.jcour = jmax;
    c.precos = 2.0 * df1 / (c.gnorm * c.gnorm);
    for (int i = 0; i < n; ++i) {
        d[i] = -g[i] * c.precos;
        diag[i] = 1.0;
    }
    c.tmax = 1.0e20;
    c.hp0 = m1o_prosca(n, d, g);
    if (c.hp0 >= 0.0) {
        omode = 7;
        goto L1000;
    }
L100:
    niter = niter + 1;
    for (int i = 0; i < n; ++i) gg[i] = g[i];
    c.ff = f;
    c.tmin = 0.0;
    for (int i = 0; i < n; ++i) c.tmin = std::max(c.tmin, std::fabs(d[i]));
    c.tmin = dxmin / c.tmin;
    c.t = 1.0;
    c.d1 = c.hp0;
L9999:
    m1o_mlis3(c, n, x, f, c.d1, c.t, c.tmin, c.tmax, d, g, rm2, rm1, c.moderl, c.isim, nsim, aux, reentry, indic,
              indica);
    if (reentry > 0) return;
    if (c.moderl != 0) {
        if (c.moderl < 0) {
            omode = c.moderl;
            goto L1000;
        } else if (c.moderl == 1) {
            c.skip_update = true;
        } else if (c.moderl == 4) {
            omode = 5;
            goto L1000;
        } else if (c.moderl == 5) {
            omode = 0;
            goto L1000;
        } else if (c.moderl == 6) {
            omode = 6;
            goto L1000;
        }
    } else {
        c.skip_update = false;
    }
    if (c.skip_update) {
    } else if (m > 0) {
        jmax = jmax + 1;
        if (jmax > m) jmax = jmax - m;
        if ((c.cold && niter > m) || (c.warm && jmin == jmax)) {
            jmin = jmin + 1;
            if (jmin > m) jmin = jmin - m;
        }
        c.jcour = jmax;
        double* sb = &sbar[(size_t)(c.jcour - 1) * n];
        double* yb = &ybar[(size_t)(c.jcour - 1) * n];
        for (int i = 0; i < n; ++i) {
            sb[i] = c.t * d[i];
            yb[i] = g[i] - gg[i];
        }
        c.ys = m1o_prosca(n, yb, sb);
        if (c.ys <= 0.0) {
            omode = 7;
            goto L1000;
        }
        c.d1 = std::sqrt(1.0 / c.ys);
        for (int i = 0; i < n; ++i) {
            sb[i] = c.d1 * sb[i];
            yb[i] = c.d1 * yb[i];
        }
        for (int i = 0; i < n; ++i) aux[i] = yb[i];   // ctonb
        c.ps = 0.0;
        for (int i = 0; i < n; ++i) c.ps = c.ps + diag[i] * aux[i] * aux[i];
        c.d1 = 1.0 / c.ps;
        for (int i = 0; i < n; ++i) diag[i] = diag[i] * c.d1;
        for (int i = 0; i < n; ++i) gg[i] = sb[i];   // ctonb
        c.ps = 0.0;
        for (int i = 0; i < n; ++i) c.ps = c.ps + gg[i] * gg[i] / diag[i];
        c.den = c.ps;
        for (int i = 0; i < n; ++i) {
            const double q = gg[i] / diag[i];
            diag[i] = 1.0 / (1.0 / diag[i] + aux[i] * aux[i] - (q * q) / c.den);
            if (diag[i] <= 0.0) diag[i] = rmin;
        }
    }
    c.ps = m1o_prosca(n, g, g);
    c.gnorm = std::sqrt(c.ps);
    c.eps1 = c.gnorm / c.gnorms;
    if (c.eps1 < epsg) {
        omode = 1;
        goto L1000;
    }
    if (niter == c.itmax) {
        omode = 4;
        goto L1000;
    }
    if (c.isim > nsim) {
        omode = 5;
        goto L1000;
    }
    for (int i = 0; i < n; ++i) d[i] = -g[i];
    m1o_dd(n, m, d, aux, jmin, jmax, diag, alpha, ybar, sbar);
    c.hp0 = m1o_prosca(n, d, g);
    if (c.hp0 >= 0.0) {
        omode = 7;
        goto L1000;
    }
    goto L100;
L1000:
    if (reverse != 0) reverse = -1;
    reentry = 0;
    nsim = c.isim;
    epsg = c.eps1;
}

static void m1o_m1qn3(M1RC& c, int n, double* x, double& f, double* g, double dxmin, double df1, double& epsg,
                      int& omode, int& niter, int& nsim, int* iz, double* dz, int ndz, int& reverse, int& indic,
                      int& indica) {
    if (c.reentry > 0) goto L9999;
    if (n <= 0 || niter <= 0 || nsim <= 0 || dxmin <= 0.0 || epsg <= 0.0) {
        omode = 2;
        if (reverse > 0) reverse = -1;
        return;
    }
    if (epsg >= 1.0) {
        omode = 1;
        niter = 0;
        nsim = 0;
        epsg = 1.0;
        if (reverse > 0) reverse = -1;
        return;
    }
    if (ndz < 5 * n + 1 || ndz < 6 * n + 1) {
        omode = 2;
        if (reverse > 0) reverse = -1;
        return;
    }
    c.m = (ndz - 4 * n) / (2 * n + 1);   // mupdts, DIS
    if (c.m < 1 || ndz < 2 * (2 + c.m) * n + c.m) {
        omode = 2;
        if (reverse > 0) reverse = -1;
        return;
    }
    iz[0] = n;
    iz[1] = 0;
    iz[2] = c.m;
    c.idiag = 0;
    c.iybar = c.idiag + n;
    c.isbar = c.iybar + n * c.m;
    c.id = c.isbar + n * c.m;
    c.igg = c.id + n;
    c.iaux = c.igg + n;
    c.ialpha = c.iaux + n;
L9999:
    m1o_m1qn3a(c, n, x, f, g, dxmin, df1, epsg, omode, niter, nsim, iz[2], iz[3], iz[4], &dz[c.id], &dz[c.igg],
               &dz[c.idiag], &dz[c.iaux], &dz[c.ialpha], &dz[c.iybar], &dz[c.isbar], reverse, c.reentry, indic,
               indica);
}

static int opt_m1qn3(orc_sys* s, int niter_in, int nsim_in, double epsrel, mdff_opt_result* R) {
    const int natm = s->natm, n = 3 * natm, ndz = 4 * n + 5 * (2 * n + 1);
    std::vector<double> x(n), g(n), dz(ndz);
    M1RC c;
    int icall = 0, iz[5] = {0, 0, 0, 0, 0}, omode = 0, niter = niter_in, nsim = nsim_in, indic = 0, reverse = 1;
    double f, phigrad = 0.0, epsg = epsrel;
    const double dxmin = 2.2250738585072014e-308, df1 = 1.0;
    auto evaluate = [&]() {
        for (int ia = 0; ia < natm; ++ia) {
            s->rx[ia] = x[ia];
            s->ry[ia] = x[natm + ia];
            s->rz[ia] = x[2 * natm + ia];
        }
        engforce(s);
        f = opt_utot(s);
        phigrad = 0.0;
        for (int ia = 0; ia < natm; ++ia) {
            g[ia] = -s->fx[ia];
            g[natm + ia] = -s->fy[ia];
            g[2 * natm + ia] = -s->fz[ia];
            phigrad = phigrad + g[ia] * g[ia] + g[natm + ia] * g[natm + ia] + g[2 * natm + ia] * g[2 * natm + ia];
        }
    };
    for (int ia = 0; ia < natm; ++ia) {
        x[ia] = s->rx[ia];
        x[natm + ia] = s->ry[ia];
        x[2 * natm + ia] = s->rz[ia];
    }
    evaluate();
    R->u_initial = f;
    while (reverse >= 0) {
        icall = icall + 1;
        m1o_m1qn3(c, n, x.data(), f, g.data(), dxmin, df1, epsg, omode, niter, nsim, iz, dz.data(), ndz, reverse,
                  indic, s->m1_indica);
        evaluate();
    }
    R->u_final = f;
    R->phigrad = phigrad;
    R->iterations = niter;
    R->nforce = icall + 1;
    R->info = omode;
    R->status = omode == 1 ? 0 : (omode == 4 || omode == 5) ? 1 : omode == 2 ? 2 : 3;
    return 0;
}

int orc_opt_sastry(orc_sys* s, int itmax, mdff_opt_result* r) {
    std::memset(r, 0, sizeof *r);
    return opt_sastry(s, itmax, r);
}

int orc_opt_m1qn3(orc_sys* s, int niter, int nsim, double epsg, mdff_opt_result* r) {
    std::memset(r, 0, sizeof *r);
    return opt_m1qn3(s, niter, nsim, epsg, r);
}

int orc_opt_lbfgs(orc_sys* s, int itmax, double eps, mdff_opt_result* r) {
    std::memset(r, 0, sizeof *r);
    return opt_lbfgs(s, itmax, eps, r);
}

int orc_engforce(orc_sys* s, double* fx, double* fy, double* fz, mdff_energies* e, double tau_nonb[9],
                 double tau_coul[9], double* ef, double* efg, double* mu) {
    engforce(s);
    copy_out(s, fx, fy, fz, e, tau_nonb, tau_coul, ef, efg, mu);
    return 0;
}

// Multipole Ewald field for given charges/dipoles (test hook for the
// linearity and alpha-independence checks): ef[3N] (no coul_unit), u in eV.
int orc_coulomb_field(orc_sys* s, const double* q, const double* mu, int damp, double* ef, double* efg6, double* u) {
    int n = s->natm;
    std::vector<double> qv(q, q + n), mv(mu, mu + 3 * (size_t)n), E, G;
    bool task[6] = {true, true, true, false, false, false};
    std::vector<double> fx = s->fx, fy = s->fy, fz = s->fz;
    double saved_upol = s->u_pol;
    s->u_pol = 0.0;
    multipole_ES(s, E, G, qv, mv, task, damp != 0, true, true, false, false, *u);
    s->u_pol = saved_upol;
    s->fx = fx; s->fy = fy; s->fz = fz;
    std::memcpy(ef, E.data(), sizeof(double) * 3 * n);
    static const int comp[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int c = 0; c < 6; ++c)
        for (int ia = 0; ia < n; ++ia) efg6[(size_t)c * n + ia] = G[(size_t)(comp[c][0] * 3 + comp[c][1]) * n + ia];
    return 0;
}

// Wall time of one Ewald field evaluation of the reference path on the host
// cores (CPU baseline): multipole_ES_dir over the Coulomb list and
// multipole_ES_rec over every kstride-th k-vector (the caller scales the
// reciprocal time by kstride), with the current dipoles; plus one BMHFTD /
// LJ pair loop.
int orc_field_time(orc_sys* s, int kstride, double* t_dir, double* t_rec, double* t_pair) {
    int n = s->natm;
    std::vector<double> mu(3 * (size_t)n, 0.0);
    for (int i = 0; i < n; ++i) mu[i] = 0.01 * (i % 7);
    std::vector<double> ef(3 * (size_t)n, 0.0), efg(9 * (size_t)n, 0.0), f(3 * (size_t)n, 0.0);
    bool task[6] = {true, true, true, false, false, false};
    double tau[3][3] = {{0}}, u = 0.0;
    auto now = []() {
#ifdef _OPENMP
        return omp_get_wtime();
#else
        return 0.0;
#endif
    };
    double t0 = now();
    multipole_ES_dir(s, s->qia, mu, task, true, true, false, false, false, u, ef, efg, f, tau);
    double t1 = now();
    KMesh full = s->km;
    KMesh sub;
    for (int k = 0; k < full.nk; k += kstride) {
        sub.kx.push_back(full.kx[k]); sub.ky.push_back(full.ky[k]); sub.kz.push_back(full.kz[k]);
        sub.kk.push_back(full.kk[k]); sub.Ak.push_back(full.Ak[k]); sub.kcoe.push_back(full.kcoe[k]);
    }
    sub.nk = (int)sub.kx.size();
    s->km = sub;
    multipole_ES_rec(s, s->qia, mu, task, true, false, false, false, u, ef, efg, f, tau);
    s->km = full;
    double t2 = now();
    std::vector<double> sx, sy, sz;
    direct_coords(s, sx, sy, sz);
    if (s->p.lbmhftd || s->p.lbmhft) engforce_bmhftd(s, sx, sy, sz);
    else if (s->p.lnmlj) engforce_nmlj(s, sx, sy, sz);
    double t3 = now();
    *t_dir = t1 - t0;
    *t_rec = t2 - t1;
    *t_pair = t3 - t2;
    return 0;
}

// ---- g(r) and reverse Monte Carlo ----------------------------------------
namespace {
struct GrSpec {
    double cut2, res;
    int nbins, ntype, npairs;
    std::vector<double> vol;   // 4 pi (res rr^2 + res^3/12) / V per bin
};

GrSpec gr_spec(const orc_sys* s, double cut, double res) {
    GrSpec g;
    g.cut2 = cut * cut;
    g.res = res;
    g.nbins = (int)(cut / res) + 1;   // rmc_main, src/rmc.f90:329
    g.ntype = s->ntype;
    g.npairs = s->ntype * (s->ntype + 1) / 2;
    g.vol.resize(g.nbins);
    for (int b = 0; b < g.nbins; ++b) {
        double rr = ((double)b + 0.5) * res;
        double vol = 4.0 * M_PI * (res * rr * rr + (res * res * res) / 12.0);
        g.vol[b] = vol / s->cell.omega;
    }
    return g;
}

// gr_main (src/radial_distrib.f90): counts of ordered pairs, row 0 all pairs,
// row 1 + ita*ntype + jta per ordered type pair
void gr_counts(const orc_sys* s, const GrSpec& g, const std::vector<double>& sx, const std::vector<double>& sy,
               const std::vector<double>& sz, std::vector<long long>& h) {
    const int n = s->natm, nt = g.ntype;
    h.assign((size_t)(1 + nt * nt) * g.nbins, 0);
    for (int ia = 0; ia < n; ++ia)
        for (int ja = 0; ja < n; ++ja) {
            if (ja == ia) continue;
            double rx, ry, rz;
            double rsq = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], rx, ry, rz);
            if (!(rsq < g.cut2)) continue;
            int igr = (int)(std::sqrt(rsq) / g.res);
            if (igr >= g.nbins) continue;
            h[igr] += 1;
            h[(size_t)(1 + s->itype[ia] * nt + s->itype[ja]) * g.nbins + igr] += 1;
        }
}

// rmc_gr (src/rmc.f90:1431-1497): normalised rows [npairs+1][nbins]
void gr_normalise(const orc_sys* s, const GrSpec& g, const std::vector<long long>& h, double* grr) {
    const int nt = g.ntype;
    for (int b = 0; b < g.nbins; ++b) {
        grr[b] = (double)h[b] / (g.vol[b] * (double)s->natm * (double)s->natm);
        int mp = 1;
        for (int it1 = 0; it1 < nt; ++it1)
            for (int it2 = it1; it2 < nt; ++it2, ++mp)
                grr[(size_t)mp * g.nbins + b] = (double)h[(size_t)(1 + it1 * nt + it2) * g.nbins + b] /
                                               (g.vol[b] * (double)s->natmi[it1] * (double)s->natmi[it2]);
    }
}

// eval_chisq_rmc (src/rmc.f90:667-690), the squares of the terms
// q = bin x (npairs + 1) + mp summed by a fixed tree (D20): 1024 strided
// partial sums in order, a halving tree over each group of 32, the same tree
// over the 32 group sums
double chisq_gr(const GrSpec& g, const double* calc, const double* exp_) {
    const int nterm = (g.npairs + 1) * g.nbins;
    std::vector<double> part(1024, 0.0);
    for (int q = 0; q < nterm; ++q) {
        int b = q / (g.npairs + 1), mp = q - b * (g.npairs + 1);
        double d = calc[(size_t)mp * g.nbins + b] - exp_[(size_t)mp * g.nbins + b];
        part[q % 1024] = part[q % 1024] + d * d;
    }
    auto tree32 = [](double* v) {
        for (int o = 16; o > 0; o >>= 1)
            for (int l = 0; l < o; ++l) v[l] = v[l] + v[l + o];
        return v[0];
    };
    double w[32];
    for (int k = 0; k < 32; ++k) w[k] = tree32(&part[32 * k]);
    return tree32(w);
}
}  // namespace

int orc_gr(orc_sys* s, double cut, double res, double* grr, int* nbins) {
    GrSpec g = gr_spec(s, cut, res);
    if (nbins) *nbins = g.nbins;
    if (!grr) return 0;
    std::vector<double> sx, sy, sz;
    direct_coords(s, sx, sy, sz);
    std::vector<long long> h;
    gr_counts(s, g, sx, sy, sz, h);
    gr_normalise(s, g, h, grr);
    return 0;
}

// rmc_main (src/rmc.f90:196-640) on the g(r) chi^2, random numbers from uni
// ---- rmc_efg ----------------------------------------------------------------
namespace {

// multipole_efg_ES (src/efg.f90:1278-1625) for point charges (rmc_main calls
// it with the efg module's mu = 0): the real-space sum over every other atom
// at its minimum image (no cutoff), the reciprocal sum of the k mesh, the
// self term -4 alpha^3 / (3 sqrt(pi)) q; no coul_unit.  V6 [6][n]: xx yy zz
// xy xz yz.
void efg_es_rmc(orc_sys* s, std::vector<double>& V6) {
    const int n = s->natm;
    std::vector<double> sx, sy, sz;
    direct_coords(s, sx, sy, sz);
    const double a = s->alphaES, alpha2 = a * a, alpha3 = alpha2 * a;
    const double selfa = -4.0 * alpha3 / 3.0 / PIROOT;
    std::vector<double> dir(6 * (size_t)n, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
    for (int ia = 0; ia < n; ++ia) {
        double g[6] = {0, 0, 0, 0, 0, 0};
        for (int ja = 0; ja < n; ++ja) {
            if (ja == ia) continue;
            const double qj = s->qia[ja];
            double rxij, ryij, rzij;
            const double d2 = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], rxij, ryij, rzij);
            const double d = std::sqrt(d2), d3 = d2 * d;
            const double dm5 = 1.0 / d2 / d3;
            const double expon = std::exp(-alpha2 * d2) / PIROOT;
            const double F1 = erfc_sel(s, a * d) + 2.0 * a * d * expon;
            const double F2 = F1 + 4.0 * alpha3 * d3 * expon / 3.0;
            g[0] = g[0] - qj * ((3.0 * rxij * rxij * F2 - d2 * F1) * dm5);
            g[1] = g[1] - qj * ((3.0 * ryij * ryij * F2 - d2 * F1) * dm5);
            g[2] = g[2] - qj * ((3.0 * rzij * rzij * F2 - d2 * F1) * dm5);
            g[3] = g[3] - qj * ((3.0 * rxij * ryij * F2) * dm5);
            g[4] = g[4] - qj * ((3.0 * rxij * rzij * F2) * dm5);
            g[5] = g[5] - qj * ((3.0 * ryij * rzij * F2) * dm5);
        }
        for (int c = 0; c < 6; ++c) dir[(size_t)c * n + ia] = g[c];
    }
    std::vector<double> mu0(3 * (size_t)n, 0.0), ef, rec(9 * (size_t)n, 0.0), f(3 * (size_t)n, 0.0);
    const bool task[6] = {true, false, false, false, false, false};
    double u = 0.0, tau[3][3] = {{0}};
    multipole_ES_rec(s, s->qia, mu0, task, false, true, false, false, u, ef, rec, f, tau);
    const int comp[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    V6.assign(6 * (size_t)n, 0.0);
    for (int c = 0; c < 6; ++c)
        for (int ia = 0; ia < n; ++ia) {
            const double self = c < 3 ? selfa * s->qia[ia] : 0.0;
            V6[(size_t)c * n + ia] = dir[(size_t)c * n + ia] + rec[(size_t)(comp[c][0] * 3 + comp[c][1]) * n + ia] + self;
        }
}

// principal values of a symmetric 3x3 tensor, ascending: cyclic Jacobi
// rotations (Rutishauser's formulation) to convergence
void eig3_jacobi(const double v6[6], double w[3]) {
    double m[3][3] = {{v6[0], v6[3], v6[4]}, {v6[3], v6[1], v6[5]}, {v6[4], v6[5], v6[2]}};
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = std::fabs(m[0][1]) + std::fabs(m[0][2]) + std::fabs(m[1][2]);
        if (off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (m[p][q] == 0.0) continue;
                const double theta = (m[q][q] - m[p][p]) / (2.0 * m[p][q]);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < 3; ++k) {   // columns p, q
                    const double mkp = m[k][p], mkq = m[k][q];
                    m[k][p] = c * mkp - sn * mkq;
                    m[k][q] = sn * mkp + c * mkq;
                }
                for (int k = 0; k < 3; ++k) {   // rows p, q
                    const double mpk = m[p][k], mqk = m[q][k];
                    m[p][k] = c * mpk - sn * mqk;
                    m[q][k] = sn * mpk + c * mqk;
                }
                m[p][q] = m[q][p] = 0.0;
            }
    }
    w[0] = m[0][0];
    w[1] = m[1][1];
    w[2] = m[2][2];
    std::sort(w, w + 3);
}

// nmr_convention (src/efg.f90:2546-2620): (Vxx, Vyy, Vzz, eta)
void nmr_conv(const double e[3], double nmr[4]) {
    double diso = (e[0] + e[1] + e[2]) / 3.0;
    if (std::fabs(diso) != 0.0 && std::fabs(diso) > 1e-3) diso = 0.0;
    const double a1 = std::fabs(e[0] - diso), a2 = std::fabs(e[1] - diso), a3 = std::fabs(e[2] - diso);
    double d11, d22, d33;
    if (a1 >= a2 && a1 >= a3) {
        d11 = e[0];
        if (a2 >= a3) { d22 = e[1]; d33 = e[2]; } else { d22 = e[2]; d33 = e[1]; }
    } else if (a2 >= a1 && a2 >= a3) {
        d11 = e[1];
        if (a1 >= a3) { d22 = e[0]; d33 = e[2]; } else { d22 = e[2]; d33 = e[0]; }
    } else {
        d11 = e[2];
        if (a1 >= a2) { d22 = e[0]; d33 = e[1]; } else { d22 = e[1]; d33 = e[0]; }
    }
    nmr[0] = d33;
    nmr[1] = d22;
    nmr[2] = d11;
    double eta = nmr[2] != 0.0 ? (nmr[0] - nmr[1]) / nmr[2] : 0.0;
    if (nmr[0] == nmr[1]) eta = 0.0;
    if (nmr[2] == 0.0) eta = 0.0;
    if (std::fabs(nmr[0]) < 1.0e-5 && std::fabs(nmr[1]) < 1.0e-5 && std::fabs(nmr[2]) < 1.0e-5) eta = 0.0;
    nmr[3] = eta;
}

struct RmcEfg {
    const mdff_rmc_efg_params* ep;
    int PANU, PANvzz, PANeta;
    const double *Uexp, *Vexp, *Eexp;
    // Fortran layouts: U (ui, mp, bin) ui fastest; vzz, eta (mp, bin) mp fastest
    std::vector<double> U, V, E;
};

// rmc_efg (src/rmc.f90:1499-1660) with eval_chisq_Uefg/vzz/eta (:693-769):
// chi[2..4]
void rmc_efg_terms(orc_sys* s, RmcEfg& R, double chi[6]) {
    const int n = s->natm, nt = s->ntype, nt1 = nt + 1;
    const mdff_rmc_efg_params& ep = *R.ep;
    std::vector<double> V6;
    efg_es_rmc(s, V6);
    std::vector<long long> cU((size_t)6 * nt1 * (R.PANU + 1), 0), cV((size_t)nt1 * (R.PANvzz + 1), 0),
        cE((size_t)nt1 * (R.PANeta + 1), 0);
    auto iU = [&](int ui, int mp, int bin) { return ((size_t)bin * nt1 + mp) * 6 + (ui - 1); };
    const double sq3 = 1.0 / std::sqrt(3.0), sq32 = sq3 * 0.5;
    for (int ia = 0; ia < n; ++ia) {
        double v[6], w[3], nmr[4];
        for (int c = 0; c < 6; ++c) v[c] = V6[(size_t)c * n + ia];
        eig3_jacobi(v, w);
        nmr_conv(w, nmr);
        const double Ui[5] = {v[2] * 0.5, v[4] * sq3, v[5] * sq3, v[3] * sq3, (v[0] - v[1]) * sq32};
        const double vzzk = (nmr[2] - ep.vzz_efg_min) / ep.resolution_vzz_efg;
        const double etak = nmr[3] / ep.resolution_eta_efg;
        // INT(x) + 1 in [0, PAN] and INT(x) in [0, PAN], with INT truncating
        if (!(vzzk > -2.0 && vzzk < (double)R.PANvzz)) continue;
        if (!(etak > -1.0 && etak < (double)R.PANeta + 1.0)) continue;
        const int kvzz = (int)vzzk + 1, keta = (int)etak;
        const int it = s->itype[ia] + 1;
        cV[(size_t)kvzz * nt1] += 1;
        cE[(size_t)keta * nt1] += 1;
        cV[(size_t)kvzz * nt1 + it] += 1;
        cE[(size_t)keta * nt1 + it] += 1;
        if (ep.lrmc_u)
            for (int ui = 1; ui <= 5; ++ui) {
                const double uk = (Ui[ui - 1] - ep.u_efg_min) / ep.resolution_u_efg;
                if (!(uk > -2.0 && uk < (double)R.PANU)) continue;
                const int ku = (int)uk + 1;
                cU[iU(ui, 0, ku)] += 1;
                cU[iU(ui, it, ku)] += 1;
                if (ui != 1) {
                    cU[iU(6, 0, ku)] += 1;
                    if (it <= 2) cU[iU(6, it, ku)] += 1;   // the reference's loop covers types 1 and 2
                }
            }
    }
    const double natm = (double)n;
    if (ep.lrmc_u)
        for (int bin = 0; bin <= R.PANU; ++bin)
            for (int ui = 1; ui <= 5; ++ui) {
                R.U[iU(ui, 0, bin)] = (double)cU[iU(ui, 0, bin)] / (ep.resolution_u_efg * natm);
                for (int it = 1; it <= nt; ++it)   // the reference divides the all-types U1 counts here
                    R.U[iU(ui, it, bin)] = (double)cU[iU(1, 0, bin)] / (ep.resolution_u_efg * (double)s->natmi[it - 1]);
            }
    if (ep.lrmc_eta)
        for (int bin = 0; bin < R.PANeta; ++bin) {
            R.E[(size_t)bin * nt1] = (double)cE[(size_t)bin * nt1] / (ep.resolution_eta_efg * natm);
            for (int it = 1; it <= nt; ++it)
                R.E[(size_t)bin * nt1 + it] =
                    (double)cE[(size_t)bin * nt1 + it] / (ep.resolution_eta_efg * (double)s->natmi[it - 1]);
        }
    if (ep.lrmc_vzz)
        for (int bin = 0; bin <= R.PANvzz; ++bin) {
            R.V[(size_t)bin * nt1] = (double)cV[(size_t)bin * nt1] / (ep.resolution_vzz_efg * natm);
            for (int it = 1; it <= nt; ++it)
                R.V[(size_t)bin * nt1 + it] =
                    (double)cV[(size_t)bin * nt1 + it] / (ep.resolution_vzz_efg * (double)s->natmi[it - 1]);
        }
    if (ep.lrmc_u) {
        double c = 0.0;
        for (int bin = 0; bin <= R.PANU; ++bin)
            for (int mp = 0; mp <= nt; ++mp)
                for (int ui = 1; ui <= 5; ++ui) {
                    const double d = R.U[iU(ui, mp, bin)] - R.Uexp[iU(ui, mp, bin)];
                    c = c + d * d;
                }
        chi[2] = c;
    }
    if (ep.lrmc_vzz) {
        double c = 0.0;
        for (int bin = 0; bin <= R.PANvzz; ++bin)
            for (int mp = 0; mp <= nt; ++mp) {
                const double d = R.V[(size_t)bin * nt1 + mp] - R.Vexp[(size_t)bin * nt1 + mp];
                c = c + d * d;
            }
        chi[3] = c;
    }
    if (ep.lrmc_eta) {
        double c = 0.0;
        for (int bin = 0; bin <= R.PANeta; ++bin)
            for (int mp = 0; mp <= nt; ++mp) {
                const double d = R.E[(size_t)bin * nt1 + mp] - R.Eexp[(size_t)bin * nt1 + mp];
                c = c + d * d;
            }
        chi[4] = c;
    }
}

}  // namespace

// eval_chisq_var_distance (src/rmc.f90:778-1063), the full recount of every
// call: for each atom and type the distances to all other atoms of that type
// (minimum image in direct coordinates, no cutoff, in the order of the
// reference's loops), sorted; dab_aver(n, it, it2) summed over the atoms ia of
// type it2 in atom order, zero distances left out; chi^2 summed over ia, it2
// and n in the reference's loop order where the mean is nonzero.
double chisq_var(const orc_sys* s, const std::vector<double>& sx, const std::vector<double>& sy,
                 const std::vector<double>& sz) {
    const int n = s->natm, nt = s->ntype;
    int nmax = 0;
    for (int t = 0; t < nt; ++t) nmax = std::max(nmax, s->natmi[t]);
    std::vector<double> dab((size_t)n * nt * nmax, 0.0);   // dab_sorted_shifted (n, it, ia)
    std::vector<double> aver((size_t)nmax * nt * nt, 0.0);  // dab_aver (n, it, it2) at [(it2 * nt + it) * nmax + n]
    std::vector<double> row;
    for (int ia = 0; ia < n; ++ia) {
        for (int it = 0; it < nt; ++it) {
            row.clear();
            for (int ja = 0; ja < n; ++ja) {
                if (ja == ia || s->itype[ja] != it) continue;
                double rx, ry, rz;
                const double rsq = pairvec(s->cell, sx[ia], sy[ia], sz[ia], sx[ja], sy[ja], sz[ja], rx, ry, rz);
                row.push_back(std::sqrt(rsq));
            }
            std::sort(row.begin(), row.end());
            double* d = &dab[((size_t)ia * nt + it) * nmax];
            for (size_t m = 0; m < row.size(); ++m) d[m] = row[m];
            const int it2 = s->itype[ia];
            for (int m = 0; m < nmax; ++m)
                if (d[m] != 0.0) aver[((size_t)it2 * nt + it) * nmax + m] += d[m];
        }
    }
    double chi = 0.0;
    for (int ia = 0; ia < n; ++ia) {
        const int it1 = s->itype[ia];
        const double ni = (double)s->natmi[it1];
        for (int it2 = 0; it2 < nt; ++it2)
            for (int m = 0; m < nmax; ++m) {
                const double a = aver[((size_t)it1 * nt + it2) * nmax + m];
                if (a != 0.0) {
                    const double mean = a / ni;
                    const double dd = dab[((size_t)ia * nt + it2) * nmax + m] - mean;
                    chi = chi + dd * dd / (mean * mean);
                }
            }
    }
    return chi;
}

int orc_rmc_efg(orc_sys* s, const mdff_rmc_params* rp, const mdff_rmc_efg_params* ep, const double* gexp,
                const double* Uexp, const double* Vexp, const double* Eexp, const double* uni, long long nuni,
                double* grr_out, double* U_out, double* V_out, double* E_out, mdff_rmc_result* res) {
    GrSpec g = gr_spec(s, rp->cut_rmc, rp->resolution_gr);
    const int n = s->natm, nt1 = s->ntype + 1;
    const bool any_efg = ep && (ep->lrmc_u || ep->lrmc_vzz || ep->lrmc_eta);
    RmcEfg R;
    if (ep) {
        R.ep = ep;
        R.PANU = (int)(2.0 * std::fabs(ep->u_efg_min) / ep->resolution_u_efg);
        R.PANvzz = (int)(2.0 * std::fabs(ep->vzz_efg_min) / ep->resolution_vzz_efg);
        R.PANeta = (int)(1.0 / ep->resolution_eta_efg);
        R.Uexp = Uexp;
        R.Vexp = Vexp;
        R.Eexp = Eexp;
        R.U.assign((size_t)6 * nt1 * (R.PANU + 1), 0.0);
        R.V.assign((size_t)nt1 * (R.PANvzz + 1), 0.0);
        R.E.assign((size_t)nt1 * (R.PANeta + 1), 0.0);
    }
    std::vector<double> aU = R.U, aV = R.V, aE = R.E;
    std::vector<double> sx, sy, sz;
    direct_coords(s, sx, sy, sz);
    auto to_cart = [&]() {
        for (int ia = 0; ia < n; ++ia) dirkar1(s->cell, sx[ia], sy[ia], sz[ia], s->rx[ia], s->ry[ia], s->rz[ia]);
    };
    std::vector<double> calc((size_t)(g.npairs + 1) * g.nbins);
    std::vector<long long> h;
    gr_counts(s, g, sx, sy, sz, h);
    gr_normalise(s, g, h, calc.data());
    double chi_old[6] = {0, 0, 0, 0, 0, 0}, chi_new[6];
    chi_old[0] = chisq_gr(g, calc.data(), gexp);
    const bool var = ep && ep->lrmc_var;
    if (var) chi_old[1] = chisq_var(s, sx, sy, sz);
    long long kall = 1, kacc = 1, u = 0;
    if (any_efg && kacc >= ep->efg_start) {
        to_cart();
        rmc_efg_terms(s, R, chi_old);
        aU = R.U; aV = R.V; aE = R.E;
    }
    chi_old[5] = (((chi_old[0] + chi_old[1]) + chi_old[2]) + chi_old[3]) + chi_old[4];
    int status = 0;
    const double dmax[3] = {rp->max_displacement / s->cell.anorm[0], rp->max_displacement / s->cell.anorm[1],
                            rp->max_displacement / s->cell.anorm[2]};
    while (kacc < rp->acceptance_max && kall < rp->max_trials) {
        ++kall;
        if (u + 4 > nuni) { status = 1; --kall; break; }
        // rmc_move (src/rmc.f90:1366-1428)
        int i = (int)(uni[u] * n);
        if (i >= n) i = n - 1;
        double* sv[3] = {&sx[i], &sy[i], &sz[i]};
        double disp[3], snew[3], sold[3];
        for (int d = 0; d < 3; ++d) {
            disp[d] = dmax[d] * (2.0 * uni[u + 1 + d] - 1.0);
            sold[d] = *sv[d];
            double v = *sv[d] + disp[d];
            if (v > 1.0 || v < 0.0) v = v - nint(v);
            snew[d] = v;
            *sv[d] = v;
        }
        u += 4;
        gr_counts(s, g, sx, sy, sz, h);
        gr_normalise(s, g, h, calc.data());
        for (int q = 0; q < 6; ++q) chi_new[q] = 0.0;
        chi_new[0] = chisq_gr(g, calc.data(), gexp);
        if (var) chi_new[1] = chisq_var(s, sx, sy, sz);
        const bool efg_now = any_efg && kacc >= ep->efg_start;
        if (efg_now) {
            to_cart();
            rmc_efg_terms(s, R, chi_new);
        }
        chi_new[5] = (((chi_new[0] + chi_new[1]) + chi_new[2]) + chi_new[3]) + chi_new[4];
        bool acc6 = false, stop = false;
        for (int q = 0; q < 6; ++q) {   // src/rmc.f90:521-540
            double dq = chi_new[q] - chi_old[q];
            bool a;
            if (dq < 0.0) a = true;
            else {
                if (u + 1 > nuni) { stop = true; break; }
                double metro = std::exp(-(dq * 0.5) / rp->temp_rmc[q]);
                a = metro >= uni[u];
                ++u;
            }
            if (q == 5) acc6 = a;
        }
        if (stop) {   // the uniforms ran out: the trial is undone exactly
            for (int d = 0; d < 3; ++d) *sv[d] = sold[d];
            status = 1;
            --kall;
            break;
        }
        if (acc6) {
            ++kacc;
            for (int q = 0; q < 6; ++q) chi_old[q] = chi_new[q];
            if (efg_now) { aU = R.U; aV = R.V; aE = R.E; }
        } else {
            for (int d = 0; d < 3; ++d) *sv[d] = snew[d] - disp[d];   // src/rmc.f90:628-636
        }
    }
    to_cart();
    if (grr_out) {
        gr_counts(s, g, sx, sy, sz, h);
        gr_normalise(s, g, h, grr_out);
    }
    if (ep) {
        if (U_out) std::copy(aU.begin(), aU.end(), U_out);
        if (V_out) std::copy(aV.begin(), aV.end(), V_out);
        if (E_out) std::copy(aE.begin(), aE.end(), E_out);
    }
    if (res) {
        res->kall = kall;
        res->kacc = kacc;
        res->uniforms_used = u;
        for (int q = 0; q < 6; ++q) res->chisq[q] = chi_old[q];
        res->status = status;
        res->pad = 0;
    }
    return 0;
}

int orc_efg_rmc(orc_sys* s, double* out6) {
    std::vector<double> V6;
    efg_es_rmc(s, V6);
    std::copy(V6.begin(), V6.end(), out6);
    return 0;
}

int orc_rmc(orc_sys* s, const mdff_rmc_params* rp, const double* gexp, const double* uni, long long nuni,
            double* grr_out, mdff_rmc_result* res) {
    return orc_rmc_efg(s, rp, nullptr, gexp, nullptr, nullptr, nullptr, uni, nuni, grr_out, nullptr, nullptr, nullptr,
                       res);
}

int orc_md_start(orc_sys* s, const double* vx, const double* vy, const double* vz, mdff_thermo* t0) {
    std::memcpy(s->vx.data(), vx, sizeof(double) * s->natm);
    std::memcpy(s->vy.data(), vy, sizeof(double) * s->natm);
    std::memcpy(s->vz.data(), vz, sizeof(double) * s->natm);
    calc_temp(s, s->temp_r, s->e_kin);
    s->itime = 0;
    engforce(s);
    s->e_nvt = 0.0;
    s->xe = s->ve = s->xe0 = 0.0;
    s->e_npt = s->p.integrator == MDFF_NPT_NHCNP ? s->p.press * s->u.press * s->cell.omega : 0.0;   // P V, at rest
    std::fill(s->xib.begin(), s->xib.end(), 0.0);
    std::fill(s->vxib.begin(), s->vxib.end(), 0.0);
    s->step_rebuilt = 0;
    if (t0) calc_thermo(s, t0, 0);
    return 0;
}

int orc_step(orc_sys* s, int nsteps, double* rx, double* ry, double* rz, double* vx, double* vy, double* vz,
             double* fx, double* fy, double* fz, mdff_thermo* th) {
    int n = s->natm;
    if (rx) std::memcpy(s->rx.data(), rx, sizeof(double) * n);
    if (ry) std::memcpy(s->ry.data(), ry, sizeof(double) * n);
    if (rz) std::memcpy(s->rz.data(), rz, sizeof(double) * n);
    if (vx) std::memcpy(s->vx.data(), vx, sizeof(double) * n);
    if (vy) std::memcpy(s->vy.data(), vy, sizeof(double) * n);
    if (vz) std::memcpy(s->vz.data(), vz, sizeof(double) * n);
    for (int k = 0; k < nsteps; ++k) {
        s->itime++;
        if (s->p.integrator == MDFF_NVT_NHCN) nhcn(s);
        else if (s->p.integrator == MDFF_NVT_NHC2) nhc2(s);
        else if (s->p.integrator == MDFF_NPT_NHCNP) nhcnp(s);
        else prop_velocity_verlet(s);
        s->step_rebuilt = 0;
        if (s->p.lvnlist) s->step_rebuilt = vnlistcheck(s) ? 1 : 0;
        if (th) calc_thermo(s, &th[k], s->itime);
    }
    if (rx) std::memcpy(rx, s->rx.data(), sizeof(double) * n);
    if (ry) std::memcpy(ry, s->ry.data(), sizeof(double) * n);
    if (rz) std::memcpy(rz, s->rz.data(), sizeof(double) * n);
    if (vx) std::memcpy(vx, s->vx.data(), sizeof(double) * n);
    if (vy) std::memcpy(vy, s->vy.data(), sizeof(double) * n);
    if (vz) std::memcpy(vz, s->vz.data(), sizeof(double) * n);
    if (fx) std::memcpy(fx, s->fx.data(), sizeof(double) * n);
    if (fy) std::memcpy(fy, s->fy.data(), sizeof(double) * n);
    if (fz) std::memcpy(fz, s->fz.data(), sizeof(double) * n);
    return 0;
}

}  // extern "C"
