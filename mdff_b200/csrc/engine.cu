// engine.cu -- host side of the B200 force engine and its C ABI.
//
// One translation unit: the kernels live in the *.cuh files included below.
// The host code owns one CUDA stream and every device buffer of a context;
// all device work for a call is queued on that stream and the call returns
// after the results it reports are on the host.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "common.cuh"
#include "nlist.cuh"
#include "pair.cuh"
#include "ewald_real.cuh"
#include "ewald_recip.cuh"
#include "solve.cuh"
#include "integrate.cuh"
#include "opt.cuh"
#include "npt.cuh"
#include "rmc.cuh"
#include "efg_post.cuh"
#include "rmc_efg.cuh"
#include "rmc_var.cuh"
#include "io.cuh"
#include <condition_variable>
#include <deque>
#include <thread>
#include "peaks.cuh"

using namespace mdff;

namespace {

struct Units { double press, boltz, time, coul; };

// Everything a captured MD step holds by value or by address that can change
// between steps: when any of it differs from the capture's, the step is
// captured again.  Zero-filled before use so that memcmp covers the padding.
struct StepKey {
    const void* ptr[6];   // Verlet lists (vdW, Coulomb): nbr, cnt; dipole pair table
    int cap[3];           // list capacities, pair-table capacity
    CellP cell;
    int g_dir, g_dd, p_mul, s_mul;
    int efg;              // the step writes the EFG
    int pmode, pnpt, pshift;   // unused (the predictor plan is device data)
    double skin;
    int n, pad;
};

// The induced-dipole predictor of one step: coefficients and launch shape.
struct PredPlan {
    double coef[16];
    int mode, npt, shift_from;
};

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
};

}  // namespace

struct mdff_ctx {
    mdff_params p;
    std::string err;
    cudaStream_t st = nullptr;
    Units u;
    // system
    int n = 0;
    int ntype = 0;
    int npol = 0;
    bool any_q = false, any_dip0 = false;
    CellP cell;
    double W[3], anorm[3];
    double cut_vdw = 0.0, cut_coul = 0.0;
    double alphaES = 0.0;
    int kES[3] = {0, 0, 0};
    double utail = 0.0, ptail = 0.0;
    std::vector<int> natmi;
    std::vector<void*> allocs;
    // device state
    double *x = nullptr, *y = nullptr, *z = nullptr;
    double *vx = nullptr, *vy = nullptr, *vz = nullptr;
    double *fx = nullptr, *fy = nullptr, *fz = nullptr;
    double *fox = nullptr, *foy = nullptr, *foz = nullptr;
    double *sx = nullptr, *sy = nullptr, *sz = nullptr;
    double *xs = nullptr, *ys = nullptr, *zs = nullptr;
    int* type = nullptr;
    double *q = nullptr, *mass = nullptr, *alpha = nullptr, *inv_alpha = nullptr, *dip0 = nullptr;
    double *mu = nullptr, *mu_ind = nullptr, *Estat = nullptr, *Eind = nullptr, *E = nullptr;
    double *cg_r = nullptr, *cg_z = nullptr, *cg_d = nullptr, *cg_Ad = nullptr, *mu_save = nullptr;
    double* hist = nullptr;
    double* coef = nullptr;
    double *opt_xi = nullptr, *opt_g = nullptr, *opt_h = nullptr, *opt_r0 = nullptr;   // structure optimisation
    double *lb_s = nullptr, *lb_y = nullptr, *lb_w = nullptr, *lb_wa = nullptr, *lb_g0 = nullptr, *lb_sc = nullptr;
    double *m1_d = nullptr, *m1_gg = nullptr, *m1_diag = nullptr, *m1_xn = nullptr, *m1_ybar = nullptr,
           *m1_sbar = nullptr, *m1_sc = nullptr;
    int* m1_flag = nullptr;          // [0] mlis3's precision test, [2..3] max |d| as 64 bits
    int m1_indica = 0;               // mlis3's SAVEd indica, zero in a fresh process
    double *efgp_t = nullptr, *efgp_nmr = nullptr, *efgp_part = nullptr;   // EFG post-processing scratch
    int* efgp_hist = nullptr;
    size_t efgp_tcap = 0, efgp_ncap = 0, efgp_pcap = 0, efgp_hcap = 0;
    double *ef = nullptr, *efg = nullptr, *fcoul = nullptr;
    PairConst* pc = nullptr;
    NList lv, lc;
    bool shared_list = false;
    CellGrid grid;
    KGrid kg;
    RecScratch rs;
    Partials part;
    DevScalars* dsc = nullptr;
    DevScalars* hsc = nullptr;   // pinned mirror
    int* d_overflow = nullptr;
    // state
    bool have_system = false, have_list = false, forces_valid = false, md_started = false;
    int itime = 0;
    int nhist = 1;
    double e_kin = 0.0, temp_r = 0.0;
    mdff_energies en;
    double tau_nonb[9], tau_coul[9];
    int last_rebuilt = 0;
    int nrebuild = 0;
    bool rec_acc_ready = false;   // rs.aks_acc holds A_k S of the charges + final dipoles
    long long kinfo[4] = {0, 0, 0, 0};   // rectangle, half space, FP32 set, FP64 low set
    int g_dir = 16, g_dd = 16;           // lanes per atom of the real-space Ewald kernels (autotuned)
    // mixed path: per-step pair table of the dipole-dipole operator (A1, B2 per
    // Coulomb list entry), written by the charge pass of each force evaluation
    float2* ddtab = nullptr;
    int* ddnbr = nullptr;
    int* ddcnt = nullptr;
    uint4* ddrec = nullptr;              // [2n] gather records of the operator
    size_t ddtab_cap = 0;                // entries allocated
    long ddtab_epoch = -1;               // position epoch it was written for
    int ddtab_lcap = 0;                  // list capacity it was written with
    bool tuned = false;
    Prof prof;
    // cell (column-major, as given) and the constant-pressure state
    double A_cur[9] = {0};
    double omega0 = 0.0, utail0 = 0.0, ptail0 = 0.0;   // set-up cell volume and tail corrections
    NptState npt;
    // the MD step as one CUDA graph, replayed once per step (graph[0]: steps
    // without the EFG, graph[1]: EFG steps); the dipole PCG is a conditional
    // WHILE node whose test runs on the device
    cudaStream_t st2 = nullptr;          // capture stream of the PCG loop body
    bool capturing = false;
    bool graph_off = false;              // a capture failed: plain launches from then on
    bool efg_due = true;                 // this evaluation writes the EFG (efg_period)
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    StepKey gkey[2];
    long glaunch[2] = {0, 0}, gbody[2] = {0, 0};   // kernels per replay outside / per PCG iteration
    long cap_body = 0;                   // kernels of one PCG iteration, counted while capturing
    bool pcg_in_graph = false;           // the last captured step solved dipoles in the graph
    PredPlan coef_up;                    // the predictor plan on the device (coef)
    bool coef_valid = false;
    double plan_host[PLAN_LEN] = {0};    // staging of the plan upload
    long long nstep_graph = 0, ncapture = 0, nstep_plain = 0;
};

namespace {

int fail(mdff_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(ctx, MDFF_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

#define TRY(expr)                  \
    do {                           \
        int r_ = (expr);           \
        if (r_ != MDFF_OK) return r_; \
    } while (0)

template <class T>
int dalloc(mdff_ctx* ctx, T** ptr, size_t count) {
    if (count == 0) count = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, sizeof(T) * count);
    if (e != cudaSuccess) return fail(ctx, MDFF_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    ctx->allocs.push_back(p);
    *ptr = (T*)p;
    return MDFF_OK;
}

// Grow-only device scratch owned by the context.
template <class T>
int dgrow(mdff_ctx* ctx, T** ptr, size_t* cap, size_t need) {
    if (*ptr && need <= *cap) return MDFF_OK;
    if (*ptr) {
        CK(cudaStreamSynchronize(ctx->st));
        cudaFree(*ptr);
        ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void*)*ptr));
        *ptr = nullptr;
    }
    TRY(dalloc(ctx, ptr, need));
    *cap = need;
    return MDFF_OK;
}

void free_all(mdff_ctx* ctx) {
    for (void* p : ctx->allocs) cudaFree(p);
    ctx->allocs.clear();
}

int check_launch(mdff_ctx* ctx, const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ctx, MDFF_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
    return MDFF_OK;
}

int sync_scalars(mdff_ctx* ctx) {
    CK(cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->prof.harvest();
    if (ctx->hsc->tc_err)
        return fail(ctx, MDFF_E_CUDA, "tensor-core structure factor: a pipeline wait gave up (code " +
                                          std::to_string(ctx->hsc->tc_err) + ")");
    return MDFF_OK;
}

// lattice (src/lattice.f90:60-175) on the host, for A given column-major.
void lattice(const double A9[9], CellP& c, double W[3], double anorm[3]) {
    double A[3][3], B[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = A9[3 * j + i];
    auto expro = [&](int out, int a, int b) {
        B[0][out] = A[1][a] * A[2][b] - A[2][a] * A[1][b];
        B[1][out] = A[2][a] * A[0][b] - A[0][a] * A[2][b];
        B[2][out] = A[0][a] * A[1][b] - A[1][a] * A[0][b];
    };
    expro(0, 1, 2);
    expro(1, 2, 0);
    expro(2, 0, 1);
    double omega = B[0][0] * A[0][0] + B[1][0] * A[1][0] + B[2][0] * A[2][0];
    for (int j = 0; j < 3; ++j) W[j] = omega / std::sqrt(B[0][j] * B[0][j] + B[1][j] * B[1][j] + B[2][j] * B[2][j]);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) B[i][j] = B[i][j] / omega;
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += A[k][i] * A[k][i];
        anorm[i] = std::sqrt(s);
    }
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { c.A[3 * i + j] = A[i][j]; c.B[3 * i + j] = B[i][j]; }
    c.omega = omega;
}

void symmetrise(mdff_params& p) {   // field_check_tag (src/field.f90:316-339)
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

// Validation of the tags on the path (field_check_tag, md_check_tag).
int check_params(mdff_ctx* ctx, const mdff_params& p) {
    if (p.ntype < 1 || p.ntype > MDFF_NTYPE_MAX) return fail(ctx, MDFF_E_ARG, "ntype out of range");
    if (p.trunc < 0 || p.trunc > 2) return fail(ctx, MDFF_E_ARG, "ctrunc should be notrunc, linear or quadratic");
    bool nonb = p.lnmlj || p.lbmhft || p.lbmhftd || p.lmorse;
    if (nonb && p.cutshortrange <= 0.0) return fail(ctx, MDFF_E_ARG, "controltag: cutshortrange is null");
    if (p.lcoulomb && p.cutlongrange <= 0.0) return fail(ctx, MDFF_E_ARG, "controltag: cutlongrange is null");
    for (int a = 0; a < p.ntype; ++a)
        for (int b = 0; b < p.ntype; ++b)
            for (int c = 0; c < p.ntype; ++c)
                if (p.dip_pol_damp_k[a][b][c] > MDFF_TT_MAX_ORDER || p.dip_pol_damp_k[a][b][c] < 0)
                    return fail(ctx, MDFF_E_ARG, "Tang-Toennies expansion order too large (dip_pol_damp_k)");
    if (p.integrator != MDFF_NVE_VV && p.integrator != MDFF_NVT_NHCN && p.integrator != MDFF_NPT_NHCNP &&
        p.integrator != MDFF_NVT_NHC2)
        return fail(ctx, MDFF_E_UNSUPPORTED,
                    "integrator: nve-vv, nvt-nhc2, nvt-nhcn and npt-nhcnp are on the engine's path");
    if (p.integrator == MDFF_NVT_NHC2 && !(p.timesca_thermo > 0.0))
        return fail(ctx, MDFF_E_ARG, "mdtag: nvt-nhc2 needs timesca_thermo > 0");
    const bool chains = p.integrator == MDFF_NVT_NHCN || p.integrator == MDFF_NPT_NHCNP;
    if (chains && (p.nhc_n < 2 || p.nhc_n > 16))
        return fail(ctx, MDFF_E_ARG, "nhc_n = 1 is not allowed with Nose Hoover chains thermostats");
    int yo = p.nhc_yosh_order;
    if (chains && !(yo == 1 || yo == 3 || yo == 5 || yo == 7 || yo == 9))
        return fail(ctx, MDFF_E_ARG, "value of yoshida order not available");
    if (chains && p.nhc_mults < 1) return fail(ctx, MDFF_E_ARG, "nhc_mults < 1");
    if (p.integrator == MDFF_NPT_NHCNP && !(p.timesca_baro > 0.0))
        return fail(ctx, MDFF_E_ARG, "mdtag: with integrator in npt_ensemble timesca_baro should be set");
    if (p.extrapolate_order < 0 || p.extrapolate_order > 5)
        return fail(ctx, MDFF_E_ARG, "extrapolate_order should be 0 <= order <= 5");
    if (p.algo_moment_from_pola != MDFF_POLA_SCF && p.algo_moment_from_pola != MDFF_POLA_PCG)
        return fail(ctx, MDFF_E_ARG, "algo_moment_from_pola should be scf or pcg");
    if (p.algo_ext_dipole != MDFF_EXT_POLY && p.algo_ext_dipole != MDFF_EXT_ASPC)
        return fail(ctx, MDFF_E_ARG, "algo_ext_dipole should be poly or aspc");
    if (p.precision != MDFF_PREC_FP64 && p.precision != MDFF_PREC_MIXED)
        return fail(ctx, MDFF_E_ARG, "precision should be MDFF_PREC_FP64 or MDFF_PREC_MIXED");
    bool pol = false;
    for (int t = 0; t < p.ntype; ++t) if (p.ldip_polar[t]) pol = true;
    if (pol && p.lsurf) return fail(ctx, MDFF_E_UNSUPPORTED, "lsurf with polarisable ions is outside the engine's path");
    return MDFF_OK;
}

// ewald_param (src/field.f90:860-908)
void ewald_param(mdff_ctx* ctx) {
    const mdff_params& p = ctx->p;
    double rcut = 0.5 * std::min(ctx->W[0], std::min(ctx->W[1], ctx->W[2]));
    double cl = std::min(p.cutlongrange, rcut);
    double eps = std::min(std::fabs(p.epsw), 0.5);
    double tol = std::sqrt(std::fabs(std::log(eps * cl)));
    double alpha = std::sqrt(std::fabs(std::log(eps * cl * tol))) / rcut;
    double tol1 = std::sqrt(-std::log(eps * cl * (2.0 * tol * alpha) * (2.0 * tol * alpha)));
    ctx->cut_coul = cl;
    ctx->alphaES = p.alphaES;
    for (int i = 0; i < 3; ++i) ctx->kES[i] = p.kES[i];
    if (p.lautoES) {
        ctx->alphaES = alpha;
        for (int i = 0; i < 3; ++i) ctx->kES[i] = (int)std::round(0.25 + ctx->anorm[i] * alpha * tol1 / PI);
    }
}

// initialize_param_non_bonded (src/field.f90:914-1101) and the damping
// tables, packed per ordered type pair.
void build_pair_consts(mdff_ctx* ctx, std::vector<PairConst>& tab) {
    const mdff_params& p = ctx->p;
    tab.assign(NT * NT, PairConst());
    std::memset(tab.data(), 0, sizeof(PairConst) * NT * NT);
    double two16 = std::pow(2.0, 1.0 / 6.0);
    ctx->utail = ctx->ptail = 0.0;
    for (int it = 0; it < ctx->ntype; ++it)
        for (int jt = 0; jt < ctx->ntype; ++jt) {
            PairConst& P = tab[it * NT + jt];
            double pp = p.plj[it][jt], qq = p.qlj[it][jt];
            double rcut = p.cutshortrange;
            P.rcutsq = rcut * rcut;
            double rcut3 = rcut * P.rcutsq;
            double ppqq = pp * qq;
            P.epsp = p.epslj[it][jt] / (qq - pp);
            P.sigsq = two16 * two16 * p.sigmalj[it][jt] * p.sigmalj[it][jt];
            P.plj = pp;
            P.qlj = qq;
            double sr2 = P.sigsq / P.rcutsq;
            double sr = std::sqrt(sr2);
            double srp = std::pow(sr, pp), srq = std::pow(sr, qq);
            P.uc = P.epsp * (pp * srq - qq * srp);
            P.uc1 = P.epsp * ppqq / (2.0 * P.rcutsq) * (srq - srp);
            P.uc2 = 0.5 * P.epsp * ((2.0 * pp + ppqq) * srq - (2.0 * qq + ppqq) * srp);
            P.fc = ppqq * P.epsp / P.sigsq;
            double ut = P.epsp * (pp * srq / (qq - 3.0) - qq * srp / (pp - 3.0)) * rcut3 * 2.0 * PI;
            double pt = ppqq * P.epsp * (srq / (qq - 3.0) - srp / (pp - 3.0)) * rcut3 * 2.0 * PI;
            if (ctx->natmi[it] != 0 && ctx->natmi[jt] != 0) {
                ctx->utail += ut * ctx->natmi[it] * ctx->natmi[jt] / ctx->cell.omega;
                ctx->ptail += pt * ctx->natmi[it] * ctx->natmi[jt] / ctx->cell.omega;
            }
            P.A = p.Abmhftd[it][jt];
            P.B = p.Bbmhftd[it][jt];
            P.C = p.Cbmhftd[it][jt];
            P.D = p.Dbmhftd[it][jt];
            P.BD = p.BDbmhftd[it][jt];
            P.epsmor = p.epsmor[it][jt];
            P.rhomor = p.rhomor[it][jt];
            P.rs = std::exp(p.rhomor[it][jt] * p.sigmamor[it][jt]);
            P.db_i = p.dip_pol_damp_b[it][it][jt];
            P.dc_i = p.dip_pol_damp_c[it][it][jt];
            P.dk_i = p.dip_pol_damp_k[it][it][jt];
            P.db_j = p.dip_pol_damp_b[jt][it][jt];
            P.dc_j = p.dip_pol_damp_c[jt][it][jt];
            P.dk_j = p.dip_pol_damp_k[jt][it][jt];
            P.ldamp = (p.ldip_damping[it][it][jt] || p.ldip_damping[jt][it][jt]) ? 1 : 0;
        }
    ctx->ptail = ctx->ptail / ctx->u.press / ctx->cell.omega / 3.0;
}

double rlist_max(const mdff_ctx* ctx, double skin) {
    double r = 0.0;
    bool nonb = ctx->p.lnmlj || ctx->p.lbmhft || ctx->p.lbmhftd || ctx->p.lmorse;
    if (nonb) r = std::max(r, ctx->cut_vdw + skin);
    if (ctx->p.lcoulomb) r = std::max(r, ctx->cut_coul + skin);
    return r;
}

int ensure_lists(mdff_ctx* ctx, int cap) {
    bool nonb = ctx->p.lnmlj || ctx->p.lbmhft || ctx->p.lbmhftd || ctx->p.lmorse;
    ctx->shared_list = !(nonb && ctx->p.lcoulomb) || (ctx->cut_vdw == ctx->cut_coul);
    auto alloc_list = [&](NList& L) -> int {
        if (L.cap >= cap && L.nbr) return MDFF_OK;
        if (L.nbr) { cudaFree(L.nbr); ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void*)L.nbr)); L.nbr = nullptr; }
        TRY(dalloc(ctx, &L.nbr, (size_t)ctx->n * cap));
        if (!L.cnt) TRY(dalloc(ctx, &L.cnt, (size_t)ctx->n));
        L.cap = cap;
        return MDFF_OK;
    };
    TRY(alloc_list(ctx->lv));
    if (!ctx->shared_list) TRY(alloc_list(ctx->lc));
    return MDFF_OK;
}

// vnlist_pbc (src/tools.f90:274-370): both lists at the current positions
// (from_frac: at the fractional coordinates already in sx, sy, sz).
int build_lists(mdff_ctx* ctx, double skin, bool from_frac = false) {
    const int n = ctx->n;
    double rl = rlist_max(ctx, skin);
    if (rl <= 0.0) return MDFF_OK;
    CellGrid& g = ctx->grid;
    for (int d = 0; d < 3; ++d) {
        int nc = (int)std::floor(ctx->W[d] / (rl * (1.0 + 1e-12)));
        g.nc[d] = std::max(1, std::min(nc, 256));
    }
    g.ncell = g.nc[0] * g.nc[1] * g.nc[2];
    if (g.ncell > g.ncell_alloc) {
        TRY(dalloc(ctx, &g.cell_count, g.ncell));
        TRY(dalloc(ctx, &g.cell_start, g.ncell + 1));
        TRY(dalloc(ctx, &g.cell_cursor, g.ncell));
        g.ncell_alloc = g.ncell;
    }
    ctx->prof.begin(PK_NLIST);
    if (!from_frac) launch_frac(ctx->st, n, ctx->x, ctx->y, ctx->z, ctx->cell, ctx->sx, ctx->sy, ctx->sz);
    launch_bin(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, g);
    ctx->prof.end(5);
    bool nonb = ctx->p.lnmlj || ctx->p.lbmhft || ctx->p.lbmhftd || ctx->p.lmorse;
    double cut_a = nonb ? ctx->cut_vdw : ctx->cut_coul;
    for (int attempt = 0; attempt < 4; ++attempt) {
        double ra = cut_a + skin, rb = ctx->cut_coul + skin;
        CK(cudaMemsetAsync(ctx->d_overflow, 0, sizeof(int), ctx->st));
        ctx->prof.begin(PK_NLIST);
        launch_nlist(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->cell, g, ra * ra, ctx->lv, rb * rb,
                     ctx->shared_list ? nullptr : &ctx->lc, ctx->d_overflow);
        ctx->prof.end(1);
        TRY(check_launch(ctx, "nlist"));
        int ovf = 0;
        CK(cudaMemcpyAsync(&ovf, ctx->d_overflow, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (ovf == 0) break;
        if (attempt == 3) return fail(ctx, MDFF_E_LISTOVF, "neighbour list capacity exceeded");
        int cap = (int)(ovf * 1.25) + 32;
        TRY(ensure_lists(ctx, cap));
    }
    ctx->lv.cut = cut_a;
    ctx->lc.cut = ctx->cut_coul;
    CK(cudaMemcpyAsync(ctx->xs, ctx->sx, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->ys, ctx->sy, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->zs, ctx->sz, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    ctx->have_list = true;
    ctx->nrebuild++;
    ctx->npt.scale_build = ctx->npt.scale;
    std::memcpy(ctx->npt.A_build, ctx->A_cur, sizeof ctx->A_cur);
    return MDFF_OK;
}

const NList& coul_list(const mdff_ctx* ctx) { return ctx->shared_list ? ctx->lv : ctx->lc; }

__global__ void k_axpy(int n, double a, const double* x, double* y) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) y[t] = fma(a, x[t], y[t]);
}

__global__ void k_add3(int n, const double* a, const double* b, double* out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = a[t] + b[t];
}

// Final assembly of multipole_ES (src/field.f90:1930-1990): self (and surface)
// terms, coul_unit, forces added to the total.
// The surface term uses the total charge and dipole moments (sums of q r and
// mu) reduced into the device scalars by the same evaluation.
__global__ void k_coul_finish(int n, const double* q, const double* mu, double* ef, double* efg, const double* fc,
                              double* fx, double* fy, double* fz, double selfa2, double cu, int do_efg, int lsurf,
                              const DevScalars* __restrict__ d, double fpi_3V) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double qi = q[i];
    const double sv[3] = {d->sums[2] + d->sums[5], d->sums[3] + d->sums[6], d->sums[4] + d->sums[7]};
    const double s0 = sv[0], s1 = sv[1], s2 = sv[2];
    for (int c = 0; c < 3; ++c) {
        double e = ef[(size_t)c * n + i] + 2.0 * selfa2 * mu[(size_t)c * n + i];
        if (lsurf) e += sv[c];
        ef[(size_t)c * n + i] = e;
    }
    if (do_efg) {
        for (int k = 0; k < 6; ++k) {
            double v = efg[(size_t)k * n + i];
            if (k < 3) v += -2.0 * selfa2 * qi;
            efg[(size_t)k * n + i] = v * cu;
        }
    }
    double f0 = fc[i], f1 = fc[n + i], f2 = fc[2 * n + i];
    if (lsurf) { f0 += -qi * s0 * fpi_3V; f1 += -qi * s1 * fpi_3V; f2 += -qi * s2 * fpi_3V; }
    fx[i] += f0 * cu;
    fy[i] += f1 * cu;
    fz[i] += f2 * cu;
}

inline int nb(int n, int t = 256) { return (n + t - 1) / t; }

double selfa(const mdff_ctx* ctx) { return ctx->alphaES / std::sqrt(PI); }
double selfa2(const mdff_ctx* ctx) { return 2.0 * selfa(ctx) * ctx->alphaES * ctx->alphaES / 3.0; }

DirFlags dir_flags(const mdff_ctx* ctx) {
    DirFlags f;
    std::memset(&f, 0, sizeof f);
    f.ntype = ctx->ntype;
    f.alpha = ctx->alphaES;
    f.cutsq = ctx->cut_coul * ctx->cut_coul;
    f.erfc_ref = ctx->p.erfc_ref ? 1 : 0;
    return f;
}

// Field of the induced dipoles: real space (dipole-dipole, undamped) +
// reciprocal space + self term; src/field.f90:3354-3357.
// Real-space part of the dipole field operator: FP64 (MODE 1 of
// k_ewald_dir) or, on the mixed path, FP32 arithmetic from the fixed-point
// coordinates (k_ewald_dd32).
void dd_field_real(mdff_ctx* ctx, const double* m, double* out) {
    const int n = ctx->n;
    ctx->prof.begin(PK_DIR);
    if (ctx->p.precision == MDFF_PREC_MIXED) {
        const int k = 1 + ensure_phase_tables(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->rs);
        const NList& L = coul_list(ctx);
        if (ctx->ddtab_epoch == ctx->rs.want_epoch && ctx->ddtab_lcap == L.cap)
            launch_ewald_ddtab(ctx->st, n, ctx->rs.fixed, m, ctx->cell, ctx->ddnbr, ctx->ddcnt, L.cap, ctx->ddtab,
                               ctx->ddrec, out, ctx->g_dd);
        else
            launch_ewald_dd32(ctx->st, n, ctx->rs.fixed, m, ctx->cell, L, ctx->cut_coul * ctx->cut_coul,
                              ctx->alphaES, out, ctx->g_dd);
        ctx->prof.end(k);
        return;
    }
    DirFlags f = dir_flags(ctx);
    f.dd = 1;
    f.field = 1;
    launch_ewald_dir(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->type, nullptr, m, ctx->cell, coul_list(ctx), ctx->pc,
                     f, out, nullptr, nullptr, ctx->part, ctx->dsc, ctx->g_dir);
    ctx->prof.end(1);
}

// self = false leaves out the self term 2 selfa2 m (the PCG iteration adds
// it in k_cg_apply).
int induced_field(mdff_ctx* ctx, const double* m, double* out, bool self = true) {
    const int n = ctx->n;
    dd_field_real(ctx, m, out);
    RecFlags rf{0, 1, 1, 0, 0, 0, ctx->p.precision, 0};
    launch_ewald_rec(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, nullptr, m, ctx->cell, ctx->kg, rf, ctx->rs, out, nullptr,
                     nullptr, ctx->part, ctx->dsc, &ctx->prof);
    if (self) {
        ctx->prof.begin(PK_SOLVER);
        k_axpy<<<nb(3 * n), 256, 0, ctx->st>>>(3 * n, 2.0 * selfa2(ctx), m, out);
        ctx->prof.end(1);
    }
    return check_launch(ctx, "induced_field");
}

// On the mixed path, let this charge pass also write the dipole-dipole pair
// table for the solver's operator (allocated for the current list capacity).
int arm_ddtab(mdff_ctx* ctx, DirFlags& f) {
    if (ctx->p.precision != MDFF_PREC_MIXED) return MDFF_OK;
    const NList& L = coul_list(ctx);
    const size_t need = (size_t)ctx->n * L.cap;
    if (need > ctx->ddtab_cap) {
        if (ctx->ddtab) CK(cudaFree(ctx->ddtab));
        if (ctx->ddnbr) CK(cudaFree(ctx->ddnbr));
        ctx->ddtab = nullptr;
        ctx->ddnbr = nullptr;
        ctx->ddtab_cap = 0;
        cudaError_t e = cudaMalloc(&ctx->ddtab, sizeof(float2) * need);
        if (e == cudaSuccess) e = cudaMalloc(&ctx->ddnbr, sizeof(int) * need);
        if (e != cudaSuccess) return fail(ctx, MDFF_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        ctx->ddtab_cap = need;
    }
    if (!ctx->ddcnt) TRY(dalloc(ctx, &ctx->ddcnt, ctx->n));
    if (!ctx->ddrec) TRY(dalloc(ctx, &ctx->ddrec, 2 * (size_t)ctx->n));
    f.ddtab = ctx->ddtab;
    f.ddnbr = ctx->ddnbr;
    f.ddcnt = ctx->ddcnt;
    ctx->ddtab_epoch = ctx->rs.want_epoch;
    ctx->ddtab_lcap = L.cap;
    return MDFF_OK;
}

// Static field of the charges (and static dipoles), damped
// (src/field.f90:3270-3272).
int static_field(mdff_ctx* ctx) {
    const int n = ctx->n;
    DirFlags f = dir_flags(ctx);
    f.qq = 1;
    f.qd = ctx->any_dip0 ? 1 : 0;
    f.dd = ctx->any_dip0 ? 1 : 0;
    f.damp = 1;
    f.field = 1;
    TRY(arm_ddtab(ctx, f));
    ctx->prof.begin(PK_DIR);
    launch_ewald_dir(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->type, ctx->q, ctx->dip0, ctx->cell, coul_list(ctx),
                     ctx->pc, f, ctx->Estat, nullptr, nullptr, ctx->part, ctx->dsc, ctx->g_dir);
    ctx->prof.end(2);
    RecFlags rf{1, ctx->any_dip0 ? 1 : 0, 1, 0, 0, 0, ctx->p.precision, 0};
    launch_ewald_rec(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->q, ctx->dip0, ctx->cell, ctx->kg, rf, ctx->rs,
                     ctx->Estat, nullptr, nullptr, ctx->part, ctx->dsc, &ctx->prof);
    ctx->prof.begin(PK_SOLVER);
    k_axpy<<<nb(3 * n), 256, 0, ctx->st>>>(3 * n, 2.0 * selfa2(ctx), ctx->dip0, ctx->Estat);
    ctx->prof.end(1);
    return check_launch(ctx, "static_field");
}

// Static field and the field of the initial guess x0 (mu_ind) together, for
// the PCG's first residual r0 = b - A x0 (kspace_reuse): the real-space parts
// are the same two sums as static_field / induced_field, the reciprocal part is
// ONE evaluation of the sources q + dip0 + x0 added to Estat (r0 only needs the
// sum), and its A_k S is the starting value of the solver's accumulator.
int fused_initial_field(mdff_ctx* ctx) {
    const int n = ctx->n, n3 = 3 * n;
    DirFlags f = dir_flags(ctx);
    f.qq = 1;
    f.qd = ctx->any_dip0 ? 1 : 0;
    f.dd = ctx->any_dip0 ? 1 : 0;
    f.damp = 1;
    f.field = 1;
    TRY(arm_ddtab(ctx, f));
    ctx->prof.begin(PK_DIR);
    launch_ewald_dir(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->type, ctx->q, ctx->dip0, ctx->cell, coul_list(ctx),
                     ctx->pc, f, ctx->Estat, nullptr, nullptr, ctx->part, ctx->dsc, ctx->g_dir);
    ctx->prof.end(2);
    dd_field_real(ctx, ctx->mu_ind, ctx->Eind);
    ctx->prof.begin(PK_OTHER);
    k_add3<<<nb(n3), 256, 0, ctx->st>>>(n3, ctx->dip0, ctx->mu_ind, ctx->mu);   // ctx->mu as scratch
    ctx->prof.end(1);
    RecFlags rf{1, 1, 1, 0, 0, 0, ctx->p.precision, 0};
    launch_ewald_rec(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->q, ctx->mu, ctx->cell, ctx->kg, rf, ctx->rs,
                     ctx->Estat, nullptr, nullptr, ctx->part, ctx->dsc, &ctx->prof);
    ctx->prof.begin(PK_SOLVER);
    launch_aks_accumulate(ctx->st, ctx->kg, ctx->rs, ctx->dsc, 1);
    k_axpy<<<nb(n3), 256, 0, ctx->st>>>(n3, 2.0 * selfa2(ctx), ctx->dip0, ctx->Estat);
    k_axpy<<<nb(n3), 256, 0, ctx->st>>>(n3, 2.0 * selfa2(ctx), ctx->mu_ind, ctx->Eind);
    ctx->prof.end(ctx->rs.low.ncol > 0 ? 4 : 3);
    return check_launch(ctx, "fused_initial_field");
}

// The predictor of the current step (extrapolate_dipole_poly,
// src/field.f90:3807-3920; ASPC predictor, src/field.f90:3924-3984):
// coefficients, mode (0: linear combination, 1: polynomial), points and the
// history slots to shift.  Constant once itime exceeds the order.
PredPlan pred_plan(const mdff_ctx* ctx) {
    const int ord = ctx->p.extrapolate_order;
    const int itime = ctx->itime;
    PredPlan pl;
    std::memset(&pl, 0, sizeof pl);
    double* coef = pl.coef;
    int mode = 0, npt = 1, shift_from = 0;   // shift history slots [shift_from..1] down by one
    if (ctx->p.algo_ext_dipole == MDFF_EXT_ASPC) {
        int eo = (itime >= ord + 1) ? ord : ((itime == 1 || itime == 0) ? 0 : itime - 1);
        static const double B[6][6] = {{1.0},
                                       {2.0, -1.0},
                                       {2.5, -2.0, 0.5},
                                       {2.8, -2.8, 1.2, -0.2},
                                       {3.0, -24.0 / 7.0, 27.0 / 14.0, -4.0 / 7.0, 1.0 / 14.0},
                                       {22.0 / 7.0, -55.0 / 14.0, 55.0 / 21.0, -22.0 / 21.0, 5.0 / 21.0, -1.0 / 42.0}};
        for (int k = 0; k <= eo; ++k) coef[k] = B[eo][k];
        npt = eo + 1;
        shift_from = eo;
    } else if (ord == 0) {
        coef[0] = 1.0;
    } else if (ord == 1) {
        if (itime > 1) { coef[0] = 2.0; coef[1] = -1.0; npt = 2; }
        else coef[0] = 1.0;
        shift_from = 1;
    } else {
        if (itime > ord) { mode = 1; npt = ord + 1; }
        else if (itime <= 1) { coef[0] = 1.0; }
        else if (itime == 2) { coef[0] = 2.0; coef[1] = -1.0; npt = 2; }
        else { mode = 1; npt = itime + 1; }
        shift_from = ord;
    }
    pl.mode = mode;
    pl.npt = npt;
    pl.shift_from = shift_from;
    return pl;
}

// The predictor's plan of this step into device memory, when it changed (on
// the stream, ahead of the step's kernels; never inside a capture, so the
// captured step reads whatever plan is current when it is replayed).
int upload_plan(mdff_ctx* ctx) {
    const PredPlan pl = pred_plan(ctx);
    if (ctx->coef_valid && std::memcmp(&pl, &ctx->coef_up, sizeof pl) == 0) return MDFF_OK;
    if (ctx->capturing) return fail(ctx, MDFF_E_STATE, "predictor plan changed inside a captured step");
    ctx->coef_up = pl;
    ctx->coef_valid = true;
    for (int k = 0; k < 16; ++k) ctx->plan_host[k] = pl.coef[k];
    ctx->plan_host[16] = pl.mode;
    ctx->plan_host[17] = pl.npt;
    ctx->plan_host[18] = pl.shift_from;
    CK(cudaMemcpyAsync(ctx->coef, ctx->plan_host, sizeof(double) * PLAN_LEN, cudaMemcpyHostToDevice, ctx->st));
    return MDFF_OK;
}

// Extrapolated initial guess from the stored history, then the history
// shifted down by the plan's slot count.
int predict(mdff_ctx* ctx, double* x) {
    const int n3 = 3 * ctx->n;
    TRY(upload_plan(ctx));
    ctx->prof.begin(PK_SOLVER);
    k_extrapolate<<<nb(n3), 256, 0, ctx->st>>>(n3, ctx->hist, ctx->coef, x);
    k_hist_shift<<<nb(n3), 256, 0, ctx->st>>>(n3, ctx->hist, ctx->coef);
    ctx->prof.end(2);
    return check_launch(ctx, "predict");
}

// Induced dipoles: moment_from_pola_scf (src/field.f90:3200-3458) or PCG.
int solve_dipoles(mdff_ctx* ctx) {
    const int n = ctx->n, n3 = 3 * n;
    const mdff_params& p = ctx->p;
    DevScalars* d = ctx->dsc;
    const bool reuse = p.kspace_reuse && p.algo_moment_from_pola == MDFF_POLA_PCG;
    ctx->rec_acc_ready = false;
    if (!reuse) TRY(static_field(ctx));
    const double inv_npol = 1.0 / (double)ctx->npol;
    int iscf = 0;
    double rmsd = 1e300;
    int vb = std::min(592, nb(n3));
    if (p.algo_moment_from_pola == MDFF_POLA_SCF) {
        bool aspc = p.algo_ext_dipole == MDFF_EXT_ASPC;
        while (((iscf < p.max_scf_pol_iter) && (rmsd > p.conv_tol_ind)) || (iscf < p.min_scf_pol_iter)) {
            iscf++;
            if (iscf != 1) {
                ctx->prof.begin(PK_SOLVER);
                k_induced_moment<<<nb(n3), 256, 0, ctx->st>>>(n, ctx->E, ctx->alpha, ctx->mu_ind);
                ctx->prof.end(1);
            } else {
                TRY(predict(ctx, ctx->mu_ind));
            }
            TRY(induced_field(ctx, ctx->mu_ind, ctx->Eind));
            if (iscf == 1 && aspc) {
                // ASPC corrector: mu = w alpha E + (1-w) mu_p (src/field.f90:3986-3991)
                int ord = p.extrapolate_order, itime = ctx->itime;
                int eo = (itime >= ord + 1) ? ord : ((itime == 1 || itime == 0) ? 0 : itime - 1);
                static const double W[6] = {0.0, 2.0 / 3.0, 0.6, 4.0 / 7.0, 5.0 / 9.0, 6.0 / 11.0};
                ctx->prof.begin(PK_SOLVER);
                k_aspc_correct<<<nb(n3), 256, 0, ctx->st>>>(n, ctx->Estat, ctx->Eind, ctx->alpha, W[eo], ctx->mu_ind);
                ctx->prof.end(1);
            }
            ctx->prof.begin(PK_SOLVER);
            k_scf_residual<<<vb, 256, 0, ctx->st>>>(n, ctx->Estat, ctx->Eind, ctx->mu_ind, ctx->inv_alpha, ctx->E,
                                                    ctx->part.buf);
            launch_reduce_partials(ctx->st, ctx->part.buf, vb, 1, &d->rr, 0);
            ctx->prof.end(2);
            TRY(sync_scalars(ctx));
            rmsd = std::sqrt(ctx->hsc->rr * inv_npol);
        }
    } else {
        TRY(predict(ctx, ctx->mu_ind));
        // zero the guess on non-polarisable atoms: Ad = A x uses the mask
        if (reuse) TRY(fused_initial_field(ctx));
        else TRY(induced_field(ctx, ctx->mu_ind, ctx->Eind));
        ctx->prof.begin(PK_SOLVER);
        k_apply_A<<<nb(n3), 256, 0, ctx->st>>>(n, ctx->mu_ind, ctx->Eind, ctx->inv_alpha, ctx->cg_Ad);
        k_cg_init<<<vb, 256, 0, ctx->st>>>(n, ctx->Estat, ctx->cg_Ad, ctx->alpha, ctx->inv_alpha, ctx->cg_r, ctx->cg_z,
                                           ctx->cg_d, ctx->part.buf);
        launch_reduce_partials(ctx->st, ctx->part.buf, vb, 2, &d->rr, 0);
        k_cg_first<<<1, 32, 0, ctx->st>>>(d, inv_npol);
        ctx->prof.end(4);
        // one PCG iteration (the body of the loop, on the device): the
        // operator, then k_cg_apply (self term, Ad, d.Ad partials),
        // k_cg_update2 (x, r, z and the r.r, r.z partials), the structure
        // factors' step, k_cg_direction2; the caller adds the scalars' update
        // (k_cg_fin, or k_cg_fincond with the loop test).  The two partial
        // sets live apart in the scratch so that each kernel reduces the
        // previous one's while writing its own.
        double* dpart = ctx->part.buf + 4096;
        auto iteration = [&]() -> int {
            TRY(induced_field(ctx, ctx->cg_d, ctx->Eind, false));
            ctx->prof.begin(PK_SOLVER);
            k_cg_apply<<<vb, 256, 0, ctx->st>>>(n, ctx->cg_d, ctx->Eind, 2.0 * selfa2(ctx), ctx->inv_alpha, ctx->cg_Ad,
                                               dpart);
            k_cg_update2<<<vb, 256, 0, ctx->st>>>(n, ctx->cg_d, ctx->cg_Ad, ctx->alpha, ctx->mu_ind, ctx->cg_r,
                                                 ctx->cg_z, d, dpart, vb, ctx->part.buf);
            // the same step on the structure factors (before rz advances)
            if (reuse) launch_aks_accumulate(ctx->st, ctx->kg, ctx->rs, d, 0);
            k_cg_direction2<<<nb(n3), 256, 0, ctx->st>>>(n3, ctx->cg_z, ctx->cg_d, d, ctx->part.buf, vb);
            ctx->prof.end(3 + (reuse ? (ctx->rs.low.ncol > 0 ? 2 : 1) : 0));
            return check_launch(ctx, "pcg iteration");
        };
        if (ctx->capturing) {
            // inside a captured MD step: a conditional WHILE node whose body is
            // one iteration and whose test (k_cg_cond) runs on the device after
            // k_cg_first and after each iteration; the host reads the count
            // and the residual after the step (solve_finish)
            cudaStreamCaptureStatus cs;
            cudaGraph_t g = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            CK(cudaStreamGetCaptureInfo(ctx->st, &cs, nullptr, &g, nullptr, nullptr));
            cudaGraphConditionalHandle h;
            CK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
            k_cg_cond<<<1, 32, 0, ctx->st>>>(d, p.max_scf_pol_iter, p.conv_tol_ind, h);
            TRY(check_launch(ctx, "pcg test"));
            CK(cudaStreamGetCaptureInfo(ctx->st, &cs, nullptr, &g, &deps, &nd));
            alignas(cudaGraphNodeParams) unsigned char cp_raw[sizeof(cudaGraphNodeParams)];   // holds a union
            std::memset(cp_raw, 0, sizeof cp_raw);
            cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_raw);
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            CK(cudaGraphAddNode(&node, g, deps, nd, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            CK(cudaStreamUpdateCaptureDependencies(ctx->st, &node, 1, cudaStreamSetCaptureDependencies));
            const cudaStream_t main_st = ctx->st;
            const long l0 = ctx->prof.launches;
            ctx->st = ctx->st2;
            cudaError_t e = cudaStreamBeginCaptureToGraph(ctx->st, body, nullptr, nullptr, 0,
                                                          cudaStreamCaptureModeThreadLocal);
            int r = MDFF_OK;
            if (e != cudaSuccess) {
                r = fail(ctx, MDFF_E_CUDA, std::string("capture of the PCG body: ") + cudaGetErrorString(e));
            } else {
                r = iteration();
                if (r == MDFF_OK) {
                    k_cg_fincond<<<1, 32, 0, ctx->st>>>(d, inv_npol, p.conv_tol_ind, p.max_scf_pol_iter, h);
                    r = check_launch(ctx, "pcg test");
                }
                cudaGraph_t out = body;
                cudaError_t e2 = cudaStreamEndCapture(ctx->st, &out);
                if (r == MDFF_OK && e2 != cudaSuccess)
                    r = fail(ctx, MDFF_E_CUDA, std::string("capture of the PCG body: ") + cudaGetErrorString(e2));
            }
            ctx->st = main_st;
            ctx->cap_body = ctx->prof.launches - l0 + 1;   // + the loop test
            ctx->prof.launches = l0 + 1;                    // the test before the loop
            TRY(r);
            ctx->pcg_in_graph = true;
            iscf = 0;
            rmsd = 0.0;
        } else {
            TRY(sync_scalars(ctx));
            rmsd = ctx->hsc->rmsd;
            while ((iscf < p.max_scf_pol_iter && rmsd > p.conv_tol_ind) || iscf < 1) {
                iscf++;
                TRY(iteration());
                k_cg_fin<<<1, 32, 0, ctx->st>>>(d, inv_npol, p.conv_tol_ind);
                ctx->prof.launches += 1;
                TRY(sync_scalars(ctx));
                rmsd = ctx->hsc->rmsd;
                if (!std::isfinite(rmsd)) return fail(ctx, MDFF_E_NONFINITE, "non-finite residual in the dipole solve");
            }
        }
    }
    TRY(check_launch(ctx, "solve_dipoles"));
    // u_pol = 1/2 mu.alpha^-1.mu (induced_moment, src/field.f90:1780-1790)
    ctx->prof.begin(PK_SOLVER);
    k_upol<<<vb, 256, 0, ctx->st>>>(n, ctx->mu_ind, ctx->inv_alpha, ctx->part.buf);
    launch_reduce_partials(ctx->st, ctx->part.buf, vb, 1, d->upol, 0);
    ctx->prof.end(2);
    // store the induced dipoles at t (src/field.f90:3440)
    CK(cudaMemcpyAsync(ctx->hist, ctx->mu_ind, sizeof(double) * n3, cudaMemcpyDeviceToDevice, ctx->st));
    ctx->rec_acc_ready = reuse;
    if (ctx->capturing) return MDFF_OK;   // solve_finish after the step
    ctx->en.scf_iter = iscf;
    ctx->en.scf_rmsd = rmsd;
    if (iscf >= p.max_scf_pol_iter && rmsd > p.conv_tol_ind && p.algo_moment_from_pola == MDFF_POLA_PCG)
        return fail(ctx, MDFF_E_NOCONV, "induced-dipole solve did not converge within max_scf_pol_iter");
    return MDFF_OK;
}

// After a step that ran as a graph: the PCG's count and residual from the
// device scalars, with the host loop's checks.
int solve_finish(mdff_ctx* ctx) {
    const DevScalars& h = *ctx->hsc;
    ctx->en.scf_iter = h.iter;
    ctx->en.scf_rmsd = h.rmsd;
    if (!std::isfinite(h.rmsd)) return fail(ctx, MDFF_E_NONFINITE, "non-finite residual in the dipole solve");
    if (h.iter >= ctx->p.max_scf_pol_iter && h.rmsd > ctx->p.conv_tol_ind)
        return fail(ctx, MDFF_E_NOCONV, "induced-dipole solve did not converge within max_scf_pol_iter");
    return MDFF_OK;
}

// Autotuner (autotune != 0): on the first force evaluation, time every
// candidate launch shape of the Ewald kernels on this system's own data with
// CUDA events on the context's stream (one warm-up launch, then three timed
// ones) and keep the fastest: lanes per atom of the real-space kernels
// (8, 16, 32), and on the mixed path the atom split of the FP32 structure
// factor and the column split of the FP32 field (x 1/2, 1, 2 of the default).
// The candidates compute the same sums in a different order; the launches
// write only scratch that the evaluation overwrites.
float time_launch(mdff_ctx* ctx, const std::function<void()>& fn) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    fn();
    cudaEventRecord(a, ctx->st);
    for (int r = 0; r < 3; ++r) fn();
    cudaEventRecord(b, ctx->st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / 3.f;
}

int autotune(mdff_ctx* ctx) {
    ctx->tuned = true;
    if (!ctx->p.lcoulomb) return MDFF_OK;
    const int n = ctx->n;
    const bool prof_on = ctx->prof.on;
    const long launches = ctx->prof.launches;
    ctx->prof.on = false;
    CK(cudaMemsetAsync(ctx->mu, 0, sizeof(double) * 3 * n, ctx->st));
    const int gs[3] = {8, 16, 32};
    // three interleaved rounds over the candidates, each scored by its fastest
    // round: a single disturbed measurement (one pass picked a shape 20 %
    // slower in the solve) does not decide the shape
    auto pick = [&](const std::function<void(int)>& run, const int* cand, int nc) {
        std::vector<float> tmin((size_t)nc, 1e30f);
        for (int round = 0; round < 3; ++round)
            for (int k = 0; k < nc; ++k) tmin[k] = std::min(tmin[k], time_launch(ctx, [&] { run(cand[k]); }));
        int best = 0;
        for (int k = 1; k < nc; ++k)
            if (tmin[k] < tmin[best]) best = k;
        return cand[best];
    };
    DirFlags f = dir_flags(ctx);
    f.qq = 1;
    f.qd = 1;
    f.dd = 1;
    f.damp = 1;
    f.field = 1;
    f.forces = 1;
    ctx->g_dir = pick([&](int g) {
        launch_ewald_dir(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->type, ctx->q, ctx->mu, ctx->cell, coul_list(ctx),
                         ctx->pc, f, ctx->ef, nullptr, ctx->fcoul, ctx->part, ctx->dsc, g);
    }, gs, 3);
    if (ctx->p.precision == MDFF_PREC_MIXED) {
        ensure_phase_tables(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->rs);
        // the pair table of this step, then the lanes per atom of its operator
        DirFlags fs = dir_flags(ctx);
        fs.qq = 1;
        fs.damp = 1;
        fs.field = 1;
        TRY(arm_ddtab(ctx, fs));
        launch_ewald_dir(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->type, ctx->q, ctx->mu, ctx->cell, coul_list(ctx),
                         ctx->pc, fs, ctx->Estat, nullptr, nullptr, ctx->part, ctx->dsc, ctx->g_dir);
        ctx->g_dd = pick([&](int g) {
            launch_ewald_ddtab(ctx->st, n, ctx->rs.fixed, ctx->mu, ctx->cell, ctx->ddnbr, ctx->ddcnt,
                               coul_list(ctx).cap, ctx->ddtab, ctx->ddrec, ctx->Eind, g);
        }, gs, 3);
        const int muls[3] = {1, 2, 4};
        RecFlags sf{1, 1, 0, 0, 0, 0, MDFF_PREC_MIXED, 0};   // structure factor only
        ctx->rs.p_mul = pick([&](int m) {
            ctx->rs.p_mul = m;
            launch_ewald_rec(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->q, ctx->mu, ctx->cell, ctx->kg, sf, ctx->rs,
                             nullptr, nullptr, nullptr, ctx->part, ctx->dsc, &ctx->prof);
        }, muls, 3);
        RecFlags fe{1, 1, 1, 0, 0, 0, MDFF_PREC_MIXED, 0};   // with the field pass
        ctx->rs.s_mul = pick([&](int m) {
            ctx->rs.s_mul = m;
            launch_ewald_rec(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->q, ctx->mu, ctx->cell, ctx->kg, fe, ctx->rs,
                             ctx->ef, nullptr, nullptr, ctx->part, ctx->dsc, &ctx->prof);
        }, muls, 3);
    }
    ctx->prof.on = prof_on;
    ctx->prof.launches = launches;
    return check_launch(ctx, "autotune");
}

int engforce_finish(mdff_ctx* ctx);

// engforce_driver (src/field.f90:1111-1166) on the device; results stay in
// device memory and ctx->hsc/en after the trailing sync.  Inside a captured
// step only the launches are recorded (engforce_finish runs after the step).
// The EFG is written when doefg and the evaluation is due one (efg_due:
// every efg_period MD steps, always outside MD).
int engforce_device(mdff_ctx* ctx) {
    const int n = ctx->n;
    const mdff_params& p = ctx->p;
    const bool efg = p.doefg && ctx->efg_due;
    if (!p.lvnlist) TRY(build_lists(ctx, 0.0));
    else if (!ctx->have_list) TRY(build_lists(ctx, p.skindiff));   // lists dropped (an interrupted RMC chain)
    ctx->prof.begin(PK_OTHER);
    launch_frac(ctx->st, n, ctx->x, ctx->y, ctx->z, ctx->cell, ctx->sx, ctx->sy, ctx->sz);
    ctx->prof.end(1);
    ctx->rs.want_epoch++;   // positions may have changed: rebuild the phase tables
    if (p.autotune && !ctx->tuned) TRY(autotune(ctx));
    std::memset(&ctx->en, 0, sizeof ctx->en);
    bool nonb = p.lnmlj || p.lbmhft || p.lbmhftd || p.lmorse;
    if (nonb) {
        PairFlags fl{p.lnmlj, p.lbmhft, p.lbmhftd, p.lmorse, p.trunc, ctx->ntype};
        ctx->prof.begin(PK_PAIR);
        launch_pair(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->type, ctx->cell, ctx->lv, ctx->pc, fl, ctx->fx, ctx->fy,
                    ctx->fz, ctx->part, ctx->dsc);
        ctx->prof.end(2);
    } else {
        CK(cudaMemsetAsync(ctx->fx, 0, sizeof(double) * n, ctx->st));
        CK(cudaMemsetAsync(ctx->fy, 0, sizeof(double) * n, ctx->st));
        CK(cudaMemsetAsync(ctx->fz, 0, sizeof(double) * n, ctx->st));
        CK(cudaMemsetAsync(ctx->dsc->nonb, 0, sizeof(double) * 12, ctx->st));
    }
    TRY(check_launch(ctx, "pair"));
    CK(cudaMemsetAsync(ctx->dsc->upol, 0, sizeof(double) * 2, ctx->st));
    if (p.lcoulomb) {
        const int n3 = 3 * n;
        if (ctx->npol > 0) {
            TRY(solve_dipoles(ctx));
            ctx->prof.begin(PK_OTHER);
            k_add3<<<nb(n3), 256, 0, ctx->st>>>(n3, ctx->dip0, ctx->mu_ind, ctx->mu);
            ctx->prof.end(1);
        } else {
            CK(cudaMemcpyAsync(ctx->mu, ctx->dip0, sizeof(double) * n3, cudaMemcpyDeviceToDevice, ctx->st));
        }
        bool dip = ctx->any_dip0 || ctx->npol > 0;
        DirFlags f = dir_flags(ctx);
        f.qq = ctx->any_q ? 1 : 0;
        f.qd = (dip && ctx->any_q) ? 1 : 0;
        f.dd = dip ? 1 : 0;
        f.damp = 1;
        f.field = p.doefield ? 1 : 0;
        f.efg = efg ? 1 : 0;
        f.forces = 1;
        CK(cudaMemsetAsync(ctx->ef, 0, sizeof(double) * n3, ctx->st));
        if (efg) CK(cudaMemsetAsync(ctx->efg, 0, sizeof(double) * 6 * n, ctx->st));
        ctx->prof.begin(PK_DIR);
        launch_ewald_dir(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->type, ctx->q, ctx->mu, ctx->cell, coul_list(ctx),
                         ctx->pc, f, ctx->ef, ctx->efg, ctx->fcoul, ctx->part, ctx->dsc, ctx->g_dir);
        ctx->prof.end(2);
        RecFlags rf{ctx->any_q ? 1 : 0, dip ? 1 : 0, p.doefield ? 1 : 0, (efg || dip) ? 1 : 0, 1, 1, p.precision,
                    ctx->rec_acc_ready ? 1 : 0};
        ctx->rec_acc_ready = false;
        launch_ewald_rec(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->q, ctx->mu, ctx->cell, ctx->kg, rf, ctx->rs, ctx->ef,
                         efg ? ctx->efg : nullptr, ctx->fcoul, ctx->part, ctx->dsc, &ctx->prof);
        int vb = std::min(592, nb(n));
        ctx->prof.begin(PK_OTHER);
        k_coul_sums<<<vb, 256, 0, ctx->st>>>(n, ctx->q, ctx->mu, ctx->x, ctx->y, ctx->z, ctx->part.buf);
        launch_reduce_partials(ctx->st, ctx->part.buf, vb, 8, ctx->dsc->sums, 0);
        const double tpi_V = 2.0 * PI / ctx->cell.omega;
        k_coul_finish<<<nb(n), 256, 0, ctx->st>>>(n, ctx->q, ctx->mu, ctx->ef, ctx->efg, ctx->fcoul, ctx->fx, ctx->fy,
                                                  ctx->fz, selfa2(ctx), ctx->u.coul, efg ? 1 : 0, p.lsurf, ctx->dsc,
                                                  2.0 * tpi_V / 3.0);
        ctx->prof.end(3);
        TRY(check_launch(ctx, "coulomb"));
    }
    if (ctx->capturing) return MDFF_OK;
    TRY(sync_scalars(ctx));
    return engforce_finish(ctx);
}

// The host side of an evaluation once its device scalars are in ctx->hsc:
// energies, virials and stresses (multipole_ES's and the pair loops' sums,
// src/field.f90:1930-2050).
int engforce_finish(mdff_ctx* ctx) {
    const mdff_params& p = ctx->p;
    const DevScalars& h = *ctx->hsc;
    {   // the solve's count and residual were set by solve_dipoles / solve_finish
        const int it = ctx->en.scf_iter;
        const double rm = ctx->en.scf_rmsd;
        std::memset(&ctx->en, 0, sizeof ctx->en);
        ctx->en.scf_iter = it;
        ctx->en.scf_rmsd = rm;
    }
    if (p.lcoulomb) {
        double cu = ctx->u.coul;
        double tpi_V = 2.0 * PI / ctx->cell.omega;
        double u_dir = h.dir[0], u_rec = h.rec[0] * 2.0 * tpi_V;
        double u_self = -selfa(ctx) * h.sums[0] - selfa2(ctx) * h.sums[1];
        double u_pol = 0.5 * h.upol[0];
        double qt[3] = {h.sums[2], h.sums[3], h.sums[4]}, mt[3] = {h.sums[5], h.sums[6], h.sums[7]};
        double u_surf = (qt[0] * qt[0] + qt[1] * qt[1] + qt[2] * qt[2]) + 2.0 * (qt[0] * mt[0] + qt[1] * mt[1] + qt[2] * mt[2]) +
                        (mt[0] * mt[0] + mt[1] * mt[1] + mt[2] * mt[2]);
        u_surf *= tpi_V / 3.0;
        double u = u_dir + u_rec + u_self + u_pol + (p.lsurf ? u_surf : 0.0);
        ctx->en.u_dir = u_dir * cu;
        ctx->en.u_rec = u_rec * cu;
        ctx->en.u_self = u_self * cu;
        ctx->en.u_surf = p.lsurf ? u_surf * cu : 0.0;
        ctx->en.u_pol = u_pol * cu;
        ctx->en.u_coul = u * cu;
        static const int map[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
        double sd = 0.25 / ctx->cell.omega, sr = 2.0 * tpi_V / ctx->cell.omega;
        std::memset(ctx->tau_coul, 0, sizeof ctx->tau_coul);
        for (int k = 0; k < 6; ++k) {
            double v = (h.dir[1 + k] * sd + h.rec[1 + k] * sr) * cu / ctx->u.press;
            int a = map[k][0], b = map[k][1];
            ctx->tau_coul[b * 3 + a] = v;
            ctx->tau_coul[a * 3 + b] = v;
        }
        ctx->en.pvirial_coul = (ctx->tau_coul[0] + ctx->tau_coul[4] + ctx->tau_coul[8]) / 3.0 * ctx->u.press;
    } else {
        std::memset(ctx->tau_coul, 0, sizeof ctx->tau_coul);
    }
    ctx->en.u_lj = h.nonb[0];
    ctx->en.vir_lj = h.nonb[1] / 3.0;
    ctx->en.u_bmhft = h.nonb[2];
    ctx->en.vir_bmhft = h.nonb[3] / 3.0;
    ctx->en.u_morse = h.nonb[4];
    ctx->en.vir_morse = h.nonb[5] / 3.0;
    ctx->en.utail = ctx->utail;
    ctx->en.ptail = ctx->ptail;
    {
        static const int map[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
        std::memset(ctx->tau_nonb, 0, sizeof ctx->tau_nonb);
        for (int k = 0; k < 6; ++k) {
            double v = h.nonb[6 + k] / ctx->cell.omega / ctx->u.press;
            int a = map[k][0], b = map[k][1];
            ctx->tau_nonb[b * 3 + a] = v;
            ctx->tau_nonb[a * 3 + b] = v;
        }
    }
    double usum = ctx->en.u_lj + ctx->en.u_bmhft + ctx->en.u_morse + ctx->en.u_coul;
    if (!std::isfinite(usum)) return fail(ctx, MDFF_E_NONFINITE, "non-finite energy");
    ctx->forces_valid = true;
    return MDFF_OK;
}

int set_units(mdff_ctx* ctx) {
    if (ctx->p.lreduced) ctx->u = {1.0, 1.0, 1.0, 1.0};
    else ctx->u = {0.00624150964712042, 8.61734229648141e-05, 98.2269514139276, 14.3996441494161};
    return MDFF_OK;
}

int upload(mdff_ctx* ctx, double* dst, const double* src, int n) {
    CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
    return MDFF_OK;
}
int download(mdff_ctx* ctx, double* dst, const double* src, int n) {
    CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
    return MDFF_OK;
}

void nhc_const(const mdff_ctx* ctx, NhcConst& c) {
    const mdff_params& p = ctx->p;
    std::memset(&c, 0, sizeof c);
    c.nhc_n = p.nhc_n;
    c.yosh = p.nhc_yosh_order;
    c.mults = p.nhc_mults;
    c.literal = p.nhc_literal ? 1 : 0;
    c.dt = p.dt * ctx->u.time;
    c.temp = p.temp * ctx->u.boltz;
    c.L = 3.0 * (double)ctx->n;
    double ts = p.timesca_thermo * ctx->u.time;
    if (p.integrator == MDFF_NVT_NHC2) {
        // nhc2 (src/integration.f90:224-229): L = 3 (natm - 1), two thermostats
        c.nhc_n = 2;
        c.L = 3.0 * ((double)ctx->n - 1.0);
        c.Q[0] = ts * ts * c.temp * c.L;
        c.Q[1] = ts * ts * c.temp;
        return;
    }
    for (int k = 0; k < p.nhc_n; ++k) c.Q[k] = ts * ts * c.temp;   // timesca_thermo**2 * temp
    c.Q[0] = c.Q[0] * c.L;
    double* w = c.w;
    switch (p.nhc_yosh_order) {
        case 1: w[0] = 1.0; break;
        case 3: w[0] = 1.0 / (2.0 - std::pow(2.0, 1.0 / 3.0)); w[1] = 1.0 - 2.0 * w[0]; w[2] = w[0]; break;
        case 5: w[0] = 1.0 / (4.0 - std::pow(4.0, 1.0 / 3.0)); w[1] = w[0]; w[2] = w[0]; w[3] = w[0]; w[4] = 1.0 - 4.0 * w[0]; break;
        case 7:
            w[0] = .78451361047756; w[1] = .235573213359357; w[2] = -1.17767998417887;
            w[3] = 1.0 - 2.0 * (w[0] + w[1] + w[2]); w[4] = w[2]; w[5] = w[1]; w[6] = w[0]; break;
        default:
            w[0] = 0.192; w[1] = 0.554910818409783619692725006662999; w[2] = 0.124659619941888644216504240951585;
            w[3] = -0.843182063596933505315033808282941; w[4] = 1.0 - 2.0 * (w[0] + w[1] + w[2] + w[3]);
            w[5] = w[3]; w[6] = w[2]; w[7] = w[1]; w[8] = w[0]; break;
    }
}

int ke_reduce(mdff_ctx* ctx, int apply_scale) {
    const int n = ctx->n;
    ctx->prof.begin(PK_INTEGRATE);
    k_scale_ke<<<nb(n), 256, 0, ctx->st>>>(n, ctx->vx, ctx->vy, ctx->vz, ctx->mass, ctx->dsc, apply_scale,
                                           ctx->part.buf);
    launch_reduce_partials(ctx->st, ctx->part.buf, nb(n), 1, ctx->dsc->ke2, 0);
    ctx->prof.end(2);
    return check_launch(ctx, "ke");
}

// calc_thermo (src/thermo.f90:116-207) from the host copies.
void fill_thermo(mdff_ctx* ctx, mdff_thermo* t, int step) {
    const double nr = ctx->p.lreduced ? (double)ctx->n : 1.0;
    double omega = ctx->cell.omega;
    t->step = step;
    t->e_kin = ctx->e_kin / nr;
    t->temp_r = ctx->temp_r;
    t->u_lj = ctx->en.u_lj / nr;
    t->u_bmhft = ctx->en.u_bmhft / nr;
    t->u_morse = ctx->en.u_morse / nr;
    t->u_coul = ctx->en.u_coul / nr;
    t->u_pol = ctx->en.u_pol / nr;
    t->u_tot = t->u_lj + t->u_coul + t->u_morse + t->u_bmhft;
    t->e_tot = t->u_tot + t->e_kin;
    const int ig = ctx->p.integrator;
    t->e_nvt = ((ig == MDFF_NVT_NHCN || ig == MDFF_NVT_NHC2) ? ctx->hsc->e_nvt
                : ig == MDFF_NPT_NHCNP                       ? ctx->npt.e_npt
                                                             : 0.0) / nr;
    t->h_tot = ig == MDFF_NVE_VV ? t->e_tot : t->e_tot + t->e_nvt;
    t->volume = omega;
    double pv = (ctx->en.vir_lj + ctx->en.vir_morse + ctx->en.vir_bmhft) / omega / nr + ctx->en.pvirial_coul / nr;
    t->pvirial_tot = pv / ctx->u.press;
    t->pressure_tot = (pv + ctx->temp_r * ctx->u.boltz / omega) / ctx->u.press;
    t->nlist_rebuilt = ctx->last_rebuilt;
    t->scf_iter = ctx->en.scf_iter;
    t->scf_rmsd = ctx->en.scf_rmsd;
}

void set_kin(mdff_ctx* ctx) {
    ctx->e_kin = 0.5 * ctx->hsc->ke2[0];
    ctx->temp_r = 2.0 * ctx->e_kin / ctx->u.boltz / (3.0 * (double)ctx->n);
}

// A new cell of the same k rectangle (constant pressure, mdff_set_cell):
// lattice, the tail corrections (proportional to 1/V and 1/V^2) and the k
// tables with their set-up membership.
int apply_cell(mdff_ctx* ctx, const double A9[9]) {
    CellP c;
    double W[3], an[3];
    lattice(A9, c, W, an);
    if (!(c.omega > 0.0)) return fail(ctx, MDFF_E_ARG, "cell volume must be positive");
    ctx->cell = c;
    for (int d = 0; d < 3; ++d) { ctx->W[d] = W[d]; ctx->anorm[d] = an[d]; }
    std::memcpy(ctx->A_cur, A9, sizeof ctx->A_cur);
    const double r = ctx->omega0 / c.omega;
    ctx->utail = ctx->utail0 * r;
    ctx->ptail = ctx->ptail0 * r * r;
    if (ctx->p.lcoulomb && ctx->kg.mask) {
        KGrid& kg = ctx->kg;
        const double a2 = ctx->alphaES * ctx->alphaES;
        k_kgrid_refresh<<<nb(kg.nrect), 256, 0, ctx->st>>>(kg.nrect, kg.nzl, kg.kmax[1], kg.kmax[2], c, a2, kg.mask,
                                                           kg.Ak, kg.kcoe, kg.Ak_hi);
        const LowK& lk = ctx->rs.low;
        if (lk.ncol > 0)
            k_lowk_refresh<<<nb(lk.ncol * lk.nzmax), 256, 0, ctx->st>>>(lk.ncol, lk.nzmax, c, a2, lk.col, lk.Ak,
                                                                        lk.kcoe);
        TRY(check_launch(ctx, "k tables"));
    }
    ctx->ddtab_epoch = -1;
    ctx->rec_acc_ready = false;
    ctx->forces_valid = false;
    return MDFF_OK;
}

void npt_const(const mdff_ctx* ctx, NptConst& c) {
    const mdff_params& p = ctx->p;
    NhcConst h;
    nhc_const(ctx, h);
    std::memset(&c, 0, sizeof c);
    c.nhc_n = h.nhc_n;
    c.yosh = h.yosh;
    c.mults = h.mults;
    c.literal = h.literal;
    c.dt = h.dt;
    c.temp = h.temp;
    c.L = h.L;
    std::memcpy(c.w, h.w, sizeof c.w);
    std::memcpy(c.Q, h.Q, sizeof c.Q);   // Q = timesca_thermo^2 temp, Q(1) x L
    const double tb = p.timesca_baro * ctx->u.time;
    for (int k = 0; k < p.nhc_n; ++k) c.Qb[k] = tb * tb * c.temp;   // Qb(1) x 9 (src/integration.f90:995-996)
    c.Qb[0] = c.Qb[0] * 9.0;
    c.W = (c.L + 1.0) * tb * tb * c.temp;
    c.press = p.press * ctx->u.press;
}

// sum m v^2 of the current velocities (scaled by s first when apply), on the host
int npt_ke2(mdff_ctx* ctx, bool apply, double s, double& ke2) {
    if (apply) CK(cudaMemcpyAsync(&ctx->dsc->s_scale, &s, sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    TRY(ke_reduce(ctx, apply ? 1 : 0));
    CK(cudaMemcpyAsync(&ctx->hsc->ke2[0], &ctx->dsc->ke2[0], sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ke2 = ctx->hsc->ke2[0];
    return MDFF_OK;
}

// virial pressure of the last force evaluation (pvirial_tot, eV / A^3)
double npt_pvirial(const mdff_ctx* ctx) {
    return (ctx->en.vir_lj + ctx->en.vir_morse + ctx->en.vir_bmhft) / ctx->cell.omega + ctx->en.pvirial_coul;
}

// nhcnp (src/integration.f90:966-1042) with the corrections listed in npt.cuh
int npt_step(mdff_ctx* ctx) {
    const int n = ctx->n;
    NptConst c;
    npt_const(ctx, c);
    NptState& st = ctx->npt;
    const double dt = c.dt, dt2 = dt * 0.5, dt4 = dt2 * 0.5;
    const double odnf = 1.0 + 3.0 / c.L;
    double ke2, s, sb;
    auto kick_ve = [&](double ke2_) {   // D15, D17
        const double omega = ctx->cell.omega;
        const double P_kin = odnf * ke2_ / (3.0 * omega);
        const double Ge = 3.0 * omega * (P_kin + npt_pvirial(ctx) - c.press);
        st.ve = st.ve + Ge * dt2;
    };
    // first half: barostat and particle chains, velocities scaled, barostat kick
    TRY(npt_ke2(ctx, false, 1.0, ke2));
    npt_chain_half(c, st, 0.5 * ke2, true, s, sb);
    TRY(npt_ke2(ctx, true, s, ke2));
    st.ve = st.ve * sb;
    kick_ve(ke2);
    // prop_pos_vel_verlet_npt (src/integration.f90:1049-1160)
    double arg = odnf * st.ve * dt4 / c.W;
    double aa = std::exp(-arg);
    double AA2 = aa * aa, BB = aa * dt2 * npt_poly(arg);
    ctx->prof.begin(PK_INTEGRATE);
    k_npt_kick<<<nb(n), 256, 0, ctx->st>>>(n, ctx->vx, ctx->vy, ctx->vz, ctx->fx, ctx->fy, ctx->fz, ctx->mass, AA2, BB,
                                           ctx->part.buf);
    ctx->prof.end(1);
    st.xe = st.xe + st.ve * dt / c.W;
    const double g = std::exp(st.xe - st.xe0);
    double A[9];
    for (int k = 0; k < 9; ++k) A[k] = ctx->A_cur[k] * g;
    st.xe0 = st.xe;
    st.scale *= g;
    TRY(apply_cell(ctx, A));
    arg = st.ve * dt2 / c.W;
    aa = std::exp(arg);
    AA2 = aa * aa;
    BB = aa * npt_poly(arg) * dt;
    ctx->prof.begin(PK_INTEGRATE);
    k_npt_drift<<<nb(n), 256, 0, ctx->st>>>(n, ctx->x, ctx->y, ctx->z, ctx->vx, ctx->vy, ctx->vz, AA2, BB);
    ctx->prof.end(1);
    TRY(check_launch(ctx, "npt drift"));
    TRY(engforce_device(ctx));
    arg = odnf * st.ve * dt4 / c.W;
    aa = std::exp(-arg);
    AA2 = aa * aa;
    BB = aa * npt_poly(arg) * dt2;
    ctx->prof.begin(PK_INTEGRATE);
    k_npt_kick<<<nb(n), 256, 0, ctx->st>>>(n, ctx->vx, ctx->vy, ctx->vz, ctx->fx, ctx->fy, ctx->fz, ctx->mass, AA2, BB,
                                           ctx->part.buf);
    launch_reduce_partials(ctx->st, ctx->part.buf, nb(n), 1, ctx->dsc->ke2, 0);
    ctx->prof.end(2);
    TRY(check_launch(ctx, "npt kick"));
    CK(cudaMemcpyAsync(&ctx->hsc->ke2[0], &ctx->dsc->ke2[0], sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ke2 = ctx->hsc->ke2[0];
    // second half: barostat kick, particle and barostat chains
    kick_ve(ke2);
    npt_chain_half(c, st, 0.5 * ke2, false, s, sb);
    TRY(npt_ke2(ctx, true, s, ke2));
    st.ve = st.ve * sb;
    st.e_npt = npt_energy(c, st, ctx->cell.omega);
    return MDFF_OK;
}

// Skin allowance of the Verlet-list check: a shrinking cell brings pairs
// beyond the list radius closer by the same factor, and that margin comes off
// the displacement allowance.
double skin_allowance(const mdff_ctx* ctx) {
    const double shrink = std::max(0.0, 1.0 - ctx->npt.scale / ctx->npt.scale_build);
    return ctx->p.skindiff - shrink * rlist_max(ctx, ctx->p.skindiff);
}

// The launches of one MD step (body of md_run's loop, src/runmd.f90:266-277)
// up to the Verlet-list check; the host syncs inside (the force evaluation's)
// are skipped while the step is being captured.
int md_launches(mdff_ctx* ctx) {
    const int n = ctx->n;
    const mdff_params& p = ctx->p;
    const double dt = p.dt * ctx->u.time;
    if (p.integrator == MDFF_NPT_NHCNP) {
        TRY(npt_step(ctx));
    } else if (p.integrator == MDFF_NVE_VV) {
        ctx->prof.begin(PK_INTEGRATE);
        k_vv_positions<<<nb(n), 256, 0, ctx->st>>>(n, ctx->x, ctx->y, ctx->z, ctx->vx, ctx->vy, ctx->vz, ctx->fx, ctx->fy,
                                                   ctx->fz, ctx->fox, ctx->foy, ctx->foz, ctx->mass, dt);
        ctx->prof.end(1);
        TRY(check_launch(ctx, "vv_positions"));
        TRY(engforce_device(ctx));
        ctx->prof.begin(PK_INTEGRATE);
        k_vv_velocities<<<nb(n), 256, 0, ctx->st>>>(n, ctx->vx, ctx->vy, ctx->vz, ctx->fx, ctx->fy, ctx->fz, ctx->fox,
                                                    ctx->foy, ctx->foz, ctx->mass, dt, ctx->part.buf);
        launch_reduce_partials(ctx->st, ctx->part.buf, nb(n), 1, ctx->dsc->ke2, 0);
        ctx->prof.end(2);
    } else {
        // nhcn (src/integration.f90:476-558) or nhc2 (:205-254): chain half,
        // prop_pos_vel_verlet, chain half; only the chain kernel differs
        NhcConst c;
        nhc_const(ctx, c);
        const bool two = p.integrator == MDFF_NVT_NHC2;
        auto chain = [&]() {
            if (two) k_nhc2_chain<<<1, 1, 0, ctx->st>>>(ctx->dsc, c, ctx->dsc->ke2);
            else k_nhc_chain<<<1, 1, 0, ctx->st>>>(ctx->dsc, c, ctx->dsc->ke2);
        };
        TRY(ke_reduce(ctx, 0));
        ctx->prof.begin(PK_INTEGRATE);
        chain();
        ctx->prof.end(1);
        TRY(ke_reduce(ctx, 1));
        ctx->prof.begin(PK_INTEGRATE);
        k_kick_drift<<<nb(n), 256, 0, ctx->st>>>(n, ctx->x, ctx->y, ctx->z, ctx->vx, ctx->vy, ctx->vz, ctx->fx, ctx->fy,
                                                 ctx->fz, ctx->mass, dt);
        ctx->prof.end(1);
        TRY(check_launch(ctx, "kick_drift"));
        TRY(engforce_device(ctx));
        ctx->prof.begin(PK_INTEGRATE);
        k_kick<<<nb(n), 256, 0, ctx->st>>>(n, ctx->vx, ctx->vy, ctx->vz, ctx->fx, ctx->fy, ctx->fz, ctx->mass, dt,
                                           ctx->part.buf);
        launch_reduce_partials(ctx->st, ctx->part.buf, nb(n), 1, ctx->dsc->ke2, 0);
        chain();
        ctx->prof.end(3);
        TRY(ke_reduce(ctx, 1));
        ctx->prof.begin(PK_INTEGRATE);
        if (two) k_nhc2_energy<<<1, 1, 0, ctx->st>>>(ctx->dsc, c);
        else k_nhc_energy<<<1, 1, 0, ctx->st>>>(ctx->dsc, c);
        ctx->prof.end(1);
    }
    TRY(check_launch(ctx, "step"));
    if (p.lvnlist) {
        // positions unchanged since the force call: sx is current
        ctx->prof.begin(PK_NLIST);
        launch_skin_check(ctx->st, n, ctx->sx, ctx->sy, ctx->sz, ctx->xs, ctx->ys, ctx->zs, ctx->cell,
                          skin_allowance(ctx), ctx->part, ctx->dsc);
        ctx->prof.end(2);
        TRY(check_launch(ctx, "skin"));
    }
    return MDFF_OK;
}

// After the step's scalars are on the host: temperature and the list rebuild
// that vnlistcheck asks for.
int step_end(mdff_ctx* ctx) {
    set_kin(ctx);
    ctx->last_rebuilt = 0;
    if (ctx->p.lvnlist && ctx->hsc->rebuild) {
        TRY(build_lists(ctx, ctx->p.skindiff));
        ctx->last_rebuilt = 1;
    }
    return MDFF_OK;
}

int md_step_plain(mdff_ctx* ctx) {
    ctx->nstep_plain++;
    TRY(md_launches(ctx));
    TRY(sync_scalars(ctx));
    return step_end(ctx);
}

// ---- the MD step as a CUDA graph --------------------------------------------
// A step whose launches do not depend on host decisions made during it is
// captured once (one graph for the EFG steps, one for the others) and
// replayed; the dipole PCG runs as a conditional WHILE node with its test on
// the device, and the host syncs once per step, after it.  Steps that need
// the host in between (constant pressure, the SCF solver, profiling, the
// predictor's start-up steps, a context whose lists or pair table are about
// to be reallocated) run as plain launches.

bool graph_eligible(const mdff_ctx* ctx) {
    const mdff_params& p = ctx->p;
    if (ctx->graph_off || ctx->prof.on) return false;
    if (p.integrator == MDFF_NPT_NHCNP) return false;
    if (!p.lvnlist || !ctx->have_list || !ctx->forces_valid) return false;
    if (p.autotune && !ctx->tuned) return false;
    if (p.lcoulomb && ctx->npol > 0 && p.algo_moment_from_pola != MDFF_POLA_PCG) return false;
    if (p.lcoulomb && p.precision == MDFF_PREC_MIXED &&
        (!ctx->ddcnt || !ctx->ddrec || (size_t)ctx->n * coul_list(ctx).cap > ctx->ddtab_cap))
        return false;
    return true;
}

StepKey step_key(const mdff_ctx* ctx) {
    StepKey k;
    std::memset(&k, 0, sizeof k);
    k.ptr[0] = ctx->lv.nbr; k.ptr[1] = ctx->lv.cnt;
    k.ptr[2] = ctx->lc.nbr; k.ptr[3] = ctx->lc.cnt;
    k.ptr[4] = ctx->ddtab;  k.ptr[5] = ctx->ddnbr;
    k.cap[0] = ctx->lv.cap; k.cap[1] = ctx->lc.cap; k.cap[2] = (int)std::min<size_t>(ctx->ddtab_cap, 0x7fffffff);
    k.cell = ctx->cell;
    k.g_dir = ctx->g_dir; k.g_dd = ctx->g_dd; k.p_mul = ctx->rs.p_mul; k.s_mul = ctx->rs.s_mul;
    k.efg = (ctx->p.doefg && ctx->efg_due) ? 1 : 0;
    // the predictor's plan is device data (upload_plan), not part of the key
    k.skin = skin_allowance(ctx);
    k.n = ctx->n;
    return k;
}

void drop_graph(mdff_ctx* ctx, int slot) {
    if (ctx->gexec[slot]) cudaGraphExecDestroy(ctx->gexec[slot]);
    if (ctx->graph[slot]) cudaGraphDestroy(ctx->graph[slot]);
    ctx->gexec[slot] = nullptr;
    ctx->graph[slot] = nullptr;
}

void drop_graphs(mdff_ctx* ctx) {
    drop_graph(ctx, 0);
    drop_graph(ctx, 1);
}

int capture_step(mdff_ctx* ctx, int slot, const StepKey& key) {
    drop_graph(ctx, slot);
    CK(cudaStreamSynchronize(ctx->st));
    const long l0 = ctx->prof.launches;
    ctx->capturing = true;
    ctx->pcg_in_graph = false;
    ctx->cap_body = 0;
    int rc = MDFF_OK;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        rc = fail(ctx, MDFF_E_CUDA, std::string("capture of the MD step: ") + cudaGetErrorString(e));
    } else {
        rc = md_launches(ctx);
        cudaError_t e2 = cudaStreamEndCapture(ctx->st, &g);
        if (rc == MDFF_OK && e2 != cudaSuccess)
            rc = fail(ctx, MDFF_E_CUDA, std::string("capture of the MD step: ") + cudaGetErrorString(e2));
    }
    ctx->capturing = false;
    const long captured = ctx->prof.launches - l0;
    ctx->prof.launches = l0;
    if (rc != MDFF_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    cudaGraphExec_t ge = nullptr;
    e = cudaGraphInstantiate(&ge, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(ctx, MDFF_E_CUDA, std::string("instantiation of the MD step graph: ") + cudaGetErrorString(e));
    }
    ctx->graph[slot] = g;
    ctx->gexec[slot] = ge;
    ctx->gkey[slot] = key;
    ctx->glaunch[slot] = captured;
    ctx->gbody[slot] = ctx->pcg_in_graph ? ctx->cap_body : 0;
    ctx->ncapture++;
    return MDFF_OK;
}

int md_step_graph(mdff_ctx* ctx) {
    if (ctx->p.lcoulomb && ctx->npol > 0) TRY(upload_plan(ctx));
    const StepKey key = step_key(ctx);
    const int slot = key.efg;
    if (!ctx->gexec[slot] || std::memcmp(&key, &ctx->gkey[slot], sizeof key) != 0) {
        if (capture_step(ctx, slot, key) != MDFF_OK) {
            // a capture that fails leaves nothing launched: run the step as
            // plain launches, and from now on
            cudaGetLastError();
            ctx->graph_off = true;
            return md_step_plain(ctx);
        }
    }
    CK(cudaGraphLaunch(ctx->gexec[slot], ctx->st));
    ctx->nstep_graph++;
    TRY(sync_scalars(ctx));
    const bool pcg = ctx->gbody[slot] > 0;
    ctx->prof.launches += ctx->glaunch[slot] + (pcg ? ctx->gbody[slot] * (long)ctx->hsc->iter : 0);
    if (pcg) {
        TRY(solve_finish(ctx));
    } else {
        ctx->en.scf_iter = 0;
        ctx->en.scf_rmsd = 0.0;
    }
    TRY(engforce_finish(ctx));
    return step_end(ctx);
}

// One MD step (body of md_run's loop, src/runmd.f90:266-277); the EFG is due
// every efg_period steps.
int md_step(mdff_ctx* ctx) {
    const mdff_params& p = ctx->p;
    ctx->itime++;
    ctx->efg_due = p.efg_period <= 1 || ctx->itime % p.efg_period == 0;
    const int rc = graph_eligible(ctx) ? md_step_graph(ctx) : md_step_plain(ctx);
    ctx->efg_due = true;
    return rc;
}

}  // namespace

// ---- structure optimisation ------------------------------------------------
// sastry (src/opt.f90:452-849): conjugate gradients on U(r) = u_tot with the
// direction normalised to unit length and each line minimised by cubic
// interpolation along it; eforce1d (:864-933) is one engforce at r + x xi.
// The scalar control flow is the reference's, statement for statement
// (labels 777, 524, 525, 676 become loops); the vectors and their dot
// products stay on the device.  As in the reference, the Verlet lists are
// the ones of the starting configuration (engforce does not rebuild them),
// trial evaluations leave their forces behind, and u_tot changes only where
// the reference assigns it.
namespace {

double opt_utot(const mdff_ctx* ctx) { return ctx->en.u_lj + ctx->en.u_coul + ctx->en.u_morse + ctx->en.u_bmhft; }

int opt_sum(mdff_ctx* ctx, int K, double out[2]) {
    launch_reduce_partials(ctx->st, ctx->part.buf, nb(ctx->n), K, ctx->dsc->opt, 0);
    TRY(sync_scalars(ctx));
    out[0] = ctx->hsc->opt[0];
    out[1] = K > 1 ? ctx->hsc->opt[1] : 0.0;
    return MDFF_OK;
}

int opt_dot(mdff_ctx* ctx, int mode, double out[2]) {
    const int n = ctx->n;
    if (mode == 0) k_opt_dots<0><<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->opt_xi, ctx->opt_g, ctx->part.buf);
    else if (mode == 1) k_opt_dots<1><<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->opt_xi, ctx->opt_g, ctx->part.buf);
    else k_opt_dots<2><<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->opt_xi, ctx->opt_g, ctx->part.buf);
    return opt_sum(ctx, 2, out);
}

// the unit steepest-descent direction from the current forces
int opt_steepest(mdff_ctx* ctx) {
    const int n = ctx->n;
    double s[2];
    k_opt_steepest<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->opt_xi, ctx->opt_g, ctx->opt_h,
                                               ctx->part.buf);
    TRY(opt_sum(ctx, 1, s));
    const double umag = std::sqrt(s[0]);
    k_opt_div<<<nb(3 * n), 256, 0, ctx->st>>>(3 * n, ctx->opt_xi, umag);
    return check_launch(ctx, "opt_steepest");
}

// r = r0 + x xi on the device positions
void opt_place(mdff_ctx* ctx, double x) {
    const int n = ctx->n;
    k_opt_move<<<nb(n), 256, 0, ctx->st>>>(n, ctx->opt_r0, ctx->opt_r0 + n, ctx->opt_r0 + 2 * (size_t)n, ctx->opt_xi,
                                           x, ctx->x, ctx->y, ctx->z);
}

// eforce1d: U and dU/dx at r0 + x xi; the positions are r0 again afterwards,
// the forces stay those of the trial point
int opt_eforce1d(mdff_ctx* ctx, double x, double& pot, double& f1d, int& neng) {
    opt_place(ctx, x);
    TRY(engforce_device(ctx));
    pot = opt_utot(ctx);
    neng = neng + 1;
    opt_place(ctx, 0.0);
    double s[2];
    TRY(opt_dot(ctx, 0, s));
    f1d = -s[0];
    return MDFF_OK;
}

// the accepted move r0 += x xi (kept in r0 and in the device positions)
int opt_accept(mdff_ctx* ctx, double x) {
    const int n = ctx->n;
    opt_place(ctx, x);
    CK(cudaMemcpyAsync(ctx->opt_r0, ctx->x, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->opt_r0 + n, ctx->y, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->opt_r0 + 2 * (size_t)n, ctx->z, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    return MDFF_OK;
}

// The reference halves a trial step without bound while U stays above the
// line's starting value ukeep (labels 524, 525).  After OPT_MAX_HALVINGS
// halvings the step is x0 to the last bit, so a U still above ukeep comes from
// the rounding of repeated evaluations at one point (the induced dipoles start
// from the previous solution); the minimisation then ends at x0 with status 3,
// as the 100-step limit ends it.
constexpr int OPT_MAX_HALVINGS = 64;

int opt_stalled(mdff_ctx* ctx, mdff_opt_result* R, double x0, double u0, double phigrad, int neng) {
    TRY(opt_accept(ctx, x0));
    R->u_final = u0;
    R->phigrad = phigrad;
    R->nforce = neng;
    R->status = 3;
    return MDFF_OK;
}

int opt_sastry(mdff_ctx* ctx, int itmax, mdff_opt_result* R) {
    const int n = ctx->n;
    if (!ctx->opt_xi) {
        TRY(dalloc(ctx, &ctx->opt_xi, 3 * (size_t)n));
        TRY(dalloc(ctx, &ctx->opt_g, 3 * (size_t)n));
        TRY(dalloc(ctx, &ctx->opt_h, 3 * (size_t)n));
        TRY(dalloc(ctx, &ctx->opt_r0, 3 * (size_t)n));
    }
    CK(cudaMemcpyAsync(ctx->opt_r0, ctx->x, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->opt_r0 + n, ctx->y, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->opt_r0 + 2 * (size_t)n, ctx->z, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    const double ftol = 2.2250738585072014e-308, epsilon = 1.0e-14;   // tiny(1.0_dp)
    int neng = 0;
    TRY(engforce_device(ctx));
    neng = neng + 1;
    double u_tot = opt_utot(ctx);
    R->u_initial = u_tot;
    R->status = 1;
    TRY(opt_steepest(ctx));
    double ds = 0.2, dutol = 1.0e-12, phigrad = 0.0, Eis = u_tot, xsol = 0.0, t[2];
    for (int its = 1; its <= itmax; ++its) {
        TRY(opt_dot(ctx, 1, t));
        phigrad = t[0];
        R->iterations = its;
        double ukeep = u_tot, x0 = 0.0, u0 = u_tot, f1_dp;
        TRY(opt_dot(ctx, 0, t));
        f1_dp = -t[0];
        if (f1_dp >= 0.0) {   // reset to the steepest-descent direction
            TRY(opt_steepest(ctx));
            ukeep = u_tot; x0 = 0.0; u0 = u_tot;
            TRY(opt_dot(ctx, 0, t));
            f1_dp = -t[0];
        }
        double x1 = ds, u1, f1d1, u2 = 0.0, f1ds = 0.0;
        TRY(opt_eforce1d(ctx, x1, u1, f1d1, neng));
        int nstep = 0;
        double uprev = std::min(u1, u0);
        for (;;) {   // label 777
            nstep = nstep + 1;
            const double dx = x1 - x0, dx2 = dx * dx, dx3 = dx * dx2;
            if (nstep > 100) {
                if (std::min(u0, u1) > ukeep) {
                    Eis = u0;
                    R->u_final = Eis; R->phigrad = phigrad; R->nforce = neng; R->status = 3;
                    return MDFF_OK;
                }
                if (u0 < u1) {
                    TRY(opt_eforce1d(ctx, x0, u0, f1_dp, neng));
                    xsol = x0; u_tot = u0; f1ds = f1_dp;
                } else {
                    xsol = x1; u_tot = u1; f1ds = f1d1;
                }
                TRY(opt_accept(ctx, xsol));
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
                    TRY(opt_eforce1d(ctx, xsol, u2, f1ds, neng));
                    if (u2 > ukeep) {
                        if (nh == OPT_MAX_HALVINGS) return opt_stalled(ctx, R, x0, u0, phigrad, neng);
                        xsol = x0 + (xsol - x0) / 2.0;
                        continue;
                    }
                    break;
                }
                if (std::fabs((uprev - u2) / u2) < dutol) {
                    TRY(opt_accept(ctx, xsol));
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
                    TRY(opt_eforce1d(ctx, xsol, u2, f1ds, neng));
                    if (u2 > ukeep) {
                        if (nh == OPT_MAX_HALVINGS) return opt_stalled(ctx, R, x0, u0, phigrad, neng);
                        xsol = x0 + (xsol - x0) / 2.0;
                        continue;
                    }
                    break;
                }
                if (std::fabs((uprev - u2) / u2) < dutol) {
                    TRY(opt_accept(ctx, xsol));
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
            TRY(engforce_device(ctx));
            neng = neng + 1;
            Eis = u_tot;
            TRY(opt_dot(ctx, 1, t));
            phigrad = t[0];
            R->u_final = Eis; R->phigrad = phigrad; R->nforce = neng; R->status = 0;
            return MDFF_OK;
        } else if (std::fabs(1.0 - u_tot / ukeep) < dutol) {
            dutol = std::fabs(1.0 - u_tot / ukeep);
        }
        TRY(opt_dot(ctx, 2, t));
        const double gg = t[0], dgg = t[1];
        if (gg == 0.0) {
            R->u_final = u_tot; R->phigrad = phigrad; R->nforce = neng; R->status = 2;
            return MDFF_OK;
        }
        const double gam = dgg / gg;
        k_opt_cg<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->opt_xi, ctx->opt_g, ctx->opt_h, gam,
                                             ctx->part.buf);
        TRY(opt_sum(ctx, 1, t));
        k_opt_div<<<nb(3 * n), 256, 0, ctx->st>>>(3 * n, ctx->opt_xi, std::sqrt(t[0]));
        TRY(check_launch(ctx, "opt_cg"));
    }
    R->u_final = u_tot; R->phigrad = phigrad; R->nforce = neng; R->status = 1;
    R->iterations = itmax;
    return MDFF_OK;
}

// ---- L-BFGS ------------------------------------------------------------------
// lbfgs_driver (src/opt.f90:972-1194) with LBFGS (src/lbfgs.f90:243-456):
// Nocedal's limited-memory BFGS, m = 5 pairs, no user diagonal, and the
// More-Thuente line search MCSRCH/MCSTEP (:655-1186) with ftol 1e-4, gtol
// 0.9, maxfev 100, stpmin 1e-20, stpmax 1e20, xtol = tiny(1.0_dp).  The
// reverse communication of the reference becomes direct calls of engforce at
// the trial points; every evaluation is one of the driver's iterations, at
// most itmax of them.  The S and Y pairs, the direction and the two-loop
// recursion stay on the device (the recursion's coefficients in device
// scalars, no host round trip); the line search's scalars come to the host.
constexpr int LB_M = 5;

struct LbState {
    int icall = 0, itmax = 0;
    double F = 0.0, gg = 0.0, phigrad = 0.0;
};

V3 lb_pos(const mdff_ctx* c) { return V3{{c->x, c->y, c->z}, 1.0}; }
V3 lb_grad(const mdff_ctx* c) { return V3{{c->fx, c->fy, c->fz}, -1.0}; }
V3 lb_buf(const double* b, int n) { return V3{{b, b + n, b + 2 * (size_t)n}, 1.0}; }

int lb_dots(mdff_ctx* ctx, V3 a0, V3 b0, V3 a1, V3 b1, int K, double out[2]) {
    const int n = ctx->n;
    if (K == 1) k_lb_dots<1><<<nb(n), 256, 0, ctx->st>>>(n, a0, b0, a1, b1, ctx->part.buf);
    else k_lb_dots<2><<<nb(n), 256, 0, ctx->st>>>(n, a0, b0, a1, b1, ctx->part.buf);
    return opt_sum(ctx, K, out);
}

// one function evaluation of the driver loop at the current device positions:
// F = u_tot, G = -f, and |G|^2 (the driver's phigrad is that of the previous
// evaluation when LBFGS returns).  Returns 1 when itmax evaluations are done.
int lb_eval(mdff_ctx* ctx, LbState& L, int& stop) {
    stop = 0;
    if (L.icall >= L.itmax) { stop = 1; return MDFF_OK; }
    TRY(engforce_device(ctx));
    L.icall = L.icall + 1;
    L.phigrad = L.gg;
    L.F = opt_utot(ctx);
    double t[2];
    TRY(lb_dots(ctx, lb_grad(ctx), lb_grad(ctx), lb_grad(ctx), lb_grad(ctx), 1, t));
    L.gg = t[0];
    return MDFF_OK;
}

// MCSTEP (src/lbfgs.f90:960-1186): one safeguarded cubic or quadratic step of
// the More-Thuente interval update.  The 0.66 of the final safeguard is a
// default-real (single-precision) constant in the reference.
void lb_mcstep(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy, double& stp, double fp,
               double dp, bool& brackt, double stpmin, double stpmax, int& info) {
    info = 0;
    if ((brackt && (stp <= std::min(stx, sty) || stp >= std::max(stx, sty))) || dx * (stp - stx) >= 0.0 ||
        stpmax < stpmin)
        return;
    const double sgnd = dp * (dx / std::fabs(dx));
    double stpf, stpc, stpq, theta, s, gamma, p, q, r;
    bool bound;
    if (fp > fx) {
        info = 1;
        bound = true;
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
        s = std::max(std::max(std::fabs(theta), std::fabs(dx)), std::fabs(dp));
        gamma = s * std::sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
        if (stp < stx) gamma = -gamma;
        p = (gamma - dx) + theta;
        q = ((gamma - dx) + gamma) + dp;
        r = p / q;
        stpc = stx + r * (stp - stx);
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2) * (stp - stx);
        if (std::fabs(stpc - stx) < std::fabs(stpq - stx)) stpf = stpc;
        else stpf = stpc + (stpq - stpc) / 2;
        brackt = true;
    } else if (sgnd < 0.0) {
        info = 2;
        bound = false;
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
        s = std::max(std::max(std::fabs(theta), std::fabs(dx)), std::fabs(dp));
        gamma = s * std::sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
        if (stp > stx) gamma = -gamma;
        p = (gamma - dp) + theta;
        q = ((gamma - dp) + gamma) + dx;
        r = p / q;
        stpc = stp + r * (stx - stp);
        stpq = stp + (dp / (dp - dx)) * (stx - stp);
        stpf = std::fabs(stpc - stp) > std::fabs(stpq - stp) ? stpc : stpq;
        brackt = true;
    } else if (std::fabs(dp) < std::fabs(dx)) {
        info = 3;
        bound = true;
        theta = 3 * (fx - fp) / (stp - stx) + dx + dp;
        s = std::max(std::max(std::fabs(theta), std::fabs(dx)), std::fabs(dp));
        gamma = s * std::sqrt(std::max(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
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
    } else {
        info = 4;
        bound = false;
        if (brackt) {
            theta = 3 * (fp - fy) / (sty - stp) + dy + dp;
            s = std::max(std::max(std::fabs(theta), std::fabs(dy)), std::fabs(dp));
            gamma = s * std::sqrt((theta / s) * (theta / s) - (dy / s) * (dp / s));
            if (stp > sty) gamma = -gamma;
            p = (gamma - dp) + theta;
            q = ((gamma - dp) + gamma) + dy;
            r = p / q;
            stpc = stp + r * (sty - stp);
            stpf = stpc;
        } else if (stp > stx) {
            stpf = stpmax;
        } else {
            stpf = stpmin;
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
    if (brackt && bound) {
        const double p66 = (double)0.66f;
        if (sty > stx) stp = std::min(stx + p66 * (sty - stx), stp);
        else stp = std::max(stx + p66 * (sty - stx), stp);
    }
}

// MCSRCH (src/lbfgs.f90:655-957) along s from the current point: info as
// there (1 success; 0 bad input or not a descent direction; 2-6 the
// tolerance, step-bound and evaluation-limit exits), stop = 1 when the
// driver's evaluation budget ran out inside the search.
int lb_mcsrch(mdff_ctx* ctx, LbState& L, const double* sdir, double& stp, double ftol, double xtol, int maxfev,
              int& info, int& nfev, int& stop) {
    const int n = ctx->n;
    const double gtol = 0.9, stpmin = 1.0e-20, stpmax = 1.0e20, p5 = 0.5, p66 = 0.66, xtrapf = 4.0;
    int infoc = 1;
    info = 0;
    stop = 0;
    if (n <= 0 || stp <= 0.0 || ftol < 0.0 || gtol < 0.0 || xtol < 0.0 || stpmin < 0.0 || stpmax < stpmin ||
        maxfev <= 0)
        return MDFF_OK;
    double t[2];
    const V3 S = lb_buf(sdir, n);
    TRY(lb_dots(ctx, lb_grad(ctx), S, S, S, 1, t));
    const double dginit = t[0];
    if (dginit >= 0.0) return MDFF_OK;
    bool brackt = false, stage1 = true;
    nfev = 0;
    const double finit = L.F, dgtest = ftol * dginit;
    double width = stpmax - stpmin, width1 = width / p5;
    CK(cudaMemcpyAsync(ctx->lb_wa, ctx->x, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->lb_wa + n, ctx->y, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->lb_wa + 2 * (size_t)n, ctx->z, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    double stx = 0.0, fx = finit, dgx = dginit, sty = 0.0, fy = finit, dgy = dginit, stmin, stmax;
    for (;;) {
        if (brackt) {
            stmin = std::min(stx, sty);
            stmax = std::max(stx, sty);
        } else {
            stmin = stx;
            stmax = stp + xtrapf * (stp - stx);
        }
        stp = std::max(stp, stpmin);
        stp = std::min(stp, stpmax);
        if ((brackt && (stp <= stmin || stp >= stmax)) || nfev >= maxfev - 1 || infoc == 0 ||
            (brackt && stmax - stmin <= xtol * stmax))
            stp = stx;
        k_lb_place<<<nb(n), 256, 0, ctx->st>>>(n, ctx->lb_wa, sdir, stp, ctx->x, ctx->y, ctx->z);
        TRY(lb_eval(ctx, L, stop));
        if (stop) return MDFF_OK;
        info = 0;
        nfev = nfev + 1;
        TRY(lb_dots(ctx, lb_grad(ctx), S, S, S, 1, t));
        const double dg = t[0], f = L.F;
        const double ftest1 = finit + stp * dgtest;
        if ((brackt && (stp <= stmin || stp >= stmax)) || infoc == 0) info = 6;
        if (stp == stpmax && f <= ftest1 && dg <= dgtest) info = 5;
        if (stp == stpmin && (f > ftest1 || dg >= dgtest)) info = 4;
        if (nfev >= maxfev) info = 3;
        if (brackt && stmax - stmin <= xtol * stmax) info = 2;
        if (f <= ftest1 && std::fabs(dg) <= gtol * (-dginit)) info = 1;
        if (info != 0) return MDFF_OK;
        if (stage1 && f <= ftest1 && dg >= std::min(ftol, gtol) * dginit) stage1 = false;
        if (stage1 && f <= fx && f > ftest1) {
            double fm = f - stp * dgtest, fxm = fx - stx * dgtest, fym = fy - sty * dgtest;
            double dgm = dg - dgtest, dgxm = dgx - dgtest, dgym = dgy - dgtest;
            lb_mcstep(stx, fxm, dgxm, sty, fym, dgym, stp, fm, dgm, brackt, stmin, stmax, infoc);
            fx = fxm + stx * dgtest;
            fy = fym + sty * dgtest;
            dgx = dgxm + dgtest;
            dgy = dgym + dgtest;
        } else {
            lb_mcstep(stx, fx, dgx, sty, fy, dgy, stp, f, dg, brackt, stmin, stmax, infoc);
        }
        if (brackt) {
            if (std::fabs(sty - stx) >= p66 * width1) stp = stx + p5 * (sty - stx);
            width1 = width;
            width = std::fabs(sty - stx);
        }
    }
}

int opt_lbfgs(mdff_ctx* ctx, int itmax, double eps, mdff_opt_result* R) {
    const int n = ctx->n, M = LB_M;
    const size_t n3 = 3 * (size_t)n;
    if (!ctx->lb_s) {
        TRY(dalloc(ctx, &ctx->lb_s, M * n3));
        TRY(dalloc(ctx, &ctx->lb_y, M * n3));
        TRY(dalloc(ctx, &ctx->lb_w, n3));
        TRY(dalloc(ctx, &ctx->lb_wa, n3));
        TRY(dalloc(ctx, &ctx->lb_g0, n3));
        TRY(dalloc(ctx, &ctx->lb_sc, 1 + M));
    }
    LbState L;
    L.itmax = itmax;
    int stop = 0;
    *R = mdff_opt_result{};
    R->status = 1;
    TRY(lb_eval(ctx, L, stop));
    R->u_initial = L.F;
    const double ftol = 1.0e-4, xtol = 2.2250738585072014e-308;   // tiny(1.0_dp)
    const int maxfev = 100;
    double rho[LB_M] = {0}, t[2];
    int iter = 0, point = 0;
    size_t npt = 0;
    const int nb3 = (int)((n3 + 255) / 256);
    // the first direction -G DIAG, DIAG = 1, and STP1 = 1 / |G|
    k_lb_negg<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, 1.0, ctx->lb_s);
    const double stp1 = 1.0 / std::sqrt(L.gg);
    auto finish = [&](int status, int info) {
        // the driver's phigrad: |G|^2 of the evaluation before the last one
        // when LBFGS ends, of the last one when the evaluations run out
        R->u_final = L.F;
        R->phigrad = status == 1 ? L.gg : L.phigrad;
        R->iterations = iter;
        R->nforce = L.icall;
        R->status = status;
        R->info = info;
        return MDFF_OK;
    };
    for (;;) {
        iter = iter + 1;
        int bound = iter - 1;
        if (iter != 1) {
            if (iter > M) bound = M;
            const double* yp = ctx->lb_y + npt;
            const double* sp = ctx->lb_s + npt;
            TRY(lb_dots(ctx, lb_buf(yp, n), lb_buf(sp, n), lb_buf(yp, n), lb_buf(yp, n), 2, t));
            const double ys = t[0], yy = t[1], diag = ys / yy;
            rho[point == 0 ? M - 1 : point - 1] = 1.0 / ys;
            k_lb_negg<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, 1.0, ctx->lb_w);
            int cp = point;
            for (int i = 0; i < bound; ++i) {
                cp = cp - 1;
                if (cp == -1) cp = M - 1;
                k_lb_dots<1><<<nb(n), 256, 0, ctx->st>>>(n, lb_buf(ctx->lb_s + cp * n3, n), lb_buf(ctx->lb_w, n),
                                                          lb_buf(ctx->lb_w, n), lb_buf(ctx->lb_w, n), ctx->part.buf);
                launch_reduce_partials(ctx->st, ctx->part.buf, nb(n), 1, ctx->lb_sc, 0);
                k_lb_twoloop<true><<<nb3, 256, 0, ctx->st>>>((int)n3, ctx->lb_w, ctx->lb_y + cp * n3, ctx->lb_sc,
                                                             rho[cp], cp);
            }
            k_lb_scale<<<nb3, 256, 0, ctx->st>>>((int)n3, ctx->lb_w, diag);
            for (int i = 0; i < bound; ++i) {
                k_lb_dots<1><<<nb(n), 256, 0, ctx->st>>>(n, lb_buf(ctx->lb_y + cp * n3, n), lb_buf(ctx->lb_w, n),
                                                          lb_buf(ctx->lb_w, n), lb_buf(ctx->lb_w, n), ctx->part.buf);
                launch_reduce_partials(ctx->st, ctx->part.buf, nb(n), 1, ctx->lb_sc, 0);
                k_lb_twoloop<false><<<nb3, 256, 0, ctx->st>>>((int)n3, ctx->lb_w, ctx->lb_s + cp * n3, ctx->lb_sc,
                                                              rho[cp], cp);
                cp = cp + 1;
                if (cp == M) cp = 0;
            }
            CK(cudaMemcpyAsync(ctx->lb_s + point * n3, ctx->lb_w, sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                               ctx->st));
            TRY(check_launch(ctx, "lbfgs two-loop recursion"));
        }
        // label 165: line search from STP = 1 (STP1 on the first iteration)
        int nfev = 0, info = 0;
        double stp = iter == 1 ? stp1 : 1.0;
        k_lb_keepg<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->lb_g0);
        TRY(lb_mcsrch(ctx, L, ctx->lb_s + point * n3, stp, ftol, xtol, maxfev, info, nfev, stop));
        if (stop) return finish(1, 0);
        if (info != 1) return finish(3, info);
        npt = point * n3;
        k_lb_pair<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->lb_g0, stp, ctx->lb_s + npt,
                                              ctx->lb_y + npt);
        point = point + 1;
        if (point == M) point = 0;
        TRY(lb_dots(ctx, lb_grad(ctx), lb_grad(ctx), lb_pos(ctx), lb_pos(ctx), 2, t));
        const double gnorm = std::sqrt(t[0]), xnorm = std::max(1.0, std::sqrt(t[1]));
        if (gnorm / xnorm <= eps) return finish(0, 0);
    }
}

// ---- M1QN3 -------------------------------------------------------------------
// m1qn3_driver (src/opt.f90:1203-1330) over M1QN3 3.3 (Gilbert & Lemarechal,
// src/m1qn3.f90) as the driver configures it: diagonal initial scaling
// (imode(1) = 0), cold start, ndz = 4n + 5(2n+1) so m = 5 (ybar, sbar)
// pairs in core (mupdts), the euclidean scalar product with identity
// changes of basis (euclid, ctonbe, ctcabe), normtype 'dfn', dxmin =
// tiny(1.0_dp), df1 = 1; the line search mlis3 (:999-1316, Wolfe tests with
// rm1 = 1e-4, rm2 = 0.99, safeguarded cubic ecube :1318-1382).  Direct calls
// of engforce replace the reverse communication; after M1QN3 ends the
// driver evaluates once more at the returned point (its loop body runs once
// with reverse = -1), and so does this.  mlis3's SAVEd indica is not reset
// between calls (its initialisation is commented out in the reference); it
// lives in the context, zero at creation as the static variable is in a
// fresh process.
struct M1Eval {
    int nevals = 0;
    double f = 0.0;
};

int m1_eval(mdff_ctx* ctx, M1Eval& E) {
    TRY(engforce_device(ctx));
    E.nevals = E.nevals + 1;
    E.f = opt_utot(ctx);
    return MDFF_OK;
}

int m1_dot_gd(mdff_ctx* ctx, const double* d, double& out) {
    double t[2];
    TRY(lb_dots(ctx, lb_grad(ctx), lb_buf(d, ctx->n), lb_grad(ctx), lb_grad(ctx), 1, t));
    out = t[0];
    return MDFF_OK;
}

// ecube (src/m1qn3.f90:1318-1382): the minimiser of the cubic through
// (t, f, fp) and (ta, fa, fpa), safeguarded into [tlower, tupper]
void m1_ecube(double& t, double f, double fp, double ta, double fa, double fpa, double tlower, double tupper) {
    const double z1 = fp + fpa - 3.0 * (fa - f) / (ta - t);
    const double b = z1 + fp;
    double discri;
    bool have_root = false;
    if (std::fabs(z1) <= 1.0) {
        discri = z1 * z1 - fp * fpa;
    } else {
        discri = fp / z1;
        discri = discri * fpa;
        discri = z1 - discri;
        if (z1 >= 0.0 && discri >= 0.0) {
            discri = std::sqrt(z1) * std::sqrt(discri);
            have_root = true;
        } else if (z1 <= 0.0 && discri <= 0.0) {
            discri = std::sqrt(-z1) * std::sqrt(-discri);
            have_root = true;
        } else {
            discri = -1.0;
        }
    }
    if (!have_root) {
        if (discri < 0.0) {
            if (fp < 0.0) t = tupper;
            if (fp >= 0.0) t = tlower;
            t = std::max(t, tlower);
            t = std::min(t, tupper);
            return;
        }
        discri = std::sqrt(discri);
    }
    if (t - ta < 0.0) discri = -discri;
    const double sign = (t - ta) / std::fabs(t - ta);
    if (b * sign > 0.0) {
        t = t + fp * (ta - t) / (b + discri);
    } else {
        const double den = z1 + b + fpa, anum = b - discri;
        if (std::fabs((t - ta) * anum) < (tupper - tlower) * std::fabs(den)) t = t + anum * (ta - t) / den;
        else t = tupper;
    }
    t = std::max(t, tlower);
    t = std::min(t, tupper);
}

// mlis3 along d from the current point (f, G on the device), fpn = d.G:
// logic 0 serious step, 1 blocked on tmax, 4 nap > napmax, 6 dxmin or
// rounding; on return the device positions are the last trial point and
// f the value there (the reference's x and f)
int m1_mlis3(mdff_ctx* ctx, M1Eval& E, const double* d, double fpn, double& t, double tmin, double tmax,
             double amd, double amf, int& nap, int napmax, int& logic) {
    const int n = ctx->n;
    if (!(n > 0 && fpn < 0.0 && t > 0.0 && tmax > 0.0 && amf > 0.0 && amd > amf && amd < 1.0)) {
        logic = 6;
        return MDFF_OK;
    }
    const double tesf = amf * fpn, tesd = amd * fpn, barmin = 0.01, barmul = 5.0, barmax = 0.3;
    // fg and the left point xn + tg d matter only to the reference's exits,
    // which return the last trial point in x
    double barr = barmin, td = 0.0, tg = 0.0, fn = E.f, ta = 0.0, fa = fn, fpa = fpn;
    if (t < tmin) {
        t = tmin;
        if (t > tmax) tmin = tmax;
    }
    while (fn + t * fpn >= fn + 0.9 * t * fpn) t = 2.0 * t;
    logic = 0;
    if (t > tmax) {
        t = tmax;
        logic = 1;
    }
    CK(cudaMemcpyAsync(ctx->m1_xn, ctx->x, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->m1_xn + n, ctx->y, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->m1_xn + 2 * (size_t)n, ctx->z, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->st));
    k_lb_place<<<nb(n), 256, 0, ctx->st>>>(n, ctx->m1_xn, d, t, ctx->x, ctx->y, ctx->z);
    for (;;) {   // label 100
        nap = nap + 1;
        if (nap > napmax) {
            logic = 4;
            return MDFF_OK;
        }
        TRY(m1_eval(ctx, E));
        const double f = E.f;
        double fp;
        TRY(m1_dot_gd(ctx, d, fp));
        const double ffn = f - fn;
        int go;   // 320 accept, 350 new left end, 500 interpolate
        if (ffn > t * tesf) {
            td = t;
            logic = 0;
            go = 500;
        } else if (fp > tesd) {
            logic = 0;
            go = 320;
        } else {
            go = logic == 0 ? 350 : 320;
        }
        if (go == 320) return MDFF_OK;
        if (go == 350) {
            tg = t;
            if (td == 0.0) {   // extrapolation
                const double taa = t, gauche = (1.0 + barmin) * t, droite = 10.0 * t;
                m1_ecube(t, f, fp, ta, fa, fpa, gauche, droite);
                ta = taa;
                if (!(t < tmax)) {
                    logic = 1;
                    t = tmax;
                }
                go = 900;
            } else {
                go = 500;
            }
        }
        if (go == 500) {   // interpolation
            if (ctx->m1_indica <= 0) {
                ta = t;
                t = 0.9 * tg + 0.1 * td;
            } else {
                const double test = barr * (td - tg), gauche = tg + test, droite = td - test, taa = t;
                m1_ecube(t, f, fp, ta, fa, fpa, gauche, droite);
                ta = taa;
                if (t > gauche && t < droite) barr = std::max(barmin, barr / barmul);
                else barr = std::min(barmul * barr, barmax);
            }
        }
        fa = f;   // label 900
        fpa = fp;
        ctx->m1_indica = 4;   // label 905: indica = indic, 4 after a simulation
        bool again = td == 0.0;
        if (!again && !(td - tg < tmin)) {
            CK(cudaMemsetAsync(ctx->m1_flag, 0, sizeof(int), ctx->st));
            k_m1_moves<<<nb(n), 256, 0, ctx->st>>>(n, ctx->m1_xn, d, t, ctx->x, ctx->y, ctx->z, ctx->m1_flag);
            int h = 0;
            CK(cudaMemcpyAsync(&h, ctx->m1_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
            CK(cudaStreamSynchronize(ctx->st));
            again = h != 0;
        }
        if (!again) {   // label 920: dxmin reached or rounding
            logic = 6;
            return MDFF_OK;
        }
        k_lb_place<<<nb(n), 256, 0, ctx->st>>>(n, ctx->m1_xn, d, t, ctx->x, ctx->y, ctx->z);   // label 950
    }
}

// dd (src/m1qn3.f90:839-923): w = H w with H the inverse-BFGS matrix of the
// stored pairs jmin..jmax (1-based, cyclic) over the diagonal diag
void m1_dd(mdff_ctx* ctx, int m, int jmin, int jmax, double* w) {
    const int n = ctx->n;
    const size_t n3 = 3 * (size_t)n;
    const int nb3 = (int)((n3 + 255) / 256);
    int jfin = jmax;
    if (jfin < jmin) jfin = jmax + m;
    for (int j = jfin; j >= jmin; --j) {
        const int jp = (j > m ? j - m : j) - 1;
        k_lb_dots<1><<<nb(n), 256, 0, ctx->st>>>(n, lb_buf(w, n), lb_buf(ctx->m1_sbar + jp * n3, n), lb_buf(w, n),
                                                  lb_buf(w, n), ctx->part.buf);
        launch_reduce_partials(ctx->st, ctx->part.buf, nb(n), 1, ctx->m1_sc, 0);
        k_lb_twoloop<true><<<nb3, 256, 0, ctx->st>>>((int)n3, w, ctx->m1_ybar + jp * n3, ctx->m1_sc, 1.0, jp);
    }
    k_m1_mul<<<nb3, 256, 0, ctx->st>>>((int)n3, w, ctx->m1_diag);
    for (int j = jmin; j <= jfin; ++j) {
        const int jp = (j > m ? j - m : j) - 1;
        k_lb_dots<1><<<nb(n), 256, 0, ctx->st>>>(n, lb_buf(w, n), lb_buf(ctx->m1_ybar + jp * n3, n), lb_buf(w, n),
                                                  lb_buf(w, n), ctx->part.buf);
        launch_reduce_partials(ctx->st, ctx->part.buf, nb(n), 1, ctx->m1_sc, 0);
        k_lb_twoloop<false><<<nb3, 256, 0, ctx->st>>>((int)n3, w, ctx->m1_sbar + jp * n3, ctx->m1_sc, 1.0, jp);
    }
}

// m1qn3a (src/m1qn3.f90:371-837) from the evaluated start: omode as there
// (1 converged, 2 zero gradient, 4 niter, 5 nsim, 6 dxmin or rounding in the
// line search, 7 not a descent direction or ys <= 0), it = its iterations
int m1_run(mdff_ctx* ctx, M1Eval& E, int niter, int nsim, double epsg, int& omode, int& it) {
    const int n = ctx->n, m = 5;
    const size_t n3 = 3 * (size_t)n;
    const int nb3 = (int)((n3 + 255) / 256);
    const double dxmin = 2.2250738585072014e-308, df1 = 1.0, rm1 = 1.0e-4, rm2 = 0.99, rmin = 1.0e-20;
    const double tmax = 1.0e20;
    double t[2], ps, hp0;
    int isim = 1;
    it = 0;
    if (epsg >= 1.0) { omode = 1; return MDFF_OK; }
    TRY(lb_dots(ctx, lb_grad(ctx), lb_grad(ctx), lb_grad(ctx), lb_grad(ctx), 1, t));
    const double gnorm = std::sqrt(t[0]), gnorms = gnorm;
    if (gnorms < rmin) { omode = 2; return MDFF_OK; }
    int jmin = 1, jmax = 0;
    const double precos = 2.0 * df1 / (gnorm * gnorm);   // Fletcher's scaling of the first direction
    k_m1_start<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, precos, ctx->m1_d, ctx->m1_diag);
    TRY(m1_dot_gd(ctx, ctx->m1_d, hp0));
    if (hp0 >= 0.0) { omode = 7; return MDFF_OK; }
    unsigned long long* dmax_bits = reinterpret_cast<unsigned long long*>(ctx->m1_flag + 2);
    for (;;) {   // label 100
        it = it + 1;
        k_lb_keepg<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->m1_gg);
        CK(cudaMemsetAsync(dmax_bits, 0, 8, ctx->st));
        k_m1_absmax<<<592, 256, 0, ctx->st>>>((int)n3, ctx->m1_d, dmax_bits);
        unsigned long long bits = 0;
        CK(cudaMemcpyAsync(&bits, dmax_bits, 8, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        double dmax;
        std::memcpy(&dmax, &bits, 8);
        const double tmin = dxmin / dmax;
        double tt = 1.0;
        int moderl = 0;
        TRY(m1_mlis3(ctx, E, ctx->m1_d, hp0, tt, tmin, tmax, rm2, rm1, isim, nsim, moderl));
        bool skip_update = false;
        if (moderl != 0) {
            if (moderl < 0) { omode = moderl; return MDFF_OK; }
            if (moderl == 1) skip_update = true;   // blocked on tmax
            else if (moderl == 4) { omode = 5; return MDFF_OK; }
            else if (moderl == 5) { omode = 0; return MDFF_OK; }
            else if (moderl == 6) { omode = 6; return MDFF_OK; }
        }
        if (!skip_update) {
            jmax = jmax + 1;
            if (jmax > m) jmax = jmax - m;
            if (it > m) {   // cold start
                jmin = jmin + 1;
                if (jmin > m) jmin = jmin - m;
            }
            const size_t jc = (size_t)(jmax - 1) * n3;
            double* sb = ctx->m1_sbar + jc;
            double* yb = ctx->m1_ybar + jc;
            k_m1_pair<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, ctx->m1_gg, ctx->m1_d, tt, sb, yb);
            TRY(lb_dots(ctx, lb_buf(yb, n), lb_buf(sb, n), lb_buf(yb, n), lb_buf(yb, n), 1, t));
            const double ys = t[0];
            if (ys <= 0.0) { omode = 7; return MDFF_OK; }
            double d1 = std::sqrt(1.0 / ys);
            k_lb_scale<<<nb3, 256, 0, ctx->st>>>((int)n3, sb, d1);
            k_lb_scale<<<nb3, 256, 0, ctx->st>>>((int)n3, yb, d1);
            // the diagonal scaled to Rayleigh's ellipsoid, then its BFGS update
            k_m1_diagsum<0><<<nb(n), 256, 0, ctx->st>>>(n, ctx->m1_diag, yb, ctx->part.buf);
            TRY(opt_sum(ctx, 1, t));
            d1 = 1.0 / t[0];
            k_lb_scale<<<nb3, 256, 0, ctx->st>>>((int)n3, ctx->m1_diag, d1);
            k_m1_diagsum<1><<<nb(n), 256, 0, ctx->st>>>(n, ctx->m1_diag, sb, ctx->part.buf);
            TRY(opt_sum(ctx, 1, t));
            k_m1_diagupd<<<nb3, 256, 0, ctx->st>>>((int)n3, ctx->m1_diag, yb, sb, t[0], rmin);
        }
        TRY(lb_dots(ctx, lb_grad(ctx), lb_grad(ctx), lb_grad(ctx), lb_grad(ctx), 1, t));
        ps = t[0];
        const double eps1 = std::sqrt(ps) / gnorms;
        if (eps1 < epsg) { omode = 1; return MDFF_OK; }
        if (it == niter) { omode = 4; return MDFF_OK; }
        if (isim > nsim) { omode = 5; return MDFF_OK; }
        k_lb_negg<<<nb(n), 256, 0, ctx->st>>>(n, ctx->fx, ctx->fy, ctx->fz, 1.0, ctx->m1_d);
        m1_dd(ctx, m, jmin, jmax, ctx->m1_d);
        TRY(check_launch(ctx, "m1qn3 direction"));
        TRY(m1_dot_gd(ctx, ctx->m1_d, hp0));
        if (hp0 >= 0.0) { omode = 7; return MDFF_OK; }
    }
}

int opt_m1qn3(mdff_ctx* ctx, int niter, int nsim, double epsg, mdff_opt_result* R) {
    const int m = 5;
    const size_t n3 = 3 * (size_t)ctx->n;
    if (!ctx->m1_d) {
        TRY(dalloc(ctx, &ctx->m1_d, n3));
        TRY(dalloc(ctx, &ctx->m1_gg, n3));
        TRY(dalloc(ctx, &ctx->m1_diag, n3));
        TRY(dalloc(ctx, &ctx->m1_xn, n3));
        TRY(dalloc(ctx, &ctx->m1_ybar, m * n3));
        TRY(dalloc(ctx, &ctx->m1_sbar, m * n3));
        TRY(dalloc(ctx, &ctx->m1_sc, 1 + m));
        double* fl = nullptr;
        TRY(dalloc(ctx, &fl, 2));
        ctx->m1_flag = reinterpret_cast<int*>(fl);
    }
    M1Eval E;
    TRY(m1_eval(ctx, E));
    R->u_initial = E.f;
    int omode = 0, it = 0;
    TRY(m1_run(ctx, E, niter, nsim, epsg, omode, it));
    // the driver's last pass: one more evaluation at the returned point
    TRY(m1_eval(ctx, E));
    double t[2];
    TRY(lb_dots(ctx, lb_grad(ctx), lb_grad(ctx), lb_grad(ctx), lb_grad(ctx), 1, t));
    R->u_final = E.f;
    R->phigrad = t[0];
    R->iterations = it;
    R->nforce = E.nevals;
    R->info = omode;
    R->status = omode == 1 ? 0 : (omode == 4 || omode == 5) ? 1 : omode == 2 ? 2 : 3;
    return MDFF_OK;
}

}  // namespace

extern "C" {

// EFG post-processing input: nconf configurations of the caller's tensors
// [nconf][6][natm] -- read in place when they are in device memory, else
// uploaded into context scratch -- or (efg6 NULL, nconf 1) the context's EFG of
// its last force evaluation.
static int efg_post_input(mdff_ctx* ctx, int nconf, const double* efg6, const double** src) {
    const size_t n = (size_t)ctx->n;
    if (nconf < 1) return fail(ctx, MDFF_E_ARG, "EFG post-processing: nconf must be >= 1");
    cudaPointerAttributes pa{};
    if (efg6 && cudaPointerGetAttributes(&pa, efg6) == cudaSuccess &&
        (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged)) {
        if (pa.device != ctx->p.device)
            return fail(ctx, MDFF_E_ARG, "EFG post-processing: tensors on another device");
        *src = efg6;
        return MDFF_OK;
    }
    cudaGetLastError();
    if (efg6) {
        TRY(dgrow(ctx, &ctx->efgp_t, &ctx->efgp_tcap, 6 * n * nconf));
        CK(cudaMemcpyAsync(ctx->efgp_t, efg6, sizeof(double) * 6 * n * nconf, cudaMemcpyHostToDevice, ctx->st));
        *src = ctx->efgp_t;
    } else {
        if (nconf != 1) return fail(ctx, MDFF_E_ARG, "EFG post-processing: the context holds one configuration");
        if (!(ctx->p.lcoulomb && ctx->p.doefg))
            return fail(ctx, MDFF_E_STATE, "no EFG in the context: pass tensors or evaluate forces with doefg");
        *src = ctx->efg;
    }
    return MDFF_OK;
}

// persistent grid of the EFG site kernel: three blocks per SM at most
static int efg_grid(mdff_ctx* ctx, int nchunk) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->p.device);
    return std::max(1, std::min(nchunk, 3 * sms));
}

int mdff_efg_nmr(mdff_ctx* ctx, int nconf, const double* efg6, double* nmr, double* U, double* S) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    cudaSetDevice(ctx->p.device);
    const double* src = nullptr;
    TRY(efg_post_input(ctx, nconf, efg6, &src));
    const size_t n = (size_t)ctx->n;
    TRY(dgrow(ctx, &ctx->efgp_nmr, &ctx->efgp_ncap, 10 * n * nconf));
    double* dn = ctx->efgp_nmr;
    double* du = dn + 4 * n * nconf;
    double* ds = du + 5 * n * nconf;
    EfgBins b{};
    const int nblk = (int)((n + EFG_THREADS - 1) / EFG_THREADS), nchunk = nblk * nconf;
    k_efg_sites<false, false><<<efg_grid(ctx, nchunk), EFG_THREADS, 0, ctx->st>>>(
        ctx->n, nblk, nchunk, src, ctx->type, b, nullptr, nullptr, dn, du, ds, nullptr);
    TRY(check_launch(ctx, "efg_sites"));
    if (nmr) CK(cudaMemcpyAsync(nmr, dn, sizeof(double) * 4 * n * nconf, cudaMemcpyDeviceToHost, ctx->st));
    if (U) CK(cudaMemcpyAsync(U, du, sizeof(double) * 5 * n * nconf, cudaMemcpyDeviceToHost, ctx->st));
    if (S) CK(cudaMemcpyAsync(S, ds, sizeof(double) * n * nconf, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

int mdff_efg_dist(mdff_ctx* ctx, int nconf, const double* efg6, const mdff_efg_dist_params* dp, double* stats,
                  double* mU, double* m2U, int* dib_vzz, int* dib_eta, int* dib_u, int* dib_s) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!dp || !(dp->resvzz > 0.0) || !(dp->reseta > 0.0) || !(dp->resu > 0.0))
        return fail(ctx, MDFF_E_ARG, "mdff_efg_dist: resolutions must be positive");
    if (ctx->ntype > EFG_NT_MAX) return fail(ctx, MDFF_E_UNSUPPORTED, "mdff_efg_dist: at most 16 types");
    cudaSetDevice(ctx->p.device);
    const double* src = nullptr;
    TRY(efg_post_input(ctx, nconf, efg6, &src));
    const int n = ctx->n, nt1 = ctx->ntype + 1;
    EfgBins b{};
    b.vzzmin = dp->vzzmin; b.resvzz = dp->resvzz; b.reseta = dp->reseta; b.umin = dp->umin; b.resu = dp->resu;
    b.ivzz = 1.0 / dp->resvzz; b.ieta = 1.0 / dp->reseta; b.iu = 1.0 / dp->resu;
    const double pv = (2.0 * std::fabs(dp->vzzmin)) / dp->resvzz, pe = 1.0 / dp->reseta;
    const double pu = (2.0 * std::fabs(dp->umin)) / dp->resu, ps = dp->smax / dp->resu;
    if (!(pv < 1e8 && pe < 1e8 && pu < 1e8 && ps < 1e8 && ps >= 0.0))
        return fail(ctx, MDFF_E_ARG, "mdff_efg_dist: bin counts out of range");
    b.PANvzz = (int)pv;                                      // efg_check_tag, src/efg.f90:233-236
    b.PANeta = (int)pe;
    b.PANU = (int)pu;
    b.PANS = (int)ps;
    b.ntype = ctx->ntype;
    const size_t nvzz = (size_t)nt1 * (b.PANvzz + 1), neta = (size_t)nt1 * (b.PANeta + 1);
    const size_t nu = (size_t)6 * nt1 * (b.PANU + 1), ns = (size_t)nt1 * (b.PANS + 1);
    const size_t nbins = nvzz + neta + nu + ns;
    if (nbins > (size_t)1 << 30) return fail(ctx, MDFF_E_ARG, "mdff_efg_dist: too many bins");
    b.ov = 0; b.oe = (int)nvzz; b.ou = (int)(nvzz + neta); b.os = (int)(nvzz + neta + nu); b.nbins = (int)nbins;
    const int nt = ctx->ntype;
    b.cv = 0;
    b.ce = b.cv + nt * (b.PANvzz + 1);
    b.cu = b.ce + nt * (b.PANeta + 1);
    b.cs = b.cu + 5 * nt * (b.PANU + 1);
    b.ncomp = b.cs + nt * (b.PANS + 1);
    const int nblk = (n + EFG_THREADS - 1) / EFG_THREADS;
    const size_t npart = (size_t)nconf * nblk * nt * EFG_NACC, nfin = (size_t)nconf * nt1 * EFG_NACC;
    TRY(dgrow(ctx, &ctx->efgp_hist, &ctx->efgp_hcap, nbins + 1));
    TRY(dgrow(ctx, &ctx->efgp_part, &ctx->efgp_pcap, npart + nfin));
    int* hist = ctx->efgp_hist;
    double* part = ctx->efgp_part;
    double* fin = part + npart;
    CK(cudaMemsetAsync(hist, 0, sizeof(int) * (nbins + 1), ctx->st));
    const int nchunk = nblk * nconf, grid = efg_grid(ctx, nchunk);
    ctx->prof.begin(PK_OTHER);
    ctx->prof.detail_begin(PD_EFG_SITES);
    if (b.ncomp <= EFG_SMEM_BINS)
        k_efg_sites<true, true><<<grid, EFG_THREADS, sizeof(int) * b.ncomp, ctx->st>>>(
            n, nblk, nchunk, src, ctx->type, b, hist, part, nullptr, nullptr, nullptr, hist + nbins);
    else
        k_efg_sites<true, false><<<grid, EFG_THREADS, 0, ctx->st>>>(n, nblk, nchunk, src, ctx->type, b, hist, part,
                                                                     nullptr, nullptr, nullptr, hist + nbins);
    TRY(check_launch(ctx, "efg_sites"));
    ctx->prof.detail_end(PD_EFG_SITES, 52.0 * n * nconf);
    k_efg_stats_fin<<<dim3((unsigned)nt1, (unsigned)nconf), EFG_THREADS, 0, ctx->st>>>(nblk, nt, part, fin);
    TRY(check_launch(ctx, "efg_stats_fin"));
    ctx->prof.end(2);
    std::vector<int> hh(nbins + 1);
    std::vector<double> ff(nfin);
    CK(cudaMemcpyAsync(hh.data(), hist, sizeof(int) * hh.size(), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(ff.data(), fin, sizeof(double) * nfin, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (dib_vzz) std::memcpy(dib_vzz, hh.data() + b.ov, sizeof(int) * nvzz);
    if (dib_eta) std::memcpy(dib_eta, hh.data() + b.oe, sizeof(int) * neta);
    if (dib_u) std::memcpy(dib_u, hh.data() + b.ou, sizeof(int) * nu);
    if (dib_s) std::memcpy(dib_s, hh.data() + b.os, sizeof(int) * ns);
    // Statistics as efg_stat forms them over its configuration loop
    // (src/efg.f90:2159-2330): the averages are zeroed once before the loop,
    // so each configuration's sums add to the previous configuration's
    // averages before the division; the extrema run over all configurations
    // from 0; <U> and <U U> are totals over all configurations divided by
    // nconf x sites at the end (:2435-2439), row 0 of <U U> left undivided.
    std::vector<double> vzzm(nt1, 0.0), vzzma(nt1, 0.0), etam(nt1, 0.0), vzzsq(nt1, 0.0), pvzz(nt1, 0.0);
    std::vector<double> vmin(nt1, 0.0), vmax(nt1, 0.0), cnt(nt1, 0.0), su(nt1 * 20, 0.0);
    for (int c = 0; c < nconf; ++c) {
        for (int t = 0; t < nt1; ++t) {
            const double* a = &ff[((size_t)c * nt1 + t) * EFG_NACC];
            const double k = a[5];
            vzzm[t] += a[0];
            vzzma[t] += a[1];
            etam[t] += a[2];
            vzzsq[t] += a[3];
            pvzz[t] += a[4];
            vmin[t] = std::min(vmin[t], a[26]);
            vmax[t] = std::max(vmax[t], a[27]);
            for (int q = 0; q < 20; ++q) su[t * 20 + q] += a[6 + q];
            cnt[t] = k;
            if (k > 0) {
                vzzm[t] /= k; vzzsq[t] /= k; vzzma[t] /= k; etam[t] /= k; pvzz[t] /= k;
            }
            const double sig = std::sqrt(vzzsq[t] - vzzma[t] * vzzma[t]);
            if (stats) {
                double* o = stats + ((size_t)c * nt1 + t) * 8;
                o[0] = vmin[t];
                o[1] = vmax[t];
                o[2] = vzzm[t];
                o[3] = vzzma[t];
                o[4] = etam[t];
                o[5] = pvzz[t];
                o[6] = vzzma[t] != 0.0 ? sig / vzzma[t] : 0.0;   // rho_z
                o[7] = sig;                                      // sigmavzz
            }
        }
    }
    for (int t = 0; t < nt1; ++t) {
        const double den = (double)nconf * cnt[t];
        if (mU)
            for (int k = 0; k < 5; ++k) mU[(size_t)t * 5 + k] = den > 0 ? su[t * 20 + k] / den : 0.0;
        if (m2U) {
            int m = 5;
            for (int k = 0; k < 5; ++k)
                for (int l = 0; l < 5; ++l) {
                    double v = 0.0;
                    if (l >= k) {
                        v = su[t * 20 + m++];
                        if (t > 0) v = den > 0 ? v / den : 0.0;
                    }
                    m2U[((size_t)t * 5 + k) * 5 + l] = v;
                }
        }
    }
    const int flag = hh[nbins];
    if (flag)
        return fail(ctx, MDFF_E_ARG,
                    "EFG value outside the distribution range (vzzmin, umin, smax) -- code " + std::to_string(flag));
    return MDFF_OK;
}

int mdff_opt_sastry(mdff_ctx* ctx, int itmax, mdff_opt_result* out) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!out || itmax < 1) return fail(ctx, MDFF_E_ARG, "mdff_opt_sastry: out must be given and itmax >= 1");
    cudaSetDevice(ctx->p.device);
    std::memset(out, 0, sizeof *out);
    return opt_sastry(ctx, itmax, out);
}

int mdff_opt_m1qn3(mdff_ctx* ctx, int niter, int nsim, double epsg, mdff_opt_result* out) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!out || niter < 1 || nsim < 1 || !(epsg > 0.0))
        return fail(ctx, MDFF_E_ARG, "mdff_opt_m1qn3: out must be given, niter >= 1, nsim >= 1 and epsg > 0");
    cudaSetDevice(ctx->p.device);
    std::memset(out, 0, sizeof *out);
    return opt_m1qn3(ctx, niter, nsim, epsg, out);
}

int mdff_opt_lbfgs(mdff_ctx* ctx, int itmax, double eps, mdff_opt_result* out) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!out || itmax < 1 || !(eps >= 0.0))
        return fail(ctx, MDFF_E_ARG, "mdff_opt_lbfgs: out must be given, itmax >= 1 and eps >= 0");
    cudaSetDevice(ctx->p.device);
    std::memset(out, 0, sizeof *out);
    return opt_lbfgs(ctx, itmax, eps, out);
}


// erfc_ex2 (the real-space kernels' erfc) and CUDA's erfc at the same points.
__global__ void k_erfc_check(int n, const double* __restrict__ x, double* __restrict__ ex2, double* __restrict__ ref) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = x[i];
    ex2[i] = mdff::erfc_ex2(v, exp(-v * v));
    ref[i] = erfc(v);
}

int mdff_erfc_check(int device, int n, const double* x, double* ex2, double* ref) {
    if (n < 1 || !x || !ex2 || !ref) return MDFF_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return MDFF_E_CUDA;
    double* d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * 3 * (size_t)n) != cudaSuccess) return MDFF_E_NOMEM;
    int rc = MDFF_OK;
    if (cudaMemcpy(d, x, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = MDFF_E_CUDA;
    if (rc == MDFF_OK) {
        k_erfc_check<<<(n + 255) / 256, 256>>>(n, d, d + n, d + 2 * (size_t)n);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(ex2, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(ref, d + 2 * (size_t)n, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = MDFF_E_CUDA;
    }
    cudaFree(d);
    return rc;
}

int mdff_measure_pipes(int device, double out[3]) {
    if (!out) return MDFF_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return MDFF_E_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256;
    void* buf = nullptr;
    if (cudaMalloc(&buf, 64) != cudaSuccess) return MDFF_E_NOMEM;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best[3] = {0, 0, 0};
    const double lanes = (double)blocks * threads * PK_ITERS;
    for (int rep = 0; rep < 4; ++rep) {
        for (int kind = 0; kind < 3; ++kind) {
            cudaEventRecord(a);
            if (kind == 0) k_peak_f64<<<blocks, threads>>>((double*)buf, 1.0);
            else if (kind == 1) k_peak_f32<<<blocks, threads>>>((float*)buf, 1.0f);
            else k_peak_f32x2<<<blocks, threads>>>((float*)buf, 1.0f);
            cudaEventRecord(b);
            cudaEventSynchronize(b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            double flops = lanes * (kind == 0 ? 8.0 : 16.0) * 2.0;
            double tf = flops / (ms * 1e-3) / 1e12;
            if (rep > 0 && tf > best[kind]) best[kind] = tf;
        }
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(buf);
    if (e != cudaSuccess) return MDFF_E_CUDA;
    for (int k = 0; k < 3; ++k) out[k] = best[k];
    return MDFF_OK;
}

int mdff_measure_tensor(int device, double out[3]) {
    if (!out) return MDFF_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return MDFF_E_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int* err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return MDFF_E_NOMEM;
    cudaMemset(err, 0, sizeof(int));
    const int niter = 4096;
    cudaFuncSetAttribute(k_peak_i8<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (128 + 256) * 64);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int ns[3] = {256, 96, 64};
    double best[3] = {0, 0, 0};
    for (int rep = 0; rep < 3; ++rep)
        for (int k = 0; k < 3; ++k) {
            const int N = ns[k];
            const size_t smem = (size_t)(128 + N) * 64;
            cudaEventRecord(a);
            if (N == 256) k_peak_i8<256><<<sms, 128, smem>>>(niter, err);
            else if (N == 96) k_peak_i8<96><<<sms, 128, smem>>>(niter, err);
            else k_peak_i8<64><<<sms, 128, smem>>>(niter, err);
            cudaEventRecord(b);
            cudaEventSynchronize(b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            const double ops = 2.0 * 128 * N * 64 * (double)niter * sms;
            const double tops = ops / (ms * 1e-3) / 1e12;
            if (rep > 0 && tops > best[k]) best[k] = tops;
        }
    int herr = 0;
    cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(err);
    if (e != cudaSuccess || herr) return MDFF_E_CUDA;
    for (int k = 0; k < 3; ++k) out[k] = best[k];
    return MDFF_OK;
}

int mdff_profile_detail(mdff_ctx* ctx, double ms[MDFF_NDETAIL], long long count[MDFF_NDETAIL],
                        double ops[MDFF_NDETAIL]) {
    static_assert(PD_NDETAIL == MDFF_NDETAIL, "detail timer count");
    if (!ctx) return MDFF_E_ARG;
    cudaSetDevice(ctx->p.device);
    CK(cudaStreamSynchronize(ctx->st));
    ctx->prof.harvest();
    for (int k = 0; k < PD_NDETAIL; ++k) {
        if (ms) ms[k] = ctx->prof.dms[k];
        if (count) count[k] = ctx->prof.dcount[k];
        if (ops) ops[k] = ctx->prof.dops[k];
    }
    return MDFF_OK;
}

int mdff_profile(mdff_ctx* ctx, int enable) {
    if (!ctx) return MDFF_E_ARG;
    ctx->prof.on = enable != 0;
    return MDFF_OK;
}

int mdff_profile_get(mdff_ctx* ctx, double ms[8], long long count[8], long long* launches, int reset) {
    if (!ctx) return MDFF_E_ARG;
    cudaSetDevice(ctx->p.device);
    CK(cudaStreamSynchronize(ctx->st));
    ctx->prof.harvest();
    for (int k = 0; k < PK_NKIND; ++k) {
        if (ms) ms[k] = ctx->prof.ms[k];
        if (count) count[k] = ctx->prof.count[k];
    }
    if (launches) *launches = ctx->prof.launches;
    if (reset) ctx->prof.reset();
    return MDFF_OK;
}

int mdff_get_velocities(mdff_ctx* ctx, double* vx, double* vy, double* vz) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    cudaSetDevice(ctx->p.device);
    TRY(download(ctx, vx, ctx->vx, ctx->n));
    TRY(download(ctx, vy, ctx->vy, ctx->n));
    TRY(download(ctx, vz, ctx->vz, ctx->n));
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

int mdff_stream(mdff_ctx* ctx, void** stream) {
    if (!ctx || !stream) return MDFF_E_ARG;
    *stream = (void*)ctx->st;
    return MDFF_OK;
}

int mdff_launch_shape(mdff_ctx* ctx, int out[4]) {
    if (!ctx || !out) return MDFF_E_ARG;
    out[0] = ctx->g_dir;
    out[1] = ctx->g_dd;
    out[2] = ctx->rs.p_mul;
    out[3] = ctx->rs.s_mul;
    return MDFF_OK;
}

int mdff_kspace_mode(mdff_ctx* ctx, int out[2]) {
    if (!ctx || !out) return MDFF_E_ARG;
    out[0] = ctx->rs.tc.on ? 1 : 0;
    out[1] = ctx->rs.low.tc ? 1 : 0;
    return MDFF_OK;
}

int mdff_graph_info(mdff_ctx* ctx, long long out[3]) {
    if (!ctx || !out) return MDFF_E_ARG;
    out[0] = ctx->nstep_graph;
    out[1] = ctx->ncapture;
    out[2] = ctx->nstep_plain;
    return MDFF_OK;
}

int mdff_kspace_info(mdff_ctx* ctx, long long out[4]) {
    if (!ctx || !out) return MDFF_E_ARG;
    if (!ctx->have_system) return fail(ctx, MDFF_E_STATE, "set_system first");
    for (int k = 0; k < 4; ++k) out[k] = ctx->kinfo[k];
    return MDFF_OK;
}

int mdff_struct_size(int which) {
    switch (which) {
        case 0: return (int)sizeof(mdff_params);
        case 1: return (int)sizeof(mdff_energies);
        case 2: return (int)sizeof(mdff_thermo);
        case 3: return (int)sizeof(mdff_param_grad);
        case 4: return (int)sizeof(mdff_opt_result);
        case 5: return (int)sizeof(mdff_efg_dist_params);
        case 6: return (int)sizeof(mdff_frame_header);
        case 7: return (int)sizeof(mdff_rmc_params);
        case 8: return (int)sizeof(mdff_rmc_result);
        case 9: return (int)sizeof(mdff_rmc_efg_params);
        default: return -1;
    }
}

void mdff_params_default(mdff_params* p) {
    std::memset(p, 0, sizeof *p);
    p->ntype = 1;
    p->lvnlist = 1;
    p->skindiff = 0.15;
    p->symmetric_pot = 1;
    p->trunc = MDFF_TRUNC_NONE;
    for (int i = 0; i < MDFF_NTYPE_MAX; ++i) {
        p->mass[i] = 1.0;
        for (int j = 0; j < MDFF_NTYPE_MAX; ++j) { p->qlj[i][j] = 12.0; p->plj[i][j] = 6.0; }
    }
    p->alphaES = 1.0;
    p->kES[0] = p->kES[1] = p->kES[2] = 10;
    p->epsw = 1e-6;
    p->conv_tol_ind = 1e-6;
    p->min_scf_pol_iter = 3;
    p->max_scf_pol_iter = 100;
    p->extrapolate_order = 0;
    p->algo_ext_dipole = MDFF_EXT_POLY;
    p->algo_moment_from_pola = MDFF_POLA_SCF;
    p->integrator = MDFF_NVE_VV;
    p->temp = 1.0;
    p->nhc_n = 4;
    p->nhc_yosh_order = 3;
    p->nhc_mults = 2;
    p->timesca_thermo = 1.0;
    p->precision = MDFF_PREC_FP64;
    p->mixed_ksplit = 2.5;
    p->mixed_keps = 1e-7;
    p->kspace_tc = 2;
    p->press = 0.0;
    p->timesca_baro = 1.0;   // md_default_tag (src/md.f90:204)
}

int mdff_create(const mdff_params* p, mdff_ctx** out) {
    if (!p || !out) return MDFF_E_ARG;
    *out = nullptr;
    mdff_ctx* ctx = new mdff_ctx();
    ctx->p = *p;
    int rc = check_params(ctx, ctx->p);
    if (rc != MDFF_OK) { *out = ctx; return rc; }
    if (ctx->p.integrator == MDFF_NVT_NHC2) ctx->p.nhc_n = 2;   // extended_coordinates_alloc (src/md.f90:335-340)
    symmetrise(ctx->p);
    set_units(ctx);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        ctx->err = std::string("no CUDA device: ") + cudaGetErrorString(e);
        *out = ctx;
        return MDFF_E_CUDA;
    }
    if (p->device < 0 || p->device >= ndev) { ctx->err = "device ordinal out of range"; *out = ctx; return MDFF_E_ARG; }
    cudaSetDevice(p->device);
    e = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->st2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&ctx->hsc, sizeof(DevScalars));
    ctx->prof.st = ctx->st;
    if (e != cudaSuccess) { ctx->err = std::string("stream/pinned alloc: ") + cudaGetErrorString(e); *out = ctx; return MDFF_E_CUDA; }
    *out = ctx;
    return MDFF_OK;
}

void mdff_destroy(mdff_ctx* ctx) {
    if (!ctx) return;
    if (ctx->st) {
        cudaSetDevice(ctx->p.device);
        cudaStreamSynchronize(ctx->st);
        ctx->prof.release();
        free_all(ctx);
        if (ctx->ddtab) cudaFree(ctx->ddtab);
        if (ctx->ddnbr) cudaFree(ctx->ddnbr);
        drop_graphs(ctx);
        cudaStreamDestroy(ctx->st);
        if (ctx->st2) cudaStreamDestroy(ctx->st2);
    }
    if (ctx->hsc) cudaFreeHost(ctx->hsc);
    delete ctx;
}

const char* mdff_last_error(const mdff_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int mdff_set_system(mdff_ctx* ctx, int natm, const int* itype, const double* rx, const double* ry, const double* rz,
                    const double A[9]) {
    if (!ctx || !ctx->st) return MDFF_E_STATE;
    if (natm < 1 || !itype || !rx || !ry || !rz || !A) return fail(ctx, MDFF_E_ARG, "invalid system arguments");
    cudaSetDevice(ctx->p.device);
    cudaStreamSynchronize(ctx->st);
    drop_graphs(ctx);   // they hold the addresses of the buffers freed here
    ctx->coef_valid = false;
    free_all(ctx);
    ctx->lv = NList();
    ctx->lc = NList();
    ctx->grid = CellGrid();
    ctx->have_system = ctx->have_list = ctx->forces_valid = ctx->md_started = false;
    const mdff_params& p = ctx->p;
    const int n = natm;
    ctx->n = n;
    ctx->ntype = p.ntype;
    lattice(A, ctx->cell, ctx->W, ctx->anorm);
    if (!(ctx->cell.omega > 0.0)) return fail(ctx, MDFF_E_ARG, "cell volume must be positive");
    std::memcpy(ctx->A_cur, A, sizeof ctx->A_cur);
    ctx->npt = NptState();
    ctx->natmi.assign(NT, 0);
    std::vector<int> t0(n);
    std::vector<double> hq(n), hm(n), ha(n), hia(n), hd(3 * (size_t)n);
    ctx->npol = 0;
    ctx->any_q = ctx->any_dip0 = false;
    for (int t = 0; t < p.ntype; ++t) {
        if (p.qch[t] != 0.0) ctx->any_q = true;
        for (int c = 0; c < 3; ++c) if (p.dip[t][c] != 0.0) ctx->any_dip0 = true;
    }
    for (int i = 0; i < n; ++i) {
        int t = itype[i] - 1;
        if (t < 0 || t >= p.ntype) return fail(ctx, MDFF_E_ARG, "itype out of range (1-based)");
        t0[i] = t;
        ctx->natmi[t]++;
        hq[i] = p.qch[t];
        hm[i] = p.mass[t];
        if (!(hm[i] > 0.0)) return fail(ctx, MDFF_E_ARG, "mass must be positive");
        ha[i] = p.ldip_polar[t] ? p.poldip_iso[t] : 0.0;
        hia[i] = ha[i] != 0.0 ? 1.0 / ha[i] : 0.0;
        if (ha[i] != 0.0) ctx->npol++;
        for (int c = 0; c < 3; ++c) hd[(size_t)c * n + i] = p.dip[t][c];
    }
    ctx->cut_vdw = p.cutshortrange;
    if (p.lcoulomb) ewald_param(ctx);
    else ctx->cut_coul = p.cutlongrange;
    std::vector<PairConst> tab;
    build_pair_consts(ctx, tab);
    ctx->omega0 = ctx->cell.omega;
    ctx->utail0 = ctx->utail;
    ctx->ptail0 = ctx->ptail;
    // device buffers
    double** d1[] = {&ctx->x, &ctx->y, &ctx->z, &ctx->vx, &ctx->vy, &ctx->vz, &ctx->fx, &ctx->fy, &ctx->fz,
                     &ctx->fox, &ctx->foy, &ctx->foz, &ctx->sx, &ctx->sy, &ctx->sz, &ctx->xs, &ctx->ys, &ctx->zs,
                     &ctx->q, &ctx->mass, &ctx->alpha, &ctx->inv_alpha};
    for (double** b : d1) TRY(dalloc(ctx, b, n));
    double** d3[] = {&ctx->dip0, &ctx->mu, &ctx->mu_ind, &ctx->Estat, &ctx->Eind, &ctx->E, &ctx->cg_r, &ctx->cg_z,
                     &ctx->cg_d, &ctx->cg_Ad, &ctx->mu_save, &ctx->ef, &ctx->fcoul};
    for (double** b : d3) TRY(dalloc(ctx, b, 3 * (size_t)n));
    TRY(dalloc(ctx, &ctx->efg, 6 * (size_t)n));
    ctx->nhist = p.extrapolate_order + 1;
    TRY(dalloc(ctx, &ctx->hist, (size_t)ctx->nhist * 3 * n));
    TRY(dalloc(ctx, &ctx->coef, PLAN_LEN));
    TRY(dalloc(ctx, &ctx->type, n));
    TRY(dalloc(ctx, &ctx->pc, NT * NT));
    TRY(dalloc(ctx, &ctx->dsc, 1));
    TRY(dalloc(ctx, &ctx->d_overflow, 1));
    TRY(dalloc(ctx, &ctx->grid.cell_of, n));
    TRY(dalloc(ctx, &ctx->grid.cell_atoms, n));
    TRY(dalloc(ctx, &ctx->grid.cell_w, n));
    CK(cudaMemsetAsync(ctx->dsc, 0, sizeof(DevScalars), ctx->st));
    CK(cudaMemsetAsync(ctx->hist, 0, sizeof(double) * ctx->nhist * 3 * (size_t)n, ctx->st));
    CK(cudaMemsetAsync(ctx->mu_ind, 0, sizeof(double) * 3 * (size_t)n, ctx->st));
    CK(cudaMemsetAsync(ctx->vx, 0, sizeof(double) * n, ctx->st));
    CK(cudaMemsetAsync(ctx->vy, 0, sizeof(double) * n, ctx->st));
    CK(cudaMemsetAsync(ctx->vz, 0, sizeof(double) * n, ctx->st));
    CK(cudaMemsetAsync(ctx->fcoul, 0, sizeof(double) * 3 * (size_t)n, ctx->st));
    CK(cudaMemsetAsync(ctx->efg, 0, sizeof(double) * 6 * (size_t)n, ctx->st));
    CK(cudaMemcpyAsync(ctx->type, t0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->pc, tab.data(), sizeof(PairConst) * NT * NT, cudaMemcpyHostToDevice, ctx->st));
    TRY(upload(ctx, ctx->q, hq.data(), n));
    TRY(upload(ctx, ctx->mass, hm.data(), n));
    TRY(upload(ctx, ctx->alpha, ha.data(), n));
    TRY(upload(ctx, ctx->inv_alpha, hia.data(), n));
    TRY(upload(ctx, ctx->dip0, hd.data(), 3 * n));
    TRY(upload(ctx, ctx->x, rx, n));
    TRY(upload(ctx, ctx->y, ry, n));
    TRY(upload(ctx, ctx->z, rz, n));
    launch_wrap_positions(ctx->st, n, ctx->x, ctx->y, ctx->z, ctx->cell);
    // Ewald k grid (kpoint_sum_init, src/kspace.f90:142-207) as a full rectangle
    if (p.lcoulomb) {
        KGrid& kg = ctx->kg;
        for (int d = 0; d < 3; ++d) kg.kmax[d] = ctx->kES[d];
        kg.ncol = (kg.kmax[0] + 1) * (2 * kg.kmax[1] + 1);
        kg.nzl = 2 * kg.kmax[2] + 1;
        kg.nrect = kg.ncol * kg.nzl;
        std::vector<double> ak(kg.nrect, 0.0), kc(kg.nrect, 0.0);
        double a2 = ctx->alphaES * ctx->alphaES;
        const CellP& c = ctx->cell;
        for (int col = 0; col < kg.ncol; ++col) {
            int nx = col / (2 * kg.kmax[1] + 1), ny = col % (2 * kg.kmax[1] + 1) - kg.kmax[1];
            for (int m = 0; m < kg.nzl; ++m) {
                int nz = m - kg.kmax[2];
                bool keep = nx > 0 || (nx == 0 && ny > 0) || (nx == 0 && ny == 0 && nz > 0);
                if (!keep) continue;
                double kx = 2.0 * PI * (double(nx) * c.B[0] + double(ny) * c.B[1] + double(nz) * c.B[2]);
                double ky = 2.0 * PI * (double(nx) * c.B[3] + double(ny) * c.B[4] + double(nz) * c.B[5]);
                double kz = 2.0 * PI * (double(nx) * c.B[6] + double(ny) * c.B[7] + double(nz) * c.B[8]);
                double kk = kx * kx + ky * ky + kz * kz;
                if (kk == 0.0) continue;
                ak[(size_t)col * kg.nzl + m] = std::exp(-kk * 0.25 / a2) / kk;
                kc[(size_t)col * kg.nzl + m] = 2.0 * (1.0 / kk + 1.0 / a2 / 4.0);
            }
        }
        ctx->kinfo[0] = kg.nrect;
        ctx->kinfo[1] = 0;
        for (double v : ak) ctx->kinfo[1] += v != 0.0;
        ctx->kinfo[2] = ctx->kinfo[3] = 0;
        kg.nfitems = kg.nfcol = 0;
        if (p.precision == MDFF_PREC_FP64) {
            // fp64_keps: leave out the vectors whose Gaussian factor
            // exp(-k^2 / 4 alpha^2) is below fp64_keps (the sphere the mixed
            // path's mixed_keps cuts), and give the FP64 kernels work lists of
            // what is left: (column, nz chunk) items for the structure factor,
            // the columns with their nz ranges for the field
            if (p.fp64_keps > 0.0) {
                const double R2 = -4.0 * a2 * std::log(p.fp64_keps);
                const int CH = kg.nzl <= 8 ? 8 : kg.nzl <= 12 ? 12 : 16;   // plan()'s chunk
                std::vector<int> items, fcols, fzr;
                for (int col = 0; col < kg.ncol; ++col) {
                    int nx = col / (2 * kg.kmax[1] + 1), ny = col % (2 * kg.kmax[1] + 1) - kg.kmax[1];
                    int lo = -1, hi = -1;
                    for (int m = 0; m < kg.nzl; ++m) {
                        const size_t r = (size_t)col * kg.nzl + m;
                        if (ak[r] == 0.0) continue;
                        int nz = m - kg.kmax[2];
                        double kx = 2.0 * PI * (double(nx) * c.B[0] + double(ny) * c.B[1] + double(nz) * c.B[2]);
                        double ky = 2.0 * PI * (double(nx) * c.B[3] + double(ny) * c.B[4] + double(nz) * c.B[5]);
                        double kz = 2.0 * PI * (double(nx) * c.B[6] + double(ny) * c.B[7] + double(nz) * c.B[8]);
                        if (kx * kx + ky * ky + kz * kz > R2) { ak[r] = 0.0; kc[r] = 0.0; continue; }
                        if (lo < 0) lo = m;
                        hi = m;
                    }
                    if (lo < 0) continue;
                    fcols.push_back(col);
                    fzr.push_back(lo);
                    fzr.push_back(hi - lo + 1);
                    for (int h = lo / CH; h <= hi / CH; ++h) { items.push_back(col); items.push_back(h); }
                }
                kg.nfitems = (int)(items.size() / 2);
                kg.nfcol = (int)fcols.size();
                if (kg.nfcol > 0) {
                    TRY(dalloc(ctx, &kg.fitems, items.size()));
                    TRY(dalloc(ctx, &kg.fcols, fcols.size()));
                    TRY(dalloc(ctx, &kg.fzr, fzr.size()));
                    CK(cudaMemcpyAsync(kg.fitems, items.data(), sizeof(int) * items.size(), cudaMemcpyHostToDevice,
                                       ctx->st));
                    CK(cudaMemcpyAsync(kg.fcols, fcols.data(), sizeof(int) * fcols.size(), cudaMemcpyHostToDevice,
                                       ctx->st));
                    CK(cudaMemcpyAsync(kg.fzr, fzr.data(), sizeof(int) * fzr.size(), cudaMemcpyHostToDevice, ctx->st));
                    CK(cudaStreamSynchronize(ctx->st));   // the host vectors go out of scope
                }
            }
            for (double v : ak) ctx->kinfo[2] += v != 0.0;
        }
        TRY(dalloc(ctx, &kg.Ak, kg.nrect));
        TRY(dalloc(ctx, &kg.kcoe, kg.nrect));
        TRY(upload(ctx, kg.Ak, ak.data(), kg.nrect));
        TRY(upload(ctx, kg.kcoe, kc.data(), kg.nrect));
        // Mixed path: the k-vectors with |k| < mixed_ksplit * alpha form the
        // FP64 low set (one contiguous nz interval per column, |k|^2 being
        // convex in nz) and are removed from the FP32 set.
        ctx->rs.low = LowK();
        std::vector<double> akhi = ak;   // the FP32 set of the mixed path
        if (p.precision == MDFF_PREC_MIXED && p.mixed_ksplit > 0.0) {
            const double ks2 = std::pow(p.mixed_ksplit * ctx->alphaES, 2);
            std::vector<int> cols;
            std::vector<double> akl, kcl;
            int nzmax = 0;
            struct Col { int nx, ny, lo, nn; };
            std::vector<Col> cl;
            for (int col = 0; col < kg.ncol; ++col) {
                int nx = col / (2 * kg.kmax[1] + 1), ny = col % (2 * kg.kmax[1] + 1) - kg.kmax[1];
                int lo = -1, hi = -2;
                for (int m = 0; m < kg.nzl; ++m) {
                    size_t r = (size_t)col * kg.nzl + m;
                    if (ak[r] == 0.0) continue;
                    int nz = m - kg.kmax[2];
                    double kx = 2.0 * PI * (double(nx) * c.B[0] + double(ny) * c.B[1] + double(nz) * c.B[2]);
                    double ky = 2.0 * PI * (double(nx) * c.B[3] + double(ny) * c.B[4] + double(nz) * c.B[5]);
                    double kz = 2.0 * PI * (double(nx) * c.B[6] + double(ny) * c.B[7] + double(nz) * c.B[8]);
                    if (kx * kx + ky * ky + kz * kz < ks2) {
                        if (lo < 0) lo = m;
                        hi = m;
                    }
                }
                if (lo < 0) continue;
                cl.push_back({nx, ny, lo, hi - lo + 1});
                nzmax = std::max(nzmax, hi - lo + 1);
            }
            LowK& lk = ctx->rs.low;
            lk.ncol = (int)cl.size();
            lk.nzmax = nzmax;
            if (lk.ncol > 0) {
                cols.resize(4 * (size_t)lk.ncol);
                akl.assign((size_t)lk.ncol * nzmax, 0.0);
                kcl.assign((size_t)lk.ncol * nzmax, 0.0);
                for (int q = 0; q < lk.ncol; ++q) {
                    const Col& C_ = cl[q];
                    int col = C_.nx * (2 * kg.kmax[1] + 1) + (C_.ny + kg.kmax[1]);
                    cols[4 * q] = C_.nx;
                    cols[4 * q + 1] = C_.ny;
                    cols[4 * q + 2] = C_.lo - kg.kmax[2];
                    cols[4 * q + 3] = C_.nn;
                    for (int m = 0; m < C_.nn; ++m) {
                        size_t r = (size_t)col * kg.nzl + C_.lo + m;
                        akl[(size_t)q * nzmax + m] = ak[r];
                        kcl[(size_t)q * nzmax + m] = kc[r];
                        akhi[r] = 0.0;
                    }
                }
                long long thr = (long long)((lk.ncol + 127) / 128) * 128 * ((nzmax + 15) / 16);
                int P = (int)std::max<long long>(1, (148LL * 1536 + thr - 1) / thr);
                P = std::min(P, std::max(1, n / 32));
                lk.natom_chunk = (n + P - 1) / P;
                lk.P = (n + lk.natom_chunk - 1) / lk.natom_chunk;
                TRY(dalloc(ctx, &lk.col, cols.size()));
                CK(cudaMemcpyAsync(lk.col, cols.data(), sizeof(int) * cols.size(), cudaMemcpyHostToDevice, ctx->st));
                TRY(dalloc(ctx, &lk.Ak, akl.size()));
                TRY(dalloc(ctx, &lk.kcoe, kcl.size()));
                TRY(upload(ctx, lk.Ak, akl.data(), (int)akl.size()));
                TRY(upload(ctx, lk.kcoe, kcl.data(), (int)kcl.size()));
                // tensor-core form: one tile of list columns per 128, atoms split
                // so that the grid covers the SMs about once
                int kxl = 0, kyl = 0, kzl = 0;
                for (const Col& C_ : cl) {
                    kxl = std::max(kxl, std::abs(C_.nx));
                    kyl = std::max(kyl, std::abs(C_.ny));
                    kzl = std::max(kzl, std::max(std::abs(C_.lo - kg.kmax[2]), std::abs(C_.lo + C_.nn - 1 - kg.kmax[2])));
                }
                lk.tc = 0;
                if (p.kspace_tc == 2) {
                    // GEMM rows nz = -kzl..-1, 1..kzl (the nz = 0 row is summed apart)
                    lk.kx = kxl; lk.ky = kyl; lk.kz = kzl; lk.nzl = 2 * kzl;
                    lk.N = std::max(16, ((2 * lk.nzl + 15) / 16) * 16);
                    lk.XYW = kxl + 2 + 2 * kyl;
                    lk.KZ = std::max(32, ((2 * lk.nzl + 31) / 32) * 32);
                    lk.ntile = (lk.ncol + 127) / 128;
                    lk.nblk = (n + tc4::SA - 1) / tc4::SA;
                    lk.npad = lk.nblk * tc4::SA;
                    const int S = std::max(1, 148 / lk.ntile);
                    lk.bps = std::min(std::max(1, (lk.nblk + S - 1) / S), tc4::MAX_ATOMS_PER_CTA / tc4::SA);
                    lk.nsplit = (lk.nblk + lk.bps - 1) / lk.bps;
                    lk.ntile_f = (n + 127) / 128;
                    const size_t smax = 227 * 1024;
                    lk.nin = tc4::Layout::depth(lk.N, lk.XYW, smax - 10 * 1024);   // static shared memory aside
                    const tc4::Layout l4(lk.N, lk.XYW, std::max(lk.nin, 2));
                    const tc4::FLayout f2(lk.KZ, lk.XYW, tc4::Cfg<2>::NB, tc4::Cfg<2>::CB);
                    const tc4::FLayout f3(lk.KZ, lk.XYW, tc4::Cfg<3>::NB, tc4::Cfg<3>::CB);
                    lk.smem = l4.smem_bytes();
                    lk.smem_f2 = f2.smem_bytes();
                    lk.smem_f3 = f3.smem_bytes();
                    lk.tc = lk.N <= tc4::LS && lk.KZ <= 128 && lk.nin >= 2 && lk.smem_f2 <= smax &&
                            lk.smem_f3 <= smax;
                    if (lk.tc) {
                        const size_t ncb2 = (lk.ncol + tc4::Cfg<2>::CB - 1) / tc4::Cfg<2>::CB;
                        const size_t ncb3 = (lk.ncol + tc4::Cfg<3>::CB - 1) / tc4::Cfg<3>::CB;
                        TRY(dalloc(ctx, &lk.xy, (size_t)lk.npad * lk.XYW));
                        TRY(dalloc(ctx, &lk.bimg, (size_t)lk.nblk * l4.b_bytes()));
                        TRY(dalloc(ctx, &lk.prm, (size_t)lk.npad));
                        TRY(dalloc(ctx, &lk.amax, (size_t)lk.npad));
                        TRY(dalloc(ctx, &lk.aimg, (size_t)lk.ntile_f * f2.a_bytes()));
                        TRY(dalloc(ctx, &lk.xyt, (size_t)lk.ntile_f * lk.XYW * 128));
                        TRY(dalloc(ctx, &lk.fimg, std::max(ncb2 * f2.stage_bytes, ncb3 * f3.stage_bytes)));
                        CK(cudaFuncSetAttribute(tc4::k_sfac_tc4, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)lk.smem));
                        CK(cudaFuncSetAttribute(tc4::k_kfield_tc4<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)lk.smem_f2));
                        CK(cudaFuncSetAttribute(tc4::k_kfield_tc4<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)lk.smem_f3));
                    }
                }
                TRY(dalloc(ctx, &lk.part, 2 * (size_t)std::max(lk.P, lk.tc ? lk.nsplit : 0) * nzmax * lk.ncol));
                TRY(dalloc(ctx, &lk.aks, 2 * (size_t)lk.ncol * nzmax));
                TRY(dalloc(ctx, &lk.aks_acc, 2 * (size_t)lk.ncol * nzmax));
                TRY(dalloc(ctx, &lk.fpart, 4 * 9 * (size_t)n));
                TRY(dalloc(ctx, &lk.tab, 16 * (size_t)n));
            }
        }
        size_t tc_part = 0;
        if (p.precision == MDFF_PREC_MIXED) {
            // Leave out the k-vectors whose Gaussian factor exp(-k^2 / 4 alpha^2)
            // is below mixed_keps (a sphere |k|^2 > -4 alpha^2 ln mixed_keps).
            if (p.mixed_keps > 0.0) {
                const double R2 = -4.0 * ctx->alphaES * ctx->alphaES * std::log(p.mixed_keps);
                for (int col = 0; col < kg.ncol; ++col) {
                    int nx = col / (2 * kg.kmax[1] + 1), ny = col % (2 * kg.kmax[1] + 1) - kg.kmax[1];
                    for (int m = 0; m < kg.nzl; ++m) {
                        int nz = m - kg.kmax[2];
                        double kx = 2.0 * PI * (double(nx) * c.B[0] + double(ny) * c.B[1] + double(nz) * c.B[2]);
                        double ky = 2.0 * PI * (double(nx) * c.B[3] + double(ny) * c.B[4] + double(nz) * c.B[5]);
                        double kz = 2.0 * PI * (double(nx) * c.B[6] + double(ny) * c.B[7] + double(nz) * c.B[8]);
                        if (kx * kx + ky * ky + kz * kz > R2) akhi[(size_t)col * kg.nzl + m] = 0.0;
                    }
                }
            }
            // per column the range of 16-wide nz chunks holding a nonzero entry,
            // and the (column, chunk) work list of the FP32 structure factor
            std::vector<int> crange(2 * (size_t)kg.ncol, 0), items;
            for (int col = 0; col < kg.ncol; ++col) {
                int lo = -1, hi = -1;
                for (int m = 0; m < kg.nzl; ++m)
                    if (akhi[(size_t)col * kg.nzl + m] != 0.0) { if (lo < 0) lo = m; hi = m; }
                if (lo < 0) continue;
                crange[2 * col] = lo / 16;
                crange[2 * col + 1] = hi / 16 - lo / 16 + 1;
                for (int h = lo / 16; h <= hi / 16; ++h) { items.push_back(col); items.push_back(h); }
            }
            kg.nitems = (int)(items.size() / 2);
            for (double v : akhi) ctx->kinfo[2] += v != 0.0;
            ctx->kinfo[3] = 0;
            for (int col = 0; col < kg.ncol; ++col)
                for (int m = 0; m < kg.nzl; ++m)
                    if (ak[(size_t)col * kg.nzl + m] != 0.0 && akhi[(size_t)col * kg.nzl + m] == 0.0 &&
                        ctx->rs.low.ncol > 0) {
                        // in the low set when below the split (the rest is outside the sphere)
                        int nx = col / (2 * kg.kmax[1] + 1), ny = col % (2 * kg.kmax[1] + 1) - kg.kmax[1];
                        int nz = m - kg.kmax[2];
                        double kx = 2.0 * PI * (double(nx) * c.B[0] + double(ny) * c.B[1] + double(nz) * c.B[2]);
                        double ky = 2.0 * PI * (double(nx) * c.B[3] + double(ny) * c.B[4] + double(nz) * c.B[5]);
                        double kz = 2.0 * PI * (double(nx) * c.B[6] + double(ny) * c.B[7] + double(nz) * c.B[8]);
                        if (kx * kx + ky * ky + kz * kz < std::pow(p.mixed_ksplit * ctx->alphaES, 2)) ctx->kinfo[3]++;
                    }
            TRY(dalloc(ctx, &kg.colrange, crange.size()));
            CK(cudaMemcpyAsync(kg.colrange, crange.data(), sizeof(int) * crange.size(), cudaMemcpyHostToDevice, ctx->st));
            TRY(dalloc(ctx, &kg.items, std::max<size_t>(2, items.size())));
            if (!items.empty())
                CK(cudaMemcpyAsync(kg.items, items.data(), sizeof(int) * items.size(), cudaMemcpyHostToDevice, ctx->st));
            TRY(dalloc(ctx, &kg.Ak_hi, kg.nrect));
            TRY(upload(ctx, kg.Ak_hi, akhi.data(), kg.nrect));
            // tensor-core structure factor: GEMM rows = the columns of the work
            // list, N = 2 x (nz rows padded to 8), atoms split so that the grid
            // covers the 148 SMs about once
            TcK& tc = ctx->rs.tc;
            const int N = ((2 * kg.nzl + 15) / 16) * 16;
            tc.on = p.kspace_tc && !items.empty() && N <= tcs::LSTRIDE;
            if (tc.on) {
                std::vector<int> sph;
                for (size_t i = 0; i < items.size(); i += 2)
                    if (sph.empty() || sph.back() != items[i]) sph.push_back(items[i]);
                tc.nsph = (int)sph.size();
                tc.ntile = (tc.nsph + 127) / 128;
                tc.N = N;
                tc.kx = kg.kmax[0]; tc.ky = kg.kmax[1]; tc.kz = kg.kmax[2]; tc.nzl = kg.nzl;
                tc.XYW = ((kg.kmax[0] + 2 + 2 * kg.kmax[1]) + 1) / 2 * 2;
                tc.nblk = (n + tcs::SA - 1) / tcs::SA;
                tc.npad = tc.nblk * tcs::SA;
                int S = std::max(1, 148 / tc.ntile);
                tc.bps = std::max(1, (tc.nblk + S - 1) / S);
                tc.bps = std::min(tc.bps, 600);      // int32 headroom of the digit accumulators
                tc.nsplit = (tc.nblk + tc.bps - 1) / tc.bps;
                const tcs::Layout lay(N, tc.XYW);
                tc.smem = lay.smem_bytes();
                TRY(dalloc(ctx, &tc.cols, tc.nsph));
                CK(cudaMemcpyAsync(tc.cols, sph.data(), sizeof(int) * tc.nsph, cudaMemcpyHostToDevice, ctx->st));
                CK(cudaStreamSynchronize(ctx->st));
                TRY(dalloc(ctx, &tc.xy, (size_t)tc.npad * tc.XYW));
                TRY(dalloc(ctx, &tc.bimg, (size_t)tc.nblk * lay.b_bytes()));
                TRY(dalloc(ctx, &tc.prm, (size_t)tc.npad));
                TRY(dalloc(ctx, &tc.amax, (size_t)tc.npad));
                CK(cudaFuncSetAttribute(tcs::k_sfac_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc.smem));
                CK(cudaFuncSetAttribute(tcs::k_sfac_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc.smem));
                tc_part = 2 * (size_t)tc.nsplit * kg.ncol * (((kg.nzl + TM - 1) / TM) * TM);
                // field pass
                tc.KZ = ((2 * kg.nzl + 31) / 32) * 32;
                tc.ntile_f = (n + 127) / 128;
                {
                    int sms = 148;
                    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device);
                    tc.grid_f = std::max(1, std::min(tc.ntile_f, sms));
                }
                const tcf::FLayout f2(tc.KZ, tc.XYW, tcf::Cfg<2>::NB, tcf::Cfg<2>::CB);
                const tcf::FLayout f3(tc.KZ, tc.XYW, tcf::Cfg<3>::NB, tcf::Cfg<3>::CB);
                tc.smem_f2 = f2.smem_bytes();
                tc.smem_f3 = f3.smem_bytes();
                const size_t ncb2 = (tc.nsph + tcf::Cfg<2>::CB - 1) / tcf::Cfg<2>::CB;
                const size_t ncb3 = (tc.nsph + tcf::Cfg<3>::CB - 1) / tcf::Cfg<3>::CB;
                TRY(dalloc(ctx, &tc.aimg, (size_t)tc.ntile_f * f2.a_bytes()));
                TRY(dalloc(ctx, &tc.xyt, (size_t)tc.ntile_f * tc.XYW * 128));
                TRY(dalloc(ctx, &tc.fimg, std::max(ncb2 * f2.stage_bytes, ncb3 * f3.stage_bytes)));
                CK(cudaFuncSetAttribute(tcf::k_kfield_tc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tc.smem_f2));
                CK(cudaFuncSetAttribute(tcf::k_kfield_tc<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tc.smem_f3));
            }
            CK(cudaStreamSynchronize(ctx->st));   // the host vectors above go out of scope
        }
        {   // k membership for cell changes (constant pressure, mdff_set_cell)
            std::vector<unsigned char> mk(kg.nrect);
            for (int r = 0; r < kg.nrect; ++r)
                mk[r] = (unsigned char)((ak[r] != 0.0 ? 1 : 0) | (akhi[r] != 0.0 ? 2 : 0));
            TRY(dalloc(ctx, &kg.mask, kg.nrect));
            CK(cudaMemcpyAsync(kg.mask, mk.data(), kg.nrect, cudaMemcpyHostToDevice, ctx->st));
            CK(cudaStreamSynchronize(ctx->st));
        }
        size_t fp = 0;
        size_t pc = std::max(tc_part, rec_scratch_doubles(n, kg, &fp, p.precision == MDFF_PREC_MIXED));
        fp = std::max(fp, (size_t)2 * tcf::NQ * 9 * n);   // tensor-core field pass: NQ column parts x 2 column slots
        TRY(dalloc(ctx, &ctx->rs.part, pc));
        TRY(dalloc(ctx, &ctx->rs.fpart, fp));
        TRY(dalloc(ctx, &ctx->rs.aks, 2 * (size_t)kg.nrect));
        TRY(dalloc(ctx, &ctx->rs.aks_acc, 2 * (size_t)kg.nrect));
        TRY(dalloc(ctx, &ctx->rs.fixed, 3 * (size_t)n));
        TRY(dalloc(ctx, &ctx->rs.tab, (size_t)n * 16));
        TRY(dalloc(ctx, &ctx->rs.aks2, (size_t)kg.ncol * (((kg.nzl + 15) / 16) * 16)));
        ctx->rs.part_cap = pc;
        ctx->rs.fpart_cap = fp;
    }
    int parts = std::max(16 * 1024, 12 * (int)(((size_t)n * 32 + 255) / 256));
    TRY(dalloc(ctx, &ctx->part.buf, parts));
    ctx->part.capacity = parts;
    // neighbour lists
    int cap = p.nlist_capacity;
    if (cap <= 0) {
        double rl = rlist_max(ctx, p.skindiff);
        double dens = (double)n / ctx->cell.omega;
        double est = 4.0 / 3.0 * PI * rl * rl * rl * dens;
        cap = (int)std::min<double>((double)n, est * 1.4 + 32.0);
        cap = std::max(cap, 32);
    }
    TRY(ensure_lists(ctx, cap));
    ctx->itime = 0;
    ctx->have_system = true;
    if (p.lvnlist) TRY(build_lists(ctx, p.skindiff));
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

int mdff_set_cell(mdff_ctx* ctx, const double A[9]) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!A) return fail(ctx, MDFF_E_ARG, "mdff_set_cell: A is NULL");
    cudaSetDevice(ctx->p.device);
    TRY(apply_cell(ctx, A));
    // the lists are rebuilt by the next force evaluation (or list read), so a
    // new cell and new positions together cost one build
    ctx->have_list = false;
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

int mdff_set_positions(mdff_ctx* ctx, const double* rx, const double* ry, const double* rz) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    cudaSetDevice(ctx->p.device);
    TRY(upload(ctx, ctx->x, rx, ctx->n));
    TRY(upload(ctx, ctx->y, ry, ctx->n));
    TRY(upload(ctx, ctx->z, rz, ctx->n));
    // a list built for other positions is not a list of these: rebuilt by
    // the next force evaluation (or list read)
    ctx->have_list = false;
    CK(cudaStreamSynchronize(ctx->st));
    ctx->forces_valid = false;
    return MDFF_OK;
}

int mdff_get_positions(mdff_ctx* ctx, double* rx, double* ry, double* rz) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    cudaSetDevice(ctx->p.device);
    TRY(download(ctx, rx, ctx->x, ctx->n));
    TRY(download(ctx, ry, ctx->y, ctx->n));
    TRY(download(ctx, rz, ctx->z, ctx->n));
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

int mdff_nlist_build(mdff_ctx* ctx) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    cudaSetDevice(ctx->p.device);
    TRY(build_lists(ctx, ctx->p.skindiff));
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

int mdff_nlist_get(mdff_ctx* ctx, int which, int* point, int* list, int cap, int* nlist) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!point || !nlist || (which != 0 && which != 1)) return fail(ctx, MDFF_E_ARG, "invalid nlist_get arguments");
    cudaSetDevice(ctx->p.device);
    if (!ctx->have_list) {
        TRY(build_lists(ctx, ctx->p.skindiff));
        CK(cudaStreamSynchronize(ctx->st));
    }
    const int n = ctx->n;
    bool nonb = ctx->p.lnmlj || ctx->p.lbmhft || ctx->p.lbmhftd || ctx->p.lmorse;
    if (which == 0 && !nonb) return fail(ctx, MDFF_E_STATE, "no vdW list without a short-range potential");
    if (which == 1 && !ctx->p.lcoulomb) return fail(ctx, MDFF_E_STATE, "no Coulomb list without lcoulomb");
    const NList* L = which == 0 ? &ctx->lv : &coul_list(ctx);
    const double want = which == 0 ? ctx->cut_vdw : ctx->cut_coul;
    if (L->cut != want) return fail(ctx, MDFF_E_STATE, "list radius mismatch");
    std::vector<int> cnt(n), nbr((size_t)n * L->cap);
    CK(cudaMemcpyAsync(cnt.data(), L->cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(nbr.data(), L->nbr, sizeof(int) * (size_t)n * L->cap, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    int total = 0;
    std::vector<int> row;
    for (int i = 0; i < n; ++i) {
        point[i] = total + 1;
        row.clear();
        const int I = i + 1;
        for (int k = 0; k < cnt[i]; ++k) {
            int j = nbr[(size_t)i * L->cap + k];
            int J = j + 1;
            if ((I > J && ((I + J) % 2 == 0)) || (I < J && ((I + J) % 2 != 0))) row.push_back(J);
        }
        std::sort(row.begin(), row.end());
        if (list && total + (int)row.size() <= cap) std::memcpy(list + total, row.data(), sizeof(int) * row.size());
        total += (int)row.size();
    }
    point[n] = total + 1;
    *nlist = total;
    if (total > cap) return fail(ctx, MDFF_E_LISTOVF, "list buffer too small");
    return MDFF_OK;
}

int mdff_engforce(mdff_ctx* ctx, double* fx, double* fy, double* fz, mdff_energies* e, double tau_nonb[9],
                  double tau_coul[9], double* ef, double* efg, double* mu) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    cudaSetDevice(ctx->p.device);
    TRY(engforce_device(ctx));
    const int n = ctx->n;
    if (fx) TRY(download(ctx, fx, ctx->fx, n));
    if (fy) TRY(download(ctx, fy, ctx->fy, n));
    if (fz) TRY(download(ctx, fz, ctx->fz, n));
    if (ef) TRY(download(ctx, ef, ctx->ef, 3 * n));
    if (efg) TRY(download(ctx, efg, ctx->efg, 6 * n));
    if (mu) TRY(download(ctx, mu, ctx->mu, 3 * n));
    CK(cudaStreamSynchronize(ctx->st));
    if (ef && !ctx->p.lcoulomb) std::memset(ef, 0, sizeof(double) * 3 * n);
    if (efg && !(ctx->p.lcoulomb && ctx->p.doefg)) std::memset(efg, 0, sizeof(double) * 6 * n);
    if (mu && !ctx->p.lcoulomb) std::memset(mu, 0, sizeof(double) * 3 * n);
    if (e) *e = ctx->en;
    if (tau_nonb) std::memcpy(tau_nonb, ctx->tau_nonb, sizeof ctx->tau_nonb);
    if (tau_coul) std::memcpy(tau_coul, ctx->tau_coul, sizeof ctx->tau_coul);
    return MDFF_OK;
}

int mdff_md_start(mdff_ctx* ctx, const double* vx, const double* vy, const double* vz, mdff_thermo* t0) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    cudaSetDevice(ctx->p.device);
    const int n = ctx->n;
    if (vx) TRY(upload(ctx, ctx->vx, vx, n));
    if (vy) TRY(upload(ctx, ctx->vy, vy, n));
    if (vz) TRY(upload(ctx, ctx->vz, vz, n));
    CK(cudaMemsetAsync(ctx->dsc->xi, 0, sizeof(double) * 16, ctx->st));
    CK(cudaMemsetAsync(ctx->dsc->vxi, 0, sizeof(double) * 16, ctx->st));
    CK(cudaMemsetAsync(&ctx->dsc->e_nvt, 0, sizeof(double), ctx->st));
    {   // xe = ve = 0 (md_check_tag, src/md.f90:349-350); the cell stays as set
        const double sc = ctx->npt.scale, sb = ctx->npt.scale_build;
        ctx->npt = NptState();
        ctx->npt.scale = sc;
        ctx->npt.scale_build = sb;
        if (ctx->p.integrator == MDFF_NPT_NHCNP) ctx->npt.e_npt = ctx->p.press * ctx->u.press * ctx->cell.omega;
    }
    ctx->itime = 0;
    TRY(ke_reduce(ctx, 0));
    TRY(engforce_device(ctx));   // syncs the scalars
    set_kin(ctx);
    ctx->last_rebuilt = 0;
    ctx->md_started = true;
    if (t0) fill_thermo(ctx, t0, 0);
    return MDFF_OK;
}

int mdff_step(mdff_ctx* ctx, int nsteps, double* rx, double* ry, double* rz, double* vx, double* vy, double* vz,
              double* fx, double* fy, double* fz, mdff_thermo* thermo) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!ctx->md_started) return fail(ctx, MDFF_E_STATE, "mdff_md_start first");
    if (nsteps < 0) return fail(ctx, MDFF_E_ARG, "nsteps < 0");
    cudaSetDevice(ctx->p.device);
    const int n = ctx->n;
    bool new_pos = rx || ry || rz;
    if (rx) TRY(upload(ctx, ctx->x, rx, n));
    if (ry) TRY(upload(ctx, ctx->y, ry, n));
    if (rz) TRY(upload(ctx, ctx->z, rz, n));
    if (vx) TRY(upload(ctx, ctx->vx, vx, n));
    if (vy) TRY(upload(ctx, ctx->vy, vy, n));
    if (vz) TRY(upload(ctx, ctx->vz, vz, n));
    if (new_pos && !ctx->forces_valid) TRY(engforce_device(ctx));
    for (int k = 0; k < nsteps; ++k) {
        TRY(md_step(ctx));
        if (thermo) fill_thermo(ctx, &thermo[k], ctx->itime);
    }
    if (rx) TRY(download(ctx, rx, ctx->x, n));
    if (ry) TRY(download(ctx, ry, ctx->y, n));
    if (rz) TRY(download(ctx, rz, ctx->z, n));
    if (vx) TRY(download(ctx, vx, ctx->vx, n));
    if (vy) TRY(download(ctx, vy, ctx->vy, n));
    if (vz) TRY(download(ctx, vz, ctx->vz, n));
    if (fx) TRY(download(ctx, fx, ctx->fx, n));
    if (fy) TRY(download(ctx, fy, ctx->fy, n));
    if (fz) TRY(download(ctx, fz, ctx->fz, n));
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Reciprocal-space energy of point charges without any device allocation.
//
// Some callers cannot let the library allocate device memory during a run:
// a host code whose device memory is entirely held by its own pool (a Fortran
// code that reserves the GPU at start-up, or a PyTorch process whose caching
// allocator already owns the free memory), or code that must not enter the
// CUDA allocator in the middle of a time step.  mdff_rec_energy_noalloc reads
// the caller's own device arrays and keeps all of its scratch in one fixed
// array in device global memory, so it calls neither cudaMalloc nor cudaFree.
//
// The scratch holds the fractional coordinates, the structure-factor partials
// and the energy partials of one call; nothing in it has to start at zero
// (every word a call reads is written earlier in the same call).  There is one
// scratch per device, so two calls that overlap on the same device (two host
// threads, or two streams without ordering between them) race on it and must
// be serialised by the caller.
namespace {

constexpr size_t NOALLOC_SCRATCH_DOUBLES = (size_t)1 << 21;   // 16 MiB of device memory per device

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];


// Energy sum over the k rectangle from the structure-factor partials, with
// A_k = exp(-k^2/4 alpha^2)/k^2 evaluated in place (no k table): the energy
// part of k_sfac_reduce.
__global__ void k_sfac_energy_inplace(int P, int ch, int nchunk, int ncol, int nzl, int ky, int kz,
                                      const double* __restrict__ part_re, const double* __restrict__ part_im,
                                      double inv4a2, CellP c, double* partials) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (t < ncol * nzl) {
        const int col = t % ncol;
        const int mz = t / ncol;
        const int ny_n = 2 * ky + 1;
        const int nx = col / ny_n, ny = col % ny_n - ky, nz = mz - kz;
        const bool keep = nx > 0 || (nx == 0 && ny > 0) || (nx == 0 && ny == 0 && nz > 0);
        if (keep) {
            const size_t plane = (size_t)ncol * ch * nchunk;
            const size_t off = (size_t)mz * ncol + col;
            double sr = 0.0, si = 0.0;
            for (int p = 0; p < P; ++p) {
                sr += part_re[(size_t)p * plane + off];
                si += part_im[(size_t)p * plane + off];
            }
            const double k0 = 2.0 * PI * (nx * c.B[0] + ny * c.B[1] + nz * c.B[2]);
            const double k1 = 2.0 * PI * (nx * c.B[3] + ny * c.B[4] + nz * c.B[5]);
            const double k2 = 2.0 * PI * (nx * c.B[6] + ny * c.B[7] + nz * c.B[8]);
            const double kk = k0 * k0 + k1 * k1 + k2 * k2;
            if (kk != 0.0) v[0] = (sr * sr + si * si) * (exp(-kk * inv4a2) / kk);
        }
    }
    block_partials<1>(v, partials);
}

// Device address of the current device's scratch.  In host code the name
// g_noalloc_scratch is a host-side stand-in, not a device address, so every
// call looks the address up with the device current.  The lookup is a host
// query that allocates nothing; doing it per call (rather than caching it)
// keeps the address right if the caller resets the device, which reloads the
// module and can move the array.
int noalloc_scratch(double** out) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return MDFF_E_CUDA;
    *out = (double*)p;
    return MDFF_OK;
}

}  // namespace

extern "C" int mdff_rec_energy_noalloc(int device, int natm, const double* rx, const double* ry, const double* rz,
                                       const double* q, const double A[9], double alpha, const int kmax[3],
                                       void* stream, double* u_rec, long long* scratch_needed) {
    if (!rx || !ry || !rz || !q || !A || !kmax || !u_rec || natm < 1 || !(alpha > 0.0)) return MDFF_E_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) return MDFF_E_CUDA;
    if (device < 0 || device >= ndev) return MDFF_E_ARG;
    for (int d = 0; d < 3; ++d)
        if (kmax[d] < 0 || kmax[d] > 64) return MDFF_E_ARG;
    // scratch layout: sx sy sz (3 natm), partials (2 plane), energy partials, result
    KGrid kg;
    for (int d = 0; d < 3; ++d) kg.kmax[d] = kmax[d];
    kg.ncol = (kmax[0] + 1) * (2 * kmax[1] + 1);
    kg.nzl = 2 * kmax[2] + 1;
    kg.nrect = kg.ncol * kg.nzl;
    const RecLaunch L = plan(natm, kg);
    const size_t plane = (size_t)L.P * L.nchunk * L.CH * kg.ncol;
    const int rb = (kg.nrect + 255) / 256;
    const size_t need = 3 * (size_t)natm + 2 * plane + (size_t)rb + 1;
    if (scratch_needed) *scratch_needed = (long long)need;
    if (need > NOALLOC_SCRATCH_DOUBLES) return MDFF_E_NOMEM;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return MDFF_E_CUDA;
    if (prev != device && cudaSetDevice(device) != cudaSuccess) return MDFF_E_CUDA;
    int rc = MDFF_OK;
    double* scr = nullptr;
    if ((rc = noalloc_scratch(&scr)) == MDFF_OK) {
        cudaStream_t st = (cudaStream_t)stream;
        CellP c;
        double W[3], anorm[3];
        lattice(A, c, W, anorm);
        double *sx = scr, *sy = scr + natm, *sz = scr + 2 * (size_t)natm;
        double* pre = scr + 3 * (size_t)natm;
        double* pim = pre + plane;
        double* epart = pim + plane;
        double* res = epart + rb;
        launch_frac(st, natm, rx, ry, rz, c, sx, sy, sz);
        dim3 g1(L.nchunk * L.ncolblk, L.P);
#define SFAC_NA(CHV) k_sfac<CHV><<<g1, SF_THREADS, 0, st>>>(natm, L.natom_chunk, sx, sy, sz, q, nullptr, c, kmax[0], \
                                                        kmax[1], kmax[2], kg.ncol, L.ncolblk, L.nchunk, 1, 0, pre, pim, \
                                                        nullptr, 0)
        if (L.CH == 16) SFAC_NA(16);
        else if (L.CH == 12) SFAC_NA(12);
        else SFAC_NA(8);
#undef SFAC_NA
        k_sfac_energy_inplace<<<rb, 256, 0, st>>>(L.P, L.CH, L.nchunk, kg.ncol, kg.nzl, kmax[1], kmax[2], pre, pim,
                                                  0.25 / (alpha * alpha), c, epart);
        launch_reduce_partials(st, epart, rb, 1, res, 0);
        double h = 0.0;
        // launch errors are read without clearing them: an error left by the
        // caller's own earlier work stays the caller's to see
        if (cudaPeekAtLastError() != cudaSuccess ||
            cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = MDFF_E_CUDA;
        else
            *u_rec = h * 2.0 * (2.0 * PI / c.omega) * 14.3996441494161;   // eV, as mdff_energies.u_rec
    }
    if (prev != device) cudaSetDevice(prev);
    return rc;
}

// ---------------------------------------------------------------------------
// On-disk formats, the streaming writer and checkpoints.
extern "C" {

int mdff_io_format(int file, int iformat, int data, const mdff_frame_header* h, const int* itype,
                   const double* cols, char* out, size_t cap, size_t* len) {
    if (!h || !itype || !cols || !len) return MDFF_E_ARG;
    std::string o;
    const int rc = mdff::io::format_frame(file, iformat, data, *h, itype, cols, o);
    if (rc != MDFF_OK) return rc;
    *len = o.size();
    if (!out || cap < o.size()) return MDFF_E_ARG;
    std::memcpy(out, o.data(), o.size());
    return MDFF_OK;
}

}  // extern "C"

struct mdff_writer {
    mdff_ctx* ctx = nullptr;
    int file = 0, iformat = 1, data = 0, ncol = 0, nslot = 0, device = 0;
    std::string path;
    mdff_frame_header h{};
    std::vector<int> itype;                 // 1-based, host
    std::FILE* f = nullptr;
    cudaStream_t cs = nullptr;
    double* dbuf = nullptr;                 // [nslot][ncol][n] device snapshots
    std::vector<double*> hbuf;              // pinned host copies
    std::vector<cudaEvent_t> ev_snap, ev_copy;
    std::vector<mdff_frame_header> hslot;   // header (cell) of each slot's frame
    std::thread th;
    std::mutex m;
    std::condition_variable cv;
    std::deque<int> queue;
    std::vector<int> free_slots;
    bool stop = false;
    int err = MDFF_OK;
    std::string errmsg;
};

namespace {

void writer_loop(mdff_writer* w) {
    cudaSetDevice(w->device);
    std::string out;
    for (;;) {
        int s;
        {
            std::unique_lock<std::mutex> lk(w->m);
            w->cv.wait(lk, [&] { return w->stop || !w->queue.empty(); });
            if (w->queue.empty()) break;
            s = w->queue.front();
            w->queue.pop_front();
        }
        int rc = MDFF_OK;
        std::string msg;
        if (cudaEventSynchronize(w->ev_copy[s]) != cudaSuccess) {
            rc = MDFF_E_CUDA;
            msg = "writer: device copy failed";
        } else {
            out.clear();
            rc = mdff::io::format_frame(w->file, w->iformat, w->data, w->hslot[s], w->itype.data(), w->hbuf[s], out);
            if (rc != MDFF_OK) msg = "writer: frame could not be formatted";
            if (rc == MDFF_OK && w->file == MDFF_FILE_CONTFF) {   // rewritten at every call
                std::FILE* g = std::fopen(w->path.c_str(), "wb");
                if (!g || std::fwrite(out.data(), 1, out.size(), g) != out.size()) {
                    rc = MDFF_E_ARG;
                    msg = "writer: cannot write " + w->path;
                }
                if (g) std::fclose(g);
            } else if (rc == MDFF_OK) {
                if (std::fwrite(out.data(), 1, out.size(), w->f) != out.size() || std::fflush(w->f) != 0) {
                    rc = MDFF_E_ARG;
                    msg = "writer: cannot write " + w->path;
                }
            }
        }
        {
            std::lock_guard<std::mutex> lk(w->m);
            if (rc != MDFF_OK && w->err == MDFF_OK) {
                w->err = rc;
                w->errmsg = msg;
            }
            w->free_slots.push_back(s);
        }
        w->cv.notify_all();
    }
}

void writer_free(mdff_writer* w) {
    if (w->th.joinable()) {
        {
            std::lock_guard<std::mutex> lk(w->m);
            w->stop = true;
        }
        w->cv.notify_all();
        w->th.join();
    }
    if (w->f) std::fclose(w->f);
    for (auto e : w->ev_snap)
        if (e) cudaEventDestroy(e);
    for (auto e : w->ev_copy)
        if (e) cudaEventDestroy(e);
    for (auto p : w->hbuf)
        if (p) cudaFreeHost(p);
    if (w->dbuf) cudaFree(w->dbuf);
    if (w->cs) cudaStreamDestroy(w->cs);
    delete w;
}

// the snapshot of slot s on the engine's stream and its copy to the host
int writer_snapshot(mdff_writer* w, int s) {
    mdff_ctx* ctx = w->ctx;
    const int n = ctx->n;
    double* d = w->dbuf + (size_t)s * w->ncol * n;
    const size_t b = sizeof(double) * n;
    // the slot's previous device-to-host copy has finished before it is overwritten
    CK(cudaStreamWaitEvent(ctx->st, w->ev_copy[s], 0));
    auto dd = [&](int c, const double* src, int k) {
        return cudaMemcpyAsync(d + (size_t)c * n, src, b * k, cudaMemcpyDeviceToDevice, ctx->st);
    };
    if (w->file == MDFF_FILE_TRAJFF || w->file == MDFF_FILE_CONTFF) {
        const int data = w->file == MDFF_FILE_CONTFF ? (MDFF_DATA_V | MDFF_DATA_F) : w->data;
        int c = 0;
        CK(dd(c++, ctx->x, 1));
        CK(dd(c++, ctx->y, 1));
        CK(dd(c++, ctx->z, 1));
        if (data & MDFF_DATA_V) {
            CK(dd(c++, ctx->vx, 1));
            CK(dd(c++, ctx->vy, 1));
            CK(dd(c++, ctx->vz, 1));
        }
        if (data & MDFF_DATA_F) {
            CK(dd(c++, ctx->fx, 1));
            CK(dd(c++, ctx->fy, 1));
            CK(dd(c++, ctx->fz, 1));
        }
        // kardir, periodicbc, dirkar of the written copy (write_trajff_xyz, src/config.f90:552-554)
        launch_wrap_positions(ctx->st, n, d, d + n, d + 2 * (size_t)n, ctx->cell);
        TRY(check_launch(ctx, "writer wrap"));
    } else if (w->file == MDFF_FILE_EFGALL) {
        CK(dd(0, ctx->efg, 6));
    } else if (w->file == MDFF_FILE_DIPFF) {
        CK(dd(0, ctx->mu, 3));
    } else {
        CK(dd(0, ctx->ef, 3));
    }
    CK(cudaEventRecord(w->ev_snap[s], ctx->st));
    CK(cudaStreamWaitEvent(w->cs, w->ev_snap[s], 0));
    CK(cudaMemcpyAsync(w->hbuf[s], d, b * w->ncol, cudaMemcpyDeviceToHost, w->cs));
    CK(cudaEventRecord(w->ev_copy[s], w->cs));
    mdff_frame_header& hs = w->hslot[s];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) hs.A[i + 3 * j] = ctx->cell.A[i * 3 + j];
    return MDFF_OK;
}

}  // namespace

extern "C" {

int mdff_writer_open(mdff_ctx* ctx, const char* path, int file, int iformat, int data, const mdff_frame_header* h,
                     int nslot, mdff_writer** out) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!path || !h || !out || nslot < 1) return fail(ctx, MDFF_E_ARG, "mdff_writer_open: bad argument");
    const int ncol = mdff::io::frame_cols(file, data);
    if (ncol < 0) return fail(ctx, MDFF_E_ARG, "mdff_writer_open: unknown file kind");
    if (iformat == 0 && file != MDFF_FILE_TRAJFF && file != MDFF_FILE_EFGALL)
        return fail(ctx, MDFF_E_UNSUPPORTED, "mdff_writer_open: only TRAJFF and EFGALL have an unformatted form");
    if (file == MDFF_FILE_EFGALL && !(ctx->p.lcoulomb && ctx->p.doefg))
        return fail(ctx, MDFF_E_STATE, "EFGALL needs lcoulomb and doefg");
    if ((file == MDFF_FILE_DIPFF || file == MDFF_FILE_EFALL) && !ctx->p.lcoulomb)
        return fail(ctx, MDFF_E_STATE, "DIPFF / EFALL need lcoulomb");
    cudaSetDevice(ctx->p.device);
    const int n = ctx->n;
    auto* w = new mdff_writer;
    w->ctx = ctx;
    w->file = file;
    w->iformat = iformat;
    w->data = data;
    w->ncol = ncol;
    w->nslot = nslot;
    w->device = ctx->p.device;
    w->path = path;
    w->h = *h;
    w->h.natm = n;
    w->h.ntype = ctx->ntype;
    for (int t = 0; t < ctx->ntype; ++t) w->h.natmi[t] = ctx->natmi[t];
    std::vector<int> t0(n);
    cudaError_t e = cudaMemcpyAsync(t0.data(), ctx->type, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    w->itype.resize(n);
    for (int i = 0; i < n; ++i) w->itype[i] = t0[i] + 1;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w->cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc((void**)&w->dbuf, sizeof(double) * (size_t)nslot * ncol * n);
    w->hbuf.assign(nslot, nullptr);
    w->ev_snap.assign(nslot, nullptr);
    w->ev_copy.assign(nslot, nullptr);
    w->hslot.assign(nslot, w->h);
    for (int s = 0; s < nslot && e == cudaSuccess; ++s) {
        e = cudaHostAlloc((void**)&w->hbuf[s], sizeof(double) * (size_t)ncol * n, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w->ev_snap[s], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w->ev_copy[s], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(w->ev_copy[s], w->cs);   // the slot starts free
        w->free_slots.push_back(s);
    }
    if (e != cudaSuccess) {
        writer_free(w);
        return fail(ctx, MDFF_E_CUDA, std::string("mdff_writer_open: ") + cudaGetErrorString(e));
    }
    if (file != MDFF_FILE_CONTFF) {
        w->f = std::fopen(path, "ab");
        if (!w->f) {
            writer_free(w);
            return fail(ctx, MDFF_E_ARG, std::string("mdff_writer_open: cannot open ") + path);
        }
    }
    w->th = std::thread(writer_loop, w);
    *out = w;
    return MDFF_OK;
}

int mdff_writer_frame(mdff_writer* w) {
    if (!w) return MDFF_E_ARG;
    mdff_ctx* ctx = w->ctx;
    cudaSetDevice(w->device);
    int s;
    {
        std::unique_lock<std::mutex> lk(w->m);
        w->cv.wait(lk, [&] { return !w->free_slots.empty() || w->err != MDFF_OK; });
        if (w->err != MDFF_OK) return fail(ctx, w->err, w->errmsg);
        s = w->free_slots.back();
        w->free_slots.pop_back();
    }
    const int rc = writer_snapshot(w, s);
    if (rc != MDFF_OK) {   // the slot goes back unused
        {
            std::lock_guard<std::mutex> lk(w->m);
            w->free_slots.push_back(s);
        }
        w->cv.notify_all();
        return rc;
    }
    {
        std::lock_guard<std::mutex> lk(w->m);
        w->queue.push_back(s);
    }
    w->cv.notify_all();
    return MDFF_OK;
}

int mdff_writer_close(mdff_writer* w) {
    if (!w) return MDFF_E_ARG;
    cudaSetDevice(w->device);
    {
        // drain: every queued frame written and its slot returned
        std::unique_lock<std::mutex> lk(w->m);
        w->cv.wait(lk, [&] { return (int)w->free_slots.size() == w->nslot; });
    }
    const int rc = w->err;
    if (rc != MDFF_OK && w->ctx) w->ctx->err = w->errmsg;
    writer_free(w);
    return rc;
}

}  // extern "C"

// ---- checkpoint -------------------------------------------------------------
namespace {
struct CkHost {
    char magic[8];
    int32_t version, n, ntype, nhist, nparam_bytes;
    int32_t itime, last_rebuilt, nrebuild, md_started, forces_valid, have_list, tuned, g_dir, g_dd, p_mul, s_mul;
    int32_t pad;
    double e_kin, temp_r;
    mdff_energies en;
    double tau_nonb[9], tau_coul[9];
    double A_cur[9];
    NptState npt;
};
constexpr char CK_MAGIC[8] = {'M', 'D', 'F', 'F', 'C', 'K', 'P', '2'};

// the device arrays of the state, in file order
std::vector<std::pair<double*, size_t>> ck_arrays(mdff_ctx* ctx) {
    const size_t n = ctx->n;
    return {{ctx->x, n},         {ctx->y, n},          {ctx->z, n},
            {ctx->vx, n},        {ctx->vy, n},         {ctx->vz, n},
            {ctx->fx, n},        {ctx->fy, n},         {ctx->fz, n},
            {ctx->fox, n},       {ctx->foy, n},        {ctx->foz, n},
            {ctx->xs, n},        {ctx->ys, n},         {ctx->zs, n},
            {ctx->mu, 3 * n},    {ctx->mu_ind, 3 * n}, {ctx->hist, (size_t)ctx->nhist * 3 * n},
            {ctx->ef, 3 * n},    {ctx->efg, 6 * n}};
}

mdff_params ck_params(const mdff_params& p) {
    mdff_params q = p;
    q.device = 0;
    q.autotune = 0;
    return q;
}

size_t ck_size(mdff_ctx* ctx) {
    size_t need = sizeof(CkHost) + sizeof(mdff_params) + sizeof(DevScalars);
    for (auto& a : ck_arrays(ctx)) need += sizeof(double) * a.second;
    return need;
}
}  // namespace

extern "C" {

int mdff_checkpoint_save(mdff_ctx* ctx, void* buf, size_t cap, size_t* len) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!len) return fail(ctx, MDFF_E_ARG, "mdff_checkpoint_save: len is NULL");
    const size_t need = ck_size(ctx);
    *len = need;
    if (!buf) return MDFF_OK;
    if (cap < need) return fail(ctx, MDFF_E_ARG, "mdff_checkpoint_save: buffer too small");
    cudaSetDevice(ctx->p.device);
    CkHost hdr{};
    std::memcpy(hdr.magic, CK_MAGIC, 8);
    hdr.version = 2;
    hdr.n = ctx->n;
    hdr.ntype = ctx->ntype;
    hdr.nhist = ctx->nhist;
    hdr.nparam_bytes = (int)sizeof(mdff_params);
    hdr.itime = ctx->itime;
    hdr.last_rebuilt = ctx->last_rebuilt;
    hdr.nrebuild = ctx->nrebuild;
    hdr.md_started = ctx->md_started;
    hdr.forces_valid = ctx->forces_valid;
    hdr.have_list = ctx->have_list;
    hdr.tuned = ctx->tuned;
    hdr.g_dir = ctx->g_dir;
    hdr.g_dd = ctx->g_dd;
    hdr.p_mul = ctx->rs.p_mul;
    hdr.s_mul = ctx->rs.s_mul;
    hdr.e_kin = ctx->e_kin;
    hdr.temp_r = ctx->temp_r;
    hdr.en = ctx->en;
    std::memcpy(hdr.tau_nonb, ctx->tau_nonb, sizeof hdr.tau_nonb);
    std::memcpy(hdr.tau_coul, ctx->tau_coul, sizeof hdr.tau_coul);
    std::memcpy(hdr.A_cur, ctx->A_cur, sizeof hdr.A_cur);
    hdr.npt = ctx->npt;
    char* o = (char*)buf;
    std::memcpy(o, &hdr, sizeof hdr);
    o += sizeof hdr;
    const mdff_params pp = ck_params(ctx->p);
    std::memcpy(o, &pp, sizeof pp);
    o += sizeof pp;
    CK(cudaMemcpyAsync(o, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->st));
    o += sizeof(DevScalars);
    for (auto& a : ck_arrays(ctx)) {
        CK(cudaMemcpyAsync(o, a.first, sizeof(double) * a.second, cudaMemcpyDeviceToHost, ctx->st));
        o += sizeof(double) * a.second;
    }
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

int mdff_checkpoint_load(mdff_ctx* ctx, const void* buf, size_t len) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!buf || len < sizeof(CkHost)) return fail(ctx, MDFF_E_ARG, "mdff_checkpoint_load: no checkpoint");
    CkHost hdr;
    std::memcpy(&hdr, buf, sizeof hdr);
    if (std::memcmp(hdr.magic, CK_MAGIC, 8) != 0 || hdr.version != 2)
        return fail(ctx, MDFF_E_ARG, "mdff_checkpoint_load: not a checkpoint of this library");
    if (hdr.n != ctx->n || hdr.ntype != ctx->ntype || hdr.nhist != ctx->nhist ||
        hdr.nparam_bytes != (int)sizeof(mdff_params))
        return fail(ctx, MDFF_E_ARG, "mdff_checkpoint_load: checkpoint of another system");
    if (len != ck_size(ctx)) return fail(ctx, MDFF_E_ARG, "mdff_checkpoint_load: size mismatch");
    drop_graphs(ctx);
    const char* in = (const char*)buf + sizeof hdr;
    const mdff_params pp = ck_params(ctx->p);
    if (std::memcmp(in, &pp, sizeof pp) != 0)
        return fail(ctx, MDFF_E_ARG, "mdff_checkpoint_load: parameters differ from the checkpoint's");
    in += sizeof pp;
    cudaSetDevice(ctx->p.device);
    // the cell of the checkpoint (constant pressure moves it), then the state
    if (std::memcmp(hdr.A_cur, ctx->A_cur, sizeof hdr.A_cur) != 0) TRY(apply_cell(ctx, hdr.A_cur));
    ctx->npt = hdr.npt;
    CK(cudaMemcpyAsync(ctx->dsc, in, sizeof(DevScalars), cudaMemcpyHostToDevice, ctx->st));
    std::memcpy((void*)ctx->hsc, in, sizeof(DevScalars));
    in += sizeof(DevScalars);
    for (auto& a : ck_arrays(ctx)) {
        CK(cudaMemcpyAsync(a.first, in, sizeof(double) * a.second, cudaMemcpyHostToDevice, ctx->st));
        in += sizeof(double) * a.second;
    }
    // the neighbour lists as they were built: from the build-time fractional
    // coordinates, so their pair order (and every sum over them) is unchanged
    if (hdr.have_list) {
        // the build-time cell (it differs from the current one under constant
        // pressure): the list's binning and distances as they were
        const CellP cur = ctx->cell;
        double W[3], an[3], Acur[9];
        std::memcpy(W, ctx->W, sizeof W);
        std::memcpy(an, ctx->anorm, sizeof an);
        std::memcpy(Acur, ctx->A_cur, sizeof Acur);
        const bool other = std::memcmp(hdr.npt.A_build, Acur, sizeof Acur) != 0 && hdr.npt.A_build[0] != 0.0;
        if (other) {
            lattice(hdr.npt.A_build, ctx->cell, ctx->W, ctx->anorm);
            std::memcpy(ctx->A_cur, hdr.npt.A_build, sizeof Acur);
        }
        CK(cudaMemcpyAsync(ctx->sx, ctx->xs, sizeof(double) * ctx->n, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->sy, ctx->ys, sizeof(double) * ctx->n, cudaMemcpyDeviceToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->sz, ctx->zs, sizeof(double) * ctx->n, cudaMemcpyDeviceToDevice, ctx->st));
        TRY(build_lists(ctx, ctx->p.lvnlist ? ctx->p.skindiff : 0.0, true));
        ctx->cell = cur;
        std::memcpy(ctx->W, W, sizeof W);
        std::memcpy(ctx->anorm, an, sizeof an);
        std::memcpy(ctx->A_cur, Acur, sizeof Acur);
        ctx->npt = hdr.npt;   // build_lists recorded its own scale and cell
    }
    launch_frac(ctx->st, ctx->n, ctx->x, ctx->y, ctx->z, ctx->cell, ctx->sx, ctx->sy, ctx->sz);
    TRY(check_launch(ctx, "checkpoint frac"));
    ctx->itime = hdr.itime;
    ctx->last_rebuilt = hdr.last_rebuilt;
    ctx->nrebuild = hdr.nrebuild;
    ctx->md_started = hdr.md_started != 0;
    ctx->forces_valid = hdr.forces_valid != 0;
    ctx->have_list = hdr.have_list != 0;
    ctx->tuned = hdr.tuned != 0;
    ctx->g_dir = hdr.g_dir;
    ctx->g_dd = hdr.g_dd;
    ctx->rs.p_mul = hdr.p_mul;
    ctx->rs.s_mul = hdr.s_mul;
    ctx->e_kin = hdr.e_kin;
    ctx->temp_r = hdr.temp_r;
    ctx->en = hdr.en;
    std::memcpy(ctx->tau_nonb, hdr.tau_nonb, sizeof hdr.tau_nonb);
    std::memcpy(ctx->tau_coul, hdr.tau_coul, sizeof hdr.tau_coul);
    ctx->rs.want_epoch++;
    ctx->rec_acc_ready = false;
    ctx->ddtab_epoch = -1;
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// g(r) and reverse Monte Carlo.
namespace {

__global__ void k_rmc_dirkar(int n, const double* __restrict__ s, CellP c, double* x, double* y, double* z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = s[i], b = s[(size_t)n + i], d = s[2 * (size_t)n + i];
    x[i] = __dadd_rn(__dadd_rn(__dmul_rn(a, c.A[0]), __dmul_rn(b, c.A[1])), __dmul_rn(d, c.A[2]));
    y[i] = __dadd_rn(__dadd_rn(__dmul_rn(a, c.A[3]), __dmul_rn(b, c.A[4])), __dmul_rn(d, c.A[5]));
    z[i] = __dadd_rn(__dadd_rn(__dmul_rn(a, c.A[6]), __dmul_rn(b, c.A[7])), __dmul_rn(d, c.A[8]));
}

// RmcConst of the context's system: nbins = INT(cut / res) + 1 (rmc_main,
// src/rmc.f90:329), the bin volumes of rmc_gr (src/rmc.f90:1469-1472)
int rmc_setup(mdff_ctx* ctx, double cut, double res, RmcConst& k) {
    if (!(cut > 0.0) || !(res > 0.0)) return fail(ctx, MDFF_E_ARG, "g(r): cut and resolution must be positive");
    if (ctx->ntype > RMC_NT_MAX) return fail(ctx, MDFF_E_UNSUPPORTED, "g(r): at most 4 types");
    const double nb = cut / res;
    if (!(nb < RMC_MAX_BINS - 1)) return fail(ctx, MDFF_E_UNSUPPORTED, "g(r): at most 4095 bins");
    std::memset(&k, 0, sizeof k);
    k.n = ctx->n;
    k.ntype = ctx->ntype;
    k.nbins = (int)nb + 1;
    k.nrow = 1 + k.ntype * k.ntype;
    k.npairs = k.ntype * (k.ntype + 1) / 2;
    k.bin.cut2 = cut * cut;
    k.bin.resg = res;
    k.bin.nbins = k.nbins;
    k.bin.ntype = k.ntype;
    k.natm = (double)ctx->n;
    for (int t = 0; t < k.ntype; ++t) k.natmi[t] = (double)ctx->natmi[t];
    const double pi4 = 4.0 * PI;
    for (int b = 0; b < k.nbins; ++b) {
        const double rr = ((double)b + 0.5) * res;
        double vol = pi4 * (res * rr * rr + (res * res * res) / 12.0);
        k.volnorm[b] = vol / ctx->cell.omega;
    }
    return MDFF_OK;
}

// fractional coordinates [3][n] of the context's positions (kardir)
int rmc_frac(mdff_ctx* ctx, double* s) {
    const int n = ctx->n;
    launch_frac(ctx->st, n, ctx->x, ctx->y, ctx->z, ctx->cell, s, s + n, s + 2 * (size_t)n);
    return check_launch(ctx, "rmc frac");
}

// normalised rows [npairs+1][nbins] of counts h [nrow][nbins] (rmc_gr)
void rmc_normalise(const RmcConst& k, const std::vector<int>& h, double* grr) {
    for (int b = 0; b < k.nbins; ++b) {
        grr[b] = (double)h[b] / (k.volnorm[b] * k.natm * k.natm);
        int mp = 1;
        for (int it1 = 0; it1 < k.ntype; ++it1)
            for (int it2 = it1; it2 < k.ntype; ++it2, ++mp)
                grr[(size_t)mp * k.nbins + b] =
                    (double)h[(size_t)(1 + it1 * k.ntype + it2) * k.nbins + b] / (k.volnorm[b] * k.natmi[it1] * k.natmi[it2]);
    }
}

}  // namespace

extern "C" {

int mdff_gr(mdff_ctx* ctx, double cut, double res, double* grr, int* nbins) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    cudaSetDevice(ctx->p.device);
    RmcConst k;
    TRY(rmc_setup(ctx, cut, res, k));
    if (nbins) *nbins = k.nbins;
    if (!grr) return MDFF_OK;
    const int n = ctx->n;
    double* s = nullptr;
    int* h = nullptr;
    CK(cudaMallocAsync((void**)&s, sizeof(double) * 3 * (size_t)n, ctx->st));
    CK(cudaMallocAsync((void**)&h, sizeof(int) * (size_t)k.nrow * k.nbins, ctx->st));
    CK(cudaMemsetAsync(h, 0, sizeof(int) * (size_t)k.nrow * k.nbins, ctx->st));
    TRY(rmc_frac(ctx, s));
    k_gr_full<<<nb(n), 256, 0, ctx->st>>>(n, s, ctx->type, ctx->cell, k.bin, h);
    TRY(check_launch(ctx, "gr"));
    std::vector<int> hh((size_t)k.nrow * k.nbins);
    CK(cudaMemcpyAsync(hh.data(), h, sizeof(int) * hh.size(), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaFreeAsync(s, ctx->st));
    CK(cudaFreeAsync(h, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    rmc_normalise(k, hh, grr);
    return MDFF_OK;
}

int mdff_rmc(mdff_ctx* ctx, const mdff_rmc_params* rp, const double* grr_exp, const double* uniforms, long long nuni,
             unsigned long long seed, double* grr_out, mdff_rmc_result* res) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!rp || !grr_exp) return fail(ctx, MDFF_E_ARG, "mdff_rmc: parameters and the experimental g(r) are required");
    if (rp->max_trials < 1 || rp->acceptance_max < 1) return fail(ctx, MDFF_E_ARG, "mdff_rmc: trial bounds");
    for (int q = 0; q < 6; ++q)
        if (!(rp->temp_rmc[q] > 0.0)) return fail(ctx, MDFF_E_ARG, "mdff_rmc: temperatures must be positive");
    if (!uniforms && rp->max_trials > 100000000LL) return fail(ctx, MDFF_E_ARG, "mdff_rmc: at most 1e8 trials per call");
    if (!(rp->max_displacement > 0.0 && 3.0 * rp->max_displacement < 1.0))
        return fail(ctx, MDFF_E_ARG, "mdff_rmc: max_displacement must be in (0, 0.33) A");
    cudaSetDevice(ctx->p.device);
    auto* k = new RmcConst;
    std::unique_ptr<RmcConst> kguard(k);
    TRY(rmc_setup(ctx, rp->cut_rmc, rp->resolution_gr, *k));
    for (int d = 0; d < 3; ++d) k->dmax[d] = rp->max_displacement / ctx->anorm[d];
    for (int q = 0; q < 6; ++q) k->temp[q] = rp->temp_rmc[q];
    const size_t ncount = (size_t)k->nrow * k->nbins;
    if (ncount * sizeof(int) > 200 * 1024) return fail(ctx, MDFF_E_UNSUPPORTED, "mdff_rmc: too many g(r) bins x types");
    const int n = ctx->n;
    const long long nu = uniforms ? nuni : 10 * rp->max_trials;
    double *s = nullptr, *gexp = nullptr, *uni = nullptr;
    int* h = nullptr;
    RmcConst* kd = nullptr;
    RmcOut* out = nullptr;
    CK(cudaMallocAsync((void**)&s, sizeof(double) * 3 * (size_t)n, ctx->st));
    CK(cudaMallocAsync((void**)&h, sizeof(int) * ncount, ctx->st));
    CK(cudaMallocAsync((void**)&gexp, sizeof(double) * (size_t)(k->npairs + 1) * k->nbins, ctx->st));
    CK(cudaMallocAsync((void**)&uni, sizeof(double) * (size_t)std::max(1LL, nu), ctx->st));
    CK(cudaMallocAsync((void**)&kd, sizeof(RmcConst), ctx->st));
    CK(cudaMallocAsync((void**)&out, sizeof(RmcOut), ctx->st));
    CK(cudaMemcpyAsync(kd, k, sizeof(RmcConst), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(gexp, grr_exp, sizeof(double) * (size_t)(k->npairs + 1) * k->nbins, cudaMemcpyHostToDevice,
                       ctx->st));
    if (uniforms) CK(cudaMemcpyAsync(uni, uniforms, sizeof(double) * (size_t)nu, cudaMemcpyHostToDevice, ctx->st));
    else k_rmc_uniforms<<<(unsigned)((nu + 255) / 256), 256, 0, ctx->st>>>(nu, seed, uni);
    CK(cudaMemsetAsync(h, 0, sizeof(int) * ncount, ctx->st));
    TRY(rmc_frac(ctx, s));
    k_gr_full<<<nb(n), 256, 0, ctx->st>>>(n, s, ctx->type, ctx->cell, k->bin, h);
    TRY(check_launch(ctx, "rmc start"));
    const int smem = (int)(ncount * sizeof(int));
    CK(cudaFuncSetAttribute(k_rmc_chain, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // neighbour lists of the chain: every atom within cut + skin; while no
    // atom has moved more than (skin - 3 max_displacement) / 2 from the
    // list's positions, a pair outside the list stays beyond cut at both ends
    // of any trial move.  When cut + skin reaches half the cell, the list
    // holds every atom and never expires.
    const double skin = 1.0;
    const double wmin = std::min(ctx->W[0], std::min(ctx->W[1], ctx->W[2]));
    const bool all_pairs = 2.0 * (rp->cut_rmc + skin) >= wmin;
    const double rl = all_pairs ? 1e300 : rp->cut_rmc + skin;
    const double dlim = all_pairs ? 1e300 : 0.5 * (skin - 3.0 * rp->max_displacement);
    int cap = all_pairs ? std::max(1, n - 1)
                        : (int)std::min<double>(n - 1, 1.3 * 4.0 / 3.0 * PI * rl * rl * rl * n / ctx->cell.omega + 64);
    int *nbr = nullptr, *ncnt = nullptr, *ovf = nullptr;
    double* sb = nullptr;
    CK(cudaMallocAsync((void**)&ncnt, sizeof(int) * (size_t)n, ctx->st));
    CK(cudaMallocAsync((void**)&ovf, sizeof(int), ctx->st));
    CK(cudaMallocAsync((void**)&sb, sizeof(double) * 3 * (size_t)n, ctx->st));
    CK(cudaMemsetAsync(out, 0, sizeof(RmcOut), ctx->st));
    int nbuild = 0;
    for (int launch = 0;; ++launch) {
        for (int attempt = 0;; ++attempt) {   // build, growing the capacity if needed
            if (!nbr) CK(cudaMallocAsync((void**)&nbr, sizeof(int) * (size_t)n * cap, ctx->st));
            CK(cudaMemsetAsync(ovf, 0, sizeof(int), ctx->st));
            k_rmc_list<<<nb(n), 256, 0, ctx->st>>>(n, s, ctx->cell, rl * rl, cap, nbr, ncnt, ovf);
            TRY(check_launch(ctx, "rmc list"));
            int ho_ovf = 0;
            CK(cudaMemcpyAsync(&ho_ovf, ovf, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
            CK(cudaStreamSynchronize(ctx->st));
            if (ho_ovf <= cap) break;
            if (attempt > 3) return fail(ctx, MDFF_E_LISTOVF, "mdff_rmc: neighbour list capacity");
            CK(cudaFreeAsync(nbr, ctx->st));
            nbr = nullptr;
            cap = std::min(n - 1, (int)(ho_ovf * 1.2) + 32);
        }
        ++nbuild;
        CK(cudaMemcpyAsync(sb, s, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, ctx->st));
        k_rmc_chain<<<1, RMC_THREADS, smem, ctx->st>>>(s, ctx->type, ctx->cell, kd, h, gexp, uni, nu,
                                                       rp->acceptance_max, rp->max_trials, nbr, ncnt, cap, sb, dlim,
                                                       out);
        TRY(check_launch(ctx, "rmc chain"));
        RmcOut st;
        CK(cudaMemcpyAsync(&st, out, sizeof st, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        if (st.status != 2) break;
        st.status = 0;
        st.maxd = 0.0;
        CK(cudaMemcpyAsync(out, &st, sizeof st, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    (void)nbuild;
    for (void* q : {(void*)nbr, (void*)ncnt, (void*)ovf, (void*)sb}) CK(cudaFreeAsync(q, ctx->st));
    k_rmc_dirkar<<<nb(n), 256, 0, ctx->st>>>(n, s, ctx->cell, ctx->x, ctx->y, ctx->z);
    RmcOut ho;
    std::vector<int> hh(ncount);
    CK(cudaMemcpyAsync(&ho, out, sizeof ho, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(hh.data(), h, sizeof(int) * ncount, cudaMemcpyDeviceToHost, ctx->st));
    for (void* p : {(void*)s, (void*)h, (void*)gexp, (void*)uni, (void*)kd, (void*)out}) CK(cudaFreeAsync(p, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    TRY(check_launch(ctx, "rmc"));
    ctx->forces_valid = false;
    if (ctx->p.lvnlist) TRY(build_lists(ctx, ctx->p.skindiff));
    if (grr_out) rmc_normalise(*k, hh, grr_out);
    if (res) {
        res->kall = ho.kall;
        res->kacc = ho.kacc;
        res->uniforms_used = ho.used;
        for (int q = 0; q < 6; ++q) res->chisq[q] = ho.chisq[q];
        res->status = ho.status;
        res->pad = 0;
    }
    CK(cudaStreamSynchronize(ctx->st));
    return MDFF_OK;
}

}  // extern "C"

namespace {

// eval_chisq_rmc's g(r) term by the fixed tree of the device chain: the
// squares of the terms q = bin x (npairs + 1) + mp in 1024 strided partial
// sums, a halving tree over each group of 32, the same tree over the groups
double rmc_chisq_gr_tree(const RmcConst& k, const double* calc, const double* gexp) {
    const int nterm = (k.npairs + 1) * k.nbins;
    std::vector<double> part(1024, 0.0);
    for (int q = 0; q < nterm; ++q) {
        const int b = q / (k.npairs + 1), mp = q - b * (k.npairs + 1);
        const double d = calc[(size_t)mp * k.nbins + b] - gexp[(size_t)mp * k.nbins + b];
        part[q % 1024] = part[q % 1024] + d * d;
    }
    auto tree32 = [](double* v) {
        for (int o = 16; o > 0; o >>= 1)
            for (int l = 0; l < o; ++l) v[l] = v[l] + v[l + o];
        return v[0];
    };
    double w[32];
    for (int g = 0; g < 32; ++g) w[g] = tree32(&part[32 * g]);
    return tree32(w);
}

// rmc_efg's normalisation (src/rmc.f90:1620-1650) and eval_chisq_Uefg /
// eval_chisq_vzz / eval_chisq_eta (:693-769), left to right in the
// reference's loop order.  Layouts are the reference's Fortran ones:
// U (ui, mp, bin) at (bin (ntype+1) + mp) 6 + ui - 1, vzz and eta (mp, bin)
// at bin (ntype+1) + mp.  Quirks kept: the per-type U rows divide the
// all-types U1 counts; eta's last bin is never normalised (it stays 0).
struct RmcEfgHost {
    int nt1, PANU, PANvzz, PANeta;
    double natm, resu, resvzz, reseta;
    std::vector<double> natmi;
};

void rmc_efg_normalise(const RmcEfgHost& e, const int* cnt, int offeta, int offU, bool lu, double* U, double* vzz,
                       double* eta) {
    const int wv = e.PANvzz + 1, we = e.PANeta + 1, wu = e.PANU + 1;
    if (lu)
        for (int bin = 0; bin <= e.PANU; ++bin)
            for (int ui = 1; ui <= 5; ++ui) {
                U[((size_t)bin * e.nt1 + 0) * 6 + ui - 1] =
                    (double)cnt[offU + ((ui - 1) * e.nt1 + 0) * wu + bin] / (e.resu * e.natm);
                for (int it = 1; it < e.nt1; ++it)
                    U[((size_t)bin * e.nt1 + it) * 6 + ui - 1] =
                        (double)cnt[offU + (0 * e.nt1 + 0) * wu + bin] / (e.resu * e.natmi[it - 1]);
            }
    for (int bin = 0; bin < e.PANeta; ++bin) {
        eta[(size_t)bin * e.nt1] = (double)cnt[offeta + bin] / (e.reseta * e.natm);
        for (int it = 1; it < e.nt1; ++it)
            eta[(size_t)bin * e.nt1 + it] = (double)cnt[offeta + it * we + bin] / (e.reseta * e.natmi[it - 1]);
    }
    for (int it = 0; it < e.nt1; ++it) eta[(size_t)e.PANeta * e.nt1 + it] = 0.0;
    for (int bin = 0; bin <= e.PANvzz; ++bin) {
        vzz[(size_t)bin * e.nt1] = (double)cnt[bin] / (e.resvzz * e.natm);
        for (int it = 1; it < e.nt1; ++it)
            vzz[(size_t)bin * e.nt1 + it] = (double)cnt[it * wv + bin] / (e.resvzz * e.natmi[it - 1]);
    }
}

}  // namespace

extern "C" {

int mdff_rmc_efg(mdff_ctx* ctx, const mdff_rmc_params* rp, const mdff_rmc_efg_params* ep, const double* grr_exp,
                 const double* dibU_exp, const double* dibvzz_exp, const double* dibeta_exp, const double* uniforms,
                 long long nuni, unsigned long long seed, double* grr_out, double* dibU_out, double* dibvzz_out,
                 double* dibeta_out, mdff_rmc_result* res) {
    if (!ctx || !ctx->have_system) return ctx ? fail(ctx, MDFF_E_STATE, "set_system first") : MDFF_E_STATE;
    if (!rp || !ep || !grr_exp) return fail(ctx, MDFF_E_ARG, "mdff_rmc_efg: parameters and the experimental g(r)");
    if (rp->max_trials < 1 || rp->acceptance_max < 1) return fail(ctx, MDFF_E_ARG, "mdff_rmc_efg: trial bounds");
    for (int q = 0; q < 6; ++q)
        if (!(rp->temp_rmc[q] > 0.0)) return fail(ctx, MDFF_E_ARG, "mdff_rmc_efg: temperatures must be positive");
    if (!(rp->max_displacement > 0.0 && 3.0 * rp->max_displacement < 1.0))
        return fail(ctx, MDFF_E_ARG, "mdff_rmc_efg: max_displacement must be in (0, 0.33) A");
    if (!(ep->resolution_vzz_efg > 0.0 && ep->resolution_eta_efg > 0.0 && ep->resolution_u_efg > 0.0))
        return fail(ctx, MDFF_E_ARG, "mdff_rmc_efg: EFG resolutions must be positive");
    if ((ep->lrmc_u && !dibU_exp) || (ep->lrmc_vzz && !dibvzz_exp) || (ep->lrmc_eta && !dibeta_exp))
        return fail(ctx, MDFF_E_ARG, "mdff_rmc_efg: an experimental distribution of an active term is missing");
    const bool any_efg_req = ep->lrmc_u || ep->lrmc_vzz || ep->lrmc_eta;
    if (any_efg_req && (!ctx->p.lcoulomb || ctx->npol > 0 || ctx->any_dip0))
        return fail(ctx, MDFF_E_UNSUPPORTED, "mdff_rmc_efg: the EFG terms take point charges (no dipoles), as "
                                             "rmc_efg's multipole_efg_ES is called with mu = 0");
    const double pu = 2.0 * std::fabs(ep->u_efg_min) / ep->resolution_u_efg;
    const double pv = 2.0 * std::fabs(ep->vzz_efg_min) / ep->resolution_vzz_efg;
    const double pe = 1.0 / ep->resolution_eta_efg;
    if (!(pu < 1e6 && pv < 1e6 && pe < 1e6)) return fail(ctx, MDFF_E_UNSUPPORTED, "mdff_rmc_efg: at most 1e6 bins");
    cudaSetDevice(ctx->p.device);
    auto* k = new RmcConst;
    std::unique_ptr<RmcConst> kguard(k);
    TRY(rmc_setup(ctx, rp->cut_rmc, rp->resolution_gr, *k));
    const int n = ctx->n, nt1 = ctx->ntype + 1;
    RmcEfgHost eh;
    eh.nt1 = nt1;
    eh.PANU = (int)pu;
    eh.PANvzz = (int)pv;
    eh.PANeta = (int)pe;
    eh.natm = (double)n;
    eh.resu = ep->resolution_u_efg;
    eh.resvzz = ep->resolution_vzz_efg;
    eh.reseta = ep->resolution_eta_efg;
    for (int t = 0; t < ctx->ntype; ++t) eh.natmi.push_back((double)ctx->natmi[t]);
    RmcEfgSpec sp;
    sp.ntype = ctx->ntype;
    sp.PANU = ep->lrmc_u ? eh.PANU : -1;
    sp.PANvzz = eh.PANvzz;
    sp.PANeta = eh.PANeta;
    sp.offeta = nt1 * (eh.PANvzz + 1);
    sp.offU = sp.offeta + nt1 * (eh.PANeta + 1);
    sp.cu = ctx->u.coul;
    sp.umin = ep->u_efg_min;
    sp.resu = ep->resolution_u_efg;
    sp.vzzmin = ep->vzz_efg_min;
    sp.resvzz = ep->resolution_vzz_efg;
    sp.reseta = ep->resolution_eta_efg;
    sp.sq3 = 1.0 / std::sqrt(3.0);
    sp.sq32 = sp.sq3 * 0.5;
    const size_t ncnt = (size_t)sp.offU + (size_t)6 * nt1 * (eh.PANU + 1);
    const size_t nU = (size_t)(eh.PANU + 1) * nt1 * 6, nV = (size_t)(eh.PANvzz + 1) * nt1,
                 nE = (size_t)(eh.PANeta + 1) * nt1;
    const size_t ngr = (size_t)k->nrow * k->nbins, ncalc = (size_t)(k->npairs + 1) * k->nbins;
    const bool any_efg = any_efg_req;
    // the distance-variance term: sorted distance lists of every atom
    const bool var = ep->lrmc_var != 0;
    VarSpec vs;
    std::memset(&vs, 0, sizeof vs);
    int varP = 1;
    if (var) {
        vs.n = n;
        vs.ntype = ctx->ntype;
        for (int t = 0; t < ctx->ntype; ++t) {
            vs.off[t] = vs.Ltot;
            vs.natmi[t] = ctx->natmi[t];
            vs.Ltot += ctx->natmi[t];
            vs.nmax = std::max(vs.nmax, ctx->natmi[t]);
        }
        int maxlen = 0;
        for (int t = 0; t < ctx->ntype; ++t)
            for (int ti = 0; ti < ctx->ntype; ++ti)
                if (ctx->natmi[ti] > 0) maxlen = std::max(maxlen, ctx->natmi[t] - (t == ti ? 1 : 0));
        if (maxlen > VAR_MAXSEG)
            return fail(ctx, MDFF_E_UNSUPPORTED, "mdff_rmc_efg: the variance term sorts at most " +
                                                     std::to_string(VAR_MAXSEG) + " distances per atom and type");
        while (varP < maxlen) varP <<= 1;
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        const size_t need = sizeof(double) * ((size_t)n * vs.Ltot + (size_t)ctx->ntype * ctx->ntype * vs.nmax +
                                              (size_t)VAR_NCH * ctx->ntype * vs.Ltot);
        if (need + ((size_t)1 << 29) > fr)
            return fail(ctx, MDFF_E_UNSUPPORTED, "mdff_rmc_efg: the variance term's distance lists need " +
                                                     std::to_string(need >> 20) + " MiB of device memory, " +
                                                     std::to_string(fr >> 20) + " MiB are free");
        CK(cudaFuncSetAttribute(k_var_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(varP * sizeof(double))));
    }
    // uniforms: the caller's, or the counter-based stream of mdff_rmc
    std::vector<double> uni;
    const long long nu = uniforms ? nuni : 10 * rp->max_trials;
    if (!uniforms) {
        if (rp->max_trials > 10000000LL) return fail(ctx, MDFF_E_ARG, "mdff_rmc_efg: at most 1e7 trials per call");
        uni.resize((size_t)nu);
        for (long long t = 0; t < nu; ++t) {
            unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(t + 1);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z = z ^ (z >> 31);
            uni[(size_t)t] = (double)(z >> 11) * (1.0 / 9007199254740992.0);
        }
    }
    const double* U_ = uniforms ? uniforms : uni.data();
    // device scratch: fractional coordinates, g(r) counts and their change, EFG counts
    double* s = nullptr;
    int *hd = nullptr, *dh = nullptr, *ce = nullptr;
    CK(cudaMallocAsync((void**)&s, sizeof(double) * 3 * (size_t)n, ctx->st));
    CK(cudaMallocAsync((void**)&hd, sizeof(int) * ngr, ctx->st));
    CK(cudaMallocAsync((void**)&dh, sizeof(int) * ngr, ctx->st));
    CK(cudaMallocAsync((void**)&ce, sizeof(int) * ncnt, ctx->st));
    CK(cudaMemsetAsync(hd, 0, sizeof(int) * ngr, ctx->st));
    TRY(rmc_frac(ctx, s));
    k_rmc_dirkar<<<nb(n), 256, 0, ctx->st>>>(n, s, ctx->cell, ctx->x, ctx->y, ctx->z);
    k_gr_full<<<nb(n), 256, 0, ctx->st>>>(n, s, ctx->type, ctx->cell, k->bin, hd);
    double *vl = nullptr, *vmean = nullptr, *vpart = nullptr, *vpsum = nullptr;
    int *vrank = nullptr, *verr = nullptr;
    const int vwb = (n * 32 + 255) / 256;   // blocks of the per-atom chi kernel (a warp per atom)
    if (var) {
        CK(cudaMallocAsync((void**)&vl, sizeof(double) * (size_t)n * vs.Ltot, ctx->st));
        CK(cudaMallocAsync((void**)&vmean, sizeof(double) * (size_t)vs.ntype * vs.ntype * vs.nmax, ctx->st));
        CK(cudaMallocAsync((void**)&vpsum, sizeof(double) * (size_t)VAR_NCH * vs.ntype * vs.Ltot, ctx->st));
        CK(cudaMallocAsync((void**)&vpart, sizeof(double) * (size_t)(vwb + 1), ctx->st));
        CK(cudaMallocAsync((void**)&vrank, sizeof(int) * (size_t)n, ctx->st));
        CK(cudaMallocAsync((void**)&verr, sizeof(int), ctx->st));
        std::vector<int> ht(n), rank(n), cntt(NT, 0);
        CK(cudaMemcpyAsync(ht.data(), ctx->type, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        for (int a = 0; a < n; ++a) rank[a] = cntt[ht[a]]++;
        CK(cudaMemcpyAsync(vrank, rank.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemsetAsync(verr, 0, sizeof(int), ctx->st));
        k_var_fill<<<dim3((n + 255) / 256, n), 256, 0, ctx->st>>>(vs, s, ctx->type, vrank, ctx->cell, vl);
        k_var_sort<<<n * vs.ntype, 1024, varP * sizeof(double), ctx->st>>>(vs, ctx->type, 0, -1, varP, vl);
        CK(cudaStreamSynchronize(ctx->st));   // rank goes out of scope
        TRY(check_launch(ctx, "rmc variance lists"));
    }
    // chi^2 of the variance term from the lists (launches; *res written on the device)
    auto var_launch = [&](double* dres) {
        k_var_mean<<<dim3(nb(n), VAR_NCH), 256, 0, ctx->st>>>(vs, ctx->type, vl, vpsum);
        k_var_mean_fin<<<nb(n), 256, 0, ctx->st>>>(vs, vpsum, vmean);
        k_var_chi<<<vwb, 256, 0, ctx->st>>>(vs, ctx->type, vl, vmean, vpart);
        launch_reduce_partials(ctx->st, vpart, vwb, 1, dres, 0);
    };
    // p moved from direct position f to t: p's own lists again, and the one
    // changed value in every other atom's list
    auto var_move = [&](int p, const double f[3], const double t[3]) {
        k_var_row<<<nb(n), 256, 0, ctx->st>>>(vs, s, ctx->type, vrank, ctx->cell, p, vl);
        k_var_sort<<<vs.ntype, 1024, varP * sizeof(double), ctx->st>>>(vs, ctx->type, 0, p, varP, vl);
        k_var_shift<<<(n * 32 + 255) / 256, 256, 0, ctx->st>>>(vs, s, ctx->type, ctx->cell, p, f[0], f[1], f[2], t[0],
                                                               t[1], t[2], vl, verr);
    };
    std::vector<int> h(ngr), hdel(ngr), htr(ngr), cnt(ncnt);
    std::vector<double> sh(3 * (size_t)n);
    CK(cudaMemcpyAsync(h.data(), hd, sizeof(int) * ngr, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(sh.data(), s, sizeof(double) * sh.size(), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    TRY(check_launch(ctx, "rmc_efg start"));
    // the chain needs the EFG alone: the short-range pair terms are switched
    // off for its evaluations (and their lists for its rebuilds), then restored
    const int saved_doefg = ctx->p.doefg;
    const int saved_nonb[4] = {ctx->p.lnmlj, ctx->p.lbmhft, ctx->p.lbmhftd, ctx->p.lmorse};
    ctx->p.doefg = 1;
    ctx->p.lnmlj = ctx->p.lbmhft = ctx->p.lbmhftd = ctx->p.lmorse = 0;
    std::vector<double> calc(ncalc), cU(nU, 0.0), cV(nV, 0.0), cE(nE, 0.0), aU(nU, 0.0), aV(nV, 0.0), aE(nE, 0.0);
    // Verlet-list validity: an atom's summed trial displacements since the
    // last build stay below half the skin
    const bool lists = ctx->p.lvnlist != 0;
    const double half_skin = 0.5 * ctx->p.skindiff;
    std::vector<double> moved(lists ? (size_t)n : 0, 0.0);
    auto efg_terms = [&](double chi[6]) -> int {
        TRY(engforce_device(ctx));
        CK(cudaMemsetAsync(ce, 0, sizeof(int) * ncnt, ctx->st));
        k_rmc_efg_hist<<<nb(n), 256, 0, ctx->st>>>(n, ctx->efg, ctx->type, sp, ce);
        CK(cudaMemcpyAsync(cnt.data(), ce, sizeof(int) * ncnt, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        TRY(check_launch(ctx, "rmc_efg histograms"));
        rmc_efg_normalise(eh, cnt.data(), sp.offeta, sp.offU, ep->lrmc_u != 0, cU.data(), cV.data(), cE.data());
        if (ep->lrmc_u) {
            double c = 0.0;
            for (int bin = 0; bin <= eh.PANU; ++bin)
                for (int mp = 0; mp < nt1; ++mp)
                    for (int ui = 0; ui < 5; ++ui) {
                        const size_t q = ((size_t)bin * nt1 + mp) * 6 + ui;
                        const double d = cU[q] - dibU_exp[q];
                        c = c + d * d;
                    }
            chi[2] = c;
        }
        if (ep->lrmc_vzz) {
            double c = 0.0;
            for (int bin = 0; bin <= eh.PANvzz; ++bin)
                for (int mp = 0; mp < nt1; ++mp) {
                    const double d = cV[(size_t)bin * nt1 + mp] - dibvzz_exp[(size_t)bin * nt1 + mp];
                    c = c + d * d;
                }
            chi[3] = c;
        }
        if (ep->lrmc_eta) {
            double c = 0.0;
            for (int bin = 0; bin <= eh.PANeta; ++bin)
                for (int mp = 0; mp < nt1; ++mp) {
                    const double d = cE[(size_t)bin * nt1 + mp] - dibeta_exp[(size_t)bin * nt1 + mp];
                    c = c + d * d;
                }
            chi[4] = c;
        }
        return MDFF_OK;
    };
    auto total = [](double chi[6]) { chi[5] = (((chi[0] + chi[1]) + chi[2]) + chi[3]) + chi[4]; };
    int rc = MDFF_OK;
#define CK_R(call)                                                                             \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            rc = fail(ctx, MDFF_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
            return;                                                                            \
        }                                                                                      \
    } while (0)
    long long kall = 1, kacc = 1, u = 0;
    int status = 0;
    double chi_old[6] = {0, 0, 0, 0, 0, 0}, chi[6];
    double var_h = 0.0;
    [&]() {
        rmc_normalise(*k, h, calc.data());
        chi_old[0] = rmc_chisq_gr_tree(*k, calc.data(), grr_exp);
        if (var) {
            var_launch(vpart + vwb);
            CK_R(cudaMemcpyAsync(&var_h, vpart + vwb, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
            CK_R(cudaStreamSynchronize(ctx->st));
            chi_old[1] = var_h;
        }
        if (any_efg && kacc >= ep->efg_start) {
            if ((rc = efg_terms(chi_old)) != MDFF_OK) return;
            aU = cU; aV = cV; aE = cE;
        }
        total(chi_old);
        const double dmax[3] = {rp->max_displacement / ctx->anorm[0], rp->max_displacement / ctx->anorm[1],
                                rp->max_displacement / ctx->anorm[2]};
        while (kacc < rp->acceptance_max && kall < rp->max_trials) {
            ++kall;
            if (u + 4 > nu) { status = 1; --kall; break; }
            int p = (int)(U_[u] * n);   // rmc_move (src/rmc.f90:1371-1424)
            if (p >= n) p = n - 1;
            double disp[3], snew[3], sold[3];
            for (int d = 0; d < 3; ++d) {
                disp[d] = dmax[d] * (2.0 * U_[u + 1 + d] - 1.0);
                sold[d] = sh[(size_t)d * n + p];
                double v = sold[d] + disp[d];
                if (v > 1.0 || v < 0.0) v = v - std::round(v);   // NINT: half away from zero
                snew[d] = v;
            }
            u += 4;
            if (lists) {
                double dc[3];
                for (int a = 0; a < 3; ++a)
                    dc[a] = ctx->cell.A[3 * a] * disp[0] + ctx->cell.A[3 * a + 1] * disp[1] + ctx->cell.A[3 * a + 2] * disp[2];
                const double step = std::sqrt(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]) + 1e-9;
                if (moved[p] + step > half_skin) {
                    if ((rc = build_lists(ctx, ctx->p.skindiff)) != MDFF_OK) return;
                    std::fill(moved.begin(), moved.end(), 0.0);
                }
                moved[p] += step;
            }
            for (int d = 0; d < 3; ++d) sh[(size_t)d * n + p] = snew[d];
            k_rmc_place<<<1, 1, 0, ctx->st>>>(n, s, p, snew[0], snew[1], snew[2], ctx->cell, ctx->x, ctx->y, ctx->z);
            CK_R(cudaMemsetAsync(dh, 0, sizeof(int) * ngr, ctx->st));
            k_rmc_grdelta<<<nb(n), 256, 0, ctx->st>>>(n, s, ctx->type, ctx->cell, k->bin, p, sold[0], sold[1],
                                                       sold[2], dh);
            CK_R(cudaMemcpyAsync(hdel.data(), dh, sizeof(int) * ngr, cudaMemcpyDeviceToHost, ctx->st));
            if (var) {
                var_move(p, sold, snew);
                var_launch(vpart + vwb);
                CK_R(cudaMemcpyAsync(&var_h, vpart + vwb, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
            }
            for (int q = 0; q < 6; ++q) chi[q] = 0.0;
            const bool efg_now = any_efg && kacc >= ep->efg_start;
            if (efg_now) {
                if ((rc = efg_terms(chi)) != MDFF_OK) return;
            } else {
                CK_R(cudaStreamSynchronize(ctx->st));
            }
            for (size_t q = 0; q < ngr; ++q) htr[q] = h[q] + hdel[q];
            rmc_normalise(*k, htr, calc.data());
            chi[0] = rmc_chisq_gr_tree(*k, calc.data(), grr_exp);
            if (var) chi[1] = var_h;
            total(chi);
            bool acc6 = false, stop = false;
            for (int q = 0; q < 6; ++q) {   // src/rmc.f90:521-540
                const double dq = chi[q] - chi_old[q];
                bool a;
                if (dq < 0.0) a = true;
                else {
                    if (u + 1 > nu) { stop = true; break; }
                    const double metro = std::exp(-(dq * 0.5) / rp->temp_rmc[q]);
                    a = metro >= U_[u];
                    ++u;
                }
                if (q == 5) acc6 = a;
            }
            if (stop || !acc6) {   // back to snew - disp (src/rmc.f90:628-636); sold when the uniforms ran out
                double back[3];
                for (int d = 0; d < 3; ++d) {
                    back[d] = stop ? sold[d] : snew[d] - disp[d];
                    sh[(size_t)d * n + p] = back[d];
                }
                k_rmc_place<<<1, 1, 0, ctx->st>>>(n, s, p, back[0], back[1], back[2], ctx->cell, ctx->x, ctx->y,
                                                  ctx->z);
                if (var) var_move(p, snew, back);
                if (stop) { status = 1; --kall; break; }
            } else {
                ++kacc;
                for (int q = 0; q < 6; ++q) chi_old[q] = chi[q];
                h = htr;
                if (efg_now) { aU = cU; aV = cV; aE = cE; }
            }
        }
    }();
#undef CK_R
    ctx->p.doefg = saved_doefg;
    ctx->p.lnmlj = saved_nonb[0];
    ctx->p.lbmhft = saved_nonb[1];
    ctx->p.lbmhftd = saved_nonb[2];
    ctx->p.lmorse = saved_nonb[3];
    int var_err = 0;
    if (var) {
        if (cudaMemcpyAsync(&var_err, verr, sizeof(int), cudaMemcpyDeviceToHost, ctx->st) != cudaSuccess) var_err = 2;
        for (void* q : {(void*)vl, (void*)vmean, (void*)vpart, (void*)vrank, (void*)verr, (void*)vpsum})
            cudaFreeAsync(q, ctx->st);
    }
    for (void* q : {(void*)s, (void*)hd, (void*)dh, (void*)ce}) cudaFreeAsync(q, ctx->st);
    cudaStreamSynchronize(ctx->st);
    if (rc == MDFF_OK && var_err)
        rc = fail(ctx, MDFF_E_STATE, "mdff_rmc_efg: the variance term's distance lists lost step with the positions");
    // lists rebuilt during the chain cover the Coulomb cut only: never leave
    // them in place, on the error path either (a failed rebuild here leaves
    // have_list false, so the next evaluation builds them)
    ctx->forces_valid = false;
    ctx->have_list = false;
    if (rc != MDFF_OK) {
        if (ctx->p.lvnlist) build_lists(ctx, ctx->p.skindiff);
        return rc;
    }
    TRY(check_launch(ctx, "rmc_efg"));
    if (ctx->p.lvnlist) TRY(build_lists(ctx, ctx->p.skindiff));
    if (grr_out) rmc_normalise(*k, h, grr_out);
    if (dibU_out) std::memcpy(dibU_out, aU.data(), sizeof(double) * nU);
    if (dibvzz_out) std::memcpy(dibvzz_out, aV.data(), sizeof(double) * nV);
    if (dibeta_out) std::memcpy(dibeta_out, aE.data(), sizeof(double) * nE);
    if (res) {
        res->kall = kall;
        res->kacc = kacc;
        res->uniforms_used = u;
        for (int q = 0; q < 6; ++q) res->chisq[q] = chi_old[q];
        res->status = status;
        res->pad = 0;
    }
    return MDFF_OK;
}

}  // extern "C"
