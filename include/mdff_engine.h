/*
 * mdff_engine.h -- C ABI of the B200 force engine for the MDFF force and
 * integration hot path.
 *
 * The reference (MDFF, Fortran 90 + MPI) has no argument-passing interface on
 * this path: engforce_driver (src/field.f90:1111) and the integrators
 * (src/integration.f90:131,476) read and write module globals.  Every entry
 * point below replaces one of those routines; the comment on each names the
 * reference routine and file:line it stands in for.  A Fortran caller binds
 * these with iso_c_binding (fortran/mdff_engine.f90); Python binds them with
 * ctypes (mdff_b200/abi.py).
 *
 * Conventions
 *   - Arrays are structure-of-arrays FP64, one array per Cartesian component,
 *     exactly like rx(natm), ry(natm), rz(natm) in src/config.f90:44-89.
 *   - Atom types and neighbour-list indices are 1-based, as in the reference.
 *   - The cell matrix A[9] is column-major (Fortran order): A[3*j+i] is
 *     component i of basis vector j, i.e. simu_cell%A(i+1,j+1).
 *   - Per-type tables in mdff_params are indexed [i][j] for the reference's
 *     (i+1,j+1); the 3-index damping tables [p][i][j] for (p+1,i+1,j+1).
 *   - Input units are the control-file units of the reference: lengths in
 *     Angstrom, energies in eV, masses in amu, charges in e, dt and
 *     timesca_thermo in ps, temp in K (src/md.f90:314-324 conversions are done
 *     inside the engine).  With lreduced != 0 every unit factor is 1
 *     (src/constants.f90:135-146).
 *   - Every call returns 0 on success or a negative MDFF_E_* code; the message
 *     is available from mdff_last_error().  The library never exits or traps.
 *   - One context per host thread; a context owns one CUDA stream and all its
 *     device buffers.  No caller pointer is retained past a call.
 */
#ifndef MDFF_ENGINE_H
#define MDFF_ENGINE_H

#ifdef __cplusplus
extern "C" {
#endif

#define MDFF_NTYPE_MAX 16          /* ntypemax, src/config.f90:40 */
#define MDFF_TT_MAX_ORDER 8        /* maximum_of_TT_expansion, src/tt_damp.f90:8 */

/* status codes */
#define MDFF_OK            0
#define MDFF_E_ARG        -1       /* invalid argument / parameter */
#define MDFF_E_CUDA       -2       /* CUDA runtime error */
#define MDFF_E_NOCONV     -3       /* induced-dipole solve did not converge */
#define MDFF_E_LISTOVF    -4       /* neighbour list capacity exceeded (host regrows and retries) */
#define MDFF_E_NONFINITE  -5       /* NaN/Inf in energies or forces */
#define MDFF_E_STATE      -6       /* call out of order (e.g. step before set_system) */
#define MDFF_E_UNSUPPORTED -7      /* feature outside the engine's scope */
#define MDFF_E_NOMEM      -8       /* device allocation failed */

/* ctrunc (src/field.f90:54-58) */
#define MDFF_TRUNC_NONE      0
#define MDFF_TRUNC_LINEAR    1
#define MDFF_TRUNC_QUADRATIC 2

/* algo_moment_from_pola (src/field.f90:150-152) */
#define MDFF_POLA_SCF 0            /* reference fixed-point iteration */
#define MDFF_POLA_PCG 1            /* preconditioned conjugate gradient (new) */

/* algo_ext_dipole (src/field.f90:146-148) */
#define MDFF_EXT_POLY 0
#define MDFF_EXT_ASPC 1

/* integrator (src/md.f90:71-76): the ones on the hot path */
#define MDFF_NVE_VV   0
#define MDFF_NVT_NHCN 1
#define MDFF_NPT_NHCNP 2           /* isotropic Martyna-Tobias-Klein barostat with Nose-Hoover chains on
                                      particles and barostat (nhcnp, src/integration.f90:715-1160) */
#define MDFF_NVT_NHC2 3            /* 'nvt-nhc2': two-thermostat Nose-Hoover chain after Frenkel and Smit
                                      (nhc2 + chain_nhc2, src/integration.f90:205-324); nhc_n is 2, L = 3(N-1) */

/* arithmetic of the bulk pair and k-space work */
#define MDFF_PREC_FP64  0          /* plain FP64 everywhere */
#define MDFF_PREC_MIXED 1          /* FP32 bulk + FP64 accumulation/scalars */

/*
 * Parameters: the union of &controltag (src/control.f90:128-160), &fieldtag
 * (src/field.f90:450-500) and &mdtag (src/md.f90:109-132) tags on the path,
 * plus engine choices.  mdff_params_default() fills the reference defaults
 * (control_default_tag, field_default_tag, md_default_tag).
 */
typedef struct mdff_params {
    int ntype;
    /* &controltag */
    int lnmlj, lbmhft, lbmhftd, lmorse, lcoulomb, lvnlist, lreduced, lsurf;
    double cutshortrange, cutlongrange, skindiff;
    /* &fieldtag: per-type properties */
    double mass[MDFF_NTYPE_MAX];
    double qch[MDFF_NTYPE_MAX];
    double dip[MDFF_NTYPE_MAX][3];             /* static dipoles */
    double poldip_iso[MDFF_NTYPE_MAX];         /* isotropic dipole polarisability, A^3 */
    int    ldip_polar[MDFF_NTYPE_MAX];
    int    symmetric_pot;
    int    trunc;                              /* MDFF_TRUNC_* */
    double epslj[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double sigmalj[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double plj[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double qlj[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double epsmor[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double sigmamor[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double rhomor[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double Abmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double Bbmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double Cbmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double Dbmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double BDbmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    int    ldip_damping[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double dip_pol_damp_b[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double dip_pol_damp_c[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    int    dip_pol_damp_k[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    /* Ewald (src/field.f90:163-168, ewald_param :860-908) */
    double alphaES;
    int    kES[3];
    int    lautoES;
    double epsw;
    int    doefield, doefg;
    /* induced dipoles (src/field.f90:128-140) */
    double conv_tol_ind;
    int    min_scf_pol_iter, max_scf_pol_iter;
    int    algo_moment_from_pola;              /* MDFF_POLA_* */
    int    extrapolate_order;
    int    algo_ext_dipole;                    /* MDFF_EXT_* */
    /* &mdtag */
    int    integrator;                         /* MDFF_NVE_VV / MDFF_NVT_NHCN / MDFF_NPT_NHCNP / MDFF_NVT_NHC2 */
    double dt;                                 /* ps */
    double temp;                               /* K */
    int    nhc_n, nhc_yosh_order, nhc_mults;
    double timesca_thermo;                     /* ps */
    /* engine choices (no reference counterpart) */
    int    precision;                          /* MDFF_PREC_* */
    int    efg_period;                         /* EFG every n MD steps when doefg (0 = every step) */
    int    nlist_capacity;                     /* neighbours per atom reserved (0 = automatic) */
    int    device;                             /* CUDA device ordinal */
    int    erfc_ref;                           /* 1: the reference's fitted erfc (src/functions.f90:28-39) */
    int    nhc_literal;                        /* 1: chain_nhcn's literal force order (stale G(2..M-1)), and
                                                  nhc2's literal thermostat energy vxi^2/(2Q) */
    double mixed_ksplit;                       /* mixed path: |k| < mixed_ksplit*alpha summed in FP64 (0: none) */
    int    kspace_reuse;                       /* PCG: one reciprocal evaluation for the static field and the first
                                                  residual, and the final structure factor from the solver's by
                                                  linearity (0: the reference's sequence of evaluations) */
    double mixed_keps;                         /* mixed path: k-vectors whose Gaussian factor exp(-k^2/4 alpha^2)
                                                  is below mixed_keps are left out (0: the whole rectangle) */
    int    autotune;                           /* 1: time the candidate launch shapes of the Ewald kernels on the
                                                  first force evaluation and keep the fastest */
    int    kspace_tc;                          /* mixed path: 1 = structure factor and field on the tensor cores
                                                  (exact int8 digit products of 24-bit fixed point) when nz rows
                                                  <= 80, the low-|k| set in FP64 on the CUDA cores; 2 = the low-|k|
                                                  set on the tensor cores as well (32-bit fixed point, FP64
                                                  operands) when its nz rows <= 32; 0 = FP32 CUDA-core kernels */
    /* &mdtag, constant pressure (integrator MDFF_NPT_NHCNP) */
    double press;                              /* GPa (md_check_tag converts with press_unit) */
    double timesca_baro;                       /* ps */
    /* engine choice (no reference counterpart) */
    double fp64_keps;                          /* FP64 path: k-vectors whose Gaussian factor exp(-k^2/4 alpha^2) is
                                                  below fp64_keps are left out, as mixed_keps does on the mixed
                                                  path (0, the default: the reference's whole half space) */
} mdff_params;

/* Energies and scalar outputs of one force evaluation (thermodynamic module
 * variables written by engforce_driver, src/thermo.f90 and field.f90). */
typedef struct mdff_energies {
    double u_lj, u_bmhft, u_morse;             /* eV */
    double u_coul;                             /* eV, includes u_pol (field.f90:1974-1990) */
    double u_dir, u_rec, u_self, u_surf, u_pol;/* eV (coul_unit applied) */
    double vir_lj, vir_bmhft, vir_morse;       /* eV (sum r.f / 3) */
    double pvirial_coul;                       /* eV/A^3 */
    double utail, ptail;                       /* long-range LJ corrections (not in u_lj) */
    int    scf_iter;                           /* induced-dipole iterations used */
    double scf_rmsd;                           /* final RMS residual of mu/alpha - E */
} mdff_energies;

/* Per-step thermodynamics (calc_thermo, src/thermo.f90:116-207). */
typedef struct mdff_thermo {
    int    step;
    double e_kin, temp_r;                      /* eV, K */
    double u_tot, e_tot, h_tot;                /* eV; h_tot is the conserved quantity */
    double u_lj, u_bmhft, u_morse, u_coul, u_pol;
    double e_nvt;                              /* NHC thermostat energy (NPT: e_npt, thermostats and barostat) */
    double pressure_tot;                       /* GPa */
    double pvirial_tot;                        /* GPa */
    int    nlist_rebuilt;                      /* 1 if the Verlet list was rebuilt after this step */
    int    scf_iter;
    double scf_rmsd;
    double volume;                             /* A^3 (changes under MDFF_NPT_NHCNP) */
} mdff_thermo;

/* Derivative of a scalar loss with respect to the force-field tables (no
 * reference counterpart; the reference has no derivatives).  Layout mirrors
 * the tables of mdff_params.  The tables are taken as symmetric in their pair
 * indices (symmetric_pot): the derivative with respect to an unordered entry
 * {a,b} is returned in the upper-triangle slot [a][b] with a <= b (for the
 * damping tables [p][a][b] with a <= b), and the lower-triangle slots are 0.
 * Bbmhftd is the inverse range 1/rho as in the reference
 * (src/field.f90:2952); d/d(rho) = -B^2 d/dB. */
typedef struct mdff_param_grad {
    double Abmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double Bbmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double Cbmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double Dbmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double BDbmhftd[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double epsmor[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double sigmamor[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double rhomor[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double poldip_iso[MDFF_NTYPE_MAX];
    double dip_pol_damp_b[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
    double dip_pol_damp_c[MDFF_NTYPE_MAX][MDFF_NTYPE_MAX][MDFF_NTYPE_MAX];
} mdff_param_grad;

/* Result of a structure optimisation (opt_main's per-configuration report,
 * src/opt.f90:369-380: Eis, phigrad, iter, neng, pot0). */
typedef struct mdff_opt_result {
    double u_initial;   /* u_tot at the starting positions (eV), pot0 */
    double u_final;     /* u_tot at the returned positions (eV), Eis */
    double phigrad;     /* sum of the squared force components at the end (eV^2/A^2) */
    int    iterations;  /* conjugate-gradient iterations (its) */
    int    nforce;      /* force evaluations (neng) */
    int    status;      /* 0: minimum reached (sastry: energy unchanged to ftol; lbfgs: |G| / max(1, |X|)
                           <= eps); 1: itmax iterations (sastry) or force evaluations (lbfgs);
                           2: zero gradient; 3: the line search failed (sastry: no progress in 100
                           steps, or U still above the line's start after 64 halvings of a trial
                           step; lbfgs: MCSRCH returned info != 1, IFLAG = -1) */
    int    info;        /* lbfgs with status 3: MCSRCH's info (0 not a descent direction or bad
                           input, 2 interval below xtol, 3 maxfev reached, 4/5 at stpmin/stpmax,
                           6 rounding errors), 0 otherwise; m1qn3: its omode; sastry: 0 */
} mdff_opt_result;

/* Distribution settings of efg_stat (the efgtag namelist, src/efg.f90:171-190):
 * bins PANvzz = int(2|vzzmin|/resvzz), PANeta = int(1/reseta),
 * PANU = int(2|umin|/resu), PANS = int(smax/resu) (src/efg.f90:233-236). */
typedef struct mdff_efg_dist_params {
    double vzzmin, resvzz, reseta, umin, resu, smax;
} mdff_efg_dist_params;

/* sizeof(mdff_params), sizeof(mdff_energies), sizeof(mdff_thermo),
 * sizeof(mdff_param_grad), sizeof(mdff_opt_result) for which = 0 .. 4 (lets a binding check its
 * mirror of these structs); no reference counterpart. */
int  mdff_struct_size(int which);   /* 5 efg_dist_params, 6 frame_header, 7 rmc_params, 8 rmc_result,
                                       9 rmc_efg_params */

/* The real-space kernels' FP64 erfc (e^{-x^2} times a degree-13 Chebyshev fit
 * of erfc(x) e^{x^2} per half-unit interval on [0, 4.5), CUDA's erfc
 * elsewhere) and CUDA's erfc, evaluated on the device at n host points x:
 * ex2[n] and ref[n].  A check of the fit; no reference counterpart. */
int  mdff_erfc_check(int device, int n, const double* x, double* ex2, double* ref);

/* Measured FMA throughput of the device in TFLOP/s: out[0] FP64, out[1]
 * FP32, out[2] packed FP32x2 (fma.rn.f32x2).  The roofline denominators of
 * the engine's FMA-bound kernels; no reference counterpart. */
int  mdff_measure_pipes(int device, double out[3]);

/* Measured tcgen05 kind::i8 tensor-core throughput of the device in TOPS
 * (dense, S32 accumulate, operands resident in shared memory): out[0] with
 * N = 256 (the peak), out[1] N = 96 and out[2] N = 64 (the tile widths of the
 * structure-factor and field GEMMs).  No reference counterpart. */
int  mdff_measure_tensor(int device, double out[3]);

/* Fill p with the reference defaults (control_default_tag, src/control.f90:199-243;
 * field_default_tag, src/field.f90:192-273; md_default_tag, src/md.f90:178-205). */
void mdff_params_default(mdff_params* p);

typedef struct mdff_ctx mdff_ctx;

/* Create a context on p->device (replaces the set-up done by field_init and
 * md_init, src/field.f90:439-560, src/md.f90:99-357).  Parameters are
 * validated as field_check_tag / md_check_tag do (src/field.f90:282-432). */
int  mdff_create(const mdff_params* p, mdff_ctx** out);

/* Release the context and every device buffer it owns. */
void mdff_destroy(mdff_ctx* ctx);

/* Message of the last failing call on ctx (never NULL). */
const char* mdff_last_error(const mdff_ctx* ctx);

/* The context's CUDA stream (cudaStream_t), so a caller can order its own
 * work or timing events against the engine's; no reference counterpart. */
int  mdff_stream(mdff_ctx* ctx, void** stream);

/* Kernel timing with CUDA events on the context's stream, per kernel group:
 * 0 Verlet list, 1 pair loop, 2 Ewald real space, 3 structure factor,
 * 4 reciprocal field, 5 dipole solver vectors, 6 integrator, 7 other.
 * The counterpart of the reference's MPI_WTIME accumulators
 * (src/time.f90:35-73, src/symbol.h:2-17).  mdff_profile_get returns the
 * accumulated milliseconds and kernel launches per group and in total, and
 * clears them when reset != 0. */
int  mdff_profile(mdff_ctx* ctx, int enable);
int  mdff_profile_get(mdff_ctx* ctx, double ms[8], long long count[8], long long* launches, int reset);
/* Detail timers of single kernels: the tensor-core structure-factor kernel
 * [0] and field kernel [1] (mixed path, inside groups 3 and 4) with the int8
 * digit-product operations they were launched for (2 M N K per product, six
 * products, unpadded problem), the EFG post-processing site kernel [2] with
 * the bytes it must read (52 per site: tensor and type), and the low-|k|
 * set's 32-bit tensor-core structure-factor [3] and field [4] kernels (ten
 * digit products) -- accumulated milliseconds, launches and work; cleared
 * with the groups.  No reference counterpart. */
#define MDFF_NDETAIL 5
int  mdff_profile_detail(mdff_ctx* ctx, double ms[MDFF_NDETAIL], long long count[MDFF_NDETAIL],
                         double ops[MDFF_NDETAIL]);

/* Sizes of the reciprocal-space sums of the context (no reference
 * counterpart): out[0] the k rectangle the kernels sweep, out[1] the k-vectors
 * of the reference's half space (kpoint_sum_init, src/kspace.f90:142-207),
 * out[2] the main set the path sums (mixed: the FP32 / tensor-core set; FP64:
 * the half space, or its part inside the fp64_keps sphere) and out[3] the FP64
 * low-|k| set of the mixed path (0 on the FP64 path). */
int  mdff_kspace_info(mdff_ctx* ctx, long long out[4]);

/* Which reciprocal-space kernels the mixed path uses (no reference
 * counterpart): out[0] = 1 when the main set runs on the tensor cores (24-bit
 * fixed point, kspace_tc >= 1), out[1] = 1 when the low-|k| set does (32-bit
 * fixed point, kspace_tc = 2); 0 for the FP32 / FP64 CUDA-core kernels. */
int  mdff_kspace_mode(mdff_ctx* ctx, int out[2]);

/* How the context's MD steps ran (no reference counterpart): out[0] steps
 * replayed from a captured CUDA graph (the whole step, the dipole PCG as a
 * conditional loop on the device, one host synchronisation per step), out[1]
 * captures made (one per EFG / non-EFG step kind, again when the lists, pair
 * table, cell, launch shapes or predictor change), out[2] steps run as plain
 * launches (constant pressure, the SCF solver, profiling, the predictor's
 * start-up steps, a step before a reallocation). */
int  mdff_graph_info(mdff_ctx* ctx, long long out[3]);

/* Launch shape in use (the autotuner's choice, or the defaults): out[0] lanes
 * per atom of the FP64 real-space Ewald kernel, out[1] of the FP32 dipole
 * operator, out[2] and out[3] the FP32 structure-factor atom split and field
 * column split in halves of the default (no reference counterpart). */
int  mdff_launch_shape(mdff_ctx* ctx, int out[4]);

/* Define the system: natm atoms, 1-based types, Cartesian positions and the
 * cell.  Replaces read_pos + typeinfo_init (src/read_pos.f90:35-219): the cell
 * goes through lattice() (src/lattice.f90:60-175), positions are wrapped with
 * kardir/periodicbc/dirkar (src/read_pos.f90:148-150), ewald_param clamps
 * cutlongrange (src/field.f90:860-908), initialize_param_non_bonded and
 * initialize_coulomb run (src/field.f90:914-1101, 1596-1662), and the Verlet
 * lists are built (src/mdff.f90:192-193).  Resets the MD state. */
int  mdff_set_system(mdff_ctx* ctx, int natm, const int* itype,
                     const double* rx, const double* ry, const double* rz,
                     const double A[9]);

/* A new cell (column-major, as mdff_set_system) for the same atoms: the
 * lattice, the tail corrections and the Ewald k tables of the same k
 * rectangle follow it (the k membership of the mixed path's sets stays as set
 * up; meant for the percent-level changes of a constant-pressure run).
 * Positions are kept as given (Cartesian).  No reference counterpart (the
 * reference moves simu_cell inside nhcnp). */
int  mdff_set_cell(mdff_ctx* ctx, const double A[9]);
/* Replace the positions (no wrap): the state engforce_driver sees when a
 * caller moved the atoms itself.  After either call the Verlet lists are
 * rebuilt by the next force evaluation or list read, so a new cell and new
 * positions together cost one build. */
int  mdff_set_positions(mdff_ctx* ctx, const double* rx, const double* ry, const double* rz);

/* Wrapped positions as the engine holds them. */
int  mdff_get_positions(mdff_ctx* ctx, double* rx, double* ry, double* rz);

/* Current velocities (internal units). */
int  mdff_get_velocities(mdff_ctx* ctx, double* vx, double* vy, double* vz);

/* One force evaluation at the current positions with the current lists:
 * replaces engforce_driver (src/field.f90:1111-1166), i.e. the LJ / BMH(FTD) /
 * Morse pair loops, the induced-dipole solve and the multipole Ewald sum.
 * fx,fy,fz (natm each) receive the total force in eV/A; tau_nonb and tau_coul
 * (3x3, column-major) the stresses in GPa; ef (3*natm, component-major:
 * ef[c*natm+i]) the electric field in e/A^2 without coul_unit, as the
 * reference returns it (field.f90:1977); efg (6*natm, components xx,yy,zz,xy,
 * xz,yz, each natm long) the field gradient times coul_unit; mu (3*natm) the
 * total dipoles.  Any output pointer may be NULL. */
int  mdff_engforce(mdff_ctx* ctx, double* fx, double* fy, double* fz,
                   mdff_energies* e, double tau_nonb[9], double tau_coul[9],
                   double* ef, double* efg, double* mu);

/* Structure optimisation of the current positions by conjugate gradients
 * with cubic line minimisation: sastry + eforce1d (src/opt.f90:452-933), the
 * default optalgo of opt_main (src/opt.f90:251-439; epsilon, dutol, ds and
 * the energy test with ftol = tiny(1.0_dp) as there).  Every function value
 * is one mdff_engforce at trial positions on the lists of the starting
 * configuration.  On return the context's positions (mdff_get_positions) and
 * forces are those of the minimum; *out gets pot0, Eis, phigrad, iter, neng.
 * itmax: the reference's 10000. */
int  mdff_opt_sastry(mdff_ctx* ctx, int itmax, mdff_opt_result* out);

/* Structure optimisation by limited-memory BFGS: lbfgs_driver (src/opt.f90:
 * 972-1194) over Nocedal's LBFGS (src/lbfgs.f90:243-456; m = 5 pairs, no
 * user diagonal) and the More-Thuente line search MCSRCH/MCSTEP
 * (:655-1186; ftol 1e-4, gtol 0.9, maxfev 100, xtol tiny(1.0_dp)) on
 * X = (rx, ry, rz), G = -f, F = u_tot -- optalgo = 'lbfgs' of opt_main.
 * eps: the reference's epsrel_lbfgs (1e-5), the test |G| / max(1, |X|) <= eps.
 * itmax bounds the force evaluations (the driver's loop, 10000 there).  Every
 * evaluation is one mdff_engforce on the lists of the starting configuration.
 * On return the positions and forces are those of the last evaluation (the
 * accepted point when status = 0); *out gets pot0 (u_initial), Eis (u_final),
 * phigrad as the driver leaves it (|G|^2 of the evaluation before the last),
 * the L-BFGS iterations and the evaluations (nforce; the reference reports
 * this count as both iter and neng). */
int  mdff_opt_lbfgs(mdff_ctx* ctx, int itmax, double eps, mdff_opt_result* out);

/* Structure optimisation by M1QN3 (optalgo = 'm1qn3' of opt_main):
 * m1qn3_driver (src/opt.f90:1203-1330) over M1QN3 3.3 (src/m1qn3.f90) in its
 * configuration there -- diagonal initial scaling, cold start, m = 5 pairs,
 * the euclidean scalar product, normtype 'dfn', dxmin = tiny(1.0_dp),
 * df1 = 1, and the Wolfe line search mlis3 (rm1 1e-4, rm2 0.99) -- on
 * X = (rx, ry, rz), G = -f, F = u_tot.  niter, nsim: the driver's 6000 and
 * 6000; epsg: epsrel_m1qn3 (1e-5), the test |G| / |G_0| < epsg.  Every
 * evaluation is one mdff_engforce on the lists of the starting
 * configuration; after M1QN3 returns, one more evaluation at the returned
 * point, as the driver's loop makes it, so the positions, forces, u_final
 * and phigrad (|G|^2) on return belong together.  iterations: M1QN3's
 * niter; nforce: all evaluations (the reference reports one less, its
 * icall); info: M1QN3's omode; status 0 (omode 1), 1 (omode 4 or 5: niter
 * or nsim reached), 2 (omode 2: zero gradient at the start), 3 (omode 6:
 * dxmin or rounding in the line search, which the driver accepts with a
 * warning; omode 7: not a descent direction or (y, s) <= 0). */
int  mdff_opt_m1qn3(mdff_ctx* ctx, int niter, int nsim, double epsg, mdff_opt_result* out);

/* EFG post-processing (efg_stat, src/efg.f90:2057-2440, and nmr_convention,
 * :2546-2650) on the device, over nconf configurations of the context's
 * system at once (the configurations of an EFGALL file).  efg6: host tensors
 * [nconf][6][natm] (xx yy zz xy xz yz), or NULL with nconf = 1 for the
 * context's EFG of its last force evaluation (doefg).
 * mdff_efg_nmr, per site (any output may be NULL): nmr[nconf][4][natm] = Vxx,
 * Vyy, Vzz, eta (|Vzz| >= |Vyy| >= |Vxx|); U[nconf][5][natm] the Czjzek
 * components (Vzz/2, Vxz/sqrt3, Vyz/sqrt3, Vxy/sqrt3, (Vxx-Vyy)/(2 sqrt3));
 * S[nconf][natm] = |U|.  The principal values come from a cyclic Jacobi
 * iteration in FP64 in place of LAPACK's DSYEV. */
int  mdff_efg_nmr(mdff_ctx* ctx, int nconf, const double* efg6, double* nmr, double* U, double* S);
/* efg_stat's statistics and distributions.  Rows t = 0 (all sites), 1..ntype.
 * stats[nconf][ntype+1][8] per configuration: vzzmin, vzzmax, <Vzz>, <|Vzz|>,
 * <eta>, fraction Vzz >= 0, rho_z = sigma/<|Vzz|>, sigma = sqrt(<Vzz^2> -
 * <|Vzz|>^2), formed as the reference's loop forms them (averages zeroed once
 * before the loop, so each configuration's sums add to the previous
 * configuration's averages; extrema running from 0 over all configurations;
 * 0 where a row has no sites or <|Vzz|> = 0).  The isotropy test (:2435-2469)
 * over all configurations: mU[ntype+1][5] = <U_k>, m2U[ntype+1][5][5] =
 * <U_k U_l> on the upper triangle (k <= l, zero below), row 0 of m2U left as
 * the plain sum as there.  Counts summed over the configurations:
 * dib_vzz[ntype+1][PANvzz+1], dib_eta[ntype+1][PANeta+1],
 * dib_u[6][ntype+1][PANU+1] (U1..U5, then U2..U5 together),
 * dib_s[ntype+1][PANS+1].  A value outside the ranges returns MDFF_E_ARG (the
 * reference STOPs).  Any output may be NULL. */
int  mdff_efg_dist(mdff_ctx* ctx, int nconf, const double* efg6, const mdff_efg_dist_params* dp, double* stats,
                   double* mU, double* m2U, int* dib_vzz, int* dib_eta, int* dib_u, int* dib_s);

/* Rebuild the Verlet lists at the current positions: vnlist_pbc
 * (src/tools.f90:274-370). */
int  mdff_nlist_build(mdff_ctx* ctx);

/* Copy a Verlet list out in the reference's own layout (verlet_vdw /
 * verlet_coul, src/config.f90:64-72): point[natm+1] and list[...], both
 * 1-based, the half list with the reference's parity ownership rule
 * (src/tools.f90:320-321) and ascending j per atom.  which = 0 for the vdW
 * list (cutshortrange + skindiff), 1 for the Coulomb list (cutlongrange +
 * skindiff).  *nlist receives the number of entries; returns MDFF_E_LISTOVF
 * if cap is too small. */
int  mdff_nlist_get(mdff_ctx* ctx, int which, int* point, int* list, int cap, int* nlist);

/* Start MD from the current positions with the given velocities (A/ps
 * scaled like the reference's internal velocities: A per internal time unit):
 * computes step-0 forces and thermodynamics as md_run does before its loop
 * (src/runmd.f90:150-165).  t0 may be NULL. */
int  mdff_md_start(mdff_ctx* ctx, const double* vx, const double* vy, const double* vz,
                   mdff_thermo* t0);

/* Advance nsteps MD steps: the body of md_run's loop (src/runmd.f90:231-454):
 * prop_velocity_verlet (src/integration.f90:131-194) or nhcn
 * (src/integration.f90:476-713), then vnlistcheck (src/tools.f90:446-535) and
 * calc_thermo (src/thermo.f90:116-207).  Non-NULL position / velocity arrays
 * are uploaded before the first step and all non-NULL arrays (positions,
 * velocities, forces) are written back after the last.  thermo, if not NULL,
 * receives nsteps records. */
int  mdff_step(mdff_ctx* ctx, int nsteps,
               double* rx, double* ry, double* rz,
               double* vx, double* vy, double* vz,
               double* fx, double* fy, double* fz,
               mdff_thermo* thermo);

/*
 * Batched force matching (no reference counterpart: the reference evaluates
 * one configuration at a time and has no derivatives).  A batch holds nconf
 * fixed configurations of uneven atom counts sharing one force field; every
 * kernel of an evaluation is one launch over the whole batch.  The physics per
 * configuration is that of mdff_engforce in FP64 (BMH / BMHFTD, Morse,
 * multipole Ewald with polarisable ions solved by PCG to conv_tol_ind), with
 * one neighbour cutoff rc[c] for both the short-range and the real-space
 * Coulomb sums, Ewald alpha[c] and k rectangle kmax[3c..3c+2] per
 * configuration.  Lennard-Jones, static dipoles and lsurf are not supported
 * (MDFF_E_UNSUPPORTED); at most 2 atom types.
 *
 * Loss:  L = 1/nconf sum_c [ w_force/(3 N_c) sum_i |F_i - F*_i|^2
 *                           + w_stress/9 sum_ab (tau_ab - tau*_ab)^2 ]
 * with F the total force (eV/A) and tau = tau_nonb + tau_coul (GPa).
 */
typedef struct mdff_batch mdff_batch;

/* natm[c] atoms per configuration; itype (1-based), rx, ry, rz concatenated
 * over the configurations; cells[9c..9c+8] the column-major cell of
 * configuration c.  *out is set even when the call fails (read
 * mdff_batch_last_error, then mdff_batch_destroy). */
int  mdff_batch_create(const mdff_params* p, int nconf, const int* natm, const int* itype,
                       const double* rx, const double* ry, const double* rz, const double* cells,
                       const double* rc, const double* alpha, const int* kmax, mdff_batch** out);
void mdff_batch_destroy(mdff_batch* b);
const char* mdff_batch_last_error(const mdff_batch* b);
int  mdff_batch_stream(mdff_batch* b, void** stream);

/* Replace the force-field tables (same ntype and lcoulomb as at creation). */
int  mdff_batch_set_params(mdff_batch* b, const mdff_params* p);

/* Forces (concatenated, eV/A), total stress tau[9c..9c+8] (GPa, column-major)
 * and potential energy energy[c] (eV) of every configuration; iters receives
 * the iterations of the dipole solve.  Any output may be NULL. */
int  mdff_batch_forces(mdff_batch* b, double* fx, double* fy, double* fz, double* tau, double* energy,
                       int* iters);

/* Target forces (concatenated) and stresses (9 per configuration) of the loss. */
int  mdff_batch_set_targets(mdff_batch* b, const double* fx, const double* fy, const double* fz,
                            const double* tau, double w_force, double w_stress);

/* The loss and, when grad != NULL, its gradient with respect to the force-field
 * tables (adjoint method: one forward and one adjoint induced-dipole solve).
 * iters (may be NULL) receives the forward and adjoint solve iterations. */
int  mdff_batch_loss_grad(mdff_batch* b, double* loss, mdff_param_grad* grad, int iters[2]);

/*
 * Reciprocal-space Ewald energy of point charges that allocates no device
 * memory (no reference counterpart).  For callers that cannot let a library
 * allocate device memory while they run: a host code whose device memory is
 * held entirely by its own pool, or one that must not enter the CUDA
 * allocator inside a time step.  Inputs are the caller's DEVICE arrays (rx,
 * ry, rz Cartesian positions and q charges, natm each) on `device`; A is the
 * host cell matrix (column-major, as in mdff_set_system), kmax the host k
 * rectangle; stream is a cudaStream_t (NULL: the legacy default stream).
 * *u_rec receives the energy in eV with the reference's coul_unit
 * (14.3996441494161 eV A / e^2) applied, the same quantity as
 * mdff_energies.u_rec of mdff_engforce for a charges-only system outside
 * reduced units (lreduced is not taken into account here).  The call copies
 * the energy into *u_rec and waits for `stream` to finish before it returns.
 *
 * Scratch is a fixed 16 MiB array in device memory per device (2^21 doubles),
 * held by every device that loads the library until the process exits: a
 * problem needing more (3 natm + the structure-factor partials) returns
 * MDFF_E_NOMEM before anything is launched, and *scratch_needed (may be NULL)
 * receives the doubles it would need.  Each call looks up the array's device
 * address on `device` (cudaGetSymbolAddress, a host query that allocates
 * nothing).  Nothing in the scratch has to start at zero: every word a call
 * reads it has written earlier in the same call.  All calls on one device
 * share the scratch: overlapping calls race and must be serialised by the
 * caller.
 */
int  mdff_rec_energy_noalloc(int device, int natm, const double* rx, const double* ry, const double* rz,
                             const double* q, const double A[9], double alpha, const int kmax[3],
                             void* stream, double* u_rec, long long* scratch_needed);

/* ---- on-disk formats and streaming (TRAJFF, CONTFF, EFGALL, DIPFF, EFALL) ----
 * File kinds and their reference writers: TRAJFF write_trajff_xyz
 * (src/config.f90:539-628), CONTFF write_CONTFF (src/config.f90:206-250),
 * EFGALL write_EFGALL (src/field.f90:4140-4195), DIPFF write_DIPFF
 * (src/field.f90:4051-4083), EFALL write_EFALL (src/field.f90:4205-4240).
 * iformat 0 = Fortran unformatted sequential (4-byte record markers; TRAJFF
 * and EFGALL), else formatted.  data (TRAJFF): trajff_data as bits,
 * 0 = rnn, MDFF_DATA_V = rvn, MDFF_DATA_F = rnf, both = rvf. */
#define MDFF_FILE_TRAJFF 0
#define MDFF_FILE_CONTFF 1
#define MDFF_FILE_EFGALL 2
#define MDFF_FILE_DIPFF  3
#define MDFF_FILE_EFALL  4
#define MDFF_DATA_V 1
#define MDFF_DATA_F 2

/* Frame header: the config module's natm, system, simu_cell%A (column-major:
 * A[0..2] = first lattice vector), ntype, atypei, natmi. */
typedef struct mdff_frame_header {
    int natm, ntype;
    double A[9];
    char system[60];                 /* blank padded, not NUL terminated */
    char atypei[MDFF_NTYPE_MAX][3];  /* blank padded */
    int natmi[MDFF_NTYPE_MAX];
} mdff_frame_header;

/* One frame formatted on the host (no device use).  itype: 1-based type per
 * atom.  cols: [ncol][natm] -- TRAJFF: x y z [vx vy vz] [fx fy fz] (by data),
 * CONTFF: the nine of rvf, EFGALL: xx yy zz xy xz yz, DIPFF: mux muy muz,
 * EFALL: Ex Ey Ez; positions are written as given (the streaming writer folds
 * them into the cell first, as the reference's writers do).  out: cap bytes;
 * *len receives the frame's length (when cap is too small nothing is written
 * and MDFF_E_ARG is returned with *len the size needed). */
int  mdff_io_format(int file, int iformat, int data, const mdff_frame_header* h, const int* itype,
                    const double* cols, char* out, size_t cap, size_t* len);

/* Streaming writer bound to a context: each mdff_writer_frame snapshots the
 * context's current state on its stream and returns; a copy stream and a
 * writer thread bring the frame to the file (appended; CONTFF rewritten).
 * h supplies system and the type labels (natm, ntype, natmi and the cell come
 * from the context).  nslot frames may be in flight (>= 1).  EFGALL / DIPFF /
 * EFALL take the tensors, dipoles or fields of the last force evaluation
 * (doefg / lcoulomb as the reference requires).  Errors of the background
 * write are returned by the next mdff_writer_frame or by mdff_writer_close,
 * which drains the queue, closes the file and frees the writer. */
typedef struct mdff_writer mdff_writer;
int  mdff_writer_open(mdff_ctx* ctx, const char* path, int file, int iformat, int data, const mdff_frame_header* h,
                      int nslot, mdff_writer** w);
int  mdff_writer_frame(mdff_writer* w);
int  mdff_writer_close(mdff_writer* w);

/* Checkpoint of the whole time-integration state: what the reference restarts
 * from (CONTFF's positions, velocities, forces) plus what it cannot restore
 * (Nose-Hoover chain variables, the induced-dipole predictor history, the
 * neighbour-list reference positions, the step counter, the tuned launch
 * shapes), so that a restarted run continues bit for bit.
 * mdff_checkpoint_save writes into buf (cap bytes; *len the size; buf NULL to
 * query; MDFF_E_ARG when cap is too small).  mdff_checkpoint_load restores it
 * into a context created with the same parameters and system
 * (mdff_set_system), in place of mdff_md_start. */
int  mdff_checkpoint_save(mdff_ctx* ctx, void* buf, size_t cap, size_t* len);
int  mdff_checkpoint_load(mdff_ctx* ctx, const void* buf, size_t len);

/* ---- pair distribution and reverse Monte Carlo (rmc.f90, radial_distrib.f90) ----
 * g(r) as rmc_gr forms it (gr_main, src/radial_distrib.f90, normalised as
 * src/rmc.f90:1469-1490): nbins = INT(cut/res) + 1; rows mp = 0 (all pairs,
 * over natm^2) then the type pairs it1 <= it2 (over natmi(it1) natmi(it2)),
 * grr[(npairs+1)][nbins], npairs = ntype (ntype+1) / 2; at most 4 types.
 * grr NULL: *nbins only. */
int  mdff_gr(mdff_ctx* ctx, double cut, double res, double* grr, int* nbins);

/* rmc_main (src/rmc.f90:196-640) on the g(r) chi^2: single-atom trial moves
 * of up to max_displacement / ANORM per fractional axis (rmc_move), g(r)
 * chi^2 against grr_exp [(npairs+1)][nbins] (eval_chisq_rmc), the
 * Metropolis test of each chi^2 component with exp(-dchi^2 / 2 T) and the
 * total deciding.  temp_rmc[0..4]: the components' temperatures (g(r), var,
 * U, Vzz, eta), temp_rmc[5] the total's (the reference reads it past the end
 * of its 5-element array).  Only the g(r) term is computed here (the others
 * are 0).  Stops when acceptance_max configurations are accepted (the start
 * counting as 1) or after max_trials moves.  Random numbers: uniforms
 * [nuni] in [0,1) used in the reference's order (particle, 3 displacements,
 * then one per component whose chi^2 did not decrease), or NULL for a
 * counter-based stream from seed.  The context's positions are replaced by
 * the chain's last state; grr_out (may be NULL) receives its g(r). */
typedef struct mdff_rmc_params {
    double max_displacement;   /* A (rmctag default 0.1) */
    double resolution_gr;      /* A */
    double cut_rmc;            /* A */
    double temp_rmc[6];
    long long acceptance_max;
    long long max_trials;
} mdff_rmc_params;
typedef struct mdff_rmc_result {
    long long kall, kacc, uniforms_used;
    double chisq[6];           /* of the last accepted configuration (g(r), var, U, Vzz, eta, total) */
    int status;                /* 1: the given uniforms ran out */
    int pad;
} mdff_rmc_result;
int  mdff_rmc(mdff_ctx* ctx, const mdff_rmc_params* rp, const double* grr_exp, const double* uniforms,
              long long nuni, unsigned long long seed, double* grr_out, mdff_rmc_result* res);

/* rmctag's EFG settings (src/rmc.f90:40-60): which EFG chi^2 terms, from
 * which acceptance count, and the bins of rmc_efg: PANU = INT(2|u_efg_min| /
 * resolution_u_efg), PANvzz = INT(2|vzz_efg_min| / resolution_vzz_efg),
 * PANeta = INT(1 / resolution_eta_efg).  Values in the units of
 * multipole_efg_ES (e / A^3, no coul_unit). */
typedef struct mdff_rmc_efg_params {
    int lrmc_u, lrmc_vzz, lrmc_eta;
    int efg_start;                 /* the EFG terms while kacc >= efg_start (default 0) */
    double resolution_u_efg, u_efg_min;
    double resolution_vzz_efg, vzz_efg_min;
    double resolution_eta_efg;
    int lrmc_var;                  /* the distance-variance term (eval_chisq_var_distance, src/rmc.f90:778-1063) */
    int pad_;
} mdff_rmc_efg_params;

/* rmc_main with its optional chi^2 terms (src/rmc.f90:420-640): per trial move
 * the g(r) term as mdff_rmc (incremental counts), and while kacc >=
 * efg_start the EFG of the whole trial configuration (rmc_efg: the engine's
 * Ewald EFG of the point charges, multipole_efg_ES with mu = 0), its NMR
 * convention, the Vzz, eta and Czjzek U1..U5 histograms and eval_chisq_Uefg /
 * vzz / eta against the experimental distributions.  One host-driven trial
 * at a time (each needs a full-device EFG evaluation).  Distributions use
 * the reference's Fortran layouts: dibU (ui = 1..6, mp = 0..ntype,
 * bin = 0..PANU) with ui fastest, dibvzz and dibeta (mp, bin) with mp
 * fastest; the *_out arrays receive those of the last accepted
 * configuration (rows the reference never fills -- U's row 6, eta's last
 * bin -- are 0).  With lrmc_var, chi^2 component 2 is the distance-variance
 * term of every trial configuration: per atom and type the sorted distances
 * to all other atoms of that type (minimum image, no cutoff), and
 * sum (d_n - <d_n>)^2 / <d_n>^2 over atoms, types and ranks, the mean taken
 * over the atoms of each type.  Its sorted lists stay in device memory
 * (natm^2 doubles): a cell whose lists do not fit in free device memory, or
 * with more than 16385 atoms of one type, returns MDFF_E_UNSUPPORTED.
 * Uniforms, temperatures, stopping and the result as mdff_rmc.  With an EFG
 * term the system must be point charges: no static or induced dipoles
 * (MDFF_E_UNSUPPORTED otherwise). */
int  mdff_rmc_efg(mdff_ctx* ctx, const mdff_rmc_params* rp, const mdff_rmc_efg_params* ep,
                  const double* grr_exp, const double* dibU_exp, const double* dibvzz_exp,
                  const double* dibeta_exp, const double* uniforms, long long nuni,
                  unsigned long long seed, double* grr_out, double* dibU_out, double* dibvzz_out,
                  double* dibeta_out, mdff_rmc_result* res);

#ifdef __cplusplus
}
#endif

#endif /* MDFF_ENGINE_H */
