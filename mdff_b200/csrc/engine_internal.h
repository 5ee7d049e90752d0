// engine_internal.h -- declarations shared by the engine's host code and its
// CUDA kernels.  Nothing here is part of the public C ABI.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mdff_engine.h"

namespace mdff {

constexpr int NT = MDFF_NTYPE_MAX;
constexpr double PI = 3.14159265358979323846264338327950;

// Simulation cell as the kernels see it (passed by value).
// A[3*i+j] = simu_cell%A(i+1,j+1); B likewise, already divided by omega
// (src/lattice.f90:60-175).
struct CellP {
    double A[9];
    double B[9];
    double omega;
};

// Constants of one ordered type pair (ti,tj), index ti*NT+tj.  Built on the
// host from mdff_params exactly as initialize_param_non_bonded
// (src/field.f90:914-1101) and the damping tables of field_check_tag
// (src/field.f90:316-339).
struct PairConst {
    // Lennard-Jones n-m
    double rcutsq, sigsq, epsp, plj, qlj, fc, uc, uc1, uc2;
    // BMH / BMHFTD
    double A, B, C, D, BD;
    // Morse
    double epsmor, rhomor, rs;
    // Tang-Toennies dipole damping: "_i" = (ti,ti,tj) damps the field of j's
    // charge at i; "_j" = (tj,ti,tj) damps the field of i's charge at j
    // (src/field.f90:2205-2217).
    double db_i, dc_i, db_j, dc_j;
    int dk_i, dk_j;
    int ldamp;   // ldip_damping(ti,ti,tj) .or. ldip_damping(tj,ti,tj)
    int pad;
};

// Per-kernel-group timing with CUDA events on the context's stream (the
// counterpart of the reference's MPI_WTIME accumulators, src/time.f90:35-73)
// and a count of kernel launches.
enum ProfKind { PK_NLIST = 0, PK_PAIR, PK_DIR, PK_SFAC, PK_KFIELD, PK_SOLVER, PK_INTEGRATE, PK_OTHER, PK_NKIND };
// Detail timers of single kernels: the tensor-core structure factor and field
// kernels with the int8 MMA operations they were launched for, the EFG site
// kernel with the bytes it reads.
enum ProfDetail { PD_TC_SFAC = 0, PD_TC_FIELD, PD_EFG_SITES, PD_TC4_SFAC, PD_TC4_FIELD, PD_NDETAIL };
struct Prof {
    bool on = false;
    cudaStream_t st = nullptr;
    struct Pending { int kind; cudaEvent_t a, b; };   // kind >= PK_NKIND: detail PK_NKIND + d
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    double ms[PK_NKIND] = {0};
    long count[PK_NKIND] = {0};
    double dms[PD_NDETAIL] = {0}, dops[PD_NDETAIL] = {0};
    long dcount[PD_NDETAIL] = {0};
    long launches = 0;
    int open_kind = -1;
    size_t open_idx = 0, detail_idx = 0;
    void detail_begin(int d) {
        if (!on) return;
        Pending p{PK_NKIND + d, get(), get()};
        cudaEventRecord(p.a, st);
        pending.push_back(p);
        detail_idx = pending.size() - 1;
    }
    void detail_end(int d, double ops) {
        if (!on) return;
        cudaEventRecord(pending[detail_idx].b, st);
        dcount[d] += 1;
        dops[d] += ops;
    }
    cudaEvent_t get() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int kind) {
        if (!on) return;
        Pending p{kind, get(), get()};
        cudaEventRecord(p.a, st);
        pending.push_back(p);
        open_kind = kind;
        open_idx = pending.size() - 1;
    }
    void end(int nkernels) {
        launches += nkernels;
        if (!on || pending.empty() || open_kind < 0) return;
        cudaEventRecord(pending[open_idx].b, st);
        count[pending[open_idx].kind] += nkernels;
        open_kind = -1;
    }
    void harvest() {   // after the stream has been synchronised
        for (auto& p : pending) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
                if (p.kind < PK_NKIND) ms[p.kind] += t;
                else dms[p.kind - PK_NKIND] += t;
            }
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void reset() {
        harvest();
        for (int k = 0; k < PK_NKIND; ++k) { ms[k] = 0.0; count[k] = 0; }
        for (int k = 0; k < PD_NDETAIL; ++k) { dms[k] = 0.0; dops[k] = 0.0; dcount[k] = 0; }
        launches = 0;
    }
    void release() {
        harvest();
        for (auto e : pool) cudaEventDestroy(e);
        pool.clear();
    }
};

// Neighbour lists in ELL layout: row i holds cnt[i] entries at nbr[i*cap ...].
// The row is the FULL list (every j != i within cut+skin); the reference's
// half list is the subset satisfying its parity ownership rule.
struct NList {
    int* nbr = nullptr;
    int* cnt = nullptr;
    int cap = 0;
    double cut = 0.0;     // verlet_*%cut
};

// Deterministic reduction scratch: each kernel writes per-block partials of K
// values; reduce_partials sums them in block order.
struct Partials {
    double* buf = nullptr;
    int capacity = 0;   // doubles
};

// Scalars kept on the device between kernels.  Reductions write straight
// into these slots, so each group is contiguous.
struct DevScalars {
    double nonb[12];    // u_lj vir_lj u_bmh vir_bmh u_mor vir_mor, stress xx yy zz xy xz yz (half-pair sums)
    double dir[8];      // real-space energy, stress sums xx yy zz xy xz yz, pad
    double rec[8];      // sum_k A_k|S|^2, stress sums xx yy zz xy xz yz, pad
    double sums[8];     // qsq musq qtot(3) mutot(3)
    double upol[2];     // sum mu.alpha^-1.mu, pad
    double ke2[2];      // sum m v^2, pad
    // solver
    double rr, rz_new;  // written together by one reduction
    double rz, dAd, beta_cg, rmsd;
    int iter, converged;
    // MD
    double s_scale, e_nvt;
    double xi[16], vxi[16];
    // neighbour-list check
    double dmax1, dmax2;
    int rebuild;
    int overflow;
    int tc_err;         // tensor-core pipeline: a bounded wait gave up (bit per wait site)
    int pad_;
    double opt[2];      // structure optimisation: reduced dot products
};

// Launchers (kernels live in the *.cuh files, compiled as one unit by engine.cu).
void launch_frac(cudaStream_t st, int n, const double* x, const double* y, const double* z, CellP c,
                 double* sx, double* sy, double* sz);
void launch_wrap_positions(cudaStream_t st, int n, double* x, double* y, double* z, CellP c);

struct CellGrid {
    int nc[3] = {1, 1, 1};
    int ncell = 1;
    int* cell_of = nullptr;     // [n]
    int* cell_count = nullptr;  // [ncell]
    int* cell_start = nullptr;  // [ncell+1]
    int* cell_cursor = nullptr; // [ncell]
    int* cell_atoms = nullptr;  // [n]
    float4* cell_w = nullptr;   // [n] cell order: FP32 wrapped fractional coordinates, atom index as bits
    int ncell_alloc = 0;
};
void launch_bin(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz, CellGrid& g);
void launch_nlist(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz, CellP c,
                  const CellGrid& g, double rskinsq_a, NList& la, double rskinsq_b, NList* lb, int* overflow);
void launch_skin_check(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz,
                       const double* xs, const double* ys, const double* zs, CellP c, double skindiff,
                       Partials& part, DevScalars* d);

// Short-range pair loop: LJ / BMH(FTD) / Morse, forces written (not added).
struct PairFlags { int lj, bmh, bmhftd, morse, trunc, ntype; };
void launch_pair(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz, const int* type,
                 CellP c, const NList& l, const PairConst* pc, PairFlags fl,
                 double* fx, double* fy, double* fz, Partials& part, DevScalars* d);

// Real-space multipole Ewald (charges + dipoles).
struct DirFlags {
    int qq, qd, dd;        // tasks
    int damp;              // damp_ind
    int field, efg, forces;// outputs (forces implies energy + stress)
    int ntype;
    double alpha;          // Ewald alpha
    double cutsq;          // verlet_coul%cut^2
    int erfc_ref;          // use the reference's fitted erfc
    // optional output of the charge pass: the Coulomb list compacted to the
    // entries inside the cutoff (ddnbr, ddcnt) with the undamped
    // dipole-dipole radial factors (A1, B2) of each entry in FP32 (ddtab)
    float2* ddtab;
    int* ddnbr;
    int* ddcnt;
};
void launch_ewald_dir(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz,
                      const int* type, const double* q, const double* mu, CellP c, const NList& l,
                      const PairConst* pc, DirFlags fl,
                      double* ef, double* efg, double* f, Partials& part, DevScalars* d, int g = 16);

// Reciprocal-space multipole Ewald.
struct KGrid {
    int kmax[3];
    int ncol;            // (kmax0+1)*(2*kmax1+1)
    int nzl;             // 2*kmax2+1
    int nrect;           // ncol*nzl
    double* Ak = nullptr;      // [nrect], 0 for excluded k
    double* kcoe = nullptr;    // [nrect]
    double* Ak_hi = nullptr;   // [nrect], Ak of the FP32 set: without the low-|k| set and outside the sphere (mixed path)
    int* colrange = nullptr;   // [ncol][2]: first 16-wide nz chunk and chunk count of the FP32 set (mixed path)
    int* items = nullptr;      // [nitems][2]: (column, chunk) work list of the FP32 structure factor
    unsigned char* mask = nullptr;   // [nrect]: bit 1 in the half space, bit 2 in the FP32 set (fixed at set-up)
    int nitems = 0;
    // FP64 path with the fp64_keps sphere: the (column, CH-wide nz chunk) work
    // list of the structure factor, and the columns holding a vector with the
    // nz index range [lo, lo + cnt) of each, for the field pass
    int* fitems = nullptr;     // [nfitems][2]
    int nfitems = 0;
    int* fcols = nullptr;      // [nfcol]
    int* fzr = nullptr;        // [nfcol][2]: lo, cnt
    int nfcol = 0;
};
// The low-|k| set of the mixed path, summed in FP64 (see ewald_recip.cuh):
// columns (nx, ny) with a contiguous nz range [nzlo, nzlo + nzn).
struct LowK {
    int ncol = 0;          // columns in the list
    int nzmax = 0;         // longest column
    int* col = nullptr;    // [ncol][4]: nx, ny, nzlo, nzn
    double* Ak = nullptr;  // [ncol][nzmax]
    double* kcoe = nullptr;
    double* part = nullptr;   // pass-1 partials [2][P][nzmax][ncol]
    double* aks = nullptr;    // [2][ncol][nzmax]
    double* fpart = nullptr;  // [LK_SPLIT][9][n]
    double* aks_acc = nullptr;   // solver accumulator of aks (reuse of structure factors)
    double2* tab = nullptr;   // [n][16] e^{2 pi i m s_z} in FP64
    int P = 1, natom_chunk = 0;
    // tensor-core form in 32-bit fixed point (kspace_tc = 2, ewald_tc4.cuh)
    int tc = 0;
    int kx = 0, ky = 0, kz = 0, nzl = 0;   // index half-ranges of the list; nz rows 2 kz + 1
    int N = 0, XYW = 0;                    // structure-factor GEMM N, X/Y table width
    int nblk = 0, npad = 0, bps = 0, nsplit = 0, ntile = 0, nin = 0;   // nin: input pipeline depth
    int KZ = 0, ntile_f = 0;               // field pass: K bytes per atom row, 128-atom tiles
    size_t smem = 0, smem_f2 = 0, smem_f3 = 0;
    double2* xy = nullptr;    // [npad][XYW] X_a[nx], Y_a[ny]
    uint8_t* bimg = nullptr;  // [nblk] B digit images
    double4* prm = nullptr;   // [npad] (q, m1, m2, m3)
    double* amax = nullptr;   // [npad]
    uint8_t* aimg = nullptr;  // [ntile_f] Z digit images
    double2* xyt = nullptr;   // [ntile_f][XYW][128]
    uint8_t* fimg = nullptr;  // per evaluation: B digit images + column constants
};

// Tensor-core structure factor of the mixed path (ewald_tc.cuh).
struct TcK {
    int on = 0;
    int nsph = 0;             // sphere columns (rows of the GEMM)
    int* cols = nullptr;      // [nsph] rectangle column index of each row
    int ntile = 0, nsplit = 0, bps = 0;   // 128-row tiles, atom splits, 16-atom blocks per split
    int nblk = 0, npad = 0;   // 16-atom blocks, padded atom count
    int N = 0, XYW = 0;       // GEMM N (2 x padded nz rows), per-atom X/Y table width
    int kx = 0, ky = 0, kz = 0, nzl = 0;
    size_t smem = 0;
    float2* xy = nullptr;     // [npad][XYW] X_a[nx], Y_a[ny]
    uint8_t* bimg = nullptr;  // [nblk] B digit images
    float4* prm = nullptr;    // [npad] (q, m1, m2, m3)
    float* amax = nullptr;    // [npad]
    // field pass
    int ntile_f = 0, KZ = 0;  // 128-atom tiles, K bytes (nz, re/im) per atom row
    int grid_f = 0;           // field CTAs: min(tiles, SMs), each an equal share of (tile, column block) units
    uint8_t* aimg = nullptr;  // [ntile_f] Z digit images
    float2* xyt = nullptr;    // [ntile_f][XYW][128] X/Y tables
    uint8_t* fimg = nullptr;  // per evaluation: B digit images + column constants
    size_t smem_f2 = 0, smem_f3 = 0;
};

struct RecScratch {
    double* part = nullptr;    // structure-factor partials
    size_t part_cap = 0;       // doubles
    double* aks = nullptr;     // [2][nrect] Ak*S (re, im)
    double* aks_acc = nullptr; // [2][nrect] solver accumulator of Ak*S (reuse of structure factors)
    double* fpart = nullptr;   // per-atom field partials [split][9][n]
    size_t fpart_cap = 0;
    uint32_t* fixed = nullptr;  // [3][n] fractional coordinates as 32-bit fixed point
    float2* tab = nullptr;      // [n][16] e^{2 pi i m s_z}
    float4* aks2 = nullptr;     // [ncol][nzp] A_k S(k) padded, FP32 pairs (re, re, im, im)
    int p_mul = 2, s_mul = 2;   // mixed path: FP32 structure-factor atom split and field column split, x mul/2
    long tab_epoch = -1;        // position epoch the table was built for
    long want_epoch = 0;        // current position epoch (set by the engine)
    LowK low;
    TcK tc;
};
struct RecFlags {
    int with_q, with_mu;
    int field;     // E
    int grad;      // full field gradient (for EFG and dipole forces)
    int energy;    // energy + stress
    int forces;    // forces q E + G mu
    int prec;      // MDFF_PREC_*
    int reuse;     // take A_k S from the solver's accumulators (no structure-factor pass)
};
void launch_ewald_rec(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz,
                      const double* q, const double* mu, CellP c, const KGrid& kg, RecFlags fl,
                      RecScratch& rs, double* ef, double* efg6, double* fo, Partials& part, DevScalars* d,
                      Prof* prof);
size_t rec_scratch_doubles(int n, const KGrid& kg, size_t* fpart, int mixed);
void launch_aks_accumulate(cudaStream_t st, const KGrid& kg, RecScratch& rs, const DevScalars* d, int copy);
int ensure_phase_tables(cudaStream_t st, int n, const double* sx, const double* sy, const double* sz, RecScratch& rs);
void launch_ewald_dd32(cudaStream_t st, int n, const uint32_t* fx, const double* mu, CellP c, const NList& l,
                       double cutsq, double alpha, double* ef, int g = 16);
// The solver's real-space dipole operator from the charge pass's pair table;
// rec is per-atom scratch of 8 words (fixed-point coordinates, FP32 dipole).
void launch_ewald_ddtab(cudaStream_t st, int n, const uint32_t* fx, const double* mu, CellP c, const int* nbr,
                        const int* cnt, int cap, const float2* tab, uint4* rec, double* ef, int g = 16);

// Solver vector kernels.

// Reduce per-block partials: out[k] = sum_b buf[b*K + k].
void launch_reduce_partials(cudaStream_t st, const double* buf, int nblocks, int K, double* out, int accumulate);

}  // namespace mdff
