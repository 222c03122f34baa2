// Internal declarations of the B200 solver library (not part of the public ABI).
//
// Data model: one device instance ("Inst") per simulated device.  Node arrays live in
// HBM as structure-of-arrays, x fastest (node k = i + Nx*(j + Ny*l), the reference's
// IDX, semiconductor_3d.c:114).  Kernels address an instance through a device-resident
// parameter record (DevP) selected by blockIdx.y, so the same kernels run one instance
// or a batch of instances per launch.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace ss {

constexpr double Q = 1.602176634e-19;
constexpr double KB = 1.380649e-23;
constexpr double EPS0 = 8.8541878128e-12;
constexpr double EPS_OX = 3.9 * EPS0;
constexpr double LN_MIN = -230.0, LN_MAX = 150.0, NFLOOR = 1e-100;
constexpr double PH_NONE = -1e300;
constexpr int NM_MAX = 16, NC_MAX = 32, AA_MAX = 12, MAXLEV = 24;
constexpr int K_SEMI = 0, K_INS = 1, K_METAL = 2;
constexpr int TPB = 256;            // threads per block of the node kernels
constexpr int RED_MAX_BLOCKS = 2048; // grid cap of reducing kernels (partials per instance)
constexpr int RED_NV = 16;          // doubles per block partial record
constexpr int COARSE_MAX = 64;      // unknowns of the coarsest multigrid level
constexpr int ION_W = 4;            // doubles per node of the ionisation constants

// per-node flag word: kind(2) | contact+1 (6) | gate+1 (6) | material (4) | car_fix (1)
__host__ __device__ inline int fl_kind(uint32_t f) { return int(f & 3u); }
__host__ __device__ inline int fl_con(uint32_t f) { return int((f >> 2) & 63u); }
__host__ __device__ inline int fl_gate(uint32_t f) { return int((f >> 8) & 63u); }
__host__ __device__ inline int fl_mat(uint32_t f) { return int((f >> 14) & 15u); }
__host__ __device__ inline bool fl_fix(uint32_t f) { return (f >> 18) & 1u; }
__host__ __device__ inline uint32_t make_flags(int kind, int con, int gate, int mat, bool fix) {
    return uint32_t(kind) | (uint32_t(con) << 2) | (uint32_t(gate) << 8) | (uint32_t(mat) << 14) |
           (uint32_t(fix ? 1 : 0) << 18);
}

// material constants the kernels need (semiconductor_3d.c:127-188, derived by mat_prepare)
struct MatD {
    double VT, lnc, lnv, ni, eps;
    double tau_n0, tau_p0, Cn, Cp, Brad, tau_Nref;
    double vsat_n, vsat_p, beta_n, beta_p, ani_n, ani_p;
    double chi, Eg;
    double ion_w[2];             // donor site weights of incomplete ionisation
    double T, Nc, Nv;            // temperature and band densities of states (metal contacts)
    double rich_n, rich_p, mtun_e, mtun_h;   // Richardson constants, tunnelling masses
    double ms_e, ms_h;                       // supply masses of gate tunnelling
    double ii_a[2][2], ii_b[2][2], ii_E0[2], ii_m[2], ii_g;   // impact ionisation (models bit 8)
    double lbB[2], lbC[2], lbL[2], lbD[2], lbE[2];           // Lombardi surface mobility (models bit 4)
    double lbc_mu1, lbc_nu, lbc_N0, lbc_e1, lbc_e2, lbc_E0, lbc_gam;   // its Coulomb term (4H-SiC)
    int insulator, ii_on, lb_on, lbc_on;
};

// contact constants the kernels need
struct ConD {
    double V, phi_m, tox, qox;   // applied voltage of the stage, work function, oxide
    int bc, te;                  // boundary type; thermionic-emission metal contact (models bit 6)
};

// one multigrid level of scalar type T (7-point stencil, 2x2x2 aggregation)
template <class T>
struct LevelT {
    int Nx, Ny, Nz, N;
    int cx, cy, cz, last;        // coarsened along x/y/z; last = coarsest (dense) level
    int apitch, pad_;            // A[q] = A[0] + q * apitch (the seven arrays are laid out back to back)
    T *A[7];                     // c, xm, xp, ym, yp, zm, zp
    T *D;                        // reciprocal red-black D-ILU pivots (or the dense inverse on the last level)
    T *x, *b, *r;
    T *pw;                       // prolongation weights (to the parent)
    double *ph;                  // reference level / VT of the Slotboom weights (set-up only)
};

// per-instance Krylov scalars (device resident; written by the reduction finalisers)
struct KrylovS {
    double rho, al, om, rho1, be, rv, ss, tt, ts, rr, r0, tgt, rbest, fl;
    double rz, rz0, pq;
    double rtol, atol;               // stop rule of the running solve (set by the host)
    int it, stall, active, status;   // status: 0 running, 1 converged, 2 breakdown/stop, 3 iteration cap
    int half, pad0, maxit, body_runs;
};

// Grid-wide barrier and reduction records of a persistent solve launch (one per
// instance): the arrival counter (set to 0 before every launch), the error word (1: a
// barrier wait ran out of time and every block left), the work done (V-cycles, Krylov
// iterations, refinement steps) for the byte accounting, and two alternating buffers of
// per-block reduction partials (up to 4 values per block).
constexpr int PG_MAXB = 512;
struct PGrid {
    unsigned count, err;
    int vcycles, iters, steps, pad;
    double red[2][PG_MAXB * 4];
};

// one level of the aggregation multigrid of a general (graph) mesh: the level's matrix in
// ELL (slot s of node k at s*N + k; the diagonal apart), its D-ILU(0) pivot reciprocals in
// a multicolour order, and towards the next level the aggregate of every node, the member
// lists of the aggregates and, per ELL entry, the coarse ELL entry it sums into (-1 inside
// an aggregate)
struct GLev {
    int N, D;
    const int *col, *rev, *color;
    double *val, *diag, *dil;
    const int *agg, *mrp, *mem, *emap;   // null at the coarsest level
    double *pw, *ph, *x, *b, *r;
    double *inv;                         // coarsest level: dense inverse (N x N), or null (ILU sweeps)
};

// everything a kernel needs about one instance
struct DevP {
    int Nx, Ny, Nz, N;
    int models, caxis, ncon, ref_mat;
    double VTref, Cref;
    const double *xs, *ys, *zs, *Lx, *Ly, *Lz;
    const uint32_t *flags;
    const double *Nd, *Na, *Nf, *bgn, *robA;
    const double *qd;             // distance to the nearest insulator / gate wall (display)
    double *ion;                  // incomplete ionisation, ION_W per node (null: every dopant ionised)
    // band corrections of electrons / holes in units of VT (the reference's qcn / qcp: MLDA
    // confinement plus the image-force lowering at metal contacts; null without either);
    // metal contacts (null without them): the continuity sink and source of the exchange
    // (tk c - tg), and the velocity-saturation weight near a contact with the axis of its normal
    double *qcn, *qcp, *tk, *tg;
    double *imgn, *imgp;          // the image-force part of qcn / qcp (metal contacts)
    double *gii;                  // impact-ionisation pair generation of the node (1/s; null: models bit 8 off)
    // deep-level traps (null without them): per node the range tr_rp[k]..tr_rp[k+1] of its
    // entries - species, density (m^-3), capture coefficients cn, cp (m^3/s)
    const int *tr_rp, *tr_s;
    const double *tr_N, *tr_cn, *tr_cp;
    const struct TrapD *tsp;      // species: type (-1 acceptor, 1 donor, 0 neutral), level reference, energy
    // Coulomb scattering on interface charge (models bit 4 with a Coulomb material; null
    // without): per node its nearest interface entry (-1: none within reach); per entry its
    // node, dual-face area, fixed charge (elementary charges) and N_C (m^-2)
    const int *qi, *if_k;
    const double *if_A, *if_Qf;
    double *if_NC;
    int n_if, pad_if;
    // general (graph) mesh, null on a tensor mesh: ELL layout with gD slots per node, slot s
    // of node k at s*N + k - neighbour (-1 past the degree), undirected edge id, slot of the
    // reverse edge, edge length, dual face area, matrix off-diagonal; node positions (3 per
    // node), least-squares gradient matrices (6 per node), colours of the D-ILU order and
    // its reciprocal pivots; edge mobilities per undirected edge
    int gD, nUE;
    const int *gcol, *gue, *grev;
    const double *gh, *ga, *gpos, *glsq;
    double *gval, *gmu_n, *gmu_p, *gdil;
    double *ggrad;               // least-squares potential gradient near walls (3 N, surface mobility)
    const float *te_vw;
    const signed char *te_ax;
    const MatD *mats;
    const ConD *cons;
    const int *cnode;             // contact-node list (semiconductor nodes of carrier contacts)
    int ncnode, nlev;
    // state
    double *phi, *phin, *phip, *n, *p;
    double *mu0n, *mu0p;          // low-field node mobility (fixed after set-up)
    double *mudn, *mudp;          // display mobility (after a resolve)
    double *fmu[6];               // face mobility k -> k+e_ax: 0-2 electrons, 3-5 holes
    // level-0 system, FP64
    double *A[7], *rhs, *sc, *dsc, *sol, *F;
    double *wk[8];                // Krylov work vectors
    double *qn0, *qp0, *dqn, *dqp, *xk, *tr;
    double *Jx, *Jy, *Jz, *Rt;    // display current density and recombination
    double *h1[3], *h2[3], *e2[3], *e3[3];   // path states; the last two sweep points' solutions
    // Anderson
    float *aaF, *aaG;             // AA_MAX slots of 3N each
    double *aaf, *aag;            // 3N each
    double *gram;                 // AA_MAX*AA_MAX
    double *aagam;                // AA_MAX coefficients
    // reductions
    double *part;                 // RED_MAX_BLOCKS*RED_NV
    unsigned *ticket;             // one counter per reduction slot (16)
    double *partc;                // terminal-current partials: 256 blocks x 96
    double *ffbuf;                // floating-block sums: 6 x 1024
    int *ffint;                   // floating-block flags / counts / roots: 16 + 1024
    unsigned long long *ffacc;    // floating-block exact accumulators: 4 sums x 1024 x XS_WORDS
    double *res;                  // scalar results (64)
    KrylovS *ks;
    // FP32 copy of the level-0 system and the FP32 Krylov vectors of the refined solves
    float *A32[7], *dsc32, *rhs32, *sol32;
    float *wk32[8];
    KrylovS *ksi;                 // Krylov record of the FP32 inner solve
    PGrid *pgrid;                 // barrier and reduction records of the persistent solves
    // multigrid (FP64 and FP32 hierarchies)
    LevelT<double> *lev;          // device array of nlev levels
    LevelT<float> *levf;
    int *ccl;                     // labels for connected-component work
    int *cclaux;
};

// a deep-level species: type -1 acceptor / +1 donor / 0 neutral; E (eV) below Ec (ref 0),
// above Ev (ref 1) or above the intrinsic level (ref 2)
struct TrapD {
    int type, ref;
    double E;
};

// Thermionic-emission metal contacts (models bit 6, semiconductor_3d.c:3390-3571): the
// entries are the semiconductor nodes of metal face contacts, each with its column of
// nodes along the inward normal (at most TE_COL deep); `touched` lists every column node
// once with its column entries in ascending order (CSR), so gathers add in entry order.
constexpr double TE_COL = 60e-9;
constexpr int TE_NE = 64;          // Simpson intervals of the tunnelling energy integral
constexpr int TE_NNMAX = 256;      // column nodes the tunnelling integral looks at
struct TeD {
    int n_te, n_tc, n_touch, models;
    const int *te_k, *te_c, *te_c0, *te_cn;
    const double *te_A;
    double *te_K, *te_G;           // 2 per entry: thermionic-emission coefficients (n, p)
    const int *tc_k;
    const double *tc_s;            // distance of a column node from the interface
    double *tc_K, *tc_G, *tc_I;    // 2 per column node: exchange terms, image-force lowering
    const int *tn_k, *tn_ptr, *tn_q;
    int ce0[NC_MAX], ce1[NC_MAX];  // entry range of every contact
};

// Gate tunnelling (models bit 5, semiconductor_3d.c:3146-3388): one path per semiconductor
// node facing an insulator that ends on a gate metal within 30 nm (plus one per Robin-gate
// node with a layer stack), its layers (material, thickness; at most 6) and its supply
// column of semiconductor nodes inward from the interface (5 nm deep).
struct TunD {
    int n_tp, n_col;
    const int *tp_k, *tp_c, *tp_nl, *tp_m, *tp_c0, *tp_cn;   // tp_m: 6 per path
    const double *tp_t, *tp_A;                               // tp_t: 6 per path
    double *tp_G;                  // 2 per path: injection from the gate (electrons, holes; 1/s)
    const int *col_k;
    const double *col_l, *col_h;   // cell length along the path axis, spacing to the next node
    double *col_K;                 // 2 per column node: escape rate per unit density
};
// gather of the continuity sink / source per node, in the reference's order: gate
// tunnelling column terms, gate injection, then the metal-contact terms
struct ScD {
    int n;
    const int *k, *pk, *pg, *pe;   // nodes; CSR pointers into qk (tunnel column entries),
    const int *qk, *qg, *qe;       // qg (paths of the node) and qe (metal-contact column entries)
};

// slots of DevP::res
enum ResSlot {
    R_PNORM = 0,     // poisson ||F/diag||
    R_DMAX = 1,      // max |dx| (Newton step)
    R_DQ = 2,        // cont_update weighted max |dq|
    R_DPSI = 3,      // max |psi - xk|
    R_FLOOR = 4,
    R_AUX = 5,
    R_I = 8,         // terminal currents I[NC_MAX] at 8..39
    R_S = 40,        // scales S[NC_MAX] at 40..71 (res has 128 doubles)
    R_IN = 72,       // electron components at 72..103
    R_OUT = 104,     // per-point output reductions at 104..110
    R_GII = 111,     // total impact-ionisation generation
    R_TOTAL = 128
};

}  // namespace ss
