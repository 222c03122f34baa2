// Host-side state of one simulated device and its GPU buffers.
#pragma once
#include <atomic>
#include <cstdint>
#include <vector>

#include "kernels.h"
#include "materials.h"
#include "semisim.h"

namespace ss {

// level-0 vector selectors understood by the linear-algebra kernels (0..7 = DevP::wk)
enum VecSel { V_RHS = 8, V_SOL = 9, V_F = 10, V_TR = 11, V_DSC = 12, V_PHI = 13 };

// multigrid shape over all instances of a launch
struct MGHost {
    int maxlev = 0, minlev = 0;
    int maxN[MAXLEV] = {0};
    int maxNx[MAXLEV] = {0};       // largest x extent of the level
    int maxRows[MAXLEV] = {0};     // largest Ny*Nz of the level
    double alpha = 1.0;
};
double bench_la_kernel(const Ctx &c, const MGHost &mg, int which, int reps);
extern int g_small_nodes;

struct Contact {
    int face = 0, i0 = 0, i1 = 0, j0 = 0, j1 = 0, k0 = 0, k1 = 0, bc = 0;
    double V = 0, phi_m = 0, tox = 10e-9, qox = 0;
    double Vprev = 0, I = 0, A = 0, In = 0, Iflr = 0, Iraw = 0;
    int snl = 0, smat[6] = {0}, ntp = 0;   // Robin-gate layer stack for tunnelling; paths of the contact
    double st[6] = {0};
    int te = 0;                  // thermionic-emission metal contact (set by prepare)
};

// a device on a general box-method mesh (api3_set_mesh_graph): the symmetric CSR graph with
// per directed edge its length and dual face area, per node its volume, position and walls
// (api3_set_walls), and the derived reverse entries, undirected edge ids and colouring
struct GraphHost {
    std::vector<int> rp, cj, rev, ue;
    std::vector<double> h, ar, vol, pos, wall;
    int nue = 0, D = 0;
};

// one V-cycle of the graph multigrid captured as a CUDA graph: its operands and executable
struct GmgCycle {
    const double *r = nullptr, *w = nullptr;
    double *z = nullptr;
    bool ilu_only = false;
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches = 0;   // kernels in the graph
};

// a level of the graph multigrid on the host: the device view and its colour classes
struct GLevHost {
    GLev dv{};
    int ncolor = 0;
    std::vector<int> cptr;       // colour q: cnodes[cptr[q] .. cptr[q+1])
    int *cnodes = nullptr;       // device
};

struct Gpu {
    bool ready = false;
    int dev = 0;
    size_t N = 0, bytes = 0;
    void *block = nullptr;       // one allocation for all node arrays
    DevP h{};                    // host copy of the device record
    DevP *d = nullptr;           // device record
    MGHost mg;
    std::vector<LevelT<double>> levs;
    cudaStream_t st = nullptr;
    LoopGraphs lg;               // device-looped Krylov solves
    cudaEvent_t tev[2] = {nullptr, nullptr};   // stream timer (test hook)
    double *pin = nullptr;       // pinned host scratch (results)
    double *scratch = nullptr;   // device scratch (bulk output)
    int *flag = nullptr;         // device int scratch
    double *ion = nullptr;       // incomplete-ionisation constants (ION_W x N), when a material needs them
    double *gii = nullptr;       // impact-ionisation generation (N), with models bit 8
    double *qc = nullptr;        // band corrections qcn, qcp (2 N), with MLDA or metal contacts
    double *xchg = nullptr;      // continuity sink / source tk, tg (2 N), with gate tunnelling or metal contacts
    void *gblock = nullptr;      // graph-mesh arrays (ELL edges, colours, gradients, edge mobilities)
    void *gmgblock = nullptr;    // graph multigrid levels (one allocation)
    std::vector<GLevHost> glev;  // graph multigrid hierarchy, level 0 = the mesh
    std::vector<GmgCycle> gcyc;  // its V-cycles captured as CUDA graphs (per operand set)
    void *gptab = nullptr;       // the hierarchy's level table for the persistent graph solves (device)
    bool gcyc_off = false;       // capture failed once: launch the V-cycle directly
    void *trblock = nullptr;     // deep-level trap entries (CSR per node) and species
    void *coblock = nullptr;     // Coulomb interface entries and every node's nearest one
    void *teblock = nullptr;     // metal-contact entries, columns and per-node arrays (one allocation)
    void *tunblock = nullptr;    // gate-tunnelling paths and columns, and the exchange gather
    TunD tun{};
    ScD sc{};
    bool tun_on = false;
    TeD te{};
    bool te_on = false;
    int *qown = nullptr;         // charge-partition owners (N, dense terminal slots), uploaded on first use
    bool qown_ok = false;
    int qown_nt = 0;             // the terminal count they were numbered for
    void *seedw = nullptr;       // learned predictor: BF16 weight pack, then FP32 biases and parameters
    float *seedb = nullptr;
    void *seedx = nullptr;       // its node features (N x 48 BF16), in the same allocation
};

struct TrapSpec { int type, ref; double E, sn, sp; };   // deep-level species (api3_trap_species)

// launch shapes of an instance's linear-algebra kernels (picked by api3b_autotune)
struct Tune {
    int rpb = 4;                  // rows per block of the row-blocked level passes
    int grid_cap = 148 * 8;       // blocks of the grid-stride node kernels
    int small_nodes = 0;          // size at which the small-level kernel takes over (0: default)
    int zcap = 65535;             // most row blocks of one row-blocked pass
    int rq = 1;                   // coarse rows per residual + restriction block
    int tuned = 0;
    double us = 0.0;              // V-cycle time of the chosen shapes (microseconds)
};

struct Inst {
    // ---- configuration (the reference's Dev, semiconductor_3d.c:234-364)
    int Nx = 0, Ny = 0, Nz = 0;
    size_t N = 0;
    std::vector<double> xs, ys, zs, Lx, Ly, Lz;
    std::vector<int> mat_idx;
    std::vector<double> Nd, Na, Nf;
    Material mats[NM_MAX];
    int n_mats = 0;
    Contact cons[NC_MAX];
    int n_cons = 0;
    std::vector<int> cnodes[NC_MAX];       // node-list contacts (api3_set_con_nodes)
    std::vector<double> careas[NC_MAX];
    int max_iter_p = 2000, max_iter_c = 1000, max_gummel = 500;
    double tol_p = 1e-9, tol_c = 1e-6, omega_p = 1, omega_c = 1;
    int converged = 0, conv_iter = 0;
    double conv_res = 0;
    int allocated = 0, have_solution = 0, dirty = 1, verbose = 0;
    double vlo = 0, vhi = 0;
    long long pcg_its = 0, bicg_its = 0, newton_its = 0, gummel_its = 0;
    double t_pois = 0, t_cont = 0, t_mob = 0, t_cur = 0, t_aa = 0, t_mg = 0;
    double ii_err = 0;           // impact ionisation: estimated remaining change of the generated current (A)
    double pcg_rtol = 1e-3, ntol_fac = 0.1, bicg_rtol = 1e-4, cont_atol_f = 1;
    int nthreads = 1, caxis = 1, models = 7;
    std::vector<int> trq_k, trq_s;        // trap requests (api3_trap_add): node, species, density
    std::vector<double> trq_N;
    int n_tr = 0;                         // compiled trap entries of the last prepare
    int unstr = 0;                        // a general (graph) mesh instead of the tensor grid
    GraphHost ggh;
    double Cref = 0;
    int ref_mat = 0;
    double Ve1[NC_MAX] = {0}, Ve2[NC_MAX] = {0}, Ve3[NC_MAX] = {0};
    int e_n = 0;
    int aa_m = 0, aa_n = 0, aa_pos = 0, aa_have = 0;
    int precision = -1;               // linear solves: 0 FP64, 1 FP32 refined in FP64, -1 library default
    long long ir_steps = 0, ir_fallbacks = 0;
    Tune tune;
    int pblocks = 0;             // grid share of its persistent solves (api3b_set_share; 0: none)
    unsigned long long upload_gen = 0;      // set-up upload this instance's device holds (prepare)
    const Inst *clone_src = nullptr;        // batched-resolve worker: the instance and upload
    unsigned long long clone_gen = 0;       //   generation its set-up was copied from
    int seed_on = 0;                  // learned sweep predictor enabled (needs a loaded model)
    long long seed_used = 0, seed_fallbacks = 0;
    // ---- derived by prepare (host copies)
    std::vector<uint32_t> flags;
    std::vector<double> bgn, robA, mu0n, mu0p;
    std::vector<int> cnode;
    int n_rob = 0;
    // ---- device
    Gpu g;
    // host mirrors of device results for the getters (valid while `mirror_ok`)
    std::vector<std::vector<double>> cache;
    std::vector<int> cache_ok;
    // terminal partition of the quasi-static charges; trap species table
    std::vector<int> qown;
    int qct[NC_MAX] = {0};
    TrapSpec tsp[512];
    int n_tsp = 0;
};

// global knobs (the reference's static tunables, read by api3_init)
struct Knobs {
    double mg_alpha = 1.0;
    int gpass = 3;               // graph multigrid: rounds of pairwise matching per level
    double gbeta = 0.5;          //   and the strength threshold of a match
    int aa_depth = AA_MAX;
    int pred_on = 1;
    int pred_order = 1;          // sweep predictor: 1 secant (the reference's), 2 quadratic through three points
    double grow_slow = 2.2;
    double cont_atol = 2e-14;
    double qf_margin = 0.0;
    int te_colvs = 1;            // metal contacts: velocity saturation tapered over the column (0: first edge only)
    int check_every = 1;        // Krylov iterations queued between status reads
};
extern Knobs g_knobs;
extern bool g_use_graphs;           // Krylov loops as device-looped CUDA graphs (SEMISIM_B200_GRAPHS=0: off)
extern std::atomic<int> g_stop;
extern volatile double g_prog[8];

// solver entry points (solver.cpp)
bool gpu_available();
int select_device(int dev);
int prepare(Inst &d);
int equilibrium(Inst &d);
int run_continuation(Inst &d);
int do_solve(Inst &d, int keep);
void finish_point(Inst &d);
void set_vrange(Inst &d, const double *Va);
void upload_voltages(Inst &d, const double *Va);
void apply_bc(Inst &d, const double *Va);
void clamp_qf(Inst &d);
void rebuild_np(Inst &d);
void upd_mob(Inst &d);
void terminal_currents(Inst &d, double *I, double *S);
Ctx make_ctx(Inst &d);
int use_mixed(const Inst &d);
int seed_available(const Inst &d);                       // learned.cu
void launch_mlp_seed(Inst &d, double s, const double *dv);
extern int g_precision_default;                          // precision of new instances (1 = refined FP32)
// general (graph) meshes (graph.cu)
void launch_poisson_g(const Ctx &c, const double *phi_sel, int build);
void launch_upd_mob_g(const Ctx &c);
void launch_cont_assemble_g(const Ctx &c, int hole);
void launch_currents_g(const Ctx &c);
void launch_upd_J_g(const Ctx &c);
void launch_mob_display_g(const Ctx &c);
void launch_node_Jc_g(const Ctx &c, int which, double *out);
void launch_emax_g(const Ctx &c);
int pcg_graph(Inst &d, int maxit, double rtol);
int bicg_graph(Inst &d, int maxit, double rtol, double atol, double *rn, double *r0, int qsign, bool ilu_only);
int persist_graph(Inst &d, int kind, int maxit, double rtol, double atol, const double *w, bool ilu_only);
// aggregation multigrid of a graph mesh (graph_mg.cu)
int gmg_build(Inst &d, cudaStream_t st);
void gmg_free(Inst &d);
void gmg_setup(Inst &d, const Ctx &c, int qsign, const double *w);
void gmg_apply(Inst &d, const Ctx &c, const double *r, double *z, const double *w, bool ilu_only);
int gmg_levels(const Inst &d);
int ff_label_g(Inst &d, int *changed);
void ff_boundary_g(Inst &d, int hole, unsigned long long *Aout, unsigned long long *Bin);   // exact accumulators
void region_grow_g(Inst &d, int c1, int type, int *mark, int *changed);
void launch_region_mark_g(Inst &d, int c1, int type, double dV, int *mark, int *changed);
// thermionic-emission metal contacts (metal.cu) and gate tunnelling (tunnel.cu)
void te_update(Inst &d);
void te_currents(Inst &d);
void tun_update(Inst &d);
void tun_currents(Inst &d);
void tun_display(Inst &d);
void exchange_scatter(Inst &d, int hole);   // continuity sink / source of both
void mat_to_dev(const Material &m, MatD &o);
void mat_prepare(Inst &d);                 // gauge Cref and the effective band densities
double tun_eval_host(const MatD *mats, int smat, int nl, const int *mat, const double *t, double psi, double phin,
                     double phip, double Vg, double pm, double Cref, double *out);
double lombardi_host(const MatD &m, double mub, double F, double Nt, double Dw, int hole);
double coulomb_inv_host(const MatD &m, double F, double n, double NC, double NA);
double mlda_factor_host(const Material &m, double a, double b, int hole);
// per-point output reductions on the device (outputs.cu)
double out_emax(Inst &d);
void out_carrier_sums(Inst &d, double *out);
double out_ins_field(Inst &d, long long *node);
int out_terminal_charges(Inst &d, const int *owner_dev, int nt, const int *gate_term, double *out);
void gpu_free(Inst &d);
int batch_pool_release(const Inst *src);   // frees the batched-resolve workers of src (batch.cpp)

// linear-algebra drivers (kernels_la.cu)
void mg_setup(const Ctx &c, const MGHost &mg, int qsign);
void vcycle(const Ctx &c, const MGHost &mg, int bsel, int xsel, int wsel, int mg_on, int gate);
// mixed = 1: FP32 inner solves (FP32 hierarchy and Krylov vectors) refined in FP64
int pcg_solve(const Ctx &c, const MGHost &mg, int maxit, double rtol, int check_every, int mixed = 0);
// persistent (one cooperative launch per solve) forms, kernels_persist.cu: 1 done, 0 not
// applicable, -1 abandoned (the caller restores the start and solves per pass)
int persist_enabled();
void persist_set(int mode, int blocks);
int persist_get_blocks();
int persist_thread_blocks(int n);
int persist_pcg(const Ctx &c, const MGHost &mg, int mixed);
int persist_bicg(const Ctx &c, const MGHost &mg, double rtol, double atol, int qsign);
int persist_refined(const Ctx &c, const MGHost &mg, int maxsteps, int *steps, int qsign);
void vcycle_knobs_init();
int persist_timeout_probe(const Ctx &c, int nb, double wait_s, int *gave_up);
int persist_trace(int n, unsigned long long *out, int *blocks);
extern int g_l0_sweeps, g_deep_levels;
int bicgstab_core(const Ctx &c, const MGHost &mg, int maxit, double rtol, double atol, int mg_on, int check_every,
                  double *rn, double *r0, int qsign, int mixed = 0);
extern thread_local long long t_ir_steps, t_ir_fallbacks;   // refinement steps / FP64 take-overs
extern double g_ir_factor, g_ir_rtol_min;
void launch_absmax_sel(const Ctx &c, int xsel, int slot);
void launch_axpy_sel(const Ctx &c, int ysel, int xsel, double a, int zsel);
void launch_fill_sel(const Ctx &c, int ysel, double v);
void launch_copy_sel(const Ctx &c, int ysel, int xsel);

// Anderson (kernels_aa.cu)
void aa_update_history(const Ctx &c, int slot, int nfill);
void aa_store_fg(const Ctx &c);
void aa_solve_mix(const Ctx &c, int m, int *ok_host);

}  // namespace ss
