// The C ABI of the solver library: the reference core's 89 api3_* entry points
// (semiconductor_3d.c:4567-5353) with identical signatures and semantics on the
// reference's single global device, plus one additive entry (api3_set_mat_mobility)
// and the b200x_* kernel-level test hooks.
//
// The solve path runs on the GPU (solver.cpp and the .cu kernels); there is no CPU
// fallback: without a CUDA device every solve returns 0 with a message on stderr.
// Set-up calls only record the device description, so they work without a GPU.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "prof.h"
#include "solver_ctx.h"

using namespace ss;

namespace {

// Instances: 0 is the reference ABI's single global device (semiconductor_3d.c:366);
// api3b_new adds more.  Every api3_* call acts on the calling thread's current
// instance (api3b_use), so independent devices can be solved from several host threads
// at once, each on its own CUDA stream.
Inst g_dev0;
std::mutex g_reg_mu;
std::vector<std::unique_ptr<Inst>> g_reg;       // g_reg[h-1] = instance h
thread_local Inst *t_cur = nullptr;
Inst &ss_cur() { return t_cur ? *t_cur : g_dev0; }

}  // namespace
#define g_dev (ss_cur())
#define g_qown (g_dev.qown)
#define g_qct (g_dev.qct)
#define g_n_trap_species (g_dev.n_tsp)
#define g_tsp (g_dev.tsp)
namespace {

const char *env_get(const char *n) { return std::getenv(n); }

void mark_changed(Inst &d) { d.dirty = 1; d.have_solution = 0; }

double fv_len(const std::vector<double> &c, int i) {   // semiconductor_3d.c:700-705
    const int N = (int)c.size();
    if (N < 2) return 1.;
    if (i == 0) return 0.5 * (c[1] - c[0]);
    if (i == N - 1) return 0.5 * (c[N - 1] - c[N - 2]);
    return 0.5 * (c[i + 1] - c[i - 1]);
}

double nanv() { return std::nan(""); }

// host mirror of one derived node quantity (api3_bulk_copy semantics)
const std::vector<double> *node_vals(Inst &d, int which) {
    if (!d.allocated || !d.have_solution || !d.g.ready || which < 0 || which > 35) return nullptr;
    if (d.cache.size() < 36) { d.cache.assign(36, {}); d.cache_ok.assign(36, 0); }
    if (!d.cache_ok[which]) {
        Ctx c = make_ctx(d);
        if (d.unstr && which >= 20 && which <= 25) launch_node_Jc_g(c, which, d.g.scratch);   // least squares
        else launch_node_val(c, which, d.g.scratch);
        d.cache[which].resize(d.N);
        cudaMemcpyAsync(d.cache[which].data(), d.g.scratch, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
        cudaStreamSynchronize(d.g.st);
        d.cache_ok[which] = 1;
    }
    return &d.cache[which];
}
double node_val1(int which, int k) {
    Inst &d = g_dev;
    if (k < 0 || (size_t)k >= d.N) return nanv();
    const std::vector<double> *v = node_vals(d, which);
    return v ? (*v)[k] : nanv();
}
void invalidate(Inst &d) { for (auto &v : d.cache_ok) v = 0; }

int kind_of(const Inst &d, size_t k) { return fl_kind(d.flags[k]); }
int con_of(const Inst &d, size_t k) { return fl_con(d.flags[k]); }

// neighbours with their Poisson coupling eps A / h and spacing (semiconductor_3d.c:5166-5186)
int qnbrs(const Inst &d, size_t k, size_t *nb, double *cf, double *hh) {
    if (d.unstr) {                                  // the graph's edges, in CSR order (at most 64)
        const GraphHost &G = d.ggh;
        const double ek = d.mats[d.mat_idx[k]].eps_r * EPS0;
        int m = 0;
        for (int e = G.rp[k]; e < G.rp[k + 1] && m < 64; e++) {
            const size_t kb = (size_t)G.cj[e];
            const double eb = d.mats[d.mat_idx[kb]].eps_r * EPS0;
            nb[m] = kb; cf[m] = (2. * ek * eb / (ek + eb)) * G.ar[e] / G.h[e]; hh[m] = G.h[e]; m++;
        }
        return m;
    }
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const int l = int(k / ((size_t)Nx * Ny)), rem = int(k - (size_t)l * Nx * Ny), j = rem / Nx, i = rem % Nx;
    int m = 0;
    const double ek = d.mats[d.mat_idx[k]].eps_r * EPS0;
    for (int dir = 0; dir < 6; dir++) {
        int ii = i, jj = j, ll = l;
        double h, ar;
        switch (dir) {
        case 0: if (i == 0) continue; ii = i - 1; h = d.xs[i] - d.xs[i - 1]; ar = d.Ly[j] * d.Lz[l]; break;
        case 1: if (i == Nx - 1) continue; ii = i + 1; h = d.xs[i + 1] - d.xs[i]; ar = d.Ly[j] * d.Lz[l]; break;
        case 2: if (j == 0) continue; jj = j - 1; h = d.ys[j] - d.ys[j - 1]; ar = d.Lx[i] * d.Lz[l]; break;
        case 3: if (j == Ny - 1) continue; jj = j + 1; h = d.ys[j + 1] - d.ys[j]; ar = d.Lx[i] * d.Lz[l]; break;
        case 4: if (l == 0) continue; ll = l - 1; h = d.zs[l] - d.zs[l - 1]; ar = d.Lx[i] * d.Ly[j]; break;
        default: if (l == Nz - 1) continue; ll = l + 1; h = d.zs[l + 1] - d.zs[l]; ar = d.Lx[i] * d.Ly[j]; break;
        }
        const size_t kb = (size_t)ll * Nx * Ny + (size_t)jj * Nx + ii;
        const double eb = d.mats[d.mat_idx[kb]].eps_r * EPS0;
        nb[m] = kb; cf[m] = (2. * ek * eb / (ek + eb)) * ar / h; hh[m] = h; m++;
    }
    return m;
}

}  // namespace

// the calling thread's current instance, for the test hooks
Inst *b200_global_dev() { return &g_dev; }

extern "C" {

// ------------------------------------------------------------------ set-up
void api3_init(void) {                                      // semiconductor_3d.c:4570-4597
    Gpu keep = g_dev.g;                                     // device buffers are reused when the size allows
    const int prec = g_dev.precision;                       // so are the instance's solver precision
    const int share = g_dev.pblocks;                        // and its grid share
    g_dev.g = Gpu();
    g_dev = Inst();
    g_dev.g = keep;
    g_dev.precision = prec;
    g_dev.pblocks = share;
    g_dev.g.ready = keep.ready;
    Inst &d = g_dev;
    const char *e = env_get("SEMISIM_PCGRTOL"); d.pcg_rtol = e ? std::atof(e) : 1e-3;
    const char *f = env_get("SEMISIM_NTOLF"); d.ntol_fac = f ? std::atof(f) : 0.1;
    const char *g = env_get("SEMISIM_BRTOL"); d.bicg_rtol = g ? std::atof(g) : 1e-4;
    d.cont_atol_f = 1.;
    d.models = 7;
    d.caxis = 1;
    const char *v = env_get("SEMISIM_VERBOSE"); d.verbose = v ? std::atoi(v) : 0;
    const char *a = env_get("SEMISIM_MGA"); if (a) g_knobs.mg_alpha = std::atof(a);
    if (const char *m = env_get("SEMISIM_GPASS")) g_knobs.gpass = std::atoi(m);
    if (const char *m = env_get("SEMISIM_GBETA")) g_knobs.gbeta = std::atof(m);
    if (const char *m = env_get("SEMISIM_AAM")) { int q = std::atoi(m); g_knobs.aa_depth = q < 0 ? 0 : (q > AA_MAX ? AA_MAX : q); }
    if (const char *m = env_get("SEMISIM_PRED")) g_knobs.pred_on = std::atoi(m) != 0;
    if (const char *m = env_get("SEMISIM_B200_PRED_ORDER")) g_knobs.pred_order = std::atoi(m) >= 2 ? 2 : 1;
    if (const char *m = env_get("SEMISIM_GROW")) { const double gg = std::atof(m); if (gg >= 1. && gg <= 4.) g_knobs.grow_slow = gg; }
    if (const char *m = env_get("SEMISIM_CATOL")) g_knobs.cont_atol = std::atof(m);
    if (const char *m = env_get("SEMISIM_QFM")) g_knobs.qf_margin = std::atof(m);
    if (const char *m = env_get("SEMISIM_TECOLVS")) g_knobs.te_colvs = std::atoi(m);
    if (const char *m = env_get("SEMISIM_B200_CHECK")) { const int q = std::atoi(m); if (q >= 1 && q <= 64) g_knobs.check_every = q; }
    if (const char *m = env_get("SEMISIM_B200_GRAPHS")) g_use_graphs = std::atoi(m) != 0;
    if (const char *m = env_get("SEMISIM_B200_PDL")) g_pdl = std::atoi(m) != 0;
    if (const char *m = env_get("SEMISIM_B200_PRECISION"))
        g_precision_default = (!std::strcmp(m, "mixed") || !std::strcmp(m, "refined") || !std::strcmp(m, "1")) ? 1 : 0;
    if (const char *m = env_get("SEMISIM_B200_IR_FACTOR")) { const double q = std::atof(m); if (q > 0. && q <= 1.) g_ir_factor = q; }
    if (const char *m = env_get("SEMISIM_B200_IR_RTOL")) { const double q = std::atof(m); if (q > 0. && q < 1.) g_ir_rtol_min = q; }
    g_n_trap_species = 0;
}

void api3_set_threads(int n) { g_dev.nthreads = n < 1 ? 1 : n; }   // host threads play no part in the solve
void api3_set_verbose(int v) { g_dev.verbose = v; }

int api3_trap_species(int type, int ref, double E, double sn, double sp) {
    for (int s = 0; s < g_n_trap_species; s++) {
        const TrapSpec &t = g_tsp[s];
        if (t.type == type && t.ref == ref && t.E == E && t.sn == sn && t.sp == sp) return s;
    }
    if (g_n_trap_species >= 512 || !(sn >= 0.) || !(sp >= 0.)) return -1;
    TrapSpec &t = g_tsp[g_n_trap_species];
    t.type = type < 0 ? -1 : (type > 0 ? 1 : 0); t.ref = ref < 0 || ref > 2 ? 2 : ref; t.E = E; t.sn = sn; t.sp = sp;
    return g_n_trap_species++;
}
int api3_trap_add(int sid, int n, const int *nodes, const double *dens) {   // semiconductor_3d.c:4629-4644
    Inst &d = g_dev;
    if (sid < 0 || sid >= g_n_trap_species || n <= 0) return 0;
    for (int q = 0; q < n; q++) {
        if (!(dens[q] > 0.)) continue;
        d.trq_k.push_back(nodes[q]); d.trq_s.push_back(sid); d.trq_N.push_back(dens[q]);
    }
    mark_changed(d);
    return 1;
}
void api3_traps_clear(void) {                                  // semiconductor_3d.c:4645
    Inst &d = g_dev;
    d.trq_k.clear(); d.trq_s.clear(); d.trq_N.clear();
    d.n_tr = 0;
    g_n_trap_species = 0;
    mark_changed(d);
}
int api3_charge_add(int n, const int *nodes, const double *rho) {
    Inst &d = g_dev;
    if (!d.allocated) return 0;
    for (int q = 0; q < n; q++) {
        const size_t k = (size_t)nodes[q];
        if (k < d.N) d.Nf[k] += rho[q];
    }
    mark_changed(d);
    return 1;
}
int api3_n_trap_entries(void) { return g_dev.n_tr; }
void api3_set_models(int flags) { g_dev.models = flags; g_dev.have_solution = 0; g_dev.dirty = 1; }
void api3_set_caxis(int ax) { g_dev.caxis = (ax >= 0 && ax <= 2) ? ax : -1; g_dev.have_solution = 0; g_dev.dirty = 1; }
int api3_get_caxis(void) { return g_dev.caxis; }

int api3_add_material(int id, double T) {
    Inst &d = g_dev;
    if (d.n_mats >= NM_MAX) return -1;
    material_init(d.mats[d.n_mats], id, T);
    mark_changed(d);
    return d.n_mats++;
}
int api3_set_mat_tau(int mi, double tn, double tp) {
    Inst &d = g_dev;
    if (mi < 0 || mi >= d.n_mats) return 0;
    d.mats[mi].tau_n0 = tn > 0. ? tn : 1e30;
    d.mats[mi].tau_p0 = tp > 0. ? tp : 1e30;
    mark_changed(d);
    return 1;
}
// Additive entry (no counterpart in the reference): pin the low-field mobility of
// material mi to constants mun / mup (m^2/Vs), independent of doping and temperature.
int api3_set_mat_mobility(int mi, double mun, double mup) {
    Inst &d = g_dev;
    if (mi < 0 || mi >= d.n_mats || !(mun > 0.) || !(mup > 0.)) return 0;
    Material &m = d.mats[mi];
    m.mas_on = 0;
    m.mu_n_min = m.mu_n_max = mun;
    m.mu_p_min = m.mu_p_max = mup;
    m.mt_min = m.mt_max_n = m.mt_max_p = 0.;
    mark_changed(d);
    return 1;
}

int api3_set_grid_coords(int Nx, int Ny, int Nz, const double *xs, const double *ys, const double *zs) {
    for (int i = 1; i < Nx; i++) if (!(xs[i] > xs[i - 1])) return 0;
    for (int j = 1; j < Ny; j++) if (!(ys[j] > ys[j - 1])) return 0;
    for (int l = 1; l < Nz; l++) if (!(zs[l] > zs[l - 1])) return 0;
    Inst &d = g_dev;
    if (Nx < 2 || Ny < 2 || Nz < 2) return 0;
    const size_t N = (size_t)Nx * Ny * Nz;
    if (N > 2000000000ULL) return 0;
    d.unstr = 0;
    d.ggh = GraphHost();
    d.Nx = Nx; d.Ny = Ny; d.Nz = Nz; d.N = N;
    d.xs.assign(xs, xs + Nx); d.ys.assign(ys, ys + Ny); d.zs.assign(zs, zs + Nz);
    d.Lx.resize(Nx); d.Ly.resize(Ny); d.Lz.resize(Nz);
    for (int i = 0; i < Nx; i++) d.Lx[i] = fv_len(d.xs, i);
    for (int j = 0; j < Ny; j++) d.Ly[j] = fv_len(d.ys, j);
    for (int l = 0; l < Nz; l++) d.Lz[l] = fv_len(d.zs, l);
    d.mat_idx.assign(N, 0);
    d.Nd.assign(N, 0.0); d.Na.assign(N, 0.0); d.Nf.assign(N, 0.0);
    d.flags.assign(N, 0);
    d.allocated = 1; d.have_solution = 0; d.dirty = 1;
    d.aa_m = AA_MAX;
    invalidate(d);
    return 1;
}
void api3_set_grid(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz) {
    if (Nx < 2) Nx = 2; if (Ny < 2) Ny = 2; if (Nz < 2) Nz = 2;
    std::vector<double> xs(Nx), ys(Ny), zs(Nz);
    for (int i = 0; i < Nx; i++) xs[i] = i * Lx / (Nx - 1.);
    for (int j = 0; j < Ny; j++) ys[j] = j * Ly / (Ny - 1.);
    for (int l = 0; l < Nz; l++) zs[l] = l * Lz / (Nz - 1.);
    (void)api3_set_grid_coords(Nx, Ny, Nz, xs.data(), ys.data(), zs.data());
}
void api3_set_solver(int mp, int mc, int mg, double tp, double tc, double op, double oc) {
    Inst &d = g_dev;
    d.max_iter_p = mp; d.max_iter_c = mc; d.max_gummel = mg;
    d.tol_p = tp; d.tol_c = tc; d.omega_p = op; d.omega_c = oc;
}
static void clip_box(int *x0, int *y0, int *z0, int *x1, int *y1, int *z1) {
    const Inst &d = g_dev;
    if (*x0 < 0) *x0 = 0; if (*y0 < 0) *y0 = 0; if (*z0 < 0) *z0 = 0;
    if (*x1 >= d.Nx) *x1 = d.Nx - 1; if (*y1 >= d.Ny) *y1 = d.Ny - 1; if (*z1 >= d.Nz) *z1 = d.Nz - 1;
}
void api3_set_region(int x0, int y0, int z0, int x1, int y1, int z1, int midx, double Nd, double Na) {
    Inst &d = g_dev;
    if (!d.allocated || midx < 0 || midx >= d.n_mats) return;
    clip_box(&x0, &y0, &z0, &x1, &y1, &z1);
    for (int l = z0; l <= z1; l++)
        for (int j = y0; j <= y1; j++)
            for (int i = x0; i <= x1; i++) {
                const size_t k = (size_t)l * d.Nx * d.Ny + (size_t)j * d.Nx + i;
                d.mat_idx[k] = midx; d.Nd[k] = Nd; d.Na[k] = Na;
                if (d.mats[midx].insulator) d.Nd[k] = d.Na[k] = 0.;
            }
    mark_changed(d);
}
void api3_add_fixed_charge(int x0, int y0, int z0, int x1, int y1, int z1, double Nf) {
    Inst &d = g_dev;
    if (!d.allocated) return;
    clip_box(&x0, &y0, &z0, &x1, &y1, &z1);
    for (int l = z0; l <= z1; l++)
        for (int j = y0; j <= y1; j++)
            for (int i = x0; i <= x1; i++) d.Nf[(size_t)l * d.Nx * d.Ny + (size_t)j * d.Nx + i] += Nf;
    mark_changed(d);
}
void api3_add_sheet_charge(int axis, int idx, int a0, int a1, int b0, int b1, double sigma) {
    Inst &d = g_dev;
    if (!d.allocated) return;
    int x0, x1, y0, y1, z0, z1;
    double L;
    if (axis == 0) { if (idx < 0 || idx >= d.Nx) return; x0 = x1 = idx; y0 = a0; y1 = a1; z0 = b0; z1 = b1; L = d.Lx[idx]; }
    else if (axis == 1) { if (idx < 0 || idx >= d.Ny) return; y0 = y1 = idx; x0 = a0; x1 = a1; z0 = b0; z1 = b1; L = d.Ly[idx]; }
    else { if (idx < 0 || idx >= d.Nz) return; z0 = z1 = idx; x0 = a0; x1 = a1; y0 = b0; y1 = b1; L = d.Lz[idx]; }
    api3_add_fixed_charge(x0, y0, z0, x1, y1, z1, sigma / L);
}
int api3_add_contact_ex(int face, int i0, int i1, int j0, int j1, int k0, int k1, int bc, double V, double pm,
                        double tox, double Nox) {
    Inst &d = g_dev;
    if (d.n_cons >= NC_MAX) return -1;
    Contact &c = d.cons[d.n_cons];
    c = Contact();
    c.face = face < 0 ? 0 : (face > 6 ? 6 : face);
    c.i0 = i0; c.i1 = i1; c.j0 = j0; c.j1 = j1; c.k0 = k0; c.k1 = k1;
    c.bc = bc < 0 ? 0 : (bc > 2 ? 2 : bc); c.V = V; c.phi_m = pm;
    c.tox = tox > 0. ? tox : 10e-9;
    c.qox = Nox * Q;
    d.cnodes[d.n_cons].clear(); d.careas[d.n_cons].clear();
    mark_changed(d);
    return d.n_cons++;
}
void api3_add_contact(int face, int i0, int i1, int j0, int j1, int bc, double V, double pm) {
    (void)api3_add_contact_ex(face, i0, i1, j0, j1, 0, 0, bc, V, pm, 10e-9, 0.);
}
void api3_clear_contacts(void) { g_dev.n_cons = 0; mark_changed(g_dev); }
int api3_set_gate_stack(int cid, int nl, const int *mat, const double *t) {
    Inst &d = g_dev;
    if (cid < 0 || cid >= d.n_cons || nl < 0 || nl > 6) return 0;
    for (int i = 0; i < nl; i++) if (mat[i] < 0 || mat[i] >= d.n_mats || !(t[i] > 0.)) return 0;
    d.cons[cid].snl = nl;             // Robin-gate layer stack of gate tunnelling (semiconductor_3d.c:4776-4787)
    for (int i = 0; i < nl; i++) { d.cons[cid].smat[i] = mat[i]; d.cons[cid].st[i] = t[i]; }
    mark_changed(d);
    return 1;
}
// a device on a general box-method mesh (semiconductor_3d.c:4788-4805, alloc_dev_graph
// :981-1041): N nodes, E directed edges as a symmetric CSR graph, per edge its length and
// dual face area, per node its control volume and position.  Nx = N, Ny = Nz = 1 with the
// volume in Lx, so the node-wise parts of the solver apply unchanged.  Returns 0 for a bad
// graph (not symmetric, self edges, non-positive lengths or volumes).
int api3_set_mesh_graph(int N, int E, const int *rp, const int *cj, const double *h, const double *ar,
                        const double *vol, const double *pos) {
    Inst &d = g_dev;
    if (N < 2 || E < 1 || !rp || !cj || !h || !ar || !vol || !pos || rp[0] != 0 || rp[N] != E) return 0;
    for (int k = 0; k < N; k++) {
        if (rp[k + 1] < rp[k] || !(vol[k] > 0.)) return 0;
        for (int e = rp[k]; e < rp[k + 1]; e++)
            if (cj[e] < 0 || cj[e] >= N || cj[e] == k || !(h[e] > 0.) || !(ar[e] >= 0.)) return 0;
    }
    GraphHost G;
    G.rp.assign(rp, rp + N + 1); G.cj.assign(cj, cj + E);
    G.h.assign(h, h + E); G.ar.assign(ar, ar + E);
    G.vol.assign(vol, vol + N); G.pos.assign(pos, pos + 3 * (size_t)N);
    G.rev.assign(E, -1); G.ue.assign(E, -1);
    for (int k = 0; k < N; k++)
        for (int e = rp[k]; e < rp[k + 1]; e++) {       // reverse entries and undirected ids
            const int j = cj[e];
            int r = -1;
            for (int t = rp[j]; t < rp[j + 1]; t++) if (cj[t] == k) { r = t; break; }
            if (r < 0) return 0;
            G.rev[e] = r;
            if (k < j) G.ue[e] = G.nue++;
        }
    for (int k = 0; k < N; k++)
        for (int e = rp[k]; e < rp[k + 1]; e++) if (cj[e] < k) G.ue[e] = G.ue[G.rev[e]];
    G.wall.assign(6 * (size_t)N, 1.);
    d.unstr = 1;
    d.ggh = std::move(G);
    d.Nx = N; d.Ny = 1; d.Nz = 1; d.N = (size_t)N;
    d.xs.assign(N, 0.); d.Lx.assign(vol, vol + N);
    for (int k = 0; k < N; k++) d.xs[k] = pos[3 * k];
    d.ys.assign(1, 0.); d.zs.assign(1, 0.); d.Ly.assign(1, 1.); d.Lz.assign(1, 1.);
    d.mat_idx.assign(N, 0);
    d.Nd.assign(N, 0.0); d.Na.assign(N, 0.0); d.Nf.assign(N, 0.0);
    d.flags.assign(N, 0);
    d.allocated = 1; d.have_solution = 0; d.dirty = 1;
    d.aa_m = AA_MAX;
    invalidate(d);
    // the continuity solves of a general mesh stop at 1e-6 unless SEMISIM_BRTOL says otherwise
    if (!env_get("SEMISIM_BRTOL")) d.bicg_rtol = 1e-6;
    return 1;
}
int api3_is_graph(void) { return g_dev.unstr; }
void api3_set_node_data(const int *mat, const double *Nd, const double *Na, const double *Nf) {
    Inst &d = g_dev;
    if (!d.allocated) return;
    for (size_t k = 0; k < d.N; k++) {
        int mi = mat[k];
        if (mi < 0 || mi >= d.n_mats) mi = 0;
        d.mat_idx[k] = mi;
        const int ins = d.mats[mi].insulator;
        d.Nd[k] = ins ? 0. : Nd[k]; d.Na[k] = ins ? 0. : Na[k]; d.Nf[k] = Nf ? Nf[k] : 0.;
    }
    mark_changed(d);
}
int api3_set_con_nodes(int cid, int n, const int *nodes, const double *areas) {
    Inst &d = g_dev;
    if (cid < 0 || cid >= d.n_cons || n < 0) return 0;
    d.cnodes[cid].clear(); d.careas[cid].clear();
    if (n == 0) return 1;
    for (int q = 0; q < n; q++) {
        if (nodes[q] < 0 || (size_t)nodes[q] >= d.N) { d.cnodes[cid].clear(); d.careas[cid].clear(); return 0; }
        d.cnodes[cid].push_back(nodes[q]);
        d.careas[cid].push_back(areas ? areas[q] : 0.);
    }
    mark_changed(d);
    return 1;
}
// the interface walls of a graph device: per node two walls, each the node's distance to it
// and the range a..b of its cell measured from it; a distance >= 0.5 m is no wall
// (semiconductor_3d.c:4835-4841)
void api3_set_walls(const double *w) {
    Inst &d = g_dev;
    if (!d.allocated || !d.unstr || !w) return;
    d.ggh.wall.assign(w, w + 6 * d.N);
    mark_changed(d);
}
int api3_get_ntp(int cid) {                                  // semiconductor_3d.c:4844-4847
    Inst &d = g_dev;
    if (cid < 0) {
        int n = 0;
        for (int c = 0; c < d.n_cons; c++) n += d.cons[c].ntp;
        return n;
    }
    return cid < d.n_cons ? d.cons[cid].ntp : 0;
}
double api3_tun_eval(int smat, int nl, const int *mat, const double *t, double psi, double phin, double phip,
                     double Vg, double pm, double *out) {      // semiconductor_3d.c:4855-4868
    Inst &d = g_dev;
    if (smat < 0 || smat >= d.n_mats || nl < 1 || nl > 6) return 0.;
    for (int i = 0; i < nl; i++) if (mat[i] < 0 || mat[i] >= d.n_mats) return 0.;
    mat_prepare(d);
    MatD md[NM_MAX];
    for (int i = 0; i < d.n_mats; i++) mat_to_dev(d.mats[i], md[i]);
    return tun_eval_host(md, smat, nl, mat, t, psi, phin, phip, Vg, pm, d.Cref, out);
}
double api3_mlda_factor(int mi, double a, double b, int hole) {   // semiconductor_3d.c:4869-4872
    if (mi < 0 || mi >= g_dev.n_mats) return 1.;
    return mlda_factor_host(g_dev.mats[mi], a, b, hole);
}
double api3_coulomb_inv(int mi, double F, double n, double NC, double NA) {   // semiconductor_3d.c:4878-4881
    if (mi < 0 || mi >= g_dev.n_mats || !g_dev.mats[mi].lbc_on) return nanv();
    MatD md;
    mat_to_dev(g_dev.mats[mi], md);
    return coulomb_inv_host(md, F, n, NC, NA);
}
int api3_set_surface_mobility(int mi, double delta, double eta, double mu1) {   // semiconductor_3d.c:4885-4893
    Inst &d = g_dev;
    if (mi < 0 || mi >= d.n_mats) return 0;
    Material &m = d.mats[mi];
    if (delta > 0.) m.lbD[0] = delta;
    if (eta > 0.) m.lbE[0] = eta;
    if (mu1 > 0.) m.lbc_mu1 = mu1;
    mark_changed(d);
    d.have_solution = 0;
    return 1;
}
double api3_lombardi(int mi, double mub, double F, double Nt, double Dw, int hole) {   // semiconductor_3d.c:4894-4897
    if (mi < 0 || mi >= g_dev.n_mats) return mub;
    MatD md;
    mat_to_dev(g_dev.mats[mi], md);
    return lombardi_host(md, mub, F, Nt, Dw, hole);
}
void api3_set_contact_V(int cid, double V) { if (cid >= 0 && cid < g_dev.n_cons) g_dev.cons[cid].V = V; }
int api3_get_ncon(void) { return g_dev.n_cons; }
double api3_get_contact_I(int cid) { return (cid >= 0 && cid < g_dev.n_cons) ? g_dev.cons[cid].I : 0.; }
double api3_get_contact_A(int cid) { return (cid >= 0 && cid < g_dev.n_cons) ? g_dev.cons[cid].A : 0.; }
double api3_get_contact_In(int cid) { return (cid >= 0 && cid < g_dev.n_cons) ? g_dev.cons[cid].In : 0.; }
double api3_get_contact_Ifloor(int cid) { return (cid >= 0 && cid < g_dev.n_cons) ? g_dev.cons[cid].Iflr : 0.; }
double api3_get_contact_Iraw(int cid) { return (cid >= 0 && cid < g_dev.n_cons) ? g_dev.cons[cid].Iraw : 0.; }
int api3_get_aa_depth(void) { return g_dev.aa_m < g_knobs.aa_depth ? g_dev.aa_m : g_knobs.aa_depth; }
double api3_get_contact_Vsolved(int cid) { return (cid >= 0 && cid < g_dev.n_cons) ? g_dev.cons[cid].Vprev : 0.; }

// ------------------------------------------------------------------ solve
void api3_request_stop(void) { g_stop.store(1); }
void api3_clear_stop(void) { g_stop.store(0); }
int api3_stop_requested(void) { return g_stop.load(); }
void api3_get_progress(double *out) { for (int i = 0; i < 8; i++) out[i] = g_prog[i]; }
int api3_solve(void) { return do_solve(g_dev, 0); }
int api3_resolve(void) { return do_solve(g_dev, 1); }

void api3_iv_sweep(int cid, double Vs, double Ve, int Npts, double *Varr, double *Jarr, int *Carr) {
    Inst &d = g_dev;
    if (cid < 0 || cid >= d.n_cons) return;
    if (Npts < 1) Npts = 1;
    if (Npts > 400) Npts = 400;
    const double dV = (Npts > 1) ? (Ve - Vs) / (Npts - 1.) : 0.;
    const double V0 = d.cons[cid].V;
    if (!prepare(d)) return;
    if (!d.have_solution) equilibrium(d);
    for (int kk = 0; kk < Npts; kk++) {
        const double V = Vs + kk * dV;
        if (g_stop.load()) { Varr[kk] = nanv(); Jarr[kk] = nanv(); Carr[kk] = -1; continue; }
        d.cons[cid].V = V;
        const int ok = run_continuation(d);
        const double A = d.cons[cid].A;
        Varr[kk] = d.cons[cid].Vprev;
        Jarr[kk] = A > 0. ? d.cons[cid].I / A : d.cons[cid].I;
        Carr[kk] = ok;
    }
    finish_point(d);
    g_prog[4] = 0.;
    d.cons[cid].V = V0;
}
void api3_iv_sweep2(int cid, double Vs, double Ve, int Npts, double *Varr, double *Iarr, double *Farr, int *Carr) {
    Inst &d = g_dev;
    if (cid < 0 || cid >= d.n_cons) return;
    if (Npts < 1) Npts = 1;
    if (Npts > 400) Npts = 400;
    const double dV = (Npts > 1) ? (Ve - Vs) / (Npts - 1.) : 0.;
    const double V0 = d.cons[cid].V;
    const int nc = d.n_cons;
    if (!prepare(d)) return;
    if (!d.have_solution) equilibrium(d);
    for (int kk = 0; kk < Npts; kk++) {
        if (g_stop.load()) {
            Varr[kk] = nanv(); Carr[kk] = -1;
            for (int c = 0; c < nc; c++) { Iarr[kk * nc + c] = nanv(); Farr[kk * nc + c] = nanv(); }
            continue;
        }
        d.cons[cid].V = Vs + kk * dV;
        const int ok = run_continuation(d);
        Varr[kk] = d.cons[cid].Vprev;
        for (int c = 0; c < nc; c++) { Iarr[kk * nc + c] = d.cons[c].I; Farr[kk * nc + c] = d.cons[c].Iflr; }
        Carr[kk] = ok;
    }
    finish_point(d);
    g_prog[4] = 0.;
    d.cons[cid].V = V0;
}

// ------------------------------------------------------------------ getters
double api3_get_Emax(void) {                                // semiconductor_3d.c:4981-5001
    Inst &d = g_dev;
    if (!d.allocated || !d.have_solution || !d.g.ready) return 0.;
    return out_emax(d);
}
int api3_get_Nx(void) { return g_dev.Nx; }
int api3_get_Ny(void) { return g_dev.Ny; }
int api3_get_Nz(void) { return g_dev.Nz; }
int api3_get_conv(void) { return g_dev.converged; }
int api3_get_iter(void) { return g_dev.conv_iter; }
double api3_get_res(void) { return g_dev.conv_res; }
double api3_get_xs(int i) { return (g_dev.allocated && i >= 0 && i < g_dev.Nx) ? g_dev.xs[i] : nanv(); }
double api3_get_ys(int j) { return (g_dev.allocated && j >= 0 && j < g_dev.Ny) ? g_dev.ys[j] : nanv(); }
double api3_get_zs(int l) { return (g_dev.allocated && l >= 0 && l < g_dev.Nz) ? g_dev.zs[l] : nanv(); }
double api3_get_Cref(void) { return g_dev.Cref; }
long long api3_get_stat(int w) {
    switch (w) {
    case 0: return g_dev.pcg_its;
    case 1: return g_dev.bicg_its;
    case 2: return g_dev.newton_its;
    case 3: return g_dev.gummel_its;
    }
    return 0;
}
void api3_set_predictor(int on) { g_knobs.pred_on = on != 0; }
int api3_get_state(double *phi, double *phin, double *phip) {
    Inst &d = g_dev;
    if (!d.allocated) return 0;
    if (!d.g.ready) {
        for (size_t k = 0; k < d.N; k++) phi[k] = phin[k] = phip[k] = 0.;
        return d.have_solution;
    }
    cudaMemcpyAsync(phi, d.g.h.phi, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    cudaMemcpyAsync(phin, d.g.h.phin, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    cudaMemcpyAsync(phip, d.g.h.phip, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    cudaStreamSynchronize(d.g.st);
    return d.have_solution;
}
int api3_set_state(const double *phi, const double *phin, const double *phip) {   // semiconductor_3d.c:5030-5041
    Inst &d = g_dev;
    if (!prepare(d)) return 0;
    if (!d.have_solution) equilibrium(d);
    double Va[NC_MAX];
    cudaMemcpyAsync(d.g.h.phi, phi, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    cudaMemcpyAsync(d.g.h.phin, phin, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    cudaMemcpyAsync(d.g.h.phip, phip, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    for (int c = 0; c < d.n_cons; c++) { Va[c] = d.cons[c].V; d.cons[c].Vprev = Va[c]; }
    set_vrange(d, Va);
    apply_bc(d, Va);
    clamp_qf(d);
    rebuild_np(d);
    upd_mob(d);
    cudaStreamSynchronize(d.g.st);
    d.have_solution = 1;
    d.e_n = 0;
    invalidate(d);
    return 1;
}
double api3_get_time(int w) {
    switch (w) {
    case 0: return g_dev.t_pois;
    case 1: return g_dev.t_cont;
    case 2: return g_dev.t_mob;
    case 3: return g_dev.t_cur;
    case 4: return g_dev.t_aa;
    case 5: return g_dev.t_mg;
    }
    return 0.;
}
double api3_mat_ni(int mi) { return (mi >= 0 && mi < g_dev.n_mats) ? g_dev.mats[mi].ni : 0.; }
double api3_mat_Eg(int mi) { return (mi >= 0 && mi < g_dev.n_mats) ? g_dev.mats[mi].Eg : 0.; }

void api3_bulk_copy(int which, double *out) {
    Inst &d = g_dev;
    if (!d.allocated) return;
    const std::vector<double> *v = node_vals(d, which);
    if (!v) {
        const bool sol = d.have_solution && d.g.ready;
        for (size_t k = 0; k < d.N; k++) out[k] = sol ? 0. : nanv();
        return;
    }
    std::memcpy(out, v->data(), d.N * 8);
}
void api3_carrier_sums(double *out) {                       // semiconductor_3d.c:5137-5147
    Inst &d = g_dev;
    out[0] = out[1] = 0.;
    if (!d.allocated || !d.have_solution || !d.g.ready) return;
    out_carrier_sums(d, out);
}

// terminal partition for the quasi-static charges (semiconductor_3d.c:5192-5246)
int api3_charge_partition(const int *cterm) {
    Inst &d = g_dev;
    if (!d.allocated || !d.have_solution || !cterm) return -1;
    const std::vector<double> *n = node_vals(d, 1), *p = node_vals(d, 2);
    if (!n || !p) return -1;
    const size_t N = d.N;
    g_qown.assign(N, -1);
    d.g.qown_ok = false;
    for (int c = 0; c < NC_MAX; c++) g_qct[c] = c < d.n_cons ? cterm[c] : -1;
    auto qtype = [&](size_t k) { return (*n)[k] >= (*p)[k] ? 1 : -1; };
    std::vector<size_t> qu;
    qu.reserve(N);
    size_t qh = 0;
    int meet = 0;
    for (size_t k = 0; k < N; k++) {
        const int c = con_of(d, k) - 1;
        if (c < 0 || c >= d.n_cons) continue;
        const int t = cterm[c];
        g_qown[k] = t;
        if (t >= 0 && d.cons[c].bc == 0 && !d.cons[c].te && (kind_of(d, k) == K_SEMI || kind_of(d, k) == K_METAL))
            qu.push_back(k);
    }
    size_t nb[64]; double cf[64], hh[64];
    while (qh < qu.size()) {
        const size_t k = qu[qh++];
        const int t = g_qown[k];
        const int m = qnbrs(d, k, nb, cf, hh);
        for (int e = 0; e < m; e++) {
            const size_t b = nb[e];
            if (con_of(d, b)) continue;
            const bool ok = kind_of(d, k) == K_METAL ? kind_of(d, b) == K_METAL
                          : (kind_of(d, k) == K_SEMI && kind_of(d, b) == K_SEMI && qtype(b) == qtype(k));
            if (!ok) continue;
            if (g_qown[b] < 0) { g_qown[b] = t; qu.push_back(b); }
            else if (g_qown[b] != t) meet++;
        }
    }
    qu.clear(); qh = 0;
    for (size_t k = 0; k < N; k++) if (g_qown[k] >= 0 && kind_of(d, k) == K_SEMI) qu.push_back(k);
    while (qh < qu.size()) {
        const size_t k = qu[qh++];
        const int t = g_qown[k];
        const int m = qnbrs(d, k, nb, cf, hh);
        for (int e = 0; e < m; e++) {
            const size_t b = nb[e];
            if (con_of(d, b) || kind_of(d, b) != K_SEMI || g_qown[b] >= 0) continue;
            g_qown[b] = t; qu.push_back(b);
        }
    }
    return meet;
}
int api3_terminal_charges(int nt, double *Qt) {             // semiconductor_3d.c:5248-5282
    Inst &d = g_dev;
    const size_t N = d.N;
    if (!d.allocated || !d.have_solution || !d.g.ready || g_qown.size() != N || nt <= 0 || !Qt) return 0;
    // owners only take the contacts' terminal ids: number the ones inside [0, nt) densely
    // (at most NC_MAX), the others count as no terminal, like -1
    int slot[NC_MAX], ids[NC_MAX], m = 0, gate_slot[NC_MAX];
    for (int c = 0; c < NC_MAX; c++) {
        const int t = g_qct[c];
        slot[c] = -1;
        if (t < 0 || t >= nt) continue;
        for (int q = 0; q < m; q++) if (ids[q] == t) slot[c] = q;
        if (slot[c] < 0) { ids[m] = t; slot[c] = m++; }
    }
    for (int c = 0; c < NC_MAX; c++) gate_slot[c] = slot[c];
    if (!d.g.qown_ok || d.g.qown_nt != nt) {                // the partition's owners, once per nt
        std::vector<int> own(N);
        for (size_t k = 0; k < N; k++) {
            const int t = g_qown[k];
            int q = -1;
            for (int r = 0; r < m && t >= 0; r++) if (ids[r] == t) { q = r; break; }
            own[k] = q;
        }
        if (!d.g.qown && cudaMalloc(&d.g.qown, N * sizeof(int)) != cudaSuccess) { d.g.qown = nullptr; return 0; }
        cudaMemcpyAsync(d.g.qown, own.data(), N * sizeof(int), cudaMemcpyHostToDevice, d.g.st);
        cudaStreamSynchronize(d.g.st);
        d.g.qown_ok = true;
        d.g.qown_nt = nt;
    }
    double acc[NC_MAX + 1];
    if (!out_terminal_charges(d, d.g.qown, m, gate_slot, acc)) return 0;
    for (int t = 0; t <= nt; t++) Qt[t] = 0.;
    for (int q = 0; q < m; q++) Qt[ids[q]] = acc[q];
    Qt[nt] = acc[m];
    return 1;
}
int api3_face_J(int ax, int carrier, double *out) {
    Inst &d = g_dev;
    if (!d.allocated || !d.have_solution || !out || ax < 0 || ax > 2 || !d.g.ready) return 0;
    if (d.unstr) return 0;                          // faces of a graph mesh have no axis (as the reference)
    launch_face_J(make_ctx(d), ax, carrier, d.g.scratch);
    cudaMemcpyAsync(out, d.g.scratch, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    cudaStreamSynchronize(d.g.st);
    return 1;
}
int api3_charge_owner(int *out) {
    Inst &d = g_dev;
    if (g_qown.size() != d.N || g_qown.empty() || !out) return 0;
    std::memcpy(out, g_qown.data(), d.N * sizeof(int));
    return 1;
}
double api3_ins_field_max(double *pos) {                    // semiconductor_3d.c:5308-5339
    Inst &d = g_dev;
    if (pos) pos[0] = pos[1] = pos[2] = nanv();
    if (!d.allocated || !d.have_solution || !d.g.ready) return nanv();
    long long kb = -1;
    const double best = out_ins_field(d, &kb);
    if (pos && kb >= 0) {
        const size_t k = (size_t)kb;
        const int l = int(k / ((size_t)d.Nx * d.Ny)), rem = int(k - (size_t)l * d.Nx * d.Ny);
        if (d.unstr) { pos[0] = d.ggh.pos[3 * k]; pos[1] = d.ggh.pos[3 * k + 1]; pos[2] = d.ggh.pos[3 * k + 2]; }
        else { pos[0] = d.xs[rem % d.Nx]; pos[1] = d.ys[rem / d.Nx]; pos[2] = d.zs[l]; }
    }
    return best;
}
// ------------------------------------------------------------------ instances (additive)
// Additive entries with no counterpart in the reference (whose core has one global
// device): more solver instances, each with its own device memory and CUDA stream.
// api3b_use selects the instance the calling thread's api3_* calls act on.
int api3b_new(void) {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_reg.emplace_back(new Inst());
    return (int)g_reg.size();
}
int api3b_use(int h) {
    if (h == 0) { t_cur = nullptr; return 1; }
    std::lock_guard<std::mutex> lk(g_reg_mu);
    if (h < 1 || h > (int)g_reg.size() || !g_reg[h - 1]) return 0;
    t_cur = g_reg[h - 1].get();
    return 1;
}
int api3b_current(void) {
    if (!t_cur) return 0;
    std::lock_guard<std::mutex> lk(g_reg_mu);
    for (size_t q = 0; q < g_reg.size(); q++)
        if (g_reg[q].get() == t_cur) return (int)q + 1;
    return -1;
}
// precision of the current instance's linear solves: 0 FP64 throughout (the reference's
// arithmetic), 1 FP32 Krylov / multigrid inner solves refined in FP64 to the same FP64
// stop rule, -1 the library default (SEMISIM_B200_PRECISION=mixed selects 1).  Returns
// the previous setting.
int api3b_set_precision(int mode) {
    Inst &d = g_dev;
    const int old = d.precision;
    d.precision = mode < -1 ? -1 : (mode > 1 ? 1 : mode);
    return old;
}
// persistent linear solves on (1) / off (0), blocks per launch (0: every SM's worth); -1
// keeps a value.  Returns the previous mode.
int api3b_set_persist(int mode, int blocks) {
    const int old = persist_enabled();
    persist_set(mode, blocks);
    return old;
}
// order of the sweep predictor (1 secant, 2 quadratic), library-wide; other values read.
// Returns the previous order.
int api3b_set_pred_order(int order) {
    const int old = g_knobs.pred_order;
    if (order == 1 || order == 2) g_knobs.pred_order = order;
    return old;
}
// grid share (blocks) of the current instance's persistent solves, 0 for none; -1 reads.
// Returns the previous share.
int api3b_set_share(int blocks) {
    const int old = g_dev.pblocks;
    if (blocks >= 0) g_dev.pblocks = blocks;
    return old;
}
// precision in effect on the current instance (0 FP64, 1 refined FP32)
int api3b_get_precision(void) { return use_mixed(g_dev); }
int api3b_free(int h) {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    if (h < 1 || h > (int)g_reg.size() || !g_reg[h - 1]) return 0;
    if (t_cur == g_reg[h - 1].get()) t_cur = nullptr;
    batch_pool_release(g_reg[h - 1].get());   // its batched-resolve workers go with it
    gpu_free(*g_reg[h - 1]);
    g_reg[h - 1].reset();
    return 1;
}

double api3_get_phi(int k) { return node_val1(0, k); }
double api3_get_n(int k) { return node_val1(1, k); }
double api3_get_p(int k) { return node_val1(2, k); }
double api3_get_Ec(int k) { return node_val1(3, k); }
double api3_get_Ev(int k) { return node_val1(4, k); }
double api3_get_Efn(int k) { return node_val1(5, k); }
double api3_get_Efp(int k) { return node_val1(6, k); }
double api3_get_Jx(int k) { return node_val1(7, k); }
double api3_get_Jy(int k) { return node_val1(8, k); }
double api3_get_Jz(int k) { return node_val1(9, k); }
double api3_get_mun(int k) { return node_val1(10, k); }
double api3_get_mup(int k) { return node_val1(11, k); }
double api3_get_R(int k) { return node_val1(12, k); }

}  // extern "C"
