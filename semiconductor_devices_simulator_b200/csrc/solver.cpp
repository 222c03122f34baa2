// Host control of the solve path over device-resident state: device set-up (prepare),
// equilibrium, damped Newton-Poisson with PCG, the continuity solves with BiCGSTAB and
// the floating-block balance, the Gummel loop with Anderson mixing and the adaptive
// continuation with the sweep predictor.  The control logic follows the reference
// routine named beside each function; all O(N) work runs in the CUDA kernels.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "exact_sum.cuh"
#include "solver_ctx.h"
#include "physics_hd.cuh"

namespace ss {

Knobs g_knobs;
std::atomic<int> g_stop{0};
volatile double g_prog[8];

static double wtime() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            std::fprintf(stderr, "semisim-b200: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                                   \
            return 0;                                                                           \
        }                                                                                       \
    } while (0)

bool gpu_available() {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

int g_device = -1;                 // CUDA device of the solver (-1: the runtime's current one)

int select_device(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || dev < 0 || dev >= n) return 0;
    g_device = dev;
    return 1;
}

int g_precision_default = 0;

int use_mixed(const Inst &d) { return (d.precision < 0 ? g_precision_default : d.precision) == 1 ? 1 : 0; }

Ctx make_ctx(Inst &d) {
    if (g_device >= 0) cudaSetDevice(g_device);
    Ctx c;
    c.dP = d.g.d;
    c.h = d.g.h;
    c.ninst = 1;
    c.maxN = (int)d.N;
    c.st = d.g.st;
    c.lg = &d.g.lg;
    c.rpb = d.tune.rpb;
    c.grid_cap = d.tune.grid_cap;
    c.small_nodes = d.tune.small_nodes;
    c.zcap = d.tune.zcap;
    c.rq = d.tune.rq;
    c.pblocks = d.pblocks;
    return c;
}

static double read_res(Inst &d, int slot) {
    cudaMemcpyAsync(d.g.pin, d.g.h.res + slot, sizeof(double), cudaMemcpyDeviceToHost, d.g.st);
    cudaStreamSynchronize(d.g.st);
    return d.g.pin[0];
}

// ------------------------------------------------------------------ device memory
static size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

struct Carver {
    char *base = nullptr;
    size_t off = 0;
    template <class T> T *take(size_t n) {
        T *p = reinterpret_cast<T *>(base ? base + off : nullptr);
        off += align_up(n * sizeof(T));
        return p;
    }
};

// Lay out every device array of an instance in one block (two passes: size, then place).
static void carve(Inst &d, Carver &cv, DevP &P, std::vector<LevelT<double>> &levs, std::vector<LevelT<float>> &levsf,
                  int nlev, const int dims[][6]) {
    const size_t N = d.N;
    P.flags = cv.take<uint32_t>(N);
    P.Nd = cv.take<double>(N); P.Na = cv.take<double>(N); P.Nf = cv.take<double>(N);
    P.bgn = cv.take<double>(N); P.robA = cv.take<double>(N); P.qd = cv.take<double>(N);
    P.xs = cv.take<double>(d.Nx); P.ys = cv.take<double>(d.Ny); P.zs = cv.take<double>(d.Nz);
    P.Lx = cv.take<double>(d.Nx); P.Ly = cv.take<double>(d.Ny); P.Lz = cv.take<double>(d.Nz);
    P.mats = cv.take<MatD>(NM_MAX);
    P.cons = cv.take<ConD>(NC_MAX);
    P.cnode = cv.take<int>(N > 0 ? N : 1);
    P.phi = cv.take<double>(N); P.phin = cv.take<double>(N); P.phip = cv.take<double>(N);
    P.n = cv.take<double>(N); P.p = cv.take<double>(N);
    P.mu0n = cv.take<double>(N); P.mu0p = cv.take<double>(N);
    P.mudn = cv.take<double>(N); P.mudp = cv.take<double>(N);
    for (int q = 0; q < 6; q++) P.fmu[q] = cv.take<double>(N);
    for (int q = 0; q < 7; q++) P.A[q] = cv.take<double>(N);
    P.rhs = cv.take<double>(N); P.sc = cv.take<double>(N); P.dsc = cv.take<double>(N);
    P.sol = cv.take<double>(N); P.F = cv.take<double>(N);
    for (int q = 0; q < 8; q++) P.wk[q] = cv.take<double>(N);
    P.qn0 = cv.take<double>(N); P.qp0 = cv.take<double>(N); P.dqn = cv.take<double>(N);
    P.dqp = cv.take<double>(N); P.xk = cv.take<double>(N); P.tr = cv.take<double>(N);
    P.Jx = cv.take<double>(N); P.Jy = cv.take<double>(N); P.Jz = cv.take<double>(N); P.Rt = cv.take<double>(N);
    for (int a = 0; a < 3; a++) { P.h1[a] = cv.take<double>(N); P.h2[a] = cv.take<double>(N); P.e2[a] = cv.take<double>(N); }
    for (int a = 0; a < 3; a++) P.e3[a] = cv.take<double>(N);
    P.aaF = cv.take<float>((size_t)AA_MAX * 3 * N);
    P.aaG = cv.take<float>((size_t)AA_MAX * 3 * N);
    P.aaf = cv.take<double>(3 * N); P.aag = cv.take<double>(3 * N);
    P.gram = cv.take<double>(AA_MAX * AA_MAX); P.aagam = cv.take<double>(AA_MAX);
    P.part = cv.take<double>((size_t)RED_MAX_BLOCKS * RED_NV);
    P.ticket = cv.take<unsigned>(16);
    P.partc = cv.take<double>(256 * 96);
    P.ffbuf = cv.take<double>(6 * 1024);
    P.ffint = cv.take<int>(16 + 1024);
    P.ffacc = cv.take<unsigned long long>((size_t)4 * 1024 * XS_WORDS);
    P.res = cv.take<double>(R_TOTAL);
    P.ks = cv.take<KrylovS>(1);
    P.ksi = cv.take<KrylovS>(1);
    P.pgrid = cv.take<PGrid>(1);
    for (int q = 0; q < 7; q++) P.A32[q] = cv.take<float>(N);
    P.dsc32 = cv.take<float>(N); P.rhs32 = cv.take<float>(N); P.sol32 = cv.take<float>(N);
    for (int q = 0; q < 8; q++) P.wk32[q] = cv.take<float>(N);
    P.lev = cv.take<LevelT<double>>(MAXLEV);
    P.levf = cv.take<LevelT<float>>(MAXLEV);
    P.ccl = cv.take<int>(N); P.cclaux = cv.take<int>(N);
    levs.assign(nlev, LevelT<double>{});
    levsf.assign(nlev, LevelT<float>{});
    // the FP64 hierarchy (plain solves) and its FP32 twin (inner solves of the refined path)
    auto shape = [&](auto &v, int L) {
        v.Nx = dims[L][0]; v.Ny = dims[L][1]; v.Nz = dims[L][2];
        v.N = v.Nx * v.Ny * v.Nz;
        v.apitch = int(align_up((size_t)v.N * sizeof(*v.A[0])) / sizeof(*v.A[0]));
        v.cx = dims[L][3]; v.cy = dims[L][4]; v.cz = dims[L][5];
        v.last = L == nlev - 1;
    };
    for (int L = 0; L < nlev; L++) {
        LevelT<double> &v = levs[L];
        shape(v, L);
        const size_t n = (size_t)v.N;
        if (L == 0) {
            for (int q = 0; q < 7; q++) v.A[q] = P.A[q];
            v.x = nullptr; v.b = nullptr;
        } else {
            for (int q = 0; q < 7; q++) v.A[q] = cv.take<double>(n);
            v.x = cv.take<double>(n); v.b = cv.take<double>(n);
        }
        v.D = cv.take<double>(v.last && L > 0 ? n * n : n);
        v.r = cv.take<double>(n);
        v.pw = cv.take<double>(n);
        v.ph = cv.take<double>(n);
    }
    for (int L = 0; L < nlev; L++) {
        LevelT<float> &v = levsf[L];
        shape(v, L);
        const size_t n = (size_t)v.N;
        if (L == 0) {
            for (int q = 0; q < 7; q++) v.A[q] = P.A32[q];
            v.x = nullptr; v.b = nullptr;
        } else {
            for (int q = 0; q < 7; q++) v.A[q] = cv.take<float>(n);
            v.x = cv.take<float>(n); v.b = cv.take<float>(n);
        }
        v.D = cv.take<float>(v.last && L > 0 ? n * n : n);
        v.r = cv.take<float>(n);
        v.pw = cv.take<float>(n);
        v.ph = levs[L].ph;              // set-up scratch, shared with the FP64 twin
    }
}

// 2x2x2 aggregation hierarchy shape (semiconductor_3d.c:1894-1921)
int mg_levels(int Nx, int Ny, int Nz, int dims[][6]) {
    int nl = 1;
    dims[0][0] = Nx; dims[0][1] = Ny; dims[0][2] = Nz; dims[0][3] = dims[0][4] = dims[0][5] = 0;
    while (nl < MAXLEV) {
        int *f = dims[nl - 1];
        if ((size_t)f[0] * f[1] * f[2] <= 64) break;
        const int cx = f[0] > 2, cy = f[1] > 2, cz = f[2] > 2;
        if (!cx && !cy && !cz) break;
        f[3] = cx; f[4] = cy; f[5] = cz;
        int *c = dims[nl];
        c[0] = cx ? (f[0] + 1) / 2 : f[0];
        c[1] = cy ? (f[1] + 1) / 2 : f[1];
        c[2] = cz ? (f[2] + 1) / 2 : f[2];
        c[3] = c[4] = c[5] = 0;
        nl++;
    }
    return nl;
}

void gpu_free(Inst &d) {
    for (auto &e : d.g.lg.exec)
        if (e) cudaGraphExecDestroy(e);
    for (auto &e : d.g.tev)
        if (e) cudaEventDestroy(e);
    if (d.g.block) cudaFree(d.g.block);
    if (d.g.d) cudaFree(d.g.d);
    if (d.g.pin) cudaFreeHost(d.g.pin);
    if (d.g.scratch) cudaFree(d.g.scratch);
    if (d.g.flag) cudaFree(d.g.flag);
    if (d.g.qown) cudaFree(d.g.qown);
    if (d.g.ion) cudaFree(d.g.ion);
    if (d.g.gii) cudaFree(d.g.gii);
    if (d.g.teblock) cudaFree(d.g.teblock);
    if (d.g.qc) cudaFree(d.g.qc);
    if (d.g.xchg) cudaFree(d.g.xchg);
    if (d.g.tunblock) cudaFree(d.g.tunblock);
    if (d.g.trblock) cudaFree(d.g.trblock);
    if (d.g.coblock) cudaFree(d.g.coblock);
    if (d.g.gblock) cudaFree(d.g.gblock);
    gmg_free(d);
    if (d.g.seedw) cudaFree(d.g.seedw);
    if (d.g.st) cudaStreamDestroy(d.g.st);
    d.g = Gpu();
}

static int gpu_alloc(Inst &d) {
    if (d.g.ready && d.g.h.Nx == d.Nx && d.g.h.Ny == d.Ny && d.g.h.Nz == d.Nz) return 1;
    gpu_free(d);
    if (!gpu_available()) {
        std::fprintf(stderr, "semisim-b200: no CUDA device available - the solver has no CPU path\n");
        return 0;
    }
    if (g_device < 0) {
        const char *e = std::getenv("SEMISIM_B200_DEVICE");
        g_device = e ? std::atoi(e) : 0;
    }
    CK(cudaSetDevice(g_device));
    static bool sync_set = false;             // host wait mode, once per process (SEMISIM_B200_SYNC)
    if (!sync_set) {
        sync_set = true;
        if (const char *m = std::getenv("SEMISIM_B200_SYNC")) {
            const unsigned fl = !std::strcmp(m, "blocking") ? cudaDeviceScheduleBlockingSync
                                : !std::strcmp(m, "yield") ? cudaDeviceScheduleYield : cudaDeviceScheduleSpin;
            if (cudaSetDeviceFlags(fl) != cudaSuccess) cudaGetLastError();   // an active context keeps its mode
        }
    }
    int dims[MAXLEV][6];
    const int nl = mg_levels(d.Nx, d.Ny, d.Nz, dims);
    Carver cv;
    DevP P{};
    std::vector<LevelT<double>> levs;
    std::vector<LevelT<float>> levsf;
    carve(d, cv, P, levs, levsf, nl, dims);       // sizing pass
    const size_t bytes = cv.off;
    void *blk = nullptr;
    CK(cudaMalloc(&blk, bytes));
    CK(cudaMemset(blk, 0, bytes));
    Carver cv2;
    cv2.base = static_cast<char *>(blk);
    P = DevP{};
    carve(d, cv2, P, levs, levsf, nl, dims);
    P.Nx = d.Nx; P.Ny = d.Ny; P.Nz = d.Nz; P.N = (int)d.N; P.nlev = nl;
    d.g.block = blk;
    d.g.bytes = bytes;
    d.g.N = d.N;
    d.g.levs = levs;
    d.g.h = P;
    CK(cudaMalloc(&d.g.d, sizeof(DevP)));
    CK(cudaStreamCreateWithFlags(&d.g.st, cudaStreamNonBlocking));
    CK(cudaMallocHost(&d.g.pin, sizeof(double) * 256));
    CK(cudaMalloc(&d.g.scratch, sizeof(double) * (d.N > 0 ? d.N : 1)));
    CK(cudaMalloc(&d.g.flag, sizeof(int) * 16));
    for (int L = 0; L < nl; L++)                     // the kernels address A[q] as A[0] + q * apitch
        for (int q = 1; q < 7; q++)
            if (levs[L].A[q] != levs[L].A[0] + (size_t)q * levs[L].apitch ||
                levsf[L].A[q] != levsf[L].A[0] + (size_t)q * levsf[L].apitch) {
                std::fprintf(stderr, "semisim-b200: level %d coupling arrays are not evenly spaced\n", L);
                gpu_free(d);
                return 0;
            }
    CK(cudaMemcpy(P.lev, levs.data(), sizeof(LevelT<double>) * nl, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(P.levf, levsf.data(), sizeof(LevelT<float>) * nl, cudaMemcpyHostToDevice));
    MGHost &mg = d.g.mg;
    mg.maxlev = mg.minlev = nl;
    for (int L = 0; L < nl; L++) {
        mg.maxN[L] = levs[L].N;
        mg.maxNx[L] = levs[L].Nx;
        mg.maxRows[L] = levs[L].Ny * levs[L].Nz;
    }
    d.g.ready = true;
    return 1;
}

// ------------------------------------------------------------------ prepare
// Contact node iteration over a node list, a face or a box (FOR_CON_ANY / FOR_CON_NODES,
// semiconductor_3d.c:1045-1065, 1422-1426)
template <class F>
static void for_con_nodes(const Inst &d, const Contact &cn, F body) {
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const int cid = int(&cn - d.cons);
    if (d.unstr || (cid >= 0 && cid < NC_MAX && !d.cnodes[cid].empty())) {   // node lists (graph: only those)
        if (cid < 0 || cid >= NC_MAX) return;
        for (size_t q = 0; q < d.cnodes[cid].size(); q++) {
            const size_t k = (size_t)d.cnodes[cid][q];
            const int l = int(k / ((size_t)Nx * Ny)), rem = int(k - (size_t)l * Nx * Ny);
            body(rem % Nx, rem / Nx, l, k, d.careas[cid][q]);
        }
        return;
    }
    int ia = 0, ib = Nx - 1, ja = 0, jb = Ny - 1, la = 0, lb = Nz - 1;
    switch (cn.face) {
    case 0: ia = ib = 0; ja = cn.i0; jb = cn.i1; la = cn.j0; lb = cn.j1; break;
    case 1: ia = ib = Nx - 1; ja = cn.i0; jb = cn.i1; la = cn.j0; lb = cn.j1; break;
    case 2: ja = jb = 0; ia = cn.i0; ib = cn.i1; la = cn.j0; lb = cn.j1; break;
    case 3: ja = jb = Ny - 1; ia = cn.i0; ib = cn.i1; la = cn.j0; lb = cn.j1; break;
    case 4: la = lb = 0; ia = cn.i0; ib = cn.i1; ja = cn.j0; jb = cn.j1; break;
    case 5: la = lb = Nz - 1; ia = cn.i0; ib = cn.i1; ja = cn.j0; jb = cn.j1; break;
    default: ia = cn.i0; ib = cn.i1; ja = cn.j0; jb = cn.j1; la = cn.k0; lb = cn.k1;
    }
    if (ia < 0) ia = 0; if (ja < 0) ja = 0; if (la < 0) la = 0;
    if (ib > Nx - 1) ib = Nx - 1; if (jb > Ny - 1) jb = Ny - 1; if (lb > Nz - 1) lb = Nz - 1;
    for (int l = la; l <= lb; l++)
        for (int j = ja; j <= jb; j++)
            for (int i = ia; i <= ib; i++) {
                const size_t k = (size_t)l * Nx * Ny + (size_t)j * Nx + i;
                const double area = cn.face <= 1 ? d.Ly[j] * d.Lz[l]
                                  : (cn.face <= 3 ? d.Lx[i] * d.Lz[l] : (cn.face <= 5 ? d.Lx[i] * d.Ly[j] : 0.));
                body(i, j, l, k, area);
            }
}

// Material band offsets in the common gauge (mat_prepare, semiconductor_3d.c:631-642)
void mat_prepare(Inst &d) {
    d.ref_mat = 0;
    for (int i = 0; i < d.n_mats; i++)
        if (!d.mats[i].insulator) { d.ref_mat = i; break; }
    const Material &r = d.mats[d.ref_mat];
    d.Cref = r.insulator ? 4.6 : r.chi + 0.5 * r.Eg + 0.5 * r.VT * std::log(r.Nc / r.Nv);
    for (int i = 0; i < d.n_mats; i++) {
        Material &m = d.mats[i];
        if (m.insulator) { m.lnc = m.lnv = -1e300; continue; }
        m.lnc = std::log(m.Nc) + (m.chi - d.Cref) / m.VT;
        m.lnv = std::log(m.Nv) + (d.Cref - m.chi - m.Eg) / m.VT;
    }
}

// device record of a material (the constants the kernels and the tunnelling arithmetic read)
void mat_to_dev(const Material &m, MatD &o) {
    std::memset(&o, 0, sizeof o);
    o.VT = m.VT; o.lnc = m.lnc; o.lnv = m.lnv; o.ni = m.ni; o.eps = m.eps_r * EPS0;
    o.tau_n0 = m.tau_n0; o.tau_p0 = m.tau_p0; o.Cn = m.Cn; o.Cp = m.Cp; o.Brad = m.Brad; o.tau_Nref = m.tau_Nref;
    o.vsat_n = m.vsat_n; o.vsat_p = m.vsat_p; o.beta_n = m.beta_n; o.beta_p = m.beta_p;
    o.ani_n = m.ani_n; o.ani_p = m.ani_p; o.chi = m.chi; o.Eg = m.Eg; o.insulator = m.insulator;
    o.ion_w[0] = m.ion_on ? m.ion_w[0] : 0.; o.ion_w[1] = m.ion_on ? m.ion_w[1] : 0.;
    o.T = m.T; o.Nc = m.Nc; o.Nv = m.Nv;
    o.rich_n = m.rich_n; o.rich_p = m.rich_p; o.mtun_e = m.mtun_e; o.mtun_h = m.mtun_h;
    o.ms_e = m.ms_e; o.ms_h = m.ms_h;
    o.ii_on = m.ii_on;
    for (int c = 0; c < 2; c++) {
        o.ii_a[c][0] = m.ii_a[c][0]; o.ii_a[c][1] = m.ii_a[c][1];
        o.ii_b[c][0] = m.ii_b[c][0]; o.ii_b[c][1] = m.ii_b[c][1];
        o.ii_E0[c] = m.ii_E0[c]; o.ii_m[c] = m.ii_m[c];
    }
    o.ii_g = m.ii_g;
    o.lb_on = m.lb_on;
    o.lbc_on = m.lbc_on;
    o.lbc_mu1 = m.lbc_mu1; o.lbc_nu = m.lbc_nu; o.lbc_N0 = m.lbc_N0; o.lbc_e1 = m.lbc_e1; o.lbc_e2 = m.lbc_e2;
    o.lbc_E0 = m.lbc_E0; o.lbc_gam = m.lbc_gam;
    for (int c = 0; c < 2; c++) {
        o.lbB[c] = m.lbB[c]; o.lbC[c] = m.lbC[c]; o.lbL[c] = m.lbL[c]; o.lbD[c] = m.lbD[c]; o.lbE[c] = m.lbE[c];
    }
}

// prepare (semiconductor_3d.c:1638-1775): node kinds, contact and gate masks, Robin gate
// areas, contact areas, band-gap narrowing; uploaded to the device with the geometry.
// Distance of every node to the nearest wall along the mesh axes (the interface distance
// semiconductor_3d.c:1100-1145 reports for display): scanning each mesh line both ways, a
// wall is the midpoint to an insulator neighbour, or the domain face of the node's gate
// contact; a metal node or the domain edge without such a gate ends the run.  1 m where no
// wall is in sight.
// MLDA factor of one population averaged over a cell z in [a, b] from a hard wall:
// 1 - exp(-(z/lambda)^2) (semiconductor_3d.c:1072-1080)
static double mlda_pop(double a, double b, double lam) {
    const double u = a / lam, v = b / lam;
    if (v < 0.05) {                                       // series: no cancellation
        const double dd = v - u;
        if (dd < 1e-12) return u * u;
        return ((v * v * v - u * u * u) / 3. - (std::pow(v, 5) - std::pow(u, 5)) / 10. +
                (std::pow(v, 7) - std::pow(u, 7)) / 42.) / dd;
    }
    if (v - u < 1e-9 * v) return 1. - std::exp(-u * u);
    return 1. - 0.5 * std::sqrt(3.14159265358979323846) * (std::erf(v) - std::erf(u)) / (v - u);
}
// two populations, lambda = hbar / sqrt(2 m kT) (semiconductor_3d.c:1081-1088)
double mlda_factor_host(const Material &m, double a, double b, int hole) {
    const double HBAR_ = 1.054571817e-34, M0_ = 9.1093837015e-31;
    const double kT = KB * m.T, m1 = hole ? m.mq_h1 : m.mq_e1, m2 = hole ? m.mq_h2 : m.mq_e2,
                 w = hole ? m.wq_h1 : m.wq_e1;
    if (!(m1 > 0.)) return 1.;
    if (a < 0.) a = 0.;
    if (b < a) b = a;
    double f = w * mlda_pop(a, b, HBAR_ / std::sqrt(2. * m1 * M0_ * kT));
    if (w < 1. && m2 > 0.) f += (1. - w) * mlda_pop(a, b, HBAR_ / std::sqrt(2. * m2 * M0_ * kT));
    return f;
}

// With qc (models bit 3) also the MLDA band corrections qcn / qcp: the sum over the walls
// within 40 nm of the log of the cell-averaged factor, clamped at -60
// (semiconductor_3d.c:1090-1145).
static void wall_distance(const Inst &d, const std::vector<unsigned char> &kind, const std::vector<int> &gate,
                          std::vector<double> &qd, bool qc, std::vector<double> &qcn, std::vector<double> &qcp) {
    const int n3[3] = {d.Nx, d.Ny, d.Nz};
    const std::vector<double> *cs[3] = {&d.xs, &d.ys, &d.zs};
    const size_t st3[3] = {1, (size_t)d.Nx, (size_t)d.Nx * d.Ny};
    qd.assign(d.N, 1.0);
    qcn.assign(qc ? d.N : 0, 0.0);
    qcp.assign(qc ? d.N : 0, 0.0);
    for (int ax = 0; ax < 3; ax++) {
        const int n = n3[ax];
        const std::vector<double> &c = *cs[ax];
        const size_t st = st3[ax];
        for (size_t k0 = 0; k0 < d.N; k0++) {
            if ((k0 / st) % (size_t)n != 0) continue;          // a line starts at index 0 along ax
            for (int side = 0; side < 2; side++) {               // 0: walls below, 1: walls above
                double w = 0.;
                bool have = false;
                for (int t = 0; t < n; t++) {
                    const int q = side ? n - 1 - t : t;
                    const size_t k = k0 + (size_t)q * st;
                    if (kind[k] != K_SEMI) { have = false; continue; }
                    const int qp = side ? q + 1 : q - 1;
                    if (qp < 0 || qp >= n) {
                        have = false;
                        const int g = gate[k];
                        if (g && d.cons[g - 1].face == 2 * ax + side) { w = c[q]; have = true; }
                    } else {
                        const unsigned char kb = kind[k0 + (size_t)qp * st];
                        if (kb == K_INS) { w = 0.5 * (c[q] + c[qp]); have = true; }
                        else if (kb != K_SEMI) have = false;
                    }
                    if (!have) continue;
                    const double lo = q > 0 ? 0.5 * (c[q - 1] + c[q]) : c[q];
                    const double hi = q < n - 1 ? 0.5 * (c[q] + c[q + 1]) : c[q];
                    double za = side ? w - hi : lo - w;
                    const double zb = side ? w - lo : hi - w, zn = std::fabs(c[q] - w);
                    if (za < 0.) za = 0.;
                    if (zn < qd[k]) qd[k] = zn;
                    if (qc && za < 40e-9) {
                        const Material &m = d.mats[d.mat_idx[k]];
                        qcn[k] += std::log(std::fmax(mlda_factor_host(m, za, zb, 0), 1e-30));
                        qcp[k] += std::log(std::fmax(mlda_factor_host(m, za, zb, 1), 1e-30));
                    }
                }
            }
        }
    }
    for (size_t k = 0; k < qcn.size(); k++) {            // keep the exponents sane
        if (qcn[k] < -60.) qcn[k] = -60.;
        if (qcp[k] < -60.) qcp[k] = -60.;
    }
}

// interface distance and MLDA corrections of a graph device from the walls the host gave
// (two per node: the node's distance, the range a..b of its cell; distance >= 0.5 m: none)
// (walls_graph, semiconductor_3d.c:1252-1271)
static void walls_graph(const Inst &d, const std::vector<unsigned char> &kind, std::vector<double> &qd, bool qc,
                        std::vector<double> &qcn, std::vector<double> &qcp) {
    const size_t N = d.N;
    qd.assign(N, 1.0);
    qcn.assign(qc ? N : 0, 0.0);
    qcp.assign(qc ? N : 0, 0.0);
    for (size_t k = 0; k < N; k++) {
        if (kind[k] != K_SEMI) continue;
        const Material &m = d.mats[d.mat_idx[k]];
        for (int w = 0; w < 2; w++) {
            const double *g = d.ggh.wall.data() + 6 * k + 3 * w;
            if (!(g[0] < 0.5)) continue;
            if (g[0] < qd[k]) qd[k] = g[0];
            if (qc && g[1] < 40e-9) {
                qcn[k] += std::log(std::fmax(mlda_factor_host(m, g[1], g[2], 0), 1e-30));
                qcp[k] += std::log(std::fmax(mlda_factor_host(m, g[1], g[2], 1), 1e-30));
            }
        }
        if (qc) {
            if (qcn[k] < -60.) qcn[k] = -60.;
            if (qcp[k] < -60.) qcp[k] = -60.;
        }
    }
}

// device arrays of a graph device: the CSR graph packed as ELL (gD slots per node, slot s of
// node k at s*N + k), the least-squares gradient matrices of the semiconductor nodes (g_lsq_setup,
// semiconductor_3d.c:2682-2700), room for the edge mobilities, matrix off-diagonals and
// pivots, and the aggregation multigrid hierarchy
static int graph_upload(Inst &d, const std::vector<unsigned char> &kind, DevP &P, cudaStream_t st) {
    if (d.g.gblock) { cudaFree(d.g.gblock); d.g.gblock = nullptr; }
    gmg_free(d);
    P.gD = 0; P.nUE = 0;
    P.gcol = P.gue = P.grev = nullptr;
    P.gh = P.ga = P.gpos = P.glsq = nullptr;
    P.gval = P.gmu_n = P.gmu_p = P.gdil = P.ggrad = nullptr;
    if (!d.unstr) return 1;
    GraphHost &G = d.ggh;
    const int N = (int)d.N;
    int D = 0;
    for (int k = 0; k < N; k++) D = std::max(D, G.rp[k + 1] - G.rp[k]);
    G.D = D;
    std::vector<int> col((size_t)D * N, -1), ue((size_t)D * N, 0), rv((size_t)D * N, 0), slot(G.cj.size());
    std::vector<double> h((size_t)D * N, 1.0), ar((size_t)D * N, 0.0);
    for (int k = 0; k < N; k++)
        for (int e = G.rp[k]; e < G.rp[k + 1]; e++) slot[e] = e - G.rp[k];
    for (int k = 0; k < N; k++)
        for (int e = G.rp[k]; e < G.rp[k + 1]; e++) {
            const size_t q = (size_t)slot[e] * N + k;
            col[q] = G.cj[e]; ue[q] = G.ue[e]; rv[q] = slot[G.rev[e]]; h[q] = G.h[e]; ar[q] = G.ar[e];
        }
    std::vector<double> lsq(6 * (size_t)N, 0.0);
    for (int k = 0; k < N; k++) {
        double m[6] = {0, 0, 0, 0, 0, 0};
        double *o = lsq.data() + 6 * (size_t)k;
        if (kind[k] == K_SEMI)
            for (int e = G.rp[k]; e < G.rp[k + 1]; e++) {
                const int b = G.cj[e];
                if (kind[b] != K_SEMI) continue;
                const double dx = G.pos[3 * b] - G.pos[3 * k], dy = G.pos[3 * b + 1] - G.pos[3 * k + 1],
                             dz = G.pos[3 * b + 2] - G.pos[3 * k + 2];
                const double w = 1. / (dx * dx + dy * dy + dz * dz + 1e-40);
                m[0] += w * dx * dx; m[1] += w * dx * dy; m[2] += w * dx * dz;
                m[3] += w * dy * dy; m[4] += w * dy * dz; m[5] += w * dz * dz;
            }
        const double tr = m[0] + m[3] + m[5], eps = 1e-6 * tr + 1e-30;
        m[0] += eps; m[3] += eps; m[5] += eps;
        const double a = m[0], b = m[1], c = m[2], dd = m[3], e = m[4], f = m[5];
        const double A = dd * f - e * e, B = -(b * f - c * e), Cc = b * e - c * dd, Dq = a * f - c * c,
                     E = -(a * e - b * c), F = a * dd - b * b;
        const double det = a * A + b * B + Cc * c;
        if (!(std::fabs(det) > 0.)) continue;
        o[0] = A / det; o[1] = B / det; o[2] = Cc / det; o[3] = Dq / det; o[4] = E / det; o[5] = F / det;
    }
    const size_t DN = (size_t)D * N, nue = G.nue > 0 ? (size_t)G.nue : 1;
    size_t off = 0;
    auto room = [&](size_t bytes) { const size_t x = off; off += align_up(bytes > 0 ? bytes : 1); return x; };
    const size_t o_col = room(DN * 4), o_ue = room(DN * 4), o_rv = room(DN * 4), o_h = room(DN * 8), o_ar = room(DN * 8),
                 o_val = room(DN * 8),
                 o_pos = room(3 * (size_t)N * 8), o_lsq = room(6 * (size_t)N * 8), o_mun = room(nue * 8),
                 o_mup = room(nue * 8), o_dil = room((size_t)N * 8), o_gg = room(3 * (size_t)N * 8);
    char *b = nullptr;
    if (cudaMalloc(&b, off) != cudaSuccess) {
        std::fprintf(stderr, "semisim-b200: out of device memory for the mesh graph\n");
        return 0;
    }
    d.g.gblock = b;
    bool ok = cudaMemsetAsync(b, 0, off, st) == cudaSuccess;
    auto up = [&](size_t x, const void *src, size_t bytes) {
        if (bytes && cudaMemcpyAsync(b + x, src, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) ok = false;
    };
    up(o_col, col.data(), DN * 4); up(o_ue, ue.data(), DN * 4); up(o_rv, rv.data(), DN * 4);
    up(o_h, h.data(), DN * 8); up(o_ar, ar.data(), DN * 8);
    up(o_pos, G.pos.data(), 3 * (size_t)N * 8);
    up(o_lsq, lsq.data(), 6 * (size_t)N * 8);
    P.gD = D; P.nUE = G.nue;
    P.gcol = (const int *)(b + o_col); P.gue = (const int *)(b + o_ue); P.grev = (const int *)(b + o_rv);
    P.gh = (const double *)(b + o_h); P.ga = (const double *)(b + o_ar); P.gpos = (const double *)(b + o_pos);
    P.glsq = (const double *)(b + o_lsq);
    P.gval = (double *)(b + o_val); P.gmu_n = (double *)(b + o_mun); P.gmu_p = (double *)(b + o_mup);
    P.gdil = (double *)(b + o_dil);
    P.ggrad = (double *)(b + o_gg);
    if (cudaStreamSynchronize(st) != cudaSuccess) ok = false;
    return ok && gmg_build(d, st) ? 1 : 0;
}

// Thermionic-emission metal contacts (semiconductor_3d.c:1376-1416, 1723-1768): one entry
// per semiconductor node of a metal face contact with its column along the inward normal
// (semiconductor nodes of no contact, until TE_COL deep), the velocity-saturation weight
// of the column nodes (0 in the first half of the column, rising to 1 at its end) and,
// per column node, its column entries in ascending order.
struct TeHost {
    std::vector<int> te_k, te_c, te_c0, te_cn, tc_k, tn_k, tn_ptr, tn_q;
    std::vector<double> te_A, tc_s;
    std::vector<float> vw;
    std::vector<signed char> ax;
    int ce0[NC_MAX], ce1[NC_MAX];
};
// graph mesh: the displacement a -> b projected on the unit vector u, and the neighbour of
// cur best aligned with u (cosine above cmin), not prev (g_proj / g_step,
// semiconductor_3d.c:1272-1284)
static double g_proj(const GraphHost &G, size_t a, size_t b, const double *u) {
    return (G.pos[3 * b] - G.pos[3 * a]) * u[0] + (G.pos[3 * b + 1] - G.pos[3 * a + 1]) * u[1] +
           (G.pos[3 * b + 2] - G.pos[3 * a + 2]) * u[2];
}
static long g_step(const GraphHost &G, size_t cur, long prev, const double *u, double cmin) {
    long best = -1;
    double bc = cmin;
    for (int e = G.rp[cur]; e < G.rp[cur + 1]; e++) {
        const int b = G.cj[e];
        if ((long)b == prev) continue;
        const double c = g_proj(G, cur, (size_t)b, u) / G.h[e];
        if (c > bc) { bc = c; best = b; }
    }
    return best;
}

static void te_build(Inst &d, const std::vector<unsigned char> &kind, const std::vector<int> &con, TeHost &H) {
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const size_t N = d.N;
    for (int c = 0; c < NC_MAX; c++) H.ce0[c] = H.ce1[c] = 0;
    for (int c = 0; c < d.n_cons; c++) {
        const Contact &cn = d.cons[c];
        H.ce0[c] = H.ce1[c] = (int)H.te_k.size();
        if (!cn.te) continue;
        const int dir = cn.face ^ 1;                       // inward normal of the face
        for_con_nodes(d, cn, [&](int, int, int, size_t k, double area) {
            if (con[k] != c + 1 || kind[k] != K_SEMI || !(area > 0.)) return;
            H.te_k.push_back((int)k); H.te_A.push_back(area); H.te_c.push_back(c);
            H.te_c0.push_back((int)H.tc_k.size());
            H.tc_k.push_back((int)k); H.tc_s.push_back(0.);
            int cnt = 1;
            double s_ = 0.;
            size_t cur = k;
            if (d.unstr) {                                  // graph: the neighbour best aligned with the normal
                double v[3] = {0., 0., 0.};
                v[cn.face / 2] = (cn.face & 1) ? -1. : 1.;
                long prev = -1;
                for (int guard = 0; guard < 100000; guard++) {
                    const long nb = g_step(d.ggh, cur, prev, v, 0.8);
                    if (nb < 0 || kind[nb] != K_SEMI || con[nb]) break;
                    const double h = g_proj(d.ggh, cur, (size_t)nb, v);
                    if (!(h > 0.)) break;
                    s_ += h;
                    H.tc_k.push_back((int)nb); H.tc_s.push_back(s_);
                    cnt++;
                    if (s_ >= TE_COL) break;
                    prev = (long)cur;
                    cur = (size_t)nb;
                }
                H.te_cn.push_back(cnt);
                return;
            }
            for (int guard = 0; guard < 100000; guard++) {
                const int l = int(cur / ((size_t)Nx * Ny)), rem = int(cur - (size_t)l * Nx * Ny);
                const int j = rem / Nx, i = rem % Nx;
                long long kn = -1;
                double h = 0.;
                switch (dir) {
                case 0: if (i > 0) { kn = (long long)cur - 1; h = d.xs[i] - d.xs[i - 1]; } break;
                case 1: if (i < Nx - 1) { kn = (long long)cur + 1; h = d.xs[i + 1] - d.xs[i]; } break;
                case 2: if (j > 0) { kn = (long long)cur - Nx; h = d.ys[j] - d.ys[j - 1]; } break;
                case 3: if (j < Ny - 1) { kn = (long long)cur + Nx; h = d.ys[j + 1] - d.ys[j]; } break;
                case 4: if (l > 0) { kn = (long long)cur - (long long)Nx * Ny; h = d.zs[l] - d.zs[l - 1]; } break;
                default: if (l < Nz - 1) { kn = (long long)cur + (long long)Nx * Ny; h = d.zs[l + 1] - d.zs[l]; } break;
                }
                if (kn < 0 || kind[kn] != K_SEMI || con[kn]) break;
                s_ += h;
                H.tc_k.push_back((int)kn); H.tc_s.push_back(s_);
                cnt++;
                if (s_ >= TE_COL) break;
                cur = (size_t)kn;
            }
            H.te_cn.push_back(cnt);
        });
        H.ce1[c] = (int)H.te_k.size();
    }
    // velocity-saturation weight of the column nodes (semiconductor_3d.c:1750-1764)
    H.vw.assign(N, 1.f);
    H.ax.assign(N, 0);
    for (size_t t = 0; t < H.te_k.size(); t++) {
        const int a = d.cons[H.te_c[t]].face / 2;
        for (int q = H.te_c0[t]; q < H.te_c0[t] + H.te_cn[t]; q++) {
            const double s_ = H.tc_s[q];
            double w;
            if (g_knobs.te_colvs) w = s_ <= 0.5 * TE_COL ? 0. : (s_ >= TE_COL ? 1. : (s_ - 0.5 * TE_COL) / (0.5 * TE_COL));
            else w = s_ > 0. ? 1. : 0.;
            const int k = H.tc_k[q];
            if ((float)w < H.vw[k]) { H.vw[k] = (float)w; H.ax[k] = (signed char)a; }
        }
    }
    // column entries of every column node, ascending
    std::vector<int> slot(N, -1);
    std::vector<std::vector<int>> lists;
    for (int q = 0; q < (int)H.tc_k.size(); q++) {
        const int k = H.tc_k[q];
        if (slot[k] < 0) { slot[k] = (int)lists.size(); lists.emplace_back(); H.tn_k.push_back(k); }
        lists[slot[k]].push_back(q);
    }
    H.tn_ptr.assign(1, 0);
    for (auto &L : lists) {
        for (int q : L) H.tn_q.push_back(q);
        H.tn_ptr.push_back((int)H.tn_q.size());
    }
}

// Gate-tunnelling paths (tun_build, semiconductor_3d.c:1146-1247): from every semiconductor
// node of no contact with an insulator neighbour of no contact, straight through the
// insulator; the path counts if it ends on the metal of a Dirichlet gate within TUN_LMAX.
// Layers: the semiconductor half cell, then one per run of equal insulator material, the
// last ending on the metal node.  A Robin gate adds one path per gate node with the
// contact's stack.  Each path has its supply column inward from the interface.
struct TunHost {
    std::vector<int> tp_k, tp_c, tp_nl, tp_m, tp_c0, tp_cn, col_k;
    std::vector<double> tp_t, tp_A, col_l, col_h;
};
static void tun_build(Inst &d, const std::vector<unsigned char> &kind, const std::vector<int> &con,
                      const std::vector<int> &rob_k, const std::vector<double> &rob_A, const std::vector<int> &rob_c,
                      TunHost &H) {
    for (int c = 0; c < d.n_cons; c++) d.cons[c].ntp = 0;
    if (!(d.models & 32)) return;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    auto nb = [&](size_t k, int dir, size_t &kn, double &h, double &ar) {
        const int l = int(k / ((size_t)Nx * Ny)), rem = int(k - (size_t)l * Nx * Ny), j = rem / Nx, i = rem % Nx;
        switch (dir) {
        case 0: if (i == 0) return false; kn = k - 1; h = d.xs[i] - d.xs[i - 1]; ar = d.Ly[j] * d.Lz[l]; return true;
        case 1: if (i == Nx - 1) return false; kn = k + 1; h = d.xs[i + 1] - d.xs[i]; ar = d.Ly[j] * d.Lz[l]; return true;
        case 2: if (j == 0) return false; kn = k - Nx; h = d.ys[j] - d.ys[j - 1]; ar = d.Lx[i] * d.Lz[l]; return true;
        case 3: if (j == Ny - 1) return false; kn = k + Nx; h = d.ys[j + 1] - d.ys[j]; ar = d.Lx[i] * d.Lz[l]; return true;
        case 4: if (l == 0) return false; kn = k - (size_t)Nx * Ny; h = d.zs[l] - d.zs[l - 1]; ar = d.Lx[i] * d.Ly[j]; return true;
        default: if (l == Nz - 1) return false; kn = k + (size_t)Nx * Ny; h = d.zs[l + 1] - d.zs[l]; ar = d.Lx[i] * d.Ly[j]; return true;
        }
    };
    auto push = [&](size_t k, double A, int c, int dir, int nl, const int *m, const double *t) {
        H.tp_k.push_back((int)k); H.tp_A.push_back(A); H.tp_c.push_back(c); H.tp_nl.push_back(nl);
        for (int i = 0; i < 6; i++) { H.tp_m.push_back(i < nl ? m[i] : 0); H.tp_t.push_back(i < nl ? t[i] : 0.); }
        H.tp_c0.push_back((int)H.col_k.size());
        int cnt = 0;
        if (dir >= 0) {                                    // supply column, inward (direction dir^1)
            size_t cur = k;
            double depth = 0.;
            const int in = dir ^ 1, ax = dir / 2;
            for (;;) {
                const int l = int(cur / ((size_t)Nx * Ny)), rem = int(cur - (size_t)l * Nx * Ny);
                const double L = ax == 0 ? d.Lx[rem % Nx] : (ax == 1 ? d.Ly[rem / Nx] : d.Lz[l]);
                size_t kn = 0;
                double h = 0., ar;
                bool more = nb(cur, in, kn, h, ar);
                if (!more || kind[kn] != K_SEMI || con[kn]) more = false;
                H.col_k.push_back((int)cur); H.col_l.push_back(L); H.col_h.push_back(more ? h : 0.);
                cnt++;
                depth += L;
                if (!more || depth >= TUN_COL) break;
                cur = kn;
            }
        }
        H.tp_cn.push_back(cnt);
        d.cons[c].ntp++;
    };
    for (int l = 0; l < Nz; l++)
        for (int j = 0; j < Ny; j++)
            for (int i = 0; i < Nx; i++) {
                const size_t k = (size_t)l * Nx * Ny + (size_t)j * Nx + i;
                if (kind[k] != K_SEMI || con[k]) continue;
                for (int dir = 0; dir < 6; dir++) {
                    size_t kb;
                    double h, ar;
                    if (!nb(k, dir, kb, h, ar) || kind[kb] != K_INS || con[kb]) continue;
                    int m[6];
                    double t[6];
                    int nl = 1, ok = 0;
                    m[0] = d.mat_idx[k]; t[0] = 0.5 * h;     // semiconductor half cell
                    double tins = 0., hin = h;
                    size_t cur = kb;
                    for (int guard = 0; guard < 100000; guard++) {
                        size_t kn;
                        double h2, ar2;
                        if (!nb(cur, dir, kn, h2, ar2)) break;   // domain edge
                        const int mi = d.mat_idx[cur];
                        const bool end = kind[kn] == K_METAL && con[kn] && d.cons[con[kn] - 1].bc == 2;
                        const double seg = 0.5 * hin + (end ? h2 : 0.5 * h2);
                        if (nl > 1 && m[nl - 1] == mi) t[nl - 1] += seg;
                        else {
                            if (nl >= 6) break;
                            m[nl] = mi; t[nl] = seg; nl++;
                        }
                        tins += seg;
                        if (tins > TUN_LMAX) break;
                        if (end) { ok = con[kn]; break; }
                        if (kind[kn] != K_INS || con[kn]) break;
                        cur = kn; hin = h2;
                    }
                    if (ok) push(k, ar, ok - 1, dir, nl, m, t);
                }
            }
    for (size_t r = 0; r < rob_k.size(); r++) {
        const Contact &cn = d.cons[rob_c[r]];
        if (cn.snl < 1) continue;
        push((size_t)rob_k[r], rob_A[r], rob_c[r], cn.face, cn.snl, cn.smat, cn.st);
    }
}

// Gate-tunnelling paths on a graph mesh (tun_build_graph / tun_push_g,
// semiconductor_3d.c:1285-1349): from every semiconductor node of no contact along each edge
// into an insulator node of no contact, on through the insulator by the neighbour best
// aligned with that edge, each layer bounded at the midpoints of the projected positions;
// the path counts if it ends on the metal of a Dirichlet gate within TUN_LMAX.  A Robin
// gate adds one path per gate node along the face's outward normal.  The supply column
// runs from the node against the path direction, a node's share half the spacing to each
// column neighbour (the interface half cell first).
static void tun_build_graph(Inst &d, const std::vector<unsigned char> &kind, const std::vector<int> &con,
                            const std::vector<int> &rob_k, const std::vector<double> &rob_A,
                            const std::vector<int> &rob_c, TunHost &H) {
    for (int c = 0; c < d.n_cons; c++) d.cons[c].ntp = 0;
    if (!(d.models & 32)) return;
    const GraphHost &G = d.ggh;
    const int N = (int)d.N;
    auto push = [&](size_t k, double A, int c, const double *u, double hw, int nl, const int *m, const double *t) {
        H.tp_k.push_back((int)k); H.tp_A.push_back(A); H.tp_c.push_back(c); H.tp_nl.push_back(nl);
        for (int i = 0; i < TUN_MAXL; i++) { H.tp_m.push_back(i < nl ? m[i] : 0); H.tp_t.push_back(i < nl ? t[i] : 0.); }
        H.tp_c0.push_back((int)H.col_k.size());
        const double v[3] = {-u[0], -u[1], -u[2]};
        size_t cur = k;
        long prev = -1;
        double depth = 0., hprev = 2. * hw;
        int cnt = 0;
        for (int guard = 0; guard < 10000; guard++) {
            long nb = g_step(G, cur, prev, v, 0.8);
            if (nb >= 0 && (kind[nb] != K_SEMI || con[nb])) nb = -1;
            const double h = nb >= 0 ? g_proj(G, cur, (size_t)nb, v) : 0.;
            if (nb >= 0 && !(h > 0.)) nb = -1;
            double L = 0.5 * hprev + (nb >= 0 ? 0.5 * h : 0.5 * hprev);
            if (!(L > 0.)) L = std::cbrt(d.Lx[cur]);
            H.col_k.push_back((int)cur); H.col_l.push_back(L); H.col_h.push_back(nb >= 0 ? h : 0.);
            cnt++;
            depth += L;
            if (nb < 0 || depth >= TUN_COL) break;
            prev = (long)cur;
            cur = (size_t)nb;
            hprev = h;
        }
        H.tp_cn.push_back(cnt);
        d.cons[c].ntp++;
    };
    for (int k = 0; k < N; k++) {
        if (kind[k] != K_SEMI || con[k]) continue;
        for (int e0 = G.rp[k]; e0 < G.rp[k + 1]; e0++) {
            const int kb = G.cj[e0];
            if (kind[kb] != K_INS || con[kb]) continue;
            const double h = G.h[e0];
            double u[3];
            for (int q = 0; q < 3; q++) u[q] = (G.pos[3 * kb + q] - G.pos[3 * k + q]) / h;
            int m[TUN_MAXL];
            double t[TUN_MAXL];
            int nl = 1, ok = 0;
            m[0] = d.mat_idx[k]; t[0] = 0.5 * h;              // semiconductor half cell
            double s0 = 0.5 * h, scur = g_proj(G, k, kb, u), tins = 0.;
            size_t cur = kb;
            long prev = k;
            for (int guard = 0; guard < 100000; guard++) {
                const long nb = g_step(G, cur, prev, u, 0.8);
                if (nb < 0) break;
                const double snb = g_proj(G, k, (size_t)nb, u);
                const bool end = kind[nb] == K_METAL && con[nb] && d.cons[con[nb] - 1].bc == 2;
                const double s1 = end ? snb : 0.5 * (scur + snb), seg = s1 - s0;
                if (!(seg > 0.)) break;
                const int mi = d.mat_idx[cur];
                if (nl > 1 && m[nl - 1] == mi) t[nl - 1] += seg;
                else {
                    if (nl >= TUN_MAXL) break;
                    m[nl] = mi; t[nl] = seg; nl++;
                }
                tins += seg;
                if (tins > TUN_LMAX) break;
                if (end) { ok = con[nb]; break; }
                if (kind[nb] != K_INS || con[nb]) break;
                s0 = s1; scur = snb; prev = (long)cur; cur = (size_t)nb;
            }
            if (ok) push((size_t)k, G.ar[e0], ok - 1, u, 0.5 * h, nl, m, t);
        }
    }
    for (size_t r = 0; r < rob_k.size(); r++) {
        const Contact &cn = d.cons[rob_c[r]];
        if (cn.snl < 1) continue;
        double u[3] = {0., 0., 0.};
        u[cn.face / 2] = (cn.face & 1) ? 1. : -1.;            // outward normal of the face
        push((size_t)rob_k[r], rob_A[r], rob_c[r], u, 0., cn.snl, cn.smat, cn.st);
    }
}

// the per-node gather of the continuity sink / source: tunnelling column entries, paths
// ending at the node, metal-contact column entries, each list in ascending order
struct ScHost {
    std::vector<int> k, pk, pg, pe, qk, qg, qe;
};
static void sc_build(size_t N, const TunHost &U, const std::vector<int> &tc_k, ScHost &H) {
    std::vector<int> slot(N, -1);
    std::vector<std::vector<int>> lk, lg, le;
    auto at = [&](int k) {
        if (slot[k] < 0) { slot[k] = (int)H.k.size(); H.k.push_back(k); lk.emplace_back(); lg.emplace_back(); le.emplace_back(); }
        return slot[k];
    };
    for (int q = 0; q < (int)U.col_k.size(); q++) lk[at(U.col_k[q])].push_back(q);
    for (int p = 0; p < (int)U.tp_k.size(); p++) lg[at(U.tp_k[p])].push_back(p);
    for (int q = 0; q < (int)tc_k.size(); q++) le[at(tc_k[q])].push_back(q);
    H.pk.assign(1, 0); H.pg.assign(1, 0); H.pe.assign(1, 0);
    for (size_t i = 0; i < H.k.size(); i++) {
        for (int q : lk[i]) H.qk.push_back(q);
        for (int p : lg[i]) H.qg.push_back(p);
        for (int q : le[i]) H.qe.push_back(q);
        H.pk.push_back((int)H.qk.size()); H.pg.push_back((int)H.qg.size()); H.pe.push_back((int)H.qe.size());
    }
}

// Deep-level traps (traps_build, semiconductor_3d.c:1428-1468): the requests compiled into
// per-node lists (semiconductor nodes only), entries of one species on one node summed in
// the order of their first request; capture coefficients sigma v_th with
// v_th = sqrt(3 kT / m*) from the node material's tunnelling masses.  Uploaded with the
// species table into one allocation.
static int traps_upload(Inst &d, const std::vector<unsigned char> &kind, DevP &P, cudaStream_t st) {
    if (d.g.trblock) { cudaFree(d.g.trblock); d.g.trblock = nullptr; }
    P.tr_rp = P.tr_s = nullptr;
    P.tr_N = P.tr_cn = P.tr_cp = nullptr;
    P.tsp = nullptr;
    d.n_tr = 0;
    if (d.trq_k.empty()) return 1;
    const size_t N = d.N;
    std::vector<int> rp(N + 1, 0);
    for (size_t q = 0; q < d.trq_k.size(); q++) {
        const size_t k = (size_t)(unsigned)d.trq_k[q];
        if (k < N && kind[k] == K_SEMI) rp[k + 1]++;
    }
    for (size_t k = 0; k < N; k++) rp[k + 1] += rp[k];
    std::vector<int> fill(rp), ts(rp[N] > 0 ? rp[N] : 1);
    std::vector<double> tN(ts.size());
    for (size_t q = 0; q < d.trq_k.size(); q++) {
        const size_t k = (size_t)(unsigned)d.trq_k[q];
        if (k >= N || kind[k] != K_SEMI) continue;
        const int sid = d.trq_s[q];
        int w = -1;
        for (int e = rp[k]; e < fill[k]; e++) if (ts[e] == sid) { w = e; break; }
        if (w >= 0) { tN[w] += d.trq_N[q]; continue; }
        w = fill[k]++;
        ts[w] = sid; tN[w] = d.trq_N[q];
    }
    int o = 0;                                            // compact the merged duplicates
    for (size_t k = 0; k < N; k++) {
        const int a = rp[k], b = fill[k];
        rp[k] = o;
        for (int e = a; e < b; e++) { ts[o] = ts[e]; tN[o] = tN[e]; o++; }
    }
    rp[N] = o;
    d.n_tr = o;
    if (o == 0) return 1;
    std::vector<double> tcn(o), tcp(o);
    const double M0_ = 9.1093837015e-31;
    for (size_t k = 0; k < N; k++) {
        if (rp[k] == rp[k + 1]) continue;
        const Material &m = d.mats[d.mat_idx[k]];
        const double me = m.mtun_e > 0. ? m.mtun_e : 0.3, mh = m.mtun_h > 0. ? m.mtun_h : 0.5;
        const double vn = std::sqrt(3. * KB * m.T / (me * M0_)), vp = std::sqrt(3. * KB * m.T / (mh * M0_));
        for (int e = rp[k]; e < rp[k + 1]; e++) {
            const TrapSpec &sp = d.tsp[ts[e]];
            tcn[e] = sp.sn * vn; tcp[e] = sp.sp * vp;
        }
    }
    std::vector<TrapD> tab(d.n_tsp > 0 ? d.n_tsp : 1);
    for (int q = 0; q < d.n_tsp; q++) { tab[q].type = d.tsp[q].type; tab[q].ref = d.tsp[q].ref; tab[q].E = d.tsp[q].E; }
    size_t off = 0;
    auto room = [&](size_t bytes) { const size_t x = off; off += align_up(bytes > 0 ? bytes : 1); return x; };
    const size_t o_rp = room((N + 1) * 4), o_s = room((size_t)o * 4), o_N = room((size_t)o * 8),
                 o_cn = room((size_t)o * 8), o_cp = room((size_t)o * 8), o_tab = room(tab.size() * sizeof(TrapD));
    char *b = nullptr;
    if (cudaMalloc(&b, off) != cudaSuccess) {
        std::fprintf(stderr, "semisim-b200: out of device memory for the traps\n");
        return 0;
    }
    d.g.trblock = b;
    bool ok = true;
    auto up = [&](size_t x, const void *src, size_t bytes) {
        if (bytes && cudaMemcpyAsync(b + x, src, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) ok = false;
    };
    up(o_rp, rp.data(), (N + 1) * 4); up(o_s, ts.data(), (size_t)o * 4); up(o_N, tN.data(), (size_t)o * 8);
    up(o_cn, tcn.data(), (size_t)o * 8); up(o_cp, tcp.data(), (size_t)o * 8); up(o_tab, tab.data(), tab.size() * sizeof(TrapD));
    P.tr_rp = (const int *)(b + o_rp); P.tr_s = (const int *)(b + o_s);
    P.tr_N = (const double *)(b + o_N); P.tr_cn = (const double *)(b + o_cn); P.tr_cp = (const double *)(b + o_cp);
    P.tsp = (const TrapD *)(b + o_tab);
    if (!ok) return 0;
    if (d.verbose) std::fprintf(stderr, "semisim-b200: %d trap entries (%d species) on the mesh\n", d.n_tr, d.n_tsp);
    return 1;
}

// Coulomb scattering on interface charge (coul_build, semiconductor_3d.c:1540-1623; models
// bit 4 with a material whose electrons have the Coulomb term): the interface entries are
// the semiconductor nodes of such a material, of no contact, next to an insulator node or
// under a face gate; an entry's area is its dual faces to insulator nodes (plus a Robin
// gate's area), its fixed charge the node's own |Nf| and its insulator neighbours' shared
// by area (plus the gate's oxide charge).  Every node of a Coulomb material then takes the
// nearest entry with an area within 150 nm, found by a breadth-first search from the entries.
static int coul_upload(Inst &d, const std::vector<unsigned char> &kind, const std::vector<int> &con,
                       const std::vector<int> &gate, const std::vector<int> &rob_k, const std::vector<double> &rob_A,
                       const std::vector<int> &rob_c, DevP &P, cudaStream_t st) {
    if (d.g.coblock) { cudaFree(d.g.coblock); d.g.coblock = nullptr; }
    P.qi = P.if_k = nullptr;
    P.if_A = P.if_Qf = nullptr;
    P.if_NC = nullptr;
    P.n_if = 0;
    if (!(d.models & 16)) return 1;
    bool any = false;
    for (int q = 0; q < d.n_mats; q++) if (d.mats[q].lbc_on && (d.mats[q].lb_on & 1)) any = true;
    if (!any) return 1;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const size_t N = d.N;
    const GraphHost &G = d.ggh;
    auto nbrs = [&](size_t k, size_t *kb, double *ar) {     // at most 64 (NBR_MAX) on a graph
        int c = 0;
        if (d.unstr) {
            for (int e = G.rp[k]; e < G.rp[k + 1] && c < 64; e++) { kb[c] = (size_t)G.cj[e]; ar[c++] = G.ar[e]; }
            return c;
        }
        const int l = int(k / ((size_t)Nx * Ny)), rem = int(k - (size_t)l * Nx * Ny), j = rem / Nx, i = rem % Nx;
        if (i > 0) { kb[c] = k - 1; ar[c++] = d.Ly[j] * d.Lz[l]; }
        if (i < Nx - 1) { kb[c] = k + 1; ar[c++] = d.Ly[j] * d.Lz[l]; }
        if (j > 0) { kb[c] = k - Nx; ar[c++] = d.Lx[i] * d.Lz[l]; }
        if (j < Ny - 1) { kb[c] = k + Nx; ar[c++] = d.Lx[i] * d.Lz[l]; }
        if (l > 0) { kb[c] = k - (size_t)Nx * Ny; ar[c++] = d.Lx[i] * d.Ly[j]; }
        if (l < Nz - 1) { kb[c] = k + (size_t)Nx * Ny; ar[c++] = d.Lx[i] * d.Ly[j]; }
        return c;
    };
    auto xyz = [&](size_t k, double *pq) {
        if (d.unstr) { for (int q = 0; q < 3; q++) pq[q] = G.pos[3 * k + q]; return; }
        const int l = int(k / ((size_t)Nx * Ny)), rem = int(k - (size_t)l * Nx * Ny);
        pq[0] = d.xs[rem % Nx]; pq[1] = d.ys[rem / Nx]; pq[2] = d.zs[l];
    };
    auto vol = [&](size_t k) {
        const int l = int(k / ((size_t)Nx * Ny)), rem = int(k - (size_t)l * Nx * Ny);
        return d.Lx[rem % Nx] * d.Ly[rem / Nx] * d.Lz[l];
    };
    auto d2 = [](const double *a, const double *b) {
        const double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
        return x * x + y * y + z * z;
    };
    std::vector<int> qi(N, -1), ik;
    size_t kb[64], kb2[64];
    double ar[64], ar2[64];
    for (size_t k = 0; k < N; k++) {
        if (kind[k] != K_SEMI || con[k] || !d.mats[d.mat_idx[k]].lbc_on) continue;
        bool is = gate[k] != 0;
        if (!is) {
            const int c = nbrs(k, kb, ar);
            for (int q = 0; q < c; q++) if (kind[kb[q]] == K_INS) { is = true; break; }
        }
        if (is) { qi[k] = (int)ik.size(); ik.push_back((int)k); }
    }
    const int cnt = (int)ik.size();
    if (!cnt) return 1;
    std::vector<double> iA(cnt, 0.), iQ(cnt, 0.);
    for (int e = 0; e < cnt; e++) {
        const size_t k = (size_t)ik[e];
        const int c = nbrs(k, kb, ar);
        double A = 0., Qf = std::fabs(d.Nf[k]) * vol(k);
        for (int q = 0; q < c; q++) {
            const size_t ko = kb[q];
            if (kind[ko] != K_INS) continue;
            A += ar[q];
            if (d.Nf[ko] != 0.) {
                const int c2 = nbrs(ko, kb2, ar2);
                double As = 0.;
                for (int q2 = 0; q2 < c2; q2++) if (kind[kb2[q2]] == K_SEMI) As += ar2[q2];
                if (As > 0.) Qf += std::fabs(d.Nf[ko]) * vol(ko) * ar[q] / As;
            }
        }
        iA[e] = A; iQ[e] = Qf;
    }
    for (size_t r = 0; r < rob_k.size(); r++) {
        const int e = qi[rob_k[r]];
        if (e < 0) continue;
        iA[e] += rob_A[r];
        iQ[e] += std::fabs(d.cons[rob_c[r]].qox) / Q * rob_A[r];
    }
    // breadth-first search from the entries with an area (a ring of N slots)
    std::vector<size_t> qu(N);
    std::vector<char> inq(N, 0);
    size_t head = 0, tail = 0, used = 0;
    for (int e = 0; e < cnt; e++) {
        const size_t k = (size_t)ik[e];
        if (iA[e] > 0.) { qu[tail] = k; tail = (tail + 1) % N; used++; inq[k] = 1; }
        else qi[k] = -1;
    }
    const double R2 = 150e-9 * 150e-9;
    while (used) {
        const size_t u = qu[head];
        head = (head + 1) % N; used--; inq[u] = 0;
        const int lab = qi[u];
        if (lab < 0) continue;
        double pl[3], pv[3], pc[3];
        xyz((size_t)ik[lab], pl);
        const int c = nbrs(u, kb, ar);
        for (int q = 0; q < c; q++) {
            const size_t v = kb[q];
            if (kind[v] != K_SEMI || !d.mats[d.mat_idx[v]].lbc_on) continue;
            xyz(v, pv);
            const double r2 = d2(pv, pl);
            if (r2 > R2) continue;
            const int cur = qi[v];
            if (cur == lab) continue;
            if (cur >= 0) { xyz((size_t)ik[cur], pc); if (r2 >= d2(pv, pc)) continue; }
            qi[v] = lab;
            if (!inq[v]) { qu[tail] = v; tail = (tail + 1) % N; used++; inq[v] = 1; }
        }
    }
    size_t off = 0;
    auto room = [&](size_t bytes) { const size_t x = off; off += align_up(bytes > 0 ? bytes : 1); return x; };
    const size_t o_qi = room(N * 4), o_ik = room((size_t)cnt * 4), o_A = room((size_t)cnt * 8),
                 o_Q = room((size_t)cnt * 8), o_NC = room((size_t)cnt * 8);
    char *b = nullptr;
    if (cudaMalloc(&b, off) != cudaSuccess) {
        std::fprintf(stderr, "semisim-b200: out of device memory for the interface entries\n");
        return 0;
    }
    d.g.coblock = b;
    bool ok = cudaMemsetAsync(b, 0, off, st) == cudaSuccess;
    auto up = [&](size_t x, const void *src, size_t bytes) {
        if (bytes && cudaMemcpyAsync(b + x, src, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) ok = false;
    };
    up(o_qi, qi.data(), N * 4); up(o_ik, ik.data(), (size_t)cnt * 4);
    up(o_A, iA.data(), (size_t)cnt * 8); up(o_Q, iQ.data(), (size_t)cnt * 8);
    P.qi = (const int *)(b + o_qi); P.if_k = (const int *)(b + o_ik);
    P.if_A = (const double *)(b + o_A); P.if_Qf = (const double *)(b + o_Q); P.if_NC = (double *)(b + o_NC);
    P.n_if = cnt;
    if (d.verbose) std::fprintf(stderr, "semisim-b200: %d interface nodes for Coulomb scattering\n", cnt);
    return ok ? 1 : 0;
}

// device copy of the tunnelling paths and the exchange gather (one allocation)
static int tun_upload(Inst &d, const TunHost &U, const ScHost &G, cudaStream_t st) {
    if (d.g.tunblock) { cudaFree(d.g.tunblock); d.g.tunblock = nullptr; }
    d.g.tun_on = false;
    d.g.tun = TunD{};
    d.g.sc = ScD{};
    const size_t np = U.tp_k.size(), nc = U.col_k.size(), ns = G.k.size();
    if (ns == 0) return 1;
    size_t off = 0;
    auto room = [&](size_t bytes) { const size_t o = off; off += align_up(bytes > 0 ? bytes : 1); return o; };
    const size_t o_tpk = room(np * 4), o_tpc = room(np * 4), o_tpnl = room(np * 4), o_tpm = room(np * 24),
                 o_tpc0 = room(np * 4), o_tpcn = room(np * 4), o_tpt = room(np * 48), o_tpA = room(np * 8),
                 o_tpG = room(np * 16), o_colk = room(nc * 4), o_coll = room(nc * 8), o_colh = room(nc * 8),
                 o_colK = room(nc * 16);
    const size_t o_sk = room(ns * 4), o_spk = room((ns + 1) * 4), o_spg = room((ns + 1) * 4), o_spe = room((ns + 1) * 4),
                 o_sqk = room(G.qk.size() * 4), o_sqg = room(G.qg.size() * 4), o_sqe = room(G.qe.size() * 4);
    char *b = nullptr;
    if (cudaMalloc(&b, off) != cudaSuccess) {
        std::fprintf(stderr, "semisim-b200: out of device memory for the gate-tunnelling paths\n");
        return 0;
    }
    d.g.tunblock = b;
    bool ok = cudaMemsetAsync(b, 0, off, st) == cudaSuccess;
    auto up = [&](size_t o, const void *src, size_t bytes) {
        if (bytes && cudaMemcpyAsync(b + o, src, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) ok = false;
    };
    up(o_tpk, U.tp_k.data(), np * 4); up(o_tpc, U.tp_c.data(), np * 4); up(o_tpnl, U.tp_nl.data(), np * 4);
    up(o_tpm, U.tp_m.data(), np * 24); up(o_tpc0, U.tp_c0.data(), np * 4); up(o_tpcn, U.tp_cn.data(), np * 4);
    up(o_tpt, U.tp_t.data(), np * 48); up(o_tpA, U.tp_A.data(), np * 8);
    up(o_colk, U.col_k.data(), nc * 4); up(o_coll, U.col_l.data(), nc * 8); up(o_colh, U.col_h.data(), nc * 8);
    up(o_sk, G.k.data(), ns * 4); up(o_spk, G.pk.data(), (ns + 1) * 4); up(o_spg, G.pg.data(), (ns + 1) * 4);
    up(o_spe, G.pe.data(), (ns + 1) * 4); up(o_sqk, G.qk.data(), G.qk.size() * 4);
    up(o_sqg, G.qg.data(), G.qg.size() * 4); up(o_sqe, G.qe.data(), G.qe.size() * 4);
    TunD &T = d.g.tun;
    T.n_tp = (int)np; T.n_col = (int)nc;
    T.tp_k = (const int *)(b + o_tpk); T.tp_c = (const int *)(b + o_tpc); T.tp_nl = (const int *)(b + o_tpnl);
    T.tp_m = (const int *)(b + o_tpm); T.tp_c0 = (const int *)(b + o_tpc0); T.tp_cn = (const int *)(b + o_tpcn);
    T.tp_t = (const double *)(b + o_tpt); T.tp_A = (const double *)(b + o_tpA); T.tp_G = (double *)(b + o_tpG);
    T.col_k = (const int *)(b + o_colk); T.col_l = (const double *)(b + o_coll); T.col_h = (const double *)(b + o_colh);
    T.col_K = (double *)(b + o_colK);
    ScD &S = d.g.sc;
    S.n = (int)ns;
    S.k = (const int *)(b + o_sk); S.pk = (const int *)(b + o_spk); S.pg = (const int *)(b + o_spg);
    S.pe = (const int *)(b + o_spe); S.qk = (const int *)(b + o_sqk); S.qg = (const int *)(b + o_sqg);
    S.qe = (const int *)(b + o_sqe);
    if (!ok) return 0;
    d.g.tun_on = np > 0;
    return 1;
}

// device copy of the metal-contact data; the per-node band lowering and sink / source
// start at zero (the reference resets them at prepare)
static int te_upload(Inst &d, const TeHost &H, DevP &P, cudaStream_t st) {
    if (d.g.teblock) { cudaFree(d.g.teblock); d.g.teblock = nullptr; }
    d.g.te_on = false;
    P.tk = P.tg = P.imgn = P.imgp = nullptr;
    P.te_vw = nullptr;
    P.te_ax = nullptr;
    const size_t N = d.N, nte = H.te_k.size(), ntc = H.tc_k.size(), ntn = H.tn_k.size();
    if (nte == 0) return 1;
    size_t off = 0;
    auto room = [&](size_t bytes) { const size_t o = off; off += align_up(bytes > 0 ? bytes : 1); return o; };
    const size_t o_imgn = room(N * 8), o_imgp = room(N * 8);
    const size_t o_vw = room(N * 4), o_ax = room(N);
    const size_t o_tek = room(nte * 4), o_tec = room(nte * 4), o_tec0 = room(nte * 4), o_tecn = room(nte * 4);
    const size_t o_teA = room(nte * 8), o_teK = room(nte * 16), o_teG = room(nte * 16);
    const size_t o_tck = room(ntc * 4), o_tcs = room(ntc * 8), o_tcK = room(ntc * 16), o_tcG = room(ntc * 16),
                 o_tcI = room(ntc * 16);
    const size_t o_tnk = room(ntn * 4), o_tnp = room((ntn + 1) * 4), o_tnq = room(ntc * 4);
    char *b = nullptr;
    if (cudaMalloc(&b, off) != cudaSuccess) {
        std::fprintf(stderr, "semisim-b200: out of device memory for the metal contacts\n");
        return 0;
    }
    d.g.teblock = b;
    CK(cudaMemsetAsync(b, 0, off, st));
    TeD &T = d.g.te;
    T = TeD{};
    T.n_te = (int)nte; T.n_tc = (int)ntc; T.n_touch = (int)ntn; T.models = d.models;
    T.te_k = (int *)(b + o_tek); T.te_c = (int *)(b + o_tec); T.te_c0 = (int *)(b + o_tec0); T.te_cn = (int *)(b + o_tecn);
    T.te_A = (double *)(b + o_teA); T.te_K = (double *)(b + o_teK); T.te_G = (double *)(b + o_teG);

    T.tc_k = (int *)(b + o_tck); T.tc_s = (double *)(b + o_tcs);
    T.tc_K = (double *)(b + o_tcK); T.tc_G = (double *)(b + o_tcG); T.tc_I = (double *)(b + o_tcI);
    T.tn_k = (int *)(b + o_tnk); T.tn_ptr = (int *)(b + o_tnp); T.tn_q = (int *)(b + o_tnq);
    for (int c = 0; c < NC_MAX; c++) { T.ce0[c] = H.ce0[c]; T.ce1[c] = H.ce1[c]; }
    bool ok = true;
    auto up = [&](const void *dst, const void *src, size_t bytes) {
        if (bytes && cudaMemcpyAsync((void *)dst, src, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) ok = false;
    };
    up(T.te_k, H.te_k.data(), nte * 4); up(T.te_c, H.te_c.data(), nte * 4);
    up(T.te_c0, H.te_c0.data(), nte * 4); up(T.te_cn, H.te_cn.data(), nte * 4);
    up(T.te_A, H.te_A.data(), nte * 8);
    up(T.tc_k, H.tc_k.data(), ntc * 4); up(T.tc_s, H.tc_s.data(), ntc * 8);
    up(T.tn_k, H.tn_k.data(), ntn * 4); up(T.tn_ptr, H.tn_ptr.data(), (ntn + 1) * 4);
    up(T.tn_q, H.tn_q.data(), ntc * 4);
    up(b + o_vw, H.vw.data(), N * 4); up(b + o_ax, H.ax.data(), N);
    P.imgn = (double *)(b + o_imgn); P.imgp = (double *)(b + o_imgp);
    P.te_vw = (const float *)(b + o_vw);
    P.te_ax = (const signed char *)(b + o_ax);
    if (!ok) return 0;
    d.g.te_on = true;
    return 1;
}

int prepare(Inst &d) {
    if (!d.allocated || d.n_mats < 1) return 0;
    if (!d.dirty && d.g.ready) return 1;       // set-up unchanged since the last upload
    const size_t N = d.N;
    mat_prepare(d);
    std::vector<unsigned char> kind(N);
    std::vector<int> con(N, 0), gate(N, 0);
    d.bgn.assign(N, 0.0);
    for (size_t k = 0; k < N; k++) {
        int mi = d.mat_idx[k];
        if (mi < 0 || mi >= d.n_mats) mi = d.mat_idx[k] = 0;
        const Material &m = d.mats[mi];
        kind[k] = m.insulator ? K_INS : K_SEMI;
        d.bgn[k] = (!m.insulator && (d.models & 1)) ? bgn_half(m, d.Nd[k] + d.Na[k]) : 0.;
    }
    int nrob = 0;
    for (int c = 0; c < d.n_cons; c++)                  // metal face contacts (semiconductor_3d.c:1655)
        d.cons[c].te = (d.models & 64) && d.cons[c].bc == 1 && d.cons[c].face <= 5;
    for (int c = 0; c < d.n_cons; c++) {
        Contact &cn = d.cons[c];
        cn.A = 0.;
        for_con_nodes(d, cn, [&](int, int, int, size_t k, double area) {
            if (cn.face <= 5) cn.A += area;
            if (cn.bc == 2 && cn.face <= 5 && kind[k] == K_SEMI) {
                gate[k] = c + 1; nrob++;
            } else if (cn.bc == 2 || kind[k] != K_SEMI) {
                kind[k] = K_METAL; con[k] = c + 1; gate[k] = 0;
            } else {
                con[k] = c + 1; gate[k] = 0;
            }
        });
    }
    d.robA.assign(N, 0.0);
    d.n_rob = 0;
    std::vector<int> rob_k, rob_c;                      // the Robin list in the reference's order
    std::vector<double> rob_A;
    for (int c = 0; c < d.n_cons; c++) {
        const Contact &cn = d.cons[c];
        if (cn.bc != 2 || cn.face > 5) continue;
        for_con_nodes(d, cn, [&](int, int, int, size_t k, double area) {
            if (gate[k] == c + 1 && !con[k] && d.n_rob < nrob && d.robA[k] == 0.0) {
                d.robA[k] = area; d.n_rob++;
                rob_k.push_back((int)k); rob_A.push_back(area); rob_c.push_back(c);
            }
        });
    }
    // box contacts: area = interface with non-contact semiconductor
    for (int c = 0; c < d.n_cons; c++) {
        Contact &cn = d.cons[c];
        if (cn.face <= 5) continue;
        double A = 0.;
        if (d.unstr) {
            const GraphHost &G = d.ggh;
            for_con_nodes(d, cn, [&](int, int, int, size_t k, double) {
                if (con[k] != c + 1) return;
                for (int e = G.rp[k]; e < G.rp[k + 1]; e++) {
                    const int kb = G.cj[e];
                    if (kind[kb] == K_SEMI && con[kb] != c + 1) A += G.ar[e];
                }
            });
            cn.A = A;
            continue;
        }
        for_con_nodes(d, cn, [&](int i, int j, int l, size_t k, double) {
            if (con[k] != c + 1) return;
            const int Nx = d.Nx, Ny = d.Ny;
            const int ii[6] = {i - 1, i + 1, i, i, i, i}, jj[6] = {j, j, j - 1, j + 1, j, j}, ll[6] = {l, l, l, l, l - 1, l + 1};
            for (int dir = 0; dir < 6; dir++) {
                if (ii[dir] < 0 || ii[dir] >= Nx || jj[dir] < 0 || jj[dir] >= Ny || ll[dir] < 0 || ll[dir] >= d.Nz) continue;
                const size_t kb = (size_t)ll[dir] * Nx * Ny + (size_t)jj[dir] * Nx + ii[dir];
                const double ar = dir < 2 ? d.Ly[j] * d.Lz[l] : (dir < 4 ? d.Lx[i] * d.Lz[l] : d.Lx[i] * d.Ly[j]);
                if (kind[kb] == K_SEMI && con[kb] != c + 1) A += ar;
            }
        });
        cn.A = A;
    }
    // flags, contact-node list, low-field mobility
    d.flags.assign(N, 0);
    d.cnode.clear();
    d.mu0n.assign(N, 0.0);
    d.mu0p.assign(N, 0.0);
    for (size_t k = 0; k < N; k++) {
        // carrier densities are fixed on contact nodes, except the semiconductor nodes of a
        // thermionic-emission contact (car_fix, semiconductor_3d.c:796-799)
        const bool fix = con[k] != 0 && !(d.cons[con[k] - 1].te && kind[k] == K_SEMI);
        d.flags[k] = make_flags(kind[k], con[k], gate[k], d.mat_idx[k], fix);
        if (con[k] && kind[k] == K_SEMI) d.cnode.push_back((int)k);
        if (kind[k] == K_SEMI) {
            const Material &m = d.mats[d.mat_idx[k]];
            const double Nt = d.Nd[k] + d.Na[k];
            d.mu0n[k] = mobility_low(m, Nt, 0);
            d.mu0p[k] = mobility_low(m, Nt, 1);
        }
    }
    std::vector<double> qd, qcn0, qcp0;
    const bool qc_on = (d.models & 8) != 0;
    if (d.unstr) {
        walls_graph(d, kind, qd, qc_on, qcn0, qcp0);
    } else {
        wall_distance(d, kind, gate, qd, qc_on, qcn0, qcp0);
    }
    // incomplete ionisation (semiconductor_3d.c:1472-1510): per node the constants
    // N_c/g_D e^(-dE_s/kT) of the two donor sites and N_v/g_A e^(-dE_A/kT), the level depths
    // falling with the node's own dopant density; the neutral majority density (slot 3)
    // follows on the device
    bool want_ion = false;
    std::vector<double> ionx;
    if (d.models & 512)
        for (int q = 0; q < d.n_mats; q++) if (d.mats[q].ion_on && !d.mats[q].insulator) want_ion = true;
    if (want_ion) {
        ionx.assign((size_t)ION_W * N, 0.0);
        for (size_t k = 0; k < N; k++) {
            if (kind[k] != K_SEMI) continue;
            const Material &m = d.mats[d.mat_idx[k]];
            if (!m.ion_on) continue;
            double *x = ionx.data() + (size_t)ION_W * k;
            if (d.Nd[k] > 0.) {
                const double c = std::cbrt(d.Nd[k]);
                for (int s_ = 0; s_ < 2; s_++) {
                    const double E = std::fmax(m.ion_Ed[s_] - m.ion_ad[s_] * c, 0.);
                    x[s_] = m.Nc / m.ion_gd * std::exp(-E / m.VT);
                }
            }
            if (d.Na[k] > 0.) {
                const double E = std::fmax(m.ion_Ea - m.ion_aa * std::cbrt(d.Na[k]), 0.);
                x[2] = m.Nv / m.ion_ga * std::exp(-E / m.VT);
            }
        }
    }
    TeHost teh;
    TunHost tuh;
    te_build(d, kind, con, teh);
    if (!d.unstr) tun_build(d, kind, con, rob_k, rob_A, rob_c, tuh);
    else tun_build_graph(d, kind, con, rob_k, rob_A, rob_c, tuh);
    ScHost sch;
    sc_build(N, tuh, teh.tc_k, sch);
    if (!gpu_alloc(d)) return 0;
    if ((d.models & 256) && !d.g.gii && cudaMalloc(&d.g.gii, N * sizeof(double)) != cudaSuccess) {
        d.g.gii = nullptr;
        std::fprintf(stderr, "semisim-b200: out of device memory for the impact-ionisation generation\n");
        return 0;
    }
    if (want_ion && !d.g.ion && cudaMalloc(&d.g.ion, (size_t)ION_W * N * sizeof(double)) != cudaSuccess) {
        d.g.ion = nullptr;
        std::fprintf(stderr, "semisim-b200: out of device memory for the ionisation constants\n");
        return 0;
    }
    // upload
    DevP &P = d.g.h;
    P.models = d.models; P.caxis = d.caxis; P.ncon = d.n_cons; P.ref_mat = d.ref_mat;
    P.VTref = d.mats[d.ref_mat].VT; P.Cref = d.Cref;
    P.ncnode = (int)d.cnode.size();
    P.ion = want_ion ? d.g.ion : nullptr;
    P.gii = (d.models & 256) ? d.g.gii : nullptr;
    if (P.gii) CK(cudaMemsetAsync(P.gii, 0, N * sizeof(double), d.g.st));
    if (!te_upload(d, teh, P, d.g.st)) return 0;
    if (!tun_upload(d, tuh, sch, d.g.st)) return 0;
    if (!traps_upload(d, kind, P, d.g.st)) return 0;
    if (!coul_upload(d, kind, con, gate, rob_k, rob_A, rob_c, P, d.g.st)) return 0;
    if (!graph_upload(d, kind, P, d.g.st)) return 0;
    // continuity sink / source of the exchange with gate and metal contacts (zero elsewhere)
    P.tk = P.tg = nullptr;
    if (d.g.te_on || d.g.tun_on) {
        if (!d.g.xchg && cudaMalloc(&d.g.xchg, 2 * N * sizeof(double)) != cudaSuccess) {
            d.g.xchg = nullptr;
            std::fprintf(stderr, "semisim-b200: out of device memory for the exchange terms\n");
            return 0;
        }
        CK(cudaMemsetAsync(d.g.xchg, 0, 2 * N * sizeof(double), d.g.st));
        P.tk = d.g.xchg; P.tg = d.g.xchg + N;
    }
    // band corrections: the MLDA part from the wall scan (zero without models bit 3); the
    // metal contacts add their image-force lowering on the device
    P.qcn = P.qcp = nullptr;
    if (qc_on || d.g.te_on) {
        if (!d.g.qc && cudaMalloc(&d.g.qc, 2 * N * sizeof(double)) != cudaSuccess) {
            d.g.qc = nullptr;
            std::fprintf(stderr, "semisim-b200: out of device memory for the band corrections\n");
            return 0;
        }
        P.qcn = d.g.qc; P.qcp = d.g.qc + N;
        if (qc_on) {
            CK(cudaMemcpyAsync(P.qcn, qcn0.data(), N * 8, cudaMemcpyHostToDevice, d.g.st));
            CK(cudaMemcpyAsync(P.qcp, qcp0.data(), N * 8, cudaMemcpyHostToDevice, d.g.st));
        } else {
            CK(cudaMemsetAsync(d.g.qc, 0, 2 * N * sizeof(double), d.g.st));
        }
    }
    MatD md[NM_MAX];
    std::memset(md, 0, sizeof md);
    for (int i = 0; i < d.n_mats; i++) mat_to_dev(d.mats[i], md[i]);
    cudaStream_t st = d.g.st;
    CK(cudaMemcpyAsync((void *)P.mats, md, sizeof md, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.flags, d.flags.data(), N * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.Nd, d.Nd.data(), N * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.Na, d.Na.data(), N * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.Nf, d.Nf.data(), N * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.bgn, d.bgn.data(), N * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.robA, d.robA.data(), N * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.qd, qd.data(), N * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(P.mu0n, d.mu0n.data(), N * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(P.mu0p, d.mu0p.data(), N * 8, cudaMemcpyHostToDevice, st));
    if (!d.cnode.empty())
        CK(cudaMemcpyAsync((void *)P.cnode, d.cnode.data(), d.cnode.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.xs, d.xs.data(), d.Nx * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.ys, d.ys.data(), d.Ny * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.zs, d.zs.data(), d.Nz * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.Lx, d.Lx.data(), d.Nx * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.Ly, d.Ly.data(), d.Ny * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((void *)P.Lz, d.Lz.data(), d.Nz * 8, cudaMemcpyHostToDevice, st));
    if (want_ion)
        CK(cudaMemcpyAsync(d.g.ion, ionx.data(), ionx.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d.g.d, &P, sizeof(DevP), cudaMemcpyHostToDevice, st));
    if (want_ion) launch_ion_neutral(make_ctx(d));
    CK(cudaStreamSynchronize(st));
    d.g.mg.alpha = g_knobs.mg_alpha;
    d.dirty = 0;
    static std::atomic<unsigned long long> gen{0};
    d.upload_gen = ++gen;
    return 1;
}

void upload_voltages(Inst &d, const double *Va) {
    ConD cd[NC_MAX];
    std::memset(cd, 0, sizeof cd);
    for (int c = 0; c < d.n_cons; c++) {
        cd[c].V = Va[c]; cd[c].phi_m = d.cons[c].phi_m; cd[c].tox = d.cons[c].tox;
        cd[c].qox = d.cons[c].qox; cd[c].bc = d.cons[c].bc; cd[c].te = d.cons[c].te;
    }
    cudaMemcpyAsync((void *)d.g.h.cons, cd, sizeof(ConD) * (d.n_cons > 0 ? d.n_cons : 1), cudaMemcpyHostToDevice,
                    d.g.st);
    cudaStreamSynchronize(d.g.st);     // cd is a stack buffer
}

// ------------------------------------------------------------------ small pieces
void set_vrange(Inst &d, const double *Va) {   // semiconductor_3d.c:3660-3668
    int any = 0;
    double lo = 0., hi = 0.;
    for (int c = 0; c < d.n_cons; c++) {
        if (d.cons[c].bc == 2 && !d.cons[c].ntp) continue;   // a tunnelling gate is a carrier terminal
        if (!any) { lo = hi = Va[c]; any = 1; }
        else { if (Va[c] < lo) lo = Va[c]; if (Va[c] > hi) hi = Va[c]; }
    }
    d.vlo = lo; d.vhi = hi;
}
static double newton_tol(const Inst &d, const double *Va) {   // semiconductor_3d.c:3670-3674
    double s = 1.;
    for (int c = 0; c < d.n_cons; c++) if (std::fabs(Va[c]) > s) s = std::fabs(Va[c]);
    return 2e-14 + 2e-15 * s;
}
void apply_bc(Inst &d, const double *Va) {
    upload_voltages(d, Va);
    launch_apply_bc(make_ctx(d), d.have_solution);
}
void clamp_qf(Inst &d) {
    launch_clamp_qf(make_ctx(d), d.vlo - g_knobs.qf_margin, d.vhi + g_knobs.qf_margin);
}
void rebuild_np(Inst &d) { launch_rebuild_np(make_ctx(d)); }
void upd_mob(Inst &d) {
    if (d.unstr) {
        const Ctx c = make_ctx(d);
        launch_coul_update(c);
        launch_upd_mob_g(c);
    } else {
        launch_upd_mob(make_ctx(d));
    }
}

void terminal_currents(Inst &d, double *I, double *S) {
    Ctx c = make_ctx(d);
    const int nc = d.n_cons;
    if (d.unstr) launch_currents_g(c);
    else launch_currents(c);
    tun_currents(d);
    te_currents(d);
    cudaMemcpyAsync(d.g.pin, d.g.h.res, sizeof(double) * R_TOTAL, cudaMemcpyDeviceToHost, d.g.st);
    cudaStreamSynchronize(d.g.st);
    for (int q = 0; q < nc; q++) {
        I[q] = d.g.pin[R_I + q];
        S[q] = d.g.pin[R_S + q];
        d.cons[q].In = d.g.pin[R_IN + q];
    }
}

static void copy_dev(Inst &d, double *dst, const double *src) {
    cudaMemcpyAsync(dst, src, d.N * 8, cudaMemcpyDeviceToDevice, d.g.st);
}
static void save_state(Inst &d, double *const *h) {
    copy_dev(d, h[0], d.g.h.phi); copy_dev(d, h[1], d.g.h.phin); copy_dev(d, h[2], d.g.h.phip);
}
static void load_state(Inst &d, double *const *h) {
    copy_dev(d, d.g.h.phi, h[0]); copy_dev(d, d.g.h.phin, h[1]); copy_dev(d, d.g.h.phip, h[2]);
}

// ------------------------------------------------------------------ Newton-Poisson
// Damped Newton with PCG and a backtracking line search on ||F/diag||
// (semiconductor_3d.c:2791-2823)
static int poisson_newton(Inst &d, const double *Va, double ntol, int maxit) {
    Ctx c = make_ctx(d);
    upload_voltages(d, Va);
    for (int it = 0; it < maxit; it++) {
        d.newton_its++;
        if (d.unstr) launch_poisson_g(c, nullptr, 1);
        else launch_poisson(c, nullptr, 1, nullptr);
        const double f0 = read_res(d, R_PNORM);
        if (!(f0 > 0.)) return f0 == 0.;
        launch_fill_sel(c, V_SOL, 0.0);
        const int maxp = d.max_iter_p > 0 ? d.max_iter_p : 2000;
        const int its = d.unstr ? pcg_graph(d, maxp, d.pcg_rtol)
                                : pcg_solve(c, d.g.mg, maxp, d.pcg_rtol, g_knobs.check_every, use_mixed(d));
        d.pcg_its += its;
        launch_absmax_sel(c, V_SOL, R_DMAX);
        const double dm = read_res(d, R_DMAX);
        if (dm != dm) return 0;
        if (dm < ntol) {
            launch_axpy_sel(c, V_PHI, V_PHI, 1.0, V_SOL);   // psi += dx
            return 1;
        }
        double lam = 1.;
        for (int ls = 0; ls < 40; ls++) {
            launch_axpy_sel(c, V_TR, V_PHI, lam, V_SOL);    // trial psi + lam dx
            if (d.unstr) launch_poisson_g(c, d.g.h.tr, 0);
            else launch_poisson(c, d.g.h.tr, 0, nullptr);
            const double f1 = read_res(d, R_PNORM);
            if (f1 <= (1. - 1e-4 * lam) * f0) break;
            lam *= 0.5;
        }
        cudaMemcpyAsync(d.g.h.phi, d.g.h.tr, d.N * 8, cudaMemcpyDeviceToDevice, d.g.st);
        if (d.verbose > 4) std::fprintf(stderr, "      newton it=%d f0=%.3e dm=%.3e lam=%.3e\n", it, f0, dm, lam);
        if (lam * dm < ntol) return 1;
    }
    return 0;
}

// ------------------------------------------------------------------ floating blocks
int float_fix(Inst &d, int hole);   // kernels_ccl.cu

// ------------------------------------------------------------------ continuity
// assemble -> BiCGSTAB from u = 1 (ILU-only retry, keep the start if worse) ->
// floating-block balance -> update (semiconductor_3d.c:2216-2232, 3580-3594)
static int solve_cont(Inst &d, int hole, double lo, double hi, double *dmax) {
    Ctx c = make_ctx(d);
    exchange_scatter(d, hole);                           // gate / metal-contact sink and source of this carrier
    if (d.unstr) launch_cont_assemble_g(c, hole);
    else launch_cont_assemble(c, hole);
    launch_fill_sel(c, V_SOL, 1.0);
    const double atol = g_knobs.cont_atol * d.cont_atol_f;
    const int maxit = d.max_iter_c > 0 ? d.max_iter_c : 1000;
    launch_copy_sel(c, 7, V_SOL);                        // x0 backup
    double rn = 0, r0 = 0;
    const long long s0 = t_ir_steps, f0 = t_ir_fallbacks;
    int its = d.unstr ? bicg_graph(d, maxit, d.bicg_rtol, atol, &rn, &r0, hole ? -1 : 1, false)
                      : bicgstab_core(c, d.g.mg, maxit, d.bicg_rtol, atol, 1, g_knobs.check_every, &rn, &r0,
                                      hole ? -1 : 1, use_mixed(d));
    d.ir_steps += t_ir_steps - s0;
    d.ir_fallbacks += t_ir_fallbacks - f0;
    if (!(rn <= std::fmax(r0, 1e-300)) && (d.unstr ? gmg_levels(d) > 1 : d.g.mg.maxlev > 1)) {
        if (d.verbose) std::fprintf(stderr, "semisim-b200: MG-BiCGSTAB diverged (%.2e > %.2e), retry ILU\n", rn, r0);
        launch_copy_sel(c, V_SOL, 7);
        its += d.unstr ? bicg_graph(d, 4 * maxit, d.bicg_rtol, atol, &rn, &r0, hole ? -1 : 1, true)
                       : bicgstab_core(c, d.g.mg, 4 * maxit, d.bicg_rtol, atol, 0, g_knobs.check_every, &rn, &r0,
                                       hole ? -1 : 1);
    }
    d.bicg_its += its;
    if (!(rn <= std::fmax(r0, 1e-300)) || !std::isfinite(rn)) {
        launch_copy_sel(c, V_SOL, 7);
        rn = INFINITY;
    }
    if (d.verbose > 2) std::fprintf(stderr, "    bicgstab(%c) its=%d |r|=%.3e\n", hole ? 'p' : 'n', its, rn);
    const int ok = std::isfinite(rn);
    if (ok) float_fix(d, hole);
    launch_cont_update(c, hole, lo, hi);
    *dmax = read_res(d, R_DQ);
    return ok;
}

// ------------------------------------------------------------------ Anderson
static void aa_reset(Inst &d) { d.aa_n = 0; d.aa_pos = 0; d.aa_have = 0; }
static void aa_step(Inst &d) {                      // semiconductor_3d.c:3709-3757
    Ctx c = make_ctx(d);
    const int M = d.aa_m < g_knobs.aa_depth ? d.aa_m : g_knobs.aa_depth;
    if (M > 0 && d.aa_have) {
        const int s = d.aa_pos;
        if (d.aa_n < M) d.aa_n++;
        aa_update_history(c, s, d.aa_n);
        d.aa_pos = (s + 1) % M;
    }
    aa_store_fg(c);
    d.aa_have = 1;
    const int m = d.aa_n;
    if (m == 0) return;
    aa_solve_mix(c, m, nullptr);
}

// ------------------------------------------------------------------ Gummel
// One Gummel solve at fixed terminal voltages (semiconductor_3d.c:3781-3930; the
// impact-ionisation branch belongs to a model this library does not build)
static int gummel(Inst &d, const double *Va, int maxit, double gtol, int *iters, double *res) {
    Ctx c = make_ctx(d);
    const int nc = d.n_cons;
    const double lo = d.vlo - g_knobs.qf_margin, hi = d.vhi + g_knobs.qf_margin, nt0 = newton_tol(d, Va);
    double I[NC_MAX], S[NC_MAX], Iold[NC_MAX];
    int haveI = 0;
    const double itol = d.tol_c > 0. ? d.tol_c : 1e-6;
    apply_bc(d, Va);
    aa_reset(d);
    poisson_newton(d, Va, std::fmax(nt0, 1e-6), 100);
    int it, conv = 0, it_mark = 0, stall = 0, ntight = 0, loose = 0;
    double dpsi = 1., dq = 1., best = 1e300, prev = 1., best_mark = 1e300;
    const int n_te = d.g.te_on ? d.g.te.n_te : 0;
    // impact ionisation: the multiplication converges slowly near breakdown; track the total
    // generation Gs and accept only when its change and the extrapolated remainder of the
    // series are below tol_ii Gs; the continuity solves run tighter meanwhile
    // (semiconductor_3d.c:3788-3799, 3815-3831)
    const int iion = (d.models & 256) != 0 && d.g.h.gii;
    const double tol_ii = std::fmax(itol, 1e-4);
    double Gs_old = -1., dG_old = 0., ii_rel = 1., ii_best = 1e300, Erem = 0.;
    const double brtol0 = d.bicg_rtol;
    if (iion && d.bicg_rtol > 1e-8) d.bicg_rtol = 1e-8;
    d.ii_err = 0.;
    for (it = 1; it <= maxit; it++) {
        if (g_stop.load()) break;
        const double t0 = wtime();
        clamp_qf(d);
        copy_dev(d, d.g.h.qn0, d.g.h.phin);
        copy_dev(d, d.g.h.qp0, d.g.h.phip);
        rebuild_np(d);
        upd_mob(d);
        tun_update(d);
        te_update(d);
        int iiok = 1;
        if (iion) {
            if (d.unstr) launch_ii_update_g(c);
            else launch_ii_update(c);
            const double Gs = read_res(d, R_GII);
            if (Gs > 0.) {
                if (Gs_old < 0.) { iiok = 0; Erem = Gs; }
                else {
                    const double dG = std::fabs(Gs - Gs_old);
                    double rho = dG_old > 0. ? dG / dG_old : 0.;
                    if (rho > 0.99) rho = 0.99;
                    Erem = dG + dG * rho / (1. - rho);
                    iiok = dG <= tol_ii * Gs && Erem <= tol_ii * Gs;
                    dG_old = dG;
                }
                ii_rel = Erem / Gs;
                Gs_old = Gs;
            } else {
                Erem = 0.;
                ii_rel = 0.;
            }
        }
        const double t1 = wtime();
        d.t_mob += t1 - t0;
        double dn = 0., dp = 0.;
        if (!solve_cont(d, 0, lo, hi, &dn)) break;
        if (!solve_cont(d, 1, lo, hi, &dp)) break;
        const double t2 = wtime();
        d.t_cont += t2 - t1;
        dq = std::fmax(dn, dp);
        terminal_currents(d, I, S);
        d.t_cur += wtime() - t2;
        int icv = haveI, icl = haveI;                     // icl: stable to 1e-4 (metal-contact noise floor)
        if (haveI)
            for (int q = 0; q < nc; q++) {
                if (std::fabs(I[q] - Iold[q]) > std::fmax(itol * std::fabs(I[q]), 3e-14 * S[q])) icv = 0;
                if (std::fabs(I[q] - Iold[q]) > std::fmax(std::fmax(itol, 1e-4) * std::fabs(I[q]), 3e-14 * S[q])) icl = 0;
            }
        if (iion && !iiok) {                              // generation below the current resolution
            double Sm = 0.;
            for (int q = 0; q < nc; q++) if (S[q] > Sm) Sm = S[q];
            if (Q * Erem <= 3e-14 * Sm) iiok = 1;
        }
        loose = icl ? loose + 1 : 0;
        std::memcpy(Iold, I, sizeof(double) * nc);
        haveI = 1;
        launch_predictor(c);                               // xk = psi; neutral-region predictor
        const double ntol = std::fmax(nt0, d.ntol_fac * std::fmin(prev, 1.));
        const double t3 = wtime();
        poisson_newton(d, Va, ntol, 100);
        d.t_pois += wtime() - t3;
        launch_dpsi(c);
        dpsi = read_res(d, R_DPSI);
        if (d.verbose > 1)
            std::fprintf(stderr, "  gummel %3d dpsi=%.3e dq=%.3e I0=%.6e aa=%d\n", it, dpsi, dq, nc ? I[0] : 0., d.aa_n);
        if (dpsi != dpsi || dq != dq) break;
        const double r = std::fmax(dpsi, dq);
        g_prog[1] = it; g_prog[2] = r; g_prog[5] = (double)(d.gummel_its + it);
        if (dq < gtol && dpsi < gtol && icv && iiok) {    // accept psi_k with its carriers
            copy_dev(d, d.g.h.phi, d.g.h.xk);
            conv = 1;
            break;
        }
        // metal contacts: potentials converged but a terminal current keeps moving (a trace
        // carrier left at the BiCGSTAB tolerance): tighten that tolerance (it stays tight
        // for this device), then the residual floor, then accept at the 1e-4 noise floor
        // (semiconductor_3d.c:3875-3904)
        if (n_te > 0 && r <= 1e3 * gtol && !icv && haveI) {
            if (++stall >= 3 + 3 * ntight) {
                int did = 0;
                if (d.bicg_rtol > 1.01e-10) { d.bicg_rtol = std::fmax(d.bicg_rtol * 1e-2, 1e-10); did = 1; }
                else if (d.cont_atol_f > 1e-6) { d.cont_atol_f *= 1e-3; did = 1; }
                if (did) {
                    stall = 0; ntight++; best_mark = 1e300; it_mark = it;
                    if (d.verbose)
                        std::fprintf(stderr, "semisim-b200: terminal current not settling - continuity tolerance %.0e, floor %.0e\n",
                                     d.bicg_rtol, g_knobs.cont_atol * d.cont_atol_f);
                } else if (loose >= 8 && iiok) {
                    copy_dev(d, d.g.h.phi, d.g.h.xk);
                    conv = 1;
                    if (d.verbose) std::fprintf(stderr, "semisim-b200: accepted at the metal-contact noise floor (res %.2e)\n", r);
                    break;
                }
            }
        } else {
            stall = 0;
        }
        prev = r;
        if (r < 0.5 * best_mark) { best_mark = r; it_mark = it; }
        if (iion && ii_rel < 0.5 * ii_best) { ii_best = ii_rel; it_mark = it; }   // slow multiplication is progress
        if (it - it_mark > 20 && r <= 1e3 * gtol && icv && iiok) {
            copy_dev(d, d.g.h.phi, d.g.h.xk);
            conv = 1;
            if (d.verbose) std::fprintf(stderr, "semisim-b200: accepted at noise floor (res %.2e)\n", r);
            break;
        }
        if (it - it_mark > 60) break;
        if (r < best) best = r;
        else if (r > 30. * best) aa_reset(d);
        const double t4 = wtime();
        aa_step(d);
        d.t_aa += wtime() - t4;
    }
    if (it > maxit) it = maxit;
    cudaStreamSynchronize(d.g.st);
    if (iion && brtol0 > 1e-8 && d.bicg_rtol == 1e-8) d.bicg_rtol = brtol0;   // (a metal-contact tightening stays)
    if (iion) d.ii_err = Q * Erem;
    d.gummel_its += it;
    *iters = it;
    *res = std::fmax(dpsi, dq);
    return conv;
}

// ------------------------------------------------------------------ continuation
static void region_shift(Inst &d, const double *dV) {      // semiconductor_3d.c:3956-3987
    Ctx c = make_ctx(d);
    int *mark = d.g.h.ccl;
    cudaMemsetAsync(mark, 0, d.N * sizeof(int), d.g.st);
    for (int q = 0; q < d.n_cons; q++) {
        if (d.cons[q].bc != 0 || std::fabs(dV[q]) < 1e-15) continue;
        int type = 0;
        for (size_t k = 0; k < d.N && !type; k++) {
            const uint32_t f = d.flags[k];
            if (fl_con(f) == q + 1 && fl_kind(f) == K_SEMI) {
                const double D = d.Nd[k] - d.Na[k];
                type = D > 0. ? 1 : (D < 0. ? -1 : 0);
            }
        }
        if (!type) continue;
        if (d.unstr) launch_region_mark_g(d, q + 1, type, dV[q], mark, d.g.flag);
        else launch_region_mark(c, q + 1, type, dV[q], mark, d.g.flag);
    }
}

int equilibrium(Inst &d) {                                  // semiconductor_3d.c:3989-4004
    double Va[NC_MAX];
    d.e_n = 0;
    for (int q = 0; q < d.n_cons; q++) Va[q] = d.cons[q].bc == 2 ? d.cons[q].V : 0.;
    Ctx c = make_ctx(d);
    launch_init_eq(c);
    set_vrange(d, Va);
    apply_bc(d, Va);
    g_prog[4] = 1.;
    const int ok = poisson_newton(d, Va, newton_tol(d, Va), 300);
    rebuild_np(d);
    upd_mob(d);
    for (int q = 0; q < d.n_cons; q++) d.cons[q].Vprev = Va[q];
    d.have_solution = 1;
    if (d.verbose) std::fprintf(stderr, "semisim-b200: equilibrium %s (newton its %lld)\n", ok ? "ok" : "NOT converged", d.newton_its);
    return ok;
}

static double gummel_tol(const Inst &d) {
    double g = d.tol_p;
    if (!(g > 0.)) g = 1e-9;
    if (g > 1e-4) g = 1e-4;
    if (g < 1e-13) g = 1e-13;
    return g;
}

// Adaptive continuation from Vprev to V, all contacts together, with the secant sweep
// predictor (semiconductor_3d.c:4018-4133)
static int cont_path(Inst &d) {
    const int nc = d.n_cons;
    double Vf[NC_MAX], Vt[NC_MAX], Va[NC_MAX], dV[NC_MAX];
    double span = 0.;
    for (int q = 0; q < nc; q++) {
        Vf[q] = d.cons[q].Vprev; Vt[q] = d.cons[q].V;
        if (std::fabs(Vt[q] - Vf[q]) > span) span = std::fabs(Vt[q] - Vf[q]);
    }
    const int maxg = d.max_gummel > 0 ? d.max_gummel : 100;
    const double gtol = gummel_tol(d);
    Ctx c = make_ctx(d);
    upd_mob(d);
    save_state(d, d.g.h.h1);
    double rx = 0.;
    if (g_knobs.pred_on && d.e_n >= 1 && span > 0.) {
        double num = 0., den = 0., err = 0.;
        int same = 1;
        for (int q = 0; q < nc; q++) {
            const double a = Vt[q] - Vf[q], b = Vf[q] - d.Ve2[q];
            num += a * b; den += b * b;
            if (std::fabs(Vf[q] - d.Ve1[q]) > 1e-12) same = 0;
        }
        if (same && den > 0.) {
            const double r = num / den;
            for (int q = 0; q < nc; q++) {
                const double a = Vt[q] - Vf[q], b = Vf[q] - d.Ve2[q];
                err = std::fmax(err, std::fabs(a - r * b));
            }
            if (r >= -2. && r <= 3. && std::fabs(r) > 1e-12 && err <= 1e-9 + 1e-6 * span) rx = r;
        }
    }
    // quadratic predictor (not in the reference): the point before the last on the same
    // line, Ve3 = Ve2 - r3 (Vf - Ve2); positions in units of the last step: Ve3 at -1 - r3,
    // Ve2 at -1, Vf at 0
    double r3 = 0.;
    if (rx != 0. && g_knobs.pred_order >= 2 && d.e_n >= 2) {
        double num = 0., den = 0., err = 0.;
        for (int q = 0; q < nc; q++) {
            const double b = Vf[q] - d.Ve2[q], e = d.Ve2[q] - d.Ve3[q];
            num += e * b; den += b * b;
        }
        if (den > 0.) {
            const double r = num / den;
            for (int q = 0; q < nc; q++)
                err = std::fmax(err, std::fabs((d.Ve2[q] - d.Ve3[q]) - r * (Vf[q] - d.Ve2[q])));
            if (r >= 0.2 && r <= 5. && err <= 1e-9 + 1e-6 * span) r3 = r;
        }
    }
    int first = 1, noseed = 0;
    double t = 0., tp = -1., dt = span > 0. ? std::fmin(1., 0.1 / span) : 1.;
    int ok_all = 0, its = 0, steps = 0;
    double res = 0.;
    g_prog[0] = 0.; g_prog[3] = 0.;
    for (int guard = 0; guard < 5000; guard++) {
        if (g_stop.load()) break;
        const double tn = std::fmin(1., t + dt);
        for (int q = 0; q < nc; q++) Va[q] = Vf[q] + tn * (Vt[q] - Vf[q]);
        set_vrange(d, Va);
        int seeded = 0;
        if (tp >= 0.) {
            launch_extrap(c, (tn - t) / (t - tp), 0, 1);
        } else if (rx != 0. && !noseed && seed_available(d)) {
            // learned correction of the sweep predictor's linear guess
            double dvs[4] = {0., 0., 0., 0.};
            for (int q = 0; q < nc && q < 4; q++) dvs[q] = Va[q] - Vf[q];
            launch_mlp_seed(d, tn * rx, dvs);
            seeded = 1;
        } else if (rx != 0. && r3 != 0.) {
            const double s = tn * rx, s1 = -1., s0 = -1. - r3;      // Lagrange weights at s
            launch_extrap3(c, (s - s1) * (s - s0) / (s1 * s0), s * (s - s0) / (s1 * (s1 - s0)),
                           s * (s - s1) / (s0 * (s0 - s1)));
        } else if (rx != 0.) {
            launch_extrap(c, tn * rx, 0, 2);
        } else {
            load_state(d, d.g.h.h1);
            if (span > 0.) {
                for (int q = 0; q < nc; q++) dV[q] = (tn - t) * (Vt[q] - Vf[q]);
                region_shift(d, dV);
            }
        }
        clamp_qf(d);
        apply_bc(d, Va);
        rebuild_np(d);
        const int ok = gummel(d, Va, maxg, gtol, &its, &res);
        if (!ok && seeded) {                       // redo the step from the linear guess
            d.seed_fallbacks++;
            noseed = 1;
            if (d.verbose) std::fprintf(stderr, "semisim-b200: learned seed failed, linear guess\n");
            continue;
        }
        if (seeded) d.seed_used++;
        if (first) {                               // the path's start (h1 until the first accepted step)
            for (int a = 0; a < 3; a++) copy_dev(d, d.g.h.e3[a], d.g.h.e2[a]);
            for (int a = 0; a < 3; a++) copy_dev(d, d.g.h.e2[a], d.g.h.h1[a]);
            first = 0;
        }
        d.conv_iter = its;
        d.conv_res = res;
        if (d.verbose)
            std::fprintf(stderr, "semisim-b200: step t=%.4f (V0=%.4f) %s its=%d res=%.2e\n", tn, nc ? Va[0] : 0.,
                         ok ? "ok" : "FAIL", its, res);
        if (ok) {
            for (int a = 0; a < 3; a++) std::swap(d.g.h.h1[a], d.g.h.h2[a]);
            cudaMemcpyAsync(d.g.d, &d.g.h, sizeof(DevP), cudaMemcpyHostToDevice, d.g.st);
            c = make_ctx(d);
            save_state(d, d.g.h.h1);
            tp = t; t = tn; steps++;
            g_prog[0] = t; g_prog[3] = steps;
            for (int q = 0; q < nc; q++) d.cons[q].Vprev = Va[q];
            if (t >= 1.) { ok_all = 1; break; }
            dt *= its <= 8 ? 2.0 : (its <= 25 ? 1.5 : g_knobs.grow_slow);
        } else {
            rx = 0.;
            if (span == 0. || dt * span < 2e-5) break;
            dt *= 0.3;
        }
    }
    if (ok_all && span > 0.) {
        for (int q = 0; q < nc; q++) { d.Ve3[q] = d.Ve2[q]; d.Ve2[q] = Vf[q]; d.Ve1[q] = Vt[q]; }
        d.e_n = d.e_n < 2 ? d.e_n + 1 : 2;
    } else if (!ok_all) d.e_n = 0;
    if (!ok_all && (span > 0. || g_stop.load())) {
        load_state(d, d.g.h.h1);
        for (int q = 0; q < nc; q++) Va[q] = d.cons[q].Vprev;
        set_vrange(d, Va);
        apply_bc(d, Va);
        rebuild_np(d);
        upd_mob(d);
        if (d.verbose) std::fprintf(stderr, "semisim-b200: continuation stopped at t=%.4f\n", t);
    }
    cudaStreamSynchronize(d.g.st);
    return ok_all;
}

// Gate-first bias path, then terminal currents with the Kirchhoff choice and their
// resolution floors (semiconductor_3d.c:4135-4173)
int run_continuation(Inst &d) {
    const int nc = d.n_cons;
    int gch = 0, cch = 0, ok_all;
    for (int q = 0; q < nc; q++) {
        if (std::fabs(d.cons[q].V - d.cons[q].Vprev) <= 1e-12) continue;
        if (d.cons[q].bc == 2) gch = 1;
        else cch = 1;
    }
    if (gch && cch) {
        double Vt[NC_MAX];
        for (int q = 0; q < nc; q++) {
            Vt[q] = d.cons[q].V;
            if (d.cons[q].bc != 2) d.cons[q].V = d.cons[q].Vprev;
        }
        g_prog[4] = 2.;
        ok_all = cont_path(d);
        for (int q = 0; q < nc; q++) d.cons[q].V = Vt[q];
        g_prog[4] = 3.;
        if (ok_all) ok_all = cont_path(d);
    } else {
        g_prog[4] = gch ? 2. : 3.;
        ok_all = cont_path(d);
    }
    double I[NC_MAX], S[NC_MAX];
    terminal_currents(d, I, S);
    double ks = 0., F = 0., fl[NC_MAX];
    int ncar = 0;
    for (int q = 0; q < nc; q++) {
        ks += I[q]; fl[q] = 3e-14 * S[q]; F += fl[q];
        if (d.cons[q].bc != 2) ncar++;
    }
    const double scl = F > 0. ? std::fmax(1., 2. * std::fabs(ks) / F) : 1.;
    for (int q = 0; q < nc; q++) {
        double Iv = I[q], fv = fl[q];
        const double fo = F - fl[q];
        if (d.cons[q].bc != 2 && ncar > 1 && fo < fv) { Iv = -(ks - I[q]); fv = fo; }
        d.cons[q].I = Iv;
        d.cons[q].Iflr = fv * scl + (ok_all ? d.ii_err : 0.);   // (a failed point keeps its partial-state floor)
        d.cons[q].Iraw = I[q];
    }
    return ok_all;
}

void finish_point(Inst &d) {
    Ctx c = make_ctx(d);
    if (d.unstr) {
        launch_upd_J_g(c);
        launch_mob_display_g(c);
    } else {
        launch_upd_J(c);
        launch_mob_display(c);
    }
    // the display update leaves the sink / source arrays holding the gate-tunnelling current
    // density at the interface nodes (A/m^2), as upd_J does (semiconductor_3d.c:3648-3657)
    if (d.g.h.tk) {
        cudaMemsetAsync(d.g.h.tk, 0, d.N * sizeof(double), d.g.st);
        cudaMemsetAsync(d.g.h.tg, 0, d.N * sizeof(double), d.g.st);
        tun_display(d);
    }
    cudaStreamSynchronize(d.g.st);
    for (auto &v : d.cache_ok) v = 0;
}

int do_solve(Inst &d, int keep) {                           // semiconductor_3d.c:4910-4916
    if (!prepare(d)) return 0;
    if (!keep || !d.have_solution) equilibrium(d);
    const int ok = run_continuation(d);
    finish_point(d);
    d.converged = ok;
    g_prog[4] = 0.;
    return ok;
}

}  // namespace ss
