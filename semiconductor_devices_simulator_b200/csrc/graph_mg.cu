// Aggregation multigrid of a general (graph) mesh (semiconductor_3d.c:2322-2680): the
// preconditioner of the graph path's PCG and BiCGSTAB.
//
// Hierarchy (host, once per mesh): every level pairs each node with its strongest free
// neighbour - coupling w = dual face area / edge length, summed over merged nodes - when
// that coupling is at least beta of the node's strongest, else the node stays alone; passes
// rounds of pairing on the contracted graph give aggregates of up to 2^passes nodes.  Levels
// are added until one has at most GMG_COARSE nodes or the aggregation stalls (more than 0.7
// of the nodes left).  The coarsest level is solved through its dense inverse (up to
// GMG_DENSE_MAX nodes), else by D-ILU sweeps.
//
// Per solve (device): Slotboom prolongation weights from the quasi-Fermi levels (continuity;
// 1 for Poisson), Petrov-Galerkin coarse operators P^T W A P summed per aggregate in the
// reference's order (W the continuity row scale, 1 for Poisson), D-ILU(0) pivots of every
// level and the coarsest inverse.  The V(1,1) cycle smooths with D-ILU(0) in a multicolour
// order (a greedy colouring of each level: one parallel sweep per colour), where the
// reference runs a chunked natural-order recurrence on its host threads.
//
// Every level is stored in ELL (slot s of node k at s*N + k), the layout of the mesh level
// the assembly kernels write, so one set of kernels serves all levels.
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <vector>

#include "device_common.cuh"
#include "prof.h"
#include "solver_ctx.h"
#include "gmg_common.cuh"

namespace ss {

constexpr int GMG_COARSE = 160;        // stop coarsening at or below this many nodes
constexpr int GMG_DENSE_MAX = 640;     // coarsest level solved through its dense inverse up to here
constexpr int GMG_SMEM_MAX = 160;      // dense inversion in shared memory up to here

// ------------------------------------------------------------------ device kernels
// level-0 reference potential in units of VT (ph0, semiconductor_3d.c:2085-2090)
__device__ __forceinline__ double gph0(const DevP &P, int k, int qsign) {
    const uint32_t f = P.flags[k];
    if (fl_kind(f) != K_SEMI || fl_fix(f)) return PH_NONE;
    return qsign > 0 ? P.phin[k] / P.VTref : -P.phip[k] / P.VTref;
}

// Slotboom prolongation weights of level f towards c: pw = exp(ph - max over the aggregate)
// (g_weights, semiconductor_3d.c:2621-2642)
__global__ void k_gmg_weights(const DevP *__restrict__ Ps, GLev f, GLev c, int L, int qsign) {
    const DevP &P = Ps[0];
    SS_GRID_LOOP(I, c.N) {
        const int q0 = f.mrp[I], q1 = f.mrp[I + 1];
        if (qsign == 0) {
            for (int q = q0; q < q1; q++) f.pw[f.mem[q]] = 1.0;
            continue;
        }
        double mx = PH_NONE;
        for (int q = q0; q < q1; q++) {
            const int i = f.mem[q];
            const double p = L == 0 ? gph0(P, i, qsign) : f.ph[i];
            if (p > mx) mx = p;
        }
        c.ph[I] = mx;
        for (int q = q0; q < q1; q++) {
            const int i = f.mem[q];
            const double p = L == 0 ? gph0(P, i, qsign) : f.ph[i];
            const double e = (p <= 0.5 * PH_NONE) ? -800.0 : p - mx;
            f.pw[i] = e < -700.0 ? 0.0 : exp(e);
        }
    }
}

// coarse operator row I = sum over the aggregate's members i (and their entries) of
// w_i a_ij pw_j (g_galerkin, semiconductor_3d.c:2575-2594); a row of identity rows only
// stays an identity row
__global__ void k_gmg_galerkin(GLev f, GLev c, const double *__restrict__ w) {
    SS_GRID_LOOP(I, c.N) {
        for (int s = 0; s < c.D; s++) c.val[(size_t)s * c.N + I] = 0.0;
        double cc = 0.0;
        for (int q = f.mrp[I]; q < f.mrp[I + 1]; q++) {
            const int i = f.mem[q];
            const double wi = w ? w[i] : 1.0;
            cc += wi * f.diag[i] * f.pw[i];
            for (int s = 0; s < f.D; s++) {
                const size_t e = (size_t)s * f.N + i;
                const int j = f.col[e];
                if (j < 0) continue;
                const double a = wi * f.val[e] * f.pw[j];
                const int em = f.emap[e];
                if (em < 0) cc += a;
                else c.val[em] += a;
            }
        }
        bool zero = cc == 0.0;
        for (int s = 0; s < c.D && zero; s++)
            if (c.val[(size_t)s * c.N + I] != 0.0) zero = false;
        c.diag[I] = zero ? 1.0 : cc;
    }
}

// D-ILU(0) pivots of one colour: D_i = a_ii - sum over earlier colours a_ij a_ji / D_j,
// guarded as the reference guards its pivots (gilu_factor, semiconductor_3d.c:2533-2551);
// reciprocals kept
__global__ void k_gmg_ilu(GLev v, const int *__restrict__ nodes, int cnt) {
    SS_GRID_LOOP(t, cnt) {
        const int i = nodes[t], ci = v.color[i];
        const double a = v.diag[i];
        double d = a;
        for (int s = 0; s < v.D; s++) {
            const size_t e = (size_t)s * v.N + i;
            const int j = v.col[e];
            if (j < 0 || v.color[j] >= ci || v.val[e] == 0.0) continue;
            d -= v.val[e] * v.val[(size_t)v.rev[e] * v.N + j] * v.dil[j];
        }
        if (!(d > 1e-8 * fabs(a))) d = a;
        if (!(d != 0.0)) d = 1.0;
        v.dil[i] = 1.0 / d;
    }
}

// one colour of the D-ILU(0) solve: forward (dir 0) y_i = (r_i - sum earlier colours a_ij
// y_j) / D_i, backward (dir 1) z_i = y_i - sum later colours a_ij z_j / D_i; r may be z
__global__ void k_gmg_ilu_apply(GLev v, const int *__restrict__ nodes, int cnt, int dir, const double *r, double *z) {
    SS_GRID_LOOP(t, cnt) gilu_apply_node(v, nodes[t], dir, r, z);
}

// y = b - A x (b null: y = A x)  (gmatvec_L, semiconductor_3d.c:2553-2561)
__global__ void k_gmg_matvec(GLev v, const double *__restrict__ x, const double *__restrict__ b,
                             double *__restrict__ y) {
    SS_GRID_LOOP(k, v.N) {
        const double s = gmatvec_row(v, x, k);
        y[k] = b ? b[k] - s : s;
    }
}

// coarse right-hand side: the weighted residual summed over each aggregate (g_restrict,
// semiconductor_3d.c:2595-2603)
__global__ void k_gmg_restrict(GLev f, int ncoarse, const double *__restrict__ r, double *__restrict__ bc,
                               const double *__restrict__ w) {
    SS_GRID_LOOP(I, ncoarse) {
        double s = 0.0;
        for (int q = f.mrp[I]; q < f.mrp[I + 1]; q++) {
            const int i = f.mem[q];
            s += w ? w[i] * r[i] : r[i];
        }
        bc[I] = s;
    }
}

// x += alpha pw x_c[aggregate]  (g_prolong, semiconductor_3d.c:2604-2608)
__global__ void k_gmg_prolong(GLev f, const double *__restrict__ xc, double *__restrict__ x, double alpha) {
    SS_GRID_LOOP(i, f.N) x[i] += alpha * f.pw[i] * xc[f.agg[i]];
}

__global__ void k_gmg_add(int N, double *__restrict__ x, const double *__restrict__ r) {
    SS_GRID_LOOP(k, N) x[k] += r[k];
}

// dense inverse of the coarsest level by Gauss-Jordan elimination with row interchanges
// (tiny pivots set to 1e-300 as semiconductor_3d.c:2620 does); one block, the matrix in
// dynamic shared memory (n <= GMG_SMEM_MAX) or in place in v.inv
__global__ void k_gmg_coarse_setup(GLev v, int smem) {
    extern __shared__ double shm[];
    const int n = v.N;
    double *M = smem ? shm : v.inv;
    __shared__ int perm[GMG_DENSE_MAX];
    __shared__ double fcol[GMG_DENSE_MAX];
    __shared__ int piv;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) M[e] = 0.0;
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        M[(size_t)r * n + r] = v.diag[r];
        for (int s = 0; s < v.D; s++) {
            const size_t e = (size_t)s * n + r;
            const int j = v.col[e];
            if (j >= 0) M[(size_t)r * n + j] += v.val[e];
        }
    }
    __syncthreads();
    for (int c = 0; c < n; c++) {
        if (threadIdx.x == 0) {
            int p = c;
            double mx = fabs(M[(size_t)c * n + c]);
            for (int r = c + 1; r < n; r++)
                if (fabs(M[(size_t)r * n + c]) > mx) { mx = fabs(M[(size_t)r * n + c]); p = r; }
            piv = p;
            perm[c] = p;
            if (!(mx > 1e-300)) M[(size_t)p * n + c] = 1e-300;
        }
        __syncthreads();
        const int p = piv;
        if (p != c)
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                const double t = M[(size_t)c * n + q];
                M[(size_t)c * n + q] = M[(size_t)p * n + q];
                M[(size_t)p * n + q] = t;
            }
        __syncthreads();
        const double dg = M[(size_t)c * n + c];
        __syncthreads();
        if (threadIdx.x == 0) M[(size_t)c * n + c] = 1.0;
        __syncthreads();
        for (int q = threadIdx.x; q < n; q += blockDim.x) M[(size_t)c * n + q] /= dg;
        for (int r = threadIdx.x; r < n; r += blockDim.x) fcol[r] = r == c ? 0.0 : M[(size_t)r * n + c];
        __syncthreads();
        // every other row r: row_r -= f_r row_c, with column c becoming -f_r / pivot
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
            const int r = e / n, q = e - r * n;
            if (r == c) continue;
            const double fr = fcol[r];
            if (q == c) M[e] = -fr * M[(size_t)c * n + c];
            else M[e] -= fr * M[(size_t)c * n + q];
        }
        __syncthreads();
    }
    for (int c = n - 1; c >= 0; c--) {
        const int p = perm[c];
        if (p != c)
            for (int r = threadIdx.x; r < n; r += blockDim.x) {
                const double t = M[(size_t)r * n + c];
                M[(size_t)r * n + c] = M[(size_t)r * n + p];
                M[(size_t)r * n + p] = t;
            }
        __syncthreads();
    }
    if (smem)
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) v.inv[e] = M[e];
}

// x = inverse b, one warp per row
__global__ void k_gmg_coarse_solve(GLev v, const double *__restrict__ b, double *__restrict__ x) {
    const int lane = threadIdx.x & 31, n = v.N;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5) {
        double s = 0.0;
        for (int q = lane; q < n; q += 32) s += v.inv[(size_t)r * n + q] * b[q];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[r] = s;
    }
}

// ------------------------------------------------------------------ host: hierarchy
namespace {

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

struct Csr {
    int N = 0;
    std::vector<int> rp, cj;
    std::vector<double> w;
};

// one round of pairwise matching (g_pair, semiconductor_3d.c:2350-2366): agg[i], returns
// the number of groups
int pair_round(const Csr &g, double beta, std::vector<int> &agg) {
    agg.assign(g.N, -1);
    int na = 0;
    for (int i = 0; i < g.N; i++) {
        if (agg[i] >= 0) continue;
        double mx = 0.0;
        for (int e = g.rp[i]; e < g.rp[i + 1]; e++) mx = std::max(mx, g.w[e]);
        int best = -1;
        double bw = -1.0;
        for (int e = g.rp[i]; e < g.rp[i + 1]; e++) {
            const int j = g.cj[e];
            if (j == i || agg[j] >= 0 || !(g.w[e] > 0.0) || g.w[e] < beta * mx) continue;
            if (g.w[e] > bw) { bw = g.w[e]; best = j; }
        }
        agg[i] = na;
        if (best >= 0) agg[best] = na;
        na++;
    }
    return na;
}

// member lists of na groups, members ascending
void members(const std::vector<int> &agg, int na, std::vector<int> &mrp, std::vector<int> &mem) {
    const int N = (int)agg.size();
    mrp.assign(na + 1, 0);
    for (int i = 0; i < N; i++) mrp[agg[i] + 1]++;
    for (int a = 0; a < na; a++) mrp[a + 1] += mrp[a];
    mem.assign(N, 0);
    std::vector<int> pos(mrp.begin(), mrp.end() - 1);
    for (int i = 0; i < N; i++) mem[pos[agg[i]]++] = i;
}

// graph of the groups: entries in first-touch order over the members' entries, couplings
// summed (g_contract / g_coarse_pattern, semiconductor_3d.c:2368-2404, 2428-2473); emap[e]
// = the group entry fine entry e adds to, -1 inside a group
Csr contract(const Csr &f, const std::vector<int> &agg, int na, std::vector<int> *emap) {
    std::vector<int> mrp, mem;
    members(agg, na, mrp, mem);
    Csr c;
    c.N = na;
    c.rp.assign(na + 1, 0);
    std::vector<int> mark(na, -1), slot(na, 0);
    if (emap) emap->assign(f.cj.size(), -1);
    for (int I = 0; I < na; I++) {
        for (int q = mrp[I]; q < mrp[I + 1]; q++) {
            const int i = mem[q];
            for (int e = f.rp[i]; e < f.rp[i + 1]; e++) {
                const int J = agg[f.cj[e]];
                if (J == I) continue;
                if (mark[J] != I) {
                    mark[J] = I;
                    slot[J] = (int)c.cj.size();
                    c.cj.push_back(J);
                    c.w.push_back(0.0);
                }
                c.w[slot[J]] += f.w[e];
                if (emap) (*emap)[e] = slot[J];
            }
        }
        c.rp[I + 1] = (int)c.cj.size();
    }
    return c;
}

// aggregates of one level: passes rounds of pairing on the successively contracted graph
// (g_aggregate, semiconductor_3d.c:2406-2424)
int aggregate(const Csr &f, int passes, double beta, std::vector<int> &agg) {
    agg.resize(f.N);
    for (int i = 0; i < f.N; i++) agg[i] = i;
    Csr cur;
    const Csr *g = &f;
    int na = f.N;
    std::vector<int> pa;
    for (int pass = 0; pass < passes && g->N > 1; pass++) {
        const int n = g->N;
        na = pair_round(*g, beta, pa);
        for (int i = 0; i < f.N; i++) agg[i] = pa[agg[i]];
        if (pass == passes - 1 || na == n) break;
        Csr nx = contract(*g, pa, na, nullptr);
        cur = std::move(nx);
        g = &cur;
    }
    return na;
}

// greedy colouring in node order: the smallest colour no earlier neighbour took
int colour(const Csr &g, std::vector<int> &color) {
    color.assign(g.N, -1);
    int nc = 0;
    std::vector<int> used;
    for (int k = 0; k < g.N; k++) {
        used.assign(nc + 1, 0);
        for (int e = g.rp[k]; e < g.rp[k + 1]; e++) {
            const int c = color[g.cj[e]];
            if (c >= 0) used[c] = 1;
        }
        int c = 0;
        while (used[c]) c++;
        color[k] = c;
        nc = std::max(nc, c + 1);
    }
    return nc;
}

struct LevelBuild {
    Csr g;                                   // pattern and aggregation strengths
    std::vector<int> agg, mrp, mem, emap;    // towards the next level (CSR entry -> coarse CSR entry)
    std::vector<int> color, cptr, cnodes;
    int ncolor = 0, D = 0;
};

// the levels of a graph (CSR rp / cj, edge lengths h, dual areas ar): patterns, aggregates,
// member lists and entry maps, down to GMG_COARSE nodes or until the aggregation stalls
// (gmg_alloc, semiconductor_3d.c:2475-2512); host only
std::vector<LevelBuild> plan(int N, const std::vector<int> &rp, const std::vector<int> &cj,
                             const std::vector<double> &h, const std::vector<double> &ar, int passes, double beta) {
    std::vector<LevelBuild> B(1);
    B[0].g.N = N;
    B[0].g.rp = rp;
    B[0].g.cj = cj;
    B[0].g.w.resize(cj.size());
    for (size_t e = 0; e < cj.size(); e++) B[0].g.w[e] = h[e] > 0.0 ? ar[e] / h[e] : 0.0;
    while ((int)B.size() < MAXLEV) {
        LevelBuild &f = B.back();
        if (f.g.N <= GMG_COARSE) break;
        std::vector<int> agg;
        const int na = aggregate(f.g, passes, beta, agg);
        if (na < 1 || (double)na > 0.7 * (double)f.g.N) break;
        f.agg = agg;
        members(f.agg, na, f.mrp, f.mem);
        LevelBuild c;
        c.g = contract(f.g, f.agg, na, &f.emap);
        B.push_back(std::move(c));
    }
    return B;
}

}  // namespace

void gmg_free(Inst &d) {
    for (auto &g : d.g.gcyc)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    d.g.gcyc.clear();
    d.g.gcyc_off = false;
    if (d.g.gmgblock) cudaFree(d.g.gmgblock);
    d.g.gmgblock = nullptr;
    if (d.g.gptab) cudaFree(d.g.gptab);
    d.g.gptab = nullptr;
    d.g.glev.clear();
}

// build the hierarchy of the graph in d.ggh (level 0 = the mesh, whose ELL arrays are
// d.g.h's graph fields) and upload the coarse levels
int gmg_build(Inst &d, cudaStream_t st) {
    gmg_free(d);
    const GraphHost &G = d.ggh;
    std::vector<LevelBuild> B = plan((int)d.N, G.rp, G.cj, G.h, G.ar, g_knobs.gpass, g_knobs.gbeta);
    const int nl = (int)B.size();
    for (auto &b : B) {
        b.ncolor = colour(b.g, b.color);
        b.cptr.assign(b.ncolor + 1, 0);
        for (int k = 0; k < b.g.N; k++) b.cptr[b.color[k] + 1]++;
        for (int c = 0; c < b.ncolor; c++) b.cptr[c + 1] += b.cptr[c];
        b.cnodes.assign(b.g.N, 0);
        std::vector<int> fill(b.cptr.begin(), b.cptr.end() - 1);
        for (int k = 0; k < b.g.N; k++) b.cnodes[fill[b.color[k]]++] = k;
        b.D = 0;
        for (int k = 0; k < b.g.N; k++) b.D = std::max(b.D, b.g.rp[k + 1] - b.g.rp[k]);
    }
    // one allocation: per level the ELL pattern (coarse levels), values, diagonal, pivots,
    // colour classes, transfer arrays and vectors, the coarsest inverse
    size_t off = 0;
    auto room = [&](size_t bytes) { const size_t x = off; off += align_up(bytes > 0 ? bytes : 1); return x; };
    struct Off { size_t col, rev, color, val, diag, dil, cn, agg, mrp, mem, emap, pw, ph, x, b, r, inv; };
    std::vector<Off> O(nl);
    for (int L = 0; L < nl; L++) {
        const LevelBuild &b = B[L];
        const size_t n = (size_t)b.g.N, DN = (size_t)b.D * n;
        Off &o = O[L];
        o = Off{};
        o.color = room(n * 4);
        if (L > 0) {
            o.col = room(DN * 4); o.rev = room(DN * 4);
            o.val = room(DN * 8); o.diag = room(n * 8); o.dil = room(n * 8);
        }
        o.cn = room(n * 4);
        if (L < nl - 1) {
            o.agg = room(n * 4); o.mrp = room((size_t)(B[L + 1].g.N + 1) * 4); o.mem = room(n * 4);
            o.emap = room(DN * 4);
        }
        o.pw = room(n * 8); o.ph = room(n * 8); o.x = room(n * 8); o.b = room(n * 8); o.r = room(n * 8);
        if (L == nl - 1 && n <= (size_t)GMG_DENSE_MAX) o.inv = room(n * n * 8);
    }
    char *blk = nullptr;
    if (cudaMalloc(&blk, off) != cudaSuccess) {
        std::fprintf(stderr, "semisim-b200: out of device memory for the graph multigrid\n");
        return 0;
    }
    d.g.gmgblock = blk;
    bool ok = cudaMemsetAsync(blk, 0, off, st) == cudaSuccess;
    std::vector<std::vector<int>> keep;                  // staging kept alive until the copies finish
    auto up = [&](size_t x, std::vector<int> v) {
        if (v.empty()) return;
        keep.push_back(std::move(v));
        if (cudaMemcpyAsync(blk + x, keep.back().data(), keep.back().size() * 4, cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
            ok = false;
    };
    d.g.glev.assign(nl, GLevHost{});
    for (int L = 0; L < nl; L++) {
        const LevelBuild &b = B[L];
        const int n = b.g.N;
        const Off &o = O[L];
        GLevHost &H = d.g.glev[L];
        GLev &v = H.dv;
        v = GLev{};
        v.N = n;
        v.D = b.D;
        if (L > 0) {
            std::vector<int> col((size_t)b.D * n, -1), rev((size_t)b.D * n, 0);
            for (int k = 0; k < n; k++)
                for (int e = b.g.rp[k]; e < b.g.rp[k + 1]; e++) {
                    const int j = b.g.cj[e];
                    int rs = -1;                             // slot of the reverse entry in row j
                    for (int t = b.g.rp[j]; t < b.g.rp[j + 1]; t++)
                        if (b.g.cj[t] == k) { rs = t - b.g.rp[j]; break; }
                    col[(size_t)(e - b.g.rp[k]) * n + k] = j;
                    rev[(size_t)(e - b.g.rp[k]) * n + k] = rs < 0 ? 0 : rs;
                }
            up(o.col, std::move(col));
            up(o.rev, std::move(rev));
            v.col = (const int *)(blk + o.col); v.rev = (const int *)(blk + o.rev);
            v.val = (double *)(blk + o.val); v.diag = (double *)(blk + o.diag); v.dil = (double *)(blk + o.dil);
        }
        up(o.color, b.color);
        v.color = (const int *)(blk + o.color);
        up(o.cn, b.cnodes);
        H.cnodes = (int *)(blk + o.cn);
        H.ncolor = b.ncolor;
        H.cptr = b.cptr;
        if (L < nl - 1) {
            const LevelBuild &c = B[L + 1];
            std::vector<int> em((size_t)b.D * n, -1);      // fine ELL entry -> coarse ELL entry
            for (int k = 0; k < n; k++)
                for (int e = b.g.rp[k]; e < b.g.rp[k + 1]; e++) {
                    const int ce = b.emap[e];
                    if (ce < 0) continue;
                    const int I = b.agg[k];
                    em[(size_t)(e - b.g.rp[k]) * n + k] = (ce - c.g.rp[I]) * c.g.N + I;
                }
            up(o.agg, b.agg);
            up(o.mrp, b.mrp);
            up(o.mem, b.mem);
            up(o.emap, std::move(em));
            v.agg = (const int *)(blk + o.agg); v.mrp = (const int *)(blk + o.mrp);
            v.mem = (const int *)(blk + o.mem); v.emap = (const int *)(blk + o.emap);
        }
        v.pw = (double *)(blk + o.pw); v.ph = (double *)(blk + o.ph);
        v.x = (double *)(blk + o.x); v.b = (double *)(blk + o.b); v.r = (double *)(blk + o.r);
        v.inv = (L == nl - 1 && n <= GMG_DENSE_MAX) ? (double *)(blk + o.inv) : nullptr;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) ok = false;
    if (d.verbose)
        std::fprintf(stderr, "semisim-b200: graph multigrid %d levels, coarsest %d unknowns\n", nl, B.back().g.N);
    return ok ? 1 : 0;
}

// ------------------------------------------------------------------ host: set-up and cycle
namespace {
dim3 grid_for(int n) {
    int b = (n + TPB - 1) / TPB;
    if (b < 1) b = 1;
    if (b > 148 * 8) b = 148 * 8;
    return dim3(b);
}
// level 0 reads the mesh's matrix arrays of the device record (valid after every upload)
void bind_level0(Inst &d) {
    GLev &v = d.g.glev[0].dv;
    const DevP &P = d.g.h;
    v.col = P.gcol; v.rev = P.grev;
    v.val = P.gval; v.diag = P.A[0]; v.dil = P.gdil;
}
void ilu_factor(Inst &d, const Ctx &c, int L) {
    const GLevHost &H = d.g.glev[L];
    for (int q = 0; q < H.ncolor; q++) {
        const int n = H.cptr[q + 1] - H.cptr[q];
        if (n > 0) SS_LAUNCH(PF_ILU_DIAG, n, k_gmg_ilu, grid_for(n), TPB, c.st, H.dv, H.cnodes + H.cptr[q], n);
    }
}
void ilu_apply(Inst &d, const Ctx &c, int L, const double *r, double *z) {
    const GLevHost &H = d.g.glev[L];
    for (int q = 0; q < H.ncolor; q++) {
        const int n = H.cptr[q + 1] - H.cptr[q];
        if (n > 0)
            SS_LAUNCH(PF_SMOOTH_B, n, k_gmg_ilu_apply, grid_for(n), TPB, c.st, H.dv, H.cnodes + H.cptr[q], n, 0, r, z);
    }
    for (int q = H.ncolor - 1; q >= 0; q--) {
        const int n = H.cptr[q + 1] - H.cptr[q];
        if (n > 0)
            SS_LAUNCH(PF_SMOOTH_R, n, k_gmg_ilu_apply, grid_for(n), TPB, c.st, H.dv, H.cnodes + H.cptr[q], n, 1, z, z);
    }
}
void matvec_L(const Ctx &c, const GLev &v, const double *x, const double *b, double *y) {
    SS_LAUNCH(PF_LEVEL_RESID, v.N, k_gmg_matvec, grid_for(v.N), TPB, c.st, v, x, b, y);
}
void vcycle(Inst &d, const Ctx &c, int L, const double *b, double *x, const double *w, bool ilu_only) {
    const int nl = (int)d.g.glev.size();
    const GLev &v = d.g.glev[L].dv;
    if (ilu_only && L == 0 && nl > 1) { ilu_apply(d, c, 0, b, x); return; }
    if (L == nl - 1) {
        if (v.inv) {
            SS_LAUNCH(PF_COARSE, v.N, k_gmg_coarse_solve, grid_for(32 * v.N), TPB, c.st, v, b, x);
        } else {                                          // coarsest too large to invert: D-ILU sweeps
            ilu_apply(d, c, L, b, x);
            for (int s = 0; s < 4; s++) {
                matvec_L(c, v, x, b, v.r);
                ilu_apply(d, c, L, v.r, v.r);
                SS_LAUNCH(PF_PROLONG, v.N, k_gmg_add, grid_for(v.N), TPB, c.st, v.N, x, v.r);
            }
        }
        return;
    }
    const GLev &cv = d.g.glev[L + 1].dv;
    ilu_apply(d, c, L, b, x);                             // pre-smoothing from x = 0
    matvec_L(c, v, x, b, v.r);                            // r = b - A x
    SS_LAUNCH(PF_RESID_RESTRICT, cv.N, k_gmg_restrict, grid_for(cv.N), TPB, c.st, v, cv.N, v.r, cv.b,
              L == 0 ? w : nullptr);
    vcycle(d, c, L + 1, cv.b, cv.x, w, false);
    SS_LAUNCH(PF_PROLONG, v.N, k_gmg_prolong, grid_for(v.N), TPB, c.st, v, cv.x, x, g_knobs.mg_alpha);
    matvec_L(c, v, x, b, v.r);                            // post-smoothing
    ilu_apply(d, c, L, v.r, v.r);
    SS_LAUNCH(PF_PROLONG, v.N, k_gmg_add, grid_for(v.N), TPB, c.st, v.N, x, v.r);
}
}  // namespace

// coarse operators, pivots and the coarsest inverse of the matrix now assembled on the mesh
// (gmg_setup, semiconductor_3d.c:2643-2653); qsign 0 Poisson, +1 electrons, -1 holes; w the
// row weights of the restriction (null: 1)
void gmg_setup(Inst &d, const Ctx &c, int qsign, const double *w) {
    const int nl = (int)d.g.glev.size();
    bind_level0(d);
    for (int L = 0; L < nl - 1; L++) {
        const GLev &f = d.g.glev[L].dv, &cv = d.g.glev[L + 1].dv;
        SS_LAUNCH(PF_WEIGHTS, cv.N, k_gmg_weights, grid_for(cv.N), TPB, c.st, c.dP, f, cv, L, qsign);
    }
    for (int L = 0; L < nl - 1; L++) {
        const GLev &f = d.g.glev[L].dv, &cv = d.g.glev[L + 1].dv;
        SS_LAUNCH(PF_GALERKIN, cv.N, k_gmg_galerkin, grid_for(cv.N), TPB, c.st, f, cv, L == 0 ? w : nullptr);
        ilu_factor(d, c, L);
    }
    const GLev &z = d.g.glev[nl - 1].dv;
    if (z.inv) {
        const int smem = z.N <= GMG_SMEM_MAX;
        const size_t bytes = smem ? (size_t)z.N * z.N * sizeof(double) : 0;
        static std::once_flag attr;          // instances may set up from several host threads
        std::call_once(attr, [] {
            cudaFuncSetAttribute(k_gmg_coarse_setup, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 GMG_SMEM_MAX * GMG_SMEM_MAX * (int)sizeof(double));
        });
        ss::g_launches++;
        ss::t_launches++;
        if (ss::g_prof_on) ss::prof_begin(PF_COARSE_SETUP, c.st);
        k_gmg_coarse_setup<<<1, 1024, bytes, c.st>>>(z, smem);
        if (ss::g_prof_on) ss::prof_end(PF_COARSE_SETUP, c.st, (double)z.N);
    } else {
        ilu_factor(d, c, nl - 1);
    }
}

// z = M^-1 r: one V-cycle (gvcycle, semiconductor_3d.c:2654-2680), or the mesh level's
// D-ILU alone (the reference's fallback after a diverged multigrid solve).  A V-cycle is
// ~100 dependent launches of a few microseconds, so each operand set (the Krylov vectors r,
// z, the row weights, ILU alone or not) is captured once as a CUDA graph and replayed; the
// kernels' arguments - the level views, the mesh level's matrix arrays, the vectors - stay
// fixed for the instance until the hierarchy is rebuilt, which drops the graphs.  With the
// per-launch profiler on, or graphs switched off, the launches go out one by one.
void gmg_apply(Inst &d, const Ctx &c, const double *r, double *z, const double *w, bool ilu_only) {
    if (g_prof_on || !g_use_graphs || d.g.gcyc_off) {
        vcycle(d, c, 0, r, z, w, ilu_only);
        return;
    }
    bind_level0(d);
    GmgCycle *hit = nullptr;
    for (auto &g : d.g.gcyc)
        if (g.r == r && g.z == z && g.w == w && g.ilu_only == ilu_only) { hit = &g; break; }
    if (!hit) {
        GmgCycle g;
        g.r = r; g.z = z; g.w = w; g.ilu_only = ilu_only;
        const unsigned long long l0 = t_launches;
        cudaGraph_t gr = nullptr;
        bool ok = cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            vcycle(d, c, 0, r, z, w, ilu_only);
            ok = cudaStreamEndCapture(c.st, &gr) == cudaSuccess && gr != nullptr;
        }
        g.launches = t_launches - l0;
        g_launches -= g.launches;                  // captured, not run
        t_launches -= g.launches;
        if (ok) ok = cudaGraphInstantiate(&g.exec, gr, 0) == cudaSuccess;
        if (gr) cudaGraphDestroy(gr);
        if (!ok) {                                 // run it the plain way from now on
            cudaGetLastError();
            if (g.exec) cudaGraphExecDestroy(g.exec);
            d.g.gcyc_off = true;
            vcycle(d, c, 0, r, z, w, ilu_only);
            return;
        }
        d.g.gcyc.push_back(g);
        hit = &d.g.gcyc.back();
    }
    cudaGraphLaunch(hit->exec, c.st);
    g_launches += hit->launches;
    t_launches += hit->launches;
}

int gmg_levels(const Inst &d) { return (int)d.g.glev.size(); }

}  // namespace ss

ss::Inst *b200_global_dev();                      // the calling thread's current instance (api.cpp)

// Test hook: set up the graph multigrid of the system now assembled on the mesh (qsign 0:
// Poisson, weights 1; +-1: the continuity row weights and Slotboom weights of that carrier)
// and return level L's coupling values in its CSR order (va, nnz) and its diagonal (dg, n);
// returns nnz, -1 without a graph device or level L
extern "C" int b200x_gmg_vals(int qsign, int L, double *va, double *dg) {
    ss::Inst &d = *b200_global_dev();
    if (!d.unstr || L < 0 || L >= (int)d.g.glev.size()) return -1;
    const ss::Ctx c = ss::make_ctx(d);
    ss::gmg_setup(d, c, qsign, qsign ? d.g.h.dsc : nullptr);
    const ss::GLev &v = d.g.glev[L].dv;
    const size_t DN = (size_t)v.D * v.N;
    std::vector<int> col(DN);
    std::vector<double> val(DN), diag(v.N);
    cudaMemcpyAsync(col.data(), v.col, DN * sizeof(int), cudaMemcpyDeviceToHost, c.st);
    cudaMemcpyAsync(val.data(), v.val, DN * sizeof(double), cudaMemcpyDeviceToHost, c.st);
    cudaMemcpyAsync(diag.data(), v.diag, v.N * sizeof(double), cudaMemcpyDeviceToHost, c.st);
    if (cudaStreamSynchronize(c.st) != cudaSuccess) return -1;
    int nnz = 0;
    for (int k = 0; k < v.N; k++)                       // ELL slot order = the level's CSR order
        for (int s = 0; s < v.D; s++) {
            const size_t e = (size_t)s * v.N + k;
            if (col[e] < 0) break;
            if (va) va[nnz] = val[e];
            nnz++;
        }
    if (dg) std::copy(diag.begin(), diag.end(), dg);
    return nnz;
}

// Test hook (no GPU needed): the graph multigrid hierarchy of a graph (api3_set_mesh_graph's
// CSR arrays) with the current pairing knobs.  Level L's node count and pattern size go to
// n_out / nnz_out; when the buffers are given, its CSR pattern (rp: n + 1, cj: nnz) and, below
// the coarsest level, every node's aggregate (agg: n).  Returns the number of levels.
extern "C" int b200x_gmg_plan(int N, const int *rp, const int *cj, const double *h, const double *ar, int L,
                              int *n_out, int *nnz_out, int *crp, int *ccj, int *agg) {
    if (N < 1 || !rp || !cj || !h || !ar) return 0;
    const int E = rp[N];
    std::vector<int> r(rp, rp + N + 1), c(cj, cj + E);
    std::vector<double> hh(h, h + E), aa(ar, ar + E);
    const auto B = ss::plan(N, r, c, hh, aa, ss::g_knobs.gpass, ss::g_knobs.gbeta);
    const int nl = (int)B.size();
    if (L < 0 || L >= nl) return nl;
    const auto &b = B[L];
    if (n_out) *n_out = b.g.N;
    if (nnz_out) *nnz_out = (int)b.g.cj.size();
    if (crp) std::copy(b.g.rp.begin(), b.g.rp.end(), crp);
    if (ccj) std::copy(b.g.cj.begin(), b.g.cj.end(), ccj);
    if (agg && L < nl - 1) std::copy(b.agg.begin(), b.agg.end(), agg);
    return nl;
}
