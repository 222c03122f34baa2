// Persistent linear solves of general (graph) meshes: one cooperative launch runs a whole
// PCG or BiCGSTAB solve preconditioned by the aggregation multigrid (its V-cycles with the
// multicolour D-ILU(0) smoother, the dense coarsest solve), with grid-wide barriers between
// the dependent passes instead of one kernel launch per colour sweep and a host round trip
// per dot product (pcg_graph / bicg_graph in graph.cu, which this replaces when it applies).
//
// Work layout:
//   * levels larger than GP_SMALL nodes: every block, grid-stride loops, one grid barrier
//     after each pass (each colour of a smoother sweep is a pass);
//   * the smaller levels down to the coarsest: block 0 alone with block barriers (the other
//     blocks wait at the next grid barrier);
//   * fused passes, each the same operations as the per-launch path in one pass: the
//     residual summed straight into the aggregates on the way down, the prolonged iterate
//     read by the residual on the way up, and the correction x += prolongation + smoother
//     output applied by the last (backward) colour sweep of each node.
// The Krylov scalars are reduced in every block (persist_common.cuh), so the stop decisions
// are the same in every block; the stop rules are the reference's (gpcg / gbicgstab,
// semiconductor_3d.c:2682-2714 with bicgstab_core's rules :2244-2320).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gmg_common.cuh"
#include "persist_common.cuh"
#include "prof.h"
#include "solver_ctx.h"

namespace ss {

constexpr int GP_TPB = 1024;
constexpr int GP_MAXC = 64;         // most colours of a level
constexpr int GP_SMALL = 4096;      // levels at or below this size run in block 0
constexpr int GP_MAXL = 16;         // most levels (the level table lives in shared memory)

// one level as the persistent kernel sees it: the level, its colour classes
struct PGLev {
    GLev v;
    int ncolor, pad;
    const int *cnodes;
    int cptr[GP_MAXC + 1];
};
struct GPArgs {
    const PGLev *lev;
    int nl, Ls;          // levels; the first one block 0 runs alone
    int kind;            // 0 PCG, 1 BiCGSTAB
    int ilu_only;        // BiCGSTAB preconditioned by the mesh level's D-ILU(0) alone
    int maxit;
    double alpha, rtol, atol;
    const double *w;     // continuity row weights (restriction of the mesh level) or null
};

// the threads that run a level: the whole grid, or block 0 alone
struct GE {
    int tid, nth;
    bool blk;
};
__device__ __forceinline__ bool ge_sync(PS &s, const GE &e) {
    if (e.blk) { __syncthreads(); return true; }
    return pg_sync(s);
}
#define GP_SYNC(E)                     \
    do {                               \
        if (!ge_sync(s, (E))) return false; \
    } while (0)

// prolonged value of level-L node i: x_i + alpha pw_i xc[agg_i]
__device__ __forceinline__ double gp_xprol(const GLev &f, const double *x, const double *xc, double al, int i) {
    return x[i] + al * f.pw[i] * xc[f.agg[i]];
}

// D-ILU(0) solve z = M^-1 r of one level: forward colours then backward colours.  With xc
// (the way up) the backward sweep of each node finishes the correction x_i += alpha pw_i
// xc[agg_i] + z_i.
__device__ bool gp_ilu(PS &s, const GE &e, const PGLev &H, const double *r, double *z, double *x, const double *xc,
                       double al) {
    const GLev &v = H.v;
    for (int c = 0; c < H.ncolor; c++) {
        const int c0 = H.cptr[c], c1 = H.cptr[c + 1];
        for (int t = c0 + e.tid; t < c1; t += e.nth) gilu_apply_node(v, H.cnodes[t], 0, r, z);
        GP_SYNC(e);
    }
    for (int c = H.ncolor - 1; c >= 0; c--) {
        const int c0 = H.cptr[c], c1 = H.cptr[c + 1];
        for (int t = c0 + e.tid; t < c1; t += e.nth) {
            const int i = H.cnodes[t];
            gilu_apply_node(v, i, 1, z, z);
            if (x) x[i] += (xc ? al * v.pw[i] * xc[v.agg[i]] : 0.0) + z[i];
        }
        GP_SYNC(e);
    }
    return true;
}

// the way down at level L: pre-smoothing x = M^-1 b from x = 0, then the weighted residual
// summed into the aggregates of level L + 1
__device__ bool gp_down(PS &s, const GE &e, const PGLev &H, const PGLev &Hc, const double *b, double *x,
                        const double *w) {
    if (!gp_ilu(s, e, H, b, x, nullptr, nullptr, 0.0)) return false;
    const GLev &f = H.v;
    for (int I = e.tid; I < Hc.v.N; I += e.nth) {
        double sum = 0.0;
        for (int q = f.mrp[I]; q < f.mrp[I + 1]; q++) {
            const int i = f.mem[q];
            const double r = b[i] - gmatvec_row(f, x, i);
            sum += w ? w[i] * r : r;
        }
        Hc.v.b[I] = sum;
    }
    GP_SYNC(e);
    return true;
}

// the way up at level L: residual of the prolonged iterate, its D-ILU(0) correction, and
// x += prolongation + correction (in the backward sweep)
__device__ bool gp_up(PS &s, const GE &e, const PGLev &H, const PGLev &Hc, const double *b, double *x, double al) {
    const GLev &f = H.v;
    const double *xc = Hc.v.x;
    for (int k = e.tid; k < f.N; k += e.nth) {
        double sum = f.diag[k] * gp_xprol(f, x, xc, al, k);
        for (int q = 0; q < f.D; q++) {
            const size_t ee = (size_t)q * f.N + k;
            const int j = f.col[ee];
            if (j >= 0) sum += f.val[ee] * gp_xprol(f, x, xc, al, j);
        }
        f.r[k] = b[k] - sum;
    }
    GP_SYNC(e);
    return gp_ilu(s, e, H, f.r, f.r, x, xc, al);
}

// x = inverse b on the coarsest level (one warp per row)
__device__ bool gp_coarse(PS &s, const GE &e, const PGLev &H, const double *b, double *x) {
    const GLev &v = H.v;
    const int lane = threadIdx.x & 31, n = v.N;
    for (int r = e.tid >> 5; r < n; r += e.nth >> 5) {
        double sum = 0.0;
        for (int q = lane; q < n; q += 32) sum += v.inv[(size_t)r * n + q] * b[q];
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        if (lane == 0) x[r] = sum;
    }
    GP_SYNC(e);
    return true;
}

// one V-cycle z = M^-1 r on the mesh level (gvcycle, semiconductor_3d.c:2654-2680)
__device__ bool gp_vcycle(const DevP &P, PS &s, const GPArgs &a, const double *b0, double *x0) {
    const GE grid{s.tid, s.nth, false};
    if (a.ilu_only) return gp_ilu(s, grid, a.lev[0], b0, x0, nullptr, nullptr, 0.0);
    const int nl = a.nl, Ls = a.Ls;
    for (int L = 0; L < Ls && L < nl - 1; L++)
        if (!gp_down(s, grid, a.lev[L], a.lev[L + 1], L ? a.lev[L].v.b : b0, L ? a.lev[L].v.x : x0,
                     L ? nullptr : a.w))
            return false;
    if (blockIdx.x == 0) {                         // the small levels: block 0 alone
        const GE blk{(int)threadIdx.x, (int)blockDim.x, true};
        for (int L = Ls; L < nl - 1; L++)
            gp_down(s, blk, a.lev[L], a.lev[L + 1], L ? a.lev[L].v.b : b0, L ? a.lev[L].v.x : x0, L ? nullptr : a.w);
        if (Ls <= nl - 1) gp_coarse(s, blk, a.lev[nl - 1], a.lev[nl - 1].v.b, a.lev[nl - 1].v.x);
        for (int L = nl - 2; L >= Ls; L--)
            gp_up(s, blk, a.lev[L], a.lev[L + 1], L ? a.lev[L].v.b : b0, L ? a.lev[L].v.x : x0, a.alpha);
    }
    if (!pg_sync(s)) return false;
    if (Ls > nl - 1 && !gp_coarse(s, grid, a.lev[nl - 1], a.lev[nl - 1].v.b, a.lev[nl - 1].v.x)) return false;
    for (int L = (Ls < nl - 1 ? Ls : nl - 1) - 1; L >= 0; L--)
        if (!gp_up(s, grid, a.lev[L], a.lev[L + 1], L ? a.lev[L].v.b : b0, L ? a.lev[L].v.x : x0, a.alpha))
            return false;
    if (blockIdx.x == 0 && threadIdx.x == 0) s.g->vcycles++;
    return true;
}

// y = A x on the mesh level, with the dot product d = u.y (u null: y.y)
__device__ __forceinline__ double gp_spmv_dot(const PGLev &H, const PS &s, const double *x, double *y, const double *u) {
    const GLev &v = H.v;
    double acc = 0.0;
    for (int k = s.tid; k < v.N; k += s.nth) {
        const double q = gmatvec_row(v, x, k);
        y[k] = q;
        acc += (u ? u[k] : q) * q;
    }
    return acc;
}

__global__ void __launch_bounds__(GP_TPB, 1) k_gpersist(const DevP *Ps, GPArgs ga) {
    const DevP &P = Ps[0];
    __shared__ KrylovS sk;
    // the level table in shared memory: after each grid barrier L1 holds nothing, and the
    // passes would otherwise re-read their level descriptors from L2
    __shared__ PGLev lt[GP_MAXL];
    {
        const int words = ga.nl * (int)(sizeof(PGLev) / sizeof(unsigned));
        const unsigned *src = reinterpret_cast<const unsigned *>(ga.lev);
        unsigned *dst = reinterpret_cast<unsigned *>(lt);
        for (int q = threadIdx.x; q < words; q += blockDim.x) dst[q] = src[q];
    }
    GPArgs a = ga;
    a.lev = lt;
    PS s;
    s.g = P.pgrid;
    s.target = 0;
    s.rb = 0;
    s.tid = blockIdx.x * blockDim.x + threadIdx.x;
    s.nth = gridDim.x * blockDim.x;
    s.wait_ns = PG_WAIT_NS;
    s.trace = nullptr;
    s.ntrace = 0;
    s.mode = 1;
    s.onecl = 0;
    if (threadIdx.x == 0) sk = *P.ks;
    __syncthreads();
    const PGLev &H0 = a.lev[0];
    const int N = P.N;
    double *x = P.sol;
    const double *b = P.rhs;
    if (a.kind == 0) {                            // PCG (gpcg)
        double *r = P.wk[0], *z = P.wk[1], *p = P.wk[2], *q = P.wk[3];
        for (int k = s.tid; k < N; k += s.nth) r[k] = b[k] - gmatvec_row(H0.v, x, k);
        if (!pg_sync(s)) return;
        if (!gp_vcycle(P, s, a, r, z)) return;
        double acc[1] = {0.0};
        for (int k = s.tid; k < N; k += s.nth) acc[0] += r[k] * z[k];
        if (!pg_sum<1>(s, acc)) return;
        if (threadIdx.x == 0) {
            sk.rz = sk.rz0 = acc[0]; sk.it = 0; sk.status = 0;
            sk.active = acc[0] > 0.0 ? 1 : 0;
            if (!sk.active) sk.status = 2;
        }
        __syncthreads();
        if (sk.active) {
            for (int k = s.tid; k < N; k += s.nth) p[k] = z[k];
            if (!pg_sync(s)) return;
        }
        while (sk.active) {
            acc[0] = gp_spmv_dot(H0, s, p, q, p);
            if (!pg_sum<1>(s, acc)) return;
            if (threadIdx.x == 0) {
                sk.it++;
                if (!(acc[0] > 0.0)) { sk.active = 0; sk.status = 2; }
                else sk.al = sk.rz / acc[0];
            }
            __syncthreads();
            if (!sk.active) break;
            for (int k = s.tid; k < N; k += s.nth) { x[k] += sk.al * p[k]; r[k] -= sk.al * q[k]; }
            if (!pg_sync(s)) return;
            if (!gp_vcycle(P, s, a, r, z)) return;
            acc[0] = 0.0;
            for (int k = s.tid; k < N; k += s.nth) acc[0] += r[k] * z[k];
            if (!pg_sum<1>(s, acc)) return;
            if (threadIdx.x == 0) {
                const double rzn = acc[0];
                if (!(rzn > sk.rtol * sk.rtol * sk.rz0)) { sk.active = 0; sk.status = 1; }
                else if (sk.it >= sk.maxit) { sk.active = 0; sk.status = 3; }
                else { sk.be = rzn / sk.rz; sk.rz = rzn; }
            }
            __syncthreads();
            if (!sk.active) break;
            for (int k = s.tid; k < N; k += s.nth) p[k] = sk.be * p[k] + z[k];
            if (!pg_sync(s)) return;
        }
    } else {                                      // BiCGSTAB (gbicgstab)
        double *r = P.wk[0], *rh = P.wk[1], *p = P.wk[2], *v = P.wk[3], *ph = P.wk[4], *sh = P.wk[5], *t = P.wk[6];
        double acc[2] = {0.0, 0.0};
        for (int k = s.tid; k < N; k += s.nth) {
            const GLev &g = H0.v;
            double sum = g.diag[k] * x[k], fl = fabs(g.diag[k] * x[k]) + fabs(b[k]);
            for (int qq = 0; qq < g.D; qq++) {
                const size_t e = (size_t)qq * N + k;
                const int j = g.col[e];
                if (j < 0) continue;
                const double tv = g.val[e] * x[j];
                sum += tv;
                fl += fabs(tv);
            }
            const double rk = b[k] - sum;
            r[k] = rk; rh[k] = rk; p[k] = 0.0; v[k] = 0.0;
            acc[0] += rk * rk;
            acc[1] += fl * fl;
        }
        if (!pg_sum<2>(s, acc)) return;
        if (threadIdx.x == 0) {
            sk.rr = acc[0]; sk.fl = acc[1];
            sk.r0 = sqrt(acc[0]);
            sk.tgt = fmax(a.rtol * sk.r0, a.atol * sqrt(acc[1]));
            sk.rho = sk.al = sk.om = 1.0; sk.rbest = sk.r0; sk.stall = 0; sk.it = 0; sk.half = 0;
            sk.active = sk.r0 > sk.tgt ? 1 : 0;
            sk.status = sk.active ? 0 : 1;
        }
        __syncthreads();
        while (sk.active) {
            double a1[1] = {0.0};
            for (int k = s.tid; k < N; k += s.nth) a1[0] += rh[k] * r[k];
            if (!pg_sum<1>(s, a1)) return;
            if (threadIdx.x == 0) {
                if (sk.it >= sk.maxit) { sk.active = 0; sk.status = 3; }
                else {
                    sk.it++;
                    sk.pad0 = fabs(a1[0]) < 1e-300;
                    sk.rho1 = a1[0];
                }
            }
            __syncthreads();
            if (!sk.active) break;
            if (sk.pad0) {                        // breakdown: restart the shadow residual
                a1[0] = 0.0;
                for (int k = s.tid; k < N; k += s.nth) { rh[k] = r[k]; p[k] = 0.0; v[k] = 0.0; a1[0] += r[k] * r[k]; }
                if (!pg_sum<1>(s, a1)) return;
                if (threadIdx.x == 0) {
                    sk.rho1 = a1[0];
                    sk.rho = sk.al = sk.om = 1.0;
                    if (!(a1[0] > 0.0)) { sk.active = 0; sk.status = 2; }
                }
                __syncthreads();
                if (!sk.active) break;
            }
            if (threadIdx.x == 0) sk.be = (sk.rho1 / sk.rho) * (sk.al / sk.om);
            __syncthreads();
            {
                const double be = sk.be, om = sk.om;
                for (int k = s.tid; k < N; k += s.nth) p[k] = be * p[k] + r[k] - be * om * v[k];
            }
            if (!pg_sync(s)) return;
            if (!gp_vcycle(P, s, a, p, ph)) return;
            a1[0] = gp_spmv_dot(H0, s, ph, v, rh);
            if (!pg_sum<1>(s, a1)) return;
            if (threadIdx.x == 0) {
                if (fabs(a1[0]) < 1e-300) { sk.active = 0; sk.status = 2; }
                else { sk.rv = a1[0]; sk.al = sk.rho1 / a1[0]; }
            }
            __syncthreads();
            if (!sk.active) break;
            const double al = sk.al;
            a1[0] = 0.0;
            for (int k = s.tid; k < N; k += s.nth) {
                const double q = r[k] - al * v[k];
                r[k] = q;
                a1[0] += q * q;
            }
            if (!pg_sum<1>(s, a1)) return;
            if (threadIdx.x == 0) {
                sk.ss = a1[0];
                if (sqrt(a1[0]) <= sk.tgt) { sk.half = 1; sk.rr = a1[0]; }
            }
            __syncthreads();
            if (sk.half) {                        // half-step exit: x += al ph
                for (int k = s.tid; k < N; k += s.nth) x[k] += al * ph[k];
                if (threadIdx.x == 0) { sk.active = 0; sk.status = 1; }
                if (!pg_sync(s)) return;
                break;
            }
            if (!gp_vcycle(P, s, a, r, sh)) return;
            acc[0] = acc[1] = 0.0;
            for (int k = s.tid; k < N; k += s.nth) {
                const double q = gmatvec_row(H0.v, sh, k);
                t[k] = q;
                acc[0] += q * q;
                acc[1] += r[k] * q;
            }
            if (!pg_sum<2>(s, acc)) return;
            if (threadIdx.x == 0) {
                sk.tt = acc[0]; sk.ts = acc[1];
                sk.om = acc[0] > 0.0 ? acc[1] / acc[0] : 0.0;
            }
            __syncthreads();
            {
                const double om = sk.om;
                a1[0] = 0.0;
                for (int k = s.tid; k < N; k += s.nth) {
                    x[k] += al * ph[k] + om * sh[k];
                    const double q = r[k] - om * t[k];
                    r[k] = q;
                    a1[0] += q * q;
                }
            }
            if (!pg_sum<1>(s, a1)) return;
            if (threadIdx.x == 0) {
                sk.rr = a1[0];
                const double rn = sqrt(a1[0]);
                if (rn <= sk.tgt || sk.om == 0.0) { sk.active = 0; sk.status = 1; }
                else {
                    if (rn < 0.99 * sk.rbest) { sk.rbest = rn; sk.stall = 0; }
                    else if (++sk.stall > 40) { sk.active = 0; sk.status = 2; }
                    if (sk.active) sk.rho = sk.rho1;
                }
            }
            __syncthreads();
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *P.ks = sk;
        s.g->iters = sk.it;
    }
}

// ---------------------------------------------------------------- host side
namespace {
int g_gp_blocks = 0;               // co-resident blocks of k_gpersist (0: not read yet)
}

// Launch the persistent graph solve (kind 0 PCG from the present sol with the stop rule
// r.z <= rtol^2 r0.z0; kind 1 BiCGSTAB with max(rtol r0, atol floor)).  The hierarchy must
// be set up.  Returns 1 when it ran (P.ks holds it, rr, r0), 0 when it does not apply
// (nothing changed), -1 when a barrier wait ran out (the caller restores the start).
int persist_graph(Inst &d, int kind, int maxit, double rtol, double atol, const double *w, bool ilu_only) {
    if (!persist_enabled() || d.g.glev.empty()) return 0;
    const int nl = (int)d.g.glev.size();
    std::vector<PGLev> tab(nl);
    int Ls = nl;
    for (int L = 0; L < nl; L++) {
        const GLevHost &H = d.g.glev[L];
        if (H.ncolor > GP_MAXC) return 0;
        if (L == nl - 1 && !H.dv.inv && nl > 1) return 0;      // coarsest by ILU sweeps: per-launch path
        PGLev &p = tab[L];
        p.v = H.dv;
        p.ncolor = H.ncolor;
        p.cnodes = H.cnodes;
        for (int c = 0; c <= H.ncolor; c++) p.cptr[c] = H.cptr[c];
        if (L > 0 && Ls == nl && H.dv.N <= GP_SMALL) Ls = L;
    }
    if (nl < 2 && !ilu_only) return 0;
    if (!d.g.gptab) {
        if (cudaMalloc(&d.g.gptab, sizeof(PGLev) * 32) != cudaSuccess) { cudaGetLastError(); return 0; }
    }
    if (nl > GP_MAXL) return 0;
    if (!g_gp_blocks) {
        int per = 0, dev = 0, nsm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_gpersist, GP_TPB, 0);
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        g_gp_blocks = per * nsm;
        cudaGetLastError();
    }
    int nb = g_gp_blocks;
    const int want = (int)((d.N + 2 * GP_TPB - 1) / (2 * GP_TPB));
    if (want < nb) nb = want < 4 ? 4 : want;
    const int cap = persist_get_blocks();
    if (cap > 0 && cap < nb) nb = cap;
    if (d.pblocks > 0 && d.pblocks < nb) nb = d.pblocks;
    if (nb > PG_MAXB) nb = PG_MAXB;
    if (nb < 1) return 0;
    Ctx c = make_ctx(d);
    cudaMemcpyAsync(d.g.gptab, tab.data(), sizeof(PGLev) * nl, cudaMemcpyHostToDevice, c.st);
    KrylovS ks0{};
    ks0.maxit = maxit;
    ks0.rtol = rtol;
    ks0.atol = atol;
    ks0.active = 1;
    cudaMemcpyAsync(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
    PGrid *g = c.h.pgrid;
    cudaMemsetAsync(g, 0, 6 * sizeof(unsigned), c.st);
    GPArgs a{};
    a.lev = reinterpret_cast<const PGLev *>(d.g.gptab);
    a.nl = nl;
    a.Ls = Ls;
    a.kind = kind;
    a.ilu_only = ilu_only ? 1 : 0;
    a.maxit = maxit;
    a.alpha = g_knobs.mg_alpha;
    a.rtol = rtol;
    a.atol = atol;
    a.w = w;
    const DevP *dp = c.dP;
    void *args[] = {(void *)&dp, (void *)&a};
    g_launches++;
    t_launches++;
    if (g_prof_on) prof_begin(PF_PERSIST, c.st);
    const cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_gpersist, dim3(nb), dim3(GP_TPB), args, 0, c.st);
    if (g_prof_on) prof_end(PF_PERSIST, c.st, 0.0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    PGrid h{};
    cudaMemcpyAsync(&h, g, 6 * sizeof(unsigned), cudaMemcpyDeviceToHost, c.st);
    cudaStreamSynchronize(c.st);
    if (h.err) {
        std::fprintf(stderr, "semisim-b200: persistent graph solve abandoned (a barrier wait ran out)\n");
        return -1;
    }
    return 1;
}

}  // namespace ss
