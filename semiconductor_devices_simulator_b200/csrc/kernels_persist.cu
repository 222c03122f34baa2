// Persistent linear solves: one cooperative launch runs a whole multigrid-preconditioned
// Krylov solve of an instance - every iteration, both V-cycles of a BiCGSTAB iteration,
// and for the refined path every FP64 refinement step around its FP32 inner solves -
// with grid-wide barriers between the dependent passes instead of kernel boundaries.
//
// Why: on a 576k-node device a V-cycle is ~26 dependent passes of 1-10 MB each.  Launched
// one kernel per pass (the device-looped CUDA graphs of kernels_la.cu) every pass costs a
// launch and a grid ramp (~6-9 us) for ~1-2 us of memory traffic; a resident grid pays a
// barrier (~1-2 us) instead and keeps the level descriptors and the small levels on chip.
//
// Layout of the work:
//   * every block runs the passes of the large levels (0 .. Ls-1) as grid-stride loops
//     over the pass's index space, one barrier after each pass;
//   * block 0 keeps the small levels (Ls .. coarsest) in its shared memory for the whole
//     solve (staged once at the start, not per V-cycle) and runs their part of every
//     V-cycle with block barriers, while the other blocks wait at the next grid barrier;
//   * reductions: each block writes its partial record, and after the barrier every block
//     sums all records in block order, so every block holds bit-identical totals and takes
//     the same stop decisions with no extra barrier.
//
// The arithmetic per node is the per-pass kernels' (the shared helpers of la_common.cuh);
// the stop rules are the reference's (pcg semiconductor_3d.c:2182-2210, bicgstab_core
// :2234-2320) as the per-pass path applies them, and the refinement the same FP64 rule.
//
// Safety: the launch is cooperative (all blocks co-resident).  Every barrier wait is
// bounded: after 2 s of waiting a block sets the error word and leaves, every other block
// leaves at its next wait, and the host restores the solve's start and repeats it on the
// per-pass path.
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <mutex>
#include <vector>

#include "la_common.cuh"
#include "persist_common.cuh"
#include "prof.h"

// the pass functions inline into the kernel (compiled apart, __noinline__, they measured
// 30 % slower: every view field was reloaded after each store)
#ifndef PG_PASS
#define PG_PASS __forceinline__
#endif

namespace ss {

enum PKind { PK_PCG = 0, PK_BICG = 1, PK_REFINED = 2 };

struct PArgs {
    int Ls;          // first level of the shared-memory part (>= 1)
    int deep;        // levels (from the finest) with two smoother applications
    int sweeps2;     // 1: the second application is on
    int maxsteps;    // refinement steps at most (PK_REFINED)
    int fuse_up;     // 1: prolongation deferred into the residual and post-smoothing passes
    int setup;       // 1: build the hierarchy first (the per-launch mg_setup of kernels_la.cu)
    int qsign;       // its Slotboom weights: 0 none (Poisson), +1 electrons, -1 holes
    unsigned long long *trace;   // barrier timeline of this launch (null: off)
    int ntrace;
    int barmode;                 // grid-barrier form (persist_common.cuh)
    int csz;                     // CTAs of a thread-block cluster (0: launched without clusters)
    int Lc;                      // first level the first cluster runs alone (cluster barriers)
    int onecl;                   // the whole grid is one cluster
    double alpha;    // prolongation factor
    double rtol, atol;   // stop rule of the FP64 BiCGSTAB start (PK_BICG)
};

// ---------------------------------------------------------------- on-chip tables
// Every descriptor a pass needs (level views, vector pointers) is copied into shared
// memory once per launch: after each grid barrier the acquire invalidates L1, so a
// descriptor read from global memory would cost a chain of dependent L2 round trips per
// pass, more than the pass's own loads on the small levels.
template <class T>
struct PTab {
    LevView<T> lev[MAXLEV];      // every level; level 0's x and b are set per V-cycle
    T *vec[8];                   // level-0 work vectors of precision T
    T *sol, *rhs;
    const T *w0;                 // level-0 row weights (continuity systems)
    const double *A64;           // the FP64 level-0 operator (coupling q at A64 + q * ap64 + k)
    int ap64;
    LevView<T> cur0;             // level 0 with the running V-cycle's b and x
};
template <class T>
__device__ __forceinline__ void ptab_fill(const DevP &P, PTab<T> &tb) {
    const int nl = P.nlev, t = threadIdx.x;
    if (t < nl) tb.lev[t] = levview<T>(P, t, 0, 0);
    if (t >= 32 && t < 40) tb.vec[t - 32] = PT<T>::wk(P, t - 32);
    if (t == 40) {
        tb.sol = PT<T>::sol(P);
        tb.rhs = PT<T>::rhs(P);
        tb.w0 = PT<T>::w0(P);
        tb.A64 = P.A[0];
        tb.ap64 = (int)(P.A[1] - P.A[0]);
    }
}
// level 0 with the V-cycle's b and x, for the passes to read from shared memory (every
// thread of the block calls it: it ends with a block barrier)
template <class T>
__device__ __forceinline__ void set_lev0(PTab<T> &tb, int bsel, int xsel) {
    if (threadIdx.x == 0) {
        tb.cur0 = tb.lev[0];
        tb.cur0.b = tb.vec[bsel];
        tb.cur0.x = tb.vec[xsel];
    }
    __syncthreads();
}

// ---------------------------------------------------------------- grid passes of a level
// (i, j, l) and node index of item t of a half sweep over one colour
struct HItem { int k, i, j, l; bool ok; };
template <class T>
__device__ __forceinline__ HItem hitem(const LevView<T> &v, int t, int tot, int color) {
    HItem h;
    h.ok = t < tot;
    if (!h.ok) { h.k = h.i = h.j = h.l = 0; return h; }
    const int hx = (v.Nx + 1) >> 1;
    const int row = t / hx, ti = t - row * hx;
    h.l = row / v.Ny;
    h.j = row - h.l * v.Ny;
    h.i = 2 * ti + ((h.j + h.l + color) & 1);
    h.ok = h.i < v.Nx;
    h.k = h.i + v.Nx * row;
    return h;
}
// new x (and the z parked in r for the other colour's sweep) of one node of a half sweep,
// without storing: the smoother update of smooth_node (la_common.cuh) split into its
// loads and its stores, so that two nodes' loads can be in flight together (a node of the
// sweep's colour reads only the other colour's nodes and itself)
template <class T>
struct SmRes { T x, r; };
template <class T>
__device__ __forceinline__ SmRes<T> smooth_eval(const LevView<T> &v, const HItem &h, int mode, int color) {
    SmRes<T> o;
    const int k = h.k;
    if (mode == 2) {
        if (color) {
            const T z = (v.b[k] - lv_apply<T>(v, v.x, k, h.i, h.j, h.l)) * v.D[k];
            o.x = v.x[k] + z;
            o.r = z;
        } else {
            o.x = v.x[k] - lv_offdiag<T>(v, v.r, k, h.i, h.j, h.l) * v.D[k];
            o.r = 0;
        }
        return o;
    }
    const T *src = mode ? v.r : v.b;
    T z;
    if (color) z = (src[k] - lv_offdiag_scaled<T>(v, src, k, h.i, h.j, h.l)) * v.D[k];
    else z = (src[k] - lv_offdiag<T>(v, mode ? v.r : v.x, k, h.i, h.j, h.l)) * v.D[k];
    o.x = mode ? v.x[k] + z : z;
    o.r = z;
    return o;
}
// the stores of smooth_eval's result (r only where the sweep parks z: black, modes 1, 2)
template <class T>
__device__ __forceinline__ void smooth_store(const LevView<T> &v, const HItem &h, const SmRes<T> &o, int mode,
                                             int color) {
    v.x[h.k] = o.x;
    if (color && mode) v.r[h.k] = o.r;
}
// prolongation of the coarse correction to node h (added by the deferred way up)
template <class T>
__device__ __forceinline__ T prol_at(const LevView<T> &f, const LevView<T> &cl, T al, int k, int i, int j, int l) {
    const int I = f.cx ? i >> 1 : i, J = f.cy ? j >> 1 : j, K = f.cz ? l >> 1 : l;
    return al * f.pw[k] * cl.x[I + cl.Nx * (J + cl.Ny * K)];
}
// half sweep of one colour, two nodes per thread and loop trip; cl non-null: post-
// smoothing with the deferred prolongation added to each node first (mode 1)
template <class T>
__device__ PG_PASS void pg_smooth(const LevView<T> &vr, int mode, int color, const PS &s,
                                       const LevView<T> *clr = nullptr, T al = 0) {
    const LevView<T> v = vr;                      // register copies of the shared-memory views
    LevView<T> clv;
    const LevView<T> *cl = nullptr;
    if (clr) { clv = *clr; cl = &clv; }
    const int hx = (v.Nx + 1) >> 1, tot = hx * v.Ny * v.Nz;
    for (int t = s.tid; t < tot; t += 2 * s.nth) {
        const HItem h1 = hitem(v, t, tot, color), h2 = hitem(v, t + s.nth, tot, color);
        SmRes<T> o1{0, 0}, o2{0, 0};
        T p1 = 0, p2 = 0;
        if (h1.ok) {
            o1 = smooth_eval<T>(v, h1, mode, color);
            if (cl) p1 = prol_at<T>(v, *cl, al, h1.k, h1.i, h1.j, h1.l);
        }
        if (h2.ok) {
            o2 = smooth_eval<T>(v, h2, mode, color);
            if (cl) p2 = prol_at<T>(v, *cl, al, h2.k, h2.i, h2.j, h2.l);
        }
        if (h1.ok) { o1.x += p1; smooth_store<T>(v, h1, o1, mode, color); }
        if (h2.ok) { o2.x += p2; smooth_store<T>(v, h2, o2, mode, color); }
    }
}
// weighted residual of every fine node summed into its 2x2x2 aggregate: 8 lanes per
// coarse node (lane bits di, dj, dl), whole warps per loop trip, two trips' loads together
template <class T>
__device__ __forceinline__ T rr_val(const LevView<T> &f, const LevView<T> &cl, const T *w, int t) {
    const int K = t >> 3, sub = t & 7;
    if (K >= cl.N) return 0;
    const Node c = unidx(K, cl.Nx, cl.Ny);
    const int di = sub & 1, dj = (sub >> 1) & 1, dl = sub >> 2;
    const int i = f.cx ? 2 * c.i + di : c.i, j = f.cy ? 2 * c.j + dj : c.j, l = f.cz ? 2 * c.l + dl : c.l;
    const bool ok = i < f.Nx && j < f.Ny && l < f.Nz && (f.cx || di == 0) && (f.cy || dj == 0) && (f.cz || dl == 0);
    if (!ok) return 0;
    const int k = i + f.Nx * (j + f.Ny * l);
    const T r = f.b[k] - lv_apply<T>(f, f.x, k, i, j, l);
    return w ? w[k] * r : r;
}
template <class T>
__device__ __forceinline__ T oct_sum(T v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    return v;
}
template <class T>
__device__ PG_PASS void pg_resid_restrict(const LevView<T> &fr, const LevView<T> &clr, const T *w, const PS &s) {
    const LevView<T> f = fr, cl = clr;            // register copies of the shared-memory views
    const int nK = ((cl.N + 3) >> 2) << 5;
    for (int t = s.tid; t < nK; t += 2 * s.nth) {
        const int t2 = t + s.nth;                 // whole warps: nK and nth are multiples of 32
        T v1 = rr_val<T>(f, cl, w, t);
        T v2 = t2 < nK ? rr_val<T>(f, cl, w, t2) : T(0);
        v1 = oct_sum<T>(v1);
        if (t2 < nK) v2 = oct_sum<T>(v2);
        if ((t & 7) == 0 && (t >> 3) < cl.N) cl.b[t >> 3] = v1;
        if (t2 < nK && (t2 & 7) == 0 && (t2 >> 3) < cl.N) cl.b[t2 >> 3] = v2;
    }
}
template <class T>
__device__ PG_PASS void pg_prolong(const LevView<T> &fr, const LevView<T> &clr, T al, const PS &s) {
    const LevView<T> f = fr, cl = clr;
    for (int k = s.tid; k < f.N; k += s.nth) {
        const Node a = unidx(k, f.Nx, f.Ny);
        f.x[k] += prol_at<T>(f, cl, al, k, a.i, a.j, a.l);
    }
}
template <class T>
__device__ PG_PASS void pg_resid(const LevView<T> &fr, const PS &s) {
    const LevView<T> f = fr;
    for (int k = s.tid; k < f.N; k += s.nth) {
        const Node a = unidx(k, f.Nx, f.Ny);
        f.r[k] = f.b[k] - lv_apply<T>(f, f.x, k, a.i, a.j, a.l);
    }
}

// The way up, with the prolongation deferred: the residual pass reads the prolonged
// x + al pw P xc at each stencil point without writing it, and each post-smoothing half
// sweep adds the prolongation to its own colour's nodes - the same operations as a
// prolongation pass followed by a residual pass, one barrier fewer.
template <class T>
__device__ __forceinline__ T xprol(const LevView<T> &f, const LevView<T> &cl, T al, int m, int i, int j, int l) {
    return f.x[m] + prol_at<T>(f, cl, al, m, i, j, l);
}
template <class T>
__device__ __forceinline__ T pr_val(const LevView<T> &f, const LevView<T> &cl, T al, int k) {
    const int NxNy = f.Nx * f.Ny;
    const Node a = unidx(k, f.Nx, f.Ny);
    const int i = a.i, j = a.j, l = a.l;
    T sum = f.a(0, k) * xprol<T>(f, cl, al, k, i, j, l);
    if (i > 0) sum += f.a(1, k) * xprol<T>(f, cl, al, k - 1, i - 1, j, l);
    if (i < f.Nx - 1) sum += f.a(2, k) * xprol<T>(f, cl, al, k + 1, i + 1, j, l);
    if (j > 0) sum += f.a(3, k) * xprol<T>(f, cl, al, k - f.Nx, i, j - 1, l);
    if (j < f.Ny - 1) sum += f.a(4, k) * xprol<T>(f, cl, al, k + f.Nx, i, j + 1, l);
    if (l > 0) sum += f.a(5, k) * xprol<T>(f, cl, al, k - NxNy, i, j, l - 1);
    if (l < f.Nz - 1) sum += f.a(6, k) * xprol<T>(f, cl, al, k + NxNy, i, j, l + 1);
    return f.b[k] - sum;
}
template <class T>
__device__ PG_PASS void pg_prolong_resid(const LevView<T> &fr, const LevView<T> &clr, T al, const PS &s) {
    const LevView<T> f = fr, cl = clr;            // register copies of the shared-memory views
    for (int k = s.tid; k < f.N; k += 2 * s.nth) {
        const int k2 = k + s.nth;
        const T r1 = pr_val<T>(f, cl, al, k);
        const T r2 = k2 < f.N ? pr_val<T>(f, cl, al, k2) : T(0);
        f.r[k] = r1;
        if (k2 < f.N) f.r[k2] = r2;
    }
}

#define PG_SYNC()                   \
    do {                            \
        if (!pg_sync(s)) return false; \
    } while (0)

// The passes of one level on the way down (pre-smoothing, residual restricted to the next
// level) and on the way up (prolongation, residual, post-smoothing), each pass followed by
// `sync` - the grid barrier, or the first cluster's hardware barrier for the levels it runs
// alone.  The same passes as the per-pass path (vcycle_t in kernels_la.cu).
template <class T, class Sync>
__device__ __forceinline__ bool pg_level_down(const PS &e, const PArgs &a, PTab<T> &tb, int L, int wsel, Sync sync) {
    const LevView<T> &v = L ? tb.lev[L] : tb.cur0;
    pg_smooth<T>(v, 0, 1, e);
    if (!sync()) return false;
    pg_smooth<T>(v, 0, 0, e);
    if (!sync()) return false;
    if (L < a.deep && a.sweeps2) {
        pg_smooth<T>(v, 2, 1, e);
        if (!sync()) return false;
        pg_smooth<T>(v, 2, 0, e);
        if (!sync()) return false;
    }
    pg_resid_restrict<T>(v, tb.lev[L + 1], (L == 0 && wsel) ? tb.w0 : nullptr, e);
    return sync();
}
template <class T, class Sync>
__device__ __forceinline__ bool pg_level_up(const PS &e, const PArgs &a, PTab<T> &tb, int L, Sync sync) {
    const T al = (T)a.alpha;
    const LevView<T> &v = L ? tb.lev[L] : tb.cur0;
    const LevView<T> &cl = tb.lev[L + 1];
    if (a.fuse_up) {
        pg_prolong_resid<T>(v, cl, al, e);
        if (!sync()) return false;
        pg_smooth<T>(v, 1, 1, e, &cl, al);
        if (!sync()) return false;
        pg_smooth<T>(v, 1, 0, e, &cl, al);
        if (!sync()) return false;
    } else {
        pg_prolong<T>(v, cl, al, e);
        if (!sync()) return false;
        pg_resid<T>(v, e);
        if (!sync()) return false;
        pg_smooth<T>(v, 1, 1, e);
        if (!sync()) return false;
        pg_smooth<T>(v, 1, 0, e);
        if (!sync()) return false;
    }
    if (L < a.deep && a.sweeps2) {
        pg_smooth<T>(v, 2, 1, e);
        if (!sync()) return false;
        pg_smooth<T>(v, 2, 0, e);
        if (!sync()) return false;
    }
    return true;
}

// one V(1,1) cycle x = M^-1 b on the level-0 vectors (bsel -> xsel).  Levels 0 .. Lc-1: the
// whole grid, grid barriers; levels Lc .. Ls-1: the first cluster alone, cluster barriers
// (0.3 us against 2.2 us for a grid barrier); levels Ls ..: block 0 in shared memory.
template <class T>
__device__ __noinline__ bool pg_vcycle(PS &s, const PArgs &a, PTab<T> &tb, const LevView<T> *sv, int nl, int bsel, int xsel,
                          int wsel) {
    const int Ls = a.Ls, Lc = (a.csz && !a.onecl) ? a.Lc : Ls;
    const T al = (T)a.alpha;
    set_lev0<T>(tb, bsel, xsel);
    auto gsync = [&]() { return pg_sync(s); };
    for (int L = 0; L < Lc; L++)
        if (!pg_level_down<T>(s, a, tb, L, wsel, gsync)) return false;
    if ((int)blockIdx.x < (Lc < Ls ? a.csz : 1)) {         // the first cluster (or block 0 alone)
        PS e = s;
        const int rank = (int)blockIdx.x;                  // a 1-D grid: the first cluster is blocks 0 .. csz-1
        e.tid = rank * blockDim.x + threadIdx.x;
        e.nth = (Lc < Ls ? a.csz : 1) * blockDim.x;
        auto csync = [&]() {
            if (Lc < Ls) cooperative_groups::this_cluster().sync();
            else __syncthreads();
            return true;
        };
        for (int L = Lc; L < Ls; L++) pg_level_down<T>(e, a, tb, L, wsel, csync);
        if (blockIdx.x == 0) {
            const LevView<T> &g = tb.lev[Ls];
            blk_copy<T>(sv[0].b, g.b, g.N);
            __syncthreads();
            blk_vcycle_small<T>(sv, Ls, nl, al);
            blk_copy<T>(g.x, sv[0].x, g.N);
        }
        csync();
        for (int L = Ls - 1; L >= Lc; L--) pg_level_up<T>(e, a, tb, L, csync);
    }
    if (!pg_sync(s)) return false;
    for (int L = Lc - 1; L >= 0; L--)
        if (!pg_level_up<T>(s, a, tb, L, gsync)) return false;
    if (blockIdx.x == 0 && threadIdx.x == 0) s.g->vcycles++;
    return true;
}

// y = A x on level 0 at node k
template <class T>
__device__ __forceinline__ T spmv_at(const LevView<T> &l0, const T *x, int k) {
    const Node nd = unidx(k, l0.Nx, l0.Ny);
    return lv_apply<T>(l0, x, k, nd.i, nd.j, nd.l);
}

// ---------------------------------------------------------------- Krylov loops
// BiCGSTAB iterations (semiconductor_3d.c:2281-2316) on the records `sk` of precision T
// while it is active; the reduction of rh.r for the next iteration rides on the x update.
template <class T>
__device__ bool pg_bicg(PS &s, const PArgs &a, PTab<T> &tb, const LevView<T> *sv, int nl, int N, KrylovS &sk) {
    T *r = tb.vec[0], *rh = tb.vec[1], *p = tb.vec[2], *v = tb.vec[3];
    T *ph = tb.vec[4], *sh = tb.vec[5], *t = tb.vec[6];
    T *x = tb.sol;
    const LevView<T> l0 = tb.lev[0];
    bool have_rho = false;
    double rho_next = 0.0;
    while (sk.active) {
        double acc[2] = {0.0, 0.0}, a1[1] = {0.0};
        if (have_rho) a1[0] = rho_next;
        else {
            for (int k = s.tid; k < N; k += s.nth) a1[0] += (double)rh[k] * (double)r[k];
            if (!pg_sum<1>(s, a1)) return false;
        }
        if (threadIdx.x == 0) {
            if (sk.it >= sk.maxit) { sk.active = 0; sk.status = 3; }
            else {
                sk.it++;
                double rho1 = a1[0];
                sk.pad0 = 0;
                if (fabs(rho1) < 1e-300) {          // breakdown: restart the shadow residual
                    rho1 = sk.rr;
                    sk.rho = sk.al = sk.om = 1.0;
                    sk.pad0 = 1;
                    if (!(rho1 > 0.0)) { sk.active = 0; sk.status = 2; }
                }
                sk.rho1 = rho1;
                sk.be = (rho1 / sk.rho) * (sk.al / sk.om);
            }
        }
        __syncthreads();
        if (!sk.active) break;
        {
            const T be = (T)sk.be, om = (T)sk.om;
            const int restart = sk.pad0;
            for (int k = s.tid; k < N; k += s.nth) {
                if (restart) { rh[k] = r[k]; p[k] = r[k]; v[k] = 0; }
                else p[k] = r[k] + be * (p[k] - om * v[k]);
            }
        }
        PG_SYNC();
        if (!pg_vcycle<T>(s, a, tb, sv, nl, 2, 4, 1)) return false;      // ph = M p
        a1[0] = 0.0;
        for (int k = s.tid; k < N; k += 2 * s.nth) {
            const int k2 = k + s.nth;
            const T q1 = spmv_at<T>(l0, ph, k);
            const T q2 = k2 < N ? spmv_at<T>(l0, ph, k2) : T(0);
            v[k] = q1;
            a1[0] += (double)rh[k] * (double)q1;
            if (k2 < N) { v[k2] = q2; a1[0] += (double)rh[k2] * (double)q2; }
        }
        if (!pg_sum<1>(s, a1)) return false;
        if (threadIdx.x == 0) {
            if (fabs(a1[0]) < 1e-300) { sk.active = 0; sk.status = 2; }
            else { sk.rv = a1[0]; sk.al = sk.rho1 / a1[0]; }
        }
        __syncthreads();
        if (!sk.active) break;
        const T al = (T)sk.al;
        a1[0] = 0.0;
        for (int k = s.tid; k < N; k += s.nth) {
            const T q = r[k] - al * v[k];
            r[k] = q;
            a1[0] += (double)q * (double)q;
        }
        if (!pg_sum<1>(s, a1)) return false;
        if (threadIdx.x == 0) {
            sk.ss = a1[0];
            if (sqrt(a1[0]) <= sk.tgt) { sk.half = 1; sk.rr = a1[0]; }
        }
        __syncthreads();
        if (sk.half) {                                // half-step exit: x += al ph
            for (int k = s.tid; k < N; k += s.nth) x[k] += al * ph[k];
            if (threadIdx.x == 0) { sk.active = 0; sk.status = 1; }
            PG_SYNC();
            break;
        }
        if (!pg_vcycle<T>(s, a, tb, sv, nl, 0, 5, 1)) return false;      // sh = M r
        acc[0] = acc[1] = 0.0;
        for (int k = s.tid; k < N; k += 2 * s.nth) {
            const int k2 = k + s.nth;
            const T q1 = spmv_at<T>(l0, sh, k);
            const T q2 = k2 < N ? spmv_at<T>(l0, sh, k2) : T(0);
            t[k] = q1;
            acc[0] += (double)q1 * (double)q1;
            acc[1] += (double)q1 * (double)r[k];
            if (k2 < N) {
                t[k2] = q2;
                acc[0] += (double)q2 * (double)q2;
                acc[1] += (double)q2 * (double)r[k2];
            }
        }
        if (!pg_sum<2>(s, acc)) return false;
        if (threadIdx.x == 0) {
            sk.tt = acc[0]; sk.ts = acc[1];
            sk.om = acc[0] > 0.0 ? acc[1] / acc[0] : 0.0;
        }
        __syncthreads();
        {
            const T om = (T)sk.om;
            acc[0] = acc[1] = 0.0;
            for (int k = s.tid; k < N; k += s.nth) {
                x[k] += al * ph[k] + om * sh[k];
                const T q = r[k] - om * t[k];
                r[k] = q;
                acc[0] += (double)q * (double)q;
                acc[1] += (double)rh[k] * (double)q;
            }
        }
        if (!pg_sum<2>(s, acc)) return false;
        if (threadIdx.x == 0) {
            sk.rr = acc[0];
            const double rn = sqrt(acc[0]);
            if (rn <= sk.tgt || sk.om == 0.0) { sk.active = 0; sk.status = 1; }
            else {
                if (rn < 0.99 * sk.rbest) { sk.rbest = rn; sk.stall = 0; }
                else if (++sk.stall > 40) { sk.active = 0; sk.status = 2; }
                if (sk.active) sk.rho = sk.rho1;
            }
        }
        have_rho = true;
        rho_next = acc[1];
        __syncthreads();
    }
    return true;
}

// PCG iterations (semiconductor_3d.c:2194-2206) on the records `sk` while active
template <class T>
__device__ bool pg_pcg(PS &s, const PArgs &a, PTab<T> &tb, const LevView<T> *sv, int nl, int N, KrylovS &sk) {
    T *r = tb.vec[0], *z = tb.vec[1], *p = tb.vec[2], *q = tb.vec[3];
    T *x = tb.sol;
    const LevView<T> l0 = tb.lev[0];
    while (sk.active) {
        double acc[1] = {0.0};
        for (int k = s.tid; k < N; k += 2 * s.nth) {
            const int k2 = k + s.nth;
            const T q1 = spmv_at<T>(l0, p, k);
            const T q2 = k2 < N ? spmv_at<T>(l0, p, k2) : T(0);
            q[k] = q1;
            acc[0] += (double)p[k] * (double)q1;
            if (k2 < N) { q[k2] = q2; acc[0] += (double)p[k2] * (double)q2; }
        }
        if (!pg_sum<1>(s, acc)) return false;
        if (threadIdx.x == 0) {
            sk.it++;
            const double pq = acc[0];
            if (!(pq > 0.0)) { sk.active = 0; sk.status = 2; sk.al = 0.0; }
            else sk.al = sk.rz / pq;
        }
        __syncthreads();
        if (!sk.active) break;
        {
            const T al = (T)sk.al;
            for (int k = s.tid; k < N; k += s.nth) { x[k] += al * p[k]; r[k] -= al * q[k]; }
        }
        PG_SYNC();
        if (!pg_vcycle<T>(s, a, tb, sv, nl, 0, 1, 0)) return false;      // z = M r
        acc[0] = 0.0;
        for (int k = s.tid; k < N; k += s.nth) acc[0] += (double)r[k] * (double)z[k];
        if (!pg_sum<1>(s, acc)) return false;
        if (threadIdx.x == 0) {
            const double rz = acc[0];
            if (!(rz > sk.rtol * sk.rtol * sk.rz0)) { sk.active = 0; sk.status = 1; }
            else if (sk.it >= sk.maxit) { sk.active = 0; sk.status = 3; }
            else { sk.be = rz / sk.rz; sk.rz = rz; }
        }
        __syncthreads();
        if (!sk.active) break;
        {
            const T be = (T)sk.be;
            for (int k = s.tid; k < N; k += s.nth) p[k] = z[k] + be * p[k];
        }
        PG_SYNC();
    }
    return true;
}

// (A x)_k of the FP64 level-0 operator and, in fl, sum_j |a_kj x_j|
template <class X>
__device__ __forceinline__ double a64_at(const double *A, int ap, const X *x, int k, int i, int j, int l, int Nx,
                                         int Ny, int Nz, double *fl) {
    const int NxNy = Nx * Ny;
    double t = A[k] * (double)x[k], sum = t, f = fabs(t);
    if (i > 0) { t = A[ap + k] * (double)x[k - 1]; sum += t; f += fabs(t); }
    if (i < Nx - 1) { t = A[2 * ap + k] * (double)x[k + 1]; sum += t; f += fabs(t); }
    if (j > 0) { t = A[3 * ap + k] * (double)x[k - Nx]; sum += t; f += fabs(t); }
    if (j < Ny - 1) { t = A[4 * ap + k] * (double)x[k + Nx]; sum += t; f += fabs(t); }
    if (l > 0) { t = A[5 * ap + k] * (double)x[k - NxNy]; sum += t; f += fabs(t); }
    if (l < Nz - 1) { t = A[6 * ap + k] * (double)x[k + NxNy]; sum += t; f += fabs(t); }
    if (fl) *fl = f;
    return sum;
}

// r = b - A x with the FP64 operator, its squared norm and the squared rounding floor
// (sum_k (sum_j |a_kj x_j| + |b_k|)^2) - the start of the FP64 BiCGSTAB and of the
// refinement (semiconductor_3d.c:2244-2268).  Writes r (FP64 work vector 0) and, when
// r32 is not null, its FP32 copy; with rh, also rh = r and p = v = 0.
template <class T>
__device__ __forceinline__ void pg_start64(const DevP &P, const PTab<T> &tb, const PS &s, float *r32, bool bicg,
                                           double (&acc)[2]) {
    const double *b = P.rhs, *x = P.sol;
    double *r = P.wk[0], *rh = P.wk[1], *p = P.wk[2], *v = P.wk[3];
    const int Nx = P.Nx, Ny = P.Ny, Nz = P.Nz, N = P.N;
    for (int k = s.tid; k < N; k += s.nth) {
        const Node a = unidx(k, Nx, Ny);
        double fl;
        const double sum = a64_at<double>(tb.A64, tb.ap64, x, k, a.i, a.j, a.l, Nx, Ny, Nz, &fl);
        fl += fabs(b[k]);
        const double rk = b[k] - sum;
        r[k] = rk;
        if (bicg) { rh[k] = rk; p[k] = 0.0; v[k] = 0.0; }
        if (r32) r32[k] = (float)rk;
        acc[0] += rk * rk;
        acc[1] += fl * fl;
    }
}

// ---------------------------------------------------------------- hierarchy set-up
// The multigrid set-up of the system now in the level-0 operator (mg_setup_t in
// kernels_la.cu, the reference's mg_setup semiconductor_3d.c:2126-2148): for T = float
// the FP32 copy of the operator and row weights, then per level the Slotboom weights with
// the next level's reference potentials and the smoother pivots (one pass: the pivots
// read only the level's own operator), the Galerkin coarse operator (one pass), and the
// coarsest level's dense inverse (block 0, in its shared memory).
template <class T>
__device__ __noinline__ bool pg_setup(const DevP &P, PS &s, const PArgs &a, const PTab<T> &tb, unsigned char *scratch) {
    const int nl = P.nlev, qsign = a.qsign;
    if constexpr (std::is_same<T, float>::value) {
        float *A32 = const_cast<float *>(tb.lev[0].A);
        const int ap = tb.lev[0].ap;
        for (int k = s.tid; k < P.N; k += s.nth) {
#pragma unroll
            for (int q = 0; q < 7; q++) A32[q * ap + k] = (float)tb.A64[q * tb.ap64 + k];
            if (qsign) P.dsc32[k] = (float)P.dsc[k];
        }
        PG_SYNC();
    }
    for (int L = 0; L < nl - 1; L++) {
        const LevView<T> &f = tb.lev[L];
        const LevelT<T> &cl = PT<T>::lev(P, L + 1);
        for (int K = s.tid; K < cl.N; K += s.nth) mg_weights_node<T>(P, f, cl, L, qsign, K);
        for (int k = s.tid; k < f.N; k += s.nth) ilu_diag_node<T>(f, k);
        PG_SYNC();
        const T *w = (L == 0 && qsign) ? tb.w0 : nullptr;
        for (int K = s.tid; K < cl.N; K += s.nth) galerkin_node<T>(f, cl, w, K);
        PG_SYNC();
    }
    if (blockIdx.x == 0 && nl > 1) {
        double *M = reinterpret_cast<double *>(scratch);
        int *perm = reinterpret_cast<int *>(M + COARSE_MAX * (COARSE_MAX + 1));
        blk_coarse_setup<T>(PT<T>::lev(P, nl - 1), M, perm, perm + COARSE_MAX);
        __syncthreads();
    }
    return true;
}
// dynamic shared memory the set-up's dense inverse needs (block 0)
constexpr size_t PG_SETUP_SMEM = sizeof(double) * COARSE_MAX * (COARSE_MAX + 1) + sizeof(int) * (COARSE_MAX + 1);

// ---------------------------------------------------------------- the solve kernels
// T: precision of the Krylov iterations and the hierarchy.  PK_PCG: the Poisson Newton
// system from the present sol (T = float: sol starts at 0 and the result is copied to the
// FP64 sol when it converged).  PK_BICG (T = double): the continuity system from the
// present sol.  PK_REFINED (T = float): FP64 refinement steps around FP32 BiCGSTAB.
template <class T, int KIND>
__global__ void __launch_bounds__(PG_TPB, 1024 / PG_TPB) k_persist(const DevP *Ps, PArgs a) {
    const DevP &P = Ps[0];
    extern __shared__ __align__(16) unsigned char sraw[];
    __shared__ LevView<T> sv[MAXLEV];
    __shared__ PTab<T> tb;
    __shared__ KrylovS sk, so;                    // the loop's record (and the outer one: PK_REFINED)
    PS s;
    s.g = P.pgrid;
    s.target = 0;
    s.rb = 0;
    s.tid = blockIdx.x * blockDim.x + threadIdx.x;
    s.nth = gridDim.x * blockDim.x;
    s.wait_ns = PG_WAIT_NS;
    s.trace = a.trace;
    s.ntrace = a.ntrace;
    s.mode = a.barmode;
    s.onecl = a.onecl;
    const int nl = P.nlev, N = P.N;
    ptab_fill<T>(P, tb);
    __syncthreads();
    if (a.setup && !pg_setup<T>(P, s, a, tb, sraw)) return;
    if (blockIdx.x == 0) {                        // the small levels stay in block 0's shared memory
        if (threadIdx.x < nl - a.Ls) sv[threadIdx.x] = smem_view<T>(P, a.Ls + threadIdx.x, a.Ls, sraw);
        __syncthreads();
        blk_stage_small<T>(P, sv, a.Ls, nl);
    }
    if (threadIdx.x == 0) {
        sk = *PT<T>::ks(P);
        so = *P.ks;
    }
    __syncthreads();
    KrylovS &rec = sk;
    if constexpr (KIND == PK_PCG) {
        T *r0 = tb.vec[0];
        if constexpr (std::is_same<T, double>::value) {
            for (int k = s.tid; k < N; k += s.nth) {
                const Node nd = unidx(k, P.Nx, P.Ny);
                r0[k] = P.rhs[k] - a64_at<double>(tb.A64, tb.ap64, P.sol, k, nd.i, nd.j, nd.l, P.Nx, P.Ny, P.Nz,
                                                  nullptr);
            }
        } else {
            float *b32 = tb.rhs, *x32 = tb.sol;
            for (int k = s.tid; k < N; k += s.nth) {
                const float b = (float)P.rhs[k];
                b32[k] = b;
                r0[k] = b;
                x32[k] = 0.f;
            }
        }
        if (!pg_sync(s)) return;
        if (!pg_vcycle<T>(s, a, tb, sv, nl, 0, 1, 0)) return;        // z = M r
        double acc[1] = {0.0};
        const T *z = tb.vec[1];
        for (int k = s.tid; k < N; k += s.nth) acc[0] += (double)r0[k] * (double)z[k];
        if (!pg_sum<1>(s, acc)) return;
        if (threadIdx.x == 0) {
            const double rz = acc[0];
            rec.rz = rec.rz0 = rz; rec.it = 0; rec.status = 0;
            rec.active = (rz > 0.0) ? 1 : 0;
            if (!(rz > 0.0)) rec.status = 2;
        }
        __syncthreads();
        if (rec.active) {
            T *p = tb.vec[2];
            for (int k = s.tid; k < N; k += s.nth) p[k] = z[k];
            if (!pg_sync(s)) return;
            if (!pg_pcg<T>(s, a, tb, sv, nl, N, rec)) return;
        }
        if constexpr (std::is_same<T, float>::value) {
            if (rec.status == 1)
                for (int k = s.tid; k < N; k += s.nth) P.sol[k] = (double)tb.sol[k];
        }
    } else if constexpr (KIND == PK_BICG) {
        double acc[2] = {0.0, 0.0};
        pg_start64<T>(P, tb, s, nullptr, true, acc);
        if (!pg_sum<2>(s, acc)) return;
        if (threadIdx.x == 0) {
            rec.rr = acc[0]; rec.fl = acc[1];
            rec.r0 = sqrt(acc[0]);
            rec.tgt = fmax(a.rtol * rec.r0, a.atol * sqrt(acc[1]));
            rec.rho = rec.al = rec.om = 1.0; rec.rbest = rec.r0; rec.stall = 0; rec.it = 0; rec.half = 0;
            if (!(rec.r0 > rec.tgt)) { rec.active = 0; rec.status = 1; }
            else { rec.active = 1; rec.status = 0; }
        }
        __syncthreads();
        if (!pg_bicg<T>(s, a, tb, sv, nl, N, rec)) return;
    } else {                                      // PK_REFINED
        double acc[2] = {0.0, 0.0};
        float *rhs32 = tb.rhs;
        pg_start64<T>(P, tb, s, rhs32, false, acc);
        if (!pg_sum<2>(s, acc)) return;
        if (threadIdx.x == 0) {
            so.rr = acc[0]; so.fl = acc[1];
            so.r0 = sqrt(acc[0]);
            so.tgt = fmax(so.rtol * so.r0, so.atol * sqrt(acc[1]));
            so.rbest = so.r0; so.stall = 0; so.it = 0; so.half = 0;
            if (!(so.r0 > so.tgt)) { so.active = 0; so.status = 1; }
            else { so.active = 1; so.status = 0; }
        }
        __syncthreads();
        int steps = 0;
        double *x = P.sol, *r64 = P.wk[0];
        const int Nx = P.Nx, Ny = P.Ny, Nz = P.Nz;
        for (; steps < a.maxsteps && so.active; steps++) {
            // inner start: d = 0, r = rh = rhs32, p = v = 0
            float *r = tb.vec[0], *rh = tb.vec[1], *p = tb.vec[2], *v = tb.vec[3], *d = tb.sol;
            double ai[1] = {0.0};
            for (int k = s.tid; k < N; k += s.nth) {
                const float bk = rhs32[k];
                r[k] = bk; rh[k] = bk; p[k] = 0.f; v[k] = 0.f; d[k] = 0.f;
                ai[0] += (double)bk * (double)bk;
            }
            if (!pg_sum<1>(s, ai)) return;
            if (threadIdx.x == 0) {
                sk.rr = ai[0];
                sk.r0 = sqrt(ai[0]);
                sk.tgt = fmax(sk.rtol * sk.r0, sk.atol * so.tgt);
                sk.rho = sk.al = sk.om = 1.0; sk.rbest = sk.r0; sk.stall = 0; sk.it = 0; sk.half = 0;
                sk.body_runs = 0;
                sk.maxit = so.maxit - so.it;
                sk.status = 0;
                sk.active = (sk.r0 > sk.tgt && sk.maxit > 0) ? 1 : 0;
            }
            __syncthreads();
            if (!pg_bicg<float>(s, a, tb, sv, nl, N, sk)) return;
            // x += d; r -= A d (FP64 operator); rhs32 = (float) r; the outer stop test
            double au[1] = {0.0};
            for (int k = s.tid; k < N; k += s.nth) {
                const Node nd = unidx(k, Nx, Ny);
                const double sum = a64_at<float>(tb.A64, tb.ap64, d, k, nd.i, nd.j, nd.l, Nx, Ny, Nz, nullptr);
                x[k] += (double)d[k];
                const double rk = r64[k] - sum;
                r64[k] = rk;
                rhs32[k] = (float)rk;
                au[0] += rk * rk;
            }
            if (!pg_sum<1>(s, au)) return;
            if (threadIdx.x == 0) {
                so.it += sk.it;
                so.body_runs++;
                so.rr = au[0];
                const double rn = sqrt(au[0]);
                if (rn <= so.tgt) { so.active = 0; so.status = 1; }
                else if (!(rn < 0.5 * so.rbest)) { so.active = 0; so.status = 4; }
                else if (so.it >= so.maxit) { so.active = 0; so.status = 3; }
                else so.rbest = rn;
            }
            __syncthreads();
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) s.g->steps = steps;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *PT<T>::ks(P) = sk;
        if (KIND == PK_REFINED) *P.ks = so;
        s.g->iters = KIND == PK_REFINED ? so.it : sk.it;
    }
}

// Test of the bounded barrier wait: the last block of the launch never arrives, so every
// other block must give up after wait_ns, set the error word and report ok = 0.
__global__ void k_pg_timeout_probe(PGrid *g, unsigned long long wait_ns, int *ok) {
    PS s;
    s.g = g;
    s.target = 0;
    s.rb = 0;
    s.tid = blockIdx.x * blockDim.x + threadIdx.x;
    s.nth = gridDim.x * blockDim.x;
    s.wait_ns = wait_ns;
    s.trace = nullptr;
    s.ntrace = 0;
    s.mode = 1;
    s.onecl = 0;
    if (blockIdx.x == gridDim.x - 1) return;     // never arrives
    const bool r = pg_sync(s);
    if (threadIdx.x == 0) ok[blockIdx.x] = r ? 1 : 0;
}

// ---------------------------------------------------------------- host side
namespace {
struct KInfo {
    const void *fn = nullptr;
    size_t smem = 0;       // dynamic shared memory the attribute allows
    int blocks = 0;        // co-resident blocks at that size
    int clusters = 0;      // co-resident clusters at that size (0: no cluster launch)
};
std::mutex g_pmu;
int g_persist_mode = -1;   // -1 unread, 0 off, 1 on
int g_persist_blocks = 0;  // blocks per launch (0: every SM's worth)
thread_local int t_persist_blocks = 0;  // this host thread's cap (0: none)
bool g_persist_broken = false;
bool g_coop_ok = false;    // the device supports cooperative launches
unsigned long long *g_trace = nullptr;   // armed barrier timeline (test hook): device buffer
int g_trace_n = 0, g_trace_used = 0;     // its barriers; 1 once a launch has filled it
int g_last_blocks = 0;                   // blocks of the last persistent launch
int g_fuse_up = 1;         // deferred prolongation on the way up (SEMISIM_B200_FUSEUP=0: off)
int g_barmode = 1;         // grid-barrier form (SEMISIM_B200_BARMODE; 1 measured faster than 0)
int g_clusters = 1;        // cluster launches: 0 off, 1 grids of one cluster, 2 every grid (SEMISIM_B200_CLUSTERS)
int g_csz = 8;             // CTAs per cluster (SEMISIM_B200_CSZ: 8 portable, 16 non-portable)
int g_clevel = 1;          // first level the first cluster runs alone (SEMISIM_B200_CLEVEL)
int g_coop = 1;            // cooperative launch attribute (SEMISIM_B200_COOP=0: plain launch of a
                           //   grid within the co-resident capacity)

template <class T, int KIND>
const void *kfn() { return reinterpret_cast<const void *>(&k_persist<T, KIND>); }

// co-resident clusters of g_csz CTAs of the kernel at `smem` bytes (0: no clusters)
int cluster_occupancy(const void *fn, size_t smem) {
    if (g_csz > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t q = {};
    q.gridDim = dim3(g_csz);
    q.blockDim = dim3(PG_TPB);
    q.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = g_csz; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
    q.attrs = at;
    q.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, fn, &q) != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}
// co-resident blocks of the kernel at `smem` bytes (0 when it cannot launch)
int occupancy(const void *fn, size_t smem) {
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per = 0, dev = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, PG_TPB, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return per * nsm;
}
}  // namespace

int persist_enabled() {
    std::lock_guard<std::mutex> lk(g_pmu);
    if (g_persist_mode < 0) {
        const char *e = std::getenv("SEMISIM_B200_PERSIST");
        g_persist_mode = (e && std::atoi(e) == 0) ? 0 : 1;
        if (const char *b = std::getenv("SEMISIM_B200_PBLOCKS")) g_persist_blocks = std::atoi(b);
        if (const char *f = std::getenv("SEMISIM_B200_FUSEUP")) g_fuse_up = std::atoi(f) != 0;
        if (const char *m = std::getenv("SEMISIM_B200_BARMODE")) g_barmode = std::atoi(m) ? 1 : 0;
        if (const char *m = std::getenv("SEMISIM_B200_CLUSTERS")) g_clusters = std::atoi(m) < 0 ? 0 : (std::atoi(m) > 2 ? 2 : std::atoi(m));
        if (const char *m = std::getenv("SEMISIM_B200_CLEVEL")) g_clevel = std::atoi(m) < 1 ? 1 : std::atoi(m);
        if (const char *m = std::getenv("SEMISIM_B200_CSZ")) g_csz = std::atoi(m) == 16 ? 16 : 8;
        if (const char *m = std::getenv("SEMISIM_B200_COOP")) g_coop = std::atoi(m) != 0;
        int dev = 0, coop = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) cudaGetLastError();
        if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess) cudaGetLastError();
        g_coop_ok = coop != 0;
    }
    return g_persist_mode == 1 && g_coop_ok && !g_persist_broken;
}
void persist_set(int mode, int blocks) {
    persist_enabled();
    std::lock_guard<std::mutex> lk(g_pmu);
    if (mode >= 0) g_persist_mode = mode ? 1 : 0;
    if (blocks >= 0) g_persist_blocks = blocks;
}
int persist_get_blocks() { return g_persist_blocks; }
int persist_thread_blocks(int n) {
    const int old = t_persist_blocks;
    if (n >= 0) t_persist_blocks = n;
    return old;
}

// Launch the persistent solve `kind` of precision T on instance 0 of the context.  Returns
// 1 when it ran (results in the Krylov records), 0 when the persistent path does not apply
// (the caller runs the per-pass path), -1 when a barrier wait ran out (the caller restores
// the start and runs the per-pass path; the persistent path is off from then on).
template <class T, int KIND>
static int persist_run(const Ctx &c, int Ls, size_t smem, const PArgs &a, PGrid *hres) {
    static KInfo info;                           // per instantiation, cached
    static std::mutex mu;
    KInfo ki;
    {
        std::lock_guard<std::mutex> lk(mu);
        KInfo &k = info;
        if (!k.fn || k.smem < smem) {
            k.fn = kfn<T, KIND>();
            k.smem = smem;
            k.blocks = occupancy(k.fn, smem);
            k.clusters = cluster_occupancy(k.fn, smem);
        }
        ki = k;
    }
    int nb = ki.blocks;
    // small systems take a part of the GPU (about two nodes per thread), so that several
    // instances' solves can run side by side
    const int want = (c.maxN + 2 * PG_TPB - 1) / (2 * PG_TPB);
    if (want < nb) nb = want < 4 ? 4 : want;
    if (g_persist_blocks > 0 && g_persist_blocks < nb) nb = g_persist_blocks;
    if (c.pblocks > 0 && c.pblocks < nb) nb = c.pblocks;
    if (t_persist_blocks > 0 && t_persist_blocks < nb) nb = t_persist_blocks;
    if (nb > PG_MAXB) nb = PG_MAXB;
    if (nb < 1) return 0;
    // clusters of g_csz CTAs: a grid of at most g_csz blocks becomes one cluster (every
    // barrier a cluster barrier, 0.3 us against 2 us for a grid barrier).  With g_clusters 2 a
    // larger grid is a whole number of clusters, the first of which runs the coarse levels
    // from Lc on alone; that costs the grid the SMs that no whole cluster covers (112 - 120
    // of 148 blocks), which a full-size solve loses more time to than the coarse levels gain,
    // so by default larger grids launch without clusters
    PArgs aa = a;
    aa.csz = 0;
    aa.onecl = 0;
    aa.Lc = a.Ls;
    if (g_clusters && ki.clusters > 0) {
        if (nb <= g_csz) {
            nb = g_csz;
            aa.csz = g_csz;
            aa.onecl = 1;
        } else if (g_clusters == 2) {
            int ncl = nb / g_csz;
            if (ncl > ki.clusters) ncl = ki.clusters;
            nb = ncl * g_csz;
            aa.csz = g_csz;
            aa.Lc = g_clevel < a.Ls ? g_clevel : a.Ls;
        }
    }
    (void)Ls;
    PGrid *g = c.h.pgrid;
    cudaMemsetAsync(g, 0, 6 * sizeof(unsigned), c.st);      // counter, error word, work counters
    const DevP *dp = c.dP;
    if (g_trace && !g_trace_used) {              // the armed timeline records this launch only
        aa.trace = g_trace;
        aa.ntrace = g_trace_n;
        g_trace_used = 1;
    }
    void *args[] = {(void *)&dp, (void *)&aa};
    g_launches++;
    t_launches++;
    const int pid = sizeof(T) == 4 ? PF_PERSIST32 : PF_PERSIST;
    if (g_prof_on) prof_begin(pid, c.st);
    g_last_blocks = nb;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nb);
    cfg.blockDim = dim3(PG_TPB);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c.st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = g_coop;
    at[1].id = cudaLaunchAttributeClusterDimension;
    at[1].val.clusterDim.x = aa.csz; at[1].val.clusterDim.y = 1; at[1].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = aa.csz ? 2 : 1;
    cudaError_t e = cudaLaunchKernelExC(&cfg, kfn<T, KIND>(), args);
    if (e != cudaSuccess && aa.csz) {            // no cluster launch here: plain cooperative grid
        cudaGetLastError();
        std::fprintf(stderr, "semisim-b200: cluster launch of the persistent solve refused (%s); without clusters "
                             "from now on\n", cudaGetErrorString(e));
        g_clusters = 0;
        aa.csz = 0;
        aa.onecl = 0;
        aa.Lc = aa.Ls;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelExC(&cfg, kfn<T, KIND>(), args);
    }
    if (g_prof_on) prof_end(pid, c.st, 0.0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        std::fprintf(stderr, "semisim-b200: persistent solve launch failed (%s); per-pass solves from now on\n",
                     cudaGetErrorString(e));
        g_persist_broken = true;
        return 0;
    }
    cudaMemcpyAsync(hres, g, 6 * sizeof(unsigned), cudaMemcpyDeviceToHost, c.st);
    cudaStreamSynchronize(c.st);
    if (hres->err) {
        std::fprintf(stderr, "semisim-b200: persistent solve abandoned (a barrier wait ran out); per-pass solves "
                             "from now on\n");
        g_persist_broken = true;
        return -1;
    }
    return 1;
}

// algorithmic bytes of one V-cycle of precision T (the passes the persistent kernel runs)
template <class T>
static double vcycle_bytes(const MGHost &mg, int Ls, int deep, int sweeps2) {
    const double w = sizeof(T) / 8.0;
    double b = 0.0;
    for (int L = 0; L < Ls; L++) {
        const double n = mg.maxN[L];
        const int sm = (L < deep && sweeps2) ? 2 : 1;
        // smoother half sweeps (black, red) per application, pre and post; residual +
        // restriction; prolongation and residual on the way up
        b += n * w * (2.0 * sm * (kProfBytesPerNode[PF_SMOOTH_B] + kProfBytesPerNode[PF_SMOOTH_R]) +
                      kProfBytesPerNode[PF_RESID_RESTRICT] + kProfBytesPerNode[PF_PROLONG] +
                      kProfBytesPerNode[PF_LEVEL_RESID]);
    }
    b += 2.0 * mg.maxN[Ls] * sizeof(T);             // b in, x out of the shared-memory levels
    return b;
}

// algorithmic bytes of the in-kernel hierarchy set-up of precision T
template <class T>
static double setup_bytes(const MGHost &mg) {
    const double w = sizeof(T) / 8.0;
    double b = sizeof(T) == 4 ? mg.maxN[0] * kProfBytesPerNode[PF_CONVERT32] : 0.0;
    for (int L = 0; L < mg.maxlev - 1; L++)
        b += mg.maxN[L] * w * (kProfBytesPerNode[PF_WEIGHTS] + kProfBytesPerNode[PF_GALERKIN] +
                               kProfBytesPerNode[PF_ILU_DIAG]);
    return b;
}

// small-level plan of precision T for the persistent kernels: the first level at or below
// the small-level size whose data fits the opt-in shared memory (never level 0)
template <class T>
static int persist_plan(const Ctx &c, const MGHost &mg, size_t *smem) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t cap = optin > 16384 ? (size_t)optin - 16384 : 0;
    *smem = 0;
    if (mg.maxlev < 2) return -1;
    vcycle_knobs_init();
    const int lim = c.small_nodes > 0 ? c.small_nodes : g_small_nodes;
    int L = 1;
    while (L < mg.maxlev - 1 && mg.maxN[L] > lim) L++;
    auto bytes = [&](int Ls) {
        size_t b = 0;
        for (int q = Ls; q < mg.maxlev; q++) b += smem_level_bytes<T>(mg.maxN[q], q == mg.maxlev - 1);
        return b;
    };
    while (L < mg.maxlev - 1 && bytes(L) > cap) L++;
    if (bytes(L) > cap) return -1;
    *smem = bytes(L);
    return L;
}

// Persistent forms of the solves of kernels_la.cu.  Each returns 1 (done: the Krylov
// records hold the result), 0 (not applicable: nothing was changed) or -1 (abandoned: the
// caller restores the start and uses the per-pass solve).
int persist_pcg(const Ctx &c, const MGHost &mg, int mixed) {
    if (c.ninst != 1 || !persist_enabled()) return 0;
    size_t smem = 0;
    PArgs a{};
    a.Ls = mixed ? persist_plan<float>(c, mg, &smem) : persist_plan<double>(c, mg, &smem);
    if (a.Ls < 1) return 0;
    a.setup = 1;
    a.qsign = 0;
    smem = std::max(smem, PG_SETUP_SMEM);
    a.deep = g_deep_levels;
    a.sweeps2 = g_l0_sweeps > 1;
    a.alpha = mg.alpha;
    a.fuse_up = g_fuse_up;
    a.barmode = g_barmode;
    PGrid h{};
    const int rc = mixed ? persist_run<float, PK_PCG>(c, a.Ls, smem, a, &h)
                         : persist_run<double, PK_PCG>(c, a.Ls, smem, a, &h);
    if (rc == 1 && g_prof_on) {
        const double vb = mixed ? vcycle_bytes<float>(mg, a.Ls, a.deep, a.sweeps2)
                                : vcycle_bytes<double>(mg, a.Ls, a.deep, a.sweeps2);
        const double kb = (mixed ? 0.5 : 1.0) * (kProfBytesPerNode[PF_KRY_SPMV_DOT] + 2 * kProfBytesPerNode[PF_KRY_UPDATE] +
                                                 kProfBytesPerNode[PF_KRY_DOT]);
        const double sb = mixed ? setup_bytes<float>(mg) : setup_bytes<double>(mg);
        prof_set_last(mixed ? PF_PERSIST32 : PF_PERSIST, sb + h.vcycles * vb + h.iters * kb * c.maxN);
    }
    return rc;
}
int persist_bicg(const Ctx &c, const MGHost &mg, double rtol, double atol, int qsign) {
    if (c.ninst != 1 || !persist_enabled()) return 0;
    size_t smem = 0;
    PArgs a{};
    a.Ls = persist_plan<double>(c, mg, &smem);
    if (a.Ls < 1) return 0;
    a.setup = 1;
    a.qsign = qsign;
    smem = std::max(smem, PG_SETUP_SMEM);
    a.deep = g_deep_levels;
    a.sweeps2 = g_l0_sweeps > 1;
    a.alpha = mg.alpha;
    a.fuse_up = g_fuse_up;
    a.barmode = g_barmode;
    a.rtol = rtol;
    a.atol = atol;
    PGrid h{};
    const int rc = persist_run<double, PK_BICG>(c, a.Ls, smem, a, &h);
    if (rc == 1 && g_prof_on) {
        const double vb = vcycle_bytes<double>(mg, a.Ls, a.deep, a.sweeps2);
        const double kb = 2 * kProfBytesPerNode[PF_KRY_SPMV_DOT] + 4 * kProfBytesPerNode[PF_KRY_UPDATE];
        prof_set_last(PF_PERSIST, setup_bytes<double>(mg) + h.vcycles * vb +
                                      (h.iters * kb + kProfBytesPerNode[PF_KRY_INIT]) * c.maxN);
    }
    return rc;
}
int persist_refined(const Ctx &c, const MGHost &mg, int maxsteps, int *steps, int qsign) {
    if (c.ninst != 1 || !persist_enabled()) return 0;
    size_t smem = 0;
    PArgs a{};
    a.Ls = persist_plan<float>(c, mg, &smem);
    if (a.Ls < 1) return 0;
    a.setup = 1;
    a.qsign = qsign;
    smem = std::max(smem, PG_SETUP_SMEM);
    a.deep = g_deep_levels;
    a.sweeps2 = g_l0_sweeps > 1;
    a.alpha = mg.alpha;
    a.fuse_up = g_fuse_up;
    a.barmode = g_barmode;
    a.maxsteps = maxsteps;
    PGrid h{};
    const int rc = persist_run<float, PK_REFINED>(c, a.Ls, smem, a, &h);
    if (rc == 1) {
        *steps = h.steps;
        if (g_prof_on) {
            const double vb = vcycle_bytes<float>(mg, a.Ls, a.deep, a.sweeps2);
            const double kb = 0.5 * (2 * kProfBytesPerNode[PF_KRY_SPMV_DOT] + 4 * kProfBytesPerNode[PF_KRY_UPDATE]);
            prof_set_last(PF_PERSIST32, setup_bytes<float>(mg) + h.vcycles * vb +
                                            (h.iters * kb + (h.steps + 1) * kProfBytesPerNode[PF_REFINE]) * c.maxN);
        }
    }
    return rc;
}

// Barrier timeline of the next persistent launch (test and measurement hook): n > 0 arms a
// timeline of n barriers; n == 0 copies the recorded one to out (3 n values: first arrival,
// last arrival, release seen by block 0, globaltimer ns; unused barriers keep ~0, 0, 0),
// disarms it and returns the blocks of that launch.
int persist_trace(int n, unsigned long long *out, int *blocks) {
    static int nmax = 0;
    if (n > 0) {
        if (g_trace) cudaFree(g_trace);
        g_trace = nullptr;
        if (cudaMalloc(&g_trace, sizeof(unsigned long long) * 3 * n) != cudaSuccess) { cudaGetLastError(); return -1; }
        std::vector<unsigned long long> init(3 * (size_t)n, 0ull);
        for (int q = 0; q < n; q++) init[3 * q] = ~0ull;
        cudaMemcpy(g_trace, init.data(), init.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice);
        g_trace_n = nmax = n;
        g_trace_used = 0;
        return 0;
    }
    if (!g_trace) return -1;
    cudaDeviceSynchronize();
    if (out) cudaMemcpy(out, g_trace, sizeof(unsigned long long) * 3 * nmax, cudaMemcpyDeviceToHost);
    cudaFree(g_trace);
    g_trace = nullptr;
    g_trace_n = 0;
    if (blocks) *blocks = g_last_blocks;
    return g_trace_used;
}

// Run the bounded-wait test on the instance's barrier record with `nb` blocks (>= 2):
// returns the error word (1 expected) and the blocks that reported ok = 0 in *gave_up
// (nb - 1 expected), or -1 when the launch failed.
int persist_timeout_probe(const Ctx &c, int nb, double wait_s, int *gave_up) {
    if (nb < 2 || nb > 64) return -1;
    int *ok = nullptr;
    if (cudaMalloc(&ok, nb * sizeof(int)) != cudaSuccess) { cudaGetLastError(); return -1; }
    cudaMemsetAsync(ok, 0xff, nb * sizeof(int), c.st);
    PGrid *g = c.h.pgrid;
    cudaMemsetAsync(g, 0, 6 * sizeof(unsigned), c.st);
    unsigned long long wn = (unsigned long long)(wait_s * 1e9);
    void *args[] = {(void *)&g, (void *)&wn, (void *)&ok};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_pg_timeout_probe, dim3(nb), dim3(32), args, 0, c.st);
    int rc = -1;
    if (e == cudaSuccess) {
        unsigned err = 0;
        std::vector<int> h(nb);
        cudaMemcpyAsync(&err, &g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, c.st);
        cudaMemcpyAsync(h.data(), ok, nb * sizeof(int), cudaMemcpyDeviceToHost, c.st);
        if (cudaStreamSynchronize(c.st) == cudaSuccess) {
            int n0 = 0;
            for (int q = 0; q < nb - 1; q++) n0 += h[q] == 0;
            *gave_up = n0;
            rc = (int)err;
        }
    } else {
        cudaGetLastError();
    }
    cudaFree(ok);
    return rc;
}

}  // namespace ss
