// Linear algebra of the solve path on 7-point stencils: level-0 SpMV fused with the
// Krylov dot products, the geometric 2x2x2 aggregation multigrid (Slotboom-weighted
// prolongation, Petrov-Galerkin coarse operators, red-black D-ILU smoother, dense
// coarsest level) and device-resident PCG / BiCGSTAB.
//
// Every multigrid and Krylov kernel is a template over the element type T of the
// vectors and matrices it streams.  T = double is the plain path (the reference's FP64
// arithmetic).  T = float is the inner solver of the refined path: an FP32 copy of the
// level-0 system, an FP32 hierarchy and FP32 Krylov vectors (dot products accumulated in
// FP64), driven by FP64 iterative refinement (FP64 residual b - A x with the FP64
// operator, FP32 correction) to the reference's own FP64 stop rule.
//
// The reference smooths with a chunked natural-order D-ILU(0) (semiconductor_3d.c:
// 1923-1972), a sequential recurrence.  Here the smoother is D-ILU(0) in red-black
// order: red nodes (i+j+l even) have only black neighbours, so the forward sweep is a
// pointwise divide on red and one stencil pass on black, the backward sweep one pass on
// red.  It changes Krylov iteration counts, not the converged solution.
//
// Krylov scalars stay on the device (KrylovS): each reducing kernel's last block
// computes the next coefficients and the stop test.  Every kernel of an iteration first
// reads the instance's `active` word, so the host can queue several iterations and
// read the status once.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include <cooperative_groups.h>

#include "device_common.cuh"
#include "prof.h"
#include "kernels.h"
#include "solver_ctx.h"
#include "la_common.cuh"

namespace cg = cooperative_groups;

namespace ss {

static inline dim3 grid_nodes(const Ctx &c) { return dim3(c.nodes_blocks(), c.ninst); }
static inline dim3 grid_n(const Ctx &c, int n) {
    int b = (n + TPB - 1) / TPB;
    if (b > c.grid_cap) b = c.grid_cap;
    if (b < 1) b = 1;
    return dim3(b, c.ninst);
}

template <class T>
__global__ void k_ilu_diag(const DevP *__restrict__ Ps, int L) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    if (L > 0 && L >= P.nlev - 1) return;
    const LevView<T> v = levview<T>(P, L, 0, 0);
    SS_GRID_LOOP(k, v.N) ilu_diag_node<T>(v, k);
}

// Row-blocked launch shape of the level passes: block (32, rpb), threadIdx.x along x (the
// x index, or the half-row index of a colour), threadIdx.y + rpb blockIdx.z the grid row
// j + Ny l, so no thread divides its linear index (rpb: Ctx, set by the autotuner).
#define SS_ROW_LOOP(row, rows) \
    for (int row = blockIdx.z * blockDim.y + threadIdx.y; row < (rows); row += gridDim.z * blockDim.y)

// x += alpha pw P xc (semiconductor_3d.c:2038-2048); the residual that follows needs
// every prolonged neighbour and is a separate pass
template <class T>
__global__ void __launch_bounds__(1024) k_prolong(const DevP *__restrict__ Ps, int L, int bsel, int xsel, double alpha,
                                                 int gate) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const LevView<T> f = levview<T>(P, L, bsel, xsel);
    const LevelT<T> cl = PT<T>::lev(P, L + 1 < MAXLEV ? L + 1 : L);
    const int nl = P.nlev;
    pdl_wait();
    if (L >= nl - 1 || gated_off<T>(P, gate)) return;
    const T al = (T)alpha;
    const int i = blockIdx.x * 32 + threadIdx.x;
    if (i >= f.Nx) return;
    const int I = f.cx ? i >> 1 : i;
    SS_ROW_LOOP(row, f.Ny * f.Nz) {
        const int l = row / f.Ny, j = row - l * f.Ny;
        const int J = f.cy ? j >> 1 : j, K = f.cz ? l >> 1 : l;
        const int k = i + f.Nx * row;
        f.x[k] += al * f.pw[k] * cl.x[I + cl.Nx * (J + cl.Ny * K)];
    }
}
template <class T>
__global__ void __launch_bounds__(1024) k_level_resid(const DevP *__restrict__ Ps, int L, int bsel, int xsel, int gate) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const LevView<T> f = levview<T>(P, L, bsel, xsel);
    const int nl = P.nlev;
    pdl_wait();
    if (L >= nl - 1 || gated_off<T>(P, gate)) return;
    const int i = blockIdx.x * 32 + threadIdx.x;
    if (i >= f.Nx) return;
    SS_ROW_LOOP(row, f.Ny * f.Nz) {
        const int l = row / f.Ny, j = row - l * f.Ny;
        const int k = i + f.Nx * row;
        f.r[k] = f.b[k] - lv_apply<T>(f, f.x, k, i, j, l);
    }
}

template <class T>
__global__ void k_coarse_setup(const DevP *__restrict__ Ps, int L) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    if (L != P.nlev - 1 || L == 0) return;
    __shared__ double M[COARSE_MAX * (COARSE_MAX + 1)];
    __shared__ int perm[COARSE_MAX];
    __shared__ int piv;
    blk_coarse_setup<T>(PT<T>::lev(P, L), M, perm, &piv);
}

template <class T>
__global__ void k_mg_weights(const DevP *__restrict__ Ps, int L, int qsign) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    if (L >= P.nlev - 1) return;
    const LevView<T> f = levview<T>(P, L, 0, 0);
    const LevelT<T> &cl = PT<T>::lev(P, L + 1);
    SS_GRID_LOOP(K, cl.N) mg_weights_node<T>(P, f, cl, L, qsign, K);
}

template <class T>
__global__ void k_galerkin(const DevP *__restrict__ Ps, int L, int wsel) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    if (L >= P.nlev - 1) return;
    const LevView<T> f = levview<T>(P, L, 0, 0);
    const LevelT<T> &cl = PT<T>::lev(P, L + 1);
    const T *w = (L == 0 && wsel) ? PT<T>::w0(P) : nullptr;
    SS_GRID_LOOP(K, cl.N) galerkin_node<T>(f, cl, w, K);
}

// FP32 copy of the level-0 operator and its row weights (start of a refined solve)
__global__ void k_to32(const DevP *__restrict__ Ps, int wsel) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
#pragma unroll
        for (int q = 0; q < 7; q++) P.A32[q][k] = (float)P.A[q][k];
        if (wsel) P.dsc32[k] = (float)P.dsc[k];
    }
}

// ------------------------------------------------------------------ vector kernels (FP64)
__global__ void k_absmax(const DevP *__restrict__ Ps, int xsel, int slot) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    const double *x = vsel<double>(P, xsel);
    double m = 0.0;
    SS_GRID_LOOP(k, P.N) {
        const double a = fabs(x[k]);
        m = (a > m || a != a) ? a : m;
    }
    if (grid_max(m, P.part, P.ticket + 3)) P.res[slot] = m;
}
// y = x + a z  (selectors)
__global__ void k_axpy(const DevP *__restrict__ Ps, int ysel, int xsel, double a, int zsel) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    double *y = vsel<double>(P, ysel);
    const double *x = vsel<double>(P, xsel), *z = vsel<double>(P, zsel);
    SS_GRID_LOOP(k, P.N) y[k] = x[k] + a * z[k];
}
__global__ void k_fill(const DevP *__restrict__ Ps, int ysel, double v) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    double *y = vsel<double>(P, ysel);
    SS_GRID_LOOP(k, P.N) y[k] = v;
}
__global__ void k_copy(const DevP *__restrict__ Ps, int ysel, int xsel) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    double *y = vsel<double>(P, ysel);
    const double *x = vsel<double>(P, xsel);
    SS_GRID_LOOP(k, P.N) y[k] = x[k];
}

void launch_absmax_sel(const Ctx &c, int xsel, int slot) { SS_LAUNCH_PDL(PF_VEC, c.maxN, k_absmax, grid_nodes(c), TPB, c.st, c.dP, xsel, slot); }
void launch_axpy_sel(const Ctx &c, int ysel, int xsel, double a, int zsel) {
    SS_LAUNCH_PDL(PF_VEC, c.maxN, k_axpy, grid_nodes(c), TPB, c.st, c.dP, ysel, xsel, a, zsel);
}
void launch_fill_sel(const Ctx &c, int ysel, double v) { SS_LAUNCH_PDL(PF_VEC, c.maxN, k_fill, grid_nodes(c), TPB, c.st, c.dP, ysel, v); }
void launch_copy_sel(const Ctx &c, int ysel, int xsel) { SS_LAUNCH_PDL(PF_VEC, c.maxN, k_copy, grid_nodes(c), TPB, c.st, c.dP, ysel, xsel); }

// ------------------------------------------------------------------ multigrid set-up
// hierarchy of the system now in A: Slotboom weights, Galerkin products, smoother
// pivots, coarsest inverse.  T = float first copies the level-0 operator to FP32.
template <class T>
static void mg_setup_t(const Ctx &c, const MGHost &mg, int qsign) {
    if (std::is_same<T, float>::value)
        SS_LAUNCH_PDL(PF_CONVERT32, c.maxN, k_to32, grid_nodes(c), TPB, c.st, c.dP, qsign != 0);
    for (int L = 0; L < mg.maxlev - 1; L++) {
        const int nc = mg.maxN[L + 1];
        SS_LAUNCH_PDL(pf<T>(PF_WEIGHTS), mg.maxN[L], k_mg_weights<T>, grid_n(c, nc), TPB, c.st, c.dP, L, qsign);
        SS_LAUNCH_PDL(pf<T>(PF_GALERKIN), mg.maxN[L], k_galerkin<T>, grid_n(c, nc), TPB, c.st, c.dP, L, qsign != 0);
        SS_LAUNCH_PDL(pf<T>(PF_ILU_DIAG), mg.maxN[L], k_ilu_diag<T>, grid_n(c, mg.maxN[L]), TPB, c.st, c.dP, L);
    }
    for (int L = 1; L < mg.maxlev; L++)
        SS_LAUNCH_PDL(pf<T>(PF_COARSE_SETUP), COARSE_MAX, k_coarse_setup<T>, dim3(1, c.ninst), TPB, c.st, c.dP, L);
}
void mg_setup(const Ctx &c, const MGHost &mg, int qsign) { mg_setup_t<double>(c, mg, qsign); }

// ------------------------------------------------------------------ V-cycle
// one V(1,1) cycle x = M^-1 b on the level-0 vectors (bsel -> xsel); mg_on = 0 applies
// the level-0 smoother alone (the reference's ILU-only fallback).
// ---- fine levels: one kernel per pass, all SMs
// Half sweep over the nodes of one colour: thread ti of row (j, l) takes
// i = 2 ti + ((j + l + colour) & 1), so every lane does work.
template <class T, int MODE, int COLOR>
__global__ void __launch_bounds__(1024) k_smooth_cm(const DevP *__restrict__ Ps, int L, int bsel, int xsel, int gate) {
    constexpr int mode = MODE, color = COLOR;
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const LevView<T> v = levview<T>(P, L, bsel, xsel);
    const int nl = P.nlev;
    pdl_wait();
    if ((L > 0 && L >= nl - 1) || gated_off<T>(P, gate)) return;
    const int ti = blockIdx.x * 32 + threadIdx.x;
    if (2 * ti >= v.Nx) return;
    SS_ROW_LOOP(row, v.Ny * v.Nz) {
        const int l = row / v.Ny, j = row - l * v.Ny;
        const int i = 2 * ti + ((j + l + color) & 1);
        if (i >= v.Nx) continue;
        smooth_node<T>(v, i + v.Nx * row, i, j, l, mode, color);
    }
}
// the half sweep of (mode, colour), one kernel instance per pair
template <class T>
using SmoothFn = void (*)(const DevP *, int, int, int, int);
template <class T>
static SmoothFn<T> smooth_fn(int mode, int color) {
    static const SmoothFn<T> tab[3][2] = {{k_smooth_cm<T, 0, 0>, k_smooth_cm<T, 0, 1>},
                                          {k_smooth_cm<T, 1, 0>, k_smooth_cm<T, 1, 1>},
                                          {k_smooth_cm<T, 2, 0>, k_smooth_cm<T, 2, 1>}};
    return tab[mode][color];
}

// Weighted residual of every fine node summed into its 2x2x2 aggregate.  Block (32, 4 Q):
// threadIdx.x runs along fine x, threadIdx.y picks one of Q coarse rows and the (j, l)
// parity inside it; pairs along x meet through a shuffle, the four parities through
// shared memory; the blocks loop over the coarse rows.  One thread per fine node (the restriction of semiconductor_3d.c:
// 2028-2037 applied to the residual of 1984-1991).
template <class T>
__global__ void __launch_bounds__(1024) k_resid_restrict2(const DevP *__restrict__ Ps, int L, int bsel, int xsel,
                                                          int wsel, int gate) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const LevView<T> f = levview<T>(P, L, bsel, xsel);
    const LevelT<T> cl = PT<T>::lev(P, L + 1 < MAXLEV ? L + 1 : L);
    const T *w = (L == 0 && wsel) ? PT<T>::w0(P) : nullptr;
    const int nl = P.nlev;
    pdl_wait();
    if (L >= nl - 1 || gated_off<T>(P, gate)) return;
    // block (32, 4 Q): Q coarse rows per pass, threadIdx.y = 4 q + (j, l) parity
    const int Q = blockDim.y >> 2, q = threadIdx.y >> 2, par = threadIdx.y & 3;
    const int dj = par & 1, dl = par >> 1;
    const int rows = cl.Ny * cl.Nz;
    const int i = blockIdx.x * 32 + threadIdx.x;
    __shared__ T sh[32][32];
    for (int R0 = blockIdx.z * Q; R0 < rows; R0 += gridDim.z * Q) {
        const int R = R0 + q;                         // coarse row J + Cy*Lc
        const bool rowok = R < rows;
        const int Lc = rowok ? R / cl.Ny : 0, Jc = rowok ? R - Lc * cl.Ny : 0;
        const int j = f.cy ? 2 * Jc + dj : Jc, l = f.cz ? 2 * Lc + dl : Lc;
        const bool ok = rowok && i < f.Nx && j < f.Ny && l < f.Nz && (f.cy || dj == 0) && (f.cz || dl == 0);
        T val = 0;
        if (ok) {
            const int k = i + f.Nx * (j + f.Ny * l);
            const T r = f.b[k] - lv_apply<T>(f, f.x, k, i, j, l);
            val = w ? w[k] * r : r;
        }
        sh[threadIdx.y][threadIdx.x] = val;
        __syncthreads();
        if (par == 0) {
            T s = sh[4 * q][threadIdx.x] + sh[4 * q + 1][threadIdx.x] + sh[4 * q + 2][threadIdx.x] +
                  sh[4 * q + 3][threadIdx.x];
            if (f.cx) {
                s += __shfl_down_sync(0xffffffffu, s, 1);
                if (rowok && !(threadIdx.x & 1) && i < f.Nx) cl.b[(i >> 1) + cl.Nx * R] = s;
            } else if (rowok && i < f.Nx) {
                cl.b[i + cl.Nx * R] = s;
            }
        }
        __syncthreads();
    }
}

// ---- small levels: the rest of the V-cycle in one thread-block cluster per instance
// The CTAs of a cluster split every pass (cluster-stride loops); a hardware cluster
// barrier (release / acquire at cluster scope) separates the passes, so each pass sees
// the global writes of the one before.  One launch replaces ~7 launches per level.
__device__ __forceinline__ int cl_first() {
    return (int)cg::this_cluster().block_rank() * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ int cl_stride() { return (int)cg::this_cluster().num_blocks() * blockDim.x; }
__device__ __forceinline__ void cl_sync() { cg::this_cluster().sync(); }

template <class T>
__device__ __forceinline__ void cta_smooth(const LevView<T> &v, int color, int mode) {
    const int hx = (v.Nx + 1) >> 1, rows = v.Ny * v.Nz;
    for (int t = cl_first(); t < hx * rows; t += cl_stride()) {
        const int row = t / hx, ti = t - row * hx;
        const int l = row / v.Ny, j = row - l * v.Ny;
        const int i = 2 * ti + ((j + l + color) & 1);
        if (i >= v.Nx) continue;
        smooth_node<T>(v, i + v.Nx * row, i, j, l, mode, color);
    }
    cl_sync();
}
template <class T>
__device__ __forceinline__ void cta_resid_restrict(const LevView<T> &f, const LevelT<T> &cl, const T *w) {
    for (int K = cl_first(); K < cl.N; K += cl_stride()) {
        const Node c = unidx(K, cl.Nx, cl.Ny);
        const Agg g = agg_range(f, c.i, c.j, c.l);
        T s = 0;
        for (int l = g.l0; l <= g.l1; l++)
            for (int j = g.j0; j <= g.j1; j++)
                for (int i = g.i0; i <= g.i1; i++) {
                    const int k = i + f.Nx * (j + f.Ny * l);
                    const T r = f.b[k] - lv_apply<T>(f, f.x, k, i, j, l);
                    s += w ? w[k] * r : r;
                }
        cl.b[K] = s;
    }
    cl_sync();
}
template <class T>
__device__ __forceinline__ void cta_prolong(const LevView<T> &f, const LevelT<T> &cl, T alpha) {
    for (int k = cl_first(); k < f.N; k += cl_stride()) {
        const Node a = unidx(k, f.Nx, f.Ny);
        const int I = f.cx ? a.i >> 1 : a.i, J = f.cy ? a.j >> 1 : a.j, K = f.cz ? a.l >> 1 : a.l;
        f.x[k] += alpha * f.pw[k] * cl.x[I + cl.Nx * (J + cl.Ny * K)];
    }
    cl_sync();
}
template <class T>
__device__ __forceinline__ void cta_resid(const LevView<T> &f) {
    for (int k = cl_first(); k < f.N; k += cl_stride()) {
        const Node a = unidx(k, f.Nx, f.Ny);
        f.r[k] = f.b[k] - lv_apply<T>(f, f.x, k, a.i, a.j, a.l);
    }
    cl_sync();
}
template <class T>
__device__ __forceinline__ void cta_dense(const LevelT<T> &v) {
    const int n = v.N;
    for (int r = cl_first(); r < n; r += cl_stride()) {
        T s = 0;
        for (int q = 0; q < n; q++) s += v.D[r * n + q] * v.b[q];
        v.x[r] = s;
    }
    cl_sync();
}

constexpr int SMALL_TPB = 1024;
template <class T>
__global__ void __launch_bounds__(SMALL_TPB) k_vcycle_small(const DevP *__restrict__ Ps, int Ls, int bsel, int xsel,
                                                            int wsel, double alpha, int gate) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    if (gated_off<T>(P, gate)) return;
    const int nl = P.nlev;
    if (nl == 1) {                                 // a single level: the smoother alone
        const LevView<T> v = levview<T>(P, 0, bsel, xsel);
        cta_smooth<T>(v, 1, 0);
        cta_smooth<T>(v, 0, 0);
        return;
    }
    for (int L = Ls; L < nl - 1; L++) {
        const LevView<T> v = levview<T>(P, L, bsel, xsel);
        cta_smooth<T>(v, 1, 0);
        cta_smooth<T>(v, 0, 0);
        cta_resid_restrict<T>(v, PT<T>::lev(P, L + 1), (L == 0 && wsel) ? PT<T>::w0(P) : nullptr);
    }
    cta_dense<T>(PT<T>::lev(P, nl - 1));
    for (int L = nl - 2; L >= Ls; L--) {
        const LevView<T> v = levview<T>(P, L, bsel, xsel);
        cta_prolong<T>(v, PT<T>::lev(P, L + 1), (T)alpha);
        cta_resid<T>(v);
        cta_smooth<T>(v, 1, 1);
        cta_smooth<T>(v, 0, 1);
    }
}

template <class T>
__global__ void __launch_bounds__(SMALL_TPB) k_vcycle_smem(const DevP *__restrict__ Ps, int Ls, double alpha,
                                                           int gate) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    extern __shared__ __align__(16) unsigned char sraw[];
    __shared__ LevView<T> sv[MAXLEV];             // the levels' views into shared memory
    const int nl = P.nlev;
    if (threadIdx.x < nl - Ls) sv[threadIdx.x] = smem_view<T>(P, Ls + threadIdx.x, Ls, sraw);
    pdl_wait();
    if (gated_off<T>(P, gate)) return;
    __syncthreads();
    blk_stage_small<T>(P, sv, Ls, nl);            // couplings, pivots, weights, coarsest inverse
    blk_copy<T>(sv[0].b, PT<T>::lev(P, Ls).b, sv[0].N);
    __syncthreads();
    blk_vcycle_small<T>(sv, Ls, nl, (T)alpha);
    blk_copy<T>(PT<T>::lev(P, Ls).x, sv[0].x, sv[0].N);
}

int g_small_nodes = 2048;           // levels at or below this size run in the cluster kernel
int g_l0_sweeps = 2;                // red-black applications per smoothing step on the finest level
int g_deep_levels = 1;              // levels (from the finest) that get the second application
static int g_cluster = 0;           // CTAs per cluster of the small-level kernel (set on first use)
static size_t g_smem_max = 0;       // dynamic shared memory of the shared-memory small-level kernel (0: off)

template <class T>
static bool cluster16_ok() {
    if (cudaFuncSetAttribute(k_vcycle_small<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t q = {};
    q.gridDim = dim3(16, 1);
    q.blockDim = dim3(SMALL_TPB);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 16; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
    q.attrs = at;
    q.numAttrs = 1;
    int ncl = 0;
    const bool ok = cudaOccupancyMaxActiveClusters(&ncl, k_vcycle_small<T>, &q) == cudaSuccess && ncl >= 1;
    cudaGetLastError();
    return ok;
}

// cluster size of the small-level kernel (16 CTAs when the device allows non-portable
// clusters of 16, else 8) and the size split, read once (SEMISIM_B200_CLUSTER / _SMALL)
static void small_init() {
    if (!g_cluster) {
        const char *e = std::getenv("SEMISIM_B200_CLUSTER");
        int cl = (e && std::atoi(e) == 8) ? 8 : 16;
        if (const char *s = std::getenv("SEMISIM_B200_SMALL")) g_small_nodes = std::atoi(s);
        if (const char *s = std::getenv("SEMISIM_B200_L0SWEEPS")) g_l0_sweeps = std::atoi(s) > 1 ? 2 : 1;
        if (const char *s = std::getenv("SEMISIM_B200_DEEP")) g_deep_levels = std::atoi(s) < 1 ? 1 : std::atoi(s);
        const bool ok64 = cluster16_ok<double>(), ok32 = cluster16_ok<float>();
        if (!ok64 || !ok32) cl = 8;
        g_cluster = cl;
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        g_smem_max = optin > 8192 ? (size_t)optin - 8192 : 0;     // room for the static shared arrays
        const char *sm = std::getenv("SEMISIM_B200_SMEM");
        if (sm && std::atoi(sm) == 0) g_smem_max = 0;
        if (g_smem_max &&
            (cudaFuncSetAttribute(k_vcycle_smem<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g_smem_max) !=
                 cudaSuccess ||
             cudaFuncSetAttribute(k_vcycle_smem<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g_smem_max) !=
                 cudaSuccess))
            g_smem_max = 0;
        cudaGetLastError();
    }
}

// the multigrid knobs read from the environment (small-level size, finest-level sweeps)
void vcycle_knobs_init() { small_init(); }

// launch the small-level V-cycle as clusters of g_cluster CTAs, one cluster per instance
template <class T>
static void launch_small(const Ctx &c, int nodes, int Ls, int bsel, int xsel, int wsel, double alpha, int gate) {
    small_init();
    g_launches++;
    t_launches++;
    if (g_prof_on) prof_begin(pf<T>(PF_COARSE), c.st);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g_cluster, c.ninst);
    cfg.blockDim = dim3(SMALL_TPB);
    cfg.stream = c.st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = g_cluster; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = g_pdl ? 2 : 1;
    cudaLaunchKernelEx(&cfg, k_vcycle_small<T>, c.dP, Ls, bsel, xsel, wsel, alpha, gate);
    if (g_prof_on) prof_end(pf<T>(PF_COARSE), c.st, nodes);
}

// row-blocked grids (block (32, c.rpb)): x extent `nx`, all rows of level L
static inline dim3 grid_rows(const Ctx &c, int L, const MGHost &mg, int nx) {
    int gz = (mg.maxRows[L] + c.rpb - 1) / c.rpb;
    if (gz > c.zcap) gz = c.zcap;
    if (gz > 65535) gz = 65535;
    return dim3((nx + 31) / 32, c.ninst, gz > 0 ? gz : 1);
}
static inline dim3 grid_half(const Ctx &c, int L, const MGHost &mg) { return grid_rows(c, L, mg, (mg.maxNx[L] + 1) / 2); }
static inline dim3 grid_full(const Ctx &c, int L, const MGHost &mg) { return grid_rows(c, L, mg, mg.maxNx[L]); }
// residual + restriction from level L: block (32, 4 rq), grid over the coarse rows
static inline dim3 block_rr(const Ctx &c) { return dim3(32, 4 * c.rq); }
static inline dim3 grid_rr(const Ctx &c, int L, const MGHost &mg) {
    int gz = (mg.maxRows[L + 1] + c.rq - 1) / c.rq;
    if (gz > 65535) gz = 65535;
    return dim3((mg.maxNx[L] + 31) / 32, c.ninst, gz > 0 ? gz : 1);
}
#define ROW_BLOCK dim3(32, c.rpb)
static int small_split(const Ctx &c, const MGHost &mg) {
    small_init();
    const int lim = c.small_nodes > 0 ? c.small_nodes : g_small_nodes;
    int Ls = 0;
    while (Ls < mg.maxlev - 1 && mg.maxN[Ls] > lim) Ls++;
    return Ls;
}
// shared-memory bytes of levels Ls.. of the shared-memory small-level kernel
template <class T>
static size_t smem_bytes(const MGHost &mg, int Ls) {
    size_t b = 0;
    for (int L = Ls; L < mg.maxlev; L++) b += smem_level_bytes<T>(mg.maxN[L], L == mg.maxlev - 1);
    return b;
}
// where the per-level kernels stop: the shared-memory kernel takes the levels from the
// first one at or below g_small_nodes whose data fits (never level 0); *smem = its bytes,
// 0 when the cluster kernel takes the small levels instead
template <class T>
static int small_plan(const Ctx &c, const MGHost &mg, size_t *smem) {
    int Ls = small_split(c, mg);
    *smem = 0;
    if (!g_smem_max || mg.maxlev < 2) return Ls;
    int L = Ls < 1 ? 1 : Ls;
    while (L < mg.maxlev - 1 && smem_bytes<T>(mg, L) > g_smem_max) L++;
    if (smem_bytes<T>(mg, L) > g_smem_max) return Ls;
    *smem = smem_bytes<T>(mg, L);
    return L;
}
template <class T>
static void launch_smem(const Ctx &c, int nodes, int Ls, double alpha, int gate, size_t bytes) {
    g_launches++;
    t_launches++;
    if (g_prof_on) prof_begin(pf<T>(PF_COARSE), c.st);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1, c.ninst);
    cfg.blockDim = dim3(SMALL_TPB);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = c.st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = g_pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k_vcycle_smem<T>, c.dP, Ls, alpha, gate);
    if (g_prof_on) prof_end(pf<T>(PF_COARSE), c.st, nodes);
}

template <class T>
static void vcycle_t(const Ctx &c, const MGHost &mg, int bsel, int xsel, int wsel, int mg_on, int gate) {
    const int SB = pf<T>(PF_SMOOTH_B), SR = pf<T>(PF_SMOOTH_R);
    if (!mg_on) {
        SS_LAUNCH_PDL(SB, c.maxN, smooth_fn<T>(0, 1), grid_half(c, 0, mg), ROW_BLOCK, c.st, c.dP, 0, bsel, xsel, gate);
        SS_LAUNCH_PDL(SR, c.maxN, smooth_fn<T>(0, 0), grid_half(c, 0, mg), ROW_BLOCK, c.st, c.dP, 0, bsel, xsel, gate);
        return;
    }
    size_t smem = 0;
    const int Ls = small_plan<T>(c, mg, &smem);
    for (int L = 0; L < Ls; L++) {
        SS_LAUNCH_PDL(SB, mg.maxN[L], smooth_fn<T>(0, 1), grid_half(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel, gate);
        SS_LAUNCH_PDL(SR, mg.maxN[L], smooth_fn<T>(0, 0), grid_half(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel, gate);
        if (L < g_deep_levels && g_l0_sweeps > 1) {     // second application (finest levels)
            SS_LAUNCH_PDL(SB, mg.maxN[L], smooth_fn<T>(2, 1), grid_half(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel, gate);
            SS_LAUNCH_PDL(SR, mg.maxN[L], smooth_fn<T>(2, 0), grid_half(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel, gate);
        }
        SS_LAUNCH_PDL(pf<T>(PF_RESID_RESTRICT), mg.maxN[L], k_resid_restrict2<T>, grid_rr(c, L, mg), block_rr(c), c.st, c.dP, L, bsel,
                  xsel, wsel, gate);
    }
    if (smem) launch_smem<T>(c, mg.maxN[Ls], Ls, mg.alpha, gate, smem);
    else launch_small<T>(c, mg.maxN[Ls], Ls, bsel, xsel, wsel, mg.alpha, gate);
    for (int L = Ls - 1; L >= 0; L--) {
        SS_LAUNCH_PDL(pf<T>(PF_PROLONG), mg.maxN[L], k_prolong<T>, grid_full(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel,
                  mg.alpha, gate);
        SS_LAUNCH_PDL(pf<T>(PF_LEVEL_RESID), mg.maxN[L], k_level_resid<T>, grid_full(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel,
                  xsel, gate);
        SS_LAUNCH_PDL(SB, mg.maxN[L], smooth_fn<T>(1, 1), grid_half(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel, gate);
        SS_LAUNCH_PDL(SR, mg.maxN[L], smooth_fn<T>(1, 0), grid_half(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel, gate);
        if (L < g_deep_levels && g_l0_sweeps > 1) {
            SS_LAUNCH_PDL(SB, mg.maxN[L], smooth_fn<T>(2, 1), grid_half(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel, gate);
            SS_LAUNCH_PDL(SR, mg.maxN[L], smooth_fn<T>(2, 0), grid_half(c, L, mg), ROW_BLOCK, c.st, c.dP, L, bsel, xsel, gate);
        }
    }
}
void vcycle(const Ctx &c, const MGHost &mg, int bsel, int xsel, int wsel, int mg_on, int gate) {
    vcycle_t<double>(c, mg, bsel, xsel, wsel, mg_on, gate);
}

// ------------------------------------------------------------------ PCG (semiconductor_3d.c:2182-2210)
// r = b - A x
template <class T>
__global__ void k_pcg_init_r(const DevP *__restrict__ Ps) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    const T *b = PT<T>::rhs(P), *x = PT<T>::sol(P);
    T *r = PT<T>::wk(P, 0);
    T *const *A = PT<T>::A0(P);
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        r[k] = b[k] - stencil_apply<T>(A, x, k, a.i, a.j, a.l, P.Nx, P.Ny, P.Nz);
    }
}
// FP32 start of a PCG solve from x = 0: b = r = (float) rhs
__global__ void k_pcg32_start(const DevP *__restrict__ Ps) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const float b = (float)P.rhs[k];
        P.rhs32[k] = b;
        P.wk32[0][k] = b;
        P.sol32[k] = 0.f;
    }
}
// rz = r.z; mode 0 initial (rz0), mode 1 iteration end (stop test, beta)
template <class T>
__global__ void k_pcg_rz(const DevP *__restrict__ Ps, int mode) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const T *r = PT<T>::wk(P, 0), *z = PT<T>::wk(P, 1);
    pdl_wait();
    if (mode && !ks_running<T>(P)) return;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) acc[0] += (double)r[k] * (double)z[k];
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *PT<T>::ks(P);
        const double rz = acc[0];
        if (!mode) {
            s.rz = s.rz0 = rz; s.it = 0; s.status = 0;
            s.active = (rz > 0.0) ? 1 : 0;
            if (!(rz > 0.0)) s.status = 2;
        } else {
            if (!(rz > s.rtol * s.rtol * s.rz0)) { s.active = 0; s.status = 1; }
            else if (s.it >= s.maxit) { s.active = 0; s.status = 3; }
            else { s.be = rz / s.rz; s.rz = rz; }
        }
    }
}
// p = z (init) or p = z + be p
template <class T>
__global__ void k_pcg_p(const DevP *__restrict__ Ps, int init) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    T *p = PT<T>::wk(P, 2);
    const T *z = PT<T>::wk(P, 1);
    pdl_wait();
    if (!ks_running<T>(P)) return;
    const T be = init ? T(0) : (T)PT<T>::ks(P)->be;
    SS_GRID_LOOP(k, P.N) p[k] = z[k] + (init ? T(0) : be * p[k]);
}
// q = A p; pq = p.q; al = rz / pq
template <class T>
__global__ void k_pcg_q(const DevP *__restrict__ Ps) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const T *p = PT<T>::wk(P, 2);
    T *q = PT<T>::wk(P, 3);
    T *const *A = PT<T>::A0(P);
    pdl_wait();
    if (!ks_running<T>(P)) return;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const T v = stencil_apply<T>(A, p, k, a.i, a.j, a.l, P.Nx, P.Ny, P.Nz);
        q[k] = v;
        acc[0] += (double)p[k] * (double)v;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 5)) {
        KrylovS &s = *PT<T>::ks(P);
        s.it++;
        const double pq = acc[0];
        if (!(pq > 0.0)) { s.active = 0; s.status = 2; s.al = 0.0; }
        else s.al = s.rz / pq;
    }
}
// x += al p; r -= al q
template <class T>
__global__ void k_pcg_xr(const DevP *__restrict__ Ps) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    T *x = PT<T>::sol(P), *r = PT<T>::wk(P, 0);
    const T *p = PT<T>::wk(P, 2), *q = PT<T>::wk(P, 3);
    pdl_wait();
    if (!ks_running<T>(P)) return;
    const T al = (T)PT<T>::ks(P)->al;
    SS_GRID_LOOP(k, P.N) { x[k] += al * p[k]; r[k] -= al * q[k]; }
}
// sol = (double) sol32 (end of an FP32 solve whose result is the whole solution)
__global__ void k_sol_from32(const DevP *__restrict__ Ps) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) P.sol[k] = (double)P.sol32[k];
}

// one PCG iteration (every kernel gated on the instance's active word)
template <class T>
static void pcg_body(const Ctx &c, const MGHost &mg) {
    SS_LAUNCH_PDL(pf<T>(PF_KRY_SPMV_DOT), c.maxN, k_pcg_q<T>, grid_nodes(c), TPB, c.st, c.dP);
    SS_LAUNCH_PDL(pf<T>(PF_KRY_UPDATE), c.maxN, k_pcg_xr<T>, grid_nodes(c), TPB, c.st, c.dP);
    vcycle_t<T>(c, mg, 0, 1, 0, 1, 1);
    SS_LAUNCH_PDL(pf<T>(PF_KRY_DOT), c.maxN, k_pcg_rz<T>, grid_nodes(c), TPB, c.st, c.dP, 1);
    SS_LAUNCH_PDL(pf<T>(PF_KRY_UPDATE), c.maxN, k_pcg_p<T>, grid_nodes(c), TPB, c.st, c.dP, 0);
}

// ------------------------------------------------------------------ BiCGSTAB (semiconductor_3d.c:2216-2320)
// work vectors: 0 r, 1 rh, 2 p, 3 v, 4 ph, 5 sh, 6 t, 7 x0 (start backup)
// r = b - A x; rh = r; p = v = 0; rr = r.r; fl = sum (sum|A x| + |b|)^2; tgt
__global__ void k_bicg_init(const DevP *__restrict__ Ps, double rtol, double atol) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    const double *b = P.rhs, *x = P.sol;
    double *r = P.wk[0], *rh = P.wk[1], *p = P.wk[2], *v = P.wk[3];
    const int NxNy = P.Nx * P.Ny;
    double acc[2] = {0.0, 0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const int i = a.i, j = a.j, l = a.l;
        double s = P.A[0][k] * x[k], fl = fabs(P.A[0][k] * x[k]) + fabs(b[k]), t;
        if (i > 0) { t = P.A[1][k] * x[k - 1]; s += t; fl += fabs(t); }
        if (i < P.Nx - 1) { t = P.A[2][k] * x[k + 1]; s += t; fl += fabs(t); }
        if (j > 0) { t = P.A[3][k] * x[k - P.Nx]; s += t; fl += fabs(t); }
        if (j < P.Ny - 1) { t = P.A[4][k] * x[k + P.Nx]; s += t; fl += fabs(t); }
        if (l > 0) { t = P.A[5][k] * x[k - NxNy]; s += t; fl += fabs(t); }
        if (l < P.Nz - 1) { t = P.A[6][k] * x[k + NxNy]; s += t; fl += fabs(t); }
        const double rk = b[k] - s;
        r[k] = rk; rh[k] = rk; p[k] = 0.0; v[k] = 0.0;
        acc[0] += rk * rk;
        acc[1] += fl * fl;
    }
    if (grid_sum<2>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
        s.rr = acc[0]; s.fl = acc[1];
        s.r0 = sqrt(acc[0]);
        s.tgt = fmax(rtol * s.r0, atol * sqrt(acc[1]));
        s.rho = s.al = s.om = 1.0; s.rbest = s.r0; s.stall = 0; s.it = 0; s.half = 0;
        if (!(s.r0 > s.tgt)) { s.active = 0; s.status = 1; }
        else { s.active = 1; s.status = 0; }
    }
}
// rho1 = rh.r; restart on breakdown; be
template <class T>
__global__ void k_bicg_rho(const DevP *__restrict__ Ps) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const T *r = PT<T>::wk(P, 0), *rh = PT<T>::wk(P, 1);
    pdl_wait();
    if (!ks_running<T>(P)) return;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) acc[0] += (double)rh[k] * (double)r[k];
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *PT<T>::ks(P);
        if (s.it >= s.maxit) { s.active = 0; s.status = 3; return; }
        s.it++;
        double rho1 = acc[0];
        s.pad0 = 0;
        if (fabs(rho1) < 1e-300) {              // breakdown: restart the shadow residual
            rho1 = s.rr;
            s.rho = s.al = s.om = 1.0;
            s.pad0 = 1;
            if (!(rho1 > 0.0)) { s.active = 0; s.status = 2; return; }
        }
        s.rho1 = rho1;
        s.be = (rho1 / s.rho) * (s.al / s.om);
    }
}
// p = r + be (p - om v); on a restart rh = r, p = r, v = 0
template <class T>
__global__ void k_bicg_p(const DevP *__restrict__ Ps) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    T *p = PT<T>::wk(P, 2), *v = PT<T>::wk(P, 3), *rh = PT<T>::wk(P, 1);
    const T *r = PT<T>::wk(P, 0);
    pdl_wait();
    if (!ks_running<T>(P)) return;
    const KrylovS &s = *PT<T>::ks(P);
    const T be = (T)s.be, om = (T)s.om;
    const int restart = s.pad0;
    SS_GRID_LOOP(k, P.N) {
        if (restart) { rh[k] = r[k]; p[k] = r[k]; v[k] = 0; }
        else p[k] = r[k] + be * (p[k] - om * v[k]);
    }
}
// v = A ph; rv = rh.v; al
template <class T>
__global__ void k_bicg_v(const DevP *__restrict__ Ps) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const T *ph = PT<T>::wk(P, 4), *rh = PT<T>::wk(P, 1);
    T *v = PT<T>::wk(P, 3);
    T *const *A = PT<T>::A0(P);
    pdl_wait();
    if (!ks_running<T>(P)) return;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const T t = stencil_apply<T>(A, ph, k, a.i, a.j, a.l, P.Nx, P.Ny, P.Nz);
        v[k] = t;
        acc[0] += (double)rh[k] * (double)t;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *PT<T>::ks(P);
        if (fabs(acc[0]) < 1e-300) { s.active = 0; s.status = 2; return; }
        s.rv = acc[0];
        s.al = s.rho1 / acc[0];
    }
}
// r -= al v; ss = r.r; half-step exit test
template <class T>
__global__ void k_bicg_s(const DevP *__restrict__ Ps) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    T *r = PT<T>::wk(P, 0);
    const T *v = PT<T>::wk(P, 3);
    pdl_wait();
    if (!ks_running<T>(P)) return;
    const T al = (T)PT<T>::ks(P)->al;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const T t = r[k] - al * v[k];
        r[k] = t;
        acc[0] += (double)t * (double)t;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *PT<T>::ks(P);
        s.ss = acc[0];
        if (sqrt(acc[0]) <= s.tgt) { s.half = 1; s.rr = acc[0]; }
    }
}
// t = A sh; tt = t.t; ts = t.r; om
template <class T>
__global__ void k_bicg_t(const DevP *__restrict__ Ps) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    const T *sh = PT<T>::wk(P, 5), *r = PT<T>::wk(P, 0);
    T *t = PT<T>::wk(P, 6);
    T *const *A = PT<T>::A0(P);
    pdl_wait();
    if (!ks_running<T>(P) || PT<T>::ks(P)->half) return;
    double acc[2] = {0.0, 0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const T q = stencil_apply<T>(A, sh, k, a.i, a.j, a.l, P.Nx, P.Ny, P.Nz);
        t[k] = q;
        acc[0] += (double)q * (double)q;
        acc[1] += (double)q * (double)r[k];
    }
    if (grid_sum<2>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *PT<T>::ks(P);
        s.tt = acc[0]; s.ts = acc[1];
        s.om = acc[0] > 0.0 ? acc[1] / acc[0] : 0.0;
    }
}
// x += al ph + om sh; r -= om t; rr = r.r; stop tests (or the half-step x update)
template <class T>
__global__ void k_bicg_x(const DevP *__restrict__ Ps) {
    pdl_launch();
    const DevP &P = Ps[blockIdx.y];
    T *x = PT<T>::sol(P), *r = PT<T>::wk(P, 0);
    const T *ph = PT<T>::wk(P, 4), *sh = PT<T>::wk(P, 5), *t = PT<T>::wk(P, 6);
    pdl_wait();
    if (!ks_running<T>(P)) return;
    const KrylovS &s0 = *PT<T>::ks(P);
    const T al = (T)s0.al, om = (T)s0.om;
    const int half = s0.half;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        if (half) { x[k] += al * ph[k]; continue; }
        x[k] += al * ph[k] + om * sh[k];
        const T q = r[k] - om * t[k];
        r[k] = q;
        acc[0] += (double)q * (double)q;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *PT<T>::ks(P);
        if (half) { s.active = 0; s.status = 1; return; }
        s.rr = acc[0];
        const double rn = sqrt(acc[0]);
        if (rn <= s.tgt || s.om == 0.0) { s.active = 0; s.status = 1; return; }
        if (rn < 0.99 * s.rbest) { s.rbest = rn; s.stall = 0; }
        else if (++s.stall > 40) { s.active = 0; s.status = 2; return; }
        s.rho = s.rho1;
    }
}

// one BiCGSTAB iteration (the continuity systems use the Slotboom-weighted hierarchy)
template <class T>
static void bicg_body(const Ctx &c, const MGHost &mg, int mg_on) {
    SS_LAUNCH_PDL(pf<T>(PF_KRY_DOT), c.maxN, k_bicg_rho<T>, grid_nodes(c), TPB, c.st, c.dP);
    SS_LAUNCH_PDL(pf<T>(PF_KRY_UPDATE), c.maxN, k_bicg_p<T>, grid_nodes(c), TPB, c.st, c.dP);
    vcycle_t<T>(c, mg, 2, 4, 1, mg_on, 1);          // ph = M p
    SS_LAUNCH_PDL(pf<T>(PF_KRY_SPMV_DOT), c.maxN, k_bicg_v<T>, grid_nodes(c), TPB, c.st, c.dP);
    SS_LAUNCH_PDL(pf<T>(PF_KRY_UPDATE), c.maxN, k_bicg_s<T>, grid_nodes(c), TPB, c.st, c.dP);
    vcycle_t<T>(c, mg, 0, 5, 1, mg_on, 2);          // sh = M r
    SS_LAUNCH_PDL(pf<T>(PF_KRY_SPMV_DOT), c.maxN, k_bicg_t<T>, grid_nodes(c), TPB, c.st, c.dP);
    SS_LAUNCH_PDL(pf<T>(PF_KRY_UPDATE), c.maxN, k_bicg_x<T>, grid_nodes(c), TPB, c.st, c.dP);
}

// ------------------------------------------------------------------ FP64 iterative refinement
// The refined continuity solve keeps x (sol) and the residual r = b - A x (wk[0]) in
// FP64 with the FP64 operator; each step solves A d = r in FP32 (the FP32 copy of A and
// the FP32 hierarchy, BiCGSTAB from d = 0 to a relative target) and applies x += d,
// r -= A d in FP64.  The stop rule is the reference's, evaluated on the FP64 residual:
// |r| <= max(rtol |r0|, atol sqrt(sum_k (sum_j |a_kj x_j| + |b_k|)^2)).
//
// start: r = b - A x, r0, the rounding floor and the target (outer record P.ks);
// rhs32 = (float) r
__global__ void k_ir_init(const DevP *__restrict__ Ps) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    const double *b = P.rhs, *x = P.sol;
    double *r = P.wk[0];
    const int NxNy = P.Nx * P.Ny;
    double acc[2] = {0.0, 0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const int i = a.i, j = a.j, l = a.l;
        double s = P.A[0][k] * x[k], fl = fabs(P.A[0][k] * x[k]) + fabs(b[k]), t;
        if (i > 0) { t = P.A[1][k] * x[k - 1]; s += t; fl += fabs(t); }
        if (i < P.Nx - 1) { t = P.A[2][k] * x[k + 1]; s += t; fl += fabs(t); }
        if (j > 0) { t = P.A[3][k] * x[k - P.Nx]; s += t; fl += fabs(t); }
        if (j < P.Ny - 1) { t = P.A[4][k] * x[k + P.Nx]; s += t; fl += fabs(t); }
        if (l > 0) { t = P.A[5][k] * x[k - NxNy]; s += t; fl += fabs(t); }
        if (l < P.Nz - 1) { t = P.A[6][k] * x[k + NxNy]; s += t; fl += fabs(t); }
        const double rk = b[k] - s;
        r[k] = rk;
        P.rhs32[k] = (float)rk;
        acc[0] += rk * rk;
        acc[1] += fl * fl;
    }
    if (grid_sum<2>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
        s.rr = acc[0]; s.fl = acc[1];
        s.r0 = sqrt(acc[0]);
        s.tgt = fmax(s.rtol * s.r0, s.atol * sqrt(acc[1]));
        s.rbest = s.r0; s.stall = 0; s.it = 0; s.half = 0;
        if (!(s.r0 > s.tgt)) { s.active = 0; s.status = 1; }
        else { s.active = 1; s.status = 0; }
    }
}
// inner start: d = 0, r = rh = rhs32, p = v = 0; inner target
// max(rtol_in |r_in|, factor * outer target) with rtol_in = ksi.rtol, factor = ksi.atol
__global__ void k_ir_inner_init(const DevP *__restrict__ Ps) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    const KrylovS &so = *P.ks;
    if (!so.active) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { P.ksi->active = 0; P.ksi->body_runs = 0; }
        return;
    }
    float *r = P.wk32[0], *rh = P.wk32[1], *p = P.wk32[2], *v = P.wk32[3], *x = P.sol32;
    const float *b = P.rhs32;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const float bk = b[k];
        r[k] = bk; rh[k] = bk; p[k] = 0.f; v[k] = 0.f; x[k] = 0.f;
        acc[0] += (double)bk * (double)bk;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ksi;
        s.rr = acc[0];
        s.r0 = sqrt(acc[0]);
        s.tgt = fmax(s.rtol * s.r0, s.atol * so.tgt);
        s.rho = s.al = s.om = 1.0; s.rbest = s.r0; s.stall = 0; s.it = 0; s.half = 0; s.body_runs = 0;
        s.maxit = so.maxit - so.it;
        s.status = 0;
        s.active = (s.r0 > s.tgt && s.maxit > 0) ? 1 : 0;
    }
}
// x += d; r -= A d (FP64 operator); rhs32 = (float) r; the outer stop test.  A step
// that does not halve the residual ends the refinement with status 4 (the FP64 solver
// takes over from the host).
__global__ void k_ir_update(const DevP *__restrict__ Ps) {
    pdl_entry();
    const DevP &P = Ps[blockIdx.y];
    if (!P.ks->active) return;
    const float *d = P.sol32;
    double *x = P.sol, *r = P.wk[0];
    const int NxNy = P.Nx * P.Ny;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const int i = a.i, j = a.j, l = a.l;
        const double dk = (double)d[k];
        double s = P.A[0][k] * dk;
        if (i > 0) s += P.A[1][k] * (double)d[k - 1];
        if (i < P.Nx - 1) s += P.A[2][k] * (double)d[k + 1];
        if (j > 0) s += P.A[3][k] * (double)d[k - P.Nx];
        if (j < P.Ny - 1) s += P.A[4][k] * (double)d[k + P.Nx];
        if (l > 0) s += P.A[5][k] * (double)d[k - NxNy];
        if (l < P.Nz - 1) s += P.A[6][k] * (double)d[k + NxNy];
        x[k] += dk;
        const double rk = r[k] - s;
        r[k] = rk;
        P.rhs32[k] = (float)rk;
        acc[0] += rk * rk;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
        s.it += P.ksi->it;
        s.body_runs++;                                // refinement steps of this solve
        s.rr = acc[0];
        const double rn = sqrt(acc[0]);
        if (rn <= s.tgt) { s.active = 0; s.status = 1; }
        else if (!(rn < 0.5 * s.rbest)) { s.active = 0; s.status = 4; }
        else if (s.it >= s.maxit) { s.active = 0; s.status = 3; }
        else s.rbest = rn;
    }
}

// ------------------------------------------------------------------ device-looped solves
// A Krylov solve runs as one CUDA graph: a conditional WHILE node whose body is one
// iteration; the body's last kernel sets the loop condition from the instances' active
// words, so the iteration loop runs on the device with no host round trip.
__global__ void k_loop_cond(const DevP *__restrict__ Ps, int ninst, cudaGraphConditionalHandle h, int body, int inner) {
    pdl_entry();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned any = 0;
    for (int i = 0; i < ninst; i++) {
        KrylovS *s = inner ? Ps[i].ksi : Ps[i].ks;
        if (body) s->body_runs++;
        any |= s->active ? 1u : 0u;
    }
    cudaGraphSetConditional(h, any);
}

static bool g_graph_warned = false;
#define GCK(x)                                                                                     \
    do {                                                                                           \
        if ((x) != cudaSuccess) {                                                                  \
            if (!g_graph_warned)                                                                   \
                std::fprintf(stderr, "semisim-b200: graph build failed (%s), iterating from the host\n", \
                             cudaGetErrorString(cudaGetLastError()));                              \
            g_graph_warned = true;                                                                 \
            if (g) cudaGraphDestroy(g);                                                            \
            return nullptr;                                                                        \
        }                                                                                          \
    } while (0)

static void loop_body(const Ctx &c, const MGHost &mg, int kind) {
    switch (kind) {
    case 0: pcg_body<double>(c, mg); break;
    case 1: bicg_body<double>(c, mg, 1); break;
    case 2: bicg_body<double>(c, mg, 0); break;
    case 3: pcg_body<float>(c, mg); break;
    default: bicg_body<float>(c, mg, 1); break;
    }
}

// the graph of `kind` (LoopGraphs); *nkern = kernels of one body pass, *nfix = kernels
// outside the loop
static cudaGraphExec_t build_loop(const Ctx &c, const MGHost &mg, int kind, int *nkern, int *nfix) {
    cudaGraph_t g = nullptr;
    GCK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    GCK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    const DevP *dp = c.dP;
    const int inner = kind >= 3 ? 1 : 0;
    int ninst = c.ninst, body0 = 0;
    const int nblk = c.nodes_blocks();
    void *args[] = {(void *)&dp, (void *)&ninst, (void *)&h, (void *)&body0, (void *)&inner};
    void *args1[] = {(void *)&dp};
    cudaKernelNodeParams kp = {};
    cudaGraphNode_t n_init = nullptr, n0, cn, n_upd;
    int fixed = 1;
    if (kind == 4) {                                  // refinement step: inner start
        kp.func = (void *)k_ir_inner_init;
        kp.gridDim = dim3(nblk, c.ninst);
        kp.blockDim = dim3(TPB);
        kp.kernelParams = args1;
        GCK(cudaGraphAddKernelNode(&n_init, g, nullptr, 0, &kp));
        fixed++;
    }
    kp = {};
    kp.func = (void *)k_loop_cond;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = args;
    GCK(cudaGraphAddKernelNode(&n0, g, n_init ? &n_init : nullptr, n_init ? 1 : 0, &kp));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    GCK(cudaGraphAddNode(&cn, g, &n0, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    GCK(cudaStreamBeginCaptureToGraph(c.st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    const unsigned long long l0 = t_launches;
    loop_body(c, mg, kind);
    launch_pdl(k_loop_cond, dim3(1), dim3(32), c.st, c.dP, c.ninst, h, 1, inner);
    const unsigned long long nb = t_launches - l0;
    *nkern = int(nb) + 1;
    g_launches -= nb;                                  // counted per executed body instead
    t_launches = l0;
    cudaGraph_t out = nullptr;
    GCK(cudaStreamEndCapture(c.st, &out));
    if (kind == 4) {                                  // refinement step: FP64 update
        kp = {};
        kp.func = (void *)k_ir_update;
        kp.gridDim = dim3(nblk, c.ninst);
        kp.blockDim = dim3(TPB);
        kp.kernelParams = args1;
        GCK(cudaGraphAddKernelNode(&n_upd, g, &cn, 1, &kp));
        fixed++;
    }
    *nfix = fixed;
    cudaGraphExec_t ex = nullptr;
    GCK(cudaGraphInstantiate(&ex, g, 0));
    cudaGraphDestroy(g);
    return ex;
}

bool g_use_graphs = true;

static KrylovS read_ks(const Ctx &c, const KrylovS *src) {
    KrylovS hs{};
    cudaMemcpyAsync(&hs, src, sizeof(KrylovS), cudaMemcpyDeviceToHost, c.st);
    cudaStreamSynchronize(c.st);
    return hs;
}

// Run the iteration loop of `kind` to completion (kind 4: one refinement step); returns
// the loop's Krylov record (the inner one for the FP32 kinds)
static KrylovS run_loop(const Ctx &c, const MGHost &mg, int kind, int maxit, int check_every) {
    const KrylovS *rec = kind >= 3 ? c.h.ksi : c.h.ks;
    LoopGraphs *lg = c.lg;
    if (lg && g_use_graphs && !g_prof_on && !lg->failed) {
        if (!lg->exec[kind]) {
            int nfix = 1;
            lg->exec[kind] = build_loop(c, mg, kind, &lg->kernels[kind], &nfix);
            if (!lg->exec[kind]) lg->failed = 1;
            else lg->kernels[kind] |= nfix << 16;
        }
        if (lg->exec[kind]) {
            cudaGraphLaunch(lg->exec[kind], c.st);
            const KrylovS hs = read_ks(c, rec);
            const unsigned long long body = (unsigned long long)(lg->kernels[kind] & 0xffff);
            const unsigned long long ran = (unsigned long long)(lg->kernels[kind] >> 16) + body * hs.body_runs;
            g_launches += ran;
            t_launches += ran;
            return hs;
        }
    }
    if (kind == 4) SS_LAUNCH_PDL(PF_KRY_INIT32, c.maxN, k_ir_inner_init, grid_nodes(c), TPB, c.st, c.dP);
    KrylovS hs{};
    for (int it = 0; it < maxit + 1;) {
        if (kind == 4 && it == 0) {
            hs = read_ks(c, rec);
            if (!hs.active) break;
        }
        for (int q = 0; q < check_every && it < maxit + 1; q++, it++) loop_body(c, mg, kind);
        hs = read_ks(c, rec);
        if (!hs.active) break;
    }
    if (kind == 4) SS_LAUNCH_PDL(PF_REFINE, c.maxN, k_ir_update, grid_nodes(c), TPB, c.st, c.dP);
    return hs;
}

// ------------------------------------------------------------------ solver drivers
// refinement statistics of the calling thread's solves (steps, FP64 take-overs)
thread_local long long t_ir_steps = 0, t_ir_fallbacks = 0;
double g_ir_factor = 0.7;      // inner target as a fraction of the outer target
double g_ir_rtol_min = 1e-5;   // smallest relative reduction asked of one FP32 solve

// PCG of the Poisson Newton system from sol = 0 (the reference's stop rule r.z <=
// rtol^2 r0.z0).  mixed: FP32 vectors and hierarchy (the Newton loop's FP64 residual
// refines it); rtol below 1e-5 and FP32 failures use the FP64 solver.
int pcg_solve(const Ctx &c, const MGHost &mg, int maxit, double rtol, int check_every, int mixed) {
    KrylovS ks0{};
    ks0.active = 1;
    ks0.maxit = maxit;
    ks0.rtol = rtol;
    if (mixed && rtol >= 1e-5) {
        cudaMemcpyAsync(c.h.ksi, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
        const int pr = persist_pcg(c, mg, 1);        // set-up and solve in one persistent launch
        if (pr == 1) {
            const KrylovS hs = read_ks(c, c.h.ksi);
            if (hs.status == 1) return hs.it;
            t_ir_fallbacks++;
            launch_fill_sel(c, V_SOL, 0.0);
            return hs.it + pcg_solve(c, mg, maxit, rtol, check_every, 0);
        }
        if (pr < 0) cudaMemcpyAsync(c.h.ksi, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
        mg_setup_t<float>(c, mg, 0);
        SS_LAUNCH_PDL(PF_KRY_INIT32, c.maxN, k_pcg32_start, grid_nodes(c), TPB, c.st, c.dP);
        vcycle_t<float>(c, mg, 0, 1, 0, 1, 0);
        SS_LAUNCH_PDL(PF_KRY_DOT32, c.maxN, k_pcg_rz<float>, grid_nodes(c), TPB, c.st, c.dP, 0);
        SS_LAUNCH_PDL(PF_KRY_UPDATE32, c.maxN, k_pcg_p<float>, grid_nodes(c), TPB, c.st, c.dP, 1);
        const KrylovS hs = run_loop(c, mg, 3, maxit, check_every);
        if (hs.status == 1) {
            SS_LAUNCH_PDL(PF_VEC, c.maxN, k_sol_from32, grid_nodes(c), TPB, c.st, c.dP);
            return hs.it;
        }
        t_ir_fallbacks++;
        launch_fill_sel(c, V_SOL, 0.0);
        return hs.it + pcg_solve(c, mg, maxit, rtol, check_every, 0);
    }
    cudaMemcpyAsync(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
    if (c.ninst == 1 && persist_enabled()) {
        launch_copy_sel(c, 7, V_SOL);                // start backup (the persistent path may be abandoned)
        const int pr = persist_pcg(c, mg, 0);        // set-up and solve in one persistent launch
        if (pr == 1) return read_ks(c, c.h.ks).it;
        if (pr < 0) {
            launch_copy_sel(c, V_SOL, 7);
            cudaMemcpyAsync(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
        }
    }
    mg_setup_t<double>(c, mg, 0);
    SS_LAUNCH_PDL(PF_KRY_INIT, c.maxN, k_pcg_init_r<double>, grid_nodes(c), TPB, c.st, c.dP);
    vcycle_t<double>(c, mg, 0, 1, 0, 1, 0);                  // z = M r
    SS_LAUNCH_PDL(PF_KRY_DOT, c.maxN, k_pcg_rz<double>, grid_nodes(c), TPB, c.st, c.dP, 0);
    SS_LAUNCH_PDL(PF_KRY_UPDATE, c.maxN, k_pcg_p<double>, grid_nodes(c), TPB, c.st, c.dP, 1);
    const KrylovS hs = run_loop(c, mg, 0, maxit, check_every);
    return hs.it;
}

// FP64-refined BiCGSTAB with FP32 inner solves (multigrid preconditioner).  A stalled
// refinement hands the solve to the FP64 solver with the same target.
static int bicgstab_refined(const Ctx &c, const MGHost &mg, int maxit, double rtol, double atol, int check_every,
                            double *rn, double *r0, int qsign) {
    KrylovS ko{}, ki{};
    ko.maxit = maxit;
    ko.rtol = rtol;
    ko.atol = atol;
    ki.rtol = g_ir_rtol_min;
    ki.atol = g_ir_factor;
    cudaMemcpyAsync(c.h.ks, &ko, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
    cudaMemcpyAsync(c.h.ksi, &ki, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
    launch_copy_sel(c, 7, V_SOL);                   // start backup
    KrylovS hs{};
    int steps = 0;
    const int pr = persist_refined(c, mg, 16, &steps, qsign);   // set-up and every step in one launch
    if (pr == 1) {
        hs = read_ks(c, c.h.ks);
        t_ir_steps += steps > 0 ? steps : 1;
    } else {
        if (pr < 0) {                                // abandoned: restore the start, per-pass solve
            launch_copy_sel(c, V_SOL, 7);
            cudaMemcpyAsync(c.h.ks, &ko, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
            cudaMemcpyAsync(c.h.ksi, &ki, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
        }
        mg_setup_t<float>(c, mg, qsign);
        SS_LAUNCH_PDL(PF_REFINE, c.maxN, k_ir_init, grid_nodes(c), TPB, c.st, c.dP);
        for (int step = 0; step < 16; step++) {
            run_loop(c, mg, 4, maxit, check_every);
            hs = read_ks(c, c.h.ks);
            t_ir_steps++;
            if (!hs.active) break;
        }
    }
    *r0 = hs.r0;
    if (hs.status == 1 || hs.status == 3) {
        *rn = sqrt(hs.rr);
        return hs.it;
    }
    // the refinement stalled: FP64 BiCGSTAB to the same target, from the better of
    // the start and the refined iterate
    t_ir_fallbacks++;
    double rcur = sqrt(hs.rr);
    if (!(rcur <= hs.r0)) {
        launch_copy_sel(c, V_SOL, 7);
        rcur = hs.r0;
    }
    const double rt = rcur > 0.0 ? hs.tgt / rcur : rtol;
    double rn2 = 0, r02 = 0;
    const int its = bicgstab_core(c, mg, maxit, rt, atol, 1, check_every, &rn2, &r02, qsign, 0);
    *rn = rn2;
    return hs.it + its;
}

// One BiCGSTAB solve of P.A sol = rhs from the present sol.  Returns the iterations;
// rn / r0 the final and initial residual norms.  mixed: FP64-refined FP32 solve (with
// the multigrid preconditioner only; the smoother-only retry stays FP64).
int bicgstab_core(const Ctx &c, const MGHost &mg, int maxit, double rtol, double atol, int mg_on, int check_every,
                  double *rn, double *r0, int qsign, int mixed) {
    if (mixed && mg_on && mg.maxlev > 1) return bicgstab_refined(c, mg, maxit, rtol, atol, check_every, rn, r0, qsign);
    KrylovS ks0{};
    ks0.maxit = maxit;
    ks0.rtol = rtol;
    ks0.atol = atol;
    cudaMemcpyAsync(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
    if (mg_on && c.ninst == 1 && persist_enabled()) {
        launch_copy_sel(c, 7, V_SOL);                // start backup (the persistent path may be abandoned)
        const int pr = persist_bicg(c, mg, rtol, atol, qsign);   // set-up and solve in one launch
        if (pr == 1) {
            const KrylovS hs = read_ks(c, c.h.ks);
            *rn = sqrt(hs.rr);
            *r0 = hs.r0;
            return hs.it;
        }
        if (pr < 0) {
            launch_copy_sel(c, V_SOL, 7);
            cudaMemcpyAsync(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
        }
    }
    if (mg_on) mg_setup_t<double>(c, mg, qsign);
    else {
        SS_LAUNCH_PDL(PF_ILU_DIAG, c.maxN, k_ilu_diag<double>, grid_nodes(c), TPB, c.st, c.dP, 0);
    }
    SS_LAUNCH_PDL(PF_KRY_INIT, c.maxN, k_bicg_init, grid_nodes(c), TPB, c.st, c.dP, rtol, atol);
    const KrylovS hs = run_loop(c, mg, mg_on ? 1 : 2, maxit, check_every);
    *rn = sqrt(hs.rr);
    *r0 = hs.r0;
    return hs.it;
}

// ------------------------------------------------------------------ kernel timing hook
// Time `reps` launches of one kernel of the solve path on the instance's present state
// (test hook for per-kernel roofline numbers; it overwrites work vectors).  Returns
// microseconds per launch.  0-10 FP64, 11-16 the FP32 twins.
double bench_la_kernel(const Ctx &c, const MGHost &mg, int which, int reps) {
    KrylovS ks0{};
    ks0.active = 1;
    ks0.maxit = 1 << 30;
    cudaMemcpy(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice);
    cudaMemcpy(c.h.ksi, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice);
    size_t sm64 = 0, sm32 = 0;
    const int Ls64 = small_plan<double>(c, mg, &sm64), Ls32 = small_plan<float>(c, mg, &sm32);
    if (which >= 11) {
        mg_setup_t<float>(c, mg, 1);
        cudaStreamSynchronize(c.st);
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const dim3 grr = grid_rr(c, 0, mg), brr = block_rr(c);
    auto one = [&]() {
        switch (which) {
        case 0: k_bicg_v<double><<<grid_nodes(c), TPB, 0, c.st>>>(c.dP); break;
        case 1: k_smooth_cm<double, 0, 1><<<grid_half(c, 0, mg), ROW_BLOCK, 0, c.st>>>(c.dP, 0, 2, 4, 0); break;
        case 2: k_smooth_cm<double, 0, 0><<<grid_half(c, 0, mg), ROW_BLOCK, 0, c.st>>>(c.dP, 0, 2, 4, 0); break;
        case 3: k_resid_restrict2<double><<<grr, brr, 0, c.st>>>(c.dP, 0, 2, 4, 1, 0); break;
        case 4: k_level_resid<double><<<grid_full(c, 0, mg), ROW_BLOCK, 0, c.st>>>(c.dP, 0, 2, 4, 0); break;
        case 5: k_prolong<double><<<grid_full(c, 0, mg), ROW_BLOCK, 0, c.st>>>(c.dP, 0, 2, 4, 1.0, 0); break;
        case 6: k_bicg_x<double><<<grid_nodes(c), TPB, 0, c.st>>>(c.dP); break;
        case 7:
            if (sm64) launch_smem<double>(c, mg.maxN[Ls64], Ls64, 1.0, 0, sm64);
            else launch_small<double>(c, mg.maxN[Ls64], Ls64, 2, 4, 1, 1.0, 0);
            break;
        case 8: vcycle_t<double>(c, mg, 2, 4, 1, 1, 0); break;
        case 9: k_copy<<<grid_nodes(c), TPB, 0, c.st>>>(c.dP, 5, 6); break;
        case 10: k_bicg_rho<double><<<grid_nodes(c), TPB, 0, c.st>>>(c.dP); break;
        case 11: k_bicg_v<float><<<grid_nodes(c), TPB, 0, c.st>>>(c.dP); break;
        case 12: k_smooth_cm<float, 0, 1><<<grid_half(c, 0, mg), ROW_BLOCK, 0, c.st>>>(c.dP, 0, 2, 4, 0); break;
        case 13: k_smooth_cm<float, 0, 0><<<grid_half(c, 0, mg), ROW_BLOCK, 0, c.st>>>(c.dP, 0, 2, 4, 0); break;
        case 14: k_resid_restrict2<float><<<grr, brr, 0, c.st>>>(c.dP, 0, 2, 4, 1, 0); break;
        case 15: vcycle_t<float>(c, mg, 2, 4, 1, 1, 0); break;
        case 16: k_ir_update<<<grid_nodes(c), TPB, 0, c.st>>>(c.dP); break;
        case 17:
            if (sm32) launch_smem<float>(c, mg.maxN[Ls32], Ls32, 1.0, 0, sm32);
            else launch_small<float>(c, mg.maxN[Ls32], Ls32, 2, 4, 1, 1.0, 0);
            break;
        default: break;
        }
    };
    for (int r = 0; r < 3; r++) one();
    cudaEventRecord(a, c.st);
    for (int r = 0; r < reps; r++) one();
    cudaEventRecord(b, c.st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return 1e3 * ms / reps;
}

}  // namespace ss
