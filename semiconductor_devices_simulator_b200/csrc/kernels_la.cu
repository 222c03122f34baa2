// Linear algebra of the solve path on 7-point stencils: level-0 SpMV fused with the
// Krylov dot products, the geometric 2x2x2 aggregation multigrid (Slotboom-weighted
// prolongation, Petrov-Galerkin coarse operators, red-black D-ILU smoother, dense
// coarsest level) and device-resident PCG / BiCGSTAB.
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
#include <vector>

#include <cooperative_groups.h>

#include "device_common.cuh"
#include "prof.h"
#include "kernels.h"
#include "solver_ctx.h"

namespace cg = cooperative_groups;

namespace ss {

static inline dim3 grid_nodes(const Ctx &c) { return dim3(c.nodes_blocks(), c.ninst); }
static inline dim3 grid_n(const Ctx &c, int n) {
    int b = (n + TPB - 1) / TPB;
    if (b > c.grid_cap) b = c.grid_cap;
    if (b < 1) b = 1;
    return dim3(b, c.ninst);
}

// vector selectors of the level-0 Krylov vectors
__device__ __forceinline__ double *vsel(const DevP &P, int s) {
    if (s < 8) return P.wk[s];
    switch (s) {
    case V_RHS: return P.rhs;
    case V_SOL: return P.sol;
    case V_F: return P.F;
    case V_TR: return P.tr;
    case V_PHI: return P.phi;
    default: return P.dsc;
    }
}

// y = A x on a level (7-point, boundary terms skipped as in semiconductor_3d.c:1975-1993)
template <class T>
__device__ __forceinline__ double stencil_apply(T *const *A, const T *x, int k, int i, int j, int l, int Nx, int Ny,
                                                int Nz) {
    const int NxNy = Nx * Ny;
    double s = (double)A[0][k] * (double)x[k];
    if (i > 0) s += (double)A[1][k] * (double)x[k - 1];
    if (i < Nx - 1) s += (double)A[2][k] * (double)x[k + 1];
    if (j > 0) s += (double)A[3][k] * (double)x[k - Nx];
    if (j < Ny - 1) s += (double)A[4][k] * (double)x[k + Nx];
    if (l > 0) s += (double)A[5][k] * (double)x[k - NxNy];
    if (l < Nz - 1) s += (double)A[6][k] * (double)x[k + NxNy];
    return s;
}
// sum over the off-diagonal couplings only
template <class T>
__device__ __forceinline__ double offdiag_apply(T *const *A, const T *x, int k, int i, int j, int l, int Nx, int Ny,
                                                int Nz) {
    const int NxNy = Nx * Ny;
    double s = 0.0;
    if (i > 0) s += (double)A[1][k] * (double)x[k - 1];
    if (i < Nx - 1) s += (double)A[2][k] * (double)x[k + 1];
    if (j > 0) s += (double)A[3][k] * (double)x[k - Nx];
    if (j < Ny - 1) s += (double)A[4][k] * (double)x[k + Nx];
    if (l > 0) s += (double)A[5][k] * (double)x[k - NxNy];
    if (l < Nz - 1) s += (double)A[6][k] * (double)x[k + NxNy];
    return s;
}
// sum of a_kj x_j / D_j over the neighbours (forward sweep of the black rows)
template <class T>
__device__ __forceinline__ double offdiag_apply_div(T *const *A, const T *x, const T *D, int k, int i, int j, int l,
                                                    int Nx, int Ny, int Nz) {
    const int NxNy = Nx * Ny;
    double s = 0.0;
    if (i > 0) s += (double)A[1][k] * (double)x[k - 1] / (double)D[k - 1];
    if (i < Nx - 1) s += (double)A[2][k] * (double)x[k + 1] / (double)D[k + 1];
    if (j > 0) s += (double)A[3][k] * (double)x[k - Nx] / (double)D[k - Nx];
    if (j < Ny - 1) s += (double)A[4][k] * (double)x[k + Nx] / (double)D[k + Nx];
    if (l > 0) s += (double)A[5][k] * (double)x[k - NxNy] / (double)D[k - NxNy];
    if (l < Nz - 1) s += (double)A[6][k] * (double)x[k + NxNy] / (double)D[k + NxNy];
    return s;
}

// ------------------------------------------------------------------ multigrid levels
// level accessors: level 0 reads the instance's system arrays and the caller's vectors
struct LevView {
    double *A[7];
    double *D, *x, *b, *r, *pw, *ph;
    int Nx, Ny, Nz, N, cx, cy, cz, last;
};
__device__ __forceinline__ LevView levview(const DevP &P, int L, int bsel, int xsel) {
    const LevelT<double> &lv = P.lev[L];
    LevView v;
#pragma unroll
    for (int q = 0; q < 7; q++) v.A[q] = L == 0 ? P.A[q] : lv.A[q];
    v.D = lv.D; v.r = lv.r; v.pw = lv.pw; v.ph = lv.ph;
    v.x = L == 0 ? vsel(P, xsel) : lv.x;
    v.b = L == 0 ? vsel(P, bsel) : lv.b;
    v.Nx = lv.Nx; v.Ny = lv.Ny; v.Nz = lv.Nz; v.N = lv.N;
    v.cx = lv.cx; v.cy = lv.cy; v.cz = lv.cz; v.last = lv.last;
    return v;
}
__device__ __forceinline__ bool ks_running(const DevP &P) { return P.ks->active != 0; }

// red-black D-ILU pivots: red D = a_kk; black D = a_kk - sum a_kr a_rk / a_rr, guarded
// as the reference guards its ILU pivots (semiconductor_3d.c:1937-1938)
__global__ void k_ilu_diag(const DevP *__restrict__ Ps, int L) {
    const DevP &P = Ps[blockIdx.y];
    if (L > 0 && L >= P.nlev - 1) return;
    const LevView v = levview(P, L, 0, 0);
    SS_GRID_LOOP(k, v.N) {
        const Node a = unidx(k, v.Nx, v.Ny);
        const double c = v.A[0][k];
        double d = c;
        if ((a.i + a.j + a.l) & 1) {
            const int NxNy = v.Nx * v.Ny;
            double s = 0.0;
            if (a.i > 0) s += v.A[1][k] * v.A[2][k - 1] / v.A[0][k - 1];
            if (a.i < v.Nx - 1) s += v.A[2][k] * v.A[1][k + 1] / v.A[0][k + 1];
            if (a.j > 0) s += v.A[3][k] * v.A[4][k - v.Nx] / v.A[0][k - v.Nx];
            if (a.j < v.Ny - 1) s += v.A[4][k] * v.A[3][k + v.Nx] / v.A[0][k + v.Nx];
            if (a.l > 0) s += v.A[5][k] * v.A[6][k - NxNy] / v.A[0][k - NxNy];
            if (a.l < v.Nz - 1) s += v.A[6][k] * v.A[5][k + NxNy] / v.A[0][k + NxNy];
            d = c - s;
            if (!(d > 1e-8 * fabs(c))) d = c;
        }
        if (!(d != 0.0)) d = 1.0;
        v.D[k] = d;
    }
}

// pre-smoothing from x = 0: black rows then red rows of the two triangular sweeps
// mode 0: x = M^-1 b (from zero).  mode 1: post-smoothing, z = M^-1 r with r the level's
// residual array, x += z (the black z is parked in r for the red sweep).
__global__ void k_smooth_black(const DevP *__restrict__ Ps, int L, int bsel, int xsel, int mode, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if ((L > 0 && L >= P.nlev - 1) || (gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const LevView v = levview(P, L, bsel, xsel);
    const double *src = mode ? v.r : v.b;
    SS_GRID_LOOP(k, v.N) {
        const Node a = unidx(k, v.Nx, v.Ny);
        if (!((a.i + a.j + a.l) & 1)) continue;
        const double s = offdiag_apply_div<double>(v.A, src, v.D, k, a.i, a.j, a.l, v.Nx, v.Ny, v.Nz);
        const double z = (src[k] - s) / v.D[k];
        if (mode) { v.x[k] += z; v.r[k] = z; }
        else v.x[k] = z;
    }
}
__global__ void k_smooth_red(const DevP *__restrict__ Ps, int L, int bsel, int xsel, int mode, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if ((L > 0 && L >= P.nlev - 1) || (gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const LevView v = levview(P, L, bsel, xsel);
    const double *src = mode ? v.r : v.b;
    const double *zb = mode ? v.r : v.x;
    SS_GRID_LOOP(k, v.N) {
        const Node a = unidx(k, v.Nx, v.Ny);
        if ((a.i + a.j + a.l) & 1) continue;
        const double s = offdiag_apply<double>(v.A, zb, k, a.i, a.j, a.l, v.Nx, v.Ny, v.Nz);
        const double z = (src[k] - s) / v.D[k];
        if (mode) v.x[k] += z;
        else v.x[k] = z;
    }
}

// coarse aggregate (I,J,L) -> fine index range (AGG_RANGE, semiconductor_3d.c:1996-1999)
struct Agg { int i0, i1, j0, j1, l0, l1; };
__device__ __forceinline__ Agg agg_range(const LevView &f, int I, int J, int K) {
    Agg g;
    g.i0 = f.cx ? 2 * I : I; g.i1 = f.cx ? 2 * I + 1 : I; if (g.i1 > f.Nx - 1) g.i1 = f.Nx - 1;
    g.j0 = f.cy ? 2 * J : J; g.j1 = f.cy ? 2 * J + 1 : J; if (g.j1 > f.Ny - 1) g.j1 = f.Ny - 1;
    g.l0 = f.cz ? 2 * K : K; g.l1 = f.cz ? 2 * K + 1 : K; if (g.l1 > f.Nz - 1) g.l1 = f.Nz - 1;
    return g;
}

// residual b - A x of the fine level summed over every aggregate (restriction), with
// the level-0 row weights w (semiconductor_3d.c:2028-2037 applied to 1984-1991)
__global__ void k_resid_restrict(const DevP *__restrict__ Ps, int L, int bsel, int xsel, int wsel, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if (L >= P.nlev - 1 || (gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const LevView f = levview(P, L, bsel, xsel);
    const LevelT<double> &cl = P.lev[L + 1];
    const double *w = (L == 0 && wsel) ? P.dsc : nullptr;
    SS_GRID_LOOP(K, cl.N) {
        const Node c = unidx(K, cl.Nx, cl.Ny);
        const Agg g = agg_range(f, c.i, c.j, c.l);
        double s = 0.0;
        for (int l = g.l0; l <= g.l1; l++)
            for (int j = g.j0; j <= g.j1; j++)
                for (int i = g.i0; i <= g.i1; i++) {
                    const int k = i + f.Nx * (j + f.Ny * l);
                    const double r = f.b[k] - stencil_apply<double>(f.A, f.x, k, i, j, l, f.Nx, f.Ny, f.Nz);
                    s += w ? w[k] * r : r;
                }
        cl.b[K] = s;
    }
}

// x += alpha pw P xc (semiconductor_3d.c:2038-2048), then nothing else: the residual
// needs every prolonged neighbour and is a separate pass
__global__ void k_prolong(const DevP *__restrict__ Ps, int L, int bsel, int xsel, double alpha, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if (L >= P.nlev - 1 || (gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const LevView f = levview(P, L, bsel, xsel);
    const LevelT<double> &cl = P.lev[L + 1];
    SS_GRID_LOOP(k, f.N) {
        const Node a = unidx(k, f.Nx, f.Ny);
        const int I = f.cx ? a.i >> 1 : a.i, J = f.cy ? a.j >> 1 : a.j, K = f.cz ? a.l >> 1 : a.l;
        f.x[k] += alpha * f.pw[k] * cl.x[I + cl.Nx * (J + cl.Ny * K)];
    }
}
__global__ void k_level_resid(const DevP *__restrict__ Ps, int L, int bsel, int xsel, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if (L >= P.nlev - 1 || (gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const LevView f = levview(P, L, bsel, xsel);
    SS_GRID_LOOP(k, f.N) {
        const Node a = unidx(k, f.Nx, f.Ny);
        f.r[k] = f.b[k] - stencil_apply<double>(f.A, f.x, k, a.i, a.j, a.l, f.Nx, f.Ny, f.Nz);
    }
}

// coarsest level: x = M^-1 b with the dense inverse formed at set-up (one block per instance)
__global__ void k_coarse_solve(const DevP *__restrict__ Ps, int L, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if (L != P.nlev - 1 || (gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const LevelT<double> &v = P.lev[L];
    const int n = v.N;
    __shared__ double sb[COARSE_MAX];
    double *b = v.b, *x = v.x;
    if (L == 0) return;                    // a single-level hierarchy is not built
    for (int q = threadIdx.x; q < n; q += blockDim.x) sb[q] = b[q];
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < n; q++) s += v.D[r * n + q] * sb[q];
        x[r] = s;
    }
}

// coarsest level set-up: dense matrix of the stencil, Gauss-Jordan inverse with partial
// pivoting (tiny pivots guarded as semiconductor_3d.c:2066 does)
__global__ void k_coarse_setup(const DevP *__restrict__ Ps, int L) {
    const DevP &P = Ps[blockIdx.y];
    if (L != P.nlev - 1 || L == 0) return;
    const LevelT<double> &v = P.lev[L];
    const int n = v.N;
    __shared__ double M[COARSE_MAX][COARSE_MAX + 1];
    __shared__ int perm[COARSE_MAX];
    __shared__ int piv;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) M[e / n][e % n] = 0.0;
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        const Node a = unidx(r, v.Nx, v.Ny);
        const int NxNy = v.Nx * v.Ny;
        M[r][r] = v.A[0][r];
        if (a.i > 0) M[r][r - 1] = v.A[1][r];
        if (a.i < v.Nx - 1) M[r][r + 1] = v.A[2][r];
        if (a.j > 0) M[r][r - v.Nx] = v.A[3][r];
        if (a.j < v.Ny - 1) M[r][r + v.Nx] = v.A[4][r];
        if (a.l > 0) M[r][r - NxNy] = v.A[5][r];
        if (a.l < v.Nz - 1) M[r][r + NxNy] = v.A[6][r];
    }
    __syncthreads();
    // in-place Gauss-Jordan inversion with row interchanges (columns unswapped at the end)
    for (int c = 0; c < n; c++) {
        if (threadIdx.x == 0) {
            int p = c;
            double mx = fabs(M[c][c]);
            for (int r = c + 1; r < n; r++)
                if (fabs(M[r][c]) > mx) { mx = fabs(M[r][c]); p = r; }
            piv = p;
            perm[c] = p;
            if (!(mx > 1e-300)) M[p][c] = 1e-300;
        }
        __syncthreads();
        const int p = piv;
        if (p != c)
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                const double t = M[c][q]; M[c][q] = M[p][q]; M[p][q] = t;
            }
        __syncthreads();
        const double dg = M[c][c];
        __syncthreads();
        if (threadIdx.x == 0) M[c][c] = 1.0;
        __syncthreads();
        for (int q = threadIdx.x; q < n; q += blockDim.x) M[c][q] /= dg;
        __syncthreads();
        // eliminate column c from every other row: each thread owns whole rows
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            if (r == c) continue;
            const double fct = M[r][c];
            M[r][c] = 0.0;
            for (int q = 0; q < n; q++) M[r][q] -= fct * M[c][q];
        }
        __syncthreads();
    }
    for (int c = n - 1; c >= 0; c--) {
        const int p = perm[c];
        if (p != c)
            for (int r = threadIdx.x; r < n; r += blockDim.x) {
                const double t = M[r][c]; M[r][c] = M[r][p]; M[r][p] = t;
            }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, q = e % n;
        v.D[r * n + q] = M[r][q];
    }
}

// Slotboom weights of one level (semiconductor_3d.c:2092-2117): qsign 0 gives pw = 1
__device__ __forceinline__ double ph0(const DevP &P, int k, int qsign) {
    const uint32_t f = P.flags[k];
    if (fl_kind(f) != K_SEMI || fl_fix(f)) return PH_NONE;
    return qsign > 0 ? P.phin[k] / P.VTref : -P.phip[k] / P.VTref;
}
__global__ void k_mg_weights(const DevP *__restrict__ Ps, int L, int qsign) {
    const DevP &P = Ps[blockIdx.y];
    if (L >= P.nlev - 1) return;
    const LevView f = levview(P, L, 0, 0);
    const LevelT<double> &cl = P.lev[L + 1];
    SS_GRID_LOOP(K, cl.N) {
        const Node c = unidx(K, cl.Nx, cl.Ny);
        const Agg g = agg_range(f, c.i, c.j, c.l);
        if (qsign == 0) {
            for (int l = g.l0; l <= g.l1; l++)
                for (int j = g.j0; j <= g.j1; j++)
                    for (int i = g.i0; i <= g.i1; i++) f.pw[i + f.Nx * (j + f.Ny * l)] = 1.0;
            continue;
        }
        double mx = PH_NONE;
        for (int l = g.l0; l <= g.l1; l++)
            for (int j = g.j0; j <= g.j1; j++)
                for (int i = g.i0; i <= g.i1; i++) {
                    const int k = i + f.Nx * (j + f.Ny * l);
                    const double p = L == 0 ? ph0(P, k, qsign) : f.ph[k];
                    if (p > mx) mx = p;
                }
        cl.ph[K] = mx;
        for (int l = g.l0; l <= g.l1; l++)
            for (int j = g.j0; j <= g.j1; j++)
                for (int i = g.i0; i <= g.i1; i++) {
                    const int k = i + f.Nx * (j + f.Ny * l);
                    const double p = L == 0 ? ph0(P, k, qsign) : f.ph[k];
                    const double e = (p <= 0.5 * PH_NONE) ? -800.0 : p - mx;
                    f.pw[k] = e < -700.0 ? 0.0 : exp(e);
                }
    }
}

// Petrov-Galerkin coarse operator P^T W A P (semiconductor_3d.c:2003-2027)
__global__ void k_galerkin(const DevP *__restrict__ Ps, int L, int wsel) {
    const DevP &P = Ps[blockIdx.y];
    if (L >= P.nlev - 1) return;
    const LevView f = levview(P, L, 0, 0);
    const LevelT<double> &cl = P.lev[L + 1];
    const double *w = (L == 0 && wsel) ? P.dsc : nullptr;
    const int NxNy = f.Nx * f.Ny;
    SS_GRID_LOOP(K, cl.N) {
        const Node c = unidx(K, cl.Nx, cl.Ny);
        const Agg g = agg_range(f, c.i, c.j, c.l);
        double cc = 0, xm = 0, xp = 0, ym = 0, yp = 0, zm = 0, zp = 0;
        for (int l = g.l0; l <= g.l1; l++)
            for (int j = g.j0; j <= g.j1; j++)
                for (int i = g.i0; i <= g.i1; i++) {
                    const int k = i + f.Nx * (j + f.Ny * l);
                    const double wk = w ? w[k] : 1.0;
                    double a;
                    cc += wk * f.A[0][k] * f.pw[k];
                    if (i > 0) { a = wk * f.A[1][k] * f.pw[k - 1]; if (i - 1 >= g.i0) cc += a; else xm += a; }
                    if (i < f.Nx - 1) { a = wk * f.A[2][k] * f.pw[k + 1]; if (i + 1 <= g.i1) cc += a; else xp += a; }
                    if (j > 0) { a = wk * f.A[3][k] * f.pw[k - f.Nx]; if (j - 1 >= g.j0) cc += a; else ym += a; }
                    if (j < f.Ny - 1) { a = wk * f.A[4][k] * f.pw[k + f.Nx]; if (j + 1 <= g.j1) cc += a; else yp += a; }
                    if (l > 0) { a = wk * f.A[5][k] * f.pw[k - NxNy]; if (l - 1 >= g.l0) cc += a; else zm += a; }
                    if (l < f.Nz - 1) { a = wk * f.A[6][k] * f.pw[k + NxNy]; if (l + 1 <= g.l1) cc += a; else zp += a; }
                }
        if (cc == 0. && xm == 0. && xp == 0. && ym == 0. && yp == 0. && zm == 0. && zp == 0.) cc = 1.;
        cl.A[0][K] = cc; cl.A[1][K] = xm; cl.A[2][K] = xp; cl.A[3][K] = ym;
        cl.A[4][K] = yp; cl.A[5][K] = zm; cl.A[6][K] = zp;
    }
}

// ------------------------------------------------------------------ vector kernels
__global__ void k_absmax(const DevP *__restrict__ Ps, int xsel, int slot) {
    const DevP &P = Ps[blockIdx.y];
    const double *x = vsel(P, xsel);
    double m = 0.0;
    SS_GRID_LOOP(k, P.N) {
        const double a = fabs(x[k]);
        m = (a > m || a != a) ? a : m;
    }
    if (grid_max(m, P.part, P.ticket + 3)) P.res[slot] = m;
}
// y = x + a z  (selectors)
__global__ void k_axpy(const DevP *__restrict__ Ps, int ysel, int xsel, double a, int zsel) {
    const DevP &P = Ps[blockIdx.y];
    double *y = vsel(P, ysel);
    const double *x = vsel(P, xsel), *z = vsel(P, zsel);
    SS_GRID_LOOP(k, P.N) y[k] = x[k] + a * z[k];
}
__global__ void k_fill(const DevP *__restrict__ Ps, int ysel, double v) {
    const DevP &P = Ps[blockIdx.y];
    double *y = vsel(P, ysel);
    SS_GRID_LOOP(k, P.N) y[k] = v;
}
__global__ void k_copy(const DevP *__restrict__ Ps, int ysel, int xsel) {
    const DevP &P = Ps[blockIdx.y];
    double *y = vsel(P, ysel);
    const double *x = vsel(P, xsel);
    SS_GRID_LOOP(k, P.N) y[k] = x[k];
}

void launch_absmax_sel(const Ctx &c, int xsel, int slot) { SS_LAUNCH(PF_VEC, c.maxN, k_absmax, grid_nodes(c), TPB, c.st, c.dP, xsel, slot); }
void launch_axpy_sel(const Ctx &c, int ysel, int xsel, double a, int zsel) {
    SS_LAUNCH(PF_VEC, c.maxN, k_axpy, grid_nodes(c), TPB, c.st, c.dP, ysel, xsel, a, zsel);
}
void launch_fill_sel(const Ctx &c, int ysel, double v) { SS_LAUNCH(PF_VEC, c.maxN, k_fill, grid_nodes(c), TPB, c.st, c.dP, ysel, v); }
void launch_copy_sel(const Ctx &c, int ysel, int xsel) { SS_LAUNCH(PF_VEC, c.maxN, k_copy, grid_nodes(c), TPB, c.st, c.dP, ysel, xsel); }

// ------------------------------------------------------------------ multigrid driver
void mg_setup(const Ctx &c, const MGHost &mg, int qsign) {
    for (int L = 0; L < mg.maxlev - 1; L++) {
        const int nc = mg.maxN[L + 1];
        SS_LAUNCH(PF_WEIGHTS, nc, k_mg_weights, grid_n(c, nc), TPB, c.st, c.dP, L, qsign);
        SS_LAUNCH(PF_GALERKIN, nc, k_galerkin, grid_n(c, nc), TPB, c.st, c.dP, L, qsign != 0);
        SS_LAUNCH(PF_ILU_DIAG, mg.maxN[L], k_ilu_diag, grid_n(c, mg.maxN[L]), TPB, c.st, c.dP, L);
    }
    for (int L = 1; L < mg.maxlev; L++) SS_LAUNCH(PF_COARSE_SETUP, COARSE_MAX, k_coarse_setup, dim3(1, c.ninst), TPB, c.st, c.dP, L);
}

// one V(1,1) cycle x = M^-1 b on the level-0 vectors (bsel -> xsel); mg_on = 0 applies
// the level-0 smoother alone (the reference's ILU-only fallback).  gate: 0 always run,
// 1 only while the instance's Krylov loop is active, 2 also not after a half-step exit.
// ---- fine levels: one kernel per pass, all SMs
// Smoother half sweep over the nodes of one colour only: thread t of a row (j,l) takes
// i = 2t + ((j + l + colour) & 1), so every lane does work (colour 1 = black, 0 = red).
__global__ void k_smooth_c(const DevP *__restrict__ Ps, int L, int bsel, int xsel, int mode, int color, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if ((L > 0 && L >= P.nlev - 1) || (gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const LevView v = levview(P, L, bsel, xsel);
    const int hx = (v.Nx + 1) >> 1, rows = v.Ny * v.Nz;
    const double *src = mode ? v.r : v.b;
    const double *zb = mode ? v.r : v.x;
    SS_GRID_LOOP(t, hx * rows) {
        const int row = t / hx, ti = t - row * hx;
        const int l = row / v.Ny, j = row - l * v.Ny;
        const int i = 2 * ti + ((j + l + color) & 1);
        if (i >= v.Nx) continue;
        const int k = i + v.Nx * row;
        double z;
        if (mode == 2) {
            // a further application of the preconditioner right after a red-black one:
            // the residual of every red node is then zero, so black z = r / D with the
            // full-stencil residual, and red z = -(sum a_rb z_b) / D
            if (color) {
                z = (v.b[k] - stencil_apply<double>(v.A, v.x, k, i, j, l, v.Nx, v.Ny, v.Nz)) / v.D[k];
                v.x[k] += z;
                v.r[k] = z;
            } else {
                z = -offdiag_apply<double>(v.A, v.r, k, i, j, l, v.Nx, v.Ny, v.Nz) / v.D[k];
                v.x[k] += z;
            }
            continue;
        }
        if (color) {
            const double s = offdiag_apply_div<double>(v.A, src, v.D, k, i, j, l, v.Nx, v.Ny, v.Nz);
            z = (src[k] - s) / v.D[k];
            if (mode) { v.x[k] += z; v.r[k] = z; }
            else v.x[k] = z;
        } else {
            const double s = offdiag_apply<double>(v.A, zb, k, i, j, l, v.Nx, v.Ny, v.Nz);
            z = (src[k] - s) / v.D[k];
            if (mode) v.x[k] += z;
            else v.x[k] = z;
        }
    }
}

// Weighted residual of every fine node summed into its 2x2x2 aggregate.  Block (32, 4):
// threadIdx.x runs along fine x, threadIdx.y picks the (j, l) parity inside the coarse
// row blockIdx.z; pairs along x meet through a shuffle, the four parities through
// shared memory.  One thread per fine node (the restriction of semiconductor_3d.c:
// 2028-2037 applied to the residual of 1984-1991).
__global__ void __launch_bounds__(128) k_resid_restrict2(const DevP *__restrict__ Ps, int L, int bsel, int xsel,
                                                         int wsel, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if (L >= P.nlev - 1 || (gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const LevView f = levview(P, L, bsel, xsel);
    const LevelT<double> &cl = P.lev[L + 1];
    const double *w = (L == 0 && wsel) ? P.dsc : nullptr;
    const int R = blockIdx.z;                         // coarse row J + Cy*Lc
    const bool rowok = R < cl.Ny * cl.Nz;
    const int Lc = rowok ? R / cl.Ny : 0, Jc = rowok ? R - Lc * cl.Ny : 0;
    const int dj = threadIdx.y & 1, dl = threadIdx.y >> 1;
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = f.cy ? 2 * Jc + dj : Jc, l = f.cz ? 2 * Lc + dl : Lc;
    const bool ok = rowok && i < f.Nx && j < f.Ny && l < f.Nz && (f.cy || dj == 0) && (f.cz || dl == 0);
    double val = 0.0;
    if (ok) {
        const int k = i + f.Nx * (j + f.Ny * l);
        const double r = f.b[k] - stencil_apply<double>(f.A, f.x, k, i, j, l, f.Nx, f.Ny, f.Nz);
        val = w ? w[k] * r : r;
    }
    __shared__ double sh[4][32];
    sh[threadIdx.y][threadIdx.x] = val;
    __syncthreads();
    if (threadIdx.y == 0) {
        double s = sh[0][threadIdx.x] + sh[1][threadIdx.x] + sh[2][threadIdx.x] + sh[3][threadIdx.x];
        if (f.cx) {
            s += __shfl_down_sync(0xffffffffu, s, 1);
            if (rowok && !(threadIdx.x & 1) && i < f.Nx) cl.b[(i >> 1) + cl.Nx * R] = s;
        } else if (rowok && i < f.Nx) {
            cl.b[i + cl.Nx * R] = s;
        }
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

__device__ __forceinline__ void cta_smooth(const LevView &v, int color, int mode) {
    const double *src = mode ? v.r : v.b;
    const double *zb = mode ? v.r : v.x;
    const int hx = (v.Nx + 1) >> 1, rows = v.Ny * v.Nz;
    for (int t = cl_first(); t < hx * rows; t += cl_stride()) {
        const int row = t / hx, ti = t - row * hx;
        const int l = row / v.Ny, j = row - l * v.Ny;
        const int i = 2 * ti + ((j + l + color) & 1);
        if (i >= v.Nx) continue;
        const int k = i + v.Nx * row;
        if (color) {
            const double s = offdiag_apply_div<double>(v.A, src, v.D, k, i, j, l, v.Nx, v.Ny, v.Nz);
            const double z = (src[k] - s) / v.D[k];
            if (mode) { v.x[k] += z; v.r[k] = z; }
            else v.x[k] = z;
        } else {
            const double s = offdiag_apply<double>(v.A, zb, k, i, j, l, v.Nx, v.Ny, v.Nz);
            const double z = (src[k] - s) / v.D[k];
            if (mode) v.x[k] += z;
            else v.x[k] = z;
        }
    }
    cl_sync();
}
__device__ __forceinline__ void cta_resid_restrict(const LevView &f, const LevelT<double> &cl, const double *w) {
    for (int K = cl_first(); K < cl.N; K += cl_stride()) {
        const Node c = unidx(K, cl.Nx, cl.Ny);
        const Agg g = agg_range(f, c.i, c.j, c.l);
        double s = 0.0;
        for (int l = g.l0; l <= g.l1; l++)
            for (int j = g.j0; j <= g.j1; j++)
                for (int i = g.i0; i <= g.i1; i++) {
                    const int k = i + f.Nx * (j + f.Ny * l);
                    const double r = f.b[k] - stencil_apply<double>(f.A, f.x, k, i, j, l, f.Nx, f.Ny, f.Nz);
                    s += w ? w[k] * r : r;
                }
        cl.b[K] = s;
    }
    cl_sync();
}
__device__ __forceinline__ void cta_prolong(const LevView &f, const LevelT<double> &cl, double alpha) {
    for (int k = cl_first(); k < f.N; k += cl_stride()) {
        const Node a = unidx(k, f.Nx, f.Ny);
        const int I = f.cx ? a.i >> 1 : a.i, J = f.cy ? a.j >> 1 : a.j, K = f.cz ? a.l >> 1 : a.l;
        f.x[k] += alpha * f.pw[k] * cl.x[I + cl.Nx * (J + cl.Ny * K)];
    }
    cl_sync();
}
__device__ __forceinline__ void cta_resid(const LevView &f) {
    for (int k = cl_first(); k < f.N; k += cl_stride()) {
        const Node a = unidx(k, f.Nx, f.Ny);
        f.r[k] = f.b[k] - stencil_apply<double>(f.A, f.x, k, a.i, a.j, a.l, f.Nx, f.Ny, f.Nz);
    }
    cl_sync();
}
__device__ __forceinline__ void cta_dense(const LevelT<double> &v) {
    const int n = v.N;
    for (int r = cl_first(); r < n; r += cl_stride()) {
        double s = 0.0;
        for (int q = 0; q < n; q++) s += v.D[r * n + q] * v.b[q];
        v.x[r] = s;
    }
    cl_sync();
}

constexpr int SMALL_TPB = 1024;
__global__ void __launch_bounds__(SMALL_TPB) k_vcycle_small(const DevP *__restrict__ Ps, int Ls, int bsel, int xsel,
                                                            int wsel, double alpha, int gate) {
    const DevP &P = Ps[blockIdx.y];
    if ((gate && !ks_running(P)) || (gate == 2 && P.ks->half)) return;
    const int nl = P.nlev;
    if (nl == 1) {                                 // a single level: the smoother alone
        const LevView v = levview(P, 0, bsel, xsel);
        cta_smooth(v, 1, 0);
        cta_smooth(v, 0, 0);
        return;
    }
    for (int L = Ls; L < nl - 1; L++) {
        const LevView v = levview(P, L, bsel, xsel);
        cta_smooth(v, 1, 0);
        cta_smooth(v, 0, 0);
        cta_resid_restrict(v, P.lev[L + 1], (L == 0 && wsel) ? P.dsc : nullptr);
    }
    cta_dense(P.lev[nl - 1]);
    for (int L = nl - 2; L >= Ls; L--) {
        const LevView v = levview(P, L, bsel, xsel);
        cta_prolong(v, P.lev[L + 1], alpha);
        cta_resid(v);
        cta_smooth(v, 1, 1);
        cta_smooth(v, 0, 1);
    }
}

int g_small_nodes = 2048;           // levels at or below this size run in the cluster kernel
int g_l0_sweeps = 2;                // red-black applications per smoothing step on the finest level
static int g_cluster = 0;           // CTAs per cluster of the small-level kernel (set on first use)

// cluster size of the small-level kernel (16 CTAs when the device allows non-portable
// clusters of 16, else 8) and the size split, read once (SEMISIM_B200_CLUSTER / _SMALL)
static void small_init() {
    if (!g_cluster) {
        const char *e = std::getenv("SEMISIM_B200_CLUSTER");
        g_cluster = (e && std::atoi(e) == 8) ? 8 : 16;
        if (const char *s = std::getenv("SEMISIM_B200_SMALL")) g_small_nodes = std::atoi(s);
        if (const char *s = std::getenv("SEMISIM_B200_L0SWEEPS")) g_l0_sweeps = std::atoi(s) > 1 ? 2 : 1;
        if (cudaFuncSetAttribute(k_vcycle_small, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
            g_cluster = 8;
        cudaGetLastError();
        cudaLaunchConfig_t q = {};
        q.gridDim = dim3(g_cluster, 1);
        q.blockDim = dim3(SMALL_TPB);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = g_cluster; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        q.attrs = at;
        q.numAttrs = 1;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, k_vcycle_small, &q) != cudaSuccess || ncl < 1) g_cluster = 8;
        cudaGetLastError();
    }
}

// launch the small-level V-cycle as clusters of g_cluster CTAs, one cluster per instance
static void launch_small(const Ctx &c, int nodes, int Ls, int bsel, int xsel, int wsel, double alpha, int gate) {
    small_init();
    g_launches++;
    t_launches++;
    if (g_prof_on) prof_begin(PF_COARSE, c.st);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g_cluster, c.ninst);
    cfg.blockDim = dim3(SMALL_TPB);
    cfg.stream = c.st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = g_cluster; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_vcycle_small, c.dP, Ls, bsel, xsel, wsel, alpha, gate);
    if (g_prof_on) prof_end(PF_COARSE, c.st, nodes);
}

static inline dim3 grid_half(const Ctx &c, int L, const MGHost &mg) {
    return grid_n(c, ((mg.maxNx[L] + 1) / 2) * (mg.maxN[L] / (mg.maxNx[L] > 0 ? mg.maxNx[L] : 1)));
}

void vcycle(const Ctx &c, const MGHost &mg, int bsel, int xsel, int wsel, int mg_on, int gate) {
    if (!mg_on) {
        SS_LAUNCH(PF_SMOOTH_B, c.maxN, k_smooth_c, grid_half(c, 0, mg), TPB, c.st, c.dP, 0, bsel, xsel, 0, 1, gate);
        SS_LAUNCH(PF_SMOOTH_R, c.maxN, k_smooth_c, grid_half(c, 0, mg), TPB, c.st, c.dP, 0, bsel, xsel, 0, 0, gate);
        return;
    }
    small_init();
    int Ls = 0;
    while (Ls < mg.maxlev - 1 && mg.maxN[Ls] > g_small_nodes) Ls++;
    for (int L = 0; L < Ls; L++) {
        SS_LAUNCH(PF_SMOOTH_B, mg.maxN[L], k_smooth_c, grid_half(c, L, mg), TPB, c.st, c.dP, L, bsel, xsel, 0, 1, gate);
        SS_LAUNCH(PF_SMOOTH_R, mg.maxN[L], k_smooth_c, grid_half(c, L, mg), TPB, c.st, c.dP, L, bsel, xsel, 0, 0, gate);
        if (L == 0 && g_l0_sweeps > 1) {     // second application on the finest level
            SS_LAUNCH(PF_SMOOTH_B, mg.maxN[L], k_smooth_c, grid_half(c, L, mg), TPB, c.st, c.dP, L, bsel, xsel, 2, 1, gate);
            SS_LAUNCH(PF_SMOOTH_R, mg.maxN[L], k_smooth_c, grid_half(c, L, mg), TPB, c.st, c.dP, L, bsel, xsel, 2, 0, gate);
        }
        const dim3 gr((mg.maxNx[L] + 31) / 32, c.ninst, mg.maxRows[L + 1]);
        SS_LAUNCH(PF_RESID_RESTRICT, mg.maxN[L + 1], k_resid_restrict2, gr, dim3(32, 4), c.st, c.dP, L, bsel, xsel, wsel, gate);
    }
    launch_small(c, mg.maxN[Ls], Ls, bsel, xsel, wsel, mg.alpha, gate);
    for (int L = Ls - 1; L >= 0; L--) {
        SS_LAUNCH(PF_PROLONG, mg.maxN[L], k_prolong, grid_n(c, mg.maxN[L]), TPB, c.st, c.dP, L, bsel, xsel, mg.alpha, gate);
        SS_LAUNCH(PF_LEVEL_RESID, mg.maxN[L], k_level_resid, grid_n(c, mg.maxN[L]), TPB, c.st, c.dP, L, bsel, xsel, gate);
        SS_LAUNCH(PF_SMOOTH_B, mg.maxN[L], k_smooth_c, grid_half(c, L, mg), TPB, c.st, c.dP, L, bsel, xsel, 1, 1, gate);
        SS_LAUNCH(PF_SMOOTH_R, mg.maxN[L], k_smooth_c, grid_half(c, L, mg), TPB, c.st, c.dP, L, bsel, xsel, 1, 0, gate);
        if (L == 0 && g_l0_sweeps > 1) {
            SS_LAUNCH(PF_SMOOTH_B, mg.maxN[L], k_smooth_c, grid_half(c, L, mg), TPB, c.st, c.dP, L, bsel, xsel, 2, 1, gate);
            SS_LAUNCH(PF_SMOOTH_R, mg.maxN[L], k_smooth_c, grid_half(c, L, mg), TPB, c.st, c.dP, L, bsel, xsel, 2, 0, gate);
        }
    }
}

__global__ void k_bicg_v(const DevP *__restrict__ Ps);
__global__ void k_bicg_x(const DevP *__restrict__ Ps);
__global__ void k_bicg_rho(const DevP *__restrict__ Ps);

// Time `reps` launches of one kernel of the solve path on the instance's present state
// (test hook for per-kernel roofline numbers; it overwrites work vectors).  Returns
// microseconds per launch.
double bench_la_kernel(const Ctx &c, const MGHost &mg, int which, int reps) {
    KrylovS ks0{};
    ks0.active = 1;
    ks0.maxit = 1 << 30;
    cudaMemcpy(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice);
    small_init();
    int Ls = 0;
    while (Ls < mg.maxlev - 1 && mg.maxN[Ls] > g_small_nodes) Ls++;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    auto one = [&]() {
        switch (which) {
        case 0: k_bicg_v<<<grid_nodes(c), TPB, 0, c.st>>>(c.dP); break;
        case 1: k_smooth_c<<<grid_half(c, 0, mg), TPB, 0, c.st>>>(c.dP, 0, 2, 4, 0, 1, 0); break;
        case 2: k_smooth_c<<<grid_half(c, 0, mg), TPB, 0, c.st>>>(c.dP, 0, 2, 4, 0, 0, 0); break;
        case 3: k_resid_restrict2<<<dim3((mg.maxNx[0] + 31) / 32, c.ninst, mg.maxRows[1]), dim3(32, 4), 0, c.st>>>(
                    c.dP, 0, 2, 4, 1, 0); break;
        case 4: k_level_resid<<<grid_nodes(c), TPB, 0, c.st>>>(c.dP, 0, 2, 4, 0); break;
        case 5: k_prolong<<<grid_nodes(c), TPB, 0, c.st>>>(c.dP, 0, 2, 4, 1.0, 0); break;
        case 6: k_bicg_x<<<grid_nodes(c), TPB, 0, c.st>>>(c.dP); break;
        case 7: launch_small(c, mg.maxN[Ls], Ls, 2, 4, 1, 1.0, 0); break;
        case 8: vcycle(c, mg, 2, 4, 1, 1, 0); break;
        case 9: k_copy<<<grid_nodes(c), TPB, 0, c.st>>>(c.dP, 5, 6); break;
        case 10: k_bicg_rho<<<grid_nodes(c), TPB, 0, c.st>>>(c.dP); break;
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

// ------------------------------------------------------------------ PCG (semiconductor_3d.c:2182-2210)
// r = b - A x; z = M r; rz = r.z
__global__ void k_pcg_init_r(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    const double *b = P.rhs, *x = P.sol;
    double *r = P.wk[0];
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        r[k] = b[k] - stencil_apply<double>(P.A, x, k, a.i, a.j, a.l, P.Nx, P.Ny, P.Nz);
    }
}
// rz = r.z; mode 0 initial (rz0), mode 1 iteration end (stop test, beta)
__global__ void k_pcg_rz(const DevP *__restrict__ Ps, int mode) {
    const DevP &P = Ps[blockIdx.y];
    if (mode && !ks_running(P)) return;
    const double *r = P.wk[0], *z = P.wk[1];
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) acc[0] += r[k] * z[k];
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
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
__global__ void k_pcg_p(const DevP *__restrict__ Ps, int init) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P)) return;
    const double be = init ? 0.0 : P.ks->be;
    double *p = P.wk[2];
    const double *z = P.wk[1];
    SS_GRID_LOOP(k, P.N) p[k] = z[k] + (init ? 0.0 : be * p[k]);
}
// q = A p; pq = p.q; al = rz / pq
__global__ void k_pcg_q(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P)) return;
    const double *p = P.wk[2];
    double *q = P.wk[3];
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const double v = stencil_apply<double>(P.A, p, k, a.i, a.j, a.l, P.Nx, P.Ny, P.Nz);
        q[k] = v;
        acc[0] += p[k] * v;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 5)) {
        KrylovS &s = *P.ks;
        s.it++;
        const double pq = acc[0];
        if (!(pq > 0.0)) { s.active = 0; s.status = 2; s.al = 0.0; }
        else s.al = s.rz / pq;
    }
}
// x += al p; r -= al q
__global__ void k_pcg_xr(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P)) return;
    const double al = P.ks->al;
    double *x = P.sol, *r = P.wk[0];
    const double *p = P.wk[2], *q = P.wk[3];
    SS_GRID_LOOP(k, P.N) { x[k] += al * p[k]; r[k] -= al * q[k]; }
}

// one PCG iteration (every kernel gated on the instance's active word)
static void pcg_body(const Ctx &c, const MGHost &mg) {
    SS_LAUNCH(PF_KRY_SPMV_DOT, c.maxN, k_pcg_q, grid_nodes(c), TPB, c.st, c.dP);
    SS_LAUNCH(PF_KRY_UPDATE, c.maxN, k_pcg_xr, grid_nodes(c), TPB, c.st, c.dP);
    vcycle(c, mg, 0, 1, 0, 1, 1);
    SS_LAUNCH(PF_KRY_DOT, c.maxN, k_pcg_rz, grid_nodes(c), TPB, c.st, c.dP, 1);
    SS_LAUNCH(PF_KRY_UPDATE, c.maxN, k_pcg_p, grid_nodes(c), TPB, c.st, c.dP, 0);
}
static void bicg_body(const Ctx &c, const MGHost &mg, int mg_on);

// ------------------------------------------------------------------ device-looped solves
// A Krylov solve runs as one CUDA graph: a conditional WHILE node whose body is one
// iteration; the body's last kernel sets the loop condition from the instances' active
// words, so the iteration loop runs on the device with no host round trip.
__global__ void k_loop_cond(const DevP *__restrict__ Ps, int ninst, cudaGraphConditionalHandle h, int body) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned any = 0;
    for (int i = 0; i < ninst; i++) {
        KrylovS *s = Ps[i].ks;
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

// kind 0: PCG; 1: BiCGSTAB with the multigrid preconditioner; 2: BiCGSTAB, smoother only
static cudaGraphExec_t build_loop(const Ctx &c, const MGHost &mg, int kind, int *nkern) {
    cudaGraph_t g = nullptr;
    GCK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    GCK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    const DevP *dp = c.dP;
    int ninst = c.ninst, body0 = 0;
    void *args[] = {(void *)&dp, (void *)&ninst, (void *)&h, (void *)&body0};
    cudaKernelNodeParams kp = {};
    kp.func = (void *)k_loop_cond;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = args;
    cudaGraphNode_t n0, cn;
    GCK(cudaGraphAddKernelNode(&n0, g, nullptr, 0, &kp));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    GCK(cudaGraphAddNode(&cn, g, &n0, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    GCK(cudaStreamBeginCaptureToGraph(c.st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    const unsigned long long l0 = t_launches;
    if (kind == 0) pcg_body(c, mg);
    else bicg_body(c, mg, kind == 1);
    k_loop_cond<<<1, 32, 0, c.st>>>(c.dP, c.ninst, h, 1);
    const unsigned long long nb = t_launches - l0;
    *nkern = int(nb) + 1;
    g_launches -= nb;                                  // counted per executed body instead
    t_launches = l0;
    cudaGraph_t out = nullptr;
    GCK(cudaStreamEndCapture(c.st, &out));
    cudaGraphExec_t ex = nullptr;
    GCK(cudaGraphInstantiate(&ex, g, 0));
    cudaGraphDestroy(g);
    return ex;
}

bool g_use_graphs = true;

// run the iteration loop of `kind` to completion; returns the final Krylov record
static KrylovS run_loop(const Ctx &c, const MGHost &mg, int kind, int maxit, int check_every) {
    KrylovS hs{};
    LoopGraphs *lg = c.lg;
    if (lg && g_use_graphs && !g_prof_on && !lg->failed) {
        if (!lg->exec[kind]) {
            lg->exec[kind] = build_loop(c, mg, kind, &lg->kernels[kind]);
            if (!lg->exec[kind]) lg->failed = 1;
        }
        if (lg->exec[kind]) {
            cudaGraphLaunch(lg->exec[kind], c.st);
            cudaMemcpyAsync(&hs, c.h.ks, sizeof(KrylovS), cudaMemcpyDeviceToHost, c.st);
            cudaStreamSynchronize(c.st);
            const unsigned long long ran = 1ull + (unsigned long long)lg->kernels[kind] * (unsigned long long)hs.body_runs;
            g_launches += ran;
            t_launches += ran;
            return hs;
        }
    }
    for (int it = 0; it < maxit + 1;) {
        for (int q = 0; q < check_every && it < maxit + 1; q++, it++) {
            if (kind == 0) pcg_body(c, mg);
            else bicg_body(c, mg, kind == 1);
        }
        cudaMemcpyAsync(&hs, c.h.ks, sizeof(KrylovS), cudaMemcpyDeviceToHost, c.st);
        cudaStreamSynchronize(c.st);
        if (!hs.active) break;
    }
    return hs;
}

int pcg_solve(const Ctx &c, const MGHost &mg, int maxit, double rtol, int check_every) {
    KrylovS ks0{};
    ks0.active = 1;
    ks0.maxit = maxit;
    ks0.rtol = rtol;
    cudaMemcpyAsync(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
    mg_setup(c, mg, 0);
    SS_LAUNCH(PF_KRY_INIT, c.maxN, k_pcg_init_r, grid_nodes(c), TPB, c.st, c.dP);
    vcycle(c, mg, 0, 1, 0, 1, 0);                  // z = M r
    SS_LAUNCH(PF_KRY_DOT, c.maxN, k_pcg_rz, grid_nodes(c), TPB, c.st, c.dP, 0);
    SS_LAUNCH(PF_KRY_UPDATE, c.maxN, k_pcg_p, grid_nodes(c), TPB, c.st, c.dP, 1);
    const KrylovS hs = run_loop(c, mg, 0, maxit, check_every);
    return hs.it;
}

// ------------------------------------------------------------------ BiCGSTAB (semiconductor_3d.c:2216-2320)
// work vectors: 0 r, 1 rh, 2 p, 3 v, 4 ph, 5 sh, 6 t, 7 x0 (start backup)
// r = b - A x; rh = r; p = v = 0; rr = r.r; fl = sum (sum|A x| + |b|)^2; tgt
__global__ void k_bicg_init(const DevP *__restrict__ Ps, double rtol, double atol) {
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
__global__ void k_bicg_rho(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P)) return;
    const double *r = P.wk[0], *rh = P.wk[1];
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) acc[0] += rh[k] * r[k];
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
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
__global__ void k_bicg_p(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P)) return;
    const KrylovS &s = *P.ks;
    const double be = s.be, om = s.om;
    const int restart = s.pad0;
    double *p = P.wk[2], *v = P.wk[3], *rh = P.wk[1];
    const double *r = P.wk[0];
    SS_GRID_LOOP(k, P.N) {
        if (restart) { rh[k] = r[k]; p[k] = r[k]; v[k] = 0.0; }
        else p[k] = r[k] + be * (p[k] - om * v[k]);
    }
}
// v = A ph; rv = rh.v; al
__global__ void k_bicg_v(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P)) return;
    const double *ph = P.wk[4], *rh = P.wk[1];
    double *v = P.wk[3];
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const double t = stencil_apply<double>(P.A, ph, k, a.i, a.j, a.l, P.Nx, P.Ny, P.Nz);
        v[k] = t;
        acc[0] += rh[k] * t;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
        if (fabs(acc[0]) < 1e-300) { s.active = 0; s.status = 2; return; }
        s.rv = acc[0];
        s.al = s.rho1 / acc[0];
    }
}
// r -= al v; ss = r.r; half-step exit test
__global__ void k_bicg_s(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P)) return;
    const double al = P.ks->al;
    double *r = P.wk[0];
    const double *v = P.wk[3];
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const double t = r[k] - al * v[k];
        r[k] = t;
        acc[0] += t * t;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
        s.ss = acc[0];
        if (sqrt(acc[0]) <= s.tgt) { s.half = 1; s.rr = acc[0]; }
    }
}
// t = A sh; tt = t.t; ts = t.r; om
__global__ void k_bicg_t(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P) || P.ks->half) return;
    const double *sh = P.wk[5], *r = P.wk[0];
    double *t = P.wk[6];
    double acc[2] = {0.0, 0.0};
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        const double q = stencil_apply<double>(P.A, sh, k, a.i, a.j, a.l, P.Nx, P.Ny, P.Nz);
        t[k] = q;
        acc[0] += q * q;
        acc[1] += q * r[k];
    }
    if (grid_sum<2>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
        s.tt = acc[0]; s.ts = acc[1];
        s.om = acc[0] > 0.0 ? acc[1] / acc[0] : 0.0;
    }
}
// x += al ph + om sh; r -= om t; rr = r.r; stop tests (or the half-step x update)
__global__ void k_bicg_x(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!ks_running(P)) return;
    const KrylovS &s0 = *P.ks;
    const double al = s0.al, om = s0.om;
    const int half = s0.half;
    double *x = P.sol, *r = P.wk[0];
    const double *ph = P.wk[4], *sh = P.wk[5], *t = P.wk[6];
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        if (half) { x[k] += al * ph[k]; continue; }
        x[k] += al * ph[k] + om * sh[k];
        const double q = r[k] - om * t[k];
        r[k] = q;
        acc[0] += q * q;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 4)) {
        KrylovS &s = *P.ks;
        if (half) { s.active = 0; s.status = 1; return; }
        s.rr = acc[0];
        const double rn = sqrt(acc[0]);
        if (rn <= s.tgt || s.om == 0.0) { s.active = 0; s.status = 1; return; }
        if (rn < 0.99 * s.rbest) { s.rbest = rn; s.stall = 0; }
        else if (++s.stall > 40) { s.active = 0; s.status = 2; return; }
        s.rho = s.rho1;
    }
}

// One BiCGSTAB solve of P.A sol = rhs from the present sol.  Returns the iterations;
// rn / r0 the final and initial residual norms.
// one BiCGSTAB iteration (the continuity systems use the Slotboom-weighted hierarchy)
static void bicg_body(const Ctx &c, const MGHost &mg, int mg_on) {
    SS_LAUNCH(PF_KRY_DOT, c.maxN, k_bicg_rho, grid_nodes(c), TPB, c.st, c.dP);
    SS_LAUNCH(PF_KRY_UPDATE, c.maxN, k_bicg_p, grid_nodes(c), TPB, c.st, c.dP);
    vcycle(c, mg, 2, 4, 1, mg_on, 1);            // ph = M p
    SS_LAUNCH(PF_KRY_SPMV_DOT, c.maxN, k_bicg_v, grid_nodes(c), TPB, c.st, c.dP);
    SS_LAUNCH(PF_KRY_UPDATE, c.maxN, k_bicg_s, grid_nodes(c), TPB, c.st, c.dP);
    vcycle(c, mg, 0, 5, 1, mg_on, 2);            // sh = M r
    SS_LAUNCH(PF_KRY_SPMV_DOT, c.maxN, k_bicg_t, grid_nodes(c), TPB, c.st, c.dP);
    SS_LAUNCH(PF_KRY_UPDATE, c.maxN, k_bicg_x, grid_nodes(c), TPB, c.st, c.dP);
}

// One BiCGSTAB solve of P.A sol = rhs from the present sol.  Returns the iterations;
// rn / r0 the final and initial residual norms.
int bicgstab_core(const Ctx &c, const MGHost &mg, int maxit, double rtol, double atol, int mg_on, int check_every,
                  double *rn, double *r0, int qsign) {
    KrylovS ks0{};
    ks0.maxit = maxit;
    ks0.rtol = rtol;
    ks0.atol = atol;
    cudaMemcpyAsync(c.h.ks, &ks0, sizeof(KrylovS), cudaMemcpyHostToDevice, c.st);
    if (mg_on) mg_setup(c, mg, qsign);
    else {
        SS_LAUNCH(PF_ILU_DIAG, c.maxN, k_ilu_diag, grid_nodes(c), TPB, c.st, c.dP, 0);
    }
    SS_LAUNCH(PF_KRY_INIT, c.maxN, k_bicg_init, grid_nodes(c), TPB, c.st, c.dP, rtol, atol);
    const KrylovS hs = run_loop(c, mg, mg_on ? 1 : 2, maxit, check_every);
    *rn = sqrt(hs.rr);
    *r0 = hs.r0;
    return hs.it;
}

}  // namespace ss
