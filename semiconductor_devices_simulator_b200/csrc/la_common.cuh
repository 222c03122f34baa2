// Device helpers of the 7-point multigrid and Krylov kernels, shared by the per-pass
// kernels (kernels_la.cu) and the persistent solve kernels (kernels_persist.cu): where
// each precision's vectors and hierarchy live in an instance record, level views, the
// stencil products, the 2x2x2 aggregate ranges, the red-black D-ILU smoother update of
// one node, and the shared-memory layout of the small levels.
#pragma once
#include <type_traits>

#include "device_common.cuh"
#include "kernels.h"
#include "solver_ctx.h"

namespace ss {

// ------------------------------------------------------------------ precision traits
// where the level-0 system, the Krylov vectors, the hierarchy and the Krylov record of
// each precision live in an instance's parameter record
template <class T> struct PT;
template <> struct PT<double> {
    static __device__ __forceinline__ double *wk(const DevP &P, int s) { return P.wk[s]; }
    static __device__ __forceinline__ double *sol(const DevP &P) { return P.sol; }
    static __device__ __forceinline__ double *rhs(const DevP &P) { return P.rhs; }
    static __device__ __forceinline__ double *const *A0(const DevP &P) { return P.A; }
    static __device__ __forceinline__ const double *w0(const DevP &P) { return P.dsc; }
    static __device__ __forceinline__ const LevelT<double> &lev(const DevP &P, int L) { return P.lev[L]; }
    static __device__ __forceinline__ KrylovS *ks(const DevP &P) { return P.ks; }
};
template <> struct PT<float> {
    static __device__ __forceinline__ float *wk(const DevP &P, int s) { return P.wk32[s]; }
    static __device__ __forceinline__ float *sol(const DevP &P) { return P.sol32; }
    static __device__ __forceinline__ float *rhs(const DevP &P) { return P.rhs32; }
    static __device__ __forceinline__ float *const *A0(const DevP &P) { return P.A32; }
    static __device__ __forceinline__ const float *w0(const DevP &P) { return P.dsc32; }
    static __device__ __forceinline__ const LevelT<float> &lev(const DevP &P, int L) { return P.levf[L]; }
    static __device__ __forceinline__ KrylovS *ks(const DevP &P) { return P.ksi; }
};

// vector selectors of the level-0 vectors (0-7 Krylov work vectors; the FP32 side has
// the work vectors, rhs and sol only)
template <class T>
__device__ __forceinline__ T *vsel(const DevP &P, int s) {
    if (s < 8) return PT<T>::wk(P, s);
    if constexpr (std::is_same<T, double>::value) {
        switch (s) {
        case V_RHS: return P.rhs;
        case V_SOL: return P.sol;
        case V_F: return P.F;
        case V_TR: return P.tr;
        case V_PHI: return P.phi;
        default: return P.dsc;
        }
    } else {
        return s == V_RHS ? P.rhs32 : P.sol32;
    }
}

// y = A x on a level (7-point, boundary terms skipped as in semiconductor_3d.c:1975-1993)
template <class T>
__device__ __forceinline__ T stencil_apply(T *const *A, const T *x, int k, int i, int j, int l, int Nx, int Ny, int Nz) {
    const int NxNy = Nx * Ny;
    T s = A[0][k] * x[k];
    if (i > 0) s += A[1][k] * x[k - 1];
    if (i < Nx - 1) s += A[2][k] * x[k + 1];
    if (j > 0) s += A[3][k] * x[k - Nx];
    if (j < Ny - 1) s += A[4][k] * x[k + Nx];
    if (l > 0) s += A[5][k] * x[k - NxNy];
    if (l < Nz - 1) s += A[6][k] * x[k + NxNy];
    return s;
}
// ------------------------------------------------------------------ multigrid levels
// level accessors: level 0 reads the instance's system arrays and the caller's vectors
template <class T>
struct LevView {
    const T *A;                  // coupling q of node k at A[q * ap + k] (q: c, xm, xp, ym, yp, zm, zp)
    T *D, *x, *b, *r, *pw;       // D: reciprocal smoother pivots
    double *ph;
    int ap, Nx, Ny, Nz, N, cx, cy, cz, last;
    __device__ __forceinline__ T a(int q, int k) const { return A[q * ap + k]; }
};
template <class T>
__device__ __forceinline__ LevView<T> levview(const DevP &P, int L, int bsel, int xsel) {
    const LevelT<T> &lv = PT<T>::lev(P, L);
    LevView<T> v;
    v.A = lv.A[0];
    v.ap = lv.apitch;
    v.D = lv.D; v.r = lv.r; v.pw = lv.pw; v.ph = lv.ph;
    v.x = L == 0 ? vsel<T>(P, xsel) : lv.x;
    v.b = L == 0 ? vsel<T>(P, bsel) : lv.b;
    v.Nx = lv.Nx; v.Ny = lv.Ny; v.Nz = lv.Nz; v.N = lv.N;
    v.cx = lv.cx; v.cy = lv.cy; v.cz = lv.cz; v.last = lv.last;
    return v;
}
// y = A x at node k = (i, j, l) of a level
template <class T>
__device__ __forceinline__ T lv_apply(const LevView<T> &v, const T *x, int k, int i, int j, int l) {
    const int NxNy = v.Nx * v.Ny;
    T s = v.a(0, k) * x[k];
    if (i > 0) s += v.a(1, k) * x[k - 1];
    if (i < v.Nx - 1) s += v.a(2, k) * x[k + 1];
    if (j > 0) s += v.a(3, k) * x[k - v.Nx];
    if (j < v.Ny - 1) s += v.a(4, k) * x[k + v.Nx];
    if (l > 0) s += v.a(5, k) * x[k - NxNy];
    if (l < v.Nz - 1) s += v.a(6, k) * x[k + NxNy];
    return s;
}
// sum over the off-diagonal couplings only
template <class T>
__device__ __forceinline__ T lv_offdiag(const LevView<T> &v, const T *x, int k, int i, int j, int l) {
    const int NxNy = v.Nx * v.Ny;
    T s = 0;
    if (i > 0) s += v.a(1, k) * x[k - 1];
    if (i < v.Nx - 1) s += v.a(2, k) * x[k + 1];
    if (j > 0) s += v.a(3, k) * x[k - v.Nx];
    if (j < v.Ny - 1) s += v.a(4, k) * x[k + v.Nx];
    if (l > 0) s += v.a(5, k) * x[k - NxNy];
    if (l < v.Nz - 1) s += v.a(6, k) * x[k + NxNy];
    return s;
}
// sum of a_kj x_j / D_j over the neighbours (forward sweep of the black rows), with the
// reciprocal pivots
template <class T>
__device__ __forceinline__ T lv_offdiag_scaled(const LevView<T> &v, const T *x, int k, int i, int j, int l) {
    const int NxNy = v.Nx * v.Ny;
    T s = 0;
    if (i > 0) s += v.a(1, k) * (x[k - 1] * v.D[k - 1]);
    if (i < v.Nx - 1) s += v.a(2, k) * (x[k + 1] * v.D[k + 1]);
    if (j > 0) s += v.a(3, k) * (x[k - v.Nx] * v.D[k - v.Nx]);
    if (j < v.Ny - 1) s += v.a(4, k) * (x[k + v.Nx] * v.D[k + v.Nx]);
    if (l > 0) s += v.a(5, k) * (x[k - NxNy] * v.D[k - NxNy]);
    if (l < v.Nz - 1) s += v.a(6, k) * (x[k + NxNy] * v.D[k + NxNy]);
    return s;
}

template <class T>
__device__ __forceinline__ bool ks_running(const DevP &P) { return PT<T>::ks(P)->active != 0; }
// gate 0: always run; 1: only while the instance's Krylov loop (of precision T) is
// active; 2: also not after a half-step exit
template <class T>
__device__ __forceinline__ bool gated_off(const DevP &P, int gate) {
    if (!gate) return false;
    const KrylovS *s = PT<T>::ks(P);
    return !s->active || (gate == 2 && s->half);
}


// coarse aggregate (I,J,L) -> fine index range (AGG_RANGE, semiconductor_3d.c:1996-1999)
struct Agg { int i0, i1, j0, j1, l0, l1; };
template <class V>
__device__ __forceinline__ Agg agg_range(const V &f, int I, int J, int K) {
    Agg g;
    g.i0 = f.cx ? 2 * I : I; g.i1 = f.cx ? 2 * I + 1 : I; if (g.i1 > f.Nx - 1) g.i1 = f.Nx - 1;
    g.j0 = f.cy ? 2 * J : J; g.j1 = f.cy ? 2 * J + 1 : J; if (g.j1 > f.Ny - 1) g.j1 = f.Ny - 1;
    g.l0 = f.cz ? 2 * K : K; g.l1 = f.cz ? 2 * K + 1 : K; if (g.l1 > f.Nz - 1) g.l1 = f.Nz - 1;
    return g;
}


// Smoother update of node k = (i, j, l) in a half sweep over one colour (1 = black,
// 0 = red), with D the reciprocal pivots.  mode 0: pre-smoothing from x = 0,
// x = M^-1 b.  mode 1: post-smoothing, z = M^-1 r with r the level's residual array,
// x += z (the black z is parked in r for the red sweep).  mode 2: a further application
// right after a red-black one: the residual of every red node is then zero, so black
// z = r / D with the full-stencil residual, and red z = -(sum a_rb z_b) / D.
template <class T>
__device__ __forceinline__ void smooth_node(const LevView<T> &v, int k, int i, int j, int l, int mode, int color) {
    if (mode == 2) {
        if (color) {
            const T z = (v.b[k] - lv_apply<T>(v, v.x, k, i, j, l)) * v.D[k];
            v.x[k] += z;
            v.r[k] = z;
        } else {
            v.x[k] -= lv_offdiag<T>(v, v.r, k, i, j, l) * v.D[k];
        }
        return;
    }
    const T *src = mode ? v.r : v.b;
    if (color) {
        const T z = (src[k] - lv_offdiag_scaled<T>(v, src, k, i, j, l)) * v.D[k];
        if (mode) { v.x[k] += z; v.r[k] = z; }
        else v.x[k] = z;
    } else {
        const T z = (src[k] - lv_offdiag<T>(v, mode ? v.r : v.x, k, i, j, l)) * v.D[k];
        if (mode) v.x[k] += z;
        else v.x[k] = z;
    }
}

// ---- small levels, shared-memory resident: one CTA per instance loads the couplings,
// pivots and weights of every level from Ls down (and b of level Ls) into shared memory,
// runs the rest of the V-cycle there with block barriers between passes, and writes x of
// level Ls back.  Layout per level: A (7 N, pitch N), D, pw, x, b, r; the coarsest level
// keeps its dense inverse (N x N), x and b.
__host__ __device__ inline size_t al16(size_t b) { return (b + 15) & ~size_t(15); }
template <class T>
__host__ __device__ inline size_t smem_level_bytes(int N, bool last) {
    if (last) return al16((size_t)N * N * sizeof(T)) + 2 * al16((size_t)N * sizeof(T));
    return al16(7 * (size_t)N * sizeof(T)) + 5 * al16((size_t)N * sizeof(T));
}
template <class T>
__device__ LevView<T> smem_view(const DevP &P, int L, int Ls, unsigned char *base) {
    size_t off = 0;
    for (int q = Ls; q < L; q++) off += smem_level_bytes<T>(PT<T>::lev(P, q).N, false);
    const LevelT<T> &g = PT<T>::lev(P, L);
    const int N = g.N;
    const size_t nb = al16((size_t)N * sizeof(T));
    unsigned char *p = base + off;
    LevView<T> v;
    v.ap = N;
    v.Nx = g.Nx; v.Ny = g.Ny; v.Nz = g.Nz; v.N = N;
    v.cx = g.cx; v.cy = g.cy; v.cz = g.cz; v.last = g.last;
    v.ph = nullptr;
    if (g.last) {
        v.A = nullptr; v.r = nullptr; v.pw = nullptr;
        v.D = reinterpret_cast<T *>(p); p += al16((size_t)N * N * sizeof(T));
        v.x = reinterpret_cast<T *>(p); p += nb;
        v.b = reinterpret_cast<T *>(p);
    } else {
        v.A = reinterpret_cast<T *>(p); p += al16(7 * (size_t)N * sizeof(T));
        v.D = reinterpret_cast<T *>(p); p += nb;
        v.pw = reinterpret_cast<T *>(p); p += nb;
        v.x = reinterpret_cast<T *>(p); p += nb;
        v.b = reinterpret_cast<T *>(p); p += nb;
        v.r = reinterpret_cast<T *>(p);
    }
    return v;
}
template <class T>
__device__ __forceinline__ void blk_copy(T *dst, const T *src, int n) {
    for (int q = threadIdx.x; q < n; q += blockDim.x) dst[q] = src[q];
}
template <class T>
__device__ __forceinline__ void blk_smooth(const LevView<T> &v, int color, int mode) {
    const int hx = (v.Nx + 1) >> 1, rows = v.Ny * v.Nz;
    for (int t = threadIdx.x; t < hx * rows; t += blockDim.x) {
        const int row = t / hx, ti = t - row * hx;
        const int l = row / v.Ny, j = row - l * v.Ny;
        const int i = 2 * ti + ((j + l + color) & 1);
        if (i >= v.Nx) continue;
        smooth_node<T>(v, i + v.Nx * row, i, j, l, mode, color);
    }
    __syncthreads();
}

// stage the set-up of levels Ls .. nl-1 into the shared-memory views sv (the block's
// threads; the caller synchronises before use)
template <class T>
__device__ __forceinline__ void blk_stage_small(const DevP &P, const LevView<T> *sv, int Ls, int nl) {
    for (int L = Ls; L < nl; L++) {
        const LevelT<T> &g = PT<T>::lev(P, L);
        const LevView<T> v = sv[L - Ls];
        if (g.last) {
            blk_copy<T>(v.D, g.D, g.N * g.N);
        } else {
            for (int q = 0; q < 7; q++) blk_copy<T>(const_cast<T *>(v.A) + q * g.N, g.A[q], g.N);
            blk_copy<T>(v.D, g.D, g.N);
            blk_copy<T>(v.pw, g.pw, g.N);
        }
    }
}
// V(1,1) cycle of the staged levels Ls .. nl-1 in shared memory, from b of level Ls
// (sv[0].b) to x of level Ls (sv[0].x), block barriers between the passes
template <class T>
__device__ void blk_vcycle_small(const LevView<T> *sv, int Ls, int nl, T al) {
    for (int L = Ls; L < nl - 1; L++) {
        const LevView<T> v = sv[L - Ls], cv = sv[L + 1 - Ls];
        blk_smooth<T>(v, 1, 0);
        blk_smooth<T>(v, 0, 0);
        // residual summed into the aggregates: 8 lanes per coarse node, lane bits (di, dj, dl)
        // pick the fine node (the same summation order for every aggregate)
        const int nK = ((cv.N + 3) >> 2) << 5;       // 8 lanes x coarse nodes, whole warps
        for (int t = threadIdx.x; t < nK; t += blockDim.x) {
            const int K = t >> 3, sub = t & 7;
            T val = 0;
            if (K < cv.N) {
                const Node c = unidx(K, cv.Nx, cv.Ny);
                const int di = sub & 1, dj = (sub >> 1) & 1, dl = sub >> 2;
                const int i = v.cx ? 2 * c.i + di : c.i, j = v.cy ? 2 * c.j + dj : c.j, l = v.cz ? 2 * c.l + dl : c.l;
                const bool ok = i < v.Nx && j < v.Ny && l < v.Nz && (v.cx || di == 0) && (v.cy || dj == 0) &&
                                (v.cz || dl == 0);
                if (ok) {
                    const int k = i + v.Nx * (j + v.Ny * l);
                    val = v.b[k] - lv_apply<T>(v, v.x, k, i, j, l);
                }
            }
            val += __shfl_xor_sync(0xffffffffu, val, 1);
            val += __shfl_xor_sync(0xffffffffu, val, 2);
            val += __shfl_xor_sync(0xffffffffu, val, 4);
            if (sub == 0 && K < cv.N) cv.b[K] = val;
        }
        __syncthreads();
    }
    {                                             // coarsest level: x = D^-1 b (dense inverse)
        const LevView<T> v = sv[nl - 1 - Ls];
        for (int r = threadIdx.x; r < v.N; r += blockDim.x) {
            T sum = 0;
            for (int q = 0; q < v.N; q++) sum += v.D[r * v.N + q] * v.b[q];
            v.x[r] = sum;
        }
        __syncthreads();
    }
    for (int L = nl - 2; L >= Ls; L--) {
        const LevView<T> v = sv[L - Ls], cv = sv[L + 1 - Ls];
        for (int k = threadIdx.x; k < v.N; k += blockDim.x) {
            const Node a = unidx(k, v.Nx, v.Ny);
            const int I = v.cx ? a.i >> 1 : a.i, J = v.cy ? a.j >> 1 : a.j, K = v.cz ? a.l >> 1 : a.l;
            v.x[k] += al * v.pw[k] * cv.x[I + cv.Nx * (J + cv.Ny * K)];
        }
        __syncthreads();
        for (int k = threadIdx.x; k < v.N; k += blockDim.x) {
            const Node a = unidx(k, v.Nx, v.Ny);
            v.r[k] = v.b[k] - lv_apply<T>(v, v.x, k, a.i, a.j, a.l);
        }
        __syncthreads();
        blk_smooth<T>(v, 1, 1);
        blk_smooth<T>(v, 0, 1);
    }
}


// ---- hierarchy set-up, per node / per coarse node / per block (shared by the per-launch
// set-up kernels of kernels_la.cu and the persistent solves)
// red-black D-ILU pivot of node k, stored as its reciprocal: red D = a_kk; black
// D = a_kk - sum a_kr a_rk / a_rr, guarded as the reference guards its ILU pivots
// (semiconductor_3d.c:1937-1938)
template <class T>
__device__ __forceinline__ void ilu_diag_node(const LevView<T> &v, int k) {
    const Node a = unidx(k, v.Nx, v.Ny);
    const T c = v.a(0, k);
    T d = c;
    if ((a.i + a.j + a.l) & 1) {
        const int NxNy = v.Nx * v.Ny;
        T s = 0;
        if (a.i > 0) s += v.a(1, k) * v.a(2, k - 1) / v.a(0, k - 1);
        if (a.i < v.Nx - 1) s += v.a(2, k) * v.a(1, k + 1) / v.a(0, k + 1);
        if (a.j > 0) s += v.a(3, k) * v.a(4, k - v.Nx) / v.a(0, k - v.Nx);
        if (a.j < v.Ny - 1) s += v.a(4, k) * v.a(3, k + v.Nx) / v.a(0, k + v.Nx);
        if (a.l > 0) s += v.a(5, k) * v.a(6, k - NxNy) / v.a(0, k - NxNy);
        if (a.l < v.Nz - 1) s += v.a(6, k) * v.a(5, k + NxNy) / v.a(0, k + NxNy);
        d = c - s;
        if (!(d > T(1e-8) * fabs(c))) d = c;
    }
    if (!(d != T(0))) d = 1;
    v.D[k] = T(1) / d;                     // the smoothers multiply by the reciprocal
}

// coarsest level set-up by one block: dense matrix of the stencil, Gauss-Jordan inverse
// with partial pivoting (tiny pivots guarded as semiconductor_3d.c:2066 does), formed in
// FP64 in the block's shared scratch M (COARSE_MAX x (COARSE_MAX + 1)) and stored in T
template <class T>
__device__ void blk_coarse_setup(const LevelT<T> &v, double *M, int *perm, int *piv) {
    const int n = v.N, ld = COARSE_MAX + 1;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) M[(e / n) * ld + e % n] = 0.0;
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        const Node a = unidx(r, v.Nx, v.Ny);
        const int NxNy = v.Nx * v.Ny;
        M[r * ld + r] = v.A[0][r];
        if (a.i > 0) M[r * ld + r - 1] = v.A[1][r];
        if (a.i < v.Nx - 1) M[r * ld + r + 1] = v.A[2][r];
        if (a.j > 0) M[r * ld + r - v.Nx] = v.A[3][r];
        if (a.j < v.Ny - 1) M[r * ld + r + v.Nx] = v.A[4][r];
        if (a.l > 0) M[r * ld + r - NxNy] = v.A[5][r];
        if (a.l < v.Nz - 1) M[r * ld + r + NxNy] = v.A[6][r];
    }
    __syncthreads();
    // in-place Gauss-Jordan inversion with row interchanges (columns unswapped at the end)
    for (int c = 0; c < n; c++) {
        if (threadIdx.x == 0) {
            int p = c;
            double mx = fabs(M[c * ld + c]);
            for (int r = c + 1; r < n; r++)
                if (fabs(M[r * ld + c]) > mx) { mx = fabs(M[r * ld + c]); p = r; }
            *piv = p;
            perm[c] = p;
            if (!(mx > 1e-300)) M[p * ld + c] = 1e-300;
        }
        __syncthreads();
        const int p = *piv;
        if (p != c)
            for (int q = threadIdx.x; q < n; q += blockDim.x) {
                const double t = M[c * ld + q]; M[c * ld + q] = M[p * ld + q]; M[p * ld + q] = t;
            }
        __syncthreads();
        const double dg = M[c * ld + c];
        __syncthreads();
        if (threadIdx.x == 0) M[c * ld + c] = 1.0;
        __syncthreads();
        for (int q = threadIdx.x; q < n; q += blockDim.x) M[c * ld + q] /= dg;
        __syncthreads();
        // eliminate column c from every other row: each thread owns whole rows
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            if (r == c) continue;
            const double fct = M[r * ld + c];
            M[r * ld + c] = 0.0;
            for (int q = 0; q < n; q++) M[r * ld + q] -= fct * M[c * ld + q];
        }
        __syncthreads();
    }
    for (int c = n - 1; c >= 0; c--) {
        const int p = perm[c];
        if (p != c)
            for (int r = threadIdx.x; r < n; r += blockDim.x) {
                const double t = M[r * ld + c]; M[r * ld + c] = M[r * ld + p]; M[r * ld + p] = t;
            }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, q = e % n;
        v.D[r * n + q] = (T)M[r * ld + q];
    }
}

// Slotboom weights of the aggregate of coarse node K (semiconductor_3d.c:2092-2117):
// qsign 0 gives pw = 1
__device__ __forceinline__ double ph0(const DevP &P, int k, int qsign) {
    const uint32_t f = P.flags[k];
    if (fl_kind(f) != K_SEMI || fl_fix(f)) return PH_NONE;
    return qsign > 0 ? P.phin[k] / P.VTref : -P.phip[k] / P.VTref;
}
template <class T>
__device__ __forceinline__ void mg_weights_node(const DevP &P, const LevView<T> &f, const LevelT<T> &cl, int L,
                                                int qsign, int K) {
    const Node c = unidx(K, cl.Nx, cl.Ny);
    const Agg g = agg_range(f, c.i, c.j, c.l);
    if (qsign == 0) {
        for (int l = g.l0; l <= g.l1; l++)
            for (int j = g.j0; j <= g.j1; j++)
                for (int i = g.i0; i <= g.i1; i++) f.pw[i + f.Nx * (j + f.Ny * l)] = 1;
        return;
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
                f.pw[k] = (T)(e < -700.0 ? 0.0 : exp(e));
            }
}

// Petrov-Galerkin coarse operator row of coarse node K, P^T W A P
// (semiconductor_3d.c:2003-2027), summed in FP64; w: the level-0 row weights or null
template <class T>
__device__ __forceinline__ void galerkin_node(const LevView<T> &f, const LevelT<T> &cl, const T *w, int K) {
    const int NxNy = f.Nx * f.Ny;
    const Node c = unidx(K, cl.Nx, cl.Ny);
    const Agg g = agg_range(f, c.i, c.j, c.l);
    double cc = 0, xm = 0, xp = 0, ym = 0, yp = 0, zm = 0, zp = 0;
    for (int l = g.l0; l <= g.l1; l++)
        for (int j = g.j0; j <= g.j1; j++)
            for (int i = g.i0; i <= g.i1; i++) {
                const int k = i + f.Nx * (j + f.Ny * l);
                const double wk = w ? (double)w[k] : 1.0;
                double a;
                cc += wk * (double)f.a(0, k) * (double)f.pw[k];
                if (i > 0) { a = wk * (double)f.a(1, k) * (double)f.pw[k - 1]; if (i - 1 >= g.i0) cc += a; else xm += a; }
                if (i < f.Nx - 1) { a = wk * (double)f.a(2, k) * (double)f.pw[k + 1]; if (i + 1 <= g.i1) cc += a; else xp += a; }
                if (j > 0) { a = wk * (double)f.a(3, k) * (double)f.pw[k - f.Nx]; if (j - 1 >= g.j0) cc += a; else ym += a; }
                if (j < f.Ny - 1) { a = wk * (double)f.a(4, k) * (double)f.pw[k + f.Nx]; if (j + 1 <= g.j1) cc += a; else yp += a; }
                if (l > 0) { a = wk * (double)f.a(5, k) * (double)f.pw[k - NxNy]; if (l - 1 >= g.l0) cc += a; else zm += a; }
                if (l < f.Nz - 1) { a = wk * (double)f.a(6, k) * (double)f.pw[k + NxNy]; if (l + 1 <= g.l1) cc += a; else zp += a; }
            }
    if (cc == 0. && xm == 0. && xp == 0. && ym == 0. && yp == 0. && zm == 0. && zp == 0.) cc = 1.;
    cl.A[0][K] = (T)cc; cl.A[1][K] = (T)xm; cl.A[2][K] = (T)xp; cl.A[3][K] = (T)ym;
    cl.A[4][K] = (T)yp; cl.A[5][K] = (T)zm; cl.A[6][K] = (T)zp;
}

}  // namespace ss
