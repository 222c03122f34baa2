// Anderson acceleration (Walker-Ni) of the Gummel map on the 3N state
// x = (psi, phi_n, phi_p) (semiconductor_3d.c:3709-3757): FP32 difference history,
// FP64 Gram matrix and normal equations, masked mixing.
#include "device_common.cuh"
#include "prof.h"
#include "solver_ctx.h"

namespace ss {

static inline dim3 grid3(const Ctx &c) {
    int b = (3 * c.maxN + TPB - 1) / TPB;
    if (b > c.grid_cap) b = c.grid_cap;
    return dim3(b < 1 ? 1 : b, c.ninst);
}

// carrier `hole` matters at node k: > 1e-6 of n + p + |Nd - Na| (semiconductor_3d.c:3696-3700)
__device__ __forceinline__ bool aa_sig(const DevP &P, int k, int hole) {
    const uint32_t f = P.flags[k];
    if (fl_kind(f) != K_SEMI || fl_fix(f)) return false;
    const double c = hole ? P.p[k] : P.n[k];
    return c > 1e-6 * (P.n[k] + P.p[k] + fabs(P.Nd[k] - P.Na[k]));
}
__device__ __forceinline__ void blk(const DevP &P, int b, const double *&x, double *&g) {
    x = b == 0 ? P.xk : (b == 1 ? P.qn0 : P.qp0);
    g = b == 0 ? P.phi : (b == 1 ? P.phin : P.phip);
}

// dF[s] = f_new - f_old, dG[s] = g - g_old (float), f_new masked
__global__ void k_aa_diff(const DevP *__restrict__ Ps, int s) {
    const DevP &P = Ps[blockIdx.y];
    const int N = P.N, L = 3 * N;
    float *dF = P.aaF + (size_t)s * L, *dG = P.aaG + (size_t)s * L;
    SS_GRID_LOOP(q, L) {
        const int b = q / N, k = q - b * N;
        const double *x; double *g;
        blk(P, b, x, g);
        const double gk = g[k];
        const double fk = (b == 0 || aa_sig(P, k, b - 1)) ? gk - x[k] : 0.0;
        dF[q] = (float)(fk - P.aaf[q]);
        dG[q] = (float)(gk - P.aag[q]);
    }
}
// Gram row/column s: gram[i][s] = dF[i] . dF[s], i < n
__global__ void k_aa_gram(const DevP *__restrict__ Ps, int s, int n) {
    const DevP &P = Ps[blockIdx.y];
    const int L = 3 * P.N;
    const float *ds = P.aaF + (size_t)s * L;
    double acc[AA_MAX];
#pragma unroll
    for (int i = 0; i < AA_MAX; i++) acc[i] = 0.0;
    SS_GRID_LOOP(q, L) {
        const double a = ds[q];
#pragma unroll
        for (int i = 0; i < AA_MAX; i++)
            if (i < n) acc[i] += (double)P.aaF[(size_t)i * L + q] * a;
    }
    if (grid_sum<AA_MAX>(acc, P.part, P.ticket + 6)) {
        for (int i = 0; i < n; i++) {
            P.gram[i * AA_MAX + s] = acc[i];
            P.gram[s * AA_MAX + i] = acc[i];
        }
    }
}
// f = masked (g - x), g_old = g
__global__ void k_aa_fg(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    const int N = P.N, L = 3 * N;
    SS_GRID_LOOP(q, L) {
        const int b = q / N, k = q - b * N;
        const double *x; double *g;
        blk(P, b, x, g);
        const double gk = g[k];
        P.aaf[q] = (b == 0 || aa_sig(P, k, b - 1)) ? gk - x[k] : 0.0;
        P.aag[q] = gk;
    }
}
// bb[i] = dF[i] . f; regularised normal equations solved by the last block
__global__ void k_aa_bb_solve(const DevP *__restrict__ Ps, int m) {
    const DevP &P = Ps[blockIdx.y];
    const int L = 3 * P.N;
    double acc[AA_MAX];
#pragma unroll
    for (int i = 0; i < AA_MAX; i++) acc[i] = 0.0;
    SS_GRID_LOOP(q, L) {
        const double fq = P.aaf[q];
#pragma unroll
        for (int i = 0; i < AA_MAX; i++)
            if (i < m) acc[i] += (double)P.aaF[(size_t)i * L + q] * fq;
    }
    if (grid_sum<AA_MAX>(acc, P.part, P.ticket + 6)) {
        double A[AA_MAX][AA_MAX], bb[AA_MAX], gam[AA_MAX];
        double tr = 0.0;
        for (int i = 0; i < m; i++) {
            bb[i] = acc[i];
            for (int j = 0; j < m; j++) A[i][j] = P.gram[i * AA_MAX + j];
            tr += A[i][i];
        }
        for (int i = 0; i < m; i++) A[i][i] += 1e-9 * tr + 1e-300;
        for (int c = 0; c < m; c++) {                 // Gaussian elimination, partial pivoting
            int pv = c;
            for (int r = c + 1; r < m; r++)
                if (fabs(A[r][c]) > fabs(A[pv][c])) pv = r;
            if (pv != c) {
                for (int q = 0; q < m; q++) { const double t = A[c][q]; A[c][q] = A[pv][q]; A[pv][q] = t; }
                const double t = bb[c]; bb[c] = bb[pv]; bb[pv] = t;
            }
            for (int r = c + 1; r < m; r++) {
                const double fct = A[r][c] / A[c][c];
                for (int q = c; q < m; q++) A[r][q] -= fct * A[c][q];
                bb[r] -= fct * bb[c];
            }
        }
        for (int r = m - 1; r >= 0; r--) {
            double t = bb[r];
            for (int q = r + 1; q < m; q++) t -= A[r][q] * gam[q];
            gam[r] = t / A[r][r];
        }
        int ok = 1;
        for (int i = 0; i < m; i++) {
            if (!(gam[i] == gam[i])) ok = 0;
            P.aagam[i] = gam[i];
        }
        P.res[R_AUX] = ok;
    }
}
// g -= sum gam_i dG[i] where the node takes part (psi off contacts, phi_n/p where significant)
__global__ void k_aa_mix(const DevP *__restrict__ Ps, int m) {
    const DevP &P = Ps[blockIdx.y];
    if (P.res[R_AUX] == 0.0) return;                 // NaN coefficients: keep the Picard step
    const int N = P.N, L = 3 * N;
    double gam[AA_MAX];
    for (int i = 0; i < m; i++) gam[i] = P.aagam[i];
    SS_GRID_LOOP(q, L) {
        const int b = q / N, k = q - b * N;
        const uint32_t f = P.flags[k];
        if (b == 0 ? fl_con(f) != 0 : fl_fix(f)) continue;
        if (b > 0 && !aa_sig(P, k, b - 1)) continue;
        const double *x; double *g;
        blk(P, b, x, g);
        double s = g[k];
        for (int i = 0; i < m; i++) s -= gam[i] * (double)P.aaG[(size_t)i * L + q];
        g[k] = s;
    }
}

void aa_update_history(const Ctx &c, int slot, int nfill) {
    SS_LAUNCH(PF_AA, 3 * c.maxN, k_aa_diff, grid3(c), TPB, c.st, c.dP, slot);
    SS_LAUNCH(PF_AA, 3 * c.maxN, k_aa_gram, grid3(c), TPB, c.st, c.dP, slot, nfill);
}
void aa_store_fg(const Ctx &c) { SS_LAUNCH(PF_AA, 3 * c.maxN, k_aa_fg, grid3(c), TPB, c.st, c.dP); }
void aa_solve_mix(const Ctx &c, int m, int *) {
    SS_LAUNCH(PF_AA, 3 * c.maxN, k_aa_bb_solve, grid3(c), TPB, c.st, c.dP, m);
    SS_LAUNCH(PF_AA, 3 * c.maxN, k_aa_mix, grid3(c), TPB, c.st, c.dP, m);
}

}  // namespace ss
