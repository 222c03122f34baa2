// Floating majority-carrier blocks of a continuity solve (semiconductor_3d.c:3159-3228).
// A connected region where carrier c is the quasi-neutral majority and that no carrier
// contact reaches is rescaled uniformly, c -> lambda c, so that its global balance
// (net outflow + recombination inside = 0) holds; Newton in ln(lambda) per block.
//
// The reference finds the blocks by a breadth-first search.  Here the components are
// labelled on the device by min-label propagation with line sweeps along x, y, z
// (each sweep carries labels the whole length of a line), the anchoring test and the
// block sums are per-node kernels adding into per-block exact accumulators (exact_sum.cuh),
// so that the sums, and the rescaled solution, do not depend on the order of the threads.
#include <cmath>
#include <cstdio>
#include <vector>

#include "device_common.cuh"
#include "exact_sum.cuh"
#include "prof.h"
#include "solver_ctx.h"

namespace ss {

constexpr int FF_MAX_BLOCKS = 1024;

__device__ __forceinline__ bool ff_maj(const DevP &P, int k, int hole) {
    const uint32_t f = P.flags[k];
    if (fl_kind(f) != K_SEMI || fl_con(f)) return false;
    const double s = P.sc[k], c = s * P.sol[k];
    const double oth = hole ? P.n[k] : P.p[k];
    const double hd = 0.5 * dnet_ion(P, k);
    const MatD &m = P.mats[fl_mat(f)];
    return c >= oth && c >= hd && s >= hd && c > 10.0 * niK(P, m, k);
}

__global__ void k_ff_init(const DevP *__restrict__ Ps, int hole) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        P.ccl[k] = ff_maj(P, k, hole) ? k : -1;
        P.cclaux[k] = 0;
    }
}
__global__ void k_ff_sweep(const DevP *__restrict__ Ps, int ax, int *changed) {
    const DevP &P = Ps[blockIdx.y];
    const int n = ax == 0 ? P.Nx : (ax == 1 ? P.Ny : P.Nz);
    const int st = ax == 0 ? 1 : (ax == 1 ? P.Nx : P.Nx * P.Ny);
    const int nlines = P.N / n;
    int *lab = P.ccl;
    int ch = 0;
    SS_GRID_LOOP(t, nlines) {
        int k0;
        if (ax == 0) k0 = t * P.Nx;
        else if (ax == 1) { const int i = t % P.Nx, l = t / P.Nx; k0 = i + l * P.Nx * P.Ny; }
        else k0 = t;
        for (int q = 1; q < n; q++) {
            const int k = k0 + q * st, a = lab[k], b = lab[k - st];
            if (a >= 0 && b >= 0 && b < a) { lab[k] = b; ch = 1; }
        }
        for (int q = n - 2; q >= 0; q--) {
            const int k = k0 + q * st, a = lab[k], b = lab[k + st];
            if (a >= 0 && b >= 0 && b < a) { lab[k] = b; ch = 1; }
        }
    }
    if (ch) *changed = 1;
}
// a block touching a semiconductor contact node is anchored
__global__ void k_ff_anchor(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const int lb = P.ccl[k];
        if (lb < 0) continue;
        const Node a = unidx(k, P.Nx, P.Ny);
        for (int dir = 0; dir < 6; dir++) {
            int kb; double h, ar;
            if (!nbr(P, a, k, dir, kb, h, ar)) continue;
            const uint32_t fb = P.flags[kb];
            if (fl_kind(fb) == K_SEMI && fl_con(fb)) { P.cclaux[lb] = 1; break; }
        }
    }
}
// list the unanchored roots; cclaux[root] = 2 + block index
__global__ void k_ff_roots(const DevP *__restrict__ Ps, int *count, int *roots) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        if (P.ccl[k] != k || P.cclaux[k] != 0) continue;
        const int b = atomicAdd(count, 1);
        if (b < FF_MAX_BLOCKS) { roots[b] = k; P.cclaux[k] = 2 + b; }
        else P.cclaux[k] = 1;          // beyond the table: left as it is
    }
}
__device__ __forceinline__ int ff_block(const DevP &P, int k) {
    const int lb = P.ccl[k];
    if (lb < 0) return -1;
    const int a = P.cclaux[lb];
    return a >= 2 ? a - 2 : -1;
}
// boundary balance of every block: Aout = sum self s_k u_k, Bin = sum nb c_b
__global__ void k_ff_boundary(const DevP *__restrict__ Ps, int hole, unsigned long long *Aout,
                              unsigned long long *Bin) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const int b = ff_block(P, k);
        if (b < 0) continue;
        const Node a = unidx(k, P.Nx, P.Ny);
        const uint32_t f = P.flags[k];
        const MatD &m = P.mats[fl_mat(f)];
        const double VT = m.VT, lk = hole ? lnvK(P, m, k) : lncK(P, m, k);
        const double ck = P.sc[k] * P.sol[k];
        double ao = 0.0, bi = 0.0;
        for (int dir = 0; dir < 6; dir++) {
            int kb; double h, ar;
            if (!nbr(P, a, k, dir, kb, h, ar)) continue;
            const uint32_t fb = P.flags[kb];
            if (fl_kind(fb) != K_SEMI || P.ccl[kb] == P.ccl[k]) continue;
            const MatD &mb = P.mats[fl_mat(fb)];
            const double lb = hole ? lnvK(P, mb, kb) : lncK(P, mb, kb);
            const double D = (P.phi[kb] - P.phi[k]) / VT + (hole ? -(lb - lk) : (lb - lk));
            const int kl = k < kb ? k : kb;
            const double g = ar * P.fmu[(hole ? 3 : 0) + (dir >> 1)][kl] * VT / h;
            const double self = hole ? g * bern(D) : g * bern(-D), nb = hole ? g * bern(-D) : g * bern(D);
            const double cb = fl_con(fb) ? (hole ? P.p[kb] : P.n[kb]) : P.sc[kb] * P.sol[kb];
            ao += self * ck;
            bi += nb * cb;
        }
        xs_add(Aout + (size_t)b * XS_WORDS, ao);
        xs_add(Bin + (size_t)b * XS_WORDS, bi);
    }
}
// recombination of every block at the trial scale lambda_b
__global__ void k_ff_recomb(const DevP *__restrict__ Ps, int hole, const double *lam, unsigned long long *G,
                            unsigned long long *dG) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const int b = ff_block(P, k);
        if (b < 0) continue;
        const Node a = unidx(k, P.Nx, P.Ny);
        const MatD &m = P.mats[fl_mat(P.flags[k])];
        const double c = lam[b] * P.sc[k] * P.sol[k];
        const double oth = hole ? P.n[k] : P.p[k];
        double R, dRn, dRp;
        recombK(P, m, k, hole ? oth : c, hole ? c : oth, R, dRn, dRp);
        const double vol = P.Lx[a.i] * P.Ly[a.j] * P.Lz[a.l];
        double g = vol * R, dg = vol * (hole ? dRp : dRn) * c;
        if (P.tk) { g += P.tk[k] * c - P.tg[k]; dg += P.tk[k] * c; }   // metal-contact exchange
        if (P.gii) g -= P.gii[k];                                        // impact-ionisation pairs
        xs_add(G + (size_t)b * XS_WORDS, g);
        xs_add(dG + (size_t)b * XS_WORDS, dg);
    }
}
// the per-block totals of two accumulator sets: out0[b], out1[b] for b < nb
__global__ void k_ff_finish(const unsigned long long *a0, const unsigned long long *a1, int nb, double *out0,
                            double *out1) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nb) out0[t] = xs_value(a0 + (size_t)t * XS_WORDS);
    else if (t < 2 * nb) out1[t - nb] = xs_value(a1 + (size_t)(t - nb) * XS_WORDS);
}
__global__ void k_ff_apply(const DevP *__restrict__ Ps, const double *scale) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const int b = ff_block(P, k);
        if (b < 0) continue;
        P.sol[k] *= scale[b];
    }
}

int float_fix(Inst &d, int hole) {
    Ctx c = make_ctx(d);
    const dim3 g(c.nodes_blocks(), 1);
    double *const g_ffbuf = d.g.h.ffbuf;
    int *const g_ffint = d.g.h.ffint;
    int *changed = g_ffint, *count = g_ffint + 1, *roots = g_ffint + 16;
    SS_LAUNCH(PF_CCL, d.N, k_ff_init, g, TPB, c.st, c.dP, hole);
    int h = 1, cycles = 0;
    const int maxcyc = d.Nx + d.Ny + d.Nz + 8;
    if (d.unstr) { ff_label_g(d, changed); h = 0; }           // labels over the graph's edges, anchors
    while (h && cycles < maxcyc) {
        cudaMemsetAsync(changed, 0, sizeof(int), c.st);
        for (int ax = 0; ax < 3; ax++) {
            const int n = ax == 0 ? d.Nx : (ax == 1 ? d.Ny : d.Nz);
            const int nb = ((int)d.N / n + TPB - 1) / TPB;
            SS_LAUNCH(PF_CCL, d.N, k_ff_sweep, dim3(nb, 1), TPB, c.st, c.dP, ax, changed);
        }
        cudaMemcpyAsync(&h, changed, sizeof(int), cudaMemcpyDeviceToHost, c.st);
        cudaStreamSynchronize(c.st);
        cycles++;
    }
    if (!d.unstr) SS_LAUNCH(PF_CCL, d.N, k_ff_anchor, g, TPB, c.st, c.dP);
    cudaMemsetAsync(count, 0, sizeof(int), c.st);
    SS_LAUNCH(PF_CCL, d.N, k_ff_roots, g, TPB, c.st, c.dP, count, roots);
    int nb = 0;
    cudaMemcpyAsync(&nb, count, sizeof(int), cudaMemcpyDeviceToHost, c.st);
    cudaStreamSynchronize(c.st);
    if (nb <= 0) return 0;
    if (nb > FF_MAX_BLOCKS) nb = FF_MAX_BLOCKS;
    double *Aout = g_ffbuf, *Bin = g_ffbuf + FF_MAX_BLOCKS, *lam = g_ffbuf + 2 * FF_MAX_BLOCKS;
    double *G = g_ffbuf + 3 * FF_MAX_BLOCKS, *dG = g_ffbuf + 4 * FF_MAX_BLOCKS;
    unsigned long long *const acc = d.g.h.ffacc;           // [sum][block][XS_WORDS]
    const size_t aw = (size_t)FF_MAX_BLOCKS * XS_WORDS;
    const int fin = (2 * nb + TPB - 1) / TPB;
    for (int q = 0; q < 2; q++) cudaMemsetAsync(acc + q * aw, 0, sizeof(unsigned long long) * nb * XS_WORDS, c.st);
    if (d.unstr) ff_boundary_g(d, hole, acc, acc + aw);
    else SS_LAUNCH(PF_CCL, d.N, k_ff_boundary, g, TPB, c.st, c.dP, hole, acc, acc + aw);
    SS_LAUNCH(PF_CCL, 2 * nb, k_ff_finish, dim3(fin), TPB, c.st, acc, acc + aw, nb, Aout, Bin);
    std::vector<double> hA(nb), hB(nb), sl(nb, 0.0), hl(nb), hG(nb), hdG(nb);
    std::vector<int> act(nb, 1);
    cudaMemcpyAsync(hA.data(), Aout, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.st);
    cudaMemcpyAsync(hB.data(), Bin, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.st);
    cudaStreamSynchronize(c.st);
    for (int it = 0; it < 60; it++) {
        int any = 0;
        for (int b = 0; b < nb; b++) { hl[b] = std::exp(sl[b]); any |= act[b]; }
        if (!any) break;
        cudaMemcpyAsync(lam, hl.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, c.st);
        for (int q = 2; q < 4; q++) cudaMemsetAsync(acc + q * aw, 0, sizeof(unsigned long long) * nb * XS_WORDS, c.st);
        SS_LAUNCH(PF_CCL, d.N, k_ff_recomb, g, TPB, c.st, c.dP, hole, lam, acc + 2 * aw, acc + 3 * aw);
        SS_LAUNCH(PF_CCL, 2 * nb, k_ff_finish, dim3(fin), TPB, c.st, acc + 2 * aw, acc + 3 * aw, nb, G, dG);
        cudaMemcpyAsync(hG.data(), G, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.st);
        cudaMemcpyAsync(hdG.data(), dG, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.st);
        cudaStreamSynchronize(c.st);
        for (int b = 0; b < nb; b++) {
            if (!act[b]) continue;
            const double l = hl[b];
            const double Gv = l * hA[b] - hB[b] + hG[b], dGv = l * hA[b] + hdG[b];
            if (!(dGv > 0.)) { act[b] = 0; continue; }
            double ds = -Gv / dGv;
            if (ds > 2.) ds = 2.;
            else if (ds < -2.) ds = -2.;
            sl[b] += ds;
            if (std::fabs(ds) < 1e-13) act[b] = 0;
        }
    }
    int nfix = 0;
    for (int b = 0; b < nb; b++) {
        const double s = sl[b];
        if (s == s && std::fabs(s) > 1e-15 && std::fabs(s) < 200.) { hl[b] = std::exp(s); nfix++; }
        else hl[b] = 1.0;
    }
    cudaMemcpyAsync(lam, hl.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, c.st);
    SS_LAUNCH(PF_CCL, d.N, k_ff_apply, g, TPB, c.st, c.dP, lam);
    cudaStreamSynchronize(c.st);
    if (d.verbose > 2) std::fprintf(stderr, "    float_fix(%c): %d blocks, %d rescaled\n", hole ? 'p' : 'n', nb, nfix);
    return nfix;
}

}  // namespace ss
