// Gate tunnelling (models bit 5): Tsu-Esaki current with WKB transmission through the layer
// stack of every path from a semiconductor node to a gate metal (semiconductor_3d.c:3230-3388).
//
// Supply: carriers pressed against the interface by the field supply it through their
// pressure on the wall (contact theorem summed over the path's column); carriers pushed away
// use the local density extrapolated to the interface.  The escape is linearised in the
// column densities (col_K, a sink K c at each column node), the injection from the gate
// (tp_G) is a source at the interface node.  One thread per path: it owns its column slots.
//
// The continuity sink / source of both exchange models (gate tunnelling and metal contacts)
// is gathered per node here, in the reference's order of summation.
#include "device_common.cuh"
#include "physics_hd.cuh"
#include "prof.h"
#include "solver_ctx.h"

namespace ss {

// one path (tun_path, semiconductor_3d.c:3326-3366)
__global__ void __launch_bounds__(64) k_tun_path(const DevP *__restrict__ Ps, TunD T) {
    const DevP &P = Ps[0];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= T.n_tp) return;
    const int k = T.tp_k[p], c = T.tp_c[p];
    const MatD &ms = P.mats[fl_mat(P.flags[k])];
    const double VT = ms.VT, A = T.tp_A[p], Vg = P.cons[c].V;
    TPath S;
    tun_stack(S, P.mats, T.tp_nl[p], T.tp_m + (size_t)p * TUN_MAXL, T.tp_t + (size_t)p * TUN_MAXL, P.phi[k], Vg,
              P.cons[c].phi_m, P.Cref);
    const int q0 = T.tp_c0[p], nq = T.tp_cn[p];
    const double Fs = S.D / ms.eps;                 // surface field, + = pushes electrons to the wall
    double neff[2];
    for (int hole = 0; hole < 2; hole++) {
        const double sg = hole ? -1.0 : 1.0, Fsc = sg * Fs;
        const double *car = hole ? P.p : P.n;
        for (int q = q0; q < q0 + nq; q++) T.col_K[2 * q + hole] = 0.0;
        if (Fsc > 0.0) {                            // pressed against the wall: contact theorem
            double P0 = 0.0, Fl = Fsc;
            for (int q = q0; q < q0 + nq; q++) {
                const int kq = T.col_k[q];
                const double Fr = (q < q0 + nq - 1 && T.col_h[q] > 0.0)
                                      ? sg * (P.phi[kq] - P.phi[T.col_k[q + 1]]) / T.col_h[q] : Fl;
                double Fm = 0.5 * (Fl + Fr);
                if (Fm < 0.0) Fm = 0.0;
                const double w = Fm * T.col_l[q] / VT;   // share of node q per unit density
                T.col_K[2 * q + hole] = w;
                P0 += w * car[kq];
                Fl = Fr;
            }
            const int kl = T.col_k[q0 + nq - 1];
            T.col_K[2 * (q0 + nq - 1) + hole] += 1.0;
            P0 += car[kl];                          // kT n(z1)
            neff[hole] = P0;
        } else {                                    // pushed away: local density at the interface
            const double qc = hole ? qcp_of(P, k) : qcn_of(P, k);
            neff[hole] = car[k] * exp(-qc + sg * (S.psis - P.phi[k]) / VT);
            T.col_K[2 * q0 + hole] = neff[hole] / fmax(car[k], NFLOOR);
        }
        if (!(neff[hole] > 1e-100)) neff[hole] = 1e-100;
    }
    const double EFn = -P.phin[k] - P.Cref, EFp = -P.phip[k] - P.Cref, EFm = -Vg - P.Cref;
    const double Ecp = EFn - VT * log(neff[0] / ms.Nc), Evp = EFp + VT * log(neff[1] / ms.Nv);
    double F[4];
    tun_flux(ms, S, Ecp, Evp, EFn, EFp, EFm, F);
    const double be = A * F[0] / neff[0], bh = A * F[2] / neff[1];   // K_q = A F_sg / n_eff dn_eff/dc_q
    for (int q = q0; q < q0 + nq; q++) {
        T.col_K[2 * q] *= be;
        T.col_K[2 * q + 1] *= bh;
    }
    T.tp_G[2 * p] = A * F[1];
    T.tp_G[2 * p + 1] = A * F[3];
}

// escape rates (1/s) of path p at the current densities (tun_escape, semiconductor_3d.c:3382-3388)
__device__ __forceinline__ void tun_escape(const DevP &P, const TunD &T, int p, double &se, double &sh) {
    double a = 0.0, b = 0.0;
    for (int q = T.tp_c0[p]; q < T.tp_c0[p] + T.tp_cn[p]; q++) {
        const int kq = T.col_k[q];
        a += T.col_K[2 * q] * P.n[kq];
        b += T.col_K[2 * q + 1] * P.p[kq];
    }
    se = a;
    sh = b;
}

// continuity sink tk and source tg of carrier `hole` at every node the exchange touches:
// tunnelling column terms, gate injection, then metal-contact column terms, each in
// ascending order (tun_scatter + te_scatter, semiconductor_3d.c:3373-3379, 3544-3553)
__global__ void k_exchange_scatter(const DevP *__restrict__ Ps, ScD S, TunD T, TeD E, int hole) {
    const DevP &P = Ps[0];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    double K = 0.0, G = 0.0;
    for (int e = S.pk[i]; e < S.pk[i + 1]; e++) K += T.col_K[2 * S.qk[e] + hole];
    for (int e = S.pg[i]; e < S.pg[i + 1]; e++) G += T.tp_G[2 * S.qg[e] + hole];
    for (int e = S.pe[i]; e < S.pe[i + 1]; e++) {
        const int q = S.qe[e];
        K += E.tc_K[2 * q + hole];
        G += E.tc_G[2 * q + hole];
    }
    const int k = S.k[i];
    P.tk[k] = K;
    P.tg[k] = G;
}

// gate terminal currents (semiconductor_3d.c:3613-3620): electrons leaving to the gate are
// current into the device through the gate, holes leaving are current out of it; one block,
// each contact's paths summed by the block in a fixed order
constexpr int TUN_CUR_TPB = 256;
__global__ void __launch_bounds__(TUN_CUR_TPB) k_tun_currents(const DevP *__restrict__ Ps, TunD T) {
    const DevP &P = Ps[0];
    __shared__ double sh[3][TUN_CUR_TPB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int c = 0; c < P.ncon; c++) {
        double v[3] = {0.0, 0.0, 0.0};
        for (int p = threadIdx.x; p < T.n_tp; p += blockDim.x) {
            if (T.tp_c[p] != c) continue;
            double se, shh;
            tun_escape(P, T, p, se, shh);
            const double G0 = T.tp_G[2 * p], G1 = T.tp_G[2 * p + 1];
            const double Ie = Q * (se - G0), Ih = -Q * (shh - G1);
            v[0] += Ie + Ih;
            v[1] += Q * (se + G0 + shh + G1);
            v[2] += Ie;
        }
        for (int w = 0; w < 3; w++) {
            double x = v[w];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) sh[w][wid] = x;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double s = 0.0;
            for (int q = 0; q < TUN_CUR_TPB / 32; q++) s += sh[threadIdx.x][q];
            P.res[(threadIdx.x == 0 ? R_I : (threadIdx.x == 1 ? R_S : R_IN)) + c] += s;
        }
        __syncthreads();
    }
}

// display: the gate-tunnelling current density at the interface nodes (A/m^2, into the
// device through the gate), the sum over the node's paths divided by their area
// (semiconductor_3d.c:3648-3657); tk / tg were cleared before
__global__ void k_tun_display(const DevP *__restrict__ Ps, ScD S, TunD T) {
    const DevP &P = Ps[0];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n || S.pg[i] == S.pg[i + 1]) return;
    double g = 0.0, a = 0.0;
    for (int e = S.pg[i]; e < S.pg[i + 1]; e++) {
        const int p = S.qg[e];
        double se, sh;
        tun_escape(P, T, p, se, sh);
        g += Q * ((se - T.tp_G[2 * p]) - (sh - T.tp_G[2 * p + 1]));
        a += T.tp_A[p];
    }
    const int k = S.k[i];
    P.tk[k] = a;
    P.tg[k] = a > 0.0 ? g / a : g;
}

// ------------------------------------------------------------------ host drivers
static int blocks(int n, int tpb) { return n > 0 ? (n + tpb - 1) / tpb : 1; }

void tun_update(Inst &d) {                       // semiconductor_3d.c:3367-3371
    if (!d.g.tun_on) return;
    Ctx c = make_ctx(d);
    SS_LAUNCH(PF_METAL, d.g.tun.n_col, k_tun_path, blocks(d.g.tun.n_tp, 64), 64, c.st, c.dP, d.g.tun);
}
void exchange_scatter(Inst &d, int hole) {
    if (!d.g.sc.n) return;
    Ctx c = make_ctx(d);
    SS_LAUNCH(PF_METAL, d.g.sc.n, k_exchange_scatter, blocks(d.g.sc.n, 128), 128, c.st, c.dP, d.g.sc, d.g.tun,
              d.g.te, hole);
}
void tun_currents(Inst &d) {
    if (!d.g.tun_on) return;
    Ctx c = make_ctx(d);
    SS_LAUNCH(PF_METAL, d.g.tun.n_col, k_tun_currents, 1, TUN_CUR_TPB, c.st, c.dP, d.g.tun);
}
void tun_display(Inst &d) {
    if (!d.g.tun_on) return;
    Ctx c = make_ctx(d);
    SS_LAUNCH(PF_METAL, d.g.sc.n, k_tun_display, blocks(d.g.sc.n, 128), 128, c.st, c.dP, d.g.sc, d.g.tun);
}

// fluxes through a stack from a semiconductor surface at psi (api3_tun_eval,
// semiconductor_3d.c:4850-4868): out = e s->g, e g->s, h s->g, h g->s (1/m^2 s); returns the
// net current density into the semiconductor through the gate (A/m^2)
double tun_eval_host(const MatD *mats, int smat, int nl, const int *mat, const double *t, double psi, double phin,
                     double phip, double Vg, double pm, double Cref, double *out) {
    TPath S;
    tun_stack(S, mats, nl, mat, t, psi, Vg, pm, Cref);
    const MatD &ms = mats[smat];
    const double Ec = -S.psis - ms.chi, Ev = Ec - ms.Eg;
    double F[4];
    tun_flux(ms, S, Ec, Ev, -phin - Cref, -phip - Cref, -Vg - Cref, F);
    if (out) for (int i = 0; i < 4; i++) out[i] = F[i];
    return Q * ((F[0] - F[1]) - (F[2] - F[3]));
}
double lombardi_host(const MatD &m, double mub, double F, double Nt, double Dw, int hole) {
    return lombardi(m, mub, F, Nt, Dw, hole, 0.0);
}
double coulomb_inv_host(const MatD &m, double F, double n, double NC, double NA) { return coul_inv(m, F, n, NC, NA); }

}  // namespace ss
