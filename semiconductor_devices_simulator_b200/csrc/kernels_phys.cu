// Physics kernels of the solve path: Poisson residual / Jacobian, Scharfetter-Gummel
// continuity assembly, face mobility, carrier and quasi-Fermi updates, boundary
// values, terminal currents, predictors and the display outputs.
//
// One thread per node, grid-stride loops; blockIdx.y selects the instance.  Every
// routine restates the reference routine cited beside it.
#include <cstdio>

#include "device_common.cuh"
#include "physics_hd.cuh"
#include "prof.h"
#include "kernels.h"

namespace ss {

int Ctx::nodes_blocks() const {
    int b = (maxN + TPB - 1) / TPB;
    if (b > grid_cap) b = grid_cap;
    if (b < 1) b = 1;
    return b;
}

static inline dim3 grid_of(const Ctx &c) { return dim3(c.nodes_blocks(), c.ninst); }

// ------------------------------------------------------------------ Poisson
// F_k = sum eps_f A_f (psi_b - psi_k)/h + V_k q (p - n + Nd - Na + Nf) + Robin gate term,
// Jacobian (-dF/dpsi) as a 7-point stencil and ||F/diag|| (semiconductor_3d.c:2732-2789).
// src: 0 psi = P.phi, 1 psi = P.tr.  build: write A, sc and F into rhs; else F into P.F
// and the norm uses the sc of the last build (as the reference's line search does).
__global__ void k_poisson(const DevP *__restrict__ Ps, int src, int build) {
    const DevP &P = Ps[blockIdx.y];
    const double *phi = src ? P.tr : P.phi;
    double *F = build ? P.rhs : P.F;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        if (fl_con(f)) {
            F[k] = 0.0;
            if (build) {
                P.A[0][k] = 1.0;
#pragma unroll
                for (int q = 1; q < 7; q++) P.A[q][k] = 0.0;
                P.sc[k] = 1.0;
            }
            continue;
        }
        const Node a = unidx(k, P.Nx, P.Ny);
        const MatD &m = P.mats[fl_mat(f)];
        const double ek = m.eps, pk = phi[k];
        double fk = 0.0, dg = 0.0, off[6];
#pragma unroll
        for (int dir = 0; dir < 6; dir++) {
            int kb; double h, ar;
            off[dir] = 0.0;
            if (!nbr(P, a, k, dir, kb, h, ar)) continue;
            const uint32_t fb = P.flags[kb];
            const double eb = P.mats[fl_mat(fb)].eps;
            const double cf = (2.0 * ek * eb / (ek + eb)) * ar / h;
            fk += cf * (phi[kb] - pk);
            dg += cf;
            if (!fl_con(fb)) off[dir] = -cf;
        }
        const double vol = P.Lx[a.i] * P.Ly[a.j] * P.Lz[a.l];
        if (fl_kind(f) == K_SEMI) {
            const double n = nK(P, m, k, pk, P.phin[k]), p = pK(P, m, k, pk, P.phip[k]);
            if (ion_node(P, k)) {                 // incompletely ionised dopants
                double Np, dNp, Nm, dNm;
                ion_eval(P, m, k, n, p, Np, dNp, Nm, dNm);
                fk += vol * Q * (p - n + Np - Nm + P.Nf[k]);
                dg += vol * Q * ((n + p) / m.VT - dNp + dNm);
            } else {
                fk += vol * Q * (p - n + P.Nd[k] - P.Na[k] + P.Nf[k]);
                dg += vol * Q * (n + p) / m.VT;
            }
            if (trap_node(P, k)) {                    // charge in deep traps
                double r, a, b, rho, drho;
                trap_eval(P, m, k, n, p, r, a, b, rho, drho);
                fk += vol * Q * rho;
                dg -= vol * Q * drho;
            }
        } else {
            fk += vol * Q * P.Nf[k];
        }
        const int g = fl_gate(f);
        if (g) {                                  // oxide Robin gate (semiconductor_3d.c:2778-2785)
            const ConD &cn = P.cons[g - 1];
            const double Cox = EPS_OX / (cn.tox > 0.0 ? cn.tox : 10e-9);
            const double pm = cn.phi_m > 0.0 ? cn.phi_m : P.Cref;
            const double VG = cn.V + P.Cref - pm;
            const double rA = P.robA[k];
            fk += rA * (Cox * (VG - pk) + cn.qox);
            dg += Cox * rA;
        }
        F[k] = fk;
        double sck;
        if (build) {
            P.A[0][k] = dg;
#pragma unroll
            for (int q = 0; q < 6; q++) P.A[1 + q][k] = off[q];
            P.sc[k] = dg;
            sck = dg;
        } else {
            sck = P.sc[k];
        }
        const double r = fk / sck;
        acc[0] += r * r;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 0)) P.res[R_PNORM] = sqrt(acc[0]);
}

void launch_poisson(const Ctx &c, const double *phi_sel, int build, double *) {
    SS_LAUNCH(PF_POISSON, c.maxN, k_poisson, grid_of(c), TPB, c.st, c.dP, phi_sel ? 1 : 0, build);
}

// n, p from the potentials (semiconductor_3d.c:2826-2834)
__global__ void k_rebuild_np(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        if (fl_kind(f) != K_SEMI) { P.n[k] = P.p[k] = 0.0; continue; }
        const MatD &m = P.mats[fl_mat(f)];
        P.n[k] = nK(P, m, k, P.phi[k], P.phin[k]);
        P.p[k] = pK(P, m, k, P.phi[k], P.phip[k]);
    }
}
void launch_rebuild_np(const Ctx &c) { SS_LAUNCH(PF_REBUILD, c.maxN, k_rebuild_np, grid_of(c), TPB, c.st, c.dP); }

// Face mobility of the edge k -> k+e_ax from the node low-field mobilities, with
// Caughey-Thomas saturation driven by the harmonic-mean field when models bit 2 is set
// (semiconductor_3d.c:2962-3006), and Lombardi surface scattering near insulator / gate walls
// when models bit 4 is set (the Coulomb term of 4H-SiC is not built).
// potential gradient along ax taken inside the semiconductor (one-sided at an interface,
// semiconductor_3d.c:2909-2917)
__device__ __forceinline__ double grad_semi(const DevP &P, const Node &a, int k, int ax) {
    int km = 0, kp = 0;
    double hm = 1.0, hp = 1.0, ar;
    const bool lo = nbr(P, a, k, 2 * ax, km, hm, ar) && fl_kind(P.flags[km]) == K_SEMI;
    const bool hi = nbr(P, a, k, 2 * ax + 1, kp, hp, ar) && fl_kind(P.flags[kp]) == K_SEMI;
    if (lo && hi) return (P.phi[kp] - P.phi[km]) / (hm + hp);
    if (hi) return (P.phi[kp] - P.phi[k]) / hp;
    if (lo) return (P.phi[k] - P.phi[km]) / hm;
    return 0.0;
}
// squared field normal to axis ax (semiconductor_3d.c:2918-2921)
__device__ __forceinline__ double fnorm2(const DevP &P, const Node &a, int k, int ax) {
    const double g1 = grad_semi(P, a, k, (ax + 1) % 3), g2 = grad_semi(P, a, k, (ax + 2) % 3);
    return g1 * g1 + g2 * g2;
}

__global__ void k_upd_mob(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    const bool sat = (P.models & 4) != 0, lb = (P.models & 16) != 0;
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        const Node a = unidx(k, P.Nx, P.Ny);
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            int kp; double h, ar;
            if (fl_kind(f) != K_SEMI || !nbr(P, a, k, 2 * ax + 1, kp, h, ar) || fl_kind(P.flags[kp]) != K_SEMI) {
                P.fmu[ax][k] = 0.0; P.fmu[3 + ax][k] = 0.0;
                continue;
            }
            const MatD &m = P.mats[fl_mat(f)];
            double mn = 0.5 * (P.mu0n[k] + P.mu0n[kp]), mp = 0.5 * (P.mu0p[k] + P.mu0p[kp]);
            if (ax == P.caxis) {
                if (m.ani_n > 0.0) mn *= m.ani_n;
                if (m.ani_p > 0.0) mp *= m.ani_p;
            }
            if (lb && m.lb_on) {
                const double Dw = exp(-0.5 * (P.qd[k] + P.qd[kp]) / 1e-8);
                if (Dw > 1e-8) {
                    Node b = a;
                    if (ax == 0) b.i++; else if (ax == 1) b.j++; else b.l++;
                    const double F = sqrt(0.5 * (fnorm2(P, a, k, ax) + fnorm2(P, b, kp, ax)));
                    const double Nt = 0.5 * (P.Nd[k] + P.Na[k] + P.Nd[kp] + P.Na[kp]);
                    double ic = 0.0;
                    if (P.if_NC && m.lbc_on) {          // Coulomb scattering, n from the reference levels
                        const double nn = 0.5 * (nK(P, m, k, P.phi[k], P.phin[k]) +
                                                 nK(P, P.mats[fl_mat(P.flags[kp])], kp, P.phi[kp], P.phin[kp]));
                        const int ea = P.qi[k], eb = P.qi[kp];
                        const double NC = ea >= 0 && eb >= 0 ? 0.5 * (P.if_NC[ea] + P.if_NC[eb])
                                        : (ea >= 0 ? P.if_NC[ea] : (eb >= 0 ? P.if_NC[eb] : 0.0));
                        ic = coul_inv(m, F, nn, NC, 0.5 * (P.Na[k] + P.Na[kp]));
                    }
                    if (m.lb_on & 1) mn = lombardi(m, mn, F, Nt, Dw, 0, ic);
                    if (m.lb_on & 2) mp = lombardi(m, mp, F, Nt, Dw, 1, 0.0);
                }
            }
            // velocity saturation, tapered off across the barrier region of a metal contact
            // (te_vsat_w, semiconductor_3d.c:810-824)
            double wv = 0.0;
            if (sat) {
                wv = 1.0;
                if (P.te_vw) {
                    auto node_w = [&](int kk) {
                        const double w = P.te_vw[kk];
                        if (w >= 1.0) return 1.0;
                        const double c2 = P.te_ax[kk] == ax ? 1.0 : 0.0;
                        return 1.0 - (1.0 - w) * c2;
                    };
                    wv = 0.5 * (node_w(k) + node_w(kp));
                }
            }
            if (wv > 0.0) {
                const double dps = P.phi[kp] - P.phi[k];
                const double Fn = heat_field(P.phin[kp] - P.phin[k], dps, h);
                const double Fp = heat_field(P.phip[kp] - P.phip[k], dps, h);
                const double sn = mob_hf(mn, Fn, m.vsat_n, m.beta_n), sp = mob_hf(mp, Fp, m.vsat_p, m.beta_p);
                mn += wv * (sn - mn);
                mp += wv * (sp - mp);
            }
            P.fmu[ax][k] = mn; P.fmu[3 + ax][k] = mp;
        }
    }
}
// N_C of every Coulomb interface entry: fixed charge plus the charged trap states of the
// node at the reference quasi-Fermi potentials, per interface area (coul_update,
// semiconductor_3d.c:1624-1636)
__global__ void k_coul_update(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(e, P.n_if) {
        const int k = P.if_k[e];
        const double A = P.if_A[e];
        if (!(A > 0.0)) { P.if_NC[e] = 0.0; continue; }
        double Qt = 0.0;
        if (trap_node(P, k)) {
            const MatD &m = P.mats[fl_mat(P.flags[k])];
            const Node a = unidx(k, P.Nx, P.Ny);
            Qt = trap_abs(P, m, k, nK(P, m, k, P.phi[k], P.phin[k]), pK(P, m, k, P.phi[k], P.phip[k])) *
                 (P.Lx[a.i] * P.Ly[a.j] * P.Lz[a.l]);
        }
        P.if_NC[e] = (P.if_Qf[e] + Qt) / A;
    }
}
void launch_coul_update(const Ctx &c) {
    if (c.h.if_NC && (c.h.models & 16))
        SS_LAUNCH(PF_UPDMOB, c.h.n_if, k_coul_update, dim3(c.nodes_blocks(), c.ninst), TPB, c.st, c.dP);
}
void launch_upd_mob(const Ctx &c) {
    launch_coul_update(c);
    SS_LAUNCH(PF_UPDMOB, c.maxN, k_upd_mob, grid_of(c), TPB, c.st, c.dP);
}

// ------------------------------------------------------------------ continuity
// Scaled Scharfetter-Gummel row for u = c/s (semiconductor_3d.c:3067-3106):
//   electrons D = dpsi/VT + d(ln Nc_eff), self = g B(-D), nb = g B(D)
//   holes     D = dpsi/VT - d(ln Nv_eff), self = g B(D),  nb = g B(-D)
// linearised recombination on the diagonal, row scale 1/(diag s_k).
__global__ void k_cont_assemble(const DevP *__restrict__ Ps, int hole) {
    const DevP &P = Ps[blockIdx.y];
    const double *car = hole ? P.p : P.n;
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        const bool semi = fl_kind(f) == K_SEMI;
        if (!semi || fl_fix(f)) {
            P.A[0][k] = 1.0;
#pragma unroll
            for (int q = 1; q < 7; q++) P.A[q][k] = 0.0;
            P.rhs[k] = semi ? 1.0 : 0.0;
            P.sc[k] = semi ? car[k] : 0.0;
            P.dsc[k] = 0.0;
            continue;
        }
        const Node a = unidx(k, P.Nx, P.Ny);
        const MatD &m = P.mats[fl_mat(f)];
        const double VT = m.VT, sk = fmax(car[k], NFLOOR);
        const double lk = hole ? lnvK(P, m, k) : lncK(P, m, k);
        const double pk = P.phi[k];
        double dg = 0.0, b = 0.0, off[6];
#pragma unroll
        for (int dir = 0; dir < 6; dir++) {
            int kb; double h, ar;
            off[dir] = 0.0;
            if (!nbr(P, a, k, dir, kb, h, ar)) continue;
            const uint32_t fb = P.flags[kb];
            if (fl_kind(fb) != K_SEMI) continue;
            const MatD &mb = P.mats[fl_mat(fb)];
            const double lb = hole ? lnvK(P, mb, kb) : lncK(P, mb, kb);
            const double D = (P.phi[kb] - pk) / VT + (hole ? -(lb - lk) : (lb - lk));
            const int kl = k < kb ? k : kb;
            const double g = ar * P.fmu[(hole ? 3 : 0) + (dir >> 1)][kl] * VT / h;
            const double bp = bern(D), bm = bern(-D);
            const double self = hole ? g * bp : g * bm;
            const double nb = hole ? g * bm : g * bp;
            dg += self;
            if (fl_fix(fb)) b += nb * car[kb];
            else off[dir] = -nb * fmax(car[kb], NFLOOR);
        }
        double R, dRn, dRp;
        recombK(P, m, k, P.n[k], P.p[k], R, dRn, dRp);
        double dR = hole ? dRp : dRn;
        if (dR < 0.0) dR = 0.0;
        const double vol = P.Lx[a.i] * P.Ly[a.j] * P.Lz[a.l];
        dg += vol * dR;
        b += vol * (dR * car[k] - R);
        if (P.tk) { dg += P.tk[k]; b += P.tg[k]; }   // metal-contact exchange: sink tk c - tg
        if (P.gii) b += P.gii[k];                   // impact ionisation (pairs)
        const double w = 1.0 / (dg * sk);
        P.A[0][k] = 1.0;
#pragma unroll
        for (int q = 0; q < 6; q++) P.A[1 + q][k] = off[q] * w;
        P.rhs[k] = b * w;
        P.sc[k] = sk;
        P.dsc[k] = dg * sk;
    }
}
void launch_cont_assemble(const Ctx &c, int hole) { SS_LAUNCH(PF_CONT_ASM, c.maxN, k_cont_assemble, grid_of(c), TPB, c.st, c.dP, hole); }

// c = s u -> quasi-Fermi potential clamped to [lo, hi], carrier, change, and the
// weighted max |change| (semiconductor_3d.c:3112-3146)
__global__ void k_cont_update(const DevP *__restrict__ Ps, int hole, double lo, double hi) {
    const DevP &P = Ps[blockIdx.y];
    double *qf = hole ? P.phip : P.phin;
    double *car = hole ? P.p : P.n;
    const double *oth = hole ? P.n : P.p;
    double *dq = hole ? P.dqp : P.dqn;
    double dmax = 0.0;
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        if (fl_kind(f) != K_SEMI || fl_fix(f)) { dq[k] = 0.0; continue; }
        const MatD &m = P.mats[fl_mat(f)];
        double u = P.sol[k];
        if (!(u > 1e-30)) u = 1e-30;
        else if (u > 1e30) u = 1e30;
        const double cc = P.sc[k] * u;
        double qn = hole ? P.phi[k] + m.VT * (log(cc) - lnvK(P, m, k)) : P.phi[k] - m.VT * (log(cc) - lncK(P, m, k));
        if (qn < lo) qn = lo;
        else if (qn > hi) qn = hi;
        const double ch = qn - qf[k];
        qf[k] = qn;
        dq[k] = ch;
        const double cn = hole ? pK(P, m, k, P.phi[k], qn) : nK(P, m, k, P.phi[k], qn);
        car[k] = cn;
        const double scale = cn + oth[k] + fabs(P.Nd[k] - P.Na[k]);
        const double r = scale > 0.0 ? cn / scale : 0.0;
        if (r > 1e-6) {
            const double w = r >= 1e-3 ? 1.0 : r * 1e3;
            dmax = fmax(dmax, w * fabs(ch));
        }
    }
    if (grid_max(dmax, P.part, P.ticket + 1)) P.res[R_DQ] = dmax;
}
void launch_cont_update(const Ctx &c, int hole, double lo, double hi) {
    SS_LAUNCH(PF_CONT_UPD, c.maxN, k_cont_update, grid_of(c), TPB, c.st, c.dP, hole, lo, hi);
}

// ------------------------------------------------------------------ boundary values
// neutral potential with both quasi-Fermi levels at V (semiconductor_3d.c:1782-1805): the
// closed form, and with deep traps or incompletely ionised dopants a safeguarded Newton on
// p - n + N_D+ - N_A- + Nf + trapped charge = 0 (decreasing in psi) from it, at most 200 steps
__device__ double neutral_psi(const DevP &P, const MatD &m, int k, double V) {
    const double D = P.Nd[k] - P.Na[k], VT = m.VT;
    double psi = V + VT * (asinh(D / (2.0 * niK(P, m, k))) - 0.5 * (lncK(P, m, k) - lnvK(P, m, k)));
    const bool io = ion_node(P, k);
    if (!trap_node(P, k) && !io) return psi;
    double lo = psi - m.Eg - 1.0, hi = psi + m.Eg + 1.0;
    for (int it = 0; it < 200; it++) {
        const double n = nK(P, m, k, psi, V), p = pK(P, m, k, psi, V);
        double a, b, c, r, dr;
        trap_eval(P, m, k, n, p, a, b, c, r, dr);
        double g = p - n + D + P.Nf[k] + r, dg = -(n + p) / VT + dr;
        if (io) {                                    // incompletely ionised dopants
            double Np, dNp, Nm, dNm;
            ion_eval(P, m, k, n, p, Np, dNp, Nm, dNm);
            g = p - n + Np - Nm + P.Nf[k] + r;
            dg = -(n + p) / VT + dr + dNp - dNm;
        }
        if (g > 0.0) lo = psi; else hi = psi;
        double nx = dg < 0.0 ? psi - g / dg : 0.5 * (lo + hi);
        if (!(nx > lo && nx < hi)) nx = 0.5 * (lo + hi);
        if (fabs(nx - psi) < 1e-13 * (1.0 + fabs(psi))) { psi = nx; break; }
        psi = nx;
    }
    return psi;
}

// the neutral majority density of every incompletely ionised node, slot 3 of its
// ionisation constants (semiconductor_3d.c:1502-1508)
__global__ void k_ion_neutral(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    if (!P.ion) return;
    SS_GRID_LOOP(k, P.N) {
        if (!ion_node(P, k)) continue;
        const MatD &m = P.mats[fl_mat(P.flags[k])];
        const double ps = neutral_psi(P, m, k, 0.0);
        const double n = nK(P, m, k, ps, 0.0), p = pK(P, m, k, ps, 0.0);
        P.ion[(size_t)ION_W * k + 3] = fabs(n - p);
    }
}
void launch_ion_neutral(const Ctx &c) { SS_LAUNCH(PF_BC, c.maxN, k_ion_neutral, grid_of(c), TPB, c.st, c.dP); }

// Dirichlet values of every contact node at the stage voltages (semiconductor_3d.c:1806-1829)
__global__ void k_apply_bc(const DevP *__restrict__ Ps, int have_solution) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        const int c = fl_con(f);
        if (!c) continue;
        const ConD &cn = P.cons[c - 1];
        const double V = cn.V;
        const MatD &m = P.mats[fl_mat(f)];
        if (fl_kind(f) == K_METAL) {
            const double pm = cn.phi_m > 0.0 ? cn.phi_m : P.Cref;
            P.phi[k] = V + P.Cref - pm; P.phin[k] = P.phip[k] = V; P.n[k] = P.p[k] = 0.0;
            continue;
        }
        if (cn.bc == 1) {
            const double pm = cn.phi_m > 0.0 ? cn.phi_m : P.Cref;
            P.phi[k] = V + P.Cref - pm;
            if (cn.te && have_solution) {          // metal contact: the carriers are unknowns
                P.n[k] = nK(P, m, k, P.phi[k], P.phin[k]);
                P.p[k] = pK(P, m, k, P.phi[k], P.phip[k]);
                continue;
            }
        } else {
            P.phi[k] = neutral_psi(P, m, k, V);
        }
        P.phin[k] = P.phip[k] = V;
        P.n[k] = nK(P, m, k, P.phi[k], V);
        P.p[k] = pK(P, m, k, P.phi[k], V);
    }
}
void launch_apply_bc(const Ctx &c, int have_solution) {
    SS_LAUNCH(PF_BC, c.maxN, k_apply_bc, grid_of(c), TPB, c.st, c.dP, have_solution);
}

// local charge-neutral equilibrium start (semiconductor_3d.c:1831-1845)
__global__ void k_init_eq(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        P.phin[k] = P.phip[k] = 0.0;
        if (fl_kind(f) == K_SEMI) {
            const MatD &m = P.mats[fl_mat(f)];
            const double ps = neutral_psi(P, m, k, 0.0);
            P.phi[k] = ps;
            P.n[k] = nK(P, m, k, ps, 0.0);
            P.p[k] = pK(P, m, k, ps, 0.0);
        } else {
            P.phi[k] = 0.0; P.n[k] = P.p[k] = 0.0;
        }
        P.Rt[k] = 0.0;
    }
}
void launch_init_eq(const Ctx &c) { SS_LAUNCH(PF_BC, c.maxN, k_init_eq, grid_of(c), TPB, c.st, c.dP); }

// quasi-Fermi potentials clamped to the terminal span (semiconductor_3d.c:3945-3952)
__global__ void k_clamp_qf(const DevP *__restrict__ Ps, double lo, double hi) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        double a = P.phin[k], b = P.phip[k];
        P.phin[k] = a < lo ? lo : (a > hi ? hi : a);
        P.phip[k] = b < lo ? lo : (b > hi ? hi : b);
    }
}
void launch_clamp_qf(const Ctx &c, double lo, double hi) { SS_LAUNCH(PF_VEC, c.maxN, k_clamp_qf, grid_of(c), TPB, c.st, c.dP, lo, hi); }

// ------------------------------------------------------------------ currents
// SG flux through the face a -> b, split into electrons / holes, with the magnitude
// scales (semiconductor_3d.c:2843-2854)
__device__ __forceinline__ void face_flux(const DevP &P, int ka, int kb, int ax, double h, double ar, double &Jn,
                                          double &Jp, double &Sn, double &Sp) {
    const MatD &ma = P.mats[fl_mat(P.flags[ka])];
    const MatD &mb = P.mats[fl_mat(P.flags[kb])];
    const double VT = ma.VT, dps = (P.phi[kb] - P.phi[ka]) / VT;
    const double Dn = dps + (lncK(P, mb, kb) - lncK(P, ma, ka));
    const double Dp = dps - (lnvK(P, mb, kb) - lnvK(P, ma, ka));
    const int kl = ka < kb ? ka : kb;
    const double gn = Q * ar * P.fmu[ax][kl] * VT / h;
    const double gp = Q * ar * P.fmu[3 + ax][kl] * VT / h;
    const double a1 = gn * P.n[kb] * bern(Dn), a2 = gn * P.n[ka] * bern(-Dn);
    const double b1 = gp * P.p[ka] * bern(Dp), b2 = gp * P.p[kb] * bern(-Dp);
    Jn = a1 - a2; Jp = b1 - b2; Sn = a1 + a2; Sp = b1 + b2;
}

// Flux out of every contact's nodes into semiconductor nodes of other contacts or none:
// I, S and the electron part per contact (semiconductor_3d.c:3598-3623).  Per-contact
// block sums with a deterministic finish in the last block.
__global__ void k_currents(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    const int nc = P.ncon;
    double *pc = P.partc;
    unsigned *ticket = P.ticket + 7;
    for (int c = 0; c < nc; c++) {
        double v[3] = {0.0, 0.0, 0.0};
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P.ncnode; q += gridDim.x * blockDim.x) {
            const int k = P.cnode[q];
            if (fl_con(P.flags[k]) != c + 1 || P.cons[c].te) continue;   // metal contacts: te_currents
            const Node a = unidx(k, P.Nx, P.Ny);
            for (int dir = 0; dir < 6; dir++) {
                int kb; double h, ar;
                if (!nbr(P, a, k, dir, kb, h, ar)) continue;
                const uint32_t fb = P.flags[kb];
                if (fl_kind(fb) != K_SEMI || fl_con(fb) == c + 1) continue;
                double Jn, Jp, Sn, Sp;
                face_flux(P, k, kb, dir >> 1, h, ar, Jn, Jp, Sn, Sp);
                v[0] += Jn + Jp; v[1] += Sn + Sp; v[2] += Jn;
            }
        }
        block_sum<3>(v);
        if (threadIdx.x == 0) {
            pc[blockIdx.x * 96 + 3 * c + 0] = v[0];
            pc[blockIdx.x * 96 + 3 * c + 1] = v[1];
            pc[blockIdx.x * 96 + 3 * c + 2] = v[2];
        }
    }
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    if (threadIdx.x < 3 * nc) {
        double s = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) s += __ldcg(pc + b * 96 + threadIdx.x);
        const int c = threadIdx.x / 3, w = threadIdx.x % 3;
        P.res[(w == 0 ? R_I : (w == 1 ? R_S : R_IN)) + c] = s;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

void launch_currents(const Ctx &c) {
    int nb = (c.h.ncnode + TPB - 1) / TPB;
    if (nb < 1) nb = 1;
    if (nb > 256) nb = 256;                    // grid-stride beyond 256 blocks (partial buffer size)
    SS_LAUNCH(PF_CURRENTS, c.h.ncnode, k_currents, dim3(nb, c.ninst), TPB, c.st, c.dP);
}

// ------------------------------------------------------------------ impact ionisation
// pair generation G = (alpha_n(F_n) |J_n| + alpha_p(F_p) |J_p|) / q over the control volume,
// F the field along each carrier's node current density (semiconductor_3d.c:4486-4523), and
// the total generation -> res[R_GII]
__global__ void k_ii_update(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        double gk = 0.0;
        const MatD &m = P.mats[fl_mat(f)];
        if (fl_kind(f) == K_SEMI && !fl_fix(f) && m.ii_on) {
            const Node a = unidx(k, P.Nx, P.Ny);
            double Jn[3], Jp[3], E[3];
#pragma unroll
            for (int ax = 0; ax < 3; ax++) {
                double sn = 0.0, sp = 0.0, h, ar, jn, jp, s1, s2;
                int cnt = 0, kb;
                if (nbr(P, a, k, 2 * ax, kb, h, ar) && fl_kind(P.flags[kb]) == K_SEMI) {
                    face_flux(P, kb, k, ax, h, ar, jn, jp, s1, s2); sn += jn / ar; sp += jp / ar; cnt++;
                }
                if (nbr(P, a, k, 2 * ax + 1, kb, h, ar) && fl_kind(P.flags[kb]) == K_SEMI) {
                    face_flux(P, k, kb, ax, h, ar, jn, jp, s1, s2); sn += jn / ar; sp += jp / ar; cnt++;
                }
                Jn[ax] = cnt ? sn / cnt : 0.0;
                Jp[ax] = cnt ? sp / cnt : 0.0;
                E[ax] = -grad_semi(P, a, k, ax);
            }
            const double vol = P.Lx[a.i] * P.Ly[a.j] * P.Lz[a.l];
            double G = 0.0;
            for (int c = 0; c < 2; c++) {
                const double *J = c ? Jp : Jn;
                const double jj = sqrt(J[0] * J[0] + J[1] * J[1] + J[2] * J[2]);
                if (!(jj > 0.0)) continue;
                const double F = fabs(E[0] * J[0] + E[1] * J[1] + E[2] * J[2]) / jj;
                G += ii_alpha(m, F, c) * jj;
            }
            gk = G / Q * vol;
        }
        P.gii[k] = gk;
        acc[0] += gk;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 9)) P.res[R_GII] = acc[0];
}
void launch_ii_update(const Ctx &c) { SS_LAUNCH(PF_DISPLAY, c.maxN, k_ii_update, grid_of(c), TPB, c.st, c.dP); }

// ------------------------------------------------------------------ Gummel helpers
// xk = psi; neutral-region psi predictor from the quasi-Fermi changes
// (semiconductor_3d.c:3853-3859)
__global__ void k_predictor(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        const double ps = P.phi[k];
        P.xk[k] = ps;
        if (fl_kind(f) != K_SEMI || fl_con(f)) continue;
        const double n = P.n[k], p = P.p[k], D = dnet_ion(P, k);
        const double den = fmax(n + p, D);
        if (!(den > 0.0)) continue;
        P.phi[k] = ps + (n * P.dqn[k] + p * P.dqp[k]) / den;
    }
}
void launch_predictor(const Ctx &c) { SS_LAUNCH(PF_VEC, c.maxN, k_predictor, grid_of(c), TPB, c.st, c.dP); }

__global__ void k_dpsi(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    double m = 0.0;
    SS_GRID_LOOP(k, P.N) {
        const double a = fabs(P.phi[k] - P.xk[k]);
        m = a > m || a != a ? a : m;
    }
    if (grid_max(m, P.part, P.ticket + 2)) P.res[R_DPSI] = m;
}
void launch_dpsi(const Ctx &c) { SS_LAUNCH(PF_VEC, c.maxN, k_dpsi, grid_of(c), TPB, c.st, c.dP); }

// ------------------------------------------------------------------ display outputs
// node current density (mean of the adjacent face fluxes per axis) and recombination
// (semiconductor_3d.c:3627-3658)
__global__ void k_upd_J(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        double *Jo[3] = {P.Jx, P.Jy, P.Jz};
        if (fl_kind(f) != K_SEMI) { P.Jx[k] = P.Jy[k] = P.Jz[k] = 0.0; P.Rt[k] = 0.0; continue; }
        const Node a = unidx(k, P.Nx, P.Ny);
        for (int ax = 0; ax < 3; ax++) {
            double s = 0.0; int cnt = 0;
            int kb; double h, ar, Jn, Jp, Sn, Sp;
            if (nbr(P, a, k, 2 * ax, kb, h, ar) && fl_kind(P.flags[kb]) == K_SEMI) {
                face_flux(P, kb, k, ax, h, ar, Jn, Jp, Sn, Sp); s += (Jn + Jp) / ar; cnt++;
            }
            if (nbr(P, a, k, 2 * ax + 1, kb, h, ar) && fl_kind(P.flags[kb]) == K_SEMI) {
                face_flux(P, k, kb, ax, h, ar, Jn, Jp, Sn, Sp); s += (Jn + Jp) / ar; cnt++;
            }
            Jo[ax][k] = cnt ? s / cnt : 0.0;
        }
        const MatD &m = P.mats[fl_mat(f)];
        double R, x, y;
        recombK(P, m, k, P.n[k], P.p[k], R, x, y);
        P.Rt[k] = R;
    }
}
void launch_upd_J(const Ctx &c) { SS_LAUNCH(PF_DISPLAY, c.maxN, k_upd_J, grid_of(c), TPB, c.st, c.dP); }

// display mobility: mean of the adjacent edge mobilities (semiconductor_3d.c:3035-3060)
__global__ void k_mob_display(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        if (fl_kind(f) != K_SEMI) { P.mudn[k] = P.mu0n[k]; P.mudp[k] = P.mu0p[k]; continue; }
        const Node a = unidx(k, P.Nx, P.Ny);
        double sn = 0.0, sp = 0.0; int c = 0;
        for (int dir = 0; dir < 6; dir++) {
            int kb; double h, ar;
            if (!nbr(P, a, k, dir, kb, h, ar) || fl_kind(P.flags[kb]) != K_SEMI) continue;
            const int kl = k < kb ? k : kb, ax = dir >> 1;
            double fn = P.fmu[ax][kl], fp = P.fmu[3 + ax][kl];
            if (ax == P.caxis) {
                const MatD &m = P.mats[fl_mat(P.flags[kl])];
                if (m.ani_n > 0.0) fn /= m.ani_n;
                if (m.ani_p > 0.0) fp /= m.ani_p;
            }
            sn += fn; sp += fp; c++;
        }
        P.mudn[k] = c ? sn / c : P.mu0n[k];
        P.mudp[k] = c ? sp / c : P.mu0p[k];
    }
}
void launch_mob_display(const Ctx &c) { SS_LAUNCH(PF_DISPLAY, c.maxN, k_mob_display, grid_of(c), TPB, c.st, c.dP); }

// derived node quantity `which` (semiconductor_3d.c:5066-5126); models outside the
// library's scope contribute their "off" values
__global__ void k_node_val(const DevP *__restrict__ Ps, int which, double *out) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        const int kd = fl_kind(f);
        const MatD &m = P.mats[fl_mat(f)];
        const double nan = __longlong_as_double(0x7ff8000000000000ULL);
        double v = 0.0;
        const Node a = unidx(k, P.Nx, P.Ny);
        switch (which) {
        case 0: v = P.phi[k]; break;
        case 1: v = P.n[k]; break;
        case 2: v = P.p[k]; break;
        case 3: v = kd == K_METAL ? nan : -P.phi[k] - m.chi - bgn_of(P, k) * m.VT; break;
        case 4: v = kd == K_METAL ? nan : -P.phi[k] - m.chi - m.Eg + bgn_of(P, k) * m.VT; break;
        case 5: v = kd == K_INS ? nan : -P.phin[k] - P.Cref; break;
        case 6: v = kd == K_INS ? nan : -P.phip[k] - P.Cref; break;
        case 7: v = P.Jx[k]; break;
        case 8: v = P.Jy[k]; break;
        case 9: v = P.Jz[k]; break;
        case 10: v = P.mudn[k]; break;
        case 11: v = P.mudp[k]; break;
        case 12: v = P.Rt[k]; break;
        case 13: v = (double)kd; break;
        case 14: v = P.Nd[k] - P.Na[k]; break;
        case 15: v = P.phin[k]; break;
        case 16: v = P.phip[k]; break;
        case 17: v = P.Nf[k]; break;
        case 18: v = (double)fl_con(f); break;
        case 19: v = bgn_of(P, k) * m.VT * 2.0; break;
        case 20: case 21: case 22: case 23: case 24: case 25: {
            const int ax = (which - 20) % 3, hole = which >= 23;
            if (kd != K_SEMI) { v = 0.0; break; }
            double s = 0.0; int cnt = 0; int kb; double h, ar, Jn, Jp, Sn, Sp;
            if (nbr(P, a, k, 2 * ax, kb, h, ar) && fl_kind(P.flags[kb]) == K_SEMI) {
                face_flux(P, kb, k, ax, h, ar, Jn, Jp, Sn, Sp); s += (hole ? Jp : Jn) / ar; cnt++;
            }
            if (nbr(P, a, k, 2 * ax + 1, kb, h, ar) && fl_kind(P.flags[kb]) == K_SEMI) {
                face_flux(P, k, kb, ax, h, ar, Jn, Jp, Sn, Sp); s += (hole ? Jp : Jn) / ar; cnt++;
            }
            v = cnt ? s / cnt : 0.0;
            break;
        }
        case 26: v = kd == K_SEMI ? niK(P, m, k) : 0.0; break;
        case 27: v = kd == K_SEMI && P.tg ? P.tg[k] : 0.0; break;   // gate tunnelling J (none: 0 after a solve)
        case 28: case 29: {                         // quantum potentials (eV): the MLDA part of qcn / qcp
            if (kd != K_SEMI) { v = nan; break; }
            const double qc = which == 28 ? qcn_of(P, k) : qcp_of(P, k);
            const double *img = which == 28 ? P.imgn : P.imgp;
            v = -(qc - (img ? img[k] : 0.0)) * m.VT;
            break;
        }
        case 30: v = kd == K_SEMI ? P.qd[k] : nan; break;        // distance to the nearest wall
        case 31: case 32: {                         // trapped charge (q/m^3) / total trap density (m^-3)
            if (kd != K_SEMI) { v = nan; break; }
            if (!trap_node(P, k)) { v = 0.0; break; }
            if (which == 32) {
                double sN = 0.0;
                for (int e = P.tr_rp[k]; e < P.tr_rp[k + 1]; e++) sN += P.tr_N[e];
                v = sN;
            } else {
                double r, a, b, rho, drho;
                trap_eval(P, m, k, P.n[k], P.p[k], r, a, b, rho, drho);
                v = rho;
            }
            break;
        }
        case 33: {                                  // impact-ionisation generation (m^-3 s^-1)
            if (kd != K_SEMI || !P.gii) { v = 0.0; break; }
            const double vol = P.Lx[a.i] * P.Ly[a.j] * P.Lz[a.l];
            v = vol > 0.0 ? P.gii[k] / vol : 0.0;
            break;
        }
        case 34: v = kd == K_SEMI ? (P.if_NC && P.qi[k] >= 0 ? P.if_NC[P.qi[k]] : 0.0) : nan; break;   // N_C (m^-2)
        case 35: {                                  // ionised net doping N_D+ - N_A-
            if (kd != K_SEMI) { v = 0.0; break; }
            double Np, dNp, Nm, dNm;
            ion_eval(P, m, k, P.n[k], P.p[k], Np, dNp, Nm, dNm);
            v = Np - Nm;
            break;
        }
        default: v = 0.0;
        }
        out[k] = v;
    }
}
void launch_node_val(const Ctx &c, int which, double *out) {
    SS_LAUNCH(PF_DISPLAY, c.maxN, k_node_val, grid_of(c), TPB, c.st, c.dP, which, out);
}

// current density through the face k -> k+e_ax, total or electrons (semiconductor_3d.c:5284-5298)
__global__ void k_face_J(const DevP *__restrict__ Ps, int ax, int carrier, double *out) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const Node a = unidx(k, P.Nx, P.Ny);
        int kb; double h, ar, Jn, Jp, Sn, Sp;
        double v = 0.0;
        if (fl_kind(P.flags[k]) == K_SEMI && nbr(P, a, k, 2 * ax + 1, kb, h, ar) && fl_kind(P.flags[kb]) == K_SEMI) {
            face_flux(P, k, kb, ax, h, ar, Jn, Jp, Sn, Sp);
            v = (carrier ? Jn : Jn + Jp) / ar;
        }
        out[k] = v;
    }
}
void launch_face_J(const Ctx &c, int ax, int carrier, double *out) {
    SS_LAUNCH(PF_DISPLAY, c.maxN, k_face_J, grid_of(c), TPB, c.st, c.dP, ax, carrier, out);
}

// ------------------------------------------------------------------ continuation
// psi, phi_n, phi_p = x1 + r (x1 - x2) (semiconductor_3d.c:4061-4087); x1/x2 select the
// history blocks: 0 h1, 1 h2, 2 e2
__global__ void k_extrap(const DevP *__restrict__ Ps, double r, int s1, int s2) {
    const DevP &P = Ps[blockIdx.y];
    double *const *X1 = s1 == 0 ? P.h1 : (s1 == 1 ? P.h2 : P.e2);
    double *const *X2 = s2 == 0 ? P.h1 : (s2 == 1 ? P.h2 : P.e2);
    double *dst[3] = {P.phi, P.phin, P.phip};
    SS_GRID_LOOP(k, P.N) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double x1 = X1[a][k], x2 = X2[a][k];
            dst[a][k] = x1 + r * (x1 - x2);
        }
    }
}
void launch_extrap(const Ctx &c, double r, int s1, int s2) {
    SS_LAUNCH(PF_VEC, c.maxN, k_extrap, grid_of(c), TPB, c.st, c.dP, r, s1, s2);
}
// quadratic sweep predictor: the Lagrange weights of the last three sweep points' solutions
__global__ void k_extrap3(const DevP *__restrict__ Ps, double w1, double w2, double w3) {
    const DevP &P = Ps[blockIdx.y];
    double *dst[3] = {P.phi, P.phin, P.phip};
    SS_GRID_LOOP(k, P.N) {
#pragma unroll
        for (int a = 0; a < 3; a++) dst[a][k] = w1 * P.h1[a][k] + w2 * P.e2[a][k] + w3 * P.e3[a][k];
    }
}
void launch_extrap3(const Ctx &c, double w1, double w2, double w3) {
    SS_LAUNCH(PF_VEC, c.maxN, k_extrap3, grid_of(c), TPB, c.st, c.dP, w1, w2, w3);
}

// ---- region shift (semiconductor_3d.c:3956-3987): flood fill of the quasi-neutral
// region attached to an ohmic contact, by line sweeps along x, y, z until nothing
// changes.  mark[k] = contact+1 of the region that claimed node k.
__device__ __forceinline__ bool region_ok(const DevP &P, int k, int c1, int type, const int *mark) {
    const uint32_t f = P.flags[k];
    if (mark[k] || fl_kind(f) != K_SEMI) return false;
    const int c = fl_con(f);
    if (c && c != c1) return false;
    const double D = P.Nd[k] - P.Na[k];
    if (D * type <= 0.0) return false;
    const double maj = type > 0 ? P.n[k] : P.p[k];
    return !(maj < 0.5 * fabs(D));
}
__global__ void k_region_seed(const DevP *__restrict__ Ps, int c1, int *mark) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        if (fl_con(f) == c1 && fl_kind(f) == K_SEMI && !mark[k]) mark[k] = c1;
    }
}
// one sweep forward and back along every line of axis ax
__global__ void k_region_sweep(const DevP *__restrict__ Ps, int ax, int c1, int type, int *mark, int *changed) {
    const DevP &P = Ps[blockIdx.y];
    const int n = ax == 0 ? P.Nx : (ax == 1 ? P.Ny : P.Nz);
    const int st = ax == 0 ? 1 : (ax == 1 ? P.Nx : P.Nx * P.Ny);
    const int nlines = P.N / n;
    int ch = 0;
    SS_GRID_LOOP(t, nlines) {
        int k0;
        if (ax == 0) k0 = t * P.Nx;
        else if (ax == 1) { const int i = t % P.Nx, l = t / P.Nx; k0 = i + l * P.Nx * P.Ny; }
        else k0 = t;
        int prev = mark[k0];
        for (int q = 1; q < n; q++) {
            const int k = k0 + q * st;
            const int mk = mark[k];
            if (!mk && prev == c1 && region_ok(P, k, c1, type, mark)) { mark[k] = c1; ch = 1; prev = c1; }
            else prev = mark[k];
        }
        prev = mark[k0 + (n - 1) * st];
        for (int q = n - 2; q >= 0; q--) {
            const int k = k0 + q * st;
            const int mk = mark[k];
            if (!mk && prev == c1 && region_ok(P, k, c1, type, mark)) { mark[k] = c1; ch = 1; prev = c1; }
            else prev = mark[k];
        }
    }
    if (ch) *changed = 1;
}
__global__ void k_region_shift(const DevP *__restrict__ Ps, int c1, double dV, const int *mark) {
    const DevP &P = Ps[blockIdx.y];
    SS_GRID_LOOP(k, P.N) {
        if (mark[k] != c1 || fl_con(P.flags[k])) continue;
        P.phi[k] += dV; P.phin[k] += dV; P.phip[k] += dV;
    }
}
// the seed and the shift of a region, for the graph-mesh growth between them
void launch_region_seed(const Ctx &c, int c1, int *mark) {
    SS_LAUNCH(PF_CCL, c.maxN, k_region_seed, grid_of(c), TPB, c.st, c.dP, c1, mark);
}
void launch_region_shift(const Ctx &c, int c1, double dV, const int *mark) {
    SS_LAUNCH(PF_CCL, c.maxN, k_region_shift, grid_of(c), TPB, c.st, c.dP, c1, dV, mark);
}
void launch_region_mark(const Ctx &c, int c1, int type, double dV, int *mark, int *changed) {
    SS_LAUNCH(PF_CCL, c.maxN, k_region_seed, grid_of(c), TPB, c.st, c.dP, c1, mark);
    int h_changed = 1, cycles = 0;
    const int maxcyc = c.h.Nx + c.h.Ny + c.h.Nz + 8;
    while (h_changed && cycles < maxcyc) {
        cudaMemsetAsync(changed, 0, sizeof(int), c.st);
        for (int ax = 0; ax < 3; ax++) {
            const int n = ax == 0 ? c.h.Nx : (ax == 1 ? c.h.Ny : c.h.Nz);
            const int nl = c.h.N / n;
            const int nb = (nl + TPB - 1) / TPB;
            SS_LAUNCH(PF_CCL, c.h.N, k_region_sweep, dim3(nb, c.ninst), TPB, c.st, c.dP, ax, c1, type, mark, changed);
        }
        cudaMemcpyAsync(&h_changed, changed, sizeof(int), cudaMemcpyDeviceToHost, c.st);
        cudaStreamSynchronize(c.st);
        cycles++;
    }
    SS_LAUNCH(PF_CCL, c.maxN, k_region_shift, grid_of(c), TPB, c.st, c.dP, c1, dV, mark);
}

}  // namespace ss
