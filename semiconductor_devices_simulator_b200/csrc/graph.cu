// Devices on a general box-method mesh (triangular prisms or any other), given as a
// symmetric graph of nodes and edges (api3_set_mesh_graph): the same finite-volume equations
// as the tensor path with the neighbours and geometry taken per edge
// (semiconductor_3d.c:4175-4565).
//
// Layout: ELL with gD slots per node, slot s of node k at s*N + k (coalesced over k):
// neighbour (-1 past the node's degree), edge length, dual face area, undirected edge id,
// the slot of the reverse edge in the neighbour's row, and the matrix off-diagonal.  Node
// control volumes sit in Lx (Nx = N, Ny = Nz = 1), so every node-wise kernel of the tensor
// path applies unchanged.
//
// Linear solves: PCG (Poisson) and right-preconditioned BiCGSTAB (continuity) with the
// reference's stop rules, preconditioned by the aggregation multigrid of graph_mg.cu.
#include <vector>

#include "device_common.cuh"
#include "exact_sum.cuh"
#include "physics_hd.cuh"
#include "prof.h"
#include "solver_ctx.h"

namespace ss {

__device__ __forceinline__ double gvol(const DevP &P, int k) { return P.Lx[k]; }

// ------------------------------------------------------------------ Poisson
// F, the diagonal (A[0]) and off-diagonals (gval) of -dF/dpsi, sc and ||F/sc||
// (poisson_core_g, semiconductor_3d.c:4181-4217, with the Robin gates of poisson_eval)
__global__ void k_poisson_g(const DevP *__restrict__ Ps, int src, int build) {
    const DevP &P = Ps[0];
    const double *phi = src ? P.tr : P.phi;
    double *F = build ? P.rhs : P.F;
    const int N = P.N, D = P.gD;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, N) {
        const uint32_t f = P.flags[k];
        if (fl_con(f)) {
            F[k] = 0.0;
            if (build) {
                P.A[0][k] = 1.0;
                for (int s = 0; s < D; s++) P.gval[(size_t)s * N + k] = 0.0;
                P.sc[k] = 1.0;
            }
            continue;
        }
        const MatD &m = P.mats[fl_mat(f)];
        const double ek = m.eps, pk = phi[k];
        double fk = 0.0, dg = 0.0;
        for (int s = 0; s < D; s++) {
            const size_t e = (size_t)s * N + k;
            const int kb = P.gcol[e];
            if (kb < 0) { if (build) P.gval[e] = 0.0; continue; }
            const uint32_t fb = P.flags[kb];
            const double eb = P.mats[fl_mat(fb)].eps;
            const double cf = (2.0 * ek * eb / (ek + eb)) * P.ga[e] / P.gh[e];
            fk += cf * (phi[kb] - pk);
            dg += cf;
            if (build) P.gval[e] = fl_con(fb) ? 0.0 : -cf;
        }
        const double vol = gvol(P, k);
        if (fl_kind(f) == K_SEMI) {
            const double n = nK(P, m, k, pk, P.phin[k]), p = pK(P, m, k, pk, P.phip[k]);
            if (ion_node(P, k)) {
                double Np, dNp, Nm, dNm;
                ion_eval(P, m, k, n, p, Np, dNp, Nm, dNm);
                fk += vol * Q * (p - n + Np - Nm + P.Nf[k]);
                dg += vol * Q * ((n + p) / m.VT - dNp + dNm);
            } else {
                fk += vol * Q * (p - n + P.Nd[k] - P.Na[k] + P.Nf[k]);
                dg += vol * Q * (n + p) / m.VT;
            }
            if (trap_node(P, k)) {
                double r, a, b, rho, drho;
                trap_eval(P, m, k, n, p, r, a, b, rho, drho);
                fk += vol * Q * rho;
                dg -= vol * Q * drho;
            }
        } else {
            fk += vol * Q * P.Nf[k];
        }
        const int g = fl_gate(f);
        if (g) {
            const ConD &cn = P.cons[g - 1];
            const double Cox = EPS_OX / (cn.tox > 0.0 ? cn.tox : 10e-9);
            const double pm = cn.phi_m > 0.0 ? cn.phi_m : P.Cref;
            const double rA = P.robA[k];
            fk += rA * (Cox * (cn.V + P.Cref - pm - pk) + cn.qox);
            dg += Cox * rA;
        }
        F[k] = fk;
        double sck;
        if (build) { P.A[0][k] = dg; P.sc[k] = dg; sck = dg; }
        else sck = P.sc[k];
        const double r = fk / sck;
        acc[0] += r * r;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 0)) P.res[R_PNORM] = sqrt(acc[0]);
}

// ------------------------------------------------------------------ mobility
// mobility tensor of a hexagonal crystal projected on the edge (ani_edge_g, :4235-4240)
__device__ __forceinline__ double ani_edge(const DevP &P, int k, int kp, double a) {
    if (P.caxis < 0 || !(a > 0.0) || a == 1.0) return 1.0;
    double dv[3], L2 = 0.0;
    for (int q = 0; q < 3; q++) { dv[q] = P.gpos[3 * kp + q] - P.gpos[3 * k + q]; L2 += dv[q] * dv[q]; }
    return L2 > 0.0 ? 1.0 + (a - 1.0) * dv[P.caxis] * dv[P.caxis] / L2 : 1.0;
}
// least-squares potential gradient of the semiconductor nodes within reach of a wall
// (qd < 0.5 m), zero elsewhere: the Lombardi field of the edges (upd_mob_ref_g, :4244-4250)
__device__ void g_grad(const DevP &P, const double *fld, int k, double *g);
__global__ void k_ggrad_g(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[0];
    SS_GRID_LOOP(k, P.N) {
        double g[3] = {0.0, 0.0, 0.0};
        if (fl_kind(P.flags[k]) == K_SEMI && P.qd[k] < 0.5) g_grad(P, P.phi, k, g);
        for (int q = 0; q < 3; q++) P.ggrad[3 * k + q] = g[q];
    }
}
// weight of velocity saturation of a node next to a metal contact for an edge of unit
// direction t (te_node_w, semiconductor_3d.c:813-817)
__device__ __forceinline__ double te_node_w_g(const DevP &P, int k, const double *t) {
    const double w = P.te_vw[k];
    if (w >= 1.0) return 1.0;
    const double c = t[P.te_ax[k]];
    return 1.0 - (1.0 - w) * c * c;
}
// edge mobilities, each undirected edge once (upd_mob_ref_g, semiconductor_3d.c:4241-4293):
// anisotropy projected on the edge, Lombardi surface scattering from the field normal to
// the edge (with the Coulomb term of 4H-SiC), Caughey-Thomas saturation tapered next to
// metal contacts
__global__ void k_upd_mob_g(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    const bool sat = (P.models & 4) != 0, lb = (P.models & 16) != 0;
    SS_GRID_LOOP(k, N) {
        const uint32_t f = P.flags[k];
        for (int s = 0; s < D; s++) {
            const size_t e = (size_t)s * N + k;
            const int kp = P.gcol[e];
            if (kp < k) continue;                  // padding (-1) and the lower half of each edge
            const int ue = P.gue[e];
            if (fl_kind(f) != K_SEMI || fl_kind(P.flags[kp]) != K_SEMI) { P.gmu_n[ue] = P.gmu_p[ue] = 0.0; continue; }
            const MatD &m = P.mats[fl_mat(f)];
            const double h = P.gh[e];
            double t[3];
            for (int q = 0; q < 3; q++) t[q] = (P.gpos[3 * kp + q] - P.gpos[3 * k + q]) / h;
            double mn = 0.5 * (P.mu0n[k] + P.mu0n[kp]), mp = 0.5 * (P.mu0p[k] + P.mu0p[kp]);
            mn *= ani_edge(P, k, kp, m.ani_n);
            mp *= ani_edge(P, k, kp, m.ani_p);
            if (lb && m.lb_on) {
                const double Dw = exp(-0.5 * (P.qd[k] + P.qd[kp]) / 1e-8);
                if (Dw > 1e-8) {
                    const double *ga = P.ggrad + 3 * (size_t)k, *gb = P.ggrad + 3 * (size_t)kp;
                    const double pa = ga[0] * t[0] + ga[1] * t[1] + ga[2] * t[2];
                    const double pb = gb[0] * t[0] + gb[1] * t[1] + gb[2] * t[2];
                    const double Fa = ga[0] * ga[0] + ga[1] * ga[1] + ga[2] * ga[2] - pa * pa;
                    const double Fb = gb[0] * gb[0] + gb[1] * gb[1] + gb[2] * gb[2] - pb * pb;
                    const double F = sqrt(fmax(0.5 * (Fa + Fb), 0.0));
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
            double wv = 0.0;
            if (sat) wv = P.te_vw ? 0.5 * (te_node_w_g(P, k, t) + te_node_w_g(P, kp, t)) : 1.0;
            if (wv > 0.0) {
                const double dps = P.phi[kp] - P.phi[k];
                const double Fn = heat_field(P.phin[kp] - P.phin[k], dps, h);
                const double Fp = heat_field(P.phip[kp] - P.phip[k], dps, h);
                const double sn = mob_hf(mn, Fn, m.vsat_n, m.beta_n), sp = mob_hf(mp, Fp, m.vsat_p, m.beta_p);
                mn += wv * (sn - mn);
                mp += wv * (sp - mp);
            }
            P.gmu_n[ue] = mn;
            P.gmu_p[ue] = mp;
        }
    }
}

// ------------------------------------------------------------------ continuity
// scaled Scharfetter-Gummel rows for u = c/s (cont_assemble_g, :4314-4351)
__global__ void k_cont_assemble_g(const DevP *__restrict__ Ps, int hole) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    const double *car = hole ? P.p : P.n;
    const double *mu = hole ? P.gmu_p : P.gmu_n;
    SS_GRID_LOOP(k, N) {
        const uint32_t f = P.flags[k];
        const bool semi = fl_kind(f) == K_SEMI;
        if (!semi || fl_fix(f)) {
            P.A[0][k] = 1.0;
            for (int s = 0; s < D; s++) P.gval[(size_t)s * N + k] = 0.0;
            P.rhs[k] = semi ? 1.0 : 0.0;
            P.sc[k] = semi ? car[k] : 0.0;
            P.dsc[k] = 0.0;
            continue;
        }
        const MatD &m = P.mats[fl_mat(f)];
        const double VT = m.VT, sk = fmax(car[k], NFLOOR);
        const double lk = hole ? lnvK(P, m, k) : lncK(P, m, k), pk = P.phi[k];
        double dg = 0.0, b = 0.0;
        for (int s = 0; s < D; s++) {
            const size_t e = (size_t)s * N + k;
            const int kb = P.gcol[e];
            P.gval[e] = 0.0;
            if (kb < 0) continue;
            const uint32_t fb = P.flags[kb];
            if (fl_kind(fb) != K_SEMI) continue;
            const MatD &mb = P.mats[fl_mat(fb)];
            const double lb = hole ? lnvK(P, mb, kb) : lncK(P, mb, kb);
            const double Dd = (P.phi[kb] - pk) / VT + (hole ? -(lb - lk) : (lb - lk));
            const double g = P.ga[e] * mu[P.gue[e]] * VT / P.gh[e];
            const double self = hole ? g * bern(Dd) : g * bern(-Dd);
            const double nb = hole ? g * bern(-Dd) : g * bern(Dd);
            dg += self;
            if (fl_fix(fb)) b += nb * car[kb];
            else P.gval[e] = -nb * fmax(car[kb], NFLOOR);
        }
        double R, dRn, dRp;
        recombK(P, m, k, P.n[k], P.p[k], R, dRn, dRp);
        double dR = hole ? dRp : dRn;
        if (dR < 0.0) dR = 0.0;
        const double vol = gvol(P, k);
        dg += vol * dR;
        b += vol * (dR * car[k] - R);
        if (P.tk) { dg += P.tk[k]; b += P.tg[k]; }   // gate / metal-contact exchange: sink tk c - tg
        if (P.gii) b += P.gii[k];                   // impact ionisation (pairs)
        const double w = 1.0 / (dg * sk);
        P.A[0][k] = 1.0;
        for (int s = 0; s < D; s++) P.gval[(size_t)s * N + k] *= w;
        P.rhs[k] = b * w;
        P.sc[k] = sk;
        P.dsc[k] = dg * sk;
    }
}

// SG flux through edge ka -> kb (face_flux_g, :4219-4229)
__device__ __forceinline__ void flux_g(const DevP &P, int ka, int kb, int ue, double h, double ar, double &Jn,
                                       double &Jp, double &Sn, double &Sp) {
    const MatD &ma = P.mats[fl_mat(P.flags[ka])];
    const MatD &mb = P.mats[fl_mat(P.flags[kb])];
    const double VT = ma.VT, dps = (P.phi[kb] - P.phi[ka]) / VT;
    const double Dn = dps + (lncK(P, mb, kb) - lncK(P, ma, ka)), Dp = dps - (lnvK(P, mb, kb) - lnvK(P, ma, ka));
    const double gn = Q * ar * P.gmu_n[ue] * VT / h, gp = Q * ar * P.gmu_p[ue] * VT / h;
    const double a1 = gn * P.n[kb] * bern(Dn), a2 = gn * P.n[ka] * bern(-Dn);
    const double b1 = gp * P.p[ka] * bern(Dp), b2 = gp * P.p[kb] * bern(-Dp);
    Jn = a1 - a2; Jp = b1 - b2; Sn = a1 + a2; Sp = b1 + b2;
}

// terminal currents: flux out of every contact's semiconductor nodes (terminal_flux_g,
// :4414-4426), per-block partials in P.partc, summed by the last block in block order
__global__ void k_currents_g(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[0];
    const int nc = P.ncon, N = P.N, D = P.gD;
    double *pc = P.partc;
    for (int c = 0; c < nc; c++) {
        double v[3] = {0.0, 0.0, 0.0};
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < P.ncnode; q += gridDim.x * blockDim.x) {
            const int k = P.cnode[q];
            if (fl_con(P.flags[k]) != c + 1 || P.cons[c].te) continue;   // metal contacts: te_currents
            for (int s = 0; s < D; s++) {
                const size_t e = (size_t)s * N + k;
                const int kb = P.gcol[e];
                if (kb < 0) continue;
                const uint32_t fb = P.flags[kb];
                if (fl_kind(fb) != K_SEMI || fl_con(fb) == c + 1) continue;
                double Jn, Jp, Sn, Sp;
                flux_g(P, k, kb, P.gue[e], P.gh[e], P.ga[e], Jn, Jp, Sn, Sp);
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
        is_last = atomicAdd(P.ticket + 7, 1u) == gridDim.x - 1;
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
    if (threadIdx.x == 0) P.ticket[7] = 0u;
}

// node current-density vector from the edge fluxes by least squares (g_node_J, :4428-4452);
// which: 0 total, 1 electrons, 2 holes
__device__ void node_J_g(const DevP &P, int k, int which, double *J) {
    const int N = P.N, D = P.gD;
    double M[6] = {0, 0, 0, 0, 0, 0}, r[3] = {0, 0, 0};
    J[0] = J[1] = J[2] = 0.0;
    if (fl_kind(P.flags[k]) != K_SEMI) return;
    for (int s = 0; s < D; s++) {
        const size_t e = (size_t)s * N + k;
        const int kb = P.gcol[e];
        if (kb < 0 || fl_kind(P.flags[kb]) != K_SEMI) continue;
        const double h = P.gh[e], ar = P.ga[e];
        double t[3], Jn, Jp, Sn, Sp;
        for (int q = 0; q < 3; q++) t[q] = (P.gpos[3 * kb + q] - P.gpos[3 * k + q]) / h;
        flux_g(P, k, kb, P.gue[e], h, ar, Jn, Jp, Sn, Sp);
        const double j = (which == 1 ? Jn : (which == 2 ? Jp : Jn + Jp)) / (ar > 0.0 ? ar : 1e-300);
        const double w = ar;
        M[0] += w * t[0] * t[0]; M[1] += w * t[0] * t[1]; M[2] += w * t[0] * t[2];
        M[3] += w * t[1] * t[1]; M[4] += w * t[1] * t[2]; M[5] += w * t[2] * t[2];
        r[0] += w * t[0] * j; r[1] += w * t[1] * j; r[2] += w * t[2] * j;
    }
    const double tr = M[0] + M[3] + M[5], eps = 1e-6 * tr + 1e-300;
    M[0] += eps; M[3] += eps; M[5] += eps;
    const double a = M[0], b = M[1], c = M[2], dd = M[3], ee = M[4], ff = M[5];
    const double A = dd * ff - ee * ee, Bq = -(b * ff - c * ee), Cc = b * ee - c * dd, Dq = a * ff - c * c,
                 E = -(a * ee - b * c), F = a * dd - b * b;
    const double det = a * A + b * Bq + c * Cc;
    if (!(fabs(det) > 0.0)) return;
    J[0] = (A * r[0] + Bq * r[1] + Cc * r[2]) / det;
    J[1] = (Bq * r[0] + Dq * r[1] + E * r[2]) / det;
    J[2] = (Cc * r[0] + E * r[1] + F * r[2]) / det;
}

// display current density and recombination (upd_J_g, :4453-4463)
__global__ void k_upd_J_g(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[0];
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        if (fl_kind(f) != K_SEMI) { P.Jx[k] = P.Jy[k] = P.Jz[k] = 0.0; P.Rt[k] = 0.0; continue; }
        double J[3];
        node_J_g(P, k, 0, J);
        P.Jx[k] = J[0]; P.Jy[k] = J[1]; P.Jz[k] = J[2];
        double R, a, b;
        recombK(P, P.mats[fl_mat(f)], k, P.n[k], P.p[k], R, a, b);
        P.Rt[k] = R;
    }
}
// display mobility: mean of the node's edge mobilities across the c-axis (mob_display_g, :4295-4312)
__global__ void k_mob_display_g(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    SS_GRID_LOOP(k, N) {
        const uint32_t f = P.flags[k];
        if (fl_kind(f) != K_SEMI) { P.mudn[k] = 0.0; P.mudp[k] = 0.0; continue; }
        double sn = 0.0, sp = 0.0;
        int c = 0;
        for (int s = 0; s < D; s++) {
            const size_t e = (size_t)s * N + k;
            const int kb = P.gcol[e];
            if (kb < 0 || fl_kind(P.flags[kb]) != K_SEMI) continue;
            const MatD &m = P.mats[fl_mat(P.flags[k < kb ? k : kb])];
            sn += P.gmu_n[P.gue[e]] / ani_edge(P, k, kb, m.ani_n);
            sp += P.gmu_p[P.gue[e]] / ani_edge(P, k, kb, m.ani_p);
            c++;
        }
        if (c) { P.mudn[k] = sn / c; P.mudp[k] = sp / c; }
        else { P.mudn[k] = P.mu0n[k]; P.mudp[k] = P.mu0p[k]; }
    }
}
// Jn / Jp components by least squares (node_val 20..25 on a graph, :5053-5056)
__global__ void k_node_Jc_g(const DevP *__restrict__ Ps, int which, double *out) {
    const DevP &P = Ps[0];
    const int ax = (which - 20) % 3, hole = which >= 23;
    SS_GRID_LOOP(k, P.N) {
        double J[3];
        node_J_g(P, k, 1 + hole, J);
        out[k] = fl_kind(P.flags[k]) == K_SEMI ? J[ax] : 0.0;
    }
}
// least-squares gradient of a node field over the node's semiconductor neighbours
// (g_grad, semiconductor_3d.c:2702-2714): g = M^-1 sum_e (f_b - f_k) dr_e / |dr_e|^2
__device__ void g_grad(const DevP &P, const double *fld, int k, double *g) {
    const int N = P.N, D = P.gD;
    double r[3] = {0, 0, 0};
    if (fl_kind(P.flags[k]) == K_SEMI)
        for (int s = 0; s < D; s++) {
            const int b = P.gcol[(size_t)s * N + k];
            if (b < 0 || fl_kind(P.flags[b]) != K_SEMI) continue;
            const double dx = P.gpos[3 * b] - P.gpos[3 * k], dy = P.gpos[3 * b + 1] - P.gpos[3 * k + 1],
                         dz = P.gpos[3 * b + 2] - P.gpos[3 * k + 2];
            const double w = (fld[b] - fld[k]) / (dx * dx + dy * dy + dz * dz + 1e-40);
            r[0] += w * dx; r[1] += w * dy; r[2] += w * dz;
        }
    const double *m = P.glsq + 6 * (size_t)k;
    g[0] = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
    g[1] = m[1] * r[0] + m[3] * r[1] + m[4] * r[2];
    g[2] = m[2] * r[0] + m[4] * r[1] + m[5] * r[2];
}
// the largest field (Emax_g, semiconductor_3d.c:4557-4565)
__global__ void k_emax_g(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[0];
    double mx = 0.0;
    SS_GRID_LOOP(k, P.N) {
        if (fl_kind(P.flags[k]) != K_SEMI) continue;
        double g[3];
        g_grad(P, P.phi, k, g);
        mx = fmax(mx, g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    }
    if (grid_max(mx, P.part, P.ticket + 8)) P.res[R_OUT] = mx;
}
// impact-ionisation pair generation on the graph: node current densities of each carrier
// and the field by least squares (ii_update, semiconductor_3d.c:4490-4523); total -> res[R_GII]
__global__ void k_ii_update_g(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[0];
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, P.N) {
        const uint32_t f = P.flags[k];
        double gk = 0.0;
        const MatD &m = P.mats[fl_mat(f)];
        if (fl_kind(f) == K_SEMI && !fl_fix(f) && m.ii_on) {
            double Jn[3], Jp[3], g[3], E[3];
            node_J_g(P, k, 1, Jn);
            node_J_g(P, k, 2, Jp);
            g_grad(P, P.phi, k, g);
            for (int q = 0; q < 3; q++) E[q] = -g[q];
            double G = 0.0;
            for (int c = 0; c < 2; c++) {
                const double *J = c ? Jp : Jn;
                const double jj = sqrt(J[0] * J[0] + J[1] * J[1] + J[2] * J[2]);
                if (!(jj > 0.0)) continue;
                const double F = fabs(E[0] * J[0] + E[1] * J[1] + E[2] * J[2]) / jj;
                G += ii_alpha(m, F, c) * jj;
            }
            gk = G / Q * gvol(P, k);
        }
        P.gii[k] = gk;
        acc[0] += gk;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 9)) P.res[R_GII] = acc[0];
}

// ------------------------------------------------------------------ linear algebra
// y = A x (ELL off-diagonals + the diagonal in A[0])
__global__ void k_matvec_g(const DevP *__restrict__ Ps, const double *__restrict__ x, double *__restrict__ y) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    SS_GRID_LOOP(k, N) {
        double s = P.A[0][k] * x[k];
        for (int q = 0; q < D; q++) {
            const size_t e = (size_t)q * N + k;
            const int j = P.gcol[e];
            if (j >= 0) s += P.gval[e] * x[j];
        }
        y[k] = s;
    }
}
// sums of a.b (and b.b) over all nodes -> res[slot], res[slot + 1]
__global__ void k_dot2_g(const DevP *__restrict__ Ps, const double *a, const double *b, int slot) {
    const DevP &P = Ps[0];
    double acc[2] = {0.0, 0.0};
    SS_GRID_LOOP(k, P.N) { acc[0] += a[k] * b[k]; acc[1] += b[k] * b[k]; }
    if (grid_sum<2>(acc, P.part, P.ticket + 9)) { P.res[slot] = acc[0]; P.res[slot + 1] = acc[1]; }
}
// y = a x + b y + c z (any of x, z may be null)
__global__ void k_lin_g(int N, double *y, double b, const double *x, double a, const double *z, double c) {
    SS_GRID_LOOP(k, N) {
        double v = b * y[k];
        if (x) v += a * x[k];
        if (z) v += c * z[k];
        y[k] = v;
    }
}
// rounding floor of a continuity system: sum over rows of (sum |A_ab x_b| + |b_a|)^2 (gfloor)
__global__ void k_floor_g(const DevP *__restrict__ Ps, const double *b, const double *x, int slot) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    double acc[1] = {0.0};
    SS_GRID_LOOP(k, N) {
        double s = fabs(P.A[0][k] * x[k]) + fabs(b[k]);
        for (int q = 0; q < D; q++) {
            const size_t e = (size_t)q * N + k;
            const int j = P.gcol[e];
            if (j >= 0) s += fabs(P.gval[e] * x[j]);
        }
        acc[0] += s * s;
    }
    if (grid_sum<1>(acc, P.part, P.ticket + 9)) P.res[slot] = acc[0];
}

// ------------------------------------------------------------------ labelling
// floating blocks: labels take the smallest label of a labelled neighbour
__global__ void k_ff_prop_g(const DevP *__restrict__ Ps, int *changed) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    int *lab = P.ccl;
    int ch = 0;
    SS_GRID_LOOP(k, N) {
        int a = lab[k];
        if (a < 0) continue;
        for (int q = 0; q < D; q++) {
            const int j = P.gcol[(size_t)q * N + k];
            if (j < 0) continue;
            const int b = lab[j];
            if (b >= 0 && b < a) a = b;
        }
        if (a < lab[k]) { lab[k] = a; ch = 1; }
    }
    if (ch) *changed = 1;
}
__global__ void k_ff_anchor_g(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    SS_GRID_LOOP(k, N) {
        const int lb = P.ccl[k];
        if (lb < 0) continue;
        for (int q = 0; q < D; q++) {
            const int j = P.gcol[(size_t)q * N + k];
            if (j < 0) continue;
            const uint32_t fb = P.flags[j];
            if (fl_kind(fb) == K_SEMI && fl_con(fb)) { P.cclaux[lb] = 1; break; }
        }
    }
}
__device__ __forceinline__ int ff_block_g(const DevP &P, int k) {
    const int lb = P.ccl[k];
    if (lb < 0) return -1;
    const int a = P.cclaux[lb];
    return a >= 2 ? a - 2 : -1;
}
// boundary balance of every block: Aout = sum self s_k u_k, Bin = sum nb c_b (float_fix_g, :4371-4385)
__global__ void k_ff_boundary_g(const DevP *__restrict__ Ps, int hole, unsigned long long *Aout,
                                unsigned long long *Bin) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    const double *mu = hole ? P.gmu_p : P.gmu_n;
    SS_GRID_LOOP(k, N) {
        const int b = ff_block_g(P, k);
        if (b < 0) continue;
        const MatD &m = P.mats[fl_mat(P.flags[k])];
        const double VT = m.VT, lk = hole ? lnvK(P, m, k) : lncK(P, m, k);
        const double ck = P.sc[k] * P.sol[k];
        double ao = 0.0, bi = 0.0;
        for (int q = 0; q < D; q++) {
            const size_t e = (size_t)q * N + k;
            const int kb = P.gcol[e];
            if (kb < 0) continue;
            const uint32_t fb = P.flags[kb];
            if (fl_kind(fb) != K_SEMI || P.ccl[kb] == P.ccl[k]) continue;
            const MatD &mb = P.mats[fl_mat(fb)];
            const double lb = hole ? lnvK(P, mb, kb) : lncK(P, mb, kb);
            const double Dd = (P.phi[kb] - P.phi[k]) / VT + (hole ? -(lb - lk) : (lb - lk));
            const double g = P.ga[e] * mu[P.gue[e]] * VT / P.gh[e];
            const double self = hole ? g * bern(Dd) : g * bern(-Dd), nb = hole ? g * bern(-Dd) : g * bern(Dd);
            const double cb = fl_con(fb) ? (hole ? P.p[kb] : P.n[kb]) : P.sc[kb] * P.sol[kb];
            ao += self * ck;
            bi += nb * cb;
        }
        xs_add(Aout + (size_t)b * XS_WORDS, ao);
        xs_add(Bin + (size_t)b * XS_WORDS, bi);
    }
}
// majority region of contact c1 grown over the graph (region_shift_g, :4525-4556)
__global__ void k_region_prop_g(const DevP *__restrict__ Ps, int c1, int type, int *mark, int *changed) {
    const DevP &P = Ps[0];
    const int N = P.N, D = P.gD;
    int ch = 0;
    SS_GRID_LOOP(k, N) {
        if (mark[k]) continue;
        const uint32_t f = P.flags[k];
        if (fl_kind(f) != K_SEMI) continue;
        const int c = fl_con(f);
        if (c && c != c1) continue;
        const double Dn = P.Nd[k] - P.Na[k];
        if (Dn * type <= 0.0) continue;
        const double maj = type > 0 ? P.n[k] : P.p[k];
        if (maj < 0.5 * fabs(Dn)) continue;
        for (int q = 0; q < D; q++) {
            const int j = P.gcol[(size_t)q * N + k];
            if (j >= 0 && mark[j] == c1) { mark[k] = c1; ch = 1; break; }
        }
    }
    if (ch) *changed = 1;
}

// ------------------------------------------------------------------ host drivers
static dim3 gblocks(const Ctx &c) { return dim3(c.nodes_blocks(), 1); }

void launch_poisson_g(const Ctx &c, const double *phi_sel, int build) {
    SS_LAUNCH(PF_POISSON, c.maxN, k_poisson_g, gblocks(c), TPB, c.st, c.dP, phi_sel ? 1 : 0, build);
}
void launch_upd_mob_g(const Ctx &c) {
    if (c.h.models & 16) SS_LAUNCH(PF_UPDMOB, c.maxN, k_ggrad_g, gblocks(c), TPB, c.st, c.dP);
    SS_LAUNCH(PF_UPDMOB, c.maxN, k_upd_mob_g, gblocks(c), TPB, c.st, c.dP);
}
void launch_cont_assemble_g(const Ctx &c, int hole) {
    SS_LAUNCH(PF_CONT_ASM, c.maxN, k_cont_assemble_g, gblocks(c), TPB, c.st, c.dP, hole);
}
void launch_currents_g(const Ctx &c) {
    int nb = (c.h.ncnode + TPB - 1) / TPB;
    if (nb < 1) nb = 1;
    if (nb > 256) nb = 256;
    SS_LAUNCH(PF_CURRENTS, c.h.ncnode, k_currents_g, dim3(nb, 1), TPB, c.st, c.dP);
}
void launch_upd_J_g(const Ctx &c) { SS_LAUNCH(PF_DISPLAY, c.maxN, k_upd_J_g, gblocks(c), TPB, c.st, c.dP); }
void launch_mob_display_g(const Ctx &c) { SS_LAUNCH(PF_DISPLAY, c.maxN, k_mob_display_g, gblocks(c), TPB, c.st, c.dP); }
void launch_node_Jc_g(const Ctx &c, int which, double *out) {
    SS_LAUNCH(PF_DISPLAY, c.maxN, k_node_Jc_g, gblocks(c), TPB, c.st, c.dP, which, out);
}
void launch_emax_g(const Ctx &c) { SS_LAUNCH(PF_DISPLAY, c.maxN, k_emax_g, gblocks(c), TPB, c.st, c.dP); }
void launch_ii_update_g(const Ctx &c) { SS_LAUNCH(PF_DISPLAY, c.maxN, k_ii_update_g, gblocks(c), TPB, c.st, c.dP); }

namespace {
double rd(Inst &d, int slot) {
    cudaMemcpyAsync(d.g.pin, d.g.h.res + slot, sizeof(double), cudaMemcpyDeviceToHost, d.g.st);
    cudaStreamSynchronize(d.g.st);
    return d.g.pin[0];
}
void rd2(Inst &d, int slot, double &a, double &b) {
    cudaMemcpyAsync(d.g.pin, d.g.h.res + slot, 2 * sizeof(double), cudaMemcpyDeviceToHost, d.g.st);
    cudaStreamSynchronize(d.g.st);
    a = d.g.pin[0];
    b = d.g.pin[1];
}
constexpr int RG = R_OUT + 8;           // result slots of the graph solves (112..115)
void matvec(const Ctx &c, const double *x, double *y) {
    SS_LAUNCH(PF_KRY_SPMV_DOT, c.maxN, k_matvec_g, gblocks(c), TPB, c.st, c.dP, x, y);
}
void lin(const Ctx &c, double *y, double b, const double *x, double a, const double *z = nullptr, double cc = 0.0) {
    SS_LAUNCH(PF_KRY_UPDATE, c.maxN, k_lin_g, gblocks(c), TPB, c.st, (int)c.h.N, y, b, x, a, z, cc);
}
double dot(Inst &d, const Ctx &c, const double *a, const double *b, double *bb = nullptr) {
    SS_LAUNCH(PF_KRY_DOT, c.maxN, k_dot2_g, gblocks(c), TPB, c.st, c.dP, a, b, RG);
    double x, y;
    rd2(d, RG, x, y);
    if (bb) *bb = y;
    return x;
}
}  // namespace

// PCG on the graph system with the reference's stop rule r.z <= rtol^2 r0.z0
// (pcg, semiconductor_3d.c:2182-2210), preconditioned by one V-cycle of the aggregation
// multigrid; x = P.sol, b = P.rhs; returns the iterations
int pcg_graph(Inst &d, int maxit, double rtol) {
    Ctx c = make_ctx(d);
    double *x = d.g.h.sol, *b = d.g.h.rhs;
    double *r = d.g.h.wk[0], *z = d.g.h.wk[1], *p = d.g.h.wk[2], *q = d.g.h.wk[3];
    gmg_setup(d, c, 0, nullptr);
    if (persist_enabled()) {                      // the whole solve in one persistent launch
        lin(c, d.g.h.wk[7], 0.0, x, 1.0);        // start backup
        const int pr = persist_graph(d, 0, maxit, rtol, 0.0, nullptr, false);
        if (pr == 1) {
            KrylovS hs{};
            cudaMemcpyAsync(&hs, c.h.ks, sizeof(KrylovS), cudaMemcpyDeviceToHost, c.st);
            cudaStreamSynchronize(c.st);
            return hs.it;
        }
        if (pr < 0) lin(c, x, 0.0, d.g.h.wk[7], 1.0);
    }
    matvec(c, x, q);
    lin(c, r, 0.0, b, 1.0, q, -1.0);
    gmg_apply(d, c, r, z, nullptr, false);
    double rz = dot(d, c, r, z), rz0 = rz;
    if (!(rz0 > 0.)) return 0;
    lin(c, p, 0.0, z, 1.0);
    int it;
    for (it = 1; it <= maxit; it++) {
        if (g_stop.load()) break;
        matvec(c, p, q);
        const double pq = dot(d, c, p, q);
        if (!(pq > 0.)) break;
        const double al = rz / pq;
        lin(c, x, 1.0, p, al);
        lin(c, r, 1.0, q, -al);
        gmg_apply(d, c, r, z, nullptr, false);
        const double rzn = dot(d, c, r, z);
        if (!(rzn > rtol * rtol * rz0)) break;
        const double be = rzn / rz;
        rz = rzn;
        lin(c, p, be, z, 1.0);
    }
    if (it > maxit) it = maxit;
    return it;
}

// right-preconditioned BiCGSTAB (bicgstab_core, semiconductor_3d.c:2230-2320): stops at
// ||r|| <= max(rtol ||r0||, atol sqrt(floor)), breakdown restarts, 40 stalled iterations;
// preconditioned by one V-cycle of the aggregation multigrid with the Slotboom weights of
// carrier qsign (or the mesh level's D-ILU alone); x = P.sol, b = P.rhs.  Returns the
// iterations; *rn the final and *r0 the initial residual.
int bicg_graph(Inst &d, int maxit, double rtol, double atol, double *rn_out, double *r0_out, int qsign,
               bool ilu_only) {
    Ctx c = make_ctx(d);
    double *x = d.g.h.sol, *b = d.g.h.rhs;
    double *r = d.g.h.wk[0], *rh = d.g.h.wk[1], *p = d.g.h.wk[2], *v = d.g.h.wk[3], *ph = d.g.h.wk[4],
           *sh = d.g.h.wk[5], *t = d.g.h.wk[6];
    const double *w = d.g.h.dsc;
    gmg_setup(d, c, qsign, w);
    if (persist_enabled()) {                      // the whole solve in one persistent launch
        lin(c, d.g.h.wk[7], 0.0, x, 1.0);        // start backup
        const int pr = persist_graph(d, 1, maxit, rtol, atol, w, ilu_only);
        if (pr == 1) {
            KrylovS hs{};
            cudaMemcpyAsync(&hs, c.h.ks, sizeof(KrylovS), cudaMemcpyDeviceToHost, c.st);
            cudaStreamSynchronize(c.st);
            *r0_out = hs.r0;
            *rn_out = std::sqrt(hs.rr);
            return hs.it;
        }
        if (pr < 0) lin(c, x, 0.0, d.g.h.wk[7], 1.0);
    }
    matvec(c, x, t);
    lin(c, r, 0.0, b, 1.0, t, -1.0);
    lin(c, rh, 0.0, r, 1.0);
    lin(c, p, 0.0, nullptr, 0.0);
    lin(c, v, 0.0, nullptr, 0.0);
    double rr;
    dot(d, c, r, r, &rr);
    SS_LAUNCH(PF_KRY_DOT, c.maxN, k_floor_g, gblocks(c), TPB, c.st, c.dP, b, x, RG + 2);
    const double fl = rd(d, RG + 2);
    const double r0 = std::sqrt(rr), tgt = std::fmax(rtol * r0, atol * std::sqrt(fl));
    *r0_out = r0;
    *rn_out = r0;
    if (!(r0 > tgt)) return 0;
    double rho = 1., al = 1., om = 1., rbest = r0;
    int stall = 0, it;
    for (it = 1; it <= maxit; it++) {
        if (g_stop.load()) break;
        double rho1 = dot(d, c, rh, r);
        if (std::fabs(rho1) < 1e-300) {             // breakdown: restart the shadow residual
            lin(c, rh, 0.0, r, 1.0);
            lin(c, p, 0.0, nullptr, 0.0);
            lin(c, v, 0.0, nullptr, 0.0);
            rho1 = dot(d, c, r, r);
            rho = al = om = 1.;
            if (!(rho1 > 0.)) break;
        }
        const double be = (rho1 / rho) * (al / om);
        lin(c, p, be, r, 1.0, v, -be * om);          // p = r + be (p - om v)
        gmg_apply(d, c, p, ph, w, ilu_only);
        matvec(c, ph, v);
        const double rv = dot(d, c, rh, v);
        if (std::fabs(rv) < 1e-300) break;
        al = rho1 / rv;
        lin(c, r, 1.0, v, -al);
        double ss;
        dot(d, c, r, r, &ss);
        if (std::sqrt(ss) <= tgt) {
            lin(c, x, 1.0, ph, al);
            rr = ss;
            break;
        }
        gmg_apply(d, c, r, sh, w, ilu_only);
        matvec(c, sh, t);
        double tt;
        const double ts = dot(d, c, r, t, &tt);     // ts = r.t, tt = t.t
        om = tt > 0. ? ts / tt : 0.;
        lin(c, x, 1.0, ph, al, sh, om);
        lin(c, r, 1.0, t, -om);
        dot(d, c, r, r, &rr);
        const double rn = std::sqrt(rr);
        if (rn <= tgt || om == 0.) break;
        if (rn < 0.99 * rbest) { rbest = rn; stall = 0; }
        else if (++stall > 40) break;
        rho = rho1;
    }
    if (it > maxit) it = maxit;
    *rn_out = std::sqrt(rr);
    return it;
}

// floating majority blocks of the graph: label, anchor, boundary (float_fix_g); the
// recombination balance and the rescaling are the tensor path's node-wise kernels
int ff_label_g(Inst &d, int *changed) {
    Ctx c = make_ctx(d);
    int h = 1, cycles = 0;
    const int maxcyc = (int)d.N + 8;
    while (h && cycles < maxcyc) {
        cudaMemsetAsync(changed, 0, sizeof(int), c.st);
        for (int q = 0; q < 8; q++) SS_LAUNCH(PF_CCL, d.N, k_ff_prop_g, gblocks(c), TPB, c.st, c.dP, changed);
        cudaMemcpyAsync(&h, changed, sizeof(int), cudaMemcpyDeviceToHost, c.st);
        cudaStreamSynchronize(c.st);
        cycles += 8;
    }
    SS_LAUNCH(PF_CCL, d.N, k_ff_anchor_g, gblocks(c), TPB, c.st, c.dP);
    return 1;
}
void ff_boundary_g(Inst &d, int hole, unsigned long long *Aout, unsigned long long *Bin) {
    Ctx c = make_ctx(d);
    SS_LAUNCH(PF_CCL, d.N, k_ff_boundary_g, gblocks(c), TPB, c.st, c.dP, hole, Aout, Bin);
}
void launch_region_mark_g(Inst &d, int c1, int type, double dV, int *mark, int *changed) {
    Ctx c = make_ctx(d);
    launch_region_seed(c, c1, mark);
    region_grow_g(d, c1, type, mark, changed);
    launch_region_shift(c, c1, dV, mark);
}
void region_grow_g(Inst &d, int c1, int type, int *mark, int *changed) {
    Ctx c = make_ctx(d);
    int h = 1, cycles = 0;
    const int maxcyc = (int)d.N + 8;
    while (h && cycles < maxcyc) {
        cudaMemsetAsync(changed, 0, sizeof(int), c.st);
        for (int q = 0; q < 8; q++) SS_LAUNCH(PF_CCL, d.N, k_region_prop_g, gblocks(c), TPB, c.st, c.dP, c1, type, mark, changed);
        cudaMemcpyAsync(&h, changed, sizeof(int), cudaMemcpyDeviceToHost, c.st);
        cudaStreamSynchronize(c.st);
        cycles += 8;
    }
}

}  // namespace ss
