// Thermionic-emission metal contacts (models bit 6) with image-force lowering and, with
// models bit 7, Tsu-Esaki tunnelling through the barrier (semiconductor_3d.c:3390-3571).
//
// A semiconductor node of a metal face contact exchanges carriers with the metal at the
// Richardson velocity v = A** T^2 / (q N) towards the density in equilibrium with the metal
// Fermi level; the interface field lowers the barrier of the carrier it pushes away from
// the metal (image force, screened by the free carriers along the node's column), and with
// tunnelling a carrier below the barrier top tunnels (WKB through the band along the column)
// to the node where its energy meets the band.
//
// One thread per contact entry computes the image-force lowering of its column, its
// emission coefficients and its tunnelling terms (the entry owns its column's slots, so
// nothing races); gathers over the column nodes (CSR, ascending entry order) give the
// per-node band lowering, and the exchange gather of tunnel.cu the continuity sink / source,
// in the reference's summation order.
#include "device_common.cuh"
#include "physics_hd.cuh"
#include "prof.h"
#include "solver_ctx.h"

namespace ss {

constexpr double PI_D = 3.14159265358979323846;

// image-force lowering along the column of entry t (te_img, semiconductor_3d.c:3422-3445):
// the interface field F sets dphi = sqrt(qF / 4 pi eps) (at most 1 V) and the barrier
// maximum x_m = dphi / 2F; the carrier pushed away from the metal sees the flat top up to
// x_m and q / (16 pi eps s) beyond, screened by exp(-2 int ds / lambda_Debye)
__global__ void k_te_img(const DevP *__restrict__ Ps, TeD T) {
    const DevP &P = Ps[0];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T.n_te) return;
    const int k = T.te_k[t], q0 = T.te_c0[t], nq = T.te_cn[t];
    const MatD &m = P.mats[fl_mat(P.flags[k])];
    const double eps = m.eps, VT = m.VT;
    double F = 0.0;
    if (nq > 1) {
        const int k1 = T.tc_k[q0 + 1];
        const double h = T.tc_s[q0 + 1];
        if (h > 0.0) F = (P.phi[k1] - P.phi[k]) / h;
    }
    const int hole = F < 0.0;
    const double Fa = fabs(F);
    double dph = Fa > 0.0 ? sqrt(Q * Fa / (4.0 * PI_D * eps)) : 0.0;
    if (dph > 1.0) dph = 1.0;
    const double xm = dph > 0.0 ? dph / (2.0 * Fa) : 0.0;
    double S = 0.0, li0 = 0.0, s0 = 0.0;
    for (int q = q0; q < q0 + nq; q++) {
        const int kq = T.tc_k[q];
        const double s = T.tc_s[q];
        const MatD &mq = P.mats[fl_mat(P.flags[kq])];
        const double cq = P.n[kq] + P.p[kq];
        const double li = cq > 0.0 ? sqrt(Q * cq / (mq.eps * mq.VT)) : 0.0;
        if (q > q0) S += 0.5 * (li + li0) * (s - s0);
        li0 = li;
        s0 = s;
        double dl = 0.0;
        if (dph > 0.0 && S < 20.0) {
            dl = s < xm ? dph - Fa * s : Q / (16.0 * PI_D * eps * s);
            dl *= exp(-2.0 * S);
        }
        T.tc_I[2 * q + hole] = dl / VT;
        T.tc_I[2 * q + 1 - hole] = 0.0;
    }
}

// band lowering of every column node: the largest of its columns replaces the node's
// previous image-force part of qcn / qcp, in the reference's order of operations
// (te_apply_img, semiconductor_3d.c:3448-3462)
__global__ void k_te_apply(const DevP *__restrict__ Ps, TeD T) {
    const DevP &P = Ps[0];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.n_touch) return;
    double mn = 0.0, mp = 0.0;
    for (int e = T.tn_ptr[i]; e < T.tn_ptr[i + 1]; e++) {
        const int q = T.tn_q[e];
        if (T.tc_I[2 * q] > mn) mn = T.tc_I[2 * q];
        if (T.tc_I[2 * q + 1] > mp) mp = T.tc_I[2 * q + 1];
    }
    const int k = T.tn_k[i];
    P.qcn[k] = (P.qcn[k] - P.imgn[k]) + mn;
    P.qcp[k] = (P.qcp[k] - P.imgp[k]) + mp;
    P.imgn[k] = mn;
    P.imgp[k] = mp;
}

// exchange with the metal at entry t (te_one, semiconductor_3d.c:3467-3533): emission
// coefficients K (sink K c) and G (source) of both carriers at the entry node, written to
// te_K / te_G and to the entry node's column slot; with models bit 7 the tunnelling terms
// of the column nodes, linearised in the turning-point densities
__global__ void __launch_bounds__(64) k_te_one(const DevP *__restrict__ Ps, TeD T) {
    const DevP &P = Ps[0];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T.n_te) return;
    const int k = T.te_k[t], c = T.te_c[t], q0 = T.te_c0[t], nq = T.te_cn[t];
    const MatD &m = P.mats[fl_mat(P.flags[k])];
    const double VT = m.VT, Tk = m.T, A = T.te_A[t], V = P.cons[c].V;
    const double vn = m.rich_n * Tk * Tk / (Q * m.Nc), vp = m.rich_p * Tk * Tk / (Q * m.Nv);
    const double n0 = nK(P, m, k, P.phi[k], V), p0 = pK(P, m, k, P.phi[k], V);
    T.te_K[2 * t] = A * vn; T.te_G[2 * t] = A * vn * n0;
    T.te_K[2 * t + 1] = A * vp; T.te_G[2 * t + 1] = A * vp * p0;
    for (int q = q0; q < q0 + nq; q++) T.tc_K[2 * q] = T.tc_K[2 * q + 1] = T.tc_G[2 * q] = T.tc_G[2 * q + 1] = 0.0;
    T.tc_K[2 * q0] = T.te_K[2 * t]; T.tc_K[2 * q0 + 1] = T.te_K[2 * t + 1];
    T.tc_G[2 * q0] = T.te_G[2 * t]; T.tc_G[2 * q0 + 1] = T.te_G[2 * t + 1];
    if (!(T.models & 128) || nq < 2) return;
    const int nn = nq < TE_NNMAX ? nq : TE_NNMAX;
    double u[TE_NNMAX];
    const double EFm = -V - P.Cref;
    for (int hole = 0; hole < 2; hole++) {
        // band along the carrier's direction: electrons u = Ec, holes u = -Ev (image force
        // included), so the algebra is the same for both
        for (int i = 0; i < nn; i++) {
            const int kq = T.tc_k[q0 + i];
            const MatD &mq = P.mats[fl_mat(P.flags[kq])];
            const double Ec = -P.phi[kq] - mq.chi - VT * (bgn_of(P, kq) + qcn_of(P, kq));
            const double Ev = -P.phi[kq] - mq.chi - mq.Eg + VT * (bgn_of(P, kq) + qcp_of(P, kq));
            u[i] = hole ? -Ev : Ec;
        }
        const double top = fmax(u[0], u[1]);
        double umin = u[1];
        for (int i = 2; i < nn; i++) if (u[i] < umin) umin = u[i];
        if (!(top - umin > 2.0 * VT)) continue;           // no barrier to tunnel through
        double mt = hole ? m.mtun_h : m.mtun_e;
        if (!(mt > 0.0)) mt = 0.3;
        const double rich = hole ? m.rich_p : m.rich_n;
        const double Cr = A * rich * Tk / (KB / Q) / Q;
        const double eFm = hole ? -EFm : EFm;
        const double h = (top - umin) / TE_NE;
        for (int jq = 0; jq <= TE_NE; jq++) {
            const double e = umin + jq * h;
            const double w = h / 3.0 * (jq == 0 || jq == TE_NE ? 1.0 : (jq & 1 ? 4.0 : 2.0));
            double sw = 0.0, fr = 1.0;
            int it = -1;
            for (int i = 0; i + 1 < nn; i++) {
                const double L = T.tc_s[q0 + i + 1] - T.tc_s[q0 + i], a0 = u[i] - e, a1 = u[i + 1] - e;
                sw += wkb_seg(mt, L, a0, a1);
                if (a1 <= 0.0) { it = i + 1; fr = a0 > 0.0 ? a0 / (a0 - a1) : 0.0; break; }
                if (sw > 230.0) break;
            }
            if (it < 1 || sw > 230.0) continue;
            const double Sx = Cr * w * exp(-sw);
            const double Lm = softplus((eFm - e) / VT);
            // the turning point lies a fraction fr into segment it-1..it: its inflow is
            // shared linearly by the two nodes, never put on the interface node itself
            const int nd = it >= 2 ? 2 : 1;
            for (int j = 0; j < nd; j++) {
                const int qi = q0 + (j == 0 ? it : it - 1);
                const double wt = nd == 1 ? 1.0 : (j == 0 ? fr : 1.0 - fr);
                if (!(wt > 0.0)) continue;
                const int ki = T.tc_k[qi];
                const double eFi = hole ? P.phip[ki] + P.Cref : -P.phin[ki] - P.Cref;
                const double ci = hole ? P.p[ki] : P.n[ki];
                const double zs = (eFi - e) / VT, Ls = softplus(zs);
                const double z = exp(fmin(zs, 700.0)), dLs = ci > 0.0 ? z / ((1.0 + z) * ci) : 0.0;
                T.tc_K[2 * qi + hole] += Sx * wt * dLs;
                T.tc_G[2 * qi + hole] += Sx * wt * (Lm - Ls + dLs * ci);
            }
        }
    }
}

// terminal current of the metal contacts (te_currents, semiconductor_3d.c:3555-3571), added
// to the face-flux currents of the other contacts: one block, each contact's entries summed
// by the block in a fixed order
constexpr int TE_CUR_TPB = 256;
__global__ void __launch_bounds__(TE_CUR_TPB) k_te_currents(const DevP *__restrict__ Ps, TeD T) {
    const DevP &P = Ps[0];
    __shared__ double sh[3][TE_CUR_TPB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int c = 0; c < P.ncon; c++) {
        if (T.ce1[c] <= T.ce0[c]) continue;
        double v[3] = {0.0, 0.0, 0.0};
        for (int t = T.ce0[c] + threadIdx.x; t < T.ce1[c]; t += blockDim.x) {
            const int k = T.te_k[t], q0 = T.te_c0[t], nq = T.te_cn[t];
            const double on = T.te_K[2 * t] * P.n[k] - T.te_G[2 * t];
            const double op = T.te_K[2 * t + 1] * P.p[k] - T.te_G[2 * t + 1];
            double tn = 0.0, tp = 0.0, sm = 0.0;
            for (int q = q0 + 1; q < q0 + nq; q++) {
                const int kq = T.tc_k[q];
                const double a = T.tc_K[2 * q] * P.n[kq], b = T.tc_K[2 * q + 1] * P.p[kq];
                tn += T.tc_G[2 * q] - a;
                tp += T.tc_G[2 * q + 1] - b;
                sm += fabs(T.tc_G[2 * q]) + a + fabs(T.tc_G[2 * q + 1]) + b;
            }
            const double Ie = Q * (on - tn), Ih = -Q * (op - tp);
            v[0] += Ie + Ih;
            v[1] += Q * (T.te_K[2 * t] * P.n[k] + T.te_G[2 * t] + T.te_K[2 * t + 1] * P.p[k] + T.te_G[2 * t + 1] + sm);
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
            for (int q = 0; q < TE_CUR_TPB / 32; q++) s += sh[threadIdx.x][q];
            P.res[(threadIdx.x == 0 ? R_I : (threadIdx.x == 1 ? R_S : R_IN)) + c] += s;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ host drivers
static int blocks(int n, int tpb) { return n > 0 ? (n + tpb - 1) / tpb : 1; }

// once per Gummel iteration, after the mobility update (te_update, semiconductor_3d.c:3534-3542)
void te_update(Inst &d) {
    if (!d.g.te_on) return;
    Ctx c = make_ctx(d);
    const TeD &T = d.g.te;
    SS_LAUNCH(PF_METAL, T.n_tc, k_te_img, blocks(T.n_te, 128), 128, c.st, c.dP, T);
    SS_LAUNCH(PF_METAL, T.n_tc, k_te_apply, blocks(T.n_touch, 128), 128, c.st, c.dP, T);
    SS_LAUNCH(PF_METAL, T.n_tc, k_te_one, blocks(T.n_te, 64), 64, c.st, c.dP, T);
}
// after the face-flux terminal currents
void te_currents(Inst &d) {
    if (!d.g.te_on) return;
    Ctx c = make_ctx(d);
    SS_LAUNCH(PF_METAL, d.g.te.n_tc, k_te_currents, 1, TE_CUR_TPB, c.st, c.dP, d.g.te);
}

}  // namespace ss
