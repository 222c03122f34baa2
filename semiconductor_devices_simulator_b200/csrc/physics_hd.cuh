// Physics shared by the device kernels and the host-side ABI probes (api3_tun_eval,
// api3_lombardi): WKB through piecewise-linear barriers and the Tsu-Esaki energy integral of
// a gate stack (semiconductor_3d.c:3258-3325), and the Lombardi surface mobility
// (semiconductor_3d.c:2924-2933).
#pragma once
#include <cmath>

#include "semisim.h"

#ifdef __CUDACC__
#define SS_HD __host__ __device__ __forceinline__
#else
#define SS_HD inline
#endif

namespace ss {

constexpr double TUN_HBAR = 1.054571817e-34, TUN_M0 = 9.1093837015e-31, TUN_HPLANCK = 6.62607015e-34;
constexpr double TUN_PI = 3.14159265358979323846;
constexpr int TUN_MAXL = 6;        // layers of a tunnelling path
constexpr int TUN_NE = 64;         // Simpson intervals per energy integral
constexpr double TUN_EMAX = 3.0;   // integration range beyond the band edge (eV)
constexpr double TUN_LMAX = 30e-9; // insulator a path may cross
constexpr double TUN_COL = 5e-9;   // depth of a path's supply column

SS_HD double softplus(double x) { return x > 35.0 ? x + log1p(exp(-x)) : log1p(exp(x)); }

// 2 int kappa dx over a layer of length L whose barrier above the carrier energy runs
// linearly from u0 to u1 (eV), kappa = sqrt(2 m q u) / hbar
SS_HD double wkb_seg(double mt, double L, double u0, double u1) {
    const double a = u0 > 0.0 ? u0 : 0.0, b = u1 > 0.0 ? u1 : 0.0;
    if (a == 0.0 && b == 0.0) return 0.0;
    const double c = 2.0 * sqrt(2.0 * mt * TUN_M0 * Q) / TUN_HBAR, du = u1 - u0;
    double I;
    if (fabs(du) < 1e-9 * (a + b)) I = L * sqrt(0.5 * (a + b));
    else I = L * (2.0 / 3.0) * (b * sqrt(b) - a * sqrt(a)) / du;
    return c * I;
}

// a layer stack between a semiconductor node and a metal: potentials linear in every layer
struct TPath {
    int nl;
    const MatD *m[TUN_MAXL];
    double t[TUN_MAXL], p0[TUN_MAXL], dp[TUN_MAXL];
    double D, psis;                // displacement (C/m^2) and the potential at the interface
};

// transmission exp(-sum WKB) through the insulator layers at energy E (eV)
SS_HD double tun_T(const TPath &P, double E, int hole) {
    double s = 0.0;
    for (int i = 0; i < P.nl; i++) {
        const MatD &m = *P.m[i];
        if (!m.insulator) continue;
        double mt = hole ? m.mtun_h : m.mtun_e;
        if (!(mt > 0.0)) mt = 0.5;
        const double ea = -P.p0[i] - m.chi, eb = -(P.p0[i] + P.dp[i]) - m.chi;   // Ec of the insulator at both ends
        double u0, u1;
        if (hole) { u0 = E - (ea - m.Eg); u1 = E - (eb - m.Eg); }
        else { u0 = ea - E; u1 = eb - E; }
        s += wkb_seg(mt, P.t[i], u0, u1);
        if (s > 745.0) return 0.0;
    }
    return exp(-s);
}

// int T(E) ln(1 + exp(+-(EF - E)/kT)) dE (eV): electrons upwards from E0, holes downwards
SS_HD double tun_int(const TPath &P, double E0, double EF, double kT, int hole) {
    const double sg = hole ? -1.0 : 1.0;
    double top = sg * (EF - E0);
    if (top < 0.0) top = 0.0;
    double span = top + 25.0 * kT;
    if (span > TUN_EMAX) span = TUN_EMAX;
    const double h = span / TUN_NE;
    double s = 0.0;
    for (int q = 0; q <= TUN_NE; q++) {
        const double E = E0 + sg * q * h;
        const double f = tun_T(P, E, hole) * softplus(sg * (EF - E) / kT);
        s += f * (q == 0 || q == TUN_NE ? 1.0 : (q & 1 ? 4.0 : 2.0));
    }
    return s * h / 3.0;
}

// potentials along a stack (semiconductor half cell first, if any) between a node at psik
// and a metal at voltage Vg with work function pm
SS_HD void tun_stack(TPath &P, const MatD *mats, int nl, const int *mi, const double *t, double psik, double Vg,
                     double pm, double Cref) {
    P.nl = nl;
    double R = 0.0;
    for (int i = 0; i < nl; i++) {
        P.m[i] = &mats[mi[i]];
        P.t[i] = t[i];
        R += t[i] / P.m[i]->eps;
    }
    if (!(pm > 0.0)) pm = Cref;
    const double psim = Vg + Cref - pm;
    double ps = psik;
    P.D = R > 0.0 ? (psim - psik) / R : 0.0;
    P.psis = psik;
    for (int i = 0; i < nl; i++) {
        P.p0[i] = ps;
        P.dp[i] = P.D * t[i] / P.m[i]->eps;
        ps += P.dp[i];
        if (i == 0 && !P.m[0]->insulator) P.psis = ps;             // potential at the interface
    }
}

// fluxes (1/m^2 s) for effective band edges Ec', Ev' and Fermi levels (eV): electrons s->g,
// g->s, holes s->g, g->s
SS_HD void tun_flux(const MatD &ms, const TPath &P, double Ecp, double Evp, double EFn, double EFp, double EFm,
                    double *F) {
    const double kT = ms.VT, h3 = TUN_HPLANCK * TUN_HPLANCK * TUN_HPLANCK;
    const double ce = 4.0 * TUN_PI * ms.ms_e * TUN_M0 * Q * Q * kT / h3, ch = 4.0 * TUN_PI * ms.ms_h * TUN_M0 * Q * Q * kT / h3;
    F[0] = ce * tun_int(P, Ecp, EFn, kT, 0);
    F[1] = ce * tun_int(P, Ecp, EFm, kT, 0);
    F[2] = ch * tun_int(P, Evp, EFp, kT, 1);
    F[3] = ch * tun_int(P, Evp, EFm, kT, 1);
}

// Lombardi: 1/mu = 1/mu_b + D (1/mu_ac + 1/mu_sr + invC), cm units inside; invC the 1/mu of
// further surface terms (Coulomb), (cm^2/Vs)^-1
SS_HD double lombardi(const MatD &m, double mub, double Fv, double Nt, double Dw, int hole, double invC) {
    double F = Fv * 1e-2;
    if (F < 1.0) F = 1.0;                          // V/cm
    double N = Nt * 1e-6;
    if (N < 1.0) N = 1.0;                          // cm^-3
    const double Bc = m.lbB[hole], Cc = m.lbC[hole], Lc = m.lbL[hole], Dc = m.lbD[hole], Ec = m.lbE[hole];
    const double muac = Bc / F + Cc * pow(N, Lc) / (cbrt(F) * (m.T / 300.0));
    const double musr = Ec > 0.0 ? 1.0 / (F * F / Dc + F * F * F / Ec) : Dc / (F * F);
    return 1.0 / (1.0 / mub + Dw * 1e4 * (1.0 / muac + 1.0 / musr + invC));
}

// n_trans (cm^-3) of the Coulomb term against the acceptor doping (cm^-3): log-log
// interpolation of four points, clamped (semiconductor_3d.c:2937-2944)
SS_HD double ntrans_sic(double NA) {
    const double a[4] = {1e15, 1e16, 5e16, 5e17}, t[4] = {2.8e16, 8e16, 2.5e17, 1.55e18};
    if (!(NA > a[0])) return t[0];
    if (NA >= a[3]) return t[3];
    int q = 0;
    while (NA > a[q + 1]) q++;
    return t[q] * pow(t[q + 1] / t[q], log(NA / a[q]) / log(a[q + 1] / a[q]));
}
// 1/mu_C (cm^2/Vs)^-1 of electrons at density n (m^-3) in a normal field Fv (V/m) near an
// interface holding NC charges per m^2, acceptor doping NA (m^-3); 0 without interface
// charge or normal field (semiconductor_3d.c:2948-2955)
SS_HD double coul_inv(const MatD &m, double Fv, double n, double NC, double NA) {
    const double F = Fv * 1e-2, r = NC * 1e-4 / m.lbc_N0;
    if (!(r > 0.0) || !(F > 0.0)) return 0.0;
    const double f = 1.0 - exp(-pow(F / m.lbc_E0, m.lbc_gam));
    if (!(f > 0.0)) return 0.0;
    const double s = pow(n * 1e-6 / (ntrans_sic(NA * 1e-6) * pow(r, m.lbc_e1)), m.lbc_nu);
    return pow(r, m.lbc_e2) * f / (m.lbc_mu1 * (m.T / 300.0) * (1.0 + s));
}

}  // namespace ss
