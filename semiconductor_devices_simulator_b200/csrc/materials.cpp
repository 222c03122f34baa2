// Material tables of the 14 reference materials.  The numbers must equal the
// reference's (semiconductor_3d.c:423-627) for results to agree; the code that holds
// them is this library's own: one descriptor per material, applied by a common routine.
#include "materials.h"

#include <cmath>
#include <cstdio>
#include <cstring>

#include "semisim.h"

namespace ss {

namespace {

// Bandgap Varshni form Eg(T) = E0 - a T^2 / (T + b)
double varshni(double E0, double a, double b, double T) { return E0 - a * T * T / (T + b); }

struct Lowfield {   // Arora / Caughey-Thomas parameters (mobilities in m^2/Vs, N in m^-3)
    double mun_max, mup_max, mun_min, mup_min, Nref_n, Nref_p, alpha_n, alpha_p;
    double mt_min, mt_max_n, mt_max_p, mt_Nref, mt_alpha;
};
struct Recomb { double tau_n0, tau_p0, Cn, Cp, Brad; };
struct Sat { double vsat_n, vsat_p, beta_n, beta_p; };

void set_lowfield(Material &m, const Lowfield &l) {
    m.mu_n_max = l.mun_max; m.mu_p_max = l.mup_max; m.mu_n_min = l.mun_min; m.mu_p_min = l.mup_min;
    m.Nref_n = l.Nref_n; m.Nref_p = l.Nref_p; m.alpha_n = l.alpha_n; m.alpha_p = l.alpha_p;
    m.mt_min = l.mt_min; m.mt_max_n = l.mt_max_n; m.mt_max_p = l.mt_max_p;
    m.mt_Nref = l.mt_Nref; m.mt_alpha = l.mt_alpha;
}
void set_recomb(Material &m, const Recomb &r) {
    m.tau_n0 = r.tau_n0; m.tau_p0 = r.tau_p0; m.Cn = r.Cn; m.Cp = r.Cp; m.Brad = r.Brad;
}
void set_sat(Material &m, const Sat &s) {
    m.vsat_n = s.vsat_n; m.vsat_p = s.vsat_p; m.beta_n = s.beta_n; m.beta_p = s.beta_p;
}

// impact-ionisation coefficients: electrons (a, b) below / above E0, holes likewise
struct Ii { double an0, bn0, an1, bn1, E0n, mn, ap0, bp0, ap1, bp1, E0p, mp, hw; };
void set_ii(Material &m, const Ii &v) {
    m.ii_on = 1;
    m.ii_a[0][0] = v.an0; m.ii_b[0][0] = v.bn0; m.ii_a[0][1] = v.an1; m.ii_b[0][1] = v.bn1; m.ii_E0[0] = v.E0n; m.ii_m[0] = v.mn;
    m.ii_a[1][0] = v.ap0; m.ii_b[1][0] = v.bp0; m.ii_a[1][1] = v.ap1; m.ii_b[1][1] = v.bp1; m.ii_E0[1] = v.E0p; m.ii_m[1] = v.mp;
    m.ii_hw = v.hw;
}

// Semiconductor band data: Eg(T) Varshni, affinity, permittivity, Nc/Nv at 300 K with
// power-law temperature exponents.
struct Band { double E0, a, b, chi, eps_r, Nc300, Nc_exp, Nv300, Nv_exp; };
void set_band(Material &m, const Band &bd) {
    const double tr = m.T / 300.0;
    m.Eg = varshni(bd.E0, bd.a, bd.b, m.T);
    m.chi = bd.chi; m.eps_r = bd.eps_r;
    m.Nc = bd.Nc300 * std::pow(tr, bd.Nc_exp);
    m.Nv = bd.Nv300 * std::pow(tr, bd.Nv_exp);
}

}  // namespace

void material_init(Material &m, int id, double T) {
    m = Material();
    m.id = id; m.T = T; m.VT = KB * T / Q;
    const double tr = T / 300.0;
    switch (id) {
    case 0: {   // Si: Masetti low-field mobility, Canali saturation laws, Klaassen BGN
        set_band(m, {1.170, 4.73e-4, 636., 4.05, 11.7, 2.86e25, 1.58, 3.10e25, 1.85});
        m.mas_on = 1; m.mt_max_n = -2.5; m.mt_max_p = -2.2;
        m.mu_n_max = 0.1417; m.mu_p_max = 0.04705; m.mu_n_min = 0.00522; m.mu_p_min = 0.00449;
        const double mm1[2] = {0.00522, 0.00449}, mm2[2] = {0.00522, 0.0}, mu1[2] = {0.00434, 0.00290};
        const double Pc[2] = {0.0, 9.23e22}, Cr[2] = {9.68e22, 2.23e23}, Cs[2] = {3.43e26, 6.10e26};
        const double ma[2] = {0.680, 0.719}, mb[2] = {2.0, 2.0};
        for (int c = 0; c < 2; c++) {
            m.mas_min1[c] = mm1[c]; m.mas_min2[c] = mm2[c]; m.mas_mu1[c] = mu1[c]; m.mas_Pc[c] = Pc[c];
            m.mas_Cr[c] = Cr[c]; m.mas_Cs[c] = Cs[c]; m.mas_a[c] = ma[c]; m.mas_b[c] = mb[c];
        }
        m.Nref_n = 9.68e22; m.Nref_p = 2.23e23; m.alpha_n = 0.680; m.alpha_p = 0.719;
        set_sat(m, {1.07e5 * std::pow(tr, -0.87), 8.37e4 * std::pow(tr, -0.52),
                    1.109 * std::pow(tr, 0.66), 1.213 * std::pow(tr, 0.17)});
        set_recomb(m, {1e-5, 1e-5, 2.8e-43, 9.9e-44, 4.73e-21});
        m.tau_Nref = 1e22;
        m.bgn_E = 6.92e-3; m.bgn_N = 1.3e23; m.bgn_C = 0.5;
        // MLDA: the 2 Delta-2 valleys (m_l 0.916, 1/3) and the 4 Delta-4 valleys (0.19);
        // heavy (0.29, 0.84) and light (0.20) holes (semiconductor_3d.c:457)
        m.mq_e1 = 0.916; m.mq_e2 = 0.19; m.wq_e1 = 1. / 3.; m.mq_h1 = 0.29; m.mq_h2 = 0.20; m.wq_h1 = 0.84;
        m.ms_e = 0.50; m.ms_h = 0.50;
        // Lombardi as parameterised in Sentaurus (semiconductor_3d.c:462-465)
        m.lb_on = 3;
        m.lbB[0] = 4.75e7; m.lbC[0] = 580.; m.lbL[0] = 0.125; m.lbD[0] = 5.82e14;
        m.lbB[1] = 9.925e6; m.lbC[1] = 2947.; m.lbL[1] = 0.0317; m.lbD[1] = 2.0546e14;
        // van Overstraeten - de Man (semiconductor_3d.c:466-472)
        set_ii(m, {7.03e7, 1.231e8, 7.03e7, 1.231e8, 4e7, 1., 1.582e8, 2.036e8, 6.71e7, 1.693e8, 4e7, 1., 0.063});
        break;
    }
    case 1:     // Ge
        set_band(m, {0.742, 4.77e-4, 235., 4.00, 16.2, 1.04e25, 1.5, 6.0e24, 1.5});
        set_lowfield(m, {0.39, 0.19, 0.040, 0.020, 1.30e23, 1.00e23, 0.56, 0.43, 0., -1.66, -2.33, 0., 0.});
        set_sat(m, {6e4, 5.4e4, 1., 1.});
        set_recomb(m, {1e-3, 1e-3, 1e-42, 1e-42, 6.4e-20});
        break;
    case 2:     // GaAs
        set_band(m, {1.519, 5.405e-4, 204., 4.07, 12.9, 4.37e23, 1.5, 8.68e24, 1.5});
        set_lowfield(m, {0.94, 0.040, 0.050, 0.0020, 6.0e22, 2.75e23, 0.394, 0.394, 0., -2.1, -2.1, 3.0, 0.});
        set_sat(m, {7.7e4, 7.7e4, 1., 1.});
        set_recomb(m, {1e-9, 1e-9, 1e-43, 1e-43, 1.5e-16});
        set_ii(m, {2.99e7, 6.848e7, 2.99e7, 6.848e7, 1e30, 1.6, 2.215e7, 6.57e7, 2.215e7, 6.57e7, 1e30, 1.75, 0.});   // :498-500
        break;
    case 3:     // InP
        set_band(m, {1.4236, 3.63e-4, 162., 4.38, 12.5, 5.7e23, 1.5, 1.1e25, 1.5});
        set_lowfield(m, {0.52, 0.015, 0.040, 0.0010, 3.00e23, 4.90e23, 0.47, 0.40, 0., -2.0, -2.0, 3.25, 0.});
        set_sat(m, {1e5, 5e4, 1., 1.});
        set_recomb(m, {1e-8, 1e-8, 1e-43, 1e-43, 8.5e-17});
        break;
    case 4:     // 4H-SiC
        set_band(m, {3.265, 6.5e-4, 1300., 3.7, 9.7, 1.73e25, 1.5, 2.64e25, 1.5});
        set_lowfield(m, {0.095, 0.0124, 0.0040, 0.00159, 1.94e23, 1.76e25, 0.61, 0.34, -0.5, -2.40, -2.15, 0., 0.});
        set_sat(m, {2.2e5, 1.6e5, 1.2, 1.});
        set_recomb(m, {1e-6, 1e-7, 5e-44, 2e-44, 1.5e-18});
        m.lb_on = 1; m.lbc_on = 1;                  // electrons, with Coulomb scattering (semiconductor_3d.c:545-548)
        m.lbc_mu1 = 40.; m.lbc_nu = 1.5; m.lbc_N0 = 1e11; m.lbc_e1 = 1.; m.lbc_e2 = 0.5; m.lbc_E0 = 2e5; m.lbc_gam = 2.;
        m.lbB[0] = 1e6; m.lbC[0] = 1.077e4; m.lbL[0] = 0.0284; m.lbD[0] = 1.7e13; m.lbE[0] = 1.7e29;
        set_ii(m, {1.76e10, 3.30e9, 1.76e10, 3.30e9, 1e30, 1., 3.41e10, 2.50e9, 3.41e10, 2.50e9, 1e30, 1., 0.});   // :528-530
        // nitrogen on the hexagonal and cubic sites (1:1), aluminium acceptors
        // (semiconductor_3d.c:553-555)
        m.ion_on = 1; m.ion_w[0] = m.ion_w[1] = 0.5;
        m.ion_Ed[0] = 0.0709; m.ion_ad[0] = 3.38e-10; m.ion_Ed[1] = 0.1237; m.ion_ad[1] = 4.65e-10; m.ion_gd = 2.;
        m.ion_Ea = 0.225; m.ion_aa = 3.2e-10; m.ion_ga = 4.;
        m.ani_n = 1. / 0.83; m.ani_p = 1. / 1.15;
        break;
    case 5:     // GaN
        set_band(m, {3.507, 9.09e-4, 830., 4.1, 8.9, 2.3e24, 1.5, 4.6e25, 1.5});
        set_lowfield(m, {0.120, 0.0030, 0.0055, 0.00030, 1.00e23, 3.00e23, 1.0, 2.0, -1.02, -3.84, -3.84, 0., 0.});
        set_sat(m, {2.5e5, 2e5, 1., 1.});
        set_recomb(m, {1e-8, 1e-8, 1e-43, 1e-43, 1.1e-16});
        set_ii(m, {2.11e11, 3.689e9, 2.11e11, 3.689e9, 1e30, 1., 4.39e8, 1.8e9, 4.39e8, 1.8e9, 1e30, 1., 0.});   // :572-574
        break;
    case 6:     // Al0.3Ga0.7As
        set_band(m, {1.882, 5.58e-4, 295., 3.827, 12.24, 7.2e23, 1.5, 1.05e25, 1.5});
        set_lowfield(m, {0.35, 0.025, 0.020, 0.0015, 6.00e22, 1.00e23, 0.394, 0.394, 0., -2.1, -2.1, 3.0, 0.});
        set_sat(m, {6e4, 5e4, 1., 1.});
        set_recomb(m, {1e-9, 1e-9, 1e-43, 1e-43, 5e-17});
        break;
    case 7:     // Al0.25Ga0.75N
        set_band(m, {3.990, 9.09e-4, 830., 3.76, 8.8, 3.2e24, 1.5, 4.6e25, 1.5});
        set_lowfield(m, {0.030, 0.0010, 0.0030, 0.00020, 1.00e23, 3.00e23, 1.0, 2.0, -1.02, -3.84, -3.84, 0., 0.});
        set_sat(m, {1.5e5, 1e5, 1., 1.});
        set_recomb(m, {1e-9, 1e-9, 1e-43, 1e-43, 1e-16});
        break;
    // insulators: gap, affinity, permittivity
    case 8:  m.insulator = 1; m.Eg = 9.0;  m.chi = 0.95; m.eps_r = 3.9;  break;   // SiO2
    case 9:  m.insulator = 1; m.Eg = 6.8;  m.chi = 1.35; m.eps_r = 9.0;  break;   // Al2O3
    case 10: m.insulator = 1; m.Eg = 5.8;  m.chi = 2.55; m.eps_r = 22.0; break;   // HfO2
    case 11: m.insulator = 1; m.Eg = 5.1;  m.chi = 2.05; m.eps_r = 7.5;  break;   // Si3N4
    case 12: m.insulator = 1; m.Eg = 10.;  m.chi = 0.;   m.eps_r = 1.0;  break;   // void
    case 13: m.insulator = 1; m.Eg = 10.;  m.chi = 0.;   m.eps_r = 1.0e3; break;  // metal inclusion
    default:
        std::fprintf(stderr, "semisim-b200: WARNING unknown material id %d, using Si\n", id);
        material_init(m, 0, T);
        return;
    }
    // Richardson constants and tunnelling masses (semiconductor_3d.c:461, 483, 494, 512, 524,
    // 569, 585, 597, 601-614)
    static const double te_tab[14][4] = {
        {1.12e6, 3.2e5, 0.26, 0.39},  {1.43e6, 4.1e5, 0.12, 0.28}, {8.16e4, 7.44e5, 0.067, 0.45},
        {9.6e4, 7.2e5, 0.08, 0.60},   {1.46e6, 9.6e5, 0.33, 0.80}, {2.64e5, 9.6e5, 0.22, 0.80},
        {1.08e5, 6.6e5, 0.092, 0.50}, {3.0e5, 9.6e5, 0.25, 1.0},   {0., 0., 0.42, 0.33},
        {0., 0., 0.35, 0.35},         {0., 0., 0.18, 0.20},        {0., 0., 0.50, 0.50},
        {0., 0., 1., 1.},             {0., 0., 1., 1.}};
    m.rich_n = te_tab[id][0]; m.rich_p = te_tab[id][1]; m.mtun_e = te_tab[id][2]; m.mtun_h = te_tab[id][3];
    if (!m.insulator && !(m.mq_e1 > 0.) && id < 8) {    // generic single confinement masses (:619-624)
        static const double me[8] = {0.916, 0.082, 0.067, 0.08, 0.37, 0.20, 0.09, 0.23};
        static const double mh[8] = {0.29, 0.28, 0.50, 0.60, 1.00, 1.00, 0.55, 1.00};
        m.mq_e1 = m.mq_e2 = me[id]; m.wq_e1 = 1.; m.mq_h1 = m.mq_h2 = mh[id]; m.wq_h1 = 1.;
        m.ms_e = me[id] < 0.5 ? me[id] : 0.5; m.ms_h = 0.5;
    }
    if (m.insulator) {
        // insulators carry no mobility / recombination data; keep the defaults neutral
        m.mt_min = m.mt_max_n = m.mt_max_p = m.mt_Nref = m.mt_alpha = 0.;
    }
    m.ni = m.insulator ? 0. : std::sqrt(m.Nc * m.Nv) * std::exp(-m.Eg / (2. * m.VT));
    m.ii_g = m.ii_hw > 0. ? std::tanh(m.ii_hw / (2. * KB * 300. / Q)) / std::tanh(m.ii_hw / (2. * m.VT)) : 1.;
}

// Low-field mobility: Masetti (mas_on) or Arora / Caughey-Thomas (semiconductor_3d.c:646-662)
double mobility_low(const Material &m, double Ntot, int hole) {
    if (Ntot < 1.) Ntot = 1.;
    const double tr = m.T / 300.;
    if (m.mas_on) {
        const int c = hole ? 1 : 0;
        const double muL = (hole ? m.mu_p_max : m.mu_n_max) * std::pow(tr, hole ? m.mt_max_p : m.mt_max_n);
        const double mu = m.mas_min1[c] * std::exp(-m.mas_Pc[c] / Ntot) +
                          (muL - m.mas_min2[c]) / (1. + std::pow(Ntot / m.mas_Cr[c], m.mas_a[c])) -
                          m.mas_mu1[c] / (1. + std::pow(m.mas_Cs[c] / Ntot, m.mas_b[c]));
        return mu > 1e-6 ? mu : 1e-6;
    }
    const double mumin = (hole ? m.mu_p_min : m.mu_n_min) * std::pow(tr, m.mt_min);
    double mumax = (hole ? m.mu_p_max : m.mu_n_max) * std::pow(tr, hole ? m.mt_max_p : m.mt_max_n);
    const double Nref = (hole ? m.Nref_p : m.Nref_n) * std::pow(tr, m.mt_Nref);
    const double alpha = (hole ? m.alpha_p : m.alpha_n) * std::pow(tr, m.mt_alpha);
    if (mumax < mumin) mumax = mumin;
    return mumin + (mumax - mumin) / (1. + std::pow(Ntot / Nref, alpha));
}

// Half the band-gap narrowing in units of VT, Klaassen form (semiconductor_3d.c:839-843)
double bgn_half(const Material &m, double N) {
    if (!(m.bgn_E > 0.) || N < 1.) return 0.;
    const double L = std::log(N / m.bgn_N);
    return 0.5 * m.bgn_E * (L + std::sqrt(L * L + m.bgn_C)) / m.VT;
}

}  // namespace ss
