// Host-side material model of the solver library.
#pragma once

namespace ss {

// Parameters of one material at temperature T (SI units).  The field set covers the
// physics of the solve path (Poisson, Scharfetter-Gummel continuity with SRH + Auger +
// radiative recombination, low-field and velocity-saturated mobility, band-gap
// narrowing) plus flags naming the reference models this library does not implement.
struct Material {
    int id = 0, insulator = 0;
    double T = 300, VT = 0, Eg = 0, chi = 0, eps_r = 1, Nc = 0, Nv = 0, ni = 0;
    // low-field mobility: Arora / Caughey-Thomas form or Masetti (mas_on)
    double mu_n_max = 0, mu_p_max = 0, mu_n_min = 0, mu_p_min = 0;
    double Nref_n = 1, Nref_p = 1, alpha_n = 1, alpha_p = 1;
    double mt_min = -0.57, mt_max_n = -2.33, mt_max_p = -2.23, mt_Nref = 2.4, mt_alpha = -0.146;
    int mas_on = 0;
    double mas_min1[2] = {0, 0}, mas_min2[2] = {0, 0}, mas_mu1[2] = {0, 0}, mas_Pc[2] = {0, 0};
    double mas_Cr[2] = {1, 1}, mas_Cs[2] = {1, 1}, mas_a[2] = {1, 1}, mas_b[2] = {1, 1};
    double vsat_n = 0, vsat_p = 0, beta_n = 1, beta_p = 1;
    double tau_n0 = 0, tau_p0 = 0, Cn = 0, Cp = 0, Brad = 0, tau_Nref = 0;
    double bgn_E = 0, bgn_N = 1, bgn_C = 0;
    double ani_n = 0, ani_p = 0;
    // incomplete ionisation (models bit 9): donors on up to two lattice sites with weights
    // ion_w, level depth dE = ion_Ed - ion_ad N^(1/3) (eV, eV m; clamped at 0) below Ec and
    // degeneracy ion_gd; acceptors one level ion_Ea - ion_aa N^(1/3) above Ev, degeneracy ion_ga
    int ion_on = 0;
    double ion_w[2] = {0, 0}, ion_Ed[2] = {0, 0}, ion_ad[2] = {0, 0}, ion_gd = 1, ion_Ea = 0, ion_aa = 0, ion_ga = 1;
    // MLDA quantum confinement (models bit 3): confinement masses (units of m0) of two
    // electron / hole populations with the weight of the first
    double mq_e1 = 0, mq_e2 = 0, wq_e1 = 1, mq_h1 = 0, mq_h2 = 0, wq_h1 = 1;
    // gate tunnelling (models bit 5): supply (density-of-states) masses of the carriers
    double ms_e = 0, ms_h = 0;
    // metal contacts (models bits 6, 7): Richardson constants A** (A m^-2 K^-2) and the
    // tunnelling effective masses (units of m0) of electrons and holes
    double rich_n = 0, rich_p = 0, mtun_e = 0, mtun_h = 0;
    // impact ionisation (models bit 8), Chynoweth law per carrier c (0 n, 1 p):
    // alpha(F) = g a exp(-(g b / F)^m) with (a, b) below / above the field E0, temperature
    // factor g = tanh(hw / 2kT0) / tanh(hw / 2kT) from the optical-phonon energy hw
    int ii_on = 0;
    double ii_a[2][2] = {{0, 0}, {0, 0}}, ii_b[2][2] = {{0, 0}, {0, 0}}, ii_E0[2] = {0, 0}, ii_m[2] = {1, 1};
    double ii_hw = 0, ii_g = 1;
    // Lombardi surface mobility (models bit 4): lb_on bit 0 electrons, bit 1 holes;
    // 1/mu = 1/mu_b + D (1/mu_ac + 1/mu_sr), mu_ac = B/F + C N^L / (F^(1/3) T/300),
    // mu_sr = D/F^2 (or 1/(F^2/D + F^3/E) with the roughness term E), cm units [0] n, [1] p
    int lb_on = 0;
    double lbB[2] = {0, 0}, lbC[2] = {0, 0}, lbL[2] = {0, 0}, lbD[2] = {0, 0}, lbE[2] = {0, 0};
    // Coulomb scattering of electrons on interface charge (4H-SiC, in the Lombardi sum):
    // mu1 (cm^2/Vs), nu, N0 (cm^-2), e1, e2, E0 (V/cm), gamma
    int lbc_on = 0;
    double lbc_mu1 = 0, lbc_nu = 0, lbc_N0 = 1, lbc_e1 = 0, lbc_e2 = 0, lbc_E0 = 1, lbc_gam = 1;
    double lnc = 0, lnv = 0;      // effective ln Nc / ln Nv in the common gauge (mat_prepare)
};

void material_init(Material &m, int id, double T);
double mobility_low(const Material &m, double Ntot, int hole);
double bgn_half(const Material &m, double N);

}  // namespace ss
