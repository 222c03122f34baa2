// Device helpers shared by the kernel files: block reductions with a deterministic
// last-block finish, grid-stride loops, and the per-node physics of the solve path.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "semisim.h"

namespace ss {

#define SS_GRID_LOOP(k, N) for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < (N); k += gridDim.x * blockDim.x)

// Programmatic dependent launch: let the next kernel of the stream start its launch now,
// then wait until the kernels this one depends on have completed and their writes are
// visible.  Every kernel launched with SS_LAUNCH_PDL calls this before touching memory;
// without that launch attribute both instructions are no-ops.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
// The two halves, for kernels that first read set-up data (instance and level records,
// array pointers, sizes: written only by host copies, never by a kernel) and only then
// wait: those loads overlap the previous kernel's tail.  Every path calls pdl_wait()
// before it reads kernel-written memory and before it returns.
__device__ __forceinline__ void pdl_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
    for (int q = 0; q < NV; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Sum NV values over the block; the result is valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
    __shared__ double sh[NV][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    warp_sum<NV>(v);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[q][wid] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) v[q] = lane < nw ? sh[q][lane] : 0.0;
        warp_sum<NV>(v);
    }
}

// Grid-wide sum of NV values with a deterministic finish: every block writes its
// partial record, the last block to arrive (atomic ticket) adds the records in block
// order.  Returns true in thread 0 of the last block, with `v` holding the totals.
// `part` holds RED_MAX_BLOCKS records of RED_NV doubles; gridDim.x <= RED_MAX_BLOCKS.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double *part, unsigned *ticket) {
    __shared__ bool is_last;
    block_sum<NV>(v);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) part[blockIdx.x * RED_NV + q] = v[q];
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; q++) v[q] += __ldcg(part + b * RED_NV + q);
    block_sum<NV>(v);
    if (threadIdx.x == 0) *ticket = 0u;
    return threadIdx.x == 0;
}

// Grid-wide max of one value (same protocol; values >= 0 or -inf)
__device__ __forceinline__ bool grid_max(double &v, double *part, unsigned *ticket) {
    __shared__ double sh[32];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? sh[lane] : -INFINITY;
        v = warp_max(v);
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x * RED_NV] = v;
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    v = -INFINITY;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v = fmax(v, __ldcg(part + b * RED_NV));
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? sh[lane] : -INFINITY;
        v = warp_max(v);
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return threadIdx.x == 0;
}

// ---------------------------------------------------------------- node physics
__device__ __forceinline__ double clampe(double e) { return e < LN_MIN ? LN_MIN : (e > LN_MAX ? LN_MAX : e); }

// Bernoulli function x/(e^x - 1): quadratic series below 1e-6, limits beyond +-700
// (semiconductor_3d.c:670-675)
__device__ __forceinline__ double bern(double x) {
    if (fabs(x) < 1e-6) return 1.0 - x / 2.0 + x * x / 12.0;
    if (x > 700.0) return 0.0;
    if (x < -700.0) return -x;
    return x / expm1(x);
}

struct Node {
    int i, j, l;
};
__device__ __forceinline__ Node unidx(int k, int Nx, int Ny) {
    Node r;
    const int NxNy = Nx * Ny;
    r.l = k / NxNy;
    const int rem = k - r.l * NxNy;
    r.j = rem / Nx;
    r.i = rem - r.j * Nx;
    return r;
}

// neighbour in direction dir (0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+) with spacing h and
// face area ar (semiconductor_3d.c:709-719); false outside the domain
__device__ __forceinline__ bool nbr(const DevP &P, const Node &a, int k, int dir, int &kb, double &h, double &ar) {
    switch (dir) {
    case 0: if (a.i == 0) return false; kb = k - 1; h = P.xs[a.i] - P.xs[a.i - 1]; ar = P.Ly[a.j] * P.Lz[a.l]; return true;
    case 1: if (a.i == P.Nx - 1) return false; kb = k + 1; h = P.xs[a.i + 1] - P.xs[a.i]; ar = P.Ly[a.j] * P.Lz[a.l]; return true;
    case 2: if (a.j == 0) return false; kb = k - P.Nx; h = P.ys[a.j] - P.ys[a.j - 1]; ar = P.Lx[a.i] * P.Lz[a.l]; return true;
    case 3: if (a.j == P.Ny - 1) return false; kb = k + P.Nx; h = P.ys[a.j + 1] - P.ys[a.j]; ar = P.Lx[a.i] * P.Lz[a.l]; return true;
    case 4: if (a.l == 0) return false; kb = k - P.Nx * P.Ny; h = P.zs[a.l] - P.zs[a.l - 1]; ar = P.Lx[a.i] * P.Ly[a.j]; return true;
    default: if (a.l == P.Nz - 1) return false; kb = k + P.Nx * P.Ny; h = P.zs[a.l + 1] - P.zs[a.l]; ar = P.Lx[a.i] * P.Ly[a.j]; return true;
    }
}

__device__ __forceinline__ double bgn_of(const DevP &P, int k) { return P.bgn ? P.bgn[k] : 0.0; }
// image-force band lowering near metal contacts (0 elsewhere; semiconductor_3d.c:736-738)
__device__ __forceinline__ double qcn_of(const DevP &P, int k) { return P.qcn ? P.qcn[k] : 0.0; }
__device__ __forceinline__ double qcp_of(const DevP &P, int k) { return P.qcp ? P.qcp[k] : 0.0; }
__device__ __forceinline__ double lncK(const DevP &P, const MatD &m, int k) { return m.lnc + bgn_of(P, k) + qcn_of(P, k); }
__device__ __forceinline__ double lnvK(const DevP &P, const MatD &m, int k) { return m.lnv + bgn_of(P, k) + qcp_of(P, k); }
__device__ __forceinline__ double niK(const DevP &P, const MatD &m, int k) {
    return m.ni * exp(bgn_of(P, k) + 0.5 * (qcn_of(P, k) + qcp_of(P, k)));
}
__device__ __forceinline__ double nK(const DevP &P, const MatD &m, int k, double psi, double qn) {
    return exp(clampe(lncK(P, m, k) + (psi - qn) / m.VT));
}
__device__ __forceinline__ double pK(const DevP &P, const MatD &m, int k, double psi, double qp) {
    return exp(clampe(lnvK(P, m, k) + (qp - psi) / m.VT));
}
// Incomplete ionisation (semiconductor_3d.c:749-786): P.ion holds per node N_c/g_D e^(-dE/kT)
// of the two donor sites, N_v/g_A e^(-dE_A/kT) (m^-3; 0 = fully ionised) and the node's
// majority density when neutral.  ion_eval gives the ionised donor and acceptor densities at
// carrier densities n, p and their psi-derivatives at fixed quasi-Fermi potentials.
__device__ __forceinline__ bool ion_node(const DevP &P, int k) {
    if (!P.ion) return false;
    const double *x = P.ion + (size_t)ION_W * k;
    return (x[0] > 0.0 && P.Nd[k] > 0.0) || (x[2] > 0.0 && P.Na[k] > 0.0);
}
__device__ __forceinline__ void ion_eval(const DevP &P, const MatD &m, int k, double n, double p, double &Np,
                                         double &dNp, double &Nm, double &dNm) {
    const double Nd = P.Nd[k], Na = P.Na[k];
    Np = Nd; Nm = Na; dNp = dNm = 0.0;
    if (!P.ion) return;
    const double *x = P.ion + (size_t)ION_W * k;
    const double VT = m.VT;
    if (Nd > 0.0 && x[0] > 0.0) {
        const double e = bgn_of(P, k) + qcn_of(P, k);
        const double ne = e != 0.0 ? n * exp(-e) : n;
        const double a = ne / x[0];
        double f = m.ion_w[0] / (1.0 + a), df = -m.ion_w[0] * a / ((1.0 + a) * (1.0 + a));
        if (m.ion_w[1] > 0.0 && x[1] > 0.0) {
            const double b = ne / x[1];
            f += m.ion_w[1] / (1.0 + b);
            df -= m.ion_w[1] * b / ((1.0 + b) * (1.0 + b));
        }
        Np = Nd * f; dNp = Nd * df / VT;
    }
    if (Na > 0.0 && x[2] > 0.0) {
        const double e = bgn_of(P, k) + qcp_of(P, k);
        const double pe = e != 0.0 ? p * exp(-e) : p;
        const double c = pe / x[2];
        Nm = Na / (1.0 + c); dNm = Na * c / ((1.0 + c) * (1.0 + c) * VT);
    }
}
// the doping scale of the quasi-neutral tests: |Nd - Na|, or the neutral majority density
__device__ __forceinline__ double dnet_ion(const DevP &P, int k) {
    if (!ion_node(P, k)) return fabs(P.Nd[k] - P.Na[k]);
    return P.ion[(size_t)ION_W * k + 3];
}

// SRH lifetime doping factor (semiconductor_3d.c:787-791)
__device__ __forceinline__ double tauf(const DevP &P, const MatD &m, int k) {
    if (!(P.models & 2) || !(m.tau_Nref > 0.)) return 1.0;
    return 1.0 / (1.0 + (P.Nd[k] + P.Na[k]) / m.tau_Nref);
}
// SRH + Auger + radiative recombination with derivatives (semiconductor_3d.c:686-697)
__device__ __forceinline__ void recomb(const MatD &m, double ni, double tf, double n, double p, double &R,
                                       double &dRn, double &dRp) {
    const double ni2 = ni * ni, np_ = n * p - ni2;
    const double den = tf * (m.tau_p0 * (n + ni) + m.tau_n0 * (p + ni)) + 1e-300;
    const double Rs = np_ / den;
    const double dsn = (p * den - np_ * tf * m.tau_p0) / (den * den);
    const double dsp = (n * den - np_ * tf * m.tau_n0) / (den * den);
    const double Au = m.Cn * n + m.Cp * p;
    R = Rs + Au * np_ + m.Brad * np_;
    dRn = dsn + m.Cn * np_ + Au * p + m.Brad * p;
    dRp = dsp + m.Cp * np_ + Au * n + m.Brad * n;
}

// Shockley-Read-Hall statistics of the trap entries of node k at densities n, p
// (semiconductor_3d.c:368-400): recombination R with dR/dn, dR/dp, and the trapped charge
// rho (elementary charges per m^3) with d rho / d psi at fixed quasi-Fermi levels; the
// occupancy f = (cn n + cp p1) / (cn (n + n1) + cp (p + p1)) with n1, p1 at the local band
// edges, so the equilibrium is exact
__device__ __forceinline__ bool trap_node(const DevP &P, int k) { return P.tr_rp && P.tr_rp[k] < P.tr_rp[k + 1]; }
__device__ __forceinline__ void trap_levels(const TrapD &s, const MatD &m, double ni, double &n1, double &p1) {
    const double VT = m.VT;
    if (s.ref == 0) { n1 = m.Nc * exp(-s.E / VT); p1 = ni * ni / n1; }
    else if (s.ref == 1) { p1 = m.Nv * exp(-s.E / VT); n1 = ni * ni / p1; }
    else { n1 = ni * exp(s.E / VT); p1 = ni * exp(-s.E / VT); }
}
__device__ __forceinline__ void trap_eval(const DevP &P, const MatD &m, int k, double n, double p, double &R,
                                          double &dRn, double &dRp, double &rho, double &drho) {
    R = dRn = dRp = rho = drho = 0.0;
    if (!trap_node(P, k)) return;
    const double VT = m.VT, ni = niK(P, m, k), ni2 = ni * ni;
    for (int q = P.tr_rp[k]; q < P.tr_rp[k + 1]; q++) {
        const TrapD &s = P.tsp[P.tr_s[q]];
        double n1, p1;
        trap_levels(s, m, ni, n1, p1);
        const double cn = P.tr_cn[q], cp = P.tr_cp[q], Nt = P.tr_N[q];
        const double den = cn * (n + n1) + cp * (p + p1) + 1e-300, np_ = n * p - ni2, A = Nt * cn * cp;
        R += A * np_ / den;
        dRn += A * (p * den - np_ * cn) / (den * den);
        dRp += A * (n * den - np_ * cp) / (den * den);
        if (s.type) {
            const double num = cn * n + cp * p1, f = num / den;
            const double df = (cn * n * den - num * (cn * n - cp * p)) / (VT * den * den);   // df/dpsi >= 0
            rho += s.type < 0 ? -Nt * f : Nt * (1.0 - f);
            drho -= Nt * df;
        }
    }
}
// charged trap states of node k (m^-3, all signs counted): occupied acceptors plus empty
// donors - the scattering centres of the trapped charge (trap_abs, semiconductor_3d.c:402-420)
__device__ __forceinline__ double trap_abs(const DevP &P, const MatD &m, int k, double n, double p) {
    if (!trap_node(P, k)) return 0.0;
    const double ni = niK(P, m, k);
    double sum = 0.0;
    for (int q = P.tr_rp[k]; q < P.tr_rp[k + 1]; q++) {
        const TrapD &s = P.tsp[P.tr_s[q]];
        if (!s.type) continue;
        double n1, p1;
        trap_levels(s, m, ni, n1, p1);
        const double cn = P.tr_cn[q], cp = P.tr_cp[q], Nt = P.tr_N[q];
        const double f = (cn * n + cp * p1) / (cn * (n + n1) + cp * (p + p1) + 1e-300);
        sum += s.type < 0 ? Nt * f : Nt * (1.0 - f);
    }
    return sum;
}
// band-to-band recombination plus the traps of the node (recombKnp, semiconductor_3d.c:823-837)
__device__ __forceinline__ void recombK(const DevP &P, const MatD &m, int k, double n, double p, double &R,
                                        double &dRn, double &dRp) {
    recomb(m, niK(P, m, k), tauf(P, m, k), n, p, R, dRn, dRp);
    if (trap_node(P, k)) {
        double r, a, b, c, e;
        trap_eval(P, m, k, n, p, r, a, b, c, e);
        R += r; dRn += a; dRp += b;
    }
}

// Caughey-Thomas velocity saturation (semiconductor_3d.c:664-668)
__device__ __forceinline__ double mob_hf(double mu0, double E, double vsat, double beta) {
    const double r = mu0 * fabs(E) / vsat;
    if (r < 1e-12) return mu0;
    return mu0 / pow(1.0 + pow(r, beta), 1.0 / beta);
}
// harmonic-mean driving field of an edge (semiconductor_3d.c:2882-2886)
__device__ __forceinline__ double heat_field(double dq, double dps, double h) {
    if (dq * dps <= 0.0) return 0.0;
    const double a = fabs(dq), b = fabs(dps);
    return 2.0 * a * b / ((a + b) * h);
}

// impact ionisation coefficient alpha(F) = g a exp(-(g b / F)^m), (a, b) below / above E0
// (semiconductor_3d.c:4478-4485)
__device__ __forceinline__ double ii_alpha(const MatD &m, double F, int c) {
    if (!(F > 1e5)) return 0.0;                    // below 1 kV/cm: nothing
    const int r = F >= m.ii_E0[c];
    double x = m.ii_g * m.ii_b[c][r] / F;
    if (m.ii_m[c] != 1.0) x = pow(x, m.ii_m[c]);
    if (x > 700.0) return 0.0;
    return m.ii_g * m.ii_a[c][r] * exp(-x);
}

}  // namespace ss
