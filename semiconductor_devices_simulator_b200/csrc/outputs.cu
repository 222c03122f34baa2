// Per-point outputs as device reductions over the resident state: the largest field in
// the semiconductor (api3_get_Emax, semiconductor_3d.c:4981-5001), the carrier totals
// (api3_carrier_sums, :5137-5147), the largest insulator field and where it is
// (api3_ins_field_max, :5308-5339) and the quasi-static terminal charges of a charge
// partition (api3_terminal_charges, :5248-5282).  Each reduces in a fixed block order, so
// the results are deterministic; the host reads a few doubles instead of whole node arrays.
#include "device_common.cuh"
#include "prof.h"
#include "solver_ctx.h"

namespace ss {

constexpr int OUT_TPB = 256, OUT_BLOCKS = 256;   // <= 256 blocks: the partial buffers' size

// coupling eps_bar A / h of the box-method edge from node k towards neighbour dir, with its
// spacing h (the reference's harmonic-mean permittivity, semiconductor_3d.c:5174-5191)
__device__ __forceinline__ bool edge(const DevP &P, int k, const Node &a, int dir, int &kb, double &cf, double &h) {
    double ar;
    if (!nbr(P, a, k, dir, kb, h, ar)) return false;
    const double ek = P.mats[fl_mat(P.flags[k])].eps, eb = P.mats[fl_mat(P.flags[kb])].eps;
    cf = (2.0 * ek * eb / (ek + eb)) * ar / h;
    return true;
}

// the same for either mesh: neighbour idx of node k (the six directions of the tensor grid,
// or the ELL slots of a graph in CSR order), with its coupling and spacing
__device__ __forceinline__ int nslots(const DevP &P) { return P.gD ? P.gD : 6; }
__device__ __forceinline__ bool edge_any(const DevP &P, int k, const Node &a, int idx, int &kb, double &cf, double &h) {
    if (!P.gD) return edge(P, k, a, idx, kb, cf, h);
    const size_t e = (size_t)idx * P.N + k;
    kb = P.gcol[e];
    if (kb < 0) return false;
    h = P.gh[e];
    const double ek = P.mats[fl_mat(P.flags[k])].eps, eb = P.mats[fl_mat(P.flags[kb])].eps;
    cf = (2.0 * ek * eb / (ek + eb)) * P.ga[e] / h;
    return true;
}

// Grid-wide arg-max of (v, idx): the largest v, the smallest idx among equal v (what a
// sequential scan in idx order with a strict comparison keeps).  idx < 2^53, so it travels
// exactly through the double partials; NO_IDX marks an empty candidate.  Thread 0 of the
// last block returns true with the result.
constexpr long long NO_IDX = 1LL << 62;
__device__ __forceinline__ bool better(double v, long long i, double w, long long j) {
    return v > w || (v == w && i < j);
}
__device__ bool grid_argmax(double &v, long long &idx, double *part, unsigned *ticket) {
    __shared__ double sv[32];
    __shared__ long long si[32];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    auto warp_red = [&]() {
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_down_sync(0xffffffffu, v, o);
            const long long j = __shfl_down_sync(0xffffffffu, idx, o);
            if (better(w, j, v, idx)) { v = w; idx = j; }
        }
    };
    warp_red();
    __syncthreads();
    if (lane == 0) { sv[wid] = v; si[wid] = idx; }
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? sv[lane] : -1.0;
        idx = lane < nw ? si[lane] : NO_IDX;
        warp_red();
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x * RED_NV] = v;
        part[blockIdx.x * RED_NV + 1] = (double)idx;
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    v = -1.0;
    idx = NO_IDX;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        const double w = __ldcg(part + b * RED_NV);
        const long long j = (long long)__ldcg(part + b * RED_NV + 1);
        if (better(w, j, v, idx)) { v = w; idx = j; }
    }
    warp_red();
    __syncthreads();
    if (lane == 0) { sv[wid] = v; si[wid] = idx; }
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? sv[lane] : -1.0;
        idx = lane < nw ? si[lane] : NO_IDX;
        warp_red();
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return threadIdx.x == 0;
}

// largest |grad psi|^2 over the semiconductor nodes (central differences inside, one-sided
// at the domain edge) -> res[R_OUT]
__global__ void k_out_emax(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    double m = 0.0;
    const int NxNy = P.Nx * P.Ny;
    SS_GRID_LOOP(k, P.N) {
        if (fl_kind(P.flags[k]) != K_SEMI) continue;
        const Node a = unidx(k, P.Nx, P.Ny);
        const int idx[3] = {a.i, a.j, a.l}, nn[3] = {P.Nx, P.Ny, P.Nz}, st[3] = {1, P.Nx, NxNy};
        const double *cs[3] = {P.xs, P.ys, P.zs};
        double g2 = 0.0;
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            const int q = idx[ax];
            const bool lo = q > 0, hi = q < nn[ax] - 1;
            const double *c = cs[ax];
            double g = 0.0;
            if (lo && hi) g = (P.phi[k + st[ax]] - P.phi[k - st[ax]]) / (c[q + 1] - c[q - 1]);
            else if (hi) g = (P.phi[k + st[ax]] - P.phi[k]) / (c[q + 1] - c[q]);
            else if (lo) g = (P.phi[k] - P.phi[k - st[ax]]) / (c[q] - c[q - 1]);
            g2 += g * g;
        }
        m = fmax(m, g2);
    }
    if (grid_max(m, P.part, P.ticket + 8)) P.res[R_OUT] = m;
}

// sum over semiconductor nodes of n and p times the node volume -> res[R_OUT + 1, + 2]
__global__ void k_out_sums(const DevP *__restrict__ Ps) {
    const DevP &P = Ps[blockIdx.y];
    double acc[2] = {0.0, 0.0};
    SS_GRID_LOOP(k, P.N) {
        if (fl_kind(P.flags[k]) != K_SEMI) continue;
        const Node a = unidx(k, P.Nx, P.Ny);
        const double v = P.Lx[a.i] * P.Ly[a.j] * P.Lz[a.l];
        acc[0] += P.n[k] * v;
        acc[1] += P.p[k] * v;
    }
    if (grid_sum<2>(acc, P.part, P.ticket + 8)) {
        P.res[R_OUT + 1] = acc[0];
        P.res[R_OUT + 2] = acc[1];
    }
}

// largest field across an insulator edge (|dpsi| / h over the edges between two
// non-semiconductor nodes of which one is an insulator; the node reported is the insulator
// end) and across the oxide of a Robin gate (|psi - (V + Cref - phi_m)| / tox).  The edge
// candidates are keyed by their scan position 6 k + dir, so ties resolve to the edge the
// reference's node-order scan meets first.  mode 0: edges -> res[R_OUT + 3] (value),
// res[R_OUT + 4] (node); mode 1: Robin gates -> res[R_OUT + 5], res[R_OUT + 6]; the node is
// -1 without a candidate.
__global__ void k_out_insfield(const DevP *__restrict__ Ps, int mode) {
    const DevP &P = Ps[blockIdx.y];
    double best = -1.0;
    long long key = NO_IDX;
    SS_GRID_LOOP(k, P.N) {
        const uint32_t fk = P.flags[k];
        if (mode == 0) {
            if (fl_kind(fk) == K_SEMI) continue;
            const Node a = unidx(k, P.Nx, P.Ny);
            const int ns = nslots(P);
            for (int dir = 0; dir < ns; dir++) {
                int b;
                double h, cf;
                if (!edge_any(P, k, a, dir, b, cf, h) || b < k) continue;
                const int kb = fl_kind(P.flags[b]);
                if (kb == K_SEMI) continue;
                if (fl_kind(fk) != K_INS && kb != K_INS) continue;
                const double F = fabs(P.phi[b] - P.phi[k]) / h;
                if (F > best) { best = F; key = (long long)ns * k + dir; }   // this thread's scan order
            }
        } else {
            if (P.robA[k] == 0.0) continue;
            const int g = fl_gate(fk);
            if (g <= 0 || g > NC_MAX) continue;
            const ConD &cn = P.cons[g - 1];
            const double tox = cn.tox > 0.0 ? cn.tox : 10e-9;
            const double pm = cn.phi_m > 0.0 ? cn.phi_m : P.Cref;
            const double F = fabs(P.phi[k] - (cn.V + P.Cref - pm)) / tox;
            if (F > best) { best = F; key = k; }
        }
    }
    if (grid_argmax(best, key, P.part, P.ticket + 8)) {
        long long at = -1;
        if (key != NO_IDX) {
            if (mode == 0) {
                const int ns = nslots(P);
                const int k = int(key / ns), dir = int(key - (long long)ns * (key / ns));
                const Node a = unidx(k, P.Nx, P.Ny);
                int b = k;
                double h, cf;
                edge_any(P, k, a, dir, b, cf, h);
                at = fl_kind(P.flags[k]) == K_INS ? k : b;
            } else {
                at = key;
            }
        }
        P.res[R_OUT + 3 + 2 * mode] = best;
        P.res[R_OUT + 4 + 2 * mode] = (double)at;
    }
}

// terminal charges of a charge partition (owner[k] = terminal slot 0..nt-1 of node k, or
// -1): the flux eps_bar A / h (psi_k - psi_b) out of every owned node through each edge to
// a node of another owner, added to the owner (and to slot nt when the other node has
// none), plus the Robin gates' oxide charge moved from the node's owner to the gate's
// terminal.  Per-block sums in P.partc (<= 256 blocks x (nt + 1) <= 33 of its 96), the last
// block adds them in block order into out[0..nt].
struct QTerm {
    int nt;
    int gate_term[NC_MAX];
};
__global__ void __launch_bounds__(OUT_TPB) k_out_qterm(const DevP *__restrict__ Ps, const int *__restrict__ owner,
                                                        QTerm q, double *out) {
    const DevP &P = Ps[blockIdx.y];
    const int nt = q.nt;
    __shared__ double sacc[33][OUT_TPB / 32];
    __shared__ bool is_last;
    double acc[33];
    for (int t = 0; t <= nt; t++) acc[t] = 0.0;
    SS_GRID_LOOP(k, P.N) {
        const int t = owner[k];
        if (t >= 0 && t < nt) {
            const Node a = unidx(k, P.Nx, P.Ny);
            const int ns = nslots(P);
            for (int dir = 0; dir < ns; dir++) {
                int b;
                double cf, h;
                if (!edge_any(P, k, a, dir, b, cf, h)) continue;
                const int tb = owner[b];
                if (tb == t) continue;
                const double f = cf * (P.phi[k] - P.phi[b]);
                acc[t] += f;
                if (tb < 0 || tb >= nt) acc[nt] += f;
            }
        }
        if (P.robA[k] != 0.0) {
            const int g = fl_gate(P.flags[k]) - 1;
            if (g >= 0 && g < NC_MAX) {
                const ConD &cn = P.cons[g];
                const double Cox = EPS_OX / (cn.tox > 0.0 ? cn.tox : 10e-9);
                const double pm = cn.phi_m > 0.0 ? cn.phi_m : P.Cref;
                const double f = P.robA[k] * Cox * (P.phi[k] - (cn.V + P.Cref - pm));
                const int tg = q.gate_term[g];
                if (t >= 0 && t < nt) acc[t] += f;
                if (tg >= 0 && tg < nt) acc[tg] -= f;
            }
        }
    }
    // block sums, one terminal at a time, in a fixed order
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int t = 0; t <= nt; t++) {
        double v = acc[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sacc[t][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x <= nt) {
        double s = 0.0;
        for (int w = 0; w < OUT_TPB / 32; w++) s += sacc[threadIdx.x][w];
        P.partc[blockIdx.x * 96 + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(P.ticket + 8, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    if (threadIdx.x <= nt) {
        double s = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) s += __ldcg(P.partc + b * 96 + threadIdx.x);
        out[threadIdx.x] = s;
    }
    if (threadIdx.x == 0) P.ticket[8] = 0u;
}

static int out_blocks(const Inst &d) {
    int nb = (int)((d.N + OUT_TPB - 1) / OUT_TPB);
    return nb < 1 ? 1 : (nb > OUT_BLOCKS ? OUT_BLOCKS : nb);
}
static void read(Inst &d, int slot, int n, double *v) {
    cudaMemcpyAsync(v, d.g.h.res + slot, n * sizeof(double), cudaMemcpyDeviceToHost, d.g.st);
    cudaStreamSynchronize(d.g.st);
}

double out_emax(Inst &d) {
    Ctx c = make_ctx(d);
    if (d.unstr) launch_emax_g(c);                  // least-squares gradients of a graph mesh
    else SS_LAUNCH(PF_DISPLAY, d.N, k_out_emax, dim3(out_blocks(d), 1), OUT_TPB, c.st, c.dP);
    double v;
    read(d, R_OUT, 1, &v);
    return std::sqrt(v);
}
void out_carrier_sums(Inst &d, double *out) {
    Ctx c = make_ctx(d);
    SS_LAUNCH(PF_DISPLAY, d.N, k_out_sums, dim3(out_blocks(d), 1), OUT_TPB, c.st, c.dP);
    read(d, R_OUT + 1, 2, out);
}
// largest insulator field and its node (-1 when there is none)
double out_ins_field(Inst &d, long long *node) {
    Ctx c = make_ctx(d);
    SS_LAUNCH(PF_DISPLAY, d.N, k_out_insfield, dim3(out_blocks(d), 1), OUT_TPB, c.st, c.dP, 0);
    SS_LAUNCH(PF_DISPLAY, d.N, k_out_insfield, dim3(out_blocks(d), 1), OUT_TPB, c.st, c.dP, 1);
    double v[4];
    read(d, R_OUT + 3, 4, v);
    double best = 0.0;                                          // the reference starts at 0 and
    long long kb = -1;                                          // keeps a strictly larger field
    if (v[1] >= 0.0 && v[0] > best) { best = v[0]; kb = (long long)v[1]; }
    if (v[3] >= 0.0 && v[2] > best) { best = v[2]; kb = (long long)v[3]; }   // gates after edges
    *node = kb;
    return best;
}
// terminal charges out[0..nt] of the owner map (device array of N terminal slots)
int out_terminal_charges(Inst &d, const int *owner_dev, int nt, const int *gate_term, double *out) {
    if (nt < 0 || nt > NC_MAX) return 0;
    Ctx c = make_ctx(d);
    QTerm q;
    q.nt = nt;
    for (int g = 0; g < NC_MAX; g++) q.gate_term[g] = gate_term[g];
    SS_LAUNCH(PF_DISPLAY, d.N, k_out_qterm, dim3(out_blocks(d), 1), OUT_TPB, c.st, c.dP, owner_dev, q, d.g.scratch);
    cudaMemcpyAsync(out, d.g.scratch, (nt + 1) * sizeof(double), cudaMemcpyDeviceToHost, d.g.st);
    cudaStreamSynchronize(d.g.st);
    return 1;
}

}  // namespace ss
