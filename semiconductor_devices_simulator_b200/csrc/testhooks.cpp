// Kernel-level test hooks (b200x_*): run one device kernel of the solve path on the
// prepared global device and copy its inputs / outputs through caller buffers.  The
// parity tests use them to compare every kernel with the oracle on seeded states.
// They are not part of the reference ABI.
#include <cmath>
#include <cstring>

#include "solver_ctx.h"

using namespace ss;

namespace ss {
int float_fix(Inst &d, int hole);
}
namespace {
Inst *dev();
}
extern Inst *b200_global_dev();

namespace {
Inst *dev() { return b200_global_dev(); }
double *arr(Inst &d, int which) {
    DevP &P = d.g.h;
    switch (which) {
    case 0: return P.phi; case 1: return P.phin; case 2: return P.phip;
    case 3: return P.n; case 4: return P.p; case 5: return P.mu0n; case 6: return P.mu0p;
    case 7: return P.sol; case 8: return P.rhs; case 9: return P.sc; case 10: return P.dsc;
    }
    if (which >= 16 && which < 22) return P.fmu[which - 16];
    if (which >= 22 && which < 25) return P.h1[which - 22];
    if (which >= 25 && which < 28) return P.e2[which - 25];
    return nullptr;
}
void dump7(Inst &d, double *const *A, size_t n, double *A7) {
    if (!A7) return;
    for (int q = 0; q < 7; q++) cudaMemcpyAsync(A7 + q * n, A[q], n * 8, cudaMemcpyDeviceToHost, d.g.st);
}
void sync(Inst &d) { cudaStreamSynchronize(d.g.st); }
double res(Inst &d, int slot) {
    double v = 0;
    cudaMemcpyAsync(&v, d.g.h.res + slot, 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    return v;
}
void voltages(Inst &d) {
    double Va[NC_MAX];
    for (int c = 0; c < d.n_cons; c++) Va[c] = d.cons[c].V;
    set_vrange(d, Va);
    upload_voltages(d, Va);
}
}  // namespace

extern "C" {

int b200x_prepare(void) {
    Inst &d = *dev();
    if (!prepare(d)) return 0;
    voltages(d);
    return 1;
}
int b200x_masks(int *kind, int *con, int *gate, double *robA) {
    Inst &d = *dev();
    if (d.flags.size() != d.N) return 0;
    for (size_t k = 0; k < d.N; k++) {
        kind[k] = fl_kind(d.flags[k]); con[k] = fl_con(d.flags[k]); gate[k] = fl_gate(d.flags[k]);
        if (robA) robA[k] = d.robA.empty() ? 0.0 : d.robA[k];
    }
    return 1;
}
// metal contacts: the exchange update at the contacts' voltages, and the entry / column
// records (the entry node's own column slot holds its emission terms here; the reference
// keeps them only in te_K / te_G)
int b200x_te_update(void) {
    Inst &d = *dev();
    if (!d.g.ready || !d.g.te_on) return 0;
    double Va[NC_MAX];
    for (int c = 0; c < d.n_cons; c++) Va[c] = d.cons[c].V;
    upload_voltages(d, Va);
    te_update(d);
    sync(d);
    return 1;
}
// gate tunnelling: the path update at the contacts' voltages, and the path / column records
int b200x_tun_update(void) {
    Inst &d = *dev();
    if (!d.g.ready || !d.g.tun_on) return 0;
    double Va[NC_MAX];
    for (int c = 0; c < d.n_cons; c++) Va[c] = d.cons[c].V;
    upload_voltages(d, Va);
    tun_update(d);
    sync(d);
    return 1;
}
int b200x_tun(int *cnt, double *tpG, double *colK, long long *tpk, long long *colk) {
    Inst &d = *dev();
    cnt[0] = cnt[1] = 0;
    if (!d.g.ready || !d.g.tun_on) return 0;
    const TunD &T = d.g.tun;
    cnt[0] = T.n_tp; cnt[1] = T.n_col;
    if (tpG) cudaMemcpyAsync(tpG, T.tp_G, 2 * (size_t)T.n_tp * 8, cudaMemcpyDeviceToHost, d.g.st);
    if (colK) cudaMemcpyAsync(colK, T.col_K, 2 * (size_t)T.n_col * 8, cudaMemcpyDeviceToHost, d.g.st);
    std::vector<int> a((size_t)T.n_tp), b((size_t)T.n_col);
    cudaMemcpyAsync(a.data(), T.tp_k, a.size() * 4, cudaMemcpyDeviceToHost, d.g.st);
    cudaMemcpyAsync(b.data(), T.col_k, b.size() * 4, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    if (tpk) for (size_t p = 0; p < a.size(); p++) tpk[p] = a[p];
    if (colk) for (size_t q = 0; q < b.size(); q++) colk[q] = b[q];
    return T.n_tp;
}
int b200x_set_qc(const double *qcn, const double *qcp) {
    Inst &d = *dev();
    if (!d.g.ready || !d.g.te_on) return 0;
    cudaMemcpyAsync(d.g.h.qcn, qcn, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    cudaMemcpyAsync(d.g.h.qcp, qcp, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    cudaMemcpyAsync(d.g.h.imgn, qcn, d.N * 8, cudaMemcpyHostToDevice, d.g.st);   // no MLDA part
    cudaMemcpyAsync(d.g.h.imgp, qcp, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    sync(d);
    return 1;
}
int b200x_te(int *cnt, double *teK, double *teG, double *tcK, double *tcG, double *tcI, double *qcn, double *qcp) {
    Inst &d = *dev();
    cnt[0] = cnt[1] = 0;
    if (!d.g.ready || !d.g.te_on) return 0;
    const TeD &T = d.g.te;
    cnt[0] = T.n_te; cnt[1] = T.n_tc;
    auto cp = [&](double *dst, const double *src, size_t n) {
        if (dst) cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyDeviceToHost, d.g.st);
    };
    cp(teK, T.te_K, 2 * (size_t)T.n_te); cp(teG, T.te_G, 2 * (size_t)T.n_te);
    cp(tcK, T.tc_K, 2 * (size_t)T.n_tc); cp(tcG, T.tc_G, 2 * (size_t)T.n_tc); cp(tcI, T.tc_I, 2 * (size_t)T.n_tc);
    cp(qcn, d.g.h.qcn, d.N); cp(qcp, d.g.h.qcp, d.N);
    sync(d);
    return T.n_te;
}
// the device's incomplete-ionisation constants (ION_W x N); 0 when every dopant is ionised
int b200x_ion(double *out) {
    Inst &d = *dev();
    if (!d.g.ready || !d.g.h.ion) return 0;
    if (out) {
        cudaMemcpyAsync(out, d.g.h.ion, (size_t)ION_W * d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
        sync(d);
    }
    return ION_W;
}
int b200x_set(int which, const double *in) {
    Inst &d = *dev();
    double *a = arr(d, which);
    if (!a) return 0;
    cudaMemcpyAsync(a, in, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    sync(d);
    return 1;
}
int b200x_get(int which, double *out) {
    Inst &d = *dev();
    double *a = arr(d, which);
    if (!a) return 0;
    cudaMemcpyAsync(out, a, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    return 1;
}
double b200x_vlo(void) { return dev()->vlo; }
double b200x_vhi(void) { return dev()->vhi; }
void b200x_apply_bc(void) {
    Inst &d = *dev();
    double Va[NC_MAX];
    for (int c = 0; c < d.n_cons; c++) Va[c] = d.cons[c].V;
    set_vrange(d, Va);
    apply_bc(d, Va);
    sync(d);
}
void b200x_rebuild_np(void) { rebuild_np(*dev()); sync(*dev()); }
// charge-neutral start state at the contact voltages now set (init_eq + boundary values +
// carriers + face mobility), without the Newton solve of an equilibrium
void b200x_init_state(void) {
    Inst &d = *dev();
    launch_init_eq(make_ctx(d));
    double Va[NC_MAX];
    for (int c = 0; c < d.n_cons; c++) Va[c] = d.cons[c].V;
    set_vrange(d, Va);
    apply_bc(d, Va);
    rebuild_np(d);
    upd_mob(d);
    sync(d);
}
void b200x_upd_mob(void) { upd_mob(*dev()); sync(*dev()); }
void b200x_clamp_qf(void) { clamp_qf(*dev()); sync(*dev()); }

// F, stencil and sc of the Poisson system at psi (build) and ||F/diag||
double b200x_poisson(const double *phi, double *F, double *A7, double *sc) {
    Inst &d = *dev();
    voltages(d);
    Ctx c = make_ctx(d);
    cudaMemcpyAsync(d.g.h.phi, phi, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    if (d.unstr) launch_poisson_g(c, nullptr, 1);    // graph: the diagonal in A7[0], couplings per edge
    else launch_poisson(c, nullptr, 1, nullptr);
    const double nrm = res(d, R_PNORM);
    if (F) cudaMemcpyAsync(F, d.g.h.rhs, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    dump7(d, d.g.h.A, d.N, A7);
    if (sc) cudaMemcpyAsync(sc, d.g.h.sc, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    return nrm;
}
void b200x_cont_assemble(int hole, double *A7, double *rhs, double *sc, double *dsc) {
    Inst &d = *dev();
    Ctx c = make_ctx(d);
    if (d.unstr) launch_cont_assemble_g(c, hole);     // graph: the diagonal in A7[0], couplings per edge
    else launch_cont_assemble(c, hole);
    dump7(d, d.g.h.A, d.N, A7);
    if (rhs) cudaMemcpyAsync(rhs, d.g.h.rhs, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    if (sc) cudaMemcpyAsync(sc, d.g.h.sc, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    if (dsc) cudaMemcpyAsync(dsc, d.g.h.dsc, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
}
double b200x_cont_update(int hole, const double *sol, double lo, double hi, double *dq) {
    Inst &d = *dev();
    Ctx c = make_ctx(d);
    cudaMemcpyAsync(d.g.h.sol, sol, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    launch_cont_update(c, hole, lo, hi);
    const double dm = res(d, R_DQ);
    if (dq) cudaMemcpyAsync(dq, hole ? d.g.h.dqp : d.g.h.dqn, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    return dm;
}
void b200x_currents(double *I, double *S, double *In) {
    Inst &d = *dev();
    double Iw[NC_MAX], Sw[NC_MAX];
    terminal_currents(d, Iw, Sw);
    for (int c = 0; c < d.n_cons; c++) { I[c] = Iw[c]; S[c] = Sw[c]; if (In) In[c] = d.cons[c].In; }
}
// multigrid hierarchy of the system now in A (qsign 0 Poisson, +-1 continuity)
int b200x_mg_setup(int qsign) {
    Inst &d = *dev();
    mg_setup(make_ctx(d), d.g.mg, qsign);
    sync(d);
    return d.g.mg.maxlev;
}
int b200x_mg_level(int L, int *dims, double *A7, double *pw) {
    Inst &d = *dev();
    if (L < 0 || L >= (int)d.g.levs.size()) return 0;
    const LevelT<double> &v = d.g.levs[L];
    if (dims) { dims[0] = v.Nx; dims[1] = v.Ny; dims[2] = v.Nz; dims[3] = v.cx; dims[4] = v.cy; dims[5] = v.cz; }
    dump7(d, v.A, (size_t)v.N, A7);
    if (pw) cudaMemcpyAsync(pw, v.pw, (size_t)v.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    return 1;
}
// BiCGSTAB on the system now in A / rhs from sol = x0 (or 1); returns iterations
int b200x_bicgstab(int maxit, double rtol, double atol, int qsign, const double *x0, double *sol, double *rn,
                   double *r0) {
    Inst &d = *dev();
    Ctx c = make_ctx(d);
    if (x0) cudaMemcpyAsync(d.g.h.sol, x0, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    else launch_fill_sel(c, V_SOL, 1.0);
    const int its = bicgstab_core(c, d.g.mg, maxit, rtol, atol, 1, 1, rn, r0, qsign, use_mixed(d));
    if (sol) cudaMemcpyAsync(sol, d.g.h.sol, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    return its;
}
// bounded barrier wait of the persistent solves: a launch whose last block never arrives;
// returns the error word (1) and the blocks that gave up (nb - 1), -1 on a launch error
int b200x_persist_probe(int nb, double wait_s, int *gave_up) {
    Inst &d = *dev();
    Ctx c = make_ctx(d);
    return persist_timeout_probe(c, nb, wait_s, gave_up);
}
// barrier timeline of the next persistent solve: n > 0 arms it, n == 0 reads it (3 n
// values per barrier: first arrival, last arrival, release; ns) and the launch's blocks
int b200x_persist_trace(int n, unsigned long long *out, int *blocks) { return persist_trace(n, out, blocks); }
// block cap of the persistent solves launched from the calling host thread (n >= 0 sets it,
// 0 removes it); returns the previous cap
int b200x_persist_tblocks(int n) { return persist_thread_blocks(n); }
// PCG on the Poisson system now in A / rhs from sol = 0
int b200x_pcg(int maxit, double rtol, double *sol) {
    Inst &d = *dev();
    Ctx c = make_ctx(d);
    launch_fill_sel(c, V_SOL, 0.0);
    const int its = pcg_solve(c, d.g.mg, maxit, rtol, 1, use_mixed(d));
    if (sol) cudaMemcpyAsync(sol, d.g.h.sol, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    return its;
}
int b200x_float_fix(int hole, double *sol) {
    Inst &d = *dev();
    cudaMemcpyAsync(d.g.h.sol, sol, d.N * 8, cudaMemcpyHostToDevice, d.g.st);
    const int r = float_fix(d, hole);
    cudaMemcpyAsync(sol, d.g.h.sol, d.N * 8, cudaMemcpyDeviceToHost, d.g.st);
    sync(d);
    return r;
}
// device memory of the instance (bytes) and the multigrid depth
long long b200x_device_bytes(void) { return (long long)dev()->g.bytes; }

// microseconds per launch of one kernel of the solve path, `reps` back-to-back launches
// on the present state (it overwrites work vectors): 0-10 linear algebra (see
// bench_la_kernel), 20 continuity assembly, 21 Poisson build
double b200x_bench(int which, int reps) {
    Inst &d = *dev();
    if (!d.g.ready || reps < 1) return -1.0;
    Ctx c = make_ctx(d);
    if (which < 20) return bench_la_kernel(c, d.g.mg, which, reps);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    auto one = [&]() {
        if (which == 20) launch_cont_assemble(c, 0);
        else launch_poisson(c, nullptr, 1, nullptr);
    };
    for (int r = 0; r < 3; r++) one();
    cudaEventRecord(a, c.st);
    for (int r = 0; r < reps; r++) one();
    cudaEventRecord(b, c.st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return 1e3 * ms / reps;
}

// thermal voltage of the reference material (the unit of the learned predictor's
// outputs); 0 before the device is prepared
double b200x_vtref(void) { return dev()->g.ready ? dev()->g.h.VTref : 0.0; }

// learned predictor on the present history: psi, phi_n, phi_p = h1 + s (h1 - e2) +
// VT * MLP (the step voltages dv: 4 values, volts); 1 = done (a model must be loaded)
int b200x_seed_run(double s, const double *dv4) {
    Inst &d = *dev();
    if (!d.g.ready || !d.g.seedw) return 0;
    double dv[4] = {0., 0., 0., 0.};
    for (int q = 0; q < 4; q++) dv[q] = dv4 ? dv4[q] : 0.;
    launch_mlp_seed(d, s, dv);
    sync(d);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}

// refinement steps and FP64 take-overs of the instance's refined continuity solves
void b200x_ir_stats(long long *steps, long long *fallbacks) {
    Inst &d = *dev();
    *steps = d.ir_steps;
    *fallbacks = d.ir_fallbacks;
}

// select the CUDA device of the solver (before its first solve); 1 = done
int b200x_set_device(int dev) { return select_device(dev); }

// CUDA-event timer on the solver's own stream: op 0 records the start, op 1 records the
// stop, waits for it and returns the elapsed milliseconds (-1 before the first solve)
double b200x_stream_timer(int op) {
    Inst &d = *dev();
    if (!d.g.ready) return -1.0;
    cudaEvent_t *ev = d.g.tev;
    if (!ev[0]) { cudaEventCreate(&ev[0]); cudaEventCreate(&ev[1]); }
    if (op == 0) { cudaEventRecord(ev[0], d.g.st); return 0.0; }
    cudaEventRecord(ev[1], d.g.st);
    cudaEventSynchronize(ev[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    return ms;
}

}  // extern "C"
