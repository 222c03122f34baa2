// Batched resolve: several bias vectors solved at once from the current instance's solved
// state.  Each bias vector goes to a worker instance (its own device memory and CUDA
// stream, driven by its own host thread) that starts from a copy of the source state, so
// the solves are independent and run concurrently on the GPU.  This serves the callers
// that multiply solves around one operating point - the C-V perturbation solves of
// main.py's cap_matrix (main.py:4034-4087) and the floating-node secant of solve_floating
// (main.py:3575-3636) - which the reference runs one after the other, each with
// api3_resolve from the restored state.
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "solver_ctx.h"

using namespace ss;
extern Inst *b200_global_dev();

namespace {
std::mutex g_pool_mu;
std::map<const Inst *, std::vector<std::unique_ptr<Inst>>> g_pool;   // workers per source instance

// the worker becomes a copy of src's configuration with src's solved state, at src's
// solved voltages (the state api3_set_state would install), device memory kept
int clone_into(Inst &w, Inst &src) {
    Gpu keep = w.g;
    // the worker's device already holds this set-up when it last copied the same upload
    const bool same = keep.ready && w.clone_src == &src && w.clone_gen == src.upload_gen && !src.dirty;
    const unsigned long long own_gen = w.upload_gen;
    w = src;                                   // configuration, derived tables, tunables
    w.g = keep;
    w.dirty = same ? 0 : 1;                    // else upload the set-up to the worker's memory
    w.upload_gen = same ? own_gen : 0;
    w.cache.clear();
    w.cache_ok.clear();
    w.seed_on = 0;                             // the learned model stays with the source
    if (!prepare(w)) return 0;
    w.clone_src = &src;
    w.clone_gen = src.upload_gen;
    const size_t bytes = w.N * sizeof(double);
    cudaStreamSynchronize(src.g.st);           // the source state is final
    cudaMemcpyAsync(w.g.h.phi, src.g.h.phi, bytes, cudaMemcpyDeviceToDevice, w.g.st);
    cudaMemcpyAsync(w.g.h.phin, src.g.h.phin, bytes, cudaMemcpyDeviceToDevice, w.g.st);
    cudaMemcpyAsync(w.g.h.phip, src.g.h.phip, bytes, cudaMemcpyDeviceToDevice, w.g.st);
    if (src.g.te_on && w.g.te_on) {            // the image-force band of the source's last iteration
        cudaMemcpyAsync(w.g.h.qcn, src.g.h.qcn, bytes, cudaMemcpyDeviceToDevice, w.g.st);
        cudaMemcpyAsync(w.g.h.qcp, src.g.h.qcp, bytes, cudaMemcpyDeviceToDevice, w.g.st);
        cudaMemcpyAsync(w.g.h.imgn, src.g.h.imgn, bytes, cudaMemcpyDeviceToDevice, w.g.st);
        cudaMemcpyAsync(w.g.h.imgp, src.g.h.imgp, bytes, cudaMemcpyDeviceToDevice, w.g.st);
    }
    double Va[NC_MAX];
    for (int c = 0; c < w.n_cons; c++) { Va[c] = src.cons[c].Vprev; w.cons[c].Vprev = Va[c]; }
    set_vrange(w, Va);
    apply_bc(w, Va);
    clamp_qf(w);
    rebuild_np(w);
    upd_mob(w);
    cudaStreamSynchronize(w.g.st);
    w.have_solution = 1;
    w.e_n = 0;                                 // no sweep-predictor history
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}
}  // namespace

namespace ss {
// release the batched-resolve workers of `src` (their device memory and streams); called
// when the source instance itself is freed, so no worker outlives it
int batch_pool_release(const Inst *src) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pool.find(src);
    if (it == g_pool.end()) return 0;
    for (auto &w : it->second) gpu_free(*w);
    g_pool.erase(it);
    return 1;
}
}  // namespace ss

extern "C" {

// Solve n bias vectors (V: n x ncon volts, contact order) from the current instance's
// solved state, each independently (as api3_resolve after restoring that state would),
// `workers` at a time (<= 0: min(n, 8)).  Per vector: terminal currents I (n x ncon), their
// resolution floors Iflr (n x ncon, may be null) and the converged flag conv (n, may be
// null).  The current instance is not changed.  Returns the number of converged solves,
// -1 without a solution to start from or on a device error.
int api3b_resolve_batch(int n, const double *V, double *I, double *Iflr, int *conv, int workers) {
    Inst &src = *b200_global_dev();
    if (n <= 0) return 0;
    if (!src.have_solution || !src.g.ready || !V || !I) return -1;
    const int nc = src.n_cons;
    int W = workers > 0 ? workers : (n < 8 ? n : 8);
    if (W > n) W = n;
    std::vector<Inst *> ws;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        auto &pool = g_pool[&src];
        while ((int)pool.size() < W) pool.emplace_back(new Inst());
        for (int q = 0; q < W; q++) ws.push_back(pool[q].get());
    }
    std::vector<int> ok(n, 0), fail(W, 0);
    auto run = [&](int q) {
        Inst &w = *ws[q];
        for (int j = q; j < n; j += W) {
            if (!clone_into(w, src)) { fail[q] = 1; return; }
            for (int c = 0; c < nc; c++) w.cons[c].V = V[(size_t)j * nc + c];
            ok[j] = do_solve(w, 1);
            for (int c = 0; c < nc; c++) {
                I[(size_t)j * nc + c] = w.cons[c].I;
                if (Iflr) Iflr[(size_t)j * nc + c] = w.cons[c].Iflr;
            }
            if (conv) conv[j] = ok[j];
        }
    };
    std::vector<std::thread> th;
    for (int q = 0; q < W; q++) th.emplace_back(run, q);
    for (auto &t : th) t.join();
    for (int q = 0; q < W; q++)
        if (fail[q]) return -1;
    int nok = 0;
    for (int j = 0; j < n; j++) nok += ok[j];
    return nok;
}

// release the worker instances of the current instance's batched resolves
int api3b_resolve_batch_free(void) { return batch_pool_release(b200_global_dev()); }

}  // extern "C"
