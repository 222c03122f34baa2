// Autotuner of the linear-algebra launch shapes of one solver instance: rows per block of
// the row-blocked level passes (block 32 x rpb) and the most row blocks of a pass (more rows
// per thread beyond it), coarse rows per block of the residual + restriction pass, the
// block count of the grid-stride node kernels, and the level size at which the small-level
// kernel takes over.  It times
// V-cycles of the instance's own multigrid hierarchy (the precision its solves use) on
// the GPU with CUDA events and keeps the fastest shapes, one parameter at a time.  Results
// are cached per mesh shape and precision for the process, so instances of the same
// shape tune once.  The shapes change no arithmetic of a pass; the small-level split
// changes which kernel sums a restriction, so Krylov iteration counts may move by round-off.
#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>

#include "solver_ctx.h"

using namespace ss;
extern Inst *b200_global_dev();

namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, Tune> g_tune_cache;

// microseconds per V-cycle of the instance with shapes t (best of two timings)
double time_vcycle(Inst &d, const Tune &t, int mixed, int reps) {
    const Tune keep = d.tune;
    d.tune = t;
    Ctx c = make_ctx(d);
    const int which = mixed ? 15 : 8;
    double best = 1e30;
    for (int r = 0; r < 2; r++) {
        const double us = bench_la_kernel(c, d.g.mg, which, reps);
        if (us > 0.0 && us < best) best = us;
    }
    d.tune = keep;
    return best;
}
}  // namespace

extern "C" {

// mode 0: back to the default shapes; 1: tune the current instance now; 2: take the cached
// shapes of this mesh shape and precision, tuning when there are none.  The instance must
// have solved once (its device memory and multigrid hierarchy exist) and no other work of
// this process should run on the GPU meanwhile.  Returns the chosen V-cycle time in
// microseconds, 0 for mode 0, -1 when the instance has not solved yet.
double api3b_autotune(int mode) {
    Inst &d = *b200_global_dev();
    if (mode == 0) {
        d.tune = Tune();
        return 0.0;
    }
    if (!d.g.ready || d.g.mg.maxlev < 1) return -1.0;
    if (d.unstr) return -1.0;                  // a graph mesh has no tensor multigrid to tune
    const int mixed = use_mixed(d);
    const auto key = std::make_tuple(d.Nx, d.Ny, d.Nz, mixed);
    if (mode == 2) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            d.tune = it->second;
            return d.tune.us;
        }
    }
    const int reps = 20;
    Tune best = Tune();
    best.us = time_vcycle(d, best, mixed, reps);
    const int small_c[] = {1024, 2048, 4096, 8192};
    const int rpb_c[] = {2, 4, 8, 16, 32};
    const int rq_c[] = {1, 2, 4, 8};
    const int cap_c[] = {148 * 4, 148 * 8, 148 * 12};
    const int zcap_c[] = {65535, 148 * 2, 148};
    for (int pass = 0; pass < 5; pass++) {
        const int *cand = pass == 0 ? small_c : (pass == 1 ? rpb_c : (pass == 2 ? cap_c : (pass == 3 ? zcap_c : rq_c)));
        const int nc = pass == 0 || pass == 4 ? 4 : (pass == 1 ? 5 : 3);
        for (int q = 0; q < nc; q++) {
            Tune t = best;
            if (pass == 0) t.small_nodes = cand[q];
            else if (pass == 1) t.rpb = cand[q];
            else if (pass == 2) t.grid_cap = cand[q];
            else if (pass == 3) t.zcap = cand[q];
            else t.rq = cand[q];
            const double us = time_vcycle(d, t, mixed, reps);
            if (d.verbose)
                std::fprintf(stderr, "semisim-b200: autotune rpb %d cap %d small %d zcap %d rq %d: %.2f us\n", t.rpb,
                             t.grid_cap, t.small_nodes, t.zcap, t.rq, us);
            if (us < 0.97 * best.us) {       // keep a change only when it clearly wins
                best = t;
                best.us = us;
            }
        }
    }
    best.tuned = 1;
    d.tune = best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
    return best.us;
}

// the current instance's launch shapes: rows per block, grid cap, small-level size, most
// row blocks per pass (the restriction's coarse rows per block are not reported)
int api3b_tune_get(int *rpb, int *grid_cap, int *small_nodes, int *zcap) {
    Inst &d = *b200_global_dev();
    *rpb = d.tune.rpb;
    *grid_cap = d.tune.grid_cap;
    *small_nodes = d.tune.small_nodes;
    if (zcap) *zcap = d.tune.zcap;
    return d.tune.tuned;
}

}  // extern "C"
