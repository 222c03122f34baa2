// Launch accounting and CUDA-event kernel timing (see prof.h).
#include "prof.h"

#include <map>
#include <utility>
#include <vector>

namespace ss {

// Algorithmic bytes per node, FP64 words counted once per array a kernel must touch:
//   Poisson build: flags 4 + psi, phi_n, phi_p, Nd, Na, Nf, bgn 56 read; A 56 + F 8 + sc 8 written
//   SG assembly: flags 4 + psi, c, n, p, bgn, Nd, Na, 6 face mobilities 104; A 56 + rhs, sc, dsc 24
//   smoother half sweeps: the colour's 6 couplings + pivot + source + result, plus the other
//   colour's values read once; residual + restriction: 7 couplings + x + b (+ weight)
//   Krylov SpMV + dot: 7 couplings + x + y + one dot operand; updates: the vectors touched
const double kProfBytesPerNode[PF_NPROF] = {
    132.0,  // PF_POISSON
    52.0,   // PF_REBUILD
    92.0,   // PF_UPDMOB
    188.0,  // PF_CONT_ASM
    92.0,   // PF_CONT_UPD
    46.0,   // PF_SMOOTH_B
    38.0,   // PF_SMOOTH_R
    80.0,   // PF_RESID_RESTRICT
    25.0,   // PF_PROLONG
    80.0,   // PF_LEVEL_RESID
    8.0,    // PF_COARSE (per coarse unknown; dense inverse in shared/L2)
    80.0,   // PF_GALERKIN
    20.0,   // PF_WEIGHTS
    64.0,   // PF_ILU_DIAG
    8.0,    // PF_COARSE_SETUP
    80.0,   // PF_KRY_SPMV_DOT
    48.0,   // PF_KRY_UPDATE
    16.0,   // PF_KRY_DOT
    96.0,   // PF_KRY_INIT
    100.0,  // PF_CURRENTS (per contact node)
    40.0,   // PF_AA (per state entry)
    60.0,   // PF_BC
    24.0,   // PF_VEC
    24.0,   // PF_CCL
    120.0,  // PF_DISPLAY
    23.0,   // PF_SMOOTH_B32 (FP32 words: half the FP64 figures)
    19.0,   // PF_SMOOTH_R32
    40.0,   // PF_RESID_RESTRICT32
    12.5,   // PF_PROLONG32
    40.0,   // PF_LEVEL_RESID32
    4.0,    // PF_COARSE32
    40.0,   // PF_GALERKIN32
    12.0,   // PF_WEIGHTS32
    32.0,   // PF_ILU_DIAG32
    4.0,    // PF_COARSE_SETUP32
    40.0,   // PF_KRY_SPMV_DOT32
    24.0,   // PF_KRY_UPDATE32
    8.0,    // PF_KRY_DOT32
    24.0,   // PF_KRY_INIT32: rhs read; r, rh, p, v, x written
    92.0,   // PF_REFINE: FP64 A 56 + x, r read and written 32, FP32 correction 4 (FP64 start: 96)
    96.0,   // PF_CONVERT32: A and row weights 64 read, 32 written
    112.0,  // PF_SEED: x1, x0 of 3 fields at the node (neighbours from cache), flags, doping; 3 fields written
    64.0,   // PF_METAL: column node state, exchange slots and the per-node results
    1.0,    // PF_PERSIST: algorithmic bytes of the whole solve, booked after it (prof_set_last)
    1.0,    // PF_PERSIST32
};
int pf_f32(int id) {
    switch (id) {
    case PF_SMOOTH_B: return PF_SMOOTH_B32;
    case PF_SMOOTH_R: return PF_SMOOTH_R32;
    case PF_RESID_RESTRICT: return PF_RESID_RESTRICT32;
    case PF_PROLONG: return PF_PROLONG32;
    case PF_LEVEL_RESID: return PF_LEVEL_RESID32;
    case PF_COARSE: return PF_COARSE32;
    case PF_GALERKIN: return PF_GALERKIN32;
    case PF_WEIGHTS: return PF_WEIGHTS32;
    case PF_ILU_DIAG: return PF_ILU_DIAG32;
    case PF_COARSE_SETUP: return PF_COARSE_SETUP32;
    case PF_KRY_SPMV_DOT: return PF_KRY_SPMV_DOT32;
    case PF_KRY_UPDATE: return PF_KRY_UPDATE32;
    case PF_KRY_DOT: return PF_KRY_DOT32;
    case PF_KRY_INIT: return PF_KRY_INIT32;
    default: return id;
    }
}
const char *kProfName[PF_NPROF] = {
    "poisson_eval", "rebuild_np", "upd_mob", "cont_assemble", "cont_update", "smooth_black", "smooth_red",
    "resid_restrict", "prolong", "level_resid", "coarse_solve", "galerkin", "mg_weights", "ilu_diag",
    "coarse_setup", "krylov_spmv_dot", "krylov_update", "krylov_dot", "krylov_init", "terminal_currents",
    "anderson", "boundary", "vector", "labelling", "display", "smooth_black_f32", "smooth_red_f32",
    "resid_restrict_f32", "prolong_f32", "level_resid_f32", "coarse_solve_f32", "galerkin_f32", "mg_weights_f32",
    "ilu_diag_f32", "coarse_setup_f32", "krylov_spmv_dot_f32", "krylov_update_f32", "krylov_dot_f32",
    "krylov_init_f32", "refine_f64", "convert_f32", "learned_seed", "metal_contacts", "persistent_solve",
    "persistent_solve_f32"};

bool g_prof_on = false;
bool g_pdl = true;
std::atomic<unsigned long long> g_launches{0};
thread_local unsigned long long t_launches = 0;

namespace {
struct Rec {
    int id;
    double nodes;
    cudaEvent_t a, b;
};
std::vector<Rec> g_recs;
size_t g_used = 0;
double g_ms[PF_NPROF], g_cnt[PF_NPROF], g_bytes[PF_NPROF];
std::map<std::pair<int, long long>, std::pair<double, double>> g_detail;   // (class, nodes) -> (ms, launches)
}  // namespace

void prof_begin(int id, cudaStream_t st) {
    if (g_used == g_recs.size()) {
        Rec r{};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        g_recs.push_back(r);
    }
    Rec &r = g_recs[g_used];
    r.id = id;
    cudaEventRecord(r.a, st);
}
void prof_end(int, cudaStream_t st, double nodes) {
    Rec &r = g_recs[g_used];
    r.nodes = nodes;
    cudaEventRecord(r.b, st);
    g_used++;
    if (g_used >= 4096) prof_collect();     // bound the pool
}
void prof_set_last(int id, double bytes) {
    for (size_t q = g_used; q-- > 0;)
        if (g_recs[q].id == id) { g_recs[q].nodes = bytes; return; }
}
void prof_collect() {
    for (size_t q = 0; q < g_used; q++) {
        Rec &r = g_recs[q];
        cudaEventSynchronize(r.b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        g_ms[r.id] += ms;
        g_cnt[r.id] += 1.0;
        g_bytes[r.id] += r.nodes * kProfBytesPerNode[r.id];
        auto &e = g_detail[{r.id, (long long)r.nodes}];
        e.first += ms;
        e.second += 1.0;
    }
    g_used = 0;
}
void prof_reset() {
    prof_collect();
    for (int i = 0; i < PF_NPROF; i++) g_ms[i] = g_cnt[i] = g_bytes[i] = 0.0;
    g_detail.clear();
}
void prof_read(int id, double *ms, double *count, double *bytes) {
    prof_collect();
    *ms = g_ms[id];
    *count = g_cnt[id];
    *bytes = g_bytes[id];
}

}  // namespace ss

extern "C" {
// 1: time every launch with CUDA events from now on; 0: stop.  Returns the kernel classes.
int b200x_prof(int on) {
    if (on) ss::prof_reset();
    else ss::prof_collect();
    ss::g_prof_on = on != 0;
    return ss::PF_NPROF;
}
// per kernel class: total ms, launches, algorithmic bytes since the last b200x_prof(1)
int b200x_prof_read(int id, double *ms, double *count, double *bytes) {
    if (id < 0 || id >= ss::PF_NPROF) return 0;
    ss::prof_read(id, ms, count, bytes);
    return 1;
}
const char *b200x_prof_name(int id) { return (id >= 0 && id < ss::PF_NPROF) ? ss::kProfName[id] : ""; }
// q-th (class, launch size) bucket: class id, nodes per launch, total ms, launches; 0 past the end
int b200x_prof_detail(int q, int *id, double *nodes, double *ms, double *count) {
    ss::prof_collect();
    int i = 0;
    for (const auto &e : ss::g_detail) {
        if (i++ != q) continue;
        *id = e.first.first; *nodes = (double)e.first.second; *ms = e.second.first; *count = e.second.second;
        return 1;
    }
    return 0;
}
// kernel launches of this library since it was loaded
unsigned long long b200x_launches(void) { return ss::g_launches.load(); }
}
