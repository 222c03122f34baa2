// Launch accounting: every kernel launch of the library goes through SS_LAUNCH, which
// counts it and, while profiling is switched on (b200x_prof), brackets it with CUDA
// events on its own stream and books the kernel's algorithmic bytes (bytes per node
// of the kernel class times the nodes of the launch).
#pragma once
#include <cuda_runtime.h>

#include <atomic>

namespace ss {

enum ProfId {
    PF_POISSON, PF_REBUILD, PF_UPDMOB, PF_CONT_ASM, PF_CONT_UPD, PF_SMOOTH_B, PF_SMOOTH_R, PF_RESID_RESTRICT,
    PF_PROLONG, PF_LEVEL_RESID, PF_COARSE, PF_GALERKIN, PF_WEIGHTS, PF_ILU_DIAG, PF_COARSE_SETUP,
    PF_KRY_SPMV_DOT, PF_KRY_UPDATE, PF_KRY_DOT, PF_KRY_INIT, PF_CURRENTS, PF_AA, PF_BC, PF_VEC, PF_CCL,
    PF_DISPLAY, PF_NPROF
};

// algorithmic bytes per node of each kernel class (FP64 arrays; see the kernel files)
extern const double kProfBytesPerNode[PF_NPROF];
extern const char *kProfName[PF_NPROF];

extern bool g_prof_on;
extern std::atomic<unsigned long long> g_launches;     // all threads
extern thread_local unsigned long long t_launches;     // this thread
void prof_begin(int id, cudaStream_t st);
void prof_end(int id, cudaStream_t st, double nodes);
void prof_collect();
void prof_reset();
void prof_read(int id, double *ms, double *count, double *bytes);

}  // namespace ss

#define SS_LAUNCH(ID, NODES, KERN, GRID, BLOCK, ST, ...)                \
    do {                                                                \
        ss::g_launches++;                                               \
        ss::t_launches++;                                               \
        if (ss::g_prof_on) ss::prof_begin((ID), (ST));                  \
        KERN<<<(GRID), (BLOCK), 0, (ST)>>>(__VA_ARGS__);                \
        if (ss::g_prof_on) ss::prof_end((ID), (ST), (double)(NODES));   \
    } while (0)
