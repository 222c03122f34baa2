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
    PF_DISPLAY,
    // FP32 twins of the linear-algebra classes (inner solves of the refined path) and the
    // FP64 refinement kernels
    PF_SMOOTH_B32, PF_SMOOTH_R32, PF_RESID_RESTRICT32, PF_PROLONG32, PF_LEVEL_RESID32, PF_COARSE32,
    PF_GALERKIN32, PF_WEIGHTS32, PF_ILU_DIAG32, PF_COARSE_SETUP32, PF_KRY_SPMV_DOT32, PF_KRY_UPDATE32,
    PF_KRY_DOT32, PF_KRY_INIT32, PF_REFINE, PF_CONVERT32,
    PF_SEED,                     // learned sweep predictor (features + MLP + seed write)
    PF_METAL,                    // metal-contact exchange (per column node)
    PF_PERSIST, PF_PERSIST32,    // persistent solve launches, FP64 and FP32 (bytes booked per launch)
    PF_NPROF
};
// kernel class of the FP32 twin of an FP64 linear-algebra class
int pf_f32(int id);
template <class T> inline int pf(int id) { return sizeof(T) == 4 ? pf_f32(id) : id; }

// algorithmic bytes per node of each kernel class (FP64 arrays; see the kernel files)
extern const double kProfBytesPerNode[PF_NPROF];
extern const char *kProfName[PF_NPROF];

extern bool g_prof_on;
extern std::atomic<unsigned long long> g_launches;     // all threads
extern thread_local unsigned long long t_launches;     // this thread
void prof_begin(int id, cudaStream_t st);
void prof_end(int id, cudaStream_t st, double nodes);
// book `bytes` algorithmic bytes for the last timed launch of class `id` (classes whose
// bytes are known only after the launch, kProfBytesPerNode 1)
void prof_set_last(int id, double bytes);
void prof_collect();
void prof_reset();
void prof_read(int id, double *ms, double *count, double *bytes);

}  // namespace ss

namespace ss {
extern bool g_pdl;   // programmatic dependent launch of the linear-algebra kernels (SEMISIM_B200_PDL=0: off)
// launch with the programmatic-stream-serialization attribute: the kernel may be
// scheduled while the previous kernel of the stream still runs, and waits in pdl_entry()
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = g_pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, static_cast<Args &&>(args)...);
}
}  // namespace ss

#define SS_LAUNCH_PDL(ID, NODES, KERN, GRID, BLOCK, ST, ...)            \
    do {                                                                \
        ss::g_launches++;                                               \
        ss::t_launches++;                                               \
        if (ss::g_prof_on) ss::prof_begin((ID), (ST));                  \
        ss::launch_pdl(KERN, (GRID), (BLOCK), (ST), __VA_ARGS__);       \
        if (ss::g_prof_on) ss::prof_end((ID), (ST), (double)(NODES));   \
    } while (0)

#define SS_LAUNCH(ID, NODES, KERN, GRID, BLOCK, ST, ...)                \
    do {                                                                \
        ss::g_launches++;                                               \
        ss::t_launches++;                                               \
        if (ss::g_prof_on) ss::prof_begin((ID), (ST));                  \
        KERN<<<(GRID), (BLOCK), 0, (ST)>>>(__VA_ARGS__);                \
        if (ss::g_prof_on) ss::prof_end((ID), (ST), (double)(NODES));   \
    } while (0)
