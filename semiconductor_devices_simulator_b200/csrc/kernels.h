// Host-side launchers of the device kernels.
#pragma once
#include <cuda_runtime.h>

#include "semisim.h"

namespace ss {

// instantiated device-looped Krylov graphs of one instance (kernels_la.cu)
// kinds: 0 PCG, 1 BiCGSTAB with the multigrid preconditioner, 2 BiCGSTAB with the
// smoother alone (all FP64); 3 FP32 PCG; 4 one FP64 refinement step around an FP32
// multigrid BiCGSTAB
constexpr int LOOP_KINDS = 5;
struct LoopGraphs {
    cudaGraphExec_t exec[LOOP_KINDS] = {};
    int kernels[LOOP_KINDS] = {};
    int failed = 0;
};

// Launch context: the device parameter records of `ninst` instances (dP), the host copy
// of instance 0's record (sizes), the stream.
struct Ctx {
    LoopGraphs *lg = nullptr;
    const DevP *dP = nullptr;
    DevP h{};
    int ninst = 1;
    int maxN = 0;
    cudaStream_t st = 0;
    int grid_cap = 148 * 8;     // blocks of the grid-stride node kernels (<= RED_MAX_BLOCKS)
    int rpb = 4;                // rows per block of the row-blocked level passes (block 32 x rpb)
    int zcap = 65535;           // most row blocks of one pass (more rows per thread beyond it)
    int rq = 1;                 // coarse rows per block of the residual + restriction pass
    int small_nodes = 0;        // levels at or below this size go to the small-level kernel (0: default)
    int pblocks = 0;            // blocks of the instance's persistent solves (0: the library-wide cap)
    int nodes_blocks() const;
};

// ---- physics (kernels_phys.cu)
void launch_poisson(const Ctx &c, const double *phi, int build, double *F);   // res[R_PNORM]
void launch_rebuild_np(const Ctx &c);
void launch_upd_mob(const Ctx &c);
void launch_coul_update(const Ctx &c);      // Coulomb interface charge (before the edge mobilities)
void launch_cont_assemble(const Ctx &c, int hole);
void launch_cont_update(const Ctx &c, int hole, double lo, double hi);          // res[R_DQ]
void launch_apply_bc(const Ctx &c, int have_solution);
void launch_init_eq(const Ctx &c);
void launch_clamp_qf(const Ctx &c, double lo, double hi);
void launch_currents(const Ctx &c);                                             // res[R_I..]
void launch_predictor(const Ctx &c);
void launch_dpsi(const Ctx &c);                                                 // res[R_DPSI]
void launch_upd_J(const Ctx &c);
void launch_mob_display(const Ctx &c);
void launch_node_val(const Ctx &c, int which, double *out);
void launch_ion_neutral(const Ctx &c);
void launch_ii_update(const Ctx &c);
void launch_ii_update_g(const Ctx &c);   // graph mesh (graph.cu)
void launch_region_seed(const Ctx &c, int c1, int *mark);
void launch_region_shift(const Ctx &c, int c1, double dV, const int *mark);
void launch_face_J(const Ctx &c, int ax, int carrier, double *out);
void launch_extrap(const Ctx &c, double r, int s1, int s2);     // history selectors 0 h1, 1 h2, 2 e2
void launch_extrap3(const Ctx &c, double w1, double w2, double w3);   // w1 h1 + w2 e2 + w3 e3
void launch_region_mark(const Ctx &c, int con1, int type, double dV, int *mark, int *changed);
void launch_floating_blocks(const Ctx &c, int hole, int *nblocks);

// ---- linear algebra (kernels_la.cu; drivers declared in solver_ctx.h)
int mg_levels(int Nx, int Ny, int Nz, int dims[][6]);

// ---- Anderson (kernels_aa.cu)
void launch_aa_step(const Ctx &c, int M, int have, int pos, int nfill, double *const *x, double *const *g,
                    int *nfill_out, int *ok);

}  // namespace ss
