// Per-node operations of the aggregation multigrid of general (graph) meshes, shared by
// its per-launch kernels (graph_mg.cu) and the persistent graph solves (graph_persist.cu).
// ELL layout: slot q of node k at q * N + k (neighbour -1 past the degree).
#pragma once
#include "device_common.cuh"

namespace ss {

// one node of a colour of the D-ILU(0) solve: forward (dir 0) y_i = (r_i - sum over earlier
// colours a_ij y_j) / D_i, backward (dir 1) z_i = y_i - sum over later colours a_ij z_j / D_i
// (gilu_apply, semiconductor_3d.c:2563-2593); r may be z
__device__ __forceinline__ void gilu_apply_node(const GLev &v, int i, int dir, const double *r, double *z) {
    const int ci = v.color[i];
    double s = 0.0;
    for (int q = 0; q < v.D; q++) {
        const size_t e = (size_t)q * v.N + i;
        const int j = v.col[e];
        if (j < 0) continue;
        const int cj = v.color[j];
        if (dir == 0 ? cj < ci : cj > ci) s += v.val[e] * z[j];
    }
    z[i] = dir == 0 ? (r[i] - s) * v.dil[i] : z[i] - s * v.dil[i];
}

// (A x)_k of a level (gmatvec_L, semiconductor_3d.c:2553-2561)
__device__ __forceinline__ double gmatvec_row(const GLev &v, const double *x, int k) {
    double s = v.diag[k] * x[k];
    for (int q = 0; q < v.D; q++) {
        const size_t e = (size_t)q * v.N + k;
        const int j = v.col[e];
        if (j >= 0) s += v.val[e] * x[j];
    }
    return s;
}

}  // namespace ss
