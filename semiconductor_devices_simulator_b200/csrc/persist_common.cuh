// Grid-wide barrier and reduction of the persistent (cooperative, one launch per linear
// solve) kernels of the tensor and graph solve paths.
//
// Barrier: every block arrives (release), thread 0 of each block waits for all arrivals
// (acquire).  Every wait is bounded: after the launch's limit a block sets the error word
// and leaves, every other block leaves at its next wait, and the host, which reads the
// error word after the launch, repeats the solve on the per-pass path.
//
// Reduction: each block writes its partial record, and after the barrier every block sums
// all records in block order, so every block holds bit-identical totals and takes the same
// decisions with no extra barrier.  Two alternating partial buffers keep a reduction from
// overwriting partials another block may still be reading.
#pragma once
#include <cooperative_groups.h>

#include "device_common.cuh"

namespace ss {

#ifndef PG_TPB_SET
#define PG_TPB_SET 1024
#endif
constexpr int PG_TPB = PG_TPB_SET;
constexpr unsigned long long PG_WAIT_NS = 2000000000ull;    // longest barrier wait of a solve (2 s)

__device__ __forceinline__ unsigned long long pg_clock() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned pg_ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// per-block state of a persistent launch
struct PS {
    PGrid *g;
    unsigned target;   // arrivals the next barrier waits for
    int rb;            // reduction buffer of the next reduction
    int tid, nth;      // thread index in the grid, threads in the grid
    unsigned long long wait_ns;   // longest wait at one barrier
    unsigned long long *trace;    // barrier timeline (null: off): per barrier first arrival,
    int ntrace;                   //   last arrival, release seen by block 0 (globaltimer ns)
    int mode;                     // barrier form: 0 fences around the arrival and the wait,
                                  //   1 release-add / acquire-load
    int onecl;                    // 1: the whole grid is one thread-block cluster, whose
                                  //   hardware barrier replaces the grid barrier
};

// Grid-wide barrier: every block arrives (release), the block waits until every block
// has arrived (acquire), then proceeds.  Returns false when the launch is being abandoned.
// Forms (PS::mode): 0 - thread 0 fences, adds and polls; 1 - thread 0 adds with release
// semantics and polls with acquire loads (no separate fences).  The block barriers before
// and after order the other threads' accesses with thread 0's.
__device__ __forceinline__ void pg_red_release(unsigned *p) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(p) : "memory");
}
// poll until the arrivals reach the target; 1 released, 0 abandoned (error word or time)
__device__ __forceinline__ int pg_poll(PS &s) {
    unsigned long long t0 = 0;
    unsigned it = 0;
    while ((int)(pg_ld_acquire(&s.g->count) - s.target) < 0) {
        if ((++it & 255u) == 0) {
            if (*(volatile unsigned *)&s.g->err) return 0;
            const unsigned long long t = pg_clock();
            if (!t0) t0 = t;
            else if (t - t0 > s.wait_ns) { atomicExch(&s.g->err, 1u); return 0; }
        }
    }
    return 1;
}
__device__ __forceinline__ bool pg_sync(PS &s) {
    __shared__ int s_ok;
    if (s.onecl) {                                 // one cluster: barrier.cluster (release / acquire)
        cooperative_groups::this_cluster().sync();
        return true;
    }
    __syncthreads();
    s.target += gridDim.x;
    const int bn = (int)(s.target / gridDim.x) - 1;          // this barrier's number in the launch
    if (threadIdx.x == 0) {
        if (s.trace && bn < s.ntrace) {
            const unsigned long long t = pg_clock();
            atomicMin(s.trace + 3 * bn, t);
            atomicMax(s.trace + 3 * bn + 1, t);
        }
        int ok;
        if (s.mode == 0) {
            __threadfence();
            atomicAdd(&s.g->count, 1u);
            ok = pg_poll(s);
            __threadfence();
        } else {
            pg_red_release(&s.g->count);
            ok = pg_poll(s);
        }
        s_ok = ok;
        if (s.trace && bn < s.ntrace && blockIdx.x == 0) s.trace[3 * bn + 2] = pg_clock();
    }
    __syncthreads();
    return s_ok != 0;
}

// Sum NV (<= 4) values over the grid; every block returns the same totals in every thread.
template <int NV>
__device__ __forceinline__ bool pg_sum(PS &s, double (&v)[NV]) {
    __shared__ double tot[4];
    block_sum<NV>(v);
    double *buf = s.g->red[s.rb];
    s.rb ^= 1;
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) buf[blockIdx.x * 4 + q] = v[q];
    if (!pg_sync(s)) return false;
    if (threadIdx.x < 32) {
        double a[NV];
#pragma unroll
        for (int q = 0; q < NV; q++) a[q] = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += 32)
#pragma unroll
            for (int q = 0; q < NV; q++) a[q] += __ldcg(buf + b * 4 + q);
        warp_sum<NV>(a);
        if (threadIdx.x == 0)
#pragma unroll
            for (int q = 0; q < NV; q++) tot[q] = a[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = tot[q];
    return true;
}


}  // namespace ss
