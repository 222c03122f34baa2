// Residual of a 7-point stencil system with its norm and rounding floor, for callers that
// cannot allocate device memory.
//
// Who needs it: a caller whose device memory belongs to another allocator (a framework's
// caching allocator with a fixed budget, where a library's own cudaMalloc would go around
// it), a caller on a latency-critical path where cudaMalloc / cudaFree are not acceptable
// (they can synchronise the whole device), or a caller that must not change the device's
// memory footprint at all after start-up.  Such a caller owns every input and output
// buffer; the only memory this entry point needs beyond them - the per-block partial sums
// of the two grid-wide reductions and the ticket counter of their last-block finish - is
// the file-scope device array below, which every GPU that loads the library holds (about
// 38 KB) until the process exits.
//
// The kernel is a variant of the BiCGSTAB start kernel of the solve path (k_bicg_init in
// kernels_la.cu): r = b - A x, ||r||_2 and the floor sqrt(sum_a (sum_b |A_ab x_b| + |b_a|)^2)
// the reference's BiCGSTAB stops against (semiconductor_3d.c:2244-2268), reading the
// caller's arrays instead of an instance's.
#include <cstdio>
#include <mutex>

#include "device_common.cuh"

namespace ss {

constexpr int NA_BLOCKS = 296;                  // 2 CTAs per SM of a B200
constexpr int NA_TPB = 256;
constexpr long long NA_MAX_NODES = 1LL << 30;   // largest system (int32 node indices)
constexpr int NA_MAX_DEVICES = 64;

struct NoAllocScratch {
    double part[NA_BLOCKS * RED_NV];            // per-block partial records
    double out[2];                              // ||r||, floor
    unsigned ticket[2];                         // last-block counter (must start at 0)
};
// the scratch of every call on this GPU: shared by all calls, keeps the last call's contents
static __device__ __align__(256) NoAllocScratch g_na_scratch;

__global__ void __launch_bounds__(NA_TPB) k_resid_floor_na(const double *__restrict__ A7, const double *__restrict__ x,
                                                           const double *__restrict__ b, double *__restrict__ r, int Nx,
                                                           int Ny, int Nz, NoAllocScratch *s) {
    const long long N = (long long)Nx * Ny * Nz;
    const double *A[7];
#pragma unroll
    for (int q = 0; q < 7; q++) A[q] = A7 + (size_t)q * (size_t)N;
    const int NxNy = Nx * Ny;
    double acc[2] = {0.0, 0.0};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < (int)N; k += gridDim.x * blockDim.x) {
        const Node a = unidx(k, Nx, Ny);
        double sum = A[0][k] * x[k], fl = fabs(A[0][k] * x[k]) + fabs(b[k]), t;
        if (a.i > 0) { t = A[1][k] * x[k - 1]; sum += t; fl += fabs(t); }
        if (a.i < Nx - 1) { t = A[2][k] * x[k + 1]; sum += t; fl += fabs(t); }
        if (a.j > 0) { t = A[3][k] * x[k - Nx]; sum += t; fl += fabs(t); }
        if (a.j < Ny - 1) { t = A[4][k] * x[k + Nx]; sum += t; fl += fabs(t); }
        if (a.l > 0) { t = A[5][k] * x[k - NxNy]; sum += t; fl += fabs(t); }
        if (a.l < Nz - 1) { t = A[6][k] * x[k + NxNy]; sum += t; fl += fabs(t); }
        const double rk = b[k] - sum;
        r[k] = rk;
        acc[0] += rk * rk;
        acc[1] += fl * fl;
    }
    if (grid_sum<2>(acc, s->part, s->ticket)) {
        s->out[0] = sqrt(acc[0]);
        s->out[1] = sqrt(acc[1]);
    }
}

namespace {
std::mutex g_na_mu;
NoAllocScratch *g_na_ptr[NA_MAX_DEVICES] = {nullptr};

// device address of the scratch on `dev` (current), looked up once per device
NoAllocScratch *scratch_on(int dev) {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (dev < 0 || dev >= NA_MAX_DEVICES) return nullptr;
    if (!g_na_ptr[dev]) {
        NoAllocScratch *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_na_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: cudaGetSymbolAddress failed on device %d: %s\n",
                         dev, cudaGetErrorString(e));
            return nullptr;
        }
        g_na_ptr[dev] = p;
    }
    return g_na_ptr[dev];
}

// the GPU that holds a caller buffer, or -1 when it is not device (or managed) memory
int device_of(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) return -1;
    return at.device;
}

// true when the byte ranges [a, a + na) and [b, b + nb) share a byte
bool overlap(const void *a, size_t na, const void *b, size_t nb) {
    const char *pa = static_cast<const char *>(a), *pb = static_cast<const char *>(b);
    return pa < pb + nb && pb < pa + na;
}

// makes `dev` current for the lifetime of the guard and restores the caller's device
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) { cudaGetLastError(); prev = -1; return; }
        ok = prev == dev || cudaSetDevice(dev) == cudaSuccess;
        if (!ok) cudaGetLastError();
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};
}  // namespace

}  // namespace ss

using namespace ss;

extern "C" {

// r = b - A x for the 7-point stencil A (7 arrays of N = Nx*Ny*Nz doubles one after the
// other: diagonal, x-, x+, y-, y+, z-, z+; node k = i + Nx*(j + Ny*l)) and norms[0] =
// ||r||_2, norms[1] = sqrt(sum_a (sum_b |A_ab x_b| + |b_a|)^2).  A7, x, b and r are device
// buffers the caller owns, all on one GPU; r must not overlap A7, x or b; norms is host
// memory.  Allocates nothing.  Returns 1 on success, 0 with a message on stderr (and no
// kernel launched) on a null pointer, a buffer that is not device memory or lies on
// another GPU than x, an r that overlaps an input, a size beyond 2^30 nodes; 0 also on
// a CUDA error.  The calling thread's current device is the same on return as before.
//
// The first call on a GPU looks up the scratch's device address (cudaGetSymbolAddress
// with that GPU current): make that first call before any stream capture.  All calls
// share the scratch and run on the default stream; calls that overlap on a GPU (from
// several host threads, or work another stream runs at the same time) race on it.
int api3b_stencil_residual_noalloc(const double *A7, const double *x, const double *b, int Nx, int Ny, int Nz,
                                   double *r, double *norms) {
    if (!A7 || !x || !b || !r || !norms) {
        std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: null pointer\n");
        return 0;
    }
    if (Nx < 1 || Ny < 1 || Nz < 1) {
        std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: bad shape %d x %d x %d\n", Nx, Ny, Nz);
        return 0;
    }
    const long long N = (long long)Nx * Ny * Nz;
    if (N > NA_MAX_NODES) {
        std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: %lld nodes exceeds the maximum of %lld\n", N,
                     NA_MAX_NODES);
        return 0;
    }
    // every caller buffer must be device memory of one GPU: a host or another GPU's
    // pointer would reach the kernel and fault there, which poisons the caller's context
    const char *names[4] = {"A7", "x", "b", "r"};
    const void *bufs[4] = {A7, x, b, r};
    int dev = -1;
    for (int q = 0; q < 4; q++) {
        const int d = device_of(bufs[q]);
        if (d < 0) {
            std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: %s is not device memory\n", names[q]);
            return 0;
        }
        if (q > 0 && d != dev) {
            std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: %s is on device %d, x on device %d\n",
                         names[q], d, dev);
            return 0;
        }
        dev = d;
    }
    // r is written while A7, x and b are read (at neighbouring nodes too): it must not
    // share memory with any of them
    const size_t vb = (size_t)N * sizeof(double);
    if (overlap(r, vb, x, vb) || overlap(r, vb, b, vb) || overlap(r, vb, A7, 7 * vb)) {
        std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: r overlaps an input (A7, x or b)\n");
        return 0;
    }
    DeviceGuard guard(dev);                     // the caller's current device comes back on return
    if (!guard.ok) {
        std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: cannot make device %d current\n", dev);
        return 0;
    }
    NoAllocScratch *s = scratch_on(dev);
    if (!s) return 0;
    if (cudaMemsetAsync(s->ticket, 0, sizeof s->ticket, 0) != cudaSuccess) return 0;   // the finish counter starts at 0
    k_resid_floor_na<<<NA_BLOCKS, NA_TPB, 0, 0>>>(A7, x, b, r, Nx, Ny, Nz, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: launch failed: %s\n", cudaGetErrorString(e));
        return 0;
    }
    double out[2] = {0.0, 0.0};
    e = cudaMemcpy(out, s->out, sizeof out, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "semisim-b200: stencil_residual_noalloc: %s\n", cudaGetErrorString(e));
        return 0;
    }
    norms[0] = out[0];
    norms[1] = out[1];
    return 1;
}

}  // extern "C"
