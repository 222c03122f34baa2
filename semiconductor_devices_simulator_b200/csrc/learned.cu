// Learned sweep predictor: a per-node MLP that corrects the sweep's linear extrapolation
// x_lin = x1 + s (x1 - x0) of (psi, phi_n, phi_p) towards the next bias point's solution.
//
//   input  48 features of node k (stencil differences of the last step, local carrier
//          levels, doping, kind, the bias step), BF16
//   layers 48 -> 128 -> 128 -> 128 -> 3, SiLU, BF16 weights and activations, FP32
//          accumulation on the tensor cores (mma.sync m16n8k16 BF16 -> FP32)
//   output (psi, phi_n, phi_p)_next - x_lin in units of the thermal voltage
//
// It only seeds the Gummel loop, which converges to the same residual tolerance; the
// solver falls back to the linear guess when a seeded step fails.  The network is
// trained on solutions the solver itself generates: the training kernels here (forward
// with saved activations, backward through the activations, weight gradients summed
// over the batch, Adam) are driven from the host through b200m_* entry points that take
// device pointers.  The reference has no learned component.
//
// One warp computes 16 nodes through all four layers: the FP32 accumulators of a layer
// are, after bias and SiLU, exactly the BF16 A fragments of the next layer's mma
// (columns 16j..16j+15 = accumulator tiles 2j and 2j+1), so activations never leave the
// registers.  Weights sit in shared memory with rows padded by 8 elements so the B
// fragment loads of a warp hit 32 distinct banks.
#include <cuda_bf16.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "prof.h"
#include "solver_ctx.h"

namespace ss {

constexpr int MI = 48, MH = 128, MO = 8, MOUT = 3;
// FP32 parameter vector: W1 [MH][MI], b1, W2 [MH][MH], b2, W3 [MH][MH], b3, W4 [MO][MH], b4
constexpr int OW1 = 0, OB1 = OW1 + MH * MI, OW2 = OB1 + MH, OB2 = OW2 + MH * MH, OW3 = OB2 + MH,
              OB3 = OW3 + MH * MH, OW4 = OB3 + MH, OB4 = OW4 + MO * MH, NPARAM = OB4 + MO;
// BF16 weight pack (same matrices, same order, no biases)
constexpr int QW1 = 0, QW2 = QW1 + MH * MI, QW3 = QW2 + MH * MH, QW4 = QW3 + MH * MH, NWB = QW4 + MO * MH;
constexpr int NBIAS = 3 * MH + MO;
// shared-memory row pitches (elements)
constexpr int P1 = MI + 8, PH = MH + 8, PT4 = MO + 8;

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t ld32(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }
// SiLU and its derivative with the fast exponential and division intrinsics (relative
// error ~1e-6, far below the BF16 rounding of the activations they feed)
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = __fdividef(1.f, 1.f + __expf(-z));
    return s * (1.f + z * (1.f - s));
}

// ------------------------------------------------------------------ features
// Features of node k from the last two solutions x1 (now) and x0 (one step back), the
// extrapolation ratio s and the new step's contact voltage changes dv (4, volts):
//   0-20   (x1 - x0) / VT of psi, phi_n, phi_p at k and its 6 neighbours
//          (self, x-, x+, y-, y+, z-, z+; a missing neighbour repeats k)
//   21-34  (psi - phi_n) / 40 VT and (phi_p - psi) / 40 VT of x1 at the same 7 nodes
//   35     s;  36-39 dv / 10 VT;  40 asinh(net doping / 1e22 m^-3) / 10
//   41     semiconductor node;  42 contact node;  43 1;  44-47 0
struct SeedIn {
    const double *x1[3], *x0[3];
    float s, dv[4];
};
__device__ __forceinline__ void node_features(const DevP &P, const SeedIn &in, int k, float *f) {
    const Node a = unidx(k, P.Nx, P.Ny);
    const int NxNy = P.Nx * P.Ny;
    int nb[7];
    nb[0] = k;
    nb[1] = a.i > 0 ? k - 1 : k;
    nb[2] = a.i < P.Nx - 1 ? k + 1 : k;
    nb[3] = a.j > 0 ? k - P.Nx : k;
    nb[4] = a.j < P.Ny - 1 ? k + P.Nx : k;
    nb[5] = a.l > 0 ? k - NxNy : k;
    nb[6] = a.l < P.Nz - 1 ? k + NxNy : k;
    const double iv = 1.0 / P.VTref, iv40 = iv / 40.0;
#pragma unroll
    for (int q = 0; q < 7; q++) {
        const int m = nb[q];
        const double p1 = in.x1[0][m], n1 = in.x1[1][m], h1 = in.x1[2][m];
        f[q] = (float)((p1 - in.x0[0][m]) * iv);
        f[7 + q] = (float)((n1 - in.x0[1][m]) * iv);
        f[14 + q] = (float)((h1 - in.x0[2][m]) * iv);
        f[21 + q] = (float)((p1 - n1) * iv40);
        f[28 + q] = (float)((h1 - p1) * iv40);
    }
    f[35] = in.s;
#pragma unroll
    for (int q = 0; q < 4; q++) f[36 + q] = (float)(in.dv[q] * iv * 0.1);
    const uint32_t fl = P.flags[k];
    f[40] = (float)(asinh((P.Nd[k] - P.Na[k]) * 1e-22) * 0.1);
    f[41] = fl_kind(fl) == K_SEMI ? 1.f : 0.f;
    f[42] = fl_con(fl) ? 1.f : 0.f;
    f[43] = 1.f;
#pragma unroll
    for (int q = 44; q < MI; q++) f[q] = 0.f;
}

__global__ void k_seed_features(const DevP *__restrict__ Ps, SeedIn in, bf16 *X) {
    const DevP &P = Ps[blockIdx.y];
    float f[MI];
    SS_GRID_LOOP(k, P.N) {
        node_features(P, in, k, f);
#pragma unroll
        for (int q = 0; q < MI; q += 2)
            *reinterpret_cast<__nv_bfloat162 *>(X + (size_t)k * MI + q) = __floats2bfloat162_rn(f[q], f[q + 1]);
    }
}

// ------------------------------------------------------------------ shared weights
struct MlpSmem {
    bf16 W1[MH * P1], W2[MH * PH], W3[MH * PH], W4[MO * PH];
    float b1[MH], b2[MH], b3[MH], b4[MO];
};
__device__ __forceinline__ void load_weights(MlpSmem &s, const bf16 *Wb, const float *bias) {
    for (int e = threadIdx.x; e < MH * MI; e += blockDim.x) s.W1[(e / MI) * P1 + e % MI] = Wb[QW1 + e];
    for (int e = threadIdx.x; e < MH * MH; e += blockDim.x) {
        s.W2[(e / MH) * PH + e % MH] = Wb[QW2 + e];
        s.W3[(e / MH) * PH + e % MH] = Wb[QW3 + e];
    }
    for (int e = threadIdx.x; e < MO * MH; e += blockDim.x) s.W4[(e / MH) * PH + e % MH] = Wb[QW4 + e];
    for (int e = threadIdx.x; e < MH; e += blockDim.x) {
        s.b1[e] = bias[0 * MH + e]; s.b2[e] = bias[1 * MH + e]; s.b3[e] = bias[2 * MH + e];
    }
    for (int e = threadIdx.x; e < MO; e += blockDim.x) s.b4[e] = bias[3 * MH + e];
}

// one hidden layer of a warp's 16 rows: acc = A W^T + b (16 x 128), A given as BF16
// fragments of KS k-slices
template <int KS, int PW>
__device__ __forceinline__ void layer_mma(float (&acc)[16][4], const uint32_t (&a)[KS][4], const bf16 *W,
                                          const float *b) {
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
#pragma unroll
    for (int nt = 0; nt < 16; nt++) {
        const float b0 = b[8 * nt + 2 * t], b1 = b[8 * nt + 2 * t + 1];
        acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
    }
#pragma unroll
    for (int ks = 0; ks < KS; ks++)
#pragma unroll
        for (int nt = 0; nt < 16; nt++) {
            const bf16 *w = W + (8 * nt + g) * PW + 16 * ks + 2 * t;
            mma16816(acc[nt], a[ks], ld32(w), ld32(w + 8));
        }
}
// SiLU of the accumulators repacked as the next layer's A fragments
__device__ __forceinline__ void act_pack(const float (&acc)[16][4], uint32_t (&a)[8][4]) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
        a[j][0] = pack2(silu(acc[2 * j][0]), silu(acc[2 * j][1]));
        a[j][1] = pack2(silu(acc[2 * j][2]), silu(acc[2 * j][3]));
        a[j][2] = pack2(silu(acc[2 * j + 1][0]), silu(acc[2 * j + 1][1]));
        a[j][3] = pack2(silu(acc[2 * j + 1][2]), silu(acc[2 * j + 1][3]));
    }
}
// A fragments of a 16 x MI feature tile in shared memory (row pitch P1)
__device__ __forceinline__ void feat_frags(const bf16 *Xs, uint32_t (&a)[3][4]) {
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
#pragma unroll
    for (int ks = 0; ks < 3; ks++) {
        const bf16 *r0 = Xs + g * P1 + 16 * ks + 2 * t, *r1 = r0 + 8 * P1;
        a[ks][0] = ld32(r0); a[ks][1] = ld32(r1); a[ks][2] = ld32(r0 + 8); a[ks][3] = ld32(r1 + 8);
    }
}
// output layer: 16 x 8 (channels 0-2 used)
__device__ __forceinline__ void out_mma(float (&o)[4], const uint32_t (&a)[8][4], const bf16 *W4, const float *b4) {
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    o[0] = b4[2 * t]; o[1] = b4[2 * t + 1]; o[2] = o[0]; o[3] = o[1];
#pragma unroll
    for (int ks = 0; ks < 8; ks++) {
        const bf16 *w = W4 + g * PH + 16 * ks + 2 * t;
        mma16816(o, a[ks], ld32(w), ld32(w + 8));
    }
}

// ------------------------------------------------------------------ seed
// x_next = x1 + s (x1 - x0) + VT * MLP(X) for psi, phi_n, phi_p of every node; X the
// node features (k_seed_features), 128 nodes per CTA pass (8 warps x 16 rows), x1 = h1 and
// x0 = e2 of the instance
constexpr int SEED_TPB = 128, SEED_ROWS = 64;            // training kernels
constexpr int INF_TPB = 256, INF_ROWS = 128;             // inference
__global__ void __launch_bounds__(INF_TPB) k_mlp_seed(const DevP *__restrict__ Ps, const bf16 *__restrict__ Wb,
                                                       const float *__restrict__ bias, SeedIn in,
                                                       const bf16 *__restrict__ X) {
    const DevP &P = Ps[blockIdx.y];
    extern __shared__ __align__(16) unsigned char smraw[];
    MlpSmem &s = *reinterpret_cast<MlpSmem *>(smraw);
    bf16 *Xs = reinterpret_cast<bf16 *>(smraw + sizeof(MlpSmem));
    load_weights(s, Wb, bias);
    const int w = threadIdx.x >> 5, g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    const double VT = P.VTref;
    const int N = P.N;
    for (int base = blockIdx.x * INF_ROWS; base < N; base += gridDim.x * INF_ROWS) {
        __syncthreads();                           // weights staged / previous tile consumed
        for (int e = threadIdx.x; e < INF_ROWS * MI / 2; e += blockDim.x) {
            const int r = e / (MI / 2), q = 2 * (e % (MI / 2));
            const int row = base + r;
            const uint32_t v = row < N ? ld32(X + (size_t)row * MI + q) : 0u;
            *reinterpret_cast<uint32_t *>(Xs + r * P1 + q) = v;
        }
        __syncthreads();
        uint32_t a0[3][4], a[8][4];
        float acc[16][4];
        feat_frags(Xs + 16 * w * P1, a0);
        layer_mma<3, P1>(acc, a0, s.W1, s.b1);
        act_pack(acc, a);
        layer_mma<8, PH>(acc, a, s.W2, s.b2);
        act_pack(acc, a);
        layer_mma<8, PH>(acc, a, s.W3, s.b3);
        act_pack(acc, a);
        float o[4];
        out_mma(o, a, s.W4, s.b4);
        if (t < 2) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int k = base + 16 * w + g + 8 * h;
                if (k >= N) continue;
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int c = 2 * t + e;
                    if (c >= MOUT) continue;
                    // channel pointers by select (no dynamically indexed arrays: no local memory)
                    const double *X1 = c == 0 ? in.x1[0] : (c == 1 ? in.x1[1] : in.x1[2]);
                    const double *X0 = c == 0 ? in.x0[0] : (c == 1 ? in.x0[1] : in.x0[2]);
                    double *D = c == 0 ? P.phi : (c == 1 ? P.phin : P.phip);
                    const double x1 = X1[k], x0 = X0[k];
                    D[k] = x1 + (double)in.s * (x1 - x0) + VT * (double)o[2 * h + e];
                }
            }
        }
    }
}

// ------------------------------------------------------------------ training kernels
// forward of a batch: X [B][MI] -> Y [B][MO]; saves Z_l (FP32 pre-activations) and H_l
// (BF16 activations) of the three hidden layers, [B][MH] each
__global__ void __launch_bounds__(SEED_TPB) k_mlp_train_fwd(const bf16 *__restrict__ X, int B, const bf16 *__restrict__ Wb,
                                                             const float *__restrict__ bias, float *Y, float *Z, bf16 *H) {
    extern __shared__ __align__(16) unsigned char smraw[];
    MlpSmem &s = *reinterpret_cast<MlpSmem *>(smraw);
    bf16 *Xs = reinterpret_cast<bf16 *>(smraw + sizeof(MlpSmem));
    load_weights(s, Wb, bias);
    const int w = threadIdx.x >> 5, g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    for (int base = blockIdx.x * SEED_ROWS; base < B; base += gridDim.x * SEED_ROWS) {
        __syncthreads();
        for (int e = threadIdx.x; e < SEED_ROWS * MI / 2; e += blockDim.x) {
            const int r = e / (MI / 2), q = 2 * (e % (MI / 2));
            const int row = base + r;
            const uint32_t v = row < B ? ld32(X + (size_t)row * MI + q) : 0u;
            *reinterpret_cast<uint32_t *>(Xs + r * P1 + q) = v;
        }
        __syncthreads();
        uint32_t a0[3][4], a[8][4];
        float acc[16][4];
        feat_frags(Xs + 16 * w * P1, a0);
        const int r0 = base + 16 * w + g, r1 = r0 + 8;
#pragma unroll
        for (int L = 0; L < 3; L++) {
            if (L == 0) layer_mma<3, P1>(acc, a0, s.W1, s.b1);
            else if (L == 1) layer_mma<8, PH>(acc, a, s.W2, s.b2);
            else layer_mma<8, PH>(acc, a, s.W3, s.b3);
            act_pack(acc, a);
            float *ZL = Z + (size_t)L * B * MH;
            bf16 *HL = H + (size_t)L * B * MH;
#pragma unroll
            for (int nt = 0; nt < 16; nt++) {
                const int col = 8 * nt + 2 * t;
                if (r0 < B) {
                    *reinterpret_cast<float2 *>(ZL + (size_t)r0 * MH + col) = make_float2(acc[nt][0], acc[nt][1]);
                    *reinterpret_cast<uint32_t *>(HL + (size_t)r0 * MH + col) = a[nt >> 1][(nt & 1) * 2];
                }
                if (r1 < B) {
                    *reinterpret_cast<float2 *>(ZL + (size_t)r1 * MH + col) = make_float2(acc[nt][2], acc[nt][3]);
                    *reinterpret_cast<uint32_t *>(HL + (size_t)r1 * MH + col) = a[nt >> 1][(nt & 1) * 2 + 1];
                }
            }
        }
        float o[4];
        out_mma(o, a, s.W4, s.b4);
        if (r0 < B) *reinterpret_cast<float2 *>(Y + (size_t)r0 * MO + 2 * t) = make_float2(o[0], o[1]);
        if (r1 < B) *reinterpret_cast<float2 *>(Y + (size_t)r1 * MO + 2 * t) = make_float2(o[2], o[3]);
    }
}

// backward through the activations: dY = 2 (Y - T) / (3 B) on the 3 channels (loss =
// mean squared error, accumulated into *loss), then dZ_3, dZ_2, dZ_1 (BF16 [B][MH]) with
// dH_l = dZ_{l+1} W_{l+1} and dZ_l = dH_l * SiLU'(Z_l); dY is stored BF16 [B][MO]
struct MlpSmemT {
    bf16 W2T[MH * PH], W3T[MH * PH], W4T[MH * PT4];
};
__global__ void __launch_bounds__(SEED_TPB) k_mlp_train_bwd(int B, const bf16 *__restrict__ Wb, const float *__restrict__ Y,
                                                             const float *__restrict__ T, const float *__restrict__ Z,
                                                             bf16 *dZ, bf16 *dY, float *loss) {
    extern __shared__ __align__(16) unsigned char smraw[];
    MlpSmemT &s = *reinterpret_cast<MlpSmemT *>(smraw);
    for (int e = threadIdx.x; e < MH * MH; e += blockDim.x) {       // transposed copies: [in][out]
        const int o = e / MH, i = e % MH;
        s.W2T[i * PH + o] = Wb[QW2 + e];
        s.W3T[i * PH + o] = Wb[QW3 + e];
    }
    for (int e = threadIdx.x; e < MH * PT4; e += blockDim.x) s.W4T[e] = __float2bfloat16(0.f);
    __syncthreads();
    for (int e = threadIdx.x; e < MO * MH; e += blockDim.x) {
        const int o = e / MH, i = e % MH;
        s.W4T[i * PT4 + o] = Wb[QW4 + e];
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    const float sc = 2.f / (3.f * (float)B);
    float lsum = 0.f;
    for (int base = blockIdx.x * SEED_ROWS; base < B; base += gridDim.x * SEED_ROWS) {
        const int r0 = base + 16 * w + g, r1 = r0 + 8;
        // dY in the accumulator layout of a 16 x 8 tile: rows r0 / r1, channels 2t, 2t+1
        float dy[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int r = h ? r1 : r0;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int c = 2 * t + e;
                if (r < B && c < MOUT) {
                    const float d = Y[(size_t)r * MO + c] - T[(size_t)r * MOUT + c];
                    lsum += d * d;
                    dy[2 * h + e] = sc * d;
                }
            }
        }
        const uint32_t y0 = pack2(dy[0], dy[1]), y1 = pack2(dy[2], dy[3]);
        if (r0 < B) *reinterpret_cast<uint32_t *>(dY + (size_t)r0 * MO + 2 * t) = y0;
        if (r1 < B) *reinterpret_cast<uint32_t *>(dY + (size_t)r1 * MO + 2 * t) = y1;
        // dH3 = dY W4 (K = 8 padded to 16)
        uint32_t a[8][4];
        float acc[16][4];
        {
            const uint32_t ay[4] = {y0, y1, 0u, 0u};
#pragma unroll
            for (int nt = 0; nt < 16; nt++) {
                acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
                const bf16 *wt = s.W4T + (8 * nt + g) * PT4 + 2 * t;
                mma16816(acc[nt], ay, ld32(wt), 0u);
            }
        }
#pragma unroll
        for (int L = 2; L >= 0; L--) {
            // dZ_L = dH_L * SiLU'(Z_L), stored and repacked as A fragments
            const float *ZL = Z + (size_t)L * B * MH;
            bf16 *dZL = dZ + (size_t)L * B * MH;
#pragma unroll
            for (int nt = 0; nt < 16; nt++) {
                const int col = 8 * nt + 2 * t;
                float2 z0 = make_float2(0.f, 0.f), z1 = z0;
                if (r0 < B) z0 = *reinterpret_cast<const float2 *>(ZL + (size_t)r0 * MH + col);
                if (r1 < B) z1 = *reinterpret_cast<const float2 *>(ZL + (size_t)r1 * MH + col);
                acc[nt][0] *= dsilu(z0.x); acc[nt][1] *= dsilu(z0.y);
                acc[nt][2] *= dsilu(z1.x); acc[nt][3] *= dsilu(z1.y);
                const uint32_t p0 = pack2(acc[nt][0], acc[nt][1]), p1 = pack2(acc[nt][2], acc[nt][3]);
                a[nt >> 1][(nt & 1) * 2] = p0;
                a[nt >> 1][(nt & 1) * 2 + 1] = p1;
                if (r0 < B) *reinterpret_cast<uint32_t *>(dZL + (size_t)r0 * MH + col) = p0;
                if (r1 < B) *reinterpret_cast<uint32_t *>(dZL + (size_t)r1 * MH + col) = p1;
            }
            if (L == 0) break;
            // dH_{L-1} = dZ_L W_L  (B operand: W_L^T, rows = input index)
            const bf16 *WT = L == 2 ? s.W3T : s.W2T;
#pragma unroll
            for (int nt = 0; nt < 16; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
            for (int ks = 0; ks < 8; ks++)
#pragma unroll
                for (int nt = 0; nt < 16; nt++) {
                    const bf16 *wt = WT + (8 * nt + g) * PH + 16 * ks + 2 * t;
                    mma16816(acc[nt], a[ks], ld32(wt), ld32(wt + 8));
                }
        }
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, lsum / (3.f * (float)B));
}

// weight and bias gradients of one layer: dW[o][i] += sum_b dZ[b][o] H[b][i],
// db[o] += sum_b dZ[b][o].  dZ [B][OUTP] BF16 (the first OUT columns used), H [B][IN]
// BF16.  8 warps, warp w owns output rows 16w..16w+15; 64 batch rows staged per pass,
// both operands read transposed from shared memory by ldmatrix.trans.
template <int OUT, int OUTP, int IN>
__global__ void __launch_bounds__(256) k_mlp_wgrad(const bf16 *__restrict__ dZ, const bf16 *__restrict__ H, int B,
                                                    float *dW, float *db) {
    constexpr int ZC = OUTP < 16 ? 16 : OUTP, PZ = ZC + 8, PHI = IN + 8, NT = IN / 8, MT = (OUT + 15) / 16;
    __shared__ __align__(16) bf16 Zs[64 * PZ];
    __shared__ __align__(16) bf16 Hs[64 * PHI];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
    float bsum = 0.f;
    for (int base = blockIdx.x * 64; base < B; base += gridDim.x * 64) {
        __syncthreads();
        for (int e = threadIdx.x; e < 64 * ZC; e += blockDim.x) {
            const int r = e / ZC, c = e % ZC;
            Zs[r * PZ + c] = (base + r < B && c < OUTP) ? dZ[(size_t)(base + r) * OUTP + c] : __float2bfloat16(0.f);
        }
        for (int e = threadIdx.x; e < 64 * IN; e += blockDim.x) {
            const int r = e / IN, c = e % IN;
            Hs[r * PHI + c] = base + r < B ? H[(size_t)(base + r) * IN + c] : __float2bfloat16(0.f);
        }
        __syncthreads();
        if (threadIdx.x < OUT)
            for (int r = 0; r < 64; r++) bsum += __bfloat162float(Zs[r * PZ + threadIdx.x]);
        if (w < MT) {
            const int m0 = 16 * w;
#pragma unroll
            for (int ks = 0; ks < 4; ks++) {
                const int k0 = 16 * ks;
                uint32_t a[4];
                {
                    const int mi = lane >> 3, r = lane & 7;
                    const bf16 *p = Zs + (k0 + r + (mi >> 1) * 8) * PZ + m0 + (mi & 1) * 8;
                    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(p);
                    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                                 : "r"(addr));
                }
#pragma unroll
                for (int nt = 0; nt < NT; nt++) {
                    uint32_t b0, b1;
                    const bf16 *p = Hs + (k0 + (lane & 15)) * PHI + 8 * nt;
                    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(p);
                    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                                 : "=r"(b0), "=r"(b1)
                                 : "r"(addr));
                    mma16816(acc[nt], a, b0, b1);
                }
            }
        }
    }
    if (threadIdx.x < OUT) atomicAdd(db + threadIdx.x, bsum);
    if (w < MT) {
        const int m0 = 16 * w;
#pragma unroll
        for (int nt = 0; nt < NT; nt++) {
            const int col = 8 * nt + 2 * t;
            if (m0 + g < OUT) {
                atomicAdd(dW + (m0 + g) * IN + col, acc[nt][0]);
                atomicAdd(dW + (m0 + g) * IN + col + 1, acc[nt][1]);
            }
            if (m0 + g + 8 < OUT) {
                atomicAdd(dW + (m0 + g + 8) * IN + col, acc[nt][2]);
                atomicAdd(dW + (m0 + g + 8) * IN + col + 1, acc[nt][3]);
            }
        }
    }
}

// Adam on the FP32 parameters with bias-corrected moments (c1 = 1 - b1^t, c2 = 1 - b2^t)
__global__ void k_mlp_adam(float *P, const float *G, float *M, float *V, int n, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
    SS_GRID_LOOP(i, n) {
        const float gr = G[i];
        const float m = b1 * M[i] + (1.f - b1) * gr, v = b2 * V[i] + (1.f - b2) * gr * gr;
        M[i] = m;
        V[i] = v;
        P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
}
// BF16 weight pack + bias vector [b1 | b2 | b3 | b4] of an FP32 parameter vector
__global__ void k_mlp_pack(const float *P, bf16 *Wb, float *bias) {
    SS_GRID_LOOP(i, NPARAM) {
        const float v = P[i];
        if (i < OB1) Wb[QW1 + i - OW1] = __float2bfloat16(v);
        else if (i < OW2) bias[i - OB1] = v;
        else if (i < OB2) Wb[QW2 + i - OW2] = __float2bfloat16(v);
        else if (i < OW3) bias[MH + i - OB2] = v;
        else if (i < OB3) Wb[QW3 + i - OW3] = __float2bfloat16(v);
        else if (i < OW4) bias[2 * MH + i - OB3] = v;
        else if (i < OB4) Wb[QW4 + i - OW4] = __float2bfloat16(v);
        else bias[3 * MH + i - OB4] = v;
    }
}

static size_t seed_smem() { return sizeof(MlpSmem) + (size_t)SEED_ROWS * P1 * sizeof(bf16); }
static size_t inf_smem() { return sizeof(MlpSmem) + (size_t)INF_ROWS * P1 * sizeof(bf16); }
static bool g_mlp_attr = false;
static void mlp_attrs() {
    if (g_mlp_attr) return;
    cudaFuncSetAttribute(k_mlp_seed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inf_smem());
    cudaFuncSetAttribute(k_mlp_train_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)seed_smem());
    cudaFuncSetAttribute(k_mlp_train_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmemT));
    g_mlp_attr = true;
}

// ------------------------------------------------------------------ solver side
int seed_available(const Inst &d) { return d.seed_on && d.g.seedw != nullptr && !d.unstr; }

// x = x1 + s (x1 - x0) + VT * MLP for the sweep predictor step (h1 = x1, e2 = x0): the
// features into the instance's feature buffer, then the network and the seed write
void launch_mlp_seed(Inst &d, double s, const double *dv) {
    mlp_attrs();
    Ctx c = make_ctx(d);
    SeedIn in;
    for (int a = 0; a < 3; a++) { in.x1[a] = d.g.h.h1[a]; in.x0[a] = d.g.h.e2[a]; }
    in.s = (float)s;
    for (int q = 0; q < 4; q++) in.dv[q] = (float)dv[q];
    bf16 *X = reinterpret_cast<bf16 *>(d.g.seedx);
    int nb = (int)((d.N + INF_ROWS - 1) / INF_ROWS);
    if (nb > 296) nb = 296;
    g_launches += 2;
    t_launches += 2;
    if (g_prof_on) prof_begin(PF_SEED, c.st);
    k_seed_features<<<dim3(c.nodes_blocks(), 1), TPB, 0, c.st>>>(c.dP, in, X);
    k_mlp_seed<<<dim3(nb, 1), INF_TPB, inf_smem(), c.st>>>(c.dP, (const bf16 *)d.g.seedw, (const float *)d.g.seedb,
                                                           in, X);
    if (g_prof_on) prof_end(PF_SEED, c.st, (double)d.N);
}

}  // namespace ss

using namespace ss;
extern Inst *b200_global_dev();

extern "C" {

// ---- public (additive) API of the learned seed, on the calling thread's instance
// load a trained model: NPARAM FP32 values (W1 [128][48], b1 [128], W2 [128][128], b2,
// W3 [128][128], b3, W4 [8][128] with rows 3-7 zero, b4 [8]) and enable the seed; the
// instance must have been set up by a solve (its device memory exists).  1 = done.
int api3b_seed_set_model(const float *params, int n) {
    Inst &d = *b200_global_dev();
    if (n != NPARAM || !params || !d.g.ready) return 0;
    Ctx c = make_ctx(d);
    if (!d.g.seedw) {                              // weights, biases, parameters, node features
        void *p = nullptr;
        const size_t wb = NWB * sizeof(bf16) + (NBIAS + NPARAM) * sizeof(float);
        const size_t xo = (wb + 255) & ~size_t(255);
        if (cudaMalloc(&p, xo + d.N * MI * sizeof(bf16)) != cudaSuccess) return 0;
        d.g.seedw = p;
        d.g.seedb = reinterpret_cast<float *>(reinterpret_cast<char *>(p) + NWB * sizeof(bf16));
        d.g.seedx = reinterpret_cast<char *>(p) + xo;
    }
    float *P = d.g.seedb + NBIAS;
    cudaMemcpyAsync(P, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice, c.st);
    k_mlp_pack<<<64, 256, 0, c.st>>>(P, (bf16 *)d.g.seedw, d.g.seedb);
    cudaStreamSynchronize(c.st);
    d.seed_on = 1;
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}
// 1: seed the sweep predictor with the loaded model, 0: linear guess only; returns the
// previous setting
int api3b_seed_enable(int on) {
    Inst &d = *b200_global_dev();
    const int old = d.seed_on;
    d.seed_on = on ? 1 : 0;
    return old;
}
// predictor steps seeded by the model, and seeded steps that failed and were redone from
// the linear guess, since the instance was created
void api3b_seed_stats(long long *used, long long *fallbacks) {
    Inst &d = *b200_global_dev();
    *used = d.seed_used;
    *fallbacks = d.seed_fallbacks;
}
int api3b_seed_nparam(void) { return NPARAM; }

// ---- training hooks (device pointers; `stream` a cudaStream_t, null = the instance's
// stream for the features, the legacy stream otherwise).  Fixed sizes: 48 features,
// hidden 128, output padded to 8.
// features of every node of the current instance from two solutions (device arrays)
int b200m_seed_features(const double *psi1, const double *phin1, const double *phip1, const double *psi0,
                        const double *phin0, const double *phip0, double s, const double *dv4, void *X, void *stream) {
    Inst &d = *b200_global_dev();
    if (!d.g.ready) return 0;
    Ctx c = make_ctx(d);
    SeedIn in;
    in.x1[0] = psi1; in.x1[1] = phin1; in.x1[2] = phip1;
    in.x0[0] = psi0; in.x0[1] = phin0; in.x0[2] = phip0;
    in.s = (float)s;
    for (int q = 0; q < 4; q++) in.dv[q] = dv4 ? (float)dv4[q] : 0.f;
    cudaStream_t st = stream ? (cudaStream_t)stream : c.st;
    k_seed_features<<<dim3(c.nodes_blocks(), 1), TPB, 0, st>>>(c.dP, in, (bf16 *)X);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}
// BF16 weight pack (NWB) and bias vector (3*128+8) of an FP32 parameter vector
int b200m_mlp_pack(const float *P, void *Wb, float *bias, void *stream) {
    k_mlp_pack<<<64, 256, 0, (cudaStream_t)stream>>>(P, (bf16 *)Wb, bias);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}
// forward of B rows: Y [B][8]; Z [3][B][128] FP32; H [3][B][128] BF16
int b200m_mlp_forward(const void *X, int B, const void *Wb, const float *bias, float *Y, float *Z, void *H,
                      void *stream) {
    mlp_attrs();
    int nb = (B + SEED_ROWS - 1) / SEED_ROWS;
    if (nb > 1184) nb = 1184;
    k_mlp_train_fwd<<<nb, SEED_TPB, seed_smem(), (cudaStream_t)stream>>>((const bf16 *)X, B, (const bf16 *)Wb, bias, Y,
                                                                          Z, (bf16 *)H);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}
// backward: gradients of loss = mean over B x 3 of (Y - T)^2 added into G (NPARAM FP32;
// zero it first), the loss added to *loss.  T [B][3]; scratch dZ [3][B][128] and dY [B][8]
// BF16.
int b200m_mlp_backward(const void *X, int B, const void *Wb, const float *Y, const float *T, const float *Z,
                       const void *H, void *dZ, void *dY, float *G, float *loss, void *stream) {
    mlp_attrs();
    cudaStream_t st = (cudaStream_t)stream;
    int nb = (B + SEED_ROWS - 1) / SEED_ROWS;
    if (nb > 1184) nb = 1184;
    k_mlp_train_bwd<<<nb, SEED_TPB, sizeof(MlpSmemT), st>>>(B, (const bf16 *)Wb, Y, T, Z, (bf16 *)dZ, (bf16 *)dY, loss);
    const bf16 *Hb = (const bf16 *)H, *dZb = (const bf16 *)dZ;
    const size_t L = (size_t)B * MH;
    int ng = (B + 63) / 64;
    if (ng > 296) ng = 296;
    k_mlp_wgrad<MH, MH, MI><<<ng, 256, 0, st>>>(dZb, (const bf16 *)X, B, G + OW1, G + OB1);
    k_mlp_wgrad<MH, MH, MH><<<ng, 256, 0, st>>>(dZb + L, Hb, B, G + OW2, G + OB2);
    k_mlp_wgrad<MH, MH, MH><<<ng, 256, 0, st>>>(dZb + 2 * L, Hb + L, B, G + OW3, G + OB3);
    k_mlp_wgrad<MOUT, MO, MH><<<ng, 256, 0, st>>>((const bf16 *)dY, Hb + 2 * L, B, G + OW4, G + OB4);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}
// one Adam step (t >= 1) on P with gradient G and moments M, V; then the BF16 pack and
// the bias vector
int b200m_mlp_adam(float *P, const float *G, float *M, float *V, float lr, int t, void *Wb, float *bias, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    k_mlp_adam<<<64, 256, 0, st>>>(P, G, M, V, NPARAM, lr, b1, b2, 1e-8f, c1, c2);
    k_mlp_pack<<<64, 256, 0, st>>>(P, (bf16 *)Wb, bias);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}
int b200m_mlp_sizes(int *nparam, int *nwb, int *nbias) {
    *nparam = NPARAM;
    *nwb = NWB;
    *nbias = NBIAS;
    return 1;
}

}  // extern "C"
