// cmf_emu.cu -- device kernels of the learned per-cell emulator (no counterpart in the reference).
//
// A 4-layer MLP (input 32 -> 128 -> 128 -> 128 -> 1, ReLU) maps local state plus 8-hop upstream
// messages of every cell to its mean outflow over the next coupling step.  BF16 operands, FP32
// accumulation on the tensor cores (mma.sync m16n8k16 tiles for training and a register-chained
// fused inference; tcgen05 MMAs into tensor memory for the production inference), FP32 master
// weights updated by Adam.
// The rollout kernel turns predicted outflows into a mass-conserving storage update along the
// same upstream CSR the physics uses; the stage scheme then recomputes depths.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/cmf_gpu.h"

namespace {

thread_local std::string g_emu_err;

int emu_err(int code, const std::string &m) {
    g_emu_err = m;
    return code;
}

#define EMU_TRY(expr)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (expr);                                                              \
        if (e_ != cudaSuccess) return emu_err(CMF_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------------------------------
// GEMM: C[M,N] (+)= op(A)[M,K] * op(B)[K,N], bf16 in, fp32 accumulate.
// A is [M][K] (transA=0) or [K][M] (transA=1); B is [K][N] (transB=0) or [N][K] (transB=1); all
// row-major with leading dimensions lda/ldb.  Tiles of 64x64 per CTA (4 warps of 32x32), K steps
// of 32 staged in shared memory with both operands stored K-contiguous ([m][k], [n][k]), so the
// m16n8k16 fragments are plain 32-bit shared loads:
//   A frag  a0={A[g][2t..]}, a1={A[g+8][2t..]}, a2={A[g][2t+8..]}, a3={A[g+8][2t+8..]}
//   B frag  b0={B[k=2t..][n=g]}, b1={B[k=2t+8..][n=g]}          (g = lane/4, t = lane%4)
//   C frag  c0,c1 = C[g][2t..], c2,c3 = C[g+8][2t..]
// Epilogue: +bias[n], optional ReLU, store fp32 and/or bf16, or atomic-add fp32 (split-K).
// M, N must be multiples of 64 and K of 32 (callers pad); K may be split over gridDim.z.
// ------------------------------------------------------------------------------------------
constexpr int TM = 64, TN = 64, TK = 32, PAD = 8;

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const __nv_bfloat16 *__restrict__ A, int lda, int transA,
                                              const __nv_bfloat16 *__restrict__ B, int ldb, int transB,
                                              float *C, int ldc, __nv_bfloat16 *Cb, int ldcb, const float *__restrict__ bias,
                                              int relu, int accumulate, int k_per_split) {
    __shared__ __align__(16) __nv_bfloat16 As[TM][TK + PAD];
    __shared__ __align__(16) __nv_bfloat16 Bs[TN][TK + PAD];
    const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;   // row tiles on x: up to 2^31-1 of them
    const int kbeg = blockIdx.z * k_per_split, kend = min(K, kbeg + k_per_split);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, t = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;
    for (int k0 = kbeg; k0 < kend; k0 += TK) {
        // stage A tile as [m][k] and B tile as [n][k]
        for (int e = tid; e < TM * TK; e += blockDim.x) {
            const int mm = e / TK, kk = e % TK;
            const int gm = m0 + mm, gk = k0 + kk;
            As[mm][kk] = transA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            const int nn = mm;
            const int gn = n0 + nn;
            Bs[nn][kk] = transB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < TK; ks += 16) {
            uint32_t af[2][4], bfr[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int r = wm + i * 16 + g;
                af[i][0] = *reinterpret_cast<const uint32_t *>(&As[r][ks + 2 * t]);
                af[i][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][ks + 2 * t]);
                af[i][2] = *reinterpret_cast<const uint32_t *>(&As[r][ks + 2 * t + 8]);
                af[i][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][ks + 2 * t + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int c = wn + j * 8 + g;
                bfr[j][0] = *reinterpret_cast<const uint32_t *>(&Bs[c][ks + 2 * t]);
                bfr[j][1] = *reinterpret_cast<const uint32_t *>(&Bs[c][ks + 2 * t + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], af[i], bfr[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int row = m0 + wm + i * 16 + g + h * 8;
                const int col = n0 + wn + j * 8 + 2 * t;
                float v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
                if (accumulate) {
                    atomicAdd(&C[(size_t)row * ldc + col], v0);
                    atomicAdd(&C[(size_t)row * ldc + col + 1], v1);
                    continue;
                }
                if (bias) { v0 += bias[col]; v1 += bias[col + 1]; }
                if (relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
                if (C) { C[(size_t)row * ldc + col] = v0; C[(size_t)row * ldc + col + 1] = v1; }
                if (Cb) {
                    Cb[(size_t)row * ldcb + col] = __float2bfloat16_rn(v0);
                    Cb[(size_t)row * ldcb + col + 1] = __float2bfloat16_rn(v1);
                }
            }
}

// ------------------------------------------------------------------------------------------
// Fused inference: y[r] = w3 . relu(W2' relu(W1' relu(W0' x_r + b0) + b1) + b2) + b3[0]
//
// One warp owns 16 rows through all four layers.  The m16n8k16 accumulator of two adjacent
// n-tiles (columns 16k..16k+7 and 16k+8..16k+15) holds, lane by lane, exactly the A fragment of
// the k-slab 16k..16k+15 of the next layer, so activations never leave registers: bias, ReLU and
// the bf16 rounding happen on the accumulator and the packed pairs feed the next layer's MMAs.
// The weights are packed once in fragment order (kMlpPack* below: [layer][kslab][ntile][lane] of
// {b0b1, b2b3}) and copied into shared memory by every CTA of a persistent grid; a warp's B
// fragment is one 8-byte shared load per lane.  The chain of MMAs, bias/ReLU/bf16 points and the
// K order are those of the layer-by-layer forward (k_gemm), so y equals its column 0 bit for bit.
// Input columns 32..63 of X are zero padding (the first layer reads k-slabs 0 and 1 only).
// ------------------------------------------------------------------------------------------
constexpr int kMlpKs0 = 2, kMlpKsH = 8, kMlpNt = 16;
constexpr int kMlpOff1 = kMlpKs0 * kMlpNt * 32;                 // uint2 offsets of each layer
constexpr int kMlpOff2 = kMlpOff1 + kMlpKsH * kMlpNt * 32;
constexpr int kMlpOff3 = kMlpOff2 + kMlpKsH * kMlpNt * 32;
constexpr int kMlpPackWords = kMlpOff3 + kMlpKsH * 32;          // last layer: one n-tile (column 0 real)
constexpr int kMlpThreads = 256, kMlpRowsPerCta = 128;

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x = lo (lower address / lower 16 bits)
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t bf16_pair(const __nv_bfloat16 *W, int ldw, int k, int n) {
    __nv_bfloat162 v;
    v.x = W[(size_t)k * ldw + n];
    v.y = W[(size_t)(k + 1) * ldw + n];
    return *reinterpret_cast<const uint32_t *>(&v);
}

// W0..W2 bf16 [K][128] row-major, W3 bf16 [128][ldw3]; one thread per packed uint2
__global__ void k_mlp_pack(const __nv_bfloat16 *__restrict__ W0, const __nv_bfloat16 *__restrict__ W1,
                           const __nv_bfloat16 *__restrict__ W2, const __nv_bfloat16 *__restrict__ W3, int ldw3, uint2 *out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kMlpPackWords) return;
    const __nv_bfloat16 *W;
    int ldw, rel;
    if (e < kMlpOff1) { W = W0; ldw = 128; rel = e; }
    else if (e < kMlpOff2) { W = W1; ldw = 128; rel = e - kMlpOff1; }
    else if (e < kMlpOff3) { W = W2; ldw = 128; rel = e - kMlpOff2; }
    else { W = W3; ldw = ldw3; rel = e - kMlpOff3; }
    const int nts = (e < kMlpOff3) ? kMlpNt : 1;
    const int lane = rel & 31, nt = (rel >> 5) % nts, ks = (rel >> 5) / nts;
    const int g = lane >> 2, t = lane & 3;
    const int n = nt * 8 + g, k = ks * 16 + 2 * t;
    out[e] = make_uint2(bf16_pair(W, ldw, k, n), bf16_pair(W, ldw, k + 8, n));
}

template <int KS>
__device__ __forceinline__ void mlp_layer(float (&acc)[kMlpNt][4], const uint32_t (&a)[kMlpKsH][4], const uint2 *__restrict__ w,
                                          int lane) {
#pragma unroll
    for (int nt = 0; nt < kMlpNt; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < KS; ks++)
#pragma unroll
        for (int nt = 0; nt < kMlpNt; nt++) {
            const uint2 b2 = w[(ks * kMlpNt + nt) * 32 + lane];
            const uint32_t b[2] = {b2.x, b2.y};
            mma_bf16(acc[nt], a[ks], b);
        }
}

// bias + ReLU + bf16 on the accumulator, repacked as the next layer's A fragments
__device__ __forceinline__ void mlp_chain(const float (&acc)[kMlpNt][4], const float *__restrict__ bias, uint32_t (&a)[kMlpKsH][4],
                                          int t) {
#pragma unroll
    for (int nt = 0; nt < kMlpNt; nt++) {
        const int col = nt * 8 + 2 * t;
        const float b0 = bias[col], b1 = bias[col + 1];
        const float v0 = fmaxf(acc[nt][0] + b0, 0.f), v1 = fmaxf(acc[nt][1] + b1, 0.f);
        const float v2 = fmaxf(acc[nt][2] + b0, 0.f), v3 = fmaxf(acc[nt][3] + b1, 0.f);
        a[nt >> 1][(nt & 1) * 2 + 0] = pack_bf16x2(v0, v1);   // row g
        a[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16x2(v2, v3);   // row g + 8
    }
}

__global__ void __launch_bounds__(kMlpThreads, 2) k_mlp_fused(const __nv_bfloat16 *__restrict__ X, int ldx, int rows,
                                                              const uint2 *__restrict__ wpack, const float *__restrict__ b0,
                                                              const float *__restrict__ b1, const float *__restrict__ b2,
                                                              const float *__restrict__ b3, float *__restrict__ y) {
    extern __shared__ __align__(16) uint2 sw[];
    __shared__ float sb[3 * 128 + 4];
    for (int e = threadIdx.x; e < kMlpPackWords; e += blockDim.x) sw[e] = wpack[e];
    for (int e = threadIdx.x; e < 128; e += blockDim.x) { sb[e] = b0[e]; sb[128 + e] = b1[e]; sb[256 + e] = b2[e]; }
    if (threadIdx.x == 0) sb[384] = b3[0];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int ntiles = (rows + kMlpRowsPerCta - 1) / kMlpRowsPerCta;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int r0 = tile * kMlpRowsPerCta + warp * 16;
        if (r0 >= rows) continue;                    // rows is a multiple of 16: groups are whole
        uint32_t a[kMlpKsH][4];
        const __nv_bfloat16 *x0 = X + (size_t)(r0 + g) * ldx, *x1 = X + (size_t)(r0 + g + 8) * ldx;
#pragma unroll
        for (int ks = 0; ks < kMlpKs0; ks++) {
            a[ks][0] = *reinterpret_cast<const uint32_t *>(x0 + ks * 16 + 2 * t);
            a[ks][1] = *reinterpret_cast<const uint32_t *>(x1 + ks * 16 + 2 * t);
            a[ks][2] = *reinterpret_cast<const uint32_t *>(x0 + ks * 16 + 8 + 2 * t);
            a[ks][3] = *reinterpret_cast<const uint32_t *>(x1 + ks * 16 + 8 + 2 * t);
        }
        float acc[kMlpNt][4];
        mlp_layer<kMlpKs0>(acc, a, sw, lane);
        mlp_chain(acc, sb, a, t);
        mlp_layer<kMlpKsH>(acc, a, sw + kMlpOff1, lane);
        mlp_chain(acc, sb + 128, a, t);
        mlp_layer<kMlpKsH>(acc, a, sw + kMlpOff2, lane);
        mlp_chain(acc, sb + 256, a, t);
        float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < kMlpKsH; ks++) {
            const uint2 b2 = sw[kMlpOff3 + ks * 32 + lane];
            const uint32_t b[2] = {b2.x, b2.y};
            mma_bf16(o, a[ks], b);
        }
        if (t == 0) {
            y[r0 + g] = o[0] + sb[384];
            y[r0 + g + 8] = o[2] + sb[384];
        }
    }
}

// dZ = dA * (act > 0) -> bf16, for ReLU layers (act stored in bf16 by the forward pass)
__global__ void k_relu_bwd(int n, const float *__restrict__ dA, const __nv_bfloat16 *__restrict__ act, __nv_bfloat16 *dZ,
                           float *dZf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = __bfloat162float(act[i]) > 0.f ? dA[i] : 0.f;
    dZ[i] = __float2bfloat16_rn(v);
    if (dZf) dZf[i] = v;
}

// column sums of a [rows][cols] fp32 matrix into out[cols] (bias gradients), one block per column
__global__ void k_colsum(int rows, int cols, const float *__restrict__ X, float *out) {
    const int c = blockIdx.x;
    float s = 0.f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) s += X[(size_t)r * cols + c];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ float w[32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += w[k];
        out[c] = t;
    }
}

// Adam on fp32 master weights, bf16 copy for the tensor cores
__global__ void k_adam(int n, float *w, __nv_bfloat16 *wb, const float *__restrict__ grad, float *m, float *v, float lr,
                       float b1, float b2, float eps, float bc1, float bc2, float wd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gr = grad[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gr;
    const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    const float upd = lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    const float wn = w[i] - upd;
    w[i] = wn;
    if (wb) wb[i] = __float2bfloat16_rn(wn);
}

// mean-squared-error gradient on column 0 of Y [rows][ldy]: dY = 2 (Y - t) / rows (other columns 0),
// bf16 copy for the tensor cores, per-block loss partials
__global__ void k_mse_grad(int rows, int valid, int ldy, const float *__restrict__ Y, const float *__restrict__ t, float *dY,
                           __nv_bfloat16 *dYb, float *loss_part) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (r < rows) {
        const float e = (r < valid) ? Y[(size_t)r * ldy] - t[r] : 0.f;
        l = e * e;
        for (int c = 0; c < ldy; c++) {
            const float v = (c == 0) ? 2.f * e / (float)valid : 0.f;
            dY[(size_t)r * ldy + c] = v;
            dYb[(size_t)r * ldy + c] = __float2bfloat16_rn(v);
        }
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    __shared__ float w[32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += w[k];
        loss_part[blockIdx.x] = s;
    }
}

// ------------------------------------------------------------------------------------------
// features: 14 local + 16 message channels + 2 hydraulic estimates = 32 per cell (bf16 rows)
//
// The upstream messages are computed first as fp32 planes (one coalesced pass per hop), then one
// assembly pass writes each cell's 32 features as four 16-byte stores; nothing writes X columns
// one at a time (rows are 128 bytes apart, so column writes would touch every row's sector per hop).
// ------------------------------------------------------------------------------------------
struct EmuNet {
    int N, R;
    const int *next, *up_ptr, *up_idx;
    const double *rivelv, *elevtn, *nxtdst, *rivwth, *rivhgt, *rivlen, *rivstomax, *qref, *rivman;
    double pmanfld;
};


// hop-0 inputs: last-step mean outflow and runoff of every member, as fp32 planes
__global__ void k_emu_seed(EmuNet n, const double *__restrict__ qprev, const double *__restrict__ runoff, float *pa, float *pb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n.N) return;
    const size_t gi = (size_t)blockIdx.y * n.N + i;
    pa[gi] = (float)qprev[gi];
    pb[gi] = (float)runoff[gi];
}

// one hop of upstream message passing: out[i] = sum over upstream j of in[j], ascending upstream order
__global__ void k_emu_hop(EmuNet n, const float *__restrict__ in_a, const float *__restrict__ in_b, float *out_a, float *out_b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n.N) return;
    const size_t mo = (size_t)blockIdx.y * n.N;
    float a = 0.f, b = 0.f;
    for (int k = n.up_ptr[i]; k < n.up_ptr[i + 1]; k++) {
        const int j = n.up_idx[k];
        a += in_a[mo + j];
        b += in_b[mo + j];
    }
    out_a[mo + i] = a;
    out_b[mo + i] = b;
}

// Features feed a bf16 network (8-bit mantissa), so they are computed in fp32 with fast
// reciprocals and the hardware log/exp approximations: one reciprocal of the discharge scale per
// cell instead of a division per feature.  Training and inference use this same kernel.
// sign(x) log(1 + |x|); below 1e-3 the two-term series a - a^2/2 (relative error < a^2/3), where
// the hardware logarithm of 1 + a would lose the small ratios (runoff over a large river's scale)
__device__ __forceinline__ float fslog(float x) {
    const float a = fabsf(x);
    return copysignf(a < 1e-3f ? a * (1.f - 0.5f * a) : __logf(1.f + a), x);
}

// two hops in one pass: out1[i] = sum over upstream j of in[j]; out2[i] = sum over upstream j of
// (sum over upstream k of j of in[k]) -- the same fp32 sums, in the same ascending order, as two
// single-hop passes.  The first pair reads the fp64 last-step outflow and runoff directly (the
// single-hop chain converts them to fp32 planes first: the same values).
template <bool FromState>
__global__ void k_emu_hop2(EmuNet n, const float *__restrict__ in_a, const float *__restrict__ in_b,
                           const double *__restrict__ qa, const double *__restrict__ qb, float *o1a, float *o1b,
                           float *o2a, float *o2b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n.N) return;
    const size_t mo = (size_t)blockIdx.y * n.N;
    auto va = [&](int j) { return FromState ? (float)qa[mo + j] : in_a[mo + j]; };
    auto vb = [&](int j) { return FromState ? (float)qb[mo + j] : in_b[mo + j]; };
    float a1 = 0.f, b1 = 0.f, a2 = 0.f, b2 = 0.f;
    for (int k = n.up_ptr[i]; k < n.up_ptr[i + 1]; k++) {
        const int j = n.up_idx[k];
        a1 += va(j);
        b1 += vb(j);
        float sa = 0.f, sb = 0.f;
        for (int q = n.up_ptr[j]; q < n.up_ptr[j + 1]; q++) {
            const int g = n.up_idx[q];
            sa += va(g);
            sb += vb(g);
        }
        a2 += sa;
        b2 += sb;
    }
    o1a[mo + i] = a1;
    o1b[mo + i] = b1;
    o2a[mo + i] = a2;
    o2b[mo + i] = b2;
}

// Manning discharge of a rectangular section of area A, hydraulic depth h and friction slope s
__device__ __forceinline__ float manning_q(float area, float h, float s, float inv_man) {
    if (!(area > 0.f) || !(h > 0.f)) return 0.f;
    return copysignf(area * __expf(0.6666667f * __logf(h)) * sqrtf(fabsf(s)) * inv_man, s);
}

// features of cell i of member blockIdx.y; planes [2*(hops+1)][M*N] (0,1 = seeds; 2h+2, 2h+3 = hop h)
__global__ void k_emu_assemble(EmuNet n, const double *__restrict__ rivsto, const double *__restrict__ fldsto,
                               const double *__restrict__ levsto, const double *__restrict__ rivdph,
                               const double *__restrict__ flddph, const double *__restrict__ fldfrc,
                               const double *__restrict__ qprev, const double *__restrict__ runoff,
                               const float *__restrict__ planes, size_t plane, int hops, __nv_bfloat16 *X, int ldx,
                               int rows_per_member) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n.N) return;
    // member blockIdx.y: state arrays are member-major [M][N], X rows [M][rows_per_member]
    const size_t mo = (size_t)blockIdx.y * n.N, gi = mo + i;
    const float qf = (float)n.qref[i];
    const float iq = __frcp_rn(qf);
    const double Sd = rivsto[gi] + fldsto[gi] + (levsto ? levsto[gi] : 0.0);
    const float S = (float)Sd;
    const float rdph = (float)rivdph[gi], fdph = (float)flddph[gi];
    const float len = (float)n.rivlen[i], wth = (float)n.rivwth[i], hgt = (float)n.rivhgt[i];
    float f[32];
    f[0] = fslog(S * __frcp_rn((float)n.rivstomax[i]));
    f[1] = rdph * __frcp_rn(hgt);
    f[2] = fslog(fdph);
    f[3] = fslog((float)qprev[gi] * iq);
    f[4] = fslog((float)runoff[gi] * iq);
    f[5] = (float)fldfrc[gi];
    const bool mouth = i >= n.R;
    const int j = mouth ? i : n.next[i];
    const float inv_dst = __frcp_rn(mouth ? 10000.f : (float)n.nxtdst[i]);
    const double sfc = n.rivelv[i] + rivdph[gi], sfcn = mouth ? n.elevtn[i] : n.rivelv[j] + rivdph[mo + j];
    const float slope = (float)(sfc - sfcn) * inv_dst;   // elevations subtracted in fp64
    f[6] = fslog(1000.f * slope);
    f[7] = fslog(1000.f * (float)(n.elevtn[i] - (mouth ? n.elevtn[i] : n.elevtn[j])) * __frcp_rn((float)n.nxtdst[i]));
    f[8] = __logf(len) - 9.5f;
    f[9] = __logf(wth) - 4.0f;
    f[10] = __logf(hgt) - 1.0f;
    f[11] = __logf(qf) - 3.0f;
    f[12] = mouth ? 1.f : 0.f;
    f[13] = fslog(S * iq * (1.f / 3600.f));
#pragma unroll
    for (int h = 0; h < 8; h++) {
        if (h < hops) {
            f[14 + 2 * h] = fslog(planes[(size_t)(2 + 2 * h) * plane + gi] * iq);
            f[15 + 2 * h] = fslog(planes[(size_t)(3 + 2 * h) * plane + gi] * iq);
        } else {
            f[14 + 2 * h] = f[15 + 2 * h] = 0.f;
        }
    }
    // hydraulic estimates: Manning discharge of the channel and of the floodplain at the current
    // water-surface slope (the state the local-inertial scheme relaxes towards within an hour)
    const float af = fmaxf((float)fldsto[gi] * __frcp_rn(len) - fdph * wth, 0.f);
    f[30] = fslog(manning_q(wth * rdph, rdph, slope, __frcp_rn((float)n.rivman[i])) * iq);
    f[31] = fslog(manning_q(af, fdph, fmaxf(-0.005f, fminf(0.005f, slope)), __frcp_rn((float)n.pmanfld)) * iq);
    uint4 *row = reinterpret_cast<uint4 *>(X + ((size_t)blockIdx.y * rows_per_member + i) * ldx);
#pragma unroll
    for (int v = 0; v < 4; v++) {
        uint4 u;
        u.x = pack_bf16x2(f[8 * v + 0], f[8 * v + 1]);
        u.y = pack_bf16x2(f[8 * v + 2], f[8 * v + 3]);
        u.z = pack_bf16x2(f[8 * v + 4], f[8 * v + 5]);
        u.w = pack_bf16x2(f[8 * v + 6], f[8 * v + 7]);
        row[v] = u;
    }
}

// Mass-conserving rollout of one coupling step from the predicted transformed mean outflow:
// Q_i = qref_i * expm1(max(base_i + y_i, 0)) with base_i = log1p(Qprev_i/qref_i) when the network
// predicts the change over the step (residual != 0) and 0 when it predicts the value itself, limited
// to the storage the cell holds plus its own runoff over DT (so storage never goes negative whatever
// its upstream delivers); storage then changes by (inflow + runoff - outflow) * DT with the inflow
// gathered over the upstream CSR.
__global__ void k_emu_rollout(EmuNet n, const float *y, int ldy, int rows_per_member, const int *active, double dt,
                              int residual, const double *runoff, const double *rivsto, const double *fldsto,
                              const double *levsto, const double *qprev, double *qout) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n.N || !active[blockIdx.y]) return;
    const size_t mo = (size_t)blockIdx.y * n.N;
    y += (size_t)blockIdx.y * rows_per_member * ldy;
    runoff += mo; rivsto += mo; fldsto += mo; if (levsto) levsto += mo; qout += mo;
    const double S = rivsto[i] + fldsto[i] + (levsto ? levsto[i] : 0.0);
    // the network predicts the change of log1p(Q/qref) over the step (residual on the last outflow)
    const double base = residual ? log1p(fmax(qprev[mo + i], 0.0) / n.qref[i]) : 0.0;
    const double yi = fmax(base + (double)y[(size_t)i * ldy], 0.0);
    double q = n.qref[i] * expm1(yi);
    q = fmin(q, S / dt + runoff[i]);
    qout[i] = fmax(q, 0.0);
}

__global__ void k_emu_update(EmuNet n, const int *active, double dt, const double *runoff, const double *qout, double *rivsto,
                             double *fldsto, double *levsto, double *rivout_pre, double *fldout_pre, double *qprev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n.N || !active[blockIdx.y]) return;
    const size_t mo = (size_t)blockIdx.y * n.N;
    runoff += mo; qout += mo; rivsto += mo; fldsto += mo; if (levsto) levsto += mo; rivout_pre += mo; fldout_pre += mo;
    qprev += mo;
    double inflow = 0.0;
    for (int k = n.up_ptr[i]; k < n.up_ptr[i + 1]; k++) inflow += qout[n.up_idx[k]];
    const double S = rivsto[i] + fldsto[i] + (levsto ? levsto[i] : 0.0);
    const double Snew = fmax(S + (inflow + runoff[i] - qout[i]) * dt, 0.0);
    rivsto[i] = Snew;   // the stage scheme re-splits river / floodplain / protected storage
    fldsto[i] = 0.0;
    if (levsto) levsto[i] = 0.0;
    rivout_pre[i] = qout[i];
    fldout_pre[i] = 0.0;
    qprev[i] = qout[i];
}


// ------------------------------------------------------------------------------------------
// Fused inference on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One CTA per SM (a persistent grid) holds all four layers' weights in shared memory once, as
// the MMAs' B operands, and runs four 128-row tiles at a time: warpgroup s (warps 4s..4s+3) owns
// tile slot s -- its activation buffer (the next MMA's A operand) and 128 of the SM's 512
// tensor-memory columns -- and a seventeenth warp issues the MMAs.  Both operands use the K-major
// no-swizzle canonical layout: 16-byte rows of 8 bf16 grouped in 8-row core matrices, byte offset
// (k/8)*(R*16) + (r/8)*128 + (r%8)*16 for an R-row operand.  Per layer of a slot: the warpgroup
// writes the A operand, arrives on the slot's `ready` mbarrier; the MMA warp, polling all four
// slots, issues that layer's tcgen05.mma chain (M=128, N=128 or 16, K=16 per instruction, fp32
// accumulator in the slot's columns) and commits it to the slot's `done` mbarrier; the warpgroup
// waits on it, reads its rows with tcgen05.ld (warp 4s+q owns TMEM lanes 32q..32q+31), adds the
// bias, applies ReLU and the bf16 rounding in one cvt and writes the next A operand.  While one
// slot runs its epilogue the tensor pipe serves the others.  The last layer (N=16, column 0 real)
// adds b3 and writes y.  Every wait is bounded: a wait that runs out raises the CTA's abort flag,
// every warpgroup leaves at its next vote, and the MMA warp drains the MMAs it issued (one more
// commit, waited for with the full bound) before the tensor memory is released.  The rounding
// points equal the layer-by-layer chain (bf16 inputs, fp32 accumulation, bf16 activations) and the
// K=16 steps run in the same order, so the outputs equal that chain bit for bit.
// ------------------------------------------------------------------------------------------
constexpr int kTcRows = 128;
constexpr int kTcSlots = 4;                           // tiles in flight per CTA
constexpr int kTcEpi = 128 * kTcSlots;                // epilogue threads (4 warpgroups)
constexpr int kTcThreads = kTcEpi + 32;               // + the MMA warp
constexpr int kTcW0 = 0;                              // byte offsets inside the packed image
constexpr int kTcW1 = kTcW0 + 128 * 32 * 2;           // layer 0: N=128, K=32
constexpr int kTcW2 = kTcW1 + 128 * 128 * 2;          // layers 1, 2: N=128, K=128
constexpr int kTcW3 = kTcW2 + 128 * 128 * 2;          // layer 3: N=16, K=128
constexpr int kTcWBytes = kTcW3 + 16 * 128 * 2;
constexpr int kTcABytes = kTcRows * 128 * 2;          // one slot's activations: 128 rows x 128 k
constexpr int kTcA = kTcWBytes;
constexpr int kTcBias = kTcA + kTcSlots * kTcABytes;  // b0 b1 b2 (3 x 128 floats), b3[0]
constexpr int kTcMisc = kTcBias + (3 * 128 + 4) * 4;  // ready[4], done[4], drain mbarriers; TMEM address; abort
constexpr int kTcSmem = kTcMisc + (2 * kTcSlots + 1) * 8 + 16;
constexpr int kTcCols = 128 * kTcSlots;               // tensor-memory columns of the CTA
#ifndef CMF_TC_WAIT_LIMIT
#define CMF_TC_WAIT_LIMIT (1 << 20)
#endif
constexpr int kTcWaitLimit = CMF_TC_WAIT_LIMIT;        // polls of an MMA completion before giving up
int g_tc_wait_limit = kTcWaitLimit;                   // host side: the bound the next launches use

__device__ int g_mlp_tc_status;                       // 0 ok; 1: an MMA completion wait ran out

__host__ __device__ constexpr uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    // start address, leading- and stride-dimension byte offsets (16-byte units), version 1,
    // base offset 0, no swizzle
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
    // D fp32, A and B bf16, both K-major, N/8 and M/16
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of element (r, k) of an R-row K-major operand in the canonical layout
__host__ __device__ constexpr uint32_t canon_off(int r, int k, int R) {
    return (uint32_t)((k >> 3) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// B operands of the four layers as one shared-memory image: element (n, k) = W[k][n]
__global__ void k_mlp_tc_pack(const __nv_bfloat16 *__restrict__ W0, const __nv_bfloat16 *__restrict__ W1,
                              const __nv_bfloat16 *__restrict__ W2, const __nv_bfloat16 *__restrict__ W3, int ldw3,
                              __nv_bfloat16 *out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int n0 = 128 * 32, n1 = 128 * 128, n3 = 16 * 128;
    if (e >= n0 + 2 * n1 + n3) return;
    int n, k, R, base;
    const __nv_bfloat16 *W;
    int ldw;
    if (e < n0) { n = e / 32; k = e % 32; R = 128; base = kTcW0; W = W0; ldw = 128; }
    else if (e < n0 + n1) { const int q = e - n0; n = q / 128; k = q % 128; R = 128; base = kTcW1; W = W1; ldw = 128; }
    else if (e < n0 + 2 * n1) { const int q = e - n0 - n1; n = q / 128; k = q % 128; R = 128; base = kTcW2; W = W2; ldw = 128; }
    else { const int q = e - n0 - 2 * n1; n = q / 128; k = q % 128; R = 16; base = kTcW3; W = W3; ldw = ldw3; }
    out[(base + canon_off(n, k, R)) / 2] = W[(size_t)k * ldw + n];
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(mbar) : "memory");
}

// bounded wait on an mbarrier phase; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int limit) {
    for (int i = 0; i < limit; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld1(uint32_t taddr, uint32_t &v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(v) : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ReLU and round-to-nearest bf16 of two fp32 values in one instruction (ReLU commutes with the
// rounding, so this equals rounding max(x, 0)); lo goes to the lower half
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// layer epilogue: bias + ReLU + bf16 of the 128 accumulator columns of row r into the next
// layer's A operand (two 32-column loads in flight)
__device__ __forceinline__ void tc_epilogue_hidden(uint32_t tmem_row, const float *bias, unsigned char *sA, int r) {
#pragma unroll
    for (int h = 0; h < 4; h += 2) {
        uint32_t v[2][32];
        tmem_ld32(tmem_row + 32 * h, v[0]);
        tmem_ld32(tmem_row + 32 * (h + 1), v[1]);
        tmem_wait_ld();
#pragma unroll
        for (int g = 0; g < 2; g++) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int c = 32 * (h + g) + 8 * q;       // first of 8 columns = k chunk c/8 of the next layer
                uint4 u;
                uint32_t *w = reinterpret_cast<uint32_t *>(&u);
#pragma unroll
                for (int j = 0; j < 4; j++)
                    w[j] = relu_bf16x2(__uint_as_float(v[g][8 * q + 2 * j]) + bias[c + 2 * j],
                                       __uint_as_float(v[g][8 * q + 2 * j + 1]) + bias[c + 2 * j + 1]);
                *reinterpret_cast<uint4 *>(sA + canon_off(r, c, kTcRows)) = u;
            }
        }
    }
}

__device__ __forceinline__ void named_bar(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(nthreads) : "memory");
}
// named barrier with an OR over the participants' flags: every participant gets the same answer
__device__ __forceinline__ bool named_bar_or(int id, int nthreads, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, %2, %3, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r) : "r"((uint32_t)v), "r"(id), "r"(nthreads) : "memory");
    return r != 0;
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
    return ok != 0;
}

__global__ void __launch_bounds__(kTcThreads, 1) k_mlp_tc(const __nv_bfloat16 *__restrict__ X, int ldx, int rows,
                                                        const uint4 *__restrict__ wimg, const float *__restrict__ b0,
                                                        const float *__restrict__ b1, const float *__restrict__ b2,
                                                        const float *__restrict__ b3, float *__restrict__ y,
                                                        int wait_limit) {
    extern __shared__ __align__(1024) unsigned char sm[];
    float *sb = reinterpret_cast<float *>(sm + kTcBias);
    uint64_t *ready = reinterpret_cast<uint64_t *>(sm + kTcMisc);
    uint64_t *done = ready + kTcSlots;
    uint64_t *drain = done + kTcSlots;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // weights and biases into shared memory
    for (int e = tid; e < kTcWBytes / 16; e += kTcThreads) reinterpret_cast<uint4 *>(sm)[e] = wimg[e];
    for (int e = tid; e < 128; e += kTcThreads) { sb[e] = b0[e]; sb[128 + e] = b1[e]; sb[256 + e] = b2[e]; }
    if (tid == 0) {
        sb[384] = b3[0];
        for (int q = 0; q < 2 * kTcSlots + 1; q++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(ready + q)) : "memory");
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {   // one warp allocates the CTA's accumulator columns and releases the allocation permit
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tslot)), "r"(kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int ntiles = (rows + kTcRows - 1) / kTcRows;
    const int stride = kTcSlots * (int)gridDim.x;             // tiles of slot s: first + j * stride
    if (warp < kTcSlots * 4) {
        // ---- epilogue warpgroup of slot s
        const int sl = warp >> 2, q = warp & 3;
        const int r = 32 * q + lane;                          // this thread's row == TMEM lane
        unsigned char *sA = sm + kTcA + sl * kTcABytes;
        const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(128 * sl);
        const uint32_t rd = smem_u32(ready + sl), dn = smem_u32(done + sl);
        const int bar = 1 + sl;                               // named barrier of the warpgroup
        uint32_t dphase = 0;
        bool go = true;
        int t = blockIdx.x * kTcSlots + sl;
        uint4 xn[4];                                          // this row's X (32 bf16) of tile t
#pragma unroll
        for (int kc = 0; kc < 4; kc++) xn[kc] = make_uint4(0u, 0u, 0u, 0u);
        if (t < ntiles && t * kTcRows + r < rows)
#pragma unroll
            for (int kc = 0; kc < 4; kc++) xn[kc] = *reinterpret_cast<const uint4 *>(X + (size_t)(t * kTcRows + r) * ldx + kc * 8);
        for (; t < ntiles && go; t += stride) {
            const int row = t * kTcRows + r;
#pragma unroll
            for (int kc = 0; kc < 4; kc++) *reinterpret_cast<uint4 *>(sA + canon_off(r, kc * 8, kTcRows)) = xn[kc];
            // the next tile's row of X, fetched while this tile's layers run
            const int tn = t + stride;
#pragma unroll
            for (int kc = 0; kc < 4; kc++) xn[kc] = make_uint4(0u, 0u, 0u, 0u);
            if (tn < ntiles && tn * kTcRows + r < rows)
#pragma unroll
                for (int kc = 0; kc < 4; kc++) xn[kc] = *reinterpret_cast<const uint4 *>(X + (size_t)(tn * kTcRows + r) * ldx + kc * 8);
            fence_async_smem();
            tc_fence_before();
            named_bar(bar, 128);
            if (r == 0) mbar_arrive(rd);
#pragma unroll 1
            for (int layer = 0; layer < 4; layer++) {
                // bounded wait for this layer's MMAs, then a warpgroup-uniform vote on the outcome
                // (an OR over the warpgroup's flags, so no thread goes on to a barrier the others left)
                bool fail = false;
                int spins = 0;
                while (!mbar_try(dn, dphase)) {
                    if (*abort_flag) { fail = true; break; }
                    if (++spins > wait_limit) { *abort_flag = 1; fail = true; break; }
                }
                if (named_bar_or(bar, 128, fail)) { go = false; break; }
                dphase ^= 1u;
                tc_fence_after();
                if (layer < 3) {
                    tc_epilogue_hidden(trow, sb + 128 * layer, sA, r);
                    fence_async_smem();
                    tc_fence_before();
                    named_bar(bar, 128);
                    if (r == 0) mbar_arrive(rd);
                } else {
                    uint32_t v;
                    tmem_ld1(trow, v);
                    tmem_wait_ld();
                    if (row < rows) y[row] = __uint_as_float(v) + sb[384];
                    tc_fence_before();
                    named_bar(bar, 128);   // the slot's columns and A buffer are free for the next tile
                }
            }
        }
    } else {
      if (lane == 0) {
        // ---- MMA warp: issues every layer of every slot as its A operand becomes ready
        const uint32_t sw = smem_u32(sm);
        const uint32_t id128 = umma_idesc_bf16_f32(128, 128), id16 = umma_idesc_bf16_f32(128, 16);
        int left[kTcSlots], layer[kTcSlots];
        uint32_t rphase[kTcSlots];
        int remaining = 0;
#pragma unroll
        for (int sl = 0; sl < kTcSlots; sl++) {
            const int t0 = blockIdx.x * kTcSlots + sl;
            left[sl] = t0 < ntiles ? 4 * ((ntiles - 1 - t0) / stride + 1) : 0;
            layer[sl] = 0;
            rphase[sl] = 0u;
            remaining += left[sl];
        }
        bool issued_any = false;
        int spins = 0;
        while (remaining > 0) {
            bool progressed = false;
#pragma unroll
            for (int sl = 0; sl < kTcSlots; sl++) {
                if (left[sl] == 0 || !mbar_try(smem_u32(ready + sl), rphase[sl])) continue;
                rphase[sl] ^= 1u;
                tc_fence_after();
                const int L = layer[sl];
                const int ksteps = L == 0 ? 2 : 8;
                const uint32_t wb = sw + (L == 0 ? kTcW0 : L == 1 ? kTcW1 : L == 2 ? kTcW2 : kTcW3);
                const uint32_t blbo = L == 3 ? 16 * 16 : 128 * 16;
                const uint32_t sa = sw + kTcA + sl * kTcABytes;
                for (int st = 0; st < ksteps; st++) {
                    const uint64_t ad = umma_smem_desc(sa + 2 * st * (128 * 16), 128 * 16, 128);
                    const uint64_t bd = umma_smem_desc(wb + 2 * st * blbo, blbo, 128);
                    umma_bf16(tmem + 128 * sl, ad, bd, L == 3 ? id16 : id128, st > 0 ? 1u : 0u);
                }
                umma_commit(smem_u32(done + sl));
                issued_any = true;
                layer[sl] = (L + 1) & 3;
                left[sl]--;
                remaining--;
                progressed = true;
            }
            if (progressed) {
                spins = 0;
            } else {
                if (*abort_flag) break;
                if (++spins > wait_limit) { *abort_flag = 1; break; }
            }
        }
        if (issued_any) {
            // every MMA this thread issued completes before the columns are released, also those
            // whose completion no warpgroup waited for after an abort: one more commit tracks all
            // of them, waited for with the full bound
            umma_commit(smem_u32(drain));
            mbar_wait(smem_u32(drain), 0u, kTcWaitLimit);
        }
      }
      __syncwarp();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (*abort_flag && tid == 0) atomicExch(&g_mlp_tc_status, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTcCols) : "memory");
}

// ------------------------------------------------------------------------------------------
// Training GEMM on the 5th-generation tensor cores: the contract of k_gemm (C (+)= op(A) op(B),
// bias + ReLU, fp32 and/or bf16 output, or split-K atomic accumulation), with the products on
// tcgen05.  CTA tile 128 rows x NT columns (NT = 128, or 64 when N is not a multiple of 128); K in
// chunks of 64 staged into two shared-memory buffers in the canonical K-major no-swizzle layout
// (operands stored transposed in global memory are written element by element); one thread issues
// the chunk's MMAs (M=128, N=NT, K=16, bf16 x bf16 -> fp32) into a tensor-memory accumulator and
// commits them to the buffer's mbarrier, which completes (bounded wait) before the buffer is refilled.
// Epilogue: thread t owns row t (TMEM lane t) and reads its NT accumulator columns 32 at a time.
// With `zstride` > 0 every K slice stores its own partial product at C + blockIdx.z * zstride
// (plain stores, no bias or ReLU); k_splitk_reduce then adds the slices to the output in slice
// order, so a split-K product is the same bits on every run.
// ------------------------------------------------------------------------------------------
constexpr int kGThreads = 128;                          // = rows of the tile = TMEM lanes
constexpr int kGK = 64;                                 // K per staged chunk
constexpr int kGTileBytes = 128 * kGK * 2;              // one 128-row operand chunk (bf16)
constexpr int kGBuf = 2 * kGTileBytes;                  // A and B chunks of one buffer
constexpr int kGSmem = 2 * kGBuf + 64;                  // two buffers, two mbarriers, TMEM address

// stages rows [r0, r0 + 128) (rows >= rmax zero) x k [k0, k0 + kc) of an operand whose element
// (r, k) is at P[r * ld + k] (kmajor) or P[k * ld + r] (r contiguous) into the canonical layout
__device__ __forceinline__ void gemm_stage(unsigned char *dst, int R, const __nv_bfloat16 *__restrict__ P, int ld,
                                           bool kmajor, int r0, int rmax, int k0, int kc) {
    const int tid = threadIdx.x;
    if (kmajor) {
        const int cpr = kc / 8;                          // 16-byte chunks per row
        for (int e = tid; e < R * cpr; e += kGThreads) {
            const int r = e / cpr, kq = e - r * cpr;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (r0 + r < rmax) v = *reinterpret_cast<const uint4 *>(P + (size_t)(r0 + r) * ld + k0 + kq * 8);
            *reinterpret_cast<uint4 *>(dst + canon_off(r, kq * 8, R)) = v;
        }
    } else {
        const int cpk = R / 8;                           // 16-byte chunks along r per k
        for (int e = tid; e < kc * cpk; e += kGThreads) {
            const int k = e / cpk, rq = e - k * cpk;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (r0 + rq * 8 < rmax) v = *reinterpret_cast<const uint4 *>(P + (size_t)(k0 + k) * ld + r0 + rq * 8);
            const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
            for (int j = 0; j < 8; j++) *reinterpret_cast<__nv_bfloat16 *>(dst + canon_off(rq * 8 + j, k, R)) = h[j];
        }
    }
}

template <int NT>
__global__ void __launch_bounds__(kGThreads) k_gemm_tc(int M, int N, int K, const __nv_bfloat16 *__restrict__ A, int lda,
                                                       int transA, const __nv_bfloat16 *__restrict__ B, int ldb, int transB,
                                                       float *C, int ldc, __nv_bfloat16 *Cb, int ldcb,
                                                       const float *__restrict__ bias, int relu, int accumulate,
                                                       int k_per_split, int wait_limit, size_t zstride) {
    extern __shared__ __align__(1024) unsigned char sm[];
    if (zstride) C += blockIdx.z * zstride;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + 2 * kGBuf);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + 2 * kGBuf + 16);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * NT;
    const int kbeg = blockIdx.z * k_per_split, kend = min(K, kbeg + k_per_split);
    if (tid == 0) {
        for (int b = 0; b < 2; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[b])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(tslot)), "r"(NT)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = umma_idesc_bf16_f32(128, NT);
    uint32_t phase[2] = {0u, 0u};
    bool issued[2] = {false, false};
    bool failed = false;
    int chunk = 0;
    for (int k0 = kbeg; k0 < kend; k0 += kGK, chunk++) {
        const int buf = chunk & 1;
        unsigned char *sA = sm + buf * kGBuf, *sB = sA + kGTileBytes;
        if (issued[buf]) {   // the MMAs that read this buffer two chunks ago must have finished
            const bool ok = mbar_wait(smem_u32(&mbar[buf]), phase[buf], wait_limit);
            if (__syncthreads_or(ok ? 0 : 1)) { failed = true; break; }   // block-uniform
            phase[buf] ^= 1u;
            issued[buf] = false;
            tc_fence_after();
        }
        const int kc = min(kGK, kend - k0);             // a multiple of 32
        gemm_stage(sA, 128, A, lda, !transA, m0, M, k0, kc);
        gemm_stage(sB, NT, B, ldb, transB != 0, n0, N, k0, kc);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            for (int s = 0; s < kc / 16; s++) {
                const uint64_t ad = umma_smem_desc(smem_u32(sA) + 2 * s * (128 * 16), 128 * 16, 128);
                const uint64_t bd = umma_smem_desc(smem_u32(sB) + 2 * s * (NT * 16), NT * 16, 128);
                umma_bf16(tmem, ad, bd, idesc, (chunk > 0 || s > 0) ? 1u : 0u);
            }
            umma_commit(smem_u32(&mbar[buf]));
        }
        issued[buf] = true;
    }
    // the outstanding commits, oldest first (after a failure: drain them with the full bound
    // before the accumulator columns are released)
    for (int q = 0; q < 2; q++) {
        const int b = (chunk + q) & 1;
        if (!issued[b]) continue;
        const bool ok = mbar_wait(smem_u32(&mbar[b]), phase[b], failed ? kTcWaitLimit : wait_limit);
        if (__syncthreads_or(ok ? 0 : 1)) failed = true;
        phase[b] ^= 1u;
    }
    tc_fence_after();
    if (failed) {
        if (tid == 0) atomicExch(&g_mlp_tc_status, 1);
    } else {
        const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
        const int row = m0 + tid;
        const bool vec = ((ldc & 3) == 0) && (((uintptr_t)C & 15) == 0);
#pragma unroll 1
        for (int c0 = 0; c0 < NT; c0 += 32) {
            uint32_t v[32];
            tmem_ld32(trow + c0, v);
            tmem_wait_ld();
            if (row >= M) continue;
            const int col = n0 + c0;
            float x[32];
#pragma unroll
            for (int j = 0; j < 32; j++) x[j] = __uint_as_float(v[j]);
            if (accumulate) {
#pragma unroll
                for (int j = 0; j < 32; j++) atomicAdd(&C[(size_t)row * ldc + col + j], x[j]);
                continue;
            }
#pragma unroll
            for (int j = 0; j < 32; j++) {
                if (bias) x[j] += bias[col + j];
                if (relu) x[j] = fmaxf(x[j], 0.f);
            }
            if (C) {
                float *dst = C + (size_t)row * ldc + col;
                if (vec) {
#pragma unroll
                    for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4 *>(dst + j) = make_float4(x[j], x[j + 1], x[j + 2], x[j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; j++) dst[j] = x[j];
                }
            }
            if (Cb) {
#pragma unroll
                for (int j = 0; j < 32; j++) Cb[(size_t)row * ldcb + col + j] = __float2bfloat16_rn(x[j]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(NT) : "memory");
}

// C[r][c] = ((C[r][c] + P_0[r][c]) + P_1[r][c]) + ...: the split-K slices in slice order
__global__ void k_splitk_reduce(int M, int N, int splits, const float *__restrict__ ws, float *C, int ldc) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t MN = (size_t)M * N;
    if (e >= MN) return;
    const int r = (int)(e / N), c = (int)(e - (size_t)r * N);
    float x = C[(size_t)r * ldc + c];
    for (int z = 0; z < splits; z++) x += ws[z * MN + e];
    C[(size_t)r * ldc + c] = x;
}

}  // namespace

extern "C" {

const char *cmf_emu_last_error(void) { return g_emu_err.c_str(); }

int cmf_emu_gemm(int M, int N, int K, const void *A, int lda, int transA, const void *B, int ldb, int transB, float *C,
                 int ldc, void *Cb, int ldcb, const float *bias, int relu, int accumulate, int ksplit, void *stream) {
    if (M % TM || N % TN || K % TK || M <= 0 || N <= 0 || K <= 0)
        return emu_err(CMF_E_ARG, "cmf_emu_gemm: M,N must be multiples of 64 and K of 32");
    if ((lda % 8) || (ldb % 8) || ((uintptr_t)A & 15) || ((uintptr_t)B & 15))
        return emu_err(CMF_E_ARG, "cmf_emu_gemm: lda, ldb must be multiples of 8 and A, B 16-byte aligned");
    int dev = 0, major = 0;
    EMU_TRY(cudaGetDevice(&dev));
    EMU_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) return emu_err(CMF_E_NO_DEVICE, "cmf_emu_gemm: needs an sm_100 device");
    if (ksplit < 1) ksplit = 1;
    const int kps = ((K / ksplit + kGK - 1) / kGK) * kGK;   // whole chunks per split
    const int splits = (K + kps - 1) / kps;
    if (splits > 1 && !accumulate) return emu_err(CMF_E_ARG, "cmf_emu_gemm: split-K needs accumulate=1");
    cudaStream_t st = (cudaStream_t)stream;
    if (N % 128 == 0) {
        EMU_TRY(cudaFuncSetAttribute(k_gemm_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
        dim3 grid((M + 127) / 128, N / 128, splits);
        k_gemm_tc<128><<<grid, kGThreads, kGSmem, st>>>(M, N, K, (const __nv_bfloat16 *)A, lda, transA, (const __nv_bfloat16 *)B,
                                                       ldb, transB, C, ldc, (__nv_bfloat16 *)Cb, ldcb, bias, relu, accumulate,
                                                       kps, g_tc_wait_limit, (size_t)0);
    } else {
        EMU_TRY(cudaFuncSetAttribute(k_gemm_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
        dim3 grid((M + 127) / 128, N / 64, splits);
        k_gemm_tc<64><<<grid, kGThreads, kGSmem, st>>>(M, N, K, (const __nv_bfloat16 *)A, lda, transA, (const __nv_bfloat16 *)B,
                                                      ldb, transB, C, ldc, (__nv_bfloat16 *)Cb, ldcb, bias, relu, accumulate,
                                                      kps, g_tc_wait_limit, (size_t)0);
    }
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

size_t cmf_emu_gemm_splitk_ws_floats(int M, int N, int K, int ksplit) {
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    if (ksplit < 1) ksplit = 1;
    const int kps = ((K / ksplit + kGK - 1) / kGK) * kGK;
    return (size_t)((K + kps - 1) / kps) * (size_t)M * (size_t)N;
}

int cmf_emu_gemm_splitk(int M, int N, int K, const void *A, int lda, int transA, const void *B, int ldb, int transB,
                        float *C, int ldc, int ksplit, float *workspace, size_t workspace_floats, void *stream) {
    if (M % TM || N % TN || K % TK || M <= 0 || N <= 0 || K <= 0)
        return emu_err(CMF_E_ARG, "cmf_emu_gemm_splitk: M,N must be multiples of 64 and K of 32");
    if ((lda % 8) || (ldb % 8) || ((uintptr_t)A & 15) || ((uintptr_t)B & 15))
        return emu_err(CMF_E_ARG, "cmf_emu_gemm_splitk: lda, ldb must be multiples of 8 and A, B 16-byte aligned");
    if (!C || !workspace) return emu_err(CMF_E_ARG, "cmf_emu_gemm_splitk: C and workspace are required");
    int dev = 0, major = 0;
    EMU_TRY(cudaGetDevice(&dev));
    EMU_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) return emu_err(CMF_E_NO_DEVICE, "cmf_emu_gemm_splitk: needs an sm_100 device");
    if (ksplit < 1) ksplit = 1;
    const int kps = ((K / ksplit + kGK - 1) / kGK) * kGK;
    const int splits = (K + kps - 1) / kps;
    const size_t MN = (size_t)M * N;
    if (workspace_floats < (size_t)splits * MN)
        return emu_err(CMF_E_ARG, "cmf_emu_gemm_splitk: workspace smaller than cmf_emu_gemm_splitk_ws_floats()");
    cudaStream_t st = (cudaStream_t)stream;
    if (N % 128 == 0) {
        EMU_TRY(cudaFuncSetAttribute(k_gemm_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
        dim3 grid((M + 127) / 128, N / 128, splits);
        k_gemm_tc<128><<<grid, kGThreads, kGSmem, st>>>(M, N, K, (const __nv_bfloat16 *)A, lda, transA, (const __nv_bfloat16 *)B,
                                                       ldb, transB, workspace, N, nullptr, 0, nullptr, 0, 0, kps,
                                                       g_tc_wait_limit, MN);
    } else {
        EMU_TRY(cudaFuncSetAttribute(k_gemm_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
        dim3 grid((M + 127) / 128, N / 64, splits);
        k_gemm_tc<64><<<grid, kGThreads, kGSmem, st>>>(M, N, K, (const __nv_bfloat16 *)A, lda, transA, (const __nv_bfloat16 *)B,
                                                      ldb, transB, workspace, N, nullptr, 0, nullptr, 0, 0, kps,
                                                      g_tc_wait_limit, MN);
    }
    EMU_TRY(cudaGetLastError());
    k_splitk_reduce<<<(unsigned)((MN + 255) / 256), 256, 0, st>>>(M, N, splits, workspace, C, ldc);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_gemm_mma(int M, int N, int K, const void *A, int lda, int transA, const void *B, int ldb, int transB, float *C,
                     int ldc, void *Cb, int ldcb, const float *bias, int relu, int accumulate, int ksplit, void *stream) {
    if (M % TM || N % TN || K % TK || M <= 0 || N <= 0 || K <= 0)
        return emu_err(CMF_E_ARG, "cmf_emu_gemm_mma: M,N must be multiples of 64 and K of 32");
    if (ksplit < 1) ksplit = 1;
    int kps = ((K / ksplit + TK - 1) / TK) * TK;
    const int splits = (K + kps - 1) / kps;
    if (splits > 1 && !accumulate) return emu_err(CMF_E_ARG, "cmf_emu_gemm: split-K needs accumulate=1");
    dim3 grid(M / TM, N / TN, splits);
    k_gemm<<<grid, 128, 0, (cudaStream_t)stream>>>(M, N, K, (const __nv_bfloat16 *)A, lda, transA, (const __nv_bfloat16 *)B,
                                                  ldb, transB, C, ldc, (__nv_bfloat16 *)Cb, ldcb, bias, relu, accumulate, kps);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_relu_bwd(int n, const float *dA, const void *act, void *dZ, float *dZf, void *stream) {
    k_relu_bwd<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, dA, (const __nv_bfloat16 *)act, (__nv_bfloat16 *)dZ, dZf);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_mse_grad(int rows, int valid, int ldy, const float *Y, const float *t, float *dY, void *dYb, float *loss_part,
                     void *stream) {
    k_mse_grad<<<(rows + 255) / 256, 256, 0, (cudaStream_t)stream>>>(rows, valid, ldy, Y, t, dY, (__nv_bfloat16 *)dYb, loss_part);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_colsum(int rows, int cols, const float *X, float *out, void *stream) {
    k_colsum<<<cols, 256, 0, (cudaStream_t)stream>>>(rows, cols, X, out);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_adam(int n, float *w, void *wb, const float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
                 int step, float wd, void *stream) {
    const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, w, (__nv_bfloat16 *)wb, grad, m, v, lr, b1, b2, eps, bc1, bc2, wd);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

size_t cmf_emu_mlp_pack_bytes(void) { return (size_t)kMlpPackWords * sizeof(uint2); }

int cmf_emu_mlp_pack(const void *W0, const void *W1, const void *W2, const void *W3, int ldw3, void *pack, void *stream) {
    if (!W0 || !W1 || !W2 || !W3 || !pack || ldw3 < 8) return emu_err(CMF_E_ARG, "cmf_emu_mlp_pack: bad arguments");
    k_mlp_pack<<<(kMlpPackWords + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16 *)W0, (const __nv_bfloat16 *)W1, (const __nv_bfloat16 *)W2, (const __nv_bfloat16 *)W3, ldw3,
        (uint2 *)pack);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_mlp_fused(const void *X, int ldx, int rows, const void *pack, const float *b0, const float *b1, const float *b2,
                      const float *b3, float *y, void *stream) {
    if (!X || !pack || !b0 || !b1 || !b2 || !b3 || !y || ldx < 32 || (ldx & 1) || rows < 0 || rows % 16)
        return emu_err(CMF_E_ARG, "cmf_emu_mlp_fused: bad arguments (ldx >= 32 and even, rows % 16 == 0)");
    if (((uintptr_t)X & 3) || ((uintptr_t)pack & 7)) return emu_err(CMF_E_ARG, "cmf_emu_mlp_fused: misaligned X or pack");
    if (rows == 0) return CMF_OK;
    int dev = 0, sms = 0;
    EMU_TRY(cudaGetDevice(&dev));
    EMU_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int smem = (int)cmf_emu_mlp_pack_bytes();
    EMU_TRY(cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int ntiles = (rows + kMlpRowsPerCta - 1) / kMlpRowsPerCta;
    const int grid = ntiles < 2 * sms ? ntiles : 2 * sms;
    k_mlp_fused<<<grid, kMlpThreads, smem, (cudaStream_t)stream>>>((const __nv_bfloat16 *)X, ldx, rows, (const uint2 *)pack,
                                                                   b0, b1, b2, b3, y);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

size_t cmf_emu_mlp_tc_pack_bytes(void) { return (size_t)kTcWBytes; }

int cmf_emu_mlp_tc_pack(const void *W0, const void *W1, const void *W2, const void *W3, int ldw3, void *pack, void *stream) {
    if (!W0 || !W1 || !W2 || !W3 || !pack || ldw3 < 16 || ((uintptr_t)pack & 15))
        return emu_err(CMF_E_ARG, "cmf_emu_mlp_tc_pack: bad arguments (ldw3 >= 16, pack 16-byte aligned)");
    const int n = 128 * 32 + 2 * 128 * 128 + 16 * 128;
    k_mlp_tc_pack<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16 *)W0, (const __nv_bfloat16 *)W1, (const __nv_bfloat16 *)W2, (const __nv_bfloat16 *)W3, ldw3,
        (__nv_bfloat16 *)pack);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_mlp_tc(const void *X, int ldx, int rows, const void *pack, const float *b0, const float *b1, const float *b2,
                   const float *b3, float *y, void *stream) {
    if (!X || !pack || !b0 || !b1 || !b2 || !b3 || !y || ldx < 32 || (ldx % 8) || rows < 0)
        return emu_err(CMF_E_ARG, "cmf_emu_mlp_tc: bad arguments (ldx >= 32 and a multiple of 8)");
    if (((uintptr_t)X & 15) || ((uintptr_t)pack & 15)) return emu_err(CMF_E_ARG, "cmf_emu_mlp_tc: X and pack must be 16-byte aligned");
    if (rows == 0) return CMF_OK;
    int dev = 0, sms = 0, major = 0;
    EMU_TRY(cudaGetDevice(&dev));
    EMU_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) return emu_err(CMF_E_NO_DEVICE, "cmf_emu_mlp_tc: needs an sm_100 device");
    EMU_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    EMU_TRY(cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    const int ntiles = (rows + kTcRows - 1) / kTcRows;
    const int want = (ntiles + kTcSlots - 1) / kTcSlots;
    const int grid = want < sms ? want : sms;
    k_mlp_tc<<<grid, kTcThreads, kTcSmem, (cudaStream_t)stream>>>((const __nv_bfloat16 *)X, ldx, rows, (const uint4 *)pack,
                                                                  b0, b1, b2, b3, y, g_tc_wait_limit);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_mlp_tc_status(void) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_mlp_tc_status, sizeof v) != cudaSuccess) return emu_err(CMF_E_CUDA, "cmf_emu_mlp_tc_status: read failed");
    if (!v) return CMF_OK;
    const int zero = 0;                                       // clear on read: the next check starts clean
    if (cudaMemcpyToSymbol(g_mlp_tc_status, &zero, sizeof zero) != cudaSuccess)
        return emu_err(CMF_E_CUDA, "cmf_emu_mlp_tc_status: reset failed");
    return emu_err(CMF_E_CUDA, "cmf_emu_mlp_tc: an MMA completion wait ran out its bound (the kernel returned early)");
}

int cmf_emu_mlp_tc_set_wait_limit(int32_t limit) {
    g_tc_wait_limit = limit < 0 ? kTcWaitLimit : limit;
    return CMF_OK;
}

// Features of every member: X rows [M][rows_per_member][ldx] bf16 (columns 0..31 written);
// planes: fp32 [2 * (hops + 1)][M * N] scratch for the message passes.
int cmf_emu_features(const cmf_emu_net *net, const cmf_emu_member *mb, int nmembers, void *X, int ldx, int rows_per_member,
                     int hops, float *planes, void *stream) {
    if (!net || !mb || !X || !planes || hops < 0 || hops > 8 || ldx < 32 || (ldx % 8) || nmembers < 1 ||
        rows_per_member < net->nseqall || ((uintptr_t)X & 15) || !net->rivman)
        return emu_err(CMF_E_ARG, "cmf_emu_features: bad arguments (hops <= 8, ldx % 8 == 0, X 16-byte aligned)");
    EmuNet n{net->nseqall, net->nseqriv, net->next, net->up_ptr, net->up_idx, net->rivelv, net->elevtn, net->nxtdst,
             net->rivwth, net->rivhgt, net->rivlen, net->rivstomax, net->qref, net->rivman, net->pmanfld};
    cudaStream_t st = (cudaStream_t)stream;
    const dim3 blocks((n.N + 255) / 256, nmembers);
    const size_t plane = (size_t)nmembers * n.N;
    auto pl = [&](int k) { return planes + (size_t)k * plane; };   // hop h: planes 2h+2 (outflow), 2h+3 (runoff)
    int h = 0;
    if (hops >= 2) {
        k_emu_hop2<true><<<blocks, 256, 0, st>>>(n, nullptr, nullptr, mb->qprev, mb->runoff, pl(2), pl(3), pl(4), pl(5));
        h = 2;
    } else if (hops == 1) {
        k_emu_seed<<<blocks, 256, 0, st>>>(n, mb->qprev, mb->runoff, pl(0), pl(1));
        k_emu_hop<<<blocks, 256, 0, st>>>(n, pl(0), pl(1), pl(2), pl(3));
        h = 1;
    }
    for (; h + 2 <= hops; h += 2)
        k_emu_hop2<false><<<blocks, 256, 0, st>>>(n, pl(2 * h), pl(2 * h + 1), nullptr, nullptr, pl(2 * h + 2),
                                                  pl(2 * h + 3), pl(2 * h + 4), pl(2 * h + 5));
    if (h < hops) k_emu_hop<<<blocks, 256, 0, st>>>(n, pl(2 * h), pl(2 * h + 1), pl(2 * h + 2), pl(2 * h + 3));
    k_emu_assemble<<<blocks, 256, 0, st>>>(n, mb->rivsto, mb->fldsto, mb->levsto, mb->rivdph, mb->flddph, mb->fldfrc,
                                           mb->qprev, mb->runoff, planes, plane, hops, (__nv_bfloat16 *)X, ldx,
                                           rows_per_member);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

int cmf_emu_rollout(const cmf_emu_net *net, const cmf_emu_member *mb, int nmembers, const int *active_dev, const float *y,
                    int ldy, int rows_per_member, double dt, int residual, double *qout, void *stream) {
    if (!net || !mb || !y || !qout || !active_dev || nmembers < 1) return emu_err(CMF_E_ARG, "cmf_emu_rollout: null argument");
    EmuNet n{net->nseqall, net->nseqriv, net->next, net->up_ptr, net->up_idx, net->rivelv, net->elevtn, net->nxtdst,
             net->rivwth, net->rivhgt, net->rivlen, net->rivstomax, net->qref, net->rivman, net->pmanfld};
    cudaStream_t st = (cudaStream_t)stream;
    const dim3 blocks((n.N + 255) / 256, nmembers);
    k_emu_rollout<<<blocks, 256, 0, st>>>(n, y, ldy, rows_per_member, active_dev, dt, residual, mb->runoff, mb->rivsto, mb->fldsto,
                                          mb->levsto, mb->qprev, qout);
    k_emu_update<<<blocks, 256, 0, st>>>(n, active_dev, dt, mb->runoff, qout, mb->rivsto, mb->fldsto, mb->levsto,
                                         mb->rivout_pre, mb->fldout_pre, mb->qprev);
    EMU_TRY(cudaGetLastError());
    return CMF_OK;
}

}  // extern "C"
