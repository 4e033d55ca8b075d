// Learned surrogate of the E3B three-body forces (no reference counterpart;
// the exact term is ThreeBodyE3B.h:255-549 / EvaluatorE3B.h:145-345, which
// stays the fallback and the measure of the surrogate's force error).
//
// Model.  For molecule m a right-handed frame (e1 along the H-O-H bisector,
// e2 toward H1, e3 = e1 x e2) and 128 rotation-invariant features: four
// channels (O_m->O_j, O_m->H_j, H1_m->O_j, H2_m->O_j over the molecules j of
// the E3B molecule list), eight Gaussian radial shells per channel under a
// cosine cutoff of 5.6 A, and per shell the sum of the weights and of the
// weighted unit vectors in m's frame.  Standardised features go through an MLP
// 128 -> 64 -> 64 -> 64 -> 9 (SiLU) whose outputs are the three-body forces on
// O, H1 and H2 of m in m's frame (scaled by the training set's force RMS);
// they are rotated back to the lab frame.  Forces are not conservative (a
// regression surrogate, scored by force RMSE); the exact O-O two-body term is
// kept.
//
// Arithmetic.  Every GEMM uses BF16 operands with FP32 accumulation on the
// tensor cores (mma.sync m16n8k16 bf16): the inference kernel keeps the 64-wide
// activations in registers between layers; training (forward, backward and
// Adam on FP32 master weights) is a chain of the same GEMM kernel and small
// element-wise kernels, all hand-written here.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include <cstring>

#include "engine.hpp"

namespace mdx {

namespace {

using S = E3BSurrogate;
constexpr int kTeam = 8;      // lanes per molecule in the feature kernel
constexpr int kListTeam = kE3BTeam;  // team layout of the E3B molecule list
constexpr float kCut = 5.6f;  // feature cutoff (A)
constexpr float kPi = 3.14159265358979f;

// radial shells: channel 0 (O-O) centres 2.4 + 0.4 b, width 0.4; channels
// 1-3 (O-H, H-O) centres 1.5 + 0.5 b, width 0.5
__device__ __forceinline__ float shell_mu(int c, int b) { return c == 0 ? 2.4f + 0.4f * b : 1.5f + 0.5f * b; }
__device__ __forceinline__ float shell_gamma(int c) { return c == 0 ? 3.125f : 2.0f; }

struct FeatArgs {
    int nmol;
    const int4 *mol_idx;
    const float4 *xs;
    const uint32_t *mcounts, *mlist;
    int mcap;
    Box box;
    const float *mean, *inv_std;
    __nv_bfloat16 *feat;  // standardised BF16 [nmol_pad x kIn] (may be null)
    float *raw;           // raw FP32 [nmol x kIn] (may be null)
    float4 *frame;        // [3 nmol]: e1, e2, e3
};

__device__ __forceinline__ float3 nrm(float3 v) { return v * rsqrtf(dot3(v, v)); }

__device__ __forceinline__ void mol_frame(const float3 o, const float3 h1, const float3 h2, float3 &e1, float3 &e2,
                                          float3 &e3) {
    const float3 a = h1 - o, b = h2 - o;
    e1 = nrm(a + b);
    float3 d = a - b;
    d = d - e1 * dot3(d, e1);
    e2 = nrm(d);
    e3 = make_float3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x);
}

// lane t of the team: channel t / 2, shells 4 (t % 2) .. 4 (t % 2) + 3
__global__ void k_features(const FeatArgs A) {
    constexpr int G = 32 / kTeam;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / kTeam, t = lane % kTeam;
    const int m = warp * G + a;
    if (m >= A.nmol) return;  // team-uniform; no shuffles below
    const int ch = t >> 1, b0 = 4 * (t & 1);
    const int4 ix = A.mol_idx[m];
    const float3 o = f3(A.xs[ix.x]);
    const float3 h1 = o + min_image(A.box, f3(A.xs[ix.y]) - o);
    const float3 h2 = o + min_image(A.box, f3(A.xs[ix.z]) - o);
    float3 e1, e2, e3;
    mol_frame(o, h1, h2, e1, e2, e3);
    const float3 src = ch == 2 ? h1 : (ch == 3 ? h2 : o);
    float acc[4][4];
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
        for (int k = 0; k < 4; k++) acc[b][k] = 0.f;
    const float gam = shell_gamma(ch);
    float mu[4];
#pragma unroll
    for (int b = 0; b < 4; b++) mu[b] = shell_mu(ch, b0 + b);
    int cnt = (int)A.mcounts[m];
    cnt = cnt < A.mcap ? cnt : A.mcap;
    constexpr int GL = 32 / kListTeam;
    const uint32_t *row = A.mlist + (size_t)(m / GL) * A.mcap * GL + (m % GL) * kListTeam;
    for (int k = 0; k < cnt; k++) {
        const int mj = (int)row[(size_t)(k / kListTeam) * 32 + (k % kListTeam)];
        const int4 jx = A.mol_idx[mj];
        const int nv = ch == 1 ? 2 : 1;
        for (int v = 0; v < nv; v++) {
            const int tgt = ch == 1 ? (v == 0 ? jx.y : jx.z) : jx.x;
            const float3 d = min_image(A.box, f3(A.xs[tgt]) - src);
            const float r2 = dot3(d, d);
            if (r2 >= kCut * kCut || r2 < 1e-6f) continue;
            const float r = sqrtf(r2);
            const float ir = 1.0f / r;
            const float u1 = dot3(d, e1) * ir, u2 = dot3(d, e2) * ir, u3 = dot3(d, e3) * ir;
            const float fc = 0.5f * (cosf(kPi * r / kCut) + 1.0f);
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const float x = r - mu[b];
                const float g = expf(-gam * x * x) * fc;
                acc[b][0] += g;
                acc[b][1] += g * u1;
                acc[b][2] += g * u2;
                acc[b][3] += g * u3;
            }
        }
    }
    const int base = ch * 32 + b0 * 4;
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int f = base + b * 4 + k;
            const float v = acc[b][k];
            if (A.raw) A.raw[(size_t)m * S::kIn + f] = v;
            if (A.feat) A.feat[(size_t)m * S::kIn + f] = __float2bfloat16((v - A.mean[f]) * A.inv_std[f]);
        }
    if (t == 0) {
        A.frame[3 * m] = make_float4(e1.x, e1.y, e1.z, 0.f);
        A.frame[3 * m + 1] = make_float4(e2.x, e2.y, e2.z, 0.f);
        A.frame[3 * m + 2] = make_float4(e3.x, e3.y, e3.z, 0.f);
    }
}

// exact three-body forces of O, H1, H2 rotated into the molecule frame
__global__ void k_targets(int nmol, const int4 *__restrict__ mol_idx, const float4 *__restrict__ frame,
                          const float4 *__restrict__ f, float *__restrict__ Y) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    const int4 ix = mol_idx[m];
    const float3 e1 = f3(frame[3 * m]), e2 = f3(frame[3 * m + 1]), e3 = f3(frame[3 * m + 2]);
    const int at[3] = {ix.x, ix.y, ix.z};
    float *y = Y + (size_t)m * S::kOut;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float3 F = f3(f[at[k]]);
        y[3 * k] = dot3(F, e1);
        y[3 * k + 1] = dot3(F, e2);
        y[3 * k + 2] = dot3(F, e3);
    }
    for (int k = 9; k < S::kOut; k++) y[k] = 0.f;
}

// per-feature mean and 1/std over the dataset (FP64 sums); one block of 256 per feature
__global__ void k_stats(size_t n, const float *__restrict__ X, float *__restrict__ mean, float *__restrict__ inv_std) {
    __shared__ double s1[256], s2[256];
    const int f = blockIdx.x;
    double a = 0.0, b = 0.0;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = X[i * S::kIn + f];
        a += v;
        b += v * v;
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double mu = s1[0] / (double)n;
        const double var = s2[0] / (double)n - mu * mu;
        mean[f] = (float)mu;
        inv_std[f] = var > 1e-12 ? (float)(1.0 / sqrt(var)) : 1.0f;
    }
}

// sum of squares of the targets (FP64) for the force scale; blocks of 256
__global__ void k_target_ss(size_t n, const float *__restrict__ Y, double *out) {
    __shared__ double sh[256];
    double a = 0.0;
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n * 9; i += (size_t)gridDim.x * blockDim.x) {
        const double v = Y[(i / 9) * S::kOut + i % 9];
        a += v * v;
    }
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, sh[0]);
}

// minibatch: row i of the batch is dataset row hash(seed, i) % n; features
// standardised to BF16, targets scaled
__global__ void k_gather_batch(int B, size_t n, uint64_t seed, const float *__restrict__ X, const float *__restrict__ Y,
                               const float *__restrict__ mean, const float *__restrict__ inv_std, float inv_scale,
                               __nv_bfloat16 *__restrict__ xb, float *__restrict__ yb) {
    const int i = blockIdx.x;
    uint64_t h = seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(i + 1));
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    const size_t r = h % n;
    for (int f = threadIdx.x; f < S::kIn; f += blockDim.x)
        xb[(size_t)i * S::kIn + f] = __float2bfloat16((X[r * S::kIn + f] - mean[f]) * inv_std[f]);
    for (int k = threadIdx.x; k < S::kOut; k += blockDim.x)
        yb[(size_t)i * S::kOut + k] = k < 9 ? Y[r * S::kOut + k] * inv_scale : 0.f;
}

// ---- GEMM: C[M x N] (+)= A[M x K] * B[K x N], BF16 operands, FP32 accumulation
// A(i, k) = A[i sa_i + k sa_k], B(k, j) = B[k sb_k + j sb_j]; M % 64 == 0,
// N % 8 == 0, K % 16 == 0 (K split over gridDim.z, partial sums added
// atomically when atomic != 0).  Block: 4 warps x 16 rows, 32 columns.
struct GemmArgs {
    int M, N, K;
    const __nv_bfloat16 *A;
    long long sa_i, sa_k;
    const __nv_bfloat16 *B;
    long long sb_k, sb_j;
    float *C;
    int ldc;
    const float *bias;  // added once (split 0), may be null
    int atomic;
};

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) k_gemm(const GemmArgs g) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    const int m0 = blockIdx.y * 64 + 16 * w;
    const int n0 = blockIdx.x * 32;
    const int ksplit = gridDim.z;
    const int kchunk = ((g.K / 16 + ksplit - 1) / ksplit) * 16;
    const int kb = blockIdx.z * kchunk, ke = min(g.K, kb + kchunk);
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[j][q] = 0.f;
    auto Aat = [&](int i, int k) { return g.A[(long long)i * g.sa_i + (long long)k * g.sa_k]; };
    auto Bat = [&](int k, int j) { return g.B[(long long)k * g.sb_k + (long long)j * g.sb_j]; };
    for (int k0 = kb; k0 < ke; k0 += 16) {
        uint32_t af[4];
        af[0] = pack2(Aat(m0 + gq, k0 + 2 * tq), Aat(m0 + gq, k0 + 2 * tq + 1));
        af[1] = pack2(Aat(m0 + gq + 8, k0 + 2 * tq), Aat(m0 + gq + 8, k0 + 2 * tq + 1));
        af[2] = pack2(Aat(m0 + gq, k0 + 2 * tq + 8), Aat(m0 + gq, k0 + 2 * tq + 9));
        af[3] = pack2(Aat(m0 + gq + 8, k0 + 2 * tq + 8), Aat(m0 + gq + 8, k0 + 2 * tq + 9));
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int nc = n0 + 8 * j;
            if (nc >= g.N) continue;
            uint32_t bf[2];
            bf[0] = pack2(Bat(k0 + 2 * tq, nc + gq), Bat(k0 + 2 * tq + 1, nc + gq));
            bf[1] = pack2(Bat(k0 + 2 * tq + 8, nc + gq), Bat(k0 + 2 * tq + 9, nc + gq));
            mma_bf16(acc[j], af, bf);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int col = n0 + 8 * j + 2 * tq;
        if (n0 + 8 * j >= g.N) continue;
        float b0 = 0.f, b1 = 0.f;
        if (g.bias && blockIdx.z == 0) {
            b0 = g.bias[col];
            b1 = g.bias[col + 1];
        }
        float *r0 = g.C + (size_t)(m0 + gq) * g.ldc + col;
        float *r1 = g.C + (size_t)(m0 + gq + 8) * g.ldc + col;
        if (g.atomic) {
            atomicAdd(r0, acc[j][0] + b0);
            atomicAdd(r0 + 1, acc[j][1] + b1);
            atomicAdd(r1, acc[j][2] + b0);
            atomicAdd(r1 + 1, acc[j][3] + b1);
        } else {
            r0[0] = acc[j][0] + b0;
            r0[1] = acc[j][1] + b1;
            r1[0] = acc[j][2] + b0;
            r1[1] = acc[j][3] + b1;
        }
    }
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

__global__ void k_silu(size_t n, const float *__restrict__ z, __nv_bfloat16 *__restrict__ a) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = __float2bfloat16(silu(z[i]));
}

// output gradient of the mean squared error over the 9 used outputs; loss sum
// (blocks of 256)
__global__ void k_out_grad(int B, const float *__restrict__ y, const float *__restrict__ t,
                           __nv_bfloat16 *__restrict__ dz, double *loss) {
    __shared__ double sh[256];
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < (size_t)B * S::kOut) {
        const int k = (int)(i % S::kOut);
        float g = 0.f;
        if (k < 9) {
            const float d = y[i] - t[i];
            l = (double)d * d;
            g = 2.0f * d / (float)(B * 9);
        }
        dz[i] = __float2bfloat16(g);
    }
    sh[threadIdx.x] = l;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, sh[0]);
}

__global__ void k_silu_back(size_t n, const float *__restrict__ da, const float *__restrict__ z,
                            __nv_bfloat16 *__restrict__ dz) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dz[i] = __float2bfloat16(da[i] * dsilu(z[i]));
}

// bias gradient: column sums of dz [B x N]
__global__ void k_colsum(int B, int N, const __nv_bfloat16 *__restrict__ dz, float *__restrict__ db) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    float s = 0.f;
    for (int i = 0; i < B; i++) s += __bfloat162float(dz[(size_t)i * N + j]);
    db[j] += s;
}

__global__ void k_adam(int n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float c1, float c2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_to_bf16(int n, const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16(w[i]);
}

// ---- inference: one warp per 16 molecules, weights in shared memory,
// activations kept in registers between layers (the m16n8k16 accumulator
// layout of two adjacent n-tiles is the A-operand layout of one k-tile)
struct InferArgs {
    int nmol;
    const __nv_bfloat16 *feat;  // [nmol_pad x kIn]
    const __nv_bfloat16 *wb;    // bf16 weights (blob offsets)
    const float *w;             // fp32 blob (biases)
    const float4 *frame;
    const int4 *mol_idx;
    float scale;
    float4 *out;  // forces: O gets +=, H1/H2 stored (side-buffer semantics)
    float *yraw;  // optional [nmol_pad x kOut] model outputs
    int add_o;
};

constexpr int kInferWarps = 4;

template <int KT, int NT>
__device__ __forceinline__ void layer(const uint32_t (&a)[KT][4], const __nv_bfloat16 *W, int ldw, const float *bias,
                                      float (&c)[NT][4], int lane) {
    const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int j = 0; j < NT; j++) {
        const float b0 = bias[8 * j + 2 * tq], b1 = bias[8 * j + 2 * tq + 1];
        c[j][0] = b0;
        c[j][1] = b1;
        c[j][2] = b0;
        c[j][3] = b1;
    }
#pragma unroll
    for (int k = 0; k < KT; k++) {
#pragma unroll
        for (int j = 0; j < NT; j++) {
            const int kr = 16 * k + 2 * tq, nc = 8 * j + gq;
            uint32_t bf[2];
            bf[0] = pack2(W[kr * ldw + nc], W[(kr + 1) * ldw + nc]);
            bf[1] = pack2(W[(kr + 8) * ldw + nc], W[(kr + 9) * ldw + nc]);
            mma_bf16(c[j], a[k], bf);
        }
    }
}

template <int NT>
__device__ __forceinline__ void to_afrag(const float (&c)[NT][4], uint32_t (&a)[NT / 2][4]) {
#pragma unroll
    for (int k = 0; k < NT / 2; k++) {
        a[k][0] = pack2(__float2bfloat16(silu(c[2 * k][0])), __float2bfloat16(silu(c[2 * k][1])));
        a[k][1] = pack2(__float2bfloat16(silu(c[2 * k][2])), __float2bfloat16(silu(c[2 * k][3])));
        a[k][2] = pack2(__float2bfloat16(silu(c[2 * k + 1][0])), __float2bfloat16(silu(c[2 * k + 1][1])));
        a[k][3] = pack2(__float2bfloat16(silu(c[2 * k + 1][2])), __float2bfloat16(silu(c[2 * k + 1][3])));
    }
}

__global__ void __launch_bounds__(kInferWarps * 32) k_mlp_infer(const InferArgs A) {
    __shared__ __nv_bfloat16 sw[S::kOffB4];      // weights (bias slots unused)
    __shared__ float sb[3 * S::kHid + S::kOut];  // b1, b2, b3, b4
    __shared__ float sy[kInferWarps][16][S::kOut];
    for (int i = threadIdx.x; i < S::kOffB4; i += blockDim.x) sw[i] = A.wb[i];
    for (int i = threadIdx.x; i < 3 * S::kHid + S::kOut; i += blockDim.x) {
        const int l = i / S::kHid;
        const int off = l == 0 ? S::kOffB1 : (l == 1 ? S::kOffB2 : (l == 2 ? S::kOffB3 : S::kOffB4));
        sb[i] = A.w[off + i - l * S::kHid];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    const int r0 = (blockIdx.x * kInferWarps + w) * 16;
    if (r0 >= A.nmol) return;  // warp-uniform, after the only block barrier
    uint32_t x[8][4];
    const __nv_bfloat16 *F = A.feat + (size_t)r0 * S::kIn;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int c = 16 * k + 2 * tq;
        x[k][0] = pack2(F[gq * S::kIn + c], F[gq * S::kIn + c + 1]);
        x[k][1] = pack2(F[(gq + 8) * S::kIn + c], F[(gq + 8) * S::kIn + c + 1]);
        x[k][2] = pack2(F[gq * S::kIn + c + 8], F[gq * S::kIn + c + 9]);
        x[k][3] = pack2(F[(gq + 8) * S::kIn + c + 8], F[(gq + 8) * S::kIn + c + 9]);
    }
    float c1[8][4];
    layer<8, 8>(x, sw + S::kOffW1, S::kHid, sb, c1, lane);
    uint32_t a1[4][4];
    to_afrag<8>(c1, a1);
    float c2[8][4];
    layer<4, 8>(a1, sw + S::kOffW2, S::kHid, sb + S::kHid, c2, lane);
    uint32_t a2[4][4];
    to_afrag<8>(c2, a2);
    float c3[8][4];
    layer<4, 8>(a2, sw + S::kOffW3, S::kHid, sb + 2 * S::kHid, c3, lane);
    uint32_t a3[4][4];
    to_afrag<8>(c3, a3);
    float c4[2][4];
    layer<4, 2>(a3, sw + S::kOffW4, S::kOut, sb + 3 * S::kHid, c4, lane);
#pragma unroll
    for (int j = 0; j < 2; j++) {
        sy[w][gq][8 * j + 2 * tq] = c4[j][0];
        sy[w][gq][8 * j + 2 * tq + 1] = c4[j][1];
        sy[w][gq + 8][8 * j + 2 * tq] = c4[j][2];
        sy[w][gq + 8][8 * j + 2 * tq + 1] = c4[j][3];
    }
    __syncwarp();
    if (lane < 16) {
        const int m = r0 + lane;
        if (A.yraw)
            for (int k = 0; k < S::kOut; k++) A.yraw[(size_t)m * S::kOut + k] = sy[w][lane][k];
        if (m < A.nmol && A.out) {
            const float3 e1 = f3(A.frame[3 * m]), e2 = f3(A.frame[3 * m + 1]), e3 = f3(A.frame[3 * m + 2]);
            const int4 ix = A.mol_idx[m];
            const float *y = sy[w][lane];
            const float s = A.scale;
            const float3 fo = (e1 * y[0] + e2 * y[1] + e3 * y[2]) * s;
            const float3 fh1 = (e1 * y[3] + e2 * y[4] + e3 * y[5]) * s;
            const float3 fh2 = (e1 * y[6] + e2 * y[7] + e3 * y[8]) * s;
            float4 o = A.add_o ? A.out[ix.x] : make_float4(0.f, 0.f, 0.f, 0.f);
            A.out[ix.x] = make_float4(o.x + fo.x, o.y + fo.y, o.z + fo.z, 0.f);
            A.out[ix.y] = make_float4(fh1.x, fh1.y, fh1.z, 0.f);
            A.out[ix.z] = make_float4(fh2.x, fh2.y, fh2.z, 0.f);
        }
    }
}

__global__ void k_add_forces(int nmol, const int4 *__restrict__ mol_idx, const float4 *__restrict__ src,
                             float4 *__restrict__ fs) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    const int4 ix = mol_idx[m];
    const int at[3] = {ix.x, ix.y, ix.z};
    for (int k = 0; k < 3; k++) {
        const float4 a = src[at[k]];
        float4 f = fs[at[k]];
        f.x += a.x;
        f.y += a.y;
        f.z += a.z;
        fs[at[k]] = f;
    }
}

// |surrogate - exact|^2 and |exact|^2 over O, H1, H2 of every molecule (FP64;
// blocks of 256)
__global__ void k_compare(int nmol, const int4 *__restrict__ mol_idx, const float4 *__restrict__ a,
                          const float4 *__restrict__ b, double *out) {
    __shared__ double s1[256], s2[256];
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    double d2 = 0.0, r2 = 0.0;
    if (m < nmol) {
        const int4 ix = mol_idx[m];
        const int at[3] = {ix.x, ix.y, ix.z};
        for (int k = 0; k < 3; k++) {
            const float4 x = a[at[k]], y = b[at[k]];
            const double dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
            d2 += dx * dx + dy * dy + dz * dz;
            r2 += (double)y.x * y.x + (double)y.y * y.y + (double)y.z * y.z;
        }
    }
    s1[threadIdx.x] = d2;
    s2[threadIdx.x] = r2;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(out, s1[0]);
        atomicAdd(out + 1, s2[0]);
    }
}

int pad16(int n) { return (n + 15) / 16 * 16; }

int sur_alloc(State &s, FixE3B &f) {
    if (!f.sur) f.sur.reset(new E3BSurrogate());
    S &u = *f.sur;
    const int nmol = (int)f.mol_ids.size();
    const int np = pad16(std::max(nmol, 1)) + 64;  // + a block of padding rows
    if (int e = u.feat.alloc((size_t)np * S::kIn)) return e;
    if (int e = u.raw.alloc((size_t)std::max(nmol, 1) * S::kIn)) return e;
    if (int e = u.frame.alloc(3 * (size_t)std::max(nmol, 1))) return e;
    if (int e = u.fexact.alloc(std::max(s.gpd.n, 1))) return e;
    if (!u.w.p) {
        if (int e = u.w.alloc(S::kParams)) return e;
        if (int e = u.wb.alloc(S::kParams)) return e;
        if (int e = u.grad.alloc(S::kParams)) return e;
        if (int e = u.adam_m.alloc(S::kParams)) return e;
        if (int e = u.adam_v.alloc(S::kParams)) return e;
        if (int e = u.mean.alloc(S::kIn)) return e;
        if (int e = u.inv_std.alloc(S::kIn)) return e;
        if (int e = u.loss.alloc(1)) return e;
        // He-uniform weights (output layer x 0.1), zero biases, seeded
        std::vector<float> h(S::kParams, 0.f);
        std::mt19937_64 rng(20261203);
        auto fill = [&](int off, int fan_in, int count, float gain) {
            const float lim = gain * std::sqrt(6.0f / (float)fan_in);
            std::uniform_real_distribution<float> U(-lim, lim);
            for (int i = 0; i < count; i++) h[off + i] = U(rng);
        };
        fill(S::kOffW1, S::kIn, S::kIn * S::kHid, 1.0f);
        fill(S::kOffW2, S::kHid, S::kHid * S::kHid, 1.0f);
        fill(S::kOffW3, S::kHid, S::kHid * S::kHid, 1.0f);
        fill(S::kOffW4, S::kHid, S::kHid * S::kOut, 0.1f);
        for (int j = 0; j < S::kHid; j++)
            for (int k = S::kOutUsed; k < S::kOut; k++) h[S::kOffW4 + j * S::kOut + k] = 0.f;
        MDX_CUDA_TRY(cudaMemcpy(u.w.p, h.data(), S::kParams * sizeof(float), cudaMemcpyHostToDevice));
        MDX_CUDA_TRY(cudaMemset(u.adam_m.p, 0, S::kParams * sizeof(float)));
        MDX_CUDA_TRY(cudaMemset(u.adam_v.p, 0, S::kParams * sizeof(float)));
        std::vector<float> z(S::kIn, 0.f), o(S::kIn, 1.f);
        MDX_CUDA_TRY(cudaMemcpy(u.mean.p, z.data(), S::kIn * sizeof(float), cudaMemcpyHostToDevice));
        MDX_CUDA_TRY(cudaMemcpy(u.inv_std.p, o.data(), S::kIn * sizeof(float), cudaMemcpyHostToDevice));
        k_to_bf16<<<(S::kParams + 255) / 256, 256, 0, s.stream>>>(S::kParams, u.w.p, u.wb.p);
        MDX_LAUNCHED();
    }
    return 0;
}

FeatArgs feat_args(State &s, FixE3B &f) {
    S &u = *f.sur;
    FeatArgs A{};
    A.nmol = (int)f.mol_ids.size();
    A.mol_idx = f.d_mol_idx.p;
    A.xs = s.gpd.xs.p;
    A.mcounts = f.mcounts.p;
    A.mlist = f.mlist.p;
    A.mcap = f.mcap;
    A.box = s.box;
    A.mean = u.mean.p;
    A.inv_std = u.inv_std.p;
    A.feat = u.feat.p;
    A.raw = nullptr;
    A.frame = u.frame.p;
    return A;
}

dim3 feat_blocks(int nmol) {
    const int warps = (nmol + (32 / kTeam) - 1) / (32 / kTeam);
    return dim3((warps * 32 + 255) / 256);
}

InferArgs infer_args(FixE3B &f, int nmol, float4 *out, int add_o) {
    S &u = *f.sur;
    InferArgs I{};
    I.nmol = nmol;
    I.feat = u.feat.p;
    I.wb = u.wb.p;
    I.w = u.w.p;
    I.frame = u.frame.p;
    I.mol_idx = f.d_mol_idx.p;
    I.scale = u.force_scale;
    I.out = out;
    I.yraw = nullptr;
    I.add_o = add_o;
    return I;
}

unsigned infer_blocks(int n) { return (unsigned)((pad16(n) / 16 + kInferWarps - 1) / kInferWarps); }

int gemm(cudaStream_t st, int M, int N, int K, const __nv_bfloat16 *A, long long sa_i, long long sa_k,
         const __nv_bfloat16 *B, long long sb_k, long long sb_j, float *C, int ldc, const float *bias, int ksplit) {
    if (M % 64 || N % 8 || K % 16) {
        set_error(MDX_ERR_ARG, "surrogate GEMM shape %d x %d x %d not tiled", M, N, K);
        return MDX_ERR_ARG;
    }
    GemmArgs g{M, N, K, A, sa_i, sa_k, B, sb_k, sb_j, C, ldc, bias, ksplit > 1 ? 1 : 0};
    k_gemm<<<dim3((N + 31) / 32, M / 64, ksplit), 128, 0, st>>>(g);
    MDX_LAUNCHED();
    return 0;
}

// forward + backward of one minibatch already in u.xb / u.yb (B rows);
// gradient into u.grad (zeroed here), loss sum into u.loss
int sur_fwd_bwd(S &u, int B, cudaStream_t st) {
    const int in[4] = {S::kIn, S::kHid, S::kHid, S::kHid};
    const int out[4] = {S::kHid, S::kHid, S::kHid, S::kOut};
    const int offW[4] = {S::kOffW1, S::kOffW2, S::kOffW3, S::kOffW4};
    const int offB[4] = {S::kOffB1, S::kOffB2, S::kOffB3, S::kOffB4};
    const __nv_bfloat16 *x = u.xb.p;
    for (int l = 0; l < 4; l++) {
        if (int e = gemm(st, B, out[l], in[l], x, in[l], 1, u.wb.p + offW[l], out[l], 1, u.z[l].p, out[l],
                         u.w.p + offB[l], 1))
            return e;
        if (l < 3) {
            const size_t n = (size_t)B * out[l];
            k_silu<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, u.z[l].p, u.act[l].p);
            MDX_LAUNCHED();
            x = u.act[l].p;
        }
    }
    MDX_CUDA_TRY(cudaMemsetAsync(u.grad.p, 0, S::kParams * sizeof(float), st));
    MDX_CUDA_TRY(cudaMemsetAsync(u.loss.p, 0, sizeof(double), st));
    {
        const size_t n = (size_t)B * S::kOut;
        k_out_grad<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(B, u.z[3].p, u.yb.p, u.dz.p, u.loss.p);
        MDX_LAUNCHED();
    }
    for (int l = 3; l >= 0; l--) {
        const __nv_bfloat16 *aprev = l == 0 ? u.xb.p : u.act[l - 1].p;
        // dW = aprev^T dz  [in x out], the batch dimension split over blocks
        const int ks = std::max(1, std::min(32, B / 256));
        if (int e = gemm(st, in[l], out[l], B, aprev, 1, in[l], u.dz.p, out[l], 1, u.grad.p + offW[l], out[l],
                         nullptr, ks))
            return e;
        k_colsum<<<(out[l] + 63) / 64, 64, 0, st>>>(B, out[l], u.dz.p, u.grad.p + offB[l]);
        MDX_LAUNCHED();
        if (l == 0) break;
        // da = dz W^T  [B x in]; dz(l-1) = da * silu'(z(l-1))
        if (int e = gemm(st, B, in[l], out[l], u.dz.p, out[l], 1, u.wb.p + offW[l], 1, out[l], u.da.p, in[l],
                         nullptr, 1))
            return e;
        const size_t n = (size_t)B * in[l];
        k_silu_back<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, u.da.p, u.z[l - 1].p, u.dz.p);
        MDX_LAUNCHED();
    }
    return 0;
}

int sur_batch_alloc(S &u, int B) {
    if (u.batch >= B) return 0;
    if (int e = u.xb.alloc((size_t)B * S::kIn)) return e;
    if (int e = u.yb.alloc((size_t)B * S::kOut)) return e;
    for (int l = 0; l < 3; l++)
        if (int e = u.act[l].alloc((size_t)B * S::kHid)) return e;
    for (int l = 0; l < 4; l++)
        if (int e = u.z[l].alloc((size_t)B * S::kHid)) return e;
    if (int e = u.dz.alloc((size_t)B * S::kHid)) return e;
    if (int e = u.da.alloc((size_t)B * S::kIn)) return e;
    u.batch = B;
    return 0;
}

FixE3B *e3b_of(mdx_fix *f) {
    if (!f || !f->f || f->f->kind != FixKind::E3B) return nullptr;
    return static_cast<FixE3B *>(f->f);
}

}  // namespace

// the surrogate's E3B forces of one step into the side buffer: exact two-body
// on O (stored), surrogate three-body added on O and stored on H1, H2
int surrogate_forces_to(State &s, FixE3B &f, float4 *out, cudaStream_t stream) {
    const int nmol = (int)f.mol_ids.size();
    if (nmol == 0) return 0;
    if (int e = e3b_twobody_to(s, f, out, stream)) return e;
    k_features<<<feat_blocks(nmol), 256, 0, stream>>>(feat_args(s, f));
    MDX_LAUNCHED();
    k_mlp_infer<<<infer_blocks(nmol), kInferWarps * 32, 0, stream>>>(infer_args(f, nmol, out, 1));
    MDX_LAUNCHED();
    return 0;
}

// FixE3B::compute with the surrogate on: the step's E3B forces added to fs
int surrogate_compute(State &s, FixE3B &f) {
    S &u = *f.sur;
    if (int e = surrogate_forces_to(s, f, u.fexact.p, s.stream)) return e;
    const int nmol = (int)f.mol_ids.size();
    k_add_forces<<<(nmol + 127) / 128, 128, 0, s.stream>>>(nmol, f.d_mol_idx.p, u.fexact.p, s.gpd.fs.p);
    MDX_LAUNCHED();
    return 0;
}

}  // namespace mdx

using namespace mdx;

static int need_prepared(mdx_state *st, FixE3B *f) {
    if (!st || !f) {
        set_error(MDX_ERR_ARG, "need a state and an E3B fix");
        return MDX_ERR_ARG;
    }
    if (!st->s->prepared || !f->prepared) {
        set_error(MDX_ERR_STATE, "call mdx_prepare first");
        return MDX_ERR_STATE;
    }
    return 0;
}

extern "C" {

// append the current frame (features + exact three-body forces in the molecule frames)
int mdx_e3b_surrogate_collect(mdx_state *st, mdx_fix *fix) {
    FixE3B *f = e3b_of(fix);
    if (int e = need_prepared(st, f)) return e;
    State &s = *st->s;
    if (int e = sur_alloc(s, *f)) return e;
    S &u = *f->sur;
    const int nmol = (int)f->mol_ids.size();
    if (u.n + nmol > u.cap) {
        size_t nc = std::max(u.cap * 2, u.n + nmol);
        nc = std::max(nc, (size_t)nmol * 16);
        DBuf<float> X2, Y2;
        if (int e = X2.alloc(nc * S::kIn)) return e;
        if (int e = Y2.alloc(nc * S::kOut)) return e;
        if (u.n) {
            MDX_CUDA_TRY(cudaMemcpyAsync(X2.p, u.X.p, u.n * S::kIn * sizeof(float), cudaMemcpyDeviceToDevice,
                                         s.stream));
            MDX_CUDA_TRY(cudaMemcpyAsync(Y2.p, u.Y.p, u.n * S::kOut * sizeof(float), cudaMemcpyDeviceToDevice,
                                         s.stream));
        }
        MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
        std::swap(u.X.p, X2.p);
        std::swap(u.X.n, X2.n);
        std::swap(u.Y.p, Y2.p);
        std::swap(u.Y.n, Y2.n);
        u.cap = nc;
    }
    if (int e = e3b_exact_to(s, *f, u.fexact.p, 0, s.stream)) return e;
    FeatArgs A = feat_args(s, *f);
    A.feat = nullptr;
    A.raw = u.X.p + u.n * S::kIn;
    k_features<<<feat_blocks(nmol), 256, 0, s.stream>>>(A);
    MDX_LAUNCHED();
    k_targets<<<(nmol + 127) / 128, 128, 0, s.stream>>>(nmol, f->d_mol_idx.p, u.frame.p, u.fexact.p,
                                                        u.Y.p + u.n * S::kOut);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    MDX_CUDA_TRY(cudaGetLastError());
    u.n += nmol;
    return 0;
}

int mdx_e3b_surrogate_dataset_size(mdx_fix *fix, int64_t *n) {
    FixE3B *f = e3b_of(fix);
    if (!f || !n) {
        set_error(MDX_ERR_ARG, "need an E3B fix");
        return MDX_ERR_ARG;
    }
    *n = f->sur ? (int64_t)f->sur->n : 0;
    return 0;
}

// standardisation statistics and force scale from the collected frames (first
// call), then `iters` Adam steps on minibatches of `batch` rows
int mdx_e3b_surrogate_train(mdx_state *st, mdx_fix *fix, int iters, int batch, float lr, uint64_t seed,
                            double *loss_first, double *loss_last) {
    FixE3B *f = e3b_of(fix);
    if (int e = need_prepared(st, f)) return e;
    State &s = *st->s;
    if (!f->sur || f->sur->n < 64) {
        set_error(MDX_ERR_STATE, "collect frames first (mdx_e3b_surrogate_collect)");
        return MDX_ERR_STATE;
    }
    if (iters < 0 || batch < 64 || batch % 64) {
        set_error(MDX_ERR_ARG, "batch must be a positive multiple of 64");
        return MDX_ERR_ARG;
    }
    S &u = *f->sur;
    cudaStream_t cs = s.stream;
    if (!u.stats) {
        k_stats<<<S::kIn, 256, 0, cs>>>(u.n, u.X.p, u.mean.p, u.inv_std.p);
        MDX_LAUNCHED();
        MDX_CUDA_TRY(cudaMemsetAsync(u.loss.p, 0, sizeof(double), cs));
        k_target_ss<<<148, 256, 0, cs>>>(u.n, u.Y.p, u.loss.p);
        MDX_LAUNCHED();
        double ss = 0.0;
        MDX_CUDA_TRY(cudaMemcpyAsync(&ss, u.loss.p, sizeof(double), cudaMemcpyDeviceToHost, cs));
        MDX_CUDA_TRY(cudaStreamSynchronize(cs));
        u.force_scale = (float)std::sqrt(ss / (double)(u.n * 9));
        if (!(u.force_scale > 0.f)) u.force_scale = 1.f;
        u.stats = true;
    }
    if (int e = sur_batch_alloc(u, batch)) return e;
    double lf = -1, ll = -1;
    for (int it = 0; it < iters; it++) {
        k_gather_batch<<<batch, 128, 0, cs>>>(batch, u.n, seed + 0x632BE59BD9B4E019ull * (uint64_t)(u.adam_t + 1),
                                              u.X.p, u.Y.p, u.mean.p, u.inv_std.p, 1.0f / u.force_scale, u.xb.p,
                                              u.yb.p);
        MDX_LAUNCHED();
        if (int e = sur_fwd_bwd(u, batch, cs)) return e;
        u.adam_t += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)u.adam_t), c2 = 1.f - std::pow(b2, (float)u.adam_t);
        k_adam<<<(S::kParams + 255) / 256, 256, 0, cs>>>(S::kParams, u.w.p, u.grad.p, u.adam_m.p, u.adam_v.p, lr, b1,
                                                        b2, c1, c2, 1e-8f);
        MDX_LAUNCHED();
        k_to_bf16<<<(S::kParams + 255) / 256, 256, 0, cs>>>(S::kParams, u.w.p, u.wb.p);
        MDX_LAUNCHED();
        if (it == 0 || it == iters - 1) {
            double l = 0.0;
            MDX_CUDA_TRY(cudaMemcpyAsync(&l, u.loss.p, sizeof(double), cudaMemcpyDeviceToHost, cs));
            MDX_CUDA_TRY(cudaStreamSynchronize(cs));
            l /= (double)batch * 9.0;
            if (it == 0) lf = l;
            ll = l;
        }
    }
    MDX_CUDA_TRY(cudaStreamSynchronize(cs));
    MDX_CUDA_TRY(cudaGetLastError());
    u.trained = true;
    if (loss_first) *loss_first = lf;
    if (loss_last) *loss_last = ll;
    return 0;
}

// surrogate on (1) / exact E3B (0) for the fix's force evaluations
int mdx_e3b_surrogate_enable(mdx_fix *fix, int on) {
    FixE3B *f = e3b_of(fix);
    if (!f) {
        set_error(MDX_ERR_ARG, "need an E3B fix");
        return MDX_ERR_ARG;
    }
    if (on && (!f->sur || !f->sur->trained)) {
        set_error(MDX_ERR_STATE, "the surrogate is not trained");
        return MDX_ERR_STATE;
    }
    if (f->sur) f->sur->enabled = on != 0;
    return 0;
}

// three-body force error of the surrogate on the current frame:
// rmse = sqrt(mean |F_sur - F_exact|^2), rms = sqrt(mean |F_exact|^2) over O, H1, H2
int mdx_e3b_surrogate_eval(mdx_state *st, mdx_fix *fix, double *rmse, double *rms) {
    FixE3B *f = e3b_of(fix);
    if (int e = need_prepared(st, f)) return e;
    if (!f->sur || !f->sur->trained) {
        set_error(MDX_ERR_STATE, "the surrogate is not trained");
        return MDX_ERR_STATE;
    }
    State &s = *st->s;
    S &u = *f->sur;
    const int nmol = (int)f->mol_ids.size();
    DBuf<float4> fs;
    DBuf<double> acc;
    if (int e = fs.alloc(s.gpd.n)) return e;
    if (int e = acc.alloc(2)) return e;
    MDX_CUDA_TRY(cudaMemsetAsync(fs.p, 0, s.gpd.n * sizeof(float4), s.stream));
    MDX_CUDA_TRY(cudaMemsetAsync(acc.p, 0, 2 * sizeof(double), s.stream));
    if (int e = e3b_exact_to(s, *f, u.fexact.p, 0, s.stream)) return e;
    k_features<<<feat_blocks(nmol), 256, 0, s.stream>>>(feat_args(s, *f));
    MDX_LAUNCHED();
    k_mlp_infer<<<infer_blocks(nmol), kInferWarps * 32, 0, s.stream>>>(infer_args(*f, nmol, fs.p, 0));
    MDX_LAUNCHED();
    k_compare<<<(nmol + 255) / 256, 256, 0, s.stream>>>(nmol, f->d_mol_idx.p, fs.p, u.fexact.p, acc.p);
    MDX_LAUNCHED();
    double h[2];
    MDX_CUDA_TRY(cudaMemcpyAsync(h, acc.p, sizeof(h), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    const double cnt = 3.0 * nmol;
    if (rmse) *rmse = std::sqrt(h[0] / cnt);
    if (rms) *rms = std::sqrt(h[1] / cnt);
    return 0;
}

// parameters: w (kParams floats), mean / inv_std (kIn floats), scale; any may be NULL
int mdx_e3b_surrogate_get_params(mdx_fix *fix, float *w, float *mean, float *inv_std, float *scale) {
    FixE3B *f = e3b_of(fix);
    if (!f || !f->sur || !f->sur->w.p) {
        set_error(MDX_ERR_STATE, "no surrogate on this fix (collect or set parameters first)");
        return MDX_ERR_STATE;
    }
    S &u = *f->sur;
    if (w) MDX_CUDA_TRY(cudaMemcpy(w, u.w.p, S::kParams * sizeof(float), cudaMemcpyDeviceToHost));
    if (mean) MDX_CUDA_TRY(cudaMemcpy(mean, u.mean.p, S::kIn * sizeof(float), cudaMemcpyDeviceToHost));
    if (inv_std) MDX_CUDA_TRY(cudaMemcpy(inv_std, u.inv_std.p, S::kIn * sizeof(float), cudaMemcpyDeviceToHost));
    if (scale) *scale = u.force_scale;
    return 0;
}

int mdx_e3b_surrogate_set_params(mdx_state *st, mdx_fix *fix, const float *w, const float *mean, const float *inv_std,
                                 float scale) {
    FixE3B *f = e3b_of(fix);
    if (int e = need_prepared(st, f)) return e;
    if (!w || !mean || !inv_std || !(scale > 0.f)) {
        set_error(MDX_ERR_ARG, "need weights, statistics and a positive scale");
        return MDX_ERR_ARG;
    }
    State &s = *st->s;
    if (int e = sur_alloc(s, *f)) return e;
    S &u = *f->sur;
    MDX_CUDA_TRY(cudaMemcpy(u.w.p, w, S::kParams * sizeof(float), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(u.mean.p, mean, S::kIn * sizeof(float), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(u.inv_std.p, inv_std, S::kIn * sizeof(float), cudaMemcpyHostToDevice));
    k_to_bf16<<<(S::kParams + 255) / 256, 256, 0, s.stream>>>(S::kParams, u.w.p, u.wb.p);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    u.force_scale = scale;
    u.stats = true;
    u.trained = true;
    return 0;
}

// raw features (nmol x kIn, FP32, molecule order of the fix) and frames
// (nmol x 9: e1, e2, e3) of the current positions
int mdx_e3b_surrogate_features(mdx_state *st, mdx_fix *fix, float *raw, float *frames) {
    FixE3B *f = e3b_of(fix);
    if (int e = need_prepared(st, f)) return e;
    State &s = *st->s;
    if (int e = sur_alloc(s, *f)) return e;
    S &u = *f->sur;
    const int nmol = (int)f->mol_ids.size();
    FeatArgs A = feat_args(s, *f);
    A.feat = nullptr;
    A.raw = u.raw.p;
    k_features<<<feat_blocks(nmol), 256, 0, s.stream>>>(A);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    // rows come per E3B molecule index; in the molecule form that index is the
    // slot, mapped back here to the fix's molecule order (FixRigid's maps)
    std::vector<int> row_of(nmol);
    for (int m = 0; m < nmol; m++) row_of[m] = m;
    if (s.mf.on) {
        std::vector<int4> mi(nmol);
        MDX_CUDA_TRY(cudaMemcpy(mi.data(), s.rigidFix()->d_mol_idx.p, nmol * sizeof(int4), cudaMemcpyDeviceToHost));
        for (int m = 0; m < nmol; m++) row_of[m] = mi[m].x >> 2;
    }
    if (raw) {
        std::vector<float> h((size_t)nmol * S::kIn);
        MDX_CUDA_TRY(cudaMemcpy(h.data(), u.raw.p, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (int m = 0; m < nmol; m++)
            std::memcpy(raw + (size_t)m * S::kIn, h.data() + (size_t)row_of[m] * S::kIn, S::kIn * sizeof(float));
    }
    if (frames) {
        std::vector<float4> h(3 * (size_t)nmol);
        MDX_CUDA_TRY(cudaMemcpy(h.data(), u.frame.p, h.size() * sizeof(float4), cudaMemcpyDeviceToHost));
        for (int m = 0; m < nmol; m++)
            for (int c = 0; c < 3; c++) {
                const float4 v = h[3 * (size_t)row_of[m] + c];
                frames[9 * (size_t)m + 3 * c] = v.x;
                frames[9 * (size_t)m + 3 * c + 1] = v.y;
                frames[9 * (size_t)m + 3 * c + 2] = v.z;
            }
    }
    return 0;
}

// model outputs for n standardised feature rows given on the host (rounded to
// BF16 on upload): y (n x kOut)
int mdx_e3b_surrogate_infer(mdx_state *st, mdx_fix *fix, const float *x, int n, float *y) {
    FixE3B *f = e3b_of(fix);
    if (int e = need_prepared(st, f)) return e;
    if (!f->sur || !x || !y || n <= 0) {
        set_error(MDX_ERR_ARG, "need a surrogate, inputs and outputs");
        return MDX_ERR_ARG;
    }
    State &s = *st->s;
    S &u = *f->sur;
    const int np = pad16(n) + 64;
    std::vector<__nv_bfloat16> hb((size_t)np * S::kIn, __float2bfloat16(0.f));
    for (size_t i = 0; i < (size_t)n * S::kIn; i++) hb[i] = __float2bfloat16(x[i]);
    DBuf<__nv_bfloat16> xd;
    DBuf<float> yd;
    if (int e = xd.alloc(hb.size())) return e;
    if (int e = yd.alloc((size_t)np * S::kOut)) return e;
    MDX_CUDA_TRY(cudaMemcpy(xd.p, hb.data(), hb.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    InferArgs I = infer_args(*f, n, nullptr, 0);
    I.feat = xd.p;
    I.yraw = yd.p;
    I.w = u.w.p;
    k_mlp_infer<<<infer_blocks(n), kInferWarps * 32, 0, s.stream>>>(I);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    MDX_CUDA_TRY(cudaMemcpy(y, yd.p, (size_t)n * S::kOut * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

// loss (mean over n x 9) and gradient (kParams floats) of one minibatch given
// on the host: x standardised features (n x kIn), t scaled targets (n x kOut);
// n a multiple of 64.  No parameter update.
int mdx_e3b_surrogate_grad(mdx_state *st, mdx_fix *fix, const float *x, const float *t, int n, float *grad,
                           double *loss) {
    FixE3B *f = e3b_of(fix);
    if (int e = need_prepared(st, f)) return e;
    if (!f->sur || !x || !t || n <= 0 || n % 64) {
        set_error(MDX_ERR_ARG, "need a surrogate and n a positive multiple of 64");
        return MDX_ERR_ARG;
    }
    State &s = *st->s;
    S &u = *f->sur;
    if (int e = sur_batch_alloc(u, n)) return e;
    std::vector<__nv_bfloat16> hb((size_t)n * S::kIn);
    for (size_t i = 0; i < hb.size(); i++) hb[i] = __float2bfloat16(x[i]);
    MDX_CUDA_TRY(cudaMemcpy(u.xb.p, hb.data(), hb.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(u.yb.p, t, (size_t)n * S::kOut * sizeof(float), cudaMemcpyHostToDevice));
    if (int e = sur_fwd_bwd(u, n, s.stream)) return e;
    double l = 0.0;
    MDX_CUDA_TRY(cudaMemcpyAsync(&l, u.loss.p, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    if (grad) MDX_CUDA_TRY(cudaMemcpy(grad, u.grad.p, S::kParams * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l / ((double)n * 9.0);
    return 0;
}

}  // extern "C"
