// P3M reciprocal-space Ewald (FixChargeEwald, src/Fixes/FixChargeEwald.cu).
//
//  spread   map_charge_to_grid_order_5_cu (:174-217): order-5 charge
//           assignment W_p_5 (:163-172), float atomics into a REAL grid
//  FFT      cuFFT R2C (the reference runs C2C on a complex grid with a zero
//           imaginary part, :1307-1309; R2C computes the same half spectrum)
//  E(k)     E_field_cu (:386-434): E_d(k) = i k_d G(k) rho(k).  The reference
//           keeps only the real part after its C2C inverse, which drops the
//           anti-Hermitian Nyquist-plane term of each component; that term is
//           zeroed here so the C2R inverse gives the identical real field.
//  inverse  one batched cuFFT C2R for the three components (:1340-1346)
//  gather   Ewald_long_range_forces_order_5_cu (:561-630): F = Q q sum W E,
//           E = -ifft / V
//  G(k)     Green_function_cu (:314-366), evaluated once per box in FP64.
//  alpha    find_optimal_parameters (:848-967), secant on the RMS errors.
//
// Deviation (documented): the reference's nearest grid point is
// make_int3((x-lo+h/2)/h), a truncation toward zero, which mis-assigns the
// stencil of an atom more than h/2 below lo (atoms drift out of the box
// between list rebuilds); floorf is used here.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "engine.hpp"

namespace mdx {

namespace {

__device__ __forceinline__ void w5(float x, float w[5]) {
    const float x2 = x * x, x4 = x2 * x2;
    w[0] = (1.0f / 384.0f) * (1.0f - 8.0f * x + 24.0f * x2 - 32.0f * x * x2 + 16.0f * x4);
    w[1] = (1.0f / 96.0f) * (19.0f - 44.0f * x + 24.0f * x2 + 16.0f * x * x2 - 16.0f * x4);
    w[2] = (1.0f / 192.0f) * (115.0f - 120.0f * x2 + 48.0f * x4);
    w[3] = (1.0f / 96.0f) * (19.0f + 44.0f * x + 24.0f * x2 - 16.0f * x * x2 - 16.0f * x4);
    w[4] = (1.0f / 384.0f) * (1.0f + 8.0f * x + 24.0f * x2 + 32.0f * x * x2 + 16.0f * x4);
}

__device__ __forceinline__ int wrapi(int p, int n) {
    p %= n;
    return p < 0 ? p + n : p;
}

struct P3MGeom {
    int3 sz;
    float3 lo, h, invh;
    float qunit;
};

__device__ __forceinline__ void stencil(const P3MGeom &g, float4 x, int3 &ng, float3 &d) {
    const float px = x.x - g.lo.x, py = x.y - g.lo.y, pz = x.z - g.lo.z;
    ng.x = (int)floorf((px + 0.5f * g.h.x) / g.h.x);
    ng.y = (int)floorf((py + 0.5f * g.h.y) / g.h.y);
    ng.z = (int)floorf((pz + 0.5f * g.h.z) / g.h.z);
    d.x = px / g.h.x - (float)ng.x;
    d.y = py / g.h.y - (float)ng.y;
    d.z = pz / g.h.z - (float)ng.z;
}

// Arguments of the P3M kernels for one system: a0 (single system) or
// tab[blockIdx.y] (batched replicas; a0 then only sizes the grid).
struct P3MArgs {
    int n;
    const float4 *xs;
    const float *qs;
    float4 *fs;
    P3MGeom g;
    float *rho;
    const float2 *rho_k;
    float2 *e_k;
    const float *e_r;
    const float *green;
    float3 tpl;  // 2 pi / L
    size_t nk, ngrid;
    float niv;   // -1 / V
    // molecule form (all-rigid water): the charged sites of molecule m are
    // H1, H2, M of mol_idx[m] (four-site, uncharged O) or O, H1, H2
    const int4 *mol_idx;
    int nmol, four_site;
    int slots;  // 1: the molecule form's layout, molecule slot m at sites 4m .. 4m+3 (no map read)
    const float4 *e4;  // the own FFT's interleaved field (batched gather), or null
};
#define MDX_P3M_ARGS const P3MArgs A = tab ? tab[blockIdx.y] : a0

// map_charge_to_grid_order_5_cu (FixChargeEwald.cu:174-217) with five lanes
// per atom: lane t adds the 25 points of stencil plane a = t.  The six atoms
// of a warp are taken W = n/6 apart (atom g W + warp) so that the float
// atomics of one warp instruction land in distant parts of the mesh instead
// of piling onto the same points (neighbouring atoms are adjacent in the
// cell-sorted order)
__device__ __forceinline__ float pick5(const float w[5], int t) {
    return t == 0 ? w[0] : t == 1 ? w[1] : t == 2 ? w[2] : t == 3 ? w[3] : w[4];
}

// stencil plane a = t of atom i's charge (25 points, as two 16-byte vector
// atomics per z row: the five z points lie in two aligned groups of four,
// the mesh side being a multiple of 4)
__device__ __forceinline__ void spread_plane(const P3MArgs &A, int i, int t) {
    const float q = A.qs[i];
    if (q == 0.f) return;
    const P3MGeom &g = A.g;
    const float qi = g.qunit * q;
    int3 ng;
    float3 d;
    stencil(g, A.xs[i], ng, d);
    float wx[5], wy[5], wz[5];
    w5(d.x, wx);
    w5(d.y, wy);
    w5(d.z, wz);
    int pz[5];
#pragma unroll
    for (int c = 0; c < 5; c++) pz[c] = wrapi(ng.z + c - 2, g.sz.z);
    const int px = wrapi(ng.x + t - 2, g.sz.x);
    const float cyz = qi * pick5(wx, t);
    const int z0 = pz[0], g0 = z0 & ~3, sh = z0 - g0;
    const int g1 = (g0 + 4) % g.sz.z;
#pragma unroll
    for (int b = 0; b < 5; b++) {
        const int py = wrapi(ng.y + b - 2, g.sz.y);
        const float cz = cyz * wy[b];
        float w[5];
#pragma unroll
        for (int c = 0; c < 5; c++) w[c] = cz * wz[c];
        float4 v1, v2;
        switch (sh) {
            case 0: v1 = make_float4(w[0], w[1], w[2], w[3]); v2 = make_float4(w[4], 0.f, 0.f, 0.f); break;
            case 1: v1 = make_float4(0.f, w[0], w[1], w[2]); v2 = make_float4(w[3], w[4], 0.f, 0.f); break;
            case 2: v1 = make_float4(0.f, 0.f, w[0], w[1]); v2 = make_float4(w[2], w[3], w[4], 0.f); break;
            default: v1 = make_float4(0.f, 0.f, 0.f, w[0]); v2 = make_float4(w[1], w[2], w[3], w[4]); break;
        }
        float *row = A.rho + ((size_t)px * g.sz.y + py) * g.sz.z;
        atomicAdd(reinterpret_cast<float4 *>(row + g0), v1);
        atomicAdd(reinterpret_cast<float4 *>(row + g1), v2);
    }
}

__global__ void k_spread5(const P3MArgs a0, const P3MArgs *__restrict__ tab) {
    pdl_wait();
    MDX_P3M_ARGS;
    const int lane = threadIdx.x & 31;
    const int t = lane % 5;
    const int W = (A.n + 5) / 6;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int i = (lane / 5) * W + w;
    if (lane >= 30 || w >= W || i >= A.n) return;
    spread_plane(A, i, t);
}

__device__ __forceinline__ int mol_site(int4 ix, int k, int four_site) {
    return four_site ? (k == 0 ? ix.y : (k == 1 ? ix.z : ix.w)) : (k == 0 ? ix.x : (k == 1 ? ix.y : ix.z));
}

// the molecule form: lanes 15 j .. 15 j + 14 of a warp take the three
// charged sites (five planes each) of one molecule, two molecules per warp,
// the two W = nmol/2 apart; no lane is spent on an uncharged oxygen
__global__ void k_spread_mol(const P3MArgs a0, const P3MArgs *__restrict__ tab) {
    pdl_wait();
    MDX_P3M_ARGS;
    const int lane = threadIdx.x & 31;
    const int W = (A.nmol + 1) / 2;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int m = (lane / 15) * W + w;
    if (lane >= 30 || w >= W || m >= A.nmol) return;
    const int4 ix = A.slots ? make_int4(4 * m, 4 * m + 1, 4 * m + 2, 4 * m + 3) : A.mol_idx[m];
    spread_plane(A, mol_site(ix, (lane % 15) / 5, A.four_site), lane % 5);
}

// E_d(k) = i k_d G rho on the half spectrum (z halved), batched output
__global__ void k_efield(const P3MArgs a0, const P3MArgs *__restrict__ tab) {
    MDX_P3M_ARGS;
    const size_t nk = A.nk;
    size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nk) return;
    const int3 sz = A.g.sz;
    const float3 twopi_over_L = A.tpl;
    const float2 *__restrict__ rho_k = A.rho_k;
    const float *__restrict__ green = A.green;
    float2 *__restrict__ ek = A.e_k;
    const int nzh = sz.z / 2 + 1;
    const int iz = (int)(id % nzh);
    const int iy = (int)((id / nzh) % sz.y);
    const int ix = (int)(id / ((size_t)nzh * sz.y));
    const float kx = twopi_over_L.x * (float)(ix > sz.x / 2 ? ix - sz.x : ix);
    const float ky = twopi_over_L.y * (float)(iy > sz.y / 2 ? iy - sz.y : iy);
    const float kz = twopi_over_L.z * (float)iz;
    const float G = green[id];
    const float2 q = rho_k[id];
    // i k G (q.x + i q.y) = (-k G q.y) + i (k G q.x); Nyquist planes dropped per component
    const float gx = (2 * ix == sz.x) ? 0.f : kx * G;
    const float gy = (2 * iy == sz.y) ? 0.f : ky * G;
    const float gz = (2 * iz == sz.z) ? 0.f : kz * G;
    ek[id] = make_float2(-gx * q.y, gx * q.x);
    ek[nk + id] = make_float2(-gy * q.y, gy * q.x);
    ek[2 * nk + id] = make_float2(-gz * q.y, gz * q.x);
}

template <bool ACC>
__global__ void k_gather(const P3MArgs a0, const P3MArgs *__restrict__ tab) {
    MDX_P3M_ARGS;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const float4 *__restrict__ xs = A.xs;
    const float *__restrict__ qs = A.qs;
    const P3MGeom &g = A.g;
    const float *__restrict__ er = A.e_r;
    const size_t ngrid = A.ngrid;
    const float neg_inv_vol = A.niv;
    float4 *__restrict__ fs = A.fs;
    const float q = qs[i];
    if (q == 0.f) {
        if (!ACC) {
            float4 f = fs[i];
            fs[i] = make_float4(0.f, 0.f, 0.f, f.w);
        }
        return;
    }
    int3 ng;
    float3 d;
    stencil(g, xs[i], ng, d);
    float wx[5], wy[5], wz[5];
    w5(d.x, wx);
    w5(d.y, wy);
    w5(d.z, wz);
    int pz[5];
#pragma unroll
    for (int c = 0; c < 5; c++) pz[c] = wrapi(ng.z + c - 2, g.sz.z);
    float ex = 0.f, ey = 0.f, ez = 0.f;
#pragma unroll
    for (int a = 0; a < 5; a++) {
        const int px = wrapi(ng.x + a - 2, g.sz.x);
#pragma unroll
        for (int b = 0; b < 5; b++) {
            const int py = wrapi(ng.y + b - 2, g.sz.y);
            const size_t row = ((size_t)px * g.sz.y + py) * g.sz.z;
            const float wab = wx[a] * wy[b];
#pragma unroll
            for (int c = 0; c < 5; c++) {
                const float w = wab * wz[c];
                const size_t o = row + pz[c];
                ex += w * __ldg(er + o);
                ey += w * __ldg(er + ngrid + o);
                ez += w * __ldg(er + 2 * ngrid + o);
            }
        }
    }
    const float s = g.qunit * q * neg_inv_vol;
    float4 f = fs[i];
    if (ACC) {
        f.x += s * ex;
        f.y += s * ey;
        f.z += s * ez;
    } else {
        f.x = s * ex;
        f.y = s * ey;
        f.z = s * ez;
    }
    fs[i] = f;
}

// sum_k G |rho_k|^2 over the full spectrum from the half spectrum (FP64)
__global__ void k_recip_energy(int3 sz, const float2 *__restrict__ rho_k, const float *__restrict__ green, size_t nk,
                               double *out) {
    double acc = 0.0;
    const int nzh = sz.z / 2 + 1;
    for (size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x; id < nk; id += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(id % nzh);
        const double w = (iz == 0 || 2 * iz == sz.z) ? 1.0 : 2.0;
        const float2 q = rho_k[id];
        acc += w * (double)green[id] * ((double)q.x * q.x + (double)q.y * q.y);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// virials_cu (FixChargeEwald.cu:731-812) on the half spectrum: the 6-vector
// sum_k w G |rho_k|^2 (delta_ab - 2 (1/k^2 + 1/(4 alpha^2)) k_a k_b), k != 0,
// w = 2 for the kz planes that stand for their conjugates; FP64 sums
__global__ void k_recip_virial(int3 sz, const float2 *__restrict__ rho_k, const float *__restrict__ green, size_t nk,
                               double3 tpl, double alpha, double *out) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int nzh = sz.z / 2 + 1;
    const double f4a = 0.25 / (alpha * alpha);
    for (size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x; id < nk; id += (size_t)gridDim.x * blockDim.x) {
        const int iz = (int)(id % nzh);
        const int iy = (int)((id / nzh) % sz.y);
        const int ix = (int)(id / ((size_t)nzh * sz.y));
        const double kx = tpl.x * (ix > sz.x / 2 ? ix - sz.x : ix);
        const double ky = tpl.y * (iy > sz.y / 2 ? iy - sz.y : iy);
        const double kz = tpl.z * iz;
        const double k2 = kx * kx + ky * ky + kz * kz;
        if (k2 == 0.0) continue;
        const double w = (iz == 0 || 2 * iz == sz.z) ? 1.0 : 2.0;
        const float2 q = rho_k[id];
        const double E = w * (double)green[id] * ((double)q.x * q.x + (double)q.y * q.y);
        const double d = -2.0 * (1.0 / k2 + f4a);
        acc[0] += (1.0 + d * kx * kx) * E;
        acc[1] += (1.0 + d * ky * ky) * E;
        acc[2] += (1.0 + d * kz * kz) * E;
        acc[3] += d * kx * ky * E;
        acc[4] += d * kx * kz * E;
        acc[5] += d * ky * kz * E;
    }
#pragma unroll
    for (int c = 0; c < 6; c++) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(out + c, v);
    }
}

// mapVirialToSingleAtom (FixChargeEwald.cu:815-818): the field virial, 0.5/V
// of the sum, goes onto the first atom's per-atom virial
__global__ void k_add_field_virial(float *__restrict__ vir, const double *__restrict__ sum6, double scale) {
    const int c = threadIdx.x;
    if (c < 6) vir[c] += (float)(scale * sum6[c]);
}

__host__ __device__ double sinc(double x) {
    if (x < 0.1 && x > -0.1) {
        double x2 = x * x;
        return 1.0 - x2 * 0.16666666667 + x2 * x2 * 0.008333333333333333 - x2 * x2 * x2 * 0.00019841269841269841;
    }
    return std::sin(x) / x;
}

const double kAmp[5][5] = {
    {2.0 / 3.0, 0, 0, 0, 0},
    {1.0 / 50.0, 5.0 / 294.0, 0, 0, 0},
    {1.0 / 588.0, 7.0 / 1440.0, 21.0 / 3872.0, 0, 0},
    {1.0 / 4320.0, 3.0 / 1936.0, 7601.0 / 2271360.0, 143.0 / 28800.0, 0},
    {1.0 / 23232.0, 7601.0 / 12628160.0, 143.0 / 69120.0, 517231.0 / 106536960.0, 106640677.0 / 11737571328.0},
};

P3MGeom geom(State &s, FixChargeEwald &f) {
    P3MGeom g;
    g.sz = f.sz;
    g.lo = s.box.lo;
    g.h = make_float3(s.box.L.x / (float)f.sz.x, s.box.L.y / (float)f.sz.y, s.box.L.z / (float)f.sz.z);
    g.invh = make_float3(1.f / g.h.x, 1.f / g.h.y, 1.f / g.h.z);
    g.qunit = (float)std::sqrt(s.units.qqr_to_eng);
    return g;
}

P3MArgs p3m_args(State &s, FixChargeEwald &f) {
    P3MArgs A{};
    A.n = s.gpd.n;
    A.xs = s.gpd.xs.p;
    A.qs = s.gpd.qs.p;
    A.fs = s.gpd.fs.p;
    A.g = geom(s, f);
    A.rho = f.rho.p;
    A.rho_k = f.rho_k.p;
    A.e_k = f.e_k.p;
    A.e_r = f.e_r.p;
    A.green = f.green.p;
    A.tpl = make_float3((float)(6.28318530717958647693 / s.box.Ld.x), (float)(6.28318530717958647693 / s.box.Ld.y),
                        (float)(6.28318530717958647693 / s.box.Ld.z));
    A.nk = (size_t)f.sz.x * f.sz.y * (f.sz.z / 2 + 1);
    A.ngrid = (size_t)f.sz.x * f.sz.y * f.sz.z;
    A.niv = (float)(-1.0 / (s.box.Ld.x * s.box.Ld.y * s.box.Ld.z));
    A.slots = 0;
    A.e4 = f.own_fft ? f.e4.p : nullptr;
    return A;
}

// ---- P3M reciprocal solve on our own FFT (cubic 32^3 / 64^3 meshes) --------
// One warp transforms one line of N = 32 R points held as v[r] = x[32 r + lane]:
// R-point DFTs inside each lane, twiddles W_N^(lane k1), then a radix-2
// decimation-in-frequency FFT of 32 points across the lanes (shuffles); lane
// l then holds X[k1 + R bitrev5(l)] in v[k1].  Unnormalised, as cuFFT.
// Three kernels replace R2C + E(k) + batched C2R:
//   k_fft_zy   per x plane: real FFT along z (half spectrum kept) then along y
//   k_fft_xe   per (ky, kz) line: FFT along x, E_d(k) = i k_d G rho (Nyquist
//              planes dropped per component, as k_efield), 3 inverse FFTs along x
//   k_ifft_yz  per (x plane, component): inverse along y, then the real inverse along z of
//              the Hermitian half spectrum, E written as float4 (Ex, Ey, Ez, 0)
// so the gather reads one 16-byte field value per stencil point.
struct FFTArgs {
    int n;                   // points per side (32 or 64)
    const float *rho;        // [n][n][n]
    float2 *mid1;            // [n][n/2+1][n] (x, kz, ky): after the z and y passes
    float2 *mid2;            // [3][n][n/2+1][n] (d, x, kz, ky): E_d after the inverse x pass
    float4 *e4;              // [n][n][n]
    const float *green;      // [n][n][n/2+1]
    const float2 *tw;        // W_32^k (32) then W_64^k (64), forward sign
    float3 tpl;              // 2 pi / L
};

__device__ __forceinline__ int brev5(int l) { return (int)(__brev((unsigned)l) >> 27); }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// this lane's twiddles: W_2h^(lane mod h) for the five lane stages and
// W_N^lane for the R = 2 step (forward sign; conjugated for the inverse)
struct LaneTw {
    float2 st[5];
    float2 wn;
};

template <int R>
__device__ __forceinline__ LaneTw lane_twiddles(int lane, const float2 *__restrict__ tw) {
    LaneTw T;
#pragma unroll
    for (int s = 0; s < 5; s++) {
        const int h = 16 >> s;
        T.st[s] = __ldg(tw + (lane & (h - 1)) * (16 / h));
    }
    T.wn = R == 2 ? __ldg(tw + 32 + lane) : make_float2(1.f, 0.f);
    return T;
}

// forward (INV = false: W = exp(-2 pi i k / N)) or inverse (W conjugated)
template <int R, bool INV>
__device__ __forceinline__ void warp_fft(float2 (&v)[R], int lane, const LaneTw &T) {
    if (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = make_float2(a.x + b.x, a.y + b.y);
        float2 w = T.wn;
        if (INV) w.y = -w.y;
        v[1] = cmul(make_float2(a.x - b.x, a.y - b.y), w);
    }
#pragma unroll
    for (int k1 = 0; k1 < R; k1++) {
#pragma unroll
        for (int s = 0; s < 5; s++) {
            const int h = 16 >> s;
            const float px = __shfl_xor_sync(0xffffffffu, v[k1].x, h);
            const float py = __shfl_xor_sync(0xffffffffu, v[k1].y, h);
            if ((lane & h) == 0) {
                v[k1] = make_float2(v[k1].x + px, v[k1].y + py);
            } else {
                float2 w = T.st[s];
                if (INV) w.y = -w.y;
                v[k1] = cmul(make_float2(px - v[k1].x, py - v[k1].y), w);
            }
        }
    }
}

template <int R>
__device__ __forceinline__ int fft_out_index(int k1, int lane) { return k1 + R * brev5(lane); }

// Inverse transform of a line held the way warp_fft leaves its output (lane
// l holds Y[k1 + R bitrev5(l)] in v[k1]): radix-2 decimation in time across
// the lanes (stages h = 1 .. 16, twiddle W_2h^(lane mod h) conjugated, on
// the bit-reversed positions), then for R = 2 the in-lane step y[l] = z0 +
// W_N^-l z1, y[l + 32] = z0 - W_N^-l z1.  Lane l then holds y[32 r + l] in
// v[r]: natural order, no permutation through shared memory.  Unnormalised.
template <int R>
__device__ __forceinline__ void warp_ifft_dit(float2 (&v)[R], int lane, const LaneTw &T) {
#pragma unroll
    for (int k1 = 0; k1 < R; k1++) {
#pragma unroll
        for (int s = 4; s >= 0; s--) {
            const int h = 16 >> s;
            const float px = __shfl_xor_sync(0xffffffffu, v[k1].x, h);
            const float py = __shfl_xor_sync(0xffffffffu, v[k1].y, h);
            float2 w = T.st[s];
            w.y = -w.y;
            if ((lane & h) == 0) {
                const float2 t = cmul(make_float2(px, py), w);
                v[k1] = make_float2(v[k1].x + t.x, v[k1].y + t.y);
            } else {
                const float2 t = cmul(v[k1], w);
                v[k1] = make_float2(px - t.x, py - t.y);
            }
        }
    }
    if (R == 2) {
        float2 w = T.wn;
        w.y = -w.y;
        const float2 z0 = v[0];
        const float2 t = cmul(v[R - 1], w);
        v[0] = make_float2(z0.x + t.x, z0.y + t.y);
        v[R - 1] = make_float2(z0.x - t.x, z0.y - t.y);
    }
}

// plane kernels: kFftPlaneWarps warps per block, fixed at compile time so a
// warp's line loop has a constant trip count and, for the small meshes,
// unrolls (the lines' loads are in flight together)
constexpr int kFftPlaneWarps = 16;

template <int R>
__global__ void __launch_bounds__(kFftPlaneWarps * 32) k_fft_zy(const FFTArgs a0, const FFTArgs *__restrict__ tab) {
    extern __shared__ float2 plane[];  // [n][n/2+1]
    constexpr int N = 32 * R, NH = N / 2 + 1;
    constexpr int nw = kFftPlaneWarps, UNR = R <= 2 ? 4 : 1;
    pdl_wait();
    const FFTArgs A = tab ? tab[blockIdx.y] : a0;  // batched replicas: blockIdx.y
    const int x = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const LaneTw T = lane_twiddles<R>(lane, A.tw);
#pragma unroll UNR
    for (int y = w; y < N; y += nw) {
        float2 v[R];
        const float *line = A.rho + ((size_t)x * N + y) * N;
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = make_float2(line[32 * r + lane], 0.f);
        warp_fft<R, false>(v, lane, T);
#pragma unroll
        for (int k1 = 0; k1 < R; k1++) {
            const int k = fft_out_index<R>(k1, lane);
            if (k < NH) plane[y * NH + k] = v[k1];
        }
    }
    __syncthreads();
#pragma unroll UNR
    for (int kz = w; kz < NH; kz += nw) {
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = plane[(32 * r + lane) * NH + kz];
        warp_fft<R, false>(v, lane, T);
#pragma unroll
        for (int k1 = 0; k1 < R; k1++) {
            const int ky = fft_out_index<R>(k1, lane);
            A.mid1[((size_t)x * NH + kz) * N + ky] = v[k1];  // a column's 64 ky in one 512-byte row
        }
    }
}

template <int R>
__global__ void __launch_bounds__(256) k_fft_xe(const FFTArgs a0, const FFTArgs *__restrict__ tab) {
    constexpr int N = 32 * R, NH = N / 2 + 1;
    pdl_wait();
    const FFTArgs A = tab ? tab[blockIdx.y] : a0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int line_id = blockIdx.x * (blockDim.x >> 5) + w;
    if (line_id >= N * NH) return;  // warp-uniform; no block barrier below
    const LaneTw T = lane_twiddles<R>(lane, A.tw);
    const int ky = line_id / NH, kz = line_id % NH;
    const size_t stride = (size_t)N * NH;
    const size_t base = (size_t)ky * NH + kz;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = A.mid1[(32 * r + lane) * stride + (size_t)kz * N + ky];
    warp_fft<R, false>(v, lane, T);
    const float kyv = A.tpl.y * (float)(ky > N / 2 ? ky - N : ky);
    const float kzv = A.tpl.z * (float)kz;
    float2 e[3][R];
#pragma unroll
    for (int k1 = 0; k1 < R; k1++) {
        const int kx = fft_out_index<R>(k1, lane);
        const float kxv = A.tpl.x * (float)(kx > N / 2 ? kx - N : kx);
        const float G = __ldg(A.green + (size_t)kx * stride + base);
        const float2 q = v[k1];
        const float gx = (2 * kx == N) ? 0.f : kxv * G;
        const float gy = (2 * ky == N) ? 0.f : kyv * G;
        const float gz = (2 * kz == N) ? 0.f : kzv * G;
        e[0][k1] = make_float2(-gx * q.y, gx * q.x);
        e[1][k1] = make_float2(-gy * q.y, gy * q.x);
        e[2][k1] = make_float2(-gz * q.y, gz * q.x);
    }
    // the inverse x transforms take the forward's bit-reversed layout as it
    // stands and leave natural order
#pragma unroll
    for (int d = 0; d < 3; d++) {
        float2 u[R];
#pragma unroll
        for (int k1 = 0; k1 < R; k1++) u[k1] = e[d][k1];
        warp_ifft_dit<R>(u, lane, T);
        float2 *out = A.mid2 + (size_t)d * N * stride;
#pragma unroll
        for (int r = 0; r < R; r++) out[(32 * r + lane) * stride + (size_t)kz * N + ky] = u[r];
    }
}

// one block per (x plane, field component): inverse along y for every kz,
// then the real inverse along z; component d of the float4 field is written
template <int R>
__global__ void __launch_bounds__(kFftPlaneWarps * 32) k_ifft_yz(const FFTArgs a0, const FFTArgs *__restrict__ tab) {
    extern __shared__ float2 plane[];  // [n][n/2+1]
    constexpr int N = 32 * R, NH = N / 2 + 1;
    constexpr int nw = kFftPlaneWarps, UNR = R <= 2 ? 4 : 1;
    pdl_wait();
    const FFTArgs A = tab ? tab[blockIdx.z] : a0;  // batched replicas: blockIdx.z
    const int x = blockIdx.x, d = blockIdx.y;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const LaneTw T = lane_twiddles<R>(lane, A.tw);
    const size_t stride = (size_t)N * NH;
    const float2 *src0 = A.mid2 + (size_t)d * N * stride + (size_t)x * stride;
#pragma unroll UNR
    for (int kz = w; kz < NH; kz += nw) {
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src0[(size_t)kz * N + 32 * r + lane];  // one contiguous ky row
        warp_fft<R, true>(v, lane, T);
#pragma unroll
        for (int k1 = 0; k1 < R; k1++) plane[fft_out_index<R>(k1, lane) * NH + kz] = v[k1];
    }
    __syncthreads();
    float *e = reinterpret_cast<float *>(A.e4) + d;
#pragma unroll UNR
    for (int y = w; y < N; y += nw) {
        const float2 *row = plane + y * NH;
        // the Hermitian half spectrum read in the bit-reversed order the
        // decimation-in-time inverse takes; the line comes out in natural
        // order (consecutive lanes, consecutive points)
        float2 v[R];
#pragma unroll
        for (int k1 = 0; k1 < R; k1++) {
            const int n = fft_out_index<R>(k1, lane);
            float2 X;
            if (n == 0 || n == N / 2) {
                X = make_float2(row[n].x, 0.f);
            } else if (n < N / 2) {
                X = row[n];
            } else {
                const float2 c = row[N - n];
                X = make_float2(c.x, -c.y);
            }
            v[k1] = X;
        }
        warp_ifft_dit<R>(v, lane, T);
        const size_t base = ((size_t)x * N + y) * N;
#pragma unroll
        for (int r = 0; r < R; r++) e[4 * (base + 32 * r + lane)] = v[r].x;
    }
}

// gather on the interleaved field, five lanes per atom (six atoms per warp):
// lane t sums the 25 points of stencil plane a = t with one 16-byte load per
// point; the five partial fields are added with shuffles
// the field at atom i's stencil plane a = t, weighted (one lane's share)
__device__ __forceinline__ float3 gather_plane(const P3MArgs &A, const float4 *__restrict__ e4, int i, int t) {
    const P3MGeom &g = A.g;
    int3 ng;
    float3 d;
    stencil(g, A.xs[i], ng, d);
    float wx[5], wy[5], wz[5];
    w5(d.x, wx);
    w5(d.y, wy);
    w5(d.z, wz);
    int pz[5];
#pragma unroll
    for (int c = 0; c < 5; c++) pz[c] = wrapi(ng.z + c - 2, g.sz.z);
    const int px = wrapi(ng.x + t - 2, g.sz.x);
    const float wa = pick5(wx, t);
    float ex = 0.f, ey = 0.f, ez = 0.f;
#pragma unroll
    for (int b = 0; b < 5; b++) {
        const int py = wrapi(ng.y + b - 2, g.sz.y);
        const size_t row = ((size_t)px * g.sz.y + py) * g.sz.z;
        const float wab = wa * wy[b];
#pragma unroll
        for (int c = 0; c < 5; c++) {
            const float w = wab * wz[c];
            const float4 e = __ldg(e4 + row + pz[c]);
            ex += w * e.x;
            ey += w * e.y;
            ez += w * e.z;
        }
    }
    return make_float3(ex, ey, ez);
}

// sum over the five lanes base .. base + 4 (valid in lane base); the whole
// warp takes part
__device__ __forceinline__ float3 group5_sum(float3 e, int base) {
    float3 s = e;
#pragma unroll
    for (int k = 1; k < 5; k++) {
        const int src = (base + k) & 31;
        s.x += __shfl_sync(0xffffffffu, e.x, src);
        s.y += __shfl_sync(0xffffffffu, e.y, src);
        s.z += __shfl_sync(0xffffffffu, e.z, src);
    }
    return s;
}

template <bool ACC>
__device__ __forceinline__ void gather4_body(const P3MArgs &A, const float4 *__restrict__ e4) {
    const int lane = threadIdx.x & 31;
    const int t = lane % 5, base = lane - t;
    const int i = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 6 + lane / 5;
    const bool valid = lane < 30 && i < A.n;
    const float q = valid ? A.qs[i] : 0.f;
    const float3 e = q != 0.f ? gather_plane(A, e4, i, t) : make_float3(0.f, 0.f, 0.f);
    const float3 sm = group5_sum(e, base);
    if (!valid || t != 0) return;
    float4 *__restrict__ fs = A.fs;
    float4 f = fs[i];
    if (q == 0.f) {
        if (!ACC) fs[i] = make_float4(0.f, 0.f, 0.f, f.w);
        return;
    }
    const float s = A.g.qunit * q * A.niv;
    if (ACC) {
        f.x += s * sm.x;
        f.y += s * sm.y;
        f.z += s * sm.z;
    } else {
        f.x = s * sm.x;
        f.y = s * sm.y;
        f.z = s * sm.z;
    }
    fs[i] = f;
}

template <bool ACC>
__global__ void k_gather4(const P3MArgs A, const float4 *__restrict__ e4) {
    pdl_wait();
    gather4_body<ACC>(A, e4);
}

// batched replicas (blockIdx.y = replica), each with its own field
template <bool ACC>
__global__ void k_gather4_tab(const P3MArgs a0, const P3MArgs *__restrict__ tab) {
    MDX_P3M_ARGS;
    if ((blockIdx.x * blockDim.x >> 5) * 6 >= (unsigned)A.n) return;  // past this replica's atoms
    gather4_body<ACC>(A, A.e4);
}

// the molecule form of the gather into a per-step buffer (STORE): the
// mapping of k_spread_mol, each charged site's force stored, the uncharged
// oxygen of a four-site molecule stored as zero
__global__ void k_gather_mol(const P3MArgs a0, const P3MArgs *__restrict__ tab, const float4 *__restrict__ e4_one) {
    pdl_wait();
    MDX_P3M_ARGS;
    const float4 *__restrict__ e4 = tab ? A.e4 : e4_one;  // batched: each replica's own field
    const int lane = threadIdx.x & 31;
    const int t = lane % 5, base = lane - t;
    const int W = (A.nmol + 1) / 2;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int m = (lane / 15) * W + w;
    const bool valid = lane < 30 && w < W && m < A.nmol;
    const int k = (lane % 15) / 5;
    int4 ix = make_int4(0, 0, 0, 0);
    int i = 0;
    float q = 0.f;
    if (valid) {
        ix = A.slots ? make_int4(4 * m, 4 * m + 1, 4 * m + 2, 4 * m + 3) : A.mol_idx[m];
        i = mol_site(ix, k, A.four_site);
        q = A.qs[i];
    }
    const float3 e = q != 0.f ? gather_plane(A, e4, i, t) : make_float3(0.f, 0.f, 0.f);
    const float3 sm = group5_sum(e, base);
    if (!valid || t != 0) return;
    const float s = A.g.qunit * q * A.niv;
    A.fs[i] = make_float4(s * sm.x, s * sm.y, s * sm.z, 0.f);
    if (A.four_site && k == 0) A.fs[ix.x] = make_float4(0.f, 0.f, 0.f, 0.f);
}

}  // namespace

FixChargeEwald::FixChargeEwald(State *s, std::string h, std::string g)
    : Fix(s, h, g, "ChargeEwald", FixKind::ChargeEwald) {
    requiresCharges = true;
}

FixChargeEwald::~FixChargeEwald() {
    if (plans) {
        cufftDestroy(plan_r2c);
        cufftDestroy(plan_c2r);
    }
}

int FixChargeEwald::setParameters(int nx, int ny, int nz, double rcut, int ord) {
    auto ok = [](int v) { return v == 32 || v == 64 || v == 128 || v == 256 || v == 512 || v == 1024; };
    if (!ok(nx) || !ok(ny) || !ok(nz)) {
        set_error(MDX_ERR_ARG, "P3M grid %d %d %d: only 2^N sizes 32..1024 are supported (FixChargeEwald.cu:976-987)",
                  nx, ny, nz);
        return MDX_ERR_ARG;
    }
    if (ord != 5) {
        set_error(MDX_ERR_UNSUPPORTED, "P3M interpolation order %d: this library implements order 5", ord);
        return MDX_ERR_UNSUPPORTED;
    }
    sz = make_int3(nx, ny, nz);
    r_cut = rcut;
    order = ord;
    return 0;
}

// total_Q2 (setTotalQ2, :883-914) in FP64 and the secant of :918-967
double FixChargeEwald::findAlpha() {
    State &s = *state;
    double Q2 = 0.0;
    for (auto &a : s.atoms) Q2 += a.q * a.q;
    Q2 *= s.units.qqr_to_eng;
    const double L[3] = {s.box.Ld.x, s.box.Ld.y, s.box.Ld.z};
    const double h[3] = {L[0] / sz.x, L[1] / sz.y, L[2] / sz.z};
    const double nAtoms = (double)s.atoms.size();
    const double rc = r_cut;
    auto dk = [&](double a) {
        double tot = 0.0;
        for (int d = 0; d < 3; d++) {
            double sum = 0.0;
            for (int m = 0; m < order; m++) sum += kAmp[order - 1][m] * std::pow(h[d] * a, 2 * m);
            tot += 1.0 / (L[d] * L[d]) * std::pow(a * h[d], order) * std::sqrt(a * L[d] / nAtoms * std::sqrt(2.0 * M_PI) * sum);
        }
        return Q2 / 3.0 * tot;
    };
    auto dr = [&](double a) { return 2 * Q2 / std::sqrt(nAtoms * rc * L[0] * L[1] * L[2]) * std::exp(-a * a * rc * rc); };
    double xa = 0.0, xb = 4.79853 / rc;
    double ya = dk(xa) - dr(xa), yb = dk(xb) - dr(xb);
    for (int it = 0; it < 100 && std::fabs(yb) / dr(xb) > 1e-5; it++) {
        double kinv = (xb - xa) / (yb - ya);
        ya = yb;
        xa = xb;
        xb = xa - ya * kinv;
        yb = dk(xb) - dr(xb);
    }
    return xb;
}

namespace {
template <int R>
int own_fft_setup();
}  // namespace

int FixChargeEwald::prepareForRun() {
    State &s = *state;
    if (r_cut < 0) r_cut = s.rCut;
    alpha = alpha_user > 0 ? alpha_user : findAlpha();
    const size_t ng = (size_t)sz.x * sz.y * sz.z;
    const size_t nk = (size_t)sz.x * sz.y * (sz.z / 2 + 1);
    if (int e = rho.alloc(ng)) return e;
    if (int e = rho_k.alloc(nk)) return e;
    if (int e = e_k.alloc(3 * nk)) return e;
    if (int e = e_r.alloc(3 * ng)) return e;
    if (int e = green.alloc(nk)) return e;
    if (int e = energy_acc.alloc(1)) return e;
    if (!plans) {
        if (cufftPlan3d(&plan_r2c, sz.x, sz.y, sz.z, CUFFT_R2C) != CUFFT_SUCCESS) {
            set_error(MDX_ERR_CUDA, "cufftPlan3d R2C failed");
            return MDX_ERR_CUDA;
        }
        int dims[3] = {sz.x, sz.y, sz.z};
        if (cufftPlanMany(&plan_c2r, 3, dims, nullptr, 1, (int)nk, nullptr, 1, (int)ng, CUFFT_C2R, 3) !=
            CUFFT_SUCCESS) {
            set_error(MDX_ERR_CUDA, "cufftPlanMany C2R failed");
            return MDX_ERR_CUDA;
        }
        plans = true;
    }
    cufftSetStream(plan_r2c, s.stream);
    cufftSetStream(plan_c2r, s.stream);
    // Green function on the half spectrum (Green_function_cu), on the device
    if (int e = computeGreen(s.stream)) return e;
    // own FFT for cubic 32^3 / 64^3 meshes (cuFFT for every other size)
    if (int e = f_recip.alloc(std::max(s.gpd.n, 1))) return e;
    own_fft = sz.x == sz.y && sz.y == sz.z && (sz.x == 32 || sz.x == 64);
    if (own_fft) {
        if (int e = e4.alloc(ng)) return e;
        if (int e = tw.alloc(96)) return e;
        std::vector<float2> h(96);
        for (int k = 0; k < 32; k++)
            h[k] = make_float2((float)std::cos(-2.0 * M_PI * k / 32.0), (float)std::sin(-2.0 * M_PI * k / 32.0));
        for (int k = 0; k < 64; k++)
            h[32 + k] = make_float2((float)std::cos(-2.0 * M_PI * k / 64.0), (float)std::sin(-2.0 * M_PI * k / 64.0));
        MDX_CUDA_TRY(cudaMemcpy(tw.p, h.data(), 96 * sizeof(float2), cudaMemcpyHostToDevice));
        if (int e = sz.x == 64 ? own_fft_setup<2>() : own_fft_setup<1>()) return e;
    }
    prepared = true;
    return 0;
}

namespace {
FFTArgs fft_args(State &s, FixChargeEwald &f) {
    FFTArgs A{};
    A.n = f.sz.x;
    A.rho = f.rho.p;
    A.mid1 = f.rho_k.p;
    A.mid2 = f.e_k.p;
    A.e4 = f.e4.p;
    A.green = f.green.p;
    A.tw = f.tw.p;
    A.tpl = make_float3((float)(6.28318530717958647693 / s.box.Ld.x), (float)(6.28318530717958647693 / s.box.Ld.y),
                        (float)(6.28318530717958647693 / s.box.Ld.z));
    return A;
}

template <int R>
int own_solve(State &s, FixChargeEwald &f, cudaStream_t st) {
    constexpr int N = 32 * R, NH = N / 2 + 1;
    const FFTArgs A = fft_args(s, f);
    // 512-thread plane blocks (measured +0.8 % per water step against 1024
    // beside the pair kernel; 256 was slower)
    const FFTArgs *nt = nullptr;
    MDX_CUDA_TRY(launch_pdl_prio(true, k_fft_zy<R>, dim3(N), dim3(kFftPlaneWarps * 32), (size_t)N * NH * sizeof(float2), st, A, nt));
    MDX_CUDA_TRY(launch_pdl_prio(true, k_fft_xe<R>, dim3((N * NH + 7) / 8), dim3(256), 0, st, A, nt));
    MDX_CUDA_TRY(launch_pdl_prio(true, k_ifft_yz<R>, dim3(N, 3), dim3(kFftPlaneWarps * 32), (size_t)N * NH * sizeof(float2), st, A, nt));
    return 0;
}

template <int R>
int own_fft_setup() {
    constexpr int N = 32 * R, NH = N / 2 + 1;
    MDX_CUDA_TRY(cudaFuncSetAttribute(k_ifft_yz<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      N * NH * (int)sizeof(float2)));
    MDX_CUDA_TRY(cudaFuncSetAttribute(k_fft_zy<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      N * NH * (int)sizeof(float2)));
    return 0;
}
}  // namespace

namespace {
// the optimal influence function of order-5 P3M on the half spectrum
// (Green_function_cu, FixChargeEwald.cu:218-294), one thread per k, FP64:
// sum over the aliasing images m within +-lim of the charge assignment
// function's transform W^(2 order) and the reference force R(k_m)
__global__ void k_green(int3 sz, double3 L, double alpha, int lim, float *__restrict__ green) {
    const int nzh = sz.z / 2 + 1;
    const size_t nk = (size_t)sz.x * sz.y * nzh;
    const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nk) return;
    const int iz = (int)(id % nzh);
    const int iy = (int)((id / nzh) % sz.y);
    const int ix = (int)(id / ((size_t)nzh * sz.y));
    const double tp = 6.28318530717958647693;
    const double h0 = L.x / sz.x, h1 = L.y / sz.y, h2 = L.z / sz.z;
    const double kx = tp * (ix > sz.x / 2 ? ix - sz.x : ix) / L.x;
    const double ky = tp * (iy > sz.y / 2 ? iy - sz.y : iy) / L.y;
    const double kz = tp * iz / L.z;
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double f4a = 0.25 / alpha / alpha;
    double val = 0.0;
    if (k2 != 0.0) {
        double s1 = 0.0, s2 = 0.0;
        for (int mx = -lim; mx <= lim; mx++)
            for (int my = -lim; my <= lim; my++)
                for (int mz = -lim; mz <= lim; mz++) {
                    const double px = kx + tp * mx / h0, py = ky + tp * my / h1, pz = kz + tp * mz / h2;
                    const double pp = px * px + py * py + pz * pz;
                    const double W = sinc(px * h0 * 0.5) * sinc(py * h1 * 0.5) * sinc(pz * h2 * 0.5);
                    const double W2 = W * W, W4 = W2 * W2, W8 = W4 * W4;
                    const double W10 = W8 * W2;  // W^(2 order), order 5
                    s1 += 12.56637061435917295385 * exp(-pp * f4a) * (kx * px + ky * py + kz * pz) / pp * W10;
                    s2 += W10;
                }
        val = s1 / (s2 * s2) / k2;
    }
    green[id] = (float)val;
}
}  // namespace

int FixChargeEwald::computeGreen(cudaStream_t st) {
    State &s = *state;
    const double L[3] = {s.box.Ld.x, s.box.Ld.y, s.box.Ld.z};
    const double h[3] = {L[0] / sz.x, L[1] / sz.y, L[2] / sz.z};
    const int lim = (int)(alpha * std::pow(h[0] * h[1] * h[2], 1.0 / 3.0) / 3.14159 * std::sqrt(-std::log(10E-7))) + 1;
    const size_t nk = (size_t)sz.x * sz.y * (sz.z / 2 + 1);
    k_green<<<(unsigned)((nk + 255) / 256), 256, 0, st>>>(sz, make_double3(L[0], L[1], L[2]), alpha, lim, green.p);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// FixChargeEwald::handleBoundsChange (FixChargeEwald.cu:1200-1229): the
// splitting parameter for the new box (unless set by hand) and the Green
// function
int FixChargeEwald::boxChanged() {
    if (!prepared) return 0;
    alpha = alpha_user > 0 ? alpha_user : findAlpha();
    return computeGreen(state->stream);
}

int FixChargeEwald::spread(cudaStream_t st) {
    State &s = *state;
    const size_t ng = (size_t)sz.x * sz.y * sz.z;
    MDX_CUDA_TRY(cudaMemsetAsync(rho.p, 0, ng * sizeof(float), st));
    MDX_CUDA_TRY(launch_pdl_prio(true, k_spread5, dim3((s.gpd.n + 47) / 48), dim3(256), 0, st, p3m_args(s, *this),
                            (const P3MArgs *)nullptr));
    return 0;
}

int FixChargeEwald::solve(cudaStream_t st) {
    State &s = *state;
    if (own_fft) return sz.x == 64 ? own_solve<2>(s, *this, st) : own_solve<1>(s, *this, st);
    const size_t nk = (size_t)sz.x * sz.y * (sz.z / 2 + 1);
    cufftSetStream(plan_r2c, st);
    cufftSetStream(plan_c2r, st);
    if (cufftExecR2C(plan_r2c, rho.p, (cufftComplex *)rho_k.p) != CUFFT_SUCCESS) {
        set_error(MDX_ERR_CUDA, "cufftExecR2C failed");
        return MDX_ERR_CUDA;
    }
    k_efield<<<(unsigned)((nk + 255) / 256), 256, 0, st>>>(p3m_args(s, *this), nullptr);
    MDX_LAUNCHED();
    if (cufftExecC2R(plan_c2r, (cufftComplex *)e_k.p, e_r.p) != CUFFT_SUCCESS) {
        set_error(MDX_ERR_CUDA, "cufftExecC2R failed");
        return MDX_ERR_CUDA;
    }
    return 0;
}

int FixChargeEwald::gather(bool accumulate, cudaStream_t st) {
    State &s = *state;
    const P3MArgs A = p3m_args(s, *this);
    if (own_fft) {
        if (accumulate)
            MDX_CUDA_TRY(launch_pdl_prio(true, k_gather4<true>, dim3((s.gpd.n + 47) / 48), dim3(256), 0, st, A,
                                    (const float4 *)e4.p));
        else
            MDX_CUDA_TRY(launch_pdl_prio(true, k_gather4<false>, dim3((s.gpd.n + 47) / 48), dim3(256), 0, st, A,
                                    (const float4 *)e4.p));
        return 0;
    }
    if (accumulate)
        k_gather<true><<<(s.gpd.n + 127) / 128, 128, 0, st>>>(A, nullptr);
    else
        k_gather<false><<<(s.gpd.n + 127) / 128, 128, 0, st>>>(A, nullptr);
    MDX_LAUNCHED();
    return 0;
}

int FixChargeEwald::gather_to(float4 *out, cudaStream_t st) {
    State &s = *state;
    P3MArgs A = p3m_args(s, *this);
    A.fs = out;
    if (own_fft) {
        MDX_CUDA_TRY(launch_pdl_prio(true, k_gather4<false>, dim3((s.gpd.n + 47) / 48), dim3(256), 0, st, A,
                                (const float4 *)e4.p));
    } else {
        k_gather<false><<<(s.gpd.n + 127) / 128, 128, 0, st>>>(A, nullptr);
        MDX_LAUNCHED();
    }
    return 0;
}

// the molecule form of spread and gather (every atom in a rigid molecule,
// all molecules four-site with uncharged oxygens or all three-site, own FFT)
bool FixChargeEwald::mol_form_ok(const FixRigid &r) const {
    const State &s = *state;
    if (!own_fft || r.mol_ids.empty() || !r.d_mol_idx.p) return false;
    const bool four = r.mol_ids[0].w >= 0;
    size_t members = 0;
    for (const int4 &m : r.mol_ids) {
        if ((m.w >= 0) != four) return false;
        if (four && s.atoms[m.x].q != 0.0) return false;
        members += four ? 4 : 3;
    }
    return members == s.atoms.size();
}

P3MArgs mol_args(State &s, FixChargeEwald &f, const FixRigid &r) {
    P3MArgs A = p3m_args(s, f);
    A.mol_idx = r.d_mol_idx.p;
    A.nmol = (int)r.mol_ids.size();
    A.four_site = r.mol_ids[0].w >= 0 ? 1 : 0;
    A.slots = s.mf.on ? 1 : 0;
    return A;
}

int FixChargeEwald::spread_mol(cudaStream_t st, const FixRigid &r) {
    State &s = *state;
    const size_t ng = (size_t)sz.x * sz.y * sz.z;
    MDX_CUDA_TRY(cudaMemsetAsync(rho.p, 0, ng * sizeof(float), st));
    const P3MArgs A = mol_args(s, *this, r);
    const int warps = (A.nmol + 1) / 2;
    // two-warp blocks: they slot in beside the pair kernel's (measured +1 % per
    // water step against 256-thread blocks)
    MDX_CUDA_TRY(launch_pdl_prio(true, k_spread_mol, dim3((warps + 1) / 2), dim3(64), 0, st, A,
                                 (const P3MArgs *)nullptr));
    return 0;
}

int FixChargeEwald::gather_mol_to(float4 *out, cudaStream_t st, const FixRigid &r) {
    State &s = *state;
    P3MArgs A = mol_args(s, *this, r);
    A.fs = out;
    const int warps = (A.nmol + 1) / 2;
    MDX_CUDA_TRY(launch_pdl_prio(true, k_gather_mol, dim3((warps + 1) / 2), dim3(64), 0, st, A,
                                 (const P3MArgs *)nullptr, (const float4 *)e4.p));
    return 0;
}

int FixChargeEwald::compute(int virialMode) {
    State &s = *state;
    if (int e = spread(s.stream)) return e;
    if (int e = solve(s.stream)) return e;
    if (int e = gather(true, s.stream)) return e;
    return virialMode ? ewald_recip_virial(s, *this) : 0;
}

// the reciprocal-space virial (FixChargeEwald::compute with virialMode,
// FixChargeEwald.cu:1455-1466): spread, R2C, k-space sum, onto atom 0
int ewald_recip_virial(State &s, FixChargeEwald &f) {
    if (int e = f.spread(s.stream)) return e;
    cufftSetStream(f.plan_r2c, s.stream);
    if (cufftExecR2C(f.plan_r2c, f.rho.p, (cufftComplex *)f.rho_k.p) != CUFFT_SUCCESS) {
        set_error(MDX_ERR_CUDA, "cufftExecR2C failed");
        return MDX_ERR_CUDA;
    }
    if (int e = f.vir_acc.alloc(6)) return e;
    MDX_CUDA_TRY(cudaMemsetAsync(f.vir_acc.p, 0, 6 * sizeof(double), s.stream));
    const size_t nk = (size_t)f.sz.x * f.sz.y * (f.sz.z / 2 + 1);
    const double3 tpl = make_double3(2.0 * M_PI / s.box.Ld.x, 2.0 * M_PI / s.box.Ld.y, 2.0 * M_PI / s.box.Ld.z);
    k_recip_virial<<<148, 256, 0, s.stream>>>(f.sz, f.rho_k.p, f.green.p, nk, tpl, f.alpha, f.vir_acc.p);
    MDX_LAUNCHED();
    const double V = s.box.Ld.x * s.box.Ld.y * s.box.Ld.z;
    k_add_field_virial<<<1, 32, 0, s.stream>>>(s.gpd.virials.p, f.vir_acc.p, 0.5 / V);
    MDX_LAUNCHED();
    return 0;
}

int ewald_recip_energy(State &s, FixChargeEwald &f, double *out) {
    if (int e = f.spread(s.stream)) return e;
    cufftSetStream(f.plan_r2c, s.stream);
    if (cufftExecR2C(f.plan_r2c, f.rho.p, (cufftComplex *)f.rho_k.p) != CUFFT_SUCCESS) {
        set_error(MDX_ERR_CUDA, "cufftExecR2C failed");
        return MDX_ERR_CUDA;
    }
    const size_t nk = (size_t)f.sz.x * f.sz.y * (f.sz.z / 2 + 1);
    MDX_CUDA_TRY(cudaMemsetAsync(f.energy_acc.p, 0, sizeof(double), s.stream));
    k_recip_energy<<<148, 256, 0, s.stream>>>(f.sz, f.rho_k.p, f.green.p, nk, f.energy_acc.p);
    MDX_LAUNCHED();
    double sumG = 0.0;
    MDX_CUDA_TRY(cudaMemcpyAsync(&sumG, f.energy_acc.p, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    double Q2 = 0.0;
    for (auto &a : s.atoms) Q2 += a.q * a.q;
    Q2 *= s.units.qqr_to_eng;
    const double V = s.box.Ld.x * s.box.Ld.y * s.box.Ld.z;
    *out = 0.5 * sumG / V - f.alpha / std::sqrt(M_PI) * Q2;
    return 0;
}

// ---- batched replicas -------------------------------------------------------
// Replicas are grouped by mesh size; each class gets contiguous pools that its
// replicas' buffers view, so a batched cuFFT plan per class covers them all.
// Spread, E(k) and gather are one launch each for every replica.
int batch_p3m_prepare(Batch &b) {
    const int R = (int)b.reps.size();
    for (int r = 0; r < R; r++) {
        FixChargeEwald *f = b.reps[r]->ewaldFix();
        Batch::FFTClass *c = nullptr;
        for (auto &k : b.fft)
            if (k->sz.x == f->sz.x && k->sz.y == f->sz.y && k->sz.z == f->sz.z) c = k.get();
        if (!c) {
            b.fft.emplace_back(new Batch::FFTClass());
            c = b.fft.back().get();
            c->sz = f->sz;
        }
        c->reps.push_back(r);
    }
    for (auto &cp : b.fft) {
        Batch::FFTClass &c = *cp;
        const int K = (int)c.reps.size();
        const size_t ng = (size_t)c.sz.x * c.sz.y * c.sz.z;
        const size_t nk = (size_t)c.sz.x * c.sz.y * (c.sz.z / 2 + 1);
        if (int e = c.rho.alloc(K * ng)) return e;
        if (int e = c.rho_k.alloc(K * nk)) return e;
        if (int e = c.e_k.alloc(K * 3 * nk)) return e;
        if (int e = c.e_r.alloc(K * 3 * ng)) return e;
        for (int j = 0; j < K; j++) {
            FixChargeEwald *f = b.reps[c.reps[j]]->ewaldFix();
            f->rho.view(c.rho.p + j * ng, ng);
            f->rho_k.view(c.rho_k.p + j * nk, nk);
            f->e_k.view(c.e_k.p + j * 3 * nk, 3 * nk);
            f->e_r.view(c.e_r.p + j * 3 * ng, 3 * ng);
        }
        c.own = true;
        for (int j = 0; j < K; j++) c.own = c.own && b.reps[c.reps[j]]->ewaldFix()->own_fft;
        if (c.own) {
            std::vector<FFTArgs> ft(K);
            for (int j = 0; j < K; j++) ft[j] = fft_args(*b.reps[c.reps[j]], *b.reps[c.reps[j]]->ewaldFix());
            if (int e = c.tab.alloc(K * sizeof(FFTArgs))) return e;
            MDX_CUDA_TRY(cudaMemcpy(c.tab.p, ft.data(), K * sizeof(FFTArgs), cudaMemcpyHostToDevice));
        } else {
            int dims[3] = {c.sz.x, c.sz.y, c.sz.z};
            if (cufftPlanMany(&c.r2c, 3, dims, nullptr, 1, (int)ng, nullptr, 1, (int)nk, CUFFT_R2C, K) !=
                    CUFFT_SUCCESS ||
                cufftPlanMany(&c.c2r, 3, dims, nullptr, 1, (int)nk, nullptr, 1, (int)ng, CUFFT_C2R, 3 * K) !=
                    CUFFT_SUCCESS) {
                set_error(MDX_ERR_CUDA, "batched cufftPlanMany failed");
                return MDX_ERR_CUDA;
            }
        }
        b.max_nk = std::max(b.max_nk, nk);
    }
    b.p3m_own = true;
    for (auto &cp : b.fft) b.p3m_own = b.p3m_own && cp->own;
    std::vector<P3MArgs> h(R);
    for (int r = 0; r < R; r++) h[r] = p3m_args(*b.reps[r], *b.reps[r]->ewaldFix());
    if (int e = b.tab_p3m.alloc(R * sizeof(P3MArgs))) return e;
    MDX_CUDA_TRY(cudaMemcpy(b.tab_p3m.p, h.data(), R * sizeof(P3MArgs), cudaMemcpyHostToDevice));
    // the molecule form of spread and gather, as the single system's fused
    // step: the charged sites of each molecule only, the reciprocal forces
    // stored into each replica's per-step buffer by the P3M branch itself
    b.p3m_mol = b.p3m_own;
    for (State *s : b.reps) b.p3m_mol = b.p3m_mol && s->ewaldFix()->mol_form_ok(*s->rigidFix());
    if (b.p3m_mol) {
        for (int r = 0; r < R; r++) {
            State &s = *b.reps[r];
            h[r] = mol_args(s, *s.ewaldFix(), *s.rigidFix());
            h[r].fs = s.ewaldFix()->f_recip.p;
        }
        if (int e = b.tab_p3m_mol.alloc(R * sizeof(P3MArgs))) return e;
        MDX_CUDA_TRY(cudaMemcpy(b.tab_p3m_mol.p, h.data(), R * sizeof(P3MArgs), cudaMemcpyHostToDevice));
    }
    return 0;
}

int batch_p3m_spread_solve(Batch &b, cudaStream_t st) {
    const unsigned R = (unsigned)b.reps.size();
    const P3MArgs *tab = reinterpret_cast<const P3MArgs *>(b.tab_p3m.p);
    P3MArgs A = p3m_args(*b.reps[0], *b.reps[0]->ewaldFix());  // sizing only
    A.n = b.max_n;
    A.nk = b.max_nk;
    for (auto &c : b.fft) MDX_CUDA_TRY(cudaMemsetAsync(c->rho.p, 0, c->rho.n * sizeof(float), st));
    if (b.p3m_mol) {
        const int warps = (b.max_mol + 1) / 2;
        k_spread_mol<<<dim3((warps + 1) / 2, R), 64, 0, st>>>(A, reinterpret_cast<const P3MArgs *>(b.tab_p3m_mol.p));
    } else {
        k_spread5<<<dim3((A.n + 47) / 48, R), 256, 0, st>>>(A, tab);
    }
    MDX_LAUNCHED();
    if (b.p3m_own) {
        // each mesh class: R2C + E(k) + 3 C2R as the single system's three
        // FFT kernels, one launch each over the class's replicas
        for (auto &c : b.fft) {
            const unsigned K = (unsigned)c->reps.size();
            const FFTArgs a0 = fft_args(*b.reps[c->reps[0]], *b.reps[c->reps[0]]->ewaldFix());
            const FFTArgs *ft = reinterpret_cast<const FFTArgs *>(c->tab.p);
            const int N = c->sz.x, NH = N / 2 + 1;
            const size_t smem = (size_t)N * NH * sizeof(float2);
            if (N == 64) {
                k_fft_zy<2><<<dim3(N, K), kFftPlaneWarps * 32, smem, st>>>(a0, ft);
                k_fft_xe<2><<<dim3((N * NH + 7) / 8, K), 256, 0, st>>>(a0, ft);
                k_ifft_yz<2><<<dim3(N, 3, K), kFftPlaneWarps * 32, smem, st>>>(a0, ft);
            } else {
                k_fft_zy<1><<<dim3(N, K), kFftPlaneWarps * 32, smem, st>>>(a0, ft);
                k_fft_xe<1><<<dim3((N * NH + 7) / 8, K), 256, 0, st>>>(a0, ft);
                k_ifft_yz<1><<<dim3(N, 3, K), kFftPlaneWarps * 32, smem, st>>>(a0, ft);
            }
            g_launches += 3;
        }
        MDX_CUDA_TRY(cudaGetLastError());
        return 0;
    }
    for (auto &c : b.fft) {
        cufftSetStream(c->r2c, st);
        if (cufftExecR2C(c->r2c, c->rho.p, (cufftComplex *)c->rho_k.p) != CUFFT_SUCCESS) {
            set_error(MDX_ERR_CUDA, "batched cufftExecR2C failed");
            return MDX_ERR_CUDA;
        }
    }
    k_efield<<<dim3((unsigned)((A.nk + 255) / 256), R), 256, 0, st>>>(A, tab);
    MDX_LAUNCHED();
    for (auto &c : b.fft) {
        cufftSetStream(c->c2r, st);
        if (cufftExecC2R(c->c2r, (cufftComplex *)c->e_k.p, c->e_r.p) != CUFFT_SUCCESS) {
            set_error(MDX_ERR_CUDA, "batched cufftExecC2R failed");
            return MDX_ERR_CUDA;
        }
    }
    return 0;
}

int batch_p3m_gather(Batch &b, cudaStream_t st) {
    const P3MArgs *tab = reinterpret_cast<const P3MArgs *>(b.tab_p3m.p);
    P3MArgs A = p3m_args(*b.reps[0], *b.reps[0]->ewaldFix());
    A.n = b.max_n;
    if (b.p3m_mol) {  // into each replica's per-step buffer (the second half adds it)
        const int warps = (b.max_mol + 1) / 2;
        k_gather_mol<<<dim3((warps + 1) / 2, (unsigned)b.reps.size()), 64, 0, st>>>(
            A, reinterpret_cast<const P3MArgs *>(b.tab_p3m_mol.p), (const float4 *)nullptr);
        MDX_LAUNCHED();
        return 0;
    }
    if (b.p3m_own) {
        k_gather4_tab<true><<<dim3((A.n + 47) / 48, (unsigned)b.reps.size()), 256, 0, st>>>(A, tab);
        MDX_LAUNCHED();
        return 0;
    }
    k_gather<true><<<dim3((A.n + 127) / 128, (unsigned)b.reps.size()), 128, 0, st>>>(A, tab);
    MDX_LAUNCHED();
    return 0;
}

}  // namespace mdx
