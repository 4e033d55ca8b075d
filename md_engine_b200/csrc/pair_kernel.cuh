// The per-site pair kernel (compute_force_iso, PairEvaluateIso.h:8-207) as
// templates over the pair evaluator and the charge evaluator it carries,
// shared by the translation units that instantiate its forms (pair.cu: LJ/cut
// and WCA with Ewald or no charges; pair_styles.cu: the other evaluators and
// the shifted-force charge pair term).
//
// Pair evaluators (LJ template value): 0 none; 1 LJ/cut (PairEvaluatorLJ.h
// :17-60); 2 WCA (PairEvaluatorWCA.h:13-38); 3 force-shifted LJ
// (PairEvaluatorLJFS.h:15-57); 4 CHARMM LJ with 1-4 parameters
// (PairEvaluatorCHARMM.h:7-44); 5 TICG soft-sphere overlap
// (PairEvaluatorTICG.h:9-52).  Parameter tables per type pair, in the
// reference's paramOrder: {rc^2, 24 eps, sig^6} (1, 2), + F(rc) (3),
// + 24 eps14, sig14^6 (4), {rc^2, C} (5).
// Charge evaluators (CK): 0 none; 1 Ewald real space with the excluded-pair
// correction (ChargeEvaluatorEwald.h:11-64); 2 damped shifted force
// (ChargeEvaluatorDSF.h:13-47).
#pragma once

#include "engine.hpp"

namespace mdx {
namespace pk {

// threads per block of the pair kernel: small blocks retire and refill SM
// slots finely, beside the P3M chain on another stream (measured against 256:
// water step +1.8 %, LJ +2.4 %)
constexpr int kPairBlock = 64;

template <int T>
__device__ __forceinline__ float team_sum(float v) {
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct PairArgs {
    int n;
    const float4 *__restrict__ xs;
    float4 *__restrict__ fs;
    const float *__restrict__ qs;
    const uint32_t *__restrict__ counts;
    const uint32_t *__restrict__ nlist;
    int cap;
    const float *__restrict__ params;
    int np;  // parameters per type pair
    int ntypes;
    Box box;
    float coef1, coef2, coef3;
    float qrc2, alpha, qqr;
    // damped shifted force charges (CK 2): 2 alpha / sqrt(pi), the force
    // shift, erfc(alpha rc) / rc and rc of the charge cutoff
    float dsf_A, dsf_shift, dsf_ecut, dsf_rc;
    float *__restrict__ virials;
    float *__restrict__ energy;  // per-atom (energy kernel)
    uint32_t lj_types;           // bit ti: type ti has a pair with eps != 0
    // GridGPU's own list layout instead of this library's (null: this
    // library's): per-block padded rows located by cumulSumMaxPerBlock for
    // ref_ntpb threads per block, counts as uint16 (GridGPU.cu:777-821,
    // cutils_func.h:23-45)
    const uint32_t *__restrict__ cum;
    const uint16_t *__restrict__ counts16;
    int ref_ntpb;
};

// erfc(x) for x >= 0 by Abramowitz & Stegun, Handbook of Mathematical
// Functions, eq. 7.1.26 (|error| <= 1.5e-7): erfc(x) = t P5(t) exp(-x^2) with
// t = 1 / (1 + p x).  exp(-x^2) is passed in: the Ewald force needs it anyway.
__device__ __forceinline__ float erfc_as(float x, float expmx2) {
    // t only feeds the A&S polynomial (error 1.5e-7): the approximate
    // reciprocal (one SFU op, a few ulp) is plenty
    const float t = rcp_ftz(fmaf(0.3275911f, x, 1.0f));
    float poly = fmaf(t, 1.061405429f, -1.453152027f);
    poly = fmaf(t, poly, 1.421413741f);
    poly = fmaf(t, poly, -0.284496736f);
    poly = fmaf(t, poly, 0.254829592f);
    return t * poly * expmx2;
}

// one neighbour: returns the scalar force factor (F = dr * s) and energy
template <int LJ, int CK, bool ENERGY>
__device__ __forceinline__ bool pair_term(const PairArgs &A, const float *sp, int nt2, int ti, float qi, float4 xj,
                                          float qj, float3 dr, float r2, float mult, float &s, float &e) {
    bool any = false;
    s = 0.f;
    e = 0.f;
    if (LJ) {
        const int tj = type_of(xj);
        const int ix = ti * A.ntypes + tj;
        const float rc2 = sp[ix];
        if (r2 < rc2) {
            any = true;
            if (LJ == 5) {
                // TICG: F = -C 3/2 (r^2/rc^2 - 1) / (rc r), E = C/2 (x-1)^2 (x+2)/2, x = r/rc
                const float C = sp[nt2 + ix];
                if (mult != 0.f && C != 0.f && r2 != 0.f) {
                    s += -C * 1.5f * rsqrt_ftz(rc2 * r2) * (r2 / rc2 - 1.0f) * mult;
                    if (ENERGY) {
                        const float x = sqrtf(r2 / rc2);
                        e += 0.5f * C * (0.5f * (x - 1.0f) * (x - 1.0f) * (x + 2.0f)) * mult;
                    }
                }
            } else {
                float eps24 = sp[nt2 + ix], sig6 = sp[2 * nt2 + ix];
                // CHARMM: a pair whose multiplier is the 1-4 one takes the 1-4
                // parameters (isNorm = multiplier != mult14)
                if (LJ == 4 && mult == A.coef3) {
                    eps24 = sp[3 * nt2 + ix];
                    sig6 = sp[4 * nt2 + ix];
                }
                // eps = 0 (e.g. TIP4P/2005 H and M sites) contributes exactly zero
                if (mult != 0.f && eps24 != 0.f) {
                    const float p1 = eps24 * 2.f * sig6 * sig6;
                    const float p2 = eps24 * sig6;
                    const float r2inv = 1.0f / r2;
                    const float r6inv = r2inv * r2inv * r2inv;
                    float fs = r6inv * r2inv * (p1 * r6inv - p2);
                    if (LJ == 3) fs -= sp[3 * nt2 + ix] * rsqrtf(r2);  // minus F(rc) / r
                    s += fs * mult;
                    if (ENERGY) {
                        const float eps = eps24 / 24.0f;
                        const float s6r6 = sig6 * r6inv;
                        if (LJ == 2) {
                            e += 0.5f * (4.0f * eps * s6r6 * (s6r6 - 1.0f) + eps) * mult;
                        } else {
                            const float rc6 = rc2 * rc2 * rc2;
                            const float s6rc6 = sig6 / rc6;
                            const float off = s6rc6 * (s6rc6 - 1.0f);
                            float u = 4.0f * eps * (s6r6 * (s6r6 - 1.0f) - off);
                            // + F(rc) (r - rc): the force-consistent sign of the
                            // linear term (the reference's comment at
                            // PairEvaluatorLJFS.h:41-44; its code adds F(rc) (rc - r))
                            if (LJ == 3) u += sp[3 * nt2 + ix] * (sqrtf(r2) - sqrtf(rc2));
                            e += 0.5f * u * mult;
                        }
                    }
                }
            }
        }
    }
    if (CK == 1) {
        // q_i q_j = 0 (e.g. the TIP4P/2005 oxygen) contributes exactly zero
        if (r2 < A.qrc2 && qi * qj != 0.f) {
            any = true;
            const float r2c = r2 < 1e-10f ? 1e-10f : r2;
            const float rinv = rsqrt_ftz(r2c);
            const float r2inv = rinv * rinv;
            const float x = A.alpha * (r2c * rinv);  // alpha r
            const float expm = exp_neg_sq(x);        // exp(-alpha^2 r^2) (the reference: __expf)
            const float qq = A.qqr * qi * qj;
            const float erfcv = erfc_as(x, expm);
            float fsc = qq * (erfcv * rinv + (2.0f * 0.5641895835477563f * A.alpha) * expm);
            if (mult < 1.0f) fsc -= (1.0f - mult) * qq * rinv;
            s += fsc * r2inv;
            if (ENERGY) {
                float eng = qq * rinv * erfcv;
                if (mult < 1.0f) eng -= (1.0f - mult) * qq * rinv;
                e += 0.5f * eng;
            }
        }
    }
    if (CK == 2) {
        // damped shifted force: F = qq (erfc(a r)/r^2 + A e^{-a^2 r^2}/r - shift)/r,
        // E = qq (erfc(a r)/r - erfc(a rc)/rc + shift (r - rc)), both times mult
        if (r2 < A.qrc2 && qi * qj != 0.f) {
            any = true;
            const float rinv = rsqrt_ftz(r2);
            const float r2inv = rinv * rinv;
            const float len = r2 * rinv;
            const float x = A.alpha * len;
            const float expm = exp_neg_sq(x);
            const float erfcv = erfc_as(x, expm);
            const float qq = A.qqr * qi * qj;
            s += qq * (erfcv * r2inv + A.dsf_A * expm * rinv - A.dsf_shift) * rinv * mult;
            if (ENERGY) e += 0.5f * qq * (erfcv * rinv - A.dsf_ecut + A.dsf_shift * (len - A.dsf_rc)) * mult;
        }
    }
    return any;
}

// one lane's share of atom i's row: U entries per trip -- all list loads,
// then all position and charge gathers, then the arithmetic, so U memory
// chains are in flight per lane instead of one dependent list->position chain
template <int T, int LJ, int CK, bool VIR, bool ENERGY>
__device__ __forceinline__ void pair_row(const PairArgs &A, const float *sp, int nt2, int i, int ti, float qi,
                                         float4 xi, const uint32_t *row, int cnt, int t, float &fx, float &fy,
                                         float &fz, float &en, float (&v)[6]) {
    // entries per lane per trip: a full-warp team (long water rows) keeps
    // three in flight within its 40-register cap (measured at 24 blocks per
    // SM: U = 3 vs 2, pair 35.1 -> 33.4 us; U = 4 at the old 256-thread
    // shape cost registers and resident warps beside the P3M chain)
    constexpr int U = T >= 32 ? 3 : 4;
    constexpr uint32_t kNone = 0xffffffffu;
    for (int k0 = t; k0 < cnt; k0 += U * T) {
        uint32_t ent[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + u * T;
            ent[u] = k < cnt ? __ldg(row + (size_t)(k / T) * 32) : kNone;
        }
        float4 xj[U];
        float qj[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int j = ent[u] == kNone ? i : (int)(ent[u] & kExclMask);
            xj[u] = __ldg(A.xs + j);
            qj[u] = CK ? __ldg(A.qs + j) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (ent[u] == kNone) continue;
            const uint32_t tag = ent[u] >> 30;
            float mult = 1.0f;
            if (tag) mult = tag == 1u ? A.coef1 : (tag == 2u ? A.coef2 : A.coef3);
            const float3 dr = min_image(A.box, make_float3(xi.x - xj[u].x, xi.y - xj[u].y, xi.z - xj[u].z));
            const float r2 = dot3(dr, dr);
            float s, eng;
            if (pair_term<LJ, CK, ENERGY>(A, sp, nt2, ti, qi, xj[u], qj[u], dr, r2, mult, s, eng)) {
                const float Fx = dr.x * s, Fy = dr.y * s, Fz = dr.z * s;
                fx += Fx;
                fy += Fy;
                fz += Fz;
                if (ENERGY) en += eng;
                if (VIR) {
                    v[0] += Fx * dr.x;
                    v[1] += Fy * dr.y;
                    v[2] += Fz * dr.z;
                    v[3] += Fx * dr.y;
                    v[4] += Fx * dr.z;
                    v[5] += Fy * dr.z;
                }
            }
        }
    }
}

// tab: one argument record per replica (batched launch, blockIdx.y = replica)
// or null (single system, a0).  With both LJ and Ewald terms, a warp whose
// atoms have no LJ partner type (water H, M) runs the row without the LJ
// term, and one whose atoms are all uncharged (water O) without the Ewald
// term: both contribute exactly zero there, and the choice is warp-uniform.
// The full-warp team (long water rows) is latency bound on the x_j gathers:
// capped at 40 registers it keeps 24 blocks (48 warps) per SM (measured:
// pair 36.9 -> 35.1 us, water step +0 to +3 %); other teams are left alone
template <int T, int LJ, int CK, bool VIR, bool ENERGY>
__global__ void __launch_bounds__(kPairBlock, T >= 32 ? 24 : 1) k_pair(const PairArgs a0, const PairArgs *__restrict__ tab, int accumulate) {
    pdl_wait();
    const PairArgs A = tab ? tab[blockIdx.y] : a0;
    extern __shared__ float sp[];
    const int nt2 = A.ntypes * A.ntypes;
    if (LJ) {
        for (int k = threadIdx.x; k < A.np * nt2; k += blockDim.x) sp[k] = A.params[k];
        __syncthreads();
    }
    constexpr int G = 32 / T;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / T, t = lane % T;
    const int i = warp * G + a;
    const bool valid = i < A.n;
    float fx = 0.f, fy = 0.f, fz = 0.f, en = 0.f;
    float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    int ti = 0, cnt = 0;
    float qi = 0.f;
    const uint32_t *row = nullptr;
    if (valid) {
        xi = A.xs[i];
        ti = type_of(xi);
        qi = CK ? A.qs[i] : 0.f;
        if (A.cum) {
            // GridGPU layout: block b of ref_ntpb threads holds ref_ntpb / T
            // atoms; its warps' rows start at (ref_ntpb / 32) * cum[b] and are
            // cum[b+1] - cum[b] entries apart; entry k sits 32 * (k / T) on
            const int per_block = A.ref_ntpb / T;
            const int blk = i / per_block, nth = i % per_block;
            const uint32_t c0 = A.cum[blk], mem = A.cum[blk + 1] - c0;
            row = A.nlist + (size_t)(A.ref_ntpb / 32) * c0 + (size_t)mem * (nth / G) + (nth % G) * T + t;
            cnt = (int)A.counts16[i];
        } else {
            cnt = (int)A.counts[i];
            cnt = cnt < A.cap ? cnt : A.cap;
            row = A.nlist + (size_t)(i / G) * A.cap * G + a * T + t;
        }
    }
    if (LJ && CK) {
        const bool lj_row = valid && ti < 32 && ((A.lj_types >> ti) & 1u);
        const bool q_row = valid && qi != 0.f;
        if (!__any_sync(0xffffffffu, lj_row)) {
            if (valid) pair_row<T, 0, CK, VIR, ENERGY>(A, sp, nt2, i, ti, qi, xi, row, cnt, t, fx, fy, fz, en, v);
        } else if (!__any_sync(0xffffffffu, q_row)) {
            if (valid) pair_row<T, LJ, 0, VIR, ENERGY>(A, sp, nt2, i, ti, qi, xi, row, cnt, t, fx, fy, fz, en, v);
        } else if (valid) {
            pair_row<T, LJ, CK, VIR, ENERGY>(A, sp, nt2, i, ti, qi, xi, row, cnt, t, fx, fy, fz, en, v);
        }
    } else if (valid) {
        pair_row<T, LJ, CK, VIR, ENERGY>(A, sp, nt2, i, ti, qi, xi, row, cnt, t, fx, fy, fz, en, v);
    }
    // late trigger (row loop done): the next kernel's blocks take SM slots
    // as this grid drains; its griddepcontrol.wait still waits for the stores
    pdl_trigger();
    // invalid lanes carry zeros; whole warp takes part in the shuffles
    if (ENERGY) {
        en = team_sum<T>(en);
        if (valid && t == 0) A.energy[i] = en;
        return;
    }
    fx = team_sum<T>(fx);
    fy = team_sum<T>(fy);
    fz = team_sum<T>(fz);
    if (VIR) {
#pragma unroll
        for (int c = 0; c < 6; c++) v[c] = team_sum<T>(v[c]);
    }
    if (valid && t == 0) {
        float4 f = A.fs[i];
        if (accumulate) {
            f.x += fx;
            f.y += fy;
            f.z += fz;
        } else {
            f.x = fx;
            f.y = fy;
            f.z = fz;
        }
        A.fs[i] = f;
        if (VIR) {
            float *vv = A.virials + 6 * (size_t)i;
#pragma unroll
            for (int c = 0; c < 6; c++) vv[c] += 0.5f * v[c];
        }
    }
}

// nrep > 1: tab holds nrep records, A is the largest replica (grid sizing)
template <int T, int LJ, int CK>
void launch_t(const PairArgs &A, const PairArgs *tab, int nrep, bool vir, bool energy, bool accumulate,
              cudaStream_t st) {
    const int G = 32 / T;
    const int warps = (A.n + G - 1) / G;
    const dim3 blocks((warps * 32 + kPairBlock - 1) / kPairBlock, nrep);
    const size_t smem = LJ ? (size_t)A.np * A.ntypes * A.ntypes * sizeof(float) : 0;
    if (energy) {
        k_pair<T, LJ, CK, false, true><<<blocks, kPairBlock, smem, st>>>(A, tab, 0);
        MDX_LAUNCHED();
    } else if (vir) {
        k_pair<T, LJ, CK, true, false><<<blocks, kPairBlock, smem, st>>>(A, tab, accumulate ? 1 : 0);
        MDX_LAUNCHED();
    } else {
        launch_pdl(k_pair<T, LJ, CK, false, false>, blocks, dim3(kPairBlock), smem, st, A, tab, accumulate ? 1 : 0);
    }
}


// the pair / charge evaluator pairs outside pair.cu's set (pair_styles.cu)
int pair_launch_styles(const PairArgs &A, const PairArgs *tab, int nrep, int team, int lj, int ck, bool vir,
                       bool energy, bool acc, cudaStream_t st);

}  // namespace pk
}  // namespace mdx
