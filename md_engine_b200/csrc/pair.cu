// Short-range pair forces: LJ/cut or WCA plus the Ewald real-space term
// offloaded into the same kernel (compute_force_iso, PairEvaluateIso.h:8-207,
// with EvaluatorLJ PairEvaluatorLJ.h:17-60, EvaluatorWCA PairEvaluatorWCA.h:13-38,
// ChargeEvaluatorEwald ChargeEvaluatorEwald.h:11-64; charge offload
// State.cpp:648-660).
//
// Layout: a team of T lanes per atom i walks i's neighbour row; a warp covers
// 32/T atoms, so every list load is one 128-byte row.  Per-type-pair
// parameters {rc^2, 24 eps, sig^6} sit in shared memory (the reference's
// paramsCoalesced order).  The team's partial forces (and the optional
// per-atom virial, x0.5 as helpers.h:34-41 / PairEvaluateIso.h:180-195) are
// reduced with register shuffles, not shared memory.
#include <cmath>
#include <cstdio>

#include "pair_kernel.cuh"

namespace mdx {

namespace {

using pk::PairArgs;
using pk::kPairBlock;

// LJ/cut and WCA with Ewald or no charges (the other pair and charge
// evaluators: pair_styles.cu)
template <int T>
int launch_kind(const PairArgs &A, const PairArgs *tab, int nrep, int lj, int ck, bool vir, bool energy, bool acc,
                cudaStream_t st) {
    if (lj == 0 && ck == 1) pk::launch_t<T, 0, 1>(A, tab, nrep, vir, energy, acc, st);
    else if (lj == 1 && ck == 1) pk::launch_t<T, 1, 1>(A, tab, nrep, vir, energy, acc, st);
    else if (lj == 1 && ck == 0) pk::launch_t<T, 1, 0>(A, tab, nrep, vir, energy, acc, st);
    else if (lj == 2 && ck == 1) pk::launch_t<T, 2, 1>(A, tab, nrep, vir, energy, acc, st);
    else if (lj == 2 && ck == 0) pk::launch_t<T, 2, 0>(A, tab, nrep, vir, energy, acc, st);
    else return pk::pair_launch_styles(A, tab, nrep, T, lj, ck, vir, energy, acc, st);
    return 0;
}

int launch_any(const PairArgs &A, int team, int lj, int ck, bool vir, bool energy, bool acc, cudaStream_t st,
               const PairArgs *tab = nullptr, int nrep = 1) {
    switch (team) {
        case 1: return launch_kind<1>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 2: return launch_kind<2>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 4: return launch_kind<4>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 8: return launch_kind<8>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 16: return launch_kind<16>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 32: return launch_kind<32>(A, tab, nrep, lj, ck, vir, energy, acc, st);
    }
    set_error(MDX_ERR_ARG, "team size %d not in {1,2,4,8,16,32}", team);
    return MDX_ERR_ARG;
}

// the charge evaluator the pair fix carries: 0 none, 1 Ewald, 2 DSF
int charge_kind(const FixPair &f) { return f.chargeFix ? 1 : (f.dsfFix ? 2 : 0); }

PairArgs make_args(State &s, FixPair &f) {
    PairArgs A;
    A.n = s.gpd.n;
    A.xs = s.gpd.xs.p;
    A.fs = s.gpd.fs.p;
    A.qs = s.gpd.qs.p;
    A.counts = s.grid.partition ? s.grid.counts_int.p : s.grid.counts.p;
    A.nlist = s.grid.nlist.p;
    A.cap = s.grid.cap;
    A.params = f.d_params.p;
    A.np = f.nparam();
    A.ntypes = (int)s.species.size();
    A.box = s.box;
    A.coef1 = s.specialNeighborCoefs[0];
    A.coef2 = s.specialNeighborCoefs[1];
    A.coef3 = s.specialNeighborCoefs[2];
    A.qrc2 = 0.f;
    A.alpha = 0.f;
    A.qqr = (float)s.units.qqr_to_eng;
    A.dsf_A = A.dsf_shift = A.dsf_ecut = A.dsf_rc = 0.f;
    if (f.chargeFix) {
        float qrc = (float)f.chargeRCut;
        A.qrc2 = qrc * qrc;
        A.alpha = (float)f.chargeFix->alpha;
    } else if (f.dsfFix) {
        // FixChargePairDSF's evaluator (generateEvaluator, FixChargePairDSF.cu)
        const FixChargePairDSF &d = *f.dsfFix;
        const float qrc = (float)d.r_cut;
        A.qrc2 = qrc * qrc;
        A.alpha = (float)d.alpha;
        A.dsf_A = (float)d.A;
        A.dsf_shift = (float)d.shift;
        A.dsf_ecut = (float)(std::erfc(d.alpha * d.r_cut) / d.r_cut);
        A.dsf_rc = qrc;
    }
    A.virials = s.gpd.virials.p;
    A.energy = nullptr;
    A.cum = nullptr;
    A.counts16 = nullptr;
    A.ref_ntpb = 0;
    // types with a pair partner the pair evaluator does not zero
    A.lj_types = 0xffffffffu;
    const int nt = A.ntypes;
    if (nt <= 32 && f.h_params.size() == (size_t)f.nparam() * nt * nt) {
        A.lj_types = 0u;
        for (int x = 0; x < nt; x++)
            for (int y = 0; y < nt; y++)
                if (f.pairActive(x, y)) A.lj_types |= 1u << x;
    }
    return A;
}

// ---- molecule form (all-rigid four-site water) ---------------------------
// One warp per molecule slot k (sites at 4k .. 4k+3, stored whole) walks k's
// molecule-pair list in two phases per 32 entries:
//  * filter: each lane takes one entry j, gathers its site 0 and forms the
//    minimum-image shift of the site-0 pair; entries whose site-0 distance is
//    within `far` (beyond it no site pair is within the cutoffs) are
//    compacted by ballot into a per-warp queue in shared memory;
//  * evaluate: whenever 32 entries are queued, each lane takes one and
//    evaluates every site pair (a of k, b of j) that can interact (bit 4a+b
//    of the LJ / charge masks: eps(a,b) != 0, q_a q_b != 0) as
//    compute_force_iso evaluates a listed pair -- LJ/WCA when
//    r^2 < rc^2(a,b), Ewald real space when r^2 < qrc^2 -- with the one
//    shift of the molecule pair (molecules are whole and a pair within the
//    cutoff is within L/2 under it, so it is the pair's minimum image) and
//    the cutoffs applied as masks, not branches: all lanes run one path.
// The molecule's own site pairs (the excluded pairs of the reference's list,
// multiplier by exclusion depth) are added by lane 0.  Forces on the four
// sites are reduced by shuffles and written by lanes 0..3 (one 64-byte store).
constexpr int kMolPairBlock = 64;
constexpr int kMolQueue = 64;  // queued entries per warp (two chunks)

struct MolPairArgs {
    int nmol;
    const float4 *__restrict__ xs;
    float4 *__restrict__ fs;
    const uint32_t *__restrict__ counts;
    const uint32_t *__restrict__ list;
    int cap;
    Box box;
    float far2, qrc2, alpha;
    uint32_t ljm, qm, selfm;  // bit 4a+b: LJ term, charge term, own-molecule pair
    // per site pair ab: rc^2, 48 eps sig^12, 24 eps sig^6, sig^6, eps, the
    // LJ/cut energy shift at rc, qqr q_a q_b, exclusion multiplier (own pairs)
    float rc2[16], p1[16], p2[16], sig6[16], eps[16], eoff[16], qq[16], mult[16];
    float *__restrict__ virials;
    float *__restrict__ energy;  // per site (energy kernel)
};

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <bool VIR>
__device__ __forceinline__ void add_vir(float (&v)[6], float3 F, float3 dr) {
    if (VIR) {
        v[0] += F.x * dr.x;
        v[1] += F.y * dr.y;
        v[2] += F.z * dr.z;
        v[3] += F.x * dr.y;
        v[4] += F.x * dr.z;
        v[5] += F.y * dr.z;
    }
}

// site pair ab at r2, multiplier mult (1 between molecules; own pairs carry
// their exclusion multiplier and the Ewald correction of the excluded part,
// ChargeEvaluatorEwald.h:11-64): scalar force factor (F = dr s) and half the
// pair energy, cutoffs applied as masks
// TOPO 1: the four-site water pattern known at compile time -- LJ between
// the sites 0 only, charges on sites 1..3 only (ljm = 0x1, qm = 0xEEE0);
// TOPO 0: any pattern, from the runtime masks
template <int TOPO>
__device__ __forceinline__ bool topo_lj(const MolPairArgs &A, int ab) {
    return TOPO == 1 ? ab == 0 : ((A.ljm >> ab) & 1u) != 0u;
}
template <int TOPO>
__device__ __forceinline__ bool topo_q(const MolPairArgs &A, int ab) {
    return TOPO == 1 ? (ab / 4 != 0 && ab % 4 != 0) : ((A.qm >> ab) & 1u) != 0u;
}

template <int LJ, bool EW, bool ENERGY, bool OWN, int TOPO>
__device__ __forceinline__ float mol_pair_term(const MolPairArgs &A, int ab, float r2, float mult, float &e) {
    float s = 0.f;
    e = 0.f;
    if (LJ && topo_lj<TOPO>(A, ab)) {
        const float in = (r2 < A.rc2[ab] && (!OWN || mult != 0.f)) ? (OWN ? mult : 1.0f) : 0.f;
        const float r2inv = rcp_ftz(r2);
        const float r6inv = r2inv * r2inv * r2inv;
        s += r6inv * r2inv * (A.p1[ab] * r6inv - A.p2[ab]) * in;
        if (ENERGY) {
            const float s6r6 = A.sig6[ab] * r6inv;
            if (LJ == 1) e += 0.5f * 4.0f * A.eps[ab] * (s6r6 * (s6r6 - 1.0f) - A.eoff[ab]) * in;
            else e += 0.5f * (4.0f * A.eps[ab] * s6r6 * (s6r6 - 1.0f) + A.eps[ab]) * in;
        }
    }
    if (EW && topo_q<TOPO>(A, ab)) {
        const float r2c = fmaxf(r2, 1e-10f);
        const float rinv = rsqrt_ftz(r2c);
        const float x = A.alpha * (r2c * rinv);
        const float expm = exp_neg_sq(x);
        const float erfcv = pk::erfc_as(x, expm);
        const float qq = A.qq[ab];
        float fsc = qq * (erfcv * rinv + (2.0f * 0.5641895835477563f * A.alpha) * expm);
        if (OWN && mult < 1.0f) fsc -= (1.0f - mult) * qq * rinv;
        const float in = r2 < A.qrc2 ? 1.0f : 0.f;
        s += fsc * (rinv * rinv) * in;
        if (ENERGY) {
            float eng = qq * rinv * erfcv;
            if (OWN && mult < 1.0f) eng -= (1.0f - mult) * qq * rinv;
            e += 0.5f * eng * in;
        }
    }
    return s;
}

// asynchronous 16-byte global -> shared copies (cp.async, cached in L1): a
// batch of neighbour molecules is staged while the warp scans the next chunk
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// one queued molecule pair: every interacting site pair of slot k (sites
// xi, the shift already taken off) and the neighbour's sites xj
template <int LJ, bool EW, bool VIR, bool ENERGY, int TOPO>
__device__ __forceinline__ void mol_pair_eval_x(const MolPairArgs &A, const float3 (&xi)[4], const float3 (&xj)[4],
                                                float3 shift, float3 (&f)[4], float (&en)[4], float (&v)[4][6]) {
    const uint32_t any = TOPO == 1 ? 0xEEE1u : ((LJ ? A.ljm : 0u) | (EW ? A.qm : 0u));
#pragma unroll
    for (int a = 0; a < 4; a++) {
        if (!((any >> (4 * a)) & 15u)) continue;
        const float3 xa = xi[a] - shift;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int ab = 4 * a + b;
            if (!((any >> ab) & 1u)) continue;
            const float3 dr = xa - xj[b];
            const float r2 = dot3(dr, dr);
            float e;
            const float sc = mol_pair_term<LJ, EW, ENERGY, false, TOPO>(A, ab, r2, 1.0f, e);
            const float3 F = dr * sc;
            f[a] += F;
            if (ENERGY) en[a] += e;
            add_vir<VIR>(v[a], F, dr);
        }
    }
}

template <int LJ, bool EW, bool VIR, bool ENERGY, int TOPO>
__device__ __forceinline__ void mol_pair_eval(const MolPairArgs &A, const float3 (&xi)[4], int j, float3 shift,
                                              float3 (&f)[4], float (&en)[4], float (&v)[4][6]) {
    float3 xj[4];
#pragma unroll
    for (int b = 0; b < 4; b++) xj[b] = f3(__ldg(A.xs + 4 * j + b));
    mol_pair_eval_x<LJ, EW, VIR, ENERGY, TOPO>(A, xi, xj, shift, f, en, v);
}

// one warp per molecule slot; the grid strides over the slots, so a grid
// capped below the device's capacity leaves room on every SM for the P3M
// chain's blocks that run beside it.  The row is scanned in 32-entry chunks
// (ids loaded two chunks ahead, first sites one chunk ahead); the entries
// within the far cutoff queue up in shared memory, and each full batch of
// 32 has its four sites staged into shared memory by cp.async while the
// warp scans the next chunk, then is evaluated one entry per lane.
// BATCH: batched replicas, the arguments of replica blockIdx.y from tab
// (a0 unused); otherwise a0
template <int LJ, bool EW, bool VIR, bool ENERGY, int TOPO, bool BATCH = false>
__global__ void __launch_bounds__(kMolPairBlock, 14) k_pair_mol(const MolPairArgs a0,
                                                                const MolPairArgs *__restrict__ tab, int accumulate) {
    pdl_wait();
    const MolPairArgs &A = BATCH ? tab[blockIdx.y] : a0;
    __shared__ int q_j[kMolPairBlock / 32][kMolQueue];
    __shared__ float4 q_s[kMolPairBlock / 32][kMolQueue];
    __shared__ float4 s_b[kMolPairBlock / 32][4][32];  // staged batch: site b of entry lane
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int *const qj = q_j[wib];
    float4 *const qs = q_s[wib];
    float4(*const sb)[32] = s_b[wib];
    const uint32_t lt = (1u << lane) - 1u;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < A.nmol; k += nwarps) {  // warp-uniform
        float3 xi[4], f[4];
        float en[4], v[4][6];
#pragma unroll
        for (int a = 0; a < 4; a++) {
            f[a] = make_float3(0.f, 0.f, 0.f);
            en[a] = 0.f;
#pragma unroll
            for (int c = 0; c < 6; c++) v[a][c] = 0.f;
        }
#pragma unroll
        for (int a = 0; a < 4; a++) xi[a] = f3(A.xs[4 * k + a]);
        int cnt = (int)A.counts[k];
        cnt = cnt < A.cap ? cnt : A.cap;
        const uint32_t *row = A.list + (size_t)k * A.cap;
        int nq = 0;           // queued entries (warp-uniform)
        bool staged = false;  // a batch of 32 queued entries is being copied into sb (warp-uniform)
        float3 bshift = make_float3(0.f, 0.f, 0.f);
        int j_cur = lane < cnt ? (int)__ldg(row + lane) : 0;
        int j_nxt = 32 + lane < cnt ? (int)__ldg(row + 32 + lane) : 0;
        float4 x_cur = lane < cnt ? __ldg(A.xs + 4 * j_cur) : make_float4(0.f, 0.f, 0.f, 0.f);
        for (int base = 0; base < cnt; base += 32) {
            float4 x_nxt = make_float4(0.f, 0.f, 0.f, 0.f);
            if (base + 32 + lane < cnt) x_nxt = __ldg(A.xs + 4 * j_nxt);
            const int j_nn = base + 64 + lane < cnt ? (int)__ldg(row + base + 64 + lane) : 0;
            const int e = base + lane;
            bool pass = false;
            const int j = j_cur;
            float3 sh = make_float3(0.f, 0.f, 0.f);
            if (e < cnt) {
                const float3 d = xi[0] - f3(x_cur);
                sh = make_float3(A.box.L.x * rint_small(d.x * A.box.invL.x),
                                 A.box.L.y * rint_small(d.y * A.box.invL.y),
                                 A.box.L.z * rint_small(d.z * A.box.invL.z));
                const float3 dm = d - sh;
                pass = dot3(dm, dm) < A.far2;
            }
            j_cur = j_nxt;
            j_nxt = j_nn;
            x_cur = x_nxt;
            const uint32_t bal = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                const int pos = nq + __popc(bal & lt);
                qj[pos] = j;
                qs[pos] = make_float4(sh.x, sh.y, sh.z, 0.f);
            }
            nq += __popc(bal);
            __syncwarp();
            // the batch staged one chunk ago: its copies had the scan above to land
            if (staged) {
                cp_async_wait_all();
                __syncwarp();
                float3 xj[4];
#pragma unroll
                for (int b = 0; b < 4; b++) xj[b] = f3(sb[b][lane]);
                mol_pair_eval_x<LJ, EW, VIR, ENERGY, TOPO>(A, xi, xj, bshift, f, en, v);
                staged = false;
                __syncwarp();
            }
            if (nq >= 32) {
                const float4 s4 = qs[lane];
                bshift = make_float3(s4.x, s4.y, s4.z);
                const float4 *src = A.xs + 4 * qj[lane];
#pragma unroll
                for (int b = 0; b < 4; b++) cp_async16(&sb[b][lane], src + b);
                cp_async_commit();
                staged = true;
                __syncwarp();
                nq -= 32;
                if (lane < nq) {
                    qj[lane] = qj[32 + lane];
                    qs[lane] = qs[32 + lane];
                }
                __syncwarp();
            }
        }
        if (staged) {
            cp_async_wait_all();
            __syncwarp();
            float3 xj[4];
#pragma unroll
            for (int b = 0; b < 4; b++) xj[b] = f3(sb[b][lane]);
            mol_pair_eval_x<LJ, EW, VIR, ENERGY, TOPO>(A, xi, xj, bshift, f, en, v);
        }
        if (lane < nq) {
            const float4 s4 = qs[lane];
            mol_pair_eval<LJ, EW, VIR, ENERGY, TOPO>(A, xi, qj[lane], make_float3(s4.x, s4.y, s4.z), f, en, v);
        }
        __syncwarp();  // the queue and the batch are reused by the warp's next slot
        // the molecule's own site pairs, once per molecule
        if (lane == 0 && A.selfm) {
#pragma unroll
            for (int a = 0; a < 4; a++) {
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    const int ab = 4 * a + b;
                    if (a == b || !((A.selfm >> ab) & 1u)) continue;
                    const float3 dr = xi[a] - xi[b];  // the molecule is whole
                    const float r2 = dot3(dr, dr);
                    float e;
                    const float sc = mol_pair_term<LJ, EW, ENERGY, true, 0>(A, ab, r2, A.mult[ab], e);
                    const float3 F = dr * sc;
                    f[a] += F;
                    if (ENERGY) en[a] += e;
                    add_vir<VIR>(v[a], F, dr);
                }
            }
        }
        if (ENERGY) {
#pragma unroll
            for (int a = 0; a < 4; a++) en[a] = warp_sum(en[a]);
            if (lane < 4) A.energy[4 * k + lane] = lane == 0 ? en[0] : (lane == 1 ? en[1] : (lane == 2 ? en[2] : en[3]));
            continue;
        }
#pragma unroll
        for (int a = 0; a < 4; a++) f[a] = make_float3(warp_sum(f[a].x), warp_sum(f[a].y), warp_sum(f[a].z));
        if (VIR) {
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int c = 0; c < 6; c++) v[a][c] = warp_sum(v[a][c]);
        }
        if (lane < 4) {
            const float3 fm = lane == 0 ? f[0] : (lane == 1 ? f[1] : (lane == 2 ? f[2] : f[3]));
            float4 fo = A.fs[4 * k + lane];
            if (accumulate) {
                fo.x += fm.x;
                fo.y += fm.y;
                fo.z += fm.z;
            } else {
                fo.x = fm.x;
                fo.y = fm.y;
                fo.z = fm.z;
            }
            A.fs[4 * k + lane] = fo;
            if (VIR) {
                float *vv = A.virials + 6 * (size_t)(4 * k + lane);
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    const float vm = lane == 0 ? v[0][c] : (lane == 1 ? v[1][c] : (lane == 2 ? v[2][c] : v[3][c]));
                    vv[c] += 0.5f * vm;
                }
            }
        }
    }
    pdl_trigger();
}

MolPairArgs make_mol_args(State &s, FixPair &f) {
    const MolForm &mf = s.mf;
    MolPairArgs A{};
    A.nmol = mf.nmol;
    A.xs = s.gpd.xs.p;
    A.fs = s.gpd.fs.p;
    A.counts = mf.counts.p;
    A.list = mf.list.p;
    A.cap = mf.cap;
    A.box = s.box;
    A.far2 = mf.far * mf.far;
    A.virials = s.gpd.virials.p;
    A.energy = nullptr;
    const int nt = (int)s.species.size();
    const int nt2 = nt * nt;
    const bool ew = f.chargeFix != nullptr;
    A.qrc2 = 0.f;
    A.alpha = 0.f;
    if (ew) {
        const float qrc = (float)f.chargeRCut;
        A.qrc2 = qrc * qrc;
        A.alpha = (float)f.chargeFix->alpha;
    }
    const float qqr = (float)s.units.qqr_to_eng;
    const float coef[3] = {s.specialNeighborCoefs[0], s.specialNeighborCoefs[1], s.specialNeighborCoefs[2]};
    A.ljm = A.qm = A.selfm = 0u;
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
            const int ab = 4 * a + b;
            const int ix = mf.type[a] * nt + mf.type[b];
            // the same FP32 products as the per-site kernel forms them
            const float rc2 = f.h_params[ix], eps24 = f.h_params[nt2 + ix], sig6 = f.h_params[2 * nt2 + ix];
            A.rc2[ab] = rc2;
            A.p1[ab] = eps24 * 2.f * sig6 * sig6;
            A.p2[ab] = eps24 * sig6;
            A.sig6[ab] = sig6;
            A.eps[ab] = eps24 / 24.0f;
            const float rc6 = rc2 * rc2 * rc2;
            const float s6rc6 = sig6 / rc6;
            A.eoff[ab] = s6rc6 * (s6rc6 - 1.0f);
            A.qq[ab] = qqr * mf.q[a] * mf.q[b];
            const int dep = mf.depth[ab];
            A.mult[ab] = dep == 0 ? 1.0f : coef[dep - 1];
            if (eps24 != 0.f) A.ljm |= 1u << ab;
            if (ew && mf.q[a] * mf.q[b] != 0.f) A.qm |= 1u << ab;
            if (a != b) A.selfm |= 1u << ab;
        }
    return A;
}

template <int LJ, bool EW, int TOPO>
void mol_launch_t(const MolPairArgs &A, int virialMode, bool energy, bool accumulate, int max_blocks,
                  cudaStream_t st) {
    int nb = (A.nmol * 32 + kMolPairBlock - 1) / kMolPairBlock;
    if (max_blocks > 0 && nb > max_blocks) nb = max_blocks;
    const dim3 blocks(nb > 0 ? nb : 1);
    const MolPairArgs *nt = nullptr;
    if (energy) {
        k_pair_mol<LJ, EW, false, true, TOPO><<<blocks, kMolPairBlock, 0, st>>>(A, nt, 0);
        MDX_LAUNCHED();
    } else if (virialMode == 1 || virialMode == 2) {
        k_pair_mol<LJ, EW, true, false, TOPO><<<blocks, kMolPairBlock, 0, st>>>(A, nt, accumulate ? 1 : 0);
        MDX_LAUNCHED();
    } else {
        launch_pdl(k_pair_mol<LJ, EW, false, false, TOPO>, blocks, dim3(kMolPairBlock), 0, st, A, nt,
                   accumulate ? 1 : 0);
    }
}

}  // namespace

int pair_launch(State &s, FixPair &f, int virialMode, bool accumulate) {
    if (s.mf.on) return pair_mol_launch(s, f, virialMode, accumulate, nullptr, s.stream);
    PairArgs A = make_args(s, f);
    bool vir = virialMode == 1 || virialMode == 2;
    return launch_any(A, s.grid.team, f.lj_kind, charge_kind(f), vir, false, accumulate, s.stream);
}

// the molecule form of the pair forces (energy: per-site energies into
// `energy` instead of forces)
int pair_mol_launch(State &s, FixPair &f, int virialMode, bool accumulate, float *energy, cudaStream_t st) {
    MolPairArgs A = make_mol_args(s, f);
    A.energy = energy;
    const bool ew = f.chargeFix != nullptr;
    const bool en = energy != nullptr;
    if (f.lj_kind != 1 && f.lj_kind != 2) {
        set_error(MDX_ERR_ARG, "pair kind %d", f.lj_kind);
        return MDX_ERR_ARG;
    }
    // the four-site water pattern (LJ on sites 0, charges on 1..3) as
    // compile-time masks; any other pattern from the runtime masks
    const bool water4 = ew && A.ljm == 0x1u && A.qm == 0xEEE0u;
    // blocks per SM of the grid.  Automatic: a pair block holds its SM for
    // most of the kernel (one molecule per warp, one wave), so with every SM
    // full the P3M chain beside it (all-rigid water) waits for the pair
    // kernel at each of its launches; a grid capped below the SMs' capacity
    // keeps room for it (measured on B200, 4,096 molecules: 10 blocks per SM
    // without E3B, 7 with the E3B kernel as a third branch).  Else uncapped.
    int bps = s.pairBlocksPerSM;
    if (bps == 0) {
        const bool p3m_beside = ew && s.rigidFix() && !has_free_atoms(s);
        bps = p3m_beside ? (s.e3bFix() ? 7 : 10) : -1;
    }
    const int mb = bps > 0 ? bps * num_sms() : 0;
    if (f.lj_kind == 1 && water4) mol_launch_t<1, true, 1>(A, virialMode, en, accumulate, mb, st);
    else if (f.lj_kind == 1 && ew) mol_launch_t<1, true, 0>(A, virialMode, en, accumulate, mb, st);
    else if (f.lj_kind == 1) mol_launch_t<1, false, 0>(A, virialMode, en, accumulate, mb, st);
    else if (water4) mol_launch_t<2, true, 1>(A, virialMode, en, accumulate, mb, st);
    else if (ew) mol_launch_t<2, true, 0>(A, virialMode, en, accumulate, mb, st);
    else mol_launch_t<2, false, 0>(A, virialMode, en, accumulate, mb, st);
    return 0;
}

// compute_energy_iso (PairEvaluateIso.h:212-358): per-site energies into the
// state's energy buffer, summed on the device in FP64 in a fixed order
int pair_energy(State &s, FixPair &f, double *out) {
    PairArgs A = make_args(s, f);
    if (s.e_site.n < (size_t)A.n || !s.e_sum.p) {
        set_error(MDX_ERR_STATE, "energy buffers not sized (prepare the state)");
        return MDX_ERR_STATE;
    }
    A.energy = s.e_site.p;
    if (s.mf.on) {
        if (int r = pair_mol_launch(s, f, 0, false, s.e_site.p, s.stream)) return r;
    } else if (int r = launch_any(A, s.grid.team, f.lj_kind, charge_kind(f), false, true, false, s.stream)) {
        return r;
    }
    return float_sum(s, s.e_site.p, A.n, out);
}

// batched replicas: one launch per form, blockIdx.y = replica of that form;
// tables built at prepare
int batch_pair_tables(Batch &b) {
    const int P = (int)b.ps.size(), Q = (int)b.mfi.size();
    if (P) {
        std::vector<PairArgs> h(P);
        b.pair_big = b.ps[0];
        for (int q = 0; q < P; q++) {
            State &s = *b.reps[b.ps[q]];
            h[q] = make_args(s, *s.pairFix());
            if (s.gpd.n > b.reps[b.pair_big]->gpd.n) b.pair_big = b.ps[q];
        }
        if (int e = b.tab_pair.alloc(P * sizeof(PairArgs))) return e;
        MDX_CUDA_TRY(cudaMemcpy(b.tab_pair.p, h.data(), P * sizeof(PairArgs), cudaMemcpyHostToDevice));
    }
    if (Q) {
        // one kernel instance serves these replicas: their force fields
        // must give the same compile-time pattern
        std::vector<MolPairArgs> hm(Q);
        const FixPair &f0 = *b.reps[b.mfi[0]]->pairFix();
        for (int q = 0; q < Q; q++) {
            State &s = *b.reps[b.mfi[q]];
            const FixPair &f = *s.pairFix();
            hm[q] = make_mol_args(s, *s.pairFix());
            hm[q].energy = nullptr;
            if (hm[q].ljm != hm[0].ljm || hm[q].qm != hm[0].qm || f.lj_kind != f0.lj_kind ||
                (f.chargeFix != nullptr) != (f0.chargeFix != nullptr)) {
                set_error(MDX_ERR_UNSUPPORTED, "batched replicas must share one pair style and site pattern (replica %d)",
                          b.mfi[q]);
                return MDX_ERR_UNSUPPORTED;
            }
        }
        if (int e = b.tab_pairmol.alloc(Q * sizeof(MolPairArgs))) return e;
        MDX_CUDA_TRY(cudaMemcpy(b.tab_pairmol.p, hm.data(), Q * sizeof(MolPairArgs), cudaMemcpyHostToDevice));
    }
    return 0;
}

// the molecule-form replicas: one warp per molecule slot, the grid (slots
// of the largest of them, replicas) with blocks past a smaller replica's
// slots idle
template <int LJ, bool EW, int TOPO>
static void batch_mol_launch_t(const MolPairArgs &A, const MolPairArgs *tab, int Q, cudaStream_t st) {
    const int nb = (A.nmol * 32 + kMolPairBlock - 1) / kMolPairBlock;
    k_pair_mol<LJ, EW, false, false, TOPO, true><<<dim3(nb > 0 ? nb : 1, Q), kMolPairBlock, 0, st>>>(A, tab, 0);
    MDX_LAUNCHED();
}

static int batch_pair_mol_launch(Batch &b, cudaStream_t stream) {
    const int Q = (int)b.mfi.size();
    State &s0 = *b.reps[b.mfi[0]];
    FixPair &f = *s0.pairFix();
    MolPairArgs A = make_mol_args(s0, f);  // sizing and pattern only: the kernel reads tab
    A.nmol = b.max_mol_mf;
    const MolPairArgs *tab = reinterpret_cast<const MolPairArgs *>(b.tab_pairmol.p);
    const bool ew = f.chargeFix != nullptr;
    const bool water4 = ew && A.ljm == 0x1u && A.qm == 0xEEE0u;
    if (f.lj_kind == 1 && water4) batch_mol_launch_t<1, true, 1>(A, tab, Q, stream);
    else if (f.lj_kind == 1 && ew) batch_mol_launch_t<1, true, 0>(A, tab, Q, stream);
    else if (f.lj_kind == 1) batch_mol_launch_t<1, false, 0>(A, tab, Q, stream);
    else if (water4) batch_mol_launch_t<2, true, 1>(A, tab, Q, stream);
    else if (ew) batch_mol_launch_t<2, true, 0>(A, tab, Q, stream);
    else batch_mol_launch_t<2, false, 0>(A, tab, Q, stream);
    return 0;
}

int batch_pair_launch(Batch &b, cudaStream_t stream) {
    if ((!b.ps.empty() && !b.tab_pair.p) || (!b.mfi.empty() && !b.tab_pairmol.p)) {
        set_error(MDX_ERR_STATE, "batch tables not built (prepare the batch)");
        return MDX_ERR_STATE;
    }
    if (!b.ps.empty()) {
        State &big = *b.reps[b.pair_big];
        FixPair &f = *big.pairFix();
        const PairArgs A = make_args(big, f);
        if (int e = launch_any(A, big.grid.team, f.lj_kind, charge_kind(f), false, false, true, stream,
                               reinterpret_cast<const PairArgs *>(b.tab_pair.p), (int)b.ps.size()))
            return e;
    }
    if (!b.mfi.empty())
        if (int e = batch_pair_mol_launch(b, stream)) return e;
    return 0;
}

int pair_force_raw(int n, const float4 *xs, float4 *fs, const float *qs, const uint32_t *counts,
                   const uint32_t *nlist, int team, int cap, const float *params, int ntypes, const Box &box,
                   const float coef[3], int lj_kind, float qrc, float alpha, float qqr, float *virials,
                   bool accumulate, cudaStream_t stream) {
    PairArgs A;
    A.n = n;
    A.xs = xs;
    A.fs = fs;
    A.qs = qs;
    A.counts = counts;
    A.nlist = nlist;
    A.cap = cap;
    A.params = params;
    A.ntypes = ntypes;
    A.box = box;
    A.coef1 = coef[0];
    A.coef2 = coef[1];
    A.coef3 = coef[2];
    A.dsf_A = A.dsf_shift = A.dsf_ecut = A.dsf_rc = 0.f;
    A.qrc2 = qrc > 0.f ? qrc * qrc : 0.f;
    A.alpha = alpha;
    A.qqr = qqr;
    A.virials = virials;
    A.energy = nullptr;
    A.lj_types = 0xffffffffu;  // parameters live on the device here: no skipping
    A.cum = nullptr;
    A.counts16 = nullptr;
    A.ref_ntpb = 0;
    bool ew = qrc > 0.f;
    if (lj_kind == 0 && !ew) return 0;
    A.np = 3;
    int r = launch_any(A, team, lj_kind, ew ? 1 : 0, virials != nullptr, false, accumulate, stream);
    if (r) return r;
    MDX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// EvaluatorWrapperImplement::compute (EvaluatorWrapper.h:49-109) on GridGPU's
// list as it hands it over: neighborCounts (uint16), neighborlist, the
// per-block prefix cumulSumMaxPerBlock for nThreadPerBlock threads per block,
// nThreadPerAtom lanes per atom.  Forces (and, when virials is given,
// 0.5 F (x) dr per atom) are added, as the reference kernel adds them.
int pair_force_gridgpu(int n, const float4 *xs, float4 *fs, const uint16_t *counts, const uint32_t *nlist,
                       const uint32_t *cum, int ntpb, int ntpa, const float *params, int ntypes, const Box &box,
                       const float coef[3], int lj_kind, const float *qs, float qcut, float alpha, float qqr,
                       float *virials, cudaStream_t stream) {
    PairArgs A{};
    A.n = n;
    A.xs = xs;
    A.fs = fs;
    A.qs = qs;
    A.counts = nullptr;
    A.nlist = nlist;
    A.cap = 1 << 16;  // uint16 counts: never clipped
    A.params = params;
    A.ntypes = ntypes;
    A.box = box;
    A.coef1 = coef[0];
    A.coef2 = coef[1];
    A.coef3 = coef[2];
    A.dsf_A = A.dsf_shift = A.dsf_ecut = A.dsf_rc = 0.f;
    A.qrc2 = qcut > 0.f ? qcut * qcut : 0.f;
    A.alpha = alpha;
    A.qqr = qqr;
    A.virials = virials;
    A.energy = nullptr;
    A.lj_types = 0xffffffffu;
    A.cum = cum;
    A.counts16 = counts;
    A.ref_ntpb = ntpb;
    const bool ew = qcut > 0.f;
    if (lj_kind == 0 && !ew) return 0;
    A.np = 3;
    if (int r = launch_any(A, ntpa, lj_kind, ew ? 1 : 0, virials != nullptr, false, true, stream)) return r;
    MDX_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mdx
