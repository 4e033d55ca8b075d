// E3B three-body water term (FixE3B, src/Fixes/FixE3B.cu; kernels
// src/Evaluators/ThreeBodyE3B.h:18-549; maths src/Evaluators/EvaluatorE3B.h).
//
// The reference rebuilds a private molecule grid + neighbour list every step
// (FixE3B::handleLocalData, FixE3B.cu:349-406: 3 host syncs + 7 memsets),
// writes five per-pair scratch arrays in a two-body kernel and combines them
// with 18 float atomics per pair in a three-body kernel.  Here:
//  * the molecule list (O-O within rf + 1 A + skin) is cut from the atom list
//    whenever the atom list is rebuilt (same skin criterion, so it holds every
//    pair within the reference's 6.2 A list radius at every step);
//  * pass 1 (k_e3b_totals): each molecule sums its own e3bTotals over its FULL
//    list -- no atomics -- and adds the O-O two-body force;
//  * pass 2 (k_e3b_forces): each molecule re-evaluates the four switched
//    O-H exponentials of every pair within RMAX_E3B and keeps the forces that
//    land on its own three atoms, evaluating EvaluatorE3B::threeBodyPairForce
//    with the lower index as molecule "1" exactly as the reference's i<j
//    ordering; no scratch arrays, no atomics, deterministic.
#include <cstdio>

#include "engine.hpp"

namespace mdx {

namespace {

template <int T>
__device__ __forceinline__ float tsum(float v) {
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// switching(r), dswitchdr(r) (EvaluatorE3B.h:91-115)
__device__ __forceinline__ float e3b_sw(const E3BParams &p, float r) {
    if (r <= p.rs) return 1.0f;
    if (r > p.rf) return 0.0f;
    float v = (p.rf - r);
    v *= v;
    v *= ((p.rf + (2.0f * r) - p.rstimes3) * p.rfminusrs_cubed_inv);
    return v;
}
__device__ __forceinline__ float e3b_dsw(const E3BParams &p, float r) {
    if (r <= p.rs || r > p.rf) return 0.0f;
    return 6.0f * (p.rf - r) * (p.rs - r) * p.rfminusrs_cubed_inv;
}
// threeBodyPairEnergy(r) and threeBodyForce(dr, r) (EvaluatorE3B.h:117-141)
// (square root, exponential and divisions in the single-instruction forms
// the reference's --use_fast_math build gives them, CMakeLists.txt:53)
__device__ __forceinline__ void e3b_ef(const E3BParams &p, float3 dr, float &e, float3 &f) {
    const float r2 = dot3(dr, dr);
    const float rinv = rsqrt_ftz(r2);
    const float r = r2 * rinv;
    const float es = ex2_ftz(-p.k3 * r * 1.4426950408889634f);
    const float sw = e3b_sw(p, r);
    e = sw * es;
    f = make_float3(0.f, 0.f, 0.f);
    if (r <= p.rf) {
        float s = p.k3 * es * rinv;
        if (r > p.rs) {
            s *= sw;
            s -= es * e3b_dsw(p, r) * rinv;
        }
        f = dr * s;
    }
}

struct MolPos {
    float3 a, b, c;  // O, H1, H2
};

__device__ __forceinline__ MolPos load_mol(const float4 *__restrict__ xs, int4 ix) {
    MolPos m;
    m.a = f3(__ldg(xs + ix.x));
    m.b = f3(__ldg(xs + ix.y));
    m.c = f3(__ldg(xs + ix.z));
    return m;
}

// geometry of the pair with molecule 1 = m1 and 2 = m2 (ThreeBodyE3B.h:128-176)
struct PairGeom {
    float es[4];     // e_b2a1, e_c2a1, e_b1a2, e_c1a2
    float3 fv[4];    // forces_b2a1, c2a1, b1a2, c1a2
};
__device__ __forceinline__ void pair_geom(const E3BParams &p, const Box &box, const MolPos &m1, const MolPos &m2,
                                          PairGeom &g) {
    e3b_ef(p, min_image(box, m2.b - m1.a), g.es[0], g.fv[0]);
    e3b_ef(p, min_image(box, m2.c - m1.a), g.es[1], g.fv[1]);
    e3b_ef(p, min_image(box, m1.b - m2.a), g.es[2], g.fv[2]);
    e3b_ef(p, min_image(box, m1.c - m2.a), g.es[3], g.fv[3]);
}

// the same with whole molecules (the molecule form: a molecule's sites are
// made whole at every rebuild and move together): each O-H separation is an
// intramolecular vector plus the O-O image d12 = x(O1) - x(O2), no further
// minimum images.  h1b/h1c, h2b/h2c: the H - O vectors of molecules 1 and 2
__device__ __forceinline__ void pair_geom_whole(const E3BParams &p, float3 d12, float3 h1b, float3 h1c, float3 h2b,
                                                float3 h2c, PairGeom &g) {
    e3b_ef(p, h2b - d12, g.es[0], g.fv[0]);
    e3b_ef(p, h2c - d12, g.es[1], g.fv[1]);
    e3b_ef(p, h1b + d12, g.es[2], g.fv[2]);
    e3b_ef(p, h1c + d12, g.es[3], g.fv[3]);
}

// EvaluatorE3B::threeBodyPairForce (EvaluatorE3B.h:145-249): the forces on
// both molecules' atoms of one unordered pair (molecule 1 = lower index)
__device__ __forceinline__ void pair_force_both(const E3BParams &p, const PairGeom &g, float4 T1, float4 T2,
                                                float3 &a1, float3 &b1, float3 &c1, float3 &a2, float3 &b2,
                                                float3 &c2) {
    const float *e = g.es;
    a1 = make_float3(0.f, 0.f, 0.f);
    b1 = a1; c1 = a1; a2 = a1; b2 = a1; c2 = a1;
    float3 fj;
    float sc;
    sc = p.Ea * (T2.y - e[0]);
    fj = sc * g.fv[1]; a1 -= fj; c2 += fj;
    sc = p.Ea * (T1.y - e[2]);
    fj = sc * g.fv[3]; a2 -= fj; c1 += fj;
    sc = p.Ea * (T2.z - e[1]);
    fj = sc * g.fv[0]; a1 -= fj; b2 += fj;
    sc = p.Ea * (T1.z - e[3]);
    fj = sc * g.fv[2]; a2 -= fj; b1 += fj;
    sc = p.Eb * (T2.x + T1.y + T1.z - 2.0f * (e[2] + e[3]));
    fj = sc * g.fv[0]; a1 -= fj; b2 += fj;
    fj = sc * g.fv[1]; a1 -= fj; c2 += fj;
    sc = p.Eb * (T1.x + T2.y + T2.z - 2.0f * (e[0] + e[1]));
    fj = sc * g.fv[2]; a2 -= fj; b1 += fj;
    fj = sc * g.fv[3]; a2 -= fj; c1 += fj;
    sc = p.Ec * (T1.x - e[1] - e[0]);
    fj = sc * g.fv[0]; a1 -= fj; b2 += fj;
    fj = sc * g.fv[1]; a1 -= fj; c2 += fj;
    sc = p.Ec * (T2.x - e[2] - e[3]);
    fj = sc * g.fv[2]; a2 -= fj; b1 += fj;
    fj = sc * g.fv[3]; a2 -= fj; c1 += fj;
}

// VEC: one 16-byte atomic (side buffers, whose .w is unused); otherwise three
// scalar atomics so that .w (the force stream's group-tag bits) is untouched
template <bool VEC>
__device__ __forceinline__ void add_force(float4 *f, float3 v) {
    if (VEC) {
        atomicAdd(f, make_float4(v.x, v.y, v.z, 0.f));
    } else {
        atomicAdd(&f->x, v.x);
        atomicAdd(&f->y, v.y);
        atomicAdd(&f->z, v.z);
    }
}

// total three-body energy of one unordered pair (EvaluatorE3B.h:251-345)
__device__ __forceinline__ float pair_energy(const E3BParams &p, const float *e, float4 T1, float4 T2) {
    float s = 0.f, sc;
    sc = p.Ea * (T2.y - e[0]); s += 0.5f * sc * e[1];
    sc = p.Ea * (T1.y - e[2]); s += 0.5f * sc * e[3];
    sc = p.Ea * (T2.z - e[1]); s += 0.5f * sc * e[0];
    sc = p.Ea * (T1.z - e[3]); s += 0.5f * sc * e[2];
    sc = p.Eb * (T2.x + T1.y + T1.z - 2.0f * (e[2] + e[3])); s += 0.5f * sc * (e[0] + e[1]);
    sc = p.Eb * (T1.x + T2.y + T2.z - 2.0f * (e[0] + e[1])); s += 0.5f * sc * (e[2] + e[3]);
    sc = p.Ec * (T1.x - e[1] - e[0]); s += 0.5f * sc * (e[0] + e[1]);
    sc = p.Ec * (T2.x - e[2] - e[3]); s += 0.5f * sc * (e[2] + e[3]);
    return s;
}

// Arguments of the E3B kernels for one system: a0 (single system) or
// tab[blockIdx.y] (batched replicas; a0 then only sizes the grid).
struct E3BArgs {
    int nmol;
    const int4 *mol_ids;
    int4 *mol_idx;
    const int *idToIdx, *mol_of_id;
    const uint32_t *ids;
    const float4 *xs;
    const uint32_t *counts, *counts_int, *nlist;
    int team_atom, cap_atom;
    Box box;
    float cut2;
    uint32_t *mcounts, *mlist;
    int mcap;
    DeviceStatus *st;
    float4 *out;      // forces (added) or the per-step side buffer (STORE)
    E3BParams p;
    float4 *totals;
    double *e_out;    // energy passes
    int twobody;      // 0: the totals pass leaves out the O-O two-body force
    // the forces pass's own list, written by the totals pass each step: the
    // partners mj > m within rmax (each unordered pair once), in mlist's
    // team layout with mcap entries per molecule (null: walk the full list)
    uint32_t *ccounts, *clist;
    // 1: the molecule form -- molecule index = slot, sites at 4m .. 4m+3
    // (mol_idx holds that identity map; the hot passes skip reading it)
    int slots;
    // the molecule form's list source: the molecule-pair list of the same
    // rebuild (counts, entries in its team layout) and the sorted positions
    const uint32_t *mf_counts, *mf_list;
    int mf_cap, mf_team;
    const float4 *mf_xs2;
};

__device__ __forceinline__ int4 e3b_sites(const E3BArgs &A, const int4 *__restrict__ mol_idx, int m) {
    return A.slots ? make_int4(4 * m, 4 * m + 1, 4 * m + 2, 4 * m + 3) : __ldg(mol_idx + m);
}
#define MDX_E3B_ARGS \
    pdl_wait();      \
    const E3BArgs A = tab ? tab[blockIdx.y] : a0

// updateMoleculeIdxsMap (FixE3B.cu:41-65) + molecule list cut from the atom
// list: O-O pairs with r^2 < (rf + 1 + skin)^2.  Team of T lanes per molecule.
template <int T>
__global__ void k_e3b_list(const E3BArgs a0, const E3BArgs *__restrict__ tab, int conditional) {
    MDX_E3B_ARGS;
    if (A.slots) return;  // a molecule-form replica: its list comes from k_e3b_list_mf
    DeviceStatus *st = A.st;
    const int nmol = A.nmol;
    const int4 *__restrict__ mol_ids = A.mol_ids;
    int4 *__restrict__ mol_idx = A.mol_idx;
    const int *__restrict__ idToIdx = A.idToIdx;
    const int *__restrict__ mol_of_id = A.mol_of_id;
    const uint32_t *__restrict__ ids = A.ids;
    const float4 *__restrict__ xs = A.xs;
    const uint32_t *__restrict__ counts = A.counts;
    const uint32_t *__restrict__ counts_int = A.counts_int;
    const uint32_t *__restrict__ nlist = A.nlist;
    const int team_atom = A.team_atom, cap_atom = A.cap_atom;
    const Box &box = A.box;
    const float cut2 = A.cut2;
    uint32_t *__restrict__ mcounts = A.mcounts;
    uint32_t *__restrict__ mlist = A.mlist;
    const int mcap = A.mcap;
    if (conditional && !st->rebuild) return;
    constexpr int G = 32 / T;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / T, t = lane % T;
    const int m = warp * G + a;
    if (m >= nmol) return;
    const unsigned team_mask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << (a * T));
    const int4 id4 = mol_ids[m];
    const int4 ix = make_int4(idToIdx[id4.x], idToIdx[id4.y], idToIdx[id4.z], id4.w >= 0 ? idToIdx[id4.w] : -1);
    if (t == 0) mol_idx[m] = ix;
    const int oi = ix.x;
    const float3 po = f3(xs[oi]);
    int cnt = (int)counts[oi];
    cnt = cnt < cap_atom ? cnt : cap_atom;
    // rows hold interacting pairs from the front and the rest from the back
    const int cfront = counts_int ? (int)counts_int[oi] : cnt;
    const int Ga = 32 / team_atom;
    const uint32_t *row = nlist + (size_t)(oi / Ga) * cap_atom * Ga + (oi % Ga) * team_atom;
    uint32_t *mrow = mlist + (size_t)(m / G) * mcap * G + a * T;
    int mc = 0;
    for (int k0 = 0; k0 < cnt; k0 += T) {
        const int k = k0 + t;
        bool hit = false;
        int mj = -1;
        if (k < cnt) {
            const int kk = k < cfront ? k : cap_atom - 1 - (k - cfront);
            const uint32_t e = row[(size_t)(kk / team_atom) * 32 + (kk % team_atom)];
            const int j = (int)(e & kExclMask);
            mj = mol_of_id[ids[j]];
            if (mj >= 0 && mj != m) {
                const float3 d = min_image(box, po - f3(xs[j]));
                hit = dot3(d, d) < cut2;
            }
        }
        const unsigned b = __ballot_sync(team_mask, hit);
        if (hit) {
            const unsigned mine = (T == 32) ? b : (b >> (a * T));
            const int pos = mc + __popc(mine & ((1u << t) - 1u));
            if (pos < mcap) mrow[(size_t)(pos / T) * 32 + (pos % T)] = (uint32_t)mj;
        }
        mc += __popc(b);
    }
    if (t == 0) {
        mcounts[m] = (uint32_t)mc;
        if (mc > mcap) atomicOr(&st->bits, kStatusMolOverflow);
        atomicMax(&st->max_mol_neighbors, (uint32_t)mc);
    }
}

// The molecule form's E3B list, cut from the molecule-pair list of the same
// rebuild: in that form the E3B molecule index is the slot (sites 4k ..
// 4k+3), so row k holds every listed slot whose site-0 distance is below the
// E3B list radius.  The molecule-pair list holds every site-0 pair within its
// larger radius, so the E3B set is the per-site path's.
template <int T>
__global__ void k_e3b_list_mf(const E3BArgs a0, const E3BArgs *__restrict__ tab) {
    MDX_E3B_ARGS;
    if (!A.slots || !A.st->rebuild) return;
    const uint32_t *__restrict__ pcounts = A.mf_counts;
    const uint32_t *__restrict__ plist = A.mf_list;
    const int pcap = A.mf_cap, pteam = A.mf_team;
    const float4 *__restrict__ xs2 = A.mf_xs2;
    constexpr int G = 32 / T;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / T, t = lane % T;
    const int m = warp * G + a;
    if (m >= A.nmol) return;
    const unsigned team_mask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << (a * T));
    const int k = m;
    const float3 po = f3(xs2[4 * k]);
    int cnt = (int)pcounts[k];
    cnt = cnt < pcap ? cnt : pcap;
    const int PG = 32 / pteam;
    const uint32_t *prow = plist + (size_t)(k / PG) * pcap * PG + (k % PG) * pteam;
    uint32_t *mrow = A.mlist + (size_t)(m / G) * A.mcap * G + a * T;
    int mc = 0;
    for (int k0 = 0; k0 < cnt; k0 += T) {
        const int e = k0 + t;
        bool hit = false;
        int mj = -1;
        if (e < cnt) {
            const int j = (int)prow[(size_t)(e / pteam) * 32 + (e % pteam)];
            const float3 d = min_image(A.box, po - f3(xs2[4 * j]));
            hit = dot3(d, d) < A.cut2;
            mj = j;
        }
        const unsigned b = __ballot_sync(team_mask, hit);
        if (hit) {
            const unsigned mine = (T == 32) ? b : (b >> (a * T));
            const int pos = mc + __popc(mine & ((1u << t) - 1u));
            if (pos < A.mcap) mrow[(size_t)(pos / T) * 32 + (pos % T)] = (uint32_t)mj;
        }
        mc += __popc(b);
    }
    if (t == 0) {
        A.mcounts[m] = (uint32_t)mc;
        if (mc > A.mcap) atomicOr(&A.st->bits, kStatusMolOverflow);
        atomicMax(&A.st->max_mol_neighbors, (uint32_t)mc);
    }
}

// pass 1: e3bTotals of molecule i (ThreeBodyE3B.h:170-211 summed from i's own
// full list) and the O-O two-body force (EvaluatorE3B::twoBodyForce, :67-78)
// STORE: write into a per-step side buffer instead of adding to the forces
// (lets E3B run concurrently with the pair kernel; the second half merges it)
// list entries per lane per trip of the totals pass: all of them in flight
// (list -> sites) before the first is evaluated
#ifndef MDX_E3B_TOT_U
#define MDX_E3B_TOT_U 2
#endif
constexpr int kTotU = MDX_E3B_TOT_U;

template <int T, bool ENERGY, bool STORE = false>
__global__ void k_e3b_totals(const E3BArgs a0, const E3BArgs *__restrict__ tab) {
    MDX_E3B_ARGS;
    const int nmol = A.nmol;
    const int4 *__restrict__ mol_idx = A.mol_idx;
    const float4 *__restrict__ xs = A.xs;
    float4 *__restrict__ fs = A.out;
    const uint32_t *__restrict__ mcounts = A.mcounts;
    const uint32_t *__restrict__ mlist = A.mlist;
    const int mcap = A.mcap;
    const Box &box = A.box;
    const E3BParams &p = A.p;
    float4 *__restrict__ totals = A.totals;
    double *__restrict__ e2_out = A.e_out;
    constexpr int G = 32 / T;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / T, t = lane % T;
    const int m = warp * G + a;
    const bool valid = m < nmol;
    float fx = 0.f, fy = 0.f, fz = 0.f, tx = 0.f, ty = 0.f, tz = 0.f, e2 = 0.f;
    int4 ix = make_int4(0, 0, 0, 0);
    uint32_t *const clist = A.clist;
    // the team's lanes (the teams of a warp walk rows of different lengths)
    const unsigned team_mask = (T == 32 ? 0xffffffffu : ((1u << T) - 1u)) << (a * T);
    int nc = 0;  // the forces pass's partners found (team-uniform)
    if (valid) {
        ix = e3b_sites(A, mol_idx, m);
        const MolPos mi = load_mol(xs, ix);
        const float3 hb = mi.b - mi.a, hc = mi.c - mi.a;  // whole molecules (A.slots)
        int cnt = (int)mcounts[m];
        cnt = cnt < mcap ? cnt : mcap;
        const uint32_t *row = mlist + (size_t)(m / G) * mcap * G + a * T + t;
        uint32_t *crow = clist ? clist + (size_t)(m / G) * mcap * G + a * T : nullptr;
        // two entries per lane per trip: both list -> molecule -> O chains are
        // in flight before either pair is evaluated.  Every lane of the team
        // makes the same trips (the partner ballot below takes the team)
        for (int k00 = 0; k00 < cnt; k00 += kTotU * T) {
            const int k0 = k00 + t;
            int4 jxs[kTotU];
            MolPos mps[kTotU];
            bool has[kTotU];
            int mjs[kTotU];
#pragma unroll
            for (int u = 0; u < kTotU; u++) {
                const int k = k0 + u * T;
                has[u] = k < cnt;
                mjs[u] = has[u] ? (int)row[(size_t)(k / T) * 32] : m;
                jxs[u] = e3b_sites(A, mol_idx, mjs[u]);
            }
            // the partner's three sites in one round of loads (L2-resident;
            // the hydrogens are used only within rmax)
#pragma unroll
            for (int u = 0; u < kTotU; u++) mps[u] = load_mol(xs, jxs[u]);
#pragma unroll
            for (int u = 0; u < kTotU; u++) {
            const float3 oj = mps[u].a;
            const float3 dr = min_image(box, mi.a - oj);
            const float r2 = dot3(dr, dr);
            if (!ENERGY && clist) {
                // the forces pass's partners: the same tests it makes
                const int mj = mjs[u];
                const bool keep = has[u] && r2 < p.list_cut2 && !(r2 > p.rmax * p.rmax) && m < mj;
                const unsigned tm = __ballot_sync(team_mask, keep) >> (a * T);
                if (keep) {
                    const int pos = nc + __popc(tm & ((1u << t) - 1u));
                    crow[(size_t)(pos / T) * 32 + pos % T] = (uint32_t)mj;
                }
                nc += __popc(tm);
            }
            if (!has[u]) continue;
            if (r2 >= p.list_cut2) continue;
            const float rinv = rsqrt_ftz(r2);
            const float r = r2 * rinv;
            const float ex = ex2_ftz(-p.k2 * r * 1.4426950408889634f);
            const float s = p.k2 * p.E2 * ex * rinv;
            fx += dr.x * s;
            fy += dr.y * s;
            fz += dr.z * s;
            if (ENERGY) e2 += 0.5f * p.E2 * ex;
            if (r <= p.rmax) {
                const MolPos &mj_ = mps[u];
                PairGeom g;
                if (A.slots) pair_geom_whole(p, dr, hb, hc, mj_.b - oj, mj_.c - oj, g);
                else pair_geom(p, box, mi, mj_, g);
                tx += g.es[0] + g.es[1];
                ty += g.es[2];
                tz += g.es[3];
            }
            }
        }
    }
    if (ENERGY) {
        e2 = tsum<T>(e2);
        if (valid && t == 0) atomicAdd(e2_out, (double)e2);
        return;
    }
    fx = tsum<T>(fx);
    fy = tsum<T>(fy);
    fz = tsum<T>(fz);
    tx = tsum<T>(tx);
    ty = tsum<T>(ty);
    tz = tsum<T>(tz);
    if (!A.twobody) fx = fy = fz = 0.f;
    if (valid && t == 0) {
        if (clist) A.ccounts[m] = (uint32_t)nc;
        totals[m] = make_float4(tx, ty, tz, 0.f);
        if (STORE) {
            // the forces pass adds into these with atomics
            fs[ix.x] = make_float4(fx, fy, fz, 0.f);
            fs[ix.y] = make_float4(0.f, 0.f, 0.f, 0.f);
            fs[ix.z] = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            float4 f = fs[ix.x];
            f.x += fx;
            f.y += fy;
            f.z += fz;
            fs[ix.x] = f;
        }
    }
}

// pass 2: three-body forces on molecule i's O, H1, H2 (ThreeBodyE3B.h:255-549)
template <int T, bool ENERGY, bool STORE = false>
__global__ void k_e3b_forces(const E3BArgs a0, const E3BArgs *__restrict__ tab) {
    MDX_E3B_ARGS;
    const int nmol = A.nmol;
    const int4 *__restrict__ mol_idx = A.mol_idx;
    const float4 *__restrict__ xs = A.xs;
    float4 *__restrict__ fs = A.out;
    const uint32_t *__restrict__ mcounts = A.mcounts;
    const uint32_t *__restrict__ mlist = A.mlist;
    const int mcap = A.mcap;
    const Box &box = A.box;
    const E3BParams &p = A.p;
    const float4 *__restrict__ totals = A.totals;
    double *__restrict__ e3_out = A.e_out;
    constexpr int G = 32 / T;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / T, t = lane % T;
    const int m = warp * G + a;
    const bool valid = m < nmol;
    float3 fa = make_float3(0.f, 0.f, 0.f), fb = fa, fc = fa;
    float e3 = 0.f;
    int4 ix = make_int4(0, 0, 0, 0);
    if (valid) {
        ix = e3b_sites(A, mol_idx, m);
        const MolPos mi = load_mol(xs, ix);
        const float4 Ti = totals[m];
        // forces: the partners the totals pass kept (mj > m within rmax);
        // the energy walks the full list (both orders, half each)
        const bool compact = !ENERGY && A.clist;
        int cnt = compact ? (int)A.ccounts[m] : (int)mcounts[m];
        cnt = cnt < mcap ? cnt : mcap;
        const uint32_t *row = (compact ? A.clist : mlist) + (size_t)(m / G) * mcap * G + a * T + t;
        // two entries per lane per trip, as the totals pass
        for (int k0 = t; k0 < cnt; k0 += 2 * T) {
            int mjs[2];
            int4 jxs[2];
            MolPos mps[2];
            float4 Tjs[2];
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int k = k0 + u * T;
                mjs[u] = k < cnt ? (int)row[(size_t)(k / T) * 32] : -1;
                jxs[u] = e3b_sites(A, mol_idx, mjs[u] < 0 ? m : mjs[u]);
            }
            // sites and totals of both partners in one round of loads
#pragma unroll
            for (int u = 0; u < 2; u++) {
                mps[u] = load_mol(xs, jxs[u]);
                Tjs[u] = __ldg(totals + (mjs[u] < 0 ? m : mjs[u]));
            }
#pragma unroll
            for (int u = 0; u < 2; u++) {
            if (mjs[u] < 0) continue;
            const int mj = mjs[u];
            const int4 jx = jxs[u];
            const MolPos &mjp = mps[u];
            const float3 dr = min_image(box, mi.a - mjp.a);
            const float r2 = dot3(dr, dr);
            if (r2 >= p.list_cut2) continue;
            if (r2 > p.rmax * p.rmax) continue;
            const float4 Tj = Tjs[u];
            const bool first = m < mj;
            PairGeom g;
            if (ENERGY) {
                if (first) pair_geom(p, box, mi, mjp, g);
                else pair_geom(p, box, mjp, mi, g);
                e3 += 0.5f * (first ? pair_energy(p, g.es, Ti, Tj) : pair_energy(p, g.es, Tj, Ti));
                continue;
            }
            // forces: each unordered pair once, from its lower-index molecule
            // (molecule 1, as the reference's i < j); the partner's share is
            // scattered with vector atomics
            if (!first) continue;
            if (A.slots) pair_geom_whole(p, dr, mi.b - mi.a, mi.c - mi.a, mjp.b - mjp.a, mjp.c - mjp.a, g);
            else pair_geom(p, box, mi, mjp, g);
            float3 a1, b1, c1, a2, b2, c2;
            pair_force_both(p, g, Ti, Tj, a1, b1, c1, a2, b2, c2);
            fa += a1;
            fb += b1;
            fc += c1;
            add_force<STORE>(fs + jx.x, a2);
            add_force<STORE>(fs + jx.y, b2);
            add_force<STORE>(fs + jx.z, c2);
            }
        }
    }
    if (ENERGY) {
        e3 = tsum<T>(e3);
        if (valid && t == 0) atomicAdd(e3_out, (double)e3);
        return;
    }
    fa.x = tsum<T>(fa.x); fa.y = tsum<T>(fa.y); fa.z = tsum<T>(fa.z);
    fb.x = tsum<T>(fb.x); fb.y = tsum<T>(fb.y); fb.z = tsum<T>(fb.z);
    fc.x = tsum<T>(fc.x); fc.y = tsum<T>(fc.y); fc.z = tsum<T>(fc.z);
    if (valid && t == 0) {
        add_force<STORE>(fs + ix.x, fa);
        add_force<STORE>(fs + ix.y, fb);
        add_force<STORE>(fs + ix.z, fc);
    }
}

// E3B virial (virialMode): per molecule i, the two-body term as the
// reference, 0.5 F (x) dr per listed O-O pair (computeVirial,
// ThreeBodyE3B.h:129, 222-245), plus -- which the reference leaves out
// (ThreeBodyE3B.h:449-451) -- the three-body forces of each unordered pair,
// counted once on its lower-index molecule: every term of pair_force_both is
// a central O-H force sc fv[k] along d[k] (H minus O), so the pair adds
// sum_k S_k fv[k] (x) d[k], S_k the sum of the coefficients of fv[k].  Added
// to the O atom's per-atom virial (xx yy zz xy xz yz).
template <int T>
__global__ void k_e3b_virial(const E3BArgs A, float *__restrict__ vir) {
    const int4 *__restrict__ mol_idx = A.mol_idx;
    const float4 *__restrict__ xs = A.xs;
    const Box &box = A.box;
    const E3BParams &p = A.p;
    constexpr int G = 32 / T;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / T, t = lane % T;
    const int m = warp * G + a;
    const bool valid = m < A.nmol;
    float w[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    auto add = [&](float s, float3 f, float3 d) {
        w[0] += s * f.x * d.x;
        w[1] += s * f.y * d.y;
        w[2] += s * f.z * d.z;
        w[3] += s * f.x * d.y;
        w[4] += s * f.x * d.z;
        w[5] += s * f.y * d.z;
    };
    int4 ix = make_int4(0, 0, 0, 0);
    if (valid) {
        ix = mol_idx[m];
        const MolPos mi = load_mol(xs, ix);
        const float4 Ti = A.totals[m];
        int cnt = (int)A.mcounts[m];
        cnt = cnt < A.mcap ? cnt : A.mcap;
        const uint32_t *row = A.mlist + (size_t)(m / G) * A.mcap * G + a * T + t;
        for (int k = t; k < cnt; k += T) {
            const int mj = (int)row[(size_t)(k / T) * 32];
            const int4 jx = __ldg(mol_idx + mj);
            MolPos mjp;
            mjp.a = f3(__ldg(xs + jx.x));
            const float3 dr = min_image(box, mi.a - mjp.a);
            const float r2 = dot3(dr, dr);
            if (r2 >= p.list_cut2) continue;
            const float r = sqrtf(r2);
            add(0.5f * p.k2 * p.E2 * expf(-p.k2 * r) / r, dr, dr);
            if (r > p.rmax || m >= mj) continue;
            mjp.b = f3(__ldg(xs + jx.y));
            mjp.c = f3(__ldg(xs + jx.z));
            const float4 Tj = __ldg(A.totals + mj);
            PairGeom g;
            pair_geom(p, box, mi, mjp, g);
            const float3 d[4] = {min_image(box, mjp.b - mi.a), min_image(box, mjp.c - mi.a),
                                 min_image(box, mi.b - mjp.a), min_image(box, mi.c - mjp.a)};
            const float *e = g.es;
            const float B1 = p.Eb * (Tj.x + Ti.y + Ti.z - 2.0f * (e[2] + e[3]));
            const float B2 = p.Eb * (Ti.x + Tj.y + Tj.z - 2.0f * (e[0] + e[1]));
            const float C1 = p.Ec * (Ti.x - e[1] - e[0]);
            const float C2 = p.Ec * (Tj.x - e[2] - e[3]);
            add(p.Ea * (Tj.z - e[1]) + B1 + C1, g.fv[0], d[0]);
            add(p.Ea * (Tj.y - e[0]) + B1 + C1, g.fv[1], d[1]);
            add(p.Ea * (Ti.z - e[3]) + B2 + C2, g.fv[2], d[2]);
            add(p.Ea * (Ti.y - e[2]) + B2 + C2, g.fv[3], d[3]);
        }
    }
#pragma unroll
    for (int c = 0; c < 6; c++) w[c] = tsum<T>(w[c]);
    if (valid && t == 0) {
#pragma unroll
        for (int c = 0; c < 6; c++) vir[6 * (size_t)ix.x + c] += w[c];
    }
}

constexpr int kMolTeam = kE3BTeam;

}  // namespace

FixE3B::FixE3B(State *s, std::string h, std::string st) : Fix(s, h, "all", "E3B", FixKind::E3B), style(st) {}

int FixE3B::prepareForRun() {
    State &s = *state;
    if (style != "E3B3" && style != "E3B2") {
        set_error(MDX_ERR_ARG, "FixE3B style must be 'E3B3' or 'E3B2'");
        return MDX_ERR_ARG;
    }
    if (s.units.type != MDX_UNITS_REAL) {
        set_error(MDX_ERR_UNSUPPORTED, "Units for E3B potential are not yet as LJ (FixE3B.cu:541)");
        return MDX_ERR_UNSUPPORTED;
    }
    const double kj = 0.23900573614;
    double E2, Ea, Eb, Ec;
    if (style == "E3B3") { E2 = 453000.0; Ea = 150.0; Eb = -1005.0; Ec = 1880.0; }
    else { E2 = 2349000.0; Ea = 1745.7; Eb = -4565.0; Ec = 7606.8; }
    // EvaluatorE3B ctor (EvaluatorE3B.h:46-64): float parameters
    prm.rs = 5.0f;
    prm.rf = 5.2f;
    prm.E2 = (float)(E2 * kj);
    prm.Ea = (float)(Ea * kj);
    prm.Eb = (float)(Eb * kj);
    prm.Ec = (float)(Ec * kj);
    prm.k2 = 4.872f;
    prm.k3 = 1.907f;
    float d = prm.rf - prm.rs;
    prm.rfminusrs_cubed_inv = 1.0f / (d * d * d);
    prm.rstimes3 = 3.0f * prm.rs;
    float lc = (float)((double)prm.rf + 1.0);  // molecule-list radius rf + padding(1.0) (FixE3B.cu:29, 657)
    prm.list_cut2 = lc * lc;
    prm.rmax = 6.157200f;
    if ((double)s.grid.cut < (double)lc + s.padding) {
        set_error(MDX_ERR_UNSUPPORTED,
                  "FixE3B needs the atom neighbour cutoff (rCut + padding = %g) >= %g (E3B list radius + padding)",
                  (double)s.grid.cut, (double)lc + s.padding);
        return MDX_ERR_UNSUPPORTED;
    }
    const int nmol = (int)mol_ids.size();
    if (int e = d_mol_ids.alloc(nmol)) return e;
    if (int e = d_mol_idx.alloc(nmol)) return e;
    if (int e = totals.alloc(nmol)) return e;
    if (int e = mcounts.alloc(nmol)) return e;
    MDX_CUDA_TRY(cudaMemcpy(d_mol_ids.p, mol_ids.data(), nmol * sizeof(int4), cudaMemcpyHostToDevice));
    std::vector<int> mof(s.atoms.size(), -1);
    for (int m = 0; m < nmol; m++) mof[mol_ids[m].x] = m;
    if (int e = d_mol_of_atom.alloc(mof.size())) return e;
    MDX_CUDA_TRY(cudaMemcpy(d_mol_of_atom.p, mof.data(), mof.size() * sizeof(int), cudaMemcpyHostToDevice));
    // the fused step can run E3B beside the pair kernel when its molecules
    // are FixRigid's, in the same order (the second half merges the forces)
    side_ok = false;
    if (FixRigid *r = s.rigidFix()) {
        if (r->mol_ids.size() == mol_ids.size()) {
            side_ok = true;
            for (size_t k = 0; k < mol_ids.size(); k++) {
                const int4 a = mol_ids[k], b = r->mol_ids[k];
                if (a.x != b.x || a.y != b.y || a.z != b.z) side_ok = false;
            }
        }
    }
    if (side_ok)
        if (int e = f_side.alloc(s.atoms.size())) return e;
    mteam = kMolTeam;
    const double vol = s.box.Ld.x * s.box.Ld.y * s.box.Ld.z;
    const double rl = (double)lc + s.padding;
    const double est = nmol / vol * 4.18879 * rl * rl * rl;
    mcap = ((int)(2.0 * est + 32) + mteam - 1) / mteam * mteam;
    const size_t groups = (size_t)(nmol + 32 / mteam - 1) / (32 / mteam);
    if (int e = mlist.alloc(groups * mcap * (32 / mteam))) return e;
    // the forces pass's list: a subset of each full row, so the same capacity
    if (int e = ccounts.alloc(nmol)) return e;
    if (int e = clist.alloc(groups * mcap * (32 / mteam))) return e;
    prepared = true;
    return 0;
}

static E3BArgs e3b_args(State &s, FixE3B &f, float4 *out) {
    E3BArgs A{};
    const float lc = (float)((double)f.prm.rf + 1.0 + s.padding);
    A.nmol = (int)f.mol_ids.size();
    A.mol_ids = f.d_mol_ids.p;
    A.mol_idx = f.d_mol_idx.p;
    A.idToIdx = s.gpd.idToIdx.p;
    A.mol_of_id = f.d_mol_of_atom.p;
    A.ids = s.gpd.ids.p;
    A.xs = s.gpd.xs.p;
    A.counts = s.grid.counts.p;
    A.counts_int = s.grid.partition ? s.grid.counts_int.p : nullptr;
    A.nlist = s.grid.nlist.p;
    A.team_atom = s.grid.team;
    A.cap_atom = s.grid.cap;
    A.box = s.box;
    A.cut2 = lc * lc;
    A.mcounts = f.mcounts.p;
    A.mlist = f.mlist.p;
    A.mcap = f.mcap;
    A.st = s.d_status.p;
    A.out = out;
    A.p = f.prm;
    A.totals = f.totals.p;
    A.e_out = nullptr;
    A.twobody = 1;
    A.ccounts = f.ccounts.p;
    A.clist = f.clist.p;
    A.slots = s.mf.on ? 1 : 0;
    if (s.mf.on) {
        A.mf_counts = s.mf.counts.p;
        A.mf_list = s.mf.list.p;
        A.mf_cap = s.mf.cap;
        A.mf_team = s.mf.team;
        A.mf_xs2 = s.gpd.xs_alt.p;
    }
    return A;
}

static dim3 e3b_blocks(int nmol, unsigned nrep = 1) {
    const int warps = (nmol + (32 / kMolTeam) - 1) / (32 / kMolTeam);
    return dim3((warps * 32 + 255) / 256, nrep);
}

// part of a list rebuild, after the sort: the O-O distances are taken on the
// sorted copy of the positions of this list build (xs_alt), which the step's first half
// running beside it on another stream does not move
int e3b_build_list(State &s, FixE3B &f, bool conditional, cudaStream_t st) {
    const int nmol = (int)f.mol_ids.size();
    if (nmol == 0 || !f.prepared) return 0;
    E3BArgs A = e3b_args(s, f, nullptr);
    A.xs = s.gpd.xs_alt.p;
    MDX_CUDA_TRY(launch_pdl(k_e3b_list<kMolTeam>, e3b_blocks(nmol), dim3(256), 0, st ? st : s.stream, A,
                            (const E3BArgs *)nullptr, conditional ? 1 : 0));
    return 0;
}

// the molecule form: after the sort by molecule, from the molecule-pair list
int e3b_build_list_mf(State &s, FixE3B &f, cudaStream_t st) {
    const int nmol = (int)f.mol_ids.size();
    if (nmol == 0 || !f.prepared) return 0;
    const E3BArgs A = e3b_args(s, f, nullptr);
    MDX_CUDA_TRY(launch_pdl(k_e3b_list_mf<kMolTeam>, e3b_blocks(nmol), dim3(256), 0, st ? st : s.stream, A,
                            (const E3BArgs *)nullptr));
    return 0;
}

int e3b_forces(State &s, FixE3B &f) { return e3b_forces_to(s, f, s.gpd.fs.p, false, s.stream); }

// side = true: store into `out` (a per-step E3B force buffer of O/H1/H2),
// otherwise add to `out` (the atom forces)
int e3b_forces_to(State &s, FixE3B &f, float4 *out, bool side, cudaStream_t stream) {
    const int nmol = (int)f.mol_ids.size();
    if (nmol == 0) return 0;
    const E3BArgs A = e3b_args(s, f, out);
    const dim3 blocks = e3b_blocks(nmol);
    const E3BArgs *nt = nullptr;
    if (side) {
        // the fused step's pair: 64-thread blocks beside the pair kernel and
        // the P3M chain (measured +0.6 % per water + E3B step against 256)
        const dim3 b64 = dim3(blocks.x * 4);
        MDX_CUDA_TRY(launch_pdl(k_e3b_totals<kMolTeam, false, true>, b64, dim3(64), 0, stream, A, nt));
        MDX_CUDA_TRY(launch_pdl(k_e3b_forces<kMolTeam, false, true>, b64, dim3(64), 0, stream, A, nt));
        return 0;
    }
    k_e3b_totals<kMolTeam, false><<<blocks, 256, 0, stream>>>(A, nullptr);
    MDX_LAUNCHED();
    k_e3b_forces<kMolTeam, false><<<blocks, 256, 0, stream>>>(A, nullptr);
    MDX_LAUNCHED();
    return 0;
}

// exact E3B forces stored into out[O], out[H1], out[H2]; twobody = 0 leaves
// out the O-O two-body term (the three-body forces alone: the surrogate's
// training target and the measure of its error)
int e3b_exact_to(State &s, FixE3B &f, float4 *out, int twobody, cudaStream_t stream) {
    const int nmol = (int)f.mol_ids.size();
    if (nmol == 0) return 0;
    E3BArgs A = e3b_args(s, f, out);
    A.twobody = twobody;
    const dim3 blocks = e3b_blocks(nmol);
    k_e3b_totals<kMolTeam, false, true><<<blocks, 256, 0, stream>>>(A, nullptr);
    MDX_LAUNCHED();
    k_e3b_forces<kMolTeam, false, true><<<blocks, 256, 0, stream>>>(A, nullptr);
    MDX_LAUNCHED();
    return 0;
}

// the O-O two-body force alone, stored into out[O] (the exact part of the
// surrogate step)
int e3b_twobody_to(State &s, FixE3B &f, float4 *out, cudaStream_t stream) {
    const int nmol = (int)f.mol_ids.size();
    if (nmol == 0) return 0;
    E3BArgs A = e3b_args(s, f, out);
    k_e3b_totals<kMolTeam, false, true><<<e3b_blocks(nmol), 256, 0, stream>>>(A, nullptr);
    MDX_LAUNCHED();
    return 0;
}

int e3b_energy(State &s, FixE3B &f, double out[2]) {
    const int nmol = (int)f.mol_ids.size();
    out[0] = out[1] = 0.0;
    if (nmol == 0) return 0;
    DBuf<double> acc;
    if (int e = acc.alloc(2)) return e;
    MDX_CUDA_TRY(cudaMemsetAsync(acc.p, 0, 2 * sizeof(double), s.stream));
    const dim3 blocks = e3b_blocks(nmol);
    // totals are needed by the energy pass: run the force-less totals first
    DBuf<float4> ftmp;
    if (int e = ftmp.alloc(s.gpd.n)) return e;
    MDX_CUDA_TRY(cudaMemcpyAsync(ftmp.p, s.gpd.fs.p, s.gpd.n * sizeof(float4), cudaMemcpyDeviceToDevice, s.stream));
    E3BArgs A = e3b_args(s, f, ftmp.p);
    k_e3b_totals<kMolTeam, false><<<blocks, 256, 0, s.stream>>>(A, nullptr);
    MDX_LAUNCHED();
    A.e_out = acc.p;
    k_e3b_totals<kMolTeam, true><<<blocks, 256, 0, s.stream>>>(A, nullptr);
    MDX_LAUNCHED();
    A.e_out = acc.p + 1;
    k_e3b_forces<kMolTeam, true><<<blocks, 256, 0, s.stream>>>(A, nullptr);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaMemcpyAsync(out, acc.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    return 0;
}

// ---- batched replicas: one launch per pass, blockIdx.y = replica ----------
int batch_e3b_tables(Batch &b) {
    const int R = (int)b.reps.size();
    std::vector<E3BArgs> h(R);
    for (int r = 0; r < R; r++) {
        State &s = *b.reps[r];
        FixE3B &f = *s.e3bFix();
        if (!f.side_ok || !f.f_side.p) {
            set_error(MDX_ERR_UNSUPPORTED, "batched E3B needs FixRigid molecules matching the E3B molecules");
            return MDX_ERR_UNSUPPORTED;
        }
        h[r] = e3b_args(s, f, f.f_side.p);
    }
    if (int e = b.tab_e3b.alloc(R * sizeof(E3BArgs))) return e;
    MDX_CUDA_TRY(cudaMemcpy(b.tab_e3b.p, h.data(), R * sizeof(E3BArgs), cudaMemcpyHostToDevice));
    return 0;
}

static int batch_e3b_sizing(Batch &b, E3BArgs *out) {
    if (!b.tab_e3b.p) {
        set_error(MDX_ERR_STATE, "batch tables not built (prepare the batch)");
        return MDX_ERR_STATE;
    }
    State &s0 = *b.reps[0];
    E3BArgs A = e3b_args(s0, *s0.e3bFix(), nullptr);
    A.nmol = b.max_mol;
    *out = A;
    return 0;
}

int batch_e3b_list(Batch &b) {
    E3BArgs A;
    if (int e = batch_e3b_sizing(b, &A)) return e;
    const E3BArgs *tab = reinterpret_cast<const E3BArgs *>(b.tab_e3b.p);
    const dim3 grid = e3b_blocks(b.max_mol, (unsigned)b.reps.size());
    // each kernel returns at once for the replicas of the other form
    if (!b.ps.empty()) {
        k_e3b_list<kMolTeam><<<grid, 256, 0, b.stream>>>(A, tab, 1);
        MDX_LAUNCHED();
    }
    if (!b.mfi.empty()) {  // from each replica's molecule-pair list
        k_e3b_list_mf<kMolTeam><<<grid, 256, 0, b.stream>>>(A, tab);
        MDX_LAUNCHED();
    }
    return 0;
}

int batch_e3b_forces(Batch &b, cudaStream_t stream) {
    E3BArgs A;
    if (int e = batch_e3b_sizing(b, &A)) return e;
    const E3BArgs *tab = reinterpret_cast<const E3BArgs *>(b.tab_e3b.p);
    const dim3 blocks = e3b_blocks(b.max_mol, (unsigned)b.reps.size());
    k_e3b_totals<kMolTeam, false, true><<<blocks, 256, 0, stream>>>(A, tab);
    MDX_LAUNCHED();
    k_e3b_forces<kMolTeam, false, true><<<blocks, 256, 0, stream>>>(A, tab);
    MDX_LAUNCHED();
    return 0;
}

int FixE3B::compute(int virialMode) {
    if (sur && sur->enabled) return surrogate_compute(*state, *this);
    if (int e = e3b_forces(*state, *this)) return e;
    return virialMode ? e3b_virial(*state, *this) : 0;
}

// after e3b_forces (the totals are current)
int e3b_virial(State &s, FixE3B &f) {
    const int nmol = (int)f.mol_ids.size();
    if (nmol == 0) return 0;
    const E3BArgs A = e3b_args(s, f, s.gpd.fs.p);
    k_e3b_virial<kMolTeam><<<e3b_blocks(nmol), 256, 0, s.stream>>>(A, s.gpd.virials.p);
    MDX_LAUNCHED();
    return 0;
}

int FixE3B::handleLocalData() { return 0; }

}  // namespace mdx
