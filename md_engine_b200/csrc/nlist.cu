// Cell-binned neighbour list (the GridGPU component, src/GridGPU.cu:824-1103).
//
// Differences from the reference's launch structure (the pair SET is the
// same, see below):
//  * no host round trips: the rebuild decision (setBuildFlag, GridGPU.cu:755),
//    the cell histogram, the exclusive scan (host cumulativeSum at
//    GridGPU.cu:902-908) and the list sizing all stay on the device; every
//    kernel of the rebuild group reads DeviceStatus::rebuild and returns
//    immediately when no rebuild is due, so the group can sit inside a
//    captured CUDA graph.
//  * search cells are >= cut/m wide (m = 2: a 5x5x5 stencil walked as 25
//    contiguous z-rows) instead of >= cut with 27 cells; the atoms tested are
//    a superset of every pair within cut, and each pair is tested once with
//    the minimum-image shift, so the pair set is unchanged.
//  * atoms are ordered by (cell, type, id) -- deterministic -- instead of the
//    atomicAdd arrival order of countNumInGridCells (GridGPU.cu:190-203).
//  * one sweep writes the list into a fixed per-atom capacity (overflow is
//    flagged in the status word) instead of count + max + prefix + assign.
//
// The predicate is the reference's FP32 expression (GridGPU.cu:326-338,
// 518-522): d = (x_j + shift) - x_i, r2 = dot(d, d) as nvcc contracts it,
// fma(dz, dz, fma(dy, dy, dx*dx)), pair kept iff r2 < cut*cut (float).
#include <algorithm>
#include <cstdio>
#include <vector>

#include "engine.hpp"

namespace mdx {

namespace {

__device__ __forceinline__ int cell_coord(float x, float lo, float inv_ds, int n) {
    int c = (int)((x - lo) * inv_ds);
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

struct CellGrid {
    float3 lo;
    float3 inv_ds;
    int3 ns;
};

__device__ __forceinline__ int cell_of_pos(const CellGrid &g, float3 p) {
    int cx = cell_coord(p.x, g.lo.x, g.inv_ds.x, g.ns.x);
    int cy = cell_coord(p.y, g.lo.y, g.inv_ds.y, g.ns.y);
    int cz = cell_coord(p.z, g.lo.z, g.inv_ds.z, g.ns.z);
    return (cx * g.ns.y + cy) * g.ns.z + cz;
}

// setBuildFlag (GridGPU.cu:755-774) + the periodicInterval gate of
// IntegratorVerlet.cu:696: rebuild iff forced, or turn % interval == 0 and
// any atom moved more than skin/2 since the last build.
__global__ void k_check(const float4 *__restrict__ xs, const float4 *__restrict__ xs_last, int n, Box box,
                        float skin2_quarter, int interval, int force, DeviceStatus *st) {
    if (!force) {
        long long t = st->turn;
        if (interval <= 0 || (t % interval) != 0) return;
    } else {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->rebuild = 1u;
        return;
    }
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int moved = 0;
    if (i < n) {
        float3 d = min_image(box, f3(xs[i]) - f3(xs_last[i]));
        moved = dot3(d, d) > skin2_quarter;
    }
    if (__syncthreads_or(moved) && threadIdx.x == 0) atomicOr(&st->rebuild, 1u);
}

// periodicWrap (GridGPU.cu:138-161) + countNumInGridCells (GridGPU.cu:190-203)
__global__ void k_wrap_bin(float4 *__restrict__ xs, int n, Box box, CellGrid g, int *__restrict__ cell_of,
                           uint32_t *__restrict__ cell_count, const DeviceStatus *st) {
    if (!st->rebuild) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = xs[i];
    float ix = floorf((p.x - box.lo.x) / box.L.x);
    float iy = floorf((p.y - box.lo.y) / box.L.y);
    float iz = floorf((p.z - box.lo.z) / box.L.z);
    if (ix != 0.f || iy != 0.f || iz != 0.f) {
        p.x = p.x - box.L.x * ix;
        p.y = p.y - box.L.y * iy;
        p.z = p.z - box.L.z * iz;
        xs[i] = p;
    }
    int c = cell_of_pos(g, f3(p));
    cell_of[i] = c;
    atomicAdd(cell_count + c, 1u);
}

// exclusive scan of the cell histogram in one block (replaces the host
// cumulativeSum, helpers.h:15-24); also clears the fill counters
__global__ void k_scan_cells(const uint32_t *__restrict__ count, uint32_t *__restrict__ start,
                             uint32_t *__restrict__ fill, int ncell, const DeviceStatus *st) {
    if (!st->rebuild) return;
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < ncell; base += blockDim.x) {
        int c = base + threadIdx.x;
        uint32_t v = c < ncell ? count[c] : 0u;
        if (c < ncell) fill[c] = 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t t = lane < nw ? warp_tot[lane] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            if (lane < nw) warp_tot[lane] = t;
        }
        __syncthreads();
        uint32_t excl = carry + (w > 0 ? warp_tot[w - 1] : 0u) + x - v;
        if (c < ncell) start[c] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) start[ncell] = carry;
}

__global__ void k_scatter(const int *__restrict__ cell_of, const uint32_t *__restrict__ start,
                          uint32_t *__restrict__ fill, int *__restrict__ perm_tmp, int n, const DeviceStatus *st) {
    if (!st->rebuild) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cell_of[i];
    uint32_t slot = atomicAdd(fill + c, 1u);
    perm_tmp[start[c] + slot] = i;
}

// deterministic order inside each cell: rank by (type, id); one warp per cell
__global__ void k_rank(const uint32_t *__restrict__ start, const int *__restrict__ perm_tmp,
                       const float4 *__restrict__ xs, const uint32_t *__restrict__ ids, int *__restrict__ perm,
                       int ncell, const DeviceStatus *st) {
    if (!st->rebuild) return;
    int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (c >= ncell) return;
    uint32_t s = start[c], e = start[c + 1];
    for (uint32_t p = s + lane; p < e; p += 32) {
        int a = perm_tmp[p];
        unsigned long long ka = ((unsigned long long)(uint32_t)type_of(xs[a]) << 32) | ids[a];
        uint32_t r = 0;
        for (uint32_t q = s; q < e; q++) {
            int b = perm_tmp[q];
            unsigned long long kb = ((unsigned long long)(uint32_t)type_of(xs[b]) << 32) | ids[b];
            r += kb < ka;
        }
        perm[s + r] = a;
    }
}

// sortPerAtomArrays (GridGPU.cu:253-293): gather every stream into the
// alternate buffers and rebuild idToIdx
__global__ void k_gather(const int *__restrict__ perm, int n, const float4 *__restrict__ xs,
                         const float4 *__restrict__ vs, const float4 *__restrict__ fs, const float *__restrict__ qs,
                         const uint32_t *__restrict__ ids, float4 *__restrict__ xs2, float4 *__restrict__ vs2,
                         float4 *__restrict__ fs2, float *__restrict__ qs2, uint32_t *__restrict__ ids2,
                         int *__restrict__ idToIdx, const DeviceStatus *st) {
    if (!st->rebuild) return;
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    int s = perm[d];
    xs2[d] = xs[s];
    vs2[d] = vs[s];
    fs2[d] = fs[s];
    qs2[d] = qs[s];
    uint32_t id = ids[s];
    ids2[d] = id;
    idToIdx[id] = d;
}

// assignNeighbors / assignFromCell (GridGPU.cu:482-734) with the exclusion
// lookup of addExclusion (GridGPU.cu:466-478).  Team of T lanes per atom;
// also copies the sorted streams back to the primary buffers.
template <int T>
__global__ void __launch_bounds__(256) k_build(
    int n, const float4 *__restrict__ xs2, const float4 *__restrict__ vs2, const float4 *__restrict__ fs2,
    const float *__restrict__ qs2, const uint32_t *__restrict__ ids2, float4 *__restrict__ xs,
    float4 *__restrict__ vs, float4 *__restrict__ fs, float *__restrict__ qs, uint32_t *__restrict__ ids,
    float4 *__restrict__ xs_last, const uint32_t *__restrict__ cell_start, CellGrid g, Box box, int m,
    float cutsq, const int *__restrict__ excl_start, const uint32_t *__restrict__ excl_ids, int use_excl,
    uint32_t *__restrict__ counts, uint32_t *__restrict__ nlist, int cap, DeviceStatus *st) {
    if (!st->rebuild) return;
    constexpr int G = 32 / T;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / T, t = lane % T;
    const int i = warp * G + a;
    if (i >= n) return;  // whole team leaves together
    const unsigned team_mask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << (a * T));
    const float4 pi4 = xs2[i];
    if (t == 0) {
        xs[i] = pi4;
        xs_last[i] = pi4;
        vs[i] = vs2[i];
        fs[i] = fs2[i];
        qs[i] = qs2[i];
        ids[i] = ids2[i];
    }
    const float3 pi = f3(pi4);
    const int cx = cell_coord(pi.x, g.lo.x, g.inv_ds.x, g.ns.x);
    const int cy = cell_coord(pi.y, g.lo.y, g.inv_ds.y, g.ns.y);
    const int cz = cell_coord(pi.z, g.lo.z, g.inv_ds.z, g.ns.z);
    int e0 = 0, e1 = 0;
    if (use_excl) {
        uint32_t myid = ids2[i];
        e0 = excl_start[myid];
        e1 = excl_start[myid + 1];
    }
    uint32_t *mylist = nlist + (size_t)(i / G) * cap * G + a * T + t;
    int cnt = 0;
    for (int dx = -m; dx <= m; dx++) {
        int kx = cx + dx;
        float sx = 0.f;
        if (kx < 0) { kx += g.ns.x; sx = -box.L.x; }
        else if (kx >= g.ns.x) { kx -= g.ns.x; sx = box.L.x; }
        for (int dy = -m; dy <= m; dy++) {
            int ky = cy + dy;
            float sy = 0.f;
            if (ky < 0) { ky += g.ns.y; sy = -box.L.y; }
            else if (ky >= g.ns.y) { ky -= g.ns.y; sy = box.L.y; }
            const int rowbase = (kx * g.ns.y + ky) * g.ns.z;
            // up to three z segments: [main, wrapped low, wrapped high]
            for (int seg = 0; seg < 3; seg++) {
                int z0, z1;
                float sz = 0.f;
                if (seg == 0) {
                    z0 = cz - m < 0 ? 0 : cz - m;
                    z1 = cz + m >= g.ns.z ? g.ns.z - 1 : cz + m;
                } else if (seg == 1) {
                    if (cz - m >= 0) continue;
                    z0 = cz - m + g.ns.z;
                    z1 = g.ns.z - 1;
                    sz = -box.L.z;
                } else {
                    if (cz + m < g.ns.z) continue;
                    z0 = 0;
                    z1 = cz + m - g.ns.z;
                    sz = box.L.z;
                }
                const int pbeg = cell_start[rowbase + z0];
                const int pend = cell_start[rowbase + z1 + 1];
                for (int p0 = pbeg; p0 < pend; p0 += T) {
                    const int p = p0 + t;
                    bool hit = false;
                    if (p < pend && p != i) {
                        const float4 pj = xs2[p];
                        const float ddx = __fsub_rn(__fadd_rn(pj.x, sx), pi.x);
                        const float ddy = __fsub_rn(__fadd_rn(pj.y, sy), pi.y);
                        const float ddz = __fsub_rn(__fadd_rn(pj.z, sz), pi.z);
                        const float r2 = __fmaf_rn(ddz, ddz, __fmaf_rn(ddy, ddy, __fmul_rn(ddx, ddx)));
                        hit = r2 < cutsq;
                    }
                    const unsigned b = __ballot_sync(team_mask, hit);
                    if (hit) {
                        const unsigned mine = (T == 32) ? b : (b >> (a * T));
                        const int pos = cnt + __popc(mine & ((1u << t) - 1u));
                        if (pos < cap) {
                            uint32_t entry = (uint32_t)p;
                            if (use_excl) {
                                const uint32_t oid = ids2[p];
                                for (int e = e0; e < e1; e++) {
                                    const uint32_t x = excl_ids[e];
                                    if ((x & kExclMask) == oid) { entry |= x & ~kExclMask; break; }
                                }
                            }
                            // k-th entry: row k/T, column within team k%T
                            mylist[(size_t)(pos / T) * 32 + (pos % T) - t] = entry;
                        }
                    }
                    cnt += __popc(b);
                }
            }
        }
    }
    if (t == 0) {
        counts[i] = (uint32_t)cnt;
        if (cnt > cap) atomicOr(&st->bits, kStatusNlistOverflow);
        atomicMax(&st->max_neighbors, (uint32_t)cnt);
    }
}

// single block: every thread must read the flag before it is cleared
__global__ void k_finish(uint32_t *__restrict__ cell_count, int ncell, DeviceStatus *st) {
    if (!st->rebuild) return;
    for (int c = threadIdx.x; c < ncell; c += blockDim.x) cell_count[c] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        st->n_builds += 1;
        st->rebuild = 0u;
    }
}

// count-only sweep used to size the list before the first build
template <int T>
__global__ void k_count_only(int n, const float4 *__restrict__ xs2, const uint32_t *__restrict__ cell_start,
                             CellGrid g, Box box, int m, float cutsq, DeviceStatus *st) {
    constexpr int G = 32 / T;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int a = lane / T, t = lane % T;
    const int i = warp * G + a;
    if (i >= n) return;
    const unsigned team_mask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << (a * T));
    const float3 pi = f3(xs2[i]);
    const int cx = cell_coord(pi.x, g.lo.x, g.inv_ds.x, g.ns.x);
    const int cy = cell_coord(pi.y, g.lo.y, g.inv_ds.y, g.ns.y);
    const int cz = cell_coord(pi.z, g.lo.z, g.inv_ds.z, g.ns.z);
    int cnt = 0;
    for (int dx = -m; dx <= m; dx++) {
        int kx = cx + dx;
        float sx = 0.f;
        if (kx < 0) { kx += g.ns.x; sx = -box.L.x; }
        else if (kx >= g.ns.x) { kx -= g.ns.x; sx = box.L.x; }
        for (int dy = -m; dy <= m; dy++) {
            int ky = cy + dy;
            float sy = 0.f;
            if (ky < 0) { ky += g.ns.y; sy = -box.L.y; }
            else if (ky >= g.ns.y) { ky -= g.ns.y; sy = box.L.y; }
            const int rowbase = (kx * g.ns.y + ky) * g.ns.z;
            for (int dz = -m; dz <= m; dz++) {
                int kz = cz + dz;
                float sz = 0.f;
                if (kz < 0) { kz += g.ns.z; sz = -box.L.z; }
                else if (kz >= g.ns.z) { kz -= g.ns.z; sz = box.L.z; }
                const int pbeg = cell_start[rowbase + kz], pend = cell_start[rowbase + kz + 1];
                for (int p0 = pbeg; p0 < pend; p0 += T) {
                    const int p = p0 + t;
                    bool hit = false;
                    if (p < pend && p != i) {
                        const float4 pj = xs2[p];
                        const float ddx = __fsub_rn(__fadd_rn(pj.x, sx), pi.x);
                        const float ddy = __fsub_rn(__fadd_rn(pj.y, sy), pi.y);
                        const float ddz = __fsub_rn(__fadd_rn(pj.z, sz), pi.z);
                        const float r2 = __fmaf_rn(ddz, ddz, __fmaf_rn(ddy, ddy, __fmul_rn(ddx, ddx)));
                        hit = r2 < cutsq;
                    }
                    cnt += __popc(__ballot_sync(team_mask, hit));
                }
            }
        }
    }
    if (t == 0) atomicMax(&st->max_neighbors, (uint32_t)cnt);
}

CellGrid make_grid(const State &s) {
    CellGrid g;
    g.lo = s.box.lo;
    g.ns = s.grid.ns;
    g.inv_ds = make_float3((float)(s.grid.ns.x / s.box.Ld.x), (float)(s.grid.ns.y / s.box.Ld.y),
                           (float)(s.grid.ns.z / s.box.Ld.z));
    return g;
}

template <int T>
void launch_build(State &s, const CellGrid &g, float cutsq) {
    GridGPU &gr = s.grid;
    GPUData &d = s.gpd;
    int warps = (d.n + (32 / T) - 1) / (32 / T);
    int blocks = (warps * 32 + 255) / 256;
    k_build<T><<<blocks, 256, 0, s.stream>>>(
        d.n, d.xs_alt.p, d.vs_alt.p, d.fs_alt.p, d.qs_alt.p, d.ids_alt.p, d.xs.p, d.vs.p, d.fs.p, d.qs.p, d.ids.p,
        d.xs_last_build.p, gr.cell_start.p, g, s.box, gr.m, cutsq, gr.excl_start.p, gr.excl_ids.p,
        gr.have_excl ? 1 : 0, gr.counts.p, gr.nlist.p, gr.cap, s.d_status.p);
    MDX_LAUNCHED();
}

template <int T>
void launch_count(State &s, const CellGrid &g, float cutsq) {
    int warps = (s.gpd.n + (32 / T) - 1) / (32 / T);
    int blocks = (warps * 32 + 255) / 256;
    k_count_only<T><<<blocks, 256, 0, s.stream>>>(s.gpd.n, s.gpd.xs_alt.p, s.grid.cell_start.p, g, s.box, s.grid.m,
                                                  cutsq, s.d_status.p);
    MDX_LAUNCHED();
}

int dispatch_team(int team, void (*f1)(), void (*f2)(), void (*f4)(), void (*f8)(), void (*f16)(), void (*f32)()) {
    switch (team) {
        case 1: f1(); return 0;
        case 2: f2(); return 0;
        case 4: f4(); return 0;
        case 8: f8(); return 0;
        case 16: f16(); return 0;
        case 32: f32(); return 0;
    }
    return MDX_ERR_ARG;
}

}  // namespace

// Exclusion list by bond-graph depth (handleExclusionsDistance /
// generateExclusionList, GridGPU.cu:1377-1518): level d+1 = neighbours of
// level-d atoms that are not closer and not the atom itself; tags 1..3.
int nlist_exclusions(State &s) {
    std::vector<std::pair<int, int>> bonds;
    for (Fix *f : s.fixes) f->getBonds(bonds);
    GridGPU &gr = s.grid;
    gr.have_excl = !bonds.empty();
    if (!gr.have_excl) return 0;
    const int nid = (int)s.atoms.size();
    std::vector<std::vector<int>> adj(nid);
    for (auto &b : bonds) {
        adj[b.first].push_back(b.second);
        adj[b.second].push_back(b.first);
    }
    std::vector<int> start(nid + 1, 0);
    std::vector<uint32_t> ent;
    std::vector<int> level(nid, -1);  // scratch: depth at which an id was reached
    std::vector<int> touched;
    for (int i = 0; i < nid; i++) {
        touched.clear();
        level[i] = 0;
        touched.push_back(i);
        std::vector<int> frontier{i};
        for (int depth = 1; depth <= 3; depth++) {
            std::vector<int> next;
            for (int a : frontier)
                for (int b : adj[a])
                    if (level[b] < 0) {
                        level[b] = depth;
                        touched.push_back(b);
                        next.push_back(b);
                    }
            std::sort(next.begin(), next.end());
            next.erase(std::unique(next.begin(), next.end()), next.end());
            for (int b : next) ent.push_back((uint32_t)b | ((uint32_t)depth << 30));
            frontier.swap(next);
        }
        for (int t : touched) level[t] = -1;
        start[i + 1] = (int)ent.size();
        gr.max_excl = std::max(gr.max_excl, start[i + 1] - start[i]);
    }
    if (int e = gr.excl_start.alloc(start.size())) return e;
    if (int e = gr.excl_ids.alloc(ent.size())) return e;
    MDX_CUDA_TRY(cudaMemcpy(gr.excl_start.p, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(gr.excl_ids.p, ent.data(), ent.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    return 0;
}

// Grid set-up (GridGPU::setBounds, GridGPU.cu:46-66): cells of width
// >= cut/m, m = 2 when the box allows 2m+1 cells per side, else 1.
int nlist_init(State &s) {
    GridGPU &gr = s.grid;
    gr.cut = (float)((double)(float)s.maxRCut() + s.padding);
    gr.skin = (float)s.padding;
    int m = 2;
    int3 ns;
    for (;; m--) {
        if (m == 0) {
            set_error(MDX_ERR_UNSUPPORTED, "box (%g %g %g) too small for neighbour cutoff %g: need >= 3 cells per side",
                      s.box.Ld.x, s.box.Ld.y, s.box.Ld.z, (double)gr.cut);
            return MDX_ERR_UNSUPPORTED;
        }
        double w = (double)gr.cut / m * (1.0 + 1e-5);
        ns = make_int3((int)(s.box.Ld.x / w), (int)(s.box.Ld.y / w), (int)(s.box.Ld.z / w));
        if (ns.x >= 2 * m + 1 && ns.y >= 2 * m + 1 && ns.z >= 2 * m + 1) break;
    }
    gr.m = m;
    gr.ns = ns;
    int ncell = ns.x * ns.y * ns.z;
    if (int e = gr.cell_start.alloc(ncell + 1)) return e;
    if (int e = gr.cell_count.alloc(ncell)) return e;
    if (int e = gr.cell_fill.alloc(ncell)) return e;
    MDX_CUDA_TRY(cudaMemsetAsync(gr.cell_count.p, 0, ncell * sizeof(uint32_t), s.stream));
    const int n = s.gpd.n;
    if (int e = gr.cell_of.alloc(n)) return e;
    if (int e = gr.perm_tmp.alloc(n)) return e;
    if (int e = gr.perm.alloc(n)) return e;
    if (int e = gr.counts.alloc(n)) return e;
    if (s.nThreadPerAtom > 0) {
        gr.team = s.nThreadPerAtom;
    } else {
        // density * list volume -> mean neighbours; about 8-16 entries per lane
        double vol = s.box.Ld.x * s.box.Ld.y * s.box.Ld.z;
        double nbar = n / vol * 4.18879 * (double)gr.cut * gr.cut * gr.cut;
        gr.team = nbar > 256 ? 8 : (nbar > 48 ? 4 : 2);
    }
    if (gr.team != 1 && gr.team != 2 && gr.team != 4 && gr.team != 8 && gr.team != 16 && gr.team != 32) {
        set_error(MDX_ERR_ARG, "nThreadPerAtom must be 1,2,4,8,16 or 32 (got %d)", gr.team);
        return MDX_ERR_ARG;
    }
    return nlist_exclusions(s);
}

// GridGPU::periodicBoundaryConditions (GridGPU.cu:824-1103).  conditional:
// run the check kernel that decides on the device (graph mode); otherwise
// the rebuild is forced (force=true) or decided by the same check.
int nlist_rebuild(State &s, bool force, bool conditional) {
    GridGPU &gr = s.grid;
    GPUData &d = s.gpd;
    const int n = d.n;
    const int ncell = gr.ns.x * gr.ns.y * gr.ns.z;
    const CellGrid g = make_grid(s);
    const float cutsq = gr.cut * gr.cut;
    const float skin2q = (float)(s.padding * s.padding) * 0.25f;
    (void)conditional;
    k_check<<<(n + 255) / 256, 256, 0, s.stream>>>(d.xs.p, d.xs_last_build.p, n, s.box, skin2q, s.periodicInterval,
                                                   force ? 1 : 0, s.d_status.p);
    MDX_LAUNCHED();
    k_wrap_bin<<<(n + 255) / 256, 256, 0, s.stream>>>(d.xs.p, n, s.box, g, gr.cell_of.p, gr.cell_count.p, s.d_status.p);
    MDX_LAUNCHED();
    k_scan_cells<<<1, 1024, 0, s.stream>>>(gr.cell_count.p, gr.cell_start.p, gr.cell_fill.p, ncell, s.d_status.p);
    MDX_LAUNCHED();
    k_scatter<<<(n + 255) / 256, 256, 0, s.stream>>>(gr.cell_of.p, gr.cell_start.p, gr.cell_fill.p, gr.perm_tmp.p, n,
                                                     s.d_status.p);
    MDX_LAUNCHED();
    k_rank<<<(ncell * 32 + 255) / 256, 256, 0, s.stream>>>(gr.cell_start.p, gr.perm_tmp.p, d.xs.p, d.ids.p, gr.perm.p,
                                                           ncell, s.d_status.p);
    MDX_LAUNCHED();
    k_gather<<<(n + 255) / 256, 256, 0, s.stream>>>(gr.perm.p, n, d.xs.p, d.vs.p, d.fs.p, d.qs.p, d.ids.p, d.xs_alt.p,
                                                    d.vs_alt.p, d.fs_alt.p, d.qs_alt.p, d.ids_alt.p, d.idToIdx.p,
                                                    s.d_status.p);
    MDX_LAUNCHED();
    if (gr.cap == 0) {
        // first build: size the per-atom capacity from a counting sweep
        MDX_CUDA_TRY(cudaMemsetAsync(&s.d_status.p->max_neighbors, 0, sizeof(uint32_t), s.stream));
        switch (gr.team) {
            case 1: launch_count<1>(s, g, cutsq); break;
            case 2: launch_count<2>(s, g, cutsq); break;
            case 4: launch_count<4>(s, g, cutsq); break;
            case 8: launch_count<8>(s, g, cutsq); break;
            case 16: launch_count<16>(s, g, cutsq); break;
            default: launch_count<32>(s, g, cutsq); break;
        }
        uint32_t mx = 0;
        MDX_CUDA_TRY(cudaMemcpyAsync(&mx, &s.d_status.p->max_neighbors, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                     s.stream));
        MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
        int c = (int)(mx * 1.35 + 32);
        c = (c + gr.team - 1) / gr.team * gr.team;
        gr.cap = c;
        size_t groups = (size_t)(n + (32 / gr.team) - 1) / (32 / gr.team);
        if (int e = gr.nlist.alloc(groups * (size_t)c * (32 / gr.team))) return e;
    }
    switch (gr.team) {
        case 1: launch_build<1>(s, g, cutsq); break;
        case 2: launch_build<2>(s, g, cutsq); break;
        case 4: launch_build<4>(s, g, cutsq); break;
        case 8: launch_build<8>(s, g, cutsq); break;
        case 16: launch_build<16>(s, g, cutsq); break;
        default: launch_build<32>(s, g, cutsq); break;
    }
    // molecule maps / molecule list of the fixes that keep atom indices
    if (FixRigid *r = s.rigidFix()) {
        if (int e = rigid_update_maps(s, *r, true)) return e;
    }
    if (FixE3B *e3 = s.e3bFix()) {
        if (int e = e3b_build_list(s, *e3, true)) return e;
    }
    k_finish<<<1, 1024, 0, s.stream>>>(gr.cell_count.p, ncell, s.d_status.p);
    MDX_LAUNCHED();
    gr.built = true;
    return 0;
}

}  // namespace mdx
