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
//  * search cells are >= cut/m wide (m <= 4: a (2m+1)^3 stencil walked as
//    (2m+1)^2 contiguous z-rows) instead of >= cut with 27 cells; the atoms tested are
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
#include <cmath>
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

// Arguments of the rebuild-group kernels for one system.  Every kernel takes
// a0 (single system) and tab (batched replicas: tab[blockIdx.y], a0 is then
// only the largest replica used to size the grid).
struct GridArgs {
    float4 *xs, *vs, *fs;
    float *qs;
    uint32_t *ids;
    float4 *xs2, *vs2, *fs2;
    float *qs2;
    uint32_t *ids2;
    float4 *xs_last;
    int *idToIdx;
    int *cell_of;
    uint32_t *cell_count, *cell_start, *cell_fill;
    int *perm_tmp, *perm;
    DeviceStatus *st;
    Box box;
    CellGrid g;
    int n, ncell, interval;
    float skin2q;
    // 1: a list build into the alternate buffers only (the molecule form's
    // per-site list for Grid.getNeighborList): idToIdx, the primary streams
    // and the build counter are left alone
    int view;
};
#define MDX_GRID_ARGS \
    pdl_wait();       \
    const GridArgs A = tab ? tab[blockIdx.y] : a0

// setBuildFlag (GridGPU.cu:755-774) + the periodicInterval gate of
// IntegratorVerlet.cu:696: rebuild iff forced, or turn % interval == 0 and
// any atom moved more than skin/2 since the last build.
__global__ void k_check(const GridArgs a0, const GridArgs *__restrict__ tab, int force) {
    MDX_GRID_ARGS;
    DeviceStatus *st = A.st;
    if (!force) {
        long long t = st->turn;
        if (A.interval <= 0 || (t % A.interval) != 0) return;
    } else {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->rebuild = 1u;
        return;
    }
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int moved = 0;
    if (i < A.n) {
        float3 d = min_image(A.box, f3(A.xs[i]) - f3(A.xs_last[i]));
        moved = dot3(d, d) > A.skin2q;
    }
    if (__syncthreads_or(moved) && threadIdx.x == 0) atomicOr(&st->rebuild, 1u);
}

// periodicWrap (GridGPU.cu:138-161) + countNumInGridCells (GridGPU.cu:190-203)
__global__ void k_wrap_bin(const GridArgs a0, const GridArgs *__restrict__ tab) {
    MDX_GRID_ARGS;
    if (!A.st->rebuild) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const Box &box = A.box;
    float4 p = A.xs[i];
    float ix = floorf((p.x - box.lo.x) / box.L.x);
    float iy = floorf((p.y - box.lo.y) / box.L.y);
    float iz = floorf((p.z - box.lo.z) / box.L.z);
    if (ix != 0.f || iy != 0.f || iz != 0.f) {
        p.x = p.x - box.L.x * ix;
        p.y = p.y - box.L.y * iy;
        p.z = p.z - box.L.z * iz;
        if (!A.view) A.xs[i] = p;  // a view build wraps its sorted copy only (k_gather)
    }
    int c = cell_of_pos(A.g, f3(p));
    A.cell_of[i] = c;
    atomicAdd(A.cell_count + c, 1u);
}

// exclusive scan of the cell histogram in one block per system (replaces the
// host cumulativeSum, helpers.h:15-24); also clears the fill counters.  The
// counts pass through shared memory in tiles of kScanTile cells: coalesced
// loads and stores, thread t scans its eight consecutive cells in registers,
// warp and block totals by shuffles, a running carry across tiles.
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;
__global__ void __launch_bounds__(kScanThreads) k_scan_cells(const GridArgs a0, const GridArgs *__restrict__ tab) {
    MDX_GRID_ARGS;
    if (!A.st->rebuild) return;
    const uint32_t *__restrict__ count = A.cell_count;
    uint32_t *__restrict__ start = A.cell_start;
    uint32_t *__restrict__ fill = A.cell_fill;
    const int ncell = A.ncell;
    __shared__ uint4 tile4[kScanTile / 4];
    __shared__ uint32_t warp_tot[32];
    uint32_t *const tile = reinterpret_cast<uint32_t *>(tile4);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int nw = kScanThreads / 32;
    uint32_t carry = 0u;
    for (int base = 0; base < ncell; base += kScanTile) {
        const int nt = min(kScanTile, ncell - base);
#pragma unroll
        for (int k = 0; k < kScanPer; k++) {
            const int c = k * kScanThreads + (int)threadIdx.x;
            tile[c] = c < nt ? count[base + c] : 0u;
        }
        __syncthreads();
        const uint4 a = tile4[2 * threadIdx.x], b = tile4[2 * threadIdx.x + 1];
        const uint32_t v[kScanPer] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        uint32_t run = 0u;
#pragma unroll
        for (int k = 0; k < kScanPer; k++) run += v[k];
        uint32_t x = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t t = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;
        }
        __syncthreads();
        uint32_t excl = carry + (w > 0 ? warp_tot[w - 1] : 0u) + x - run;
        uint32_t e[kScanPer];
#pragma unroll
        for (int k = 0; k < kScanPer; k++) {
            e[k] = excl;
            excl += v[k];
        }
        tile4[2 * threadIdx.x] = make_uint4(e[0], e[1], e[2], e[3]);
        tile4[2 * threadIdx.x + 1] = make_uint4(e[4], e[5], e[6], e[7]);
        carry += warp_tot[nw - 1];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kScanPer; k++) {
            const int c = k * kScanThreads + (int)threadIdx.x;
            if (c < nt) {
                start[base + c] = tile[c];
                fill[base + c] = 0u;
            }
        }
        __syncthreads();  // tile and warp_tot are reused by the next tile
    }
    if (threadIdx.x == 0) start[ncell] = carry;
}

__global__ void k_scatter(const GridArgs a0, const GridArgs *__restrict__ tab) {
    MDX_GRID_ARGS;
    if (!A.st->rebuild) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    int c = A.cell_of[i];
    uint32_t slot = atomicAdd(A.cell_fill + c, 1u);
    A.perm_tmp[A.cell_start[c] + slot] = i;
}

// deterministic order inside each cell: rank by (type, id); one warp per cell
__global__ void k_rank(const GridArgs a0, const GridArgs *__restrict__ tab) {
    MDX_GRID_ARGS;
    if (!A.st->rebuild) return;
    int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (c >= A.ncell) return;
    const int *__restrict__ perm_tmp = A.perm_tmp;
    const float4 *__restrict__ xs = A.xs;
    const uint32_t *__restrict__ ids = A.ids;
    uint32_t s = A.cell_start[c], e = A.cell_start[c + 1];
    for (uint32_t p = s + lane; p < e; p += 32) {
        int a = perm_tmp[p];
        unsigned long long ka = ((unsigned long long)(uint32_t)type_of(xs[a]) << 32) | ids[a];
        uint32_t r = 0;
        for (uint32_t q = s; q < e; q++) {
            int b = perm_tmp[q];
            unsigned long long kb = ((unsigned long long)(uint32_t)type_of(xs[b]) << 32) | ids[b];
            r += kb < ka;
        }
        A.perm[s + r] = a;
    }
}

// sortPerAtomArrays (GridGPU.cu:253-293): gather every stream into the
// alternate buffers and rebuild idToIdx
__global__ void k_gather(const GridArgs a0, const GridArgs *__restrict__ tab) {
    MDX_GRID_ARGS;
    if (!A.st->rebuild) return;
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= A.n) return;
    int s = A.perm[d];
    if (A.view) {
        // the view build's copy, wrapped as k_wrap_bin wraps in place
        const Box &box = A.box;
        float4 p = A.xs[s];
        const float ix = floorf((p.x - box.lo.x) / box.L.x);
        const float iy = floorf((p.y - box.lo.y) / box.L.y);
        const float iz = floorf((p.z - box.lo.z) / box.L.z);
        if (ix != 0.f || iy != 0.f || iz != 0.f) {
            p.x = p.x - box.L.x * ix;
            p.y = p.y - box.L.y * iy;
            p.z = p.z - box.L.z * iz;
        }
        A.xs2[d] = p;
    } else {
        A.xs2[d] = A.xs[s];
    }
    A.vs2[d] = A.vs[s];
    A.fs2[d] = A.fs[s];
    A.qs2[d] = A.qs[s];
    uint32_t id = A.ids[s];
    A.ids2[d] = id;
    if (!A.view) A.idToIdx[id] = d;
}

// the sorted streams back into the primary buffers (the captured graph keeps
// the same pointers), and the positions of this list build for the skin check
__global__ void k_copyback(const GridArgs a0, const GridArgs *__restrict__ tab) {
    MDX_GRID_ARGS;
    if (!A.st->rebuild) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const float4 p = A.xs2[i];
    A.xs[i] = p;
    A.xs_last[i] = p;
    A.vs[i] = A.vs2[i];
    A.fs[i] = A.fs2[i];
    A.qs[i] = A.qs2[i];
    A.ids[i] = A.ids2[i];
}

// assignNeighbors / assignFromCell (GridGPU.cu:482-734) with the exclusion
// lookup of addExclusion (GridGPU.cu:466-478), one warp per home cell.
// The candidates of the cell -- its (2m+1)^2 stencil rows, each row's z range
// and each row trimmed to the cells that can hold a point within cut of the
// home atoms' bounding box (conservative margin of 1e-3 cell) -- are laid out
// as one sequence of contiguous segments of the sorted streams.  The warp
// walks that sequence 32 candidates at a time, one candidate per lane,
// already shifted by its periodic image (x_j + shift, the reference's first
// rounding), for HG home atoms at once held in registers.  The sequence is
// first expanded into shared memory (sorted index and image code per
// candidate, windows of kCandWin) so a chunk costs one shared load; every lane tests
// its candidate against each of them with the reference's predicate and two
// ballots give the hit and the "can interact" masks.  The warp owns whole
// rows, so a single pass writes them: interacting pairs at the front,
// provably zero ones at the back, each slot from the running counts (the same
// in every lane) plus a popcount of the lower lanes' hits -- deterministic,
// and the entries written for one home atom at a time are consecutive slots
// of its row.  Exclusion depths come from the id-window bit planes (the id
// list only for atoms with far exclusions).  COUNT counts alone to size the
// first build.
constexpr int kBuildCellsPerBlock = 4;            // one warp per cell
constexpr int kStencilMax = 4;                    // largest m (cells >= cut/m)
constexpr int kBuildSegMax = 2 * (2 * kStencilMax + 1) * (2 * kStencilMax + 1);  // two z segments per row
constexpr int kCandWin = 1536;                    // expanded candidates per warp and window
constexpr int kCandIdxBits = 27;                  // sorted index bits of an expanded candidate
constexpr int kCandPad = 64;                      // harmless entries after a window (branch-free prefetch)
constexpr uint32_t kNoShift = 13u;                // image code (1,1,1): no shift

struct BuildArgs {
    const float4 *xs2, *vs2, *fs2;
    const float *qs2;
    const uint32_t *ids2;
    float4 *xs, *vs, *fs;
    float *qs;
    uint32_t *ids;
    float4 *xs_last;
    const uint32_t *cell_start;
    const int *excl_start;
    const uint32_t *excl_ids;
    const ulonglong2 *excl_win;
    const uint8_t *excl_far;
    const uint32_t *ljmask;
    uint32_t *counts, *counts_int, *nlist;
    DeviceStatus *st;
    CellGrid g;
    Box box;
    int ncell, m, use_excl, part_q, cap;
    float cutsq;
};

// exclusion depth of the pair (home id myid, candidate id oid): bit planes of
// the id window (w, in registers), else the id list of an atom with far
// exclusions
__device__ __forceinline__ uint32_t excl_depth(const BuildArgs &A, uint32_t myid, bool far, ulonglong2 w,
                                               uint32_t oid) {
    const uint32_t dd = oid - myid + 32u;
    uint32_t depth = 0u;
    if (dd < 64u) depth = (uint32_t)((w.x >> dd) & 1ull) | ((uint32_t)((w.y >> dd) & 1ull) << 1);
    if (far && depth == 0u) {
        for (int e = A.excl_start[myid]; e < A.excl_start[myid + 1]; e++) {
            const uint32_t x = A.excl_ids[e];
            if ((x & kExclMask) == oid) {
                depth = x >> 30;
                break;
            }
        }
    }
    return depth;
}

// SPLIT: interacting pairs to the front of a row, provably zero ones to the
// back (ljmask, part_q); EXCL: exclusion depths from the id window.  Both are
// compile-time so that the candidate loop carries no tests for them.
template <int TP, int HG, bool COUNT, bool SPLIT, bool EXCL>
__global__ void __launch_bounds__(kBuildCellsPerBlock * 32, 7) k_build_cells(const BuildArgs a0,
                                                                            const BuildArgs *__restrict__ tab) {
    pdl_wait();
    const BuildArgs A = tab ? tab[blockIdx.y] : a0;
    if (!COUNT && !A.st->rebuild) return;
    constexpr int GP = 32 / TP;
    // segment table: offset in the sequence | image code << kCandIdxBits,
    // and the first sorted index (two words per segment: seven blocks fit
    // an SM beside the candidate windows)
    __shared__ uint32_t sh_seg_offc_all[kBuildCellsPerBlock][kBuildSegMax + 1];
    __shared__ int sh_seg_beg_all[kBuildCellsPerBlock][kBuildSegMax];
    __shared__ uint32_t sh_cand_all[kBuildCellsPerBlock][kCandWin + kCandPad];
    __shared__ float4 sh_shift[27];  // image shift by code (ix+1) + 3 (iy+1) + 9 (iz+1)
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    if (threadIdx.x < 27) {
        const int t = threadIdx.x;
        sh_shift[t] = make_float4((float)(t % 3 - 1) * A.box.L.x, (float)(t / 3 % 3 - 1) * A.box.L.y,
                                  (float)(t / 9 - 1) * A.box.L.z, 0.f);
    }
    __syncthreads();  // the only block-wide barrier: warps own cells from here on
    const int c = blockIdx.x * kBuildCellsPerBlock + wib;
    if (c >= A.ncell) return;
    uint32_t *const sh_seg_offc = sh_seg_offc_all[wib];
    int *const sh_seg_beg = sh_seg_beg_all[wib];
    uint32_t *const sh_cand = sh_cand_all[wib];
    const CellGrid &g = A.g;
    const int cs = (int)A.cell_start[c], ce = (int)A.cell_start[c + 1];
    if (ce <= cs) return;
    const int cz = c % g.ns.z, cy = (c / g.ns.z) % g.ns.y, cx = c / (g.ns.z * g.ns.y);
    const int m = A.m, side = 2 * m + 1;
    const float cutsq = A.cutsq;
    const uint32_t cap = (uint32_t)A.cap;
    uint32_t *const nlist = A.nlist;
    const float dsx = 1.0f / g.inv_ds.x, dsy = 1.0f / g.inv_ds.y, dsz = 1.0f / g.inv_ds.z;
    const uint32_t lt = (1u << lane) - 1u;
    // bounding box of the home atoms' positions
    float bxl = 3.0e38f, bxh = -3.0e38f, byl = 3.0e38f, byh = -3.0e38f, bzl = 3.0e38f, bzh = -3.0e38f;
    for (int i = cs + lane; i < ce; i += 32) {
        const float4 p4 = A.xs2[i];
        bxl = fminf(bxl, p4.x);
        bxh = fmaxf(bxh, p4.x);
        byl = fminf(byl, p4.y);
        byh = fmaxf(byh, p4.y);
        bzl = fminf(bzl, p4.z);
        bzh = fmaxf(bzh, p4.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        bxl = fminf(bxl, __shfl_xor_sync(0xffffffffu, bxl, o));
        bxh = fmaxf(bxh, __shfl_xor_sync(0xffffffffu, bxh, o));
        byl = fminf(byl, __shfl_xor_sync(0xffffffffu, byl, o));
        byh = fmaxf(byh, __shfl_xor_sync(0xffffffffu, byh, o));
        bzl = fminf(bzl, __shfl_xor_sync(0xffffffffu, bzl, o));
        bzh = fmaxf(bzh, __shfl_xor_sync(0xffffffffu, bzh, o));
    }
    // segment table: lane r builds stencil row r's z segments, rows in
    // chunks of 32 with the running totals carried
    int seg_base = 0, cand_base = 0;
    for (int r0 = 0; r0 < side * side; r0 += 32) {
        // up to two segments per row (the stencil wraps at most once):
        // the parts of the z range below, inside and above the box
        int nseg = 0, b0 = 0, l0 = 0, b1 = 0, l1 = 0;
        uint32_t cxy = 0u, cz0 = 0u, cz1 = 0u;  // image codes
        const int r = r0 + lane;
        if (r < side * side) {
            const int kx = cx - m + r / side, ky = cy - m + r % side;
            const int kxw = kx < 0 ? kx + g.ns.x : (kx >= g.ns.x ? kx - g.ns.x : kx);
            const uint32_t ix = kx < 0 ? 0u : (kx >= g.ns.x ? 2u : 1u);
            const int kyw = ky < 0 ? ky + g.ns.y : (ky >= g.ns.y ? ky - g.ns.y : ky);
            const uint32_t iy = ky < 0 ? 0u : (ky >= g.ns.y ? 2u : 1u);
            cxy = ix + 3u * iy;
            // distance from the home box to this row of cells (image
            // frame), shrunk by the margin
            const float clx = g.lo.x + (float)kx * dsx;
            const float cly = g.lo.y + (float)ky * dsy;
            float dxm = fmaxf(fmaxf(clx - bxh, bxl - (clx + dsx)), 0.f);
            float dym = fmaxf(fmaxf(cly - byh, byl - (cly + dsy)), 0.f);
            dxm = fmaxf(dxm - 1e-3f * dsx, 0.f);
            dym = fmaxf(dym - 1e-3f * dsy, 0.f);
            const float rz2 = cutsq - dxm * dxm - dym * dym;
            if (rz2 > 0.f) {
                const float rz = sqrtf(rz2) + 1e-3f * dsz;
                const int zlo = max(cz - m, (int)floorf((bzl - rz - g.lo.z) * g.inv_ds.z));
                const int zhi = min(cz + m, (int)floorf((bzh + rz - g.lo.z) * g.inv_ds.z));
                const int rowbase = (kxw * g.ns.y + kyw) * g.ns.z;
#pragma unroll
                for (int part = 0; part < 3; part++) {
                    const int za = part == 0 ? zlo : (part == 1 ? max(zlo, 0) : max(zlo, g.ns.z));
                    const int ze = part == 0 ? min(zhi, -1) : (part == 1 ? min(zhi, g.ns.z - 1) : zhi);
                    const int wrap = part == 0 ? g.ns.z : (part == 1 ? 0 : -g.ns.z);
                    const uint32_t czp = 9u * (uint32_t)part;
                    if (za <= ze) {
                        const int pbeg = (int)A.cell_start[rowbase + za + wrap];
                        const int pend = (int)A.cell_start[rowbase + ze + wrap + 1];
                        if (pend > pbeg) {
                            if (nseg == 0) {
                                b0 = pbeg;
                                l0 = pend - pbeg;
                                cz0 = czp;
                            } else {
                                b1 = pbeg;
                                l1 = pend - pbeg;
                                cz1 = czp;
                            }
                            nseg++;
                        }
                    }
                }
            }
        }
        // inclusive scans of the segment counts and lengths
        int so = nseg, lo = l0 + l1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int a = __shfl_up_sync(0xffffffffu, so, o);
            const int b = __shfl_up_sync(0xffffffffu, lo, o);
            if (lane >= o) {
                so += a;
                lo += b;
            }
        }
        const int slot = seg_base + so - nseg, off = cand_base + lo - (l0 + l1);
        if (nseg > 0) {
            sh_seg_beg[slot] = b0;
            sh_seg_offc[slot] = (uint32_t)off | ((cxy + cz0) << kCandIdxBits);
        }
        if (nseg > 1) {
            sh_seg_beg[slot + 1] = b1;
            sh_seg_offc[slot + 1] = (uint32_t)(off + l0) | ((cxy + cz1) << kCandIdxBits);
        }
        // the first window straight from the rows, every lane its own
        // segments (later windows of a long sequence expand from the table)
        {
            const uint32_t w0c = (cxy + cz0) << kCandIdxBits, w1c = (cxy + cz1) << kCandIdxBits;
            const int e0 = min(off + l0, kCandWin), e1 = min(off + l0 + l1, kCandWin);
            for (int t = off; t < e0; t++) sh_cand[t] = (uint32_t)(b0 - off + t) | w0c;
            for (int t = off + l0; t < e1; t++) sh_cand[t] = (uint32_t)(b1 - off - l0 + t) | w1c;
        }
        seg_base += __shfl_sync(0xffffffffu, so, 31);
        cand_base += __shfl_sync(0xffffffffu, lo, 31);
    }
    if (lane == 0) sh_seg_offc[seg_base] = (uint32_t)cand_base;  // total candidates

    __syncwarp();
    const int nseg = seg_base;
    const int total = cand_base;
    if (total >= (1 << kCandIdxBits)) {  // the packed table offset cannot hold it
        if (lane == 0) atomicOr(&A.st->bits, kStatusNlistOverflow);
        return;
    }

    // the prefetch reads up to kCandPad entries past a window: the cell's
    // first site, unshifted (in bounds, never counted)
    auto pad = [&](int wn) {
        for (int t = wn + lane; t < wn + kCandPad; t += 32) sh_cand[t] = (uint32_t)cs | (kNoShift << kCandIdxBits);
    };
    // expand candidates [w0, w0 + wn) of the segment sequence into sh_cand
    auto expand = [&](int w0, int wn) {
        __syncwarp();
        for (int sg = 0; sg < nseg; sg++) {
            constexpr uint32_t kOffMask = (1u << kCandIdxBits) - 1u;
            const uint32_t oc = sh_seg_offc[sg];
            const int off = (int)(oc & kOffMask);
            const int lo = max(off, w0), hi = min((int)(sh_seg_offc[sg + 1] & kOffMask), w0 + wn);
            const uint32_t beg = (uint32_t)(sh_seg_beg[sg] - off), code = oc & ~kOffMask;
            for (int t = lo + lane; t < hi; t += 32) sh_cand[t - w0] = (beg + (uint32_t)t) | code;
        }
        pad(wn);
        __syncwarp();
    };
    const bool single = total <= kCandWin;
    if (single) {
        pad(total);
        __syncwarp();
    }
    // home atoms HG at a time, in registers (warp-uniform values)
    for (int g0 = cs; g0 < ce; g0 += HG) {
        float hx[HG], hy[HG], hz[HG], hq[HG];
        uint32_t hmask[HG], hid[HG], ci[HG], cn[HG];
        ulonglong2 hwin[HG];
        bool hfar[HG];
        uint32_t *hrow[HG];
#pragma unroll
        for (int k = 0; k < HG; k++) {
            const int i = g0 + k;
            const bool v = i < ce;
            const int ii = v ? i : cs;
            const float4 p4 = A.xs2[ii];
            // an absent home slot sits far outside the box: r^2 overflows to
            // infinity and it never hits
            hx[k] = v ? p4.x : 3.0e37f;
            hy[k] = v ? p4.y : 3.0e37f;
            hz[k] = v ? p4.z : 3.0e37f;
            hq[k] = SPLIT && A.part_q ? A.qs2[ii] : 0.f;
            hmask[k] = SPLIT ? A.ljmask[type_of(p4)] : 0xffffffffu;
            hid[k] = EXCL ? A.ids2[ii] : 0u;
            hfar[k] = EXCL ? A.excl_far[hid[k]] != 0 : false;
            hwin[k] = EXCL ? A.excl_win[hid[k]] : make_ulonglong2(0ull, 0ull);
            hrow[k] = nlist + (size_t)(ii / GP) * cap * GP + (ii % GP) * TP;
            ci[k] = 0u;
            cn[k] = 0u;
        }
        for (int w0 = 0; w0 < total; w0 += kCandWin) {
            const int wn = min(kCandWin, total - w0);
            if (!single) expand(w0, wn);
            // candidate: sorted index, raw position, image shift, charge, id;
            // the next chunk's loads are issued before the current one is
            // tested (indices up to wn + 63 < wn + kCandPad: no bounds test)
            uint32_t pn = 0u, idn = 0u;
            float4 pjn, shn;
            float qn = 0.f;
            auto fetch = [&](int k) {
                const uint32_t e = sh_cand[k];
                pn = e & ((1u << kCandIdxBits) - 1u);
                shn = sh_shift[e >> kCandIdxBits];
                pjn = A.xs2[pn];
                if (SPLIT) qn = A.qs2[pn];
                if (EXCL) idn = A.ids2[pn];
            };
            fetch(lane);
#pragma unroll 2
            for (int c0 = 0; c0 < wn; c0 += 32) {
                const uint32_t p = pn;
                const bool cval = c0 + lane < wn;
                const float cxj = __fadd_rn(pjn.x, shn.x);
                const float cyj = __fadd_rn(pjn.y, shn.y);
                const float czj = __fadd_rn(pjn.z, shn.z);
                const uint32_t tj = (uint32_t)type_of(pjn);
                const float qj = qn;
                const uint32_t oid = idn;
                fetch(c0 + 32 + lane);
                bool hit[HG], act[HG];
                uint32_t hm[HG], am[HG];
#pragma unroll
                for (int k = 0; k < HG; k++) {
                    const float ddx = __fsub_rn(cxj, hx[k]);
                    const float ddy = __fsub_rn(cyj, hy[k]);
                    const float ddz = __fsub_rn(czj, hz[k]);
                    const float r2 = __fmaf_rn(ddz, ddz, __fmaf_rn(ddy, ddy, __fmul_rn(ddx, ddx)));
                    hit[k] = cval && r2 < cutsq && p != (uint32_t)(g0 + k);
                    hm[k] = __ballot_sync(0xffffffffu, hit[k]);
                    act[k] = true;
                    am[k] = hm[k];
                    if (SPLIT && !COUNT) {
                        act[k] = ((hmask[k] >> tj) & 1u) != 0u || hq[k] * qj != 0.f;
                        am[k] = __ballot_sync(0xffffffffu, hit[k] && act[k]);
                    }
                }
#pragma unroll
                for (int k = 0; k < HG; k++) {
                    if (COUNT) {
                        ci[k] += __popc(hm[k]);
                        continue;
                    }
                    if (hm[k] == 0u) continue;  // warp-uniform: no hit for this home in the chunk
                    const uint32_t before = __popc(hm[k] & lt);
                    const uint32_t bi = __popc(am[k] & lt);
                    const uint32_t pos = act[k] ? ci[k] + bi : cap - 1u - cn[k] - (before - bi);
                    uint32_t entry = p;
                    // a depth needs an id within 32 of the home's (the bit
                    // window) or a home with far exclusions; most chunks have
                    // neither
                    if (EXCL && (hfar[k] || __any_sync(0xffffffffu, hit[k] && oid - hid[k] + 32u < 64u)))
                        entry |= excl_depth(A, hid[k], hfar[k], hwin[k], oid) << 30;
                    if (hit[k] && ci[k] + cn[k] + before < cap) hrow[k][(pos / TP) * 32u + pos % TP] = entry;
                    const uint32_t na = __popc(am[k]);
                    ci[k] += na;
                    cn[k] += __popc(hm[k]) - na;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < HG; k++) {
            if (lane == k && g0 + k < ce) {
                const int i = g0 + k;
                const uint32_t cnt = ci[k] + cn[k];
                if (COUNT) {
                    atomicMax(&A.st->max_neighbors, cnt);
                } else {
                    A.counts[i] = cnt;
                    A.counts_int[i] = ci[k];
                    if (cnt > cap) atomicOr(&A.st->bits, kStatusNlistOverflow);
                    atomicMax(&A.st->max_neighbors, cnt);
                }
            }
        }
    }
}

// single block: every thread must read the flag before it is cleared
__global__ void k_finish(const GridArgs a0, const GridArgs *__restrict__ tab) {
    MDX_GRID_ARGS;
    DeviceStatus *st = A.st;
    if (!st->rebuild) return;
    for (int c = threadIdx.x; c < A.ncell; c += blockDim.x) A.cell_count[c] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        if (!A.view) st->n_builds += 1;
        st->rebuild = 0u;
    }
}

// ---- molecule form (all-rigid four-site water) ---------------------------
// The sort unit is the molecule: its cell is the cell of its site 0, slots
// are ordered by (cell, molecule index), and slot d's sites land at 4d .. 4d+3
// of every per-atom stream.
struct MolGridArgs {
    float4 *xs, *vs, *fs;
    float *qs;
    uint32_t *ids;
    float4 *xs2, *vs2, *fs2;
    float *qs2;
    uint32_t *ids2;
    float4 *xs_last;
    int *idToIdx;
    int4 *mol_idx;      // FixRigid's molecule -> atom indices (rewritten by the sort)
    int4 *mol_idx_e3b;  // FixE3B's copy of the same molecules (may be null)
    int *cell_of;
    uint32_t *cell_count, *cell_start, *cell_fill;
    int *perm_tmp, *perm;
    uint32_t *counts, *list;
    int cap, team;
    DeviceStatus *st;
    Box box;
    CellGrid g;
    int nmol, ncell, m;
    float cut2;
};

// one system (m0) or, for batched replicas, tab[blockIdx.y] (m0 then only
// sizes the grid; blocks past a smaller replica's work return at once)
#define MDX_MG_ARGS \
    pdl_wait();     \
    const MolGridArgs M = tab ? tab[blockIdx.y] : m0

__device__ __forceinline__ float4 wrap_pos(const Box &box, float4 p, bool &moved) {
    // periodicWrap (GridGPU.cu:138-161), per site
    const float ix = floorf((p.x - box.lo.x) / box.L.x);
    const float iy = floorf((p.y - box.lo.y) / box.L.y);
    const float iz = floorf((p.z - box.lo.z) / box.L.z);
    moved = ix != 0.f || iy != 0.f || iz != 0.f;
    if (moved) {
        p.x = p.x - box.L.x * ix;
        p.y = p.y - box.L.y * iy;
        p.z = p.z - box.L.z * iz;
    }
    return p;
}

// site 0 wrapped into the box (periodicWrap's formula), the other sites put
// at their minimum-image offset from it, so every molecule is stored whole
// (as SETTLE leaves it after every step); the molecule binned by its site 0
__global__ void k_mf_wrap_bin(const MolGridArgs m0, const MolGridArgs *__restrict__ tab) {
    MDX_MG_ARGS;
    if (!M.st->rebuild) return;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M.nmol) return;
    const int4 ix = M.mol_idx[m];
    const int at[4] = {ix.x, ix.y, ix.z, ix.w};
    bool moved;
    const float4 r0 = M.xs[at[0]];
    const float4 p0 = wrap_pos(M.box, r0, moved);
    if (moved) M.xs[at[0]] = p0;
#pragma unroll
    for (int k = 1; k < 4; k++) {
        const float4 r = M.xs[at[k]];
        const float3 d = min_image(M.box, f3(r) - f3(r0));
        const float4 p = make_float4(p0.x + d.x, p0.y + d.y, p0.z + d.z, r.w);
        if (p.x != r.x || p.y != r.y || p.z != r.z) M.xs[at[k]] = p;
    }
    const int c = cell_of_pos(M.g, f3(p0));
    M.cell_of[m] = c;
    atomicAdd(M.cell_count + c, 1u);
}

__global__ void k_mf_scatter(const MolGridArgs m0, const MolGridArgs *__restrict__ tab) {
    MDX_MG_ARGS;
    if (!M.st->rebuild) return;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M.nmol) return;
    const int c = M.cell_of[m];
    const uint32_t slot = atomicAdd(M.cell_fill + c, 1u);
    M.perm_tmp[M.cell_start[c] + slot] = m;
}

// deterministic order inside each cell: by molecule index; one warp per cell
__global__ void k_mf_rank(const MolGridArgs m0, const MolGridArgs *__restrict__ tab) {
    MDX_MG_ARGS;
    if (!M.st->rebuild) return;
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= M.ncell) return;
    const uint32_t s = M.cell_start[c], e = M.cell_start[c + 1];
    for (uint32_t p = s + lane; p < e; p += 32) {
        const int a = M.perm_tmp[p];
        uint32_t r = 0;
        for (uint32_t q = s; q < e; q++) r += M.perm_tmp[q] < a;
        M.perm[s + r] = a;
    }
}

// slot d <- molecule perm[d]: its four sites into 4d .. 4d+3 of the
// alternate streams and idToIdx rewritten; one thread per site
__global__ void k_mf_gather(const MolGridArgs m0, const MolGridArgs *__restrict__ tab) {
    MDX_MG_ARGS;
    if (!M.st->rebuild) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * M.nmol) return;
    const int d = t >> 2, site = t & 3;
    const int4 ix = M.mol_idx[M.perm[d]];
    const int s = site == 0 ? ix.x : (site == 1 ? ix.y : (site == 2 ? ix.z : ix.w));
    M.xs2[t] = M.xs[s];
    M.vs2[t] = M.vs[s];
    M.fs2[t] = M.fs[s];
    M.qs2[t] = M.qs[s];
    const uint32_t id = M.ids[s];
    M.ids2[t] = id;
    M.idToIdx[id] = t;
}

// the sorted streams back into the primary buffers, the positions of this
// build for the skin check, and the molecule maps (molecule perm[d] at slot d)
__global__ void k_mf_copyback(const MolGridArgs m0, const MolGridArgs *__restrict__ tab) {
    MDX_MG_ARGS;
    if (!M.st->rebuild) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 4 * M.nmol) return;
    const float4 p = M.xs2[i];
    M.xs[i] = p;
    M.xs_last[i] = p;
    M.vs[i] = M.vs2[i];
    M.fs[i] = M.fs2[i];
    M.qs[i] = M.qs2[i];
    M.ids[i] = M.ids2[i];
    if ((i & 3) == 0) {
        const int d = i >> 2;
        const int4 nx = make_int4(i, i + 1, i + 2, i + 3);
        M.mol_idx[M.perm[d]] = nx;
        if (M.mol_idx_e3b) M.mol_idx_e3b[M.perm[d]] = nx;
    }
}

// the molecule-pair list: one block per slot, one thread per row of its
// (2m+1)^2-row stencil (each row one or two contiguous runs of slots: the
// grid has at least 2m+1 cells per side, so no cell is seen twice).  A
// candidate is kept when the minimum-image distance of the site-0 positions
// is below the list radius.  Two passes over the row: count, a block scan of
// the row counts, then the writes -- rows in stencil order, candidates in slot
// order (deterministic) -- into the team layout: slot k's e-th entry at
// (k/G) cap G + (e/T) 32 + (k%G) T + e%T, G = 32/T.  Every row's cell-start
// loads and candidate loads are in flight at once instead of one row after
// another.
constexpr int kMfBuildThreads = 64;  // >= 49 rows (m <= 3)

__device__ __forceinline__ void mf_row_runs(const MolGridArgs &M, int r, int cx, int cy, int cz, int (&b)[2],
                                            int (&e)[2]) {
    const CellGrid &g = M.g;
    const int mm = M.m, side = 2 * mm + 1;
    int kx = cx - mm + r / side, ky = cy - mm + r % side;
    kx = kx < 0 ? kx + g.ns.x : (kx >= g.ns.x ? kx - g.ns.x : kx);
    ky = ky < 0 ? ky + g.ns.y : (ky >= g.ns.y ? ky - g.ns.y : ky);
    const int rowbase = (kx * g.ns.y + ky) * g.ns.z;
    const int zlo = cz - mm, zhi = cz + mm;
    int za[2], zb[2], nr;
    if (zlo < 0) {
        za[0] = zlo + g.ns.z; zb[0] = g.ns.z - 1; za[1] = 0; zb[1] = zhi; nr = 2;
    } else if (zhi >= g.ns.z) {
        za[0] = zlo; zb[0] = g.ns.z - 1; za[1] = 0; zb[1] = zhi - g.ns.z; nr = 2;
    } else {
        za[0] = zlo; zb[0] = zhi; za[1] = 0; zb[1] = -1; nr = 1;
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
        b[q] = 0;
        e[q] = 0;
        if (q < nr) {
            b[q] = (int)M.cell_start[rowbase + za[q]];
            e[q] = (int)M.cell_start[rowbase + zb[q] + 1];
        }
    }
}

__global__ void __launch_bounds__(kMfBuildThreads) k_mf_build(const MolGridArgs m0,
                                                               const MolGridArgs *__restrict__ tab) {
    MDX_MG_ARGS;
    if (!M.st->rebuild) return;
    const int k = blockIdx.x;
    if (k >= M.nmol) return;  // block-uniform
    __shared__ uint32_t sh_cnt[kMfBuildThreads];
    const int r = threadIdx.x;
    const int side = 2 * M.m + 1;
    const bool has_row = r < side * side;
    const float3 p = f3(M.xs2[4 * k]);
    const int c = cell_of_pos(M.g, p);
    const int cz = c % M.g.ns.z, cy = (c / M.g.ns.z) % M.g.ns.y, cx = c / (M.g.ns.z * M.g.ns.y);
    int b[2] = {0, 0}, e[2] = {0, 0};
    if (has_row) mf_row_runs(M, r, cx, cy, cz, b, e);
    // pass 1: this row's hits
    uint32_t n = 0;
#pragma unroll
    for (int q = 0; q < 2; q++)
        for (int j = b[q]; j < e[q]; j++) {
            if (j == k) continue;
            const float3 d = min_image(M.box, f3(M.xs2[4 * j]) - p);
            n += dot3(d, d) < M.cut2 ? 1u : 0u;
        }
    // exclusive scan of the row counts over the block (rows in order)
    sh_cnt[r] = n;
    __syncthreads();
    uint32_t off = 0, tot = 0;
    for (int q = 0; q < kMfBuildThreads; q++) {
        const uint32_t v = sh_cnt[q];
        off += q < r ? v : 0u;
        tot += v;
    }
    // pass 2: the writes
    const int T = M.team, G = 32 / T;
    uint32_t *const row = M.list + (size_t)(k / G) * M.cap * G + (k % G) * T;
    const uint32_t cap = (uint32_t)M.cap;
    uint32_t pos = off;
#pragma unroll
    for (int q = 0; q < 2; q++)
        for (int j = b[q]; j < e[q]; j++) {
            if (j == k) continue;
            const float3 d = min_image(M.box, f3(M.xs2[4 * j]) - p);
            if (dot3(d, d) < M.cut2) {
                if (pos < cap) row[(pos / T) * 32u + pos % T] = (uint32_t)j;
                pos++;
            }
        }
    if (r == 0) {
        M.counts[k] = tot;
        if (tot > cap) atomicOr(&M.st->bits, kStatusNlistOverflow);
        atomicMax(&M.st->max_mol_neighbors, tot);
    }
}

CellGrid make_grid(const State &s) {
    CellGrid g;
    g.lo = s.box.lo;
    g.ns = s.grid.ns;
    g.inv_ds = make_float3((float)(s.grid.ns.x / s.box.Ld.x), (float)(s.grid.ns.y / s.box.Ld.y),
                           (float)(s.grid.ns.z / s.box.Ld.z));
    return g;
}

GridArgs grid_args(State &s) {
    GridGPU &gr = s.grid;
    GPUData &d = s.gpd;
    GridArgs A{};
    A.xs = d.xs.p;
    A.vs = d.vs.p;
    A.fs = d.fs.p;
    A.qs = d.qs.p;
    A.ids = d.ids.p;
    A.xs2 = d.xs_alt.p;
    A.vs2 = d.vs_alt.p;
    A.fs2 = d.fs_alt.p;
    A.qs2 = d.qs_alt.p;
    A.ids2 = d.ids_alt.p;
    A.xs_last = d.xs_last_build.p;
    A.idToIdx = d.idToIdx.p;
    A.cell_of = gr.cell_of.p;
    A.cell_count = gr.cell_count.p;
    A.cell_start = gr.cell_start.p;
    A.cell_fill = gr.cell_fill.p;
    A.perm_tmp = gr.perm_tmp.p;
    A.perm = gr.perm.p;
    A.st = s.d_status.p;
    A.box = s.box;
    A.g = make_grid(s);
    A.n = d.n;
    A.ncell = gr.ns.x * gr.ns.y * gr.ns.z;
    A.interval = s.periodicInterval;
    A.skin2q = (float)(s.padding * s.padding) * 0.25f;
    A.view = 0;
    return A;
}

CellGrid mol_grid(const State &s) {
    CellGrid g;
    g.lo = s.box.lo;
    g.ns = s.mf.ns;
    g.inv_ds = make_float3((float)(s.mf.ns.x / s.box.Ld.x), (float)(s.mf.ns.y / s.box.Ld.y),
                           (float)(s.mf.ns.z / s.box.Ld.z));
    return g;
}

MolGridArgs mol_grid_args(State &s) {
    MolForm &mf = s.mf;
    GPUData &d = s.gpd;
    MolGridArgs M{};
    M.xs = d.xs.p;
    M.vs = d.vs.p;
    M.fs = d.fs.p;
    M.qs = d.qs.p;
    M.ids = d.ids.p;
    M.xs2 = d.xs_alt.p;
    M.vs2 = d.vs_alt.p;
    M.fs2 = d.fs_alt.p;
    M.qs2 = d.qs_alt.p;
    M.ids2 = d.ids_alt.p;
    M.xs_last = d.xs_last_build.p;
    M.idToIdx = d.idToIdx.p;
    M.mol_idx = s.rigidFix()->d_mol_idx.p;
    // (FixE3B's map is the identity slot map in this form, never rewritten)
    M.mol_idx_e3b = nullptr;
    M.cell_of = mf.cell_of.p;
    M.cell_count = mf.cell_count.p;
    M.cell_start = mf.cell_start.p;
    M.cell_fill = mf.cell_fill.p;
    M.perm_tmp = mf.perm_tmp.p;
    M.perm = mf.perm.p;
    M.counts = mf.counts.p;
    M.list = mf.list.p;
    M.cap = mf.cap;
    M.team = mf.team;
    M.st = s.d_status.p;
    M.box = s.box;
    M.g = mol_grid(s);
    M.nmol = mf.nmol;
    M.ncell = mf.ns.x * mf.ns.y * mf.ns.z;
    M.m = mf.m;
    M.cut2 = mf.cut * mf.cut;
    return M;
}

// the scan / finish kernels over the molecule grid's cell arrays
GridArgs mol_scan_args(State &s) {
    GridArgs A = grid_args(s);
    A.cell_count = s.mf.cell_count.p;
    A.cell_start = s.mf.cell_start.p;
    A.cell_fill = s.mf.cell_fill.p;
    A.ncell = s.mf.ns.x * s.mf.ns.y * s.mf.ns.z;
    return A;
}

BuildArgs build_args(State &s, const CellGrid &g, float cutsq) {
    GridGPU &gr = s.grid;
    GPUData &d = s.gpd;
    BuildArgs A{};
    A.xs2 = d.xs_alt.p;
    A.vs2 = d.vs_alt.p;
    A.fs2 = d.fs_alt.p;
    A.qs2 = d.qs_alt.p;
    A.ids2 = d.ids_alt.p;
    A.xs = d.xs.p;
    A.vs = d.vs.p;
    A.fs = d.fs.p;
    A.qs = d.qs.p;
    A.ids = d.ids.p;
    A.xs_last = d.xs_last_build.p;
    A.cell_start = gr.cell_start.p;
    A.excl_start = gr.excl_start.p;
    A.excl_ids = gr.excl_ids.p;
    A.excl_win = gr.excl_win.p;
    A.excl_far = gr.excl_far.p;
    A.ljmask = gr.partition ? gr.ljmask.p : nullptr;
    A.counts = gr.counts.p;
    A.counts_int = gr.counts_int.p;
    A.nlist = gr.nlist.p;
    A.st = s.d_status.p;
    A.g = g;
    A.box = s.box;
    A.ncell = g.ns.x * g.ns.y * g.ns.z;
    A.m = gr.m;
    A.use_excl = gr.have_excl ? 1 : 0;
    A.part_q = gr.part_q ? 1 : 0;
    A.cap = gr.cap;
    A.cutsq = cutsq;
    return A;
}

template <int T, int HG, bool COUNT>
auto build_kernel(bool split, bool excl) {
    if constexpr (COUNT) {
        return k_build_cells<T, HG, true, false, false>;
    } else {
        return split ? (excl ? k_build_cells<T, HG, false, true, true> : k_build_cells<T, HG, false, true, false>)
                     : (excl ? k_build_cells<T, HG, false, false, true> : k_build_cells<T, HG, false, false, false>);
    }
}

template <int T, bool COUNT>
void launch_build_hg(int hg, dim3 grid, cudaStream_t st, const BuildArgs &A, const BuildArgs *tab) {
    const bool split = A.ljmask != nullptr, excl = A.use_excl != 0;
    auto k = hg == 4 ? build_kernel<T, 4, COUNT>(split, excl) : build_kernel<T, 2, COUNT>(split, excl);
    if (tab) {
        k<<<grid, kBuildCellsPerBlock * 32, 0, st>>>(A, tab);
        MDX_LAUNCHED();
    } else {
        launch_pdl(k, grid, dim3(kBuildCellsPerBlock * 32), 0, st, A, tab);
    }
}

// grid.x covers ncell (or the largest replica's) cells, one warp each
template <bool COUNT>
void launch_build_any(int team, int hg, dim3 grid, cudaStream_t st, const BuildArgs &A, const BuildArgs *tab) {
    switch (team) {
        case 1: launch_build_hg<1, COUNT>(hg, grid, st, A, tab); break;
        case 2: launch_build_hg<2, COUNT>(hg, grid, st, A, tab); break;
        case 4: launch_build_hg<4, COUNT>(hg, grid, st, A, tab); break;
        case 8: launch_build_hg<8, COUNT>(hg, grid, st, A, tab); break;
        case 16: launch_build_hg<16, COUNT>(hg, grid, st, A, tab); break;
        default: launch_build_hg<32, COUNT>(hg, grid, st, A, tab); break;
    }
}

inline dim3 build_grid(int ncell, int nrep) {
    return dim3((ncell + kBuildCellsPerBlock - 1) / kBuildCellsPerBlock, nrep);
}

void launch_build(State &s, const CellGrid &g, float cutsq, cudaStream_t st) {
    const BuildArgs A = build_args(s, g, cutsq);
    launch_build_any<false>(s.grid.team, s.grid.home_group, build_grid(A.ncell, 1), st, A, nullptr);
}

void launch_count(State &s, const CellGrid &g, float cutsq) {
    BuildArgs A = build_args(s, g, cutsq);
    A.use_excl = 0;
    A.ljmask = nullptr;
    A.part_q = 0;
    A.cap = 0;
    launch_build_any<true>(s.grid.team, s.grid.home_group, build_grid(A.ncell, 1), s.stream, A, nullptr);
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
    gr.h_excl_start.assign(s.atoms.size() + 1, 0);
    gr.h_excl_ids.clear();
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
    std::vector<ulonglong2> win(nid, make_ulonglong2(0ull, 0ull));
    std::vector<uint8_t> far(nid, 0);
    for (int i = 0; i < nid; i++)
        for (int e = start[i]; e < start[i + 1]; e++) {
            const long long d = (long long)(ent[e] & kExclMask) - i + 32;
            const uint32_t depth = ent[e] >> 30;
            if (d < 0 || d >= 64) {
                far[i] = 1;
                continue;
            }
            if (depth & 1u) win[i].x |= 1ull << d;
            if (depth & 2u) win[i].y |= 1ull << d;
        }
    if (int e = gr.excl_win.alloc(nid)) return e;
    if (int e = gr.excl_far.alloc(nid)) return e;
    MDX_CUDA_TRY(cudaMemcpy(gr.excl_win.p, win.data(), nid * sizeof(ulonglong2), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(gr.excl_far.p, far.data(), nid * sizeof(uint8_t), cudaMemcpyHostToDevice));
    gr.h_excl_start = start;
    gr.h_excl_ids = ent;
    if (int e = gr.excl_start.alloc(start.size())) return e;
    if (int e = gr.excl_ids.alloc(ent.size())) return e;
    MDX_CUDA_TRY(cudaMemcpy(gr.excl_start.p, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(gr.excl_ids.p, ent.data(), ent.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    return 0;
}

// Which listed pairs can interact: bit tj of ljmask[ti] is set when the pair
// fix's evaluator can give (ti, tj) a force (eps != 0; eps14 != 0 for
// LJCHARMM; C != 0 for TICG); with a charge fix (Ewald or DSF), pairs with
// q_i q_j != 0 also interact.  Everything else contributes exactly zero
// force, energy and virial in compute_force_iso (the pair evaluators scale by
// eps or C, the charge evaluators by q_i q_j) and is kept at the back of the
// row.
int nlist_set_interactions(State &s) {
    GridGPU &gr = s.grid;
    FixPair *pf = s.pairFix();
    const int nt = (int)s.species.size();
    gr.partition = false;
    gr.part_q = false;
    if (!pf || nt > 32 || pf->h_params.size() != (size_t)pf->nparam() * nt * nt) return 0;
    std::vector<uint32_t> mask(nt, 0u);
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++)
            if (pf->pairActive(a, b)) mask[a] |= 1u << b;
    if (int e = gr.ljmask.alloc(nt)) return e;
    MDX_CUDA_TRY(cudaMemcpy(gr.ljmask.p, mask.data(), nt * sizeof(uint32_t), cudaMemcpyHostToDevice));
    gr.partition = true;
    gr.part_q = pf->chargeFix != nullptr || pf->dsfFix != nullptr;
    return 0;
}

// Grid set-up (GridGPU::setBounds, GridGPU.cu:46-66): cells of width
// >= cut/m instead of >= cut, m chosen below.
int nlist_init(State &s) {
    GridGPU &gr = s.grid;
    gr.cut = (float)((double)(float)s.maxRCut() + s.padding);
    gr.skin = (float)s.padding;
    // minimum image: one periodic image of a pair at most can lie within cut
    if (2.0 * (double)gr.cut >= std::min(s.box.Ld.x, std::min(s.box.Ld.y, s.box.Ld.z))) {
        set_error(MDX_ERR_UNSUPPORTED, "neighbour cutoff %g (rCut + padding) must be below half the box (%g %g %g)",
                  (double)gr.cut, s.box.Ld.x, s.box.Ld.y, s.box.Ld.z);
        return MDX_ERR_UNSUPPORTED;
    }
    // cells of at least cut/m, m as large as keeps a mean of 2 atoms per
    // cell (finer cells trim the candidate volume toward the cutoff sphere).
    // A (2m+1)-cell stencil row wraps the box at most once when there are
    // >= 2m cells per side; a cell it visits under two images holds at most
    // one image within cut < L/2.  m = 1 needs 3 cells per side.
    if (s.gridStencil < 0 || s.gridStencil > kStencilMax) {
        set_error(MDX_ERR_ARG, "gridStencil must be 0 (automatic) or 1..%d (got %d)", kStencilMax, s.gridStencil);
        return MDX_ERR_ARG;
    }
    int m = s.gridStencil > 0 ? s.gridStencil : kStencilMax;
    int3 ns;
    for (;; m--) {
        if (m == 0) {
            set_error(MDX_ERR_UNSUPPORTED, "box (%g %g %g) too small for neighbour cutoff %g: need >= 3 cells per side",
                      s.box.Ld.x, s.box.Ld.y, s.box.Ld.z, (double)gr.cut);
            return MDX_ERR_UNSUPPORTED;
        }
        double w = (double)gr.cut / m * (1.0 + 1e-5);
        ns = make_int3((int)(s.box.Ld.x / w), (int)(s.box.Ld.y / w), (int)(s.box.Ld.z / w));
        const int need = std::max(3, 2 * m);
        if (ns.x < need || ns.y < need || ns.z < need) continue;
        if (m == 1 || s.gridStencil > 0 || (double)s.gpd.n >= 2.0 * ns.x * ns.y * ns.z) break;
    }
    if (s.gpd.n >= (1 << kCandIdxBits)) {
        set_error(MDX_ERR_UNSUPPORTED, "neighbour list build limited to %d atoms (got %d)", 1 << kCandIdxBits, s.gpd.n);
        return MDX_ERR_UNSUPPORTED;
    }
    gr.m = m;
    gr.ns = ns;
    int ncell = ns.x * ns.y * ns.z;
    // list build: home atoms tested four at a time when cells hold that many
    if (s.gridHomeGroup != 0 && s.gridHomeGroup != 2 && s.gridHomeGroup != 4) {
        set_error(MDX_ERR_ARG, "gridHomeGroup must be 0 (automatic), 2 or 4 (got %d)", s.gridHomeGroup);
        return MDX_ERR_ARG;
    }
    gr.home_group = s.gridHomeGroup ? s.gridHomeGroup : ((double)s.gpd.n >= 4.0 * ncell ? 4 : 2);
    if (int e = gr.cell_start.alloc(ncell + 1)) return e;
    if (int e = gr.cell_count.alloc(ncell)) return e;
    if (int e = gr.cell_fill.alloc(ncell)) return e;
    MDX_CUDA_TRY(cudaMemsetAsync(gr.cell_count.p, 0, ncell * sizeof(uint32_t), s.stream));
    const int n = s.gpd.n;
    if (int e = gr.cell_of.alloc(n)) return e;
    if (int e = gr.perm_tmp.alloc(n)) return e;
    if (int e = gr.perm.alloc(n)) return e;
    if (int e = gr.counts.alloc(n)) return e;
    if (int e = gr.counts_int.alloc(n)) return e;
    if (s.nThreadPerAtom > 0) {
        gr.team = s.nThreadPerAtom;
    } else {
        // density * list volume -> mean neighbours; a wide team for long rows
        // (water, 558 entries: 32 lanes measured 11 % faster than 16 in the
        // pair kernel, which reads only the interacting front of each row)
        double vol = s.box.Ld.x * s.box.Ld.y * s.box.Ld.z;
        double nbar = n / vol * 4.18879 * (double)gr.cut * gr.cut * gr.cut;
        gr.team = nbar > 400 ? 32 : (nbar > 256 ? 16 : (nbar > 128 ? 8 : (nbar > 48 ? 4 : 2)));
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
// bstream (optional): the list build, the E3B molecule list and k_finish go
// to that stream after the sort, so the caller can run the step's first half
// and the P3M chain beside them; it waits on s.ev_join[2] (recorded at the
// end of bstream) before anything that reads the lists.
static int nlist_rebuild_mf(State &s, bool force, cudaStream_t bstream);

int nlist_rebuild(State &s, bool force, bool conditional, cudaStream_t bstream) {
    if (s.mf.on) return nlist_rebuild_mf(s, force, bstream);
    GridGPU &gr = s.grid;
    GPUData &d = s.gpd;
    const int n = d.n;
    const int ncell = gr.ns.x * gr.ns.y * gr.ns.z;
    const CellGrid g = make_grid(s);
    const float cutsq = gr.cut * gr.cut;
    (void)conditional;
    const GridArgs A = grid_args(s);
    const int nb = (n + 255) / 256;
    const GridArgs *nt = nullptr;
    MDX_CUDA_TRY(launch_pdl(k_check, dim3(nb), dim3(256), 0, s.stream, A, nt, force ? 1 : 0));
    MDX_CUDA_TRY(launch_pdl(k_wrap_bin, dim3(nb), dim3(256), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_scan_cells, dim3(1), dim3(kScanThreads), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_scatter, dim3(nb), dim3(256), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_rank, dim3((ncell * 32 + 255) / 256), dim3(256), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_gather, dim3(nb), dim3(256), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_copyback, dim3(nb), dim3(256), 0, s.stream, A, nt));
    // molecule maps of the fixes that keep atom indices
    if (FixRigid *r = s.rigidFix()) {
        if (int e = rigid_update_maps(s, *r, true)) return e;
    }
    if (gr.cap == 0) {
        // first build: size the per-atom capacity from a counting sweep
        MDX_CUDA_TRY(cudaMemsetAsync(&s.d_status.p->max_neighbors, 0, sizeof(uint32_t), s.stream));
        launch_count(s, g, cutsq);
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
    cudaStream_t bs = s.stream;
    if (bstream) {
        MDX_CUDA_TRY(cudaEventRecord(s.ev_sorted, s.stream));
        MDX_CUDA_TRY(cudaStreamWaitEvent(bstream, s.ev_sorted, 0));
        bs = bstream;
    }
    launch_build(s, g, cutsq, bs);
    if (FixE3B *e3 = s.e3bFix()) {
        if (int e = e3b_build_list(s, *e3, true, bs)) return e;
    }
    MDX_CUDA_TRY(launch_pdl(k_finish, dim3(1), dim3(1024), 0, bs, A, (const GridArgs *)nullptr));
    if (bs != s.stream) MDX_CUDA_TRY(cudaEventRecord(s.ev_join[2], bs));
    gr.built = true;
    return 0;
}

// The molecule form's rebuild group: the same skin check, then the sort by
// molecule, then (on bstream when given, beside the step's first half) the
// molecule-pair list and the E3B molecule list cut from it.
static int nlist_rebuild_mf(State &s, bool force, cudaStream_t bstream) {
    const GridArgs A = grid_args(s);
    const GridArgs Am = mol_scan_args(s);
    const MolGridArgs M = mol_grid_args(s);
    const GridArgs *nt = nullptr;
    const MolGridArgs *mnt = nullptr;
    const int nb_atoms = (s.gpd.n + 255) / 256;
    const int nb_mol = (M.nmol + 255) / 256;
    MDX_CUDA_TRY(launch_pdl(k_check, dim3(nb_atoms), dim3(256), 0, s.stream, A, nt, force ? 1 : 0));
    MDX_CUDA_TRY(launch_pdl(k_mf_wrap_bin, dim3(nb_mol), dim3(256), 0, s.stream, M, mnt));
    MDX_CUDA_TRY(launch_pdl(k_scan_cells, dim3(1), dim3(kScanThreads), 0, s.stream, Am, nt));
    MDX_CUDA_TRY(launch_pdl(k_mf_scatter, dim3(nb_mol), dim3(256), 0, s.stream, M, mnt));
    MDX_CUDA_TRY(launch_pdl(k_mf_rank, dim3((M.ncell * 32 + 255) / 256), dim3(256), 0, s.stream, M, mnt));
    MDX_CUDA_TRY(launch_pdl(k_mf_gather, dim3((4 * M.nmol + 255) / 256), dim3(256), 0, s.stream, M, mnt));
    MDX_CUDA_TRY(launch_pdl(k_mf_copyback, dim3((4 * M.nmol + 255) / 256), dim3(256), 0, s.stream, M, mnt));
    cudaStream_t bs = s.stream;
    if (bstream) {
        MDX_CUDA_TRY(cudaEventRecord(s.ev_sorted, s.stream));
        MDX_CUDA_TRY(cudaStreamWaitEvent(bstream, s.ev_sorted, 0));
        bs = bstream;
    }
    MDX_CUDA_TRY(launch_pdl(k_mf_build, dim3(M.nmol), dim3(kMfBuildThreads), 0, bs, M, mnt));
    if (FixE3B *e3 = s.e3bFix()) {
        if (int e = e3b_build_list_mf(s, *e3, bs)) return e;
    }
    MDX_CUDA_TRY(launch_pdl(k_finish, dim3(1), dim3(1024), 0, bs, Am, nt));
    if (bs != s.stream) MDX_CUDA_TRY(cudaEventRecord(s.ev_join[2], bs));
    s.grid.built = true;
    return 0;
}

// The per-site list (the reference's GridGPU list) of the current positions
// built into the sort's alternate buffers only: the molecule form's primary
// streams, idToIdx, molecule maps and skin-check positions are untouched.
// The list's atom indices refer to that sorted copy (ids_alt holds its ids).
int nlist_build_atoms_view(State &s) {
    GridGPU &gr = s.grid;
    const int n = s.gpd.n;
    const CellGrid g = make_grid(s);
    const float cutsq = gr.cut * gr.cut;
    GridArgs A = grid_args(s);
    A.view = 1;
    const int nb = (n + 255) / 256;
    const int ncell = gr.ns.x * gr.ns.y * gr.ns.z;
    const GridArgs *nt = nullptr;
    MDX_CUDA_TRY(launch_pdl(k_check, dim3(nb), dim3(256), 0, s.stream, A, nt, 1));
    MDX_CUDA_TRY(launch_pdl(k_wrap_bin, dim3(nb), dim3(256), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_scan_cells, dim3(1), dim3(kScanThreads), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_scatter, dim3(nb), dim3(256), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_rank, dim3((ncell * 32 + 255) / 256), dim3(256), 0, s.stream, A, nt));
    MDX_CUDA_TRY(launch_pdl(k_gather, dim3(nb), dim3(256), 0, s.stream, A, nt));
    if (gr.cap == 0) {
        MDX_CUDA_TRY(cudaMemsetAsync(&s.d_status.p->max_neighbors, 0, sizeof(uint32_t), s.stream));
        launch_count(s, g, cutsq);
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
    launch_build(s, g, cutsq, s.stream);
    MDX_CUDA_TRY(launch_pdl(k_finish, dim3(1), dim3(1024), 0, s.stream, A, nt));
    return 0;
}

// Molecule form set-up (see MolForm): decides whether the system allows it
// and sizes its grid and list.  pairForm 1 keeps the per-site form; 2 makes
// an unsuitable system an error; 0 takes the molecule form when it can.
int molform_init(State &s) {
    MolForm &mf = s.mf;
    mf.on = false;
    if (s.pairForm == 1) return 0;
    auto refuse = [&](const char *why) -> int {
        if (s.pairForm != 2) return 0;
        set_error(MDX_ERR_UNSUPPORTED, "pairForm 2 (molecule form) not possible: %s", why);
        return MDX_ERR_UNSUPPORTED;
    };
    FixRigid *r = s.rigidFix();
    FixPair *pf = s.pairFix();
    if (!r || !r->foursite) return refuse("needs FixRigid with four-site molecules");
    if (!pf) return refuse("needs a pair fix");
    if (pf->lj_kind != 1 && pf->lj_kind != 2) return refuse("the molecule form evaluates LJ/cut or WCA");
    if (s.dsfFix()) return refuse("the molecule form evaluates Ewald real-space charges");
    if (has_free_atoms(s)) return refuse("every atom must belong to a rigid molecule");
    if (FixE3B *e3 = s.e3bFix())
        if (!e3->side_ok) return refuse("FixE3B's molecules must be FixRigid's, in the same order");
    const int nmol = (int)r->mol_ids.size();
    if (nmol == 0) return refuse("no molecules");
    auto site = [&](const int4 &m, int k) { return k == 0 ? m.x : (k == 1 ? m.y : (k == 2 ? m.z : m.w)); };
    // every molecule alike: site types and charges (as stored, FP32)
    const int4 m0 = r->mol_ids[0];
    for (int k = 0; k < 4; k++) {
        mf.type[k] = s.atoms[site(m0, k)].type;
        mf.q[k] = (float)s.atoms[site(m0, k)].q;
    }
    for (const int4 &m : r->mol_ids)
        for (int k = 0; k < 4; k++) {
            const HostAtom &a = s.atoms[site(m, k)];
            if (a.type != mf.type[k] || (float)a.q != mf.q[k]) return refuse("molecules differ in site types or charges");
        }
    // exclusions only inside a molecule, by the same depth in every molecule
    const GridGPU &gr = s.grid;
    std::vector<int> site_of(s.atoms.size(), -1), mol_of(s.atoms.size(), -1);
    for (int mi = 0; mi < nmol; mi++)
        for (int k = 0; k < 4; k++) {
            site_of[site(r->mol_ids[mi], k)] = k;
            mol_of[site(r->mol_ids[mi], k)] = mi;
        }
    for (int k = 0; k < 16; k++) mf.depth[k] = 0;
    bool first = true;
    for (int mi = 0; mi < nmol; mi++) {
        int dep[16] = {0};
        for (int k = 0; k < 4; k++) {
            const int id = site(r->mol_ids[mi], k);
            if (!gr.have_excl) break;
            for (int e = gr.h_excl_start[id]; e < gr.h_excl_start[id + 1]; e++) {
                const int o = (int)(gr.h_excl_ids[e] & kExclMask);
                if (mol_of[o] != mi) return refuse("an exclusion joins two molecules");
                dep[4 * k + site_of[o]] = (int)(gr.h_excl_ids[e] >> 30);
            }
        }
        if (first) {
            for (int k = 0; k < 16; k++) mf.depth[k] = dep[k];
            first = false;
        } else {
            for (int k = 0; k < 16; k++)
                if (dep[k] != mf.depth[k]) return refuse("molecules differ in their exclusions");
        }
    }
    // site 0 to any other site: the rigid geometry (+ a margin for the
    // FP32 positions SETTLE leaves)
    const double dmax = std::max(r->rc.r_OH, r->rc.r_OM) + 1e-3;
    const double pair_cut = (double)s.maxRCut();
    const double cut = pair_cut + s.padding + 2.0 * dmax;
    const double Lmin = std::min(s.box.Ld.x, std::min(s.box.Ld.y, s.box.Ld.z));
    if (2.0 * cut >= Lmin) return refuse("the molecule list radius must stay below half the box");
    // a site pair within the pair cutoff lies within pair_cut + 4 dmax under
    // the site-0 image shift, which must be the unique image within L/2
    if (2.0 * (pair_cut + 4.0 * dmax) >= Lmin) return refuse("box too small for one image shift per molecule pair");
    if (2.0 * dmax >= (double)gr.cut) return refuse("a molecule must lie within the neighbour cutoff");
    // cells >= cut / m with at least 2m + 1 per side; the finest such grid
    // that keeps a mean of two molecules per cell
    int m = 3;
    int3 ns{0, 0, 0};
    for (;; m--) {
        if (m == 0) return refuse("box too small for the molecule grid");
        const double w = cut / m * (1.0 + 1e-5);
        ns = make_int3((int)(s.box.Ld.x / w), (int)(s.box.Ld.y / w), (int)(s.box.Ld.z / w));
        if (ns.x < 2 * m + 1 || ns.y < 2 * m + 1 || ns.z < 2 * m + 1) continue;
        if (m == 1 || (double)nmol >= 2.0 * ns.x * ns.y * ns.z) break;
    }
    mf.m = m;
    mf.ns = ns;
    mf.nmol = nmol;
    mf.dmax = (float)dmax;
    mf.cut = (float)cut;
    mf.far = (float)(pair_cut + 2.0 * dmax);
    mf.team = 32;  // one warp per molecule in the pair kernel: each row is contiguous
    const double vol = s.box.Ld.x * s.box.Ld.y * s.box.Ld.z;
    const double nbar = nmol / vol * 4.18879 * cut * cut * cut;
    mf.cap = ((int)(1.5 * nbar + 64) + mf.team - 1) / mf.team * mf.team;
    const int ncell = ns.x * ns.y * ns.z;
    if (int e = mf.cell_start.alloc(ncell + 1)) return e;
    if (int e = mf.cell_count.alloc(ncell)) return e;
    if (int e = mf.cell_fill.alloc(ncell)) return e;
    MDX_CUDA_TRY(cudaMemsetAsync(mf.cell_count.p, 0, ncell * sizeof(uint32_t), s.stream));
    if (int e = mf.cell_of.alloc(nmol)) return e;
    if (int e = mf.perm_tmp.alloc(nmol)) return e;
    if (int e = mf.perm.alloc(nmol)) return e;
    if (int e = mf.counts.alloc(nmol)) return e;
    const int G = 32 / mf.team;
    const size_t groups = (size_t)(nmol + G - 1) / G;
    if (int e = mf.list.alloc(groups * (size_t)mf.cap * G)) return e;
    // the sort reads the molecule maps first: after an upload every atom sits
    // at index == id, so the maps are the molecules' ids
    MDX_CUDA_TRY(cudaMemcpy(r->d_mol_idx.p, r->mol_ids.data(), nmol * sizeof(int4), cudaMemcpyHostToDevice));
    // E3B works by slot in this form (its molecules are FixRigid's): its map
    // is the identity slot map, slot k at sites 4k .. 4k+3
    if (FixE3B *e3 = s.e3bFix()) {
        std::vector<int4> ident(nmol);
        for (int k = 0; k < nmol; k++) ident[k] = make_int4(4 * k, 4 * k + 1, 4 * k + 2, 4 * k + 3);
        MDX_CUDA_TRY(cudaMemcpy(e3->d_mol_idx.p, ident.data(), nmol * sizeof(int4), cudaMemcpyHostToDevice));
    }
    mf.on = true;
    return 0;
}

// the box changed size (a barostat): the cell grids keep their stencil
// widths m and take as many cells per side as the new box holds at that
// width (cells never narrower than the list radius / m); the caller forces a
// rebuild.  The minimum-image and stencil conditions of nlist_init and
// molform_init are checked again.
// a box that grew without bound (a barostat run away) ends the run with an
// error instead of an overflowing grid
static int grid_cells_fit(int3 ns) {
    const long long n = (long long)ns.x * ns.y * ns.z;
    if (n > (1LL << 27)) {
        set_error(MDX_ERR_UNSUPPORTED, "the box grew to %d x %d x %d neighbour cells (more than 2^27)", ns.x, ns.y,
                  ns.z);
        return MDX_ERR_UNSUPPORTED;
    }
    return 0;
}

int nlist_box_changed(State &s) {
    GridGPU &gr = s.grid;
    const double Lmin = std::min(s.box.Ld.x, std::min(s.box.Ld.y, s.box.Ld.z));
    if (2.0 * (double)gr.cut >= Lmin) {
        set_error(MDX_ERR_UNSUPPORTED, "the box shrank below twice the neighbour cutoff %g", (double)gr.cut);
        return MDX_ERR_UNSUPPORTED;
    }
    {
        const double w = (double)gr.cut / gr.m * (1.0 + 1e-5);
        const int3 ns = make_int3((int)(s.box.Ld.x / w), (int)(s.box.Ld.y / w), (int)(s.box.Ld.z / w));
        const int need = std::max(3, 2 * gr.m);
        if (ns.x < need || ns.y < need || ns.z < need) {
            set_error(MDX_ERR_UNSUPPORTED, "the box shrank below the neighbour grid's %d cells per side", need);
            return MDX_ERR_UNSUPPORTED;
        }
        if (int e = grid_cells_fit(ns)) return e;
        const int ncell = ns.x * ns.y * ns.z;
        if (int e = gr.cell_start.alloc(ncell + 1)) return e;
        if (int e = gr.cell_count.alloc(ncell)) return e;
        if (int e = gr.cell_fill.alloc(ncell)) return e;
        MDX_CUDA_TRY(cudaMemsetAsync(gr.cell_count.p, 0, ncell * sizeof(uint32_t), s.stream));
        gr.ns = ns;
    }
    if (s.mf.on) {
        MolForm &mf = s.mf;
        if (2.0 * (double)mf.cut >= Lmin) {
            set_error(MDX_ERR_UNSUPPORTED, "the box shrank below twice the molecule list radius %g", (double)mf.cut);
            return MDX_ERR_UNSUPPORTED;
        }
        const double w = (double)mf.cut / mf.m * (1.0 + 1e-5);
        const int3 ns = make_int3((int)(s.box.Ld.x / w), (int)(s.box.Ld.y / w), (int)(s.box.Ld.z / w));
        if (ns.x < 2 * mf.m + 1 || ns.y < 2 * mf.m + 1 || ns.z < 2 * mf.m + 1) {
            set_error(MDX_ERR_UNSUPPORTED, "the box shrank below the molecule grid's %d cells per side", 2 * mf.m + 1);
            return MDX_ERR_UNSUPPORTED;
        }
        if (int e = grid_cells_fit(ns)) return e;
        const int ncell = ns.x * ns.y * ns.z;
        if (int e = mf.cell_start.alloc(ncell + 1)) return e;
        if (int e = mf.cell_count.alloc(ncell)) return e;
        if (int e = mf.cell_fill.alloc(ncell)) return e;
        MDX_CUDA_TRY(cudaMemsetAsync(mf.cell_count.p, 0, ncell * sizeof(uint32_t), s.stream));
        mf.ns = ns;
    }
    return 0;
}

// batched replicas: the same group, one launch per kernel for all replicas
// of a form (blockIdx.y = replica of that form); every kernel returns at once
// for a replica whose skin check did not fire.  Tables are built at prepare,
// before any capture.
int batch_nlist_tables(Batch &b) {
    const int R = (int)b.reps.size();
    std::vector<GridArgs> hg(R);
    for (int r = 0; r < R; r++) hg[r] = grid_args(*b.reps[r]);
    if (int e = b.tab_grid.alloc(R * sizeof(GridArgs))) return e;
    MDX_CUDA_TRY(cudaMemcpy(b.tab_grid.p, hg.data(), R * sizeof(GridArgs), cudaMemcpyHostToDevice));
    const int P = (int)b.ps.size();
    if (P) {
        std::vector<GridArgs> hp(P);
        std::vector<BuildArgs> hb(P);
        for (int q = 0; q < P; q++) {
            State &s = *b.reps[b.ps[q]];
            hp[q] = hg[b.ps[q]];
            hb[q] = build_args(s, make_grid(s), s.grid.cut * s.grid.cut);
            // one list-build kernel serves the batch: its exclusion and
            // front/back split forms are compile-time, so they must agree
            if ((hb[q].use_excl != 0) != (hb[0].use_excl != 0) ||
                (hb[q].ljmask != nullptr) != (hb[0].ljmask != nullptr)) {
                set_error(MDX_ERR_UNSUPPORTED,
                          "batched replicas must agree on exclusions and on the interacting-pair split (replica %d)",
                          b.ps[q]);
                return MDX_ERR_UNSUPPORTED;
            }
        }
        if (int e = b.tab_grid_ps.alloc(P * sizeof(GridArgs))) return e;
        if (int e = b.tab_build.alloc(P * sizeof(BuildArgs))) return e;
        MDX_CUDA_TRY(cudaMemcpy(b.tab_grid_ps.p, hp.data(), P * sizeof(GridArgs), cudaMemcpyHostToDevice));
        MDX_CUDA_TRY(cudaMemcpy(b.tab_build.p, hb.data(), P * sizeof(BuildArgs), cudaMemcpyHostToDevice));
    }
    const int Q = (int)b.mfi.size();
    if (Q) {
        std::vector<MolGridArgs> hm(Q);
        std::vector<GridArgs> hs(Q);
        b.max_mcell = 0;
        for (int q = 0; q < Q; q++) {
            State &s = *b.reps[b.mfi[q]];
            hm[q] = mol_grid_args(s);
            hs[q] = mol_scan_args(s);
            b.max_mcell = std::max(b.max_mcell, hs[q].ncell);
        }
        if (int e = b.tab_molgrid.alloc(Q * sizeof(MolGridArgs))) return e;
        if (int e = b.tab_molscan.alloc(Q * sizeof(GridArgs))) return e;
        MDX_CUDA_TRY(cudaMemcpy(b.tab_molgrid.p, hm.data(), Q * sizeof(MolGridArgs), cudaMemcpyHostToDevice));
        MDX_CUDA_TRY(cudaMemcpy(b.tab_molscan.p, hs.data(), Q * sizeof(GridArgs), cudaMemcpyHostToDevice));
    }
    return 0;
}

// the per-site replicas' sort and list build (nlist_rebuild's kernels)
static void batch_rebuild_sites(Batch &b, cudaStream_t st) {
    const int P = (int)b.ps.size();
    const GridArgs *tg = reinterpret_cast<const GridArgs *>(b.tab_grid_ps.p);
    const BuildArgs *tb = reinterpret_cast<const BuildArgs *>(b.tab_build.p);
    State &s0 = *b.reps[b.ps[0]];
    GridArgs A = grid_args(s0);  // sizing only: the kernels read tab
    A.n = b.max_n_ps;
    A.ncell = b.max_cell_ps;
    BuildArgs B = build_args(s0, make_grid(s0), s0.grid.cut * s0.grid.cut);
    B.ncell = b.max_cell_ps;
    const dim3 nb((b.max_n_ps + 255) / 256, P);
    k_wrap_bin<<<nb, 256, 0, st>>>(A, tg);
    k_scan_cells<<<dim3(1, P), kScanThreads, 0, st>>>(A, tg);
    k_scatter<<<nb, 256, 0, st>>>(A, tg);
    k_rank<<<dim3((b.max_cell_ps * 32 + 255) / 256, P), 256, 0, st>>>(A, tg);
    k_gather<<<nb, 256, 0, st>>>(A, tg);
    k_copyback<<<nb, 256, 0, st>>>(A, tg);
    int hg = 2;
    for (int r : b.ps) hg = std::max(hg, b.reps[r]->grid.home_group);
    launch_build_any<false>(s0.grid.team, hg, build_grid(b.max_cell_ps, P), st, B, tb);
    g_launches += 6;
}

// the molecule-form replicas' sort by molecule and molecule-pair list
// (nlist_rebuild_mf's kernels)
static void batch_rebuild_mols(Batch &b, cudaStream_t st) {
    const int Q = (int)b.mfi.size();
    const GridArgs *ts = reinterpret_cast<const GridArgs *>(b.tab_molscan.p);
    const MolGridArgs *tm = reinterpret_cast<const MolGridArgs *>(b.tab_molgrid.p);
    State &s0 = *b.reps[b.mfi[0]];
    GridArgs Am = mol_scan_args(s0);  // sizing only: the kernels read the tables
    Am.ncell = b.max_mcell;
    MolGridArgs M = mol_grid_args(s0);
    M.nmol = b.max_mol_mf;
    M.ncell = b.max_mcell;
    const int nb_mol = (b.max_mol_mf + 255) / 256, nb_site = (4 * b.max_mol_mf + 255) / 256;
    k_mf_wrap_bin<<<dim3(nb_mol, Q), 256, 0, st>>>(M, tm);
    k_scan_cells<<<dim3(1, Q), kScanThreads, 0, st>>>(Am, ts);
    k_mf_scatter<<<dim3(nb_mol, Q), 256, 0, st>>>(M, tm);
    k_mf_rank<<<dim3((b.max_mcell * 32 + 255) / 256, Q), 256, 0, st>>>(M, tm);
    k_mf_gather<<<dim3(nb_site, Q), 256, 0, st>>>(M, tm);
    k_mf_copyback<<<dim3(nb_site, Q), 256, 0, st>>>(M, tm);
    k_mf_build<<<dim3(b.max_mol_mf, Q), kMfBuildThreads, 0, st>>>(M, tm);
    g_launches += 7;
}

int batch_nlist_rebuild(Batch &b) {
    const int R = (int)b.reps.size();
    if (!b.tab_grid.p) {
        set_error(MDX_ERR_STATE, "batch tables not built (prepare the batch)");
        return MDX_ERR_STATE;
    }
    const GridArgs *tg = reinterpret_cast<const GridArgs *>(b.tab_grid.p);
    State &s0 = *b.reps[0];
    GridArgs A = grid_args(s0);  // sizing only
    A.n = b.max_n;
    cudaStream_t st = b.stream;
    k_check<<<dim3((b.max_n + 255) / 256, R), 256, 0, st>>>(A, tg, 0);
    MDX_LAUNCHED();
    if (!b.ps.empty()) batch_rebuild_sites(b, st);
    if (!b.mfi.empty()) batch_rebuild_mols(b, st);
    // the per-site replicas' molecule maps (the molecule form's copyback
    // rewrote its own)
    if (!b.ps.empty())
        if (int e = batch_rigid_maps(b)) return e;
    if (s0.e3bFix())
        if (int e = batch_e3b_list(b)) return e;
    if (!b.ps.empty()) {
        GridArgs Ap = A;
        Ap.n = b.max_n_ps;
        k_finish<<<dim3(1, (unsigned)b.ps.size()), 1024, 0, st>>>(Ap, reinterpret_cast<const GridArgs *>(b.tab_grid_ps.p));
        MDX_LAUNCHED();
    }
    if (!b.mfi.empty()) {
        GridArgs Am = mol_scan_args(*b.reps[b.mfi[0]]);
        Am.ncell = b.max_mcell;
        k_finish<<<dim3(1, (unsigned)b.mfi.size()), 1024, 0, st>>>(Am, reinterpret_cast<const GridArgs *>(b.tab_molscan.p));
        MDX_LAUNCHED();
    }
    MDX_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mdx
