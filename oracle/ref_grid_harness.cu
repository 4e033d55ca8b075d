// Harness around the REFERENCE's own neighbour-grid kernels -- TEST
// INFRASTRUCTURE ONLY.
//
// oracle/ref.mk compiles the reference's src/GridGPU.cu where it lies, for
// sm_100a with the reference's nvcc flags, against the stand-in headers of
// oracle/ref_shim_grid/ (State, Fix, Bond, Mod and the Boost.Python names
// GridGPU.cu mentions; the split include path makes them shadow the
// reference's own, which pull in Boost and Python).  Every kernel launched
// here is the reference's: setBuildFlag, periodicWrap, countNumInGridCells,
// sortPerAtomArrays, countNumNeighbors, computeMaxMemSizePerWarp,
// setCumulativeSumPerBlock, assignNeighbors.  The only code written here is
// the C entry points that allocate plain device arrays in place of GPUData,
// launch those kernels in the order of GridGPU::periodicBoundaryConditions
// (GridGPU.cu:824-1103, a forced build, one atom per ring polymer, no
// exclusions) with the grid geometry of GridGPU::setBounds (:46-67), and
// read the padded per-block list back by the addressing of
// GridGPU::getNeighborList (:1520-1600).
#include "GridGPU.cu"
#include "GPUArrayDevice.cpp"  // the device-array base class GridGPU.cu's arrays derive from

#include <algorithm>
#include <cstring>

namespace {

template <class T>
T *dalloc(size_t n) {
    T *p = nullptr;
    cudaMalloc(&p, (n ? n : 1) * sizeof(T));
    return p;
}

}  // namespace

extern "C" {

// setBuildFlag (GridGPU.cu:755-774) on positions a and b (n x 4 floats):
// 1 if any atom moved more than padding / 2 (minimum image), else 0
int ref_grid_skin_flag(int n, const float *xa4, const float *xb4, const float lo[3], const float L[3],
                       float padding) {
    real4 *a = dalloc<real4>(n), *b = dalloc<real4>(n);
    int *flag = dalloc<int>(1);
    cudaMemcpy(a, xa4, n * sizeof(real4), cudaMemcpyHostToDevice);
    cudaMemcpy(b, xb4, n * sizeof(real4), cudaMemcpyHostToDevice);
    cudaMemset(flag, 0, sizeof(int));
    BoundsGPU bounds(make_real3(lo[0], lo[1], lo[2]), make_real3(L[0], L[1], L[2]), make_real3(1, 1, 1));
    setBuildFlag<<<NBLOCK(n), PERBLOCK, PERBLOCK * sizeof(short)>>>(a, b, n, bounds, padding * padding, flag, 32);
    int h = -1;
    cudaError_t e = cudaMemcpy(&h, flag, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(a);
    cudaFree(b);
    cudaFree(flag);
    return e == cudaSuccess ? h : -(int)e - 10;
}

// A forced GridGPU build of n atoms (positions xs4, ids 0..n-1) in the box
// (lo, L), cells of at least min_dim, cutoff neigh_cut (rCut + padding),
// nThreadPerBlock ntpb, nThreadPerAtom ntpa.  Out: counts[id] and, per atom
// id, its neighbours' ids in list order at nbr[id * maxn ..]; wrapped[id]
// the wrapped position the list was built on.  Returns 0, or a CUDA error
// code, or -1 if an atom has more than maxn neighbours.
int ref_grid_build(int n, const float *xs4, const float lo[3], const float L[3], const float min_dim[3],
                   float neigh_cut, int ntpb, int ntpa, int maxn, int *counts, uint32_t *nbr, float *wrapped) {
    const int warpSize = 32;
    // GridGPU::setBounds: whole cells of at least min_dim (truncation), then
    // the EPSILON widening of periodicBoundaryConditions
    const double tr[3] = {L[0], L[1], L[2]};
    int3 ns;
    ns.x = (int)(tr[0] / (double)min_dim[0]);
    ns.y = (int)(tr[1] / (double)min_dim[1]);
    ns.z = (int)(tr[2] / (double)min_dim[2]);
    real3 ds = make_real3((real)(tr[0] / ns.x), (real)(tr[1] / ns.y), (real)(tr[2] / ns.z));
    real3 os = make_real3(lo[0], lo[1], lo[2]);
    ds += make_real3(EPSILON, EPSILON, EPSILON);
    os -= make_real3(EPSILON, EPSILON, EPSILON);
    BoundsGPU bounds(make_real3(lo[0], lo[1], lo[2]), make_real3(L[0], L[1], L[2]), make_real3(1, 1, 1));
    const int ncell = ns.x * ns.y * ns.z;

    std::vector<uint> hids(n);
    for (int i = 0; i < n; i++) hids[i] = (uint)i;
    real4 *xa = dalloc<real4>(n), *xb = dalloc<real4>(n), *va = dalloc<real4>(n), *vb = dalloc<real4>(n);
    real4 *fa = dalloc<real4>(n), *fb = dalloc<real4>(n);
    uint *ia = dalloc<uint>(n), *ib = dalloc<uint>(n);
    real *qa = dalloc<real>(n), *qb = dalloc<real>(n);
    int *idToIdx = dalloc<int>(n);
    uint32_t *perCell = dalloc<uint32_t>(ncell + 1);
    uint16_t *perAtom = dalloc<uint16_t>(n + 1);
    const int nblocks = NBLOCKTEAM(n, ntpb, ntpa);
    uint32_t *perBlock = dalloc<uint32_t>(nblocks + 1);
    // computeMaxMemSizePerWarp writes nThreadPerAtom entries for every block
    // of its own grid (NBLOCKVAR(n, ntpb) blocks), up to ntpa - 1 past the
    // NBLOCKTEAM(n, ntpb, ntpa) entries the reference allocates
    const int nmax = std::max(nblocks, NBLOCKVAR(n, ntpb) * ntpa);
    uint16_t *maxInBlock = dalloc<uint16_t>(nmax);
    cudaMemset(maxInBlock, 0, nmax * sizeof(uint16_t));
    cudaMemcpy(xa, xs4, n * sizeof(real4), cudaMemcpyHostToDevice);
    cudaMemcpy(ia, hids.data(), n * sizeof(uint), cudaMemcpyHostToDevice);
    cudaMemset(va, 0, n * sizeof(real4));
    cudaMemset(fa, 0, n * sizeof(real4));

    periodicWrap<<<NBLOCK(n), PERBLOCK>>>(xa, n, bounds.unskewed());
    cudaMemset(perCell, 0, (ncell + 1) * sizeof(uint32_t));
    cudaMemset(perAtom, 0, (n + 1) * sizeof(uint16_t));
    countNumInGridCells<<<NBLOCK(n), PERBLOCK>>>(xa, n, perCell, perAtom, os, ds, ns);
    std::vector<uint32_t> hc(ncell + 1);
    cudaMemcpy(hc.data(), perCell, (ncell + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cumulativeSum(hc.data(), ncell + 1);
    cudaMemcpy(perCell, hc.data(), (ncell + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice);
    sortPerAtomArrays<<<NBLOCK(n), PERBLOCK>>>(xa, xa, xb, va, vb, fa, fb, ia, ib, qa, qb, idToIdx, false, perCell,
                                               perAtom, n, os, ds, ns, 1);
    const real3 trace = bounds.unskewed().trace();
    cudaMemset(perAtom, 0, (n + 1) * sizeof(uint16_t));
    const real cut2 = neigh_cut * neigh_cut;
    if (ntpa == 1)
        countNumNeighbors<0><<<nblocks, ntpb>>>(xb, n, perAtom, perCell, os, ds, ns, bounds.periodic, trace, cut2,
                                                ntpa);
    else
        countNumNeighbors<1><<<nblocks, ntpb, ntpb * sizeof(uint16_t)>>>(xb, n, perAtom, perCell, os, ds, ns,
                                                                       bounds.periodic, trace, cut2, ntpa);
    computeMaxMemSizePerWarp<<<NBLOCKVAR(n, ntpb), ntpb, ntpb * sizeof(uint16_t)>>>(n, perAtom, maxInBlock, warpSize,
                                                                                  ntpa);
    setCumulativeSumPerBlock<<<NBLOCKVAR(nblocks + 1, ntpb), ntpb>>>(nblocks, perBlock, maxInBlock);
    uint32_t cumul = 0;
    cudaMemcpy(&cumul, perBlock + nblocks, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    size_t total = (size_t)cumul * (ntpb / warpSize);
    if (total == 0) total = 1;
    // 1.5x, as periodicBoundaryConditions sizes it
    uint *nlist = dalloc<uint>(total + total / 2 + 64);
    int *exIdx = dalloc<int>(1);
    uint *exIds = dalloc<uint>(1);
    if (ntpa == 1)
        assignNeighbors<0, false><<<nblocks, ntpb, 0>>>(xb, n, 1, ib, perCell, perBlock, os, ds, ns, bounds.periodic,
                                                       trace, cut2, nlist, warpSize, exIdx, exIds, 0, ntpa);
    else
        assignNeighbors<1, false><<<nblocks, ntpb, ntpb * sizeof(uint32_t)>>>(
            xb, n, 1, ib, perCell, perBlock, os, ds, ns, bounds.periodic, trace, cut2, nlist, warpSize, exIdx, exIds,
            0, ntpa);
    cudaError_t e = cudaDeviceSynchronize();

    // GridGPU::getNeighborList's reading of the padded per-block layout
    int rc = (int)e;
    if (e == cudaSuccess) {
        std::vector<uint16_t> hcount(n);
        std::vector<uint32_t> hblock(nblocks + 1);
        std::vector<uint> hl(total), hid(n);
        std::vector<real4> hx(n);
        cudaMemcpy(hcount.data(), perAtom, n * sizeof(uint16_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(hblock.data(), perBlock, (nblocks + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(hl.data(), nlist, total * sizeof(uint), cudaMemcpyDeviceToHost);
        cudaMemcpy(hid.data(), ib, n * sizeof(uint), cudaMemcpyDeviceToHost);
        cudaMemcpy(hx.data(), xb, n * sizeof(real4), cudaMemcpyDeviceToHost);
        const int perBlockAtoms = ntpb / ntpa;
        const int warpsPerBlock = ntpb / warpSize;
        for (int i = 0; i < n && rc == 0; i++) {
            const int c = hcount[i];
            const uint id = hid[i];
            if (c > maxn) {
                rc = -1;
                break;
            }
            counts[id] = c;
            std::memcpy(wrapped + 4 * (size_t)id, &hx[i], sizeof(real4));
            const int blk = i / perBlockAtoms;
            const uint32_t memPerWarp = hblock[blk + 1] - hblock[blk];
            const int nth = i % perBlockAtoms;
            const int atomsPerWarp = warpSize / ntpa;
            const size_t base = (size_t)warpsPerBlock * hblock[blk] + memPerWarp * (nth / atomsPerWarp) +
                                (nth % atomsPerWarp) * ntpa;
            for (int k = 0; k < c; k++)
                nbr[(size_t)id * maxn + k] = hid[hl[base + (k % ntpa) + (size_t)warpSize * (k / ntpa)]];
        }
    }
    cudaFree(xa); cudaFree(xb); cudaFree(va); cudaFree(vb); cudaFree(fa); cudaFree(fb);
    cudaFree(ia); cudaFree(ib); cudaFree(qa); cudaFree(qb); cudaFree(idToIdx);
    cudaFree(perCell); cudaFree(perAtom); cudaFree(perBlock); cudaFree(maxInBlock);
    cudaFree(nlist); cudaFree(exIdx); cudaFree(exIds);
    return rc;
}

}  // extern "C"
