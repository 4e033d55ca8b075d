// mdx_kinetic_noalloc: the FP64 sum of m v^2 (the kinetic-energy reduction
// behind mdx_kinetic) without any device allocation.
//
// Who needs it: host programs that cannot call cudaMalloc/cudaFree while they
// drive a simulation -- e.g. a host that hands all device memory out of its
// own pre-reserved pool and forbids other components from allocating, or an
// inner loop that must not pay the implicit device synchronisation that
// cudaMalloc/cudaFree can cause.  mdx_kinetic allocates its per-block partial
// sums on every call; this variant keeps them in a fixed file-scope device
// array instead, so a call allocates nothing.
//
// Limits and sharing rules:
//  * the scratch holds kNoAllocMaxBlocks = 8192 partial sums (64 KiB): at
//    256 atoms per block the state may hold at most 2,097,152 atoms; larger
//    states are rejected with MDX_ERR_ARG;
//  * every GPU that loads this library holds the 64 KiB until process exit;
//  * all calls share the one array (per device) and it keeps the contents of
//    the last call: each call writes every partial it later reads, so nothing
//    needs clearing, but calls whose kernels overlap on the GPU (different
//    streams, no ordering between them) race on the array;
//  * the first call for a state on a device looks up the array's device
//    address with cudaGetSymbolAddress (set-up, once per device), with the
//    state's own device made current for the call (the caller's current
//    device is restored afterwards); make that first call before any stream
//    capture begins.
#include <mutex>

#include "engine.hpp"

namespace mdx {

namespace {

constexpr int kNoAllocMaxBlocks = 8192;
constexpr int kNoAllocThreads = 256;
constexpr int kMaxDevices = 64;

// partial sums [0, kNoAllocMaxBlocks) and the final sum at [kNoAllocMaxBlocks]
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxBlocks + 1];

std::mutex g_noalloc_mu;
double *g_noalloc_ptr[kMaxDevices] = {nullptr};

// device address of the scratch array on device `dev`, which must be the
// current device (set-up on the first call per device; the host-side symbol
// is not a device address)
int noalloc_scratch(int dev, double **out) {
    if (dev < 0 || dev >= kMaxDevices) {
        set_error(MDX_ERR_UNSUPPORTED, "device %d beyond the %d devices this entry point tracks", dev, kMaxDevices);
        return MDX_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        MDX_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return 0;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// each block writes its partial sum of m v^2 (massless sites skipped) to scratch[blockIdx.x]
__global__ void k_mv2_noalloc(int n, const float4 *__restrict__ vs, double *__restrict__ scratch) {
    __shared__ double sh[kNoAllocThreads / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mv2 = 0.0;
    if (i < n) {
        const float4 v = vs[i];
        if (v.w < kInvMassBool) mv2 = ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z) / (double)v.w;
    }
    mv2 = warp_sum(mv2);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mv2;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (kNoAllocThreads / 32) ? sh[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) scratch[blockIdx.x] = t;
    }
}

// one block sums the partials in a fixed order into scratch[kNoAllocMaxBlocks]
__global__ void k_mv2_noalloc_final(int nblocks, double *__restrict__ scratch) {
    __shared__ double sh[kNoAllocThreads / 32];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc += scratch[b];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (kNoAllocThreads / 32) ? sh[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) scratch[kNoAllocMaxBlocks] = t;
    }
}

// the two kernels and the copy-out on the state's stream; `dev` is current
int kinetic_noalloc_on_device(State &s, int n, int nblocks, int dev, double *sum_mv2) {
    double *scratch = nullptr;
    if (int e = noalloc_scratch(dev, &scratch)) return e;
    if (nblocks > 0) {
        k_mv2_noalloc<<<nblocks, kNoAllocThreads, 0, s.stream>>>(n, s.gpd.vs.p, scratch);
        MDX_LAUNCHED();
    }
    k_mv2_noalloc_final<<<1, kNoAllocThreads, 0, s.stream>>>(nblocks, scratch);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaGetLastError());
    MDX_CUDA_TRY(cudaMemcpyAsync(sum_mv2, scratch + kNoAllocMaxBlocks, sizeof(double), cudaMemcpyDeviceToHost,
                                 s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    return 0;
}

}  // namespace

}  // namespace mdx

using namespace mdx;

extern "C" int mdx_kinetic_noalloc(mdx_state *st, double *sum_mv2) {
    if (!st || !sum_mv2) {
        set_error(MDX_ERR_ARG, "null argument");
        return MDX_ERR_ARG;
    }
    State &s = *st->s;
    if (!s.prepared || !s.uploaded) {
        set_error(MDX_ERR_STATE, "call mdx_prepare (or run) first");
        return MDX_ERR_STATE;
    }
    const int n = s.gpd.n;
    const int nblocks = (n + kNoAllocThreads - 1) / kNoAllocThreads;
    if (nblocks > kNoAllocMaxBlocks) {
        set_error(MDX_ERR_ARG, "mdx_kinetic_noalloc: %d atoms exceed its fixed scratch (at most %d atoms)", n,
                  kNoAllocMaxBlocks * kNoAllocThreads);
        return MDX_ERR_ARG;
    }
    // the state's device is current for the look-up and the launches; the
    // caller's current device is put back before returning
    int prev = 0;
    MDX_CUDA_TRY(cudaGetDevice(&prev));
    if (s.device >= 0 && s.device != prev) MDX_CUDA_TRY(cudaSetDevice(s.device));
    const int rc = kinetic_noalloc_on_device(s, n, nblocks, s.device >= 0 ? s.device : prev, sum_mv2);
    if (s.device >= 0 && s.device != prev) {
        const cudaError_t back = cudaSetDevice(prev);
        if (rc == 0 && back != cudaSuccess) {
            set_error(MDX_ERR_CUDA, "cudaSetDevice(%d): %s", prev, cudaGetErrorString(back));
            return MDX_ERR_CUDA;
        }
    }
    return rc;
}
