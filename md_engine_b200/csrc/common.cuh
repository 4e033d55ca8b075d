// Shared device/host helpers for the B200 force hot path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "mdx.h"

namespace mdx {

// Exclusion tag bits of a neighbour entry (bits 30-31 = depth 1..3), the
// same packing as the reference's EXCL_MASK (globalDefs.h:40).
constexpr uint32_t kExclMask = ~(3u << 30);
// Inverse-mass sentinel for massless sites and its threshold
// (globalDefs.h:37-38: INVMASSLESS 1e30, INVMASSBOOL 1e18).
constexpr float kInvMassless = 1.0e30f;
constexpr float kInvMassBool = 1.0e18f;

// Device status word bits (written with atomicOr, read by the host between
// runs; nothing here traps or waits on the device).
enum StatusBits : uint32_t {
    kStatusNlistOverflow = 1u << 0,   // an atom had more neighbours than the list capacity
    kStatusMolOverflow   = 1u << 1,   // molecule (E3B) list overflow
    kStatusNanForce      = 1u << 2,   // non-finite force seen
    kStatusSettleFail    = 1u << 3,   // SETTLE cos^2 <= 0 (degenerate triangle)
    kStatusConstraint    = 1u << 4,   // bond length drift beyond tolerance
    kStatusBoxTooSmall   = 1u << 5,   // cut + skin >= half box
    kStatusP3MMiss       = 1u << 6,   // charge assignment stencil out of grid
};

struct DeviceStatus {
    uint32_t bits;
    uint32_t max_neighbors;      // largest per-atom count seen at the last build
    uint32_t max_mol_neighbors;  // largest per-molecule count seen
    uint32_t rebuild;            // 1 when the current step rebuilds the list
    uint64_t n_builds;           // number of list builds executed on device
    int64_t turn;                // device-side turn counter
};

// Box, the analogue of BoundsGPU (BoundsGPU.h) for a fully periodic
// orthorhombic box.  Float and double copies so that the SETTLE kernels can
// take minimum images in FP64 (BoundsGPU.h:102-108).
struct Box {
    float3 lo, L, invL;
    double3 lod, Ld, invLd;
};

__host__ __device__ inline float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__host__ __device__ inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline void operator+=(float3 &a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
__host__ __device__ inline void operator-=(float3 &a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
__host__ __device__ inline float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__host__ __device__ inline double3 d3(float4 a) { return make_double3(a.x, a.y, a.z); }
__host__ __device__ inline double3 operator+(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline double3 operator-(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline double3 operator*(double3 a, double s) { return make_double3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline double3 operator*(double s, double3 a) { return make_double3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline void operator+=(double3 &a, double3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
__host__ __device__ inline void operator-=(double3 &a, double3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
__host__ __device__ inline void operator/=(double3 &a, double s) { a.x /= s; a.y /= s; a.z /= s; }
__host__ __device__ inline double dotd(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline double lend(double3 a) { return sqrt(dotd(a, a)); }
__host__ __device__ inline double3 crossd(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// programmatic dependent launch (sm_90+): pdl_trigger lets the next kernel of
// the stream be scheduled now (without it, once this block exits); pdl_wait
// blocks until the previous kernel of the stream has completed and its writes
// are visible.  Both are no-ops for a kernel launched without the
// programmatic-serialization attribute.  Triggers sit late in a kernel: a
// dependent scheduled early holds SM slots idle that kernels of other streams
// (the pair kernel beside the P3M chain) would use.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Single-instruction approximations (PTX ISA rsqrt/ex2/rcp .approx.ftz): the
// hot loops' arguments are normal floats, so flushing denormals changes no
// result while it drops the range handling of the non-ftz forms.
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ex2_ftz(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rcp_ftz(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// exp(-x^2) as 2^(-x^2 log2 e)
__device__ __forceinline__ float exp_neg_sq(float x) { return ex2_ftz(-(x * x) * 1.4426950408889634f); }

// nearest integer of |x| < 2^22 as rintf gives it (ties to even), by two
// round-to-nearest additions of 1.5 * 2^23: the sum's unit in the last place
// is 1, so the addition itself rounds x to an integer.  Two FP32 adds on the
// FMA pipe in place of a rounding instruction; __fadd_rn keeps the compiler
// from folding the pair.
__device__ __forceinline__ float rint_small(float x) {
    return __fadd_rn(__fadd_rn(x, 12582912.0f), -12582912.0f);
}

// minimum image (BoundsGPU::minImage, BoundsGPU.h:91-108); the scaled
// separations are a few box lengths at most
__device__ inline float3 min_image(const Box &b, float3 v) {
    v.x -= b.L.x * rint_small(v.x * b.invL.x);
    v.y -= b.L.y * rint_small(v.y * b.invL.y);
    v.z -= b.L.z * rint_small(v.z * b.invL.z);
    return v;
}
__device__ inline double3 min_image(const Box &b, double3 v) {
    v.x -= b.Ld.x * rint(v.x * b.invLd.x);
    v.y -= b.Ld.y * rint(v.y * b.invLd.y);
    v.z -= b.Ld.z * rint(v.z * b.invLd.z);
    return v;
}

__device__ inline int type_of(float4 x) { return __float_as_int(x.w); }

}  // namespace mdx

#define MDX_CUDA_TRY(expr)                                                     \
    do {                                                                       \
        cudaError_t _e = (expr);                                               \
        if (_e != cudaSuccess) {                                               \
            ::mdx::set_error(MDX_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, \
                             #expr, cudaGetErrorString(_e));                   \
            return MDX_ERR_CUDA;                                               \
        }                                                                      \
    } while (0)

namespace mdx {
void set_error(int code, const char *fmt, ...);
}
