// Time integration: velocity Verlet (IntegratorVerlet.cu:23-61, 307-338,
// 610-627), the rigid-water hooks of FixRigid (SETTLE positions/velocities in
// FP64, M-site placement and force redistribution, FixRigid.cu:475-1132) and
// the Nose-Hoover chain of FixNoseHoover (FixNoseHoover.cu:413-604, 795-866).
//
// Fused form (default): one per-molecule kernel does NH rescale + kick + drift
// + SETTLE positions + M-site, and one does kick + M-site force
// redistribution + SETTLE velocities + the FP64 sum of m v^2; the last block
// of that kernel runs the chain update on the device, so no host round trip is
// needed per step (the reference syncs for the kinetic energy every step,
// FixNoseHoover.cu:1044-1056).  Atoms outside rigid molecules use per-atom
// kernels with the same arithmetic.
#include <cstdio>

#include "engine.hpp"

namespace mdx {

// ---------------------------------------------------------------- NH chain
// exp(x) for the chain's arguments, -dt/8 .. -dt/2 times a thermostat
// velocity (|x| well below 1/64 for any stable run): the Taylor polynomial of
// degree 8 (truncation below 1e-22 relative, under FP64 rounding) evaluated
// by Estrin's scheme -- pairs of terms, then x^2, x^4, x^8 -- a dependent
// depth of four multiply-adds on the device's serial tail instead of
// Horner's nine; larger arguments use exp().  Host and device run the same
// code.
__host__ __device__ inline double nh_exp(double x) {
    if (fabs(x) >= 0.015625) return exp(x);
    const double x2 = x * x;
    const double x4 = x2 * x2;
    const double b0 = 1.0 + x;
    const double b1 = fma(x, 1.0 / 6.0, 0.5);
    const double b2 = fma(x, 1.0 / 120.0, 1.0 / 24.0);
    const double b3 = fma(x, 1.0 / 5040.0, 1.0 / 720.0);
    const double c0 = fma(x2, b1, b0);
    const double c1 = fma(x2, b3, b2);
    const double d0 = fma(x4, c1, c0);
    return fma(x4 * x4, 1.0 / 40320.0, d0);
}

// thermostatIntegrate (FixNoseHoover.cu:795-866), nTimesteps = n_ys = 1, for
// a chain of compile-time length N (loops unrolled, so a chain held in
// registers stays there); C has the fields of NHChain used here.  Divisions
// by the chain masses are products with their reciprocals.
template <int N, class C>
__host__ __device__ __forceinline__ double nh_integrate_n(C &c, bool stepInit) {
    const double nkt = c.ndf * c.kB * c.T;
    if (!stepInit) c.force[0] = (c.ke - nkt) * c.inv_mass[0];
    const double ts = c.dt;
    const double t2 = 0.5 * ts, t4 = 0.25 * ts, t8 = 0.125 * ts;
    c.vel[N - 1] += t4 * c.force[N - 1];
#pragma unroll
    for (int k = N - 2; k > 0; --k) {
        double pf = nh_exp(-t8 * c.vel[k + 1]);
        c.vel[k] *= pf;
        c.vel[k] += t4 * c.force[k];
        c.vel[k] *= pf;
    }
    double pf = nh_exp(-t8 * c.vel[1]);
    c.vel[0] *= pf;
    c.vel[0] += t4 * c.force[0];
    c.vel[0] *= pf;
    const double sf = nh_exp(-t2 * c.vel[0]);
    c.ke *= sf * sf;
    c.vel[0] *= pf;
    c.force[0] = (c.ke - nkt) * c.inv_mass[0];
    c.vel[0] += t4 * c.force[0];
    c.vel[0] *= pf;
#pragma unroll
    for (int k = 1; k < N - 1; ++k) {
        pf = nh_exp(-t8 * c.vel[k + 1]);
        c.vel[k] *= pf;
        c.force[k] = (c.mass[k - 1] * c.vel[k - 1] * c.vel[k - 1] - c.kB * c.T) * c.inv_mass[k];
        c.vel[k] += t4 * c.force[k];
        c.vel[k] *= pf;
    }
    c.force[N - 1] = (c.mass[N - 2] * c.vel[N - 2] * c.vel[N - 2] - c.kB * c.T) * c.inv_mass[N - 1];
    c.vel[N - 1] += t4 * c.force[N - 1];
    return sf;
}

// the chain has kNHChain links (FixNoseHoover's default chain length)
__host__ __device__ double nh_integrate(NHChain &c, bool stepInit) {
    return nh_integrate_n<kNHChain>(c, stepInit);
}

// device copy: [0] = state after stepInit of the coming step ("next"),
// [1] = state after the last stepFinal ("final", what the reference holds
// between runs); the pending velocity scale of the coming step is next.scale
// and the stepFinal part of it is final.scale.
namespace {

struct StepConsts {
    float dt, dtf;
    int n_atoms, n_mol;
    Box box;
};

__device__ __forceinline__ float4 kick(float4 v, float4 f, float dtf) {
    const float w = v.w;
    const float s = dtf * w;
    v.x += s * f.x;
    v.y += s * f.y;
    v.z += s * f.z;
    return v;
}

// SETTLE positions (settlePositions, FixRigid.cu:849-1132), FP64
__device__ void settle_pos(const RigidConsts &rc, const Box &box, double dt, const float4 x0[3], float4 x[3],
                           float4 v[3], DeviceStatus *st) {
    const double ra = rc.ra, rb = rc.rb, rcc = rc.rc, inv2Rc = rc.inv2Rc, wH = rc.wH;
    const double3 pO0 = d3(x0[0]), pH10 = d3(x0[1]), pH20 = d3(x0[2]);
    double3 pO = d3(x[0]), pH1 = d3(x[1]), pH2 = d3(x[2]);
    double3 vO = d3(v[0]), vH1 = d3(v[1]), vH2 = d3(v[2]);
    const double3 b0v = min_image(box, pH10 - pO0);
    const double3 c0v = min_image(box, pH20 - pO0);
    const double3 oh1 = min_image(box, pH1 - pO);
    const double3 oh2 = min_image(box, pH2 - pO);
    pH1 = pO + oh1;
    pH2 = pO + oh2;
    const double3 com = pO + (oh1 + oh2) * wH;
    const double3 a1 = (oh1 + oh2) * (-1.0 * wH);
    const double3 b1 = pH1 - com;
    const double3 c1 = pH2 - com;
    double3 ax3 = crossd(b0v, c0v);
    double3 ax1 = crossd(a1, ax3);
    double3 ax2 = crossd(ax3, ax1);
    // unit axes: one reciprocal square root each instead of a square root
    // and three divisions
    ax1 = ax1 * rsqrt(dotd(ax1, ax1));
    ax2 = ax2 * rsqrt(dotd(ax2, ax2));
    ax3 = ax3 * rsqrt(dotd(ax3, ax3));
    auto rot = [&](double3 u) { return make_double3(dotd(ax1, u), dotd(ax2, u), dotd(ax3, u)); };
    const double3 rb0 = rot(b0v), rc0 = rot(c0v), ra1 = rot(a1), rb1 = rot(b1), rc1 = rot(c1);
    const double sinPhi = ra1.z / ra;
    const double cosPhiSqr = 1.0 - sinPhi * sinPhi;
    double cosPhi = 0.0, sinPsi = 0.0, cosPsi = 0.0;
    if (cosPhiSqr <= 0) {
        atomicOr(&st->bits, kStatusSettleFail);
    } else {
        cosPhi = sqrt(cosPhiSqr);
        sinPsi = (rb1.z - rc1.z) * (inv2Rc / cosPhi);
        const double cosPsiSqr = 1.0 - sinPsi * sinPsi;
        if (cosPsiSqr <= 0) atomicOr(&st->bits, kStatusSettleFail);
        else cosPsi = sqrt(cosPsiSqr);
    }
    const double3 a2 = make_double3(0.0, ra * cosPhi, rb * sinPhi);
    const double3 b2 = make_double3(-1.0 * rcc * cosPsi, -rb * cosPhi - rcc * sinPsi * sinPhi,
                                    -rb * sinPhi + rcc * sinPsi * cosPhi);
    const double3 c2 = make_double3(rcc * cosPsi, -1.0 * rb * cosPhi + rcc * sinPsi * sinPhi,
                                    -1.0 * rb * sinPhi - rcc * sinPsi * cosPhi);
    const double alpha = b2.x * (rb0.x - rc0.x) + b2.y * rb0.y + c2.y * rc0.y;
    const double beta = b2.x * (rc0.y - rb0.y) + b2.y * rb0.x + c2.y * rc0.x;
    const double gamma = rb0.x * rb1.y - rb1.x * rb0.y + rc0.x * rc1.y - rc1.x * rc0.y;
    const double a2b2 = alpha * alpha + beta * beta;
    const double sinT = (alpha * gamma - (beta * sqrt(a2b2 - gamma * gamma))) / a2b2;
    const double cosT = sqrt(1.0 - sinT * sinT);
    const double3 a3 = make_double3(-a2.y * sinT, a2.y * cosT, ra1.z);
    const double3 b3 = make_double3(b2.x * cosT - b2.y * sinT, b2.x * sinT + b2.y * cosT, b2.z);
    const double3 c3 = make_double3(c2.x * cosT - c2.y * sinT, c2.x * sinT + c2.y * cosT, c2.z);
    // back-rotation with the transposed frame
    const double3 t1 = make_double3(ax1.x, ax2.x, ax3.x), t2 = make_double3(ax1.y, ax2.y, ax3.y),
                  t3 = make_double3(ax1.z, ax2.z, ax3.z);
    auto back = [&](double3 u) { return make_double3(dotd(t1, u), dotd(t2, u), dotd(t3, u)); };
    const double3 ap = back(a3), bp = back(b3), cp = back(c3);
    const double invdt = 1.0 / dt;
    const double3 nO = ap + com, nH1 = bp + com, nH2 = cp + com;
    vO += (ap - a1) * invdt;
    vH1 += (bp - b1) * invdt;
    vH2 += (cp - c1) * invdt;
    x[0] = make_float4((float)nO.x, (float)nO.y, (float)nO.z, x[0].w);
    x[1] = make_float4((float)nH1.x, (float)nH1.y, (float)nH1.z, x[1].w);
    x[2] = make_float4((float)nH2.x, (float)nH2.y, (float)nH2.z, x[2].w);
    v[0] = make_float4((float)vO.x, (float)vO.y, (float)vO.z, v[0].w);
    v[1] = make_float4((float)vH1.x, (float)vH1.y, (float)vH1.z, v[1].w);
    v[2] = make_float4((float)vH2.x, (float)vH2.y, (float)vH2.z, v[2].w);
}

// SETTLE velocities (settleVelocities, FixRigid.cu:657-846), FP64
__device__ void settle_vel(const RigidConsts &rc, const Box &box, const float4 x[3], float4 v[3]) {
    double3 vO = d3(v[0]), vH1 = d3(v[1]), vH2 = d3(v[2]);
    const double3 xO = d3(x[0]), xH1 = d3(x[1]), xH2 = d3(x[2]);
    const double3 rOH1 = min_image(box, xO - xH1) * rc.invOH;
    const double3 rOH2 = min_image(box, xO - xH2) * rc.invOH;
    const double3 rHH = min_image(box, xH1 - xH2) * rc.invHH;
    const double3 rel = make_double3(dotd(vO - vH1, rOH1), dotd(vO - vH2, rOH2), dotd(vH1 - vH2, rHH));
    const double *M = rc.Minv;
    const double3 vc = make_double3(M[0] * rel.x + M[1] * rel.y + M[2] * rel.z,
                                    M[3] * rel.x + M[4] * rel.y + M[5] * rel.z,
                                    M[6] * rel.x + M[7] * rel.y + M[8] * rel.z);
    vO += (rOH1 * vc.x + rOH2 * vc.y) * (-1.0 * rc.invmO);
    vH1 += (rOH1 * (-1.0) * vc.x + rHH * vc.z) * (-1.0 * rc.invmH);
    vH2 += (rOH2 * (-1.0) * vc.y - rHH * vc.z) * (-1.0 * rc.invmH);
    v[0] = make_float4((float)vO.x, (float)vO.y, (float)vO.z, v[0].w);
    v[1] = make_float4((float)vH1.x, (float)vH1.y, (float)vH1.z, v[1].w);
    v[2] = make_float4((float)vH2.x, (float)vH2.y, (float)vH2.z, v[2].w);
}

// validateConstraints (FixRigid.cu:351-447): bit 0 set when a side length
// (O-H1, O-H2, H1-H2) is off its fixed value by more than 1e-3 (a NaN
// length counts as off); with v, bit 1 set when a relative velocity along a
// bond, dot(r_ij, v_j - v_i), exceeds 1e-3 (the reference's one-sided test)
__device__ __forceinline__ uint32_t rigid_violation(const RigidConsts &rc, const Box &box, const float4 x[3],
                                                    const float4 *v) {
    const float tol = 1e-3f;
    const float3 r01 = min_image(box, f3(x[1]) - f3(x[0]));
    const float3 r02 = min_image(box, f3(x[2]) - f3(x[0]));
    const float3 r12 = min_image(box, f3(x[2]) - f3(x[1]));
    const float oh = (float)rc.r_OH, hh = (float)rc.r_HH;
    uint32_t bad = 0u;
    if (!(fabsf(sqrtf(dot3(r01, r01)) - oh) <= tol) || !(fabsf(sqrtf(dot3(r02, r02)) - oh) <= tol) ||
        !(fabsf(sqrtf(dot3(r12, r12)) - hh) <= tol))
        bad |= 1u;
    if (v) {
        const float3 v01 = f3(v[1]) - f3(v[0]), v02 = f3(v[2]) - f3(v[0]), v12 = f3(v[2]) - f3(v[1]);
        if (dot3(r01, v01) > tol || dot3(r02, v02) > tol || dot3(r12, v12) > tol) bad |= 2u;
    }
    return bad;
}

// setMSite (FixRigid.cu:560-599), FP32 as the reference
__device__ __forceinline__ float4 msite(const RigidConsts &rc, const Box &box, const float4 x[3], float w) {
    const float3 o = f3(x[0]);
    const float3 rij = min_image(box, f3(x[1]) - o);
    const float3 rik = min_image(box, f3(x[2]) - o);
    const float3 s = rij + rik;
    const float l = sqrtf(dot3(s, s));
    const float om = (float)rc.r_OM;
    const float3 m = o + om * (s * (1.0f / l));
    return make_float4(m.x, m.y, m.z, w);
}

int rigid_blocks(int nmol) { return (nmol + kMolBlock - 1) / kMolBlock; }

// Arguments of the per-molecule kernels for one system: a0 (single system)
// or tab[blockIdx.y] (batched replicas; a0 then only sizes the grid).
struct MolArgs {
    int nmol;
    const int4 *mol_ids;
    int4 *mol_idx;
    const int *idToIdx;
    float4 *xs, *vs, *fs;
    RigidConsts rc;
    Box box;
    float dt, dtf;
    NHChain *chain;
    DeviceStatus *st;
    double *partials;
    int part_off, nparts;
    unsigned int *counter;
    int nh;
    double *ke_out;
    const float4 *fextra;
    const float4 *frecip;  // P3M reciprocal forces of every site (may be null)
    int nblk;  // blocks of k_second_mol that carry this system's molecules
    // 1: the molecule form's layout, thread m takes slot m whose sites are
    // 4m .. 4m+3 (coalesced, no map read); 0: molecule m's sites from mol_idx
    int slots;
};

__device__ __forceinline__ int4 mol_sites(const MolArgs &A, int m) {
    return A.slots ? make_int4(4 * m, 4 * m + 1, 4 * m + 2, 4 * m + 3) : A.mol_idx[m];
}
#define MDX_MOL_ARGS \
    pdl_wait();      \
    const MolArgs A = tab ? tab[blockIdx.y] : a0

// rebuild-group kernel: molecule -> current atom indices (idToIdx after sort)
__global__ void k_rigid_maps(const MolArgs a0, const MolArgs *__restrict__ tab, int conditional) {
    MDX_MOL_ARGS;
    // a molecule-form replica's sort rewrites its map itself
    if (A.slots || (conditional && !A.st->rebuild)) return;
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= A.nmol) return;
    const int *__restrict__ idToIdx = A.idToIdx;
    int4 a = A.mol_ids[m];
    A.mol_idx[m] = make_int4(idToIdx[a.x], idToIdx[a.y], idToIdx[a.z], a.w >= 0 ? idToIdx[a.w] : -1);
}

// ---- first half ---------------------------------------------------------
// per-atom: NH rescale (rescale_no_tags_cu) + nve_v + nve_x (+ zero force)
template <bool NH>
__global__ void k_first_atoms(int n, float4 *__restrict__ xs, float4 *__restrict__ vs, float4 *__restrict__ fs,
                              const uint32_t *__restrict__ ids, const uint8_t *__restrict__ rigid_by_id, float dt,
                              float dtf, const NHChain *__restrict__ chain) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (rigid_by_id && rigid_by_id[ids[i]]) return;
    float4 v = vs[i];
    float4 f = fs[i];
    if (NH) {
        const float s = (float)chain[0].scale;
        v.x *= s;
        v.y *= s;
        v.z *= s;
    }
    if (v.w > kInvMassBool) {
        vs[i] = make_float4(0.f, 0.f, 0.f, v.w);
        fs[i] = make_float4(0.f, 0.f, 0.f, f.w);
        return;
    }
    v = kick(v, f, dtf);
    vs[i] = v;
    float4 x = xs[i];
    x.x += dt * v.x;
    x.y += dt * v.y;
    x.z += dt * v.z;
    xs[i] = x;
    fs[i] = make_float4(0.f, 0.f, 0.f, f.w);
}

// per-molecule fused: NH rescale + save_prev_val + nve_v + nve_x + SETTLE + M-site
template <bool NH>
__global__ void k_first_mol(const MolArgs a0, const MolArgs *__restrict__ tab) {
    MDX_MOL_ARGS;
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= A.nmol) return;
    float4 *__restrict__ xs = A.xs;
    float4 *__restrict__ vs = A.vs;
    float4 *__restrict__ fs = A.fs;
    const RigidConsts &rc = A.rc;
    const Box &box = A.box;
    const float dt = A.dt, dtf = A.dtf;
    const NHChain *__restrict__ chain = A.chain;
    DeviceStatus *st = A.st;
    const int4 ix = mol_sites(A, m);
    const int id3[3] = {ix.x, ix.y, ix.z};
    float4 x0[3], x[3], v[3];
    // the M site's words read with the rest, not after the SETTLE
    float vmw = 0.f, fmw = 0.f, xmw = 0.f;
    if (rc.foursite) {
        vmw = vs[ix.w].w;
        fmw = fs[ix.w].w;
        xmw = xs[ix.w].w;
    }
    const float s = NH ? (float)chain[0].scale : 1.0f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        x0[k] = xs[id3[k]];
        v[k] = vs[id3[k]];
        const float4 f = fs[id3[k]];
        if (NH) {
            v[k].x *= s;
            v[k].y *= s;
            v[k].z *= s;
        }
        v[k] = kick(v[k], f, dtf);
        x[k] = make_float4(x0[k].x + dt * v[k].x, x0[k].y + dt * v[k].y, x0[k].z + dt * v[k].z, x0[k].w);
        fs[id3[k]] = make_float4(0.f, 0.f, 0.f, f.w);
    }
    settle_pos(rc, box, (double)dt, x0, x, v, st);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        xs[id3[k]] = x[k];
        vs[id3[k]] = v[k];
    }
    if (rc.foursite) {
        vs[ix.w] = make_float4(0.f, 0.f, 0.f, vmw);
        fs[ix.w] = make_float4(0.f, 0.f, 0.f, fmw);
        xs[ix.w] = msite(rc, box, x, xmw);
    }
    // late trigger: the dependent's blocks become resident during this
    // grid's tail; their griddepcontrol.wait still waits for all of it
    pdl_trigger();
}

// ---- second half --------------------------------------------------------
__device__ __forceinline__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}

// the time-dependent part of a chain, held in registers by the last block
struct NHRegs {
    double vel[kNHChain], force[kNHChain], mass[kNHChain], inv_mass[kNHChain];
    double ke, ndf, kB, T, dt;
};

__device__ __forceinline__ void store_chain(NHChain &d, const NHRegs &c, double last_ke, double scale) {
#pragma unroll
    for (int k = 0; k < kNHChain; k++) {
        d.vel[k] = c.vel[k];
        d.force[k] = c.force[k];
    }
    d.ke = c.ke;
    d.last_ke = last_ke;
    d.scale = scale;
}

// Last-block epilogue: fixed-order FP64 sum of the block partials, then the
// Nose-Hoover stepFinal + next stepInit on one thread, and the turn counter.
// nparts partials are summed; the counter target is this kernel's grid size
__device__ void finish_step(double *partials, int nparts, unsigned int *counter, NHChain *chain, int nh,
                            DeviceStatus *st, double *ke_out, unsigned int nblk) {
    __shared__ bool last;
    __threadfence();
    if (threadIdx.x == 0) {
        unsigned int prev = atomicAdd(counter, 1u);
        last = (prev == nblk - 1u);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // thread 0 reads the chain into registers (a copy of the struct would
    // sit in local memory on this serial path) while the partials are read
    NHRegs c;
    double mvv = 0.0;
    if (threadIdx.x == 0 && nh) {
        const NHChain &g = chain[0];
#pragma unroll
        for (int k = 0; k < kNHChain; k++) {
            c.vel[k] = __ldcg(&g.vel[k]);
            c.force[k] = __ldcg(&g.force[k]);
            c.mass[k] = __ldcg(&g.mass[k]);
            c.inv_mass[k] = __ldcg(&g.inv_mass[k]);
        }
        c.ndf = __ldcg(&g.ndf);
        c.kB = __ldcg(&g.kB);
        c.T = __ldcg(&g.T);
        c.dt = __ldcg(&g.dt);
        mvv = __ldcg(&g.mvv_to_eng);
    }
    // every thread of the last block sums a fixed strided share of the
    // partials (L2 reads), then a fixed-order block reduction: deterministic
    __shared__ double red[32];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) acc += __ldcg(partials + b);
    const double tot_all = block_sum(acc, red);
    if (threadIdx.x == 0) {
        const double tot = tot_all;
        *counter = 0u;
        if (ke_out) *ke_out = tot;
        if (nh) {
            // constants stay in chain[0/1]
            c.ke = tot * mvv;
            const double last_ke = c.ke;
            const double sf1 = nh_integrate_n<kNHChain>(c, false);  // stepFinal
            store_chain(chain[1], c, last_ke, sf1);
            const double sf2 = nh_integrate_n<kNHChain>(c, true);   // stepInit of the next step
            store_chain(chain[0], c, last_ke, sf1 * sf2);
        }
        st->turn += 1;
    }
}

// per-atom: postForce_cu (IntegratorVerlet.cu:610-627) + m v^2 partials
__global__ void k_second_atoms(int n, float4 *__restrict__ vs, const float4 *__restrict__ fs,
                               const uint32_t *__restrict__ ids, const uint8_t *__restrict__ rigid_by_id, float dtf,
                               double *__restrict__ partials, int part_off, int nparts, unsigned int *counter,
                               NHChain *chain, int nh, DeviceStatus *st, double *ke_out, int do_finish) {
    __shared__ double sh[32];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mv2 = 0.0;
    if (i < n && !(rigid_by_id && rigid_by_id[ids[i]])) {
        float4 v = vs[i];
        if (v.w > kInvMassBool) {
            vs[i] = make_float4(0.f, 0.f, 0.f, v.w);
        } else {
            v = kick(v, fs[i], dtf);
            vs[i] = v;
            mv2 = ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z) / (double)v.w;
        }
    }
    const double b = block_sum(mv2, sh);
    if (threadIdx.x == 0) partials[part_off + blockIdx.x] = b;
    if (do_finish) finish_step(partials, nparts, counter, chain, nh, st, ke_out, gridDim.x);
}

// per-molecule fused: postForce + distributeMSite + settleVelocities +
// validateConstraints + m v^2 partials (+ last-block NH / turn)
// fextra (may be null): per-molecule-atom forces computed beside the pair
// kernel (E3B), indexed like fs, merged into O/H1/H2 here
__global__ void k_second_mol(const MolArgs a0, const MolArgs *__restrict__ tab) {
    MDX_MOL_ARGS;
    if ((int)blockIdx.x >= A.nblk) return;  // the whole block: not counted
    __shared__ double sh[32];
    const int nmol = A.nmol;
    const float4 *__restrict__ xs = A.xs;
    float4 *__restrict__ vs = A.vs;
    float4 *__restrict__ fs = A.fs;
    const RigidConsts &rc = A.rc;
    const Box &box = A.box;
    const float dtf = A.dtf;
    DeviceStatus *st = A.st;
    const float4 *__restrict__ fextra = A.fextra;
    const float4 *__restrict__ frecip = A.frecip;
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    double mv2 = 0.0;
    if (m < nmol) {
        const int4 ix = mol_sites(A, m);
        const int id3[3] = {ix.x, ix.y, ix.z};
        float4 x[3], v[3], f[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            x[k] = xs[id3[k]];
            f[k] = fs[id3[k]];
            if (fextra) {
                const float4 fe = fextra[id3[k]];
                f[k].x += fe.x;
                f[k].y += fe.y;
                f[k].z += fe.z;
            }
            if (frecip) {
                const float4 fr = frecip[id3[k]];
                f[k].x += fr.x;
                f[k].y += fr.y;
                f[k].z += fr.z;
            }
            v[k] = kick(vs[id3[k]], f[k], dtf);
        }
        if (rc.foursite) {
            float4 fm = fs[ix.w];
            if (frecip) {
                const float4 fr = frecip[ix.w];
                fm.x += fr.x;
                fm.y += fr.y;
                fm.z += fr.z;
            }
            const float4 vm = vs[ix.w];
            const float g = (float)rc.gamma;
            const float3 fOd = f3(fm) * g;
            const float3 fHd = f3(fm) * 0.5f * (1.0f - g);
            const float3 dvO = dtf * v[0].w * fOd;
            const float3 dvH = dtf * v[1].w * fHd;
            v[0].x += dvO.x; v[0].y += dvO.y; v[0].z += dvO.z;
            v[1].x += dvH.x; v[1].y += dvH.y; v[1].z += dvH.z;
            v[2].x += dvH.x; v[2].y += dvH.y; v[2].z += dvH.z;
            f[0].x += fOd.x; f[0].y += fOd.y; f[0].z += fOd.z;
            f[1].x += fHd.x; f[1].y += fHd.y; f[1].z += fHd.z;
            f[2].x += fHd.x; f[2].y += fHd.y; f[2].z += fHd.z;
            vs[ix.w] = make_float4(0.f, 0.f, 0.f, vm.w);
            fs[ix.w] = make_float4(0.f, 0.f, 0.f, fm.w);
        }
        if (rc.foursite || fextra || frecip) {
#pragma unroll
            for (int k = 0; k < 3; k++) fs[id3[k]] = f[k];
        }
        settle_vel(rc, box, x, v);
        // validateConstraints (FixRigid.cu:351-447), side lengths: flag,
        // never print or trap
        if (rigid_violation(rc, box, x, nullptr)) atomicOr(&st->bits, kStatusConstraint);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            vs[id3[k]] = v[k];
            mv2 += ((double)v[k].x * v[k].x + (double)v[k].y * v[k].y + (double)v[k].z * v[k].z) / (double)v[k].w;
        }
    }
    const double b = block_sum(mv2, sh);
    if (threadIdx.x == 0) A.partials[A.part_off + blockIdx.x] = b;
    // the next step's first half may be scheduled now: it waits for this
    // grid (the last block's chain update included) before reading anything
    pdl_trigger();
    finish_step(A.partials, A.nparts, A.counter, A.chain, A.nh, st, A.ke_out, (unsigned int)A.nblk);
}

// ---- stand-alone hooks (one kernel per reference hook) ------------------
// validateConstraints as its own hook: counts the molecules whose side
// lengths or bond velocities are off (into *bad), leaves the status word alone
__global__ void k_validate_hook(int nmol, const int4 *__restrict__ mol_idx, const float4 *__restrict__ xs,
                                const float4 *__restrict__ vs, RigidConsts rc, Box box, uint32_t *bad) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    const int4 ix = mol_idx[m];
    const float4 x[3] = {xs[ix.x], xs[ix.y], xs[ix.z]};
    const float4 v[3] = {vs[ix.x], vs[ix.y], vs[ix.z]};
    if (rigid_violation(rc, box, x, v)) atomicAdd(bad, 1u);
}

__global__ void k_save_prev(int nmol, const int4 *__restrict__ mol_idx, const float4 *__restrict__ xs,
                            float4 *__restrict__ xs0) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    const int4 ix = mol_idx[m];
    xs0[3 * m] = xs[ix.x];
    xs0[3 * m + 1] = xs[ix.y];
    xs0[3 * m + 2] = xs[ix.z];
}

__global__ void k_settle_pos_hook(int nmol, const int4 *__restrict__ mol_idx, float4 *__restrict__ xs,
                                  float4 *__restrict__ vs, const float4 *__restrict__ xs0, RigidConsts rc, Box box,
                                  float dt, DeviceStatus *st) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    const int4 ix = mol_idx[m];
    const int id3[3] = {ix.x, ix.y, ix.z};
    float4 x0[3], x[3], v[3];
    for (int k = 0; k < 3; k++) {
        x0[k] = xs0[3 * m + k];
        x[k] = xs[id3[k]];
        v[k] = vs[id3[k]];
    }
    settle_pos(rc, box, (double)dt, x0, x, v, st);
    for (int k = 0; k < 3; k++) {
        xs[id3[k]] = x[k];
        vs[id3[k]] = v[k];
    }
    if (rc.foursite) xs[ix.w] = msite(rc, box, x, xs[ix.w].w);
}

__global__ void k_distribute_hook(int nmol, const int4 *__restrict__ mol_idx, float4 *__restrict__ vs,
                                  float4 *__restrict__ fs, RigidConsts rc, float dtf) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol || !rc.foursite) return;
    const int4 ix = mol_idx[m];
    float4 fO = fs[ix.x], fH1 = fs[ix.y], fH2 = fs[ix.z], fM = fs[ix.w];
    float4 vO = vs[ix.x], vH1 = vs[ix.y], vH2 = vs[ix.z];
    const float g = (float)rc.gamma;
    const float3 fOd = f3(fM) * g, fHd = f3(fM) * 0.5f * (1.0f - g);
    const float3 dvO = dtf * vO.w * fOd, dvH = dtf * vH1.w * fHd;
    vO.x += dvO.x; vO.y += dvO.y; vO.z += dvO.z;
    vH1.x += dvH.x; vH1.y += dvH.y; vH1.z += dvH.z;
    vH2.x += dvH.x; vH2.y += dvH.y; vH2.z += dvH.z;
    vs[ix.x] = vO; vs[ix.y] = vH1; vs[ix.z] = vH2;
    vs[ix.w] = make_float4(0.f, 0.f, 0.f, kInvMassless);
    fO.x += fOd.x; fO.y += fOd.y; fO.z += fOd.z;
    fH1.x += fHd.x; fH1.y += fHd.y; fH1.z += fHd.z;
    fH2.x += fHd.x; fH2.y += fHd.y; fH2.z += fHd.z;
    fs[ix.x] = fO; fs[ix.y] = fH1; fs[ix.z] = fH2;
    fs[ix.w] = make_float4(0.f, 0.f, 0.f, fM.w);
}

__global__ void k_settle_vel_hook(int nmol, const int4 *__restrict__ mol_idx, const float4 *__restrict__ xs,
                                  float4 *__restrict__ vs, RigidConsts rc, Box box) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    const int4 ix = mol_idx[m];
    const int id3[3] = {ix.x, ix.y, ix.z};
    float4 x[3], v[3];
    for (int k = 0; k < 3; k++) {
        x[k] = xs[id3[k]];
        v[k] = vs[id3[k]];
    }
    settle_vel(rc, box, x, v);
    for (int k = 0; k < 3; k++) vs[id3[k]] = v[k];
}

// nve_v + nve_x for every atom (IntegratorVerlet.cu:23-61)
__global__ void k_verlet_first_all(int n, float4 *__restrict__ xs, float4 *__restrict__ vs, float4 *__restrict__ fs,
                                   float dt, float dtf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = vs[i];
    float4 f = fs[i];
    if (v.w > kInvMassBool) {
        vs[i] = make_float4(0.f, 0.f, 0.f, v.w);
        fs[i] = make_float4(0.f, 0.f, 0.f, f.w);
        return;
    }
    v = kick(v, f, dtf);
    vs[i] = v;
    fs[i] = make_float4(0.f, 0.f, 0.f, f.w);
    float4 x = xs[i];
    x.x += dt * v.x;
    x.y += dt * v.y;
    x.z += dt * v.z;
    xs[i] = x;
}

__global__ void k_verlet_second_all(int n, float4 *__restrict__ vs, const float4 *__restrict__ fs, float dtf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = vs[i];
    if (v.w > kInvMassBool) {
        vs[i] = make_float4(0.f, 0.f, 0.f, v.w);
        return;
    }
    vs[i] = kick(v, fs[i], dtf);
}

// rescale_no_tags_cu (FixNoseHoover.cu:40-51) with the scale read on device
__global__ void k_scale_v(int n, float4 *__restrict__ vs, const NHChain *__restrict__ chain) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float s = (float)chain[0].scale;
    float4 v = vs[i];
    v.x *= s;
    v.y *= s;
    v.z *= s;
    vs[i] = v;
}

__global__ void k_mv2(int n, const float4 *__restrict__ vs, double *__restrict__ partials) {
    __shared__ double sh[32];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mv2 = 0.0;
    if (i < n) {
        float4 v = vs[i];
        if (v.w < kInvMassBool) mv2 = ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z) / (double)v.w;
    }
    const double b = block_sum(mv2, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

// momentum sum (SumVectorXYZOverW) partials: 4 doubles per block
__global__ void k_momentum(int n, const float4 *__restrict__ vs, double *__restrict__ partials) {
    __shared__ double sh[32];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double p[4] = {0, 0, 0, 0};
    if (i < n) {
        float4 v = vs[i];
        double m = 1.0 / (double)v.w;
        p[0] = v.x * m;
        p[1] = v.y * m;
        p[2] = v.z * m;
        p[3] = m;
    }
    for (int c = 0; c < 4; c++) {
        const double b = block_sum(p[c], sh);
        __syncthreads();
        if (threadIdx.x == 0) partials[4 * blockIdx.x + c] = b;
    }
}

__global__ void k_sub_v(int n, float4 *__restrict__ vs, float3 dv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = vs[i];
    v.x -= dv.x;
    v.y -= dv.y;
    v.z -= dv.z;
    vs[i] = v;
}

__global__ void k_reduce_vec(int n, const double *__restrict__ src, int stride, int comp, double *out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += src[(size_t)i * stride + comp];
    const double b = block_sum(acc, sh);
    if (threadIdx.x == 0) out[comp] = b;
}

__global__ void k_reduce_float(int n, const float *__restrict__ src, int stride, int comp, double *out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += (double)src[(size_t)i * stride + comp];
    const double b = block_sum(acc, sh);
    if (threadIdx.x == 0) out[comp] = b;
}

// zero force xyz (group tag in .w kept) and per-atom virials
__global__ void k_zero_f(int n, float4 *__restrict__ fs, float *__restrict__ vir) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 f = fs[i];
    fs[i] = make_float4(0.f, 0.f, 0.f, f.w);
    if (vir)
        for (int c = 0; c < 6; c++) vir[6 * (size_t)i + c] = 0.f;
}

// FixNoseHoover::postRun (FixNoseHoover.cu:405-411) applies the scale left
// pending by the last stepFinal; the stepInit part stays pending for the
// next run so a continued run sees the same chain as the reference's
// re-prepared one
__global__ void k_nh_end_of_run(int n, float4 *__restrict__ vs, NHChain *chain) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double sf1 = chain[1].scale;
    if (i < n) {
        float4 v = vs[i];
        const float s = (float)sf1;
        v.x *= s;
        v.y *= s;
        v.z *= s;
        vs[i] = v;
    }
}
__global__ void k_nh_end_of_run_fix(NHChain *chain) {
    chain[0].scale /= chain[1].scale;
    chain[1].scale = 1.0;
}

}  // namespace

MolArgs mol_args(State &s, FixRigid &r) {
    MolArgs A{};
    FixNoseHoover *nh = s.nhFix();
    A.nmol = (int)r.mol_ids.size();
    A.mol_ids = r.d_mol_ids.p;
    A.mol_idx = r.d_mol_idx.p;
    A.idToIdx = s.gpd.idToIdx.p;
    A.xs = s.gpd.xs.p;
    A.vs = s.gpd.vs.p;
    A.fs = s.gpd.fs.p;
    A.rc = r.rc;
    A.box = s.box;
    A.dt = (float)s.dt;
    A.dtf = (float)(0.5 * s.dt * s.units.ftm_to_v);
    A.chain = nh ? nh->d_chain.p : nullptr;
    A.st = s.d_status.p;
    A.partials = s.red_partials.p;
    A.part_off = 0;
    A.nparts = rigid_blocks(A.nmol);
    A.counter = s.red_counter.p;
    A.nh = nh ? 1 : 0;
    A.ke_out = s.red_out.p;
    A.fextra = nullptr;
    A.frecip = nullptr;
    A.nblk = rigid_blocks(A.nmol);
    A.slots = 0;
    return A;
}

int rigid_update_maps(State &s, FixRigid &r, bool conditional) {
    const int nmol = (int)r.mol_ids.size();
    if (nmol == 0 || !r.d_mol_ids.p) return 0;
    MDX_CUDA_TRY(launch_pdl(k_rigid_maps, dim3((nmol + 255) / 256), dim3(256), 0, s.stream, mol_args(s, r),
                            (const MolArgs *)nullptr, conditional ? 1 : 0));
    return 0;
}

// rigid-membership by id (static), lazily built
static uint8_t *rigid_flags(State &s) {
    static thread_local std::map<State *, DBuf<uint8_t> *> cache;
    FixRigid *r = s.rigidFix();
    if (!r) return nullptr;
    auto it = cache.find(&s);
    if (it != cache.end() && it->second->n == s.atoms.size()) return it->second->p;
    std::vector<uint8_t> h(s.atoms.size(), 0);
    for (auto &m : r->mol_ids) {
        h[m.x] = h[m.y] = h[m.z] = 1;
        if (m.w >= 0) h[m.w] = 1;
    }
    auto *b = new DBuf<uint8_t>();
    if (b->alloc(h.size())) return nullptr;
    cudaMemcpy(b->p, h.data(), h.size(), cudaMemcpyHostToDevice);
    cache[&s] = b;
    return b->p;
}

int rigid_flags_prepare(State &s) { return (s.rigidFix() && !rigid_flags(s)) ? MDX_ERR_CUDA : 0; }

bool has_free_atoms(State &s) {
    FixRigid *r = s.rigidFix();
    if (!r) return true;
    size_t members = 0;
    for (auto &m : r->mol_ids) members += m.w >= 0 ? 4 : 3;
    return members < s.atoms.size();
}

int step_first_half(State &s, bool fused) {
    const int n = s.gpd.n;
    const float dt = (float)s.dt;
    const float dtf = (float)(0.5 * s.dt * s.units.ftm_to_v);
    FixNoseHoover *nh = s.nhFix();
    FixRigid *r = s.rigidFix();
    const NHChain *chain = nh ? nh->d_chain.p : nullptr;
    if (!fused) {
        // reference hook order: stepInit (NH rescale, rigid save_prev) ->
        // nve_v + nve_x on all atoms -> postNVE_X (SETTLE, M-site)
        if (nh) {
            k_scale_v<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.vs.p, nh->d_chain.p);
            MDX_LAUNCHED();
        }
        if (r) {
            if (int e = rigid_hook(s, *r, 0)) return e;
        }
        k_verlet_first_all<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.xs.p, s.gpd.vs.p, s.gpd.fs.p, dt, dtf);
        MDX_LAUNCHED();
        if (r) {
            if (int e = rigid_hook(s, *r, 1)) return e;
        }
        return 0;
    }
    if (has_free_atoms(s)) {
        const uint8_t *rf = r ? rigid_flags(s) : nullptr;
        if (nh)
            k_first_atoms<true><<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.xs.p, s.gpd.vs.p, s.gpd.fs.p,
                                                                      s.gpd.ids.p, rf, dt, dtf, chain);
        else
            k_first_atoms<false><<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.xs.p, s.gpd.vs.p, s.gpd.fs.p,
                                                                       s.gpd.ids.p, rf, dt, dtf, chain);
        MDX_LAUNCHED();
    }
    if (r) {
        MolArgs A = mol_args(s, *r);
        A.slots = s.mf.on ? 1 : 0;
        if (nh)
            MDX_CUDA_TRY(launch_pdl(k_first_mol<true>, dim3(rigid_blocks(A.nmol)), dim3(kMolBlock), 0, s.stream, A,
                                    (const MolArgs *)nullptr));
        else
            MDX_CUDA_TRY(launch_pdl(k_first_mol<false>, dim3(rigid_blocks(A.nmol)), dim3(kMolBlock), 0, s.stream, A,
                                    (const MolArgs *)nullptr));
    }
    return 0;
}

int step_second_half(State &s, bool fused, const float4 *fextra, const float4 *frecip) {
    const int n = s.gpd.n;
    const float dtf = (float)(0.5 * s.dt * s.units.ftm_to_v);
    FixNoseHoover *nh = s.nhFix();
    FixRigid *r = s.rigidFix();
    NHChain *chain = nh ? nh->d_chain.p : nullptr;
    const int ab = (n + 255) / 256;
    const int mb = r ? rigid_blocks((int)r->mol_ids.size()) : 0;
    const bool free_atoms = has_free_atoms(s);
    int nparts = (free_atoms ? ab : 0) + mb;
    if ((size_t)(std::max(nparts, ab) + 8) > s.red_partials.n) {
        set_error(MDX_ERR_STATE, "reduction buffer not sized by prepare");
        return MDX_ERR_STATE;
    }
    if (!fused) {
        k_verlet_second_all<<<ab, 256, 0, s.stream>>>(n, s.gpd.vs.p, s.gpd.fs.p, dtf);
        MDX_LAUNCHED();
        if (r) {
            if (int e = rigid_hook(s, *r, 2)) return e;
            if (int e = rigid_hook(s, *r, 3)) return e;
        }
        // stepFinal: reduce m v^2 then the chain on the device (single block)
        k_mv2<<<ab, 256, 0, s.stream>>>(n, s.gpd.vs.p, s.red_partials.p);
        MDX_LAUNCHED();
        k_second_atoms<<<1, 32, 0, s.stream>>>(0, s.gpd.vs.p, s.gpd.fs.p, nullptr, nullptr, dtf, s.red_partials.p,
                                               ab, ab + 1, s.red_counter.p, chain, nh ? 1 : 0, s.d_status.p,
                                               s.red_out.p, 1);
        MDX_LAUNCHED();
        return 0;
    }
    const uint8_t *rf = r ? rigid_flags(s) : nullptr;
    if (free_atoms) {
        k_second_atoms<<<ab, 256, 0, s.stream>>>(n, s.gpd.vs.p, s.gpd.fs.p, s.gpd.ids.p, rf, dtf, s.red_partials.p, 0,
                                                 nparts, s.red_counter.p, chain, nh ? 1 : 0, s.d_status.p,
                                                 s.red_out.p, r ? 0 : 1);
        MDX_LAUNCHED();
    }
    if (r) {
        MolArgs A = mol_args(s, *r);
        A.part_off = free_atoms ? ab : 0;
        A.nparts = nparts;
        A.fextra = fextra;
        A.frecip = frecip;
        A.slots = s.mf.on ? 1 : 0;
        MDX_CUDA_TRY(launch_pdl(k_second_mol, dim3(mb), dim3(kMolBlock), 0, s.stream, A, (const MolArgs *)nullptr));
    }
    return 0;
}

// which: 0 save_prev, 1 settle positions (+M-site), 2 distribute M-site, 3 settle velocities
int rigid_hook(State &s, FixRigid &r, int which) {
    const int nmol = (int)r.mol_ids.size();
    if (nmol == 0) return 0;
    const int nb = (nmol + 127) / 128;
    const float dtf = (float)(0.5 * s.dt * s.units.ftm_to_v);
    if (int e = r.xs0.alloc(3 * nmol)) return e;
    switch (which) {
        case 0:
            k_save_prev<<<nb, 128, 0, s.stream>>>(nmol, r.d_mol_idx.p, s.gpd.xs.p, r.xs0.p);
            break;
        case 1:
            k_settle_pos_hook<<<nb, 128, 0, s.stream>>>(nmol, r.d_mol_idx.p, s.gpd.xs.p, s.gpd.vs.p, r.xs0.p, r.rc,
                                                        s.box, (float)s.dt, s.d_status.p);
            break;
        case 2:
            k_distribute_hook<<<nb, 128, 0, s.stream>>>(nmol, r.d_mol_idx.p, s.gpd.vs.p, s.gpd.fs.p, r.rc, dtf);
            break;
        case 3:
            k_settle_vel_hook<<<nb, 128, 0, s.stream>>>(nmol, r.d_mol_idx.p, s.gpd.xs.p, s.gpd.vs.p, r.rc, s.box);
            break;
        default:
            return MDX_ERR_ARG;
    }
    MDX_LAUNCHED();
    return 0;
}

// validateConstraints (FixRigid.cu:351-447) on the current positions and
// velocities: *n_bad = molecules off their constraints
int rigid_validate(State &s, FixRigid &r, uint32_t *n_bad) {
    const int nmol = (int)r.mol_ids.size();
    *n_bad = 0;
    if (nmol == 0) return 0;
    if (int e = r.d_bad.alloc(1)) return e;
    MDX_CUDA_TRY(cudaMemsetAsync(r.d_bad.p, 0, sizeof(uint32_t), s.stream));
    k_validate_hook<<<(nmol + 127) / 128, 128, 0, s.stream>>>(nmol, r.d_mol_idx.p, s.gpd.xs.p, s.gpd.vs.p, r.rc,
                                                               s.box, r.d_bad.p);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaMemcpyAsync(n_bad, r.d_bad.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    return 0;
}

// FixRigid::prepareForRun (FixRigid.cu:1740-1880) with solveInitialConstraints:
// SETTLE the current configuration onto itself, place M, settle velocities,
// remove the centre-of-mass velocity
int rigid_prepare(State &s, FixRigid &r) {
    if (int e = rigid_update_maps(s, r, false)) return e;
    if (int e = rigid_hook(s, r, 0)) return e;
    if (int e = rigid_hook(s, r, 1)) return e;
    if (int e = rigid_hook(s, r, 3)) return e;
    return remove_com_velocity(s);
}

int remove_com_velocity(State &s) {
    const int n = s.gpd.n;
    const int nb = (n + 255) / 256;
    DBuf<double> part, out;
    if (int e = part.alloc(4 * nb)) return e;
    if (int e = out.alloc(4)) return e;
    k_momentum<<<nb, 256, 0, s.stream>>>(n, s.gpd.vs.p, part.p);
    MDX_LAUNCHED();
    for (int c = 0; c < 4; c++) {
        k_reduce_vec<<<1, 256, 0, s.stream>>>(nb, part.p, 4, c, out.p);
        MDX_LAUNCHED();
    }
    double h[4];
    MDX_CUDA_TRY(cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    float3 dv = make_float3((float)(h[0] / h[3]), (float)(h[1] / h[3]), (float)(h[2] / h[3]));
    k_sub_v<<<nb, 256, 0, s.stream>>>(n, s.gpd.vs.p, dv);
    MDX_LAUNCHED();
    return 0;
}

int kinetic_sum(State &s, double *out) {
    const int n = s.gpd.n;
    const int nb = (n + 255) / 256;
    DBuf<double> part, o;
    if (int e = part.alloc(nb)) return e;
    if (int e = o.alloc(1)) return e;
    k_mv2<<<nb, 256, 0, s.stream>>>(n, s.gpd.vs.p, part.p);
    MDX_LAUNCHED();
    k_reduce_vec<<<1, 256, 0, s.stream>>>(nb, part.p, 1, 0, o.p);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaMemcpyAsync(out, o.p, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    return 0;
}

// FP64 sum of n floats on the device (one block, fixed order) into *out_host
int float_sum(State &s, const float *src, int n, double *out_host) {
    k_reduce_float<<<1, 256, 0, s.stream>>>(n, src, 1, 0, s.e_sum.p);
    MDX_LAUNCHED();
    MDX_CUDA_TRY(cudaMemcpyAsync(out_host, s.e_sum.p, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    return 0;
}

int virial_sum(State &s, double out6[6]) {
    DBuf<double> o;
    if (int e = o.alloc(6)) return e;
    for (int c = 0; c < 6; c++) {
        k_reduce_float<<<1, 256, 0, s.stream>>>(s.gpd.n, s.gpd.virials.p, 6, c, o.p);
        MDX_LAUNCHED();
    }
    MDX_CUDA_TRY(cudaMemcpyAsync(out6, o.p, 6 * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    return 0;
}

// FixNoseHoover::prepareFinal (FixNoseHoover.cu:240-290) then stepInit's
// half of the chain for the first step; the result is uploaded.
int nh_prepare(State &s, FixNoseHoover &nh) {
    double mv2 = 0.0;
    if (int e = kinetic_sum(s, &mv2)) return e;
    NHChain &c = nh.h;
    int ndf = 0;
    for (auto &a : s.atoms) ndf += a.ndf;
    c.n = kNHChain;
    c.T = nh.T;
    c.freq = 1.0 / nh.tau;
    c.ndf = ndf;
    c.kB = s.units.boltz;
    c.dt = s.dt;
    c.mvv_to_eng = s.units.mvv_to_eng;
    if (!nh.chain_on_device) {
        for (int k = 0; k < 10; k++) c.vel[k] = c.force[k] = 0.0;
    }
    c.ke = mv2 * s.units.mvv_to_eng;
    c.mass[0] = c.ndf * c.kB * c.T / (c.freq * c.freq);
    for (int k = 1; k < c.n; k++) c.mass[k] = c.kB * c.T / (c.freq * c.freq);
    for (int k = 0; k < c.n; k++) c.inv_mass[k] = 1.0 / c.mass[k];
    c.force[0] = (c.ke - c.ndf * c.kB * c.T) / c.mass[0];
    for (int k = 1; k < c.n; k++) c.force[k] = (c.mass[k - 1] * c.vel[k - 1] * c.vel[k - 1] - c.kB * c.T) / c.mass[k];
    NHChain pair[2];
    pair[1] = c;
    pair[1].scale = 1.0;
    NHChain nx = c;
    nx.scale = nh_integrate(nx, true);
    pair[0] = nx;
    if (int e = nh.d_chain.alloc(2)) return e;
    MDX_CUDA_TRY(cudaMemcpy(nh.d_chain.p, pair, sizeof(pair), cudaMemcpyHostToDevice));
    nh.h = nx;
    nh.chain_on_device = true;
    return 0;
}

int nh_end_of_run(State &s) {
    FixNoseHoover *nh = s.nhFix();
    if (!nh || !nh->d_chain.p) return 0;
    const int n = s.gpd.n;
    k_nh_end_of_run<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.vs.p, nh->d_chain.p);
    MDX_LAUNCHED();
    k_nh_end_of_run_fix<<<1, 1, 0, s.stream>>>(nh->d_chain.p);
    MDX_LAUNCHED();
    return 0;
}

int zero_forces(State &s) {
    const int n = s.gpd.n;
    k_zero_f<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.fs.p, s.gpd.virials.p);
    MDX_LAUNCHED();
    return 0;
}

// ---- batched replicas: one launch per phase, blockIdx.y = replica ----------
int batch_mol_tables(Batch &b) {
    const int R = (int)b.reps.size();
    std::vector<MolArgs> h1(R), h2(R);
    for (int r = 0; r < R; r++) {
        State &s = *b.reps[r];
        FixRigid *fr = s.rigidFix();
        h1[r] = mol_args(s, *fr);
        h1[r].slots = s.mf.on ? 1 : 0;
        // the P3M branch's per-step reciprocal forces (molecule-form gather)
        h1[r].frecip = b.p3m_mol ? s.ewaldFix()->f_recip.p : nullptr;
        h2[r] = h1[r];
        FixE3B *e3 = s.e3bFix();
        h2[r].fextra = (e3 && e3->side_ok) ? e3->f_side.p : nullptr;
    }
    if (int e = b.tab_first.alloc(R * sizeof(MolArgs))) return e;
    if (int e = b.tab_second.alloc(R * sizeof(MolArgs))) return e;
    MDX_CUDA_TRY(cudaMemcpy(b.tab_first.p, h1.data(), R * sizeof(MolArgs), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(b.tab_second.p, h2.data(), R * sizeof(MolArgs), cudaMemcpyHostToDevice));
    return 0;
}

static int batch_sizing(Batch &b, MolArgs *out) {
    if (!b.tab_first.p) {
        set_error(MDX_ERR_STATE, "batch tables not built (prepare the batch)");
        return MDX_ERR_STATE;
    }
    State &s0 = *b.reps[0];
    MolArgs A = mol_args(s0, *s0.rigidFix());
    A.nmol = b.max_mol;
    A.nblk = rigid_blocks(b.max_mol);
    *out = A;
    return 0;
}

namespace {
// Mod::scaleSystem (Mod.cu:201-240) for the atoms outside rigid molecules:
// x -> c + (x - c) s about the box centre c
__global__ void k_scale_free(int n, float4 *__restrict__ xs, const uint32_t *__restrict__ ids,
                             const uint8_t *__restrict__ rigid_by_id, double3 c, double s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (rigid_by_id && rigid_by_id[ids[i]]) return;
    float4 x = xs[i];
    x.x = (float)(c.x + ((double)x.x - c.x) * s);
    x.y = (float)(c.y + ((double)x.y - c.y) * s);
    x.z = (float)(c.z + ((double)x.z - c.z) * s);
    xs[i] = x;
}

// FixRigid::scaleRigidBodies (rigid_scaleSystem_cu, FixRigid.cu:164-242):
// the centre of mass of O, H1, H2 (the hydrogens at the oxygen's image)
// moves to c + (com - c) s and every site of the molecule moves with it, so
// the rigid geometry (and the M site) is kept
__global__ void k_scale_mol(const MolArgs A, double3 c, double s) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= A.nmol) return;
    const int4 ix = mol_sites(A, m);
    const Box &b = A.box;
    const float4 o = A.xs[ix.x], h1 = A.xs[ix.y], h2 = A.xs[ix.z];
    auto mi = [&](double d, double L, double iL) { return d - L * rint(d * iL); };
    const double3 d1 = make_double3(mi((double)h1.x - o.x, b.Ld.x, b.invLd.x), mi((double)h1.y - o.y, b.Ld.y, b.invLd.y),
                                    mi((double)h1.z - o.z, b.Ld.z, b.invLd.z));
    const double3 d2 = make_double3(mi((double)h2.x - o.x, b.Ld.x, b.invLd.x), mi((double)h2.y - o.y, b.Ld.y, b.invLd.y),
                                    mi((double)h2.z - o.z, b.Ld.z, b.invLd.z));
    const double wH = A.rc.wH;
    const double3 com = make_double3(o.x + (d1.x + d2.x) * wH, o.y + (d1.y + d2.y) * wH, o.z + (d1.z + d2.z) * wH);
    const double3 sh = make_double3((c.x + (com.x - c.x) * s) - com.x, (c.y + (com.y - c.y) * s) - com.y,
                                    (c.z + (com.z - c.z) * s) - com.z);
    const int id4[4] = {ix.x, ix.y, ix.z, ix.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (id4[k] < 0) continue;
        float4 x = A.xs[id4[k]];
        x.x = (float)((double)x.x + sh.x);
        x.y = (float)((double)x.y + sh.y);
        x.z = (float)((double)x.z + sh.z);
        A.xs[id4[k]] = x;
    }
}
}  // namespace

// Mod::scaleSystem (Mod.cu:301-330) on the device positions, about the
// centre of the current box (which the caller then scales): free atoms
// scaled, rigid molecules moved with their centres of mass
int scale_positions(State &s, double sc) {
    const double3 c = make_double3(s.box.lod.x + 0.5 * s.box.Ld.x, s.box.lod.y + 0.5 * s.box.Ld.y,
                                   s.box.lod.z + 0.5 * s.box.Ld.z);
    FixRigid *r = s.rigidFix();
    const int n = s.gpd.n;
    if (has_free_atoms(s)) {
        k_scale_free<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.xs.p, s.gpd.ids.p, r ? rigid_flags(s) : nullptr,
                                                           c, sc);
        MDX_LAUNCHED();
    }
    if (r && !r->mol_ids.empty()) {
        MolArgs A = mol_args(s, *r);
        A.slots = s.mf.on ? 1 : 0;
        k_scale_mol<<<(A.nmol + 255) / 256, 256, 0, s.stream>>>(A, c, sc);
        MDX_LAUNCHED();
    }
    MDX_CUDA_TRY(cudaGetLastError());
    return 0;
}

int batch_rigid_maps(Batch &b) {
    MolArgs A;
    if (int e = batch_sizing(b, &A)) return e;
    k_rigid_maps<<<dim3((A.nmol + 255) / 256, (unsigned)b.reps.size()), 256, 0, b.stream>>>(
        A, reinterpret_cast<const MolArgs *>(b.tab_first.p), 1);
    MDX_LAUNCHED();
    return 0;
}

int batch_first_half(Batch &b) {
    MolArgs A;
    if (int e = batch_sizing(b, &A)) return e;
    k_first_mol<true><<<dim3(A.nblk, (unsigned)b.reps.size()), kMolBlock, 0, b.stream>>>(
        A, reinterpret_cast<const MolArgs *>(b.tab_first.p));
    MDX_LAUNCHED();
    return 0;
}

int batch_second_half(Batch &b, bool with_e3b) {
    MolArgs A;
    if (int e = batch_sizing(b, &A)) return e;
    k_second_mol<<<dim3(A.nblk, (unsigned)b.reps.size()), kMolBlock, 0, b.stream>>>(
        A, reinterpret_cast<const MolArgs *>(with_e3b ? b.tab_second.p : b.tab_first.p));
    MDX_LAUNCHED();
    return 0;
}

}  // namespace mdx
