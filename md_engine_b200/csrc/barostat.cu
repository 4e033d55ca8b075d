// Pressure control: FixPressureBerendsen (src/Fixes/FixPressureBerendsen.cu)
// and what a box change drags along (Mod::scaleSystem, Mod.cu:301-330;
// FixChargeEwald::handleBoundsChange, FixChargeEwald.cu:1200-1229; the
// neighbour grids).  Host-side control: the barostat reads the scalar
// pressure back after the step of each of its turns, as the reference's
// stepFinal does with its device synchronisation.
#include <algorithm>
#include <cmath>

#include "engine.hpp"

namespace mdx {

int pressure_now(State &s, double *pressure, double virial6[6]) {
    const int n = s.gpd.n;
    DBuf<float4> keep;
    if (int e = keep.alloc(n)) return e;
    MDX_CUDA_TRY(cudaMemcpyAsync(keep.p, s.gpd.fs.p, (size_t)n * sizeof(float4), cudaMemcpyDeviceToDevice, s.stream));
    if (int e = s.computeForces(1)) return e;
    double v6[6];
    if (int e = virial_sum(s, v6)) return e;
    double mv2 = 0.0;
    if (int e = kinetic_sum(s, &mv2)) return e;
    MDX_CUDA_TRY(cudaMemcpyAsync(s.gpd.fs.p, keep.p, (size_t)n * sizeof(float4), cudaMemcpyDeviceToDevice, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    if (int e = s.checkStatus()) return e;
    const double V = s.box.Ld.x * s.box.Ld.y * s.box.Ld.z;
    // DataComputerPressure::computeScalar_CPU: (sum m v^2 + trace W) / 3V
    *pressure = (mv2 * s.units.mvv_to_eng + v6[0] + v6[1] + v6[2]) / (3.0 * V) * s.units.nktv_to_press;
    if (virial6)
        for (int c = 0; c < 6; c++) virial6[c] = v6[c];
    return 0;
}

int box_rescale(State &s, double sc) {
    if (!(sc > 0.0) || !std::isfinite(sc)) {
        set_error(MDX_ERR_ARG, "box scale factor must be positive and finite (got %g)", sc);
        return MDX_ERR_ARG;
    }
    // positions first, about the centre of the old box
    if (int e = scale_positions(s, sc)) return e;
    // BoundsGPU::scale: the box about its centre
    for (int d = 0; d < 3; d++) {
        const double c = 0.5 * (s.lo[d] + s.hi[d]);
        const double h = 0.5 * (s.hi[d] - s.lo[d]) * sc;
        s.lo[d] = c - h;
        s.hi[d] = c + h;
    }
    s.setBox();
    s.box_gen++;
    if (FixChargeEwald *ew = s.ewaldFix())
        if (int e = ew->boxChanged()) return e;
    if (int e = nlist_box_changed(s)) return e;
    // the positions moved by up to (sc - 1) L / 2 and the cells changed: a
    // fresh list (sorted, wrapped into the new box)
    if (int e = nlist_rebuild(s, true, false)) return e;
    MDX_CUDA_TRY(cudaGetLastError());
    return 0;
}

int barostat_apply(State &s, FixPressureBerendsen &b) {
    double p = 0.0;
    if (int e = pressure_now(s, &p, nullptr)) return e;
    // FixPressureBerendsen::stepFinal (FixPressureBerendsen.cu:26-51)
    double dil = std::pow(1.0 - s.dt / b.period * (b.pressure - p) / b.bulkModulus, 1.0 / 3.0);
    if (!std::isfinite(dil)) dil = 1.0 - b.maxDilation;  // a negative base: compress at the limit
    dil = std::min(std::max(dil, 1.0 - b.maxDilation), 1.0 + b.maxDilation);
    b.lastPressure = p;
    b.lastDilation = dil;
    b.applications++;
    return box_rescale(s, dil);
}

int64_t barostat_next(State &s, int64_t t) {
    FixPressureBerendsen *b = s.barostatFix();
    if (!b || b->applyEvery <= 0) return -1;
    const int64_t W = b->applyEvery;
    return ((t + W - 1) / W) * W;
}


// ---------------------------------------------------------------- MTK NPT
namespace {
constexpr float kMassless = 1.0e18f;  // 1/m of a massless site (vs.w above it)

// nve_v (IntegratorVerlet.cu:23-42): v += dtf f / m; the forces are kept for
// the barostat's additive velocity term
__global__ void k_mtk_kick(int n, float4 *__restrict__ vs, const float4 *__restrict__ fs, float dtf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = vs[i];
    if (v.w > kMassless) return;
    const float4 f = fs[i];
    const float s = dtf * v.w;
    v.x += s * f.x;
    v.y += s * f.y;
    v.z += s * f.z;
    vs[i] = v;
}

// nve_x (IntegratorVerlet.cu:44-61): x += dt v
__global__ void k_mtk_drift(int n, float4 *__restrict__ xs, const float4 *__restrict__ vs, float dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = vs[i];
    if (v.w > kMassless) return;
    float4 x = xs[i];
    x.x += dt * v.x;
    x.y += dt * v.y;
    x.z += dt * v.z;
    xs[i] = x;
}

// rescale_no_tags_cu (FixNoseHoover.cu:40-51)
__global__ void k_mtk_scale(int n, float4 *__restrict__ vs, float s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = vs[i];
    v.x *= s;
    v.y *= s;
    v.z *= s;
    vs[i] = v;
}

// barostat_vel_no_tags_cu (FixNoseHoover.cu:84-103): v = (v m + dtf f/m a) m
__global__ void k_mtk_baro_vel(int n, float4 *__restrict__ vs, const float4 *__restrict__ fs, float add,
                               float mult, float dtf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = vs[i];
    if (v.w > kMassless) return;
    const float4 f = fs[i];
    const float s = dtf * v.w * add;
    v.x = (v.x * mult + s * f.x) * mult;
    v.y = (v.y * mult + s * f.y) * mult;
    v.z = (v.z * mult + s * f.z) * mult;
    vs[i] = v;
}

struct Mtk {
    State &s;
    FixNoseHoover &nh;
    double kT() const { return s.units.boltz * nh.T; }
    int natoms() const { return (int)s.atoms.size(); }
    double ndf() const { return nh.h.ndf; }
    double volume() const { return s.box.Ld.x * s.box.Ld.y * s.box.Ld.z; }
    int launch_n() const { return s.gpd.n; }
    // calculateKineticEnergy (FixNoseHoover.cu:1044-1074): sum m v^2
    int kinetic(double *ke) {
        double mv2 = 0.0;
        if (int e = kinetic_sum(s, &mv2)) return e;
        *ke = mv2 * s.units.mvv_to_eng;
        return 0;
    }
    // DataComputerPressure's scalar pressure from the virials of the last
    // force evaluation and the kinetic sum ke
    int pressure(double ke, double *p) {
        double v6[6];
        if (int e = virial_sum(s, v6)) return e;
        *p = (ke + v6[0] + v6[1] + v6[2]) / (3.0 * volume()) * s.units.nktv_to_press;
        return 0;
    }
    // updateBarostatMasses (FixNoseHoover.cu:628-667), ISO
    void barostatMasses() {
        const double f = 1.0 / nh.ptau;
        for (int i = 0; i < 3; i++) nh.pressMass[i] = (ndf() + 3.0) * kT() / (f * f);
    }
    // updateBarostatThermalMasses (FixNoseHoover.cu:669-700)
    void barostatThermalMasses() {
        const double f = 1.0 / nh.ptau;
        nh.pThermMass[0] = 3.0 * 4.0 * kT() / (2.0 * f);
        for (int i = 1; i < kNHChain; i++) nh.pThermMass[i] = kT() / (f * f);
        for (int i = 1; i < kNHChain; i++)
            nh.pThermForce[i] = (nh.pThermMass[i - 1] * nh.pThermVel[i - 1] * nh.pThermVel[i - 1] - kT()) /
                                nh.pThermMass[i];
    }
    double keBarostat() const {
        double k = 0.0;
        for (int i = 0; i < 3; i++) k += nh.pressMass[i] * nh.pressVel[i] * nh.pressVel[i];
        return k;
    }
    // barostatThermostatIntegrate (FixNoseHoover.cu:702-793), one Yoshida
    // weight, one substep
    void barostatThermostat(bool stepInit) {
        const int N = kNHChain;
        double *v = nh.pThermVel, *F = nh.pThermForce, *M = nh.pThermMass;
        if (!stepInit) F[0] = (keBarostat() - kT()) / M[0];
        const double ts = s.dt, t2 = 0.5 * ts, t4 = 0.25 * ts, t8 = 0.125 * ts;
        v[N - 1] += t4 * F[N - 1];
        for (int k = N - 2; k > 0; --k) {
            const double pf = std::exp(-t8 * v[k + 1]);
            v[k] = (v[k] * pf + t4 * F[k]) * pf;
        }
        double pf = std::exp(-t8 * v[1]);
        v[0] = (v[0] * pf + t4 * F[0]) * pf;
        const double sc = std::exp(-t2 * v[0]);
        for (int i = 0; i < 3; i++) nh.pressVel[i] *= sc;
        v[0] *= pf;
        F[0] = (keBarostat() - kT()) / M[0];
        v[0] += t4 * F[0];
        v[0] *= pf;
        for (int k = 1; k < N - 1; ++k) {
            pf = std::exp(-t8 * v[k + 1]);
            v[k] *= pf;
            F[k] = (M[k - 1] * v[k - 1] * v[k - 1] - kT()) / M[k];
            v[k] += t4 * F[k];
            v[k] *= pf;
        }
        F[N - 1] = (M[N - 2] * v[N - 2] * v[N - 2] - kT()) / M[N - 1];
        v[N - 1] += t4 * F[N - 1];
    }
    // barostatVelocityIntegrate (FixNoseHoover.cu:868-943), ISO
    void barostatVelocity(double ke, double p) {
        const double tcur = ke / (ndf() * s.units.boltz);
        const double alpha = s.units.boltz * tcur * ndf() / (natoms() * 3.0);
        for (int i = 0; i < 3; i++) {
            const double G = alpha / nh.pressMass[i] +
                             (p - nh.pressure) * volume() / (nh.pressMass[i] * s.units.nktv_to_press);
            nh.pressVel[i] += G * s.dt * 0.5;
        }
    }
    // scaleVelocitiesBarostat (FixNoseHoover.cu:945-1015)
    int barostatVelocities() {
        const double alpha = (nh.pressVel[0] + nh.pressVel[1] + nh.pressVel[2]) / (3.0 * natoms());
        const double x = (nh.pressVel[0] + alpha) * s.dt * 0.25;
        const double x2 = x * x, x4 = x2 * x2, x6 = x4 * x2, x8 = x4 * x4;
        const double add = x2 / 6.0 + x4 / 120.0 + x6 / 5040.0 + x8 / 362880.0;
        const double mult = std::exp(-x);
        const int n = launch_n();
        k_mtk_baro_vel<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.vs.p, s.gpd.fs.p, (float)add, (float)mult,
                                                              (float)(0.5 * s.dt * s.units.ftm_to_v));
        MDX_LAUNCHED();
        return 0;
    }
    int thermostat(bool stepInit, double ke) {
        nh.h.ke = ke;
        nh.pendingScale *= nh_integrate(nh.h, stepInit);
        return 0;
    }
    int rescale() {
        if (nh.pendingScale == 1.0) return 0;
        const int n = launch_n();
        k_mtk_scale<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.vs.p, (float)nh.pendingScale);
        MDX_LAUNCHED();
        nh.pendingScale = 1.0;
        return 0;
    }
};
}  // namespace

int mtk_prepare(State &s, FixNoseHoover &nh) {
    if (s.rigidFix()) {
        set_error(MDX_ERR_UNSUPPORTED, "FixNoseHoover's barostat is implemented for systems without FixRigid "
                                       "(rigid water: FixPressureBerendsen)");
        return MDX_ERR_UNSUPPORTED;
    }
    if (s.barostatFix()) {
        set_error(MDX_ERR_UNSUPPORTED, "one barostat per state: FixNoseHoover's or FixPressureBerendsen");
        return MDX_ERR_UNSUPPORTED;
    }
    Mtk m{s, nh};
    // the virials of the current positions for the first stepInit
    if (int e = s.computeForces(1)) return e;
    double ke = 0.0;
    if (int e = m.kinetic(&ke)) return e;
    // the particle chain as prepareFinal sets it, its velocities those the
    // last run left (the device copy's "final" state)
    NHChain &c = nh.h;
    if (nh.d_chain.p) {
        NHChain fin;
        MDX_CUDA_TRY(cudaMemcpy(&fin, nh.d_chain.p + 1, sizeof(NHChain), cudaMemcpyDeviceToHost));
        for (int k = 0; k < kNHChain; k++) c.vel[k] = fin.vel[k];
    }
    int ndf = 0;
    for (auto &a : s.atoms) ndf += a.ndf;
    c.n = kNHChain;
    c.T = nh.T;
    c.freq = 1.0 / nh.tau;
    c.ndf = ndf;
    c.kB = s.units.boltz;
    c.dt = s.dt;
    c.mvv_to_eng = s.units.mvv_to_eng;
    c.ke = ke;
    c.mass[0] = c.ndf * c.kB * c.T / (c.freq * c.freq);
    for (int k = 1; k < c.n; k++) c.mass[k] = c.kB * c.T / (c.freq * c.freq);
    for (int k = 0; k < c.n; k++) c.inv_mass[k] = 1.0 / c.mass[k];
    c.force[0] = (c.ke - c.ndf * c.kB * c.T) / c.mass[0];
    for (int k = 1; k < c.n; k++) c.force[k] = (c.mass[k - 1] * c.vel[k - 1] * c.vel[k - 1] - c.kB * c.T) / c.mass[k];
    // the barostat variables restart at rest, as prepareFinal resets them
    for (int i = 0; i < 3; i++) nh.pressVel[i] = nh.pressMass[i] = 0.0;
    for (int k = 0; k < kNHChain; k++) nh.pThermVel[k] = nh.pThermForce[k] = nh.pThermMass[k] = 0.0;
    m.barostatMasses();
    m.barostatThermalMasses();
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    return s.checkStatus();
}

// the chain as a run leaves it, for the next run's prepareFinal
int mtk_finish(State &s, FixNoseHoover &nh) {
    // postRun (FixNoseHoover.cu:406-411) applies the scale still pending
    Mtk m{s, nh};
    if (int e = m.rescale()) return e;
    if (!nh.d_chain.p) {
        MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
        return 0;
    }
    NHChain pair[2] = {nh.h, nh.h};
    pair[0].scale = pair[1].scale = 1.0;
    MDX_CUDA_TRY(cudaMemcpyAsync(nh.d_chain.p, pair, sizeof(pair), cudaMemcpyHostToDevice, s.stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
    return 0;
}

int mtk_step(State &s, FixNoseHoover &nh) {
    Mtk m{s, nh};
    const int n = s.gpd.n;
    const float dtf = (float)(0.5 * s.dt * s.units.ftm_to_v);
    double ke = 0.0, p = 0.0;
    // stepInit (FixNoseHoover.cu:413-518)
    m.barostatMasses();
    m.barostatThermalMasses();
    m.barostatThermostat(true);
    if (int e = m.thermostat(true, nh.h.ke)) return e;
    if (int e = m.rescale()) return e;
    if (int e = m.kinetic(&ke)) return e;
    if (int e = m.pressure(ke, &p)) return e;
    m.barostatVelocity(ke, p);
    // nve_v, postNVE_V (barostat velocity scaling, rescaleVolume), nve_x
    k_mtk_kick<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.vs.p, s.gpd.fs.p, dtf);
    MDX_LAUNCHED();
    if (int e = m.barostatVelocities()) return e;
    if (int e = box_rescale(s, std::exp(nh.pressVel[0] * s.dt))) return e;
    k_mtk_drift<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.xs.p, s.gpd.vs.p, (float)s.dt);
    MDX_LAUNCHED();
    // force with virials, postForce
    if (int e = s.computeForces(1)) return e;
    k_mtk_kick<<<(n + 255) / 256, 256, 0, s.stream>>>(n, s.gpd.vs.p, s.gpd.fs.p, dtf);
    MDX_LAUNCHED();
    // stepFinal (FixNoseHoover.cu:544-605)
    if (int e = m.barostatVelocities()) return e;
    if (int e = m.kinetic(&ke)) return e;
    if (int e = m.pressure(ke, &p)) return e;
    nh.lastPressure = p;
    m.barostatVelocity(ke, p);
    if (int e = m.thermostat(false, ke)) return e;
    m.barostatMasses();
    m.barostatThermalMasses();
    m.barostatThermostat(false);
    MDX_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace mdx

using namespace mdx;

#define B_ARG(cond, msg)                   \
    do {                                   \
        if (!(cond)) {                     \
            set_error(MDX_ERR_ARG, "%s", msg); \
            return MDX_ERR_ARG;            \
        }                                  \
    } while (0)

extern "C" {

int mdx_fix_pressure_berendsen_create(mdx_state *st, const char *handle, double pressure, double period,
                                      int apply_every, mdx_fix **out) {
    B_ARG(st && handle && out, "null argument");
    B_ARG(period > 0.0, "period must be positive");
    B_ARG(apply_every > 0, "applyEvery must be positive");
    Fix *f = new FixPressureBerendsen(st->s, handle, pressure, period, apply_every);
    *out = new mdx_fix{f, st};
    return 0;
}

int mdx_fix_pressure_berendsen_set(mdx_fix *fix, const char *key, double value) {
    B_ARG(fix && key, "null argument");
    B_ARG(fix->f->kind == FixKind::Barostat, "not a FixPressureBerendsen");
    FixPressureBerendsen &b = *static_cast<FixPressureBerendsen *>(fix->f);
    const std::string k = key;
    if (k == "maxDilation") {
        // setParameters(maxDilation) (FixPressureBerendsen.cu:57-59)
        B_ARG(value > 0.0 && value < 1.0, "maxDilation must be in (0, 1)");
        b.maxDilation = value;
    } else if (k == "bulkModulus") {
        B_ARG(value > 0.0, "bulkModulus must be positive");
        b.bulkModulus = value;
    } else if (k == "pressure") {
        b.pressure = value;
    } else if (k == "period") {
        B_ARG(value > 0.0, "period must be positive");
        b.period = value;
    } else {
        set_error(MDX_ERR_ARG, "unknown FixPressureBerendsen key '%s'", key);
        return MDX_ERR_ARG;
    }
    return 0;
}

int mdx_fix_pressure_berendsen_get(mdx_fix *fix, const char *key, double *value) {
    B_ARG(fix && key && value, "null argument");
    B_ARG(fix->f->kind == FixKind::Barostat, "not a FixPressureBerendsen");
    const FixPressureBerendsen &b = *static_cast<FixPressureBerendsen *>(fix->f);
    const std::string k = key;
    if (k == "maxDilation") *value = b.maxDilation;
    else if (k == "bulkModulus") *value = b.bulkModulus;
    else if (k == "pressure") *value = b.pressure;
    else if (k == "period") *value = b.period;
    else if (k == "lastPressure") *value = b.lastPressure;
    else if (k == "lastDilation") *value = b.lastDilation;
    else if (k == "applications") *value = (double)b.applications;
    else {
        set_error(MDX_ERR_ARG, "unknown FixPressureBerendsen key '%s'", key);
        return MDX_ERR_ARG;
    }
    return 0;
}

int mdx_state_scale_system(mdx_state *st, double scale) {
    B_ARG(st, "null state");
    State &s = *st->s;
    if (!s.prepared) {
        set_error(MDX_ERR_STATE, "state not prepared (call mdx_prepare or run first)");
        return MDX_ERR_STATE;
    }
    try {
        if (int e = box_rescale(s, scale)) return e;
        MDX_CUDA_TRY(cudaStreamSynchronize(s.stream));
        return s.checkStatus();
    } catch (const std::exception &ex) {
        set_error(MDX_ERR_STATE, "exception: %s", ex.what());
        return MDX_ERR_STATE;
    }
}

}  // extern "C"
