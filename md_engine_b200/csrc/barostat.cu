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
