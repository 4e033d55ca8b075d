// Host-side State / fixes: parameter tables, upload/download, run
// preparation (State::prepareForRun, State.cpp:562-647; Integrator::
// basicPrepare / prepareFixes / prepareFinal, Integrator.cu:142-219).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>

#include "engine.hpp"

namespace mdx {

uint64_t g_launches = 0;

int high_priority() {
    static int prio = 1;  // not yet read
    if (prio == 1) {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) greatest = 0;
        prio = greatest;
    }
    return prio;
}

static thread_local char g_err[1024] = "";
void set_error(int code, const char *fmt, ...) {
    (void)code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
const char *last_error() { return g_err; }

// ---------------------------------------------------------------- State
int num_sms() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
        cache[dev] = n;
    }
    return cache[dev];
}

State::State() {
    units.setLJ();
}

State::~State() {
    if (h_status) cudaFreeHost(h_status);
    for (int k = 0; k < 3; k++) {
        if (side[k]) cudaStreamDestroy(side[k]);
        if (ev_join[k]) cudaEventDestroy(ev_join[k]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_sorted) cudaEventDestroy(ev_sorted);
    if (stream && own_stream) cudaStreamDestroy(stream);
}

int State::typeFromHandle(const std::string &h) const {
    for (size_t i = 0; i < species.size(); i++)
        if (species[i].handle == h) return (int)i;
    return -1;
}

void State::setBox() {
    box.lod = make_double3(lo[0], lo[1], lo[2]);
    box.Ld = make_double3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    box.invLd = make_double3(1.0 / box.Ld.x, 1.0 / box.Ld.y, 1.0 / box.Ld.z);
    box.lo = make_float3((float)lo[0], (float)lo[1], (float)lo[2]);
    box.L = make_float3((float)box.Ld.x, (float)box.Ld.y, (float)box.Ld.z);
    box.invL = make_float3(1.0f / box.L.x, 1.0f / box.L.y, 1.0f / box.L.z);
}

double State::maxRCut() {
    // State::getMaxRCut (State.cpp:502-511), a float max over fixes' cutoffs
    float m = (float)rCut;
    for (Fix *f : fixes)
        for (double x : f->getRCuts()) m = std::fmax(m, (float)x);
    return m;
}

FixPair *State::pairFix() {
    for (Fix *f : fixes)
        if (f->kind == FixKind::Pair) return static_cast<FixPair *>(f);
    return nullptr;
}
FixChargeEwald *State::ewaldFix() {
    for (Fix *f : fixes)
        if (f->kind == FixKind::ChargeEwald) return static_cast<FixChargeEwald *>(f);
    return nullptr;
}
FixChargePairDSF *State::dsfFix() {
    for (Fix *f : fixes)
        if (f->kind == FixKind::ChargeDSF) return static_cast<FixChargePairDSF *>(f);
    return nullptr;
}
FixE3B *State::e3bFix() {
    for (Fix *f : fixes)
        if (f->kind == FixKind::E3B) return static_cast<FixE3B *>(f);
    return nullptr;
}
FixRigid *State::rigidFix() {
    for (Fix *f : fixes)
        if (f->kind == FixKind::Rigid) return static_cast<FixRigid *>(f);
    return nullptr;
}
FixPressureBerendsen *State::barostatFix() {
    for (Fix *f : fixes)
        if (f->kind == FixKind::Barostat) return static_cast<FixPressureBerendsen *>(f);
    return nullptr;
}
FixNoseHoover *State::nhFix() {
    for (Fix *f : fixes)
        if (f->kind == FixKind::NoseHoover) return static_cast<FixNoseHoover *>(f);
    return nullptr;
}

// State::copyAtomDataToGPU (State.cpp:529-610): type bits in xs.w, 1/m in
// vs.w (INVMASSLESS for massless sites), group tag bits in fs.w
int State::upload() {
    const int n = (int)atoms.size();
    if (device < 0) MDX_CUDA_TRY(cudaGetDevice(&device));
    if (!stream) {
        MDX_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        own_stream = true;
    }
    for (int k = 0; k < 3; k++) {
        if (!side[k]) MDX_CUDA_TRY(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
        if (!ev_join[k]) MDX_CUDA_TRY(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
    }
    if (!ev_fork) MDX_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    if (!ev_sorted) MDX_CUDA_TRY(cudaEventCreateWithFlags(&ev_sorted, cudaEventDisableTiming));
    if (!h_status) MDX_CUDA_TRY(cudaMallocHost(&h_status, sizeof(DeviceStatus)));
    if (int e = d_status.alloc(1)) return e;
    MDX_CUDA_TRY(cudaMemset(d_status.p, 0, sizeof(DeviceStatus)));
    DeviceStatus init{};
    init.turn = turn;
    MDX_CUDA_TRY(cudaMemcpy(d_status.p, &init, sizeof(init), cudaMemcpyHostToDevice));
    GPUData &d = gpd;
    d.n = n;
    for (DBuf<float4> *b : {&d.xs, &d.vs, &d.fs, &d.xs_alt, &d.vs_alt, &d.fs_alt, &d.xs_last_build})
        if (int e = b->alloc(n)) return e;
    if (int e = d.qs.alloc(n)) return e;
    if (int e = d.qs_alt.alloc(n)) return e;
    if (int e = d.ids.alloc(n)) return e;
    if (int e = d.ids_alt.alloc(n)) return e;
    if (int e = d.idToIdx.alloc(n)) return e;
    if (int e = d.virials.alloc(6 * (size_t)n)) return e;
    if (int e = red_counter.alloc(1)) return e;
    if (int e = red_out.alloc(4)) return e;
    if (int e = e_site.alloc(n)) return e;
    if (int e = e_sum.alloc(1)) return e;
    MDX_CUDA_TRY(cudaMemset(red_counter.p, 0, sizeof(unsigned int)));
    MDX_CUDA_TRY(cudaMemset(d.virials.p, 0, 6 * (size_t)n * sizeof(float)));
    std::vector<float4> xs(n), vs(n), fs(n);
    std::vector<float> qs(n);
    std::vector<uint32_t> ids(n);
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) {
        const HostAtom &a = atoms[i];
        float tbits;
        std::memcpy(&tbits, &a.type, sizeof(float));
        xs[i] = make_float4((float)a.pos[0], (float)a.pos[1], (float)a.pos[2], tbits);
        float im = a.mass == 0.0 ? kInvMassless : (float)(1.0 / a.mass);
        vs[i] = make_float4((float)a.vel[0], (float)a.vel[1], (float)a.vel[2], im);
        float gbits;
        std::memcpy(&gbits, &a.groupTag, sizeof(float));
        fs[i] = make_float4((float)a.force[0], (float)a.force[1], (float)a.force[2], gbits);
        qs[i] = (float)a.q;
        ids[i] = (uint32_t)i;
        idx[i] = i;
    }
    MDX_CUDA_TRY(cudaMemcpy(d.xs.p, xs.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(d.vs.p, vs.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(d.fs.p, fs.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(d.xs_last_build.p, xs.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(d.qs.p, qs.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(d.ids.p, ids.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
    MDX_CUDA_TRY(cudaMemcpy(d.idToIdx.p, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    uploaded = true;
    return 0;
}

// device -> host atoms, back in id order
int State::download() {
    if (!uploaded) return 0;
    const int n = gpd.n;
    std::vector<float4> xs(n), vs(n), fs(n);
    std::vector<uint32_t> ids(n);
    MDX_CUDA_TRY(cudaStreamSynchronize(stream));
    MDX_CUDA_TRY(cudaMemcpy(xs.data(), gpd.xs.p, n * sizeof(float4), cudaMemcpyDeviceToHost));
    MDX_CUDA_TRY(cudaMemcpy(vs.data(), gpd.vs.p, n * sizeof(float4), cudaMemcpyDeviceToHost));
    MDX_CUDA_TRY(cudaMemcpy(fs.data(), gpd.fs.p, n * sizeof(float4), cudaMemcpyDeviceToHost));
    MDX_CUDA_TRY(cudaMemcpy(ids.data(), gpd.ids.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    DeviceStatus st;
    MDX_CUDA_TRY(cudaMemcpy(&st, d_status.p, sizeof(st), cudaMemcpyDeviceToHost));
    turn = st.turn;
    for (int i = 0; i < n; i++) {
        HostAtom &a = atoms[ids[i]];
        a.pos[0] = xs[i].x; a.pos[1] = xs[i].y; a.pos[2] = xs[i].z;
        a.vel[0] = vs[i].x; a.vel[1] = vs[i].y; a.vel[2] = vs[i].z;
        a.force[0] = fs[i].x; a.force[1] = fs[i].y; a.force[2] = fs[i].z;
    }
    return 0;
}

int State::checkStatus() {
    MDX_CUDA_TRY(cudaMemcpyAsync(h_status, d_status.p, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, stream));
    MDX_CUDA_TRY(cudaStreamSynchronize(stream));
    const uint32_t b = h_status->bits;
    if (b & kStatusNlistOverflow) {
        if (mf.on)
            set_error(MDX_ERR_OVERFLOW, "molecule-pair list capacity %d exceeded (max count %u)", mf.cap,
                      h_status->max_mol_neighbors);
        else
            set_error(MDX_ERR_OVERFLOW, "neighbour list capacity %d exceeded (max count %u)", grid.cap,
                      h_status->max_neighbors);
        return MDX_ERR_OVERFLOW;
    }
    if (b & kStatusMolOverflow) {
        set_error(MDX_ERR_OVERFLOW, "E3B molecule list capacity exceeded (max count %u)", h_status->max_mol_neighbors);
        return MDX_ERR_OVERFLOW;
    }
    if (b & kStatusSettleFail) {
        set_error(MDX_ERR_NUMERIC, "SETTLE failed: cos^2 <= 0 (degenerate water triangle)");
        return MDX_ERR_NUMERIC;
    }
    if (b & kStatusConstraint) {
        set_error(MDX_ERR_NUMERIC, "rigid-water bond length drifted beyond 1e-3 A (validateConstraints)");
        return MDX_ERR_NUMERIC;
    }
    return 0;
}

int State::buildNeighborList(bool force) { return nlist_rebuild(*this, force, false); }

// IntegratorUtil::force (IntegratorUtil.cpp:15-30): zero forces, then every
// fix's compute in fix order (pair fixes first, orderPreference -1)
int State::computeForces(int virialMode) {
    if (int e = zero_forces(*this)) return e;
    std::vector<Fix *> order(fixes.begin(), fixes.end());
    std::stable_sort(order.begin(), order.end(),
                     [](Fix *a, Fix *b) { return a->orderPreference < b->orderPreference; });
    for (Fix *f : order)
        if (int e = f->compute(virialMode)) return e;
    MDX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// run preparation in the reference order (IntegratorVerlet::run, :649-684)
int State::prepare() {
    if (!bounds_set) {
        set_error(MDX_ERR_STATE, "state.bounds not set");
        return MDX_ERR_STATE;
    }
    if (atoms.empty()) {
        set_error(MDX_ERR_STATE, "no atoms");
        return MDX_ERR_STATE;
    }
    if (dt <= 0) {
        set_error(MDX_ERR_STATE, "dt must be positive");
        return MDX_ERR_STATE;
    }
    setBox();
    // charge offload (State::handleChargeOffloading, State.cpp:648-660)
    requiresCharges = false;
    FixPair *pf = pairFix();
    FixChargeEwald *ew = ewaldFix();
    FixChargePairDSF *dsf = dsfFix();
    if (ew && dsf) {
        set_error(MDX_ERR_UNSUPPORTED, "one charge fix per state: FixChargeEwald or FixChargePairDSF");
        return MDX_ERR_UNSUPPORTED;
    }
    if (ew) {
        requiresCharges = true;
        if (ew->r_cut < 0) ew->r_cut = rCut;
    }
    if (dsf) requiresCharges = true;
    if (pf) {
        pf->chargeFix = ew;
        pf->dsfFix = dsf;
        pf->chargeRCut = ew ? ew->r_cut : (dsf ? dsf->r_cut : 0.0);
        if (ew) ew->offloaded = true;
    }
    // reset NDF (Atom ndf 3, FixRigid::assignNDF sets 2 / 0)
    for (auto &a : atoms) a.ndf = 3;
    if (FixRigid *r = rigidFix()) {
        if (int e = r->setConsts()) return e;
        for (auto &m : r->mol_ids) {
            atoms[m.x].ndf = atoms[m.y].ndf = atoms[m.z].ndf = 2;
            if (m.w >= 0) atoms[m.w].ndf = 0;
        }
    }
    if (int e = upload()) return e;
    if (int e = nlist_init(*this)) return e;
    {
        // reduction partials for the per-step kinetic sums (allocated here, never
        // while a graph is being captured)
        const int ab = (gpd.n + 255) / 256;
        const int mb = rigidFix() ? ((int)rigidFix()->mol_ids.size() + kMolBlock - 1) / kMolBlock : 0;
        if (int e = red_partials.alloc(ab + mb + 8)) return e;
        if (int e = rigid_flags_prepare(*this)) return e;
    }
    // prepareFixes(false): pair, charge, E3B
    for (Fix *f : fixes) {
        if (f->kind == FixKind::Rigid || f->kind == FixKind::NoseHoover) continue;
        if (int e = f->prepareForRun()) return e;
    }
    if (FixRigid *r = rigidFix()) {
        if (int e = r->prepareForRun()) return e;  // device molecule arrays
    }
    if (int e = nlist_set_interactions(*this)) return e;
    if (int e = molform_init(*this)) return e;
    // first build (GridGPU::periodicBoundaryConditions(-1, true), Integrator.cu:216)
    if (int e = nlist_rebuild(*this, true, false)) return e;
    if (int e = computeForces(0)) return e;  // forceInitial
    if (FixRigid *r = rigidFix()) {
        // prepareFixes(true): SETTLE the initial configuration, M sites,
        // velocity constraints, COM velocity removal.  As in the reference
        // (FixRigid.cu:1825-1834 distributes M-site virials only), the initial
        // M-site force is not moved onto O/H before the first half kick.
        if (int e = rigid_prepare(*this, *r)) return e;
    }
    if (FixNoseHoover *nh = nhFix()) {
        if (int e = nh_prepare(*this, *nh)) return e;
    }
    MDX_CUDA_TRY(cudaStreamSynchronize(stream));
    MDX_CUDA_TRY(cudaGetLastError());
    if (int e = checkStatus()) return e;
    prepared = true;
    return 0;
}

// ---------------------------------------------------------------- FixPair
static const char *pair_type_name(int kind) {
    switch (kind) {
        case 1: return "LJCut";
        case 2: return "LJCutWCA";
        case 3: return "LJCutFS";
        case 4: return "LJCHARMM";
        default: return "TICG";
    }
}

FixPair::FixPair(State *s, std::string h, int kind, std::string mix)
    : Fix(s, h, "all", pair_type_name(kind), FixKind::Pair), lj_kind(kind), mixing(mix) {
    orderPreference = -1;  // FixPair.h:34
    // the parameter handles each style's constructor initializes
    if (kind == 5) {
        params["C"] = {};
    } else {
        params["eps"] = {};
        params["sig"] = {};
    }
    if (kind == 4) {
        params["eps14"] = {};
        params["sig14"] = {};
    }
    params["rCut"] = {};
}

bool FixPair::pairActive(int a, int b) const {
    const int nt = (int)state->species.size();
    const size_t nt2 = (size_t)nt * nt, k = (size_t)a * nt + b;
    if (h_params.size() != (size_t)nparam() * nt2) return true;
    if (h_params[nt2 + k] != 0.f) return true;  // 24 eps, or C (TICG)
    return lj_kind == 4 && h_params[3 * nt2 + k] != 0.f;  // 24 eps14
}

// ---------------------------------------------------------------- FixChargePairDSF
FixChargePairDSF::FixChargePairDSF(State *s, std::string h, std::string g)
    : Fix(s, h, g, "ChargePairDSF", FixKind::ChargeDSF) {
    requiresCharges = true;
    setParameters(0.25, 9.0);  // the constructor's defaults (FixChargePairDSF.cu)
}

// FixChargePairDSF::setParameters: A = 2 alpha / sqrt(pi),
// shift = erfc(alpha rc) / rc^2 + A exp(-alpha^2 rc^2) / rc
void FixChargePairDSF::setParameters(double alpha_, double r_cut_) {
    alpha = alpha_;
    r_cut = r_cut_;
    A = 2.0 / std::sqrt(M_PI) * alpha;
    shift = std::erfc(alpha * r_cut) / (r_cut * r_cut) + A * std::exp(-alpha * alpha * r_cut * r_cut) / r_cut;
}

int FixChargePairDSF::prepareForRun() {
    if (!state->pairFix()) {
        set_error(MDX_ERR_UNSUPPORTED, "FixChargePairDSF is evaluated inside a pair fix's kernel: add a pair fix");
        return MDX_ERR_UNSUPPORTED;
    }
    prepared = true;
    return 0;
}

void FixPair::ensureSize() {
    const size_t nt = state->species.size();
    for (auto &kv : params) {
        std::vector<double> &v = kv.second;
        const size_t old = (size_t)std::llround(std::sqrt((double)v.size()));
        if (old == nt && v.size() == nt * nt) continue;
        std::vector<double> nv(nt * nt, std::numeric_limits<double>::quiet_NaN());
        for (size_t i = 0; i < old && i < nt; i++)
            for (size_t j = 0; j < old && j < nt; j++) nv[i * nt + j] = v[i * old + j];
        v.swap(nv);
    }
}

int FixPair::setParameter(const std::string &param, int a, int b, double v) {
    if (params.find(param) == params.end()) {
        set_error(MDX_ERR_ARG, "unknown pair parameter '%s'", param.c_str());
        return MDX_ERR_ARG;
    }
    const int nt = (int)state->species.size();
    if (a < 0 || b < 0 || a >= nt || b >= nt) {
        set_error(MDX_ERR_ARG, "invalid atom types for setParameter");
        return MDX_ERR_ARG;
    }
    ensureSize();
    params[param][a * nt + b] = v;
    params[param][b * nt + a] = v;
    return 0;
}

// prepareParameters (FixPair.cpp:13-63) with each style's lambdas: FixLJCut
// (FixLJCut.cu:83-122), FixWCA (FixWCA.cu:60-106), FixLJCutFS
// (FixLJCutFS.cu:84-130), FixLJCHARMM (FixLJCHARMM.cu:113-180), FixTICG
// (FixTICG.cu:68-83).  Off-diagonal entries left unset are mixed from the
// diagonal ones (eps geometric, sig geometric or arithmetic, rCut the larger
// one, the diagonal rCut defaulting to state.rCut); TICG mixes nothing
// (check_populate: every entry must be set).
int FixPair::prepareForRun() {
    State &s = *state;
    ensureSize();
    const int nt = (int)s.species.size();
    const size_t nt2 = (size_t)nt * nt;
    auto fill = [&](std::vector<double> v, bool geo, bool fillDiag, double diag) {
        if (fillDiag)
            for (int i = 0; i < nt; i++)
                if (std::isnan(v[i * nt + i])) v[i * nt + i] = diag;
        for (int i = 0; i < nt; i++)
            for (int j = 0; j < nt; j++)
                if (std::isnan(v[i * nt + j])) {
                    double a = v[i * nt + i], b = v[j * nt + j];
                    v[i * nt + j] = geo ? std::sqrt((float)a * (float)b) : ((float)a + (float)b) / 2.0;
                }
        return v;
    };
    auto fill_rcut = [&]() {
        // fillRCut = fmax(a, b), diagonal default state->rCut
        std::vector<double> rc = params["rCut"];
        for (int i = 0; i < nt; i++)
            if (std::isnan(rc[i * nt + i])) rc[i * nt + i] = (float)s.rCut;
        for (int i = 0; i < nt; i++)
            for (int j = 0; j < nt; j++)
                if (std::isnan(rc[i * nt + j])) rc[i * nt + j] = std::fmax((float)rc[i * nt + i], (float)rc[j * nt + j]);
        return rc;
    };
    auto all_set = [&](const std::vector<double> &v, const char *what) {
        for (size_t k = 0; k < nt2; k++)
            if (std::isnan(v[k])) {
                set_error(MDX_ERR_STATE, "pair parameter %s not set for every pair of species", what);
                return false;
            }
        return true;
    };
    h_params.assign((size_t)nparam() * nt2, 0.f);
    if (lj_kind == 5) {
        // TICG: {rCut^2, C}, no mixing
        const std::vector<double> &C = params["C"], &rc = params["rCut"];
        if (!all_set(C, "C") || !all_set(rc, "rCut")) return MDX_ERR_STATE;
        for (size_t k = 0; k < nt2; k++) {
            const float r = (float)rc[k];
            h_params[k] = r * r;
            h_params[nt2 + k] = (float)C[k];
        }
    } else {
        const double c14 = s.specialNeighborCoefs[2];
        if (lj_kind == 4) {
            // an unset 1-4 diagonal entry is the ordinary one times the 1-4
            // coefficient, for eps14 and for sig14 (FixLJCHARMM.cu:147-155)
            for (const char *h : {"eps14", "sig14"}) {
                std::vector<double> &v14 = params[h];
                const std::vector<double> &v = params[h[0] == 'e' ? "eps" : "sig"];
                for (int i = 0; i < nt; i++)
                    if (std::isnan(v14[i * nt + i])) v14[i * nt + i] = (float)v[i * nt + i] * (float)c14;
            }
        }
        std::vector<double> eps = fill(params["eps"], true, false, 0);
        std::vector<double> sig = fill(params["sig"], mixing != "arithmetic", false, 0);
        if (!all_set(eps, "eps") || !all_set(sig, "sig")) return MDX_ERR_STATE;
        std::vector<double> rc;
        if (lj_kind == 2) {
            rc.resize(nt2);
            for (size_t k = 0; k < nt2; k++) rc[k] = (float)sig[k] * (float)std::pow(2.0, 1.0 / 6.0);
        } else {
            rc = fill_rcut();
        }
        for (size_t k = 0; k < nt2; k++) {
            const float r = (float)rc[k];
            h_params[k] = r * r;                                    // processRCut
            h_params[nt2 + k] = 24.0f * (float)eps[k];              // processEps
            h_params[2 * nt2 + k] = (float)std::pow((float)sig[k], 6);  // processSig
        }
        if (lj_kind == 3) {
            // F(rCut): the unshifted LJ force magnitude at the pair's cutoff,
            // from its processed parameters (the table EvaluatorLJFS::force
            // reads as params[3]; see EvaluatorLJFS::forcePy, PairEvaluatorLJFS.cu)
            for (size_t k = 0; k < nt2; k++) {
                const float rc2 = h_params[k], eps24 = h_params[nt2 + k], sig6 = h_params[2 * nt2 + k];
                const float p1 = eps24 * 2.0f * sig6 * sig6, p2 = eps24 * sig6;
                const float r2inv = 1.0f / rc2, rinv = std::sqrt(r2inv);
                const float r6inv = r2inv * r2inv * r2inv;
                h_params[3 * nt2 + k] = r6inv * rinv * (p1 * r6inv - p2);
            }
        }
        if (lj_kind == 4) {
            std::vector<double> eps14 = fill(params["eps14"], true, false, 0);
            std::vector<double> sig14 = fill(params["sig14"], mixing != "arithmetic", false, 0);
            if (!all_set(eps14, "eps14") || !all_set(sig14, "sig14")) return MDX_ERR_STATE;
            for (size_t k = 0; k < nt2; k++) {
                h_params[3 * nt2 + k] = 24.0f * (float)eps14[k];
                h_params[4 * nt2 + k] = (float)std::pow((float)sig14[k], 6);
            }
        }
    }
    if (int e = d_params.alloc(h_params.size())) return e;
    MDX_CUDA_TRY(cudaMemcpy(d_params.p, h_params.data(), h_params.size() * sizeof(float), cudaMemcpyHostToDevice));
    prepared = true;
    return 0;
}

std::vector<double> FixPair::getRCuts() {
    // FixPair::getRCuts: the largest pair cutoff
    State &s = *state;
    const int nt = (int)s.species.size();
    double m = s.rCut;
    if (lj_kind == 2) {
        ensureSize();
        for (int k = 0; k < nt * nt; k++) {
            double sg = params["sig"][k];
            if (!std::isnan(sg)) m = std::max(m, sg * std::pow(2.0, 1.0 / 6.0));
        }
        return {m};
    }
    (void)nt;
    ensureSize();
    for (double v : params["rCut"])
        if (!std::isnan(v)) m = std::max(m, v);
    return {m};
}

int FixPair::compute(int virialMode) { return pair_launch(*state, *this, virialMode, true); }

// ---------------------------------------------------------------- FixRigid
FixRigid::FixRigid(State *s, std::string h, std::string st) : Fix(s, h, "all", "Rigid", FixKind::Rigid), style(st) {}

int FixRigid::createRigid(int o, int h1, int h2, int m) {
    State &s = *state;
    const int n = (int)s.atoms.size();
    if (o < 0 || h1 < 0 || h2 < 0 || o >= n || h1 >= n || h2 >= n || m >= n) {
        set_error(MDX_ERR_ARG, "createRigid: atom id out of range");
        return MDX_ERR_ARG;
    }
    // mass ordering check (FixRigid.cu:1580-1594)
    const double mo = s.atoms[o].mass, mh1 = s.atoms[h1].mass, mh2 = s.atoms[h2].mass;
    bool ordered = mo > mh1 && mo > mh2 && mh1 == mh2;
    if (m >= 0) ordered = ordered && mh1 > s.atoms[m].mass;
    if (!ordered) {
        set_error(MDX_ERR_ARG, "Ids in FixRigid::createRigid must be as O, H1, H2, M");
        return MDX_ERR_ARG;
    }
    if (m >= 0) foursite = true;
    else threesite = true;
    mol_ids.push_back(make_int4(o, h1, h2, m));
    return 0;
}

void FixRigid::getBonds(std::vector<std::pair<int, int>> &out) {
    for (auto &m : mol_ids) {
        out.push_back({m.x, m.y});
        out.push_back({m.x, m.z});
        out.push_back({m.y, m.z});
        if (m.w >= 0) out.push_back({m.x, m.w});
    }
}

// setStyleBondLengths, set_fixed_sides, populateRigidData (FixRigid.cu:1137-1436)
int FixRigid::setConsts() {
    State &s = *state;
    if (mol_ids.empty()) {
        set_error(MDX_ERR_STATE, "There needs to be at least one water in FixRigid");
        return MDX_ERR_STATE;
    }
    if (foursite && threesite) {
        set_error(MDX_ERR_UNSUPPORTED, "both 3-site and 4-site models in one FixRigid");
        return MDX_ERR_UNSUPPORTED;
    }
    if (s.units.type != MDX_UNITS_REAL) {
        set_error(MDX_ERR_UNSUPPORTED, "real units must be used for rigid water (FixRigid.cu:1425)");
        return MDX_ERR_UNSUPPORTED;
    }
    double r_OH, r_HH, r_OM = 0, gamma = 0;
    if (style == "TIP4P/2005") { r_OH = 0.9572; r_HH = 1.5139; r_OM = 0.1546; gamma = 0.73612446364836; }
    else if (style == "TIP4P") { r_OH = 0.9572; r_HH = 1.5139; r_OM = 0.15; gamma = 0.74397533; }
    else if (style == "TIP3P") { r_OH = 0.9572; r_HH = 1.5139; }
    else if (style == "SPC" || style == "SPC/E") { r_OH = 1.0; r_HH = 1.633; }
    else {
        set_error(MDX_ERR_ARG, "unsupported FixRigid style '%s'", style.c_str());
        return MDX_ERR_ARG;
    }
    if (foursite && r_OM == 0) {
        set_error(MDX_ERR_ARG, "style '%s' is a 3-site model but M sites were given", style.c_str());
        return MDX_ERR_ARG;
    }
    const double mO = s.atoms[mol_ids[0].x].mass, mH = s.atoms[mol_ids[0].y].mass;
    const double mW = mO + 2.0 * mH;
    rc.wO = mO / mW;
    rc.wH = mH / mW;
    rc.mO = mO;
    rc.mH = mH;
    rc.invmO = 1.0 / mO;
    rc.invmH = 1.0 / mH;
    rc.r_OH = r_OH;
    rc.r_HH = r_HH;
    rc.r_OM = r_OM;
    rc.gamma = gamma;
    rc.invOH = 1.0 / r_OH;
    rc.invHH = 1.0 / r_HH;
    rc.foursite = foursite ? 1 : 0;
    const double half_hh = 0.5 * r_HH;
    const double rab = std::sqrt(r_OH * r_OH - half_hh * half_hh);
    const double ht = std::atan(half_hh / rab);
    const double h1 = 1.5 * M_PI + ht, h2 = 1.5 * M_PI - ht;
    const double comy = (std::sin(h1) + std::sin(h2)) * r_OH * rc.wH;
    rc.ra = -comy;
    rc.rb = rab - rc.ra;
    rc.rc = half_hh;
    rc.inv2Rc = 1.0 / r_HH;
    // constraint matrix (populateRigidData) and its inverse times mO
    const double inv = mO / mH;
    double M[9];
    M[0] = 1.0 + inv;
    M[1] = 1.0 - 0.5 * r_HH * r_HH / (r_OH * r_OH);
    M[2] = inv * 0.5 * r_HH / r_OH;
    M[3] = M[1];
    M[4] = M[0];
    M[5] = M[2];
    M[6] = M[2];
    M[7] = M[5];
    M[8] = 2.0 * inv;
    const double det = M[0] * (M[4] * M[8] - M[5] * M[7]) - M[1] * (M[3] * M[8] - M[5] * M[6]) +
                       M[2] * (M[3] * M[7] - M[4] * M[6]);
    double I[9];
    I[0] = (M[4] * M[8] - M[5] * M[7]) / det;
    I[1] = (M[2] * M[7] - M[1] * M[8]) / det;
    I[2] = (M[1] * M[5] - M[2] * M[4]) / det;
    I[3] = (M[5] * M[6] - M[3] * M[8]) / det;
    I[4] = (M[0] * M[8] - M[2] * M[6]) / det;
    I[5] = (M[2] * M[3] - M[0] * M[5]) / det;
    I[6] = (M[3] * M[7] - M[4] * M[6]) / det;
    I[7] = (M[1] * M[6] - M[0] * M[7]) / det;
    I[8] = (M[0] * M[4] - M[1] * M[3]) / det;
    for (int k = 0; k < 9; k++) rc.Minv[k] = I[k] * mO;
    return 0;
}

int FixRigid::prepareForRun() {
    const int nmol = (int)mol_ids.size();
    if (int e = d_mol_ids.alloc(nmol)) return e;
    if (int e = d_mol_idx.alloc(nmol)) return e;
    MDX_CUDA_TRY(cudaMemcpy(d_mol_ids.p, mol_ids.data(), nmol * sizeof(int4), cudaMemcpyHostToDevice));
    prepared = true;
    return 0;
}

// ---------------------------------------------------------------- FixNoseHoover
FixNoseHoover::FixNoseHoover(State *s, std::string h, std::string g)
    : Fix(s, h, g, "NoseHoover", FixKind::NoseHoover) {
    orderPreference = 50;
}

int FixNoseHoover::setTemperature(double T_, double tau_) {
    if (T_ <= 0 || tau_ <= 0) {
        set_error(MDX_ERR_ARG, "temperature and time constant must be positive");
        return MDX_ERR_ARG;
    }
    T = T_;
    tau = tau_;
    return 0;
}

int FixNoseHoover::setPressure(const std::string &mode, double P, double tau_) {
    if (mode != "ISO") {
        set_error(MDX_ERR_UNSUPPORTED, "FixNoseHoover::setPressure: mode '%s' (this library implements ISO)",
                  mode.c_str());
        return MDX_ERR_UNSUPPORTED;
    }
    if (tau_ <= 0) {
        set_error(MDX_ERR_ARG, "pressure time constant must be positive");
        return MDX_ERR_ARG;
    }
    barostatting = true;
    pressure = P;
    ptau = tau_;
    return 0;
}

int FixNoseHoover::prepareFinal() { return nh_prepare(*state, *this); }

}  // namespace mdx
