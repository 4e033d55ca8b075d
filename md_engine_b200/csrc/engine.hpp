// C++ host side of the hot path: State / GPUData / GridGPU / Fix / Integrator,
// mirroring the reference's operator API (src/State.h, src/GPUData.h,
// src/GridGPU.h, src/Fixes/Fix.h, src/Integrators/IntegratorVerlet.h).
#pragma once
#include <cuda_bf16.h>
#include <cufft.h>

#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace mdx {

extern uint64_t g_launches;  // kernels launched by this library
// threads per block of the fused per-molecule step kernels: two warps, so a
// few thousand molecules spread over many SMs (each thread's FP64 SETTLE is a
// long dependent chain) with half as many block partials for the kinetic
// sum's last-block tail as one-warp blocks (measured +0.6 % per water step)
constexpr int kMolBlock = 64;
// lanes per molecule in the E3B list and kernels (the molecule list is laid
// out for teams of this size)
constexpr int kE3BTeam = 16;
#define MDX_LAUNCHED() (++::mdx::g_launches)

// Programmatic dependent launch for the kernels of the fused step: the kernel
// may be scheduled while its predecessor in the stream is still running (once
// every block of that one has called pdl_trigger()); it calls pdl_wait()
// before touching anything the predecessor writes, which returns when that
// grid has completed and its memory is visible.  A CUDA graph captured from
// such launches keeps them as programmatic edges, so consecutive kernels of a
// step no longer pay a full drain-and-launch gap.
// high: the launch also carries the device's greatest stream priority (the
// P3M chain, the critical path of a water step, beside the pair kernel),
// kept as a node priority by graphs instantiated with
// cudaGraphInstantiateFlagUseNodePriority
int high_priority();
// SMs of the current device (cached per device)
int num_sms();
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl_prio(bool high, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                   cudaStream_t st, Args... args) {
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    attr[1].id = cudaLaunchAttributePriority;
    attr[1].val.priority = high ? high_priority() : 0;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = high ? 2 : 1;
    MDX_LAUNCHED();
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    return launch_pdl_prio(false, kern, grid, block, smem, st, args...);
}

template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    bool own = true;  // false: a view into memory owned elsewhere (a pool)
    int alloc(size_t count) {
        if (count <= n && p) return 0;
        if (!own) {
            set_error(MDX_ERR_STATE, "buffer is a pool view of %zu elements; %zu requested", n, count);
            return MDX_ERR_STATE;
        }
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            n = 0;
            set_error(MDX_ERR_CUDA, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
            return MDX_ERR_CUDA;
        }
        n = count;
        return 0;
    }
    void release() {
        if (p && own) cudaFree(p);
        p = nullptr;
        n = 0;
        own = true;
    }
    void view(T *q, size_t count) {
        release();
        p = q;
        n = count;
        own = false;
    }
    ~DBuf() { release(); }
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
};

struct Units {  // src/Units.cpp:5-32
    int type = MDX_UNITS_LJ;
    double boltz = 1, hbar = 1, mvv_to_eng = 1, qqr_to_eng = 1, nktv_to_press = 1, ftm_to_v = 1;
    void setLJ() {
        type = MDX_UNITS_LJ;
        boltz = hbar = mvv_to_eng = qqr_to_eng = nktv_to_press = ftm_to_v = 1.0;
    }
    void setReal() {
        type = MDX_UNITS_REAL;
        boltz = 0.0019872067;
        hbar = 15.178728314015;
        mvv_to_eng = 48.88821291 * 48.88821291;
        nktv_to_press = 68568.415;
        qqr_to_eng = 332.06371;
        ftm_to_v = (double)(1.0f / (48.88821291 * 48.88821291));
    }
};

struct Species {
    std::string handle;
    double mass;
    int atomic_num;
};

struct HostAtom {
    double pos[3], vel[3], force[3];
    double mass, q;
    int type, ndf;
    uint32_t groupTag;
};

class State;
class Fix;
// configuration IO (WriteConfig.cpp, ReadConfig.cpp): host-only, in config_io.cu
struct ConfigWriter;
struct ConfigReader;
// the smallest turn >= t at which an active writer fires, or -1
int64_t config_next_write(const State &s, int64_t t);
// writes every active writer due at `turn` (state's host copy current)
int config_write_due(State &s, int64_t turn);
// a new fix's readFromRestart: parameters / molecules from the configuration
// the state's reader is on (no-op without one)
int config_fix_restart(State &s, Fix &f);
// the state is going away: its writers stop writing, its reader is freed
void config_state_detach(State &s);

// ---------------------------------------------------------------- GPUData
// Per-atom device streams (src/GPUData.h:18-28): xs (type bits in .w),
// vs (1/m in .w), fs (group tag bits in .w), ids, qs, idToIdx, virials.
// Streams are sorted by cell at each list rebuild; the *_alt buffers are
// the scatter targets, copied back so that captured graphs see fixed
// pointers.
struct GPUData {
    DBuf<float4> xs, vs, fs, xs_alt, vs_alt, fs_alt, xs_last_build;
    DBuf<float> qs, qs_alt;
    DBuf<uint32_t> ids, ids_alt;
    DBuf<int> idToIdx;
    DBuf<float> virials;  // 6 per atom
    int n = 0;
};

// ---------------------------------------------------------------- GridGPU
// Cell-binned neighbour list (src/GridGPU.h).  Layout: "team-interleaved
// ELL": atoms are grouped 32/team per warp; an atom's k-th entry lives at
// group*cap*(32/team) + (k/team)*32 + slot*team + k%team, so a warp's team
// lanes read 128 contiguous bytes per row.
struct GridGPU {
    int team = 8;        // threads per atom in build and force kernels
    int cap = 0;         // per-atom capacity (multiple of team)
    int3 ns{0, 0, 0};    // cells per dimension
    int m = 2;           // stencil half width in cells (cells >= cut/m)
    int home_group = 2;  // home atoms a warp of the list build tests at once
    float cut = 0.f;     // neighCut = rCut + padding (float, as GridGPU)
    float skin = 0.f;    // padding
    DBuf<uint32_t> cell_start, cell_count, cell_fill, block_sums;
    DBuf<int> cell_of;     // per atom (unsorted order)
    DBuf<int> perm_tmp, perm;  // sort scratch
    DBuf<uint32_t> counts; // per atom neighbour count (all pairs within cut)
    DBuf<uint32_t> counts_int;  // per atom count of pairs that can interact
    DBuf<uint32_t> nlist;  // entries: interacting ones from the front of the
                           // row, provably zero ones (no LJ, q_i q_j = 0) from the back
    DBuf<uint32_t> ljmask;  // per type: bit tj set when LJ/WCA eps(ti,tj) != 0
    bool partition = false; // rows are split as above
    bool part_q = false;    // charges take part in the split (Ewald active)
    DBuf<int> excl_start;  // by id
    DBuf<uint32_t> excl_ids;
    // per id: exclusion depth of the ids id-32 .. id+31 as two bit planes
    // (bit d of .x: depth bit 0 of id-32+d, .y: depth bit 1); excl_far[id]
    // is set when some exclusion of id lies outside that window
    DBuf<ulonglong2> excl_win;
    DBuf<uint8_t> excl_far;
    int max_excl = 0;
    bool have_excl = false;
    bool built = false;
    // host copies of the exclusion lists by id (start, id | depth << 30)
    std::vector<int> h_excl_start;
    std::vector<uint32_t> h_excl_ids;
};

// ---------------------------------------------------------------- MolForm
// Molecule form of the step for all-rigid four-site water: every atom in a
// FixRigid molecule, every molecule alike in site types, charges and
// exclusions, no exclusion between molecules.  The per-atom streams then hold
// molecule slot k's sites (O, H1, H2, M) at 4k .. 4k+3, slots ordered by the
// cell of their site 0 at each rebuild, and the pair kernel walks a
// molecule-pair list (site 0 within cut = pair cutoff + padding + 2 dmax,
// dmax bounding every site's distance from site 0) evaluating every site
// pair of a listed molecule pair from one 64-byte gather.  The pair set is
// unchanged: every site pair within the pair cutoff now is within the list
// radius of site 0 at the last build while no atom has moved more than half
// the padding.  The per-site list of the reference stays available (built on
// demand into the sort's alternate buffers for Grid.getNeighborList).
struct MolForm {
    bool on = false;
    int nmol = 0;
    int team = 32;      // lanes per molecule in the pair kernel (list layout)
    int cap = 0;        // entries per molecule row
    int3 ns{0, 0, 0};   // cells per dimension of the molecule grid
    int m = 2;          // stencil half width (cells >= cut / m)
    float cut = 0.f;    // list radius on site 0
    float far = 0.f;    // pair cutoff + 2 dmax: no site pair interacts beyond it
    float dmax = 0.f;
    int type[4] = {0, 0, 0, 0};
    float q[4] = {0.f, 0.f, 0.f, 0.f};
    int depth[16] = {0};  // exclusion depth of site pair (a, b) within a molecule
    DBuf<uint32_t> cell_start, cell_count, cell_fill;
    DBuf<int> cell_of, perm_tmp, perm;  // by molecule; perm[slot] = FixRigid molecule index
    DBuf<uint32_t> counts, list;       // molecule-pair list (slots), team layout
};

// ---------------------------------------------------------------- Fixes
enum class FixKind { Pair, ChargeEwald, ChargeDSF, E3B, Rigid, NoseHoover, Barostat };

class Fix {
   public:
    State *state;
    std::string handle, group, type;
    FixKind kind;
    int orderPreference = 0;
    bool prepared = false;
    bool active = false;
    bool requiresCharges = false;
    Fix(State *s, std::string h, std::string g, std::string t, FixKind k) : state(s), handle(h), group(g), type(t), kind(k) {}
    virtual ~Fix() {}
    // hooks of src/Fixes/Fix.h:79-281 (return 0 on success, MDX_ERR_* otherwise)
    virtual int prepareForRun() { prepared = true; return 0; }
    virtual int stepInit() { return 0; }
    virtual int postNVE_X() { return 0; }
    virtual int compute(int virialMode) { (void)virialMode; return 0; }
    virtual int preStepFinal() { return 0; }
    virtual int stepFinal() { return 0; }
    virtual int handleLocalData() { return 0; }
    virtual std::vector<double> getRCuts() { return {}; }
    virtual void getBonds(std::vector<std::pair<int, int>> &out) { (void)out; }
};

class FixChargeEwald;
class FixChargePairDSF;
class FixRigid;

// FixPair and its pair styles (src/Fixes/FixPair.cpp): 1 FixLJCut
// (FixLJCut.cu), 2 FixWCA (FixWCA.cu), 3 FixLJCutFS (FixLJCutFS.cu),
// 4 FixLJCHARMM (FixLJCHARMM.cu), 5 FixTICG (FixTICG.cu)
class FixPair : public Fix {
   public:
    int lj_kind;
    std::string mixing;
    // unprocessed per-type tables; NaN = unset (DEFAULT_FILL)
    std::map<std::string, std::vector<double>> params;
    // processed tables in the reference's paramOrder, nparam() x T x T:
    // {rCut^2, 24 eps, sig^6} (LJ/cut, WCA), + F(rCut) (LJCutFS),
    // + 24 eps14, sig14^6 (LJCHARMM), {rCut^2, C} (TICG)
    DBuf<float> d_params;
    std::vector<float> h_params;
    FixChargeEwald *chargeFix = nullptr;     // offloaded real-space Ewald (State.cpp:648-660)
    FixChargePairDSF *dsfFix = nullptr;      // offloaded damped shifted force charges
    double chargeRCut = 0;
    int nparam() const { return lj_kind == 3 ? 4 : (lj_kind == 4 ? 5 : (lj_kind == 5 ? 2 : 3)); }
    // whether the pair evaluator can give a non-zero force for types (a, b)
    bool pairActive(int a, int b) const;
    FixPair(State *s, std::string h, int kind, std::string mix);
    int setParameter(const std::string &param, int a, int b, double v);
    int prepareForRun() override;
    int compute(int virialMode) override;
    std::vector<double> getRCuts() override;
    void ensureSize();
};

class FixChargeEwald : public Fix {
   public:
    int3 sz{64, 64, 64};
    int order = 5;
    double r_cut = -1;
    double alpha = 0;
    double alpha_user = 0;
    bool offloaded = false;
    cufftHandle plan_r2c = 0, plan_c2r = 0;
    bool plans = false;
    DBuf<float> rho;        // real grid
    DBuf<float2> rho_k;     // half spectrum
    DBuf<float2> e_k;       // 3 half spectra
    DBuf<float> e_r;        // 3 real grids
    DBuf<float> green;      // half spectrum Green function
    DBuf<double> energy_acc;
    // own FFT path (cubic 32^3 / 64^3 meshes): field interleaved as float4
    bool own_fft = false;
    DBuf<double> vir_acc;  // reciprocal-space virial sum (6)
    DBuf<float4> e4;
    DBuf<float2> tw;        // W_32^k then W_64^k
    FixChargeEwald(State *s, std::string h, std::string g);
    ~FixChargeEwald() override;
    int setParameters(int nx, int ny, int nz, double rcut, int ord);
    int prepareForRun() override;
    int compute(int virialMode) override;
    std::vector<double> getRCuts() override { return {r_cut}; }
    double findAlpha();
    int computeGreen(cudaStream_t st);  // the influence function for the current box
    int boxChanged();                   // alpha and the Green function after a box change
    int spread(cudaStream_t st);   // zero + spread
    int solve(cudaStream_t st);    // FFT, E-field, inverse FFTs
    int gather(bool accumulate, cudaStream_t st);
    int gather_to(float4 *out, cudaStream_t st);  // reciprocal forces stored into out
    // molecule form of spread / gather_to (rigid water, own FFT)
    bool mol_form_ok(const FixRigid &r) const;
    int spread_mol(cudaStream_t st, const FixRigid &r);
    int gather_mol_to(float4 *out, cudaStream_t st, const FixRigid &r);
    DBuf<float4> f_recip;                         // per-step reciprocal forces (fused step)
};

// FixChargePairDSF (src/Fixes/FixChargePairDSF.cu): damped shifted force
// charges (Fennell & Gezelter, J. Chem. Phys. 124, 234104 (2006)), a pair
// term offloaded into the pair fix's kernel
class FixChargePairDSF : public Fix {
   public:
    double alpha = 0.25, r_cut = 9.0, A = 0, shift = 0;
    FixChargePairDSF(State *s, std::string h, std::string g);
    void setParameters(double alpha_, double r_cut_);
    int prepareForRun() override;
    std::vector<double> getRCuts() override { return {r_cut}; }
};

struct E3BParams {  // EvaluatorE3B (EvaluatorE3B.h:9-65), FixE3B.cu:515-593
    float rs, rf, E2, Ea, Eb, Ec, k2, k3;
    float rfminusrs_cubed_inv, rstimes3;
    float list_cut2;  // (rf + padding)^2, the reference's molecule-list radius
    float rmax;       // RMAX_E3B (ThreeBodyE3B.h:16)
};

// Learned surrogate of the E3B three-body forces (no reference counterpart):
// per-molecule local-frame features -> MLP (3 x 64 SiLU, BF16 operands, FP32
// accumulation) -> the three-body forces on O, H1, H2 in the molecule's frame.
struct E3BSurrogate {
    static constexpr int kIn = 128, kHid = 64, kOut = 16, kOutUsed = 9;
    // parameter blob (floats): W1 [kIn x kHid], b1, W2 [kHid x kHid], b2, W3, b3, W4 [kHid x kOut], b4
    static constexpr int kOffW1 = 0, kOffB1 = kIn * kHid, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
                         kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kHid, kOffW4 = kOffB3 + kHid,
                         kOffB4 = kOffW4 + kHid * kOut, kParams = kOffB4 + kOut;
    DBuf<float> w, grad, adam_m, adam_v;  // FP32 master weights, gradient, Adam moments
    DBuf<__nv_bfloat16> wb;               // BF16 copy used by every GEMM (same offsets)
    DBuf<float> mean, inv_std;            // feature standardisation
    float force_scale = 1.f;              // targets are local-frame forces / force_scale
    bool stats = false, trained = false, enabled = false;
    int64_t adam_t = 0;
    // dataset (raw features, local-frame exact three-body forces)
    DBuf<float> X, Y;
    size_t n = 0, cap = 0;
    // per-step scratch
    DBuf<__nv_bfloat16> feat;
    DBuf<float> raw;
    DBuf<float4> frame;
    DBuf<float4> fexact;
    // training scratch
    DBuf<__nv_bfloat16> xb, act[3], dz;
    DBuf<float> z[4], yb, da;
    DBuf<double> loss;
    int batch = 0;
};

class FixE3B : public Fix {
   public:
    std::string style;
    std::unique_ptr<E3BSurrogate> sur;
    std::vector<int4> mol_ids;
    E3BParams prm{};
    DBuf<int4> d_mol_ids, d_mol_idx;
    DBuf<int> d_mol_of_atom;  // by atom index, -1 if none (rebuilt with the list)
    DBuf<uint32_t> mcounts, mlist;  // molecule neighbour list (full, team layout)
    DBuf<uint32_t> ccounts, clist;  // per step: the forces pass's partners (mj > m within rmax)
    DBuf<float4> totals;
    DBuf<float4> f_side;  // per-step E3B forces when run beside the pair kernel
    bool side_ok = false; // molecules identical to FixRigid's, in the same order
    int mteam = 8, mcap = 0;
    FixE3B(State *s, std::string h, std::string st);
    int prepareForRun() override;
    int compute(int virialMode) override;
    int handleLocalData() override;
};

struct RigidConsts {  // FixRigidData (FixRigid.h:23-77)
    double ra, rb, rc, inv2Rc;
    double wO, wH, mO, mH, invmO, invmH;
    double r_OH, r_HH, r_OM, gamma;
    double invOH, invHH;
    double Minv[9];
    int foursite;
};

class FixRigid : public Fix {
   public:
    std::string style;
    std::vector<int4> mol_ids;
    RigidConsts rc{};
    DBuf<int4> d_mol_ids, d_mol_idx;
    DBuf<float4> xs0;  // previous constrained O,H1,H2 (stand-alone hook path)
    DBuf<uint32_t> d_bad;  // validateConstraints hook: molecules off their constraints
    bool foursite = false, threesite = false;
    FixRigid(State *s, std::string h, std::string st);
    int createRigid(int o, int h1, int h2, int m);
    int prepareForRun() override;
    void getBonds(std::vector<std::pair<int, int>> &out) override;
    int setConsts();
};

// FixPressureBerendsen (src/Fixes/FixPressureBerendsen.cu): every
// applyEvery turns, after the step, the scalar pressure P (DataComputerPressure)
// sets the box dilation (1 - dt / period (P0 - P) / bulkModulus)^(1/3),
// clamped to 1 +- maxDilation; atoms and molecules are scaled about the box
// centre (Mod::scaleSystem)
class FixPressureBerendsen : public Fix {
   public:
    double pressure, period;
    int applyEvery;
    double bulkModulus = 10.0;  // FixPressureBerendsen.cu:12 (as LAMMPS)
    double maxDilation = 1e-5;
    double lastPressure = 0.0, lastDilation = 1.0;
    int64_t applications = 0;
    FixPressureBerendsen(State *s, std::string h, double p, double per, int every)
        : Fix(s, h, "all", "Berendsen", FixKind::Barostat), pressure(p), period(per), applyEvery(every) {}
};
// scalar pressure (DataComputerPressure, FP64) from a virial-mode force
// evaluation at the current positions (the forces are kept); virial6 may be null
int pressure_now(State &s, double *pressure, double virial6[6]);
// Mod::scaleSystem on the device positions about the box centre
int scale_positions(State &s, double sc);
// the box scaled by sc about its centre, with everything that follows it:
// positions, the P3M splitting and Green function, the cell grids, a forced
// list rebuild
int box_rescale(State &s, double sc);
int nlist_box_changed(State &s);
// FixPressureBerendsen::stepFinal
int barostat_apply(State &s, FixPressureBerendsen &b);
// the smallest turn >= t at which the state's barostat fires, or -1
int64_t barostat_next(State &s, int64_t t);

constexpr int kNHChain = 10;  // chain links (FixNoseHoover's default chainLength)
struct NHChain {  // FixNoseHoover chain state (FixNoseHoover.h), FP64
    double vel[10], force[10], mass[10];
    double inv_mass[10];  // 1 / mass, set with mass
    double ke;       // sum m v^2 * mvv_to_eng
    double T, freq, ndf, kB, dt;
    double mvv_to_eng;
    int n;
    double scale;    // pending velocity scale for the next stepInit
    double last_ke;
};

class FixNoseHoover : public Fix {
   public:
    double T = 0, tau = 0;
    NHChain h{};
    DBuf<NHChain> d_chain;
    DBuf<double> partials;
    DBuf<unsigned int> counter;
    bool chain_on_device = false;
    // barostatting (setPressure("ISO", P, timeConstant), FixNoseHoover.cu:
    // 153-219): the MTK propagator of FixNoseHoover.cu:413-604 on the host in
    // FP64, as the reference runs it, with the box change, velocity scalings
    // and reductions on the device
    bool barostatting = false;
    double pressure = 0, ptau = 0;
    double pressVel[3] = {0, 0, 0}, pressMass[3] = {0, 0, 0};
    double pThermVel[kNHChain] = {}, pThermForce[kNHChain] = {}, pThermMass[kNHChain] = {};
    double pendingScale = 1.0;    // thermostat factors not yet applied to the velocities
    double lastPressure = 0.0;    // the instantaneous pressure of the last stepFinal
    FixNoseHoover(State *s, std::string h, std::string g);
    int setTemperature(double T_, double tau_);
    int setPressure(const std::string &mode, double P, double tau_);
    int prepareFinal();
};
// an NPT run with FixNoseHoover's barostat: initialisation (prepareFinal,
// FixNoseHoover.cu:240-404) and one step in the reference's hook order
double nh_integrate(NHChain &c, bool stepInit);  // thermostatIntegrate on a chain (FP64)
int mtk_prepare(State &s, FixNoseHoover &nh);
int mtk_step(State &s, FixNoseHoover &nh);
int mtk_finish(State &s, FixNoseHoover &nh);

// ---------------------------------------------------------------- State
class State {
   public:
    Units units;
    double rCut = -1, padding = 0.5, dt = 0.005;
    int64_t turn = 0;
    int periodicInterval = 50;
    int nThreadPerAtom = 0, nThreadPerBlock = 256;  // 0 = automatic team size
    // 0 automatic (molecule form when the system allows it), 1 per-site
    // (atom) form, 2 molecule form (an error at prepare when not allowed)
    int pairForm = 0;
    // molecule form: cap on the pair kernel's grid in blocks per SM (0
    // automatic, -1 uncapped: one warp per molecule); a capped grid strides
    // over the molecules and leaves every SM room for the P3M chain running
    // beside it
    int pairBlocksPerSM = 0;
    MolForm mf;
    // list build tunables, 0 = automatic: cells of >= cut/gridStencil (1..4),
    // home atoms tested at once per warp (2 or 4)
    int gridStencil = 0, gridHomeGroup = 0;
    float specialNeighborCoefs[3] = {0.f, 0.f, 0.5f};
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool bounds_set = false;
    std::vector<Species> species;
    std::vector<HostAtom> atoms;  // index == id
    std::vector<Fix *> fixes;     // active fixes in order
    Box box{};
    GPUData gpd;
    GridGPU grid;
    DBuf<DeviceStatus> d_status;
    DeviceStatus *h_status = nullptr;  // pinned
    DBuf<double> red_partials;
    DBuf<double> red_out;
    DBuf<unsigned int> red_counter;
    // per-site pair energies and their FP64 sum (energy evaluations outside
    // the step; sized at upload so that no evaluation allocates)
    DBuf<float> e_site;
    DBuf<double> e_sum;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    int device = -1;  // the CUDA device the state's buffers and streams live on (set at upload)
    // concurrent branches of the fused step: P3M, E3B, and the list build of
    // a rebuild step
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[3] = {nullptr, nullptr, nullptr}, ev_sorted = nullptr;
    bool uploaded = false;   // device copy is authoritative
    bool prepared = false;
    bool requiresCharges = false;
    // host-side bookkeeping of the reference's State used by configuration
    // IO: group tags (bit 0 = "all", State.cpp:31), molecules
    // (State::createMolecule), active writers, the configuration reader
    int periodic[3] = {1, 1, 1};
    std::map<std::string, uint32_t> groupTags{{"all", 1u}};
    std::vector<std::vector<int>> molecules;
    std::vector<ConfigWriter *> writers;
    ConfigReader *reader = nullptr;
    // bumped at every box change (a barostat): captured step graphs hold the
    // box by value and are rebuilt when it moves
    uint64_t box_gen = 0;
    State();
    ~State();
    int typeFromHandle(const std::string &h) const;
    void setBox();
    int upload();
    int download();
    int prepare();
    int buildNeighborList(bool force);
    int computeForces(int virialMode);
    int checkStatus();
    FixPair *pairFix();
    FixChargeEwald *ewaldFix();
    FixChargePairDSF *dsfFix();
    FixE3B *e3bFix();
    FixRigid *rigidFix();
    FixNoseHoover *nhFix();
    FixPressureBerendsen *barostatFix();
    double maxRCut();
};

// ---------------------------------------------------------------- Batch
// Independent replicas (each a full State with its own box, temperature and
// size) advanced together: every phase of the step is ONE launch whose
// gridDim.y is the replica count and whose blockIdx.y selects the replica's
// argument record in a device table; gridDim.x is sized for the largest
// replica and blocks past a smaller replica's work return at once.  The whole
// step (rebuild group included) is captured into one CUDA graph per chunk.
class Batch {
   public:
    std::vector<State *> reps;
    cudaStream_t stream = nullptr;
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    bool prepared = false;
    int periodicInterval = 10;
    int64_t turn = 0;
    // argument tables (device), one record per replica, built at prepare
    DBuf<char> tab_pair, tab_grid, tab_build, tab_p3m, tab_e3b, tab_first, tab_second;
    // replicas by form: ps (per-site list) and mfi (molecule form); the pair
    // kernel and the rebuild group launch once per form over that form's
    // replicas (tab_grid: every replica, for the skin check; tab_grid_ps,
    // tab_build, tab_pair: the per-site ones; tab_molgrid, tab_molscan,
    // tab_pairmol: the molecule-form ones, in the order of ps / mfi)
    std::vector<int> ps, mfi;
    DBuf<char> tab_grid_ps, tab_molgrid, tab_molscan, tab_pairmol;
    int max_n_ps = 0, max_cell_ps = 0, max_mol_mf = 0, max_mcell = 0;
    int pair_big = 0;
    int max_n = 0, max_mol = 0, max_cell = 0;
    size_t max_nk = 0;
    // P3M: replicas grouped by mesh size; each class owns contiguous pools
    // that the replicas' FixChargeEwald buffers view, so one batched cuFFT
    // plan per class transforms every replica of that class
    struct FFTClass {
        int3 sz{0, 0, 0};
        std::vector<int> reps;
        DBuf<float> rho, e_r;
        DBuf<float2> rho_k, e_k;
        cufftHandle r2c = 0, c2r = 0;
        // cubic 32^3 / 64^3 meshes: this library's FFT kernels over the
        // class's replicas (a table of their field pointers), no cuFFT
        bool own = false;
        DBuf<char> tab;
    };
    bool p3m_own = false;  // every class on the own FFT: the gather reads the float4 fields
    // and every replica's molecules fit the molecule form of spread and
    // gather: spread and gather by molecule, the gather on the P3M branch
    // into each replica's per-step reciprocal buffer
    bool p3m_mol = false;
    DBuf<char> tab_p3m_mol;
    std::vector<std::unique_ptr<FFTClass>> fft;
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
    std::map<std::pair<int, int>, uint64_t> graph_kernels;
    Batch();
    ~Batch();
    int biggest_rep() const;
    int prepare();
    int step();
    int enqueue(int nsteps, bool with_group);
    int launchGraph(int nsteps, bool with_group);
    int run(int nturns, double *ms);
    int runTimed(int nturns, int chunk, size_t flush_bytes, double *ms_total);
    int checkStatus();
    void clearGraphs();
    // back to the configured, unprepared replicas (their initial host state)
    void reset();
    // time `steps` steps for each neighbour team size in cands, keep the fastest
    int autotune(int steps, const int *cands, int ncand, int *best, double *best_ms);
    int64_t turn0 = 0;
    bool turn0_set = false;
};
int batch_pair_tables(Batch &b);
int batch_nlist_tables(Batch &b);
int batch_mol_tables(Batch &b);
int batch_e3b_tables(Batch &b);
int batch_pair_launch(Batch &b, cudaStream_t stream);
int batch_nlist_rebuild(Batch &b);
int batch_p3m_prepare(Batch &b);
int batch_p3m_spread_solve(Batch &b, cudaStream_t stream);
int batch_p3m_gather(Batch &b, cudaStream_t stream);
int batch_e3b_list(Batch &b);
int batch_e3b_forces(Batch &b, cudaStream_t stream);
int batch_first_half(Batch &b);
int batch_second_half(Batch &b, bool with_e3b);
int batch_rigid_maps(Batch &b);

// ---------------------------------------------------------------- kernels
// neighbour list (nlist.cu)
int nlist_rebuild(State &s, bool force, bool conditional, cudaStream_t bstream = nullptr);
int nlist_init(State &s);
int nlist_exclusions(State &s);
int nlist_set_interactions(State &s);
int molform_init(State &s);
int nlist_build_atoms_view(State &s);
// pair (pair.cu)
int pair_launch(State &s, FixPair &f, int virialMode, bool accumulate);
int pair_energy(State &s, FixPair &f, double *out);
int pair_mol_launch(State &s, FixPair &f, int virialMode, bool accumulate, float *energy, cudaStream_t st);
int pair_force_raw(int n, const float4 *xs, float4 *fs, const float *qs, const uint32_t *counts,
                   const uint32_t *nlist, int team, int cap, const float *params, int ntypes, const Box &box,
                   const float coef[3], int lj_kind, float qrc, float alpha, float qqr, float *virials,
                   bool accumulate, cudaStream_t stream);
int pair_force_gridgpu(int n, const float4 *xs, float4 *fs, const uint16_t *counts, const uint32_t *nlist,
                       const uint32_t *cum, int ntpb, int ntpa, const float *params, int ntypes, const Box &box,
                       const float coef[3], int lj_kind, const float *qs, float qcut, float alpha, float qqr,
                       float *virials, cudaStream_t stream);
// e3b (e3b.cu)
int e3b_build_list(State &s, FixE3B &f, bool conditional, cudaStream_t st = nullptr);
int e3b_build_list_mf(State &s, FixE3B &f, cudaStream_t st);
int e3b_forces(State &s, FixE3B &f);
int e3b_forces_to(State &s, FixE3B &f, float4 *out, bool side, cudaStream_t stream);
int e3b_energy(State &s, FixE3B &f, double out[2]);
int e3b_exact_to(State &s, FixE3B &f, float4 *out, int twobody, cudaStream_t stream);
int e3b_virial(State &s, FixE3B &f);
int ewald_recip_virial(State &s, FixChargeEwald &f);
int e3b_twobody_to(State &s, FixE3B &f, float4 *out, cudaStream_t stream);
// learned E3B three-body surrogate (surrogate.cu)
int surrogate_forces_to(State &s, FixE3B &f, float4 *out, cudaStream_t stream);
int surrogate_compute(State &s, FixE3B &f);
// rigid + integration (integrate.cu)
int rigid_update_maps(State &s, FixRigid &r, bool conditional);
int step_first_half(State &s, bool fused);
int step_second_half(State &s, bool fused, const float4 *fextra = nullptr, const float4 *frecip = nullptr);
bool has_free_atoms(State &s);
int rigid_prepare(State &s, FixRigid &r);
int rigid_hook(State &s, FixRigid &r, int which);
int rigid_validate(State &s, FixRigid &r, uint32_t *n_bad);
int kinetic_sum(State &s, double *out);
int nh_prepare(State &s, FixNoseHoover &nh);
int zero_forces(State &s);
int device_sum(State &s, const double *src, int n, double *out_host);
int float_sum(State &s, const float *src, int n, double *out_host);
int virial_sum(State &s, double out[6]);
int remove_com_velocity(State &s);
int nh_end_of_run(State &s);
int rigid_flags_prepare(State &s);

}  // namespace mdx

struct mdx_state {
    mdx::State *s;
};
struct mdx_fix {
    mdx::Fix *f;
    mdx_state *owner;
};
struct mdx_batch {
    mdx::Batch *b;
};
