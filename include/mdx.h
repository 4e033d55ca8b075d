/*
 * mdx.h -- C ABI of the B200-native DASH force hot path (libmdx.so).
 *
 * Plain C types only: opaque handles, pointers and sizes, int status codes
 * (0 = MDX_OK).  No C++ exceptions cross this boundary; the message of the
 * last failure on the calling thread is returned by mdx_last_error().
 *
 * Each entry point names the reference (dreid1991/md_engine, "DASH")
 * interface it replaces, by file:line within that project.  Handles are not
 * thread safe; one state per host thread / CUDA stream.  Device memory is
 * owned by the library handle and released by its destroy call.
 */
#ifndef MDX_H
#define MDX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDX_OK 0
#define MDX_ERR_ARG 1         /* invalid argument / unknown handle or key   */
#define MDX_ERR_CUDA 2        /* CUDA runtime or cuFFT failure              */
#define MDX_ERR_STATE 3       /* call not valid in the current state        */
#define MDX_ERR_OVERFLOW 4    /* neighbour-list capacity exceeded           */
#define MDX_ERR_UNSUPPORTED 5 /* configuration outside the implemented path */
#define MDX_ERR_NUMERIC 6     /* NaN force / SETTLE failure / constraint    */

#define MDX_UNITS_REAL 0
#define MDX_UNITS_LJ 1

typedef struct mdx_state mdx_state;
typedef struct mdx_fix mdx_fix;
typedef struct mdx_integrator mdx_integrator;

/* ---- library ------------------------------------------------------------ */
const char *mdx_last_error(void);
int mdx_version(void);
/* select the CUDA device for subsequent state creation on this host thread
 * (DeviceManager::setDevice, src/DeviceManager.cpp) */
int mdx_set_device(int device);
/* number of CUDA kernels this library has launched since load (for the
 * benchmark's launch count; cuFFT's own kernels are not included) */
uint64_t mdx_kernel_launch_count(void);

/* ---- State (src/State.h:63-146, src/State.cpp:28-68) --------------------- */
int mdx_state_create(mdx_state **out);
int mdx_state_destroy(mdx_state *st);
/* Units::setReal / Units::setLJ (src/Units.cpp:5-32) */
int mdx_state_set_units(mdx_state *st, int unit_type);
/* state.bounds = Bounds(state, lo=..., hi=...) (src/Bounds.cpp) */
int mdx_state_set_bounds(mdx_state *st, const double lo[3], const double hi[3]);
/* State attributes exported at src/State.cpp:1220-1247: keys "rCut",
 * "padding", "dt" (double); "periodicInterval", "nThreadPerAtom",
 * "nThreadPerBlock", "turn" (int).  Tunables of this library's list build
 * (0 = automatic, the default): "gridStencil" (cells of at least
 * (rCut + padding) / gridStencil, 1..4), "gridHomeGroup" (2 or 4 home atoms
 * tested at once per warp).  "pairForm": 0 automatic (the molecule form for
 * all-rigid four-site water), 1 per-site list, 2 molecule form.
 * "pairBlocksPerSM": molecule form, cap on the pair kernel's grid in blocks
 * per SM (0 = automatic, -1 = uncapped: one warp per molecule).  Read-only:
 * "nlistCapacity", "cellsPerSide", "molListCapacity", "molListEntries" (the
 * molecule-pair list's entries, summed over its rows). */
int mdx_state_set_double(mdx_state *st, const char *key, double value);
int mdx_state_get_double(mdx_state *st, const char *key, double *value);
int mdx_state_set_int(mdx_state *st, const char *key, int64_t value);
int mdx_state_get_int(mdx_state *st, const char *key, int64_t *value);
/* State::setSpecialNeighborCoefs (src/State.cpp:406-410) */
int mdx_state_set_special_neighbor_coefs(mdx_state *st, double onetwo, double onethree, double onefour);
/* AtomParams::addSpecies (src/AtomParams.cpp); returns the type index */
int mdx_state_add_species(mdx_state *st, const char *handle, double mass, int atomic_num, int *type_out);
/* State::addAtom (src/State.cpp) for n atoms; ids are assigned 0..N-1 in
 * call order and the first new id is returned.  pos/q may not be NULL. */
int mdx_state_add_atoms(mdx_state *st, int n, const char *const *species_handles, const double *pos,
                        const double *q, int *first_id_out);
int mdx_state_n_atoms(mdx_state *st, int *n_out);
/* atom.vel = ... for ids[i] (vel is 3 doubles per id) */
int mdx_state_set_velocities(mdx_state *st, int n, const int *ids, const double *vel);
/* host copies by atom id (each pointer may be NULL): positions, velocities,
 * forces as 3 doubles per atom.  Syncs the device copy back first. */
int mdx_state_get_atoms(mdx_state *st, double *pos, double *vel, double *force);
/* overwrite device positions/velocities by atom id from host buffers
 * (3 doubles per atom; either may be NULL) after a prepared run */
int mdx_state_put_atoms(mdx_state *st, const double *pos, const double *vel);
/* State::activateFix / deactivateFix (src/State.cpp:445-500) */
int mdx_state_activate_fix(mdx_state *st, mdx_fix *fix);
int mdx_state_deactivate_fix(mdx_state *st, mdx_fix *fix);
/* device status bits (see common.cuh StatusBits) and the largest neighbour
 * count seen at the last build */
int mdx_state_status(mdx_state *st, uint32_t *bits, uint32_t *max_neighbors, uint64_t *n_builds);
/* use a caller-owned cudaStream_t (NULL = the library's own stream) */
int mdx_state_set_stream(mdx_state *st, void *cuda_stream);
int mdx_state_synchronize(mdx_state *st);

/* ---- fixes (src/Fixes/Fix.h:79-281) ------------------------------------- */
/* FixLJCut(state, handle, mixingRules) (src/Fixes/FixLJCut.cu:14-28) */
int mdx_fix_lj_cut_create(mdx_state *st, const char *handle, const char *mixing, mdx_fix **out);
/* FixWCA(state, handle, mixingRules) (src/Fixes/FixWCA.cu) */
int mdx_fix_wca_create(mdx_state *st, const char *handle, const char *mixing, mdx_fix **out);
/* FixLJCutFS(state, handle, mixingRules) (src/Fixes/FixLJCutFS.cu:12-26):
 * force-shifted LJ (PairEvaluatorLJFS.h:15-57), parameters eps, sig, rCut */
int mdx_fix_lj_cut_fs_create(mdx_state *st, const char *handle, const char *mixing, mdx_fix **out);
/* FixLJCHARMM(state, handle, mixingRules) (src/Fixes/FixLJCHARMM.cu:15-32):
 * LJ with separate 1-4 parameters (PairEvaluatorCHARMM.h:7-44), parameters
 * eps, sig, eps14, sig14, rCut; a pair whose exclusion multiplier equals the
 * 1-4 coefficient takes eps14/sig14 */
int mdx_fix_lj_charmm_create(mdx_state *st, const char *handle, const char *mixing, mdx_fix **out);
/* FixTICG(state, handle, mixingRules) (src/Fixes/FixTICG.cu:11-22): soft
 * sphere overlap (PairEvaluatorTICG.h:9-52), parameters C and rCut, set for
 * every pair of species (no mixing) */
int mdx_fix_ticg_create(mdx_state *st, const char *handle, const char *mixing, mdx_fix **out);
/* FixChargePairDSF(state, handle, group) + setParameters(alpha, r_cut)
 * (src/Fixes/FixChargePairDSF.cu): damped shifted force charges
 * (ChargeEvaluatorDSF.h:13-47), evaluated inside the pair fix's kernel;
 * defaults alpha 0.25, r_cut 9.0.  One charge fix (Ewald or DSF) per state. */
int mdx_fix_charge_pair_dsf_create(mdx_state *st, const char *handle, const char *group, mdx_fix **out);
int mdx_fix_charge_pair_dsf_set_parameters(mdx_fix *fix, double alpha, double r_cut);
/* FixPair::setParameter(param, handleA, handleB, val) (src/Fixes/FixPair.cpp:143-168);
 * param is one of the fix's handles: "eps", "sig", "rCut" (LJ/cut, WCA,
 * LJCutFS), + "eps14", "sig14" (LJCHARMM), "C", "rCut" (TICG) */
int mdx_fix_pair_set_parameter(mdx_fix *fix, const char *param, const char *handle_a, const char *handle_b,
                               double value);
/* FixPair::getParameter(param, handleA, handleB) (FixPair.cpp:173-200): the
 * raw value set (or read from a restart); -1000 (DEFAULT_FILL) when unset */
int mdx_fix_pair_get_parameter(mdx_fix *fix, const char *param, const char *handle_a, const char *handle_b,
                               double *value);
/* FixChargeEwald(state, handle, group) (src/Fixes/FixChargeEwald.cu:828-839) */
int mdx_fix_charge_ewald_create(mdx_state *st, const char *handle, const char *group, mdx_fix **out);
/* FixChargeEwald::setParameters(sz, rcut, order) (src/Fixes/FixChargeEwald.cu:969-1021);
 * rcut < 0 means state rCut.  Grid sizes 32..1024 powers of two, order 5. */
int mdx_fix_charge_ewald_set_parameters(mdx_fix *fix, int nx, int ny, int nz, double rcut, int order);
/* explicit splitting parameter (the reference solves it by secant in
 * find_optimal_parameters, src/Fixes/FixChargeEwald.cu:918-967; <= 0 restores that) */
int mdx_fix_charge_ewald_set_alpha(mdx_fix *fix, double alpha);
int mdx_fix_charge_ewald_get_alpha(mdx_fix *fix, double *alpha);
/* FixE3B(state, handle, style) (src/Fixes/FixE3B.cu:16-36), style "E3B3" or "E3B2" */
int mdx_fix_e3b_create(mdx_state *st, const char *handle, const char *style, mdx_fix **out);
/* FixE3B::addMolecule(O, H1, H2, M) (src/Fixes/FixE3B.cu:753-792) */
int mdx_fix_e3b_add_molecule(mdx_fix *fix, int id_o, int id_h1, int id_h2, int id_m);
/* FixRigid(state, handle, style) (src/Fixes/FixRigid.cu:18-37) */
int mdx_fix_rigid_create(mdx_state *st, const char *handle, const char *style, mdx_fix **out);
/* FixRigid::createRigid(O, H1, H2, M) (src/Fixes/FixRigid.cu:1560-1610); id_m < 0 for 3-site */
int mdx_fix_rigid_create_rigid(mdx_fix *fix, int id_o, int id_h1, int id_h2, int id_m);
/* FixNoseHoover(state, handle, group) + setTemperature(T, timeConstant)
 * (src/Fixes/FixNoseHoover.cu:97-130, 221-226) */
int mdx_fix_nose_hoover_create(mdx_state *st, const char *handle, const char *group, mdx_fix **out);
int mdx_fix_nose_hoover_set_temperature(mdx_fix *fix, double temperature, double time_constant);
/* FixNoseHoover::setPressure("ISO", pressure, timeConstant)
 * (FixNoseHoover.cu:193-202): the fix also barostats, with the MTK
 * propagator of stepInit / postNVE_V / stepFinal (FixNoseHoover.cu:413-605,
 * 628-1032) run on the host in FP64 around device kernels, the box scaled
 * about its centre every step.  Systems without FixRigid ("ANISO" and rigid
 * bodies: MDX_ERR_UNSUPPORTED).  A barostatting state runs through
 * mdx_integrator_run only. */
int mdx_fix_nose_hoover_set_pressure(mdx_fix *fix, const char *mode, double pressure, double time_constant);
/* "lastPressure" (the instantaneous pressure of the last stepFinal),
 * "pressVel", "pressMass" (the isotropic barostat's velocity and mass) */
int mdx_fix_nose_hoover_get(mdx_fix *fix, const char *key, double *value);
int mdx_fix_destroy(mdx_fix *fix);

/* ---- integrator (src/Integrators/IntegratorVerlet.cu:649-770) ----------- */
int mdx_integrator_verlet_create(mdx_state *st, mdx_integrator **out);
/* IntegratorVerlet::run(numTurns); returns particle-timesteps per second
 * measured with CUDA events around the stepping loop */
int mdx_integrator_run(mdx_integrator *it, int num_turns, double *ptsps_out);
/* 0: fused, CUDA-graph captured timestep (default); 1: one kernel per
 * reference hook, no graph (the reference's launch structure) */
int mdx_integrator_set_mode(mdx_integrator *it, int mode);
int mdx_integrator_destroy(mdx_integrator *it);
/* IntegratorVerlet::run with host buffers (the State's atoms are the host
 * buffers in the reference, State.cpp:529-610): positions/velocities (3
 * doubles per atom, by id; NULL keeps the resident copy) are copied in,
 * num_turns steps run on the fused graph path, and positions / velocities /
 * forces (NULL to skip) are copied back, all within this call.  The arrays
 * cross as FP64 through pinned staging; the FP32 rounding (to nearest) and
 * the placement by id happen on the device. */
int mdx_integrator_run_host(mdx_integrator *it, int num_turns, const double *pos_in, const double *vel_in,
                            double *pos_out, double *vel_out, double *force_out);
/* Benchmark support (no reference counterpart): run num_turns in chunks of
 * `chunk` timesteps on the fused graph path; each chunk is bracketed by CUDA
 * events on the library stream and preceded, outside the timed window, by a
 * flush_bytes device write that evicts L2.  *device_ms = summed chunk time. */
int mdx_integrator_run_timed(mdx_integrator *it, int num_turns, int chunk, size_t flush_bytes, double *device_ms);
/* Integrator::tune (src/Integrators/Integrator.cu:272-376), which times the
 * force kernels for each NTPB x NTPA at the start of a run and keeps the
 * fastest: here the shape is the molecule-form pair grid's blocks per SM
 * (caps: candidates, -1 = uncapped, 0 = the built-in default), timed on the
 * force phase of the fused step (the pair kernel beside the P3M chain and
 * E3B), `reps` phases per timing; the fastest is kept as the state's
 * pairBlocksPerSM and returned with its ms per phase.  Positions and
 * velocities are untouched.  Systems without that shape: *best_cap = 0,
 * *best_ms = 0, nothing timed. */
int mdx_integrator_autotune(mdx_integrator *it, int reps, const int *caps, int ncaps, int *best_cap,
                            double *best_ms);
/* Benchmark support (no reference counterpart): average device time of one
 * launch of a hot-path stage over `iters` launches, L2 flushed between them.
 * stage 0 pair forces, 1 P3M reciprocal (spread+FFT+field+gather), 2 E3B,
 * 3 neighbour-list rebuild (forced), 4 fused first half, 5 fused second half;
 * the fused step's P3M chain as it runs there: 6 spread, 7 solve (FFT, field,
 * inverse FFT), 8 gather, 9 all three */
int mdx_time_stage(mdx_state *st, int stage, int iters, size_t flush_bytes, double *avg_ms);

/* ---- stage-level hot path ------------------------------------------------ */
/* Integrator::basicPrepare + prepareFixes + forceInitial + prepareFinal
 * (src/Integrators/Integrator.cu:142-219): upload, build, prepare, forces. */
int mdx_prepare(mdx_state *st);
/* GridGPU::periodicBoundaryConditions(-1, forceBuild) (src/GridGPU.cu:824-1103) */
int mdx_nlist_build(mdx_state *st, int force_build);
/* Grid.getNeighborList (src/GridGPU.cu:1520-1648): per-id neighbour ids,
 * sorted ascending.  counts[id]; nbr[id*max_per_atom + k] (atom ids);
 * tags[id*max_per_atom + k] = exclusion depth (0..3), may be NULL.  nbr NULL:
 * the counts alone (to size nbr).  In the molecule form (rigid water, no
 * per-site list in the step) the per-site list of the current positions is
 * built by the call itself, beside the step's buffers. */
int mdx_nlist_get(mdx_state *st, int max_per_atom, int *counts, int *nbr, int *tags);
/* IntegratorUtil::force(virialMode) (src/Integrators/IntegratorUtil.cpp:15-30):
 * zero forces, run every fix's compute() */
int mdx_compute_forces(mdx_state *st, int virial_mode);
/* Fix::singlePointEng summed per term: out[0] pair (LJ/WCA + Ewald real),
 * out[1] Ewald reciprocal, out[2] E3B two-body, out[3] E3B three-body;
 * FP64 device reductions */
int mdx_potential_energy(mdx_state *st, double out[4]);
/* sum over atoms of m v^2 (FP64) and the degrees of freedom */
int mdx_kinetic(mdx_state *st, double *sum_mv2, double *ndf);
/* The same FP64 sum of m v^2 as mdx_kinetic, for host programs that cannot
 * allocate device memory while they run (e.g. a host that serves all device
 * memory from its own pre-reserved pool, or a loop that must avoid the
 * implicit device synchronisation of cudaMalloc/cudaFree).  No counterpart
 * in the reference.  It allocates nothing: its block partials live in a fixed
 * 64 KiB file-scope device array (held on every GPU that loads the library
 * until exit), so states of more than 2,097,152 atoms are rejected with
 * MDX_ERR_ARG.  The call runs on the state's own device (made current for
 * the call; the caller's current device is restored after).  The first call
 * on a device looks the array up (set-up, once per device) and should come
 * before any stream capture; all calls share the array, so calls whose
 * kernels overlap on the GPU race. */
int mdx_kinetic_noalloc(mdx_state *st, double *sum_mv2);
/* DataComputerPressure::computeScalar_CPU (src/DataStorageUser/
 * DataComputerPressure.cu:76-92): scalar pressure (sum m v^2 + virial trace)
 * / (3 V) * nktv_to_press from a virial-mode force evaluation at the current
 * positions (pair, P3M reciprocal, E3B); virial6 (may be NULL) gets the total
 * virial.  The forces the integrator holds are restored afterwards. */
int mdx_pressure(mdx_state *st, double *pressure, double virial6[6]);
/* per-atom virials (6 per atom, xx yy zz xy xz yz) by id, FP64 total in sum6 */
int mdx_get_virials(mdx_state *st, double *per_atom, double sum6[6]);
/* single hooks, for stage-level parity (src/Fixes/FixRigid.cu:1234-1279, 1916-1984) */
int mdx_rigid_settle_positions(mdx_state *st, mdx_fix *rigid);   /* save_prev_val before x move is the caller's */
int mdx_rigid_save_prev(mdx_state *st, mdx_fix *rigid);
int mdx_rigid_settle_velocities(mdx_state *st, mdx_fix *rigid);
int mdx_rigid_distribute_msite(mdx_state *st, mdx_fix *rigid);
/* validateConstraints (src/Fixes/FixRigid.cu:351-447) on the current
 * positions and velocities: *n_bad = molecules whose O-H1, O-H2 or H1-H2
 * length is off by more than 1e-3 (NaN counts as off) or whose relative
 * velocity along a bond exceeds 1e-3; returns MDX_ERR_NUMERIC when n_bad > 0
 * (the reference prints instead).  The fused step applies the same length
 * test to every molecule after SETTLE and reports it as MDX_ERR_NUMERIC. */
int mdx_rigid_validate(mdx_state *st, mdx_fix *rigid, uint32_t *n_bad);
int mdx_verlet_first_half(mdx_state *st);   /* nve_v + nve_x (IntegratorVerlet.cu:23-61) */
int mdx_verlet_second_half(mdx_state *st);  /* postForce_cu (IntegratorVerlet.cu:610-627) */

/* ---- raw device-pointer entry points (PairEvaluateIso.h:8-207) ----------
 * mdx_pair_force_raw: the pair kernel over a neighbour list in this
 * library's own layout (mdx_pair_force_gridgpu below takes GridGPU's): atom i is in
 * warp group g = i / (32/team), slot a = i % (32/team); its k-th entry is at
 * nlist[g*cap*(32/team) + (k/team)*32 + a*team + k%team]; entries are atom
 * indices with the exclusion depth in bits 30-31.  params = {rc2, 24*eps,
 * sig^6} per type pair (3 * ntypes^2 floats, row-major, the reference's
 * paramsCoalesced order).  lj_kind 0 none / 1 LJ / 2 WCA; qrc <= 0 disables
 * the Ewald real-space term.  virials (6 floats per atom) may be NULL.
 * accumulate != 0 adds to fs instead of overwriting.  All pointers device. */
int mdx_pair_force_raw(int n, const float *xs4, float *fs4, const float *qs, const uint32_t *counts,
                       const uint32_t *nlist, int team, int cap, const float *params, int ntypes,
                       const double lo[3], const double hi[3], const float coef[3], int lj_kind, float qrc,
                       float alpha, float qqr_to_eng, float *virials, int accumulate, void *cuda_stream);

/* EvaluatorWrapperImplement::compute (src/Evaluators/EvaluatorWrapper.h:10-16,
 * 49-109) on GridGPU's list exactly as the reference hands it over
 * (GridGPU.cu:777-821, cutils_func.h:23-45): neighbor_counts (uint16 per
 * atom), neighborlist with atom i's k-th entry at
 *   (NTPB/32)*cum[b] + (cum[b+1]-cum[b])*w + s*NTPA + k%NTPA + 32*(k/NTPA)
 * where b = i/(NTPB/NTPA), w and s the warp and slot of i within block b
 * (cum = cumul_sum_max_per_block, NTPB/NTPA = n_thread_per_block/atom);
 * entries carry the exclusion depth in bits 30-31.  parameters = {rc2,
 * 24 eps, sig^6} per type pair; lj_kind 0 none / 1 LJ / 2 WCA (the pair
 * evaluator the reference's template names), q_cutoff <= 0 disables the
 * Ewald real-space term (alpha and qqr_to_eng are ChargeEvaluatorEwald's
 * members).  Forces are added to fs4; with virial_mode 1 or 2, 0.5 F (x) dr
 * per atom is added to virials (6 floats per atom).  warp_size must be 32
 * and n_per_ring_poly 1.  All pointers device. */
int mdx_pair_force_gridgpu(int n_atoms, int n_per_ring_poly, const float *xs4, float *fs4,
                           const uint16_t *neighbor_counts, const uint32_t *neighborlist,
                           const uint32_t *cumul_sum_max_per_block, int warp_size, const float *parameters,
                           int num_types, const double lo[3], const double hi[3], float onetwo_str,
                           float onethree_str, float onefour_str, float *virials, const float *qs, float q_cutoff,
                           int virial_mode, int n_thread_per_block, int n_thread_per_atom, int lj_kind, float alpha,
                           float qqr_to_eng, void *cuda_stream);

/* ---- learned E3B three-body surrogate (no reference counterpart; the exact
 *      term is src/Fixes/ThreeBodyE3B.h:255-549, which stays the fallback) --
 * Per molecule: a frame (e1 along the H-O-H bisector, e2 toward H1, e3 =
 * e1 x e2) and 128 invariant features (O->O, O->H, H1->O, H2->O channels x 8
 * Gaussian shells x {weight sum, weighted unit vector in the frame}); an MLP
 * 128-64-64-64-9 (SiLU; BF16 operands, FP32 accumulation) gives the
 * three-body forces on O, H1, H2 in the frame.  collect appends the current
 * frame's features and exact three-body forces to a device dataset; train
 * standardises (first call) and runs Adam; enable switches the fix's force
 * evaluations (fused step and compute) between exact (0) and surrogate (1);
 * eval compares surrogate and exact three-body forces on the current frame.
 * The exact O-O two-body term is always evaluated exactly.  Parameters are
 * kParams = 17,616 floats: W1[128x64] b1 W2[64x64] b2 W3[64x64] b3 W4[64x16]
 * b4[16] (outputs 9..15 unused). */
int mdx_e3b_surrogate_collect(mdx_state *st, mdx_fix *e3b);
int mdx_e3b_surrogate_dataset_size(mdx_fix *e3b, int64_t *n);
int mdx_e3b_surrogate_train(mdx_state *st, mdx_fix *e3b, int iters, int batch, float lr, uint64_t seed,
                            double *loss_first, double *loss_last);
int mdx_e3b_surrogate_enable(mdx_fix *e3b, int on);
int mdx_e3b_surrogate_eval(mdx_state *st, mdx_fix *e3b, double *rmse, double *rms);
int mdx_e3b_surrogate_get_params(mdx_fix *e3b, float *w, float *mean, float *inv_std, float *scale);
int mdx_e3b_surrogate_set_params(mdx_state *st, mdx_fix *e3b, const float *w, const float *mean,
                                 const float *inv_std, float scale);
/* raw features (nmol x 128) and frames (nmol x 9) of the current positions */
int mdx_e3b_surrogate_features(mdx_state *st, mdx_fix *e3b, float *raw, float *frames);
/* model outputs (n x 16) for n standardised feature rows (n x 128) */
int mdx_e3b_surrogate_infer(mdx_state *st, mdx_fix *e3b, const float *x, int n, float *y);
/* mean-squared-error loss and its gradient (17,616 floats) for n rows of
 * standardised features x (n x 128) and scaled targets t (n x 16); n % 64 == 0 */
int mdx_e3b_surrogate_grad(mdx_state *st, mdx_fix *e3b, const float *x, const float *t, int n, float *grad,
                           double *loss);

/* ---- batched replicas (no reference counterpart: DASH runs one State per
 *      process, src/Integrators/IntegratorVerlet.cu:649-770) --------------
 * Many independent rigid-water systems, each a configured mdx_state with its
 * own box, size and FixNoseHoover temperature, advanced together: every phase
 * of the step is one launch covering all replicas and each chunk of steps is
 * one CUDA graph.  Every replica needs a pair fix, FixChargeEwald, FixRigid
 * (all atoms in molecules) and FixNoseHoover, the same fix set (E3B in all or
 * none), periodicInterval and species count.  The batch does not own the
 * states; destroy the batch before its states.  run returns the device time
 * of the whole call in device_ms (may be NULL); run_timed brackets chunks of
 * `chunk` turns with CUDA events after an L2 flush of flush_bytes and returns
 * their summed device time. */
typedef struct mdx_batch mdx_batch;
int mdx_batch_create(mdx_batch **out);
int mdx_batch_add(mdx_batch *b, mdx_state *st);
int mdx_batch_size(mdx_batch *b, int *n);
int mdx_batch_prepare(mdx_batch *b);
int mdx_batch_run(mdx_batch *b, int num_turns, double *device_ms);
int mdx_batch_run_timed(mdx_batch *b, int num_turns, int chunk, size_t flush_bytes, double *device_ms);
/* autotuner (replaces Integrator::tune, src/Integrators/Integrator.cu:272-376):
 * resets the replicas to their configured initial state, times `steps` batched
 * steps for each neighbour team size in teams[0..nteams) and leaves the batch
 * prepared with the fastest (best_team, device ms per step in best_ms).  Call
 * it before the production run: the timing runs start from the initial state. */
int mdx_batch_autotune(mdx_batch *b, int steps, const int *teams, int nteams, int *best_team, double *best_ms);
int mdx_batch_destroy(mdx_batch *b);

/* ---- pressure control (src/Fixes/FixPressureBerendsen.cu) ----------------- */
/* FixPressureBerendsen(state, handle, pressure, period, applyEvery)
 * (FixPressureBerendsen.cu:8-12, Python signature :62-67): every applyEvery
 * turns, after the step, the scalar pressure P sets the dilation
 * (1 - dt/period (pressure - P)/bulkModulus)^(1/3), clamped to
 * 1 +- maxDilation (stepFinal, :26-51); the box scales about its centre,
 * free atoms with it and rigid molecules by their centres of mass
 * (Mod::scaleSystem, Mod.cu:301-330).  The P3M splitting and Green function
 * follow the box (FixChargeEwald::handleBoundsChange, FixChargeEwald.cu:
 * 1200-1229) and the neighbour list is rebuilt.  A state with an active
 * barostat runs through mdx_integrator_run only (its steps are launched one
 * by one rather than replayed from captured graphs). */
int mdx_fix_pressure_berendsen_create(mdx_state *st, const char *handle, double pressure, double period,
                                      int apply_every, mdx_fix **out);
/* keys "maxDilation" (setParameters, :57-59), "bulkModulus" (default 10),
 * "pressure", "period" */
int mdx_fix_pressure_berendsen_set(mdx_fix *fix, const char *key, double value);
/* the keys above and, read-only, "lastPressure", "lastDilation",
 * "applications" (the pressure and dilation of the last application) */
int mdx_fix_pressure_berendsen_get(mdx_fix *fix, const char *key, double *value);
/* Mod::scaleSystem(state, (s, s, s)) with everything that follows a box
 * change, on a prepared state */
int mdx_state_scale_system(mdx_state *st, double scale);

/* ---- configuration IO (src/WriteConfig.cpp, src/ReadConfig.cpp) ---------- */
typedef struct mdx_writer mdx_writer;
/* WriteConfig(state, fn, handle, format, writeEvery, groupHandle,
 * unwrapMolecules) (WriteConfig.cpp:389-416, Python signature at
 * WriteConfig.cpp:442-453).  format "base64" (writeXMLfileBase64,
 * WriteConfig.cpp:91-162), "xyz" (writeXYZFile, :206-251), "lammpstrj"
 * (writeLAMMPSTRJFile, :165-203), anything else the plain "xml" form
 * (writeXMLfile, :253-343, with the fixes' restart chunks).  fn gets the
 * format's suffix; a '*' in fn is replaced by the turn and makes every write
 * its own file, else writes append to one file opened (and emptied) here.
 * group_handle NULL = "all". */
int mdx_write_config_create(mdx_state *st, const char *fn, const char *handle, const char *format, int write_every,
                            const char *group_handle, int unwrap_molecules, mdx_writer **out);
/* WriteConfig attributes (WriteConfig.cpp:446-451): "writeEvery",
 * "unwrapMolecules", "writingVelocities", "writingForces" (xyz columns) */
int mdx_write_config_set(mdx_writer *w, const char *key, int64_t value);
/* WriteConfig::writePy (WriteConfig.cpp:433-439) for turn < 0 (the state's
 * turn; xyz in real units guesses atomic numbers from the masses first), else
 * WriteConfig::write(turn) (:427-432) */
int mdx_write_config_write(mdx_writer *w, int64_t turn);
/* WriteConfig::finish (closes the single-file XML's <data>) and release */
int mdx_write_config_destroy(mdx_writer *w);
/* State::activateWriteConfig / deactivateWriteConfig (State.cpp:475-480): an
 * active writer fires inside mdx_integrator_run after the step of every turn
 * that is a multiple of its writeEvery (Integrator::asyncOperations,
 * Integrator.cu:77-113) */
int mdx_state_activate_write_config(mdx_state *st, mdx_writer *w);
int mdx_state_deactivate_write_config(mdx_state *st, mdx_writer *w);
/* Integrator::writeOutput (Integrator.cu:265-269): every active writer now */
int mdx_write_output(mdx_state *st);
/* ReadConfig::loadFile (ReadConfig.cpp:319-332) */
int mdx_read_config_load(mdx_state *st, const char *fn);
/* ReadConfig::next (op 0), prev (op 1), moveBy(by) (op 2)
 * (ReadConfig.cpp:259-315): *found = 0 when there is no such configuration;
 * else the state's atoms, species, bounds, turn, rCut, padding, dt, groups and
 * molecules are replaced by the configuration's (ReadConfig::read,
 * ReadConfig.cpp:176-257), and fixes created afterwards read their restart
 * chunk from it (FixPair::readFromRestart, FixPair.cpp:211-240;
 * FixRigid::readFromRestart, FixRigid.cu:1458-1514).  Atom ids must be
 * 0..numAtoms-1 (this library's ids are indices). */
int mdx_read_config_move(mdx_state *st, int op, int by, int *found);
/* State::createGroup(handle, ids) (State.cpp:878-889): the next free tag bit */
int mdx_state_create_group(mdx_state *st, const char *handle, int n, const int *ids);
int mdx_state_group_tag(mdx_state *st, const char *handle, uint32_t *bit);
/* State::createMolecule(ids) (State.cpp createMoleculePy): written to
 * <molecules> and unwrapped by writers with unwrapMolecules */
int mdx_state_create_molecule(mdx_state *st, int n, const int *ids);
/* the state's bounds and species as a read configuration left them */
int mdx_state_get_bounds(mdx_state *st, double lo[3], double hi[3]);
/* species k (handle copied into handle[0..cap)); k < 0 only sets *count */
int mdx_state_get_species(mdx_state *st, int k, char *handle, int cap, double *mass, int *atomic_num, int *count);

#ifdef __cplusplus
}
#endif
#endif /* MDX_H */
