// IntegratorVerlet (src/Integrators/IntegratorVerlet.cu:649-770).
//
// The run loop keeps the reference's per-step hook order (§ stepInit ->
// nve_v/nve_x -> postNVE_X -> force -> postForce -> preStepFinal ->
// stepFinal) but, in the default fused mode, a chunk of periodicInterval
// steps is captured once into a CUDA graph: [neighbour-list check + rebuild
// group, each kernel returning at once unless the device decided to rebuild]
// followed by the steps.  Nothing in a step waits on the host.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <map>
#include <vector>

#include "engine.hpp"

namespace mdx {

namespace {
// host-buffer run support: scatter by id into the sorted device streams and
// gather them back in id order
// host-buffer runs: (n,3) FP64 arrays by atom id in, rounded to FP32 here
// (the host cast's round-to-nearest), and widened back out; .w is kept
__global__ void k_put_by_id(int n, const double *__restrict__ in, const int *__restrict__ idToIdx,
                            float4 *__restrict__ dst) {
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const int i = idToIdx[id];
    const float w = dst[i].w;
    const double *v = in + 3 * (size_t)id;
    dst[i] = make_float4((float)v[0], (float)v[1], (float)v[2], w);
}
__global__ void k_get_by_id(int n, const float4 *__restrict__ src, const uint32_t *__restrict__ ids,
                            double *__restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = src[i];
    double *o = out + 3 * (size_t)ids[i];
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
}
}  // namespace

class IntegratorVerlet {
   public:
    State *s;
    int mode = 0;  // 0 fused + graphs, 1 hook-by-hook without graphs
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
    std::map<std::pair<int, int>, uint64_t> graph_kernels;  // our kernels per graph
    explicit IntegratorVerlet(State *st) : s(st) {}
    ~IntegratorVerlet() {
        clearGraphs();
        if (h_stage) cudaFreeHost(h_stage);
    }
    void clearGraphs() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
        graph_kernels.clear();
    }
    int forces() {
        // IntegratorUtil::force: pair fixes first (orderPreference -1)
        if (FixPair *p = s->pairFix())
            if (int e = p->compute(0)) return e;
        for (Fix *f : s->fixes) {
            if (f->kind == FixKind::Pair) continue;
            if (int e = f->compute(0)) return e;
        }
        return 0;
    }
    // fused step: the P3M chain (spread, R2C, E(k), C2R) and E3B run on two
    // side streams beside the pair kernel; they join before the P3M gather
    // and the second half (which merges the E3B forces)
    int stepFused() {
        FixPair *pf = s->pairFix();
        FixChargeEwald *ew = s->ewaldFix();
        FixE3B *e3 = s->e3bFix();
        const bool e3side = e3 && e3->side_ok && s->rigidFix();
        if (int e = step_first_half(*s, true)) return e;
        if (ew || e3side) MDX_CUDA_TRY(cudaEventRecord(s->ev_fork, s->stream));
        // all-rigid systems: the gather also runs on the side stream, into a
        // per-step buffer the second half adds (so it overlaps the pair kernel)
        const bool recip_side = ew && s->rigidFix() && !has_free_atoms(*s);
        if (ew) {
            MDX_CUDA_TRY(cudaStreamWaitEvent(s->side[0], s->ev_fork, 0));
            // all-rigid water: spread and gather by molecule (charged sites only)
            const bool by_mol = recip_side && ew->mol_form_ok(*s->rigidFix());
            if (int e = by_mol ? ew->spread_mol(s->side[0], *s->rigidFix()) : ew->spread(s->side[0])) return e;
            if (int e = ew->solve(s->side[0])) return e;
            if (recip_side)
                if (int e = by_mol ? ew->gather_mol_to(ew->f_recip.p, s->side[0], *s->rigidFix())
                                   : ew->gather_to(ew->f_recip.p, s->side[0]))
                    return e;
            MDX_CUDA_TRY(cudaEventRecord(s->ev_join[0], s->side[0]));
        }
        if (e3side) {
            MDX_CUDA_TRY(cudaStreamWaitEvent(s->side[1], s->ev_fork, 0));
            if (build_pending) MDX_CUDA_TRY(cudaStreamWaitEvent(s->side[1], s->ev_join[2], 0));
            if (e3->sur && e3->sur->enabled) {
                if (int e = surrogate_forces_to(*s, *e3, e3->f_side.p, s->side[1])) return e;
            } else {
                if (int e = e3b_forces_to(*s, *e3, e3->f_side.p, true, s->side[1])) return e;
            }
            MDX_CUDA_TRY(cudaEventRecord(s->ev_join[1], s->side[1]));
        }
        if (build_pending) {
            // the lists are read from here on
            MDX_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->ev_join[2], 0));
            build_pending = false;
        }
        if (pf)
            if (int e = pair_launch(*s, *pf, 0, false)) return e;
        if (e3 && !e3side)
            if (int e = e3b_forces(*s, *e3)) return e;
        if (ew) {
            MDX_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->ev_join[0], 0));
            if (!recip_side)
                if (int e = ew->gather(true, s->stream)) return e;
        }
        if (e3side) MDX_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->ev_join[1], 0));
        return step_second_half(*s, true, e3side ? e3->f_side.p : nullptr, recip_side ? ew->f_recip.p : nullptr);
    }
    // the force phase of the fused step alone (fork, the pair kernel beside
    // the P3M chain and E3B, join): what the pair grid's cap trades off
    int forcePhase() {
        FixPair *pf = s->pairFix();
        FixChargeEwald *ew = s->ewaldFix();
        FixE3B *e3 = s->e3bFix();
        FixRigid &r = *s->rigidFix();
        MDX_CUDA_TRY(cudaEventRecord(s->ev_fork, s->stream));
        MDX_CUDA_TRY(cudaStreamWaitEvent(s->side[0], s->ev_fork, 0));
        if (int e = ew->spread_mol(s->side[0], r)) return e;
        if (int e = ew->solve(s->side[0])) return e;
        if (int e = ew->gather_mol_to(ew->f_recip.p, s->side[0], r)) return e;
        MDX_CUDA_TRY(cudaEventRecord(s->ev_join[0], s->side[0]));
        if (e3) {
            MDX_CUDA_TRY(cudaStreamWaitEvent(s->side[1], s->ev_fork, 0));
            if (int e = e3b_forces_to(*s, *e3, e3->f_side.p, true, s->side[1])) return e;
            MDX_CUDA_TRY(cudaEventRecord(s->ev_join[1], s->side[1]));
        }
        if (int e = pair_launch(*s, *pf, 0, false)) return e;
        MDX_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->ev_join[0], 0));
        if (e3) MDX_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->ev_join[1], 0));
        return 0;
    }

    // Integrator::tune (Integrator.cu:272-376) times the force kernels for
    // each NTPB x NTPA at the start of a run and keeps the fastest.  Here, for
    // the molecule form of all-rigid water with P3M (and E3B) beside the pair
    // kernel, the tuned shape is the pair grid's blocks per SM: each
    // candidate's force phase is captured as a graph of `reps` repetitions
    // and timed by CUDA events (median of three launches); the fastest is
    // kept in State::pairBlocksPerSM (-1: uncapped).  Positions and
    // velocities are not touched, the force array is saved and put back.
    // Other systems have no such shape: best = 0, nothing is timed.
    int autotunePairGrid(int reps, const int *caps, int ncaps, int *best, double *best_ms) {
        *best = 0;
        *best_ms = 0.0;
        if (!s->prepared) {
            clearGraphs();
            if (int e = s->prepare()) return e;
        }
        FixChargeEwald *ew = s->ewaldFix();
        FixE3B *e3 = s->e3bFix();
        const bool ok = s->pairFix() && ew && s->mf.on && s->rigidFix() && !has_free_atoms(*s) &&
                        ew->mol_form_ok(*s->rigidFix()) && (!e3 || e3->side_ok) &&
                        !(e3 && e3->sur && e3->sur->enabled);
        if (!ok || reps <= 0 || ncaps <= 0) return 0;
        const int n = s->gpd.n;
        DBuf<float4> fsave;
        if (int e = fsave.alloc(n)) return e;
        MDX_CUDA_TRY(cudaMemcpyAsync(fsave.p, s->gpd.fs.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, s->stream));
        const int keep = s->pairBlocksPerSM;
        cudaEvent_t a, b;
        MDX_CUDA_TRY(cudaEventCreate(&a));
        MDX_CUDA_TRY(cudaEventCreate(&b));
        double best_t = 0.0;
        int best_c = keep;
        for (int k = 0; k < ncaps; k++) {
            s->pairBlocksPerSM = caps[k];
            cudaGraph_t g;
            MDX_CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = g_launches;
            int e = 0;
            for (int r = 0; r < reps && !e; r++) e = forcePhase();
            g_launches = before;
            cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
            if (e) return e;
            if (ce != cudaSuccess) {
                set_error(MDX_ERR_CUDA, "autotune capture failed: %s", cudaGetErrorString(ce));
                return MDX_ERR_CUDA;
            }
            cudaGraphExec_t ex;
            MDX_CUDA_TRY(cudaGraphInstantiate(&ex, g, cudaGraphInstantiateFlagUseNodePriority));
            cudaGraphDestroy(g);
            MDX_CUDA_TRY(cudaGraphLaunch(ex, s->stream));  // warm
            float t[3];
            for (int q = 0; q < 3; q++) {
                MDX_CUDA_TRY(cudaEventRecord(a, s->stream));
                MDX_CUDA_TRY(cudaGraphLaunch(ex, s->stream));
                MDX_CUDA_TRY(cudaEventRecord(b, s->stream));
                MDX_CUDA_TRY(cudaEventSynchronize(b));
                MDX_CUDA_TRY(cudaEventElapsedTime(&t[q], a, b));
            }
            cudaGraphExecDestroy(ex);
            std::sort(t, t + 3);
            const double ms = (double)t[1] / reps;
            if (k == 0 || ms < best_t) {
                best_t = ms;
                best_c = caps[k];
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        MDX_CUDA_TRY(cudaMemcpyAsync(s->gpd.fs.p, fsave.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, s->stream));
        MDX_CUDA_TRY(cudaStreamSynchronize(s->stream));
        s->pairBlocksPerSM = best_c;
        clearGraphs();  // the step graphs take the chosen shape
        *best = best_c;
        *best_ms = best_t;
        return s->checkStatus();
    }

    int stepBody() {
        if (mode == 0) return stepFused();
        if (int e = step_first_half(*s, false)) return e;
        if (int e = forces()) return e;
        if (int e = step_second_half(*s, false)) return e;
        return 0;
    }
    // fused graphs: the list build of a rebuild step runs on side stream 2
    // beside the step's first half and P3M chain; the pair kernel and E3B of
    // that step wait for it (build_pending)
    bool build_pending = false;
    int enqueue(int nsteps, bool with_group) {
        if (with_group) {
            // (the per-site form's first build sizes its list with a host sync)
            const bool overlap = mode == 0 && (s->grid.cap != 0 || s->mf.on);
            if (int e = nlist_rebuild(*s, false, true, overlap ? s->side[2] : nullptr)) return e;
            build_pending = overlap;
        }
        for (int k = 0; k < nsteps; k++)
            if (int e = stepBody()) return e;
        if (build_pending) MDX_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->ev_join[2], 0));
        build_pending = false;
        return 0;
    }
    uint64_t graph_box_gen = 0;
    int getGraph(int nsteps, bool with_group, cudaGraphExec_t *out) {
        if (graph_box_gen != s->box_gen) {
            clearGraphs();
            graph_box_gen = s->box_gen;
        }
        auto key = std::make_pair(nsteps, with_group ? 1 : 0);
        auto it = graphs.find(key);
        if (it != graphs.end()) {
            *out = it->second;
            return 0;
        }
        cudaGraph_t g;
        MDX_CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        const uint64_t before = g_launches;
        int e = enqueue(nsteps, with_group);
        const uint64_t captured = g_launches - before;
        g_launches = before;  // counted again at every replay
        cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
        if (e) return e;
        if (ce != cudaSuccess) {
            set_error(MDX_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
            return MDX_ERR_CUDA;
        }
        cudaGraphExec_t ex;
        MDX_CUDA_TRY(cudaGraphInstantiate(&ex, g, cudaGraphInstantiateFlagUseNodePriority));
        cudaGraphDestroy(g);
        graphs[key] = ex;
        graph_kernels[key] = captured;
        *out = ex;
        return 0;
    }
    int launchGraph(int nsteps, bool with_group) {
        cudaGraphExec_t ex;
        if (int e = getGraph(nsteps, with_group, &ex)) return e;
        MDX_CUDA_TRY(cudaGraphLaunch(ex, s->stream));
        g_launches += graph_kernels[std::make_pair(nsteps, with_group ? 1 : 0)];
        return 0;
    }
    // the (steps, rebuild group) chunk shapes that nturns steps from the
    // current turn split into, given a window of `chunk` steps (chunk <= 0:
    // one window); each window is cut at every periodicInterval boundary
    std::vector<std::pair<int, bool>> chunkShapes(int nturns, int chunk) const {
        std::vector<std::pair<int, bool>> out;
        const int P = s->periodicInterval > 0 ? s->periodicInterval : 1;
        int64_t t = s->turn;
        int done = 0;
        while (done < nturns) {
            int todo = chunk > 0 ? std::min(chunk, nturns - done) : nturns - done;
            while (todo > 0) {
                const bool check = (t % P) == 0;
                int c = check ? P : (int)(P - (t % P));
                c = std::min(c, todo);
                out.emplace_back(c, check);
                t += c;
                todo -= c;
                done += c;
            }
        }
        return out;
    }
    // capture and instantiate, ahead of time, every graph a run of nturns
    // steps in windows of `chunk` will launch, so that no capture or
    // instantiation happens between a window's timing events
    int precapture(int nturns, int chunk) {
        for (const auto &sh : chunkShapes(nturns, chunk)) {
            cudaGraphExec_t ex;
            if (int e = getGraph(sh.first, sh.second, &ex)) return e;
        }
        return 0;
    }
    // bench support: nturns in chunks of `chunk`, each chunk bracketed by
    // CUDA events on the library stream, L2 flushed (a write larger than L2)
    // before every chunk outside the timed windows; returns summed device ms
    int runTimed(int nturns, int chunk, size_t flush_bytes, double *ms_total) {
        if (s->barostatFix() || (s->nhFix() && s->nhFix()->barostatting)) {
            set_error(MDX_ERR_UNSUPPORTED, "a barostat changes the box between steps: use mdx_integrator_run");
            return MDX_ERR_UNSUPPORTED;
        }
        if (!s->prepared) {
            clearGraphs();
            if (int e = s->prepare()) return e;
        }
        DBuf<char> flush;
        if (flush_bytes)
            if (int e = flush.alloc(flush_bytes)) return e;
        // every graph shape of the timed windows exists before the first event
        if (int e = precapture(nturns, chunk)) return e;
        std::vector<cudaEvent_t> ev;
        const int P = s->periodicInterval > 0 ? s->periodicInterval : 1;
        int done = 0;
        while (done < nturns) {
            if (flush_bytes) MDX_CUDA_TRY(cudaMemsetAsync(flush.p, (int)(done & 0xff), flush_bytes, s->stream));
            cudaEvent_t a, b;
            MDX_CUDA_TRY(cudaEventCreate(&a));
            MDX_CUDA_TRY(cudaEventCreate(&b));
            MDX_CUDA_TRY(cudaEventRecord(a, s->stream));
            int todo = std::min(chunk, nturns - done);
            while (todo > 0) {
                const int64_t t = s->turn;
                const bool check = (t % P) == 0;
                int c = check ? P : (int)(P - (t % P));
                c = std::min(c, todo);
                if (int e = launchGraph(c, check)) return e;
                s->turn += c;
                todo -= c;
                done += c;
            }
            MDX_CUDA_TRY(cudaEventRecord(b, s->stream));
            ev.push_back(a);
            ev.push_back(b);
        }
        MDX_CUDA_TRY(cudaStreamSynchronize(s->stream));
        double tot = 0.0;
        for (size_t k = 0; k < ev.size(); k += 2) {
            float ms = 0.f;
            MDX_CUDA_TRY(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            tot += ms;
            cudaEventDestroy(ev[k]);
            cudaEventDestroy(ev[k + 1]);
        }
        *ms_total = tot;
        return s->checkStatus();
    }

    // run with host buffers in/out (the call a host program makes): inputs are
    // copied from pinned staging and scattered by id, outputs gathered by id
    // and copied back, all inside the call
    double *h_stage = nullptr;  // pinned: 3 arrays of (n,3) FP64
    size_t h_stage_n = 0;
    DBuf<double> d_stage;
    int runHost(int nturns, const double *pin, const double *vin, double *pout, double *vout, double *fout) {
        if (s->barostatFix() || (s->nhFix() && s->nhFix()->barostatting)) {
            set_error(MDX_ERR_UNSUPPORTED, "a barostat changes the box between steps: use mdx_integrator_run");
            return MDX_ERR_UNSUPPORTED;
        }
        if (!s->prepared) {
            clearGraphs();
            if (int e = s->prepare()) return e;
        }
        const int n = s->gpd.n;
        const size_t a3 = 3 * (size_t)n;  // doubles per array
        if (h_stage_n < 3 * a3) {
            if (h_stage) cudaFreeHost(h_stage);
            MDX_CUDA_TRY(cudaMallocHost(&h_stage, 3 * a3 * sizeof(double)));
            h_stage_n = 3 * a3;
        }
        if (int e = d_stage.alloc(3 * a3)) return e;
        // the step graphs of this call exist before any copy is queued
        if (int e = precapture(nturns, 0)) return e;
        // inputs: a plain copy into pinned memory, one async copy each, the
        // FP32 rounding and the scatter by id on the device
        const double *ins[2] = {pin, vin};
        float4 *dsts[2] = {s->gpd.xs.p, s->gpd.vs.p};
        for (int k = 0; k < 2; k++) {
            if (!ins[k]) continue;
            double *h = h_stage + k * a3;
            std::memcpy(h, ins[k], a3 * sizeof(double));
            MDX_CUDA_TRY(cudaMemcpyAsync(d_stage.p + k * a3, h, a3 * sizeof(double), cudaMemcpyHostToDevice,
                                         s->stream));
            k_put_by_id<<<(n + 255) / 256, 256, 0, s->stream>>>(n, d_stage.p + k * a3, s->gpd.idToIdx.p, dsts[k]);
            MDX_LAUNCHED();
        }
        const int P = s->periodicInterval > 0 ? s->periodicInterval : 1;
        int done = 0;
        while (done < nturns) {
            const int64_t t = s->turn;
            const bool check = (t % P) == 0;
            int c = check ? P : (int)(P - (t % P));
            c = std::min(c, nturns - done);
            if (int e = launchGraph(c, check)) return e;
            s->turn += c;
            done += c;
        }
        if (nturns > 0)
            if (int e = nh_end_of_run(*s)) return e;
        double *outs[3] = {pout, vout, fout};
        const float4 *srcs[3] = {s->gpd.xs.p, s->gpd.vs.p, s->gpd.fs.p};
        for (int k = 0; k < 3; k++) {
            if (!outs[k]) continue;
            k_get_by_id<<<(n + 255) / 256, 256, 0, s->stream>>>(n, srcs[k], s->gpd.ids.p, d_stage.p + k * a3);
            MDX_LAUNCHED();
            MDX_CUDA_TRY(cudaMemcpyAsync(h_stage + k * a3, d_stage.p + k * a3, a3 * sizeof(double),
                                         cudaMemcpyDeviceToHost, s->stream));
        }
        MDX_CUDA_TRY(cudaMemcpyAsync(s->h_status, s->d_status.p, sizeof(DeviceStatus), cudaMemcpyDeviceToHost,
                                     s->stream));
        MDX_CUDA_TRY(cudaStreamSynchronize(s->stream));
        for (int k = 0; k < 3; k++)
            if (outs[k]) std::memcpy(outs[k], h_stage + k * a3, a3 * sizeof(double));
        if (s->h_status->bits) return s->checkStatus();
        return 0;
    }

    // an NPT run with FixNoseHoover's barostat (the MTK propagator): host
    // steps in the reference's hook order, the box moving every step
    int runMtk(FixNoseHoover &nh, int nturns, double *ptsps) {
        if (int e = mtk_prepare(*s, nh)) return e;
        cudaEvent_t e0, e1;
        MDX_CUDA_TRY(cudaEventCreate(&e0));
        MDX_CUDA_TRY(cudaEventCreate(&e1));
        MDX_CUDA_TRY(cudaEventRecord(e0, s->stream));
        for (int k = 0; k < nturns; k++) {
            if (int e = mtk_step(*s, nh)) return e;
            const int64_t t = s->turn;
            s->turn += 1;
            MDX_CUDA_TRY(cudaMemcpyAsync(&s->d_status.p->turn, &s->turn, sizeof(int64_t), cudaMemcpyHostToDevice,
                                         s->stream));
            if (config_next_write(*s, t) == t) {
                if (int e = s->checkStatus()) return e;
                if (int e = config_write_due(*s, t)) return e;
            }
        }
        MDX_CUDA_TRY(cudaEventRecord(e1, s->stream));
        MDX_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        MDX_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (int e = s->checkStatus()) return e;
        if (int e = mtk_finish(*s, nh)) return e;
        if (ptsps) *ptsps = ms > 0 ? (double)s->atoms.size() * nturns / (ms * 1e-3) : 0.0;
        return s->download();
    }

    int run(int nturns, double *ptsps) {
        if (nturns < 0) {
            set_error(MDX_ERR_ARG, "numTurns must be >= 0");
            return MDX_ERR_ARG;
        }
        if (!s->prepared) {
            clearGraphs();
            if (int e = s->prepare()) return e;
        }
        if (FixNoseHoover *nh = s->nhFix())
            if (nh->barostatting) return runMtk(*nh, nturns, ptsps);
        const int P = s->periodicInterval > 0 ? s->periodicInterval : 1;
        cudaEvent_t e0, e1;
        MDX_CUDA_TRY(cudaEventCreate(&e0));
        MDX_CUDA_TRY(cudaEventCreate(&e1));
        MDX_CUDA_TRY(cudaEventRecord(e0, s->stream));
        int done = 0;
        while (done < nturns) {
            const int64_t t = s->turn;
            const bool check = (t % P) == 0;
            int chunk = check ? P : (int)(P - (t % P));
            if (chunk > nturns - done) chunk = nturns - done;
            // configuration writers (Integrator::asyncOperations,
            // Integrator.cu:77-113) and the barostat (its stepFinal): due at
            // turn T, they act after that turn's step, so the chunk ends there
            const int64_t wt = config_next_write(*s, t);
            if (wt >= 0 && wt - t + 1 < chunk) chunk = (int)(wt - t + 1);
            FixPressureBerendsen *baro = s->barostatFix();
            const int64_t bt = barostat_next(*s, t);
            if (bt >= 0 && bt - t + 1 < chunk) chunk = (int)(bt - t + 1);
            // with a barostat the box moves every few steps: launched step by
            // step (captured graphs hold the box by value)
            if (mode == 0 && !baro) {
                if (int e = launchGraph(chunk, check)) return e;
            } else {
                if (int e = enqueue(chunk, check)) return e;
            }
            s->turn += chunk;
            done += chunk;
            if (bt >= 0 && s->turn == bt + 1) {
                MDX_CUDA_TRY(cudaStreamSynchronize(s->stream));
                if (int e = s->checkStatus()) return e;
                if (int e = barostat_apply(*s, *baro)) return e;
            }
            if (wt >= 0 && s->turn == wt + 1) {
                if (int e = s->checkStatus()) return e;
                if (int e = config_write_due(*s, wt)) return e;
            }
        }
        MDX_CUDA_TRY(cudaEventRecord(e1, s->stream));
        if (nturns > 0)
            if (int e = nh_end_of_run(*s)) return e;
        MDX_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        MDX_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        MDX_CUDA_TRY(cudaGetLastError());
        if (int e = s->checkStatus()) return e;
        if (ptsps) *ptsps = ms > 0 ? (double)s->atoms.size() * nturns / (ms * 1e-3) : 0.0;
        if (FixNoseHoover *nh = s->nhFix()) {
            NHChain c[2];
            MDX_CUDA_TRY(cudaMemcpy(c, nh->d_chain.p, sizeof(c), cudaMemcpyDeviceToHost));
            nh->h = c[0];
        }
        return s->download();
    }
};

}  // namespace mdx

struct mdx_integrator {
    mdx::IntegratorVerlet *it;
};

using namespace mdx;

extern "C" {

int mdx_integrator_verlet_create(mdx_state *st, mdx_integrator **out) {
    if (!st || !out) {
        set_error(MDX_ERR_ARG, "null argument");
        return MDX_ERR_ARG;
    }
    *out = new mdx_integrator{new IntegratorVerlet(st->s)};
    return 0;
}

int mdx_integrator_run(mdx_integrator *it, int num_turns, double *ptsps_out) {
    if (!it) {
        set_error(MDX_ERR_ARG, "null integrator");
        return MDX_ERR_ARG;
    }
    try {
        return it->it->run(num_turns, ptsps_out);
    } catch (...) {
        set_error(MDX_ERR_STATE, "exception in run");
        return MDX_ERR_STATE;
    }
}

int mdx_integrator_autotune(mdx_integrator *it, int reps, const int *caps, int ncaps, int *best_cap,
                            double *best_ms) {
    if (!it || !caps || !best_cap || !best_ms || reps <= 0 || ncaps <= 0) {
        set_error(MDX_ERR_ARG, "bad argument");
        return MDX_ERR_ARG;
    }
    for (int k = 0; k < ncaps; k++)
        if (caps[k] < -1 || caps[k] > 32) {
            set_error(MDX_ERR_ARG, "pair grid caps are -1 (uncapped) or 0..32 blocks per SM (got %d)", caps[k]);
            return MDX_ERR_ARG;
        }
    try {
        return it->it->autotunePairGrid(reps, caps, ncaps, best_cap, best_ms);
    } catch (...) {
        set_error(MDX_ERR_STATE, "exception in autotune");
        return MDX_ERR_STATE;
    }
}

int mdx_integrator_run_timed(mdx_integrator *it, int num_turns, int chunk, size_t flush_bytes, double *device_ms) {
    if (!it || !device_ms || num_turns < 0 || chunk <= 0) {
        set_error(MDX_ERR_ARG, "bad argument");
        return MDX_ERR_ARG;
    }
    if (it->it->mode != 0) {
        set_error(MDX_ERR_STATE, "timed runs use the fused graph mode");
        return MDX_ERR_STATE;
    }
    try {
        return it->it->runTimed(num_turns, chunk, flush_bytes, device_ms);
    } catch (...) {
        set_error(MDX_ERR_STATE, "exception in run");
        return MDX_ERR_STATE;
    }
}

int mdx_integrator_run_host(mdx_integrator *it, int num_turns, const double *pos_in, const double *vel_in,
                            double *pos_out, double *vel_out, double *force_out) {
    if (!it || num_turns < 0) {
        set_error(MDX_ERR_ARG, "bad argument");
        return MDX_ERR_ARG;
    }
    if (it->it->mode != 0) {
        set_error(MDX_ERR_STATE, "host-buffer runs use the fused graph mode");
        return MDX_ERR_STATE;
    }
    try {
        return it->it->runHost(num_turns, pos_in, vel_in, pos_out, vel_out, force_out);
    } catch (...) {
        set_error(MDX_ERR_STATE, "exception in run");
        return MDX_ERR_STATE;
    }
}

int mdx_integrator_set_mode(mdx_integrator *it, int mode) {
    if (!it || (mode != 0 && mode != 1)) {
        set_error(MDX_ERR_ARG, "mode must be 0 (fused graph) or 1 (hook by hook)");
        return MDX_ERR_ARG;
    }
    it->it->mode = mode;
    it->it->clearGraphs();
    return 0;
}

int mdx_integrator_destroy(mdx_integrator *it) {
    if (!it) return 0;
    delete it->it;
    delete it;
    return 0;
}

}  // extern "C"
