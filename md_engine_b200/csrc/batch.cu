// Batched replicas: many independent water systems (each a full State with its
// own box, size and thermostat temperature) advanced together.  The reference
// has no such form (one State per process, IntegratorVerlet.cu:649-770); each
// replica keeps the reference's per-step semantics exactly, and only the
// launch structure changes: every phase of the fused step is one launch whose
// gridDim.y is the replica count (blockIdx.y picks the replica's argument
// record), the FFTs are batched per mesh size, and a chunk of steps (with the
// rebuild group in front) is captured once into a CUDA graph.
//
// Requirements checked at prepare: every replica is rigid water (all atoms in
// FixRigid molecules) with a pair fix + FixChargeEwald + FixNoseHoover, the
// same fix set (E3B in all or none), the same periodicInterval, and the same
// neighbour team size.
#include <algorithm>
#include <cstdio>

#include "engine.hpp"

namespace mdx {

Batch::Batch() = default;

Batch::~Batch() {
    clearGraphs();
    for (auto &c : fft) {
        if (c->r2c) cufftDestroy(c->r2c);
        if (c->c2r) cufftDestroy(c->c2r);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (auto &e : ev_join)
        if (e) cudaEventDestroy(e);
    for (auto &s : side)
        if (s) cudaStreamDestroy(s);
    if (stream) cudaStreamDestroy(stream);
}

void Batch::clearGraphs() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
    graph_kernels.clear();
}

int Batch::biggest_rep() const {
    int best = 0;
    for (int r = 1; r < (int)reps.size(); r++)
        if (reps[r]->gpd.n > reps[best]->gpd.n) best = r;
    return best;
}

void Batch::reset() {
    clearGraphs();
    for (State *s : reps) {
        if (FixChargeEwald *ew = s->ewaldFix()) {
            // views into the pools below: let the fix own its buffers again
            ew->rho.release();
            ew->rho_k.release();
            ew->e_k.release();
            ew->e_r.release();
        }
        s->prepared = false;
        s->grid.cap = 0;
        s->turn = turn0;
    }
    for (auto &c : fft) {
        if (c->r2c) cufftDestroy(c->r2c);
        if (c->c2r) cufftDestroy(c->c2r);
    }
    fft.clear();
    for (DBuf<char> *t : {&tab_pair, &tab_grid, &tab_grid_ps, &tab_build, &tab_p3m, &tab_e3b, &tab_first,
                          &tab_second, &tab_molgrid, &tab_molscan, &tab_pairmol, &tab_p3m_mol})
        t->release();
    max_n = max_mol = max_cell = 0;
    ps.clear();
    mfi.clear();
    max_nk = 0;
    prepared = false;
}

// The reference's Integrator::tune (Integrator.cu:272-376) times 30 force
// evaluations for every (threads per block, threads per atom) pair; here the
// whole batched step is timed for each neighbour team size (threads per
// atom; the pair kernel's list layout and the build follow it) from the same
// initial state, and the batch is left prepared with the fastest.
int Batch::autotune(int steps, const int *cands, int ncand, int *best, double *best_ms) {
    if (steps <= 0 || ncand <= 0 || !cands) {
        set_error(MDX_ERR_ARG, "need steps > 0 and candidate team sizes");
        return MDX_ERR_ARG;
    }
    if (!turn0_set) {
        turn0 = reps.empty() ? 0 : reps[0]->turn;
        turn0_set = true;
    }
    int arg = -1;
    double tbest = 1e300;
    for (int k = 0; k < ncand; k++) {
        const int t = cands[k];
        if (t != 1 && t != 2 && t != 4 && t != 8 && t != 16 && t != 32) {
            set_error(MDX_ERR_ARG, "team size %d not in {1,2,4,8,16,32}", t);
            return MDX_ERR_ARG;
        }
        reset();
        for (State *s : reps) s->nThreadPerAtom = t;
        if (int e = prepare()) return e;
        if (int e = run(periodicInterval, nullptr)) return e;  // capture the graphs
        double ms = 0.0;
        if (int e = runTimed(steps, periodicInterval, 0, &ms)) return e;
        if (ms < tbest) {
            tbest = ms;
            arg = t;
        }
    }
    reset();
    for (State *s : reps) s->nThreadPerAtom = arg;
    if (int e = prepare()) return e;
    if (best) *best = arg;
    if (best_ms) *best_ms = tbest / steps;
    return 0;
}

int Batch::prepare() {
    if (reps.empty()) {
        set_error(MDX_ERR_STATE, "batch has no replicas");
        return MDX_ERR_STATE;
    }
    if (!turn0_set) {
        turn0 = reps[0]->turn;
        turn0_set = true;
    }
    State &s0 = *reps[0];
    const bool e3b0 = s0.e3bFix() != nullptr;
    for (State *s : reps) {
        if (!s->pairFix() || !s->ewaldFix() || !s->rigidFix() || !s->nhFix()) {
            set_error(MDX_ERR_UNSUPPORTED, "batched replicas need a pair fix, FixChargeEwald, FixRigid and "
                                           "FixNoseHoover in every replica");
            return MDX_ERR_UNSUPPORTED;
        }
        if ((s->e3bFix() != nullptr) != e3b0 || s->periodicInterval != s0.periodicInterval ||
            s->species.size() != s0.species.size()) {
            set_error(MDX_ERR_UNSUPPORTED, "replicas differ in fix set, periodicInterval or species");
            return MDX_ERR_UNSUPPORTED;
        }
        if (s->e3bFix() && s->e3bFix()->sur && s->e3bFix()->sur->enabled) {
            set_error(MDX_ERR_UNSUPPORTED, "batched replicas run the exact E3B kernel; disable the surrogate");
            return MDX_ERR_UNSUPPORTED;
        }
        size_t members = 0;
        for (auto &m : s->rigidFix()->mol_ids) members += m.w >= 0 ? 4 : 3;
        if (members != s->atoms.size()) {
            set_error(MDX_ERR_UNSUPPORTED, "batched replicas must be rigid water only (every atom in a molecule)");
            return MDX_ERR_UNSUPPORTED;
        }
    }
    // one neighbour team size for all (the pair and build kernels are templated on it)
    int team = s0.nThreadPerAtom;
    for (State *s : reps)
        if (s->nThreadPerAtom) team = s->nThreadPerAtom;
    if (!team) team = 8;
    for (State *s : reps) {
        if (s->nThreadPerAtom && s->nThreadPerAtom != team) {
            set_error(MDX_ERR_UNSUPPORTED, "replicas ask for different nThreadPerAtom");
            return MDX_ERR_UNSUPPORTED;
        }
        s->nThreadPerAtom = team;
    }
    // each replica in its own form: the molecule form where its box holds
    // the molecule list's minimum image (pairForm 0 or 2), else the per-site
    // form; a phase whose kernels differ by form launches once per form
    for (State *s : reps)
        if (!s->prepared)
            if (int e = s->prepare()) return e;
    MDX_CUDA_TRY(cudaDeviceSynchronize());
    max_n = max_mol = max_cell = 0;
    ps.clear();
    mfi.clear();
    max_n_ps = max_cell_ps = max_mol_mf = 0;
    for (int r = 0; r < (int)reps.size(); r++) {
        State *s = reps[r];
        max_n = std::max(max_n, s->gpd.n);
        max_mol = std::max(max_mol, (int)s->rigidFix()->mol_ids.size());
        max_cell = std::max(max_cell, s->grid.ns.x * s->grid.ns.y * s->grid.ns.z);
        if (s->mf.on) {
            mfi.push_back(r);
            max_mol_mf = std::max(max_mol_mf, (int)s->rigidFix()->mol_ids.size());
        } else {
            ps.push_back(r);
            max_n_ps = std::max(max_n_ps, s->gpd.n);
            max_cell_ps = std::max(max_cell_ps, s->grid.ns.x * s->grid.ns.y * s->grid.ns.z);
            if (s->grid.team != team) {
                set_error(MDX_ERR_STATE, "replica built with team %d, batch uses %d", s->grid.team, team);
                return MDX_ERR_STATE;
            }
        }
    }
    periodicInterval = s0.periodicInterval > 0 ? s0.periodicInterval : 1;
    turn = s0.turn;
    for (State *s : reps)
        if (s->turn != turn) {
            set_error(MDX_ERR_STATE, "replicas are at different turns");
            return MDX_ERR_STATE;
        }
    if (!stream) {
        MDX_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        for (auto &s : side) MDX_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        MDX_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        for (auto &e : ev_join) MDX_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    // every argument table is built here: nothing may allocate once the
    // step is being captured
    if (int e = batch_p3m_prepare(*this)) return e;
    if (int e = batch_pair_tables(*this)) return e;
    if (int e = batch_nlist_tables(*this)) return e;
    if (int e = batch_mol_tables(*this)) return e;
    if (e3b0)
        if (int e = batch_e3b_tables(*this)) return e;
    MDX_CUDA_TRY(cudaDeviceSynchronize());
    prepared = true;
    return 0;
}

// the fused step of IntegratorVerlet (P3M chain and E3B on side streams beside
// the pair kernel) with every launch covering all replicas
int Batch::step() {
    const bool e3b = reps[0]->e3bFix() != nullptr;
    if (int e = batch_first_half(*this)) return e;
    MDX_CUDA_TRY(cudaEventRecord(ev_fork, stream));
    MDX_CUDA_TRY(cudaStreamWaitEvent(side[0], ev_fork, 0));
    if (int e = batch_p3m_spread_solve(*this, side[0])) return e;
    if (p3m_mol)  // the gather on the P3M branch, beside the pair kernel
        if (int e = batch_p3m_gather(*this, side[0])) return e;
    MDX_CUDA_TRY(cudaEventRecord(ev_join[0], side[0]));
    if (e3b) {
        MDX_CUDA_TRY(cudaStreamWaitEvent(side[1], ev_fork, 0));
        if (int e = batch_e3b_forces(*this, side[1])) return e;
        MDX_CUDA_TRY(cudaEventRecord(ev_join[1], side[1]));
    }
    if (int e = batch_pair_launch(*this, stream)) return e;
    MDX_CUDA_TRY(cudaStreamWaitEvent(stream, ev_join[0], 0));
    if (!p3m_mol)
        if (int e = batch_p3m_gather(*this, stream)) return e;
    if (e3b) MDX_CUDA_TRY(cudaStreamWaitEvent(stream, ev_join[1], 0));
    return batch_second_half(*this, e3b);
}

int Batch::enqueue(int nsteps, bool with_group) {
    if (with_group)
        if (int e = batch_nlist_rebuild(*this)) return e;
    for (int k = 0; k < nsteps; k++)
        if (int e = step()) return e;
    return 0;
}

int Batch::launchGraph(int nsteps, bool with_group) {
    const auto key = std::make_pair(nsteps, with_group ? 1 : 0);
    auto it = graphs.find(key);
    if (it == graphs.end()) {
        cudaGraph_t g;
        MDX_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const uint64_t before = g_launches;
        int e = enqueue(nsteps, with_group);
        const uint64_t captured = g_launches - before;
        g_launches = before;
        cudaError_t ce = cudaStreamEndCapture(stream, &g);
        if (e) return e;
        if (ce != cudaSuccess) {
            set_error(MDX_ERR_CUDA, "batch graph capture failed: %s", cudaGetErrorString(ce));
            return MDX_ERR_CUDA;
        }
        cudaGraphExec_t ex;
        MDX_CUDA_TRY(cudaGraphInstantiate(&ex, g, cudaGraphInstantiateFlagUseNodePriority));
        cudaGraphDestroy(g);
        it = graphs.emplace(key, ex).first;
        graph_kernels[key] = captured;
    }
    MDX_CUDA_TRY(cudaGraphLaunch(it->second, stream));
    g_launches += graph_kernels[key];
    return 0;
}

int Batch::checkStatus() {
    for (State *s : reps) {
        s->turn = turn;
        if (int e = s->checkStatus()) return e;
    }
    return 0;
}

int Batch::run(int nturns, double *ms) {
    if (nturns < 0) {
        set_error(MDX_ERR_ARG, "numTurns must be >= 0");
        return MDX_ERR_ARG;
    }
    if (!prepared)
        if (int e = prepare()) return e;
    cudaEvent_t e0, e1;
    MDX_CUDA_TRY(cudaEventCreate(&e0));
    MDX_CUDA_TRY(cudaEventCreate(&e1));
    MDX_CUDA_TRY(cudaEventRecord(e0, stream));
    const int P = periodicInterval;
    int done = 0;
    while (done < nturns) {
        const bool check = (turn % P) == 0;
        int c = check ? P : (int)(P - (turn % P));
        c = std::min(c, nturns - done);
        if (int e = launchGraph(c, check)) return e;
        turn += c;
        done += c;
    }
    MDX_CUDA_TRY(cudaEventRecord(e1, stream));
    MDX_CUDA_TRY(cudaEventSynchronize(e1));
    float t = 0.f;
    MDX_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = t;
    // FixNoseHoover::postRun per replica, then the status of every replica
    if (nturns > 0)
        for (State *s : reps)
            if (int e = nh_end_of_run(*s)) return e;
    return checkStatus();
}

int Batch::runTimed(int nturns, int chunk, size_t flush_bytes, double *ms_total) {
    if (!prepared)
        if (int e = prepare()) return e;
    DBuf<char> flush;
    if (flush_bytes)
        if (int e = flush.alloc(flush_bytes)) return e;
    const int P = periodicInterval;
    std::vector<cudaEvent_t> ev;
    int done = 0;
    while (done < nturns) {
        if (flush_bytes) MDX_CUDA_TRY(cudaMemsetAsync(flush.p, (int)(done & 0xff), flush_bytes, stream));
        cudaEvent_t a, b;
        MDX_CUDA_TRY(cudaEventCreate(&a));
        MDX_CUDA_TRY(cudaEventCreate(&b));
        MDX_CUDA_TRY(cudaEventRecord(a, stream));
        int todo = std::min(chunk, nturns - done);
        while (todo > 0) {
            const bool check = (turn % P) == 0;
            int c = check ? P : (int)(P - (turn % P));
            c = std::min(c, todo);
            if (int e = launchGraph(c, check)) return e;
            turn += c;
            todo -= c;
            done += c;
        }
        MDX_CUDA_TRY(cudaEventRecord(b, stream));
        ev.push_back(a);
        ev.push_back(b);
    }
    MDX_CUDA_TRY(cudaStreamSynchronize(stream));
    double tot = 0.0;
    for (size_t k = 0; k < ev.size(); k += 2) {
        float ms = 0.f;
        MDX_CUDA_TRY(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
        tot += ms;
        cudaEventDestroy(ev[k]);
        cudaEventDestroy(ev[k + 1]);
    }
    *ms_total = tot;
    return checkStatus();
}

}  // namespace mdx

using namespace mdx;

extern "C" {

int mdx_batch_create(mdx_batch **out) {
    if (!out) {
        set_error(MDX_ERR_ARG, "null argument");
        return MDX_ERR_ARG;
    }
    *out = new mdx_batch{new Batch()};
    return 0;
}

int mdx_batch_add(mdx_batch *b, mdx_state *st) {
    if (!b || !st) {
        set_error(MDX_ERR_ARG, "null argument");
        return MDX_ERR_ARG;
    }
    if (b->b->prepared) {
        set_error(MDX_ERR_STATE, "batch already prepared");
        return MDX_ERR_STATE;
    }
    for (State *s : b->b->reps)
        if (s == st->s) {
            set_error(MDX_ERR_ARG, "state already in the batch");
            return MDX_ERR_ARG;
        }
    b->b->reps.push_back(st->s);
    return 0;
}

int mdx_batch_size(mdx_batch *b, int *n) {
    if (!b || !n) {
        set_error(MDX_ERR_ARG, "null argument");
        return MDX_ERR_ARG;
    }
    *n = (int)b->b->reps.size();
    return 0;
}

int mdx_batch_prepare(mdx_batch *b) {
    if (!b) {
        set_error(MDX_ERR_ARG, "null batch");
        return MDX_ERR_ARG;
    }
    try {
        return b->b->prepare();
    } catch (...) {
        set_error(MDX_ERR_STATE, "exception in batch prepare");
        return MDX_ERR_STATE;
    }
}

int mdx_batch_run(mdx_batch *b, int num_turns, double *device_ms) {
    if (!b) {
        set_error(MDX_ERR_ARG, "null batch");
        return MDX_ERR_ARG;
    }
    try {
        return b->b->run(num_turns, device_ms);
    } catch (...) {
        set_error(MDX_ERR_STATE, "exception in batch run");
        return MDX_ERR_STATE;
    }
}

int mdx_batch_run_timed(mdx_batch *b, int num_turns, int chunk, size_t flush_bytes, double *device_ms) {
    if (!b || !device_ms || num_turns < 0 || chunk <= 0) {
        set_error(MDX_ERR_ARG, "bad argument");
        return MDX_ERR_ARG;
    }
    try {
        return b->b->runTimed(num_turns, chunk, flush_bytes, device_ms);
    } catch (...) {
        set_error(MDX_ERR_STATE, "exception in batch run");
        return MDX_ERR_STATE;
    }
}

int mdx_batch_autotune(mdx_batch *b, int steps, const int *teams, int nteams, int *best_team, double *best_ms) {
    if (!b) {
        set_error(MDX_ERR_ARG, "null batch");
        return MDX_ERR_ARG;
    }
    try {
        return b->b->autotune(steps, teams, nteams, best_team, best_ms);
    } catch (...) {
        set_error(MDX_ERR_STATE, "exception in batch autotune");
        return MDX_ERR_STATE;
    }
}

int mdx_batch_destroy(mdx_batch *b) {
    if (!b) return 0;
    delete b->b;
    delete b;
    return 0;
}

}  // extern "C"
