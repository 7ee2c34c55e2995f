// rg_amr.cu -- the coarse step of a run whose tree and state are resident on
// the device (rg_tree_attach), as one native call.
//
// Replays Simulation::run's coarse step (RAMSES-CPP src/core/Simulation.cpp:
// 366-397: refine the domain below levelmin, amr_step(levelmin, 1), flag every
// level from levelmin down, restrict) and Simulation::amr_step (:522-635:
// refine / remove the finer levels, CFL step capped by the coarser level's dt
// over its sub-cycles, set_unew, the finer sub-steps, godunov_fine, set_uold,
// restrict_fine, flag_fine of the next finer level) with every grid and hydro
// call on the device.  The clock (each level's dtnew / dtold and the time)
// lives in device memory for the step: the CFL step, its cap by the coarser
// level's dt over its sub-cycles and the time updates are single-thread
// kernels with the host's arithmetic, since the control flow depends only on
// the level counts, which the host keeps; so the host reads no dt back.
// Sub-cycling 2 from levelmin on, 1 below, as
// Simulation's nsubcycle_ default.  Physics modules the hydro configs switch
// off (turbulence, sinks, stars, cooling, RT) are not called.
#include <algorithm>
#include <cstring>

#include "rg_internal.cuh"

namespace rg {
namespace {

constexpr int kMaxLevel = kClockLevels - 1;
// device clock: dtnew[0..32], dtold[0..32], t (ClockStep's layout)
constexpr int kDtOld = kClockDtOld, kClockT = kClockTime, kClockN = kClockT + 1;

enum RunMode { RUN_EAGER, RUN_CAPTURE, RUN_REPLAY };

struct AmrRunState {
    double* ck = nullptr;  // device clock
    long long nstep = 0, cell_updates = 0;
    const rg_amr_config* cfg = nullptr;
    // the current run (the level-step segments between two of the host's
    // waits): its index in the coarse step, how it is issued, and whether an
    // eager visit may count as the warm-up of a capture
    int run = 0;
    RunMode mode = RUN_EAGER;
    bool open = false, warm_ok = false;
    long long topo = -1;
};

__global__ void k_arm_cfl(DevStatus* st, double dt_start) {
    st->dtmin_bits = (unsigned long long)__double_as_longlong(dt_start);
}


int count_grids(const rg_ctx* c, int il) {
    if (il < 0 || il > c->nlevelmax) return 0;
    return c->h_numbl[(size_t)il * (c->ncpu + c->nboundary)];
}

int nsubcycle(const rg_amr_config& cfg, int il) { return il >= cfg.levelmin ? 2 : 1; }

// The coarse step as CUDA graphs.  Between tree changes a level step issues
// the same kernels with the same arguments every time: the CFL pass with
// set_unew and the clock update before the finer sub-steps, and after them
// the level step proper (dt, primitives, face, fold with set_uold),
// restrict_fine and flag_fine; on a level without finer octs both halves and
// the time update form one segment.  The host waits only at the change
// probes, so the segments between two probes -- a run -- form one graph.  At
// a run's first visit at a topology version every cache its segments touch is
// prepared (the plans, the face shapes, the flux scratch size, the level oct
// lists: prepare_run) and the run is captured whole; it is replayed from then
// on until the tree changes (the topology version moves), a scratch buffer it
// names is reallocated or the configuration differs.  When the preparation
// cannot finish (a level whose face shape waits to be timed) the run goes
// eagerly once, which warms the rest, and is captured at its next visit.  A
// replay is launched at the run's start; the host still walks the step's
// recursion (the probes and the counts depend on it), issuing nothing.  A
// captured run calls nothing that waits or allocates: a segment that is not
// ready for capture ends the capture there, the part captured so far is
// launched and the rest of the run goes eagerly.
bool segment_ok(rg_ctx* c, int il) {
    if (!c->amr_graphs_on || c->timing || c->tree_dirty || !c->d_tscr) return false;
    Plan* P = existing_plan(c, il);
    if (!P) return false;
    // a level without a leaf cell launches no face kernel (no shape, no scratch)
    if (P->ncells > 0 && P->nactive > 0) {
        if (P->face_variant < 0) return false;
        const size_t need = (size_t)(2 * c->params.ndim + 1) * (c->params.ndim + 2) * (size_t)P->ncells;
        if (c->cap_flux < need || !c->d_flux) return false;
    }
    // the finer level's oct list, which restrict_fine and flag_fine read
    const int L = il + 1;
    if (L <= c->nlevelmax && count_grids(c, L) > 0)
        if ((int)c->lvl_ver.size() <= L || c->lvl_ver[(size_t)L] != c->topo_version) return false;
    return true;
}

bool same_cfg(const rg_amr_config& a, const rg_amr_config& b) {
    return a.levelmin == b.levelmin && a.nexpand == b.nexpand && a.courant_factor == b.courant_factor &&
           a.err_grad_d == b.err_grad_d && a.err_grad_p == b.err_grad_p && a.err_grad_u == b.err_grad_u &&
           a.pressure_cap == b.pressure_cap && a.boxlen == b.boxlen;
}

// Everything a run can touch made ready ahead of a capture: every stepped
// level's plan, flux scratch and face shape, every level's oct list.  A run
// warmed this way is captured at its first visit; false (nothing captured)
// when a level waits for its shape to be timed, or the tree scratch is not
// there yet.
int prepare_run(rg_ctx* c, const rg_amr_config& cfg, bool* ready) {
    *ready = false;
    if (!c->d_tscr) return RG_OK;
    bool ok = true;
    for (int L = cfg.levelmin; L <= c->nlevelmax && ok; ++L)
        if (count_grids(c, L) > 0)
            if (int rc = prepare_level_step(c, L, &ok)) return rc;
    if (!ok) return RG_OK;
    for (int L = 1; L <= c->nlevelmax; ++L) {
        if (count_grids(c, L) == 0) continue;
        const int* octs = nullptr;
        int noct = 0;
        if (int rc = level_octs_cached(c, L, &octs, &noct)) return rc;
    }
    *ready = !c->tree_dirty;
    return RG_OK;
}

int run_begin(rg_ctx* c, AmrRunState& S) {
    // settle the topology first: a run never changes it, so its version holds
    // for every segment of the run
    if (int rc = refresh_tree(c)) return rc;
    RunGraph& g = c->amr_graphs[S.run];
    const long long v = c->topo_version;
    const bool base = c->amr_graphs_on && !c->timing && !c->tree_dirty && c->d_tscr;
    S.open = true;
    S.topo = v;
    S.warm_ok = false;
    if (base && g.exec && g.topo == v && g.flux == c->d_flux && g.tscr == c->d_tscr && same_cfg(g.cfg, *S.cfg)) {
        // issued at once: the device works through the run while the host
        // walks the same recursion to the run's end, issuing nothing
        S.mode = RUN_REPLAY;
        ++c->amr_replayed;
        return check_cuda(c, cudaGraphLaunch(g.exec, c->stream), "coarse-step graph");
    }
    bool warm = base && g.failed != v && g.warm == v && same_cfg(g.cfg, *S.cfg);
    if (base && g.failed != v && !warm) {
        // first visit at this topology: warm the caches here and capture now
        if (int rc = prepare_run(c, *S.cfg, &warm)) return rc;
        warm = warm && c->topo_version == v;
    }
    if (warm) {
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            S.mode = RUN_CAPTURE;
            g.flux = c->d_flux;
            g.tscr = c->d_tscr;
            return RG_OK;
        }
        cudaGetLastError();
        g.failed = v;
    }
    S.mode = RUN_EAGER;
    S.warm_ok = base;
    return RG_OK;
}

// end a capture and launch what it holds (the whole run, or the part before a
// segment that could not be captured); keep it for replays when it is whole
int run_launch_capture(rg_ctx* c, AmrRunState& S, bool whole) {
    RunGraph& g = c->amr_graphs[S.run];
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    bool good = e == cudaSuccess && graph != nullptr;
    if (good && g.exec) {
        // after a tree change a run usually issues the same kernels with new
        // sizes and pointers: updating the old executable graph in place costs
        // a fraction of instantiating a new one (launches already queued keep
        // the old parameters)
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(g.exec, graph, &info) == cudaSuccess) {
            exec = g.exec;
        } else {
            cudaGetLastError();
            cudaGraphExecDestroy(g.exec);
        }
        g.exec = nullptr;
    } else if (g.exec) {
        cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    if (good && !exec) good = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!good || g.flux != c->d_flux || g.tscr != c->d_tscr) {
        // the captured work cannot be issued: the step is incomplete
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        g.failed = S.topo;
        c->broken = true;
        return set_error(c, RG_ERR_CUDA, "a captured run of the coarse step could not be instantiated");
    }
    const cudaError_t le = cudaGraphLaunch(exec, c->stream);
    if (whole) {
        g.exec = exec;
        g.topo = S.topo;
        g.cfg = *S.cfg;
        ++c->amr_captured;
    } else {
        cudaGraphExecDestroy(exec);  // the launch keeps what it needs
        g.failed = S.topo;
    }
    return check_cuda(c, le, "coarse-step graph");
}

int run_end(rg_ctx* c, AmrRunState& S) {
    if (!S.open) return RG_OK;
    S.open = false;
    RunGraph& g = c->amr_graphs[S.run];
    int rc = RG_OK;
    if (S.mode == RUN_CAPTURE) {
        rc = run_launch_capture(c, S, true);
    } else if (S.warm_ok && c->topo_version == S.topo && !c->tree_dirty) {
        g.warm = S.topo;
        g.cfg = *S.cfg;
    }
    ++S.run;
    return rc;
}

// an error inside a run: leave the stream out of capture
void run_abort(rg_ctx* c, AmrRunState& S) {
    if (S.open && S.mode == RUN_CAPTURE) {
        cudaGraph_t graph = nullptr;
        cudaStreamEndCapture(c->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        c->amr_graphs[S.run].failed = S.topo;
    }
    S.open = false;
}

template <class F>
int run_segment(rg_ctx* c, AmrRunState& S, bool ok, F&& body) {
    if (S.mode == RUN_REPLAY) return RG_OK;
    if (S.mode == RUN_CAPTURE && !ok) {
        if (int rc = run_launch_capture(c, S, false)) return rc;
        S.mode = RUN_EAGER;
        S.warm_ok = false;
    }
    return body();
}


// The refinements and removals that open a level step, make_grid_fine(L)
// for L = lo..hi then remove_grid_fine(L) for L = hi..lo, skipping the calls
// that cannot change the tree by the probe `ch` and by what the calls before
// them changed: make_grid_fine(L) runs when list L has refinement candidates
// or make_grid_fine(L - 1) created octs, remove_grid_fine(L) when list L has
// removal candidates or remove_grid_fine(L + 1) freed octs.  Every call that
// is skipped would have found no candidate, so the tree ends as the full
// sequence leaves it.
int refine_and_remove(rg_ctx* c, int lo, int hi, const TreeChanges& ch, int* made_total = nullptr) {
    int made = 0, freed = 0, total = 0;
    for (int L = lo; L <= hi; ++L) {
        const bool run = (L < 64 && (ch.refine >> L) & 1ull) || made > 0;
        made = 0;
        if (run)
            if (int rc = tree_make_grid_fine(c, L, &made)) return rc;
        total += made;
    }
    for (int L = hi; L >= lo; --L) {
        const bool run = (L < 64 && (ch.kill >> L) & 1ull) || freed > 0;
        freed = 0;
        if (run)
            if (int rc = tree_remove_grid_fine(c, L, &freed)) return rc;
    }
    if (made_total) *made_total = total;
    return RG_OK;
}

// probed: what the caller's probe of this step's refinement levels leaves to
// do, with nothing changing the tree since (nullptr: probe here)
int amr_step(rg_ctx* c, const rg_amr_config& cfg, AmrRunState& S, int il, int icount,
             const TreeChanges* probed = nullptr) {
    const int lmin = cfg.levelmin, lmax = c->nlevelmax;
    if (il > lmax) return RG_OK;
    if (count_grids(c, il) == 0 && il > 0) return RG_OK;
    if (lmin < lmax && (il == lmin || icount > 1)) {
        // one probe instead of a scan and a read-back per call; the host waits
        // for it, so the run of segments before it ends here
        const uint64_t m = level_bits(il + 1, std::min(lmax, c->nlevelmax - 1));
        TreeChanges ch;
        if (probed) {
            ch = *probed;
        } else if (m) {
            if (int rc = run_end(c, S)) return rc;
            if (int rc = tree_changes_pending(c, m, &ch)) return rc;
        }
        if (ch.any(m))
            if (int rc = refine_and_remove(c, il + 1, lmax + 1, ch)) return rc;
        if (!probed && m)
            if (int rc = run_begin(c, S)) return rc;
    }
    const double dx = cfg.boxlen / (double)(c->nx * (1 << il));
    const int nsub = nsubcycle(cfg, il);
    const bool finer = il < lmax && count_grids(c, il + 1) > 0;
    double* ck = S.ck;
    // before the finer sub-steps: the CFL pass, which also does set_unew (both
    // read the level's uold, nothing between them writes it; the clock update only
    // reads the CFL word), and the level's new dt
    // On a level without finer octs the level step follows at once: the CFL
    // pass then also forms the primitives (uold changes in between for none
    // of the cells they are read from) and sets the step values.
    auto pre = [&]() -> int {
        ClockStep cs;
        cs.ck = ck;
        cs.il = il;
        cs.nsub_coarser = il > lmin ? nsubcycle(cfg, il - 1) : 0;
        cs.finer = finer ? 0 : (il < lmax ? 1 : 2);
        cs.nsub = nsub;
        cs.dt_start = c->params.boxlen / 1e-10;
        cs.set_step = finer ? 0 : 1;
        cs.dx = dx;
        return courant_step_device(c, il, dx, cfg.courant_factor, cfg.pressure_cap, true, true, &cs, !finer);
    };
    // after them: the level step with set_uold folded into the fold kernels (a
    // level target's result goes to uold as well; the fold reads only unew and
    // the flux scratch), restrict_fine, flag_fine of the next finer level.
    // This level's dtnew is still the one set above: the finer steps only
    // change the finer levels' entries.
    auto post = [&]() -> int {
        if (int rc = godunov_level_device_dt(c, il, ck + il, dx, true, !finer)) return rc;
        if (Plan* P = existing_plan(c, il); P == nullptr || P->ncells == 0)
            if (int rc = rg_set_uold(c, il)) return rc;
        if (il < lmax)
            if (int rc = tree_restrict_fine(c, il)) return rc;
        return tree_flag_fine(c, il + 1, cfg.err_grad_d, cfg.err_grad_p, cfg.err_grad_u, -1.0, cfg.nexpand, icount,
                              il > 0 ? nsubcycle(cfg, il - 1) : 1);
    };
    if (!finer) {
        if (int rc = run_segment(c, S, segment_ok(c, il), [&]() -> int {
                if (int rc = pre()) return rc;
                return post();
            }))
            return rc;
        S.nstep++;
    } else {
        if (int rc = run_segment(c, S, segment_ok(c, il), pre)) return rc;
        for (int i = 1; i <= nsub; ++i)
            if (int rc = amr_step(c, cfg, S, il + 1, i)) return rc;
        if (int rc = run_segment(c, S, segment_ok(c, il), post)) return rc;
    }
    S.cell_updates += rg_level_cell_updates(c, il);
    return RG_OK;
}

int coarse_step(rg_ctx* c, const rg_amr_config& cfgr, AmrRunState& S) {
    const rg_amr_config* cfg = &cfgr;
    const int lmin = cfg->levelmin, lmax = c->nlevelmax;
    TreeChanges ch;
    bool created = false;
    if (lmin < lmax) {
        // one probe for the refinements of the levels below levelmin (complete
        // after the initialisation, so normally nothing) and for the
        // refinements and removals that open amr_step(levelmin, 1), which
        // follows them directly; make_grid_fine of a level below levelmin runs
        // when the probe or the refinement of the level before asks for it
        if (int rc = tree_changes_pending(c, level_bits(1, lmin - 1) | level_bits(lmin + 1, lmax), &ch)) return rc;
        int made = 0;
        for (int il = 1; il <= lmin - 1; ++il) {
            const bool run = (il < 64 && (ch.refine >> il) & 1ull) || made > 0;
            made = 0;
            if (run)
                if (int rc = tree_make_grid_fine(c, il, &made)) return rc;
            created = created || made > 0;
        }
    }
    // the refinements and removals that open amr_step(levelmin, 1), issued
    // here so that the run of segments starts after them (when nothing was
    // created below levelmin the probe still holds for them)
    TreeChanges done;
    done.refine = done.kill = 0;
    if (lmin < lmax) {
        const uint64_t m = level_bits(lmin + 1, std::min(lmax, c->nlevelmax - 1));
        if (created && m)
            if (int rc = tree_changes_pending(c, m, &ch)) return rc;
        if (ch.any(m))
            if (int rc = refine_and_remove(c, lmin + 1, lmax + 1, ch)) return rc;
    }
    if (int rc = run_begin(c, S)) return rc;
    if (int rc = amr_step(c, *cfg, S, lmin, 1, lmin < lmax ? &done : nullptr)) return rc;
    // the step's tail: flag_fine from levelmin down and the restrictions below
    // levelmin, one segment like the level steps' (it reads the oct lists of
    // levels 1..levelmin, which must be current for a capture)
    auto tail = [&]() -> int {
        if (int rc = tree_flag_fine(c, lmin, cfg->err_grad_d, cfg->err_grad_p, cfg->err_grad_u, -1.0, cfg->nexpand,
                                    2, 2))
            return rc;
        // the levels below levelmin (all cells flagged, restrictions) in two
        // launches when they are small, else call by call
        bool fused = false;
        if (int rc = tree_tail_below_min(c, lmin, lmin < lmax, &fused)) return rc;
        if (fused) return RG_OK;
        for (int il = lmin - 1; il >= 1; --il)
            if (int rc = tree_flag_fine(c, il, cfg->err_grad_d, cfg->err_grad_p, cfg->err_grad_u, -1.0, cfg->nexpand,
                                        2, 2))
                return rc;
        if (lmin < lmax)
            for (int il = lmin - 1; il >= 0; --il)
                if (int rc = tree_restrict_fine(c, il)) return rc;
        return RG_OK;
    };
    bool tail_ok = c->amr_graphs_on && !c->timing && !c->tree_dirty && c->d_tscr;
    for (int L = 1; tail_ok && L <= lmin && L <= lmax; ++L)
        if (count_grids(c, L) > 0 && ((int)c->lvl_ver.size() <= L || c->lvl_ver[(size_t)L] != c->topo_version))
            tail_ok = false;
    if (int rc = run_segment(c, S, tail_ok, tail)) return rc;
    // what flag_fine(1) leaves on the host, which a replay does not
    if (lmin > 1 && lmax > 1) c->auth_dirty = true;
    if (int rc = run_end(c, S)) return rc;
    return check_cuda(c, cudaGetLastError(), "coarse-step clock kernels");
}

}  // namespace
}  // namespace rg

using namespace rg;

extern "C" int rg_amr_graphs(rg_ctx* c, int on, int64_t* captured, int64_t* replayed) {
    if (!c) return RG_ERR_ARG;
    if (on >= 0) c->amr_graphs_on = on != 0;
    if (captured) *captured = c->amr_captured;
    if (replayed) *replayed = c->amr_replayed;
    return RG_OK;
}

extern "C" int rg_amr_coarse_step(rg_ctx* c, const rg_amr_config* cfg, rg_amr_clock* clock) {
    if (!c) return RG_ERR_ARG;
    if (c->broken) return set_error(c, RG_ERR_CUDA, c->err.empty() ? "context unusable after a device fault" : c->err);
    if (!cfg || !clock) return set_error(c, RG_ERR_ARG, "config and clock required");
    if (!c->tree_resident) return set_error(c, RG_ERR_STATE, "no device-resident tree: call rg_tree_attach first");
    if (c->nlevelmax > kMaxLevel) return set_error(c, RG_ERR_UNSUPPORTED, "nlevelmax above 32");
    if (cfg->levelmin < 1 || cfg->levelmin > c->nlevelmax) return set_error(c, RG_ERR_ARG, "levelmin outside 1..nlevelmax");
    if (!(cfg->boxlen > 0.0)) return set_error(c, RG_ERR_ARG, "boxlen must be positive");
    cudaSetDevice(c->device);
    c->next_level = -1;  // replayed level steps skip that host bookkeeping
    AmrRunState S;
    double h[kClockN];
    std::copy(clock->dtnew, clock->dtnew + kMaxLevel + 1, h);
    std::copy(clock->dtold, clock->dtold + kMaxLevel + 1, h + kDtOld);
    h[kClockT] = clock->t;
    if (!c->d_clock)  // kept for the context's lifetime: captured level steps name it
        if (int rc = check_cuda(c, dev_alloc(c, &c->d_clock, sizeof(h)), "coarse-step clock")) return rc;
    if (!c->h_clock) {
        if (int rc = check_cuda(c, cudaMallocHost((void**)&c->h_clock, sizeof(h)), "coarse-step clock (host)"))
            return rc;
        c->clock_known = false;
    }
    S.ck = c->d_clock;
    // the device keeps the clock of the last step: send it only when the
    // caller's differs
    if (!c->clock_known || std::memcmp(c->h_clock, h, sizeof(h)) != 0) {
        c->clock_known = false;
        std::memcpy(c->h_clock, h, sizeof(h));
        if (int rc = check_cuda(c, cudaMemcpyAsync(S.ck, c->h_clock, sizeof(h), cudaMemcpyHostToDevice, c->stream),
                                "clock upload"))
            return rc;
    }
    S.nstep = clock->nstep;
    S.cell_updates = clock->cell_updates;
    S.cfg = cfg;
    // the CFL word's start value, as every CFL pass arms it (launch_courant);
    // each level's clock update (the CFL pass's last block) re-arms it after reading
    k_arm_cfl<<<1, 1, 0, c->stream>>>(c->d_status, c->params.boxlen / 1e-10);
    const int rc_step = coarse_step(c, *cfg, S);
    if (rc_step) run_abort(c, S);
    // the clock comes back with the step (the copy waits for it); on an error
    // the caller's clock is left as it was
    c->clock_known = false;
    const int rc_copy =
        check_cuda(c, cudaMemcpyAsync(c->h_clock, S.ck, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "clock");
    const int rc_sync = check_cuda(c, cudaStreamSynchronize(c->stream), "coarse step");
    if (rc_step) return rc_step;
    if (rc_copy) return rc_copy;
    if (rc_sync) return rc_sync;
    std::memcpy(h, c->h_clock, sizeof(h));
    c->clock_known = true;
    std::copy(h, h + kMaxLevel + 1, clock->dtnew);
    std::copy(h + kDtOld, h + kDtOld + kMaxLevel + 1, clock->dtold);
    clock->t = h[kClockT];
    clock->nstep = S.nstep;
    clock->cell_updates = S.cell_updates;
    return RG_OK;
}
