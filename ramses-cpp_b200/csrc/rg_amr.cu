// rg_amr.cu -- the coarse step of a run whose tree and state are resident on
// the device (rg_tree_attach), as one native call.
//
// Replays Simulation::run's coarse step (RAMSES-CPP src/core/Simulation.cpp:
// 366-397: refine the domain below levelmin, amr_step(levelmin, 1), flag every
// level from levelmin down, restrict) and Simulation::amr_step (:522-635:
// refine / remove the finer levels, CFL step capped by the coarser level's dt
// over its sub-cycles, set_unew, the finer sub-steps, godunov_fine, set_uold,
// restrict_fine, flag_fine of the next finer level) with every grid and hydro
// call on the device: the host only reads the level counts (kept on the host)
// and one dt per level step.  Sub-cycling 2 from levelmin on, 1 below, as
// Simulation's nsubcycle_ default.  Physics modules the hydro configs switch
// off (turbulence, sinks, stars, cooling, RT) are not called.
#include <algorithm>

#include "rg_internal.cuh"

namespace rg {
namespace {

constexpr int kMaxLevel = 32;

struct AmrRunState {
    double dtnew[kMaxLevel + 1] = {}, dtold[kMaxLevel + 1] = {};
    double t = 0.0;
    long long nstep = 0, cell_updates = 0;
};

int count_grids(const rg_ctx* c, int il) {
    if (il < 0 || il > c->nlevelmax) return 0;
    return c->h_numbl[(size_t)il * (c->ncpu + c->nboundary)];
}

int nsubcycle(const rg_amr_config& cfg, int il) { return il >= cfg.levelmin ? 2 : 1; }

int amr_step(rg_ctx* c, const rg_amr_config& cfg, AmrRunState& S, int il, int icount) {
    const int lmin = cfg.levelmin, lmax = c->nlevelmax;
    if (il > lmax) return RG_OK;
    if (count_grids(c, il) == 0 && il > 0) return RG_OK;
    if (lmin < lmax && (il == lmin || icount > 1)) {
        for (int i = il; i <= lmax; ++i)
            if (int rc = tree_make_grid_fine(c, i + 1)) return rc;
        for (int i = lmax; i >= il; --i)
            if (int rc = tree_remove_grid_fine(c, i + 1)) return rc;
    }
    const double dx = cfg.boxlen / (double)(c->nx * (1 << il));
    S.dtold[il] = S.dtnew[il];
    if (int rc = rg_courant_step(c, il, dx, cfg.courant_factor, cfg.pressure_cap, &S.dtnew[il])) return rc;
    if (il > lmin) {
        const double cand = S.dtnew[il - 1] / (double)nsubcycle(cfg, il - 1);
        S.dtnew[il] = std::min(S.dtnew[il], cand);
    }
    const double dt = S.dtnew[il];
    if (int rc = rg_set_unew(c, il)) return rc;
    const int nsub = nsubcycle(cfg, il);
    if (il < lmax) {
        if (count_grids(c, il + 1) > 0) {
            for (int i = 1; i <= nsub; ++i)
                if (int rc = amr_step(c, cfg, S, il + 1, i)) return rc;
        } else {
            S.dtold[il + 1] = S.dtnew[il] / (double)nsub;
            S.dtnew[il + 1] = S.dtnew[il] / (double)nsub;
            S.t += dt;
            S.nstep++;
        }
    } else {
        S.t += dt;
        S.nstep++;
    }
    if (int rc = rg_godunov_level(c, il, dt, dx)) return rc;
    S.cell_updates += rg_level_cell_updates(c, il);
    if (int rc = rg_set_uold(c, il)) return rc;
    if (il < lmax)
        if (int rc = tree_restrict_fine(c, il)) return rc;
    return tree_flag_fine(c, il + 1, cfg.err_grad_d, cfg.err_grad_p, cfg.err_grad_u, -1.0, cfg.nexpand, icount,
                          il > 0 ? nsubcycle(cfg, il - 1) : 1);
}

}  // namespace
}  // namespace rg

using namespace rg;

extern "C" int rg_amr_coarse_step(rg_ctx* c, const rg_amr_config* cfg, rg_amr_clock* clock) {
    if (!c) return RG_ERR_ARG;
    if (c->broken) return set_error(c, RG_ERR_CUDA, c->err.empty() ? "context unusable after a device fault" : c->err);
    if (!cfg || !clock) return set_error(c, RG_ERR_ARG, "config and clock required");
    if (!c->tree_resident) return set_error(c, RG_ERR_STATE, "no device-resident tree: call rg_tree_attach first");
    if (c->nlevelmax > kMaxLevel) return set_error(c, RG_ERR_UNSUPPORTED, "nlevelmax above 32");
    if (cfg->levelmin < 1 || cfg->levelmin > c->nlevelmax) return set_error(c, RG_ERR_ARG, "levelmin outside 1..nlevelmax");
    if (!(cfg->boxlen > 0.0)) return set_error(c, RG_ERR_ARG, "boxlen must be positive");
    cudaSetDevice(c->device);
    AmrRunState S;
    std::copy(clock->dtnew, clock->dtnew + kMaxLevel + 1, S.dtnew);
    std::copy(clock->dtold, clock->dtold + kMaxLevel + 1, S.dtold);
    S.t = clock->t;
    S.nstep = clock->nstep;
    S.cell_updates = clock->cell_updates;
    const int lmin = cfg->levelmin, lmax = c->nlevelmax;
    if (lmin < lmax)
        for (int il = 1; il <= lmin - 1; ++il)
            if (int rc = tree_make_grid_fine(c, il)) return rc;
    if (int rc = amr_step(c, *cfg, S, lmin, 1)) return rc;
    for (int il = lmin; il >= 1; --il)
        if (int rc = tree_flag_fine(c, il, cfg->err_grad_d, cfg->err_grad_p, cfg->err_grad_u, -1.0, cfg->nexpand, 2, 2))
            return rc;
    if (lmin < lmax)
        for (int il = lmin - 1; il >= 0; --il)
            if (int rc = tree_restrict_fine(c, il)) return rc;
    std::copy(S.dtnew, S.dtnew + kMaxLevel + 1, clock->dtnew);
    std::copy(S.dtold, S.dtold + kMaxLevel + 1, clock->dtold);
    clock->t = S.t;
    clock->nstep = S.nstep;
    clock->cell_updates = S.cell_updates;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "coarse step");
}
