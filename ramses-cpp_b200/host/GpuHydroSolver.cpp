// GpuHydroSolver.cpp -- RAMSES-CPP hydro solver whose level step runs on a B200.
//
// Drop-in for the reference's patch seam: placed under patch/ and compiled
// with -DRAMSES_HAS_PATCH_HYDRO, it provides create_hydro_solver
// (include/ramses/core/SolverFactory.hpp:23, default at
// src/core/SolverFactory.cpp:5-9), so Simulation gets this class instead of
// HydroSolver and nothing else in the reference changes.  It overrides the
// virtual hot-path entry points of HydroSolver (HydroSolver.hpp:19-22:
// godunov_fine, set_unew, set_uold, compute_courant_step) and forwards them
// to librgpu.so through the C ABI of include/rgpu.h.
//
// State: the device keeps uold and unew of the whole grid between calls.
// AmrGrid still owns the host vectors, and the reference's TreeUpdater works
// on them between hydro calls: it reads uold (flag_fine, restrict_fine,
// make_grid_fine's interpolation), writes the refined cells' uold
// (restrict_fine) and the new cells' uold and unew (make_grid_fine), and
// never reads unew.  So a level step moves only its own cells: set_unew (or
// compute_courant_step, whichever comes first in the step) uploads the cells
// the step reads -- the level's cells and the coarser cells of its ghost
// stencils -- from the host uold, and set_uold downloads the level's cells of
// both arrays once the step is done; godunov_fine moves nothing.  The tree
// arrays are re-sent when the tree changed, detected from next[] and the
// level heads alone: every refinement or removal allocates or frees octs, and
// moving an oct between the free list and a level list rewrites a next[]
// entry (the predecessor's or the oct's own) or a head.  The state is sent
// whole at the start and whenever ngridmax changes (resize_grids relabels the
// cells).  Unsupported configurations (non-thermal energies, passive scalars,
// barotropic EOS, boundary patches) throw: there is no silent CPU fallback.
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "ramses/core/Parameters.hpp"
#include "ramses/core/SolverFactory.hpp"
#include "ramses/solvers/hydro/HydroSolver.hpp"
#include "rgpu.h"

namespace ramses {

class GpuHydroSolver : public HydroSolver {
public:
    GpuHydroSolver(AmrGrid& grid, Config& config) : HydroSolver(grid, config) {}
    ~GpuHydroSolver() override {
        if (ctx_) rg_destroy(ctx_);
    }

    real_t compute_courant_step(int ilevel, real_t dx, real_t gamma, real_t courant_factor) override {
        ensure_context();
        sync_topology();
        if (gamma != params_.gamma)
            throw std::runtime_error("GpuHydroSolver: compute_courant_step with a gamma other than the grid's");
        check(rg_upload_level(ctx_, ilevel, grid_.uold_vec.data()), "rg_upload_level");
        uploaded_level_ = ilevel;
        double dt = 0.0;
        check(rg_courant_step(ctx_, ilevel, dx, courant_factor, 1, &dt), "rg_courant_step");
        return dt;
    }

    void set_unew(int ilevel) override {
        ensure_context();
        sync_topology();
        if (uploaded_level_ != ilevel)  // compute_courant_step of this step already sent the level
            check(rg_upload_level(ctx_, ilevel, grid_.uold_vec.data()), "rg_upload_level");
        uploaded_level_ = -1;
        check(rg_set_unew(ctx_, ilevel), "rg_set_unew");
    }

    void godunov_fine(int ilevel, real_t dt, real_t dx) override {
        ensure_context();
        sync_topology();
        uploaded_level_ = -1;
        check(rg_godunov_level(ctx_, ilevel, dt, dx), "rg_godunov_level");
    }

    void set_uold(int ilevel) override {
        ensure_context();
        sync_topology();
        uploaded_level_ = -1;
        check(rg_set_uold(ctx_, ilevel), "rg_set_uold");
        check(rg_download_level(ctx_, ilevel, grid_.uold_vec.data(), grid_.unew_vec.data()), "rg_download_level");
    }

private:
    rg_ctx* ctx_ = nullptr;
    rg_params params_{};
    std::vector<int> sent_next_, sent_headl_;
    int sent_ngridmax_ = -1;
    int uploaded_level_ = -1;

    void check(int rc, const char* what) {
        if (rc != RG_OK)
            throw std::runtime_error(std::string("GpuHydroSolver: ") + what + " failed: " +
                                     (ctx_ ? rg_last_error(ctx_) : "no context"));
    }

    rg_params read_params() {
        // the knobs godunov_fine looks up per interface (HydroSolver.cpp:55,62,216-217,456)
        rg_params p{};
        p.ndim = NDIM;
        p.nvar = grid_.nvar;
        p.slope_type = config_.get_int("hydro_params", "slope_type", 1);
        p.riemann = rg_riemann_from_string(config_.get("hydro_params", "riemann", "llf").c_str());
        p.interpol_type = config_.get_int("refine_params", "interpol_type", 1);
        p.interpol_var = config_.get_int("refine_params", "interpol_var",
                                         config_.get_int("hydro_params", "interpol_var", 0));
        p.gamma = grid_.gamma;
        p.courant_factor = config_.get_double("hydro_params", "courant_factor", 0.8);
        p.exact_niter = 10;
        p.exact_tol = 1e-6;
        p.exact_guess = RG_GUESS_TWO_SHOCK;
        p.boxlen = params::boxlen;
        p.flags = 0;
        return p;
    }

    void ensure_context() {
        if (nener_ != 0 || params::barotropic_eos)
            throw std::runtime_error("GpuHydroSolver: non-thermal energies / barotropic EOS are not supported");
        rg_params p = read_params();
        if (!ctx_) {
            ctx_ = rg_create(&p, -1);
            if (!ctx_) throw std::runtime_error("GpuHydroSolver: rg_create failed");
            check(std::strlen(rg_last_error(ctx_)) == 0 ? RG_OK : RG_ERR_CUDA, "rg_create");
            params_ = p;
        } else if (std::memcmp(&p, &params_, sizeof(p)) != 0) {
            check(rg_set_params(ctx_, &p), "rg_set_params");
            params_ = p;
        }
    }

    static bool same(const std::vector<int>& a, const std::vector<int>& b) {
        return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(int)) == 0;
    }

    void sync_topology() {
        const bool resized = sent_ngridmax_ != grid_.ngridmax;
        const bool changed = resized || !same(sent_next_, grid_.next) || !same(sent_headl_, grid_.headl_vec);
        if (!changed) return;
        rg_grid_view v{};
        v.ncoarse = grid_.ncoarse;
        v.ngridmax = grid_.ngridmax;
        v.ncell = grid_.ncell;
        v.nvar = grid_.nvar;
        v.nx = grid_.nx;
        v.ny = grid_.ny;
        v.nz = grid_.nz;
        v.ncpu = grid_.ncpu;
        v.nboundary = grid_.nboundary;
        v.nlevelmax = grid_.nlevelmax;
        v.son = grid_.son.data();
        v.father = grid_.father.data();
        v.nbor = grid_.nbor.data();
        v.next = grid_.next.data();
        v.headl = grid_.headl_vec.data();
        v.bound_type = grid_.bound_type.empty() ? nullptr : grid_.bound_type.data();
        v.nbound_type = (int)grid_.bound_type.size();
        check(rg_sync_topology(ctx_, &v), "rg_sync_topology");
        if (resized)  // the first call, or resize_grids relabelled every cell
            check(rg_upload_state(ctx_, grid_.uold_vec.data(), grid_.unew_vec.data()), "rg_upload_state");
        uploaded_level_ = -1;
        sent_next_ = grid_.next;
        sent_headl_ = grid_.headl_vec;
        sent_ngridmax_ = grid_.ngridmax;
    }
};

std::unique_ptr<HydroSolver> create_hydro_solver(AmrGrid& grid, Config& config) {
    return std::make_unique<GpuHydroSolver>(grid, config);
}

}  // namespace ramses
