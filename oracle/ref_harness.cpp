// ref_harness.cpp -- extern "C" driver around the RAMSES-CPP reference.
//
// TEST INFRASTRUCTURE ONLY.  Linked against the reference's own objects,
// compiled from its sources in place by oracle/Makefile into oracle/_ref.
// Tests and the CPU-baseline leg of the benchmark load it with ctypes to run
// the unmodified reference path on synthetic grids:
//   - AmrGrid::allocate / TreeUpdater::{flag_fine, make_grid_fine,
//     remove_grid_fine, restrict_fine} build and evolve the tree exactly as
//     Simulation::initialize / amr_step do (src/core/Simulation.cpp:226-253,
//     522-635);
//   - HydroSolver::{set_unew, godunov_fine, set_uold, compute_courant_step}
//     are the hot path under test;
//   - RiemannSolver::solve_* and SlopeLimiter::compute_slope are exposed for
//     unit-level parity.
// Built with -DRG_GPU_PATCH (oracle/Makefile target "dropin") the same
// harness gets its solver from ramses-cpp_b200/host/GpuHydroSolver.cpp through
// the reference's create_hydro_solver seam, so tests run the unmodified
// reference API with the GPU level step dropped in.
// The namelist text is written to a temporary file because Config can only
// parse files (src/core/Config.cpp:25).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <unistd.h>

#include "ramses/core/AmrGrid.hpp"
#include "ramses/core/Config.hpp"
#include "ramses/core/Parameters.hpp"
#include "ramses/core/TreeUpdater.hpp"
#include "ramses/io/RamsesWriter.hpp"
#include "ramses/solvers/hydro/HydroSolver.hpp"
#include "ramses/solvers/hydro/RiemannSolver.hpp"
#include "ramses/solvers/hydro/SlopeLimiter.hpp"
#ifdef RG_GPU_PATCH
#include "ramses/core/SolverFactory.hpp"
#endif

namespace {
struct Harness {
    ramses::AmrGrid grid;
    ramses::Config config;
    std::unique_ptr<ramses::TreeUpdater> updater;
    std::unique_ptr<ramses::HydroSolver> hydro;
};
}  // namespace

extern "C" {

int rh_ndim(void) { return NDIM; }

void* rh_create(const char* nml_text, int nx, int ny, int nz, int ngridmax, int nvar, int levelmin,
                int nlevelmax, double gamma, double boxlen) {
    auto* h = new Harness();
    char path[] = "/tmp/rh_nml_XXXXXX";
    int fd = mkstemp(path);
    if (fd < 0) { delete h; return nullptr; }
    size_t len = strlen(nml_text);
    if (write(fd, nml_text, len) != (ssize_t)len) { close(fd); unlink(path); delete h; return nullptr; }
    close(fd);
    bool ok = h->config.parse(path);
    unlink(path);
    if (!ok) { delete h; return nullptr; }
    ramses::params::nx = nx;
    ramses::params::ny = ny;
    ramses::params::nz = nz;
    ramses::params::boxlen = boxlen;
    ramses::params::levelmin = levelmin;
    ramses::params::nlevelmax = nlevelmax;
    h->grid.allocate(nx, ny, nz, ngridmax, nvar, 1, nlevelmax);
    h->grid.gamma = gamma;
#ifdef RG_GPU_PATCH
    // the drop-in build: the solver comes from the patch's create_hydro_solver
    h->hydro = ramses::create_hydro_solver(h->grid, h->config);
#else
    h->hydro = std::make_unique<ramses::HydroSolver>(h->grid, h->config);
#endif
    h->hydro->set_nener(0);
    h->hydro->set_nvar_hydro(nvar);
    ramses::HydroSolver* hs = h->hydro.get();
    h->grid.set_interpol_hook([hs](const ramses::real_t u1[7][64], ramses::real_t u2[8][64]) { hs->interpol_hydro(u1, u2); });
    h->updater = std::make_unique<ramses::TreeUpdater>(h->grid, h->config);
    return h;
}

void rh_destroy(void* hp) { delete static_cast<Harness*>(hp); }

long long rh_get(void* hp, const char* name) {
    auto& g = static_cast<Harness*>(hp)->grid;
    std::string n(name);
    if (n == "ncoarse") return g.ncoarse;
    if (n == "ngridmax") return g.ngridmax;
    if (n == "ncell") return g.ncell;
    if (n == "nvar") return g.nvar;
    if (n == "nx") return g.nx;
    if (n == "ny") return g.ny;
    if (n == "nz") return g.nz;
    if (n == "ncpu") return g.ncpu;
    if (n == "nboundary") return g.nboundary;
    if (n == "nlevelmax") return g.nlevelmax;
    if (n == "numbf") return g.numbf;
    if (n == "headf") return g.headf;
    if (n == "tailf") return g.tailf;
    if (n == "headl_size") return (long long)g.headl_vec.size();
    return -1;
}

void* rh_ptr(void* hp, const char* name) {
    auto& g = static_cast<Harness*>(hp)->grid;
    std::string n(name);
    if (n == "uold") return g.uold_vec.data();
    if (n == "unew") return g.unew_vec.data();
    if (n == "son") return g.son.data();
    if (n == "father") return g.father.data();
    if (n == "nbor") return g.nbor.data();
    if (n == "next") return g.next.data();
    if (n == "prev") return g.prev.data();
    if (n == "headl") return g.headl_vec.data();
    if (n == "flag1") return g.flag1.data();
    if (n == "flag2") return g.flag2.data();
    if (n == "cpu_map") return g.cpu_map.data();
    if (n == "taill") return g.taill_vec.data();
    if (n == "numbl") return g.numbl_vec.data();
    if (n == "xg") return g.xg.data();
    return nullptr;
}

int rh_count_grids(void* hp, int ilevel) { return static_cast<Harness*>(hp)->grid.count_grids_at_level(ilevel); }

void rh_cell_center(void* hp, int icell, double* xc) { static_cast<Harness*>(hp)->grid.get_cell_center(icell, xc); }

void rh_flag_fine(void* hp, int il, double ed, double ep, double ev, double eb2, int nexp, int icount, int nsub) {
    static_cast<Harness*>(hp)->updater->flag_fine(il, ed, ep, ev, eb2, {}, nexp, icount, nsub);
}
void rh_make_grid_fine(void* hp, int il) { static_cast<Harness*>(hp)->updater->make_grid_fine(il); }
void rh_remove_grid_fine(void* hp, int il) { static_cast<Harness*>(hp)->updater->remove_grid_fine(il); }
void rh_restrict_fine(void* hp, int il) { static_cast<Harness*>(hp)->updater->restrict_fine(il); }

void rh_set_unew(void* hp, int il) { static_cast<Harness*>(hp)->hydro->set_unew(il); }
void rh_set_uold(void* hp, int il) { static_cast<Harness*>(hp)->hydro->set_uold(il); }
void rh_godunov_fine(void* hp, int il, double dt, double dx) { static_cast<Harness*>(hp)->hydro->godunov_fine(il, dt, dx); }
double rh_courant(void* hp, int il, double dx, double gamma, double cfl) {
    return static_cast<Harness*>(hp)->hydro->compute_courant_step(il, dx, gamma, cfl);
}
void rh_interpol_hydro(void* hp, const double* u1, double* u2) {
    ramses::real_t a[7][64], b[8][64];
    memcpy(a, u1, sizeof(a));
    static_cast<Harness*>(hp)->hydro->interpol_hydro(a, b);
    memcpy(u2, b, sizeof(b));
}

// The reference's hydro snapshot file (RamsesWriter::write_hydro,
// src/io/RamsesWriter.cpp:145-226) for the harness's current state.
void rh_write_hydro(void* hp, const char* path) {
    ramses::SnapshotInfo info{};
    info.gamma = static_cast<Harness*>(hp)->grid.gamma;
    ramses::RamsesWriter(path).write_hydro(static_cast<Harness*>(hp)->grid, info);
}

// Direct access to the public static kernels of the hot path.
int rh_riemann(const char* name, const double* ql, const double* qr, double* flux, double gamma) {
    std::string n(name);
    if (n == "hllc") ramses::RiemannSolver::solve_hllc(ql, qr, flux, gamma);
    else if (n == "hll") ramses::RiemannSolver::solve_hll(ql, qr, flux, gamma);
    else if (n == "exact") ramses::RiemannSolver::solve_godunov_nr(ql, qr, flux, gamma);
    else if (n == "acoustic") ramses::RiemannSolver::solve_acoustic(ql, qr, flux, gamma);
    else ramses::RiemannSolver::solve_llf(ql, qr, flux, gamma);
    return 0;
}
double rh_slope(double ql, double qc, double qr, int slope_type, double theta, double nu) {
    return ramses::SlopeLimiter::compute_slope(ql, qc, qr, slope_type, theta, nu);
}

}  // extern "C"
