// rg_api.cu -- the extern "C" boundary of librgpu.so (declared in include/rgpu.h).
//
// Mirrors the HydroSolver entry points that Simulation::amr_step calls
// (RAMSES-CPP src/core/Simulation.cpp:550,564,589,614): every call takes the
// same arguments as its HydroSolver counterpart plus the context, returns an
// int status and never throws across the boundary.
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "rg_face.cuh"
#include "rg_internal.cuh"

namespace rg {

int set_error(rg_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int check_cuda(rg_ctx* c, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return RG_OK;
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    // errors that poison the context (faults) make every later call fail fast
    if (e == cudaErrorIllegalAddress || e == cudaErrorLaunchFailure || e == cudaErrorIllegalInstruction ||
        e == cudaErrorMisalignedAddress || e == cudaErrorHardwareStackError || e == cudaErrorAssert)
        c->broken = true;
    if (e == cudaErrorMemoryAllocation) return set_error(c, RG_ERR_NOMEM, m);
    return set_error(c, RG_ERR_CUDA, m);
}

static const char* dev_err_name(int e) {
    switch (e) {
        case DE_TOPO_CYCLE: return "cyclic linked list or father chain";
        case DE_LIST: return "level linked list inconsistent with next[]";
        case DE_SAME_OUTSIDE:
            return "same-level branch names a cell outside the level (the reference would read stale traces)";
        case DE_NBOR_DEPTH: return "neighbour lookup deeper than 64 father levels";
        case DE_EVENT_OVERFLOW: return "event list overflow";
        case DE_BAD_INDEX: return "neighbour index beyond ncell";
        default: return "unknown device error";
    }
}

int check_device_status(rg_ctx* c) {
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                               c->stream),
                            "status copy"))
        return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "stream sync")) return rc;
    if (c->h_status->err != DE_NONE) {
        int e = c->h_status->err, info = c->h_status->info;
        cudaMemsetAsync(c->d_status, 0, 2 * sizeof(int), c->stream);
        cudaStreamSynchronize(c->stream);
        int code = (e == DE_SAME_OUTSIDE) ? RG_ERR_UNSUPPORTED : RG_ERR_TOPOLOGY;
        return set_error(c, code, std::string("device check: ") + dev_err_name(e) + " (index " + std::to_string(info) + ")");
    }
    return RG_OK;
}

}  // namespace rg

using namespace rg;

namespace {

template <typename T>
int grow(rg_ctx* c, T** p, size_t* cap, size_t n, const char* what) {
    if (*cap >= n && *p) return RG_OK;
    dev_free(c, *p);
    *p = nullptr;
    *cap = 0;
    if (dev_alloc(c, (void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
        return set_error(c, RG_ERR_NOMEM, std::string("device allocation failed: ") + what);
    }
    *cap = n;
    return RG_OK;
}

int validate_params(rg_ctx* c, const rg_params* p) {
    if (!p) return set_error(c, RG_ERR_ARG, "params is NULL");
    if (p->ndim != 1 && p->ndim != 3) return set_error(c, RG_ERR_UNSUPPORTED, "ndim must be 1 or 3");
    if (p->nvar != p->ndim + 2)
        return set_error(c, RG_ERR_UNSUPPORTED, "nvar must be ndim+2 (passive scalars and non-thermal energies are not implemented on the GPU path)");
    if (p->slope_type < 0 || p->slope_type > 8) return set_error(c, RG_ERR_ARG, "slope_type out of 0..8");
    if (p->riemann < 0 || p->riemann > 4) return set_error(c, RG_ERR_ARG, "riemann out of range");
    if (!(p->gamma > 1.0)) return set_error(c, RG_ERR_ARG, "gamma must be > 1");
    if (p->flags != 0) return set_error(c, RG_ERR_ARG, "flags must be 0");
    return RG_OK;
}

#define CTX_GUARD(c)                                                              \
    do {                                                                          \
        if (!(c)) return RG_ERR_ARG;                                              \
        if ((c)->broken) return set_error((c), RG_ERR_CUDA, (c)->err.empty() ? "context unusable after a device fault" : (c)->err); \
        cudaSetDevice((c)->device);                                               \
    } while (0)

void invalidate_plans(rg_ctx* c) {
    for (auto& p : c->plans) free_plan(c, p);
}

// dt of every box of an ensemble level (synchronises the stream)
int box_dts(rg_ctx* c, const Plan& P, double* out) {
    std::vector<BoxStep> h((size_t)P.nbox);
    if (int rc = check_cuda(c, cudaMemcpyAsync(h.data(), P.boxes, h.size() * sizeof(BoxStep), cudaMemcpyDeviceToHost,
                                               c->stream),
                            "box dt copy"))
        return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "box dt sync")) return rc;
    for (size_t b = 0; b < h.size(); ++b) out[b] = h[b].dt;
    return RG_OK;
}

int get_plan(rg_ctx* c, int ilevel, Plan** out) {
    if (!c->have_topology) return set_error(c, RG_ERR_STATE, "rg_sync_topology has not been called");
    if (int rc = refresh_tree(c)) return rc;
    if (ilevel < 0 || ilevel > c->nlevelmax) return set_error(c, RG_ERR_ARG, "ilevel outside 0..nlevelmax");
    if ((int)c->plans.size() < c->nlevelmax + 1) c->plans.resize(c->nlevelmax + 1);
    Plan& p = c->plans[ilevel];
    if (!p.valid) {
        if (int rc = build_plan(c, ilevel, p)) {
            free_plan(c, p);
            return rc;
        }
        if (int rc = build_lattice(c, p)) {
            free_plan(c, p);
            return rc;
        }
        if ((int)c->tuned.size() > ilevel) {
            const TunedShape& t = c->tuned[ilevel];
            if (t.variant >= 0 && p.ncells <= 8LL * t.ncells && 8LL * p.ncells >= t.ncells) {
                p.face_variant = t.variant;
                p.face_batch = t.batch;
                p.face_ms = t.ms;
            }
        }
    }
    *out = &p;
    return RG_OK;
}

// The flux scratch is shared by all levels and baked into captured graphs:
// growing it invalidates every graph.
int ensure_flux(rg_ctx* c, const Plan& P) {
    size_t need = (size_t)(2 * c->params.ndim + 1) * (c->params.ndim + 2) * (size_t)P.ncells;
    if (c->cap_flux >= need && c->d_flux) return RG_OK;
    cudaStreamSynchronize(c->stream);
    for (auto& p : c->plans)
        if (p.graph) {
            cudaGraphExecDestroy(p.graph);
            p.graph = nullptr;
        }
    return grow(c, &c->d_flux, &c->cap_flux, need, "flux scratch");
}

// rg_level_run's clock: start values, then after each substep t += dt, one
// more step, and the WHILE node's condition for the next iteration
__global__ void k_run_init(DevStatus* st, double t, long long steps) {
    st->run_t = t;
    st->run_steps = steps;
}

__global__ void k_run_limit(DevStatus* st, long long limit) { st->run_limit = limit; }

__global__ void k_run_advance(DevStatus* st, cudaGraphConditionalHandle h, double t_end) {
    st->run_t = st->run_t + st->dt;
    st->run_steps += 1;
    cudaGraphSetConditional(h, (st->run_t < t_end && st->run_steps < st->run_limit) ? 1u : 0u);
}

// substeps per launch of the run kernel or graph: bounds how long one launch
// runs (tens of milliseconds to seconds) whatever max_steps the caller asks
constexpr long long kRunChunk = 65536;

void record_updates(rg_ctx* c, int ilevel, const Plan& P) {
    if ((int)c->cell_updates.size() < c->nlevelmax + 1) c->cell_updates.resize(c->nlevelmax + 1, 0);
    c->cell_updates[ilevel] = P.nactive;
}

}  // namespace

namespace rg {
int create_pool(rg_ctx* c) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = c->device;
    if (int rc = check_cuda(c, cudaMemPoolCreate(&c->pool, &props), "device memory pool")) return rc;
    unsigned long long keep = ~0ULL;  // freed memory stays in the pool for the next plan
    return check_cuda(c, cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool");
}

cudaError_t dev_alloc(rg_ctx* c, void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, c->pool, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
    }
    return e;
}

void dev_free(rg_ctx* c, void* p) {
    if (p) cudaFreeAsync(p, c->stream);
}

void remember_shape(rg_ctx* c, const Plan& P) {
    if (P.ilevel < 0) return;
    if ((int)c->tuned.size() <= P.ilevel) c->tuned.resize((size_t)P.ilevel + 1);
    c->tuned[(size_t)P.ilevel] = TunedShape{P.face_variant, P.face_batch, P.ncells, P.face_ms};
}

int refresh_tree(rg_ctx* c) {
    if (!c->tree_dirty) return RG_OK;
    c->tree_dirty = false;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "tree refresh")) return rc;
    // the plans and oct lists of the levels the changes cannot reach stay
    // (make_grid_fine and remove_grid_fine mark the levels they reach)
    auto dirty = [](uint64_t m, size_t L) { return L > 63 || ((m >> L) & 1ull); };
    for (size_t L = 0; L < c->plans.size(); ++L)
        if (dirty(c->plans_dirty, L)) free_plan(c, c->plans[L]);
    const long long old = c->topo_version;
    c->topo_version++;
    for (size_t L = 0; L < c->lvl_ver.size(); ++L)
        if (c->lvl_ver[L] == old && !dirty(c->lists_dirty, L)) c->lvl_ver[L] = c->topo_version;
    c->plans_dirty = c->lists_dirty = 0;
    // list ranks (pointer jumping over every oct) only when a list must be
    // walked again: make_grid_fine and remove_grid_fine keep the cached lists
    // of the levels they change in order themselves
    c->ranked = false;
    if (int rc = compute_cell_levels(c)) return rc;
    return check_device_status(c);
}

void drop_amr_graphs(rg_ctx* c) {
    for (auto& kv : c->amr_graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->amr_graphs.clear();
}

Plan* existing_plan(rg_ctx* c, int ilevel) {
    if (!c->have_topology || ilevel < 0 || ilevel >= (int)c->plans.size()) return nullptr;
    Plan& p = c->plans[ilevel];
    return p.valid ? &p : nullptr;
}
}  // namespace rg

extern "C" {

const char* rg_version(void) { return "rgpu 1 (sm_100a, FP64 Godunov level step)"; }

int rg_riemann_from_string(const char* name) {
    // HydroSolver.cpp:456-461: exact, case-sensitive comparisons; LLF otherwise.
    if (!name) return RG_RIEMANN_LLF;
    if (!strcmp(name, "hllc")) return RG_RIEMANN_HLLC;
    if (!strcmp(name, "hll")) return RG_RIEMANN_HLL;
    if (!strcmp(name, "exact")) return RG_RIEMANN_EXACT;
    if (!strcmp(name, "acoustic")) return RG_RIEMANN_ACOUSTIC;
    return RG_RIEMANN_LLF;
}

rg_ctx* rg_create(const rg_params* params, int device) {
    rg_ctx* c = new (std::nothrow) rg_ctx();
    if (!c) return nullptr;
    if (validate_params(c, params)) {
        c->broken = true;
        return c;
    }
    c->params = *params;
    if (c->params.boxlen <= 0) c->params.boxlen = 1.0;
    if (device < 0) {
        if (cudaGetDevice(&device) != cudaSuccess) device = 0;
    }
    c->device = device;
    if (check_cuda(c, cudaSetDevice(device), "cudaSetDevice") ||
        check_cuda(c, cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device), "SM count") ||
        check_cuda(c, cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking), "stream") ||
        create_pool(c)) {
        c->broken = true;
        return c;
    }
    c->stream = c->own_stream;
    if (check_cuda(c, dev_alloc(c, &c->d_status, sizeof(DevStatus)), "status") ||
        check_cuda(c, cudaMallocHost(&c->h_status, sizeof(DevStatus)), "pinned status") ||
        check_cuda(c, cudaMemsetAsync(c->d_status, 0, sizeof(DevStatus), c->stream), "status init") ||
        check_cuda(c, cudaStreamSynchronize(c->stream), "status init")) {
        c->broken = true;
        return c;
    }
    for (auto& e : c->ev) cudaEventCreate(&e);
    const char* t = getenv("RG_TIMING");
    c->timing = t && t[0] == '1';
    const char* g = getenv("RG_AMR_GRAPHS");
    c->amr_graphs_on = !(g && g[0] == '0');
    return c;
}

void rg_destroy(rg_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    invalidate_plans(c);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& set : c->acc_ev)
        for (auto& e : set) cudaEventDestroy(e);
    int* ip[] = {c->d_son, c->d_father, c->d_nbor, c->d_next, c->d_bound, c->d_jump, c->d_dist, c->d_jump2,
                 c->d_dist2, c->d_cell_level, c->d_cpos, c->d_tmap, c->d_pmark, c->d_scan};
    for (int* p : ip) dev_free(c, p);
    dev_free(c, c->d_uold);
    dev_free(c, c->d_unew);
    dev_free(c, c->d_prim);
    dev_free(c, c->d_flux);
    dev_free(c, c->d_mlp);
    dev_free(c, c->d_stage);
    dev_free(c, c->d_status);
    int* tp[] = {c->d_prev, c->d_flag1, c->d_flag2, c->d_cpu_map, c->d_fq, c->d_tscr};
    for (int* p : tp) dev_free(c, p);
    dev_free(c, c->d_xg);
    for (int* p : c->lvl_octs) dev_free(c, p);
    drop_amr_graphs(c);
    dev_free(c, c->d_clock);
    if (c->h_clock) cudaFreeHost(c->h_clock);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->pool) cudaMemPoolDestroy(c->pool);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

const char* rg_last_error(const rg_ctx* c) {
    if (!c) return "null context";
    return c->err.c_str();
}

int rg_set_params(rg_ctx* c, const rg_params* params) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (int rc = validate_params(c, params)) return rc;
    if (params->ndim != c->params.ndim && c->have_topology)
        return set_error(c, RG_ERR_ARG, "ndim cannot change after rg_sync_topology");
    c->params = *params;
    if (c->params.boxlen <= 0) c->params.boxlen = 1.0;
    // graphs bake the solver choice and constants in: drop them, keep the plans
    // (and forget tuned shapes: another solver may prefer another one)
    c->tuned.clear();
    for (auto& p : c->plans)
        if (p.graph) {
            cudaGraphExecDestroy(p.graph);
            p.graph = nullptr;
        }
    drop_amr_graphs(c);
    return RG_OK;
}

int rg_sync_topology(rg_ctx* c, const rg_grid_view* g) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    c->tree_resident = false;  // the host's tree is the one in use from now on
    c->tree_dirty = false;
    if (!g || !g->son || !g->father || !g->nbor || !g->next || !g->headl) return set_error(c, RG_ERR_ARG, "null grid array");
    if (g->ngridmax < 1 || g->ncoarse < 1 || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->ncpu < 1 || g->nlevelmax < 1)
        return set_error(c, RG_ERR_ARG, "bad grid sizes");
    int ttd = 1 << c->params.ndim;
    if ((long long)g->ncell != (long long)g->ncoarse + (long long)ttd * g->ngridmax)
        return set_error(c, RG_ERR_ARG, "ncell != ncoarse + 2^ndim * ngridmax");
    if ((long long)g->nx * g->ny * g->nz != g->ncoarse) return set_error(c, RG_ERR_ARG, "ncoarse != nx*ny*nz");
    if (g->nvar != c->params.nvar) return set_error(c, RG_ERR_ARG, "grid nvar differs from params.nvar");
    if (g->nboundary != 0)
        return set_error(c, RG_ERR_UNSUPPORTED, "nboundary != 0 (boundary patches are not read by the reference either)");
    if (g->ncpu != 1) return set_error(c, RG_ERR_UNSUPPORTED, "ncpu must be 1 (the hydro path has no halo exchange)");
    cudaStreamSynchronize(c->stream);
    invalidate_plans(c);
    c->plans_dirty = c->lists_dirty = ~0ull;
    bool resized = g->ncell != c->ncell;
    c->ncoarse = g->ncoarse;
    c->ngridmax = g->ngridmax;
    c->ncell = g->ncell;
    c->nvar = g->nvar;
    c->nx = g->nx;
    c->ny = g->ny;
    c->nz = g->nz;
    c->ncpu = g->ncpu;
    c->nboundary = g->nboundary;
    c->nlevelmax = g->nlevelmax;
    c->nbound_type = (g->bound_type && g->nbound_type > 0) ? g->nbound_type : 0;
    size_t ncell1 = (size_t)c->ncell + 1, ngm = (size_t)c->ngridmax;
    size_t cap;
    cap = c->cap_cell;
    if (int rc = grow(c, &c->d_son, &cap, ncell1, "son")) return rc;
    cap = c->cap_cell;
    if (int rc = grow(c, &c->d_cell_level, &cap, ncell1, "cell_level")) return rc;
    cap = c->cap_cell;
    if (int rc = grow(c, &c->d_cpos, &cap, ncell1, "cpos")) return rc;
    cap = c->cap_cell;
    if (int rc = grow(c, &c->d_tmap, &cap, ncell1, "tmap")) return rc;
    cap = c->cap_cell;
    if (int rc = grow(c, &c->d_pmark, &cap, ncell1, "pmark")) return rc;
    c->cap_cell = std::max(c->cap_cell, ncell1);
    cap = c->cap_grid;
    if (int rc = grow(c, &c->d_father, &cap, ngm, "father")) return rc;
    cap = c->cap_grid;
    if (int rc = grow(c, &c->d_next, &cap, ngm, "next")) return rc;
    cap = c->cap_grid;
    if (int rc = grow(c, &c->d_jump, &cap, ngm, "jump")) return rc;
    cap = c->cap_grid;
    if (int rc = grow(c, &c->d_dist, &cap, ngm, "dist")) return rc;
    cap = c->cap_grid;
    if (int rc = grow(c, &c->d_jump2, &cap, ngm, "jump2")) return rc;
    cap = c->cap_grid;
    if (int rc = grow(c, &c->d_dist2, &cap, ngm, "dist2")) return rc;
    cap = c->cap_grid * 6;
    if (int rc = grow(c, &c->d_nbor, &cap, 6 * ngm, "nbor")) return rc;
    c->cap_grid = std::max(c->cap_grid, ngm);
    dev_free(c, c->d_bound);
    c->d_bound = nullptr;
    if (c->nbound_type) {
        if (check_cuda(c, dev_alloc(c, &c->d_bound, sizeof(int) * c->nbound_type), "bound_type")) return RG_ERR_NOMEM;
        cudaMemcpyAsync(c->d_bound, g->bound_type, sizeof(int) * c->nbound_type, cudaMemcpyHostToDevice, c->stream);
    }
    size_t nheadl = (size_t)(c->ncpu + c->nboundary) * (c->nlevelmax + 1);
    c->h_headl.assign(g->headl, g->headl + nheadl);
    cudaStream_t s = c->stream;
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->d_son, g->son, sizeof(int) * c->ncell, cudaMemcpyHostToDevice, s), "son upload")) return rc;
    cudaMemsetAsync(c->d_son + c->ncell, 0, sizeof(int), s);
    cudaMemcpyAsync(c->d_father, g->father, sizeof(int) * ngm, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(c->d_nbor, g->nbor, sizeof(int) * 6 * ngm, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(c->d_next, g->next, sizeof(int) * ngm, cudaMemcpyHostToDevice, s);
    if (int rc = check_cuda(c, cudaStreamSynchronize(s), "topology upload")) return rc;
    if (resized) {
        size_t ns = (size_t)c->nvar * c->ncell;
        cap = c->cap_state;
        if (int rc = grow(c, &c->d_uold, &cap, ns, "uold")) return rc;
        cap = c->cap_state;
        if (int rc = grow(c, &c->d_unew, &cap, ns, "unew")) return rc;
        cap = c->cap_state;
        if (int rc = grow(c, &c->d_prim, &cap, ns, "prim")) return rc;
        c->cap_state = std::max(c->cap_state, ns);
        c->have_state = false;
    }
    c->have_topology = true;
    c->topo_version++;
    if (int rc = rank_lists(c)) return rc;
    if (int rc = compute_cell_levels(c)) return rc;
    return check_device_status(c);
}

int rg_upload_state(rg_ctx* c, const double* uold, const double* unew) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (!c->have_topology) return set_error(c, RG_ERR_STATE, "rg_sync_topology has not been called");
    size_t bytes = sizeof(double) * (size_t)c->nvar * c->ncell;
    if (uold && check_cuda(c, cudaMemcpyAsync(c->d_uold, uold, bytes, cudaMemcpyHostToDevice, c->stream), "uold upload"))
        return RG_ERR_CUDA;
    if (unew && check_cuda(c, cudaMemcpyAsync(c->d_unew, unew, bytes, cudaMemcpyHostToDevice, c->stream), "unew upload"))
        return RG_ERR_CUDA;
    if (uold || unew) c->have_state = true;
    return RG_OK;
}

int rg_download_state(rg_ctx* c, double* uold, double* unew) {
    CTX_GUARD(c);
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state on the device");
    size_t bytes = sizeof(double) * (size_t)c->nvar * c->ncell;
    if (uold && check_cuda(c, cudaMemcpyAsync(uold, c->d_uold, bytes, cudaMemcpyDeviceToHost, c->stream), "uold download"))
        return RG_ERR_CUDA;
    if (unew && check_cuda(c, cudaMemcpyAsync(unew, c->d_unew, bytes, cudaMemcpyDeviceToHost, c->stream), "unew download"))
        return RG_ERR_CUDA;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "download sync");
}

int rg_device_state(rg_ctx* c, double** uold_dev, double** unew_dev) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (!c->have_topology) return set_error(c, RG_ERR_STATE, "rg_sync_topology has not been called");
    if (uold_dev) *uold_dev = c->d_uold;
    if (unew_dev) *unew_dev = c->d_unew;
    c->have_state = true;
    return RG_OK;
}

int rg_set_unew(rg_ctx* c, int ilevel) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    return launch_set_unew(c, *P);
}

int rg_set_uold(rg_ctx* c, int ilevel) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    return launch_set_uold(c, *P);
}

static int check_learned(rg_ctx* c) {
    if (c->params.riemann == RG_RIEMANN_EXACT && c->params.exact_guess == RG_GUESS_LEARNED && !c->mlp_valid)
        return set_error(c, RG_ERR_STATE, "exact_guess is RG_GUESS_LEARNED but no network was trained or set");
    return RG_OK;
}

int rg_godunov_level(rg_ctx* c, int ilevel, double dt, double dx) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state uploaded");
    if (int rc = check_learned(c)) return rc;
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->nbox > 0) return set_error(c, RG_ERR_STATE, "ensemble level: every box has its own dt, use rg_level_substep");
    record_updates(c, ilevel, *P);
    // no son == 0 cell (a fully refined level): godunov_fine computes nothing
    // (HydroSolver.cpp:119), so neither is anything launched or moved
    if (P->ncells == 0 || P->nactive == 0) return RG_OK;
    if (int rc = ensure_flux(c, *P)) return rc;
    if (int rc = launch_set_dt_host(c, dt, dx)) return rc;
    if (int rc = launch_godunov(c, *P)) return rc;
    // after the first real call the primitives of this level are in place:
    // time the face-kernel shapes on them (writes only the flux scratch)
    if (P->face_variant < 0 && ++P->substeps_run >= 1) return autotune_face(c, *P, step_consts(c));
    return RG_OK;
}

int rg_godunov_level_host(rg_ctx* c, int ilevel, double dt, double dx, const double* uold, double* unew) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (!uold || !unew) return set_error(c, RG_ERR_ARG, "uold and unew must be host arrays of nvar*ncell doubles");
    if (int rc = check_learned(c)) return rc;
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->nbox > 0) return set_error(c, RG_ERR_STATE, "ensemble level: every box has its own dt, use rg_level_substep");
    record_updates(c, ilevel, *P);
    // no son == 0 cell (a fully refined level): godunov_fine computes nothing
    // (HydroSolver.cpp:119), so neither is anything launched or moved
    if (P->ncells == 0 || P->nactive == 0) return RG_OK;
    if (int rc = ensure_flux(c, *P)) return rc;
    if (int rc = upload_level_host(c, *P, uold, unew)) return rc;
    if (int rc = launch_set_dt_host(c, dt, dx)) return rc;
    if (int rc = launch_godunov(c, *P)) return rc;
    if (P->face_variant < 0 && ++P->substeps_run >= 1)
        if (int rc = autotune_face(c, *P, step_consts(c))) return rc;
    if (int rc = download_level_host(c, *P, unew)) return rc;
    return check_device_status(c);
}

int rg_courant_step(rg_ctx* c, int ilevel, double dx, double courant_factor, int pressure_cap, double* dt_out) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (!dt_out) return set_error(c, RG_ERR_ARG, "dt_out is NULL");
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state uploaded");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->nbox > 0) return set_error(c, RG_ERR_STATE, "ensemble level: read the per-box steps with rg_level_box_dt");
    if (int rc = launch_courant(c, *P, dx, pressure_cap, courant_factor)) return rc;
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                               c->stream),
                            "dt copy"))
        return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "courant sync")) return rc;
    unsigned long long b = c->h_status->dtmin_bits;
    double dt;
    memcpy(&dt, &b, sizeof(dt));
    *dt_out = dt;
    return RG_OK;
}

}  // extern "C"

namespace rg {
int courant_step_device(rg_ctx* c, int ilevel, double dx, double courant_factor, int pressure_cap, bool set_unew,
                        bool armed, const ClockStep* clock, bool with_prim) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state uploaded");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->nbox > 0) return set_error(c, RG_ERR_STATE, "ensemble level: read the per-box steps with rg_level_box_dt");
    return launch_courant(c, *P, dx, pressure_cap, courant_factor, set_unew, armed, clock, with_prim);
}

int prepare_level_step(rg_ctx* c, int ilevel, bool* ready) {
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->nbox > 0) {
        *ready = false;
        return RG_OK;
    }
    if (P->ncells == 0 || P->nactive == 0) return RG_OK;
    if (int rc = ensure_flux(c, *P)) return rc;
    if (P->face_variant < 0) {
        // a level the tuner would time waits for its first eager substep
        if (P->ncells >= (1 << 17) && !c->no_autotune) {
            *ready = false;
            return RG_OK;
        }
        if (int rc = autotune_face(c, *P, step_consts(c))) return rc;
    }
    return RG_OK;
}

int godunov_level_device_dt(rg_ctx* c, int ilevel, const double* dt_dev, double dx, bool set_uold, bool prim_ready) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state uploaded");
    if (int rc = check_learned(c)) return rc;
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->nbox > 0) return set_error(c, RG_ERR_STATE, "ensemble level: every box has its own dt, use rg_level_substep");
    record_updates(c, ilevel, *P);
    // no son == 0 cell (a fully refined level): godunov_fine computes nothing
    // (HydroSolver.cpp:119), so neither is anything launched or moved
    if (P->ncells == 0 || P->nactive == 0) return RG_OK;
    if (int rc = ensure_flux(c, *P)) return rc;
    if (int rc = launch_godunov(c, *P, set_uold, dt_dev, dx, prim_ready)) return rc;  // the primitive pass sets dt
    if (P->face_variant < 0 && ++P->substeps_run >= 1) return autotune_face(c, *P, step_consts(c));
    return RG_OK;
}
}  // namespace rg

extern "C" {

int rg_level_substep(rg_ctx* c, int ilevel, double dx, int pressure_cap, int use_graph, double* dt_used) {
    CTX_GUARD(c);
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state uploaded");
    if (int rc = check_learned(c)) return rc;
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    record_updates(c, ilevel, *P);
    if (int rc = ensure_flux(c, *P)) return rc;
    const bool leaf = P->nactive == P->ncells;  // no refined cell: fused substep
    const double cfl = c->params.courant_factor;
    const int cap_key = pressure_cap ? 1 : 0;
    if (leaf) {
        // the CFL word and primitives are current if the previous call was a
        // fused substep of this level with the same arguments
        const bool ready = leaf_fusable(*P) && c->next_level == ilevel && c->next_cap == cap_key &&
                           c->next_dx == dx && c->next_cfl == cfl;
        c->next_level = -1;
        if (!ready) {
            if (int rc = launch_leaf_prefix(c, *P, dx, pressure_cap, cfl)) return rc;
        } else if (c->timing) {
            cudaEventRecord(c->ev[0], c->stream);
        }
    }
    auto enqueue = [&]() -> int {
        if (leaf) return launch_leaf_core(c, *P, dx, pressure_cap, cfl);
        if (int rc = launch_courant(c, *P, dx, pressure_cap, cfl)) return rc;
        if (int rc = launch_finalize_dt(c, dx)) return rc;
        if (int rc = launch_set_unew(c, *P)) return rc;
        if (int rc = launch_godunov(c, *P)) return rc;
        return launch_set_uold(c, *P);
    };
    if (P->face_variant < 0) {
        // first substep of this plan: run it eagerly, then tune the face
        // kernel on its primitives before any graph captures the launch shape
        if (int rc = enqueue()) return rc;
        if (int rc = autotune_face(c, *P, step_consts(c))) return rc;
    } else if (use_graph) {
        // a graph bakes dx, the courant factor and the pressure cap into its launches
        if (!P->graph || P->graph_cap != cap_key || P->graph_dx != dx || P->graph_cfl != cfl) {
            if (P->graph) {
                cudaGraphExecDestroy(P->graph);
                P->graph = nullptr;
            }
            bool timing = c->timing;
            c->timing = false;
            cudaGraph_t g = nullptr;
            if (int rc = check_cuda(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture")) {
                c->timing = timing;
                return rc;
            }
            int rc_enq = enqueue();
            cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            c->timing = timing;
            if (rc_enq) {
                if (g) cudaGraphDestroy(g);
                return rc_enq;
            }
            if (int rc = check_cuda(c, e, "end capture")) return rc;
            cudaError_t ei = cudaGraphInstantiate(&P->graph, g, 0);
            cudaGraphDestroy(g);
            if (int rc = check_cuda(c, ei, "graph instantiate")) return rc;
            P->graph_cap = cap_key;
            P->graph_dx = dx;
            P->graph_cfl = cfl;
        }
        if (int rc = check_cuda(c, cudaGraphLaunch(P->graph, c->stream), "graph launch")) return rc;
    } else {
        if (int rc = enqueue()) return rc;
    }
    if (leaf && leaf_fusable(*P) && P->ncells > 0) {
        c->next_level = ilevel;
        c->next_cap = cap_key;
        c->next_dx = dx;
        c->next_cfl = cfl;
    }
    if (dt_used) {
        if (P->nbox > 0) {
            std::vector<double> dts((size_t)P->nbox);
            if (int rc = box_dts(c, *P, dts.data())) return rc;
            *dt_used = *std::min_element(dts.begin(), dts.end());
            return RG_OK;
        }
        if (int rc = check_cuda(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                                   c->stream),
                                "dt copy"))
            return rc;
        if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "substep sync")) return rc;
        *dt_used = c->h_status->dt;
    }
    return RG_OK;
}

int rg_level_substep_host(rg_ctx* c, int ilevel, double dx, int pressure_cap, double* uold, double* unew,
                          double* dt_used) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state comes from the host
    if (!uold) return set_error(c, RG_ERR_ARG, "uold must be a host array of nvar*ncell doubles");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->nactive != P->ncells) return set_error(c, RG_ERR_STATE, "host substeps need a level without refined cells");
    if (P->ncells == 0) return RG_OK;
    if (int rc = upload_level_host(c, *P, uold, nullptr)) return rc;
    c->have_state = true;
    if (int rc = rg_level_substep(c, ilevel, dx, pressure_cap, 1, nullptr)) return rc;
    if (unew)
        if (int rc = download_level_host(c, *P, unew, c->d_unew)) return rc;
    if (int rc = download_level_host(c, *P, uold, c->d_uold)) return rc;
    if (dt_used) {
        if (int rc = check_cuda(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                                   c->stream),
                                "dt copy"))
            return rc;
        if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "dt copy")) return rc;
        *dt_used = c->h_status->dt;
    }
    return RG_OK;
}

int rg_level_run(rg_ctx* c, int ilevel, double dx, int pressure_cap, double t_start, double t_end, int64_t max_steps,
                 double* t_out, int64_t* steps_out) {
    CTX_GUARD(c);
    if (!t_out || !steps_out) return set_error(c, RG_ERR_ARG, "t_out and steps_out required");
    *t_out = t_start;
    *steps_out = 0;
    if (max_steps < 1 || !(t_start < t_end)) return RG_OK;  // the host loop would not enter
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state uploaded");
    if (int rc = check_learned(c)) return rc;
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->ncells == 0 || P->nactive != P->ncells || !leaf_fusable(*P) || P->nbox > 0)
        return set_error(c, RG_ERR_UNSUPPORTED,
                         "rg_level_run needs a level without refined cells whose stencils stay inside it (one box)");
    double t = t_start;
    long long n = 0;
    if (P->face_variant < 0) {
        // the first substep of a plan runs eagerly and chooses the face shape
        double dt = 0.0;
        if (int rc = rg_level_substep(c, ilevel, dx, pressure_cap, 0, &dt)) return rc;
        t = t + dt;
        n = 1;
        if (int rc = get_plan(c, ilevel, &P)) return rc;
        if (!(t < t_end) || n >= max_steps) {
            *t_out = t;
            *steps_out = n;
            return RG_OK;
        }
    }
    record_updates(c, ilevel, *P);
    if (int rc = ensure_flux(c, *P)) return rc;
    const double cfl = c->params.courant_factor;
    const int cap_key = pressure_cap ? 1 : 0;
    const bool ready = c->next_level == ilevel && c->next_cap == cap_key && c->next_dx == dx && c->next_cfl == cfl;
    c->next_level = -1;
    if (!ready)
        if (int rc = launch_leaf_prefix(c, *P, dx, pressure_cap, cfl)) return rc;
    k_run_init<<<1, 1, 0, c->stream>>>(c->d_status, t, n);
    // launches of at most kRunChunk substeps until t_end or max_steps
    auto read_clock = [&]() -> int {
        if (int rc = check_cuda(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(DevStatus),
                                                   cudaMemcpyDeviceToHost, c->stream),
                                "run clock"))
            return rc;
        if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "run")) return rc;
        t = c->h_status->run_t;
        n = c->h_status->run_steps;
        return c->h_status->err ? check_device_status(c) : RG_OK;
    };
    if (P->ncells <= kRunBlockCells) {
        // small level: the loop in a single-block kernel
        while (t < t_end && n < max_steps) {
            const long long limit = std::min<long long>(max_steps, n + kRunChunk);
            if (int rc = launch_run_block(c, *P, dx, pressure_cap, t_end, limit)) return rc;
            if (int rc = read_clock()) return rc;
        }
        c->next_level = ilevel;
        c->next_cap = cap_key;
        c->next_dx = dx;
        c->next_cfl = cfl;
        *t_out = t;
        *steps_out = n;
        return check_device_status(c);
    }
    // one graph: a WHILE node whose body is the substep (dt finalize, face,
    // fold with the next CFL word and primitives) and the clock advance
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto fail = [&](int rc) {
        if (exec) cudaGraphExecDestroy(exec);
        if (g) cudaGraphDestroy(g);
        return rc;
    };
    if (int rc = check_cuda(c, cudaGraphCreate(&g, 0), "run graph")) return rc;
    cudaGraphConditionalHandle h;
    if (int rc = check_cuda(c, cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault), "run handle"))
        return fail(rc);
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (int rc = check_cuda(c, cudaGraphAddNode(&node, g, nullptr, 0, &np), "run loop node")) return fail(rc);
    cudaGraph_t body = np.conditional.phGraph_out[0];
    const bool timing = c->timing;
    c->timing = false;
    if (int rc = check_cuda(c, cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0,
                                                             cudaStreamCaptureModeThreadLocal),
                            "run capture")) {
        c->timing = timing;
        return fail(rc);
    }
    int rc_enq = launch_leaf_core(c, *P, dx, pressure_cap, cfl);
    k_run_advance<<<1, 1, 0, c->stream>>>(c->d_status, h, t_end);
    cudaGraph_t captured = nullptr;
    cudaError_t ec = cudaStreamEndCapture(c->stream, &captured);
    c->timing = timing;
    if (rc_enq) return fail(rc_enq);
    if (int rc = check_cuda(c, ec, "run capture end")) return fail(rc);
    if (int rc = check_cuda(c, cudaGraphInstantiate(&exec, g, 0), "run graph instantiate")) return fail(rc);
    while (t < t_end && n < max_steps) {
        k_run_limit<<<1, 1, 0, c->stream>>>(c->d_status, std::min<long long>(max_steps, n + kRunChunk));
        if (int rc = check_cuda(c, cudaGraphLaunch(exec, c->stream), "run graph launch")) return fail(rc);
        if (int rc = read_clock()) return fail(rc);
    }
    fail(RG_OK);
    c->next_level = ilevel;  // the last fold left the next substep's CFL word and primitives
    c->next_cap = cap_key;
    c->next_dx = dx;
    c->next_cfl = cfl;
    *t_out = t;
    *steps_out = n;
    return check_device_status(c);
}

int rg_set_level_boxes(rg_ctx* c, int ilevel, int nbox, const int* first_oct, const double* dx) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (nbox < 1 || !first_oct || !dx) return set_error(c, RG_ERR_ARG, "nbox >= 1, first_oct[nbox+1] and dx[nbox] required");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->level0) return set_error(c, RG_ERR_ARG, "ensemble boxes need a level above the coarse level");
    if (P->nactive != P->ncells) return set_error(c, RG_ERR_STATE, "ensemble level has refined cells");
    if (first_oct[0] != 0 || first_oct[nbox] != P->noct)
        return set_error(c, RG_ERR_ARG, "first_oct must start at 0 and end at the level's oct count " +
                                            std::to_string(P->noct));
    std::vector<int> obox((size_t)P->noct);
    std::vector<BoxStep> boxes((size_t)nbox);
    for (int b = 0; b < nbox; ++b) {
        if (first_oct[b + 1] <= first_oct[b]) return set_error(c, RG_ERR_ARG, "box " + std::to_string(b) + " is empty");
        if (!(dx[b] > 0.0) || !std::isfinite(dx[b])) return set_error(c, RG_ERR_ARG, "dx must be positive");
        for (int k = first_oct[b]; k < first_oct[b + 1]; ++k) obox[(size_t)k] = b;
        boxes[(size_t)b] = BoxStep{0ULL, 0.0, dx[b], 0.0, 0.0, 0, 0};
    }
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "boxes sync")) return rc;
    dev_free(c, P->obox);
    dev_free(c, P->boxes);
    P->obox = nullptr;
    P->boxes = nullptr;
    P->nbox = 0;
    if (int rc = check_cuda(c, dev_alloc(c, &P->obox, obox.size() * sizeof(int)), "dev_alloc(c, boxes)")) return rc;
    if (int rc = check_cuda(c, dev_alloc(c, &P->boxes, boxes.size() * sizeof(BoxStep)), "dev_alloc(c, boxes)")) return rc;
    if (int rc = check_cuda(c, cudaMemcpyAsync(P->obox, obox.data(), obox.size() * sizeof(int), cudaMemcpyHostToDevice,
                                               c->stream),
                            "boxes upload"))
        return rc;
    if (int rc = check_cuda(c, cudaMemcpyAsync(P->boxes, boxes.data(), boxes.size() * sizeof(BoxStep),
                                               cudaMemcpyHostToDevice, c->stream),
                            "boxes upload"))
        return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "boxes upload")) return rc;
    P->nbox = nbox;
    if (P->graph) {
        cudaGraphExecDestroy(P->graph);
        P->graph = nullptr;
    }
    return RG_OK;
}

int rg_set_level_lattices(rg_ctx* c, int ilevel, int nbox, const int* extent, const int* lat_id, const int* lat_p) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state or the CFL word may change
    if (nbox < 1 || !extent || !lat_id || !lat_p) return set_error(c, RG_ERR_ARG, "nbox, extent, lat_id and lat_p required");
    Plan* P = existing_plan(c, ilevel);
    if (!P || P->nbox != nbox) return set_error(c, RG_ERR_STATE, "set the level's boxes (rg_set_level_boxes) first");
    if (c->params.ndim != 3) return set_error(c, RG_ERR_UNSUPPORTED, "box lattices are a 3D form");
    if (int rc = set_box_lattices(c, *P, extent, lat_id, lat_p)) return rc;
    if (P->graph) {
        cudaGraphExecDestroy(P->graph);
        P->graph = nullptr;
    }
    // the tuned shape was timed without the brick kernel
    P->face_variant = -1;
    return RG_OK;
}

int rg_level_output(rg_ctx* c, int ilevel, double* out, int64_t cap) {
    CTX_GUARD(c);
    if (!out) return set_error(c, RG_ERR_ARG, "out is NULL");
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state on the device");
    if (c->params.nvar != c->params.ndim + 2)
        return set_error(c, RG_ERR_UNSUPPORTED, "snapshot records of extra variables are not formed on the device");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    const size_t n = (size_t)(1 << c->params.ndim) * c->params.nvar * (size_t)P->noct;
    if (P->level0) return set_error(c, RG_ERR_ARG, "the coarse level has no octs to write");
    if ((int64_t)n > cap) return set_error(c, RG_ERR_ARG, "out holds fewer than 2^ndim * nvar * noct doubles");
    if (n == 0) return RG_OK;
    if (int rc = ensure_flux(c, *P)) return rc;  // the flux scratch is large enough to stage the records
    if (c->cap_flux < n) return set_error(c, RG_ERR_STATE, "staging too small");
    if (int rc = launch_level_output(c, *P, c->d_flux)) return rc;
    if (int rc = check_cuda(c, cudaMemcpyAsync(out, c->d_flux, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                            "level output copy"))
        return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "level output sync");
}

int rg_level_box_dt(rg_ctx* c, int ilevel, double* dt_out, int nbox) {
    CTX_GUARD(c);
    Plan* P = existing_plan(c, ilevel);
    if (!P || P->nbox == 0) return set_error(c, RG_ERR_STATE, "level has no ensemble boxes");
    if (!dt_out || nbox != P->nbox) return set_error(c, RG_ERR_ARG, "dt_out must hold the level's box count");
    return box_dts(c, *P, dt_out);
}

int rg_synchronize(rg_ctx* c) {
    CTX_GUARD(c);
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "synchronize")) return rc;
    if (c->timing) {
        for (int i = 0; i < 3; ++i) cudaEventElapsedTime(&c->last_ms[i], c->ev[i], c->ev[i + 1]);
        cudaGetLastError();
    }
    return check_device_status(c);
}

int rg_set_stream(rg_ctx* c, void* stream) {
    CTX_GUARD(c);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->own_stream;
    if (s == c->stream) return RG_OK;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "stream switch")) return rc;
    for (auto& p : c->plans)
        if (p.graph) {
            cudaGraphExecDestroy(p.graph);
            p.graph = nullptr;
        }
    c->stream = s;
    return RG_OK;
}

int rg_get_stream(rg_ctx* c, void** stream) {
    CTX_GUARD(c);
    if (!stream) return set_error(c, RG_ERR_ARG, "stream is NULL");
    *stream = (void*)c->stream;
    return RG_OK;
}

int rg_level_octs(rg_ctx* c, int ilevel, int* octs_out, int cap, int* n_out) {
    CTX_GUARD(c);
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (n_out) *n_out = P->noct;
    int n = std::min(cap, P->noct);
    if (n > 0 && octs_out) {
        if (int rc = check_cuda(c, cudaMemcpyAsync(octs_out, P->octs, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream), "octs copy")) return rc;
        return check_cuda(c, cudaStreamSynchronize(c->stream), "octs sync");
    }
    return RG_OK;
}

int rg_level_plan_info(rg_ctx* c, int ilevel, rg_plan_info* out) {
    CTX_GUARD(c);
    if (!out) return set_error(c, RG_ERR_ARG, "out is NULL");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    *out = rg_plan_info{P->ncells, P->ntarg, P->nevents, P->nextra_prim, P->nlong};
    return RG_OK;
}

int rg_level_nbor_cells(rg_ctx* c, int ilevel, int* out, int cap) {
    CTX_GUARD(c);
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    int ns = 2 * c->params.ndim, ttd = 1 << c->params.ndim;
    if ((long long)cap < (long long)P->ncells * 6) return set_error(c, RG_ERR_ARG, "output too small (need ncells*6)");
    std::vector<int> h((size_t)ns * P->ncells);
    if (P->ncells) {
        if (int rc = check_cuda(c, cudaMemcpyAsync(h.data(), P->icn, sizeof(int) * h.size(), cudaMemcpyDeviceToHost, c->stream), "icn copy")) return rc;
        if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "icn sync")) return rc;
    }
    for (int p = 0; p < P->ncells; ++p) {
        int cpu = P->level0 ? p : (p % P->noct) * ttd + p / P->noct;
        for (int j = 0; j < 6; ++j) out[(size_t)cpu * 6 + j] = (j < ns) ? h[(size_t)j * P->ncells + p] : 0;
    }
    return RG_OK;
}

int64_t rg_level_cell_updates(rg_ctx* c, int ilevel) {
    if (!c || ilevel < 0 || ilevel >= (int)c->cell_updates.size()) return 0;
    return c->cell_updates[ilevel];
}

int rg_exact_stats(rg_ctx* c, int64_t* iters, int64_t* calls, int reset) {
    CTX_GUARD(c);
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                               c->stream),
                            "stats copy"))
        return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "stats sync")) return rc;
    if (iters) *iters = (int64_t)c->h_status->exact_iters;
    if (calls) *calls = (int64_t)c->h_status->exact_calls;
    if (reset) {
        // exact_iters and exact_calls are adjacent in DevStatus
        cudaMemsetAsync(&c->d_status->exact_iters, 0, 2 * sizeof(unsigned long long), c->stream);
        return check_cuda(c, cudaStreamSynchronize(c->stream), "stats reset");
    }
    return RG_OK;
}

int rg_set_autotune(rg_ctx* c, int on) {
    CTX_GUARD(c);
    c->no_autotune = (on == 0);
    drop_amr_graphs(c);
    return RG_OK;
}

int rg_face_config(rg_ctx* c, int ilevel, int* variant, int* batch, float* ms) {
    CTX_GUARD(c);
    Plan* P = existing_plan(c, ilevel);
    if (!P) return set_error(c, RG_ERR_STATE, "no plan for this level yet");
    if (variant) *variant = P->face_variant;
    if (batch) *batch = P->face_batch;
    if (ms) *ms = P->face_ms;
    return RG_OK;
}

int rg_set_face_config(rg_ctx* c, int ilevel, int variant, int batch) {
    CTX_GUARD(c);
    if (variant < 0 || variant >= kNumFaceVariants || batch < 1)
        return set_error(c, RG_ERR_ARG, "variant must be in [0, 11), batch >= 1");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    P->face_variant = variant;
    P->face_batch = batch;
    remember_shape(c, *P);
    if (P->graph) {
        cudaGraphExecDestroy(P->graph);
        P->graph = nullptr;
    }
    drop_amr_graphs(c);
    return RG_OK;
}

int rg_exact_batch(rg_ctx* c, int n, const double* ql_dev, const double* qr_dev, const double* gamma_dev,
                   double* flux_dev, double* pstar_dev, int* iters_dev, int guess, int niter, double tol) {
    CTX_GUARD(c);
    if (n < 0 || !ql_dev || !qr_dev) return set_error(c, RG_ERR_ARG, "bad batch arguments");
    if (niter < 1 || !(tol > 0)) return set_error(c, RG_ERR_ARG, "niter >= 1 and tol > 0 required");
    const float* mlp = nullptr;
    if (guess == RG_GUESS_LEARNED) {
        if (!c->mlp_valid) return set_error(c, RG_ERR_STATE, "no network trained or set");
        mlp = c->d_mlp;
    }
    if (n == 0) return RG_OK;
    return launch_exact_batch(c, n, ql_dev, qr_dev, gamma_dev, flux_dev, pstar_dev, iters_dev, mlp, niter, tol);
}

int rg_stress_states(rg_ctx* c, int n, uint64_t seed, double* ql_dev, double* qr_dev, double* gamma_dev) {
    CTX_GUARD(c);
    if (n < 1 || !ql_dev || !qr_dev) return set_error(c, RG_ERR_ARG, "bad stress arguments");
    return launch_stress_states(c, n, (unsigned long long)seed, ql_dev, qr_dev, gamma_dev);
}

int rg_mlp_nparam(void) { return MLP_NPARAM; }

int rg_mlp_train(rg_ctx* c, int nsamples, int epochs, int batch, float lr, uint64_t seed, float* loss_out) {
    CTX_GUARD(c);
    drop_amr_graphs(c);  // captured steps name the network (or its absence)
    return mlp_train(c, nsamples, epochs, batch, lr, (unsigned long long)seed, loss_out);
}

int rg_mlp_get(rg_ctx* c, float* params) {
    CTX_GUARD(c);
    if (!params) return set_error(c, RG_ERR_ARG, "params is NULL");
    if (!c->mlp_valid) return set_error(c, RG_ERR_STATE, "no network trained or set");
    if (int rc = check_cuda(c, cudaMemcpyAsync(params, c->d_mlp, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost,
                                               c->stream),
                            "mlp copy"))
        return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "mlp sync");
}

int rg_mlp_set(rg_ctx* c, const float* params) {
    CTX_GUARD(c);
    if (!params) return set_error(c, RG_ERR_ARG, "params is NULL");
    drop_amr_graphs(c);  // captured steps name the network (or its absence)
    if (int rc = mlp_ensure(c)) return rc;
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->d_mlp, params, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice,
                                               c->stream),
                            "mlp copy"))
        return rc;
    c->mlp_valid = true;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "mlp sync");
}

int rg_mlp_grad(rg_ctx* c, int n, const float* x, const float* t, float* grad, float* loss) {
    CTX_GUARD(c);
    if (n < 1 || !x || !t || !grad || !loss) return set_error(c, RG_ERR_ARG, "bad gradient-check arguments");
    if (!c->mlp_valid) return set_error(c, RG_ERR_STATE, "no network trained or set");
    return mlp_grad(c, n, x, t, grad, loss);
}

int rg_set_timing(rg_ctx* c, int on) {
    CTX_GUARD(c);
    c->timing = on != 0;
    c->timing_acc = on == 2;
    c->acc_n = 0;
    return RG_OK;
}

int rg_kernel_ms_totals(rg_ctx* c, double* ms, int64_t* cells, int64_t* steps, int reset) {
    CTX_GUARD(c);
    if (!ms || !cells || !steps) return set_error(c, RG_ERR_ARG, "ms[3], cells and steps must be non-null");
    if (!c->timing_acc) return set_error(c, RG_ERR_STATE, "accumulating timing is off (rg_set_timing(ctx, 2))");
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "kernel timing")) return rc;
    ms[0] = ms[1] = ms[2] = 0.0;
    long long n = 0;
    for (size_t i = 0; i < c->acc_n; ++i) {
        for (int k = 0; k < 3; ++k) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, c->acc_ev[i][k], c->acc_ev[i][k + 1]) == cudaSuccess) ms[k] += t;
        }
        n += c->acc_cells[i];
    }
    cudaGetLastError();
    *cells = n;
    *steps = (int64_t)c->acc_n;
    if (reset) c->acc_n = 0;
    return RG_OK;
}

int rg_last_kernel_ms(rg_ctx* c, float* out, int n) {
    CTX_GUARD(c);
    for (int i = 0; i < n && i < 3; ++i) out[i] = c->last_ms[i];
    return c->timing ? RG_OK : set_error(c, RG_ERR_STATE, "timing disabled (set RG_TIMING=1)");
}

int rg_upload_level(rg_ctx* c, int ilevel, const double* uold) {
    CTX_GUARD(c);
    c->next_level = -1;  // the state changes
    if (!uold) return set_error(c, RG_ERR_ARG, "uold must be a host array of nvar*ncell doubles");
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state uploaded (rg_upload_state first)");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (P->ncells == 0) return RG_OK;
    return upload_level_host(c, *P, uold, nullptr);
}

int rg_download_level(rg_ctx* c, int ilevel, double* uold, double* unew) {
    CTX_GUARD(c);
    if (!c->have_state) return set_error(c, RG_ERR_STATE, "no state uploaded (rg_upload_state first)");
    Plan* P;
    if (int rc = get_plan(c, ilevel, &P)) return rc;
    if (int rc = download_level_cells(c, *P, uold, unew)) return rc;
    return check_device_status(c);
}

int rg_pool_usage(rg_ctx* c, uint64_t* reserved, uint64_t* used) {
    CTX_GUARD(c);
    if (!reserved || !used) return set_error(c, RG_ERR_ARG, "reserved and used must be non-null");
    unsigned long long r = 0, u = 0;  // the attributes are 64-bit values
    if (int rc = check_cuda(c, cudaMemPoolGetAttribute(c->pool, cudaMemPoolAttrReservedMemCurrent, &r),
                            "cudaMemPoolGetAttribute"))
        return rc;
    if (int rc = check_cuda(c, cudaMemPoolGetAttribute(c->pool, cudaMemPoolAttrUsedMemCurrent, &u),
                            "cudaMemPoolGetAttribute"))
        return rc;
    *reserved = r;
    *used = u;
    return RG_OK;
}

/* ---- device-resident tree ---------------------------------------------- */
int rg_tree_attach(rg_ctx* c, const rg_grid_view* g, const rg_tree_arrays* t, int levelmin) {
    CTX_GUARD(c);
    if (!g || !t) return set_error(c, RG_ERR_ARG, "grid view and tree arrays required");
    if (c->params.ndim != 3 || c->params.nvar != 5)
        return set_error(c, RG_ERR_UNSUPPORTED, "device tree operations need ndim 3 and nvar 5");
    if (!t->prev || !t->taill || !t->numbl || !t->flag1 || !t->flag2 || !t->cpu_map || !t->xg || !t->uold || !t->unew)
        return set_error(c, RG_ERR_ARG, "null tree array");
    if (int rc = rg_sync_topology(c, g)) return rc;
    if (int rc = rg_upload_state(c, t->uold, t->unew)) return rc;
    const size_t ngm = (size_t)c->ngridmax, nc = (size_t)c->ncell, nh = c->h_headl.size();
    int** ip[] = {&c->d_prev, &c->d_fq, &c->d_flag1, &c->d_flag2, &c->d_cpu_map};
    const size_t isz[] = {ngm, ngm, nc, nc, nc};
    for (int i = 0; i < 5; ++i) {
        dev_free(c, *ip[i]);
        *ip[i] = nullptr;
        if (int rc = check_cuda(c, dev_alloc(c, ip[i], sizeof(int) * isz[i]), "tree arrays")) return rc;
    }
    dev_free(c, c->d_xg);
    c->d_xg = nullptr;
    if (int rc = check_cuda(c, dev_alloc(c, &c->d_xg, sizeof(double) * 3 * ngm), "tree coordinates")) return rc;
    // the free list, walked from its head, becomes the ring's initial content
    if (t->numbf < 0 || (size_t)t->numbf > ngm) return set_error(c, RG_ERR_TOPOLOGY, "numbf out of range");
    c->h_fq.assign(ngm, 0);
    int g_at = t->headf, n = 0, last = 0;
    while (g_at > 0 && n < t->numbf) {
        if ((size_t)g_at > ngm) return set_error(c, RG_ERR_TOPOLOGY, "free list entry out of range");
        c->h_fq[(size_t)n++] = g_at;
        last = g_at;
        g_at = g->next[g_at - 1];
    }
    if (n != t->numbf || g_at != 0 || last != t->tailf)
        return set_error(c, RG_ERR_TOPOLOGY, "free list (headf, next, tailf, numbf) is inconsistent");
    c->fq_head = 0;
    c->numbf = n;
    c->h_taill.assign(t->taill, t->taill + nh);
    c->h_numbl.assign(t->numbl, t->numbl + nh);
    c->levelmin = levelmin;
    cudaStream_t s = c->stream;
    cudaMemcpyAsync(c->d_prev, t->prev, sizeof(int) * ngm, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(c->d_fq, c->h_fq.data(), sizeof(int) * ngm, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(c->d_flag1, t->flag1, sizeof(int) * nc, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(c->d_flag2, t->flag2, sizeof(int) * nc, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(c->d_cpu_map, t->cpu_map, sizeof(int) * nc, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(c->d_xg, t->xg, sizeof(double) * 3 * ngm, cudaMemcpyHostToDevice, s);
    if (int rc = check_cuda(c, cudaStreamSynchronize(s), "tree upload")) return rc;
    c->tree_resident = true;
    c->tree_dirty = false;
    c->auth_dirty = true;
    return RG_OK;
}

int rg_tree_fetch(rg_ctx* c, rg_tree_arrays* t) {
    CTX_GUARD(c);
    if (!c->tree_resident) return set_error(c, RG_ERR_STATE, "no device-resident tree");
    if (!t) return set_error(c, RG_ERR_ARG, "tree arrays required");
    const size_t ngm = (size_t)c->ngridmax, nc = (size_t)c->ncell, nh = c->h_headl.size();
    const size_t ns = (size_t)c->nvar * nc;
    cudaStream_t s = c->stream;
    struct {
        void* dst;
        const void* src;
        size_t bytes;
    } cp[] = {{t->son, c->d_son, sizeof(int) * nc},        {t->father, c->d_father, sizeof(int) * ngm},
              {t->nbor, c->d_nbor, sizeof(int) * 6 * ngm}, {t->next, c->d_next, sizeof(int) * ngm},
              {t->prev, c->d_prev, sizeof(int) * ngm},     {t->flag1, c->d_flag1, sizeof(int) * nc},
              {t->flag2, c->d_flag2, sizeof(int) * nc},    {t->cpu_map, c->d_cpu_map, sizeof(int) * nc},
              {t->xg, c->d_xg, sizeof(double) * 3 * ngm},  {t->uold, c->d_uold, sizeof(double) * ns},
              {t->unew, c->d_unew, sizeof(double) * ns}};
    for (auto& e : cp)
        if (e.dst)
            if (int rc = check_cuda(c, cudaMemcpyAsync(e.dst, e.src, e.bytes, cudaMemcpyDeviceToHost, s), "tree fetch"))
                return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(s), "tree fetch")) return rc;
    if (t->headl) std::copy(c->h_headl.begin(), c->h_headl.end(), t->headl);
    if (t->taill) std::copy(c->h_taill.begin(), c->h_taill.end(), t->taill);
    if (t->numbl) std::copy(c->h_numbl.begin(), c->h_numbl.end(), t->numbl);
    (void)nh;
    const int ngmi = c->ngridmax;
    t->numbf = c->numbf;
    t->headf = c->numbf > 0 ? c->h_fq[(size_t)c->fq_head] : 0;
    t->tailf = c->numbf > 0 ? c->h_fq[(size_t)((c->fq_head + c->numbf - 1) % ngmi)] : 0;
    return RG_OK;
}

int rg_flag_fine(rg_ctx* c, int ilevel, double err_grad_d, double err_grad_p, double err_grad_u, double err_grad_b2,
                 int nexpand, int icount, int nsubcycle) {
    CTX_GUARD(c);
    return tree_flag_fine(c, ilevel, err_grad_d, err_grad_p, err_grad_u, err_grad_b2, nexpand, icount, nsubcycle);
}

int rg_make_grid_fine(rg_ctx* c, int ilevel) {
    CTX_GUARD(c);
    return tree_make_grid_fine(c, ilevel);
}

int rg_remove_grid_fine(rg_ctx* c, int ilevel) {
    CTX_GUARD(c);
    return tree_remove_grid_fine(c, ilevel);
}

int rg_restrict_fine(rg_ctx* c, int ilevel) {
    CTX_GUARD(c);
    return tree_restrict_fine(c, ilevel);
}

int rg_count_grids(rg_ctx* c, int ilevel, int* n) {
    CTX_GUARD(c);
    if (!n) return set_error(c, RG_ERR_ARG, "n is NULL");
    if (!c->tree_resident) return set_error(c, RG_ERR_STATE, "no device-resident tree");
    *n = 0;
    if (ilevel < 0 || ilevel > c->nlevelmax) return RG_OK;  // AmrGrid::numbl returns 0 out of range
    *n = c->h_numbl[(size_t)ilevel * (c->ncpu + c->nboundary)];
    return RG_OK;
}

int rg_tree_sizes(rg_ctx* c, int* ngridmax, int* ncell) {
    CTX_GUARD(c);
    if (!c->have_topology) return set_error(c, RG_ERR_STATE, "rg_sync_topology has not been called");
    if (ngridmax) *ngridmax = c->ngridmax;
    if (ncell) *ncell = c->ncell;
    return RG_OK;
}

}  // extern "C"
