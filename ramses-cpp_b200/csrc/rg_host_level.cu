// rg_host_level.cu -- level-sparse host <-> device state transfer for
// callers whose state lives in host memory between level steps.
//
// In a RAMSES-CPP run the tree maintenance (TreeUpdater) and Simulation read
// and write AmrGrid's host uold/unew between hydro calls, so a drop-in hydro
// solver must take its inputs from, and return its outputs to, host memory
// on every godunov_fine call (HydroSolver.cpp:18-573).  The step of level L
// reads uold only at the level's cells and at the cells outside the level
// that its stencils reach (the plan's extra primitive cells), reads unew only
// at its update targets (the level's cells and the coarser cells that
// receive refluxes), and writes unew only at those targets.  So instead of
// the whole state (2 x nvar x ncell doubles up, nvar x ncell down) a call
// moves exactly those cells.  From page-locked host arrays whose level cells
// form few runs of consecutive ids (a uniform level: one run per child slot)
// each run is one DMA straight between the caller's array and the device
// state.  Otherwise (pageable arrays, as AmrGrid's std::vectors are, or a
// fragmented level) the cells are gathered on the host into pinned staging,
// run by run where runs are long, moved in one copy each way and scattered on
// the device: the CUDA driver stages a pageable copy through its own buffers with
// a wait per row, so many small pageable copies would cost far more than the
// host gather.
#include <algorithm>
#include <cstring>
#include <vector>

#include "rg_internal.cuh"

namespace rg {

namespace {

__device__ __forceinline__ int plan_cell(const TreeView& T, const PlanView& P, int p) {
    if (P.level0) return p + 1;
    int icx = p / P.noct, k = p - icx * P.noct;
    return T.ncoarse + icx * T.ngridmax + P.octs[k];
}

// read ids: level cells then extra primitive cells; target ids: level cells
// then extra targets
__global__ void k_level_ids(TreeView T, PlanView P, int* read_ids, int* targ_ids) {
    const int nread = P.ncells + P.nextra_prim;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nread || t < P.ntarg; t += gridDim.x * blockDim.x) {
        const int lvl = t < P.ncells ? plan_cell(T, P, t) : 0;
        if (t < nread) read_ids[t] = t < P.ncells ? lvl : P.xprim[t - P.ncells];
        if (t < P.ntarg) targ_ids[t] = t < P.ncells ? lvl : P.textra[t - P.ncells];
    }
}

// staging layout: [nvar][nread] uold values, then [nvar][ntarg] unew values
// (ntarg = 0 when only uold is uploaded)
__global__ void k_scatter_level(const int* __restrict__ read_ids, int nread, const int* __restrict__ targ_ids,
                                int ntarg, int nvar, size_t ncell, const double* __restrict__ stage, double* uold,
                                double* unew) {
    const double* sn = stage + (size_t)nvar * nread;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nread || t < ntarg; t += gridDim.x * blockDim.x) {
        if (t < nread) {
            const size_t id = (size_t)read_ids[t] - 1;
            for (int iv = 0; iv < nvar; ++iv) uold[iv * ncell + id] = stage[(size_t)iv * nread + t];
        }
        if (t < ntarg) {
            const size_t id = (size_t)targ_ids[t] - 1;
            for (int iv = 0; iv < nvar; ++iv) unew[iv * ncell + id] = sn[(size_t)iv * ntarg + t];
        }
    }
}

// ids[0..n) of two state arrays (b may be null) into stage [2][nvar][n]
__global__ void k_gather_ids2(const int* __restrict__ ids, int n, int nvar, size_t ncell, const double* __restrict__ a,
                              const double* __restrict__ b, double* stage) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const size_t id = (size_t)ids[t] - 1;
        for (int iv = 0; iv < nvar; ++iv) {
            if (a) stage[(size_t)iv * n + t] = a[iv * ncell + id];
            if (b) stage[((size_t)nvar + iv) * n + t] = b[iv * ncell + id];
        }
    }
}

__global__ void k_gather_targets(const int* __restrict__ targ_ids, int ntarg, int nvar, size_t ncell,
                                  const double* __restrict__ unew, double* stage) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntarg; t += gridDim.x * blockDim.x) {
        const size_t id = (size_t)targ_ids[t] - 1;
        for (int iv = 0; iv < nvar; ++iv) stage[(size_t)iv * ntarg + t] = unew[iv * ncell + id];
    }
}

int blocks(rg_ctx* c, long long n) {
    long long b = (n + 255) / 256, cap = (long long)c->sm_count * 16;
    return (int)std::max(1LL, std::min(b, cap));
}

int grow_stage(rg_ctx* c, size_t doubles) {
    if (c->cap_hstage < doubles) {
        if (c->h_stage) cudaFreeHost(c->h_stage);
        c->h_stage = nullptr;
        c->cap_hstage = 0;
        if (int rc = check_cuda(c, cudaMallocHost(&c->h_stage, doubles * sizeof(double)), "pinned level staging"))
            return rc;
        c->cap_hstage = doubles;
    }
    if (c->cap_dstage < doubles) {
        dev_free(c, c->d_stage);
        c->d_stage = nullptr;
        c->cap_dstage = 0;
        if (int rc = check_cuda(c, dev_alloc(c, &c->d_stage, doubles * sizeof(double)), "device level staging"))
            return rc;
        c->cap_dstage = doubles;
    }
    return RG_OK;
}

}  // namespace

// Host and device copies of the plan's read and target cell ids (built once
// per plan; synchronises the stream).
int level_ids(rg_ctx* c, Plan& P) {
    if (P.ids_ready) return RG_OK;
    const int nread = P.ncells + P.nextra_prim;
    dev_free(c, P.read_ids);
    P.read_ids = nullptr;
    if (int rc = check_cuda(c, dev_alloc(c, &P.read_ids, sizeof(int) * ((size_t)nread + P.ntarg + 1)), "level ids"))
        return rc;
    P.targ_ids = P.read_ids + nread;
    k_level_ids<<<blocks(c, std::max(nread, P.ntarg)), 256, 0, c->stream>>>(tree_view(c), P.view(), P.read_ids,
                                                                          P.targ_ids);
    P.h_read.resize((size_t)nread);
    P.h_targ.resize((size_t)P.ntarg);
    if (nread && check_cuda(c, cudaMemcpyAsync(P.h_read.data(), P.read_ids, sizeof(int) * nread,
                                               cudaMemcpyDeviceToHost, c->stream),
                            "level ids copy"))
        return RG_ERR_CUDA;
    if (P.ntarg && check_cuda(c, cudaMemcpyAsync(P.h_targ.data(), P.targ_ids, sizeof(int) * P.ntarg,
                                                 cudaMemcpyDeviceToHost, c->stream),
                              "level ids copy"))
        return RG_ERR_CUDA;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "level ids sync")) return rc;
    auto runs = [](const std::vector<int>& ids) {
        std::vector<std::pair<int, int>> r;
        for (size_t t = 0; t < ids.size(); ++t) {
            if (!r.empty() && ids[t] == r.back().first + r.back().second) ++r.back().second;
            else r.emplace_back(ids[t], 1);
        }
        return r;
    };
    P.read_runs = runs(P.h_read);
    P.targ_runs = runs(P.h_targ);
    P.h_cells.assign(P.h_read.begin(), P.h_read.begin() + P.ncells);
    P.cell_runs = runs(P.h_cells);
    P.ids_ready = true;
    return RG_OK;
}

namespace {
// Levels whose cells form at most this many id runs are moved run by run
// (DMA straight between the caller's arrays and the device state); more
// fragmented levels are gathered into pinned staging instead.
constexpr size_t kMaxRuns = 256;

// one 2D copy per run covers the run in all nvar planes (pitch = one plane)
int copy_runs(rg_ctx* c, const std::vector<std::pair<int, int>>& runs, double* dst, const double* src,
              cudaMemcpyKind kind) {
    const size_t pitch = sizeof(double) * (size_t)c->ncell;
    for (const auto& r : runs) {
        const size_t off = (size_t)r.first - 1;
        if (int rc = check_cuda(c, cudaMemcpy2DAsync(dst + off, pitch, src + off, pitch, sizeof(double) * (size_t)r.second,
                                                     (size_t)c->nvar, kind, c->stream),
                                "level run copy"))
            return rc;
    }
    return RG_OK;
}

// true when the whole state array [nvar][ncell] at p is page-locked host memory
bool state_pinned(rg_ctx* c, const double* p) {
    const size_t n = (size_t)c->nvar * (size_t)c->ncell;
    if (n == 0) return false;
    for (const double* q : {p, p + (n - 1)}) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (a.type != cudaMemoryTypeHost) return false;
    }
    return true;
}

// dst[iv][t] = src[iv][ids[t] - 1] for the level's ids, by runs when they are
// long on average, else cell by cell
void gather_host(const std::vector<int>& ids, const std::vector<std::pair<int, int>>& runs, const double* src,
                 size_t ncell, int nv, double* dst) {
    const size_t n = ids.size();
    const bool by_runs = runs.size() * 8 <= n;
    for (int iv = 0; iv < nv; ++iv) {
        const double* s = src + (size_t)iv * ncell;
        double* d = dst + (size_t)iv * n;
        if (by_runs) {
            for (const auto& r : runs) {
                std::memcpy(d, s + ((size_t)r.first - 1), sizeof(double) * (size_t)r.second);
                d += r.second;
            }
        } else {
            for (size_t t = 0; t < n; ++t) d[t] = s[ids[t] - 1];
        }
    }
}

// dst[iv][ids[t] - 1] = src[iv][t], the inverse of gather_host
void scatter_host(const std::vector<int>& ids, const std::vector<std::pair<int, int>>& runs, const double* src,
                  size_t ncell, int nv, double* dst) {
    const size_t n = ids.size();
    const bool by_runs = runs.size() * 8 <= n;
    for (int iv = 0; iv < nv; ++iv) {
        const double* s = src + (size_t)iv * n;
        double* d = dst + (size_t)iv * ncell;
        if (by_runs) {
            for (const auto& r : runs) {
                std::memcpy(d + ((size_t)r.first - 1), s, sizeof(double) * (size_t)r.second);
                s += r.second;
            }
        } else {
            for (size_t t = 0; t < n; ++t) d[ids[t] - 1] = s[t];
        }
    }
}
}  // namespace

int upload_level_host(rg_ctx* c, Plan& P, const double* uold, const double* unew) {
    if (int rc = level_ids(c, P)) return rc;
    if (P.read_runs.size() <= kMaxRuns && (!unew || P.targ_runs.size() <= kMaxRuns) && state_pinned(c, uold) &&
        (!unew || state_pinned(c, unew))) {
        if (int rc = copy_runs(c, P.read_runs, c->d_uold, uold, cudaMemcpyHostToDevice)) return rc;
        if (unew) return copy_runs(c, P.targ_runs, c->d_unew, unew, cudaMemcpyHostToDevice);
        return RG_OK;
    }
    const int nv = c->nvar, nread = (int)P.h_read.size(), ntarg = unew ? (int)P.h_targ.size() : 0;
    const size_t ncell = (size_t)c->ncell;
    const size_t n = (size_t)nv * ((size_t)nread + ntarg);
    if (n == 0) return RG_OK;
    if (int rc = grow_stage(c, n)) return rc;
    // the previous call's download has completed (it synchronised), so the
    // pinned buffer is free to refill
    double* s = c->h_stage;
    gather_host(P.h_read, P.read_runs, uold, ncell, nv, s);
    if (unew) gather_host(P.h_targ, P.targ_runs, unew, ncell, nv, s + (size_t)nv * nread);
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->d_stage, s, n * sizeof(double), cudaMemcpyHostToDevice, c->stream),
                            "level upload"))
        return rc;
    k_scatter_level<<<blocks(c, std::max(nread, ntarg)), 256, 0, c->stream>>>(
        P.read_ids, nread, P.targ_ids, ntarg, nv, ncell, c->d_stage, c->d_uold, c->d_unew);
    return check_cuda(c, cudaGetLastError(), "level scatter");
}

int download_level_host(rg_ctx* c, Plan& P, double* unew, const double* src_dev) {
    if (P.targ_runs.size() <= kMaxRuns && state_pinned(c, unew)) {
        if (int rc = copy_runs(c, P.targ_runs, unew, src_dev ? src_dev : c->d_unew, cudaMemcpyDeviceToHost)) return rc;
        return check_cuda(c, cudaStreamSynchronize(c->stream), "level download sync");
    }
    const int nv = c->nvar, ntarg = (int)P.h_targ.size();
    const size_t ncell = (size_t)c->ncell;
    const size_t n = (size_t)nv * ntarg;
    if (n == 0) return check_cuda(c, cudaStreamSynchronize(c->stream), "level download sync");
    if (int rc = grow_stage(c, n)) return rc;
    k_gather_targets<<<blocks(c, ntarg), 256, 0, c->stream>>>(P.targ_ids, ntarg, nv, ncell, src_dev ? src_dev : c->d_unew,
                                                              c->d_stage);
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->h_stage, c->d_stage, n * sizeof(double), cudaMemcpyDeviceToHost,
                                               c->stream),
                            "level download"))
        return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "level download sync")) return rc;
    scatter_host(P.h_targ, P.targ_runs, c->h_stage, ncell, nv, unew);
    return RG_OK;
}

int download_level_cells(rg_ctx* c, Plan& P, double* uold, double* unew) {
    if (int rc = level_ids(c, P)) return rc;
    const int n = P.ncells;
    if (n == 0 || (!uold && !unew)) return check_cuda(c, cudaStreamSynchronize(c->stream), "level download sync");
    if (P.cell_runs.size() <= kMaxRuns && (!uold || state_pinned(c, uold)) && (!unew || state_pinned(c, unew))) {
        if (uold)
            if (int rc = copy_runs(c, P.cell_runs, uold, c->d_uold, cudaMemcpyDeviceToHost)) return rc;
        if (unew)
            if (int rc = copy_runs(c, P.cell_runs, unew, c->d_unew, cudaMemcpyDeviceToHost)) return rc;
        return check_cuda(c, cudaStreamSynchronize(c->stream), "level download sync");
    }
    const int nv = c->nvar;
    const size_t ncell = (size_t)c->ncell, m = (size_t)nv * n;
    if (int rc = grow_stage(c, 2 * m)) return rc;
    k_gather_ids2<<<blocks(c, n), 256, 0, c->stream>>>(P.read_ids, n, nv, ncell, uold ? c->d_uold : nullptr,
                                                       unew ? c->d_unew : nullptr, c->d_stage);
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->h_stage, c->d_stage, 2 * m * sizeof(double), cudaMemcpyDeviceToHost,
                                               c->stream),
                            "level download"))
        return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "level download sync")) return rc;
    if (uold) scatter_host(P.h_cells, P.cell_runs, c->h_stage, ncell, nv, uold);
    if (unew) scatter_host(P.h_cells, P.cell_runs, c->h_stage + m, ncell, nv, unew);
    return RG_OK;
}

}  // namespace rg
