// rg_noalloc.cu -- a level step that allocates nothing when it is called.
//
// Who needs it: host codes that must not touch the CUDA allocator once their
// set-up is done -- a simulation running under a fixed device-memory budget
// that was fully committed at start-up, a caller that shares the GPU with a
// framework whose caching allocator owns all free memory, or a time loop that
// forbids cudaMalloc/cudaFree inside it because they synchronise the device.
// rg_godunov_level grows its flux scratch with cudaMalloc on first use of a
// level; rg_godunov_level_noalloc instead keeps that scratch in the
// file-scope array below, which the CUDA runtime places in device memory when
// the library is loaded, and takes the state buffers from the caller.
//
// Limits and sharing, stated once for every caller:
//   - the array holds RG_NOALLOC_SCRATCH_DOUBLES doubles (64 MiB): a level of
//     up to 279,620 cells in 3D (64^3 fits) or 1,398,101 cells in 1D; larger
//     levels are rejected with RG_ERR_ARG and a message, nothing is launched;
//   - every GPU that loads the library holds the 64 MiB until the process exits;
//   - all calls (all contexts, all streams) share the one array and it keeps
//     whatever the last call wrote.  Nothing in it has to start at zero: each
//     flux slot the fold kernel reads is written by the face kernel of the same
//     call.  Calls whose kernels overlap on the GPU race on the array; the
//     caller must order them (one stream, or events between streams).
//
// What the caller hands over: uold_dev and unew_dev are device memory of the
// context's device, each at least nvar*ncell doubles from the pointer on
// (checked with cudaPointerGetAttributes and the driver's address-range
// query; neither allocates).  unew_dev must already hold the level's starting
// unew -- normally a copy of uold_dev, as rg_set_unew makes it -- because the
// fold adds the flux updates to it; only the level's update targets (its
// cells and the coarser cells that take refluxes) are written.
#include <mutex>
#include <string>

#include "rg_internal.cuh"

#define RG_NOALLOC_SCRATCH_DOUBLES (8u * 1024u * 1024u)  // 64 MiB of FP64

// The scratch itself: flux slots [2*ndim][nvar][ncells] of one level.
static __device__ __align__(256) double g_noalloc_flux[RG_NOALLOC_SCRATCH_DOUBLES];

namespace {

// Host code cannot take the address of g_noalloc_flux (the host-side symbol
// is only a stand-in); the device address comes from cudaGetSymbolAddress,
// once per device, with that device current.  Resolved on the first call on
// each device.
constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {nullptr};

int scratch_address(rg_ctx* c, double** out) {
    if (c->device < 0 || c->device >= kMaxDevices) return rg::set_error(c, RG_ERR_ARG, "device id out of range");
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[c->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_flux);
        if (e != cudaSuccess) return rg::check_cuda(c, e, "cudaGetSymbolAddress(static flux scratch)");
        g_addr[c->device] = static_cast<double*>(p);
    }
    *out = g_addr[c->device];
    return RG_OK;
}

// cuMemGetAddressRange through the runtime's driver entry point (librgpu.so
// links the runtime only): the base and size of the allocation holding a
// device pointer.  Null when the driver does not offer it.
using AddressRangeFn = int (*)(unsigned long long* base, size_t* size, unsigned long long ptr);

AddressRangeFn address_range_fn() {
    static AddressRangeFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &f, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<AddressRangeFn>(nullptr);
        }
        return reinterpret_cast<AddressRangeFn>(f);
    }();
    return fn;
}

// A caller's state buffer: device memory of this context's device with room
// for nvar*ncell doubles from p on.
int check_state_buffer(rg_ctx* c, const void* p, const char* name) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return rg::set_error(c, RG_ERR_ARG, std::string(name) + " is not a pointer the CUDA runtime knows");
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
        return rg::set_error(c, RG_ERR_ARG, std::string(name) + " is not device memory");
    if (a.type == cudaMemoryTypeDevice && a.device != c->device)
        return rg::set_error(c, RG_ERR_ARG, std::string(name) + " belongs to device " + std::to_string(a.device) +
                                                ", the context runs on device " + std::to_string(c->device));
    const size_t need = sizeof(double) * (size_t)c->nvar * (size_t)c->ncell;
    if (AddressRangeFn range = address_range_fn()) {
        unsigned long long base = 0;
        size_t size = 0;
        const unsigned long long addr = reinterpret_cast<unsigned long long>(p);
        // memory the driver cannot size (an allocation of another allocator
        // mapped by hand) passes unchecked; the pointer attributes above hold
        if (range(&base, &size, addr) == 0 && addr + need > base + size)
            return rg::set_error(c, RG_ERR_ARG,
                                 std::string(name) + " holds " + std::to_string((base + size - addr) / sizeof(double)) +
                                     " doubles from the pointer on; the grid needs nvar*ncell = " +
                                     std::to_string(need / sizeof(double)));
    }
    return RG_OK;
}

}  // namespace

extern "C" int rg_godunov_level_noalloc(rg_ctx* c, int ilevel, double dt, double dx, const double* uold_dev,
                                        double* unew_dev) {
    if (!c) return RG_ERR_ARG;
    if (c->broken) return rg::set_error(c, RG_ERR_CUDA, c->err.empty() ? "context unusable after a device fault" : c->err);
    if (!uold_dev || !unew_dev) return rg::set_error(c, RG_ERR_ARG, "uold_dev and unew_dev must be device pointers");
    c->next_level = -1;  // this call uses the context's CFL word and primitive array
    if (int rc = rg::check_cuda(c, cudaSetDevice(c->device), "cudaSetDevice")) return rc;
    if (!c->have_topology) return rg::set_error(c, RG_ERR_STATE, "rg_sync_topology has not been called");
    // a resident tree whose links changed since the last plan build: the
    // plans' oct lists and neighbour ids follow the old tree, and rebuilding
    // them allocates
    if (c->tree_dirty)
        return rg::set_error(c, RG_ERR_STATE,
                             "the resident tree changed since the level plans were built; make one allocating call "
                             "for the level (rg_godunov_level or rg_set_unew) first");
    if (c->params.riemann == RG_RIEMANN_EXACT && c->params.exact_guess == RG_GUESS_LEARNED && !c->mlp_valid)
        return rg::set_error(c, RG_ERR_STATE, "exact_guess is RG_GUESS_LEARNED but no network was trained or set");
    if (int rc = check_state_buffer(c, uold_dev, "uold_dev")) return rc;
    if (int rc = check_state_buffer(c, unew_dev, "unew_dev")) return rc;
    rg::Plan* P = rg::existing_plan(c, ilevel);
    if (P && P->nbox > 0) return rg::set_error(c, RG_ERR_STATE, "ensemble level: every box has its own dt");
    if (!P)
        return rg::set_error(c, RG_ERR_STATE,
                             "no level plan: building one allocates, so call rg_godunov_level (or rg_set_unew) "
                             "for this level once after rg_sync_topology or a change of the resident tree, "
                             "before the allocation-free calls");
    const size_t need = (size_t)(2 * c->params.ndim) * (c->params.ndim + 2) * (size_t)P->ncells;
    if (need > RG_NOALLOC_SCRATCH_DOUBLES)
        return rg::set_error(c, RG_ERR_ARG,
                             "level has " + std::to_string(P->ncells) + " cells and needs " + std::to_string(need) +
                                 " scratch doubles; the static scratch holds " +
                                 std::to_string((size_t)RG_NOALLOC_SCRATCH_DOUBLES) + " (64 MiB)");
    double* flux = nullptr;
    if (int rc = scratch_address(c, &flux)) return rc;
    if (int rc = rg::launch_set_dt_host(c, dt, dx)) return rc;
    return rg::launch_godunov_ext(c, *P, uold_dev, unew_dev, c->d_prim, flux);
}
