// rg_output.cu -- snapshot hydro records from the device state.
//
// RamsesWriter::write_hydro (RAMSES-CPP src/io/RamsesWriter.cpp:145-226)
// writes, per level and per child slot ic and variable iv, one record of the
// level's octs in list order: density floored at smallr = 1e-10, velocities
// u_i / d, and pressure max((E - 0.5 d v^2 - e_nonthermal) (gamma - 1), 0).  A
// run whose state lives on the device would otherwise download the whole
// uold for every output; here the level's records are formed on the device
// (same floors, same operation order, so the same bits) and only they cross
// PCIe.
#include "rg_internal.cuh"
#include "rg_physics.cuh"

namespace rg {

namespace {

template <int NDIM>
__global__ void k_level_output(TreeView T, PlanView P, const double* __restrict__ uold, double gamma, double* out) {
    constexpr int NV = NDIM + 2;
    const size_t ncell = (size_t)T.ncell;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P.ncells; p += gridDim.x * blockDim.x) {
        const int icx = P.level0 ? 0 : p / P.noct, k = P.level0 ? p : p - icx * P.noct;
        const size_t id = (size_t)(P.level0 ? p + 1 : T.ncoarse + icx * T.ngridmax + P.octs[k]) - 1;
        const size_t n = (size_t)P.noct;
        double* o = out + (size_t)icx * NV * n + k;
        const double d = smax(uold[id], 1e-10);
        o[0] = d;
        double v2 = 0;
#pragma unroll
        for (int j = 1; j <= NDIM; ++j) {
            const double v = uold[j * ncell + id] / d;
            o[j * n] = v;
            v2 += v * v;
        }
        const double e_nonthermal = 0.0;
        o[(NDIM + 1) * n] = smax((uold[(NDIM + 1) * ncell + id] - 0.5 * d * v2 - e_nonthermal) * (gamma - 1.0), 0.0);
    }
}

}  // namespace

int launch_level_output(rg_ctx* c, const Plan& P, double* out_dev) {
    if (P.ncells == 0) return RG_OK;
    const int blocks = (int)std::min<long long>((P.ncells + 255) / 256, (long long)c->sm_count * 16);
    if (c->params.ndim == 1)
        k_level_output<1><<<blocks, 256, 0, c->stream>>>(tree_view(c), P.view(), c->d_uold, c->params.gamma, out_dev);
    else
        k_level_output<3><<<blocks, 256, 0, c->stream>>>(tree_view(c), P.view(), c->d_uold, c->params.gamma, out_dev);
    return check_cuda(c, cudaGetLastError(), "level output");
}

}  // namespace rg
