// rg_nav.cuh -- tree navigation shared by the plan builder and the tree
// maintenance kernels: AmrGrid::get_nbor_cells and get_nbor_cells_coarse
// (RAMSES-CPP src/core/AmrGrid.cpp:402-444, 513-550) on the device mirror.
#pragma once

#include "rg_internal.cuh"

namespace rg {
namespace {

__device__ __forceinline__ void raise_err(DevStatus* st, int code, int info) {
    if (atomicCAS(&st->err, 0, code) == 0) st->info = info;
}

__device__ __forceinline__ int coarse_nbor(const TreeView& T, int icell, int idim, int side) {
    if (icell <= 0 || icell > T.ncoarse) return 0;
    int nx = T.nx, ny = T.ny, nz = T.nz;
    int idx = icell - 1;
    int iz = idx / (nx * ny), rem = idx % (nx * ny);
    int iy = rem / nx, ix = rem % nx;
    int c0 = ix, c1 = iy, c2 = iz;
    int d = (side == 0) ? -1 : 1;
    if (idim == 0) c0 = (c0 + d + nx) % nx;
    else if (idim == 1) c1 = (c1 + d + ny) % ny;
    else c2 = (c2 + d + nz) % nz;
    return c2 * nx * ny + c1 * nx + c0 + 1;
}

// AmrGrid::get_nbor_cells for one direction; the recursion through the father
// oct (AmrGrid.cpp:429-440) becomes a bounded loop.
__device__ int nbor_cell_dir(const TreeView& T, int igrid, int ic, int idim, int side, DevStatus* st) {
    for (int depth = 0; depth < 64; ++depth) {
        int bit = ((ic - 1) >> idim) & 1;
        int ig_idx = (side == 0) ? (bit ? 0 : 2 * idim + 1) : (bit ? 2 * idim + 2 : 0);
        int ic_pos = ((ic - 1) ^ (1 << idim)) + 1;
        int ig;
        if (ig_idx == 0) {
            ig = igrid;
        } else {
            int v = T.nbor[(size_t)(ig_idx - 1) * T.ngridmax + igrid - 1];
            ig = (v > T.ncell) ? 0 : v;
        }
        if (ig > 0) {
            if (ig_idx == 0) return T.ncoarse + (ic_pos - 1) * T.ngridmax + ig;
            int ch = (ig <= T.ncell) ? T.son[ig - 1] : 0;
            return (ch > 0) ? T.ncoarse + (ic_pos - 1) * T.ngridmax + ch : ig;
        }
        if (ig < 0) return ig;
        int ifather = T.father[igrid - 1];
        if (ifather <= T.ncoarse) return coarse_nbor(T, ifather, idim, side);
        igrid = ((ifather - T.ncoarse - 1) % T.ngridmax) + 1;
        ic = ((ifather - T.ncoarse - 1) / T.ngridmax) + 1;
    }
    raise_err(st, DE_NBOR_DEPTH, igrid);
    return 0;
}

}  // namespace
}  // namespace rg
