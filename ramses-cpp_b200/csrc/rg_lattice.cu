// rg_lattice.cu -- detection of levels that form one complete periodic lattice.
//
// A uniform grid's finest level (the reference's levelmin = levelmax runs, and
// the base level of an AMR run before refinement) holds every cell of an
// Ex x Ey x Ez periodic lattice.  On such a level the plan's neighbour cells
// (AmrGrid::get_nbor_cells, AmrGrid.cpp:402-444) and ghost stencils are the
// lattice neighbours, which lets the brick face kernel (rg_face_brick.cuh)
// stage whole 8^3 bricks of cells in shared memory instead of gathering every
// stencil cell through the plan's index arrays.  Nothing is assumed: the
// lattice is accepted only if, for every cell and interface slot, the plan's
// neighbour id, both ghost-stencil ids and the interface kind equal what the
// lattice gives; otherwise the level keeps the general kernels.
#include <vector>

#include "rg_internal.cuh"

namespace rg {

namespace {

constexpr int LTPB = 256;

// Lattice coordinates of level cell p from its oct's father chain: at every
// level a cell's coordinate is twice its father cell's plus its own bit
// ((ic-1) = ix + 2 iy + 4 iz); coarse cells are numbered x fastest.
// Returns the number of doublings (all cells of a complete level agree).
__device__ int cell_coords(const TreeView& T, const PlanView& P, int p, int* x, int* y, int* z) {
    const int icx = p / P.noct, k = p - icx * P.noct;
    int ig = P.octs[k];
    int cx = icx & 1, cy = (icx >> 1) & 1, cz = (icx >> 2) & 1, scale = 1;
    for (int guard = 0; guard < 40; ++guard) {
        const int fc = T.father[ig - 1];
        scale *= 2;
        if (fc <= 0) return -1;
        if (fc <= T.ncoarse) {
            const int idx = fc - 1;
            cx += scale * (idx % T.nx);
            cy += scale * ((idx / T.nx) % T.ny);
            cz += scale * (idx / (T.nx * T.ny));
            *x = cx;
            *y = cy;
            *z = cz;
            return scale;
        }
        const int j = fc - T.ncoarse - 1, icf = j / T.ngridmax;
        ig = j - icf * T.ngridmax + 1;
        cx += scale * (icf & 1);
        cy += scale * ((icf >> 1) & 1);
        cz += scale * ((icf >> 2) & 1);
    }
    return -1;
}

__global__ void k_lattice_fill(TreeView T, PlanView P, int scale0, int ex, int ey, int ez, int* lat_id, int* lat_p,
                               int* bad) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P.ncells; p += gridDim.x * blockDim.x) {
        int x, y, z;
        const int sc = cell_coords(T, P, p, &x, &y, &z);
        if (sc != scale0 || x < 0 || y < 0 || z < 0 || x >= ex || y >= ey || z >= ez) {
            atomicExch(bad, 1);
            continue;
        }
        const size_t site = (size_t)x + (size_t)ex * ((size_t)y + (size_t)ey * z);
        if (atomicCAS(&lat_p[site], -1, p) != -1) {
            atomicExch(bad, 1);
            continue;
        }
        const int icx = p / P.noct;
        lat_id[site] = T.ncoarse + icx * T.ngridmax + P.octs[p - icx * P.noct];
    }
}

__device__ __forceinline__ int wrap(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

__global__ void k_lattice_check(TreeView T, PlanView P, int ex, int ey, int ez, const int* __restrict__ lat_id,
                                const int* __restrict__ lat_p, int kind0, int* bad) {
    const size_t n = (size_t)ex * ey * ez;
    for (size_t site = (size_t)blockIdx.x * blockDim.x + threadIdx.x; site < n;
         site += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(site % ex), y = (int)((site / ex) % ey), z = (int)(site / ((size_t)ex * ey));
        const int p = lat_p[site];
        if (p < 0) {
            atomicExch(bad, 1);
            continue;
        }
        const int c = lat_id[site];
        for (int s = 0; s < 6; ++s) {
            const int idim = s >> 1, side = s & 1, d = side ? 1 : -1;
            auto at = [&](int off) {
                int xx = x, yy = y, zz = z;
                if (idim == 0) xx = wrap(x + off, ex);
                else if (idim == 1) yy = wrap(y + off, ey);
                else zz = wrap(z + off, ez);
                return lat_id[(size_t)xx + (size_t)ex * ((size_t)yy + (size_t)ey * zz)];
            };
            const int nb = at(d), far = at(2 * d);
            const size_t nc = (size_t)P.ncells;
            const int want_nl = side ? c : far, want_nr = side ? far : c;
            if (P.icn[s * nc + p] != nb || P.stc[((size_t)s * 2 + 0) * nc + p] != want_nl ||
                P.stc[((size_t)s * 2 + 1) * nc + p] != want_nr || P.kind[s * nc + p] != kind0)
                atomicExch(bad, 1);
        }
    }
}

// Box lattices supplied by the host (one periodic lattice per ensemble box):
// every site's plan position must hold that site's cell, every plan position
// must appear once, and the plan's neighbours, ghost stencils and kinds must
// be the box lattice's (periodic inside the box).
__global__ void k_box_lattice_check(TreeView T, PlanView P, int nbox, const int* __restrict__ ext,
                                    const int* __restrict__ off, const int* __restrict__ lat_id,
                                    const int* __restrict__ lat_p, int kind0, int* seen, int* bad) {
    const int n = P.ncells;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        int lo = 0, hi = nbox - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (off[mid] <= g) lo = mid;
            else hi = mid - 1;
        }
        const int b = lo, ex = ext[3 * b], ey = ext[3 * b + 1], ez = ext[3 * b + 2];
        const int site = g - off[b];
        const int x = site % ex, y = (site / ex) % ey, z = site / (ex * ey);
        const int p = lat_p[g], c = lat_id[g];
        if (p < 0 || p >= n || atomicExch(&seen[p], 1) != 0) {
            atomicExch(bad, 1);
            continue;
        }
        const int icx = p / P.noct;
        if (c != T.ncoarse + icx * T.ngridmax + P.octs[p - icx * P.noct]) {
            atomicExch(bad, 1);
            continue;
        }
        for (int s = 0; s < 6; ++s) {
            const int idim = s >> 1, side = s & 1, d = side ? 1 : -1;
            auto at = [&](int o) {
                int xx = x, yy = y, zz = z;
                if (idim == 0) xx = wrap(x + o, ex);
                else if (idim == 1) yy = wrap(y + o, ey);
                else zz = wrap(z + o, ez);
                return lat_id[off[b] + xx + ex * (yy + ey * zz)];
            };
            const int nb = at(d), far = at(2 * d);
            const size_t nc = (size_t)n;
            const int want_nl = side ? c : far, want_nr = side ? far : c;
            if (P.icn[s * nc + p] != nb || P.stc[((size_t)s * 2 + 0) * nc + p] != want_nl ||
                P.stc[((size_t)s * 2 + 1) * nc + p] != want_nr || P.kind[s * nc + p] != kind0)
                atomicExch(bad, 1);
        }
    }
}

int lblocks(rg_ctx* c, long long n) {
    long long b = (n + LTPB - 1) / LTPB, cap = (long long)c->sm_count * 16;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

// Accepts the level as a lattice (P.lattice = 1, lat_id/lat_p filled) or
// leaves it general.  Synchronises the stream.  Errors are CUDA errors only;
// a level that is not a lattice is not an error.
int build_lattice(rg_ctx* c, Plan& P) {
    P.lattice = 0;
    if (c->params.ndim != 3 || P.level0 || P.ncells == 0 || P.nactive != P.ncells || P.ilevel < 2) return RG_OK;
    const long long side = 1LL << (P.ilevel - 1);
    const long long ex = (long long)c->nx * side, ey = (long long)c->ny * side, ez = (long long)c->nz * side;
    if (ex * ey * ez != P.ncells || ex % 8 || ey % 8 || ez % 8) return RG_OK;
    // the interface kind of every face of a uniform leaf level: the first one's
    int8_t kind0 = 0;
    if (int rc = check_cuda(c, cudaMemcpyAsync(&kind0, P.kind, 1, cudaMemcpyDeviceToHost, c->stream), "lattice kind"))
        return rc;
    int* d_bad = nullptr;
    if (int rc = check_cuda(c, dev_alloc(c, &d_bad, sizeof(int)), "lattice flag")) return rc;
    if (int rc = check_cuda(c, dev_alloc(c, &P.lat_id, sizeof(int) * (size_t)P.ncells), "lattice ids")) return rc;
    if (int rc = check_cuda(c, dev_alloc(c, &P.lat_p, sizeof(int) * (size_t)P.ncells), "lattice positions")) return rc;
    cudaMemsetAsync(P.lat_p, 0xff, sizeof(int) * (size_t)P.ncells, c->stream);
    cudaMemsetAsync(d_bad, 0, sizeof(int), c->stream);
    if (int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "lattice kind sync")) return rc;
    const int kd = kind0;
    if ((kd & KIND_MASK) != K_GHOST && (kd & KIND_MASK) != K_SAME) {
        dev_free(c, d_bad);
        dev_free(c, P.lat_id);
        dev_free(c, P.lat_p);
        P.lat_id = P.lat_p = nullptr;
        return RG_OK;
    }
    const int scale0 = (int)side;  // cells per coarse cell and side
    k_lattice_fill<<<lblocks(c, P.ncells), LTPB, 0, c->stream>>>(tree_view(c), P.view(), scale0, (int)ex, (int)ey,
                                                                 (int)ez, P.lat_id, P.lat_p, d_bad);
    k_lattice_check<<<lblocks(c, P.ncells), LTPB, 0, c->stream>>>(tree_view(c), P.view(), (int)ex, (int)ey, (int)ez,
                                                                  P.lat_id, P.lat_p, kd, d_bad);
    int bad = 1;
    cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    dev_free(c, d_bad);
    if (int rc = check_cuda(c, e, "lattice check")) return rc;
    if (bad) {
        dev_free(c, P.lat_id);
        dev_free(c, P.lat_p);
        P.lat_id = P.lat_p = nullptr;
        return RG_OK;
    }
    P.lattice = 1;
    P.lat_e[0] = (int)ex;
    P.lat_e[1] = (int)ey;
    P.lat_e[2] = (int)ez;
    P.lat_kind = kd;
    return RG_OK;
}

int set_box_lattices(rg_ctx* c, Plan& P, const int* ext, const int* lat_id, const int* lat_p) {
    const int nbox = P.nbox;
    std::vector<int> hext(ext, ext + 3 * (size_t)nbox), hoff((size_t)nbox), hbrick((size_t)nbox + 1);
    long long sites = 0, bricks = 0;
    for (int b = 0; b < nbox; ++b) {
        const int ex = hext[3 * b], ey = hext[3 * b + 1], ez = hext[3 * b + 2];
        if (ex < 8 || ey < 8 || ez < 8 || ex % 8 || ey % 8 || ez % 8)
            return set_error(c, RG_ERR_ARG, "box " + std::to_string(b) + ": lattice extents must be multiples of 8");
        hoff[(size_t)b] = (int)sites;
        hbrick[(size_t)b] = (int)bricks;
        sites += (long long)ex * ey * ez;
        bricks += (long long)(ex / 8) * (ey / 8) * (ez / 8);
    }
    hbrick[(size_t)nbox] = (int)bricks;
    if (sites != P.ncells) return set_error(c, RG_ERR_ARG, "box lattices do not cover the level's cells once");
    int8_t kind0 = 0;
    int* d_bad = nullptr;
    int* d_seen = nullptr;
    auto fail = [&](int rc) {
        dev_free(c, d_bad);
        dev_free(c, d_seen);
        dev_free(c, P.lat_id);
        dev_free(c, P.lat_p);
        dev_free(c, P.bl_ext);
        dev_free(c, P.bl_off);
        dev_free(c, P.bl_brick_off);
        P.lat_id = P.lat_p = P.bl_ext = P.bl_off = P.bl_brick_off = nullptr;
        P.box_lattice = 0;
        return rc;
    };
    fail(RG_OK);
    const size_t n = (size_t)P.ncells;
    if (check_cuda(c, dev_alloc(c, &d_bad, sizeof(int)), "box lattice flag") ||
        check_cuda(c, dev_alloc(c, &d_seen, sizeof(int) * n), "box lattice marks") ||
        check_cuda(c, dev_alloc(c, &P.lat_id, sizeof(int) * n), "box lattice ids") ||
        check_cuda(c, dev_alloc(c, &P.lat_p, sizeof(int) * n), "box lattice positions") ||
        check_cuda(c, dev_alloc(c, &P.bl_ext, sizeof(int) * hext.size()), "box lattice extents") ||
        check_cuda(c, dev_alloc(c, &P.bl_off, sizeof(int) * hoff.size()), "box lattice offsets") ||
        check_cuda(c, dev_alloc(c, &P.bl_brick_off, sizeof(int) * hbrick.size()), "box lattice bricks"))
        return fail(RG_ERR_NOMEM);
    cudaStream_t s = c->stream;
    cudaMemcpyAsync(&kind0, P.kind, 1, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(P.lat_id, lat_id, sizeof(int) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(P.lat_p, lat_p, sizeof(int) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(P.bl_ext, hext.data(), sizeof(int) * hext.size(), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(P.bl_off, hoff.data(), sizeof(int) * hoff.size(), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(P.bl_brick_off, hbrick.data(), sizeof(int) * hbrick.size(), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d_seen, 0, sizeof(int) * n, s);
    cudaMemsetAsync(d_bad, 0, sizeof(int), s);
    if (int rc = check_cuda(c, cudaStreamSynchronize(s), "box lattice upload")) return fail(rc);
    if ((kind0 & KIND_MASK) != K_GHOST && (kind0 & KIND_MASK) != K_SAME)
        return fail(set_error(c, RG_ERR_ARG, "box lattices need a level whose faces are all ghost faces"));
    k_box_lattice_check<<<lblocks(c, P.ncells), LTPB, 0, s>>>(tree_view(c), P.view(), nbox, P.bl_ext, P.bl_off,
                                                             P.lat_id, P.lat_p, kind0, d_seen, d_bad);
    int bad = 1;
    cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (int rc = check_cuda(c, cudaStreamSynchronize(s), "box lattice check")) return fail(rc);
    dev_free(c, d_bad);
    dev_free(c, d_seen);
    d_bad = d_seen = nullptr;
    if (bad) return fail(set_error(c, RG_ERR_ARG, "box lattices do not match the level's neighbours"));
    P.box_lattice = 1;
    P.bl_nbricks = (int)bricks;
    P.lat_kind = kind0;
    return RG_OK;
}

}  // namespace rg
