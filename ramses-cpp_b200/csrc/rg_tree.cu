// rg_tree.cu -- AMR tree maintenance on the device (TreeUpdater on the GPU).
//
// The reference (RAMSES-CPP) rebuilds its tree on the host between hydro
// steps: TreeUpdater::flag_fine, smooth_fine, test_flag, ensure_ref_rules,
// make_grid_fine, remove_grid_fine and restrict_fine
// (src/core/TreeUpdater.cpp:27-636), with the oct free list and level lists of
// AmrGrid (src/core/AmrGrid.cpp:259-302), the coordinate lookups of
// get_27_cell_neighbors (:474-511) and the prolongation interpol_hydro
// (src/solvers/hydro/HydroSolver.cpp:734-876).  Here the tree stays in device
// memory for a whole run and every one of those operations is a few kernels
// over the level's octs; the host keeps only the list heads, tails and counts
// and a mirror of the free list's order.
//
// Every loop of the reference that looks sequential is one of two kinds:
//   - per cell or per oct with disjoint writes (flags, gradients, restriction,
//     nesting rules, the new octs' neighbours and interpolated states): the
//     writes of one iteration never feed a later iteration's reads, so one
//     thread per cell or oct gives the same bits;
//   - order-carrying (which oct id a refined cell gets, the level and free
//     lists' links): the reference walks cells in list order, pops ids from
//     the head of the FIFO free list and appends to list tails, so the k-th
//     refined cell in list order gets the k-th free id and the lists end up
//     as the compacted sequences; an exclusive scan over the list order
//     reproduces both.
// Scope: refinement of levels above the coarse level (the coarse level,
// ilevel 1 in the reference's numbering, is refined at initialisation on the
// host; below levelmin its flags are all set, which is handled), ncpu == 1,
// nvar == ndim + 2 = 5 and no boundary patches, as on the rest of this path.
// A free list too short for a refinement grows the arrays as the reference's
// resize_grids does (tree_grow).
// The per-flagged-cell printf of flag_fine (TreeUpdater.cpp:519) is not
// reproduced: it writes to stdout and changes no state.
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "rg_face.cuh"
#include "rg_nav.cuh"

namespace rg {

namespace {

constexpr int TPB = 256;
inline int nblk(long long n) { return (int)std::max(1LL, std::min((n + TPB - 1) / TPB, 1LL << 30)); }

struct TreeMut {
    int ncoarse, ngridmax, ncell;
    int* son;
    int* father;
    int* nbor;
    int* next;
    int* prev;
    int* flag1;
    int* flag2;
    int* cpu_map;
    double* xg;
    double* uold;
    double* unew;
};

TreeMut tree_mut(rg_ctx* c) {
    return TreeMut{c->ncoarse, c->ngridmax, c->ncell, c->d_son, c->d_father, c->d_nbor, c->d_next, c->d_prev,
                   c->d_flag1, c->d_flag2, c->d_cpu_map, c->d_xg, c->d_uold, c->d_unew};
}

// cell id (1-based) of position p = icx * noct + k of a level's cells
__device__ __forceinline__ int lvl_cell(const TreeMut& M, const int* octs, int noct, int p) {
    const int icx = p / noct, k = p - icx * noct;
    return M.ncoarse + icx * M.ngridmax + octs[k];
}

// AmrGrid::get_nbor_cells_exact (AmrGrid.cpp:449-472) for one direction: the
// neighbour cell at the same level, or 0 when that oct does not exist
__device__ __forceinline__ int nbor_exact_dir(const TreeMut& M, int igrid, int ic, int idim, int side) {
    const int bit = ((ic - 1) >> idim) & 1;
    const int ig_idx = (side == 0) ? (bit ? 0 : 2 * idim + 1) : (bit ? 2 * idim + 2 : 0);
    const int ic_pos = ((ic - 1) ^ (1 << idim)) + 1;
    if (ig_idx == 0) return M.ncoarse + (ic_pos - 1) * M.ngridmax + igrid;
    int ig = M.nbor[(size_t)(ig_idx - 1) * M.ngridmax + igrid - 1];
    if (ig > M.ncell) ig = 0;  // get_nbor_grids (AmrGrid.cpp:389-400)
    if (ig <= 0) return 0;
    const int ch = M.son[ig - 1];
    return ch > 0 ? M.ncoarse + (ic_pos - 1) * M.ngridmax + ch : 0;
}

// ---------------------------------------------------------------- flag_fine
// TreeUpdater.cpp:414-446: reset, then keep cells whose son oct has a
// refined or flagged cell (always flag below levelmin)
__global__ void k_flag_init(TreeMut M, const int* __restrict__ octs, int noct, int below_min) {
    const int n = 8 * noct;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int idc = lvl_cell(M, octs, noct, p) - 1;
        int f = 0;
        if (below_min) {
            f = 1;
        } else {
            const int ch = M.son[idc];
            if (ch > 0)
                for (int s = 0; s < 8; ++s) {
                    const int ids = M.ncoarse + s * M.ngridmax + ch - 1;
                    if (M.son[ids] > 0 || M.flag1[ids] == 1) {
                        f = 1;
                        break;
                    }
                }
        }
        M.flag1[idc] = f;
    }
}

// smooth_fine (TreeUpdater.cpp:211-259): unflagged cells with a flagged
// same-level neighbour; marks first, then applied (the reference's ok_flag)
__global__ void k_smooth_mark(TreeMut M, const int* __restrict__ octs, int noct, int* ok) {
    const int n = 8 * noct;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int icx = p / noct, k = p - icx * noct, ig = octs[k], ic = icx + 1;
        const int idc = M.ncoarse + icx * M.ngridmax + ig - 1;
        int o = 0;
        if (M.flag1[idc] == 0) {
            // the six lookups first, so that their loads are in flight together
            int nc[6];
#pragma unroll
            for (int s = 0; s < 6; ++s) nc[s] = nbor_exact_dir(M, ig, ic, s >> 1, s & 1);
            int nf = 0;
#pragma unroll
            for (int s = 0; s < 6; ++s)
                if (nc[s] > 0 && nc[s] <= M.ncell && M.flag1[nc[s] - 1] == 1) ++nf;
            o = nf > 0;
        }
        ok[p] = o;
    }
}

__global__ void k_smooth_apply(TreeMut M, const int* __restrict__ octs, int noct, const int* __restrict__ ok) {
    const int n = 8 * noct;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        if (ok[p] == 1) M.flag1[lvl_cell(M, octs, noct, p) - 1] = 1;
}

struct CellState {
    double d, v[3], p;
};

// get_cell_state of flag_fine (TreeUpdater.cpp:346-385), hydro variables, no
// non-thermal energies
__device__ __forceinline__ CellState cell_state(const TreeMut& M, int cell, double gamma) {
    CellState s{};
    const size_t nc = (size_t)M.ncell, i = (size_t)cell - 1;
    s.d = smax(M.uold[i], 1e-10);
    double v2 = 0.0;
#pragma unroll
    for (int idim = 0; idim < 3; ++idim) {
        s.v[idim] = M.uold[(size_t)(2 + idim - 1) * nc + i] / s.d;
        v2 = v2 + s.v[idim] * s.v[idim];
    }
    const double ek = 0.5 * s.d * v2;
    const double em = 0.0, e_nonthermal = 0.0;
    const double e_tot = M.uold[(size_t)4 * nc + i];
    s.p = smax((e_tot - ek - em - e_nonthermal) * (gamma - 1.0), s.d * 1e-10);
    return s;
}

__device__ __forceinline__ double err_grad(double l, double c, double r, double floor_val) {
    return 2.0 * smax(fabs(r - c) / (r + c + floor_val), fabs(c - l) / (c + l + floor_val));
}

__device__ __forceinline__ double err_grad_u(double vl, double vc, double vr, double pl, double pc, double pr,
                                             double dl, double dc, double dr, double gamma) {
    const double floor_val = 1e-10;
    const double cg = sqrt(smax(gamma * pl / dl, floor_val * floor_val));
    const double cm = sqrt(smax(gamma * pc / dc, floor_val * floor_val));
    const double cd = sqrt(smax(gamma * pr / dr, floor_val * floor_val));
    return 2.0 * smax(fabs(vr - vc) / (cd + cm + fabs(vr) + fabs(vc) + floor_val),
                      fabs(vc - vl) / (cm + cg + fabs(vc) + fabs(vl) + floor_val));
}

// gradient criteria (TreeUpdater.cpp:491-535), 3D hydro: density, pressure,
// velocity (no magnetic energy on the hydro path)
__global__ void k_flag_grad(TreeMut M, const int* __restrict__ octs, int noct, double ed, double ep, double ev,
                            double gamma) {
    const int n = 8 * noct;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int icx = p / noct, k = p - icx * noct, ig = octs[k], ic = icx + 1;
        const int idc = M.ncoarse + icx * M.ngridmax + ig - 1;
        if (M.flag1[idc] != 0) continue;
        // every direction's neighbour ids first (independent lookups, their
        // loads in flight together); the directions are then tested in order
        // up to the first that flags the cell, as in the reference
        int nl[3], nr[3];
#pragma unroll
        for (int idim = 0; idim < 3; ++idim) {
            nl[idim] = nbor_exact_dir(M, ig, ic, idim, 0);
            nr[idim] = nbor_exact_dir(M, ig, ic, idim, 1);
        }
#pragma unroll
        for (int idim = 0; idim < 3; ++idim) {
            if (nl[idim] == 0) nl[idim] = M.nbor[(size_t)(2 * idim) * M.ngridmax + ig - 1];
            if (nr[idim] == 0) nr[idim] = M.nbor[(size_t)(2 * idim + 1) * M.ngridmax + ig - 1];
        }
        const CellState sc = cell_state(M, idc + 1, gamma);
        bool ok = false;
        for (int idim = 0; idim < 3 && !ok; ++idim) {
            const int id_l = nl[idim], id_r = nr[idim];
            const CellState sl = (id_l > 0 && id_l <= M.ncell) ? cell_state(M, id_l, gamma) : sc;
            const CellState sr = (id_r > 0 && id_r <= M.ncell) ? cell_state(M, id_r, gamma) : sc;
            if (ed > 0.0 && err_grad(sl.d, sc.d, sr.d, 1e-10) > ed) ok = true;
            else if (ep > 0.0 && err_grad(sl.p, sc.p, sr.p, 1e-10) > ep) ok = true;
            else if (ev > 0.0 && err_grad_u(sl.v[idim], sc.v[idim], sr.v[idim], sl.p, sc.p, sr.p, sl.d, sc.d, sr.d,
                                            gamma) > ev)
                ok = true;
        }
        if (ok) M.flag1[idc] = 1;
    }
}

// test_flag (TreeUpdater.cpp:263-307): cells whose son oct has a refined or
// flagged cell stay flagged
__global__ void k_test_flag(TreeMut M, const int* __restrict__ octs, int noct) {
    const int n = 8 * noct;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int idc = lvl_cell(M, octs, noct, p) - 1;
        const int ch = M.son[idc];
        if (ch <= 0) continue;
        for (int s = 0; s < 8; ++s) {
            const int ids = M.ncoarse + s * M.ngridmax + ch - 1;
            if (M.son[ids] > 0 || M.flag1[ids] == 1) {
                M.flag1[idc] = 1;
                break;
            }
        }
    }
}

// AmrGrid::get_cell_level (AmrGrid.hpp:69-80)
__device__ __forceinline__ int cell_level(const TreeMut& M, int icell) {
    if (icell <= M.ncoarse) return 0;
    int cur = ((icell - M.ncoarse - 1) % M.ngridmax) + 1;
    int level = 1;
    for (int guard = 0; guard < 64 && cur > 0; ++guard) {
        const int fc = M.father[cur - 1];
        if (fc <= M.ncoarse) break;
        cur = ((fc - M.ncoarse - 1) % M.ngridmax) + 1;
        ++level;
    }
    return level;
}

struct Geo {
    int nx, ny, nz;
    double boxlen;
};

// AmrGrid::get_cell_center (AmrGrid.cpp:331-365), 3D
__device__ void cell_center(const TreeMut& M, const Geo& G, int icell, double* xc) {
    xc[0] = 0.5 * G.boxlen;
    xc[1] = 0.5 * G.boxlen;
    xc[2] = 0.5 * G.boxlen;
    if (icell <= M.ncoarse) {
        int idx = icell - 1;
        const int iz = idx / (G.nx * G.ny);
        idx %= (G.nx * G.ny);
        const int iy = idx / G.nx, ix = idx % G.nx;
        const double dxc = G.boxlen / (double)max(G.nx, max(G.ny, G.nz));
        xc[0] = (ix + 0.5) * dxc;
        xc[1] = (iy + 0.5) * dxc;
        xc[2] = (iz + 0.5) * dxc;
        return;
    }
    const int ig = ((icell - M.ncoarse - 1) % M.ngridmax) + 1;
    const int idc = (icell - M.ncoarse - 1) / M.ngridmax;
    const int ixyz[3] = {idc & 1, (idc & 2) >> 1, (idc & 4) >> 2};
    const int level = cell_level(M, icell);
    const double dx = G.boxlen / (double)(G.nx * (1 << level));
    const double scale = G.boxlen / (double)G.nx;
#pragma unroll
    for (int d = 0; d < 3; ++d) xc[d] = M.xg[(size_t)d * M.ngridmax + ig - 1] * scale + (double)(ixyz[d] - 0.5) * dx;
}

// AmrGrid::find_cell_by_coords (AmrGrid.cpp:367-387), 3D
__device__ int cell_at(const TreeMut& M, const Geo& G, const double* x, int level) {
    const double dxc = G.boxlen / (double)max(G.nx, max(G.ny, G.nz));
    const int ix = min(max((int)(x[0] / dxc), 0), G.nx - 1);
    const int iy = min(max((int)(x[1] / dxc), 0), G.ny - 1);
    const int iz = min(max((int)(x[2] / dxc), 0), G.nz - 1);
    int cur = iz * G.nx * G.ny + iy * G.nx + ix + 1;
    const double scale = G.boxlen / (double)G.nx;
    for (int lev = 1; lev <= level && M.son[cur - 1] > 0; ++lev) {
        const int ig = M.son[cur - 1];
        const int ixc = x[0] > M.xg[ig - 1] * scale ? 1 : 0;
        const int iyc = x[1] > M.xg[(size_t)M.ngridmax + ig - 1] * scale ? 1 : 0;
        const int izc = x[2] > M.xg[(size_t)2 * M.ngridmax + ig - 1] * scale ? 1 : 0;
        const int ic = izc * 4 + iyc * 2 + ixc + 1;
        cur = M.ncoarse + (ic - 1) * M.ngridmax + ig;
    }
    return cur;
}

// ensure_ref_rules (TreeUpdater.cpp:578-634): an oct stays flagged only when
// all 27 cells around its father exist at the father's level and are refined
// (get_27_cell_neighbors, AmrGrid.cpp:474-511, by coordinates).  One thread
// per (oct, neighbour): each lookup is a descent of the tree through
// dependent loads, so the 27 of an oct run side by side instead of one after
// another.  A failing neighbour clears the oct's flags; the reference stops
// at the first failure, which writes the same zeros.
__global__ void k_ensure_ref_rules(TreeMut M, Geo G, const int* __restrict__ octs, int noct) {
    const long long n = 27LL * noct;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q / 27), j = (int)(q % 27);
        const int ig = octs[k];
        const int fc = M.father[ig - 1];
        bool ok = fc > 0;
        if (ok && fc > M.ncell) ok = false;  // get_27_cell_neighbors returns no neighbours
        if (ok) {
            const int level = cell_level(M, fc);
            double xc[3];
            cell_center(M, G, fc, xc);
            const double dxl = G.boxlen / (double)(G.nx * (1 << level));
            const int dz = j / 9 - 1, dy = (j / 3) % 3 - 1, dx = j % 3 - 1;
            double x[3] = {xc[0], xc[1], xc[2]};
            x[0] += dx * dxl;
            x[1] += dy * dxl;
            x[2] += dz * dxl;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (x[d] < 0.0) x[d] += G.boxlen;
                else if (x[d] >= G.boxlen) x[d] -= G.boxlen;
            }
            const int nb = cell_at(M, G, x, level);
            if (cell_level(M, nb) != level || M.son[nb - 1] == 0) ok = false;
        }
        if (!ok)
            for (int s = 0; s < 8; ++s) M.flag1[M.ncoarse + s * M.ngridmax + ig - 1] = 0;
    }
}

// flag_fine on the coarse level below levelmin (TreeUpdater.cpp:396-413): every
// coarse cell flagged and owned by this process
__global__ void k_flag_coarse_below_min(TreeMut M) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M.ncoarse; i += gridDim.x * blockDim.x) {
        M.cpu_map[i] = 1;
        M.flag1[i] = 1;
    }
}

// make_grid_fine(1) candidates (TreeUpdater.cpp:33-41): counted only; refining
// the coarse level is left to the host
__global__ void k_coarse_candidates(TreeMut M, int* count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M.ncoarse; i += gridDim.x * blockDim.x)
        if (M.flag1[i] == 1 && M.flag2[i] == 1 && M.son[i] == 0) atomicAdd(count, 1);
}

// ---------------------------------------------------------------- make_grid_fine
__global__ void k_authorize(TreeMut M) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M.ncell; i += gridDim.x * blockDim.x)
        M.flag2[i] = (M.cpu_map[i] == 1) ? 1 : 0;
}

// candidates in the reference's order: octs in list order, child slots inside
__global__ void k_refine_mark(TreeMut M, const int* __restrict__ octs, int noct, int* mark) {
    const int n = 8 * noct;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int k = q >> 3, icx = q & 7;
        const int idc = M.ncoarse + icx * M.ngridmax + octs[k] - 1;
        mark[q] = (M.flag1[idc] == 1 && M.flag2[idc] == 1 && M.son[idc] == 0) ? 1 : 0;
    }
}

// interpol_hydro (HydroSolver.cpp:734-876), 3D, no non-thermal energies or
// passive scalars, no barotropic EOS
__device__ void interpol_3d(const double u1[7][5], double u2[8][5], int interpol_var, int interpol_type, double gam,
                            double smalle) {
    constexpr int NV = 5;
    double q1[7][NV], q2[8][NV];
    if (interpol_var == 0) {
        for (int i = 0; i < 7; ++i)
            for (int iv = 0; iv < NV; ++iv) q1[i][iv] = u1[i][iv];
    } else if (interpol_var == 1) {
        for (int i = 0; i < 7; ++i) {
            const double d = smax(u1[i][0], 1e-10);
            q1[i][0] = u1[i][0];
            double e_kin = 0.0;
            for (int idim = 1; idim <= 3; ++idim) {
                q1[i][idim] = u1[i][idim];
                e_kin = e_kin + 0.5 * u1[i][idim] * u1[i][idim] / d;
            }
            const double e_nonthermal = 0.0;
            q1[i][4] = u1[i][4] - e_kin - e_nonthermal;
        }
    } else {
        for (int i = 0; i < 7; ++i) ctoprim<3>(u1[i], q1[i], gam, smalle);
    }
    for (int iv = 0; iv < NV; ++iv) {
        double slopes[3] = {0.0, 0.0, 0.0};
        for (int idim = 0; idim < 3; ++idim) {
            const double dlft = q1[0][iv] - q1[2 * idim + 1][iv];
            const double drgt = q1[2 * idim + 2][iv] - q1[0][iv];
            if (dlft * drgt > 0.0) {
                const double sgn = (dlft >= 0.0) ? 1.0 : -1.0;
                int itype = interpol_type;
                if (interpol_type == 4) itype = (interpol_var == 2 && iv >= 1 && iv <= 3) ? 3 : 2;
                if (itype == 1) slopes[idim] = sgn * 0.5 * smin(fabs(dlft), fabs(drgt));
                else if (itype == 2) slopes[idim] = sgn * smin3(fabs(dlft), fabs(drgt), 0.25 * fabs(dlft + drgt));
                else if (itype == 3) slopes[idim] = 0.25 * (dlft + drgt);
                else slopes[idim] = 0.0;
            }
        }
        for (int i = 0; i < 8; ++i) {
            const int ix = i & 1, iy = (i & 2) >> 1, iz = (i & 4) >> 2;
            q2[i][iv] = q1[0][iv] + (ix - 0.5) * slopes[0] + (iy - 0.5) * slopes[1] + (iz - 0.5) * slopes[2];
        }
    }
    if (interpol_var == 0) {
        for (int i = 0; i < 8; ++i)
            for (int iv = 0; iv < NV; ++iv) u2[i][iv] = q2[i][iv];
    } else if (interpol_var == 1) {
        for (int i = 0; i < 8; ++i) {
            const double d = smax(q2[i][0], 1e-10);
            u2[i][0] = d;
            double e_kin = 0.0;
            for (int idim = 1; idim <= 3; ++idim) {
                u2[i][idim] = q2[i][idim];
                e_kin = e_kin + 0.5 * q2[i][idim] * q2[i][idim] / d;
            }
            const double e_nonthermal = 0.0;
            u2[i][4] = q2[i][4] + e_kin + e_nonthermal;
        }
    } else {
        const double oneover_n2d = 1.0 / 8;
        for (int di = 1; di <= 3; ++di) {
            double mom_sum = 0.0;
            for (int i = 0; i < 8; ++i) mom_sum = mom_sum + q2[i][0] * q2[i][di] * oneover_n2d;
            const double mom_err = mom_sum - u1[0][di];
            for (int i = 0; i < 8; ++i) {
                const double d = smax(q2[i][0], 1e-10);
                q2[i][di] = (d * q2[i][di] - mom_err) / d;
            }
        }
        for (int i = 0; i < 8; ++i) {
            const double d = smax(q2[i][0], 1e-10);
            const double p = smax(q2[i][4], 1e-20);
            u2[i][0] = d;
            double v2 = 0.0;
            for (int di = 1; di <= 3; ++di) {
                u2[i][di] = d * q2[i][di];
                v2 = v2 + q2[i][di] * q2[i][di];
            }
            const double e_thermal = p / (gam - 1.0), e_kinetic = 0.5 * d * v2, e_nonthermal = 0.0;
            u2[i][4] = e_thermal + e_kinetic + e_nonthermal;
        }
    }
}

// one refined cell: its new oct (the j-th free id), links to father and
// neighbours, coordinates, prolonged state (TreeUpdater.cpp:76-149)
__global__ void k_refine(TreeMut M, TreeView T, Geo G, const int* __restrict__ octs, int noct,
                         const int* __restrict__ mark, const int* __restrict__ rank, const int* __restrict__ fq,
                         int fq_head, int ilevel, int interpol_var, int interpol_type, double gamma, double smalle,
                         const int* __restrict__ bound_type, int nbound_type, int* newlist, DevStatus* st) {
    const int n = 8 * noct;
    const size_t nc = (size_t)M.ncell;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        if (!mark[q]) continue;
        const int k = q >> 3, icx = q & 7, ig = octs[k], ic = icx + 1;
        const int idc = M.ncoarse + icx * M.ngridmax + ig - 1;
        const int j = rank[q];
        const int new_ig = fq[(int)(((long long)fq_head + j) % M.ngridmax)];
        newlist[j] = new_ig;
        M.son[idc] = new_ig;
        M.father[new_ig - 1] = idc + 1;
        int icn[6];
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            icn[s] = nbor_cell_dir(T, ig, ic, s >> 1, s & 1, st);
            M.nbor[(size_t)s * M.ngridmax + new_ig - 1] = icn[s];
        }
        const double dx_level = 1.0 / (double)(1 << (ilevel - 1));
        const int ixyz[3] = {icx & 1, (icx & 2) >> 1, (icx & 4) >> 2};
#pragma unroll
        for (int d = 0; d < 3; ++d)
            M.xg[(size_t)d * M.ngridmax + new_ig - 1] =
                M.xg[(size_t)d * M.ngridmax + ig - 1] + (double)(ixyz[d] - 0.5) * dx_level;
        double u1[7][5], u2[8][5];
        for (int iv = 0; iv < 5; ++iv) u1[0][iv] = M.uold[(size_t)iv * nc + idc];
        for (int i = 1; i <= 6; ++i) {
            const int id_n = icn[i - 1];
            if (id_n > 0) {
                for (int iv = 0; iv < 5; ++iv) u1[i][iv] = M.uold[(size_t)iv * nc + id_n - 1];
            } else {
                for (int iv = 0; iv < 5; ++iv) u1[i][iv] = u1[0][iv];
                const int ib = -id_n;
                if (ib > 0 && ib <= nbound_type && bound_type[ib - 1] == 1) {
                    const int idim = (i - 1) / 2;
                    u1[i][1 + idim] *= -1.0;
                }
            }
        }
        interpol_3d(u1, u2, interpol_var, interpol_type, gamma, smalle);
        for (int isc = 0; isc < 8; ++isc) {
            const size_t child = (size_t)M.ncoarse + (size_t)isc * M.ngridmax + new_ig - 1;
            for (int iv = 0; iv < 5; ++iv) {
                M.uold[(size_t)iv * nc + child] = u2[isc][iv];
                M.unew[(size_t)iv * nc + child] = u2[isc][iv];
            }
            M.cpu_map[child] = 1;
        }
    }
}

// links of list[0..n) chained in order after `before` (0: a list of its own):
// add_to_level_list (AmrGrid.cpp:289-302) and the free list's tail pushes
// (free_grid, :282-284)
__global__ void k_link_chain(int* next, int* prev, const int* __restrict__ list, int n, int before) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int g = list[j];
        prev[g - 1] = j > 0 ? list[j - 1] : before;
        next[g - 1] = j + 1 < n ? list[j + 1] : 0;
        if (j == 0 && before > 0) next[before - 1] = g;
    }
}

// ---------------------------------------------------------------- remove_grid_fine
__global__ void k_kill_mark(TreeMut M, const int* __restrict__ octs, int noct, int* mark) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < noct; k += gridDim.x * blockDim.x) {
        const int ig = octs[k];
        const int fc = M.father[ig - 1];
        int rm = 0;
        if (fc > 0 && M.flag1[fc - 1] == 0) {
            rm = 1;
            for (int s = 0; s < 8; ++s)
                if (M.son[M.ncoarse + s * M.ngridmax + ig - 1] > 0) {
                    rm = 0;
                    break;
                }
        }
        mark[k] = rm;
    }
}

// make_grid_fine and remove_grid_fine candidates among a level's octs:
// k_refine_mark's and k_kill_mark's tests, without writing marks; `bit` (the
// level's) is or-ed into bits[0] for a refinement, bits[1] for a removal
__global__ void k_change_probe(TreeMut M, const int* __restrict__ octs, int noct, unsigned* bits, unsigned bit) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < noct; k += gridDim.x * blockDim.x) {
        const int ig = octs[k];
        bool refine = false, refined_child = false;
        for (int s = 0; s < 8; ++s) {
            const int idc = M.ncoarse + s * M.ngridmax + ig - 1;
            if (M.son[idc] > 0) refined_child = true;
            else if (M.flag1[idc] == 1 && M.flag2[idc] == 1) refine = true;
        }
        const int fc = M.father[ig - 1];
        if (refine) atomicOr(bits, bit);
        if (fc > 0 && M.flag1[fc - 1] == 0 && !refined_child) atomicOr(bits + 1, bit);
    }
}

// unlink and free the marked octs (TreeUpdater.cpp:164-181, free_grid
// AmrGrid.cpp:270-287): compacted kept list, freed ids in list order, the
// freed ids appended to the free-list ring
__global__ void k_kill(TreeMut M, const int* __restrict__ octs, int noct, const int* __restrict__ mark,
                       const int* __restrict__ rank, int* kept, int* freed, int* fq, int fq_tail) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < noct; k += gridDim.x * blockDim.x) {
        const int ig = octs[k];
        const int r = rank[k];
        if (!mark[k]) {
            kept[k - r] = ig;
            continue;
        }
        freed[r] = ig;
        fq[(int)(((long long)fq_tail + r) % M.ngridmax)] = ig;
        for (int s = 0; s < 6; ++s) M.nbor[(size_t)s * M.ngridmax + ig - 1] = 0;
        const int fc = M.father[ig - 1];
        if (fc > 0) M.son[fc - 1] = 0;
        M.father[ig - 1] = 0;
        for (int s = 0; s < 8; ++s) {
            const int idc = M.ncoarse + s * M.ngridmax + ig - 1;
            M.son[idc] = 0;
            M.flag1[idc] = 0;
            M.flag2[idc] = 0;
        }
    }
}

// ---------------------------------------------------------------- restrict_fine
// father = mean of its 8 children, summed in child order (TreeUpdater.cpp:188-207).
// The 40 child values are loaded before any store, so they are in flight
// together (a store to the father could alias a later load otherwise).
__device__ __forceinline__ void restrict_oct(const TreeMut& M, int ig) {
    const size_t nc = (size_t)M.ncell;
    const int fc = M.father[ig - 1];
    if (fc <= 0) return;
    double v[5][8];
#pragma unroll
    for (int iv = 0; iv < 5; ++iv)
#pragma unroll
        for (int s = 0; s < 8; ++s) v[iv][s] = M.uold[(size_t)iv * nc + M.ncoarse + (size_t)s * M.ngridmax + ig - 1];
#pragma unroll
    for (int iv = 0; iv < 5; ++iv) {
        double sum = 0;
#pragma unroll
        for (int s = 0; s < 8; ++s) sum += v[iv][s];
        M.uold[(size_t)iv * nc + fc - 1] = sum / 8;
    }
}

__global__ void k_restrict(TreeMut M, const int* __restrict__ octs, int noct) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < noct; k += gridDim.x * blockDim.x) restrict_oct(M, octs[k]);
}

// The coarse step's work below levelmin in two launches.  k_tail_flags_restrict:
// its first nb_r blocks do restrict_fine(levelmin-1) over the levelmin list
// (octs, noct), the others flag_fine(il) for il = levelmin-1..2 over the
// lists F (k_flag_init's below-levelmin case: every cell flagged) and for the
// coarse cells (k_flag_coarse_below_min) -- independent writes (uold of the
// levelmin-1 cells, flags).  k_tail_cascade: restrict_fine(il) for il =
// levelmin-2..0 over the lists R given coarsest last, in one block with a
// barrier between levels so that each restriction reads the one before it
// (the threads of a block see each other's global writes after
// __syncthreads); these levels are small (585 octs in the lists below
// levelmin-1 for a levelmin of 7), so one block's latency is below the
// launches it replaces.
struct LevelLists {
    const int* octs[32];
    int noct[32];
    int n;
};

__global__ void k_tail_flags_restrict(TreeMut M, const int* __restrict__ octs, int noct, int nb_r, LevelLists F) {
    const int b = (int)blockIdx.x;
    if (b < nb_r) {
        for (int k = b * blockDim.x + threadIdx.x; k < noct; k += nb_r * blockDim.x) restrict_oct(M, octs[k]);
        return;
    }
    const int fb = b - nb_r, nfb = (int)gridDim.x - nb_r;
    const int stride = nfb * blockDim.x;
    for (int j = 0; j < F.n; ++j) {
        const int nj = F.noct[j], n = 8 * nj;
        for (int p = fb * blockDim.x + threadIdx.x; p < n; p += stride) M.flag1[lvl_cell(M, F.octs[j], nj, p) - 1] = 1;
    }
    for (int i = fb * blockDim.x + threadIdx.x; i < M.ncoarse; i += stride) {
        M.cpu_map[i] = 1;
        M.flag1[i] = 1;
    }
}

__global__ void __launch_bounds__(1024) k_tail_cascade(TreeMut M, LevelLists R) {
    for (int j = 0; j < R.n; ++j) {
        if (j > 0) __syncthreads();
        const int* octs = R.octs[j];
        for (int k = threadIdx.x; k < R.noct[j]; k += blockDim.x) restrict_oct(M, octs[k]);
    }
}

// ---------------------------------------------------------------- host side
int hidx(const rg_ctx* c, int ilevel) { return ilevel * (c->ncpu + c->nboundary); }

// A change of the tree's links reaches the plans of levels lo..hi (bits of
// levels above 63 are implied) and the oct list of level `list` (-1: none).
void mark_changed(rg_ctx* c, int lo, int hi, int list) {
    for (int L = lo < 0 ? 0 : lo; L <= hi && L <= 63; ++L) c->plans_dirty |= 1ull << L;
    if (list >= 0 && list <= 63) c->lists_dirty |= 1ull << list;
}

// The cached oct list of level L (current before the change) made the
// level's list after it: `keep` entries from the old list's start, then the
// `add` octs (device, in list order) after them.  false (nothing done) when
// the list is not cached; it is then walked again after the refresh.
bool keep_cached_list(rg_ctx* c, int L, int keep, const int* add, int nadd) {
    if (L < 0 || (int)c->lvl_ver.size() <= L || c->lvl_ver[(size_t)L] != c->topo_version) return false;
    const size_t l = (size_t)L;
    const int need = keep + nadd;
    if (need > c->lvl_cap[l]) {
        const int cap = (need + 1023) / 1024 * 1024;
        int* grown = nullptr;
        if (dev_alloc(c, &grown, sizeof(int) * (size_t)cap) != cudaSuccess) return false;
        if (keep > 0) cudaMemcpyAsync(grown, c->lvl_octs[l], sizeof(int) * (size_t)keep, cudaMemcpyDeviceToDevice, c->stream);
        dev_free(c, c->lvl_octs[l]);
        c->lvl_octs[l] = grown;
        c->lvl_cap[l] = cap;
    }
    if (nadd > 0)
        cudaMemcpyAsync(c->lvl_octs[l] + keep, add, sizeof(int) * (size_t)nadd, cudaMemcpyDeviceToDevice, c->stream);
    c->lvl_n[l] = need;
    return true;
}

// RG_OK to go on, kNoOp when the call does nothing (ilevel >= nlevelmax, where
// the reference returns at once), else an error code (error codes are negative)
constexpr int kNoOp = 1;
int check_tree(rg_ctx* c, int ilevel) {
    if (!c->tree_resident) return set_error(c, RG_ERR_STATE, "no device-resident tree: call rg_tree_attach first");
    if (ilevel >= c->nlevelmax) return kNoOp;
    if (ilevel < 1) return set_error(c, RG_ERR_ARG, "level below 1");
    c->next_level = -1;  // the state or the topology may change
    return refresh_tree(c);
}

// scratch carved from one pool allocation: [octs ngm][mark 8ngm+1][rank 8ngm+1][list ngm][list2 ngm]
struct TreeScratch {
    int *octs, *mark, *rank, *list, *list2;
};

int tree_scratch(rg_ctx* c, TreeScratch* s) {
    const size_t ngm = (size_t)c->ngridmax, need = 20 * ngm + 16;
    if (c->cap_tscr < need) {
        dev_free(c, c->d_tscr);
        c->d_tscr = nullptr;
        c->cap_tscr = 0;
        if (int rc = check_cuda(c, dev_alloc(c, &c->d_tscr, need * sizeof(int)), "tree scratch")) return rc;
        c->cap_tscr = need;
    }
    s->octs = c->d_tscr;
    s->mark = s->octs + ngm;
    s->rank = s->mark + 8 * ngm + 1;
    s->list = s->rank + 8 * ngm + 1;
    s->list2 = s->list + ngm;
    return RG_OK;
}

__global__ void k_set_int(int* dst, int v) { *dst = v; }

// one link write in stream order (a kernel argument, so nothing waits)
int set_dev_int(rg_ctx* c, int* dst, int v) {
    k_set_int<<<1, 1, 0, c->stream>>>(dst, v);
    return check_cuda(c, cudaGetLastError(), "tree link");
}

// ---------------------------------------------------------------- growing the oct arrays
// AmrGrid::resize_grids (AmrGrid.cpp:117-248): cell ncoarse + (ic-1)*ngridmax
// + ig keeps its (ic, ig) under the new ngridmax, so per-cell planes move
// slot by slot; per-oct planes keep their first ngm0 entries; everything new
// is zero; cell ids stored in father and nbor (values above ncoarse) are
// relabelled the same way.
__device__ __forceinline__ int relabel_cell(int id, int ncoarse, int ngm0, int ngm1) {
    if (id <= ncoarse) return id;
    const int r = id - 1 - ncoarse;
    return ncoarse + (r / ngm0) * ngm1 + r % ngm0 + 1;
}

template <class T>
__global__ void k_relocate_cells(const T* __restrict__ src, T* __restrict__ dst, int nplanes, size_t plane0,
                                 size_t plane1, int ncoarse, int ngm0, int ngm1) {
    const size_t n = (size_t)nplanes * plane1, ncell1 = (size_t)ncoarse + 8 * (size_t)ngm1;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t v = i / plane1, j = i - v * plane1;
        T x = T(0);
        if (j < (size_t)ncoarse) {
            x = src[v * plane0 + j];
        } else if (j < ncell1) {
            const size_t r = j - ncoarse, ic = r / ngm1, ig = r - ic * ngm1;
            if (ig < (size_t)ngm0) x = src[v * plane0 + ncoarse + ic * ngm0 + ig];
        }
        dst[i] = x;
    }
}

template <class T>
__global__ void k_relocate_octs(const T* __restrict__ src, T* __restrict__ dst, int nplanes, int ncoarse, int ngm0,
                                int ngm1, bool relabel) {
    const size_t n = (size_t)nplanes * ngm1;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t v = i / ngm1, ig = i - v * ngm1;
        T x = T(0);
        if (ig < (size_t)ngm0) x = src[v * ngm0 + ig];
        if constexpr (sizeof(T) == sizeof(int))
            if (relabel) x = relabel_cell(x, ncoarse, ngm0, ngm1);
        dst[i] = x;
    }
}

// the new octs first..last appended to the free list after `before` (its
// old tail, 0 when it was empty), as resize_grids links them
__global__ void k_link_new_octs(int* next, int* prev, int first, int last, int before) {
    for (int g = first + blockIdx.x * blockDim.x + threadIdx.x; g <= last; g += gridDim.x * blockDim.x) {
        prev[g - 1] = g > first ? g - 1 : before;
        next[g - 1] = g < last ? g + 1 : 0;
        if (g == first && before > 0) next[before - 1] = first;
    }
}

// *p (nplanes planes of plane0 entries) replaced by a relocated copy with
// planes of plane1 entries; cells: per-cell layout, else per-oct
template <class T>
int relocate(rg_ctx* c, T** p, bool cells, int nplanes, size_t plane0, size_t plane1, int ngm0, int ngm1,
             bool relabel, const char* what) {
    T* dst = nullptr;
    const size_t n = (size_t)nplanes * plane1;
    if (dev_alloc(c, &dst, sizeof(T) * n) != cudaSuccess)
        return set_error(c, RG_ERR_NOMEM, std::string("device allocation failed while growing the tree: ") + what);
    if (cells)
        k_relocate_cells<T><<<nblk((long long)n), TPB, 0, c->stream>>>(*p, dst, nplanes, plane0, plane1, c->ncoarse,
                                                                     ngm0, ngm1);
    else
        k_relocate_octs<T><<<nblk((long long)n), TPB, 0, c->stream>>>(*p, dst, nplanes, c->ncoarse, ngm0, ngm1,
                                                                    relabel);
    dev_free(c, *p);
    *p = dst;
    return check_cuda(c, cudaGetLastError(), what);
}

// *p replaced by an uninitialised array of n entries (scratch whose content is rebuilt)
template <class T>
int renew(rg_ctx* c, T** p, size_t n, const char* what) {
    dev_free(c, *p);
    *p = nullptr;
    if (dev_alloc(c, p, sizeof(T) * (n ? n : 1)) != cudaSuccess)
        return set_error(c, RG_ERR_NOMEM, std::string("device allocation failed while growing the tree: ") + what);
    return RG_OK;
}

// Doubles ngridmax until the free list holds `need` octs, as get_free_grid's
// resize_grids(2 * ngridmax) does each time the list runs dry
// (AmrGrid.cpp:259-261).  Growing before the refinement instead of in the
// middle of it gives the same arrays: make_grid_fine recomputes every cell id
// it still holds under the new ngridmax (TreeUpdater.cpp:62-75), the octs it
// takes from the free list are the old entries first and then ngm0+1, ngm0+2,
// ... in both cases, and a taken oct's free-list links are reset either way.
int tree_grow_arrays(rg_ctx* c, int need);

int tree_grow(rg_ctx* c, int need) {
    const int rc = tree_grow_arrays(c, need);
    if (rc != RG_OK && rc != RG_ERR_UNSUPPORTED) {
        // some arrays may already have the new layout and others not: the
        // tree and the state are lost, and every later call says so
        c->tree_resident = false;
        c->have_topology = false;
        c->have_state = false;
        c->tree_dirty = false;
        for (auto& p : c->plans) free_plan(c, p);
    }
    return rc;
}

int tree_grow_arrays(rg_ctx* c, int need) {
    const int ngm0 = c->ngridmax, nc0 = c->ncell, nv = c->nvar;
    long long ngm1 = ngm0, avail = c->numbf;
    while (avail < need) {
        avail += ngm1;
        ngm1 *= 2;
    }
    const long long nc1 = (long long)c->ncoarse + 8 * ngm1;
    if (nc1 + 1 > (long long)INT32_MAX)
        return set_error(c, RG_ERR_UNSUPPORTED, "growing ngridmax to " + std::to_string(ngm1) +
                                                    " would overflow 32-bit cell ids");
    const int g1 = (int)ngm1, n1 = (int)nc1;
    // per-cell state and flags, moved slot by slot
    if (int rc = relocate(c, &c->d_uold, true, nv, nc0, n1, ngm0, g1, false, "uold")) return rc;
    if (int rc = relocate(c, &c->d_unew, true, nv, nc0, n1, ngm0, g1, false, "unew")) return rc;
    if (int rc = relocate(c, &c->d_son, true, 1, (size_t)nc0 + 1, (size_t)n1 + 1, ngm0, g1, false, "son")) return rc;
    if (int rc = relocate(c, &c->d_flag1, true, 1, nc0, n1, ngm0, g1, false, "flag1")) return rc;
    if (int rc = relocate(c, &c->d_flag2, true, 1, nc0, n1, ngm0, g1, false, "flag2")) return rc;
    if (int rc = relocate(c, &c->d_cpu_map, true, 1, nc0, n1, ngm0, g1, false, "cpu_map")) return rc;
    // per-oct links, neighbours and coordinates
    if (int rc = relocate(c, &c->d_father, false, 1, ngm0, g1, ngm0, g1, true, "father")) return rc;
    if (int rc = relocate(c, &c->d_nbor, false, 6, ngm0, g1, ngm0, g1, true, "nbor")) return rc;
    if (int rc = relocate(c, &c->d_next, false, 1, ngm0, g1, ngm0, g1, false, "next")) return rc;
    if (int rc = relocate(c, &c->d_prev, false, 1, ngm0, g1, ngm0, g1, false, "prev")) return rc;
    if (int rc = relocate(c, &c->d_xg, false, 3, ngm0, g1, ngm0, g1, false, "xg")) return rc;
    // scratch sized by the tree, rebuilt by the next refresh or step
    const size_t cell1 = (size_t)n1 + 1;
    int** cell_scr[] = {&c->d_cell_level, &c->d_cpos, &c->d_tmap, &c->d_pmark};
    for (int** p : cell_scr)
        if (int rc = renew(c, p, cell1, "cell scratch")) return rc;
    int** oct_scr[] = {&c->d_jump, &c->d_dist, &c->d_jump2, &c->d_dist2};
    for (int** p : oct_scr)
        if (int rc = renew(c, p, (size_t)g1, "oct scratch")) return rc;
    if (int rc = renew(c, &c->d_prim, (size_t)nv * n1, "primitives")) return rc;
    c->cap_cell = cell1;
    c->cap_grid = (size_t)g1;
    c->cap_state = (size_t)nv * n1;
    // the free list: its old entries in order, then ngm0+1 .. ngm1
    std::vector<int> fq((size_t)g1, 0);
    for (int j = 0; j < c->numbf; ++j) fq[(size_t)j] = c->h_fq[(size_t)((c->fq_head + j) % ngm0)];
    const int before = c->numbf > 0 ? fq[(size_t)c->numbf - 1] : 0;
    for (int g = ngm0 + 1; g <= g1; ++g) fq[(size_t)(c->numbf + g - ngm0 - 1)] = g;
    c->h_fq.swap(fq);
    if (int rc = renew(c, &c->d_fq, (size_t)g1, "free list")) return rc;
    if (int rc = check_cuda(c, cudaMemcpyAsync(c->d_fq, c->h_fq.data(), sizeof(int) * (size_t)g1,
                                               cudaMemcpyHostToDevice, c->stream),
                            "free list upload"))
        return rc;
    k_link_new_octs<<<nblk(g1 - ngm0), TPB, 0, c->stream>>>(c->d_next, c->d_prev, ngm0 + 1, g1, before);
    c->fq_head = 0;
    c->numbf += g1 - ngm0;
    c->ngridmax = g1;
    c->ncell = n1;
    c->next_level = -1;
    c->tree_dirty = true;  // cell ids moved: plans, ranks and cell levels are stale
    c->plans_dirty = c->lists_dirty = ~0ull;
    if (int rc = check_cuda(c, cudaGetLastError(), "tree growth kernels")) return rc;
    // the upload above reads the host ring: keep it alive until the copy is done
    return check_cuda(c, cudaStreamSynchronize(c->stream), "tree growth");
}

}  // namespace

int tree_flag_fine(rg_ctx* c, int ilevel, double ed, double ep, double ev, double eb2, int nexp, int icount,
                   int nsub) {
    if (int rc = check_tree(c, ilevel)) return rc == kNoOp ? RG_OK : rc;  // no-op at and above nlevelmax (TreeUpdater.cpp:329)
    if (eb2 > 0.0) return set_error(c, RG_ERR_UNSUPPORTED, "err_grad_b2 needs MHD variables");
    TreeMut M = tree_mut(c);
    cudaStream_t s = c->stream;
    const int lmin = c->levelmin;
    if (ilevel == 1) {
        // below levelmin every coarse cell ends flagged, and smoothing a fully
        // flagged level changes nothing; refinement criteria on the coarse
        // level itself are not covered here
        if (ilevel >= lmin)
            return set_error(c, RG_ERR_UNSUPPORTED, "coarse-level refinement criteria (levelmin 1) stay on the host");
        k_flag_coarse_below_min<<<nblk(c->ncoarse), TPB, 0, s>>>(M);
        c->auth_dirty = true;
        return check_cuda(c, cudaGetLastError(), "coarse flags");
    }
    TreeScratch S;
    if (int rc = tree_scratch(c, &S)) return rc;
    int noct = 0;
    const int* octs = nullptr;
    if (int rc = level_octs_cached(c, ilevel, &octs, &noct)) return rc;
    if (noct == 0) return RG_OK;
    S.octs = const_cast<int*>(octs);  // read only below
    const int n = 8 * noct;
    auto smooth = [&]() {
        k_smooth_mark<<<nblk(n), TPB, 0, s>>>(M, S.octs, noct, S.mark);
        k_smooth_apply<<<nblk(n), TPB, 0, s>>>(M, S.octs, noct, S.mark);
    };
    k_flag_init<<<nblk(n), TPB, 0, s>>>(M, S.octs, noct, ilevel < lmin ? 1 : 0);
    // below levelmin every cell of the level is now flagged, and smoothing a
    // fully flagged level flags nothing more: the smoothing passes run from
    // levelmin on only
    if (ilevel >= lmin) smooth();
    if (ilevel >= lmin && (ed > 0.0 || ep > 0.0 || ev > 0.0))
        k_flag_grad<<<nblk(n), TPB, 0, s>>>(M, S.octs, noct, ed, ep, ev, c->params.gamma);
    if (ilevel > lmin && icount < nsub) k_test_flag<<<nblk(n), TPB, 0, s>>>(M, S.octs, noct);
    if (ilevel >= lmin)
        for (int i = 0; i < nexp; ++i) smooth();
    if (ilevel > lmin && icount < nsub)
        k_ensure_ref_rules<<<nblk(27LL * noct), TPB, 0, s>>>(M, Geo{c->nx, c->ny, c->nz, c->params.boxlen}, S.octs,
                                                              noct);
    // nothing to read back: the host does not wait here, and a check the
    // kernels failed is reported by the next call that synchronises
    return check_cuda(c, cudaGetLastError(), "flag_fine kernels");
}

int tree_make_grid_fine(rg_ctx* c, int ilevel, int* changed) {
    if (changed) *changed = 0;
    if (int rc = check_tree(c, ilevel)) return rc == kNoOp ? RG_OK : rc;  // no-op at and above nlevelmax (TreeUpdater.cpp:28)
    TreeScratch S;
    if (int rc = tree_scratch(c, &S)) return rc;
    TreeMut M = tree_mut(c);
    cudaStream_t s = c->stream;
    if (c->auth_dirty) {
        k_authorize<<<nblk(c->ncell), TPB, 0, s>>>(M);
        c->auth_dirty = false;
    }
    if (ilevel == 1) {
        int* d_count = S.mark;
        int count = 0;
        cudaMemsetAsync(d_count, 0, sizeof(int), s);
        k_coarse_candidates<<<nblk(c->ncoarse), TPB, 0, s>>>(M, d_count);
        cudaMemcpyAsync(&count, d_count, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (int rc = check_cuda(c, cudaStreamSynchronize(s), "coarse candidates")) return rc;
        if (count > 0) return set_error(c, RG_ERR_UNSUPPORTED, "refining coarse cells stays on the host");
        return RG_OK;
    }
    int noct = 0;
    const int* octs = nullptr;
    if (int rc = level_octs_cached(c, ilevel, &octs, &noct)) return rc;
    if (noct == 0) return check_cuda(c, cudaStreamSynchronize(s), "authorize");
    S.octs = const_cast<int*>(octs);  // read only below
    const int n8 = 8 * noct;
    k_refine_mark<<<nblk(n8), TPB, 0, s>>>(M, S.octs, noct, S.mark);
    int n = 0;
    if (int rc = exclusive_scan(c, S.mark, S.rank, n8, &n)) return rc;
    if (n == 0) return RG_OK;
    if (n > c->numbf) {
        // the free list is too short: grow the arrays as the reference does,
        // then start over on the relabelled tree (authorisation is idempotent)
        if (int rc = tree_grow(c, n)) return rc;
        return tree_make_grid_fine(c, ilevel, changed);
    }
    const StepK K = step_consts(c);
    k_refine<<<nblk(n8), TPB, 0, s>>>(M, tree_view(c), Geo{c->nx, c->ny, c->nz, c->params.boxlen}, S.octs, noct,
                                      S.mark, S.rank, c->d_fq, c->fq_head, ilevel, c->params.interpol_var,
                                      c->params.interpol_type, c->params.gamma, K.smalle, c->d_bound, c->nbound_type,
                                      S.list, c->d_status);
    // the new octs, in order, are the next n entries of the free-list ring
    const int ngm = c->ngridmax, L = ilevel + 1;
    const int first = c->h_fq[(size_t)c->fq_head], last = c->h_fq[(size_t)((c->fq_head + n - 1) % ngm)];
    const int old_tail = c->h_taill[(size_t)hidx(c, L)];
    k_link_chain<<<nblk(n), TPB, 0, s>>>(c->d_next, c->d_prev, S.list, n, old_tail);
    if (old_tail == 0) c->h_headl[(size_t)hidx(c, L)] = first;
    c->h_taill[(size_t)hidx(c, L)] = last;
    c->h_numbl[(size_t)hidx(c, L)] += n;
    c->fq_head = (c->fq_head + n) % ngm;
    c->numbf -= n;
    c->auth_dirty = true;  // the new cells have cpu_map 1 and flag2 0
    if (c->numbf > 0)
        if (int rc = set_dev_int(c, c->d_prev + c->h_fq[(size_t)c->fq_head] - 1, 0)) return rc;
    c->tree_dirty = true;
    // refining level-L cells changes their son links (the plan of level L),
    // adds octs to list L + 1 (its plan and list), and changes which cells
    // exist at level L + 1, hence the neighbour and ghost-stencil cells of
    // levels L + 1 and L + 2; level L - 1 is included as a margin.  The new
    // octs follow list L + 1's old tail in rank order (k_link_chain), so its
    // cached list stays in order with them appended.
    const int L1 = ilevel + 1;
    const int kept = ((int)c->lvl_n.size() > L1) ? c->lvl_n[(size_t)L1] : 0;
    mark_changed(c, ilevel - 1, ilevel + 2, keep_cached_list(c, L1, kept, S.list, n) ? -1 : L1);
    if (changed) *changed = n;
    if (int rc = check_cuda(c, cudaGetLastError(), "make_grid_fine kernels")) return rc;
    return check_device_status(c);
}

int tree_remove_grid_fine(rg_ctx* c, int ilevel, int* changed) {
    if (changed) *changed = 0;
    if (int rc = check_tree(c, ilevel)) return rc == kNoOp ? RG_OK : rc;  // no-op at and above nlevelmax (TreeUpdater.cpp:152)
    TreeScratch S;
    if (int rc = tree_scratch(c, &S)) return rc;
    int noct = 0;
    const int* octs = nullptr;
    if (int rc = level_octs_cached(c, ilevel, &octs, &noct)) return rc;
    if (noct == 0) return RG_OK;
    S.octs = const_cast<int*>(octs);  // read only below
    TreeMut M = tree_mut(c);
    cudaStream_t s = c->stream;
    k_kill_mark<<<nblk(noct), TPB, 0, s>>>(M, S.octs, noct, S.mark);
    int nkill = 0;
    if (int rc = exclusive_scan(c, S.mark, S.rank, noct, &nkill)) return rc;
    if (nkill == 0) return RG_OK;
    const int ngm = c->ngridmax, m = noct - nkill;
    const int fq_tail = (c->fq_head + c->numbf) % ngm;
    const int old_tailf = c->numbf > 0 ? c->h_fq[(size_t)((fq_tail - 1 + ngm) % ngm)] : 0;
    k_kill<<<nblk(noct), TPB, 0, s>>>(M, S.octs, noct, S.mark, S.rank, S.list, S.list2, c->d_fq, fq_tail);
    c->auth_dirty = true;  // the freed cells have cpu_map 1 and flag2 0
    k_link_chain<<<nblk(std::max(m, 1)), TPB, 0, s>>>(c->d_next, c->d_prev, S.list, m, 0);
    k_link_chain<<<nblk(nkill), TPB, 0, s>>>(c->d_next, c->d_prev, S.list2, nkill, old_tailf);
    std::vector<int> freed((size_t)nkill);
    int ends[2] = {0, 0};
    cudaMemcpyAsync(freed.data(), S.list2, sizeof(int) * nkill, cudaMemcpyDeviceToHost, s);
    if (m > 0) {
        cudaMemcpyAsync(&ends[0], S.list, sizeof(int), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&ends[1], S.list + m - 1, sizeof(int), cudaMemcpyDeviceToHost, s);
    }
    if (int rc = check_cuda(c, cudaStreamSynchronize(s), "remove_grid_fine")) return rc;
    for (int j = 0; j < nkill; ++j) c->h_fq[(size_t)((fq_tail + j) % ngm)] = freed[(size_t)j];
    c->numbf += nkill;
    c->h_headl[(size_t)hidx(c, ilevel)] = ends[0];
    c->h_taill[(size_t)hidx(c, ilevel)] = ends[1];
    c->h_numbl[(size_t)hidx(c, ilevel)] -= nkill;
    c->tree_dirty = true;
    // removing level-L octs changes list L (its plan and list), the son links
    // of their fathers (the plan of level L - 1) and the ghost-stencil cells of
    // level L + 1; level L - 2 is included as a margin.  The kept octs, in
    // list order (k_kill), are the level's list now.
    mark_changed(c, ilevel - 2, ilevel + 1, keep_cached_list(c, ilevel, 0, S.list, m) ? -1 : ilevel);
    if (changed) *changed = nkill;
    if (int rc = check_cuda(c, cudaGetLastError(), "remove_grid_fine kernels")) return rc;
    return check_device_status(c);
}

int tree_changes_pending(rg_ctx* c, uint64_t levels, TreeChanges* out) {
    *out = TreeChanges{};
    if (!c->tree_resident) return set_error(c, RG_ERR_STATE, "no device-resident tree: call rg_tree_attach first");
    levels &= level_bits(1, c->nlevelmax - 1);  // both operations are no-ops at and above nlevelmax
    // the results are 32-bit masks: levels from 32 on stay "may change"
    const uint64_t probed = levels & level_bits(1, 31);
    // a level whose every cell has a son has no candidate of either kind (a
    // refinement needs a cell without a son, a removal an oct without a
    // refined cell); the host's counts show it, since every oct has one father
    // cell: list L + 1 holds 8 octs per oct of list L (per coarse cell for
    // L = 1, whose cells are the coarse cells)
    uint64_t scan = 0;
    for (int L = 1; L <= 31; ++L) {
        if (!(probed & (1ull << L))) continue;
        const long long cells = L == 1 ? c->ncoarse : 8LL * c->h_numbl[(size_t)hidx(c, L)];
        const bool full = L + 1 <= c->nlevelmax && c->h_numbl[(size_t)hidx(c, L + 1)] == cells;
        if (!full) scan |= 1ull << L;
    }
    if (scan == 0) {
        out->refine &= ~probed;
        out->kill &= ~probed;
        out->kill |= probed & 2ull;  // remove_grid_fine(1) is not probed
        return RG_OK;
    }
    c->next_level = -1;
    if (int rc = refresh_tree(c)) return rc;
    TreeScratch S;
    if (int rc = tree_scratch(c, &S)) return rc;
    cudaStream_t s = c->stream;
    TreeMut M = tree_mut(c);
    if (c->auth_dirty) {  // what the first make_grid_fine of the range does first
        k_authorize<<<nblk(c->ncell), TPB, 0, s>>>(M);
        c->auth_dirty = false;
    }
    // [refine bits, kill bits, coarse candidates]
    unsigned* d_bits = reinterpret_cast<unsigned*>(S.list);
    cudaMemsetAsync(d_bits, 0, 3 * sizeof(unsigned), s);
    // make_grid_fine(1)'s test: a coarse cell flagged and authorised without a son
    if (scan & 2ull) k_coarse_candidates<<<nblk(c->ncoarse), TPB, 0, s>>>(M, reinterpret_cast<int*>(d_bits + 2));
    for (int L = 2; L <= 31; ++L) {
        if (!(scan & (1ull << L))) continue;
        const int* octs = nullptr;
        int noct = 0;
        if (int rc = level_octs_cached(c, L, &octs, &noct)) return rc;
        if (noct > 0) k_change_probe<<<nblk(noct), TPB, 0, s>>>(M, octs, noct, d_bits, 1u << L);
    }
    unsigned h[3] = {~0u, ~0u, 1u};
    if (int rc = check_cuda(c, cudaMemcpyAsync(h, d_bits, sizeof(h), cudaMemcpyDeviceToHost, s), "change probe"))
        return rc;
    if (int rc = check_cuda(c, cudaStreamSynchronize(s), "change probe")) return rc;
    uint64_t refine = h[0], kill = h[1];
    if (h[2] != 0) refine |= 2ull;
    kill |= 2ull;  // remove_grid_fine(1) is not probed
    out->refine = (out->refine & ~probed) | (refine & probed);
    out->kill = (out->kill & ~probed) | (kill & probed);
    return RG_OK;
}

int tree_restrict_fine(rg_ctx* c, int ilevel) {
    // restrict_fine(ilevel) reads level ilevel + 1; the reference walks an
    // empty list when ilevel + 1 > nlevelmax
    if (!c->tree_resident) return set_error(c, RG_ERR_STATE, "no device-resident tree: call rg_tree_attach first");
    if (ilevel < 0 || ilevel > c->nlevelmax) return set_error(c, RG_ERR_ARG, "level outside 0..nlevelmax");
    c->next_level = -1;
    if (ilevel + 1 > c->nlevelmax) return RG_OK;
    if (int rc = refresh_tree(c)) return rc;
    TreeScratch S;
    if (int rc = tree_scratch(c, &S)) return rc;
    int noct = 0;
    const int* octs = nullptr;
    if (int rc = level_octs_cached(c, ilevel + 1, &octs, &noct)) return rc;
    if (noct == 0) return RG_OK;
    S.octs = const_cast<int*>(octs);  // read only below
    k_restrict<<<nblk(noct), TPB, 0, c->stream>>>(tree_mut(c), S.octs, noct);
    return check_cuda(c, cudaGetLastError(), "restrict_fine kernel");
}

// The tail of the coarse step below levelmin: flag_fine(il) for il =
// levelmin-1..1 and restrict_fine(il) for il = levelmin-1..0 (the
// restrictions when `restrictions` is set), as the calls one by one leave the
// tree and the state, in a few launches (k_tail_flags_restrict, k_restrict
// for the larger lists, k_tail_cascade for the small ones).
// *done stays false (nothing issued) when the lists below levelmin are not
// small or not cached, and the caller makes the calls one by one.  Enqueue
// only.
int tree_tail_below_min(rg_ctx* c, int lmin, bool restrictions, bool* done) {
    *done = false;
    if (!c->tree_resident || c->tree_dirty || lmin < 2 || lmin > c->nlevelmax || lmin > 32 || c->levelmin != lmin)
        return RG_OK;
    for (int L = 1; L <= lmin; ++L)
        if ((int)c->lvl_ver.size() <= L || (c->lvl_ver[(size_t)L] != c->topo_version && c->h_numbl[(size_t)hidx(c, L)] > 0))
            return RG_OK;
    // lists below levelmin beyond a few thousand octs: call by call
    long long below = 0;
    for (int L = 1; L <= lmin - 1; ++L) below += c->h_numbl[(size_t)hidx(c, L)];
    if (below > 65536) return RG_OK;
    LevelLists F{}, R{};
    for (int L = lmin - 1; L >= 2; --L) {
        const int* octs = nullptr;
        int noct = 0;
        if (int rc = level_octs_cached(c, L, &octs, &noct)) return rc;
        F.octs[F.n] = octs;
        F.noct[F.n++] = noct;
    }
    // lists with more octs than the cascade's block takes in a few rounds get
    // their own launch (those come first: the lists grow with the level)
    const int* big[32];
    int nbig[32], nb = 0;
    if (restrictions)
        for (int L = lmin - 1; L >= 1; --L) {
            const int* octs = nullptr;
            int noct = 0;
            if (int rc = level_octs_cached(c, L, &octs, &noct)) return rc;
            if (R.n == 0 && noct > 2048) {
                big[nb] = octs;
                nbig[nb++] = noct;
                continue;
            }
            R.octs[R.n] = octs;
            R.noct[R.n++] = noct;
        }
    const int* top = nullptr;
    int ntop = 0;
    if (restrictions)
        if (int rc = level_octs_cached(c, lmin, &top, &ntop)) return rc;
    long long nflag = c->ncoarse;
    for (int j = 0; j < F.n; ++j) nflag += 8LL * F.noct[j];
    c->next_level = -1;
    TreeMut M = tree_mut(c);
    const int nb_r = ntop > 0 ? nblk(ntop) : 0;
    k_tail_flags_restrict<<<nb_r + nblk(nflag), TPB, 0, c->stream>>>(M, top, ntop, nb_r, F);
    for (int i = 0; i < nb; ++i) k_restrict<<<nblk(nbig[i]), TPB, 0, c->stream>>>(M, big[i], nbig[i]);
    if (R.n > 0) k_tail_cascade<<<1, 1024, 0, c->stream>>>(M, R);
    c->auth_dirty = true;  // k_flag_coarse_below_min's part: the coarse cells' cpu_map
    *done = true;
    return check_cuda(c, cudaGetLastError(), "tail below levelmin");
}

}  // namespace rg
