// rg_face.cuh -- device helpers of the face step shared by the face kernels.
//
// Face states and fluxes of HydroSolver::godunov_fine (RAMSES-CPP
// src/solvers/hydro/HydroSolver.cpp:93-474) on rotated primitive states: the
// cell's own MUSCL-Hancock trace (compute_slopes + trace, :653-732), the
// neighbour's face state by the ghost (:162-453), same-level (:148-161) or
// boundary (:130-145) branch, and the Riemann solver selected at :456-461.
#pragma once

#include "rg_internal.cuh"
#include "rg_mlp.cuh"
#include "rg_physics.cuh"

namespace rg {

struct StepK {
    double gamma, smalle, smallp;
    int slope_type, interpol_type, interpol_var, exact_niter;
    double exact_tol;
    const float* mlp;  // learned Newton start of the exact solver, or nullptr
};

__device__ __forceinline__ int cell_of(const TreeView& T, const PlanView& P, int p) {
    if (P.level0) return p + 1;
    int icx = p / P.noct, k = p - icx * P.noct;
    return T.ncoarse + icx * T.ngridmax + P.octs[k];
}

// Primitive state of cell id, rotated so the velocity along idim sits at 1.
template <int NDIM>
__device__ __forceinline__ void load_rot(const double* __restrict__ prim, size_t ncell, int id, int idim, double* q) {
    constexpr int NV = Dims<NDIM>::NV;
    const double* b = prim + (size_t)(id - 1);
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) q[iv] = __ldg(b + iv * ncell);
    rot_swap<NDIM>(q, idim);
}

// Neighbour primitive for a slope stencil: the cell's own state when the
// neighbour id is <= 0, with the normal velocity flipped for a reflecting
// boundary entry (HydroSolver.cpp:661-664, 194-204).
template <int NDIM>
__device__ __forceinline__ void load_nb_rot(const TreeView& T, const double* __restrict__ prim, size_t ncell, int id,
                                            int idim, const double* qself, double* q) {
    constexpr int NV = Dims<NDIM>::NV;
    if (id > 0) {
        load_rot<NDIM>(prim, ncell, id, idim, q);
        return;
    }
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) q[iv] = qself[iv];
    int ib = -id;
    if (ib > 0 && ib <= T.nbound_type && T.bound_type[ib - 1] == 1) q[1] *= -1.0;
}

// Own trace (compute_slopes + trace, HydroSolver.cpp:653-732) on rotated data.
template <int NDIM>
__device__ __forceinline__ void own_trace(const double* qc, const double* ql, const double* qr, double dt,
                                          const DxDiv& D, const StepK& K, double* qm, double* qp) {
    constexpr int NV = Dims<NDIM>::NV;
    double dq[NV];
    double nu = D.div(qc[1] * dt);
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
        if (K.slope_type == 0) dq[iv] = 0.0;
        else if ((K.slope_type == 5 || K.slope_type == 6) && iv != 0) dq[iv] = 0.0;
        else dq[iv] = D.div(compute_slope(ql[iv], qc[iv], qr[iv], K.slope_type, 1.5, nu));
    }
    trace<NDIM>(qc, dq, dt, D.dx, qm, qp, K.gamma);
}

// Ghost trace of a coarser (or same-level) neighbour, 2D/3D form
// (HydroSolver.cpp:357-440): interpolation slopes over 2dx.
template <int NDIM>
__device__ __forceinline__ void ghost_trace(const double* qc, const double* ql, const double* qr, double dt,
                                            const DxDiv& D, const StepK& K, double* qm, double* qp) {
    constexpr int NV = Dims<NDIM>::NV;
    double dq[NV];
    const DxDiv Dc{2.0 * D.dx, 0.5 * D.inv, D.pow2};  // dx_coarse = 2 dx, still a power of two
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
        double dlft = qc[iv] - ql[iv];
        double drgt = qr[iv] - qc[iv];
        double slope = 0.0;
        if (K.interpol_type > 0 && dlft * drgt > 0.0) slope = interp_slope(dlft, drgt, K.interpol_type);
        dq[iv] = Dc.div(slope);
    }
    trace<NDIM>(qc, dq, dt, Dc.dx, qm, qp, K.gamma);
}

// Ghost face state of the 1D build (HydroSolver.cpp:219-356): the coarse
// neighbour's child states, then a slope_type slope against the active cell.
__device__ __forceinline__ void ghost_1d(const double* __restrict__ uold, size_t ncell, const TreeView& T, int n, int nl, int nr,
                         int side, const double* q_act, double dt, const DxDiv& D, const StepK& K, double* qm,
                         double* qp) {
    constexpr int NV = 3;
    double uc[NV], ul[NV], ur[NV];
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) uc[iv] = uold[(size_t)iv * ncell + n - 1];
    for (int k = 0; k < 2; ++k) {
        int id = k ? nr : nl;
        double* uo = k ? ur : ul;
        if (id > 0) {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) uo[iv] = uold[(size_t)iv * ncell + id - 1];
        } else {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) uo[iv] = uc[iv];
            int ib = -id;
            if (ib > 0 && ib <= T.nbound_type && T.bound_type[ib - 1] == 1) uo[1] *= -1.0;
        }
    }
    const double gamma = K.gamma;
    const int ivar = K.interpol_var, itp = K.interpol_type;
    double q1[3][NV];
    const double* us[3] = {ul, uc, ur};
    for (int k = 0; k < 3; ++k) {
        const double* u = us[k];
        double* q = q1[k];
        if (ivar == 0) {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) q[iv] = u[iv];
        } else if (ivar == 1) {
            double d = smax(u[0], 1e-10);
            q[0] = u[0];
            q[1] = 0.0;
            double e_kin = 0.5 * u[1] * u[1] / d;
            q[2] = u[2] - e_kin - 0.0;
        } else {
            ctoprim<1>(u, q, gamma, K.smalle);
        }
    }
    double slopes[NV];
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
        slopes[iv] = 0.0;
        double dlft = q1[1][iv] - q1[0][iv];
        double drgt = q1[2][iv] - q1[1][iv];
        if (dlft * drgt > 0.0) {
            int itype = itp;
            if (itp == 4) itype = (ivar == 2 && iv == 1) ? 3 : 2;
            if (itype >= 1 && itype <= 3) slopes[iv] = interp_slope(dlft, drgt, itype);
        }
    }
    double uch[2][NV];
    for (int k = 0; k < 2; ++k) {
        double q2[NV];
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) q2[iv] = k ? q1[1][iv] + 0.5 * slopes[iv] : q1[1][iv] - 0.5 * slopes[iv];
        double* u = uch[k];
        if (ivar == 0) {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) u[iv] = q2[iv];
        } else if (ivar == 1) {
            double d = smax(q2[0], 1e-10);
            u[0] = d;
            u[1] = 0.0;
            double e_kin = 0.5 * q2[1] * q2[1] / d;
            u[2] = q2[2] + e_kin + 0.0;
        } else {
            double d = smax(q2[0], 1e-10);
            u[0] = d;
            u[1] = 0.0;
            double e_kin = 0.5 * d * q2[1] * q2[1];
            u[2] = q2[2] / (gamma - 1.0) + e_kin + 0.0;
        }
    }
    double qg2[NV], qg[NV];
    ctoprim<1>(uch[side == 0 ? 0 : 1], qg2, gamma, K.smalle);
    ctoprim<1>(uch[side == 0 ? 1 : 0], qg, gamma, K.smalle);
    double dq[NV];
    double nu = D.div(qg[1] * dt);
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
        double dlft, drgt;
        if (side == 0) {
            dlft = qg[iv] - qg2[iv];
            drgt = q_act[iv] - qg[iv];
        } else {
            dlft = qg[iv] - q_act[iv];
            drgt = qg2[iv] - qg[iv];
        }
        if ((K.slope_type == 5 || K.slope_type == 6) && iv != 0) dq[iv] = 0.0;
        else dq[iv] = D.div(compute_slope(qg[iv] - dlft, qg[iv], qg[iv] + drgt, K.slope_type, 1.5, nu));
    }
    trace<1>(qg, dq, dt, D.dx, qm, qp, gamma);
}

// Step values of the box of level cell p (ensemble levels).
__device__ __forceinline__ void step_of_box(const PlanView& P, int p, double& dt, DxDiv& D) {
    const BoxStep& B = P.boxes[box_of(P, p)];
    dt = B.dt;
    D = DxDiv{B.dx, B.inv_dx, B.dx_pow2 != 0};
}

template <int NDIM, int RS>
__device__ __forceinline__ int riemann(const double* ql, const double* qr, double* f, const StepK& K) {
    if constexpr (RS == RG_RIEMANN_HLLC) solve_hllc<NDIM>(ql, qr, f, K.gamma, K.smallp);
    else if constexpr (RS == RG_RIEMANN_HLL) solve_hll<NDIM>(ql, qr, f, K.gamma);
    else if constexpr (RS == RG_RIEMANN_ACOUSTIC) solve_acoustic<NDIM>(ql, qr, f, K.gamma, K.smallp);
    else if constexpr (RS == RG_RIEMANN_EXACT)
        return solve_exact<NDIM>(ql, qr, f, K.gamma, K.smallp, K.exact_niter, K.exact_tol,
                                 mlp_guess<NDIM>(K.mlp, ql, qr, K.gamma, K.smallp));
    else solve_llf<NDIM>(ql, qr, f, K.gamma);
    return 0;
}

// Face state of the neighbour across slot (idim, side), rotated.  Writes the
// state the Riemann problem needs: the neighbour's right-face state (qm) for
// side 0, its left-face state (qp) for side 1.  qside, if not null, is the
// rotated primitive state of neighbour cell n already in registers (the own
// trace's stencil cell on that side); otherwise it is loaded here.
// LEVEL0: 1 the plan is level 0's, 0 it is not, -1 read P.level0
template <int NDIM, int LEVEL0 = -1>
__device__ __forceinline__ void neighbour_face(const TreeView& T, const PlanView& P, const double* __restrict__ prim,
                                               const double* __restrict__ uold, size_t ncell, int p, int c, int idim,
                                               int side, int kd, int n, const double* qc, const double* qside,
                                               double dt, const DxDiv& D, const StepK& K, double* qf) {
    constexpr int NV = Dims<NDIM>::NV;
    double qm[NV], qp[NV];
    int kind = kd & KIND_MASK;
    int s = 2 * idim + side;
    if (kind == K_BOUND) {
        double qb[NV], dq0[NV];
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) {
            qb[iv] = qc[iv];
            dq0[iv] = 0.0;
        }
        if (kd & KIND_REFLECT) qb[1] *= -1.0;
        trace<NDIM>(qb, dq0, dt, D.dx, qm, qp, K.gamma);
    } else {
        if (LEVEL0 == 1 || (LEVEL0 < 0 && P.level0)) {
            // level 0 traces are unrotated first-order states (HydroSolver.cpp:77-91)
            double qn[NV], dq0[NV], qmn[NV], qpn[NV];
            load_rot<NDIM>(prim, ncell, n, 0, qn);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) dq0[iv] = 0.0;
            trace<NDIM>(qn, dq0, dt, D.dx, qmn, qpn, K.gamma);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) {
                qm[iv] = qmn[iv];
                qp[iv] = qpn[iv];
            }
            rot_swap<NDIM>(qm, idim);
            rot_swap<NDIM>(qp, idim);
        } else {
            int nl = P.stc[((size_t)s * 2 + 0) * P.ncells + p];
            int nr = P.stc[((size_t)s * 2 + 1) * P.ncells + p];
            if constexpr (NDIM == 1) {
                if (kind == K_GHOST) {
                    ghost_1d(uold, ncell, T, n, nl, nr, side, qc, dt, D, K, qm, qp);
                    goto have_face;
                }
            }
            {
                // the neighbour's state is the own trace's stencil cell on this
                // side (qside, already loaded), and on a same-level face the
                // neighbour's stencil cell towards this cell is the cell itself
                double qnl[NV], qnr[NV], qload[NV];
                const double* qn = qside;
                if (!qn) {
                    load_rot<NDIM>(prim, ncell, n, idim, qload);
                    qn = qload;
                }
                if (side == 0 && nr == c) {
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) qnr[iv] = qc[iv];
                } else {
                    load_nb_rot<NDIM>(T, prim, ncell, nr, idim, qn, qnr);
                }
                if (side == 1 && nl == c) {
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) qnl[iv] = qc[iv];
                } else {
                    load_nb_rot<NDIM>(T, prim, ncell, nl, idim, qn, qnl);
                }
                if (kind == K_GHOST) ghost_trace<NDIM>(qn, qnl, qnr, dt, D, K, qm, qp);
                else own_trace<NDIM>(qn, qnl, qnr, dt, D, K, qm, qp);
            }
        have_face:;
        }
    }
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) qf[iv] = side == 0 ? qm[iv] : qp[iv];
}

// The persistent tiled face kernel.  Work unit: a tile of 32 consecutive
// level cells (one warp wide).  A block holds R tiles x ndim directions, one
// warp per (tile, direction): the warp computes, for its 32 cells, the own
// trace along the direction, the two neighbour face states and the two Riemann
// fluxes (HydroSolver.cpp:93-474).  The fluxes go to global memory (the
// neighbours' reflux events read them) and to shared memory, where the
// direction-0 warp then forms each cell's own flux sum in the reference's
// (idim, side) order (HydroSolver.cpp:485-486), so the fold reads 5 doubles
// for the own update instead of 2*ndim*5.  Blocks are persistent: a grid sized
// from the occupancy of the chosen variant pulls batches of tiles from a
// counter in device memory; the last block to finish resets the counter for
// the next launch (nothing ever waits on another block).
constexpr int TILE = 32;

// LEVEL0: instantiated for level 0 (the coarse cells, first-order traces) or
// for the other levels, so neither instance carries the other's code
template <int NDIM, int RS, int R, int MINB, bool BOXED, bool LEVEL0 = false>
__global__ void __launch_bounds__(TILE * NDIM * R, MINB)
    k_face_tiles(TreeView T, PlanView P, const double* __restrict__ prim, const double* __restrict__ uold,
                 double* __restrict__ flux, double* __restrict__ fsum, DevStatus* st, StepK K, int batch) {
    constexpr int NV = Dims<NDIM>::NV, NS = Dims<NDIM>::NS;
    __shared__ double sf[R][NS][NV][TILE];
    __shared__ int s_base;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = warp / NDIM, idim = warp - r * NDIM;
    const size_t ncell = (size_t)T.ncell;
    const int nc = P.ncells;
    const int ntiles = (nc + TILE - 1) / TILE;
    const double dt0 = st->dt;
    const DxDiv D0{st->dx, st->inv_dx, st->dx_pow2 != 0};
    unsigned long long iters = 0, calls = 0;
    for (;;) {
        if (threadIdx.x == 0) s_base = (int)atomicAdd(&st->face_next, (unsigned)(batch * R));
        __syncthreads();
        const int base = s_base;
        __syncthreads();
        if (base >= ntiles) break;
        const int end = min(base + batch * R, ntiles);
        for (int t0 = base; t0 < end; t0 += R) {
            const int tile = t0 + r;
            const int p = tile * TILE + lane;
            const bool valid = tile < end && p < nc;
            int kd0 = K_NONE;
            if (valid) {
                const int s0 = 2 * idim;
                kd0 = P.kind[(size_t)s0 * nc + p];
                if (kd0 != K_NONE) {
                    const int kd1 = P.kind[(size_t)(s0 + 1) * nc + p];
                    const int c = cell_of(T, P, p);
                    double dt = dt0;
                    DxDiv D = D0;
                    if constexpr (BOXED) step_of_box(P, p, dt, D);
                    double qc[NV], qmo[NV], qpo[NV];
                    load_rot<NDIM>(prim, ncell, c, idim, qc);
                    if constexpr (LEVEL0) {
                        double qn[NV], dq0[NV];
                        load_rot<NDIM>(prim, ncell, c, 0, qn);
#pragma unroll
                        for (int iv = 0; iv < NV; ++iv) dq0[iv] = 0.0;
                        trace<NDIM>(qn, dq0, dt, D.dx, qmo, qpo, K.gamma);
                        rot_swap<NDIM>(qmo, idim);
                        rot_swap<NDIM>(qpo, idim);
                    } else {
                        const int l = P.icn[(size_t)s0 * nc + p], rr = P.icn[(size_t)(s0 + 1) * nc + p];
                        double ql[NV], qr[NV];
                        load_nb_rot<NDIM>(T, prim, ncell, l, idim, qc, ql);
                        load_nb_rot<NDIM>(T, prim, ncell, rr, idim, qc, qr);
                        own_trace<NDIM>(qc, ql, qr, dt, D, K, qmo, qpo);
                    }
#pragma unroll
                    for (int side = 0; side < 2; ++side) {
                        const int kd = side ? kd1 : kd0;
                        const int s = s0 + side;
                        double f[NV];
                        if ((kd & KIND_MASK) == K_ZERO) {
#pragma unroll
                            for (int iv = 0; iv < NV; ++iv) f[iv] = 0.0;
                        } else {
                            const int n = P.icn[(size_t)s * nc + p];
                            double qf[NV];
                            neighbour_face<NDIM, LEVEL0 ? 1 : 0>(T, P, prim, uold, ncell, p, c, idim, side, kd, n, qc, nullptr,
                                                 dt, D, K, qf);
                            if (side == 0) iters += riemann<NDIM, RS>(qf, qpo, f, K);
                            else iters += riemann<NDIM, RS>(qmo, qf, f, K);
                            ++calls;
                            rot_swap<NDIM>(f, idim);
                        }
#pragma unroll
                        for (int iv = 0; iv < NV; ++iv) {
                            flux[((size_t)s * NV + iv) * nc + p] = f[iv];
                            sf[r][s][iv][lane] = f[iv];
                        }
                    }
                }
            }
            __syncthreads();
            if (idim == 0 && valid && kd0 != K_NONE) {
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) {
                    double fs = 0.0;
#pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        const double sign = (s & 1) ? -1.0 : 1.0;
                        fs = fs + sign * sf[r][s][iv][lane];
                    }
                    fsum[(size_t)iv * nc + p] = fs;
                }
            }
            __syncthreads();
        }
    }
    if (RS == RG_RIEMANN_EXACT) {
        for (int o = 16; o > 0; o >>= 1) {
            iters += __shfl_xor_sync(0xffffffffu, iters, o);
            calls += __shfl_xor_sync(0xffffffffu, calls, o);
        }
        if (lane == 0 && calls) {
            atomicAdd(&st->exact_iters, iters);
            atomicAdd(&st->exact_calls, calls);
        }
    }
    // the last block out resets the work counter for the next launch
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&st->face_done, 1u) == gridDim.x - 1) {
            st->face_next = 0;
            st->face_done = 0;
            __threadfence();
        }
    }
}

// Variant table: tiles per block (R) and the launch-bounds minimum of
// resident blocks (caps registers per thread).  Index = variant id.  Ids
// kFirstPipeVariant.. select the software-pipelined kernel (rg_face_pipe.cuh)
// with launch-bounds minimum 4 and 3 (levels above level 0 in 2D/3D builds;
// elsewhere they fall back to the default variant); ids 9 and 10 the brick
// kernel (launch-bounds minimum 3 and 2) on levels that form one complete
// periodic lattice, the default variant elsewhere.
#define RG_FACE_VARIANTS(X) X(0, 1, 6) X(1, 1, 8) X(2, 1, 10) X(3, 1, 9) X(4, 2, 4) X(5, 2, 5) X(6, 2, 6)
constexpr int kFirstPipeVariant = 7;
constexpr int kFirstBrickVariant = 9;  // 9, 10: brick kernel (rg_face_brick.cuh), lattice levels only
constexpr int kNumFaceVariants = 11;
constexpr int kDefaultFaceVariant = 1;
// Ensemble levels (per-box dt and dx read per cell) instantiate only the
// default tiled shape, this one, and the first pipelined variant; every other
// id runs the default shape there.
constexpr int kBoxedAltVariant = 4;
inline bool boxed_variant_distinct(int v) {
    return v == kDefaultFaceVariant || v == kBoxedAltVariant || v == kFirstPipeVariant || v == kFirstBrickVariant;
}

template <int NDIM, int RS, int R, int MINB, bool BOXED = false, bool LEVEL0 = false>
int launch_face_one(rg_ctx* c, const Plan& P, const StepK& K, int batch, const double* uold, const double* prim,
                    double* flux, double* fsum) {
    auto kern = k_face_tiles<NDIM, RS, R, MINB, BOXED, LEVEL0>;
    const int block = TILE * NDIM * R;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
    per_sm = per_sm > 1 ? per_sm : 1;
    const int ntiles = (P.ncells + TILE - 1) / TILE;
    const int grabs = (ntiles + batch * R - 1) / (batch * R);
    int grid = per_sm * c->sm_count;
    if (grabs < grid) grid = grabs;
    if (grid < 1) grid = 1;
    kern<<<grid, block, 0, c->stream>>>(tree_view(c), P.view(), prim, uold, flux, fsum, c->d_status, K, batch);
    return check_cuda(c, cudaGetLastError(), "face kernel");
}

template <int NDIM, int RS>
int launch_face_rs(rg_ctx* c, const Plan& P, const StepK& K, int variant, int batch, const double* uold,
                   const double* prim, double* flux, double* fsum) {
    // level 0 (coarse cells): the default shape only
    if (P.level0) return launch_face_one<NDIM, RS, 1, 8, false, true>(c, P, K, batch, uold, prim, flux, fsum);
    if (P.nbox > 0) {
        // ensemble levels (per-box dt and dx): two shapes are instantiated
        if (variant == kBoxedAltVariant) return launch_face_one<NDIM, RS, 2, 4, true>(c, P, K, batch, uold, prim, flux, fsum);
        return launch_face_one<NDIM, RS, 1, 8, true>(c, P, K, batch, uold, prim, flux, fsum);
    }
#define RG_FACE_CASE(id, r, mb) \
    case id: return launch_face_one<NDIM, RS, r, mb>(c, P, K, batch, uold, prim, flux, fsum);
    switch (variant) {
        RG_FACE_VARIANTS(RG_FACE_CASE)
        default: return launch_face_one<NDIM, RS, 1, 8>(c, P, K, batch, uold, prim, flux, fsum);
    }
#undef RG_FACE_CASE
}

template <int NDIM>
int launch_face_nd(rg_ctx* c, const Plan& P, const StepK& K, int variant, int batch, const double* uold,
                   const double* prim, double* flux, double* fsum) {
    switch (c->params.riemann) {
        case RG_RIEMANN_HLLC: return launch_face_rs<NDIM, RG_RIEMANN_HLLC>(c, P, K, variant, batch, uold, prim, flux, fsum);
        case RG_RIEMANN_HLL: return launch_face_rs<NDIM, RG_RIEMANN_HLL>(c, P, K, variant, batch, uold, prim, flux, fsum);
        case RG_RIEMANN_EXACT: return launch_face_rs<NDIM, RG_RIEMANN_EXACT>(c, P, K, variant, batch, uold, prim, flux, fsum);
        case RG_RIEMANN_ACOUSTIC:
            return launch_face_rs<NDIM, RG_RIEMANN_ACOUSTIC>(c, P, K, variant, batch, uold, prim, flux, fsum);
        default: return launch_face_rs<NDIM, RG_RIEMANN_LLF>(c, P, K, variant, batch, uold, prim, flux, fsum);
    }
}

// instantiated in rg_face_1d.cu / rg_face_3d.cu (compiled in parallel)
int launch_face_nd1(rg_ctx* c, const Plan& P, const StepK& K, int variant, int batch, const double* uold,
                    const double* prim, double* flux, double* fsum);
int launch_face_nd3(rg_ctx* c, const Plan& P, const StepK& K, int variant, int batch, const double* uold,
                    const double* prim, double* flux, double* fsum);

StepK step_consts(const rg_ctx* c);
int launch_face_tiles(rg_ctx* c, const Plan& P, const StepK& K, const double* uold, const double* prim,
                      double* flux, double* fsum);
int autotune_face(rg_ctx* c, Plan& P, const StepK& K);

}  // namespace rg
