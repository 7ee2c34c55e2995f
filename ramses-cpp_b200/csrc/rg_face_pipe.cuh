// rg_face_pipe.cuh -- software-pipelined face kernel for levels above level 0
// in 2D/3D builds.
//
// Same arithmetic and the same outputs as k_face_tiles (rg_face.cuh): per
// (cell, direction) the own MUSCL-Hancock trace, the two neighbour face
// states and the two Riemann fluxes of HydroSolver::godunov_fine (RAMSES-CPP
// src/solvers/hydro/HydroSolver.cpp:93-474), the fluxes to global memory and
// the cell's own flux sum in the reference's (idim, side) order.
//
// What differs is how the stencil reaches the arithmetic.  The tiled kernel
// loads each stencil cell into registers when it needs it, so a warp waits on
// two chains of dependent gathers (plan index -> primitive) per tile and the
// SM, at the occupancy its registers allow, is mostly stalled on memory.
// Here each lane gathers the primitives of the NEXT tile's five stencil cells
// -- the cell, its two neighbours along the direction and the neighbours' far
// stencil cells -- into shared memory with cp.async while it computes the
// current tile, and the plan indices of the tile after that into registers.
// The copies need no registers, so the kernel runs without spills at four
// blocks per SM and its gathers are in flight a whole tile ahead.
//
// Tiles are assigned round-robin (tile = block + k * grid): every tile costs
// the same, and the pipeline must know its next tile in advance.  The
// neighbour's inner stencil cell is the cell itself on every same-level face;
// on a coarse-fine face it is another cell and is loaded directly (rare).
#pragma once

#include "rg_face.cuh"

namespace rg {

constexpr int PIPE_SLOTS = 5;  // cell, left, right, left neighbour's left, right neighbour's right

struct PipeIdx {
    int kd0, kd1, c, l, r, nl0, nr0, nl1, nr1;
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Plan indices of (tile, lane, idim); kd0 = K_NONE outside the level.  All
// loads are independent of each other (no load waits on another).
__device__ __forceinline__ PipeIdx pipe_idx(const TreeView& T, const PlanView& P, int tile, int ntiles, int lane,
                                            int idim) {
    PipeIdx I{K_NONE, K_NONE, 0, 0, 0, 0, 0, 0, 0};
    const int nc = P.ncells, p = tile * TILE + lane;
    if (tile < ntiles && p < nc) {
        const size_t s0 = 2 * (size_t)idim, n = (size_t)nc;
        I.kd0 = P.kind[s0 * n + p];
        I.kd1 = P.kind[(s0 + 1) * n + p];
        I.c = cell_of(T, P, p);
        I.l = P.icn[s0 * n + p];
        I.r = P.icn[(s0 + 1) * n + p];
        I.nl0 = P.stc[(s0 * 2 + 0) * n + p];
        I.nr0 = P.stc[(s0 * 2 + 1) * n + p];
        I.nl1 = P.stc[((s0 + 1) * 2 + 0) * n + p];
        I.nr1 = P.stc[((s0 + 1) * 2 + 1) * n + p];
    }
    return I;
}

__device__ __forceinline__ bool pipe_has_face(int kd) {
    const int k = kd & KIND_MASK;
    return k == K_GHOST || k == K_SAME;
}

// Gathers the stencil primitives of one lane into its slots of stage buffer
// B ([slot*NV + iv][TILE] doubles).  Slots whose cell id is <= 0 are not
// copied: the compute step substitutes as load_nb_rot does.
template <int NDIM>
__device__ __forceinline__ void pipe_prefetch(const double* __restrict__ prim, size_t ncell, const PipeIdx& I,
                                              double* B, int lane) {
    constexpr int NV = Dims<NDIM>::NV;
    if (I.kd0 == K_NONE) return;
    const int ids[PIPE_SLOTS] = {I.c, I.l, I.r, pipe_has_face(I.kd0) ? I.nl0 : 0,
                                 pipe_has_face(I.kd1) ? I.nr1 : 0};
#pragma unroll
    for (int s = 0; s < PIPE_SLOTS; ++s) {
        const int id = ids[s];
        if (id > 0) {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv)
                cp_async8(B + (s * NV + iv) * TILE + lane, prim + (size_t)iv * ncell + (id - 1));
        }
    }
}

// Rotated primitive state of slot s, or the substitute of load_nb_rot for
// id <= 0 (the reference state, normal velocity flipped on a reflecting
// boundary entry).
template <int NDIM>
__device__ __forceinline__ void pipe_state(const TreeView& T, const double* B, int lane, int s, int id, int idim,
                                           const double* qself, double* q) {
    constexpr int NV = Dims<NDIM>::NV;
    if (id > 0) {
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) q[iv] = B[(s * NV + iv) * TILE + lane];
        rot_swap<NDIM>(q, idim);
        return;
    }
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) q[iv] = qself[iv];
    const int ib = -id;
    if (ib > 0 && ib <= T.nbound_type && T.bound_type[ib - 1] == 1) q[1] *= -1.0;
}

template <int NDIM, int RS, int MINB, bool BOXED>
__global__ void __launch_bounds__(TILE * NDIM, MINB)
    k_face_pipe(TreeView T, PlanView P, const double* __restrict__ prim, double* __restrict__ flux,
                double* __restrict__ fsum, DevStatus* st, StepK K) {
    constexpr int NV = Dims<NDIM>::NV, NS = Dims<NDIM>::NS;
    __shared__ __align__(16) double sbuf[NDIM][2][PIPE_SLOTS * NV * TILE];
    __shared__ double sf[NS][NV][TILE];
    const int idim = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t ncell = (size_t)T.ncell;
    const int nc = P.ncells;
    const int ntiles = (nc + TILE - 1) / TILE;
    const int G = gridDim.x;
    const double dt0 = st->dt;
    const DxDiv D0{st->dx, st->inv_dx, st->dx_pow2 != 0};
    unsigned long long iters = 0, calls = 0;

    PipeIdx I0 = pipe_idx(T, P, blockIdx.x, ntiles, lane, idim);
    pipe_prefetch<NDIM>(prim, ncell, I0, sbuf[idim][0], lane);
    cp_async_commit();
    PipeIdx I1 = pipe_idx(T, P, blockIdx.x + G, ntiles, lane, idim);
    int stage = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += G) {
        // gathers for the next tile, indices for the one after
        pipe_prefetch<NDIM>(prim, ncell, I1, sbuf[idim][stage ^ 1], lane);
        cp_async_commit();
        const PipeIdx I2 = pipe_idx(T, P, tile + 2 * G, ntiles, lane, idim);
        cp_async_wait<1>();  // this lane's copies of the current tile have landed
        const double* B = sbuf[idim][stage];
        const int p = tile * TILE + lane;
        if (I0.kd0 != K_NONE) {
            const int c = I0.c;
            double dt = dt0;
            DxDiv D = D0;
            if constexpr (BOXED) step_of_box(P, p, dt, D);
            double qc[NV], ql[NV], qr[NV], qmo[NV], qpo[NV];
            pipe_state<NDIM>(T, B, lane, 0, c, idim, nullptr, qc);
            pipe_state<NDIM>(T, B, lane, 1, I0.l, idim, qc, ql);
            pipe_state<NDIM>(T, B, lane, 2, I0.r, idim, qc, qr);
            own_trace<NDIM>(qc, ql, qr, dt, D, K, qmo, qpo);
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const int kd = side ? I0.kd1 : I0.kd0;
                const int kind = kd & KIND_MASK;
                const int s = 2 * idim + side;
                double f[NV];
                if (kind == K_ZERO) {
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) f[iv] = 0.0;
                } else {
                    double qf[NV];
                    if (kind == K_BOUND) {
                        // boundary branch of neighbour_face: first-order state of the cell
                        double qb[NV], dq0[NV], qm[NV], qp[NV];
#pragma unroll
                        for (int iv = 0; iv < NV; ++iv) {
                            qb[iv] = qc[iv];
                            dq0[iv] = 0.0;
                        }
                        if (kd & KIND_REFLECT) qb[1] *= -1.0;
                        trace<NDIM>(qb, dq0, dt, D.dx, qm, qp, K.gamma);
#pragma unroll
                        for (int iv = 0; iv < NV; ++iv) qf[iv] = side == 0 ? qm[iv] : qp[iv];
                    } else {
                        // neighbour state qn, its stencil cells qnl / qnr
                        const double* qn = side ? qr : ql;
                        double qnl[NV], qnr[NV], qm[NV], qp[NV];
                        if (side == 0) {
                            pipe_state<NDIM>(T, B, lane, 3, I0.nl0, idim, qn, qnl);
                            if (I0.nr0 == c) {
#pragma unroll
                                for (int iv = 0; iv < NV; ++iv) qnr[iv] = qc[iv];
                            } else {
                                load_nb_rot<NDIM>(T, prim, ncell, I0.nr0, idim, qn, qnr);
                            }
                        } else {
                            if (I0.nl1 == c) {
#pragma unroll
                                for (int iv = 0; iv < NV; ++iv) qnl[iv] = qc[iv];
                            } else {
                                load_nb_rot<NDIM>(T, prim, ncell, I0.nl1, idim, qn, qnl);
                            }
                            pipe_state<NDIM>(T, B, lane, 4, I0.nr1, idim, qn, qnr);
                        }
                        if (kind == K_GHOST) ghost_trace<NDIM>(qn, qnl, qnr, dt, D, K, qm, qp);
                        else own_trace<NDIM>(qn, qnl, qnr, dt, D, K, qm, qp);
#pragma unroll
                        for (int iv = 0; iv < NV; ++iv) qf[iv] = side == 0 ? qm[iv] : qp[iv];
                    }
                    if (side == 0) iters += riemann<NDIM, RS>(qf, qpo, f, K);
                    else iters += riemann<NDIM, RS>(qmo, qf, f, K);
                    ++calls;
                    rot_swap<NDIM>(f, idim);
                }
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) {
                    flux[((size_t)s * NV + iv) * nc + p] = f[iv];
                    sf[s][iv][lane] = f[iv];
                }
            }
        }
        __syncthreads();
        if (idim == 0 && I0.kd0 != K_NONE) {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) {
                double fs = 0.0;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const double sign = (s & 1) ? -1.0 : 1.0;
                    fs = fs + sign * sf[s][iv][lane];
                }
                fsum[(size_t)iv * nc + p] = fs;
            }
        }
        __syncthreads();
        I0 = I1;
        I1 = I2;
        stage ^= 1;
    }
    cp_async_wait<0>();
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
}

template <int NDIM, int RS, int MINB, bool BOXED = false>
int launch_face_pipe(rg_ctx* c, const Plan& P, const StepK& K, const double* prim, double* flux, double* fsum) {
    auto kern = k_face_pipe<NDIM, RS, MINB, BOXED>;
    const int block = TILE * NDIM;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
    per_sm = per_sm > 1 ? per_sm : 1;
    const int ntiles = (P.ncells + TILE - 1) / TILE;
    int grid = per_sm * c->sm_count;
    if (ntiles < grid) grid = ntiles;
    if (grid < 1) grid = 1;
    kern<<<grid, block, 0, c->stream>>>(tree_view(c), P.view(), prim, flux, fsum, c->d_status, K);
    return check_cuda(c, cudaGetLastError(), "pipelined face kernel");
}

}  // namespace rg
