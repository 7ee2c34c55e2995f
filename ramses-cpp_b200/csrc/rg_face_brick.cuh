// rg_face_brick.cuh -- face kernel for levels that form one complete periodic
// lattice (detected and verified by rg_lattice.cu).
//
// Same arithmetic and outputs as k_face_tiles (rg_face.cuh): per (cell,
// direction) the own MUSCL-Hancock trace, the two neighbours' face states by
// the ghost (or same-level) branch and the two Riemann fluxes of
// HydroSolver::godunov_fine (RAMSES-CPP src/solvers/hydro/HydroSolver.cpp:
// 93-474); fluxes to the scratch and each cell's own flux sum in the
// reference's (idim, side) order.
//
// A block owns an 8x8x8 brick of cells (on ensemble levels: of one box, whose
// own dt and dx it uses).  It first copies the primitives of
// the brick and a 2-cell periodic halo (12^3 cells, the reach of the own and
// ghost stencils) from HBM into shared memory -- one read of each value per
// brick, through the lattice's id map, instead of per-thread gathers through
// the plan's neighbour and stencil arrays -- and then every thread computes
// all three directions of its cells from shared memory, accumulating the own
// flux sum in registers in slot order.
#pragma once

#include "rg_face.cuh"

namespace rg {

constexpr int BRICK = 8, BHALO = 2, BSIDE = BRICK + 2 * BHALO, BSITES = BSIDE * BSIDE * BSIDE;
constexpr int BRICK_THREADS = 256;
constexpr size_t BRICK_SMEM = sizeof(double) * 5 * BSITES;  // 69,120 bytes (3D: nvar 5)

// Rotated primitive state of shared-memory site `site`: the normal velocity
// read from plane o1 into slot 1, the tangential ones from o2 and o3 (planes
// of the direction, set once per direction by brick_planes), so the rotation
// costs no data movement after the loads.
__device__ __forceinline__ void brick_state(const double* __restrict__ sq, int site, int o1, int o2, int o3,
                                            double* q) {
    q[0] = sq[site];
    q[1] = sq[o1 + site];
    q[2] = sq[o2 + site];
    q[3] = sq[o3 + site];
    q[4] = sq[4 * BSITES + site];
}

// Planes of slots 1..3 for direction idim: rot_swap<3>'s exchange of slot 1
// with slot 1 + idim, applied to where the values are read from.
__device__ __forceinline__ void brick_planes(int idim, int& o1, int& o2, int& o3) {
    o1 = (1 + idim) * BSITES;
    o2 = (idim == 1 ? 1 : 2) * BSITES;
    o3 = (idim == 2 ? 1 : 3) * BSITES;
}

// Lattice geometry of a level: one lattice (nbox == 0: extents ex, ey, ez) or
// one lattice per ensemble box (extents ext[3b..3b+2], sites from off[b] in
// the concatenated maps, bricks from brick_off[b]).
struct BrickGeom {
    int ex, ey, ez, nbox;
    const int* ext;
    const int* off;
    const int* brick_off;
};

// The face work of one brick (index `brick` in the level's brick order), by
// the whole block: stage the brick and its halo in sq (shared, [NV][BSITES]),
// then every cell's fluxes and own flux sum.  Newton statistics of the exact
// solver are added to iters / calls.
template <int RS, bool BOXED>
__device__ __forceinline__ void brick_face(const PlanView& P, const BrickGeom& G, const int* __restrict__ lat_id,
                                           const int* __restrict__ lat_p, int kind, const double* __restrict__ prim,
                                           size_t ncell, double* __restrict__ flux, double* __restrict__ fsum,
                                           const DevStatus* st, const StepK& K, int brick, double* sq,
                                           unsigned long long& iters, unsigned long long& calls) {
    constexpr int NV = 5;
    int ex = G.ex, ey = G.ey, ez = G.ez, local = brick;
    double dt = st->dt;
    DxDiv D{st->dx, st->inv_dx, st->dx_pow2 != 0};
    if constexpr (BOXED) {
        int lo = 0, hi = G.nbox - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (G.brick_off[mid] <= brick) lo = mid;
            else hi = mid - 1;
        }
        local = brick - G.brick_off[lo];
        ex = G.ext[3 * lo];
        ey = G.ext[3 * lo + 1];
        ez = G.ext[3 * lo + 2];
        lat_id += G.off[lo];
        lat_p += G.off[lo];
        const BoxStep& B = P.boxes[lo];
        dt = B.dt;
        D = DxDiv{B.dx, B.inv_dx, B.dx_pow2 != 0};
    }
    const int nbx = ex / BRICK, nby = ey / BRICK;
    const int bx = local % nbx, by = (local / nbx) % nby, bz = local / (nbx * nby);
    const int x0 = bx * BRICK - BHALO, y0 = by * BRICK - BHALO, z0 = bz * BRICK - BHALO;
    for (int t = threadIdx.x; t < BSITES; t += blockDim.x) {
        const int a = t % BSIDE, b = (t / BSIDE) % BSIDE, cz = t / (BSIDE * BSIDE);
        int x = x0 + a, y = y0 + b, z = z0 + cz;
        x = x < 0 ? x + ex : (x >= ex ? x - ex : x);
        y = y < 0 ? y + ey : (y >= ey ? y - ey : y);
        z = z < 0 ? z + ez : (z >= ez ? z - ez : z);
        const size_t id = (size_t)lat_id[(size_t)x + (size_t)ex * ((size_t)y + (size_t)ey * z)] - 1;
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) sq[iv * BSITES + t] = __ldg(prim + iv * ncell + id);
    }
    __syncthreads();
    const int nc = P.ncells;
    const bool ghost = (kind & KIND_MASK) == K_GHOST;
    for (int u = threadIdx.x; u < BRICK * BRICK * BRICK; u += blockDim.x) {
        const int x = u % BRICK, y = (u / BRICK) % BRICK, z = u / (BRICK * BRICK);
        const int site = (x + BHALO) + BSIDE * ((y + BHALO) + BSIDE * (z + BHALO));
        const int p = lat_p[(size_t)(bx * BRICK + x) + (size_t)ex * ((size_t)(by * BRICK + y) + (size_t)ey * (bz * BRICK + z))];
        double fs[NV];
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) fs[iv] = 0.0;
#pragma unroll 1
        for (int idim = 0; idim < 3; ++idim) {
            const int stride = idim == 0 ? 1 : (idim == 1 ? BSIDE : BSIDE * BSIDE);
            int o1, o2, o3;
            brick_planes(idim, o1, o2, o3);
            double qc[NV], ql[NV], qr[NV], qmo[NV], qpo[NV];
            brick_state(sq, site, o1, o2, o3, qc);
            brick_state(sq, site - stride, o1, o2, o3, ql);
            brick_state(sq, site + stride, o1, o2, o3, qr);
            own_trace<3>(qc, ql, qr, dt, D, K, qmo, qpo);
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                // neighbour n = c -/+ e, its stencil (n - e, n + e) = (c - 2e, c) / (c, c + 2e)
                double qn[NV], qfar[NV], qm[NV], qp[NV], f[NV];
                brick_state(sq, side ? site + stride : site - stride, o1, o2, o3, qn);
                brick_state(sq, side ? site + 2 * stride : site - 2 * stride, o1, o2, o3, qfar);
                const double* qnl = side ? qc : qfar;
                const double* qnr = side ? qfar : qc;
                if (ghost) ghost_trace<3>(qn, qnl, qnr, dt, D, K, qm, qp);
                else own_trace<3>(qn, qnl, qnr, dt, D, K, qm, qp);
                if (side == 0) iters += riemann<3, RS>(qm, qpo, f, K);
                else iters += riemann<3, RS>(qmo, qp, f, K);
                ++calls;
                rot_swap<3>(f, idim);
                const int s = 2 * idim + side;
                const double sign = side ? -1.0 : 1.0;
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) {
                    flux[((size_t)s * NV + iv) * nc + p] = f[iv];
                    fs[iv] = fs[iv] + sign * f[iv];
                }
            }
        }
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) fsum[(size_t)iv * nc + p] = fs[iv];
    }
}

template <int RS, int MINB, bool BOXED>
__global__ void __launch_bounds__(BRICK_THREADS, MINB)
    k_face_brick(PlanView P, BrickGeom G, const int* __restrict__ lat_id, const int* __restrict__ lat_p, int kind,
                 const double* __restrict__ prim, size_t ncell, double* __restrict__ flux,
                 double* __restrict__ fsum, DevStatus* st, StepK K) {
    extern __shared__ __align__(16) double sq[];  // [NV][BSITES]
    unsigned long long iters = 0, calls = 0;
    brick_face<RS, BOXED>(P, G, lat_id, lat_p, kind, prim, ncell, flux, fsum, st, K, (int)blockIdx.x, sq, iters,
                          calls);
    if (RS == RG_RIEMANN_EXACT) {
        for (int o = 16; o > 0; o >>= 1) {
            iters += __shfl_xor_sync(0xffffffffu, iters, o);
            calls += __shfl_xor_sync(0xffffffffu, calls, o);
        }
        if ((threadIdx.x & 31) == 0 && calls) {
            atomicAdd(&st->exact_iters, iters);
            atomicAdd(&st->exact_calls, calls);
        }
    }
}

template <int RS, int MINB, bool BOXED = false>
int launch_face_brick(rg_ctx* c, const Plan& P, const StepK& K, const double* prim, double* flux, double* fsum) {
    auto kern = k_face_brick<RS, MINB, BOXED>;
    static bool attr_set[64] = {};  // per device: the shared-memory opt-in is a function attribute
    const int dev = c->device & 63;
    if (!attr_set[dev]) {
        if (int rc = check_cuda(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        (int)BRICK_SMEM),
                                "brick kernel shared memory"))
            return rc;
        attr_set[dev] = true;
    }
    const BrickGeom G{P.lat_e[0], P.lat_e[1], P.lat_e[2], P.nbox, P.bl_ext, P.bl_off, P.bl_brick_off};
    const int nbricks =
        BOXED ? P.bl_nbricks : (P.lat_e[0] / BRICK) * (P.lat_e[1] / BRICK) * (P.lat_e[2] / BRICK);
    kern<<<nbricks, BRICK_THREADS, BRICK_SMEM, c->stream>>>(P.view(), G, P.lat_id, P.lat_p, P.lat_kind, prim,
                                                            (size_t)c->ncell, flux, fsum, c->d_status, K);
    return check_cuda(c, cudaGetLastError(), "brick face kernel");
}

}  // namespace rg
