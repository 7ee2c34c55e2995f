// rg_face.cu -- persistent, tiled face kernel and its autotuner.
//
// Work unit: a tile of 32 consecutive level cells (one warp wide).  A block
// holds R tiles x ndim directions, one warp per (tile, direction): the warp
// computes, for its 32 cells, the own trace along the direction, the two
// neighbour face states and the two Riemann fluxes (HydroSolver.cpp:93-474 of
// RAMSES-CPP).  The fluxes go to global memory (the neighbours' reflux events
// read them) and to shared memory, where the direction-0 warp then forms each
// cell's own flux sum in the reference's (idim, side) order
// (HydroSolver.cpp:485-486), so the fold reads 5 doubles for the own update
// instead of 2*ndim*5.
//
// Blocks are persistent: a grid sized from the occupancy of the chosen
// variant pulls batches of tiles from a counter in device memory; the last
// block to finish resets the counter for the next launch (no waiting on
// anything).  The autotuner times every (variant, batch) pair once per level
// plan on the level's own data and keeps the fastest.
#include <algorithm>
#include <cstdio>

#include "rg_face.cuh"

namespace rg {

namespace {

constexpr int TILE = 32;

template <int NDIM, int RS, int R, int MINB>
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
    const double dt = st->dt;
    const DxDiv D{st->dx, st->inv_dx, st->dx_pow2 != 0};
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
                    double qc[NV], qmo[NV], qpo[NV];
                    load_rot<NDIM>(prim, ncell, c, idim, qc);
                    if (P.level0) {
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
                            neighbour_face<NDIM>(T, P, prim, uold, ncell, p, c, idim, side, kd, n, qc, dt, D, K, qf);
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
// resident blocks (caps registers per thread).
struct Variant {
    int R, minb;
};
constexpr Variant kVariants[] = {{1, 5}, {1, 6}, {1, 8}, {2, 3}, {2, 4}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);
constexpr int kBatches[] = {1, 4, 16};

template <int NDIM, int RS, int R, int MINB>
int launch_one(rg_ctx* c, const Plan& P, const StepK& K, int batch, const double* uold, const double* prim,
               double* flux, double* fsum) {
    auto kern = k_face_tiles<NDIM, RS, R, MINB>;
    const int block = TILE * NDIM * R;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
    per_sm = std::max(per_sm, 1);
    const int ntiles = (P.ncells + TILE - 1) / TILE;
    const int grabs = (ntiles + batch * R - 1) / (batch * R);
    const int grid = std::max(1, std::min(grabs, per_sm * c->sm_count));
    kern<<<grid, block, 0, c->stream>>>(tree_view(c), P.view(), prim, uold, flux, fsum, c->d_status, K, batch);
    return check_cuda(c, cudaGetLastError(), "face kernel");
}

template <int NDIM, int RS>
int launch_rs(rg_ctx* c, const Plan& P, const StepK& K, int variant, int batch, const double* uold,
              const double* prim, double* flux, double* fsum) {
    switch (variant) {
        case 0: return launch_one<NDIM, RS, 1, 5>(c, P, K, batch, uold, prim, flux, fsum);
        case 1: return launch_one<NDIM, RS, 1, 6>(c, P, K, batch, uold, prim, flux, fsum);
        case 2: return launch_one<NDIM, RS, 1, 8>(c, P, K, batch, uold, prim, flux, fsum);
        case 3: return launch_one<NDIM, RS, 2, 3>(c, P, K, batch, uold, prim, flux, fsum);
        default: return launch_one<NDIM, RS, 2, 4>(c, P, K, batch, uold, prim, flux, fsum);
    }
}

template <int NDIM>
int launch_nd(rg_ctx* c, const Plan& P, const StepK& K, int variant, int batch, const double* uold,
              const double* prim, double* flux, double* fsum) {
    switch (c->params.riemann) {
        case RG_RIEMANN_HLLC: return launch_rs<NDIM, RG_RIEMANN_HLLC>(c, P, K, variant, batch, uold, prim, flux, fsum);
        case RG_RIEMANN_HLL: return launch_rs<NDIM, RG_RIEMANN_HLL>(c, P, K, variant, batch, uold, prim, flux, fsum);
        case RG_RIEMANN_EXACT: return launch_rs<NDIM, RG_RIEMANN_EXACT>(c, P, K, variant, batch, uold, prim, flux, fsum);
        case RG_RIEMANN_ACOUSTIC:
            return launch_rs<NDIM, RG_RIEMANN_ACOUSTIC>(c, P, K, variant, batch, uold, prim, flux, fsum);
        default: return launch_rs<NDIM, RG_RIEMANN_LLF>(c, P, K, variant, batch, uold, prim, flux, fsum);
    }
}

}  // namespace

int launch_face_tiles(rg_ctx* c, const Plan& P, const StepK& K, const double* uold, const double* prim,
                      double* flux, double* fsum) {
    if (P.ncells == 0) return RG_OK;
    int v = P.face_variant >= 0 ? P.face_variant : 1;
    int b = P.face_batch > 0 ? P.face_batch : 4;
    if (c->params.ndim == 1) return launch_nd<1>(c, P, K, v, b, uold, prim, flux, fsum);
    return launch_nd<3>(c, P, K, v, b, uold, prim, flux, fsum);
}

// Times every (variant, batch) on the level's current data (the face kernel
// only writes the flux scratch, so repeating it changes no state) and keeps
// the fastest.  Small levels keep the default.  Must run outside a capture.
int autotune_face(rg_ctx* c, Plan& P, const StepK& K) {
    if (P.face_variant >= 0) return RG_OK;
    P.face_variant = 1;
    P.face_batch = 4;
    if (P.ncells < (1 << 14) || c->no_autotune) return RG_OK;
    const int ns = 2 * c->params.ndim, nv = c->params.ndim + 2;
    double* fsum = c->d_flux + (size_t)ns * nv * P.ncells;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bv = 1, bb = 4;
    for (int v = 0; v < kNumVariants; ++v) {
        for (int b : kBatches) {
            float tmin = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                cudaEventRecord(e0, c->stream);
                int nd = c->params.ndim;
                int rc = nd == 1 ? launch_nd<1>(c, P, K, v, b, c->d_uold, c->d_prim, c->d_flux, fsum)
                                 : launch_nd<3>(c, P, K, v, b, c->d_uold, c->d_prim, c->d_flux, fsum);
                if (rc) {
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                    return rc;
                }
                cudaEventRecord(e1, c->stream);
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) tmin = std::min(tmin, ms);  // first launch warms caches and code
            }
            if (tmin < best) {
                best = tmin;
                bv = v;
                bb = b;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P.face_variant = bv;
    P.face_batch = bb;
    P.face_ms = best;
    return check_cuda(c, cudaGetLastError(), "face autotune");
}

}  // namespace rg
