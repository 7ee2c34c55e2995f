// rg_step.cu -- the per-substep kernels of the Godunov level step.
//
// One level substep (Simulation.cpp:548-614 of RAMSES-CPP) is, on the device:
//   k_courant   per-cell CFL candidate + exact min-reduction
//               (HydroSolver::compute_courant_step, HydroSolver.cpp:878-977)
//   k_set_unew  unew <- uold on the level           (HydroSolver.cpp:575-590)
//   k_prim      conservative -> primitive, once per cell the level reads
//               (the reference recomputes it ~34x per cell update)
//   k_face      per (cell, dimension): the cell's own MUSCL-Hancock trace,
//               the neighbours' face states (ghost / same-level / boundary
//               branches) and the two Riemann fluxes of the cell's faces
//               (HydroSolver.cpp:93-115,118-474)
//   k_fold      per target cell: its updates applied in the CPU order --
//               refluxes from neighbours processed earlier, its own flux sum
//               and clamps, refluxes from later neighbours
//               (HydroSolver.cpp:476-547)
//   k_set_uold  uold <- unew where son == 0          (HydroSolver.cpp:592-611)
// All FP64; compiled with -fmad=false so every result is bit-identical to the
// reference's x86-64 build for the HLLC/HLL/LLF/acoustic solvers.
#include <algorithm>

#include "rg_face.cuh"
#include "rg_fold.cuh"
#include "rg_internal.cuh"
#include "rg_physics.cuh"

namespace rg {

namespace {

template <int NDIM, int RS>
__global__ void __launch_bounds__(128) k_face(TreeView T, PlanView P, const double* __restrict__ prim,
                                              const double* __restrict__ uold, double* __restrict__ flux,
                                              const DevStatus* __restrict__ st, StepK K,
                                              unsigned long long* __restrict__ exact_iters) {
    constexpr int NV = Dims<NDIM>::NV;
    const size_t ncell = (size_t)T.ncell;
    const int nc = P.ncells;
    const double dt = st->dt;
    const DxDiv D{st->dx, st->inv_dx, st->dx_pow2 != 0};
    const long long total = (long long)nc * NDIM;
    unsigned long long iters = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int idim = (int)(t / nc), p = (int)(t - (long long)idim * nc);
        int s0 = 2 * idim;
        int kd0 = P.kind[(size_t)s0 * nc + p];
        if (kd0 == K_NONE) continue;
        int kd1 = P.kind[(size_t)(s0 + 1) * nc + p];
        int c = cell_of(T, P, p);
        double qc[NV], qmo[NV], qpo[NV], ql[NV], qr[NV];
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
            int l = P.icn[(size_t)s0 * nc + p], r = P.icn[(size_t)(s0 + 1) * nc + p];
            load_nb_rot<NDIM>(T, prim, ncell, l, idim, qc, ql);
            load_nb_rot<NDIM>(T, prim, ncell, r, idim, qc, qr);
            own_trace<NDIM>(qc, ql, qr, dt, D, K, qmo, qpo);
        }
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            int kd = side ? kd1 : kd0;
            int s = s0 + side;
            double f[NV];
            if ((kd & KIND_MASK) == K_ZERO) {
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) f[iv] = 0.0;
            } else {
                int n = P.icn[(size_t)s * nc + p];
                double qf[NV];
                neighbour_face<NDIM>(T, P, prim, uold, ncell, p, c, idim, side, kd, n, qc, side ? qr : ql, dt, D, K,
                                     qf);
                if (side == 0) iters += riemann<NDIM, RS>(qf, qpo, f, K);
                else iters += riemann<NDIM, RS>(qmo, qf, f, K);
                rot_swap<NDIM>(f, idim);
            }
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) flux[((size_t)s * NV + iv) * nc + p] = f[iv];
        }
    }
    if (RS == RG_RIEMANN_EXACT && exact_iters && iters) atomicAdd(exact_iters, iters);
}

__device__ __forceinline__ void set_step_values(DevStatus* st, double dt, double dx);

// dt_dev != nullptr: also the step values (dt, dt/dx, 1/dx) from the dt in
// device memory, by one thread (nothing in this kernel reads them; the face
// and fold kernels after it do).
template <int NDIM>
__global__ void k_prim(TreeView T, PlanView P, const double* __restrict__ uold, double* __restrict__ prim,
                       double gamma, double smalle, DevStatus* st = nullptr, const double* dt_dev = nullptr,
                       double dx = 0.0) {
    constexpr int NV = Dims<NDIM>::NV;
    const size_t ncell = (size_t)T.ncell;
    if (dt_dev && blockIdx.x == 0 && threadIdx.x == 0) set_step_values(st, *dt_dev, dx);
    const int total = P.ncells + P.nextra_prim;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int c = (t < P.ncells) ? cell_of(T, P, t) : P.xprim[t - P.ncells];
        double u[NV], q[NV];
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) u[iv] = uold[(size_t)iv * ncell + c - 1];
        ctoprim<NDIM>(u, q, gamma, smalle);
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) prim[(size_t)iv * ncell + c - 1] = q[iv];
    }
}

// dt/dx of the box a target belongs to (ensemble levels): a target's updates
// all come from its own box, so its first event's source tells the box.
template <int NDIM>
__device__ __forceinline__ double box_dtdx(const PlanView& P, int a) {
    constexpr int TTD = Dims<NDIM>::TTD;
    const int cp = P.tev[a] >> 3;
    return P.boxes[box_of(P, P.level0 ? cp : (cp % TTD) * P.noct + cp / TTD)].dtdx;
}

// LEAF: the level has no refined cell, so set_unew (unew <- uold) and
// set_uold (uold <- unew) of its cells are folded in: a level target starts
// from uold and its result is written to both arrays.  Coarser targets start
// from unew as always.
// uold_out != nullptr (a level with refined cells in an AMR step): set_uold
// folded in -- every level target (all of the level's son == 0 cells, each
// with at least its own update) also writes its result to uold_out.
// (blocks bid of nb; a thread a target)
template <int NDIM, bool LEAF, bool FSUM>
__device__ __forceinline__ void fold_short(int bid, int nb, const TreeView& T, const PlanView& P,
                                           const double* __restrict__ flux, double* __restrict__ unew,
                                           const DevStatus* __restrict__ st, double gamma, double* __restrict__ uold,
                                           const double* __restrict__ fsum, double* __restrict__ uold_out) {
    constexpr int NV = Dims<NDIM>::NV;
    const size_t ncell = (size_t)T.ncell;
    const int nc = P.ncells;
    const double dtdx0 = st->dtdx;
    for (int t = bid * blockDim.x + threadIdx.x; t < P.ntarg; t += nb * blockDim.x) {
        int a = P.toff[t], b = P.toff[t + 1];
        if (a == b || b - a > kLongEvents) continue;  // long targets: fold_long
        const double dtdx = P.obox ? box_dtdx<NDIM>(P, a) : dtdx0;
        int cell = (t < nc) ? cell_of(T, P, t) : P.textra[t - nc];
        const bool from_old = LEAF && t < nc;
        const double* src = from_old ? uold : unew;
        double u[NV];
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) u[iv] = src[(size_t)iv * ncell + cell - 1];
        if (P.obox) fold_events<NDIM, FSUM, false>(P, a, b, flux, fsum, gamma, dtdx, u);
        else fold_events<NDIM, FSUM>(P, a, b, flux, fsum, gamma, dtdx, u);
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) unew[(size_t)iv * ncell + cell - 1] = u[iv];
        if (from_old) {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) uold[(size_t)iv * ncell + cell - 1] = u[iv];
        } else if (uold_out && t < nc) {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) uold_out[(size_t)iv * ncell + cell - 1] = u[iv];
        }
    }
}

// The targets fold_short skips, those with more than kLongEvents updates (in
// AMR runs, coarse cells that take the refluxes of many finer faces: 192 at
// the edge of the finest level of the 64^3-base Sedov run), one warp each.  A
// thread walking such a chain waits on its loads event after event, and the
// few long chains set the whole fold's duration.  Here the lanes fetch 32
// events at a time and form each one's term -- dtdx * sign * flux * factor
// for a reflux, the own flux sum for the own update, the expressions of
// fold_events -- and the terms are then applied in event order:
//   - a coarser target takes refluxes only, whose subtractions act on each
//     variable separately, so lane iv walks variable iv's terms in order
//     from shared memory;
//   - a level cell (whose own update mixes the variables through its clamps)
//     applies them on values broadcast from the lane that formed them, every
//     lane computing the whole state.
// Either way the result is the sequential fold's arithmetic, bit for bit.
constexpr int kLongThreads = 256, kLongChunk = 32, kLongPad = kLongChunk + 1;

template <int NDIM, bool LEAF, bool FSUM>
__device__ __forceinline__ void fold_long(int bid, int nb, const TreeView& T, const PlanView& P,
                                          const int* __restrict__ tlong, int nlong, const double* __restrict__ flux,
                                          double* __restrict__ unew, const DevStatus* __restrict__ st, double gamma,
                                          double* __restrict__ uold, const double* __restrict__ fsum,
                                          double* __restrict__ uold_out) {
    constexpr int NV = Dims<NDIM>::NV, NS = Dims<NDIM>::NS, TTD = Dims<NDIM>::TTD;
    // per warp: the terms of one chunk, variable-major, rows padded so the
    // NV walking lanes read from different banks
    __shared__ double terms[kLongThreads / 32][NV * kLongPad];
    double* my = terms[threadIdx.x >> 5];
    const size_t ncell = (size_t)T.ncell;
    const int nc = P.ncells, lane = threadIdx.x & 31;
    const int nwarp = (int)(((size_t)nb * blockDim.x) >> 5);
    const double factor = 1.0 / (1 << NDIM);
    for (int w = (int)(((size_t)bid * blockDim.x + threadIdx.x) >> 5); w < nlong; w += nwarp) {
        const int t = tlong[w];
        const int a = P.toff[t], b = P.toff[t + 1];
        const double dtdx = P.obox ? box_dtdx<NDIM>(P, a) : st->dtdx;
        if (t >= nc) {
            const int cell = P.textra[t - nc];
            double u = lane < NV ? unew[(size_t)lane * ncell + cell - 1] : 0.0;
            for (int e0 = a; e0 < b; e0 += kLongChunk) {
                const int e = e0 + lane;
                if (e < b) {
                    const int key = P.tev[e];
                    const int slot = key & 7, cp = key >> 3;
                    const int ps = P.level0 ? cp : (cp % TTD) * P.noct + cp / TTD;
                    const double sign = (slot & 1) ? -1.0 : 1.0;
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv)
                        my[iv * kLongPad + lane] = dtdx * sign * flux[((size_t)slot * NV + iv) * nc + ps] * factor;
                }
                __syncwarp();
                const int m = (b - e0 < kLongChunk) ? b - e0 : kLongChunk;
                if (lane < NV) {
                    const double* s = my + lane * kLongPad;
#pragma unroll 8
                    for (int j = 0; j < m; ++j) u = u - s[j];
                }
                __syncwarp();
            }
            if (lane < NV) unew[(size_t)lane * ncell + cell - 1] = u;
            continue;
        }
        const int cell = cell_of(T, P, t);
        const bool from_old = LEAF;
        const double* src = from_old ? uold : unew;
        double u[NV];
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) u[iv] = src[(size_t)iv * ncell + cell - 1];
        for (int e0 = a; e0 < b; e0 += 32) {
            const int e = e0 + lane;
            int own = 0;
            double val[NV];
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) val[iv] = 0.0;
            if (e < b) {
                const int key = P.tev[e];
                const int slot = key & 7, cp = key >> 3;
                const int ps = P.level0 ? cp : (cp % TTD) * P.noct + cp / TTD;
                if (slot == OWN_SLOT) {
                    own = 1;
                    if constexpr (FSUM) {
#pragma unroll
                        for (int iv = 0; iv < NV; ++iv) val[iv] = fsum[(size_t)iv * nc + ps];
                    } else {
#pragma unroll
                        for (int sl = 0; sl < NS; ++sl) {
                            const double sign = (sl & 1) ? -1.0 : 1.0;
#pragma unroll
                            for (int iv = 0; iv < NV; ++iv)
                                val[iv] = val[iv] + sign * flux[((size_t)sl * NV + iv) * nc + ps];
                        }
                    }
                } else {
                    const double sign = (slot & 1) ? -1.0 : 1.0;
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) val[iv] = dtdx * sign * flux[((size_t)slot * NV + iv) * nc + ps] * factor;
                }
            }
            const int m = (b - e0 < 32) ? b - e0 : 32;
            for (int j = 0; j < m; ++j) {
                const int oj = __shfl_sync(0xffffffffu, own, j);
                double vj[NV];
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) vj[iv] = __shfl_sync(0xffffffffu, val[iv], j);
                if (oj) {
                    own_update<NDIM>(vj, gamma, dtdx, u);
                } else {
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) u[iv] = u[iv] - vj[iv];
                }
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) unew[(size_t)iv * ncell + cell - 1] = u[iv];
            if (from_old) {
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) uold[(size_t)iv * ncell + cell - 1] = u[iv];
            } else if (uold_out) {
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) uold_out[(size_t)iv * ncell + cell - 1] = u[iv];
            }
        }
    }
}

inline int grid_for(rg_ctx* c, long long work, int block) {
    long long b = (work + block - 1) / block;
    long long cap = (long long)c->sm_count * 32;
    if (b > cap) b = cap;
    return (int)std::max(1LL, b);
}

// One launch for a level's targets: its first long_blocks blocks walk the
// long targets a warp each, the others the rest a thread each.  The two sets
// are disjoint and each target is folded by one thread or warp, so the split
// changes no result; scheduled first, the long chains overlap the short ones.
template <int NDIM, bool LEAF = false, bool FSUM = false>
__global__ void __launch_bounds__(kLongThreads)
    k_fold(TreeView T, PlanView P, const int* __restrict__ tlong, int nlong, int long_blocks,
           const double* __restrict__ flux, double* __restrict__ unew, const DevStatus* __restrict__ st, double gamma,
           double* __restrict__ uold = nullptr, const double* __restrict__ fsum = nullptr,
           double* __restrict__ uold_out = nullptr) {
    const int b = (int)blockIdx.x;
    if (b < long_blocks)
        fold_long<NDIM, LEAF, FSUM>(b, long_blocks, T, P, tlong, nlong, flux, unew, st, gamma, uold, fsum, uold_out);
    else
        fold_short<NDIM, LEAF, FSUM>(b - long_blocks, (int)gridDim.x - long_blocks, T, P, flux, unew, st, gamma, uold,
                                     fsum, uold_out);
}

template <int NDIM, bool LEAF = false, bool FSUM = false>
void launch_fold(rg_ctx* c, const Plan& P, const TreeView& T, const PlanView& V, const double* flux, double* unew,
                 double gamma, double* uold = nullptr, const double* fsum = nullptr, double* uold_out = nullptr) {
    const int long_blocks =
        P.nlong > 0 ? (int)std::min<long long>(((long long)P.nlong * 32 + kLongThreads - 1) / kLongThreads, 4096) : 0;
    const int grid = long_blocks + grid_for(c, P.ntarg, kLongThreads);
    k_fold<NDIM, LEAF, FSUM><<<grid, kLongThreads, 0, c->stream>>>(T, V, P.tlong, P.nlong, long_blocks, flux, unew,
                                                                   c->d_status, gamma, uold, fsum, uold_out);
}

// The block's minimum of `best` (every thread of the block calls this, none
// may have returned) min-ed into *dst with one global atomic per block: the
// warps' minima meet in shared memory first, so thousands of warps do not
// queue on the one word.  The minimum of bit patterns is the same in any
// order.
__device__ __forceinline__ void block_atomic_min(unsigned long long best, unsigned long long* dst) {
    __shared__ unsigned long long s_min;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
        best = other < best ? other : best;
    }
    if (threadIdx.x == 0) s_min = ~0ULL;
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && best != ~0ULL) atomicMin(&s_min, best);
    __syncthreads();
    if (threadIdx.x == 0 && s_min != ~0ULL) atomicMin(dst, s_min);
}

// Leaf-level fold that also prepares the next substep: on a level whose
// stencils and updates stay inside it (no extra primitive cells, no extra
// targets), the new state of every level cell is in registers here, so its
// primitives (the next face step's input) and its CFL candidate (min-reduced
// into the re-armed CFL word; per box on ensemble levels) are formed at once
// instead of in a separate pass over uold.  Warps walk aligned runs of 32
// targets so the per-box min can use a segmented shuffle.
template <int NDIM, bool BOXED>
__global__ void k_fold_next(TreeView T, PlanView P, const double* __restrict__ flux, double* __restrict__ unew,
                            DevStatus* st, double gamma, double smalle, double* __restrict__ uold,
                            const double* __restrict__ fsum, double* __restrict__ prim, double dx, double cfl,
                            int pressure_cap) {
    constexpr int NV = Dims<NDIM>::NV;
    const size_t ncell = (size_t)T.ncell;
    const int nt = P.ntarg;
    const double dtdx0 = st->dtdx;
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long best_all = ~0ULL;
    for (long long base = warp * 32; base < nt; base += nwarps * 32) {
        const int t = (int)(base + lane);
        unsigned long long best = ~0ULL;
        int box = -1;
        if (t < nt) {
            const int a = P.toff[t], b = P.toff[t + 1];
            const int cell = cell_of(T, P, t);
            double u[NV], q[NV];
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) u[iv] = uold[(size_t)iv * ncell + cell - 1];
            if (a < b) {
                const double dtdx = BOXED ? box_dtdx<NDIM>(P, a) : dtdx0;
                fold_events<NDIM, true, !BOXED>(P, a, b, flux, fsum, gamma, dtdx, u);
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) {
                    unew[(size_t)iv * ncell + cell - 1] = u[iv];
                    uold[(size_t)iv * ncell + cell - 1] = u[iv];
                }
            }
            ctoprim<NDIM>(u, q, gamma, smalle);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) prim[(size_t)iv * ncell + cell - 1] = q[iv];
            if (T.son[cell - 1] == 0) {
                if (BOXED) box = box_of(P, t);
                unsigned long long bits;
                if (cfl_candidate<NDIM>(u, BOXED ? P.boxes[box].dx : dx, gamma, cfl, pressure_cap, &bits))
                    best = bits;
            }
        }
        if constexpr (BOXED) {
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long ob = __shfl_down_sync(0xffffffffu, best, o);
                const int obx = __shfl_down_sync(0xffffffffu, box, o);
                if (lane + o < 32 && obx == box && ob < best) best = ob;
            }
            const int prev = __shfl_up_sync(0xffffffffu, box, 1);
            if (box >= 0 && (lane == 0 || prev != box) && best != ~0ULL) atomicMin(&P.boxes[box].dtmin_bits, best);
        } else {
            best_all = best < best_all ? best : best_all;
        }
    }
    if constexpr (!BOXED) {
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, best_all, o);
            best_all = other < best_all ? other : best_all;
        }
        if (lane == 0 && best_all != ~0ULL) atomicMin(&st->dtmin_bits, best_all);
    }
}

__global__ void k_copy_level(TreeView T, PlanView P, int nvar, const double* __restrict__ src, double* __restrict__ dst,
                             int only_leaf) {
    const size_t ncell = (size_t)T.ncell;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P.ncells; p += gridDim.x * blockDim.x) {
        int c = cell_of(T, P, p);
        if (only_leaf && T.son[c - 1] != 0) continue;
        for (int iv = 0; iv < nvar; ++iv) dst[(size_t)iv * ncell + c - 1] = src[(size_t)iv * ncell + c - 1];
    }
}

// unew_copy != nullptr: set_unew of the level in the same pass (every level
// cell's uold copied into unew_copy, refined cells included, as
// HydroSolver::set_unew does).
template <int NDIM>
__global__ void k_courant(TreeView T, PlanView P, const double* __restrict__ uold, DevStatus* st, double dx,
                          double gamma, double cfl, int pressure_cap, double* __restrict__ unew_copy,
                          ClockStep clock, double* __restrict__ prim, double smalle) {
    constexpr int NV = NDIM + 2;
    const size_t ncell = (size_t)T.ncell;
    unsigned long long best = ~0ULL;
    // with prim: the extra (ghost-stencil) cells after the level's, primitives only
    const int total = prim ? P.ncells + P.nextra_prim : P.ncells;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
        int id = (p < P.ncells) ? cell_of(T, P, p) : P.xprim[p - P.ncells];
        if (prim) {
            // k_prim's pass (ctoprim of uold), folded in
            double u[NV], q[NV];
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) u[iv] = uold[(size_t)iv * ncell + id - 1];
            ctoprim<NDIM>(u, q, gamma, smalle);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) prim[(size_t)iv * ncell + id - 1] = q[iv];
            if (p >= P.ncells) continue;
        }
        if (unew_copy) {
#pragma unroll
            for (int iv = 0; iv < NDIM + 2; ++iv) unew_copy[(size_t)iv * ncell + id - 1] = uold[(size_t)iv * ncell + id - 1];
        }
        if (T.son[id - 1] > 0) continue;
        const double* u = uold + (id - 1);
        double d = smax(u[0], 1e-10), v2 = 0.0;
#pragma unroll
        for (int i = 1; i <= NDIM; ++i) {
            double v = u[i * ncell] / d;
            v2 = v2 + v * v;
        }
        double e_non = 0.0, sum_gamma_p = 0.0;
        double pr = smax((u[(NDIM + 1) * ncell] - 0.5 * d * v2 - e_non) * (gamma - 1.0), d * 1e-10);
        if (pressure_cap) pr = smin(pr, d * 1e2);
        double cs2 = cs2_of(d, pr, gamma);
        cs2 = cs2 + sum_gamma_p / d;
        double cs = sqrt(smax(cs2, 1e-10));
        double u_wave = NDIM * cs;
#pragma unroll
        for (int i = 1; i <= NDIM; ++i) u_wave = u_wave + fabs(u[i * ncell] / d);
        double a_grav = 0.0;
#pragma unroll
        for (int i = 1; i <= NDIM; ++i) a_grav = a_grav + fabs(0.0);
        double alpha = a_grav * dx / (u_wave * u_wave);
        alpha = smax(alpha, 0.0001);
        double dtc = (dx / u_wave) * (sqrt(1.0 + 2.0 * cfl * alpha) - 1.0) / alpha;
        // positive doubles order like their bit patterns; NaN patterns sort
        // above every finite value, matching std::min's NaN fall-through.
        unsigned long long b = (unsigned long long)__double_as_longlong(dtc);
        if (dtc >= 0.0 && b < best) best = b;
    }
    block_atomic_min(best, &st->dtmin_bits);
    if (!clock.ck) return;
    // the last block to finish (every other block's minimum is in the word by
    // then: each block's thread 0 puts it there before it fences and counts)
    // does the clock update and resets the count for the next pass
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&st->cfl_done, 1u) == gridDim.x - 1) {
            __threadfence();
            st->cfl_done = 0;
            clock_step_apply(clock, st, atomicOr(&st->dtmin_bits, 0ULL));  // the word read at L2
            if (clock.set_step) set_step_values(st, clock.ck[clock.il], clock.dx);
        }
    }
}

// The clock update alone (a level without cells in its plan).
__global__ void k_clock_step(DevStatus* st, ClockStep clock) {
    clock_step_apply(clock, st, st->dtmin_bits);
    if (clock.set_step) set_step_values(st, clock.ck[clock.il], clock.dx);
}

// CFL candidate and primitives in one pass over uold (leaf-level substep).
template <int NDIM>
__global__ void k_courant_prim(TreeView T, PlanView P, const double* __restrict__ uold, double* __restrict__ prim,
                               DevStatus* st, double dx, double gamma, double smalle, double cfl, int pressure_cap) {
    constexpr int NV = Dims<NDIM>::NV;
    const size_t ncell = (size_t)T.ncell;
    const int total = P.ncells + P.nextra_prim;
    unsigned long long best = ~0ULL;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int id = (t < P.ncells) ? cell_of(T, P, t) : P.xprim[t - P.ncells];
        double u[NV], q[NV];
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) u[iv] = uold[(size_t)iv * ncell + id - 1];
        ctoprim<NDIM>(u, q, gamma, smalle);
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) prim[(size_t)iv * ncell + id - 1] = q[iv];
        if (t >= P.ncells || T.son[id - 1] > 0) continue;
        unsigned long long b;
        if (cfl_candidate<NDIM>(u, dx, gamma, cfl, pressure_cap, &b) && b < best) best = b;
    }
    block_atomic_min(best, &st->dtmin_bits);
}

__global__ void k_courant_init(DevStatus* st, double dt_start) {
    st->dtmin_bits = (unsigned long long)__double_as_longlong(dt_start);
}
__device__ __forceinline__ void set_step_values(DevStatus* st, double dt, double dx) {
    st->dt = dt;
    st->dx = dx;
    st->dtdx = dt / dx;
    double inv = 1.0 / dx;
    st->inv_dx = inv;
    st->dx_pow2 = is_pow2_with_normal_inverse(dx, inv) ? 1 : 0;
}
// Takes the step from the CFL word and re-arms the word at dt_start, ready for
// the candidates of the next step (the fused fold adds them).
__global__ void k_dt_finalize(DevStatus* st, double dx, double dt_start) {
    set_step_values(st, __longlong_as_double((long long)st->dtmin_bits), dx);
    st->dtmin_bits = (unsigned long long)__double_as_longlong(dt_start);
}
__global__ void k_dt_set(DevStatus* st, double dt, double dx) { set_step_values(st, dt, dx); }
__global__ void k_dt_set_dev(DevStatus* st, const double* dt, double dx) { set_step_values(st, *dt, dx); }

// ---- ensemble levels: one CFL step per box
__global__ void k_box_courant_init(BoxStep* boxes, int nbox, double dt_start) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbox; b += gridDim.x * blockDim.x)
        boxes[b].dtmin_bits = (unsigned long long)__double_as_longlong(dt_start);
}
__global__ void k_box_dt_finalize(BoxStep* boxes, int nbox, double dt_start) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbox; b += gridDim.x * blockDim.x) {
        BoxStep& B = boxes[b];
        const double dt = __longlong_as_double((long long)B.dtmin_bits), dx = B.dx;
        B.dtmin_bits = (unsigned long long)__double_as_longlong(dt_start);
        B.dt = dt;
        B.dtdx = dt / dx;
        const double inv = 1.0 / dx;
        B.inv_dx = inv;
        B.dx_pow2 = is_pow2_with_normal_inverse(dx, inv) ? 1 : 0;
    }
}

// k_courant_prim of an ensemble level: each cell's CFL candidate uses its
// box's dx and goes to its box's min-reduction word.  Warps walk aligned runs
// of 32 consecutive level cells; a box owns contiguous oct positions, so the
// lanes of one box form one run and a segmented shuffle min leaves one atomic
// per run.
template <int NDIM>
__global__ void k_courant_prim_boxes(TreeView T, PlanView P, const double* __restrict__ uold,
                                     double* __restrict__ prim, double gamma, double smalle, double cfl,
                                     int pressure_cap) {
    constexpr int NV = Dims<NDIM>::NV;
    const size_t ncell = (size_t)T.ncell;
    const int total = P.ncells + P.nextra_prim;
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * 32; base < total; base += nwarps * 32) {
        const int t = (int)(base + lane);
        unsigned long long best = ~0ULL;
        int box = -1;
        if (t < total) {
            int id = (t < P.ncells) ? cell_of(T, P, t) : P.xprim[t - P.ncells];
            double u[NV], q[NV];
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) u[iv] = uold[(size_t)iv * ncell + id - 1];
            ctoprim<NDIM>(u, q, gamma, smalle);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) prim[(size_t)iv * ncell + id - 1] = q[iv];
            if (t < P.ncells && T.son[id - 1] == 0) {
                box = box_of(P, t);
                unsigned long long b;
                if (cfl_candidate<NDIM>(u, P.boxes[box].dx, gamma, cfl, pressure_cap, &b)) best = b;
            }
        }
        // segmented min over runs of equal box in lane order
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long ob = __shfl_down_sync(0xffffffffu, best, o);
            const int obx = __shfl_down_sync(0xffffffffu, box, o);
            if (lane + o < 32 && obx == box && ob < best) best = ob;
        }
        const int prev = __shfl_up_sync(0xffffffffu, box, 1);
        if (box >= 0 && (lane == 0 || prev != box) && best != ~0ULL) atomicMin(&P.boxes[box].dtmin_bits, best);
    }
}

}  // namespace

StepK step_consts(const rg_ctx* c) {
    const rg_params& p = c->params;
    StepK K;
    K.gamma = p.gamma;
    K.smalle = 1e-10 * 1e-10 / p.gamma / (p.gamma - 1.0);
    K.smallp = 1e-10 * 1e-10 / p.gamma;
    K.slope_type = p.slope_type;
    K.interpol_type = p.interpol_type;
    K.interpol_var = p.interpol_var;
    K.exact_niter = p.exact_niter > 0 ? p.exact_niter : 10;
    K.exact_tol = p.exact_tol > 0 ? p.exact_tol : 1e-6;
    K.mlp = (p.riemann == RG_RIEMANN_EXACT && p.exact_guess == RG_GUESS_LEARNED && c->mlp_valid) ? c->d_mlp : nullptr;
    return K;
}

namespace {


template <int NDIM, int RS>
void launch_face_t(rg_ctx* c, const Plan& P, const StepK& K) {
    long long work = (long long)P.ncells * NDIM;
    int block = 128;
    k_face<NDIM, RS><<<grid_for(c, work, block), block, 0, c->stream>>>(
        tree_view(c), P.view(), c->d_prim, c->d_uold, c->d_flux, c->d_status, K, nullptr);
}

template <int NDIM>
void launch_face_n(rg_ctx* c, const Plan& P, const StepK& K) {
    switch (c->params.riemann) {
        case RG_RIEMANN_HLLC: launch_face_t<NDIM, RG_RIEMANN_HLLC>(c, P, K); break;
        case RG_RIEMANN_HLL: launch_face_t<NDIM, RG_RIEMANN_HLL>(c, P, K); break;
        case RG_RIEMANN_EXACT: launch_face_t<NDIM, RG_RIEMANN_EXACT>(c, P, K); break;
        case RG_RIEMANN_ACOUSTIC: launch_face_t<NDIM, RG_RIEMANN_ACOUSTIC>(c, P, K); break;
        default: launch_face_t<NDIM, RG_RIEMANN_LLF>(c, P, K); break;
    }
}

template <int NDIM>
int launch_godunov_t(rg_ctx* c, const Plan& P, bool set_uold, const double* dt_dev, double dx, bool prim_ready) {
    constexpr int NV = NDIM + 2, NS = 2 * NDIM;
    if (P.ncells == 0) return RG_OK;
    // the caller sized the shared flux scratch (ensure_flux) outside any capture:
    // 2*ndim flux slots plus the own flux sum, [*][nvar][ncells]
    if (c->cap_flux < (size_t)(NS + 1) * NV * P.ncells) return set_error(c, RG_ERR_STATE, "flux scratch not sized");
    StepK K = step_consts(c);
    TreeView T = tree_view(c);
    PlanView V = P.view();
    double* fsum = c->d_flux + (size_t)NS * NV * P.ncells;
    cudaEvent_t* E = c->timing ? step_events(c, P.ncells) : nullptr;
    if (E) cudaEventRecord(E[0], c->stream);
    int nprim = P.ncells + P.nextra_prim;
    if (!prim_ready)
        k_prim<NDIM><<<grid_for(c, nprim, 256), 256, 0, c->stream>>>(T, V, c->d_uold, c->d_prim, K.gamma, K.smalle,
                                                                     c->d_status, dt_dev, dx);
    if (E) cudaEventRecord(E[1], c->stream);
    if (int rc = launch_face_tiles(c, P, K, c->d_uold, c->d_prim, c->d_flux, fsum)) return rc;
    if (E) cudaEventRecord(E[2], c->stream);
    double* uold_out = set_uold ? c->d_uold : nullptr;
    launch_fold<NDIM, false, true>(c, P, T, V, c->d_flux, c->d_unew, K.gamma, nullptr, fsum, uold_out);
    if (E) cudaEventRecord(E[3], c->stream);
    return check_cuda(c, cudaGetLastError(), "godunov kernels");
}

template <int NDIM, int RS>
void launch_face_ext_t(rg_ctx* c, const Plan& P, const StepK& K, const double* uold, const double* prim,
                       double* flux) {
    long long work = (long long)P.ncells * NDIM;
    k_face<NDIM, RS><<<grid_for(c, work, 128), 128, 0, c->stream>>>(tree_view(c), P.view(), prim, uold, flux,
                                                                     c->d_status, K, nullptr);
}

// Same kernels as launch_godunov_t, on caller-given state, primitive and flux
// buffers (used by the entry point whose flux scratch is a static array).
template <int NDIM>
int launch_godunov_ext_t(rg_ctx* c, const Plan& P, const double* uold, double* unew, double* prim, double* flux) {
    if (P.ncells == 0) return RG_OK;
    StepK K = step_consts(c);
    TreeView T = tree_view(c);
    PlanView V = P.view();
    int nprim = P.ncells + P.nextra_prim;
    k_prim<NDIM><<<grid_for(c, nprim, 256), 256, 0, c->stream>>>(T, V, uold, prim, K.gamma, K.smalle);
    switch (c->params.riemann) {
        case RG_RIEMANN_HLLC: launch_face_ext_t<NDIM, RG_RIEMANN_HLLC>(c, P, K, uold, prim, flux); break;
        case RG_RIEMANN_HLL: launch_face_ext_t<NDIM, RG_RIEMANN_HLL>(c, P, K, uold, prim, flux); break;
        case RG_RIEMANN_EXACT: launch_face_ext_t<NDIM, RG_RIEMANN_EXACT>(c, P, K, uold, prim, flux); break;
        case RG_RIEMANN_ACOUSTIC: launch_face_ext_t<NDIM, RG_RIEMANN_ACOUSTIC>(c, P, K, uold, prim, flux); break;
        default: launch_face_ext_t<NDIM, RG_RIEMANN_LLF>(c, P, K, uold, prim, flux); break;
    }
    launch_fold<NDIM>(c, P, T, V, flux, unew, K.gamma);
    return check_cuda(c, cudaGetLastError(), "godunov kernels (caller buffers)");
}

}  // namespace

cudaEvent_t* step_events(rg_ctx* c, long long ncells) {
    if (!c->timing_acc) return c->ev;
    if (c->acc_n == c->acc_ev.size()) {
        std::array<cudaEvent_t, 4> e{};
        for (auto& x : e) cudaEventCreate(&x);
        c->acc_ev.push_back(e);
        c->acc_cells.push_back(0);
    }
    c->acc_cells[c->acc_n] = ncells;
    return c->acc_ev[c->acc_n++].data();
}

int launch_godunov(rg_ctx* c, const Plan& P, bool set_uold, const double* dt_dev, double dx, bool prim_ready) {
    if (c->params.ndim == 1) return launch_godunov_t<1>(c, P, set_uold, dt_dev, dx, prim_ready);
    return launch_godunov_t<3>(c, P, set_uold, dt_dev, dx, prim_ready);
}

int launch_godunov_ext(rg_ctx* c, const Plan& P, const double* uold, double* unew, double* prim, double* flux) {
    if (c->params.ndim == 1) return launch_godunov_ext_t<1>(c, P, uold, unew, prim, flux);
    return launch_godunov_ext_t<3>(c, P, uold, unew, prim, flux);
}

// CFL candidates and primitives of a leaf level from uold, into the armed CFL
// word (the first substep, or any substep whose previous one did not prepare
// them).
template <int NDIM>
void launch_leaf_prefix_t(rg_ctx* c, const Plan& P, double dx, int pressure_cap, double cfl) {
    StepK K = step_consts(c);
    TreeView T = tree_view(c);
    PlanView V = P.view();
    const int nprim = P.ncells + P.nextra_prim;
    const double start = c->params.boxlen / 1e-10;
    if (P.nbox > 0) {
        const int bb = (P.nbox + 127) / 128;
        k_box_courant_init<<<bb, 128, 0, c->stream>>>(P.boxes, P.nbox, start);
        k_courant_prim_boxes<NDIM><<<grid_for(c, nprim, 256), 256, 0, c->stream>>>(T, V, c->d_uold, c->d_prim,
                                                                                   K.gamma, K.smalle, cfl,
                                                                                   pressure_cap);
    } else {
        k_courant_init<<<1, 1, 0, c->stream>>>(c->d_status, start);
        k_courant_prim<NDIM><<<grid_for(c, nprim, 256), 256, 0, c->stream>>>(T, V, c->d_uold, c->d_prim,
                                                                             c->d_status, dx, K.gamma, K.smalle,
                                                                             cfl, pressure_cap);
    }
}

// dt from the CFL word, the face step and the fold (the fused fold on levels
// that allow it, which leaves the next substep's CFL word and primitives).
template <int NDIM>
int launch_leaf_core_t(rg_ctx* c, const Plan& P, double dx, int pressure_cap, double cfl) {
    StepK K = step_consts(c);
    TreeView T = tree_view(c);
    PlanView V = P.view();
    const double start = c->params.boxlen / 1e-10;
    if (P.nbox > 0) k_box_dt_finalize<<<(P.nbox + 127) / 128, 128, 0, c->stream>>>(P.boxes, P.nbox, start);
    else k_dt_finalize<<<1, 1, 0, c->stream>>>(c->d_status, dx, start);
    if (c->timing) cudaEventRecord(c->ev[1], c->stream);
    double* fsum = c->d_flux + (size_t)(2 * NDIM) * (NDIM + 2) * P.ncells;
    if (int rc = launch_face_tiles(c, P, K, c->d_uold, c->d_prim, c->d_flux, fsum)) return rc;
    if (c->timing) cudaEventRecord(c->ev[2], c->stream);
    const int g = grid_for(c, P.ntarg, 256);
    if (leaf_fusable(P)) {
        if (P.nbox > 0)
            k_fold_next<NDIM, true><<<g, 256, 0, c->stream>>>(T, V, c->d_flux, c->d_unew, c->d_status, K.gamma,
                                                              K.smalle, c->d_uold, fsum, c->d_prim, dx, cfl,
                                                              pressure_cap);
        else
            k_fold_next<NDIM, false><<<g, 256, 0, c->stream>>>(T, V, c->d_flux, c->d_unew, c->d_status, K.gamma,
                                                               K.smalle, c->d_uold, fsum, c->d_prim, dx, cfl,
                                                               pressure_cap);
    } else {
        launch_fold<NDIM, true, true>(c, P, T, V, c->d_flux, c->d_unew, K.gamma, c->d_uold, fsum);
    }
    if (c->timing) cudaEventRecord(c->ev[3], c->stream);
    return check_cuda(c, cudaGetLastError(), "leaf substep kernels");
}

// Substep of a level without refined cells: CFL + primitives in one pass,
// set_unew/set_uold folded into the fold kernel; on levels whose stencils stay
// inside them the fold also prepares the next substep's CFL word and
// primitives, and the prefix is skipped while they are current (three
// launches instead of five).
int launch_leaf_prefix(rg_ctx* c, const Plan& P, double dx, int pressure_cap, double cfl) {
    if (P.ncells == 0) return RG_OK;
    if (c->timing) cudaEventRecord(c->ev[0], c->stream);
    if (c->params.ndim == 1) launch_leaf_prefix_t<1>(c, P, dx, pressure_cap, cfl);
    else launch_leaf_prefix_t<3>(c, P, dx, pressure_cap, cfl);
    return check_cuda(c, cudaGetLastError(), "leaf substep CFL");
}

int launch_leaf_core(rg_ctx* c, const Plan& P, double dx, int pressure_cap, double cfl) {
    if (P.ncells == 0) return RG_OK;
    if (c->cap_flux < (size_t)(2 * c->params.ndim + 1) * (c->params.ndim + 2) * P.ncells)
        return set_error(c, RG_ERR_STATE, "flux scratch not sized");
    if (c->params.ndim == 1) return launch_leaf_core_t<1>(c, P, dx, pressure_cap, cfl);
    return launch_leaf_core_t<3>(c, P, dx, pressure_cap, cfl);
}

int launch_set_unew(rg_ctx* c, const Plan& P) {
    if (P.ncells == 0) return RG_OK;
    k_copy_level<<<grid_for(c, P.ncells, 256), 256, 0, c->stream>>>(tree_view(c), P.view(), c->nvar, c->d_uold,
                                                                     c->d_unew, 0);
    return check_cuda(c, cudaGetLastError(), "set_unew");
}

int launch_set_uold(rg_ctx* c, const Plan& P) {
    if (P.ncells == 0) return RG_OK;
    k_copy_level<<<grid_for(c, P.ncells, 256), 256, 0, c->stream>>>(tree_view(c), P.view(), c->nvar, c->d_unew,
                                                                     c->d_uold, 1);
    return check_cuda(c, cudaGetLastError(), "set_uold");
}

int launch_courant(rg_ctx* c, const Plan& P, double dx, int pressure_cap, double cfl, bool set_unew, bool armed,
                   const ClockStep* clock, bool with_prim) {
    double start = c->params.boxlen / 1e-10;
    if (!armed) k_courant_init<<<1, 1, 0, c->stream>>>(c->d_status, start);
    const ClockStep cs = clock ? *clock : ClockStep{};
    if (P.ncells > 0) {
        double* copy = set_unew ? c->d_unew : nullptr;
        double* prim = with_prim ? c->d_prim : nullptr;
        const long long work = with_prim ? (long long)P.ncells + P.nextra_prim : P.ncells;
        const StepK K = step_consts(c);
        if (c->params.ndim == 1)
            k_courant<1><<<grid_for(c, work, 256), 256, 0, c->stream>>>(tree_view(c), P.view(), c->d_uold,
                                                                        c->d_status, dx, c->params.gamma, cfl,
                                                                        pressure_cap, copy, cs, prim, K.smalle);
        else
            k_courant<3><<<grid_for(c, work, 256), 256, 0, c->stream>>>(tree_view(c), P.view(), c->d_uold,
                                                                        c->d_status, dx, c->params.gamma, cfl,
                                                                        pressure_cap, copy, cs, prim, K.smalle);
    } else if (cs.ck) {
        k_clock_step<<<1, 1, 0, c->stream>>>(c->d_status, cs);
    }
    return check_cuda(c, cudaGetLastError(), "courant");
}

int launch_finalize_dt(rg_ctx* c, double dx) {
    k_dt_finalize<<<1, 1, 0, c->stream>>>(c->d_status, dx, c->params.boxlen / 1e-10);
    return check_cuda(c, cudaGetLastError(), "dt finalize");
}

int launch_set_dt_host(rg_ctx* c, double dt, double dx) {
    k_dt_set<<<1, 1, 0, c->stream>>>(c->d_status, dt, dx);
    return check_cuda(c, cudaGetLastError(), "dt set");
}

int launch_set_dt_device(rg_ctx* c, const double* dt, double dx) {
    k_dt_set_dev<<<1, 1, 0, c->stream>>>(c->d_status, dt, dx);
    return check_cuda(c, cudaGetLastError(), "dt set (device)");
}

// ---------------------------------------------------------------- small-level runs
// rg_level_run on a small level (at most kRunBlockCells cells): the whole
// loop in ONE block of one kernel.  Each substep is the fused leaf substep of
// the three kernels above with block barriers in place of kernel boundaries:
// dt from the CFL word (re-armed), every cell's fluxes and own flux sum (the
// per-(cell, direction) work of k_face_tiles, same functions, same order),
// then every target's ordered fold with the next primitives and CFL
// candidates (k_fold_next), then the clock.  Global writes of one phase are
// visible to the whole block after the barrier, and only one block exists,
// so nothing waits across blocks; max_steps bounds the loop.
namespace {

constexpr int kRunBlock = 512;

template <int NDIM, int RS>
__global__ void __launch_bounds__(kRunBlock) k_level_run_block(TreeView T, PlanView P, double* __restrict__ uold,
                                                              double* __restrict__ unew, double* __restrict__ prim,
                                                              double* __restrict__ flux, double* __restrict__ fsum,
                                                              DevStatus* st, StepK K, double dx, double cfl,
                                                              int pressure_cap, double dt_start, double t_end,
                                                              long long max_steps) {
    constexpr int NV = Dims<NDIM>::NV, NS = Dims<NDIM>::NS;
    const size_t ncell = (size_t)T.ncell;
    const int nc = P.ncells, nt = P.ntarg;
    __shared__ int s_go;
    __shared__ unsigned long long s_best;
    unsigned long long iters = 0, calls = 0;
    for (long long guard = 0; guard < max_steps; ++guard) {
        if (threadIdx.x == 0) {
            set_step_values(st, __longlong_as_double((long long)st->dtmin_bits), dx);
            st->dtmin_bits = (unsigned long long)__double_as_longlong(dt_start);
            s_best = ~0ULL;
        }
        __syncthreads();
        const double dt = st->dt;
        const DxDiv D{st->dx, st->inv_dx, st->dx_pow2 != 0};
        // fluxes and own flux sums
        for (int p = threadIdx.x; p < nc; p += blockDim.x) {
            const int c = cell_of(T, P, p);
            double fs[NV];
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) fs[iv] = 0.0;
            bool any = false;
#pragma unroll 1
            for (int idim = 0; idim < NDIM; ++idim) {
                const int s0 = 2 * idim;
                const int kd0 = P.kind[(size_t)s0 * nc + p];
                if (kd0 == K_NONE) continue;
                any = true;
                const int kd1 = P.kind[(size_t)(s0 + 1) * nc + p];
                double qc[NV], qmo[NV], qpo[NV], ql[NV], qr[NV];
                load_rot<NDIM>(prim, ncell, c, idim, qc);
                const int l = P.icn[(size_t)s0 * nc + p], rr = P.icn[(size_t)(s0 + 1) * nc + p];
                load_nb_rot<NDIM>(T, prim, ncell, l, idim, qc, ql);
                load_nb_rot<NDIM>(T, prim, ncell, rr, idim, qc, qr);
                own_trace<NDIM>(qc, ql, qr, dt, D, K, qmo, qpo);
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
                        neighbour_face<NDIM>(T, P, prim, uold, ncell, p, c, idim, side, kd, n, qc, nullptr, dt, D, K,
                                             qf);
                        if (side == 0) iters += riemann<NDIM, RS>(qf, qpo, f, K);
                        else iters += riemann<NDIM, RS>(qmo, qf, f, K);
                        ++calls;
                        rot_swap<NDIM>(f, idim);
                    }
                    const double sign = side ? -1.0 : 1.0;
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) {
                        flux[((size_t)s * NV + iv) * nc + p] = f[iv];
                        fs[iv] = fs[iv] + sign * f[iv];
                    }
                }
            }
            if (any)
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) fsum[(size_t)iv * nc + p] = fs[iv];
        }
        __syncthreads();
        // ordered fold, next primitives and CFL candidates
        unsigned long long best = ~0ULL;
        for (int t = threadIdx.x; t < nt; t += blockDim.x) {
            const int a = P.toff[t], b = P.toff[t + 1];
            const int cell = cell_of(T, P, t);
            double u[NV], q[NV];
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) u[iv] = uold[(size_t)iv * ncell + cell - 1];
            if (a < b) {
                fold_events<NDIM, true, true>(P, a, b, flux, fsum, K.gamma, st->dtdx, u);
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) {
                    unew[(size_t)iv * ncell + cell - 1] = u[iv];
                    uold[(size_t)iv * ncell + cell - 1] = u[iv];
                }
            }
            ctoprim<NDIM>(u, q, K.gamma, K.smalle);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) prim[(size_t)iv * ncell + cell - 1] = q[iv];
            if (T.son[cell - 1] == 0) {
                unsigned long long bits;
                if (cfl_candidate<NDIM>(u, dx, K.gamma, cfl, pressure_cap, &bits) && bits < best) best = bits;
            }
        }
        if (best != ~0ULL) atomicMin(&s_best, best);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_best != ~0ULL) atomicMin(&st->dtmin_bits, s_best);
            st->run_t = st->run_t + dt;
            st->run_steps += 1;
            s_go = (st->run_t < t_end && st->run_steps < max_steps) ? 1 : 0;
        }
        __syncthreads();
        if (!s_go) break;
    }
    if (RS == RG_RIEMANN_EXACT) {
        if (calls) {
            atomicAdd(&st->exact_iters, iters);
            atomicAdd(&st->exact_calls, calls);
        }
    }
}

template <int NDIM>
int launch_run_block_t(rg_ctx* c, const Plan& P, double dx, int pressure_cap, double t_end, long long max_steps) {
    StepK K = step_consts(c);
    const double start = c->params.boxlen / 1e-10, cfl = c->params.courant_factor;
    double* fsum = c->d_flux + (size_t)(2 * NDIM) * (NDIM + 2) * P.ncells;
#define RG_RUN_ARGS                                                                                                  \
    tree_view(c), P.view(), c->d_uold, c->d_unew, c->d_prim, c->d_flux, fsum, c->d_status, K, dx, cfl, pressure_cap, \
        start, t_end, max_steps
    switch (c->params.riemann) {
        case RG_RIEMANN_HLLC: k_level_run_block<NDIM, RG_RIEMANN_HLLC><<<1, kRunBlock, 0, c->stream>>>(RG_RUN_ARGS); break;
        case RG_RIEMANN_HLL: k_level_run_block<NDIM, RG_RIEMANN_HLL><<<1, kRunBlock, 0, c->stream>>>(RG_RUN_ARGS); break;
        case RG_RIEMANN_EXACT: k_level_run_block<NDIM, RG_RIEMANN_EXACT><<<1, kRunBlock, 0, c->stream>>>(RG_RUN_ARGS); break;
        case RG_RIEMANN_ACOUSTIC:
            k_level_run_block<NDIM, RG_RIEMANN_ACOUSTIC><<<1, kRunBlock, 0, c->stream>>>(RG_RUN_ARGS);
            break;
        default: k_level_run_block<NDIM, RG_RIEMANN_LLF><<<1, kRunBlock, 0, c->stream>>>(RG_RUN_ARGS); break;
    }
#undef RG_RUN_ARGS
    return check_cuda(c, cudaGetLastError(), "small-level run kernel");
}

}  // namespace

int launch_run_block(rg_ctx* c, const Plan& P, double dx, int pressure_cap, double t_end, long long max_steps) {
    if (c->params.ndim == 1) return launch_run_block_t<1>(c, P, dx, pressure_cap, t_end, max_steps);
    return launch_run_block_t<3>(c, P, dx, pressure_cap, t_end, max_steps);
}

}  // namespace rg
