// rg_fold.cuh -- the ordered update of one target cell and the CFL candidate
// of one cell, used by the fold kernels and the small-level run kernel
// (rg_step.cu).
#pragma once

#include "rg_face.cuh"
#include "rg_internal.cuh"
#include "rg_physics.cuh"

namespace rg {
namespace {

// The ordered updates of one target (HydroSolver.cpp:476-547): refluxes from
// neighbours and the cell's own flux-sum update with its clamps, applied in
// the CPU loop order to u (the target's starting state).
// FSUM: the face kernel stored each cell's own flux sum (fsum [nvar][ncells]),
// so the own update reads it instead of re-adding the 2*ndim slots.
// Own update with its clamps (HydroSolver.cpp:485-547).
template <int NDIM>
__device__ __forceinline__ void own_update(const double* fs, double gamma, double dtdx, double* u) {
    constexpr int NV = Dims<NDIM>::NV;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) u[iv] = u[iv] + dtdx * fs[iv];
    double d = sclamp(u[0], 1e-10, 1e6);
    u[0] = d;
#pragma unroll
    for (int i = 1; i <= NDIM; ++i) u[i] = sclamp(u[i], -d * 10.0, d * 10.0);
    double v2 = 0.0;
#pragma unroll
    for (int i = 1; i <= NDIM; ++i) {
        double v = u[i] / d;
        v2 = v2 + v * v;
    }
    constexpr int IE = NDIM + 1;
    double ei = u[IE] - 0.5 * d * v2;
    if (ei < d * 1e-10 / (gamma - 1.0)) {
        double e_non = 0;
        u[IE] = d * 1e-10 / (gamma - 1.0) + 0.5 * d * v2 + e_non;
    }
    u[IE] = smin(u[IE], d * 1e8);
}

// BATCH: fetch all events' values before applying them (more loads in flight
// per thread).  It pays on a single grid; on a 43M-cell ensemble, with a
// 12 GB flux scratch, 35 planes in flight per warp measured slower.
template <int NDIM, bool FSUM, bool BATCH = true>
__device__ __forceinline__ void fold_events(const PlanView& P, int a, int b, const double* __restrict__ flux,
                                            const double* __restrict__ fsum, double gamma, double dtdx, double* u) {
    constexpr int NV = Dims<NDIM>::NV, NS = Dims<NDIM>::NS, TTD = Dims<NDIM>::TTD;
    const int nc = P.ncells;
    const double factor = 1.0 / (1 << NDIM);
    if (BATCH && FSUM && b - a == NS + 1) {
        // a cell with all 2*ndim neighbours refluxing into it and its own
        // update (every cell of a uniform level): fetch every event's values
        // first, then apply them in the same order with the same arithmetic
        double v[NS + 1][NV];
        int slots[NS + 1];
#pragma unroll
        for (int e = 0; e <= NS; ++e) {
            const int key = P.tev[a + e];
            const int slot = key & 7, cp = key >> 3;
            const int ps = P.level0 ? cp : (cp % TTD) * P.noct + cp / TTD;
            slots[e] = slot;
            const double* src = slot == OWN_SLOT ? fsum + ps : flux + (size_t)slot * NV * nc + ps;
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) v[e][iv] = src[(size_t)iv * nc];
        }
#pragma unroll
        for (int e = 0; e <= NS; ++e) {
            if (slots[e] == OWN_SLOT) {
                own_update<NDIM>(v[e], gamma, dtdx, u);
            } else {
                const double sign = (slots[e] & 1) ? -1.0 : 1.0;
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) u[iv] = u[iv] - dtdx * sign * v[e][iv] * factor;
            }
        }
        return;
    }
    int e = a;
    if constexpr (FSUM && NDIM == 3) {
        // four events at a time: their values are fetched together, then
        // applied one by one in event order with the same arithmetic
        constexpr int C = 4;
        for (; e + C <= b; e += C) {
            double v[C][NV];
            int slots[C];
#pragma unroll
            for (int j = 0; j < C; ++j) {
                const int key = P.tev[e + j];
                const int slot = key & 7, cp = key >> 3;
                const int ps = P.level0 ? cp : (cp % TTD) * P.noct + cp / TTD;
                slots[j] = slot;
                const double* src = slot == OWN_SLOT ? fsum + ps : flux + (size_t)slot * NV * nc + ps;
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) v[j][iv] = src[(size_t)iv * nc];
            }
#pragma unroll
            for (int j = 0; j < C; ++j) {
                if (slots[j] == OWN_SLOT) {
                    own_update<NDIM>(v[j], gamma, dtdx, u);
                } else {
                    const double sign = (slots[j] & 1) ? -1.0 : 1.0;
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) u[iv] = u[iv] - dtdx * sign * v[j][iv] * factor;
                }
            }
        }
    }
    for (; e < b; ++e) {
        int key = P.tev[e];
        int slot = key & 7, cp = key >> 3;
        int ps = P.level0 ? cp : (cp % TTD) * P.noct + cp / TTD;
        if (slot == OWN_SLOT) {
            double fs[NV];
            if constexpr (FSUM) {
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) fs[iv] = fsum[(size_t)iv * nc + ps];
            } else {
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) fs[iv] = 0.0;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    double sign = (s & 1) ? -1.0 : 1.0;
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) fs[iv] = fs[iv] + sign * flux[((size_t)s * NV + iv) * nc + ps];
                }
            }
            own_update<NDIM>(fs, gamma, dtdx, u);
        } else {
            double sign = (slot & 1) ? -1.0 : 1.0;
#pragma unroll
            for (int iv = 0; iv < NV; ++iv)
                u[iv] = u[iv] - dtdx * sign * flux[((size_t)slot * NV + iv) * nc + ps] * factor;
        }
    }
}

// CFL candidate of one cell from its conservative state, the reference
// formula (HydroSolver::compute_courant_step, HydroSolver.cpp:878-977) with or
// without its p <= 100 rho cap; negative or NaN candidates are not returned
// (flag false), matching std::min's NaN fall-through.
template <int NDIM>
__device__ __forceinline__ bool cfl_candidate(const double* u, double dx, double gamma, double cfl, int pressure_cap,
                                              unsigned long long* bits) {
    double d = smax(u[0], 1e-10), v2 = 0.0;
#pragma unroll
    for (int i = 1; i <= NDIM; ++i) {
        double v = u[i] / d;
        v2 = v2 + v * v;
    }
    double e_non = 0.0;
    double pr = smax((u[NDIM + 1] - 0.5 * d * v2 - e_non) * (gamma - 1.0), d * 1e-10);
    if (pressure_cap) pr = smin(pr, d * 1e2);
    // The reference adds sum_gamma_p / d with sum_gamma_p = 0 (no non-thermal
    // energies): +0 leaves cs2 unchanged (cs2 > 0, or NaN stays NaN).
    double cs2 = cs2_of(d, pr, gamma);
    double cs = sqrt(smax(cs2, 1e-10));
    double u_wave = NDIM * cs;
#pragma unroll
    for (int i = 1; i <= NDIM; ++i) u_wave = u_wave + fabs(u[i] / d);
    // alpha = max(a_grav dx / u_wave^2, 1e-4) with a_grav = 0 (no gravity) is
    // exactly 1e-4 when dx is finite and u_wave^2 > 0; the sqrt term then
    // depends on cfl alone.  Other cases take the literal formula.
    const double uw2 = u_wave * u_wave;
    double alpha, sq;
    if (isfinite(dx) && uw2 > 0.0) {
        alpha = 0.0001;
        sq = sqrt(1.0 + 2.0 * cfl * 0.0001) - 1.0;
    } else {
        const double a_grav = 0.0;
        alpha = smax(a_grav * dx / uw2, 0.0001);
        sq = sqrt(1.0 + 2.0 * cfl * alpha) - 1.0;
    }
    double dtc = (dx / u_wave) * sq / alpha;
    *bits = (unsigned long long)__double_as_longlong(dtc);
    return dtc >= 0.0;
}

}  // namespace
}  // namespace rg
