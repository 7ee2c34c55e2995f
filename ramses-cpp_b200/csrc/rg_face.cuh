// rg_face.cuh -- device helpers of the face step shared by the face kernels.
//
// Face states and fluxes of HydroSolver::godunov_fine (RAMSES-CPP
// src/solvers/hydro/HydroSolver.cpp:93-474) on rotated primitive states: the
// cell's own MUSCL-Hancock trace (compute_slopes + trace, :653-732), the
// neighbour's face state by the ghost (:162-453), same-level (:148-161) or
// boundary (:130-145) branch, and the Riemann solver selected at :456-461.
#pragma once

#include "rg_internal.cuh"
#include "rg_physics.cuh"

namespace rg {

struct StepK {
    double gamma, smalle, smallp;
    int slope_type, interpol_type, interpol_var, exact_niter;
    double exact_tol;
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

template <int NDIM, int RS>
__device__ __forceinline__ int riemann(const double* ql, const double* qr, double* f, const StepK& K) {
    if constexpr (RS == RG_RIEMANN_HLLC) solve_hllc<NDIM>(ql, qr, f, K.gamma, K.smallp);
    else if constexpr (RS == RG_RIEMANN_HLL) solve_hll<NDIM>(ql, qr, f, K.gamma);
    else if constexpr (RS == RG_RIEMANN_ACOUSTIC) solve_acoustic<NDIM>(ql, qr, f, K.gamma, K.smallp);
    else if constexpr (RS == RG_RIEMANN_EXACT) return solve_exact<NDIM>(ql, qr, f, K.gamma, K.smallp, K.exact_niter, K.exact_tol, -1.0);
    else solve_llf<NDIM>(ql, qr, f, K.gamma);
    return 0;
}

// Face state of the neighbour across slot (idim, side), rotated.  Writes the
// state the Riemann problem needs: the neighbour's right-face state (qm) for
// side 0, its left-face state (qp) for side 1.
template <int NDIM>
__device__ __forceinline__ void neighbour_face(const TreeView& T, const PlanView& P, const double* __restrict__ prim,
                                               const double* __restrict__ uold, size_t ncell, int p, int c, int idim,
                                               int side, int kd, int n, const double* qc, double dt,
                                               const DxDiv& D, const StepK& K, double* qf) {
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
        if (P.level0) {
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
                double qn[NV], qnl[NV], qnr[NV];
                load_rot<NDIM>(prim, ncell, n, idim, qn);
                load_nb_rot<NDIM>(T, prim, ncell, nl, idim, qn, qnl);
                load_nb_rot<NDIM>(T, prim, ncell, nr, idim, qn, qnr);
                if (kind == K_GHOST) ghost_trace<NDIM>(qn, qnl, qnr, dt, D, K, qm, qp);
                else own_trace<NDIM>(qn, qnl, qnr, dt, D, K, qm, qp);
            }
        have_face:;
        }
    }
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) qf[iv] = side == 0 ? qm[iv] : qp[iv];
}

StepK step_consts(const rg_ctx* c);
int launch_face_tiles(rg_ctx* c, const Plan& P, const StepK& K, const double* uold, const double* prim,
                      double* flux, double* fsum);
int autotune_face(rg_ctx* c, Plan& P, const StepK& K);

}  // namespace rg
