// rg_physics.cuh -- per-cell and per-interface physics of the Godunov step.
//
// Device restatement of the reference's arithmetic (paths relative to the
// RAMSES-CPP tree):
//   ctoprim            src/solvers/hydro/HydroSolver.cpp:613-651
//   compute_slope      src/solvers/hydro/SlopeLimiter.cpp:7-60
//   trace              src/solvers/hydro/HydroSolver.cpp:680-732
//   ghost slopes       src/solvers/hydro/HydroSolver.cpp:357-440 (2D/3D), 219-356 (1D)
//   Riemann solvers    src/solvers/hydro/RiemannSolver.cpp:15-427
//   get_cs2            src/solvers/physics/EquationOfState.cpp:26-51
// Every expression keeps the reference's association order and min/max tie
// rules.  The library is compiled with -fmad=false, so no multiply-add is
// contracted and every IEEE operation rounds exactly as the x86-64 g++ -O3
// build of the reference (which has no FMA without -march).  Division and
// square root are the correctly rounded IEEE operations in both; only pow()
// (exact solver) differs by at most a few ulp between libm and CUDA.
#pragma once

#include <math_constants.h>

#include <cuda_runtime.h>

namespace rg {

// std::max / std::min / std::clamp semantics: first argument wins ties and
// NaN comparisons fall through exactly as in libstdc++.
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smin3(double a, double b, double c) {
    double m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    return m;
}
__device__ __forceinline__ double sclamp(double v, double lo, double hi) {
    return (v < lo) ? lo : ((hi < v) ? hi : v);
}

template <int NDIM>
struct Dims {
    static constexpr int NV = NDIM + 2;  // rho, momenta/velocities, energy/pressure
    static constexpr int IP = NDIM + 1;  // pressure / energy index
    static constexpr int TTD = 1 << NDIM;
    static constexpr int NS = 2 * NDIM;  // interface slots per cell
};

// Exchange element 1 (the normal velocity slot) with element 1+idim using
// compile-time indices only, so the state arrays stay in registers.
template <int NDIM>
__device__ __forceinline__ void rot_swap(double* q, int idim) {
    if constexpr (NDIM >= 2) {
        if (idim == 1) {
            double t = q[1];
            q[1] = q[2];
            q[2] = t;
        }
    }
    if constexpr (NDIM >= 3) {
        if (idim == 2) {
            double t = q[1];
            q[1] = q[3];
            q[3] = t;
        }
    }
}

// Division by the cell size.  When dx is a power of two (the usual
// boxlen / (nx 2^L) with power-of-two nx and boxlen), x / dx and x * (1/dx)
// are the same correctly rounded value of the same real number for every x,
// so the multiply replaces the divide without changing a bit.
struct DxDiv {
    double dx, inv;
    bool pow2;
    __device__ __forceinline__ double div(double x) const { return pow2 ? x * inv : x / dx; }
};

__device__ __forceinline__ bool is_pow2_with_normal_inverse(double dx, double inv) {
    unsigned long long b = (unsigned long long)__double_as_longlong(dx);
    unsigned long long bi = (unsigned long long)__double_as_longlong(inv);
    unsigned e = (unsigned)((b >> 52) & 0x7ff), ei = (unsigned)((bi >> 52) & 0x7ff);
    return dx > 0.0 && (b & 0xfffffffffffffULL) == 0 && e != 0 && e != 0x7ff && ei != 0 && ei != 0x7ff;
}

__device__ __forceinline__ double cs2_of(double d, double p, double gamma) {
    double cs2 = gamma * p;
    return smax(cs2 / smax(d, 1e-10), 1e-20);
}

// Conservative -> primitive.  smalle is a per-call constant
// (1e-10*1e-10/gamma/(gamma-1)) computed once by the caller with the same
// operation order.
template <int NDIM>
__device__ __forceinline__ void ctoprim(const double* u, double* q, double gamma, double smalle) {
    constexpr int IP = Dims<NDIM>::IP;
    double d = smax(u[0], 1e-10);
    q[0] = d;
    double oneoverrho = 1.0 / d;
    double eken = 0.0;
#pragma unroll
    for (int i = 1; i <= NDIM; ++i) {
        q[i] = u[i] * oneoverrho;
        eken = eken + 0.5 * q[i] * q[i];
    }
    double erad = 0.0;
    double eint = smax(u[IP] * oneoverrho - eken - erad, smalle);
    q[IP] = (gamma - 1.0) * d * eint;
}

__device__ __forceinline__ double compute_slope(double ql, double qc, double qr, int slope_type, double theta,
                                                double nu) {
    if (slope_type == 0) return 0.0;
    double dlft = qc - ql;
    double drgt = qr - qc;
    if (slope_type == 4 || slope_type == 5) {
        double dlft_s, drgt_s;
        if (slope_type == 4) {
            dlft_s = 2.0 / (1.0 + nu) * dlft;
            drgt_s = 2.0 / (1.0 - nu) * drgt;
        } else if (nu >= 0.0) {
            dlft_s = 2.0 / (nu + 1e-10) * dlft;
            drgt_s = 2.0 / (1.0 - nu) * drgt;
        } else {
            dlft_s = 2.0 / (1.0 + nu) * dlft;
            drgt_s = 2.0 / (-nu + 1e-10) * drgt;
        }
        double dcen = 0.5 * (dlft + drgt);
        double dsgn = (dcen >= 0.0) ? 1.0 : -1.0;
        double dlim = smin(fabs(dlft_s), fabs(drgt_s));
        if (dlft * drgt <= 0.0) dlim = 0.0;
        return dsgn * dlim;
    }
    if (slope_type == 6) return 0.5 * (dlft + drgt);
    if (dlft * drgt <= 0.0) return 0.0;
    double dcen = 0.5 * (dlft + drgt);
    double dsgn = (dcen >= 0.0) ? 1.0 : -1.0;
    double dlim;
    if (slope_type == 1) dlim = smin(fabs(dlft), fabs(drgt));
    else if (slope_type == 2 || slope_type == 3) dlim = smin3(2.0 * fabs(dlft), 2.0 * fabs(drgt), fabs(dcen));
    else if (slope_type == 7) dlim = 2.0 * fabs(dlft) * fabs(drgt) / (fabs(dlft) + fabs(drgt));
    else if (slope_type == 8) dlim = smin3(theta * fabs(dlft), theta * fabs(drgt), fabs(dcen));
    else dlim = smin(fabs(dlft), fabs(drgt));
    return dsgn * dlim;
}

// Interpolation slope of the ghost branch (types 1 minmod/2, 2 moncen/4-style,
// 3 central/4; anything else gives 0).
__device__ __forceinline__ double interp_slope(double dlft, double drgt, int itype) {
    double sgn = (dlft >= 0.0) ? 1.0 : -1.0;
    if (itype == 1) return sgn * 0.5 * smin(fabs(dlft), fabs(drgt));
    if (itype == 2) return sgn * smin3(fabs(dlft), fabs(drgt), 0.25 * fabs(dlft + drgt));
    if (itype == 3) return 0.25 * (dlft + drgt);
    return 0.0;
}

// MUSCL-Hancock predictor on a rotated state (normal velocity at index 1).
template <int NDIM>
__device__ __forceinline__ void trace(const double* q, const double* dq, double dt, double dx, double* qm,
                                      double* qp, double gamma) {
    constexpr int NV = Dims<NDIM>::NV, IP = Dims<NDIM>::IP;
    double r = smax(q[0], 1e-10), u = q[1], p = smax(q[IP], r * 1e-20);
    double sr0 = -u * dq[0] - dq[1] * r;
    double su0 = -u * dq[1] - dq[IP] / r;
    double cs2 = cs2_of(r, p, gamma);
    double sp0 = -u * dq[IP] - dq[1] * r * cs2;
    double hdx = 0.5 * dx, hdt = 0.5 * dt;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
        double dqi = dq[iv];
        double dq_dt = 0;
        if (iv == 0) dq_dt = sr0;
        else if (iv == 1) dq_dt = su0;
        else if (iv == IP) dq_dt = sp0;
        double a = hdx * dqi, b = hdt * dq_dt;
        qp[iv] = q[iv] - a + b;
        qm[iv] = q[iv] + a + b;
        if (iv == 0) {
            if (qp[iv] < 1e-10) qp[iv] = r;
            if (qm[iv] < 1e-10) qm[iv] = r;
        }
    }
}

template <int NDIM>
__device__ __forceinline__ void compute_flux(const double* q, double* f, double gamma) {
    constexpr int IP = Dims<NDIM>::IP;
    double rho = q[0], u = q[1], p = q[IP];
    double v2 = 0;
#pragma unroll
    for (int i = 1; i <= NDIM; ++i) v2 = v2 + q[i] * q[i];
    double e_kin = 0.5 * rho * v2;
    double e_int = p / (gamma - 1.0);
    double E = e_kin + e_int + 0.0;
    f[0] = rho * u;
    f[1] = rho * u * u + p;
#pragma unroll
    for (int i = 2; i <= NDIM; ++i) f[i] = rho * u * q[i];
    f[IP] = (E + p) * u;
}

template <int NDIM>
__device__ __forceinline__ void prim_to_cons(const double* q, double* u, double gamma) {
    constexpr int IP = Dims<NDIM>::IP;
    u[0] = q[0];
    double v2 = 0;
#pragma unroll
    for (int i = 1; i <= NDIM; ++i) {
        u[i] = q[0] * q[i];
        v2 = v2 + q[i] * q[i];
    }
    double e_kin = 0.5 * q[0] * v2;
    double e_int = q[IP] / (gamma - 1.0);
    u[IP] = e_kin + e_int + 0.0;
}

template <int NDIM>
__device__ __forceinline__ void solve_llf(const double* ql, const double* qr, double* flux, double gamma) {
    constexpr int NV = Dims<NDIM>::NV, IP = Dims<NDIM>::IP;
    double fl[NV], fr[NV], ul[NV], ur[NV];
    compute_flux<NDIM>(ql, fl, gamma);
    compute_flux<NDIM>(qr, fr, gamma);
    prim_to_cons<NDIM>(ql, ul, gamma);
    prim_to_cons<NDIM>(qr, ur, gamma);
    double al = sqrt(cs2_of(ql[0], ql[IP], gamma));
    double ar = sqrt(cs2_of(qr[0], qr[IP], gamma));
    double a_max = smax(fabs(ql[1]) + al, fabs(qr[1]) + ar);
#pragma unroll
    for (int i = 0; i < NV; ++i) flux[i] = 0.5 * (fl[i] + fr[i]) - 0.5 * a_max * (ur[i] - ul[i]);
}

template <int NDIM>
__device__ __forceinline__ void solve_hll(const double* ql, const double* qr, double* flux, double gamma) {
    constexpr int NV = Dims<NDIM>::NV, IP = Dims<NDIM>::IP;
    double fl[NV], fr[NV], ul[NV], ur[NV];
    compute_flux<NDIM>(ql, fl, gamma);
    compute_flux<NDIM>(qr, fr, gamma);
    prim_to_cons<NDIM>(ql, ul, gamma);
    prim_to_cons<NDIM>(qr, ur, gamma);
    double al = sqrt(cs2_of(ql[0], ql[IP], gamma));
    double ar = sqrt(cs2_of(qr[0], qr[IP], gamma));
    double sl = smin(0.0, smin(ql[1] - al, qr[1] - ar));
    double sr = smax(0.0, smax(ql[1] + al, qr[1] + ar));
    if (sr - sl < 1e-20) {
#pragma unroll
        for (int i = 0; i < NV; ++i) flux[i] = 0.5 * (fl[i] + fr[i]);
    } else {
        double inv_srs = 1.0 / (sr - sl);
#pragma unroll
        for (int i = 0; i < NV; ++i) flux[i] = (sr * fl[i] - sl * fr[i] + sr * sl * (ur[i] - ul[i])) * inv_srs;
    }
}

// smallp = 1e-10*1e-10/gamma (RiemannSolver.cpp:71) is the same value in every
// call, so the caller computes it once, in the same operation order.
template <int NDIM>
__device__ __forceinline__ void solve_hllc(const double* ql, const double* qr, double* flux, double gamma,
                                           double smallp) {
    constexpr int NV = Dims<NDIM>::NV, IP = Dims<NDIM>::IP;
    double rl = smax(ql[0], 1e-10), ul = ql[1], pl = smax(ql[IP], rl * smallp);
    double rr = smax(qr[0], 1e-10), ur = qr[1], pr = smax(qr[IP], rr * smallp);
    double cl = sqrt(cs2_of(rl, ql[IP], gamma));
    double cr = sqrt(cs2_of(rr, qr[IP], gamma));
    double cmax = smax(cl, cr);
    double sl = smin(ul, ur) - cmax;
    double sr = smax(ul, ur) + cmax;
    if (sl > 0.0) {
        compute_flux<NDIM>(ql, flux, gamma);
        return;
    }
    if (sr < 0.0) {
        compute_flux<NDIM>(qr, flux, gamma);
        return;
    }
    double rcl = rl * (ul - sl);
    double rcr = rr * (sr - ur);
    double div = rcr + rcl;
    if (div < 1e-5) {
        double fa[NV], fb[NV];
        compute_flux<NDIM>(ql, fa, gamma);
        compute_flux<NDIM>(qr, fb, gamma);
#pragma unroll
        for (int i = 0; i < NV; ++i) flux[i] = 0.5 * (fa[i] + fb[i]);
        return;
    }
    double ustar = (rcr * ur + rcl * ul + (pl - pr)) / div;
    ustar = smax(-1e6, smin(1e6, ustar));
    double pstar = (rcr * pl + rcl * pr + rcl * rcr * (ul - ur)) / div;
    pstar = smax(pstar, 0.0);
    // Upwind side: left star state when ustar > 0, else right.
    const bool left = ustar > 0.0;
    const double* qo = left ? ql : qr;
    double ro = left ? rl : rr, uo = left ? ul : ur, po = left ? pl : pr, so = left ? sl : sr;
    double den = left ? smin(sl - ustar, -1e-10) : smax(sr - ustar, 1e-10);
    double rstar = ro * (so - uo) / den;
    double qs[NV];
    qs[0] = rstar;
    qs[1] = ustar;
#pragma unroll
    for (int i = 2; i <= NDIM; ++i) qs[i] = qo[i];
    qs[IP] = smax(pstar - 0.0, rstar * smallp);
    double f0[NV], u0[NV], us[NV];
    compute_flux<NDIM>(qo, f0, gamma);
    prim_to_cons<NDIM>(qo, u0, gamma);
    prim_to_cons<NDIM>(qs, us, gamma);
    us[IP] = ((so - uo) * u0[IP] - po * uo + pstar * ustar) / den;
#pragma unroll
    for (int i = 0; i < NV; ++i) flux[i] = f0[i] + so * (us[i] - u0[i]);
}

template <int NDIM>
__device__ __forceinline__ void solve_acoustic(const double* ql, const double* qr, double* flux, double gamma,
                                               double smallp) {
    constexpr int NV = Dims<NDIM>::NV, IP = Dims<NDIM>::IP;
    const double smallc = 1e-10;
    double rl = smax(ql[0], 1e-10), ul = ql[1], pl = smax(ql[IP], rl * smallp);
    double rr = smax(qr[0], 1e-10), ur = qr[1], pr = smax(qr[IP], rr * smallp);
    double cl = sqrt(cs2_of(rl, ql[IP], gamma));
    double cr = sqrt(cs2_of(rr, qr[IP], gamma));
    double wl = cl * rl, wr = cr * rr;
    double pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr + 1e-20);
    double ustar = ((wr * ur + wl * ul) + (pl - pr)) / (wl + wr + 1e-20);
    double sgnm = (ustar >= 0.0) ? 1.0 : -1.0;
    double ro, uo, po, co;
    if (sgnm == 1.0) { ro = rl; uo = ul; po = pl; co = cl; }
    else { ro = rr; uo = ur; po = pr; co = cr; }
    double rstar = ro + (pstar - po) / smax(co * co, 1e-20);
    rstar = smax(rstar, 1e-10);
    double cstar = sqrt(smax(gamma * pstar / rstar, 1e-20));
    cstar = smax(cstar, smallc);
    double spout = co - sgnm * uo;
    double spin = cstar - sgnm * ustar;
    double ushock = 0.5 * (spin + spout);
    ushock = smax(ushock, -sgnm * ustar);
    if (pstar >= po) { spout = ushock; spin = spout; }
    double rg, ug, pg;
    if (spout < 0.0) { rg = ro; ug = uo; pg = po; }
    else if (spin >= 0.0) { rg = rstar; ug = ustar; pg = pstar; }
    else {
        double frac = spout / (spout - spin + 1e-20);
        rg = frac * rstar + (1.0 - frac) * ro;
        ug = frac * ustar + (1.0 - frac) * uo;
        pg = frac * pstar + (1.0 - frac) * po;
    }
    double qg[NV];
    qg[0] = rg;
    qg[1] = ug;
#pragma unroll
    for (int i = 2; i <= NDIM; ++i) qg[i] = (sgnm == 1.0) ? ql[i] : qr[i];
    qg[IP] = smax(pg - 0.0, rg * smallp);
    compute_flux<NDIM>(qg, flux, gamma);
}

// Exact solver (two-shock Newton iteration, RiemannSolver.cpp:194-307).
// niter/tol default to the reference's 10 and 1e-6; p_guess > 0 replaces the
// initial guess of :215 (learned mode).  Returns the Newton update count.
//
// Converged mode (tol below the reference's 1e-6) safeguards the iteration:
// the function the update zeroes, g(p) = u_L*(p) - u_R*(p) with the
// two-shock mass fluxes W_k(p) = sqrt(gamma p_k rho_k (1 + (gamma+1)/(2 gamma)
// (p - p_k)/p_k)), is continuous, strictly decreasing and convex on p >= 0,
// so every evaluated p tells on which side of the root it lies.  The solver
// keeps that bracket [lo, hi] and replaces a Newton step that leaves it by
// its midpoint (a bracketed Newton-bisection hybrid, the safeguarded Newton
// method of Numerical Recipes, 3rd ed., sec. 9.4 "rtsafe"); it stops as soon
// as a Newton update is below tol relative (the reference's test, taken
// before the bracket so that an update below one ulp still ends the loop) or
// the bracket has closed to tol relative.  Newton is monotone from the left of
// the root, so the bracket only acts after an overshoot from the right and
// where rounding noise in g near an ill-conditioned (near-vacuum) root makes
// the steps wander; then the bracket halves each step and the iteration ends
// well inside the cap.  Reference mode (tol >= 1e-6) runs the reference's
// loop unchanged.
template <int NDIM>
__device__ __forceinline__ int solve_exact_p(const double* ql, const double* qr, double* flux, double gamma,
                                             double smallp, int niter, double tol, double p_guess,
                                             double* pstar_out) {
    constexpr int IP = Dims<NDIM>::IP;
    const double gamma6 = (gamma + 1.0) / (2.0 * gamma);
    double rl = smax(ql[0], 1e-10), ul = ql[1], pl = smax(ql[IP], rl * smallp);
    double rr = smax(qr[0], 1e-10), ur = qr[1], pr = smax(qr[IP], rr * smallp);
    double cl_sq = gamma * pl * rl;
    double cr_sq = gamma * pr * rr;
    double wl = sqrt(smax(cl_sq, 0.0));
    double wr = sqrt(smax(cr_sq, 0.0));
    double pstar = (wr * pl + wl * pr + wl * wr * (ul - ur)) / (wl + wr + 1e-20);
    pstar = smax(pstar, 0.0);
    if (p_guess > 0.0) pstar = p_guess;
    double pold = pstar;
    int it = 0;
    const bool safe = tol < 1e-6;
    double lo = 0.0, hi = CUDART_INF;  // converged mode: g(lo) > 0 > g(hi)
    for (int iter = 0; iter < niter; ++iter) {
        double wwl_sq = cl_sq * (1.0 + gamma6 * (pold - pl) / (pl + 1e-20));
        double wwr_sq = cr_sq * (1.0 + gamma6 * (pold - pr) / (pr + 1e-20));
        double wwl = sqrt(smax(wwl_sq, 0.0));
        double wwr = sqrt(smax(wwr_sq, 0.0));
        // std::pow(w, 3.0) in the reference (RiemannSolver.cpp:226): the cube
        // by two products is as close to glibc's result (a few ulp at most)
        // as CUDA's general pow, at a fraction of its cost
        double ql_nr = (2.0 * (wwl * wwl * wwl)) / (wwl * wwl + cl_sq + 1e-20);
        double qr_nr = (2.0 * (wwr * wwr * wwr)) / (wwr * wwr + cr_sq + 1e-20);
        double usl = ul - (pold - pl) / (wwl + 1e-20);
        double usr = ur + (pold - pr) / (wwr + 1e-20);
        double delp = (qr_nr * ql_nr / (qr_nr + ql_nr + 1e-20)) * (usl - usr);
        delp = smax(delp, -pold);
        ++it;
        if (safe) {
            const double gv = usl - usr;
            if (gv > 0.0) lo = smax(lo, pold);
            else if (gv < 0.0) hi = smin(hi, pold);
            else break;  // g(pold) == 0: the root itself
            // the next point: Newton's (clamped at 0 like the reference's
            // update, which is how a vacuum root p* = 0 is reached) while it
            // stays inside the bracket, else the bracket's midpoint
            double pn = pold + delp;
            if (fabs(delp / (pn + 1e-10)) < tol) {  // the reference's test, on the Newton update
                pold = pn;
                break;
            }
            if (!((pn > lo || pn == 0.0) && pn < hi))
                pn = hi < CUDART_INF ? 0.5 * (lo + hi) : 2.0 * lo + 1e-300;
            pold = pn;
            if (hi - lo <= tol * (lo + 1e-10)) break;
            continue;
        }
        pold = pold + delp;
        if (fabs(delp / (pold + 1e-10)) < tol) break;
    }
    if (safe) {
        // Polish: the converged root truncated to its 30 leading significant
        // bits, then two plain Newton updates from there.  Where the root is
        // ill-conditioned, where it ends inside the search depends on the start
        // by a few ulp, and a flux sampled through a nearly stationary contact
        // magnifies that; from the truncated value the arithmetic no longer
        // depends on the start, so any two starts that converged to within
        // 2^-30 of each other give the same bits.  From 2^-30 the two updates
        // are back at the root's own rounding level.
        pold = __longlong_as_double(__double_as_longlong(pold) & ~((1LL << 22) - 1));
        for (int k = 0; k < 2; ++k) {
            double wwl = sqrt(smax(cl_sq * (1.0 + gamma6 * (pold - pl) / (pl + 1e-20)), 0.0));
            double wwr = sqrt(smax(cr_sq * (1.0 + gamma6 * (pold - pr) / (pr + 1e-20)), 0.0));
            double ql_nr = (2.0 * (wwl * wwl * wwl)) / (wwl * wwl + cl_sq + 1e-20);
            double qr_nr = (2.0 * (wwr * wwr * wwr)) / (wwr * wwr + cr_sq + 1e-20);
            double usl = ul - (pold - pl) / (wwl + 1e-20);
            double usr = ur + (pold - pr) / (wwr + 1e-20);
            double delp = (qr_nr * ql_nr / (qr_nr + ql_nr + 1e-20)) * (usl - usr);
            pold = pold + smax(delp, -pold);
        }
    }
    pstar = pold;
    if (pstar_out) *pstar_out = pstar;
    double wwl_f = sqrt(smax(cl_sq * (1.0 + gamma6 * (pstar - pl) / (pl + 1e-20)), 0.0));
    double wwr_f = sqrt(smax(cr_sq * (1.0 + gamma6 * (pstar - pr) / (pr + 1e-20)), 0.0));
    double ustar = 0.5 * (ul + (pl - pstar) / (wwl_f + 1e-20) + ur - (pr - pstar) / (wwr_f + 1e-20));
    bool left = ustar > 0;
    double ro = left ? rl : rr, po = left ? pl : pr;
    double rstar_val;
    if (pstar >= po) {
        rstar_val = ro * ((gamma + 1.0) * pstar + (gamma - 1.0) * po) / ((gamma - 1.0) * pstar + (gamma + 1.0) * po);
    } else {
        rstar_val = ro * pow(pstar / (po + 1e-20), 1.0 / gamma);
    }
    rstar_val = smax(rstar_val, 1e-10);
    double cl_h = sqrt(cs2_of(rl, pl, gamma));
    double cr_h = sqrt(cs2_of(rr, pr, gamma));
    double cm = smax(cl_h, cr_h);
    double sl_h = smin(ul, ur) - cm;
    double sr_h = smax(ul, ur) + cm;
    double uo;
    if (sl_h > 0.0) { ro = rl; uo = ul; po = pl; }
    else if (sr_h < 0.0) { ro = rr; uo = ur; po = pr; }
    else { ro = rstar_val; uo = ustar; po = pstar; }
    double e_int = po / (gamma - 1.0);
    double e_kin = 0.5 * ro * uo * uo;
#pragma unroll
    for (int i = 2; i <= NDIM; ++i) {
        double vt = left ? ql[i] : qr[i];
        e_kin = e_kin + 0.5 * ro * vt * vt;
    }
    double E = e_int + e_kin;
    flux[0] = ro * uo;
    flux[1] = ro * uo * uo + po;
#pragma unroll
    for (int i = 2; i <= NDIM; ++i) flux[i] = flux[0] * (left ? ql[i] : qr[i]);
    flux[IP] = (E + po) * uo;
    return it;
}

template <int NDIM>
__device__ __forceinline__ int solve_exact(const double* ql, const double* qr, double* flux, double gamma,
                                           double smallp, int niter, double tol, double p_guess) {
    return solve_exact_p<NDIM>(ql, qr, flux, gamma, smallp, niter, tol, p_guess, nullptr);
}

}  // namespace rg
