/*
 * rg_oracle.c -- CPU restatement of RAMSES-CPP's Godunov level step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the B200
 * library: tests, the smoke check and the CPU-baseline leg of the benchmark
 * call it to produce the expected answer.  No product code path links it.
 *
 * It restates, in plain C, the arithmetic and the operation order of the
 * reference's CPU hot path (paths relative to the RAMSES-CPP tree):
 *   src/solvers/hydro/HydroSolver.cpp:18-573   godunov_fine
 *   src/solvers/hydro/HydroSolver.cpp:575-611  set_unew / set_uold
 *   src/solvers/hydro/HydroSolver.cpp:613-732  ctoprim, compute_slopes, trace
 *   src/solvers/hydro/HydroSolver.cpp:878-977  compute_courant_step
 *   src/solvers/hydro/RiemannSolver.cpp        llf, hll, hllc, exact, acoustic
 *   src/solvers/hydro/SlopeLimiter.cpp:7-60    compute_slope
 *   src/solvers/physics/EquationOfState.cpp:26-51  get_cs2 (ideal gas)
 *   src/core/AmrGrid.cpp:389-444,513-550       neighbour lookups
 *   src/core/Constants.cpp:8-43                iii/jjj tables (derived here)
 * Every expression keeps the reference's evaluation order so that, compiled
 * without FMA contraction, results are bit-identical to the reference built
 * the same way.  The pin tests compare it with the reference compiled from its
 * own sources (oracle/_ref) and with committed golden vectors.
 *
 * Supported: ndim 1..3, nvar = ndim+2+npassive, no non-thermal energies, no
 * barotropic EOS, no gravity force (f == 0), nboundary == 0 (the reference
 * never sets boundaries from its namelist, so every run is periodic).
 */
#include "rg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXV 20

/* std::max / std::min / std::clamp semantics (first argument wins ties). */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smin3(double a, double b, double c) {
    double m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    return m;
}
static inline double sclamp(double v, double lo, double hi) {
    return (v < lo) ? lo : ((hi < v) ? hi : v);
}
static inline void swapd(double* a, double* b) { double t = *a; *a = *b; *b = t; }

/* ---------------------------------------------------------------- topology */

/* Neighbour-slot tables.  Constants.cpp:8-43 lists iii/jjj for the 8 cells of
 * an oct; both follow from the cell bit layout ic-1 = ix + 2 iy + 4 iz: the
 * neighbour across direction (idim, side) is the cell with bit idim flipped,
 * in the same oct when that bit points inward, else in neighbour oct
 * 2*idim+side+1. */
int orc_iii(int idim, int inbor, int ic) {
    int bit = ((ic - 1) >> idim) & 1;
    if (inbor == 0) return bit ? 0 : 2 * idim + 1;
    return bit ? 2 * idim + 2 : 0;
}
int orc_jjj(int idim, int ic) { return ((ic - 1) ^ (1 << idim)) + 1; }

void orc_get_nbor_grids(const rg_grid_view* g, int igrid, int ign[7]) {
    ign[0] = igrid;
    for (int i = 1; i <= 6; ++i) {
        int val = g->nbor[(size_t)(i - 1) * g->ngridmax + igrid - 1];
        ign[i] = (val > g->ncell) ? 0 : val;
    }
}

void orc_get_nbor_cells_coarse(const rg_grid_view* g, int icell, int icn[6]) {
    for (int i = 0; i < 6; ++i) icn[i] = 0;
    if (icell <= 0 || icell > g->ncoarse) return;
    int nx = g->nx, ny = g->ny, nz = g->nz;
    int idx = icell - 1;
    int iz = idx / (nx * ny), rem = idx % (nx * ny);
    int iy = rem / nx, ix = rem % nx;
    int n[3] = {nx, ny, nz};
    for (int idim = 0; idim < 3; ++idim) {
        for (int side = 0; side < 2; ++side) {
            int c[3] = {ix, iy, iz};
            c[idim] = (c[idim] + (side == 0 ? -1 : 1) + n[idim]) % n[idim];
            icn[idim * 2 + side] = c[2] * nx * ny + c[1] * nx + c[0] + 1;
        }
    }
}

/* AmrGrid::get_nbor_cells, with the recursion to the father oct unrolled
 * into a loop per direction.  Returns 0 on success, -1 if the father chain
 * is deeper than 64 (a cycle). */
int orc_get_nbor_cells(const rg_grid_view* g, int ndim, const int ign[7], int ic,
                       int icn[6], int igrid) {
    for (int i = 0; i < 6; ++i) icn[i] = 0;
    if (igrid <= 0) return 0;
    for (int idim = 0; idim < ndim; ++idim) {
        for (int inbor = 0; inbor < 2; ++inbor) {
            int cur_igrid = igrid, cur_ic = ic;
            int cur_ign[7];
            memcpy(cur_ign, ign, sizeof(cur_ign));
            int result = 0, depth = 0;
            for (;;) {
                int ig_idx = orc_iii(idim, inbor, cur_ic);
                int ic_pos = orc_jjj(idim, cur_ic);
                int ig = cur_ign[ig_idx];
                if (ig > 0) {
                    if (ig_idx == 0) {
                        result = g->ncoarse + (ic_pos - 1) * g->ngridmax + ig;
                    } else {
                        int ig_child = (ig <= g->ncell) ? g->son[ig - 1] : 0;
                        result = (ig_child > 0) ? g->ncoarse + (ic_pos - 1) * g->ngridmax + ig_child : ig;
                    }
                    break;
                } else if (ig < 0) {
                    result = ig;
                    break;
                }
                int ifather = g->father[cur_igrid - 1];
                if (ifather <= g->ncoarse) {
                    int ifn[6];
                    orc_get_nbor_cells_coarse(g, ifather, ifn);
                    result = ifn[idim * 2 + inbor];
                    break;
                }
                int p_ig = ((ifather - g->ncoarse - 1) % g->ngridmax) + 1;
                int p_ic = ((ifather - g->ncoarse - 1) / g->ngridmax) + 1;
                orc_get_nbor_grids(g, p_ig, cur_ign);
                cur_igrid = p_ig;
                cur_ic = p_ic;
                if (++depth > 64) return -1;
            }
            icn[idim * 2 + inbor] = result;
        }
    }
    return 0;
}

/* Neighbours of an arbitrary cell id (coarse or oct cell), as the ghost
 * branch computes them (HydroSolver.cpp:179-187). */
static int nbor_cells_of(const rg_grid_view* g, int ndim, int id, int icn[6]) {
    if (id <= g->ncoarse) {
        orc_get_nbor_cells_coarse(g, id, icn);
        return 0;
    }
    int ig_p = ((id - g->ncoarse - 1) % g->ngridmax) + 1;
    int ic_p = ((id - g->ncoarse - 1) / g->ngridmax) + 1;
    int ign_p[7];
    orc_get_nbor_grids(g, ig_p, ign_p);
    return orc_get_nbor_cells(g, ndim, ign_p, ic_p, icn, ig_p);
}

/* cell_levels[] of HydroSolver.cpp:22-38: father-chain depth of every cell of
 * an oct that has a father; 0 elsewhere.  Returns -1 on a cyclic chain. */
int orc_cell_levels(const rg_grid_view* g, int ndim, int* cell_levels /* [ncell+1] */) {
    int ttd = 1 << ndim;
    memset(cell_levels, 0, sizeof(int) * ((size_t)g->ncell + 1));
    for (int ig = 1; ig <= g->ngridmax; ++ig) {
        if (g->father[ig - 1] > 0) {
            int level = 1, curr = ig, guard = 0;
            while (curr > 0) {
                int fc = g->father[curr - 1];
                if (fc <= g->ncoarse) break;
                curr = ((fc - g->ncoarse - 1) % g->ngridmax) + 1;
                level++;
                if (++guard > 4096) return -1;
            }
            for (int ic = 1; ic <= ttd; ++ic) cell_levels[g->ncoarse + (ic - 1) * g->ngridmax + ig] = level;
        }
    }
    return 0;
}

int orc_level_octs(const rg_grid_view* g, int ilevel, int* octs, int cap) {
    if (ilevel < 0 || ilevel > g->nlevelmax) return 0;
    int n = 0;
    int ig = g->headl[(size_t)ilevel * (g->ncpu + g->nboundary)];
    while (ig > 0) {
        if (n < cap) octs[n] = ig;
        n++;
        if (n > g->ngridmax) return -1; /* cycle */
        ig = g->next[ig - 1];
    }
    return n;
}

/* ------------------------------------------------------------------ physics */

static inline double cs2_of(double d, double p, double gamma) {
    /* EquationOfState::get_cs2, ideal gas, no non-thermal energies */
    double cs2 = gamma * p;
    return smax(cs2 / smax(d, 1e-10), 1e-20);
}

void orc_ctoprim(const double* u, double* q, double gamma, int ndim, int nvar) {
    const double smallr = 1e-10, smallc = 1e-10;
    double smalle = smallc * smallc / gamma / (gamma - 1.0);
    double d = smax(u[0], smallr);
    q[0] = d;
    double oneoverrho = 1.0 / d;
    double eken = 0.0;
    for (int i = 1; i <= ndim; ++i) {
        q[i] = u[i] * oneoverrho;
        eken += 0.5 * q[i] * q[i];
    }
    int iener = ndim + 1;
    double erad = 0.0;
    double eint = smax(u[iener] * oneoverrho - eken - erad, smalle);
    q[iener] = (gamma - 1.0) * d * eint;
    for (int iv = iener + 1; iv < nvar; ++iv) q[iv] = u[iv] * oneoverrho;
}

double orc_compute_slope(double ql, double qc, double qr, int slope_type, double theta, double nu) {
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

void orc_trace(const double* q, const double* dq, double dt, double dx, double* qm, double* qp,
               double gamma, int ndim, int nvar) {
    double r = smax(q[0], 1e-10), u = q[1], p = smax(q[ndim + 1], r * 1e-20);
    double sr0 = -u * dq[0] - dq[1] * r;
    double su0 = -u * dq[1] - dq[ndim + 1] / r;
    double cs2 = cs2_of(r, p, gamma);
    double sp0 = -u * dq[ndim + 1] - dq[1] * r * cs2;
    for (int iv = 0; iv < nvar; ++iv) {
        double dqi = dq[iv];
        double dq_dt = 0;
        if (iv == 0) dq_dt = sr0;
        else if (iv == 1) dq_dt = su0;
        else if (iv == ndim + 1) dq_dt = sp0;
        qp[iv] = q[iv] - 0.5 * dx * dqi + 0.5 * dt * dq_dt;
        qm[iv] = q[iv] + 0.5 * dx * dqi + 0.5 * dt * dq_dt;
        if (iv == 0) {
            if (qp[iv] < 1e-10) qp[iv] = r;
            if (qm[iv] < 1e-10) qm[iv] = r;
        }
    }
}

static void compute_flux(const double* q, double* f, double gamma, int ndim) {
    double rho = q[0], u = q[1];
    int ip = ndim + 1;
    double p = q[ip];
    double v2 = 0;
    for (int i = 1; i <= ndim; ++i) v2 += q[i] * q[i];
    double e_kin = 0.5 * rho * v2;
    double e_int = p / (gamma - 1.0);
    double e_nonthermal = 0.0;
    double p_tot = p;
    double E = e_kin + e_int + e_nonthermal;
    f[0] = rho * u;
    f[1] = rho * u * u + p_tot;
    for (int i = 2; i <= ndim; ++i) f[i] = rho * u * q[i];
    f[ip] = (E + p_tot) * u;
}

static void prim_to_cons(const double* q, double* u, double gamma, int ndim) {
    u[0] = q[0];
    double v2 = 0;
    for (int i = 1; i <= ndim; ++i) {
        u[i] = q[0] * q[i];
        v2 += q[i] * q[i];
    }
    int ip = ndim + 1;
    double e_kin = 0.5 * q[0] * v2;
    double e_int = q[ip] / (gamma - 1.0);
    double e_nonthermal = 0.0;
    u[ip] = e_kin + e_int + e_nonthermal;
}

void orc_solve_llf(const double* ql, const double* qr, double* flux, double gamma, int ndim) {
    double fl[MAXV], fr[MAXV], ul[MAXV], ur[MAXV];
    compute_flux(ql, fl, gamma, ndim);
    compute_flux(qr, fr, gamma, ndim);
    prim_to_cons(ql, ul, gamma, ndim);
    prim_to_cons(qr, ur, gamma, ndim);
    int ip = ndim + 1;
    double al = sqrt(cs2_of(ql[0], ql[ip], gamma));
    double ar = sqrt(cs2_of(qr[0], qr[ip], gamma));
    double a_max = smax(fabs(ql[1]) + al, fabs(qr[1]) + ar);
    for (int i = 0; i < ndim + 2; ++i) flux[i] = 0.5 * (fl[i] + fr[i]) - 0.5 * a_max * (ur[i] - ul[i]);
}

void orc_solve_hll(const double* ql, const double* qr, double* flux, double gamma, int ndim) {
    double fl[MAXV], fr[MAXV], ul[MAXV], ur[MAXV];
    compute_flux(ql, fl, gamma, ndim);
    compute_flux(qr, fr, gamma, ndim);
    prim_to_cons(ql, ul, gamma, ndim);
    prim_to_cons(qr, ur, gamma, ndim);
    int ip = ndim + 1;
    double al = sqrt(cs2_of(ql[0], ql[ip], gamma));
    double ar = sqrt(cs2_of(qr[0], qr[ip], gamma));
    double sl = smin(0.0, smin(ql[1] - al, qr[1] - ar));
    double sr = smax(0.0, smax(ql[1] + al, qr[1] + ar));
    if (sr - sl < 1e-20) {
        for (int i = 0; i < ndim + 2; ++i) flux[i] = 0.5 * (fl[i] + fr[i]);
    } else {
        double inv_srs = 1.0 / (sr - sl);
        for (int i = 0; i < ndim + 2; ++i) flux[i] = (sr * fl[i] - sl * fr[i] + sr * sl * (ur[i] - ul[i])) * inv_srs;
    }
}

void orc_solve_hllc(const double* ql, const double* qr, double* flux, double gamma, int ndim) {
    const double smallc = 1e-10, smallr = smallc;
    const double smallp = smallc * smallc / gamma;
    int ip = ndim + 1;
    double rl = smax(ql[0], smallr), ul = ql[1], pl = smax(ql[ip], rl * smallp);
    double rr = smax(qr[0], smallr), ur = qr[1], pr = smax(qr[ip], rr * smallp);
    double cl = sqrt(cs2_of(rl, ql[ip], gamma));
    double cr = sqrt(cs2_of(rr, qr[ip], gamma));
    double sl = smin(ul, ur) - smax(cl, cr);
    double sr = smax(ul, ur) + smax(cl, cr);
    if (sl > 0.0) {
        compute_flux(ql, flux, gamma, ndim);
    } else if (sr < 0.0) {
        compute_flux(qr, flux, gamma, ndim);
    } else {
        double rcl = rl * (ul - sl);
        double rcr = rr * (sr - ur);
        double div = rcr + rcl;
        if (div < 1e-5) {
            double fa[MAXV], fb[MAXV];
            compute_flux(ql, fa, gamma, ndim);
            compute_flux(qr, fb, gamma, ndim);
            for (int i = 0; i < ndim + 2; ++i) flux[i] = 0.5 * (fa[i] + fb[i]);
            return;
        }
        double ustar = (rcr * ur + rcl * ul + (pl - pr)) / div;
        ustar = smax(-1e6, smin(1e6, ustar));
        double pstar = (rcr * pl + rcl * pr + rcl * rcr * (ul - ur)) / div;
        pstar = smax(pstar, 0.0);
        double qs[MAXV] = {0}, f0[MAXV], u0[MAXV], us[MAXV];
        if (ustar > 0.0) {
            double den = smin(sl - ustar, -1e-10);
            double rstar = rl * (sl - ul) / den;
            qs[0] = rstar;
            qs[1] = ustar;
            for (int i = 2; i <= ndim; ++i) qs[i] = ql[i];
            double sum_prad_star = 0.0;
            qs[ip] = smax(pstar - sum_prad_star, rstar * smallp);
            compute_flux(ql, f0, gamma, ndim);
            prim_to_cons(ql, u0, gamma, ndim);
            prim_to_cons(qs, us, gamma, ndim);
            us[ip] = ((sl - ul) * u0[ip] - pl * ul + pstar * ustar) / den;
            for (int i = 0; i < ndim + 2; ++i) flux[i] = f0[i] + sl * (us[i] - u0[i]);
        } else {
            double den = smax(sr - ustar, 1e-10);
            double rstar = rr * (sr - ur) / den;
            qs[0] = rstar;
            qs[1] = ustar;
            for (int i = 2; i <= ndim; ++i) qs[i] = qr[i];
            double sum_prad_star = 0.0;
            qs[ip] = smax(pstar - sum_prad_star, rstar * smallp);
            compute_flux(qr, f0, gamma, ndim);
            prim_to_cons(qr, u0, gamma, ndim);
            prim_to_cons(qs, us, gamma, ndim);
            us[ip] = ((sr - ur) * u0[ip] - pr * ur + pstar * ustar) / den;
            for (int i = 0; i < ndim + 2; ++i) flux[i] = f0[i] + sr * (us[i] - u0[i]);
        }
    }
}

/* Exact (two-shock Newton) solver, RiemannSolver.cpp:194-307.  niter and tol
 * are the reference's 10 and 1e-6 unless overridden; p0 (if > 0) replaces the
 * initial guess of :215 (the learned-guess mode); *iters receives the number
 * of Newton updates made. */
void orc_solve_exact(const double* ql, const double* qr, double* flux, double gamma, int ndim,
                     int niter, double tol, double p0, int* iters, double* pstar_out) {
    const double smallc = 1e-10, smallr = smallc;
    const double smallp = smallc * smallc / gamma;
    const double gamma6 = (gamma + 1.0) / (2.0 * gamma);
    int ip = ndim + 1;
    double rl = smax(ql[0], smallr), ul = ql[1], pl = smax(ql[ip], rl * smallp);
    double rr = smax(qr[0], smallr), ur = qr[1], pr = smax(qr[ip], rr * smallp);
    double cl_sq = gamma * pl * rl;
    double cr_sq = gamma * pr * rr;
    double wl = sqrt(smax(cl_sq, 0.0));
    double wr = sqrt(smax(cr_sq, 0.0));
    double pstar = (wr * pl + wl * pr + wl * wr * (ul - ur)) / (wl + wr + 1e-20);
    pstar = smax(pstar, 0.0);
    if (p0 > 0.0) pstar = p0;
    double pold = pstar;
    int it = 0;
    /* Converged mode (tol below the reference's 1e-6), this library's own
     * addition: g(p) = usl - usr is strictly decreasing and convex in p >= 0,
     * so the signs of the evaluated g bracket the root; a Newton step that
     * leaves the bracket is replaced by its midpoint (bracketed Newton-
     * bisection, Numerical Recipes 3rd ed. sec. 9.4), and the loop also ends
     * when the bracket has closed to tol relative.  Reference mode runs
     * RiemannSolver.cpp:220-235 as written. */
    const int safe = tol < 1e-6;
    double lo = 0.0, hi = INFINITY;
    for (int iter = 0; iter < niter; ++iter) {
        double wwl_sq = cl_sq * (1.0 + gamma6 * (pold - pl) / (pl + 1e-20));
        double wwr_sq = cr_sq * (1.0 + gamma6 * (pold - pr) / (pr + 1e-20));
        double wwl = sqrt(smax(wwl_sq, 0.0));
        double wwr = sqrt(smax(wwr_sq, 0.0));
        double ql_nr = (2.0 * pow(wwl, 3)) / (wwl * wwl + cl_sq + 1e-20);
        double qr_nr = (2.0 * pow(wwr, 3)) / (wwr * wwr + cr_sq + 1e-20);
        double usl = ul - (pold - pl) / (wwl + 1e-20);
        double usr = ur + (pold - pr) / (wwr + 1e-20);
        double delp = (qr_nr * ql_nr / (qr_nr + ql_nr + 1e-20)) * (usl - usr);
        delp = smax(delp, -pold);
        it++;
        if (safe) {
            double gv = usl - usr, pn;
            if (gv > 0.0) lo = smax(lo, pold);
            else if (gv < 0.0) hi = smin(hi, pold);
            else break;
            pn = pold + delp;
            if (fabs(delp / (pn + 1e-10)) < tol) { pold = pn; break; }
            if (!((pn > lo || pn == 0.0) && pn < hi)) pn = hi < INFINITY ? 0.5 * (lo + hi) : 2.0 * lo + 1e-300;
            pold = pn;
            if (hi - lo <= tol * (lo + 1e-10)) break;
            continue;
        }
        pold = pold + delp;
        if (fabs(delp / (pold + 1e-10)) < tol) break;
    }
    if (safe) {
        /* polish: the root truncated to 30 significant bits, then two plain
         * Newton updates, so the result no longer depends on the start */
        union { double d; unsigned long long u; } b;
        b.d = pold;
        b.u &= ~((1ULL << 22) - 1);
        pold = b.d;
        for (int k = 0; k < 2; ++k) {
            double wwl = sqrt(smax(cl_sq * (1.0 + gamma6 * (pold - pl) / (pl + 1e-20)), 0.0));
            double wwr = sqrt(smax(cr_sq * (1.0 + gamma6 * (pold - pr) / (pr + 1e-20)), 0.0));
            double ql_nr = (2.0 * pow(wwl, 3)) / (wwl * wwl + cl_sq + 1e-20);
            double qr_nr = (2.0 * pow(wwr, 3)) / (wwr * wwr + cr_sq + 1e-20);
            double usl = ul - (pold - pl) / (wwl + 1e-20);
            double usr = ur + (pold - pr) / (wwr + 1e-20);
            double delp = (qr_nr * ql_nr / (qr_nr + ql_nr + 1e-20)) * (usl - usr);
            pold = pold + smax(delp, -pold);
        }
    }
    pstar = pold;
    if (iters) *iters = it;
    if (pstar_out) *pstar_out = pstar;

    double wwl_f = sqrt(smax(cl_sq * (1.0 + gamma6 * (pstar - pl) / (pl + 1e-20)), 0.0));
    double wwr_f = sqrt(smax(cr_sq * (1.0 + gamma6 * (pstar - pr) / (pr + 1e-20)), 0.0));
    double ustar = 0.5 * (ul + (pl - pstar) / (wwl_f + 1e-20) + ur - (pr - pstar) / (wwr_f + 1e-20));
    double ro, uo, po;
    double sgnm = (ustar > 0) ? 1.0 : -1.0;
    if (sgnm == 1.0) { ro = rl; uo = ul; po = pl; }
    else { ro = rr; uo = ur; po = pr; }
    double rstar_val;
    if (pstar >= po) {
        rstar_val = ro * ((gamma + 1.0) * pstar + (gamma - 1.0) * po) / ((gamma - 1.0) * pstar + (gamma + 1.0) * po);
    } else {
        rstar_val = ro * pow(pstar / (po + 1e-20), 1.0 / gamma);
    }
    rstar_val = smax(rstar_val, smallr);
    double cl_h = sqrt(cs2_of(rl, pl, gamma));
    double cr_h = sqrt(cs2_of(rr, pr, gamma));
    double sl_h = smin(ul, ur) - smax(cl_h, cr_h);
    double sr_h = smax(ul, ur) + smax(cl_h, cr_h);
    if (sl_h > 0.0) { ro = rl; uo = ul; po = pl; }
    else if (sr_h < 0.0) { ro = rr; uo = ur; po = pr; }
    else { ro = rstar_val; uo = ustar; po = pstar; }
    double e_int = po / (gamma - 1.0);
    double e_kin = 0.5 * ro * uo * uo;
    for (int i = 2; i <= ndim; ++i) {
        double vt = (ustar > 0.0) ? ql[i] : qr[i];
        e_kin += 0.5 * ro * vt * vt;
    }
    double E = e_int + e_kin;
    flux[0] = ro * uo;
    flux[1] = ro * uo * uo + po;
    for (int i = 2; i <= ndim; ++i) flux[i] = flux[0] * ((ustar > 0.0) ? ql[i] : qr[i]);
    flux[ip] = (E + po) * uo;
}

void orc_solve_acoustic(const double* ql, const double* qr, double* flux, double gamma, int ndim) {
    const double smallc = 1e-10, smallr = smallc;
    const double smallp = smallc * smallc / gamma;
    int ip = ndim + 1;
    double rl = smax(ql[0], smallr), ul = ql[1], pl = smax(ql[ip], rl * smallp);
    double rr = smax(qr[0], smallr), ur = qr[1], pr = smax(qr[ip], rr * smallp);
    double cl = sqrt(cs2_of(rl, ql[ip], gamma));
    double cr = sqrt(cs2_of(rr, qr[ip], gamma));
    double wl = cl * rl, wr = cr * rr;
    double pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr + 1e-20);
    double ustar = ((wr * ur + wl * ul) + (pl - pr)) / (wl + wr + 1e-20);
    double sgnm = (ustar >= 0.0) ? 1.0 : -1.0;
    double ro, uo, po, co;
    if (sgnm == 1.0) { ro = rl; uo = ul; po = pl; co = cl; }
    else { ro = rr; uo = ur; po = pr; co = cr; }
    double rstar = ro + (pstar - po) / smax(co * co, 1e-20);
    rstar = smax(rstar, smallr);
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
    double qg[MAXV] = {0};
    qg[0] = rg;
    qg[1] = ug;
    for (int i = 2; i <= ndim; ++i) qg[i] = (sgnm == 1.0) ? ql[i] : qr[i];
    double sum_prad_star = 0.0;
    qg[ip] = smax(pg - sum_prad_star, rg * smallp);
    compute_flux(qg, flux, gamma, ndim);
}

static void riemann(const rg_params* p, const double* ql, const double* qr, double* flux, int* iters) {
    int nd = p->ndim;
    switch (p->riemann) {
        case RG_RIEMANN_HLLC: orc_solve_hllc(ql, qr, flux, p->gamma, nd); break;
        case RG_RIEMANN_HLL: orc_solve_hll(ql, qr, flux, p->gamma, nd); break;
        case RG_RIEMANN_EXACT:
            orc_solve_exact(ql, qr, flux, p->gamma, nd, p->exact_niter > 0 ? p->exact_niter : 10,
                            p->exact_tol > 0 ? p->exact_tol : 1e-6, -1.0, iters, NULL);
            break;
        case RG_RIEMANN_ACOUSTIC: orc_solve_acoustic(ql, qr, flux, p->gamma, nd); break;
        default: orc_solve_llf(ql, qr, flux, p->gamma, nd); break;
    }
}

/* Interpolation slope of the ghost branch (HydroSolver.cpp:256-269,365-374). */
static double interp_slope(double dlft, double drgt, int itype) {
    double sgn = (dlft >= 0.0) ? 1.0 : -1.0;
    if (itype == 1) return sgn * 0.5 * smin(fabs(dlft), fabs(drgt));
    if (itype == 2) return sgn * smin3(fabs(dlft), fabs(drgt), 0.25 * fabs(dlft + drgt));
    if (itype == 3) return 0.25 * (dlft + drgt);
    return 0.0;
}

/* ------------------------------------------------------------ level step */

#define UOLD(icell, iv) uold[(size_t)((iv) - 1) * ncell + (icell) - 1]
#define UNEW(icell, iv) unew[(size_t)((iv) - 1) * ncell + (icell) - 1]

static int btype_of(const rg_grid_view* g, int ib_default_one, int id) {
    int ib = -id;
    if (ib > 0 && ib <= g->nbound_type && g->bound_type) return g->bound_type[ib - 1];
    return ib_default_one;
}

typedef struct {
    const rg_grid_view* g;
    const rg_params* p;
    const double* uold;
    double* unew;
    double* qm; /* [ncell][3][nvar] */
    double* qp;
    int* cell_levels;
    int ilevel, ndim, nvar;
    long ncell;
    double dt, dx, dtdx;
    long long exact_iters, exact_calls;
} step_t;

/* GHOST branch, 2D/3D form (HydroSolver.cpp:171-218,357-446). */
static int ghost_face_3d(step_t* s, int id_n, int idim, double* qm_nb, double* qp_nb) {
    const rg_grid_view* g = s->g;
    const double* uold = s->uold;
    long ncell = s->ncell;
    int nvar = s->nvar, ndim = s->ndim;
    double gamma = s->p->gamma;
    double u_c[MAXV], q_c[MAXV];
    for (int iv = 1; iv <= nvar; ++iv) u_c[iv - 1] = UOLD(id_n, iv);
    int icn_p[6];
    if (nbor_cells_of(g, ndim, id_n, icn_p)) return -1;
    int id_l = icn_p[idim * 2], id_r = icn_p[idim * 2 + 1];
    double u_l[MAXV], u_r[MAXV];
    for (int k = 0; k < 2; ++k) {
        int id = k ? id_r : id_l;
        double* uo = k ? u_r : u_l;
        if (id > 0) {
            for (int iv = 1; iv <= nvar; ++iv) uo[iv - 1] = UOLD(id, iv);
        } else {
            for (int iv = 0; iv < nvar; ++iv) uo[iv] = u_c[iv];
            if (btype_of(g, 0, id) == 1 && id < 0) uo[1 + idim] *= -1.0;
        }
    }
    /* The reference swaps the velocities, computes a slope on the conservative
     * variables that it then overwrites, and swaps back; both interpol_var
     * branches then reduce to: primitives of the natural state, rotated. */
    double q_l[MAXV], q_r[MAXV], dq[MAXV];
    orc_ctoprim(u_c, q_c, gamma, ndim, nvar);
    orc_ctoprim(u_l, q_l, gamma, ndim, nvar);
    orc_ctoprim(u_r, q_r, gamma, ndim, nvar);
    if (idim > 0) {
        swapd(&q_c[1], &q_c[1 + idim]);
        swapd(&q_l[1], &q_l[1 + idim]);
        swapd(&q_r[1], &q_r[1 + idim]);
    }
    double dx_coarse = 2.0 * s->dx;
    int it = s->p->interpol_type;
    for (int iv = 0; iv < nvar; ++iv) {
        double dlft = q_c[iv] - q_l[iv];
        double drgt = q_r[iv] - q_c[iv];
        double slope = 0.0;
        if (it > 0 && dlft * drgt > 0.0) slope = interp_slope(dlft, drgt, it);
        dq[iv] = slope / dx_coarse;
    }
    orc_trace(q_c, dq, s->dt, dx_coarse, qm_nb, qp_nb, gamma, ndim, nvar);
    return 0;
}

/* GHOST branch, 1D form (HydroSolver.cpp:219-356): child states of the
 * coarse neighbour, then a slope_type ghost slope against the active cell. */
static int ghost_face_1d(step_t* s, int idc, int id_n, int side, double* qm_nb, double* qp_nb) {
    const rg_grid_view* g = s->g;
    const double* uold = s->uold;
    long ncell = s->ncell;
    int nvar = s->nvar, ndim = s->ndim, idim = 0;
    double gamma = s->p->gamma;
    double dt = s->dt, dx = s->dx;
    int slope_type = s->p->slope_type, interpol_type = s->p->interpol_type, interpol_var = s->p->interpol_var;
    double u_c[MAXV], u_l[MAXV], u_r[MAXV];
    for (int iv = 1; iv <= nvar; ++iv) u_c[iv - 1] = UOLD(id_n, iv);
    int icn_p[6];
    if (nbor_cells_of(g, ndim, id_n, icn_p)) return -1;
    int id_l = icn_p[0], id_r = icn_p[1];
    for (int k = 0; k < 2; ++k) {
        int id = k ? id_r : id_l;
        double* uo = k ? u_r : u_l;
        if (id > 0) {
            for (int iv = 1; iv <= nvar; ++iv) uo[iv - 1] = UOLD(id, iv);
        } else {
            for (int iv = 0; iv < nvar; ++iv) uo[iv] = u_c[iv];
            if (btype_of(g, 0, id) == 1 && id < 0) uo[1 + idim] *= -1.0;
        }
    }
    double q1_l[MAXV] = {0}, q1_c[MAXV] = {0}, q1_r[MAXV] = {0};
    const double* us[3] = {u_l, u_c, u_r};
    double* q1s[3] = {q1_l, q1_c, q1_r};
    for (int k = 0; k < 3; ++k) {
        const double* u = us[k];
        double* q = q1s[k];
        if (interpol_var == 0) {
            for (int iv = 0; iv < nvar; ++iv) q[iv] = u[iv];
        } else if (interpol_var == 1) {
            double d = smax(u[0], 1e-10);
            q[0] = u[0];
            double e_kin = 0.5 * u[1] * u[1] / d;
            int iener = ndim + 1;
            double e_nonthermal = 0.0;
            q[iener] = u[iener] - e_kin - e_nonthermal;
            for (int iv = iener + 1; iv < nvar; ++iv) q[iv] = u[iv];
        } else {
            orc_ctoprim(u, q, gamma, ndim, nvar);
        }
    }
    double slopes[MAXV] = {0};
    for (int iv = 0; iv < nvar; ++iv) {
        double dlft = q1_c[iv] - q1_l[iv];
        double drgt = q1_r[iv] - q1_c[iv];
        if (dlft * drgt > 0.0) {
            int itype = interpol_type;
            if (interpol_type == 4) itype = (interpol_var == 2 && iv == 1) ? 3 : 2;
            if (itype >= 1 && itype <= 3) slopes[iv] = interp_slope(dlft, drgt, itype);
        }
    }
    double q2L[MAXV] = {0}, q2R[MAXV] = {0}, uL[MAXV] = {0}, uR[MAXV] = {0};
    for (int iv = 0; iv < nvar; ++iv) {
        q2L[iv] = q1_c[iv] - 0.5 * slopes[iv];
        q2R[iv] = q1_c[iv] + 0.5 * slopes[iv];
    }
    for (int k = 0; k < 2; ++k) {
        const double* q = k ? q2R : q2L;
        double* u = k ? uR : uL;
        if (interpol_var == 0) {
            for (int iv = 0; iv < nvar; ++iv) u[iv] = q[iv];
        } else if (interpol_var == 1) {
            double d = smax(q[0], 1e-10);
            u[0] = d;
            double e_kin = 0.5 * q[1] * q[1] / d;
            int iener = ndim + 1;
            double e_nonthermal = 0.0;
            u[iener] = q[iener] + e_kin + e_nonthermal;
            for (int iv = iener + 1; iv < nvar; ++iv) u[iv] = q[iv];
        } else {
            double d = smax(q[0], 1e-10);
            u[0] = d;
            double e_kin = 0.5 * d * q[1] * q[1];
            int iener = ndim + 1;
            double pq = q[iener];
            double e_nonthermal = 0.0;
            u[iener] = pq / (gamma - 1.0) + e_kin + e_nonthermal;
            for (int iv = iener + 1; iv < nvar; ++iv) u[iv] = d * q[iv];
        }
    }
    /* the 1D state vectors above leave u[1] unset in modes 1 and 2 when the
     * reference does: its mode-1/2 helpers never write index 1 either. */
    double q_g2[MAXV] = {0}, q_g[MAXV] = {0};
    if (side == 0) {
        orc_ctoprim(uL, q_g2, gamma, ndim, nvar);
        orc_ctoprim(uR, q_g, gamma, ndim, nvar);
    } else {
        orc_ctoprim(uR, q_g2, gamma, ndim, nvar);
        orc_ctoprim(uL, q_g, gamma, ndim, nvar);
    }
    double u_act[MAXV], q_act[MAXV];
    for (int iv = 1; iv <= nvar; ++iv) u_act[iv - 1] = UOLD(idc, iv);
    orc_ctoprim(u_act, q_act, gamma, ndim, nvar);
    double dq_g[MAXV] = {0};
    for (int iv = 0; iv < nvar; ++iv) {
        double dlft, drgt;
        if (side == 0) {
            dlft = q_g[iv] - q_g2[iv];
            drgt = q_act[iv] - q_g[iv];
        } else {
            dlft = q_g[iv] - q_act[iv];
            drgt = q_g2[iv] - q_g[iv];
        }
        double nu = q_g[1] * dt / dx;
        if ((slope_type == 5 || slope_type == 6) && iv != 0) dq_g[iv] = 0.0;
        else dq_g[iv] = orc_compute_slope(q_g[iv] - dlft, q_g[iv], q_g[iv] + drgt, slope_type, 1.5, nu) / dx;
    }
    orc_trace(q_g, dq_g, dt, dx, qm_nb, qp_nb, gamma, ndim, nvar);
    return 0;
}

#define QM(idc0, idim, iv) s->qm[((size_t)(idc0) * 3 + (idim)) * nvar + (iv)]
#define QP(idc0, idim, iv) s->qp[((size_t)(idc0) * 3 + (idim)) * nvar + (iv)]

/* compute_fluxes lambda of HydroSolver.cpp:118-555 for one cell. */
static int cell_fluxes(step_t* s, int idc0, const int icn[6]) {
    const rg_grid_view* g = s->g;
    const double* uold = s->uold;
    double* unew = s->unew;
    long ncell = s->ncell;
    int nvar = s->nvar, ndim = s->ndim, ilevel = s->ilevel;
    double gamma = s->p->gamma, dt = s->dt, dx = s->dx, dtdx = s->dtdx;
    if (g->son[idc0] != 0) return 0;
    double flux_sum[MAXV] = {0};
    for (int idim = 0; idim < ndim; ++idim) {
        for (int side = 0; side < 2; ++side) {
            int id_n = icn[idim * 2 + side];
            double ql_f[MAXV], qr_f[MAXV], flux[MAXV];
            int is_refined = (id_n > 0 && (g->son[id_n - 1] > 0 || s->cell_levels[id_n] > ilevel));
            if (is_refined) {
                for (int iv = 0; iv < nvar; ++iv) flux[iv] = 0.0;
            } else {
                if (id_n <= 0) {
                    int btype = btype_of(g, 1, id_n);
                    double u_nb[MAXV], q_nb[MAXV], qm_nb[MAXV], qp_nb[MAXV], dq0[MAXV] = {0};
                    for (int iv = 1; iv <= nvar; ++iv) u_nb[iv - 1] = UOLD(idc0 + 1, iv);
                    if (btype == 1) u_nb[1 + idim] *= -1.0;
                    orc_ctoprim(u_nb, q_nb, gamma, ndim, nvar);
                    if (idim > 0) swapd(&q_nb[1], &q_nb[1 + idim]);
                    orc_trace(q_nb, dq0, dt, dx, qm_nb, qp_nb, gamma, ndim, nvar);
                    if (idim > 0) {
                        swapd(&qm_nb[1], &qm_nb[1 + idim]);
                        swapd(&qp_nb[1], &qp_nb[1 + idim]);
                    }
                    for (int iv = 0; iv < nvar; ++iv) {
                        if (side == 0) { ql_f[iv] = qm_nb[iv]; qr_f[iv] = QP(idc0, idim, iv); }
                        else { ql_f[iv] = QM(idc0, idim, iv); qr_f[iv] = qp_nb[iv]; }
                    }
                } else if (!g->son[id_n - 1] && s->cell_levels[id_n] == ilevel) {
                    int n0 = id_n - 1;
                    for (int iv = 0; iv < nvar; ++iv) {
                        if (side == 0) { ql_f[iv] = QM(n0, idim, iv); qr_f[iv] = QP(idc0, idim, iv); }
                        else { ql_f[iv] = QM(idc0, idim, iv); qr_f[iv] = QP(n0, idim, iv); }
                    }
                } else {
                    double qm_nb[MAXV] = {0}, qp_nb[MAXV] = {0};
                    if (ndim == 1) {
                        if (ghost_face_1d(s, idc0 + 1, id_n, side, qm_nb, qp_nb)) return -1;
                    } else {
                        if (ghost_face_3d(s, id_n, idim, qm_nb, qp_nb)) return -1;
                        if (idim > 0) {
                            swapd(&qm_nb[1], &qm_nb[1 + idim]);
                            swapd(&qp_nb[1], &qp_nb[1 + idim]);
                        }
                    }
                    for (int iv = 0; iv < nvar; ++iv) {
                        if (side == 0) { ql_f[iv] = qm_nb[iv]; qr_f[iv] = QP(idc0, idim, iv); }
                        else { ql_f[iv] = QM(idc0, idim, iv); qr_f[iv] = qp_nb[iv]; }
                    }
                }
                if (idim > 0) {
                    swapd(&ql_f[1], &ql_f[1 + idim]);
                    swapd(&qr_f[1], &qr_f[1 + idim]);
                }
                int iters = 0;
                riemann(s->p, ql_f, qr_f, flux, &iters);
                if (s->p->riemann == RG_RIEMANN_EXACT) {
                    s->exact_iters += iters;
                    s->exact_calls++;
                }
                double mass_flux = flux[0];
                for (int iv = ndim + 2; iv < nvar; ++iv) flux[iv] = mass_flux * ((mass_flux > 0) ? ql_f[iv] : qr_f[iv]);
                if (idim > 0) swapd(&flux[1], &flux[1 + idim]);
                if (id_n > 0 && s->cell_levels[id_n] < ilevel) {
                    double factor = 1.0 / (1 << ndim);
                    double sign = (side == 0) ? 1.0 : -1.0;
                    for (int iv = 1; iv <= nvar; ++iv) UNEW(id_n, iv) -= dtdx * sign * flux[iv - 1] * factor;
                }
            }
            double sign = (side == 0) ? 1.0 : -1.0;
            for (int iv = 0; iv < nvar; ++iv) flux_sum[iv] += sign * flux[iv];
        }
    }
    for (int iv = 1; iv <= nvar; ++iv) UNEW(idc0 + 1, iv) = UNEW(idc0 + 1, iv) + dtdx * flux_sum[iv - 1];
    double d_curr = sclamp(UNEW(idc0 + 1, 1), 1e-10, 1e6);
    UNEW(idc0 + 1, 1) = d_curr;
    for (int i = 1; i <= ndim; ++i) UNEW(idc0 + 1, 1 + i) = sclamp(UNEW(idc0 + 1, 1 + i), -d_curr * 10.0, d_curr * 10.0);
    double v2_curr = 0.0;
    for (int i = 1; i <= ndim; ++i) {
        double v = UNEW(idc0 + 1, 1 + i) / d_curr;
        v2_curr += v * v;
    }
    int iener = ndim + 2;
    double ei_curr = UNEW(idc0 + 1, iener) - 0.5 * d_curr * v2_curr;
    if (ei_curr < d_curr * 1e-10 / (gamma - 1.0)) {
        double e_non = 0;
        UNEW(idc0 + 1, iener) = d_curr * 1e-10 / (gamma - 1.0) + 0.5 * d_curr * v2_curr + e_non;
    }
    UNEW(idc0 + 1, iener) = smin(UNEW(idc0 + 1, iener), d_curr * 1e8);
    return 0;
}

int orc_godunov_fine(const rg_grid_view* g, const rg_params* p, int ilevel, double dt, double dx,
                     const double* uold, double* unew, long long* exact_iters, long long* exact_calls) {
    int ndim = p->ndim, nvar = p->nvar;
    if (ndim < 1 || ndim > 3 || nvar < ndim + 2 || nvar > MAXV || g->nboundary != 0) return -3;
    long ncell = g->ncell;
    int ttd = 1 << ndim;
    step_t s;
    memset(&s, 0, sizeof(s));
    s.g = g; s.p = p; s.uold = uold; s.unew = unew;
    s.ilevel = ilevel; s.ndim = ndim; s.nvar = nvar; s.ncell = ncell;
    s.dt = dt; s.dx = dx; s.dtdx = dt / dx;
    s.cell_levels = (int*)malloc(sizeof(int) * ((size_t)ncell + 1));
    if (!s.cell_levels) return -8;
    if (orc_cell_levels(g, ndim, s.cell_levels)) { free(s.cell_levels); return -4; }
    int noct = 0;
    int* octs = NULL;
    if (ilevel > 0) {
        noct = orc_level_octs(g, ilevel, NULL, 0);
        if (noct < 0) { free(s.cell_levels); return -4; }
        octs = (int*)malloc(sizeof(int) * (size_t)(noct > 0 ? noct : 1));
        orc_level_octs(g, ilevel, octs, noct);
    }
    int do_level_0 = (ilevel == 0);
    if (noct == 0 && !do_level_0) { free(octs); free(s.cell_levels); return 0; }
    s.qm = (double*)calloc((size_t)ncell * 3 * nvar, sizeof(double));
    s.qp = (double*)calloc((size_t)ncell * 3 * nvar, sizeof(double));
    if (!s.qm || !s.qp) { free(s.qm); free(s.qp); free(octs); free(s.cell_levels); return -8; }
    double gamma = p->gamma;
    int rc = 0;

    /* pass 1: traces (HydroSolver.cpp:76-115) */
    if (do_level_0) {
        for (int idc0 = 0; idc0 < g->ncoarse; ++idc0) {
            double u_c[MAXV], q_c[MAXV];
            for (int iv = 1; iv <= nvar; ++iv) u_c[iv - 1] = UOLD(idc0 + 1, iv);
            orc_ctoprim(u_c, q_c, gamma, ndim, nvar);
            for (int idim = 0; idim < ndim; ++idim) {
                double dq[MAXV] = {0}, qm_t[MAXV], qp_t[MAXV];
                orc_trace(q_c, dq, dt, dx, qm_t, qp_t, gamma, ndim, nvar);
                for (int iv = 0; iv < nvar; ++iv) {
                    s.qm[((size_t)idc0 * 3 + idim) * nvar + iv] = qm_t[iv];
                    s.qp[((size_t)idc0 * 3 + idim) * nvar + iv] = qp_t[iv];
                }
            }
        }
    }
    for (int k = 0; k < noct && rc == 0; ++k) {
        int ig = octs[k];
        int ign[7];
        orc_get_nbor_grids(g, ig, ign);
        for (int ic = 1; ic <= ttd; ++ic) {
            int idc0 = g->ncoarse + (ic - 1) * g->ngridmax + ig - 1;
            int icn[6];
            if (orc_get_nbor_cells(g, ndim, ign, ic, icn, ig)) { rc = -4; break; }
            double u_c[MAXV], q_c[MAXV];
            for (int iv = 1; iv <= nvar; ++iv) u_c[iv - 1] = UOLD(idc0 + 1, iv);
            orc_ctoprim(u_c, q_c, gamma, ndim, nvar);
            for (int idim = 0; idim < ndim; ++idim) {
                double dq[MAXV], q_rot[MAXV];
                for (int iv = 0; iv < nvar; ++iv) q_rot[iv] = q_c[iv];
                /* compute_slopes (HydroSolver.cpp:653-678) */
                if (p->slope_type == 0) {
                    for (int iv = 0; iv < nvar; ++iv) dq[iv] = 0.0;
                } else {
                    double ql[MAXV], qr[MAXV];
                    for (int k2 = 0; k2 < 2; ++k2) {
                        int id = icn[idim * 2 + k2];
                        double* qo = k2 ? qr : ql;
                        if (id > 0) {
                            double u_nb[MAXV];
                            for (int iv = 1; iv <= nvar; ++iv) u_nb[iv - 1] = UOLD(id, iv);
                            orc_ctoprim(u_nb, qo, gamma, ndim, nvar);
                        } else {
                            for (int iv = 0; iv < nvar; ++iv) qo[iv] = q_c[iv];
                            if (id < 0 && btype_of(g, 0, id) == 1) qo[1 + idim] *= -1.0;
                        }
                    }
                    double nu = q_c[1 + idim] * dt / dx;
                    for (int iv = 0; iv < nvar; ++iv) {
                        if ((p->slope_type == 5 || p->slope_type == 6) && iv != 0) dq[iv] = 0.0;
                        else dq[iv] = orc_compute_slope(ql[iv], q_c[iv], qr[iv], p->slope_type, 1.5, nu) / dx;
                    }
                }
                if (idim > 0) {
                    swapd(&q_rot[1], &q_rot[1 + idim]);
                    swapd(&dq[1], &dq[1 + idim]);
                }
                double qm_t[MAXV], qp_t[MAXV];
                orc_trace(q_rot, dq, dt, dx, qm_t, qp_t, gamma, ndim, nvar);
                if (idim > 0) {
                    swapd(&qm_t[1], &qm_t[1 + idim]);
                    swapd(&qp_t[1], &qp_t[1 + idim]);
                }
                for (int iv = 0; iv < nvar; ++iv) {
                    s.qm[((size_t)idc0 * 3 + idim) * nvar + iv] = qm_t[iv];
                    s.qp[((size_t)idc0 * 3 + idim) * nvar + iv] = qp_t[iv];
                }
            }
        }
    }

    /* pass 2: fluxes, reflux and the per-cell update (HydroSolver.cpp:557-572) */
    if (rc == 0 && do_level_0) {
        for (int idc0 = 0; idc0 < g->ncoarse && rc == 0; ++idc0) {
            int icn[6];
            orc_get_nbor_cells_coarse(g, idc0 + 1, icn);
            rc = cell_fluxes(&s, idc0, icn);
        }
    }
    for (int k = 0; k < noct && rc == 0; ++k) {
        int ig = octs[k];
        int ign[7];
        orc_get_nbor_grids(g, ig, ign);
        for (int ic = 1; ic <= ttd && rc == 0; ++ic) {
            int idc0 = g->ncoarse + (ic - 1) * g->ngridmax + ig - 1;
            int icn[6];
            if (orc_get_nbor_cells(g, ndim, ign, ic, icn, ig)) { rc = -4; break; }
            rc = cell_fluxes(&s, idc0, icn);
        }
    }
    if (exact_iters) *exact_iters = s.exact_iters;
    if (exact_calls) *exact_calls = s.exact_calls;
    free(s.qm); free(s.qp); free(octs); free(s.cell_levels);
    return rc;
}

int orc_set_unew(const rg_grid_view* g, int ndim, int nvar, int ilevel, const double* uold, double* unew) {
    long ncell = g->ncell;
    int ttd = 1 << ndim;
    if (ilevel == 0)
        for (int i = 1; i <= g->ncoarse; ++i)
            for (int iv = 1; iv <= nvar; ++iv) UNEW(i, iv) = UOLD(i, iv);
    int n = orc_level_octs(g, ilevel, NULL, 0);
    if (n < 0) return -4;
    int ig = (ilevel < 0 || ilevel > g->nlevelmax) ? 0 : g->headl[(size_t)ilevel * (g->ncpu + g->nboundary)];
    while (ig > 0) {
        for (int ic = 1; ic <= ttd; ++ic) {
            int idc = g->ncoarse + (ic - 1) * g->ngridmax + ig;
            for (int iv = 1; iv <= nvar; ++iv) UNEW(idc, iv) = UOLD(idc, iv);
        }
        ig = g->next[ig - 1];
    }
    return 0;
}

int orc_set_uold(const rg_grid_view* g, int ndim, int nvar, int ilevel, double* uold, const double* unew) {
    long ncell = g->ncell;
    int ttd = 1 << ndim;
    if (ilevel == 0)
        for (int i = 1; i <= g->ncoarse; ++i)
            if (g->son[i - 1] == 0)
                for (int iv = 1; iv <= nvar; ++iv) UOLD(i, iv) = UNEW(i, iv);
    int n = orc_level_octs(g, ilevel, NULL, 0);
    if (n < 0) return -4;
    int ig = (ilevel < 0 || ilevel > g->nlevelmax) ? 0 : g->headl[(size_t)ilevel * (g->ncpu + g->nboundary)];
    while (ig > 0) {
        for (int ic = 1; ic <= ttd; ++ic) {
            int idc = g->ncoarse + (ic - 1) * g->ngridmax + ig;
            if (g->son[idc - 1] == 0)
                for (int iv = 1; iv <= nvar; ++iv) UOLD(idc, iv) = UNEW(idc, iv);
        }
        ig = g->next[ig - 1];
    }
    return 0;
}

/* compute_courant_step (HydroSolver.cpp:878-977) for one cell; pressure_cap
 * selects the reference's p <= 100 rho clamp (:909,948). */
static double courant_cell(const double* uold, long ncell, int id, int ndim, double gamma, double dx,
                           double cfl, int pressure_cap) {
    double d = smax(UOLD(id, 1), 1e-10), v2 = 0.0;
    for (int i = 1; i <= ndim; ++i) {
        double v = UOLD(id, 1 + i) / d;
        v2 += v * v;
    }
    int iener = ndim + 2;
    double e_nonthermal = 0.0, sum_gamma_p = 0.0;
    double p = smax((UOLD(id, iener) - 0.5 * d * v2 - e_nonthermal) * (gamma - 1.0), d * 1e-10);
    if (pressure_cap) p = smin(p, d * 1e2);
    double cs2 = cs2_of(d, p, gamma);
    cs2 += sum_gamma_p / d;
    double cs = sqrt(smax(cs2, 1e-10));
    double u_wave = ndim * cs;
    for (int idim = 1; idim <= ndim; ++idim) u_wave += fabs(UOLD(id, 1 + idim) / d);
    double a_grav = 0.0;
    for (int idim = 1; idim <= ndim; ++idim) a_grav += fabs(0.0);
    double alpha = a_grav * dx / (u_wave * u_wave);
    alpha = smax(alpha, 0.0001);
    return (dx / u_wave) * (sqrt(1.0 + 2.0 * cfl * alpha) - 1.0) / alpha;
}

double orc_courant_step(const rg_grid_view* g, int ndim, int nvar, int ilevel, double dx, double gamma,
                        double cfl, double boxlen, int pressure_cap, const double* uold) {
    (void)nvar;
    long ncell = g->ncell;
    int ttd = 1 << ndim;
    double dt_max = boxlen / 1e-10;
    if (ilevel == 0) {
        for (int id = 1; id <= g->ncoarse; ++id) {
            if (g->son[id - 1] > 0) continue;
            dt_max = smin(dt_max, courant_cell(uold, ncell, id, ndim, gamma, dx, cfl, pressure_cap));
        }
        return dt_max;
    }
    int ig = (ilevel > g->nlevelmax) ? 0 : g->headl[(size_t)ilevel * (g->ncpu + g->nboundary)];
    long guard = 0;
    while (ig > 0 && guard++ <= g->ngridmax) {
        for (int ic = 1; ic <= ttd; ++ic) {
            int id = g->ncoarse + (ic - 1) * g->ngridmax + ig;
            if (g->son[id - 1] > 0) continue;
            dt_max = smin(dt_max, courant_cell(uold, ncell, id, ndim, gamma, dx, cfl, pressure_cap));
        }
        ig = g->next[ig - 1];
    }
    return dt_max;
}

long long orc_level_cell_updates(const rg_grid_view* g, int ndim, int ilevel) {
    int ttd = 1 << ndim;
    long long n = 0;
    if (ilevel == 0) {
        for (int i = 0; i < g->ncoarse; ++i) n += (g->son[i] == 0);
        return n;
    }
    int ig = (ilevel > g->nlevelmax) ? 0 : g->headl[(size_t)ilevel * (g->ncpu + g->nboundary)];
    long guard = 0;
    while (ig > 0 && guard++ <= g->ngridmax) {
        for (int ic = 1; ic <= ttd; ++ic) n += (g->son[g->ncoarse + (ic - 1) * g->ngridmax + ig - 1] == 0);
        ig = g->next[ig - 1];
    }
    return n;
}
