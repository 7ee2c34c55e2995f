/*
 * rg_oracle.h -- CPU restatement of RAMSES-CPP's Godunov level step.
 * TEST INFRASTRUCTURE ONLY (see rg_oracle.c): the parity checker, never a
 * product code path.  Return codes follow include/rgpu.h (0 ok, <0 error).
 */
#ifndef RG_ORACLE_H
#define RG_ORACLE_H

#include "../include/rgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

int orc_iii(int idim, int inbor, int ic);
int orc_jjj(int idim, int ic);
void orc_get_nbor_grids(const rg_grid_view* g, int igrid, int ign[7]);
void orc_get_nbor_cells_coarse(const rg_grid_view* g, int icell, int icn[6]);
int orc_get_nbor_cells(const rg_grid_view* g, int ndim, const int ign[7], int ic, int icn[6], int igrid);
int orc_cell_levels(const rg_grid_view* g, int ndim, int* cell_levels);
int orc_level_octs(const rg_grid_view* g, int ilevel, int* octs, int cap);

void orc_ctoprim(const double* u, double* q, double gamma, int ndim, int nvar);
double orc_compute_slope(double ql, double qc, double qr, int slope_type, double theta, double nu);
void orc_trace(const double* q, const double* dq, double dt, double dx, double* qm, double* qp,
               double gamma, int ndim, int nvar);
void orc_solve_llf(const double* ql, const double* qr, double* flux, double gamma, int ndim);
void orc_solve_hll(const double* ql, const double* qr, double* flux, double gamma, int ndim);
void orc_solve_hllc(const double* ql, const double* qr, double* flux, double gamma, int ndim);
void orc_solve_acoustic(const double* ql, const double* qr, double* flux, double gamma, int ndim);
void orc_solve_exact(const double* ql, const double* qr, double* flux, double gamma, int ndim,
                     int niter, double tol, double p0, int* iters, double* pstar_out);

int orc_godunov_fine(const rg_grid_view* g, const rg_params* p, int ilevel, double dt, double dx,
                     const double* uold, double* unew, long long* exact_iters, long long* exact_calls);
int orc_set_unew(const rg_grid_view* g, int ndim, int nvar, int ilevel, const double* uold, double* unew);
int orc_set_uold(const rg_grid_view* g, int ndim, int nvar, int ilevel, double* uold, const double* unew);
double orc_courant_step(const rg_grid_view* g, int ndim, int nvar, int ilevel, double dx, double gamma,
                        double cfl, double boxlen, int pressure_cap, const double* uold);
long long orc_level_cell_updates(const rg_grid_view* g, int ndim, int ilevel);

#ifdef __cplusplus
}
#endif

#endif
