/*
 * mgp_oracle.h -- CPU restatement of the MGPoisson2D multigrid hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The tests check the CUDA library in
 * mgpoisson2d_b200/ against this code, and bench.py times it as the CPU baseline.  The product never
 * links, loads or calls it.
 *
 * It restates, in C, the Fortran 90 routines of EdSantilli/MGPoisson2D
 * (src/libBaseTools/arrayutils.f90, src/libMGPoisson/poisson2d.f90,
 * src/libMGPoisson/MGPoisson2D.f90, src/libMGPoisson/MGPoisson2D_DD.f90) with
 * the same loop order, the same FP64 operation order (built with
 * -ffp-contract=off) and the same quirks.  Each function cites the routine it
 * follows.  Parity pinning: the reference cannot be built here (no Fortran
 * compiler) and ships no golden numbers, so the restatement is pinned by the
 * reference's own known-answer tests (manufactured solutions and their
 * convergence rates, src/tests/test.f90), reproduced in tests/.
 *
 * Arrays use the mgp_array layout of include/mgp2d.h; ld must be set (> 0).
 * Index (i,j) below is relative to the valid region's lower corner.
 *
 * gs_order selects the Gauss-Seidel visiting order:
 *   0 = lexicographic, as the reference (P2:1560-1959, DD:288-306);
 *   1 = the device order: for the 9-point sweep, four colours (i mod 2,
 *       j mod 2) = (0,0),(1,1),(1,0),(0,1) over the interior cells, then the
 *       boundary cells (edges colour by colour, then the corners); for the
 *       deferred-correction 5-point sweep, the reference's own red-black
 *       order (DD:262-285).
 */
#ifndef MGP_ORACLE_H
#define MGP_ORACLE_H
#include "../include/mgp2d.h"

#ifdef __cplusplus
extern "C" {
#endif

int or_estimate_maxdepth(int *maxdepth, const mgp_box *valid);
int or_create_mgschedule(int *refx, int *refy, int *maxdepth, const mgp_box *valid);

int or_fill_ghosts(const mgp_box *valid, mgp_array *phi, const mgp_bdry *bc,
                   const mgp_geo *geo, int homog, int do_neum);
int or_extrapolate_ghosts(const mgp_box *valid, mgp_array *phi, int order);

int or_compute_invdiags(const mgp_box *valid, mgp_array *invd, const mgp_geo *geo,
                        const mgp_bdry *bc, int homog);
/* 1: compute_invdiags includes the Dirichlet ghost's dependence on the cell
 * (an extension; the reference leaves it out, P2:29-33).  Default 0. */
void or_set_dirichlet_coupled_diagonal(int on);
int or_compute_laplacian(const mgp_box *valid, mgp_array *lap, mgp_array *phi,
                         const mgp_geo *geo, const mgp_bdry *bc, int homog, int jscale);
int or_compute_residual(const mgp_box *valid, mgp_array *res, const mgp_array *rhs,
                        mgp_array *phi, const mgp_geo *geo, const mgp_bdry *bc,
                        int homog, int jscale);
int or_relax_gs(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                const mgp_geo *geo, const mgp_bdry *bc, int homog, const mgp_array *invd,
                double omega, double tol, int maxiters, int zerophi, int verbosity,
                int gs_order);
/* relax_jacobi, P2:1358-1451. */
int or_relax_jacobi(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs, const mgp_geo *geo,
                    const mgp_bdry *bc, int homog, const mgp_array *invd, double omega, double tol, int maxiters,
                    int zerophi, int verbosity);
int or_solve_bicgstab2(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                       const mgp_geo *geo, const mgp_bdry *bc, int homog,
                       const mgp_array *invd, double tol, int max_iters, int max_restarts,
                       int zerophi, int verbosity, int gs_order);

int or_restrict(const mgp_box *fine_valid, const mgp_array *fine, const mgp_box *crse_valid,
                mgp_array *crse, int offi, int offj);
int or_prolong(const mgp_box *fine_valid, mgp_array *fine, const mgp_box *crse_valid,
               mgp_array *crse, const mgp_geo *fine_geo, const mgp_geo *crse_geo,
               const mgp_bdry *crse_bc, int order);

/* compute_pd P2:404-795, fill_boundary_fluxes AU:1574-1622, compute_grad
 * P2:809-850, compute_div P2:860-879. */
int or_compute_pd(const mgp_box *valid, mgp_array *pd, const mgp_array *phi, int dir, int nodedir);
int or_fill_boundary_fluxes(const mgp_box *valid, mgp_array *xflux, mgp_array *yflux, const mgp_bdry *bc, int homog);
int or_compute_grad(const mgp_box *valid, mgp_array *xflux, mgp_array *yflux, mgp_array *phi, const mgp_geo *geo,
                    const mgp_bdry *bc, int homog);
int or_compute_div(const mgp_box *valid, mgp_array *div, const mgp_array *xflux, const mgp_array *yflux);
double or_pnorm(const mgp_box *valid, const mgp_array *bd, int p);
double or_inner_prod(const mgp_box *valid, const mgp_array *a, const mgp_array *b);
double or_integrate2d(const mgp_box *valid, const mgp_array *bd, const mgp_geo *geo, int jscale);

/* The operator's own face fluxes on the four boundary faces (what
 * compute_grad, P2:809-850, returns there); used by the known-answer tests to
 * build Neumann data as test.f90:1980-2004 does.  xlo/xhi hold ny values,
 * ylo/yhi hold nx values.  phi must have its ghosts set by the caller. */
int or_boundary_fluxes(const mgp_box *valid, const mgp_array *phi, const mgp_geo *geo,
                       double *xlo, double *xhi, double *ylo, double *yhi);

/* Deferred-correction operator set, module DeferredPoisson2D. */
int or_dd_compute_invdiags(const mgp_box *valid, mgp_array *invd, const mgp_geo *geo);
int or_dd_compute_laplacian(const mgp_box *valid, mgp_array *lap, mgp_array *phi,
                            const mgp_geo *geo, const mgp_bdry *bc, int homog);
int or_dd_compute_residual(const mgp_box *valid, mgp_array *res, const mgp_array *rhs,
                           mgp_array *phi, const mgp_geo *geo, const mgp_bdry *bc, int homog);
int or_dd_relax_gs(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                   const mgp_geo *geo, const mgp_bdry *bc, int homog, const mgp_array *invd,
                   double omega, double tol, int maxiters, int zerophi, int verbosity,
                   int gs_order);

/* Drivers.  relres (maxiters+1 doubles) and the report are optional. */
int or_vcycle(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
              const mgp_bdry *bc, int homog, double tol, int maxiters, int maxdepth_user,
              int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
              int verbosity, int gs_order, mgp_report *report);
int or_fmg(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
           const mgp_bdry *bc, int homog, double tol, int maxiters, int maxdepth_user,
           int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
           int verbosity, int gs_order, mgp_report *report);
int or_dc_vcycle(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
                 const mgp_bdry *bc, int homog, double tol, int maxiters, int maxdepth_user,
                 int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
                 int verbosity, int gs_order, mgp_report *report);

#ifdef __cplusplus
}
#endif
#endif
