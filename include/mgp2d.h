/*
 * mgp2d.h -- C ABI of the B200 multigrid solver for the 2-D mapped-grid,
 * variable-coefficient Poisson operator  L[phi] = d_xi(J g^{xi xi} d_xi phi + J g^{xi eta} d_eta phi)
 *                                               + d_eta(J g^{eta xi} d_xi phi + J g^{eta eta} d_eta phi).
 *
 * Every entry point replaces one module procedure of the Fortran library
 * MGPoisson2D (src/libMGPoisson, src/libBaseTools).  The citation beside each
 * declaration names the routine it replaces (file:line).  Argument meaning,
 * defaults and numerical behaviour follow that routine; differences are listed
 * in the comment.
 *
 * Conventions
 *  - Arrays are Fortran column-major (i / x fastest), exactly the memory of
 *    box_data%data (arrayutils.f90:83-96).  An mgp_array names the first
 *    element of the allocation (bx%ilo, bx%jlo) plus its leading dimension and
 *    ghost counts, so a Fortran caller passes c_loc(bd%data) without a copy.
 *  - Pointers may be host or device memory; the library asks the CUDA driver
 *    which one each pointer is (cudaPointerGetAttributes).  Host arrays are
 *    staged through device buffers inside the call.
 *  - All arithmetic is IEEE FP64 without fused multiply-add, in the same
 *    operation order as the Fortran routines (MGP_FLAG_MIXED, an opt-in
 *    extension, runs the V-cycle's grid levels in FP32).
 *  - Every function returns an mgp_status (0 = MGP_OK).  Nothing calls exit();
 *    where the Fortran library prints and stops, this library returns an
 *    error code and records a message readable through mgp_last_error().
 */
#ifndef MGP2D_H
#define MGP2D_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- BC types and modes: same values as arrayutils.f90:27-49 ---- */
#define MGP_BCTYPE_UNDEFINED (-2)
#define MGP_BCTYPE_NONE      (-1)
#define MGP_BCTYPE_NEUM        0
#define MGP_BCTYPE_DIRI        1
#define MGP_BCTYPE_PERIODIC    2
#define MGP_BCTYPE_CF          3
#define MGP_BCTYPE_EXTRAP0     4
#define MGP_BCTYPE_EXTRAP1     5
#define MGP_BCTYPE_EXTRAP2     6

#define MGP_BCMODE_UNIFORM     0
#define MGP_BCMODE_NONUNIFORM  1
#define MGP_BCMODE_LAH         2

/* Sides, in the order of the bdry_data components (arrayutils.f90:55-70). */
#define MGP_XLO 0
#define MGP_XHI 1
#define MGP_YLO 2
#define MGP_YHI 3

/* The sentinel the Fortran library writes into corner ghosts (precision.f90:53). */
#define MGP_BOGUS_VAL 1.2345e300

typedef enum mgp_status {
    MGP_OK        = 0,
    MGP_EINVAL    = 1,  /* bad argument: the Fortran code would print and stop  */
    MGP_ENOMEM    = 2,  /* device or host allocation failed                     */
    MGP_EDIVERGED = 3,  /* non-finite residual (NaN/Inf in the data)            */
    MGP_EMAXITER  = 4,  /* maxiters reached (only with MGP_FLAG_REPORT_MAXITER) */
    MGP_ETIMEOUT  = 5,  /* a bounded device wait ran out                         */
    MGP_ECUDA     = 6,  /* a CUDA runtime call failed                            */
    MGP_ENOTSUP   = 7   /* a path the Fortran library also stops on              */
} mgp_status;

/* type(box), arrayutils.f90:10-15.  nx = ihi-ilo+1, ny = jhi-jlo+1. */
typedef struct mgp_box {
    int ilo, ihi, jlo, jhi;
    int nx, ny;
    double dx, dy;
} mgp_box;

/* box_data%data seen from C.  Valid element (i,j), counted from the valid
 * region's lower corner (0 <= i < nx of the centring), lives at
 *     data[(i + ngx) + (j + ngy) * ld].
 * ld = 0 means the natural leading dimension (valid extent + 2*ngx). */
typedef struct mgp_array {
    double *data;
    int ld;
    int ngx, ngy;
} mgp_array;

/* type(bdry_data), arrayutils.f90:55-70.  data[s] points at 1 value (UNIFORM,
 * LAH) or at the side length of values (NONUNIFORM: ny for x sides, nx for y
 * sides), indexed from the valid region's lower corner. */
typedef struct mgp_bdry {
    int type[4];
    int mode[4];
    const double *data[4];
} mgp_bdry;

/* type(geo_data), arrayutils.f90:109-116.  J is cell-centred; Jgup_xx and
 * Jgup_xy live on x-faces ((nx+1) x ny valid); Jgup_yx and Jgup_yy on y-faces
 * (nx x (ny+1) valid). */
typedef struct mgp_geo {
    mgp_array J, Jgup_xx, Jgup_xy, Jgup_yx, Jgup_yy;
    double dx, dy;
} mgp_geo;

/* Per-solve record, filled by the solve entry points when non-NULL.  relres
 * (optional, caller-owned, maxiters+1 doubles) receives the relative residual
 * history that the Fortran drivers print at verbosity >= 1. */
typedef struct mgp_report {
    int status;
    int iterations;      /* outer iterations performed                        */
    int maxdepth;        /* multigrid depth used (levels 0..maxdepth)         */
    int diverged;        /* 1 if the last correction was undone (MG:630-639)  */
    double rscale;       /* |r0|_2 (1 if it was zero)                          */
    double final_relres;
    double *relres;      /* in: caller array or NULL; out: history            */
    double seconds;      /* wall time of the solve on the device              */
    /* With MGP_FLAG_TIME_SMOOTHER: device time of the level-0 smoothing calls
     * and the number of level-0 sweeps they ran. */
    double smooth0_seconds;
    long long smooth0_sweeps;
} mgp_report;

/* Solver flags (mgp_solver_create; mgp_set_flags for the Fortran-signature
 * drivers and operator calls).  0 reproduces the Fortran library exactly. */
/* compute_invdiags adds the order-3 Dirichlet ghost's dependence on the cell
 * (the ghost moves by -3 per unit change of the cell, arrayutils.f90:1162-1166).
 * The Fortran routine leaves it out (poisson2d.f90:29-33); with that diagonal
 * the Gauss-Seidel sweep amplifies errors at Dirichlet corners and the V-cycle
 * diverges on every problem with two adjacent Dirichlet sides. */
#define MGP_FLAG_DIRICHLET_COUPLED_DIAG 1
/* Time the finest level's smoothing with CUDA events (reported in
 * mgp_report.smooth0_seconds); the events are read after the solve. */
#define MGP_FLAG_TIME_SMOOTHER 2
/* vcycle only: accelerate the V-cycle with BiCGStab.  The solve runs
 * right-preconditioned BiCGStab on the correction equation L_h e = r0
 * (homogeneous BCs), one unchanged V-cycle per preconditioner application,
 * and stops on the same relative-residual test.  report.iterations and the
 * relres history count V-cycles (two per BiCGStab step); final_relres is the
 * true residual rhs - L[phi] recomputed at the end.  No reference counterpart:
 * the Fortran vcycle is a stationary iteration only.  On strongly stretched
 * grids it needs several times fewer V-cycles for the same tolerance. */
#define MGP_FLAG_KRYLOV 4
/* vcycle and dc_vcycle: run the V-cycle's grid levels (every level above the
 * single-CTA coarse cycle) in FP32 inside the FP64 outer iteration.  The
 * residual, the solution update, the convergence test and the coarse levels
 * with the bottom solve stay FP64; geometry and inverse diagonals are the
 * FP64 hierarchy's values rounded to FP32.  Combine with MGP_FLAG_KRYLOV (the
 * FP32 cycle is then the preconditioner).  No reference counterpart. */
#define MGP_FLAG_MIXED 8
/* MG kind only: end the V-cycle at the first level of at most 64 cells and
 * solve that level exactly, with the inverse of its operator (homogeneous
 * BCs) built and factored when the solver is created, in place of the bottom
 * relaxation and solve_bicgstab2 to 1e-6 (MGPoisson2D.f90:733-761).  Needs a
 * Dirichlet side (a nonsingular bottom operator); without one, or when no
 * level is that small, or for cycles that start below that level (fmg), the
 * reference bottom runs.  No reference counterpart: the V-cycle is then a
 * different (stronger) preconditioner, for use with MGP_FLAG_KRYLOV. */
#define MGP_FLAG_DIRECT_COARSE 16
/* vcycle only: accelerate the V-cycle with restarted GMRES instead of
 * BiCGStab (takes precedence over MGP_FLAG_KRYLOV): right-preconditioned
 * GMRES(m) on L_h e = r0 with one V-cycle per preconditioner application,
 * one pass of classical Gram-Schmidt, m = 128 (fewer if the 2m + 1 stored
 * vectors would take more than a quarter of the free device memory).
 * report.iterations and the relres history count V-cycles (the GMRES
 * residual estimate); final_relres is the true residual recomputed at the
 * end, and the solve restarts from it if it has not passed.  No reference
 * counterpart. */
#define MGP_FLAG_GMRES 32
/* with MGP_FLAG_DIRECT_COARSE: the exact bottom is the first level of at
 * most 1024 cells (the level where the single-CTA coarse cycle would start)
 * instead of 64, so no coarse cycle runs: its operator's inverse is built by
 * Gauss-Jordan elimination with partial pivoting on the device when the
 * solver is created (n + 3 launches, 40 n^2 bytes of scratch) and applied by
 * one kernel over many CTAs, one warp per row.  Where that level has more
 * than 1024 cells, or lies below a level of at most 64, MGP_FLAG_DIRECT_COARSE
 * alone applies.  No reference counterpart. */
#define MGP_FLAG_DIRECT_LARGE 64
/* mgp_batch only: solve the batch in lockstep.  Every phase of the V-cycle --
 * a level's smoothing sweeps, its ghost fill, the residual restricted to the
 * next level, the coarse cycles, the prolongations, the update and the
 * residual norms -- runs as one launch over the job table of every problem
 * not yet converged (one job per problem: the tiles or cell blocks of its
 * level), with one host synchronisation per V-cycle for all the norms.  The
 * solver is the stationary V-cycle (MGPoisson2D.f90:565-645, FP64 or with
 * MGP_FLAG_MIXED), each problem stopping on its own test; each solution has
 * the bits of solving that problem alone.  Applies when every problem is MG
 * kind without MGP_FLAG_KRYLOV or MGP_FLAG_GMRES, numcycles is 1, the
 * smoothing counts are even, every problem has a Dirichlet side and no
 * periodic one, and its bottom fits one CTA; otherwise the batch runs its
 * problems concurrently as without the flag.  No reference counterpart. */
#define MGP_FLAG_LOCKSTEP 128
/* vcycle, fmg, dc_vcycle (one-shot, resident, batch and server): a solve that
 * stops because it ran maxiters V-cycles without reaching tol returns
 * MGP_EMAXITER instead of MGP_OK (the report and phi are filled as usual).
 * Without the flag such a solve returns MGP_OK, as the Fortran drivers do
 * (MGPoisson2D.f90:596-645 leave the loop and return), and the caller reads
 * report.final_relres.  A solve stopped by a growing residual (report.diverged)
 * still returns MGP_OK.  No reference counterpart. */
#define MGP_FLAG_REPORT_MAXITER 256
/* with MGP_FLAG_MIXED: a numerics study of BF16 storage on the coarse grid
 * levels.  The FP32 copies of every level below the finest -- the operator's
 * face coefficients, J and the inverse diagonal when the solver is created,
 * the correction and right-hand side each time a kernel writes them -- are
 * rounded to the nearest BF16 value (round to nearest even), so the V-cycle
 * computes in FP32 on the values a BF16 copy would hold.  The storage stays
 * FP32, so the flag adds launches and saves no bytes: it measures the
 * V-cycle counts and the error of that variant, not its speed.  The finest
 * level, the FP64 outer iteration and the FP64 coarse levels (the single-CTA
 * cycle and the exact bottom) are unchanged.  Not used by lockstep batches.
 * No reference counterpart. */
#define MGP_FLAG_BF16_COARSE 512

/* Solver kinds for the resident-hierarchy handle. */
#define MGP_KIND_MG 0   /* module MGPoisson2D (vcycle, fmg)                  */
#define MGP_KIND_DD 1   /* module DeferredMGPoisson2D (vcycle)               */

typedef struct mgp_solver mgp_solver;

/* ------------------------------------------------------------------------ */
/* Library                                                                    */
/* ------------------------------------------------------------------------ */
const char *mgp_version(void);
const char *mgp_last_error(void);
/* Process-wide flags used by the calls that carry no flags argument.  Returns
 * the previous value. */
int mgp_set_flags(int flags);
/* Number of CUDA kernels this process has launched through the library. */
long long mgp_kernel_launch_count(void);
/* Diagnostic with no reference counterpart (the Fortran library has no
 * device waits).  Runs one cooperative grid of nctas CTAs through nbarriers
 * of the grid barrier that the coarse cycle uses on large bottoms, with every
 * wait bounded by wait_s seconds; CTA skip_cta (-1: none) exits before the
 * first barrier, so the other CTAs' waits run out.  Returns MGP_OK when every
 * barrier opened, MGP_ETIMEOUT when a wait ran out (the kernel still ends:
 * after the first timeout no barrier waits again), MGP_ENOTSUP without
 * cooperative launch.  seconds (nullable) receives the kernel's device time. */
int mgp_selftest_grid_barrier(int nctas, int skip_cta, int nbarriers, double wait_s, double *seconds);

/* ------------------------------------------------------------------------ */
/* Schedule (MGPoisson2D.f90:38-129)                                          */
/* ------------------------------------------------------------------------ */
/* estimate_maxdepth, MGPoisson2D.f90:38-62. */
int mgp_estimate_maxdepth(int *maxdepth, const mgp_box *valid);
/* create_mgschedule, MGPoisson2D.f90:67-129.  refx/refy hold maxdepth ints. */
int mgp_create_mgschedule(int *refx, int *refy, int *maxdepth, const mgp_box *valid);

/* compute_pd, poisson2d.f90:404-795: d(phi)/d(dir) (1 = x, 2 = y) onto the
 * faces nodal in `nodedir` (1: x-faces, (nx+1) x ny; 2: y-faces,
 * nx x (ny+1)); the transverse derivative uses the operator's boundary
 * stencils (simple_bdry_stencil = .false.).  The nodal derivative reads
 * phi's ghosts as given. */
int mgp_compute_pd(const mgp_box *valid, mgp_array *pd, const mgp_array *phi, int dir, int nodedir);
/* compute_grad, poisson2d.f90:809-850: J Grad[phi] on x- and y-faces (fills
 * phi's ghosts first, do_neum = .false.; Neumann faces take the BC data).
 * The workspaces of the Fortran signature are internal.  Only valid faces
 * are written; ghost rows of the flux arrays are left as they are. */
int mgp_compute_grad(const mgp_box *valid, mgp_array *xflux, mgp_array *yflux, mgp_array *phi,
                     const mgp_geo *geo, const mgp_bdry *bc, int homog);
/* fill_boundary_fluxes, arrayutils.f90:1574-1622 (valid faces only, as above). */
int mgp_fill_boundary_fluxes(const mgp_box *valid, mgp_array *xflux, mgp_array *yflux,
                             const mgp_bdry *bc, int homog);
/* compute_div, poisson2d.f90:860-879: J Div[flux] = (xflux(i+1)-xflux(i))/dx
 * + (yflux(j+1)-yflux(j))/dy on cells. */
int mgp_compute_div(const mgp_box *valid, mgp_array *div, const mgp_array *xflux, const mgp_array *yflux);


/* ------------------------------------------------------------------------ */
/* Operator-level calls (module Poisson2D and arrayutils)                     */
/* ------------------------------------------------------------------------ */
/* fill_ghosts, arrayutils.f90:1277-1492 (do_neum is the optional do_neum_opt). */
int mgp_fill_ghosts(const mgp_box *valid, mgp_array *phi, const mgp_bdry *bc,
                    const mgp_geo *geo, int homog, int do_neum);
/* extrapolate_ghosts, arrayutils.f90:1497-1566. */
int mgp_extrapolate_ghosts(const mgp_box *valid, mgp_array *phi, int order);
/* compute_invdiags, poisson2d.f90:16-388. */
int mgp_compute_invdiags(const mgp_box *valid, mgp_array *invdiags,
                         const mgp_geo *geo, const mgp_bdry *bc, int homog);
/* compute_laplacian, poisson2d.f90:886-1319 (jscale = opt_jscale). */
int mgp_compute_laplacian(const mgp_box *valid, mgp_array *lap, mgp_array *phi,
                          const mgp_geo *geo, const mgp_bdry *bc, int homog, int jscale);
/* compute_residual, poisson2d.f90:1327-1353. */
int mgp_compute_residual(const mgp_box *valid, mgp_array *res, const mgp_array *rhs,
                         mgp_array *phi, const mgp_geo *geo, const mgp_bdry *bc,
                         int homog, int jscale);
/* relax_jacobi, poisson2d.f90:1358-1451: weighted Jacobi iterations
 * (phi <- omega (phi + r invdiag) + (1 - omega) phi over every cell, then the
 * residual again); tol > 0 stops on |r|/|r0| <= tol. */
int mgp_relax_jacobi(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs, const mgp_geo *geo,
                     const mgp_bdry *bc, int homog, const mgp_array *invdiags, double omega, double tol,
                     int maxiters, int zerophi, int verbosity);
/* relax_gs, poisson2d.f90:1460-1988.  The device sweep visits the four
 * colours (i mod 2, j mod 2) = (0,0),(1,1),(1,0),(0,1) in turn instead of the
 * lexicographic order; ghosts are refreshed once per sweep as in P2:1556. */
int mgp_relax_gs(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                 const mgp_geo *geo, const mgp_bdry *bc, int homog,
                 const mgp_array *invdiags, double omega, double tol, int maxiters,
                 int zerophi, int verbosity);
/* solve_bicgstab2, poisson2d.f90:2253-2477. */
int mgp_solve_bicgstab2(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                        const mgp_geo *geo, const mgp_bdry *bc, int homog,
                        const mgp_array *invdiags, double tol, int max_iters,
                        int max_restarts, int zerophi, int verbosity);
/* No counterpart in the reference.  solve_bicgstab2 for callers that cannot
 * allocate device memory -- a service that reserves its whole device-memory
 * budget at start-up and forbids allocation afterwards, or code running while
 * another component owns the device allocator (cudaMalloc can fail there, and
 * cudaMalloc/cudaFree synchronise the device).  Same arguments and results as
 * mgp_solve_bicgstab2, but every array must be device memory (phi with exactly
 * one ghost layer), the grid at most MGP_NOALLOC_MAX_SIDE cells per side
 * (MGP_EINVAL otherwise), and the work arrays live in one file-scope
 * __device__ array (about 1.2 MB) that every device loading the library keeps
 * until the process exits.  The first call on a device looks up that array's
 * address with the device current; make that first call before any stream
 * capture.  All calls share the array: calls whose kernels overlap on the
 * device race on it.  Runs on the default stream and returns when done. */
#define MGP_NOALLOC_MAX_SIDE 128
int mgp_solve_bicgstab2_noalloc(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                                const mgp_geo *geo, const mgp_bdry *bc, int homog,
                                const mgp_array *invdiags, double tol, int max_iters,
                                int max_restarts, int zerophi, int verbosity);
/* restrict, MGPoisson2D.f90:135-257.  offi/offj: 0 = node, 1 = cell
 * (BD_NODE/BD_CELL, arrayutils.f90:76-77); crse/fine give the cell-centred
 * valid boxes of the two levels. */
int mgp_restrict(const mgp_box *fine_valid, const mgp_array *fine,
                 const mgp_box *crse_valid, mgp_array *crse, int offi, int offj);
/* prolong, MGPoisson2D.f90:262-394.  Adds the interpolated correction to fine.
 * Ratios (2,2) follow the Fortran routine; (2,1) and (1,2), where the Fortran
 * routine stops, use the same constant + linear form in the coarsened
 * direction only. */
int mgp_prolong(const mgp_box *fine_valid, mgp_array *fine, const mgp_box *crse_valid,
                mgp_array *crse, const mgp_geo *fine_geo, const mgp_geo *crse_geo,
                const mgp_bdry *crse_bc, int order);
/* pnorm, arrayutils.f90:753-796 (p = 0 max, 1, 2, other p). */
int mgp_pnorm(const mgp_box *valid, const mgp_array *bd, int p, double *out);
/* inner_prod, arrayutils.f90:637-661. */
int mgp_inner_prod(const mgp_box *valid, const mgp_array *a, const mgp_array *b, double *out);

/* ------------------------------------------------------------------------ */
/* Drivers with the Fortran argument lists (the hierarchy is built and freed  */
/* inside every call, as the Fortran drivers do)                              */
/* ------------------------------------------------------------------------ */
/* MGPoisson2D::vcycle, MGPoisson2D.f90:400-670. */
int mgp_vcycle(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
               const mgp_bdry *bc, int homog, int amrrefx, int amrrefy, double tol,
               int maxiters, int maxdepth_user, int numcycles, int smooth_down,
               int smooth_up, int smooth_bottom, int zerophi, int verbosity,
               mgp_report *report);
/* MGPoisson2D::fmg, MGPoisson2D.f90:860-1122. */
int mgp_fmg(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
            const mgp_bdry *bc, int homog, int amrrefx, int amrrefy, double tol,
            int maxiters, int maxdepth_user, int numcycles, int smooth_down,
            int smooth_up, int smooth_bottom, int zerophi, int verbosity,
            mgp_report *report);
/* DeferredMGPoisson2D::vcycle, MGPoisson2D_DD.f90:589-862.  rhs is scaled by
 * J on entry and divided by J on exit, as in DD:772-773 and DD:837-838. */
int mgp_dc_vcycle(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
                  const mgp_bdry *bc, int homog, int amrrefx, int amrrefy, double tol,
                  int maxiters, int maxdepth_user, int numcycles, int smooth_down,
                  int smooth_up, int smooth_bottom, int zerophi, int verbosity,
                  mgp_report *report);

/* ------------------------------------------------------------------------ */
/* Resident hierarchy.  The set-up half of the drivers above (schedule,       */
/* geometry restriction, inverse diagonals; MG:432-562, DD:622-761) runs once */
/* in mgp_solver_create and stays in HBM; each solve call then runs only the  */
/* iteration half (MG:565-645, MG:1010-1096, DD:765-839).                     */
/* ------------------------------------------------------------------------ */
/* bc supplies the BC types; values are taken per solve call. */
int mgp_solver_create(const mgp_box *valid, const mgp_geo *geo, const mgp_bdry *bc,
                      int kind, int flags, int maxdepth_user, mgp_solver **out);
int mgp_solver_destroy(mgp_solver *s);
/* CUDA stream (cudaStream_t) the solver's work is queued on; NULL = default. */
int mgp_solver_set_stream(mgp_solver *s, void *stream);
int mgp_solver_maxdepth(const mgp_solver *s, int *maxdepth);
int mgp_solver_vcycle(mgp_solver *s, mgp_array *phi, mgp_array *rhs, const mgp_bdry *bc,
                      int homog, double tol, int maxiters, int numcycles, int smooth_down,
                      int smooth_up, int smooth_bottom, int zerophi, int verbosity,
                      mgp_report *report);
int mgp_solver_fmg(mgp_solver *s, mgp_array *phi, mgp_array *rhs, const mgp_bdry *bc,
                   int homog, double tol, int maxiters, int numcycles, int smooth_down,
                   int smooth_up, int smooth_bottom, int zerophi, int verbosity,
                   mgp_report *report);
int mgp_solver_dc_vcycle(mgp_solver *s, mgp_array *phi, mgp_array *rhs, const mgp_bdry *bc,
                         int homog, double tol, int maxiters, int numcycles, int smooth_down,
                         int smooth_up, int smooth_bottom, int zerophi, int verbosity,
                         mgp_report *report);

/* ------------------------------------------------------------------------ */
/* Metric terms and right-hand sides generated on the device from an analytic */
/* map (the Fortran test program builds them on the host, test.f90:566-716).  */
/* Arrays may be device or host memory; device arrays are written in place.   */
/* ------------------------------------------------------------------------ */
#define MGP_MAP_IDENTITY   0   /* x = xi, y = eta                                  */
#define MGP_MAP_WAVY_EXP   1   /* params {a, beta}: x = xi + a sin(2 pi xi) sin(2 pi eta),
                                  y = (e^{beta eta} - 1)/(e^beta - 1)             */
#define MGP_MAP_SKEW_LAYER 2   /* params {tan(angle), ratio, t*, n_ref}: y grows by
                                  `ratio` per cell (of n_ref cells) up to t* cells
                                  from y = 0, uniformly beyond, normalised to
                                  [0,1]; x = xi + tan(angle) y                     */
/* J, Jgup_xx, Jgup_xy, Jgup_yx, Jgup_yy over the whole allocation of each array
 * (valid points and ghosts), by one-cell differences of the map half a cell
 * either side: J = x_xi y_eta - x_eta y_xi, Jgup_xx = (x_eta^2 + y_eta^2)/J,
 * Jgup_xy = Jgup_yx = -(x_xi x_eta + y_xi y_eta)/J, Jgup_yy = (x_xi^2 + y_xi^2)/J.
 * Sets geo->dx, geo->dy from the box. */
int mgp_map_geometry(const mgp_box *valid, int map, const double *params, mgp_geo *geo);
/* rhs = J (f - <f>_J), f = sum_k amp[k] cos(pi m_x[k] x) cos(pi m_y[k] y) at the
 * mapped cell centres, <f>_J its J-weighted mean. */
int mgp_map_fourier_rhs(const mgp_box *valid, int map, const double *params, int nmodes,
                        const double *amp, const int *m_x, const int *m_y, const mgp_array *J,
                        mgp_array *rhs);

/* ------------------------------------------------------------------------ */
/* Many solves at once.  No reference counterpart: the Fortran library solves */
/* one problem per call.  Both front ends run the single-problem solver       */
/* unchanged on several host workers, each with its own CUDA stream, so the   */
/* latency-bound kernels of different problems overlap on the device; every  */
/* result is identical to solving its problem alone.                          */
/* ------------------------------------------------------------------------ */
typedef struct mgp_batch mgp_batch;
/* nprob independent problems (arrays of nprob boxes, geometries and BC types),
 * each with its own resident hierarchy; nstreams workers. */
int mgp_batch_create(int nprob, const mgp_box *valid, const mgp_geo *geo, const mgp_bdry *bc, int kind,
                     int flags, int maxdepth_user, int nstreams, mgp_batch **out);
int mgp_batch_destroy(mgp_batch *b);
int mgp_batch_size(const mgp_batch *b, int *nprob);
/* vcycle on every problem: phi, rhs, bc and reports (nullable) are arrays of
 * nprob.  Returns the first nonzero status; each report holds its own. */
int mgp_batch_vcycle(mgp_batch *b, mgp_array *phi, mgp_array *rhs, const mgp_bdry *bc, int homog,
                     double tol, int maxiters, int numcycles, int smooth_down, int smooth_up,
                     int smooth_bottom, int zerophi, mgp_report *reports);
/* Knobs of the lockstep path (MGP_FLAG_LOCKSTEP), which change speed and never
 * results: groups = how many groups of problems run their lockstep loops
 * concurrently, each on its own stream (1 .. nstreams; 0 restores the
 * default, min(4, nstreams)); pairs = 1 runs two sweeps per launch on the
 * levels whose descriptors allow it (when the smoothing counts are multiples
 * of 4).  mgpoisson2d_b200.api.Batch.autotune times the combinations and
 * caches the fastest.  No reference counterpart. */
int mgp_batch_set_tuning(mgp_batch *b, int groups, int pairs);
int mgp_batch_get_tuning(const mgp_batch *b, int *groups, int *pairs);

typedef struct mgp_server mgp_server;
/* A solve server with nworkers slots.  Requests start in arrival order as a
 * slot frees up and the device memory their hierarchy needs fits within
 * mem_budget bytes (0: 90% of the memory free at creation), evicting idle
 * cached hierarchies first.  The hierarchy of a request with a nonzero key
 * stays resident and serves later requests with the same key and box. */
int mgp_server_create(int nworkers, size_t mem_budget, int flags, mgp_server **out);
/* Queue one vcycle solve (the mgp_solver_vcycle arguments).  Every array the
 * request names must stay alive until mgp_server_wait returns for it. */
int mgp_server_submit(mgp_server *s, unsigned long long key, const mgp_box *valid,
                      const mgp_geo *geo, const mgp_bdry *bc, mgp_array *phi, mgp_array *rhs,
                      int homog, double tol, int maxiters, int numcycles, int smooth_down,
                      int smooth_up, int smooth_bottom, int zerophi, long long *ticket);
/* Block until the ticket's solve is done; report, latency (submit to done) and
 * queue time (submit to start), in seconds, are each nullable. */
int mgp_server_wait(mgp_server *s, long long ticket, mgp_report *report, double *latency_s,
                    double *queue_s);
int mgp_server_destroy(mgp_server *s);

#ifdef __cplusplus
}
#endif
#endif /* MGP2D_H */
