/*
 * mgp_oracle.c -- CPU restatement of the MGPoisson2D multigrid hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see mgp_oracle.h).  Built with -ffp-contract=off
 * so every product and sum is rounded on its own, like the Fortran code.
 *
 * Reference citations use the file tags
 *   AU = src/libBaseTools/arrayutils.f90     P2 = src/libMGPoisson/poisson2d.f90
 *   MG = src/libMGPoisson/MGPoisson2D.f90    DD = src/libMGPoisson/MGPoisson2D_DD.f90
 *
 * Memory that the Fortran drivers allocate and never initialise (the ghost
 * layers of the correction arrays e(d)) starts at zero here.
 */
#include "mgp_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- views ------------------------------------------------------------- */
typedef struct { double *b; long ld; } V;   /* b -> valid element (0,0) */

static V view(const mgp_array *a)
{
    V v;
    v.ld = a->ld;
    v.b = a->data + a->ngx + (long)a->ngy * a->ld;
    return v;
}
#define AT(v, i, j) ((v).b[(long)(i) + (long)(j) * (v).ld])

typedef struct { V J, xx, xy, yx, yy; double dx, dy; } G;

static G gview(const mgp_geo *g)
{
    G r;
    r.J = view(&g->J);
    r.xx = view(&g->Jgup_xx);
    r.xy = view(&g->Jgup_xy);
    r.yx = view(&g->Jgup_yx);
    r.yy = view(&g->Jgup_yy);
    r.dx = g->dx;
    r.dy = g->dy;
    return r;
}

/* Whole allocation of an array (ghosts included): the Fortran `a%data = ...`. */
static long alloc_rows(const mgp_array *a, int ny) { return ny + 2L * a->ngy; }
static long alloc_cols(const mgp_array *a, int nx) { return nx + 2L * a->ngx; }

static const double zero = 0.0, one = 1.0, two = 2.0, three = 3.0, four = 4.0,
                    five = 5.0, six = 6.0, half = 0.5, fourth = 0.25, eighth = 0.125,
                    sixteenth = 0.0625, threehalves = 1.5;

enum { RLO = 0, RMID = 1, RHI = 2 };

static int g_err_quiet = 0;
static int fail(int code, const char *msg)
{
    if (!g_err_quiet) fprintf(stderr, "oracle: %s\n", msg);
    return code;
}

/* ---- schedule: MG:38-62, MG:67-129 -------------------------------------- */
int or_estimate_maxdepth(int *maxdepth, const mgp_box *valid)
{
    int mgnx = valid->nx, mgny = valid->ny, d;
    for (d = 0; d <= *maxdepth - 1; ++d) {
        if (mgnx % 2 == 0)
            mgnx /= 2;
        else if (mgny % 2 == 0)
            mgny /= 2;
        else
            break;
    }
    if (d + 1 < *maxdepth) *maxdepth = d + 1;
    return MGP_OK;
}

int or_create_mgschedule(int *refx, int *refy, int *maxdepth, const mgp_box *valid)
{
    const int min_nx = 4, min_ny = 4;
    int mgnx = valid->nx, mgny = valid->ny, d;
    double mgdx = valid->dx, mgdy = valid->dy, max_dx;
    for (d = 0; d < *maxdepth; ++d) refx[d] = refy[d] = 0;
    for (d = 0; d <= *maxdepth - 1; ++d) {
        if ((mgnx % 2 != 0) || (mgny % 2 != 0)) break;
        max_dx = mgdx > mgdy ? mgdx : mgdy;
        refx[d] = (mgdx <= max_dx / 2) ? 2 : 1;
        refy[d] = (mgdy <= max_dx / 2) ? 2 : 1;
        if (refx[d] * refy[d] == 1) refx[d] = refy[d] = 2;
        mgnx /= refx[d];
        mgny /= refy[d];
        if ((mgnx < min_nx) || (mgny < min_ny)) break;
        mgdx = mgdx * (double)refx[d];
        mgdy = mgdy * (double)refy[d];
    }
    *maxdepth = d;
    return MGP_OK;
}

/* ---- ghost fills: AU:871-1064, AU:1069-1272, AU:1277-1492 --------------- */

/* Relative index into a NONUNIFORM data array of a y side when the Fortran
 * code indexes it with a j-range (AU:1198, AU:1211, AU:1224 and the `(j)` of
 * the north-face flux in P2): absolute index jabs in an array whose lower
 * bound is ilo. */
static int yside_index(const mgp_box *b, int jabs, int *k)
{
    *k = jabs - b->ilo;
    if (*k < 0 || *k >= b->nx) return fail(MGP_EINVAL, "y-side boundary data indexed outside its bounds (reference indexes it with j)");
    return MGP_OK;
}

static int neum_dir_side(const mgp_box *bx, V p, const mgp_bdry *bc, const G *g, int homog,
                         int dir, int side)
{
    const int nx = bx->nx, ny = bx->ny;
    double dx = bx->dx, dy = bx->dy, dpn, dpf, cross;
    int i, j, e, s;
    const double *bcd;
    int bcmode;
    if (dir == 1) {
        if (side < 1) { s = MGP_XLO; e = -1; i = 0; dx = -dx; }
        else          { s = MGP_XHI; e = 1; i = nx - 1; }
    } else {
        if (side < 1) { s = MGP_YLO; e = -1; j = 0; dy = -dy; }
        else          { s = MGP_YHI; e = 1; j = ny - 1; }
    }
    bcd = bc->data[s];
    bcmode = bc->mode[s];
    if (dir == 1) {
        if (bcmode == MGP_BCMODE_LAH) {
            for (j = 0; j < ny; ++j) AT(p, i + e, j) = AT(p, i, j);
        } else if (homog) {
            j = 0;
            dpn = -((three * AT(p, i, j) - four * AT(p, i, j + 1) + AT(p, i, j + 2)) * half / dy);
            dpf = -((three * AT(p, i - e, j) - four * AT(p, i - e, j + 1) + AT(p, i - e, j + 2)) * half / dy);
            cross = half * (three * dpn - dpf) * AT(g->xy, i, j);
            AT(p, i + e, j) = AT(p, i, j) - (-cross) * dx / AT(g->xx, i, j);
            for (j = 1; j <= ny - 2; ++j) {
                dpn = (AT(p, i, j + 1) - AT(p, i, j - 1)) * half / dy;
                dpf = (AT(p, i - e, j + 1) - AT(p, i - e, j - 1)) * half / dy;
                cross = (threehalves * dpn - half * dpf) * AT(g->xy, i, j);
                AT(p, i + e, j) = AT(p, i, j) - (-cross) * dx / AT(g->xx, i, j);
            }
            j = ny - 1;
            dpn = (three * AT(p, i, j) - four * AT(p, i, j - 1) + AT(p, i, j - 2)) * half / dy;
            dpf = (three * AT(p, i - e, j) - four * AT(p, i - e, j - 1) + AT(p, i - e, j - 2)) * half / dy;
            cross = half * (three * dpn - dpf) * AT(g->xy, i, j);
            AT(p, i + e, j) = AT(p, i, j) - (-cross) * dx / AT(g->xx, i, j);
        } else {
            /* UNIFORM uses bcd(1); NONUNIFORM bcd(j).  The centred loop runs
             * over jlo..jhi and reads the y ghosts (AU:965, AU:985). */
            int nonu = (bcmode != MGP_BCMODE_UNIFORM);
#define BV(k) (nonu ? bcd[(k)] : bcd[0])
            j = 0;
            dpn = -((three * AT(p, i, j) - four * AT(p, i, j + 1) + AT(p, i, j + 2)) * half / dy);
            dpf = -((three * AT(p, i - e, j) - four * AT(p, i - e, j + 1) + AT(p, i - e, j + 2)) * half / dy);
            cross = half * (three * dpn - dpf) * AT(g->xy, i, j);
            AT(p, i + e, j) = AT(p, i, j) - (BV(j) - cross) * dx / AT(g->xx, i, j);
            for (j = 0; j <= ny - 1; ++j) {
                dpn = (AT(p, i, j + 1) - AT(p, i, j - 1)) * half / dy;
                dpf = (AT(p, i - e, j + 1) - AT(p, i - e, j - 1)) * half / dy;
                cross = (threehalves * dpn - half * dpf) * AT(g->xy, i, j);
                AT(p, i + e, j) = AT(p, i, j) - (BV(j) - cross) * dx / AT(g->xx, i, j);
            }
            j = ny - 1;
            dpn = (three * AT(p, i, j) - four * AT(p, i, j - 1) + AT(p, i, j - 2)) * half / dy;
            dpf = (three * AT(p, i - e, j) - four * AT(p, i - e, j - 1) + AT(p, i - e, j - 2)) * half / dy;
            cross = half * (three * dpn - dpf) * AT(g->xy, i, j);
            AT(p, i + e, j) = AT(p, i, j) - (BV(j) - cross) * dx / AT(g->xx, i, j);
#undef BV
        }
    } else {
        if (bcmode == MGP_BCMODE_LAH) {
            for (i = 0; i < nx; ++i) AT(p, i, j + e) = AT(p, i, j);
        } else {
            /* homog, UNIFORM and NONUNIFORM share one loop structure here:
             * one-sided at ilo, centred over ilo..ihi, one-sided at ihi
             * (AU:994-1062). */
            int kind = homog ? 0 : (bcmode == MGP_BCMODE_UNIFORM ? 1 : 2);
#define BV(k) (kind == 0 ? 0.0 : (kind == 1 ? bcd[0] : bcd[(k)]))
#define UPD(ii) do { if (kind == 0) AT(p, ii, j + e) = AT(p, ii, j) - (-cross) * dy / AT(g->yy, ii, j); \
                     else AT(p, ii, j + e) = AT(p, ii, j) - (BV(ii) - cross) * dy / AT(g->yy, ii, j); } while (0)
            i = 0;
            dpn = -((three * AT(p, i, j) - four * AT(p, i + 1, j) + AT(p, i + 2, j)) * half / dx);
            dpf = -((three * AT(p, i, j - e) - four * AT(p, i + 1, j - e) + AT(p, i + 2, j - e)) * half / dx);
            cross = half * (three * dpn - dpf) * AT(g->yx, i, j);
            UPD(i);
            for (i = 0; i <= nx - 1; ++i) {
                dpn = (AT(p, i + 1, j) - AT(p, i - 1, j)) * half / dx;
                dpf = (AT(p, i + 1, j - e) - AT(p, i - 1, j - e)) * half / dx;
                cross = (threehalves * dpn - half * dpf) * AT(g->yx, i, j);
                UPD(i);
            }
            i = nx - 1;
            dpn = (three * AT(p, i, j) - four * AT(p, i - 1, j) + AT(p, i - 2, j)) * half / dx;
            dpf = (three * AT(p, i, j - e) - four * AT(p, i - 1, j - e) + AT(p, i - 2, j - e)) * half / dx;
            cross = half * (three * dpn - dpf) * AT(g->yx, i, j);
            UPD(i);
#undef UPD
#undef BV
        }
    }
    return MGP_OK;
}

/* fill_ghosts_diri_dir_side with order 3 (the order fill_ghosts hard-wires,
 * AU:1284-1287); AU:1161-1177 and AU:1215-1231. */
static int diri_dir_side(const mgp_box *bx, V p, const mgp_bdry *bc, int homog, int dir, int side)
{
    const int nx = bx->nx, ny = bx->ny;
    const double sixteenfifth = 16.0 / 5.0, fifth = 1.0 / 5.0;
    int i, j, e, s, k, koff = 0;
    if (dir == 1) {
        if (side < 1) { s = MGP_XLO; e = -1; i = 0; }
        else          { s = MGP_XHI; e = 1; i = nx - 1; }
    } else {
        if (side < 1) { s = MGP_YLO; e = -1; j = 0; }
        else          { s = MGP_YHI; e = 1; j = ny - 1; }
    }
    const double *bcd = bc->data[s];
    int bcmode = bc->mode[s];
    if (dir == 1) {
        for (k = 0; k < ny; ++k) {
            double p0 = AT(p, i, k), p1 = AT(p, i - e, k), p2 = AT(p, i - 2 * e, k);
            if (bcmode == MGP_BCMODE_LAH)       AT(p, i + e, k) = -p0;
            else if (homog)                     AT(p, i + e, k) = -(three * p0) + p1 - fifth * p2;
            else if (bcmode == MGP_BCMODE_UNIFORM) AT(p, i + e, k) = sixteenfifth * bcd[0] - three * p0 + p1 - fifth * p2;
            else                                AT(p, i + e, k) = sixteenfifth * bcd[k] - three * p0 + p1 - fifth * p2;
        }
    } else {
        /* NONUNIFORM y sides read bcd(jlo:jhi) of an array declared
         * (ilo:ihi) (AU:1224-1228): element jlo+k for column k. */
        if (bcmode == MGP_BCMODE_NONUNIFORM && !homog) {
            koff = bx->jlo - bx->ilo;
            if (koff < 0 || koff + nx - 1 >= nx)
                return fail(MGP_EINVAL, "nonuniform Dirichlet data on a y side needs jlo == ilo (reference indexes it with jlo:jhi)");
        }
        for (k = 0; k < nx; ++k) {
            double p0 = AT(p, k, j), p1 = AT(p, k, j - e), p2 = AT(p, k, j - 2 * e);
            if (bcmode == MGP_BCMODE_LAH)       AT(p, k, j + e) = -p0;
            else if (homog)                     AT(p, k, j + e) = -(three * p0) + p1 - fifth * p2;
            else if (bcmode == MGP_BCMODE_UNIFORM) AT(p, k, j + e) = sixteenfifth * bcd[0] - three * p0 + p1 - fifth * p2;
            else                                AT(p, k, j + e) = sixteenfifth * bcd[koff + k] - three * p0 + p1 - fifth * p2;
        }
    }
    return MGP_OK;
}

int or_fill_ghosts(const mgp_box *valid, mgp_array *phi, const mgp_bdry *bc,
                   const mgp_geo *geo, int homog, int do_neum)
{
    const int nx = valid->nx, ny = valid->ny;
    V p = view(phi);
    G g;
    int s, rc, i, j;
    long jlo_all = -phi->ngy, jhi_all = ny - 1 + phi->ngy;
    long ilo_all = -phi->ngx, ihi_all = nx - 1 + phi->ngx;
    if (phi->ngx > 1 || phi->ngy > 1) return fail(MGP_EINVAL, "fill_ghosts: Can only handle 1 ghost layer max.");
    if (nx < 3 || ny < 3) return fail(MGP_EINVAL, "fill_ghosts: grid needs at least 3 cells per direction");
    g = gview(geo);
    for (s = 0; s < 4; ++s) {
        int dir = (s < 2) ? 1 : 2, side = (s % 2 == 0) ? -1 : 1;
        switch (bc->type[s]) {
        case MGP_BCTYPE_NEUM:
            if (do_neum) { rc = neum_dir_side(valid, p, bc, &g, homog, dir, side); if (rc) return rc; }
            break;
        case MGP_BCTYPE_DIRI:
            rc = diri_dir_side(valid, p, bc, homog, dir, side);
            if (rc) return rc;
            break;
        case MGP_BCTYPE_PERIODIC:
            if (s == MGP_XLO) for (j = 0; j < ny; ++j) AT(p, -1, j) = AT(p, nx - 1, j);
            if (s == MGP_XHI) for (j = 0; j < ny; ++j) AT(p, nx, j) = AT(p, 0, j);
            if (s == MGP_YLO) for (i = 0; i < nx; ++i) AT(p, i, -1) = AT(p, i, ny - 1);
            if (s == MGP_YHI) for (i = 0; i < nx; ++i) AT(p, i, ny) = AT(p, i, 0);
            break;
        case MGP_BCTYPE_EXTRAP0:
        case MGP_BCTYPE_EXTRAP1:
        case MGP_BCTYPE_EXTRAP2: {
            int t = bc->type[s];
            long a, lo = (dir == 1) ? jlo_all : ilo_all, hi = (dir == 1) ? jhi_all : ihi_all;
            for (a = lo; a <= hi; ++a) {
                double v0, v1, v2, *dst;
                if (s == MGP_XLO)      { v0 = AT(p, 0, a); v1 = AT(p, 1, a); v2 = AT(p, 2, a); dst = &AT(p, -1, a); }
                else if (s == MGP_XHI) { v0 = AT(p, nx - 1, a); v1 = AT(p, nx - 2, a); v2 = AT(p, nx - 3, a); dst = &AT(p, nx, a); }
                else if (s == MGP_YLO) { v0 = AT(p, a, 0); v1 = AT(p, a, 1); v2 = AT(p, a, 2); dst = &AT(p, a, -1); }
                else                   { v0 = AT(p, a, ny - 1); v1 = AT(p, a, ny - 2); v2 = AT(p, a, ny - 3); dst = &AT(p, a, ny); }
                if (t == MGP_BCTYPE_EXTRAP0) *dst = v0;
                else if (t == MGP_BCTYPE_EXTRAP1) *dst = two * v0 - v1;
                else *dst = three * (v0 - v1) + v2;
            }
            break;
        }
        case MGP_BCTYPE_NONE:
            break;
        case MGP_BCTYPE_CF:
            /* c2x/c2y are used uninitialised in the reference (AU:1296-1302). */
            return fail(MGP_ENOTSUP, "fill_ghosts: BCTYPE_CF is not supported");
        default:
            return fail(MGP_EINVAL, "fill_ghosts: invalid BCTYPE_");
        }
    }
    /* corners, AU:1460-1490 */
    if (bc->type[MGP_XLO] != MGP_BCTYPE_PERIODIC && bc->type[MGP_YLO] != MGP_BCTYPE_PERIODIC) {
        AT(p, -1, -1) = MGP_BOGUS_VAL;
        AT(p, -1, ny) = MGP_BOGUS_VAL;
        AT(p, nx, -1) = MGP_BOGUS_VAL;
        AT(p, nx, ny) = MGP_BOGUS_VAL;
    } else if (bc->type[MGP_XLO] == MGP_BCTYPE_PERIODIC && bc->type[MGP_YLO] == MGP_BCTYPE_PERIODIC) {
        AT(p, -1, -1) = AT(p, nx - 1, ny - 1);
        AT(p, -1, ny) = AT(p, nx - 1, 0);
        AT(p, nx, -1) = AT(p, 0, ny - 1);
        AT(p, nx, ny) = AT(p, 0, 0);
    } else if (bc->type[MGP_XLO] == MGP_BCTYPE_PERIODIC) {
        AT(p, -1, -1) = AT(p, nx - 1, -1);
        AT(p, -1, ny) = AT(p, nx - 1, ny);
        AT(p, nx, -1) = AT(p, 0, -1);
        AT(p, nx, ny) = AT(p, 0, ny);
    } else {
        AT(p, -1, -1) = AT(p, -1, ny - 1);
        AT(p, nx, -1) = AT(p, nx, ny - 1);
        AT(p, -1, ny) = AT(p, -1, 0);
        AT(p, nx, ny) = AT(p, nx, 0);
    }
    return MGP_OK;
}

/* extrapolate_ghosts, AU:1497-1566.  x columns over the full j range of the
 * allocation first, then y rows over the full i range. */
int or_extrapolate_ghosts(const mgp_box *valid, mgp_array *phi, int order)
{
    const int nx = valid->nx, ny = valid->ny;
    V p = view(phi);
    long a;
    if (phi->ngx > 1 || phi->ngy > 1) return fail(MGP_EINVAL, "extrapolate_ghosts: 1 ghost layer max");
    if (order < 0 || order > 3) return fail(MGP_EINVAL, "extrapolate_ghosts: order is not supported");
    if (phi->ngx > 0) {
        for (a = -phi->ngy; a <= ny - 1 + phi->ngy; ++a) {
            double l0 = AT(p, 0, a), l1 = AT(p, 1, a), l2 = AT(p, 2, a), l3 = (nx > 3) ? AT(p, 3, a) : 0.0;
            double h0 = AT(p, nx - 1, a), h1 = AT(p, nx - 2, a), h2 = AT(p, nx - 3, a), h3 = (nx > 3) ? AT(p, nx - 4, a) : 0.0;
            switch (order) {
            case 0: AT(p, -1, a) = l0; AT(p, nx, a) = h0; break;
            case 1: AT(p, -1, a) = two * l0 - l1; AT(p, nx, a) = two * h0 - h1; break;
            case 2: AT(p, -1, a) = three * (l0 - l1) + l2; AT(p, nx, a) = three * (h0 - h1) + h2; break;
            default: AT(p, -1, a) = four * (l0 + l2) - six * l1 - l3; AT(p, nx, a) = four * (h0 + h2) - six * h1 - h3; break;
            }
        }
    }
    if (phi->ngy > 0) {
        for (a = -phi->ngx; a <= nx - 1 + phi->ngx; ++a) {
            double l0 = AT(p, a, 0), l1 = AT(p, a, 1), l2 = AT(p, a, 2), l3 = (ny > 3) ? AT(p, a, 3) : 0.0;
            double h0 = AT(p, a, ny - 1), h1 = AT(p, a, ny - 2), h2 = AT(p, a, ny - 3), h3 = (ny > 3) ? AT(p, a, ny - 4) : 0.0;
            switch (order) {
            case 0: AT(p, a, -1) = l0; AT(p, a, ny) = h0; break;
            case 1: AT(p, a, -1) = two * l0 - l1; AT(p, a, ny) = two * h0 - h1; break;
            case 2: AT(p, a, -1) = three * (l0 - l1) + l2; AT(p, a, ny) = three * (h0 - h1) + h2; break;
            default: AT(p, a, -1) = four * (l0 + l2) - six * l1 - l3; AT(p, a, ny) = four * (h0 + h2) - six * h1 - h3; break;
            }
        }
    }
    return MGP_OK;
}

/* ---- the mapped 9-point operator: P2:886-1319 ---------------------------- */

typedef struct { double p, pe, pw, pn, ps, ee, ew, en, es, ene, enw, ese, esw; } st9;

/* The transverse values of the nine region blocks of compute_laplacian.
 * c points at phi(i,j); xr/yr = RLO, RMID, RHI. */
static inline void gather(const double *c, long ld, int xr, int yr, st9 *s)
{
#define P(di, dj) c[(di) + (long)(dj) * ld]
    double p = P(0, 0), pe = P(1, 0), pw = P(-1, 0), pn = P(0, 1), ps = P(0, -1);
    double ee, ew, en, es, ene, enw, ese, esw;
    s->p = p; s->pe = pe; s->pw = pw; s->pn = pn; s->ps = ps;
    if (yr == RLO) {
        if (xr == RLO) {                      /* P2:937-958 */
            ee = P(1, 0); en = P(0, 1);
            ew = three * (p - ee) + P(2, 0);
            es = three * (p - en) + P(0, 2);
            ene = P(1, 1);
            enw = three * (en - ene) + P(2, 1);
            ese = three * (ee - ene) + P(1, 2);
            esw = half * ((three * (es - ese) + P(2, -1)) + (three * (ew - enw) + P(-1, 2)));
        } else if (xr == RMID) {              /* P2:986-1002 */
            ee = P(1, 0); ew = P(-1, 0); en = P(0, 1);
            es = three * (p - en) + P(0, 2);
            ene = P(1, 1); enw = P(-1, 1);
            ese = three * (ee - ene) + P(1, 2);
            esw = three * (ew - enw) + P(-1, 2);
        } else {                              /* P2:1021-1039 */
            ew = P(-1, 0); en = P(0, 1);
            ee = three * (p - ew) + P(-2, 0);
            es = three * (p - en) + P(0, 2);
            enw = P(-1, 1);
            ene = three * (pn - enw) + P(-2, 1);
            esw = three * (pw - enw) + P(-1, 2);
            ese = half * ((three * (es - esw) + P(-2, -1)) + (three * (ee - ene) + P(1, 2)));
        }
    } else if (yr == RMID) {
        if (xr == RLO) {                      /* P2:1068-1085 */
            ee = P(1, 0); en = P(0, 1); es = P(0, -1);
            ew = three * (p - ee) + P(2, 0);
            ene = P(1, 1); ese = P(1, -1);
            enw = three * (en - ene) + P(2, 1);
            esw = three * (es - ese) + P(2, -1);
        } else if (xr == RMID) {              /* P2:1103-1125 */
            ee = P(1, 0); ew = P(-1, 0); en = P(0, 1); es = P(0, -1);
            ene = P(1, 1); enw = P(-1, 1); ese = P(1, -1); esw = P(-1, -1);
        } else {                              /* P2:1128-1147 */
            ew = P(-1, 0); en = P(0, 1); es = P(0, -1);
            ee = three * (p - ew) + P(-2, 0);
            enw = P(-1, 1); esw = P(-1, -1);
            ene = three * (en - enw) + P(-2, 1);
            ese = three * (es - esw) + P(-2, -1);
        }
    } else {
        if (xr == RLO) {                      /* P2:1176-1194 */
            ee = P(1, 0); es = P(0, -1);
            ew = three * (p - ee) + P(2, 0);
            en = three * (p - es) + P(0, -2);
            ese = P(1, -1);
            ene = three * (ee - ese) + P(1, -2);
            esw = three * (es - ese) + P(2, -1);
            enw = half * ((three * (ew - esw) + P(-1, -2)) + (three * (en - ene) + P(2, 1)));
        } else if (xr == RMID) {              /* P2:1223-1239 */
            ee = P(1, 0); ew = P(-1, 0); es = P(0, -1);
            en = three * (p - es) + P(0, -2);
            ese = P(1, -1); esw = P(-1, -1);
            ene = three * (ee - ese) + P(1, -2);
            enw = three * (ew - esw) + P(-1, -2);
        } else {                              /* P2:1258-1276 */
            ew = P(-1, 0); es = P(0, -1);
            ee = three * (p - ew) + P(-2, 0);
            en = three * (p - es) + P(0, -2);
            esw = P(-1, -1);
            enw = three * (ew - esw) + P(-1, -2);
            ese = three * (es - esw) + P(-2, -1);
            ene = half * ((three * (en - enw) + P(-2, 1)) + (three * (ee - ese) + P(1, -2)));
        }
    }
#undef P
    s->ee = ee; s->ew = ew; s->en = en; s->es = es;
    s->ene = ene; s->enw = enw; s->ese = ese; s->esw = esw;
}

/* Neumann replacement values of the four face fluxes. */
typedef struct {
    int neum[4];
    int homog;
    const double *d[4];
    int mode[4];
    int kyhi;   /* relative index the north-face data is read at (P2: data_yhi(j)) */
} NB;

static int nb_init(NB *nb, const mgp_box *b, const mgp_bdry *bc, int homog)
{
    int s;
    nb->homog = homog;
    for (s = 0; s < 4; ++s) {
        nb->neum[s] = (bc->type[s] == MGP_BCTYPE_NEUM);
        nb->d[s] = bc->data[s];
        nb->mode[s] = bc->mode[s];
    }
    nb->kyhi = 0;
    if (nb->neum[MGP_YHI] && !homog && bc->mode[MGP_YHI] != MGP_BCMODE_UNIFORM)
        return yside_index(b, b->jhi, &nb->kyhi);
    return MGP_OK;
}

static inline double nbval(const NB *nb, int s, int k)
{
    if (nb->homog) return zero;
    if (nb->mode[s] == MGP_BCMODE_UNIFORM) return nb->d[s][0];
    return nb->d[s][k];
}

/* One cell of compute_laplacian (P2:958-982 pattern).  Returns lap. */
static inline double lap_cell(const st9 *s, const G *g, int i, int j, double idx, double idy,
                              int xr, int yr, const NB *nb)
{
    double xfe = AT(g->xx, i + 1, j) * (s->pe - s->p) * idx + AT(g->xy, i + 1, j) * fourth * (s->ene - s->ese + s->en - s->es) * idy;
    double xfw = AT(g->xx, i, j) * (s->p - s->pw) * idx + AT(g->xy, i, j) * fourth * (s->en - s->es + s->enw - s->esw) * idy;
    double yfn = AT(g->yy, i, j + 1) * (s->pn - s->p) * idy + AT(g->yx, i, j + 1) * fourth * (s->ene - s->enw + s->ee - s->ew) * idx;
    double yfs = AT(g->yy, i, j) * (s->p - s->ps) * idy + AT(g->yx, i, j) * fourth * (s->ee - s->ew + s->ese - s->esw) * idx;
    if (xr == RLO && nb->neum[MGP_XLO]) xfw = nbval(nb, MGP_XLO, j);
    if (yr == RLO && nb->neum[MGP_YLO]) yfs = nbval(nb, MGP_YLO, i);
    if (xr == RHI && nb->neum[MGP_XHI]) xfe = nbval(nb, MGP_XHI, j);
    if (yr == RHI && nb->neum[MGP_YHI]) yfn = nbval(nb, MGP_YHI, nb->kyhi);
    return (xfe - xfw) * idx + (yfn - yfs) * idy;
}

static inline int xregion(int i, int nx, int perx_lo, int perx_hi)
{
    if (i == 0 && !perx_lo) return RLO;
    if (i == nx - 1 && !perx_hi) return RHI;
    return RMID;
}

static int check_op(const mgp_box *b, const mgp_bdry *bc)
{
    int s;
    for (s = 0; s < 4; ++s)
        if (bc->mode[s] == MGP_BCMODE_LAH) return fail(MGP_EINVAL, "Poisson2d::compute_invdiags received BCMODE_LAH.");
    if (b->nx < 3 || b->ny < 3) return fail(MGP_EINVAL, "operator needs at least 3 cells per direction");
    return MGP_OK;
}

int or_compute_laplacian(const mgp_box *valid, mgp_array *lap, mgp_array *phi,
                         const mgp_geo *geo, const mgp_bdry *bc, int homog, int jscale)
{
    const int nx = valid->nx, ny = valid->ny;
    int rc, i, j, px0, px1, py0, py1;
    NB nb;
    V L = view(lap), P;
    G g;
    double idx, idy;
    st9 s;
    if ((rc = check_op(valid, bc))) return rc;
    if ((rc = nb_init(&nb, valid, bc, homog))) return rc;
    g = gview(geo);
    idx = one / geo->dx;
    idy = one / geo->dy;
    if ((rc = or_fill_ghosts(valid, phi, bc, geo, homog, 0))) return rc;   /* P2:935 */
    P = view(phi);
    px0 = bc->type[MGP_XLO] == MGP_BCTYPE_PERIODIC; px1 = bc->type[MGP_XHI] == MGP_BCTYPE_PERIODIC;
    py0 = bc->type[MGP_YLO] == MGP_BCTYPE_PERIODIC; py1 = bc->type[MGP_YHI] == MGP_BCTYPE_PERIODIC;
    for (j = 0; j < ny; ++j) {
        int yr = xregion(j, ny, py0, py1);
        for (i = 0; i < nx; ++i) {
            int xr = xregion(i, nx, px0, px1);
            gather(&AT(P, i, j), P.ld, xr, yr, &s);
            AT(L, i, j) = lap_cell(&s, &g, i, j, idx, idy, xr, yr, &nb);
        }
    }
    if (jscale)   /* P2:1311-1317 */
        for (j = 0; j < ny; ++j)
            for (i = 0; i < nx; ++i) AT(L, i, j) = AT(L, i, j) / AT(g.J, i, j);
    return MGP_OK;
}

int or_compute_residual(const mgp_box *valid, mgp_array *res, const mgp_array *rhs,
                        mgp_array *phi, const mgp_geo *geo, const mgp_bdry *bc,
                        int homog, int jscale)
{
    int rc, i, j;
    V R, F;
    if ((rc = or_compute_laplacian(valid, res, phi, geo, bc, homog, jscale))) return rc;
    R = view(res);
    F = view(rhs);
    for (j = 0; j < valid->ny; ++j)
        for (i = 0; i < valid->nx; ++i) AT(R, i, j) = AT(F, i, j) - AT(R, i, j);   /* P2:1351 */
    return MGP_OK;
}

/* compute_invdiags, P2:16-388: the same stencil applied to a unit impulse at
 * (i,j) with every neighbour and ghost zero, then inverted. */
static int g_diri_coupled = 0;
void or_set_dirichlet_coupled_diagonal(int on) { g_diri_coupled = on; }

int or_compute_invdiags(const mgp_box *valid, mgp_array *invd, const mgp_geo *geo,
                        const mgp_bdry *bc, int homog)
{
    const int nx = valid->nx, ny = valid->ny;
    int rc, i, j, px0, px1, py0, py1;
    NB nb;
    V D = view(invd);
    G g;
    double idx, idy, patch[25];
    st9 s;
    if ((rc = check_op(valid, bc))) return rc;
    if ((rc = nb_init(&nb, valid, bc, homog))) return rc;
    g = gview(geo);
    idx = one / geo->dx;
    idy = one / geo->dy;
    memset(patch, 0, sizeof patch);
    patch[12] = one;
    px0 = bc->type[MGP_XLO] == MGP_BCTYPE_PERIODIC; px1 = bc->type[MGP_XHI] == MGP_BCTYPE_PERIODIC;
    py0 = bc->type[MGP_YLO] == MGP_BCTYPE_PERIODIC; py1 = bc->type[MGP_YHI] == MGP_BCTYPE_PERIODIC;
    for (j = 0; j < ny; ++j) {
        int yr = xregion(j, ny, py0, py1);
        for (i = 0; i < nx; ++i) {
            int xr = xregion(i, nx, px0, px1);
            if (g_diri_coupled) {
                /* The order-3 Dirichlet ghost of the cell's own row/column
                 * moves by -3 per unit change of the cell (AU:1162-1166). */
                patch[11] = (xr == RLO && bc->type[MGP_XLO] == MGP_BCTYPE_DIRI) ? -three : zero;
                patch[13] = (xr == RHI && bc->type[MGP_XHI] == MGP_BCTYPE_DIRI) ? -three : zero;
                patch[7] = (yr == RLO && bc->type[MGP_YLO] == MGP_BCTYPE_DIRI) ? -three : zero;
                patch[17] = (yr == RHI && bc->type[MGP_YHI] == MGP_BCTYPE_DIRI) ? -three : zero;
            }
            gather(&patch[12], 5, xr, yr, &s);
            AT(D, i, j) = lap_cell(&s, &g, i, j, idx, idy, xr, yr, &nb);
        }
    }
    for (j = 0; j < ny; ++j)
        for (i = 0; i < nx; ++i) AT(D, i, j) = one / AT(D, i, j);   /* P2:386 */
    return MGP_OK;
}

int or_boundary_fluxes(const mgp_box *valid, const mgp_array *phi, const mgp_geo *geo,
                       double *xlo, double *xhi, double *ylo, double *yhi)
{
    const int nx = valid->nx, ny = valid->ny;
    V P = view(phi);
    G g = gview(geo);
    double idx = one / geo->dx, idy = one / geo->dy;
    st9 s;
    int i, j;
    for (j = 0; j < ny; ++j) {
        int yr = xregion(j, ny, 0, 0);
        gather(&AT(P, 0, j), P.ld, RLO, yr, &s);
        xlo[j] = AT(g.xx, 0, j) * (s.p - s.pw) * idx + AT(g.xy, 0, j) * fourth * (s.en - s.es + s.enw - s.esw) * idy;
        gather(&AT(P, nx - 1, j), P.ld, RHI, yr, &s);
        xhi[j] = AT(g.xx, nx, j) * (s.pe - s.p) * idx + AT(g.xy, nx, j) * fourth * (s.ene - s.ese + s.en - s.es) * idy;
    }
    for (i = 0; i < nx; ++i) {
        int xr = xregion(i, nx, 0, 0);
        gather(&AT(P, i, 0), P.ld, xr, RLO, &s);
        ylo[i] = AT(g.yy, i, 0) * (s.p - s.ps) * idy + AT(g.yx, i, 0) * fourth * (s.ee - s.ew + s.ese - s.esw) * idx;
        gather(&AT(P, i, ny - 1), P.ld, xr, RHI, &s);
        yhi[i] = AT(g.yy, i, ny) * (s.pn - s.p) * idy + AT(g.yx, i, ny) * fourth * (s.ene - s.enw + s.ee - s.ew) * idx;
    }
    return MGP_OK;
}

static mgp_array alloc_like(int nx, int ny, int ngx, int ngy);

/* ---- gradient and divergence: P2:404-879, AU:1571-1622 ------------------ */
/* compute_pd (P2:404-795): d(phi)/d(dir) onto the faces nodal in `nodedir`
 * (1: x-faces, (nx+1) x ny; 2: y-faces, nx x (ny+1)).  The nodal derivative
 * reads the ghosts; the transverse one uses interior differences, one-sided
 * ones at the sides across it (P2:455-478, P2:618-641) and the
 * compute_laplacian region values on the faces along the sides
 * (simple_bdry_stencil = .false., P2:488-611, P2:651-793). */
int or_compute_pd(const mgp_box *valid, mgp_array *pd, const mgp_array *phi, int dir, int nodedir)
{
    const int nx = valid->nx, ny = valid->ny;
    V D = view(pd), P = view(phi);
    st9 s;
    int i, j;
    if ((dir != 1 && dir != 2) || (nodedir != 1 && nodedir != 2)) return fail(MGP_EINVAL, "compute_pd: bad direction");
    if (nx < 3 || ny < 3) return fail(MGP_EINVAL, "compute_pd needs at least 3 cells per direction");
    if (dir == 1 && nodedir == 1) {   /* P2:446-449 */
        const double scale = one / valid->dx;
        for (j = 0; j < ny; ++j)
            for (i = 0; i <= nx; ++i) AT(D, i, j) = scale * (AT(P, i, j) - AT(P, i - 1, j));
    } else if (dir == 2 && nodedir == 2) {   /* P2:614-617 */
        const double scale = one / valid->dy;
        for (j = 0; j <= ny; ++j)
            for (i = 0; i < nx; ++i) AT(D, i, j) = scale * (AT(P, i, j) - AT(P, i, j - 1));
    } else if (dir == 1) {   /* d/dx onto y-faces, P2:450-612 */
        const double scale = fourth / valid->dx;
        for (j = 1; j < ny; ++j)
            for (i = 1; i < nx - 1; ++i)
                AT(D, i, j) = scale * (AT(P, i + 1, j) - AT(P, i - 1, j) + AT(P, i + 1, j - 1) - AT(P, i - 1, j - 1));
        for (j = 1; j < ny; ++j) {
            AT(D, 0, j) = -scale * (three * AT(P, 0, j) - four * AT(P, 1, j) + AT(P, 2, j) + three * AT(P, 0, j - 1) -
                                    four * AT(P, 1, j - 1) + AT(P, 2, j - 1));
            AT(D, nx - 1, j) = scale * (three * AT(P, nx - 1, j) - four * AT(P, nx - 2, j) + AT(P, nx - 3, j) +
                                        three * AT(P, nx - 1, j - 1) - four * AT(P, nx - 2, j - 1) +
                                        AT(P, nx - 3, j - 1));
        }
        for (i = 0; i < nx; ++i) {
            const int xr = xregion(i, nx, 0, 0);
            gather(&AT(P, i, 0), P.ld, xr, RLO, &s);
            AT(D, i, 0) = scale * (s.ee - s.ew + s.ese - s.esw);
            gather(&AT(P, i, ny - 1), P.ld, xr, RHI, &s);
            AT(D, i, ny) = scale * (s.ene - s.enw + s.ee - s.ew);
        }
    } else {   /* d/dy onto x-faces, P2:613-794 */
        const double scale = fourth / valid->dy;
        for (j = 1; j < ny - 1; ++j)
            for (i = 1; i < nx; ++i)
                AT(D, i, j) = scale * (AT(P, i, j + 1) - AT(P, i, j - 1) + AT(P, i - 1, j + 1) - AT(P, i - 1, j - 1));
        for (i = 1; i < nx; ++i) {
            AT(D, i, 0) = -scale * (three * AT(P, i, 0) - four * AT(P, i, 1) + AT(P, i, 2) + three * AT(P, i - 1, 0) -
                                    four * AT(P, i - 1, 1) + AT(P, i - 1, 2));
            AT(D, i, ny - 1) = scale * (three * AT(P, i, ny - 1) - four * AT(P, i, ny - 2) + AT(P, i, ny - 3) +
                                        three * AT(P, i - 1, ny - 1) - four * AT(P, i - 1, ny - 2) +
                                        AT(P, i - 1, ny - 3));
        }
        for (j = 0; j < ny; ++j) {
            const int yr = xregion(j, ny, 0, 0);
            gather(&AT(P, 0, j), P.ld, RLO, yr, &s);
            AT(D, 0, j) = scale * (s.en - s.es + s.enw - s.esw);
            gather(&AT(P, nx - 1, j), P.ld, RHI, yr, &s);
            AT(D, nx, j) = scale * (s.ene - s.ese + s.en - s.es);
        }
    }
    return MGP_OK;
}

/* fill_boundary_fluxes (AU:1574-1622): the faces on Neumann sides take the
 * BC flux (0 when homogeneous).  UNIFORM values (and zeros) go to the whole
 * face column or row, ghost rows included (the `(ilo,:)` sections);
 * NONUNIFORM values to the valid faces. */
int or_fill_boundary_fluxes(const mgp_box *valid, mgp_array *xflux, mgp_array *yflux, const mgp_bdry *bc, int homog)
{
    const int nx = valid->nx, ny = valid->ny;
    V X = view(xflux), Y = view(yflux);
    int s, k;
    for (s = 0; s < 4; ++s) {
        const int isx = s < 2, n = isx ? ny : nx;
        const int ng = isx ? xflux->ngy : yflux->ngx;
        const int edge = (s == MGP_XLO || s == MGP_YLO) ? 0 : (isx ? nx : ny);
        if (bc->type[s] != MGP_BCTYPE_NEUM) continue;
        for (k = -ng; k < n + ng; ++k) {
            double v;
            if (homog || bc->mode[s] == MGP_BCMODE_LAH) v = zero;
            else if (bc->mode[s] == MGP_BCMODE_UNIFORM) v = bc->data[s][0];
            else if (k >= 0 && k < n) v = bc->data[s][k];
            else continue;
            if (isx) AT(X, edge, k) = v;
            else AT(Y, k, edge) = v;
        }
    }
    return MGP_OK;
}

/* compute_grad (P2:809-850): J Grad[phi] on the faces; phi's ghosts are
 * filled first (do_neum = .false.). */
int or_compute_grad(const mgp_box *valid, mgp_array *xflux, mgp_array *yflux, mgp_array *phi, const mgp_geo *geo,
                    const mgp_bdry *bc, int homog)
{
    const int nx = valid->nx, ny = valid->ny;
    mgp_array xwk = alloc_like(nx + 1, ny, 0, 0), ywk = alloc_like(nx, ny + 1, 0, 0);
    V X = view(xflux), Y = view(yflux), XW, YW;
    G g = gview(geo);
    int rc = MGP_OK, i, j;
    if (!xwk.data || !ywk.data) { rc = fail(MGP_ENOMEM, "compute_grad: out of memory"); goto done; }
    XW = view(&xwk);
    YW = view(&ywk);
    if ((rc = or_fill_ghosts(valid, phi, bc, geo, homog, 0))) goto done;
    if ((rc = or_compute_pd(valid, xflux, phi, 1, 1))) goto done;
    if ((rc = or_compute_pd(valid, &xwk, phi, 2, 1))) goto done;
    for (j = 0; j < ny; ++j)
        for (i = 0; i <= nx; ++i) AT(X, i, j) = AT(g.xx, i, j) * AT(X, i, j) + AT(g.xy, i, j) * AT(XW, i, j);
    if ((rc = or_compute_pd(valid, &ywk, phi, 1, 2))) goto done;
    if ((rc = or_compute_pd(valid, yflux, phi, 2, 2))) goto done;
    for (j = 0; j <= ny; ++j)
        for (i = 0; i < nx; ++i) AT(Y, i, j) = AT(g.yx, i, j) * AT(YW, i, j) + AT(g.yy, i, j) * AT(Y, i, j);
    rc = or_fill_boundary_fluxes(valid, xflux, yflux, bc, homog);
done:
    free(xwk.data);
    free(ywk.data);
    return rc;
}

/* compute_div (P2:860-879): J Div[flux] = (xflux(i+1)-xflux(i))/dx + (yflux(j+1)-yflux(j))/dy. */
int or_compute_div(const mgp_box *valid, mgp_array *div, const mgp_array *xflux, const mgp_array *yflux)
{
    const double invdx = one / valid->dx, invdy = one / valid->dy;
    V D = view(div), X = view(xflux), Y = view(yflux);
    int i, j;
    for (j = 0; j < valid->ny; ++j)
        for (i = 0; i < valid->nx; ++i)
            AT(D, i, j) = invdx * (AT(X, i + 1, j) - AT(X, i, j)) + invdy * (AT(Y, i, j + 1) - AT(Y, i, j));
    return MGP_OK;
}

/* ---- reductions: AU:637-661, AU:670-710, AU:753-796 --------------------- */
double or_pnorm(const mgp_box *valid, const mgp_array *bd, int p)
{
    V B = view(bd);
    double volScale = valid->dx * valid->dy, pn = zero;
    int i, j;
    if (p == 0) {
        for (j = 0; j < valid->ny; ++j)
            for (i = 0; i < valid->nx; ++i) { double a = fabs(AT(B, i, j)); if (a > pn) pn = a; }
    } else if (p == 1) {
        for (j = 0; j < valid->ny; ++j)
            for (i = 0; i < valid->nx; ++i) pn = pn + volScale * fabs(AT(B, i, j));
    } else if (p == 2) {
        for (j = 0; j < valid->ny; ++j)
            for (i = 0; i < valid->nx; ++i) { double v = AT(B, i, j); pn = pn + volScale * (v * v); }
        pn = sqrt(pn);
    } else {
        for (j = 0; j < valid->ny; ++j)
            for (i = 0; i < valid->nx; ++i) pn = pn + volScale * pow(fabs(AT(B, i, j)), p);
        pn = pow(pn, one / p);
    }
    return pn;
}

double or_inner_prod(const mgp_box *valid, const mgp_array *a, const mgp_array *b)
{
    V A = view(a), B = view(b);
    double vol = valid->dx * valid->dy, ip = zero;
    int i, j;
    for (j = 0; j < valid->ny; ++j) {
        double dot = zero;
        for (i = 0; i < valid->nx; ++i) dot = dot + AT(A, i, j) * AT(B, i, j);
        ip = ip + vol * dot;
    }
    return ip;
}

double or_integrate2d(const mgp_box *valid, const mgp_array *bd, const mgp_geo *geo, int jscale)
{
    V B = view(bd), J = view(&geo->J);
    double volScale = geo->dx * geo->dy, sum = zero;
    int i, j;
    for (j = 0; j < valid->ny; ++j)
        for (i = 0; i < valid->nx; ++i)
            sum = jscale ? sum + volScale * AT(J, i, j) * AT(B, i, j) : sum + volScale * AT(B, i, j);
    return sum;
}

/* ---- relax_gs: P2:1460-1988 --------------------------------------------- */

static void zero_all(mgp_array *a, int nx, int ny)
{
    long r, c, rows = alloc_rows(a, ny), cols = alloc_cols(a, nx);
    for (r = 0; r < rows; ++r)
        for (c = 0; c < cols; ++c) a->data[c + r * a->ld] = zero;
}

/* One Gauss-Seidel update of cell (i,j) (P2:1768-1771). */
static inline void gs_cell(V P, V F, V D, const G *g, int i, int j, double idx, double idy,
                           int xr, int yr, const NB *nb, double omega)
{
    st9 s;
    double lphi, newphi;
    gather(&AT(P, i, j), P.ld, xr, yr, &s);
    lphi = lap_cell(&s, g, i, j, idx, idy, xr, yr, nb);
    newphi = AT(P, i, j) + (AT(F, i, j) - lphi) * AT(D, i, j);
    AT(P, i, j) = omega * newphi + (one - omega) * AT(P, i, j);
}

/* One sweep: ghosts once, then the cells in lexicographic or 4-colour order. */
static int gs_sweep(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs, const mgp_geo *geo,
                    const mgp_bdry *bc, int homog, const NB *nb, const mgp_array *invd,
                    double omega, int gs_order)
{
    const int nx = valid->nx, ny = valid->ny;
    int rc, i, j, c, px0, px1, py0, py1;
    V P, F = view(rhs), D = view(invd);
    G g = gview(geo);
    double idx = one / geo->dx, idy = one / geo->dy;
    if ((rc = or_fill_ghosts(valid, phi, bc, geo, homog, 0))) return rc;   /* P2:1556 */
    P = view(phi);
    px0 = bc->type[MGP_XLO] == MGP_BCTYPE_PERIODIC; px1 = bc->type[MGP_XHI] == MGP_BCTYPE_PERIODIC;
    py0 = bc->type[MGP_YLO] == MGP_BCTYPE_PERIODIC; py1 = bc->type[MGP_YHI] == MGP_BCTYPE_PERIODIC;
    if (gs_order == 0) {
        for (j = 0; j < ny; ++j) {
            int yr = xregion(j, ny, py0, py1);
            i = 0;
            gs_cell(P, F, D, &g, i, j, idx, idy, xregion(i, nx, px0, px1), yr, nb, omega);
            if (yr == RMID)
                for (i = 1; i < nx - 1; ++i) gs_cell(P, F, D, &g, i, j, idx, idy, RMID, RMID, nb, omega);
            else
                for (i = 1; i < nx - 1; ++i) gs_cell(P, F, D, &g, i, j, idx, idy, RMID, yr, nb, omega);
            i = nx - 1;
            gs_cell(P, F, D, &g, i, j, idx, idy, xregion(i, nx, px0, px1), yr, nb, omega);
        }
    } else {
        /* The device order.  Colours (i mod 2, j mod 2) = (0,0), (1,1), (1,0),
         * (0,1) -- the cells with i+j even first, which is red-black order
         * for 5-point couplings.  First the four colours over the interior
         * cells (region MID in both directions: their stencil reaches one
         * cell, so a colour is an independent set), then the boundary cells
         * (whose stencil reaches two cells inward): edge cells colour by
         * colour, then the four corners one after another. */
        static const int ci_of[4] = {0, 1, 1, 0}, cj_of[4] = {0, 1, 0, 1};
        for (c = 0; c < 4; ++c) {
            int ci = ci_of[c], cj = cj_of[c];
            for (j = cj; j < ny; j += 2) {
                int yr = xregion(j, ny, py0, py1);
                if (yr != RMID) continue;
                for (i = ci; i < nx; i += 2) {
                    int xr = xregion(i, nx, px0, px1);
                    if (xr == RMID) gs_cell(P, F, D, &g, i, j, idx, idy, xr, yr, nb, omega);
                }
            }
        }
        for (c = 0; c < 4; ++c) {
            int ci = ci_of[c], cj = cj_of[c];
            for (j = cj; j < ny; j += 2) {
                int yr = xregion(j, ny, py0, py1);
                for (i = ci; i < nx; i += 2) {
                    int xr = xregion(i, nx, px0, px1);
                    if ((xr == RMID) != (yr == RMID)) gs_cell(P, F, D, &g, i, j, idx, idy, xr, yr, nb, omega);
                }
            }
        }
        {
            static const int cx[4] = {0, 1, 0, 1}, cy[4] = {0, 0, 1, 1};
            for (c = 0; c < 4; ++c) {
                int ii = cx[c] ? nx - 1 : 0, jj = cy[c] ? ny - 1 : 0;
                int xr = xregion(ii, nx, px0, px1), yr = xregion(jj, ny, py0, py1);
                if (xr != RMID && yr != RMID) gs_cell(P, F, D, &g, ii, jj, idx, idy, xr, yr, nb, omega);
            }
        }
    }
    return MGP_OK;
}

static mgp_array alloc_like(int nx, int ny, int ngx, int ngy)
{
    mgp_array a;
    a.ngx = ngx;
    a.ngy = ngy;
    a.ld = nx + 2 * ngx;
    a.data = (double *)calloc((size_t)(nx + 2 * ngx) * (size_t)(ny + 2 * ngy), sizeof(double));
    return a;
}

int or_relax_gs(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                const mgp_geo *geo, const mgp_bdry *bc, int homog, const mgp_array *invd,
                double omega, double tol, int maxiters, int zerophi, int verbosity, int gs_order)
{
    int rc, iter;
    NB nb;
    mgp_array r = {0};
    double rscale = 0, relres;
    if (maxiters == 0) return MGP_OK;
    if ((rc = check_op(valid, bc))) return rc;
    if ((rc = nb_init(&nb, valid, bc, homog))) return rc;
    if (zerophi) zero_all(phi, valid->nx, valid->ny);
    if (tol > zero) {
        r = alloc_like(valid->nx, valid->ny, 0, 0);
        if (!r.data) return fail(MGP_ENOMEM, "relax_gs: out of memory");
        if ((rc = or_compute_residual(valid, &r, rhs, phi, geo, bc, homog, 0))) { free(r.data); return rc; }
        rscale = or_pnorm(valid, &r, 2);
        if (rscale == zero) rscale = one;
        if (verbosity >= 3) printf("scale |res| = %.16e\n", rscale);
    }
    for (iter = 1; iter <= maxiters; ++iter) {
        if ((rc = gs_sweep(valid, phi, rhs, geo, bc, homog, &nb, invd, omega, gs_order))) break;
        if (tol > zero) {
            if ((rc = or_compute_residual(valid, &r, rhs, phi, geo, bc, homog, 0))) break;
            relres = or_pnorm(valid, &r, 2) / rscale;
            if (verbosity >= 3) printf("iter %d: rel |res| = %.16e\n", iter, relres);
            if (relres <= tol) break;
        }
    }
    free(r.data);
    return rc;
}

/* relax_jacobi (P2:1358-1451): phi += r*invdiag for every cell, weighted by
 * omega, then the residual again; tol > 0 stops on the relative residual. */
int or_relax_jacobi(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs, const mgp_geo *geo,
                    const mgp_bdry *bc, int homog, const mgp_array *invd, double omega, double tol, int maxiters,
                    int zerophi, int verbosity)
{
    const int nx = valid->nx, ny = valid->ny;
    mgp_array r;
    V R, PH, D;
    double rscale = one, relres;
    int rc, iter, i, j;
    if (maxiters == 0) return MGP_OK;
    if ((rc = check_op(valid, bc))) return rc;
    r = alloc_like(nx, ny, 0, 0);
    if (!r.data) return fail(MGP_ENOMEM, "relax_jacobi: out of memory");
    R = view(&r); PH = view(phi); D = view(invd);
    if (zerophi) zero_all(phi, nx, ny);
    if ((rc = or_compute_residual(valid, &r, rhs, phi, geo, bc, homog, 0))) goto done;
    if (tol > zero) {
        rscale = or_pnorm(valid, &r, 2);
        if (rscale == zero) rscale = one;
        if (verbosity >= 3) printf("scale |res| = %.16e\n", rscale);
    }
    for (iter = 1; iter <= maxiters; ++iter) {
        for (j = 0; j < ny; ++j)
            for (i = 0; i < nx; ++i) {
                const double newphi = AT(PH, i, j) + AT(R, i, j) * AT(D, i, j);
                AT(PH, i, j) = omega * newphi + (one - omega) * AT(PH, i, j);
            }
        if ((rc = or_compute_residual(valid, &r, rhs, phi, geo, bc, homog, 0))) break;
        if (tol > zero) {
            relres = or_pnorm(valid, &r, 2) / rscale;
            if (verbosity >= 3) printf("iter %d: rel |res| = %.16e\n", iter, relres);
            if (relres <= tol) break;
        }
    }
done:
    free(r.data);
    return rc;
}

/* ---- solve_bicgstab2: P2:2253-2477 and DD:339-566 ------------------------ */

typedef struct {
    int dd;          /* 0: Poisson2D operators, 1: DeferredPoisson2D operators */
    int norm_type;   /* 2 (P2:2278) or 0 (DD:364)                              */
    double omega;    /* preconditioner weight: 1-1/3 (P2:2378) or 4/5 (DD:365) */
    int gs_order;
} KOps;

static int k_residual(const KOps *o, const mgp_box *b, mgp_array *res, const mgp_array *rhs, mgp_array *phi,
                      const mgp_geo *geo, const mgp_bdry *bc, int homog)
{
    return o->dd ? or_dd_compute_residual(b, res, rhs, phi, geo, bc, homog)
                 : or_compute_residual(b, res, rhs, phi, geo, bc, homog, 0);
}
static int k_laplacian(const KOps *o, const mgp_box *b, mgp_array *lap, mgp_array *phi,
                       const mgp_geo *geo, const mgp_bdry *bc, int homog)
{
    return o->dd ? or_dd_compute_laplacian(b, lap, phi, geo, bc, homog)
                 : or_compute_laplacian(b, lap, phi, geo, bc, homog, 0);
}
static int k_relax(const KOps *o, const mgp_box *b, mgp_array *phi, const mgp_array *rhs, const mgp_geo *geo,
                   const mgp_bdry *bc, const mgp_array *invd)
{
    return o->dd ? or_dd_relax_gs(b, phi, rhs, geo, bc, 1, invd, o->omega, -one, 2, 0, 0, o->gs_order)
                 : or_relax_gs(b, phi, rhs, geo, bc, 1, invd, o->omega, -one, 2, 0, 0, o->gs_order);
}

/* Whole-allocation elementwise ops on arrays of identical shape. */
#define FOR_ALL(a, nx, ny, body)                                                     \
    do {                                                                             \
        long _r, _c, _rows = alloc_rows((a), (ny)), _cols = alloc_cols((a), (nx));   \
        for (_r = 0; _r < _rows; ++_r)                                               \
            for (_c = 0; _c < _cols; ++_c) { long _k = _c + _r * (a)->ld; body; }    \
    } while (0)

static int bicgstab_impl(const KOps *o, const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                         const mgp_geo *geo, const mgp_bdry *bc, int homog, const mgp_array *invd,
                         double tol, int max_iters, int max_restarts, int zerophi, int verbosity)
{
    const double reps = 1.0e-12, hang = 1.0e-7, small = 1.0e-30;
    const int nx = valid->nx, ny = valid->ny;
    mgp_array e, pt, st, r, rt, p, t, v;
    double rho[4] = {0, 0, 0, 0}, norm[2], alpha[2] = {0, 0}, beta[2] = {0, 0}, omega[2] = {0, 0};
    double initial_norm, initial_rnorm, m;
    int recount = 0, i = 0, restarts = 0, init = 1, rc = MGP_OK;
    V R, RT, Pv, Tv, Vv, E, PT, ST, D, PH;
    long a, b2;

    if (max_iters == 0) return MGP_OK;
    if (zerophi) zero_all(phi, nx, ny);
    e = alloc_like(nx, ny, phi->ngx, phi->ngy);
    pt = alloc_like(nx, ny, phi->ngx, phi->ngy);
    st = alloc_like(nx, ny, phi->ngx, phi->ngy);
    r = alloc_like(nx, ny, rhs->ngx, rhs->ngy);
    rt = alloc_like(nx, ny, rhs->ngx, rhs->ngy);
    p = alloc_like(nx, ny, rhs->ngx, rhs->ngy);
    t = alloc_like(nx, ny, rhs->ngx, rhs->ngy);
    v = alloc_like(nx, ny, rhs->ngx, rhs->ngy);
    if (!e.data || !pt.data || !st.data || !r.data || !rt.data || !p.data || !t.data || !v.data) {
        rc = fail(MGP_ENOMEM, "bicgstab: out of memory");
        goto done;
    }
    R = view(&r); RT = view(&rt); Pv = view(&p); Tv = view(&t); Vv = view(&v);
    E = view(&e); PT = view(&pt); ST = view(&st); D = view(invd); PH = view(phi);

    if ((rc = k_residual(o, valid, &r, rhs, phi, geo, bc, homog))) goto done;
    memcpy(rt.data, r.data, sizeof(double) * (size_t)alloc_rows(&r, ny) * (size_t)alloc_cols(&r, nx));
    norm[0] = or_pnorm(valid, &r, o->norm_type);
    initial_norm = norm[0];
    initial_rnorm = norm[0];
    norm[1] = norm[0];

    while (((i < max_iters) && (norm[0] > tol * norm[1])) && (norm[1] > zero)) {
        i = i + 1;
        norm[1] = norm[0];
        alpha[1] = alpha[0];
        beta[1] = beta[0];
        omega[1] = omega[0];
        rho[3] = rho[2];
        rho[2] = rho[1];
        rho[1] = or_inner_prod(valid, &rt, &r);
        if (rho[1] == zero) {
            FOR_ALL(phi, nx, ny, phi->data[_k] = phi->data[_k] + e.data[_c + _r * e.ld]);
            goto done;
        }
        if (init) {
            FOR_ALL(&p, nx, ny, p.data[_k] = r.data[_k]);
            init = 0;
        } else {
            beta[1] = (rho[1] / rho[2]) * (alpha[1] / omega[1]);
            FOR_ALL(&p, nx, ny, p.data[_k] = beta[1] * (p.data[_k] - omega[1] * v.data[_k]) + r.data[_k]);
        }
        for (b2 = 0; b2 < ny; ++b2)
            for (a = 0; a < nx; ++a) AT(PT, a, b2) = AT(Pv, a, b2) * AT(D, a, b2);
        if ((rc = k_relax(o, valid, &pt, &p, geo, bc, invd))) goto done;
        if ((rc = k_laplacian(o, valid, &v, &pt, geo, bc, 1))) goto done;
        m = or_inner_prod(valid, &rt, &v);
        alpha[0] = rho[1] / m;
        if (fabs(m) > small * fabs(rho[1])) {
            FOR_ALL(&r, nx, ny, r.data[_k] = r.data[_k] - alpha[0] * v.data[_k]);
            norm[0] = or_pnorm(valid, &r, o->norm_type);
            FOR_ALL(&e, nx, ny, e.data[_k] = e.data[_k] + alpha[0] * pt.data[_k]);
        } else {
            FOR_ALL(&r, nx, ny, r.data[_k] = zero);
            norm[0] = zero;
        }
        if ((norm[0] > tol * initial_norm) && (norm[0] > reps * initial_rnorm)) {
            for (b2 = 0; b2 < ny; ++b2)
                for (a = 0; a < nx; ++a) AT(ST, a, b2) = AT(R, a, b2) * AT(D, a, b2);
            if ((rc = k_relax(o, valid, &st, &r, geo, bc, invd))) goto done;
            if ((rc = k_laplacian(o, valid, &t, &st, geo, bc, 1))) goto done;
            omega[0] = or_inner_prod(valid, &t, &r) / or_inner_prod(valid, &t, &t);
            FOR_ALL(&e, nx, ny, e.data[_k] = e.data[_k] + omega[0] * st.data[_k]);
            FOR_ALL(&r, nx, ny, r.data[_k] = r.data[_k] - omega[0] * t.data[_k]);
            norm[0] = or_pnorm(valid, &r, o->norm_type);
        }
        if (verbosity >= 3) printf("iter %d: rel |res| = %.16e\n", i, norm[0]);
        if ((norm[0] <= tol * initial_norm) || (norm[0] <= reps * initial_rnorm)) break;
        if ((omega[0] == zero) || (norm[0] > (one - hang) * norm[1])) {
            if (recount == 0) {
                recount = 1;
            } else {
                recount = 0;
                FOR_ALL(phi, nx, ny, phi->data[_k] = phi->data[_k] + e.data[_c + _r * e.ld]);
                /* P2:2438-2443 leaves the loop here; the add after the loop
                 * (P2:2466) then adds e a second time, as in the reference. */
                if (restarts == max_restarts) break;
                if ((rc = k_residual(o, valid, &r, rhs, phi, geo, bc, homog))) goto done;
                norm[0] = or_pnorm(valid, &r, o->norm_type);
                rho[1] = rho[2] = rho[3] = zero;
                alpha[0] = beta[0] = omega[0] = zero;
                FOR_ALL(&rt, nx, ny, rt.data[_k] = r.data[_k]);
                FOR_ALL(&e, nx, ny, e.data[_k] = zero);
                restarts = restarts + 1;
                init = 1;
            }
        }
    }
    if (verbosity >= 3) printf("%d iterations. final rel |res| = %.16e\n", i, norm[0]);
    FOR_ALL(phi, nx, ny, phi->data[_k] = phi->data[_k] + e.data[_c + _r * e.ld]);
    (void)PH; (void)E; (void)RT; (void)Tv; (void)Vv;
done:
    free(e.data); free(pt.data); free(st.data); free(r.data);
    free(rt.data); free(p.data); free(t.data); free(v.data);
    return rc;
}

int or_solve_bicgstab2(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                       const mgp_geo *geo, const mgp_bdry *bc, int homog,
                       const mgp_array *invd, double tol, int max_iters, int max_restarts,
                       int zerophi, int verbosity, int gs_order)
{
    KOps o = {0, 2, one - 1.0 / 3.0, gs_order};
    int rc;
    if ((rc = check_op(valid, bc))) return rc;
    return bicgstab_impl(&o, valid, phi, rhs, geo, bc, homog, invd, tol, max_iters, max_restarts,
                         zerophi, verbosity);
}

/* ---- restrict: MG:135-257 ----------------------------------------------- */
int or_restrict(const mgp_box *fb, const mgp_array *fine, const mgp_box *cb, mgp_array *crse,
                int offi, int offj)
{
    V F = view(fine), C = view(crse);
    int refx, refy, fi, fj, ci, cj;
    double scale;
    if (offi == 1 && offj == 1) {
        refx = fb->nx / cb->nx;
        refy = fb->ny / cb->ny;
        scale = one / (refx * refy);
        zero_all(crse, cb->nx, cb->ny);
        for (fj = 0; fj < fb->ny; ++fj) {
            cj = fj / refy;
            for (fi = 0; fi < fb->nx; ++fi) {
                ci = fi / refx;
                AT(C, ci, cj) = AT(C, ci, cj) + scale * AT(F, fi, fj);
            }
        }
    } else if (offi == 0 && offj == 1) {     /* x-faces: inject in x, average in y */
        refx = fb->nx / cb->nx;
        refy = fb->ny / cb->ny;
        scale = one / refy;
        zero_all(crse, cb->nx + 1, cb->ny);
        for (fj = 0; fj < fb->ny; ++fj) {
            cj = fj / refy;
            for (ci = 0; ci <= cb->nx; ++ci) {
                fi = ci * refx;
                AT(C, ci, cj) = AT(C, ci, cj) + scale * AT(F, fi, fj);
            }
        }
    } else if (offi == 1 && offj == 0) {     /* y-faces: average in x, inject in y */
        refx = fb->nx / cb->nx;
        refy = fb->ny / cb->ny;
        scale = one / refx;
        zero_all(crse, cb->nx, cb->ny + 1);
        for (cj = 0; cj <= cb->ny; ++cj) {
            fj = cj * refy;
            for (fi = 0; fi < fb->nx; ++fi) {
                ci = fi / refx;
                AT(C, ci, cj) = AT(C, ci, cj) + scale * AT(F, fi, fj);
            }
        }
    } else {
        refx = fb->nx / cb->nx;
        refy = fb->ny / cb->ny;
        for (cj = 0; cj <= cb->ny; ++cj)
            for (ci = 0; ci <= cb->nx; ++ci) AT(C, ci, cj) = AT(F, ci * refx, cj * refy);
    }
    return MGP_OK;
}

/* ---- prolong: MG:262-394 -------------------------------------------------
 * (2,2) follows the reference.  (2,1) and (1,2), where the reference stops
 * (MG:385-388), use the constant, linear and second-difference terms of the
 * (2,2) form in the coarsened direction only (an extension, no oracle in the
 * reference). */
int or_prolong(const mgp_box *fb, mgp_array *fine, const mgp_box *cb, mgp_array *crse,
               const mgp_geo *fine_geo, const mgp_geo *crse_geo, const mgp_bdry *crse_bc, int order)
{
    const int homog = 1, do_neum = 1;
    int refx, refy, fi, fj, ci, cj, rax, ray, remove_avg, rc;
    double dxprod, mx, my, mc;
    V Fv, Cv;
    rax = (crse_bc->type[MGP_XLO] == MGP_BCTYPE_PERIODIC && crse_bc->type[MGP_XHI] == MGP_BCTYPE_PERIODIC) ||
          (crse_bc->type[MGP_XLO] == MGP_BCTYPE_NEUM && crse_bc->type[MGP_XHI] == MGP_BCTYPE_NEUM);
    ray = (crse_bc->type[MGP_YLO] == MGP_BCTYPE_PERIODIC && crse_bc->type[MGP_YHI] == MGP_BCTYPE_PERIODIC) ||
          (crse_bc->type[MGP_YLO] == MGP_BCTYPE_NEUM && crse_bc->type[MGP_YHI] == MGP_BCTYPE_NEUM);
    remove_avg = rax && ray;
    dxprod = fine_geo->dx * fine_geo->dy;
    if (dxprod > crse_geo->dx * crse_geo->dy) return fail(MGP_EINVAL, "prolong: crse and fine geos passed in wrong order");
    refx = fb->nx / cb->nx;
    refy = fb->ny / cb->ny;
    if (!((refx == 2 || refx == 1) && (refy == 2 || refy == 1) && refx * refy > 1))
        return fail(MGP_ENOTSUP, "prolong: Needs updatin'");
    Fv = view(fine);
    Cv = view(crse);
    for (cj = 0; cj < cb->ny; ++cj) {
        fj = refy * cj;
        for (ci = 0; ci < cb->nx; ++ci) {
            double c = AT(Cv, ci, cj);
            fi = refx * ci;
            AT(Fv, fi, fj) = AT(Fv, fi, fj) + c;
            if (refx == 2) AT(Fv, fi + 1, fj) = AT(Fv, fi + 1, fj) + c;
            if (refy == 2) AT(Fv, fi, fj + 1) = AT(Fv, fi, fj + 1) + c;
            if (refx == 2 && refy == 2) AT(Fv, fi + 1, fj + 1) = AT(Fv, fi + 1, fj + 1) + c;
        }
    }
    if (order >= 1) {
        if ((rc = or_fill_ghosts(cb, crse, crse_bc, crse_geo, homog, do_neum))) return rc;
        Cv = view(crse);
        for (cj = 0; cj < cb->ny; ++cj) {
            fj = refy * cj;
            for (ci = 0; ci < cb->nx; ++ci) {
                fi = refx * ci;
                mx = half * (AT(Cv, ci + 1, cj) - AT(Cv, ci - 1, cj));
                my = half * (AT(Cv, ci, cj + 1) - AT(Cv, ci, cj - 1));
                if (refx == 2 && refy == 2) {
                    AT(Fv, fi, fj) = AT(Fv, fi, fj) + fourth * (-mx - my);
                    AT(Fv, fi + 1, fj) = AT(Fv, fi + 1, fj) + fourth * (mx - my);
                    AT(Fv, fi, fj + 1) = AT(Fv, fi, fj + 1) + fourth * (-mx + my);
                    AT(Fv, fi + 1, fj + 1) = AT(Fv, fi + 1, fj + 1) + fourth * (mx + my);
                } else if (refx == 2) {
                    AT(Fv, fi, fj) = AT(Fv, fi, fj) + fourth * (-mx);
                    AT(Fv, fi + 1, fj) = AT(Fv, fi + 1, fj) + fourth * (mx);
                } else {
                    AT(Fv, fi, fj) = AT(Fv, fi, fj) + fourth * (-my);
                    AT(Fv, fi, fj + 1) = AT(Fv, fi, fj + 1) + fourth * (my);
                }
            }
        }
    }
    if (order >= 2) {
        for (cj = 0; cj < cb->ny; ++cj) {
            fj = refy * cj;
            for (ci = 0; ci < cb->nx; ++ci) {
                double q;
                fi = refx * ci;
                mx = fourth * (AT(Cv, ci + 1, cj) - two * AT(Cv, ci, cj) + AT(Cv, ci - 1, cj));
                my = fourth * (AT(Cv, ci, cj + 1) - two * AT(Cv, ci, cj) + AT(Cv, ci, cj - 1));
                if (refx == 2 && refy == 2) {
                    q = eighth * (mx + my);
                    AT(Fv, fi, fj) = AT(Fv, fi, fj) + q;
                    AT(Fv, fi + 1, fj) = AT(Fv, fi + 1, fj) + q;
                    AT(Fv, fi, fj + 1) = AT(Fv, fi, fj + 1) + q;
                    AT(Fv, fi + 1, fj + 1) = AT(Fv, fi + 1, fj + 1) + q;
                } else if (refx == 2) {
                    q = eighth * mx;
                    AT(Fv, fi, fj) = AT(Fv, fi, fj) + q;
                    AT(Fv, fi + 1, fj) = AT(Fv, fi + 1, fj) + q;
                } else {
                    q = eighth * my;
                    AT(Fv, fi, fj) = AT(Fv, fi, fj) + q;
                    AT(Fv, fi, fj + 1) = AT(Fv, fi, fj + 1) + q;
                }
            }
        }
        if (refx == 2 && refy == 2) {
            if ((rc = or_extrapolate_ghosts(cb, crse, 3))) return rc;
            Cv = view(crse);
            for (cj = 0; cj < cb->ny; ++cj) {
                fj = refy * cj;
                for (ci = 0; ci < cb->nx; ++ci) {
                    fi = refx * ci;
                    mc = sixteenth * (AT(Cv, ci + 1, cj + 1) - AT(Cv, ci + 1, cj - 1) - AT(Cv, ci - 1, cj + 1) + AT(Cv, ci - 1, cj - 1));
                    AT(Fv, fi, fj) = AT(Fv, fi, fj) + fourth * mc;
                    AT(Fv, fi + 1, fj) = AT(Fv, fi + 1, fj) - fourth * mc;
                    AT(Fv, fi, fj + 1) = AT(Fv, fi, fj + 1) - fourth * mc;
                    AT(Fv, fi + 1, fj + 1) = AT(Fv, fi + 1, fj + 1) + fourth * mc;
                }
            }
        }
    }
    if (remove_avg) {   /* MG:371-383 */
        V Jv = view(&fine_geo->J);
        double sum = zero, vol = zero, avg;
        for (fj = 0; fj < fb->ny; ++fj)
            for (fi = 0; fi < fb->nx; ++fi) {
                double dvol = dxprod * AT(Jv, fi, fj);
                sum = sum + dvol * AT(Fv, fi, fj);
                vol = vol + dvol;
            }
        avg = sum / vol;
        FOR_ALL(fine, fb->nx, fb->ny, fine->data[_k] = fine->data[_k] - avg);
    }
    return MGP_OK;
}

/* ---- deferred-correction operators: DD:16-334 --------------------------- */
int or_dd_compute_invdiags(const mgp_box *valid, mgp_array *invd, const mgp_geo *geo)
{
    V D = view(invd);
    G g = gview(geo);
    double idx2 = one / (geo->dx * geo->dx), idy2 = one / (geo->dy * geo->dy);
    int i, j;
    for (j = 0; j < valid->ny; ++j)
        for (i = 0; i < valid->nx; ++i)
            AT(D, i, j) = (AT(g.xx, i + 1, j) + AT(g.xx, i, j)) * idx2 + (AT(g.yy, i, j + 1) + AT(g.yy, i, j)) * idy2;
    for (j = 0; j < valid->ny; ++j)
        for (i = 0; i < valid->nx; ++i) AT(D, i, j) = -one / AT(D, i, j);
    return MGP_OK;
}

int or_dd_compute_laplacian(const mgp_box *valid, mgp_array *lap, mgp_array *phi,
                            const mgp_geo *geo, const mgp_bdry *bc, int homog)
{
    const int nx = valid->nx, ny = valid->ny;
    V L = view(lap), P;
    G g = gview(geo);
    double idx = one / geo->dx, idy = one / geo->dy, xyscale = fourth * idx * idy;
    int i, j, rc;
    if ((rc = or_extrapolate_ghosts(valid, phi, 0))) return rc;
    P = view(phi);
    for (j = 0; j < ny; ++j)
        for (i = 0; i < nx; ++i) {
            double pe = AT(P, i + 1, j), pw = AT(P, i - 1, j), pn = AT(P, i, j + 1), ps = AT(P, i, j - 1);
            double pne = AT(P, i + 1, j + 1), pnw = AT(P, i - 1, j + 1), psw = AT(P, i - 1, j - 1), pse = AT(P, i + 1, j - 1);
            double gxye = AT(g.xy, i + 1, j) * (pne - pse + pn - ps);
            double gxyw = AT(g.xy, i, j) * (pn - ps + pnw - psw);
            double gyxn = AT(g.yx, i, j + 1) * (pne - pnw + pe - pw);
            double gyxs = AT(g.yx, i, j) * (pe - pw + pse - psw);
            AT(L, i, j) = (gxye - gxyw + gyxn - gyxs) * xyscale;
        }
    if ((rc = or_fill_ghosts(valid, phi, bc, geo, homog, 1))) return rc;
    for (j = 0; j < ny; ++j)
        for (i = 0; i < nx; ++i) {
            double p = AT(P, i, j), pe = AT(P, i + 1, j), pw = AT(P, i - 1, j), pn = AT(P, i, j + 1), ps = AT(P, i, j - 1);
            double xfe = AT(g.xx, i + 1, j) * (pe - p) * idx;
            double xfw = AT(g.xx, i, j) * (p - pw) * idx;
            double yfn = AT(g.yy, i, j + 1) * (pn - p) * idy;
            double yfs = AT(g.yy, i, j) * (p - ps) * idy;
            AT(L, i, j) = AT(L, i, j) + (xfe - xfw) * idx + (yfn - yfs) * idy;
        }
    return MGP_OK;
}

int or_dd_compute_residual(const mgp_box *valid, mgp_array *res, const mgp_array *rhs,
                           mgp_array *phi, const mgp_geo *geo, const mgp_bdry *bc, int homog)
{
    int rc, i, j;
    V R, F;
    if ((rc = or_dd_compute_laplacian(valid, res, phi, geo, bc, homog))) return rc;
    R = view(res);
    F = view(rhs);
    for (j = 0; j < valid->ny; ++j)
        for (i = 0; i < valid->nx; ++i) AT(R, i, j) = AT(F, i, j) - AT(R, i, j);
    return MGP_OK;
}

static inline void dd_gs_cell(V P, V M, V D, const G *g, int i, int j, double idx, double idy, double omega)
{
    double p = AT(P, i, j), pe = AT(P, i + 1, j), pw = AT(P, i - 1, j), pn = AT(P, i, j + 1), ps = AT(P, i, j - 1);
    double xfe = AT(g->xx, i + 1, j) * (pe - p) * idx;
    double xfw = AT(g->xx, i, j) * (p - pw) * idx;
    double yfn = AT(g->yy, i, j + 1) * (pn - p) * idy;
    double yfs = AT(g->yy, i, j) * (p - ps) * idy;
    double lphi = (xfe - xfw) * idx + (yfn - yfs) * idy;
    double newphi = AT(P, i, j) + (AT(M, i, j) - lphi) * AT(D, i, j);
    AT(P, i, j) = omega * newphi + (one - omega) * AT(P, i, j);
}

int or_dd_relax_gs(const mgp_box *valid, mgp_array *phi, const mgp_array *rhs,
                   const mgp_geo *geo, const mgp_bdry *bc, int homog, const mgp_array *invd,
                   double omega, double tol, int maxiters, int zerophi, int verbosity, int gs_order)
{
    const int nx = valid->nx, ny = valid->ny;
    G g = gview(geo);
    double idx = one / geo->dx, idy = one / geo->dy, xyscale = half * idx * idy, rscale = one, relres;
    mgp_array r = {0}, modrhs;
    V P, M, D = view(invd), F = view(rhs);
    int i, j, iter, color, rc = MGP_OK;
    if (maxiters == 0) return MGP_OK;
    if (zerophi) zero_all(phi, nx, ny);
    if (tol > zero) {
        r = alloc_like(nx, ny, 0, 0);
        if ((rc = or_dd_compute_residual(valid, &r, rhs, phi, geo, bc, homog))) { free(r.data); return rc; }
        rscale = or_pnorm(valid, &r, 2);
        if (rscale == zero) rscale = one;
    }
    /* modrhs = rhs - lagged corner cross terms (DD:226-250) */
    modrhs = alloc_like(nx, ny, 0, 0);
    M = view(&modrhs);
    for (j = 0; j < ny; ++j)
        for (i = 0; i < nx; ++i) AT(M, i, j) = AT(F, i, j);
    if ((rc = or_extrapolate_ghosts(valid, phi, 0))) goto out;
    P = view(phi);
    for (j = 0; j < ny; ++j)
        for (i = 0; i < nx; ++i) {
            double pne = AT(P, i + 1, j + 1), pnw = AT(P, i - 1, j + 1), psw = AT(P, i - 1, j - 1), pse = AT(P, i + 1, j - 1);
            double gxye = AT(g.xy, i + 1, j) * (pne - pse);
            double gxyw = AT(g.xy, i, j) * (pnw - psw);
            double gyxn = AT(g.yx, i, j + 1) * (pne - pnw);
            double gyxs = AT(g.yx, i, j) * (pse - psw);
            AT(M, i, j) = AT(M, i, j) - (gxye - gxyw + gyxn - gyxs) * xyscale;
        }
    for (iter = 1; iter <= maxiters; ++iter) {
        if ((rc = or_fill_ghosts(valid, phi, bc, geo, homog, 1))) goto out;   /* DD:259 */
        if (gs_order == 0) {
            for (j = 0; j < ny; ++j)
                for (i = 0; i < nx; ++i) dd_gs_cell(P, M, D, &g, i, j, idx, idy, omega);
        } else {
            for (color = 0; color <= 1; ++color)   /* DD:262-285, parity relative to (ilo, jlo) */
                for (j = 0; j < ny; ++j)
                    for (i = (color + j) % 2; i < nx; i += 2) dd_gs_cell(P, M, D, &g, i, j, idx, idy, omega);
        }
        if (tol > zero) {
            if ((rc = or_dd_compute_residual(valid, &r, rhs, phi, geo, bc, homog))) goto out;
            relres = or_pnorm(valid, &r, 2) / rscale;
            if (verbosity >= 3) printf("iter %d: rel |res| = %.16e\n", iter, relres);
            if (relres <= tol) break;
        }
    }
out:
    free(modrhs.data);
    free(r.data);
    return rc;
}

/* ---- the multigrid drivers: MG:400-1189, DD:589-1045 -------------------- */

typedef struct {
    mgp_box valid;
    mgp_array e, r, w, invd;
    mgp_array J, xx, xy, yx, yy;
    mgp_geo geo;
    mgp_bdry bc;
    double bczero[4];
} Lvl;

typedef struct {
    int maxdepth;
    int *refx, *refy;
    Lvl *lv;
    int dd;          /* deferred-correction operators and LAH BCs */
    int gs_order;
} Hier;

static void hier_free(Hier *h)
{
    int d;
    if (h->lv) {
        for (d = 0; d <= h->maxdepth; ++d) {
            Lvl *L = &h->lv[d];
            free(L->e.data); free(L->r.data); free(L->w.data); free(L->invd.data);
            free(L->J.data); free(L->xx.data); free(L->xy.data); free(L->yx.data); free(L->yy.data);
        }
    }
    free(h->lv);
    free(h->refx);
    free(h->refy);
    memset(h, 0, sizeof *h);
}

static void copy_valid(const mgp_array *src, mgp_array *dst, int nx, int ny)
{
    V S = view(src), D = view(dst);
    int i, j;
    for (j = 0; j < ny; ++j)
        for (i = 0; i < nx; ++i) AT(D, i, j) = AT(S, i, j);
}

/* MG:432-562 (dd = 0) and DD:622-761 (dd = 1). */
static int hier_build(Hier *h, const mgp_box *valid, const mgp_geo *geo, const mgp_bdry *bc,
                      int maxdepth_user, int dd, int gs_order)
{
    int d, s, rc;
    mgp_box v = *valid;
    memset(h, 0, sizeof *h);
    h->dd = dd;
    h->gs_order = gs_order;
    h->maxdepth = maxdepth_user < 0 ? 1000 : maxdepth_user;
    or_estimate_maxdepth(&h->maxdepth, valid);
    h->refx = (int *)calloc((size_t)h->maxdepth + 1, sizeof(int));
    h->refy = (int *)calloc((size_t)h->maxdepth + 1, sizeof(int));
    if (!h->refx || !h->refy) return fail(MGP_ENOMEM, "vcycle: Out of memory");
    or_create_mgschedule(h->refx, h->refy, &h->maxdepth, valid);
    h->lv = (Lvl *)calloc((size_t)h->maxdepth + 1, sizeof(Lvl));
    if (!h->lv) return fail(MGP_ENOMEM, "vcycle: Out of memory");
    for (d = 0; d <= h->maxdepth; ++d) {
        Lvl *L = &h->lv[d];
        L->valid = v;
        for (s = 0; s < 4; ++s) {
            L->bc.type[s] = bc->type[s];
            L->bc.mode[s] = dd ? MGP_BCMODE_LAH : MGP_BCMODE_UNIFORM;
            L->bczero[s] = zero;
            L->bc.data[s] = &L->bczero[s];
        }
        L->e = alloc_like(v.nx, v.ny, 1, 1);
        L->r = alloc_like(v.nx, v.ny, 0, 0);
        L->w = alloc_like(v.nx, v.ny, 0, 0);
        L->invd = alloc_like(v.nx, v.ny, 0, 0);
        L->J = alloc_like(v.nx, v.ny, 0, 0);
        L->xx = alloc_like(v.nx + 1, v.ny, 0, 0);
        L->xy = alloc_like(v.nx + 1, v.ny, 0, 0);
        L->yx = alloc_like(v.nx, v.ny + 1, 0, 0);
        L->yy = alloc_like(v.nx, v.ny + 1, 0, 0);
        if (!L->e.data || !L->r.data || !L->w.data || !L->invd.data || !L->J.data || !L->xx.data ||
            !L->xy.data || !L->yx.data || !L->yy.data)
            return fail(MGP_ENOMEM, "Out of memory");
        L->geo.J = L->J; L->geo.Jgup_xx = L->xx; L->geo.Jgup_xy = L->xy;
        L->geo.Jgup_yx = L->yx; L->geo.Jgup_yy = L->yy;
        L->geo.dx = v.dx;
        L->geo.dy = v.dy;
        if (d == 0) {
            copy_valid(&geo->J, &L->J, v.nx, v.ny);
            copy_valid(&geo->Jgup_xx, &L->xx, v.nx + 1, v.ny);
            copy_valid(&geo->Jgup_xy, &L->xy, v.nx + 1, v.ny);
            copy_valid(&geo->Jgup_yx, &L->yx, v.nx, v.ny + 1);
            copy_valid(&geo->Jgup_yy, &L->yy, v.nx, v.ny + 1);
        } else {
            Lvl *U = &h->lv[d - 1];
            or_restrict(&U->valid, &U->J, &v, &L->J, 1, 1);
            or_restrict(&U->valid, &U->xx, &v, &L->xx, 0, 1);
            or_restrict(&U->valid, &U->xy, &v, &L->xy, 0, 1);
            or_restrict(&U->valid, &U->yx, &v, &L->yx, 1, 0);
            or_restrict(&U->valid, &U->yy, &v, &L->yy, 1, 0);
        }
        if (dd)
            rc = or_dd_compute_invdiags(&v, &L->invd, &L->geo);
        else
            rc = or_compute_invdiags(&v, &L->invd, &L->geo, &L->bc, 1);
        if (rc) return rc;
        if (d < h->maxdepth) {
            /* coarsen_box, AU:154-170 (relative indices: ilo, jlo even) */
            v.ilo /= h->refx[d]; v.ihi /= h->refx[d]; v.nx = v.ihi - v.ilo + 1; v.dx = v.dx * h->refx[d];
            v.jlo /= h->refy[d]; v.jhi /= h->refy[d]; v.ny = v.jhi - v.jlo + 1; v.dy = v.dy * h->refy[d];
        }
    }
    return MGP_OK;
}

static void set_guess(Lvl *L)   /* e = r * invdiag on the valid region (MG:600, MG:805) */
{
    V E = view(&L->e), R = view(&L->r), D = view(&L->invd);
    int i, j;
    for (j = 0; j < L->valid.ny; ++j)
        for (i = 0; i < L->valid.nx; ++i) AT(E, i, j) = AT(R, i, j) * AT(D, i, j);
}

/* vcycle_noinit, MG:675-854 (dd = 0) and DD:867-1045 (dd = 1). */
static int vcycle_noinit(Hier *h, int depth, int numcycles, int nd, int nu, int nb)
{
    Lvl *L = &h->lv[depth];
    int rc, c;
    const double relax_omega = h->dd ? 4.0 / 5.0 : one;
    const double bottom_tol = 1.0e-6;
    const int bottom_maxiters = 80, bottom_maxrestarts = 5;
#define RELAX(nu_)                                                                                      \
    (h->dd ? or_dd_relax_gs(&L->valid, &L->e, &L->r, &L->geo, &L->bc, 1, &L->invd, relax_omega, -one, \
                            (nu_), 0, 0, h->gs_order)                                                  \
           : or_relax_gs(&L->valid, &L->e, &L->r, &L->geo, &L->bc, 1, &L->invd, relax_omega, -one,    \
                         (nu_), 0, 0, h->gs_order))
    if (depth == h->maxdepth) {
        KOps o;
        if (h->dd) set_guess(L);   /* DD:931 */
        if ((rc = RELAX(nb))) return rc;
        o.dd = h->dd;
        o.norm_type = h->dd ? 0 : 2;
        o.omega = h->dd ? 4.0 / 5.0 : one - 1.0 / 3.0;
        o.gs_order = h->gs_order;
        return bicgstab_impl(&o, &L->valid, &L->e, &L->r, &L->geo, &L->bc, 1, &L->invd, bottom_tol,
                             bottom_maxiters, bottom_maxrestarts, 0, 0);
    }
    if (h->dd) set_guess(L);   /* DD:971 */
    if ((rc = RELAX(nd))) return rc;
    rc = h->dd ? or_dd_compute_residual(&L->valid, &L->w, &L->r, &L->e, &L->geo, &L->bc, 1)
               : or_compute_residual(&L->valid, &L->w, &L->r, &L->e, &L->geo, &L->bc, 1, 0);
    if (rc) return rc;
    or_restrict(&L->valid, &L->w, &h->lv[depth + 1].valid, &h->lv[depth + 1].r, 1, 1);
    if (!h->dd) set_guess(&h->lv[depth + 1]);   /* MG:805-806 */
    for (c = 1; c <= numcycles; ++c)
        if ((rc = vcycle_noinit(h, depth + 1, numcycles, nd, nu, nb))) return rc;
    {
        Lvl *C = &h->lv[depth + 1];
        if ((rc = or_prolong(&L->valid, &L->e, &C->valid, &C->e, &L->geo, &C->geo, &C->bc, 1))) return rc;
    }
    if ((rc = RELAX(nu))) return rc;
#undef RELAX
    return MGP_OK;
}

/* fmg_noinit, MG:1127-1189. */
static int fmg_noinit(Hier *h, int depth, int numcycles, int nd, int nu, int nb)
{
    Lvl *L = &h->lv[depth];
    int rc, c;
    zero_all(&L->e, L->valid.nx, L->valid.ny);
    if (depth < h->maxdepth) {
        Lvl *C = &h->lv[depth + 1];
        or_restrict(&L->valid, &L->r, &C->valid, &C->r, 1, 1);
        if ((rc = fmg_noinit(h, depth + 1, numcycles, nd, nu, nb))) return rc;
        if ((rc = or_prolong(&L->valid, &L->e, &C->valid, &C->e, &L->geo, &C->geo, &C->bc, 2))) return rc;
    }
    for (c = 1; c <= numcycles; ++c)
        if ((rc = vcycle_noinit(h, depth, numcycles, nd, nu, nb))) return rc;
    return MGP_OK;
}

static int check_solver_box(const mgp_box *valid)
{
    if (valid->ilo < 0 || valid->jlo < 0 || (valid->ilo % 2) || (valid->jlo % 2))
        return fail(MGP_EINVAL, "solver: ilo and jlo must be even and non-negative");
    if (valid->nx != valid->ihi - valid->ilo + 1 || valid->ny != valid->jhi - valid->jlo + 1)
        return fail(MGP_EINVAL, "solver: box extents are inconsistent");
    return MGP_OK;
}

/* kind 0 = vcycle (MG:400-670), 1 = fmg (MG:860-1122), 2 = DD vcycle (DD:589-862). */
static int driver(int kind, const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
                  const mgp_bdry *bc, int homog, double tol, int maxiters, int maxdepth_user, int numcycles,
                  int nd, int nu, int nb, int zerophi, int verbosity, int gs_order, mgp_report *rep)
{
    Hier h;
    int rc, iter, i, j, dd = (kind == 2), done_iters = 0, diverged = 0;
    double rscale = 0.0, *relres = NULL, rel_prev;
    const int nx = valid->nx, ny = valid->ny;
    V F, J, E0;
    Lvl *L0;
    if ((rc = check_solver_box(valid))) return rc;
    if ((rc = hier_build(&h, valid, geo, bc, maxdepth_user, dd, gs_order))) { hier_free(&h); return rc; }
    relres = (double *)calloc((size_t)maxiters + 1, sizeof(double));
    if (!relres) { hier_free(&h); return fail(MGP_ENOMEM, "Out of memory"); }
    if (verbosity >= 1) printf("max MG depth = %d\n", h.maxdepth);
    if (zerophi) zero_all(phi, nx, ny);
    F = view(rhs);
    J = view(&geo->J);
    if (dd)   /* DD:772-773 */
        for (j = 0; j < ny; ++j)
            for (i = 0; i < nx; ++i) AT(F, i, j) = AT(F, i, j) * AT(J, i, j);
    L0 = &h.lv[0];
    E0 = view(&L0->e);
    (void)E0;
    if ((rc = or_compute_residual(valid, &L0->r, rhs, phi, geo, bc, homog, 0))) goto out;
    rscale = or_pnorm(valid, &L0->r, 2);
    if (rscale == zero) { relres[0] = rscale; rscale = one; }
    else relres[0] = one;
    rel_prev = relres[0];
    if (verbosity >= 1) printf("V-Cycle iter 0: rel |res| = %.16e\n", relres[0]);
    for (iter = 1; iter <= maxiters; ++iter) {
        if (kind == 0) set_guess(L0);   /* MG:600 */
        if (kind == 1) rc = fmg_noinit(&h, 0, numcycles, nd, nu, nb);
        else rc = vcycle_noinit(&h, 0, numcycles, nd, nu, nb);
        if (rc) goto out;
        FOR_ALL(phi, nx, ny, phi->data[_k] = phi->data[_k] + L0->e.data[_c + _r * L0->e.ld]);
        if ((rc = or_compute_residual(valid, &L0->r, rhs, phi, &L0->geo, bc, homog, 0))) goto out;
        relres[iter] = or_pnorm(valid, &L0->r, 2) / rscale;
        done_iters = iter;
        if (verbosity >= 1) printf("V-Cycle iter %d: rel |res| = %.16e\n", iter, relres[iter]);
        if (relres[iter] <= tol) break;
        if (relres[iter] > relres[iter - 1]) {   /* MG:630-639 */
            FOR_ALL(phi, nx, ny, phi->data[_k] = phi->data[_k] - L0->e.data[_c + _r * L0->e.ld]);
            diverged = 1;
            break;
        }
        rel_prev = relres[iter];
    }
    (void)rel_prev;
    if (dd)   /* DD:837-838 */
        for (j = 0; j < ny; ++j)
            for (i = 0; i < nx; ++i) AT(F, i, j) = AT(F, i, j) / AT(J, i, j);
out:
    if (rep) {
        rep->status = rc;
        rep->iterations = done_iters;
        rep->maxdepth = h.maxdepth;
        rep->diverged = diverged;
        rep->rscale = rscale;
        rep->final_relres = relres[done_iters];
        if (rep->relres)
            for (i = 0; i <= done_iters; ++i) rep->relres[i] = relres[i];
    }
    free(relres);
    hier_free(&h);
    return rc;
}

int or_vcycle(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
              const mgp_bdry *bc, int homog, double tol, int maxiters, int maxdepth_user,
              int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
              int verbosity, int gs_order, mgp_report *report)
{
    return driver(0, valid, phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles,
                  smooth_down, smooth_up, smooth_bottom, zerophi, verbosity, gs_order, report);
}

int or_fmg(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
           const mgp_bdry *bc, int homog, double tol, int maxiters, int maxdepth_user,
           int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
           int verbosity, int gs_order, mgp_report *report)
{
    return driver(1, valid, phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles,
                  smooth_down, smooth_up, smooth_bottom, zerophi, verbosity, gs_order, report);
}

int or_dc_vcycle(const mgp_box *valid, mgp_array *phi, mgp_array *rhs, const mgp_geo *geo,
                 const mgp_bdry *bc, int homog, double tol, int maxiters, int maxdepth_user,
                 int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
                 int verbosity, int gs_order, mgp_report *report)
{
    return driver(2, valid, phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles,
                  smooth_down, smooth_up, smooth_bottom, zerophi, verbosity, gs_order, report);
}
