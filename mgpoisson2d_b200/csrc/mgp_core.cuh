// mgp_core.cuh -- device-side building blocks of the B200 multigrid solver.
//
// Compiled with -fmad=false, so each product and sum is rounded on its own
// in the order the Fortran routines write them: a cell computed here in FP64
// is bit-identical to the same cell computed by the Fortran code (and by the
// CPU oracle).  The templates are also instantiated for FP32 fields, the grid
// levels of the mixed-precision V-cycle.
//
// Citations: AU = arrayutils.f90, P2 = poisson2d.f90, MG = MGPoisson2D.f90,
// DD = MGPoisson2D_DD.f90 (EdSantilli/MGPoisson2D, src/).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mgp {

constexpr double kBogus = 1.2345e300;   // precision.f90:53
enum { RLO = 0, RMID = 1, RHI = 2 };
enum { T_NONE = -1, T_NEUM = 0, T_DIRI = 1, T_PERIODIC = 2, T_CF = 3, T_EX0 = 4, T_EX1 = 5, T_EX2 = 6 };
enum { M_UNIFORM = 0, M_NONUNIFORM = 1, M_LAH = 2 };
enum { S_XLO = 0, S_XHI = 1, S_YLO = 2, S_YHI = 3 };

// A 2-D field; p points at valid element (0,0), ld is the row pitch.  The
// solver's own arithmetic is FP64 (DF); the mixed-precision V-cycle keeps
// its grid levels in FP32 (DF32).
template <class T>
struct DFT {
    T* p;
    int ld;
};
using DF = DFT<double>;
using DF32 = DFT<float>;
#define AT(f, i, j) ((f).p[(long)(i) + (long)(j) * (long)(f).ld])

template <class T>
struct GeoT {
    DFT<T> J, xx, xy, yx, yy;   // J cell-centred; xx, xy on x-faces; yx, yy on y-faces
    double dx, dy, idx, idy;
};
using Geo = GeoT<double>;
using Geo32 = GeoT<float>;

// The value fill_ghosts puts in non-periodic corner ghosts (precision.f90:53);
// FP32 fields hold a large finite stand-in.
template <class T>
__device__ __forceinline__ T bogus();
template <>
__device__ __forceinline__ double bogus<double>() { return kBogus; }
template <>
__device__ __forceinline__ float bogus<float>() { return 1.2345e30f; }

// Boundary conditions of one level (type(bdry_data), AU:55-70).
struct BCd {
    int type[4];
    int mode[4];
    const double* d[4];   // NONUNIFORM values in device memory, else nullptr
    double u[4];          // UNIFORM values
    int kyhi;             // index of the north-face Neumann value the operator reads (P2: data_yhi(j), j = jhi)
    int koffy;            // offset of y-side NONUNIFORM Dirichlet values (AU:1224: bcd(jlo:jhi))
};

// One multigrid level as the kernels see it.
struct Lv {
    int nx, ny;
    Geo g;
    BCd bc;
    DF e;      // correction, 1 ghost layer
    DF e2;     // second buffer of e for the two-buffer sweep (grid-path levels)
    DF r;      // right-hand side of the residual equation
    DF w;      // work (residual before restriction)
    DF invd;   // inverse diagonal
    DF ea;     // extra arrays for the bottom solver (1 ghost): e_loc, p_tilde, s_tilde
    DF pt, st;
    DF rr, rt, pp, tt, vv;   // bottom solver, no ghosts
};

// Asynchronous 8-byte global -> shared copy (cp.async, sm_80+): the thread does
// not wait for the load, so a loop of them keeps many loads in flight.
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// The same by shared-space address, without a memory clobber: the copies of
// a staging loop are ordered against later reads by cp_async_wait_all.
__device__ __forceinline__ void cp_async8s(unsigned sdst, const double* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sdst), "l"(gsrc));
}
__device__ __forceinline__ void cp_async16s(unsigned sdst, const double* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sdst), "l"(gsrc));
}

__device__ __forceinline__ int region(int i, int n, bool per_lo, bool per_hi) {
    if (i == 0 && !per_lo) return RLO;
    if (i == n - 1 && !per_hi) return RHI;
    return RMID;
}

// ---------------------------------------------------------------------------
// The mapped 9-point operator, P2:886-1319
// ---------------------------------------------------------------------------
template <class T>
struct St9T {
    T p, pe, pw, pn, ps, ee, ew, en, es, ene, enw, ese, esw;
};
using St9 = St9T<double>;

// Reads phi around the cell from global memory.
template <class T>
struct GLoadT {
    const T* c;
    long ld;
    __device__ __forceinline__ T operator()(int di, int dj) const { return c[di + (long)dj * ld]; }
};
using GLoad = GLoadT<double>;

// A unit impulse at the cell, zero elsewhere; the four own-row/column ghosts
// may carry the Dirichlet coupling (-3) for the coupled diagonal.
struct DeltaLoad {
    double gw, ge, gs, gn;
    __device__ __forceinline__ double operator()(int di, int dj) const {
        if (di == 0 && dj == 0) return 1.0;
        if (dj == 0 && di == -1) return gw;
        if (dj == 0 && di == 1) return ge;
        if (di == 0 && dj == -1) return gs;
        if (di == 0 && dj == 1) return gn;
        return 0.0;
    }
};

// The transverse values of the nine region blocks of compute_laplacian.
template <class L, class T>
__device__ __forceinline__ void gather9(const L& P, int xr, int yr, St9T<T>& s) {
    const T p = P(0, 0), pe = P(1, 0), pw = P(-1, 0), pn = P(0, 1), ps = P(0, -1);
    const T three = T(3.0), half = T(0.5);
    T ee, ew, en, es, ene, enw, ese, esw;
    s.p = p; s.pe = pe; s.pw = pw; s.pn = pn; s.ps = ps;
    if (yr == RLO) {
        if (xr == RLO) {              // P2:937-958
            ee = P(1, 0); en = P(0, 1);
            ew = three * (p - ee) + P(2, 0);
            es = three * (p - en) + P(0, 2);
            ene = P(1, 1);
            enw = three * (en - ene) + P(2, 1);
            ese = three * (ee - ene) + P(1, 2);
            esw = half * ((three * (es - ese) + P(2, -1)) + (three * (ew - enw) + P(-1, 2)));
        } else if (xr == RMID) {      // P2:986-1002
            ee = P(1, 0); ew = P(-1, 0); en = P(0, 1);
            es = three * (p - en) + P(0, 2);
            ene = P(1, 1); enw = P(-1, 1);
            ese = three * (ee - ene) + P(1, 2);
            esw = three * (ew - enw) + P(-1, 2);
        } else {                      // P2:1021-1039
            ew = P(-1, 0); en = P(0, 1);
            ee = three * (p - ew) + P(-2, 0);
            es = three * (p - en) + P(0, 2);
            enw = P(-1, 1);
            ene = three * (pn - enw) + P(-2, 1);
            esw = three * (pw - enw) + P(-1, 2);
            ese = half * ((three * (es - esw) + P(-2, -1)) + (three * (ee - ene) + P(1, 2)));
        }
    } else if (yr == RMID) {
        if (xr == RLO) {              // P2:1068-1085
            ee = P(1, 0); en = P(0, 1); es = P(0, -1);
            ew = three * (p - ee) + P(2, 0);
            ene = P(1, 1); ese = P(1, -1);
            enw = three * (en - ene) + P(2, 1);
            esw = three * (es - ese) + P(2, -1);
        } else if (xr == RMID) {      // P2:1103-1125
            ee = P(1, 0); ew = P(-1, 0); en = P(0, 1); es = P(0, -1);
            ene = P(1, 1); enw = P(-1, 1); ese = P(1, -1); esw = P(-1, -1);
        } else {                      // P2:1128-1147
            ew = P(-1, 0); en = P(0, 1); es = P(0, -1);
            ee = three * (p - ew) + P(-2, 0);
            enw = P(-1, 1); esw = P(-1, -1);
            ene = three * (en - enw) + P(-2, 1);
            ese = three * (es - esw) + P(-2, -1);
        }
    } else {
        if (xr == RLO) {              // P2:1176-1194
            ee = P(1, 0); es = P(0, -1);
            ew = three * (p - ee) + P(2, 0);
            en = three * (p - es) + P(0, -2);
            ese = P(1, -1);
            ene = three * (ee - ese) + P(1, -2);
            esw = three * (es - ese) + P(2, -1);
            enw = half * ((three * (ew - esw) + P(-1, -2)) + (three * (en - ene) + P(2, 1)));
        } else if (xr == RMID) {      // P2:1223-1239
            ee = P(1, 0); ew = P(-1, 0); es = P(0, -1);
            en = three * (p - es) + P(0, -2);
            ese = P(1, -1); esw = P(-1, -1);
            ene = three * (ee - ese) + P(1, -2);
            enw = three * (ew - esw) + P(-1, -2);
        } else {                      // P2:1258-1276
            ew = P(-1, 0); es = P(0, -1);
            ee = three * (p - ew) + P(-2, 0);
            en = three * (p - es) + P(0, -2);
            esw = P(-1, -1);
            enw = three * (ew - esw) + P(-1, -2);
            ese = three * (es - esw) + P(-2, -1);
            ene = half * ((three * (en - enw) + P(-2, 1)) + (three * (ee - ese) + P(1, -2)));
        }
    }
    s.ee = ee; s.ew = ew; s.en = en; s.es = es;
    s.ene = ene; s.enw = enw; s.ese = ese; s.esw = esw;
}

__device__ __forceinline__ double nbval(const BCd& b, int homog, int s, int k) {
    if (homog) return 0.0;
    if (b.mode[s] == M_UNIFORM) return b.u[s];
    return b.d[s][k];
}

// The metric values the operator reads at one cell: its four faces.
template <class T>
struct FacesT {
    T xxe, xxw, xye, xyw;   // Jgup_xx, Jgup_xy at x-faces i+1 (east) and i (west)
    T yyn, yys, yxn, yxs;   // Jgup_yy, Jgup_yx at y-faces j+1 (north) and j (south)
};
using Faces = FacesT<double>;

template <class T>
__device__ __forceinline__ FacesT<T> faces_of(const GeoT<T>& g, int i, int j) {
    FacesT<T> f;
    f.xxe = AT(g.xx, i + 1, j); f.xxw = AT(g.xx, i, j);
    f.xye = AT(g.xy, i + 1, j); f.xyw = AT(g.xy, i, j);
    f.yyn = AT(g.yy, i, j + 1); f.yys = AT(g.yy, i, j);
    f.yxn = AT(g.yx, i, j + 1); f.yxs = AT(g.yx, i, j);
    return f;
}

// (xfe - xfw)/dx + (yfn - yfs)/dy with Neumann faces replaced by the BC flux.
template <class T>
__device__ __forceinline__ T lap9f(const St9T<T>& s, const FacesT<T>& f, T idx, T idy, int i, int j, int xr, int yr,
                                   const BCd& b, int homog) {
    const T q = T(0.25);
    T xfe = f.xxe * (s.pe - s.p) * idx + f.xye * q * (s.ene - s.ese + s.en - s.es) * idy;
    T xfw = f.xxw * (s.p - s.pw) * idx + f.xyw * q * (s.en - s.es + s.enw - s.esw) * idy;
    T yfn = f.yyn * (s.pn - s.p) * idy + f.yxn * q * (s.ene - s.enw + s.ee - s.ew) * idx;
    T yfs = f.yys * (s.p - s.ps) * idy + f.yxs * q * (s.ee - s.ew + s.ese - s.esw) * idx;
    if (xr == RLO && b.type[S_XLO] == T_NEUM) xfw = T(nbval(b, homog, S_XLO, j));
    if (yr == RLO && b.type[S_YLO] == T_NEUM) yfs = T(nbval(b, homog, S_YLO, i));
    if (xr == RHI && b.type[S_XHI] == T_NEUM) xfe = T(nbval(b, homog, S_XHI, j));
    if (yr == RHI && b.type[S_YHI] == T_NEUM) yfn = T(nbval(b, homog, S_YHI, b.kyhi));
    return (xfe - xfw) * idx + (yfn - yfs) * idy;
}

template <class T>
__device__ __forceinline__ T lap9(const St9T<T>& s, const GeoT<T>& g, int i, int j, int xr, int yr, const BCd& b,
                                  int homog) {
    return lap9f(s, faces_of(g, i, j), T(g.idx), T(g.idy), i, j, xr, yr, b, homog);
}

struct Per {
    bool xl, xh, yl, yh;
};
__device__ __forceinline__ Per periodic_of(const BCd& b) {
    Per p;
    p.xl = b.type[S_XLO] == T_PERIODIC; p.xh = b.type[S_XHI] == T_PERIODIC;
    p.yl = b.type[S_YLO] == T_PERIODIC; p.yh = b.type[S_YHI] == T_PERIODIC;
    return p;
}

// L[phi] at (i,j) in regions (xr, yr); phi's ghosts must be set.
template <class T>
__device__ __forceinline__ T apply9r(const DFT<T>& phi, const GeoT<T>& g, const BCd& b, int homog, int i, int j,
                                     int xr, int yr) {
    St9T<T> s;
    gather9(GLoadT<T>{&AT(phi, i, j), phi.ld}, xr, yr, s);
    return lap9(s, g, i, j, xr, yr, b, homog);
}

// L[phi] at (i,j); phi's ghosts must be set.
template <class T>
__device__ __forceinline__ T apply9(const DFT<T>& phi, const GeoT<T>& g, const BCd& b, int homog, int nx, int ny,
                                    int i, int j) {
    const Per pr = periodic_of(b);
    return apply9r(phi, g, b, homog, i, j, region(i, nx, pr.xl, pr.xh), region(j, ny, pr.yl, pr.yh));
}

// Diagonal of the operator at (i,j) (compute_invdiags, P2:16-388), before inversion.
__device__ __forceinline__ double diag9(const Geo& g, const BCd& b, int homog, int nx, int ny, int i, int j,
                                        bool diri_coupled) {
    const Per pr = periodic_of(b);
    const int xr = region(i, nx, pr.xl, pr.xh), yr = region(j, ny, pr.yl, pr.yh);
    DeltaLoad D{0.0, 0.0, 0.0, 0.0};
    if (diri_coupled) {
        if (xr == RLO && b.type[S_XLO] == T_DIRI) D.gw = -3.0;
        if (xr == RHI && b.type[S_XHI] == T_DIRI) D.ge = -3.0;
        if (yr == RLO && b.type[S_YLO] == T_DIRI) D.gs = -3.0;
        if (yr == RHI && b.type[S_YHI] == T_DIRI) D.gn = -3.0;
    }
    St9 s;
    gather9(D, xr, yr, s);
    return lap9(s, g, i, j, xr, yr, b, homog);
}

// One Gauss-Seidel update of (i,j) in regions (xr, yr) (P2:1768-1771).
template <class T>
__device__ __forceinline__ void gs9r(const DFT<T>& phi, const DFT<T>& rhs, const DFT<T>& invd, const GeoT<T>& g,
                                     const BCd& b, int homog, int i, int j, int xr, int yr, double omega) {
    const T lphi = apply9r(phi, g, b, homog, i, j, xr, yr);
    const T p = AT(phi, i, j);
    const T newphi = p + (AT(rhs, i, j) - lphi) * AT(invd, i, j);
    AT(phi, i, j) = T(omega) * newphi + T(1.0 - omega) * p;
}

// The same, regions from the position.
template <class T>
__device__ __forceinline__ void gs9(const DFT<T>& phi, const DFT<T>& rhs, const DFT<T>& invd, const GeoT<T>& g,
                                    const BCd& b, int homog, int nx, int ny, int i, int j, double omega) {
    const Per pr = periodic_of(b);
    gs9r(phi, rhs, invd, g, b, homog, i, j, region(i, nx, pr.xl, pr.xh), region(j, ny, pr.yl, pr.yh), omega);
}

// ---------------------------------------------------------------------------
// The ghost values a Gauss-Seidel sweep starts from: fill_ghosts with
// do_neum = .false. (P2:1556) for sides of type DIRI, NEUM (left as stored)
// and PERIODIC, computed from interior values only, so all ghost cells can
// be filled at once.  P(i,j) reads phi as it stands at the sweep start.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T ghost_diri(const BCd& b, int homog, int s, int k, T p0, T p1, T p2);

// y-side ghost (i,j), 0 <= i < nx.
template <class P>
__device__ __forceinline__ auto sweep_ghost_y(const P& p, const BCd& b, int homog, int ny, int i, int j) {
    const int s = (j < 0) ? S_YLO : S_YHI;
    const int t = b.type[s];
    if (t == T_DIRI) {
        const int jj = (j < 0) ? 0 : ny - 1, e = (j < 0) ? -1 : 1;
        return ghost_diri(b, homog, s, i, p(i, jj), p(i, jj - e), p(i, jj - 2 * e));
    }
    if (t == T_PERIODIC) return p(i, (j < 0) ? ny - 1 : 0);
    return p(i, j);
}

// x-side ghost (i,j), 0 <= j < ny.
template <class P>
__device__ __forceinline__ auto sweep_ghost_x(const P& p, const BCd& b, int homog, int nx, int i, int j) {
    const int s = (i < 0) ? S_XLO : S_XHI;
    const int t = b.type[s];
    if (t == T_DIRI) {
        const int ii = (i < 0) ? 0 : nx - 1, e = (i < 0) ? -1 : 1;
        return ghost_diri(b, homog, s, j, p(ii, j), p(ii - e, j), p(ii - 2 * e, j));
    }
    if (t == T_PERIODIC) return p((i < 0) ? nx - 1 : 0, j);
    return p(i, j);
}

// Any ghost cell; corners as AU:1460-1490.
template <class P>
__device__ __forceinline__ auto sweep_ghost(const P& p, const BCd& b, int homog, int nx, int ny, int i, int j) {
    const bool xin = (i >= 0 && i < nx), yin = (j >= 0 && j < ny);
    if (xin && !yin) return sweep_ghost_y(p, b, homog, ny, i, j);
    if (yin && !xin) return sweep_ghost_x(p, b, homog, nx, i, j);
    const bool px = b.type[S_XLO] == T_PERIODIC, py = b.type[S_YLO] == T_PERIODIC;
    if (!px && !py) return bogus<decltype(p(0, 0))>();
    const int wi = (i < 0) ? nx - 1 : 0, wj = (j < 0) ? ny - 1 : 0;
    if (px && py) return p(wi, wj);
    if (px) return sweep_ghost_y(p, b, homog, ny, wi, j);
    return sweep_ghost_x(p, b, homog, nx, i, wj);
}

// Reads a field directly.
template <class T>
struct DFLoadT {
    DFT<T> f;
    __device__ __forceinline__ T operator()(int i, int j) const { return AT(f, i, j); }
};
using DFLoad = DFLoadT<double>;

// k / d by a multiply: exact for 0 <= k < 65536 and 1 <= d <= 1024 (every
// pair checked on the host).  The magic number costs one divide; compute it
// off the critical path.
__device__ __forceinline__ unsigned long long fastdiv_magic(int d) {
    return ((1ull << 32) + (unsigned)d - 1) / (unsigned)d;
}
__device__ __forceinline__ int fastdiv(int k, unsigned long long m) {
    return (int)(((unsigned long long)(unsigned)k * m) >> 32);
}

// The same with a 24-bit magic number, which one 32-bit divide makes:
// m = ceil(2^24 / d), and floor(k * m / 2^24) = floor(k / d) whenever
// k * (d - 1) < 2^24 (so for k < 16384 with d <= 1024, and k < 65536 with
// d <= 256; both ranges checked exhaustively on the host).
__device__ __forceinline__ unsigned fastdiv24_magic(int d) {
    return ((1u << 24) + (unsigned)d - 1u) / (unsigned)d;
}
__device__ __forceinline__ int fastdiv24(int k, unsigned m) {
    return (int)(((unsigned long long)(unsigned)k * m) >> 24);
}

// Colour c of the 4-colour sweep: (i mod 2, j mod 2) = (0,0), (1,1), (1,0), (0,1).
__device__ __forceinline__ int colour_ci(int c) { return (c == 1 || c == 2) ? 1 : 0; }
__device__ __forceinline__ int colour_cj(int c) { return (c == 1 || c == 3) ? 1 : 0; }

// ---------------------------------------------------------------------------
// Ghost fills, AU:871-1492.  Each function returns the final value of one
// ghost cell of one side, given the array state the Fortran loop sees.
// ---------------------------------------------------------------------------

// Dirichlet, order 3 (AU:1161-1177, AU:1215-1231).  k = index along the side.
template <class T>
__device__ __forceinline__ T ghost_diri(const BCd& b, int homog, int s, int k, T p0, T p1, T p2) {
    const T sixteenfifth = T(16.0 / 5.0), fifth = T(1.0 / 5.0), three = T(3.0);
    if (b.mode[s] == M_LAH) return -p0;
    if (homog) return -(three * p0) + p1 - fifth * p2;
    if (b.mode[s] == M_UNIFORM) return sixteenfifth * T(b.u[s]) - three * p0 + p1 - fifth * p2;
    const T g = T((s < 2) ? b.d[s][k] : b.d[s][b.koffy + k]);
    return sixteenfifth * g - three * p0 + p1 - fifth * p2;
}

// Neumann on an x side (AU:926-985), ghost of row j.  Which formula last wrote
// row j depends on homog: homogeneous fills are one-sided at both ends;
// inhomogeneous fills rewrite jlo with the centred formula (which reads the y
// ghosts at jlo-1).
template <class T>
__device__ __forceinline__ T ghost_neum_x(const DFT<T>& p, const GeoT<T>& g, const BCd& b, int homog, int s, int nx,
                                               int ny, int j) {
    const bool lo = (s == S_XLO);
    const int e = lo ? -1 : 1, i = lo ? 0 : nx - 1;
    const T dx = T(lo ? -g.dx : g.dx), dy = T(g.dy);
    if (b.mode[s] == M_LAH) return AT(p, i, j);
    T dpn, dpf, cross;
    const T c3 = T(3.0), c4 = T(4.0), half = T(0.5), c15 = T(1.5);
    const bool onesided_lo = (j == 0) && homog;
    const bool onesided_hi = (j == ny - 1);
    if (onesided_lo) {
        dpn = -((c3 * AT(p, i, j) - c4 * AT(p, i, j + 1) + AT(p, i, j + 2)) * half / dy);
        dpf = -((c3 * AT(p, i - e, j) - c4 * AT(p, i - e, j + 1) + AT(p, i - e, j + 2)) * half / dy);
        cross = half * (c3 * dpn - dpf) * AT(g.xy, i, j);
    } else if (onesided_hi) {
        dpn = (c3 * AT(p, i, j) - c4 * AT(p, i, j - 1) + AT(p, i, j - 2)) * half / dy;
        dpf = (c3 * AT(p, i - e, j) - c4 * AT(p, i - e, j - 1) + AT(p, i - e, j - 2)) * half / dy;
        cross = half * (c3 * dpn - dpf) * AT(g.xy, i, j);
    } else {
        dpn = (AT(p, i, j + 1) - AT(p, i, j - 1)) * half / dy;
        dpf = (AT(p, i - e, j + 1) - AT(p, i - e, j - 1)) * half / dy;
        cross = (c15 * dpn - half * dpf) * AT(g.xy, i, j);
    }
    if (homog) return AT(p, i, j) - (-cross) * dx / AT(g.xx, i, j);
    const T bv = T((b.mode[s] == M_UNIFORM) ? b.u[s] : b.d[s][j]);
    return AT(p, i, j) - (bv - cross) * dx / AT(g.xx, i, j);
}

// Neumann on a y side (AU:990-1062), ghost of column i.  Column ilo always
// ends with the centred formula (it reads the x ghosts), ihi one-sided.
template <class T>
__device__ __forceinline__ T ghost_neum_y(const DFT<T>& p, const GeoT<T>& g, const BCd& b, int homog, int s, int nx,
                                               int ny, int i) {
    const bool lo = (s == S_YLO);
    const int e = lo ? -1 : 1, j = lo ? 0 : ny - 1;
    const T dy = T(lo ? -g.dy : g.dy), dx = T(g.dx);
    if (b.mode[s] == M_LAH) return AT(p, i, j);
    T dpn, dpf, cross;
    const T c3 = T(3.0), c4 = T(4.0), half = T(0.5), c15 = T(1.5);
    if (i == nx - 1) {
        dpn = (c3 * AT(p, i, j) - c4 * AT(p, i - 1, j) + AT(p, i - 2, j)) * half / dx;
        dpf = (c3 * AT(p, i, j - e) - c4 * AT(p, i - 1, j - e) + AT(p, i - 2, j - e)) * half / dx;
        cross = half * (c3 * dpn - dpf) * AT(g.yx, i, j);
    } else {
        dpn = (AT(p, i + 1, j) - AT(p, i - 1, j)) * half / dx;
        dpf = (AT(p, i + 1, j - e) - AT(p, i - 1, j - e)) * half / dx;
        cross = (c15 * dpn - half * dpf) * AT(g.yx, i, j);
    }
    if (homog) return AT(p, i, j) - (-cross) * dy / AT(g.yy, i, j);
    const T bv = T((b.mode[s] == M_UNIFORM) ? b.u[s] : b.d[s][i]);
    return AT(p, i, j) - (bv - cross) * dy / AT(g.yy, i, j);
}

// Number of ghost cells a side's fill writes, and the first index.
__device__ __forceinline__ void side_range(const BCd& b, int s, int nx, int ny, int do_neum, int& lo, int& cnt) {
    const int t = b.type[s];
    const int n = (s < 2) ? ny : nx;
    lo = 0;
    cnt = 0;
    if (t == T_NEUM) { if (do_neum) cnt = n; }
    else if (t == T_DIRI || t == T_PERIODIC) cnt = n;
    else if (t == T_EX0 || t == T_EX1 || t == T_EX2) { lo = -1; cnt = n + 2; }   // whole column/row incl. ghosts
}

// Ghost k of side s (k counted from `lo` of side_range).  Returns false if the
// side writes nothing there.  Writes the value.
template <class T>
__device__ __forceinline__ void fill_side_elem(const DFT<T>& p, const GeoT<T>& g, const BCd& b, int homog, int s, int nx,
                                               int ny, int k) {
    const int t = b.type[s];
    if (s < 2) {
        const bool lo = (s == S_XLO);
        const int i = lo ? 0 : nx - 1, e = lo ? -1 : 1;
        T v;
        if (t == T_NEUM) v = ghost_neum_x(p, g, b, homog, s, nx, ny, k);
        else if (t == T_DIRI) v = ghost_diri(b, homog, s, k, AT(p, i, k), AT(p, i - e, k), AT(p, i - 2 * e, k));
        else if (t == T_PERIODIC) v = lo ? AT(p, nx - 1, k) : AT(p, 0, k);
        else {
            const T v0 = AT(p, i, k), v1 = AT(p, i - e, k), v2 = AT(p, i - 2 * e, k);
            v = (t == T_EX0) ? v0 : (t == T_EX1) ? T(2.0) * v0 - v1 : T(3.0) * (v0 - v1) + v2;
        }
        AT(p, i + e, k) = v;
    } else {
        const bool lo = (s == S_YLO);
        const int j = lo ? 0 : ny - 1, e = lo ? -1 : 1;
        T v;
        if (t == T_NEUM) v = ghost_neum_y(p, g, b, homog, s, nx, ny, k);
        else if (t == T_DIRI) v = ghost_diri(b, homog, s, k, AT(p, k, j), AT(p, k, j - e), AT(p, k, j - 2 * e));
        else if (t == T_PERIODIC) v = lo ? AT(p, k, ny - 1) : AT(p, k, 0);
        else {
            const T v0 = AT(p, k, j), v1 = AT(p, k, j - e), v2 = AT(p, k, j - 2 * e);
            v = (t == T_EX0) ? v0 : (t == T_EX1) ? T(2.0) * v0 - v1 : T(3.0) * (v0 - v1) + v2;
        }
        AT(p, k, j + e) = v;
    }
}

// Corner ghosts, AU:1460-1490.  Corner c = 0..3: (-1,-1), (-1,ny), (nx,-1), (nx,ny).
template <class T>
__device__ __forceinline__ void fill_corner(const DFT<T>& p, const BCd& b, int nx, int ny, int c) {
    const bool px = b.type[S_XLO] == T_PERIODIC, py = b.type[S_YLO] == T_PERIODIC;
    const int ci = (c >= 2) ? nx : -1, cj = (c & 1) ? ny : -1;
    T v;
    if (!px && !py) v = bogus<T>();
    else if (px && py) v = AT(p, ci < 0 ? nx - 1 : 0, cj < 0 ? ny - 1 : 0);
    else if (px) v = AT(p, ci < 0 ? nx - 1 : 0, cj);
    else v = AT(p, ci, cj < 0 ? ny - 1 : 0);
    AT(p, ci, cj) = v;
}

// extrapolate_ghosts value for an x-ghost column (lo/hi) at row a, AU:1497-1566.
template <class T>
__device__ __forceinline__ T extrap_val(int order, T v0, T v1, T v2, T v3) {
    switch (order) {
        case 0: return v0;
        case 1: return T(2.0) * v0 - v1;
        case 2: return T(3.0) * (v0 - v1) + v2;
        default: return T(4.0) * (v0 + v2) - T(6.0) * v1 - v3;
    }
}

// ---------------------------------------------------------------------------
// Transfers, MG:135-394
// ---------------------------------------------------------------------------
// Cell-centred restriction (MG:145-158): sum in the Fortran loop order.
template <class T>
__device__ __forceinline__ T restrict_cc(const DFT<T>& f, int ci, int cj, int refx, int refy, double scale) {
    T acc = T(0.0);
    const T sc = T(scale);
    for (int a = 0; a < refy; ++a)
        for (int c = 0; c < refx; ++c) acc = acc + sc * AT(f, ci * refx + c, cj * refy + a);
    return acc;
}

// Fine += constant + linear (+ second-difference) terms for one coarse cell.
// The adds happen in the Fortran order: all constant adds (MG:304-314), then
// the linear ones (MG:316-333), then the quadratic ones (MG:335-352).  Each
// fine cell belongs to one coarse cell, so doing them per cell in sequence
// gives the same bits.
template <class TF, class TC>
__device__ __forceinline__ void prolong_cell(const DFT<TF>& fine, const DFT<TC>& crse, int ci, int cj, int refx, int refy,
                                             int order) {
    using R = TC;   // arithmetic in the coarse field's type
    const R half = R(0.5), quarter = R(0.25), two = R(2.0), eighth = R(0.125);
    const R c = AT(crse, ci, cj);
    const int fi = refx * ci, fj = refy * cj;
    R f00 = R(AT(fine, fi, fj));
    R f10 = refx == 2 ? R(AT(fine, fi + 1, fj)) : R(0.0);
    R f01 = refy == 2 ? R(AT(fine, fi, fj + 1)) : R(0.0);
    R f11 = (refx == 2 && refy == 2) ? R(AT(fine, fi + 1, fj + 1)) : R(0.0);
    f00 = f00 + c; f10 = f10 + c; f01 = f01 + c; f11 = f11 + c;
    if (order >= 1) {
        const R mx = half * (AT(crse, ci + 1, cj) - AT(crse, ci - 1, cj));
        const R my = half * (AT(crse, ci, cj + 1) - AT(crse, ci, cj - 1));
        if (refx == 2 && refy == 2) {
            f00 = f00 + quarter * (-mx - my);
            f10 = f10 + quarter * (mx - my);
            f01 = f01 + quarter * (-mx + my);
            f11 = f11 + quarter * (mx + my);
        } else if (refx == 2) {
            f00 = f00 + quarter * (-mx);
            f10 = f10 + quarter * (mx);
        } else {
            f00 = f00 + quarter * (-my);
            f01 = f01 + quarter * (my);
        }
    }
    if (order >= 2) {
        const R mx = quarter * (AT(crse, ci + 1, cj) - two * AT(crse, ci, cj) + AT(crse, ci - 1, cj));
        const R my = quarter * (AT(crse, ci, cj + 1) - two * AT(crse, ci, cj) + AT(crse, ci, cj - 1));
        const R q = (refx == 2 && refy == 2) ? eighth * (mx + my) : (refx == 2 ? eighth * mx : eighth * my);
        f00 = f00 + q; f10 = f10 + q; f01 = f01 + q; f11 = f11 + q;
    }
    AT(fine, fi, fj) = TF(f00);
    if (refx == 2) AT(fine, fi + 1, fj) = TF(f10);
    if (refy == 2) AT(fine, fi, fj + 1) = TF(f01);
    if (refx == 2 && refy == 2) AT(fine, fi + 1, fj + 1) = TF(f11);
}

// ---------------------------------------------------------------------------
// Deferred-correction operators, DD:45-334
// ---------------------------------------------------------------------------
// Value of phi at (i,j) after extrapolate_ghosts(phi, 0): indices clamped to the valid region.
template <class T>
__device__ __forceinline__ T clampv(const DFT<T>& p, int nx, int ny, int i, int j) {
    i = i < 0 ? 0 : (i > nx - 1 ? nx - 1 : i);
    j = j < 0 ? 0 : (j > ny - 1 ? ny - 1 : j);
    return AT(p, i, j);
}

// Value of phi at a neighbour after fill_ghosts with LAH BCs (AU:935-936, AU:1135-1136):
// Dirichlet ghost = -cell, Neumann ghost = cell, periodic = wrapped.  (i,j) is a
// valid cell and (di,dj) a unit step.
template <class T>
__device__ __forceinline__ T lahv(const DFT<T>& p, const BCd& b, int nx, int ny, int i, int j, int di, int dj) {
    const int ii = i + di, jj = j + dj;
    int s = -1;
    if (ii < 0) s = S_XLO;
    else if (ii >= nx) s = S_XHI;
    else if (jj < 0) s = S_YLO;
    else if (jj >= ny) s = S_YHI;
    if (s < 0) return AT(p, ii, jj);
    const int t = b.type[s];
    if (t == T_PERIODIC) {
        const int wi = (ii + nx) % nx, wj = (jj + ny) % ny;
        return AT(p, wi, wj);
    }
    if (t == T_DIRI) return -AT(p, i, j);
    if (t == T_NEUM) return AT(p, i, j);
    return AT(p, ii, jj);   // other types leave the ghost as stored
}

// The three DD routines below are written for both field types; for FP64 the
// operations are those of the Fortran routines in their order (T(x) of a
// double is x), for FP32 the same operations in single precision.

// Lagged corner cross terms of the DD smoother's modified rhs (DD:226-250).
template <class T>
__device__ __forceinline__ T dd_modrhs(const DFT<T>& phi, const DFT<T>& rhs, const GeoT<T>& g, int nx, int ny, int i,
                                       int j) {
    const T xyscale = T(0.5 * g.idx * g.idy);
    const T pne = clampv(phi, nx, ny, i + 1, j + 1), pnw = clampv(phi, nx, ny, i - 1, j + 1);
    const T psw = clampv(phi, nx, ny, i - 1, j - 1), pse = clampv(phi, nx, ny, i + 1, j - 1);
    const T gxye = AT(g.xy, i + 1, j) * (pne - pse);
    const T gxyw = AT(g.xy, i, j) * (pnw - psw);
    const T gyxn = AT(g.yx, i, j + 1) * (pne - pnw);
    const T gyxs = AT(g.yx, i, j) * (pse - psw);
    return AT(rhs, i, j) - (gxye - gxyw + gyxn - gyxs) * xyscale;
}

// DD compute_laplacian (DD:45-119) at (i,j), reading phi's valid cells only.
template <class T>
__device__ __forceinline__ T dd_apply(const DFT<T>& phi, const GeoT<T>& g, const BCd& b, int nx, int ny, int i, int j) {
    const T xyscale = T(0.25 * g.idx * g.idy), idx = T(g.idx), idy = T(g.idy);
    T pe = clampv(phi, nx, ny, i + 1, j), pw = clampv(phi, nx, ny, i - 1, j);
    T pn = clampv(phi, nx, ny, i, j + 1), ps = clampv(phi, nx, ny, i, j - 1);
    const T pne = clampv(phi, nx, ny, i + 1, j + 1), pnw = clampv(phi, nx, ny, i - 1, j + 1);
    const T psw = clampv(phi, nx, ny, i - 1, j - 1), pse = clampv(phi, nx, ny, i + 1, j - 1);
    const T gxye = AT(g.xy, i + 1, j) * (pne - pse + pn - ps);
    const T gxyw = AT(g.xy, i, j) * (pn - ps + pnw - psw);
    const T gyxn = AT(g.yx, i, j + 1) * (pne - pnw + pe - pw);
    const T gyxs = AT(g.yx, i, j) * (pe - pw + pse - psw);
    const T cross = (gxye - gxyw + gyxn - gyxs) * xyscale;
    const T p = AT(phi, i, j);
    pe = lahv(phi, b, nx, ny, i, j, 1, 0);
    pw = lahv(phi, b, nx, ny, i, j, -1, 0);
    pn = lahv(phi, b, nx, ny, i, j, 0, 1);
    ps = lahv(phi, b, nx, ny, i, j, 0, -1);
    const T xfe = AT(g.xx, i + 1, j) * (pe - p) * idx;
    const T xfw = AT(g.xx, i, j) * (p - pw) * idx;
    const T yfn = AT(g.yy, i, j + 1) * (pn - p) * idy;
    const T yfs = AT(g.yy, i, j) * (p - ps) * idy;
    return cross + (xfe - xfw) * idx + (yfn - yfs) * idy;
}

// One DD Gauss-Seidel update (DD:288-306); phi's ghosts hold the LAH fill.
template <class T>
__device__ __forceinline__ void dd_gs(const DFT<T>& phi, const DFT<T>& modrhs, const DFT<T>& invd, const GeoT<T>& g,
                                      int i, int j, double omega) {
    const T idx = T(g.idx), idy = T(g.idy);
    const T p = AT(phi, i, j), pe = AT(phi, i + 1, j), pw = AT(phi, i - 1, j);
    const T pn = AT(phi, i, j + 1), ps = AT(phi, i, j - 1);
    const T xfe = AT(g.xx, i + 1, j) * (pe - p) * idx;
    const T xfw = AT(g.xx, i, j) * (p - pw) * idx;
    const T yfn = AT(g.yy, i, j + 1) * (pn - p) * idy;
    const T yfs = AT(g.yy, i, j) * (p - ps) * idy;
    const T lphi = (xfe - xfw) * idx + (yfn - yfs) * idy;
    const T newphi = p + (AT(modrhs, i, j) - lphi) * AT(invd, i, j);
    AT(phi, i, j) = T(omega) * newphi + T(1.0 - omega) * p;
}

}  // namespace mgp
