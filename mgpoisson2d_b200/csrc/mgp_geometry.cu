// mgp_geometry.cu -- metric terms and right-hand sides generated on the
// device from an analytic map x(xi, eta), y(xi, eta).
//
// The Fortran test program builds J and J g^{ij} on the host from its map
// (test.f90:566-716); a caller that serves many problems would then copy
// five metric arrays per problem to the device.  Here the map is evaluated
// where the arrays live.  The metric formulas are the general ones,
//   J = x_xi y_eta - x_eta y_xi,
//   J g^{xi xi} = (x_eta^2 + y_eta^2) / J,
//   J g^{xi eta} = J g^{eta xi} = -(x_xi x_eta + y_xi y_eta) / J,
//   J g^{eta eta} = (x_xi^2 + y_xi^2) / J,
// with the derivatives taken as one-cell differences of the map at the
// points half a cell either side (the same construction as the host
// generator, so the two agree to rounding of the map's transcendentals).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "../../include/mgp2d.h"
#include "mgp_kernels.cuh"

namespace mgp {
int record_error(int code, const char* msg);
}

using namespace mgp;

namespace {

// A map with its constants resolved on the host.
struct MapC {
    int kind;
    double a;       // WAVY_EXP: amplitude          SKEW_LAYER: tan(angle)
    double beta;    // WAVY_EXP: beta               SKEW_LAYER: log(ratio) (0: no stretch)
    double den;     // WAVY_EXP: expm1(beta)        SKEW_LAYER: the layer's width in cells t*
    double nref;    // SKEW_LAYER: cells the stretch is laid out over
    double total;   // SKEW_LAYER: the stretched coordinate at eta = 1, before normalising
};

// Stretched coordinate of the wall layer at t cells from the wall: cell
// heights grow by exp(lr) per cell up to t*, constant beyond; linear below 0.
__host__ __device__ inline double layer_prim(double t, double lr, double tstar) {
    if (t < 0.0) return t;
    const double inner = expm1(lr * fmin(t, tstar)) / lr;
    const double outer = exp(lr * tstar) * fmax(t - tstar, 0.0);
    return inner + outer;
}

__device__ inline void map_eval(const MapC& m, double xi, double eta, double& x, double& y) {
    const double twopi = 6.283185307179586;
    if (m.kind == MGP_MAP_WAVY_EXP) {
        x = xi + m.a * sin(twopi * xi) * sin(twopi * eta);
        y = expm1(m.beta * eta) / m.den;
    } else if (m.kind == MGP_MAP_SKEW_LAYER) {
        y = (m.beta == 0.0) ? eta : layer_prim(eta * m.nref, m.beta, m.den) / m.total;
        x = xi + m.a * y;
    } else {
        x = xi;
        y = eta;
    }
}

// x_xi, x_eta, y_xi, y_eta at (xi, eta).
__device__ inline void derivs(const MapC& m, double xi, double eta, double dx, double dy, double d[4]) {
    const double sx = 1.0 / dx, sy = 1.0 / dy, hx = 0.5 * dx, hy = 0.5 * dy;
    double xe, ye, xw, yw, xn, yn, xs, ys;
    map_eval(m, xi + hx, eta, xe, ye);
    map_eval(m, xi - hx, eta, xw, yw);
    map_eval(m, xi, eta + hy, xn, yn);
    map_eval(m, xi, eta - hy, xs, ys);
    d[0] = (xe - xw) * sx;
    d[1] = (xn - xs) * sy;
    d[2] = (ye - yw) * sx;
    d[3] = (yn - ys) * sy;
}

// One metric array over its whole allocation (valid points and ghosts).
// what: 0 J (cells), 1 Jgup_xx, 2 Jgup_xy (x-faces), 3 Jgup_yx, 4 Jgup_yy (y-faces).
__global__ void k_metric(DF out, int what, MapC m, int ilo, int jlo, double dx, double dy, int nvx, int nvy, int gx,
                         int gy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - gx;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - gy;
    if (i >= nvx + gx || j >= nvy + gy) return;
    const double offx = (what == 1 || what == 2) ? 0.0 : 0.5;
    const double offy = (what == 3 || what == 4) ? 0.0 : 0.5;
    const double xi = ((double)(ilo + i) + offx) * dx, eta = ((double)(jlo + j) + offy) * dy;
    double d[4];
    derivs(m, xi, eta, dx, dy, d);
    const double J = d[0] * d[3] - d[1] * d[2];
    double v;
    switch (what) {
        case 0: v = J; break;
        case 1: v = (d[1] * d[1] + d[3] * d[3]) / J; break;
        case 2:
        case 3: v = -(d[0] * d[1] + d[2] * d[3]) / J; break;
        default: v = (d[0] * d[0] + d[2] * d[2]) / J; break;
    }
    AT(out, i, j) = v;
}

// f = sum_k a_k cos(pi m_k x) cos(pi n_k y) at the cell centres.
__global__ void k_fourier(DF f, MapC m, int ilo, int jlo, double dx, double dy, int nx, int ny, int nmodes,
                          const double* amp, const int* mm, const int* nn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    const double pi = 3.141592653589793;
    double x, y;
    map_eval(m, ((double)(ilo + i) + 0.5) * dx, ((double)(jlo + j) + 0.5) * dy, x, y);
    double acc = 0.0;
    for (int k = 0; k < nmodes; ++k) acc = acc + amp[k] * cos(pi * mm[k] * x) * cos(pi * nn[k] * y);
    AT(f, i, j) = acc;
}

// rhs = J (f - mean_J f), mean_J f = out[0] / out[1].
__global__ void k_center_scale(DF f, DF J, const double* out, int nx, int ny) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    AT(f, i, j) = AT(J, i, j) * (AT(f, i, j) - out[0] / out[1]);
}

int resolve(int map, const double* params, MapC* m) {
    m->kind = map;
    m->a = m->beta = m->den = m->nref = m->total = 0.0;
    if (map == MGP_MAP_IDENTITY) return MGP_OK;
    if (!params) return record_error(MGP_EINVAL, "map: null parameters");
    if (map == MGP_MAP_WAVY_EXP) {
        m->a = params[0];
        m->beta = params[1];
        m->den = std::expm1(m->beta);
        if (!(m->beta > 0.0)) return record_error(MGP_EINVAL, "map: WAVY_EXP needs beta > 0");
        return MGP_OK;
    }
    if (map == MGP_MAP_SKEW_LAYER) {
        m->a = params[0];
        const double ratio = params[1];
        m->den = params[2];
        m->nref = params[3];
        if (!(ratio > 0.0) || !(m->nref > 0.0) || m->den < 0.0)
            return record_error(MGP_EINVAL, "map: SKEW_LAYER needs ratio > 0, n_ref > 0, t* >= 0");
        m->beta = (std::fabs(ratio - 1.0) < 1e-14) ? 0.0 : std::log(ratio);
        if (m->beta != 0.0) m->total = layer_prim(m->nref, m->beta, m->den);
        return MGP_OK;
    }
    return record_error(MGP_EINVAL, "map: unknown map kind");
}

bool on_device(const void* p) {
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int array_ld(const mgp_array* a, int nvx) { return a->ld ? a->ld : nvx + 2 * a->ngx; }

// Runs `fill` on the caller array, or on a device copy of it when it is host
// memory (copied in first when `in`, back to the host after when `out`).
template <class F>
int with_device(const mgp_array* a, int nvx, int nvy, const char* what, bool in, bool out, F fill) {
    if (!a || !a->data || a->ngx < 0 || a->ngy < 0) return record_error(MGP_EINVAL, what);
    const int ld = array_ld(a, nvx);
    if (ld < nvx + 2 * a->ngx) return record_error(MGP_EINVAL, what);
    DF f;
    f.ld = ld;
    const size_t n = (size_t)ld * (nvy + 2 * a->ngy);
    if (on_device(a->data)) {
        f.p = a->data + a->ngx + (size_t)a->ngy * ld;
        return fill(f, a->ngx, a->ngy);
    }
    double* buf = nullptr;
    if (cudaMalloc(&buf, n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return record_error(MGP_ENOMEM, "map: cudaMalloc failed");
    }
    f.p = buf + a->ngx + (size_t)a->ngy * ld;
    if (in && cudaMemcpy(buf, a->data, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(buf);
        return record_error(MGP_ECUDA, "map: copy to the device failed");
    }
    int rc = fill(f, a->ngx, a->ngy);
    if (!rc && out && cudaMemcpy(a->data, buf, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        rc = record_error(MGP_ECUDA, "map: copy to the host failed");
    }
    cudaFree(buf);
    return rc;
}

}  // namespace

extern "C" {

int mgp_map_geometry(const mgp_box* valid, int map, const double* params, mgp_geo* geo) {
    if (!valid || !geo || valid->nx <= 0 || valid->ny <= 0 || !(valid->dx > 0) || !(valid->dy > 0))
        return record_error(MGP_EINVAL, "map_geometry: bad box or null geometry");
    MapC m;
    int rc = resolve(map, params, &m);
    if (rc) return rc;
    const int nx = valid->nx, ny = valid->ny;
    struct Arr {
        mgp_array* a;
        int what, nvx, nvy;
        const char* name;
    } arrs[5] = {{&geo->J, 0, nx, ny, "map_geometry: bad J"},
                 {&geo->Jgup_xx, 1, nx + 1, ny, "map_geometry: bad Jgup_xx"},
                 {&geo->Jgup_xy, 2, nx + 1, ny, "map_geometry: bad Jgup_xy"},
                 {&geo->Jgup_yx, 3, nx, ny + 1, "map_geometry: bad Jgup_yx"},
                 {&geo->Jgup_yy, 4, nx, ny + 1, "map_geometry: bad Jgup_yy"}};
    for (const Arr& a : arrs) {
        rc = with_device(a.a, a.nvx, a.nvy, a.name, true, true, [&](const DF& f, int gx, int gy) -> int {
            const dim3 blk(32, 8), grd((a.nvx + 2 * gx + 31) / 32, (a.nvy + 2 * gy + 7) / 8);
            k_metric<<<grd, blk>>>(f, a.what, m, valid->ilo, valid->jlo, valid->dx, valid->dy, a.nvx, a.nvy, gx,
                                   gy);
            count_launch();
            if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
                cudaGetLastError();
                return record_error(MGP_ECUDA, "map_geometry: kernel failed");
            }
            return MGP_OK;
        });
        if (rc) return rc;
    }
    geo->dx = valid->dx;
    geo->dy = valid->dy;
    return MGP_OK;
}

int mgp_map_fourier_rhs(const mgp_box* valid, int map, const double* params, int nmodes, const double* amp,
                        const int* m_x, const int* m_y, const mgp_array* J, mgp_array* rhs) {
    if (!valid || !J || !rhs || nmodes < 0 || (nmodes > 0 && (!amp || !m_x || !m_y)))
        return record_error(MGP_EINVAL, "map_fourier_rhs: null argument");
    MapC m;
    int rc = resolve(map, params, &m);
    if (rc) return rc;
    const int nx = valid->nx, ny = valid->ny;
    double* dbuf = nullptr;   // amplitudes, then reduction partials and outputs
    int* ibuf = nullptr;
    const size_t nd = (size_t)nmodes + 2 * kRedBlocksMax + 8;
    if (cudaMalloc(&dbuf, nd * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&ibuf, (2 * (size_t)nmodes + 1) * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        if (dbuf) cudaFree(dbuf);
        return record_error(MGP_ENOMEM, "map_fourier_rhs: cudaMalloc failed");
    }
    if (nmodes > 0 && (cudaMemcpy(dbuf, amp, nmodes * sizeof(double), cudaMemcpyDefault) != cudaSuccess ||
                       cudaMemcpy(ibuf, m_x, nmodes * sizeof(int), cudaMemcpyDefault) != cudaSuccess ||
                       cudaMemcpy(ibuf + nmodes, m_y, nmodes * sizeof(int), cudaMemcpyDefault) != cudaSuccess)) {
        cudaGetLastError();
        cudaFree(dbuf);
        cudaFree(ibuf);
        return record_error(MGP_ECUDA, "map_fourier_rhs: copy of the modes failed");
    }
    // J on the device (a copy when it is host memory)
    rc = with_device(J, nx, ny, "map_fourier_rhs: bad J", true, false, [&](const DF& jd, int, int) -> int {
        return with_device(rhs, nx, ny, "map_fourier_rhs: bad rhs", true, true, [&](const DF& f, int, int) -> int {
            const dim3 blk(32, 8), grd((nx + 31) / 32, (ny + 7) / 8);
            k_fourier<<<grd, blk>>>(f, m, valid->ilo, valid->jlo, valid->dx, valid->dy, nx, ny, nmodes, dbuf, ibuf,
                                    ibuf + nmodes);
            count_launch();
            double* partials = dbuf + nmodes;
            double* out = partials + 2 * kRedBlocksMax;
            if (launch_reduce(RED_JSUM, f, jd, nx, ny, valid->dx * valid->dy, partials, out, 0) != cudaSuccess)
                return record_error(MGP_ECUDA, "map_fourier_rhs: reduction failed");
            k_center_scale<<<grd, blk>>>(f, jd, out, nx, ny);
            count_launch();
            if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
                cudaGetLastError();
                return record_error(MGP_ECUDA, "map_fourier_rhs: kernel failed");
            }
            return MGP_OK;
        });
    });
    cudaFree(dbuf);
    cudaFree(ibuf);
    return rc;
}

}  // extern "C"
