// mgp_noalloc.cu -- solve_bicgstab2 for callers that cannot allocate device
// memory.
//
// mgp_solve_bicgstab2 allocates eight work arrays (and staging buffers) on
// every call.  Some callers cannot do that: a service that reserves its whole
// device-memory budget at start-up and forbids allocation afterwards, or code
// that runs while another component owns the device allocator -- cudaMalloc
// can fail there, and cudaMalloc/cudaFree also synchronise the device, which
// a caller keeping work queued on its own streams cannot accept.  This entry
// point takes the caller's device arrays and keeps its work arrays in one
// file-scope __device__ array, so it allocates nothing.
//
// The scratch array holds the work arrays of one solve on grids of at most
// MGP_NOALLOC_MAX_SIDE x MGP_NOALLOC_MAX_SIDE cells, about 1.2 MB, and every
// device that loads the library keeps it until the process exits.  All calls
// share it: two calls whose kernels overlap on the device (different streams,
// or different host threads) race on it and corrupt each other's results.
// Each call rewrites every scratch value it reads before reading it, so a
// call never depends on what the previous call left there.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/mgp2d.h"
#include "mgp_kernels.cuh"

namespace mgp {
int record_error(int code, const char* msg);
}

using namespace mgp;

namespace {

constexpr int kSide = MGP_NOALLOC_MAX_SIDE;
constexpr size_t kGhosted = (size_t)(kSide + 2) * (kSide + 2);
constexpr size_t kPlain = (size_t)kSide * kSide;
constexpr size_t kBcDoubles = 2 * (2 * (size_t)kSide + 2);
// e_loc, p_tilde, s_tilde (with ghosts); r, r_tilde, p, t, v, w; BC values; status
constexpr size_t kScratchDoubles = 3 * kGhosted + 6 * kPlain + kBcDoubles + 1;

static __device__ __align__(256) double g_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device.  The first call on a
// device resolves it (cudaGetSymbolAddress) with that device current.
int scratch_address(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return record_error(MGP_ECUDA, "solve_bicgstab2_noalloc: no current CUDA device");
    }
    if (dev < 0 || dev >= kMaxDevices) return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: device index too large");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return record_error(MGP_ECUDA, "solve_bicgstab2_noalloc: cudaGetSymbolAddress failed");
        }
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return MGP_OK;
}

bool on_device(const void* p) {
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int device_view(const mgp_array* a, int nxv, const char* what, DF* out) {
    if (!a || !a->data || a->ngx < 0 || a->ngy < 0) return record_error(MGP_EINVAL, what);
    const int ld = a->ld ? a->ld : nxv + 2 * a->ngx;
    if (ld < nxv + 2 * a->ngx) return record_error(MGP_EINVAL, what);
    if (!on_device(a->data)) return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: arrays must be device memory");
    out->ld = ld;
    out->p = a->data + a->ngx + (long)a->ngy * ld;
    return MGP_OK;
}

// type(bdry_data) -> BCd, with NONUNIFORM values copied into the scratch.
int scratch_bc(const mgp_bdry* b, const mgp_box* v, int homog, double* dst, BCd* out) {
    if (!b) return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: null bdry_data");
    std::memset(out, 0, sizeof *out);
    size_t off = 0;
    for (int s = 0; s < 4; ++s) {
        const int t = b->type[s], m = b->mode[s];
        if (t == MGP_BCTYPE_CF) return record_error(MGP_ENOTSUP, "fill_ghosts: BCTYPE_CF is not supported");
        if (t < MGP_BCTYPE_NONE || t > MGP_BCTYPE_EXTRAP2) return record_error(MGP_EINVAL, "fill_ghosts: invalid BCTYPE_");
        if (m == MGP_BCMODE_LAH) return record_error(MGP_EINVAL, "Poisson2d::compute_invdiags received BCMODE_LAH.");
        if (m != MGP_BCMODE_UNIFORM && m != MGP_BCMODE_NONUNIFORM) return record_error(MGP_EINVAL, "Bad BCMODE");
        out->type[s] = t;
        out->mode[s] = m;
        const int n = (s < 2) ? v->ny : v->nx;
        if (m == MGP_BCMODE_NONUNIFORM) {
            if (!b->data[s]) return record_error(MGP_EINVAL, "null NONUNIFORM boundary data");
            if (cudaMemcpy(dst + off, b->data[s], (size_t)n * sizeof(double), cudaMemcpyDefault) != cudaSuccess) {
                cudaGetLastError();
                return record_error(MGP_ECUDA, "solve_bicgstab2_noalloc: boundary data copy failed");
            }
            out->d[s] = dst + off;
            off += n;
        } else if (b->data[s]) {
            if (cudaMemcpy(&out->u[s], b->data[s], sizeof(double), cudaMemcpyDefault) != cudaSuccess) {
                cudaGetLastError();
                return record_error(MGP_ECUDA, "solve_bicgstab2_noalloc: boundary data copy failed");
            }
        }
    }
    if (b->type[3] == MGP_BCTYPE_NEUM && !homog && b->mode[3] == MGP_BCMODE_NONUNIFORM) {
        out->kyhi = v->jhi - v->ilo;   // poisson2d.f90 reads bc%data_yhi(j) at j = jhi
        if (out->kyhi < 0 || out->kyhi >= v->nx)
            return record_error(MGP_EINVAL, "north Neumann data is read at index jhi, outside its bounds");
    }
    for (int s = 2; s < 4; ++s)
        if (b->type[s] == MGP_BCTYPE_DIRI && !homog && b->mode[s] == MGP_BCMODE_NONUNIFORM && v->jlo != v->ilo)
            return record_error(MGP_EINVAL, "y-side nonuniform Dirichlet data needs jlo == ilo");
    return MGP_OK;
}

DF carve(double*& cur, int nx, int ny, int g) {
    DF f;
    f.ld = nx + 2 * g;
    f.p = cur + (size_t)g * f.ld + g;
    cur += (size_t)f.ld * (ny + 2 * g);
    return f;
}

}  // namespace

extern "C" int mgp_solve_bicgstab2_noalloc(const mgp_box* valid, mgp_array* phi, const mgp_array* rhs,
                                           const mgp_geo* geo, const mgp_bdry* bc, int homog,
                                           const mgp_array* invdiags, double tol, int max_iters, int max_restarts,
                                           int zerophi, int verbosity) {
    (void)verbosity;
    if (!valid || !geo) return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: null argument");
    const int nx = valid->nx, ny = valid->ny;
    if (nx != valid->ihi - valid->ilo + 1 || ny != valid->jhi - valid->jlo + 1)
        return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: box extents are inconsistent");
    if (nx < 4 || ny < 4) return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: at least 4 cells per direction");
    if (nx > kSide || ny > kSide)
        return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: grid larger than MGP_NOALLOC_MAX_SIDE cells per side");
    if (!phi || phi->ngx != 1 || phi->ngy != 1)
        return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: phi needs exactly one ghost layer");
    if (max_iters == 0) return MGP_OK;
    double* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;

    BicgArgs a;
    std::memset(&a, 0, sizeof a);
    Lv& L = a.L;
    L.nx = nx;
    L.ny = ny;
    if ((rc = device_view(phi, nx, "solve_bicgstab2_noalloc: bad phi", &a.phi))) return rc;
    if ((rc = device_view(rhs, nx, "solve_bicgstab2_noalloc: bad rhs", &a.rhs))) return rc;
    if ((rc = device_view(invdiags, nx, "solve_bicgstab2_noalloc: bad invdiags", &L.invd))) return rc;
    if ((rc = device_view(&geo->J, nx, "solve_bicgstab2_noalloc: bad J", &L.g.J))) return rc;
    if ((rc = device_view(&geo->Jgup_xx, nx + 1, "solve_bicgstab2_noalloc: bad Jgup_xx", &L.g.xx))) return rc;
    if ((rc = device_view(&geo->Jgup_xy, nx + 1, "solve_bicgstab2_noalloc: bad Jgup_xy", &L.g.xy))) return rc;
    if ((rc = device_view(&geo->Jgup_yx, nx, "solve_bicgstab2_noalloc: bad Jgup_yx", &L.g.yx))) return rc;
    if ((rc = device_view(&geo->Jgup_yy, nx, "solve_bicgstab2_noalloc: bad Jgup_yy", &L.g.yy))) return rc;
    if (!(geo->dx > 0) || !(geo->dy > 0)) return record_error(MGP_EINVAL, "solve_bicgstab2_noalloc: bad dx, dy");
    L.g.dx = geo->dx;
    L.g.dy = geo->dy;
    L.g.idx = 1.0 / geo->dx;
    L.g.idy = 1.0 / geo->dy;

    double* cur = base;
    L.ea = carve(cur, nx, ny, 1);
    L.pt = carve(cur, nx, ny, 1);
    L.st = carve(cur, nx, ny, 1);
    L.rr = carve(cur, nx, ny, 0);
    L.rt = carve(cur, nx, ny, 0);
    L.pp = carve(cur, nx, ny, 0);
    L.tt = carve(cur, nx, ny, 0);
    L.vv = carve(cur, nx, ny, 0);
    L.w = carve(cur, nx, ny, 0);
    double* bcdst = base + 3 * kGhosted + 6 * kPlain;
    int* status = reinterpret_cast<int*>(base + kScratchDoubles - 1);
    if ((rc = scratch_bc(bc, valid, homog, bcdst, &L.bc))) return rc;

    a.homog = homog;
    a.tol = tol;
    a.max_iters = max_iters;
    a.max_restarts = max_restarts;
    a.zerophi = zerophi;
    a.dd = 0;
    a.status = status;
    if (cudaMemsetAsync(status, 0, sizeof(int), 0) != cudaSuccess ||
        launch_bicgstab(a, 0) != cudaSuccess) {
        cudaGetLastError();
        return record_error(MGP_ECUDA, "solve_bicgstab2_noalloc: launch failed");
    }
    int st = 0;
    if (cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return record_error(MGP_ECUDA, "solve_bicgstab2_noalloc: kernel failed");
    }
    if (st) return record_error(MGP_EDIVERGED, "solve_bicgstab2_noalloc: non-finite residual");
    return MGP_OK;
}
