// mgp_host.cu -- host side of the B200 multigrid solver: hierarchy set-up,
// the V-cycle / FMG / deferred-correction drivers, array staging and the C ABI
// declared in include/mgp2d.h.
//
// The drivers follow MGPoisson2D.f90 (vcycle MG:400-670, vcycle_noinit
// MG:675-854, fmg MG:860-1122, fmg_noinit MG:1127-1189) and
// MGPoisson2D_DD.f90 (vcycle DD:589-862, vcycle_noinit DD:867-1045) step for
// step; the levels small enough for one CTA run their whole sub-cycle in
// k_coarse_cycle.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/mgp2d.h"
#include "mgp_kernels.cuh"

using namespace mgp;

namespace {

thread_local std::string g_err;
int g_flags = 0;

int set_err(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(x)                                                                                     \
    do {                                                                                          \
        cudaError_t e_ = (x);                                                                     \
        if (e_ != cudaSuccess) return set_err(MGP_ECUDA, "%s: %s", #x, cudaGetErrorString(e_));   \
    } while (0)
#define RC(x)                   \
    do {                        \
        int r_ = (x);           \
        if (r_) return r_;      \
    } while (0)

// GMRES restart length and the blocks of its many-vector reductions.
constexpr int kGmresRestart = 128;
constexpr int kGmresBlocks = 296;

// Levels with at most this many cells run inside the single-CTA coarse cycle.
constexpr long kCoarseCells = 1024;
// When the schedule stops above that (an odd side), the coarse cycle runs on
// the coarsest level alone; beyond this many cells it runs as a cooperative
// grid of one CTA per 256 cells (at most one per SM) instead of one CTA.
constexpr long kGridCoarseCells = 8192;
// Largest coarse-cycle level run by one thread-block cluster (cells).
constexpr long kClusterCoarseCells = 1L << 17;

// ---------------------------------------------------------------------------
// Device memory of solvers comes from a stream-ordered pool per device, owned
// by this library, that keeps up to kPoolKeepBytes of freed memory for the
// next solver instead of handing it back to the driver.  The Fortran-signature
// drivers build and free a whole hierarchy in every call (as MG:469-533 and
// MG:646-668 allocate and deallocate it); cudaMalloc and cudaFree of it cost
// milliseconds, a reuse from the pool microseconds.  Where the device has no
// memory pools the plain calls are used.
// ---------------------------------------------------------------------------
// The pool keeps an eighth of the device's memory (at least 4 GB) once
// freed: enough for a resident hierarchy with GMRES's stored vectors and a
// one-shot call's own beside it (2.7 GB each at 1024^2), so the one-shot
// drivers reuse memory instead of returning and re-mapping it per call.
constexpr unsigned long long kPoolKeepMinBytes = 4ull << 30;

cudaMemPool_t solver_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    static bool tried[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!tried[dev]) {
        tried[dev] = true;
        int supported = 0;
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        size_t freeb = 0, totalb = 0;
        if (cudaMemGetInfo(&freeb, &totalb) != cudaSuccess) {
            cudaGetLastError();
            totalb = 0;
        }
        unsigned long long keep = std::max<unsigned long long>(kPoolKeepMinBytes, totalb / 8);
        if (cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev) == cudaSuccess && supported &&
            cudaMemPoolCreate(&p, &props) == cudaSuccess &&
            cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess)
            pools[dev] = p;
        else
            cudaGetLastError();
    }
    return pools[dev];
}

// Memory the pool holds but no solver uses (freed, kept for reuse).
size_t pool_cached_bytes() {
    cudaMemPool_t p = solver_pool();
    if (!p) return 0;
    unsigned long long reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
        cudaMemPoolGetAttribute(p, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return reserved > used ? (size_t)(reserved - used) : 0;
}

// The current device's total memory, queried once per device.
size_t device_total_bytes() {
    static std::mutex mu;
    static size_t total[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 0;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!total[dev]) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) total[dev] = tot;
        else cudaGetLastError();
    }
    return total[dev];
}

// Allocation ordered on stream st (usable there at once, elsewhere after st is synchronised).
cudaError_t dmalloc(void** p, size_t bytes, cudaStream_t st) {
    if (cudaMemPool_t pool = solver_pool()) return cudaMallocFromPoolAsync(p, bytes, pool, st);
    return cudaMalloc(p, bytes);
}
template <class T>
cudaError_t dmalloc(T** p, size_t bytes, cudaStream_t st) {
    return dmalloc(reinterpret_cast<void**>(p), bytes, st);
}
// The caller has synchronised every stream that used p.
void dfree(void* p, cudaStream_t st) {
    if (!p) return;
    if (solver_pool()) cudaFreeAsync(p, st);
    else cudaFree(p);
}

// Small pinned host buffers (a solver's reduction read-back) from 4 KB slabs
// that are never returned: page-locking costs far more than the buffer.
constexpr size_t kPinnedSlot = 64;
struct PinnedSlots {
    std::mutex mu;
    std::vector<void*> free_slots;
    void* get() {
        std::lock_guard<std::mutex> lock(mu);
        if (free_slots.empty()) {
            char* slab = nullptr;
            if (cudaMallocHost(&slab, 4096) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            for (size_t k = 0; k < 4096 / kPinnedSlot; ++k) free_slots.push_back(slab + k * kPinnedSlot);
        }
        void* p = free_slots.back();
        free_slots.pop_back();
        return p;
    }
    void put(void* p) {
        if (!p) return;
        std::lock_guard<std::mutex> lock(mu);
        free_slots.push_back(p);
    }
};
PinnedSlots& pinned_slots() {
    static PinnedSlots* slots = new PinnedSlots();   // never destroyed: solvers may outlive static teardown
    return *slots;
}

// ---------------------------------------------------------------------------
// Device memory: every field of a solver comes out of one allocation.
// ---------------------------------------------------------------------------
template <class T>
struct Spec {
    DFT<T>* dst;
    int nxv, nyv, g;
    size_t off;   // element offset of the field's block
};

template <class T>
struct ArenaT {
    std::vector<Spec<T>> specs;
    size_t elems = 0;
    T* base = nullptr;
    void add(DFT<T>* dst, int nxv, int nyv, int g) {
        // arrays with ghosts keep spare columns, so the sweep's TMA window (from
        // the 16-byte-aligned column left of the ghost column -1) still covers
        // the ghost column nx
        const int spare = g ? 16 / (int)sizeof(T) - 1 : 0;
        const int ld = ((nxv + 2 * g + spare + 31) / 32) * 32;
        const size_t pad = g ? 32 : 0;
        const size_t n = (size_t)(nyv + 2 * g) * ld + 2 * pad;
        Spec<T> s{dst, nxv, nyv, g, elems};
        specs.push_back(s);
        dst->ld = ld;
        elems += (n + 31) / 32 * 32;
    }
    int commit(cudaStream_t st) {
        if (elems == 0) return MGP_OK;
        if (dmalloc(&base, elems * sizeof(T), st) != cudaSuccess) {
            cudaGetLastError();
            base = nullptr;
            return set_err(MGP_ENOMEM, "device allocation of %zu bytes failed", elems * sizeof(T));
        }
        for (auto& s : specs) {
            const size_t pad = s.g ? 32 : 0;
            s.dst->p = base + s.off + pad + (size_t)s.g * s.dst->ld;
        }
        CK(cudaMemsetAsync(base, 0, elems * sizeof(T), st));   // fresh arrays start at zero
        return MGP_OK;
    }
    void release() {   // after a device synchronisation (solver_free)
        dfree(base, nullptr);
        base = nullptr;
        specs.clear();
        elems = 0;
    }
};
using Arena = ArenaT<double>;
using Arena32 = ArenaT<float>;

// ---------------------------------------------------------------------------
// Argument checks and staging of caller arrays
// ---------------------------------------------------------------------------
int check_box(const mgp_box* v) {
    if (!v) return set_err(MGP_EINVAL, "null box");
    if (v->nx != v->ihi - v->ilo + 1 || v->ny != v->jhi - v->jlo + 1)
        return set_err(MGP_EINVAL, "box extents are inconsistent (nx=%d ilo=%d ihi=%d)", v->nx, v->ilo, v->ihi);
    if (v->nx < 3 || v->ny < 3) return set_err(MGP_EINVAL, "the operator needs at least 3 cells per direction");
    if (!(v->dx > 0) || !(v->dy > 0)) return set_err(MGP_EINVAL, "dx and dy must be positive");
    return MGP_OK;
}

int array_ld(const mgp_array* a, int nxv) { return a->ld ? a->ld : nxv + 2 * a->ngx; }

int check_array(const mgp_array* a, int nxv, const char* what) {
    if (!a || !a->data) return set_err(MGP_EINVAL, "%s: null array", what);
    if (a->ngx < 0 || a->ngy < 0) return set_err(MGP_EINVAL, "%s: negative ghost count", what);
    if (array_ld(a, nxv) < nxv + 2 * a->ngx) return set_err(MGP_EINVAL, "%s: leading dimension too small", what);
    return MGP_OK;
}

// Copy the part of a caller array that the device field holds (valid cells
// and up to `gmax` ghost layers).  cudaMemcpyDefault lets the driver tell host
// from device memory.
int stage_in(const mgp_array* u, int nxv, int nyv, const DF& d, int gmax, cudaStream_t st) {
    const int gx = u->ngx < gmax ? u->ngx : gmax, gy = u->ngy < gmax ? u->ngy : gmax;
    const long uld = array_ld(u, nxv);
    const double* src = u->data + (u->ngx - gx) + (long)(u->ngy - gy) * uld;
    double* dst = d.p - gx - (long)gy * d.ld;
    CK(cudaMemcpy2DAsync(dst, (size_t)d.ld * 8, src, (size_t)uld * 8, (size_t)(nxv + 2 * gx) * 8, nyv + 2 * gy,
                         cudaMemcpyDefault, st));
    return MGP_OK;
}

int stage_out(const DF& d, const mgp_array* u, int nxv, int nyv, int gmax, cudaStream_t st) {
    const int gx = u->ngx < gmax ? u->ngx : gmax, gy = u->ngy < gmax ? u->ngy : gmax;
    const long uld = array_ld(u, nxv);
    double* dst = u->data + (u->ngx - gx) + (long)(u->ngy - gy) * uld;
    const double* src = d.p - gx - (long)gy * d.ld;
    CK(cudaMemcpy2DAsync(dst, (size_t)uld * 8, src, (size_t)d.ld * 8, (size_t)(nxv + 2 * gx) * 8, nyv + 2 * gy,
                         cudaMemcpyDefault, st));
    return MGP_OK;
}

int read_scalar(const double* p, double* out) {
    CK(cudaMemcpy(out, p, sizeof(double), cudaMemcpyDefault));
    return MGP_OK;
}

// type(bdry_data) -> BCd.  NONUNIFORM values are copied to `dbuf` (device,
// 2*(nx+ny) doubles).  homog selects which checks apply.
int make_bc(const mgp_bdry* b, const mgp_box* v, int homog, double* dbuf, BCd* out, cudaStream_t st) {
    if (!b) return set_err(MGP_EINVAL, "null bdry_data");
    std::memset(out, 0, sizeof *out);
    size_t off = 0;
    for (int s = 0; s < 4; ++s) {
        const int t = b->type[s], m = b->mode[s];
        if (t == MGP_BCTYPE_CF) return set_err(MGP_ENOTSUP, "fill_ghosts: BCTYPE_CF is not supported");
        if (t < MGP_BCTYPE_NONE || t > MGP_BCTYPE_EXTRAP2) return set_err(MGP_EINVAL, "fill_ghosts: invalid BCTYPE_");
        if (m < MGP_BCMODE_UNIFORM || m > MGP_BCMODE_LAH) return set_err(MGP_EINVAL, "define_bdry_data: Bad BCMODE");
        out->type[s] = t;
        out->mode[s] = m;
        const int n = (s < 2) ? v->ny : v->nx;
        if (m == MGP_BCMODE_NONUNIFORM) {
            if (!b->data[s]) return set_err(MGP_EINVAL, "null NONUNIFORM boundary data");
            CK(cudaMemcpyAsync(dbuf + off, b->data[s], (size_t)n * 8, cudaMemcpyDefault, st));
            out->d[s] = dbuf + off;
            off += n;
        } else {
            double u = 0.0;
            if (b->data[s]) RC(read_scalar(b->data[s], &u));
            out->u[s] = u;
        }
    }
    // The Fortran operator reads the north-face Neumann data at index jhi
    // (poisson2d.f90:1208, 1248, 1298 `bc%data_yhi(j)`); keep that, and refuse
    // the cases where that index is outside the array.
    if (b->type[3] == MGP_BCTYPE_NEUM && !homog && b->mode[3] == MGP_BCMODE_NONUNIFORM) {
        out->kyhi = v->jhi - v->ilo;
        if (out->kyhi < 0 || out->kyhi >= v->nx)
            return set_err(MGP_EINVAL, "north Neumann data is read at index jhi, outside its bounds");
    }
    // Y-side NONUNIFORM Dirichlet data is read as bcd(jlo:jhi) (arrayutils.f90:1224).
    for (int s = 2; s < 4; ++s)
        if (b->type[s] == MGP_BCTYPE_DIRI && !homog && b->mode[s] == MGP_BCMODE_NONUNIFORM) {
            out->koffy = v->jlo - v->ilo;
            if (out->koffy != 0)
                return set_err(MGP_EINVAL, "y-side nonuniform Dirichlet data needs jlo == ilo");
        }
    return MGP_OK;
}

Geo make_geo(DF J, DF xx, DF xy, DF yx, DF yy, double dx, double dy) {
    Geo g;
    g.J = J; g.xx = xx; g.xy = xy; g.yx = yx; g.yy = yy;
    g.dx = dx; g.dy = dy;
    g.idx = 1.0 / dx;
    g.idy = 1.0 / dy;
    return g;
}

// ---------------------------------------------------------------------------
// Schedule (MG:38-129)
// ---------------------------------------------------------------------------
void estimate_maxdepth(int* maxdepth, const mgp_box* v) {
    int mgnx = v->nx, mgny = v->ny, d;
    for (d = 0; d <= *maxdepth - 1; ++d) {
        if (mgnx % 2 == 0) mgnx /= 2;
        else if (mgny % 2 == 0) mgny /= 2;
        else break;
    }
    if (d + 1 < *maxdepth) *maxdepth = d + 1;
}

void create_mgschedule(std::vector<int>& refx, std::vector<int>& refy, int* maxdepth, const mgp_box* v) {
    const int min_nx = 4, min_ny = 4;
    int mgnx = v->nx, mgny = v->ny, d;
    double mgdx = v->dx, mgdy = v->dy;
    refx.assign(*maxdepth + 1, 0);
    refy.assign(*maxdepth + 1, 0);
    for (d = 0; d <= *maxdepth - 1; ++d) {
        if ((mgnx % 2 != 0) || (mgny % 2 != 0)) break;
        const double max_dx = mgdx > mgdy ? mgdx : mgdy;
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
}

}  // namespace

// ---------------------------------------------------------------------------
// The resident hierarchy
// ---------------------------------------------------------------------------
struct mgp_solver {
    int kind = MGP_KIND_MG;
    int flags = 0;
    int maxdepth = 0;
    int dc = 0;   // first level handled by the coarse CTA
    mgp_box valid{};
    int types[4] = {0, 0, 0, 0};
    std::vector<int> refx, refy;
    std::vector<Lv> lv;
    Lv* d_lv = nullptr;
    Lv* d_shadow = nullptr; // coarse levels' shared-memory layout (offsets), or nullptr
    int shadow_bytes = 0;
    // MGP_FLAG_DIRECT_COARSE: level db (>= dc) is the V-cycle's bottom, solved
    // with d_ainv, its operator's inverse (transposed); db = -1 without.
    // direct_large: db == dc, d_ainv row-major, applied by launch_direct_apply
    int db = -1;
    double* d_ainv = nullptr;
    bool direct_large = false;
    // coarse cycle as a cooperative grid of grid_ctas CTAs (0: one CTA)
    int grid_ctas = 0;
    int coarse_cluster = 0;   // the grid_ctas CTAs form one thread-block cluster (2: one-CTA reduction order)
    GridCtl gctl{};
    int* d_ref = nullptr;   // refx then refy
    int* d_status = nullptr;
    Arena fixed;            // geometry, inverse diagonals
    Arena state;            // everything a solve writes; zeroed at the start of each solve
    DF phi0{}, rhs0{};
    // MGP_FLAG_KRYLOV: BiCGStab vectors on level 0 (residual, shadow residual,
    // search direction, A*y and A*z)
    DF kr{}, krh{}, kp{}, kv{}, kt{};
    // MGP_FLAG_GMRES: 2m + 1 level-0 vectors (basis v_0..v_m, then the
    // preconditioned z_0..z_{m-1}), each (nx + 2) x (ny + 2) with a ghost
    // layer, and the reduction scratch (partials, two Gram-Schmidt columns,
    // a norm, the update coefficients)
    double* gm_base = nullptr;
    double* gm_red = nullptr;
    int gm_m = 0;
    size_t gm_vec = 0, gm_ld = 0;
    std::vector<SweepTma> tma;   // per level, for the fused sweep
    // MGP_FLAG_MIXED: FP32 copies of the grid-path levels 0 .. dc-1
    struct Lv32 {
        int nx = 0, ny = 0;
        Geo32 g{};
        DF32 e{}, e2{}, r{}, w{}, invd{};
    };
    std::vector<Lv32> lv32;
    std::vector<SweepTma> tma32;
    Arena32 fixed32, state32;
    // V-cycles captured as CUDA graphs, keyed by their arguments and by which
    // buffer holds e on each grid-path level when the cycle starts
    struct VGraph {
        int d;
        bool mix;
        int numcycles, nd, nu, nb;
        std::vector<const void*> e_in, e_out;
        cudaGraphExec_t exec;
        long long launches;
    };
    std::vector<VGraph> graphs;
    cudaStream_t cap = nullptr;   // capture-only stream
    double* d_bcbuf = nullptr;
    double* d_red = nullptr;    // reduction partials + outputs
    double* h_red = nullptr;    // pinned
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // MGP_FLAG_TIME_SMOOTHER: event pairs around the level-0 smoothing calls
    std::vector<cudaEvent_t> tev;
    size_t tev_used = 0;
    long long t_sweeps = 0;
};

namespace {

constexpr int kRedSlots = 2 * kRedBlocksMax + 8;   // two partials per reduction block, then the outputs

void solver_free(mgp_solver* s) {
    if (!s) return;
    // nothing of the solver's may still run when its memory goes back to the
    // pool (its stream may already be gone: a server worker's, say), as
    // cudaFree would have waited for the device
    cudaDeviceSynchronize();
    for (void* p : {(void*)s->d_lv, (void*)s->d_shadow, (void*)s->d_ainv, (void*)s->gm_base, (void*)s->gm_red,
                    (void*)s->gctl.bar, (void*)s->gctl.part, (void*)s->d_ref, (void*)s->d_status,
                    (void*)s->d_bcbuf, (void*)s->d_red})
        dfree(p, nullptr);
    pinned_slots().put(s->h_red);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    for (cudaEvent_t e : s->tev) cudaEventDestroy(e);
    for (auto& g : s->graphs) cudaGraphExecDestroy(g.exec);
    if (s->cap) cudaStreamDestroy(s->cap);
    s->fixed.release();
    s->state.release();
    s->fixed32.release();
    s->state32.release();
    delete s;
}

double* red_partials(mgp_solver* s) { return s->d_red; }
double* red_out(mgp_solver* s) { return s->d_red + 2 * kRedBlocksMax; }

// The mixed-precision V-cycle: MGP_FLAG_MIXED on a vcycle/fmg solver whose
// grid path has at least one level.
bool mixed(const mgp_solver* s) {
    return (s->flags & MGP_FLAG_MIXED) && (s->kind == MGP_KIND_MG || s->kind == MGP_KIND_DD) && s->dc > 0;
}

// Inverse of an n x n matrix (row-major) by Gauss-Jordan elimination with
// partial pivoting; false if a pivot falls below 1e-13 of the largest entry
// (the matrix is singular to working precision).
bool invert_dense(std::vector<double> a, int n, std::vector<double>* inv) {
    std::vector<double>& b = *inv;
    b.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) b[(size_t)i * n + i] = 1.0;
    double amax = 0.0;
    for (double v : a) amax = std::max(amax, std::fabs(v));
    if (!(amax > 0.0)) return false;
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[(size_t)r * n + c]) > std::fabs(a[(size_t)p * n + c])) p = r;
        const double piv = a[(size_t)p * n + c];
        if (!(std::fabs(piv) > 1e-13 * amax)) return false;
        if (p != c)
            for (int k = 0; k < n; ++k) {
                std::swap(a[(size_t)p * n + k], a[(size_t)c * n + k]);
                std::swap(b[(size_t)p * n + k], b[(size_t)c * n + k]);
            }
        const double ip = 1.0 / piv;
        for (int k = 0; k < n; ++k) {
            a[(size_t)c * n + k] *= ip;
            b[(size_t)c * n + k] *= ip;
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = a[(size_t)r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
                b[(size_t)r * n + k] -= f * b[(size_t)c * n + k];
            }
        }
    }
    return true;
}

// MGP_FLAG_DIRECT_LARGE: level dc (at most kDirectLargeCells cells) becomes
// the bottom.  Its operator is assembled as in build_direct_coarse and
// inverted on the device (launch_invert); a pivot below 1e-13 of the largest
// entry keeps the reference bottom, as the host inversion does.
int build_direct_large(mgp_solver* s, cudaStream_t st) {
    const Lv& L = s->lv[s->dc];
    const int n = L.nx * L.ny;
    const size_t sz = (size_t)(L.nx + 2) * (L.ny + 2);
    double *scratch = nullptr, *A = nullptr;
    int* iw = nullptr;
    // scratch: the columns' 2 n fields, later the elimination's 4 n^2 + 2 + (n + 1) kGjPanel doubles
    const size_t ns = std::max(2 * sz * n, 4 * (size_t)n * n + 2 + (size_t)(n + 1) * kGjPanel);
    if (dmalloc(&scratch, sizeof(double) * ns, st) != cudaSuccess ||
        dmalloc(&A, sizeof(double) * n * n, st) != cudaSuccess ||
        dmalloc(&iw, sizeof(int) * (2 * n + 1), st) != cudaSuccess) {
        cudaGetLastError();
        dfree(scratch, st);
        dfree(A, st);
        return set_err(MGP_ENOMEM, "device allocation failed");
    }
    int fail = 1;
    cudaError_t e = launch_direct_columns(L, scratch, A, st);
    if (e == cudaSuccess) e = launch_invert(A, n, A, scratch, iw, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&fail, iw + 2 * n, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    dfree(scratch, st);
    dfree(iw, st);
    if (e != cudaSuccess || fail) {
        dfree(A, st);
        if (e != cudaSuccess) return set_err(MGP_ECUDA, "direct coarse operator: %s", cudaGetErrorString(e));
        return MGP_OK;   // singular to working precision: keep the reference bottom
    }
    s->d_ainv = A;
    s->db = s->dc;
    s->direct_large = true;
    return MGP_OK;
}

// MGP_FLAG_DIRECT_COARSE: the first level from dc down with at most
// kDirectCells cells becomes the bottom, solved with its operator's inverse.
// The operator (homogeneous BCs) is assembled on the device column by column,
// so the inverse is that of the very operator the V-cycle's residuals use.
// Kept only with a Dirichlet side: otherwise the operator is singular.
int build_direct_coarse(mgp_solver* s, cudaStream_t st) {
    bool diri = false;
    for (int k = 0; k < 4; ++k) diri = diri || s->types[k] == MGP_BCTYPE_DIRI;
    if (!diri) return MGP_OK;
    if ((s->flags & MGP_FLAG_DIRECT_LARGE) && (long)s->lv[s->dc].nx * s->lv[s->dc].ny <= kDirectLargeCells &&
        (long)s->lv[s->dc].nx * s->lv[s->dc].ny > kDirectCells)
        return build_direct_large(s, st);
    int db = -1;
    for (int d = s->dc; d <= s->maxdepth; ++d)
        if ((long)s->lv[d].nx * s->lv[d].ny <= kDirectCells) {
            db = d;
            break;
        }
    if (db < 0) return MGP_OK;
    const Lv& L = s->lv[db];
    const int n = L.nx * L.ny;
    const size_t sz = (size_t)(L.nx + 2) * (L.ny + 2);
    double *scratch = nullptr, *A = nullptr;
    if (dmalloc(&scratch, sizeof(double) * 2 * sz * n, st) != cudaSuccess ||
        dmalloc(&A, sizeof(double) * n * n, st) != cudaSuccess) {
        cudaGetLastError();
        dfree(scratch, st);
        return set_err(MGP_ENOMEM, "device allocation failed");
    }
    std::vector<double> h((size_t)n * n), inv;
    cudaError_t e = launch_direct_columns(L, scratch, A, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), A, sizeof(double) * n * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    dfree(scratch, st);
    if (e != cudaSuccess) {
        dfree(A, st);
        return set_err(MGP_ECUDA, "direct coarse operator: %s", cudaGetErrorString(e));
    }
    if (!invert_dense(h, n, &inv)) {   // singular to working precision: keep the reference bottom
        dfree(A, st);
        return MGP_OK;
    }
    for (int k = 0; k < n; ++k)
        for (int m = 0; m < n; ++m) h[(size_t)m * n + k] = inv[(size_t)k * n + m];
    e = cudaMemcpyAsync(A, h.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        dfree(A, st);
        return set_err(MGP_ECUDA, "direct coarse operator: %s", cudaGetErrorString(e));
    }
    s->d_ainv = A;
    s->db = db;
    return MGP_OK;
}

// FP32 copies of the grid-path levels: geometry and inverse diagonals rounded
// from the FP64 hierarchy (built first, so the coarse operators are the FP64
// restrictions), corrections, right-hand sides and work arrays in FP32.
int build_fp32_levels(mgp_solver* s) {
    cudaStream_t st = s->stream;
    s->lv32.assign(s->dc, mgp_solver::Lv32{});
    for (int d = 0; d < s->dc; ++d) {
        const Lv& L = s->lv[d];
        auto& M = s->lv32[d];
        M.nx = L.nx;
        M.ny = L.ny;
        s->fixed32.add(&M.g.J, L.nx, L.ny, 0);
        s->fixed32.add(&M.g.xx, L.nx + 1, L.ny, 0);
        s->fixed32.add(&M.g.xy, L.nx + 1, L.ny, 0);
        s->fixed32.add(&M.g.yx, L.nx, L.ny + 1, 0);
        s->fixed32.add(&M.g.yy, L.nx, L.ny + 1, 0);
        s->fixed32.add(&M.invd, L.nx, L.ny, 0);
        s->state32.add(&M.e, L.nx, L.ny, 1);
        s->state32.add(&M.e2, L.nx, L.ny, 1);
        s->state32.add(&M.r, L.nx, L.ny, 0);
        s->state32.add(&M.w, L.nx, L.ny, 0);
        M.g.dx = L.g.dx;
        M.g.dy = L.g.dy;
        M.g.idx = L.g.idx;
        M.g.idy = L.g.idy;
    }
    RC(s->fixed32.commit(st));
    RC(s->state32.commit(st));
    s->tma32.assign(s->dc, SweepTma{});
    for (int d = 0; d < s->dc; ++d) {
        const Lv& L = s->lv[d];
        auto& M = s->lv32[d];
        CK(launch_convert(M.g.J, L.g.J, L.nx, L.ny, 0, 0, st));
        CK(launch_convert(M.g.xx, L.g.xx, L.nx + 1, L.ny, 0, 0, st));
        CK(launch_convert(M.g.xy, L.g.xy, L.nx + 1, L.ny, 0, 0, st));
        CK(launch_convert(M.g.yx, L.g.yx, L.nx, L.ny + 1, 0, 0, st));
        CK(launch_convert(M.g.yy, L.g.yy, L.nx, L.ny + 1, 0, 0, st));
        CK(launch_convert(M.invd, L.invd, L.nx, L.ny, 0, 0, st));
        if (d >= 1 && (s->flags & MGP_FLAG_BF16_COARSE)) {
            CK(launch_round_bf16(M.g.J, L.nx, L.ny, 0, st));
            CK(launch_round_bf16(M.g.xx, L.nx + 1, L.ny, 0, st));
            CK(launch_round_bf16(M.g.xy, L.nx + 1, L.ny, 0, st));
            CK(launch_round_bf16(M.g.yx, L.nx, L.ny + 1, 0, st));
            CK(launch_round_bf16(M.g.yy, L.nx, L.ny + 1, 0, st));
            CK(launch_round_bf16(M.invd, L.nx, L.ny, 0, st));
        }
        sweep_tma_prepare(&s->tma32[d], M.e, M.e2, M.r, M.invd, M.g, M.nx, M.ny);
    }
    return MGP_OK;
}

// Schedule, allocation, geometry restriction and inverse diagonals:
// MG:432-562 and DD:622-761.
int solver_build(mgp_solver* s, const mgp_box* valid, const mgp_geo* geo, const mgp_bdry* bc, int maxdepth_user) {
    cudaStream_t st = s->stream;
    RC(check_box(valid));
    if (valid->ilo < 0 || valid->jlo < 0 || (valid->ilo % 2) || (valid->jlo % 2))
        return set_err(MGP_EINVAL, "solver: ilo and jlo must be even and non-negative");
    if (valid->nx < 4 || valid->ny < 4) return set_err(MGP_EINVAL, "solver: at least 4 cells per direction");
    if (!geo || !bc) return set_err(MGP_EINVAL, "null geometry or bdry_data");
    RC(check_array(&geo->J, valid->nx, "J"));
    RC(check_array(&geo->Jgup_xx, valid->nx + 1, "Jgup_xx"));
    RC(check_array(&geo->Jgup_xy, valid->nx + 1, "Jgup_xy"));
    RC(check_array(&geo->Jgup_yx, valid->nx, "Jgup_yx"));
    RC(check_array(&geo->Jgup_yy, valid->nx, "Jgup_yy"));
    for (int k = 0; k < 4; ++k) {
        if (bc->type[k] == MGP_BCTYPE_CF) return set_err(MGP_ENOTSUP, "BCTYPE_CF is not supported");
        if (bc->type[k] < MGP_BCTYPE_NONE || bc->type[k] > MGP_BCTYPE_EXTRAP2)
            return set_err(MGP_EINVAL, "invalid BC type");
        s->types[k] = bc->type[k];
    }
    s->valid = *valid;
    int md = maxdepth_user < 0 ? 1000 : maxdepth_user;
    estimate_maxdepth(&md, valid);
    create_mgschedule(s->refx, s->refy, &md, valid);
    if (md >= 32) return set_err(MGP_EINVAL, "multigrid depth %d exceeds 31", md);
    s->maxdepth = md;
    s->lv.assign(md + 1, Lv{});
    // level boxes (coarsen_box, AU:154-170)
    std::vector<mgp_box> boxes(md + 1);
    boxes[0] = *valid;
    for (int d = 1; d <= md; ++d) {
        mgp_box b = boxes[d - 1];
        b.ilo /= s->refx[d - 1]; b.ihi /= s->refx[d - 1]; b.nx = b.ihi - b.ilo + 1; b.dx = b.dx * s->refx[d - 1];
        b.jlo /= s->refy[d - 1]; b.jhi /= s->refy[d - 1]; b.ny = b.jhi - b.jlo + 1; b.dy = b.dy * s->refy[d - 1];
        boxes[d] = b;
    }
    s->dc = md;
    for (int d = 0; d <= md; ++d)
        if ((long)boxes[d].nx * boxes[d].ny <= kCoarseCells) { s->dc = d; break; }
    for (int d = 0; d <= md; ++d) {
        Lv& L = s->lv[d];
        const int nx = boxes[d].nx, ny = boxes[d].ny;
        L.nx = nx;
        L.ny = ny;
        s->fixed.add(&L.g.J, nx, ny, 0);
        s->fixed.add(&L.g.xx, nx + 1, ny, 0);
        s->fixed.add(&L.g.xy, nx + 1, ny, 0);
        s->fixed.add(&L.g.yx, nx, ny + 1, 0);
        s->fixed.add(&L.g.yy, nx, ny + 1, 0);
        s->fixed.add(&L.invd, nx, ny, 0);
        s->state.add(&L.e, nx, ny, 1);
        if (d < s->dc) s->state.add(&L.e2, nx, ny, 1);
        s->state.add(&L.r, nx, ny, 0);
        s->state.add(&L.w, nx, ny, 0);
        if (d == md) {
            s->state.add(&L.ea, nx, ny, 1);
            s->state.add(&L.pt, nx, ny, 1);
            s->state.add(&L.st, nx, ny, 1);
            s->state.add(&L.rr, nx, ny, 0);
            s->state.add(&L.rt, nx, ny, 0);
            s->state.add(&L.pp, nx, ny, 0);
            s->state.add(&L.tt, nx, ny, 0);
            s->state.add(&L.vv, nx, ny, 0);
        }
        L.g.dx = boxes[d].dx;
        L.g.dy = boxes[d].dy;
        L.g.idx = 1.0 / boxes[d].dx;
        L.g.idy = 1.0 / boxes[d].dy;
        for (int k = 0; k < 4; ++k) {
            L.bc.type[k] = bc->type[k];
            L.bc.mode[k] = (s->kind == MGP_KIND_DD) ? MGP_BCMODE_LAH : MGP_BCMODE_UNIFORM;   // MG:516-522, DD:713-719
            L.bc.u[k] = 0.0;
            L.bc.d[k] = nullptr;
        }
    }
    s->state.add(&s->phi0, valid->nx, valid->ny, 1);
    s->state.add(&s->rhs0, valid->nx, valid->ny, 0);
    if ((s->flags & MGP_FLAG_KRYLOV) && s->kind == MGP_KIND_MG)
        for (DF* f : {&s->kr, &s->krh, &s->kp, &s->kv, &s->kt}) s->state.add(f, valid->nx, valid->ny, 0);
    RC(s->fixed.commit(st));
    RC(s->state.commit(st));
    s->h_red = static_cast<double*>(pinned_slots().get());
    static_assert(sizeof(double) * 8 <= kPinnedSlot, "reduction read-back slot");
    if (dmalloc(&s->d_bcbuf, sizeof(double) * 2 * (valid->nx + valid->ny + 2), st) != cudaSuccess ||
        dmalloc(&s->d_red, sizeof(double) * kRedSlots, st) != cudaSuccess ||
        dmalloc(&s->d_lv, sizeof(Lv) * (md + 1), st) != cudaSuccess ||
        dmalloc(&s->d_ref, sizeof(int) * 2 * (md + 1), st) != cudaSuccess ||
        dmalloc(&s->d_status, sizeof(int), st) != cudaSuccess || !s->h_red) {
        cudaGetLastError();
        return set_err(MGP_ENOMEM, "device allocation failed");
    }
    CK(cudaEventCreate(&s->ev0));
    CK(cudaEventCreate(&s->ev1));
    // level-0 geometry is copied (MG:538-545); coarser levels restrict it (MG:550-554)
    Lv& L0 = s->lv[0];
    RC(stage_in(&geo->J, valid->nx, valid->ny, L0.g.J, 0, st));
    RC(stage_in(&geo->Jgup_xx, valid->nx + 1, valid->ny, L0.g.xx, 0, st));
    RC(stage_in(&geo->Jgup_xy, valid->nx + 1, valid->ny, L0.g.xy, 0, st));
    RC(stage_in(&geo->Jgup_yx, valid->nx, valid->ny + 1, L0.g.yx, 0, st));
    RC(stage_in(&geo->Jgup_yy, valid->nx, valid->ny + 1, L0.g.yy, 0, st));
    for (int d = 1; d <= md; ++d) {
        Lv &U = s->lv[d - 1], &L = s->lv[d];
        const int rx = s->refx[d - 1], ry = s->refy[d - 1];
        CK(launch_restrict(U.g.J, L.g.J, L.nx, L.ny, rx, ry, 0, st));
        CK(launch_restrict(U.g.xx, L.g.xx, L.nx, L.ny, rx, ry, 1, st));
        CK(launch_restrict(U.g.xy, L.g.xy, L.nx, L.ny, rx, ry, 1, st));
        CK(launch_restrict(U.g.yx, L.g.yx, L.nx, L.ny, rx, ry, 2, st));
        CK(launch_restrict(U.g.yy, L.g.yy, L.nx, L.ny, rx, ry, 2, st));
    }
    for (int d = 0; d <= md; ++d) {
        Lv& L = s->lv[d];
        if (s->kind == MGP_KIND_DD) CK(launch_dd_invdiag(L.invd, L.g, L.nx, L.ny, st));   // DD:16-39
        else CK(launch_invdiag(L.invd, L.g, L.bc, 1, L.nx, L.ny, (s->flags & MGP_FLAG_DIRICHLET_COUPLED_DIAG) ? 1 : 0,
                               st));                                                      // P2:16-388
    }
    if ((s->flags & MGP_FLAG_DIRECT_COARSE) && s->kind == MGP_KIND_MG) RC(build_direct_coarse(s, st));
    if ((s->flags & MGP_FLAG_GMRES) && s->kind == MGP_KIND_MG) {
        s->gm_ld = (size_t)valid->nx + 2;
        s->gm_vec = s->gm_ld * (valid->ny + 2);
        // m = kGmresRestart unless the 2m + 1 vectors would take more than a
        // quarter of the memory free for solvers (the device's free memory
        // and what the pool keeps); a request of at most 1/16 of the device
        // skips the query
        int m = kGmresRestart;
        const size_t want = (size_t)(2 * m + 1) * s->gm_vec * sizeof(double);
        if (want > device_total_bytes() / 16) {
            size_t freeb = 0, totalb = 0;
            CK(cudaMemGetInfo(&freeb, &totalb));
            freeb += pool_cached_bytes();
            while (m > 8 && (size_t)(2 * m + 1) * s->gm_vec * sizeof(double) > freeb / 4) m /= 2;
        }
        s->gm_m = m;
        if (dmalloc(&s->gm_base, (size_t)(2 * m + 1) * s->gm_vec * sizeof(double), st) != cudaSuccess ||
            dmalloc(&s->gm_red, sizeof(double) * ((size_t)kGmresBlocks * (m + 1) + 2 * (m + 1)), st) !=
                cudaSuccess) {
            cudaGetLastError();
            return set_err(MGP_ENOMEM, "device allocation failed");
        }
    }
    // shared-memory layout of the coarse levels for k_coarse_cycle_smem
    {
        std::vector<Lv> sh(s->lv);
        size_t off = 0;
        auto place = [&](DF& f, int nxv, int nyv, int g) {
            f.ld = nxv + 2 * g;
            f.p = (double*)(uintptr_t)(off + (size_t)g * f.ld + g);
            off += (size_t)f.ld * (nyv + 2 * g);
        };
        for (int d = s->dc; d <= md; ++d) {
            Lv& L = sh[d];
            place(L.e, L.nx, L.ny, 1);
            place(L.r, L.nx, L.ny, 0);
            place(L.w, L.nx, L.ny, 0);
            place(L.invd, L.nx, L.ny, 0);
            place(L.g.J, L.nx, L.ny, 0);
            place(L.g.xx, L.nx + 1, L.ny, 0);
            place(L.g.xy, L.nx + 1, L.ny, 0);
            place(L.g.yx, L.nx, L.ny + 1, 0);
            place(L.g.yy, L.nx, L.ny + 1, 0);
            if (d == md) {
                place(L.ea, L.nx, L.ny, 1);
                place(L.pt, L.nx, L.ny, 1);
                place(L.st, L.nx, L.ny, 1);
                place(L.rr, L.nx, L.ny, 0);
                place(L.rt, L.nx, L.ny, 0);
                place(L.pp, L.nx, L.ny, 0);
                place(L.tt, L.nx, L.ny, 0);
                place(L.vv, L.nx, L.ny, 0);
            }
        }
        const size_t bytes = off * sizeof(double);
        if (md - s->dc + 1 <= kMaxCoarseLevels && bytes <= (size_t)kCoarseSmemMax) {
            if (dmalloc(&s->d_shadow, sizeof(Lv) * (md + 1), st) != cudaSuccess) {
                cudaGetLastError();
                return set_err(MGP_ENOMEM, "device allocation failed");
            }
            CK(cudaMemcpyAsync(s->d_shadow, sh.data(), sizeof(Lv) * (md + 1), cudaMemcpyHostToDevice, st));
            s->shadow_bytes = (int)bytes;
        }
    }
    // Coarse levels that one CTA cannot stage in shared memory: up to
    // kClusterCoarseCells, one thread-block cluster of 16 (or 8) CTAs with
    // hardware barriers; above that, or where no such cluster fits and the
    // level has more than kGridCoarseCells cells, a cooperative grid, one CTA
    // per 256 cells, at most one per SM and at most what the device keeps
    // resident; otherwise one CTA on global memory.
    {
        const int grid_max = coarse_grid_ctas_max();
        const long coarse_cells = (long)s->lv[s->dc].nx * s->lv[s->dc].ny;
        const bool staged = s->shadow_bytes > 0;
        const int cluster_max = !staged && coarse_cells <= kClusterCoarseCells ? coarse_cluster_ctas_max() : 0;
        if (cluster_max > 1) {
            // levels a lockstep batch also serves (one CTA there) keep the
            // one-CTA reduction order, so a problem has the same bits in both
            s->grid_ctas = cluster_max;
            s->coarse_cluster = coarse_cells <= kGridCoarseCells ? 2 : 1;
        } else if (!staged && coarse_cells > kGridCoarseCells && grid_max > 1) {
            int dev = 0, nsm = 0;
            CK(cudaGetDevice(&dev));
            CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
            s->grid_ctas = (int)std::min<long>(std::min(std::max(nsm, 1), grid_max),
                                               std::max<long>(2, coarse_cells / 256));
        }
        if (s->grid_ctas > 1) {
            if (dmalloc(&s->gctl.bar, 2 * sizeof(unsigned), st) != cudaSuccess ||
                dmalloc(&s->gctl.part, 2 * sizeof(double) * s->grid_ctas, st) != cudaSuccess) {
                cudaGetLastError();
                return set_err(MGP_ENOMEM, "device allocation failed");
            }
            s->gctl.status = s->d_status;
            s->gctl.wait_ns = kGridWaitNsDefault;
        }
    }
    s->tma.assign(md + 1, SweepTma{});
    for (int d = 0; d < s->dc; ++d) {
        Lv& L = s->lv[d];
        if (L.e2.p) sweep_tma_prepare(&s->tma[d], L.e, L.e2, L.r, L.invd, L.g, L.nx, L.ny);
    }
    if (mixed(s)) RC(build_fp32_levels(s));
    std::vector<int> ref(2 * (md + 1), 0);
    for (int d = 0; d < md; ++d) { ref[d] = s->refx[d]; ref[md + 1 + d] = s->refy[d]; }
    CK(cudaMemcpyAsync(s->d_lv, s->lv.data(), sizeof(Lv) * (md + 1), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->d_ref, ref.data(), sizeof(int) * 2 * (md + 1), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return MGP_OK;
}

// ---- pieces of vcycle_noinit on the grid-wide kernels -------------------- //
int smooth_body(mgp_solver* s, int d, int nu);

// Level-0 smoothing, bracketed by an event pair when MGP_FLAG_TIME_SMOOTHER is set.
template <class Body>
int timed_smooth(mgp_solver* s, int d, int nu, Body body) {
    const bool timed = (d == 0) && (s->flags & MGP_FLAG_TIME_SMOOTHER) && nu > 0;
    if (!timed) return body();
    if (s->tev_used + 2 > s->tev.size()) {
        for (int k = 0; k < 2; ++k) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            s->tev.push_back(e);
        }
    }
    CK(cudaEventRecord(s->tev[s->tev_used], s->stream));
    RC(body());
    CK(cudaEventRecord(s->tev[s->tev_used + 1], s->stream));
    s->tev_used += 2;
    s->t_sweeps += nu;
    return MGP_OK;
}

int smooth(mgp_solver* s, int d, int nu) {
    return timed_smooth(s, d, nu, [&]() { return smooth_body(s, d, nu); });
}

int smooth_body(mgp_solver* s, int d, int nu) {
    Lv& L = s->lv[d];
    cudaStream_t st = s->stream;
    if (nu <= 0) return MGP_OK;
    if (s->kind == MGP_KIND_DD) {
        CK(launch_dd_modrhs(L.w, L.e, L.r, L.g, L.nx, L.ny, st));   // DD:226-250
        for (int k = 0; k < nu; ++k) {
            CK(launch_fill(L.e, L.g, L.bc, 1, 1, L.nx, L.ny, st));   // DD:259
            CK(launch_dd_colour(L.e, L.w, L.invd, L.g, L.nx, L.ny, 4.0 / 5.0, 0, st));
            CK(launch_dd_colour(L.e, L.w, L.invd, L.g, L.nx, L.ny, 4.0 / 5.0, 1, st));
        }
    } else if (L.e2.p && sweep_fusable(L.bc)) {
        // on small levels two sweeps per launch where the level allows it
        // (the same bits as two launches)
        const bool pairs = sweep_pair_ok(&s->tma[d], L.bc);
        for (int k = 0; k < nu;) {
            if (pairs && nu - k >= 2) {
                CK(launch_sweep9_pair(L.e, L.e2, L.r, L.invd, L.g, L.bc, 1, L.nx, L.ny, 1.0, &s->tma[d], s->d_status,
                                      st));
                k += 2;
            } else {
                CK(launch_sweep9(L.e, L.e2, L.r, L.invd, L.g, L.bc, 1, L.nx, L.ny, 1.0, &s->tma[d], s->d_status,
                                 st));
                k += 1;
            }
            const DF t = L.e;
            L.e = L.e2;
            L.e2 = t;
        }
    } else {
        for (int k = 0; k < nu; ++k) CK(launch_gs_sweep(L.e, L.r, L.invd, L.g, L.bc, 1, L.nx, L.ny, 1.0, st));
    }
    return MGP_OK;
}

int residual_level(mgp_solver* s, int d) {
    Lv& L = s->lv[d];
    cudaStream_t st = s->stream;
    if (s->kind == MGP_KIND_DD) {
        CK(launch_dd_apply(L.w, L.e, L.r, L.g, L.bc, L.nx, L.ny, 1, st));
        CK(launch_fill(L.e, L.g, L.bc, 1, 1, L.nx, L.ny, st));
    } else {
        CK(launch_fill(L.e, L.g, L.bc, 1, 0, L.nx, L.ny, st));
        CK(launch_apply(L.w, L.e, L.r, L.g, L.bc, 1, L.nx, L.ny, 1, 0, st));
    }
    return MGP_OK;
}

// prolong(e(d), e(d+1), ..., order), MG:262-394.
int prolong_level(mgp_solver* s, int d, int order) {
    Lv &F = s->lv[d], &Cl = s->lv[d + 1];
    cudaStream_t st = s->stream;
    const int rx = s->refx[d], ry = s->refy[d];
    CK(launch_fill(Cl.e, Cl.g, Cl.bc, 1, 1, Cl.nx, Cl.ny, st));   // MG:318
    CK(launch_prolong(F.e, Cl.e, Cl.nx, Cl.ny, rx, ry, order, st));
    if (order >= 2 && rx == 2 && ry == 2) {
        CK(launch_extrapolate(Cl.e, Cl.nx, Cl.ny, 1, 1, 3, st));   // MG:354
        CK(launch_prolong_cross(F.e, Cl.e, Cl.nx, Cl.ny, st));
    }
    const bool rax = (Cl.bc.type[0] == T_PERIODIC && Cl.bc.type[1] == T_PERIODIC) ||
                     (Cl.bc.type[0] == T_NEUM && Cl.bc.type[1] == T_NEUM);
    const bool ray = (Cl.bc.type[2] == T_PERIODIC && Cl.bc.type[3] == T_PERIODIC) ||
                     (Cl.bc.type[2] == T_NEUM && Cl.bc.type[3] == T_NEUM);
    if (rax && ray) {
        CK(launch_reduce(RED_JSUM, F.e, F.g.J, F.nx, F.ny, F.g.dx * F.g.dy, red_partials(s), red_out(s), st));
        CK(launch_sub_mean(F.e, red_out(s), F.nx, F.ny, 1, 1, st));
    }
    return MGP_OK;
}

int coarse_cycle(mgp_solver* s, int d, int numcycles, int nd, int nu, int nb) {
    if (s->direct_large && d == s->db) {   // the exact bottom at dc
        const Lv& L = s->lv[d];
        CK(launch_direct_apply(L.e, L.r, s->d_ainv, L.nx, L.ny, s->stream));
        return MGP_OK;
    }
    CoarseArgs a;
    a.lv = s->d_lv;
    a.d0 = d;
    // the exact bottom serves cycles that reach it from above (fmg's cycles
    // that start below it keep the reference bottom)
    const bool direct = s->d_ainv && !s->direct_large && d <= s->db;
    a.maxdepth = direct ? s->db : s->maxdepth;
    a.ainv = direct ? s->d_ainv : nullptr;
    a.numcycles = numcycles;
    a.nd = nd; a.nu = nu; a.nb = nb;
    a.dd = (s->kind == MGP_KIND_DD);
    a.refx = s->d_ref;
    a.refy = s->d_ref + s->maxdepth + 1;
    a.status = s->d_status;
    a.shadow = s->d_shadow;
    a.smem_bytes = s->shadow_bytes;
    a.grid_ctas = s->grid_ctas;
    a.cluster = s->coarse_cluster;
    a.gctl = s->gctl;
    if (a.grid_ctas > 1 && !a.cluster) CK(cudaMemsetAsync(s->gctl.bar, 0, 2 * sizeof(unsigned), s->stream));
    CK(launch_coarse_cycle(a, s->stream));
    return MGP_OK;
}

// vcycle_noinit(depth), MG:675-854 / DD:867-1045.
int vcycle_noinit(mgp_solver* s, int d, int numcycles, int nd, int nu, int nb) {
    if (d >= s->dc) return coarse_cycle(s, d, numcycles, nd, nu, nb);
    Lv &L = s->lv[d], &Cl = s->lv[d + 1];
    cudaStream_t st = s->stream;
    const bool dd = (s->kind == MGP_KIND_DD);
    if (dd) CK(launch_set_guess(L.e, L.r, L.invd, L.nx, L.ny, st));   // DD:971
    RC(smooth(s, d, nd));
    if (dd) {
        RC(residual_level(s, d));
        CK(launch_restrict(L.w, Cl.r, Cl.nx, Cl.ny, s->refx[d], s->refy[d], 0, st));
    } else {   // residual (MG:793-795), restriction and the coarse guess (MG:805-806) in one pass
        CK(launch_fill(L.e, L.g, L.bc, 1, 0, L.nx, L.ny, st));
        CK(launch_resid_restrict(L.e, L.r, L.g, L.bc, 1, L.nx, L.ny, Cl.r, Cl.e, Cl.invd, Cl.nx, Cl.ny, s->refx[d],
                                 s->refy[d], 1, st));
    }
    for (int c = 1; c <= numcycles; ++c) RC(vcycle_noinit(s, d + 1, numcycles, nd, nu, nb));
    RC(prolong_level(s, d, 1));
    RC(smooth(s, d, nu));
    return MGP_OK;
}

// The mixed-precision V-cycle from grid level d < dc: the same schedule and
// kernels as vcycle_noinit on the FP32 copies of the grid-path levels (the 9-
// point sweeps and residual for MG, the DD smoother and residual for DD); the
// restriction into level dc writes the FP64 right-hand side of the coarse
// CTA's levels (which, with the bottom solve, stay FP64) and the prolongation
// from level dc reads its FP64 correction.
int vcycle32(mgp_solver* s, int d, int numcycles, int nd, int nu, int nb) {
    auto& L = s->lv32[d];
    const Lv& F = s->lv[d];   // BCs of the level
    cudaStream_t st = s->stream;
    const bool dd = (s->kind == MGP_KIND_DD);
    // MGP_FLAG_BF16_COARSE: the fields of levels >= 1 take BF16 values each
    // time a kernel writes them to memory
    const bool b16 = (s->flags & MGP_FLAG_BF16_COARSE) != 0;
    auto round16 = [&](const DF32& f, int lvl, int nx_, int ny_, int g) -> cudaError_t {
        return (b16 && lvl >= 1) ? launch_round_bf16(f, nx_, ny_, g, st) : cudaSuccess;
    };
    if (dd) CK(launch_set_guess(L.e, L.r, L.invd, L.nx, L.ny, st));   // DD:971
    auto smooth32 = [&](int nu_) -> int {
        return timed_smooth(s, d, nu_, [&]() -> int {
            if (dd) {
                if (nu_ <= 0) return MGP_OK;
                CK(launch_dd_modrhs(L.w, L.e, L.r, L.g, L.nx, L.ny, st));   // DD:226-250
                for (int k = 0; k < nu_; ++k) {
                    CK(launch_fill(L.e, L.g, F.bc, 1, 1, L.nx, L.ny, st));   // DD:259
                    CK(launch_dd_colour(L.e, L.w, L.invd, L.g, L.nx, L.ny, 4.0 / 5.0, 0, st));
                    CK(launch_dd_colour(L.e, L.w, L.invd, L.g, L.nx, L.ny, 4.0 / 5.0, 1, st));
                    CK(round16(L.e, d, L.nx, L.ny, 1));
                }
                return MGP_OK;
            }
            // on small levels two sweeps per launch where the level allows it
            // (the same bits as two launches; half the launches and loads)
            const bool pairs = sweep_pair_ok(&s->tma32[d], F.bc);
            for (int k = 0; k < nu_;) {
                if (pairs && nu_ - k >= 2) {
                    CK(launch_sweep9_pair(L.e, L.e2, L.r, L.invd, L.g, F.bc, 1, L.nx, L.ny, 1.0, &s->tma32[d],
                                          s->d_status, st));
                    k += 2;
                } else {
                    CK(launch_sweep9(L.e, L.e2, L.r, L.invd, L.g, F.bc, 1, L.nx, L.ny, 1.0, &s->tma32[d],
                                     s->d_status, st));
                    k += 1;
                }
                std::swap(L.e, L.e2);
                CK(round16(L.e, d, L.nx, L.ny, 1));
            }
            return MGP_OK;
        });
    };
    RC(smooth32(nd));
    const int rx = s->refx[d], ry = s->refy[d];
    const bool fine_next = d + 1 < s->dc;
    Lv& C = s->lv[d + 1];
    if (dd) {
        CK(launch_dd_apply(L.w, L.e, L.r, L.g, F.bc, L.nx, L.ny, 1, st));
        CK(launch_fill(L.e, L.g, F.bc, 1, 1, L.nx, L.ny, st));
        if (fine_next) {
            auto& N = s->lv32[d + 1];
            CK(launch_restrict(L.w, N.r, N.nx, N.ny, rx, ry, st));
            CK(round16(N.r, d + 1, N.nx, N.ny, 0));
        } else {
            CK(launch_restrict(L.w, C.r, C.nx, C.ny, rx, ry, st));
        }
    } else {   // residual (MG:793-795), restriction and the coarse guess (MG:805-806) in one pass
        CK(launch_fill(L.e, L.g, F.bc, 1, 0, L.nx, L.ny, st));
        if (fine_next) {
            auto& N = s->lv32[d + 1];
            CK(launch_resid_restrict(L.e, L.r, L.g, F.bc, 1, L.nx, L.ny, N.r, N.e, N.invd, N.nx, N.ny, rx, ry, 1, st));
            CK(round16(N.r, d + 1, N.nx, N.ny, 0));
            CK(round16(N.e, d + 1, N.nx, N.ny, 1));
        } else {
            CK(launch_resid_restrict(L.e, L.r, L.g, F.bc, 1, L.nx, L.ny, C.r, C.e, C.invd, C.nx, C.ny, rx, ry, 1, st));
        }
    }
    if (fine_next) {
        auto& N = s->lv32[d + 1];
        for (int c = 1; c <= numcycles; ++c) RC(vcycle32(s, d + 1, numcycles, nd, nu, nb));
        CK(launch_fill(N.e, N.g, C.bc, 1, 1, N.nx, N.ny, st));    // MG:318
        CK(round16(N.e, d + 1, N.nx, N.ny, 1));
        CK(launch_prolong(L.e, N.e, N.nx, N.ny, rx, ry, 1, st));
        CK(round16(L.e, d, L.nx, L.ny, 1));
    } else {
        for (int c = 1; c <= numcycles; ++c) RC(vcycle_noinit(s, d + 1, numcycles, nd, nu, nb));
        CK(launch_fill(C.e, C.g, C.bc, 1, 1, C.nx, C.ny, st));
        CK(launch_prolong(L.e, C.e, C.nx, C.ny, rx, ry, 1, st));
        CK(round16(L.e, d, L.nx, L.ny, 1));
    }
    const bool rax = (C.bc.type[0] == T_PERIODIC && C.bc.type[1] == T_PERIODIC) ||
                     (C.bc.type[0] == T_NEUM && C.bc.type[1] == T_NEUM);
    const bool ray = (C.bc.type[2] == T_PERIODIC && C.bc.type[3] == T_PERIODIC) ||
                     (C.bc.type[2] == T_NEUM && C.bc.type[3] == T_NEUM);
    if (rax && ray) {   // MG:371-383
        CK(launch_reduce(RED_JSUM, L.e, L.g.J, L.nx, L.ny, L.g.dx * L.g.dy, red_partials(s), red_out(s), st));
        CK(launch_sub_mean(L.e, red_out(s), L.nx, L.ny, 1, 1, st));
        CK(round16(L.e, d, L.nx, L.ny, 1));
    }
    RC(smooth32(nu));
    return MGP_OK;
}

// fmg_noinit(depth), MG:1127-1189.
int fmg_noinit(mgp_solver* s, int d, int numcycles, int nd, int nu, int nb) {
    Lv& L = s->lv[d];
    cudaStream_t st = s->stream;
    CK(launch_fillval(L.e, 0.0, L.nx, L.ny, 1, 1, st));
    if (d < s->maxdepth) {
        Lv& Cl = s->lv[d + 1];
        CK(launch_restrict(L.r, Cl.r, Cl.nx, Cl.ny, s->refx[d], s->refy[d], 0, st));
        RC(fmg_noinit(s, d + 1, numcycles, nd, nu, nb));
        RC(prolong_level(s, d, 2));
    }
    for (int c = 1; c <= numcycles; ++c) RC(vcycle_noinit(s, d, numcycles, nd, nu, nb));
    return MGP_OK;
}

// vcycle_noinit(d) replayed from a CUDA graph: the first call with a given
// key captures the cycle's launches (on a capture-only stream, so nothing
// runs), later calls launch the graph on the solver's stream.  The host-side
// e/e2 buffer swaps the capture made are applied again after every replay.
// Off when the level-0 smoothing is timed with events.
int vcycle_run(mgp_solver* s, int d, int numcycles, int nd, int nu, int nb, bool mix) {
    auto run = [&]() { return mix ? vcycle32(s, d, numcycles, nd, nu, nb) : vcycle_noinit(s, d, numcycles, nd, nu, nb); };
    if ((s->flags & MGP_FLAG_TIME_SMOOTHER) || d >= s->dc) return run();
    // which buffer holds e on each grid-path level
    auto state = [&]() {
        std::vector<const void*> v;
        for (int k = d; k < s->dc; ++k) v.push_back(mix ? (const void*)s->lv32[k].e.p : (const void*)s->lv[k].e.p);
        return v;
    };
    auto set_state = [&](const std::vector<const void*>& v) {
        for (int k = d; k < s->dc; ++k) {
            if (mix) {
                auto& L = s->lv32[k];
                if ((const void*)L.e.p != v[k - d]) std::swap(L.e, L.e2);
            } else {
                Lv& L = s->lv[k];
                if ((const void*)L.e.p != v[k - d]) std::swap(L.e, L.e2);
            }
        }
    };
    const std::vector<const void*> cur = state();
    for (const auto& g : s->graphs) {
        if (g.d == d && g.mix == mix && g.numcycles == numcycles && g.nd == nd && g.nu == nu && g.nb == nb &&
            g.e_in == cur) {
            CK(cudaGraphLaunch(g.exec, s->stream));
            count_launch((int)g.launches);
            set_state(g.e_out);
            return MGP_OK;
        }
    }
    CK(sweep_kernels_init());
    CK(coarse_kernels_init());
    if (!s->cap) CK(cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking));
    const cudaStream_t saved = s->stream;
    const long long l0 = thread_launch_count();   // other threads' solvers may be launching meanwhile
    s->stream = s->cap;
    CK(cudaStreamBeginCapture(s->cap, cudaStreamCaptureModeThreadLocal));
    const int rc = run();
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s->cap, &graph);
    s->stream = saved;
    mgp_solver::VGraph g{d, mix, numcycles, nd, nu, nb, cur, state(), nullptr, thread_launch_count() - l0};
    set_state(cur);   // the capture ran nothing: put the buffers back as they were
    count_launch((int)-g.launches);
    if (rc || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (rc) return rc;
        return set_err(MGP_ECUDA, "V-cycle graph capture failed: %s", cudaGetErrorString(ce));
    }
    const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        cudaGetLastError();
        return set_err(MGP_ECUDA, "V-cycle graph instantiation failed: %s", cudaGetErrorString(ie));
    }
    s->graphs.push_back(g);
    CK(cudaGraphLaunch(g.exec, s->stream));
    count_launch((int)g.launches);
    set_state(g.e_out);
    return MGP_OK;
}

// dst = src over the valid region of level 0.
int copy_valid(const DF& dst, const DF& src, int nx, int ny, cudaStream_t st);

// One V-cycle on level 0 for the right-hand side x (MG:600-606): e = x * invd,
// vcycle_noinit(0); the correction ends in L0.e.  With MGP_FLAG_MIXED the
// cycle runs on the FP32 copies: x is rounded into the FP32 right-hand side
// and the FP32 correction (with its ghosts) is widened into L0.e.
int vcycle_top(mgp_solver* s, const DF& x, int numcycles, int nd, int nu, int nb) {
    Lv& L0 = s->lv[0];
    const int nx = L0.nx, ny = L0.ny;
    cudaStream_t st = s->stream;
    if (!mixed(s)) {
        if (x.p != L0.r.p) RC(copy_valid(L0.r, x, nx, ny, st));
        CK(launch_set_guess(L0.e, L0.r, L0.invd, nx, ny, st));
        return vcycle_run(s, 0, numcycles, nd, nu, nb, false);
    }
    auto& M = s->lv32[0];
    CK(launch_convert(M.r, x, nx, ny, 0, 0, st));
    CK(launch_set_guess(M.e, M.r, M.invd, nx, ny, st));
    RC(vcycle_run(s, 0, numcycles, nd, nu, nb, true));
    CK(launch_convert(L0.e, M.e, nx, ny, 1, 1, st));
    return MGP_OK;
}

// dst = src over the valid region of level 0.
int copy_valid(const DF& dst, const DF& src, int nx, int ny, cudaStream_t st) {
    CK(cudaMemcpy2DAsync(dst.p, dst.ld * sizeof(double), src.p, src.ld * sizeof(double), nx * sizeof(double), ny,
                         cudaMemcpyDeviceToDevice, st));
    return MGP_OK;
}

// Reads reduction slots 0..n-1 back to s->h_red (one copy, one synchronisation).
int fetch_reductions(mgp_solver* s, int n) {
    CK(cudaMemcpyAsync(s->h_red, red_out(s), n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MGP_OK;
}

// MGP_FLAG_KRYLOV: right-preconditioned BiCGStab (van der Vorst, SIAM J. Sci.
// Stat. Comput. 13, 1992) on L_h e = r0, where L_h is the level-0 operator
// with homogeneous BCs and the preconditioner is one V-cycle started from
// e = r * invdiags (the same call the stationary loop makes, MG:600-606).
// Corrections go straight into phi0; kr carries the recursive residual.  When
// it passes the tolerance, the true residual rhs - L[phi] is recomputed with
// the caller's BCs; if that one has not passed, BiCGStab restarts from it.
// On entry L0.r holds r0.  relres[k] is the residual after k V-cycles; the
// last entry is the true residual.
int krylov_loop(mgp_solver* s, const BCd& ubc, int homog, double tol, int maxiters, int numcycles, int nd, int nu,
                int nb, double rscale, std::vector<double>& relres, int* iters_out, int verbosity) {
    Lv& L0 = s->lv[0];   // L0.e moves between two buffers as the fused sweep swaps them
    const int nx = s->valid.nx, ny = s->valid.ny;
    const double vol = s->valid.dx * s->valid.dy;
    cudaStream_t st = s->stream;
    double* out = red_out(s);
    int k = 0;
    // y = M^-1 x in L0.e, then Ay = L_h y
    auto precond_apply = [&](const DF& x, const DF& Ay) -> int {
        RC(vcycle_top(s, x, numcycles, nd, nu, nb));
        CK(launch_fill(L0.e, L0.g, L0.bc, 1, 0, nx, ny, st));
        CK(launch_apply(Ay, L0.e, L0.r, L0.g, L0.bc, 1, nx, ny, 0, 0, st));
        return MGP_OK;
    };
    auto record = [&](double res) -> int {
        relres[k] = res / rscale;
        *iters_out = k;
        if (verbosity >= 1) printf("BiCGStab V-Cycle %d: rel |res| = %.16e\n", k, relres[k]);
        return std::isfinite(relres[k]) ? MGP_OK : MGP_EDIVERGED;
    };
    *iters_out = 0;
    if (relres[0] <= tol) return MGP_OK;
    RC(copy_valid(s->kr, L0.r, nx, ny, st));
    for (;;) {   // one pass per (re)start
        RC(copy_valid(s->krh, s->kr, nx, ny, st));
        RC(copy_valid(s->kp, s->kr, nx, ny, st));
        CK(launch_reduce(RED_DOT, s->krh, s->kr, nx, ny, vol, red_partials(s), out, st));
        RC(fetch_reductions(s, 1));
        double rho = s->h_red[0];
        bool passed = false;
        while (k < maxiters) {
            // first half: alpha, s = r - alpha v
            RC(precond_apply(s->kp, s->kv));
            ++k;
            CK(launch_reduce(RED_DOT, s->krh, s->kv, nx, ny, vol, red_partials(s), out, st));
            RC(fetch_reductions(s, 1));
            const double alpha = rho / s->h_red[0];
            if (!std::isfinite(alpha)) { relres[k] = relres[k - 1]; break; }   // breakdown: restart
            CK(launch_axpby(s->phi0, L0.e, 1.0, alpha, nx, ny, 0, 0, st));
            CK(launch_axpby(s->kr, s->kv, 1.0, -alpha, nx, ny, 0, 0, st));
            CK(launch_reduce(RED_SUMSQ, s->kr, s->kr, nx, ny, vol, red_partials(s), out, st));
            RC(fetch_reductions(s, 1));
            RC(record(s->h_red[0]));
            if (relres[k] <= tol) { passed = true; break; }
            if (k >= maxiters) break;
            // second half: omega, r = s - omega t
            RC(precond_apply(s->kr, s->kt));
            ++k;
            CK(launch_reduce(RED_DOT, s->kt, s->kr, nx, ny, vol, red_partials(s), out, st));
            CK(launch_reduce(RED_DOT, s->kt, s->kt, nx, ny, vol, red_partials(s), out + 1, st));
            RC(fetch_reductions(s, 2));
            const double omega = s->h_red[0] / s->h_red[1];
            if (!std::isfinite(omega) || omega == 0.0) { relres[k] = relres[k - 1]; break; }
            CK(launch_axpby(s->phi0, L0.e, 1.0, omega, nx, ny, 0, 0, st));
            CK(launch_axpby(s->kr, s->kt, 1.0, -omega, nx, ny, 0, 0, st));
            CK(launch_reduce(RED_SUMSQ, s->kr, s->kr, nx, ny, vol, red_partials(s), out, st));
            CK(launch_reduce(RED_DOT, s->krh, s->kr, nx, ny, vol, red_partials(s), out + 1, st));
            RC(fetch_reductions(s, 2));
            RC(record(s->h_red[0]));
            if (relres[k] <= tol) { passed = true; break; }
            const double rho_new = s->h_red[1];
            const double beta = (rho_new / rho) * (alpha / omega);
            if (!std::isfinite(beta) || rho_new == 0.0) break;   // breakdown: restart
            rho = rho_new;
            CK(launch_axpby(s->kp, s->kv, 1.0, -omega, nx, ny, 0, 0, st));   // p = r + beta (p - omega v)
            CK(launch_axpby(s->kp, s->kr, beta, 1.0, nx, ny, 0, 0, st));
        }
        // true residual with the caller's BCs (MG:579)
        CK(launch_fill(s->phi0, L0.g, ubc, homog, 0, nx, ny, st));
        CK(launch_apply(L0.r, s->phi0, s->rhs0, L0.g, ubc, homog, nx, ny, 1, 0, st));
        CK(launch_reduce(RED_SUMSQ, L0.r, L0.r, nx, ny, vol, red_partials(s), out, st));
        RC(fetch_reductions(s, 1));
        RC(record(s->h_red[0]));
        *iters_out = k;
        if ((passed && relres[k] <= tol) || k >= maxiters) return MGP_OK;
        RC(copy_valid(s->kr, L0.r, nx, ny, st));
    }
}

// MGP_FLAG_GMRES: restarted, right-preconditioned GMRES(m) (Saad and Schultz,
// SIAM J. Sci. Stat. Comput. 7, 1986) on L_h e = r0, with L_h and the V-cycle
// preconditioner as in krylov_loop.  Each step: z_j = M^-1 v_j (one V-cycle),
// w = L_h z_j, w orthogonalised against v_0..v_j by one pass of classical
// Gram-Schmidt (the coefficients stay on the device; one host
// synchronisation per step fetches them with |w|), and Givens rotations on
// the host give the residual norm.  At convergence, breakdown or m steps,
// phi0 += Z y and the true residual is recomputed with the caller's BCs;
// the solve restarts from it if it has not passed, so a residual estimate
// that drifted with lost orthogonality ends in a restart, not in a wrong
// answer.  (A second pass, taken whenever |w| fell below half its norm
// before, ran on every step with the V-cycle preconditioner, since
// L_h M^-1 is close to the identity, and left the V-cycle count unchanged.)  Inner products are
// unweighted; the weighted norms of the history differ by sqrt(dx dy).
int gmres_loop(mgp_solver* s, const BCd& ubc, int homog, double tol, int maxiters, int numcycles, int nd, int nu,
               int nb, double rscale, std::vector<double>& relres, int* iters_out, int verbosity) {
    Lv& L0 = s->lv[0];
    const int nx = s->valid.nx, ny = s->valid.ny, m = s->gm_m, ld = (int)s->gm_ld;
    const double vol = s->valid.dx * s->valid.dy, sv = std::sqrt(vol);
    cudaStream_t st = s->stream;
    auto V = [&](int k) { return DF{s->gm_base + (size_t)k * s->gm_vec + ld + 1, ld}; };
    auto Z = [&](int k) { return DF{s->gm_base + (size_t)(m + 1 + k) * s->gm_vec + ld + 1, ld}; };
    const MVec mv{V(0).p, ld, (long)s->gm_vec}, mz{Z(0).p, ld, (long)s->gm_vec};
    double* part = s->gm_red;
    double* h1 = part + (size_t)kGmresBlocks * (m + 1);   // h1[m + 1], |w|^2, then y[m]
    double* nrm = h1 + (m + 1);
    double* dy = nrm + 1;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), hc(m + 2), y(m);
    int k = 0;
    auto record = [&](double res) -> int {
        relres[k] = res / rscale;
        *iters_out = k;
        if (verbosity >= 1) printf("GMRES V-Cycle %d: rel |res| = %.16e\n", k, relres[k]);
        return std::isfinite(relres[k]) ? MGP_OK : MGP_EDIVERGED;
    };
    *iters_out = 0;
    if (relres[0] <= tol) return MGP_OK;
    for (;;) {   // one pass per (re)start; L0.r holds the residual
        CK(launch_mdot(L0.r, MVec{L0.r.p, L0.r.ld, 0}, 1, nx, ny, part, kGmresBlocks, nrm, st));
        CK(cudaMemcpyAsync(hc.data(), nrm, sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const double beta = std::sqrt(hc[0]);
        if (!(beta > 0.0) || !std::isfinite(beta)) return std::isfinite(beta) ? MGP_OK : MGP_EDIVERGED;
        CK(launch_axpby(V(0), L0.r, 0.0, 1.0 / beta, nx, ny, 0, 0, st));
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int jend = 0;
        for (int j = 0; j < m && k < maxiters; ++j) {
            RC(vcycle_top(s, V(j), numcycles, nd, nu, nb));   // M^-1 v_j in L0.e
            CK(launch_axpby(Z(j), L0.e, 0.0, 1.0, nx, ny, 1, 1, st));
            CK(launch_fill(Z(j), L0.g, L0.bc, 1, 0, nx, ny, st));
            CK(launch_apply(V(j + 1), Z(j), L0.r, L0.g, L0.bc, 1, nx, ny, 0, 0, st));
            ++k;
            const cudaError_t gse =
                launch_gs_pass(V(j + 1), mv, j + 1, nx, ny, part, (long)kGmresBlocks * (m + 1), kGmresBlocks, h1, nrm, st);
            if (gse == cudaErrorNotSupported) {   // more blocks of cells than partial sums: a pass per step
                CK(launch_mdot(V(j + 1), mv, j + 1, nx, ny, part, kGmresBlocks, h1, st));
                CK(launch_maxpy(V(j + 1), mv, j + 1, h1, -1.0, nx, ny, st));
                CK(launch_mdot(V(j + 1), MVec{V(j + 1).p, ld, 0}, 1, nx, ny, part, kGmresBlocks, nrm, st));
            } else {
                CK(gse);
            }
            CK(cudaMemcpyAsync(hc.data(), h1, sizeof(double) * (m + 2), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            double* col = &H[(size_t)j * (m + 1)];   // column j of the Hessenberg matrix
            for (int i = 0; i <= j; ++i) col[i] = hc[i];
            const double hn = std::sqrt(hc[m + 1]);
            col[j + 1] = hn;
            for (int i = 0; i < j; ++i) {   // earlier rotations
                const double t = cs[i] * col[i] + sn[i] * col[i + 1];
                col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1];
                col[i] = t;
            }
            const double den = std::hypot(col[j], col[j + 1]);
            cs[j] = den > 0.0 ? col[j] / den : 1.0;
            sn[j] = den > 0.0 ? col[j + 1] / den : 0.0;
            col[j] = den;
            col[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            if (!(den > 0.0)) {   // breakdown: column j is singular and stays out of H y = g; restart
                if (jend == 0) RC(record(beta * sv));   // nothing to add: phi0 and its residual stand
                break;
            }
            jend = j + 1;
            RC(record(std::fabs(g[j + 1]) * sv));
            if (relres[k] <= tol || !(hn > 0.0)) break;   // converged, or the space is exhausted
            CK(launch_axpby(V(j + 1), V(j + 1), 1.0 / hn, 0.0, nx, ny, 0, 0, st));
        }
        if (jend == 0) return MGP_OK;   // maxiters reached before a step
        for (int i = jend - 1; i >= 0; --i) {   // H y = g, upper triangular
            double t = g[i];
            for (int l = i + 1; l < jend; ++l) t -= H[(size_t)l * (m + 1) + i] * y[l];
            y[i] = t / H[(size_t)i * (m + 1) + i];
        }
        CK(cudaMemcpyAsync(dy, y.data(), sizeof(double) * jend, cudaMemcpyHostToDevice, st));
        CK(launch_maxpy(s->phi0, mz, jend, dy, 1.0, nx, ny, st));
        CK(cudaStreamSynchronize(st));   // y's host copy is read by the transfer above
        // true residual with the caller's BCs (MG:579)
        CK(launch_fill(s->phi0, L0.g, ubc, homog, 0, nx, ny, st));
        CK(launch_apply(L0.r, s->phi0, s->rhs0, L0.g, ubc, homog, nx, ny, 1, 0, st));
        CK(launch_reduce(RED_SUMSQ, L0.r, L0.r, nx, ny, vol, red_partials(s), red_out(s), st));
        RC(fetch_reductions(s, 1));
        RC(record(s->h_red[0]));
        if (relres[k] <= tol || k >= maxiters) return MGP_OK;
    }
}

// 0 = vcycle (MG:400-670), 1 = fmg (MG:860-1122), 2 = DD vcycle (DD:589-862)
int solver_solve(mgp_solver* s, int which, mgp_array* phi, mgp_array* rhs, const mgp_bdry* bc, int homog, double tol,
                 int maxiters, int numcycles, int nd, int nu, int nb, int zerophi, int verbosity, mgp_report* rep) {
    const int nx = s->valid.nx, ny = s->valid.ny;
    cudaStream_t st = s->stream;
    if (which == 2 && s->kind != MGP_KIND_DD) return set_err(MGP_EINVAL, "solver was not created for the DD path");
    if (which != 2 && s->kind == MGP_KIND_DD) return set_err(MGP_EINVAL, "solver was created for the DD path");
    if (maxiters < 0 || numcycles < 0 || nd < 0 || nu < 0 || nb < 0) return set_err(MGP_EINVAL, "negative count");
    RC(check_array(phi, nx, "phi"));
    RC(check_array(rhs, nx, "rhs"));
    if (!bc) return set_err(MGP_EINVAL, "null bdry_data");
    for (int k = 0; k < 4; ++k)
        if (bc->type[k] != s->types[k]) return set_err(MGP_EINVAL, "BC types differ from the ones the solver was built with");
    BCd ubc;
    RC(make_bc(bc, &s->valid, homog, s->d_bcbuf, &ubc, st));
    Lv& L0 = s->lv[0];
    const double vol = s->valid.dx * s->valid.dy;
    std::vector<double> relres((size_t)maxiters + 1, 0.0);
    int iters = 0, diverged = 0, status = MGP_OK;
    double rscale = 0.0;

    s->tev_used = 0;
    s->t_sweeps = 0;
    CK(cudaEventRecord(s->ev0, st));
    // every solve starts from fresh (zeroed) work arrays, like the Fortran drivers' allocations
    CK(cudaMemsetAsync(s->state.base, 0, s->state.elems * sizeof(double), st));
    if (s->state32.base) CK(cudaMemsetAsync(s->state32.base, 0, s->state32.elems * sizeof(float), st));
    CK(cudaMemsetAsync(s->d_status, 0, sizeof(int), st));
    RC(stage_in(phi, nx, ny, s->phi0, 1, st));
    RC(stage_in(rhs, nx, ny, s->rhs0, 0, st));
    if (zerophi) CK(launch_fillval(s->phi0, 0.0, nx, ny, 1, 1, st));
    if (which == 2) CK(launch_muldiv(s->rhs0, L0.g.J, 1, nx, ny, st));   // DD:772-773
    // r(0) = rhs - L[phi] with the caller's BCs (MG:579)
    CK(launch_fill(s->phi0, L0.g, ubc, homog, 0, nx, ny, st));
    CK(launch_apply(L0.r, s->phi0, s->rhs0, L0.g, ubc, homog, nx, ny, 1, 0, st));
    CK(launch_reduce(RED_SUMSQ, L0.r, L0.r, nx, ny, vol, red_partials(s), red_out(s), st));
    CK(cudaMemcpyAsync(s->h_red, red_out(s), sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    rscale = s->h_red[0];
    if (rscale == 0.0) { relres[0] = rscale; rscale = 1.0; }
    else relres[0] = 1.0;
    if (verbosity >= 1) printf("max MG depth = %d\nV-Cycle iter 0: rel |res| = %.16e\n", s->maxdepth, relres[0]);
    if (!std::isfinite(rscale)) status = MGP_EDIVERGED;
    const bool gmres = which == 0 && (s->flags & MGP_FLAG_GMRES) && s->gm_base;
    const bool krylov = which == 0 && !gmres && (s->flags & MGP_FLAG_KRYLOV) && s->kr.p;
    if ((krylov || gmres) && status == MGP_OK) {
        const int rc = gmres ? gmres_loop(s, ubc, homog, tol, maxiters, numcycles, nd, nu, nb, rscale, relres, &iters,
                                          verbosity)
                             : krylov_loop(s, ubc, homog, tol, maxiters, numcycles, nd, nu, nb, rscale, relres,
                                           &iters, verbosity);
        if (rc == MGP_EDIVERGED) status = rc;
        else if (rc) return rc;
    }
    for (int iter = 1; !krylov && !gmres && iter <= maxiters && status == MGP_OK; ++iter) {
        if (which == 0) RC(vcycle_top(s, L0.r, numcycles, nd, nu, nb));   // MG:600-606
        else if (which == 1) RC(fmg_noinit(s, 0, numcycles, nd, nu, nb));
        else if (!mixed(s)) RC(vcycle_run(s, 0, numcycles, nd, nu, nb, false));
        else {   // DD with FP32 grid levels: the residual rounded in, the correction widened out
            auto& M = s->lv32[0];
            CK(launch_convert(M.r, L0.r, nx, ny, 0, 0, st));
            RC(vcycle_run(s, 0, numcycles, nd, nu, nb, true));
            CK(launch_convert(L0.e, M.e, nx, ny, 1, 1, st));
        }
        CK(launch_axpby(s->phi0, L0.e, 1.0, 1.0, nx, ny, 1, 1, st));   // MG:611 (whole array)
        CK(launch_fill(s->phi0, L0.g, ubc, homog, 0, nx, ny, st));
        CK(launch_apply(L0.r, s->phi0, s->rhs0, L0.g, ubc, homog, nx, ny, 1, 0, st));
        CK(launch_reduce(RED_SUMSQ, L0.r, L0.r, nx, ny, vol, red_partials(s), red_out(s), st));
        CK(cudaMemcpyAsync(s->h_red, red_out(s), sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        relres[iter] = s->h_red[0] / rscale;
        iters = iter;
        if (verbosity >= 1) printf("V-Cycle iter %d: rel |res| = %.16e\n", iter, relres[iter]);
        if (!std::isfinite(relres[iter])) { status = MGP_EDIVERGED; break; }
        if (relres[iter] <= tol) break;
        if (relres[iter] > relres[iter - 1]) {   // MG:630-639
            CK(launch_axpby(s->phi0, L0.e, 1.0, -1.0, nx, ny, 1, 1, st));
            diverged = 1;
            break;
        }
    }
    int dstat = 0;
    CK(cudaMemcpyAsync(&dstat, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    RC(stage_out(s->phi0, phi, nx, ny, 1, st));
    if (which == 2) {   // DD:837-838
        CK(launch_muldiv(s->rhs0, L0.g.J, 0, nx, ny, st));
        RC(stage_out(s->rhs0, rhs, nx, ny, 0, st));
    }
    CK(cudaEventRecord(s->ev1, st));
    CK(cudaStreamSynchronize(st));
    if (status == MGP_OK && dstat)
        status = (dstat == DST_TIMEOUT) ? MGP_ETIMEOUT : (dstat == DST_MISALIGNED) ? MGP_ECUDA : MGP_EDIVERGED;
    if (status == MGP_OK && (s->flags & MGP_FLAG_REPORT_MAXITER) && !diverged && !(relres[iters] <= tol))
        status = MGP_EMAXITER;
    if (rep) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        rep->status = status;
        rep->iterations = iters;
        rep->maxdepth = s->maxdepth;
        rep->diverged = diverged;
        rep->rscale = rscale;
        rep->final_relres = relres[iters];
        rep->seconds = ms * 1e-3;
        double sm = 0.0;
        for (size_t k = 0; k + 1 < s->tev_used; k += 2) {
            float t = 0.f;
            cudaEventElapsedTime(&t, s->tev[k], s->tev[k + 1]);
            sm += t * 1e-3;
        }
        rep->smooth0_seconds = sm;
        rep->smooth0_sweeps = s->t_sweeps;
        if (rep->relres)
            for (int k = 0; k <= iters; ++k) rep->relres[k] = relres[k];
    }
    if (status == MGP_ETIMEOUT) return set_err(status, "a device wait ran out of its iteration limit");
    if (status == MGP_ECUDA) return set_err(status, "misaligned shared-memory window in the sweep");
    if (status == MGP_EMAXITER) return set_err(status, "maxiters reached before the tolerance");
    if (status) return set_err(status, "non-finite residual");
    return MGP_OK;
}

int solver_new(const mgp_box* valid, const mgp_geo* geo, const mgp_bdry* bc, int kind, int flags, int maxdepth_user,
               cudaStream_t stream, mgp_solver** out) {
    if (!out) return set_err(MGP_EINVAL, "null output pointer");
    *out = nullptr;
    if (kind != MGP_KIND_MG && kind != MGP_KIND_DD) return set_err(MGP_EINVAL, "unknown solver kind");
    mgp_solver* s = new mgp_solver();
    s->kind = kind;
    s->flags = flags;
    s->stream = stream;
    const int rc = solver_build(s, valid, geo, bc, maxdepth_user);
    if (rc) {
        solver_free(s);
        return rc;
    }
    *out = s;
    return MGP_OK;
}

int oneshot(int which, const mgp_box* valid, mgp_array* phi, mgp_array* rhs, const mgp_geo* geo, const mgp_bdry* bc,
            int homog, double tol, int maxiters, int maxdepth_user, int numcycles, int nd, int nu, int nb, int zerophi,
            int verbosity, mgp_report* rep) {
    mgp_solver* s = nullptr;
    RC(solver_new(valid, geo, bc, which == 2 ? MGP_KIND_DD : MGP_KIND_MG, g_flags, maxdepth_user, nullptr, &s));
    const int rc = solver_solve(s, which, phi, rhs, bc, homog, tol, maxiters, numcycles, nd, nu, nb, zerophi, verbosity,
                                rep);
    solver_free(s);
    return rc;
}

// ---------------------------------------------------------------------------
// Operator-level calls: a short-lived context that stages the arguments.
// ---------------------------------------------------------------------------
struct OpCtx {
    std::vector<void*> bufs;
    cudaStream_t st = nullptr;
    ~OpCtx() {
        for (void* p : bufs) cudaFree(p);
    }
    int field(DF* f, int nxv, int nyv, int g) {
        const int ld = ((nxv + 2 * g + 31) / 32) * 32;
        const size_t pad = g ? 32 : 0;
        const size_t n = (size_t)(nyv + 2 * g) * ld + 2 * pad;
        double* p = nullptr;
        if (cudaMalloc(&p, n * 8) != cudaSuccess) {
            cudaGetLastError();
            return set_err(MGP_ENOMEM, "cudaMalloc failed");
        }
        bufs.push_back(p);
        CK(cudaMemsetAsync(p, 0, n * 8, st));
        f->ld = ld;
        f->p = p + pad + (size_t)g * ld;
        return MGP_OK;
    }
    int dbuf(double** p, size_t n) {
        if (cudaMalloc(p, n * 8) != cudaSuccess) {
            cudaGetLastError();
            return set_err(MGP_ENOMEM, "cudaMalloc failed");
        }
        bufs.push_back(*p);
        return MGP_OK;
    }
    int ibuf(int** p) {
        if (cudaMalloc(p, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            return set_err(MGP_ENOMEM, "cudaMalloc failed");
        }
        bufs.push_back(*p);
        CK(cudaMemsetAsync(*p, 0, sizeof(int), st));
        return MGP_OK;
    }
    // Geometry of a level: the five arrays.
    int geo(const mgp_geo* g, const mgp_box* v, Geo* out) {
        if (!g) return set_err(MGP_EINVAL, "null geometry");
        DF J, xx, xy, yx, yy;
        RC(check_array(&g->J, v->nx, "J"));
        RC(check_array(&g->Jgup_xx, v->nx + 1, "Jgup_xx"));
        RC(check_array(&g->Jgup_xy, v->nx + 1, "Jgup_xy"));
        RC(check_array(&g->Jgup_yx, v->nx, "Jgup_yx"));
        RC(check_array(&g->Jgup_yy, v->nx, "Jgup_yy"));
        RC(field(&J, v->nx, v->ny, 0));
        RC(field(&xx, v->nx + 1, v->ny, 0));
        RC(field(&xy, v->nx + 1, v->ny, 0));
        RC(field(&yx, v->nx, v->ny + 1, 0));
        RC(field(&yy, v->nx, v->ny + 1, 0));
        RC(stage_in(&g->J, v->nx, v->ny, J, 0, st));
        RC(stage_in(&g->Jgup_xx, v->nx + 1, v->ny, xx, 0, st));
        RC(stage_in(&g->Jgup_xy, v->nx + 1, v->ny, xy, 0, st));
        RC(stage_in(&g->Jgup_yx, v->nx, v->ny + 1, yx, 0, st));
        RC(stage_in(&g->Jgup_yy, v->nx, v->ny + 1, yy, 0, st));
        *out = make_geo(J, xx, xy, yx, yy, g->dx, g->dy);
        return MGP_OK;
    }
    int in(const mgp_array* a, int nxv, int nyv, int g, DF* f, const char* what) {
        RC(check_array(a, nxv, what));
        RC(field(f, nxv, nyv, g));
        return stage_in(a, nxv, nyv, *f, g, st);
    }
    int bc(const mgp_bdry* b, const mgp_box* v, int homog, BCd* out) {
        double* d = nullptr;
        RC(dbuf(&d, 2 * (size_t)(v->nx + v->ny + 2)));
        return make_bc(b, v, homog, d, out, st);
    }
    int finish() {
        CK(cudaStreamSynchronize(st));
        CK(cudaGetLastError());
        return MGP_OK;
    }
};

int no_lah(const mgp_bdry* bc) {
    for (int k = 0; k < 4; ++k)
        if (bc && bc->mode[k] == MGP_BCMODE_LAH) return set_err(MGP_EINVAL, "Poisson2d::compute_invdiags received BCMODE_LAH.");
    return MGP_OK;
}

int ghost_cap(const mgp_array* a) {
    if (a->ngx > 1 || a->ngy > 1) return set_err(MGP_EINVAL, "fill_ghosts: Can only handle 1 ghost layer max.");
    return MGP_OK;
}

}  // namespace

// Lets other translation units of the library record the message that
// mgp_last_error() returns.
namespace mgp {
int record_error(int code, const char* msg) { return set_err(code, "%s", msg); }

// For the batch and server front ends (mgp_batch.cu): a solver whose set-up
// runs on the given stream, and the device bytes it holds.
int solver_create_on(const mgp_box* valid, const mgp_geo* geo, const mgp_bdry* bc, int kind, int flags,
                     int maxdepth_user, cudaStream_t st, mgp_solver** out) {
    return solver_new(valid, geo, bc, kind, flags, maxdepth_user, st, out);
}
size_t solver_device_bytes(const mgp_solver* s) {
    if (!s) return 0;
    size_t bytes = (s->fixed.elems + s->state.elems) * sizeof(double) +
                   (s->fixed32.elems + s->state32.elems) * sizeof(float) + (size_t)s->shadow_bytes;
    if (s->gm_base) bytes += (size_t)(2 * s->gm_m + 1) * s->gm_vec * sizeof(double);   // GMRES's stored vectors
    if (s->d_ainv && s->db >= 0) {   // the exact bottom's inverse
        const size_t n = (size_t)s->lv[s->db].nx * s->lv[s->db].ny;
        bytes += n * n * sizeof(double);
    }
    return bytes;
}
// Memory the solvers' pool on the current device holds but no solver uses
// (freed, kept for reuse; see solver_pool): free for the next solver.
size_t solver_pool_cached_bytes() { return pool_cached_bytes(); }

// ===========================================================================
// Lockstep batches (mgp_batch_* with MGP_FLAG_LOCKSTEP): the stationary
// V-cycle of MG:565-645 for many resident hierarchies at once.  Every phase of
// the cycle -- a level's smoothing sweeps, its ghost fill, the fused
// residual-restriction, the coarse cycles, the fills and prolongations on the
// way up, the update, the residual norm -- is one launch over the phase's job
// table, one job per unconverged problem (tiles or cell blocks of its level),
// instead of a launch per problem.  Each job does what the single-problem
// kernel does for its cells, so each problem's solution has the bits of its
// own stationary V-cycle; only the residual norms are summed in another (fixed)
// order.  One host synchronisation per V-cycle reads every problem's norm,
// and the job tables are rebuilt when a problem leaves.
// ===========================================================================
struct Lockstep {
    char* dev = nullptr;   // job tables and their block prefixes
    size_t cap = 0;
    double* part = nullptr;   // norm partials, one per cell block
    size_t part_cap = 0;
    double* norms = nullptr;  // per job
    double* vols = nullptr;
    double* h_norms = nullptr;   // pinned
    int ncap = 0;
    int* status = nullptr;    // the sweeps' status word
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // the iteration captured as a CUDA graph for one set of active problems
    // (replayed while that set does not change; re-captured when the set has
    // stayed the same for two iterations in a row)
    cudaStream_t capture = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<int> exec_act;
    long long exec_launches = 0;
};

namespace {

struct Packer {
    std::vector<char> host;
    size_t add(const void* p, size_t bytes) {
        const size_t off = (host.size() + 255) / 256 * 256;
        host.resize(off + bytes);
        if (bytes) std::memcpy(host.data() + off, p, bytes);
        return off;
    }
};

// One launch's jobs: the host copy until upload, then device pointers.
template <class J>
struct Table {
    std::vector<J> jobs;
    std::vector<int> pre{0};
    size_t oj = 0, op = 0;
    const J* dj = nullptr;
    const int* dp = nullptr;
    void push(const J& j, int blocks) {
        jobs.push_back(j);
        pre.push_back(pre.back() + blocks);
    }
    int n() const { return (int)jobs.size(); }
    int blocks() const { return pre.back(); }
    void pack(Packer& pk) {
        oj = pk.add(jobs.data(), jobs.size() * sizeof(J));
        op = pk.add(pre.data(), pre.size() * sizeof(int));
    }
    void bind(char* base) {
        dj = reinterpret_cast<const J*>(base + oj);
        dp = reinterpret_cast<const int*>(base + op);
    }
};

int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

bool fill_one_phase(const BCd& b, int do_neum) {   // no side's fill reads another side's ghosts
    for (int k = 0; k < 4; ++k) {
        const int t = b.type[k];
        if (t == T_DIRI || t == T_NONE || (t == T_NEUM && !do_neum)) continue;
        return false;
    }
    return true;
}

template <class T>
struct SweepGroups {   // a level's sweep jobs by tile width, and those that sweep twice per launch
    Table<SweepJobT<T>> w32, w64, w32k2;
};

template <class T>
void add_sweep_job(SweepGroups<T>& sg, const SweepTma& t, const DFT<T>& e, const DFT<T>& e2, const DFT<T>& r,
                   const DFT<T>& invd, const GeoT<T>& g, const BCd& b, int nx, int ny, bool pairs) {
    SweepJobT<T> J;
    std::memset(&J, 0, sizeof J);
    const bool a_is_e = (const void*)e.p == t.pa;
    const bool k2 = pairs && t.ok2;   // the level's two-sweep descriptors exist
    J.m[0] = k2 ? (a_is_e ? t.ma2 : t.mb2) : (a_is_e ? t.ma : t.mb);
    J.m[1] = k2 ? (a_is_e ? t.mb2 : t.ma2) : (a_is_e ? t.mb : t.ma);
    J.buf[0] = e;
    J.buf[1] = e2;
    J.rhs = r;
    J.invd = invd;
    J.g = g;
    J.b = b;
    J.nx = nx;
    J.ny = ny;
    J.gx = cdiv(nx, t.tx);
    J.gy = cdiv(ny, 32);
    J.part = make_int4(nx / J.gx, nx % J.gx, ny / J.gy, ny % J.gy);
    J.s0 = 0;
    (k2 ? sg.w32k2 : t.tx == 64 ? sg.w64 : sg.w32).push(J, J.gx * J.gy);
}

// Everything one V-cycle iteration launches, for one set of active problems.
struct Plan {
    int D = 0;        // levels with sweeps (max grid-path depth)
    bool mix = false;
    std::vector<SweepGroups<double>> sw64;
    std::vector<SweepGroups<float>> sw32;
    std::vector<Table<FillJob<double>>> fpre64, fpost64;
    std::vector<Table<FillJob<float>>> fpre32, fpost32;
    std::vector<int> fpre_ph, fpost_ph;
    std::vector<Table<ResidJob<double, double>>> res64;
    std::vector<Table<ResidJob<float, float>>> res32;
    std::vector<Table<ResidJob<float, double>>> res3264;
    std::vector<Table<ProlongJob<double, double>>> pro64;
    std::vector<Table<ProlongJob<float, float>>> pro32;
    std::vector<Table<ProlongJob<float, double>>> pro3264;
    Table<CoarseJob> coarse;
    int coarse_smem = 0;
    Table<DirectJob> direct;   // problems whose bottom is the coarse-cycle level, solved by its inverse
    Table<CellJob<float, double>> r_to32;   // mixed: level-0 rhs rounded to FP32
    Table<CellJob<float, float>> guess32;   // e = r invd on FP32 level 0
    Table<CellJob<double, double>> guess64; // e = r invd on FP64 level 0
    Table<CellJob<double, float>> e_to64;   // mixed: the correction widened
    Table<CellJob<double, double>> update;  // phi += e (valid cells and ghosts)
    Table<FillJob<double>> fill_phi;        // caller BCs
    int fill_phi_ph = 1;
    Table<NormJob> norm;
    std::vector<double> vol;
};

CoarseArgs coarse_args_of(mgp_solver* s, int d, int nd, int nu, int nb) {
    CoarseArgs a;
    std::memset(&a, 0, sizeof a);
    a.lv = s->d_lv;
    a.d0 = d;
    const bool direct = s->d_ainv && !s->direct_large && d <= s->db;
    a.maxdepth = direct ? s->db : s->maxdepth;
    a.ainv = direct ? s->d_ainv : nullptr;
    a.numcycles = 1;
    a.nd = nd;
    a.nu = nu;
    a.nb = nb;
    a.dd = 0;
    a.refx = s->d_ref;
    a.refy = s->d_ref + s->maxdepth + 1;
    a.status = s->d_status;
    a.shadow = s->d_shadow;
    a.smem_bytes = s->shadow_bytes;
    a.grid_ctas = 0;
    a.cluster = 0;
    return a;
}

void build_plan(Plan& P, const std::vector<mgp_solver*>& ss, const std::vector<int>& act, const std::vector<BCd>& ubc,
                int homog, int nd, int nu, int nb, bool pairs) {
    P = Plan();
    for (int p : act) P.D = std::max(P.D, ss[p]->dc);
    P.mix = !act.empty() && mixed(ss[act[0]]);
    const int D = P.D;
    P.sw64.resize(D); P.sw32.resize(D);
    P.fpre64.resize(D); P.fpre32.resize(D); P.fpost64.resize(D); P.fpost32.resize(D);
    P.fpre_ph.assign(D, 1); P.fpost_ph.assign(D, 1);
    P.res64.resize(D); P.res32.resize(D); P.res3264.resize(D);
    P.pro64.resize(D); P.pro32.resize(D); P.pro3264.resize(D);
    for (int p : act) {
        mgp_solver* s = ss[p];
        const bool mx = mixed(s);
        for (int d = 0; d < s->dc; ++d) {
            const Lv& F = s->lv[d];
            Lv& C = s->lv[d + 1];
            const int rx = s->refx[d], ry = s->refy[d];
            const bool next_grid = d + 1 < s->dc;
            if (!fill_one_phase(F.bc, 0)) P.fpre_ph[d] = 3;
            if (!fill_one_phase(C.bc, 1)) P.fpost_ph[d] = 3;
            const int fblk = cdiv(2 * (F.nx + F.ny) + 12, 256), cblk = cdiv(2 * (C.nx + C.ny) + 12, 256);
            const int gbx = cdiv(F.nx, 32), gby = cdiv(F.ny, 8);
            const int cbx = cdiv(C.nx, 32), cby = cdiv(C.ny, 8);
            if (mx) {
                auto& L = s->lv32[d];
                add_sweep_job(P.sw32[d], s->tma32[d], L.e, L.e2, L.r, L.invd, L.g, F.bc, L.nx, L.ny, pairs);
                P.fpre32[d].push(FillJob<float>{L.e, L.g, F.bc, L.nx, L.ny, 1, 0}, fblk);
                if (next_grid) {
                    auto& N = s->lv32[d + 1];
                    P.res32[d].push(ResidJob<float, float>{L.e, L.r, L.g, F.bc, N.r, N.e, N.invd, L.nx, L.ny, N.nx, N.ny,
                                                           rx, ry, gbx},
                                    gbx * gby);
                    P.fpost32[d].push(FillJob<float>{N.e, N.g, C.bc, N.nx, N.ny, 1, 1}, cblk);
                    P.pro32[d].push(ProlongJob<float, float>{L.e, N.e, N.nx, N.ny, rx, ry, cbx}, cbx * cby);
                } else {
                    P.res3264[d].push(ResidJob<float, double>{L.e, L.r, L.g, F.bc, C.r, C.e, C.invd, L.nx, L.ny, C.nx,
                                                              C.ny, rx, ry, gbx},
                                      gbx * gby);
                    P.fpost64[d].push(FillJob<double>{C.e, C.g, C.bc, C.nx, C.ny, 1, 1}, cblk);
                    P.pro3264[d].push(ProlongJob<float, double>{L.e, C.e, C.nx, C.ny, rx, ry, cbx}, cbx * cby);
                }
            } else {
                add_sweep_job(P.sw64[d], s->tma[d], F.e, F.e2, F.r, F.invd, F.g, F.bc, F.nx, F.ny, pairs);
                P.fpre64[d].push(FillJob<double>{F.e, F.g, F.bc, F.nx, F.ny, 1, 0}, fblk);
                P.res64[d].push(ResidJob<double, double>{F.e, F.r, F.g, F.bc, C.r, C.e, C.invd, F.nx, F.ny, C.nx, C.ny,
                                                         rx, ry, gbx},
                                gbx * gby);
                P.fpost64[d].push(FillJob<double>{C.e, C.g, C.bc, C.nx, C.ny, 1, 1}, cblk);
                P.pro64[d].push(ProlongJob<double, double>{F.e, C.e, C.nx, C.ny, rx, ry, cbx}, cbx * cby);
            }
        }
        if (s->direct_large && s->db == s->dc) {
            const Lv& B = s->lv[s->dc];
            P.direct.push(DirectJob{B.e, B.r, s->d_ainv, B.nx, B.ny}, direct_apply_blocks(B.nx, B.ny));
        } else {
            CoarseJob cj;
            cj.a = coarse_args_of(s, s->dc, nd, nu, nb);
            P.coarse.push(cj, 1);
            if (s->d_shadow) P.coarse_smem = std::max(P.coarse_smem, s->shadow_bytes);
        }
        const Lv& L0 = s->lv[0];
        const int nx = L0.nx, ny = L0.ny;
        const int bx0 = cdiv(nx, 32), by0 = cdiv(ny, 8), bxg = cdiv(nx + 2, 32), byg = cdiv(ny + 2, 8);
        if (mx) {
            auto& M = s->lv32[0];
            P.r_to32.push(CellJob<float, double>{M.r, L0.r, DF32{}, nx, ny, 0, bx0}, bx0 * by0);
            P.guess32.push(CellJob<float, float>{M.e, M.r, M.invd, nx, ny, 0, bx0}, bx0 * by0);
            P.e_to64.push(CellJob<double, float>{L0.e, M.e, DF{}, nx, ny, 1, bxg}, bxg * byg);
        } else {
            P.guess64.push(CellJob<double, double>{L0.e, L0.r, L0.invd, nx, ny, 0, bx0}, bx0 * by0);
        }
        P.update.push(CellJob<double, double>{s->phi0, L0.e, DF{}, nx, ny, 1, bxg}, bxg * byg);
        if (!fill_one_phase(ubc[p], 0)) P.fill_phi_ph = 3;
        P.fill_phi.push(FillJob<double>{s->phi0, L0.g, ubc[p], nx, ny, homog, 0}, cdiv(2 * (nx + ny) + 12, 256));
        P.norm.push(NormJob{s->phi0, s->rhs0, L0.r, L0.g, ubc[p], nx, ny, homog, bx0}, bx0 * by0);
        P.vol.push_back(s->valid.dx * s->valid.dy);
    }
}

template <class F>
void for_tables(Plan& P, F f) {
    for (auto& g : P.sw64) { f(g.w32); f(g.w64); f(g.w32k2); }
    for (auto& g : P.sw32) { f(g.w32); f(g.w64); f(g.w32k2); }
    for (auto& t : P.fpre64) f(t);
    for (auto& t : P.fpre32) f(t);
    for (auto& t : P.fpost64) f(t);
    for (auto& t : P.fpost32) f(t);
    for (auto& t : P.res64) f(t);
    for (auto& t : P.res32) f(t);
    for (auto& t : P.res3264) f(t);
    for (auto& t : P.pro64) f(t);
    for (auto& t : P.pro32) f(t);
    for (auto& t : P.pro3264) f(t);
    f(P.coarse); f(P.direct); f(P.r_to32); f(P.guess32); f(P.guess64); f(P.e_to64); f(P.update); f(P.fill_phi); f(P.norm);
}

int upload_plan(Plan& P, Lockstep* ls, cudaStream_t st) {
    Packer pk;
    for_tables(P, [&](auto& t) { t.pack(pk); });
    const size_t ov = pk.add(P.vol.data(), P.vol.size() * sizeof(double));
    if (pk.host.size() > ls->cap) {
        CK(cudaStreamSynchronize(st));
        dfree(ls->dev, st);
        ls->dev = nullptr;
        ls->cap = 0;
        const size_t cap = pk.host.size() + pk.host.size() / 2;
        if (dmalloc(&ls->dev, cap, st) != cudaSuccess) {
            cudaGetLastError();
            return set_err(MGP_ENOMEM, "lockstep: device allocation failed");
        }
        ls->cap = cap;
    }
    // the tables the previous iteration's kernels read are no longer in use
    // (the host synchronised on its norms); stream order covers the rest
    CK(cudaMemcpyAsync(ls->dev, pk.host.data(), pk.host.size(), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));   // the pageable source must stay valid until copied
    for_tables(P, [&](auto& t) { t.bind(ls->dev); });
    const size_t nb = (size_t)P.norm.blocks();
    if (nb > ls->part_cap) {
        dfree(ls->part, st);
        ls->part = nullptr;
        ls->part_cap = 0;
        if (dmalloc(&ls->part, nb * sizeof(double), st) != cudaSuccess) {
            cudaGetLastError();
            return set_err(MGP_ENOMEM, "lockstep: device allocation failed");
        }
        ls->part_cap = nb;
    }
    ls->vols = reinterpret_cast<double*>(ls->dev + ov);
    return MGP_OK;
}

// n sweeps of every job of a level (n even; with two-sweep jobs a multiple of
// 4, so every job's correction ends in its first buffer).
template <class T>
int sweeps(SweepGroups<T>& g, int n, Lockstep* ls, cudaStream_t st) {
    for (int k = 0; k < n; ++k) {
        CK(launch_sweep9_jobs<T>(g.w32.dj, g.w32.dp, g.w32.n(), g.w32.blocks(), 32, 1, k & 1, ls->status, st));
        CK(launch_sweep9_jobs<T>(g.w64.dj, g.w64.dp, g.w64.n(), g.w64.blocks(), 64, 1, k & 1, ls->status, st));
    }
    for (int k = 0; k < n / 2; ++k)
        CK(launch_sweep9_jobs<T>(g.w32k2.dj, g.w32k2.dp, g.w32k2.n(), g.w32k2.blocks(), 32, 2, k & 1, ls->status,
                                 st));
    return MGP_OK;
}

// One V-cycle iteration of every problem in the plan: vcycle_top, the cycle, phi += e, the new residual and its norm.
int lockstep_iteration(Plan& P, Lockstep* ls, int nd, int nu, cudaStream_t st) {
    CK(launch_cell_jobs(P.r_to32.dj, P.r_to32.dp, P.r_to32.n(), P.r_to32.blocks(), 1, st));
    CK(launch_cell_jobs(P.guess32.dj, P.guess32.dp, P.guess32.n(), P.guess32.blocks(), 3, st));
    CK(launch_cell_jobs(P.guess64.dj, P.guess64.dp, P.guess64.n(), P.guess64.blocks(), 3, st));
    for (int d = 0; d < P.D; ++d) {   // down: smooth, fill, residual-restriction-guess (MG:784-806)
        RC(sweeps(P.sw64[d], nd, ls, st));
        RC(sweeps(P.sw32[d], nd, ls, st));
        CK(launch_fill_jobs(P.fpre64[d].dj, P.fpre64[d].dp, P.fpre64[d].n(), P.fpre64[d].blocks(), P.fpre_ph[d], st));
        CK(launch_fill_jobs(P.fpre32[d].dj, P.fpre32[d].dp, P.fpre32[d].n(), P.fpre32[d].blocks(), P.fpre_ph[d], st));
        CK(launch_resid_jobs(P.res64[d].dj, P.res64[d].dp, P.res64[d].n(), P.res64[d].blocks(), st));
        CK(launch_resid_jobs(P.res32[d].dj, P.res32[d].dp, P.res32[d].n(), P.res32[d].blocks(), st));
        CK(launch_resid_jobs(P.res3264[d].dj, P.res3264[d].dp, P.res3264[d].n(), P.res3264[d].blocks(), st));
    }
    CK(launch_coarse_jobs(P.coarse.dj, P.coarse.n(), P.coarse_smem, st));
    CK(launch_direct_jobs(P.direct.dj, P.direct.dp, P.direct.n(), P.direct.blocks(), st));
    for (int d = P.D - 1; d >= 0; --d) {   // up: fill the coarse correction, prolong, smooth (MG:818-845)
        CK(launch_fill_jobs(P.fpost64[d].dj, P.fpost64[d].dp, P.fpost64[d].n(), P.fpost64[d].blocks(), P.fpost_ph[d],
                            st));
        CK(launch_fill_jobs(P.fpost32[d].dj, P.fpost32[d].dp, P.fpost32[d].n(), P.fpost32[d].blocks(), P.fpost_ph[d],
                            st));
        CK(launch_prolong_jobs(P.pro64[d].dj, P.pro64[d].dp, P.pro64[d].n(), P.pro64[d].blocks(), st));
        CK(launch_prolong_jobs(P.pro32[d].dj, P.pro32[d].dp, P.pro32[d].n(), P.pro32[d].blocks(), st));
        CK(launch_prolong_jobs(P.pro3264[d].dj, P.pro3264[d].dp, P.pro3264[d].n(), P.pro3264[d].blocks(), st));
        RC(sweeps(P.sw64[d], nu, ls, st));
        RC(sweeps(P.sw32[d], nu, ls, st));
    }
    CK(launch_cell_jobs(P.e_to64.dj, P.e_to64.dp, P.e_to64.n(), P.e_to64.blocks(), 1, st));
    CK(launch_cell_jobs(P.update.dj, P.update.dp, P.update.n(), P.update.blocks(), 0, st));   // MG:611
    CK(launch_fill_jobs(P.fill_phi.dj, P.fill_phi.dp, P.fill_phi.n(), P.fill_phi.blocks(), P.fill_phi_ph, st));
    CK(launch_norm_jobs(P.norm.dj, P.norm.dp, P.norm.n(), P.norm.blocks(), ls->part, ls->vols, ls->norms, st));
    return MGP_OK;
}

}  // namespace

Lockstep* lockstep_new() { return new Lockstep(); }

void lockstep_free(Lockstep* ls) {
    if (!ls) return;
    cudaDeviceSynchronize();
    if (ls->exec) cudaGraphExecDestroy(ls->exec);
    if (ls->capture) cudaStreamDestroy(ls->capture);
    dfree(ls->dev, nullptr);
    dfree(ls->part, nullptr);
    dfree(ls->norms, nullptr);
    dfree(ls->status, nullptr);
    if (ls->h_norms) cudaFreeHost(ls->h_norms);
    if (ls->e0) cudaEventDestroy(ls->e0);
    if (ls->e1) cudaEventDestroy(ls->e1);
    delete ls;
}

// Whether the lockstep path serves these solvers with these counts: the MG
// stationary V-cycle (no Krylov or GMRES flags), one coarse visit per level,
// even smoothing counts (so every phase but the sweeps finds each level's
// correction in its first buffer), every level swept with TMA descriptors, no
// periodic side and a Dirichlet side (no mean removal), bottoms that fit one
// CTA, and one precision for all.
bool lockstep_ok(const std::vector<mgp_solver*>& ss, int numcycles, int nd, int nu) {
    if (ss.empty() || numcycles != 1 || (nd & 1) || (nu & 1) || nd < 0 || nu < 0) return false;
    const bool mx = mixed(ss[0]);
    for (mgp_solver* s : ss) {
        if (s->kind != MGP_KIND_MG || (s->flags & (MGP_FLAG_KRYLOV | MGP_FLAG_GMRES | MGP_FLAG_BF16_COARSE)) ||
            (s->direct_large && s->db != s->dc) || (long)s->lv[s->dc].nx * s->lv[s->dc].ny > kGridCoarseCells ||
            mixed(s) != mx)
            return false;
        bool diri = false;
        for (int k = 0; k < 4; ++k) {
            if (s->types[k] == MGP_BCTYPE_PERIODIC) return false;
            diri = diri || s->types[k] == MGP_BCTYPE_DIRI;
        }
        if (!diri) return false;
        for (int d = 0; d < s->dc; ++d) {
            const SweepTma& t = mx ? s->tma32[d] : s->tma[d];
            if (!t.ok || !s->lv[d].e2.p || !sweep_fusable(s->lv[d].bc)) return false;
        }
    }
    return true;
}

int lockstep_vcycle(const std::vector<mgp_solver*>& ss, Lockstep* ls, mgp_array* phi, mgp_array* rhs,
                    const mgp_bdry* bc, int homog, double tol, int maxiters, int nd, int nu, int nb, int zerophi,
                    mgp_report* reports, cudaStream_t st, int pairs_wanted) {
    const int n = (int)ss.size();
    const bool pairs = pairs_wanted && nd % 4 == 0 && nu % 4 == 0;
    if (maxiters < 0 || nb < 0) return set_err(MGP_EINVAL, "negative count");
    if (ls->ncap < n) {
        dfree(ls->norms, st);
        if (ls->h_norms) cudaFreeHost(ls->h_norms);
        ls->norms = nullptr;
        ls->h_norms = nullptr;
        if (dmalloc(&ls->norms, sizeof(double) * n, st) != cudaSuccess ||
            cudaMallocHost(&ls->h_norms, sizeof(double) * n) != cudaSuccess) {
            cudaGetLastError();
            ls->ncap = 0;
            return set_err(MGP_ENOMEM, "lockstep: allocation failed");
        }
        ls->ncap = n;
    }
    if (!ls->status && dmalloc(&ls->status, sizeof(int), st) != cudaSuccess) {
        cudaGetLastError();
        return set_err(MGP_ENOMEM, "lockstep: allocation failed");
    }
    if (!ls->e0) CK(cudaEventCreate(&ls->e0));
    if (!ls->e1) CK(cudaEventCreate(&ls->e1));
    CK(sweep_kernels_init());
    CK(coarse_kernels_init());
    CK(cudaEventRecord(ls->e0, st));
    CK(cudaMemsetAsync(ls->status, 0, sizeof(int), st));
    std::vector<BCd> ubc(n);
    for (int p = 0; p < n; ++p) {   // solver_solve's set-up, per problem
        mgp_solver* s = ss[p];
        const int nx = s->valid.nx, ny = s->valid.ny;
        RC(check_array(&phi[p], nx, "phi"));
        RC(check_array(&rhs[p], nx, "rhs"));
        for (int k = 0; k < 4; ++k)
            if (bc[p].type[k] != s->types[k]) return set_err(MGP_EINVAL, "BC types differ from the solver's");
        RC(make_bc(&bc[p], &s->valid, homog, s->d_bcbuf, &ubc[p], st));
        CK(cudaMemsetAsync(s->state.base, 0, s->state.elems * sizeof(double), st));
        if (s->state32.base) CK(cudaMemsetAsync(s->state32.base, 0, s->state32.elems * sizeof(float), st));
        CK(cudaMemsetAsync(s->d_status, 0, sizeof(int), st));
        RC(stage_in(&phi[p], nx, ny, s->phi0, 1, st));
        RC(stage_in(&rhs[p], nx, ny, s->rhs0, 0, st));
        if (zerophi) CK(launch_fillval(s->phi0, 0.0, nx, ny, 1, 1, st));
    }
    std::vector<std::vector<double>> hist(n, std::vector<double>((size_t)maxiters + 1, 0.0));
    std::vector<double> rscale(n, 1.0);
    std::vector<int> iters(n, 0), diverged(n, 0), status(n, MGP_OK);
    std::vector<int> act(n);
    for (int p = 0; p < n; ++p) act[p] = p;
    Plan P;
    // r(0) = rhs - L[phi] with the caller's BCs (MG:579) and its norm
    build_plan(P, ss, act, ubc, homog, nd, nu, nb, pairs);
    RC(upload_plan(P, ls, st));
    CK(launch_fill_jobs(P.fill_phi.dj, P.fill_phi.dp, P.fill_phi.n(), P.fill_phi.blocks(), P.fill_phi_ph, st));
    CK(launch_norm_jobs(P.norm.dj, P.norm.dp, P.norm.n(), P.norm.blocks(), ls->part, ls->vols, ls->norms, st));
    CK(cudaMemcpyAsync(ls->h_norms, ls->norms, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<int> next;
    for (int p = 0; p < n; ++p) {
        double r = ls->h_norms[p];
        if (r == 0.0) { hist[p][0] = 0.0; r = 1.0; }
        else hist[p][0] = 1.0;
        rscale[p] = r;
        if (!std::isfinite(r)) status[p] = MGP_EDIVERGED;
        else if (hist[p][0] > tol && maxiters > 0) next.push_back(p);
    }
    act.swap(next);
    std::vector<int> prev;
    if (ls->exec) {   // a graph of an earlier call holds that call's tables and BC values
        cudaGraphExecDestroy(ls->exec);
        ls->exec = nullptr;
        ls->exec_act.clear();
    }
    for (int iter = 1; iter <= maxiters && !act.empty(); ++iter) {
        if (ls->exec && act == ls->exec_act) {   // the same problems as the captured iteration
            CK(cudaGraphLaunch(ls->exec, st));
            count_launch((int)ls->exec_launches);
        } else {
            if (ls->exec) {
                cudaGraphExecDestroy(ls->exec);
                ls->exec = nullptr;
                ls->exec_act.clear();
            }
            build_plan(P, ss, act, ubc, homog, nd, nu, nb, pairs);
            RC(upload_plan(P, ls, st));
            if (act == prev) {   // the set held for an iteration: capture it for the ones to come
                if (!ls->capture) CK(cudaStreamCreateWithFlags(&ls->capture, cudaStreamNonBlocking));
                const long long l0 = thread_launch_count();
                CK(cudaStreamBeginCapture(ls->capture, cudaStreamCaptureModeThreadLocal));
                const int rc = lockstep_iteration(P, ls, nd, nu, ls->capture);
                cudaGraph_t graph = nullptr;
                const cudaError_t ce = cudaStreamEndCapture(ls->capture, &graph);
                const long long nl = thread_launch_count() - l0;
                count_launch((int)-nl);
                cudaGraphExec_t ex = nullptr;
                if (!rc && ce == cudaSuccess && cudaGraphInstantiate(&ex, graph, 0) == cudaSuccess) {
                    ls->exec = ex;
                    ls->exec_act = act;
                    ls->exec_launches = nl;
                }
                if (graph) cudaGraphDestroy(graph);
                cudaGetLastError();
                if (rc) return rc;
            }
            if (ls->exec) {
                CK(cudaGraphLaunch(ls->exec, st));
                count_launch((int)ls->exec_launches);
            } else {
                RC(lockstep_iteration(P, ls, nd, nu, st));
            }
        }
        prev = act;
        CK(cudaMemcpyAsync(ls->h_norms, ls->norms, sizeof(double) * act.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        next.clear();
        std::vector<int> undo;
        for (size_t k = 0; k < act.size(); ++k) {
            const int p = act[k];
            const double rr = ls->h_norms[k] / rscale[p];
            hist[p][iter] = rr;
            iters[p] = iter;
            if (!std::isfinite(rr)) { status[p] = MGP_EDIVERGED; continue; }
            if (rr <= tol) continue;
            if (rr > hist[p][iter - 1]) {   // MG:630-639: undo the correction and stop
                diverged[p] = 1;
                undo.push_back(p);
                continue;
            }
            next.push_back(p);
        }
        if (!undo.empty()) {
            Table<CellJob<double, double>> t;
            for (int p : undo) {
                mgp_solver* s = ss[p];
                const int nx = s->valid.nx, ny = s->valid.ny, bx = cdiv(nx + 2, 32), by = cdiv(ny + 2, 8);
                t.push(CellJob<double, double>{s->phi0, s->lv[0].e, DF{}, nx, ny, 1, bx}, bx * by);
            }
            Packer pk;
            t.pack(pk);
            CK(cudaMemcpyAsync(ls->dev, pk.host.data(), pk.host.size(), cudaMemcpyHostToDevice, st));
            t.bind(ls->dev);
            CK(launch_cell_jobs(t.dj, t.dp, t.n(), t.blocks(), 2, st));
            CK(cudaStreamSynchronize(st));
        }
        act.swap(next);
    }
    for (int p = 0; p < n; ++p) RC(stage_out(ss[p]->phi0, &phi[p], ss[p]->valid.nx, ss[p]->valid.ny, 1, st));
    CK(cudaEventRecord(ls->e1, st));
    CK(cudaStreamSynchronize(st));
    int sweep_status = 0;
    CK(cudaMemcpy(&sweep_status, ls->status, sizeof(int), cudaMemcpyDeviceToHost));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ls->e0, ls->e1);
    int first = MGP_OK;
    for (int p = 0; p < n; ++p) {
        int dstat = 0;
        CK(cudaMemcpy(&dstat, ss[p]->d_status, sizeof(int), cudaMemcpyDeviceToHost));
        if (!dstat) dstat = sweep_status;
        if (status[p] == MGP_OK && dstat)
            status[p] = (dstat == DST_TIMEOUT) ? MGP_ETIMEOUT : (dstat == DST_MISALIGNED) ? MGP_ECUDA : MGP_EDIVERGED;
        if (status[p] == MGP_OK && (ss[p]->flags & MGP_FLAG_REPORT_MAXITER) && !diverged[p] &&
            !(hist[p][iters[p]] <= tol))
            status[p] = MGP_EMAXITER;
        if (reports) {
            mgp_report& r = reports[p];
            double* dst = r.relres;
            std::memset(&r, 0, sizeof r);
            r.relres = dst;
            r.status = status[p];
            r.iterations = iters[p];
            r.maxdepth = ss[p]->maxdepth;
            r.diverged = diverged[p];
            r.rscale = rscale[p];
            r.final_relres = hist[p][iters[p]];
            r.seconds = ms * 1e-3;
            if (dst)
                for (int k = 0; k <= iters[p]; ++k) dst[k] = hist[p][k];
        }
        if (status[p] && !first) first = status[p];
    }
    if (first == MGP_ETIMEOUT) return set_err(first, "a device wait ran out of its iteration limit");
    if (first == MGP_ECUDA) return set_err(first, "misaligned shared-memory window in the sweep");
    if (first == MGP_EMAXITER) return set_err(first, "maxiters reached before the tolerance");
    if (first) return set_err(first, "non-finite residual");
    return MGP_OK;
}
}  // namespace mgp

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* mgp_version(void) { return "mgp2d-b200 0.1 (sm_100a, FP64)"; }
const char* mgp_last_error(void) { return g_err.c_str(); }
long long mgp_kernel_launch_count(void) { return launch_count(); }

int mgp_selftest_grid_barrier(int nctas, int skip_cta, int nbarriers, double wait_s, double* seconds) {
    if (nctas < 2 || nbarriers < 1 || nbarriers > (1 << 20) || !(wait_s > 0.0) || wait_s > 10.0 ||
        skip_cta >= nctas)
        return set_err(MGP_EINVAL, "selftest_grid_barrier: bad argument");
    const int cap = barrier_selftest_ctas_max();
    if (cap < 2) return set_err(MGP_ENOTSUP, "selftest_grid_barrier: no cooperative launch on this device");
    if (nctas > cap) return set_err(MGP_EINVAL, "selftest_grid_barrier: more CTAs than the device keeps resident");
    GridCtl g{};
    unsigned* bar = nullptr;
    int* status = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = MGP_OK, dstat = 0;
    if (cudaMalloc(&bar, 2 * sizeof(unsigned)) != cudaSuccess || cudaMalloc(&status, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        rc = set_err(MGP_ENOMEM, "cudaMalloc failed");
    }
    float ms = 0.f;
    if (!rc) {
        g.bar = bar;
        g.status = status;
        g.wait_ns = (unsigned long long)(wait_s * 1e9);
        if (cudaMemset(bar, 0, 2 * sizeof(unsigned)) != cudaSuccess || cudaMemset(status, 0, sizeof(int)) != cudaSuccess ||
            cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
            cudaEventRecord(e0, 0) != cudaSuccess || launch_barrier_selftest(g, nctas, skip_cta, nbarriers, 0) != cudaSuccess ||
            cudaEventRecord(e1, 0) != cudaSuccess || cudaMemcpy(&dstat, status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = set_err(MGP_ECUDA, cudaGetErrorString(cudaGetLastError()));
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (bar) cudaFree(bar);
    if (status) cudaFree(status);
    if (seconds) *seconds = ms * 1e-3;
    if (rc) return rc;
    if (dstat == DST_TIMEOUT) return set_err(MGP_ETIMEOUT, "a grid barrier wait ran out of its limit");
    if (dstat) return set_err(MGP_ECUDA, "unexpected device status");
    return MGP_OK;
}

int mgp_set_flags(int flags) {
    const int old = g_flags;
    g_flags = flags;
    return old;
}

int mgp_estimate_maxdepth(int* maxdepth, const mgp_box* valid) {
    if (!maxdepth || !valid) return set_err(MGP_EINVAL, "null argument");
    estimate_maxdepth(maxdepth, valid);
    return MGP_OK;
}

int mgp_create_mgschedule(int* refx, int* refy, int* maxdepth, const mgp_box* valid) {
    if (!refx || !refy || !maxdepth || !valid) return set_err(MGP_EINVAL, "null argument");
    std::vector<int> rx, ry;
    const int in = *maxdepth;
    create_mgschedule(rx, ry, maxdepth, valid);
    for (int d = 0; d < in; ++d) {
        refx[d] = rx[d];
        refy[d] = ry[d];
    }
    return MGP_OK;
}

int mgp_fill_ghosts(const mgp_box* valid, mgp_array* phi, const mgp_bdry* bc, const mgp_geo* geo, int homog,
                    int do_neum) {
    RC(check_box(valid));
    RC(check_array(phi, valid->nx, "phi"));
    RC(ghost_cap(phi));
    OpCtx c;
    DF p;
    Geo g;
    BCd b;
    RC(c.in(phi, valid->nx, valid->ny, 1, &p, "phi"));
    RC(c.geo(geo, valid, &g));
    RC(c.bc(bc, valid, homog, &b));
    CK(launch_fill(p, g, b, homog, do_neum, valid->nx, valid->ny, c.st));
    RC(stage_out(p, phi, valid->nx, valid->ny, 1, c.st));
    return c.finish();
}

int mgp_extrapolate_ghosts(const mgp_box* valid, mgp_array* phi, int order) {
    RC(check_box(valid));
    RC(check_array(phi, valid->nx, "phi"));
    RC(ghost_cap(phi));
    if (order < 0 || order > 3) return set_err(MGP_EINVAL, "extrapolate_ghosts: order is not supported");
    OpCtx c;
    DF p;
    RC(c.in(phi, valid->nx, valid->ny, 1, &p, "phi"));
    CK(launch_extrapolate(p, valid->nx, valid->ny, phi->ngx, phi->ngy, order, c.st));
    RC(stage_out(p, phi, valid->nx, valid->ny, 1, c.st));
    return c.finish();
}

int mgp_compute_invdiags(const mgp_box* valid, mgp_array* invdiags, const mgp_geo* geo, const mgp_bdry* bc,
                         int homog) {
    RC(check_box(valid));
    RC(no_lah(bc));
    RC(check_array(invdiags, valid->nx, "invdiags"));
    OpCtx c;
    DF d;
    Geo g;
    BCd b;
    RC(c.field(&d, valid->nx, valid->ny, 0));
    RC(c.geo(geo, valid, &g));
    RC(c.bc(bc, valid, homog, &b));
    CK(launch_invdiag(d, g, b, homog, valid->nx, valid->ny, (g_flags & MGP_FLAG_DIRICHLET_COUPLED_DIAG) ? 1 : 0, c.st));
    RC(stage_out(d, invdiags, valid->nx, valid->ny, 0, c.st));
    return c.finish();
}

int mgp_compute_laplacian(const mgp_box* valid, mgp_array* lap, mgp_array* phi, const mgp_geo* geo,
                          const mgp_bdry* bc, int homog, int jscale) {
    RC(check_box(valid));
    RC(no_lah(bc));
    RC(check_array(lap, valid->nx, "lap"));
    RC(check_array(phi, valid->nx, "phi"));
    RC(ghost_cap(phi));
    OpCtx c;
    DF l, p;
    Geo g;
    BCd b;
    RC(c.field(&l, valid->nx, valid->ny, 0));
    RC(c.in(phi, valid->nx, valid->ny, 1, &p, "phi"));
    RC(c.geo(geo, valid, &g));
    RC(c.bc(bc, valid, homog, &b));
    CK(launch_fill(p, g, b, homog, 0, valid->nx, valid->ny, c.st));
    CK(launch_apply(l, p, l, g, b, homog, valid->nx, valid->ny, 0, jscale, c.st));
    RC(stage_out(l, lap, valid->nx, valid->ny, 0, c.st));
    RC(stage_out(p, phi, valid->nx, valid->ny, 1, c.st));
    return c.finish();
}

int mgp_compute_pd(const mgp_box* valid, mgp_array* pd, const mgp_array* phi, int dir, int nodedir) {
    RC(check_box(valid));
    if ((dir != 1 && dir != 2) || (nodedir != 1 && nodedir != 2))
        return set_err(MGP_EINVAL, "compute_pd: direction and nodal direction must be 1 or 2");
    const int nx = valid->nx, ny = valid->ny, fx = nx + (nodedir == 1), fy = ny + (nodedir == 2);
    RC(check_array(pd, fx, "pd"));
    RC(check_array(phi, nx, "phi"));
    RC(ghost_cap(phi));
    if (dir == nodedir && ((dir == 1 && phi->ngx < 1) || (dir == 2 && phi->ngy < 1)))
        return set_err(MGP_EINVAL, "compute_pd: the nodal derivative needs a ghost layer");
    OpCtx c;
    DF d, p;
    RC(c.field(&d, fx, fy, 0));
    RC(c.in(phi, nx, ny, 1, &p, "phi"));
    CK(launch_pd(d, p, nx, ny, valid->dx, valid->dy, dir, nodedir, c.st));
    RC(stage_out(d, pd, fx, fy, 0, c.st));
    return c.finish();
}

int mgp_compute_grad(const mgp_box* valid, mgp_array* xflux, mgp_array* yflux, mgp_array* phi, const mgp_geo* geo,
                     const mgp_bdry* bc, int homog) {
    RC(check_box(valid));
    const int nx = valid->nx, ny = valid->ny;
    RC(check_array(xflux, nx + 1, "xflux"));
    RC(check_array(yflux, nx, "yflux"));
    RC(check_array(phi, nx, "phi"));
    RC(ghost_cap(phi));
    if (phi->ngx < 1 || phi->ngy < 1) return set_err(MGP_EINVAL, "compute_grad: phi needs a ghost layer");
    OpCtx c;
    DF x, y, p;
    Geo g;
    BCd b;
    RC(c.field(&x, nx + 1, ny, 0));
    RC(c.field(&y, nx, ny + 1, 0));
    RC(c.in(phi, nx, ny, 1, &p, "phi"));
    RC(c.geo(geo, valid, &g));
    RC(c.bc(bc, valid, homog, &b));
    CK(launch_fill(p, g, b, homog, 0, nx, ny, c.st));   // P2:828
    CK(launch_grad(x, y, p, g, b, homog, nx, ny, c.st));
    RC(stage_out(x, xflux, nx + 1, ny, 0, c.st));
    RC(stage_out(y, yflux, nx, ny + 1, 0, c.st));
    RC(stage_out(p, phi, nx, ny, 1, c.st));
    return c.finish();
}

int mgp_fill_boundary_fluxes(const mgp_box* valid, mgp_array* xflux, mgp_array* yflux, const mgp_bdry* bc,
                             int homog) {
    RC(check_box(valid));
    const int nx = valid->nx, ny = valid->ny;
    OpCtx c;
    DF x, y;
    BCd b;
    RC(c.in(xflux, nx + 1, ny, 0, &x, "xflux"));
    RC(c.in(yflux, nx, ny + 1, 0, &y, "yflux"));
    RC(c.bc(bc, valid, homog, &b));
    CK(launch_boundary_fluxes(x, y, b, homog, nx, ny, c.st));
    RC(stage_out(x, xflux, nx + 1, ny, 0, c.st));
    RC(stage_out(y, yflux, nx, ny + 1, 0, c.st));
    return c.finish();
}

int mgp_compute_div(const mgp_box* valid, mgp_array* div, const mgp_array* xflux, const mgp_array* yflux) {
    RC(check_box(valid));
    const int nx = valid->nx, ny = valid->ny;
    RC(check_array(div, nx, "div"));
    OpCtx c;
    DF d, x, y;
    RC(c.field(&d, nx, ny, 0));
    RC(c.in(xflux, nx + 1, ny, 0, &x, "xflux"));
    RC(c.in(yflux, nx, ny + 1, 0, &y, "yflux"));
    CK(launch_div(d, x, y, nx, ny, valid->dx, valid->dy, c.st));
    RC(stage_out(d, div, nx, ny, 0, c.st));
    return c.finish();
}

int mgp_compute_residual(const mgp_box* valid, mgp_array* res, const mgp_array* rhs, mgp_array* phi,
                         const mgp_geo* geo, const mgp_bdry* bc, int homog, int jscale) {
    RC(check_box(valid));
    RC(no_lah(bc));
    RC(check_array(res, valid->nx, "res"));
    RC(check_array(phi, valid->nx, "phi"));
    RC(ghost_cap(phi));
    OpCtx c;
    DF r, f, p;
    Geo g;
    BCd b;
    RC(c.field(&r, valid->nx, valid->ny, 0));
    RC(c.in(rhs, valid->nx, valid->ny, 0, &f, "rhs"));
    RC(c.in(phi, valid->nx, valid->ny, 1, &p, "phi"));
    RC(c.geo(geo, valid, &g));
    RC(c.bc(bc, valid, homog, &b));
    CK(launch_fill(p, g, b, homog, 0, valid->nx, valid->ny, c.st));
    CK(launch_apply(r, p, f, g, b, homog, valid->nx, valid->ny, 1, jscale, c.st));
    RC(stage_out(r, res, valid->nx, valid->ny, 0, c.st));
    RC(stage_out(p, phi, valid->nx, valid->ny, 1, c.st));
    return c.finish();
}

int mgp_relax_jacobi(const mgp_box* valid, mgp_array* phi, const mgp_array* rhs, const mgp_geo* geo,
                     const mgp_bdry* bc, int homog, const mgp_array* invdiags, double omega, double tol, int maxiters,
                     int zerophi, int verbosity) {
    RC(check_box(valid));
    RC(no_lah(bc));
    RC(check_array(phi, valid->nx, "phi"));
    RC(ghost_cap(phi));
    if (maxiters == 0) return MGP_OK;
    const int nx = valid->nx, ny = valid->ny;
    OpCtx c;
    DF p, f, d, r;
    Geo g;
    BCd b;
    double* red = nullptr;
    RC(c.in(phi, nx, ny, 1, &p, "phi"));
    RC(c.in(rhs, nx, ny, 0, &f, "rhs"));
    RC(c.in(invdiags, nx, ny, 0, &d, "invdiags"));
    RC(c.field(&r, nx, ny, 0));
    RC(c.dbuf(&red, kRedSlots));
    RC(c.geo(geo, valid, &g));
    RC(c.bc(bc, valid, homog, &b));
    if (zerophi) CK(launch_fillval(p, 0.0, nx, ny, 1, 1, c.st));
    const double vol = valid->dx * valid->dy;
    double rscale = 1.0, h = 0.0;
    auto residual = [&]() -> int {   // compute_residual (P2:1327-1353)
        CK(launch_fill(p, g, b, homog, 0, nx, ny, c.st));
        CK(launch_apply(r, p, f, g, b, homog, nx, ny, 1, 0, c.st));
        return MGP_OK;
    };
    auto norm = [&](double* out) -> int {
        CK(launch_reduce(RED_SUMSQ, r, r, nx, ny, vol, red, red + 2 * kRedBlocksMax, c.st));
        CK(cudaMemcpyAsync(out, red + 2 * kRedBlocksMax, 8, cudaMemcpyDeviceToHost, c.st));
        CK(cudaStreamSynchronize(c.st));
        return MGP_OK;
    };
    RC(residual());
    if (tol > 0.0) {
        RC(norm(&rscale));
        if (rscale == 0.0) rscale = 1.0;
    }
    for (int it = 1; it <= maxiters; ++it) {
        CK(launch_jacobi(p, r, d, omega, nx, ny, c.st));   // P2:1419-1424
        RC(residual());
        if (tol > 0.0) {
            RC(norm(&h));
            if (verbosity >= 3) printf("iter %d: rel |res| = %.16e\n", it, h / rscale);
            if (h / rscale <= tol) break;
        }
    }
    RC(stage_out(p, phi, nx, ny, 1, c.st));
    return c.finish();
}

int mgp_relax_gs(const mgp_box* valid, mgp_array* phi, const mgp_array* rhs, const mgp_geo* geo, const mgp_bdry* bc,
                 int homog, const mgp_array* invdiags, double omega, double tol, int maxiters, int zerophi,
                 int verbosity) {
    RC(check_box(valid));
    RC(no_lah(bc));
    RC(check_array(phi, valid->nx, "phi"));
    RC(ghost_cap(phi));
    if (maxiters == 0) return MGP_OK;
    if (valid->nx < 4 || valid->ny < 4)
        return set_err(MGP_EINVAL, "relax_gs: the device sweep needs at least 4 cells per direction");
    const int nx = valid->nx, ny = valid->ny;
    OpCtx c;
    DF p, p2, f, d, r;
    Geo g;
    BCd b;
    double* red = nullptr;
    RC(c.field(&p2, nx, ny, 1));
    RC(c.in(phi, nx, ny, 1, &p, "phi"));
    RC(c.in(rhs, nx, ny, 0, &f, "rhs"));
    RC(c.in(invdiags, nx, ny, 0, &d, "invdiags"));
    RC(c.field(&r, nx, ny, 0));
    RC(c.dbuf(&red, kRedSlots));
    RC(c.geo(geo, valid, &g));
    RC(c.bc(bc, valid, homog, &b));
    if (zerophi) CK(launch_fillval(p, 0.0, nx, ny, 1, 1, c.st));
    const double vol = valid->dx * valid->dy;
    double rscale = 1.0, h = 0.0;
    auto resnorm = [&](double* out) -> int {
        CK(launch_fill(p, g, b, homog, 0, nx, ny, c.st));
        CK(launch_apply(r, p, f, g, b, homog, nx, ny, 1, 0, c.st));
        CK(launch_reduce(RED_SUMSQ, r, r, nx, ny, vol, red, red + 2 * kRedBlocksMax, c.st));
        CK(cudaMemcpyAsync(out, red + 2 * kRedBlocksMax, 8, cudaMemcpyDeviceToHost, c.st));
        CK(cudaStreamSynchronize(c.st));
        return MGP_OK;
    };
    if (tol > 0.0) {
        RC(resnorm(&rscale));
        if (rscale == 0.0) rscale = 1.0;
    }
    const bool fused = sweep_fusable(b);
    for (int it = 1; it <= maxiters; ++it) {
        if (fused) {
            CK(launch_sweep9(p, p2, f, d, g, b, homog, nx, ny, omega, nullptr, nullptr, c.st));
            const DF t = p;
            p = p2;
            p2 = t;
        } else {
            CK(launch_gs_sweep(p, f, d, g, b, homog, nx, ny, omega, c.st));
        }
        if (tol > 0.0) {
            RC(resnorm(&h));
            if (verbosity >= 3) printf("iter %d: rel |res| = %.16e\n", it, h / rscale);
            if (h / rscale <= tol) break;
        }
    }
    RC(stage_out(p, phi, nx, ny, 1, c.st));
    return c.finish();
}

int mgp_solve_bicgstab2(const mgp_box* valid, mgp_array* phi, const mgp_array* rhs, const mgp_geo* geo,
                        const mgp_bdry* bc, int homog, const mgp_array* invdiags, double tol, int max_iters,
                        int max_restarts, int zerophi, int verbosity) {
    (void)verbosity;
    RC(check_box(valid));
    RC(no_lah(bc));
    RC(check_array(phi, valid->nx, "phi"));
    RC(ghost_cap(phi));
    if (valid->nx < 4 || valid->ny < 4)
        return set_err(MGP_EINVAL, "solve_bicgstab2: the device sweep needs at least 4 cells per direction");
    const int nx = valid->nx, ny = valid->ny;
    OpCtx c;
    BicgArgs a;
    std::memset(&a, 0, sizeof a);
    Lv& L = a.L;
    L.nx = nx;
    L.ny = ny;
    RC(c.in(phi, nx, ny, 1, &a.phi, "phi"));
    RC(c.in(rhs, nx, ny, 0, &a.rhs, "rhs"));
    RC(c.in(invdiags, nx, ny, 0, &L.invd, "invdiags"));
    RC(c.geo(geo, valid, &L.g));
    RC(c.bc(bc, valid, homog, &L.bc));
    RC(c.field(&L.w, nx, ny, 0));
    RC(c.field(&L.ea, nx, ny, 1));
    RC(c.field(&L.pt, nx, ny, 1));
    RC(c.field(&L.st, nx, ny, 1));
    RC(c.field(&L.rr, nx, ny, 0));
    RC(c.field(&L.rt, nx, ny, 0));
    RC(c.field(&L.pp, nx, ny, 0));
    RC(c.field(&L.tt, nx, ny, 0));
    RC(c.field(&L.vv, nx, ny, 0));
    RC(c.ibuf(&a.status));
    a.homog = homog;
    a.tol = tol;
    a.max_iters = max_iters;
    a.max_restarts = max_restarts;
    a.zerophi = zerophi;
    a.dd = 0;
    CK(launch_bicgstab(a, c.st));
    RC(stage_out(a.phi, phi, nx, ny, 1, c.st));
    int dstat = 0;
    CK(cudaMemcpyAsync(&dstat, a.status, sizeof(int), cudaMemcpyDeviceToHost, c.st));
    RC(c.finish());
    if (dstat) return set_err(MGP_EDIVERGED, "solve_bicgstab2: non-finite residual");
    return MGP_OK;
}

int mgp_restrict(const mgp_box* fine_valid, const mgp_array* fine, const mgp_box* crse_valid, mgp_array* crse,
                 int offi, int offj) {
    RC(check_box(fine_valid));
    if (!crse_valid) return set_err(MGP_EINVAL, "null box");
    if (crse_valid->nx < 1 || crse_valid->ny < 1) return set_err(MGP_EINVAL, "empty coarse box");
    const int rx = fine_valid->nx / crse_valid->nx, ry = fine_valid->ny / crse_valid->ny;
    if (rx < 1 || ry < 1 || rx * crse_valid->nx != fine_valid->nx || ry * crse_valid->ny != fine_valid->ny)
        return set_err(MGP_EINVAL, "restrict: boxes are not refinements of each other");
    const int kind = (offi == 1 && offj == 1) ? 0 : (offi == 0 && offj == 1) ? 1 : (offi == 1 && offj == 0) ? 2 : 3;
    const int fx = fine_valid->nx + (offi == 0), fy = fine_valid->ny + (offj == 0);
    const int cx = crse_valid->nx + (offi == 0), cy = crse_valid->ny + (offj == 0);
    OpCtx c;
    DF f, cr;
    RC(c.in(fine, fx, fy, 0, &f, "fine"));
    RC(check_array(crse, cx, "crse"));
    const int cg = (crse->ngx > 0 || crse->ngy > 0) ? 1 : 0;
    RC(c.field(&cr, cx, cy, cg));   // crse%data = zero (ghosts included)
    CK(launch_restrict(f, cr, crse_valid->nx, crse_valid->ny, rx, ry, kind, c.st));
    RC(stage_out(cr, crse, cx, cy, cg, c.st));
    return c.finish();
}

int mgp_prolong(const mgp_box* fine_valid, mgp_array* fine, const mgp_box* crse_valid, mgp_array* crse,
                const mgp_geo* fine_geo, const mgp_geo* crse_geo, const mgp_bdry* crse_bc, int order) {
    RC(check_box(fine_valid));
    RC(check_box(crse_valid));
    if (!fine_geo || !crse_geo) return set_err(MGP_EINVAL, "null geometry");
    if (fine_geo->dx * fine_geo->dy > crse_geo->dx * crse_geo->dy)
        return set_err(MGP_EINVAL, "prolong: crse and fine geos passed in wrong order");
    const int rx = fine_valid->nx / crse_valid->nx, ry = fine_valid->ny / crse_valid->ny;
    if (!((rx == 1 || rx == 2) && (ry == 1 || ry == 2) && rx * ry > 1) || rx * crse_valid->nx != fine_valid->nx ||
        ry * crse_valid->ny != fine_valid->ny)
        return set_err(MGP_ENOTSUP, "prolong: Needs updatin'");
    RC(ghost_cap(crse));
    OpCtx c;
    DF f, cr;
    Geo fg, cg;
    BCd b;
    RC(c.in(fine, fine_valid->nx, fine_valid->ny, 1, &f, "fine"));
    RC(c.in(crse, crse_valid->nx, crse_valid->ny, 1, &cr, "crse"));
    RC(c.geo(fine_geo, fine_valid, &fg));
    RC(c.geo(crse_geo, crse_valid, &cg));
    RC(c.bc(crse_bc, crse_valid, 1, &b));
    double* red = nullptr;
    RC(c.dbuf(&red, kRedSlots));
    if (order >= 1) CK(launch_fill(cr, cg, b, 1, 1, crse_valid->nx, crse_valid->ny, c.st));
    CK(launch_prolong(f, cr, crse_valid->nx, crse_valid->ny, rx, ry, order, c.st));
    if (order >= 2 && rx == 2 && ry == 2) {
        CK(launch_extrapolate(cr, crse_valid->nx, crse_valid->ny, crse->ngx, crse->ngy, 3, c.st));
        CK(launch_prolong_cross(f, cr, crse_valid->nx, crse_valid->ny, c.st));
    }
    const bool rax = (b.type[0] == T_PERIODIC && b.type[1] == T_PERIODIC) || (b.type[0] == T_NEUM && b.type[1] == T_NEUM);
    const bool ray = (b.type[2] == T_PERIODIC && b.type[3] == T_PERIODIC) || (b.type[2] == T_NEUM && b.type[3] == T_NEUM);
    if (rax && ray) {
        const int gx = fine->ngx > 0 ? 1 : 0, gy = fine->ngy > 0 ? 1 : 0;
        CK(launch_reduce(RED_JSUM, f, fg.J, fine_valid->nx, fine_valid->ny, fine_geo->dx * fine_geo->dy, red,
                         red + 2 * kRedBlocksMax, c.st));
        CK(launch_sub_mean(f, red + 2 * kRedBlocksMax, fine_valid->nx, fine_valid->ny, gx, gy, c.st));
    }
    RC(stage_out(f, fine, fine_valid->nx, fine_valid->ny, 1, c.st));
    RC(stage_out(cr, crse, crse_valid->nx, crse_valid->ny, 1, c.st));
    return c.finish();
}

int mgp_pnorm(const mgp_box* valid, const mgp_array* bd, int p, double* out) {
    RC(check_box(valid));
    if (!out) return set_err(MGP_EINVAL, "null output");
    if (p != 0 && p != 1 && p != 2) return set_err(MGP_ENOTSUP, "pnorm: p must be 0, 1 or 2");
    OpCtx c;
    DF a;
    double* red = nullptr;
    RC(c.in(bd, valid->nx, valid->ny, 0, &a, "bd"));
    RC(c.dbuf(&red, kRedSlots));
    const int kind = p == 0 ? RED_MAXABS : p == 1 ? RED_ABSSUM : RED_SUMSQ;
    CK(launch_reduce(kind, a, a, valid->nx, valid->ny, valid->dx * valid->dy, red, red + 2 * kRedBlocksMax, c.st));
    CK(cudaMemcpyAsync(out, red + 2 * kRedBlocksMax, 8, cudaMemcpyDeviceToHost, c.st));
    return c.finish();
}

int mgp_inner_prod(const mgp_box* valid, const mgp_array* a, const mgp_array* b, double* out) {
    RC(check_box(valid));
    if (!out) return set_err(MGP_EINVAL, "null output");
    OpCtx c;
    DF x, y;
    double* red = nullptr;
    RC(c.in(a, valid->nx, valid->ny, 0, &x, "a"));
    RC(c.in(b, valid->nx, valid->ny, 0, &y, "b"));
    RC(c.dbuf(&red, kRedSlots));
    CK(launch_reduce(RED_DOT, x, y, valid->nx, valid->ny, valid->dx * valid->dy, red, red + 2 * kRedBlocksMax, c.st));
    CK(cudaMemcpyAsync(out, red + 2 * kRedBlocksMax, 8, cudaMemcpyDeviceToHost, c.st));
    return c.finish();
}

int mgp_vcycle(const mgp_box* valid, mgp_array* phi, mgp_array* rhs, const mgp_geo* geo, const mgp_bdry* bc, int homog,
               int amrrefx, int amrrefy, double tol, int maxiters, int maxdepth_user, int numcycles, int smooth_down,
               int smooth_up, int smooth_bottom, int zerophi, int verbosity, mgp_report* report) {
    (void)amrrefx;
    (void)amrrefy;   // unused by the Fortran driver too (MG:409)
    return oneshot(0, valid, phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles, smooth_down, smooth_up,
                   smooth_bottom, zerophi, verbosity, report);
}

int mgp_fmg(const mgp_box* valid, mgp_array* phi, mgp_array* rhs, const mgp_geo* geo, const mgp_bdry* bc, int homog,
            int amrrefx, int amrrefy, double tol, int maxiters, int maxdepth_user, int numcycles, int smooth_down,
            int smooth_up, int smooth_bottom, int zerophi, int verbosity, mgp_report* report) {
    (void)amrrefx;
    (void)amrrefy;
    return oneshot(1, valid, phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles, smooth_down, smooth_up,
                   smooth_bottom, zerophi, verbosity, report);
}

int mgp_dc_vcycle(const mgp_box* valid, mgp_array* phi, mgp_array* rhs, const mgp_geo* geo, const mgp_bdry* bc,
                  int homog, int amrrefx, int amrrefy, double tol, int maxiters, int maxdepth_user, int numcycles,
                  int smooth_down, int smooth_up, int smooth_bottom, int zerophi, int verbosity, mgp_report* report) {
    (void)amrrefx;
    (void)amrrefy;
    return oneshot(2, valid, phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles, smooth_down, smooth_up,
                   smooth_bottom, zerophi, verbosity, report);
}

int mgp_solver_create(const mgp_box* valid, const mgp_geo* geo, const mgp_bdry* bc, int kind, int flags,
                      int maxdepth_user, mgp_solver** out) {
    return solver_new(valid, geo, bc, kind, flags, maxdepth_user, nullptr, out);
}

int mgp_solver_destroy(mgp_solver* s) {
    solver_free(s);
    return MGP_OK;
}

int mgp_solver_set_stream(mgp_solver* s, void* stream) {
    if (!s) return set_err(MGP_EINVAL, "null solver");
    s->stream = (cudaStream_t)stream;
    return MGP_OK;
}

int mgp_solver_maxdepth(const mgp_solver* s, int* maxdepth) {
    if (!s || !maxdepth) return set_err(MGP_EINVAL, "null argument");
    *maxdepth = s->maxdepth;
    return MGP_OK;
}

int mgp_solver_vcycle(mgp_solver* s, mgp_array* phi, mgp_array* rhs, const mgp_bdry* bc, int homog, double tol,
                      int maxiters, int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
                      int verbosity, mgp_report* report) {
    if (!s) return set_err(MGP_EINVAL, "null solver");
    return solver_solve(s, 0, phi, rhs, bc, homog, tol, maxiters, numcycles, smooth_down, smooth_up, smooth_bottom,
                        zerophi, verbosity, report);
}

int mgp_solver_fmg(mgp_solver* s, mgp_array* phi, mgp_array* rhs, const mgp_bdry* bc, int homog, double tol,
                   int maxiters, int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
                   int verbosity, mgp_report* report) {
    if (!s) return set_err(MGP_EINVAL, "null solver");
    return solver_solve(s, 1, phi, rhs, bc, homog, tol, maxiters, numcycles, smooth_down, smooth_up, smooth_bottom,
                        zerophi, verbosity, report);
}

int mgp_solver_dc_vcycle(mgp_solver* s, mgp_array* phi, mgp_array* rhs, const mgp_bdry* bc, int homog, double tol,
                         int maxiters, int numcycles, int smooth_down, int smooth_up, int smooth_bottom, int zerophi,
                         int verbosity, mgp_report* report) {
    if (!s) return set_err(MGP_EINVAL, "null solver");
    return solver_solve(s, 2, phi, rhs, bc, homog, tol, maxiters, numcycles, smooth_down, smooth_up, smooth_bottom,
                        zerophi, verbosity, report);
}

}  // extern "C"
