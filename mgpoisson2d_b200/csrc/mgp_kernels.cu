// mgp_kernels.cu -- CUDA kernels of the B200 multigrid solver (sm_100a).
//
// Three execution shapes:
//  * grid kernels, one thread per cell, for the large levels (FP64, and FP32
//    for the grid levels of the mixed-precision V-cycle);
//  * one 256-thread CTA that runs a whole coarse sub-V-cycle, bottom solve
//    included (vcycle_noinit from a given depth down, MG:675-854 and
//    DD:867-1045), so the latency-bound small levels cost one launch;
//  * the same sub-cycle as a cooperative grid of CTAs when the coarsest
//    level is too large for one CTA (the schedule stopped at an odd side).
// All call the same cell functions of mgp_core.cuh, so the FP64 ones produce
// the same bits as each other and as the Fortran loop bodies.
#include <atomic>

#include <mutex>
#include <utility>

#include <cuda_bf16.h>

#include "mgp_kernels.cuh"

namespace mgp {

static std::atomic<long long> g_launches{0};
thread_local long long t_launches = 0;   // this thread's launches (a capture counts its own)
long long launch_count() { return g_launches.load(); }
long long thread_launch_count() { return t_launches; }
void count_launch(int n) {
    g_launches += n;
    t_launches += n;
}

static inline dim3 cells_grid(int nx, int ny, dim3 blk) {
    return dim3((unsigned)((nx + blk.x - 1) / blk.x), (unsigned)((ny + blk.y - 1) / blk.y));
}
static const dim3 kBlk2(32, 8);
constexpr int kBlk2N = 256;   // threads of a kBlk2 block (a power of two: the per-block reduction trees)

// Programmatic dependent launch for the V-cycle's small kernels (the sweeps
// do the same in mgp_sweep.cu): launched with the programmatic serialization
// attribute, a kernel may be scheduled while the kernel ahead of it in the
// stream is still running; pdl_wait() at its start returns once that kernel
// has completed and its writes are visible (at once when nothing is
// pending), before this kernel reads or writes anything that kernel may
// touch, so the semantics are those of plain stream order and the gain is
// the launch and scheduling latency.  pdl_allow() lets the next kernel be
// scheduled in turn.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_allow() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... KArgs, class... Args>
static cudaError_t launch_dep(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

#define CELL_IJ                                              \
    const int i = blockIdx.x * blockDim.x + threadIdx.x;   \
    const int j = blockIdx.y * blockDim.y + threadIdx.y;

// ---------------------------------------------------------------------------
// Ghost fill (fill_ghosts, AU:1277-1492)
// ---------------------------------------------------------------------------
// phase 0: x sides, 1: y sides, 2: corners, 3: all four sides and corners at once
// (used when no side's fill reads another side's ghosts).
template <class T>
__global__ void k_fill(DFT<T> p, GeoT<T> g, BCd b, int homog, int do_neum, int nx, int ny, int phase) {
    pdl_wait();
    pdl_allow();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int lo[4], cnt[4];
    for (int s = 0; s < 4; ++s) side_range(b, s, nx, ny, do_neum, lo[s], cnt[s]);
    int k = t;
    const int s0 = (phase == 1) ? 2 : 0, s1 = (phase == 0) ? 2 : 4;
    if (phase != 2) {
        for (int s = s0; s < s1; ++s) {
            if (k < cnt[s]) { fill_side_elem(p, g, b, homog, s, nx, ny, lo[s] + k); return; }
            k -= cnt[s];
        }
    }
    if (phase >= 2 && k < 4) fill_corner(p, b, nx, ny, k);
}

// The three phases of k_fill (x sides, y sides, corners) in one CTA, a
// barrier between them: the same element operations in the same phase order.
constexpr int kFill3Threads = 1024;
template <class T>
__global__ void __launch_bounds__(kFill3Threads) k_fill3(DFT<T> p, GeoT<T> g, BCd b, int homog, int do_neum, int nx,
                                                          int ny) {
    pdl_wait();
    pdl_allow();
    int lo[4], cnt[4];
    for (int s = 0; s < 4; ++s) side_range(b, s, nx, ny, do_neum, lo[s], cnt[s]);
    for (int ph = 0; ph < 2; ++ph) {
        const int s0 = 2 * ph, n = cnt[s0] + cnt[s0 + 1];
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            if (k < cnt[s0]) fill_side_elem(p, g, b, homog, s0, nx, ny, lo[s0] + k);
            else fill_side_elem(p, g, b, homog, s0 + 1, nx, ny, lo[s0 + 1] + k - cnt[s0]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) fill_corner(p, b, nx, ny, threadIdx.x);
}

static bool fill_single_phase(const BCd& b, int do_neum) {
    for (int s = 0; s < 4; ++s) {
        const int t = b.type[s];
        if (t == T_DIRI || t == T_NONE) continue;
        if (t == T_NEUM && !do_neum) continue;
        return false;
    }
    return true;
}

template <class T>
cudaError_t fill_impl(const DFT<T>& p, const GeoT<T>& g, const BCd& b, int homog, int do_neum, int nx, int ny,
                      cudaStream_t st) {
    const int n = 2 * (nx + ny) + 12;
    const int blk = 256, grd = (n + blk - 1) / blk;
    cudaError_t e = cudaSuccess;
    if (fill_single_phase(b, do_neum)) {
        e = launch_dep(k_fill<T>, dim3(grd), dim3(blk), 0, st, p, g, b, homog, do_neum, nx, ny, 3);
        count_launch();
    } else if (n <= 8 * kFill3Threads) {
        e = launch_dep(k_fill3<T>, dim3(1), dim3(kFill3Threads), 0, st, p, g, b, homog, do_neum, nx, ny);
        count_launch();
    } else {
        for (int ph = 0; ph < 3 && e == cudaSuccess; ++ph)
            e = launch_dep(k_fill<T>, dim3(grd), dim3(blk), 0, st, p, g, b, homog, do_neum, nx, ny, ph);
        count_launch(3);
    }
    return e;
}
cudaError_t launch_fill(const DF& p, const Geo& g, const BCd& b, int homog, int do_neum, int nx, int ny,
                        cudaStream_t st) {
    return fill_impl(p, g, b, homog, do_neum, nx, ny, st);
}
cudaError_t launch_fill(const DF32& p, const Geo32& g, const BCd& b, int homog, int do_neum, int nx, int ny,
                        cudaStream_t st) {
    return fill_impl(p, g, b, homog, do_neum, nx, ny, st);
}

// extrapolate_ghosts (AU:1497-1566): x columns over the whole j range of the
// allocation, then y rows over the whole i range.
__global__ void k_extrap(DF p, int nx, int ny, int ngx, int ngy, int order, int phase) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (phase == 0) {
        const int a = t - ngy;
        if (a > ny - 1 + ngy) return;
        const double l3 = nx > 3 ? AT(p, 3, a) : 0.0, h3 = nx > 3 ? AT(p, nx - 4, a) : 0.0;
        const double vl = extrap_val(order, AT(p, 0, a), AT(p, 1, a), AT(p, 2, a), l3);
        const double vh = extrap_val(order, AT(p, nx - 1, a), AT(p, nx - 2, a), AT(p, nx - 3, a), h3);
        AT(p, -1, a) = vl;
        AT(p, nx, a) = vh;
    } else {
        const int a = t - ngx;
        if (a > nx - 1 + ngx) return;
        const double l3 = ny > 3 ? AT(p, a, 3) : 0.0, h3 = ny > 3 ? AT(p, a, ny - 4) : 0.0;
        const double vl = extrap_val(order, AT(p, a, 0), AT(p, a, 1), AT(p, a, 2), l3);
        const double vh = extrap_val(order, AT(p, a, ny - 1), AT(p, a, ny - 2), AT(p, a, ny - 3), h3);
        AT(p, a, -1) = vl;
        AT(p, a, ny) = vh;
    }
}

cudaError_t launch_extrapolate(const DF& p, int nx, int ny, int ngx, int ngy, int order, cudaStream_t st) {
    if (ngx > 0) {
        const int n = ny + 2 * ngy;
        k_extrap<<<(n + 255) / 256, 256, 0, st>>>(p, nx, ny, ngx, ngy, order, 0);
        count_launch();
    }
    if (ngy > 0) {
        const int n = nx + 2 * ngx;
        k_extrap<<<(n + 255) / 256, 256, 0, st>>>(p, nx, ny, ngx, ngy, order, 1);
        count_launch();
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Operator apply / residual (compute_laplacian P2:886-1319, compute_residual P2:1327-1353)
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_apply(DFT<T> out, DFT<T> phi, DFT<T> rhs, GeoT<T> g, BCd b, int homog, int nx, int ny, int mode,
                        int jscale) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    T lap = apply9(phi, g, b, homog, nx, ny, i, j);
    if (jscale) lap = lap / AT(g.J, i, j);
    AT(out, i, j) = mode ? AT(rhs, i, j) - lap : lap;
}

cudaError_t launch_apply(const DF& out, const DF& phi, const DF& rhs, const Geo& g, const BCd& b, int homog,
                         int nx, int ny, int mode, int jscale, cudaStream_t st) {
    k_apply<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(out, phi, rhs, g, b, homog, nx, ny, mode, jscale);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_apply(const DF32& out, const DF32& phi, const DF32& rhs, const Geo32& g, const BCd& b, int homog,
                         int nx, int ny, int mode, int jscale, cudaStream_t st) {
    k_apply<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(out, phi, rhs, g, b, homog, nx, ny, mode, jscale);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Gradient and divergence (compute_pd P2:404-795, compute_grad P2:809-850,
// compute_div P2:860-879, fill_boundary_fluxes AU:1574-1622)
// ---------------------------------------------------------------------------
// d(phi)/d(dir) on face (i,j) of the faces nodal in `nodedir` (1: x-faces,
// i in [0,nx], j in [0,ny); 2: y-faces).  Same operations, in the same order,
// as compute_pd; the nodal derivative reads the ghosts.
__device__ double pd_face(const DF& P, int nx, int ny, double dx, double dy, int dir, int nodedir, int i, int j) {
    St9 s;
    if (dir == 1 && nodedir == 1) {   // P2:446-449
        const double scale = 1.0 / dx;
        return scale * (AT(P, i, j) - AT(P, i - 1, j));
    }
    if (dir == 2 && nodedir == 2) {   // P2:614-617
        const double scale = 1.0 / dy;
        return scale * (AT(P, i, j) - AT(P, i, j - 1));
    }
    if (dir == 1) {   // d/dx on y-faces, P2:450-612
        const double scale = 0.25 / dx;
        if (j == 0) {
            gather9(GLoad{&AT(P, i, 0), P.ld}, region(i, nx, false, false), RLO, s);
            return scale * (s.ee - s.ew + s.ese - s.esw);
        }
        if (j == ny) {
            gather9(GLoad{&AT(P, i, ny - 1), P.ld}, region(i, nx, false, false), RHI, s);
            return scale * (s.ene - s.enw + s.ee - s.ew);
        }
        if (i == 0)
            return -scale * (3.0 * AT(P, 0, j) - 4.0 * AT(P, 1, j) + AT(P, 2, j) + 3.0 * AT(P, 0, j - 1) -
                             4.0 * AT(P, 1, j - 1) + AT(P, 2, j - 1));
        if (i == nx - 1)
            return scale * (3.0 * AT(P, nx - 1, j) - 4.0 * AT(P, nx - 2, j) + AT(P, nx - 3, j) +
                            3.0 * AT(P, nx - 1, j - 1) - 4.0 * AT(P, nx - 2, j - 1) + AT(P, nx - 3, j - 1));
        return scale * (AT(P, i + 1, j) - AT(P, i - 1, j) + AT(P, i + 1, j - 1) - AT(P, i - 1, j - 1));
    }
    // d/dy on x-faces, P2:613-794
    const double scale = 0.25 / dy;
    if (i == 0) {
        gather9(GLoad{&AT(P, 0, j), P.ld}, RLO, region(j, ny, false, false), s);
        return scale * (s.en - s.es + s.enw - s.esw);
    }
    if (i == nx) {
        gather9(GLoad{&AT(P, nx - 1, j), P.ld}, RHI, region(j, ny, false, false), s);
        return scale * (s.ene - s.ese + s.en - s.es);
    }
    if (j == 0)
        return -scale * (3.0 * AT(P, i, 0) - 4.0 * AT(P, i, 1) + AT(P, i, 2) + 3.0 * AT(P, i - 1, 0) -
                         4.0 * AT(P, i - 1, 1) + AT(P, i - 1, 2));
    if (j == ny - 1)
        return scale * (3.0 * AT(P, i, ny - 1) - 4.0 * AT(P, i, ny - 2) + AT(P, i, ny - 3) +
                        3.0 * AT(P, i - 1, ny - 1) - 4.0 * AT(P, i - 1, ny - 2) + AT(P, i - 1, ny - 3));
    return scale * (AT(P, i, j + 1) - AT(P, i, j - 1) + AT(P, i - 1, j + 1) - AT(P, i - 1, j - 1));
}

// The value fill_boundary_fluxes writes on face k of Neumann side s.
__device__ __forceinline__ double bflux(const BCd& b, int homog, int s, int k) {
    if (homog || b.mode[s] == M_LAH) return 0.0;
    if (b.mode[s] == M_UNIFORM) return b.u[s];
    return b.d[s][k];
}

__global__ void k_pd(DF pd, DF phi, int nx, int ny, double dx, double dy, int dir, int nodedir) {
    CELL_IJ
    if (i >= nx + (nodedir == 1) || j >= ny + (nodedir == 2)) return;
    AT(pd, i, j) = pd_face(phi, nx, ny, dx, dy, dir, nodedir, i, j);
}

cudaError_t launch_pd(const DF& pd, const DF& phi, int nx, int ny, double dx, double dy, int dir, int nodedir,
                      cudaStream_t st) {
    k_pd<<<cells_grid(nx + 1, ny + 1, kBlk2), kBlk2, 0, st>>>(pd, phi, nx, ny, dx, dy, dir, nodedir);
    count_launch();
    return cudaGetLastError();
}

// J Grad[phi] on one face family (ghosts of phi filled), Neumann faces
// replaced by the BC flux (fill_boundary_fluxes).
__global__ void k_grad(DF flux, DF phi, Geo g, BCd b, int homog, int nx, int ny, int nodedir) {
    CELL_IJ
    if (nodedir == 1) {
        if (i > nx || j >= ny) return;
        const double pdn = pd_face(phi, nx, ny, g.dx, g.dy, 1, 1, i, j);
        const double pdt = pd_face(phi, nx, ny, g.dx, g.dy, 2, 1, i, j);
        double v = AT(g.xx, i, j) * pdn + AT(g.xy, i, j) * pdt;   // P2:833-834
        if (i == 0 && b.type[S_XLO] == T_NEUM) v = bflux(b, homog, S_XLO, j);
        if (i == nx && b.type[S_XHI] == T_NEUM) v = bflux(b, homog, S_XHI, j);
        AT(flux, i, j) = v;
    } else {
        if (i >= nx || j > ny) return;
        const double pdt = pd_face(phi, nx, ny, g.dx, g.dy, 1, 2, i, j);
        const double pdn = pd_face(phi, nx, ny, g.dx, g.dy, 2, 2, i, j);
        double v = AT(g.yx, i, j) * pdt + AT(g.yy, i, j) * pdn;   // P2:843-844
        if (j == 0 && b.type[S_YLO] == T_NEUM) v = bflux(b, homog, S_YLO, i);
        if (j == ny && b.type[S_YHI] == T_NEUM) v = bflux(b, homog, S_YHI, i);
        AT(flux, i, j) = v;
    }
}

cudaError_t launch_grad(const DF& xflux, const DF& yflux, const DF& phi, const Geo& g, const BCd& b, int homog,
                        int nx, int ny, cudaStream_t st) {
    k_grad<<<cells_grid(nx + 1, ny, kBlk2), kBlk2, 0, st>>>(xflux, phi, g, b, homog, nx, ny, 1);
    k_grad<<<cells_grid(nx, ny + 1, kBlk2), kBlk2, 0, st>>>(yflux, phi, g, b, homog, nx, ny, 2);
    count_launch(2);
    return cudaGetLastError();
}

__global__ void k_boundary_fluxes(DF xflux, DF yflux, BCd b, int homog, int nx, int ny) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    for (int s = 0; s < 4; ++s) {
        if (b.type[s] != T_NEUM) continue;
        if (s < 2 && k < ny) AT(xflux, s == S_XLO ? 0 : nx, k) = bflux(b, homog, s, k);
        if (s >= 2 && k < nx) AT(yflux, k, s == S_YLO ? 0 : ny) = bflux(b, homog, s, k);
    }
}

cudaError_t launch_boundary_fluxes(const DF& xflux, const DF& yflux, const BCd& b, int homog, int nx, int ny,
                                   cudaStream_t st) {
    const int n = nx > ny ? nx : ny;
    k_boundary_fluxes<<<(n + 255) / 256, 256, 0, st>>>(xflux, yflux, b, homog, nx, ny);
    count_launch();
    return cudaGetLastError();
}

__global__ void k_div(DF div, DF xflux, DF yflux, int nx, int ny, double dx, double dy) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    const double invdx = 1.0 / dx, invdy = 1.0 / dy;
    AT(div, i, j) = invdx * (AT(xflux, i + 1, j) - AT(xflux, i, j)) + invdy * (AT(yflux, i, j + 1) - AT(yflux, i, j));
}

cudaError_t launch_div(const DF& div, const DF& xflux, const DF& yflux, int nx, int ny, double dx, double dy,
                       cudaStream_t st) {
    k_div<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(div, xflux, yflux, nx, ny, dx, dy);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Gauss-Seidel (relax_gs, P2:1460-1988) in the device order:
//   1. ghosts once (P2:1556);
//   2. colours (i mod 2, j mod 2) = (0,0),(1,1),(1,0),(0,1) over the interior
//      cells -- their stencil reaches one cell, so each colour is an
//      independent set (one launch per colour);
//   3. the boundary cells, whose stencil reaches two cells inward (the
//      quadratic extrapolation, P2:947-951): the edge cells colour by colour,
//      then the four corners in turn (one CTA).
// No cell of a sub-pass reads another cell of the same sub-pass.
// ---------------------------------------------------------------------------
__global__ void k_gs_colour(DF phi, DF rhs, DF invd, Geo g, BCd b, int homog, int nx, int ny, double omega,
                            int ci, int cj) {
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ci;
    const int j = 2 * (blockIdx.y * blockDim.y + threadIdx.y) + cj;
    if (i >= nx || j >= ny) return;
    const Per pr = periodic_of(b);
    if (region(i, nx, pr.xl, pr.xh) != RMID || region(j, ny, pr.yl, pr.yh) != RMID) return;
    gs9(phi, rhs, invd, g, b, homog, nx, ny, i, j, omega);
}

// Perimeter cell k (0 <= k < 2nx + 2(ny-2)): rows j = 0 and ny-1, then columns i = 0 and nx-1.
__device__ __forceinline__ void perimeter_cell(int k, int nx, int ny, int& i, int& j) {
    if (k < nx) { i = k; j = 0; }
    else if (k < 2 * nx) { i = k - nx; j = ny - 1; }
    else if (k < 2 * nx + ny - 2) { i = 0; j = 1 + k - 2 * nx; }
    else { i = nx - 1; j = 1 + k - 2 * nx - (ny - 2); }
}

// ---------------------------------------------------------------------------
// Scopes of the cooperative building blocks (b_*): every thread of one CTA
// (BlockScope), or of a cooperative grid whose CTAs are all resident
// (GridScope: grid-stride loops, a grid barrier in place of __syncthreads,
// reductions combined across CTAs in CTA order).  With one CTA both run the
// same loops; BlockScope is what the single-CTA kernels use.
// ---------------------------------------------------------------------------
__shared__ GridCtl s_gctl;   // the grid kernel's barrier and partials (set on entry)
__shared__ int s_gred;       // grid reductions so far (parity of the partials buffer)

// A CTA gives up on a grid barrier after s_gctl.wait_ns of %globaltimer or
// kGridWaitLimit polls (each sleeps up to 256 ns), whichever comes first, and
// records DST_TIMEOUT.  From then on the grid's barriers are out of step, so
// every CTA that finds the status word set -- on entering a barrier or while
// polling one -- stops waiting at once: the kernel runs to its end in
// bounded time (its results are void and the host reports MGP_ETIMEOUT).
constexpr long kGridWaitLimit = 1L << 24;

__device__ __forceinline__ unsigned long long grid_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ void grid_barrier() {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile int* stv = s_gctl.status;
        if (*stv == DST_OK) {
            unsigned* bar = s_gctl.bar;
            volatile unsigned* gen = bar + 1;
            const unsigned g0 = *gen;
            __threadfence();
            if (atomicAdd(bar, 1u) == gridDim.x - 1) {   // the last to arrive opens the next generation
                atomicExch(bar, 0u);
                __threadfence();
                atomicAdd(bar + 1, 1u);
            } else {
                const unsigned long long t0 = grid_ns();
                unsigned nap = 32;
                for (long k = 0; *gen == g0; ++k) {
                    if (*stv != DST_OK) break;   // another CTA gave up
                    if (k > kGridWaitLimit || grid_ns() - t0 > s_gctl.wait_ns) {
                        set_status(s_gctl.status, DST_TIMEOUT);
                        break;
                    }
                    __nanosleep(nap);
                    nap = nap < 256 ? 2 * nap : nap;
                }
            }
            __threadfence();
        }
    }
    __syncthreads();
}

// rrank / rsize / ractive: the loop that accumulates a reduction's
// per-thread partial sums (RLOOP).
struct BlockScope {
    static constexpr bool kGrid = false;
    static constexpr bool kCluster = false;
    __device__ static int rank() { return threadIdx.x; }
    __device__ static int size() { return blockDim.x; }
    __device__ static void sync() { __syncthreads(); }
    __device__ static int rrank() { return threadIdx.x; }
    __device__ static int rsize() { return blockDim.x; }
    __device__ static bool ractive() { return true; }
};
struct GridScope {
    __device__ static int cta() { return blockIdx.x; }
    __device__ static int ncta() { return gridDim.x; }
    static constexpr bool kGrid = true;
    static constexpr bool kCluster = false;
    __device__ static int rank() { return blockIdx.x * blockDim.x + threadIdx.x; }
    __device__ static int size() { return gridDim.x * blockDim.x; }
    __device__ static void sync() { grid_barrier(); }
    __device__ static int rrank() { return rank(); }
    __device__ static int rsize() { return size(); }
    __device__ static bool ractive() { return true; }
};
// The CTAs of one thread-block cluster that is the whole grid (co-scheduled
// on one GPC by the hardware): GridScope's loops and CTA-ordered reductions,
// with the cluster's hardware barrier (release / acquire at cluster scope,
// which orders the global-memory accesses of every thread of the cluster) in
// place of the polled global-memory barrier.  Like __syncthreads it needs no
// time limit: every CTA of a cluster is resident before any runs, and the
// coarse cycle's control flow is the same in every CTA (each one combines
// the reductions' partials in the same order).
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// kOrdered: its reductions are accumulated by the first CTA alone, thread t
// summing cells t, t + blockDim, ... as BlockScope's thread t does, and
// combined by the same block tree (the CTAs have BlockScope's kCoarseThreads
// threads), so every result -- the sweeps, whose colour passes do not depend
// on which thread updates a cell, and the reductions -- has the bits of the
// one-CTA kernel; the result reaches the other CTAs through global memory.
// Otherwise every CTA accumulates its share and the CTAs' partials are
// combined in CTA order, as in GridScope.
// Ranks count within the cluster (%cluster_ctarank), so a grid of several
// clusters runs one coarse cycle per cluster.
template <bool kOrdered>
struct ClusterScope {
    static constexpr bool kGrid = true;
    static constexpr bool kCluster = kOrdered;
    __device__ static int cta() {
        unsigned r;
        asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
        return (int)r;
    }
    __device__ static int ncta() {
        unsigned r;
        asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
        return (int)r;
    }
    __device__ static int rank() { return cta() * blockDim.x + threadIdx.x; }
    __device__ static int size() { return ncta() * blockDim.x; }
    __device__ static void sync() { cluster_barrier(); }
    __device__ static int rrank() { return kOrdered ? (int)threadIdx.x : rank(); }
    __device__ static int rsize() { return kOrdered ? (int)blockDim.x : size(); }
    __device__ static bool ractive() { return !kOrdered || cta() == 0; }
};
#define SLOOP(k, n) for (int k = S::rank(); k < (n); k += S::size())
#define RLOOP(k, n) for (int k = S::rrank(); S::ractive() && k < (n); k += S::rsize())

// Step 3 of the sweep; every thread of the scope calls it.
template <class S>
__device__ void b_gs_boundary(const DF& phi, const DF& rhs, const DF& invd, const Geo& g, const BCd& b, int homog,
                              int nx, int ny, double omega) {
    const Per pr = periodic_of(b);
    const int np = 2 * nx + 2 * (ny - 2);
    for (int c = 0; c < 4; ++c) {
        const int ci = colour_ci(c), cj = colour_cj(c);
        SLOOP(k, np) {
            int i, j;
            perimeter_cell(k, nx, ny, i, j);
            if ((i & 1) != ci || (j & 1) != cj) continue;
            const bool xm = region(i, nx, pr.xl, pr.xh) == RMID, ym = region(j, ny, pr.yl, pr.yh) == RMID;
            if (xm != ym) gs9(phi, rhs, invd, g, b, homog, nx, ny, i, j, omega);
        }
        S::sync();
    }
    if (S::rank() == 0) {
        for (int c = 0; c < 4; ++c) {
            const int i = (c & 1) ? nx - 1 : 0, j = (c & 2) ? ny - 1 : 0;
            if (region(i, nx, pr.xl, pr.xh) != RMID && region(j, ny, pr.yl, pr.yh) != RMID)
                gs9(phi, rhs, invd, g, b, homog, nx, ny, i, j, omega);
        }
    }
    S::sync();
}

__global__ void __launch_bounds__(1024) k_gs_boundary(DF phi, DF rhs, DF invd, Geo g, BCd b, int homog, int nx,
                                                      int ny, double omega) {
    b_gs_boundary<BlockScope>(phi, rhs, invd, g, b, homog, nx, ny, omega);
}

cudaError_t launch_gs_sweep(const DF& phi, const DF& rhs, const DF& invd, const Geo& g, const BCd& b, int homog,
                            int nx, int ny, double omega, cudaStream_t st) {
    cudaError_t err = launch_fill(phi, g, b, homog, 0, nx, ny, st);   // P2:1556
    if (err != cudaSuccess) return err;
    const dim3 grd = cells_grid((nx + 1) / 2, (ny + 1) / 2, kBlk2);
    static const int ci[4] = {0, 1, 1, 0}, cj[4] = {0, 1, 0, 1};
    for (int c = 0; c < 4; ++c)
        k_gs_colour<<<grd, kBlk2, 0, st>>>(phi, rhs, invd, g, b, homog, nx, ny, omega, ci[c], cj[c]);
    const Per pr = {b.type[S_XLO] == T_PERIODIC, b.type[S_XHI] == T_PERIODIC, b.type[S_YLO] == T_PERIODIC,
                    b.type[S_YHI] == T_PERIODIC};
    int n = 4;
    if (!(pr.xl && pr.xh && pr.yl && pr.yh)) {
        k_gs_boundary<<<1, 1024, 0, st>>>(phi, rhs, invd, g, b, homog, nx, ny, omega);
        n = 5;
    }
    count_launch(n);
    return cudaGetLastError();
}

// compute_invdiags (P2:16-388)
__global__ void k_invdiag(DF invd, Geo g, BCd b, int homog, int nx, int ny, int coupled) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    AT(invd, i, j) = 1.0 / diag9(g, b, homog, nx, ny, i, j, coupled != 0);
}

cudaError_t launch_invdiag(const DF& invd, const Geo& g, const BCd& b, int homog, int nx, int ny, int coupled,
                           cudaStream_t st) {
    k_invdiag<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(invd, g, b, homog, nx, ny, coupled);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Restriction (MG:135-257) and prolongation (MG:262-394)
// ---------------------------------------------------------------------------
__global__ void k_restrict(DF f, DF c, int ncx, int ncy, int refx, int refy, int kind) {
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    const int cj = blockIdx.y * blockDim.y + threadIdx.y;
    if (kind == 0) {
        if (ci >= ncx || cj >= ncy) return;
        AT(c, ci, cj) = restrict_cc(f, ci, cj, refx, refy, 1.0 / (refx * refy));
    } else if (kind == 1) {   // x-faces: inject in x, average in y (MG:192-199)
        if (ci > ncx || cj >= ncy) return;
        const double scale = 1.0 / refy;
        double acc = 0.0;
        for (int a = 0; a < refy; ++a) acc = acc + scale * AT(f, ci * refx, cj * refy + a);
        AT(c, ci, cj) = acc;
    } else if (kind == 2) {   // y-faces: average in x, inject in y (MG:234-241)
        if (ci >= ncx || cj > ncy) return;
        const double scale = 1.0 / refx;
        double acc = 0.0;
        for (int a = 0; a < refx; ++a) acc = acc + scale * AT(f, ci * refx + a, cj * refy);
        AT(c, ci, cj) = acc;
    } else {
        if (ci > ncx || cj > ncy) return;
        AT(c, ci, cj) = AT(f, ci * refx, cj * refy);
    }
}

cudaError_t launch_restrict(const DF& f, const DF& c, int ncx, int ncy, int refx, int refy, int kind,
                            cudaStream_t st) {
    k_restrict<<<cells_grid(ncx + 1, ncy + 1, kBlk2), kBlk2, 0, st>>>(f, c, ncx, ncy, refx, refy, kind);
    count_launch();
    return cudaGetLastError();
}

// The V-cycle's residual, restriction and coarse initial guess in one pass
// (MG:793-795 then MG:805-806): a thread per fine cell computes its residual
// rhs - L[phi] (k_apply's operations) into shared memory; the threads of
// the block's coarse cells then sum their refx x refy fine residuals in
// restrict_cc's order and type, write the coarse right-hand side and, with
// guess, e = r * invdiag on the coarse level.  The fine residual never goes
// to global memory: 6 words per fine cell instead of 9, one launch instead of
// three, the same bits as k_apply, k_restrict_cc and k_set_guess in turn.
// Blocks are kBlk2 (32 x 8) fine cells, so refx, refy in {1, 2} tile them.
template <class T, class TC>
__global__ void __launch_bounds__(kBlk2N) k_resid_restrict(DFT<T> phi, DFT<T> rhs, GeoT<T> g, BCd b, int homog, int nx,
                                                           int ny, DFT<TC> rc, DFT<TC> ec, DFT<TC> invdc, int ncx,
                                                           int ncy, int refx, int refy, int guess) {
    __shared__ T w[8][33];
    pdl_wait();
    pdl_allow();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * 32 + tx, j = blockIdx.y * 8 + ty;
    T v = T(0.0);
    if (i < nx && j < ny) v = AT(rhs, i, j) - apply9(phi, g, b, homog, nx, ny, i, j);
    w[ty][tx] = v;
    __syncthreads();
    if ((tx % refx) || (ty % refy)) return;
    const int ci = i / refx, cj = j / refy;
    if (ci >= ncx || cj >= ncy) return;
    T acc = T(0.0);
    const T sc = T(1.0 / (refx * refy));
    for (int a = 0; a < refy; ++a)
        for (int c = 0; c < refx; ++c) acc = acc + sc * w[ty + a][tx + c];
    const TC r = TC(acc);
    AT(rc, ci, cj) = r;
    if (guess) AT(ec, ci, cj) = r * AT(invdc, ci, cj);
}

template <class T, class TC>
cudaError_t resid_restrict_impl(const DFT<T>& phi, const DFT<T>& rhs, const GeoT<T>& g, const BCd& b, int homog,
                                int nx, int ny, const DFT<TC>& rc, const DFT<TC>& ec, const DFT<TC>& invdc, int ncx,
                                int ncy, int refx, int refy, int guess, cudaStream_t st) {
    if (kBlk2.x != 32 || kBlk2.y != 8 || refx < 1 || refx > 2 || refy < 1 || refy > 2) return cudaErrorInvalidValue;
    const cudaError_t e = launch_dep(k_resid_restrict<T, TC>, cells_grid(nx, ny, kBlk2), kBlk2, 0, st, phi, rhs, g, b,
                                     homog, nx, ny, rc, ec, invdc, ncx, ncy, refx, refy, guess);
    count_launch();
    return e;
}
cudaError_t launch_resid_restrict(const DF& phi, const DF& rhs, const Geo& g, const BCd& b, int homog, int nx, int ny,
                                  const DF& rc, const DF& ec, const DF& invdc, int ncx, int ncy, int refx, int refy,
                                  int guess, cudaStream_t st) {
    return resid_restrict_impl(phi, rhs, g, b, homog, nx, ny, rc, ec, invdc, ncx, ncy, refx, refy, guess, st);
}
cudaError_t launch_resid_restrict(const DF32& phi, const DF32& rhs, const Geo32& g, const BCd& b, int homog, int nx,
                                  int ny, const DF32& rc, const DF32& ec, const DF32& invdc, int ncx, int ncy, int refx,
                                  int refy, int guess, cudaStream_t st) {
    return resid_restrict_impl(phi, rhs, g, b, homog, nx, ny, rc, ec, invdc, ncx, ncy, refx, refy, guess, st);
}
cudaError_t launch_resid_restrict(const DF32& phi, const DF32& rhs, const Geo32& g, const BCd& b, int homog, int nx,
                                  int ny, const DF& rc, const DF& ec, const DF& invdc, int ncx, int ncy, int refx,
                                  int refy, int guess, cudaStream_t st) {
    return resid_restrict_impl(phi, rhs, g, b, homog, nx, ny, rc, ec, invdc, ncx, ncy, refx, refy, guess, st);
}

// Cell-centred restriction of an FP32 field, into FP32 or (for the FP64
// coarse levels) FP64; the sum runs in the fine field's type.
template <class TF, class TC>
__global__ void k_restrict_cc(DFT<TF> f, DFT<TC> c, int ncx, int ncy, int refx, int refy) {
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    const int cj = blockIdx.y * blockDim.y + threadIdx.y;
    if (ci >= ncx || cj >= ncy) return;
    AT(c, ci, cj) = TC(restrict_cc(f, ci, cj, refx, refy, 1.0 / (refx * refy)));
}
cudaError_t launch_restrict(const DF32& f, const DF32& c, int ncx, int ncy, int refx, int refy, cudaStream_t st) {
    k_restrict_cc<<<cells_grid(ncx, ncy, kBlk2), kBlk2, 0, st>>>(f, c, ncx, ncy, refx, refy);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_restrict(const DF32& f, const DF& c, int ncx, int ncy, int refx, int refy, cudaStream_t st) {
    k_restrict_cc<<<cells_grid(ncx, ncy, kBlk2), kBlk2, 0, st>>>(f, c, ncx, ncy, refx, refy);
    count_launch();
    return cudaGetLastError();
}


// Cross term of the order-2 prolongation (MG:354-369); crse ghosts hold the
// order-3 extrapolation.
__device__ __forceinline__ void prolong_cross_cell(const DF& fine, const DF& crse, int ci, int cj) {
    const int fi = 2 * ci, fj = 2 * cj;
    const double mc = 0.0625 * (AT(crse, ci + 1, cj + 1) - AT(crse, ci + 1, cj - 1) - AT(crse, ci - 1, cj + 1) +
                                AT(crse, ci - 1, cj - 1));
    AT(fine, fi, fj) = AT(fine, fi, fj) + 0.25 * mc;
    AT(fine, fi + 1, fj) = AT(fine, fi + 1, fj) - 0.25 * mc;
    AT(fine, fi, fj + 1) = AT(fine, fi, fj + 1) - 0.25 * mc;
    AT(fine, fi + 1, fj + 1) = AT(fine, fi + 1, fj + 1) + 0.25 * mc;
}

template <class TF, class TC>
__global__ void k_prolong(DFT<TF> fine, DFT<TC> crse, int ncx, int ncy, int refx, int refy, int order) {
    pdl_wait();
    pdl_allow();
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    const int cj = blockIdx.y * blockDim.y + threadIdx.y;
    if (ci >= ncx || cj >= ncy) return;
    prolong_cell(fine, crse, ci, cj, refx, refy, order);
}

__global__ void k_prolong_cross(DF fine, DF crse, int ncx, int ncy) {
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    const int cj = blockIdx.y * blockDim.y + threadIdx.y;
    if (ci >= ncx || cj >= ncy) return;
    prolong_cross_cell(fine, crse, ci, cj);
}

cudaError_t launch_prolong(const DF& fine, const DF& crse, int ncx, int ncy, int refx, int refy, int order,
                           cudaStream_t st) {
    const cudaError_t e = launch_dep(k_prolong<double, double>, cells_grid(ncx, ncy, kBlk2), kBlk2, 0, st, fine, crse, ncx,
                                     ncy, refx, refy, order);
    count_launch();
    return e;
}

cudaError_t launch_prolong(const DF32& fine, const DF32& crse, int ncx, int ncy, int refx, int refy, int order,
                           cudaStream_t st) {
    const cudaError_t e = launch_dep(k_prolong<float, float>, cells_grid(ncx, ncy, kBlk2), kBlk2, 0, st, fine, crse, ncx,
                                     ncy, refx, refy, order);
    count_launch();
    return e;
}
cudaError_t launch_prolong(const DF32& fine, const DF& crse, int ncx, int ncy, int refx, int refy, int order,
                           cudaStream_t st) {
    const cudaError_t e = launch_dep(k_prolong<float, double>, cells_grid(ncx, ncy, kBlk2), kBlk2, 0, st, fine, crse, ncx,
                                     ncy, refx, refy, order);
    count_launch();
    return e;
}

cudaError_t launch_prolong_cross(const DF& fine, const DF& crse, int ncx, int ncy, cudaStream_t st) {
    k_prolong_cross<<<cells_grid(ncx, ncy, kBlk2), kBlk2, 0, st>>>(fine, crse, ncx, ncy);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Elementwise helpers
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_set_guess(DFT<T> e, DFT<T> r, DFT<T> invd, int nx, int ny) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    AT(e, i, j) = AT(r, i, j) * AT(invd, i, j);
}

cudaError_t launch_set_guess(const DF& e, const DF& r, const DF& invd, int nx, int ny, cudaStream_t st) {
    k_set_guess<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(e, r, invd, nx, ny);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_set_guess(const DF32& e, const DF32& r, const DF32& invd, int nx, int ny, cudaStream_t st) {
    k_set_guess<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(e, r, invd, nx, ny);
    count_launch();
    return cudaGetLastError();
}

// dst = src (rounded to dst's type) over i in [-gx, nx+gx), j in [-gy, ny+gy).
template <class TD, class TS>
__global__ void k_convert(DFT<TD> dst, DFT<TS> src, int nx, int ny, int gx, int gy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - gx;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - gy;
    if (i >= nx + gx || j >= ny + gy) return;
    AT(dst, i, j) = TD(AT(src, i, j));
}
cudaError_t launch_convert(const DF32& dst, const DF& src, int nx, int ny, int gx, int gy, cudaStream_t st) {
    k_convert<<<cells_grid(nx + 2 * gx, ny + 2 * gy, kBlk2), kBlk2, 0, st>>>(dst, src, nx, ny, gx, gy);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_convert(const DF& dst, const DF32& src, int nx, int ny, int gx, int gy, cudaStream_t st) {
    k_convert<<<cells_grid(nx + 2 * gx, ny + 2 * gy, kBlk2), kBlk2, 0, st>>>(dst, src, nx, ny, gx, gy);
    count_launch();
    return cudaGetLastError();
}

// Every value of an FP32 field (ghosts included) replaced by the nearest
// BF16 value (round to nearest even): the values a BF16 copy of the field
// would hold, read back into FP32 arithmetic.
__global__ void k_round_bf16(DF32 f, int nx, int ny, int g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - g;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - g;
    if (i >= nx + g || j >= ny + g) return;
    AT(f, i, j) = __bfloat162float(__float2bfloat16_rn(AT(f, i, j)));
}
cudaError_t launch_round_bf16(const DF32& f, int nx, int ny, int g, cudaStream_t st) {
    k_round_bf16<<<cells_grid(nx + 2 * g, ny + 2 * g, kBlk2), kBlk2, 0, st>>>(f, nx, ny, g);
    count_launch();
    return cudaGetLastError();
}

// One weighted Jacobi update (relax_jacobi, P2:1419-1424).
__global__ void k_jacobi(DF phi, DF r, DF invd, double omega, int nx, int ny) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    const double p = AT(phi, i, j);
    const double newphi = p + AT(r, i, j) * AT(invd, i, j);
    AT(phi, i, j) = omega * newphi + (1.0 - omega) * p;
}

cudaError_t launch_jacobi(const DF& phi, const DF& r, const DF& invd, double omega, int nx, int ny, cudaStream_t st) {
    k_jacobi<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(phi, r, invd, omega, nx, ny);
    count_launch();
    return cudaGetLastError();
}

__global__ void k_axpby(DF y, DF x, double a, double b, int nx, int ny, int gx, int gy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - gx;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - gy;
    if (i >= nx + gx || j >= ny + gy) return;
    // a == 1: y + b*x (the Fortran `y = y + b*x`); b == 1 too: y + x.
    const double yv = AT(y, i, j), xv = AT(x, i, j);
    double v;
    if (a == 1.0 && b == 1.0) v = yv + xv;
    else if (a == 1.0 && b == -1.0) v = yv - xv;
    else if (a == 1.0) v = yv + b * xv;
    else if (a == 0.0) v = b * xv;
    else v = a * yv + b * xv;
    AT(y, i, j) = v;
}

cudaError_t launch_axpby(const DF& y, const DF& x, double a, double b, int nx, int ny, int gx, int gy,
                         cudaStream_t st) {
    k_axpby<<<cells_grid(nx + 2 * gx, ny + 2 * gy, kBlk2), kBlk2, 0, st>>>(y, x, a, b, nx, ny, gx, gy);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Many-vector kernels of the GMRES outer iteration (MGP_FLAG_GMRES).  Vector k
// of a set is at V.p + k * V.stride, cell (i,j) at [i + j * V.ld]; valid cells
// only.  Deterministic: fixed per-block trees, blocks combined in order.
// ---------------------------------------------------------------------------
constexpr int kMdotThreads = 256;

// partials[k * gridDim.x + b] = sum over block b's cells of w * v_k (k = blockIdx.y).
__global__ void __launch_bounds__(kMdotThreads) k_mdot(DF w, MVec V, int nx, int ny, double* partials) {
    __shared__ double sh[kMdotThreads];
    const double* v = V.p + (long)blockIdx.y * V.stride;
    const long n = (long)nx * ny;
    double acc = 0.0;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)(c / nx);
        acc = acc + AT(w, i, j) * v[i + (long)j * V.ld];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = kMdotThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[(long)blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

// out[k] = sum of partials[k * nb .. k * nb + nb) (k = blockIdx.x), in block order.
__global__ void __launch_bounds__(kMdotThreads) k_mdot_final(const double* partials, int nb, double* out) {
    __shared__ double sh[kMdotThreads];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) acc = acc + partials[(long)blockIdx.x * nb + b];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = kMdotThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

cudaError_t launch_mdot(const DF& w, const MVec& V, int nv, int nx, int ny, double* partials, int nb, double* out,
                        cudaStream_t st) {
    k_mdot<<<dim3(nb, nv), kMdotThreads, 0, st>>>(w, V, nx, ny, partials);
    k_mdot_final<<<nv, kMdotThreads, 0, st>>>(partials, nb, out);
    count_launch(2);
    return cudaGetLastError();
}

// The multi-dot with kDotVecs basis vectors per launch row: a thread reads
// w at a cell once for all of its row's vectors, so a pass reads w
// ceil(nv / kDotVecs) times and each v_k once, where one row per vector read
// w nv times.  partials[k * gridDim.x + b] = block b's sum of w * v_k.
constexpr int kDotVecs = 8;

__global__ void __launch_bounds__(kMdotThreads) k_mdot8(DF w, MVec V, int nv, int nx, int ny, double* partials) {
    __shared__ double sh[kDotVecs][kMdotThreads];
    const int k0 = blockIdx.y * kDotVecs, kn = min(kDotVecs, nv - k0);
    const long n = (long)nx * ny;
    double acc[kDotVecs];
#pragma unroll
    for (int q = 0; q < kDotVecs; ++q) acc[q] = 0.0;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)(c / nx);
        const double wv = AT(w, i, j);
        const double* v = V.p + (long)k0 * V.stride + i + (long)j * V.ld;
#pragma unroll
        for (int q = 0; q < kDotVecs; ++q)
            if (q < kn) acc[q] = acc[q] + wv * v[(long)q * V.stride];
    }
#pragma unroll
    for (int q = 0; q < kDotVecs; ++q) sh[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int h = kMdotThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
#pragma unroll
            for (int q = 0; q < kDotVecs; ++q) sh[q][threadIdx.x] = sh[q][threadIdx.x] + sh[q][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x < kn) partials[(long)(k0 + threadIdx.x) * gridDim.x + blockIdx.x] = sh[threadIdx.x][0];
}

// w -= sum_{k < nv} h[k] v_k (the k_maxpy update, bit for bit) and, per
// block of cells, the sum of the new w^2 into partials[block] (blocks in
// row-major order of the launch grid).
__global__ void k_maxpy_nrm(DF w, MVec V, int nv, const double* h, int nx, int ny, double* partials) {
    __shared__ double sh[kBlk2N];
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int t = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    double sq = 0.0;
    if (i < nx && j < ny) {
        double acc = AT(w, i, j);
        for (int k = 0; k < nv; ++k) acc = acc + (-1.0 * h[k]) * V.p[(long)k * V.stride + i + (long)j * V.ld];
        AT(w, i, j) = acc;
        sq = acc * acc;
    }
    sh[t] = sq;
    __syncthreads();
    for (int s = nt / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] = sh[t] + sh[t + s];
        __syncthreads();
    }
    if (t == 0) partials[(long)blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

cudaError_t launch_gs_pass(const DF& w, const MVec& V, int nv, int nx, int ny, double* partials, long cap, int nb,
                           double* h, double* hnorm, cudaStream_t st) {
    const dim3 gu = cells_grid(nx, ny, kBlk2);
    const long nbu = (long)gu.x * gu.y;
    if (nv < 1 || (long)nb * nv > cap || nbu > cap || kBlk2.x * kBlk2.y != kBlk2N) return cudaErrorNotSupported;
    k_mdot8<<<dim3(nb, (nv + kDotVecs - 1) / kDotVecs), kMdotThreads, 0, st>>>(w, V, nv, nx, ny, partials);
    k_mdot_final<<<nv, kMdotThreads, 0, st>>>(partials, nb, h);
    // the coefficients are summed; their partials are free for the norm's
    k_maxpy_nrm<<<gu, kBlk2, 0, st>>>(w, V, nv, h, nx, ny, partials);
    k_mdot_final<<<1, kMdotThreads, 0, st>>>(partials, (int)nbu, hnorm);
    count_launch(4);
    return cudaGetLastError();
}

// w += sign * sum_{k < nv} coef[k] v_k over the valid cells (coef in device memory).
__global__ void k_maxpy(DF w, MVec V, int nv, const double* coef, double sign, int nx, int ny) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    double acc = AT(w, i, j);
    for (int k = 0; k < nv; ++k) acc = acc + (sign * coef[k]) * V.p[(long)k * V.stride + i + (long)j * V.ld];
    AT(w, i, j) = acc;
}

cudaError_t launch_maxpy(const DF& w, const MVec& V, int nv, const double* coef, double sign, int nx, int ny,
                         cudaStream_t st) {
    k_maxpy<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(w, V, nv, coef, sign, nx, ny);
    count_launch();
    return cudaGetLastError();
}

__global__ void k_muldiv(DF y, DF x, int mul, int nx, int ny) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    AT(y, i, j) = mul ? AT(y, i, j) * AT(x, i, j) : AT(y, i, j) / AT(x, i, j);
}

cudaError_t launch_muldiv(const DF& y, const DF& x, int mul, int nx, int ny, cudaStream_t st) {
    k_muldiv<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(y, x, mul, nx, ny);
    count_launch();
    return cudaGetLastError();
}

__global__ void k_fillval(DF y, double v, int nx, int ny, int gx, int gy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - gx;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - gy;
    if (i >= nx + gx || j >= ny + gy) return;
    AT(y, i, j) = v;
}

// y -= out[0] / out[1] over the whole allocation (prolong's mean removal, MG:371-383).
template <class T>
__global__ void k_sub_mean(DFT<T> y, const double* out, int nx, int ny, int gx, int gy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x - gx;
    const int j = blockIdx.y * blockDim.y + threadIdx.y - gy;
    if (i >= nx + gx || j >= ny + gy) return;
    AT(y, i, j) = AT(y, i, j) - T(out[0] / out[1]);
}

cudaError_t launch_sub_mean(const DF& y, const double* out, int nx, int ny, int gx, int gy, cudaStream_t st) {
    k_sub_mean<<<cells_grid(nx + 2 * gx, ny + 2 * gy, kBlk2), kBlk2, 0, st>>>(y, out, nx, ny, gx, gy);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_sub_mean(const DF32& y, const double* out, int nx, int ny, int gx, int gy, cudaStream_t st) {
    k_sub_mean<<<cells_grid(nx + 2 * gx, ny + 2 * gy, kBlk2), kBlk2, 0, st>>>(y, out, nx, ny, gx, gy);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_fillval(const DF& y, double v, int nx, int ny, int gx, int gy, cudaStream_t st) {
    k_fillval<<<cells_grid(nx + 2 * gx, ny + 2 * gy, kBlk2), kBlk2, 0, st>>>(y, v, nx, ny, gx, gy);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Deterministic reductions (pnorm AU:753-796, inner_prod AU:637-661,
// the J-weighted mean of prolong MG:371-383).  Fixed assignment of cells to
// threads and a fixed tree, so the result does not depend on scheduling.
// ---------------------------------------------------------------------------
constexpr int kRedThreads = 256;
constexpr int kRedBlocks = kRedBlocksMax;

template <class T>
__device__ __forceinline__ double red_term(int kind, const DFT<T>& a, const DFT<T>& b, int i, int j, double& w) {
    const double v = AT(a, i, j);
    switch (kind) {
        case RED_SUMSQ: return v * v;
        case RED_MAXABS: return fabs(v);
        case RED_DOT: return v * AT(b, i, j);
        case RED_ABSSUM: return fabs(v);
        default: { const double jj = AT(b, i, j); w = jj; return jj * v; }
    }
}

// Block b sums cells [b * per, (b + 1) * per) of the n = nx * ny valid cells
// in column-major order: consecutive threads on consecutive cells of a row
// (coalesced), each thread four independent partial sums (loads in flight),
// combined in a fixed order, then a fixed tree over the block.
template <class T>
__global__ void __launch_bounds__(kRedThreads) k_reduce_partial(int kind, DFT<T> a, DFT<T> b, int nx, int ny,
                                                                int per, double* partials) {
    __shared__ double s0[kRedThreads], s1[kRedThreads];
    const int n = nx * ny, c0 = blockIdx.x * per, m = max(0, min(n, c0 + per) - c0);
    const int step = blockDim.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0}, accw[4] = {0.0, 0.0, 0.0, 0.0};
    int i = (c0 + (int)threadIdx.x) % nx, j = (c0 + (int)threadIdx.x) / nx;
    int q = threadIdx.x;
    for (; q + 3 * step < m; q += 4 * step) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            double w = 0.0;
            const double t = red_term(kind, a, b, i, j, w);
            acc[u] = (kind == RED_MAXABS) ? fmax(acc[u], t) : acc[u] + t;
            accw[u] = accw[u] + w;
            for (i += step; i >= nx; i -= nx) ++j;
        }
    }
    for (; q < m; q += step) {
        double w = 0.0;
        const double t = red_term(kind, a, b, i, j, w);
        acc[0] = (kind == RED_MAXABS) ? fmax(acc[0], t) : acc[0] + t;
        accw[0] = accw[0] + w;
        for (i += step; i >= nx; i -= nx) ++j;
    }
    s0[threadIdx.x] = (kind == RED_MAXABS) ? fmax(fmax(acc[0], acc[1]), fmax(acc[2], acc[3]))
                                           : (acc[0] + acc[1]) + (acc[2] + acc[3]);
    s1[threadIdx.x] = (accw[0] + accw[1]) + (accw[2] + accw[3]);
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s0[threadIdx.x] = (kind == RED_MAXABS) ? fmax(s0[threadIdx.x], s0[threadIdx.x + s])
                                                   : s0[threadIdx.x] + s0[threadIdx.x + s];
            s1[threadIdx.x] = s1[threadIdx.x] + s1[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = s0[0];
        partials[2 * blockIdx.x + 1] = s1[0];
    }
}

__global__ void k_reduce_final(int kind, const double* partials, int nb, double vol, double* out) {
    __shared__ double s0[512], s1[512];
    double acc = 0.0, accw = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        acc = (kind == RED_MAXABS) ? fmax(acc, partials[2 * k]) : acc + partials[2 * k];
        accw = accw + partials[2 * k + 1];
    }
    s0[threadIdx.x] = acc;
    s1[threadIdx.x] = accw;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s0[threadIdx.x] = (kind == RED_MAXABS) ? fmax(s0[threadIdx.x], s0[threadIdx.x + s])
                                                   : s0[threadIdx.x] + s0[threadIdx.x + s];
            s1[threadIdx.x] = s1[threadIdx.x] + s1[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (kind == RED_SUMSQ) out[0] = sqrt(vol * s0[0]);
        else if (kind == RED_MAXABS) out[0] = s0[0];
        else if (kind == RED_JSUM) { out[0] = vol * s0[0]; out[1] = vol * s1[0]; }
        else out[0] = vol * s0[0];
    }
}

template <class T>
cudaError_t reduce_impl(int kind, const DFT<T>& a, const DFT<T>& b, int nx, int ny, double vol, double* partials,
                        double* out, cudaStream_t st) {
    const long n = (long)nx * ny;
    if (n >= (1L << 31)) return cudaErrorInvalidValue;
    // at least four cells a thread, so the four partial sums all fill
    int nb = (int)((n + 4 * kRedThreads - 1) / (4 * kRedThreads));
    if (nb > kRedBlocks) nb = kRedBlocks;
    if (nb < 1) nb = 1;
    const int per = (int)((n + nb - 1) / nb);
    k_reduce_partial<<<nb, kRedThreads, 0, st>>>(kind, a, b, nx, ny, per, partials);
    k_reduce_final<<<1, 512, 0, st>>>(kind, partials, nb, vol, out);
    count_launch(2);
    return cudaGetLastError();
}
cudaError_t launch_reduce(int kind, const DF& a, const DF& b, int nx, int ny, double vol, double* partials,
                          double* out, cudaStream_t st) {
    return reduce_impl(kind, a, b, nx, ny, vol, partials, out, st);
}
cudaError_t launch_reduce(int kind, const DF32& a, const DF32& b, int nx, int ny, double vol, double* partials,
                          double* out, cudaStream_t st) {
    return reduce_impl(kind, a, b, nx, ny, vol, partials, out, st);
}

// ---------------------------------------------------------------------------
// Deferred-correction operators (DD:16-334)
// ---------------------------------------------------------------------------
__global__ void k_dd_invdiag(DF invd, Geo g, int nx, int ny) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    const double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
    const double d = (AT(g.xx, i + 1, j) + AT(g.xx, i, j)) * idx2 + (AT(g.yy, i, j + 1) + AT(g.yy, i, j)) * idy2;
    AT(invd, i, j) = -1.0 / d;
}

cudaError_t launch_dd_invdiag(const DF& invd, const Geo& g, int nx, int ny, cudaStream_t st) {
    k_dd_invdiag<<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(invd, g, nx, ny);
    count_launch();
    return cudaGetLastError();
}

template <class T>
__global__ void k_dd_apply(DFT<T> out, DFT<T> phi, DFT<T> rhs, GeoT<T> g, BCd b, int nx, int ny, int mode) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    const T lap = dd_apply(phi, g, b, nx, ny, i, j);
    AT(out, i, j) = mode ? AT(rhs, i, j) - lap : lap;
}

template <class T>
cudaError_t dd_apply_impl(const DFT<T>& out, const DFT<T>& phi, const DFT<T>& rhs, const GeoT<T>& g, const BCd& b,
                          int nx, int ny, int mode, cudaStream_t st) {
    k_dd_apply<T><<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(out, phi, rhs, g, b, nx, ny, mode);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_dd_apply(const DF& out, const DF& phi, const DF& rhs, const Geo& g, const BCd& b, int nx, int ny,
                            int mode, cudaStream_t st) {
    return dd_apply_impl(out, phi, rhs, g, b, nx, ny, mode, st);
}
cudaError_t launch_dd_apply(const DF32& out, const DF32& phi, const DF32& rhs, const Geo32& g, const BCd& b, int nx,
                            int ny, int mode, cudaStream_t st) {
    return dd_apply_impl(out, phi, rhs, g, b, nx, ny, mode, st);
}

template <class T>
__global__ void k_dd_modrhs(DFT<T> out, DFT<T> phi, DFT<T> rhs, GeoT<T> g, int nx, int ny) {
    CELL_IJ
    if (i >= nx || j >= ny) return;
    AT(out, i, j) = dd_modrhs(phi, rhs, g, nx, ny, i, j);
}

template <class T>
cudaError_t dd_modrhs_impl(const DFT<T>& out, const DFT<T>& phi, const DFT<T>& rhs, const GeoT<T>& g, int nx, int ny,
                           cudaStream_t st) {
    k_dd_modrhs<T><<<cells_grid(nx, ny, kBlk2), kBlk2, 0, st>>>(out, phi, rhs, g, nx, ny);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_dd_modrhs(const DF& out, const DF& phi, const DF& rhs, const Geo& g, int nx, int ny,
                             cudaStream_t st) {
    return dd_modrhs_impl(out, phi, rhs, g, nx, ny, st);
}
cudaError_t launch_dd_modrhs(const DF32& out, const DF32& phi, const DF32& rhs, const Geo32& g, int nx, int ny,
                             cudaStream_t st) {
    return dd_modrhs_impl(out, phi, rhs, g, nx, ny, st);
}

// Red-black colour of DD:262-285 (parity of i+j relative to the valid corner).
template <class T>
__global__ void k_dd_colour(DFT<T> phi, DFT<T> modrhs, DFT<T> invd, GeoT<T> g, int nx, int ny, double omega,
                            int colour) {
    const int jj = blockIdx.y * blockDim.y + threadIdx.y;
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= ny) return;
    const int i = 2 * ii + ((colour + jj) & 1);
    if (i >= nx) return;
    dd_gs(phi, modrhs, invd, g, i, jj, omega);
}

template <class T>
cudaError_t dd_colour_impl(const DFT<T>& phi, const DFT<T>& modrhs, const DFT<T>& invd, const GeoT<T>& g, int nx,
                           int ny, double omega, int colour, cudaStream_t st) {
    k_dd_colour<T><<<cells_grid((nx + 1) / 2, ny, kBlk2), kBlk2, 0, st>>>(phi, modrhs, invd, g, nx, ny, omega,
                                                                         colour);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_dd_colour(const DF& phi, const DF& modrhs, const DF& invd, const Geo& g, int nx, int ny,
                             double omega, int colour, cudaStream_t st) {
    return dd_colour_impl(phi, modrhs, invd, g, nx, ny, omega, colour, st);
}
cudaError_t launch_dd_colour(const DF32& phi, const DF32& modrhs, const DF32& invd, const Geo32& g, int nx, int ny,
                             double omega, int colour, cudaStream_t st) {
    return dd_colour_impl(phi, modrhs, invd, g, nx, ny, omega, colour, st);
}

// ---------------------------------------------------------------------------
// Building blocks of the coarse cycle (every thread of the scope calls them;
// BLOOP is a block-stride loop for the single-CTA kernels' own staging)
// ---------------------------------------------------------------------------
#define BLOOP(k, n) for (int k = threadIdx.x; k < (n); k += blockDim.x)

template <class S>
__device__ void b_fill(const DF& p, const Geo& g, const BCd& b, int homog, int do_neum, int nx, int ny) {
    int lo[4], cnt[4];
    for (int s = 0; s < 4; ++s) side_range(b, s, nx, ny, do_neum, lo[s], cnt[s]);
    SLOOP(k, cnt[0] + cnt[1]) {
        if (k < cnt[0]) fill_side_elem(p, g, b, homog, 0, nx, ny, lo[0] + k);
        else fill_side_elem(p, g, b, homog, 1, nx, ny, lo[1] + k - cnt[0]);
    }
    S::sync();
    SLOOP(k, cnt[2] + cnt[3]) {
        if (k < cnt[2]) fill_side_elem(p, g, b, homog, 2, nx, ny, lo[2] + k);
        else fill_side_elem(p, g, b, homog, 3, nx, ny, lo[3] + k - cnt[2]);
    }
    S::sync();
    if (S::rank() < 4) fill_corner(p, b, nx, ny, S::rank());
    S::sync();
}

// Block-wide sum / max with a fixed combination order (warp shuffles, then the
// warps' partials in one warp), so the result does not depend on scheduling;
// in GridScope the CTAs' results are then combined in CTA order by every CTA
// (partials double-buffered: the barrier inside the next reduction keeps a
// fast CTA from overwriting partials a slow one still reads).
template <class S, bool kMax>
__device__ double b_reduce(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_down_sync(0xffffffffu, v, o);
        v = kMax ? fmax(v, u) : v + u;
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        double x = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_down_sync(0xffffffffu, x, o);
            x = kMax ? fmax(x, u) : x + u;
        }
        if (threadIdx.x == 0) sh[32] = x;
    }
    __syncthreads();
    if constexpr (!S::kGrid) {
        return sh[32];
    } else if constexpr (S::kCluster) {
        volatile double* part = s_gctl.part + (s_gred & 1) * S::ncta();
        if (S::cta() == 0 && threadIdx.x == 0) part[0] = sh[32];
        S::sync();
        if (threadIdx.x == 0) {
            sh[33] = part[0];
            s_gred = s_gred + 1;
        }
        __syncthreads();
        return sh[33];
    } else {
        volatile double* part = s_gctl.part + (s_gred & 1) * S::ncta();
        if (threadIdx.x == 0) part[S::cta()] = sh[32];
        S::sync();
        if (threadIdx.x == 0) {
            double t = part[0];
            for (int c = 1; c < S::ncta(); ++c) t = kMax ? fmax(t, part[c]) : t + part[c];
            sh[33] = t;
            s_gred = s_gred + 1;
        }
        __syncthreads();
        return sh[33];
    }
}
template <class S>
__device__ double b_sum(double v, double* sh) { return b_reduce<S, false>(v, sh); }
template <class S>
__device__ double b_max(double v, double* sh) { return b_reduce<S, true>(v, sh); }

// A thread's partial of a reduction over the cells k = rrank, rrank + rsize,
// ... (k = i + j nx), combined in that order: acc = op(acc, f(i, j)).  Four
// cells' values are loaded before they are combined, and the cell index
// advances by addition, so the loads overlap; the order of the combines, and
// so the result, is the plain loop's.
template <class S, bool kMax, class F>
__device__ __forceinline__ double r_accum(int nx, int ny, F f) {
    double acc = 0.0;
    if (!S::ractive()) return acc;
    const int n = nx * ny, step = S::rsize();
    const int di = step % nx, dj = step / nx;
    int k = S::rrank(), i = k % nx, j = k / nx;
    auto adv = [&](int& ii, int& jj) {
        ii += di;
        jj += dj;
        if (ii >= nx) {
            ii -= nx;
            ++jj;
        }
    };
    auto op = [](double x, double v) { return kMax ? fmax(x, v) : x + v; };
    for (; k + 3 * step < n; k += 4 * step) {
        int i1 = i, j1 = j;
        adv(i1, j1);
        int i2 = i1, j2 = j1;
        adv(i2, j2);
        int i3 = i2, j3 = j2;
        adv(i3, j3);
        const double v0 = f(i, j), v1 = f(i1, j1), v2 = f(i2, j2), v3 = f(i3, j3);
        acc = op(acc, v0);
        acc = op(acc, v1);
        acc = op(acc, v2);
        acc = op(acc, v3);
        i = i3;
        j = j3;
        adv(i, j);
    }
    for (; k < n; k += step) {
        acc = op(acc, f(i, j));
        adv(i, j);
    }
    return acc;
}

// pnorm (AU:753-796) with p = 2 or 0.
template <class S>
__device__ double b_pnorm(const DF& a, int nx, int ny, int p, double vol, double* sh) {
    if (p == 0) return b_max<S>(r_accum<S, true>(nx, ny, [&](int i, int j) { return fabs(AT(a, i, j)); }), sh);
    const double acc = r_accum<S, false>(nx, ny, [&](int i, int j) {
        const double v = AT(a, i, j);
        return v * v;
    });
    return sqrt(vol * b_sum<S>(acc, sh));
}

template <class S>
__device__ double b_dot(const DF& a, const DF& c, int nx, int ny, double vol, double* sh) {
    const double acc = r_accum<S, false>(nx, ny, [&](int i, int j) { return AT(a, i, j) * AT(c, i, j); });
    return vol * b_sum<S>(acc, sh);
}

// y = a*y + b*x over [-g, n+g) in both directions (g = 1 for ghosted arrays).
template <class S>
__device__ void b_axpby(const DF& y, const DF& x, double a, double bb, int nx, int ny, int g) {
    const int w = nx + 2 * g, h = ny + 2 * g;
    SLOOP(k, w * h) {
        const int i = k % w - g, j = k / w - g;
        const double yv = AT(y, i, j), xv = AT(x, i, j);
        double v;
        if (a == 1.0 && bb == 1.0) v = yv + xv;
        else if (a == 1.0 && bb == -1.0) v = yv - xv;
        else if (a == 1.0) v = yv + bb * xv;
        else if (a == 0.0) v = bb * xv;
        else v = a * yv + bb * xv;
        AT(y, i, j) = v;
    }
    S::sync();
}

template <class S>
__device__ void b_setval(const DF& y, double v, int nx, int ny, int g) {
    const int w = nx + 2 * g, h = ny + 2 * g;
    SLOOP(k, w * h) AT(y, k % w - g, k / w - g) = v;
    S::sync();
}

template <class S>
__device__ void b_mul(const DF& out, const DF& a, const DF& c, int nx, int ny) {
    SLOOP(k, nx * ny) AT(out, k % nx, k / nx) = AT(a, k % nx, k / nx) * AT(c, k % nx, k / nx);
    S::sync();
}

// 9-point sweeps (MG smoother), P2:1460-1988.
// One sweep in the device order by the whole block, for sides of type DIRI,
// NEUM and PERIODIC: the sweep-start ghost fill in one pass (every ghost
// depends on interior values only), the interior colours over precomputed
// ranges, the edge cells colour by colour along each non-periodic side, then
// the corners -- at once when the grid is at least 4 x 4 (their stencils,
// two cells deep, then neither read nor write each other), else in turn.
template <class S>
__device__ void b_sweep9(const DF& phi_, const DF& rhs_, const DF& invd_, const Geo& g_, const BCd& b, int homog,
                         int nx, int ny, double omega) {
    // field descriptors in registers: the level structs live in shared memory,
    // and every barrier would otherwise make the compiler reload them
    const DF phi = phi_, rhs = rhs_, invd = invd_;
    const Geo g = g_;
    const Per pr = periodic_of(b);
    const int mi0 = pr.xl ? 0 : 1, mi1 = pr.xh ? nx : nx - 1;
    const int mj0 = pr.yl ? 0 : 1, mj1 = pr.yh ? ny : ny - 1;
    // interior colour ranges and their divide-free index maps, set up before the fill
    // (the multiply is exact while cnt * (cw - 1) < 2^24, which every level
    // of up to 1024 cells meets; a larger level -- a depth capped by the
    // caller -- divides)
    int ci0[4], cj0[4], ccw[4], cnt[4];
    unsigned cm[4];
    bool fast[4];
    for (int c = 0; c < 4; ++c) {
        ci0[c] = mi0 + ((mi0 & 1) != colour_ci(c));
        cj0[c] = mj0 + ((mj0 & 1) != colour_cj(c));
        ccw[c] = (mi1 > ci0[c]) ? (mi1 - ci0[c] + 1) / 2 : 0;
        const int ch = (mj1 > cj0[c]) ? (mj1 - cj0[c] + 1) / 2 : 0;
        cnt[c] = ccw[c] * ch;
        cm[c] = fastdiv24_magic(ccw[c] > 0 ? ccw[c] : 1);
        fast[c] = (long)cnt[c] * (ccw[c] > 0 ? ccw[c] - 1 : 0) < (1L << 24);
    }
    const int ng = 2 * (nx + 2) + 2 * ny;
    SLOOP(k, ng) {
        int i, j;
        if (k < nx + 2) { i = k - 1; j = -1; }
        else if (k < 2 * (nx + 2)) { i = k - (nx + 2) - 1; j = ny; }
        else if (k < 2 * (nx + 2) + ny) { i = -1; j = k - 2 * (nx + 2); }
        else { i = nx; j = k - 2 * (nx + 2) - ny; }
        AT(phi, i, j) = sweep_ghost(DFLoad{phi}, b, homog, nx, ny, i, j);
    }
    S::sync();
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        SLOOP(k, cnt[c]) {
            const int kj = fast[c] ? fastdiv24(k, cm[c]) : k / ccw[c];
            gs9r(phi, rhs, invd, g, b, homog, ci0[c] + 2 * (k - kj * ccw[c]), cj0[c] + 2 * kj, RMID, RMID, omega);
        }
        S::sync();
    }
    const bool sxl = !pr.xl, sxh = !pr.xh, syl = !pr.yl, syh = !pr.yh;
    for (int c = 0; c < 4; ++c) {
        const int ci = colour_ci(c), cj = colour_cj(c);
        const int ia = mi0 + ((mi0 & 1) != ci), ja = mj0 + ((mj0 & 1) != cj);
        const int ni = (mi1 > ia) ? (mi1 - ia + 1) / 2 : 0, nj = (mj1 > ja) ? (mj1 - ja + 1) / 2 : 0;
        const int n0 = (syl && cj == 0) ? ni : 0;
        const int n1 = n0 + ((syh && ((ny - 1) & 1) == cj) ? ni : 0);
        const int n2 = n1 + ((sxl && ci == 0) ? nj : 0);
        const int n3 = n2 + ((sxh && ((nx - 1) & 1) == ci) ? nj : 0);
        SLOOP(k, n3) {
            if (k < n0) gs9r(phi, rhs, invd, g, b, homog, ia + 2 * k, 0, RMID, RLO, omega);
            else if (k < n1) gs9r(phi, rhs, invd, g, b, homog, ia + 2 * (k - n0), ny - 1, RMID, RHI, omega);
            else if (k < n2) gs9r(phi, rhs, invd, g, b, homog, 0, ja + 2 * (k - n1), RLO, RMID, omega);
            else gs9r(phi, rhs, invd, g, b, homog, nx - 1, ja + 2 * (k - n2), RHI, RMID, omega);
        }
        S::sync();
    }
    const bool apart = nx >= 4 && ny >= 4;
    if (apart ? S::rank() < 4 : S::rank() == 0) {
        for (int c = apart ? S::rank() : 0; c < (apart ? S::rank() + 1 : 4); ++c) {
            const int i = (c & 1) ? nx - 1 : 0, j = (c & 2) ? ny - 1 : 0;
            const int xr = region(i, nx, pr.xl, pr.xh), yr = region(j, ny, pr.yl, pr.yh);
            if (xr != RMID && yr != RMID) gs9r(phi, rhs, invd, g, b, homog, i, j, xr, yr, omega);
        }
    }
    S::sync();
}

__device__ __forceinline__ bool fusable_sides(const BCd& b) {
    for (int s = 0; s < 4; ++s)
        if (b.type[s] != T_DIRI && b.type[s] != T_NEUM && b.type[s] != T_PERIODIC) return false;
    return true;
}

template <class S>
__device__ void b_relax9(const Lv& L, const DF& phi, const DF& rhs, int homog, double omega, int sweeps) {
    const int nx = L.nx, ny = L.ny;
    if (fusable_sides(L.bc)) {
        for (int it = 0; it < sweeps; ++it) b_sweep9<S>(phi, rhs, L.invd, L.g, L.bc, homog, nx, ny, omega);
        return;
    }
    const int hx = (nx + 1) / 2, hy = (ny + 1) / 2;
    const Per pr = periodic_of(L.bc);
    for (int it = 0; it < sweeps; ++it) {
        b_fill<S>(phi, L.g, L.bc, homog, 0, nx, ny);
        for (int c = 0; c < 4; ++c) {   // interior cells, colour by colour
            const int ci = colour_ci(c), cj = colour_cj(c);
            SLOOP(k, hx * hy) {
                const int i = 2 * (k % hx) + ci, j = 2 * (k / hx) + cj;
                if (i < nx && j < ny && region(i, nx, pr.xl, pr.xh) == RMID && region(j, ny, pr.yl, pr.yh) == RMID)
                    gs9(phi, rhs, L.invd, L.g, L.bc, homog, nx, ny, i, j, omega);
            }
            S::sync();
        }
        b_gs_boundary<S>(phi, rhs, L.invd, L.g, L.bc, homog, nx, ny, omega);
    }
}

// 5-point red-black sweeps of the deferred-correction smoother (DD:153-334).
// modrhs is computed once per call, into L.w.
template <class S>
__device__ void b_relax_dd(const Lv& L, const DF& phi, const DF& rhs, int homog, double omega, int sweeps) {
    const int nx = L.nx, ny = L.ny;
    if (sweeps == 0) return;
    SLOOP(k, nx * ny) AT(L.w, k % nx, k / nx) = dd_modrhs(phi, rhs, L.g, nx, ny, k % nx, k / nx);
    S::sync();
    const int hx = (nx + 1) / 2;
    for (int it = 0; it < sweeps; ++it) {
        b_fill<S>(phi, L.g, L.bc, homog, 1, nx, ny);   // DD:259, neum_ghosts = .true.
        for (int colour = 0; colour < 2; ++colour) {
            SLOOP(k, hx * ny) {
                const int j = k / hx, i = 2 * (k % hx) + ((colour + j) & 1);
                if (i < nx) dd_gs(phi, L.w, L.invd, L.g, i, j, omega);
            }
            S::sync();
        }
    }
}

// out = rhs - L[phi] (mode 1) or L[phi] (mode 0); fills phi's ghosts first as the Fortran routines do.
template <class S>
__device__ void b_apply(const Lv& L, const DF& out, const DF& phi, const DF& rhs, int homog, int mode, int dd) {
    const int nx = L.nx, ny = L.ny;
    if (dd) {
        SLOOP(k, nx * ny) {
            const int i = k % nx, j = k / nx;
            const double lap = dd_apply(phi, L.g, L.bc, nx, ny, i, j);
            AT(out, i, j) = mode ? AT(rhs, i, j) - lap : lap;
        }
        S::sync();
        b_fill<S>(phi, L.g, L.bc, homog, 1, nx, ny);   // ghost state the DD routine leaves (DD:99)
    } else {
        b_fill<S>(phi, L.g, L.bc, homog, 0, nx, ny);   // P2:935
        SLOOP(k, nx * ny) {
            const int i = k % nx, j = k / nx;
            const double lap = apply9(phi, L.g, L.bc, homog, nx, ny, i, j);
            AT(out, i, j) = mode ? AT(rhs, i, j) - lap : lap;
        }
        S::sync();
    }
}

template <class S>
__device__ void b_relax(const Lv& L, const DF& phi, const DF& rhs, int homog, double omega, int sweeps, int dd) {
    if (dd) b_relax_dd<S>(L, phi, rhs, homog, omega, sweeps);
    else b_relax9<S>(L, phi, rhs, homog, omega, sweeps);
}

// solve_bicgstab2 (P2:2253-2477; DD:339-566 with dd = 1).  Status: DST_OK or DST_NONFINITE.
template <class S>
__device__ int b_bicgstab(const Lv& L, const DF& phi, const DF& rhs, int homog, double tol, int max_iters,
                          int max_restarts, int zerophi, int dd, double* sh) {
    const double reps = 1.0e-12, hang = 1.0e-7, small = 1.0e-30;
    const int norm_type = dd ? 0 : 2;
    const double relax_omega = dd ? 4.0 / 5.0 : 1.0 - 1.0 / 3.0;
    const int nx = L.nx, ny = L.ny;
    const double vol = L.g.dx * L.g.dy;
    const DF &e = L.ea, &pt = L.pt, &st = L.st, &r = L.rr, &rt = L.rt, &p = L.pp, &t = L.tt, &v = L.vv;
    double rho[4] = {0, 0, 0, 0}, norm[2], alpha[2] = {0, 0}, beta[2] = {0, 0}, omg[2] = {0, 0};
    int recount = 0, i = 0, restarts = 0, init = 1;
    if (max_iters == 0) return 0;
    if (zerophi) b_setval<S>(phi, 0.0, nx, ny, 1);
    b_apply<S>(L, r, phi, rhs, homog, 1, dd);
    b_axpby<S>(rt, r, 0.0, 1.0, nx, ny, 0);
    b_setval<S>(e, 0.0, nx, ny, 1);
    b_setval<S>(pt, 0.0, nx, ny, 1);
    b_setval<S>(st, 0.0, nx, ny, 1);
    norm[0] = b_pnorm<S>(r, nx, ny, norm_type, vol, sh);
    const double initial_norm = norm[0], initial_rnorm = norm[0];
    norm[1] = norm[0];
    while (((i < max_iters) && (norm[0] > tol * norm[1])) && (norm[1] > 0.0)) {
        i = i + 1;
        norm[1] = norm[0];
        alpha[1] = alpha[0];
        beta[1] = beta[0];
        omg[1] = omg[0];
        rho[3] = rho[2];
        rho[2] = rho[1];
        rho[1] = b_dot<S>(rt, r, nx, ny, vol, sh);
        if (rho[1] == 0.0) {
            b_axpby<S>(phi, e, 1.0, 1.0, nx, ny, 1);
            return 0;
        }
        if (init) {
            b_axpby<S>(p, r, 0.0, 1.0, nx, ny, 0);
            init = 0;
        } else {
            beta[1] = (rho[1] / rho[2]) * (alpha[1] / omg[1]);
            SLOOP(k, nx * ny) {
                const int a = k % nx, c = k / nx;
                AT(p, a, c) = beta[1] * (AT(p, a, c) - omg[1] * AT(v, a, c)) + AT(r, a, c);
            }
            S::sync();
        }
        b_mul<S>(pt, p, L.invd, nx, ny);
        b_relax<S>(L, pt, p, 1, relax_omega, 2, dd);
        b_apply<S>(L, v, pt, p, 1, 0, dd);
        const double m = b_dot<S>(rt, v, nx, ny, vol, sh);
        alpha[0] = rho[1] / m;
        if (fabs(m) > small * fabs(rho[1])) {
            b_axpby<S>(r, v, 1.0, -alpha[0], nx, ny, 0);
            norm[0] = b_pnorm<S>(r, nx, ny, norm_type, vol, sh);
            b_axpby<S>(e, pt, 1.0, alpha[0], nx, ny, 1);
        } else {
            b_setval<S>(r, 0.0, nx, ny, 0);
            norm[0] = 0.0;
        }
        if ((norm[0] > tol * initial_norm) && (norm[0] > reps * initial_rnorm)) {
            b_mul<S>(st, r, L.invd, nx, ny);
            b_relax<S>(L, st, r, 1, relax_omega, 2, dd);
            b_apply<S>(L, t, st, r, 1, 0, dd);
            const double tr = b_dot<S>(t, r, nx, ny, vol, sh);
            const double tt = b_dot<S>(t, t, nx, ny, vol, sh);
            omg[0] = tr / tt;
            b_axpby<S>(e, st, 1.0, omg[0], nx, ny, 1);
            b_axpby<S>(r, t, 1.0, -omg[0], nx, ny, 0);
            norm[0] = b_pnorm<S>(r, nx, ny, norm_type, vol, sh);
        }
        if ((norm[0] <= tol * initial_norm) || (norm[0] <= reps * initial_rnorm)) break;
        if ((omg[0] == 0.0) || (norm[0] > (1.0 - hang) * norm[1])) {
            if (recount == 0) {
                recount = 1;
            } else {
                recount = 0;
                b_axpby<S>(phi, e, 1.0, 1.0, nx, ny, 1);
                if (restarts == max_restarts) break;   // then e is added again below (P2:2466)
                b_apply<S>(L, r, phi, rhs, homog, 1, dd);
                norm[0] = b_pnorm<S>(r, nx, ny, norm_type, vol, sh);
                rho[1] = rho[2] = rho[3] = 0.0;
                alpha[0] = beta[0] = omg[0] = 0.0;
                b_axpby<S>(rt, r, 0.0, 1.0, nx, ny, 0);
                b_setval<S>(e, 0.0, nx, ny, 1);
                restarts = restarts + 1;
                init = 1;
            }
        }
    }
    b_axpby<S>(phi, e, 1.0, 1.0, nx, ny, 1);
    return isfinite(norm[0]) ? DST_OK : DST_NONFINITE;
}

// ---------------------------------------------------------------------------
// The coarse sub-cycle: vcycle_noinit(d0) run to the bottom in one CTA.
// ---------------------------------------------------------------------------
template <class S>
__device__ void b_prolong(const Lv& F, const Lv& Cl, int refx, int refy, int order, double* sh) {
    // fill_ghosts(crse, homog=.true., do_neum=.true.) (MG:318), then the fused add
    b_fill<S>(Cl.e, Cl.g, Cl.bc, 1, 1, Cl.nx, Cl.ny);
    SLOOP(k, Cl.nx * Cl.ny) prolong_cell(F.e, Cl.e, k % Cl.nx, k / Cl.nx, refx, refy, order);
    S::sync();
    const bool rax = (Cl.bc.type[0] == T_PERIODIC && Cl.bc.type[1] == T_PERIODIC) ||
                     (Cl.bc.type[0] == T_NEUM && Cl.bc.type[1] == T_NEUM);
    const bool ray = (Cl.bc.type[2] == T_PERIODIC && Cl.bc.type[3] == T_PERIODIC) ||
                     (Cl.bc.type[2] == T_NEUM && Cl.bc.type[3] == T_NEUM);
    if (rax && ray) {   // MG:371-383
        const double dxprod = F.g.dx * F.g.dy;
        double s = 0.0, vv = 0.0;
        RLOOP(k, F.nx * F.ny) {
            const double jj = AT(F.g.J, k % F.nx, k / F.nx);
            s = s + jj * AT(F.e, k % F.nx, k / F.nx);
            vv = vv + jj;
        }
        const double sum = dxprod * b_sum<S>(s, sh), vol = dxprod * b_sum<S>(vv, sh);
        const double avg = sum / vol;
        const int w = F.nx + 2, h = F.ny + 2;
        SLOOP(k, w * h) AT(F.e, k % w - 1, k / w - 1) = AT(F.e, k % w - 1, k / w - 1) - avg;
        S::sync();
    }
}

template <class S>
__device__ void b_set_guess(const Lv& L) {
    SLOOP(k, L.nx * L.ny) AT(L.e, k % L.nx, k / L.nx) = AT(L.r, k % L.nx, k / L.nx) * AT(L.invd, k % L.nx, k / L.nx);
    S::sync();
}

// e = A^{-1} r on the bottom level (MGP_FLAG_DIRECT_COARSE).  ainv holds the
// inverse transposed, ainv[m * n + k] = (A^{-1})_{k m}; row k takes four
// threads, each summing a quarter of the row, combined by two shuffles.
static_assert(4 * kDirectCells <= kCoarseThreads, "four threads per row of the bottom inverse");
template <class S>
__device__ void b_direct(const Lv& L, const double* ainv) {
    const int nx = L.nx, n = L.nx * L.ny;
    const int k = S::rank() >> 2, q = S::rank() & 3;
    double s = 0.0;
    if (k < n) {
        const int m0 = q * n / 4, m1 = (q + 1) * n / 4;
        int i = m0 % nx, j = m0 / nx;
        for (int m = m0; m < m1; ++m) {
            s = s + ainv[(size_t)m * n + k] * AT(L.r, i, j);
            if (++i == nx) {
                i = 0;
                ++j;
            }
        }
    }
    s = s + __shfl_xor_sync(0xffffffffu, s, 1);
    s = s + __shfl_xor_sync(0xffffffffu, s, 2);
    if (k < n && q == 0) AT(L.e, k % nx, k / nx) = s;
    S::sync();
}

// vcycle_noinit(d0) down to the bottom and back, on the levels lv[d0..maxdepth]
// (every thread of the block runs it).  Returns a nonzero status on a
// non-finite bottom residual.
template <class S>
__device__ int coarse_body(const Lv* lv, const CoarseArgs& a, double* sh) {
    int cnt[32];
    const double relax_omega = a.dd ? 4.0 / 5.0 : 1.0;
    int d = a.d0;
    int st = 0;
visit:
    {
        const Lv& L = lv[d];
        if (a.dd) b_set_guess<S>(L);   // DD:931, DD:971
        if (d == a.maxdepth) {
            if (a.ainv) {   // exact bottom solve
                b_direct<S>(L, a.ainv);
                goto up;
            }
            b_relax<S>(L, L.e, L.r, 1, relax_omega, a.nb, a.dd);
            const int s = b_bicgstab<S>(L, L.e, L.r, 1, 1.0e-6, 80, 5, 0, a.dd, sh);
            if (s) st = s;
            goto up;
        }
        b_relax<S>(L, L.e, L.r, 1, relax_omega, a.nd, a.dd);
        b_apply<S>(L, L.w, L.e, L.r, 1, 1, a.dd);
        const Lv& Cl = lv[d + 1];
        const int rx = a.refx[d], ry = a.refy[d];
        SLOOP(k, Cl.nx * Cl.ny) AT(Cl.r, k % Cl.nx, k / Cl.nx) =
            restrict_cc(L.w, k % Cl.nx, k / Cl.nx, rx, ry, 1.0 / (rx * ry));
        S::sync();
        if (!a.dd) b_set_guess<S>(Cl);   // MG:805-806
        if (a.numcycles == 0) goto finish;   // `do curcycle = 1, numcycles` runs no coarse visit
        cnt[d] = 0;
        d = d + 1;
        goto visit;
    }
up:
    if (d == a.d0) return st;
    d = d - 1;
    cnt[d] = cnt[d] + 1;
    if (cnt[d] < a.numcycles) {
        d = d + 1;
        goto visit;
    }
finish:
    {
        const Lv& L = lv[d];
        b_prolong<S>(L, lv[d + 1], a.refx[d], a.refy[d], 1, sh);
        b_relax<S>(L, L.e, L.r, 1, relax_omega, a.nu, a.dd);
    }
    goto up;
}

__global__ void __launch_bounds__(kCoarseThreads, 1) k_coarse_cycle(CoarseArgs a) {
    __shared__ double sh[kCoarseThreads];
    const int s = coarse_body<BlockScope>(a.lv, a, sh);
    if (threadIdx.x == 0) set_status(a.status, s);
}

__device__ void b_copy(const DF& dst, const DF& src, int i0, int i1, int j0, int j1) {
    const int w = i1 - i0, n = w * (j1 - j0);
    BLOOP(k, n) AT(dst, i0 + k % w, j0 + k / w) = AT(src, i0 + k % w, j0 + k / w);
}

// global -> shared with asynchronous copies; the caller waits (cp_async_wait_all).
__device__ void b_copy_in(const DF& dst, const DF& src, int i0, int i1, int j0, int j1) {
    const int w = i1 - i0, n = w * (j1 - j0);
    BLOOP(k, n) cp_async8(&AT(dst, i0 + k % w, j0 + k / w), &AT(src, i0 + k % w, j0 + k / w));
}

__device__ __forceinline__ void rebase(DF& f, double* base) { f.p = base + (size_t)(uintptr_t)f.p; }

// The same cycle with every coarse level held in shared memory: the levels'
// arrays are copied in (the corrections with their ghosts, the operands, the
// finest level's right-hand side), the cycle runs, the corrections go back.
__device__ __forceinline__ void coarse_cycle_smem(const CoarseArgs& a) {
    extern __shared__ double smem[];
    __shared__ double sh[kCoarseThreads];
    __shared__ Lv sl[kMaxCoarseLevels];
    const int nl = a.maxdepth - a.d0 + 1;
    if (threadIdx.x < nl) {
        Lv L = a.shadow[a.d0 + threadIdx.x];
        rebase(L.e, smem); rebase(L.r, smem); rebase(L.w, smem); rebase(L.invd, smem);
        rebase(L.g.J, smem); rebase(L.g.xx, smem); rebase(L.g.xy, smem); rebase(L.g.yx, smem); rebase(L.g.yy, smem);
        if (a.d0 + (int)threadIdx.x == a.maxdepth && !a.ainv) {
            rebase(L.ea, smem); rebase(L.pt, smem); rebase(L.st, smem);
            rebase(L.rr, smem); rebase(L.rt, smem); rebase(L.pp, smem); rebase(L.tt, smem); rebase(L.vv, smem);
        }
        sl[threadIdx.x] = L;
    }
    __syncthreads();
    for (int k = 0; k < nl; ++k) {
        const Lv &S = sl[k], &G = a.lv[a.d0 + k];
        const int nx = S.nx, ny = S.ny;
        b_copy_in(S.e, G.e, -1, nx + 1, -1, ny + 1);
        b_copy_in(S.invd, G.invd, 0, nx, 0, ny);
        b_copy_in(S.g.J, G.g.J, 0, nx, 0, ny);
        b_copy_in(S.g.xx, G.g.xx, 0, nx + 1, 0, ny);
        b_copy_in(S.g.xy, G.g.xy, 0, nx + 1, 0, ny);
        b_copy_in(S.g.yx, G.g.yx, 0, nx, 0, ny + 1);
        b_copy_in(S.g.yy, G.g.yy, 0, nx, 0, ny + 1);
        if (k == 0) b_copy_in(S.r, G.r, 0, nx, 0, ny);
    }
    cp_async_wait_all();
    __syncthreads();
    const int s = coarse_body<BlockScope>(sl - a.d0, a, sh);
    for (int k = 0; k < nl; ++k) {
        const Lv &S = sl[k], &G = a.lv[a.d0 + k];
        b_copy(G.e, S.e, -1, S.nx + 1, -1, S.ny + 1);
    }
    if (threadIdx.x == 0) set_status(a.status, s);
}

__global__ void __launch_bounds__(kCoarseThreads, 1) k_coarse_cycle_smem(CoarseArgs a) { coarse_cycle_smem(a); }

// The coarse cycles of a lockstep batch: a CTA per problem, each with its own
// arguments (staged in shared memory when its levels fit, else in place).
__global__ void __launch_bounds__(kCoarseThreads, 1) k_coarse_jobs(const CoarseJob* __restrict__ jobs) {
    const CoarseArgs& a = jobs[blockIdx.x].a;
    if (a.shadow && a.smem_bytes > 0) {
        coarse_cycle_smem(a);
    } else {
        __shared__ double sh[kCoarseThreads];
        const int s = coarse_body<BlockScope>(a.lv, a, sh);
        if (threadIdx.x == 0) set_status(a.status, s);
    }
}

cudaError_t launch_coarse_jobs(const CoarseJob* jobs, int njobs, int smem_bytes, cudaStream_t st) {
    if (njobs < 1) return cudaSuccess;
    static std::mutex mu;
    static unsigned long long done = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (dev >= 64 || !((done >> dev) & 1ull)) {
            e = cudaFuncSetAttribute(k_coarse_jobs, cudaFuncAttributeMaxDynamicSharedMemorySize, kCoarseSmemMax);
            if (e != cudaSuccess) return e;
            if (dev < 64) done |= 1ull << dev;
        }
    }
    k_coarse_jobs<<<njobs, kCoarseThreads, smem_bytes, st>>>(jobs);
    count_launch();
    return cudaGetLastError();
}

__global__ void __launch_bounds__(kCoarseThreads) k_direct_columns(Lv L, double* scratch, double* A) {
    const int nx = L.nx, ny = L.ny, n = nx * ny, k = blockIdx.x;
    const int ld = nx + 2;
    const size_t sz = (size_t)ld * (ny + 2);
    const DF phi{scratch + 2 * sz * k + ld + 1, ld}, out{scratch + (2 * k + 1) * sz + ld + 1, ld};
    b_setval<BlockScope>(phi, 0.0, nx, ny, 1);
    if (threadIdx.x == 0) AT(phi, k % nx, k / nx) = 1.0;
    __syncthreads();
    b_apply<BlockScope>(L, out, phi, out, 1, 0, 0);
    BLOOP(m, n) A[(size_t)m * n + k] = AT(out, m % nx, m / nx);
}

cudaError_t launch_direct_columns(const Lv& L, double* scratch, double* A, cudaStream_t st) {
    k_direct_columns<<<L.nx * L.ny, kCoarseThreads, 0, st>>>(L, scratch, A);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Gauss-Jordan inversion on the device (the exact bottom of
// MGP_FLAG_DIRECT_LARGE).  X = [A | I], n x 2n row-major, is reduced one
// pivot at a time.  Step c's pivot is the unused row with the largest
// |X[r][c]| (the lowest such row on ties); rows are never swapped: mark[r]
// records the step that took row r, prow[c] the pivot row of step c, and at
// the end row prow[c] of the right half is row c of A^-1.  Each update is
// X[r][k] - X[r][c] * (X[p][k] * (1 / X[p][c])), the pivot row scaled first,
// as in the textbook elimination; columns up to c are not read again.
// ---------------------------------------------------------------------------
constexpr int kGjThreads = 256;
constexpr int kGjRows = 32;   // rows of X per CTA and step

// X = [A | I]; mark[r] = n (unused); amax = max |A| over the entries that are
// not NaN (fmax's rule), as the bit pattern of a non-negative double, whose
// integer order is its numeric order: every CTA's maximum goes in by an
// atomic max on a word zeroed before the launch, which gives the exact
// maximum whatever the order.  An amax of 0 fails the first pivot test.
__global__ void __launch_bounds__(kGjThreads) k_gj_init(const double* A, int n, double* X, int* mark,
                                                        unsigned long long* amax_bits) {
    const long nn = (long)n * n;
    double m = 0.0;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < nn; q += (long)gridDim.x * blockDim.x) {
        const long r = q / n, k = q - r * n;
        const double a = A[q];
        X[r * 2 * n + k] = a;
        X[r * 2 * n + n + k] = (r == k) ? 1.0 : 0.0;
        m = fmax(m, fabs(a));
    }
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) mark[r] = n;
    __shared__ double sh[kGjThreads];
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int h = kGjThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicMax(amax_bits, (unsigned long long)__double_as_longlong(sh[0]));
}

// ainv[c][m] = X[prow[c]][n + m] (nothing after a failed step: prow is then incomplete).
__global__ void k_gj_extract(const double* X, const int* prow, const int* fail, int n, double* ainv) {
    if (*fail) return;
    const long nn = (long)n * n;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < nn; q += (long)gridDim.x * blockDim.x) {
        const long c = q / n, m = q - c * n;
        ainv[q] = X[(long)prow[c] * 2 * n + n + m];
    }
}

// The elimination runs blocked: kGjPanel pivots per pair of launches, each
// launch reading one buffer and writing the other, with every operation of
// the one-pivot steps above in its order (so the same bits as a launch per
// pivot).  k_gj_panel (one CTA, a
// thread per row) runs the steps on the panel's columns only: the pivot
// search, the pivot row scaled by 1 / pivot, the other rows' entries updated
// x - f * s; it records f[r][j] (row r's entry in the step's pivot column:
// the multiplier of step j) and 1 / pivot.  k_gj_trailing then replays the
// steps on the columns right of the panel: per column the pivot rows' new
// values s_j (the recurrence the steps apply to the pivot rows), then per row
// x = (r == p_j) ? s_j : x - f[r][j] * s_j for j in order.
constexpr int kGjPanelThreads = 1024;   // the largest bottom: a thread per row
static_assert(kGjPanelThreads >= kDirectLargeCells, "a panel thread per row of the largest bottom");

__global__ void __launch_bounds__(kGjPanelThreads) k_gj_panel(const double* __restrict__ X, int n, int c0, int b,
                                                              int* mark, int* prow, const double* amax, int* fail,
                                                              double* f, double* ipiv) {
    __shared__ double sv[kGjPanelThreads / 32];
    __shared__ int sr[kGjPanelThreads / 32];
    __shared__ double prowv[kGjPanel];
    if (*fail) return;
    const double amx = *amax;   // read once: the stores below may alias it as far as the compiler knows
    const int r = threadIdx.x;
    const bool live = r < n;
    double x[kGjPanel];
#pragma unroll
    for (int j = 0; j < kGjPanel; ++j) x[j] = (live && j < b) ? X[(long)r * 2 * n + c0 + j] : 0.0;
    int mk = live ? mark[r] : -1;
    const int lane = r & 31, wid = r >> 5;
#pragma unroll
    for (int j = 0; j < kGjPanel; ++j) {
        if (j >= b) break;
        const int c = c0 + j;
        // pivot: the unused row with the largest |x[j]|, the lowest on ties
        double best = (live && mk >= c) ? fabs(x[j]) : -1.0;
        int br = (live && mk >= c) ? r : n;
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_down_sync(0xffffffffu, best, o);
            const int orr = __shfl_down_sync(0xffffffffu, br, o);
            if (ob > best || (ob == best && orr < br)) { best = ob; br = orr; }
        }
        if (lane == 0) { sv[wid] = best; sr[wid] = br; }
        __syncthreads();
        // every warp combines the warps' candidates by the same tree, so all
        // agree on the pivot without another barrier (the next writes of
        // sv / sr come after the barrier below, which every warp reaches
        // only when done reading them)
        best = lane < kGjPanelThreads / 32 ? sv[lane] : -1.0;
        br = lane < kGjPanelThreads / 32 ? sr[lane] : n;
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_down_sync(0xffffffffu, best, o);
            const int orr = __shfl_down_sync(0xffffffffu, br, o);
            if (ob > best || (ob == best && orr < br)) { best = ob; br = orr; }
        }
        const int p = __shfl_sync(0xffffffffu, br, 0);
        if (p >= n) {
            if (r == 0) *fail = 1;
            return;
        }
        if (r == p) {
#pragma unroll
            for (int q = 0; q < kGjPanel; ++q) prowv[q] = x[q];
        }
        __syncthreads();
        const double piv = prowv[j];
        if (!(fabs(piv) > 1e-13 * amx)) {
            if (r == 0) *fail = 1;
            return;
        }
        const double ip = 1.0 / piv;
        if (r == p) {
            mk = c;
            mark[p] = c;
            prow[c] = p;
        }
        if (r == 0) ipiv[j] = ip;
        const double fj = x[j];   // the multiplier; x[j] keeps it (only columns right of j change)
#pragma unroll
        for (int q = 0; q < kGjPanel; ++q) {
            if (q <= j || q >= b) continue;
            const double sk = prowv[q] * ip;
            x[q] = (r == p) ? sk : x[q] - fj * sk;
        }
        // prowv is rewritten by the next step's pivot row only after the
        // next step's first barrier, which every thread reaches after this read
    }
    // f[r][j] = row r's entry in step j's pivot column, written once for the
    // panel as one 128-byte row a thread (16-byte stores) instead of an
    // 8-byte store a step
    if (live) {
        double2* fr = reinterpret_cast<double2*>(f + (long)r * kGjPanel);
#pragma unroll
        for (int j = 0; j < kGjPanel; j += 2) fr[j / 2] = make_double2(x[j], x[j + 1]);
    }
}

// Columns [c0 + b, 2n) of rows [r0, r0 + kGjRows): grid (columns / kGjThreads, rows / kGjRows).
__global__ void __launch_bounds__(kGjThreads) k_gj_trailing(const double* __restrict__ X, double* __restrict__ Y,
                                                            int n, int c0, int b, const int* prow, const double* f,
                                                            const double* ipiv, const int* fail) {
    __shared__ double fp[kGjPanel][kGjPanel];   // f[p_j][i]
    __shared__ double fr[kGjRows][kGjPanel];    // f[r][j] of this CTA's rows
    __shared__ int pr[kGjPanel];
    __shared__ double ip[kGjPanel];
    if (*fail) return;
    const int r0 = blockIdx.y * kGjRows, r1 = min(n, r0 + kGjRows);
    for (int q = threadIdx.x; q < b; q += blockDim.x) {
        pr[q] = prow[c0 + q];
        ip[q] = ipiv[q];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < b * b; q += blockDim.x) fp[q / b][q % b] = f[(long)pr[q / b] * kGjPanel + q % b];
    for (int q = threadIdx.x; q < (r1 - r0) * b; q += blockDim.x) fr[q / b][q % b] = f[(long)(r0 + q / b) * kGjPanel + q % b];
    __syncthreads();
    const int k = c0 + b + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 2 * n) return;
    double sj[kGjPanel];
#pragma unroll
    for (int j = 0; j < kGjPanel; ++j) {
        if (j >= b) break;
        double x = X[(long)pr[j] * 2 * n + k];
#pragma unroll
        for (int i = 0; i < kGjPanel; ++i)
            if (i < j) x = x - fp[j][i] * sj[i];
        sj[j] = x * ip[j];
    }
    for (int r = r0; r < r1; ++r) {
        double x = X[(long)r * 2 * n + k];
#pragma unroll
        for (int j = 0; j < kGjPanel; ++j) {
            if (j >= b) break;
            x = (r == pr[j]) ? sj[j] : x - fr[r - r0][j] * sj[j];
        }
        Y[(long)r * 2 * n + k] = x;
    }
}

cudaError_t launch_invert(const double* A, int n, double* ainv, double* work, int* iwork, cudaStream_t st) {
    double *X0 = work, *X1 = work + 2L * n * n, *amax = work + 4L * n * n;
    double *f = amax + 2, *ipiv = f + (long)n * kGjPanel;   // f 16-byte aligned (the panel's double2 stores)
    int *mark = iwork, *prow = iwork + n, *fail = iwork + 2 * n;
    if (n > kGjPanelThreads) return cudaErrorNotSupported;
    const int nb = std::min(1184, (int)((2L * n * n + kGjThreads - 1) / kGjThreads));
    cudaError_t e = cudaMemsetAsync(amax, 0, sizeof(double), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(fail, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    k_gj_init<<<nb, kGjThreads, 0, st>>>(A, n, X0, mark, reinterpret_cast<unsigned long long*>(amax));
    int launches = 2, cur = 0;
    for (int c0 = 0; c0 < n; c0 += kGjPanel) {
        const int b = std::min(kGjPanel, n - c0);
        double* Xc = cur ? X1 : X0;
        double* Xn = cur ? X0 : X1;
        k_gj_panel<<<1, kGjPanelThreads, 0, st>>>(Xc, n, c0, b, mark, prow, amax, fail, f, ipiv);
        const int ncols = 2 * n - (c0 + b);
        if (ncols > 0) {
            const dim3 grid((ncols + kGjThreads - 1) / kGjThreads, (n + kGjRows - 1) / kGjRows);
            k_gj_trailing<<<grid, kGjThreads, 0, st>>>(Xc, Xn, n, c0, b, prow, f, ipiv, fail);
            cur ^= 1;
            ++launches;
        }
        ++launches;
    }
    k_gj_extract<<<nb, kGjThreads, 0, st>>>(cur ? X1 : X0, prow, fail, n, ainv);
    count_launch(launches);
    return cudaGetLastError();
}

// e_k = sum_m ainv[k][m] r_m: r staged in shared memory, one warp per row k,
// lanes over m in steps of 32, then a butterfly of shuffles (a fixed order).
constexpr int kDirectApplyThreads = 256;
__global__ void __launch_bounds__(kDirectApplyThreads) k_direct_apply(DF e, DF r, const double* ainv, int nx,
                                                                      int n) {
    __shared__ double rs[kDirectLargeCells];
    // the inverse is fixed: its rows go to L2 while the kernel ahead finishes
    {
        const char* base = reinterpret_cast<const char*>(ainv + (long)blockIdx.x * (kDirectApplyThreads / 32) * n);
        const long bytes = (long)min(kDirectApplyThreads / 32, n - (int)blockIdx.x * (kDirectApplyThreads / 32)) * n * 8;
        for (long o = (long)threadIdx.x * 128; o < bytes; o += (long)blockDim.x * 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(base + o));
    }
    pdl_wait();
    pdl_allow();
    for (int m = threadIdx.x; m < n; m += blockDim.x) rs[m] = AT(r, m % nx, m / nx);
    __syncthreads();
    const int k = blockIdx.x * (kDirectApplyThreads / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (k >= n) return;
    const double* row = ainv + (long)k * n;
    double s = 0.0;
#pragma unroll 8
    for (int m = lane; m < n; m += 32) s = s + row[m] * rs[m];
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) AT(e, k % nx, k / nx) = s;
}

cudaError_t launch_direct_apply(const DF& e, const DF& r, const double* ainv, int nx, int ny, cudaStream_t st) {
    const int n = nx * ny, w = kDirectApplyThreads / 32;
    const cudaError_t err = launch_dep(k_direct_apply, dim3((n + w - 1) / w), dim3(kDirectApplyThreads), 0, st, e, r,
                                       ainv, nx, n);
    count_launch();
    return err;
}

// The exact bottoms of a lockstep batch (MGP_FLAG_DIRECT_LARGE): job k owns
// blocks [pre[k], pre[k+1]), each k_direct_apply's rows of the job's level.
__global__ void __launch_bounds__(kDirectApplyThreads) k_direct_jobs(const DirectJob* __restrict__ jobs,
                                                                     const int* __restrict__ pre, int njobs) {
    __shared__ double rs[kDirectLargeCells];
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(pre + mid) <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const DirectJob& J = jobs[lo];
    const int n = J.nx * J.ny;
    for (int m = threadIdx.x; m < n; m += blockDim.x) rs[m] = AT(J.r, m % J.nx, m / J.nx);
    __syncthreads();
    const int k = ((int)blockIdx.x - pre[lo]) * (kDirectApplyThreads / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (k >= n) return;
    const double* row = J.ainv + (long)k * n;
    double sacc = 0.0;
#pragma unroll 8
    for (int m = lane; m < n; m += 32) sacc = sacc + row[m] * rs[m];
    for (int o = 16; o > 0; o >>= 1) sacc = sacc + __shfl_xor_sync(0xffffffffu, sacc, o);
    if (lane == 0) AT(J.e, k % J.nx, k / J.nx) = sacc;
}

int direct_apply_blocks(int nx, int ny) {
    const int w = kDirectApplyThreads / 32;
    return (nx * ny + w - 1) / w;
}

cudaError_t launch_direct_jobs(const DirectJob* jobs, const int* pre, int njobs, int nblocks, cudaStream_t st) {
    if (njobs < 1 || nblocks < 1) return cudaSuccess;
    k_direct_jobs<<<nblocks, kDirectApplyThreads, 0, st>>>(jobs, pre, njobs);
    count_launch();
    return cudaGetLastError();
}

// Per device: opt the shared-memory coarse kernel into its largest window.
cudaError_t coarse_kernels_init() {
    static std::mutex mu;
    static unsigned long long done = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && ((done >> dev) & 1ull)) return cudaSuccess;
    e = cudaFuncSetAttribute(k_coarse_cycle_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, kCoarseSmemMax);
    if (e == cudaSuccess && dev < 64) done |= 1ull << dev;
    return e;
}

// The coarse sub-cycle over a cooperative grid of a.grid_ctas CTAs (all
// resident: one per SM at most), for hierarchies whose coarsest level is too
// large for one CTA (the schedule stops coarsening at an odd side).
__global__ void __launch_bounds__(kCoarseThreads, 1) k_coarse_cycle_grid(CoarseArgs a) {
    __shared__ double sh[kCoarseThreads];
    if (threadIdx.x == 0) {
        s_gctl = a.gctl;
        s_gred = 0;
    }
    __syncthreads();
    const int s = coarse_body<GridScope>(a.lv, a, sh);
    if (GridScope::rank() == 0) set_status(a.status, s);
}

// The coarse sub-cycle over one thread-block cluster of a.grid_ctas CTAs
// (a.cluster set): the same body as k_coarse_cycle_grid with hardware
// cluster barriers, for coarsest levels that one CTA cannot stage in shared
// memory, where the grid version's time is its barriers.  kOrdered
// (a.cluster == 2): the one-CTA kernel's reduction order and bits.
static_assert(kClusterThreads == kCoarseThreads, "the cluster CTAs reduce in the one-CTA kernel's order");
// Two CTAs an SM (128 registers, some spilled): a cluster CTA fits beside a
// sweep CTA of another stream, so under a server's concurrent solves a
// cluster does not wait for sixteen idle SMs in one GPC (served p99 at 10
// requests/s 156-1162 ms over four runs with one CTA an SM, 158-207 ms with
// two); alone it is 6 % slower on a 145 x 215 level.
template <bool kOrdered>
__global__ void __launch_bounds__(kClusterThreads, 2) k_coarse_cycle_cluster(CoarseArgs a) {
    __shared__ double sh[64];
    if (threadIdx.x == 0) {
        s_gctl = a.gctl;
        s_gred = 0;
    }
    __syncthreads();
    const int s = coarse_body<ClusterScope<kOrdered>>(a.lv, a, sh);
    if (ClusterScope<kOrdered>::rank() == 0) set_status(a.status, s);
}

// Largest cluster of k_coarse_cycle_cluster (16, else 8) that the current
// device can place at least once, or 0.
int coarse_cluster_ctas_max() {
    static std::mutex mu;
    static int cached[64];
    static unsigned long long known = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && ((known >> dev) & 1ull)) return cached[dev];
    int best = 0;
    if (cudaFuncSetAttribute(k_coarse_cycle_cluster<true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
            cudaSuccess &&
        cudaFuncSetAttribute(k_coarse_cycle_cluster<false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
            cudaSuccess) {
        for (int n : {16, 8}) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(n);
            cfg.blockDim = dim3(kClusterThreads);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = n;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int nclusters = 0;
            int nclusters2 = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, k_coarse_cycle_cluster<true>, &cfg) == cudaSuccess &&
                cudaOccupancyMaxActiveClusters(&nclusters2, k_coarse_cycle_cluster<false>, &cfg) == cudaSuccess &&
                nclusters >= 1 && nclusters2 >= 1) {
                best = n;
                break;
            }
        }
    }
    cudaGetLastError();
    if (dev < 64) {
        cached[dev] = best;
        known |= 1ull << dev;
    }
    return best;
}

// How many CTAs of k_coarse_cycle_grid the current device can keep resident
// at once (0 if it cannot launch cooperative grids).
int coarse_grid_ctas_max() {
    int dev = 0, coop = 0, nsm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_coarse_cycle_grid, kCoarseThreads, 0) !=
            cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return coop ? nsm * per_sm : 0;
}

__global__ void __launch_bounds__(32) k_barrier_selftest(GridCtl g, int skip, int nbar) {
    if (threadIdx.x == 0) {
        s_gctl = g;
        s_gred = 0;
    }
    __syncthreads();
    if ((int)blockIdx.x == skip) return;   // this CTA never arrives
    for (int k = 0; k < nbar; ++k) grid_barrier();
}

int barrier_selftest_ctas_max() {
    int dev = 0, coop = 0, nsm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_barrier_selftest, 32, 0) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return coop ? nsm * per_sm : 0;
}

cudaError_t launch_barrier_selftest(const GridCtl& g, int nctas, int skip, int nbar, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nctas);
    cfg.blockDim = dim3(32);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_barrier_selftest, g, skip, nbar);
    count_launch();
    return e;
}

cudaError_t launch_coarse_cycle(const CoarseArgs& a, cudaStream_t st) {
    if (a.grid_ctas > 1 && a.cluster) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(a.grid_ctas);
        cfg.blockDim = dim3(kClusterThreads);
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = a.grid_ctas;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        const cudaError_t e = a.cluster == 2 ? cudaLaunchKernelEx(&cfg, k_coarse_cycle_cluster<true>, a)
                                             : cudaLaunchKernelEx(&cfg, k_coarse_cycle_cluster<false>, a);
        count_launch();
        return e;
    }
    if (a.grid_ctas > 1) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(a.grid_ctas);
        cfg.blockDim = dim3(kCoarseThreads);
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelEx(&cfg, k_coarse_cycle_grid, a);
        count_launch();
        return e;
    }
    if (a.shadow && a.smem_bytes > 0) {
        const cudaError_t e = coarse_kernels_init();
        if (e != cudaSuccess) return e;
        k_coarse_cycle_smem<<<1, kCoarseThreads, a.smem_bytes, st>>>(a);
    } else {
        k_coarse_cycle<<<1, kCoarseThreads, 0, st>>>(a);
    }
    count_launch();
    return cudaGetLastError();
}

__global__ void __launch_bounds__(kCoarseThreads, 1) k_bicgstab(BicgArgs a) {
    __shared__ double sh[kCoarseThreads];
    const int s = b_bicgstab<BlockScope>(a.L, a.phi, a.rhs, a.homog, a.tol, a.max_iters, a.max_restarts, a.zerophi,
                                         a.dd, sh);
    if (threadIdx.x == 0) set_status(a.status, s);
}

cudaError_t launch_bicgstab(const BicgArgs& a, cudaStream_t st) {
    k_bicgstab<<<1, kCoarseThreads, 0, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

__global__ void __launch_bounds__(kCoarseThreads) k_relax_block(Lv L, DF phi, DF rhs, int homog, double omega,
                                                               int sweeps, int dd) {
    b_relax<BlockScope>(L, phi, rhs, homog, omega, sweeps, dd);
}

cudaError_t launch_relax_block(const Lv& L, const DF& phi, const DF& rhs, int homog, double omega, int sweeps,
                               int dd, int* status, cudaStream_t st) {
    (void)status;
    k_relax_block<<<1, kCoarseThreads, 0, st>>>(L, phi, rhs, homog, omega, sweeps, dd);
    count_launch();
    return cudaGetLastError();
}

}  // namespace mgp
