// mgp_kernels.cuh -- kernel launchers shared by the host drivers (mgp_host.cu)
// and the kernels (mgp_kernels.cu).
#pragma once
#include <cuda.h>

#include "mgp_core.cuh"

namespace mgp {

// Most blocks a reduction uses (4 per SM of a B200): launch_reduce's partials
// take two doubles per block.
constexpr int kRedBlocksMax = 592;

// Reduction kinds of launch_reduce.
enum RedKind { RED_SUMSQ = 0, RED_MAXABS = 1, RED_DOT = 2, RED_JSUM = 3, RED_ABSSUM = 4 };

// Values of a solver's device status word.  A kernel records the first error
// it meets and never overwrites one already there (set_status), so the host
// sees the cause, not a later consequence.
enum DevStatus {
    DST_OK = 0,
    DST_TIMEOUT = 2,      // a bounded device wait (TMA tile barrier, grid barrier) ran out
    DST_NONFINITE = 3,    // a non-finite residual in a device-side solve (bottom BiCGStab)
    DST_MISALIGNED = 4,   // the sweep's shared-memory window was not 128-byte aligned
};
#ifdef __CUDACC__
__device__ __forceinline__ void set_status(int* s, int v) {
    if (s && v) atomicCAS(s, 0, v);
}
#endif

// A grid barrier gives up after this long by default (%globaltimer
// nanoseconds): far above any real wait between two barriers of the coarse
// cycle (milliseconds at most).
constexpr unsigned long long kGridWaitNsDefault = 1000000000ull;

// Barrier and reduction partials of a cooperative grid running the
// coarse cycle (k_coarse_cycle_grid).
struct GridCtl {
    unsigned* bar;   // [0] arrivals, [1] generation; arrivals 0 at launch
    double* part;    // 2 x (CTAs) partial sums
    int* status;     // DST_TIMEOUT if a barrier wait gives up; once nonzero, barriers stop waiting
    unsigned long long wait_ns;   // a CTA's longest wait at one barrier
};

struct CoarseArgs {
    const Lv* lv;        // device array of levels
    int d0;              // level the cycle starts at (vcycle_noinit(d0) semantics)
    int maxdepth;
    int numcycles;
    int nd, nu, nb;      // smoothing counts
    int dd;              // 1: DeferredPoisson2D operators
    const int* refx;     // device arrays, maxdepth entries
    const int* refy;
    int* status;         // device int: 0 ok, nonzero = error code
    const Lv* shadow;    // device array: the levels' layout in shared memory (offsets), or nullptr
    int smem_bytes;      // dynamic shared memory the staged levels need
    const double* ainv;  // MGP_FLAG_DIRECT_COARSE: inverse of level maxdepth's operator, transposed, or nullptr
    int grid_ctas;       // > 1: run as a cooperative grid of this many CTAs (gctl set)
    int cluster;         // with grid_ctas > 1: the grid is one thread-block cluster (hardware barriers);
                         // 2: its reductions in the one-CTA kernel's order (the same bits)
    GridCtl gctl;
};

// Largest bottom level solved by its precomputed inverse (cells); b_direct
// gives each row four threads of the coarse CTA.
constexpr int kDirectCells = 64;
// Largest bottom of MGP_FLAG_DIRECT_LARGE (cells): the coarse-cycle level,
// solved by launch_direct_apply.
constexpr int kDirectLargeCells = 1024;
// Pivots per panel of the blocked device Gauss-Jordan (launch_invert); its
// scratch is 4 n^2 + 2 + (n + 1) kGjPanel doubles.
constexpr int kGjPanel = 16;

constexpr int kMaxCoarseLevels = 16;
// Largest staged coarse hierarchy (bytes of dynamic shared memory).
constexpr int kCoarseSmemMax = 200 * 1024;

// Parameters of the single-CTA BiCGStab (solve_bicgstab2).
struct BicgArgs {
    Lv L;
    DF phi, rhs;
    int homog;
    double tol;
    int max_iters, max_restarts, zerophi;
    int dd;
    int* status;
};

constexpr int kCoarseThreads = 256;
constexpr int kClusterThreads = 256;   // threads per CTA of the cluster coarse cycle

long long launch_count();
long long thread_launch_count();   // launches the calling thread made (count_launch on it)
void count_launch(int n = 1);

cudaError_t launch_fill(const DF& p, const Geo& g, const BCd& b, int homog, int do_neum, int nx, int ny,
                        cudaStream_t st);
cudaError_t launch_extrapolate(const DF& p, int nx, int ny, int ngx, int ngy, int order, cudaStream_t st);

// ---- FP32 grid levels of the mixed-precision V-cycle --------------------- //
cudaError_t launch_fill(const DF32& p, const Geo32& g, const BCd& b, int homog, int do_neum, int nx, int ny,
                        cudaStream_t st);
cudaError_t launch_apply(const DF32& out, const DF32& phi, const DF32& rhs, const Geo32& g, const BCd& b, int homog,
                         int nx, int ny, int mode, int jscale, cudaStream_t st);
// Cell-centred restriction into an FP32 or an FP64 coarse field.
cudaError_t launch_restrict(const DF32& f, const DF32& c, int ncx, int ncy, int refx, int refy, cudaStream_t st);
cudaError_t launch_restrict(const DF32& f, const DF& c, int ncx, int ncy, int refx, int refy, cudaStream_t st);
// Prolongation from an FP32 or an FP64 coarse field (arithmetic in the coarse type).
cudaError_t launch_prolong(const DF32& fine, const DF32& crse, int ncx, int ncy, int refx, int refy, int order,
                           cudaStream_t st);
cudaError_t launch_prolong(const DF32& fine, const DF& crse, int ncx, int ncy, int refx, int refy, int order,
                           cudaStream_t st);
cudaError_t launch_set_guess(const DF32& e, const DF32& r, const DF32& invd, int nx, int ny, cudaStream_t st);
// rc = restrict(rhs - L[phi]) onto the coarse cells, and with guess
// ec = rc * invdc: k_apply (mode 1), the cell restriction and k_set_guess in
// one pass, the same bits.  phi's ghosts must be filled.
cudaError_t launch_resid_restrict(const DF& phi, const DF& rhs, const Geo& g, const BCd& b, int homog, int nx, int ny,
                                  const DF& rc, const DF& ec, const DF& invdc, int ncx, int ncy, int refx, int refy,
                                  int guess, cudaStream_t st);
cudaError_t launch_resid_restrict(const DF32& phi, const DF32& rhs, const Geo32& g, const BCd& b, int homog, int nx,
                                  int ny, const DF32& rc, const DF32& ec, const DF32& invdc, int ncx, int ncy, int refx,
                                  int refy, int guess, cudaStream_t st);
cudaError_t launch_resid_restrict(const DF32& phi, const DF32& rhs, const Geo32& g, const BCd& b, int homog, int nx,
                                  int ny, const DF& rc, const DF& ec, const DF& invdc, int ncx, int ncy, int refx,
                                  int refy, int guess, cudaStream_t st);
cudaError_t launch_sub_mean(const DF32& y, const double* out, int nx, int ny, int gx, int gy, cudaStream_t st);
cudaError_t launch_reduce(int kind, const DF32& a, const DF32& b, int nx, int ny, double vol, double* partials,
                          double* out, cudaStream_t st);
// dst = src rounded to dst's type, over i in [-gx, nx+gx), j in [-gy, ny+gy).
cudaError_t launch_convert(const DF32& dst, const DF& src, int nx, int ny, int gx, int gy, cudaStream_t st);
cudaError_t launch_convert(const DF& dst, const DF32& src, int nx, int ny, int gx, int gy, cudaStream_t st);
cudaError_t launch_round_bf16(const DF32& f, int nx, int ny, int g, cudaStream_t st);
// mode: 0 lap, 1 rhs - lap; jscale divides lap by J first.
cudaError_t launch_apply(const DF& out, const DF& phi, const DF& rhs, const Geo& g, const BCd& b, int homog,
                         int nx, int ny, int mode, int jscale, cudaStream_t st);
cudaError_t launch_gs_sweep(const DF& phi, const DF& rhs, const DF& invd, const Geo& g, const BCd& b, int homog,
                            int nx, int ny, double omega, cudaStream_t st);
// One sweep in a single launch, reading pin and writing pout (mgp_sweep.cu).
// Sides must be DIRI, NEUM or PERIODIC (sweep_fusable).
bool sweep_fusable(const BCd& b);
// TMA descriptors of the seven fields one sweep stages; phi element (i,j) is
// map coordinate (i - pcb, j - prb), the operands' (i,j) is (i,j).
struct SweepMaps {
    CUtensorMap pin, rhs, invd, xx, xy, yx, yy;
    int pcb, prb;
};
// ---- lockstep batches -------------------------------------------------- //
// One launch runs the same phase of many problems.  Each launch has a job
// table and pre[0..njobs]: job k owns blocks [pre[k], pre[k + 1]) of a 1-D
// grid of pre[njobs] blocks (a block finds its job by binary search).
// One level's sweep: phi in buf[s0 ^ flip] (descriptors m[s0 ^ flip]),
// written to the other buffer.
template <class T>
struct alignas(64) SweepJobT {
    SweepMaps m[2];
    DFT<T> buf[2], rhs, invd;
    GeoT<T> g;
    BCd b;
    int4 part;   // (nx / gx, nx % gx, ny / gy, ny % gy)
    int nx, ny, gx, gy, s0;
};
// fill_ghosts of one field.
template <class T>
struct FillJob {
    DFT<T> p;
    GeoT<T> g;
    BCd b;
    int nx, ny, homog, do_neum;
};
// rc = restrict(rhs - L[phi]), ec = rc * invdc (k_resid_restrict); gbx blocks of 32 x 8 fine cells along x.
template <class T, class TC>
struct ResidJob {
    DFT<T> phi, rhs;
    GeoT<T> g;
    BCd b;
    DFT<TC> rc, ec, invdc;
    int nx, ny, ncx, ncy, refx, refy, gbx;
};
// fine += prolong(crse), order 1 (k_prolong); gbx blocks of 32 x 8 coarse cells along x.
template <class TF, class TC>
struct ProlongJob {
    DFT<TF> fine;
    DFT<TC> crse;
    int ncx, ncy, refx, refy, gbx;
};
// Cell-wise work on the valid region plus g ghost layers (k_cell_jobs: y + x,
// x converted to y's type, y - x, x * z).  gbx blocks of 32 x 8 along x.
template <class TD, class TS>
struct CellJob {
    DFT<TD> y;
    DFT<TS> x;
    DFT<TD> z;
    int nx, ny, g, gbx;
};
// r = rhs - L[phi] on level 0 (caller BCs) and the block's sum of r^2 into
// partials[block]; gbx blocks of 32 x 8 along x.
struct NormJob {
    DF phi, rhs, r;
    Geo g;
    BCd b;
    int nx, ny, homog, gbx;
};
// The coarse cycle of one problem (one CTA each; CoarseArgs with its shadow layout).
struct CoarseJob {
    CoarseArgs a;
};
// e = A^-1 r on a problem's exact bottom (MGP_FLAG_DIRECT_LARGE; k_direct_apply's blocks).
struct DirectJob {
    DF e, r;
    const double* ainv;
    int nx, ny;
};

// Descriptors for sweeping one level with phi in either of its two buffers.
struct SweepTma {
    SweepMaps ma, mb;
    const void *pa = nullptr, *pb = nullptr, *rhs = nullptr, *invd = nullptr, *xx = nullptr;
    int tx = 32;   // tile width the descriptors' boxes are cut for
    bool ok = false;
    SweepMaps ma2, mb2;   // boxes for two sweeps per launch (small FP32 levels)
    bool ok2 = false;
};
// Builds the descriptors when the arrays allow it (16-byte aligned bases and
// pitches, phi with a ghost layer and pitch >= nx + 3); else t->ok = false
// and the sweep stages with cp.async.
void sweep_tma_prepare(SweepTma* t, const DF& ea, const DF& eb, const DF& rhs, const DF& invd, const Geo& g, int nx,
                       int ny);
void sweep_tma_prepare(SweepTma* t, const DF32& ea, const DF32& eb, const DF32& rhs, const DF32& invd,
                       const Geo32& g, int nx, int ny);
// status (nullable) receives DST_TIMEOUT if a CTA's staging never completed,
// DST_MISALIGNED if the shared-memory window was not 128-byte aligned
// (neither is expected).
cudaError_t launch_sweep9(const DF& pin, const DF& pout, const DF& rhs, const DF& invd, const Geo& g, const BCd& b,
                          int homog, int nx, int ny, double omega, const SweepTma* tma, int* status,
                          cudaStream_t st);
cudaError_t launch_sweep9(const DF32& pin, const DF32& pout, const DF32& rhs, const DF32& invd, const Geo32& g,
                          const BCd& b, int homog, int nx, int ny, double omega, const SweepTma* tma, int* status,
                          cudaStream_t st);
// Two sweeps in one launch on a level whose descriptors allow it
// (sweep_pair_ok: small levels of 32-wide tiles, no periodic side): the
// result of two launch_sweep9 calls, bit for bit, written to pout.
bool sweep_pair_ok(const SweepTma* tma, const BCd& b);
cudaError_t launch_sweep9_pair(const DF32& pin, const DF32& pout, const DF32& rhs, const DF32& invd, const Geo32& g,
                               const BCd& b, int homog, int nx, int ny, double omega, const SweepTma* tma,
                               int* status, cudaStream_t st);
cudaError_t launch_sweep9_pair(const DF& pin, const DF& pout, const DF& rhs, const DF& invd, const Geo& g,
                               const BCd& b, int homog, int nx, int ny, double omega, const SweepTma* tma,
                               int* status, cudaStream_t st);
// Lockstep launches: jobs and pre in device memory (pre[njobs] blocks in all).
template <class T>
cudaError_t launch_sweep9_jobs(const SweepJobT<T>* jobs, const int* pre, int njobs, int nblocks, int tx, int k,
                               int flip, int* status, cudaStream_t st);
template <class T>
cudaError_t launch_fill_jobs(const FillJob<T>* jobs, const int* pre, int njobs, int nblocks, int phases,
                             cudaStream_t st);
template <class T, class TC>
cudaError_t launch_resid_jobs(const ResidJob<T, TC>* jobs, const int* pre, int njobs, int nblocks, cudaStream_t st);
template <class TF, class TC>
cudaError_t launch_prolong_jobs(const ProlongJob<TF, TC>* jobs, const int* pre, int njobs, int nblocks,
                                cudaStream_t st);
// kind 0: y = y + x; 1: y = x converted; 2: y = y - x; 3: y = x * z
template <class TD, class TS>
cudaError_t launch_cell_jobs(const CellJob<TD, TS>* jobs, const int* pre, int njobs, int nblocks, int kind,
                             cudaStream_t st);
// r = rhs - L[phi], then norms[k] = sqrt(vol_k * sum of job k's r^2) in block order (vol in volk).
cudaError_t launch_norm_jobs(const NormJob* jobs, const int* pre, int njobs, int nblocks, double* partials,
                             const double* volk, double* norms, cudaStream_t st);
cudaError_t launch_coarse_jobs(const CoarseJob* jobs, int njobs, int smem_bytes, cudaStream_t st);
int direct_apply_blocks(int nx, int ny);
cudaError_t launch_direct_jobs(const DirectJob* jobs, const int* pre, int njobs, int nblocks, cudaStream_t st);
cudaError_t launch_invdiag(const DF& invd, const Geo& g, const BCd& b, int homog, int nx, int ny, int coupled,
                           cudaStream_t st);
// kind: 0 cell, 1 x-face, 2 y-face, 3 node.  ncx/ncy = coarse cell counts.
cudaError_t launch_restrict(const DF& f, const DF& c, int ncx, int ncy, int refx, int refy, int kind,
                            cudaStream_t st);
// Constant, linear and (order 2) second-difference terms; crse ghosts must be filled.
cudaError_t launch_prolong(const DF& fine, const DF& crse, int ncx, int ncy, int refx, int refy, int order,
                           cudaStream_t st);
cudaError_t launch_prolong_cross(const DF& fine, const DF& crse, int ncx, int ncy, cudaStream_t st);
cudaError_t launch_set_guess(const DF& e, const DF& r, const DF& invd, int nx, int ny, cudaStream_t st);
cudaError_t launch_jacobi(const DF& phi, const DF& r, const DF& invd, double omega, int nx, int ny, cudaStream_t st);
// y[i,j] = a*y + b*x over i in [-gx, nx+gx), j in [-gy, ny+gy).
// A set of vectors for GMRES: vector k at p + k * stride, cell (i,j) at [i + j * ld].
struct MVec {
    double* p;
    int ld;
    long stride;
};
// out[k] = sum over valid cells of w * v_k, k < nv (partials: nb * nv doubles).
cudaError_t launch_mdot(const DF& w, const MVec& V, int nv, int nx, int ny, double* partials, int nb, double* out,
                        cudaStream_t st);
// One classical Gram-Schmidt pass: h[k] = w . v_k (k < nv), w -= sum_k h[k] v_k,
// then *hnorm = |w|^2.  partials holds cap doubles; cudaErrorNotSupported
// when the pass's partial sums would not fit (the caller then uses
// launch_mdot and launch_maxpy).
cudaError_t launch_gs_pass(const DF& w, const MVec& V, int nv, int nx, int ny, double* partials, long cap, int nb,
                           double* h, double* hnorm, cudaStream_t st);
// w += sign * sum_{k < nv} coef[k] v_k (coef in device memory).
cudaError_t launch_maxpy(const DF& w, const MVec& V, int nv, const double* coef, double sign, int nx, int ny,
                         cudaStream_t st);
cudaError_t launch_axpby(const DF& y, const DF& x, double a, double b, int nx, int ny, int gx, int gy,
                         cudaStream_t st);
// y = y * x (mul=1) or y / x (mul=0) over the valid region.
cudaError_t launch_muldiv(const DF& y, const DF& x, int mul, int nx, int ny, cudaStream_t st);
cudaError_t launch_fillval(const DF& y, double v, int nx, int ny, int gx, int gy, cudaStream_t st);
cudaError_t launch_sub_mean(const DF& y, const double* out, int nx, int ny, int gx, int gy, cudaStream_t st);
// Reduction over the valid region into out[0] (and out[1] for RED_JSUM: volume).
cudaError_t launch_reduce(int kind, const DF& a, const DF& b, int nx, int ny, double vol, double* partials,
                          double* out, cudaStream_t st);
// Gradient and divergence (compute_pd, compute_grad, compute_div,
// fill_boundary_fluxes); phi's ghosts filled by the caller.
cudaError_t launch_pd(const DF& pd, const DF& phi, int nx, int ny, double dx, double dy, int dir, int nodedir,
                      cudaStream_t st);
cudaError_t launch_grad(const DF& xflux, const DF& yflux, const DF& phi, const Geo& g, const BCd& b, int homog,
                        int nx, int ny, cudaStream_t st);
cudaError_t launch_boundary_fluxes(const DF& xflux, const DF& yflux, const BCd& b, int homog, int nx, int ny,
                                   cudaStream_t st);
cudaError_t launch_div(const DF& div, const DF& xflux, const DF& yflux, int nx, int ny, double dx, double dy,
                       cudaStream_t st);
// Deferred-correction operators.
cudaError_t launch_dd_invdiag(const DF& invd, const Geo& g, int nx, int ny, cudaStream_t st);
cudaError_t launch_dd_apply(const DF& out, const DF& phi, const DF& rhs, const Geo& g, const BCd& b, int nx, int ny,
                            int mode, cudaStream_t st);
cudaError_t launch_dd_modrhs(const DF& out, const DF& phi, const DF& rhs, const Geo& g, int nx, int ny,
                             cudaStream_t st);
cudaError_t launch_dd_colour(const DF& phi, const DF& modrhs, const DF& invd, const Geo& g, int nx, int ny,
                             double omega, int colour, cudaStream_t st);
// The same three on FP32 fields (the grid levels of a mixed-precision DD V-cycle).
cudaError_t launch_dd_apply(const DF32& out, const DF32& phi, const DF32& rhs, const Geo32& g, const BCd& b, int nx,
                            int ny, int mode, cudaStream_t st);
cudaError_t launch_dd_modrhs(const DF32& out, const DF32& phi, const DF32& rhs, const Geo32& g, int nx, int ny,
                             cudaStream_t st);
cudaError_t launch_dd_colour(const DF32& phi, const DF32& modrhs, const DF32& invd, const Geo32& g, int nx, int ny,
                             double omega, int colour, cudaStream_t st);
// Per-device kernel attributes (idempotent; call before any stream capture).
cudaError_t sweep_kernels_init();
cudaError_t coarse_kernels_init();
// Single-CTA kernels.
cudaError_t launch_coarse_cycle(const CoarseArgs& a, cudaStream_t st);
// Largest cooperative grid of the coarse cycle the current device keeps resident (0: none).
int coarse_grid_ctas_max();
int coarse_cluster_ctas_max();
// A cooperative grid of nctas CTAs (all resident) passing nbar grid barriers;
// CTA `skip` (if >= 0) exits before the first one, so the others' waits run
// out.  Exercises the bounded wait of the coarse cycle's grid barrier.
cudaError_t launch_barrier_selftest(const GridCtl& g, int nctas, int skip, int nbar, cudaStream_t st);
int barrier_selftest_ctas_max();
// A[m * n + k] = (L e_k)_m for the level's operator with homogeneous BCs
// (n = nx * ny columns, one CTA each; scratch holds 2 n fields of
// (nx + 2) x (ny + 2)).
cudaError_t launch_direct_columns(const Lv& L, double* scratch, double* A, cudaStream_t st);
// Inverse of the n x n row-major A by Gauss-Jordan elimination with partial
// pivoting on the device, into ainv (row-major, may alias A).  work holds
// 4 n^2 + 2 + (n + 1) kGjPanel doubles (16-byte aligned), iwork 2 n + 1 ints;
// *fail (in iwork) ends nonzero when a pivot fell below 1e-13 of the largest
// |A| entry (singular to working precision).  Launches 2 n / kGjPanel + 2
// kernels.
cudaError_t launch_invert(const double* A, int n, double* ainv, double* work, int* iwork, cudaStream_t st);
// e = ainv r on the level's cells (n = nx * ny <= kDirectLargeCells; cells
// numbered i fastest), one warp per row.
cudaError_t launch_direct_apply(const DF& e, const DF& r, const double* ainv, int nx, int ny, cudaStream_t st);
cudaError_t launch_bicgstab(const BicgArgs& a, cudaStream_t st);
cudaError_t launch_relax_block(const Lv& L, const DF& phi, const DF& rhs, int homog, double omega, int sweeps,
                               int dd, int* status, cudaStream_t st);

}  // namespace mgp
