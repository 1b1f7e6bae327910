// mgp_sweep.cu -- one Gauss-Seidel sweep of the mapped 9-point operator in a
// single launch (relax_gs, poisson2d.f90:1460-1988, in the device order).
//
// The sweep reads phi from `pin` and writes the swept field to `pout` (two
// buffers), so no CTA ever reads a value another CTA has already replaced.
// Each CTA owns one tile of a balanced partition of the grid (tiles at most
// TX x TY and, when there is more than one, at least TX/2 x TY/2, so every
// corner's neighbourhood lies inside the tile that owns the corner: with
// g = ceil(n / TX) tiles along a side, n / g lies in [TX/2, TX] for n > TX
// and equals TX only when g divides n).
//
// A CTA first stages everything its tile's update reads -- phi with its
// halo, rhs, the inverse diagonal and the four metric face arrays, each on
// exactly the region the sub-passes touch -- into shared memory with
// coalesced loads, applies the sweep-start ghost fill there (P2:1556), then
// runs the sweep's sub-passes from shared memory only, on shrinking regions:
//   * the four colours (0,0),(1,1),(1,0),(0,1) over interior cells -- the
//     stencil reaches one cell, so pass c is exact on the tile grown by
//     (3 - c + E) cells;
//   * on tiles that touch a non-periodic side, the boundary pass: edge cells
//     colour by colour (away from corners a colour along an edge reads only
//     neighbours of the colour updated just before it, so one extra cell of
//     halo suffices, E = 2), then the four corners in turn.
// The halo cells are recomputed by every CTA that needs them, with the same
// operations in the same order, so the result is bit-identical to running the
// sub-passes over the whole grid one after another.  The same argument lets
// one launch run K sweeps (K = 2 on small levels, whose sweeps last about
// one CTA's latency): with a halo of K times the one-sweep halo, sweep s of K
// works on the tile grown by (K - 1 - s)(4 + E) cells, and the tile comes out
// as after K launches, bit for bit.
//
// Staging: on the solver's own arrays (aligned, with spare columns) one
// thread issues seven TMA tile loads (five on the wide FP32 tiles;
// cp.async.bulk.tensor.2d) of the CTA's
// window of each field, completing on one mbarrier; elsewhere (caller arrays
// of any pitch and alignment) the threads stage with cp.async.
//
// The kernel is compiled for FP64 fields (the solver's arithmetic; the
// update is gs9's, bit for bit) and for FP32 fields (the grid levels of the
// mixed-precision V-cycle), where each thread updates two interior cells at
// once in packed FP32x2 arithmetic with fused multiply-adds (gs9_pair).  The
// result depends on neither the tiling nor the launch: the same inputs give
// the same bits.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "mgp_kernels.cuh"

namespace mgp {

namespace {

constexpr int kTY = 32;
constexpr int kH1 = 6;   // phi halo of one sweep: 4 for the colour passes + E = 2 for the boundary pass
// A CTA gives up on its tile loads after kWaitLimit polls or kWaitNs, far
// above any real wait (microseconds); each poll sleeps up to kSuspendNs.
constexpr long kWaitLimit = 1L << 22;
constexpr unsigned long long kWaitNs = 200000000ull;
constexpr unsigned kSuspendNs = 20000;

// Tile and shared-memory window of one field type and tile width: 32 x 32
// tiles (FP64: two CTAs of 114 KB per SM; FP32: three of 59 KB) and, for
// FP32 levels large enough to fill the GPU, 64 x 32 tiles, which spread each
// thread's fixed work over more cells and recompute a smaller share of halo.
// The wide tiles stage five arrays, not seven: rhs and the inverse diagonal,
// read once per update and only at the updated cell, come from global memory
// there, so the window (70 KB) leaves room for three CTAs per SM -- a tile's
// colour passes are latency-bound, and more CTAs in flight hide it.  All
// staged arrays share one
// window -- origin (pox, poy) with pox the column at or below tile corner - kH
// that is a multiple of kAlign (a 16-byte boundary, as TMA needs), pitch PW --
// so one offset addresses a cell in every array: phi and the cell operands
// at o, the west/east x-faces at o and o + 1, the south/north y-faces at o
// and o + PW.  The operands are needed on tile + (3 + E) <= tile + 5 cells
// (faces one further), inside the phi footprint tile + kH.
template <class T, int TX_, int K_ = 1>
struct Win {
    static constexpr int TX = TX_;
    static constexpr int kH = K_ * kH1;   // phi halo of K_ sweeps per launch
    static constexpr int kAlign = 16 / (int)sizeof(T);   // 2 doubles, 4 floats
    static constexpr int PW = (TX + 2 * kH + (kAlign - 1) + kAlign - 1) / kAlign * kAlign;   // 46 / 48 / 80
    static constexpr int PH = kTY + 2 * kH;                                                        // 44
    static constexpr int kA = (PW * PH * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);     // 128-B aligned
    static constexpr bool kRI = !(sizeof(T) == 4 && TX_ == 64);   // rhs and inverse diagonal staged
    static constexpr int NA = kRI ? 7 : 5;                          // staged arrays
    static constexpr int oF = kA, oD = 2 * kA;                      // (when kRI)
    static_assert(oD == oF + kA, "rhs and inverse diagonal adjacent");
    static constexpr int oXX = (kRI ? 3 : 1) * kA, oXY = oXX + kA, oYX = oXX + 2 * kA, oYY = oXX + 3 * kA;
    static constexpr int oBarBytes = NA * kA * (int)sizeof(T);   // the TMA mbarrier (8 bytes)
    static constexpr size_t kSmemBytes = (size_t)oBarBytes + 16;
    static constexpr unsigned kBoxBytes = PW * PH * sizeof(T);
    // threads: the wide tiles' colour passes hold 256 to 333 cell pairs (up to
    // 389 on tiles at the domain edge), so 12 warps cover them, and three
    // CTAs of 384 threads leave 56 registers a thread
    static constexpr int kThreads = kRI ? 512 : 384;
    static_assert(K_ == 1 || TX_ == 32, "two sweeps per launch: 32-wide tiles only");
    // CTAs per SM the window and the thread count allow
    static constexpr int kMinBlocks = (int)((228 * 1024) / (kSmemBytes + 1024)) < 2048 / kThreads
                                          ? (int)((228 * 1024) / (kSmemBytes + 1024))
                                          : 2048 / kThreads;
};

static_assert(Win<double, 32>::PW == 46 && Win<float, 32>::PW == 48 && Win<float, 64>::PW == 80, "window pitch");
static_assert(Win<double, 32>::kMinBlocks == 2 && Win<float, 32>::kMinBlocks == 3 && Win<float, 64>::kMinBlocks == 3,
              "CTAs per SM");
static_assert(Win<float, 32, 2>::PW == 60 && Win<float, 32, 2>::PH == 56 && Win<float, 32, 2>::kMinBlocks == 2,
              "two-sweep window");
static_assert(Win<double, 32, 2>::PW == 58 && Win<double, 32, 2>::kMinBlocks == 1, "two-sweep FP64 window");

template <class T>
struct SLoadT {
    const T* c;
    int ld;
    __device__ __forceinline__ T operator()(int di, int dj) const { return c[di + dj * ld]; }
};

// phi at the start of the sweep: the staged copy where it holds (i,j), else
// global memory (the far side of a periodic domain).
template <class T, int PW>
struct PinLoad {
    const T* s;
    int pox, poy, pi0, pi1, pj0, pj1;
    DFT<T> pin;
    __device__ __forceinline__ T operator()(int i, int j) const {
        if (i >= pi0 && i < pi1 && j >= pj0 && j < pj1) return s[(j - poy) * PW + (i - pox)];
        return AT(pin, i, j);
    }
};

// Copy rows [j0,j1) x columns [i0,i1) of a global field into a shared array
// whose (0,0) is cell (ox, oy) and whose row pitch is w.  Warp w8 takes rows
// j0 + w8, j0 + w8 + 8, ...; where a row's global and shared addresses have
// the same 16-byte phase its lanes copy pairs of doubles, else single ones.
__device__ __forceinline__ void stage(double* s, int w, int ox, int oy, const DF& f, int i0, int i1, int j0, int j1) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(s);
    for (int j = j0 + warp; j < j1; j += nw) {
        const double* g = f.p + (long)j * f.ld + i0;
        unsigned sa = sbase + (unsigned)(((j - oy) * w + (i0 - ox)) * 8);
        const int n = i1 - i0;
        if (n <= 0) continue;
        if (((unsigned)(uintptr_t)g ^ sa) & 8) {
            for (int k = lane; k < n; k += 32) cp_async8s(sa + 8 * k, g + k);
            continue;
        }
        int k0 = 0;
        if (sa & 8) {   // leading single
            if (lane == 0) cp_async8s(sa, g);
            k0 = 1;
        }
        const int np = (n - k0) >> 1;
        for (int k = lane; k < np; k += 32) cp_async16s(sa + 8 * (k0 + 2 * k), g + k0 + 2 * k);
        if (((n - k0) & 1) && lane == 31) cp_async8s(sa + 8 * (n - 1), g + n - 1);   // trailing single
    }
}

// The same for FP32 fields, one element per copy.
__device__ __forceinline__ void stage(float* s, int w, int ox, int oy, const DF32& f, int i0, int i1, int j0, int j1) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(s);
    for (int j = j0 + warp; j < j1; j += nw) {
        const float* g = f.p + (long)j * f.ld + i0;
        const unsigned sa = sbase + (unsigned)(((j - oy) * w + (i0 - ox)) * 4);
        for (int k = lane; k < i1 - i0; k += 32)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa + 4 * k), "l"(g + k));
    }
}

// ---- TMA staging ---------------------------------------------------------- //
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
// Test phase `parity`; a thread whose phase is not complete sleeps in the
// instruction until it completes or kSuspendNs pass.
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for phase 0 of the barrier (kWaitLimit polls and kWaitNs at
// most); false if it did not complete.  Between polls the warp sleeps, 32 ns
// at first and at most 256 ns, so a CTA waiting for its tile takes few issue
// slots from the CTAs computing beside it.
__device__ __forceinline__ bool mbar_wait0(unsigned bar) {
    const unsigned long long t0 = global_ns();
    unsigned nap = 32;
    for (long k = 0; k < kWaitLimit; ++k) {
        if (mbar_try_wait(bar, 0)) return true;
        if (global_ns() - t0 > kWaitNs) break;
        __nanosleep(nap);
        nap = nap < 256 ? 2 * nap : nap;
    }
    return false;
}
// Programmatic dependent launch: a grid launched with the programmatic
// serialization attribute may start before the grid ahead of it in the stream
// has finished; griddepcontrol.wait returns once that grid has completed and
// its writes are visible (at once when there is none), and launch_dependents
// lets the next such grid start as SM resources free up.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// One 2-D tile (the map's box) of `map` at element coordinates (x, y); x is a
// multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
        ::"r"(dst), "l"((unsigned long long)map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Interior colour c on the tile grown by (3 - c + E + G), G the extra grow of
// an early sweep of a multi-sweep launch: first cell (ci0, cj0), cw cells
// per row, n cells, and the magic number for k / cw (n <= 37 x 25 and cw <=
// 37, well inside the exact range of the 24-bit multiply).  Lane
// c of each group of four computes colour c; every lane then reads all four
// by shuffle, so a warp spends one divide, not four per thread.
__device__ __forceinline__ void colour_ranges(int X0, int X1, int Y0, int Y1, int E, int G, int mi0, int mi1,
                                              int mj0, int mj1, int* ci0, int* cj0, int* ccw, int* cn, unsigned* cm) {
    const int c = threadIdx.x & 3;
    const int grow = 3 - c + E + G;
    int i0 = max(X0 - grow, mi0), i1 = min(X1 + grow, mi1);
    int j0 = max(Y0 - grow, mj0), j1 = min(Y1 + grow, mj1);
    i0 += (i0 & 1) != colour_ci(c);
    j0 += (j0 & 1) != colour_cj(c);
    const int cw = (i1 - i0 + 1) / 2, ch = (j1 - j0 + 1) / 2;
    const int n = (cw > 0 && ch > 0) ? cw * ch : 0;
    const unsigned m = fastdiv24_magic(cw > 0 ? cw : 1);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        ci0[k] = __shfl_sync(0xffffffffu, i0, k);
        cj0[k] = __shfl_sync(0xffffffffu, j0, k);
        ccw[k] = __shfl_sync(0xffffffffu, cw, k);
        cn[k] = __shfl_sync(0xffffffffu, n, k);
        cm[k] = __shfl_sync(0xffffffffu, m, k);
    }
}

template <class T>
struct Tile {
    T* s;   // seven arrays of PW x PH, origin (pox, poy)
    int pox, poy;
};

// One Gauss-Seidel update of (i,j) from shared memory (same operations as gs9).
// f and d are rhs and the inverse diagonal at (i,j).
template <class W, class T>
__device__ __forceinline__ void gs9_tile(const Tile<T>& t, T idx, T idy, const BCd& b, int homog, int i, int j, int xr,
                                         int yr, T om, T om1, T f, T d) {
    T* c = t.s + (j - t.poy) * W::PW + (i - t.pox);
    St9T<T> s;
    gather9(SLoadT<T>{c, W::PW}, xr, yr, s);
    FacesT<T> fc;
    fc.xxw = c[W::oXX]; fc.xxe = c[W::oXX + 1];
    fc.xyw = c[W::oXY]; fc.xye = c[W::oXY + 1];
    fc.yys = c[W::oYY]; fc.yyn = c[W::oYY + W::PW];
    fc.yxs = c[W::oYX]; fc.yxn = c[W::oYX + W::PW];
    const T lphi = lap9f(s, fc, idx, idy, i, j, xr, yr, b, homog);
    const T p = c[0];
    const T newphi = p + (f - lphi) * d;
    c[0] = om * newphi + om1 * p;
}

// Two interior updates at once in packed FP32 arithmetic (add / mul / fma on
// a pair of floats, one instruction for both lanes): cells a and b of the
// same colour, each lane the operations of gs9_tile on an interior cell in
// the same order, except that the seven places where a product is added to
// another term -- each flux's two terms, the operator's x and y parts, the
// update p + (f - Lp) d and the relaxation om new + om1 p -- are fused
// multiply-adds, rounded once.  (The code generator fuses packed multiplies
// into adds on its own; writing the fused form makes the arithmetic defined
// by the source.)  Differences are a + b * (-1): an exact product and one
// rounding, the same as a - b.  Where the colour has an odd number of cells
// the last thread's b is a itself and only a is written back.
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

// f and d hold rhs and the inverse diagonal at the two cells.
template <class W>
__device__ __forceinline__ void gs9_pair(float* a, float* b, bool write_b, float2 f, float2 d, float2 idx, float2 idy,
                                         float2 om, float2 om1) {
    constexpr int P = W::PW;
    const auto L = [a, b](int o) { return make_float2(a[o], b[o]); };
    const float2 p = L(0), pe = L(1), pw = L(-1), pn = L(P), ps = L(-P);
    const float2 ene = L(1 + P), enw = L(-1 + P), ese = L(1 - P), esw = L(-1 - P);
    const float2 q = make_float2(0.25f, 0.25f);
    // interior cell: ee = pe, ew = pw, en = pn, es = ps (lap9f's four fluxes)
    const float2 xfe = f2fma(f2mul(L(W::oXX + 1), f2sub(pe, p)), idx,
                             f2mul(f2mul(f2mul(L(W::oXY + 1), q), f2sub(f2add(f2sub(ene, ese), pn), ps)), idy));
    const float2 xfw = f2fma(f2mul(L(W::oXX), f2sub(p, pw)), idx,
                             f2mul(f2mul(f2mul(L(W::oXY), q), f2sub(f2add(f2sub(pn, ps), enw), esw)), idy));
    const float2 yfn = f2fma(f2mul(L(W::oYY + P), f2sub(pn, p)), idy,
                             f2mul(f2mul(f2mul(L(W::oYX + P), q), f2sub(f2add(f2sub(ene, enw), pe), pw)), idx));
    const float2 yfs = f2fma(f2mul(L(W::oYY), f2sub(p, ps)), idy,
                             f2mul(f2mul(f2mul(L(W::oYX), q), f2sub(f2add(f2sub(pe, pw), ese), esw)), idx));
    const float2 lphi = f2fma(f2sub(xfe, xfw), idx, f2mul(f2sub(yfn, yfs), idy));
    const float2 newphi = f2fma(f2sub(f, lphi), d, p);
    const float2 r = f2fma(om, newphi, f2mul(om1, p));
    a[0] = r.x;
    if (write_b) b[0] = r.y;
}

// The sweep of tile (bx, by) of a level, by one CTA (the body of k_sweep9
// and of the lockstep batch's k_sweep9_jobs).  m and b may live in kernel
// parameter space or in global memory.
template <bool kTma, class T, int TX, int K>
__device__ __forceinline__ void sweep_tile(const SweepMaps& m, const DFT<T>& pin, const DFT<T>& pout,
                                           const DFT<T>& rhs, const DFT<T>& invd, const GeoT<T>& g, const BCd& b,
                                           int homog, int nx, int ny, int4 part, double omega, int* status, int bx,
                                           int by) {
    using W = Win<T, TX, K>;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    // tile bounds: part = (nx / gx, nx % gx, ny / gy, ny % gy); the first
    // nx % gx columns of tiles are one cell wider
    const int X0 = bx * part.x + min(bx, part.y), X1 = X0 + part.x + (bx < part.y ? 1 : 0);
    const int Y0 = by * part.z + min(by, part.w), Y1 = Y0 + part.z + (by < part.w ? 1 : 0);
    const Per pr = periodic_of(b);
    const bool edge_tile = (!pr.xl && X0 == 0) || (!pr.xh && X1 >= nx) || (!pr.yl && Y0 == 0) || (!pr.yh && Y1 >= ny);
    const int E = edge_tile ? 2 : 0;
    const T idx = T(g.idx), idy = T(g.idy);
    const T om = T(omega), om1 = T(1.0 - omega);
    Tile<T> t;
    t.s = smem;
    t.pox = (X0 - W::kH) & ~(W::kAlign - 1);
    t.poy = Y0 - W::kH;
    // one scalar update, rhs and the inverse diagonal from the window or global memory
    const auto gs = [&](int i, int j, int xr, int yr) {
        T f, d;
        if constexpr (W::kRI) {
            const int o = (j - t.poy) * W::PW + (i - t.pox);
            f = t.s[o + W::oF];
            d = t.s[o + W::oD];
        } else {
            f = AT(rhs, i, j);
            d = AT(invd, i, j);
        }
        gs9_tile<W>(t, idx, idy, b, homog, i, j, xr, yr, om, om1, f, d);
    };

    // interior colour ranges (i in [mi0, mi1), j in [mj0, mj1)) on shrinking
    // regions, and their divide-free index maps, set up while the loads fly
    const int mi0 = pr.xl ? 0 : 1, mi1 = pr.xh ? nx : nx - 1;
    const int mj0 = pr.yl ? 0 : 1, mj1 = pr.yh ? ny : ny - 1;
    int ci0[4], cj0[4], ccw[4], cn[4];
    unsigned cm[4];

    // 1. stage phi on tile + (4 + E) and the operands on tile + (3 + E)
    // (the first of K sweeps works on the tile grown by G0 = (K - 1)(4 + E))
    const int G0 = (K - 1) * (4 + E);
    const int hp = G0 + 4 + E, hc = G0 + 3 + E;
    const int pi0 = max(X0 - hp, -1), pi1 = min(X1 + hp, nx + 1), pj0 = max(Y0 - hp, -1), pj1 = min(Y1 + hp, ny + 1);
    const int ci0s = max(X0 - hc, 0), ci1s = min(X1 + hc, nx), cj0s = max(Y0 - hc, 0), cj1s = min(Y1 + hc, ny);
    if (kTma) {
        // the whole window of every array; what lies outside a field reads as 0 and is never used
        const unsigned sb = (unsigned)__cvta_generic_to_shared(smem), bar = sb + W::oBarBytes;
        constexpr unsigned kS = sizeof(T);
        if (sb & 127) {   // TMA destinations must be 128-byte aligned
            if (threadIdx.x == 0) set_status(status, DST_MISALIGNED);
            return;
        }
        if (threadIdx.x == 0) mbar_init(bar, 1);
        __syncthreads();
        // The descriptors exist only for a solver's own arrays, whose faces
        // and inverse diagonal do not change during a solve: their tiles are
        // requested before the wait for the previous grid (the solver
        // launches these sweeps as programmatic dependents of the kernel
        // before them), phi and rhs after it.
        if (threadIdx.x == 0) {
            mbar_expect_tx(bar, W::NA * W::kBoxBytes);
            if constexpr (W::kRI) tma_load_2d(sb + W::oD * kS, &m.invd, t.pox, t.poy, bar);
            tma_load_2d(sb + W::oXX * kS, &m.xx, t.pox, t.poy, bar);
            tma_load_2d(sb + W::oXY * kS, &m.xy, t.pox, t.poy, bar);
            tma_load_2d(sb + W::oYX * kS, &m.yx, t.pox, t.poy, bar);
            tma_load_2d(sb + W::oYY * kS, &m.yy, t.pox, t.poy, bar);
        }
        grid_dependency_wait();
        if (threadIdx.x == 0) {
            tma_load_2d(sb, &m.pin, t.pox - m.pcb, t.poy - m.prb, bar);
            if constexpr (W::kRI) tma_load_2d(sb + W::oF * kS, &m.rhs, t.pox, t.poy, bar);
        }
        colour_ranges(X0, X1, Y0, Y1, E, G0, mi0, mi1, mj0, mj1, ci0, cj0, ccw, cn, cm);
        // one warp polls the barrier; the others sleep in the block barrier
        // instead of taking issue slots from the CTAs that are computing
        const bool landed = threadIdx.x >= 32 || mbar_wait0(bar);
        if (!__syncthreads_and(landed)) {   // never seen; leave the tile unwritten and report
            if (threadIdx.x == 0) {
                set_status(status, DST_TIMEOUT);
                mbar_wait0(bar);   // let copies still in flight land before the CTA exits
            }
            return;
        }
    } else {
        grid_dependency_wait();
        stage(smem, W::PW, t.pox, t.poy, pin, pi0, pi1, pj0, pj1);
        if constexpr (W::kRI) {
            stage(smem + W::oF, W::PW, t.pox, t.poy, rhs, ci0s, ci1s, cj0s, cj1s);
            stage(smem + W::oD, W::PW, t.pox, t.poy, invd, ci0s, ci1s, cj0s, cj1s);
        }
        stage(smem + W::oXX, W::PW, t.pox, t.poy, g.xx, ci0s, ci1s + 1, cj0s, cj1s);
        stage(smem + W::oXY, W::PW, t.pox, t.poy, g.xy, ci0s, ci1s + 1, cj0s, cj1s);
        stage(smem + W::oYX, W::PW, t.pox, t.poy, g.yx, ci0s, ci1s, cj0s, cj1s + 1);
        stage(smem + W::oYY, W::PW, t.pox, t.poy, g.yy, ci0s, ci1s, cj0s, cj1s + 1);
        colour_ranges(X0, X1, Y0, Y1, E, G0, mi0, mi1, mj0, mj1, ci0, cj0, ccw, cn, cm);
        cp_async_wait_all();
        __syncthreads();
    }
    // 2.-4. once per sweep.  Sweep s of K works on the tile grown by
    //    G = (K - 1 - s)(4 + E): what the next sweep reads of it (tile +
    //    G) comes out exact, as the halo argument above gives for one sweep.
    for (int sw = 0; sw < K; ++sw) {
        const int G = (K - 1 - sw) * (4 + E);
        if (sw > 0) colour_ranges(X0, X1, Y0, Y1, E, G, mi0, mi1, mj0, mj1, ci0, cj0, ccw, cn, cm);
        // 2. sweep-start ghost fill on the staged ghost cells (the ghost rows and
        //    columns of tiles on the domain boundary only), on the sweep's footprint
        const int qi0 = max(X0 - (G + 4 + E), -1), qi1 = min(X1 + G + 4 + E, nx + 1);
        const int qj0 = max(Y0 - (G + 4 + E), -1), qj1 = min(Y1 + G + 4 + E, ny + 1);
        if (qi0 < 0 || qi1 > nx || qj0 < 0 || qj1 > ny) {
            const PinLoad<T, W::PW> P{smem, t.pox, t.poy, pi0, pi1, pj0, pj1, pin};
            const int lw = qi1 - qi0, lh = qj1 - qj0;
            for (int k = threadIdx.x; k < 2 * (lw + lh); k += blockDim.x) {
                int i, j;
                if (k < lw) { i = qi0 + k; j = qj0; }
                else if (k < 2 * lw) { i = qi0 + k - lw; j = qj1 - 1; }
                else if (k < 2 * lw + lh) { i = qi0; j = qj0 + k - 2 * lw; }
                else { i = qi1 - 1; j = qj0 + k - 2 * lw - lh; }
                if (i >= 0 && i < nx && j >= 0 && j < ny) continue;
                smem[(j - t.poy) * W::PW + (i - t.pox)] = sweep_ghost(P, b, homog, nx, ny, i, j);
            }
        }
        __syncthreads();

        // 3. interior colour passes on shrinking regions.  Interior cells are
        //    i in [mi0, mi1), j in [mj0, mj1) (a pass has at most 21 x 21 of them
        //    on a 32 x 32 tile, 37 x 21 on a 64 x 32 one).  FP64: a thread per
        //    cell.  FP32: a thread per two cells, k and k + ceil(n/2) of the
        //    colour's list, so a warp's lanes still read consecutive cells of the
        //    colour (two-way bank conflicts, as one cell per thread).
        if constexpr (sizeof(T) == 4) {
            const float2 idx2 = make_float2(idx, idx), idy2 = make_float2(idy, idy);
            const float2 om2 = make_float2(om, om), om12 = make_float2(om1, om1);
    #pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int nh = (cn[c] + 1) >> 1;
                for (int k = threadIdx.x; k < nh; k += blockDim.x) {
                    const int kb = (k + nh < cn[c]) ? k + nh : k;
                    const int ja = fastdiv24(k, cm[c]), jb = fastdiv24(kb, cm[c]);
                    const int ia = ci0[c] + 2 * (k - ja * ccw[c]), ib = ci0[c] + 2 * (kb - jb * ccw[c]);
                    T* ca = t.s + (cj0[c] + 2 * ja - t.poy) * W::PW + (ia - t.pox);
                    T* cb = t.s + (cj0[c] + 2 * jb - t.poy) * W::PW + (ib - t.pox);
                    float2 f2, d2;
                    if constexpr (W::kRI) {
                        f2 = make_float2(ca[W::oF], cb[W::oF]);
                        d2 = make_float2(ca[W::oD], cb[W::oD]);
                    } else {
                        const long ra = cj0[c] + 2 * ja, rb = cj0[c] + 2 * jb;
                        const long ga = ra * rhs.ld + ia, gb = rb * rhs.ld + ib;
                        const long ha = ra * invd.ld + ia, hb = rb * invd.ld + ib;
                        f2 = make_float2(__ldg(rhs.p + ga), __ldg(rhs.p + gb));
                        d2 = make_float2(__ldg(invd.p + ha), __ldg(invd.p + hb));
                    }
                    gs9_pair<W>(ca, cb, kb != k, f2, d2, idx2, idy2, om2, om12);
                }
                __syncthreads();
            }
        } else {
    #pragma unroll
            for (int c = 0; c < 4; ++c) {
                for (int k = threadIdx.x; k < cn[c]; k += blockDim.x) {
                    const int kj = fastdiv24(k, cm[c]);
                    const int i = ci0[c] + 2 * (k - kj * ccw[c]), j = cj0[c] + 2 * kj;
                    gs(i, j, RMID, RMID);
                }
                __syncthreads();
            }
        }

        // 4. boundary pass (edge tiles only; uniform per CTA): per colour, the
        //    edge cells of that colour along each non-periodic side within the
        //    tile grown by G + 1, then the corners in turn
        if (edge_tile) {
            const int ei0 = max(X0 - 1 - G, mi0), ei1 = min(X1 + 1 + G, mi1);
            const int ej0 = max(Y0 - 1 - G, mj0), ej1 = min(Y1 + 1 + G, mj1);
            const bool sxl = !pr.xl && X0 == 0, sxh = !pr.xh && X1 >= nx;
            const bool syl = !pr.yl && Y0 == 0, syh = !pr.yh && Y1 >= ny;
            for (int c = 0; c < 4; ++c) {
                const int ci = colour_ci(c), cj = colour_cj(c);
                const int ia = ei0 + ((ei0 & 1) != ci), ja = ej0 + ((ej0 & 1) != cj);
                const int ni = (ei1 > ia) ? (ei1 - ia + 1) / 2 : 0, nj = (ej1 > ja) ? (ej1 - ja + 1) / 2 : 0;
                const int n0 = (syl && cj == 0) ? ni : 0;
                const int n1 = n0 + ((syh && ((ny - 1) & 1) == cj) ? ni : 0);
                const int n2 = n1 + ((sxl && ci == 0) ? nj : 0);
                const int n3 = n2 + ((sxh && ((nx - 1) & 1) == ci) ? nj : 0);
                if (n3 == 0) continue;   // no cell of this colour on the tile's sides (uniform per CTA): no barrier
                for (int k = threadIdx.x; k < n3; k += blockDim.x) {
                    if (k < n0) gs(ia + 2 * k, 0, RMID, RLO);
                    else if (k < n1) gs(ia + 2 * (k - n0), ny - 1, RMID, RHI);
                    else if (k < n2) gs(0, ja + 2 * (k - n1), RLO, RMID);
                    else gs(nx - 1, ja + 2 * (k - n2), RHI, RMID);
                }
                __syncthreads();
            }
            // the corners inside the tile grown by G, in turn (uniform per CTA;
            // most edge tiles hold none and skip the phase and its barrier)
            unsigned corners = 0;
            for (int c = 0; c < 4; ++c) {
                const int i = (c & 1) ? nx - 1 : 0, j = (c & 2) ? ny - 1 : 0;
                if (i < X0 - G || i >= X1 + G || j < Y0 - G || j >= Y1 + G) continue;
                const int xr = region(i, nx, pr.xl, pr.xh), yr = region(j, ny, pr.yl, pr.yh);
                if (xr != RMID && yr != RMID) corners |= 1u << c;
            }
            if (corners) {
                if (threadIdx.x == 0) {
                    for (int c = 0; c < 4; ++c) {
                        if (!((corners >> c) & 1u)) continue;
                        const int i = (c & 1) ? nx - 1 : 0, j = (c & 2) ? ny - 1 : 0;
                        gs(i, j, region(i, nx, pr.xl, pr.xh), region(j, ny, pr.yl, pr.yh));
                    }
                }
                __syncthreads();
            }
        }
    }   // sweeps

    // 5. write the tile, and the ghost cells next to it (the state fill_ghosts
    //    leaves: filled at the start of the sweep)
    const int wi0 = (X0 == 0) ? -1 : X0, wi1 = (X1 >= nx) ? nx + 1 : X1;
    const int wj0 = (Y0 == 0) ? -1 : Y0, wj1 = (Y1 >= ny) ? ny + 1 : Y1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = wj0 + warp; j < wj1; j += (blockDim.x >> 5)) {
        const T* srow = smem + (j - t.poy) * W::PW - t.pox;
        T* grow = &AT(pout, 0, j);
        for (int i = wi0 + lane; i < wi1; i += 32) grow[i] = srow[i];
    }
}

template <bool kTma, class T, int TX, int K = 1>
__global__ void __launch_bounds__((Win<T, TX, K>::kThreads), (Win<T, TX, K>::kMinBlocks))
    k_sweep9(const __grid_constant__ SweepMaps m, DFT<T> pin, DFT<T> pout, DFT<T> rhs, DFT<T> invd, GeoT<T> g,
             const __grid_constant__ BCd b, int homog, int nx, int ny, int4 part, double omega, int* status) {
    allow_dependents();
    sweep_tile<kTma, T, TX, K>(m, pin, pout, rhs, invd, g, b, homog, nx, ny, part, omega, status, blockIdx.x,
                               blockIdx.y);
}

// Lockstep batches: one launch sweeps the same level of many problems.  Job
// k owns blocks [pre[k], pre[k + 1]) of the grid, one per tile of its level
// (row-major over its gx x gy tiles); a block finds its job by binary
// search.  flip selects the buffer each job's phi is read from (the job's s0
// xor flip), so one job table serves every sweep of a smoothing call.
// Descriptors in a job table may have been rewritten since the last launch
// that read them (tables are rebuilt when the set of unconverged problems
// changes): the tensor-map proxy is made to see the new ones before use.
template <class T, int TX, int K>
__global__ void __launch_bounds__((Win<T, TX, K>::kThreads), (Win<T, TX, K>::kMinBlocks))
    k_sweep9_jobs(const SweepJobT<T>* __restrict__ jobs, const int* __restrict__ pre, int njobs, int flip,
                  double omega, int* status) {
    allow_dependents();
    const int blk = blockIdx.x;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {   // the last job with pre[job] <= blk
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(pre + mid) <= blk) lo = mid;
        else hi = mid - 1;
    }
    const SweepJobT<T>& J = jobs[lo];
    const int q = blk - __ldg(pre + lo), side = J.s0 ^ flip;
    const SweepMaps& m = J.m[side];
    if (threadIdx.x == 0) {
        for (const CUtensorMap* d : {&m.pin, &m.rhs, &m.invd, &m.xx, &m.xy, &m.yx, &m.yy})
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(d) : "memory");
    }
    __syncthreads();
    sweep_tile<true, T, TX, K>(m, J.buf[side], J.buf[side ^ 1], J.rhs, J.invd, J.g, J.b, 1, J.nx, J.ny, J.part, omega,
                               status, q % J.gx, q / J.gx);
}

}  // namespace

bool sweep_fusable(const BCd& b) {
    for (int s = 0; s < 4; ++s) {
        const int t = b.type[s];
        if (t != T_DIRI && t != T_NEUM && t != T_PERIODIC) return false;
    }
    return true;
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

template <class T>
constexpr CUtensorMapDataType map_type() {
    return sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
}

// A 2-D map of `width` x `height` elements at `base`, row pitch ld, box PW x PH.
template <class W, class T>
bool encode(CUtensorMap* m, const T* base, long width, long height, int ld) {
    const PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || ((uintptr_t)base & 15) || (((long)ld * (long)sizeof(T)) & 15) || width > ld || width <= 0 ||
        height <= 0)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)height};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(T)};
    const cuuint32_t box[2] = {(cuuint32_t)W::PW, (cuuint32_t)W::PH};
    const cuuint32_t es[2] = {1, 1};
    return fn(m, map_type<T>(), 2, const_cast<T*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <class W, class T>
bool prepare_maps(SweepMaps* m, const DFT<T>& e, const DFT<T>& rhs, const DFT<T>& invd, const GeoT<T>& g, int nx,
                  int ny) {
    // phi from the 16-byte-aligned column kAlign left of column 0 (so the
    // ghost column -1 is inside), and row -1; the ghost column nx must lie
    // inside the pitch
    m->pcb = -W::kAlign;
    m->prb = -1;
    if (e.ld < nx + 1 + W::kAlign) return false;
    return encode<W>(&m->pin, &AT(e, m->pcb, -1), e.ld, ny + 2, e.ld) && encode<W>(&m->rhs, rhs.p, nx, ny, rhs.ld) &&
           encode<W>(&m->invd, invd.p, nx, ny, invd.ld) && encode<W>(&m->xx, g.xx.p, nx + 1, ny, g.xx.ld) &&
           encode<W>(&m->xy, g.xy.p, nx + 1, ny, g.xy.ld) && encode<W>(&m->yx, g.yx.p, nx, ny + 1, g.yx.ld) &&
           encode<W>(&m->yy, g.yy.p, nx, ny + 1, g.yy.ld);
}

template <class T, int TX, int K>
cudaError_t set_attr_jobs() {
    return cudaFuncSetAttribute(k_sweep9_jobs<T, TX, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)Win<T, TX, K>::kSmemBytes);
}

template <class T, int TX, int K = 1>
cudaError_t set_attr() {
    cudaError_t e = cudaFuncSetAttribute(k_sweep9<true, T, TX, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)Win<T, TX, K>::kSmemBytes);
    if constexpr (K == 1) {   // several sweeps per launch: the solver's own arrays (TMA) only
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_sweep9<false, T, TX, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)Win<T, TX, K>::kSmemBytes);
    }
    return e;
}

int sm_count() {
    static std::mutex mu;
    static int n[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> lock(mu);
    if (!n[dev] && cudaDeviceGetAttribute(&n[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        n[dev] = 148;
    }
    return n[dev];
}

// Tile width for a level: FP32 levels take 64-wide tiles when those alone
// fill every SM with as many CTAs as fit; smaller levels, whose sweep lasts
// about one CTA's latency, keep the narrower tiles and their larger grid.
template <class T>
int tile_width(int nx, int ny) {
    if (sizeof(T) == 8) return 32;
    const long wide = (long)((nx + 63) / 64) * ((ny + kTY - 1) / kTY);
    return wide >= (long)Win<float, 64>::kMinBlocks * sm_count() ? 64 : 32;
}

template <class T>
void tma_prepare(SweepTma* t, const DFT<T>& ea, const DFT<T>& eb, const DFT<T>& rhs, const DFT<T>& invd,
                 const GeoT<T>& g, int nx, int ny) {
    t->tx = tile_width<T>(nx, ny);
    bool wide = false;
    if constexpr (sizeof(T) == 4) {
        wide = t->tx == 64;
        if (wide)
            t->ok = prepare_maps<Win<T, 64>>(&t->ma, ea, rhs, invd, g, nx, ny) &&
                    prepare_maps<Win<T, 64>>(&t->mb, eb, rhs, invd, g, nx, ny);
    }
    if (!wide)
        t->ok = prepare_maps<Win<T, 32>>(&t->ma, ea, rhs, invd, g, nx, ny) &&
                prepare_maps<Win<T, 32>>(&t->mb, eb, rhs, invd, g, nx, ny);
    // two sweeps per launch: levels of 32-wide tiles that one wave of the
    // two-sweep CTAs covers (their sweeps last about one CTA's latency)
    const long tiles = (long)((nx + 31) / 32) * ((ny + kTY - 1) / kTY);
    t->ok2 = t->ok && !wide && tiles <= (long)Win<T, 32, 2>::kMinBlocks * sm_count() &&
             prepare_maps<Win<T, 32, 2>>(&t->ma2, ea, rhs, invd, g, nx, ny) &&
             prepare_maps<Win<T, 32, 2>>(&t->mb2, eb, rhs, invd, g, nx, ny);
    t->pa = ea.p;
    t->pb = eb.p;
    t->rhs = rhs.p;
    t->invd = invd.p;
    t->xx = g.xx.p;
}

template <class T, int TX, int K = 1>
cudaError_t launch_tiles(const SweepMaps* m, const DFT<T>& pin, const DFT<T>& pout, const DFT<T>& rhs,
                         const DFT<T>& invd, const GeoT<T>& g, const BCd& b, int homog, int nx, int ny, double omega,
                         int* status, cudaStream_t st) {
    using W = Win<T, TX, K>;
    dim3 grd((nx + TX - 1) / TX, (ny + kTY - 1) / kTY);
    const int4 part = make_int4(nx / (int)grd.x, nx % (int)grd.x, ny / (int)grd.y, ny % (int)grd.y);
    if (m) {
        // a solver's sweep: a programmatic dependent of the kernel before it
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grd;
        cfg.blockDim = dim3(W::kThreads);
        cfg.dynamicSmemBytes = W::kSmemBytes;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, k_sweep9<true, T, TX, K>, *m, pin, pout, rhs, invd, g, b, homog, nx, ny,
                                  part, omega, status);
    }
    if constexpr (K == 1) {
        static const SweepMaps none{};
        k_sweep9<false, T, TX><<<grd, W::kThreads, W::kSmemBytes, st>>>(none, pin, pout, rhs, invd, g, b, homog, nx,
                                                                        ny, part, omega, status);
        return cudaGetLastError();
    }
    return cudaErrorNotSupported;
}

template <class T>
cudaError_t sweep_impl(const DFT<T>& pin, const DFT<T>& pout, const DFT<T>& rhs, const DFT<T>& invd,
                       const GeoT<T>& g, const BCd& b, int homog, int nx, int ny, double omega, const SweepTma* tma,
                       int* status, cudaStream_t st) {
    cudaError_t e = sweep_kernels_init();
    if (e != cudaSuccess) return e;
    const SweepMaps* m = nullptr;
    if (tma && tma->ok && (const void*)rhs.p == tma->rhs && (const void*)invd.p == tma->invd &&
        (const void*)g.xx.p == tma->xx)
        m = ((const void*)pin.p == tma->pa) ? &tma->ma : ((const void*)pin.p == tma->pb) ? &tma->mb : nullptr;
    const int tx = m ? tma->tx : tile_width<T>(nx, ny);
    bool wide = false;
    if constexpr (sizeof(T) == 4) {
        wide = tx == 64;
        if (wide) e = launch_tiles<T, 64>(m, pin, pout, rhs, invd, g, b, homog, nx, ny, omega, status, st);
    }
    if (!wide) e = launch_tiles<T, 32>(m, pin, pout, rhs, invd, g, b, homog, nx, ny, omega, status, st);
    count_launch();
    return e;
}

}  // namespace

// Per device: dynamic shared memory above 48 KB must be opted into.
cudaError_t sweep_kernels_init() {
    static std::mutex mu;
    static unsigned long long done = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && (done >> dev) & 1ull) return cudaSuccess;
    e = set_attr<double, 32>();
    if (e == cudaSuccess) e = set_attr<float, 32>();
    if (e == cudaSuccess) e = set_attr<float, 64>();
    if (e == cudaSuccess) e = set_attr<float, 32, 2>();
    if (e == cudaSuccess) e = set_attr<double, 32, 2>();
    if (e == cudaSuccess) e = set_attr_jobs<double, 32, 1>();
    if (e == cudaSuccess) e = set_attr_jobs<double, 32, 2>();
    if (e == cudaSuccess) e = set_attr_jobs<float, 32, 1>();
    if (e == cudaSuccess) e = set_attr_jobs<float, 64, 1>();
    if (e == cudaSuccess) e = set_attr_jobs<float, 32, 2>();
    if (e == cudaSuccess && dev < 64) done |= 1ull << dev;
    return e;
}

void sweep_tma_prepare(SweepTma* t, const DF& ea, const DF& eb, const DF& rhs, const DF& invd, const Geo& g, int nx,
                       int ny) {
    tma_prepare(t, ea, eb, rhs, invd, g, nx, ny);
}
void sweep_tma_prepare(SweepTma* t, const DF32& ea, const DF32& eb, const DF32& rhs, const DF32& invd,
                       const Geo32& g, int nx, int ny) {
    tma_prepare(t, ea, eb, rhs, invd, g, nx, ny);
}

cudaError_t launch_sweep9(const DF& pin, const DF& pout, const DF& rhs, const DF& invd, const Geo& g, const BCd& b,
                          int homog, int nx, int ny, double omega, const SweepTma* tma, int* status,
                          cudaStream_t st) {
    return sweep_impl(pin, pout, rhs, invd, g, b, homog, nx, ny, omega, tma, status, st);
}
cudaError_t launch_sweep9(const DF32& pin, const DF32& pout, const DF32& rhs, const DF32& invd, const Geo32& g,
                          const BCd& b, int homog, int nx, int ny, double omega, const SweepTma* tma, int* status,
                          cudaStream_t st) {
    return sweep_impl(pin, pout, rhs, invd, g, b, homog, nx, ny, omega, tma, status, st);
}

bool sweep_pair_ok(const SweepTma* tma, const BCd& b) {
    if (!tma || !tma->ok2 || !sweep_fusable(b)) return false;
    for (int s = 0; s < 4; ++s)   // a periodic ghost would be read from global memory, one sweep stale
        if (b.type[s] == T_PERIODIC) return false;
    return true;
}

template <class T>
cudaError_t sweep_pair_impl(const DFT<T>& pin, const DFT<T>& pout, const DFT<T>& rhs, const DFT<T>& invd,
                            const GeoT<T>& g, const BCd& b, int homog, int nx, int ny, double omega,
                            const SweepTma* tma, int* status, cudaStream_t st) {
    if (!sweep_pair_ok(tma, b) || (const void*)rhs.p != tma->rhs || (const void*)invd.p != tma->invd ||
        (const void*)g.xx.p != tma->xx)
        return cudaErrorNotSupported;
    const SweepMaps* m =
        ((const void*)pin.p == tma->pa) ? &tma->ma2 : ((const void*)pin.p == tma->pb) ? &tma->mb2 : nullptr;
    if (!m) return cudaErrorNotSupported;
    cudaError_t e = sweep_kernels_init();
    if (e == cudaSuccess) e = launch_tiles<T, 32, 2>(m, pin, pout, rhs, invd, g, b, homog, nx, ny, omega, status, st);
    count_launch();
    return e;
}

cudaError_t launch_sweep9_pair(const DF32& pin, const DF32& pout, const DF32& rhs, const DF32& invd, const Geo32& g,
                               const BCd& b, int homog, int nx, int ny, double omega, const SweepTma* tma,
                               int* status, cudaStream_t st) {
    return sweep_pair_impl(pin, pout, rhs, invd, g, b, homog, nx, ny, omega, tma, status, st);
}
cudaError_t launch_sweep9_pair(const DF& pin, const DF& pout, const DF& rhs, const DF& invd, const Geo& g,
                               const BCd& b, int homog, int nx, int ny, double omega, const SweepTma* tma,
                               int* status, cudaStream_t st) {
    return sweep_pair_impl(pin, pout, rhs, invd, g, b, homog, nx, ny, omega, tma, status, st);
}

namespace {
template <class T, int TX, int K>
cudaError_t jobs_launch(const SweepJobT<T>* jobs, const int* pre, int njobs, int nblocks, int flip, int* status,
                        cudaStream_t st) {
    using W = Win<T, TX, K>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(W::kThreads);
    cfg.dynamicSmemBytes = W::kSmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_sweep9_jobs<T, TX, K>, jobs, pre, njobs, flip, 1.0, status);
}
}  // namespace

template <class T>
cudaError_t launch_sweep9_jobs(const SweepJobT<T>* jobs, const int* pre, int njobs, int nblocks, int tx, int k,
                               int flip, int* status, cudaStream_t st) {
    if (njobs < 1 || nblocks < 1) return cudaSuccess;
    cudaError_t e = sweep_kernels_init();
    if (e != cudaSuccess) return e;
    if (tx == 32 && k == 1) e = jobs_launch<T, 32, 1>(jobs, pre, njobs, nblocks, flip, status, st);
    else if (tx == 32 && k == 2) e = jobs_launch<T, 32, 2>(jobs, pre, njobs, nblocks, flip, status, st);
    else if (sizeof(T) == 4 && tx == 64 && k == 1) e = jobs_launch<float, 64, 1>(
        reinterpret_cast<const SweepJobT<float>*>(jobs), pre, njobs, nblocks, flip, status, st);
    else return cudaErrorInvalidValue;
    count_launch();
    return e;
}
template cudaError_t launch_sweep9_jobs<double>(const SweepJobT<double>*, const int*, int, int, int, int, int, int*,
                                                cudaStream_t);
template cudaError_t launch_sweep9_jobs<float>(const SweepJobT<float>*, const int*, int, int, int, int, int, int*,
                                               cudaStream_t);

}  // namespace mgp
