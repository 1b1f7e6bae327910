// mgp_sweep.cu -- one Gauss-Seidel sweep of the mapped 9-point operator in a
// single launch (relax_gs, poisson2d.f90:1460-1988, in the device order).
//
// The sweep reads phi from `pin` and writes the swept field to `pout` (two
// buffers), so no CTA ever reads a value another CTA has already replaced.
// Each CTA owns one tile of a balanced partition of the grid (tiles at most
// TX x TY and, when there is more than one, at least TX/2 x TY/2, so every
// corner's neighbourhood lies inside the tile that owns the corner).
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
// sub-passes over the whole grid one after another.
#include "mgp_kernels.cuh"

namespace mgp {

namespace {

constexpr int kTX = 32, kTY = 32;
constexpr int kH = 6;   // phi halo: 4 for the colour passes + E = 2 for the boundary pass
constexpr int kG = 5;   // operand halo: the largest pass region, tile + 3 + E
constexpr int kSweepThreads = 256;

constexpr int PW = kTX + 2 * kH, PH = kTY + 2 * kH;         // phi
constexpr int CW = kTX + 2 * kG, CH = kTY + 2 * kG;         // rhs, invdiag (cells)
constexpr int XW = CW + 1, YH = CH + 1;                      // x-faces (XW x CH), y-faces (CW x YH)
constexpr int kSmemDoubles = PW * PH + 2 * CW * CH + 2 * XW * CH + 2 * CW * YH;
constexpr size_t kSmemBytes = kSmemDoubles * sizeof(double);

struct SLoad {
    const double* c;
    int ld;
    __device__ __forceinline__ double operator()(int di, int dj) const { return c[di + dj * ld]; }
};

// The value fill_ghosts (do_neum = .false.) gives ghost (i,j) at the start of
// the sweep, for sides of type DIRI, NEUM (left as stored) and PERIODIC.
__device__ double sweep_ghost(const DF& pin, const BCd& b, int homog, int nx, int ny, int i, int j) {
    const bool xin = (i >= 0 && i < nx), yin = (j >= 0 && j < ny);
    if (xin && !yin) {
        const int s = (j < 0) ? S_YLO : S_YHI;
        const int t = b.type[s];
        if (t == T_DIRI) {
            const int jj = (j < 0) ? 0 : ny - 1, e = (j < 0) ? -1 : 1;
            return ghost_diri(b, homog, s, i, AT(pin, i, jj), AT(pin, i, jj - e), AT(pin, i, jj - 2 * e));
        }
        if (t == T_PERIODIC) return AT(pin, i, (j < 0) ? ny - 1 : 0);
        return AT(pin, i, j);
    }
    if (yin && !xin) {
        const int s = (i < 0) ? S_XLO : S_XHI;
        const int t = b.type[s];
        if (t == T_DIRI) {
            const int ii = (i < 0) ? 0 : nx - 1, e = (i < 0) ? -1 : 1;
            return ghost_diri(b, homog, s, j, AT(pin, ii, j), AT(pin, ii - e, j), AT(pin, ii - 2 * e, j));
        }
        if (t == T_PERIODIC) return AT(pin, (i < 0) ? nx - 1 : 0, j);
        return AT(pin, i, j);
    }
    // corners (AU:1460-1490)
    const bool px = b.type[S_XLO] == T_PERIODIC, py = b.type[S_YLO] == T_PERIODIC;
    if (!px && !py) return kBogus;
    const int wi = (i < 0) ? nx - 1 : 0, wj = (j < 0) ? ny - 1 : 0;
    if (px && py) return AT(pin, wi, wj);
    if (px) return sweep_ghost(pin, b, homog, nx, ny, wi, j);   // a y-side ghost
    return sweep_ghost(pin, b, homog, nx, ny, i, wj);           // an x-side ghost
}

// Copy rows [j0,j1) x columns [i0,i1) of a global field into a shared array
// whose (0,0) is cell (ox, oy) and whose row pitch is w.
__device__ __forceinline__ void stage(double* s, int w, int ox, int oy, const DF& f, int i0, int i1, int j0, int j1) {
    const int cw = i1 - i0, n = cw * (j1 - j0);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int i = i0 + k % cw, j = j0 + k / cw;
        cp_async8(&s[(j - oy) * w + (i - ox)], &AT(f, i, j));
    }
}

struct Tile {
    double *ph, *f, *d, *xx, *xy, *yx, *yy;
    int pox, poy, cox, coy;
};

// One Gauss-Seidel update of (i,j) from shared memory (same operations as gs9).
__device__ __forceinline__ void gs9_tile(const Tile& t, double idx, double idy, const BCd& b, int homog, int i, int j,
                                         int xr, int yr, double omega) {
    double* c = t.ph + (j - t.poy) * PW + (i - t.pox);
    St9 s;
    gather9(SLoad{c, PW}, xr, yr, s);
    const int ci = i - t.cox, cj = j - t.coy;
    Faces fc;
    fc.xxe = t.xx[cj * XW + ci + 1]; fc.xxw = t.xx[cj * XW + ci];
    fc.xye = t.xy[cj * XW + ci + 1]; fc.xyw = t.xy[cj * XW + ci];
    fc.yyn = t.yy[(cj + 1) * CW + ci]; fc.yys = t.yy[cj * CW + ci];
    fc.yxn = t.yx[(cj + 1) * CW + ci]; fc.yxs = t.yx[cj * CW + ci];
    const double lphi = lap9f(s, fc, idx, idy, i, j, xr, yr, b, homog);
    const double p = c[0];
    const double newphi = p + (t.f[cj * CW + ci] - lphi) * t.d[cj * CW + ci];
    c[0] = omega * newphi + (1.0 - omega) * p;
}

__global__ void __launch_bounds__(kSweepThreads) k_sweep9(DF pin, DF pout, DF rhs, DF invd, Geo g, BCd b, int homog,
                                                          int nx, int ny, double omega) {
    extern __shared__ double smem[];
    const int X0 = (int)((long)blockIdx.x * nx / gridDim.x), X1 = (int)((long)(blockIdx.x + 1) * nx / gridDim.x);
    const int Y0 = (int)((long)blockIdx.y * ny / gridDim.y), Y1 = (int)((long)(blockIdx.y + 1) * ny / gridDim.y);
    const Per pr = periodic_of(b);
    const bool edge_tile = (!pr.xl && X0 == 0) || (!pr.xh && X1 >= nx) || (!pr.yl && Y0 == 0) || (!pr.yh && Y1 >= ny);
    const int E = edge_tile ? 2 : 0;

    Tile t;
    t.ph = smem;
    t.f = t.ph + PW * PH;
    t.d = t.f + CW * CH;
    t.xx = t.d + CW * CH;
    t.xy = t.xx + XW * CH;
    t.yx = t.xy + XW * CH;
    t.yy = t.yx + CW * YH;
    t.pox = X0 - kH; t.poy = Y0 - kH;
    t.cox = X0 - kG; t.coy = Y0 - kG;

    // 1. stage phi on tile + (4 + E) and the operands on tile + (3 + E)
    const int hp = 4 + E, hc = 3 + E;
    const int pi0 = max(X0 - hp, -1), pi1 = min(X1 + hp, nx + 1), pj0 = max(Y0 - hp, -1), pj1 = min(Y1 + hp, ny + 1);
    const int ci0 = max(X0 - hc, 0), ci1 = min(X1 + hc, nx), cj0 = max(Y0 - hc, 0), cj1 = min(Y1 + hc, ny);
    stage(t.ph, PW, t.pox, t.poy, pin, pi0, pi1, pj0, pj1);
    stage(t.f, CW, t.cox, t.coy, rhs, ci0, ci1, cj0, cj1);
    stage(t.d, CW, t.cox, t.coy, invd, ci0, ci1, cj0, cj1);
    stage(t.xx, XW, t.cox, t.coy, g.xx, ci0, ci1 + 1, cj0, cj1);
    stage(t.xy, XW, t.cox, t.coy, g.xy, ci0, ci1 + 1, cj0, cj1);
    stage(t.yx, CW, t.cox, t.coy, g.yx, ci0, ci1, cj0, cj1 + 1);
    stage(t.yy, CW, t.cox, t.coy, g.yy, ci0, ci1, cj0, cj1 + 1);
    cp_async_wait_all();
    __syncthreads();
    // 2. sweep-start ghost fill on the staged ghost cells
    {
        const int lw = pi1 - pi0, n = lw * (pj1 - pj0);
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const int i = pi0 + k % lw, j = pj0 + k / lw;
            if (i >= 0 && i < nx && j >= 0 && j < ny) continue;
            t.ph[(j - t.poy) * PW + (i - t.pox)] = sweep_ghost(pin, b, homog, nx, ny, i, j);
        }
    }
    __syncthreads();

    // 3. interior colour passes on shrinking regions
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
        const int ci = colour_ci(c), cj = colour_cj(c);
        const int grow = 3 - c + E;
        int i0 = max(X0 - grow, 0), i1 = min(X1 + grow, nx);
        int j0 = max(Y0 - grow, 0), j1 = min(Y1 + grow, ny);
        i0 += (i0 & 1) != ci;
        j0 += (j0 & 1) != cj;
        const int cw = (i1 - i0 + 1) / 2, chh = (j1 - j0 + 1) / 2;
        for (int k = threadIdx.x; k < cw * chh; k += blockDim.x) {
            const int i = i0 + 2 * (k % cw), j = j0 + 2 * (k / cw);
            if (i >= i1 || j >= j1) continue;
            const int xr = region(i, nx, pr.xl, pr.xh), yr = region(j, ny, pr.yl, pr.yh);
            if (xr != RMID || yr != RMID) continue;
            gs9_tile(t, g.idx, g.idy, b, homog, i, j, xr, yr, omega);
        }
        __syncthreads();
    }

    // 4. boundary pass (edge tiles only; uniform per CTA)
    if (edge_tile) {
        const int i0 = max(X0 - 1, 0), i1 = min(X1 + 1, nx);
        const int j0 = max(Y0 - 1, 0), j1 = min(Y1 + 1, ny);
        const int w = i1 - i0, h = j1 - j0;
        for (int c = 0; c < 4; ++c) {
            const int ci = colour_ci(c), cj = colour_cj(c);
            for (int k = threadIdx.x; k < w * h; k += blockDim.x) {
                const int i = i0 + k % w, j = j0 + k / w;
                if ((i & 1) != ci || (j & 1) != cj) continue;
                const int xr = region(i, nx, pr.xl, pr.xh), yr = region(j, ny, pr.yl, pr.yh);
                if ((xr == RMID) == (yr == RMID)) continue;   // edges only
                gs9_tile(t, g.idx, g.idy, b, homog, i, j, xr, yr, omega);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            for (int c = 0; c < 4; ++c) {
                const int i = (c & 1) ? nx - 1 : 0, j = (c & 2) ? ny - 1 : 0;
                if (i < X0 || i >= X1 || j < Y0 || j >= Y1) continue;
                const int xr = region(i, nx, pr.xl, pr.xh), yr = region(j, ny, pr.yl, pr.yh);
                if (xr != RMID && yr != RMID) gs9_tile(t, g.idx, g.idy, b, homog, i, j, xr, yr, omega);
            }
        }
        __syncthreads();
    }

    // 5. write the tile, and the ghost cells next to it (the state fill_ghosts
    //    leaves: filled at the start of the sweep)
    const int wi0 = (X0 == 0) ? -1 : X0, wi1 = (X1 >= nx) ? nx + 1 : X1;
    const int wj0 = (Y0 == 0) ? -1 : Y0, wj1 = (Y1 >= ny) ? ny + 1 : Y1;
    const int ww = wi1 - wi0, wh = wj1 - wj0;
    for (int k = threadIdx.x; k < ww * wh; k += blockDim.x) {
        const int i = wi0 + k % ww, j = wj0 + k / ww;
        AT(pout, i, j) = t.ph[(j - t.poy) * PW + (i - t.pox)];
    }
}

}  // namespace

bool sweep_fusable(const BCd& b) {
    for (int s = 0; s < 4; ++s) {
        const int t = b.type[s];
        if (t != T_DIRI && t != T_NEUM && t != T_PERIODIC) return false;
    }
    return true;
}

cudaError_t launch_sweep9(const DF& pin, const DF& pout, const DF& rhs, const DF& invd, const Geo& g, const BCd& b,
                          int homog, int nx, int ny, double omega, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_sweep9, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    dim3 grd((nx + kTX - 1) / kTX, (ny + kTY - 1) / kTY);
    k_sweep9<<<grd, kSweepThreads, kSmemBytes, st>>>(pin, pout, rhs, invd, g, b, homog, nx, ny, omega);
    count_launch();
    return cudaGetLastError();
}

}  // namespace mgp
