// mgp_lockstep.cu -- the phases of a V-cycle for many problems at once (the
// lockstep batch of mgp_batch_* with MGP_FLAG_LOCKSTEP).  No counterpart in
// the Fortran library, which solves one problem per call.
//
// Every kernel here takes a job table: job k owns blocks [pre[k], pre[k+1])
// of a 1-D grid, and each block finds its job by binary search over pre.
// Within a job the block does exactly what the single-problem kernel does
// for the same cells (fill_ghosts, the fused residual-restriction, prolong,
// the elementwise steps), so a problem's bits do not depend on the batch it
// runs in.  The residual norms are summed per job over its blocks in block
// order, a fixed order for a given problem.
#include <cuda_runtime.h>

#include "mgp_kernels.cuh"

namespace mgp {

namespace {

constexpr int kBX = 32, kBY = 8;   // cell blocks (as kBlk2)

// The last job k with pre[k] <= blk.
__device__ __forceinline__ int job_of(const int* __restrict__ pre, int njobs, int blk) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(pre + mid) <= blk) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// fill_ghosts (k_fill): 256 perimeter elements a block.
template <class T>
__global__ void __launch_bounds__(256) k_fill_jobs(const FillJob<T>* __restrict__ jobs, const int* __restrict__ pre,
                                                   int njobs, int phase) {
    const int k = job_of(pre, njobs, blockIdx.x);
    const FillJob<T>& J = jobs[k];
    const int t = (blockIdx.x - pre[k]) * blockDim.x + threadIdx.x;
    int lo[4], cnt[4];
    for (int s = 0; s < 4; ++s) side_range(J.b, s, J.nx, J.ny, J.do_neum, lo[s], cnt[s]);
    int q = t;
    const int s0 = (phase == 1) ? 2 : 0, s1 = (phase == 0) ? 2 : 4;
    if (phase != 2) {
        for (int s = s0; s < s1; ++s) {
            if (q < cnt[s]) {
                fill_side_elem(J.p, J.g, J.b, J.homog, s, J.nx, J.ny, lo[s] + q);
                return;
            }
            q -= cnt[s];
        }
    }
    if (phase >= 2 && q < 4) fill_corner(J.p, J.b, J.nx, J.ny, q);
}

// k_resid_restrict for a job's 32 x 8 block of fine cells.
template <class T, class TC>
__global__ void __launch_bounds__(kBX * kBY) k_resid_jobs(const ResidJob<T, TC>* __restrict__ jobs,
                                                          const int* __restrict__ pre, int njobs) {
    __shared__ T w[kBY][kBX + 1];
    const int k = job_of(pre, njobs, blockIdx.x);
    const ResidJob<T, TC>& J = jobs[k];
    const int q = blockIdx.x - pre[k];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = (q % J.gbx) * kBX + tx, j = (q / J.gbx) * kBY + ty;
    T v = T(0.0);
    if (i < J.nx && j < J.ny) v = AT(J.rhs, i, j) - apply9(J.phi, J.g, J.b, 1, J.nx, J.ny, i, j);
    w[ty][tx] = v;
    __syncthreads();
    if ((tx % J.refx) || (ty % J.refy)) return;
    const int ci = i / J.refx, cj = j / J.refy;
    if (ci >= J.ncx || cj >= J.ncy) return;
    T acc = T(0.0);
    const T sc = T(1.0 / (J.refx * J.refy));
    for (int a = 0; a < J.refy; ++a)
        for (int c = 0; c < J.refx; ++c) acc = acc + sc * w[ty + a][tx + c];
    const TC r = TC(acc);
    AT(J.rc, ci, cj) = r;
    AT(J.ec, ci, cj) = r * AT(J.invdc, ci, cj);
}

// k_prolong (order 1) for a job's 32 x 8 block of coarse cells.
template <class TF, class TC>
__global__ void __launch_bounds__(kBX * kBY) k_prolong_jobs(const ProlongJob<TF, TC>* __restrict__ jobs,
                                                            const int* __restrict__ pre, int njobs) {
    const int k = job_of(pre, njobs, blockIdx.x);
    const ProlongJob<TF, TC>& J = jobs[k];
    const int q = blockIdx.x - pre[k];
    const int ci = (q % J.gbx) * kBX + threadIdx.x, cj = (q / J.gbx) * kBY + threadIdx.y;
    if (ci >= J.ncx || cj >= J.ncy) return;
    prolong_cell(J.fine, J.crse, ci, cj, J.refx, J.refy, 1);
}

// Elementwise steps over the valid region plus g ghost layers.  kind 0:
// y = y + x (k_axpby with a = b = 1), 1: y = x converted (k_convert), 2:
// y = y - x (k_axpby with a = 1, b = -1), 3: y = x * z (k_set_guess).
template <class TD, class TS>
__global__ void __launch_bounds__(kBX * kBY) k_cell_jobs(const CellJob<TD, TS>* __restrict__ jobs,
                                                         const int* __restrict__ pre, int njobs, int kind) {
    const int k = job_of(pre, njobs, blockIdx.x);
    const CellJob<TD, TS>& J = jobs[k];
    const int q = blockIdx.x - pre[k];
    const int i = (q % J.gbx) * kBX + threadIdx.x - J.g, j = (q / J.gbx) * kBY + threadIdx.y - J.g;
    if (i >= J.nx + J.g || j >= J.ny + J.g) return;
    if (kind == 0) AT(J.y, i, j) = AT(J.y, i, j) + TD(AT(J.x, i, j));
    else if (kind == 1) AT(J.y, i, j) = TD(AT(J.x, i, j));
    else if (kind == 2) AT(J.y, i, j) = AT(J.y, i, j) - TD(AT(J.x, i, j));
    else AT(J.y, i, j) = TD(AT(J.x, i, j)) * AT(J.z, i, j);
}

// r = rhs - L[phi] (k_apply, mode 1) and the block's sum of r^2.
__global__ void __launch_bounds__(kBX * kBY) k_norm_jobs(const NormJob* __restrict__ jobs, const int* __restrict__ pre,
                                                         int njobs, double* partials) {
    __shared__ double sh[kBX * kBY];
    const int k = job_of(pre, njobs, blockIdx.x);
    const NormJob& J = jobs[k];
    const int q = blockIdx.x - pre[k];
    const int i = (q % J.gbx) * kBX + threadIdx.x, j = (q / J.gbx) * kBY + threadIdx.y;
    double sq = 0.0;
    if (i < J.nx && j < J.ny) {
        const double r = AT(J.rhs, i, j) - apply9(J.phi, J.g, J.b, J.homog, J.nx, J.ny, i, j);
        AT(J.r, i, j) = r;
        sq = r * r;
    }
    const int t = threadIdx.y * kBX + threadIdx.x;
    sh[t] = sq;
    __syncthreads();
    for (int s = kBX * kBY / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] = sh[t] + sh[t + s];
        __syncthreads();
    }
    if (t == 0) partials[blockIdx.x] = sh[0];
}

// norms[k] = sqrt(vol[k] * sum of job k's partials in block order): a CTA per job.
__global__ void __launch_bounds__(256) k_norm_final(const double* __restrict__ partials, const int* __restrict__ pre,
                                                    const double* __restrict__ vol, double* norms) {
    __shared__ double sh[256];
    const int k = blockIdx.x, b0 = pre[k], b1 = pre[k + 1];
    double acc = 0.0;
    for (int b = b0 + (int)threadIdx.x; b < b1; b += blockDim.x) acc = acc + partials[b];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) norms[k] = sqrt(vol[k] * sh[0]);
}

}  // namespace

template <class T>
cudaError_t launch_fill_jobs(const FillJob<T>* jobs, const int* pre, int njobs, int nblocks, int phases,
                             cudaStream_t st) {
    if (njobs < 1 || nblocks < 1) return cudaSuccess;
    if (phases == 1) {
        k_fill_jobs<<<nblocks, 256, 0, st>>>(jobs, pre, njobs, 3);
        count_launch();
    } else {
        for (int ph = 0; ph < 3; ++ph) k_fill_jobs<<<nblocks, 256, 0, st>>>(jobs, pre, njobs, ph);
        count_launch(3);
    }
    return cudaGetLastError();
}
template cudaError_t launch_fill_jobs<double>(const FillJob<double>*, const int*, int, int, int, cudaStream_t);
template cudaError_t launch_fill_jobs<float>(const FillJob<float>*, const int*, int, int, int, cudaStream_t);

template <class T, class TC>
cudaError_t launch_resid_jobs(const ResidJob<T, TC>* jobs, const int* pre, int njobs, int nblocks, cudaStream_t st) {
    if (njobs < 1 || nblocks < 1) return cudaSuccess;
    k_resid_jobs<<<nblocks, dim3(kBX, kBY), 0, st>>>(jobs, pre, njobs);
    count_launch();
    return cudaGetLastError();
}
template cudaError_t launch_resid_jobs<double, double>(const ResidJob<double, double>*, const int*, int, int,
                                                       cudaStream_t);
template cudaError_t launch_resid_jobs<float, float>(const ResidJob<float, float>*, const int*, int, int, cudaStream_t);
template cudaError_t launch_resid_jobs<float, double>(const ResidJob<float, double>*, const int*, int, int,
                                                      cudaStream_t);

template <class TF, class TC>
cudaError_t launch_prolong_jobs(const ProlongJob<TF, TC>* jobs, const int* pre, int njobs, int nblocks,
                                cudaStream_t st) {
    if (njobs < 1 || nblocks < 1) return cudaSuccess;
    k_prolong_jobs<<<nblocks, dim3(kBX, kBY), 0, st>>>(jobs, pre, njobs);
    count_launch();
    return cudaGetLastError();
}
template cudaError_t launch_prolong_jobs<double, double>(const ProlongJob<double, double>*, const int*, int, int,
                                                         cudaStream_t);
template cudaError_t launch_prolong_jobs<float, float>(const ProlongJob<float, float>*, const int*, int, int,
                                                       cudaStream_t);
template cudaError_t launch_prolong_jobs<float, double>(const ProlongJob<float, double>*, const int*, int, int,
                                                        cudaStream_t);

template <class TD, class TS>
cudaError_t launch_cell_jobs(const CellJob<TD, TS>* jobs, const int* pre, int njobs, int nblocks, int kind,
                             cudaStream_t st) {
    if (njobs < 1 || nblocks < 1) return cudaSuccess;
    k_cell_jobs<<<nblocks, dim3(kBX, kBY), 0, st>>>(jobs, pre, njobs, kind);
    count_launch();
    return cudaGetLastError();
}
template cudaError_t launch_cell_jobs<double, double>(const CellJob<double, double>*, const int*, int, int, int,
                                                     cudaStream_t);
template cudaError_t launch_cell_jobs<float, float>(const CellJob<float, float>*, const int*, int, int, int,
                                                   cudaStream_t);
template cudaError_t launch_cell_jobs<float, double>(const CellJob<float, double>*, const int*, int, int, int,
                                                    cudaStream_t);
template cudaError_t launch_cell_jobs<double, float>(const CellJob<double, float>*, const int*, int, int, int,
                                                    cudaStream_t);

cudaError_t launch_norm_jobs(const NormJob* jobs, const int* pre, int njobs, int nblocks, double* partials,
                             const double* vol, double* norms, cudaStream_t st) {
    if (njobs < 1 || nblocks < 1) return cudaSuccess;
    k_norm_jobs<<<nblocks, dim3(kBX, kBY), 0, st>>>(jobs, pre, njobs, partials);
    k_norm_final<<<njobs, 256, 0, st>>>(partials, pre, vol, norms);
    count_launch(2);
    return cudaGetLastError();
}

}  // namespace mgp
