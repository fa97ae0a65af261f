// The coarsest level's exact solve, set up without library calls: A = L L^T (FP64 Cholesky) and
// the packed inverse factor M = tril(L^-1) + triu(L^-T, 1) that vx_coarse_apply_factor applies with
// two triangular passes (the reference's two triangular solves, src/voxel_mg.py:152-159).
//
// The coarsest matrix of a voxel grid is banded: a node couples only to the 27 nodes around it, so
// |i - j| <= bw = 3 ((ny+1)(nz+1) + (nz+1) + 1) + 2 in the author DOF order, and L keeps that band.
// The factorisation therefore costs about n bw^2 / 2 multiply-adds instead of n^3 / 6:
//   * band_load:      the lower band of A into band storage lb[i (bw+1) + (j - i + bw)] = L[i][j];
//   * per block column k of CB = 64 columns, two launches:
//       band_potrf:   one CTA (a thread per row) factors the CB x CB diagonal block in shared memory
//                     and inverts it;
//       band_update:  one CTA per lower tile (I, J) of the rows the block column reaches (at most
//                     bw below it) forms the panel rows L_I = A_I L_kk^-T and L_J the same way (a
//                     64 x 64 product with the block's inverse), writes L_I (diagonal tiles only),
//                     and subtracts L_I L_J^T from the band;
//   * band_inverse:   X = L^-1 column by column: a CTA owns 32 consecutive columns (one warp each),
//                     streams the band rows of L through shared memory by cp.async, and each warp
//                     runs the forward substitution x_i = -(sum_p L[i][p] x_p) / L[i][i] over the
//                     window of its last bw + 1 values; every x_i goes to M[i][j] and M[j][i].
// A non-positive pivot sets *info to its 1-based column (the factorisation continues with pivot 1
// so every value stays finite); the caller reads *info once.
#include "vx_common.cuh"
#include <algorithm>
#include <atomic>

namespace vx {

constexpr int CB = 64;            // block columns of the banded Cholesky
constexpr int CBP = CB + 1;       // padded shared-memory row
constexpr int POTRF_T = 256;    // copies by all threads; the first CB own a row of the diagonal block
constexpr int UPDATE_T = 256;
constexpr int INV_STAGES = 4;     // L rows in flight in band_inverse

__device__ __forceinline__ int64_t bidx(int i, int j, int bw) { return int64_t(i) * (bw + 1) + (j - i + bw); }

__global__ void band_load_kernel(int n, int bw, const double* __restrict__ A, double* __restrict__ lb) {
    vx::pdl_begin();
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(n) * (bw + 1)) return;
    const int i = int(t / (bw + 1)), c = int(t % (bw + 1)), j = i - bw + c;
    lb[t] = j >= 0 ? A[int64_t(i) * n + j] : 0.0;
}

// Factor the diagonal block of block column k0 (w = min(CB, n - k0) columns) and write it back; its
// inverse goes to dinv (CB x CB, row-major, lower triangle), and the block column's rows below it
// (the A values band_update turns into the panel) to apanel ((bw + 1) x CB), so that band_update
// can store finished panel rows in place while other tiles still read the originals.
// Thread r < CB owns row r of the block (right-looking: two barriers per column); the inverse is
// column-parallel (thread c runs the forward substitution of column c, no barrier); every thread
// shares the copies.
// Dynamic shared memory: D and X, CB x CBP each.
__global__ void __launch_bounds__(POTRF_T) band_potrf_kernel(int n, int bw, int k0, double* __restrict__ lb,
                                                             double* __restrict__ dinv, double* __restrict__ apanel,
                                                             int* __restrict__ info) {
    vx::pdl_begin();
    extern __shared__ __align__(16) double psm[];
    double (*D)[CBP] = reinterpret_cast<double (*)[CBP]>(psm);
    double (*X)[CBP] = reinterpret_cast<double (*)[CBP]>(psm + CB * CBP);
    const int w = min(CB, n - k0);
    const int base = k0 + w, rend = min(n, k0 + w + bw);
    const int t = threadIdx.x;
    for (int i = t; i < (rend - base) * CB; i += POTRF_T) {
        const int r = base + i / CB, c = i % CB, col = k0 + c;
        apanel[i] = (c < w && r - col <= bw) ? lb[bidx(r, col, bw)] : 0.0;
    }
    for (int i = t; i < CB * CB; i += POTRF_T) {
        const int r = i / CB, c = i % CB;
        D[r][c] = (r < w && c <= r && r - c <= bw) ? lb[bidx(k0 + r, k0 + c, bw)] : 0.0;
        X[r][c] = 0.0;
    }
    __syncthreads();
    for (int j = 0; j < w; ++j) {
        double d = D[j][j];
        if (!(d > 0.0)) {                                     // not positive definite: flag, keep finite
            if (t == j) atomicCAS(info, 0, k0 + j + 1);
            d = 1.0;
        }
        const double piv = sqrt(d);
        if (t > j && t < w) D[t][j] = D[t][j] / piv;          // column j of L below the pivot
        __syncthreads();
        if (t == j) D[j][j] = piv;
        if (t > j && t < w) {
            const double l = D[t][j];
            for (int c = j + 1; c <= t; ++c) D[t][c] -= l * D[c][j];
        }
        __syncthreads();
    }
    // inverse of the lower-triangular block, column c by thread c:
    // X[c][c] = 1 / D[c][c], X[r][c] = -(sum_{c<=p<r} D[r][p] X[p][c]) / D[r][r]
    if (t < w) {
        X[t][t] = 1.0 / D[t][t];
        for (int r = t + 1; r < w; ++r) {
            double s = 0.0;
            for (int p = t; p < r; ++p) s += D[r][p] * X[p][t];
            X[r][t] = -s / D[r][r];
        }
    }
    __syncthreads();
    for (int i = t; i < CB * CB; i += POTRF_T) {
        const int r = i / CB, c = i % CB;
        if (r < w && c <= r && r - c <= bw) lb[bidx(k0 + r, k0 + c, bw)] = D[r][c];
        dinv[i] = X[r][c];
    }
}

// One lower tile (I, J) of the rows below block column k0: rows ri = base + I*CB + r, rj = base +
// J*CB + c, base = k0 + w.  Dynamic shared memory: the block inverse and the two panels (3 CB x CBP).
__global__ void __launch_bounds__(UPDATE_T) band_update_kernel(int n, int bw, int k0, int tiles,
                                                               double* __restrict__ lb, const double* __restrict__ dinv,
                                                               const double* __restrict__ apanel) {
    vx::pdl_begin();
    extern __shared__ __align__(16) double sm[];
    double (*Xi)[CBP] = reinterpret_cast<double (*)[CBP]>(sm);
    double (*PI)[CBP] = reinterpret_cast<double (*)[CBP]>(sm + CB * CBP);
    double (*PJ)[CBP] = reinterpret_cast<double (*)[CBP]>(sm + 2 * CB * CBP);
    // tile index -> (I, J), I >= J
    int I = 0, rem = blockIdx.x;
    while (rem > I) { rem -= I + 1; ++I; }
    const int J = rem;
    const int w = min(CB, n - k0);
    const int base = k0 + w;
    const int rend = min(n, k0 + w + bw);              // rows the block column reaches
    const int ri0 = base + I * CB, rj0 = base + J * CB;
    if (ri0 >= rend) return;                           // (never: the grid covers the window exactly)
    for (int t = threadIdx.x; t < CB * CB; t += UPDATE_T) {
        const int r = t / CB, c = t % CB;
        Xi[r][c] = dinv[t];
        const int ri = ri0 + r, rj = rj0 + r;
        PI[r][c] = ri < rend ? apanel[int64_t(ri - base) * CB + c] : 0.0;
        PJ[r][c] = rj < rend ? apanel[int64_t(rj - base) * CB + c] : 0.0;
    }
    __syncthreads();
    // panels: P <- P X^T (P[r][m] = sum_{p<=m} A[r][p] X[m][p]); 16 outputs per thread, then written back
    constexpr int PER = CB * CB / UPDATE_T;
    double oi[PER], oj[PER];
    #pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int t = threadIdx.x + q * UPDATE_T, r = t / CB, m = t % CB;
        double si = 0.0, sj = 0.0;
        for (int p = 0; p <= m; ++p) {
            si += PI[r][p] * Xi[m][p];
            sj += PJ[r][p] * Xi[m][p];
        }
        oi[q] = si;
        oj[q] = sj;
    }
    __syncthreads();
    #pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int t = threadIdx.x + q * UPDATE_T, r = t / CB, m = t % CB;
        PI[r][m] = oi[q];
        PJ[r][m] = oj[q];
    }
    __syncthreads();
    if (I == J) {                                      // the panel rows of tile I are final: store them
        for (int t = threadIdx.x; t < CB * CB; t += UPDATE_T) {
            const int r = t / CB, c = t % CB, ri = ri0 + r, col = k0 + c;
            if (c < w && ri < rend && ri - col <= bw) lb[bidx(ri, col, bw)] = PI[r][c];
        }
    }
    // trailing update of the tile: A[ri][rj] -= sum_m L[ri][m] L[rj][m] (lower triangle, in the band)
    for (int t = threadIdx.x; t < CB * CB; t += UPDATE_T) {
        const int r = t / CB, c = t % CB, ri = ri0 + r, rj = rj0 + c;
        if (ri >= rend || rj >= rend || rj > ri || ri - rj > bw) continue;
        double s = 0.0;
        for (int m = 0; m < w; ++m) s += PI[r][m] * PJ[c][m];
        lb[bidx(ri, rj, bw)] -= s;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src) : "memory");
}

// X = L^-1 into the packed matrix (lower part X, upper part X^T).  CTA = nw warps, columns
// j0 .. j0+nw-1 (warp w: column j0 + w); shared memory: INV_STAGES staged band rows of L, then one
// window of bw + 1 values per warp (x_p of its column at slot p mod (bw + 1)).
__global__ void band_inverse_kernel(int n, int bw, const double* __restrict__ lb, double* __restrict__ packed) {
    vx::pdl_begin();
    extern __shared__ __align__(16) double sm[];
    const int W = bw + 1;
    const int nw = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* rows = sm;                                  // [INV_STAGES][W]
    double* win = sm + INV_STAGES * W + warp * W;       // this warp's window
    const int j0 = blockIdx.x * nw;
    const int j = j0 + warp;
    const bool active = j < n;
    auto stage = [&](int i) {                           // band row i of L into its slot (cooperative)
        if (i >= n) return;
        double* dst = rows + (i % INV_STAGES) * W;
        const double* src = lb + int64_t(i) * W;
        for (int c = threadIdx.x; c < W; c += blockDim.x) cp_async8(dst + c, src + c);
    };
    const int i_first = j0;                             // the first row any warp of the CTA needs
    for (int s = 0; s < INV_STAGES - 1; ++s) {
        stage(i_first + s);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    int slot_i = 0;                                     // window slot of row i (i mod W), advanced per step
    if (active) slot_i = j % W;
    for (int i = i_first; i < n; ++i) {
        asm volatile("cp.async.wait_group %0;" ::"n"(INV_STAGES - 2) : "memory");
        __syncthreads();                                // row i visible; the slot staged below is free
        stage(i + INV_STAGES - 1);
        asm volatile("cp.async.commit_group;" ::: "memory");
        const double* Lr = rows + (i % INV_STAGES) * W;  // Lr[c] = L[i][i - bw + c]
        if (active && i >= j) {
            double x;
            if (i == j) {
                x = 1.0 / Lr[bw];
            } else {
                const int p0 = max(j, i - bw);
                double s = 0.0;
                for (int p = p0 + lane; p < i; p += 32) {
                    int sp = slot_i - (i - p);
                    if (sp < 0) sp += W;
                    s += Lr[p - i + bw] * win[sp];
                }
                s = warp_sum(s);
                x = -s / Lr[bw];
            }
            __syncwarp();
            if (lane == 0) {
                win[slot_i] = x;
                packed[int64_t(i) * n + j] = x;
                if (i != j) packed[int64_t(j) * n + i] = x;
            }
            __syncwarp();
            if (++slot_i == W) slot_i = 0;
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

int inverse_warps(int bw) {
    const size_t budget = 227 * 1024;
    const size_t row = size_t(bw + 1) * sizeof(double);
    int nw = 32;
    while (nw > 1 && (INV_STAGES + nw) * row > budget) nw >>= 1;
    return (INV_STAGES + nw) * row > budget ? 0 : nw;
}

}  // namespace vx

using namespace vx;

// doubles of the `work` buffer vx_coarse_factor needs: the band of L, the block inverse, the panel copy
extern "C" int64_t vx_coarse_factor_workspace(int n, int bw) {
    if (n <= 0 || bw < 0) return -1;
    bw = std::min(bw, n - 1);
    return int64_t(n) * (bw + 1) + int64_t(CB) * CB + int64_t(bw + 1) * CB;
}

extern "C" int vx_coarse_factor(int n, int bw, const double* A, double* packed, double* work, int* info,
                                cudaStream_t stream) {
    VX_CHECK_ARG(n > 0 && bw >= 0, VX_ERR_INVALID_ARGUMENT, "vx_coarse_factor: bad size n=%d bw=%d", n, bw);
    VX_CHECK_ARG(A && packed && work && info, VX_ERR_NULL_POINTER, "vx_coarse_factor: NULL pointer");
    VX_CHECK_ARG(A != packed, VX_ERR_INVALID_ARGUMENT, "vx_coarse_factor: packed may not alias A");
    bw = std::min(bw, n - 1);
    const int nw = inverse_warps(bw);
    VX_CHECK_ARG(nw > 0, VX_ERR_INVALID_ARGUMENT, "vx_coarse_factor: bandwidth %d is too wide", bw);
    double* lb = work;
    double* dinv = work + int64_t(n) * (bw + 1);
    double* apanel = dinv + int64_t(CB) * CB;
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), stream);
    if (e != cudaSuccess) {
        set_error("vx_coarse_factor: memset: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    const size_t psm = size_t(2) * CB * CBP * sizeof(double);
    const size_t usm = size_t(3) * CB * CBP * sizeof(double);
    const size_t ism = size_t(INV_STAGES + nw) * (bw + 1) * sizeof(double);
    static std::atomic<uint64_t> opt_p, opt_u, opt_i;
    int st = smem_opt_in(opt_p, (const void*)band_potrf_kernel, psm, "vx_coarse_factor");
    if (!st) st = smem_opt_in(opt_u, (const void*)band_update_kernel, usm, "vx_coarse_factor");
    if (!st) st = smem_opt_in(opt_i, (const void*)band_inverse_kernel, 227 * 1024, "vx_coarse_factor");
    if (st) return st;
    const int64_t band = int64_t(n) * (bw + 1);
    vx::launch(band_load_kernel, unsigned((band + 255) / 256), 256, 0, stream, n, bw, A, lb);
    for (int k0 = 0; k0 < n; k0 += CB) {
        vx::launch(band_potrf_kernel, 1, POTRF_T, psm, stream, n, bw, k0, lb, dinv, apanel, info);
        const int w = std::min(CB, n - k0);
        const int rows = std::min(n, k0 + w + bw) - (k0 + w);
        if (rows <= 0) continue;
        const int T = (rows + CB - 1) / CB;
        vx::launch(band_update_kernel, unsigned(T * (T + 1) / 2), UPDATE_T, usm, stream, n, bw, k0, T, lb,
                   (const double*)dinv, (const double*)apanel);
    }
    vx::launch(band_inverse_kernel, unsigned((n + nw - 1) / nw), unsigned(nw * 32), ism, stream, n, bw,
               (const double*)lb, packed);
    VX_CHECK_LAUNCH("vx_coarse_factor");
    return VX_OK;
}
