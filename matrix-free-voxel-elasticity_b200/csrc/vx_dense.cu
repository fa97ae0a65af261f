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
//       band_update:  four CTAs per lower 64 x 64 tile (I, J) of the rows the block column reaches
//                     (at most bw below it), one per 32 x 32 quadrant, form their rows of the panels
//                     L_I = A_I L_kk^-T and L_J (a product with the block's inverse), write L_I
//                     (diagonal tiles only) and subtract L_I L_J^T from the band;
//   * band_inverse_blocked: X = L^-1 by blocks of 32 rows x 16 columns, a band GEMM per block and
//                     the diagonal block inverses band_potrf kept (bands up to about 550 wide);
//   * band_inverse:   (wider bands) X = L^-1 column by column: a CTA owns 32 consecutive columns (one warp each),
//                     streams the band rows of L through shared memory by cp.async, and each warp
//                     runs the forward substitution x_i = -(sum_p L[i][p] x_p) / L[i][i] over the
//                     window of its last bw + 1 values; every x_i goes to M[i][j] and M[j][i].
// A non-positive pivot sets *info to its 1-based column (the factorisation continues with pivot 1
// so every value stays finite); the caller reads *info once.
#include "vx_common.cuh"
#include <algorithm>
#include <atomic>
#include <type_traits>

namespace vx {

constexpr int CB = 64;            // block columns of the banded Cholesky
constexpr int CBP = CB + 1;       // padded shared-memory row
constexpr int POTRF_T = 256;    // copies by all threads; the first CB own a row of the diagonal block
constexpr int UPDATE_T = 256;
constexpr int INV_STAGES = 4;     // L rows in flight in band_inverse

__device__ __forceinline__ int64_t bidx(int i, int j, int bw) { return int64_t(i) * (bw + 1) + (j - i + bw); }

// Several factorisations of one size run side by side, factorisation m = blockIdx.y of every launch:
// matrix slot[m] of A (and packed, info), workspace m of `work` (the band, the diagonal block
// inverses, the panel copy).
constexpr int FB_MAX = 64;
struct FactorBatch {
    const double* A;
    double* packed;
    double* work;
    int* info;
    int64_t mat;             // doubles from one matrix slot to the next (n * n)
    int64_t ws;              // doubles of one workspace
    int nblk;                // CB-column blocks
    int slot[FB_MAX];
};
struct FactorPtrs {
    const double* A;
    double* packed;
    double* lb;
    double* dinv_all;
    double* apanel;
    int* info;
};
__device__ __forceinline__ FactorPtrs fptrs(const FactorBatch& fb, int n, int bw) {
    const int m = blockIdx.y, s = fb.slot[m];
    FactorPtrs p;
    p.A = fb.A + s * fb.mat;
    p.packed = fb.packed + s * fb.mat;
    p.lb = fb.work + m * fb.ws;
    p.dinv_all = p.lb + int64_t(n) * (bw + 1);
    p.apanel = p.dinv_all + int64_t(fb.nblk) * CB * CB;
    p.info = fb.info + s;
    return p;
}

__global__ void band_load_kernel(int n, int bw, const __grid_constant__ FactorBatch fb) {
    vx::pdl_begin();
    const FactorPtrs P = fptrs(fb, n, bw);
    const double* __restrict__ A = P.A;
    double* __restrict__ lb = P.lb;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(n) * (bw + 1)) return;
    const int i = int(t / (bw + 1)), c = int(t % (bw + 1)), j = i - bw + c;
    lb[t] = j >= 0 ? A[int64_t(i) * n + j] : 0.0;
}

// Factor the diagonal block of block column k0 (w = min(CB, n - k0) columns) and write it back; its
// inverse goes to dinv (CB x CB, row-major, lower triangle), and the block column's rows below it
// (the A values band_update turns into the panel) to apanel ((bw + 1) x CB), so that band_update
// can store finished panel rows in place while other tiles still read the originals.
// The block's CB pivots are a chain of dependent steps, so it is factored by four warps with the
// rows in registers (right-looking; threads i and CB + i hold the even and the odd columns of row i;
// per pivot: the pivot thread's reciprocal square root (the pivot is d rsqrt(d)), a named barrier of
// the four warps, the column through shared memory, a rank-1 update of the row in registers, split
// between the two threads of the row).  Three variants measured no faster: one barrier per pivot
// with every row forming the reciprocal square root from a double-buffered column (+8%), a
// look-ahead in which row j + 1 forms the next pivot before finishing its update (+2%), and (with
// two factoring warps) the update of a whole row by one thread.  Meanwhile warps 4-7 copy the
// panel rows; a block smaller than CB (the last) is padded with the identity.
// The inverse X = L^-1 goes by 32 x 32 blocks: warps 0 and 1 run the forward substitutions of
// X11 and X22 (lane = column, in registers, four partial sums per row), then all eight warps form
// X21 = -X22 (L21 X11).  Every loop is unrolled, so the row and column registers are addressed at
// compile time (a variant with the pivot loop rolled and the row shifted through the registers ran
// slower).
constexpr int HB = CB / 2, HBP = HB + 1;   // half blocks of the block inverse
constexpr int FT = 2 * CB;     // factoring threads: a row's even and odd columns
__device__ __forceinline__ void potrf_bar() { asm volatile("bar.sync 1, %0;" ::"n"(FT) : "memory"); }

// FACTOR = false: the band already holds a Cholesky factor; only the diagonal block's inverse is
// formed (block k0 = blockIdx.x CB, every block in one launch; no panel copy, nothing written back).
template <bool FACTOR>
__global__ void __launch_bounds__(POTRF_T) band_potrf_kernel(int n, int bw, int k0, const __grid_constant__ FactorBatch fb) {
    static_assert(CB == 64 && POTRF_T > FT, "four factoring warps, the others copy");
    vx::pdl_begin();
    if constexpr (!FACTOR) k0 = blockIdx.x * CB;
    const FactorPtrs P = fptrs(fb, n, bw);
    double* __restrict__ lb = P.lb;
    double* __restrict__ dinv = P.dinv_all + int64_t(k0 / CB) * CB * CB;
    double* __restrict__ apanel = P.apanel;
    int* __restrict__ info = P.info;
    extern __shared__ __align__(16) double psm[];
    __shared__ double colj[CB], rinv[CB];
    double (*D)[CBP] = reinterpret_cast<double (*)[CBP]>(psm);
    double (*X)[CBP] = reinterpret_cast<double (*)[CBP]>(psm + CB * CBP);
    double (*Tm)[HBP] = reinterpret_cast<double (*)[HBP]>(psm + 2 * CB * CBP);   // L21 X11
    const int w = min(CB, n - k0);
    const int base = k0 + w, rend = min(n, k0 + w + bw);
    const int t = threadIdx.x;
    {                                                  // the block: every load issued, then stored
        constexpr int NL = CB * CB / POTRF_T;
        double v[NL];
        #pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int i = t + u * POTRF_T, r = i / CB, c = i % CB;
            v[u] = (r < w && c <= r && r - c <= bw) ? lb[bidx(k0 + r, k0 + c, bw)] : (r >= w && r == c ? 1.0 : 0.0);
        }                                              // (identity padding of a short block)
        #pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int i = t + u * POTRF_T;
            D[i / CB][i % CB] = v[u];
        }
    }
    __syncthreads();
    if (!FACTOR && t < CB) rinv[t] = 1.0 / D[t][t];
    if (FACTOR && t < FT) {
        // row t % CB; warps 0-1 hold its even columns, warps 2-3 its odd ones (H = t / CB)
        const int row = t % CB;
        auto factor_rows = [&](auto hc) {
            constexpr int H = decltype(hc)::value;
            double a[CB / 2];                          // a[i] = row, column 2 i + H
            #pragma unroll
            for (int i = 0; i < CB / 2; ++i) a[i] = D[row][2 * i + H];
            #pragma unroll
            for (int j = 0; j < CB; ++j) {
                if ((j & 1) == H && row == j) {
                    double d = a[j / 2];
                    if (!(d > 0.0)) {                  // not positive definite: flag, keep finite
                        if (j < w) atomicCAS(info, 0, k0 + j + 1);
                        d = 1.0;
                    }
                    const double ri = rsqrt(d);
                    a[j / 2] = d * ri;
                    rinv[j] = ri;
                }
                potrf_bar();
                if ((j & 1) == H && row > j) {
                    a[j / 2] *= rinv[j];               // L[row][j]
                    colj[row] = a[j / 2];
                }
                potrf_bar();
                if (row > j) {
                    const double l = colj[row];
                    #pragma unroll
                    for (int c = j + 1; c < CB; ++c)   // c > row: never read (upper part)
                        if ((c & 1) == H) a[c / 2] -= l * colj[c];
                }
                potrf_bar();                           // colj is rewritten by the next pivot
            }
            #pragma unroll
            for (int i = 0; i < CB / 2; ++i) D[row][2 * i + H] = 2 * i + H <= row ? a[i] : 0.0;
        };
        if (t < CB) factor_rows(std::integral_constant<int, 0>{});
        else factor_rows(std::integral_constant<int, 1>{});
    } else if (FACTOR) {                               // meanwhile warps 4-7 copy the panel rows
        // in batches whose loads are all issued before their stores: the band and the panel share
        // one workspace, so the compiler may not move a load above an earlier store by itself
        constexpr int CPB = 16, CPT = POTRF_T - FT;
        const int total = (rend - base) * CB;
        for (int i0 = t - FT; i0 < total; i0 += CPB * CPT) {
            double v[CPB];
            #pragma unroll
            for (int u = 0; u < CPB; ++u) {
                const int i = i0 + u * CPT, r = base + i / CB, c = i % CB, col = k0 + c;
                v[u] = (i < total && c < w && r - col <= bw) ? lb[bidx(r, col, bw)] : 0.0;
            }
            #pragma unroll
            for (int u = 0; u < CPB; ++u)
                if (i0 + u * CPT < total) apanel[i0 + u * CPT] = v[u];
        }
    }
    __syncthreads();
    // X = L^-1 by 32 x 32 blocks: X11 (warp 0) and X22 (warp 1) by forward substitution, lane = column,
    // in registers; then X21 = -X22 (L21 X11) by all threads
    if (t < 2 * HB) {
        const int o = (t / HB) * HB, c = t % HB;
        double x[HB];
        #pragma unroll
        for (int r = 0; r < HB; ++r) {
            double s[4] = {0.0, 0.0, 0.0, 0.0};
            #pragma unroll
            for (int p = 0; p < r; ++p) s[p & 3] += D[o + r][o + p] * x[p];
            x[r] = ((r == c ? 1.0 : 0.0) - ((s[0] + s[1]) + (s[2] + s[3]))) * rinv[o + r];
        }
        #pragma unroll
        for (int r = 0; r < HB; ++r) X[o + r][o + c] = x[r];
    } else {
        for (int i = t - 2 * HB; i < HB * HB; i += POTRF_T - 2 * HB) X[i / HB][HB + i % HB] = 0.0;
    }
    __syncthreads();
    const int tc = t % HB, tr = t / HB;                // column and first row of this thread's outputs
    constexpr int NR = HB * HB / POTRF_T;              // outputs per thread, rows tr + RS m
    constexpr int RS = POTRF_T / HB;
    {
        double s[NR];
        #pragma unroll
        for (int m = 0; m < NR; ++m) s[m] = 0.0;
        #pragma unroll
        for (int p = 0; p < HB; ++p) {                 // Tm = L21 X11
            const double xv = X[p][tc];
            #pragma unroll
            for (int m = 0; m < NR; ++m) s[m] += D[HB + tr + RS * m][p] * xv;
        }
        #pragma unroll
        for (int m = 0; m < NR; ++m) Tm[tr + RS * m][tc] = s[m];
    }
    __syncthreads();
    {
        double s[NR];
        #pragma unroll
        for (int m = 0; m < NR; ++m) s[m] = 0.0;
        #pragma unroll
        for (int p = 0; p < HB; ++p) {                 // X21 = -X22 Tm (X22 lower triangular, zeros above)
            const double tv = Tm[p][tc];
            #pragma unroll
            for (int m = 0; m < NR; ++m) s[m] += X[HB + tr + RS * m][HB + p] * tv;
        }
        #pragma unroll
        for (int m = 0; m < NR; ++m) X[HB + tr + RS * m][tc] = -s[m];
    }
    __syncthreads();
    #pragma unroll
    for (int i = t; i < CB * CB; i += POTRF_T) {
        const int r = i / CB, c = i % CB;
        if (FACTOR && r < w && c <= r && r - c <= bw) lb[bidx(k0 + r, k0 + c, bw)] = D[r][c];
        dinv[i] = (r < w && c < w) ? X[r][c] : 0.0;
    }
}

// One quadrant (qa, qb) of a lower tile (I, J) of the rows below block column k0, CTA 4 tile + 2 qa + qb:
// rows ri = base + I CB + UQ qa + r, rj = base + J CB + UQ qb + c (r, c < UQ), base = k0 + w.  Four
// CTAs per tile (each needs only its UQ rows of the two panels) keep the chain step short: about
// 0.33M multiply-adds per CTA instead of 0.79M for a whole tile.  Dynamic shared memory: the block
// inverse (CB x CBP) and the two half panels (2 UQ x CBP).  Thread t: rows t / 16 + 16 a, columns
// t % 16 + 16 b of each product (a < 2; b < 4 for the panels, b < 2 for the trailing update), so the
// accumulations run as independent chains.  The upper quadrant of a diagonal tile has nothing below
// the diagonal and returns at once; its lower-left quadrants store the finished panel rows.
constexpr int UQ = CB / 2;
__global__ void __launch_bounds__(UPDATE_T) band_update_kernel(int n, int bw, int k0, int tiles,
                                                               const __grid_constant__ FactorBatch fb) {
    static_assert(UPDATE_T == 256 && CB == 64, "16 x 16 threads over 32-row quadrants");
    vx::pdl_begin();
    const FactorPtrs P = fptrs(fb, n, bw);
    double* __restrict__ lb = P.lb;
    const double* __restrict__ dinv = P.dinv_all + int64_t(k0 / CB) * CB * CB;
    const double* __restrict__ apanel = P.apanel;
    extern __shared__ __align__(16) double sm[];
    double (*Xi)[CBP] = reinterpret_cast<double (*)[CBP]>(sm);
    double (*PI)[CBP] = reinterpret_cast<double (*)[CBP]>(sm + CB * CBP);
    double (*PJ)[CBP] = reinterpret_cast<double (*)[CBP]>(sm + (CB + UQ) * CBP);
    const int tile = int(blockIdx.x) >> 2, qa = (int(blockIdx.x) >> 1) & 1, qb = int(blockIdx.x) & 1;
    int I = 0, rem = tile;                             // tile index -> (I, J), I >= J
    while (rem > I) { rem -= I + 1; ++I; }
    const int J = rem;
    if (I == J && qa < qb) return;                     // upper quadrant of a diagonal tile
    const bool same = I == J && qa == qb;              // both panels are the same rows
    const int w = min(CB, n - k0);
    const int base = k0 + w;
    const int rend = min(n, k0 + w + bw);              // rows the block column reaches
    const int ri0 = base + I * CB + UQ * qa, rj0 = base + J * CB + UQ * qb;
    if (ri0 >= rend) return;                           // the quadrant lies beyond the reach (rj0 <= ri0)
    #pragma unroll
    for (int u = 0; u < CB * CB / UPDATE_T; ++u) {
        const int i = threadIdx.x + u * UPDATE_T;
        Xi[i / CB][i % CB] = dinv[i];
    }
    #pragma unroll
    for (int u = 0; u < UQ * CB / UPDATE_T; ++u) {
        const int i = threadIdx.x + u * UPDATE_T, r = i / CB, c = i % CB;
        const int ri = ri0 + r, rj = rj0 + r;
        PI[r][c] = ri < rend ? apanel[int64_t(ri - base) * CB + c] : 0.0;
        if (!same) PJ[r][c] = rj < rend ? apanel[int64_t(rj - base) * CB + c] : 0.0;
    }
    __syncthreads();
    const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
    // panels: P <- P X^T, P[r][m] = sum_p A[r][p] X[m][p] (X lower triangular: the full sum is exact)
    double oi[2][4], oj[2][4];
    #pragma unroll
    for (int a = 0; a < 2; ++a) {
        #pragma unroll
        for (int b = 0; b < 4; ++b) { oi[a][b] = 0.0; oj[a][b] = 0.0; }
    }
    if (same) {
        #pragma unroll 4
        for (int p = 0; p < CB; ++p) {
            double ai[2], x[4];
            #pragma unroll
            for (int a = 0; a < 2; ++a) ai[a] = PI[tr + 16 * a][p];
            #pragma unroll
            for (int b = 0; b < 4; ++b) x[b] = Xi[tc + 16 * b][p];
            #pragma unroll
            for (int a = 0; a < 2; ++a) {
                #pragma unroll
                for (int b = 0; b < 4; ++b) oi[a][b] = fma(ai[a], x[b], oi[a][b]);
            }
        }
    } else {
        #pragma unroll 4
        for (int p = 0; p < CB; ++p) {
            double ai[2], aj[2], x[4];
            #pragma unroll
            for (int a = 0; a < 2; ++a) { ai[a] = PI[tr + 16 * a][p]; aj[a] = PJ[tr + 16 * a][p]; }
            #pragma unroll
            for (int b = 0; b < 4; ++b) x[b] = Xi[tc + 16 * b][p];
            #pragma unroll
            for (int a = 0; a < 2; ++a) {
                #pragma unroll
                for (int b = 0; b < 4; ++b) {
                    oi[a][b] = fma(ai[a], x[b], oi[a][b]);
                    oj[a][b] = fma(aj[a], x[b], oj[a][b]);
                }
            }
        }
    }
    __syncthreads();
    #pragma unroll
    for (int a = 0; a < 2; ++a) {
        #pragma unroll
        for (int b = 0; b < 4; ++b) {
            PI[tr + 16 * a][tc + 16 * b] = oi[a][b];
            if (!same) PJ[tr + 16 * a][tc + 16 * b] = oj[a][b];
        }
    }
    __syncthreads();
    double (*QJ)[CBP] = same ? PI : PJ;
    if (I == J && qb == 0) {                           // these panel rows of tile I are final: store them
        for (int t = threadIdx.x; t < UQ * CB; t += UPDATE_T) {
            const int r = t / CB, c = t % CB, ri = ri0 + r, col = k0 + c;
            if (c < w && ri < rend && ri - col <= bw) lb[bidx(ri, col, bw)] = PI[r][c];
        }
    }
    // trailing update of the quadrant: A[ri][rj] -= sum_m L[ri][m] L[rj][m] (lower triangle, in the band)
    double o[2][2];
    #pragma unroll
    for (int a = 0; a < 2; ++a) {
        #pragma unroll
        for (int b = 0; b < 2; ++b) o[a][b] = 0.0;
    }
    #pragma unroll 4
    for (int m = 0; m < CB; ++m) {
        double pi[2], pj[2];
        #pragma unroll
        for (int a = 0; a < 2; ++a) pi[a] = PI[tr + 16 * a][m];
        #pragma unroll
        for (int b = 0; b < 2; ++b) pj[b] = QJ[tc + 16 * b][m];
        #pragma unroll
        for (int a = 0; a < 2; ++a) {
            #pragma unroll
            for (int b = 0; b < 2; ++b) o[a][b] = fma(pi[a], pj[b], o[a][b]);
        }
    }
    double cur[2][2];                                  // every old value read before any write
    #pragma unroll
    for (int a = 0; a < 2; ++a) {
        #pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int ri = ri0 + tr + 16 * a, rj = rj0 + tc + 16 * b;
            const bool in = ri < rend && rj < rend && rj <= ri && ri - rj <= bw;
            cur[a][b] = in ? lb[bidx(ri, rj, bw)] : 0.0;
        }
    }
    #pragma unroll
    for (int a = 0; a < 2; ++a) {
        #pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int ri = ri0 + tr + 16 * a, rj = rj0 + tc + 16 * b;
            if (ri >= rend || rj >= rend || rj > ri || ri - rj > bw) continue;
            lb[bidx(ri, rj, bw)] = cur[a][b] - o[a][b];
        }
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
__global__ void band_inverse_kernel(int n, int bw, const __grid_constant__ FactorBatch fb) {
    vx::pdl_begin();
    const FactorPtrs P = fptrs(fb, n, bw);
    const double* __restrict__ lb = P.lb;
    double* __restrict__ packed = P.packed;
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

// X = L^-1 by blocks of IRB rows for TC columns per CTA (columns c0 .. c0 + TC - 1).  Walking down
// the row blocks i0 = IRB floor(c0 / IRB), + IRB, ...:
//     S   = L[i0 .. i0 + IRB)[i0 - bw .. i0) X[i0 - bw .. i0)[cols]     (the band left of the block)
//     X_I = Dinv_I (E_I - S)                                          (E_I: the identity's rows)
// with Dinv_I the inverse of L's IRB x IRB diagonal block (the diagonal sub-blocks of the CB-block
// inverses band_potrf kept, dinv_all).  The last WR >= bw + IRB rows of X for these columns live in a
// shared-memory ring (rows above c0 are zero and never written); the band rows of L are staged per
// block, transposed; S is a band GEMM split over the warps along the band (a 4 x 4 register tile per
// lane); each finished block goes to M[i][j] (rows, coalesced over columns) and, through shared
// memory, to M[j][i] (coalesced over rows).  Thread t: column t % TC, rows t / TC + (INVB_T / TC) m.
// The first CTA's walk over all n / IRB row blocks is the critical path, and each step's band product
// (IRB x bw x TC multiply-adds on one SM) sets its length: INV_TC = 16 columns per CTA halves the step
// of 32 columns for twice the CTAs (the band rows are staged by each CTA, from L2).
constexpr int IRB = 32, INVB_T = 256, INV_TC = 16;
constexpr int LTP = IRB + 2;   // row of the transposed band stage: 16-byte aligned, stores 4-way at most

template <int TC>
struct InvbLayout {
    int bw, WR;
    size_t ls, ring, dv, st, red, bytes;
    __host__ __device__ explicit InvbLayout(int bw_) : bw(bw_) {
        WR = (bw + IRB + IRB - 1) / IRB * IRB;
        ls = size_t(bw) * LTP;                       // staged band rows, transposed: [q][row]
        ring = size_t(WR) * TC;
        dv = size_t(IRB) * (IRB + 1);
        st = size_t(IRB) * (TC + 1);
        red = size_t(INVB_T / 32) * IRB * TC;        // per-warp partial products
        bytes = (ls + ring + dv + st + red) * sizeof(double);
    }
};

template <int TC>
__global__ void __launch_bounds__(INVB_T) band_inverse_blocked_kernel(int n, int bw, const __grid_constant__ FactorBatch fb) {
    static_assert(TC >= 8 && TC <= 32 && INVB_T % TC == 0 && IRB * TC % INVB_T == 0, "thread layout");
    constexpr int RG = INVB_T / TC;                    // row groups
    constexpr int MR = IRB / RG;                       // rows per thread
    vx::pdl_begin();
    const FactorPtrs P = fptrs(fb, n, bw);
    const double* __restrict__ lb = P.lb;
    const double* __restrict__ dinv_all = P.dinv_all;
    double* __restrict__ packed = P.packed;
    extern __shared__ __align__(16) double sm[];
    const InvbLayout<TC> Lo(bw);
    double* Ls = sm;                                   // [bw][LTP]: Ls[q][r] = L[i0 + r][i0 - bw + q], q < bw
    double* Wr = Ls + Lo.ls;                           // [WR][TC] ring of X rows
    double* Dv = Wr + Lo.ring;                         // [IRB][IRB + 1]
    double* St = Dv + Lo.dv;                           // [IRB][TC + 1]
    double* Red = St + Lo.st;                          // [warps][IRB x TC] partial band products
    const int t = threadIdx.x, c = t % TC, rg = t / TC, lane = t & 31, wid = t >> 5;
    const int c0 = blockIdx.x * TC;
    const int WR = Lo.WR;
    for (int i = t; i < WR * TC; i += INVB_T) Wr[i] = 0.0;
    // row blocks aligned to IRB (the diagonal block inverses are IRB-aligned sub-blocks of the CB-block
    // inverses); rows above c0 come out zero for these columns
    for (int i0 = c0 / IRB * IRB; i0 < n; i0 += IRB) {
        __syncthreads();                               // the previous block's reads of Ls, Dv, St are done
        // stage the band rows (zero outside row i's band and beyond n), transposed, and the diagonal
        // block inverse: warp w copies rows w, w + 8, ..., lanes along the row.  The staging is on the
        // chain of every block step, so each thread issues all of its loads (up to SQ 32-column
        // chunks of its four rows, one round trip for bands up to 32 SQ wide) before any store.
        constexpr int SQ = 9;
        const double* dsrc = dinv_all + int64_t(i0 / CB) * CB * CB + (i0 % CB) * CB + (i0 % CB);
        double dv[IRB * IRB / INVB_T];
        #pragma unroll
        for (int u = 0; u < IRB * IRB / INVB_T; ++u) {
            const int i = t + u * INVB_T, r = i / IRB, k = i % IRB;
            dv[u] = (k <= r) ? dsrc[r * CB + k] : 0.0;
        }
        for (int qb = 0; qb < bw; qb += 32 * SQ) {
            double v[4][SQ];
            #pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int rr = wid + 8 * j, row = i0 + rr;
                const double* src = lb + int64_t(row) * (bw + 1) - rr;   // src[q] = L[row][i0 - bw + q]
                #pragma unroll
                for (int u = 0; u < SQ; ++u) {
                    const int q = qb + lane + 32 * u;
                    v[j][u] = (q < bw && q >= rr && row < n) ? src[q] : 0.0;
                }
            }
            #pragma unroll
            for (int j = 0; j < 4; ++j)
                #pragma unroll
                for (int u = 0; u < SQ; ++u) {
                    const int q = qb + lane + 32 * u;
                    if (q < bw) Ls[q * LTP + wid + 8 * j] = v[j][u];
                }
        }
        #pragma unroll
        for (int u = 0; u < IRB * IRB / INVB_T; ++u) {
            const int i = t + u * INVB_T;
            Dv[(i / IRB) * (IRB + 1) + i % IRB] = dv[u];
        }
        __syncthreads();
        // S = Ls X_window over the band columns that can be non-zero (rows >= c0): warp w takes the
        // w-th eighth of those columns for the whole IRB x TC block, lane = a 4 x 4 register tile
        // (rows 4 (lane / 4) .., columns 4 (lane % 4) ..) read as 16-byte pairs from the transposed
        // band stage and the ring; the warps' partial tiles are then summed through shared memory.
        static_assert(IRB == 32 && TC == 16 && INVB_T == 256, "8 warps x 32 lanes x 4 x 4 tiles cover 32 x 16");
        {
            const int q0 = max(0, c0 - (i0 - bw));
            const int len = bw - q0, chunk = (len + 7) / 8;
            const int qs = q0 + wid * max(chunk, 0), qe = min(bw, qs + max(chunk, 0));
            const int tr = 4 * (lane >> 2), tcol = 4 * (lane & 3);
            double acc[4][4];
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                #pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
            int slot = (i0 - bw + qs) % WR;
            if (slot < 0) slot += WR;
            #pragma unroll 2
            for (int q = qs; q < qe; ++q) {
                const double2 l01 = *reinterpret_cast<const double2*>(Ls + q * LTP + tr);
                const double2 l23 = *reinterpret_cast<const double2*>(Ls + q * LTP + tr + 2);
                const double2 w01 = *reinterpret_cast<const double2*>(Wr + slot * TC + tcol);
                const double2 w23 = *reinterpret_cast<const double2*>(Wr + slot * TC + tcol + 2);
                const double l[4] = {l01.x, l01.y, l23.x, l23.y}, x[4] = {w01.x, w01.y, w23.x, w23.y};
                #pragma unroll
                for (int i = 0; i < 4; ++i)
                    #pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] += l[i] * x[j];
                if (++slot == WR) slot = 0;
            }
            double* rw = Red + wid * (IRB * TC);
            #pragma unroll
            for (int i = 0; i < 4; ++i)
                #pragma unroll
                for (int j = 0; j < 4; ++j) rw[(tr + i) * TC + tcol + j] = acc[i][j];
        }
        __syncthreads();
        #pragma unroll
        for (int m = 0; m < MR; ++m) {
            const int r = rg + RG * m;
            double sum = 0.0;
            #pragma unroll
            for (int w = 0; w < INVB_T / 32; ++w) sum += Red[w * (IRB * TC) + r * TC + c];
            St[r * (TC + 1) + c] = ((i0 + r == c0 + c) ? 1.0 : 0.0) - sum;
        }
        __syncthreads();
        // X_I = Dinv_I (E_I - S)
        double x[MR];
        #pragma unroll
        for (int m = 0; m < MR; ++m) {
            const int r = rg + RG * m;
            double a0 = 0.0, a1 = 0.0;
            int k = 0;
            for (; k + 1 <= r; k += 2) {
                a0 += Dv[r * (IRB + 1) + k] * St[k * (TC + 1) + c];
                a1 += Dv[r * (IRB + 1) + k + 1] * St[(k + 1) * (TC + 1) + c];
            }
            if (k == r) a0 += Dv[r * (IRB + 1) + k] * St[k * (TC + 1) + c];
            x[m] = a0 + a1;
        }
        __syncthreads();                               // every read of St done before it holds X_I
        #pragma unroll
        for (int m = 0; m < MR; ++m) {
            const int r = rg + RG * m, i = i0 + r, j = c0 + c;
            const bool ok = i < n && j < n && i >= j;
            const double v = ok ? x[m] : 0.0;
            int ws = i % WR;
            Wr[ws * TC + c] = v;
            St[r * (TC + 1) + c] = v;
            if (ok) packed[int64_t(i) * n + j] = v;    // lower part, coalesced over columns
        }
        __syncthreads();
        // upper part M[j][i] = X[i][j], coalesced over rows: lane = row of the block
        #pragma unroll
        for (int m = 0; m < TC / 8; ++m) {
            const int cc = wid + 8 * m, r = lane, i = i0 + r, j = c0 + cc;
            if (i < n && j < n && i > j) packed[int64_t(j) * n + i] = St[r * (TC + 1) + cc];
        }
    }
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
    const int64_t nblk = (n + CB - 1) / CB;
    return int64_t(n) * (bw + 1) + nblk * CB * CB + int64_t(bw + 1) * CB;
}

// count factorisations of one size (matrix slots slots[0..count) of A, packed and info; workspace m
// of work for the m-th), every launch covering all of them (blockIdx.y).
static int coarse_factor_batch(const char* what, int n, int bw, int count, const int* slots, const double* A,
                               double* packed, double* work, int* info, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0 && bw >= 0, VX_ERR_INVALID_ARGUMENT, "%s: bad size n=%d bw=%d", what, n, bw);
    VX_CHECK_ARG(A && packed && work && info, VX_ERR_NULL_POINTER, "%s: NULL pointer", what);
    VX_CHECK_ARG(A != packed, VX_ERR_INVALID_ARGUMENT, "%s: packed may not alias A", what);
    VX_CHECK_ARG(count >= 1 && count <= FB_MAX, VX_ERR_INVALID_ARGUMENT, "%s: count %d outside 1..%d", what, count,
                 FB_MAX);
    bw = std::min(bw, n - 1);
    const int nw = inverse_warps(bw);
    VX_CHECK_ARG(nw > 0, VX_ERR_INVALID_ARGUMENT, "%s: bandwidth %d is too wide", what, bw);
    FactorBatch fb{};
    fb.A = A;
    fb.packed = packed;
    fb.work = work;
    fb.info = info;
    fb.mat = int64_t(n) * n;
    fb.ws = vx_coarse_factor_workspace(n, bw);
    fb.nblk = (n + CB - 1) / CB;
    for (int m = 0; m < count; ++m) {
        VX_CHECK_ARG(slots[m] >= 0, VX_ERR_INVALID_ARGUMENT, "%s: negative slot", what);
        fb.slot[m] = slots[m];
        cudaError_t e = cudaMemsetAsync(info + slots[m], 0, sizeof(int), stream);
        if (e != cudaSuccess) {
            set_error("%s: memset: %s", what, cudaGetErrorString(e));
            return VX_ERR_CUDA;
        }
    }
    const size_t psm = size_t(2 * CB * CBP + HB * HBP) * sizeof(double);
    const size_t usm = size_t(CB + 2 * UQ) * CBP * sizeof(double);
    const size_t ism = size_t(INV_STAGES + nw) * (bw + 1) * sizeof(double);
    static std::atomic<uint64_t> opt_p, opt_u, opt_i, opt_b;
    int st = smem_opt_in(opt_p, (const void*)band_potrf_kernel<true>, psm, what);
    if (!st) st = smem_opt_in(opt_u, (const void*)band_update_kernel, usm, what);
    if (!st) st = smem_opt_in(opt_i, (const void*)band_inverse_kernel, 227 * 1024, what);
    if (!st) st = smem_opt_in(opt_b, (const void*)band_inverse_blocked_kernel<INV_TC>, 227 * 1024, what);
    if (st) return st;
    const unsigned B = unsigned(count);
    const int64_t band = int64_t(n) * (bw + 1);
    vx::launch(band_load_kernel, dim3(unsigned((band + 255) / 256), B), 256, 0, stream, n, bw, fb);
    for (int k0 = 0; k0 < n; k0 += CB) {
        vx::launch(band_potrf_kernel<true>, dim3(1, B), POTRF_T, psm, stream, n, bw, k0, fb);
        const int w = std::min(CB, n - k0);
        const int rows = std::min(n, k0 + w + bw) - (k0 + w);
        if (rows <= 0) continue;
        const int T = (rows + CB - 1) / CB;
        vx::launch(band_update_kernel, dim3(unsigned(4 * (T * (T + 1) / 2)), B), UPDATE_T, usm, stream, n, bw, k0, T, fb);
    }
    const InvbLayout<INV_TC> il(bw);
    if (il.bytes <= 227 * 1024) {
        vx::launch(band_inverse_blocked_kernel<INV_TC>, dim3(unsigned((n + INV_TC - 1) / INV_TC), B), INVB_T, il.bytes, stream, n,
                   bw, fb);
    } else {
        vx::launch(band_inverse_kernel, dim3(unsigned((n + nw - 1) / nw), B), unsigned(nw * 32), ism, stream, n, bw,
                   fb);
    }
    VX_CHECK_LAUNCH(what);
    return VX_OK;
}

extern "C" int vx_coarse_factor(int n, int bw, const double* A, double* packed, double* work, int* info,
                                cudaStream_t stream) {
    const int slot0 = 0;
    return coarse_factor_batch("vx_coarse_factor", n, bw, 1, &slot0, A, packed, work, info, stream);
}

// Several coarsest systems of one size at once (the serving batches' per-job coarse solves): slots
// are host indices into the matrix stacks A / packed (n x n each) and info; work holds count
// workspaces of vx_coarse_factor_workspace(n, bw) doubles.
extern "C" int vx_batch_coarse_factor(int n, int bw, int count, const int* slots, const double* A, double* packed,
                                      double* work, int* info, cudaStream_t stream) {
    VX_CHECK_ARG(slots, VX_ERR_NULL_POINTER, "vx_batch_coarse_factor: NULL slots");
    VX_CHECK_ARG(count >= 1, VX_ERR_INVALID_ARGUMENT, "vx_batch_coarse_factor: count %d", count);
    for (int c0 = 0; c0 < count; c0 += FB_MAX) {      // chunks reuse the workspaces, in stream order
        const int st = coarse_factor_batch("vx_batch_coarse_factor", n, bw, std::min(FB_MAX, count - c0), slots + c0, A,
                                           packed, work, info, stream);
        if (st) return st;
    }
    return VX_OK;
}

// The packed inverse factor from a Cholesky factor the caller already has (dense row-major lower
// triangle, half-bandwidth bw): the band is loaded from L, every diagonal block inverted in one
// launch, then the blocked band inverse.  work: vx_coarse_factor_workspace(n, bw) doubles.
extern "C" int vx_coarse_pack_factor(int n, int bw, const double* L, double* packed, double* work,
                                     cudaStream_t stream) {
    const char* what = "vx_coarse_pack_factor";
    VX_CHECK_ARG(n > 0 && bw >= 0, VX_ERR_INVALID_ARGUMENT, "%s: bad size n=%d bw=%d", what, n, bw);
    VX_CHECK_ARG(L && packed && work, VX_ERR_NULL_POINTER, "%s: NULL pointer", what);
    VX_CHECK_ARG(L != packed, VX_ERR_INVALID_ARGUMENT, "%s: packed may not alias L", what);
    bw = std::min(bw, n - 1);
    const int nw = inverse_warps(bw);
    VX_CHECK_ARG(nw > 0, VX_ERR_INVALID_ARGUMENT, "%s: bandwidth %d is too wide", what, bw);
    FactorBatch fb{};
    fb.A = L;
    fb.packed = packed;
    fb.work = work;
    fb.info = nullptr;
    fb.mat = int64_t(n) * n;
    fb.ws = vx_coarse_factor_workspace(n, bw);
    fb.nblk = (n + CB - 1) / CB;
    fb.slot[0] = 0;
    const size_t psm = size_t(2 * CB * CBP + HB * HBP) * sizeof(double);
    const size_t ism = size_t(INV_STAGES + nw) * (bw + 1) * sizeof(double);
    static std::atomic<uint64_t> opt_p, opt_i, opt_b;
    int st = smem_opt_in(opt_p, (const void*)band_potrf_kernel<false>, psm, what);
    if (!st) st = smem_opt_in(opt_i, (const void*)band_inverse_kernel, 227 * 1024, what);
    if (!st) st = smem_opt_in(opt_b, (const void*)band_inverse_blocked_kernel<INV_TC>, 227 * 1024, what);
    if (st) return st;
    const int64_t band = int64_t(n) * (bw + 1);
    vx::launch(band_load_kernel, dim3(unsigned((band + 255) / 256), 1), 256, 0, stream, n, bw, fb);
    vx::launch(band_potrf_kernel<false>, dim3(unsigned(fb.nblk), 1), POTRF_T, psm, stream, n, bw, 0, fb);
    const InvbLayout<INV_TC> il(bw);
    if (il.bytes <= 227 * 1024) {
        vx::launch(band_inverse_blocked_kernel<INV_TC>, dim3(unsigned((n + INV_TC - 1) / INV_TC), 1), INVB_T, il.bytes, stream, n,
                   bw, fb);
    } else {
        vx::launch(band_inverse_kernel, dim3(unsigned((n + nw - 1) / nw), 1), unsigned(nw * 32), ism, stream, n, bw,
                   fb);
    }
    VX_CHECK_LAUNCH(what);
    return VX_OK;
}
