// Multigrid kernels of the rediscretised voxel hierarchy: trilinear restriction / prolongation,
// modulus and mask coarsening, dense coarse assembly and the dense coarse solve.
// The transfers evaluate the separable per-axis passes in the reference's order (x, then y,
// then z; restriction adds the right neighbour before the left), so FP64 results agree with the
// reference's NumPy transfers to the last bit or within an ulp.
#include "vx_common.cuh"

namespace vx {

__device__ __forceinline__ void node_coords(const Grid& g, int64_t n, int& ix, int& iy, int& iz) {
    iz = int(n % (g.nz + 1));
    iy = int((n / (g.nz + 1)) % (g.ny + 1));
    ix = int(n / (int64_t(g.nz + 1) * (g.ny + 1)));
}

// Launch shape of the restriction: threads along z (TZ_T x TY_T per CTA), grid (z chunks, y rows /
// TY_T, x planes), so no thread divides to find its node; offsets in 32 bits (fewer than 2^31 DOFs).
constexpr int TZ_T = 64, TY_T = 2;
inline dim3 transfer_grid(const Grid& g) {
    return dim3(unsigned((g.nz + 1 + TZ_T - 1) / TZ_T), unsigned((g.ny + 1 + TY_T - 1) / TY_T), unsigned(g.nx + 1));
}
__device__ __forceinline__ int node32(const Grid& g, int ix, int iy, int iz) { return (ix * (g.ny + 1) + iy) * (g.nz + 1) + iz; }

// coarse node (I,J,K) of fine grid f: rc = sum w(a) w(b) w(d) f(2I+a, 2J+b, 2K+d), w(0)=1, w(+-1)=1/2.
// Arithmetic in arith_t<T> (bf16 storage: FP32).
template <typename T>
__global__ void __launch_bounds__(TZ_T * TY_T) restrict_kernel(Grid f, Grid c, const T* __restrict__ fine,
                                                              const uint8_t* __restrict__ cmask, T* __restrict__ coarse) {
    vx::pdl_begin();
    using A = arith_t<T>;
    const int K = blockIdx.x * TZ_T + threadIdx.x, J = blockIdx.y * TY_T + threadIdx.y, I = blockIdx.z;
    if (K > c.nz || J > c.ny) return;
    const int n = node32(c, I, J, K);
    const unsigned bits = cmask ? unsigned(cmask[n]) : 7u;
    auto ld = [&](int i) { return Storage<T>::load(fine + i); };
    for (int comp = 0; comp < 3; ++comp) {
        A ty[3][3];   // after the x pass, at fine (y = 2J + b - 1, z = 2K + d - 1)
        for (int b = 0; b < 3; ++b)
            for (int d = 0; d < 3; ++d) {
                const int fy = 2 * J + b - 1, fz = 2 * K + d - 1;
                A v = A(0);
                if (fy >= 0 && fy <= f.ny && fz >= 0 && fz <= f.nz) {
                    v = ld(3 * node32(f, 2 * I, fy, fz) + comp);
                    if (2 * I + 1 <= f.nx) v = v + A(0.5) * ld(3 * node32(f, 2 * I + 1, fy, fz) + comp);
                    if (I >= 1) v = v + A(0.5) * ld(3 * node32(f, 2 * I - 1, fy, fz) + comp);
                }
                ty[b][d] = v;
            }
        A tz[3];
        for (int d = 0; d < 3; ++d) {
            A v = ty[1][d];
            if (2 * J + 1 <= f.ny) v = v + A(0.5) * ty[2][d];
            if (J >= 1) v = v + A(0.5) * ty[0][d];
            tz[d] = v;
        }
        A v = tz[1];
        if (2 * K + 1 <= f.nz) v = v + A(0.5) * tz[2];
        if (K >= 1) v = v + A(0.5) * tz[0];
        Storage<T>::store(coarse + 3 * n + comp, ((bits >> comp) & 1u) ? v : A(0));
    }
}

// x(i,j,k) += (P ec)(i,j,k) * mask; P is the separable trilinear interpolation.  One thread per fine
// node in a 1-D launch: consecutive threads read and write consecutive nodes of x (measured faster
// than the 3-D launch of the restriction, whose threads gather from three fine planes).
template <typename T>
__global__ void prolong_add_kernel(Grid f, Grid c, const T* __restrict__ coarse, const uint8_t* __restrict__ fmask,
                                   T* __restrict__ x) {
    vx::pdl_begin();
    using A = arith_t<T>;
    const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= f.nodes()) return;
    int i, j, k;
    node_coords(f, n, i, j, k);
    const unsigned bits = fmask ? unsigned(fmask[n]) : 7u;
    const int I0 = i >> 1, J0 = j >> 1, K0 = k >> 1;
    const bool ox = i & 1, oy = j & 1, oz = k & 1;
    for (int comp = 0; comp < 3; ++comp) {
        A py[2];
        for (int d = 0; d <= int(oz); ++d) {
            A px[2];
            for (int b = 0; b <= int(oy); ++b) {
                const int64_t a0 = 3 * c.node(I0, J0 + b, K0 + d) + comp;
                const A c0 = Storage<T>::load(coarse + a0);
                px[b] = ox ? A(0.5) * (c0 + Storage<T>::load(coarse + a0 + 3 * int64_t(c.ny + 1) * (c.nz + 1))) : c0;
            }
            py[d] = oy ? A(0.5) * (px[0] + px[1]) : px[0];
        }
        const A v = oz ? A(0.5) * (py[0] + py[1]) : py[0];
        if ((bits >> comp) & 1u) Storage<T>::store(x + 3 * n + comp, Storage<T>::load(x + 3 * n + comp) + v);
    }
}

template <typename S>
__global__ void coarsen_modulus_kernel(Grid f, Grid c, const S* __restrict__ Ef, S* __restrict__ Ec) {
    vx::pdl_begin();
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= c.elems()) return;
    const int ez = int(e % c.nz), ey = int((e / c.nz) % c.ny), ex = int(e / (int64_t(c.nz) * c.ny));
    double s = 0.0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int d = 0; d < 2; ++d) s += double(Storage<S>::load(Ef + f.elem(2 * ex + a, 2 * ey + b, 2 * ez + d)));
    Storage<S>::store(Ec + e, decltype(Storage<S>::load(Ef))(s * 0.125));
}

__global__ void coarsen_mask_kernel(Grid f, Grid c, const uint8_t* __restrict__ mf, uint8_t* __restrict__ mc) {
    vx::pdl_begin();
    const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= c.nodes()) return;
    int I, J, K;
    node_coords(c, n, I, J, K);
    mc[n] = mf[f.node(2 * I, 2 * J, 2 * K)];
}

struct Ke576 { double k[576]; };

// one thread per (row DOF, neighbour offset, column component); A is zeroed beforehand
__global__ void assemble_dense_kernel(Grid g, const __grid_constant__ Ke576 ke, const double* __restrict__ E,
                                      const uint8_t* __restrict__ mask, double* __restrict__ A) {
    vx::pdl_begin();
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t nn = g.nodes();
    if (t >= nn * 3 * 81) return;
    const int64_t row = t / 81;
    const int rem = int(t % 81);
    const int off = rem / 3, cd = rem % 3;
    const int64_t nr = row / 3;
    const int cr = int(row % 3);
    int ix, iy, iz;
    node_coords(g, nr, ix, iy, iz);
    const int ox = off % 3 - 1, oy = (off / 3) % 3 - 1, oz = off / 9 - 1;
    const int mx = ix + ox, my = iy + oy, mz = iz + oz;
    if (mx < 0 || mx > g.nx || my < 0 || my > g.ny || mz < 0 || mz > g.nz) return;
    constexpr int nat[8] = {0, 1, 3, 2, 4, 5, 7, 6};
    double v = 0.0;
    for (int bx = 0; bx < 2; ++bx) for (int by = 0; by < 2; ++by) for (int bz = 0; bz < 2; ++bz) {
        const int ex = ix - 1 + bx, ey = iy - 1 + by, ez = iz - 1 + bz;   // element containing the row node
        if (ex < 0 || ex >= g.nx || ey < 0 || ey >= g.ny || ez < 0 || ez >= g.nz) continue;
        const int qx = mx - ex, qy = my - ey, qz = mz - ez;              // column node's offset in it
        if (qx < 0 || qx > 1 || qy < 0 || qy > 1 || qz < 0 || qz > 1) continue;
        const int li = nat[(1 - bx) + 2 * (1 - by) + 4 * (1 - bz)];
        const int lj = nat[qx + 2 * qy + 4 * qz];
        v += E[g.elem(ex, ey, ez)] * ke.k[(3 * li + cr) * 24 + 3 * lj + cd];
    }
    const int64_t col = 3 * g.node(mx, my, mz) + cd;
    const double mr = mask ? double((mask[nr] >> cr) & 1u) : 1.0;
    const double mcv = mask ? double((mask[col / 3] >> cd) & 1u) : 1.0;
    double out = mr * v * mcv;
    if (col == row) out += 1.0 - mr;
    A[row * (nn * 3) + col] = out;
}

// sum over j in [j0, j1) of row[j] * v(j) by one CTA of CT threads (stride CT), reduced in a fixed
// order.  A CTA per row keeps each thread's dependent chain short: with a warp per row, every warp
// is resident at once and the launch lasts as long as one warp's walk along a full row.
constexpr int CT = 256;
template <typename V>
__device__ __forceinline__ double block_row_dot(const double* __restrict__ row, int j0, int j1, V v) {
    __shared__ double red[CT / 32];
    double s = 0.0;
    for (int j = j0 + int(threadIdx.x); j < j1; j += CT) s = fma(row[j], v(j), s);
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < CT / 32; ++k) t += red[k];
    return t;                                                   // valid in thread 0
}

// z = (Ainv r) * mask, one CTA per row, FP64 accumulation
template <typename TR, typename T>
__global__ void __launch_bounds__(CT) coarse_apply_kernel(int n, const double* __restrict__ Ainv,
                                                          const TR* __restrict__ r, const uint8_t* __restrict__ mask,
                                                          T* __restrict__ z) {
    vx::pdl_begin();
    using A = arith_t<T>;
    const int row = blockIdx.x;
    const double s = block_row_dot(Ainv + int64_t(row) * n, 0, n, [&](int j) { return double(Storage<TR>::load(r + j)); });
    if (threadIdx.x == 0) {
        const bool fr = mask ? ((mask[row / 3] >> (row % 3)) & 1u) : true;
        Storage<T>::store(z + row, fr ? A(s) : A(0));
    }
}

// Packed inverse factor: M = tril(Linv) + triu(Linv^T, 1), Linv = L^-1 of A = L L^T, so
// A^-1 r = Linv^T (Linv r) reads row i of M left of the diagonal (pass 1) and right of it (pass 2).
// 32x32 tiles through shared memory keep the transposed reads coalesced.
__global__ void coarse_pack_kernel(int n, const double* __restrict__ linv, double* __restrict__ m) {
    vx::pdl_begin();
    __shared__ double tile[32][33];
    const int bi = blockIdx.y * 32, bj = blockIdx.x * 32;      // output tile rows bi.., cols bj..
    const int tx = threadIdx.x, ty = threadIdx.y;              // 32 x 8 threads
    if (bj > bi) {                                             // strictly-upper tile: read Linv^T
        for (int k = ty; k < 32; k += 8) {
            const int r = bj + k, c = bi + tx;                 // source element Linv[r][c]
            tile[k][tx] = (r < n && c < n) ? linv[int64_t(r) * n + c] : 0.0;
        }
        __syncthreads();
        for (int k = ty; k < 32; k += 8) {
            const int i = bi + k, j = bj + tx;
            if (i < n && j < n) m[int64_t(i) * n + j] = tile[tx][k];
        }
    } else {                                                   // lower or diagonal tile
        for (int k = ty; k < 32; k += 8) {
            const int i = bi + k, j = bj + tx;
            if (i < n && j < n) {
                if (j <= i) m[int64_t(i) * n + j] = linv[int64_t(i) * n + j];
                else m[int64_t(i) * n + j] = linv[int64_t(j) * n + i];    // diagonal tile, upper part
            }
        }
    }
}

// pass 1: y = Linv r (row i, columns 0..i of M), one CTA per row, FP64 accumulation.
// Batches: system blockIdx.y has its factor at m + slot * n^2, its vectors at slot * vs, y at slot * n.
template <typename TR>
__global__ void __launch_bounds__(CT) coarse_lower_kernel(int n, const double* __restrict__ m,
                                                          const TR* __restrict__ r, double* __restrict__ y, int64_t vs) {
    vx::pdl_begin();
    const int row = blockIdx.x;
    m += int64_t(n) * n * blockIdx.y;
    r += vs * blockIdx.y;
    y += int64_t(n) * blockIdx.y;
    const double s = block_row_dot(m + int64_t(row) * n, 0, row + 1, [&](int j) { return double(Storage<TR>::load(r + j)); });
    if (threadIdx.x == 0) y[row] = s;
}

// pass 2: z = Linv^T y (row i: the diagonal Linv[i][i] and columns i+1.. of M), masked
template <typename T>
__global__ void __launch_bounds__(CT) coarse_upper_kernel(int n, const double* __restrict__ m,
                                                          const double* __restrict__ y,
                                                          const uint8_t* __restrict__ mask, T* __restrict__ z, int64_t vs) {
    vx::pdl_begin();
    using A = arith_t<T>;
    const int row = blockIdx.x;
    m += int64_t(n) * n * blockIdx.y;
    y += int64_t(n) * blockIdx.y;
    z += vs * blockIdx.y;
    if (mask) mask += (vs / 3) * blockIdx.y;
    const double s = block_row_dot(m + int64_t(row) * n, row, n, [&](int j) { return y[j]; });
    if (threadIdx.x == 0) {
        const bool fr = mask ? ((mask[row / 3] >> (row % 3)) & 1u) : true;
        Storage<T>::store(z + row, fr ? A(s) : A(0));
    }
}

__global__ void mask_from_dofs_kernel(int64_t nodes, const double* __restrict__ m, uint8_t* __restrict__ out) {
    vx::pdl_begin();
    const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    out[n] = uint8_t((m[3 * n] != 0.0) | ((m[3 * n + 1] != 0.0) << 1) | ((m[3 * n + 2] != 0.0) << 2));
}

inline unsigned blocks_for(int64_t n, int t) { return unsigned((n + t - 1) / t); }

int check_even(int nx, int ny, int nz, const char* what) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    if (nx + 1 > 65535 || (ny + 1 + TY_T - 1) / TY_T > 65535) {      // grid dimensions of the transfer launches
        set_error("%s: fine grid (%d, %d, %d) is too long in x or y for one launch", what, nx, ny, nz);
        return VX_ERR_INVALID_ARGUMENT;
    }
    if ((nx | ny | nz) & 1) {
        set_error("%s: fine grid (%d, %d, %d) must have even extents", what, nx, ny, nz);
        return VX_ERR_INVALID_ARGUMENT;
    }
    return VX_OK;
}

}  // namespace vx

using namespace vx;

extern "C" int vx_restrict(int prec, int nx, int ny, int nz, const void* fine, const uint8_t* coarse_mask,
                           void* coarse, cudaStream_t stream) {
    int st = check_even(nx, ny, nz, "vx_restrict");
    if (st) return st;
    VX_CHECK_ARG(fine && coarse, VX_ERR_NULL_POINTER, "vx_restrict: NULL pointer");
    Grid f{nx, ny, nz}, c{nx / 2, ny / 2, nz / 2};
    const bool ok = dispatch_prec(prec, [&](auto t) {             // auxiliary vectors on both sides
        using R = typename decltype(t)::R;
        vx::launch(restrict_kernel<R>, transfer_grid(c), dim3(TZ_T, TY_T), 0, stream, f, c, (const R*)fine, coarse_mask, (R*)coarse);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_restrict: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_restrict");
    return VX_OK;
}

extern "C" int vx_prolong_add(int prec, int nx, int ny, int nz, const void* coarse, const uint8_t* fine_mask,
                              void* x, cudaStream_t stream) {
    int st = check_even(nx, ny, nz, "vx_prolong_add");
    if (st) return st;
    VX_CHECK_ARG(coarse && x, VX_ERR_NULL_POINTER, "vx_prolong_add: NULL pointer");
    Grid f{nx, ny, nz}, c{nx / 2, ny / 2, nz / 2};
    const bool ok = dispatch_prec(prec, [&](auto t) {             // iterates on both sides
        using X = typename decltype(t)::X;
        vx::launch(prolong_add_kernel<X>, blocks_for(f.nodes(), 256), 256, 0, stream, f, c, (const X*)coarse, fine_mask, (X*)x);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_prolong_add: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_prolong_add");
    return VX_OK;
}

extern "C" int vx_coarsen_modulus(int prec, int nx, int ny, int nz, const void* E_fine, void* E_coarse,
                                  cudaStream_t stream) {
    int st = check_even(nx, ny, nz, "vx_coarsen_modulus");
    if (st) return st;
    VX_CHECK_ARG(E_fine && E_coarse, VX_ERR_NULL_POINTER, "vx_coarsen_modulus: NULL pointer");
    Grid f{nx, ny, nz}, c{nx / 2, ny / 2, nz / 2};
    const unsigned gb = blocks_for(c.elems(), 256);
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using M = typename decltype(t)::M;
        vx::launch(coarsen_modulus_kernel<M>, gb, 256, 0, stream, f, c, (const M*)E_fine, (M*)E_coarse);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_coarsen_modulus: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_coarsen_modulus");
    return VX_OK;
}

extern "C" int vx_coarsen_mask(int nx, int ny, int nz, const uint8_t* mask_fine, uint8_t* mask_coarse,
                               cudaStream_t stream) {
    int st = check_even(nx, ny, nz, "vx_coarsen_mask");
    if (st) return st;
    VX_CHECK_ARG(mask_fine && mask_coarse, VX_ERR_NULL_POINTER, "vx_coarsen_mask: NULL pointer");
    Grid f{nx, ny, nz}, c{nx / 2, ny / 2, nz / 2};
    vx::launch(coarsen_mask_kernel, blocks_for(c.nodes(), 256), 256, 0, stream, f, c, mask_fine, mask_coarse);
    VX_CHECK_LAUNCH("vx_coarsen_mask");
    return VX_OK;
}

extern "C" int vx_assemble_dense(int nx, int ny, int nz, const double* ke, const double* E,
                                 const uint8_t* node_mask, double* A, cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(ke && E && A, VX_ERR_NULL_POINTER, "vx_assemble_dense: NULL pointer");
    Grid g{nx, ny, nz};
    const int64_t n = 3 * g.nodes();
    VX_CHECK_ARG(n <= 65536, VX_ERR_INVALID_ARGUMENT, "vx_assemble_dense: %lld DOFs is too many for a dense matrix",
                 (long long)n);
    Ke576 k;
    for (int i = 0; i < 576; ++i) k.k[i] = ke[i];
    cudaError_t e = cudaMemsetAsync(A, 0, size_t(n) * size_t(n) * sizeof(double), stream);
    if (e != cudaSuccess) { set_error("vx_assemble_dense: memset: %s", cudaGetErrorString(e)); return VX_ERR_CUDA; }
    vx::launch(assemble_dense_kernel, blocks_for(g.nodes() * 243, 256), 256, 0, stream, g, k, E, node_mask, A);
    VX_CHECK_LAUNCH("vx_assemble_dense");
    return VX_OK;
}

extern "C" int vx_coarse_apply(int prec, int n, const double* Ainv, const void* r, const uint8_t* node_mask,
                               void* z, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_coarse_apply: n must be positive");
    VX_CHECK_ARG(Ainv && r && z, VX_ERR_NULL_POINTER, "vx_coarse_apply: NULL pointer");
    const bool ok = dispatch_prec(prec, [&](auto t) {             // r auxiliary, z an iterate
        using R = typename decltype(t)::R;
        using X = typename decltype(t)::X;
        vx::launch(coarse_apply_kernel<R, X>, unsigned(n), CT, 0, stream, n, Ainv, (const R*)r, node_mask, (X*)z);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_coarse_apply: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_coarse_apply");
    return VX_OK;
}

extern "C" int vx_mask_from_dofs(int64_t nodes, const double* dof_mask, uint8_t* node_mask, cudaStream_t stream) {
    VX_CHECK_ARG(nodes > 0, VX_ERR_INVALID_ARGUMENT, "vx_mask_from_dofs: nodes must be positive");
    VX_CHECK_ARG(dof_mask && node_mask, VX_ERR_NULL_POINTER, "vx_mask_from_dofs: NULL pointer");
    vx::launch(mask_from_dofs_kernel, blocks_for(nodes, 256), 256, 0, stream, nodes, dof_mask, node_mask);
    VX_CHECK_LAUNCH("vx_mask_from_dofs");
    return VX_OK;
}

extern "C" int vx_coarse_pack(int n, const double* linv, double* m, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_coarse_pack: n must be positive");
    VX_CHECK_ARG(linv && m, VX_ERR_NULL_POINTER, "vx_coarse_pack: NULL pointer");
    VX_CHECK_ARG(linv != m, VX_ERR_INVALID_ARGUMENT, "vx_coarse_pack: m may not alias linv");
    const unsigned t = unsigned((n + 31) / 32);
    vx::launch(coarse_pack_kernel, dim3(t, t), dim3(32, 8), 0, stream, n, linv, m);
    VX_CHECK_LAUNCH("vx_coarse_pack");
    return VX_OK;
}

extern "C" int vx_coarse_apply_factor(int prec, int n, const double* m, const void* r, const uint8_t* node_mask,
                                      double* y, void* z, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_coarse_apply_factor: n must be positive");
    VX_CHECK_ARG(m && r && y && z, VX_ERR_NULL_POINTER, "vx_coarse_apply_factor: NULL pointer");
    const bool ok = dispatch_prec(prec, [&](auto t) {             // r auxiliary, z an iterate
        using R = typename decltype(t)::R;
        using X = typename decltype(t)::X;
        vx::launch(coarse_lower_kernel<R>, unsigned(n), CT, 0, stream, n, m, (const R*)r, y, int64_t(0));
        vx::launch(coarse_upper_kernel<X>, unsigned(n), CT, 0, stream, n, m, y, node_mask, (X*)z, int64_t(0));
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_coarse_apply_factor: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_coarse_apply_factor");
    return VX_OK;
}

// The same for `slots` independent coarse systems: factors back to back (slot k at m + k n^2), the
// right-hand side, mask and solution of slot k at k * vs DOFs (vs a multiple of 3), y holding
// slots * n doubles.
extern "C" int vx_batch_coarse_apply_factor(int prec, int n, int slots, int64_t vs, const double* m, const void* r,
                                            const uint8_t* node_mask, double* y, void* z, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0 && slots >= 1 && slots <= 65535 && vs >= n && vs % 3 == 0, VX_ERR_INVALID_ARGUMENT,
                 "vx_batch_coarse_apply_factor: bad n/slots/stride");
    VX_CHECK_ARG(m && r && y && z, VX_ERR_NULL_POINTER, "vx_batch_coarse_apply_factor: NULL pointer");
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using R = typename decltype(t)::R;
        using X = typename decltype(t)::X;
        vx::launch(coarse_lower_kernel<R>, dim3(n, slots), CT, 0, stream, n, m, (const R*)r, y, vs);
        vx::launch(coarse_upper_kernel<X>, dim3(n, slots), CT, 0, stream, n, m, y, node_mask, (X*)z, vs);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_batch_coarse_apply_factor: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_batch_coarse_apply_factor");
    return VX_OK;
}
