// x-slab domain decomposition: the two kernels that make a slab-local operator the global one.
//
// A slab owns elements ex in [a, b) and holds node planes a..b; the planes a and b are shared with
// the neighbouring slabs.  On a shared plane the global product is the sum of the two slabs'
// element-layer contributions.  Each slab computes its contribution with layer_partial (the single
// element layer next to the plane), the slabs swap them, and plane_fix rewrites the plane from
// lo + hi, the lower slab's contribution first.  Both slabs therefore evaluate every shared value
// with the same operands in the same order, so the duplicated planes stay bitwise identical.
#include "vx_common.cuh"

namespace vx {

struct KeS { double k[576]; };

// out[3 p + c] = M K_layer(M u) at node p of plane `side` (0: the layer's lower node plane, 1: its
// upper one), in the arithmetic type.  u and node_mask cover the layer's two node planes, E its
// ny * nz elements (author order).  Node-owned dense gather: no atomics, deterministic.
template <typename X, typename M>
__global__ void __launch_bounds__(128) layer_partial_kernel(int ny, int nz, const __grid_constant__ KeS ke,
                                                            const M* __restrict__ E, const X* __restrict__ u,
                                                            const uint8_t* __restrict__ node_mask, int side,
                                                            arith_t<X>* __restrict__ out) {
    vx::pdl_begin();
    using A = arith_t<X>;
    __shared__ A K[576];
    for (int i = threadIdx.x; i < 576; i += blockDim.x) K[i] = A(ke.k[i]);
    __syncthreads();
    const int P = (ny + 1) * (nz + 1);
    const int p = int(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int iz = p % (nz + 1), iy = p / (nz + 1);
    constexpr int nat[8] = {0, 1, 3, 2, 4, 5, 7, 6};   // native node index of binary offset code
    A acc[3] = {A(0), A(0), A(0)};
    for (int oy = 0; oy < 2; ++oy) for (int oz = 0; oz < 2; ++oz) {
        const int ey = iy - oy, ez = iz - oz;            // element with this node at offset (side, oy, oz)
        if (ey < 0 || ey >= ny || ez < 0 || ez >= nz) continue;
        const A Ee = A(Storage<M>::load(E + (int64_t(ey) * nz + ez)));
        const int li = nat[side + 2 * oy + 4 * oz];
        for (int b = 0; b < 8; ++b) {
            const int m = nat[b];
            const int nb = ((b & 1) * (ny + 1) + ey + ((b >> 1) & 1)) * (nz + 1) + ez + ((b >> 2) & 1);
            const unsigned bits = node_mask ? unsigned(node_mask[nb]) : 7u;
            A uv[3];
            #pragma unroll
            for (int c = 0; c < 3; ++c) uv[c] = (bits >> c) & 1u ? A(Storage<X>::load(u + 3 * nb + c)) : A(0);
            #pragma unroll
            for (int c = 0; c < 3; ++c) {
                const A* kr = K + (3 * li + c) * 24 + 3 * m;
                acc[c] += Ee * (kr[0] * uv[0] + kr[1] * uv[1] + kr[2] * uv[2]);
            }
        }
    }
    const int tn = side * P + p;
    const unsigned bits = node_mask ? unsigned(node_mask[tn]) : 7u;
    #pragma unroll
    for (int c = 0; c < 3; ++c) out[3 * p + c] = (bits >> c) & 1u ? acc[c] : A(0);
}

enum PlaneMode { PLANE_APPLY = 0, PLANE_JACOBI = 1, PLANE_RESIDUAL = 2, PLANE_TRUE_RES = 3 };

constexpr int PT = 256;   // threads per plane-fix CTA

// One shared node plane (P nodes, 3 P DOFs) rewritten from s = lo + hi, with A x = s on free DOFs
// and x on fixed ones -- the epilogues of the fused operator kernels:
//   APPLY     out = A x                                   (TY = arithmetic type)
//   JACOBI    out = x + omega invd (r - A x)              (TY = iterate storage)
//   RESIDUAL  out = scale * (free ? r - A x : 0)          (TY = auxiliary storage)
//   TRUE_RES  out = r - A x                               (TY = iterate storage, FP64 outer loop)
// With `dot` (APPLY and TRUE_RES), dot[cta] = this CTA's sum of x.out (APPLY) or out^2 (TRUE_RES)
// over the rewritten plane when this slab owns it (`owned`), else 0: the slab's fused kernel left
// its shared planes out of its sums (vx_apply_dot_planes / vx_true_residual_planes), so every
// shared DOF is counted once over all slabs.  (Subtracting the slab-local terms instead would
// cancel: near convergence they are far larger than the true residual.)
template <typename X, typename R, typename TY, int MODE>
__global__ void __launch_bounds__(PT) plane_fix_kernel(int64_t n3, const arith_t<X>* __restrict__ lo,
                                                       const arith_t<X>* __restrict__ hi,
                                                       const uint8_t* __restrict__ node_mask, const X* __restrict__ x,
                                                       const R* __restrict__ r, const R* __restrict__ invd,
                                                       double omega, double scale, TY* __restrict__ out,
                                                       double* __restrict__ dot, int owned) {
    vx::pdl_begin();
    using A = arith_t<X>;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    double corr = 0.0;
    if (i < n3) {
        const unsigned bits = node_mask ? unsigned(node_mask[i / 3]) : 7u;
        const bool fr = (bits >> (i % 3)) & 1u;
        const A xr = A(Storage<X>::load(x + i));
        const A ax = fr ? A(lo[i] + hi[i]) : xr;
        A o;
        if constexpr (MODE == PLANE_APPLY) {
            o = ax;
        } else if constexpr (MODE == PLANE_JACOBI) {
            o = xr + A(omega) * A(Storage<R>::load(invd + i)) * (A(Storage<R>::load(r + i)) - ax);
        } else if constexpr (MODE == PLANE_RESIDUAL) {
            o = fr ? A(scale) * (A(Storage<R>::load(r + i)) - ax) : A(0);
        } else {
            o = A(Storage<R>::load(r + i)) - ax;
        }
        if constexpr (MODE == PLANE_APPLY || MODE == PLANE_TRUE_RES) {
            if (dot && owned) corr = (MODE == PLANE_APPLY ? double(xr) : double(o)) * double(o);
        }
        Storage<TY>::store(out + i, o);
    }
    if constexpr (MODE == PLANE_APPLY || MODE == PLANE_TRUE_RES) {
        if (dot) {                                          // uniform across the CTA
            __shared__ double red[PT / 32];
            #pragma unroll
            for (int o = 16; o > 0; o >>= 1) corr += __shfl_down_sync(0xffffffffu, corr, o);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = corr;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (int w = 0; w < PT / 32; ++w) t += red[w];
                dot[blockIdx.x] = t;
            }
        }
    }
}

// out = lo + hi in storage S (the restricted coarse right-hand side on a shared plane)
template <typename S>
__global__ void plane_sum_kernel(int64_t n, const S* __restrict__ lo, const S* __restrict__ hi, S* __restrict__ out) {
    vx::pdl_begin();
    using A = arith_t<S>;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Storage<S>::store(out + i, A(Storage<S>::load(lo + i)) + A(Storage<S>::load(hi + i)));
}

}  // namespace vx

using namespace vx;

extern "C" int vx_layer_partial(int prec, int ny, int nz, const double* ke, const void* E, const void* u,
                                const uint8_t* node_mask, int side, void* out, cudaStream_t stream) {
    int st = check_grid(1, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(ke && E && u && out, VX_ERR_NULL_POINTER, "vx_layer_partial: NULL pointer");
    VX_CHECK_ARG(side == 0 || side == 1, VX_ERR_INVALID_ARGUMENT, "vx_layer_partial: side must be 0 or 1");
    KeS k;
    for (int i = 0; i < 576; ++i) k.k[i] = ke[i];
    const int P = (ny + 1) * (nz + 1);
    const unsigned grid = unsigned((P + 127) / 128);
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using X = typename decltype(t)::X;
        using M = typename decltype(t)::M;
        vx::launch(layer_partial_kernel<X, M>, grid, 128, 0, stream, ny, nz, k, (const M*)E, (const X*)u,
                   node_mask, side, (arith_t<X>*)out);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_layer_partial: unknown precision %d", prec);
    VX_CHECK_LAUNCH("vx_layer_partial");
    return VX_OK;
}

extern "C" int64_t vx_plane_fix_partials(int64_t nodes) { return (3 * nodes + PT - 1) / PT; }

extern "C" int vx_plane_fix(int prec, int mode, int64_t nodes, const void* lo, const void* hi,
                            const uint8_t* node_mask, const void* x, const void* r, const void* invd, double omega,
                            double scale, void* out, double* dot, int owned, cudaStream_t stream) {
    VX_CHECK_ARG(nodes > 0 && nodes < (int64_t(1) << 29), VX_ERR_INVALID_ARGUMENT, "vx_plane_fix: bad plane size");
    VX_CHECK_ARG(mode >= PLANE_APPLY && mode <= PLANE_TRUE_RES, VX_ERR_INVALID_ARGUMENT, "vx_plane_fix: bad mode %d", mode);
    VX_CHECK_ARG(lo && hi && x && out, VX_ERR_NULL_POINTER, "vx_plane_fix: NULL pointer");
    VX_CHECK_ARG(mode == PLANE_APPLY || r, VX_ERR_NULL_POINTER, "vx_plane_fix: r is required");
    VX_CHECK_ARG(mode != PLANE_JACOBI || invd, VX_ERR_NULL_POINTER, "vx_plane_fix: invd is required");
    VX_CHECK_ARG(mode != PLANE_TRUE_RES || prec == VX_F64, VX_ERR_INVALID_ARGUMENT,
                 "vx_plane_fix: the true residual is FP64 only");
    VX_CHECK_ARG(!dot || mode == PLANE_APPLY || mode == PLANE_TRUE_RES, VX_ERR_INVALID_ARGUMENT,
                 "vx_plane_fix: dot corrections exist for modes 0 and 3 only");
    const int64_t n3 = 3 * nodes;
    const unsigned grid = unsigned((n3 + PT - 1) / PT);
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using X = typename decltype(t)::X;
        using R = typename decltype(t)::R;
        using A = arith_t<X>;
        const A* l = (const A*)lo;
        const A* h = (const A*)hi;
        switch (mode) {
            case PLANE_APPLY:
                vx::launch(plane_fix_kernel<X, R, A, PLANE_APPLY>, grid, PT, 0, stream, n3, l, h, node_mask,
                           (const X*)x, (const R*)r, (const R*)invd, omega, scale, (A*)out, dot, owned);
                break;
            case PLANE_JACOBI:
                vx::launch(plane_fix_kernel<X, R, X, PLANE_JACOBI>, grid, PT, 0, stream, n3, l, h, node_mask,
                           (const X*)x, (const R*)r, (const R*)invd, omega, scale, (X*)out, dot, owned);
                break;
            case PLANE_RESIDUAL:
                vx::launch(plane_fix_kernel<X, R, R, PLANE_RESIDUAL>, grid, PT, 0, stream, n3, l, h, node_mask,
                           (const X*)x, (const R*)r, (const R*)invd, omega, scale, (R*)out, dot, owned);
                break;
            default:
                vx::launch(plane_fix_kernel<X, R, X, PLANE_TRUE_RES>, grid, PT, 0, stream, n3, l, h, node_mask,
                           (const X*)x, (const R*)r, (const R*)invd, omega, scale, (X*)out, dot, owned);
        }
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_plane_fix: unknown precision %d", prec);
    VX_CHECK_LAUNCH("vx_plane_fix");
    return VX_OK;
}

extern "C" int vx_plane_sum(int prec, int64_t n, const void* lo, const void* hi, void* out, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0 && n < (int64_t(1) << 31), VX_ERR_INVALID_ARGUMENT, "vx_plane_sum: bad size");
    VX_CHECK_ARG(lo && hi && out, VX_ERR_NULL_POINTER, "vx_plane_sum: NULL pointer");
    const unsigned grid = unsigned((n + 255) / 256);
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using R = typename decltype(t)::R;
        vx::launch(plane_sum_kernel<R>, grid, 256, 0, stream, n, (const R*)lo, (const R*)hi, (R*)out);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_plane_sum: unknown precision %d", prec);
    VX_CHECK_LAUNCH("vx_plane_sum");
    return VX_OK;
}
