// Deterministic reductions and vector kernels.  Every reduction uses a fixed grid (a function of
// n only) and a fixed summation order, so results are bitwise reproducible run to run and do
// not depend on what else is running on the device.
#include "vx_common.cuh"

namespace vx {

constexpr int RT = 256;             // threads per reducing CTA
constexpr int64_t RMAX = 1184;      // at most 8 CTAs per SM on 148 SMs

int64_t reduce_ctas(int64_t n) {
    int64_t g = (n + RT * 8 - 1) / (RT * 8);
    return g < 1 ? 1 : (g > RMAX ? RMAX : g);
}

template <typename S>
struct Vec3 { const S* p[3]; };

__device__ __forceinline__ double warp_sum(double v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[RT / 32];
    v = warp_sum(v);
    __syncthreads();                      // red[] may still be read by a previous call
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < RT / 32 ? red[threadIdx.x] : 0.0;
        s = warp_sum(s);
    }
    return s;   // valid in thread 0
}

// partials[k * G + blockIdx.x] = sum over this CTA's strided elements of a_k * b_k
template <typename S>
__global__ void __launch_bounds__(RT) dots_stage1(int64_t n, int count, Vec3<S> a, Vec3<S> b, double* partials) {
    vx::pdl_begin();
    const int64_t G = gridDim.x;
    for (int k = 0; k < count; ++k) {
        double s = 0.0;
        for (int64_t i = int64_t(blockIdx.x) * RT + threadIdx.x; i < n; i += G * RT)
            s = fma(double(Storage<S>::load(a.p[k] + i)), double(Storage<S>::load(b.p[k] + i)), s);
        s = block_sum(s);
        if (threadIdx.x == 0) partials[k * G + blockIdx.x] = s;
    }
}

// out[k] = sum_j partials[k * G + j] in a fixed order (one CTA)
__global__ void __launch_bounds__(RT) reduce_stage2(int64_t G, int count, const double* partials, double* out) {
    vx::pdl_begin();
    for (int k = 0; k < count; ++k) {
        double s = 0.0;
        for (int64_t j = threadIdx.x; j < G; j += RT) s += partials[k * G + j];
        s = block_sum(s);
        if (threadIdx.x == 0) out[k] = s;
    }
}

template <typename S>
__global__ void axpby_kernel(int64_t n, double alpha, const S* __restrict__ x, double beta, S* __restrict__ y) {
    vx::pdl_begin();
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    using C = decltype(Storage<S>::load(x));
    Storage<S>::store(y + i, C(alpha) * Storage<S>::load(x + i) + C(beta) * Storage<S>::load(y + i));
}

template <typename A, typename B>
__global__ void cast_kernel(int64_t n, const A* __restrict__ src, B* __restrict__ dst, double scale) {
    vx::pdl_begin();
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = double(Storage<A>::load(src + i));
    using C = decltype(Storage<B>::load(dst));
    Storage<B>::store(dst + i, scale == 1.0 ? C(v) : C(scale * v));
}

template <typename S>
__global__ void simp_kernel(int64_t n, const double* __restrict__ rho, double emin, double de, double penal, S* E) {
    vx::pdl_begin();
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double r = rho[i];
    const double v = emin + de * pow(r, penal);
    using C = decltype(Storage<S>::load(E));
    Storage<S>::store(E + i, C(v));
}

inline unsigned nblocks(int64_t n, int t) { return unsigned((n + t - 1) / t); }

template <typename A>
int cast_to(int64_t n, const A* src, int dst_prec, void* dst, double scale, cudaStream_t s) {
    const unsigned g = nblocks(n, 256);
    if (dst_prec == VX_F64) vx::launch(cast_kernel<A, double>, g, 256, 0, s, n, src, (double*)dst, scale);
    else if (dst_prec == VX_F32) vx::launch(cast_kernel<A, float>, g, 256, 0, s, n, src, (float*)dst, scale);
    else if (dst_prec == VX_BF16_F32) vx::launch(cast_kernel<A, __nv_bfloat16>, g, 256, 0, s, n, src, (__nv_bfloat16*)dst, scale);
    else { set_error("vx_cast: unknown destination precision %d", dst_prec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_cast");
    return VX_OK;
}

}  // namespace vx

using namespace vx;

extern "C" int64_t vx_partials_size(int64_t n) { return n > 0 ? reduce_ctas(n) : 1; }

extern "C" int vx_dots(int prec, int64_t n, int count, const void* const* a, const void* const* b,
                       double* partials, double* out, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0 && count >= 1 && count <= 3, VX_ERR_INVALID_ARGUMENT, "vx_dots: need n > 0 and 1 <= count <= 3");
    VX_CHECK_ARG(a && b && partials && out, VX_ERR_NULL_POINTER, "vx_dots: NULL pointer");
    const int64_t G = reduce_ctas(n);
    if (prec == VX_F64) {
        Vec3<double> va{}, vb{};
        for (int k = 0; k < count; ++k) { va.p[k] = (const double*)a[k]; vb.p[k] = (const double*)b[k]; }
        vx::launch(dots_stage1<double>, unsigned(G), RT, 0, stream, n, count, va, vb, partials);
    } else if (prec == VX_F32) {
        Vec3<float> va{}, vb{};
        for (int k = 0; k < count; ++k) { va.p[k] = (const float*)a[k]; vb.p[k] = (const float*)b[k]; }
        vx::launch(dots_stage1<float>, unsigned(G), RT, 0, stream, n, count, va, vb, partials);
    } else {
        set_error("vx_dots: unsupported precision %d", prec);
        return VX_ERR_INVALID_ARGUMENT;
    }
    VX_CHECK_LAUNCH("vx_dots(stage 1)");
    vx::launch(reduce_stage2, 1, RT, 0, stream, G, count, partials, out);
    VX_CHECK_LAUNCH("vx_dots(stage 2)");
    return VX_OK;
}

extern "C" int vx_reduce_partials(int64_t G, int count, const double* partials, double* out, cudaStream_t stream) {
    VX_CHECK_ARG(G > 0 && count >= 1, VX_ERR_INVALID_ARGUMENT, "vx_reduce_partials: bad sizes");
    VX_CHECK_ARG(partials && out, VX_ERR_NULL_POINTER, "vx_reduce_partials: NULL pointer");
    vx::launch(reduce_stage2, 1, RT, 0, stream, G, count, partials, out);
    VX_CHECK_LAUNCH("vx_reduce_partials");
    return VX_OK;
}

extern "C" int vx_axpby(int prec, int64_t n, double alpha, const void* x, double beta, void* y, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_axpby: n must be positive");
    VX_CHECK_ARG(x && y, VX_ERR_NULL_POINTER, "vx_axpby: NULL pointer");
    if (prec == VX_F64) vx::launch(axpby_kernel<double>, nblocks(n, 256), 256, 0, stream, n, alpha, (const double*)x, beta, (double*)y);
    else if (prec == VX_F32) vx::launch(axpby_kernel<float>, nblocks(n, 256), 256, 0, stream, n, alpha, (const float*)x, beta, (float*)y);
    else { set_error("vx_axpby: unsupported precision %d", prec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_axpby");
    return VX_OK;
}

extern "C" int vx_cast(int64_t n, int src_prec, const void* src, int dst_prec, void* dst, double scale,
                       cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_cast: n must be positive");
    VX_CHECK_ARG(src && dst, VX_ERR_NULL_POINTER, "vx_cast: NULL pointer");
    if (src_prec == VX_F64) return cast_to<double>(n, (const double*)src, dst_prec, dst, scale, stream);
    if (src_prec == VX_F32) return cast_to<float>(n, (const float*)src, dst_prec, dst, scale, stream);
    if (src_prec == VX_BF16_F32) return cast_to<__nv_bfloat16>(n, (const __nv_bfloat16*)src, dst_prec, dst, scale, stream);
    set_error("vx_cast: unknown source precision %d", src_prec);
    return VX_ERR_INVALID_ARGUMENT;
}

extern "C" int vx_simp_modulus(int prec, int64_t n, const double* rho, double emin, double emax, double penal,
                               void* E, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_simp_modulus: n must be positive");
    VX_CHECK_ARG(rho && E, VX_ERR_NULL_POINTER, "vx_simp_modulus: NULL pointer");
    const unsigned g = nblocks(n, 256);
    if (prec == VX_F64) vx::launch(simp_kernel<double>, g, 256, 0, stream, n, rho, emin, emax - emin, penal, (double*)E);
    else if (prec == VX_F32) vx::launch(simp_kernel<float>, g, 256, 0, stream, n, rho, emin, emax - emin, penal, (float*)E);
    else if (prec == VX_BF16_F32) vx::launch(simp_kernel<__nv_bfloat16>, g, 256, 0, stream, n, rho, emin, emax - emin, penal, (__nv_bfloat16*)E);
    else { set_error("vx_simp_modulus: unknown precision %d", prec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_simp_modulus");
    return VX_OK;
}
