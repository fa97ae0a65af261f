// Solver kernels with device-resident scalars, and a CUDA-graph WHILE loop.
//
// The outer Krylov loops keep every scalar (r.z, p.q, alpha, beta, |b - A x|, the iteration and
// matvec counters, the converged flag) in a small FP64 array S on the device.  Each reduction is
// two-stage and deterministic: the producing kernel writes one partial per CTA, a one-CTA
// "finalize" kernel sums them in a fixed order and applies the scalar recurrence.  With the loop
// body captured as the body of a conditional WHILE graph node, a complete solve is a single graph
// launch with no host round trip per iteration; the condition kernel stops the loop on
// convergence, on breakdown or at maxiter.
#include "vx_common.cuh"

namespace vx {

constexpr int FT = 256;

enum Slot {
    S_RZ = 0, S_PQ = 1, S_ALPHA = 2, S_RR = 3, S_REL = 4, S_NB = 5, S_BETA = 6, S_RZN = 7, S_RZD = 8,
    S_TOL = 9, S_DONE = 10, S_IT = 11, S_MAXIT = 12, S_MV = 13, S_BREAK = 14, S_CHECK = 15, S_COUNT = 16
};

enum FinOp {
    FIN_PQ = 0,        // S[PQ] = sum; alpha = rz / pq (breakdown if pq == 0); it += 1; mv += 1
    FIN_TRUE = 1,      // S[RR] = sum; rel = sqrt(rr) / nb; mv += 1; done if rel <= tol
    FIN_BETA_PR = 2,   // rzn = sum0, rzd = sum1; beta = rzd / rz; rz = rzn      (flexible / Polak-Ribiere)
    FIN_BETA_FR = 3,   // rzn = sum0; beta = rzn / rz; rz = rzn                  (Fletcher-Reeves)
    FIN_NB = 4,        // nb = sqrt(sum)
    FIN_RZ = 5,        // rz = sum0
    FIN_RR_ONLY = 6    // rr = sum; rel = sqrt(rr) / nb (no counters, no flag)
};

__device__ __forceinline__ double warp_sum(double v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ double block_sum_ft(double v) {
    __shared__ double red[FT / 32];
    v = warp_sum(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) s = warp_sum(threadIdx.x < FT / 32 ? red[threadIdx.x] : 0.0);
    return s;
}

// Slot blockIdx.y (a batch of independent systems solved in lockstep) uses S + 16 slot and
// partials + slot * pstride; unbatched launches have one slot.
__global__ void __launch_bounds__(FT) finalize_kernel(int op, int64_t G, const double* __restrict__ partials,
                                                      double* __restrict__ S, int64_t pstride) {
    vx::pdl_begin();
    S += S_COUNT * int64_t(blockIdx.y);
    partials += pstride * int64_t(blockIdx.y);
    double s0 = 0.0, s1 = 0.0;
    for (int64_t j = threadIdx.x; j < G; j += FT) s0 += partials[j];
    s0 = block_sum_ft(s0);
    if (op == FIN_BETA_PR) {
        for (int64_t j = threadIdx.x; j < G; j += FT) s1 += partials[G + j];
        s1 = block_sum_ft(s1);
    }
    if (threadIdx.x != 0) return;
    switch (op) {
        case FIN_PQ:
            if (S[S_DONE] != 0.0) break;            // a converged warm start: the body is a no-op
            S[S_PQ] = s0;
            S[S_MV] += 1.0;
            if (s0 == 0.0 || !isfinite(s0)) { S[S_BREAK] = 1.0; S[S_ALPHA] = 0.0; }   // no step is taken
            else { S[S_ALPHA] = S[S_RZ] / s0; S[S_IT] += 1.0; }
            break;
        case FIN_TRUE:
            if (S[S_DONE] != 0.0) break;
            S[S_RR] = s0;
            S[S_REL] = sqrt(s0) / S[S_NB];
            S[S_MV] += 1.0;
            if (S[S_REL] <= S[S_TOL]) S[S_DONE] = 1.0;
            if (!isfinite(S[S_REL])) S[S_BREAK] = 1.0;
            break;
        case FIN_BETA_PR:
            S[S_RZN] = s0;
            S[S_RZD] = s1;
            S[S_BETA] = s1 / S[S_RZ];
            S[S_RZ] = s0;
            break;
        case FIN_BETA_FR:
            S[S_RZN] = s0;
            S[S_BETA] = s0 / S[S_RZ];
            S[S_RZ] = s0;
            break;
        case FIN_NB: S[S_NB] = sqrt(s0); break;
        case FIN_RZ: S[S_RZ] = s0; break;
        case FIN_RR_ONLY:
            S[S_RR] = s0;
            S[S_REL] = sqrt(s0) / S[S_NB];
            break;
    }
}

// x += alpha p; r -= alpha q (r update skipped when it is about to be replaced by b - A x).
// Nothing moves once the loop has converged or broken down.
// Vector kernels of a batch: slot blockIdx.y works on its n entries at slot * vs and on S + 16 slot.
template <typename T>
__global__ void cg_update_kernel(int64_t n, const double* __restrict__ S, T* __restrict__ x, const T* __restrict__ p,
                                 T* __restrict__ r, const T* __restrict__ q, int update_r, int64_t vs) {
    vx::pdl_begin();
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t o = vs * int64_t(blockIdx.y);
    S += S_COUNT * int64_t(blockIdx.y);
    x += o;
    p += o;
    if (update_r) { r += o; q += o; }
    if (S[S_DONE] != 0.0 || S[S_BREAK] != 0.0) return;
    const T a = T(S[S_ALPHA]);
    x[i] = x[i] + a * p[i];
    if (update_r) r[i] = r[i] - a * q[i];
}

// p = z + beta p and, when z_old is given, z_old = z; z and z_old in the preconditioner's storage TZ
// (a copy in z's own type is exact and moves half the bytes of an FP64 copy of an FP32 z)
template <typename T, typename TZ>
__global__ void cg_direction_kernel(int64_t n, const double* __restrict__ S, const TZ* __restrict__ z, T* __restrict__ p,
                                    TZ* __restrict__ z_old, int64_t vs) {
    vx::pdl_begin();
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t o = vs * int64_t(blockIdx.y);
    S += S_COUNT * int64_t(blockIdx.y);
    z += o;
    p += o;
    if (z_old) z_old += o;
    const TZ zr = z[i];
    p[i] = T(Storage<TZ>::cvt(zr)) + T(S[S_BETA]) * p[i];
    if (z_old) z_old[i] = zr;
}

// The same direction update preceded by the deferred x += alpha p of this iteration (p still the old
// direction), skipped once the loop has converged or broken down: one read of p serves both.
template <typename T, typename TZ>
__global__ void cg_direction_update_kernel(int64_t n, const double* __restrict__ S, const TZ* __restrict__ z,
                                           T* __restrict__ p, TZ* __restrict__ z_old, T* __restrict__ x) {
    vx::pdl_begin();
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T pi = p[i];
    if (S[S_DONE] == 0.0 && S[S_BREAK] == 0.0) x[i] = x[i] + T(S[S_ALPHA]) * pi;
    const TZ zr = z[i];
    p[i] = T(Storage<TZ>::cvt(zr)) + T(S[S_BETA]) * pi;
    if (z_old) z_old[i] = zr;
}

// partials for r . zn and r . (zn - zo), fixed grid G (a function of n), fixed order
// (slot blockIdx.y: vectors at slot * vs, partials at slot * 2G)
template <typename T, typename TZ>
__global__ void __launch_bounds__(FT) dots_pr_kernel(int64_t n, const T* __restrict__ r, const TZ* __restrict__ zn,
                                                     const TZ* __restrict__ zo, double* __restrict__ partials, int64_t vs) {
    vx::pdl_begin();
    const int64_t G = gridDim.x;
    {
        const int64_t o = vs * int64_t(blockIdx.y);
        r += o;
        zn += o;
        if (zo) zo += o;
        partials += 2 * G * int64_t(blockIdx.y);
    }
    double a = 0.0, b = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * FT + threadIdx.x; i < n; i += G * FT) {
        const double ri = double(r[i]), zi = double(Storage<TZ>::load(zn + i));
        a = fma(ri, zi, a);
        if (zo) b = fma(ri, zi - double(Storage<TZ>::load(zo + i)), b);
    }
    a = block_sum_ft(a);
    if (threadIdx.x == 0) partials[blockIdx.x] = a;
    if (zo) {
        b = block_sum_ft(b);
        if (threadIdx.x == 0) partials[G + blockIdx.x] = b;
    }
}

// z = d * r (Jacobi) with partial r . z
template <typename T>
__global__ void __launch_bounds__(FT) jacobi_precond_dot_kernel(int64_t n, const T* __restrict__ d, const T* __restrict__ r,
                                                                T* __restrict__ z, double* __restrict__ partials) {
    vx::pdl_begin();
    const int64_t G = gridDim.x;
    double a = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * FT + threadIdx.x; i < n; i += G * FT) {
        const T zi = d[i] * r[i];
        z[i] = zi;
        a = fma(double(r[i]), double(zi), a);
    }
    a = block_sum_ft(a);
    if (threadIdx.x == 0) partials[blockIdx.x] = a;
}

// V-cycle entry: r_mg = (TM) r64 (skipped when r_mg is NULL), x = omega * invd * r_mg
// V-cycle entry: r_mg = r64 in auxiliary storage, x = omega * invd * r_mg (the first pre-sweep from x = 0)
template <typename TX, typename TR>
__global__ void vcycle_entry_kernel(int64_t n, const double* __restrict__ r64, TR* __restrict__ rmg,
                                    const TR* __restrict__ invd, double omega, TX* __restrict__ x) {
    vx::pdl_begin();
    using A = arith_t<TX>;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const A r = A(Storage<TR>::round(arith_t<TR>(r64[i])));   // the level residual as stored
    if (rmg) Storage<TR>::store(rmg + i, r);
    Storage<TX>::store(x + i, A(omega) * A(Storage<TR>::load(invd + i)) * r);
}

// The same entry preceded by the CG residual update r64 -= alpha q (alpha = S[S_ALPHA]), which is
// skipped, like vx_cg_update's, once the loop has converged or broken down.
template <typename TX, typename TR>
__global__ void vcycle_entry_update_kernel(int64_t n, const double* __restrict__ S, double* __restrict__ r64,
                                           const double* __restrict__ q, TR* __restrict__ rmg,
                                           const TR* __restrict__ invd, double omega, TX* __restrict__ x) {
    vx::pdl_begin();
    using A = arith_t<TX>;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double rv = r64[i];
    if (S[S_DONE] == 0.0 && S[S_BREAK] == 0.0) {
        rv = rv - S[S_ALPHA] * q[i];
        r64[i] = rv;
    }
    const A r = A(Storage<TR>::round(arith_t<TR>(rv)));
    if (rmg) Storage<TR>::store(rmg + i, r);
    Storage<TX>::store(x + i, A(omega) * A(Storage<TR>::load(invd + i)) * r);
}

// out = omega * a * b: a, b auxiliary, out an iterate
template <typename TX, typename TR>
__global__ void scaled_product_kernel(int64_t n, double omega, const TR* __restrict__ a, const TR* __restrict__ b,
                                      TX* __restrict__ out) {
    vx::pdl_begin();
    using A = arith_t<TX>;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Storage<TX>::store(out + i, A(omega) * A(Storage<TR>::load(a + i)) * A(Storage<TR>::load(b + i)));
}

__global__ void set_scalars_kernel(double* S, int first, int count, double value) {
    vx::pdl_begin();
    const int i = threadIdx.x;
    if (i < count) S[first + i] = value;
}

// Another loop body runs while any of the `slots` systems is still running.
__global__ void condition_kernel(cudaGraphConditionalHandle h, const double* __restrict__ S, int slots) {
    vx::pdl_begin();
    if (threadIdx.x == 0) {
        bool go = false;
        for (int k = 0; k < slots; ++k) {
            const double* s = S + S_COUNT * k;
            // S[S_CHECK] = iterations per loop body: the next body must not pass maxiter
            go = go || (s[S_DONE] == 0.0 && s[S_BREAK] == 0.0 && s[S_IT] + s[S_CHECK] <= s[S_MAXIT]);
        }
        cudaGraphSetConditional(h, go ? 1u : 0u);
    }
}

int64_t fixed_ctas(int64_t n) {
    int64_t g = (n + FT * 8 - 1) / (FT * 8);
    return g < 1 ? 1 : (g > 1184 ? 1184 : g);
}

inline unsigned nb(int64_t n, int t) { return unsigned((n + t - 1) / t); }

struct WhileGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle handle = 0;
    cudaGraph_t body = nullptr;
};

}  // namespace vx

using namespace vx;

extern "C" int vx_solver_slots(void) { return S_COUNT; }

extern "C" int64_t vx_solver_partials(int64_t n) { return fixed_ctas(n); }

extern "C" int vx_solver_finalize(int op, int64_t G, const double* partials, double* S, cudaStream_t stream) {
    VX_CHECK_ARG(op >= 0 && op <= FIN_RR_ONLY && G > 0, VX_ERR_INVALID_ARGUMENT, "vx_solver_finalize: bad op/G");
    VX_CHECK_ARG(partials && S, VX_ERR_NULL_POINTER, "vx_solver_finalize: NULL pointer");
    vx::launch(finalize_kernel, 1, FT, 0, stream, op, G, partials, S, int64_t(0));
    VX_CHECK_LAUNCH("vx_solver_finalize");
    return VX_OK;
}

extern "C" int vx_cg_update(int prec, int64_t n, const double* S, void* x, const void* p, void* r, const void* q,
                            int update_r, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_cg_update: n must be positive");
    VX_CHECK_ARG(S && x && p && (!update_r || (r && q)), VX_ERR_NULL_POINTER, "vx_cg_update: NULL pointer");
    if (prec == VX_F64)
        vx::launch(cg_update_kernel<double>, nb(n, 256), 256, 0, stream, n, S, (double*)x, (const double*)p, (double*)r,
                                                                 (const double*)q, update_r, int64_t(0));
    else if (prec == VX_F32)
        vx::launch(cg_update_kernel<float>, nb(n, 256), 256, 0, stream, n, S, (float*)x, (const float*)p, (float*)r,
                                                                (const float*)q, update_r, int64_t(0));
    else { set_error("vx_cg_update: unsupported precision %d", prec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_cg_update");
    return VX_OK;
}

extern "C" int vx_cg_direction(int prec, int zprec, int64_t n, const double* S, const void* z, void* p, void* z_old,
                               cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_cg_direction: n must be positive");
    VX_CHECK_ARG(S && z && p, VX_ERR_NULL_POINTER, "vx_cg_direction: NULL pointer");
    if (prec == VX_F64 && zprec == VX_F64)
        vx::launch(cg_direction_kernel<double, double>, nb(n, 256), 256, 0, stream, n, S, (const double*)z, (double*)p, (double*)z_old, int64_t(0));
    else if (prec == VX_F64 && zprec == VX_F32)
        vx::launch(cg_direction_kernel<double, float>, nb(n, 256), 256, 0, stream, n, S, (const float*)z, (double*)p, (float*)z_old, int64_t(0));
    else if (prec == VX_F64 && zprec == VX_BF16_F32)
        vx::launch(cg_direction_kernel<double, __nv_bfloat16>, nb(n, 256), 256, 0, stream, n, S, (const __nv_bfloat16*)z, (double*)p,
                                                                                   (__nv_bfloat16*)z_old, int64_t(0));
    else if (prec == VX_F32 && zprec == VX_F32)
        vx::launch(cg_direction_kernel<float, float>, nb(n, 256), 256, 0, stream, n, S, (const float*)z, (float*)p, (float*)z_old, int64_t(0));
    else { set_error("vx_cg_direction: unsupported precisions %d/%d", prec, zprec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_cg_direction");
    return VX_OK;
}

extern "C" int vx_cg_direction_update(int zprec, int64_t n, const double* S, const void* z, double* p, void* z_old,
                                      double* x, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_cg_direction_update: n must be positive");
    VX_CHECK_ARG(S && z && p && x, VX_ERR_NULL_POINTER, "vx_cg_direction_update: NULL pointer");
    const bool ok = dispatch_prec(zprec, [&](auto t) {
        using X = typename decltype(t)::X;
        vx::launch(cg_direction_update_kernel<double, X>, nb(n, 256), 256, 0, stream, n, S, (const X*)z, p, (X*)z_old, x);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_cg_direction_update: unsupported precision %d", zprec);
    VX_CHECK_LAUNCH("vx_cg_direction_update");
    return VX_OK;
}

extern "C" int vx_dots_pr(int prec, int zprec, int64_t n, const void* r, const void* zn, const void* zo,
                          double* partials, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_dots_pr: n must be positive");
    VX_CHECK_ARG(r && zn && partials, VX_ERR_NULL_POINTER, "vx_dots_pr: NULL pointer");
    const unsigned G = unsigned(fixed_ctas(n));
    if (prec == VX_F64 && zprec == VX_F64)
        vx::launch(dots_pr_kernel<double, double>, G, FT, 0, stream, n, (const double*)r, (const double*)zn, (const double*)zo, partials, int64_t(0));
    else if (prec == VX_F64 && zprec == VX_F32)
        vx::launch(dots_pr_kernel<double, float>, G, FT, 0, stream, n, (const double*)r, (const float*)zn, (const float*)zo, partials, int64_t(0));
    else if (prec == VX_F64 && zprec == VX_BF16_F32)
        vx::launch(dots_pr_kernel<double, __nv_bfloat16>, G, FT, 0, stream, n, (const double*)r, (const __nv_bfloat16*)zn,
                                                                    (const __nv_bfloat16*)zo, partials, int64_t(0));
    else if (prec == VX_F32 && zprec == VX_F32)
        vx::launch(dots_pr_kernel<float, float>, G, FT, 0, stream, n, (const float*)r, (const float*)zn, (const float*)zo, partials, int64_t(0));
    else { set_error("vx_dots_pr: unsupported precisions %d/%d", prec, zprec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_dots_pr");
    return VX_OK;
}

extern "C" int vx_jacobi_precond_dot(int prec, int64_t n, const void* d, const void* r, void* z, double* partials,
                                     cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_jacobi_precond_dot: n must be positive");
    VX_CHECK_ARG(d && r && z && partials, VX_ERR_NULL_POINTER, "vx_jacobi_precond_dot: NULL pointer");
    const unsigned G = unsigned(fixed_ctas(n));
    if (prec == VX_F64)
        vx::launch(jacobi_precond_dot_kernel<double>, G, FT, 0, stream, n, (const double*)d, (const double*)r, (double*)z, partials);
    else if (prec == VX_F32)
        vx::launch(jacobi_precond_dot_kernel<float>, G, FT, 0, stream, n, (const float*)d, (const float*)r, (float*)z, partials);
    else { set_error("vx_jacobi_precond_dot: unsupported precision %d", prec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_jacobi_precond_dot");
    return VX_OK;
}

extern "C" int vx_vcycle_entry(int prec, int64_t n, const double* r64, void* r_mg, const void* inv_diag, double omega,
                               void* x, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_vcycle_entry: n must be positive");
    VX_CHECK_ARG(r64 && inv_diag && x, VX_ERR_NULL_POINTER, "vx_vcycle_entry: NULL pointer");
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using X = typename decltype(t)::X;
        using R = typename decltype(t)::R;
        vx::launch(vcycle_entry_kernel<X, R>, nb(n, 256), 256, 0, stream, n, r64, (R*)r_mg, (const R*)inv_diag, omega, (X*)x);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_vcycle_entry: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_vcycle_entry");
    return VX_OK;
}

extern "C" int vx_vcycle_entry_update(int prec, int64_t n, const double* S, double* r64, const double* q, void* r_mg,
                                      const void* inv_diag, double omega, void* x, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_vcycle_entry_update: n must be positive");
    VX_CHECK_ARG(S && r64 && q && inv_diag && x, VX_ERR_NULL_POINTER, "vx_vcycle_entry_update: NULL pointer");
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using X = typename decltype(t)::X;
        using R = typename decltype(t)::R;
        vx::launch(vcycle_entry_update_kernel<X, R>, nb(n, 256), 256, 0, stream, n, S, r64, q, (R*)r_mg, (const R*)inv_diag,
                                                                         omega, (X*)x);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_vcycle_entry_update: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_vcycle_entry_update");
    return VX_OK;
}

extern "C" int vx_scaled_product(int prec, int64_t n, double omega, const void* a, const void* b, void* out,
                                 cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_scaled_product: n must be positive");
    VX_CHECK_ARG(a && b && out, VX_ERR_NULL_POINTER, "vx_scaled_product: NULL pointer");
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using X = typename decltype(t)::X;
        using R = typename decltype(t)::R;
        vx::launch(scaled_product_kernel<X, R>, nb(n, 256), 256, 0, stream, n, omega, (const R*)a, (const R*)b, (X*)out);
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_scaled_product: unsupported precision %d", prec);
    VX_CHECK_LAUNCH("vx_scaled_product");
    return VX_OK;
}

extern "C" int vx_set_scalars(double* S, int first, int count, double value, cudaStream_t stream) {
    VX_CHECK_ARG(S, VX_ERR_NULL_POINTER, "vx_set_scalars: NULL S");
    VX_CHECK_ARG(first >= 0 && count >= 1 && first + count <= S_COUNT, VX_ERR_INVALID_ARGUMENT,
                 "vx_set_scalars: slots out of range");
    vx::launch(set_scalars_kernel, 1, 32, 0, stream, S, first, count, value);
    VX_CHECK_LAUNCH("vx_set_scalars");
    return VX_OK;
}

// ----------------------------------------------------------------------------- WHILE graphs
extern "C" int vx_graph_while_begin(cudaStream_t stream, void** handle) {
    VX_CHECK_ARG(handle, VX_ERR_NULL_POINTER, "vx_graph_while_begin: NULL handle");
    VX_CHECK_ARG(stream != nullptr, VX_ERR_INVALID_ARGUMENT, "vx_graph_while_begin: capture needs a non-default stream");
    // load the condition kernel now: with lazy module loading its first launch would otherwise
    // happen inside the capture
    cudaFuncAttributes attr;
    cudaError_t e = cudaFuncGetAttributes(&attr, condition_kernel);
    if (e != cudaSuccess) {
        set_error("vx_graph_while_begin: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    auto* w = new WhileGraph();
    e = cudaGraphCreate(&w->graph, 0);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&w->handle, w->graph, 1, cudaGraphCondAssignDefault);
    cudaGraphNode_t node;
    cudaGraphNodeParams p = {};
    if (e == cudaSuccess) {
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = w->handle;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        e = cudaGraphAddNode(&node, w->graph, nullptr, 0, &p);
    }
    if (e == cudaSuccess) {
        w->body = p.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(stream, w->body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    }
    if (e != cudaSuccess) {
        if (w->graph) cudaGraphDestroy(w->graph);
        delete w;
        set_error("vx_graph_while_begin: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    *handle = w;
    return VX_OK;
}

static int graph_while_end(void* handle, const double* S, int slots, cudaStream_t stream) {
    VX_CHECK_ARG(handle && S, VX_ERR_NULL_POINTER, "vx_graph_while_end: NULL pointer");
    VX_CHECK_ARG(slots >= 1, VX_ERR_INVALID_ARGUMENT, "vx_graph_while_end: slots must be positive");
    auto* w = static_cast<WhileGraph*>(handle);
    vx::launch(condition_kernel, 1, 32, 0, stream, w->handle, S, slots);
    cudaError_t e = cudaGetLastError();
    cudaGraph_t captured = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(stream, &captured);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&w->exec, w->graph, 0);
    if (e != cudaSuccess) {
        set_error("vx_graph_while_end: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    return VX_OK;
}

extern "C" int vx_graph_while_end(void* handle, const double* S, cudaStream_t stream) {
    return graph_while_end(handle, S, 1, stream);
}

// The batch form: the loop runs while any of `slots` systems (scalars S + 16 k) is running.
extern "C" int vx_batch_graph_while_end(void* handle, const double* S, int slots, cudaStream_t stream) {
    return graph_while_end(handle, S, slots, stream);
}

// ----------------------------------------------------------------------------- batches
// `slots` independent systems of n unknowns, slot k's vectors at k * stride, scalars at S + 16 k:
// the kernels above with the slot in blockIdx.y (one launch for the whole batch).
extern "C" int vx_batch_finalize(int op, int64_t G, int slots, const double* partials, int64_t pstride, double* S,
                                 cudaStream_t stream) {
    VX_CHECK_ARG(op >= 0 && op <= FIN_RR_ONLY && G > 0 && slots >= 1 && slots <= 65535, VX_ERR_INVALID_ARGUMENT,
                 "vx_batch_finalize: bad op/G/slots");
    VX_CHECK_ARG(partials && S, VX_ERR_NULL_POINTER, "vx_batch_finalize: NULL pointer");
    vx::launch(finalize_kernel, dim3(1, slots), FT, 0, stream, op, G, partials, S, pstride);
    VX_CHECK_LAUNCH("vx_batch_finalize");
    return VX_OK;
}

extern "C" int vx_batch_cg_update(int prec, int64_t n, int slots, int64_t stride, const double* S, void* x,
                                  const void* p, void* r, const void* q, int update_r, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0 && slots >= 1 && slots <= 65535, VX_ERR_INVALID_ARGUMENT, "vx_batch_cg_update: bad n/slots");
    VX_CHECK_ARG(S && x && p && (!update_r || (r && q)), VX_ERR_NULL_POINTER, "vx_batch_cg_update: NULL pointer");
    VX_CHECK_ARG(prec == VX_F64, VX_ERR_INVALID_ARGUMENT, "vx_batch_cg_update: unsupported precision %d", prec);
    vx::launch(cg_update_kernel<double>, dim3(nb(n, 256), slots), 256, 0, stream, n, S, (double*)x, (const double*)p,
               (double*)r, (const double*)q, update_r, stride);
    VX_CHECK_LAUNCH("vx_batch_cg_update");
    return VX_OK;
}

extern "C" int vx_batch_cg_direction(int zprec, int64_t n, int slots, int64_t stride, const double* S, const void* z,
                                     double* p, void* z_old, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0 && slots >= 1 && slots <= 65535, VX_ERR_INVALID_ARGUMENT, "vx_batch_cg_direction: bad n/slots");
    VX_CHECK_ARG(S && z && p, VX_ERR_NULL_POINTER, "vx_batch_cg_direction: NULL pointer");
    if (zprec == VX_F64)
        vx::launch(cg_direction_kernel<double, double>, dim3(nb(n, 256), slots), 256, 0, stream, n, S, (const double*)z, p,
                   (double*)z_old, stride);
    else if (zprec == VX_F32)
        vx::launch(cg_direction_kernel<double, float>, dim3(nb(n, 256), slots), 256, 0, stream, n, S, (const float*)z, p,
                   (float*)z_old, stride);
    else { set_error("vx_batch_cg_direction: unsupported precision %d", zprec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_batch_cg_direction");
    return VX_OK;
}

// per-slot partials of r . zn (and r . (zn - zo)) at slot * 2 vx_solver_partials(n)
extern "C" int vx_batch_dots_pr(int zprec, int64_t n, int slots, int64_t stride, const double* r, const void* zn,
                                const void* zo, double* partials, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0 && slots >= 1 && slots <= 65535, VX_ERR_INVALID_ARGUMENT, "vx_batch_dots_pr: bad n/slots");
    VX_CHECK_ARG(r && zn && partials, VX_ERR_NULL_POINTER, "vx_batch_dots_pr: NULL pointer");
    const unsigned G = unsigned(fixed_ctas(n));
    if (zprec == VX_F64)
        vx::launch(dots_pr_kernel<double, double>, dim3(G, slots), FT, 0, stream, n, r, (const double*)zn,
                   (const double*)zo, partials, stride);
    else if (zprec == VX_F32)
        vx::launch(dots_pr_kernel<double, float>, dim3(G, slots), FT, 0, stream, n, r, (const float*)zn,
                   (const float*)zo, partials, stride);
    else { set_error("vx_batch_dots_pr: unsupported precision %d", zprec); return VX_ERR_INVALID_ARGUMENT; }
    VX_CHECK_LAUNCH("vx_batch_dots_pr");
    return VX_OK;
}

// 0: not capturing, 1: capture active, 2: capture invalidated, -1: query failed
extern "C" int vx_capture_status(cudaStream_t stream) {
    cudaStreamCaptureStatus st;
    if (cudaStreamIsCapturing(stream, &st) != cudaSuccess) return -1;
    return st == cudaStreamCaptureStatusNone ? 0 : (st == cudaStreamCaptureStatusActive ? 1 : 2);
}

extern "C" int vx_graph_launch(void* handle, cudaStream_t stream) {
    VX_CHECK_ARG(handle, VX_ERR_NULL_POINTER, "vx_graph_launch: NULL handle");
    auto* w = static_cast<WhileGraph*>(handle);
    VX_CHECK_ARG(w->exec, VX_ERR_INVALID_ARGUMENT, "vx_graph_launch: graph was not instantiated");
    cudaError_t e = cudaGraphLaunch(w->exec, stream);
    if (e != cudaSuccess) {
        set_error("vx_graph_launch: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    return VX_OK;
}

// Number of nodes in the captured loop body (introspection for tests).
extern "C" int64_t vx_graph_body_nodes(void* handle) {
    if (!handle) return -1;
    auto* w = static_cast<WhileGraph*>(handle);
    size_t n = 0;
    if (cudaGraphGetNodes(w->body, nullptr, &n) != cudaSuccess) return -1;
    return int64_t(n);
}

extern "C" int vx_graph_destroy(void* handle) {
    if (!handle) return VX_OK;
    auto* w = static_cast<WhileGraph*>(handle);
    if (w->exec) cudaGraphExecDestroy(w->exec);
    if (w->graph) cudaGraphDestroy(w->graph);
    delete w;
    return VX_OK;
}
