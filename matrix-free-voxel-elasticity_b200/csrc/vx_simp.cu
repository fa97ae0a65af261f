// SIMP kernels: the matrix-free hat ("cone") density filter and the optimality-criteria (top88)
// update with its bisection on the Lagrange multiplier resident on the device.
#include "vx_common.cuh"

#include <cmath>

namespace vx {

constexpr int FILTER_MAX_R = 3;                                   // rmin < 4 elements
constexpr int FILTER_MAX_TAPS = (2 * FILTER_MAX_R + 1) * (2 * FILTER_MAX_R + 1) * (2 * FILTER_MAX_R + 1);

struct FilterTaps {
    int n;
    signed char d[FILTER_MAX_TAPS][3];
    double w[FILTER_MAX_TAPS];
};

// mode 0: y = H x; 1: y = (H x) / s; 2: y = H (x / s).  Taps in (dx, dy, dz) lexicographic order, the
// order of the reference's stencil loops (donor filter_r2.py:55-72).
__global__ void cone_filter_kernel(Grid g, const __grid_constant__ FilterTaps t, const double* __restrict__ x,
                                   const double* __restrict__ s, int mode, double* __restrict__ y) {
    vx::pdl_begin();
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= g.elems()) return;
    const int ez = int(e % g.nz), ey = int((e / g.nz) % g.ny), ex = int(e / (int64_t(g.nz) * g.ny));
    double acc = 0.0;
    for (int i = 0; i < t.n; ++i) {
        const int jx = ex + t.d[i][0], jy = ey + t.d[i][1], jz = ez + t.d[i][2];
        if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz) continue;
        const int64_t j = g.elem(jx, jy, jz);
        const double v = mode == 2 ? x[j] / s[j] : x[j];
        acc += t.w[i] * v;
    }
    y[e] = mode == 1 ? acc / s[e] : acc;
}

// OC state slots (a 16-double array shared with the WHILE-graph condition kernel, whose slots
// 10 done, 11 iterations, 12 max iterations, 14 breakdown, 15 iterations per body it reads)
enum OcSlot { OC_L1 = 0, OC_L2 = 1, OC_LMID = 2, OC_VOL = 3, OC_VOLFRAC = 4, OC_TOL = 5, OC_NEL = 6,
              OC_DONE = 10, OC_IT = 11 };

__device__ __forceinline__ double oc_design(double x, double dc, double dv, double lmid, double move) {
    const double step = sqrt(fmax(-dc / dv / lmid, 0.0));
    return fmin(fmax(x * step, fmax(x - move, 0.0)), fmin(x + move, 1.0));
}

// one bisection probe: lmid = (l1 + l2) / 2, partials of sum_i w_i x_new_i (fixed grid and order)
__global__ void __launch_bounds__(256) oc_probe_kernel(int64_t n, const double* __restrict__ x,
                                                       const double* __restrict__ dc, const double* __restrict__ dv,
                                                       const double* __restrict__ w, double move,
                                                       const double* __restrict__ S, double* __restrict__ partials) {
    vx::pdl_begin();
    __shared__ double red[8];
    const double lmid = 0.5 * (S[OC_L2] + S[OC_L1]);
    double acc = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * 256 + threadIdx.x; i < n; i += int64_t(gridDim.x) * 256)
        acc = fma(w[i], oc_design(x[i], dc[i], dv[i], lmid, move), acc);
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < 8; ++k) s += red[k];
        partials[blockIdx.x] = s;
    }
}

// volume = sum / n; l1 or l2 := lmid; done when (l2 - l1) / (l1 + l2) <= tol (the top88 test,
// experiments/session_h/run_w1b.py:53-62)
__global__ void oc_finalize_kernel(int64_t G, const double* __restrict__ partials, double* __restrict__ S) {
    vx::pdl_begin();
    __shared__ double red[8];
    double acc = 0.0;
    for (int64_t j = threadIdx.x; j < G; j += 256) acc += partials[j];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int k = 0; k < 8; ++k) s += red[k];
    const double lmid = 0.5 * (S[OC_L2] + S[OC_L1]);
    const double vol = s / S[OC_NEL];
    S[OC_LMID] = lmid;
    S[OC_VOL] = vol;
    if (vol > S[OC_VOLFRAC]) S[OC_L1] = lmid;
    else S[OC_L2] = lmid;
    S[OC_IT] += 1.0;
    if ((S[OC_L2] - S[OC_L1]) / (S[OC_L1] + S[OC_L2]) <= S[OC_TOL]) S[OC_DONE] = 1.0;
}

// x_new with the multiplier of the last probe
__global__ void oc_apply_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ dc,
                                const double* __restrict__ dv, double move, const double* __restrict__ S,
                                double* __restrict__ x_new) {
    vx::pdl_begin();
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x_new[i] = oc_design(x[i], dc[i], dv[i], S[OC_LMID], move);
}

int64_t oc_ctas(int64_t n) {
    int64_t g = (n + 256 * 8 - 1) / (256 * 8);
    return g < 1 ? 1 : (g > 1184 ? 1184 : g);
}

}  // namespace vx

using namespace vx;

extern "C" int vx_cone_filter(int nx, int ny, int nz, double rmin, const double* x, const double* s, int mode,
                              double* y, cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(x && y && (mode == 0 || s), VX_ERR_NULL_POINTER, "vx_cone_filter: NULL pointer");
    VX_CHECK_ARG(mode >= 0 && mode <= 2, VX_ERR_INVALID_ARGUMENT, "vx_cone_filter: mode must be 0, 1 or 2");
    VX_CHECK_ARG(rmin > 0 && rmin <= FILTER_MAX_R + 1, VX_ERR_INVALID_ARGUMENT,
                 "vx_cone_filter: rmin must be in (0, %d]", FILTER_MAX_R + 1);
    VX_CHECK_ARG(x != y, VX_ERR_INVALID_ARGUMENT, "vx_cone_filter: y may not alias x");
    FilterTaps t{};
    const int R = std::max(0, int(std::ceil(rmin)) - 1);
    for (int dx = -R; dx <= R; ++dx)
        for (int dy = -R; dy <= R; ++dy)
            for (int dz = -R; dz <= R; ++dz) {
                const double w = rmin - std::sqrt(double(dx * dx + dy * dy + dz * dz));
                if (w <= 0) continue;
                t.d[t.n][0] = (signed char)dx; t.d[t.n][1] = (signed char)dy; t.d[t.n][2] = (signed char)dz;
                t.w[t.n] = w;
                ++t.n;
            }
    Grid g{nx, ny, nz};
    vx::launch(cone_filter_kernel, unsigned((g.elems() + 255) / 256), 256, 0, stream, g, t, x, s, mode, y);
    VX_CHECK_LAUNCH("vx_cone_filter");
    return VX_OK;
}

extern "C" int64_t vx_oc_partials(int64_t n) { return n > 0 ? oc_ctas(n) : 1; }

extern "C" int vx_oc_probe(int64_t n, const double* x, const double* dc, const double* dv, const double* w,
                           double move, const double* S, double* partials, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_oc_probe: n must be positive");
    VX_CHECK_ARG(x && dc && dv && w && S && partials, VX_ERR_NULL_POINTER, "vx_oc_probe: NULL pointer");
    vx::launch(oc_probe_kernel, unsigned(oc_ctas(n)), 256, 0, stream, n, x, dc, dv, w, move, S, partials);
    VX_CHECK_LAUNCH("vx_oc_probe");
    return VX_OK;
}

extern "C" int vx_oc_finalize(int64_t n, const double* partials, double* S, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_oc_finalize: n must be positive");
    VX_CHECK_ARG(partials && S, VX_ERR_NULL_POINTER, "vx_oc_finalize: NULL pointer");
    vx::launch(oc_finalize_kernel, 1, 256, 0, stream, oc_ctas(n), partials, S);
    VX_CHECK_LAUNCH("vx_oc_finalize");
    return VX_OK;
}

extern "C" int vx_oc_apply(int64_t n, const double* x, const double* dc, const double* dv, double move,
                           const double* S, double* x_new, cudaStream_t stream) {
    VX_CHECK_ARG(n > 0, VX_ERR_INVALID_ARGUMENT, "vx_oc_apply: n must be positive");
    VX_CHECK_ARG(x && dc && dv && S && x_new, VX_ERR_NULL_POINTER, "vx_oc_apply: NULL pointer");
    vx::launch(oc_apply_kernel, unsigned((n + 255) / 256), 256, 0, stream, n, x, dc, dv, move, S, x_new);
    VX_CHECK_LAUNCH("vx_oc_apply");
    return VX_OK;
}
