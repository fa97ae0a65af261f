// Shared definitions for libvoxel_b200: status codes, the thread-local error string, launch checks,
// storage types and the 45-entry parity-block pattern of an affine brick Hex8 element.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <atomic>
#include <cstdio>
#include <string>
#include <utility>

#include "../../include/voxel_b200.h"

namespace vx {

// Last error message of the calling host thread (returned by vx_last_error()).
void set_error(const char* fmt, ...);

#define VX_CHECK_ARG(cond, code, ...)            \
    do {                                         \
        if (!(cond)) {                           \
            ::vx::set_error(__VA_ARGS__);        \
            return (code);                       \
        }                                        \
    } while (0)

#define VX_CHECK_LAUNCH(what)                                                              \
    do {                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess) {                                                           \
            ::vx::set_error("%s: launch failed: %s", (what), cudaGetErrorString(e_));      \
            return VX_ERR_LAUNCH;                                                          \
        }                                                                                  \
    } while (0)

inline bool aligned(const void* p, size_t bytes) { return (reinterpret_cast<uintptr_t>(p) % bytes) == 0; }

// ---------------------------------------------------------------------------- launches
// Every kernel of the library is launched with programmatic stream serialization: the next kernel
// in the stream may be scheduled while this one drains, which hides the launch gap between the
// many short kernels of a solver iteration (also inside captured graphs).  Correctness does not
// depend on it: every kernel begins with pdl_begin(), whose griddepcontrol.wait returns only once
// the previous kernel has completed and its memory is visible (at once when there is none); its
// trigger then lets the following kernel be scheduled.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" :::);
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                          Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Launch-time opt-in to more than 48 KB of dynamic shared memory, once per kernel and device (the
// attribute is per device; `done` is the kernel's own bit set of configured devices, updated
// atomically, so concurrent first launches at worst set the attribute twice).  The solvers run
// every loop body once un-captured before capturing it, so the first call for a kernel never
// happens inside a stream capture.
inline int smem_opt_in(std::atomic<uint64_t>& done, const void* kern, size_t smem, const char* what) {
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = dev < 64 ? uint64_t(1) << dev : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return VX_OK;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) {
        set_error("%s: cudaFuncSetAttribute: %s", what, cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    done.fetch_or(bit, std::memory_order_acq_rel);
    return VX_OK;
}

// Grid extents: element grid (nx, ny, nz); nodes (nx+1)(ny+1)(nz+1); author layout, z fastest.
struct Grid {
    int nx, ny, nz;
    __host__ __device__ int64_t nodes() const { return int64_t(nx + 1) * (ny + 1) * (nz + 1); }
    __host__ __device__ int64_t elems() const { return int64_t(nx) * ny * nz; }
    __host__ __device__ int64_t node(int ix, int iy, int iz) const {
        return (int64_t(ix) * (ny + 1) + iy) * (nz + 1) + iz;
    }
    __host__ __device__ int64_t elem(int ex, int ey, int ez) const {
        return (int64_t(ex) * ny + ey) * nz + ez;
    }
};

int check_grid(int nx, int ny, int nz);

// ---------------------------------------------------------------------------- storage conversion
template <typename S> struct Storage;
// load: value in arithmetic type; raw/cvt: load without touching the value, convert at use;
// round: the arithmetic value that storing v would leave in memory
template <> struct Storage<double> {
    using raw_t = double;
    __device__ static double round(double v) { return v; }
    __device__ static double load(const double* p) { return *p; }
    __device__ static double raw(const double* p) { return *p; }
    __device__ static double cvt(double v) { return v; }
    __device__ static void store(double* p, double v) { *p = v; }
};
template <> struct Storage<float> {
    using raw_t = float;
    __device__ static float round(float v) { return v; }
    __device__ static float load(const float* p) { return *p; }
    __device__ static float raw(const float* p) { return *p; }
    __device__ static float cvt(float v) { return v; }
    __device__ static void store(float* p, float v) { *p = v; }
};
template <> struct Storage<__nv_bfloat16> {
    using raw_t = __nv_bfloat16;
    __device__ static float round(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
    __device__ static float load(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    __device__ static __nv_bfloat16 raw(const __nv_bfloat16* p) { return *p; }
    __device__ static float cvt(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ static void store(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};
// arithmetic type of a storage type (bf16 -> float)
template <typename S> using arith_t = decltype(Storage<S>::load(static_cast<const S*>(nullptr)));

// ---------------------------------------------------------------------------- storage selectors
// Iterate (X), auxiliary-vector (R) and modulus (M) storage of each VX_* selector.
template <int P> struct PrecT;
template <> struct PrecT<VX_F64> { using X = double; using R = double; using M = double; };
template <> struct PrecT<VX_F32> { using X = float; using R = float; using M = float; };
template <> struct PrecT<VX_BF16_F32> { using X = __nv_bfloat16; using R = __nv_bfloat16; using M = __nv_bfloat16; };
template <> struct PrecT<VX_F32_BF16AUX> { using X = float; using R = __nv_bfloat16; using M = __nv_bfloat16; };

// Calls f(PrecT<P>{}) for the runtime selector `prec`; false if it is not a selector.
template <typename F>
bool dispatch_prec(int prec, F&& f) {
    switch (prec) {
        case VX_F64: f(PrecT<VX_F64>{}); return true;
        case VX_F32: f(PrecT<VX_F32>{}); return true;
        case VX_BF16_F32: f(PrecT<VX_BF16_F32>{}); return true;
        case VX_F32_BF16AUX: f(PrecT<VX_F32_BF16AUX>{}); return true;
        default: return false;
    }
}

// ---------------------------------------------------------------------------- parity blocks
// The parity (Walsh-Hadamard) form of an affine-brick Hex8 element matrix: T ke T^T / 64 is block
// diagonal with 8 groups of 3x3; group g couples component x at parity g^1, y at g^2, z at g^4
// (parity p = px + 2 py + 4 pz).  Translations (parity 0) have zero rows, so 45 of the 72 entries
// are structurally non-zero.  The kernels take the 72 coefficients by value and use only these 45.
struct Blocks {
    double c[72];   // c[9*g + 3*a + b] = block g, row a (component a), column b
};
template <typename T> struct BlocksT { T c[72]; };

// true if entry (g, a, b) of the parity blocks is structurally non-zero for a brick element
__host__ __device__ constexpr bool parity_nonzero(int g, int a, int b) {
    // parity of component a in group g is g ^ (1 << a); a zero parity (translation) has no stiffness
    return ((g ^ (1 << a)) != 0) && ((g ^ (1 << b)) != 0) &&
           // cross-coupling pattern (a != b): measured structure of T ke T^T for a brick
           (a == b || !((g == 3 && (a == 2 || b == 2)) || (g == 5 && (a == 1 || b == 1)) ||
                        (g == 6 && (a == 0 || b == 0))));
}

}  // namespace vx
