// Tensor-core element-block operator (an experiment kept for measurement, not used by the solvers).
//
// The dense form of the Hex8 product, y = sum_e E_e P_e^T K0 P_e u, run on sm_100's tensor cores:
// a tile of 128 consecutive elements of one element row (fixed x, y; z = z0 .. z0 + 127) gathers
// its element vectors u_e (8 nodes x 3 components, the node mask applied, zero-padded to 32) as
// the rows of A (128 x 32, TF32), B is K0 (rows padded to 32), and one elected thread issues four
// tcgen05.mma.kind::tf32 (K = 8 each) into a 128 x 32 FP32 accumulator in tensor memory.  Each
// thread then reads its element's row back with tcgen05.ld, scales it by E_e and adds it to the
// output nodes: the z neighbours of a warp combine their shared nodes with a shuffle, every other
// node sum is an FP32 atomic add (y is cleared first).
//
// Operands sit in shared memory in the K-major, no-swizzle canonical layout: 8-row x 16-byte core
// matrices, 128 bytes each; the core matrix of row group i and 16-byte K chunk j at (8 i + j) * 128
// bytes, so adjacent K chunks are 128 bytes apart (leading byte offset) and adjacent row groups
// 1024 bytes (stride byte offset).  The k-th MMA (K columns 8k .. 8k+7, two chunks) starts 256 k
// bytes in.
//
// The form does 576 multiply-adds per element (the parity form 150 operations) at tensor-core
// rate, but it has to move every element vector through shared memory and scatter 24 results per
// element, where the parity form keeps its separable stages in registers.  vx_tc_element_product
// with mode 1 writes the 24 scaled results per element unscattered, which times the block product
// alone.
#include "vx_common.cuh"

#include <algorithm>
#include <atomic>

namespace vx {
namespace {

constexpr int TC_M = 128;                  // elements per tile (MMA M)
constexpr int TC_N = 32;                   // output DOFs, 24 padded (MMA N)
constexpr int TC_K = 32;                   // input DOFs, 24 padded (4 MMAs of K = 8)
constexpr uint32_t TC_A_BYTES = TC_M * TC_K * 4;      // 16 KB
constexpr uint32_t TC_B_BYTES = TC_N * TC_K * 4;      // 4 KB
constexpr int TC_WAIT_LIMIT = 1 << 22;

__device__ int g_tc_fault;

struct TcArgs {
    Grid g;
    const float* u;
    const float* E;
    const uint8_t* node_mask;   // may be null
    float* y;
    int mode;                   // 0: scatter into nodes, 1: 24 outputs per element
    float K0[24 * 24];          // row-major, row = output DOF
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// K-major, no-swizzle shared-memory matrix descriptor (version 1, base offset 0, legacy LBO mode)
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;                // descriptor version for sm_100
    return d;                              // layout type 0: no swizzle
}
// instruction descriptor: TF32 x TF32 -> F32, both K-major, M = 128, N = 32
constexpr uint32_t tc_idesc() {
    return (1u << 4)                       // D format F32
         | (2u << 7) | (2u << 10)          // A, B format TF32
         | (uint32_t(TC_N >> 3) << 17)
         | (uint32_t(TC_M >> 4) << 24);
}
// byte offset of (row, k) in a K-major canonical tile with 8 K chunks of 16 bytes per row group
__device__ __forceinline__ uint32_t canon(int row, int k) {
    return uint32_t(((row >> 3) * 8 + (k >> 2)) * 128 + (row & 7) * 16 + (k & 3) * 4);
}
__device__ __forceinline__ float to_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}

__global__ void __launch_bounds__(TC_M, 4) tc_element_kernel(const __grid_constant__ TcArgs a) {
    pdl_begin();
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* As = smem;                                   // 16 KB
    unsigned char* Bs = smem + TC_A_BYTES;                      // 4 KB
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + TC_A_BYTES + TC_B_BYTES);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const Grid g = a.g;

    // B = K0 (zero padded), A's padding columns 24..31: written once
    for (int i = t; i < TC_N * TC_K; i += TC_M) {
        const int n = i / TC_K, k = i % TC_K;
        *reinterpret_cast<float*>(Bs + canon(n, k)) = (n < 24 && k < 24) ? to_tf32(a.K0[n * 24 + k]) : 0.f;
    }
    #pragma unroll
    for (int k = 24; k < TC_K; k += 4)
        *reinterpret_cast<float4*>(As + canon(t, k)) = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {   // 32 tensor-memory columns: the 128 x 32 FP32 accumulator
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_addr(tslot)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    const uint64_t adesc0 = kmajor_desc(smem_addr(As), 128, 1024);
    const uint64_t bdesc0 = kmajor_desc(smem_addr(Bs), 128, 1024);

    const int ztiles = (g.nz + TC_M - 1) / TC_M;
    const int64_t tiles = int64_t(g.nx) * g.ny * ztiles;
    const int nz1 = g.nz + 1, plane = (g.ny + 1) * nz1;
    // offsets of the element's native nodes (the element matrix's node order)
    constexpr int OX[8] = {0, 1, 1, 0, 0, 1, 1, 0}, OY[8] = {0, 0, 1, 1, 0, 0, 1, 1}, OZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    unsigned phase = 0;
    bool ok = true;
    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int zt = int(tile % ztiles);
        const int64_t row = tile / ztiles;
        const int ey = int(row % g.ny), ex = int(row / g.ny);
        const int ez = zt * TC_M + t;
        const bool valid = ez < g.nz;
        const int ezc = valid ? ez : g.nz - 1;
        // ---- gather this thread's element vector into row t of A (TF32, node mask applied)
        float v[24];
        #pragma unroll
        for (int n = 0; n < 8; ++n) {
            const int node = (ex + OX[n]) * plane + (ey + OY[n]) * nz1 + ezc + OZ[n];
            const unsigned m = a.node_mask ? unsigned(a.node_mask[node]) : 7u;
            #pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float x = a.u[3 * node + c];
                v[3 * n + c] = (valid && ((m >> c) & 1u)) ? to_tf32(x) : 0.f;
            }
        }
        #pragma unroll
        for (int k = 0; k < 24; k += 4)
            *reinterpret_cast<float4*>(As + canon(t, k)) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // ---- one thread issues D = A B^T over K = 32 (four K = 8 steps) and commits to the barrier
        if (t == 0) {
            #pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t ad = adesc0 + uint64_t((256 * kk) >> 4);
                const uint64_t bd = bdesc0 + uint64_t((256 * kk) >> 4);
                const uint32_t acc = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(ad), "l"(bd), "r"(tc_idesc()), "r"(acc) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_addr(bar)) : "memory");
        }
        // ---- bounded wait for the accumulator
        bool done = false;
        for (int i = 0; i < TC_WAIT_LIMIT && !done; ++i) {
            uint32_t r;
            asm volatile("{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\tselp.u32 %0, 1, 0, q;\n\t}"
                         : "=r"(r) : "r"(smem_addr(bar)), "r"(phase) : "memory");
            done = r != 0;
        }
        phase ^= 1u;
        if (!__syncthreads_and(done)) {
            if (t == 0) atomicExch(&g_tc_fault, 1);
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // ---- row t of the accumulator: this element's 24 results (columns 24..31 are padding)
        uint32_t d[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
              "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
              "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
              "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
            : "r"(tmem + (uint32_t(warp * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const float Ee = valid ? a.E[(int64_t(ex) * g.ny + ey) * g.nz + ez] : 0.f;
        float o[24];
        #pragma unroll
        for (int i = 0; i < 24; ++i) o[i] = Ee * __uint_as_float(d[i]);
        if (a.mode == 1) {
            if (valid) {
                float* yp = a.y + 24 * ((int64_t(ex) * g.ny + ey) * g.nz + ez);
                #pragma unroll
                for (int i = 0; i < 24; ++i) yp[i] = o[i];
            }
        } else {
            // nodes at z + 1 (native 4..7) meet the next element's nodes at z (native 0..3):
            // lane l + 1 adds lane l's share, the last lane of a warp adds its own atomically
            #pragma unroll
            for (int n = 0; n < 4; ++n) {
                #pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float up = __shfl_up_sync(0xffffffffu, o[3 * (n + 4) + c], 1);
                    const float s = o[3 * n + c] + (lane > 0 ? up : 0.f);
                    if (valid) {
                        const int node = (ex + OX[n]) * plane + (ey + OY[n]) * nz1 + ez;
                        atomicAdd(a.y + 3 * node + c, s);
                    }
                }
            }
            const bool tail = lane == 31 || !(ez + 1 < g.nz) || t == TC_M - 1;
            if (valid && tail) {
                #pragma unroll
                for (int n = 4; n < 8; ++n) {
                    const int node = (ex + OX[n]) * plane + (ey + OY[n]) * nz1 + ez + 1;
                    #pragma unroll
                    for (int c = 0; c < 3; ++c) atomicAdd(a.y + 3 * node + c, o[3 * n + c]);
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();                       // every row read before the next tile's MMA
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
}

}  // namespace
}  // namespace vx

using namespace vx;

// Tensor-core element-block operator (FP32 storage, TF32 products, FP32 accumulation).  mode 0:
// y = K(E) (m . u) over the nodes (y overwritten; the node mask, if given, zeroes constrained
// components of u); mode 1: y[24 e + i] = E_e (K0 P_e (m . u))_i per element.  Experimental: no
// counterpart in the reference's solvers (its donor ships a BF16 WMMA element-block matvec).
extern "C" int vx_tc_element_product(int nx, int ny, int nz, const double* ke, const float* E, const uint8_t* node_mask,
                                     const float* u, float* y, int mode, cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(ke && E && u && y, VX_ERR_NULL_POINTER, "vx_tc_element_product: NULL pointer");
    VX_CHECK_ARG(mode == 0 || mode == 1, VX_ERR_INVALID_ARGUMENT, "vx_tc_element_product: mode %d", mode);
    TcArgs a{};
    a.g = Grid{nx, ny, nz};
    a.u = u; a.E = E; a.node_mask = node_mask; a.y = y; a.mode = mode;
    for (int i = 0; i < 576; ++i) a.K0[i] = float(ke[i]);
    if (mode == 0) {
        cudaError_t e = cudaMemsetAsync(y, 0, sizeof(float) * 3 * size_t(a.g.nodes()), stream);
        if (e != cudaSuccess) {
            set_error("vx_tc_element_product: %s", cudaGetErrorString(e));
            return VX_ERR_CUDA;
        }
    }
    const size_t smem = TC_A_BYTES + TC_B_BYTES + 16;
    static std::atomic<uint64_t> cfg;
    st = smem_opt_in(cfg, (const void*)tc_element_kernel, smem, "vx_tc_element_product");
    if (st) return st;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t tiles = int64_t(nx) * ny * ((nz + TC_M - 1) / TC_M);
    const unsigned grid = unsigned(std::min<int64_t>(tiles, int64_t(sms) * 4));
    launch(tc_element_kernel, grid, TC_M, smem, stream, a);
    VX_CHECK_LAUNCH("vx_tc_element_product");
    return VX_OK;
}

// Fault flag of the tensor-core kernel's bounded accumulator wait (0 in every correct run);
// cleared when `clear` is non-zero.  Synchronous with respect to the device.
extern "C" int vx_tc_status(int* status, int clear) {
    VX_CHECK_ARG(status, VX_ERR_NULL_POINTER, "vx_tc_status: NULL status");
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_tc_fault, sizeof(int));
    if (e == cudaSuccess && clear && v) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_tc_fault, &zero, sizeof(int));
    }
    if (e != cudaSuccess) {
        set_error("vx_tc_status: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    *status = v;
    return VX_OK;
}
