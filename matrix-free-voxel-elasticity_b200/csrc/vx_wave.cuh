// parity_wave: the streaming Hex8 operator as a wavefront of warps (FP64 and FP32 iterates).
//
// Same arithmetic as parity_stream_xp (parity form, separable X / Y / Z stages shared between
// neighbouring elements, E folded into the Z stage, cube-pattern block product, node-owned tiles
// with recomputed halo elements, no atomics), organised for B200's latency budget:
//
//  * A CTA is NW = 16 warps, one per node row (warp r <-> node row iy0 - 1 + r, lane <-> node column
//    iz0 - 1 + lane).  Every warp computes the element row iy of its node row; rows 1..15 and lanes
//    1..30 own their nodes, so the halo overhead is 16/15 in y and 32/30 in z (1.14x in all).
//  * The node planes a warp needs -- its own row and the row above, both components x, y, z --
//    are staged by cp.async into a per-warp shared-memory ring DEPTH steps deep, together with the
//    element modulus and the node masks.  Each thread copies exactly the words it later reads, so
//    a thread's own cp.async.wait_group is the only synchronisation the staging needs, and loads
//    in flight occupy no registers.
//  * The only exchange between warps is the inverse-Y contribution a row sends to the row above
//    (6 values per lane per step).  It goes through shared memory under a pair of mbarriers per row
//    and buffer (full: the producer row arrives after writing, empty: the consumer arrives after
//    reading), so rows advance as a wavefront: a warp waits only for its lower neighbour, and there
//    is no CTA-wide barrier in the streaming loop.  Every wait is bounded; a wait that runs out
//    raises a device fault flag (vx_device_status) and the CTA abandons its work.
//  * The z exchange stays in registers (shuffles); the x stage is carried along the march.
//  * FP64 processes one element plane per step (about 100 registers, 16 warps per SM); FP32 two
//    element planes per step as packed f32x2 pairs (sm_100 FFMA2 / FADD2 / FMUL2).
//  * CTAs are persistent, one per SM: work items are (x chunk, y tile, z tile) in that order,
//    dealt round-robin, so the CTAs in flight work on neighbouring tiles of one x chunk and the
//    halo rows they share are served from L2.  The staging ring streams across item boundaries,
//    so a CTA pays the load latency once, not once per item.
#pragma once

#include "vx_common.cuh"
#include "vx_pair.cuh"
#include <type_traits>

namespace vx {

// ---------------------------------------------------------------- scalar "pairs" (FP64, one plane)
__device__ __forceinline__ double add2(double a, double b) { return a + b; }
__device__ __forceinline__ double sub2(double a, double b) { return a - b; }
__device__ __forceinline__ double mul2(double a, double b) { return a * b; }
__device__ __forceinline__ double fma2(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ double cmul2(double c, double a) { return c * a; }
__device__ __forceinline__ double cfma2(double c, double a, double acc) { return fma(c, a, acc); }
__device__ __forceinline__ double shfl_down2(double a, int d) { return __shfl_down_sync(0xffffffffu, a, d); }
__device__ __forceinline__ double shfl_up2(double a, int d) { return __shfl_up_sync(0xffffffffu, a, d); }

template <typename TC> struct WaveCfg;
template <> struct WaveCfg<double> {
    static constexpr int PL = 1;      // element planes per step
    static constexpr int NW = 16;     // warps (node rows) per CTA
    static constexpr int DEPTH = 4;   // staging ring slots (steps)
    using P = double;
    __device__ static P pk(const double* v) { return v[0]; }
    __device__ static double get(P p, int) { return p; }
    __device__ static P zero() { return 0.0; }
    __device__ static P neg(P p) { return -p; }
};
template <> struct WaveCfg<float> {
    static constexpr int PL = 2;
    static constexpr int NW = 16;
    static constexpr int DEPTH = 4;
    using P = V2<float>;
    __device__ static P pk(const float* v) { return mk2(v[0], v[1]); }
    __device__ static float get(P p, int h) { return h ? p.hi() : p.lo(); }
    __device__ static P zero() { return mk2(0.f, 0.f); }
    __device__ static P neg(P p) { return mk2(-p.lo(), -p.hi()); }
};

constexpr int WAVE_TZ = 30;   // owned node columns per tile (lanes 1..30)

// Work decomposition of one launch (host-computed): items (chunk, ytile, ztile), chunk-major.
struct WaveSched {
    int tz, ty;          // z tiles, y tiles
    int cx;              // node planes per x chunk
    int chunks;
    int items;           // chunks * ty * tz
};

// ---------------------------------------------------------------- staging helpers
template <typename T> using stage_t = std::conditional_t<(sizeof(T) >= 4), T, uint32_t>;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copy base[idx] (0 <= idx < count) asynchronously into *dst.  Values narrower than 4 bytes travel
// as the aligned 32-bit word that holds them; where that word reaches outside [base, base + count)
// the value is read alone by a plain load instead, so nothing outside the array is touched.
template <typename T>
__device__ __forceinline__ void stage1(stage_t<T>* dst, const T* base, int idx, int count) {
    if constexpr (sizeof(T) >= 4) {
        cp_async<sizeof(T)>(dst, base + idx);
    } else {
        using U = std::conditional_t<sizeof(T) == 1, uint8_t, uint16_t>;
        const uintptr_t at = reinterpret_cast<uintptr_t>(base + idx);
        const uintptr_t w0 = at & ~uintptr_t(3);
        if (w0 >= reinterpret_cast<uintptr_t>(base) && w0 + 4 <= reinterpret_cast<uintptr_t>(base + count)) {
            cp_async<4>(dst, reinterpret_cast<const void*>(w0));
        } else {
            const uint32_t v = uint32_t(*reinterpret_cast<const U*>(base + idx));
            *dst = v << (8 * (at & 3));
        }
    }
}
// The value that stage1(dst, base, idx, ...) left in *dst (p = base + idx).
template <typename T>
__device__ __forceinline__ T unstage(const stage_t<T>& s, const T* p) {
    if constexpr (sizeof(T) >= 4) {
        return s;
    } else {
        using U = std::conditional_t<sizeof(T) == 1, uint8_t, uint16_t>;
        const U bits = U(s >> (8 * (reinterpret_cast<uintptr_t>(p) & 3)));
        return *reinterpret_cast<const T*>(&bits);
    }
}

// Bulk (TMA-engine) copy of `bytes` (a multiple of 16) from 16-byte aligned global memory into shared
// memory, completing as transaction bytes on the mbarrier `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// Orders this thread's earlier generic-proxy accesses of shared memory before later async-proxy
// writes to it (a staging slot that was read is refilled by bulk copies).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One staged row: elements [first, first + cnt) of an array of `total` elements of `es` bytes whose
// base is 16-byte aligned.  The bulk copy starts at the 16-byte boundary at or below the first
// element (`off` bytes before it) and covers whole 16-byte units; `bulk` is false when that would
// read past the array's end (the row is then copied element by element).
struct RowSpan {
    const unsigned char* src;
    uint32_t len;
    uint32_t off;
    bool bulk;
};
__device__ __forceinline__ RowSpan row_span(const void* base, int first, int cnt, int es, int total) {
    const uintptr_t b = reinterpret_cast<uintptr_t>(base);
    const uintptr_t g0 = b + uintptr_t(first) * uintptr_t(es);
    const uintptr_t a0 = g0 & ~uintptr_t(15);
    const uint32_t off = uint32_t(g0 - a0);
    const uint32_t len = (off + uint32_t(cnt) * uint32_t(es) + 15u) & ~15u;
    RowSpan r;
    r.src = reinterpret_cast<const unsigned char*>(a0);
    r.len = len;
    r.off = off;
    r.bulk = a0 + len <= b + uintptr_t(total) * uintptr_t(es);
    return r;
}

// ---------------------------------------------------------------- mbarriers (CTA scope)
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Device fault flag of the streaming kernels: set when a bounded wait ran out (never in a correct
// run).  Read and cleared by vx_device_status.
__device__ int g_wave_fault;
constexpr int WAVE_WAIT_LIMIT = 1 << 22;

// Bounded wait of a whole warp for the phase `parity` of `bar` (the outcome is warp-uniform); gives
// up early once another warp of the CTA aborted.  Returns false when the wait ran out or the CTA
// aborted; running out raises the fault flag and aborts the CTA.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, volatile int* abort_flag) {
    for (int i = 0; i < WAVE_WAIT_LIMIT; ++i) {
        const bool ok = mbar_try_wait(bar, parity);
        if (__all_sync(0xffffffffu, ok)) return true;
        if (__any_sync(0xffffffffu, *abort_flag != 0)) return false;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicExch(&g_wave_fault, 1);
        *abort_flag = 1;
    }
    __syncwarp();
    return false;
}

// ---------------------------------------------------------------- the kernel
// Shared memory of one launch.  Per warp, a ring of DEPTH staging slots; a slot holds PL node planes.
// cp.async staging (BULK = false): each thread's words, [slot][plane][item][lane].  Bulk staging
// (BULK = true): whole rows as the bulk copies leave them -- own and upper u rows (96 values each),
// the element modulus row, the two mask rows -- each starting `off` bytes into a 16-byte aligned
// buffer.  Then the exchange buffers of every row and the mbarriers: full/empty of the exchange
// (4 per row), the bulk staging's full barrier per row and slot, the abort flag.
template <typename TC, typename TU, typename TE, typename TY, typename TR, int EPI, int MASK, bool CUBIC, bool BULK>
struct WaveLayout {
    using Cfg = WaveCfg<TC>;
    static constexpr int PL = Cfg::PL, NW = Cfg::NW, D = Cfg::DEPTH;
    using P = typename Cfg::P;
    static constexpr bool HAS_M = MASK == MASK_NODE;
    static constexpr size_t U_B = sizeof(stage_t<TU>) * D * PL * 6 * 32;    // own + upper row, 3 components
    static constexpr size_t E_B = sizeof(stage_t<TE>) * D * PL * 32;
    static constexpr size_t M_B = HAS_M ? sizeof(uint32_t) * D * PL * 2 * 32 : 0;
    static constexpr uint32_t RBU = (15 + 96 * sizeof(TU) + 15) / 16 * 16;   // bulk row buffers
    static constexpr uint32_t RBE = (15 + 32 * sizeof(TE) + 15) / 16 * 16;
    static constexpr uint32_t RBM = HAS_M ? (15 + 32 + 15) / 16 * 16 : 0;
    static constexpr uint32_t ROWSET = 2 * RBU + RBE + 2 * RBM;              // one plane's rows
    static constexpr size_t WARP_B = BULK ? size_t(D) * PL * ROWSET : (U_B + E_B + M_B + 15) / 16 * 16;
    static constexpr size_t HS_B = sizeof(P) * 2 * 6 * 32;                  // per row, two buffers
    static constexpr size_t BAR_OFF = NW * (WARP_B + HS_B);
    static constexpr int NBARS = 4 * NW + (BULK ? NW * D : 0);
    static constexpr size_t BYTES = BAR_OFF + sizeof(uint64_t) * NBARS + 16;
};

template <typename TC, typename TU, typename TE, typename TY, typename TR, int EPI, int MASK, bool CUBIC, bool BULK>
__global__ void __launch_bounds__(WaveCfg<TC>::NW * 32, 1)
parity_wave(const __grid_constant__ OpArgs2<TC, TU, TE, TY, TR> args, const __grid_constant__ WaveSched ws) {
    vx::pdl_begin();
    using Cfg = WaveCfg<TC>;
    using L = WaveLayout<TC, TU, TE, TY, TR, EPI, MASK, CUBIC, BULK>;
    constexpr int PL = Cfg::PL, NWW = Cfg::NW, D = Cfg::DEPTH, A = D - 2;
    using P = typename Cfg::P;
    using SU = stage_t<TU>;
    using SE = stage_t<TE>;
    constexpr bool HAS_M = MASK == MASK_NODE;
    constexpr bool HAS_R = EPI == EPI_JACOBI || EPI == EPI_RESIDUAL || EPI == EPI_TRUE_RES;
    constexpr bool HAS_D = EPI == EPI_JACOBI;
    const auto& a = args.a;
    const Grid g = a.g;
    const int lane = threadIdx.x & 31;
    const int row = threadIdx.x >> 5;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* wb = smem_raw + size_t(row) * L::WARP_B;
    SU* su = reinterpret_cast<SU*>(wb);
    SE* se = reinterpret_cast<SE*>(wb + L::U_B);
    uint32_t* sm = reinterpret_cast<uint32_t*>(wb + L::U_B + L::E_B);
    P* hs = reinterpret_cast<P*>(smem_raw + NWW * L::WARP_B);             // [NWW][2][6][32]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + L::BAR_OFF);  // full[NWW][2], empty[NWW][2]
    uint64_t* sbar = bars + 4 * NWW + row * D;                            // bulk staging: this row's slots
    volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + L::NBARS);
#define SU_(s, h, c) su[(((s) * PL + (h)) * 6 + (c)) * 32 + lane]
#define SE_(s, h) se[((s) * PL + (h)) * 32 + lane]
#define SM_(s, h, w) sm[(((s) * PL + (h)) * 2 + (w)) * 32 + lane]
#define HS_(r, b, k) hs[(((r) * 2 + (b)) * 6 + (k)) * 32 + lane]
    if (threadIdx.x < 4 * NWW) mbar_init(bars + threadIdx.x, 32);
    if constexpr (BULK) {
        if (threadIdx.x < NWW * D) mbar_init(bars + 4 * NWW + threadIdx.x, 1);
    }
    if (threadIdx.x == 0) *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();

    const int nyz_nodes = (g.ny + 1) * (g.nz + 1);
    const int nyz_elems = g.ny * g.nz;
    const int n_nodes = (g.nx + 1) * nyz_nodes;
    const int n_elems = g.nx * nyz_elems;
    const int stride = gridDim.x;

    // A cursor walks this CTA's items (blockIdx.x, + gridDim.x, ...) one step at a time; step -1 of
    // an item only stages its first node planes.
    struct Cursor {
        int item, j, steps, x0, x1;
        int cn_own, cn_nb, ce;        // clamped column offsets: own node, upper node, own element
        int iy, iz;
        int lo, hi, elo, ehi;         // bulk rows: first and last node / element column of the tile
        int row_o, row_u, row_e;      // their row offsets within a plane (own, upper node row; element row)
    };
    auto open = [&](Cursor& c, int item) {
        c.item = item;
        c.j = -1;
        if (item >= ws.items) return;
        const int col = item % (ws.tz * ws.ty), chunk = item / (ws.tz * ws.ty);
        const int zt = col % ws.tz, yt = col / ws.tz;
        c.x0 = chunk * ws.cx;
        c.x1 = min(c.x0 + ws.cx, g.nx + 1);
        c.steps = (c.x1 - c.x0 + 1 + PL - 1) / PL;
        c.iz = zt * WAVE_TZ - 1 + lane;
        c.iy = yt * (NWW - 1) - 1 + row;
        const int izc = min(max(c.iz, 0), g.nz), iyc = min(max(c.iy, 0), g.ny), iyn = min(max(c.iy + 1, 0), g.ny);
        c.cn_own = iyc * (g.nz + 1) + izc;
        c.cn_nb = iyn * (g.nz + 1) + izc;
        c.ce = min(max(c.iy, 0), g.ny - 1) * g.nz + min(max(c.iz, 0), g.nz - 1);
        const int z0 = zt * WAVE_TZ;
        c.lo = max(z0 - 1, 0);
        c.hi = min(z0 + 30, g.nz);
        c.elo = max(z0 - 1, 0);
        c.ehi = min(z0 + 30, g.nz - 1);
        c.row_o = iyc * (g.nz + 1);
        c.row_u = iyn * (g.nz + 1);
        c.row_e = min(max(c.iy, 0), g.ny - 1) * g.nz;
    };
    auto advance = [&](Cursor& c) {
        if (c.item >= ws.items) return;
        if (++c.j >= c.steps) open(c, c.item + stride);
    };

    // stage the node planes of step j of cursor c (x0 + PL j + h, h < PL) into slot s
    auto stage_step = [&](const Cursor& c, int s) {
        #pragma unroll
        for (int h = 0; h < PL; ++h) {
            const int q = min(max(c.x0 + PL * c.j + h, 0), g.nx);
            const int no = q * nyz_nodes + c.cn_own, nn = q * nyz_nodes + c.cn_nb;
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                stage1<TU>(&SU_(s, h, k), a.u, 3 * no + k, 3 * n_nodes);
                stage1<TU>(&SU_(s, h, 3 + k), a.u, 3 * nn + k, 3 * n_nodes);
            }
            const int qe = min(max(c.x0 + PL * c.j + h - 1, 0), g.nx - 1);
            stage1<TE>(&SE_(s, h), a.E, qe * nyz_elems + c.ce, n_elems);
            if constexpr (HAS_M) {
                stage1<uint8_t>(&SM_(s, h, 0), a.node_mask, no, n_nodes);
                stage1<uint8_t>(&SM_(s, h, 1), a.node_mask, nn, n_nodes);
            }
        }
    };

    // bulk staging of step j of cursor c into slot s: lane 0 issues one bulk copy per row (an edge
    // row near the array's end is copied by the lanes, each the values it will read)
    unsigned char* wbulk = wb;
    auto stage_bulk = [&](const Cursor& c, int s) {
        __syncwarp();
        fence_proxy_async();
        const int ln = min(max(c.iz, c.lo), c.hi) - c.lo, le = min(max(c.iz, c.elo), c.ehi) - c.elo;
        const int ncols = c.hi - c.lo + 1, necols = c.ehi - c.elo + 1;
        auto spans = [&](int h, RowSpan* sp) {
            const int q = min(max(c.x0 + PL * c.j + h, 0), g.nx);
            const int qe = min(max(c.x0 + PL * c.j + h - 1, 0), g.nx - 1);
            sp[0] = row_span(a.u, 3 * (q * nyz_nodes + c.row_o + c.lo), 3 * ncols, int(sizeof(TU)), 3 * n_nodes);
            sp[1] = row_span(a.u, 3 * (q * nyz_nodes + c.row_u + c.lo), 3 * ncols, int(sizeof(TU)), 3 * n_nodes);
            sp[2] = row_span(a.E, qe * nyz_elems + c.row_e + c.elo, necols, int(sizeof(TE)), n_elems);
            if constexpr (HAS_M) {
                sp[3] = row_span(a.node_mask, q * nyz_nodes + c.row_o + c.lo, ncols, 1, n_nodes);
                sp[4] = row_span(a.node_mask, q * nyz_nodes + c.row_u + c.lo, ncols, 1, n_nodes);
            }
        };
        constexpr int NR = HAS_M ? 5 : 3;
        const uint32_t dst_off[5] = {0u, L::RBU, 2 * L::RBU, 2 * L::RBU + L::RBE, 2 * L::RBU + L::RBE + L::RBM};
        uint32_t tx = 0;
        #pragma unroll
        for (int h = 0; h < PL; ++h) {
            RowSpan sp[5];
            spans(h, sp);
            #pragma unroll
            for (int r = 0; r < NR; ++r) tx += sp[r].bulk ? sp[r].len : 0u;
        }
        if (lane == 0) mbar_arrive_expect_tx(sbar + s, tx);
        #pragma unroll
        for (int h = 0; h < PL; ++h) {
            RowSpan sp[5];
            spans(h, sp);
            unsigned char* rows = wbulk + (size_t(s) * PL + h) * L::ROWSET;
            #pragma unroll
            for (int r = 0; r < NR; ++r) {
                unsigned char* dst = rows + dst_off[r];
                if (sp[r].bulk) {
                    if (lane == 0) bulk_g2s(dst, sp[r].src, sp[r].len, sbar + s);
                } else if (r < 2) {
                    #pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const int i = 3 * ln + k;
                        reinterpret_cast<TU*>(dst + sp[r].off)[i] = reinterpret_cast<const TU*>(sp[r].src + sp[r].off)[i];
                    }
                } else if (r == 2) {
                    reinterpret_cast<TE*>(dst + sp[r].off)[le] = reinterpret_cast<const TE*>(sp[r].src + sp[r].off)[le];
                } else {
                    dst[sp[r].off + ln] = sp[r].src[sp[r].off + ln];
                }
            }
        }
    };
    // bulk fills issued and not yet waited for (bit per slot), and the phase parity of each slot's
    // latest fill: what an aborting warp still has to wait for before its CTA may exit
    unsigned pending = 0u, pend_par = 0u;
    auto issue = [&](const Cursor& c, int t) {
        const int s = t % D;
        if constexpr (BULK) {
            stage_bulk(c, s);
            pending |= 1u << s;
            pend_par = (pend_par & ~(1u << s)) | ((unsigned(t / D) & 1u) << s);
        } else {
            stage_step(c, s);
        }
    };
    // this thread may read stream step t's slot: its own copies landed (cp.async), or the warp's
    // bulk copies completed on the slot's barrier (phase = how often the slot was filled before)
    auto wait_step = [&](int t) -> bool {
        if constexpr (BULK) {
            const int s = t % D;
            const bool ok = mbar_wait(sbar + s, unsigned(t / D) & 1u, abort_flag);
            if (ok) pending &= ~(1u << s);
            return ok;
        } else {
            cp_async_wait<A>();
            return true;
        }
    };

    Cursor prod, cons;
    open(prod, blockIdx.x);
    open(cons, blockIdx.x);
    // prefill: the first A steps of the stream go to slots 0 .. A-1
    #pragma unroll
    for (int t = 0; t < A; ++t) {
        if (prod.item < ws.items) issue(prod, t);
        if constexpr (!BULK) cp_async_commit();
        advance(prod);
    }

    TC carry[3] = {TC(0), TC(0), TC(0)};
    double acc = 0.0;
    int cstep = 0;            // compute steps so far (exchange buffer and phase)
    bool live = true;
    for (int t = 0; live && cons.item < ws.items; ++t) {
        // ---- producer: stream step t + A into its slot (an empty group past the end keeps the count)
        if (prod.item < ws.items) issue(prod, t + A);
        if constexpr (!BULK) cp_async_commit();
        advance(prod);
        if (!wait_step(t)) { live = false; break; }         // step t's staging has landed
        if (cons.j < 0) {                                    // first step of an item: staging only
            #pragma unroll
            for (int k = 0; k < 3; ++k) carry[k] = TC(0);
            advance(cons);
            continue;
        }
        const int sp = (t + D - 1) % D, sc = t % D;         // slot of node plane e, of planes e+1..e+PL
        const int e = cons.x0 - 1 + PL * cons.j;

        // ---- epilogue operands of this step's output planes e .. e+PL-1 (plain loads; used at the end)
        const bool owner = lane >= 1 && lane <= WAVE_TZ && row >= 1 && cons.iy <= g.ny && cons.iz <= g.nz;
        const int col = cons.iy * (g.nz + 1) + cons.iz;      // owners only
        TC rr[PL][3], dd[PL][3];
        if constexpr (HAS_R) {
            #pragma unroll
            for (int h = 0; h < PL; ++h) {
                const int ixo = e + h;
                if (owner && ixo >= cons.x0 && ixo < cons.x1) {
                    const TR* rp = a.r + 3 * (ixo * nyz_nodes + col);
                    #pragma unroll
                    for (int k = 0; k < 3; ++k) rr[h][k] = TC(Storage<TR>::load(rp + k));
                    if constexpr (HAS_D) {
                        const TR* dp = a.invd + 3 * (ixo * nyz_nodes + col);
                        #pragma unroll
                        for (int k = 0; k < 3; ++k) dd[h][k] = TC(Storage<TR>::load(dp + k));
                    }
                } else {
                    #pragma unroll
                    for (int k = 0; k < 3; ++k) { rr[h][k] = TC(0); dd[h][k] = TC(0); }
                }
            }
        }

        // ---- node planes e .. e+PL from the ring: raw own row, masked own and upper rows
        TC uo[PL + 1][3], un[PL + 1][3], ur[PL][3];
        unsigned bo[PL + 1];
        #pragma unroll
        for (int h = 0; h <= PL; ++h) {
            const int s = h == 0 ? sp : sc, hh = h == 0 ? PL - 1 : h - 1;
            const int q = min(max(e + h, 0), g.nx);
            unsigned mo = 7u, mn = 7u;
            const TU* pvo;
            const TU* pvn;
            if constexpr (BULK) {
                const unsigned char* rows = wbulk + (size_t(s) * PL + hh) * L::ROWSET;
                const int ln = min(max(cons.iz, cons.lo), cons.hi) - cons.lo;
                const int no = q * nyz_nodes + cons.row_o + cons.lo, nn = q * nyz_nodes + cons.row_u + cons.lo;
                const uint32_t oo = uint32_t(3 * (no & 15) * int(sizeof(TU))) & 15u;
                const uint32_t on = uint32_t(3 * (nn & 15) * int(sizeof(TU))) & 15u;
                pvo = reinterpret_cast<const TU*>(rows + oo) + 3 * ln;
                pvn = reinterpret_cast<const TU*>(rows + L::RBU + on) + 3 * ln;
                if constexpr (HAS_M) {
                    mo = rows[2 * L::RBU + L::RBE + (no & 15) + ln];
                    mn = rows[2 * L::RBU + L::RBE + L::RBM + (nn & 15) + ln];
                }
            } else {
                if constexpr (HAS_M) {
                    mo = unstage<uint8_t>(SM_(s, hh, 0), a.node_mask + (q * nyz_nodes + cons.cn_own));
                    mn = unstage<uint8_t>(SM_(s, hh, 1), a.node_mask + (q * nyz_nodes + cons.cn_nb));
                }
            }
            bo[h] = mo;
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                TC vo, vn;
                if constexpr (BULK) {
                    vo = TC(Storage<TU>::load(pvo + k));
                    vn = TC(Storage<TU>::load(pvn + k));
                } else {
                    vo = TC(Storage<TU>::cvt(unstage<TU>(SU_(s, hh, k), a.u)));
                    vn = TC(Storage<TU>::cvt(unstage<TU>(SU_(s, hh, 3 + k), a.u)));
                }
                if (h < PL) ur[h][k] = vo;
                uo[h][k] = ((mo >> k) & 1u) ? vo : TC(0);
                un[h][k] = ((mn >> k) & 1u) ? vn : TC(0);
            }
        }
        const bool elem_ok = cons.iy >= 0 && cons.iy < g.ny && cons.iz >= 0 && cons.iz < g.nz && lane < 31;
        TC ev[PL];
        #pragma unroll
        for (int h = 0; h < PL; ++h) {
            const int ex = e + h;
            TC val;
            if constexpr (BULK) {
                const unsigned char* rows = wbulk + (size_t(sc) * PL + h) * L::ROWSET;
                const int le = min(max(cons.iz, cons.elo), cons.ehi) - cons.elo;
                const int first = min(max(ex, 0), g.nx - 1) * nyz_elems + cons.row_e + cons.elo;
                const uint32_t oe = uint32_t((first & 15) * int(sizeof(TE))) & 15u;
                val = TC(Storage<TE>::load(reinterpret_cast<const TE*>(rows + 2 * L::RBU + oe) + le));
            } else {
                val = TC(Storage<TE>::cvt(unstage<TE>(SE_(sc, h), a.E + (min(max(ex, 0), g.nx - 1) * nyz_elems + cons.ce))));
            }
            ev[h] = (elem_ok && ex >= 0 && ex < g.nx) ? val : TC(0);
        }
        const P E = Cfg::pk(ev);
        const P nE = Cfg::neg(E);

        // ---- X stage (own and upper rows), Y stage
        P Y[3][2][2];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            TC lo_o[PL], hi_o[PL], lo_n[PL], hi_n[PL];
            #pragma unroll
            for (int h = 0; h < PL; ++h) {
                lo_o[h] = uo[h][k]; hi_o[h] = uo[h + 1][k];
                lo_n[h] = un[h][k]; hi_n[h] = un[h + 1][k];
            }
            const P lo = Cfg::pk(lo_o), hi = Cfg::pk(hi_o), lon = Cfg::pk(lo_n), hin = Cfg::pk(hi_n);
            const P X0 = add2(lo, hi), X1 = sub2(lo, hi);
            const P B0 = add2(lon, hin), B1 = sub2(lon, hin);
            Y[k][0][0] = add2(X0, B0); Y[k][0][1] = sub2(X0, B0);
            Y[k][1][0] = add2(X1, B1); Y[k][1][1] = sub2(X1, B1);
        }
        // ---- Z stage, modulus folded: v = E (Y(iz) +- Y(iz+1))
        P v[3][8];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            #pragma unroll
            for (int px = 0; px < 2; ++px) {
                #pragma unroll
                for (int py = 0; py < 2; ++py) {
                    const P ya = Y[k][px][py];
                    const P yb = shfl_down2(ya, 1);
                    const P ea = mul2(E, ya);
                    const int p = px + 2 * py;
                    if (p != 0) v[k][p] = fma2(E, yb, ea);
                    v[k][p + 4] = fma2(nE, yb, ea);
                }
            }
            v[k][0] = Cfg::zero();
        }
        // ---- parity-block product
        if constexpr (CUBIC) {
            const auto& K = args.K;
            {   const P bs = cmul2(K.b0, add2(add2(v[0][1], v[1][2]), v[2][4]));
                v[0][1] = cfma2(K.amb0, v[0][1], bs); v[1][2] = cfma2(K.amb0, v[1][2], bs); v[2][4] = cfma2(K.amb0, v[2][4], bs); }
            {   const P a1 = v[1][3], a2 = v[2][5];
                v[1][3] = cfma2(K.d1, a2, cmul2(K.c1, a1)); v[2][5] = cfma2(K.d1, a1, cmul2(K.c1, a2)); }
            {   const P a0 = v[0][3], a2 = v[2][6];
                v[0][3] = cfma2(K.d2, a2, cmul2(K.c2, a0)); v[2][6] = cfma2(K.d2, a0, cmul2(K.c2, a2)); }
            {   const P a0 = v[0][5], a1 = v[1][6];
                v[0][5] = cfma2(K.d4, a1, cmul2(K.c4, a0)); v[1][6] = cfma2(K.d4, a0, cmul2(K.c4, a1)); }
            {   const P t3 = cmul2(K.e3, add2(v[0][2], v[1][1])); v[0][2] = t3; v[1][1] = t3; v[2][7] = cmul2(K.f3, v[2][7]); }
            {   const P t5 = cmul2(K.e5, add2(v[0][4], v[2][1])); v[0][4] = t5; v[2][1] = t5; v[1][7] = cmul2(K.f5, v[1][7]); }
            {   const P t6 = cmul2(K.e6, add2(v[1][4], v[2][2])); v[1][4] = t6; v[2][2] = t6; v[0][7] = cmul2(K.f6, v[0][7]); }
            {   const P ks = cmul2(K.k7, add2(add2(v[0][6], v[1][5]), v[2][3]));
                v[0][6] = cfma2(K.hmk7, v[0][6], ks); v[1][5] = cfma2(K.hmk7, v[1][5], ks); v[2][3] = cfma2(K.hmk7, v[2][3], ks); }
        } else {
            #pragma unroll
            for (int gi = 0; gi < 8; ++gi) {
                const int pa[3] = {gi ^ 1, gi ^ 2, gi ^ 4};
                const P in[3] = {v[0][pa[0]], v[1][pa[1]], v[2][pa[2]]};
                #pragma unroll
                for (int r = 0; r < 3; ++r) {
                    if (pa[r] == 0) continue;
                    P sacc = Cfg::zero();
                    bool first = true;
                    #pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        if (!parity_nonzero(gi, r, cc)) continue;
                        const auto coef = args.C2.c[9 * gi + 3 * r + cc];
                        sacc = first ? cmul2(coef, in[cc]) : cfma2(coef, in[cc], sacc);
                        first = false;
                    }
                    v[r][pa[r]] = sacc;
                }
            }
        }
        // ---- inverse Z (face iz: own G0 + G1 of lane - 1), inverse Y
        P H0[3][2], H1[3][2];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            #pragma unroll
            for (int px = 0; px < 2; ++px) {
                P FY[2];
                #pragma unroll
                for (int py = 0; py < 2; ++py) {
                    const int p = px + 2 * py;
                    const P f1 = v[k][p + 4];
                    if (p == 0) {
                        FY[py] = sub2(f1, shfl_up2(f1, 1));
                    } else {
                        const P f0 = v[k][p];
                        FY[py] = add2(add2(f0, f1), shfl_up2(sub2(f0, f1), 1));
                    }
                }
                H0[k][px] = add2(FY[0], FY[1]);
                H1[k][px] = sub2(FY[0], FY[1]);
            }
        }
        // ---- exchange with the neighbouring rows: H1 goes up, the row below's H1 comes in
        const int b = cstep & 1;
        const unsigned ph = unsigned(cstep >> 1) & 1u;
        if (row < NWW - 1) {
            if (cstep >= 2 && !mbar_wait(bars + 2 * NWW + 2 * row + b, ph ^ 1u, abort_flag)) { live = false; break; }
            #pragma unroll
            for (int k = 0; k < 3; ++k) { HS_(row, b, k) = H1[k][0]; HS_(row, b, 3 + k) = H1[k][1]; }
            mbar_arrive(bars + 2 * row + b);
        }
        P lowr[6];
        if (row > 0) {
            if (!mbar_wait(bars + 2 * (row - 1) + b, ph, abort_flag)) { live = false; break; }
            #pragma unroll
            for (int k = 0; k < 6; ++k) lowr[k] = HS_(row - 1, b, k);
            mbar_arrive(bars + 2 * NWW + 2 * (row - 1) + b);
        } else {
            #pragma unroll
            for (int k = 0; k < 6; ++k) lowr[k] = Cfg::zero();
        }
        ++cstep;

        // ---- edge totals and inverse X; node plane e (+ e+1 for pairs) is complete
        TC yo[PL][3];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            const P fx0 = add2(H0[k][0], lowr[k]);
            const P fx1 = add2(H0[k][1], lowr[3 + k]);
            const P s_ = add2(fx0, fx1), d_ = sub2(fx0, fx1);
            if constexpr (PL == 1) {
                yo[0][k] = carry[k] + Cfg::get(s_, 0);
                carry[k] = Cfg::get(d_, 0);
            } else {
                yo[0][k] = carry[k] + Cfg::get(s_, 0);
                yo[1][k] = Cfg::get(d_, 0) + Cfg::get(s_, 1);
                carry[k] = Cfg::get(d_, 1);
            }
        }
        if (owner) {
            #pragma unroll
            for (int h = 0; h < PL; ++h) {
                const int ixo = e + h;
                if (ixo < cons.x0 || ixo >= cons.x1) continue;
                TY* yp = a.y + 3 * (ixo * nyz_nodes + col);
                #pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const bool fr = (bo[h] >> k) & 1u;
                    const TC xr = ur[h][k];
                    const TC ax = (MASK == MASK_NONE || fr) ? yo[h][k] : xr;
                    TC o;
                    if constexpr (EPI == EPI_RAW) {
                        o = ax;
                    } else if constexpr (EPI == EPI_APPLY_DOT) {
                        o = ax;
                        if (ixo >= a.dot_x0 && ixo < a.dot_x1) acc += double(xr) * double(ax);
                    } else if constexpr (EPI == EPI_JACOBI) {
                        o = xr + a.omega * dd[h][k] * (rr[h][k] - ax);
                    } else if constexpr (EPI == EPI_RESIDUAL) {
                        o = fr ? rr[h][k] - ax : TC(0);
                    } else {
                        o = rr[h][k] - ax;
                        if (ixo >= a.dot_x0 && ixo < a.dot_x1) acc += double(o) * double(o);
                    }
                    Storage<TY>::store(yp + k, o);
                }
            }
        }
        advance(cons);
    }
    cp_async_wait_all();
    if constexpr (BULK) {
        // after an abort, bulk copies issued for later steps may still be landing in this warp's
        // slots: wait for them (bounded, ignoring the abort) before the CTA's shared memory goes away
        for (int s = 0; s < D; ++s) {
            if (!((pending >> s) & 1u)) continue;
            const unsigned par = (pend_par >> s) & 1u;
            bool ok = false;
            for (int i = 0; i < WAVE_WAIT_LIMIT && !ok; ++i) ok = __all_sync(0xffffffffu, mbar_try_wait(sbar + s, par));
            if (!ok && lane == 0) atomicExch(&g_wave_fault, 1);
        }
    }
    if constexpr (EPI == EPI_TRUE_RES || EPI == EPI_APPLY_DOT) {
        block_sum_store<NWW * 32>(acc, a.partials + blockIdx.x);
    }
#undef SU_
#undef SE_
#undef SM_
#undef HS_
}

// Work decomposition for a grid: z tiles of 30 columns, y tiles of NW-1 rows, and the x chunk
// length that keeps the `ctas` SMs busiest: useful node planes over the SMs' capacity for as many
// rounds of items as the busiest CTA runs (each item also computes the element plane before its
// chunk; pairs of planes want an even plane count per item).
inline WaveSched wave_sched(const Grid& g, int nw, int pl, int ctas) {
    WaveSched s{};
    s.tz = (g.nz + 1 + WAVE_TZ - 1) / WAVE_TZ;
    s.ty = (g.ny + 1 + (nw - 1) - 1) / (nw - 1);
    const int cols = s.tz * s.ty;
    double best = -1.0;
    for (int k = 1; k <= 128 && k <= g.nx + 1; ++k) {
        const int cx = (g.nx + 1 + k - 1) / k;
        const int chunks = (g.nx + 1 + cx - 1) / cx;
        const int64_t items = int64_t(chunks) * cols;
        const int64_t rounds = (items + ctas - 1) / ctas;
        const int steps = (cx + 1 + pl - 1) / pl + 1;            // compute steps + the staging-only step
        const double eff = double(g.nx + 1) * cols / (double(rounds) * ctas * steps * pl);
        if (eff > best + 1e-9) {
            best = eff;
            s.cx = cx;
            s.chunks = chunks;
        }
    }
    s.items = s.chunks * cols;
    return s;
}

}  // namespace vx
