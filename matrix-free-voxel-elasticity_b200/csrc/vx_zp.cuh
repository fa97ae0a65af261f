// parity_zp: the streaming Hex8 operator with a PAIR of z node columns per thread (FP64 and FP32
// iterates).
//
// Same arithmetic as parity_stream_xp (parity form, separable X / Y / Z stages
// shared between neighbouring elements, E folded into the Z stage, cube-pattern block product,
// node-owned tiles with recomputed halo elements, no atomics, bitwise deterministic), with the work
// of a thread shaped to cut what is not arithmetic:
//
//  * Thread (row r, lane l) holds the node columns n0 = Z0 + 2 l and n1 = n0 + 1 (Z0 = 62 t - 1 for
//    z tile t) of node row iy = Y0 - 1 + r and computes the two elements A (at n0) and B (at n1) of
//    element row iy.  The pair is one V2 value throughout (packed f32x2 in FP32), so element A
//    needs no exchange and element B one value from lane l + 1: half the z shuffles of one column
//    per lane.  Lanes own n1 of lane 0 up to n0 of lane 31: 62 columns per tile (halo 64 / 62).
//  * Memory is touched in SPAN layout: a warp's row of 64 node columns is 192 consecutive words
//    (x, y, z interleaved), and lane l moves words l, l + 32, ..., l + 160, so every warp-wide load
//    or store covers consecutive addresses (one or two 128-byte lines for FP32).  The pair layout
//    the arithmetic wants (words 6 l .. 6 l + 5) is read from shared memory, where both layouts
//    meet; results go back through a per-warp shared-memory span before the coalesced stores.
//  * A CTA is NW warps, one per node row; rows 1 .. NW-1 own their nodes (halo NW / (NW-1) in y).
//    The only exchange between warps is the inverse-Y contribution a row sends to the row above,
//    through shared memory under full / empty mbarrier pairs (two buffers; lane 0 arrives once the
//    warp's writes or reads are done), so the rows advance as a
//    wavefront with no CTA-wide barrier in the march.  Every wait is bounded; a wait that runs out
//    raises the device fault flag (vx_device_status) and the CTA abandons its work.
//  * Each warp stages its own and upper row spans (and, in FP32, the element moduli) by cp.async
//    into a ring of D slots, A planes beyond the two a step reads; cp.async.wait_group plus a warp
//    barrier make a slot readable.  Node masks (and FP64 moduli) are prefetched into registers one
//    plane ahead and pass through small shared-memory spans; right-hand sides and inverse diagonals
//    are loaded (coalesced) at the top of the step that consumes them at its end.
//  * The CTA marches along x over a chunk of node planes, one element plane per step; node plane e
//    is complete after element plane e and is written (or fused into the epilogue) at once.
#pragma once

#include "vx_async.cuh"
#include "vx_pair.cuh"

#include <type_traits>

namespace vx {

// NW warps per CTA, one CTA per SM.  An SM sub-partition holds 16K registers and takes every fourth
// warp, so 12 warps allow 168 registers per thread (FP64), 16 warps 128 (FP32).  D ring slots with
// A planes in flight; E_ASYNC: element moduli staged in the ring (FP64 prefetches them into
// registers and keeps three slots, so that its 12 warps fit in shared memory).
template <typename TC> struct ZpCfg;
template <> struct ZpCfg<double> {
    static constexpr int NW = 12, D = 3, A = 1;
    static constexpr bool E_ASYNC = false;
};
template <> struct ZpCfg<float> {
    static constexpr int NW = 16, D = 4, A = 2;
    static constexpr bool E_ASYNC = true;
};
constexpr int ZP_TZ = 62;   // owned node columns per tile
constexpr int ZP_W = 192;   // words of a row span: 64 node columns x 3 components

// Shared memory of one CTA.  Per warp: the ring (D slots: own row span, upper row span, element
// modulus span with E_ASYNC; each copied in whole 16-byte chunks from the aligned chunk at or below
// its first word, so it starts `shift` words into its buffer), the output span, the modulus span
// (without E_ASYNC) and three planes of node-mask spans (own and upper row); then the exchange
// buffers (per row two buffers of six pairs), the mbarriers (full / empty per row and buffer) and
// the abort flag.
template <typename TC, typename TU, typename TE>
struct ZpLayout {
    using Cfg = ZpCfg<TC>;
    static constexpr int NW = Cfg::NW, D = Cfg::D, A = Cfg::A;
    static constexpr bool E_ASYNC = Cfg::E_ASYNC && sizeof(TE) >= 4;
    static constexpr size_t r16(size_t b) { return (b + 15) / 16 * 16; }
    static constexpr int CH = 16 / sizeof(TU);              // words per 16-byte chunk
    static constexpr int ROW_W = ZP_W + CH;                 // a row span and its alignment shift
    static constexpr int ECH = sizeof(TE) >= 4 ? 16 / int(sizeof(TE)) : 1;
    static constexpr int E_W = 64 + ECH;
    static constexpr size_t SLOT_E = E_ASYNC ? E_W * sizeof(TE) : 0;
    static constexpr size_t SLOT_B = r16(2 * ROW_W * sizeof(TU) + SLOT_E);
    static constexpr size_t AX_OFF = D * SLOT_B;
    static constexpr size_t EX_OFF = AX_OFF + r16(ZP_W * sizeof(TC));
    static constexpr size_t MK_OFF = EX_OFF + (E_ASYNC ? 0 : r16(64 * sizeof(TE)));
    static constexpr size_t WARP_B = r16(MK_OFF + 3 * 2 * 64);
    static constexpr size_t HS_B = sizeof(V2<TC>) * 2 * 6 * 32;
    static constexpr size_t BAR_OFF = NW * (WARP_B + HS_B);
    static constexpr size_t BYTES = BAR_OFF + sizeof(uint64_t) * 4 * NW + 16;
};

// two consecutive words of a span (8- or 16-byte aligned: word offsets 6 l + 2 m)
template <typename T> struct Vec2T;
template <> struct Vec2T<double> { using type = double2; };
template <> struct Vec2T<float> { using type = float2; };

template <typename TC, typename TU, typename TE, typename TY, typename TR, int EPI, int MASK, bool CUBIC>
__global__ void __launch_bounds__(ZpCfg<TC>::NW * 32, 1)
parity_zp(const __grid_constant__ OpArgs2<TC, TU, TE, TY, TR> args) {
    vx::pdl_begin();
    using L = ZpLayout<TC, TU, TE>;
    constexpr int NWW = L::NW, D = L::D, A = L::A;
    using P = V2<TC>;
    using V2U = typename Vec2T<TU>::type;
    constexpr bool HAS_M = MASK == MASK_NODE;
    constexpr bool HAS_R = EPI == EPI_JACOBI || EPI == EPI_RESIDUAL || EPI == EPI_TRUE_RES;
    constexpr bool HAS_D = EPI == EPI_JACOBI;
    constexpr bool E_ASYNC = L::E_ASYNC;
    static_assert(sizeof(TU) == 4 || sizeof(TU) == 8, "iterates staged as 4- or 8-byte words");
    static_assert(D == A + 2, "a slot is refilled the step after its plane was last read");
    const auto& a = args.a;
    const Grid g = a.g;
    const int lane = threadIdx.x & 31;
    const int row = threadIdx.x >> 5;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* wb = smem_raw + size_t(row) * L::WARP_B;
    TC* axs = reinterpret_cast<TC*>(wb + L::AX_OFF);                      // output span
    TE* exs = reinterpret_cast<TE*>(wb + L::EX_OFF);                      // modulus span (!E_ASYNC)
    uint8_t* mks = wb + L::MK_OFF;                                         // [3 planes][own, upper][64]
    P* hs = reinterpret_cast<P*>(smem_raw + NWW * L::WARP_B);              // [NWW][2][6][32]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + L::BAR_OFF);   // full[NWW][2], empty[NWW][2]
    volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 4 * NWW);
    auto own_span = [&](int s) { return reinterpret_cast<TU*>(wb + size_t(s) * L::SLOT_B); };
    auto up_span = [&](int s) { return reinterpret_cast<TU*>(wb + size_t(s) * L::SLOT_B) + L::ROW_W; };
    auto e_span = [&](int s) { return reinterpret_cast<TE*>(wb + size_t(s) * L::SLOT_B + 2 * L::ROW_W * sizeof(TU)); };
#define HS_(r, b, k) hs[(((r) * 2 + (b)) * 6 + (k)) * 32 + lane]
    if (threadIdx.x < 4 * NWW) mbar_init(bars + threadIdx.x, 1);     // one arrival: lane 0 after a warp barrier
    if (threadIdx.x == 0) *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();

    // ---- geometry (clamped offsets: always in bounds; a node outside the grid only meets
    // elements outside it, whose modulus is 0, so the finite value read there adds nothing)
    const int nyz_nodes = (g.ny + 1) * (g.nz + 1);
    const int nyz_elems = g.ny * g.nz;
    const int plane3 = 3 * nyz_nodes;
    const int iy = blockIdx.y * (NWW - 1) - 1 + row;
    const int Z0 = blockIdx.x * ZP_TZ - 1;                      // node column of span position 0
    const int n0 = Z0 + 2 * lane, n1 = n0 + 1;
    const int x0 = blockIdx.z * a.cx;
    const int x1 = min(x0 + a.cx, g.nx + 1);                    // owned node planes [x0, x1)
    const int iyc = min(max(iy, 0), g.ny), iyn = min(max(iy + 1, 0), g.ny), iye = min(max(iy, 0), g.ny - 1);
    const int rowo = 3 * iyc * (g.nz + 1), rowu = 3 * iyn * (g.nz + 1);   // word offsets in a plane
    const int rowe = iye * g.nz, rowm = iyc * (g.nz + 1), rowmu = iyn * (g.nz + 1);
    int zw[6];                                                  // span word f = lane + 32 j
    unsigned owned_w = 0u;
    #pragma unroll
    for (int j = 0; j < 6; ++j) {
        const int f = lane + 32 * j, c = Z0 + f / 3;
        zw[j] = 3 * min(max(c, 0), g.nz) + f % 3;
        if (f / 3 >= 1 && f / 3 <= ZP_TZ && c <= g.nz) owned_w |= 1u << j;
    }
    int ze[2], zm[2];                                           // span column lane + 32 j
    #pragma unroll
    for (int j = 0; j < 2; ++j) {
        ze[j] = min(max(Z0 + lane + 32 * j, 0), g.nz - 1);
        zm[j] = min(max(Z0 + lane + 32 * j, 0), g.nz);
    }
    const bool erow = iy >= 0 && iy < g.ny;
    const bool eA_ok = erow && n0 >= 0 && n0 < g.nz;
    const bool eB_ok = erow && n1 >= 0 && n1 < g.nz && lane < 31;
    const bool orow = row >= 1 && iy <= g.ny;                  // this row owns its nodes

    auto nplane = [&](int q) { return min(max(q, 0), g.nx); };
    auto eplane = [&](int q) { return min(max(q, 0), g.nx - 1); };
    // Ring group gi: node plane x0 - 1 + gi (own and upper row spans) and the element plane before
    // it.  A span is copied in 16-byte chunks from the 16-byte aligned chunk at or below its first
    // word (lane c copies chunk c), so source and shared-memory addresses agree modulo 16 bytes and
    // the span starts `shift` words into its buffer.  A chunk that reaches outside the array (only
    // around the grid's first and last node) is copied word by word, zeros standing in for the words
    // outside (they belong to columns beyond the grid, which only meet elements of modulus 0).
    const int n_words = 3 * ((g.nx + 1) * nyz_nodes);
    const int n_elems = g.nx * nyz_elems;
    auto span_start = [&](int q, int rw) { return plane3 * nplane(q) + rw + 3 * Z0; };
    auto e_start = [&](int q) { return nyz_elems * eplane(q - 1) + rowe + Z0; };
    // words from `src` up to the first 16-byte boundary of the array (its word misalignment)
    const int mis_u = int((reinterpret_cast<uintptr_t>(a.u) / sizeof(TU)) & (L::CH - 1));
    const int mis_e = int((reinterpret_cast<uintptr_t>(a.E) / sizeof(TE)) & (L::ECH - 1));
    auto stage_span = [&](auto* dst, const auto* src, int start, int mis, int total, auto chunk_words, int nchunks) {
        constexpr int CW = decltype(chunk_words)::value;
        using T = std::remove_cv_t<std::remove_pointer_t<decltype(src)>>;
        const int base = start - ((start + mis) & (CW - 1));
        #pragma unroll
        for (int c0 = 0; c0 < nchunks; c0 += 32) {
            const int c = c0 + lane;
            if (c < nchunks) {
                const int w = base + c * CW;
                T* d = dst + c * CW;
                if (w >= 0 && w + CW <= total) {
                    cp_async_cg16(d, src + w);
                } else {
                    #pragma unroll
                    for (int t = 0; t < CW; ++t) {
                        if (w + t >= 0 && w + t < total) cp_async<sizeof(T)>(d + t, src + w + t);
                        else d[t] = T(0);
                    }
                }
            }
        }
    };
    auto stage = [&](int gi) {
        const int sl_ = gi % D;
        const int q = x0 - 1 + gi;
        stage_span(own_span(sl_), a.u, span_start(q, rowo), mis_u, n_words, std::integral_constant<int, L::CH>{},
                   L::ROW_W / L::CH);
        stage_span(up_span(sl_), a.u, span_start(q, rowu), mis_u, n_words, std::integral_constant<int, L::CH>{},
                   L::ROW_W / L::CH);
        if constexpr (E_ASYNC) {
            stage_span(e_span(sl_), a.E, e_start(q), mis_e, n_elems, std::integral_constant<int, L::ECH>{},
                       L::E_W / L::ECH);
        }
    };
    // the six words of this lane's pair in a staged row span starting `shift` words in
    auto read_pair = [&](const TU* row_buf, int shift, TU w[6]) {
        const TU* p = row_buf + shift + 6 * lane;
        if ((shift & 1) == 0) {
            #pragma unroll
            for (int m = 0; m < 3; ++m) {
                const V2U t = *reinterpret_cast<const V2U*>(p + 2 * m);
                w[2 * m] = t.x;
                w[2 * m + 1] = t.y;
            }
        } else {
            #pragma unroll
            for (int k = 0; k < 6; ++k) w[k] = p[k];
        }
    };
    // node-mask bytes of plane q, span columns lane and lane + 32 of the own and upper row
    struct MaskLd { uint8_t o[2], u[2]; };
    auto mask_issue = [&](int q) {
        MaskLd m{};
        if constexpr (HAS_M) {
            const uint8_t* mb = a.node_mask + nyz_nodes * nplane(q);
            #pragma unroll
            for (int j = 0; j < 2; ++j) { m.o[j] = mb[rowm + zm[j]]; m.u[j] = mb[rowmu + zm[j]]; }
        }
        return m;
    };
    auto mask_put = [&](const MaskLd& m, int slot) {
        if constexpr (HAS_M) {
            uint8_t* d = mks + slot * 128;
            #pragma unroll
            for (int j = 0; j < 2; ++j) { d[lane + 32 * j] = m.o[j]; d[64 + lane + 32 * j] = m.u[j]; }
        }
    };
    // pair-layout mask word of a plane: byte 0 own n0, 1 own n1, 2 upper n0, 3 upper n1
    auto mask_pair = [&](int slot) -> uint32_t {
        if constexpr (HAS_M) {
            const uint8_t* d = mks + slot * 128;
            const uint32_t o = *reinterpret_cast<const uint16_t*>(d + 2 * lane);
            const uint32_t u = *reinterpret_cast<const uint16_t*>(d + 64 + 2 * lane);
            return o | (u << 16);
        } else {
            return 0x07070707u;
        }
    };
    // moduli not staged in the ring: element plane ex, span columns lane and lane + 32
    struct ELd { typename Storage<TE>::raw_t v[2]; };
    auto e_issue = [&](int ex) {
        ELd r{};
        if constexpr (!E_ASYNC) {
            const TE* eb = a.E + (nyz_elems * eplane(ex) + rowe);
            #pragma unroll
            for (int j = 0; j < 2; ++j) r.v[j] = Storage<TE>::raw(eb + ze[j]);
        }
        return r;
    };
    auto e_put = [&](const ELd& r) {
        if constexpr (!E_ASYNC) {
            #pragma unroll
            for (int j = 0; j < 2; ++j) exs[lane + 32 * j] = r.v[j];
        }
    };

    const int steps = x1 - x0 + 1;                              // element planes x0 - 1 .. x1 - 1
    #pragma unroll
    for (int gi = 0; gi <= A; ++gi) {
        if (gi <= steps) stage(gi);
        cp_async_commit();
    }
    mask_put(mask_issue(x0 - 1), 0);
    mask_put(mask_issue(x0), 1);
    MaskLd m_pf = mask_issue(x0 + 1);
    e_put(e_issue(x0 - 1));
    ELd e_pf = e_issue(x0);

    auto msk = [](uint32_t m, int byte, int k_, TU v) -> TC {
        return ((m >> (8 * byte + k_)) & 1u) ? TC(v) : TC(0);
    };
    // masked own and upper values of a node plane's pair, from its ring slot
    auto plane_pair = [&](int slot, int q, uint32_t m, P own[3], P upper[3]) {
        TU wo[6], wu[6];
        read_pair(own_span(slot), (span_start(q, rowo) + mis_u) & (L::CH - 1), wo);
        read_pair(up_span(slot), (span_start(q, rowu) + mis_u) & (L::CH - 1), wu);
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            own[k] = mk2(msk(m, 0, k, wo[k]), msk(m, 1, k, wo[3 + k]));
            upper[k] = mk2(msk(m, 2, k, wu[k]), msk(m, 3, k, wu[3 + k]));
        }
    };
    P lo[3], lon[3];                                            // node plane e, masked: own, upper row
    uint32_t m_lo;
    cp_async_wait<A>();                                          // group 0 (plane x0 - 1) has landed
    __syncwarp();
    m_lo = mask_pair(0);
    plane_pair(0, x0 - 1, m_lo, lo, lon);

    P carry[3] = {mk2(TC(0), TC(0)), mk2(TC(0), TC(0)), mk2(TC(0), TC(0))};
    double acc = 0.0;
    for (int i = 0; i < steps; ++i) {
        const int e = x0 - 1 + i;                                // element plane; node planes e, e+1
        __syncwarp();                                            // last step's reads before refills
        if (i + A + 1 <= steps) stage(i + A + 1);
        cp_async_commit();

        // ---- epilogue operands of node plane e, span layout (coalesced; consumed at the end)
        const bool out = e >= x0 && orow;
        TC rr[6], dd[6];
        if constexpr (HAS_R) {
            if (out) {
                const TR* rp = a.r + (plane3 * e + rowo);
                const TR* dp = a.invd + (plane3 * e + rowo);
                #pragma unroll
                for (int j = 0; j < 6; ++j) {
                    rr[j] = TC(Storage<TR>::load(rp + zw[j]));
                    if constexpr (HAS_D) dd[j] = TC(Storage<TR>::load(dp + zw[j]));
                }
            }
        }

        cp_async_wait<A>();                                      // groups 0 .. i + 1 have landed
        __syncwarp();                                            // ... for every lane of the warp
        const int sl = i % D, sh = (i + 1) % D;                  // slots of node planes e, e + 1
        const uint32_t m_hi = mask_pair((i + 1) % 3);

        // ---- X stage (own and upper rows), Y stage, on the node pair
        P hi[3], hin[3];
        plane_pair(sh, e + 1, m_hi, hi, hin);
        P Y[3][2][2];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            const P X0 = add2(lo[k], hi[k]), X1 = sub2(lo[k], hi[k]);
            const P B0 = add2(lon[k], hin[k]), B1 = sub2(lon[k], hin[k]);
            Y[k][0][0] = add2(X0, B0); Y[k][0][1] = sub2(X0, B0);
            Y[k][1][0] = add2(X1, B1); Y[k][1][1] = sub2(X1, B1);
        }
        // ---- element moduli of the pair (A, B)
        TC eA, eB;
        if constexpr (E_ASYNC) {
            const TE* es = e_span(sh) + ((e_start(e + 1) + mis_e) & (L::ECH - 1)) + 2 * lane;
            eA = TC(Storage<TE>::cvt(es[0]));
            eB = TC(Storage<TE>::cvt(es[1]));
        } else {
            eA = TC(Storage<TE>::cvt(exs[2 * lane]));
            eB = TC(Storage<TE>::cvt(exs[2 * lane + 1]));
        }
        const bool eplane_ok = e >= 0 && e < g.nx;
        const P E = mk2(eplane_ok && eA_ok ? eA : TC(0), eplane_ok && eB_ok ? eB : TC(0));
        const P nE = mk2(-E.lo(), -E.hi());

        // ---- Z stage on the element pair: element A spans (n0, n1), element B (n1, n0 of lane + 1)
        P v[3][8];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            #pragma unroll
            for (int px = 0; px < 2; ++px) {
                #pragma unroll
                for (int py = 0; py < 2; ++py) {
                    const P ya = Y[k][px][py];
                    const P yb = mk2(ya.hi(), __shfl_down_sync(0xffffffffu, ya.lo(), 1));
                    const P ea = mul2(E, ya);
                    const int p = px + 2 * py;
                    if (p != 0) v[k][p] = fma2(E, yb, ea);
                    v[k][p + 4] = fma2(nE, yb, ea);
                }
            }
            v[k][0] = mk2(TC(0), TC(0));
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
                    P sacc = mk2(TC(0), TC(0));
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
        // ---- inverse Z back onto the node pair: node n0 takes element A's G0 and element B of
        // lane - 1's G1, node n1 element B's G0 and element A's G1; then inverse Y
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
                        FY[py] = sub2(f1, mk2(__shfl_up_sync(0xffffffffu, f1.hi(), 1), f1.lo()));
                    } else {
                        const P f0 = v[k][p];
                        const P g1 = sub2(f0, f1);
                        FY[py] = add2(add2(f0, f1), mk2(__shfl_up_sync(0xffffffffu, g1.hi(), 1), g1.lo()));
                    }
                }
                H0[k][px] = add2(FY[0], FY[1]);
                H1[k][px] = sub2(FY[0], FY[1]);
            }
        }
        // ---- exchange with the neighbouring rows: H1 goes up, the row below's H1 comes in
        const int b = i & 1;
        const unsigned ph = unsigned(i >> 1) & 1u;
        bool ok = true;
        if (row < NWW - 1) {
            ok = i < 2 || mbar_wait(bars + 2 * NWW + 2 * row + b, ph ^ 1u, abort_flag);
            if (ok) {
                #pragma unroll
                for (int k = 0; k < 3; ++k) { HS_(row, b, k) = H1[k][0]; HS_(row, b, 3 + k) = H1[k][1]; }
                __syncwarp();
                if (lane == 0) mbar_arrive(bars + 2 * row + b);
            }
        }
        P lowr[6];
        if (ok && row > 0) {
            ok = mbar_wait(bars + 2 * (row - 1) + b, ph, abort_flag);
            if (ok) {
                #pragma unroll
                for (int k = 0; k < 6; ++k) lowr[k] = HS_(row - 1, b, k);
                __syncwarp();
                if (lane == 0) mbar_arrive(bars + 2 * NWW + 2 * (row - 1) + b);
            }
        } else {
            #pragma unroll
            for (int k = 0; k < 6; ++k) lowr[k] = mk2(TC(0), TC(0));
        }
        if (!ok) break;

        // ---- edge totals and inverse X: node plane e is complete
        P yo[3];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            const P fx0 = add2(H0[k][0], lowr[k]);
            const P fx1 = add2(H0[k][1], lowr[3 + k]);
            yo[k] = add2(carry[k], add2(fx0, fx1));
            carry[k] = sub2(fx0, fx1);
        }
        // the operator's value on the pair's words (constrained components take the raw iterate),
        // into the output span
        const int sh_lo = (span_start(e, rowo) + mis_u) & (L::CH - 1);
        if (out) {
            TU xw[6];
            if constexpr (MASK != MASK_NONE) read_pair(own_span(sl), sh_lo, xw);
            #pragma unroll
            for (int m = 0; m < 3; ++m) {
                TC v2[2];
                #pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int w = 2 * m + t, h = w / 3, k = w % 3;
                    const bool fr = (m_lo >> (8 * h + k)) & 1u;
                    const TC yv = h == 0 ? yo[k].lo() : yo[k].hi();
                    if constexpr (MASK == MASK_NONE) v2[t] = yv;
                    else v2[t] = fr ? yv : TC(xw[w]);
                }
                typename Vec2T<TC>::type t2;
                t2.x = v2[0];
                t2.y = v2[1];
                *reinterpret_cast<typename Vec2T<TC>::type*>(axs + 6 * lane + 2 * m) = t2;
            }
        }
        __syncwarp();
        // ---- span epilogue: coalesced outputs of node plane e
        if (out) {
            const TU* xo = own_span(sl) + sh_lo;
            const uint8_t* mo = mks + (i % 3) * 128;
            TY* yp = a.y + (plane3 * e + rowo);
            #pragma unroll
            for (int j = 0; j < 6; ++j) {
                if (!((owned_w >> j) & 1u)) continue;
                const int f = lane + 32 * j;
                const TC ax = axs[f];
                const TC xr = TC(xo[f]);
                TC o;
                if constexpr (EPI == EPI_RAW) {
                    o = ax;
                } else if constexpr (EPI == EPI_APPLY_DOT) {
                    o = ax;
                    if (e >= a.dot_x0 && e < a.dot_x1) acc += double(xr) * double(ax);
                } else if constexpr (EPI == EPI_JACOBI) {
                    o = xr + a.omega * dd[j] * (rr[j] - ax);
                } else if constexpr (EPI == EPI_RESIDUAL) {
                    const bool fr = MASK == MASK_NONE || ((mo[f / 3] >> (f % 3)) & 1u);
                    o = fr ? rr[j] - ax : TC(0);
                } else {
                    o = rr[j] - ax;
                    if (e >= a.dot_x0 && e < a.dot_x1) acc += double(o) * double(o);
                }
                Storage<TY>::store(yp + zw[j], o);
            }
        }
        // ---- the next planes: masks of plane e + 2 and moduli of element plane e + 1 land in their
        // spans, the next prefetches are issued
        #pragma unroll
        for (int k = 0; k < 3; ++k) { lo[k] = hi[k]; lon[k] = hin[k]; }
        m_lo = m_hi;
        mask_put(m_pf, (i + 2) % 3);
        m_pf = mask_issue(e + 3);
        e_put(e_pf);
        e_pf = e_issue(e + 2);
    }
    cp_async_wait_all();
    if constexpr (EPI == EPI_TRUE_RES || EPI == EPI_APPLY_DOT) {
        const int64_t bid = (int64_t(blockIdx.z) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        block_sum_store<NWW * 32>(acc, a.partials + bid);
    }
#undef HS_
}

// Chunking of a grid for parity_zp: z tiles of 62 columns, y tiles of NW-1 rows, and the x chunk
// that keeps `sms` SMs (one CTA each) busiest: useful node planes over the capacity of the waves the
// launch needs (a chunk of cx planes takes cx + 1 steps).  Chunking stops at 16384 CTAs (one
// partial sum each), the size of vx_true_residual_noalloc's built-in scratch.
struct ZpGrid { int tz, ty, chunks, cx; };
inline ZpGrid zp_grid(const Grid& g, int nw, int sms) {
    ZpGrid r{};
    r.tz = (g.nz + 1 + ZP_TZ - 1) / ZP_TZ;
    r.ty = (g.ny + 1 + (nw - 1) - 1) / (nw - 1);
    const int64_t cols = int64_t(r.tz) * r.ty;
    double best = -1.0;
    for (int k = 1; k <= 256 && k <= g.nx + 1; ++k) {
        const int cx = (g.nx + 1 + k - 1) / k;
        const int chunks = (g.nx + 1 + cx - 1) / cx;
        const int64_t ctas = int64_t(chunks) * cols;
        if (ctas > 16384 && k > 1) break;        // more CTAs than the no-allocation scratch holds
        const int64_t waves = (ctas + sms - 1) / sms;
        const double eff = double(g.nx + 1) * cols / (double(waves) * sms * (cx + 1));
        if (eff > best + 1e-9) {
            best = eff;
            r.cx = cx;
            r.chunks = chunks;
        }
    }
    return r;
}

}  // namespace vx
