// Matrix-free Hex8 voxel operator kernels (author layout, z fastest).
//
// parity_stream: y = K(E) u in the parity (Walsh-Hadamard) form, node-owned and atomic-free.
//   A CTA is NW warps x 32 lanes; lane <-> z node column, warp <-> y node row, and the CTA marches
//   along x (the slowest axis) over a chunk of node planes.  Thread (row, lane) holds node column
//   (iy, iz) = (y0 - 1 + row, z0 - 1 + lane) and element (ex, iy, iz).  The 2x2x2 transform is done
//   separably and SHARED between neighbouring elements:
//     X stage  (per x-edge, in registers: previous plane carried)      2 adds / component
//     Y stage  (per xy-face, neighbour row through shared memory)      4 adds
//     Z stage  (per element, neighbour lane through a shuffle, E folded in)
//     parity-block product (45 structurally non-zero coefficients, constant bank)
//     inverse Z / Y / X with the face, edge and node accumulations done the same way.
//   Rows 0 / NW-1 and lanes 0 / 31 are halo: a CTA owns nodes rows 1..NW-2, lanes 1..30, and
//   recomputes the elements of its one-node halo, so no output needs atomics and results are
//   bitwise deterministic.  Elements outside the grid get modulus 0, which removes every branch
//   on the grid boundary.
// dense_gather: the reference's node-owned dense 24x24 mapping (independent control path).
// diag / energy / coarse-grid helpers.
#include "vx_common.cuh"
#include <climits>
#include "vx_pair.cuh"

#include <algorithm>
#include <atomic>
#include <type_traits>
#include <cmath>

namespace vx {

constexpr int NW = 16;          // warps per CTA (node rows incl. 2 halo rows)
constexpr int TYR = NW - 2;     // owned node rows per CTA
constexpr int TZ = 30;          // owned node columns per CTA
constexpr int CX_MAX = 32;      // owned node planes per CTA (x chunk), upper bound

enum Epi { EPI_RAW = 0, EPI_JACOBI = 1, EPI_RESIDUAL = 2, EPI_TRUE_RES = 3, EPI_APPLY_DOT = 4 };
enum MaskKind { MASK_NONE = 0, MASK_NODE = 1, MASK_DOF = 2 };

// TR: type of the auxiliary vectors r and invd (the output type TY unless a storage mode keeps
// them narrower than the iterate)
template <typename TC, typename TU, typename TE, typename TY, typename TR = TY>
struct OpArgs {
    Grid g;
    const TU* u;              // operand (smoother: current iterate x)
    const TE* E;              // element modulus (or rho when SIMP)
    TY* y;                    // output
    const uint8_t* node_mask; // MASK_NODE: bit c set <=> DOF c free
    const double* dof_mask;   // MASK_DOF: 3 doubles per node, non-zero = free
    const TR* r;              // JACOBI / RESIDUAL / TRUE_RES right-hand side
    const TR* invd;           // JACOBI inverse diagonal
    TC omega;
    double* partials;         // TRUE_RES (|res|^2) / APPLY_DOT (p.q): one double per CTA
    int dot_x0, dot_x1;       // node planes [dot_x0, dot_x1) enter the partial sums
    double emin, de, penal;   // SIMP modulus E = emin + de * rho^penal
    int cx;                   // owned node planes per CTA (x chunk)
    bool cubic;               // host side: the blocks have the cube pattern (CubeK)
    BlocksT<TC> C;
};

template <typename T>
__device__ __forceinline__ T shfl_down1(T v) { return __shfl_down_sync(0xffffffffu, v, 1); }
template <typename T>
__device__ __forceinline__ T shfl_up1(T v) { return __shfl_up_sync(0xffffffffu, v, 1); }

template <typename TC, typename TE, bool SIMP>
__device__ __forceinline__ TC load_modulus(const TE* E, int64_t e, double emin, double de, double penal) {
    if constexpr (SIMP) {
        const double rho = double(Storage<TE>::load(E + e));
        return TC(emin + de * pow(rho, penal));
    } else {
        return TC(Storage<TE>::load(E + e));
    }
}

// Block reduce of one double per thread; thread 0 writes partials[block].
template <int NT>
__device__ __forceinline__ void block_sum_store(double v, double* out) {
    __shared__ double red[NT / 32];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double s = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) *out = s;
    }
}

template <typename TC, typename TU, typename TE, typename TY, int EPI, int MASK, bool REV, bool SIMP>
__global__ void __launch_bounds__(NW * 32, 1)
parity_stream(const __grid_constant__ OpArgs<TC, TU, TE, TY> a) {
    vx::pdl_begin();
    const int lane = threadIdx.x & 31;
    const int row = threadIdx.x >> 5;
    const Grid g = a.g;
    const int iz = blockIdx.x * TZ - 1 + lane;
    const int iy = blockIdx.y * TYR - 1 + row;
    const int x0 = blockIdx.z * a.cx;
    const int x1 = min(x0 + a.cx, g.nx + 1);               // owned node planes [x0, x1)
    const bool in_node = iy >= 0 && iy <= g.ny && iz >= 0 && iz <= g.nz;
    const bool owner = in_node && lane >= 1 && lane <= TZ && row >= 1 && row <= TYR;
    const bool elem_ok = iy >= 0 && iy < g.ny && iz >= 0 && iz < g.nz && lane < 31 && row < NW - 1;
    const int rown = row + 1 < NW ? row + 1 : row;        // clamped neighbour rows (halo rows only)
    const int rowp = row > 0 ? row - 1 : 0;

    // X-stage results for the row below, then inverse-Y contributions for the row above
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TC* xs = reinterpret_cast<TC*>(smem_raw);
    TC* hs = xs + NW * 6 * 32;
#define XS(r, k) xs[((r) * 6 + (k)) * 32 + lane]
#define HS(r, k) hs[((r) * 6 + (k)) * 32 + lane]

    const int64_t plane_nodes = int64_t(g.ny + 1) * (g.nz + 1);
    const int64_t col = int64_t(iy) * (g.nz + 1) + iz;     // node offset within a plane
    const int64_t ecol = int64_t(iy) * g.nz + iz;          // element offset within a plane
    const int64_t plane_elems = int64_t(g.ny) * g.nz;

    auto load_node = [&](int ix, TC* uu, TC* um, unsigned& bits) {
        uu[0] = uu[1] = uu[2] = TC(0);
        bits = 7u;
        if (in_node && ix >= 0 && ix <= g.nx) {
            const int64_t n = int64_t(ix) * plane_nodes + col;
            #pragma unroll
            for (int c = 0; c < 3; ++c) uu[c] = TC(Storage<TU>::load(a.u + 3 * n + (REV ? 2 - c : c)));
            if constexpr (MASK == MASK_NODE) bits = a.node_mask ? unsigned(a.node_mask[n]) : 7u;
            if constexpr (MASK == MASK_DOF) {
                bits = 0;
                #pragma unroll
                for (int c = 0; c < 3; ++c) bits |= (a.dof_mask[3 * n + (REV ? 2 - c : c)] != 0.0) << c;
            }
        }
        #pragma unroll
        for (int c = 0; c < 3; ++c) um[c] = ((bits >> c) & 1u) ? uu[c] : TC(0);
    };
    auto load_E = [&](int ex) -> TC {
        if (elem_ok && ex >= 0 && ex < g.nx)
            return load_modulus<TC, TE, SIMP>(a.E, int64_t(ex) * plane_elems + ecol, a.emin, a.de, a.penal);
        return TC(0);
    };

    TC up[3], uprev_raw[3], carry[3] = {TC(0), TC(0), TC(0)};
    unsigned bits_prev = 7u;
    // prefetched next plane
    TC un_raw[3], un[3];
    unsigned bits_n;
    load_node(x0 - 1, un_raw, un, bits_n);
    TC En = load_E(x0 - 1);
    double acc = 0.0;

    for (int ix = x0 - 1; ix <= x1; ++ix) {
        TC ucur_raw[3] = {un_raw[0], un_raw[1], un_raw[2]};
        TC ucur[3] = {un[0], un[1], un[2]};
        const unsigned bits_cur = bits_n;
        const TC Ee = En;                                   // element plane ex = ix - 1
        if (ix < x1) {                                      // prefetch plane ix + 1
            load_node(ix + 1, un_raw, un, bits_n);
            En = load_E(ix);
        }
        // epilogue operands of node plane ix - 1
        TC rr[3] = {TC(0), TC(0), TC(0)}, dd[3] = {TC(0), TC(0), TC(0)};
        const bool out_now = owner && ix - 1 >= x0;
        const int64_t nout = int64_t(ix - 1) * plane_nodes + col;
        if constexpr (EPI == EPI_JACOBI || EPI == EPI_RESIDUAL || EPI == EPI_TRUE_RES) {
            if (out_now) {
                #pragma unroll
                for (int c = 0; c < 3; ++c) rr[c] = TC(Storage<TY>::load(a.r + 3 * nout + (REV ? 2 - c : c)));
                if constexpr (EPI == EPI_JACOBI) {
                    #pragma unroll
                    for (int c = 0; c < 3; ++c) dd[c] = TC(Storage<TY>::load(a.invd + 3 * nout + (REV ? 2 - c : c)));
                }
            }
        }

        if (ix >= x0) {
            // ---- X stage: edge (ix-1 -> ix) at (iy, iz)
            TC X0[3], X1[3];
            #pragma unroll
            for (int c = 0; c < 3; ++c) { X0[c] = up[c] + ucur[c]; X1[c] = up[c] - ucur[c]; }
            #pragma unroll
            for (int c = 0; c < 3; ++c) { XS(row, c) = X0[c]; XS(row, 3 + c) = X1[c]; }
            __syncthreads();
            // ---- Y stage: face (iy -> iy+1); Y[c][px][py]
            TC Y[3][2][2];
            #pragma unroll
            for (int c = 0; c < 3; ++c) {
                const TC b0 = XS(rown, c), b1 = XS(rown, 3 + c);
                Y[c][0][0] = X0[c] + b0; Y[c][0][1] = X0[c] - b0;
                Y[c][1][0] = X1[c] + b1; Y[c][1][1] = X1[c] - b1;
            }
            // ---- Z stage with the modulus folded in: v[c][p], p = px + 2 py + 4 pz (p = 0 unused)
            TC v[3][8];
            #pragma unroll
            for (int c = 0; c < 3; ++c) {
                #pragma unroll
                for (int px = 0; px < 2; ++px) {
                    #pragma unroll
                    for (int py = 0; py < 2; ++py) {
                        const TC ya = Y[c][px][py];
                        const TC m = Ee * shfl_down1(ya);
                        const int p = px + 2 * py;
                        if (p != 0) v[c][p] = fma(Ee, ya, m);
                        v[c][p + 4] = fma(Ee, ya, -m);
                    }
                }
                v[c][0] = TC(0);
            }
            // ---- parity-block product, in place per group
            #pragma unroll
            for (int gi = 0; gi < 8; ++gi) {
                const int pa[3] = {gi ^ 1, gi ^ 2, gi ^ 4};
                TC in[3] = {v[0][pa[0]], v[1][pa[1]], v[2][pa[2]]};
                #pragma unroll
                for (int r = 0; r < 3; ++r) {
                    if (pa[r] == 0) continue;
                    TC s = TC(0);
                    bool first = true;
                    #pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        if (!parity_nonzero(gi, r, cc)) continue;
                        const TC coef = a.C.c[9 * gi + 3 * r + cc];
                        s = first ? coef * in[cc] : fma(coef, in[cc], s);
                        first = false;
                    }
                    v[r][pa[r]] = s;
                }
            }
            // ---- inverse Z: G0 -> face iz (own), G1 -> face iz+1 (lane + 1)
            TC FY[3][2][2];
            #pragma unroll
            for (int c = 0; c < 3; ++c) {
                #pragma unroll
                for (int px = 0; px < 2; ++px) {
                    #pragma unroll
                    for (int py = 0; py < 2; ++py) {
                        const int p = px + 2 * py;
                        const TC f0 = v[c][p], f1 = v[c][p + 4];
                        if (p == 0) {
                            FY[c][px][py] = f1 - shfl_up1(f1);
                        } else {
                            const TC g1 = f0 - f1;
                            FY[c][px][py] = (f0 + f1) + shfl_up1(g1);
                        }
                    }
                }
            }
            // ---- inverse Y: H0 -> edge iy (own), H1 -> edge iy+1 (row + 1)
            TC H0[3][2];
            #pragma unroll
            for (int c = 0; c < 3; ++c) {
                #pragma unroll
                for (int px = 0; px < 2; ++px) {
                    H0[c][px] = FY[c][px][0] + FY[c][px][1];
                    HS(row, 3 * px + c) = FY[c][px][0] - FY[c][px][1];
                }
            }
            __syncthreads();
            // ---- edge totals and inverse X
            TC yout[3];
            #pragma unroll
            for (int c = 0; c < 3; ++c) {
                const TC fx0 = H0[c][0] + (row > 0 ? HS(rowp, c) : TC(0));
                const TC fx1 = H0[c][1] + (row > 0 ? HS(rowp, 3 + c) : TC(0));
                yout[c] = carry[c] + (fx0 + fx1);
                carry[c] = fx0 - fx1;
            }
            // ---- epilogue for node plane ix - 1
            if (out_now) {
                TY* yo = a.y + 3 * nout;
                #pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const bool free_dof = (bits_prev >> c) & 1u;
                    TC ax;                                   // operator applied (Dirichlet form)
                    if constexpr (MASK == MASK_NONE) ax = yout[c];
                    else ax = free_dof ? yout[c] : uprev_raw[c];
                    TC o;
                    if constexpr (EPI == EPI_RAW) {
                        o = ax;
                    } else if constexpr (EPI == EPI_APPLY_DOT) {
                        o = ax;
                        if (ix - 1 >= a.dot_x0 && ix - 1 < a.dot_x1) acc += double(uprev_raw[c]) * double(ax);
                    } else if constexpr (EPI == EPI_JACOBI) {
                        o = uprev_raw[c] + a.omega * dd[c] * (rr[c] - ax);
                    } else if constexpr (EPI == EPI_RESIDUAL) {
                        o = free_dof ? rr[c] - ax : TC(0);
                    } else {  // EPI_TRUE_RES
                        o = rr[c] - ax;
                        if (ix - 1 >= a.dot_x0 && ix - 1 < a.dot_x1) acc += double(o) * double(o);
                    }
                    Storage<TY>::store(yo + (REV ? 2 - c : c), o);
                }
            }
        }
        #pragma unroll
        for (int c = 0; c < 3; ++c) { up[c] = ucur[c]; uprev_raw[c] = ucur_raw[c]; }
        bits_prev = bits_cur;
    }
    if constexpr (EPI == EPI_TRUE_RES || EPI == EPI_APPLY_DOT) {
        const int64_t bid = (int64_t(blockIdx.z) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        block_sum_store<NW * 32>(acc, a.partials + bid);
    }
#undef XS
#undef HS
}


// ============================================================================= packed coefficients
template <typename TC> struct Blocks2 { typename Coef<TC>::type c[72]; };

// Cube elements (equal edge lengths): the parity blocks have the pattern
//   g0 [a b b; b a b; b b a]      g1/g2/g4 [c d; d c] on their two non-translation components
//   g3/g5/g6 [e e; e e] (+ f on the third component)      g7 [h k k; k h k; k k h]
// so a block product needs 33 operations instead of 45, with 16 constants.
template <typename TC> struct CubeK {
    typename Coef<TC>::type amb0, b0, c1, d1, c2, d2, c4, d4, e3, f3, e5, f5, e6, f6, hmk7, k7;
};

template <typename TC, typename TU, typename TE, typename TY, typename TR = TY>
struct OpArgs2 {
    OpArgs<TC, TU, TE, TY, TR> a;
    Blocks2<TC> C2;
    CubeK<TC> K;
};
}  // namespace vx

#include "vx_zp.cuh"

namespace vx {

// true if the 72 parity coefficients have the cube pattern above (to 1e-14 of the largest); the
// constants are then taken from fixed positions
inline bool cube_pattern(const double* c) {
    double m = 0;
    for (int i = 0; i < 72; ++i) m = std::max(m, std::fabs(c[i]));
    const double tol = 1e-14 * m;
    auto B = [&](int g, int r, int col) { return c[9 * g + 3 * r + col]; };
    auto eq = [&](double x, double y) { return std::fabs(x - y) <= tol; };
    for (int g = 0; g < 8; ++g)
        for (int r = 0; r < 3; ++r)
            for (int col = 0; col < 3; ++col)
                if (!eq(B(g, r, col), B(g, col, r))) return false;
    const bool g0 = eq(B(0, 0, 0), B(0, 1, 1)) && eq(B(0, 0, 0), B(0, 2, 2)) && eq(B(0, 0, 1), B(0, 0, 2)) &&
                    eq(B(0, 0, 1), B(0, 1, 2));
    const bool g1 = eq(B(1, 1, 1), B(1, 2, 2));
    const bool g2 = eq(B(2, 0, 0), B(2, 2, 2));
    const bool g4 = eq(B(4, 0, 0), B(4, 1, 1));
    const bool g3 = eq(B(3, 0, 0), B(3, 0, 1)) && eq(B(3, 0, 0), B(3, 1, 1));
    const bool g5 = eq(B(5, 0, 0), B(5, 0, 2)) && eq(B(5, 0, 0), B(5, 2, 2));
    const bool g6 = eq(B(6, 1, 1), B(6, 1, 2)) && eq(B(6, 1, 1), B(6, 2, 2));
    const bool g7 = eq(B(7, 0, 0), B(7, 1, 1)) && eq(B(7, 0, 0), B(7, 2, 2)) && eq(B(7, 0, 1), B(7, 0, 2)) &&
                    eq(B(7, 0, 1), B(7, 1, 2));
    return g0 && g1 && g2 && g4 && g3 && g5 && g6 && g7;
}

template <typename TC>
CubeK<TC> cube_constants(const BlocksT<TC>& C) {
    auto B = [&](int g, int r, int col) { return C.c[9 * g + 3 * r + col]; };
    auto k = [](TC v) {
        if constexpr (std::is_same<TC, float>::value) return make_float2(v, v);
        else return v;
    };
    CubeK<TC> K;
    K.amb0 = k(B(0, 0, 0) - B(0, 0, 1)); K.b0 = k(B(0, 0, 1));
    K.c1 = k(B(1, 1, 1)); K.d1 = k(B(1, 1, 2));
    K.c2 = k(B(2, 0, 0)); K.d2 = k(B(2, 0, 2));
    K.c4 = k(B(4, 0, 0)); K.d4 = k(B(4, 0, 1));
    K.e3 = k(B(3, 0, 0)); K.f3 = k(B(3, 2, 2));
    K.e5 = k(B(5, 0, 0)); K.f5 = k(B(5, 1, 1));
    K.e6 = k(B(6, 1, 1)); K.f6 = k(B(6, 0, 0));
    K.hmk7 = k(B(7, 0, 0) - B(7, 0, 1)); K.k7 = k(B(7, 0, 1));
    return K;
}

// ============================================================================= parity_stream_xp
// Third-generation streaming operator: one z node column per thread, TWO consecutive element
// planes per step, processed as a pair (packed f32x2 in FP32).  Because both halves of a pair sit at
// the same (y, z) position, the y exchange (shared memory) and the z exchange (shuffles) move whole
// pairs with no repacking, and there are two block barriers per two element planes.  Each step
// consumes the loads issued one step (two planes) earlier and refills the same registers after use;
// masking and packing happen at consumption.  Loads use clamped addresses and need no validity
// test (elements outside the grid have modulus 0).  Cube elements take the 33-operation block
// product (CubeK).  Ownership, halo recomputation and determinism as in parity_stream.
// Warps per CTA and CTAs per SM: FP32 runs two 8-warp CTAs per SM (at most 128 registers), so one
// CTA computes while the other waits at a barrier; FP64 needs ~200 registers and runs one.
template <typename TC> struct XpCfg;
template <> struct XpCfg<float> { static constexpr int NW = 8, MINB = 2; };
template <> struct XpCfg<double> { static constexpr int NW = 8, MINB = 1; };

template <typename TC, typename TU, typename TE, typename TY, typename TR, int EPI, int MASK>
struct XpPlane {
    typename Storage<TU>::raw_t u1[3], u2[3];       // node planes e+1, e+2
    typename Storage<TE>::raw_t e0, e1;             // element planes e, e+1
    uint8_t m1, m2;
    typename Storage<TR>::raw_t r0[3], r1[3], d0[3], d1[3];   // epilogue operands, node planes e, e+1
};

template <typename TC, typename TU, typename TE, typename TY, typename TR, int EPI, int MASK, bool CUBIC>
__global__ void __launch_bounds__(XpCfg<TC>::NW * 32, XpCfg<TC>::MINB)
parity_stream_xp(const __grid_constant__ OpArgs2<TC, TU, TE, TY, TR> args) {
    vx::pdl_begin();
    constexpr int NWS = XpCfg<TC>::NW;
    constexpr int TYS = NWS - 2;
    using P = V2<TC>;
    using Plane = XpPlane<TC, TU, TE, TY, TR, EPI, MASK>;
    const auto& a = args.a;
    const int lane = threadIdx.x & 31;
    const int row = threadIdx.x >> 5;
    const Grid g = a.g;
    const int iz = blockIdx.x * TZ - 1 + lane;
    const int iy = blockIdx.y * TYS - 1 + row;
    const int x0 = blockIdx.z * a.cx;
    const int x1 = min(x0 + a.cx, g.nx + 1);                 // owned node planes [x0, x1)
    const bool in_node = iy >= 0 && iy <= g.ny && iz >= 0 && iz <= g.nz;
    const bool owner = in_node && lane >= 1 && lane <= TZ && row >= 1 && row <= TYS;
    const bool elem_ok = iy >= 0 && iy < g.ny && iz >= 0 && iz < g.nz && lane < 31 && row < NWS - 1;
    const bool compute = row < NWS - 1;                      // warp-uniform
    const int rown = row + 1 < NWS ? row + 1 : row;
    const int rowp = row > 0 ? row - 1 : 0;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    P* xs = reinterpret_cast<P*>(smem_raw);
    P* hs = xs + NWS * 6 * 32;
#define XSP(r, k) xs[((r) * 6 + (k)) * 32 + lane]
#define HSP(r, k) hs[((r) * 6 + (k)) * 32 + lane]

    // Clamped (always in-bounds) addresses.  A node outside the grid only touches elements outside
    // the grid, whose modulus is 0, so the finite value read at the clamped address contributes
    // nothing and needs no validity test.  Offsets fit in 32 bits (fewer than 2^31 DOFs).
    const int plane_nodes = (g.ny + 1) * (g.nz + 1);
    const int plane_elems = g.ny * g.nz;
    const int iyc = min(max(iy, 0), g.ny), izc = min(max(iz, 0), g.nz);
    const int iye = min(max(iy, 0), g.ny - 1), ize = min(max(iz, 0), g.nz - 1);
    const int cn = iyc * (g.nz + 1) + izc;
    const TU* ub = a.u + 3 * cn;
    const TE* eb = a.E + (iye * g.nz + ize);
    const uint8_t* mb = a.node_mask + cn;
    const int col = iy * (g.nz + 1) + iz;                    // unclamped: owners only

    auto nplane = [&](int ix) { return min(max(ix, 0), g.nx); };
    auto eplane = [&](int ex) { return min(max(ex, 0), g.nx - 1); };
    auto load_step = [&](int e, Plane& pl) {
        const int n1 = 3 * plane_nodes * nplane(e + 1), n2 = 3 * plane_nodes * nplane(e + 2);
        #pragma unroll
        for (int k = 0; k < 3; ++k) { pl.u1[k] = Storage<TU>::raw(ub + n1 + k); pl.u2[k] = Storage<TU>::raw(ub + n2 + k); }
        pl.e0 = Storage<TE>::raw(eb + plane_elems * eplane(e));
        pl.e1 = Storage<TE>::raw(eb + plane_elems * eplane(e + 1));
        if constexpr (MASK == MASK_NODE) {
            pl.m1 = mb[plane_nodes * nplane(e + 1)];
            pl.m2 = mb[plane_nodes * nplane(e + 2)];
        }
        if constexpr (EPI == EPI_JACOBI || EPI == EPI_RESIDUAL || EPI == EPI_TRUE_RES) {
            const TR* r0 = a.r + (3 * cn + 3 * plane_nodes * nplane(e));
            const TR* r1 = a.r + (3 * cn + 3 * plane_nodes * nplane(e + 1));
            #pragma unroll
            for (int k = 0; k < 3; ++k) { pl.r0[k] = Storage<TR>::raw(r0 + k); pl.r1[k] = Storage<TR>::raw(r1 + k); }
            if constexpr (EPI == EPI_JACOBI) {
                const TR* d0 = a.invd + (3 * cn + 3 * plane_nodes * nplane(e));
                const TR* d1 = a.invd + (3 * cn + 3 * plane_nodes * nplane(e + 1));
                #pragma unroll
                for (int k = 0; k < 3; ++k) { pl.d0[k] = Storage<TR>::raw(d0 + k); pl.d1[k] = Storage<TR>::raw(d1 + k); }
            }
        }
    };

    // node plane e (x0 - 1 initially): masked and raw operand, mask bits
    TC up[3], upraw[3];
    unsigned bits_up;
    {
        const int e = x0 - 1;
        const int n = 3 * plane_nodes * nplane(e);
        unsigned b = 7u;
        if constexpr (MASK == MASK_NODE) b = unsigned(mb[plane_nodes * nplane(e)]);
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            upraw[k] = TC(Storage<TU>::load(ub + n + k));
            up[k] = ((b >> k) & 1u) ? upraw[k] : TC(0);
        }
        bits_up = b;
    }
    TC carry[3] = {TC(0), TC(0), TC(0)};
    double acc = 0.0;
    Plane cur;
    load_step(x0 - 1, cur);

    for (int e = x0 - 1; e <= x1 - 1; e += 2) {               // element planes e, e + 1
        // ---- consume the loads of this step
        unsigned b1 = 7u, b2 = 7u;
        if constexpr (MASK == MASK_NODE) { b1 = unsigned(cur.m1); b2 = unsigned(cur.m2); }
        TC u1r[3], u1m[3], u2m[3], u2r[3];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            u1r[k] = TC(Storage<TU>::cvt(cur.u1[k]));
            u2r[k] = TC(Storage<TU>::cvt(cur.u2[k]));
            u1m[k] = ((b1 >> k) & 1u) ? u1r[k] : TC(0);
            u2m[k] = ((b2 >> k) & 1u) ? u2r[k] : TC(0);
        }
        const P E = mk2(elem_ok && e >= 0 && e < g.nx ? TC(Storage<TE>::cvt(cur.e0)) : TC(0),
                        elem_ok && e + 1 >= 0 && e + 1 < g.nx ? TC(Storage<TE>::cvt(cur.e1)) : TC(0));
        TC rr0[3], rr1[3], dd0[3], dd1[3];
        if constexpr (EPI == EPI_JACOBI || EPI == EPI_RESIDUAL || EPI == EPI_TRUE_RES) {
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                rr0[k] = TC(Storage<TR>::cvt(cur.r0[k]));
                rr1[k] = TC(Storage<TR>::cvt(cur.r1[k]));
                if constexpr (EPI == EPI_JACOBI) { dd0[k] = TC(Storage<TR>::cvt(cur.d0[k])); dd1[k] = TC(Storage<TR>::cvt(cur.d1[k])); }
            }
        }
        if (e + 2 <= x1 - 1) load_step(e + 2, cur);          // refill: next step's planes

        // ---- X stage: pair (edge e -> e+1, edge e+1 -> e+2)
        P X0[3], X1[3];
        #pragma unroll
        for (int k = 0; k < 3; ++k) {
            const P lo = mk2(up[k], u1m[k]), hi = mk2(u1m[k], u2m[k]);
            X0[k] = add2(lo, hi);
            X1[k] = sub2(lo, hi);
        }
        #pragma unroll
        for (int k = 0; k < 3; ++k) { XSP(row, k) = X0[k]; XSP(row, 3 + k) = X1[k]; }
        __syncthreads();
        P H0[3][2];
        if (compute) {
            P Y[3][2][2];
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                const P b0 = XSP(rown, k), b1_ = XSP(rown, 3 + k);
                Y[k][0][0] = add2(X0[k], b0); Y[k][0][1] = sub2(X0[k], b0);
                Y[k][1][0] = add2(X1[k], b1_); Y[k][1][1] = sub2(X1[k], b1_);
            }
            // ---- Z stage, modulus folded: v = E (Y(iz) +- Y(iz+1)) for both elements of the pair
            const P nE = mk2(-E.lo(), -E.hi());
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
                v[k][0] = mk2(TC(0), TC(0));
            }
            if constexpr (CUBIC) {
                const auto& K = args.K;
                {   // g0: x@1 y@2 z@4, (a - b) I + b 1 1^T
                    const P bs = cmul2(K.b0, add2(add2(v[0][1], v[1][2]), v[2][4]));
                    v[0][1] = cfma2(K.amb0, v[0][1], bs);
                    v[1][2] = cfma2(K.amb0, v[1][2], bs);
                    v[2][4] = cfma2(K.amb0, v[2][4], bs);
                }
                {   // g1: y@3 z@5
                    const P a1 = v[1][3], a2 = v[2][5];
                    v[1][3] = cfma2(K.d1, a2, cmul2(K.c1, a1));
                    v[2][5] = cfma2(K.d1, a1, cmul2(K.c1, a2));
                }
                {   // g2: x@3 z@6
                    const P a0 = v[0][3], a2 = v[2][6];
                    v[0][3] = cfma2(K.d2, a2, cmul2(K.c2, a0));
                    v[2][6] = cfma2(K.d2, a0, cmul2(K.c2, a2));
                }
                {   // g4: x@5 y@6
                    const P a0 = v[0][5], a1 = v[1][6];
                    v[0][5] = cfma2(K.d4, a1, cmul2(K.c4, a0));
                    v[1][6] = cfma2(K.d4, a0, cmul2(K.c4, a1));
                }
                {   // g3: x@2 y@1 (e e; e e), z@7 (f)
                    const P t = cmul2(K.e3, add2(v[0][2], v[1][1]));
                    v[0][2] = t; v[1][1] = t;
                    v[2][7] = cmul2(K.f3, v[2][7]);
                }
                {   // g5: x@4 z@1 (e e; e e), y@7 (f)
                    const P t = cmul2(K.e5, add2(v[0][4], v[2][1]));
                    v[0][4] = t; v[2][1] = t;
                    v[1][7] = cmul2(K.f5, v[1][7]);
                }
                {   // g6: y@4 z@2 (e e; e e), x@7 (f)
                    const P t = cmul2(K.e6, add2(v[1][4], v[2][2]));
                    v[1][4] = t; v[2][2] = t;
                    v[0][7] = cmul2(K.f6, v[0][7]);
                }
                {   // g7: x@6 y@5 z@3, (h - k) I + k 1 1^T
                    const P ks = cmul2(K.k7, add2(add2(v[0][6], v[1][5]), v[2][3]));
                    v[0][6] = cfma2(K.hmk7, v[0][6], ks);
                    v[1][5] = cfma2(K.hmk7, v[1][5], ks);
                    v[2][3] = cfma2(K.hmk7, v[2][3], ks);
                }
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
            // ---- inverse Z: face iz gets G0 (own) + G1 of lane - 1
            P FY[3][2][2];
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                #pragma unroll
                for (int px = 0; px < 2; ++px) {
                    #pragma unroll
                    for (int py = 0; py < 2; ++py) {
                        const int p = px + 2 * py;
                        const P f1 = v[k][p + 4];
                        if (p == 0) {
                            const P from = shfl_up2(f1, 1);
                            FY[k][px][py] = sub2(f1, from);
                        } else {
                            const P f0 = v[k][p];
                            const P g1 = sub2(f0, f1);
                            const P from = shfl_up2(g1, 1);
                            FY[k][px][py] = add2(add2(f0, f1), from);
                        }
                    }
                }
            }
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                #pragma unroll
                for (int px = 0; px < 2; ++px) {
                    H0[k][px] = add2(FY[k][px][0], FY[k][px][1]);
                    HSP(row, 3 * px + k) = sub2(FY[k][px][0], FY[k][px][1]);
                }
            }
        }
        __syncthreads();
        if (compute) {
            // ---- edge totals, inverse X: node e <- carry + sA, node e+1 <- dA + sB, carry <- dB
            TC y0[3], y1[3];
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                // row 0 (halo, never an owner) reads its own entry: its sums are not stored
                const P fx0 = add2(H0[k][0], HSP(rowp, k));
                const P fx1 = add2(H0[k][1], HSP(rowp, 3 + k));
                const P sm = add2(fx0, fx1), df = sub2(fx0, fx1);
                y0[k] = carry[k] + sm.lo();
                y1[k] = df.lo() + sm.hi();
                carry[k] = df.hi();
            }
            if (owner) {
                #pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int ixo = e + h;                       // node plane written by this half
                    if (ixo < x0 || ixo >= x1) continue;
                    const unsigned bb = h == 0 ? bits_up : b1;
                    TY* yo = a.y + 3 * (ixo * plane_nodes + col);
                    #pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const TC yv = h == 0 ? y0[k] : y1[k];
                        const TC xr = h == 0 ? upraw[k] : u1r[k];
                        const bool fr = (bb >> k) & 1u;
                        const TC ax = (MASK == MASK_NONE || fr) ? yv : xr;
                        TC o;
                        if constexpr (EPI == EPI_RAW) {
                            o = ax;
                        } else if constexpr (EPI == EPI_APPLY_DOT) {
                            o = ax;
                            if (ixo >= a.dot_x0 && ixo < a.dot_x1) acc += double(xr) * double(ax);
                        } else if constexpr (EPI == EPI_JACOBI) {
                            const TC r_ = h == 0 ? rr0[k] : rr1[k], d_ = h == 0 ? dd0[k] : dd1[k];
                            o = xr + a.omega * d_ * (r_ - ax);
                        } else if constexpr (EPI == EPI_RESIDUAL) {
                            const TC r_ = h == 0 ? rr0[k] : rr1[k];
                            o = fr ? r_ - ax : TC(0);
                        } else {
                            const TC r_ = h == 0 ? rr0[k] : rr1[k];
                            o = r_ - ax;
                            if (ixo >= a.dot_x0 && ixo < a.dot_x1) acc += double(o) * double(o);
                        }
                        Storage<TY>::store(yo + k, o);
                    }
                }
            }
        }
        // ---- the step's last node plane (e + 2) becomes the next step's first
        #pragma unroll
        for (int k = 0; k < 3; ++k) { up[k] = u2m[k]; upraw[k] = u2r[k]; }
        bits_up = b2;
    }
    if constexpr (EPI == EPI_TRUE_RES || EPI == EPI_APPLY_DOT) {
        const int64_t bid = (int64_t(blockIdx.z) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        block_sum_store<NWS * 32>(acc, a.partials + bid);
    }
#undef XSP
#undef HSP
}

// CTA tiling of the streaming operators: parity_stream_xp (author layout, node or no mask) tiles
// (y, z) node columns as (NW-2) x 30 with NW = 8 warps; parity_stream
// (natural-layout / SIMP / DOF-mask product) as 14 x 30.  x-chunk: the longest chunk (least halo recomputation) with >= 4 CTAs per SM.
struct Tiling { int tz, ty; };
inline Tiling tiling(int prec, bool v2) {
    if (!v2) return {TZ, TYR};
    return {TZ, (prec == VX_F64 ? XpCfg<double>::NW : XpCfg<float>::NW) - 2};
}

inline int stream_cx(const Grid& g, Tiling t) {
    const int64_t yz = int64_t((g.nz + 1 + t.tz - 1) / t.tz) * ((g.ny + 1 + t.ty - 1) / t.ty);
    int cx = CX_MAX;
    while (cx > 4 && yz * ((g.nx + 1 + cx - 1) / cx) < 4 * 148) cx /= 2;
    // at most 16384 CTAs (one partial sum each, the no-allocation residual's built-in scratch)
    while (cx < g.nx + 1 && yz * ((g.nx + 1 + cx - 1) / cx) > 16384) cx *= 2;
    return cx;
}

inline dim3 stream_grid(const Grid& g, Tiling t, int cx) {
    return dim3((g.nz + 1 + t.tz - 1) / t.tz, (g.ny + 1 + t.ty - 1) / t.ty, (g.nx + 1 + cx - 1) / cx);
}

// SM count of the current device (cached per device).
inline int sm_count() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
    if (dev >= 64) {
        int n = 148;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n;
    }
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n <= 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

template <typename TC>
inline ZpGrid zp_grid_for(const Grid& g) {
    return zp_grid(g, ZpCfg<TC>::NW, sm_count());
}

// Streaming kernel for FP64 / FP32 iterates (process-wide; the other storage forms always run
// parity_stream_xp): VX_KERNEL_XP (element-plane pairs, the default) or VX_KERNEL_ZP (node-column
// pairs).
static std::atomic<int> g_stream_kernel{VX_KERNEL_XP};

// CTAs (= partial sums) of a fused reducing launch of precision `prec` on grid g
int64_t stream_ctas(const Grid& g, int prec) {
    const int kind = g_stream_kernel.load(std::memory_order_relaxed);
    if (prec == VX_F32 || prec == VX_F64) {
        if (kind == VX_KERNEL_ZP) {
            const ZpGrid z = prec == VX_F32 ? zp_grid_for<float>(g) : zp_grid_for<double>(g);
            return int64_t(z.tz) * z.ty * z.chunks;
        }
    }
    const Tiling t = tiling(prec, true);
    dim3 d = stream_grid(g, t, stream_cx(g, t));
    return int64_t(d.x) * d.y * d.z;
}

template <typename TC, typename TU, typename TE, typename TY, typename TR, int EPI, int MASK>
OpArgs2<TC, TU, TE, TY, TR> packed_args(const OpArgs<TC, TU, TE, TY, TR>& a) {
    OpArgs2<TC, TU, TE, TY, TR> a2;
    a2.a = a;
    for (int i = 0; i < 72; ++i) {
        if constexpr (std::is_same<TC, float>::value) a2.C2.c[i] = make_float2(a.C.c[i], a.C.c[i]);
        else a2.C2.c[i] = a.C.c[i];
    }
    if (a.cubic) a2.K = cube_constants<TC>(a.C);
    return a2;
}

template <typename TC, typename TU, typename TE, typename TY, int EPI, int MASK, bool REV, bool SIMP, typename TR = TY>
int launch_stream(const OpArgs<TC, TU, TE, TY, TR>& a_in, cudaStream_t s, const char* what) {
    constexpr bool v2 = !REV && !SIMP && MASK != MASK_DOF;
    static_assert(v2 || std::is_same<TR, TY>::value, "parity_stream takes r and invd of the output type");
    // iterates in FP64 / FP32: either streaming kernel (parity_zp stages 4- or 8-byte words)
    constexpr bool zp_ok = v2 && (std::is_same<TU, double>::value || std::is_same<TU, float>::value);
    OpArgs<TC, TU, TE, TY, TR> a = a_in;
    const bool cubic = a.cubic;
    static std::atomic<uint64_t> configured[2];            // per kernel of this instantiation: devices opted in
    const int kind = zp_ok ? g_stream_kernel.load(std::memory_order_relaxed) : VX_KERNEL_XP;
    if constexpr (zp_ok) {
        if (kind == VX_KERNEL_ZP) {
            const ZpGrid z = zp_grid_for<TC>(a.g);
            a.cx = z.cx;
            const OpArgs2<TC, TU, TE, TY, TR> a2 = packed_args<TC, TU, TE, TY, TR, EPI, MASK>(a);
            using Lz = ZpLayout<TC, TU, TE>;
            static std::atomic<uint64_t> cfg_zp[2];
            auto kz = cubic ? parity_zp<TC, TU, TE, TY, TR, EPI, MASK, true> : parity_zp<TC, TU, TE, TY, TR, EPI, MASK, false>;
            int st = smem_opt_in(cfg_zp[cubic ? 1 : 0], (const void*)kz, Lz::BYTES, what);
            if (st) return st;
            vx::launch(kz, dim3(z.tz, z.ty, z.chunks), unsigned(Lz::NW * 32), Lz::BYTES, s, a2);
            VX_CHECK_LAUNCH(what);
            return VX_OK;
        }
    }
    {
        const Tiling t = tiling(std::is_same<TC, double>::value ? VX_F64 : VX_F32, v2);
        a.cx = stream_cx(a.g, t);
        size_t smem, threads;
        if constexpr (v2) {
            threads = XpCfg<TC>::NW * 32;
            smem = size_t(2) * XpCfg<TC>::NW * 6 * 32 * sizeof(V2<TC>);
        } else {
            threads = NW * 32;
            smem = size_t(2) * NW * 6 * 32 * sizeof(TC);
        }
        if constexpr (v2) {
            const OpArgs2<TC, TU, TE, TY, TR> a2 = packed_args<TC, TU, TE, TY, TR, EPI, MASK>(a);
            if (cubic) {
                auto k = parity_stream_xp<TC, TU, TE, TY, TR, EPI, MASK, true>;
                int st = smem_opt_in(configured[1], (const void*)k, smem, what);
                if (st) return st;
                vx::launch(k, stream_grid(a.g, t, a.cx), unsigned(threads), smem, s, a2);
            } else {
                auto k = parity_stream_xp<TC, TU, TE, TY, TR, EPI, MASK, false>;
                int st = smem_opt_in(configured[0], (const void*)k, smem, what);
                if (st) return st;
                vx::launch(k, stream_grid(a.g, t, a.cx), unsigned(threads), smem, s, a2);
            }
        } else {
            auto k = parity_stream<TC, TU, TE, TY, EPI, MASK, REV, SIMP>;
            int st = smem_opt_in(configured[0], (const void*)k, smem, what);
            if (st) return st;
            vx::launch(k, stream_grid(a.g, t, a.cx), unsigned(threads), smem, s, a);
        }
        VX_CHECK_LAUNCH(what);
        return VX_OK;
    }
}

template <typename TC>
BlocksT<TC> convert_blocks(const double* blocks) {
    BlocksT<TC> b;
    for (int i = 0; i < 72; ++i) b.c[i] = TC(blocks[i]);
    return b;
}

// ------------------------------------------------------------------------- dense control path
template <typename T>
__global__ void dense_gather(Grid g, const T* __restrict__ ke, const T* __restrict__ E,
                             const T* __restrict__ u, T* __restrict__ y) {
    vx::pdl_begin();
    __shared__ T K[576];
    for (int i = threadIdx.x; i < 576; i += blockDim.x) K[i] = ke[i];
    __syncthreads();
    const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= g.nodes()) return;
    const int iz = int(n % (g.nz + 1));
    const int iy = int((n / (g.nz + 1)) % (g.ny + 1));
    const int ix = int(n / (int64_t(g.nz + 1) * (g.ny + 1)));
    // native node index of binary offset (bx, by, bz): 0,1,3,2,4,5,7,6
    constexpr int nat[8] = {0, 1, 3, 2, 4, 5, 7, 6};
    T acc[3] = {T(0), T(0), T(0)};
    for (int bx = 0; bx < 2; ++bx) for (int by = 0; by < 2; ++by) for (int bz = 0; bz < 2; ++bz) {
        const int ex = ix - 1 + bx, ey = iy - 1 + by, ez = iz - 1 + bz;
        if (ex < 0 || ex >= g.nx || ey < 0 || ey >= g.ny || ez < 0 || ez >= g.nz) continue;
        const T Ee = E[g.elem(ex, ey, ez)];
        const int li = nat[(1 - bx) + 2 * (1 - by) + 4 * (1 - bz)];
        for (int b = 0; b < 8; ++b) {
            const int m = nat[b];
            const int64_t nb = g.node(ex + (b & 1), ey + ((b >> 1) & 1), ez + ((b >> 2) & 1));
            const T u0 = u[3 * nb], u1 = u[3 * nb + 1], u2 = u[3 * nb + 2];
            for (int c = 0; c < 3; ++c) {
                const T* kr = K + (3 * li + c) * 24 + 3 * m;
                acc[c] += Ee * (kr[0] * u0 + kr[1] * u1 + kr[2] * u2);
            }
        }
    }
    for (int c = 0; c < 3; ++c) y[3 * n + c] = acc[c];
}

// ------------------------------------------------------------------------- diagonal
// mode 0: diag K; mode 1: 1/diag on free DOFs, 1 on fixed; mode 2: diag on free DOFs, 1 on fixed.
template <typename T, bool REV, int MASK, bool SIMP>
__global__ void diag_kernel(Grid g, BlocksT<T> kd /* c[0..23]: diagonal of ke */, const T* __restrict__ E,
                            const uint8_t* __restrict__ node_mask, const double* __restrict__ dof_mask,
                            double emin, double de, double penal, int mode, T* __restrict__ d) {
    vx::pdl_begin();
    const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= g.nodes()) return;
    const int iz = int(n % (g.nz + 1));
    const int iy = int((n / (g.nz + 1)) % (g.ny + 1));
    const int ix = int(n / (int64_t(g.nz + 1) * (g.ny + 1)));
    constexpr int nat[8] = {0, 1, 3, 2, 4, 5, 7, 6};   // native index of binary offset code
    T acc[3] = {T(0), T(0), T(0)};
    for (int bx = 0; bx < 2; ++bx) for (int by = 0; by < 2; ++by) for (int bz = 0; bz < 2; ++bz) {
        const int ex = ix - 1 + bx, ey = iy - 1 + by, ez = iz - 1 + bz;
        if (ex < 0 || ex >= g.nx || ey < 0 || ey >= g.ny || ez < 0 || ez >= g.nz) continue;
        const T Ee = load_modulus<T, T, SIMP>(E, g.elem(ex, ey, ez), emin, de, penal);
        const int li = nat[(1 - bx) + 2 * (1 - by) + 4 * (1 - bz)];
        for (int c = 0; c < 3; ++c) acc[c] += Ee * kd.c[3 * li + c];
    }
    unsigned bits = 7u;
    if constexpr (MASK == MASK_NODE) bits = node_mask ? unsigned(node_mask[n]) : 7u;
    if constexpr (MASK == MASK_DOF) {
        bits = 0;
        for (int c = 0; c < 3; ++c) bits |= (dof_mask[3 * n + (REV ? 2 - c : c)] != 0.0) << c;
    }
    for (int c = 0; c < 3; ++c) {
        const bool fr = (bits >> c) & 1u;
        T v = acc[c];
        if (mode == 1) v = fr ? T(1) / v : T(1);
        else if (mode == 2) v = fr ? v : T(1);
        d[3 * n + (REV ? 2 - c : c)] = v;
    }
}

// ------------------------------------------------------------------------- element energy
struct Ke { double k[576]; };

template <bool REV, int MASK>
__global__ void energy_kernel(Grid g, const __grid_constant__ Ke ke, const double* __restrict__ u,
                              const double* __restrict__ dof_mask, double* __restrict__ ce,
                              const double* __restrict__ rho, double emin, double de, double penal,
                              double* __restrict__ dc) {
    vx::pdl_begin();
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= g.elems()) return;
    const int ez = int(e % g.nz);
    const int ey = int((e / g.nz) % g.ny);
    const int ex = int(e / (int64_t(g.nz) * g.ny));
    constexpr int ox[8] = {0, 1, 1, 0, 0, 1, 1, 0}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1},
                  oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    double ue[24];
    #pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int64_t n = g.node(ex + ox[i], ey + oy[i], ez + oz[i]);
        #pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t k = 3 * n + (REV ? 2 - c : c);
            double val = u[k];
            if constexpr (MASK == MASK_DOF) val = dof_mask[k] != 0.0 ? val : 0.0;
            ue[3 * i + c] = val;
        }
    }
    double s = 0.0;
    #pragma unroll 4
    for (int r = 0; r < 24; ++r) {
        double t = 0.0;
        #pragma unroll
        for (int c = 0; c < 24; ++c) t = fma(ke.k[24 * r + c], ue[c], t);
        s = fma(ue[r], t, s);
    }
    ce[e] = s;
    if (dc) {
        const double rr = rho[e];
        dc[e] = -penal * pow(rr, penal - 1.0) * de * s;
    }
}

}  // namespace vx

using namespace vx;

// =========================================================================== C ABI
extern "C" int vx_matvec(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                         const void* u, void* y, const uint8_t* node_mask, cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(blocks && E && u && y, VX_ERR_NULL_POINTER, "vx_matvec: NULL pointer");
    int rc = VX_OK;
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using X = typename decltype(t)::X;                 // operand u: an iterate
        using M = typename decltype(t)::M;
        using TC = arith_t<X>;                              // y in the arithmetic type
        OpArgs<TC, X, M, TC> a{};
        a.g = Grid{nx, ny, nz}; a.u = (const X*)u; a.E = (const M*)E; a.y = (TC*)y; a.node_mask = node_mask;
        a.C = convert_blocks<TC>(blocks);
        a.cubic = cube_pattern(blocks);
        rc = node_mask ? launch_stream<TC, X, M, TC, EPI_RAW, MASK_NODE, false, false>(a, stream, "vx_matvec")
                       : launch_stream<TC, X, M, TC, EPI_RAW, MASK_NONE, false, false>(a, stream, "vx_matvec");
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "vx_matvec: unknown precision %d", prec);
    return rc;
}

extern "C" int vx_modal8(const double* blocks, const double* E, const double* u, double* y,
                         int nx, int ny, int nz, cudaStream_t stream) {
    return vx_matvec(VX_F64, nx, ny, nz, blocks, E, u, y, nullptr, stream);
}

extern "C" int vx_matvec_dense(int prec, int nx, int ny, int nz, const double* ke, const void* E,
                               const void* u, void* y, cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(ke && E && u && y, VX_ERR_NULL_POINTER, "vx_matvec_dense: NULL pointer");
    Grid g{nx, ny, nz};
    const int64_t n = g.nodes();
    const unsigned blocksz = 128;
    const unsigned grid = unsigned((n + blocksz - 1) / blocksz);
    if (prec == VX_F64) {
        vx::launch(dense_gather<double>, grid, blocksz, 0, stream, g, ke, (const double*)E, (const double*)u, (double*)y);
    } else if (prec == VX_F32) {
        // ke is device FP32 here
        vx::launch(dense_gather<float>, grid, blocksz, 0, stream, g, (const float*)ke, (const float*)E, (const float*)u, (float*)y);
    } else {
        set_error("vx_matvec_dense: unsupported precision %d", prec);
        return VX_ERR_INVALID_ARGUMENT;
    }
    VX_CHECK_LAUNCH("vx_matvec_dense");
    return VX_OK;
}

extern "C" int vx_diagonal(int prec, int nx, int ny, int nz, const double* ke, const void* E,
                           const uint8_t* node_mask, int inverse, void* d, cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(ke && E && d, VX_ERR_NULL_POINTER, "vx_diagonal: NULL pointer");
    Grid g{nx, ny, nz};
    const int64_t n = g.nodes();
    const unsigned grid = unsigned((n + 255) / 256);
    if (prec == VX_F64) {
        BlocksT<double> kd{};
        for (int i = 0; i < 24; ++i) kd.c[i] = ke[25 * i];
        vx::launch(diag_kernel<double, false, MASK_NODE, false>, grid, 256, 0, stream, 
            g, kd, (const double*)E, node_mask, nullptr, 0, 0, 0, inverse ? 1 : 0, (double*)d);
    } else if (prec == VX_F32) {
        BlocksT<float> kd{};
        for (int i = 0; i < 24; ++i) kd.c[i] = float(ke[25 * i]);
        vx::launch(diag_kernel<float, false, MASK_NODE, false>, grid, 256, 0, stream, 
            g, kd, (const float*)E, node_mask, nullptr, 0, 0, 0, inverse ? 1 : 0, (float*)d);
    } else {
        set_error("vx_diagonal: unsupported precision %d", prec);
        return VX_ERR_INVALID_ARGUMENT;
    }
    VX_CHECK_LAUNCH("vx_diagonal");
    return VX_OK;
}

extern "C" int vx_element_energy(int nx, int ny, int nz, const double* ke, const double* u, double* ce,
                                 const double* rho, double emin, double emax, double penal, double* dc,
                                 cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(ke && u && ce, VX_ERR_NULL_POINTER, "vx_element_energy: NULL pointer");
    VX_CHECK_ARG(!dc || rho, VX_ERR_NULL_POINTER, "vx_element_energy: dc requested without rho");
    Grid g{nx, ny, nz};
    Ke k;
    for (int i = 0; i < 576; ++i) k.k[i] = ke[i];
    const int64_t n = g.elems();
    vx::launch(energy_kernel<false, MASK_NONE>, unsigned((n + 127) / 128), 128, 0, stream, 
        g, k, u, nullptr, ce, rho, emin, emax - emin, penal, dc);
    VX_CHECK_LAUNCH("vx_element_energy");
    return VX_OK;
}

// Natural layout = author layout of the grid (nz, ny, nx) with the x<->z axes swapped; the
// kernels read component c from storage slot 2-c (REV) and use the axis-permuted element matrix.
namespace {
void permute_ke_xz(const double* ke, double* kp) {
    // native offsets; kernel-native node i' has offsets (z_i, y_i, x_i) of physical node pi(i')
    const int ox[8] = {0, 1, 1, 0, 0, 1, 1, 0}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1}, oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    int pi[8];
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j)
            if (ox[j] == oz[i] && oy[j] == oy[i] && oz[j] == ox[i]) pi[i] = j;
    for (int i = 0; i < 8; ++i) for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 8; ++j) for (int b = 0; b < 3; ++b)
            kp[(3 * i + a) * 24 + 3 * j + b] = ke[(3 * pi[i] + (2 - a)) * 24 + 3 * pi[j] + (2 - b)];
}
}  // namespace

extern "C" int vx_product(int nx, int ny, int nz, const double* rho, const double* u, const double* ke,
                          const double* mask, double emin, double emax, double penal,
                          double* y, double* ce, double* diag, cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(rho && u && ke && mask, VX_ERR_NULL_POINTER, "vx_product: NULL pointer");
    // kernel grid: (nz, ny, nx) author layout == natural layout of (nx, ny, nz)
    Grid g{nz, ny, nx};
    double kp[576], blocks[72], disc = 0.0;
    permute_ke_xz(ke, kp);
    if (y) {
        st = vx_parity_blocks(kp, blocks, &disc);
        if (st) return st;
        OpArgs<double, double, double, double> a{};
        a.g = g; a.u = u; a.E = rho; a.y = y; a.dof_mask = mask;
        a.emin = emin; a.de = emax - emin; a.penal = penal;
        a.C = convert_blocks<double>(blocks);
        st = launch_stream<double, double, double, double, EPI_RAW, MASK_DOF, true, true>(a, stream, "vx_product");
        if (st) return st;
    }
    if (ce) {
        Ke k;
        for (int i = 0; i < 576; ++i) k.k[i] = kp[i];
        const int64_t n = g.elems();
        vx::launch(energy_kernel<true, MASK_DOF>, unsigned((n + 127) / 128), 128, 0, stream, 
            g, k, u, mask, ce, nullptr, 0.0, 0.0, 0.0, nullptr);
        VX_CHECK_LAUNCH("vx_product(ce)");
    }
    if (diag) {
        BlocksT<double> kd{};
        for (int i = 0; i < 24; ++i) kd.c[i] = kp[25 * i];
        vx::launch(diag_kernel<double, true, MASK_DOF, true>, unsigned((g.nodes() + 255) / 256), 256, 0, stream, 
            g, kd, rho, nullptr, mask, emin, emax - emin, penal, 2, diag);
        VX_CHECK_LAUNCH("vx_product(diag)");
    }
    return VX_OK;
}

// Fused smoother / residual / outer-CG operator forms (author layout, node mask optional).
namespace {
// The fused smoother / residual / reducing forms.  Operand x and the Jacobi output are iterates;
// the right-hand side, the inverse diagonal and the residual output are auxiliary vectors; the
// reducing forms (apply_dot, true_residual) exist for VX_F64 and VX_F32.
template <int EPI>
int fused_dispatch(const char* what, int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                   const uint8_t* node_mask, const void* x, const void* r, const void* invd, double omega,
                   void* out, double* partials, cudaStream_t stream, int dot_x0 = 0, int dot_x1 = INT_MAX) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(blocks && E && x && out, VX_ERR_NULL_POINTER, "%s: NULL pointer", what);
    VX_CHECK_ARG(x != out, VX_ERR_INVALID_ARGUMENT, "%s: output may not alias the operand", what);
    constexpr bool reducing = EPI == EPI_TRUE_RES || EPI == EPI_APPLY_DOT;
    VX_CHECK_ARG(!reducing || prec == VX_F64 || prec == VX_F32, VX_ERR_INVALID_ARGUMENT,
                 "%s: unsupported precision %d", what, prec);
    int rc = VX_OK;
    const bool ok = dispatch_prec(prec, [&](auto t) {
        using X = typename decltype(t)::X;
        using R = typename decltype(t)::R;
        using M = typename decltype(t)::M;
        using TC = arith_t<X>;
        using TY = std::conditional_t<EPI == EPI_RESIDUAL, R, X>;
        if constexpr (reducing && !std::is_same<X, R>::value) {
            rc = VX_ERR_INVALID_ARGUMENT;                   // excluded above
        } else if constexpr (reducing && std::is_same<X, __nv_bfloat16>::value) {
            rc = VX_ERR_INVALID_ARGUMENT;
        } else {
            OpArgs<TC, X, M, TY, R> a{};
            a.g = Grid{nx, ny, nz};
            a.u = (const X*)x; a.E = (const M*)E; a.y = (TY*)out; a.node_mask = node_mask;
            a.r = (const R*)r; a.invd = (const R*)invd; a.omega = TC(omega); a.partials = partials;
            a.dot_x0 = dot_x0; a.dot_x1 = dot_x1;
            a.C = convert_blocks<TC>(blocks);
            a.cubic = cube_pattern(blocks);
            rc = node_mask ? launch_stream<TC, X, M, TY, EPI, MASK_NODE, false, false, R>(a, stream, what)
                           : launch_stream<TC, X, M, TY, EPI, MASK_NONE, false, false, R>(a, stream, what);
        }
    });
    VX_CHECK_ARG(ok, VX_ERR_INVALID_ARGUMENT, "%s: unsupported precision %d", what, prec);
    return rc;
}
}  // namespace

extern "C" int vx_jacobi_sweep(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                               const uint8_t* node_mask, const void* x, const void* r, const void* inv_diag,
                               double omega, void* x_out, cudaStream_t stream) {
    VX_CHECK_ARG(r && inv_diag, VX_ERR_NULL_POINTER, "vx_jacobi_sweep: NULL r / inv_diag");
    return fused_dispatch<EPI_JACOBI>("vx_jacobi_sweep", prec, nx, ny, nz, blocks, E, node_mask, x, r,
                                      inv_diag, omega, x_out, nullptr, stream);
}

extern "C" int vx_residual(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                           const uint8_t* node_mask, const void* x, const void* r, void* res,
                           cudaStream_t stream) {
    VX_CHECK_ARG(r, VX_ERR_NULL_POINTER, "vx_residual: NULL r");
    return fused_dispatch<EPI_RESIDUAL>("vx_residual", prec, nx, ny, nz, blocks, E, node_mask, x, r,
                                        nullptr, 0.0, res, nullptr, stream);
}

extern "C" int64_t vx_operator_partials(int prec, int nx, int ny, int nz) {
    if (check_grid(nx, ny, nz) || (prec != VX_F64 && prec != VX_F32)) return -1;
    return stream_ctas(Grid{nx, ny, nz}, prec);
}

extern "C" int vx_apply_dot(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                            const uint8_t* node_mask, const void* p, void* q, double* partials,
                            cudaStream_t stream) {
    VX_CHECK_ARG(partials, VX_ERR_NULL_POINTER, "vx_apply_dot: NULL partials");
    return fused_dispatch<EPI_APPLY_DOT>("vx_apply_dot", prec, nx, ny, nz, blocks, E, node_mask, p, nullptr,
                                         nullptr, 0.0, q, partials, stream);
}

extern "C" int vx_true_residual(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                                const uint8_t* node_mask, const void* x, const void* b, void* res,
                                double* partials, cudaStream_t stream) {
    VX_CHECK_ARG(b && partials, VX_ERR_NULL_POINTER, "vx_true_residual: NULL b / partials");
    return fused_dispatch<EPI_TRUE_RES>("vx_true_residual", prec, nx, ny, nz, blocks, E, node_mask, x, b,
                                        nullptr, 0.0, res, partials, stream);
}

// The reducing forms with the sums restricted to node planes x_lo <= ix < x_hi (the output is
// written everywhere): an x-slab leaves its shared planes out and adds them once they are final.
extern "C" int vx_apply_dot_planes(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                                   const uint8_t* node_mask, const void* p, void* q, double* partials, int x_lo,
                                   int x_hi, cudaStream_t stream) {
    VX_CHECK_ARG(partials, VX_ERR_NULL_POINTER, "vx_apply_dot_planes: NULL partials");
    VX_CHECK_ARG(0 <= x_lo && x_lo <= x_hi && x_hi <= nx + 1, VX_ERR_INVALID_ARGUMENT,
                 "vx_apply_dot_planes: bad plane range [%d, %d)", x_lo, x_hi);
    return fused_dispatch<EPI_APPLY_DOT>("vx_apply_dot_planes", prec, nx, ny, nz, blocks, E, node_mask, p, nullptr,
                                         nullptr, 0.0, q, partials, stream, x_lo, x_hi);
}

extern "C" int vx_true_residual_planes(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                                       const uint8_t* node_mask, const void* x, const void* b, void* res,
                                       double* partials, int x_lo, int x_hi, cudaStream_t stream) {
    VX_CHECK_ARG(b && partials, VX_ERR_NULL_POINTER, "vx_true_residual_planes: NULL b / partials");
    VX_CHECK_ARG(0 <= x_lo && x_lo <= x_hi && x_hi <= nx + 1, VX_ERR_INVALID_ARGUMENT,
                 "vx_true_residual_planes: bad plane range [%d, %d)", x_lo, x_hi);
    return fused_dispatch<EPI_TRUE_RES>("vx_true_residual_planes", prec, nx, ny, nz, blocks, E, node_mask, x, b,
                                        nullptr, 0.0, res, partials, stream, x_lo, x_hi);
}

// ----------------------------------------------------------------------------- allocation-free form
// Callers that cannot allocate device memory -- a serving loop that must not call cudaMalloc while
// requests are in flight, a plugin living inside another framework's memory arena, a process under
// a hard device-memory cap -- get one entry point that needs no scratch buffer from them:
// vx_true_residual_noalloc keeps the per-CTA partial sums of |b - A x|^2 in a fixed device array
// compiled into this library (NOALLOC_MAX_CTAS doubles = 128 KiB, resident on every device that
// loads the library until the process exits).
#include <mutex>

namespace vx {
constexpr int64_t NOALLOC_MAX_CTAS = 16384;
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_CTAS];
constexpr int NOALLOC_MAX_DEVICES = 64;
static double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
static std::mutex g_noalloc_mutex;

// Device address of g_noalloc_partials on the current device, looked up once per device.  In host
// code the array's name is only a host-side stand-in, so kernels must be given this address.
static int noalloc_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error("vx_true_residual_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        set_error("vx_true_residual_noalloc: device %d is beyond the %d supported", dev, NOALLOC_MAX_DEVICES);
        return VX_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || p == nullptr) {
            set_error("vx_true_residual_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return VX_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return VX_OK;
}
}  // namespace vx

extern "C" int vx_true_residual_noalloc(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                                        const uint8_t* node_mask, const void* x, const void* b, void* res,
                                        double* norm2, cudaStream_t stream) {
    int st = check_grid(nx, ny, nz);
    if (st) return st;
    VX_CHECK_ARG(blocks && E && x && b && res && norm2, VX_ERR_NULL_POINTER,
                 "vx_true_residual_noalloc: NULL pointer");
    VX_CHECK_ARG(prec == VX_F64 || prec == VX_F32, VX_ERR_INVALID_ARGUMENT,
                 "vx_true_residual_noalloc: unsupported precision %d", prec);
    const int64_t G = stream_ctas(Grid{nx, ny, nz}, prec);
    VX_CHECK_ARG(G <= NOALLOC_MAX_CTAS, VX_ERR_INVALID_ARGUMENT,
                 "vx_true_residual_noalloc: grid (%d, %d, %d) needs %lld partial sums but the built-in scratch "
                 "holds %lld; use vx_true_residual with a caller-provided buffer",
                 nx, ny, nz, (long long)G, (long long)NOALLOC_MAX_CTAS);
    double* scratch = nullptr;
    st = noalloc_scratch(&scratch);
    if (st) return st;
    // every CTA overwrites its own slot before the reduction reads it: nothing needs clearing
    st = fused_dispatch<EPI_TRUE_RES>("vx_true_residual_noalloc", prec, nx, ny, nz, blocks, E, node_mask, x, b,
                                      nullptr, 0.0, res, scratch, stream);
    if (st) return st;
    return vx_reduce_partials(G, 1, scratch, norm2, stream);
}

extern "C" int vx_set_stream_kernel(int kind) {
    if (kind != VX_KERNEL_ZP && kind != VX_KERNEL_XP) {
        set_error("vx_set_stream_kernel: unknown kernel %d", kind);
        return -1;
    }
    return g_stream_kernel.exchange(kind);
}

// Fault flag of the streaming kernels' bounded waits (0 in every correct run): copied to *status;
// cleared when `clear` is non-zero.  Synchronous with respect to the device.
extern "C" int vx_device_status(int* status, int clear) {
    VX_CHECK_ARG(status, VX_ERR_NULL_POINTER, "vx_device_status: NULL status");
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, vx::g_stream_fault, sizeof(int));
    if (e == cudaSuccess && clear && v) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(vx::g_stream_fault, &zero, sizeof(int));
    }
    if (e != cudaSuccess) {
        set_error("vx_device_status: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    *status = v;
    return VX_OK;
}
