// Host-side parts of libvoxel_b200: error reporting, argument checks, the Hex8 element matrix and
// its parity blocks.
#include "vx_common.cuh"

#include <cmath>
#include <cstdarg>
#include <cstring>

namespace vx {

static thread_local char g_error[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

int check_grid(int nx, int ny, int nz) {
    if (nx < 1 || ny < 1 || nz < 1) {
        set_error("invalid grid (%d, %d, %d): every extent must be >= 1", nx, ny, nz);
        return VX_ERR_INVALID_ARGUMENT;
    }
    if (ny + 1 > 6 * 65535) {      // the streaming kernels tile y over the launch grid's y extent
        set_error("invalid grid (%d, %d, %d): ny must be below %d", nx, ny, nz, 6 * 65535);
        return VX_ERR_INVALID_ARGUMENT;
    }
    const double dofs = 3.0 * (nx + 1.0) * (ny + 1.0) * (nz + 1.0);
    if (dofs >= 2147483647.0) {
        set_error("grid (%d, %d, %d) has %.0f DOFs; the limit is 2^31 - 1", nx, ny, nz, dofs);
        return VX_ERR_INVALID_ARGUMENT;
    }
    return VX_OK;
}

}  // namespace vx

using namespace vx;

extern "C" const char* vx_last_error(void) { return g_error; }

extern "C" int vx_version(void) { return 10000; }   // 1.0.0

// Native Hex8 node offsets (the reference's XYZ table, code/hex_modal/modal.py:9-10).
static const int kOff[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                               {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

extern "C" int vx_element_matrix(double hx, double hy, double hz, double nu, double* ke) {
    VX_CHECK_ARG(ke, VX_ERR_NULL_POINTER, "vx_element_matrix: NULL ke");
    VX_CHECK_ARG(hx > 0 && hy > 0 && hz > 0 && nu > -1.0 && nu < 0.5, VX_ERR_INVALID_ARGUMENT,
                 "vx_element_matrix: need positive lengths and -1 < nu < 0.5");
    const double h[3] = {hx, hy, hz};
    const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = 1.0 / (2.0 * (1.0 + nu));
    double D[6][6] = {};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) D[i][j] = lam;
        D[i][i] += 2.0 * mu;
        D[3 + i][3 + i] = mu;
    }
    std::memset(ke, 0, 576 * sizeof(double));
    const double gq = 1.0 / std::sqrt(3.0);
    for (int q = 0; q < 8; ++q) {
        double xi[3];
        for (int a = 0; a < 3; ++a) xi[a] = (2.0 * kOff[q][a] - 1.0) * gq;
        double dN[8][3];
        for (int i = 0; i < 8; ++i) {
            double s[3], f[3];
            for (int a = 0; a < 3; ++a) { s[a] = 2.0 * kOff[i][a] - 1.0; f[a] = 1.0 + s[a] * xi[a]; }
            dN[i][0] = s[0] * f[1] * f[2] / (4.0 * h[0]);
            dN[i][1] = s[1] * f[0] * f[2] / (4.0 * h[1]);
            dN[i][2] = s[2] * f[0] * f[1] / (4.0 * h[2]);
        }
        double B[6][24] = {};
        for (int i = 0; i < 8; ++i) {
            const double dx = dN[i][0], dy = dN[i][1], dz = dN[i][2];
            B[0][3 * i] = dx; B[1][3 * i + 1] = dy; B[2][3 * i + 2] = dz;
            B[3][3 * i] = dy; B[3][3 * i + 1] = dx;
            B[4][3 * i + 1] = dz; B[4][3 * i + 2] = dy;
            B[5][3 * i] = dz; B[5][3 * i + 2] = dx;
        }
        double DB[6][24];
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 24; ++c) {
                double t = 0.0;
                for (int k = 0; k < 6; ++k) t += D[r][k] * B[k][c];
                DB[r][c] = t;
            }
        const double w = h[0] * h[1] * h[2] / 8.0;
        for (int r = 0; r < 24; ++r)
            for (int c = 0; c < 24; ++c) {
                double t = 0.0;
                for (int k = 0; k < 6; ++k) t += B[k][r] * DB[k][c];
                ke[24 * r + c] += t * w;
            }
    }
    return VX_OK;
}

extern "C" int vx_element(double h, double nu, double* ke) { return vx_element_matrix(h, h, h, nu, ke); }

extern "C" int vx_parity_blocks(const double* ke, double* blocks, double* discarded_relative) {
    VX_CHECK_ARG(ke && blocks, VX_ERR_NULL_POINTER, "vx_parity_blocks: NULL pointer");
    // T[3p+c][3i+c] = (-1)^popcount(p & code_i), code_i = x + 2y + 4z of native node i
    int code[8];
    for (int i = 0; i < 8; ++i) code[i] = kOff[i][0] + 2 * kOff[i][1] + 4 * kOff[i][2];
    // full = T ke T^T / 64 (24x24)
    static thread_local double tk[24][24], full[24][24];
    for (int p = 0; p < 8; ++p)
        for (int c = 0; c < 3; ++c)
            for (int col = 0; col < 24; ++col) {
                double t = 0.0;
                for (int i = 0; i < 8; ++i) {
                    const double s = (__builtin_popcount(p & code[i]) & 1) ? -1.0 : 1.0;
                    t += s * ke[(3 * i + c) * 24 + col];
                }
                tk[3 * p + c][col] = t;
            }
    for (int r = 0; r < 24; ++r)
        for (int q = 0; q < 8; ++q)
            for (int c = 0; c < 3; ++c) {
                double t = 0.0;
                for (int i = 0; i < 8; ++i) {
                    const double s = (__builtin_popcount(q & code[i]) & 1) ? -1.0 : 1.0;
                    t += tk[r][3 * i + c] * s;
                }
                full[r][3 * q + c] = t / 64.0;
            }
    double kept2 = 0.0, all2 = 0.0;
    bool in_block[24][24] = {};
    for (int g = 0; g < 8; ++g) {
        int idx[3];
        for (int a = 0; a < 3; ++a) idx[a] = 3 * (g ^ (1 << a)) + a;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                blocks[9 * g + 3 * a + b] = full[idx[a]][idx[b]];
                in_block[idx[a]][idx[b]] = true;
            }
    }
    double maxc = 0.0;
    for (int i = 0; i < 72; ++i) maxc = std::fmax(maxc, std::fabs(blocks[i]));
    for (int r = 0; r < 24; ++r)
        for (int c = 0; c < 24; ++c) {
            all2 += full[r][c] * full[r][c];
            if (!in_block[r][c]) kept2 += full[r][c] * full[r][c];
        }
    const double disc = all2 > 0 ? std::sqrt(kept2 / all2) : INFINITY;
    if (discarded_relative) *discarded_relative = disc;
    if (!std::isfinite(disc) || disc > 2e-14) {
        set_error("vx_parity_blocks: element is outside the parity-block model (discarded %.3g)", disc);
        return VX_ERR_UNSUPPORTED;
    }
    // the kernels use only the 45 structural non-zeros; reject anything else
    for (int g = 0; g < 8; ++g)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                if (!parity_nonzero(g, a, b) && std::fabs(blocks[9 * g + 3 * a + b]) > 1e-12 * maxc) {
                    set_error("vx_parity_blocks: coefficient (%d,%d,%d) = %.3g outside the brick pattern",
                              g, a, b, blocks[9 * g + 3 * a + b]);
                    return VX_ERR_UNSUPPORTED;
                }
    return VX_OK;
}
