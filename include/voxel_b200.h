/*
 * libvoxel_b200 -- matrix-free Hex8 voxel elasticity on NVIDIA B200 (sm_100a).
 *
 * Plain C ABI: device pointers, sizes and a cudaStream_t in; an int status out (VX_OK == 0).
 * The library never allocates or frees device memory: the caller owns every buffer, including
 * the small `partials` scratch of the reducing kernels (sized by vx_partials_size()).  Calls are
 * asynchronous on `stream` and never synchronise the device.  On failure the call returns a
 * non-zero status and vx_last_error() gives a message for the calling host thread.
 *
 * Layouts.  "Author" layout (the hot path, as in the reference's src/voxel_mg.py:20-38): node
 * n = (ix*(ny+1)+iy)*(nz+1)+iz, DOF 3n+c, element e = (ex*ny+ey)*nz+ez -- x slowest, z fastest.
 * "Natural" layout (the reference's C product, experiments/session_a/inputs/reference.cc:23-28):
 * x fastest.  Grids are element counts (nx, ny, nz), each >= 1, with 3*(nx+1)(ny+1)(nz+1) < 2^31.
 *
 * Dirichlet masks.  The hot path encodes the reference's 0/1 DOF mask (src/voxel_mg.py:129-130)
 * as one byte per node: bit c set <=> DOF 3n+c is free.  A NULL node mask means "all free".
 */
#ifndef VOXEL_B200_H
#define VOXEL_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------- status */
enum {
    VX_OK = 0,
    VX_ERR_INVALID_ARGUMENT = 1, /* bad shape, size or enum value                               */
    VX_ERR_NULL_POINTER = 2,     /* a required pointer is NULL                                  */
    VX_ERR_ALIGNMENT = 3,        /* a pointer is not aligned to its element size                */
    VX_ERR_LAUNCH = 4,           /* CUDA launch error                                           */
    VX_ERR_UNSUPPORTED = 5,      /* element outside the parity-block model, or unsupported mode */
    VX_ERR_TIMEOUT = 6,          /* a bounded device wait ran out                               */
    VX_ERR_CUDA = 7              /* another CUDA runtime error                                  */
};

/* Precision / storage selectors.  The multigrid kernels see two kinds of vector: ITERATES (the
 * smoother's x and x_out, the operand u of a product, the coarse solve's z, both sides of the
 * prolongation, the V-cycle output) and AUXILIARY vectors (right-hand sides r, residuals res, the
 * inverse diagonal, both sides of the restriction).  Storage per selector:
 *                     iterate   auxiliary   modulus E   arithmetic
 *   VX_F64            double    double      double      FP64
 *   VX_F32            float     float       float       FP32
 *   VX_BF16_F32       bf16      bf16        bf16        FP32  (vx_matvec writes y in float)
 *   VX_F32_BF16AUX    float     bf16        bf16        FP32
 * VX_F32_BF16AUX keeps only the iterate in FP32: rounding the iterate to bf16 after every sweep
 * adds rough noise that costs outer iterations, rounding the rest does not. */
enum {
    VX_F64 = 0,
    VX_F32 = 1,
    VX_BF16_F32 = 2,
    VX_F32_BF16AUX = 3
};

const char* vx_last_error(void);
int vx_version(void);

/* ---------------------------------------------------------------------------- element (host) */

/* Hex8 element matrix (24x24, row-major, native node order) of an isotropic hx*hy*hz brick with
 * unit Young's modulus, 2x2x2 Gauss quadrature.
 * Replaces: code/hex_modal/modal.py:19-40 quadrature(lengths, nu). */
int vx_element_matrix(double hx, double hy, double hz, double nu, double* ke);

/* Cube element of edge h.  Same signature and result as the reference's C oracle
 * Replaces: experiments/session_a/inputs/reference.cc:12-15 element(h, nu, ke). */
int vx_element(double h, double nu, double* ke);

/* Parity blocks (8 x 3 x 3 = 72 doubles, row-major per block) of T ke T^T / 64 and the relative
 * norm of what the block model discards; returns VX_ERR_UNSUPPORTED if it exceeds 2e-14.
 * Replaces: code/hex_modal/modal.py:55-77 Modal(ke).blocks / .discarded_relative. */
int vx_parity_blocks(const double* ke, double* blocks, double* discarded_relative);

/* ---------------------------------------------------------------------------- operator */

/* y = K(E) u on the author layout, computed in the parity form with no atomics (deterministic).
 * `blocks` is a HOST pointer to the 72 parity coefficients (vx_parity_blocks); the kernel carries
 * them in its parameter (constant) bank.  Overwrites y (the reference kernel accumulated into a
 * caller-zeroed y; the result is the same).
 * Replaces: code/hex_modal_cuda/cuda.py:18-21 modal8(blocks, E, u, y, nx, ny, nz) and the
 * session-I variant experiments/session_i/dependencies/cuda.py:83-110 modal8_muladd. */
int vx_modal8(const double* blocks, const double* E, const double* u, double* y,
              int nx, int ny, int nz, cudaStream_t stream);

/* General operator application on the author layout.
 *   prec      VX_F64 (E,u,y double), VX_F32 (float), VX_BF16_F32 (E,u bf16; y float)
 *   node_mask NULL: y = K u (the reference's raw(u, E), src/voxel_mg.py:50-53)
 *             else: y = M K (M u) + (I - M) u (src/voxel_mg.py:129-130 Level.apply)
 * Replaces: src/voxel_mg.py:41-58 NumpyProduct.raw; experiments/session_a/donor/src/gpu_fem/
 * cuda_operators.py:658-699 OperatorSuite.matvec_full (node_fp64/node_fp32/fused paths). */
int vx_matvec(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
              const void* u, void* y, const uint8_t* node_mask, cudaStream_t stream);

/* Reference-style dense node-owned gather (24x24 rows, FP64/FP32), kept as an independent
 * control path for testing.  Replaces: cuda_operators.py:204-285 node_matvec_fp64/fp32. */
int vx_matvec_dense(int prec, int nx, int ny, int nz, const double* ke, const void* E,
                    const void* u, void* y, cudaStream_t stream);

/* Jacobi diagonal of K(E): diag, or with `inverse` != 0 the smoother's inverse diagonal
 * 1/diag on free DOFs and 1 on fixed DOFs (node_mask may be NULL).  prec VX_F64 or VX_F32
 * (E and d of that type).  `ke` is a HOST pointer to the 24x24 element matrix.
 * Replaces: src/voxel_mg.py:55-58 NumpyProduct.diagonal, :126-127 Level.inv_diag;
 * cuda_operators.py:371-424 jacobi_diag_fp64/fp32. */
int vx_diagonal(int prec, int nx, int ny, int nz, const double* ke, const void* E,
                const uint8_t* node_mask, int inverse, void* d, cudaStream_t stream);

/* Element energy ce_e = u_e^T ke u_e (FP64), the SIMP sensitivity kernel.  With `rho` non-NULL
 * it also writes dc_e = -penal * rho_e^(penal-1) * (emax - emin) * ce_e to `dc` (may be NULL).
 * Replaces: cuda_operators.py:304-358 elem_compliance_fp64; reference.cc:31-35 (ce);
 * code/hex_modal/modal.py:89-98 product() gradient. */
int vx_element_energy(int nx, int ny, int nz, const double* ke, const double* u, double* ce,
                      const double* rho, double emin, double emax, double penal, double* dc,
                      cudaStream_t stream);

/* The reference C product on the device, natural layout, same argument meaning:
 *   E = emin + (emax-emin) rho^penal; y = M K (M u) + (I-M) u; ce_e = (Mu)_e^T ke (Mu)_e;
 *   diag = diag K on free DOFs, 1 on fixed.  mask: 3N doubles, non-zero = free.
 * Any of y, ce, diag may be NULL to skip it.
 * Replaces: experiments/session_a/inputs/reference.cc:16-39 product(). */
int vx_product(int nx, int ny, int nz, const double* rho, const double* u, const double* ke,
               const double* mask, double emin, double emax, double penal,
               double* y, double* ce, double* diag, cudaStream_t stream);

/* SIMP modulus E = emin + (emax - emin) rho^penal, written in `prec` (VX_F64/VX_F32/VX_BF16_F32:
 * bf16 E).  Replaces: reference.cc:25; experiments/session_i/run_gpu.py:128. */
int vx_simp_modulus(int prec, int64_t n, const double* rho, double emin, double emax, double penal,
                    void* E, cudaStream_t stream);

/* ---------------------------------------------------------------------------- multigrid */

/* Fused damped-Jacobi sweep: x_out = x + omega * inv_diag * (r - A x), A = M K M + (I-M).
 * x_out may not alias x.  All vectors of `prec` (VX_BF16_F32: x in bf16 as the operand AND
 * written rounded to bf16, r/inv_diag/x_out float); E of the operator's storage type.
 * Replaces one smoothing step of src/voxel_mg.py:161-175 vcycle. */
int vx_jacobi_sweep(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                    const uint8_t* node_mask, const void* x, const void* r, const void* inv_diag,
                    double omega, void* x_out, cudaStream_t stream);

/* Fused masked residual: res = (r - A x) * M.  Replaces src/voxel_mg.py:168. */
int vx_residual(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                const uint8_t* node_mask, const void* x, const void* r, void* res,
                cudaStream_t stream);

/* Restriction R = P^T (27-point, separable trilinear weights) onto the coarse grid of
 * fine (nx,ny,nz) (all even), times the coarse node mask.  prec VX_F64/VX_F32.
 * Replaces: src/voxel_mg.py:83-89,100-105 restrict (+ the coarse mask of :169). */
int vx_restrict(int prec, int nx, int ny, int nz, const void* fine, const uint8_t* coarse_mask,
                void* coarse, cudaStream_t stream);

/* x += (P ec) * M on the fine grid (nx,ny,nz) from coarse (nx/2,ny/2,nz/2).
 * Replaces: src/voxel_mg.py:74-80,92-97 prolong (+ the add and mask of :171). */
int vx_prolong_add(int prec, int nx, int ny, int nz, const void* coarse, const uint8_t* fine_mask,
                   void* x, cudaStream_t stream);

/* Coarse modulus (2x2x2 mean) and injected node mask of the fine grid (nx,ny,nz), all even.
 * E in `prec` storage (VX_BF16_F32: bf16).  Replaces src/voxel_mg.py:108-116. */
int vx_coarsen_modulus(int prec, int nx, int ny, int nz, const void* E_fine, void* E_coarse,
                       cudaStream_t stream);
int vx_coarsen_mask(int nx, int ny, int nz, const uint8_t* mask_fine, uint8_t* mask_coarse,
                    cudaStream_t stream);

/* Dense constrained coarse matrix A = M K M + (I - M), n x n row-major FP64 with n = 3 * nodes;
 * deterministic (no atomics).  `ke` is a HOST pointer.  Replaces src/voxel_mg.py:61-70. */
int vx_assemble_dense(int nx, int ny, int nz, const double* ke, const double* E,
                      const uint8_t* node_mask, double* A, cudaStream_t stream);

/* Dense symmetric coarse solve z = (Ainv r) * M with a precomputed FP64 inverse (n x n), r and z
 * in `prec` (accumulation in FP64).  Replaces src/voxel_mg.py:152-159 coarse_solve + :163. */
int vx_coarse_apply(int prec, int n, const double* Ainv, const void* r, const uint8_t* node_mask,
                    void* z, cudaStream_t stream);

/* The coarse solve from the inverse Cholesky factor instead of the inverse: with A = L L^T and
 * Linv = L^-1, vx_coarse_pack writes M = tril(Linv) + triu(Linv^T, 1) (n x n row-major; m may not
 * alias linv), and vx_coarse_apply_factor computes z = (Linv^T (Linv r)) * M in two passes over the
 * two triangles of M (y: n doubles of caller scratch).  Same bytes per apply as vx_coarse_apply,
 * but the set-up needs no n^3 product.  Replaces the two triangular solves of
 * src/voxel_mg.py:152-159 coarse_solve.  r auxiliary, z an iterate of `prec`. */
int vx_coarse_pack(int n, const double* linv, double* m, cudaStream_t stream);
int vx_coarse_apply_factor(int prec, int n, const double* m, const void* r, const uint8_t* node_mask,
                           double* y, void* z, cudaStream_t stream);

/* Node masks <-> the reference's 0/1 DOF masks (double, 3 per node, author layout). */
int vx_mask_from_dofs(int64_t nodes, const double* dof_mask, uint8_t* node_mask, cudaStream_t stream);

/* ---------------------------------------------------------------------------- CG vector kernels */

/* Number of doubles the `partials` scratch of the reducing kernels needs for vectors of length n
 * (per reduction slot; kernels reducing k quantities need k times this). */
int64_t vx_partials_size(int64_t n);

/* Deterministic dot products (fixed reduction order; bitwise reproducible run to run):
 * out[k] (device double) = sum_i a_k[i] * b_k[i] for k < count (count <= 3), in FP64, vectors
 * of `prec` (VX_F64 or VX_F32).  `partials` holds count * vx_partials_size(n) doubles.
 * Replaces the `@` / linalg.norm reductions of src/voxel_mg.py:192-211 and donor simp_r2.py. */
int vx_dots(int prec, int64_t n, int count, const void* const* a, const void* const* b,
            double* partials, double* out, cudaStream_t stream);

/* y := alpha * x + beta * y (host scalars; VX_F64 / VX_F32). */
int vx_axpby(int prec, int64_t n, double alpha, const void* x, double beta, void* y, cudaStream_t stream);

/* Cast between storage precisions (VX_F64 <-> VX_F32 <-> bf16), optional scale (dst = scale*src). */
int vx_cast(int64_t n, int src_prec, const void* src, int dst_prec, void* dst, double scale,
            cudaStream_t stream);

/* ---------------------------------------------------------------------------- SIMP */

/* Matrix-free hat density filter on the element grid (author layout), weights max(0, rmin - |d|),
 * support ceil(rmin) - 1 (rmin <= 4): mode 0 y = H x; mode 1 y = (H x) / s; mode 2 y = H (x / s),
 * s = H 1 the row sums.  Replaces: experiments/session_a/donor/src/gpu_fem/filter_r2.py:40-76,
 * 93-171 (cone stencil, forward, transpose); the CSR filter of experiments/session_h/run_w1b.py:97-125. */
int vx_cone_filter(int nx, int ny, int nz, double rmin, const double* x, const double* s, int mode,
                   double* y, cudaStream_t stream);

/* top88 optimality-criteria update with the bisection on the multiplier on the device
 * (experiments/session_h/run_w1b.py:46-62, 82-94).  State S (16 doubles): S[0] l1, S[1] l2,
 * S[2] last lmid, S[3] last volume, S[4] volfrac, S[5] tol, S[6] element count, S[10] done,
 * S[11] probes, S[12] max probes, S[15] = 1.  A probe: lmid = (l1 + l2) / 2,
 * x_new = clip(x sqrt(max(-dc / dv / lmid, 0)), max(x - move, 0), min(x + move, 1)), volume =
 * sum w x_new / n with w = H (1 / s) (= mean of the filtered x_new); vx_oc_finalize moves l1 or l2 and
 * sets done when (l2 - l1) / (l1 + l2) <= tol.  vx_oc_apply writes x_new for the last lmid. */
int64_t vx_oc_partials(int64_t n);
int vx_oc_probe(int64_t n, const double* x, const double* dc, const double* dv, const double* w, double move,
                const double* S, double* partials, cudaStream_t stream);
int vx_oc_finalize(int64_t n, const double* partials, double* S, cudaStream_t stream);
int vx_oc_apply(int64_t n, const double* x, const double* dc, const double* dv, double move, const double* S,
                double* x_new, cudaStream_t stream);

/* Operator forms fused with the outer Krylov loop (FP64/FP32, author layout, node mask optional):
 *   vx_apply_dot:     q = A p and partials[cta] = sum p.q over the CTA's owned nodes
 *   vx_true_residual: res = b - A x and partials[cta] = sum res^2
 * `partials` holds vx_operator_partials(prec, nx, ny, nz) doubles; sum them with vx_reduce_partials or
 * vx_solver_finalize.  Replace the `apply_A(p)` + `p @ q` and `b - apply_A(x)` + `norm` pairs of
 * src/voxel_mg.py:192-203 and donor simp_r2.py:255-270. */
int64_t vx_operator_partials(int prec, int nx, int ny, int nz);
int vx_apply_dot(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                 const uint8_t* node_mask, const void* p, void* q, double* partials, cudaStream_t stream);
int vx_true_residual(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                     const uint8_t* node_mask, const void* x, const void* b, void* res, double* partials,
                     cudaStream_t stream);
int vx_reduce_partials(int64_t G, int count, const double* partials, double* out, cudaStream_t stream);
/* The same two forms with the partial sums restricted to node planes x_lo <= ix < x_hi (0 <= x_lo
 * <= x_hi <= nx + 1); the output vector is written everywhere.  An x-slab (below) leaves its
 * shared planes out and adds them after they are rewritten (vx_plane_fix with `dot`). */
int vx_apply_dot_planes(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                        const uint8_t* node_mask, const void* p, void* q, double* partials, int x_lo, int x_hi,
                        cudaStream_t stream);
int vx_true_residual_planes(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                            const uint8_t* node_mask, const void* x, const void* b, void* res, double* partials,
                            int x_lo, int x_hi, cudaStream_t stream);

/* Fault flag of the streaming operator kernels.  Their warps hand partial sums to each other
 * through shared-memory barriers whose waits are bounded; a wait that ran out (which a correct run
 * never does) sets this flag, and the output of that launch is invalid.  *status receives the flag
 * (0 or 1); a non-zero `clear` resets it.  Synchronous with respect to the device.  No counterpart
 * in the reference (its kernels have no waits between threads). */
int vx_device_status(int* status, int clear);

/* Streaming operator kernel for FP64 / FP32 iterates (VX_F64, VX_F32), process-wide; the bf16
 * iterate form always uses the element-plane-pair kernel.  Both compute the same arithmetic in the
 * same order (FP32 results are bitwise equal; in FP64 the compiler contracts different
 * multiply-add pairs, a difference of one rounding); they differ in how work is laid out:
 *   VX_KERNEL_XP  a pair of element planes per thread, CTA barriers between rows (default)
 *   VX_KERNEL_ZP  a pair of z node columns per thread, coalesced row spans staged by cp.async,
 *                 warps in a wavefront handing partial sums over mbarriers
 * vx_operator_partials follows the selection, so scratch sized before a change may be too small
 * after it.  Returns the previous selection, or -1 for an unknown kind.  No counterpart in the
 * reference. */
enum { VX_KERNEL_XP = 0, VX_KERNEL_ZP = 1 };
int vx_set_stream_kernel(int kind);

/* Tensor-core element-block operator, an experiment measured against the streaming kernels and not
 * used by the solvers: the dense 24 x 24 element matrix applied to 128 elements at a time by
 * tcgen05.mma (TF32 operands from FP32 storage, FP32 accumulation in tensor memory).
 * ke: host 24 x 24 element matrix (row-major); E: element moduli (float); node_mask: optional,
 * zeroes the constrained components of u; mode 0: y = K(E) u over the nodes (y overwritten, 3N
 * floats); mode 1: the 24 scaled element results per element, y[24 e + i] (24 Ne floats).
 * Results carry TF32 rounding (about 1e-3 relative).  The form the reference's donor ships is a
 * BF16 WMMA element-block matvec (experiments/session_a/donor/src/gpu_fem/cuda_fused_matvec.py:147-281). */
int vx_tc_element_product(int nx, int ny, int nz, const double* ke, const float* E, const uint8_t* node_mask,
                          const float* u, float* y, int mode, cudaStream_t stream);
/* Fault flag of vx_tc_element_product's bounded accumulator wait, as vx_device_status. */
int vx_tc_status(int* status, int clear);

/* The coarsest level's exact solve, set up without library calls (replaces the host Cholesky and the
 * two triangular solves of src/voxel_mg.py:152-159, experiments/session_i/run_gpu.py:281-286).
 * A: the dense n x n constrained matrix (vx_assemble_dense, row-major, symmetric positive definite),
 * bw: its half-bandwidth (a voxel grid's coarsest matrix: 3 ((ny+1)(nz+1) + (nz+1) + 1) + 2, at most
 * n - 1).  Writes packed = tril(L^-1) + triu(L^-T, 1) with A = L L^T for vx_coarse_apply_factor, and
 * *info (device int) = 0, or the 1-based column of the first non-positive pivot.  `work` holds
 * vx_coarse_factor_workspace(n, bw) doubles.  Bands wider than the kernel's shared-memory window
 * (about 5800) are rejected with VX_ERR_INVALID_ARGUMENT ("too wide"). */
int64_t vx_coarse_factor_workspace(int n, int bw);
int vx_coarse_factor(int n, int bw, const double* A, double* packed, double* work, int* info, cudaStream_t stream);
/* Several coarsest systems of one size at once (a serving batch's per-job coarse solves), every
 * launch of the factorisation covering all of them: slots (host, `count` entries) index the n x n
 * matrix stacks A and packed (slot k at k n^2) and info (slot k at k); work holds `count` workspaces
 * of vx_coarse_factor_workspace(n, bw) doubles.  Results equal vx_coarse_factor's on each matrix.
 * No counterpart in the reference. */
int vx_batch_coarse_factor(int n, int bw, int count, const int* slots, const double* A, double* packed,
                           double* work, int* info, cudaStream_t stream);
/* The packed inverse factor tril(L^-1) + triu(L^-T, 1) from a Cholesky factor L the caller already
 * has (dense row-major n x n, lower triangle read, half-bandwidth bw): what the reference's
 * Multigrid(..., coarse_factor, ...) receives (src/voxel_mg.py:120-160).  work: as vx_coarse_factor.
 * No factorisation: the diagonal blocks are inverted side by side, then the blocked band inverse. */
int vx_coarse_pack_factor(int n, int bw, const double* L, double* packed, double* work, cudaStream_t stream);

/* ---------------------------------------------------------------------------- batches
 * `slots` independent systems of one size solved in lockstep (the serving loop's batches): slot k's
 * vectors start k * stride entries after the given pointers, its scalars at S + 16 k, its partial
 * sums at partials + k * 2 vx_solver_partials(n) (vx_batch_dots_pr) -- one launch for the whole batch.
 * The single-system forms above are the one-slot case.  No counterpart in the reference (it solves
 * one system at a time). */
int vx_batch_finalize(int op, int64_t G, int slots, const double* partials, int64_t pstride, double* S,
                      cudaStream_t stream);
int vx_batch_cg_update(int prec, int64_t n, int slots, int64_t stride, const double* S, void* x, const void* p,
                       void* r, const void* q, int update_r, cudaStream_t stream);
int vx_batch_cg_direction(int zprec, int64_t n, int slots, int64_t stride, const double* S, const void* z, double* p,
                          void* z_old, cudaStream_t stream);
int vx_batch_dots_pr(int zprec, int64_t n, int slots, int64_t stride, const double* r, const void* zn, const void* zo,
                     double* partials, cudaStream_t stream);
/* vx_coarse_apply_factor for `slots` coarse systems of n DOFs: packed factors back to back (slot k at
 * m + k n^2), slot k's right-hand side, node mask and solution at k * vs DOFs, y of slots * n doubles. */
int vx_batch_coarse_apply_factor(int prec, int n, int slots, int64_t vs, const double* m, const void* r,
                                 const uint8_t* node_mask, double* y, void* z, cudaStream_t stream);
/* vx_graph_while_end whose loop runs while any of `slots` systems (scalars S + 16 k) is running. */
int vx_batch_graph_while_end(void* handle, const double* S, int slots, cudaStream_t stream);

/* res = b - A x and *norm2 = sum res^2 (a device double), like vx_true_residual followed by
 * vx_reduce_partials, but needing no scratch buffer from the caller: for code that may not
 * allocate device memory (a request loop that must never call cudaMalloc mid-flight, a plugin
 * inside another framework's memory arena, a process under a hard memory cap).  The partial sums
 * live in a fixed array compiled into the library: 16384 doubles (128 KiB) on every device that
 * loads it, kept until the process exits.  The streaming kernels keep one partial per CTA
 * (vx_operator_partials(prec, ...)) and chunk x only while the CTAs stay within 16384, so every grid
 * fits whose y-z tiling does (all but extremely flat ones); a launch that would need more than 16384
 * partials is rejected with VX_ERR_INVALID_ARGUMENT.  The
 * first call on each device looks up the array's device address (cudaGetSymbolAddress) and keeps
 * it for the process: make that first call before any stream capture, and do not use the entry
 * point across a reset of the device's primary context (cudaDeviceReset), which would leave the
 * kept address stale.  All calls share the one array: calls whose executions overlap on the GPU
 * (different streams, concurrent host threads) race and must be serialised by the caller.
 * No counterpart in the reference (it allocates every temporary through CuPy). */
int vx_true_residual_noalloc(int prec, int nx, int ny, int nz, const double* blocks, const void* E,
                             const uint8_t* node_mask, const void* x, const void* b, void* res,
                             double* norm2, cudaStream_t stream);

/* ---------------------------------------------------------------------------- device-scalar solvers
 * The Krylov loops of the reference (src/voxel_mg.py:181-217 fcg; donor simp_r2.py:187-295 pcg) with
 * every scalar in a device array S of vx_solver_slots() doubles:
 *   S[0] r.z  S[1] p.q  S[2] alpha  S[3] |b-Ax|^2  S[4] rel  S[5] |b|  S[6] beta  S[7] r.z_new
 *   S[8] r.(z_new-z_old)  S[9] tol  S[10] done  S[11] iterations  S[12] maxiter  S[13] matvecs
 *   S[14] breakdown  S[15] iterations per loop body
 * vx_solver_finalize(op, G, partials, S) sums G partials in a fixed order and applies op:
 *   0 p.q -> alpha = rz/pq, it++, mv++      1 |b-Ax|^2 -> rel, mv++, done if rel <= tol
 *   2 Polak-Ribiere beta (two partial rows)  3 Fletcher-Reeves beta   4 |b|   5 r.z   6 rel only */
int vx_solver_slots(void);
int64_t vx_solver_partials(int64_t n);
int vx_solver_finalize(int op, int64_t G, const double* partials, double* S, cudaStream_t stream);
int vx_cg_update(int prec, int64_t n, const double* S, void* x, const void* p, void* r, const void* q,
                 int update_r, cudaStream_t stream);
/* p = z + beta p, and z_old = z when z_old is not NULL.  p (and r of vx_dots_pr) are of `prec`;
 * z, z_old (and zn, zo) are iterates of the preconditioner's selector `zprec`, so a mixed-precision
 * loop keeps z_old in FP32 (an exact copy of the FP32 z).  vx_dots_pr writes the partials of r.zn
 * and, with zo, of r.(zn - zo) (Polak-Ribiere, src/voxel_mg.py:205-208). */
int vx_cg_direction(int prec, int zprec, int64_t n, const double* S, const void* z, void* p, void* z_old,
                    cudaStream_t stream);
int vx_dots_pr(int prec, int zprec, int64_t n, const void* r, const void* zn, const void* zo,
               double* partials, cudaStream_t stream);
/* FP64 x += S[alpha] p (skipped once S says done or breakdown) followed by vx_cg_direction, with p
 * read once: the x update of src/voxel_mg.py:199 deferred into the direction update of :209 on the
 * iterations that do not test the true residual.  z, z_old iterates of `zprec`. */
int vx_cg_direction_update(int zprec, int64_t n, const double* S, const void* z, double* p, void* z_old,
                           double* x, cudaStream_t stream);
int vx_jacobi_precond_dot(int prec, int64_t n, const void* d, const void* r, void* z, double* partials,
                          cudaStream_t stream);
/* V-cycle entry: r_mg = (prec) r64 (skipped if r_mg is NULL) and x = omega * inv_diag * r_mg;
 * the first damped-Jacobi step of src/voxel_mg.py:165 fused with the cast of :178. */
int vx_vcycle_entry(int prec, int64_t n, const double* r64, void* r_mg, const void* inv_diag, double omega,
                    void* x, cudaStream_t stream);
/* vx_vcycle_entry preceded by the CG update r64 -= S[alpha] q (skipped once S says done or
 * breakdown), so the residual is read once for both: the r update of src/voxel_mg.py:200 fused
 * into the preconditioner's first step. */
int vx_vcycle_entry_update(int prec, int64_t n, const double* S, double* r64, const double* q, void* r_mg,
                           const void* inv_diag, double omega, void* x, cudaStream_t stream);
int vx_scaled_product(int prec, int64_t n, double omega, const void* a, const void* b, void* out,
                      cudaStream_t stream);
int vx_set_scalars(double* S, int first, int count, double value, cudaStream_t stream);

/* A CUDA-graph WHILE loop: begin captures the loop body from `stream` (non-default); end appends
 * the condition kernel (continue while !done && !breakdown && it + S[15] <= maxiter) and
 * instantiates; launch runs the whole loop as one graph launch. */
int vx_graph_while_begin(cudaStream_t stream, void** handle);
int vx_graph_while_end(void* handle, const double* S, cudaStream_t stream);
int vx_graph_launch(void* handle, cudaStream_t stream);
/* Number of nodes in a WHILE graph's captured body (-1 on error). */
int64_t vx_graph_body_nodes(void* handle);
/* Capture state of `stream`: 0 none, 1 active, 2 invalidated, -1 query failed. */
int vx_capture_status(cudaStream_t stream);
int vx_graph_destroy(void* handle);

/* ---------------------------------------------------------------------------- x-slab decomposition
 * A slab holds elements ex in [a, b) and node planes a..b of a global grid (author layout: x is the
 * slowest index, so a slab's vectors are contiguous slices of the global ones).  The planes a and b
 * are shared with the neighbouring slabs.  On a shared plane the global operator is the sum of the
 * two slabs' element-layer contributions; the reference runs one process on one grid
 * (experiments/session_i/run_gpu.py:304 A, src/voxel_mg.py:120-178 Level/Multigrid), and these two
 * entry points make a slab-local operator the global one.
 *
 * vx_layer_partial: out (3 (ny+1)(nz+1) values, arithmetic type: FP64 for VX_F64, FP32 otherwise)
 * = M K_layer (M u) on node plane `side` (0 lower, 1 upper) of the single element layer whose
 * modulus is E (ny*nz, auxiliary storage) and whose two node planes are u (iterate storage) and
 * node_mask (NULL: all free).  `ke` is a HOST pointer to the 24x24 element matrix.
 *
 * vx_plane_fix: rewrites one shared plane (`nodes` nodes) of an operator form's output from
 * s = lo + hi (the lower slab's contribution first, so both holders compute identical values),
 * with A x = s on free DOFs and x on fixed ones:
 *   mode 0  out = A x                                 (arithmetic type; vx_matvec's output)
 *   mode 1  out = x + omega inv_diag (r - A x)        (iterate; vx_jacobi_sweep's output)
 *   mode 2  out = scale * (free ? r - A x : 0)        (auxiliary; vx_residual's output; scale 1/2
 *                                                      splits a shared plane before restriction)
 *   mode 3  out = r - A x                             (VX_F64 only; vx_true_residual's output)
 * With `dot` (modes 0 and 3; NULL otherwise), dot[cta] (vx_plane_fix_partials(nodes) doubles) =
 * the CTA's sum of x . out (mode 0) or out^2 (mode 3) over the rewritten plane if `owned` is
 * non-zero, else 0.  With vx_apply_dot_planes / vx_true_residual_planes leaving the slab's shared
 * planes out of their sums, the two kernels' partials summed over all slabs count each DOF once.
 * vx_plane_sum: out = lo + hi (n values of the selector's auxiliary storage): the restricted
 * right-hand side on a shared coarse plane. */
int vx_layer_partial(int prec, int ny, int nz, const double* ke, const void* E, const void* u,
                     const uint8_t* node_mask, int side, void* out, cudaStream_t stream);
int64_t vx_plane_fix_partials(int64_t nodes);
int vx_plane_fix(int prec, int mode, int64_t nodes, const void* lo, const void* hi, const uint8_t* node_mask,
                 const void* x, const void* r, const void* inv_diag, double omega, double scale, void* out,
                 double* dot, int owned, cudaStream_t stream);
int vx_plane_sum(int prec, int64_t n, const void* lo, const void* hi, void* out, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* VOXEL_B200_H */
