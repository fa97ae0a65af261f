"""CPU oracle for the matrix-free Hex8 voxel-elasticity path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or the timed CPU baseline.  The product path
(the ``voxel_b200`` package and its CUDA library) never imports it.

Every function below is a plain NumPy restatement of one reference function,
written independently and cited as ``file:line`` inside the reference project
nejeoui/matrix-free-voxel-elasticity.  The restatement is pinned against golden
vectors produced by the reference itself (``tests/golden/make_golden.py``
imports the reference's own Python modules and its compiled C++ product and
writes ``tests/golden/*.npz``); ``tests/test_oracle.py`` checks every pin.

Layouts.  "Author" layout (the hot-path layout): node ``n = (ix*(ny+1)+iy)*(nz+1)+iz``,
DOF ``3n+c``, element ``e = (ex*ny+ey)*nz+ez`` -- x slowest, z fastest.  "Natural"
layout (fixtures, C reference): x fastest.
"""
from __future__ import annotations

import math

import numpy as np

# Native Hex8 node order of the element matrix (code/hex_modal/modal.py:9-10, src/voxel_mg.py:27-28).
NATIVE_OFFSETS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                           [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
# Binary code (bx + 2 by + 4 bz) of each native node (code/hex_modal/modal.py:11).
NATIVE_CODE = NATIVE_OFFSETS[:, 0] + 2 * NATIVE_OFFSETS[:, 1] + 4 * NATIVE_OFFSETS[:, 2]


# ------------------------------------------------------------------------------------ element
def quadrature(lengths, nu):
    """Hex8 element matrix of an isotropic brick, 2x2x2 Gauss, engineering-strain Voigt order,
    unit Young's modulus.  Restates code/hex_modal/modal.py:19-40 (== reference.cc element())."""
    h = np.asarray(lengths, dtype=np.float64).reshape(3)
    lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = 1.0 / (2.0 * (1.0 + nu))
    D = np.diag([lam + 2 * mu] * 3 + [mu] * 3)
    D[0, 1] = D[0, 2] = D[1, 0] = D[1, 2] = D[2, 0] = D[2, 1] = lam
    s = 2.0 * NATIVE_OFFSETS - 1.0                       # node sign per axis
    g = 1.0 / math.sqrt(3.0)
    ke = np.zeros((24, 24))
    for gp in s * g:                                     # Gauss points at the node sign pattern
        # dN_i/dx_a = s_ia * prod_{b != a}(1 + s_ib xi_b) / (4 h_a)
        f = 1.0 + s * gp[None, :]                        # (8, 3)
        dN = np.empty((8, 3))
        dN[:, 0] = s[:, 0] * f[:, 1] * f[:, 2] / (4 * h[0])
        dN[:, 1] = s[:, 1] * f[:, 0] * f[:, 2] / (4 * h[1])
        dN[:, 2] = s[:, 2] * f[:, 0] * f[:, 1] / (4 * h[2])
        B = np.zeros((6, 24))
        B[0, 0::3], B[1, 1::3], B[2, 2::3] = dN[:, 0], dN[:, 1], dN[:, 2]
        B[3, 0::3], B[3, 1::3] = dN[:, 1], dN[:, 0]
        B[4, 1::3], B[4, 2::3] = dN[:, 2], dN[:, 1]
        B[5, 0::3], B[5, 2::3] = dN[:, 2], dN[:, 0]
        ke += B.T @ D @ B * (h.prod() / 8.0)
    return ke


def parity_transform():
    """24x24 Walsh-Hadamard change of basis T[3p+c, 3i+c] = (-1)^popcount(p & code_i)
    (code/hex_modal/modal.py:12-14)."""
    Hn = np.array([[(-1.0) ** bin(p & n).count("1") for n in range(8)] for p in range(8)])
    return np.kron(Hn[:, NATIVE_CODE], np.eye(3))


def parity_groups():
    """Index triples of the 8 parity blocks: group g holds (x @ g^1, y @ g^2, z @ g^4)
    (code/hex_modal/modal.py:15)."""
    return np.array([[3 * (g ^ (1 << a)) + a for a in range(3)] for g in range(8)])


def parity_blocks(ke, tolerance=2e-14):
    """Parity blocks C[g] (8x3x3) of T ke T^T / 64; raises ValueError when ke is outside the block
    model (code/hex_modal/modal.py:55-77).  Returns (blocks, discarded_relative)."""
    T = parity_transform()
    full = T @ np.asarray(ke, dtype=np.float64).reshape(24, 24) @ T.T / 64.0
    kept = np.zeros_like(full)
    blocks = np.empty((8, 3, 3))
    for g, idx in enumerate(parity_groups()):
        blocks[g] = full[np.ix_(idx, idx)]
        kept[np.ix_(idx, idx)] = blocks[g]
    discarded = float(np.linalg.norm(full - kept) / np.linalg.norm(full))
    if not np.isfinite(discarded) or discarded > tolerance:
        raise ValueError(f"element outside the parity-block model: {discarded}")
    return blocks, discarded


# ------------------------------------------------------------------------------------ layouts
def n_nodes(shape):
    nx, ny, nz = (int(s) for s in shape)
    return (nx + 1) * (ny + 1) * (nz + 1)


def edof_author(shape):
    """(Ne, 24) DOF table in author layout, native node order (src/voxel_mg.py:32-38)."""
    nx, ny, nz = (int(s) for s in shape)
    e = np.arange(nx * ny * nz)
    ex, ey, ez = e // (ny * nz), (e // nz) % ny, e % nz
    cols = []
    for ox, oy, oz in NATIVE_OFFSETS:
        node = ((ex + ox) * (ny + 1) + ey + oy) * (nz + 1) + ez + oz
        cols.extend([3 * node, 3 * node + 1, 3 * node + 2])
    return np.stack(cols, axis=1)


def element_nodes(shape):
    """(Ne, 8) node of each element per binary lane b = bx + 2 by + 4 bz (src/voxel_kernels.py:46-53)."""
    nx, ny, nz = (int(s) for s in shape)
    e = np.arange(nx * ny * nz)
    ex, ey, ez = e // (ny * nz), (e // nz) % ny, e % nz
    b = np.arange(8)
    return (((ex[:, None] + (b & 1)) * (ny + 1) + ey[:, None] + ((b >> 1) & 1)) * (nz + 1)
            + ez[:, None] + ((b >> 2) & 1))


def to_author(a, shape, nodal=False):
    """Natural (x fastest) -> author (z fastest) (experiments/session_a/dependencies/common.py:35-39)."""
    nx, ny, nz = (int(s) for s in shape)
    if nodal:
        return np.ascontiguousarray(np.asarray(a).reshape(nz + 1, ny + 1, nx + 1, 3)
                                    .transpose(2, 1, 0, 3)).ravel()
    return np.ascontiguousarray(np.asarray(a).reshape(nz, ny, nx).transpose(2, 1, 0)).ravel()


def to_natural(a, shape, nodal=False):
    """Author -> natural (experiments/session_a/dependencies/common.py:42-46)."""
    nx, ny, nz = (int(s) for s in shape)
    if nodal:
        return np.ascontiguousarray(np.asarray(a).reshape(nx + 1, ny + 1, nz + 1, 3)
                                    .transpose(2, 1, 0, 3)).ravel()
    return np.ascontiguousarray(np.asarray(a).reshape(nx, ny, nz).transpose(2, 1, 0)).ravel()


# ------------------------------------------------------------------------------------ products
def product_raw(shape, ke, u, E, dtype=np.float64):
    """y = sum_e E_e ke u_e (unmasked, caller pre-masks u) (src/voxel_mg.py:50-53)."""
    edof = edof_author(shape)
    ke = np.asarray(ke, dtype=dtype)
    u = np.asarray(u, dtype=dtype)
    E = np.asarray(E, dtype=dtype)
    contrib = (E[:, None] * (u[edof] @ ke.T)).astype(dtype)
    y = np.zeros(3 * n_nodes(shape), dtype=dtype)
    np.add.at(y, edof, contrib)
    return y


def product_diagonal(shape, ke, E, dtype=np.float64):
    """diag K(E) (src/voxel_mg.py:55-58)."""
    edof = edof_author(shape)
    d = np.zeros(3 * n_nodes(shape), dtype=dtype)
    np.add.at(d, edof, (np.asarray(E, dtype=dtype)[:, None] * np.diag(ke)[None, :]).astype(dtype))
    return d


def element_energy(shape, ke, u):
    """ce_e = u_e^T ke u_e (donor cuda_operators.py:304-358; reference.cc:31-35 on masked u)."""
    ue = np.asarray(u, dtype=np.float64)[edof_author(shape)]
    return np.einsum("ei,ij,ej->e", ue, np.asarray(ke, dtype=np.float64), ue)


def apply_dirichlet(shape, ke, E, mask, u):
    """A u = M K (M u) + (I - M) u (src/voxel_mg.py:129-130)."""
    m = np.asarray(mask, dtype=np.float64)
    return product_raw(shape, ke, u * m, E) * m + u * (1.0 - m)


def simp_modulus(rho, emin, emax=1.0, penal=3.0):
    """E = emin + (emax - emin) rho^p (reference.cc:25)."""
    return emin + (emax - emin) * np.asarray(rho, dtype=np.float64) ** penal


def c_reference_product(shape, rho, u, ke, mask, emin, emax=1.0, penal=3.0):
    """Natural-layout restatement of reference.cc product() (experiments/session_a/inputs/reference.cc:16-39):
    returns (y, ce, diag) with y = M K (M u) + (I - M) u, ce on the masked state, diag = 1 on fixed DOFs."""
    m_a = to_author(mask, shape, True)
    u_a = to_author(u, shape, True)
    E_a = to_author(simp_modulus(rho, emin, emax, penal), shape)
    um = u_a * (m_a != 0)
    y = product_raw(shape, ke, um, E_a)
    d = product_diagonal(shape, ke, E_a)
    fixed = m_a == 0
    y[fixed] = u_a[fixed]
    d[fixed] = 1.0
    ce = element_energy(shape, ke, um)
    return to_natural(y, shape, True), to_natural(ce, shape), to_natural(d, shape, True)


def assemble_dense(shape, ke, E, mask):
    """Dense constrained matrix M K M + (I - M) in FP64 (src/voxel_mg.py:61-70)."""
    edof = edof_author(shape)
    n = 3 * n_nodes(shape)
    K = np.zeros((n, n))
    E = np.asarray(E, dtype=np.float64)
    for e in range(edof.shape[0]):
        K[np.ix_(edof[e], edof[e])] += E[e] * ke
    m = np.asarray(mask, dtype=np.float64)
    return m[:, None] * K * m[None, :] + np.diag(1.0 - m)


# ------------------------------------------------------------------------------------ transfers
def prolong(uc, coarse_shape):
    """Trilinear prolongation P on (nx+1, ny+1, nz+1, 3) nodal arrays (src/voxel_mg.py:74-80,92-97)."""
    nx, ny, nz = (int(s) for s in coarse_shape)
    v = np.asarray(uc).reshape(nx + 1, ny + 1, nz + 1, 3)
    for axis in range(3):
        n = v.shape[axis]
        shape = list(v.shape)
        shape[axis] = 2 * n - 1
        out = np.empty(shape, dtype=v.dtype)
        even = [slice(None)] * 4
        odd = [slice(None)] * 4
        even[axis] = slice(0, None, 2)
        odd[axis] = slice(1, None, 2)
        lo = [slice(None)] * 4
        hi = [slice(None)] * 4
        lo[axis] = slice(0, n - 1)
        hi[axis] = slice(1, n)
        out[tuple(even)] = v
        out[tuple(odd)] = 0.5 * (v[tuple(lo)] + v[tuple(hi)])
        v = out
    return np.ascontiguousarray(v).ravel()


def restrict(rf, fine_shape):
    """Restriction R = P^T, separable per axis (src/voxel_mg.py:83-89,100-105)."""
    nx, ny, nz = (int(s) for s in fine_shape)
    v = np.asarray(rf).reshape(nx + 1, ny + 1, nz + 1, 3)
    for axis in range(3):
        w = np.moveaxis(v, axis, 0)
        out = w[0::2].copy()
        half = 0.5 * w[1::2]
        out[:-1] += half
        out[1:] += half
        v = np.moveaxis(out, 0, axis)
    return np.ascontiguousarray(v).ravel()


def coarsen_modulus(E, shape):
    """2x2x2 mean of element moduli (src/voxel_mg.py:108-111)."""
    nx, ny, nz = (int(s) for s in shape)
    return np.ascontiguousarray(np.asarray(E).reshape(nx // 2, 2, ny // 2, 2, nz // 2, 2)
                                .mean(axis=(1, 3, 5))).ravel()


def coarsen_mask(mask, shape):
    """Injection of the nodal mask to coarse nodes (src/voxel_mg.py:114-116)."""
    nx, ny, nz = (int(s) for s in shape)
    return np.ascontiguousarray(np.asarray(mask).reshape(nx + 1, ny + 1, nz + 1, 3)[::2, ::2, ::2, :]).ravel()


def hierarchy_shapes(shape, max_coarse_x=16):
    """Halve all axes while x > max_coarse_x and every extent is even (src/voxel_mg.py:220-225)."""
    shapes = [tuple(int(s) for s in shape)]
    while shapes[-1][0] > max_coarse_x and all(s % 2 == 0 for s in shapes[-1]):
        shapes.append(tuple(s // 2 for s in shapes[-1]))
    return shapes


# ------------------------------------------------------------------------------------ multigrid
class Level:
    """One level of the rediscretised hierarchy (src/voxel_mg.py:120-130)."""

    def __init__(self, shape, ke, E, mask, dtype=np.float64):
        self.shape, self.dtype = tuple(shape), dtype
        self.ke = np.asarray(ke, dtype=dtype)
        self.E = np.asarray(E).astype(dtype)
        self.mask = np.asarray(mask).astype(dtype)
        self.fixed = (1 - self.mask).astype(dtype)
        d = product_diagonal(shape, self.ke, self.E, dtype)
        self.inv_diag = (1 / np.where(self.mask != 0, d, dtype(1))).astype(dtype)

    def apply(self, u):
        return product_raw(self.shape, self.ke, u * self.mask, self.E, self.dtype) * self.mask + u * self.fixed


class Multigrid:
    """V(pre, post) cycle with damped Jacobi and a dense coarse solve (src/voxel_mg.py:133-178)."""

    def __init__(self, shapes, ke, E_fine, mask_fine, coarse_factor, dtype=np.float64,
                 pre=4, post=4, omegas=None):
        self.dtype, self.pre, self.post = dtype, pre, post
        self.levels = []
        E, mask = np.asarray(E_fine), np.asarray(mask_fine)
        for i, shape in enumerate(shapes):
            if i:
                E = coarsen_modulus(E, shapes[i - 1])
                mask = coarsen_mask(mask, shapes[i - 1])
            self.levels.append(Level(shape, np.asarray(ke) * 2 ** i, E, mask, dtype))
        self.coarse_factor = np.asarray(coarse_factor).astype(dtype)
        n = len(self.levels) - 1
        self.omegas = list(omegas) if omegas is not None else [0.6] * n

    def coarse_solve(self, r):
        from scipy.linalg import solve_triangular
        y = solve_triangular(self.coarse_factor, r, lower=True)
        return solve_triangular(self.coarse_factor.T, y, lower=False)

    def vcycle(self, r, level=0):
        L = self.levels[level]
        if level == len(self.levels) - 1:
            return self.coarse_solve(r) * L.mask
        w = self.omegas[level]
        x = w * L.inv_diag * r
        for _ in range(self.pre - 1):
            x = x + w * L.inv_diag * (r - L.apply(x))
        res = (r - L.apply(x)) * L.mask
        nxt = self.levels[level + 1]
        rc = restrict(res, L.shape) * nxt.mask
        x = x + prolong(self.vcycle(rc, level + 1), nxt.shape) * L.mask
        for _ in range(self.post):
            x = x + w * L.inv_diag * (r - L.apply(x))
        return x

    def __call__(self, r):
        return self.vcycle(r.astype(self.dtype)).astype(r.dtype)


def coarse_factor(shapes, ke, E_fine, mask_fine):
    """Cholesky factor of the coarsest constrained operator (experiments/session_i/run_gpu.py:278-285)."""
    E, m = np.asarray(E_fine), np.asarray(mask_fine)
    for i in range(1, len(shapes)):
        E, m = coarsen_modulus(E, shapes[i - 1]), coarsen_mask(m, shapes[i - 1])
    A = assemble_dense(shapes[-1], np.asarray(ke) * 2 ** (len(shapes) - 1), E, m)
    return np.linalg.cholesky(A)


def spectral_omegas(levels, iterations=30, seed=20260923):
    """omega_l = 4 / (3 lambda_l), lambda_l by seeded power iteration on D^-1 A over free DOFs
    (src/voxel_mg.py:228-244).  Returns (omegas, lambdas)."""
    omegas, lambdas = [], []
    for L in levels[:-1]:
        rng = np.random.default_rng(seed)
        v = rng.standard_normal(L.mask.size).astype(L.dtype) * L.mask
        v = v / np.linalg.norm(v)
        lam = 0.0
        for _ in range(iterations):
            w = L.inv_diag * L.apply(v) * L.mask
            lam = float(np.linalg.norm(w))
            v = w / lam
        lambdas.append(lam)
        omegas.append(4.0 / (3.0 * lam))
    return omegas, lambdas


def fcg(apply_A, b, precondition, tol, maxiter, check_every=5, fixed_iterations=None):
    """Flexible PCG, Polak-Ribiere beta, FP64 outer, true-residual test with replacement
    (src/voxel_mg.py:181-217).  Returns (x, iterations, converged, rel, matvecs)."""
    nb = float(np.linalg.norm(b))
    x = np.zeros_like(b)
    r = b.copy()
    z = precondition(r)
    p = z.copy()
    rz = float(r @ z)
    matvecs = 0
    limit = maxiter if fixed_iterations is None else fixed_iterations
    it = 0
    for it in range(1, limit + 1):
        q = apply_A(p)
        matvecs += 1
        alpha = rz / float(p @ q)
        x = x + alpha * p
        r_new = r - alpha * q
        if fixed_iterations is None and it % check_every == 0:
            true = b - apply_A(x)
            matvecs += 1
            rel = float(np.linalg.norm(true)) / nb
            if rel <= tol:
                return x, it, True, rel, matvecs
            r_new = true
        z_new = precondition(r_new)
        rz_new = float(r_new @ z_new)
        beta = float(r_new @ (z_new - z)) / rz
        p = z_new + beta * p
        r, z, rz = r_new, z_new, rz_new
    true = b - apply_A(x)
    matvecs += 1
    rel = float(np.linalg.norm(true)) / nb
    return x, it, bool(rel <= tol), rel, matvecs


# ------------------------------------------------------------------------------------ donor PCG
def pcg(matvec, b, M_inv, x0=None, tol=1e-5, maxiter=20000, mask=None, check_every=50):
    """Jacobi-PCG (Fletcher-Reeves beta) with true-residual test and replacement every
    `check_every` iterations (donor simp_r2.py:187-295).  Returns (x, iters, converged, rel)."""
    dt = b.dtype
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=dt)
    if mask is not None:
        x = x * mask
    r = b - matvec(x)
    if mask is not None:
        r = r * mask
    z = M_inv * r
    p = z.copy()
    rz = dt.type(r @ z)
    b_norm = float(np.linalg.norm(b))
    if b_norm <= 0:
        return x, 0, True, 0.0
    tol_abs = tol * b_norm
    r_norm = float(np.linalg.norm(r))
    if r_norm <= tol_abs:
        return x, 0, True, r_norm / b_norm
    k = max(1, int(check_every))
    converged, iters = False, 0
    for _ in range(maxiter):
        Ap = matvec(p)
        if mask is not None:
            Ap = Ap * mask
        pAp = dt.type(p @ Ap)
        if float(pAp) == 0.0:
            break
        alpha = rz / pAp
        x = x + alpha * p
        iters += 1
        if iters % k == 0 or iters >= maxiter:
            r = b - matvec(x)
            if mask is not None:
                r = r * mask
            r_norm = float(np.linalg.norm(r))
            if r_norm <= tol_abs:
                converged = True
                break
        else:
            r = r - alpha * Ap
        z = M_inv * r
        rz_new = dt.type(r @ z)
        beta = rz_new / rz
        p = z + beta * p
        rz = rz_new
    if not converged:
        r = b - matvec(x)
        if mask is not None:
            r = r * mask
        r_norm = float(np.linalg.norm(r))
    return x, iters, converged, r_norm / b_norm


def pcg_ir(matvec64, b64, matvec32, M_inv32, tol=1e-5, mask32=None, inner_tol=1e-1, max_outer=40,
           inner_maxiter=4000, check_every=50, x0=None):
    """Mixed-precision iterative refinement: FP64 residual, scaled FP32 PCG correction, divergence
    guard with undo and tenfold tighter inner tolerance (donor simp_r2.py:298-385).
    Returns (x, outer, inner_total, converged, rel)."""
    nb = float(np.linalg.norm(b64))
    if nb <= 0:
        return np.zeros_like(b64), 0, 0, True, 0.0
    x = np.zeros_like(b64) if x0 is None else np.array(x0, dtype=np.float64)
    inner_total, outer = 0, 0
    tol_in, rel_prev, d_last, scale_last = inner_tol, None, None, 0.0
    for outer in range(1, max_outer + 1):
        r = b64 - matvec64(x)
        rel = float(np.linalg.norm(r)) / nb
        if rel <= tol:
            return x, outer - 1, inner_total, True, rel
        if rel_prev is not None and rel > rel_prev and d_last is not None:
            x = x - d_last.astype(np.float64) * scale_last
            d_last = None
            tol_in *= 0.1
            if tol_in < 1e-5:
                return x, outer, inner_total, False, rel_prev
            continue
        rel_prev = rel
        scale = float(np.linalg.norm(r))
        d32, it32, _, _ = pcg(matvec32, (r / scale).astype(np.float32), M_inv32, tol=tol_in,
                              maxiter=inner_maxiter, mask=mask32, check_every=check_every)
        inner_total += it32
        d_last, scale_last = d32, scale
        x = x + d32.astype(np.float64) * scale
    r = b64 - matvec64(x)
    rel = float(np.linalg.norm(r)) / nb
    return x, outer, inner_total, bool(rel <= tol), rel


# ------------------------------------------------------------------------------------ SIMP
def cone_stencil(x, shape, rmin):
    """y_e = sum_{|d| < rmin} (rmin - |d|) x_{e+d} over in-grid neighbours, author element order
    (donor filter_r2.py:40-76; support R = ceil(rmin) - 1, filter_r2.py:119-124)."""
    nx, ny, nz = (int(s) for s in shape)
    R = max(0, int(math.ceil(rmin)) - 1)
    xv = np.asarray(x, dtype=np.float64).reshape(nx, ny, nz)
    y = np.zeros_like(xv)
    for dx in range(-R, R + 1):
        for dy in range(-R, R + 1):
            for dz in range(-R, R + 1):
                w = rmin - math.sqrt(dx * dx + dy * dy + dz * dz)
                if w <= 0:
                    continue
                dst = tuple(slice(max(0, -d), n - max(0, d)) for d, n in zip((dx, dy, dz), (nx, ny, nz)))
                src = tuple(slice(max(0, d), n - max(0, -d)) for d, n in zip((dx, dy, dz), (nx, ny, nz)))
                y[dst] += w * xv[src]
    return y.ravel()


class ConeFilter:
    """Hat density filter: forward H rho / s, transpose H (g / s) (donor filter_r2.py:93-171;
    same operator as the CSR DensityFilter of experiments/session_h/run_w1b.py:97-125)."""

    def __init__(self, shape, rmin):
        self.shape, self.rmin = tuple(int(s) for s in shape), float(rmin)
        self.s = cone_stencil(np.ones(int(np.prod(self.shape))), self.shape, self.rmin)

    def forward(self, rho):
        return cone_stencil(rho, self.shape, self.rmin) / self.s

    def transpose(self, g):
        return cone_stencil(np.asarray(g) / self.s, self.shape, self.rmin)


def oc_top88(x, dc, dv, volfrac, move, density=None, l2=1e9, tol=1e-3):
    """top88 optimality-criteria update with relative bisection on the multiplier; the volume is
    measured on density(x_new) (experiments/session_h/run_w1b.py:46-62)."""
    density = density or (lambda v: v)
    l1 = 0.0
    x_new = x
    while (l2 - l1) / (l1 + l2) > tol:
        lmid = 0.5 * (l2 + l1)
        x_new = np.clip(x * np.sqrt(np.maximum(-dc / dv / lmid, 0.0)),
                        np.maximum(x - move, 0.0), np.minimum(x + move, 1.0))
        if density(x_new).mean() > volfrac:
            l1 = lmid
        else:
            l2 = lmid
    return x_new


# ------------------------------------------------------------------------------------ problems
def cantilever_equal_split(shape):
    """Clamped x=0 face; total load -1 in z split equally over the nodes (ix=nx, iy=0..ny, iz=0).
    Author layout.  Restates the synthetic smoke case of tests/test_mg_cpu.py:140-155."""
    nx, ny, nz = (int(s) for s in shape)
    mask = np.ones((nx + 1, ny + 1, nz + 1, 3))
    mask[0] = 0.0
    force = np.zeros((nx + 1, ny + 1, nz + 1, 3))
    force[nx, :, 0, 2] = -1.0 / (ny + 1)
    return mask.ravel(), force.ravel()


def cantilever_line_load(shape):
    """Clamped x=0 face and consistent line load (-1/ny interior, -1/(2 ny) ends) along y at
    x=nx, z=0, natural layout (experiments/session_i/make_inputs.py:31-39)."""
    nx, ny, nz = (int(s) for s in shape)
    mask = np.ones((nz + 1, ny + 1, nx + 1, 3))
    mask[:, :, 0, :] = 0.0
    force = np.zeros((nz + 1, ny + 1, nx + 1, 3))
    line = np.full(ny + 1, -1.0 / ny)
    line[[0, -1]] = -0.5 / ny
    force[0, :, nx, 2] = line
    return mask.ravel(), force.ravel()


def upsample(rho_natural, shape, factor):
    """Nearest-neighbour repeat of a natural-layout element field (experiments/session_i/make_inputs.py:42-50)."""
    nx, ny, nz = (int(s) for s in shape)
    r = np.asarray(rho_natural).reshape(nz, ny, nx)
    for axis in range(3):
        r = np.repeat(r, factor, axis=axis)
    return np.ascontiguousarray(r.ravel()), (nx * factor, ny * factor, nz * factor)


def gaussian_random_field(shape, ell, seed):
    """Seeded GRF density in [1e-3, 1] (author element layout): white noise smoothed by
    exp(-2 pi^2 ell^2 |k|^2) in Fourier space, standardised, then a logistic map.
    This is the synthetic-input recipe for the GMG workloads (no reference counterpart)."""
    nx, ny, nz = (int(s) for s in shape)
    w = np.random.default_rng(seed).standard_normal((nx, ny, nz))
    kx, ky, kz = np.meshgrid(np.fft.fftfreq(nx), np.fft.fftfreq(ny), np.fft.fftfreq(nz), indexing="ij")
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * np.exp(-2 * np.pi ** 2 * ell ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))))
    g = (g - g.mean()) / g.std()
    return (1e-3 + (1 - 1e-3) / (1 + np.exp(-g))).ravel()


def simp_top88(shape, x, steps, volfrac, rmin, move, emin=1e-9, penal=3.0, oc_tol=1e-6, solve=None):
    """Density-filtered SIMP with the top88 OC (experiments/session_h/run_w1b.py:163-205, update
    'top88'): rho = H x / s; solve K(E(rho)) u = f; dc = -p rho^(p-1)(1-emin) u_e^T ke u_e;
    dc_x = H(dc / s), dv_x = H(1 / s); x <- oc_top88(x, dc_x, dv_x, volfrac, move, density).
    `solve(E) -> u` must return the displacement for modulus E.  Returns (x, rho, compliances)."""
    ke = quadrature([1, 1, 1], 0.3)
    filt = ConeFilter(shape, rmin)
    mask, force = cantilever_equal_split(shape)
    rho = filt.forward(x)
    dv_x = filt.transpose(np.ones_like(x))
    comps = []
    for _ in range(steps):
        E = simp_modulus(rho, emin, 1.0, penal)
        u = solve(E)
        comps.append(float(force @ u))
        ce = element_energy(shape, ke, u)
        dc = -penal * rho ** (penal - 1) * (1 - emin) * ce
        dc_x = filt.transpose(dc)
        x = oc_top88(x, dc_x, dv_x, volfrac, move, density=filt.forward, tol=oc_tol)
        rho = filt.forward(x)
    return x, rho, comps
