"""Drop-in mirror of the reference's src/voxel_mg.py over torch CUDA tensors.

Same names, arguments and return values as the reference module (src/voxel_mg.py:32-244); the
`xp` argument is accepted and ignored (the reference passed numpy or cupy).  Vectors are CUDA
tensors in author layout; masks are the reference's 0/1 DOF masks (3N floats) -- the node masks
the kernels use are derived from them.  Every product and transfer runs in libvoxel_b200.

Two routes.  Any callable `apply_A` / `precondition` runs the reference's host-driven loop (its
control flow and host synchronisations), so a caller can switch without changing code.  When
`fcg` receives a Dirichlet apply this module can see into -- `dirichlet(product, E, mask)` (the
reference's `lambda u: P.raw(u * mask, E) * mask + u * (1 - mask)`) or a `Level.apply` -- and a
`Multigrid` built from voxel_b200 Products, the solve runs on voxel_b200.solver's FCGSolver
instead: fused CG kernels, device scalars and the whole loop in one CUDA-graph launch, with the
same iterates.  `Multigrid.coarse_solve` applies the inverse Cholesky factor with two
bandwidth-bound triangular passes (no library call).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .element import XYZ  # noqa: F401  (re-exported like the reference's XYZ)
from .layout import edof_author  # noqa: F401
from .operators import PREC, Product, VoxelOperator, _ptr, node_mask_from_dofs, stream_ptr
from .solver import FCGSolver, MGHierarchy, _lower_inverse, hierarchy_shapes  # noqa: F401



def _t(a, dtype=None):
    if isinstance(a, torch.Tensor):
        t = a if a.is_cuda else a.cuda()
    else:
        t = torch.as_tensor(np.asarray(a), device="cuda")
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def _node_mask(mask, shape):
    m = _t(mask)
    if m.dtype == torch.uint8 and m.numel() == (shape[0] + 1) * (shape[1] + 1) * (shape[2] + 1):
        return m
    return node_mask_from_dofs(m.to(torch.float64))


def assemble_dense(shape, ke, E, mask):
    """Dense constrained matrix M K M + (I - M) in FP64 on the device (src/voxel_mg.py:61-70)."""
    shape = tuple(int(s) for s in shape)
    n = 3 * (shape[0] + 1) * (shape[1] + 1) * (shape[2] + 1)
    A = torch.empty(n, n, dtype=torch.float64, device="cuda")
    _lib.call("vx_assemble_dense", *shape, _lib.dptr(np.ascontiguousarray(np.asarray(ke, dtype=np.float64))),
              _ptr(_t(E, torch.float64), "E"), _ptr(_node_mask(mask, shape), "mask"), A.data_ptr(), stream_ptr())
    return A


def prolong(xp, uc, coarse_shape):
    """Trilinear prolongation P (src/voxel_mg.py:92-97)."""
    nx, ny, nz = (int(s) for s in coarse_shape)
    uc = _t(uc)
    fine = (2 * nx, 2 * ny, 2 * nz)
    out = torch.zeros(3 * (fine[0] + 1) * (fine[1] + 1) * (fine[2] + 1), dtype=uc.dtype, device="cuda")
    _lib.call("vx_prolong_add", PREC[uc.dtype], *fine, _ptr(uc, "uc"), None, out.data_ptr(), stream_ptr())
    return out


def restrict(xp, rf, fine_shape):
    """Restriction R = P^T (src/voxel_mg.py:100-105)."""
    fine = tuple(int(s) for s in fine_shape)
    rf = _t(rf)
    c = (fine[0] // 2, fine[1] // 2, fine[2] // 2)
    out = torch.empty(3 * (c[0] + 1) * (c[1] + 1) * (c[2] + 1), dtype=rf.dtype, device="cuda")
    _lib.call("vx_restrict", PREC[rf.dtype], *fine, _ptr(rf, "rf"), None, out.data_ptr(), stream_ptr())
    return out


def coarsen_modulus(xp, E, shape):
    """2x2x2 mean of element moduli (src/voxel_mg.py:108-111)."""
    shape = tuple(int(s) for s in shape)
    E = _t(E)
    out = torch.empty(E.numel() // 8, dtype=E.dtype, device="cuda")
    _lib.call("vx_coarsen_modulus", PREC[E.dtype], *shape, _ptr(E, "E"), out.data_ptr(), stream_ptr())
    return out


def coarsen_mask(xp, mask, shape):
    """Injection of the nodal DOF mask (src/voxel_mg.py:114-116); node masks (uint8) stay node masks."""
    nx, ny, nz = (int(s) for s in shape)
    m = _t(mask)
    if m.dtype == torch.uint8:
        out = torch.empty((nx // 2 + 1) * (ny // 2 + 1) * (nz // 2 + 1), dtype=torch.uint8, device="cuda")
        _lib.call("vx_coarsen_mask", nx, ny, nz, _ptr(m, "mask"), out.data_ptr(), stream_ptr())
        return out
    return m.reshape(nx + 1, ny + 1, nz + 1, 3)[::2, ::2, ::2, :].contiguous().reshape(-1)


class Level:
    """One level: E, mask, fixed = 1 - mask, inv_diag and the Dirichlet apply (src/voxel_mg.py:120-130)."""

    def __init__(self, xp, shape, product, E, mask, dtype):
        self.xp, self.shape, self.product, self.dtype = xp, tuple(shape), product, dtype
        self.E = _t(E, dtype)
        self.mask = _t(mask, dtype)
        self.fixed = (1 - self.mask).to(dtype)
        self.node_mask = _node_mask(mask, self.shape)
        d = product.diagonal(self.E)
        one = torch.ones((), dtype=dtype, device="cuda")
        self.inv_diag = (1 / torch.where(self.mask != 0, d, one)).to(dtype)
        self.op = product.op if isinstance(product, Product) else None

    def apply(self, u):
        if self.op is not None:
            return self.op.matvec(u.contiguous(), self.E, self.node_mask)
        return self.product.raw(u * self.mask, self.E) * self.mask + u * self.fixed


class Dirichlet:
    """u -> M K(E) (M u) + (I - M) u for a voxel_b200 Product: the reference's outer operator
    `lambda u: P.raw(u * mask, E) * mask + u * (1 - mask)` (experiments/session_i/run_gpu.py:304) as an
    object that fcg can recognise and run on the device solver."""

    def __init__(self, product, E, mask):
        if not isinstance(product, Product):
            raise ValueError("dirichlet() needs a voxel_b200 Product")
        self.product, self.op = product, product.op
        self.E = _t(E, product.dtype)
        self.mask = _t(mask)
        self.node_mask = _node_mask(mask, product.shape)

    def __call__(self, u):
        return self.op.matvec(u.contiguous(), self.E, self.node_mask)


def dirichlet(product, E, mask):
    """The Dirichlet apply of `product` (see Dirichlet)."""
    return Dirichlet(product, E, mask)


class Multigrid:
    """V-cycle preconditioner (src/voxel_mg.py:133-178).  `products` are per-level product objects
    (finest first) exposing raw(u, E) and diagonal(E); `coarse_factor` is the lower Cholesky factor
    of the coarsest constrained matrix.  With voxel_b200 Products each smoothing step is one fused
    kernel (x + w D^-1 (r - A x)); with other products the reference's composition is used."""

    def __init__(self, xp, shapes, products, E_fine, mask_fine, coarse_factor, dtype,
                 pre=4, post=4, omegas=None):
        self.xp, self.dtype, self.pre, self.post = xp, dtype, pre, post
        self.levels = []
        E, mask = _t(E_fine), _t(mask_fine)
        for i, (shape, prod) in enumerate(zip(shapes, products)):
            if i:
                E = coarsen_modulus(xp, E, shapes[i - 1])
                mask = coarsen_mask(xp, mask, shapes[i - 1])
            self.levels.append(Level(xp, shape, prod, E, mask, dtype))
        self.coarse_factor = _t(coarse_factor, dtype)
        n_smooth = len(self.levels) - 1
        self.omegas = list(omegas) if omegas is not None else [0.6] * n_smooth
        assert len(self.omegas) == n_smooth
        # the coarse solve: L^-1 of the FP64 factor packed with its transpose (two triangular passes),
        # formed by the library from the caller's banded factor
        f64 = _t(coarse_factor, torch.float64).contiguous()
        n = f64.shape[0]
        cs = [int(v) for v in shapes[-1]]
        bw = min(n - 1, 3 * ((cs[1] + 1) * (cs[2] + 1) + (cs[2] + 1) + 1) + 2)
        self._packed = torch.empty_like(f64)
        work = torch.empty(int(_lib.load().vx_coarse_factor_workspace(n, bw)), dtype=torch.float64, device="cuda")
        _lib.call("vx_coarse_pack_factor", n, bw, f64.data_ptr(), self._packed.data_ptr(), work.data_ptr(),
                  stream_ptr())
        self._coarse_y = torch.empty(n, dtype=torch.float64, device="cuda")
        # what the device route needs: FP64 finest modulus, products of one element matrix ke * 2^l
        self._shapes = [tuple(int(v) for v in sh) for sh in shapes]
        self._E64 = _t(E_fine, torch.float64)
        self._node_mask = self.levels[0].node_mask
        ok = all(isinstance(p, Product) for p in products) and dtype in (torch.float32, torch.float64)
        if ok:
            ke0 = products[0].op.ke
            ok = all(np.allclose(p.op.ke, ke0 * 2 ** l, rtol=1e-15, atol=0) for l, p in enumerate(products))
        self._ke0 = products[0].op.ke if ok else None
        self._device = {}

    def coarse_solve(self, r):
        """A_c^-1 r from the packed inverse factor (the reference's two triangular solves)."""
        r = r.contiguous()
        z = torch.empty_like(r)
        prec = _lib.VX_F64 if r.dtype == torch.float64 else _lib.VX_F32
        _lib.call("vx_coarse_apply_factor", prec, r.numel(), self._packed.data_ptr(), _ptr(r, "r"), None,
                  self._coarse_y.data_ptr(), z.data_ptr(), stream_ptr())
        return z

    def device_solver(self, op64, E64, node_mask, tol, maxiter, check_every, fixed_iterations):
        """The FCGSolver over this hierarchy's data (cached per outer operator and settings), or None
        when the hierarchy was not built from voxel_b200 Products of one element matrix."""
        if self._ke0 is None:
            return None
        key = (id(op64), E64.data_ptr(), float(tol), int(maxiter), int(check_every), fixed_iterations)
        s = self._device.get(key)
        if s is None:
            if "M" not in self._device:
                self._device["M"] = MGHierarchy(self._shapes[0], self._ke0, self._E64, self._node_mask, self.dtype,
                                                self.pre, self.post, list(self.omegas), shapes=self._shapes)
            s = FCGSolver(op64, E64, node_mask, self._device["M"], tol=tol, maxiter=maxiter,
                          check_every=check_every, fixed_iterations=fixed_iterations)
            self._device[key] = s
        self._device["M"].set_omegas(list(self.omegas))
        return s

    def _sweep(self, L, x, r, w):
        if L.op is not None:
            return L.op.jacobi(x.contiguous(), r.contiguous(), L.inv_diag, L.E, L.node_mask, w)
        return x + w * L.inv_diag * (r - L.apply(x))

    def vcycle(self, r, level=0):
        L = self.levels[level]
        if level == len(self.levels) - 1:
            return self.coarse_solve(r) * L.mask
        w = self.omegas[level]
        x = w * L.inv_diag * r
        for _ in range(self.pre - 1):
            x = self._sweep(L, x, r, w)
        if L.op is not None:
            res = L.op.residual(x.contiguous(), r.contiguous(), L.E, L.node_mask)
        else:
            res = (r - L.apply(x)) * L.mask
        nxt = self.levels[level + 1]
        rc = restrict(self.xp, res, L.shape) * nxt.mask
        x = x + prolong(self.xp, self.vcycle(rc, level + 1), nxt.shape) * L.mask
        for _ in range(self.post):
            x = self._sweep(L, x, r, w)
        return x

    def __call__(self, r):
        return self.vcycle(r.to(self.dtype)).to(r.dtype)


def _outer(apply_A):
    """(op64, E64, node_mask) of an apply this module can see into, else None."""
    if isinstance(apply_A, Dirichlet):
        src = apply_A
    elif isinstance(getattr(apply_A, "__self__", None), Level) and getattr(apply_A, "__func__", None) is Level.apply:
        src = apply_A.__self__
    else:
        return None
    if src.op is None or src.op.dtype != torch.float64:
        return None
    return src.op, src.E, src.node_mask


def fcg(xp, apply_A, b, precondition, tol, maxiter, check_every=5, fixed_iterations=None):
    """Flexible PCG (Polak-Ribiere beta), FP64 outer, true-residual stopping test with residual
    replacement (src/voxel_mg.py:181-217).  Returns (x, iterations, converged, rel, matvecs).
    A `dirichlet(...)` / `Level.apply` outer operator with a voxel_b200 Multigrid runs on the
    device solver (same iterates; see the module docstring)."""
    outer = _outer(apply_A)
    if outer is not None and isinstance(precondition, Multigrid) and b.dtype == torch.float64:
        s = precondition.device_solver(*outer, tol, maxiter, check_every, fixed_iterations)
        if s is not None:
            x, it, ok, rel, mv = s.solve(b.contiguous())
            return x.clone(), it, ok, rel, mv
    nb = float(torch.linalg.vector_norm(b))
    x = torch.zeros_like(b)
    r = b.clone()
    z = precondition(r)
    p = z.clone()
    rz = float(r @ z)
    matvecs = 0
    limit = fixed_iterations if fixed_iterations is not None else maxiter
    it = 0
    for it in range(1, limit + 1):
        q = apply_A(p)
        matvecs += 1
        pq = float(p @ q)
        alpha = rz / pq
        x = x + alpha * p
        r_new = r - alpha * q
        if fixed_iterations is None and it % check_every == 0:
            true = b - apply_A(x)
            matvecs += 1
            rel = float(torch.linalg.vector_norm(true)) / nb
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
    rel = float(torch.linalg.vector_norm(true)) / nb
    return x, it, bool(rel <= tol), rel, matvecs


def spectral_omegas(xp, levels, iterations=30, seed=20260923):
    """omega_l = 4 / (3 lambda_l) from a seeded power iteration on D^-1 A over free DOFs
    (src/voxel_mg.py:228-244).  Returns (omegas, lambdas)."""
    omegas, lambdas = [], []
    for L in levels[:-1]:
        rng = np.random.default_rng(seed)
        v = torch.as_tensor(rng.standard_normal(L.mask.numel()), device="cuda").to(L.dtype) * L.mask
        v = v / torch.linalg.vector_norm(v)
        lam = 0.0
        for _ in range(iterations):
            w = L.inv_diag * L.apply(v) * L.mask
            lam = float(torch.linalg.vector_norm(w))
            v = w / lam
        lambdas.append(lam)
        omegas.append(4.0 / (3.0 * lam))
    return omegas, lambdas
