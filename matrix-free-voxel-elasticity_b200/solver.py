"""Device-resident solvers: the rediscretised GMG V-cycle, flexible (Polak-Ribiere) PCG with an
FP64 outer loop, the donor's Jacobi-PCG (Fletcher-Reeves) and mixed-precision iterative
refinement.

Semantics follow the reference exactly -- src/voxel_mg.py:133-217 (Multigrid, fcg) and
experiments/session_a/donor/src/gpu_fem/simp_r2.py:187-385 (pcg, pcg_ir) -- but every scalar
lives on the device (a 16-slot FP64 array S), every reduction is deterministic, and the loop
body is captured once as the body of a CUDA-graph WHILE node, so a whole solve is one graph
launch with no host round trip per iteration (`graph=False` runs the same kernel sequence from
the host, one iteration at a time).
"""
from __future__ import annotations

import atexit
import ctypes
import sys
import weakref
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .operators import PREC, STORAGE, VoxelOperator, _ptr, stream_ptr

# scalar slots of S (csrc/vx_solver.cu)
(S_RZ, S_PQ, S_ALPHA, S_RR, S_REL, S_NB, S_BETA, S_RZN, S_RZD, S_TOL, S_DONE, S_IT, S_MAXIT, S_MV,
 S_BREAK, S_CHECK) = range(16)
FIN_PQ, FIN_TRUE, FIN_BETA_PR, FIN_BETA_FR, FIN_NB, FIN_RZ, FIN_RR_ONLY = range(7)

def hierarchy_shapes(shape, max_coarse_x=16):
    """Halve every axis while x > max_coarse_x and all extents are even (src/voxel_mg.py:220-225)."""
    shapes = [tuple(int(s) for s in shape)]
    while shapes[-1][0] > max_coarse_x and all(s % 2 == 0 for s in shapes[-1]):
        shapes.append(tuple(s // 2 for s in shapes[-1]))
    return shapes


def _s():
    return stream_ptr()


def all_free_mask(shape, device="cuda"):
    nx, ny, nz = shape
    return torch.full(((nx + 1) * (ny + 1) * (nz + 1),), 7, dtype=torch.uint8, device=device)


class _Level:
    __slots__ = ("shape", "op", "op64", "E64", "E", "mask", "invd", "omega", "r", "x", "xt", "res", "n")


def _lower_inverse(L: torch.Tensor, leaf: int = 2048) -> torch.Tensor:
    """L^-1 of a lower-triangular FP64 matrix by recursive halving:
    [[A, 0], [B, C]]^-1 = [[A^-1, 0], [-C^-1 B A^-1, C^-1]]; blocks of at most `leaf` rows are
    inverted by a triangular solve.  About n^3/3 multiply-adds, nearly all in matrix products."""
    n = L.shape[0]
    if n <= leaf:
        eye = torch.eye(n, dtype=L.dtype, device=L.device)
        return torch.linalg.solve_triangular(L, eye, upper=False).contiguous()
    h = n // 2
    out = torch.zeros((n, n), dtype=L.dtype, device=L.device)       # row-major, whatever L's layout
    ai = _lower_inverse(L[:h, :h], leaf)
    ci = _lower_inverse(L[h:, h:], leaf)
    out[:h, :h] = ai
    out[h:, h:] = ci
    out[h:, :h] = -(ci @ (L[h:, :h] @ ai))
    return out


class MGHierarchy:
    """Rediscretised geometric multigrid (src/voxel_mg.py:1-21,74-178): level l has element matrix
    ke * 2^l, modulus the 2x2x2 mean of level l-1, mask injected from level l-1; damped Jacobi
    V(pre, post) in `dtype` (float64 or float32); the coarsest level is solved in FP64 with the
    inverse Cholesky factor of its dense constrained matrix (two triangular passes per cycle, the
    reference's two triangular solves).

    BF16 storage (no reference counterpart), FP32 arithmetic in both: aux_dtype=bfloat16 stores the
    level moduli and the auxiliary vectors (right-hand sides, residuals, inverse diagonals) in bf16
    and keeps the iterates in `dtype` float32; dtype=bfloat16 stores the iterates in bf16 too.  The
    coarsest solve accumulates in FP64 either way."""

    def __init__(self, shape, ke, E, node_mask=None, dtype=torch.float32, pre=2, post=2, omegas=None,
                 max_coarse_x=16, shapes=None, aux_dtype=None, coarse_blocks=None):
        """coarse_blocks = B: the grid is B jobs stacked along x with one zero-modulus element layer
        between neighbours at the coarsest level (see batch.BatchedSolver); the coarsest level is then
        B independent dense systems, each with its own factor, solved by one batched launch."""
        aux_dtype = dtype if aux_dtype is None else aux_dtype
        if (dtype, aux_dtype) not in STORAGE:
            raise ValueError(f"unsupported V-cycle storage: iterate {dtype}, auxiliary {aux_dtype}")
        self.shapes = [tuple(s) for s in (shapes or hierarchy_shapes(shape, max_coarse_x))]
        self.dtype, self.aux_dtype = dtype, aux_dtype
        self.prec, self.pre, self.post = STORAGE[(dtype, aux_dtype)], int(pre), int(post)
        self.ke = np.asarray(ke, dtype=np.float64).reshape(24, 24)
        E64 = E.to(torch.float64).contiguous()
        mask = node_mask if node_mask is not None else all_free_mask(self.shapes[0])
        self.levels = []
        for i, s in enumerate(self.shapes):
            if i:
                prev = self.shapes[i - 1]
                Ec = torch.empty(s[0] * s[1] * s[2], dtype=torch.float64, device="cuda")
                _lib.call("vx_coarsen_modulus", _lib.VX_F64, *prev, _ptr(E64, "E"), Ec.data_ptr(), _s())
                mc = torch.empty((s[0] + 1) * (s[1] + 1) * (s[2] + 1), dtype=torch.uint8, device="cuda")
                _lib.call("vx_coarsen_mask", *prev, _ptr(mask, "mask"), mc.data_ptr(), _s())
                E64, mask = Ec, mc
            L = _Level()
            L.shape = s
            L.op = VoxelOperator(s, self.ke * 2 ** i, dtype, aux_dtype)
            L.op64 = L.op if dtype == torch.float64 else VoxelOperator(s, self.ke * 2 ** i, torch.float64)
            L.E64, L.mask = E64, mask
            L.E = E64 if aux_dtype == torch.float64 else E64.to(aux_dtype)
            inv64 = L.op64.diagonal(E64, mask, inverse=True)
            L.invd = inv64 if aux_dtype == torch.float64 else inv64.to(aux_dtype)
            L.n = L.op.ndof
            L.r = torch.zeros(L.n, dtype=aux_dtype, device="cuda")
            L.x = torch.zeros(L.n, dtype=dtype, device="cuda")
            L.xt = torch.zeros(L.n, dtype=dtype, device="cuda")
            # the residual goes to the free iterate buffer when both have one storage type
            L.res = None if aux_dtype == dtype else torch.zeros(L.n, dtype=aux_dtype, device="cuda")
            self.levels.append(L)
        c = self.levels[-1]
        self.blocks = int(coarse_blocks) if coarse_blocks else 0
        if self.blocks:
            nxc, nyc, nzc = c.shape
            if (nxc + 1) % self.blocks:
                raise ValueError(f"coarsest grid {c.shape} does not split into {self.blocks} jobs")
            pc = (nxc + 1) // self.blocks                       # job pitch: nx_job + 1 separator element
            self.job_coarse = (pc - 1, nyc, nzc)
            nb_ = 3 * pc * (nyc + 1) * (nzc + 1)
            self.A_coarse = torch.empty(self.blocks, nb_, nb_, dtype=torch.float64, device="cuda")
            self._coarse_y = torch.zeros(self.blocks * nb_, dtype=torch.float64, device="cuda")
            self.coarse_packed = torch.empty_like(self.A_coarse)
            self._factor_info = torch.zeros(self.blocks, dtype=torch.int32, device="cuda")
            for k in range(self.blocks):
                self._assemble_block(k)
        else:
            A = torch.empty(c.n, c.n, dtype=torch.float64, device="cuda")
            _lib.call("vx_assemble_dense", *c.shape, _lib.dptr(np.ascontiguousarray(self.ke * 2 ** (len(self.shapes) - 1))),
                      _ptr(c.E64, "E"), _ptr(c.mask, "mask"), A.data_ptr(), _s())
            self.A_coarse = A
            self.coarse_packed = torch.empty_like(A)              # tril(L^-1) + triu(L^-T, 1)
            self._coarse_y = torch.zeros(c.n, dtype=torch.float64, device="cuda")
        # the same calls as update_modulus, so a refreshed pooled hierarchy and a fresh one are
        # bitwise identical; the factorisation is checked once here (the check synchronises)
        info = self._coarse_inverse()
        if int(info.abs().max()) != 0:
            raise ValueError(f"coarsest-level matrix is not positive definite (cholesky info {info.tolist()})")
        n_smooth = len(self.levels) - 1
        if omegas is None:
            self.omegas = [0.6] * n_smooth                      # the reference default (voxel_mg.py:148)
            self.lambdas = None
        elif isinstance(omegas, str) and omegas == "spectral":
            self.omegas, self.lambdas = self.spectral_omegas()
        elif np.isscalar(omegas):
            self.omegas, self.lambdas = [float(omegas)] * n_smooth, None
        else:
            self.omegas, self.lambdas = [float(w) for w in omegas], None
        self.set_omegas(self.omegas)

    def set_omegas(self, omegas):
        n_smooth = len(self.levels) - 1
        if len(omegas) != n_smooth:
            raise ValueError(f"need {n_smooth} omegas, got {len(omegas)}")
        self.omegas = [float(w) for w in omegas]
        for L, w in zip(self.levels, self.omegas + [0.0]):
            L.omega = w

    @property
    def finest(self):
        return self.levels[0]

    def update_mask(self):
        """Re-inject the coarse levels' node masks from the finest one (after the finest mask tensor
        was rewritten in place); update_modulus must follow, as the diagonals and the coarsest
        matrix depend on the masks."""
        for i in range(1, len(self.levels)):
            prev, L = self.levels[i - 1], self.levels[i]
            _lib.call("vx_coarsen_mask", *prev.shape, prev.mask.data_ptr(), L.mask.data_ptr(), _s())

    def update_modulus(self, E):
        """New finest modulus (FP64, same grid): refresh every level's moduli, inverse diagonal and
        the coarsest inverse factor IN PLACE, so captured graphs that use this hierarchy stay valid."""
        L0 = self.levels[0]
        if E.data_ptr() != L0.E64.data_ptr():
            L0.E64.copy_(E)
        self.refresh_levels()
        c = self.levels[-1]
        if self.blocks:
            for k in range(self.blocks):
                self._assemble_block(k)
        else:
            _lib.call("vx_assemble_dense", *c.shape, _lib.dptr(np.ascontiguousarray(self.ke * 2 ** (len(self.shapes) - 1))),
                      c.E64.data_ptr(), c.mask.data_ptr(), self.A_coarse.data_ptr(), _s())
        # no error check here (it would synchronise the stream); a non-SPD coarse matrix shows up as a
        # non-finite residual and a non-converged solve
        self._coarse_inverse()

    def refresh_levels(self):
        """Every level's moduli (coarsened from the finest), their narrow copies and the inverse
        diagonals, one launch each per level (in place)."""
        for i, L in enumerate(self.levels):
            if i:
                prev = self.levels[i - 1]
                _lib.call("vx_coarsen_modulus", _lib.VX_F64, *prev.shape, prev.E64.data_ptr(), L.E64.data_ptr(), _s())
            if L.E.data_ptr() != L.E64.data_ptr():
                L.E.copy_(L.E64)
            inv64 = L.op64.diagonal(L.E64, L.mask, inverse=True)
            L.invd.copy_(inv64)

    def _assemble_block(self, k):
        """Coarsest dense matrix of stacked job k (from its own segment of the coarsest moduli and mask)."""
        c = self.levels[-1]
        nx, ny, nz = self.job_coarse
        pc = nx + 1
        E_off = k * pc * ny * nz
        m_off = k * pc * (ny + 1) * (nz + 1)
        _lib.call("vx_assemble_dense", nx, ny, nz, _lib.dptr(np.ascontiguousarray(self.ke * 2 ** (len(self.shapes) - 1))),
                  c.E64.data_ptr() + 8 * E_off, c.mask.data_ptr() + m_off, self.A_coarse[k].data_ptr(), _s())

    def refresh_block(self, k):
        """Re-assemble and re-factor stacked job k's coarsest system (after its moduli changed)."""
        self.refresh_blocks([k])

    def refresh_blocks(self, ks, assemble=True):
        """Re-assemble (optionally) and re-factor the coarsest systems of stacked jobs ks, the
        factorisations side by side in the same launches (vx_batch_coarse_factor)."""
        ks = [int(k) for k in ks]
        if not ks:
            return
        if assemble:
            for k in ks:
                self._assemble_block(k)
        n = self.A_coarse.shape[1]
        nx, ny, nz = self.job_coarse
        bw = min(n - 1, 3 * ((ny + 1) * (nz + 1) + (nz + 1) + 1) + 2)
        ws = int(_lib.load().vx_coarse_factor_workspace(n, bw))
        if getattr(self, "_factor_work", None) is None or self._factor_work.numel() < ws * min(len(ks), 64):
            self._factor_work = torch.empty(ws * min(self.blocks, 64), dtype=torch.float64, device="cuda")
        slots = (ctypes.c_int * len(ks))(*ks)
        _lib.call("vx_batch_coarse_factor", n, bw, len(ks), slots, self.A_coarse.data_ptr(),
                  self.coarse_packed.data_ptr(), self._factor_work.data_ptr(), self._factor_info.data_ptr(), _s())

    def _coarse_inverse(self):
        """Factor the coarsest matrix A = L L^T (FP64 Cholesky) and pack L^-1 with its transpose for
        vx_coarse_apply_factor.  The matrix is banded (a node couples to its 27 neighbours), so
        vx_coarse_factor factors the band and forms L^-1 by banded forward substitution in the
        library's own kernels.  A coarsest grid too wide for that kernel's shared-memory window takes
        a dense Cholesky and a recursive block inversion instead.  Everything is queued on the current
        stream without a host synchronisation.  Returns the factorisation's device-side info tensor
        (0 when A is positive definite)."""
        if self.blocks:
            self.refresh_blocks(range(self.blocks), assemble=False)
            return self._factor_info
        n = self.A_coarse.shape[0]
        nx, ny, nz = self.levels[-1].shape
        bw = min(n - 1, 3 * ((ny + 1) * (nz + 1) + (nz + 1) + 1) + 2)
        if getattr(self, "_factor_work", None) is None:
            need = int(_lib.load().vx_coarse_factor_workspace(n, bw))
            self._factor_work = torch.empty(max(need, 1), dtype=torch.float64, device="cuda")
            self._factor_info = torch.zeros(1, dtype=torch.int32, device="cuda")
        try:
            _lib.call("vx_coarse_factor", n, bw, self.A_coarse.data_ptr(), self.coarse_packed.data_ptr(),
                      self._factor_work.data_ptr(), self._factor_info.data_ptr(), _s())
            return self._factor_info
        except ValueError as e:
            if "too wide" not in str(e):
                raise
        factor, info = torch.linalg.cholesky_ex(self.A_coarse)
        linv = _lower_inverse(factor).contiguous()                  # the kernel reads it row-major
        _lib.call("vx_coarse_pack", linv.shape[0], linv.data_ptr(), self.coarse_packed.data_ptr(), _s())
        return info

    def footprint_bytes(self) -> int:
        b = 0
        for L in self.levels:
            for t in (L.x, L.xt, L.r, L.invd, L.res, L.E):
                b += 0 if t is None else t.numel() * t.element_size()
            b += L.E64.numel() * 8 + L.mask.numel()
        work = getattr(self, "_factor_work", None)
        return b + self.coarse_packed.numel() * 8 * 2 + (0 if work is None else work.numel() * 8)   # A, packed, band

    def spectral_omegas(self, iterations=30, seed=20260923):
        """omega_l = 4 / (3 lambda_l), lambda_l from a seeded FP64 power iteration on D^-1 A over the
        free DOFs (src/voxel_mg.py:228-244).  Returns (omegas, lambdas)."""
        omegas, lams = [], []
        for L in self.levels[:-1]:
            rng = np.random.default_rng(seed)
            m = ((L.mask.to(torch.int32)[:, None] >> torch.arange(3, device="cuda")) & 1).reshape(-1).double()
            v = torch.as_tensor(rng.standard_normal(L.n), device="cuda") * m
            v = v / torch.linalg.vector_norm(v)
            inv64 = L.op64.diagonal(L.E64, L.mask, inverse=True)
            lam = None
            for _ in range(iterations):                 # the norms stay on the device: no host round trip
                w = inv64 * L.op64.matvec(v, L.E64, L.mask) * m
                lam = torch.linalg.vector_norm(w)
                v = w / lam
            lams.append(lam)
        lambdas = [float(x) for x in lams]              # one synchronisation for all levels
        omegas = [4.0 / (3.0 * x) for x in lambdas]
        return omegas, lambdas

    # ------------------------------------------------------------------ kernel emission
    @property
    def fuses_residual_update(self) -> bool:
        """emit(r64, update=...) can apply the CG update r64 -= alpha q in its first kernel."""
        return len(self.levels) > 1

    def emit(self, r64: torch.Tensor, update=None) -> torch.Tensor:
        """Launch one V-cycle on the current stream: z = M(r64); returns the buffer holding z (in
        the hierarchy's dtype).  r64 is the FP64 finest residual; it is read, and written only when
        `update` = (q, S) asks the entry kernel to apply r64 -= S[alpha] q first (multi-level
        hierarchies, see fuses_residual_update)."""
        L0 = self.levels[0]
        if len(self.levels) == 1:
            src = r64
            if self.aux_dtype != torch.float64:
                _lib.call("vx_cast", L0.n, _lib.VX_F64, _ptr(r64, "r"), PREC[self.aux_dtype], L0.r.data_ptr(), 1.0, _s())
                src = L0.r
            self._coarse_apply(L0, src)
            return L0.x
        r0 = r64 if self.dtype == torch.float64 else L0.r
        r_mg = None if self.dtype == torch.float64 else L0.r.data_ptr()
        if update is None:
            _lib.call("vx_vcycle_entry", self.prec, L0.n, _ptr(r64, "r"), r_mg, L0.invd.data_ptr(), L0.omega,
                      L0.x.data_ptr(), _s())
        else:
            q, S = update
            _lib.call("vx_vcycle_entry_update", self.prec, L0.n, _ptr(S, "S", torch.float64), _ptr(r64, "r"),
                      _ptr(q, "q", torch.float64, L0.n), r_mg, L0.invd.data_ptr(), L0.omega, L0.x.data_ptr(), _s())
        return self._level(0, r0)

    def _level(self, l, r):
        L = self.levels[l]
        if l == len(self.levels) - 1:
            self._coarse_apply(L, r)
            return L.x
        bufs = [L.x, L.xt]
        ci = 0
        for _ in range(self.pre - 1):
            L.op.jacobi(bufs[ci], r, L.invd, L.E, L.mask, L.omega, out=bufs[1 - ci])
            ci ^= 1
        res = bufs[1 - ci] if L.res is None else L.res
        L.op.residual(bufs[ci], r, L.E, L.mask, out=res)
        nxt = self.levels[l + 1]
        _lib.call("vx_restrict", self.prec, *L.shape, res.data_ptr(), nxt.mask.data_ptr(), nxt.r.data_ptr(), _s())
        if l + 1 < len(self.levels) - 1:
            _lib.call("vx_scaled_product", self.prec, nxt.n, nxt.omega, nxt.invd.data_ptr(), nxt.r.data_ptr(),
                      nxt.x.data_ptr(), _s())
        xc = self._level(l + 1, nxt.r)
        _lib.call("vx_prolong_add", self.prec, *L.shape, xc.data_ptr(), L.mask.data_ptr(), bufs[ci].data_ptr(), _s())
        for _ in range(self.post):
            L.op.jacobi(bufs[ci], r, L.invd, L.E, L.mask, L.omega, out=bufs[1 - ci])
            ci ^= 1
        return bufs[ci]

    def _coarse_apply(self, L, r):
        if self.blocks:
            nb_ = self.A_coarse.shape[1]
            _lib.call("vx_batch_coarse_apply_factor", self.prec, nb_, self.blocks, nb_, self.coarse_packed.data_ptr(),
                      r.data_ptr(), L.mask.data_ptr(), self._coarse_y.data_ptr(), L.x.data_ptr(), _s())
        else:
            _lib.call("vx_coarse_apply_factor", self.prec, L.n, self.coarse_packed.data_ptr(), r.data_ptr(),
                      L.mask.data_ptr(), self._coarse_y.data_ptr(), L.x.data_ptr(), _s())

    def __call__(self, r64):
        """z = M(r) as a fresh FP64 tensor (the reference's Multigrid.__call__ casts back to r's dtype)."""
        return self.emit(r64.contiguous()).to(torch.float64)


class JacobiPreconditioner:
    """z = inv_diag * r in FP64 (the `precondition=lambda r: inv * r` of a Jacobi-preconditioned fcg)."""

    def __init__(self, op64: VoxelOperator, E64, node_mask):
        self.dtype, self.prec = torch.float64, _lib.VX_F64
        self.op64, self.mask = op64, node_mask
        self.invd = op64.diagonal(E64, node_mask, inverse=True)
        self.z = torch.zeros(op64.ndof, dtype=torch.float64, device="cuda")

    def emit(self, r64):
        _lib.call("vx_scaled_product", _lib.VX_F64, self.z.numel(), 1.0, self.invd.data_ptr(), r64.data_ptr(),
                  self.z.data_ptr(), _s())
        return self.z

    def update_modulus(self, E):
        self.invd.copy_(self.op64.diagonal(E, self.mask, inverse=True))

    def footprint_bytes(self):
        return self.invd.numel() * 16


@dataclass
class SolveResult:
    x: torch.Tensor
    iterations: int
    converged: bool
    rel: float
    matvecs: int

    def __iter__(self):     # unpacks like the reference's (x, it, converged, rel, matvecs)
        return iter((self.x, self.iterations, self.converged, self.rel, self.matvecs))


_LIVE_GRAPHS = weakref.WeakSet()


@atexit.register
def _destroy_graphs():
    # before the CUDA runtime tears down at process exit
    for g in list(_LIVE_GRAPHS):
        g.close()


@dataclass
class PCGResult:
    x: torch.Tensor
    iterations: int
    converged: bool
    rel: float

    def __iter__(self):     # unpacks like the donor's (x, iters, converged, rel_resid)
        return iter((self.x, self.iterations, self.converged, self.rel))


class _GraphLoop:
    """Owns a WHILE graph (csrc/vx_solver.cu) whose body is captured from `emit_body`.

    The body is first run once un-captured: with CUDA's lazy module loading, a kernel's first
    launch loads its module, which must not happen inside a capture.  That warm-up writes the
    solver's buffers on `stream`, so it is ordered after all work already queued on the caller's
    stream: the caching allocator may have handed those buffers memory that kernels still queued
    there (temporaries of the set-up, e.g. the coarse factorisation) are using.  Callers
    re-initialise the solver state after building the graph."""

    def __init__(self, stream: torch.cuda.Stream, S: torch.Tensor, emit_body):
        self.handle = ctypes.c_void_p()
        sp = ctypes.c_void_p(stream.cuda_stream)
        stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(stream):
            emit_body()                                     # warm-up (loads every kernel of the body)
            _lib.call("vx_graph_while_begin", sp, ctypes.byref(self.handle))
            _lib.CAPTURE_STREAM = sp
            before = _lib.launches
            try:
                emit_body()
            finally:
                _lib.CAPTURE_STREAM = None
                # kernels per body execution, plus the condition kernel
                self.body_kernels = _lib.launches - before + 1
                _lib.launches = before
                _lib.call("vx_graph_while_end", self.handle, S.data_ptr(), sp)
        _LIVE_GRAPHS.add(self)

    def launch(self, stream):
        _lib.call("vx_graph_launch", self.handle, ctypes.c_void_p(stream.cuda_stream))

    def account(self, bodies: int):
        """Add the kernels of `bodies` executions of the loop body to the launch counter."""
        _lib.launches += int(bodies) * self.body_kernels

    def close(self):
        if self.handle:
            _lib.load().vx_graph_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        if not sys.is_finalizing():
            self.close()


class FCGSolver:
    """Flexible PCG (Polak-Ribiere beta) in FP64 with the reference fcg's semantics
    (src/voxel_mg.py:181-217): true residual every `check_every` iterations with residual
    replacement, `fixed_iterations` mode, returns (x, it, converged, rel, matvecs).  The operator
    is the Dirichlet form M K M + (I - M) in FP64; `precond.emit(r)` launches z = M(r)."""

    def __init__(self, op64: VoxelOperator, E64, node_mask, precond, tol=1e-8, maxiter=200, check_every=5,
                 fixed_iterations=None, graph=True):
        if op64.dtype != torch.float64:
            raise ValueError("the outer operator must be float64")
        self.op, self.E, self.mask, self.M = op64, E64.contiguous(), node_mask, precond
        self.tol, self.maxiter, self.fixed = float(tol), int(maxiter), fixed_iterations
        self.check_every = max(1, int(check_every))
        n = op64.ndof
        self.n = n
        f64 = dict(dtype=torch.float64, device="cuda")
        self.b = torch.zeros(n, **f64)
        self.x = torch.zeros(n, **f64)
        self.r = torch.zeros(n, **f64)
        self.p = torch.zeros(n, **f64)
        self.q = torch.zeros(n, **f64)
        self.z_old = torch.zeros(n, dtype=precond.dtype, device="cuda")     # z's own storage: an exact copy
        self.S = torch.zeros(16, **f64)
        self.S_host = torch.zeros(16, dtype=torch.float64, pin_memory=True)
        # f . x after a launched solve (launch(..., dot_with=f)): device value and its pinned copy
        self.dot_partials = torch.zeros(int(_lib.load().vx_partials_size(n)), **f64)
        self.dot_dev = torch.zeros(1, **f64)
        self.dot_host = torch.zeros(1, dtype=torch.float64, pin_memory=True)
        self._dot_with = None
        self.last_dot = None
        self.G_op = op64.partials_size
        self.G_vec = int(_lib.load().vx_solver_partials(n))
        self.partials = torch.zeros(max(self.G_op, 2 * self.G_vec), **f64)
        self.zprec = PREC[precond.dtype]
        self.stream = torch.cuda.Stream()
        self.use_graph = bool(graph)
        self._graph = None
        self._graph_k = None
        self._pending = None
        self._event = None

    def footprint_bytes(self) -> int:
        return 6 * self.n * 8 + self.M.footprint_bytes() + self.E.numel() * 8

    # ------------------------------------------------------------------ kernel emission
    def _fin(self, op, G):
        _lib.call("vx_solver_finalize", op, G, self.partials.data_ptr(), self.S.data_ptr(), _s())

    def _iteration(self, check: bool):
        op, S, pp = self.op, self.S.data_ptr(), self.partials.data_ptr()
        # Off the check iterations the updates ride on kernels that stream the same vectors anyway:
        # r -= alpha q in the preconditioner's first kernel, x += alpha p in the direction update.
        # At a check iteration x is updated here and r is replaced by b - A x.
        fuse = not check and getattr(self.M, "fuses_residual_update", False)
        op.apply_dot(self.p, self.E, self.mask, self.q, self.partials)          # q = A p, p.q
        self._fin(FIN_PQ, self.G_op)
        if not fuse:
            _lib.call("vx_cg_update", _lib.VX_F64, self.n, S, self.x.data_ptr(), self.p.data_ptr(),
                      self.r.data_ptr(), self.q.data_ptr(), 0 if check else 1, _s())
        if check:                                                                # r = b - A x (replacement)
            op.true_residual(self.x, self.b, self.E, self.mask, self.r, self.partials)
            self._fin(FIN_TRUE, self.G_op)
        z = self.M.emit(self.r, update=(self.q, self.S)) if fuse else self.M.emit(self.r)
        _lib.call("vx_dots_pr", _lib.VX_F64, self.zprec, self.n, self.r.data_ptr(), z.data_ptr(),
                  self.z_old.data_ptr(), pp, _s())
        self._fin(FIN_BETA_PR, self.G_vec)
        if fuse:
            _lib.call("vx_cg_direction_update", self.zprec, self.n, S, z.data_ptr(), self.p.data_ptr(),
                      self.z_old.data_ptr(), self.x.data_ptr(), _s())
        else:
            _lib.call("vx_cg_direction", _lib.VX_F64, self.zprec, self.n, S, z.data_ptr(), self.p.data_ptr(),
                      self.z_old.data_ptr(), _s())

    def _body(self, k, checking):
        for j in range(k):
            self._iteration(checking and j == k - 1)

    def _init(self, b, x0=None):
        S = self.S.data_ptr()
        self.b.copy_(b)
        self.p.zero_()
        _lib.call("vx_set_scalars", S, 0, 16, 0.0, _s())
        _lib.call("vx_set_scalars", S, S_TOL, 1, self.tol if self.fixed is None else -1.0, _s())
        _lib.call("vx_dots_pr", _lib.VX_F64, _lib.VX_F64, self.n, self.b.data_ptr(), self.b.data_ptr(), None,
                  self.partials.data_ptr(), _s())
        self._fin(FIN_NB, self.G_vec)
        if x0 is None:
            self.x.zero_()
            self.r.copy_(self.b)
        else:                                                   # warm start: r = b - A x0
            self.x.copy_(x0)
            self.op.true_residual(self.x, self.b, self.E, self.mask, self.r, self.partials)
            self._fin(FIN_TRUE, self.G_op)
        z = self.M.emit(self.r)
        _lib.call("vx_dots_pr", _lib.VX_F64, self.zprec, self.n, self.r.data_ptr(), z.data_ptr(), None,
                  self.partials.data_ptr(), _s())
        self._fin(FIN_RZ, self.G_vec)
        _lib.call("vx_cg_direction", _lib.VX_F64, self.zprec, self.n, S, z.data_ptr(), self.p.data_ptr(),
                  self.z_old.data_ptr(), _s())                                  # p = z (beta = 0), z_old = z

    def _read(self):
        self.S_host.copy_(self.S, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.S_host.numpy().copy()

    def launch(self, b: torch.Tensor, x0: torch.Tensor | None = None, stream: torch.cuda.Stream | None = None,
               dot_with: torch.Tensor | None = None):
        """Enqueue a solve of A x = b on `stream` (default: the solver's own) without waiting: the
        initialisation, the whole-loop graph and an asynchronous read-back of the scalars.  Call
        finish() for the result; done() polls without blocking.  With `dot_with` = f, the dot
        product f . x (e.g. the compliance) is computed on the same stream after the loop and read
        back with the scalars: finish() leaves it in `last_dot` without another synchronisation."""
        if b.numel() != self.n:
            raise ValueError(f"b has {b.numel()} entries, expected {self.n}")
        st = stream or self.stream
        checking = self.fixed is None
        k = self.check_every if checking else 1
        limit = self.fixed if self.fixed is not None else self.maxiter
        full = limit // k
        caller = torch.cuda.current_stream()
        st.wait_stream(caller)
        if st != caller:                 # b and x0 are read on st: keep their memory until it is done
            b.record_stream(st)
            if x0 is not None:
                x0.record_stream(st)
        if full > 0 and self.use_graph and (self._graph is None or self._graph_k != (k, checking)):
            self._graph = _GraphLoop(st, self.S, lambda: self._body(k, checking))
            self._graph_k = (k, checking)
        with torch.cuda.stream(st):
            self._init(b, x0)
            S = self.S.data_ptr()
            _lib.call("vx_set_scalars", S, S_MAXIT, 1, float(limit), _s())
            _lib.call("vx_set_scalars", S, S_CHECK, 1, float(k), _s())
            if full > 0 and self.use_graph:
                self._graph.launch(st)
            self.S_host.copy_(self.S, non_blocking=True)
            self._dot_with = dot_with
            if dot_with is not None:
                if st != caller:
                    dot_with.record_stream(st)
                self._emit_dot()
                self.dot_host.copy_(self.dot_dev, non_blocking=True)
            self._event = torch.cuda.Event()
            self._event.record(st)
        self._pending = (st, k, checking, limit, full, x0 is not None)

    def _emit_dot(self):
        f = self._dot_with
        A = (ctypes.c_void_p * 3)(_ptr(f, "dot_with", torch.float64, self.n), None, None)
        B = (ctypes.c_void_p * 3)(self.x.data_ptr(), None, None)
        _lib.call("vx_dots", _lib.VX_F64, self.n, 1, A, B, self.dot_partials.data_ptr(), self.dot_dev.data_ptr(), _s())

    def done(self) -> bool:
        return self._pending is None or self._event.query()

    def finish(self) -> SolveResult:
        """Wait for the launched solve and return its result (host work only for the rare tails:
        iterations past the last full loop body, the host-driven loop, or non-convergence)."""
        st, k, checking, limit, full, warm = self._pending
        self._pending = None
        self._event.synchronize()
        with torch.cuda.stream(st):
            s = self.S_host.numpy().copy()
            s_launch = s.copy()
            if full > 0 and self.use_graph:
                self._graph.account(max(1, -(-int(s[S_IT]) // k)))
            if not self.use_graph and not (warm and s[S_DONE]):
                for _ in range(full):
                    self._body(k, checking)
                    s = self._read()
                    if s[S_DONE] or s[S_BREAK]:
                        break
            done, it = bool(s[S_DONE]), int(s[S_IT])
            while not done and not s[S_BREAK] and it < limit:                 # iterations past the last full body
                self._iteration(checking and (it + 1) % k == 0)
                s = self._read()
                done, it = bool(s[S_DONE]), int(s[S_IT])
            if not done:                                                       # final true residual (voxel_mg.py:213-216)
                self.op.true_residual(self.x, self.b, self.E, self.mask, self.q, self.partials)
                self._fin(FIN_TRUE, self.G_op)
                s = self._read()
            if self._dot_with is not None:
                if int(s[S_IT]) != int(s_launch[S_IT]):                      # x moved after the dot: redo it
                    self._emit_dot()
                    self.dot_host.copy_(self.dot_dev, non_blocking=True)
                    torch.cuda.current_stream().synchronize()
                self.last_dot = float(self.dot_host[0])
                self._dot_with = None
        torch.cuda.current_stream().wait_stream(st)
        rel = float(s[S_REL])
        return SolveResult(self.x, int(s[S_IT]), bool(rel <= self.tol), rel, int(s[S_MV]))

    def solve(self, b: torch.Tensor, x0: torch.Tensor | None = None) -> SolveResult:
        """Solve A x = b (optionally warm-started at x0: then r0 = b - A x0 and a converged x0
        returns after 0 iterations).  x is the solver's own buffer."""
        self.launch(b, x0)
        return self.finish()


class JacobiPCG:
    """The donor's Jacobi-preconditioned CG with a true-residual test and residual replacement every
    `check_every` iterations, Fletcher-Reeves beta (experiments/session_a/donor/src/gpu_fem/
    simp_r2.py:187-295), in FP64 or FP32 (`op.dtype`).  Returns (x, iters, converged, rel)."""

    def __init__(self, op: VoxelOperator, E, node_mask, tol=1e-5, maxiter=20000, check_every=50, inv_diag=None,
                 graph=True):
        if op.dtype not in (torch.float64, torch.float32):
            raise ValueError("Jacobi-PCG runs in float64 or float32")
        self.op, self.E, self.mask = op, E.contiguous(), node_mask
        self.dtype, self.prec = op.dtype, op.prec
        self.tol, self.maxiter, self.k = float(tol), int(maxiter), max(1, int(check_every))
        n = op.ndof
        self.n = n
        t = dict(dtype=self.dtype, device="cuda")
        self.invd = inv_diag if inv_diag is not None else op.diagonal(self.E, node_mask, inverse=True)
        self.b = torch.zeros(n, **t)
        self.x = torch.zeros(n, **t)
        self.r = torch.zeros(n, **t)
        self.z = torch.zeros(n, **t)
        self.p = torch.zeros(n, **t)
        self.q = torch.zeros(n, **t)
        self.S = torch.zeros(16, dtype=torch.float64, device="cuda")
        self.S_host = torch.zeros(16, dtype=torch.float64, pin_memory=True)
        self.G_op = op.partials_size
        self.G_vec = int(_lib.load().vx_solver_partials(n))
        self.partials = torch.zeros(max(self.G_op, 2 * self.G_vec), dtype=torch.float64, device="cuda")
        self.stream = torch.cuda.Stream()
        self.use_graph = bool(graph)
        self._graph = None

    def _fin(self, op, G):
        _lib.call("vx_solver_finalize", op, G, self.partials.data_ptr(), self.S.data_ptr(), _s())

    def _iteration(self, check):
        op, S = self.op, self.S.data_ptr()
        op.apply_dot(self.p, self.E, self.mask, self.q, self.partials)
        self._fin(FIN_PQ, self.G_op)
        _lib.call("vx_cg_update", self.prec, self.n, S, self.x.data_ptr(), self.p.data_ptr(), self.r.data_ptr(),
                  self.q.data_ptr(), 0 if check else 1, _s())
        if check:
            op.true_residual(self.x, self.b, self.E, self.mask, self.r, self.partials)
            self._fin(FIN_TRUE, self.G_op)
        _lib.call("vx_jacobi_precond_dot", self.prec, self.n, self.invd.data_ptr(), self.r.data_ptr(),
                  self.z.data_ptr(), self.partials.data_ptr(), _s())
        self._fin(FIN_BETA_FR, self.G_vec)
        _lib.call("vx_cg_direction", self.prec, self.prec, self.n, S, self.z.data_ptr(), self.p.data_ptr(), None, _s())

    def _read(self):
        self.S_host.copy_(self.S, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.S_host.numpy().copy()

    def solve(self, b, x0=None, tol=None, maxiter=None):
        tol = self.tol if tol is None else float(tol)
        maxiter = self.maxiter if maxiter is None else int(maxiter)
        caller = torch.cuda.current_stream()
        self.stream.wait_stream(caller)
        k = self.k
        if self.use_graph and self._graph is None and maxiter // k > 0:
            self._graph = _GraphLoop(self.stream, self.S, lambda: [self._iteration(j == k - 1) for j in range(k)])
        with torch.cuda.stream(self.stream):
            S = self.S.data_ptr()
            m = self.mask
            self.b.copy_(b)
            if x0 is None:
                self.x.zero_()
            else:
                self.x.copy_(x0)
                if m is not None:                                   # x = x0 * mask
                    bits = ((m.to(torch.int32)[:, None] >> torch.arange(3, device="cuda")) & 1).reshape(-1)
                    self.x.mul_(bits.to(self.dtype))
            _lib.call("vx_set_scalars", S, 0, 16, 0.0, _s())
            _lib.call("vx_set_scalars", S, S_TOL, 1, tol, _s())
            _lib.call("vx_dots_pr", self.prec, self.prec, self.n, self.b.data_ptr(), self.b.data_ptr(), None,
                      self.partials.data_ptr(), _s())
            self._fin(FIN_NB, self.G_vec)
            self.op.true_residual(self.x, self.b, self.E, self.mask, self.r, self.partials)   # r = b - A x
            self._fin(FIN_RR_ONLY, self.G_op)
            _lib.call("vx_jacobi_precond_dot", self.prec, self.n, self.invd.data_ptr(), self.r.data_ptr(),
                      self.z.data_ptr(), self.partials.data_ptr(), _s())
            self._fin(FIN_RZ, self.G_vec)
            _lib.call("vx_set_scalars", S, S_BETA, 1, 0.0, _s())
            self.p.zero_()
            _lib.call("vx_cg_direction", self.prec, self.prec, self.n, S, self.z.data_ptr(), self.p.data_ptr(), None, _s())
            s = self._read()
            if s[S_NB] <= 0:
                return PCGResult(self.x, 0, True, 0.0)
            if s[S_REL] <= tol:
                return PCGResult(self.x, 0, True, float(s[S_REL]))
            _lib.call("vx_set_scalars", S, S_MAXIT, 1, float(maxiter), _s())
            _lib.call("vx_set_scalars", S, S_CHECK, 1, float(k), _s())
            if maxiter // k > 0:
                if self.use_graph:
                    self._graph.launch(self.stream)
                else:
                    for _ in range(maxiter // k):
                        for j in range(k):
                            self._iteration(j == k - 1)
                        s = self._read()
                        if s[S_DONE] or s[S_BREAK]:
                            break
            s = self._read()
            it = int(s[S_IT])
            if maxiter // k > 0 and self.use_graph:
                self._graph.account(max(1, -(-it // k)))
            while not s[S_DONE] and not s[S_BREAK] and it < maxiter:          # tail: check at maxiter
                self._iteration((it + 1) % k == 0 or it + 1 >= maxiter)
                s = self._read()
                it = int(s[S_IT])
            if not s[S_DONE]:
                self.op.true_residual(self.x, self.b, self.E, self.mask, self.q, self.partials)
                self._fin(FIN_RR_ONLY, self.G_op)
                s = self._read()
        caller.wait_stream(self.stream)
        return PCGResult(self.x, int(s[S_IT]), bool(s[S_DONE]), float(s[S_REL]))


@dataclass
class IRResult:
    x: torch.Tensor
    outer: int
    inner: int
    converged: bool
    rel: float

    def __iter__(self):     # unpacks like the donor's (x, outer, inner_total, converged, rel)
        return iter((self.x, self.outer, self.inner, self.converged, self.rel))


class PCGIR:
    """Mixed-precision iterative refinement (donor experiments/session_a/donor/src/gpu_fem/
    simp_r2.py:298-385): the FP64 residual r = b - A x, an FP32 Jacobi-PCG correction of the scaled
    system A d = r / |r| to `inner_tol`, x += |r| d; a divergence guard undoes a correction that
    raised the residual and tightens the inner tolerance tenfold (giving up below 1e-5).  Every
    vector operation is a library kernel; the outer loop reads one norm per pass.
    Returns IRResult (x, outer, inner, converged, rel)."""

    def __init__(self, op64: VoxelOperator, E64, node_mask, tol=1e-5, inner_tol=1e-1, max_outer=40,
                 inner_maxiter=4000, check_every=50, graph=True, inv_diag32=None, E32=None):
        """inv_diag32 / E32: the inner FP32 system's inverse diagonal and modulus (default: the FP32
        inverse diagonal and the FP32 rounding of E64)."""
        if op64.dtype != torch.float64:
            raise ValueError("the outer operator must be float64")
        self.op64, self.E64, self.mask = op64, E64.contiguous(), node_mask
        self.tol, self.inner_tol = float(tol), float(inner_tol)
        self.max_outer, self.inner_maxiter = int(max_outer), int(inner_maxiter)
        n = op64.ndof
        self.n = n
        op32 = VoxelOperator(op64.shape, op64.ke, torch.float32)
        if E32 is None:
            self.E32 = torch.empty(self.E64.numel(), dtype=torch.float32, device="cuda")
            _lib.call("vx_cast", self.E64.numel(), _lib.VX_F64, self.E64.data_ptr(), _lib.VX_F32, self.E32.data_ptr(), 1.0, _s())
        else:
            self.E32 = E32.to(torch.float32).contiguous()
        self.inner = JacobiPCG(op32, self.E32, node_mask, tol=inner_tol, maxiter=inner_maxiter,
                               check_every=check_every, graph=graph,
                               inv_diag=None if inv_diag32 is None else inv_diag32.to(torch.float32).contiguous())
        f64 = dict(dtype=torch.float64, device="cuda")
        self.x = torch.zeros(n, **f64)
        self.r = torch.zeros(n, **f64)
        self.corr = torch.zeros(n, **f64)                    # the last correction |r| d, for the undo
        self.rhs32 = torch.zeros(n, dtype=torch.float32, device="cuda")
        self.partials = torch.zeros(op64.partials_size, **f64)
        self.norm = torch.zeros(1, **f64)

    def _residual_norm(self, b):
        self.op64.true_residual(self.x, b, self.E64, self.mask, self.r, self.partials)
        _lib.call("vx_reduce_partials", self.partials.numel(), 1, self.partials.data_ptr(), self.norm.data_ptr(), _s())
        return float(self.norm) ** 0.5

    def solve(self, b: torch.Tensor, x0: torch.Tensor | None = None) -> IRResult:
        b = b.contiguous()
        nb = float(torch.linalg.vector_norm(b))
        if nb <= 0:
            self.x.zero_()
            return IRResult(self.x, 0, 0, True, 0.0)
        if x0 is None:
            self.x.zero_()
        else:
            self.x.copy_(x0)
        n, inner_total = self.n, 0
        tol_in, rel_prev, have_last = self.inner_tol, None, False
        outer = 0
        for outer in range(1, self.max_outer + 1):
            scale = self._residual_norm(b)
            rel = scale / nb
            if rel <= self.tol:
                return IRResult(self.x, outer - 1, inner_total, True, rel)
            if rel_prev is not None and rel > rel_prev and have_last:      # divergence guard: undo
                _lib.call("vx_axpby", _lib.VX_F64, n, -1.0, self.corr.data_ptr(), 1.0, self.x.data_ptr(), _s())
                have_last = False
                tol_in *= 0.1
                if tol_in < 1e-5:
                    return IRResult(self.x, outer, inner_total, False, rel_prev)
                continue
            rel_prev = rel
            _lib.call("vx_cast", n, _lib.VX_F64, self.r.data_ptr(), _lib.VX_F32, self.rhs32.data_ptr(), 1.0 / scale, _s())
            d = self.inner.solve(self.rhs32, tol=tol_in)
            inner_total += d.iterations
            _lib.call("vx_cast", n, _lib.VX_F32, d.x.data_ptr(), _lib.VX_F64, self.corr.data_ptr(), scale, _s())
            _lib.call("vx_axpby", _lib.VX_F64, n, 1.0, self.corr.data_ptr(), 1.0, self.x.data_ptr(), _s())
            have_last = True
        rel = self._residual_norm(b) / nb
        return IRResult(self.x, outer, inner_total, bool(rel <= self.tol), rel)
