"""Several elasticity solves of one grid shape in lockstep: the serving loop's batches.

B jobs on an (nx, ny, nz) grid are stacked along x into one grid of B (nx + s) - s elements, with s =
2^(levels-1) zero-modulus element layers between neighbours whose interior node planes are fixed
(Dirichlet).  A zero modulus couples nothing, so the stacked operator is block diagonal, and s keeps
every job aligned on every level of the hierarchy (one separator element on the coarsest).  Every
stencil, transfer and V-cycle kernel therefore runs ONCE for all B jobs of a level: the same-level
kernels of concurrent jobs are fused into one launch, and each job's nodes see exactly the
arithmetic they would see alone.  What is per job -- the Krylov scalars, the dot products, the
coarsest dense solve -- runs as slot-indexed launches (one launch for the batch), so jobs converge,
stop and are replaced independently: a finished slot takes the next request between graph replays
while the others continue (continuous batching).

The iteration is the reference fcg's with the true residual every iteration (check_every 1,
src/voxel_mg.py:181-217); a chunk of iterations is captured once in a CUDA graph and replayed.
There is no counterpart in the reference (it solves one system at a time).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .element import quadrature
from .operators import PREC, VoxelOperator, node_mask_from_dofs, stream_ptr
from .solver import (FIN_BETA_PR, FIN_NB, FIN_PQ, FIN_RZ, FIN_TRUE, MGHierarchy, S_BREAK, S_CHECK, S_DONE, S_IT,
                     S_MAXIT, S_MV, S_REL, S_TOL, hierarchy_shapes)

_MG = {"fp64": (torch.float64, torch.float64), "mixed": (torch.float32, torch.float32),
       "bf16": (torch.float32, torch.bfloat16)}


def _s():
    return stream_ptr()


@dataclass(frozen=True)
class StackGeometry:
    """Where `slots` jobs of `shape` sit in the stacked grid (element x ranges [k pitch, k pitch + nx))."""
    shape: tuple
    slots: int
    levels: int
    separator: int          # zero-modulus element layers between neighbours on the finest level
    pitch: int              # node planes (and element planes) from one job's start to the next
    grid: tuple             # the stacked grid
    shapes: tuple           # its hierarchy, level by level

    @property
    def job_shapes(self):
        nx, ny, nz = self.shape
        return tuple((nx >> l, ny >> l, nz >> l) for l in range(self.levels))


def stack_geometry(shape, slots, max_coarse_x=16) -> StackGeometry:
    """The stacked grid of `slots` jobs with the job's own hierarchy depth (hierarchy_shapes)."""
    nx, ny, nz = (int(v) for v in shape)
    levels = len(hierarchy_shapes((nx, ny, nz), max_coarse_x))
    sep = 2 ** (levels - 1)
    pitch = nx + sep
    gx = slots * pitch - sep
    shapes = tuple((gx >> l, ny >> l, nz >> l) for l in range(levels))
    return StackGeometry((nx, ny, nz), int(slots), levels, sep, pitch, (gx, ny, nz), shapes)


class BatchedSolver:
    """`slots` independent solves K(E_k) u_k = f_k on grids of shape `shape` (author layout), mixed or
    FP64 GMG-preconditioned flexible CG, fused into shared launches (module docstring).

    Host protocol: admit([(slot, E, f, tol)]) for free slots, run() (a captured chunk of the loop for
    every slot; finished and free slots are no-ops), poll() for the per-slot state, result(slot) and
    retire(slot) for finished slots; repeat."""

    def __init__(self, shape, slots, mask=None, ke=None, precision="mixed", pre=2, post=2, omega=0.6,
                 max_coarse_x=16, maxiter=200, chunk=4):
        if precision not in _MG:
            raise ValueError(f"precision must be one of {tuple(_MG)}")
        if int(slots) < 1:
            raise ValueError("slots must be positive")
        self.geo = geo = stack_geometry(shape, slots, max_coarse_x)
        self.shape, self.B, self.levels, self.pitch = geo.shape, geo.slots, geo.levels, geo.pitch
        nx, ny, nz = self.shape
        self.ke = quadrature([1.0, 1.0, 1.0], 0.3) if ke is None else np.asarray(ke, dtype=np.float64).reshape(24, 24)
        self.plane = (ny + 1) * (nz + 1)                   # nodes per node plane
        self.n_job = 3 * (nx + 1) * self.plane             # DOFs of one job
        self.stride = 3 * self.pitch * self.plane          # DOFs from one job to the next
        self.e_stride = self.pitch * ny * nz               # elements from one job to the next
        self.n_elem_job = nx * ny * nz
        # node mask: each job's own (default: the clamped x = 0 face), separator planes fixed
        if mask is None:
            job_mask = torch.full(((nx + 1) * self.plane,), 7, dtype=torch.uint8, device="cuda")
            job_mask[: self.plane] = 0
        else:
            m = mask.to("cuda") if isinstance(mask, torch.Tensor) else torch.as_tensor(np.asarray(mask), device="cuda")
            job_mask = m.contiguous() if m.dtype == torch.uint8 else node_mask_from_dofs(m.to(torch.float64))
        self.node_mask = torch.zeros((geo.grid[0] + 1) * self.plane, dtype=torch.uint8, device="cuda")
        E64 = torch.zeros(geo.grid[0] * ny * nz, dtype=torch.float64, device="cuda")
        for k in range(self.B):
            o = k * self.pitch * self.plane
            self.node_mask[o:o + job_mask.numel()] = job_mask
            E64[k * self.e_stride:k * self.e_stride + self.n_elem_job] = 1.0    # harmless until admitted
        dt, aux = _MG[precision]
        self.M = MGHierarchy(geo.grid, self.ke, E64, self.node_mask, dt, pre, post, omega, shapes=list(geo.shapes),
                             aux_dtype=aux, coarse_blocks=self.B)
        self.E64 = self.M.levels[0].E64                    # the hierarchy's own finest moduli
        self.op = VoxelOperator(geo.grid, self.ke, torch.float64)
        n = self.op.ndof
        f64 = dict(dtype=torch.float64, device="cuda")
        self.b, self.x, self.r, self.p, self.q = (torch.zeros(n, **f64) for _ in range(5))
        self.z_old = torch.zeros(n, dtype=dt, device="cuda")
        self.zprec = PREC[dt]
        self.S = torch.zeros(self.B, 16, **f64)
        self.S[:, S_DONE] = 1.0                            # an empty slot counts as finished
        self.S_host = torch.zeros(self.B, 16, dtype=torch.float64, pin_memory=True)
        self.G = int(_lib.load().vx_solver_partials(self.n_job))
        self.partials = torch.zeros(self.B * 2 * self.G, **f64)
        self.op_partials = torch.zeros(self.op.partials_size, **f64)       # the stacked forms' sums (unused)
        self.maxiter = int(maxiter)
        self.chunk = int(chunk)
        self.stream = torch.cuda.Stream()
        self._graph = None
        self._event = None

    def footprint_bytes(self) -> int:
        n = self.op.ndof
        return int(6 * 8 * n + self.z_old.numel() * self.z_old.element_size() + self.M.footprint_bytes())

    # ------------------------------------------------------------------ per-slot views
    def seg(self, t, k):
        """Slot k's DOFs of a stacked vector."""
        return t[k * self.stride:k * self.stride + self.n_job]

    def modulus(self, k):
        """Slot k's finest element moduli (a view)."""
        return self.E64[k * self.e_stride:k * self.e_stride + self.n_elem_job]

    # ------------------------------------------------------------------ kernels of one iteration
    def _fin(self, op):
        _lib.call("vx_batch_finalize", op, self.G, self.B, self.partials.data_ptr(), 2 * self.G, self.S.data_ptr(), _s())

    def _dots(self, a, b, c=None, zprec=_lib.VX_F64):
        _lib.call("vx_batch_dots_pr", zprec, self.n_job, self.B, self.stride, a.data_ptr(), b.data_ptr(),
                  None if c is None else c.data_ptr(), self.partials.data_ptr(), _s())

    def _iteration(self):
        """One fcg iteration for every slot (true residual every iteration, src/voxel_mg.py:192-209)."""
        S = self.S.data_ptr()
        self.op.apply_dot(self.p, self.E64, self.node_mask, self.q, self.op_partials)      # q = A p (stacked)
        self._dots(self.p, self.q)
        self._fin(FIN_PQ)
        _lib.call("vx_batch_cg_update", _lib.VX_F64, self.n_job, self.B, self.stride, S, self.x.data_ptr(),
                  self.p.data_ptr(), None, None, 0, _s())                                  # x += alpha p
        self.op.true_residual(self.x, self.b, self.E64, self.node_mask, self.r, self.op_partials)
        self._dots(self.r, self.r)
        self._fin(FIN_TRUE)
        z = self.M.emit(self.r)                                                           # the V-cycle, stacked
        self._dots(self.r, z, self.z_old, self.zprec)
        self._fin(FIN_BETA_PR)
        _lib.call("vx_batch_cg_direction", self.zprec, self.n_job, self.B, self.stride, S, z.data_ptr(),
                  self.p.data_ptr(), self.z_old.data_ptr(), _s())                         # p = z + beta p

    # ------------------------------------------------------------------ host protocol
    def admit(self, jobs):
        """Start solves in free slots: jobs = [(slot, E, f, tol)], E (Ne) the job's element moduli,
        f (3N) its load, author layout on this grid shape.  Refreshes the slots' hierarchy segments
        and coarse factors, sets r = b, z = M(r), p = z and the slots' scalars (others untouched)."""
        if not jobs:
            return
        st = self.stream
        st.wait_stream(torch.cuda.current_stream())
        for _, E, f, _ in jobs:
            for t in (E, f):
                if isinstance(t, torch.Tensor) and t.is_cuda:
                    t.record_stream(st)
        with torch.cuda.stream(st):
            for k, E, f, tol in jobs:
                self.modulus(k).copy_(torch.as_tensor(E).to(device="cuda", dtype=torch.float64).reshape(-1))
                self.seg(self.b, k).copy_(torch.as_tensor(f).to(device="cuda", dtype=torch.float64).reshape(-1))
            # every level's moduli and diagonals in one launch per level (the other slots' values come
            # out unchanged), then the new slots' coarsest systems factored side by side
            self.M.refresh_levels()
            self.M.refresh_blocks([k for k, *_ in jobs])
            for k, E, f, tol in jobs:
                self.seg(self.x, k).zero_()
                self.seg(self.p, k).zero_()
                self.seg(self.z_old, k).zero_()
                self.seg(self.r, k).copy_(self.seg(self.b, k))
                row = torch.zeros(16, dtype=torch.float64)
                row[S_TOL], row[S_MAXIT], row[S_CHECK] = float(tol), float(self.maxiter), 1.0
                self.S[k].copy_(row)
            z = self.M.emit(self.r)                          # one V-cycle for all the new slots
            for k, *_ in jobs:
                S_k = self.S[k].data_ptr()
                part = self.partials[k * 2 * self.G:(k + 1) * 2 * self.G].data_ptr()
                bk = self.seg(self.b, k).data_ptr()
                _lib.call("vx_dots_pr", _lib.VX_F64, _lib.VX_F64, self.n_job, bk, bk, None, part, _s())
                _lib.call("vx_solver_finalize", FIN_NB, self.G, part, S_k, _s())
                _lib.call("vx_dots_pr", _lib.VX_F64, self.zprec, self.n_job, self.seg(self.r, k).data_ptr(),
                          self.seg(z, k).data_ptr(), None, part, _s())
                _lib.call("vx_solver_finalize", FIN_RZ, self.G, part, S_k, _s())
                _lib.call("vx_cg_direction", _lib.VX_F64, self.zprec, self.n_job, S_k, self.seg(z, k).data_ptr(),
                          self.seg(self.p, k).data_ptr(), self.seg(self.z_old, k).data_ptr(), _s())   # beta = 0

    def run(self, iterations=None):
        """Enqueue `iterations` (default: the captured chunk) fcg iterations for every slot on the
        solver's stream, then an asynchronous read-back of the scalars (ready() / poll())."""
        k = self.chunk if iterations is None else int(iterations)
        st = self.stream
        st.wait_stream(torch.cuda.current_stream())
        if k == self.chunk:
            if self._graph is None:
                with torch.cuda.stream(st):
                    for _ in range(k):                    # loads every kernel before the capture; the running
                        self._iteration()                 # slots' solves move on by these k iterations
                st.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=st):
                    for _ in range(k):
                        self._iteration()
                self._graph = g
            with torch.cuda.stream(st):
                self._graph.replay()
        else:
            with torch.cuda.stream(st):
                for _ in range(k):
                    self._iteration()
        with torch.cuda.stream(st):
            self.S_host.copy_(self.S, non_blocking=True)
            self._event = torch.cuda.Event()
            self._event.record(st)

    def ready(self):
        return self._event is None or self._event.query()

    def poll(self):
        """After the last run(): (finished, iterations, rel, matvecs) per slot (numpy arrays); a slot is
        finished once converged, broken down or at maxiter."""
        if self._event is not None:
            self._event.synchronize()
        s = self.S_host.numpy()
        finished = (s[:, S_DONE] != 0) | (s[:, S_BREAK] != 0) | (s[:, S_IT] >= s[:, S_MAXIT])
        return finished, s[:, S_IT].astype(int), s[:, S_REL].copy(), s[:, S_MV].astype(int)

    def result(self, k):
        """(x_k copy, iterations, converged, rel, compliance f_k . x_k) of slot k, after poll()."""
        return self.results([k])[0]

    def results(self, ks):
        """result() of several slots with one synchronisation."""
        S = self.S_host.numpy()
        with torch.cuda.stream(self.stream):
            xs = [self.seg(self.x, k).clone() for k in ks]
            comps = torch.stack([torch.dot(self.seg(self.b, k), x) for k, x in zip(ks, xs)]).cpu() if ks else []
        return [(x, int(S[k, S_IT]), bool(S[k, S_REL] <= S[k, S_TOL]), float(S[k, S_REL]), float(c))
                for k, x, c in zip(ks, xs, comps)]

    def retire(self, k):
        """Slot k becomes free (its work stays a no-op until a new job is admitted)."""
        with torch.cuda.stream(self.stream):
            self.S[k, S_DONE] = 1.0

    def solve(self, jobs):
        """Admit jobs = [(E, f, tol)] into slots 0.. and run until every one finishes.
        Returns [(x, iterations, converged, rel, compliance)]."""
        if len(jobs) > self.B:
            raise ValueError(f"{len(jobs)} jobs for {self.B} slots")
        for k in range(self.B):
            self.retire(k)
        self.admit([(k, E, f, tol) for k, (E, f, tol) in enumerate(jobs)])
        out = [None] * len(jobs)
        while any(o is None for o in out):
            self.run()
            fin, *_ = self.poll()
            for k in range(len(jobs)):
                if out[k] is None and fin[k]:
                    out[k] = self.result(k)
        return out
