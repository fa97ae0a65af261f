"""Public solve API: one voxel elasticity problem resident on the device.

`ElasticitySolver` owns the FP64 outer operator, the preconditioner (GMG V-cycle in FP64 or FP32,
or Jacobi) and the graph-captured flexible-CG loop; `solve(...)` is the host-buffer entry point
(numpy in, numpy out) a caller of the reference's `fcg(..., Multigrid(...))` path would use.
"""
from __future__ import annotations

from collections import OrderedDict

import numpy as np
import torch

from .element import quadrature
from .operators import VoxelOperator, node_mask_from_dofs
from .solver import FCGSolver, JacobiPreconditioner, MGHierarchy, hierarchy_shapes

PRECISIONS = ("fp64", "mixed", "bf16", "bf16-all", "jacobi")
# V-cycle storage: (iterate dtype, auxiliary-vector and modulus dtype)
_MG_STORAGE = {"fp64": (torch.float64, torch.float64), "mixed": (torch.float32, torch.float32),
               "bf16": (torch.float32, torch.bfloat16), "bf16-all": (torch.bfloat16, torch.bfloat16)}


def _dev(a, dtype=torch.float64):
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda").to(dtype).contiguous()


class ElasticitySolver:
    """K(E) u = f on a (nx, ny, nz) voxel cantilever-type problem, author layout.

    precision: "fp64" (FP64 V-cycle), "mixed" (FP32 V-cycle inside the FP64 outer loop; FP64 for the
    outer residual, dots, step lengths and the coarsest solve), "bf16" (as mixed, with the V-cycle's
    moduli, right-hand sides, residuals and inverse diagonals stored in bf16, iterates in FP32),
    "bf16-all" (the iterates in bf16 as well; costs outer iterations) or "jacobi" (FP64 Jacobi-PCG
    via fcg).
    omega: a float, a per-level list, or "spectral" (4 / (3 lambda_l), src/voxel_mg.py:228-244).
    """

    def __init__(self, shape, E, mask, ke=None, precision="mixed", pre=2, post=2, omega=0.6, max_coarse_x=16,
                 levels=None, tol=1e-8, maxiter=200, check_every=1, graph=True, spectral_seed=20260923):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}")
        self.shape = tuple(int(s) for s in shape)
        self.ke = quadrature([1.0, 1.0, 1.0], 0.3) if ke is None else np.asarray(ke, dtype=np.float64).reshape(24, 24)
        self.E = _dev(E).clone()          # owned: update_modulus rewrites it in place
        m = mask.to("cuda", non_blocking=True) if isinstance(mask, torch.Tensor) else _dev(mask)
        self.node_mask = m.contiguous() if m.dtype == torch.uint8 else node_mask_from_dofs(m.to(torch.float64))
        self.op64 = VoxelOperator(self.shape, self.ke, torch.float64)
        self.precision = precision
        if precision == "jacobi":
            self.M = JacobiPreconditioner(self.op64, self.E, self.node_mask)
        else:
            shapes = hierarchy_shapes(self.shape, max_coarse_x)
            if levels is not None:
                if levels > len(shapes):
                    raise ValueError(f"{self.shape} supports at most {len(shapes)} levels with max_coarse_x={max_coarse_x}")
                shapes = shapes[:levels]
            dt, aux = _MG_STORAGE[precision]
            spectral = isinstance(omega, str) and omega == "spectral"
            self.M = MGHierarchy(self.shape, self.ke, self.E, self.node_mask, dt, pre, post,
                                 None if spectral else omega, shapes=shapes, aux_dtype=aux)
            self.spectral_seed = spectral_seed
            self._spectral = spectral
            if spectral:
                # lambda_l from the FP64 level operators, as the reference estimates it once on the
                # FP64 hierarchy shared by all arms (experiments/session_i/run_gpu.py:287-288)
                self.refresh_omegas()
        self.fcg = FCGSolver(self.op64, self.E, self.node_mask, self.M, tol=tol, maxiter=maxiter,
                             check_every=check_every, graph=graph)

    def refresh_omegas(self, iterations=30):
        """Re-estimate omega_l = 4 / (3 lambda_l) for the current moduli (spectral damping)."""
        om, lam = self.M.spectral_omegas(iterations=iterations, seed=self.spectral_seed)
        self.M.set_omegas(om)
        self.lambdas = lam
        return om, lam

    @property
    def levels(self):
        return getattr(self.M, "shapes", [self.shape])

    def footprint_bytes(self):
        return self.fcg.footprint_bytes()

    def solve(self, f, x0=None):
        """Solve with right-hand side f (CUDA tensor or array, author layout), optionally warm-started
        at x0.  Returns SolveResult (x, iterations, converged, rel, matvecs); x is the solver's own
        buffer (copy it to keep it)."""
        return self.fcg.solve(_dev(f), None if x0 is None else _dev(x0))

    def update_modulus(self, E):
        """New element moduli on the same grid: refreshes the hierarchy in place (graphs stay valid)."""
        E = _dev(E)
        if E.data_ptr() != self.E.data_ptr():
            self.E.copy_(E)
        self.M.update_modulus(self.E)

    def update(self, E, mask=None):
        """A new problem on the same grid: moduli and (optionally) the 0/1 DOF or uint8 node mask,
        refreshed in place -- every level's moduli, masks and diagonals and the coarsest factor are
        recomputed from the new inputs; buffers and captured graphs are reused."""
        if mask is not None:
            m = mask.to("cuda", non_blocking=True) if isinstance(mask, torch.Tensor) else _dev(mask)
            nm = m.contiguous() if m.dtype == torch.uint8 else node_mask_from_dofs(m.to(torch.float64))
            self.node_mask.copy_(nm)
            if hasattr(self.M, "update_mask"):
                self.M.update_mask()
        self.update_modulus(E)
        if getattr(self, "_spectral", False):
            self.refresh_omegas()

    def compliance(self, f, x):
        return float(_dev(f) @ x)


_SOLVERS = OrderedDict()      # set-up key -> ElasticitySolver, least recently used first
_SOLVER_CACHE_SIZE = 4
_COPY_STREAMS = {}            # device index -> side stream for host-to-device staging


def _stage_inputs(mask, E, force):
    """Device copies of solve()'s inputs, mask first and force last.  Pinned CPU tensors go through a
    side stream, so the current stream can refresh the hierarchy and factor the coarsest system as
    soon as the mask and the moduli have arrived, while the force is still in transit; the current
    stream waits on an event before each use.  Other inputs (numpy arrays, pageable tensors) are
    copied on the current stream as before.  Returns (mask, E, force, wait) with wait(i) making the
    current stream wait for input i (0 mask, 1 E, 2 force)."""
    pinned = all(isinstance(a, torch.Tensor) and not a.is_cuda and a.is_pinned() for a in (mask, E, force))
    if not pinned:
        return mask, E, force, lambda i: None
    cur = torch.cuda.current_stream()
    side = _COPY_STREAMS.get(cur.device.index)
    if side is None:
        side = _COPY_STREAMS[cur.device.index] = torch.cuda.Stream(device=cur.device)
    side.wait_stream(cur)                         # nothing earlier on the current stream is overtaken
    out, events = [], []
    with torch.cuda.stream(side):
        for a in (mask, E, force):
            d = a.to("cuda", non_blocking=True)
            d.record_stream(cur)                  # freed only after the current stream's uses
            ev = torch.cuda.Event()
            ev.record(side)
            out.append(d)
            events.append(ev)
    return out[0], out[1], out[2], lambda i: cur.wait_event(events[i])


def clear_solver_cache():
    """Drop the solvers that solve() keeps for recent set-ups (their device memory returns to the
    caching allocator)."""
    _SOLVERS.clear()


def solve(shape, E, force, mask, *, ke=None, precision="mixed", tol=1e-8, maxiter=200, check_every=1, pre=2,
          post=2, omega=0.6, max_coarse_x=16, levels=None, out=None):
    """Host-buffer entry point: E (Ne), force and 0/1 DOF mask (3N), numpy, author layout.
    Returns (u as numpy, dict(iterations, converged, rel, matvecs, compliance)).  With `out` (a host
    float64 array or CPU tensor of 3N entries, e.g. pinned memory reused across calls) the solution
    is written there and `out` is returned: a pinned buffer takes the copy at full PCIe / C2C speed,
    where a fresh pageable array is staged by the driver at a fraction of it.

    Solvers are kept for the last few set-ups (grid, element, precision, cycle, damping, levels):
    a call with a known set-up copies its inputs into that solver and recomputes every level's
    moduli, masks, diagonals and the coarsest factor from them, reusing the device buffers and
    the captured solve graph.  With pinned CPU tensors as inputs the force is copied to the device
    while the hierarchy refresh and the coarsest factorisation run."""
    shape = tuple(int(v) for v in shape)
    ke_key = None if ke is None else np.asarray(ke, dtype=np.float64).tobytes()
    om_key = tuple(omega) if isinstance(omega, (list, tuple)) else omega
    key = (shape, ke_key, precision, int(check_every), int(pre), int(post), om_key, int(max_coarse_x), levels)
    s = _SOLVERS.pop(key, None)
    mask, E, force, wait = _stage_inputs(mask, E, force)
    wait(0)
    wait(1)
    if s is None:
        s = ElasticitySolver(shape, E, mask, ke=ke, precision=precision, pre=pre, post=post, omega=omega,
                             max_coarse_x=max_coarse_x, levels=levels, tol=tol, maxiter=maxiter,
                             check_every=check_every)
    else:
        s.update(E, mask)
    _SOLVERS[key] = s
    while len(_SOLVERS) > _SOLVER_CACHE_SIZE:
        _SOLVERS.popitem(last=False)
    s.fcg.tol, s.fcg.maxiter = float(tol), int(maxiter)
    wait(2)
    f = _dev(force)
    s.fcg.launch(f, dot_with=f)                    # the compliance f . u comes back with the solver scalars
    res = s.fcg.finish()
    if out is None:
        u = res.x.cpu().numpy()
    else:
        o = out if isinstance(out, torch.Tensor) else torch.from_numpy(out)
        if o.dtype != torch.float64 or o.numel() != res.x.numel() or o.is_cuda or not o.is_contiguous():
            raise ValueError(f"out must be a contiguous host float64 buffer of {res.x.numel()} entries")
        o.view(-1).copy_(res.x)
        u = out if not isinstance(out, torch.Tensor) else out.numpy()
    return u, dict(iterations=res.iterations, converged=res.converged, rel=res.rel, matvecs=res.matvecs,
                   compliance=float(s.fcg.last_dot))
