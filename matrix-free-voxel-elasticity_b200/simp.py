"""SIMP topology optimisation on the device: the hat density filter, the top88 optimality-criteria
update with its bisection resident on the device, the compliance as a torch.autograd.Function whose
backward is the element-energy kernel, and the optimisation loop.

Reference semantics: the cone filter of experiments/session_a/donor/src/gpu_fem/filter_r2.py:93-183
(same operator as the CSR DensityFilter of experiments/session_h/run_w1b.py:97-125), the top88 OC of
run_w1b.py:46-62 / 82-94 and the density-filtered loop of run_w1b.py:163-205 (`update="top88_gpu"`).
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib
from .api import ElasticitySolver
from .element import quadrature
from .operators import VoxelOperator, _ptr, simp_modulus, stream_ptr
from .solver import _GraphLoop

OC_L1, OC_L2, OC_LMID, OC_VOL, OC_VOLFRAC, OC_TOL, OC_NEL = range(7)
OC_DONE, OC_IT, OC_MAXIT, OC_BREAK, OC_CHECK = 10, 11, 12, 14, 15


class ConeFilter:
    """Matrix-free hat filter on an (nelx, nely, nelz) element grid, author element order:
    forward(rho) = (H rho) / s, transpose(g) = H (g / s), s = H 1."""

    def __init__(self, nelx, nely, nelz, rmin, dtype=torch.float64):
        if dtype != torch.float64:
            raise ValueError("the filter runs in float64")
        self.shape = (int(nelx), int(nely), int(nelz))
        self.n_elem = self.shape[0] * self.shape[1] * self.shape[2]
        self.dtype = dtype
        self._rmin = None
        self.set_rmin(rmin)

    def set_rmin(self, rmin):
        rmin = float(rmin)
        if self._rmin is not None and abs(rmin - self._rmin) < 1e-12:
            return
        self._rmin = rmin
        self._s = self._apply(torch.ones(self.n_elem, dtype=torch.float64, device="cuda"), 0)

    @property
    def rmin(self):
        return self._rmin

    @property
    def row_sums(self):
        return self._s

    def _apply(self, x, mode, out=None):
        x = x.contiguous()
        y = torch.empty_like(x) if out is None else out
        _lib.call("vx_cone_filter", *self.shape, self._rmin, _ptr(x, "x", torch.float64, self.n_elem),
                  None if mode == 0 else self._s.data_ptr(), int(mode), _ptr(y, "y", torch.float64, self.n_elem),
                  stream_ptr())
        return y

    def forward(self, rho, out=None):
        return self._apply(rho, 1, out)

    def transpose(self, g, out=None):
        return self._apply(g, 2, out)

    density, gradient = forward, transpose          # the names of run_w1b.DensityFilter

    def check_adjoint(self, seed=0):
        """|<H a, b> - <a, H^T b>| / max(...) -- guards the chain rule (filter_r2.py:173-183)."""
        g = torch.Generator(device="cuda").manual_seed(seed)
        a = torch.rand(self.n_elem, dtype=torch.float64, device="cuda", generator=g)
        b = torch.rand(self.n_elem, dtype=torch.float64, device="cuda", generator=g)
        lhs, rhs = float(self.forward(a) @ b), float(a @ self.transpose(b))
        return abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-300)


class OCUpdater:
    """top88 optimality-criteria update; the bisection runs on the device as one WHILE graph."""

    def __init__(self, filt: ConeFilter, graph=True):
        self.filt = filt
        n = filt.n_elem
        self.n = n
        self.w = filt.transpose(torch.ones(n, dtype=torch.float64, device="cuda"))   # H (1 / s)
        self.S = torch.zeros(16, dtype=torch.float64, device="cuda")
        self.S_host = torch.zeros(16, dtype=torch.float64, pin_memory=True)
        self.partials = torch.zeros(int(_lib.load().vx_oc_partials(n)), dtype=torch.float64, device="cuda")
        self.x = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.dc = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.dv = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.x_new = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.move = None
        self.stream = torch.cuda.Stream()
        self.use_graph = graph
        self._graph = None
        self.probes = 0

    def _body(self):
        _lib.call("vx_oc_probe", self.n, self.x.data_ptr(), self.dc.data_ptr(), self.dv.data_ptr(), self.w.data_ptr(),
                  self.move, self.S.data_ptr(), self.partials.data_ptr(), stream_ptr())
        _lib.call("vx_oc_finalize", self.n, self.partials.data_ptr(), self.S.data_ptr(), stream_ptr())

    def __call__(self, x, dc, dv, volfrac, move, tol=1e-3, l2=1e9, max_probes=400):
        """x_new of oc_top88(x, dc, dv, volfrac, move, density=filter.forward, l2, tol)."""
        if self.move is not None and move != self.move:
            self._graph = None                         # the move limit is baked into the graph
        self.move = float(move)
        caller = torch.cuda.current_stream()
        self.stream.wait_stream(caller)
        with torch.cuda.stream(self.stream):
            self.x.copy_(x)
            self.dc.copy_(dc)
            self.dv.copy_(dv)
        if self.use_graph and self._graph is None:
            self._graph = _GraphLoop(self.stream, self.S, self._body)
        with torch.cuda.stream(self.stream):
            init = torch.zeros(16, dtype=torch.float64)
            init[OC_L1], init[OC_L2], init[OC_VOLFRAC], init[OC_TOL] = 0.0, float(l2), float(volfrac), float(tol)
            init[OC_NEL], init[OC_MAXIT], init[OC_CHECK] = float(self.n), float(max_probes), 1.0
            self.S.copy_(init, non_blocking=False)
            if self.use_graph:
                self._graph.launch(self.stream)
            else:
                for _ in range(max_probes):
                    self._body()
                    self.S_host.copy_(self.S)
                    if self.S_host[OC_DONE]:
                        break
            _lib.call("vx_oc_apply", self.n, self.x.data_ptr(), self.dc.data_ptr(), self.dv.data_ptr(), self.move,
                      self.S.data_ptr(), self.x_new.data_ptr(), stream_ptr())
            self.S_host.copy_(self.S, non_blocking=True)
            torch.cuda.current_stream().synchronize()
        caller.wait_stream(self.stream)
        self.probes = int(self.S_host[OC_IT])
        if self.use_graph:
            self._graph.account(self.probes)
        if not self.S_host[OC_DONE]:
            raise RuntimeError(f"OC bisection did not reach tol {tol} in {max_probes} probes")
        return self.x_new.clone()


def oc_top88(x, dc, dv, volfrac, move, filt: ConeFilter, l2=1e9, tol=1e-3):
    """One-shot top88 OC update with the volume of filt.forward(x_new) (run_w1b.py:46-62)."""
    return OCUpdater(filt)(x, dc, dv, volfrac, move, tol=tol, l2=l2)


class SimpState:
    """What the compliance Function needs: the solver (its hierarchy is refreshed per design), the load,
    the SIMP material law and the warm-start displacement."""

    def __init__(self, solver: ElasticitySolver, force, emin=1e-9, e0=1.0, penal=3.0, warm_start=True):
        self.solver, self.force = solver, force.to(torch.float64).contiguous()
        self.emin, self.e0, self.penal = float(emin), float(e0), float(penal)
        self.warm_start = warm_start
        self.u = None
        self.last = None
        self.retried = False          # the last forward solve was retried from zero
        self.iterations = 0           # its iterations, the retry included
        self.op = solver.op64

    def modulus(self, rho):
        return simp_modulus(rho.contiguous(), self.emin, self.e0, self.penal)


class Compliance(torch.autograd.Function):
    """c(rho) = f^T u(rho), K(E(rho)) u = f, E = Emin + (E0 - Emin) rho^p.
    backward: dc/drho_e = -p rho_e^(p-1) (E0 - Emin) u_e^T K0 u_e (self-adjoint: no second solve),
    the element-energy kernel (reference sensitivity: donor simp_r2.py:722-726)."""

    @staticmethod
    def forward(ctx, rho, state: SimpState):
        state.solver.update_modulus(state.modulus(rho.detach()))
        warm = state.u if state.warm_start else None
        res = state.solver.solve(state.force, warm)
        state.retried = False
        iterations = res.iterations
        if not res.converged and warm is not None:
            # fail-closed (donor simp_r2.py:682-707): a warm-started miss is retried from zero, and the
            # retry's iterations are counted
            state.retried = True
            res = state.solver.solve(state.force, None)
            iterations += res.iterations
        if not res.converged:
            from .donor import LinearSolveNotConverged
            raise LinearSolveNotConverged(
                f"linear solve missed tol={state.solver.fcg.tol:g} (relative residual {res.rel:.3e} after "
                f"{iterations} iterations{', retried from zero' if state.retried else ''}); "
                "the result is invalid under the fail-closed rule")
        u = res.x.clone()
        state.u = u
        state.last = res
        state.iterations = iterations
        ctx.state = state
        ctx.save_for_backward(rho.detach(), u)
        return torch.dot(state.force, u).reshape(())

    @staticmethod
    def backward(ctx, grad_c):
        rho, u = ctx.saved_tensors
        st = ctx.state
        _, dc = st.op.energy(u, rho=rho.contiguous(), emin=st.emin, emax=st.e0, penal=st.penal)
        return grad_c * dc, None


def compliance(rho, state):
    return Compliance.apply(rho, state)


def run_simp(shape, volfrac=0.12, rmin=1.5, move=0.2, oc_tol=1e-6, steps=100, emin=1e-9, penal=3.0,
             precision="mixed", solve_tol=1e-6, noise=0.01, seed=0, levels=None, pre=2, post=2, omega="spectral",
             omega_every=10, omega_iterations=10, callback=None, check_every=1):
    """Density-filtered SIMP on the equal-split cantilever (run_w1b.simp_run, update='top88_gpu'):
    x starts at volfrac plus seeded uniform noise; each step solves (mixed GMG-PCG warm-started at
    solve_tol), differentiates the compliance through Compliance.backward, filters the sensitivity
    and applies the top88 OC with its bisection to oc_tol.  check_every: the solves' true-residual
    cadence (the reference fcg's default is 5).  Returns (x, rho, history)."""
    from .problems import cantilever_equal_split
    n = int(np.prod(shape))
    g = np.random.default_rng(seed)
    x = torch.as_tensor(volfrac + g.uniform(-noise, noise, n), device="cuda")
    filt = ConeFilter(*shape, rmin)
    oc = OCUpdater(filt)
    mask, force = cantilever_equal_split(shape)
    rho = filt.forward(x)
    solver = ElasticitySolver(shape, simp_modulus(rho, emin, 1.0, penal), mask, precision=precision, pre=pre, post=post,
                              omega=omega, levels=levels, tol=solve_tol, maxiter=500, check_every=check_every)
    if omega == "spectral":
        solver.refresh_omegas(omega_iterations)
    state = SimpState(solver, force, emin=emin, e0=1.0, penal=penal)
    dv_x = filt.transpose(torch.ones(n, dtype=torch.float64, device="cuda"))
    history = []
    for k in range(steps):
        t0 = time.perf_counter()
        if omega == "spectral" and k % omega_every == 0 and k:
            solver.update_modulus(simp_modulus(rho, emin, 1.0, penal))
            solver.refresh_omegas(omega_iterations)     # the design's contrast grows: keep omega * lambda < 2
        r = rho.clone().requires_grad_(True)
        c = compliance(r, state)
        c.backward()
        dc_x = filt.transpose(r.grad)
        x_new = oc(x, dc_x, dv_x, volfrac, move, tol=oc_tol)
        rho = filt.forward(x_new)
        change = float((x_new - x).abs().max())
        x = x_new
        torch.cuda.synchronize()
        history.append({"step": k, "compliance": float(c.detach()), "iterations": state.iterations,
                        "retried_from_zero": state.retried,
                        "rel": state.last.rel, "change": change, "volume": float(rho.mean()),
                        "oc_probes": oc.probes, "seconds": time.perf_counter() - t0})
        if callback:
            callback(history[-1])
    return x, rho, history
