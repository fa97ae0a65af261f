"""The donor SIMP code's solver and driver interfaces, as drop-ins over the device kernels.

The reference's session-A experiments call the donor module
experiments/session_a/donor/src/gpu_fem/simp_r2.py by these names and signatures:

* `pcg(matvec, b, M_inv, x0=None, tol=1e-5, maxiter=20000, mask=None, check_every=50,
  residual_history=None) -> (x, iters, converged, rel_resid)`  (simp_r2.py:187-295): Jacobi-PCG,
  Fletcher-Reeves beta, the stopping test on the true residual b - A x every `check_every`
  iterations with residual replacement, a pAp == 0 breakdown guard;
* `pcg_ir(matvec64, b64, matvec32, M_inv32, tol=1e-5, mask32=None, inner_tol=1e-1, max_outer=40,
  inner_maxiter=4000, check_every=50, trace=None, x0=None) -> (x, outer, inner_total, converged,
  rel)`  (simp_r2.py:298-385): FP64 residual, FP32 correction of the scaled residual, a divergence
  guard that undoes a step and tightens the inner tolerance tenfold;
* `LinearSolveNotConverged` (simp_r2.py:47-53), `project` / `dproject` (:388-404, the Heaviside
  projection and its derivative), `DEFAULT_SCHEDULE` / `schedule_at` (:410-431), `oc_update`
  (:484-545, OC bisecting on the projected volume, bracket seeded from the last multiplier) and
  `run_simp` (:552-918, the continuation loop under the fail-closed rule: a warm-started solve that
  misses tolerance is retried from zero, a second miss raises).

Any callable works as `matvec` (the loop then runs like the donor's, with its per-iteration
breakdown check).  A `DirichletOperator` of this package routes the whole solve to the
device-scalar solvers instead: `solver.JacobiPCG` (one CUDA-graph WHILE launch per solve) and
`solver.PCGIR`, with the same iterates.  Vectors are CUDA tensors.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from .element import quadrature
from .operators import VoxelOperator, node_mask_from_dofs, simp_modulus
from .solver import PCGIR, JacobiPCG


class LinearSolveNotConverged(RuntimeError):
    """A linear solve missed its tolerance twice (a warm-started attempt and a retry from zero): the
    run is invalid under the fail-closed rule (donor simp_r2.py:47-53)."""


class DirichletOperator:
    """matvec(u) = M K(E) (M u) + (I - M) u on one grid, modulus and mask (float64 or float32): the
    donor's `matvec` (OperatorSuite.matvec_full with the mask applied on both sides).  Calling it
    launches one fused kernel; handing it to pcg / pcg_ir runs the whole solve on the device."""

    def __init__(self, shape, E, mask, ke=None, dtype=torch.float64):
        self.shape = tuple(int(s) for s in shape)
        self.dtype = dtype
        ke = quadrature([1.0, 1.0, 1.0], 0.3) if ke is None else np.asarray(ke, dtype=np.float64).reshape(24, 24)
        self.op = VoxelOperator(self.shape, ke, dtype)
        self.E = E.to(device="cuda", dtype=dtype).contiguous()
        m = mask.to("cuda")
        self.node_mask = m.contiguous() if m.dtype == torch.uint8 else node_mask_from_dofs(m.to(torch.float64))
        self.calls = 0

    def set_modulus(self, E):
        self.E.copy_(E.to(self.dtype))

    def inverse_diagonal(self):
        """1 / diag K on free DOFs, 0 on fixed ones (the donor's M_inv, simp_r2.py:674-675)."""
        d = self.op.diagonal(self.E)
        free = torch.stack([(self.node_mask.to(torch.int32) >> c) & 1 for c in range(3)], 1).reshape(-1)
        return torch.where(d > 0, 1.0 / torch.clamp(d, min=1e-300), torch.zeros_like(d)) * free.to(self.dtype)

    def __call__(self, u):
        self.calls += 1
        return self.op.matvec(u.contiguous(), self.E, self.node_mask)


def _norm(v):
    return float(torch.linalg.vector_norm(v.double()))


def pcg(matvec, b, M_inv, x0=None, tol=1e-5, maxiter=20000, mask=None, check_every=50, residual_history=None):
    """Jacobi-PCG tested on the true residual (donor simp_r2.py:187-295).  Returns (x, iters,
    converged, rel_resid) with rel_resid = |b - A x| / |b| formed explicitly."""
    if isinstance(matvec, DirichletOperator) and residual_history is None and b.dtype == matvec.dtype:
        s = JacobiPCG(matvec.op, matvec.E, matvec.node_mask, tol=tol, maxiter=maxiter, check_every=check_every,
                      inv_diag=M_inv.to(matvec.dtype).contiguous())
        x, it, ok, rel = s.solve(b.contiguous(), x0)
        return x.clone(), it, ok, rel
    dt = b.dtype
    x = torch.zeros_like(b) if x0 is None else x0.to(dt).clone()
    if mask is not None:
        x *= mask
    r = b - matvec(x)
    if mask is not None:
        r *= mask
    z = M_inv * r
    p = z.clone()
    rz = torch.dot(r, z)
    b_norm = _norm(b)
    if b_norm <= 0:
        return x, 0, True, 0.0
    tol_abs = tol * b_norm
    r_norm = _norm(r)
    if residual_history is not None:
        residual_history.append(r_norm / b_norm)
    if r_norm <= tol_abs:
        return x, 0, True, r_norm / b_norm
    k = max(1, int(check_every))
    converged, iters = False, 0
    for _ in range(maxiter):
        Ap = matvec(p)
        if mask is not None:
            Ap *= mask
        pAp = torch.dot(p, Ap)
        if float(pAp) == 0.0:
            break
        alpha = rz / pAp
        x = x + alpha * p
        iters += 1
        if iters % k == 0 or iters >= maxiter:
            r = b - matvec(x)                       # the convergence test and the replacement
            if mask is not None:
                r *= mask
            r_norm = _norm(r)
            if residual_history is not None:
                residual_history.append(r_norm / b_norm)
            if r_norm <= tol_abs:
                converged = True
                break
        else:
            r = r - alpha * Ap
        z = M_inv * r
        rz_new = torch.dot(r, z)
        beta = rz_new / rz
        p = z + beta * p
        rz = rz_new
    if not converged:
        r = b - matvec(x)
        if mask is not None:
            r *= mask
        r_norm = _norm(r)
    return x, iters, converged, r_norm / b_norm


def pcg_ir(matvec64, b64, matvec32, M_inv32, tol=1e-5, mask32=None, inner_tol=1e-1, max_outer=40,
           inner_maxiter=4000, check_every=50, trace=None, x0=None):
    """Mixed-precision iterative refinement (donor simp_r2.py:298-385).  Returns (x64, outer,
    inner_total, converged, rel_resid) with rel_resid the true FP64 residual."""
    if (isinstance(matvec64, DirichletOperator) and isinstance(matvec32, DirichletOperator) and trace is None
            and matvec64.shape == matvec32.shape and matvec64.dtype == torch.float64
            and matvec32.dtype == torch.float32):
        ir = PCGIR(matvec64.op, matvec64.E, matvec64.node_mask, tol=tol, inner_tol=inner_tol, max_outer=max_outer,
                   inner_maxiter=inner_maxiter, check_every=check_every, inv_diag32=M_inv32.to(torch.float32),
                   E32=matvec32.E)
        x, outer, inner, ok, rel = ir.solve(b64.contiguous(), x0)
        return x.clone(), outer, inner, ok, rel
    nb = _norm(b64)
    if nb <= 0:
        return torch.zeros_like(b64), 0, 0, True, 0.0
    x = torch.zeros_like(b64) if x0 is None else x0.to(torch.float64).clone()
    inner_total, outer = 0, 0
    tol_in, rel_prev, d_last, scale_last = inner_tol, None, None, 0.0
    for outer in range(1, max_outer + 1):
        r = b64 - matvec64(x)
        rel = _norm(r) / nb
        if trace is not None:
            trace.append(rel)
        if rel <= tol:
            return x, outer - 1, inner_total, True, rel
        if rel_prev is not None and rel > rel_prev and d_last is not None:     # divergence guard: undo
            x = x - d_last.to(torch.float64) * scale_last
            d_last = None
            tol_in *= 0.1
            if tol_in < 1e-5:
                return x, outer, inner_total, False, rel_prev
            continue
        rel_prev = rel
        scale = _norm(r)
        d32, it32, _ok, _res = pcg(matvec32, (r / scale).to(torch.float32), M_inv32, tol=tol_in,
                                   maxiter=inner_maxiter, mask=mask32, check_every=check_every)
        inner_total += it32
        d_last, scale_last = d32, scale
        x = x + d32.to(torch.float64) * scale
    r = b64 - matvec64(x)
    rel = _norm(r) / nb
    if trace is not None:
        trace.append(rel)
    return x, outer, inner_total, bool(rel <= tol), rel


def project(rho_bar, beta, eta=0.5):
    """Smoothed Heaviside projection (donor simp_r2.py:388-394)."""
    if beta <= 1e-12:
        return rho_bar
    tb_eta = math.tanh(beta * eta)
    den = tb_eta + math.tanh(beta * (1.0 - eta))
    return (tb_eta + torch.tanh(beta * (rho_bar - eta))) / den


def dproject(rho_bar, beta, eta=0.5):
    """d project / d rho_bar (donor simp_r2.py:397-404)."""
    if beta <= 1e-12:
        return torch.ones_like(rho_bar)
    tb_eta = math.tanh(beta * eta)
    den = tb_eta + math.tanh(beta * (1.0 - eta))
    ch = torch.cosh(beta * (rho_bar - eta))
    return beta / (den * ch * ch)


# (until_iter, penal, beta, move, rmin_target) -- the donor's four-phase continuation (simp_r2.py:410-416)
DEFAULT_SCHEDULE = [(15, 1.5, 1.0, 0.20, 1.50), (40, 3.5, 4.0, 0.15, 1.35), (65, 4.5, 16.0, 0.08, 1.25),
                    (120, 4.5, 32.0, 0.05, 1.20)]


def schedule_at(it, schedule=None):
    """(penal, beta, move, rmin, in_last_phase) at outer iteration `it` (1-based) (simp_r2.py:419-431)."""
    sch = schedule or DEFAULT_SCHEDULE
    for until, p, beta, move, rmin in sch:
        if it <= until:
            return p, beta, move, rmin, until == sch[-1][0]
    p, beta, move, rmin = sch[-1][1:]
    return p, beta, move, rmin, True


def oc_update(rho, dc, dv, volfrac, move, filt, beta, eta, rho_lb, bisect_tol=1e-8, max_bisect=80, lam_hint=None):
    """One OC step whose bisection enforces the volume of the PROJECTED filtered density, the bracket
    seeded from the previous multiplier (donor simp_r2.py:484-545).  Returns (rho_new, achieved
    volume, multiplier, probes)."""
    dcn = torch.clamp(dc, max=-1e-30)
    dvp = torch.clamp(dv, min=1e-30)

    def design(lmid):
        step = torch.sqrt(-dcn / (lmid * dvp))
        rn = torch.clamp(torch.minimum(torch.maximum(rho * step, rho - move), rho + move), rho_lb, 1.0)
        return rn, float(project(filt.forward(rn), beta, eta).mean())

    probes = 0
    if lam_hint is not None and lam_hint > 0:
        l1, l2 = lam_hint / 4.0, lam_hint * 4.0
        for _ in range(30):                           # expand until the root is bracketed
            _, v1 = design(l1)
            _, v2 = design(l2)
            probes += 2
            if v1 > volfrac and v2 <= volfrac:
                break
            if v1 <= volfrac:
                l1 /= 8.0
            if v2 > volfrac:
                l2 *= 8.0
            if l1 < 1e-30 or l2 > 1e30:
                l1, l2 = 0.0, 1e9
                break
    else:
        l1, l2 = 0.0, 1e9
    rho_new, achieved = design(0.5 * (l1 + l2))
    probes += 1
    lam = 0.5 * (l1 + l2)
    for _ in range(max_bisect):
        if (l2 - l1) <= bisect_tol * (l1 + l2 + 1e-30):
            break
        lam = 0.5 * (l1 + l2)
        rho_new, achieved = design(lam)
        probes += 1
        if achieved > volfrac:
            l1 = lam
        else:
            l2 = lam
    return rho_new, achieved, lam, probes


class _Solve:
    """One equilibrium solve of the loop, fail-closed: a warm-started attempt that misses `tol` is
    retried from zero (its iterations counted), and a second miss raises LinearSolveNotConverged
    (donor simp_r2.py:682-707).  solver: "gmg" (this package's mixed GMG-FCG), "pcg" (donor Jacobi-PCG
    on the device) or "pcg_ir" (donor iterative refinement, FP32 inner solves)."""

    def __init__(self, shape, mask, force, solver, tol, maxiter, levels):
        from .api import ElasticitySolver
        self.kind, self.tol, self.maxiter = solver, float(tol), int(maxiter)
        self.shape, self.force = shape, force
        n = int(np.prod(shape))
        E0 = torch.ones(n, dtype=torch.float64, device="cuda")
        if solver == "gmg":
            self.es = ElasticitySolver(shape, E0, mask, precision="mixed", pre=2, post=2, omega="spectral",
                                       levels=levels, tol=tol, maxiter=maxiter, check_every=5)
        elif solver in ("pcg", "pcg_ir"):
            self.A64 = DirichletOperator(shape, E0, mask)
            if solver == "pcg_ir":
                self.A32 = DirichletOperator(shape, E0, self.A64.node_mask, dtype=torch.float32)
        else:
            raise ValueError(f"unknown solver {solver!r}")

    def __call__(self, E, x0):
        """Returns (u, iterations incl. a retry, rel, retried, ir_outer)."""
        if self.kind == "gmg":
            self.es.update_modulus(E)
            self.es.refresh_omegas(10)
            attempt = lambda start: self.es.solve(self.force, start)
            res = attempt(x0)
            it, ok, rel, retried = res.iterations, res.converged, res.rel, False
            if not ok and x0 is not None:
                retried = True
                res = attempt(None)
                it += res.iterations
                ok, rel = res.converged, res.rel
            u, outer = res.x.clone(), None
        else:
            self.A64.set_modulus(E)
            if self.kind == "pcg":
                M_inv = self.A64.inverse_diagonal()
                u, it, ok, rel = pcg(self.A64, self.force, M_inv, x0=x0, tol=self.tol, maxiter=self.maxiter)
                retried, outer = False, None
                if not ok and x0 is not None:
                    retried = True
                    u, it2, ok, rel = pcg(self.A64, self.force, M_inv, x0=None, tol=self.tol, maxiter=self.maxiter)
                    it += it2
            else:
                self.A32.set_modulus(E)
                u, outer, it, ok, rel = pcg_ir(self.A64, self.force, self.A32, self.A32.inverse_diagonal(),
                                               tol=self.tol, inner_maxiter=self.maxiter, x0=x0)
                retried = False
        if not ok:
            raise LinearSolveNotConverged(
                f"linear solve missed tol={self.tol:g} (relative residual {rel:.3e} after {it} iterations"
                f"{', retried from zero' if retried else ''}); the run is invalid under the fail-closed rule")
        return u, it, rel, retried, outer


def run_simp(shape, mask, force, volfrac=0.30, rmin=1.5, penal=None, E0=1.0, Emin=1e-9, rho_lb=1e-3, eta=0.5,
             cg_tol=1e-5, cg_maxiter=20000, warm_start=True, max_outer=400, schedule=None, conv_drho=0.01,
             conv_dc_rel=1e-4, conv_window=10, fixed_budget=None, solver="gmg", levels=None, verbose=False):
    """The donor's SIMP driver (simp_r2.py:552-918) on the device: continuation in penalisation,
    projection sharpness, move limit and filter radius (`schedule_at`); density filter, Heaviside
    projection and its chain rule; OC on the projected volume; the fail-closed solve; the outer
    convergence test (physical change <= conv_drho and compliance spread over conv_window <=
    conv_dc_rel, after the last phase); and one final solve on the design the run ends on.
    `mask` / `force`: 0/1 DOF mask and load (author layout), e.g. from problems.donor_cantilever.
    Returns the donor's result record (a subset of its keys) with `rho_final_device`."""
    from .simp import ConeFilter
    shape = tuple(int(s) for s in shape)
    n_elem = int(np.prod(shape))
    mask_t = torch.as_tensor(np.asarray(mask, dtype=np.float64), device="cuda")
    F = torch.as_tensor(np.asarray(force, dtype=np.float64), device="cuda") * mask_t
    ke = quadrature([1.0, 1.0, 1.0], 0.3)
    op = VoxelOperator(shape, ke, torch.float64)
    solve = _Solve(shape, mask_t, F, solver, cg_tol, cg_maxiter, levels)
    filt = ConeFilter(*shape, rmin)
    adj_err = filt.check_adjoint()
    rho = torch.full((n_elem,), float(volfrac), dtype=torch.float64, device="cuda")
    u = torch.zeros_like(F)
    history, solve_log = [], []
    total_iters = total_retries = 0
    converged_outer, stop_reason = False, "guard"
    it = 0
    budget = fixed_budget or max_outer
    rho_phys_prev, lam_prev = None, None
    t_start = time.perf_counter()
    t_solve_total = t_adj_total = t_oc_total = 0.0
    while it < budget:
        it += 1
        p_it, beta_it, move_it, rmin_it, last_phase = schedule_at(it, schedule)
        if penal is not None:
            p_it = penal
        filt.set_rmin(rmin_it)
        rho_bar = filt.forward(rho)
        rho_phys = project(rho_bar, beta_it, eta)
        E_e = Emin + (E0 - Emin) * rho_phys ** p_it
        t0 = time.perf_counter()
        u, iters, resid, retried, outer_ir = solve(E_e, u if (warm_start and it > 1) else None)
        torch.cuda.synchronize()
        t_solve = time.perf_counter() - t0
        total_iters += iters
        total_retries += int(retried)
        solve_log.append({"iter": it, "cg_iters": iters, "rel_resid": resid, "ir_outer": outer_ir,
                          "warm": bool(warm_start and it > 1), "retried_from_zero": retried, "solve_s": t_solve,
                          "penal": p_it, "beta": beta_it, "rmin": filt.rmin})
        t1 = time.perf_counter()
        c = float(torch.dot(F, u))
        _, dc_drp = op.energy(u, rho=rho_phys.contiguous(), emin=Emin, emax=E0, penal=p_it)  # -p rho^(p-1)(E0-Emin) ce
        dprj = dproject(rho_bar, beta_it, eta)
        dc_drho = filt.transpose(dc_drp * dprj)
        dv_drho = filt.transpose(dprj / n_elem)
        torch.cuda.synchronize()
        t_adj = time.perf_counter() - t1
        t2 = time.perf_counter()
        rho_old = rho
        rho, achieved_vol, lam, probes = oc_update(rho, dc_drho, dv_drho, volfrac, move_it, filt, beta_it, eta,
                                                   rho_lb, lam_hint=lam_prev)
        lam_prev = lam
        t_oc = time.perf_counter() - t2
        change = float((rho - rho_old).abs().max())
        change_phys = float((rho_phys - rho_phys_prev).abs().max()) if rho_phys_prev is not None else float("inf")
        rho_phys_prev = rho_phys
        t_solve_total += t_solve
        t_adj_total += t_adj
        t_oc_total += t_oc
        history.append({"iter": it, "compliance": c, "change": change,
                        "change_phys": None if math.isinf(change_phys) else change_phys,
                        "vol_phys": achieved_vol, "vol_raw": float(rho.mean()),
                        "grayness": float((4.0 * rho_phys * (1.0 - rho_phys)).mean()), "cg_iters": iters,
                        "rel_resid": resid, "penal": p_it, "beta": beta_it, "move": move_it, "rmin": filt.rmin,
                        "solve_s": t_solve, "adjoint_s": t_adj, "oc_s": t_oc, "oc_probes": probes,
                        "retried": retried})
        if verbose:
            print(f"  it {it:4d}  c={c:.6f}  dr={change:.4f}  V={achieved_vol:.4f}  cg={iters:5d}  r={resid:.2e}"
                  f"  p={p_it:.1f} b={beta_it:.0f}" + ("  [retry]" if retried else ""), flush=True)
        if fixed_budget is None and last_phase and len(history) > conv_window:
            recent = [h["compliance"] for h in history[-(conv_window + 1):]]
            spread = (max(recent) - min(recent)) / max(abs(recent[-1]), 1e-30)
            if change_phys <= conv_drho and spread <= conv_dc_rel:
                converged_outer, stop_reason = True, "outer_criterion"
                break
    if fixed_budget is not None:
        stop_reason = "fixed_budget"
    p_end, beta_end = schedule_at(it, schedule)[:2]
    if penal is not None:
        p_end = penal
    rho_phys = project(filt.forward(rho), beta_end, eta)
    E_end = Emin + (E0 - Emin) * rho_phys ** p_end
    u_f, it_f, res_f, _, _ = solve(E_end, None)                # the final design's own solve, fail-closed
    total_iters += it_f
    solve_log.append({"iter": it + 1, "cg_iters": it_f, "rel_resid": res_f, "ir_outer": None, "warm": False,
                      "retried_from_zero": False, "solve_s": None, "penal": p_end, "beta": beta_end,
                      "rmin": filt.rmin, "final_iterate": True})
    wall = time.perf_counter() - t_start
    return {"solver": solver, "nelx": shape[0], "nely": shape[1], "nelz": shape[2], "n_elem": n_elem,
            "ndof": int(F.numel()), "volfrac": volfrac, "rmin_initial": rmin, "rmin_final": filt.rmin,
            "filter_adjoint_err": adj_err, "E0": E0, "Emin": Emin, "rho_lb": rho_lb, "eta": eta, "cg_tol": cg_tol,
            "cg_maxiter": cg_maxiter, "warm_start": warm_start, "outer_iters": it,
            "outer_converged": converged_outer, "stop_reason": stop_reason,
            "final_compliance": float(torch.dot(F, u_f)),
            "final_compliance_pre_update": history[-1]["compliance"] if history else float("nan"),
            "final_vol_phys": float(rho_phys.mean()),
            "final_grayness": float((4.0 * rho_phys * (1.0 - rho_phys)).mean()),
            "rho_phys_min": float(rho_phys.min()), "E_min_achieved": float(E_end.min()),
            "total_cg_iters": total_iters, "warm_start_retries": total_retries,
            "max_cg_iters_single_solve": max((s["cg_iters"] for s in solve_log), default=0),
            "max_rel_resid": max((s["rel_resid"] for s in solve_log), default=0.0), "solves_at_cap": 0,
            "wall_s": wall, "t_linear_solve_s": t_solve_total, "t_adjoint_s": t_adj_total, "t_oc_s": t_oc_total,
            "history": history, "solve_log": solve_log, "rho_final_device": rho_phys}
