"""Benchmark: time-to-1e-8 solve of the voxel elasticity cantilever on B200, mixed precision
(FP32 GMG V-cycle inside the FP64 flexible CG) vs plain FP64, plus matvec GDOF/s and the
roofline of the dominant kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload gmg_576x288x288|gmg_128x64x64|jacobi_32x16x16|...] [--no-large]

Default workload: the 576x288x288 cantilever (144.6M DOF, 6-level V(2,2)), the largest
single-GPU configuration.  One step = one complete solve (hierarchy already built, inputs
resident) of the workload; the timed region is K steps bracketed by a barrier + synchronize,
timed with CUDA events, max over ranks.  The workload's vectors are far larger than L2
(126 MB), and L2 is flushed by writing a 256 MB buffer between timed steps, outside the event
bracket.  `e2e` is the same solve through the public host-buffer API (voxel_b200.solve):
pinned host inputs in, host solution out, hierarchy refresh included.  With N > 1 (torchrun)
every rank solves its own replica of the workload (the path does not need a collective): weak
scaling.

CPU baseline: on the 144.6M-DOF grid the reference's NumPy solve needs tens of GB of temporaries
and about an hour, so the reference's own compiled C++ product (reference.cc, oracle/_ref,
single-threaded) is timed on a 1/16 slab of the grid and scaled to one solve by the operator
applications the solve performs -- an extrapolation, labelled as such.  The 128x64x64 section
keeps a measured CPU solve (the NumPy restatement of src/voxel_mg.py, all host threads).

`--impl reference` times the reference's CPU implementation on the same workload (rank 0 only):
the C++ product sample above for the 144.6M-DOF grid, the NumPy restatement's full solve for the
smaller grids.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

WORKLOADS = {
    # name: (shape, density spec, V-cycle levels, description)
    "gmg_128x64x64": ((128, 64, 64), ("grf", 8.0, 0), 4,
                      "cantilever 128x64x64 (1.64M DOF), GRF l=8 seed 0 -> [1e-3,1], E0=1 Emin=1e-9 p=3, "
                      "4-level V(2,2) damped Jacobi omega=0.6, tol 1e-8"),
    "gmg_576x288x288": ((576, 288, 288), ("grf", 16.0, 0), 6,
                        "cantilever 576x288x288 (144.6M DOF), GRF l=16 seed 0 -> [1e-3,1], E0=1 Emin=1e-9 p=3, "
                        "6-level V(2,2) damped Jacobi omega=0.6, tol 1e-8"),
    "gmg_256x128x128": ((256, 128, 128), ("grf", 8.0, 0), 5,
                        "cantilever 256x128x128 (12.7M DOF), GRF l=8 seed 0 -> [1e-3,1], E0=1 Emin=1e-9 p=3, "
                        "5-level V(2,2) damped Jacobi omega=0.6, tol 1e-8"),
    "serving": ((256, 128, 128), ("grf", 8.0, 0), None,
                "256 solve requests, Poisson arrivals (seeded, offered load 1.2x the serial FP64 capacity), "
                "grids uniform from 48x24x24/96x48x48/160x80x80/256x128x128, seeded GRF densities l=8, "
                "tol uniform from {1e-6, 1e-8}, mixed GMG-PCG V(2,2) omega=0.6, HBM budget 150 GB"),
    "simp_192x96x96": ((192, 96, 96), ("simp", 0.12, 0), 5,
                       "SIMP topology optimisation, 100 iterations: cantilever 192x96x96 (5.45M DOF), volume fraction "
                       "0.12, p=3, start 0.12+U(-0.01,0.01) seed 0, hat filter rmin 1.5, OC move 0.2 bisection to 1e-6, "
                       "mixed GMG-PCG V(2,2) spectral omega, solves warm-started to 1e-6, 5 levels"),
    "jacobi_32x16x16": ((32, 16, 16), ("uniform", 0), None,
                        "cantilever 32x16x16 (28,611 DOF), uniform(0.01,1) seed 0, Jacobi-PCG, tol 1e-8"),
}
CHECK_EVERY = 5   # the reference fcg's default true-residual cadence


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="gmg_576x288x288")
    ap.add_argument("--no-large", action="store_true", help="skip the 144.6M-DOF section")
    ap.add_argument("--profile", action="store_true", help="short run for a profiler: no CPU baseline, no large")
    ap.add_argument("--host-loop", action="store_true",
                    help="launch the CG loop body from the host instead of the WHILE graph (the same kernels; "
                         "a profiler then lists every launch)")
    ap.add_argument("--slabs", type=int, default=0,
                    help="x-slab decomposition of the workload's grid: under torchrun one slab per rank "
                         "(exchange over NCCL), else this many slabs on one GPU (exchange by device copies)")
    ap.add_argument("--kernels", action="store_true",
                    help="only launch the hot kernels on the workload's data (for an ncu capture); prints their times")
    ap.add_argument("--stream-kernel", choices=("xp", "zp"), default="xp",
                    help="streaming operator kernel for FP64 / FP32 iterates (vx_set_stream_kernel)")
    ap.add_argument("--tc", action="store_true",
                    help="with --kernels: the tensor-core element-block operator (4 launches) instead")
    return ap.parse_args()


# ----------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ----------------------------------------------------------------------------------- problems
def build_inputs(name, device="cuda"):
    import torch
    import voxel_b200 as vx
    shape, dens, levels, _ = WORKLOADS[name]
    rho = vx.problems.density(dens, shape, device=device)
    E = vx.problems.simp_modulus(rho, 1e-9)
    mask, force = vx.problems.cantilever_equal_split(shape, device=device)
    return shape, levels, rho, E, mask, force


# DRAM bytes per grid node of one launch, from single-kernel ncu captures of the same kernels on the
# 256x128x128 grid (4,276,737 nodes): dram__bytes_read.sum + dram__bytes_write.sum / nodes.  Scaled by
# the node count of the measured launch (the traffic of these streaming kernels grows with the nodes).
NCU_TRAFFIC_PER_NODE = {"jacobi_sweep_f32": (175.528960e6 + 36.767744e6) / 4276737,
                        "apply_dot_f64": (140.506880e6 + 71.061504e6) / 4276737}
NCU_TRAFFIC_SOURCE = "ncu dram bytes of the same kernel on 256x128x128, per node, scaled by nodes"


def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------------------------------- timing
def max_over_ranks(t_local, world, device):
    """The slowest rank's time (every rank gets it); the timed region ends when the last replica does."""
    if world <= 1:
        return float(t_local)
    import torch
    import torch.distributed as dist
    tt = torch.tensor([float(t_local)], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt)


def whole_job_time_per_solve(t_max, world):
    """N replicas each finish one solve per step within t_max: whole-job time per solve."""
    return t_max / world

def time_solves(solver, force, steps, warmup, flush, rank_sync):
    import torch
    for _ in range(warmup):
        solver.solve(force)
    torch.cuda.synchronize()
    times, results = [], []
    rank_sync()
    torch.cuda.nvtx.range_push("timed")                   # ncu --nvtx --nvtx-include timed/
    for _ in range(steps):
        flush.fill_(1.0)                                   # evict L2 (outside the timed bracket)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        res = solver.solve(force)
        e.record()
        e.synchronize()
        times.append(s.elapsed_time(e) / 1e3)
        results.append(res)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    rank_sync()
    return times, results[-1]


def kernel_time(fn, reps, flush):
    """Average device time of one launch of fn (CUDA events on the launching stream), L2 flushed
    before each launch, over `reps` launches."""
    import torch
    fn()
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(reps):
        flush.fill_(1.0)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        e.synchronize()
        tot += s.elapsed_time(e)
    return tot / reps / 1e3


def stream_bytes(nodes, elems, vec_bytes, e_bytes, n_vec_in, n_vec_out, mask=True):
    """Algorithmic HBM bytes of one streaming-operator launch: each array crosses HBM once."""
    return nodes * 3 * vec_bytes * (n_vec_in + n_vec_out) + elems * e_bytes + (nodes if mask else 0)


def vec_bytes(nodes, elems, vector_sizes, e_bytes, mask=True):
    """Algorithmic bytes of a launch reading/writing vectors of the given element sizes once each."""
    return nodes * 3 * sum(vector_sizes) + elems * e_bytes + (nodes if mask else 0)


def mg_mode(M):
    """Short name of a hierarchy's storage mode: f64, f32, bf16 (bf16 auxiliaries) or bf16all."""
    import torch
    if M.dtype == torch.bfloat16:
        return "bf16all"
    if M.aux_dtype == torch.bfloat16:
        return "bf16"
    return "f32" if M.dtype == torch.float32 else "f64"


def kernel_table(solver, vx, torch, flush, reps=10):
    """Per-kernel device time and algorithmic bytes of the hot kernels on the solver's own data."""
    fcg, M = solver.fcg, solver.M
    op64 = fcg.op
    N, Ne = op64.nodes, op64.n_elem
    rows = {}
    tmp = torch.zeros_like(fcg.x)
    t = kernel_time(lambda: op64.apply_dot(fcg.p, fcg.E, fcg.mask, fcg.q, fcg.partials), reps, flush)
    rows["apply_dot_f64"] = (t, stream_bytes(N, Ne, 8, 8, 1, 1))
    t = kernel_time(lambda: op64.true_residual(fcg.x, fcg.b, fcg.E, fcg.mask, tmp, fcg.partials), reps, flush)
    rows["true_residual_f64"] = (t, stream_bytes(N, Ne, 8, 8, 2, 1))
    if hasattr(M, "levels") and len(M.levels) > 1:
        L = M.levels[0]
        xb, rb = L.x.element_size(), L.r.element_size()
        name = mg_mode(M)
        t = kernel_time(lambda: L.op.jacobi(L.x, L.r, L.invd, L.E, L.mask, L.omega, out=L.xt), reps, flush)
        rows[f"jacobi_sweep_{name}"] = (t, vec_bytes(N, Ne, (xb, rb, rb, xb), rb))
        res = L.xt if L.res is None else L.res
        t = kernel_time(lambda: L.op.residual(L.x, L.r, L.E, L.mask, out=res), reps, flush)
        rows[f"residual_{name}"] = (t, vec_bytes(N, Ne, (xb, rb, rb), rb))
    return rows


def coarse_factor_time(solver, flush, reps=3):
    """Device time of the coarsest level's factorisation (banded Cholesky and packed inverse factor,
    vx_coarse_factor) on the solver's own coarse matrix.  Every hierarchy refresh runs it, so it is
    part of each e2e call."""
    M = solver.M
    if getattr(M, "A_coarse", None) is None or M.A_coarse.dim() != 2:
        return None
    n = int(M.A_coarse.shape[0])
    nx, ny, nz = M.levels[-1].shape
    bw = min(n - 1, 3 * ((ny + 1) * (nz + 1) + (nz + 1) + 1) + 2)
    return {"ms": kernel_time(M._coarse_inverse, reps, flush) * 1e3, "n": n, "bw": bw}


# ----------------------------------------------------------------------------------- arms
def solve_arm(shape, E, mask, force, precision, kw, args, flush, rank_sync):
    """Build a solver of `precision`, time it (CUDA events, L2 flushed), return (solver, times, result)."""
    from voxel_b200.api import ElasticitySolver
    s = ElasticitySolver(shape, E, mask, precision=precision, **kw)
    times, res = time_solves(s, force, args.steps, args.warmup, flush, rank_sync)
    return s, times, res


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    import voxel_b200 as vx
    from voxel_b200 import _lib
    from voxel_b200.api import ElasticitySolver, clear_solver_cache

    def rank_sync():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")     # 256 MB > L2
    shape, levels, rho, E, mask, force = build_inputs(args.workload)
    del rho
    precision = "jacobi" if levels is None else "mixed"
    kw = dict(tol=1e-8, maxiter=5000 if levels is None else 200, check_every=50 if levels is None else CHECK_EVERY,
              graph=not args.host_loop)
    if levels is not None:
        kw.update(pre=2, post=2, omega=0.6, levels=levels)
    solver = ElasticitySolver(shape, E, mask, precision=precision, **kw)

    hbm, peak_kind = peaks()
    with ClockSampler(local_rank) as clocks:
        launches0 = _lib.launches
        times, res = time_solves(solver, force, args.steps, args.warmup, flush, rank_sync)
        launches = (_lib.launches - launches0)
    launches_per_solve = launches // (args.steps + args.warmup)
    t_local = float(np.mean(times))
    t_max = max_over_ranks(t_local, world, "cuda")
    compliance = float(force @ res.x)
    out = {"metric": "time-to-1e-8 solve, mixed-precision GMG-PCG (FP32 V-cycle in FP64 flexible CG)"
                     if levels is not None else "time-to-1e-8 solve, FP64 Jacobi-PCG",
           "value": whole_job_time_per_solve(t_max, world), "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": t_max * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64 outer / f32 preconditioner" if levels is not None else "f64", "data": "synthetic",
           "config": {"workload": args.workload, "description": WORKLOADS[args.workload][3],
                      "check_every": kw["check_every"]},
           "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
           "l2": "inputs larger than L2, and flushed (256 MB write) between timed steps",
           "solve": {"iterations": res.iterations, "converged": res.converged, "rel_residual": res.rel,
                     "matvecs": res.matvecs, "compliance": compliance, "step_s": times},
           "gpu_launches": int(launches_per_solve * args.steps)}

    # FP64 and bf16-storage arms (same hierarchy shapes)
    if levels is not None:
        del solver
        torch.cuda.empty_cache()
        s64, times64, r64 = solve_arm(shape, E, mask, force, "fp64", kw, args, flush, rank_sync)
        out["fp64"] = {"value": float(np.mean(times64)), "iterations": r64.iterations,
                       "compliance": float(force @ r64.x), "rel_residual": r64.rel}
        out["speedup_mixed_vs_fp64"] = float(np.mean(times64)) / t_local
        del s64
        torch.cuda.empty_cache()
        sb, times_b, rb = solve_arm(shape, E, mask, force, "bf16", kw, args, flush, rank_sync)
        out["bf16"] = {"value": float(np.mean(times_b)), "iterations": rb.iterations,
                       "compliance": float(force @ rb.x), "rel_residual": rb.rel,
                       "speedup_vs_fp64": float(np.mean(times64)) / float(np.mean(times_b))}
        del sb
        torch.cuda.empty_cache()
        solver = ElasticitySolver(shape, E, mask, precision=precision, **kw)
        solver.solve(force)

    # roofline of the dominant kernel (largest share of one solve) on the solver's own data
    table = kernel_table(solver, vx, torch, flush)
    counts = per_solve_counts(solver, res, levels)
    share = {k: table[k][0] * counts.get(k, 0) for k in table}
    dom = max(share, key=share.get)
    t_dom, b_dom = table[dom]
    tpn = NCU_TRAFFIC_PER_NODE.get(dom)
    out["roofline"] = {"kernel": dom, "bound": "hbm", "achieved": b_dom / t_dom / 1e9, "peak": hbm, "unit": "GB/s",
                       "frac": b_dom / t_dom / 1e9 / hbm, "traffic": None if tpn is None else tpn * solver.op64.nodes,
                       "traffic_source": NCU_TRAFFIC_SOURCE, "peak_kind": peak_kind,
                       "bytes_per_launch": b_dom, "launch_s": t_dom,
                       "kernels": {k: {"launch_us": v[0] * 1e6, "GB/s": v[1] / v[0] / 1e9, "frac_hbm": v[1] / v[0] / 1e9 / hbm,
                                       "per_solve": counts.get(k, 0)} for k, v in table.items()}}
    out["matvec"] = {"GDOF/s_f64_apply": 3 * solver.op64.nodes / table["apply_dot_f64"][0] / 1e9}
    out["coarse_factor"] = coarse_factor_time(solver, flush)
    out["clocks"] = clocks.summary()
    products = products_per_solve(res, levels, 2, 2, kw["check_every"])
    del solver
    torch.cuda.empty_cache()

    # e2e through the public host-buffer API (pinned inputs, refresh + solve + result read back)
    Eh = E.cpu().pin_memory()
    fh = force.cpu().pin_memory()
    mh = mask.cpu().pin_memory()
    del E, mask
    e2e = []
    api_kw = dict(kw)
    api_kw.pop("levels", None)
    api_kw.pop("graph", None)
    uh = torch.empty(fh.numel(), dtype=torch.float64, pin_memory=True)       # the caller's result buffer
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        if i >= args.warmup:
            torch.cuda.nvtx.range_push("e2e")             # ncu --nvtx --nvtx-include e2e/
        t0 = time.perf_counter()
        u, info = vx.solve(shape, Eh, fh, mh, precision=precision, levels=levels, out=uh, **api_kw)
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e.append(time.perf_counter() - t0)
            torch.cuda.nvtx.range_pop()
    out["e2e"] = {"value": float(np.mean(e2e)), "unit": "s", "h2d_bytes_per_step": int(Eh.numel() * 8 + fh.numel() * 8 + mh.numel() * 8),
                  "d2h_bytes_per_step": int(fh.numel() * 8),
                  "includes": "H2D of E/force/0-1 DOF mask from pinned memory, hierarchy refresh (moduli, masks, "
                              "diagonals, coarsest factor), solve, D2H of u into a pinned buffer (vx.solve(..., out=))",
                  "compliance": info["compliance"], "step_s": e2e}
    del uh
    clear_solver_cache()
    del Eh, fh, mh
    torch.cuda.empty_cache()

    if rank == 0 and world == 1 and not args.profile and not args.no_large:
        if args.workload == "gmg_576x288x288":
            out["gmg_128x64x64"] = small_section(args, flush, rank_sync)
            out["serving"] = serving_section(n=64, per_stream_slots=8)
            simp_line = run_simp_bench(args)
            out["simp_192x96x96"] = {k: simp_line[k] for k in ("metric", "value", "unit", "ms_per_step", "simp",
                                                               "fd_check", "clocks")}
        else:
            out["large"] = large_section(args, flush, rank_sync)
        out["matvec_sweep"] = matvec_sweep(flush)
    if rank == 0 and world == 1 and not args.profile:
        if args.workload == "gmg_576x288x288":
            out["cpu_baseline"] = cpu_reference_product_baseline(args.workload, products, steps=1)
        else:
            out["cpu_baseline"] = cpu_baseline(args.workload)
    return out


def products_per_solve(res, levels, pre, post, check_every):
    """Fine-grid operator applications of one mixed GMG-FCG solve (the unit the CPU baseline's
    product time is scaled by): per iteration one outer A p, a true residual every `check_every`
    iterations, and per V-cycle (pre - 1) + 1 + post products on every smoothed level (the first
    pre-sweep starts from x = 0 and needs none), each coarser level 1/8 of the one above."""
    it = int(res.iterations) if res is not None else REFERENCE_ITERATIONS
    levels_f = sum(8.0 ** -l for l in range(levels - 1))
    per_cycle = ((pre - 1) + 1 + post) * levels_f
    return float(it * (1.0 + per_cycle) + it / check_every + 1 + per_cycle + 1)


# FCG iterations of the 576x288x288 workload's mixed solve to 1e-8 (measured on the B200: the b200
# arm's solve.iterations); the reference arm scales its C++ product time by it.
REFERENCE_ITERATIONS = 20


def cpu_reference_product_baseline(workload, products, steps=1):
    """The reference's own C++ product (experiments/session_a/inputs/reference.cc, compiled into
    oracle/_ref by oracle/Makefile; single-threaded) on a 1/16 slab of the workload's grid: the
    slab's natural-layout z extent is nz/16 (the per-element cost is uniform).  Returns the slab
    time scaled to the full grid and, by `products`, to one solve (extrapolated, not measured).
    Without oracle/_ref the NumPy restatement of the reference product takes its place (kind port)."""
    sys.path.insert(0, str(REPO))
    from oracle import ref_product, voxel_oracle as vo
    (nx, ny, nz), _, _, _ = WORKLOADS[workload]
    slab = (nx, ny, max(1, nz // 16))
    scale = nz / slab[2]
    rng = np.random.default_rng(0)
    ne = slab[0] * slab[1] * slab[2]
    rho = 1e-3 + (1 - 1e-3) * rng.random(ne)
    u = rng.standard_normal(3 * (slab[0] + 1) * (slab[1] + 1) * (slab[2] + 1))
    mask = np.ones((slab[2] + 1, slab[1] + 1, slab[0] + 1, 3))
    mask[:, :, 0, :] = 0.0                                     # natural layout, clamped x = 0 face
    mask = mask.ravel()
    ke = vo.quadrature([1, 1, 1], 0.3)
    if ref_product.available():
        ref = ref_product.ReferenceProduct()
        fn, kind, what = (lambda: ref.product(slab, rho, u, ke, mask, 1e-9)), "reference", \
            "reference.cc product() (oracle/_ref, g++ -O3, one thread)"
    else:
        fn, kind, what = (lambda: vo.c_reference_product(slab, rho, u, ke, mask, 1e-9)), "port", \
            "NumPy restatement of reference.cc product() (oracle/voxel_oracle.py)"
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    t_slab = float(np.mean(ts))
    t_full = t_slab * scale
    return {"value": t_full * products, "unit": "s", "cores": 1, "kind": kind, "extrapolated": True,
            "sample": f"{what} on a {slab[0]}x{slab[1]}x{slab[2]} slab (1/{scale:g} of the grid's elements), "
                      f"scaled by element count to one full-grid product ({t_full:.3f} s) and by the "
                      f"{products:.1f} fine-grid operator applications of one solve; the CPU solve itself is not run",
            "product_s": t_full, "slab_s": ts, "products_per_solve": products, "host_cpus": os.cpu_count()}


def small_section(args, flush, rank_sync):
    """128x64x64 (1.64M DOF): mixed and FP64 solves on the B200 and the reference algorithm's
    measured CPU solve (NumPy restatement, all host threads) on the same inputs."""
    import torch
    name = "gmg_128x64x64"
    shape, levels, rho, E, mask, force = build_inputs(name)
    del rho
    kw = dict(tol=1e-8, maxiter=200, check_every=CHECK_EVERY, pre=2, post=2, omega=0.6, levels=levels)
    out = {"workload": name, "description": WORKLOADS[name][3]}
    for prec in ("mixed", "fp64"):
        s, times, res = solve_arm(shape, E, mask, force, prec, kw, args, flush, rank_sync)
        out[prec] = {"s": float(np.mean(times)), "iterations": res.iterations, "rel": res.rel,
                     "compliance": float(force @ res.x)}
        if prec == "mixed":
            out["coarse_factor"] = coarse_factor_time(s, flush)
        del s
    torch.cuda.empty_cache()
    cpu = cpu_baseline(name)
    out["cpu_port"] = cpu
    out["speedup_mixed_vs_cpu"] = cpu["value"] / out["mixed"]["s"]
    return out


def run_slab_bench(args, rank, world, local_rank):
    """The workload's mixed GMG-PCG solve on an x-slab decomposition of its grid (strong scaling:
    the global problem is fixed).  Under torchrun slab i is rank i's and shared planes travel over
    NCCL; in one process `--slabs K` slabs share the GPU and exchange by device copies, which
    measures the decomposition's own cost (layer contributions, plane fixes, owned-prefix dots,
    the host-driven loop) against the single-grid solver."""
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    from voxel_b200 import _lib
    from voxel_b200.api import ElasticitySolver
    from voxel_b200.slab import SlabSolver

    def rank_sync():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    nparts = world if world > 1 else args.slabs
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    shape, levels, rho, E, mask, force = build_inputs(args.workload)
    del rho
    kw = dict(tol=1e-8, maxiter=200, check_every=CHECK_EVERY, pre=2, post=2, omega=0.6, levels=levels)
    s = SlabSolver(shape, E, mask, nparts, precision="mixed", graph=not args.host_loop, **kw)
    with ClockSampler(local_rank) as clocks:
        launches0 = _lib.launches
        times, res = time_solves(s, force, args.steps, args.warmup, flush, rank_sync)
        launches = _lib.launches - launches0
    t_max = max_over_ranks(float(np.mean(times)), world, "cuda")
    x = s.gather()
    out = {"metric": "time-to-1e-8 solve, mixed-precision GMG-PCG on an x-slab decomposition", "value": t_max,
           "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max * 1e3,
           "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
           "dtype": "f64 outer / f32 preconditioner", "data": "synthetic",
           "config": {"workload": args.workload, "description": WORKLOADS[args.workload][3], "slabs": nparts,
                      "bounds": s.M.bounds, "check_every": CHECK_EVERY,
                      "parallelism": f"x-slab x{nparts} over NCCL" if world > 1 else f"x-slab x{nparts} on one GPU",
                      "l2": "flushed (256 MB write) between timed steps"},
           "solve": {"iterations": res.iterations, "converged": res.converged, "rel_residual": res.rel,
                     "compliance": float(force @ x), "step_s": times},
           "gpu_launches": int(launches // (args.steps + args.warmup) * args.steps), "clocks": clocks.summary()}
    if world == 1:
        del s
        torch.cuda.empty_cache()
        for graph in (True, False):
            one = ElasticitySolver(shape, E, mask, precision="mixed", graph=graph, **kw)
            t1, r1 = time_solves(one, force, args.steps, args.warmup, flush, rank_sync)
            out["single_grid_graph" if graph else "single_grid_host_loop"] = {
                "value": float(np.mean(t1)), "iterations": r1.iterations, "compliance": float(force @ r1.x)}
            del one
    return out


def per_solve_counts(solver, res, levels):
    it = res.iterations
    if levels is None:
        return {"apply_dot_f64": it, "true_residual_f64": it // 50 + 1}
    k = solver.fcg.check_every
    checks = it // k + (0 if it % k == 0 else 1)
    M = solver.M
    n_sweeps = (M.pre - 1) + M.post
    name = mg_mode(M)
    return {"apply_dot_f64": it, "true_residual_f64": checks, f"jacobi_sweep_{name}": (it + 1) * n_sweeps,
            f"residual_{name}": it + 1}


def large_section(args, flush, rank_sync):
    """144.6M-DOF grid: time-to-1e-8 of FP64 and the three mixed-precision preconditioners (FP32,
    bf16 auxiliaries, all-bf16), with the hot kernels of each."""
    import torch
    import voxel_b200 as vx
    from voxel_b200.api import ElasticitySolver
    name = "gmg_576x288x288"
    shape, levels, rho, E, mask, force = build_inputs(name)
    del rho
    kw = dict(tol=1e-8, maxiter=200, check_every=CHECK_EVERY, pre=2, post=2, omega=0.6, levels=levels)
    hbm, _ = peaks()
    out = {"workload": name, "description": WORKLOADS[name][3]}
    steps, warm = max(2, min(args.steps, 3)), 1
    for prec in ("mixed", "bf16", "bf16-all", "fp64"):
        s = ElasticitySolver(shape, E, mask, precision=prec, **kw)
        times, res = time_solves(s, force, steps, warm, flush, rank_sync)
        out[prec] = {"s": float(np.mean(times)), "iterations": res.iterations, "rel": res.rel,
                     "compliance": float(force @ res.x)}
        table = kernel_table(s, vx, torch, flush, reps=5)
        out[prec]["kernels"] = {k: {"launch_ms": v[0] * 1e3, "GB/s": v[1] / v[0] / 1e9,
                                    "frac_hbm": v[1] / v[0] / 1e9 / hbm} for k, v in table.items()}
        del s
        torch.cuda.empty_cache()
    for prec in ("mixed", "bf16", "bf16-all"):
        out[f"speedup_{prec}_vs_fp64"] = out["fp64"]["s"] / out[prec]["s"]
    return out


SWEEP_GRIDS = ((32, 16, 16), (128, 64, 64), (192, 96, 96), (256, 128, 128), (576, 288, 288))


def matvec_sweep(flush, reps=5):
    """Dirichlet product y = M K M u + (I - M) u alone (one launch, inputs resident, L2 flushed), on
    the grids of every workload, in FP64, FP32 and bf16 storage (u and E in bf16, y in FP32)."""
    import torch
    import voxel_b200 as vx
    hbm, _ = peaks()
    ke = vx.quadrature([1, 1, 1], 0.3)
    rows = []
    for shape in SWEEP_GRIDS:
        mask, _ = vx.problems.cantilever_equal_split(shape)
        nm = vx.node_mask_from_dofs(mask)
        del mask
        g = torch.Generator(device="cuda").manual_seed(1)
        for dt, ydt, label in ((torch.float64, torch.float64, "f64"), (torch.float32, torch.float32, "f32"),
                               (torch.bfloat16, torch.float32, "bf16")):
            op = vx.VoxelOperator(shape, ke, dt)
            u = torch.randn(op.ndof, device="cuda", dtype=torch.float32, generator=g).to(dt)
            E = torch.rand(op.n_elem, device="cuda", dtype=torch.float32, generator=g).to(dt)
            y = torch.empty(op.ndof, device="cuda", dtype=ydt)
            t = kernel_time(lambda: op.matvec(u, E, nm, out=y), reps, flush)
            b = vec_bytes(op.nodes, op.n_elem, (u.element_size(), y.element_size()), E.element_size())
            rows.append({"grid": "x".join(map(str, shape)), "dofs": op.ndof, "storage": label, "us": t * 1e6,
                         "GDOF/s": op.ndof / t / 1e9, "GB/s": b / t / 1e9, "frac_hbm": b / t / 1e9 / hbm})
            del op, u, E, y
        torch.cuda.empty_cache()
    return rows


def cpu_baseline(workload, timed=True):
    """The reference algorithm's NumPy path (oracle restatement of src/voxel_mg.py) on this host,
    same workload: one full solve (about 10-30 s on 8 cores for the 128x64x64 case)."""
    sys.path.insert(0, str(REPO))
    from oracle import voxel_oracle as vo
    shape, dens, levels, _ = WORKLOADS[workload]
    if dens[0] == "grf":
        rho = vo.gaussian_random_field(shape, dens[1], dens[2])
    else:
        rho = np.random.default_rng(dens[1]).uniform(0.01, 1.0, int(np.prod(shape)))
    E = vo.simp_modulus(rho, 1e-9)
    mask, force = vo.cantilever_equal_split(shape)
    ke = vo.quadrature([1, 1, 1], 0.3)
    A = lambda u: vo.apply_dirichlet(shape, ke, E, mask, u)
    t0 = time.perf_counter()
    if levels is None:
        inv = 1 / np.where(mask != 0, vo.product_diagonal(shape, ke, E), 1.0)
        x, it, ok, rel, mv = vo.fcg(A, force, lambda v: inv * v, 1e-8, 5000, check_every=50)
        sample = "one full Jacobi-PCG solve (fcg, check_every 50)"
    else:
        shapes = vo.hierarchy_shapes(shape, 16)[:levels]
        fac = vo.coarse_factor(shapes, ke, E, mask)
        M = vo.Multigrid(shapes, ke, E, mask, fac, np.float32, pre=2, post=2)
        x, it, ok, rel, mv = vo.fcg(A, force, M, 1e-8, 200, check_every=CHECK_EVERY)
        sample = "one full mixed (FP32 V-cycle) GMG-FCG solve incl. hierarchy setup"
    dt = time.perf_counter() - t0
    try:
        from threadpoolctl import threadpool_info
        cores = max([i.get("num_threads", 1) for i in threadpool_info()] + [1])
    except Exception:
        cores = os.cpu_count()
    return {"value": dt, "unit": "s", "cores": cores, "kind": "port", "sample": sample,
            "iterations": it, "rel_residual": rel, "compliance": float(force @ x),
            "host_cpus": os.cpu_count()}


def run_reference(args, rank):
    if rank != 0:
        return None
    if args.workload in ("serving", "simp_192x96x96"):
        return {"impl": "reference", "unavailable": f"no CPU arm for {args.workload}: the CPU port of one solve of its "
                "largest grid alone takes minutes; the CPU baseline is timed on the gmg and jacobi workloads"}
    shape, _, levels, desc = WORKLOADS[args.workload]
    times = []
    for i in range(args.warmup + args.steps):
        if args.workload == "gmg_576x288x288":
            # one step = the reference's C++ product on a 1/16 slab, scaled to one solve
            r = cpu_reference_product_baseline(args.workload, products_per_solve(None, levels, 2, 2, CHECK_EVERY))
        elif i < args.warmup:
            continue            # the NumPy path has no warm-up state; warm-up steps are skipped
        else:
            r = cpu_baseline(args.workload)
        if i >= args.warmup:
            times.append(r["value"])
    v = float(np.mean(times))
    r["value"] = v
    return {"impl": "reference", "metric": "time-to-1e-8 solve, mixed-precision GMG-PCG (FP32 V-cycle in FP64 flexible CG)"
            if levels is not None else "time-to-1e-8 solve, FP64 Jacobi-PCG", "value": v, "unit": "s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 outer / f32 preconditioner" if levels is not None else "f64",
            "data": "synthetic", "config": {"workload": args.workload, "description": desc,
                                            "check_every": 50 if levels is None else CHECK_EVERY},
            "cpu_baseline": r, "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_s": times}


def run_kernels(args):
    """Hot kernels only, on the workload's solver data: 3 launches each (for ncu -k/-c captures)."""
    import torch
    import voxel_b200 as vx
    from voxel_b200.api import ElasticitySolver
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    shape, levels, rho, E, mask, force = build_inputs(args.workload)
    if args.tc:
        from voxel_b200.operators import tc_element_product
        nm = vx.node_mask_from_dofs(mask)
        E32 = E.to(torch.float32)
        u32 = torch.randn(force.numel(), dtype=torch.float32, device="cuda",
                          generator=torch.Generator(device="cuda").manual_seed(0))
        y = torch.empty_like(u32)
        ts = []
        for i in range(4):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            tc_element_product(shape, vx.quadrature([1, 1, 1], 0.3), E32, u32, nm, out=y)
            b.record()
            b.synchronize()
            ts.append(a.elapsed_time(b) * 1e3)
        print(json.dumps({"tc_element_product_us": ts[1:]}))
        return
    s = ElasticitySolver(shape, E, mask, precision="mixed", levels=levels, pre=2, post=2, omega=0.6)
    # launch order of the streaming operator: apply_dot f64 x4, true_residual f64 x4, jacobi f32 x4,
    # residual f32 x4 (one warm-up + 3 timed each)
    table = kernel_table(s, vx, torch, flush, reps=3)
    print(json.dumps({k: {"us": v[0] * 1e6, "GB/s": v[1] / v[0] / 1e9} for k, v in table.items()}))


def run_simp_bench(args):
    """The 192x96x96 SIMP run: 100 density-filtered SIMP iterations on the device, with the autograd
    sensitivity checked by central differences (64 seeded elements, step 1e-6) at the start design."""
    import torch
    import voxel_b200 as vx
    from voxel_b200 import simp
    from voxel_b200.api import ElasticitySolver
    shape, _, levels, desc = WORKLOADS["simp_192x96x96"]
    n = int(np.prod(shape))
    steps = 100
    # ---- finite-difference check of d compliance / d rho at the start design (FP64 solves to 1e-12)
    rho0 = torch.as_tensor(0.12 + np.random.default_rng(0).uniform(-0.01, 0.01, n), device="cuda")
    mask, force = vx.problems.cantilever_equal_split(shape)
    s64 = ElasticitySolver(shape, vx.problems.simp_modulus(rho0, 1e-9), mask, precision="fp64", omega="spectral",
                           levels=levels, tol=1e-12, maxiter=500, check_every=1)
    st = simp.SimpState(s64, force)
    r = rho0.clone().requires_grad_(True)
    simp.compliance(r, st).backward()
    grad = r.grad.cpu().numpy()
    idx = np.random.default_rng(6).choice(n, 64, replace=False)
    h = 1e-6
    u0 = st.u.clone()
    fd = []
    t_fd = time.perf_counter()
    for e in idx:
        vals = []
        for sgn in (1.0, -1.0):
            rr = rho0.clone()
            rr[int(e)] += sgn * h
            st.u = u0.clone()
            vals.append(float(simp.compliance(rr, st)))
        fd.append((vals[0] - vals[1]) / (2 * h))
    t_fd = time.perf_counter() - t_fd
    fd = np.array(fd)
    relerr = np.abs(fd - grad[idx]) / np.abs(grad[idx])
    del s64, st
    torch.cuda.empty_cache()
    # ---- the optimisation (every step: solve, backward, filter transpose, OC bisection, filter)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    with ClockSampler(0) as clocks:
        x, rho, hist = simp.run_simp(shape, volfrac=0.12, rmin=1.5, move=0.2, oc_tol=1e-6, steps=steps, penal=3.0,
                                     precision="mixed", solve_tol=1e-6, noise=0.01, seed=0, levels=levels,
                                     check_every=CHECK_EVERY)
        ev1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    per_step = [h_["seconds"] for h_ in hist]
    return {"metric": "SIMP iteration time (solve + autograd sensitivity + filter + OC bisection), 192x96x96",
            "value": float(np.mean(per_step[1:])), "unit": "s", "n_gpus": 1, "steps": steps, "warmup": 1,
            "ms_per_step": 1e3 * float(np.mean(per_step[1:])), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 outer / f32 preconditioner", "data": "synthetic",
            "config": {"workload": "simp_192x96x96", "description": desc,
                       "timing": "per-step wall time with a device synchronize per step; step 0 (graph capture) excluded",
                       "check_every": CHECK_EVERY},
            "simp": {"total_s_incl_setup": wall, "device_s": ev0.elapsed_time(ev1) / 1e3,
                     "median_step_s": float(np.median(per_step[1:])),
                     "compliance_first_last": [hist[0]["compliance"], hist[-1]["compliance"]],
                     "volume_last": hist[-1]["volume"], "change_last": hist[-1]["change"],
                     "solve_iterations_mean": float(np.mean([h_["iterations"] for h_ in hist])),
                     "oc_probes_mean": float(np.mean([h_["oc_probes"] for h_ in hist]))},
            "clocks": clocks.summary(),
            "fd_check": {"elements": 64, "step": h, "solve_tol": 1e-12, "max_rel_err": float(relerr.max()),
                         "median_rel_err": float(np.median(relerr)), "seconds": t_fd}}


# cached device memory a server keeps for solvers built inside the stream (the cold shape), so that
# no cudaMalloc synchronises the device while jobs are in flight
RESERVE_BYTES = 8e9


def serving_section(n=256, repeats=1, clocks_index=0, per_stream_slots=16):
    """The mixed-size request stream (Poisson arrivals at 1.2x the serial FP64 capacity) through three
    servers: the batched one (jobs of a shape fused into shared launches, one shape built cold inside
    the stream), the per-stream one (a graph per job on its own stream, pooled solvers) and serial
    plain FP64.  Returns the summaries (p50/p99 latency, solves/s)."""
    import torch
    import voxel_b200 as vx
    from voxel_b200 import serving
    shapes = ((48, 24, 24), (96, 48, 48), (160, 80, 80), (256, 128, 128))
    svc = {}
    for s_ in shapes:                       # serial FP64 service time per shape sets the arrival rate
        rho = vx.problems.gaussian_random_field(s_, 8.0, 7)
        mask, force = vx.problems.cantilever_equal_split(s_)
        sol = vx.ElasticitySolver(s_, vx.problems.simp_modulus(rho, 1e-9), mask, precision="fp64", tol=1e-8,
                                  check_every=1)
        sol.solve(force)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = sol.solve(force)
        torch.cuda.synchronize()
        svc[s_] = time.perf_counter() - t0
        if not r.converged:
            raise RuntimeError(f"serial FP64 reference solve on {s_} did not converge: {r}")
        del sol
    torch.cuda.empty_cache()
    mean_service = float(np.mean(list(svc.values())))
    reqs = serving.request_stream(n=n, shapes=shapes, load=1.2, mean_service=mean_service, seed=0)
    out = {"requests": n, "serial_fp64_service_s": {"x".join(map(str, k)): v for k, v in svc.items()}}
    cold = (96, 48, 48)
    runs = []
    with ClockSampler(clocks_index) as clocks:
        for rep in range(repeats):
            done, summ = serving.serve_batched(reqs, shapes=shapes, precision="mixed", chunk=4,
                                               prewarm=[s_ for s_ in shapes if s_ != cold], budget_bytes=150e9,
                                               reserve_bytes=RESERVE_BYTES)
            summ["not_converged"] = [(c.rid, c.shape, c.iterations, c.rel) for c in done if not c.converged][:10]
            runs.append(summ)
            torch.cuda.empty_cache()
        out["batched"] = runs[0] if repeats == 1 else {"runs": runs, "p99_ms": [r["p99_ms"] for r in runs],
                                                       "p50_ms": [r["p50_ms"] for r in runs]}
        slots = per_stream_slots
        warm_shapes = [s_ for s_ in shapes if s_ != cold]
        pruns = []
        for rep in range(repeats):                 # a fresh pool per run: the cold shape is cold every time
            backend = serving.CudaBackend(precision="mixed")
            backend.prewarm(warm_shapes, slots, 150e9)
            warm = serving.request_stream(n=8, shapes=warm_shapes, rate=1e6, seed=99)
            for r in warm:
                r.arrival = 0.0
            sched = serving.Scheduler(serving._PoolCharge(backend), budget_bytes=150e9, max_slots=slots)
            sched.run(warm)
            serving.reserve_device_memory(RESERVE_BYTES)     # the cold shape's solvers come from the cache
            torch.cuda.synchronize()
            sched.peak_inflight = 0
            done, makespan = sched.run(reqs)
            ps = serving.summarize(done, makespan)
            ps.update(peak_inflight=sched.peak_inflight, prewarmed_solvers_per_shape=slots,
                      cold_shapes=["x".join(map(str, cold))])
            pruns.append(ps)
            del backend, sched
            torch.cuda.empty_cache()
        out["per_stream"] = pruns[0] if repeats == 1 else {"runs": pruns, "p99_ms": [r["p99_ms"] for r in pruns],
                                                            "p50_ms": [r["p50_ms"] for r in pruns]}
        serial_done, serial_summary = serving.serve(reqs, precision="fp64", max_slots=1, prewarm=True)
        out["serial_fp64"] = serial_summary
        torch.cuda.empty_cache()
        # a burst: 64 requests of the two small shapes at once, where many same-shape jobs are live
        burst = serving.request_stream(n=64, shapes=shapes[:2], rate=1e6, seed=5)
        for r in burst:
            r.arrival = 0.0
        _, bb = serving.serve_batched(burst, shapes=shapes[:2], precision="mixed", chunk=4, budget_bytes=150e9)
        torch.cuda.empty_cache()
        _, bp = serving.serve(burst, precision="mixed", max_slots=16, prewarm=True)
        torch.cuda.empty_cache()
        out["burst_small"] = {"requests": 64, "shapes": ["x".join(map(str, s_)) for s_ in shapes[:2]],
                              "batched": bb, "per_stream": bp}
    out["clocks"] = clocks.summary()
    return out


def run_serving(args):
    """Continuous batching (fused launches per shape) vs the per-stream server vs serial plain FP64 on
    the same request stream; the batched server is run three times (p99 repeatability)."""
    n = 256 if not args.profile else 32
    sec = serving_section(n=n, repeats=3 if not args.profile else 1,
                          clocks_index=int(os.environ.get("LOCAL_RANK", "0")))
    b = sec["per_stream"]
    p99 = float(np.median(b["p99_ms"])) if "runs" in b else b["p99_ms"]
    return {"metric": "serving p99 latency, mixed-size stream (per-job graphs on concurrent streams, mixed "
                      "GMG-PCG; the fused-launch batched server and serial FP64 beside it)",
            "value": p99, "unit": "ms", "n_gpus": 1, "steps": n, "warmup": 0,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64 outer / f32 preconditioner",
            "data": "synthetic", "config": {"workload": "serving", "description": WORKLOADS["serving"][3]},
            "serving": sec, "clocks": sec.pop("clocks")}


def main():
    args = parse()
    if args.impl == "b200" and args.stream_kernel != "xp":
        from voxel_b200 import _lib
        _lib.set_stream_kernel(args.stream_kernel)
    if args.kernels:
        run_kernels(args)
        return
    if args.workload == "serving" and args.impl == "b200":
        print(json.dumps(run_serving(args)))
        return
    if args.workload == "simp_192x96x96" and args.impl == "b200":
        print(json.dumps(run_simp_bench(args)))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
        if out is not None:
            print(json.dumps(out))
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_slab_bench(args, rank, world, local) if args.slabs else run_b200(args, rank, world, local)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
