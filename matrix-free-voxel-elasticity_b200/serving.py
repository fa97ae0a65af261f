"""Continuous-batching solve server.

Requests (elasticity solves on grids of different sizes, each with its own density and tolerance)
arrive over time.  The scheduler admits a request as soon as a slot is free and its device memory
footprint (vectors + multigrid hierarchy + coarsest dense inverse) fits the HBM budget, so work
that arrives while other solves run starts immediately and overlaps with them on the GPU: every
in-flight job owns a CUDA stream, its density, its hierarchy and its captured whole-solve graph,
and the host only polls completion events.  Solvers are pooled per grid shape: a new request on a
shape whose solver is free refreshes the moduli in place (the captured graph stays valid) instead
of rebuilding.  Kernels are deterministic, so a result does not depend on what else ran with it.

The scheduling core (`Scheduler`) is independent of CUDA; `CudaBackend` runs jobs on the device.
There is no counterpart in the reference (it has no serving loop).
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    shape: tuple
    density: object            # author-layout element densities (numpy or CUDA tensor)
    tol: float
    arrival: float             # seconds after the stream starts


@dataclass
class Completion:
    rid: int
    shape: tuple
    tol: float
    arrival: float
    admitted: float
    finished: float
    iterations: int
    converged: bool
    rel: float
    compliance: float
    x: object = None

    @property
    def latency(self):
        return self.finished - self.arrival


def footprint_estimate(shape, precision="mixed", levels=None, max_coarse_x=16) -> int:
    """Device bytes of one resident job: FP64 outer vectors, moduli, hierarchy, coarsest inverse."""
    from .solver import hierarchy_shapes
    shapes = hierarchy_shapes(shape, max_coarse_x)
    if levels is not None:
        shapes = shapes[:levels]
    ex, ea = {"fp64": (8, 8), "bf16": (4, 2), "bf16-all": (2, 2)}.get(precision, (4, 4))   # iterate, auxiliary
    total = 0
    for i, (nx, ny, nz) in enumerate(shapes):
        nodes, elems = (nx + 1) * (ny + 1) * (nz + 1), nx * ny * nz
        if i == 0:
            total += 6 * 24 * nodes + 2 * 8 * elems        # b x r p q z_old; E and its owned copy
        res = 0 if ex == ea else 3 * ea * nodes            # separate residual buffer
        total += 3 * nodes * (2 * ex + 2 * ea) + res + elems * (8 + ea) + nodes
    nx, ny, nz = shapes[-1]
    nc = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    return int(total + 5 * 8 * nc * nc + (64 << 20))   # A, factor, inverse, identity, L^-1; workspace


def percentile(values, q):
    return float(np.percentile(np.asarray(values, dtype=np.float64), q)) if len(values) else float("nan")


def summarize(completions, makespan):
    lat = [c.latency for c in completions]
    return {"requests": len(completions), "makespan_s": makespan,
            "solves_per_s": len(completions) / makespan if makespan > 0 else float("nan"),
            "p50_ms": 1e3 * percentile(lat, 50), "p99_ms": 1e3 * percentile(lat, 99),
            "mean_ms": 1e3 * float(np.mean(lat)) if lat else float("nan"),
            "all_converged": all(c.converged for c in completions)}


class Scheduler:
    """FIFO admission by slots and memory budget; completion by polling.  `backend` provides
    footprint(req) (bytes a start would add), start(req) -> handle, done(handle) -> bool,
    finish(handle, req) -> dict, release(handle) -> bytes freed (None: the job's footprint) and
    reclaim(bytes_needed) -> bytes freed from idle pooled state; optionally resident_bytes(), the
    bytes already held when a run starts (a pre-built pool)."""

    def __init__(self, backend, budget_bytes=150e9, max_slots=16, clock=time.perf_counter, poll_s=50e-6):
        self.backend, self.budget, self.max_slots = backend, float(budget_bytes), int(max_slots)
        self.clock, self.poll_s = clock, poll_s
        self.peak_inflight = 0
        self.peak_bytes = 0.0

    def run(self, requests):
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        active = []            # (req, handle, bytes, admitted)
        done = []
        used = float(self.backend.resident_bytes()) if hasattr(self.backend, "resident_bytes") else 0.0
        t0 = self.clock()
        while pending or active:
            now = self.clock() - t0
            progressed = False
            while pending and pending[0].arrival <= now and len(active) < self.max_slots:
                req = pending[0]
                need = float(self.backend.footprint(req))
                if need > self.budget:
                    raise ValueError(f"request {req.rid} needs {need / 1e9:.1f} GB, over the whole budget")
                if used + need > self.budget:
                    used -= self.backend.reclaim(used + need - self.budget)
                    if used + need > self.budget:
                        break                                   # wait for a running job to finish
                pending.popleft()
                handle = self.backend.start(req)
                used += need
                active.append((req, handle, need, self.clock() - t0))
                self.peak_inflight = max(self.peak_inflight, len(active))
                self.peak_bytes = max(self.peak_bytes, used)
                progressed = True
            still = []
            for req, handle, need, adm in active:
                if self.backend.done(handle):
                    info = self.backend.finish(handle, req)
                    fin = self.clock() - t0
                    freed = self.backend.release(handle)
                    used -= need if freed is None else freed
                    done.append(Completion(req.rid, tuple(req.shape), req.tol, req.arrival, adm, fin, **info))
                    progressed = True
                else:
                    still.append((req, handle, need, adm))
            active = still
            if not progressed:
                if not active and pending:
                    wait = pending[0].arrival - (self.clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.01))
                else:
                    time.sleep(self.poll_s)
        return done, self.clock() - t0


class CudaBackend:
    """Runs each request on a pooled ElasticitySolver with its own stream."""

    def __init__(self, precision="mixed", pre=2, post=2, omega=0.6, max_coarse_x=16, keep_solution=False,
                 maxiter=200, check_every=1):
        import torch
        self.torch = torch
        self.precision, self.pre, self.post, self.omega = precision, pre, post, omega
        self.max_coarse_x, self.keep, self.maxiter, self.check_every = max_coarse_x, keep_solution, maxiter, check_every
        self.free = {}              # shape -> [solver, ...] idle, resident
        self.free_bytes = {}        # id(solver) -> footprint
        self.forces = {}

    def footprint(self, req):
        return footprint_estimate(req.shape, self.precision, max_coarse_x=self.max_coarse_x)

    def _force(self, shape):
        from .problems import cantilever_equal_split
        if shape not in self.forces:
            self.forces[shape] = cantilever_equal_split(shape)
        return self.forces[shape]

    def start(self, req):
        from .api import ElasticitySolver
        from .problems import simp_modulus
        torch = self.torch
        shape = tuple(req.shape)
        mask, force = self._force(shape)
        rho = req.density if isinstance(req.density, torch.Tensor) else torch.as_tensor(req.density)
        rho = rho.to("cuda", torch.float64, non_blocking=True)
        pool = self.free.get(shape, [])
        if pool:
            s = pool.pop()
            self.free_bytes.pop(id(s), None)
            s.fcg.stream.wait_stream(torch.cuda.current_stream())    # rho was produced there
            with torch.cuda.stream(s.fcg.stream):
                s.update_modulus(simp_modulus(rho, 1e-9))
        else:
            s = ElasticitySolver(shape, simp_modulus(rho, 1e-9), mask, precision=self.precision, pre=self.pre,
                                 post=self.post, omega=self.omega, max_coarse_x=self.max_coarse_x, tol=req.tol,
                                 maxiter=self.maxiter, check_every=self.check_every)
        s.fcg.tol = float(req.tol)
        s.fcg.launch(force, dot_with=force)                    # the compliance comes back with the scalars
        return s

    def done(self, s):
        return s.fcg.done()

    def finish(self, s, req):
        res = s.fcg.finish()
        x = res.x.clone() if self.keep else None       # finish() ordered the caller's stream after the solve
        return {"iterations": res.iterations, "converged": res.converged, "rel": res.rel,
                "compliance": s.fcg.last_dot, "x": x}

    def prewarm(self, shapes, per_shape, budget_bytes=None):
        """Build `per_shape` idle solvers for each grid shape (hierarchy, buffers and the captured
        loop graph), so that serving never allocates device memory (cudaMalloc synchronises the
        device and would stall every job in flight).  Stops early at `budget_bytes` of footprint."""
        from .api import ElasticitySolver
        torch = self.torch
        used = self.resident_bytes()
        for shape in shapes:
            shape = tuple(shape)
            mask, force = self._force(shape)
            fp = footprint_estimate(shape, self.precision, max_coarse_x=self.max_coarse_x)
            for _ in range(per_shape - len(self.free.get(shape, []))):
                if budget_bytes is not None and used + fp > budget_bytes:
                    break
                E = torch.ones(shape[0] * shape[1] * shape[2], dtype=torch.float64, device="cuda")
                s = ElasticitySolver(shape, E, mask, precision=self.precision, pre=self.pre, post=self.post,
                                     omega=self.omega, max_coarse_x=self.max_coarse_x, tol=1e-6,
                                     maxiter=self.maxiter, check_every=self.check_every)
                s.fcg.launch(force)                            # captures the loop graph
                s.fcg.finish()
                self.release(s)
                used += fp
        torch.cuda.synchronize()

    def release(self, s):
        """The solver goes back to the pool and stays resident: nothing is freed."""
        self.free.setdefault(s.shape, []).append(s)
        self.free_bytes[id(s)] = footprint_estimate(s.shape, self.precision, max_coarse_x=self.max_coarse_x)
        return 0.0

    def reclaim(self, need):
        """Drop idle pooled solvers (largest first) until `need` bytes are freed; returns bytes freed."""
        freed = 0.0
        order = sorted(((self.free_bytes.get(id(s), 0), shape, s) for shape, lst in self.free.items() for s in lst),
                       key=lambda t: -t[0])
        for b, shape, s in order:
            if freed >= need:
                break
            self.free[shape].remove(s)
            self.free_bytes.pop(id(s), None)
            freed += b
        if freed:
            self.torch.cuda.empty_cache()
        return freed

    def resident_bytes(self):
        return sum(self.free_bytes.values())


def serve(requests, precision="mixed", budget_bytes=150e9, max_slots=16, keep_solution=False, prewarm=False, **kw):
    """Run a request stream through the continuous-batching server; returns (completions, summary).
    Pooled idle solvers are charged to the budget (they stay resident for reuse).  With `prewarm`,
    max_slots idle solvers per requested grid shape are built first (within the budget), so the
    stream itself never allocates device memory."""
    backend = CudaBackend(precision=precision, keep_solution=keep_solution, **kw)
    if prewarm:
        shapes = sorted({tuple(r.shape) for r in requests})
        backend.prewarm(shapes, max_slots, budget_bytes)
    sched = Scheduler(_PoolCharge(backend), budget_bytes=budget_bytes, max_slots=max_slots)
    done, makespan = sched.run(requests)
    out = summarize(done, makespan)
    out.update(peak_inflight=sched.peak_inflight, peak_budget_gb=sched.peak_bytes / 1e9)
    return sorted(done, key=lambda c: c.rid), out


class _PoolCharge:
    """Adapter: idle pooled solvers are charged to the budget until reclaimed, so the budget bounds
    everything resident (running and pooled)."""

    def __init__(self, backend):
        self.b = backend

    def footprint(self, req):
        pool = self.b.free.get(tuple(req.shape), [])
        return 0.0 if pool else self.b.footprint(req)      # a pooled solver is already charged

    def start(self, req):
        return self.b.start(req)

    def done(self, h):
        return self.b.done(h)

    def finish(self, h, req):
        return self.b.finish(h, req)

    def release(self, h):
        return self.b.release(h)

    def resident_bytes(self):
        return self.b.resident_bytes()

    def reclaim(self, need):
        return self.b.reclaim(need)


def request_stream(n=256, shapes=((48, 24, 24), (96, 48, 48), (160, 80, 80), (256, 128, 128)), tols=(1e-6, 1e-8),
                   rate=None, mean_service=None, load=1.2, seed=0, densities_per_shape=4, ell=8.0, device="cuda"):
    """The mixed-size request stream: Poisson arrivals (seeded), shapes uniform from `shapes`,
    seeded GRF densities (l = ell, a few per shape, reused), tolerances uniform from `tols`.  The
    arrival rate is `rate`, or load / mean_service."""
    from .problems import gaussian_random_field
    rng = np.random.default_rng(seed)
    dens = {s: [gaussian_random_field(s, ell, 1000 + 17 * k + i, device=device) for i in range(densities_per_shape)]
            for k, s in enumerate(shapes)}
    if rate is None:
        rate = load / float(mean_service)
    t = 0.0
    reqs = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        s = shapes[rng.integers(len(shapes))]
        reqs.append(Request(i, s, dens[s][rng.integers(densities_per_shape)], float(tols[rng.integers(len(tols))]), t))
    return reqs


def reserve_device_memory(nbytes):
    """Grow the caching allocator by `nbytes` (one block allocated and freed), so that solvers and
    batches built while a stream is being served take their memory from the cache: a cudaMalloc
    there would synchronise the device and stall every job in flight."""
    import torch
    if nbytes and nbytes > 0:
        t = torch.empty(int(nbytes), dtype=torch.uint8, device="cuda")
        del t


# ------------------------------------------------------------------------------ batched serving
def default_slots(shape, max_slots=16, dofs_per_batch=32e6):
    """Slots of a shape's batch: as many jobs as fit about `dofs_per_batch` stacked DOFs, at most max_slots."""
    nx, ny, nz = shape
    per = 3.0 * (nx + 1) * (ny + 1) * (nz + 1)
    return int(max(1, min(max_slots, dofs_per_batch // per)))


def batch_ladder(max_slots):
    """Capacities of a shape's batches: 1, 2, 4, ... up to max_slots (the last one max_slots)."""
    caps, c = [], 1
    while c < max_slots:
        caps.append(c)
        c *= 2
    caps.append(int(max_slots))
    return caps


def serve_batched(requests, shapes=None, slots=None, precision="mixed", chunk=4, maxiter=200, budget_bytes=150e9,
                  prewarm=None, keep_solution=False, clock=time.perf_counter, poll_s=50e-6, reserve_bytes=0):
    """Continuous batching with fused launches.  Each grid shape has a ladder of batch.BatchedSolvers
    of capacities 1, 2, 4, ... up to slots[shape] (batch_ladder), each with its own stream and
    captured chunk graph; every kernel of a chunk serves all the jobs of its batch at once.  A batch
    costs what its capacity costs, whatever its occupancy, so arrivals go where they waste least:
    between chunks, requests that have arrived fill the free slots of batches already running their
    shape's jobs (continuous batching), and the rest start the smallest idle empty batch that holds
    them all (else the largest idle one).  Finished jobs leave their slot at once; every batch of
    every shape runs concurrently.  A shape's batches are built when first needed unless the shape
    is listed in `prewarm` (default: every shape), so a cold shape pays its set-up inside the stream
    (`reserve_bytes` of cached memory make that set-up allocation-free).  The batches' footprint must
    fit the budget.  Returns (completions sorted by request id, summary)."""
    import torch
    from .batch import BatchedSolver
    from .problems import cantilever_equal_split, simp_modulus
    shapes = sorted({tuple(r.shape) for r in requests} if shapes is None else {tuple(s) for s in shapes})
    slots = {s: (slots or {}).get(s, default_slots(s)) for s in shapes}
    prewarm = set(shapes) if prewarm is None else {tuple(s) for s in prewarm}
    forces = {s: cantilever_equal_split(s)[1] for s in shapes}
    ladders = {s: batch_ladder(slots[s]) for s in shapes}
    batches = {s: [None] * len(ladders[s]) for s in shapes}     # built lazily
    used = 0.0

    def build(s, i):
        nonlocal used
        bs = BatchedSolver(s, ladders[s][i], precision=precision, chunk=chunk, maxiter=maxiter)
        used += bs.footprint_bytes()
        if used > budget_bytes:
            raise ValueError(f"batches need {used / 1e9:.1f} GB, over the {budget_bytes / 1e9:.0f} GB budget")
        # one throw-away job captures the chunk graph before any request is timed on it
        E1 = torch.ones(s[0] * s[1] * s[2], dtype=torch.float64, device="cuda")
        bs.solve([(E1, forces[s], 1e-2)])
        bs.retire(0)
        bs.active, bs.inflight = {}, False          # slot -> (request, admitted time)
        batches[s][i] = bs
        return bs

    for s in shapes:
        if s in prewarm:
            for i in range(len(ladders[s])):
                build(s, i)
    reserve_device_memory(reserve_bytes)            # for the cold shapes' batches
    torch.cuda.synchronize()
    pending = {s: deque() for s in shapes}
    arrivals = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
    done = []
    peak = 0
    cold = [s for s in shapes if s not in prewarm]
    t0 = clock()

    def live():
        return [b for s in shapes for b in batches[s] if b is not None]

    def admit(bs, s, rs):
        free = [k for k in range(bs.B) if k not in bs.active]
        jobs = []
        for k, r in zip(free, rs):
            rho = r.density if isinstance(r.density, torch.Tensor) else torch.as_tensor(r.density)
            E = simp_modulus(rho.to("cuda", torch.float64), 1e-9)
            jobs.append((k, E, forces[s], r.tol))
            bs.active[k] = (r, clock() - t0)
        bs.admit(jobs)

    while arrivals or any(pending.values()) or any(b.active for b in live()):
        now = clock() - t0
        progressed = False
        while arrivals and arrivals[0].arrival <= now:
            r = arrivals.popleft()
            pending[tuple(r.shape)].append(r)
        # admission between chunks
        for s in shapes:
            q = pending[s]
            if not q:
                continue
            for bs in batches[s]:                   # running batches with free slots first
                if q and bs is not None and bs.active and not bs.inflight and len(bs.active) < bs.B:
                    take = [q.popleft() for _ in range(min(len(q), bs.B - len(bs.active)))]
                    admit(bs, s, take)
                    progressed = True
            while q:
                idle = [i for i, b in enumerate(batches[s]) if b is None or (not b.active and not b.inflight)]
                if not idle:
                    break
                fit = [i for i in idle if ladders[s][i] >= len(q)]
                i = fit[0] if fit else idle[-1]
                bs = batches[s][i] or build(s, i)
                take = [q.popleft() for _ in range(min(len(q), bs.B))]
                admit(bs, s, take)
                progressed = True
        peak = max(peak, sum(len(b.active) for b in live()))
        # launch a chunk on every batch with jobs and nothing in flight
        for bs in live():
            if bs.active and not bs.inflight:
                bs.run()
                bs.inflight = True
                progressed = True
        # completion
        for s in shapes:
            for bs in batches[s]:
                if bs is None or not bs.inflight or not bs.ready():
                    continue
                bs.inflight = False
                fin, *_ = bs.poll()
                ks = [k for k in list(bs.active) if fin[k]]
                for k, (x, it, ok, rel, comp) in zip(ks, bs.results(ks)):
                    r, adm = bs.active.pop(k)
                    bs.retire(k)
                    done.append(Completion(r.rid, s, r.tol, r.arrival, adm, clock() - t0, it, ok, rel, comp,
                                           x if keep_solution else None))
                progressed = True
        if not progressed:
            if not any(b.active for b in live()) and not any(pending.values()) and arrivals:
                wait = arrivals[0].arrival - (clock() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.01))
            else:
                time.sleep(poll_s)
    makespan = clock() - t0
    out = summarize(done, makespan)
    out.update(peak_inflight=peak, slots={"x".join(map(str, s)): ladders[s] for s in shapes},
               batches_gb=used / 1e9, cold_shapes=["x".join(map(str, s)) for s in cold])
    return sorted(done, key=lambda c: c.rid), out
