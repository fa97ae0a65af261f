"""CPU tests of the serving scheduler (no GPU): admission by slots and HBM budget, FIFO order,
overlap of jobs that arrive while others run, latency bookkeeping -- against a fake backend whose
jobs take a fixed simulated time."""
import pytest

vx = pytest.importorskip("voxel_b200")
from voxel_b200.serving import Request, Scheduler, footprint_estimate, summarize  # noqa: E402


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class FakeBackend:
    """Each job runs `duration[shape]` simulated seconds after it starts; memory = `size[shape]`."""

    def __init__(self, clock, duration, size):
        self.clock, self.duration, self.size = clock, duration, size
        self.running, self.log = {}, []

    def footprint(self, req):
        return self.size[req.shape]

    def start(self, req):
        self.running[req.rid] = self.clock() + self.duration[req.shape]
        self.log.append(("start", req.rid, self.clock()))
        return req.rid

    def done(self, h):
        self.clock.t += 1e-4                 # every poll advances simulated time
        return self.clock() >= self.running[h]

    def finish(self, h, req):
        return {"iterations": 10, "converged": True, "rel": 1e-9, "compliance": 1.0}

    def release(self, h):
        self.running.pop(h)

    def reclaim(self, need):
        return 0.0


def _run(reqs, budget, slots, duration, size):
    clock = FakeClock()
    be = FakeBackend(clock, duration, size)
    sched = Scheduler(be, budget_bytes=budget, max_slots=slots, clock=clock, poll_s=0.0)
    import voxel_b200.serving as srv
    real_sleep = srv.time.sleep
    srv.time.sleep = lambda s: setattr(clock, "t", clock.t + max(s, 1e-4))
    try:
        done, makespan = sched.run(reqs)
    finally:
        srv.time.sleep = real_sleep
    return done, makespan, be, sched


def test_jobs_overlap_up_to_the_slot_limit():
    reqs = [Request(i, (4, 2, 2), None, 1e-8, 0.0) for i in range(6)]
    done, makespan, be, sched = _run(reqs, budget=1e12, slots=3, duration={(4, 2, 2): 1.0}, size={(4, 2, 2): 1.0})
    assert len(done) == 6 and sched.peak_inflight == 3
    assert 1.9 < makespan < 2.2                     # two waves of three overlapping jobs
    first_wave = {c.rid for c in done if c.admitted == min(d.admitted for d in done)}
    assert first_wave == {0, 1, 2}                  # FIFO admission


def test_admission_respects_the_memory_budget():
    big, small = (8, 4, 4), (4, 2, 2)
    reqs = [Request(0, big, None, 1e-8, 0.0), Request(1, big, None, 1e-8, 0.0), Request(2, small, None, 1e-8, 0.0)]
    done, makespan, be, sched = _run(reqs, budget=10.0, slots=8, duration={big: 1.0, small: 0.1},
                                     size={big: 6.0, small: 1.0})
    assert sched.peak_bytes <= 10.0
    byid = {c.rid: c for c in done}
    assert byid[1].admitted >= byid[0].finished - 1e-3        # the second big job waited for memory
    assert byid[2].admitted >= byid[1].admitted               # FIFO: the small job is not overtaken


def test_arrivals_during_running_jobs_are_admitted_immediately():
    reqs = [Request(0, (4, 2, 2), None, 1e-8, 0.0), Request(1, (4, 2, 2), None, 1e-8, 0.5)]
    done, makespan, be, sched = _run(reqs, budget=1e12, slots=4, duration={(4, 2, 2): 1.0}, size={(4, 2, 2): 1.0})
    byid = {c.rid: c for c in done}
    assert abs(byid[1].admitted - 0.5) < 0.01 and byid[1].admitted < byid[0].finished
    s = summarize(done, makespan)
    assert s["requests"] == 2 and s["p50_ms"] > 0 and s["p99_ms"] >= s["p50_ms"]


def test_request_over_the_whole_budget_is_rejected():
    reqs = [Request(0, (4, 2, 2), None, 1e-8, 0.0)]
    with pytest.raises(ValueError):
        _run(reqs, budget=0.5, slots=1, duration={(4, 2, 2): 1.0}, size={(4, 2, 2): 1.0})


def test_footprint_grows_with_the_grid():
    a = footprint_estimate((48, 24, 24))
    b = footprint_estimate((256, 128, 128))
    assert 0 < a < b and b < 4e9


class PoolingBackend(FakeBackend):
    """Finished jobs stay resident in a pool (release frees nothing); a new job on a pooled shape
    needs no memory; reclaim frees idle pooled jobs."""

    def __init__(self, clock, duration, size, pooled=()):
        super().__init__(clock, duration, size)
        self.pool = list(pooled)
        self.reclaimed = 0.0

    def resident_bytes(self):
        return sum(self.size[s] for s in self.pool)

    def footprint(self, req):
        return 0.0 if req.shape in self.pool else self.size[req.shape]

    def start(self, req):
        if req.shape in self.pool:
            self.pool.remove(req.shape)
        self.running[req.rid] = (self.clock() + self.duration[req.shape], req.shape)
        return req.rid

    def done(self, h):
        self.clock.t += 1e-4
        return self.clock() >= self.running[h][0]

    def release(self, h):
        self.pool.append(self.running.pop(h)[1])
        return 0.0

    def reclaim(self, need):
        freed = 0.0
        while self.pool and freed < need:
            freed += self.size[self.pool.pop(0)]
        self.reclaimed += freed
        return freed


def test_pooled_solvers_stay_charged_until_reclaimed():
    big, small = (8, 4, 4), (4, 2, 2)
    clock = FakeClock()
    be = PoolingBackend(clock, {big: 1.0, small: 0.5}, {big: 6.0, small: 1.0}, pooled=[small, small])
    sched = Scheduler(be, budget_bytes=10.0, max_slots=8, clock=clock, poll_s=0.0)
    reqs = [Request(0, small, None, 1e-8, 0.0), Request(1, big, None, 1e-8, 0.0), Request(2, big, None, 1e-8, 0.0)]
    import voxel_b200.serving as srv
    real_sleep = srv.time.sleep
    srv.time.sleep = lambda s: setattr(clock, "t", clock.t + max(s, 1e-4))
    try:
        done, makespan = sched.run(reqs)
    finally:
        srv.time.sleep = real_sleep
    assert len(done) == 3
    assert sched.peak_bytes <= 10.0                 # pool (2) + one big (6); the second big must wait
    byid = {c.rid: c for c in done}
    assert byid[2].admitted >= byid[1].finished - 1e-3
    assert be.reclaimed > 0                         # idle pooled memory was given back for the second big job
