"""The serving loop on the device: a mixed-size request stream run concurrently (jobs overlapping on
separate streams, pooled solvers reused) gives each request the result it gets alone.
Tolerance: equal iteration counts and displacement relative difference <= 1e-10.  Every kernel of
the solve is deterministic; the batched loop sums its dot products in another grouping than the
single-job solver, so the two agree to rounding, not bitwise."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import serving  # noqa: E402


def _requests():
    shapes = [(16, 8, 8), (32, 16, 16), (48, 24, 24)]
    reqs = serving.request_stream(n=12, shapes=shapes, tols=(1e-6, 1e-8), rate=1e6, seed=3, densities_per_shape=2)
    for r in reqs:
        r.arrival = 0.0                      # everything arrives at once: maximal overlap
    return reqs


def test_results_in_the_mix_equal_results_alone():
    reqs = _requests()
    done, summary = serving.serve(reqs, precision="mixed", max_slots=6, keep_solution=True)
    assert summary["requests"] == 12 and summary["all_converged"]
    assert summary["peak_inflight"] > 1
    for c in done:
        r = reqs[c.rid]
        mask, force = vx.problems.cantilever_equal_split(r.shape)
        s = vx.ElasticitySolver(r.shape, vx.problems.simp_modulus(r.density, 1e-9), mask, precision="mixed",
                                tol=r.tol, maxiter=200, check_every=1)
        alone = s.solve(force)
        assert alone.iterations == c.iterations
        diff = float(torch.linalg.vector_norm(alone.x - c.x) / torch.linalg.vector_norm(alone.x))
        print(f"request {c.rid} {r.shape}: bitwise {torch.equal(alone.x, c.x)}, rel diff {diff:.2e}")
        assert diff <= 1e-10, (c.rid, diff)


def test_budget_limits_concurrency():
    reqs = _requests()
    big = max(serving.footprint_estimate(s) for s in {r.shape for r in reqs})
    done, summary = serving.serve(reqs, precision="mixed", max_slots=6, budget_bytes=2.2 * big)
    assert summary["requests"] == 12 and summary["all_converged"]
    assert summary["peak_budget_gb"] * 1e9 <= 2.2 * big


def test_batched_serving_results_equal_results_alone():
    """serve_batched: the jobs of a shape share every launch of their batch (stacked grid); each result
    equals the job solved alone, and jobs of several shapes and more jobs than slots go through."""
    reqs = _requests()
    slots = {(16, 8, 8): 2, (32, 16, 16): 3, (48, 24, 24): 2}
    done, summary = serving.serve_batched(reqs, slots=slots, keep_solution=True, chunk=2)
    assert summary["requests"] == 12 and summary["all_converged"]
    assert summary["peak_inflight"] > 3
    for c in done:
        r = reqs[c.rid]
        mask, force = vx.problems.cantilever_equal_split(r.shape)
        s = vx.ElasticitySolver(r.shape, vx.problems.simp_modulus(r.density, 1e-9), mask, precision="mixed",
                                tol=r.tol, maxiter=200, check_every=1)
        alone = s.solve(force)
        assert alone.iterations == c.iterations, (c.rid, alone.iterations, c.iterations)
        diff = float(torch.linalg.vector_norm(alone.x - c.x) / torch.linalg.vector_norm(alone.x))
        assert diff <= 1e-10, (c.rid, diff)
