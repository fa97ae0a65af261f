"""The stacked batch solver (voxel_b200.batch): several jobs of one shape fused into shared launches
give each job the solution it gets alone -- against the single-job ElasticitySolver (same iterations,
displacement to 1e-10), bitwise against the same job alone in the batch, and for a job admitted
while another is half-way through its solve (continuous batching)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200.batch import BatchedSolver  # noqa: E402

SHAPE = (48, 24, 24)


def job(seed, tol):
    rho = vx.problems.gaussian_random_field(SHAPE, 8.0, seed)
    E = vx.problems.simp_modulus(rho, 1e-9)
    _, f = vx.problems.cantilever_equal_split(SHAPE)
    return E, f, tol


def rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_equals_single_solves(precision):
    jobs = [job(1, 1e-8), job(2, 1e-6), job(3, 1e-8)]
    bs = BatchedSolver(SHAPE, 3, precision=precision, chunk=4)
    out = bs.solve(jobs)
    mask, _ = vx.problems.cantilever_equal_split(SHAPE)
    for (E, f, tol), (x, it, ok, r, comp) in zip(jobs, out):
        es = vx.ElasticitySolver(SHAPE, E, mask, precision=precision, pre=2, post=2, omega=0.6, tol=tol, check_every=1)
        ref = es.solve(f)
        assert ok and ref.converged and it == ref.iterations
        assert rel(x, ref.x) <= 1e-10
        assert abs(comp - float(f @ ref.x)) <= 1e-10 * abs(comp)
    assert vx._lib.device_status() == 0


def test_mix_alone_and_midflight_admission_are_bitwise_equal():
    a, b, c = job(4, 1e-8), job(5, 1e-8), job(6, 1e-6)
    alone = BatchedSolver(SHAPE, 3, chunk=2).solve([b])[0]
    mixed = BatchedSolver(SHAPE, 3, chunk=2).solve([a, c, b])[2]
    assert torch.equal(alone[0], mixed[0]) and alone[1:4] == mixed[1:4]
    # continuous batching: b joins slot 1 while a is half-way through its solve in slot 0
    bs = BatchedSolver(SHAPE, 3, chunk=2)
    bs.admit([(0, *a)])
    bs.run()
    bs.run()
    fin, it, *_ = bs.poll()
    assert not fin[0] and it[0] > 0
    bs.admit([(1, *b)])
    done = {}
    while len(done) < 2:
        bs.run()
        fin, *_ = bs.poll()
        for k in (0, 1):
            if fin[k] and k not in done:
                done[k] = bs.result(k)
                bs.retire(k)
    assert torch.equal(done[1][0], alone[0]) and done[1][1] == alone[1]
    ref_a = BatchedSolver(SHAPE, 1, chunk=2).solve([a])[0]
    assert torch.equal(done[0][0], ref_a[0]) and done[0][1] == ref_a[1]
