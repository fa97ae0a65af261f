"""The donor drop-ins (voxel_b200.donor) against the donor code's own golden runs
(tests/golden/jacobi_32x16x16.npz: experiments/session_a/donor/src/gpu_fem/simp_r2.py pcg and
pcg_ir on the 32x16x16 cantilever, NumPy standing in for CuPy): both routes -- any callable
`matvec` (the donor's loop) and a DirichletOperator (the device-scalar graph solvers) -- reproduce
the donor's iteration counts and solution; the projection pair, the fail-closed rule and the
continuation driver."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import donor  # noqa: E402


def cu(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def rel(a, b):
    a = a.detach().double().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case():
    g = golden("jacobi_32x16x16.npz")
    shape = tuple(int(s) for s in g["shape"])
    ke = vo.quadrature([1, 1, 1], 0.3)
    inv = 1 / np.where(g["mask"] != 0, vo.product_diagonal(shape, ke, g["E"]), 1.0)
    return g, shape, inv


@pytest.mark.parametrize("route", ["callable", "operator"])
def test_pcg_reproduces_the_donor_run(case, route):
    g, shape, inv = case
    A = donor.DirichletOperator(shape, cu(g["E"]), cu(g["mask"]))
    mv = A if route == "operator" else (lambda u: A(u))
    x, it, ok, r = donor.pcg(mv, cu(g["force"]), cu(inv), tol=1e-8, maxiter=5000, mask=cu(g["mask"]), check_every=50)
    assert ok and it == int(g["pcg_it"])
    assert rel(x, g["pcg_x"]) < 1e-8
    # the residual at the stopping test is a few ulps of |b| (1e-8 relative): its last digits follow
    # the rounding of the product, so it agrees with the donor's to a few per cent, and both pass
    assert r <= 1e-8 and abs(r - float(g["pcg_rel"])) <= 0.1 * float(g["pcg_rel"])


def test_pcg_residual_history_and_zero_rhs(case):
    g, shape, inv = case
    A = donor.DirichletOperator(shape, cu(g["E"]), cu(g["mask"]))
    hist = []
    x, it, ok, r = donor.pcg(A, cu(g["force"]), cu(inv), tol=1e-8, maxiter=5000, mask=cu(g["mask"]),
                             check_every=50, residual_history=hist)
    assert ok and it == int(g["pcg_it"]) and len(hist) == 1 + -(-it // 50)      # the start and every check
    assert hist[-1] == pytest.approx(r)
    x0, it0, ok0, r0 = donor.pcg(A, torch.zeros_like(cu(g["force"])), cu(inv))
    assert ok0 and it0 == 0 and r0 == 0.0


@pytest.mark.parametrize("route", ["callable", "operator"])
def test_pcg_ir_reproduces_the_donor_run(case, route):
    g, shape, inv = case
    A64 = donor.DirichletOperator(shape, cu(g["E"]), cu(g["mask"]))
    A32 = donor.DirichletOperator(shape, cu(g["E"]), cu(g["mask"]), dtype=torch.float32)
    m64, m32 = (A64, A32) if route == "operator" else ((lambda u: A64(u)), (lambda u: A32(u)))
    x, outer, inner, ok, r = donor.pcg_ir(m64, cu(g["force"]), m32, cu(inv, torch.float32), tol=1e-8,
                                          mask32=cu(g["mask"], torch.float32), inner_tol=1e-1, max_outer=40,
                                          inner_maxiter=4000, check_every=50)
    assert ok and r <= 1e-8 and outer == int(g["ir_outer"])
    # FP32 arithmetic in the inner products (the donor rounded FP64 products): a few inner iterations apart
    assert abs(inner - int(g["ir_inner"])) <= 0.05 * int(g["ir_inner"])
    comp = float(cu(g["force"]) @ x)
    assert abs(comp - float(g["fcg_compliance"])) <= 1e-8 * abs(float(g["fcg_compliance"]))


def test_projection_and_its_derivative():
    x = torch.linspace(0, 1, 101, dtype=torch.float64, device="cuda")
    for beta in (0.0, 1.0, 16.0):
        p = donor.project(x, beta).cpu().numpy()
        if beta == 0:
            assert np.array_equal(p, x.cpu().numpy())
        t, d = np.tanh(beta * 0.5), np.tanh(beta * 0.5) + np.tanh(beta * 0.5)
        ref = (t + np.tanh(beta * (x.cpu().numpy() - 0.5))) / d if beta else x.cpu().numpy()
        assert np.allclose(p, ref, rtol=1e-14, atol=1e-15)
        h = 1e-6
        fd = ((donor.project(x + h, beta) - donor.project(x - h, beta)) / (2 * h)).cpu().numpy()
        assert np.allclose(donor.dproject(x, beta).cpu().numpy(), fd, rtol=1e-6, atol=1e-7)


def test_compliance_fails_closed_after_a_retry_from_zero():
    shape = (16, 8, 8)
    mask, force = vx.problems.cantilever_equal_split(shape)
    rho = torch.full((int(np.prod(shape)),), 0.5, dtype=torch.float64, device="cuda")
    s = vx.ElasticitySolver(shape, vx.problems.simp_modulus(rho, 1e-9), mask, precision="mixed", tol=1e-14,
                            maxiter=2, check_every=1)
    st = vx.simp.SimpState(s, force)
    st.u = torch.zeros(s.op64.ndof, dtype=torch.float64, device="cuda")     # a warm start that cannot meet 1e-14
    with pytest.raises(donor.LinearSolveNotConverged, match="retried from zero"):
        vx.compliance(rho.clone().requires_grad_(True), st)
    assert st.retried


def test_donor_run_simp_continuation_and_fail_closed():
    shape = (24, 12, 6)
    mask, force, _ = vx.problems.donor_cantilever(*shape, Lx=2.0, Ly=1.0, Lz=0.5, load="patch")
    res = donor.run_simp(shape, mask, force, volfrac=0.3, fixed_budget=18, solver="gmg", cg_tol=1e-6, levels=2)
    h = res["history"]
    assert res["stop_reason"] == "fixed_budget" and res["outer_iters"] == 18 and len(h) == 18
    assert [x["penal"] for x in h[14:16]] == [1.5, 3.5] and [x["beta"] for x in h[14:16]] == [1.0, 4.0]
    assert all(abs(x["vol_phys"] - 0.3) <= 1e-6 for x in h)                 # OC on the projected volume
    assert h[-1]["compliance"] < h[0]["compliance"]
    assert res["max_rel_resid"] <= 1e-6 and res["total_cg_iters"] > 0
    assert res["solve_log"][-1]["final_iterate"]
    with pytest.raises(donor.LinearSolveNotConverged):
        donor.run_simp(shape, mask, force, volfrac=0.3, fixed_budget=2, solver="pcg", cg_tol=1e-12, cg_maxiter=3)
