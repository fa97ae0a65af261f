"""The BF16-storage preconditioner variants (no reference counterpart), FP32 arithmetic, inside
the FP64 flexible-CG outer loop:
  "bf16"      moduli and auxiliary vectors (right-hand sides, residuals, inverse diagonals) in
              bf16, iterates in FP32 (selector VX_F32_BF16AUX);
  "bf16-all"  iterates in bf16 too (selector VX_BF16_F32).

Kernel parity is checked against the FP64 oracle evaluated on the same bf16-rounded inputs.  A
bf16 output is the FP32 result rounded once to bf16, so it lies within 2^-8 of the oracle relative
to its own magnitude plus FP32 rounding of the terms (tolerance 4.5e-3 in max-norm relative); an
FP32 output is within FP32 rounding (1e-5).  Solves must reach the same FP64 relative residual
(1e-8) as the FP64 and FP32 variants and agree with the reference's records and published known
answers to the bars stated per test."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import _lib  # noqa: E402
from voxel_b200 import solver as vs  # noqa: E402
from voxel_b200.api import ElasticitySolver  # noqa: E402

KE = vo.quadrature([1, 1, 1], 0.3)
BF16_TOL = 4.5e-3


def bf(a):
    """(bf16 device tensor, its exact FP64 values on the host)"""
    t = torch.as_tensor(np.ascontiguousarray(a)).to("cuda").to(torch.bfloat16)
    return t, t.double().cpu().numpy()


def maxrel(a, b):
    a = a.double().cpu().numpy() if isinstance(a, torch.Tensor) else a
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("shape", [(24, 12, 12), (33, 29, 61), (48, 24, 24)])
@pytest.mark.parametrize("iterate", [torch.bfloat16, torch.float32])
def test_bf16_smoother_and_residual_match_oracle(shape, iterate):
    rng = np.random.default_rng(sum(shape))
    n = 3 * vo.n_nodes(shape)
    E, Eh = bf(1e-3 + rng.random(int(np.prod(shape))))
    x, xh = bf(rng.standard_normal(n))
    x = x.to(iterate)
    r, rh = bf(rng.standard_normal(n))
    mask, _ = vo.cantilever_equal_split(shape)
    nm = vx.node_mask_from_dofs(torch.as_tensor(mask, device="cuda"))
    invd, dh = bf(1 / np.where(mask != 0, vo.product_diagonal(shape, KE, Eh), 1.0))
    op = vx.VoxelOperator(shape, KE, iterate, torch.bfloat16)
    Ax = vo.apply_dirichlet(shape, KE, Eh, mask, xh)
    out = op.jacobi(x, r, invd, E, nm, 0.6)
    assert out.dtype == iterate
    tol = BF16_TOL if iterate == torch.bfloat16 else 1e-5
    assert maxrel(out, xh + 0.6 * dh * (rh - Ax)) < tol
    res = op.residual(x, r, E, nm)
    assert res.dtype == torch.bfloat16
    assert maxrel(res, (rh - Ax) * mask) < BF16_TOL
    y = op.matvec(x, E, nm)
    assert y.dtype == torch.float32 and maxrel(y, Ax) < 1e-5


@pytest.mark.parametrize("shape", [(48, 24, 24), (16, 8, 8)])
def test_bf16_transfers_and_coarse_solve(shape):
    rng = np.random.default_rng(7)
    coarse = tuple(s // 2 for s in shape)
    nf, nc = 3 * vo.n_nodes(shape), 3 * vo.n_nodes(coarse)
    f, fh = bf(rng.standard_normal(nf))
    out = torch.empty(nc, dtype=torch.bfloat16, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    _lib.call("vx_restrict", _lib.VX_BF16_F32, *shape, f.data_ptr(), None, out.data_ptr(), s)
    assert maxrel(out, vo.restrict(fh, shape)) < BF16_TOL
    c, ch = bf(rng.standard_normal(nc))
    x, xh = bf(rng.standard_normal(nf))
    _lib.call("vx_prolong_add", _lib.VX_BF16_F32, *shape, c.data_ptr(), None, x.data_ptr(), s)
    assert maxrel(x, xh + vo.prolong(ch, coarse)) < BF16_TOL
    # dense coarse solve: FP64 inverse, bf16 in and out
    m = 3 * vo.n_nodes((2, 2, 2))
    A = rng.standard_normal((m, m))
    Ainv = torch.as_tensor(A @ A.T + m * np.eye(m), device="cuda")
    rv, rvh = bf(rng.standard_normal(m))
    z = torch.empty(m, dtype=torch.bfloat16, device="cuda")
    _lib.call("vx_coarse_apply", _lib.VX_BF16_F32, m, Ainv.data_ptr(), rv.data_ptr(), None, z.data_ptr(), s)
    assert maxrel(z, Ainv.cpu().numpy() @ rvh) < BF16_TOL


def test_bf16_vcycle_is_a_close_preconditioner():
    """M(r) of each storage mode against the FP64 V-cycle on the 128x64x64 hierarchy."""
    shape = (128, 64, 64)
    rho = vx.problems.gaussian_random_field(shape, 8.0, 0)
    E = vx.problems.simp_modulus(rho, 1e-9)
    mask, force = vx.problems.cantilever_equal_split(shape)
    nm = vx.node_mask_from_dofs(mask)
    out = {}
    for key, (dt, aux) in {"fp64": (torch.float64, None), "fp32": (torch.float32, None),
                           "bf16": (torch.float32, torch.bfloat16), "bf16-all": (torch.bfloat16, None)}.items():
        M = vs.MGHierarchy(shape, KE, E, nm, dt, pre=2, post=2, omegas=0.6, aux_dtype=aux)
        out[key] = M(force)
    ref = out["fp64"]
    d = {k: float(torch.linalg.vector_norm(v - ref) / torch.linalg.vector_norm(ref)) for k, v in out.items()}
    print("V-cycle relative difference to FP64: " + ", ".join(f"{k} {v:.2e}" for k, v in d.items()))
    assert d["fp32"] < 1e-5 and d["bf16"] < 3e-2 and d["bf16-all"] < 3e-2


@pytest.mark.parametrize("precision,extra", [("bf16", 1), ("bf16-all", 12)])
def test_bf16_gmg_128x64x64_solve_reaches_the_fp64_residual(precision, extra):
    """The FP64 outer loop reaches 1e-8 with either storage mode; "bf16" needs at most one more
    iteration than FP32 (emulated and measured: the same 15), "bf16-all" pays for rounding its
    iterates (about 21-25)."""
    c = golden("gmg_128x64x64.json")
    shape = (128, 64, 64)
    rho = vx.problems.gaussian_random_field(shape, 8.0, 0)
    E = vx.problems.simp_modulus(rho, 1e-9)
    mask, force = vx.problems.cantilever_equal_split(shape)
    s = ElasticitySolver(shape, E, mask, precision=precision, pre=2, post=2, omega=0.6, check_every=1)
    x, it, ok, r, mv = s.solve(force)
    print(f"{precision} 128x64x64: {it} iterations (fp32/fp64: 15), rel {r:.3e}")
    assert ok and r <= 1e-8 and it <= c["fp32"]["iterations"] + extra
    # the solution satisfies the FP64 residual bound: compliance agrees to the solve tolerance
    assert abs(float(force @ x) - c["fp64"]["compliance"]) <= 1e-7 * c["fp64"]["compliance"]
    assert torch.all(x[mask == 0] == 0)


def test_bf16_published_kat_q64x2():
    """256 x 128 x 128 (6.4M DOF), reference V(4,4) spectral: published compliance 807.19637074."""
    from test_solver_gpu import _kat
    x, it, ok, comp, obs = _kat("q64x2", "bf16")
    print(f"bf16 q64x2: {it} iterations (published {obs[0]['iterations']}), compliance {comp!r}")
    assert ok and it <= obs[0]["iterations"] + 1
    ref_c = np.array([o["compliance"] for o in obs])
    assert np.min(np.abs(comp - ref_c)) <= 1e-8 * ref_c.mean()
