"""The node-column-pair operator kernel (parity_zp, the default for FP64 / FP32 iterates): every
fused form against the oracle on ragged grids (tiles cut in y, z and x), and bitwise agreement with
the element-plane-pair kernel, which computes the same operations in the same order.
Tolerances: 1e-13 relative (FP64), 1e-5 (FP32) against the FP64 oracle; the kernels among
themselves: bitwise."""
import numpy as np
import pytest
import torch

from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu

vx = pytest.importorskip("voxel_b200")
from voxel_b200 import _lib  # noqa: E402

KE = vo.quadrature([1, 1, 1], 0.3)
# (150, 40, 70): 2 z tiles (71 columns), 4 y tiles; (64, 31, 29): one ragged z tile; (9, 61, 2): one
# node plane chunk per CTA at most; (5, 3, 125): 3 z tiles, nz + 1 a multiple of 2 but not of 62
GRIDS = [(150, 40, 70), (64, 31, 29), (9, 61, 2), (5, 3, 125)]


def maxrel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def cu(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def problem(shape, seed):
    rng = np.random.default_rng(seed)
    E = 1e-9 + (1 - 1e-9) * rng.random(int(np.prod(shape))) ** 3
    u = rng.standard_normal(3 * vo.n_nodes(shape))
    r = rng.standard_normal(u.size)
    mask, _ = vo.cantilever_equal_split(shape)
    mask = mask * (rng.random(mask.size) > 0.05)           # scattered extra constraints
    return E, u, r, mask


@pytest.fixture
def kernel():
    prev = _lib.set_stream_kernel("zp")
    yield
    _lib.set_stream_kernel(prev)


def forms(op, ut, Et, nm, rt, invd):
    """Every fused form of one operator: outputs and the partial-sum totals."""
    out = {"raw": op.matvec(ut, Et), "dirichlet": op.matvec(ut, Et, nm),
           "jacobi": op.jacobi(ut, rt, invd, Et, nm, 0.6), "residual": op.residual(ut, rt, Et, nm)}
    part = torch.zeros(op.partials_size, dtype=torch.float64, device="cuda")
    q = torch.empty_like(ut)
    op.apply_dot(ut, Et, nm, q, part)
    out["apply_dot"], out["pq"] = q, part.sum()
    res = torch.empty_like(ut)
    part = torch.zeros(op.partials_size, dtype=torch.float64, device="cuda")
    op.true_residual(ut, rt, Et, nm, res, part)
    out["true_residual"], out["rr"] = res, part.sum()
    return out


@pytest.mark.parametrize("shape", GRIDS)
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-5)])
def test_every_form_matches_the_oracle(kernel, shape, dtype, tol):
    E, u, r, mask = problem(shape, sum(shape))
    rd = (lambda a: a.astype(np.float32).astype(np.float64)) if dtype == torch.float32 else (lambda a: a)
    Eh, uh, rh = rd(E), rd(u), rd(r)
    op = vx.VoxelOperator(shape, KE, dtype)
    nm = vx.node_mask_from_dofs(cu(mask))
    Et, ut, rt = cu(Eh, dtype), cu(uh, dtype), cu(rh, dtype)
    invd = op.diagonal(Et, nm, inverse=True)
    dn = invd.double().cpu().numpy()
    Au = vo.apply_dirichlet(shape, KE, Eh, mask, uh)
    o = forms(op, ut, Et, nm, rt, invd)
    h = lambda t: t.double().cpu().numpy()
    assert maxrel(h(o["raw"]), vo.product_raw(shape, KE, uh, Eh)) < tol
    assert maxrel(h(o["dirichlet"]), Au) < tol
    assert maxrel(h(o["jacobi"]), uh + 0.6 * dn * (rh - Au)) < tol
    assert maxrel(h(o["residual"]), (rh - Au) * mask) < tol
    assert maxrel(h(o["apply_dot"]), Au) < tol
    assert abs(float(o["pq"]) - float(uh @ Au)) <= 10 * tol * float(np.abs(uh * Au).sum())
    ref = rh - Au
    assert maxrel(h(o["true_residual"]), ref) < tol
    assert abs(float(o["rr"]) - float(ref @ ref)) <= 10 * tol * float(ref @ ref)
    assert vx._lib.device_status() == 0


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_both_kernels_agree(dtype):
    """zp and xp: FP32 outputs agree to the bit (packed f32x2 intrinsics, never contracted);
    FP64 outputs to 1e-15 of the largest entry (the compiler fuses different multiply-add pairs of
    the block product and the inverse Z stage into FMAs in each kernel).  The partial sums are
    grouped per CTA, so their totals agree to rounding only."""
    shape = (150, 40, 70)
    E, u, r, mask = problem(shape, 7)
    op = vx.VoxelOperator(shape, KE, dtype)
    nm = vx.node_mask_from_dofs(cu(mask))
    Et, ut, rt = cu(E, dtype), cu(u, dtype), cu(r, dtype)
    invd = op.diagonal(Et, nm, inverse=True)
    outs = {}
    prev = _lib.set_stream_kernel("zp")
    try:
        for kind in ("zp", "xp"):
            _lib.set_stream_kernel(kind)
            outs[kind] = forms(op, ut, Et, nm, rt, invd)
    finally:
        _lib.set_stream_kernel(prev)
    for kind in ("xp",):
        for key in ("raw", "dirichlet", "jacobi", "residual", "apply_dot", "true_residual"):
            a_, b_ = outs["zp"][key], outs[kind][key]
            if dtype == torch.float32:
                assert torch.equal(a_, b_), (kind, key)
            else:
                assert float((a_ - b_).abs().max()) <= 1e-15 * float(b_.abs().max()), (kind, key)
        for key in ("pq", "rr"):
            a, b = float(outs["zp"][key]), float(outs[kind][key])
            assert abs(a - b) <= 1e-12 * abs(b), (kind, key)


def test_bf16_auxiliary_storage_forms(kernel):
    """FP32 iterates with bf16 modulus, right-hand side and inverse diagonal (moduli prefetched into
    registers, not staged)."""
    shape = (150, 40, 70)
    E, u, r, mask = problem(shape, 3)
    op = vx.VoxelOperator(shape, KE, torch.float32, torch.bfloat16)
    nm = vx.node_mask_from_dofs(cu(mask))
    Eb, rb = cu(E, torch.bfloat16), cu(r, torch.bfloat16)
    ut = cu(u, torch.float32)
    op32 = vx.VoxelOperator(shape, KE, torch.float32)
    invd = op32.diagonal(Eb.float(), nm, inverse=True).to(torch.bfloat16)
    En, rn, un, dn = (t.double().cpu().numpy() for t in (Eb, rb, ut, invd))
    Au = vo.apply_dirichlet(shape, KE, En, mask, un)
    x = op.jacobi(ut, rb, invd, Eb, nm, 0.6).double().cpu().numpy()
    assert maxrel(x, un + 0.6 * dn * (rn - Au)) < 1e-5
    res = op.residual(ut, rb, Eb, nm).double().cpu().numpy()
    assert maxrel(res, (rn - Au) * mask) < 5e-3                   # the residual is stored in bf16


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_repeated_launches_are_bitwise_equal(kernel, dtype):
    shape = (150, 40, 70)
    E, u, _, mask = problem(shape, 4)
    op = vx.VoxelOperator(shape, KE, dtype)
    nm = vx.node_mask_from_dofs(cu(mask))
    Et, ut = cu(E, dtype), cu(u, dtype)
    part = torch.empty(op.partials_size, dtype=torch.float64, device="cuda")
    outs = []
    for _ in range(3):
        q = torch.empty_like(ut)
        op.apply_dot(ut, Et, nm, q, part)
        outs.append((q, part.clone()))
    for q, p in outs[1:]:
        assert torch.equal(q, outs[0][0]) and torch.equal(p, outs[0][1])
