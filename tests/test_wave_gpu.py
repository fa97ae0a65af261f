"""The persistent wavefront operator kernel (FP64 and FP32 iterates): grids whose work items
outnumber the CTAs, so every CTA streams several (x chunk, y tile, z tile) items back to back; ragged
tiles in y and z; every fused form against the oracle; bitwise determinism across launches."""
import numpy as np
import pytest
import torch

from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu

vx = pytest.importorskip("voxel_b200")
from voxel_b200 import _lib  # noqa: E402


@pytest.fixture(autouse=True)
def wave_kernel():
    prev = _lib.set_stream_kernel("wave")
    yield
    _lib.set_stream_kernel(prev)


KE = vo.quadrature([1, 1, 1], 0.3)
# (150, 40, 70): 3 x 3 tiles of (y, z) over 151 node planes -> more items than SMs
GRIDS = [(150, 40, 70), (64, 31, 29), (9, 61, 2)]


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


@pytest.mark.parametrize("shape", GRIDS)
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-5)])
def test_every_form_matches_the_oracle(shape, dtype, tol):
    E, u, r, mask = problem(shape, sum(shape))
    rd = (lambda a: a.astype(np.float32).astype(np.float64)) if dtype == torch.float32 else (lambda a: a)
    Eh, uh, rh = rd(E), rd(u), rd(r)
    op = vx.VoxelOperator(shape, KE, dtype)
    nm = vx.node_mask_from_dofs(cu(mask))
    Et, ut, rt = cu(Eh, dtype), cu(uh, dtype), cu(rh, dtype)
    Au = vo.apply_dirichlet(shape, KE, Eh, mask, uh)
    assert maxrel(op.matvec(ut, Et).double().cpu().numpy(), vo.product_raw(shape, KE, uh, Eh)) < tol
    assert maxrel(op.matvec(ut, Et, nm).double().cpu().numpy(), Au) < tol
    invd = op.diagonal(Et, nm, inverse=True)
    dn = invd.double().cpu().numpy()
    assert maxrel(op.jacobi(ut, rt, invd, Et, nm, 0.6).double().cpu().numpy(), uh + 0.6 * dn * (rh - Au)) < tol
    assert maxrel(op.residual(ut, rt, Et, nm).double().cpu().numpy(), (rh - Au) * mask) < tol
    G = op.partials_size
    assert 1 <= G <= torch.cuda.get_device_properties(0).multi_processor_count
    part = torch.empty(G, dtype=torch.float64, device="cuda")
    q = torch.empty_like(ut)
    op.apply_dot(ut, Et, nm, q, part)
    assert maxrel(q.double().cpu().numpy(), Au) < tol
    assert abs(float(part.sum()) - float(uh @ Au)) <= 10 * tol * float(np.abs(uh * Au).sum())
    res = torch.empty_like(ut)
    op.true_residual(ut, rt, Et, nm, res, part)
    ref = rh - Au
    assert maxrel(res.double().cpu().numpy(), ref) < tol
    assert abs(float(part.sum()) - float(ref @ ref)) <= 10 * tol * float(ref @ ref)
    assert vx._lib.device_status() == 0


def test_bf16_auxiliary_storage_forms():
    """FP32 iterates with bf16 modulus, right-hand side and inverse diagonal (the narrow values are
    staged as the 32-bit words that hold them)."""
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
def test_repeated_launches_are_bitwise_equal(dtype):
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


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_bulk_and_cp_async_staging_agree_bitwise(dtype):
    """16-byte aligned arrays are staged by bulk (TMA-engine) row copies, others element by element
    with cp.async; both feed the same arithmetic, so the results are bitwise equal."""
    shape = (150, 40, 70)
    E, u, r, mask = problem(shape, 6)
    op = vx.VoxelOperator(shape, KE, dtype)
    nm = vx.node_mask_from_dofs(cu(mask))
    Et, ut, rt = cu(E, dtype), cu(u, dtype), cu(r, dtype)

    def shifted(t):                      # same values at an address 1 element past a 16-byte boundary
        buf = torch.empty(t.numel() + 1, dtype=t.dtype, device="cuda")
        buf[1:].copy_(t)
        v = buf[1:]
        assert v.data_ptr() % 16 != 0
        return v
    nms = torch.empty(nm.numel() + 1, dtype=torch.uint8, device="cuda")
    nms[1:].copy_(nm)
    invd = op.diagonal(Et, nm, inverse=True)
    outs = []
    for (E_, u_, r_, m_) in ((Et, ut, rt, nm), (shifted(Et), shifted(ut), shifted(rt), nms[1:])):
        y = op.matvec(u_, E_, m_)
        j = op.jacobi(u_, r_, invd, E_, m_, 0.6)
        part = torch.empty(op.partials_size, dtype=torch.float64, device="cuda")
        res = torch.empty_like(ut)
        op.true_residual(u_, r_, E_, m_, res, part)
        outs.append((y, j, res, part.clone()))
    for a_, b_ in zip(outs[0], outs[1]):
        assert torch.equal(a_, b_)
