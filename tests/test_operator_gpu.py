"""GPU parity of the operator kernels (libvoxel_b200 through its C ABI) against the CPU oracle and
the reference's golden vectors.  Tolerances: FP64 max-norm relative 1e-13,
FP32 1e-5, BF16-storage (FP32 arithmetic on bf16-rounded inputs) 1e-5 against the oracle run on
the same rounded inputs."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu

vx = pytest.importorskip("voxel_b200")

SHAPES = [(1, 1, 1), (3, 2, 4), (5, 3, 7), (6, 4, 2), (2, 17, 3), (33, 29, 61), (40, 15, 31), (7, 31, 30)]
KE = vo.quadrature([1, 1, 1], 0.3)


def maxrel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def case(shape, seed=0, emin=1e-9):
    rng = np.random.default_rng(seed)
    E = emin + (1 - emin) * rng.random(int(np.prod(shape))) ** 3
    u = rng.standard_normal(3 * vo.n_nodes(shape))
    return E, u


def cu(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.mark.parametrize("shape", SHAPES)
def test_matvec_fp64_matches_oracle(shape):
    E, u = case(shape, 1)
    op = vx.VoxelOperator(shape, KE)
    y = op.matvec(cu(u), cu(E)).cpu().numpy()
    assert maxrel(y, vo.product_raw(shape, KE, u, E)) < 1e-13


@pytest.mark.parametrize("shape", [(3, 2, 4), (33, 29, 61), (12, 20, 45)])
def test_matvec_dirichlet_fp64(shape):
    E, u = case(shape, 2)
    mask, _ = vo.cantilever_equal_split(shape)
    rng = np.random.default_rng(3)
    mask = mask * (rng.random(mask.size) > 0.1)              # ragged extra constraints
    op = vx.VoxelOperator(shape, KE)
    nm = vx.node_mask_from_dofs(cu(mask))
    y = op.matvec(cu(u), cu(E), node_mask=nm).cpu().numpy()
    assert maxrel(y, vo.apply_dirichlet(shape, KE, E, mask, u)) < 1e-13


def test_brick_element_and_fixture_ke():
    shape = (9, 14, 33)
    E, u = case(shape, 4)
    for ke in (vo.quadrature([1.0, 0.5, 2.0], 0.25), golden("element.npz")["ke_fixture"]):
        y = vx.VoxelOperator(shape, ke).matvec(cu(u), cu(E)).cpu().numpy()
        assert maxrel(y, vo.product_raw(shape, ke, u, E)) < 1e-13


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-5)])
def test_brick_element_fused_forms(dtype, tol):
    """A brick element has no cube symmetry: the kernels take the general 45-coefficient product
    (a cube takes the 33-operation form); both must match the oracle in every fused form."""
    shape = (17, 10, 21)
    ke = vo.quadrature([1.0, 0.5, 2.0], 0.25)
    E, u = case(shape, 8)
    r = np.random.default_rng(9).standard_normal(u.size)
    mask, _ = vo.cantilever_equal_split(shape)
    nm = vx.node_mask_from_dofs(cu(mask))
    op = vx.VoxelOperator(shape, ke, dtype)
    rd = lambda a: a.astype(np.float32).astype(np.float64) if dtype == torch.float32 else a
    Eh, uh, rh = rd(E), rd(u), rd(r)
    Au = vo.apply_dirichlet(shape, ke, Eh, mask, uh)
    invd = rd(1 / np.where(mask != 0, vo.product_diagonal(shape, ke, Eh), 1.0))
    x = op.jacobi(cu(uh, dtype), cu(rh, dtype), cu(invd, dtype), cu(Eh, dtype), nm, 0.6)
    assert maxrel(x.double().cpu().numpy(), uh + 0.6 * invd * (rh - Au)) < tol
    res = op.residual(cu(uh, dtype), cu(rh, dtype), cu(Eh, dtype), nm)
    assert maxrel(res.double().cpu().numpy(), (rh - Au) * mask) < tol
    q = torch.empty(u.size, dtype=dtype, device="cuda")
    part = torch.empty(op.partials_size, dtype=torch.float64, device="cuda")
    op.apply_dot(cu(uh, dtype), cu(Eh, dtype), nm, q, part)
    assert maxrel(q.double().cpu().numpy(), Au) < tol
    assert abs(float(part.sum()) - float(uh @ Au)) <= tol * abs(float(uh @ Au)) * 10


def test_modal8_entry_point_matches_reference_emulation():
    g = golden("element.npz")
    shape = tuple(int(s) for s in g["emu_shape"])
    y = torch.zeros(3 * vo.n_nodes(shape), dtype=torch.float64, device="cuda")
    blocks = np.ascontiguousarray(g["blocks_unit"].reshape(72))
    E, u = cu(g["emu_E"]), cu(g["emu_u"])
    vx._lib.call("vx_modal8", vx._lib.dptr(blocks), E.data_ptr(), u.data_ptr(), y.data_ptr(), *shape,
                 torch.cuda.current_stream().cuda_stream)
    assert maxrel(y.cpu().numpy(), g["emu_assembled"]) < 1e-13
    assert maxrel(y.cpu().numpy(), g["emu_modal8_fp64"]) < 1e-13


@pytest.mark.parametrize("shape", [(5, 3, 7), (33, 29, 61)])
def test_matvec_fp32(shape):
    E, u = case(shape, 5)
    y = vx.VoxelOperator(shape, KE, torch.float32).matvec(cu(u, torch.float32), cu(E, torch.float32))
    ref = vo.product_raw(shape, KE, u.astype(np.float32).astype(np.float64), E.astype(np.float32).astype(np.float64))
    assert y.dtype == torch.float32
    assert maxrel(y.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("shape", [(5, 3, 7), (33, 29, 61)])
def test_matvec_bf16_storage(shape):
    E, u = case(shape, 6)
    ub, Eb = cu(u, torch.bfloat16), cu(E, torch.bfloat16)
    y = vx.VoxelOperator(shape, KE, torch.bfloat16).matvec(ub, Eb)
    assert y.dtype == torch.float32
    ref = vo.product_raw(shape, KE, ub.double().cpu().numpy(), Eb.double().cpu().numpy())
    assert maxrel(y.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("shape", [(3, 2, 4), (20, 9, 13)])
def test_dense_control_path(shape):
    E, u = case(shape, 7)
    y = vx.VoxelOperator(shape, KE).matvec_dense(cu(u), cu(E)).cpu().numpy()
    assert maxrel(y, vo.product_raw(shape, KE, u, E)) < 1e-13


def test_matvec_is_bitwise_deterministic():
    shape = (33, 29, 61)
    E, u = case(shape, 8)
    op = vx.VoxelOperator(shape, KE)
    a = op.matvec(cu(u), cu(E))
    b = op.matvec(cu(u), cu(E))
    assert torch.equal(a, b)


@pytest.mark.parametrize("shape", [(5, 3, 7), (33, 29, 61)])
def test_diagonal_and_inverse(shape):
    E, _ = case(shape, 9)
    mask, _ = vo.cantilever_equal_split(shape)
    op = vx.VoxelOperator(shape, KE)
    d = op.diagonal(cu(E)).cpu().numpy()
    ref = vo.product_diagonal(shape, KE, E)
    assert maxrel(d, ref) < 1e-14
    inv = op.diagonal(cu(E), vx.node_mask_from_dofs(cu(mask)), inverse=True).cpu().numpy()
    assert maxrel(inv, 1 / np.where(mask != 0, ref, 1.0)) < 1e-14


def test_element_energy_and_sensitivity():
    shape = (11, 6, 9)
    rho = np.random.default_rng(10).uniform(0.01, 1, int(np.prod(shape)))
    _, u = case(shape, 10)
    op = vx.VoxelOperator(shape, KE)
    ce, dc = op.energy(cu(u), rho=cu(rho), emin=1e-9, emax=1.0, penal=3.0)
    ref = vo.element_energy(shape, KE, u)
    assert maxrel(ce.cpu().numpy(), ref) < 1e-13
    assert maxrel(dc.cpu().numpy(), -3 * rho ** 2 * (1 - 1e-9) * ref) < 1e-13


def test_c_product_on_device_matches_reference_golden():
    g = golden("products.npz")
    shape = tuple(int(s) for s in g["smoke_shape"])
    for rho, ke, emin, key in ((g["smoke_rho"], g["smoke_ke"], 1e-6, "smoke"), (g["het_rho"], KE, 1e-9, "het")):
        y, ce, d = vx.product(shape, cu(rho), cu(g["smoke_u"]), ke, cu(g["smoke_mask"]), emin)
        assert maxrel(y.cpu().numpy(), g[f"{key}_c_y"]) < 1e-13
        assert maxrel(ce.cpu().numpy(), g[f"{key}_c_ce"]) < 1e-13
        assert maxrel(d.cpu().numpy(), g[f"{key}_c_diag"]) < 1e-14


def test_c_product_natural_layout_large_odd_grid():
    shape = (23, 17, 35)
    rng = np.random.default_rng(11)
    rho = rng.uniform(0.01, 1, int(np.prod(shape)))
    u = rng.standard_normal(3 * vo.n_nodes(shape))
    mask, _ = vo.cantilever_line_load(shape)
    y, ce, d = vx.product(shape, cu(rho), cu(u), KE, cu(mask), 1e-9)
    ry, rce, rd = vo.c_reference_product(shape, rho, u, KE, mask, 1e-9)
    assert maxrel(y.cpu().numpy(), ry) < 1e-13
    assert maxrel(ce.cpu().numpy(), rce) < 1e-13
    assert maxrel(d.cpu().numpy(), rd) < 1e-14


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-5)])
def test_fused_jacobi_and_residual(dtype, tol):
    shape = (17, 30, 29)
    E, x = case(shape, 12)
    r = np.random.default_rng(13).standard_normal(x.size)
    mask, _ = vo.cantilever_equal_split(shape)
    op = vx.VoxelOperator(shape, KE, dtype)
    nm = vx.node_mask_from_dofs(cu(mask))
    Et, xt, rt = cu(E, dtype), cu(x, dtype), cu(r, dtype)
    invd = op.diagonal(Et, nm, inverse=True)
    xd, rd, Ed, invd_np = (t.double().cpu().numpy() for t in (xt, rt, Et, invd))
    Ax = vo.apply_dirichlet(shape, KE, Ed, mask, xd)
    out = op.jacobi(xt, rt, invd, Et, nm, 0.6).double().cpu().numpy()
    assert maxrel(out, xd + 0.6 * invd_np * (rd - Ax)) < tol
    res = op.residual(xt, rt, Et, nm).double().cpu().numpy()
    assert maxrel(res, (rd - Ax) * mask) < tol


def test_apply_dot_and_true_residual():
    shape = (33, 29, 61)
    E, p = case(shape, 14)
    b = np.random.default_rng(15).standard_normal(p.size)
    mask, _ = vo.cantilever_equal_split(shape)
    op = vx.VoxelOperator(shape, KE)
    nm = vx.node_mask_from_dofs(cu(mask))
    G = op.partials_size
    partials = torch.empty(G, dtype=torch.float64, device="cuda")
    q = torch.empty_like(cu(p))
    op.apply_dot(cu(p), cu(E), nm, q, partials)
    pq = float(vx.reduce_partials(partials, G)[0])
    Ap = vo.apply_dirichlet(shape, KE, E, mask, p)
    assert maxrel(q.cpu().numpy(), Ap) < 1e-13
    assert abs(pq - p @ Ap) <= 1e-12 * abs(p @ Ap)
    res = torch.empty_like(q)
    op.true_residual(cu(p), cu(b), cu(E), nm, res, partials)
    rr = float(vx.reduce_partials(partials, G)[0])
    assert maxrel(res.cpu().numpy(), b - Ap) < 1e-13
    assert abs(rr - np.sum((b - Ap) ** 2)) <= 1e-12 * np.sum((b - Ap) ** 2)


def test_dots_deterministic_and_accurate():
    rng = np.random.default_rng(16)
    for n in (1, 1000, 3 * 577 * 289 + 5):
        a, b, c = (rng.standard_normal(n) for _ in range(3))
        o1 = vx.dots([(cu(a), cu(b)), (cu(a), cu(c))]).cpu().numpy()
        o2 = vx.dots([(cu(a), cu(b)), (cu(a), cu(c))]).cpu().numpy()
        assert np.array_equal(o1, o2)
        assert abs(o1[0] - a @ b) <= 1e-12 * np.sum(np.abs(a * b))
        assert abs(o1[1] - a @ c) <= 1e-12 * np.sum(np.abs(a * c))


def test_invalid_arguments_raise():
    op = vx.VoxelOperator((4, 4, 4), KE)
    E = torch.ones(64, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        op.matvec(torch.ones(10, dtype=torch.float64, device="cuda"), E)
    with pytest.raises(ValueError):
        op.matvec(torch.ones(375, dtype=torch.float32, device="cuda"), E)
    with pytest.raises(ValueError):
        vx.VoxelOperator((0, 4, 4), KE)


def test_stream_pointer_follows_the_current_stream():
    """operators.stream_ptr (read once per launch by the host-driven loops) is the raw handle of
    torch's current stream, on the default stream and inside a stream context."""
    from voxel_b200.operators import stream_ptr
    assert stream_ptr() == torch.cuda.current_stream().cuda_stream
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        assert stream_ptr() == s.cuda_stream == torch.cuda.current_stream().cuda_stream
    assert stream_ptr() == torch.cuda.current_stream().cuda_stream
    assert stream_ptr(torch.cuda.current_device()) == torch.cuda.current_stream().cuda_stream
