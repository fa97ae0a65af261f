"""Out-of-bounds read detection: every input of a kernel sits inside a larger device buffer whose
surroundings are NaN, so a read outside its array poisons the output; every output sits inside a
guard band that must still be NaN afterwards (no write outside).  Results are also compared with
the oracle.  Shapes cover several CTA tilings in every direction, both precisions, every fused
epilogue, the transfers and the coarse-grid kernels."""
import numpy as np
import pytest
import torch

from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import _lib  # noqa: E402

PAD = 4096
SHAPES = [(96, 48, 48), (48, 24, 24), (24, 12, 12), (16, 8, 8), (33, 29, 61), (9, 31, 62)]
KE = vo.quadrature([1, 1, 1], 0.3)


def guarded(a, dtype):
    """(view, whole): a device copy of `a` inside NaN guard bands (ints: 0xAB guard bytes)."""
    a = np.ascontiguousarray(a)
    n = a.size
    if dtype == torch.uint8:
        whole = torch.full((n + 2 * PAD,), 0xAB, dtype=torch.uint8, device="cuda")
    else:
        whole = torch.full((n + 2 * PAD,), float("nan"), dtype=dtype, device="cuda")
    view = whole[PAD:PAD + n]
    view.copy_(torch.as_tensor(a).to(dtype))
    return view, whole


def out_buf(n, dtype):
    whole = torch.full((n + 2 * PAD,), float("nan"), dtype=dtype, device="cuda")
    return whole[PAD:PAD + n], whole


def bands_intact(whole, n):
    return bool(torch.isnan(whole[:PAD]).all() and torch.isnan(whole[PAD + n:]).all())


def case(shape, seed):
    rng = np.random.default_rng(seed)
    E = 1e-9 + (1 - 1e-9) * rng.random(int(np.prod(shape))) ** 3
    x = rng.standard_normal(3 * vo.n_nodes(shape))
    r = rng.standard_normal(3 * vo.n_nodes(shape))
    mask, _ = vo.cantilever_equal_split(shape)
    return E, x, r, mask


def maxrel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-5)])
def test_operator_epilogues_stay_in_bounds(shape, dtype, tol):
    E, x, r, mask = case(shape, sum(shape))
    op = vx.VoxelOperator(shape, KE, dtype)
    nm_np = np.zeros(vo.n_nodes(shape), dtype=np.uint8)
    m3 = mask.reshape(-1, 3)
    nm_np[:] = (m3[:, 0] != 0) | ((m3[:, 1] != 0) << 1) | ((m3[:, 2] != 0) << 2)
    Eg, _ = guarded(E, dtype)
    xg, _ = guarded(x, dtype)
    rg, _ = guarded(r, dtype)
    nm, _ = guarded(nm_np, torch.uint8)
    Ed, xd, rd = (t.double().cpu().numpy() for t in (Eg, xg, rg))
    Ax = vo.apply_dirichlet(shape, KE, Ed, mask, xd)
    n = op.ndof
    # raw and Dirichlet products
    y, yw = out_buf(n, dtype)
    op.matvec(xg, Eg, out=y)
    assert bands_intact(yw, n) and maxrel(y.double().cpu().numpy(), vo.product_raw(shape, KE, xd, Ed)) < tol
    op.matvec(xg, Eg, node_mask=nm, out=y)
    assert bands_intact(yw, n) and maxrel(y.double().cpu().numpy(), Ax) < tol
    # smoother and residual
    invd64 = 1 / np.where(mask != 0, vo.product_diagonal(shape, KE, Ed), 1.0)
    dg, _ = guarded(invd64, dtype)
    dd = dg.double().cpu().numpy()
    op.jacobi(xg, rg, dg, Eg, nm, 0.6, out=y)
    assert bands_intact(yw, n) and maxrel(y.double().cpu().numpy(), xd + 0.6 * dd * (rd - Ax)) < tol
    op.residual(xg, rg, Eg, nm, out=y)
    assert bands_intact(yw, n) and maxrel(y.double().cpu().numpy(), (rd - Ax) * mask) < tol
    # fused reductions
    G = op.partials_size
    pg, pw = out_buf(G, torch.float64)
    op.apply_dot(xg, Eg, nm, y, pg)
    assert bands_intact(yw, n) and bands_intact(pw, G) and not torch.isnan(pg).any()
    op.true_residual(xg, rg, Eg, nm, y, pg)
    assert bands_intact(yw, n) and bands_intact(pw, G) and not torch.isnan(pg).any()
    assert maxrel(y.double().cpu().numpy(), rd - Ax) < tol
    # diagonal
    dout, dw = out_buf(n, dtype)
    op.diagonal(Eg, nm, inverse=True, out=dout)
    assert bands_intact(dw, n) and maxrel(dout.double().cpu().numpy(), invd64) < tol


@pytest.mark.parametrize("shape", [s for s in SHAPES if all(v % 2 == 0 for v in s)])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_transfers_and_coarsening_stay_in_bounds(shape, dtype):
    E, x, r, mask = case(shape, 1 + sum(shape))
    coarse = tuple(s // 2 for s in shape)
    nf, nc = 3 * vo.n_nodes(shape), 3 * vo.n_nodes(coarse)
    fg, _ = guarded(x, dtype)
    cg_, _ = guarded(r[:nc], dtype)
    ref_r = vo.restrict(fg.double().cpu().numpy(), shape)
    out, ow = out_buf(nc, dtype)
    _lib.call("vx_restrict", vx.operators.PREC[dtype], *shape, fg.data_ptr(), None, out.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    assert bands_intact(ow, nc) and maxrel(out.double().cpu().numpy(), ref_r) < 1e-6
    xf, xw = out_buf(nf, dtype)
    xf.zero_()
    _lib.call("vx_prolong_add", vx.operators.PREC[dtype], *shape, cg_.data_ptr(), None, xf.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    assert bands_intact(xw, nf) and maxrel(xf.double().cpu().numpy(), vo.prolong(cg_.double().cpu().numpy(), coarse)) < 1e-6
    Eg, _ = guarded(E, torch.float64)
    Ec, Ew = out_buf(E.size // 8, torch.float64)
    _lib.call("vx_coarsen_modulus", _lib.VX_F64, *shape, Eg.data_ptr(), Ec.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert bands_intact(Ew, E.size // 8) and maxrel(Ec.cpu().numpy(), vo.coarsen_modulus(E, shape)) < 1e-15
