"""Transfers on grids that span several CTAs in every direction with ragged edges (odd node counts,
partial CTAs in y and z): FP64 restriction and prolongation are bit-for-bit the oracle's (the
kernels evaluate the same per-axis passes in the same order, right neighbour before left); FP32 and
bf16 within their storage rounding; coarse and fine node masks applied; restriction is the
transpose of prolongation."""
import numpy as np
import pytest
import torch

from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import _lib  # noqa: E402

# fine element grids (even): coarse nz + 1 in {2, 3, 19, 33, 41, 66}, coarse ny + 1 from 2 to 66
SHAPES = [(140, 40, 80), (2, 2, 2), (4, 66, 4), (36, 18, 64), (8, 130, 130), (576 // 8, 288 // 8, 288 // 8)]
PREC = {torch.float64: _lib.VX_F64, torch.float32: _lib.VX_F32, torch.bfloat16: _lib.VX_BF16_F32}


def _s():
    return torch.cuda.current_stream().cuda_stream


def _masks(shape, rng):
    n = vo.n_nodes(shape)
    m = rng.integers(0, 8, size=n).astype(np.uint8)
    m[rng.random(n) < 0.5] = 7
    return m


def _dof(mask):
    return np.stack([(mask >> c) & 1 for c in range(3)], axis=1).ravel().astype(np.float64)


@pytest.mark.parametrize("shape", SHAPES)
def test_fp64_transfers_equal_the_oracle_bit_for_bit(shape):
    rng = np.random.default_rng(sum(shape))
    coarse = tuple(s // 2 for s in shape)
    nf, nc = 3 * vo.n_nodes(shape), 3 * vo.n_nodes(coarse)
    rf = rng.standard_normal(nf)
    uc = rng.standard_normal(nc)
    x0 = rng.standard_normal(nf)
    rf_d, uc_d = torch.as_tensor(rf, device="cuda"), torch.as_tensor(uc, device="cuda")
    for masked in (False, True):
        cm = _masks(coarse, rng) if masked else None
        fm = _masks(shape, rng) if masked else None
        cm_d = torch.as_tensor(cm, device="cuda") if masked else None   # kept alive until the kernels ran
        fm_d = torch.as_tensor(fm, device="cuda") if masked else None
        out = torch.empty(nc, dtype=torch.float64, device="cuda")
        _lib.call("vx_restrict", _lib.VX_F64, *shape, rf_d.data_ptr(), cm_d.data_ptr() if masked else None,
                  out.data_ptr(), _s())
        ref = vo.restrict(rf, shape) * (_dof(cm) if masked else 1.0)
        assert np.array_equal(out.cpu().numpy(), ref)
        x = torch.as_tensor(x0, device="cuda").clone()
        _lib.call("vx_prolong_add", _lib.VX_F64, *shape, uc_d.data_ptr(), fm_d.data_ptr() if masked else None,
                  x.data_ptr(), _s())
        p = vo.prolong(uc, coarse)
        ref = np.where(_dof(fm) > 0, x0 + p, x0) if masked else x0 + p
        assert np.array_equal(x.cpu().numpy(), ref)


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
@pytest.mark.parametrize("shape", [SHAPES[0], SHAPES[4]])
def test_reduced_precision_transfers(shape, dtype):
    rng = np.random.default_rng(7 + sum(shape))
    coarse = tuple(s // 2 for s in shape)
    nf, nc = 3 * vo.n_nodes(shape), 3 * vo.n_nodes(coarse)
    rf = torch.as_tensor(rng.standard_normal(nf), device="cuda").to(dtype)
    uc = torch.as_tensor(rng.standard_normal(nc), device="cuda").to(dtype)
    x = torch.as_tensor(rng.standard_normal(nf), device="cuda").to(dtype)
    x0 = x.double().cpu().numpy()
    tol = 1e-6 if dtype == torch.float32 else 1e-2
    out = torch.empty(nc, dtype=dtype, device="cuda")
    _lib.call("vx_restrict", PREC[dtype], *shape, rf.data_ptr(), None, out.data_ptr(), _s())
    ref = vo.restrict(rf.double().cpu().numpy(), shape)
    assert np.abs(out.double().cpu().numpy() - ref).max() <= tol * np.abs(ref).max()
    _lib.call("vx_prolong_add", PREC[dtype], *shape, uc.data_ptr(), None, x.data_ptr(), _s())
    ref = x0 + vo.prolong(uc.double().cpu().numpy(), coarse)
    assert np.abs(x.double().cpu().numpy() - ref).max() <= tol * np.abs(ref).max()


def test_restriction_is_the_transpose_of_prolongation():
    """<R r, u> = <r, P u> on a grid of several CTAs in every direction (FP64, relative 1e-13)."""
    shape = SHAPES[0]
    coarse = tuple(s // 2 for s in shape)
    rng = np.random.default_rng(3)
    r = torch.as_tensor(rng.standard_normal(3 * vo.n_nodes(shape)), device="cuda")
    u = torch.as_tensor(rng.standard_normal(3 * vo.n_nodes(coarse)), device="cuda")
    Rr = torch.empty_like(u)
    _lib.call("vx_restrict", _lib.VX_F64, *shape, r.data_ptr(), None, Rr.data_ptr(), _s())
    Pu = torch.zeros_like(r)
    _lib.call("vx_prolong_add", _lib.VX_F64, *shape, u.data_ptr(), None, Pu.data_ptr(), _s())
    a, b = float(Rr @ u), float(r @ Pu)
    assert abs(a - b) <= 1e-13 * max(abs(a), abs(b))
