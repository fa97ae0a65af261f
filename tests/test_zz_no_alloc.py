"""The allocation-free residual entry point (vx_true_residual_noalloc) against the existing
vx_true_residual + vx_reduce_partials pair, called through the C ABI.

It exists for callers that cannot allocate device memory (a request loop that must not call
cudaMalloc while work is in flight, a plugin confined to another framework's memory arena): its
reduction scratch is a fixed array inside the library.  The file is named to be collected last."""
import numpy as np
import pytest
import torch

from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import _lib  # noqa: E402

KE = vo.quadrature([1, 1, 1], 0.3)


def _case(shape, seed):
    rng = np.random.default_rng(seed)
    E = torch.as_tensor(1e-9 + (1 - 1e-9) * rng.random(int(np.prod(shape))) ** 3, device="cuda")
    x = torch.as_tensor(rng.standard_normal(3 * vo.n_nodes(shape)), device="cuda")
    b = torch.as_tensor(rng.standard_normal(3 * vo.n_nodes(shape)), device="cuda")
    mask, _ = vo.cantilever_equal_split(shape)
    nm = vx.node_mask_from_dofs(torch.as_tensor(mask, device="cuda"))
    return E, x, b, nm


def _noalloc(op, E, nm, x, b):
    res = torch.empty_like(x)
    n2 = torch.empty(1, dtype=torch.float64, device="cuda")
    _lib.call("vx_true_residual_noalloc", _lib.VX_F64, *op.shape, op._bp, E.data_ptr(), nm.data_ptr(),
              x.data_ptr(), b.data_ptr(), res.data_ptr(), n2.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return res, n2


def _existing(op, E, nm, x, b):
    G = op.partials_size
    partials = torch.empty(G, dtype=torch.float64, device="cuda")
    res = torch.empty_like(x)
    op.true_residual(x, b, E, nm, res, partials)
    return res, vx.reduce_partials(partials, G)


@pytest.mark.parametrize("shape", [(33, 29, 61), (7, 5, 3)])
def test_noalloc_matches_existing_entry_point_on_two_calls(shape):
    op = vx.VoxelOperator(shape, KE)
    for seed in (1, 2):                          # two calls in a row reuse the built-in scratch
        E, x, b, nm = _case(shape, seed)
        res_a, n_a = _noalloc(op, E, nm, x, b)
        res_b, n_b = _existing(op, E, nm, x, b)
        torch.cuda.synchronize()
        assert torch.equal(res_a, res_b)                       # same kernel, same arithmetic
        assert abs(float(n_a) - float(n_b)) <= 1e-13 * abs(float(n_b))
        assert abs(float(n_a) - float((res_b * res_b).sum())) <= 1e-12 * float(n_b)


def test_noalloc_rejects_grids_beyond_its_scratch():
    shape = (2047, 400, 400)                     # needs far more than 16384 CTA partial sums
    assert _lib.load().vx_operator_partials(_lib.VX_F64, *shape) > 16384
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    blocks = np.ascontiguousarray(vx.Modal(KE).blocks.reshape(72))
    st = _lib.load().vx_true_residual_noalloc(_lib.VX_F64, *shape, _lib.dptr(blocks), dummy.data_ptr(), None,
                                              dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                              dummy.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == _lib.VX_ERR_INVALID_ARGUMENT
    assert "16384" in _lib.last_error()
