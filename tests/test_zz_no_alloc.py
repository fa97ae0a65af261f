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
    _lib.call("vx_true_residual_noalloc", op.prec, *op.shape, op._bp, E.data_ptr(), nm.data_ptr(),
              x.data_ptr(), b.data_ptr(), res.data_ptr(), n2.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return res, n2


def _existing(op, E, nm, x, b):
    G = op.partials_size
    partials = torch.empty(G, dtype=torch.float64, device="cuda")
    res = torch.empty_like(x)
    op.true_residual(x, b, E, nm, res, partials)
    return res, vx.reduce_partials(partials, G)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-6)])
@pytest.mark.parametrize("shape", [(33, 29, 61), (7, 5, 3), (150, 40, 70)])
def test_noalloc_matches_existing_entry_point_on_two_calls(shape, dtype, tol):
    op = vx.VoxelOperator(shape, KE, dtype)
    for seed in (1, 2):                          # two calls in a row reuse the built-in scratch
        E, x, b, nm = _case(shape, seed)
        E, x, b = E.to(dtype), x.to(dtype), b.to(dtype)
        res_a, n_a = _noalloc(op, E, nm, x, b)
        res_b, n_b = _existing(op, E, nm, x, b)
        torch.cuda.synchronize()
        assert torch.equal(res_a, res_b)                       # same kernel, same arithmetic
        assert abs(float(n_a) - float(n_b)) <= tol * abs(float(n_b))
        assert abs(float(n_a) - float((res_b.double() ** 2).sum())) <= 10 * tol * float(n_b)


def test_noalloc_scratch_covers_every_accepted_grid():
    """Every streaming kernel keeps one partial sum per CTA and chunks x only while the CTAs stay
    within the built-in 16384-double scratch, so it holds the partials of every grid whose y-z
    tiling fits (all but extremely flat ones); a grid beyond the library's 2^31-DOF limit is refused
    with a clear error before any device work."""
    prev = _lib.set_stream_kernel("xp")
    try:
        for kind in ("xp", "zp"):
            _lib.set_stream_kernel(kind)
            for prec in (_lib.VX_F64, _lib.VX_F32):
                for shape in ((2047, 400, 400), (1, 1, 1), (576, 288, 288), (1, 1500, 1500)):
                    G = _lib.load().vx_operator_partials(prec, *shape)
                    assert 1 <= G <= 16384, (kind, prec, shape, G)
    finally:
        _lib.set_stream_kernel(prev)
    shape = (4000, 600, 600)                     # 4.3e9 DOFs
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    blocks = np.ascontiguousarray(vx.Modal(KE).blocks.reshape(72))
    st = _lib.load().vx_true_residual_noalloc(_lib.VX_F64, *shape, _lib.dptr(blocks), dummy.data_ptr(), None,
                                              dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                              dummy.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == _lib.VX_ERR_INVALID_ARGUMENT
    assert "2^31" in _lib.last_error() or "DOF" in _lib.last_error()
