"""The tensor-core element-block operator (tcgen05.mma, TF32 operands, FP32 accumulation in tensor
memory): per-element block products and the scattered operator against the FP64 oracle.
Tolerance: 3e-3 relative to the largest entry (TF32 keeps 10 mantissa bits of each operand)."""
import numpy as np
import pytest
import torch

from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import _lib  # noqa: E402
from voxel_b200.operators import tc_element_product  # noqa: E402

KE = vo.quadrature([1, 1, 1], 0.3)
OX, OY, OZ = [0, 1, 1, 0, 0, 1, 1, 0], [0, 0, 1, 1, 0, 0, 1, 1], [0, 0, 0, 0, 1, 1, 1, 1]


def element_vectors(shape, u):
    """(Ne, 24) element DOF vectors in the element matrix's native node order, author layout."""
    nx, ny, nz = shape
    U = u.reshape(nx + 1, ny + 1, nz + 1, 3)
    cols = [U[OX[n]:OX[n] + nx, OY[n]:OY[n] + ny, OZ[n]:OZ[n] + nz, :] for n in range(8)]
    return np.concatenate(cols, axis=-1).reshape(-1, 24)


@pytest.mark.parametrize("shape", [(3, 4, 200), (5, 2, 31), (2, 3, 128)])
def test_block_products_and_operator_match_the_oracle(shape):
    rng = np.random.default_rng(sum(shape))
    E = (1e-3 + rng.random(int(np.prod(shape)))).astype(np.float32)
    u = rng.standard_normal(3 * vo.n_nodes(shape)).astype(np.float32)
    mask, _ = vo.cantilever_equal_split(shape)
    Et, ut = torch.as_tensor(E, device="cuda"), torch.as_tensor(u, device="cuda")
    nm = vx.node_mask_from_dofs(torch.as_tensor(mask, device="cuda"))
    um = u.astype(np.float64) * mask
    # per element: E_e K0 u_e
    ye = tc_element_product(shape, KE, Et, ut, nm, per_element=True).double().cpu().numpy()
    ref = element_vectors(shape, um) @ KE.T * E.astype(np.float64)[:, None]
    assert np.abs(ye - ref).max() <= 3e-3 * np.abs(ref).max()
    # scattered over the nodes: K(E) (m . u)
    y = tc_element_product(shape, KE, Et, ut, nm).double().cpu().numpy()
    ref = vo.product_raw(shape, KE, um, E.astype(np.float64))
    assert np.abs(y - ref).max() <= 3e-3 * np.abs(ref).max()
    v = ctypes_status()
    assert v == 0


def ctypes_status():
    import ctypes
    v = ctypes.c_int(0)
    _lib.check(_lib.load().vx_tc_status(ctypes.byref(v), 1), "vx_tc_status")
    return v.value
