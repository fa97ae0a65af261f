"""CPU checks of the C ABI: the library loads and exports every entry point include/voxel_b200.h
declares; host-side entry points (element matrix, parity blocks, argument validation) work
without a GPU.  No device compute is called here."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import REPO
from oracle import voxel_oracle as vo

vx = pytest.importorskip("voxel_b200")
HEADERS = sorted((REPO / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vx_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(vx._lib.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_table_covers_header():
    assert declared_functions() <= set(vx._lib.SIGNATURES), declared_functions() - set(vx._lib.SIGNATURES)


def test_host_element_and_blocks_match_oracle():
    for lengths, nu in (([1, 1, 1], 0.3), ([1.0, 0.5, 2.0], 0.25), ([0.25] * 3, 0.3)):
        ke = vx.quadrature(lengths, nu)
        assert np.abs(ke - vo.quadrature(lengths, nu)).max() <= 1e-15 * np.abs(ke).max() * 4
        b, disc = vo.parity_blocks(ke)
        m = vx.Modal(ke)
        assert np.abs(m.blocks - b).max() <= 1e-15 * np.abs(b).max() * 8
        assert m.discarded_relative < 2e-14
    assert np.abs(vx.element(1.0, 0.3) - vo.quadrature([1, 1, 1], 0.3)).max() < 1e-16


def test_element_outside_block_model_is_rejected():
    ke = vo.quadrature([1, 1, 1], 0.3)
    ke[0, 5] += 1e-3
    ke[5, 0] += 1e-3
    with pytest.raises(ValueError):
        vx.Modal(ke)


def test_status_codes_and_messages():
    lib = vx._lib.load()
    ke = np.zeros(576)
    assert lib.vx_element_matrix(-1.0, 1.0, 1.0, 0.3, vx._lib.dptr(ke)) == vx._lib.VX_ERR_INVALID_ARGUMENT
    assert "positive" in vx._lib.last_error()
    # shape validation happens before any device work
    assert lib.vx_matvec(0, 0, 4, 4, vx._lib.dptr(np.zeros(72)), None, None, None, None, None) != 0
    assert lib.vx_partials_size(10) >= 1
    assert lib.vx_version() >= 10000


def test_argument_validation_happens_before_any_device_work():
    """Every check below fails before a kernel is launched or device memory touched, so it runs on
    a machine without a GPU: the limits (fewer than 2^31 DOFs; launch-grid extents), precision
    selectors, NULL pointers, aliasing, and the modes each entry point supports."""
    lib = vx._lib.load()
    L = vx._lib
    host = np.zeros(1024)
    p = L.dptr(host)                                   # a valid-looking pointer that is never used
    blocks = L.dptr(np.zeros(72))
    INV, NUL = L.VX_ERR_INVALID_ARGUMENT, L.VX_ERR_NULL_POINTER

    # 3 * 1001^3 >= 2^31 DOFs
    assert lib.vx_matvec(L.VX_F64, 1000, 1000, 1000, blocks, p, p, p, None, None) == INV
    assert "2^31" in L.last_error()
    assert lib.vx_jacobi_sweep(L.VX_F64, 0, 4, 4, blocks, p, None, p, p, p, 0.6, p, None) == INV
    # unknown storage selectors
    assert lib.vx_matvec(9, 4, 4, 4, blocks, p, p, p, None, None) == INV
    assert lib.vx_restrict(9, 4, 4, 4, p, None, p, None) == INV
    assert lib.vx_prolong_add(-1, 4, 4, 4, p, None, p, None) == INV
    assert lib.vx_coarse_apply_factor(7, 10, p, p, None, p, p, None) == INV
    assert lib.vx_vcycle_entry(5, 10, p, p, p, 0.6, p, None) == INV
    assert lib.vx_cg_direction_update(4, 10, p, p, p, None, p, None) == INV
    # the reducing forms exist for VX_F64 and VX_F32 only
    assert lib.vx_apply_dot(L.VX_BF16_F32, 4, 4, 4, blocks, p, None, p, L.dptr(np.zeros(8)), p, None) == INV
    assert lib.vx_apply_dot(L.VX_F32_BF16AUX, 4, 4, 4, blocks, p, None, p, L.dptr(np.zeros(8)), p, None) == INV
    # transfers need even fine grids
    assert lib.vx_restrict(L.VX_F32, 5, 4, 4, p, None, p, None) == INV
    assert "even" in L.last_error()
    # NULL pointers and aliasing
    assert lib.vx_matvec(L.VX_F64, 4, 4, 4, blocks, None, p, p, None, None) == NUL
    assert lib.vx_residual(L.VX_F64, 4, 4, 4, blocks, p, None, p, p, p, None) == INV          # out aliases x
    assert lib.vx_coarse_pack(10, p, p, None) == INV                                       # m aliases linv
    assert lib.vx_coarse_apply(L.VX_F64, 0, p, p, None, p, None) == INV
    # SIMP filter radius limits and modes
    assert lib.vx_cone_filter(4, 4, 4, 9.0, p, p, 1, L.dptr(np.zeros(64)), None) == INV
    assert lib.vx_cone_filter(4, 4, 4, 1.5, p, p, 3, L.dptr(np.zeros(64)), None) == INV
    # the solver scalar array has 16 slots
    assert lib.vx_set_scalars(p, 15, 2, 0.0, None) == INV
