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
