"""Hex8 element matrix and its parity (Walsh-Hadamard) blocks, computed by libvoxel_b200's host
code.  Mirrors code/hex_modal/modal.py:19-40 (quadrature) and :55-77 (Modal)."""
from __future__ import annotations

import numpy as np

from . import _lib

# Native Hex8 node order of `ke` (code/hex_modal/modal.py:9-10, src/voxel_mg.py:27-28).
XYZ = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])


def quadrature(lengths, nu) -> np.ndarray:
    """24x24 element matrix of an isotropic brick (unit Young's modulus, 2x2x2 Gauss)."""
    hx, hy, hz = (float(v) for v in np.broadcast_to(np.asarray(lengths, dtype=float), (3,)))
    ke = np.zeros(576)
    _lib.call("vx_element_matrix", hx, hy, hz, float(nu), _lib.dptr(ke))
    return ke.reshape(24, 24)


def element(h, nu) -> np.ndarray:
    """Cube element of edge h (the reference C oracle's element(h, nu, ke))."""
    ke = np.zeros(576)
    _lib.call("vx_element", float(h), float(nu), _lib.dptr(ke))
    return ke.reshape(24, 24)


class Modal:
    """Parity blocks of an element matrix; raises ValueError outside the block model."""

    def __init__(self, ke, tolerance=2e-14):
        self.ke = np.ascontiguousarray(np.asarray(ke, dtype=np.float64).reshape(24, 24))
        blocks = np.zeros(72)
        disc = np.zeros(1)
        _lib.call("vx_parity_blocks", _lib.dptr(self.ke), _lib.dptr(blocks), _lib.dptr(disc))
        self.discarded_relative = float(disc[0])
        if self.discarded_relative > tolerance:
            raise ValueError(f"Element is outside the declared parity-block model: {self.discarded_relative}")
        self.blocks = blocks.reshape(8, 3, 3)
