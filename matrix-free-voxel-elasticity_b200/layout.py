"""Index maps and layout converters (author layout: x slowest, z fastest).

Mirrors src/voxel_mg.py:32-38 (edof_author), src/voxel_kernels.py:46-53 (element_nodes) and
experiments/session_a/dependencies/common.py:35-46 (to_author / to_natural).  The converters
work on numpy arrays and torch tensors alike; the index tables are host-side setup utilities
(the kernels compute indices analytically).
"""
from __future__ import annotations

import numpy as np

from .element import XYZ


def n_nodes(shape) -> int:
    nx, ny, nz = (int(s) for s in shape)
    return (nx + 1) * (ny + 1) * (nz + 1)


def n_elems(shape) -> int:
    nx, ny, nz = (int(s) for s in shape)
    return nx * ny * nz


def to_author(a, shape, nodal=False):
    """Natural (x fastest) -> author (z fastest)."""
    nx, ny, nz = (int(s) for s in shape)
    if hasattr(a, "permute"):
        if nodal:
            return a.reshape(nz + 1, ny + 1, nx + 1, 3).permute(2, 1, 0, 3).contiguous().reshape(-1)
        return a.reshape(nz, ny, nx).permute(2, 1, 0).contiguous().reshape(-1)
    if nodal:
        return np.ascontiguousarray(a.reshape(nz + 1, ny + 1, nx + 1, 3).transpose(2, 1, 0, 3)).ravel()
    return np.ascontiguousarray(a.reshape(nz, ny, nx).transpose(2, 1, 0)).ravel()


def to_natural(a, shape, nodal=False):
    nx, ny, nz = (int(s) for s in shape)
    if hasattr(a, "permute"):
        if nodal:
            return a.reshape(nx + 1, ny + 1, nz + 1, 3).permute(2, 1, 0, 3).contiguous().reshape(-1)
        return a.reshape(nx, ny, nz).permute(2, 1, 0).contiguous().reshape(-1)
    if nodal:
        return np.ascontiguousarray(a.reshape(nx + 1, ny + 1, nz + 1, 3).transpose(2, 1, 0, 3)).ravel()
    return np.ascontiguousarray(a.reshape(nx, ny, nz).transpose(2, 1, 0)).ravel()


def edof_author(shape) -> np.ndarray:
    """(Ne, 24) DOF indices in author layout for the native node order of ke."""
    nx, ny, nz = (int(s) for s in shape)
    ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    nodes = [((ex + x) * (ny + 1) + ey + y) * (nz + 1) + ez + z for x, y, z in XYZ]
    return np.stack([3 * n + c for n in nodes for c in range(3)], axis=1)


def element_nodes(shape) -> np.ndarray:
    """(Ne, 8) global node of each element per binary lane b = bx + 2 by + 4 bz."""
    nx, ny, nz = (int(s) for s in shape)
    e = np.arange(nx * ny * nz)
    ez, ey, ex = e % nz, (e // nz) % ny, e // (nz * ny)
    b = np.arange(8)
    return (((ex[:, None] + (b & 1)) * (ny + 1) + ey[:, None] + ((b >> 1) & 1)) * (nz + 1)
            + ez[:, None] + ((b >> 2) & 1))
