"""Problem builders (author layout, on the device): the cantilever boundary conditions and the
seeded density fields of the benchmark workloads.

* `cantilever_equal_split`: x = 0 face clamped, total load -1 in z split equally over the nodes
  (ix = nx, iy = 0..ny, iz = 0) -- the rule of the reference's synthetic MG test case
  (tests/test_mg_cpu.py:140-155).
* `cantilever_line_load`: the consistent line load of experiments/session_i/make_inputs.py:31-39
  (natural layout, as the reference's fixtures store it).
* `uniform_density`, `gaussian_random_field`: seeded synthetic densities (there is no public
  dataset on this path); the GRF is white noise smoothed by exp(-2 pi^2 l^2 |k|^2), standardised
  and mapped through a logistic to [1e-3, 1].
"""
from __future__ import annotations

import numpy as np
import torch


def cantilever_equal_split(shape, device="cuda"):
    """(dof_mask, force) float64 tensors, author layout."""
    nx, ny, nz = (int(s) for s in shape)
    mask = torch.ones(nx + 1, ny + 1, nz + 1, 3, dtype=torch.float64, device=device)
    mask[0] = 0.0
    force = torch.zeros(nx + 1, ny + 1, nz + 1, 3, dtype=torch.float64, device=device)
    force[nx, :, 0, 2] = -1.0 / (ny + 1)
    return mask.reshape(-1), force.reshape(-1)


def cantilever_node_mask(shape, device="cuda"):
    """uint8 node mask of the clamped x = 0 face (bit c set <=> DOF c free)."""
    nx, ny, nz = (int(s) for s in shape)
    m = torch.full((nx + 1, ny + 1, nz + 1), 7, dtype=torch.uint8, device=device)
    m[0] = 0
    return m.reshape(-1)


def cantilever_line_load(shape):
    """(mask, force) numpy float64, NATURAL layout (x fastest)."""
    nx, ny, nz = (int(s) for s in shape)
    mask = np.ones((nz + 1, ny + 1, nx + 1, 3))
    mask[:, :, 0, :] = 0.0
    force = np.zeros((nz + 1, ny + 1, nx + 1, 3))
    line = np.full(ny + 1, -1.0 / ny)
    line[[0, -1]] = -0.5 / ny
    force[0, :, nx, 2] = line
    return mask.ravel(), force.ravel()


def _clamped_face(nx, ny, nz):
    """DOF mask with every DOF of the x = 0 face fixed (author layout, numpy)."""
    mask = np.ones((nx + 1, ny + 1, nz + 1, 3))
    mask[0] = 0.0
    return mask


def _face_indices(n_nodes, h, centre, half, tol=1e-12, exact=False):
    """Node indices along one face axis whose coordinate i*h lies within the patch; the nearest
    node when none does.  `exact` uses the |coord - centre| <= half test of the torsion patches."""
    coords = np.arange(n_nodes) * h
    if exact:
        sel = np.abs(coords - centre) <= half + tol
    else:
        sel = (coords >= centre - half - tol) & (coords <= centre + half + tol)
    idx = np.nonzero(sel)[0]
    return idx if idx.size else np.array([int(round(centre / h))])


def donor_cantilever(nelx, nely, nelz, Lx=2.0, Ly=1.0, Lz=0.5, load="patch", patch_frac=None,
                     patch_size=0.1, total_load=-1.0):
    """The donor SIMP benchmark's cantilever (experiments/session_a/donor/src/gpu_fem/simp_r2.py:64-131):
    the x = 0 face clamped; a transverse (y) load on the x = nelx face, either at the node nearest
    the face centre ("point") or spread evenly over the nodes of a square patch of fixed physical
    side centred there ("patch"; side patch_frac * Lz when given, else patch_size).  Returns
    (dof_mask, force, patch_nodes) as numpy float64 arrays in author layout."""
    nx, ny, nz = int(nelx), int(nely), int(nelz)
    mask = _clamped_face(nx, ny, nz)
    force = np.zeros((nx + 1, ny + 1, nz + 1, 3))
    hy, hz = Ly / ny, Lz / nz
    if load == "point":
        jy, jz = int(round((Ly / 2.0) / hy)), int(round((Lz / 2.0) / hz))
        force[nx, jy, jz, 1] = total_load
        count = 1
    elif load == "patch":
        side = float(patch_size) if patch_frac is None else float(patch_frac) * Lz
        jy = _face_indices(ny + 1, hy, Ly / 2.0, side / 2.0)
        jz = _face_indices(nz + 1, hz, Lz / 2.0, side / 2.0)
        count = jy.size * jz.size
        force[nx, jy[:, None], jz[None, :], 1] = total_load / count
    else:
        raise ValueError(f"unknown load model {load!r}")
    return mask.reshape(-1), force.reshape(-1), count


def donor_torsion(nelx, nely, nelz, Lx=3.0, Ly=1.0, Lz=1.0, patch_size=0.15, total_load=1.0):
    """The donor's torsion shaft (simp_r2.py:134-178): the x = 0 face clamped; on the x = nelx face a
    couple from two patches at y = Ly and y = 0 (the z band of width patch_size around Lz / 2),
    forces (-1/2, +1/2) and (+1/2, -1/2) times total_load in (y, z), each spread evenly over its
    patch.  Returns (dof_mask, force, patch_nodes)."""
    nx, ny, nz = int(nelx), int(nely), int(nelz)
    mask = _clamped_face(nx, ny, nz)
    force = np.zeros((nx + 1, ny + 1, nz + 1, 3))
    hy, hz = Ly / ny, Lz / nz
    jz = _face_indices(nz + 1, hz, Lz / 2.0, patch_size / 2.0, exact=True)
    count = 0
    for y_target, sy, sz in ((Ly, -0.5, 0.5), (0.0, 0.5, -0.5)):
        jy = _face_indices(ny + 1, hy, y_target, patch_size / 2.0, exact=True)
        k = jy.size * jz.size
        force[nx, jy[:, None], jz[None, :], 1] += total_load * sy / k
        force[nx, jy[:, None], jz[None, :], 2] += total_load * sz / k
        count += k
    return mask.reshape(-1), force.reshape(-1), count


def upsample_natural(rho, shape, factor):
    """Nearest-neighbour repeat of a natural-layout element field (make_inputs.py:42-50)."""
    nx, ny, nz = (int(s) for s in shape)
    r = np.asarray(rho).reshape(nz, ny, nx)
    for axis in range(3):
        r = np.repeat(r, factor, axis=axis)
    return np.ascontiguousarray(r.ravel()), (nx * factor, ny * factor, nz * factor)


def uniform_density(shape, seed=0, low=0.01, high=1.0, device="cuda"):
    n = int(np.prod(shape))
    return torch.as_tensor(np.random.default_rng(seed).uniform(low, high, n), device=device)


def gaussian_random_field(shape, ell, seed, device="cuda"):
    """Seeded GRF density in [1e-3, 1] (FP64, author element layout), FFT on the device."""
    nx, ny, nz = (int(s) for s in shape)
    w = torch.as_tensor(np.random.default_rng(seed).standard_normal((nx, ny, nz)), device=device)
    kx = torch.fft.fftfreq(nx, dtype=torch.float64, device=device)[:, None, None]
    ky = torch.fft.fftfreq(ny, dtype=torch.float64, device=device)[None, :, None]
    kz = torch.fft.fftfreq(nz, dtype=torch.float64, device=device)[None, None, :]
    filt = torch.exp(-2 * np.pi ** 2 * ell ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    g = torch.fft.ifftn(torch.fft.fftn(w) * filt).real
    del w, filt
    g = (g - g.mean()) / g.std(correction=0)
    return (1e-3 + (1 - 1e-3) / (1 + torch.exp(-g))).reshape(-1).contiguous()


def simp_modulus(rho, emin=1e-9, e0=1.0, penal=3.0):
    return emin + (e0 - emin) * rho ** penal


# The benchmark workloads (synthetic inputs with the shapes and distributions the workloads name).
WORKLOADS = {
    "jacobi_32x16x16": dict(shape=(32, 16, 16), density=("uniform", 0), emin=1e-9, solver="jacobi",
                            tol=1e-8),
    "gmg_128x64x64": dict(shape=(128, 64, 64), density=("grf", 8.0, 0), emin=1e-9, solver="gmg", levels=4,
                          pre=2, post=2, omega=0.6, tol=1e-8),
    "gmg_576x288x288": dict(shape=(576, 288, 288), density=("grf", 16.0, 0), emin=1e-9, solver="gmg", levels=6,
                            pre=2, post=2, omega=0.6, tol=1e-8),
}


def density(spec, shape, device="cuda"):
    kind = spec[0]
    if kind == "uniform":
        return uniform_density(shape, seed=spec[1], device=device)
    if kind == "grf":
        return gaussian_random_field(shape, spec[1], spec[2], device=device)
    raise ValueError(f"unknown density {spec}")
