"""Input cases and result records in the reference's formats.

Inputs (experiments/session_a/inputs/*.npz, experiments/session_i/make_inputs.py:31-76): an npz with
`shape` (nx, ny, nz), `rho` (element densities), `mask` (0/1 per DOF), `force` and `ke` (24 x 24),
all in the NATURAL layout (x fastest; elements (z, y, x), nodes (z, y, x, 3)); the modulus is
E = floor + (1 - floor) rho^3 with the floor of the protocol (1e-6 in session I).  `load_case`
reads one into the author layout the solvers use; `upsample_case` / `regenerate` are
make_inputs' nearest-neighbour upsampling and its boundary data (clamped x = 0 face, consistent
line load in -z along y at x = nx, z = 0).

Records (experiments/session_i/run_gpu.py:236-240,313-350): `ResultWriter` keeps the reference's
result.json -- the top-level sections (cases, to_tolerance, fixed_work, products, ...), rewritten
after every appended row -- and `solve_record` runs one solve and returns the row the reference
writes for it: iterations, native_converged, native_true_residual, outer_matvecs,
solver_seconds, the physical check (the independent true residual from the reference's C product
-- run here on the device by vx_product --, compliance, force work, their relative error,
physical_passed), solution_sha256 (of the natural-layout solution bytes) and solution_norm.
"""
from __future__ import annotations

import hashlib
import json
import time
from dataclasses import dataclass, field
from datetime import datetime, timezone
from pathlib import Path

import numpy as np
import torch

from .layout import to_author, to_natural

CASE_KEYS = ("shape", "rho", "mask", "force", "ke")


@dataclass
class Case:
    """One input case.  Natural-layout arrays as stored; author-layout views for the solvers."""
    shape: tuple
    rho: np.ndarray
    mask: np.ndarray
    force: np.ndarray
    ke: np.ndarray
    floor: float = 1e-6
    penal: float = 3.0
    name: str = ""
    sha256: str = ""
    author: dict = field(default_factory=dict)

    def modulus(self) -> np.ndarray:
        """E = floor + (1 - floor) rho^penal, natural layout (reference.cc:25)."""
        return self.floor + (1.0 - self.floor) * self.rho ** self.penal

    def author_layout(self):
        """(E, mask, force) in the author layout (cached)."""
        if not self.author:
            self.author = {"E": to_author(self.modulus(), self.shape),
                           "mask": to_author(self.mask, self.shape, True),
                           "force": to_author(self.force, self.shape, True)}
        return self.author["E"], self.author["mask"], self.author["force"]


def _sha(path) -> str:
    return hashlib.sha256(Path(path).read_bytes()).hexdigest()


def load_case(path, floor=1e-6, penal=3.0) -> Case:
    """Read a reference input npz (natural layout); raises ValueError on a missing key or sizes that
    do not match `shape`."""
    path = Path(path)
    with np.load(path) as f:
        missing = [k for k in CASE_KEYS if k not in f.files]
        if missing:
            raise ValueError(f"{path}: missing {missing} (expected keys {CASE_KEYS})")
        d = {k: np.asarray(f[k]) for k in CASE_KEYS}
    shape = tuple(int(s) for s in d["shape"])
    nx, ny, nz = shape
    ne, nd = nx * ny * nz, 3 * (nx + 1) * (ny + 1) * (nz + 1)
    for k, n in (("rho", ne), ("mask", nd), ("force", nd)):
        if d[k].size != n:
            raise ValueError(f"{path}: {k} has {d[k].size} entries, the grid {shape} needs {n}")
    if d["ke"].size != 576:
        raise ValueError(f"{path}: ke must be 24 x 24")
    return Case(shape, d["rho"].astype(np.float64).ravel(), d["mask"].astype(np.float64).ravel(),
                d["force"].astype(np.float64).ravel(), d["ke"].astype(np.float64).reshape(24, 24),
                float(floor), float(penal), path.stem, _sha(path))


def save_case(path, case: Case, compressed=False):
    """Write a case in the reference's npz schema (make_inputs writes uncompressed)."""
    (np.savez_compressed if compressed else np.savez)(
        path, shape=np.array(case.shape), rho=case.rho, mask=case.mask, force=case.force, ke=case.ke)


def regenerate(shape):
    """Boundary data at any resolution (make_inputs.py:31-39): clamped x = 0 face; consistent line load
    in -z along y at x = nx, z = 0 (-1/ny interior, -1/(2 ny) ends).  Natural layout."""
    nx, ny, nz = (int(n) for n in shape)
    mask = np.ones((nz + 1, ny + 1, nx + 1, 3))
    mask[:, :, 0, :] = 0.0
    force = np.zeros((nz + 1, ny + 1, nx + 1, 3))
    line = np.full(ny + 1, -1.0 / ny)
    line[[0, -1]] = -0.5 / ny
    force[0, :, nx, 2] = line
    return mask.ravel(), force.ravel()


def upsample_case(case: Case, factor: int, name=None) -> Case:
    """Repeat each element `factor` times per axis and regenerate the boundary data (make_inputs.py:42-50)."""
    nx, ny, nz = case.shape
    r = case.rho.reshape(nz, ny, nx)
    for axis in range(3):
        r = np.repeat(r, factor, axis=axis)
    shape = (nx * factor, ny * factor, nz * factor)
    mask, force = regenerate(shape)
    return Case(shape, np.ascontiguousarray(r.ravel()), mask, force, case.ke.copy(), case.floor, case.penal,
                name or f"{case.name}x{factor}")


def solve_record(case: Case, solver, arm="", rep=0, true_residual_limit=1e-7, energy_limit=1e-6):
    """Solve case with an ElasticitySolver built on it and return the reference's to_tolerance row
    (run_gpu.py:313-324 plus physical_check, :90-101)."""
    from .operators import product
    E, mask, force = case.author_layout()
    f = torch.as_tensor(force, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = solver.solve(f)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    u_nat = torch.as_tensor(to_natural(res.x.cpu().numpy(), case.shape, True), device="cuda")
    y, ce, _ = product(case.shape, torch.as_tensor(case.rho, device="cuda"), u_nat, case.ke,
                       torch.as_tensor(case.mask, device="cuda"), case.floor, 1.0, case.penal, want=("y", "ce"))
    f_nat = torch.as_tensor(case.force, device="cuda")
    residual = float(torch.linalg.vector_norm(y - f_nat) / torch.linalg.vector_norm(f_nat))
    modulus = torch.as_tensor(case.modulus(), device="cuda")
    compliance, work = float(modulus @ ce), float(f_nat @ u_nat)
    energy_error = abs(compliance / work - 1.0) if work != 0 else float("inf")
    sol = u_nat.cpu().numpy()
    finite = bool(np.isfinite(sol).all())
    fixed_zero = bool(np.all(sol[case.mask == 0] == 0))
    valid = bool(res.converged and res.rel <= solver.fcg.tol and residual <= true_residual_limit
                 and energy_error <= energy_limit and finite and fixed_zero)
    return {"case": case.name, "arm": arm, "rep": rep, "iterations": int(res.iterations),
            "native_converged": bool(res.converged), "native_true_residual": float(res.rel),
            "outer_matvecs": int(res.matvecs), "solver_seconds": seconds,
            "independent_true_residual": residual, "compliance": compliance, "force_work": work,
            "energy_force_relative_error": energy_error, "physical_passed": valid,
            "solution_sha256": hashlib.sha256(np.ascontiguousarray(sol).tobytes()).hexdigest(),
            "solution_norm": float(np.linalg.norm(sol))}


class ResultWriter:
    """result.json in the reference's layout (run_gpu.py:236-240): created at construction, rewritten
    after every append, closed with a status."""

    SECTIONS = ("cases", "to_tolerance", "fixed_work", "profiles", "telemetry", "ladder", "products",
                "product_checks", "variant_differences")

    def __init__(self, out_dir, protocol_sha256=None, dry_run=False, exist_ok=False):
        self.dir = Path(out_dir)
        self.dir.mkdir(parents=True, exist_ok=exist_ok)
        self.path = self.dir / "result.json"
        self.result = {"started_utc": _now(), "status": "running", "dry_run": bool(dry_run),
                       "protocol_sha256": protocol_sha256, **{k: [] for k in self.SECTIONS},
                       "gpu_executed": False, "performance_claim": False, "novelty_claim": False}
        self.write()

    def append(self, section, row):
        if section not in self.SECTIONS:
            raise ValueError(f"unknown section {section!r}; one of {self.SECTIONS}")
        self.result[section].append(row)
        self.write()

    def set(self, **kv):
        self.result.update(kv)
        self.write()

    def write(self):
        tmp = self.path.with_suffix(".json.tmp")
        tmp.write_text(json.dumps(self.result, indent=1, allow_nan=False) + "\n")
        tmp.replace(self.path)

    def finish(self, status="complete"):
        self.result["status"] = status
        self.result["finished_utc"] = _now()
        self.write()
        return self.result


def _now():
    return datetime.now(timezone.utc).strftime("%Y-%m-%dT%H:%M:%SZ")
