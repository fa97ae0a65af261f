"""ctypes binding of the reference's compiled C++ product (oracle/_ref/libreference.so).

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY (see oracle/voxel_oracle.py).  The library is built from the
reference's own sources by ``make -C oracle`` (experiments/session_a/inputs/reference.cc:12-39);
its exported ABI is
    void element(double h, double nu, double* ke);
    void product(int nx, int ny, int nz, const double* rho, const double* u, const double* ke,
                 const double* mask, double emin, double emax, double penal,
                 double* y, double* ce, double* diag);
mirroring the reference's own ctypes wrapper (experiments/session_a/dependencies/common.py:57-69).
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIBRARY = Path(__file__).resolve().parent / "_ref" / "libreference.so"


def available() -> bool:
    return LIBRARY.exists()


class ReferenceProduct:
    def __init__(self, library=LIBRARY):
        self.lib = ctypes.CDLL(str(library))
        arr = np.ctypeslib.ndpointer(dtype=np.float64, ndim=1, flags="C_CONTIGUOUS")
        self.lib.product.argtypes = [ctypes.c_int] * 3 + [arr] * 4 + [ctypes.c_double] * 3 + [arr] * 3
        self.lib.product.restype = None
        self.lib.element.argtypes = [ctypes.c_double, ctypes.c_double, arr]
        self.lib.element.restype = None

    def element(self, h, nu):
        ke = np.zeros(576)
        self.lib.element(float(h), float(nu), ke)
        return ke.reshape(24, 24)

    def product(self, shape, rho, u, ke, mask, emin, emax=1.0, penal=3.0):
        """Natural layout in and out: returns (y, ce, diag)."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        mask = np.ascontiguousarray(mask, dtype=np.float64)
        y, ce, d = np.empty_like(u), np.empty_like(rho), np.empty_like(u)
        self.lib.product(*(int(s) for s in shape), rho, u,
                         np.ascontiguousarray(ke, dtype=np.float64).ravel(), mask,
                         float(emin), float(emax), float(penal), y, ce, d)
        return y, ce, d
