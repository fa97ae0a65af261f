"""The reference's physical acceptance test of a solution (experiments/session_i/run_gpu.py:90-101,
limits from experiments/session_i/protocol.json:87-88), applied to GPU solutions:

* the independent true residual |f - A u| / |f|, with A u computed by the reference's own compiled
  C++ product (reference.cc, oracle/_ref; its NumPy restatement where it is not built), <= 1e-7;
* energy-force consistency |sum_e E_e u_e^T ke u_e / f.u - 1| <= 1e-6;
* every entry finite and every fixed DOF exactly zero.

Test infrastructure: inputs in the author layout (numpy), converted to the C product's natural
layout here."""
import numpy as np

from oracle import ref_product
from oracle import voxel_oracle as vo

TRUE_RESIDUAL_LIMIT = 1e-7
ENERGY_FORCE_LIMIT = 1e-6


def physical_check(shape, ke, rho, floor, mask, force, u, penal=3.0):
    rho, mask, force, u = (np.asarray(a, dtype=np.float64) for a in (rho, mask, force, u))
    rho_n = vo.to_natural(rho, shape)
    m_n, f_n, u_n = (vo.to_natural(a, shape, True) for a in (mask, force, u))
    if ref_product.available():
        y, ce, _ = ref_product.ReferenceProduct().product(shape, rho_n, u_n, ke, m_n, floor, 1.0, penal)
        source = "reference.cc"
    else:
        y, ce, _ = vo.c_reference_product(shape, rho_n, u_n, ke, m_n, floor, 1.0, penal)
        source = "numpy restatement of reference.cc"
    residual = float(np.linalg.norm(y - f_n) / np.linalg.norm(f_n))
    modulus = floor + (1.0 - floor) * rho_n ** penal
    compliance, work = float(modulus @ ce), float(f_n @ u_n)
    energy_error = abs(compliance / work - 1.0) if work != 0 else float("inf")
    finite = bool(np.isfinite(u).all())
    fixed_zero = bool(np.all(u[mask == 0] == 0))
    ok = residual <= TRUE_RESIDUAL_LIMIT and energy_error <= ENERGY_FORCE_LIMIT and finite and fixed_zero
    return {"independent_true_residual": residual, "compliance": compliance, "force_work": work,
            "energy_force_relative_error": energy_error, "finite": finite, "fixed_dofs_zero": fixed_zero,
            "product": source, "passed": bool(ok)}
