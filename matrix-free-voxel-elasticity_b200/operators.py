"""Device-side voxel operator over torch tensors, calling libvoxel_b200 kernels.

`VoxelOperator` holds one grid and element matrix and exposes every operator form the solvers
need: the raw product K(E) u, the Dirichlet operator M K M + (I - M), the Jacobi (inverse)
diagonal, fused smoother / residual / outer-CG forms, the element energy and the transfers.
`Product` is the reference's duck-typed "product" protocol (`raw(u, E)`, `diagonal(E)`,
src/voxel_mg.py:41-58, experiments/session_i/run_gpu.py:43-66) on top of it.

All tensors are CUDA, contiguous, author layout.  Nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .element import Modal
from .layout import n_elems, n_nodes

PREC = {torch.float64: _lib.VX_F64, torch.float32: _lib.VX_F32, torch.bfloat16: _lib.VX_BF16_F32}
# (iterate dtype, auxiliary dtype) -> storage selector; the modulus is stored like the auxiliary vectors
STORAGE = {(torch.float64, torch.float64): _lib.VX_F64, (torch.float32, torch.float32): _lib.VX_F32,
           (torch.bfloat16, torch.bfloat16): _lib.VX_BF16_F32, (torch.float32, torch.bfloat16): _lib.VX_F32_BF16AUX}


_RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_CUR_DEVICE = getattr(torch._C, "_cuda_getDevice", None)


def stream_ptr(device=None) -> int:
    """cudaStream_t of the current stream (of the current device when `device` is None).  The
    host-driven loops ask for it once per launch, so on the current device it is read with torch's
    raw-stream accessor, without building a Stream object and resolving the device index."""
    if device is None and _RAW_STREAM is not None and _CUR_DEVICE is not None and torch.cuda.is_initialized():
        return _RAW_STREAM(_CUR_DEVICE())
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t, what, dtype=None, numel=None, allow_none=False):
    if t is None:
        if allow_none:
            return None
        raise ValueError(f"{what}: tensor is required")
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{what}: expected a CUDA tensor, got {type(t).__name__}"
                         f"{'' if not isinstance(t, torch.Tensor) else ' on ' + str(t.device)}")
    if not t.is_contiguous():
        raise ValueError(f"{what}: tensor must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{what}: expected dtype {dtype}, got {t.dtype}")
    if numel is not None and t.numel() != numel:
        raise ValueError(f"{what}: expected {numel} elements, got {t.numel()}")
    return t.data_ptr()


def node_mask_from_dofs(dof_mask: torch.Tensor) -> torch.Tensor:
    """uint8 node mask (bit c set <=> DOF c free) from the reference's 0/1 DOF mask (3N floats)."""
    m = dof_mask if dof_mask.dtype == torch.float64 else dof_mask.to(torch.float64)
    m = m.contiguous()
    nodes = m.numel() // 3
    out = torch.empty(nodes, dtype=torch.uint8, device=m.device)
    _lib.call("vx_mask_from_dofs", nodes, _ptr(m, "dof_mask"), _ptr(out, "node_mask"), stream_ptr(m.device))
    return out


def dofs_from_node_mask(node_mask: torch.Tensor, dtype=torch.float64) -> torch.Tensor:
    bits = node_mask.to(torch.int32)
    return torch.stack([(bits >> c) & 1 for c in range(3)], dim=1).reshape(-1).to(dtype)


class VoxelOperator:
    """K(E) on a (nx, ny, nz) voxel grid in `dtype` storage (float64, float32, or bfloat16 with
    FP32 arithmetic).  `aux_dtype` (default `dtype`) is the storage of the modulus and of the
    auxiliary vectors (right-hand side, inverse diagonal, residual output); float32 iterates with
    bfloat16 auxiliaries is the VX_F32_BF16AUX mode."""

    def __init__(self, shape, ke, dtype=torch.float64, aux_dtype=None):
        self.shape = tuple(int(s) for s in shape)
        if len(self.shape) != 3 or min(self.shape) < 1:
            raise ValueError(f"invalid grid {shape}")
        self.ke = np.ascontiguousarray(np.asarray(ke, dtype=np.float64).reshape(24, 24))
        self.blocks = np.ascontiguousarray(Modal(self.ke).blocks.reshape(72))
        aux_dtype = dtype if aux_dtype is None else aux_dtype
        if (dtype, aux_dtype) not in STORAGE:
            raise ValueError(f"unsupported storage: iterate {dtype}, auxiliary {aux_dtype}")
        self.dtype, self.aux_dtype = dtype, aux_dtype
        self.prec = STORAGE[(dtype, aux_dtype)]
        self.nodes = n_nodes(self.shape)
        self.ndof = 3 * self.nodes
        self.n_elem = n_elems(self.shape)
        self._bp = _lib.dptr(self.blocks)
        self._kp = _lib.dptr(self.ke)

    # --------------------------------------------------------------- helpers
    @property
    def partials_size(self) -> int:
        """doubles of scratch the fused reducing forms (apply_dot / true_residual) need"""
        return int(_lib.load().vx_operator_partials(self.prec, *self.shape))

    def _vec(self, t, what, dtype=None):
        return _ptr(t, what, dtype or self.dtype, self.ndof)

    def _E(self, E, dtype=None):
        return _ptr(E, "E", dtype or self.aux_dtype, self.n_elem)

    def _mask(self, m):
        return _ptr(m, "node_mask", torch.uint8, self.nodes, allow_none=True)

    def _out(self, out, like_dtype=None):
        dt = like_dtype or (torch.float32 if self.dtype == torch.bfloat16 else self.dtype)
        if out is None:
            return torch.empty(self.ndof, dtype=dt, device="cuda")
        return out

    # --------------------------------------------------------------- products
    def matvec(self, u, E, node_mask=None, out=None):
        """y = K u (node_mask None) or y = M K (M u) + (I - M) u."""
        y = self._out(out)
        _lib.call("vx_matvec", self.prec, *self.shape, self._bp, self._E(E), self._vec(u, "u"),
                  _ptr(y, "y", torch.float32 if self.dtype == torch.bfloat16 else self.dtype, self.ndof),
                  self._mask(node_mask), stream_ptr())
        return y

    def matvec_dense(self, u, E, out=None):
        """Independent control path: node-owned dense 24x24 gather (FP64/FP32)."""
        if self.dtype not in (torch.float64, torch.float32):
            raise ValueError("matvec_dense supports float64/float32")
        y = self._out(out)
        ke = torch.as_tensor(self.ke, dtype=self.dtype, device="cuda").contiguous()
        _lib.call("vx_matvec_dense", self.prec, *self.shape, ke.data_ptr(), self._E(E), self._vec(u, "u"),
                  self._vec(y, "y"), stream_ptr())
        return y

    def diagonal(self, E, node_mask=None, inverse=False, out=None):
        dt = torch.float32 if self.dtype == torch.bfloat16 else self.dtype
        d = self._out(out, dt)
        _lib.call("vx_diagonal", PREC[dt], *self.shape, self._kp, self._E(E, dt), self._mask(node_mask),
                  int(bool(inverse)), _ptr(d, "d", dt, self.ndof), stream_ptr())
        return d

    def jacobi(self, x, r, inv_diag, E, node_mask, omega, out=None):
        """out = x + omega * inv_diag * (r - A x), A the Dirichlet operator (bfloat16: every
        vector in bf16, FP32 arithmetic)."""
        o = self._out(out, self.dtype)
        _lib.call("vx_jacobi_sweep", self.prec, *self.shape, self._bp, self._E(E), self._mask(node_mask),
                  self._vec(x, "x"), self._vec(r, "r", self.aux_dtype), self._vec(inv_diag, "inv_diag", self.aux_dtype),
                  float(omega), self._vec(o, "out"), stream_ptr())
        return o

    def residual(self, x, r, E, node_mask, out=None):
        """out = (r - A x) * M."""
        o = self._out(out, self.aux_dtype)
        _lib.call("vx_residual", self.prec, *self.shape, self._bp, self._E(E), self._mask(node_mask),
                  self._vec(x, "x"), self._vec(r, "r", self.aux_dtype), self._vec(o, "out", self.aux_dtype),
                  stream_ptr())
        return o

    def apply_dot(self, p, E, node_mask, q, partials):
        """q = A p; partials[cta] = sum p.q over the CTA's nodes (reduce with reduce_partials)."""
        _lib.call("vx_apply_dot", self.prec, *self.shape, self._bp, self._E(E), self._mask(node_mask),
                  self._vec(p, "p"), self._vec(q, "q"), _ptr(partials, "partials", torch.float64), stream_ptr())

    def true_residual(self, x, b, E, node_mask, res, partials):
        """res = b - A x; partials[cta] = sum res^2 over the CTA's nodes."""
        _lib.call("vx_true_residual", self.prec, *self.shape, self._bp, self._E(E), self._mask(node_mask),
                  self._vec(x, "x"), self._vec(b, "b"), self._vec(res, "res"),
                  _ptr(partials, "partials", torch.float64), stream_ptr())

    def energy(self, u, rho=None, emin=1e-9, emax=1.0, penal=3.0, ce=None, dc=None):
        """ce_e = u_e^T ke u_e (FP64); with rho also dc_e = -p rho^(p-1) (emax-emin) ce_e."""
        ce = torch.empty(self.n_elem, dtype=torch.float64, device="cuda") if ce is None else ce
        if rho is not None and dc is None:
            dc = torch.empty(self.n_elem, dtype=torch.float64, device="cuda")
        _lib.call("vx_element_energy", *self.shape, self._kp, self._vec(u, "u", torch.float64),
                  _ptr(ce, "ce", torch.float64, self.n_elem),
                  _ptr(rho, "rho", torch.float64, self.n_elem, allow_none=True),
                  float(emin), float(emax), float(penal),
                  _ptr(dc, "dc", torch.float64, self.n_elem, allow_none=True), stream_ptr())
        return (ce, dc) if rho is not None else ce


class Product:
    """The reference's product protocol on the device: raw(u, E) -> K(E) u with u pre-masked,
    diagonal(E) -> diag K(E) (src/voxel_mg.py:41-58).  Returns fresh tensors (the reference's
    CudaModal reused one output buffer, code/hex_modal_cuda/cuda.py:96-101)."""

    def __init__(self, shape, ke, dtype=torch.float64):
        self.op = VoxelOperator(shape, ke, dtype)
        self.shape, self.dtype, self.ndof = self.op.shape, dtype, self.op.ndof

    def raw(self, u, E):
        return self.op.matvec(u, E)

    def diagonal(self, E):
        return self.op.diagonal(E)


def reduce_partials(partials: torch.Tensor, G: int, count: int = 1, out: torch.Tensor | None = None):
    out = torch.empty(count, dtype=torch.float64, device=partials.device) if out is None else out
    _lib.call("vx_reduce_partials", int(G), int(count), _ptr(partials, "partials", torch.float64),
              _ptr(out, "out", torch.float64), stream_ptr())
    return out


def dots(pairs, partials=None, out=None):
    """Deterministic FP64 dot products of up to 3 (a, b) pairs of equal-length CUDA vectors."""
    a0 = pairs[0][0]
    n = a0.numel()
    prec = PREC[a0.dtype]
    G = int(_lib.load().vx_partials_size(n))
    if partials is None:
        partials = torch.empty(G * len(pairs), dtype=torch.float64, device=a0.device)
    out = torch.empty(len(pairs), dtype=torch.float64, device=a0.device) if out is None else out
    A = (ctypes.c_void_p * 3)(*[_ptr(a, "a", a0.dtype, n) for a, _ in pairs])
    B = (ctypes.c_void_p * 3)(*[_ptr(b, "b", a0.dtype, n) for _, b in pairs])
    _lib.call("vx_dots", prec, n, len(pairs), A, B, _ptr(partials, "partials", torch.float64),
              _ptr(out, "out", torch.float64), stream_ptr())
    return out


def simp_modulus(rho, emin, emax=1.0, penal=3.0, dtype=torch.float64, out=None):
    out = torch.empty(rho.numel(), dtype=dtype, device=rho.device) if out is None else out
    _lib.call("vx_simp_modulus", PREC[out.dtype], rho.numel(), _ptr(rho, "rho", torch.float64), float(emin),
              float(emax), float(penal), _ptr(out, "E"), stream_ptr())
    return out


def cast(src, dtype, scale=1.0, out=None):
    out = torch.empty(src.numel(), dtype=dtype, device=src.device) if out is None else out
    _lib.call("vx_cast", src.numel(), PREC[src.dtype], _ptr(src, "src"), PREC[out.dtype], _ptr(out, "dst"),
              float(scale), stream_ptr())
    return out


def product(shape, rho, u, ke, mask, emin, emax=1.0, penal=3.0, want=("y", "ce", "diag")):
    """The reference C product (experiments/session_a/inputs/reference.cc:16-39) on the device,
    natural layout: returns (y, ce, diag) (None where not requested)."""
    nx, ny, nz = (int(s) for s in shape)
    nd = 3 * n_nodes(shape)
    ne = n_elems(shape)
    ke = np.ascontiguousarray(np.asarray(ke, dtype=np.float64).reshape(24, 24))
    y = torch.empty(nd, dtype=torch.float64, device="cuda") if "y" in want else None
    ce = torch.empty(ne, dtype=torch.float64, device="cuda") if "ce" in want else None
    d = torch.empty(nd, dtype=torch.float64, device="cuda") if "diag" in want else None
    _lib.call("vx_product", nx, ny, nz, _ptr(rho, "rho", torch.float64, ne), _ptr(u, "u", torch.float64, nd),
              _lib.dptr(ke), _ptr(mask, "mask", torch.float64, nd), float(emin), float(emax), float(penal),
              _ptr(y, "y", allow_none=True), _ptr(ce, "ce", allow_none=True), _ptr(d, "diag", allow_none=True),
              stream_ptr())
    return y, ce, d


def tc_element_product(shape, ke, E, u, node_mask=None, per_element=False, out=None):
    """The tensor-core element-block operator (an experiment, not used by the solvers): the dense
    24 x 24 element matrix applied 128 elements at a time by tcgen05.mma with TF32 operands and FP32
    accumulation.  E, u: float32 CUDA tensors (Ne, 3N); node_mask: optional uint8 node mask.
    Returns y = K(E) (m . u) over the nodes (3N floats), or with per_element=True the 24 scaled
    element results per element (Ne x 24).  Results carry TF32 rounding (~1e-3 relative)."""
    shape = tuple(int(v) for v in shape)
    ne, nn = n_elems(shape), n_nodes(shape)
    k = np.ascontiguousarray(np.asarray(ke, dtype=np.float64).reshape(576))
    n_out = 24 * ne if per_element else 3 * nn
    y = torch.empty(n_out, dtype=torch.float32, device=u.device) if out is None else out
    _lib.call("vx_tc_element_product", *shape, _lib.dptr(k), _ptr(E, "E", torch.float32, ne),
              _ptr(node_mask, "node_mask", torch.uint8, nn, allow_none=True), _ptr(u, "u", torch.float32, 3 * nn),
              _ptr(y, "y", torch.float32, n_out), int(bool(per_element)), stream_ptr())
    return y.view(ne, 24) if per_element else y
