"""ctypes binding of libvoxel_b200.so (the C ABI declared in include/voxel_b200.h).

There is no fallback: if the library is missing or a call fails, an exception is raised.
Status codes map to Python exceptions in the reference's style: invalid shapes/arguments and
elements outside the parity-block model raise ValueError (as the reference's Modal does,
code/hex_modal/modal.py:65-66), CUDA failures raise RuntimeError.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_int64, c_void_p, c_char_p, c_uint8
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libvoxel_b200.so"

VX_OK, VX_ERR_INVALID_ARGUMENT, VX_ERR_NULL_POINTER, VX_ERR_ALIGNMENT = 0, 1, 2, 3
VX_ERR_LAUNCH, VX_ERR_UNSUPPORTED, VX_ERR_TIMEOUT, VX_ERR_CUDA = 4, 5, 6, 7
VX_F64, VX_F32, VX_BF16_F32, VX_F32_BF16AUX = 0, 1, 2, 3

_P = c_void_p          # device or host pointer
_D = POINTER(c_double)  # host double array

# name -> (restype, argtypes); every entry point of include/voxel_b200.h
SIGNATURES = {
    "vx_last_error": (c_char_p, []),
    "vx_version": (c_int, []),
    "vx_element_matrix": (c_int, [c_double, c_double, c_double, c_double, _D]),
    "vx_element": (c_int, [c_double, c_double, _D]),
    "vx_parity_blocks": (c_int, [_D, _D, _D]),
    "vx_modal8": (c_int, [_D, _P, _P, _P, c_int, c_int, c_int, _P]),
    "vx_matvec": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, _P, _P, _P]),
    "vx_matvec_dense": (c_int, [c_int, c_int, c_int, c_int, _P, _P, _P, _P, _P]),
    "vx_diagonal": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, c_int, _P, _P]),
    "vx_element_energy": (c_int, [c_int, c_int, c_int, _D, _P, _P, _P, c_double, c_double, c_double, _P, _P]),
    "vx_product": (c_int, [c_int, c_int, c_int, _P, _P, _D, _P, c_double, c_double, c_double, _P, _P, _P, _P]),
    "vx_simp_modulus": (c_int, [c_int, c_int64, _P, c_double, c_double, c_double, _P, _P]),
    "vx_jacobi_sweep": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, _P, _P, _P, c_double, _P, _P]),
    "vx_residual": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, _P, _P, _P, _P]),
    "vx_operator_partials": (c_int64, [c_int, c_int, c_int, c_int]),
    "vx_apply_dot": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, _P, _P, _P, _P]),
    "vx_true_residual": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, _P, _P, _P, _P, _P]),
    "vx_restrict": (c_int, [c_int, c_int, c_int, c_int, _P, _P, _P, _P]),
    "vx_prolong_add": (c_int, [c_int, c_int, c_int, c_int, _P, _P, _P, _P]),
    "vx_coarsen_modulus": (c_int, [c_int, c_int, c_int, c_int, _P, _P, _P]),
    "vx_coarsen_mask": (c_int, [c_int, c_int, c_int, _P, _P, _P]),
    "vx_assemble_dense": (c_int, [c_int, c_int, c_int, _D, _P, _P, _P, _P]),
    "vx_coarse_apply": (c_int, [c_int, c_int, _P, _P, _P, _P, _P]),
    "vx_mask_from_dofs": (c_int, [c_int64, _P, _P, _P]),
    "vx_partials_size": (c_int64, [c_int64]),
    "vx_dots": (c_int, [c_int, c_int64, c_int, POINTER(c_void_p), POINTER(c_void_p), _P, _P, _P]),
    "vx_reduce_partials": (c_int, [c_int64, c_int, _P, _P, _P]),
    "vx_apply_dot_planes": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, _P, _P, _P, c_int, c_int, _P]),
    "vx_true_residual_planes": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, _P, _P, _P, _P, c_int, c_int, _P]),
    "vx_true_residual_noalloc": (c_int, [c_int, c_int, c_int, c_int, _D, _P, _P, _P, _P, _P, _P, _P]),
    "vx_device_status": (c_int, [POINTER(c_int), c_int]),
    "vx_set_stream_kernel": (c_int, [c_int]),
    "vx_tc_element_product": (c_int, [c_int, c_int, c_int, _D, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                      c_void_p]),
    "vx_tc_status": (c_int, [POINTER(c_int), c_int]),
    "vx_coarse_factor_workspace": (c_int64, [c_int, c_int]),
    "vx_coarse_factor": (c_int, [c_int, c_int, _P, _P, _P, _P, _P]),
    "vx_batch_coarse_factor": (c_int, [c_int, c_int, c_int, POINTER(c_int), _P, _P, _P, _P, _P]),
    "vx_coarse_pack_factor": (c_int, [c_int, c_int, _P, _P, _P, _P]),
    # batches of independent systems
    "vx_batch_finalize": (c_int, [c_int, c_int64, c_int, _P, c_int64, _P, _P]),
    "vx_batch_cg_update": (c_int, [c_int, c_int64, c_int, c_int64, _P, _P, _P, _P, _P, c_int, _P]),
    "vx_batch_cg_direction": (c_int, [c_int, c_int64, c_int, c_int64, _P, _P, _P, _P, _P]),
    "vx_batch_dots_pr": (c_int, [c_int, c_int64, c_int, c_int64, _P, _P, _P, _P, _P]),
    "vx_batch_coarse_apply_factor": (c_int, [c_int, c_int, c_int, c_int64, _P, _P, _P, _P, _P, _P]),
    "vx_batch_graph_while_end": (c_int, [_P, _P, c_int, _P]),
    "vx_axpby": (c_int, [c_int, c_int64, c_double, _P, c_double, _P, _P]),
    "vx_cast": (c_int, [c_int64, c_int, _P, c_int, _P, c_double, _P]),
    # solver kernels with device-resident scalars and WHILE graphs
    "vx_solver_slots": (c_int, []),
    "vx_solver_partials": (c_int64, [c_int64]),
    "vx_solver_finalize": (c_int, [c_int, c_int64, _P, _P, _P]),
    "vx_cg_update": (c_int, [c_int, c_int64, _P, _P, _P, _P, _P, c_int, _P]),
    "vx_cg_direction": (c_int, [c_int, c_int, c_int64, _P, _P, _P, _P, _P]),
    "vx_dots_pr": (c_int, [c_int, c_int, c_int64, _P, _P, _P, _P, _P]),
    "vx_jacobi_precond_dot": (c_int, [c_int, c_int64, _P, _P, _P, _P, _P]),
    "vx_vcycle_entry": (c_int, [c_int, c_int64, _P, _P, _P, c_double, _P, _P]),
    "vx_coarse_pack": (c_int, [c_int, _P, _P, _P]),
    "vx_cg_direction_update": (c_int, [c_int, c_int64, _P, _P, _P, _P, _P, _P]),
    "vx_coarse_apply_factor": (c_int, [c_int, c_int, _P, _P, _P, _P, _P, _P]),
    "vx_vcycle_entry_update": (c_int, [c_int, c_int64, _P, _P, _P, _P, _P, c_double, _P, _P]),
    "vx_scaled_product": (c_int, [c_int, c_int64, c_double, _P, _P, _P, _P]),
    "vx_set_scalars": (c_int, [_P, c_int, c_int, c_double, _P]),
    "vx_graph_while_begin": (c_int, [_P, ctypes.POINTER(c_void_p)]),
    "vx_graph_while_end": (c_int, [_P, _P, _P]),
    "vx_graph_launch": (c_int, [_P, _P]),
    "vx_graph_destroy": (c_int, [_P]),
    "vx_capture_status": (c_int, [_P]),
    "vx_graph_body_nodes": (c_int64, [_P]),
    # SIMP
    "vx_cone_filter": (c_int, [c_int, c_int, c_int, c_double, _P, _P, c_int, _P, _P]),
    "vx_oc_partials": (c_int64, [c_int64]),
    "vx_oc_probe": (c_int, [c_int64, _P, _P, _P, _P, c_double, _P, _P, _P]),
    "vx_oc_finalize": (c_int, [c_int64, _P, _P, _P]),
    "vx_oc_apply": (c_int, [c_int64, _P, _P, _P, c_double, _P, _P, _P]),
    # x-slab decomposition
    "vx_layer_partial": (c_int, [c_int, c_int, c_int, _D, _P, _P, _P, c_int, _P, _P]),
    "vx_plane_fix": (c_int, [c_int, c_int, c_int64, _P, _P, _P, _P, _P, _P, c_double, c_double, _P, _P, c_int, _P]),
    "vx_plane_fix_partials": (c_int64, [c_int64]),
    "vx_plane_sum": (c_int, [c_int, c_int64, _P, _P, _P, _P]),
}

_lib = None


def load():
    """Load the library (once) and bind every signature; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"libvoxel_b200.so not found at {LIB_PATH}; build it with "
                           "`python -c 'import __graft_entry__ as g; g.build()'` (needs nvcc)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    _lib = lib
    return lib


def last_error() -> str:
    return load().vx_last_error().decode(errors="replace")


def check(status: int, what: str = "") -> None:
    if status == VX_OK:
        return
    msg = f"{what}: {last_error()}" if what else last_error()
    if status in (VX_ERR_INVALID_ARGUMENT, VX_ERR_UNSUPPORTED, VX_ERR_NULL_POINTER, VX_ERR_ALIGNMENT):
        raise ValueError(msg)
    if status == VX_ERR_TIMEOUT:
        raise TimeoutError(msg)
    raise RuntimeError(msg)


# While a WHILE-graph body is being captured this holds the capture stream: every call then checks
# that the capture is still valid, so the first operation that invalidates it is named.
CAPTURE_STREAM = None

# Kernel launches issued by each entry point (entry points not listed launch none or one:
# host-only entry points are in HOST_ONLY).  Used to count this library's launches.
KERNELS_PER_CALL = {"vx_tc_element_product": 1, "vx_coarse_pack_factor": 3, "vx_dots": 2, "vx_assemble_dense": 1, "vx_true_residual_noalloc": 2, "vx_coarse_apply_factor": 2,
                    "vx_batch_coarse_apply_factor": 2}
HOST_ONLY = {"vx_last_error", "vx_version", "vx_element_matrix", "vx_element", "vx_parity_blocks",
             "vx_operator_partials", "vx_partials_size", "vx_solver_slots", "vx_solver_partials",
             "vx_graph_while_begin", "vx_graph_destroy", "vx_capture_status", "vx_graph_launch",
             "vx_oc_partials", "vx_graph_body_nodes", "vx_plane_fix_partials", "vx_device_status",
             "vx_coarse_factor_workspace", "vx_set_stream_kernel",
             "vx_tc_status"}
launches = 0          # kernels launched directly (graph launches are counted by the solvers)


_FNS = {}             # name -> bound entry point (getattr on a CDLL is not free)


def call(name: str, *args) -> None:
    global launches
    fn = _FNS.get(name)
    if fn is None:
        fn = _FNS[name] = getattr(load(), name)
    check(fn(*args), name)
    if name in ("vx_coarse_factor", "vx_batch_coarse_factor"):   # load, a factor and an update per block, inverse
        launches += 2 * ((int(args[0]) + 63) // 64) + 1
    elif name not in HOST_ONLY:
        launches += KERNELS_PER_CALL.get(name, 1)
    if CAPTURE_STREAM is not None and _lib.vx_capture_status(CAPTURE_STREAM) == 2:
        raise RuntimeError(f"{name} invalidated the stream capture")


def device_status(clear: bool = True) -> int:
    """The streaming kernels' fault flag (0 unless a bounded device wait ran out); waits for the device."""
    v = c_int(0)
    check(load().vx_device_status(ctypes.byref(v), int(bool(clear))), "vx_device_status")
    return int(v.value)


STREAM_KERNELS = {"xp": 0, "zp": 1}


def set_stream_kernel(kind: str) -> str:
    """Select the streaming operator kernel for FP64 / FP32 iterates ("xp" or "zp"); returns
    the previous selection.  Operators size their partial sums at each call, so a change takes
    effect at the next launch; captured graphs keep the kernel they were captured with."""
    prev = int(load().vx_set_stream_kernel(STREAM_KERNELS[kind]))
    if prev < 0:
        raise ValueError(kind)
    return {v: k for k, v in STREAM_KERNELS.items()}[prev]


def dptr(a) -> _D:
    """Host double* of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(_D)
