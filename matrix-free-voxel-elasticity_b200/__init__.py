"""voxel_b200 -- matrix-free Hex8 voxel elasticity on NVIDIA B200 (sm_100a).

A drop-in for the matvec / Jacobi-PCG / geometric-multigrid path of the reference
(nejeoui/matrix-free-voxel-elasticity: src/voxel_kernels.py, src/voxel_mg.py): a Python host over
PyTorch CUDA tensors calling hand-written sm_100a kernels in libvoxel_b200.so through a thin
ctypes C ABI (include/voxel_b200.h).  There is no CPU fallback.
"""
from . import _lib
from .element import XYZ, Modal, element, quadrature
from .layout import edof_author, element_nodes, n_elems, n_nodes, to_author, to_natural
from .operators import (Product, VoxelOperator, cast, dofs_from_node_mask, dots, node_mask_from_dofs,
                        product, reduce_partials, simp_modulus)
from . import problems, solver, voxel_mg  # noqa: E402
from .solver import FCGSolver, JacobiPCG, JacobiPreconditioner, MGHierarchy, PCGIR, SolveResult, hierarchy_shapes
from .api import ElasticitySolver, clear_solver_cache, solve
from . import batch, donor, records, serving, simp, slab  # noqa: E402
from .simp import Compliance, ConeFilter, OCUpdater, compliance, oc_top88, run_simp
from .slab import SlabComm, SlabSolver, slab_bounds

__all__ = ["XYZ", "Modal", "element", "quadrature", "edof_author", "element_nodes", "n_elems", "n_nodes",
           "to_author", "to_natural", "Product", "VoxelOperator", "cast", "dofs_from_node_mask", "dots",
           "node_mask_from_dofs", "product", "reduce_partials", "simp_modulus", "problems", "solver", "voxel_mg",
           "FCGSolver", "JacobiPCG", "JacobiPreconditioner", "MGHierarchy", "PCGIR", "SolveResult", "hierarchy_shapes",
           "ElasticitySolver", "clear_solver_cache", "solve", "simp", "Compliance", "ConeFilter", "OCUpdater", "compliance", "oc_top88",
           "run_simp", "batch", "donor", "records", "serving", "slab", "SlabComm", "SlabSolver", "slab_bounds"]
