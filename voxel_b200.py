"""Import shim: `import voxel_b200` loads the package kept in ./matrix-free-voxel-elasticity_b200/
(a directory name that is not a Python identifier) and replaces this module with it."""
import importlib.util as _ilu
import sys as _sys
from pathlib import Path as _Path

_PKG = _Path(__file__).resolve().parent / "matrix-free-voxel-elasticity_b200"
_spec = _ilu.spec_from_file_location("voxel_b200", _PKG / "__init__.py", submodule_search_locations=[str(_PKG)])
_mod = _ilu.module_from_spec(_spec)
_sys.modules["voxel_b200"] = _mod
_spec.loader.exec_module(_mod)
