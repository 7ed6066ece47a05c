"""``import bmmpy`` for code written against the reference's Python package.

Put ``bmmpy_b200/compat`` on ``sys.path`` (or PYTHONPATH) and ``import bmmpy``
gives the B200 build under the reference's module name: the same public
classes and functions (bmmpy_b200's Python surface, which mirrors
bmmpy/__init__.py), the submodules ``bmmpy.ga``, ``bmmpy.search``,
``bmmpy.solver``, ``bmmpy.apply``, ``bmmpy.matrix``, ``bmmpy.workflows``,
``bmmpy.candidate``, and ``bmmpy._bmmpy``, the native module (pybind11 over
include/bmmpy/).  Every search runs on the GPU.
"""

from __future__ import annotations

import importlib
import sys

import bmmpy_b200 as _impl
from bmmpy_b200 import *  # noqa: F401,F403
from bmmpy_b200 import __all__ as _impl_all

for _name in ("ga", "search", "solver", "apply", "matrix", "workflows", "candidate"):
    _mod = importlib.import_module(f"bmmpy_b200.{_name}")
    sys.modules[f"{__name__}.{_name}"] = _mod
    globals()[_name] = _mod
try:
    from bmmpy_b200 import _bmmpy  # noqa: F401

    sys.modules[f"{__name__}._bmmpy"] = _bmmpy
except ImportError:  # the native module is built by python -m bmmpy_b200.build
    pass

__all__ = list(_impl_all)
__version__ = getattr(_impl, "__version__", None)
