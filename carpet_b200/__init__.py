"""carpet_b200 -- B200-native grid transfers for Carpet-style AMR.

The host-side mirror of CarpetLib's transfer interface (transfer.py) over
the C-ABI library libcgx.so (include/cgx.h, csrc/).  Device memory comes
from torch; the kernels are the library's own sm_100a CUDA.

The library is loaded on first use of a name that needs it (module
``__getattr__``), not on import of the package: the pure-Python modules
(``hierarchy`` with ``native=False``, ``bo``) run without libcgx.so, which
keeps the library out of processes that only need the box algebra.
"""
from __future__ import annotations

import importlib

_TRANSFER_NAMES = ("CELL", "OP_COPY", "OP_ENO", "OP_LAGRANGE", "OP_NONE", "OP_RESTRICT", "OP_SYNC",
                   "OP_WENO", "VERTEX", "Batch", "Chain", "CgxError", "Data", "Graph", "copy_data",
                   "set_fp_mode", "set_restriction", "transfer_data")

__all__ = list(_TRANSFER_NAMES)


def __getattr__(name):
    if name in _TRANSFER_NAMES:
        mod = importlib.import_module(".transfer", __name__)
        value = getattr(mod, name)
        globals()[name] = value
        return value
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
