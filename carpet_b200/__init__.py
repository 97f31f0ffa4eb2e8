"""carpet_b200 -- B200-native grid transfers for Carpet-style AMR.

The host-side mirror of CarpetLib's transfer interface (transfer.py) over
the C-ABI library libcgx.so (include/cgx.h, csrc/).  Device memory comes
from torch; the kernels are the library's own sm_100a CUDA.
"""
from .transfer import (CELL, OP_COPY, OP_ENO, OP_LAGRANGE, OP_NONE, OP_RESTRICT, OP_SYNC,
                       OP_WENO, VERTEX, Batch, CgxError, Data, Graph, copy_data, set_fp_mode,
                       set_restriction, transfer_data)

__all__ = ["CgxError", "Data", "transfer_data", "copy_data", "Batch", "Graph", "set_fp_mode",
           "set_restriction", "OP_NONE", "OP_SYNC", "OP_RESTRICT", "OP_COPY", "OP_LAGRANGE", "OP_ENO", "OP_WENO",
           "VERTEX", "CELL"]
