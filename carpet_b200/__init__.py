"""carpet_b200 -- B200-native grid transfers for Carpet-style AMR.

The host-side mirror of CarpetLib's transfer interface (transfer.py) over
the C-ABI library libcgx.so (include/cgx.h, csrc/).  Device memory comes
from torch; the kernels are the library's own sm_100a CUDA.
"""
from .transfer import (CELL, OP_COPY, OP_ENO, OP_LAGRANGE, OP_NONE, OP_RESTRICT, OP_SYNC,
                       VERTEX, Batch, Data, Graph, copy_data, set_fp_mode, transfer_data)

__all__ = ["Data", "transfer_data", "copy_data", "Batch", "Graph", "set_fp_mode",
           "OP_NONE", "OP_SYNC", "OP_RESTRICT", "OP_COPY", "OP_LAGRANGE", "OP_ENO",
           "VERTEX", "CELL"]
