"""ctypes binding of libcgx.so (include/cgx.h).

The library is the product: there is no Python or CPU fallback.  Importing
this module without the built library raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcgx.so")

OK, EINVAL, EUNSUPPORTED, ENOMEM, ECUDA, EDEVICE = range(6)
FP_EXACT, FP_FMA = 0, 1


class cgx_array(C.Structure):
    _fields_ = [("data", C.c_void_p), ("padext", C.c_int * 3), ("bbox", C.c_int * 9)]


class cgx_pair_box(C.Structure):
    _fields_ = [("dst_comp", C.c_int), ("src_comp", C.c_int), ("dstbox", C.c_int * 9),
                ("srcbox", C.c_int * 9)]


class CgxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cgx error {code}: {msg}")
        self.code = code


if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is not built; run python -m carpet_b200.build")

lib = C.CDLL(LIB_PATH)
lib.cgx_last_error.restype = C.c_char_p
lib.cgx_version.restype = C.c_char_p

_P = C.POINTER
_i9 = C.c_int * 9
_i3 = C.c_int * 3

lib.cgx_transfer.argtypes = [C.c_int, C.c_int, _P(cgx_array), _P(cgx_array), _P(C.c_double),
                             C.c_int, _i9, _i9, C.c_void_p, C.c_double, C.c_int, C.c_int,
                             C.c_void_p]
lib.cgx_copy.argtypes = [C.c_int, C.c_int, _P(cgx_array), _P(cgx_array), _i9, _i9, C.c_void_p,
                         C.c_void_p]
lib.cgx_batch_add.argtypes = [C.c_void_p, C.c_int, C.c_int, _P(cgx_array), _P(cgx_array),
                              _P(C.c_double), C.c_int, _i9, _i9, C.c_void_p, C.c_double,
                              C.c_int, C.c_int]
lib.cgx_batch_create.argtypes = [_P(C.c_void_p)]
for fn in ("cgx_batch_destroy", "cgx_batch_clear"):
    getattr(lib, fn).argtypes = [C.c_void_p]
for fn in ("cgx_batch_upload", "cgx_batch_launch", "cgx_batch_launch_per_box", "cgx_batch_check"):
    getattr(lib, fn).argtypes = [C.c_void_p, C.c_void_p]
lib.cgx_batch_stats.argtypes = [C.c_void_p] + [_P(C.c_int64)] * 4
lib.cgx_batch_kernels.argtypes = [C.c_void_p, _P(C.c_int)]
lib.cgx_batch_autotune.argtypes = [C.c_void_p, C.c_int, C.c_void_p, _P(C.c_int)]
lib.cgx_batch_set_config.argtypes = [C.c_void_p, C.c_int, C.c_int]
lib.cgx_batch_add_many.argtypes = [C.c_void_p, C.c_int, C.c_int, _P(cgx_array), C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_int, _P(C.c_double), C.c_void_p, C.c_void_p,
                                   C.c_double, C.c_int, C.c_int]
_pb = _P(cgx_pair_box)
lib.cgx_sched_sync.argtypes = [C.c_int, C.c_void_p, C.c_void_p, _pb, C.c_int, _P(C.c_int)]
lib.cgx_sched_prolong.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p, C.c_int, C.c_int, C.c_int, _pb, C.c_int, _P(C.c_int)]
lib.cgx_sched_restrict.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                   C.c_int, C.c_int, _pb, C.c_int, _P(C.c_int)]
lib.cgx_sched_old2new.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p, C.c_int, _pb, C.c_int, _P(C.c_int), _pb, C.c_int,
                                  _P(C.c_int)]
lib.cgx_graph_begin.argtypes = [C.c_void_p]
lib.cgx_graph_end.argtypes = [C.c_void_p, _P(C.c_void_p)]
lib.cgx_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
lib.cgx_graph_destroy.argtypes = [C.c_void_p]
lib.cgx_find_source_timelevel.argtypes = [_P(C.c_double), C.c_int, C.c_double, C.c_int, C.c_int,
                                          _P(C.c_int), _P(C.c_int)]
lib.cgx_stream_sync.argtypes = [C.c_void_p]
lib.cgx_batch_set_group.argtypes = [C.c_void_p, C.c_int]
lib.cgx_batch_set_max_ctas.argtypes = [C.c_void_p, C.c_int, C.c_int]
lib.cgx_debug_skip_tma_plane.argtypes = [C.c_int]
lib.cgx_chain_debug_hold.argtypes = [C.c_void_p, C.c_int]
lib.cgx_chain_create.argtypes = [_P(C.c_void_p)]
lib.cgx_chain_destroy.argtypes = [C.c_void_p]
lib.cgx_chain_add.argtypes = [C.c_void_p, C.c_void_p]
for fn in ("cgx_chain_upload", "cgx_chain_launch", "cgx_chain_check"):
    getattr(lib, fn).argtypes = [C.c_void_p, C.c_void_p]
lib.cgx_chain_stats.argtypes = [C.c_void_p] + [_P(C.c_int64)] * 4


def check(rc: int):
    if rc != OK:
        raise CgxError(rc, lib.cgx_last_error().decode())


def box9(b) -> C.Array:
    return _i9(*[int(x) for x in b])


def ints3(v):
    return None if v is None else C.cast(_i3(*[int(x) for x in v]), C.c_void_p)
