"""ctypes bindings for the oracle (TEST INFRASTRUCTURE).

Two libraries sit behind the same calling convention:

* ``port`` -- ``oracle/_build/libcgxoracle.so``, the CPU restatement of
  CarpetLib's grid-transfer operators in ``oracle/cgx_oracle.c``;
* ``ref``  -- ``oracle/_ref/libcarpetref{,_fma}.so``, CarpetLib's own operator
  sources compiled unchanged (``oracle/Makefile``), present only where the
  reference sources were available at build time.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  The product never does.

Arrays are numpy float64 arrays of shape (nz, ny, nx_pad) -- x fastest --
with the logical extent given by their bbox; boxes are int[9]
{lower[3], upper[3], stride[3]}.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "_build", "libcgxoracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libcarpetref.so")
REF_FMA_PATH = os.path.join(HERE, "_ref", "libcarpetref_fma.so")

# operator_type (CarpetLib/src/operators.hh:8-25)
OP_ERROR, OP_NONE, OP_SYNC, OP_RESTRICT, OP_COPY, OP_LAGRANGE, OP_ENO, OP_WENO, OP_TVD, \
    OP_LAGRANGE_MONOTONE = range(10)
# centering (CarpetLib/src/defs.hh:134)
VERTEX, CELL = 1, 2

_i3 = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


class OracleError(RuntimeError):
    pass


def _ints(v) -> C.Array:
    a = (C.c_int * len(v))(*[int(x) for x in v])
    return a


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def padext(a: np.ndarray):
    """padded extent (x, y, z) of an array stored as (nz, ny, nx_pad)"""
    return (a.shape[2], a.shape[1], a.shape[0])


def box_sizes(b: Sequence[int]):
    return tuple(max(0, (b[3 + d] - b[d] + b[6 + d]) // b[6 + d]) for d in range(3))


class Port:
    """The restated oracle (cgx_oracle.c)."""

    def __init__(self, path: str = PORT_PATH):
        if not os.path.exists(path):
            raise OracleError(f"oracle library missing: {path} (run make -C oracle port)")
        self.lib = C.CDLL(path)
        self.lib.cgxo_last_error.restype = C.c_char_p

    def _check(self, rc):
        if rc:
            raise OracleError(self.lib.cgxo_last_error().decode())

    # --- operators with the common operator signature -------------------
    def _op(self, fn, pre, src, srcbbox, dst, dstbbox, srcreg, dstreg, post=()):
        args = list(pre) + [
            _dptr(src), _ints(padext(src)), _ints(box_sizes(srcbbox)),
            _dptr(dst), _ints(padext(dst)), _ints(box_sizes(dstbbox)),
            _ints(srcbbox), _ints(dstbbox), _ints(srcreg), _ints(dstreg),
        ] + list(post)
        self._check(fn(*args))

    def copy_3d(self, src, srcbbox, dst, dstbbox, srcreg, dstreg, slab=None):
        self._op(self.lib.cgxo_copy_3d, (), src, srcbbox, dst, dstbbox, srcreg,
                 dstreg, (None if slab is None else _ints(slab),))

    def prolongate_3d_rf2(self, order, src, srcbbox, dst, dstbbox, reg, fma=False):
        self._op(self.lib.cgxo_prolongate_3d_rf2, (order, int(fma)), src, srcbbox,
                 dst, dstbbox, reg, reg)

    def prolongate_3d_cc_rf2(self, order, src, srcbbox, dst, dstbbox, reg, fma=False):
        self._op(self.lib.cgxo_prolongate_3d_cc_rf2, (order, int(fma)), src,
                 srcbbox, dst, dstbbox, reg, reg)

    def prolongate_3d_cc_eno_rf2(self, order, src, srcbbox, dst, dstbbox, reg, fma=False):
        self._op(self.lib.cgxo_prolongate_3d_cc_eno_rf2, (order, int(fma)), src,
                 srcbbox, dst, dstbbox, reg, reg)

    def prolongate_3d_o5_monotone_rf2(self, src, srcbbox, dst, dstbbox, reg, fma=False):
        self._op(self.lib.cgxo_prolongate_3d_o5_monotone_rf2, (int(fma),), src, srcbbox, dst,
                 dstbbox, reg, reg)

    def prolongate_3d_eno(self, src, srcbbox, dst, dstbbox, reg, fma=False):
        self._op(self.lib.cgxo_prolongate_3d_eno, (int(fma),), src, srcbbox, dst,
                 dstbbox, reg, reg)

    def restrict_3d_rf2(self, src, srcbbox, dst, dstbbox, reg):
        self._op(self.lib.cgxo_restrict_3d_rf2, (), src, srcbbox, dst, dstbbox,
                 reg, reg)

    def restrict_3d_cc_rf2(self, src, srcbbox, dst, dstbbox, reg, fma=False):
        self._op(self.lib.cgxo_restrict_3d_cc_rf2, (int(fma),), src, srcbbox, dst,
                 dstbbox, reg, reg)

    def restrict_3d_cc_ho_rf2(self, order, src, srcbbox, dst, dstbbox, reg, fma=False):
        """restrict_3d_cc_o3_rf2 (order 3) / restrict_3d_cc_o5_rf2 (order 5)"""
        fn = {3: self.lib.cgxo_restrict_3d_cc_o3_rf2, 5: self.lib.cgxo_restrict_3d_cc_o5_rf2}[order]
        self._op(fn, (int(fma),), src, srcbbox, dst, dstbbox, reg, reg)

    def set_restriction(self, use_higher_order: bool, order: int = 1):
        """the use_higher_order_restriction / restriction_order_space parameters"""
        self.lib.cgxo_set_restriction(int(use_higher_order), int(order))

    def _ti(self, fn, srcs, times, srcbbox, dst, dstbbox, reg, t, fma):
        pre = [int(fma)]
        for s, ts in zip(srcs, times):
            pre += [_dptr(s), C.c_double(ts)]
        s0 = srcs[0]
        self._check(fn(*pre, _ints(padext(s0)), _ints(box_sizes(srcbbox)),
                       _dptr(dst), C.c_double(t), _ints(padext(dst)),
                       _ints(box_sizes(dstbbox)), _ints(srcbbox), _ints(dstbbox),
                       _ints(reg), _ints(reg)))

    def interpolate_3d_2tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t, fma=False):
        self._ti(self.lib.cgxo_interpolate_3d_2tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t, fma)

    def interpolate_3d_3tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t, fma=False):
        self._ti(self.lib.cgxo_interpolate_3d_3tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t, fma)

    def interpolate_eno_3d_3tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t, fma=False):
        self._ti(self.lib.cgxo_interpolate_eno_3d_3tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t, fma)

    def interpolate_3d_4tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t, fma=False):
        self._ti(self.lib.cgxo_interpolate_3d_4tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t, fma)

    def interpolate_3d_5tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t, fma=False):
        self._ti(self.lib.cgxo_interpolate_3d_5tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t, fma)

    def find_source_timelevel(self, times, time, order_time, op):
        tl0, ntl = C.c_int(), C.c_int()
        ts = (C.c_double * len(times))(*times)
        self._check(self.lib.cgxo_find_source_timelevel(
            ts, len(times), C.c_double(time), order_time, op, C.byref(tl0),
            C.byref(ntl)))
        return tl0.value, ntl.value

    def time_weights(self, kind, times, t):
        w = (C.c_double * 8)()
        ts = (C.c_double * 5)(*list(times) + [0.0] * (5 - len(times)))
        self._check(self.lib.cgxo_time_weights(kind, ts, C.c_double(t), w))
        return list(w)

    def transfer(self, op, cent, dst, dstbbox, srcs, srcbbox, times, dstbox,
                 srcbox, time, order_space, order_time, slab=None, fma=False):
        """One box-pair of gdata::transfer_data on one process."""
        arr = (_dp * len(srcs))(*[_dptr(s) for s in srcs])
        ts = (C.c_double * len(times))(*times)
        self._check(self.lib.cgxo_transfer(
            int(fma), op, cent, _dptr(dst), _ints(padext(dst)), _ints(dstbbox), arr,
            _ints(padext(srcs[0])), _ints(srcbbox), ts, len(times), _ints(dstbox),
            _ints(srcbox), None if slab is None else _ints(slab), C.c_double(time),
            order_space, order_time))


class Ref:
    """CarpetLib's own operators, compiled unchanged from the reference."""

    def __init__(self, fma: bool = False):
        path = REF_FMA_PATH if fma else REF_PATH
        if not os.path.exists(path):
            raise OracleError(f"reference build missing: {path}")
        # RTLD_LOCAL keeps the two builds' identical C++ symbols apart
        self.lib = C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        self.lib.cgxref_last_error.restype = C.c_char_p

    @staticmethod
    def available(fma: bool = False) -> bool:
        return os.path.exists(REF_FMA_PATH if fma else REF_PATH)

    def set_openmp(self, on: bool):
        self.lib.cgxref_set_openmp(int(on))

    def _check(self, rc):
        if rc:
            raise OracleError(self.lib.cgxref_last_error().decode())

    def _op(self, fn, pre, src, srcbbox, dst, dstbbox, srcreg, dstreg, post=()):
        args = list(pre) + [
            _dptr(src), _ints(padext(src)), _ints(box_sizes(srcbbox)),
            _dptr(dst), _ints(padext(dst)), _ints(box_sizes(dstbbox)),
            _ints(srcbbox), _ints(dstbbox), _ints(srcreg), _ints(dstreg),
        ] + list(post)
        self._check(fn(*args))

    def copy_3d(self, src, srcbbox, dst, dstbbox, srcreg, dstreg, slab=None):
        self._op(self.lib.cgxref_copy_3d, (), src, srcbbox, dst, dstbbox, srcreg,
                 dstreg, (None if slab is None else _ints(slab),))

    def prolongate_3d_rf2(self, order, src, srcbbox, dst, dstbbox, reg):
        self._op(self.lib.cgxref_prolongate_3d_rf2, (order,), src, srcbbox, dst,
                 dstbbox, reg, reg)

    def prolongate_3d_cc_rf2(self, order, src, srcbbox, dst, dstbbox, reg):
        self._op(self.lib.cgxref_prolongate_3d_cc_rf2, (order,), src, srcbbox, dst,
                 dstbbox, reg, reg)

    def prolongate_3d_o5_monotone_rf2(self, src, srcbbox, dst, dstbbox, reg):
        self._op(self.lib.cgxref_prolongate_3d_o5_monotone_rf2, (), src, srcbbox, dst,
                 dstbbox, reg, reg)

    def prolongate_3d_cc_eno_rf2(self, order, src, srcbbox, dst, dstbbox, reg):
        self._op(self.lib.cgxref_prolongate_3d_cc_eno_rf2, (order,), src, srcbbox, dst,
                 dstbbox, reg, reg)

    def restrict_3d_rf2(self, src, srcbbox, dst, dstbbox, reg):
        self._op(self.lib.cgxref_restrict_3d_rf2, (), src, srcbbox, dst, dstbbox,
                 reg, reg)

    def restrict_3d_cc_rf2(self, src, srcbbox, dst, dstbbox, reg):
        self._op(self.lib.cgxref_restrict_3d_cc_rf2, (), src, srcbbox, dst, dstbbox,
                 reg, reg)

    def restrict_3d_cc_ho_rf2(self, order, src, srcbbox, dst, dstbbox, reg):
        fn = {3: self.lib.cgxref_restrict_3d_cc_o3_rf2, 5: self.lib.cgxref_restrict_3d_cc_o5_rf2}[order]
        self._op(fn, (), src, srcbbox, dst, dstbbox, reg, reg)

    def _ti(self, fn, srcs, times, srcbbox, dst, dstbbox, reg, t):
        pre = []
        for s, ts in zip(srcs, times):
            pre += [_dptr(s), C.c_double(ts)]
        s0 = srcs[0]
        self._check(fn(*pre, _ints(padext(s0)), _ints(box_sizes(srcbbox)),
                       _dptr(dst), C.c_double(t), _ints(padext(dst)),
                       _ints(box_sizes(dstbbox)), _ints(srcbbox), _ints(dstbbox),
                       _ints(reg), _ints(reg)))

    def interpolate_3d_2tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t):
        self._ti(self.lib.cgxref_interpolate_3d_2tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t)

    def interpolate_3d_3tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t):
        self._ti(self.lib.cgxref_interpolate_3d_3tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t)

    def interpolate_eno_3d_3tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t):
        self._ti(self.lib.cgxref_interpolate_eno_3d_3tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t)

    def interpolate_3d_4tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t):
        self._ti(self.lib.cgxref_interpolate_3d_4tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t)

    def interpolate_3d_5tl(self, srcs, times, srcbbox, dst, dstbbox, reg, t):
        self._ti(self.lib.cgxref_interpolate_3d_5tl, srcs, times, srcbbox, dst,
                 dstbbox, reg, t)


def alloc(bbox: Sequence[int], pad_x_even: bool = True, fill: Optional[float] = None):
    """An array for a bbox, stored (nz, ny, nx_pad)."""
    nx, ny, nz = box_sizes(bbox)
    px = nx + (nx & 1) if pad_x_even else nx
    a = np.empty((nz, ny, px), dtype=np.float64)
    if fill is not None:
        a.fill(fill)
    return a
