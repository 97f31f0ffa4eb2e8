"""Host-side mirror of CarpetLib's transfer interface.

``Data`` stands for ``data<T>`` (CarpetLib/src/data.hh): the storage of one
grid-function component at one timelevel, with its extent (a bbox) and
padded shape, resident in device memory.  ``transfer_data`` and
``copy_data`` take the arguments of ``gdata::transfer_data`` /
``gdata::copy_data`` (CarpetLib/src/gdata.hh:182-191) for one process and
call the C-ABI; errors that abort in CarpetLib raise ``CgxError`` here.

``Batch`` collects many box-pairs (the ``sendrecv_pseudoregion`` walk of
``ggf::transfer_from_all``, CarpetLib/src/ggf.cc:500-591) and runs them in
one persistent kernel; ``Graph`` captures launches into a CUDA graph.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import CgxError, box9, check, cgx_array, ints3, lib

# operator_type (CarpetLib/src/operators.hh:8-25), centering (defs.hh:134)
OP_ERROR, OP_NONE, OP_SYNC, OP_RESTRICT, OP_COPY, OP_LAGRANGE, OP_ENO, OP_WENO, OP_TVD, \
    OP_LAGRANGE_MONOTONE = range(10)
VERTEX, CELL = 1, 2


def set_fp_mode(fma: bool):
    check(lib.cgx_set_fp_mode(_lib.FP_FMA if fma else _lib.FP_EXACT))


def set_restriction(use_higher_order: bool, order: int = 1):
    """CarpetLib's use_higher_order_restriction / restriction_order_space
    (CarpetLib/param.ccl, data.cc:1061-1097): cell-centred restriction then
    uses the third- or fifth-order stencil; takes effect for transfers built
    afterwards"""
    check(lib.cgx_set_restriction(int(bool(use_higher_order)), int(order)))


def box_sizes(b: Sequence[int]):
    return tuple(max(0, (b[3 + d] - b[d] + b[6 + d]) // b[6 + d]) for d in range(3))


class Data:
    """One component at one timelevel: a device array over ``extent``.

    Stored as a float64 tensor of shape (padext_z, padext_y, padext_x); the x
    extent is padded to an even number of elements so that every row starts
    on a 16-byte boundary."""

    def __init__(self, extent: Sequence[int], tensor: Optional[torch.Tensor] = None,
                 device: str = "cuda"):
        self.extent = [int(x) for x in extent]
        nx, ny, nz = box_sizes(self.extent)
        if tensor is None:
            tensor = torch.empty((nz, ny, nx + (nx & 1)), dtype=torch.float64, device=device)
        if tensor.dtype != torch.float64 or not tensor.is_contiguous() or tensor.dim() != 3:
            raise ValueError("Data needs a contiguous 3-d float64 tensor")
        pz, py, px = tensor.shape
        if px < nx or py < ny or pz < nz:
            raise ValueError("tensor smaller than the extent")
        self.tensor = tensor

    @property
    def padext(self):
        pz, py, px = self.tensor.shape
        return (px, py, pz)

    def cgx(self) -> cgx_array:
        a = cgx_array()
        a.data = self.tensor.data_ptr()
        a.padext[:] = self.padext
        a.bbox[:] = self.extent
        return a


def _stream(stream):
    if stream is None:
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, torch.cuda.Stream):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(stream)


def _arrays(srcs):
    arr = (cgx_array * len(srcs))()
    for i, s in enumerate(srcs):
        arr[i] = s.cgx()
    return arr


def transfer_data(dst: Data, srcs: Sequence[Data], times: Sequence[float], dstbox, srcbox,
                  time: float, order_space: int, order_time: int, op: int = OP_LAGRANGE,
                  cent: int = VERTEX, slab_offset=None, stream=None):
    """gdata::transfer_data for one box-pair on one process
    (CarpetLib/src/gdata.cc:124-286): timelevel selection, spatial operator
    per timelevel and time interpolation, fused in one launch."""
    d = dst.cgx()
    arr = _arrays(srcs)
    ts = (C.c_double * len(times))(*times)
    check(lib.cgx_transfer(op, cent, C.byref(d), arr, ts, len(srcs), box9(dstbox), box9(srcbox),
                           ints3(slab_offset), float(time), int(order_space), int(order_time),
                           _stream(stream)))


def copy_data(dst: Data, src: Data, dstbox, srcbox, op: int = OP_LAGRANGE, cent: int = VERTEX,
              slab_offset=None, stream=None):
    """gdata::copy_data (CarpetLib/src/gdata.cc:110-122)."""
    d, s = dst.cgx(), src.cgx()
    check(lib.cgx_copy(op, cent, C.byref(d), C.byref(s), box9(dstbox), box9(srcbox),
                       ints3(slab_offset), _stream(stream)))


def find_source_timelevel(times, time, order_time, op):
    tl0, ntl = C.c_int(), C.c_int()
    ts = (C.c_double * len(times))(*times)
    check(lib.cgx_find_source_timelevel(ts, len(times), float(time), int(order_time), int(op),
                                        C.byref(tl0), C.byref(ntl)))
    return tl0.value, ntl.value


class Batch:
    """Many box-pairs run by one persistent kernel."""

    def __init__(self):
        h = C.c_void_p()
        check(lib.cgx_batch_create(C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:
            lib.cgx_batch_destroy(self.h)
            self.h = None

    def clear(self):
        check(lib.cgx_batch_clear(self.h))

    def add(self, dst: Data, srcs: Sequence[Data], times, dstbox, srcbox, time, order_space,
            order_time, op=OP_LAGRANGE, cent=VERTEX, slab_offset=None):
        d = dst.cgx()
        arr = _arrays(srcs)
        ts = (C.c_double * len(times))(*times)
        check(lib.cgx_batch_add(self.h, op, cent, C.byref(d), arr, ts, len(srcs), box9(dstbox),
                                box9(srcbox), ints3(slab_offset), float(time), int(order_space),
                                int(order_time)))

    def add_many(self, pairs, times, time, order_space, order_time, op=OP_LAGRANGE, cent=VERTEX):
        """add a list of (dst Data, [src Data per timelevel], dstbox, srcbox)
        in one library call (cgx_batch_add_many)"""
        if not pairs:
            return
        index, arrays = {}, []

        def idx(d: Data):
            k = id(d)
            if k not in index:
                index[k] = len(arrays)
                arrays.append(d)
            return index[k]
        nsrc = len(pairs[0][1])
        di = np.array([idx(p[0]) for p in pairs], dtype=np.int32)
        si = np.array([[idx(s) for s in p[1]] for p in pairs], dtype=np.int32).reshape(-1)
        db = np.array([p[2] for p in pairs], dtype=np.int32).reshape(-1)
        sb = np.array([p[3] for p in pairs], dtype=np.int32).reshape(-1)
        arr = (cgx_array * len(arrays))(*[a.cgx() for a in arrays])
        ts = (C.c_double * len(times))(*times)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        check(lib.cgx_batch_add_many(self.h, op, cent, arr, len(pairs), vp(di), vp(si), nsrc, ts, vp(db),
                                     vp(sb), float(time), int(order_space), int(order_time)))

    def set_max_ctas(self, tma_per_sm: int = 0, stream_per_sm: int = 0):
        """CTAs per SM of the batch's TMA prolongation and streaming kernels
        (0: as many as fit); room for another stream's kernel on every SM"""
        check(lib.cgx_batch_set_max_ctas(self.h, int(tma_per_sm), int(stream_per_sm)))

    def set_group(self, group: int):
        """pairs added from now on belong to dependency group ``group``
        (cgx_batch_set_group; used by Chain)"""
        check(lib.cgx_batch_set_group(self.h, int(group)))

    def add_raw(self, op, cent, dst: cgx_array, srcs_arr, ts, nsrc, dstbox, srcbox, time,
                order_space, order_time):
        """add() for callers that already hold cgx_array structs"""
        check(lib.cgx_batch_add(self.h, op, cent, C.byref(dst), srcs_arr, ts, nsrc, dstbox,
                                srcbox, None, float(time), int(order_space), int(order_time)))

    def stats(self):
        v = [C.c_int64() for _ in range(4)]
        check(lib.cgx_batch_stats(self.h, *[C.byref(x) for x in v]))
        return dict(pairs=v[0].value, tiles=v[1].value, points=v[2].value, bytes=v[3].value)

    def autotune(self, reps: int = 3, stream=None):
        """pick the fastest tile configuration of every prolongation variant
        in the batch (runs the batch; leaves it uploaded); returns
        {variant: configuration}"""
        out = (C.c_int * 40)()
        check(lib.cgx_batch_autotune(self.h, reps, _stream(stream), out))
        return {v: out[v] for v in range(40) if out[v] >= 0}

    def set_config(self, config: int, variant: int = -1):
        """pin the tile configuration of one prolongation variant (all: -1);
        takes effect at the next upload()"""
        check(lib.cgx_batch_set_config(self.h, variant, config))

    def kernels(self) -> int:
        """kernels one launch() issues for the current upload"""
        n = C.c_int()
        check(lib.cgx_batch_kernels(self.h, C.byref(n)))
        return n.value

    def upload(self, stream=None):
        check(lib.cgx_batch_upload(self.h, _stream(stream)))

    def launch(self, stream=None):
        check(lib.cgx_batch_launch(self.h, _stream(stream)))

    def launch_per_box(self, stream=None):
        check(lib.cgx_batch_launch_per_box(self.h, _stream(stream)))

    def check(self, stream=None):
        check(lib.cgx_batch_check(self.h, _stream(stream)))


class Chain:
    """A sequence of batches run as one persistent launch (cgx_chain_*):
    each dependency group (Batch.set_group) sees the batches in order, the
    groups' tiles share the GPU.  The batches must outlive the chain."""

    def __init__(self, batches=()):
        h = C.c_void_p()
        check(lib.cgx_chain_create(C.byref(h)))
        self.h = h
        self.batches = []
        for b in batches:
            self.add(b)

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:
            lib.cgx_chain_destroy(self.h)
            self.h = None

    def add(self, b: Batch):
        check(lib.cgx_chain_add(self.h, b.h))
        self.batches.append(b)

    def upload(self, stream=None):
        check(lib.cgx_chain_upload(self.h, _stream(stream)))

    def launch(self, stream=None):
        check(lib.cgx_chain_launch(self.h, _stream(stream)))

    def check(self, stream=None):
        check(lib.cgx_chain_check(self.h, _stream(stream)))

    def stats(self):
        v = [C.c_int64() for _ in range(4)]
        check(lib.cgx_chain_stats(self.h, *[C.byref(x) for x in v]))
        return dict(pairs=v[0].value, tiles=v[1].value, points=v[2].value, bytes=v[3].value)


class Graph:
    """CUDA graph of the calls made inside ``with g.capture(stream):``."""

    def __init__(self):
        self.h = None

    class _Cap:
        def __init__(self, g, stream):
            self.g, self.s = g, stream

        def __enter__(self):
            check(lib.cgx_graph_begin(self.s))

        def __exit__(self, et, ev, tb):
            h = C.c_void_p()
            rc = lib.cgx_graph_end(self.s, C.byref(h))
            if et is None:
                check(rc)
                self.g.h = h

    def capture(self, stream):
        return Graph._Cap(self, _stream(stream))

    def launch(self, stream=None):
        check(lib.cgx_graph_launch(self.h, _stream(stream)))

    def __del__(self):
        if getattr(self, "h", None) and lib is not None:
            lib.cgx_graph_destroy(self.h)
            self.h = None
