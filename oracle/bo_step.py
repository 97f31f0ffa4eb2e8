"""One coarse Berger-Oliger step of grid transfers on the host through
CarpetLib's own operators (TEST INFRASTRUCTURE: the CPU baseline and the
reference arm of bench.py; the product never imports it).

The hierarchy's grid functions live in numpy arrays (one per level x
timelevel x grid function x component, x padded to even as on the device).
A step replays the phases of ``carpet_b200.bo.step_phases`` -- the call
order of Carpet/src/Evolve.cc:44-121 -- and runs every phase's box-pairs,
one grid function after the other, through ``cgxref_transfer_pairs``
(oracle/ref_api.cc): CarpetLib's data<T>::transfer_time path with its
per-call temporaries, compiled from the reference sources (oracle/_ref).

Nothing here loads libcgx.so: the hierarchy comes from
``carpet_b200.hierarchy.nested(..., native=False)``.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List

import numpy as np

from carpet_b200.bo import phase_pairs, step_totals

from .binding import REF_PATH, OracleError, alloc, padext

HERE = os.path.dirname(os.path.abspath(__file__))
REF_FAST_PATH = os.path.join(HERE, "_ref", "libcarpetref_fast.so")

KIND = {"sync": 0, "prolong": 1, "restrict": 2}


class cgxref_arr(C.Structure):
    _fields_ = [("data", C.c_void_p), ("padext", C.c_int * 3), ("bbox", C.c_int * 9)]


def host_supports_fast() -> bool:
    """the fast build needs AVX2 and FMA (x86-64-v3)"""
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return False
    return " avx2" in flags and " fma" in flags and " bmi2" in flags


def builds():
    """(name, path) of the reference builds present on this host"""
    out = []
    if os.path.exists(REF_PATH):
        out.append(("O2, no contraction (canonical order)", REF_PATH))
    if os.path.exists(REF_FAST_PATH) and host_supports_fast():
        out.append(("O3 -march=x86-64-v3, FMA contraction", REF_FAST_PATH))
    return out


class RefStep:
    """Host storage of ``ngf`` grid functions x ``ntl`` timelevels of a
    nested hierarchy and the transfer phases of a coarse step over it."""

    def __init__(self, h, ngf: int, ntl: int = 3, path: str = REF_PATH, order: int = 5,
                 seed: int = 7, threads: bool = True):
        if not os.path.exists(path):
            raise OracleError(f"reference build missing: {path}")
        self.lib = C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        self.lib.cgxref_last_error.restype = C.c_char_p
        self.lib.cgxref_set_openmp(int(threads))
        self.h, self.ngf, self.ntl, self.order = h, ngf, ntl, order
        rng = np.random.default_rng(seed)
        # arrays[l][pool][g][c]
        self.arrays: List = []
        for lev in h.levels:
            pools = []
            for _ in range(ntl):
                gfs = []
                for _ in range(ngf):
                    comps = []
                    for comp in lev.comps:
                        a = alloc(comp.exterior)
                        a[...] = rng.standard_normal(a.shape)
                        comps.append(a)
                    gfs.append(comps)
                pools.append(gfs)
            self.arrays.append(pools)
        self._calls = {}

    def _arr(self, a, bbox) -> cgxref_arr:
        x = cgxref_arr()
        x.data = a.ctypes.data
        x.padext[:] = padext(a)
        x.bbox[:] = [int(v) for v in bbox]
        return x

    def _build(self, key):
        """per grid function: the marshalled pair list of one phase"""
        from carpet_b200 import bo
        kind, l, rots, ntl = key
        h, T = self.h, self.ntl
        pairs, dl, sl = phase_pairs(h, key)
        dpool = bo.pool_index(rots[0], 0, T)
        if kind == "sync":
            spools = [dpool]
            times, time = [0.0], 0.0
        elif kind == "prolong":
            spools = [bo.pool_index(rots[1], t, T) for t in range(ntl)]
            times, time = bo.prolong_times(ntl)
        else:
            spools = [bo.pool_index(rots[1], 0, T)]
            times, time = [0.0], 0.0
        dcomps, scomps = h.levels[dl].comps, h.levels[sl].comps
        n = len(pairs)
        dboxes = np.array([p.dstbox for p in pairs], dtype=np.int32).reshape(n, 9)
        sboxes = np.array([p.srcbox for p in pairs], dtype=np.int32).reshape(n, 9)
        calls = []
        for g in range(self.ngf):
            dst = (cgxref_arr * n)(*[self._arr(self.arrays[dl][dpool][g][p.dst_comp],
                                               dcomps[p.dst_comp].exterior) for p in pairs])
            src = (cgxref_arr * (n * ntl))(*[self._arr(self.arrays[sl][sp][g][p.src_comp],
                                                       scomps[p.src_comp].exterior)
                                             for p in pairs for sp in spools])
            calls.append((dst, src))
        ts = (C.c_double * 3)(*(list(times) + [0.0] * (3 - len(times))))
        nbytes, _ = step_totals(h, [key], self.order)
        return (KIND[kind], n, ntl, dboxes, sboxes, ts, time, calls, nbytes)

    def run_phase(self, key, ngf=None) -> int:
        """runs one phase for the first ``ngf`` grid functions; returns the
        algorithmic bytes moved"""
        if key not in self._calls:
            self._calls[key] = self._build(key)
        kind, n, ntl, dboxes, sboxes, ts, time, calls, nbytes = self._calls[key]
        ng = self.ngf if ngf is None else ngf
        for dst, src in calls[:ng]:
            rc = self.lib.cgxref_transfer_pairs(
                kind, self.order, n, dst, src, ntl, dboxes.ctypes.data_as(C.c_void_p),
                sboxes.ctypes.data_as(C.c_void_p), ts, C.c_double(time))
            if rc:
                raise OracleError(self.lib.cgxref_last_error().decode())
        return nbytes * ng

    def run(self, keys, ngf=None) -> int:
        return sum(self.run_phase(k, ngf) for k in keys)
