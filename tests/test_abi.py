"""The C-ABI library on the CPU: it loads, exports every entry point that
include/cgx.h declares, and its host-side argument checks reject what
CarpetLib rejects -- before any device work, so no GPU is needed."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cgx.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(cgx_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    from carpet_b200 import _lib
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(_lib.lib, n), n


def test_version_string():
    from carpet_b200._lib import lib
    assert b"sm_100a" in lib.cgx_version()


def test_find_source_timelevel_matches_oracle(port):
    from carpet_b200.transfer import find_source_timelevel
    from carpet_b200._lib import CgxError
    from oracle.binding import OracleError
    rng = np.random.default_rng(3)
    for it in range(300):
        n = int(rng.integers(1, 4))
        t0, dt = float(rng.uniform(-1, 1)), float(rng.choice([0.5, 0.25, 1e-3]))
        times = [t0 - i * dt for i in range(n)]
        pick = rng.random()
        if pick < 0.3:
            time = times[int(rng.integers(0, n))]
        elif pick < 0.9:
            time = float(rng.uniform(times[-1], times[0]))
        else:
            time = times[0] + dt
        ot = int(rng.integers(0, 3))
        op = int(rng.choice([4, 5, 6]))
        try:
            want = port.find_source_timelevel(times, time, ot, op)
        except OracleError:
            want = None
        try:
            got = find_source_timelevel(times, time, ot, op)
        except CgxError:
            got = None
        assert got == want, (times, time, ot, op)


def _arr(bbox):
    from carpet_b200._lib import cgx_array
    a = cgx_array()
    a.data = 0x1000  # never dereferenced: every call below fails validation
    sz = [max(0, (bbox[3 + d] - bbox[d] + bbox[6 + d]) // bbox[6 + d]) for d in range(3)]
    a.padext[:] = [sz[0] + (sz[0] & 1), sz[1], sz[2]]
    a.bbox[:] = bbox
    return a


@pytest.mark.parametrize("case", ["stride", "outside", "extrapolate", "sync_prolong",
                                  "order", "stencil", "empty", "cc_eno"])
def test_host_checks_reject_bad_calls(case):
    from carpet_b200._lib import lib, box9, cgx_array, EINVAL, EUNSUPPORTED
    fine = [0, 0, 0, 20, 20, 20, 1, 1, 1]
    coarse = [-8, -8, -8, 28, 28, 28, 2, 2, 2]
    reg = [4, 4, 4, 9, 9, 9, 1, 1, 1]
    op, cent, order, times, time, ot = 5, 1, 5, [0.0], 0.0, 0
    if case == "stride":
        coarse = [-9, -9, -9, 27, 27, 27, 3, 3, 3]
    elif case == "outside":
        reg = [15, 15, 15, 25, 25, 25, 1, 1, 1]
    elif case == "extrapolate":
        times, time, ot = [1.0, 0.5, 0.0], 2.0, 2
    elif case == "sync_prolong":
        op = 2
    elif case == "order":
        order = 4
    elif case == "stencil":
        coarse = [2, 2, 2, 22, 22, 22, 2, 2, 2]
    elif case == "empty":
        reg = [5, 5, 5, 4, 4, 4, 1, 1, 1]
    elif case == "cc_eno":
        op, cent, order = 6, 2, 3
    dst = _arr(fine)
    srcs = (cgx_array * len(times))(*[_arr(coarse) for _ in times])
    ts = (C.c_double * len(times))(*times)
    rc = lib.cgx_transfer(op, cent, C.byref(dst), srcs, ts, len(times), box9(reg), box9(coarse),
                          None, time, order, ot, None)
    assert rc in (EINVAL, EUNSUPPORTED), lib.cgx_last_error()
    assert lib.cgx_last_error()
