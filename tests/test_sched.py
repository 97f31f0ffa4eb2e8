"""The library's C++ host schedules (cgx_sched_*, the dh send/recv region
lists) against the Python restatement in carpet_b200.hierarchy /
carpet_b200.moving, on nested and moving-box hierarchies: the same pairs
(as sets) for sync, boundary prolongation, restriction and the regrid fill."""
import time

from carpet_b200 import moving
from carpet_b200.hierarchy import nested


def as_set(pairs):
    return {(p.dst_comp, p.src_comp, tuple(p.dstbox), tuple(p.srcbox)) for p in pairs}


def same_schedules(a, b):
    for l in range(len(a.levels)):
        assert as_set(a.sync[l]) == as_set(b.sync[l]), ("sync", l)
        if l:
            assert as_set(a.prolong[l]) == as_set(b.prolong[l]), ("prolong", l)
            assert as_set(a.restrict[l]) == as_set(b.restrict[l]), ("restrict", l)


def test_nested_schedules_native_equal_python():
    for args in ((3, 33, (2, 2, 2), 3, 9, 5), (2, 33, [(1, 1, 1), (2, 1, 1)], 3, 3, 3),
                 (4, (33, 41, 37), (3, 2, 1), 2, 4, 3)):
        n, pts, parts, ghost, buffer, order = args
        same_schedules(nested(n, pts, parts, ghost, buffer, order, native=True),
                       nested(n, pts, parts, ghost, buffer, order, native=False))


def test_moving_schedules_and_fill_native_equal_python():
    spec = moving.MovingSpec(nlevels=4, n0=65, nbox=33, parts0=(2, 1, 1), parts=(1, 2, 1), ghost=3,
                             buffer=3, order=5)
    for step in (0, 8, 16):
        a, b = moving.build(spec, step, native=True), moving.build(spec, step, native=False)
        same_schedules(a, b)
    h0, h1 = moving.build(spec, 0), moving.build(spec, 8)
    for l in range(1, spec.nlevels):
        c1, p1 = moving.old2new(h0, h1, l, native=True)
        c2, p2 = moving.old2new(h0, h1, l, native=False)
        assert as_set(c1) == as_set(c2) and as_set(p1) == as_set(p2), l


def test_native_schedule_is_fast_on_the_moving_workload():
    """the full 8-level moving-box regrid schedule in well under a second"""
    spec = moving.MovingSpec()
    t = time.perf_counter()
    h0, h1 = moving.build(spec, 0), moving.build(spec, 8)
    for l in range(1, spec.nlevels):
        moving.old2new(h0, h1, l)
    assert time.perf_counter() - t < 5.0
