"""Host logic of the grid-function groups of carpet_b200.amr.BergerOliger,
on the CPU with stand-in streams and batches: the groups partition the grid
functions, each group's phases keep the reference's call order on a stream
of their own, every side stream forks from the calling stream before its
first launch (after group 0's first g * stagger phases when staggered), and
the calling stream joins every side stream at the end.  The bench step's
phase list (Carpet/src/Evolve.cc:44-121 order) is the one checked.
"""
from types import SimpleNamespace

import pytest

from carpet_b200.amr import BergerOliger
from carpet_b200.hierarchy import nested


class FakeStream:
    def __init__(self, name, log):
        self.name, self.log = name, log

    def wait_stream(self, other):
        self.log.append(("wait", self.name, other.name))


class FakeBatch:
    def __init__(self, key, grp, log):
        self.key, self.grp, self.log = key, grp, log

    def launch(self, stream):
        self.log.append(("launch", self.key, self.grp, stream.name))

    def launch_per_box(self, stream):
        self.log.append(("per_box", self.key, self.grp, stream.name))


@pytest.fixture(scope="module")
def hier():
    return nested(5, 33, ghost=3, buffer=9, order=5)


def make(h, ngf, groups, stagger=0):
    st = SimpleNamespace(ngf=ngf, ntl=3)
    bo = BergerOliger(h, st, groups=groups, stagger=stagger)
    log = []
    bo._side = [FakeStream(f"side{g}", log) for g in range(1, groups)]
    bo.batch = lambda key, grp=0: FakeBatch(key, grp, log)
    return bo, log


@pytest.mark.parametrize("ngf,groups", [(25, 1), (25, 2), (25, 3), (25, 5), (5, 5), (7, 3)])
def test_groups_partition_grid_functions(hier, ngf, groups):
    bo, _ = make(hier, ngf, groups)
    parts = [list(bo.gfs(g)) for g in range(groups)]
    assert sum(parts, []) == list(range(ngf))
    sizes = [len(p) for p in parts]
    assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1


def test_groups_validated(hier):
    with pytest.raises(ValueError):
        make(hier, 4, 0)
    with pytest.raises(ValueError):
        make(hier, 4, 5)
    with pytest.raises(ValueError):
        make(hier, 4, 2, stagger=-1)


@pytest.mark.parametrize("groups,stagger", [(2, 0), (3, 0), (2, 1), (3, 2), (2, 500)])
def test_group_chains_fork_and_join(hier, groups, stagger):
    bo, log = make(hier, 25, groups, stagger)
    keys = bo.step_phases()
    main = FakeStream("main", log)
    bo.run(keys, main)
    # each group: every phase once, in order, on its own stream
    for g in range(groups):
        mine = [e for e in log if e[0] == "launch" and e[2] == g]
        assert [e[1] for e in mine] == keys
        assert {e[3] for e in mine} == {"main" if g == 0 else f"side{g}"}
    for g in range(1, groups):
        name = f"side{g}"
        fork = log.index(("wait", name, "main"))
        first = next(i for i, e in enumerate(log) if e[0] == "launch" and e[3] == name)
        assert fork < first
        # group 0's phases issued on the calling stream before the fork
        before = [e for e in log[:fork] if e[0] == "launch" and e[2] == 0]
        assert len(before) == min(g * stagger, len(keys))
        # joined after its last launch
        join = log.index(("wait", "main", name))
        last = max(i for i, e in enumerate(log) if e[0] == "launch" and e[3] == name)
        assert join > last
    assert log[-(groups - 1):] == [("wait", "main", f"side{g}") for g in range(1, groups)]


def test_one_group_runs_on_the_calling_stream(hier):
    bo, log = make(hier, 25, 1)
    keys = bo.step_phases()
    main = FakeStream("main", log)
    bo.run(keys, main, per_box=True)
    assert log == [("per_box", k, 0, "main") for k in keys]
