"""Host logic of the uneven-batch scheduler: in-order packing of (device,
energy-chunk) work items under an HBM budget."""

import pytest

from libnegf_b200.batch import pack


def _flatten(groups):
    return [(k, s, c) for g in groups for (k, s, c) in g]


def test_everything_fits_in_one_group():
    assert pack([("a", 3, 10), ("b", 2, 20)], 1000) == [[("a", 0, 3), ("b", 0, 2)]]


def test_groups_respect_the_budget_and_keep_order():
    items = [(k, n, per) for k, n, per in [(0, 5, 7), (1, 9, 3), (2, 4, 11), (3, 16, 2)]]
    groups = pack(items, 30)
    for g in groups:
        assert sum(c * dict((k, per) for k, _, per in items)[k] for k, _, c in g) <= 30
    # every energy of every item exactly once, in order
    seen = {}
    for k, s, c in _flatten(groups):
        assert s == seen.get(k, 0)
        seen[k] = s + c
    assert seen == {0: 5, 1: 9, 2: 4, 3: 16}


def test_unit_larger_than_budget_goes_alone():
    groups = pack([("x", 2, 50), ("y", 1, 5)], 40)
    assert groups == [[("x", 0, 1)], [("x", 1, 1)], [("y", 0, 1)]]


@pytest.mark.parametrize("budget", [1, 17, 64, 10 ** 9])
def test_counts_are_conserved(budget):
    items = [(i, (7 * i) % 13 + 1, (5 * i) % 9 + 1) for i in range(20)]
    total = {k: n for k, n, _ in items}
    got = {}
    for k, s, c in _flatten(pack(items, budget)):
        got[k] = got.get(k, 0) + c
    assert got == total


def test_halve_conserves_and_orders():
    from libnegf_b200.batch import halve
    g = [(0, 0, 3), (1, 2, 5), (2, 0, 1)]
    a, b = halve(g)
    got = {}
    for k, s, c in a + b:
        got.setdefault(k, []).append((s, c))
    assert got == {0: [(0, 3)], 1: [(2, 1), (3, 4)], 2: [(0, 1)]}
    assert sum(c for _, _, c in a) == 4


class _Req:
    def __init__(self, n, per):
        self.energies = list(range(n))
        self.per_energy = per


class _Queue:
    """Stand-in for the server's state that _take_group reads and updates."""

    def __init__(self, reqs, budget):
        import collections
        self._queue = collections.deque((r, 0, len(r.energies)) for r in reqs)
        self.budget = budget


def test_server_takes_fifo_groups_and_splits_the_last_request():
    # NegfServer._take_group: the head of the queue under the budget, the last
    # request possibly in part; the rest stays queued in order
    from libnegf_b200.server import NegfServer
    a, b, c = _Req(4, 10), _Req(6, 10), _Req(3, 10)
    q = _Queue([a, b, c], budget=70)
    g1 = NegfServer._take_group(q)
    assert g1 == [(a, 0, 4), (b, 0, 3)]
    assert list(q._queue) == [(b, 3, 3), (c, 0, 3)]
    g2 = NegfServer._take_group(q)
    assert g2 == [(b, 3, 3), (c, 0, 3)]
    assert not q._queue


def test_server_takes_a_single_energy_larger_than_the_budget():
    from libnegf_b200.server import NegfServer
    big = _Req(2, 500)
    q = _Queue([big], budget=100)
    assert NegfServer._take_group(q) == [(big, 0, 1)]
    assert list(q._queue) == [(big, 1, 1)]
    assert NegfServer._take_group(q) == [(big, 1, 1)]
    assert not q._queue


def test_autotune_candidates_and_signature():
    from libnegf_b200.autotune import candidates, signature

    class D:
        def __init__(self, sizes):
            self.sizes = sizes

    small = [D([32, 64]), D([100])]
    assert candidates(small) == [dict(gemm_form=2, gj_nb=0), dict(gemm_form=1, gj_nb=0)]
    big = [D([256, 256])]
    c = candidates(big)
    assert dict(gemm_form=2, gj_nb=32) in c and dict(gemm_form=1, gj_nb=8) in c
    # panels that do not fit shared memory are not candidates (n = 1024: nb = 32 needs 512 KiB)
    assert all(x["gj_nb"] != 32 for x in candidates([D([1024])]))
    assert signature(small, "fp64") == ("fp64", 128) and signature(big, "mixed") == ("mixed", 256)


def test_native_server_grouping_rule():
    # negf_server_group_sizes: the native worker's FIFO grouping under a budget
    from libnegf_b200.server import group_sizes
    assert group_sizes([10, 20, 30, 100, 5, 5], 50) == [2, 1, 1, 2]
    assert group_sizes([], 10) == []
    assert group_sizes([200], 10) == [1]
    assert group_sizes([5] * 7, 15) == [3, 3, 1]
    assert sum(group_sizes(list(range(1, 30)), 40)) == 29


def test_native_server_needs_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from libnegf_b200 import NegfError
    from libnegf_b200.server import NativeServer
    with pytest.raises(NegfError):
        NativeServer()
