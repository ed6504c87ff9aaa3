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
