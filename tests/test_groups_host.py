"""Host-side checks of the grouped operators (no GPU needed)."""
from __future__ import annotations

import pytest


def test_empty_group_is_rejected():
    from em3d_b200.groups import AcousticOperatorGroup, OperatorGroup

    with pytest.raises(ValueError, match="at least one problem"):
        OperatorGroup([])
    with pytest.raises(ValueError, match="at least one problem"):
        AcousticOperatorGroup([])


def test_group_by_grid_buckets_in_first_seen_order():
    from types import SimpleNamespace

    from em3d_b200 import groups

    def prob(n, L=(1.0, 1.0, 1.0)):
        return SimpleNamespace(grid=SimpleNamespace(N=(n, n, n), L=L))

    made = []

    class Fake:
        def __init__(self, ps):
            made.append(len(ps))

    orig = groups.OperatorGroup
    groups.OperatorGroup = Fake
    try:
        out = groups.group_by_grid([prob(32), prob(48), prob(32), prob(32, (1.0, 1.0, 2.0)), prob(48)])
    finally:
        groups.OperatorGroup = orig
    assert [idx for idx, _ in out.values()] == [[0, 2], [1, 4], [3]]
    assert made == [2, 2, 1]
