"""Kernel variants on the host (no GPU): a plan's variant reads back as set,
invalid variants are rejected, and counts-relevant plan fields stay put."""
from __future__ import annotations

import pytest

import graphindor_b200 as gi


def test_variant_round_trip_and_validation():
    s = gi.Schedule_IEP(gi.Pattern(5, "0101110101010101010011000"), 1 << 14, 1 << 18, 1 << 16)
    before = s.export()
    v = s.variant
    assert v["leaf_flat"] in (0, 1) and v["occupancy"] == 0 and v["lane_budget"] > 0
    assert v["split"] == v["leaf_handoff"] == v["mid_handoff"] == 0
    s.variant = {"leaf_flat": 1, "lane_budget": 512, "occupancy": 16, "split": 8, "leaf_handoff": 16}
    assert s.variant == {"leaf_flat": 1, "lane_budget": 512, "occupancy": 16, "split": 8, "leaf_handoff": 16,
                         "mid_handoff": 0, "edge_triangles": 0}
    s.variant = {"lane_budget": 0}  # 0 keeps the budget
    assert s.variant["lane_budget"] == 512
    with pytest.raises(gi.GIError):
        s.variant = {"occupancy": 3}
    with pytest.raises(gi.GIError):
        s.variant = {"lane_budget": -1}
    with pytest.raises(gi.GIError):
        s.variant = {"split": -2}
    assert s.export() == before


def test_edge_triangle_variant_only_for_plans_that_allow_it():
    d = gi.Schedule_IEP(gi.Pattern(4, "0111101111001100"), 1 << 16, 1 << 20, 1 << 18)  # diamond
    d.variant = {"edge_triangles": 1}
    assert d.variant["edge_triangles"] == 1
    for n, adj in ((4, "0110100110010110"), (3, "011101110"), (5, "0101110101010101010011000")):
        s = gi.Schedule_IEP(gi.Pattern(n, adj), 1 << 16, 1 << 20, 1 << 18)
        s.variant = {"edge_triangles": 1}
        assert s.variant["edge_triangles"] == 0, adj
