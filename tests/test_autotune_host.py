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
                         "mid_handoff": 0}
    s.variant = {"lane_budget": 0}  # 0 keeps the budget
    assert s.variant["lane_budget"] == 512
    with pytest.raises(gi.GIError):
        s.variant = {"occupancy": 3}
    with pytest.raises(gi.GIError):
        s.variant = {"lane_budget": -1}
    with pytest.raises(gi.GIError):
        s.variant = {"split": -2}
    assert s.export() == before
