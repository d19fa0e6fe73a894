"""The hp-adaptive configuration at its own scale (128 x 128 jittered walled
mesh, N 4 -> 12, two split levels, adaptation every 20 steps, two crossing
pulses) against the reference's own CPU adapt, in lockstep: three rounds in
which p-refinement and element splitting (to split level 2, with 2:1 mortar
faces) both fire. Refine flags, p/h decisions, element orders, split levels,
Hilbert statuses, face orders and every other topology array must be
bit-identical after each round; the fields bit-identical in FP64_STRICT and
within 1e-12 relative L2 in FP64, after each adaptation and after five more
steps on the final nonconforming mesh. The harness is tests/hp_lockstep.py.
"""
from __future__ import annotations

import pytest

from tests import hp_lockstep

pytestmark = pytest.mark.gpu


def test_hp_configuration_lockstep_with_reference(ref_available):
    rep = hp_lockstep.run(rounds=3, extra_steps=5)
    rounds = rep["rounds"]
    # Both kinds of refinement happen, and the second split level is reached.
    assert sum(r["p_refine"] for r in rounds) > 0
    assert sum(r["h_refine"] for r in rounds) > 0
    assert 2 in rep["split_levels_reached"] and 1 in rep["split_levels_reached"]
    assert len(rounds[-1]["orders_after"]) >= 3
    for r in rounds:
        for name, fm in r["forms"].items():
            where = (r["round"], name)
            assert fm["refine_flags_equal"], where
            assert fm["p_h_decisions_equal"], where
            assert fm["topology_mismatches"] == [], (where, fm["topology_mismatches"])
            fa = fm["fields_after_adapt"]
            if name == "fp64_strict":
                assert fa["bitwise"], (where, fa)
            else:
                assert max(fa["rel_l2"].values()) < hp_lockstep.FIELD_TOL, (where, fa)
    fx = rep["fields_after_extra_steps"]
    assert fx["fp64_strict"]["bitwise"], fx
    assert max(fx["fp64"]["rel_l2"].values()) < hp_lockstep.FIELD_TOL, fx
    assert rep["flags_parity"]
