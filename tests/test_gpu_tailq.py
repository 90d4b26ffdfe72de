"""GPU parity of rtt_plan_tail_queue (the reference's dmma_plan_tile_tail_queue,
src/dmma_tile_tail_queue.h:190) against the oracle restatement, which
test_oracle_pin.py pins to the reference: chunk counts and gate reasons exact."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import rtt_spgemm as R
from test_oracle_pin import EARLY_CASES, TAIL_CASES, TAIL_MODEL, TAIL_POLICY, early_case, tail_tasks

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", list(TAIL_CASES))
def test_tail_planner_matches_oracle(case):
    pol, mod, tk = TAIL_CASES[case]
    pol, mod = {**TAIL_POLICY, **pol}, {**TAIL_MODEL, **mod}
    s, m, o = tail_tasks(**tk)
    ch, plan = R.plan_tail_queue(s, m, o, pol, mod)
    want_ch, want = O.plan_tail_queue(s, m, o, pol, mod)
    assert plan["reason"] == want["reason"], case
    assert np.array_equal(ch, want_ch)
    for k in ("output_tasks", "ordinary_tasks", "heavy_tasks", "chunks", "descriptor_bytes",
              "heavy_flag_bytes", "partial_workspace_bytes"):
        assert plan[k] == want[k], k
    assert plan["heavy_fraction"] == pytest.approx(want["heavy_fraction"])


def test_tail_planner_disabled_and_empty():
    ch, plan = R.plan_tail_queue([5, 900], [1, 800], [3, 4], dict(enabled=0))
    assert plan["reason"] == 0 and list(ch) == [0, 0]
    ch, plan = R.plan_tail_queue([], [], [])
    assert plan["reason"] == 4 and plan["output_tasks"] == 0


@pytest.mark.parametrize("case", list(EARLY_CASES))
def test_early_split_planner_matches_oracle(case):
    pol, mod, sms, (s, m, o) = early_case(case)
    ch, plan = R.plan_early_split(s, m, o, pol, mod, sms)
    want_ch, want = O.plan_early_split(s, m, o, pol, mod, sms)
    assert np.array_equal(ch, want_ch), case
    for k, v in want.items():
        assert plan[k] == v, (case, k)


def test_early_split_policy_defaults():
    assert R.early_split_policy_default() == pytest.approx(O.EARLY_SPLIT_POLICY)
