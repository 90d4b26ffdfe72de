"""The autotuner's host logic on the CPU: shape classes, the choice of the
fastest candidate, persistence per device, reuse of a stored choice, and
candidates that fail."""
from __future__ import annotations

import json

from rtt_spgemm import autotune as T


def test_shape_class_buckets():
    assert T.shape_class("AB", 884736, 23393656, 27) == "AB|r19|d4|s0"
    # R-MAT-like skew: longest row 6350, mean 14.6
    assert T.shape_class("AAT", 65536, 955117, 6350) == "AAT|r16|d3|s8"
    assert T.shape_class("AB", 0, 0, 0) == "AB|r0|d0|s0"


def test_tune_picks_fastest_and_persists(tmp_path):
    path = tmp_path / "tune.json"
    cands = [{"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": s} for s in (0, 7, -1)]
    speed = {0: 3.0, 7: 1.0, -1: 2.0}
    calls = []

    def runner(cfg):
        calls.append(cfg["split_target"])
        return speed[cfg["split_target"]]

    t = T.Tuner(path, candidates=cands, device_name="dev0", repeats=2)
    best = t.choose("AB|r10|d2|s0", runner)
    assert best["split_target"] == 7
    assert len(calls) == 3 * 3  # one untimed + two timed runs per candidate
    stored = json.loads(path.read_text())
    e = stored["devices"]["dev0"]["AB|r10|d2|s0"]
    assert e["config"]["split_target"] == 7 and len(e["candidates"]) == 3
    # a new tuner reads the file and does not run again
    calls.clear()
    t2 = T.Tuner(path, candidates=cands, device_name="dev0")
    assert t2.choose("AB|r10|d2|s0", runner)["split_target"] == 7 and not calls
    # another device tunes on its own
    t3 = T.Tuner(path, candidates=cands, device_name="dev1", repeats=1)
    t3.choose("AB|r10|d2|s0", runner)
    assert calls


def test_failing_candidate_is_skipped(tmp_path):
    cands = [{"dmma_pair_cutoff": 0, "b_staging": 1, "split_target": 0},
             {"dmma_pair_cutoff": 0, "b_staging": 0, "split_target": 0}]

    def runner(cfg):
        if cfg["b_staging"]:
            raise RuntimeError("no room")
        return 1.0

    t = T.Tuner(tmp_path / "t.json", candidates=cands, device_name="d")
    assert t.choose("k", runner)["b_staging"] == 0
    e = json.loads((tmp_path / "t.json").read_text())["devices"]["d"]["k"]
    assert e["candidates"][0]["ms"] is None
