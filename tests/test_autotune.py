"""CPU checks of the autotuner's selection logic with stand-in workloads (no GPU): the best
candidate wins, a candidate that fails is recorded but never chosen, and BFS is scored by
searches per second rather than by calls per second (its call count depends on the order of
evaluation, so the faster run can make fewer calls)."""
import json

from harmonize_b200 import autotune


def test_tuner_picks_the_best_and_scores_bfs_by_time(tmp_path, monkeypatch):
    def photon(prog, variant=0, patience=0, fill_links=0):
        if variant == 3:
            raise RuntimeError("does not fit")
        # variant 1 with patience 16 and fill 4 is fastest
        ms = 10.0 - (variant == 1) * 3.0 - (patience == 16) - (fill_links == 4) * 0.5
        return {"evals": 1_000_000, "device_ms": ms}

    def bfs(prog, variant=0, patience=0, fill_links=0):
        # variant 4 makes the most calls per second but takes longest; variant 2 is fastest
        if variant == 4:
            return {"evals": 90_000_000, "device_ms": 9.0}
        if variant == 2:
            return {"evals": 20_000_000, "device_ms": 4.0}
        return {"evals": 30_000_000, "device_ms": 7.0}

    monkeypatch.setattr(autotune, "_single_spec_workloads", lambda: {"photon": photon, "bfs": bfs})
    monkeypatch.setattr(autotune, "TUNED_PATH", str(tmp_path / "tuned.json"))
    table = autotune.tune(["photon", "bfs"], reps=0, programs=("async",))

    p = table["photon/async"]
    assert (p["variant"], p["patience"], p["fill_links"]) == (1, 16, 4) and p["unit"] == "calls/s"
    assert any("error" in s and s["variant"] == 3 for s in p["sweep"])
    b = table["bfs/async"]
    assert b["variant"] == 2 and b["unit"] == "searches/s" and abs(b["score"] - 250.0) < 1e-9

    saved = json.load(open(tmp_path / "tuned.json"))
    assert saved["bfs/async"]["variant"] == 2
    monkeypatch.setattr(autotune, "TUNED_PATH", str(tmp_path / "tuned.json"))
    assert autotune.tuned_config("bfs", "async") == {"variant": 2, "patience": b["patience"],
                                                     "fill_links": b["fill_links"]}
    assert autotune.tuned_config("collatz", "async") == {"variant": 0, "patience": 0, "fill_links": 0}
