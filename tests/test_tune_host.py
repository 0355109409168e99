"""Host logic of the autotuner (multicore-matching_b200/tune.py): which launch
options it keeps for a workload class, and that the shipped table
(tuned.json, read by DeviceGraph.tune_for) follows that rule.  No device: the
timing rows are given."""
from __future__ import annotations

import importlib.util
import json
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _tune():
    spec = importlib.util.spec_from_file_location("mm_tune", ROOT / "multicore-matching_b200" / "tune.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rows(times):
    return [{"finish_div": d, "blocks_per_sm": b, "ms": ms, "rounds": 20, "same": True}
            for (d, b), ms in times.items()]


def test_default_kept_unless_clearly_faster():
    t = _tune()
    # fastest within 3% of the default: the default stays
    choice, dflt, wins = t.pick(_rows({(12, 2): 1.00, (16, 1): 0.98, (-1, 2): 1.5}))
    assert not wins and (choice["finish_div"], choice["blocks_per_sm"]) == (12, 2) and choice is dflt
    # more than 3% faster: taken
    choice, dflt, wins = t.pick(_rows({(12, 2): 1.00, (16, 1): 0.95, (6, 1): 0.96}))
    assert wins and (choice["finish_div"], choice["blocks_per_sm"]) == (16, 1) and dflt["ms"] == 1.00
    # the default itself fastest
    choice, _, wins = t.pick(_rows({(12, 2): 0.90, (16, 1): 0.95}))
    assert not wins and choice["ms"] == 0.90


def test_shipped_table_is_consistent():
    """Every class in tuned.json names options from the tuner's search space, and
    a choice other than the default beat the default by more than 3%."""
    t = _tune()
    table = json.loads((ROOT / "multicore-matching_b200" / "tuned.json").read_text())
    assert table
    for name, c in table.items():
        assert c["finish_div"] in t.FIN_DIVS and c["blocks_per_sm"] in t.BLOCKS, name
        assert c["type"] in (6, 7, 8, 9), name
        if (c["finish_div"], c["blocks_per_sm"]) != t.DEFAULT:
            assert c["ms"] < 0.97 * c["default_ms"], name
        else:
            assert c["ms"] == c["default_ms"], name
