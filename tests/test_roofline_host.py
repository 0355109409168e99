"""The bench's byte accounting (roofline_bytes in the package), on per-round
counters given by hand.  reference_bytes is the reference round loop's byte
count, sum over rounds of 24 |A_r| + (4 + 4 weighted) E_r, with E_r the
entries its request and respond loops inspect; the other figures are the
kernels' own bytes per phase.  No device."""
from __future__ import annotations

import numpy as np


def _stats(mm, rows):
    st = np.zeros((len(rows), mm.STATS_COLS), dtype=np.int64)
    for r, row in enumerate(rows):
        for col, v in row.items():
            st[r, col] = v
    return st


def test_reference_bytes_and_edges(mm):
    st = _stats(mm, [
        {mm.ST_ACTIVE: 1000, mm.ST_BLUE: 520, mm.ST_REQ_ENTRIES: 4000, mm.ST_RESP_ENTRIES: 3500,
         mm.ST_MATCHED: 300, mm.ST_WINDOW_ENTRIES: 900},
        {mm.ST_ACTIVE: 600, mm.ST_BLUE: 310, mm.ST_REQ_ENTRIES: 2000, mm.ST_RESP_ENTRIES: 1000,
         mm.ST_MATCHED: 100, mm.ST_WINDOW_ENTRIES: 700, mm.ST_STAGED_DEG: 256, mm.ST_STAGED_ITEMS: 3},
    ])
    w = mm.roofline_bytes(st, True)
    assert w["edges"] == 4000 + 3500 + 2000 + 1000
    assert w["reference_bytes"] == 24 * 1000 + 8 * 7500 + 24 * 600 + 8 * 3000
    u = mm.roofline_bytes(st, False)
    assert u["reference_bytes"] == 24 * 1000 + 4 * 7500 + 24 * 600 + 4 * 3000
    # the kernels' own bytes per phase
    assert list(w["window_bytes"]) == [32 * 520 + 8 * 900, 32 * 310 + 8 * 700]
    assert list(u["window_bytes"]) == [32 * 520 + 4 * 900, 32 * 310 + 4 * 700]
    assert list(w["fallback_bytes"]) == [0, 8 * 256 + 36 * 3]
    assert list(w["commit_bytes"]) == [41 * 1000 - 12 * 300, 41 * 600 - 12 * 100]
    assert w["init_bytes"] == 41 * 1000 and u["init_bytes"] == 33 * 1000
    assert w["kernel_bytes"] == (w["window_bytes"].sum() + w["fallback_bytes"].sum() + w["commit_bytes"].sum()
                                 + w["finish_bytes"].sum() + w["init_bytes"])


def test_rounds_played_by_the_finish_phase_have_no_scan_or_commit_bytes(mm):
    # round 1 hands over to the finish phase, which plays rounds 1-3 itself:
    # its counters sit in round 1's row, the rounds after it carry only the
    # reference's counts
    rows = [{mm.ST_ACTIVE: 1000, mm.ST_BLUE: 500, mm.ST_REQ_ENTRIES: 3000, mm.ST_MATCHED: 400,
             mm.ST_WINDOW_ENTRIES: 800},
            {mm.ST_ACTIVE: 200, mm.ST_BLUE: 100, mm.ST_REQ_ENTRIES: 400, mm.ST_MATCHED: 150,
             mm.ST_FINISH_ITEMS: 200, mm.ST_FINISH_ENTRIES: 900},
            {mm.ST_ACTIVE: 50, mm.ST_BLUE: 30, mm.ST_REQ_ENTRIES: 60, mm.ST_MATCHED: 40},
            {mm.ST_ACTIVE: 10, mm.ST_BLUE: 5, mm.ST_MATCHED: 0}]
    w = mm.roofline_bytes(_stats(mm, rows), True)
    assert list(w["window_bytes"][1:]) == [0, 0, 0]
    assert list(w["commit_bytes"][1:]) == [0, 0, 0]
    assert w["window_bytes"][0] == 32 * 500 + 8 * 800
    assert list(w["finish_bytes"]) == [0, 84 * 200 + 5 * 900, 0, 0]
    # the reference's count covers every round it executes
    assert w["reference_bytes"] == 24 * (1000 + 200 + 50 + 10) + 8 * (3000 + 400 + 60)
    # a called-off attempt is followed by a window scan in the same round: kept
    rows[1][mm.ST_WINDOW_ENTRIES] = 120
    w = mm.roofline_bytes(_stats(mm, rows), True)
    assert w["window_bytes"][1] == 32 * 100 + 8 * 120 and w["commit_bytes"][2] == 41 * 50 - 12 * 40
