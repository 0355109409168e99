"""The full-size configurations against the reference's own results.

* R-MAT, 2^23 vertices, edge factor 16, seed 1, weighted and random maximal
  (GPU types 9 and 7, srand(12345) as bin/match.cpp:382 draws the seeds): the
  whole match[] by SHA-256, the round count and the next rand() value, against
  tests/golden/full_size.json, which tests/golden/make_golden.py --full wrote
  from the reference's GraphMatchingTBBWeighted / GraphMatchingTBBRandom
  (src/matchtbb.cu:498-623) built from its sources.
* The 4096-graph batch (independent graphs of 2^10 to 2^18 vertices: grids,
  random geometric and Erdos-Renyi graphs, weighted maximal) matched in one
  batched call: each graph of an evenly spaced sample of 48 against the
  reference run on that graph alone (match[] and rounds), and every graph of a
  wider sample valid and maximal by the reference's testMatching restated.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
BARRIER = 0x88B81733


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.set_device(0)
    return torch


def test_rmat23_matches_reference_record(mm, orc, torch_cuda):
    rec = json.loads((ROOT / "tests" / "golden" / "full_size.json").read_text())
    g = mm.Graph.rmat(23, 16, 0.57, 0.19, 0.19, seed=1)
    assert (g.n, g.nnz) == (rec["n"], rec["nnz"])
    seeds = orc.rand_seeds(12345, 256)
    with mm.DeviceGraph(g, device=0) as dg:
        for case in rec["cases"]:
            got, rounds = dg.match(case["type"], seeds)
            assert rounds == case["rounds"], case["type"]
            # the reference drew exactly `rounds` values: the next one is seeds[rounds]
            assert int(seeds[rounds]) == case["next_rand"]
            assert hashlib.sha256(np.ascontiguousarray(got, np.int32).tobytes()).hexdigest() == case["sha256"]
            d = torch_cuda.from_numpy(got).cuda()
            chk = dg.check(d.data_ptr())
            w, s = dg.weight(d.data_ptr())
            assert chk["valid"] and chk["matchable"] == 0
            assert s == case["size"] and abs(w - case["weight"]) <= 1e-9 * case["weight"]


def test_batch4096_graphs_match_reference(mm, orc, torch_cuda):
    sys.path.insert(0, str(ROOT))
    import bench

    u, batch = bench.make_batch(mm, 4096, seed=3)
    off = batch["offsets"]
    seeds = orc.rand_seeds(12345, 256)
    with mm.DeviceGraph(u, device=0) as dg:
        dg.set_batch(off)
        out = torch_cuda.empty(u.n, dtype=torch_cuda.int32, device="cuda")
        rounds = dg.match_batch(9, seeds, out.data_ptr())
        got = out.cpu().numpy()
    assert len(rounds) == 4096
    for i, x in batch["sample"]:
        want, _, nxt = orc.ref_run(x, 11, BARRIER, 12345)
        assert np.array_equal(got[off[i]:off[i + 1]], want), i
        assert rounds[i] == int(np.nonzero(seeds == nxt)[0][0]), i
    for i in np.linspace(0, 4095, 256).astype(int):
        lo, hi = int(off[i]), int(off[i + 1])
        r = np.asarray(u.ranges, np.int64)[lo:hi]
        e0 = int(r[0, 0])
        x = mm.Graph(hi - lo, (r - e0).astype(np.int32), u.nbrs[e0:int(r[-1, 1])] - lo,
                     u.weights[e0:int(r[-1, 1])], f"batch-{i}")
        chk = orc.check(x, got[lo:hi])
        assert chk["valid"] and chk["matchable"] == 0, i
