"""Autotuner for the launch options of the matching kernels (mm_graph_tune).

The kernels' shapes inside a launch (window length 32, window steps of 8
entries, a lane per vertex refilled from 64-item chunks, 256-entry fallback
segments, 512 threads) were fixed by measurement.  What varies with the workload is where the round
kernel hands over to the finish phase (the first round whose active set is at
most 1/d of round 0's: too early and components are too large, so the attempt
is called off and its scans are wasted; too late and the grid pays for more
rounds) and how many blocks per SM the two kernels use.  This tuner times each
(d, blocks per SM) pair on a workload with CUDA events (best of `repeats`),
checks that every candidate gives the same matching and round count (the
options never change the result), and picks the fastest.

    python multicore-matching_b200/tune.py [--classes rmat23,rgg20,grid512,er20,batch4096]

writes the table to profiles/tuning.md and the choices per workload class to
multicore-matching_b200/tuned.json; DeviceGraph.tune_for(class) applies one.
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
TUNED = PKG / "tuned.json"
FIN_DIVS = (-1, 4, 6, 8, 10, 12, 16, 24)
BLOCKS = (1, 2)
DEFAULT = (12, 2)  # the library's defaults (mm_graph_tune value 0)


def tune(mm, dg, type_, seeds, batch=False, fin_divs=FIN_DIVS, blocks=BLOCKS, repeats=5):
    """Time every (finish divisor, blocks per SM) pair on one device graph.
    Returns rows {finish_div, blocks_per_sm, ms, rounds, same} and the best row."""
    import torch

    out = torch.empty(max(dg.n, 1), dtype=torch.int32, device="cuda")

    def run():
        if batch:
            return int(dg.match_batch(type_, seeds, out.data_ptr()).max())
        return dg.match_device(type_, seeds, out.data_ptr())

    rows, ref = [], None
    for d in fin_divs:
        for b in blocks:
            dg.tune(d, b)
            run()  # warm-up
            best = 1e30
            for _ in range(repeats):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                r = run()
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            got = out.cpu().numpy()
            if ref is None:
                ref = (got.copy(), r)
            rows.append({"finish_div": d, "blocks_per_sm": b, "ms": best, "rounds": r,
                         "same": bool(np.array_equal(got, ref[0]) and r == ref[1])})
    dg.tune(0, 0)
    return rows, min(rows, key=lambda x: x["ms"])


def pick(rows, default=DEFAULT, margin=0.03):
    """The choice for a workload class from tune()'s rows: the fastest pair if it
    beats the library's default by more than `margin` (a fraction of the
    default's time), else the default.  Returns (choice row, default row, tuned?)."""
    dflt = next(r for r in rows if (r["finish_div"], r["blocks_per_sm"]) == tuple(default))
    best = min(rows, key=lambda x: x["ms"])
    wins = best["ms"] < (1.0 - margin) * dflt["ms"]
    return (best if wins else dflt), dflt, wins


def workloads(mm):
    """The workload classes: name -> (graph factory, type, batch offsets or None)."""
    sys.path.insert(0, str(ROOT))
    import bench

    def batch():
        u, b = bench.make_batch(mm, 4096, seed=3)
        return u, b["offsets"]

    return {
        "rmat23": (lambda: (mm.Graph.rmat(23, 16, 0.57, 0.19, 0.19, seed=1), None), 9),
        "rgg20": (lambda: (mm.Graph.rgg(1 << 20, 13.0, seed=7), None), 9),
        "er20": (lambda: (mm.Graph.er(1 << 20, 8.0, seed=1), None), 9),
        "grid512": (lambda: (mm.Graph.grid(512, 512), None), 7),
        "batch4096": (batch, 9),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--classes", default="rmat23,rgg20,er20,grid512,batch4096")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    from __graft_entry__ import load_package

    mm = load_package()
    import torch

    torch.cuda.set_device(args.device)
    seeds = mm.rand_seeds(12345, 255)
    tuned = json.loads(TUNED.read_text()) if TUNED.exists() else {}
    lines = ["# Launch options tuned per workload class (one B200)", "",
             "Command: `python multicore-matching_b200/tune.py` (writes this file and "
             "`multicore-matching_b200/tuned.json`).", "",
             "Device time of one matching (best of 5 CUDA-event timings), for each finish-phase divisor d "
             "(the phase starts at the first round whose active set is at most 1/d of round 0's; -1: never) and "
             "blocks per SM.  Every candidate gave the same matching and round count.", ""]
    for name in args.classes.split(","):
        make, type_ = workloads(mm)[name]
        g, off = make()
        with mm.DeviceGraph(g, device=args.device) as dg:
            if off is not None:
                dg.set_batch(off)
            dg.prepare(type_)
            rows, best = tune(mm, dg, type_, seeds, batch=off is not None)
        assert all(r["same"] for r in rows), name
        # keep the default unless the tuned choice is clearly faster
        choice, dflt, wins = pick(rows)
        tuned[name] = {"finish_div": choice["finish_div"], "blocks_per_sm": choice["blocks_per_sm"],
                       "ms": choice["ms"], "default_ms": dflt["ms"], "type": type_}
        lines += [f"## {name} (type {type_}, n = {g.n:,}, {g.nnz:,} entries)", "",
                  "| d \\\\ blocks per SM | " + " | ".join(str(b) for b in BLOCKS) + " |",
                  "|---|" + "---:|" * len(BLOCKS)]
        for d in FIN_DIVS:
            cells = [f"{next(r['ms'] for r in rows if r['finish_div'] == d and r['blocks_per_sm'] == b):.3f}"
                     for b in BLOCKS]
            lines.append(f"| {d} | " + " | ".join(cells) + " |")
        lines += ["", f"Default (d = {DEFAULT[0]}, {DEFAULT[1]} blocks per SM): {dflt['ms']:.3f} ms; fastest: "
                      f"d = {best['finish_div']}, {best['blocks_per_sm']} blocks per SM, {best['ms']:.3f} ms; "
                      f"chosen: d = {choice['finish_div']}, {choice['blocks_per_sm']} "
                      f"({'tuned' if wins else 'default kept: the fastest is within 3%'}).", ""]
        print(name, tuned[name], flush=True)
    TUNED.write_text(json.dumps(tuned, indent=1) + "\n")
    (ROOT / "profiles" / "tuning.md").write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
