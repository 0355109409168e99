"""Generate the golden fixtures from the reference's OWN code.

Runs the reference's GraphMatchingTBBRandom / GraphMatchingTBBWeighted
(src/matchtbb.cu:498-623; the GPU maximal types 7 / 9 run the same algorithm)
and the same classes built with the fixed 20-round cap (GPU types 6 / 8),
compiled from the reference sources into oracle/_ref by oracle/Makefile, after
srand(seed) exactly as bin/match.cpp:382 does.  Also records the reference's
sequential CPU matchers (types 0, 4) on the same graphs for quality
comparisons.

Output: tests/golden/golden.npz (small, committed), and with --full
tests/golden/full_size.json: the SHA-256, round count and next rand() value of
the reference's matching of the full-size R-MAT graph (2^23 vertices, edge
factor 16, seed 1), too large to store whole.  Needs the reference build
(oracle/_ref; run where the reference sources are, not on the GPU machine):

    python tests/golden/make_golden.py [--full]
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from __graft_entry__ import load_oracle, load_package  # noqa: E402
from graphs_small import random_graph  # noqa: E402

BARRIER = 0x88B81733
FULL_LIMIT = 5000  # store whole match vectors up to this many vertices, else a hash


def graph_cases(mm):
    """(name, graph) pairs; generator parameters are part of the name."""
    yield "grid_8x8", mm.Graph.grid(8, 8)
    yield "grid_64x64", mm.Graph.grid(64, 64)
    yield "grid_512x512", mm.Graph.grid(512, 512)
    yield "rgg_4096_s7", mm.Graph.rgg(4096, 13.0, seed=7)
    yield "rgg_65536_s7", mm.Graph.rgg(65536, 13.0, seed=7)
    yield "rmat_12_s1", mm.Graph.rmat(12, 16, seed=1)
    yield "rmat_16_s1", mm.Graph.rmat(16, 16, seed=1)
    yield "er_4096_s3", mm.Graph.er(4096, 8.0, seed=3)


def adversarial_cases():
    rng = np.random.default_rng(2024)
    for i in range(24):
        n = int(rng.integers(1, 48))
        g = random_graph(rng, n, avg_deg=float(rng.uniform(0.5, 6)), symmetric=bool(i % 3),
                         gaps=bool(i % 4 == 1), shuffle_ranges=bool(i % 5 == 2),
                         empty_reversed=0.2 if i % 6 == 3 else 0.0, dup=0.1, loops=0.1)
        yield f"adv_{i:02d}", g


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()


def main() -> None:
    mm = load_package()
    orc = load_oracle()
    if not orc.ref_available():
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    arrays: dict[str, np.ndarray] = {}
    index = []
    cases = list(graph_cases(mm)) + list(adversarial_cases())
    for name, g in cases:
        if name.startswith("adv_"):
            arrays[f"{name}/ranges"] = g.ranges
            arrays[f"{name}/nbrs"] = g.nbrs
            arrays[f"{name}/weights"] = g.weights
        seeds_list = (1, 12345) if not name.startswith("adv_") else (7,)
        barriers = (BARRIER,) if not name.startswith("adv_") else (BARRIER, 0x30000000, 0xF0000000)
        for seed in seeds_list:
            for barrier in barriers:
                for gpu_type, ref_type, fixed in ((6, 10, True), (7, 10, False), (8, 11, True), (9, 11, False)):
                    m, _, nxt = orc.ref_run(g, ref_type, barrier, seed, fixed_rounds=fixed)
                    seeds = orc.rand_seeds(seed, 256)
                    # rounds the reference drew: position of the next rand() value in the stream
                    hits = np.nonzero(seeds == nxt)[0]
                    rounds = int(hits[0]) if len(hits) else -1
                    if fixed:
                        rounds = 20  # the GPU fixed-round loop always draws NR_MATCH_ROUNDS values
                    valid, weight, size = orc.ref_check(g, m)
                    key = f"{name}/t{gpu_type}/s{seed}/b{barrier:08x}"
                    entry = {"key": key, "graph": name, "type": gpu_type, "seed": seed, "barrier": barrier,
                             "rounds": rounds, "next_rand": int(nxt), "valid": bool(valid),
                             "weight": float(weight), "size": int(size), "n": int(g.n),
                             "sha256": digest(m)}
                    if g.n <= FULL_LIMIT:
                        arrays[key] = m.astype(np.int32)
                    index.append(entry)
        # sequential reference matchers (quality baselines, types 0 / 4)
        if not name.startswith("adv_"):
            for ref_type in (0, 4):
                m, _, _ = orc.ref_run(g, ref_type, BARRIER, 12345)
                valid, weight, size = orc.ref_check(g, m)
                index.append({"key": f"{name}/cpu{ref_type}", "graph": name, "type": ref_type, "seed": 12345,
                              "barrier": BARRIER, "rounds": 0, "next_rand": 0, "valid": bool(valid),
                              "weight": float(weight), "size": int(size), "n": int(g.n), "sha256": digest(m)})
        print(f"{name}: n={g.n} nnz={g.nnz}", flush=True)
    arrays["index_json"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / "golden.npz", **arrays)
    print(f"wrote {len(index)} cases to {HERE / 'golden.npz'}")


def full_size() -> None:
    """The reference's matchings of the full-size R-MAT graph (GPU types 7 and 9,
    srand(12345) as bin/match.cpp:382), recorded by hash."""
    mm = load_package()
    orc = load_oracle()
    if not orc.ref_available():
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    g = mm.Graph.rmat(23, 16, 0.57, 0.19, 0.19, seed=1)
    seeds = orc.rand_seeds(12345, 256)
    out = {"graph": "rmat_23_ef16_s1", "n": int(g.n), "nnz": int(g.nnz), "cases": []}
    for gpu_type, ref_type in ((7, 10), (9, 11)):
        m, _, nxt = orc.ref_run(g, ref_type, BARRIER, 12345)
        rounds = int(np.nonzero(seeds == nxt)[0][0])
        valid, weight, size = orc.ref_check(g, m)
        out["cases"].append({"type": gpu_type, "seed": 12345, "barrier": BARRIER, "rounds": rounds,
                             "next_rand": int(nxt), "valid": bool(valid), "weight": float(weight), "size": int(size),
                             "sha256": digest(m)})
        print(out["cases"][-1], flush=True)
    (HERE / "full_size.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    if "--full" in sys.argv:
        full_size()
    else:
        main()
