"""The N > 1 path on CPU: batch sharding over ranks (gloo, world size 2).

A single graph does not shard (every rank matches its own replica); a batch of
independent graphs does: shard_batch splits the graphs into contiguous ranges of
about equal adjacency entries, every rank computing the same split with no
message, and bench.py's make_batch generates only the rank's own range.  These
tests check the split, and that two gloo ranks' shards agree on it, are
disjoint, cover the batch and concatenate to the single-process batch.  Each
rank then matches the graphs of its shard (the oracle's restatement stands in
for the kernel: no GPU here) and rank 0 gathers the results over the process
group; they must equal the single-process batch's, graph by graph."""
from __future__ import annotations

import importlib.util
import os
import socket
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _check_split(parts, sizes, world):
    assert len(parts) == world
    assert parts[0][0] == 0 and parts[-1][1] == len(sizes)
    for (a, b), (c, d) in zip(parts, parts[1:]):
        assert a <= b == c <= d
    return [float(np.sum(sizes[a:b])) for a, b in parts]


def test_shard_batch_edge_cases(mm):
    assert mm.shard_batch([], 3) == [(0, 0), (0, 0), (0, 0)]
    assert mm.shard_batch([5, 5, 5], 1) == [(0, 3)]
    assert mm.shard_batch([1, 1, 1, 1], 2) == [(0, 2), (2, 4)]
    parts = mm.shard_batch([1, 1], 4)  # more ranks than graphs: some ranks get none
    _check_split(parts, np.ones(2), 4)
    assert sum(b - a for a, b in parts) == 2
    assert mm.shard_batch([0, 0, 0], 2) in ([(0, 0), (0, 3)], [(0, 3), (3, 3)], [(0, 1), (1, 3)])
    with pytest.raises(ValueError):
        mm.shard_batch([1, -1], 2)
    with pytest.raises(ValueError):
        mm.shard_batch([1, 2], 0)


@pytest.mark.parametrize("world", [2, 3, 8])
def test_shard_batch_balances_log_uniform_sizes(mm, world):
    rng = np.random.default_rng(world)
    sizes = np.exp(rng.uniform(np.log(1 << 10), np.log(1 << 18), 4096 * world)) * 10
    loads = _check_split(mm.shard_batch(sizes, world), sizes, world)
    # every cut is within one graph of its target: imbalance below the largest graph
    assert max(loads) - min(loads) <= 2 * sizes.max()
    assert max(loads) / (sizes.sum() / world) < 1.01


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _match_graphs(mm, u, offsets, type_=9):
    """Weighted maximal matching of each graph of a batch union, one graph at a
    time (the oracle's restatement): [(match in the graph's numbering, rounds)]."""
    import sys

    sys.path.insert(0, str(ROOT))
    import oracle

    seeds = oracle.rand_seeds(12345, 256)
    r = np.asarray(u.ranges, np.int64).reshape(-1, 2)
    out = []
    for i in range(len(offsets) - 1):
        lo, hi = int(offsets[i]), int(offsets[i + 1])
        e0, e1 = int(r[lo, 0]), int(r[hi - 1, 1])
        x = mm.Graph(hi - lo, (r[lo:hi] - e0).astype(np.int32), u.nbrs[e0:e1] - lo, u.weights[e0:e1])
        m, rounds, _ = oracle.match(x, type_, seeds, 0x88B81733)
        out.append((np.asarray(m, np.int32), int(rounds)))
    return out


def _rank_main(rank, world, port, out_dir, count, seed):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import sys

        sys.path.insert(0, str(ROOT))
        from __graft_entry__ import load_package

        mm = load_package()
        bench = _bench()
        g, batch = bench.make_batch(mm, count, seed, rank, world)
        mine = {"range": batch["range"], "n": g.n, "nnz": g.nnz, "count": batch["count"], "total": batch["total"]}
        every = [None] * world
        dist.all_gather_object(every, mine)
        # the split every rank computed must be the same one
        ranges = [e["range"] for e in every]
        assert all(e["total"] == count * world for e in every)
        assert ranges[0][0] == 0 and ranges[-1][1] == count * world
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        np.savez(Path(out_dir) / f"rank{rank}.npz", ranges=np.asarray(g.ranges), nbrs=np.asarray(g.nbrs),
                 weights=np.asarray(g.weights), offsets=batch["offsets"], lo_hi=np.asarray(batch["range"]))
        # each rank matches its own graphs; rank 0 gathers every rank's results
        matched = _match_graphs(mm, g, batch["offsets"])
        every = [None] * world if rank == 0 else None
        dist.gather_object(matched, every, dst=0)
        if rank == 0:
            flat = [x for part in every for x in part]
            np.savez(Path(out_dir) / "gathered.npz", match=np.concatenate([m for m, _ in flat]),
                     rounds=np.asarray([r for _, r in flat]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_batch(mm, tmp_path):
    import torch.multiprocessing as mp

    count, seed, world = 4, 3, 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), count, seed), nprocs=world,
                       join=True, start_method="spawn")
    shards = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    bench = _bench()
    full, fb = bench.make_batch(mm, count * world, seed)  # one process, the same 8 graphs
    # concatenating the shards (ids shifted by the earlier shards' sizes) gives the full batch
    v0 = e0 = 0
    ranges, nbrs, weights, offs = [], [], [], [np.zeros(1, np.int64)]
    for s in shards:
        ranges.append(s["ranges"].reshape(-1, 2).astype(np.int64) + e0)
        nbrs.append(s["nbrs"].astype(np.int64) + v0)
        weights.append(s["weights"])
        offs.append(s["offsets"][1:].astype(np.int64) + v0)
        v0 += int(s["offsets"][-1])
        e0 += s["nbrs"].size
    assert np.array_equal(np.concatenate(ranges), np.asarray(full.ranges).reshape(-1, 2))
    assert np.array_equal(np.concatenate(nbrs), np.asarray(full.nbrs))
    assert np.array_equal(np.concatenate(weights), np.asarray(full.weights))
    assert np.array_equal(np.concatenate(offs), fb["offsets"].astype(np.int64))
    lo_hi = [tuple(s["lo_hi"]) for s in shards]
    assert lo_hi[0][0] == 0 and lo_hi[0][1] == lo_hi[1][0] and lo_hi[1][1] == count * world
    # the gathered per-rank matchings equal the single-process batch's
    got = np.load(tmp_path / "gathered.npz")
    want = _match_graphs(mm, full, fb["offsets"])
    assert np.array_equal(got["match"], np.concatenate([m for m, _ in want]))
    assert got["rounds"].tolist() == [r for _, r in want]
