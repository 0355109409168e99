"""Benchmark: edges traversed per second and ms to a maximal matching on B200.

Workload (default): weighted maximal greedy matching (reference type 9) of an
R-MAT power-law graph with 2^23 vertices, edge factor 16,
(a, b, c, d) = (0.57, 0.19, 0.19, 0.05), symmetrised, self-loops and
duplicates removed, FP32 weights in (0, 1], graph seed 1, colouring seeds from
srand(12345) as the reference CLI draws them (bin/match.cpp:382), select
barrier 0x88B81733 (bin/match.cpp:183).

One step = one matching of the whole graph to maximality: the round kernel,
the finish kernel and (only if the finish phase is called off) the resumed
round kernel, three launches on one stream.

  value     edges traversed / s with the graph resident in HBM (the reference's
            t1 -> t2 "match time", bin/match.cpp:436-437).  Edges traversed =
            adjacency entries the reference's request and respond loops
            inspect, summed over rounds (the count the TBB matcher does),
            measured by an instrumented run.
  e2e       the same metric end to end through the C ABI with host buffers:
            upload + validation + preparation + matching + download + free per
            step (the reference's t0 -> t3 "total time").
  roofline  achieved = the reference's algorithmic bytes of one matching,
            sum_r [24 |A_r| + 8 E_r] (weighted; 4 E_r random), over the step's
            CUDA-event time, against the measured HBM copy bandwidth; traffic =
            DRAM bytes of one matching's launches from an ncu capture recorded
            in profiles/dram_traffic_<workload>.json.  The design's own byte
            count of the kernels it runs, and per-round phase times (barrier
            timestamps), are reported beside it.
  cpu_baseline  the reference's own GraphMatchingTBBWeighted (same algorithm,
            src/matchtbb.cu:567-623) compiled from its sources into
            oracle/_ref, on all host cores, on the same graph and seeds; its
            match[] is also compared with the GPU result ("parity").  Beside it
            the same matcher on one thread, and the sequential matchers
            (types 4 and 5 for weighted workloads, type 0 for random ones).
  forms     (N = 1) plain vs batched vs learned: the 4096-graph batch matched
            in one batched call and as 4096 separate calls, and the learned
            colouring's shipped policy on the 2^22 R-MAT and RGG multilevel
            hierarchies against the plain path.

--impl reference runs only that CPU matcher, on the same metric.
Multi-GPU (torchrun): for a single graph every rank matches its own replica
(one graph does not shard); for the batch workload every rank matches its own
shard of a batch of 4096 graphs per GPU, split by estimated adjacency entries
(independent graphs: no collective).  value is the sum over ranks of edges
divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from __graft_entry__ import load_package  # noqa: E402

METRIC = "edges traversed/s and ms to maximal matching, 1 B200, plain vs learned/batched"
BARRIER = 0x88B81733
MATCH_SEED = 12345

WORKLOADS = {
    "rmat23_weighted_maximal": dict(kind="rmat", scale=23, ef=16, seed=1, type=9),
    "rgg20_weighted_maximal": dict(kind="rgg", n=1 << 20, deg=13.0, seed=7, type=9),
    "grid512_random_maximal": dict(kind="grid", w=512, h=512, type=7),
    "rmat20_weighted_maximal": dict(kind="rmat", scale=20, ef=16, seed=1, type=9),
    "rmat22_weighted_maximal": dict(kind="rmat", scale=22, ef=16, seed=1, type=9),
    "batch4096_weighted_maximal": dict(kind="batch", count=4096, seed=3, type=9),
}
BATCH_SAMPLE = 48  # graphs of a batch the CPU baseline and the parity check run


def make_batch(mm, count, seed, rank=0, world=1):
    """Independent graphs, vertex counts log-uniform in [2^10, 2^18], each a 2D grid,
    a random geometric graph (average degree 13) or an Erdos-Renyi graph (average
    degree 8), weights in (0, 1] from a hash of the endpoint pair; their disjoint
    union, its offsets, and an evenly spaced sample of (index, graph).

    On N GPUs the batch has count * N graphs (count per GPU: weak scaling).  Every
    rank draws all graphs' sizes and kinds, splits them by estimated adjacency
    entries with shard_batch, and generates and matches only its own range; graph
    i is the same on any number of GPUs (its own seed), and N = 1 is the single-GPU
    batch."""
    rng = np.random.default_rng(seed)
    plan = []
    for _ in range(count * world):
        n = int(round(np.exp(rng.uniform(np.log(1 << 10), np.log(1 << 18)))))
        plan.append((n, int(rng.integers(3))))
    est = [n * (4, 13, 8)[kind] for n, kind in plan]
    lo, hi = mm.shard_batch(est, world)[rank]
    graphs = []
    for i in range(lo, hi):
        n, kind = plan[i]
        gs = seed * 100003 + i
        if kind == 0:
            wd = int(np.sqrt(n))
            graphs.append(mm.Graph.grid(wd, max(1, n // wd)).with_pair_weights(gs))
        elif kind == 1:
            graphs.append(mm.Graph.rgg(n, 13.0, seed=gs))
        else:
            graphs.append(mm.Graph.er(n, 8.0, seed=gs))
    u, off = mm.Graph.union(graphs)
    pick = np.linspace(0, len(graphs) - 1, min(BATCH_SAMPLE, len(graphs))).astype(int)
    sample = [(int(i) + lo, graphs[int(i)]) for i in pick]
    return u, {"offsets": off, "sample": sample, "count": len(graphs), "total": count * world, "range": (lo, hi)}


def make_graph(mm, spec, rank=0, world=1):
    """(graph, batch): batch is None, or the offsets and sample of a batch workload
    (this rank's shard of it on N GPUs)."""
    if spec["kind"] == "batch":
        return make_batch(mm, spec["count"], spec["seed"], rank, world)
    return make_single(mm, spec), None


def make_single(mm, spec):
    if spec["kind"] == "rmat":
        return mm.Graph.rmat(spec["scale"], spec["ef"], 0.57, 0.19, 0.19, seed=spec["seed"])
    if spec["kind"] == "rgg":
        return mm.Graph.rgg(spec["n"], spec["deg"], seed=spec["seed"])
    if spec["kind"] == "grid":
        return mm.Graph.grid(spec["w"], spec["h"])
    raise KeyError(spec["kind"])


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 20 ms from before the
    warm-up to the end of the timed steps and a hold period that keeps running
    the same step until the sampling spans at least min_s seconds (a short timed
    region alone would fall between two samples)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, min_s: float = 1.0):
        self.dev = device_index
        self.min_s = min_s
        self.proc = None
        self.lines = []
        self.started = threading.Event()
        self.t0 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            self.started.wait(timeout=2.0)  # nvidia-smi takes a moment to start
        except (OSError, FileNotFoundError):
            self.proc = None
        self.t0 = time.perf_counter()
        return self

    def _read(self):
        for line in self.proc.stdout:
            if self.t0 is not None:
                self.lines.append(line.strip())
            self.started.set()

    def remaining(self) -> float:
        """Seconds the hold period must still run."""
        return self.min_s - (time.perf_counter() - self.t0) if self.proc else 0.0

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "window": f"warm-up, timed steps and a hold on the same step, >= {self.min_s:g} s"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, spec, workload):
    """--impl reference: the reference's own CPU matcher on this machine's cores."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    mm = load_package()
    import oracle  # the CPU baseline leg is the one place bench.py runs oracle/

    g, batch = make_graph(mm, spec)
    t = spec["type"]
    ref_type = {6: 10, 7: 10, 8: 11, 9: 11}[t]
    fixed = t in (6, 8)
    cores = os.cpu_count() or 1
    seeds = oracle.rand_seeds(MATCH_SEED, 256)
    kind = "reference" if oracle.ref_available() else "port"
    # a batch is timed on its sample of graphs, one reference call per graph
    work = [g] if batch is None else [x for _, x in batch["sample"]]
    edges = 0.0
    for x in work:
        _, _, ost = oracle.match(x, t, seeds, BARRIER, nthreads=cores)
        edges += float(ost[:, oracle.ST_REQ_ENTRIES].sum() + ost[:, oracle.ST_RESP_ENTRIES].sum())
    times = []
    for i in range(args.warmup + args.steps):
        ms = 0.0
        for x in work:
            if kind == "reference":
                ms += oracle.ref_run(x, ref_type, BARRIER, MATCH_SEED, nthreads=cores, fixed_rounds=fixed)[1]
            else:
                t0 = time.perf_counter()
                oracle.match(x, t, seeds, BARRIER, nthreads=cores)
                ms += (time.perf_counter() - t0) * 1e3
        if i >= args.warmup:
            times.append(ms)
    ms = statistics.mean(times)
    value = edges / (ms / 1e3)
    sample = (f"full {workload} graph, one maximal matching per step" if batch is None else
              f"{len(work)} of the batch's {batch['count']} graphs (evenly spaced), one reference call each per step")
    line = {"metric": METRIC, "value": value, "unit": "edges/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+int32", "data": "synthetic",
            "config": {"workload": workload, "n": g.n, "nnz": g.nnz, "type": t, "barrier": BARRIER,
                       "srand": MATCH_SEED, "parallelism": "host cores", "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": "edges/s", "cores": cores, "kind": kind, "sample": sample,
                             "matcher": f"GraphMatchingTBB{'Weighted' if ref_type == 11 else 'Random'}"
                                        f"{' (20-round cap)' if fixed else ''}"},
            "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline(mm, g, t, gpu_match, workload, batch=None):
    """Reference TBB matcher on all host cores + parity of the GPU result (rank 0, N=1 only).

    For a batch: the reference runs each graph of the batch's sample on its own,
    and the GPU's slice of each is compared with it."""
    import oracle  # the CPU baseline leg is the one place bench.py runs oracle/

    cores = os.cpu_count() or 1
    ref_type = {6: 10, 7: 10, 8: 11, 9: 11}[t]
    fixed = t in (6, 8)
    seeds = oracle.rand_seeds(MATCH_SEED, 256)
    kind = "reference" if oracle.ref_available() else "port"
    if batch is None:
        items = [(g, gpu_match)]
    else:
        off = batch["offsets"]
        items = [(x, gpu_match[off[i]:off[i + 1]]) for i, x in batch["sample"]]
    ms_total, edges, parity, valid, maximal, w_gpu, s_gpu = 0.0, 0.0, True, True, True, 0.0, 0
    for x, got in items:
        _, _, ost = oracle.match(x, t, seeds, BARRIER, nthreads=cores)
        edges += float(ost[:, oracle.ST_REQ_ENTRIES].sum() + ost[:, oracle.ST_RESP_ENTRIES].sum())
        if kind == "reference":
            ref_m, ms, _ = oracle.ref_run(x, ref_type, BARRIER, MATCH_SEED, nthreads=cores, fixed_rounds=fixed)
        else:
            t0 = time.perf_counter()
            ref_m, _, _ = oracle.match(x, t, seeds, BARRIER, nthreads=cores)
            ms = (time.perf_counter() - t0) * 1e3
        ms_total += ms
        parity &= bool(np.array_equal(ref_m, got))
        chk = oracle.check(x, got)
        valid &= chk["valid"]
        maximal &= chk["matchable"] == 0
        wx, sx = oracle.weight(x, got)
        w_gpu += wx
        s_gpu += sx
    # the same TBB matcher on one thread (the reference's scaling normaliser,
    # scaling.sh:17, results/randomscale.p:17-27) and the sequential matchers
    # (bin/match.cpp:136-158: types 0, 4, 5), for one graph
    one, seq = None, []
    if oracle.ref_available() and batch is None:
        _, ms1, _ = oracle.ref_run(g, ref_type, BARRIER, MATCH_SEED, nthreads=1, fixed_rounds=fixed)
        one = {"ms": ms1, "value": edges / (ms1 / 1e3), "cores": 1}
        for st in ((4, 5) if t in (8, 9) else (0,)):
            seq_m, seq_ms, _ = oracle.ref_run(g, st, BARRIER, MATCH_SEED, nthreads=1)
            w_seq, s_seq = oracle.weight(g, seq_m)
            seq.append({"type": st, "ms": seq_ms, "weight": w_seq, "size": s_seq, "cores": 1})
    sample = (f"full {workload} graph, one matching" if batch is None else
              f"{len(items)} of the batch's {batch['count']} graphs (evenly spaced), one reference call each")
    return {"kind": kind, "cores": cores, "ms": ms_total, "value": edges / (ms_total / 1e3),
            "sample": sample, "parity": parity, "valid": valid, "maximal": maximal,
            "gpu_weight": w_gpu, "gpu_size": s_gpu, "tbb_1_thread": one, "sequential": seq}


def compare_batch(mm, local, seeds):
    """The 4096-graph batch workload (independent graphs, 2^10 to 2^18 vertices,
    grid / random geometric / Erdos-Renyi, weighted maximal): one batched call
    against the same graphs as 4096 separate plain calls, device time (CUDA
    events) and rounds; per-graph parity with the reference on the sample."""
    import torch

    t = 9
    u, batch = make_batch(mm, 4096, seed=3)
    off = batch["offsets"]
    out = torch.empty(u.n, dtype=torch.int32, device="cuda")
    res = {"graphs": len(off) - 1, "n": u.n, "nnz": u.nnz}
    with mm.DeviceGraph(u, device=local) as dg:
        dg.set_batch(off)
        dg.prepare(t)
        for _ in range(2):
            dg.match_batch(t, seeds, out.data_ptr())
        torch.cuda.synchronize()
        times = []
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            rounds = dg.match_batch(t, seeds, out.data_ptr())
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        got = out.cpu().numpy()
        st_r, st = dg.stats(t, seeds, out.data_ptr())
        edges = mm.roofline_bytes(st, True)["edges"]
    res["batched"] = {"ms": min(times), "rounds_max": int(rounds.max()), "rounds_sum": int(rounds.sum()),
                      "calls": 1, "edges_per_s": edges / (min(times) / 1e3)}
    # the same graphs one call each (the plain path: what the reference's matcher, one graph per call, does)
    ranges = np.asarray(u.ranges, dtype=np.int64).reshape(-1, 2)
    graphs = []
    for i in range(len(off) - 1):
        lo, hi = int(off[i]), int(off[i + 1])
        e0, e1 = int(ranges[lo, 0]), int(ranges[hi - 1, 1]) if hi > lo else int(ranges[lo, 0])
        r = (ranges[lo:hi] - e0).astype(np.int32)
        graphs.append(mm.Graph(hi - lo, r, u.nbrs[e0:e1] - lo, u.weights[e0:e1], f"batch-{i}"))
    dgs = [mm.DeviceGraph(x, device=local) for x in graphs]
    try:
        for d in dgs:
            d.prepare(t)
        torch.cuda.synchronize()
        rs, ms_dev = [], 0.0
        t0 = time.perf_counter()
        for i, d in enumerate(dgs):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            rs.append(d.match_device(t, seeds, out.data_ptr() + 4 * int(off[i])) if graphs[i].n else 0)
            b.record()
            b.synchronize()
            ms_dev += a.elapsed_time(b)
        wall = (time.perf_counter() - t0) * 1e3
    finally:
        for d in dgs:
            d.close()
    same = bool(np.array_equal(out.cpu().numpy(), got)) and [int(x) for x in rounds] == [int(x) for x in rs]
    res["plain_calls"] = {"ms_device": ms_dev, "ms_wall": wall, "rounds_max": int(max(rs)), "rounds_sum": int(sum(rs)),
                          "calls": len(dgs), "same_result_as_batched": same}
    cpu = cpu_baseline(mm, u, t, got, "batch4096_weighted_maximal", batch)
    res["parity_sample"] = {"graphs": len(batch["sample"]), "bit_exact_vs_reference": cpu["parity"],
                            "valid": cpu["valid"], "maximal": cpu["maximal"]}
    return res


def compare_learned(mm, local, seeds):
    """The learned colouring's shipped policy against the plain path on the
    2^22 R-MAT and RGG multilevel hierarchies (coarsened to 1% of the vertices):
    rounds, device time (best of 3) and matching weight summed over levels."""
    spec = __import__("importlib.util").util.spec_from_file_location(
        "multicore_matching_b200.policy", ROOT / "multicore-matching_b200" / "policy.py")
    pol = __import__("importlib.util").util.module_from_spec(spec)
    spec.loader.exec_module(pol)
    mlp = pol.load_policy()
    out = {}
    for name, g in (("rmat22", mm.Graph.rmat(22, 16, 0.57, 0.19, 0.19, seed=1)),
                    ("rgg22", mm.Graph.rgg(1 << 22, 13.0, seed=7))):
        levels = pol.hierarchy(mm, g, 9, seeds, device=local)
        rows = pol.evaluate(mm, levels[:-1], 9, seeds, mlp, repeats=3, device=local)
        tot = {arm: {"rounds": int(sum(r[arm]["rounds"] for r in rows)), "ms": float(sum(r[arm]["ms"] for r in rows)),
                     "weight": float(sum(r[arm]["weight"] for r in rows)),
                     "valid_maximal": all(r[arm]["valid"] and r[arm]["maximal"] for r in rows)}
               for arm in ("plain", "learned")}
        tot["levels"] = len(rows)
        tot["weight_change"] = tot["learned"]["weight"] / max(tot["plain"]["weight"], 1e-300) - 1.0
        out[name] = tot
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 400; 20 for --impl reference, whose steps are CPU matchings)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat23_weighted_maximal", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the plain vs batched vs learned comparisons")
    ap.add_argument("--ncu-case", action="store_true",
                    help="build + prepare, then one host-stepped matching only (for ncu captures of the kernels)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.impl == "reference" else 400
    args.warmup = max(args.warmup, 3)
    spec = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, spec, args.workload)

    world, rank, local = dist_setup()
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    mm = load_package()
    t = spec["type"]
    weighted = t in (8, 9)
    g, batch = make_graph(mm, spec, rank, world)
    seeds = mm.rand_seeds(MATCH_SEED, 255)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    dg = mm.DeviceGraph(g, device=local)
    if batch is not None:
        dg.set_batch(batch["offsets"])
    dg.prepare(t)
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    if args.ncu_case:
        r, ms_k, launches = dg.profile(t, seeds, out.data_ptr(), stream=sptr)
        torch.cuda.synchronize()
        print(json.dumps({"ncu_case": args.workload, "rounds": r, "launches": launches,
                          "ms_window": [round(float(x), 4) for x in ms_k[:, 0]],
                          "ms_fallback": [round(float(x), 4) for x in ms_k[:, 1]],
                          "ms_commit": [round(float(x), 4) for x in ms_k[:, 2]],
                          "ms_rounds_total": round(float(ms_k[:, 3].sum()), 4)}))
        dg.close()
        return 0
    # instrumented run: rounds and the work each round does
    rounds, st = dg.stats(t, seeds, out.data_ptr(), stream=sptr)
    work = mm.roofline_bytes(st, weighted)
    edges = work["edges"]
    # all ranks' edges: every rank matches its own replica, or its own shard of a batch
    edges_all = edges * world
    if dist and batch is not None:
        et = torch.tensor([float(edges)], dtype=torch.float64, device="cuda")
        dist.all_reduce(et, op=dist.ReduceOp.SUM)
        edges_all = float(et.item())

    # L2 is 126 MB; the CSR alone is > 1 GB, and a 512 MB write flushes L2 between steps.
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        for _ in range(args.warmup):
            dg.match_device(t, seeds, out.data_ptr(), stream=sptr)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.fill_(i & 0xFF)
                evs[i][0].record(stream)
                r = dg.match_device(t, seeds, out.data_ptr(), stream=sptr)
                evs[i][1].record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        # hold: the same step until the clock samples span at least a second
        while clocks.remaining() > 0:
            with torch.cuda.stream(stream):
                for _ in range(50):
                    flush.fill_(1)
                    dg.match_device(t, seeds, out.data_ptr(), stream=sptr)
            torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ms = statistics.mean(step_ms)
    if dist:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = edges_all / (ms / 1e3)
    # per-round phase times of the round kernel (barrier timestamps of the same launch shape)
    prof = []
    for _ in range(3):
        flush.fill_(1)
        _, ms_k, launches = dg.profile(t, seeds, out.data_ptr(), stream=sptr)
        prof.append(ms_k)
    nr = min(x.shape[0] for x in prof)
    ms_k = np.mean(np.stack([x[:nr] for x in prof]), axis=0)  # [executed rounds, (window, fallback, commit, sum)]
    gpu_launches = args.steps * launches
    phase_bytes = {"window": work["window_bytes"][:nr], "fallback": work["fallback_bytes"][:nr],
                   "commit": work["commit_bytes"][:nr]}
    kernel_bytes = work["kernel_bytes"]
    # the reference's algorithmic bytes of this rank's matching over the step's device time
    achieved = work["reference_bytes"] / (ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    # the scans are bound by random single-sector reads: their measured ceiling on this device
    gather_peak = mm.probe_gather_rate(local, max(g.n, 1))
    # the same random one-byte gathers over a 1 GiB table: most miss L2 (and the
    # TLB's reach), the regime of the window reads and the commit's key reads
    try:
        gather_dram = mm.probe_gather_rate(local, 1 << 30)
    except mm.MatchError:
        gather_dram = None
    colour_gathers = float(st[:, mm.ST_WINDOW_ENTRIES].sum() + st[:, mm.ST_STAGED_DEG].sum())
    # DRAM bytes of one matching's launches from an ncu capture of this workload, where one exists
    traffic = None
    tfile = ROOT / "profiles" / f"dram_traffic_{args.workload}.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("dram_bytes_per_step")

    # end to end through the C ABI with host buffers (pinned)
    ranges_h = torch.from_numpy(np.ascontiguousarray(g.ranges, dtype=np.int32)).pin_memory()
    nbrs_h = torch.from_numpy(g.nbrs).pin_memory()
    w_h = torch.from_numpy(g.weights).pin_memory() if weighted else None
    match_h = torch.empty(g.n, dtype=torch.int32).pin_memory()
    lib = mm.lib()
    import ctypes

    e2e_ms, e2e_parts = [], []
    for i in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = ctypes.c_void_p()
        mm._check(lib.mm_graph_create(g.n, ranges_h.data_ptr(), g.nnz, nbrs_h.data_ptr(),
                                      None if w_h is None else w_h.data_ptr(), local, ctypes.byref(h)))
        if batch is not None:
            mm._check(lib.mm_graph_set_batch(h, len(batch["offsets"]) - 1, batch["offsets"].ctypes.data))
        t1 = time.perf_counter()
        rr = ctypes.c_int()
        sd = np.ascontiguousarray(seeds)
        mm._check(lib.mm_match(h, t, BARRIER, sd.ctypes.data, len(sd), match_h.data_ptr(), ctypes.byref(rr), None))
        t2 = time.perf_counter()
        lib.mm_graph_destroy(h)
        t3 = time.perf_counter()
        dt = (t3 - t0) * 1e3
        if i > 0:
            e2e_ms.append(dt)
            e2e_parts.append(((t1 - t0) * 1e3, (t2 - t1) * 1e3, (t3 - t2) * 1e3))
    e2e = statistics.mean(e2e_ms)
    if dist:
        tt = torch.tensor([e2e], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e = float(tt.item())
    e2e_split = [statistics.mean(x[k] for x in e2e_parts) for k in range(3)]
    # where one step's time goes, each call followed by a device synchronisation: upload,
    # batch set-up, reverse-key build (mm_graph_prepare), first and second match
    def synced():
        torch.cuda.synchronize()
        return time.perf_counter()

    h = ctypes.c_void_p()
    ts = [synced()]
    mm._check(lib.mm_graph_create(g.n, ranges_h.data_ptr(), g.nnz, nbrs_h.data_ptr(),
                                  None if w_h is None else w_h.data_ptr(), local, ctypes.byref(h)))
    ts.append(synced())
    if batch is not None:
        mm._check(lib.mm_graph_set_batch(h, len(batch["offsets"]) - 1, batch["offsets"].ctypes.data))
    tp = [synced()]
    mm._check(lib.mm_graph_prepare(h, t))
    tp.append(synced())
    for _ in range(2):
        mm._check(lib.mm_match(h, t, BARRIER, sd.ctypes.data, len(sd), match_h.data_ptr(), ctypes.byref(rr), None))
        tp.append(synced())
    lib.mm_graph_destroy(h)
    e2e_detail = {"ms_create_synced": (ts[1] - ts[0]) * 1e3, "ms_set_batch_synced": (tp[0] - ts[1]) * 1e3,
                  "ms_prepare": (tp[1] - tp[0]) * 1e3, "ms_match_first": (tp[2] - tp[1]) * 1e3,
                  "ms_match_again": (tp[3] - tp[2]) * 1e3}
    h2d = g.n * 8 + g.nnz * 4 + (g.nnz * 4 if weighted else 0) + 255 * 4
    d2h = g.n * 4
    e2e_value = edges_all / (e2e / 1e3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        gpu_m = torch.empty(g.n, dtype=torch.int32, device="cuda")
        dg.match_device(t, seeds, gpu_m.data_ptr(), stream=sptr)
        torch.cuda.synchronize()
        cpu = cpu_baseline(mm, g, t, gpu_m.cpu().numpy(), args.workload, batch)
    dg.close()
    del flush
    forms = None
    if rank == 0 and world == 1 and not args.no_forms and batch is None:
        torch.cuda.empty_cache()
        mm.lib().mm_release_cached_memory(local)
        forms = {"batch4096_weighted_maximal": compare_batch(mm, local, seeds),
                 "learned_multilevel22_weighted_maximal": compare_learned(mm, local, seeds)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+int32", "data": "synthetic",
            "config": {"workload": args.workload, "n": g.n, "nnz": g.nnz, "type": t, "barrier": BARRIER,
                       "graphs": 1 if batch is None else batch["total"],
                       "srand": MATCH_SEED, "rounds": rounds,
                       "parallelism": (f"replicas x{world}" if batch is None else
                                       f"batch shards x{world} (graphs split by estimated entries, no collective)"),
                       "l2": "inputs > L2 (CSR > 1 GB) and a 512 MB L2 flush between steps"},
            "ms_to_maximal": ms, "edges_per_step": edges_all,
            "e2e": {"value": e2e_value, "unit": "edges/s", "ms_per_step": e2e, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_create": e2e_split[0], "ms_first_match": e2e_split[1],
                    "ms_destroy": e2e_split[2], **e2e_detail},
            "roofline": {"bound": "hbm",
                         "kernel": "one matching: k_rounds then k_finish (a resumed k_rounds only if the finish "
                                   "phase is called off)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_step": work["reference_bytes"],
                         "bytes_formula": "sum over rounds r of 24 |A_r| + (4 + 4 weighted) E_r: the reference's "
                                          "round loop (A_r active vertices, E_r entries its request and respond "
                                          "loops inspect)",
                         "launches_per_step": launches,
                         "design_bytes_per_step": kernel_bytes,
                         "design_frac": kernel_bytes / (ms / 1e3) / 1e9 / peak,
                         "phases": {k: {"ms": float(ms_k[:, c].sum()), "bytes": float(phase_bytes[k].sum()),
                                        "gbs": float(phase_bytes[k].sum() / max(ms_k[:, c].sum(), 1e-9) / 1e6),
                                        "frac": float(phase_bytes[k].sum() / max(ms_k[:, c].sum(), 1e-9) / 1e6 / peak)}
                                    for c, k in enumerate(("window", "fallback", "commit"))},
                         "per_round_work": {k: [int(x) for x in st[:nr, c]] for k, c in
                                            (("active", mm.ST_ACTIVE), ("blue", mm.ST_BLUE),
                                             ("blue_entries", mm.ST_BLUE_DEG), ("window_entries", mm.ST_WINDOW_ENTRIES),
                                             ("fallback_entries", mm.ST_STAGED_DEG), ("matched", mm.ST_MATCHED))},
                         "per_round_ms": {"window": [round(float(x), 4) for x in ms_k[:, 0]],
                                          "fallback": [round(float(x), 4) for x in ms_k[:, 1]],
                                          "commit": [round(float(x), 4) for x in ms_k[:, 2]]},
                         "random_reads": {"ceiling_per_s": gather_peak, "ceiling": "mm_probe_gather_rate, table of n bytes",
                                          "ceiling_1gib_per_s": gather_dram,
                                          "colour_gathers_per_step": colour_gathers,
                                          "colour_gathers_per_s": colour_gathers / (ms / 1e3)}},
            "gpu_launches": gpu_launches,
            "clocks": clocks.summary(),
        }
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": "edges/s", "cores": cpu["cores"],
                                    "kind": cpu["kind"], "sample": cpu["sample"], "ms": cpu["ms"],
                                    "matcher": "GraphMatchingTBB (src/matchtbb.cu) on all host cores",
                                    "tbb_1_thread": cpu["tbb_1_thread"], "sequential": cpu["sequential"]}
            line["parity"] = {"bit_exact_vs_reference": cpu["parity"], "valid": cpu["valid"],
                              "maximal": cpu["maximal"], "weight": cpu["gpu_weight"], "size": cpu["gpu_size"]}
        if forms is not None:
            line["forms"] = forms
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
