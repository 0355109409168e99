"""B200 greedy graph matching: Python host bindings.

Thin ctypes layer over the in-tree native libraries:

  * ``libmmatch.so`` -- the product: sm_100a kernels behind the C ABI of
    ``include/mm_match.h`` (GraphMatchingGPU* of the reference,
    src/matchgpu.h:29-84, as plain C).
  * ``libmmgen.so`` -- deterministic synthetic graphs in the reference's CSR
    layout (``mtc::Graph``, src/graph.h:41-60).

There is no CPU fallback: if ``libmmatch.so`` is missing or fails to load,
every matching call raises.  Build with ``build.build_all()``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

PKG = Path(__file__).resolve().parent

# Match encoding (src/matchgpu.cu:157-164, src/matchcpu.h:40-41).
BLUE, RED, DEAD = 0, 1, 2

# Matching types (bin/match.cpp:145-148).
RANDOM, RANDOM_MAXIMAL, WEIGHTED, WEIGHTED_MAXIMAL = 6, 7, 8, 9
TYPES = (RANDOM, RANDOM_MAXIMAL, WEIGHTED, WEIGHTED_MAXIMAL)

# Kernel families of mm_match_ex.
PATH_AUTO, PATH_PULL, PATH_PUSH = 0, 1, 2

# Default select barrier of the reference CLI (bin/match.cpp:183): p(blue) ~ 0.534.
DEFAULT_BARRIER = 0x88B81733

STATS_COLS = 13
POLICY_FLOATS = 129  # MM_POLICY_FLOATS: W1[16][6], b1[16], W2[16], b2
PROFILE_KERNELS = 4  # window scan, fallback scan, commit/recolour, their sum
(ST_ACTIVE, ST_BLUE, ST_RED, ST_REQ_ENTRIES, ST_RESP_ENTRIES, ST_BLUE_DEG, ST_RED_DEG, ST_MATCHED,
 ST_STAGED_DEG, ST_STAGED_ITEMS, ST_WINDOW_ENTRIES, ST_FINISH_ITEMS, ST_FINISH_ENTRIES) = range(13)

STATUS = {0: "MM_OK", 1: "MM_ERR_ARG", 2: "MM_ERR_GRAPH", 3: "MM_ERR_CUDA", 4: "MM_ERR_NOMEM",
          5: "MM_ERR_UNSUPPORTED", 6: "MM_ERR_SEEDS", 7: "MM_ERR_DEVICE"}


class MatchError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def max_rounds(type_: int) -> int:
    """Round cap: NR_MATCH_ROUNDS = 20 for types 6/8, 255 for 7/9 (src/matchcpu.h:24-25)."""
    return 20 if type_ in (RANDOM, WEIGHTED) else 255


# --------------------------------------------------------------------------
# library loading

_LIBS: dict[str, ctypes.CDLL] = {}

_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong
_U = ctypes.c_uint32

_MM_SIGS = {
    "mm_graph_create": (_I, [_I, _P, _LL, _P, _P, _I, ctypes.POINTER(_P)]),
    "mm_graph_create_device": (_I, [_I, _P, _LL, _P, _P, ctypes.POINTER(_P)]),
    "mm_graph_prepare": (_I, [_P, _I]),
    "mm_release_cached_memory": (_I, [_I]),
    "mm_graph_destroy": (None, [_P]),
    "mm_graph_n": (_I, [_P]),
    "mm_graph_nnz": (_LL, [_P]),
    "mm_graph_weighted": (_I, [_P]),
    "mm_graph_device_ranges": (_P, [_P]),
    "mm_graph_device_neighbours": (_P, [_P]),
    "mm_graph_device_weights": (_P, [_P]),
    "mm_max_rounds": (_I, [_I]),
    "mm_match": (_I, [_P, _I, _U, _P, _I, _P, ctypes.POINTER(_I), _P]),
    "mm_match_device": (_I, [_P, _I, _U, _P, _I, _P, ctypes.POINTER(_I), _P]),
    "mm_match_ex": (_I, [_P, _I, _U, _P, _I, _P, ctypes.POINTER(_I), _I, _P]),
    "mm_match_drawn": (_I, [_P, _I, _U, _P, _P, _P, ctypes.POINTER(_I), _P]),
    "mm_match_stats": (_I, [_P, _I, _U, _P, _I, _P, ctypes.POINTER(_I), _P, _I, _I, _P]),
    "mm_matching_weight": (_I, [_P, _P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_LL), _P]),
    "mm_matching_check": (_I, [_P, _P, _P, ctypes.POINTER(_I), _P]),
    "mm_graph_contract": (_I, [_P, _P, ctypes.POINTER(_P), _P]),
    "mm_graph_copy_out": (_I, [_P, _P, _P, _P]),
    "mm_graph_set_batch": (_I, [_P, _I, _P]),
    "mm_match_batch": (_I, [_P, _I, _U, _P, _I, _P, _P, _P]),
    "mm_match_policy": (_I, [_P, _I, _U, _P, _I, _P, ctypes.c_float, _P, ctypes.POINTER(_I), _P, _I, _P]),
    "mm_probe_gather_rate": (_I, [_I, _LL, ctypes.POINTER(ctypes.c_double)]),
    "mm_match_profile": (_I, [_P, _I, _U, _P, _I, _P, ctypes.POINTER(_I), _P, _I, ctypes.POINTER(_I), _P]),
    "mm_match_noalloc": (_I, [_I, _P, _LL, _P, _P, _I, _U, _P, _I, _P, ctypes.POINTER(_I), _P]),
    "mm_debug": (_I, [_I, _LL, ctypes.POINTER(_LL)]),
    "mm_graph_tune": (_I, [_P, _I, _I]),
    "mm_last_error": (ctypes.c_char_p, []),
    "mm_version": (ctypes.c_char_p, []),
}

_GEN_SIGS = {
    "mmg_grid": (_P, [_I, _I]),
    "mmg_rgg": (_P, [_I, ctypes.c_double, ctypes.c_ulonglong, _I]),
    "mmg_rmat": (_P, [_I, _I, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong, _I]),
    "mmg_er": (_P, [_I, ctypes.c_double, ctypes.c_ulonglong, _I]),
    "mmg_n": (_I, [_P]),
    "mmg_nnz": (_LL, [_P]),
    "mmg_ranges": (_P, [_P]),
    "mmg_nbrs": (_P, [_P]),
    "mmg_weights": (_P, [_P]),
    "mmg_free": (None, [_P]),
}


def _load(name: str, sigs: dict) -> ctypes.CDLL:
    if name in _LIBS:
        return _LIBS[name]
    path = PKG / name
    if not path.exists():
        raise OSError(f"{path} is not built; run multicore-matching_b200/build.py")
    lib = ctypes.CDLL(str(path))
    for fn, (res, args) in sigs.items():
        f = getattr(lib, fn)
        f.restype = res
        f.argtypes = args
    _LIBS[name] = lib
    return lib


def lib() -> ctypes.CDLL:
    """The product library (libmmatch.so)."""
    return _load("libmmatch.so", _MM_SIGS)


def genlib() -> ctypes.CDLL:
    return _load("libmmgen.so", _GEN_SIGS)


def mm_symbols() -> list[str]:
    """Every function include/mm_match.h declares (for the export check)."""
    return list(_MM_SIGS)


def _check(status: int) -> None:
    if status != 0:
        raise MatchError(status, lib().mm_last_error().decode(errors="replace"))


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


# --------------------------------------------------------------------------
# host-side graphs


@dataclass
class Graph:
    """CSR graph in the reference's layout: ranges[v] = (begin, end) into nbrs/weights."""

    n: int
    ranges: np.ndarray   # int32 [n, 2]
    nbrs: np.ndarray     # int32 [nnz]
    weights: Optional[np.ndarray] = None  # float32 [nnz] or None (unit)
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.nbrs.shape[0])

    def degrees(self) -> np.ndarray:
        d = self.ranges[:, 1].astype(np.int64) - self.ranges[:, 0]
        return np.maximum(d, 0)

    def contiguous_arrays(self):
        return (np.ascontiguousarray(self.ranges, dtype=np.int32),
                np.ascontiguousarray(self.nbrs, dtype=np.int32),
                None if self.weights is None else np.ascontiguousarray(self.weights, dtype=np.float32))

    @staticmethod
    def from_generated(handle: int, name: str) -> "Graph":
        g = genlib()
        if not handle:
            raise ValueError(f"graph generator failed for {name}")
        try:
            n = g.mmg_n(handle)
            nnz = g.mmg_nnz(handle)
            ranges = np.ctypeslib.as_array(ctypes.cast(g.mmg_ranges(handle), ctypes.POINTER(ctypes.c_int32)),
                                           shape=(max(n, 1) * 2,))[: 2 * n].copy().reshape(n, 2)
            if nnz:
                nbrs = np.ctypeslib.as_array(ctypes.cast(g.mmg_nbrs(handle), ctypes.POINTER(ctypes.c_int32)),
                                             shape=(nnz,)).copy()
                w = np.ctypeslib.as_array(ctypes.cast(g.mmg_weights(handle), ctypes.POINTER(ctypes.c_float)),
                                          shape=(nnz,)).copy()
            else:
                nbrs = np.zeros(0, np.int32)
                w = np.zeros(0, np.float32)
        finally:
            g.mmg_free(handle)
        return Graph(n, ranges, nbrs, w, name)

    @staticmethod
    def grid(width: int, height: int) -> "Graph":
        return Graph.from_generated(genlib().mmg_grid(width, height), f"grid{width}x{height}")

    @staticmethod
    def rgg(n: int, avg_deg: float = 13.0, seed: int = 7, unit: bool = False) -> "Graph":
        return Graph.from_generated(genlib().mmg_rgg(n, avg_deg, seed, int(unit)), f"rgg{n}")

    @staticmethod
    def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1, unit: bool = False) -> "Graph":
        return Graph.from_generated(genlib().mmg_rmat(scale, edge_factor, a, b, c, seed, int(unit)),
                                    f"rmat{scale}")

    @staticmethod
    def er(n: int, avg_deg: float = 8.0, seed: int = 1, unit: bool = False) -> "Graph":
        return Graph.from_generated(genlib().mmg_er(n, avg_deg, seed, int(unit)), f"er{n}")

    def with_pair_weights(self, seed: int = 1) -> "Graph":
        """The same lists with weights in (0, 1] from a hash of the unordered
        endpoint pair, so both entries of an edge carry the same weight."""
        deg = self.degrees()
        owner = np.repeat(np.arange(self.n, dtype=np.uint64), deg)
        r = np.asarray(self.ranges, dtype=np.int64).reshape(-1, 2)
        if self.n and r[0, 0] == 0 and (r[1:, 0] == r[:-1, 1]).all() and r[-1, 1] == self.nnz:
            pos = np.arange(self.nnz, dtype=np.int64)  # contiguous lists
        else:
            pos = np.concatenate([np.arange(b, b + d) for (b, _), d in zip(r, deg)]) if self.n else []
            pos = np.asarray(pos, dtype=np.int64)
        other = self.nbrs[pos].astype(np.uint64)
        lo, hi = np.minimum(owner, other), np.maximum(owner, other)
        x = ((lo << np.uint64(32)) | hi) ^ np.uint64((0x9E3779B97F4A7C15 * (seed + 1)) & 0xFFFFFFFFFFFFFFFF)
        with np.errstate(over="ignore"):
            x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            x ^= x >> np.uint64(31)
        w = np.zeros(self.nnz, dtype=np.float32)
        w[pos] = ((x >> np.uint64(40)).astype(np.float64) + 1.0) / 16777216.0
        return Graph(self.n, self.ranges, self.nbrs, w, self.name)

    @staticmethod
    def union(graphs) -> tuple:
        """Disjoint union of graphs (vertex and entry ids shifted), and the vertex
        offsets of each graph: the input of mm_graph_set_batch."""
        ns = np.array([g.n for g in graphs], dtype=np.int64)
        ms = np.array([g.nnz for g in graphs], dtype=np.int64)
        voff = np.concatenate([[0], np.cumsum(ns)])
        eoff = np.concatenate([[0], np.cumsum(ms)])
        if voff[-1] >= (1 << 31) or eoff[-1] >= (1 << 31):
            raise ValueError("the union exceeds int32 vertex or entry ids")
        ranges = np.empty((int(voff[-1]), 2), dtype=np.int32)
        nbrs = np.empty(int(eoff[-1]), dtype=np.int32)
        weights = np.empty(int(eoff[-1]), dtype=np.float32)
        for g, v0, e0 in zip(graphs, voff[:-1], eoff[:-1]):
            r = np.asarray(g.ranges, dtype=np.int64).reshape(-1, 2)
            ranges[v0:v0 + g.n] = r + e0
            nbrs[e0:e0 + g.nnz] = np.asarray(g.nbrs, dtype=np.int64) + v0
            weights[e0:e0 + g.nnz] = 1.0 if g.weights is None else g.weights
        return Graph(int(voff[-1]), ranges, nbrs, weights, f"union{len(graphs)}"), voff.astype(np.int32)


def rand_seeds(seed: int, count: int = 255) -> np.ndarray:
    """The host rand() values the reference draws per round after srand(seed)
    (bin/match.cpp:382; src/matchgpu.cu:609, 816)."""
    libc = ctypes.CDLL(None)
    libc.srand(ctypes.c_uint(seed))
    libc.rand.restype = ctypes.c_int
    return np.array([libc.rand() for _ in range(count)], dtype=np.uint32)


# --------------------------------------------------------------------------
# device graphs


class DeviceGraph:
    """A graph uploaded to the GPU (mm_graph); the object the GPU matchers own."""

    def __init__(self, g, device: int = -1, with_weights: bool = True):
        ranges = np.ascontiguousarray(np.asarray(g.ranges).reshape(-1, 2), dtype=np.int32)
        nbrs = np.ascontiguousarray(g.nbrs, dtype=np.int32)
        w = None if (g.weights is None or not with_weights) else np.ascontiguousarray(g.weights, dtype=np.float32)
        self._lib = lib()
        h = ctypes.c_void_p()
        _check(self._lib.mm_graph_create(int(g.n), _ptr(ranges), int(nbrs.shape[0]), _ptr(nbrs), _ptr(w), device,
                                         ctypes.byref(h)))
        self.handle = h.value
        self.n = int(g.n)
        self.nnz = int(nbrs.shape[0])

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.mm_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def prepare(self, type_: int) -> None:
        _check(self._lib.mm_graph_prepare(self.handle, type_))

    def match(self, type_: int, seeds: np.ndarray, barrier: int = DEFAULT_BARRIER, stream: int = 0):
        """Host-output matching (mm_match): returns (match int32[n], rounds)."""
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        out = np.empty(max(self.n, 1), dtype=np.int32)
        rounds = ctypes.c_int(0)
        _check(self._lib.mm_match(self.handle, type_, barrier, _ptr(seeds), len(seeds), _ptr(out),
                                  ctypes.byref(rounds), stream or None))
        return out[: self.n], rounds.value

    def match_device(self, type_: int, seeds: np.ndarray, d_out: int, barrier: int = DEFAULT_BARRIER,
                     path: int = PATH_AUTO, stream: int = 0) -> int:
        """Device-output matching into the device pointer d_out; returns rounds."""
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        rounds = ctypes.c_int(0)
        _check(self._lib.mm_match_ex(self.handle, type_, barrier, _ptr(seeds), len(seeds), d_out,
                                     ctypes.byref(rounds), path, stream or None))
        return rounds.value

    def stats(self, type_: int, seeds: np.ndarray, d_out: int, barrier: int = DEFAULT_BARRIER,
              path: int = PATH_AUTO, stream: int = 0):
        """Instrumented run: returns (rounds, int64[rounds, STATS_COLS])."""
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        rounds = ctypes.c_int(0)
        st = np.zeros((255, STATS_COLS), dtype=np.int64)
        _check(self._lib.mm_match_stats(self.handle, type_, barrier, _ptr(seeds), len(seeds), d_out,
                                        ctypes.byref(rounds), _ptr(st), 255, path, stream or None))
        return rounds.value, st[: rounds.value]


    def contract(self, d_match: int, d_cmap: int = 0) -> "DeviceGraph":
        """The coarse graph of the device matching at d_match (mm_graph_contract)."""
        h = ctypes.c_void_p()
        _check(self._lib.mm_graph_contract(self.handle, d_match, ctypes.byref(h), d_cmap or None))
        return DeviceGraph.adopt(h.value, self._lib)

    @classmethod
    def adopt(cls, handle: int, library=None) -> "DeviceGraph":
        """Wrap a graph the library created (it is destroyed with this object)."""
        obj = cls.__new__(cls)
        obj._lib = library or lib()
        obj.handle = handle
        obj.n = int(obj._lib.mm_graph_n(handle))
        obj.nnz = int(obj._lib.mm_graph_nnz(handle))
        return obj

    def to_host(self):
        """(ranges int32[n, 2], neighbours int32[nnz], weights float32[nnz]) copied to the host."""
        r = np.empty((max(self.n, 1), 2), dtype=np.int32)
        nb = np.empty(max(self.nnz, 1), dtype=np.int32)
        w = np.empty(max(self.nnz, 1), dtype=np.float32)
        _check(self._lib.mm_graph_copy_out(self.handle, _ptr(r), _ptr(nb), _ptr(w)))
        return r[: self.n], nb[: self.nnz], w[: self.nnz]

    def tune(self, finish_div: int = 0, blocks_per_sm: int = 0) -> None:
        """Launch options of this graph's matchings (mm_graph_tune); 0 = default."""
        _check(self._lib.mm_graph_tune(self.handle, 1, int(finish_div)))
        _check(self._lib.mm_graph_tune(self.handle, 2, int(blocks_per_sm)))

    def tune_for(self, workload_class: str) -> dict:
        """Apply the autotuner's choice for a workload class (tuned.json, written by
        tune.py); unknown classes keep the defaults.  Returns the choice."""
        import json

        path = PKG / "tuned.json"
        choice = json.loads(path.read_text()).get(workload_class, {}) if path.exists() else {}
        self.tune(choice.get("finish_div", 0), choice.get("blocks_per_sm", 0))
        return choice

    def set_batch(self, offsets: np.ndarray) -> None:
        """Mark the graph as a disjoint union of independent graphs (mm_graph_set_batch)."""
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        _check(self._lib.mm_graph_set_batch(self.handle, len(offsets) - 1, _ptr(offsets)))
        self.ngraphs = len(offsets) - 1

    def match_batch(self, type_: int, seeds: np.ndarray, d_out: int, barrier: int = DEFAULT_BARRIER,
                    stream: int = 0) -> np.ndarray:
        """One launch matching every graph of the batch; returns each graph's rounds."""
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        rounds = np.zeros(self.ngraphs, dtype=np.int32)
        _check(self._lib.mm_match_batch(self.handle, type_, barrier, _ptr(seeds), len(seeds), d_out, _ptr(rounds),
                                        stream or None))
        return rounds

    def match_policy(self, type_: int, seeds: np.ndarray, d_out: int, mlp: np.ndarray, level: float = 0.0,
                     d_trace: int = 0, trace_rounds: int = 0, barrier: int = DEFAULT_BARRIER, stream: int = 0) -> int:
        """Matching with the learned colouring (mm_match_policy); returns rounds."""
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        mlp = np.ascontiguousarray(mlp, dtype=np.float32)
        if mlp.shape != (POLICY_FLOATS,):
            raise ValueError(f"policy weights must be {POLICY_FLOATS} floats")
        rounds = ctypes.c_int(0)
        _check(self._lib.mm_match_policy(self.handle, type_, barrier, _ptr(seeds), len(seeds), _ptr(mlp),
                                         float(level), d_out, ctypes.byref(rounds), d_trace or None, trace_rounds,
                                         stream or None))
        return rounds.value

    def weight(self, d_match: int, stream: int = 0):
        """(weight, size) of the device matching at d_match, as getWeight computes them."""
        wt = ctypes.c_double(0.0)
        sz = ctypes.c_longlong(0)
        _check(self._lib.mm_matching_weight(self.handle, d_match, ctypes.byref(wt), ctypes.byref(sz), stream or None))
        return wt.value, sz.value

    def check(self, d_match: int, stream: int = 0) -> dict:
        """testMatching's counters for the device matching at d_match."""
        counts = np.zeros(5, dtype=np.int64)
        valid = ctypes.c_int(0)
        _check(self._lib.mm_matching_check(self.handle, d_match, _ptr(counts), ctypes.byref(valid), stream or None))
        return {"valid": bool(valid.value), "under": int(counts[0]), "multi": int(counts[1]),
                "invalid": int(counts[2]), "matchable": int(counts[3]), "unmatched": int(counts[4])}

    def profile(self, type_: int, seeds: np.ndarray, d_out: int, barrier: int = DEFAULT_BARRIER, stream: int = 0):
        """Timed run of the round kernel with barrier timestamps.

        Returns (rounds, ms[r, k], launches): one row per round the kernel
        executed, k = 0 window scan (blue preference windows + proposals),
        1 fallback scan of longer lists, 2 commit (commit + recolour +
        compaction), 3 their sum; launches is 1."""
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        rounds = ctypes.c_int(0)
        launches = ctypes.c_int(0)
        ms = np.zeros((255, PROFILE_KERNELS), np.float32)
        _check(self._lib.mm_match_profile(self.handle, type_, barrier, _ptr(seeds), len(seeds), d_out,
                                          ctypes.byref(rounds), _ptr(ms), 255, ctypes.byref(launches),
                                          stream or None))
        executed = int(np.count_nonzero(ms[:, 3] > 0))
        return rounds.value, ms[:executed], launches.value


def shard_batch(sizes, world: int) -> list:
    """Split a batch of independent graphs 0..len(sizes)-1 over `world` GPUs:
    contiguous index ranges [lo, hi), one per rank, of about equal total size
    (sizes: each graph's adjacency entries, or an estimate).  Every rank
    computes the same split from the same sizes, so no message is exchanged,
    and the graphs never cross ranks, so matching needs no collective.  Each
    cut is placed at the graph boundary nearest to its share of the total."""
    if world < 1:
        raise ValueError("world must be at least 1")
    s = np.asarray(sizes, dtype=np.float64).reshape(-1)
    if (s < 0).any() or not np.isfinite(s).all():
        raise ValueError("sizes must be finite and non-negative")
    m = s.size
    cum = np.concatenate([[0.0], np.cumsum(s)])
    bounds = [0]
    for k in range(1, world):
        target = cum[-1] * k / world
        b = min(int(np.searchsorted(cum, target, side="left")), m)
        if b > 0 and target - cum[b - 1] <= cum[b] - target:
            b -= 1
        bounds.append(max(b, bounds[-1]))
    bounds.append(m)
    return [(bounds[k], bounds[k + 1]) for k in range(world)]


def multilevel(g, type_: int, seeds: np.ndarray, target: float = 0.01, device: int = 0,
               barrier: int = DEFAULT_BARRIER, max_levels: int = 64) -> list:
    """Multilevel coarsening: match (type_), contract, repeat until at most
    target * n vertices remain (or a level matches nothing).  Returns one dict per
    level: n, nnz, and for every level but the last rounds, matched vertices,
    weight, valid, maximal, ms_match (device time of the matching) and
    ms_contract."""
    import torch

    levels = []
    dg = DeviceGraph(g, device=device)
    n0 = g.n
    try:
        while True:
            info = {"n": dg.n, "nnz": dg.nnz}
            if dg.n <= target * n0 or len(levels) >= max_levels:
                levels.append(info)
                break
            out = torch.empty(max(dg.n, 1), dtype=torch.int32, device="cuda")
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record()
            rounds = dg.match_device(type_, seeds, out.data_ptr(), barrier)
            b.record()
            coarse = dg.contract(out.data_ptr())
            c.record()
            torch.cuda.synchronize()
            chk = dg.check(out.data_ptr())
            wt, sz = dg.weight(out.data_ptr())
            info.update(rounds=rounds, matched=sz, weight=wt, valid=chk["valid"], maximal=chk["matchable"] == 0,
                        ms_match=a.elapsed_time(b), ms_contract=b.elapsed_time(c))
            levels.append(info)
            stuck = coarse.n == dg.n
            dg.close()
            dg = coarse
            if stuck:
                levels.append({"n": dg.n, "nnz": dg.nnz})
                break
    finally:
        dg.close()
    return levels


def probe_gather_rate(device: int = 0, table_bytes: int = 8 << 20) -> float:
    """Random one-byte gathers per second the device sustains (mm_probe_gather_rate)."""
    rate = ctypes.c_double(0.0)
    _check(lib().mm_probe_gather_rate(device, table_bytes, ctypes.byref(rate)))
    return rate.value


def roofline_bytes(stats: np.ndarray, weighted: bool) -> dict:
    """Algorithmic work of one matching from its per-round counters.

    reference_bytes: the bytes the reference's round loop must move,
        sum_r [24 |A_r| + (4 + 4 w) E_r] with E_r the entries its request and
        respond loops inspect (gathers of match/requests assumed L2-resident).
    window_bytes[r]: the window scan: 32 per blue vertex (worklist item 16,
        reverse key 8, request 8) and per window entry read 8 (weighted:
        neighbour + position) or 4 (random: neighbour).
    fallback_bytes[r]: the fallback scan: (4 + 4 w) per entry and 36 per list
        piece (item 16, proposal 20).
    commit_bytes[r]: the commit phase: 41 per active vertex (item 16,
        request or best key 8, colour 1, next worklist item 16) minus 12 per
        matched vertex (match value 4 written, no next item).
    init_bytes: the set-up pass, 33 per vertex (range 8, colour 1, best key 8,
        worklist item 16), 41 with the weighted types' window offset.
    finish_bytes[r]: the finish phase (round r): 84 per item (worklist item 16,
        record 64, match value 4) and 5 per adjacency entry its list scans read
        (neighbour id 4, colour 1).
    edges: sum_r E_r (edges traversed, for TEPS).
    """
    ew = 8 if weighted else 4
    act = stats[:, ST_ACTIVE].astype(np.float64)
    e = stats[:, ST_REQ_ENTRIES].astype(np.float64) + stats[:, ST_RESP_ENTRIES]
    blue = stats[:, ST_BLUE].astype(np.float64)
    matched = stats[:, ST_MATCHED].astype(np.float64)
    win = stats[:, ST_WINDOW_ENTRIES].astype(np.float64)
    fb = stats[:, ST_STAGED_DEG].astype(np.float64)
    pieces = stats[:, ST_STAGED_ITEMS].astype(np.float64)
    window = 32 * blue + (8 if weighted else 4) * win
    fallback = ew * fb + 36 * pieces
    commit = 41 * act - 12 * matched
    finish = 84 * stats[:, ST_FINISH_ITEMS].astype(np.float64) + 5 * stats[:, ST_FINISH_ENTRIES].astype(np.float64)
    # From the round in which the finish phase completed, the rounds are played
    # inside it: no window, fallback or commit pass runs.  (A called-off attempt
    # is followed by a window scan in the same round.)
    ran = np.nonzero(stats[:, ST_FINISH_ITEMS] > 0)[0]
    if len(ran):
        r = int(ran[-1])
        if not (stats[r:, ST_WINDOW_ENTRIES].any() or stats[r:, ST_STAGED_DEG].any()):
            window[r:] = 0.0
            fallback[r:] = 0.0
            commit[r:] = 0.0
    init = (41 if weighted else 33) * float(act[0]) if len(act) else 0.0
    return {
        "edges": float(e.sum()),
        "reference_bytes": float((24 * act + ew * e).sum()),
        "window_bytes": window,
        "fallback_bytes": fallback,
        "commit_bytes": commit,
        "finish_bytes": finish,
        "init_bytes": init,
        "kernel_bytes": float(window.sum() + fallback.sum() + commit.sum() + finish.sum() + init),
    }


def version() -> str:
    return lib().mm_version().decode()
