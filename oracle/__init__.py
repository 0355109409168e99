"""Oracle -- TEST INFRASTRUCTURE ONLY.

The CPU checker for the CUDA matching path.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline legs may import this package; the product
(multicore-matching_b200, libmmatch.so) never does and has no CPU fallback.

Two layers:
  * ``libmm_oracle.so`` (oracle/mm_oracle.c): plain-C restatement of the
    reference GPU round loop, src/matchgpu.cu:184-851, with per-round counters.
  * ``_ref/libmmref.so`` / ``_ref/libmmref20.so``: the reference's OWN
    src/graph.cu, src/matchcpu.cu and src/matchtbb.cu compiled by
    oracle/Makefile (TBB matchers 10/11 = GPU types 7/9; the 20-round build =
    GPU types 6/8; sequential matchers 0/4/5 for the CPU baseline).  Built only
    where the reference sources exist; on other machines the .so files that
    were built next to the sources are used if present.

Parity of the restatement is pinned by tests/test_oracle.py against the
reference build and against the fixtures in tests/golden/.
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
STATS_COLS = 9  # MMO_ST_COLS of mm_oracle.c
(ST_ACTIVE, ST_BLUE, ST_RED, ST_REQ_ENTRIES, ST_RESP_ENTRIES, ST_BLUE_DEG, ST_RED_DEG, ST_MATCHED,
 ST_DEAD) = range(9)

_P, _I, _LL, _U = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_uint32
_cache: dict = {}


def _load(path: Path, sigs: dict) -> ctypes.CDLL:
    key = str(path)
    if key not in _cache:
        if not path.exists():
            raise OSError(f"{path} is not built (make -C oracle)")
        lib = ctypes.CDLL(key)
        for fn, (res, args) in sigs.items():
            f = getattr(lib, fn)
            f.restype = res
            f.argtypes = args
        _cache[key] = lib
    return _cache[key]


def lib() -> ctypes.CDLL:
    return _load(HERE / "libmm_oracle.so", {
        "mmo_colour_hash": (_U, [_U, _U]),
        "mmo_match": (_I, [_I, _P, _P, _P, _I, _U, _P, _I, _P, _P, _I, _I]),
        "mmo_rand_seeds": (None, [_U, _I, _P]),
        "mmo_weight": (None, [_I, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_LL)]),
        "mmo_check": (_I, [_I, _P, _P, _P, _P]),
    })


_REF_SIGS = {
    "mmref_run": (_I, [_I, _I, _P, _LL, _P, _P, _U, _U, _I, _P, ctypes.POINTER(ctypes.c_double),
                       ctypes.POINTER(_U)]),
    "mmref_check": (_I, [_I, _P, _LL, _P, _P, _P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_LL)]),
    "mmref_check_counts": (_I, [_I, _P, _LL, _P, _P, _P, _P]),
    "mmref_read": (_I, [ctypes.c_char_p, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_LL), _P, _P,
                        _P]),
    "mmref_cli": (_I, [ctypes.c_char_p, _I, _I, _U, _U, _I, _I, _P, ctypes.POINTER(_U)]),
    "mmref_shuffle": (_I, [ctypes.c_char_p, _I, _U, _I, _P, _P, ctypes.POINTER(_U)]),
}


def ref_available() -> bool:
    return (HERE / "_ref" / "libmmref.so").exists() and (HERE / "_ref" / "libmmref20.so").exists()


def ref_lib(fixed_rounds: bool = False) -> ctypes.CDLL:
    name = "libmmref20.so" if fixed_rounds else "libmmref.so"
    return _load(HERE / "_ref" / name, _REF_SIGS)


def _arrays(g):
    ranges = np.ascontiguousarray(g.ranges, dtype=np.int32)
    nbrs = np.ascontiguousarray(g.nbrs, dtype=np.int32)
    w = None if g.weights is None else np.ascontiguousarray(g.weights, dtype=np.float32)
    return ranges, nbrs, w


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def colour_hash(v: int, seed: int) -> int:
    return int(lib().mmo_colour_hash(v, seed))


def rand_seeds(seed: int, count: int = 255) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint32)
    lib().mmo_rand_seeds(seed, count, _p(out))
    return out


def match(g, type_: int, seeds: np.ndarray, barrier: int, nthreads: int = 0):
    """Restated GPU matching: returns (match int32[n], rounds, stats int64[rounds, 9])."""
    ranges, nbrs, w = _arrays(g)
    if type_ in (8, 9) and w is None:
        w = np.ones(len(nbrs), dtype=np.float32)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
    out = np.zeros(max(g.n, 1), dtype=np.int32)
    stats = np.zeros((256, STATS_COLS), dtype=np.int64)
    rounds = lib().mmo_match(g.n, _p(ranges), _p(nbrs), _p(w), type_, barrier, _p(seeds), len(seeds),
                             _p(out), _p(stats), 256, nthreads)
    if rounds < 0:
        raise ValueError("oracle: not enough seeds")
    return out[: g.n], rounds, stats[:rounds]


def check(g, m: np.ndarray) -> dict:
    """Validity and maximality counters (testMatching, src/matchcpu.cu:127-246)."""
    ranges, nbrs, _ = _arrays(g)
    m = np.ascontiguousarray(m, dtype=np.int32)
    out = np.zeros(4, dtype=np.int64)
    ok = lib().mmo_check(g.n, _p(ranges), _p(nbrs), _p(m), _p(out))
    return {"valid": bool(ok), "under": int(out[0]), "multi": int(out[1]), "invalid": int(out[2]),
            "matchable": int(out[3])}


def weight(g, m: np.ndarray):
    """(weight, size) as getWeight computes them (src/matchcpu.cu:64-97)."""
    ranges, nbrs, w = _arrays(g)
    m = np.ascontiguousarray(m, dtype=np.int32)
    wt = ctypes.c_double(0)
    sz = ctypes.c_longlong(0)
    lib().mmo_weight(g.n, _p(ranges), _p(nbrs), _p(w), _p(m), ctypes.byref(wt), ctypes.byref(sz))
    return wt.value, sz.value


def ref_run(g, type_: int, barrier: int, seed: int, nthreads: int = 0, fixed_rounds: bool = False):
    """Run the reference's own matcher `type_` (0, 4, 5, 10, 11) after srand(seed).

    Returns (match int32[n], ms, next rand() value)."""
    ranges, nbrs, w = _arrays(g)
    out = np.zeros(max(g.n, 1), dtype=np.int32)
    ms = ctypes.c_double(0)
    nxt = ctypes.c_uint32(0)
    rc = ref_lib(fixed_rounds).mmref_run(type_, g.n, _p(ranges), g.nnz, _p(nbrs), _p(w), barrier, seed,
                                         nthreads, _p(out), ctypes.byref(ms), ctypes.byref(nxt))
    if rc != 0:
        raise ValueError(f"reference matcher type {type_} unavailable")
    return out[: g.n], ms.value, nxt.value


def ref_check(g, m: np.ndarray):
    """The reference's testMatching + getWeight: (valid, weight, size)."""
    ranges, nbrs, w = _arrays(g)
    m = np.ascontiguousarray(m, dtype=np.int32)
    wt = ctypes.c_double(0)
    sz = ctypes.c_longlong(0)
    ok = ref_lib().mmref_check(g.n, _p(ranges), g.nnz, _p(nbrs), _p(w), _p(m), ctypes.byref(wt),
                               ctypes.byref(sz))
    return bool(ok), wt.value, sz.value


def ref_check_counts(g, m: np.ndarray) -> dict:
    """The reference's own testMatching counters (src/matchcpu.cu:127-246), as it prints them."""
    ranges, nbrs, w = _arrays(g)
    m = np.ascontiguousarray(m, dtype=np.int32)
    out = np.full(4, -1, dtype=np.int64)
    ok = ref_lib().mmref_check_counts(g.n, _p(ranges), g.nnz, _p(nbrs), _p(w), _p(m), _p(out))
    return {"valid": bool(ok), "under": int(out[0]), "multi": int(out[1]), "invalid": int(out[2]),
            "matchable": int(out[3])}


def _is_mtx(path) -> int:
    return 1 if str(path).endswith(".mtx") else 0


def ref_read(path):
    """The reference's Graph::readMETIS / readMatrixMarket (src/graph.cu:86-511) on `path`
    (MatrixMarket when it ends in .mtx).  Returns (n, nrEdges, ranges[n,2], nbrs, weights)
    or None when the reader threw."""
    n, e, nnz = _I(0), _I(0), _LL(0)
    p = str(path).encode()
    rc = ref_lib().mmref_read(p, _is_mtx(path), ctypes.byref(n), ctypes.byref(e), ctypes.byref(nnz), None, None, None)
    if rc == 2:
        return None
    if rc != 0:
        raise OSError(f"cannot open {path}")
    ranges = np.zeros((n.value, 2), dtype=np.int32)
    nbrs = np.zeros(nnz.value, dtype=np.int32)
    w = np.zeros(nnz.value, dtype=np.float32)
    ref_lib().mmref_read(p, _is_mtx(path), ctypes.byref(n), ctypes.byref(e), ctypes.byref(nnz), _p(ranges), _p(nbrs),
                         _p(w))
    return n.value, e.value, ranges, nbrs, w


def ref_shuffle(path, seed: int, reps: int, n: int, nnz: int):
    """srand(seed) and `reps` reference Graph::random_shuffle calls (src/graph.cu:513-548).
    Returns (ranges[n,2], nbrs, next rand() value)."""
    ranges = np.zeros((max(n, 1), 2), dtype=np.int32)
    nbrs = np.zeros(max(nnz, 1), dtype=np.int32)
    nxt = _U(0)
    rc = ref_lib().mmref_shuffle(str(path).encode(), _is_mtx(path), seed, reps, _p(ranges), _p(nbrs),
                                 ctypes.byref(nxt))
    if rc != 0:
        raise ValueError(f"reference shuffle failed ({rc})")
    return ranges[:n], nbrs[:nnz], nxt.value


# GPU type -> (reference TBB matcher, fixed-round build): the TBB matchers run the
# same colour/request/respond/match rounds (src/matchtbb.cu) as the GPU types.
GPU_TO_TBB = {6: (10, True), 7: (10, False), 8: (11, True), 9: (11, False)}


def ref_cli(path, gpu_type: int, barrier: int, seed: int, shuffle: bool, reps: int, n: int):
    """The reference CLI loop (bin/match.cpp:380-420) with the TBB matcher that equals
    GPU type `gpu_type`.  Returns (matches int32[reps, n], next rand() value)."""
    tbb, fixed = GPU_TO_TBB[gpu_type]
    out = np.zeros((reps, max(n, 1)), dtype=np.int32)
    nxt = _U(0)
    rc = ref_lib(fixed).mmref_cli(str(path).encode(), _is_mtx(path), tbb, barrier, seed, int(shuffle), reps,
                                  _p(out), ctypes.byref(nxt))
    if rc != 0:
        raise ValueError(f"reference CLI loop failed ({rc})")
    return out[:, :n], nxt.value
