"""The allocation-free entry point, mm_match_noalloc, against the default entry.

mm_match_noalloc serves callers that cannot allocate device memory while they
run (cudaMalloc / cudaFree synchronise the device; some callers own a fixed
memory budget).  It keeps its scratch in a fixed device array inside the
library, so this test also checks that a second call in a row -- which finds
the previous call's leftovers in that array -- gives the same answer.
Collected last (file name), so a stop-at-first-failure run has run everything
else before it; it also passes alone in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BARRIER = 0x88B81733


def noalloc(mm, torch, g, type_, seeds, d_ranges, d_nbrs, d_w, barrier=BARRIER, out=None):
    if out is None:
        out = torch.full((max(g.n, 1),), -9, dtype=torch.int32, device="cuda")
    else:
        out.fill_(-9)
    rounds = ctypes.c_int(0)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
    st = mm.lib().mm_match_noalloc(g.n, d_ranges, g.nnz, d_nbrs, d_w, type_, barrier, seeds.ctypes.data,
                                   len(seeds), out.data_ptr(), ctypes.byref(rounds), None)
    torch.cuda.synchronize()
    return st, out[: g.n].cpu().numpy(), rounds.value


def test_noalloc_entry_matches_default_entry(mm, orc):
    import torch

    assert torch.cuda.is_available()
    torch.cuda.set_device(0)
    graphs = [mm.Graph.rgg(1 << 14, 13.0, seed=7), mm.Graph.grid(200, 150), mm.Graph.rmat(14, 16, seed=4)]
    for g in graphs:
        ranges = torch.from_numpy(np.ascontiguousarray(g.ranges, dtype=np.int32)).cuda()
        nbrs = torch.from_numpy(g.nbrs).cuda()
        w = torch.from_numpy(g.weights).cuda()
        with mm.DeviceGraph(g, device=0) as dg:
            for seed in (1, 12345):
                seeds = mm.rand_seeds(seed, 255)
                for t in mm.TYPES:
                    want = torch.empty(g.n, dtype=torch.int32, device="cuda")
                    want_rounds = dg.match_device(t, seeds, want.data_ptr())
                    torch.cuda.synchronize()
                    want = want.cpu().numpy()
                    out = torch.empty(max(g.n, 1), dtype=torch.int32, device="cuda")
                    for call in range(2):  # two calls in a row share the fixed scratch
                        torch.cuda.synchronize()
                        free0 = torch.cuda.mem_get_info()[0]
                        st, got, rounds = noalloc(mm, torch, g, t, seeds, ranges.data_ptr(), nbrs.data_ptr(),
                                                  w.data_ptr(), out=out)
                        if call == 1:  # after the first call the array is in place: nothing more is taken
                            assert torch.cuda.mem_get_info()[0] == free0, (g.name, t, seed)
                        assert st == 0, mm.lib().mm_last_error()
                        assert rounds == want_rounds, (g.name, t, seed, call)
                        assert np.array_equal(got, want), (g.name, t, seed, call, int((got != want).sum()))


def test_noalloc_limits_and_errors(mm):
    import torch

    torch.cuda.set_device(0)
    lib = mm.lib()
    seeds = mm.rand_seeds(1, 255)
    r = ctypes.c_int(0)
    # beyond the fixed scratch: a clear status, nothing launched
    st = lib.mm_match_noalloc((1 << 20) + 1, 1, 0, None, None, 7, BARRIER, seeds.ctypes.data, 255, 1,
                              ctypes.byref(r), None)
    assert st == 5 and b"exceeds the fixed scratch" in lib.mm_last_error()
    # an invalid graph is rejected before any matching kernel reads it
    ranges = torch.tensor([[0, 2], [2, 3], [3, 3]], dtype=torch.int32, device="cuda")
    nbrs = torch.tensor([1, 7, 0], dtype=torch.int32, device="cuda")
    out = torch.empty(3, dtype=torch.int32, device="cuda")
    st = lib.mm_match_noalloc(3, ranges.data_ptr(), 3, nbrs.data_ptr(), None, 7, BARRIER, seeds.ctypes.data, 255,
                              out.data_ptr(), ctypes.byref(r), None)
    assert st == 2
    # ranges are read as int2 pairs: a misaligned view is refused before any kernel runs
    wide = torch.zeros(8, dtype=torch.int32, device="cuda")
    st = lib.mm_match_noalloc(3, wide.data_ptr() + 4, 3, nbrs.data_ptr(), None, 7, BARRIER, seeds.ctypes.data, 255,
                              out.data_ptr(), ctypes.byref(r), None)
    assert st == 1 and b"8-byte aligned" in lib.mm_last_error()
