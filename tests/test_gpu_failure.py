"""Failure handling without any GPU fault.

* A grid-barrier wait that runs out: block 0 leaves one barrier out (testing
  hook MM_DEBUG_SKIP_BARRIER) and the waits are bounded by a small poll limit
  (MM_DEBUG_SPIN_LIMIT), so every block gives up and returns.  The call must
  report MM_ERR_DEVICE, and the same graph object must then give the
  reference's matching.  This covers the round kernel's barriers and the
  finish kernel's.
* Out of device memory: an allocation limit on the library's pool
  (MM_DEBUG_ALLOC_LIMIT) makes graph creation and the first matching fail with
  MM_ERR_NOMEM, leaving no allocation behind (MM_DEBUG_POOL_USED), and the
  library works normally once the limit is lifted.

The reference's only guards are its error exits (src/matchgpu.cu:45-50,
481-482) and the round cap (src/matchgpu.cu:604).
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BARRIER = 0x88B81733
SPIN, SKIP, ALLOC, USED = 1, 2, 3, 4


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.set_device(0)
    return torch


def debug(mm, key, value=0):
    out = ctypes.c_longlong(0)
    assert mm.lib().mm_debug(key, value, ctypes.byref(out)) == 0
    return out.value


def test_barrier_wait_that_runs_out(mm, orc, torch_cuda):
    g = mm.Graph.rgg(1 << 14, 13.0, seed=5)
    seeds = orc.rand_seeds(12345, 256)
    want, rounds, _ = orc.match(g, 9, seeds, BARRIER)
    with mm.DeviceGraph(g, device=0) as dg:
        out = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
        _, st = dg.stats(9, seeds, out.data_ptr())
        fin = np.nonzero(st[:, mm.ST_FINISH_ITEMS] > 0)[0]
        assert len(fin) >= 1  # the round at which the finish kernel took over
        # after round 1's window scan (round kernel); after the finish kernel's first pass
        for mark in (4, 3 * int(fin[-1]) + 1):
            debug(mm, SPIN, 1 << 12)
            debug(mm, SKIP, mark)
            try:
                with pytest.raises(mm.MatchError) as e:
                    dg.match(9, seeds)
                assert e.value.status == 7, mark  # MM_ERR_DEVICE
            finally:
                debug(mm, SKIP, -1)
                debug(mm, SPIN, 0)
            got, r = dg.match(9, seeds)
            assert r == rounds and np.array_equal(got, want), mark


def test_out_of_memory_leaves_nothing_behind(mm, orc, torch_cuda):
    g = mm.Graph.rmat(14, 16, seed=3)
    seeds = orc.rand_seeds(7, 256)
    want, rounds, _ = orc.match(g, 9, seeds, BARRIER)
    used0 = debug(mm, USED)
    debug(mm, ALLOC, used0)  # no new device memory at all
    try:
        with pytest.raises(mm.MatchError) as e:
            mm.DeviceGraph(g, device=0)
        assert e.value.status == 4  # MM_ERR_NOMEM
    finally:
        debug(mm, ALLOC, -1)
    assert debug(mm, USED) == used0
    with mm.DeviceGraph(g, device=0) as dg:
        used1 = debug(mm, USED)
        debug(mm, ALLOC, used1)  # the graph is in place; its first matching needs more
        try:
            with pytest.raises(mm.MatchError) as e:
                dg.match(9, seeds)
            assert e.value.status == 4
        finally:
            debug(mm, ALLOC, -1)
        assert debug(mm, USED) == used1
        got, r = dg.match(9, seeds)
        assert r == rounds and np.array_equal(got, want)
    assert debug(mm, USED) == used0
