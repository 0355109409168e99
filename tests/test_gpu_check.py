"""GPU validator and weight (mm_matching_check / mm_matching_weight) against the
oracle's restatement of the reference's testMatching and getWeight
(src/matchcpu.cu:64-97, 127-246), on real matchings and on invalid ones built
on the host (singletons, triples, pairs that are not neighbours, corrupt values)."""
from __future__ import annotations

import numpy as np
import pytest

from graphs_small import random_graph

pytestmark = pytest.mark.gpu

BARRIER = 0x88B81733
WEIGHT_RTOL = 1e-12  # the device sums in a fixed tree, the reference in vertex order


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _device_check(mm, torch, dg, m):
    d = torch.from_numpy(np.ascontiguousarray(m, dtype=np.int32)).cuda()
    chk = dg.check(d.data_ptr())
    wt, sz = dg.weight(d.data_ptr())
    torch.cuda.synchronize()
    return chk, wt, sz


def _compare(mm, orc, torch, g, dg, m):
    chk, wt, sz = _device_check(mm, torch, dg, m)
    want = orc.check(g, m)
    for k in ("valid", "under", "multi", "invalid", "matchable"):
        assert chk[k] == want[k], (k, chk, want)
    assert chk["unmatched"] == int((np.asarray(m) < 4).sum())
    w_want, s_want = orc.weight(g, m)
    assert sz == s_want
    if np.isnan(w_want) or np.isinf(w_want):  # adversarial weights: NaN / inf propagate alike
        assert (np.isnan(wt) and np.isnan(w_want)) or wt == w_want
    else:
        assert wt == pytest.approx(w_want, rel=WEIGHT_RTOL, abs=1e-9)


def _corruptions(m, n, rng):
    """Invalid variants of a matching: each breaks it in one of testMatching's ways."""
    out = []
    matched = np.nonzero(m >= 4)[0]
    unmatched = np.nonzero(m < 4)[0]
    if len(matched) >= 2:
        x = m.copy()  # a singleton: one vertex of a pair loses its partner
        x[matched[0]] = 1
        out.append(x)
        x = m.copy()  # a triple: an unmatched vertex joins a pair's value
        if len(unmatched):
            x[unmatched[0]] = m[matched[0]]
            out.append(x)
        x = m.copy()  # two pairs swap a partner: values shared by non-neighbours likely
        a, b = matched[0], matched[-1]
        x[a], x[b] = m[b], m[a]
        out.append(x)
    x = m.copy()  # random corruption of a few values, including large ones
    idx = rng.choice(n, size=min(n, 7), replace=False)
    x[idx] = rng.integers(-3, n + 10, size=len(idx))
    out.append(x)
    x = m.copy()  # two unmatched neighbours forced to one value (valid if adjacent)
    if len(unmatched) >= 2:
        x[unmatched[:2]] = 4 + int(unmatched[:2].min())
        out.append(x)
    return out


def test_check_and_weight_match_oracle(mm, orc, torch_cuda):
    rng = np.random.default_rng(5)
    graphs = [mm.Graph.grid(64, 64), mm.Graph.rgg(1 << 13, 13.0, seed=7), mm.Graph.rmat(13, 16, seed=3),
              mm.Graph.er(1 << 12, 8.0, seed=2)]
    for g in graphs:
        seeds = orc.rand_seeds(12345, 256)
        with mm.DeviceGraph(g, device=0) as dg:
            for t in mm.TYPES:
                m, _, _ = orc.match(g, t, seeds, BARRIER)
                _compare(mm, orc, torch_cuda, g, dg, m)
                for x in _corruptions(m, g.n, rng):
                    _compare(mm, orc, torch_cuda, g, dg, x)


def test_check_on_unsorted_and_asymmetric_graphs(mm, orc, torch_cuda):
    rng = np.random.default_rng(9)
    for seed in range(6):
        g = random_graph(np.random.default_rng(seed), 200 + 50 * seed, 6.0, symmetric=seed % 3 != 0,
                         gaps=seed % 2 == 1, shuffle_ranges=seed % 3 == 1, sort_lists=seed % 2 == 0)
        seeds = orc.rand_seeds(seed + 1, 256)
        with mm.DeviceGraph(g, device=0) as dg:
            for t in (7, 9):
                m, _, _ = orc.match(g, t, seeds, BARRIER)
                _compare(mm, orc, torch_cuda, g, dg, m)
                for x in _corruptions(m, g.n, rng):
                    _compare(mm, orc, torch_cuda, g, dg, x)


def test_check_full_size_rgg(mm, orc, torch_cuda):
    g = mm.Graph.rgg(1 << 20, 13.0, seed=7)
    seeds = orc.rand_seeds(12345, 256)
    with mm.DeviceGraph(g, device=0) as dg:
        out = torch_cuda.empty(g.n, dtype=torch_cuda.int32, device="cuda")
        dg.match_device(9, seeds, out.data_ptr())
        chk = dg.check(out.data_ptr())
        wt, sz = dg.weight(out.data_ptr())
        torch_cuda.cuda.synchronize()
    m = out.cpu().numpy()
    want = orc.check(g, m)
    assert chk["valid"] and chk["matchable"] == 0 == want["matchable"]
    w_want, s_want = orc.weight(g, m)
    assert sz == s_want and wt == pytest.approx(w_want, rel=WEIGHT_RTOL)


def test_check_arguments_are_statuses(mm, torch_cuda):
    g = mm.Graph.grid(4, 4)
    with mm.DeviceGraph(g, device=0) as dg:
        assert dg._lib.mm_matching_check(dg.handle, None, None, None, None) == 1  # MM_ERR_ARG
        assert dg._lib.mm_matching_weight(dg.handle, None, None, None, None) == 1
