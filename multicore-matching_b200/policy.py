"""Learned colouring policy: trace collection, training and evaluation.

The reference colours every vertex blue with one probability, the select
barrier (0x88B81733 / 2^32 = 0.534, bin/match.cpp:183).  mm_match_policy lets a
per-vertex MLP (6 -> 16 -> 1) choose that probability from local features
(FEATURES below), and on graphs with symmetric structure retires, from round 3
on, a red vertex of at most 128 entries as soon as none of its neighbours is
unmatched, instead of waiting until it is coloured blue.

Training has two stages.

1. Off-policy, from traces of the plain colouring.  The plain method is a
   logged randomised experiment: every vertex's colour is a coin flip of known
   probability p0.  So a policy's expected number of vertices leaving the
   active set per round can be estimated by inverse propensity weighting,

       J(pi) = mean over traced (vertex, round) of  y * (pi(x) / p0  if blue,
                                                         (1 - pi(x)) / (1 - p0) if red)

   with y = 1 if the vertex left the active set in that round (matched, or
   retired as unmatchable).  The estimate holds every other vertex's colour at
   the plain policy's, which stops being true once all vertices move at once,
   so the fit is kept in a trust region around p0 (|pi - p0| <= delta).
2. On-policy refinement: evolution strategies on the quantity that matters,
   the total rounds of the learned colouring over the training hierarchies,
   with a penalty once the matching weight falls more than 0.5% below the
   plain method's.

The plain method stays the fallback and the yardstick: evaluate() reports
rounds, time and matching weight of the plain method, of the policy kernel
with the constant plain probability (the effect of early retirement alone) and
of the learned policy on the same graphs.

Used offline only: the trained weights are a 129-float blob (policy_mlp.f32
next to this file) that mm_match_policy reads.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

FEATURES = ("log2(1+degree)", "previous role (0 red, 0.5 blue unproposed, 1 blue lost)", "max incident weight",
            "mean incident weight", "min(round, 32)/32", "level/16")
N_FEAT, N_HID = 6, 16
N_FLOATS = N_HID * N_FEAT + N_HID + N_HID + 1  # W1[16][6], b1[16], W2[16], b2
HERE = Path(__file__).resolve().parent
WEIGHTS = HERE / "policy_mlp.f32"
P0 = 0x88B81733 / 4294967296.0
# the kernel clamps the blue probability to [1/16, 15/16]
P_MIN, P_MAX = 1 / 16, 15 / 16


def constant_policy(p: float = P0) -> np.ndarray:
    """Weights of the policy that colours every vertex blue with probability p."""
    w = np.zeros(N_FLOATS, dtype=np.float32)
    w[-1] = np.float32(np.log(p / (1.0 - p)))
    return w


def hand_built(feature: int, k: float, centre: float = 0.0) -> np.ndarray:
    """Weights of the policy p = sigmoid(logit(p0) + k * (x[feature] - centre)) for
    a non-negative feature (one hidden unit passes it through): e.g. feature 0
    (log2(1 + degree)) splits neighbours of different degree, feature 4 (the
    round) makes a schedule.  For probing what the colouring can change."""
    w = np.zeros(N_FLOATS, dtype=np.float32)
    w[feature] = 1.0                   # W1[0][feature]: hidden 0 = relu(x[feature])
    w[N_HID * N_FEAT + N_HID] = k      # W2[0]
    w[-1] = np.float32(np.log(P0 / (1.0 - P0)) - k * centre)
    return w


def load_policy(path: Path = WEIGHTS) -> np.ndarray:
    w = np.fromfile(path, dtype=np.float32)
    if w.shape != (N_FLOATS,):
        raise ValueError(f"{path}: {w.size} floats, expected {N_FLOATS}")
    return w


def make_net(torch):
    return torch.nn.Sequential(torch.nn.Linear(N_FEAT, N_HID), torch.nn.ReLU(), torch.nn.Linear(N_HID, 1))


def _get(net) -> np.ndarray:
    l1, l2 = net[0], net[2]
    parts = [l1.weight, l1.bias, l2.weight.reshape(-1), l2.bias]
    return np.concatenate([p.detach().cpu().numpy().reshape(-1) for p in parts]).astype(np.float32)


def _set(net, flat):
    import torch

    l1, l2 = net[0], net[2]
    off = 0
    for p in (l1.weight, l1.bias, l2.weight, l2.bias):
        k = p.numel()
        p.data.copy_(torch.tensor(flat[off:off + k], dtype=torch.float32).reshape(p.shape))
        off += k


def policy_prob(mlp: np.ndarray, X: np.ndarray) -> np.ndarray:
    """The policy's blue probability (numpy, as the kernel computes it)."""
    W1 = mlp[:N_HID * N_FEAT].reshape(N_HID, N_FEAT)
    b1 = mlp[N_HID * N_FEAT:N_HID * N_FEAT + N_HID]
    W2 = mlp[N_HID * N_FEAT + N_HID:N_HID * N_FEAT + 2 * N_HID]
    b2 = mlp[-1]
    out = np.maximum(X @ W1.T + b1, 0) @ W2 + b2
    return np.clip(1 / (1 + np.exp(-out)), P_MIN, P_MAX)


def collect(mm, dg, type_, seeds, mlp, level, max_rounds=64):
    """Run the policy on a device graph with tracing; returns (X, colour, y, rounds)."""
    import torch

    n = dg.n
    tr = torch.full((max_rounds * n * 8,), float("nan"), dtype=torch.float32, device="cuda")
    out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    rounds = dg.match_policy(type_, seeds, out.data_ptr(), mlp, level, tr.data_ptr(), max_rounds)
    t = tr.view(max_rounds, n, 8)
    t = t[: min(rounds, max_rounds)].reshape(-1, 8)
    t = t[~torch.isnan(t[:, 6])]
    return t[:, :6].cpu().numpy(), t[:, 6].cpu().numpy(), t[:, 7].cpu().numpy(), rounds


def fit_ips(X, c, y, prop, delta=0.2, steps=2000, lr=3e-3, seed=0, device="cuda"):
    """Stage 1: maximise the inverse-propensity estimate of vertices leaving per
    round, with the policy kept within delta of the plain probability p0 (a
    quadratic penalty outside).  prop: the logging policy's blue probability
    per sample."""
    import torch

    torch.manual_seed(seed)
    net = make_net(torch).to(device)
    _set(net, constant_policy())
    Xt = torch.tensor(X, dtype=torch.float32, device=device)
    ct = torch.tensor(c, dtype=torch.float32, device=device)
    yt = torch.tensor(y, dtype=torch.float32, device=device)
    pt = torch.tensor(prop, dtype=torch.float32, device=device).clamp(P_MIN, P_MAX)
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    batch = min(len(X), 1 << 18)
    for _ in range(steps):
        idx = torch.randint(0, len(X), (batch,), device=device)
        pi = torch.sigmoid(net(Xt[idx]).squeeze(1)).clamp(P_MIN, P_MAX)
        w = torch.where(ct[idx] > 0.5, pi / pt[idx], (1 - pi) / (1 - pt[idx]))
        outside = torch.relu((pi - P0).abs() - delta)
        loss = -(yt[idx] * w).mean() + 100.0 * (outside * outside).mean()
        opt.zero_grad()
        loss.backward()
        opt.step()
    return _get(net)


def es_refine(objective, w0, iters=40, pairs=12, sigma=0.05, lr=0.03, seed=0, log=None):
    """Stage 2: antithetic evolution strategies with rank-shaped fitness and
    Adam steps, maximising objective(weights) from w0.  Returns the final
    search centre and the best single candidate (the latter is partly luck:
    choose between them on held-out seeds)."""
    rng = np.random.default_rng(seed)
    w = w0.astype(np.float64)
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    best_w, best_f = w0.copy(), objective(w0)
    for it in range(iters):
        eps = rng.standard_normal((pairs, w.size))
        cand = np.concatenate([w + sigma * eps, w - sigma * eps]).astype(np.float32)
        f = np.array([objective(c) for c in cand])
        k = int(np.argmax(f))
        if f[k] > best_f:
            best_f, best_w = float(f[k]), cand[k].copy()
        ranks = np.empty(len(f))
        ranks[np.argsort(f)] = np.arange(len(f))
        shaped = ranks / (len(f) - 1) - 0.5
        grad = ((shaped[:pairs] - shaped[pairs:])[:, None] * eps).sum(0) / (pairs * sigma)
        m = 0.9 * m + 0.1 * grad
        v = 0.999 * v + 0.001 * grad * grad
        w = w + lr * (m / (1 - 0.9 ** (it + 1))) / (np.sqrt(v / (1 - 0.999 ** (it + 1))) + 1e-8)
        if log:
            log(f"es {it}: mean {f.mean():.4f} best {best_f:.4f}")
    return w.astype(np.float32), best_w.astype(np.float32)


def hierarchy(mm, g, type_, seeds, target=0.01, min_shrink=0.05, max_levels=64, device=0):
    """Host copies of the plain method's multilevel hierarchy: the graph and its
    coarse levels down to target * n vertices, or until a level removes fewer
    than min_shrink of its vertices (graphs with many isolated vertices, such as
    R-MAT, stall above the target), at most max_levels coarse levels."""
    import torch

    graphs = [g]
    dg = mm.DeviceGraph(g, device=device)
    try:
        while dg.n > target * g.n and len(graphs) <= max_levels:
            out = torch.empty(max(dg.n, 1), dtype=torch.int32, device="cuda")
            dg.match_device(type_, seeds, out.data_ptr())
            coarse = dg.contract(out.data_ptr())
            stalled = coarse.n > (1.0 - min_shrink) * dg.n
            dg.close()
            dg = coarse
            r, nb, w = dg.to_host()
            graphs.append(mm.Graph(dg.n, r, nb, w, f"{g.name}-L{len(graphs)}"))
            if stalled:
                break
    finally:
        dg.close()
    return graphs


def evaluate(mm, graphs, type_, seeds, mlp, repeats=5, device=0):
    """Plain (mm_match_device), the policy kernel at the plain probability, and
    the learned colouring on the same graphs: rounds, device time (ms, best of
    repeats) and matching weight per level."""
    import torch

    arms = (("plain", None), ("retire", constant_policy()), ("learned", mlp))
    rows = []
    for level, g in enumerate(graphs):
        with mm.DeviceGraph(g, device=device) as dg:
            dg.prepare(type_)
            out = torch.empty(max(g.n, 1), dtype=torch.int32, device="cuda")
            res = {}
            for name, w in arms:
                best = 1e30
                for _ in range(repeats):
                    a = torch.cuda.Event(enable_timing=True)
                    b = torch.cuda.Event(enable_timing=True)
                    a.record()
                    if w is None:
                        r = dg.match_device(type_, seeds, out.data_ptr())
                    else:
                        r = dg.match_policy(type_, seeds, out.data_ptr(), w, float(level))
                    b.record()
                    torch.cuda.synchronize()
                    best = min(best, a.elapsed_time(b))
                chk = dg.check(out.data_ptr())
                wt, sz = dg.weight(out.data_ptr())
                res[name] = {"rounds": r, "ms": best, "weight": wt, "matched": sz, "valid": chk["valid"],
                             "maximal": chk["matchable"] == 0}
            rows.append({"level": level, "n": g.n, "nnz": g.nnz, **res})
    return rows
