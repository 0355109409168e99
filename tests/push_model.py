"""Sequential Python model of the push-path round loop (design check only).

It restates, one vertex at a time, what the CUDA kernels of
multicore-matching_b200/csrc/mm_push.cu compute: reverse proposal keys,
blue-only scans with atomic-max proposals, commit by key comparison and the
select of the next round fused into the commit.  tests/test_push_model.py runs
it against the oracle on small adversarial graphs, so the reformulation is
checked on the CPU before any kernel runs.
"""
from __future__ import annotations

import struct

import numpy as np

M32 = 0xFFFFFFFF


def weight_order(w: float) -> int:
    u = struct.unpack("<I", struct.pack("<f", w))[0]
    if u == 0x80000000:
        u = 0
    return (~u & M32) if (u & 0x80000000) else (u | 0x80000000)


def cand_key(j: int, w: float, weighted: bool) -> int:
    if weighted:
        return ((weight_order(w) << 32) | (~j & M32)) if w > -1.0 else 0
    return ~j & M32


def reverse_keys(n, ranges, nbrs, w, weighted):
    """revkey[(v, j)] for every adjacency slot of every owner v."""
    rk = {}
    for v in range(n):
        b, e = int(ranges[v, 0]), int(ranges[v, 1])
        for j in range(b, e):
            t = int(nbrs[j])
            if t == v:
                rk[(v, j)] = 0
                continue
            best = 0
            tb, te = int(ranges[t, 0]), int(ranges[t, 1])
            for p in range(tb, te):
                if int(nbrs[p]) == v:
                    best = max(best, cand_key(p, float(w[p]), weighted))
            rk[(v, j)] = best
    return rk


def reverse_keys_sorted(n, ranges, nbrs, w, weighted, chunk=2048):
    """The binary-search build of k_chunk_owner + k_revkey_sorted, index for index:
    slots numbered by the degree prefix, owners found per chunk (in a table of at most
    chunk + 1 prefixes, else by search between the chunk's owner bounds); of the two
    entries of a pair only the one whose partner list is shorter (ties by id)
    searches it, stores the best key of the run it finds and max-combines its own
    key into the run's entries.  Returns the keys by (owner, entry) or None when
    some list has a descending pair."""
    deg = np.maximum(ranges[:, 1] - ranges[:, 0], 0).astype(np.int64)
    contiguous = bool(n > 0 and ranges[0, 0] == 0 and np.all(ranges[:, 1] >= ranges[:, 0])
                      and np.all(ranges[1:, 0] == ranges[:-1, 1]) and ranges[-1, 1] == len(nbrs))
    slot_off = np.concatenate([[0], np.cumsum(deg)[:-1]]) if n else np.zeros(0, np.int64)
    S = int(deg.sum())

    def prefix(v):
        return int(ranges[v, 0]) if contiguous else int(slot_off[v])

    def owner_of(lo, hi, s):
        while lo < hi:
            mid = (lo + hi + 1) >> 1
            if prefix(mid) <= s:
                lo = mid
            else:
                hi = mid - 1
        return lo

    chunks = (S + chunk - 1) // chunk
    chunk_v = [owner_of(0, n - 1, min(c * chunk, S - 1)) for c in range(chunks + 1)]
    rk, bad = {}, False
    pulled, pushed = set(), set()  # the kernel stores pulls plainly: no slot may be in both
    for c in range(chunks):
        s0 = c * chunk
        v0, v1 = chunk_v[c], chunk_v[c + 1]
        cnt = v1 - v0 + 1
        pre = [prefix(v0 + i) - s0 for i in range(cnt)] if cnt <= chunk + 1 else None
        for k in range(chunk):
            s = s0 + k
            if s >= S:
                break
            if pre is not None:
                lo, hi = 0, cnt - 1
                while lo < hi:
                    mid = (lo + hi + 1) >> 1
                    if pre[mid] <= k:
                        lo = mid
                    else:
                        hi = mid - 1
                v = v0 + lo
            else:
                v = owner_of(v0, v1, s)
            pos = s if contiguous else int(ranges[v, 0]) + (s - int(slot_off[v]))
            assert ranges[v, 0] <= pos < ranges[v, 1]
            u = int(nbrs[pos])
            if pos + 1 < ranges[v, 1] and nbrs[pos + 1] < u:
                bad = True
            rk.setdefault((v, pos), 0)
            if u == v:
                continue
            dv, du = int(deg[v]), int(deg[u])
            if du > dv or (du == dv and u > v):
                continue  # u's entries search v's list and push into this slot
            lo, hi = int(ranges[u, 0]), int(ranges[u, 0]) + du
            while lo < hi:
                mid = (lo + hi) >> 1
                if nbrs[mid] < v:
                    lo = mid + 1
                else:
                    hi = mid
            mine = cand_key(pos, float(w[pos]), weighted)
            key, q = 0, lo
            while q < int(ranges[u, 0]) + du and nbrs[q] == v:
                key = max(key, cand_key(q, float(w[q]), weighted))
                if mine:
                    rk[(u, q)] = max(rk.get((u, q), 0), mine)
                    pushed.add((u, q))
                q += 1
            pulled.add((v, pos))
            if key:
                rk[(v, pos)] = key
    assert not (pulled & pushed)
    return None if bad else rk


def is_symmetric(n, ranges, nbrs, w, weighted):
    """The upload test of the symmetric path: contiguous ranges in vertex order,
    strictly increasing lists, and the entries (v, u[, w]) are those (u, v[, w])
    transposed."""
    if n == 0 or ranges[0, 0] != 0 or ranges[-1, 1] != len(nbrs):
        return False
    if np.any(ranges[:, 1] < ranges[:, 0]) or np.any(ranges[1:, 0] != ranges[:-1, 1]):
        return False
    ent = {}
    for v in range(n):
        lst = [int(x) for x in nbrs[ranges[v, 0]:ranges[v, 1]]]
        if any(b <= a for a, b in zip(lst, lst[1:])):
            return False
        for j in range(int(ranges[v, 0]), int(ranges[v, 1])):
            key = (v, int(nbrs[j]))
            ent[key] = np.float32(w[j]).tobytes() if weighted else b""
    return all(ent.get((u, v)) == x for (v, u), x in ent.items())


FIN_SINGLE, FIN_MEMBER, FIN_ROOT = 1, 2, 3


def finish_model(n, ranges, nbrs, w, weighted, maximal, cap, seeds, barrier, colour_hash, col, match, active, t,
                 lim):
    """The finish phase of the round kernel (mm_push.cu: finish_classify,
    fin_search, finish_resolve, fin_play) at the start of round t, vertex by
    vertex.  col holds the colours of round t; match the final values of the
    vertices no longer active.  Returns the rounds executed, with match filled
    in for every active vertex, or None if the attempt is called off (then
    nothing has changed)."""
    BLUE, RED, DEAD, MATCHED = 0, 1, 2, 3

    def lst(x):
        return range(int(ranges[x, 0]), max(int(ranges[x, 1]), int(ranges[x, 0])))

    def search(v):
        mem, ents = [v], []  # ents: (owner slot, target slot, preference key)
        f = 0
        while f < len(mem):
            x = mem[f]
            js = lst(x)
            if len(js) > lim["maxdeg"]:
                return "big", None
            rows = [list(js)[i:i + 32] for i in range(0, len(js), 32)]
            for row in rows:
                cs = [col[int(nbrs[j])] for j in row]
                if any(c == DEAD for c in cs):
                    return "big", None
                if any(c <= RED and int(nbrs[j]) < v for j, c in zip(row, cs)):
                    return "notroot", None
                for j, c in zip(row, cs):
                    if c > RED:
                        continue
                    u = int(nbrs[j])
                    if u in mem:
                        slot = mem.index(u)
                    else:
                        if len(mem) == lim["members"]:
                            return "big", None
                        slot = len(mem)
                        mem.append(u)
                    if len(ents) == lim["entries"]:
                        return "big", None
                    # a weight that can never be picked still marks an unmatched neighbour (key 1)
                    ents.append((f, slot, (cand_key(j, float(w[j]), weighted) or 1) if weighted else (~j & M32)))
            f += 1
        return "root", (mem, ents)

    # pass 1: classify, search the root candidates' components
    cls = {}
    for v in active:
        js = lst(v)
        if len(js) > lim["maxdeg"]:
            return None
        cs = [col[int(nbrs[j])] for j in js]
        if any(c == DEAD for c in cs):
            return None
        inner = [int(nbrs[j]) for j, c in zip(js, cs) if c <= RED]
        cls[v] = FIN_SINGLE if not inner else (FIN_MEMBER if min(inner) < v else FIN_ROOT)
    for v in active:
        if cls[v] == FIN_ROOT and search(v)[0] == "big":
            return None
    # pass 2: resolve
    last_all = -1
    for v in active:
        if cls[v] == FIN_SINGLE:
            blue, r, last = col[v] == BLUE, t, t
            while True:
                last = r
                if blue:
                    match[v] = 2
                    break
                r += 1
                if r >= cap:
                    match[v] = 1
                    break
                blue = colour_hash(v, int(seeds[r])) < barrier
            last_all = max(last_all, last)
        elif cls[v] == FIN_ROOT:
            res, comp = search(v)
            if res != "root":
                continue
            mem, ents = comp
            k = len(mem)
            act, val, blue, last = [True] * k, [0] * k, [False] * k, [-1] * k
            r = t
            while r < cap and any(act):
                for l in range(k):
                    if act[l]:
                        blue[l] = colour_hash(mem[l], int(seeds[r])) < barrier
                        last[l] = r
                st = [(BLUE if blue[l] else RED) if act[l] else (DEAD if val[l] == 2 else MATCHED) for l in range(k)]
                best, choice, crk, got = [0] * k, [0] * k, [0] * k, [0] * k
                for l in range(k):
                    if not (act[l] and blue[l]):
                        continue
                    for (o, tg, pref) in ents:
                        if o != l:
                            continue
                        key = pref if st[tg] == RED else (0 if st[tg] == MATCHED else 1)
                        if key > best[l]:
                            best[l], choice[l] = key, tg
                    if best[l] >= 2:
                        crk[l] = (((best[l] >> 32) << 32) | (~mem[l] & M32)) if weighted else (~mem[l] & M32)
                        got[choice[l]] = max(got[choice[l]], crk[l])
                done = [False] * k
                for l in range(k):
                    if not act[l]:
                        continue
                    if blue[l]:
                        if best[l] >= 2 and (got[choice[l]] & M32) == (crk[l] & M32):
                            val[l] = 4 + min(mem[l], mem[choice[l]])
                            done[l] = True
                        elif best[l] == 0:
                            val[l] = 2
                            done[l] = True
                    elif got[l]:
                        val[l] = 4 + min(mem[l], ~got[l] & M32)
                        done[l] = True
                for l in range(k):
                    if done[l]:
                        act[l] = False
                r += 1
            for l in range(k):
                match[mem[l]] = (0 if blue[l] else 1) if act[l] else val[l]
            last_all = max(last_all, max(last))
    return min(last_all + 2, cap) if maximal else cap


def push_match(g, type_, seeds, barrier, colour_hash, finish=None, isolated=False):
    """finish: None, or the finish phase's limits {div, members, entries, maxdeg}.
    isolated: on the symmetric path, resolve the vertices without neighbours at
    set-up, as the round kernel does (each leaves in the first round in which it
    is blue, or stays red to the cap; the last round in which one is active
    joins the round count), instead of carrying them through the rounds."""
    n = g.n
    ranges = np.asarray(g.ranges)
    nbrs = np.asarray(g.nbrs)
    w = np.ones(len(nbrs), np.float32) if g.weights is None else np.asarray(g.weights, np.float32)
    weighted = type_ in (8, 9)
    maximal = type_ in (7, 9)
    cap = 255 if maximal else 20
    rk = reverse_keys(n, ranges, nbrs, w, weighted)
    BLUE, RED, DEAD, MATCHED = 0, 1, 2, 3
    col = [BLUE if colour_hash(v, int(seeds[0])) < barrier else RED for v in range(n)]
    match = [None] * n
    active = list(range(n))
    best = [0] * n
    rounds = None
    t = 0
    symmetric = is_symmetric(n, ranges, nbrs, w, weighted)
    sym = finish is not None and symmetric
    iso_last = -1
    if isolated and symmetric:
        lim = min(cap, len(seeds))
        keep = []
        for v in active:
            if int(ranges[v, 1]) > int(ranges[v, 0]):
                keep.append(v)
                continue
            r, blue = 0, col[v] == BLUE
            while not blue and r + 1 < lim:
                r += 1
                blue = colour_hash(v, int(seeds[r])) < barrier
            if blue:
                match[v], last = 2, r
            else:
                match[v], last = 1, (cap - 1 if lim == cap else lim)
            iso_last = max(iso_last, last)
        active = keep

    def with_isolated(r):
        return max(r, min(iso_last + 2, cap)) if maximal and iso_last >= 0 else r

    act0 = len(active)
    fin_next = act0
    while True:
        if sym and t > 0 and active and len(active) * finish["div"] <= act0 and len(active) <= fin_next:
            r = finish_model(n, ranges, nbrs, w, weighted, maximal, cap, seeds, barrier, colour_hash, col, match,
                             active, t, finish)
            if r is not None:
                out = np.zeros(n, np.int32)
                for v in range(n):
                    out[v] = match[v] if match[v] is not None else col[v]
                return out, with_isolated(r)
            fin_next = len(active) // 2
        # phase A: blue vertices scan and propose
        req = {}
        dead = set()
        for v in active:
            if col[v] != BLUE:
                continue
            b, e = int(ranges[v, 0]), int(ranges[v, 1])
            alive = 0
            key = 0
            for j in range(b, e):
                c = col[int(nbrs[j])]
                alive |= c != MATCHED
                if c == RED:
                    key = max(key, cand_key(j, float(w[j]), weighted))
                    if not weighted:
                        break
            if not alive:
                col[v] = DEAD
                match[v] = 2
                dead.add(v)
            elif key == 0:
                req[v] = (-2, 0)
            else:
                j = ~key & M32
                tgt = int(nbrs[j])
                r = rk[(v, j)]
                if r:
                    best[tgt] = max(best[tgt], r)
                req[v] = (tgt, r & M32)
        # phase B: commit, recolour, compact
        has_next = t + 1 < cap
        nxt = []
        for v in active:
            if v in dead:
                continue
            if col[v] == BLUE:
                tgt, lo = req[v]
                if lo and (best[tgt] & M32) == lo:
                    match[v] = 4 + min(v, tgt)
                    col[v] = MATCHED
                    continue
            else:  # red
                k = best[v]
                if k:
                    u = int(nbrs[~k & M32])
                    match[v] = 4 + min(v, u)
                    col[v] = MATCHED
                    continue
            nxt.append(v)
        # colours of the next round only after every commit of this round
        if has_next:
            for v in nxt:
                col[v] = BLUE if colour_hash(v, int(seeds[t + 1])) < barrier else RED
        active = nxt
        if not (has_next and active):
            rounds = min(t + 2, cap) if (maximal and not active) else cap
            break
        t += 1
    out = np.zeros(n, np.int32)
    for v in range(n):
        out[v] = match[v] if match[v] is not None else col[v]
    return out, with_isolated(rounds)
