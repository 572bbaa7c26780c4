"""The device loader's element order (lsim_b200/csrc/fsimb_loader.cu) rests on
one claim: the reference's Kahn FIFO order (fsim/simulation.cpp:718-751) is
the order of waves, and within a wave the order of (position of the
element's last predecessor, index of that predecessor's last edge to it).
This file checks the claim on the CPU, on random graphs with repeated
edges, sources split over several wire lines and edges that skip levels:
a step-for-step mirror of the loader's wave procedure (push with a max key,
count, scan, ordered emit) against a plain Kahn FIFO."""
from collections import deque

import numpy as np
import pytest


def random_netlist(rng, n_pi, n_gates, n_po, max_in=4):
    """Wire lines (source, [sinks]) in file order over ids PIs, POs, gates."""
    N = n_pi + n_po + n_gates
    g0 = n_pi + n_po
    edges = []
    for g in range(g0, N):
        k = int(rng.integers(1, max_in + 1))
        for _ in range(k):
            # any PI or earlier gate: repeated sources give repeated edges
            cand = int(rng.integers(0, n_pi + (g - g0)))
            src = cand if cand < n_pi else g0 + (cand - n_pi)
            edges.append((src, g))
    for p in range(n_pi, n_pi + n_po):
        src = g0 + int(rng.integers(0, n_gates))
        edges.append((src, p))
    order = rng.permutation(len(edges))  # file order of the edges
    lines = []
    for e in order:
        s, d = edges[e]
        if lines and lines[-1][0] == s and rng.random() < 0.7:
            lines[-1][1].append(d)
        else:
            lines.append((s, [d]))  # a source may get several lines
    return N, lines


def kahn_fifo(N, n_pi, n_po, lines):
    adj = [[] for _ in range(N)]
    indeg = [0] * N
    for s, sinks in lines:
        for d in sinks:
            adj[s].append(d)
            indeg[d] += 1
    order = list(range(n_pi))
    head = 0
    while head < len(order):
        u = order[head]
        head += 1
        for v in adj[u]:
            indeg[v] -= 1
            if indeg[v] == 0:
                order.append(v)
    order = [x for x in order if not (n_pi <= x < n_pi + n_po)]
    return order + list(range(n_pi, n_pi + n_po))


def waves(N, n_pi, n_po, lines):
    """Mirror of k_wave_push / k_wave_count / scan / k_wave_emit."""
    # adjacency in insertion order: rank of each line among its source's lines
    outdeg = [0] * N
    for s, sinks in lines:
        outdeg[s] += len(sinks)
    adj_off = np.concatenate([[0], np.cumsum(outdeg)]).astype(np.int64)
    fill = [0] * N
    adj = [0] * int(adj_off[-1])
    indeg = [0] * N
    for s, sinks in lines:
        base = adj_off[s] + fill[s]
        for j, d in enumerate(sinks):
            adj[base + j] = d
            indeg[d] += 1
        fill[s] += len(sinks)
    is_po = lambda v: n_pi <= v < n_pi + n_po  # noqa: E731
    key = [0] * N
    wait = list(indeg)
    pos = [-1] * N
    front = list(range(n_pi))
    for i in range(n_pi):
        pos[i] = i
    base, out = 0, list(front)
    while front:
        n = len(front)
        nbase = base + n
        for i, u in enumerate(front):  # push
            for r in range(adj_off[u], adj_off[u + 1]):
                v = adj[r]
                key[v] = max(key[v], ((base + i) << 32) | (r - adj_off[u]))
                wait[v] -= 1
        cnt = []
        for i, u in enumerate(front):  # count
            c = 0
            for r in range(adj_off[u], adj_off[u + 1]):
                v = adj[r]
                if wait[v] == 0 and key[v] == (((base + i) << 32) | (r - adj_off[u])) and not is_po(v):
                    c += 1
            cnt.append(c)
        offs = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
        nxt = [None] * int(offs[-1])
        for i, u in enumerate(front):  # emit
            o = offs[i]
            for r in range(adj_off[u], adj_off[u + 1]):
                v = adj[r]
                if wait[v] == 0 and key[v] == (((base + i) << 32) | (r - adj_off[u])) and not is_po(v):
                    nxt[o] = v
                    pos[v] = nbase + o
                    o += 1
        out += nxt
        base, front = nbase, nxt
    return out + list(range(n_pi, n_pi + n_po))


@pytest.mark.parametrize("seed", range(40))
def test_wave_order_is_the_kahn_fifo_order(seed):
    rng = np.random.default_rng(seed)
    n_pi = int(rng.integers(1, 12))
    n_gates = int(rng.integers(1, 300))
    n_po = int(rng.integers(1, 10))
    N, lines = random_netlist(rng, n_pi, n_gates, n_po, max_in=int(rng.integers(1, 5)))
    assert waves(N, n_pi, n_po, lines) == kahn_fifo(N, n_pi, n_po, lines)
