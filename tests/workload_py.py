"""Pure-Python restatement of the seeded workload generator.

The product generator lives in the C++ library (lsim_b200/csrc/fsimb_gen.cpp,
reached through lsim_b200.gen).  This module writes the same circuits,
pattern words and collapsed fault lists without loading that library, so
that the benchmark's reference arm can build its inputs while running
nothing but LSIM's own simulator (oracle/_ref) and the CPU oracle.  Every
function mirrors its C++ counterpart step for step (same random stream, same
draws in the same order); tests/test_workload_py.py checks the texts for
equality with lsim_b200.gen.

Test infrastructure only: the product path never imports it.
"""
import numpy as np

_M64 = (1 << 64) - 1
INV, AND, OR, XOR, NAND, NOR, XNOR, MUX, CLKBUF, PI, PO = range(11)


class Rng:
    """xoshiro256** seeded through splitmix64 (fsimb_gen.cpp, struct Rng)."""

    def __init__(self, seed):
        x = seed & _M64
        s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & _M64
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
            s.append(z ^ (z >> 31))
        self.s = s

    def next(self):
        s0, s1, s2, s3 = self.s
        v = (s1 * 5) & _M64
        r = ((((v << 7) | (v >> 57)) & _M64) * 9) & _M64
        t = (s1 << 17) & _M64
        s2 ^= s0
        s3 ^= s1
        s1 ^= s2
        s0 ^= s3
        s2 ^= t
        s3 = ((s3 << 45) | (s3 >> 19)) & _M64
        self.s = [s0, s1, s2, s3]
        return r

    def below(self, n):
        return self.next() % n if n else 0

    def unit(self):
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


def _circuit(n_gates, n_pi, n_po, n_levels, p_fanin3=0.5, type_mask=0x17F, seed=0, window=4,
             hub_frac=0.0, hub_fo=(8, 64), fo_range=(1, 3), p_unused=0.5, shuffle_ids=True):
    """Generator state (fsimb_gen.cpp generate_ckt): gate types, fanins,
    PO drivers and file ids."""
    rng = Rng((seed * 0x100000001B3 + 0x5151) & _M64)
    nPI, nPO, nG = n_pi, n_po, n_gates
    L = max(1, min(n_levels, max(1, nG)))
    nodes = nPI + nG
    lvl_begin = [0] * (L + 2)
    lvl_begin[1] = nPI
    for l in range(1, L + 1):
        sz = nG // L + (1 if l - 1 < nG % L else 0)
        lvl_begin[l + 1] = lvl_begin[l] + sz
    fo = [0] * nodes
    target = [0] * nodes
    hub_mode = hub_frac > 0.0
    if hub_mode:
        for v in range(nodes):
            if rng.unit() < hub_frac:
                target[v] = hub_fo[0] + rng.below(hub_fo[1] - hub_fo[0] + 1)
            else:
                target[v] = fo_range[0] + rng.below(fo_range[1] - fo_range[0] + 1)
    urn = [[] for _ in range(L + 1)]
    unused = [[] for _ in range(L + 1)]

    def add_node(v, l):
        if hub_mode:
            urn[l].extend([v] * target[v])
        else:
            urn[l].append(v)
        unused[l].append(v)

    for i in range(nPI):
        add_node(i, 0)

    def pick_unused(l):
        u = unused[l]
        while u:
            i = rng.below(len(u))
            v = u[i]
            u[i] = u[-1]
            u.pop()
            if fo[v] == 0:
                return v
        return -1

    def pick_urn(lo, hi):
        total = 0
        for l in range(lo, hi + 1):
            total += len(urn[l])
        if total == 0:
            span = lvl_begin[hi + 1] - lvl_begin[lo]
            if span == 0:
                return -1
            return lvl_begin[lo] + rng.below(span)
        r = rng.below(total)
        for l in range(lo, hi + 1):
            ul = urn[l]
            if r < len(ul):
                v = ul[r]
                if hub_mode:
                    ul[r] = ul[-1]
                    ul.pop()
                else:
                    ul.append(v)
                return v
            r -= len(ul)
        return -1

    allowed = [t for t in range(9) if type_mask & (1 << t)] or [AND]
    gtype = [0] * nG
    fanins = [None] * nG
    for l in range(1, L + 1):
        lo = l - window if l > window else 0
        for v in range(lvl_begin[l], lvl_begin[l + 1]):
            g = v - nPI
            t = allowed[rng.below(len(allowed))]
            if t == INV or t == CLKBUF:
                k = 1
            elif t == MUX:
                k = 3
            else:
                k = 3 if rng.unit() < p_fanin3 else 2
            gtype[g] = t
            s = pick_unused(l - 1)
            if s < 0:
                s = pick_urn(l - 1, l - 1)
            chosen = [s & 0xFFFFFFFF]
            for _ in range(1, k):
                c = -1
                attempt = 0
                while attempt < 16 and c < 0:
                    cand = -1
                    if rng.unit() < p_unused:
                        ll = lo
                        while ll < l and cand < 0:
                            cand = pick_unused(ll)
                            ll += 1
                    if cand < 0:
                        cand = pick_urn(lo, l - 1)
                    if (cand & 0xFFFFFFFF) not in chosen:
                        c = cand
                    attempt += 1
                if c < 0:
                    for x in range(lvl_begin[lo], lvl_begin[l]):
                        if x not in chosen:
                            c = x
                            break
                if c < 0:
                    break
                chosen.append(c)
            if t == MUX and len(chosen) < 3:
                gtype[g] = AND
            for q in chosen:
                fo[q] += 1
            fanins[g] = chosen
            add_node(v, l)

    po_drv = []
    taken = bytearray(nodes)
    l = L
    while l >= 1 and len(po_drv) < nPO:
        sinks = [v for v in range(lvl_begin[l], lvl_begin[l + 1]) if fo[v] == 0]
        for i in range(len(sinks), 1, -1):
            j = rng.below(i)
            sinks[i - 1], sinks[j] = sinks[j], sinks[i - 1]
        for v in sinks:
            if len(po_drv) >= nPO:
                break
            po_drv.append(v)
            taken[v] = 1
        if l == 1:
            break
        l -= 1
    l = L
    while l >= 1 and len(po_drv) < nPO:
        for v in range(lvl_begin[l], lvl_begin[l + 1]):
            if len(po_drv) >= nPO:
                break
            if not taken[v]:
                po_drv.append(v)
                taken[v] = 1
        if l == 1:
            break
        l -= 1
    i = 0
    while len(po_drv) < nPO:
        po_drv.append(i % max(1, nPI))
        i += 1
    for i in range(len(po_drv), 1, -1):
        j = rng.below(i)
        po_drv[i - 1], po_drv[j] = po_drv[j], po_drv[i - 1]

    gate_fid = list(range(nPI + nPO, nPI + nPO + nG))
    if shuffle_ids:
        for i in range(len(gate_fid), 1, -1):
            j = rng.below(i)
            gate_fid[i - 1], gate_fid[j] = gate_fid[j], gate_fid[i - 1]
    return dict(n_pi=nPI, n_po=nPO, n_gates=nG, gtype=gtype, fanins=fanins, po_drv=po_drv,
                gate_fid=gate_fid)


def _ckt_text(c):
    nPI, nPO, nG = c["n_pi"], c["n_po"], c["n_gates"]
    gate_fid, gtype, fanins = c["gate_fid"], c["gtype"], c["fanins"]
    Nf = nPI + nPO + nG

    def fid(node):
        return node if node < nPI else gate_fid[node - nPI]

    sinks = [[] for _ in range(Nf)]
    for g in range(nG):
        for k, d in enumerate(fanins[g]):
            pin = k + 1
            if gtype[g] == MUX and pin == 3:
                pin = 5
            sinks[fid(d)].append((gate_fid[g], pin))
    for i, d in enumerate(c["po_drv"]):
        sinks[fid(d)].append((nPI + i, 1))
    n_wires = sum(1 for s in sinks if s)
    ftype = [0] * Nf
    for g in range(nG):
        ftype[gate_fid[g]] = gtype[g]
    out = ["%d\n%d\n%d\n%d\n" % (nPI, nPO, nG, n_wires)]
    for f in range(Nf):
        s = sinks[f]
        if s:
            out.append("%d 0 %d %s\n" % (f, len(s), " ".join("%d %d" % pr for pr in s)))
    out.append(" ".join(str(ftype[f]) for f in range(nPI + nPO, Nf)) + "\n")
    if nG == 0:
        out.append("\n")
    return "".join(out)


def circuit(n_gates, n_pi, n_po, n_levels, p_fanin3=0.5, type_mask=0x17F, seed=0, window=4,
            hub_frac=0.0, hub_fo=(8, 64), fo=(1, 3), p_unused=0.5, shuffle_ids=True):
    """The .ckt text lsim_b200.gen.circuit writes for the same arguments."""
    return _ckt_text(_circuit(n_gates, n_pi, n_po, n_levels, p_fanin3, type_mask, seed, window,
                              hub_frac, hub_fo, fo, p_unused, shuffle_ids))


def pattern_words(n_pi, n_patterns, seed=0, biased_pi_frac=0.0, p_one_biased=0.2, rounds=None):
    """Pattern words [rounds][n_pi] of fsimb_gen.cpp generate_patterns; only
    the first `rounds` rounds (default: all) are drawn."""
    rng = Rng((seed * 0x9E3779B97F4A7C15 + 0x7A7A) & _M64)
    W = (n_patterns + 63) // 64
    R = W if rounds is None else min(W, rounds)
    biased = [rng.unit() < biased_pi_frac for _ in range(n_pi)]
    thr = int(np.floor(p_one_biased * 65536.0 + 0.5))  # std::lround of a non-negative value
    out = np.zeros((R, n_pi), dtype=np.uint64)
    for w in range(R):
        bits = 64 if n_patterns // (64 * (w + 1)) else n_patterns % 64
        mask = _M64 if bits == 64 else (1 << bits) - 1
        row = out[w]
        for b in range(n_pi):
            if not biased[b]:
                v = rng.next()
            else:
                v = 0
                for q in range(16):
                    r = rng.next()
                    for h in range(4):
                        if ((r >> (16 * h)) & 0xFFFF) < thr:
                            v |= 1 << (q * 4 + h)
            row[b] = v & mask
    return out


def collapsed_faults(c, tpg):
    """The collapsed output + input-pin fault list of fsimb_gen.cpp
    build_fault_list (kind 2) for generator state `c`, given the netlist's
    file id -> topological index map `tpg` (from the oracle's reader).
    Returns arrays (site_fid, pin, value) in the list's order."""
    nPI, nPO, nG = c["n_pi"], c["n_po"], c["n_gates"]
    gate_fid, gtype, fanins = c["gate_fid"], c["gtype"], c["fanins"]
    N = nPI + nPO + nG
    tpg = np.asarray(tpg, dtype=np.int64)
    order = np.empty(N, dtype=np.int64)
    order[tpg] = np.arange(N)

    def fid(node):
        return node if node < nPI else gate_fid[node - nPI]

    # fanin lists by topological index, pin order
    typ = np.zeros(N, dtype=np.int64)
    fin = [[] for _ in range(N)]
    for i in range(nPI):
        typ[tpg[i]] = PI
    for g in range(nG):
        e = tpg[gate_fid[g]]
        typ[e] = gtype[g]
        fin[e] = [int(tpg[fid(d)]) for d in fanins[g]]
    for i, d in enumerate(c["po_drv"]):
        e = tpg[nPI + i]
        typ[e] = PO
        fin[e] = [int(tpg[fid(d)])]
    cnt = np.array([len(f) for f in fin], dtype=np.int64)
    fi_off = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(cnt, out=fi_off[1:])
    E = int(fi_off[N])
    fi_idx = np.fromiter((d for f in fin for d in f), dtype=np.int64, count=E)
    fo_cnt = np.bincount(fi_idx, minlength=N)
    owner = np.repeat(np.arange(N), cnt)              # consumer of each fanin entry
    kpos = np.arange(E) - fi_off[owner]               # pin position
    pin_line = np.where(fo_cnt[fi_idx] == 1, fi_idx, N + np.arange(E))
    # equivalences (gates h >= n_pi, POs included)
    t = typ[owner]
    lines_o = owner
    a, b = [], []
    for tt, iv, ov in ((AND, 0, 0), (NAND, 0, 1), (OR, 1, 1), (NOR, 1, 0)):
        m = t == tt
        a.append(2 * pin_line[m] + iv)
        b.append(2 * lines_o[m] + ov)
    for tt, pairs in ((INV, ((0, 1), (1, 0))), (CLKBUF, ((0, 0), (1, 1))), (PO, ((0, 0), (1, 1)))):
        m = (t == tt) & (kpos == 0)
        for iv, ov in pairs:
            a.append(2 * pin_line[m] + iv)
            b.append(2 * lines_o[m] + ov)
    a = np.concatenate(a)
    b = np.concatenate(b)
    n_nodes = 2 * (N + E)
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    g = coo_matrix((np.ones(len(a), dtype=np.int8), (a, b)), shape=(n_nodes, n_nodes))
    _, comp = connected_components(g, directed=False)
    # members: inner-gate outputs and inner-gate input pins
    g0, g1 = nPI, nPI + nG
    gates = np.arange(g0, g1)
    ms, mp, mv, mc = [], [], [], []
    for v in (0, 1):
        ms.append(gates)
        mp.append(np.zeros(len(gates), dtype=np.int64))
        mv.append(np.full(len(gates), v))
        mc.append(comp[2 * gates + v])
    inner = (owner >= g0) & (owner < g1)
    pe = np.nonzero(inner)[0]
    d = fi_idx[pe]
    line = pin_line[pe]
    same = line == d
    site = np.where(same, d, owner[pe])
    pin = np.where(same, 0, kpos[pe] + 1)
    for v in (0, 1):
        ms.append(site)
        mp.append(pin)
        mv.append(np.full(len(pe), v))
        mc.append(comp[2 * line + v])
    ms, mp, mv, mc = (np.concatenate(x) for x in (ms, mp, mv, mc))
    key = (((mp != 0).astype(np.int64) << 40) | (ms << 8) | mp) * 2 + mv
    o = np.lexsort((key, mc))
    first = np.ones(len(o), dtype=bool)
    first[1:] = mc[o][1:] != mc[o][:-1]
    rep = o[first]
    rs, rp, rv = ms[rep], mp[rep], mv[rep]
    o2 = np.lexsort((rv, rp, rs))
    return order[rs[o2]], rp[o2], rv[o2]


def c2_inputs(rounds, n_output_faults):
    """What the reference arm needs of the 200,000-gate workload: the .ckt
    text, the number of faults in its collapsed list, a plain .flst of its
    first `n_output_faults` output faults (the reference's .flst cannot
    express pin faults), pattern words of its first `rounds` rounds, and the
    whole collapsed list as file ids, pins and values."""
    from tests.oracle_lib import Oracle
    c = _circuit(200000, 1000, 1000, 150, p_fanin3=0.6, seed=0)
    ckt = _ckt_text(c)
    o = Oracle(ckt, "0\n", "0\n")
    site, pin, val = collapsed_faults(c, o.tpg())
    out = np.nonzero(pin == 0)[0][:n_output_faults]
    flst = "%d\n%s\n" % (len(out), "\n".join("%d %d" % (site[i], val[i]) for i in out))
    words = pattern_words(1000, 65536, seed=0, rounds=rounds)
    return dict(ckt=ckt, n_faults=len(site), flst=flst, words=words, n_pi=1000, P=65536,
                fault_fids=site, fault_pins=pin, fault_values=val)


def flst_pins(fids, pins, values):
    """An extended (@pins) .flst text of faults given by file id."""
    rows = "\n".join("%d %d %d" % (f, v, p) for f, p, v in zip(fids, pins, values))
    return "@pins\n%d\n%s\n" % (len(fids), rows)
