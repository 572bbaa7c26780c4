"""Seeded synthetic workloads in LSIM's .ckt / .flst / .ptn formats.

The generator (lsim_b200/csrc/fsimb_gen.cpp) builds levelized combinational
DAGs: gates spread evenly over the levels, types drawn uniformly from the
allowed set, fan-in 2-3 (1 for NOT/BUF, 3 for MUX), inputs from at most
``window`` levels back with preferential attachment, the first input always
from the previous level; POs are driven by sink gates of the top levels.

``WORKLOADS`` holds the benchmark configurations:
  c1  2,000 gates, 64 PI / 64 PO, 30 levels, SA0/SA1 on every gate output
      (4,000 faults), 4,096 uniform patterns (seed 0);
  c2  200,000 gates, 1,000 PI / 1,000 PO, 150 levels, mean fan-in 2.2,
      SA0/SA1 on every gate output and input pin collapsed by equivalence,
      65,536 uniform patterns;
  c3  2,000,000 gates, 5,000 PI / 5,000 PO, 400 levels, 10% of gates with a
      fanout target of 8-64 (the rest 1-3), SA0/SA1 on every gate output
      (4,000,000 faults), 16,384 patterns with half of the PIs at P(1) = 0.2.

``batch_configs`` draws the batched configuration (c4): circuits with gate
counts log-uniform in 500-50,000, 10-120 levels, SA0/SA1 on every gate
output and 1,024-16,384 uniform patterns each.
"""
import ctypes

from . import _lib

# GateType numbering (fsim/base_ppg.hpp:19-32)
INV, AND, OR, XOR, NAND, NOR, XNOR, MUX, CLKBUF = range(9)
BENCH_TYPES = (1 << AND) | (1 << OR) | (1 << NAND) | (1 << NOR) | (1 << XOR) | (1 << XNOR) | \
    (1 << INV) | (1 << CLKBUF)
ALL_TYPES = BENCH_TYPES | (1 << MUX)
FAULT_KINDS = {"outputs": 0, "pins": 1, "collapsed": 2}

WORKLOADS = {
    "c1": dict(n_gates=2000, n_pi=64, n_po=64, n_levels=30, p_fanin3=0.5, seed=0,
               n_patterns=4096, faults="outputs"),
    "c2": dict(n_gates=200000, n_pi=1000, n_po=1000, n_levels=150, p_fanin3=0.6, seed=0,
               n_patterns=65536, faults="collapsed"),
    # c2 shape (same level width, fan-in and fault model), 50,000 gates, one
    # 2,048-pattern tile: the profiling case for the sweep kernel
    "c2s": dict(n_gates=50000, n_pi=1000, n_po=1000, n_levels=38, p_fanin3=0.6, seed=0,
                n_patterns=2048, faults="collapsed"),
    "c3": dict(n_gates=2000000, n_pi=5000, n_po=5000, n_levels=400, p_fanin3=0.6, seed=0,
               n_patterns=16384, faults="outputs", hub_frac=0.1, biased_pi_frac=0.5,
               p_one_biased=0.2),
}


def circuit(n_gates, n_pi, n_po, n_levels, p_fanin3=0.5, type_mask=BENCH_TYPES, seed=0,
            window=4, hub_frac=0.0, hub_fo=(8, 64), fo=(1, 3), p_unused=0.5, shuffle_ids=True):
    cfg = _lib.GenConfig(ctypes.sizeof(_lib.GenConfig), seed, n_gates, n_pi, n_po, n_levels,
                         window, p_fanin3, type_mask, hub_frac, hub_fo[0], hub_fo[1], fo[0], fo[1],
                         p_unused, 1 if shuffle_ids else 0)
    ptr, n = ctypes.c_void_p(), ctypes.c_size_t()
    _lib.check(_lib.lib().fsimb_gen_circuit(ctypes.byref(cfg), ctypes.byref(ptr), ctypes.byref(n)))
    return _lib.take_text(ptr, n)


def faults(ckt, kind="outputs"):
    b = ckt.encode()
    ptr, n = ctypes.c_void_p(), ctypes.c_size_t()
    _lib.check(_lib.lib().fsimb_gen_faults(b, len(b), FAULT_KINDS[kind], ctypes.byref(ptr),
                                           ctypes.byref(n)))
    return _lib.take_text(ptr, n)


def patterns(n_pi, n_patterns, seed=0, biased_pi_frac=0.0, p_one_biased=0.2):
    ptr, n = ctypes.c_void_p(), ctypes.c_size_t()
    _lib.check(_lib.lib().fsimb_gen_patterns(seed, n_patterns, n_pi, biased_pi_frac, p_one_biased,
                                             ctypes.byref(ptr), ctypes.byref(n)))
    return _lib.take_text(ptr, n)


def generate(n_gates, n_pi, n_po, n_levels, n_patterns, faults="outputs", seed=0,
             p_fanin3=0.5, type_mask=BENCH_TYPES, window=4, hub_frac=0.0, biased_pi_frac=0.0,
             p_one_biased=0.2, pattern_seed=None):
    """Returns {'ckt', 'flst', 'ptn'} texts for one seeded workload."""
    ckt = circuit(n_gates, n_pi, n_po, n_levels, p_fanin3=p_fanin3, type_mask=type_mask,
                  seed=seed, window=window, hub_frac=hub_frac)
    fl = globals()["faults"](ckt, faults)
    pt = patterns(n_pi, n_patterns, seed=seed if pattern_seed is None else pattern_seed,
                  biased_pi_frac=biased_pi_frac, p_one_biased=p_one_biased)
    return {"ckt": ckt, "flst": fl, "ptn": pt}


def workload(name, **overrides):
    cfg = dict(WORKLOADS[name])
    cfg.update(overrides)
    return generate(**cfg)


def batch_configs(n_circuits=256, seed=0, gates=(500, 50000), levels=(10, 120),
                  patterns=(1024, 16384), faults="outputs", type_mask=BENCH_TYPES):
    """Per-circuit ``generate`` arguments of a batch, drawn from ``seed``.

    Gate counts are log-uniform in ``gates``, levels uniform in ``levels``
    (at most a quarter of the gate count), pattern counts uniform in
    ``patterns``; PIs and POs are a 32nd of the gates, 16-1,000."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_circuits):
        g = int(round(np.exp(rng.uniform(np.log(gates[0]), np.log(gates[1])))))
        lv = int(rng.integers(levels[0], levels[1] + 1))
        lv = max(2, min(lv, g // 4))
        io = int(min(1000, max(16, g // 32)))
        P = int(rng.integers(patterns[0], patterns[1] + 1))
        out.append(dict(n_gates=g, n_pi=io, n_po=io, n_levels=lv, p_fanin3=0.5,
                        seed=seed * 100003 + i + 1, n_patterns=P, faults=faults,
                        type_mask=type_mask))
    return out


def serve_configs(n_circuits=32, seed=0, gates=(1000, 500000), levels=(20, 150)):
    """Resident circuits of the serving configuration (c5): gate counts
    log-uniform in ``gates``, levels uniform in ``levels`` but at least one
    level per 1,500 gates (the level width of the 200k-gate configuration is
    1,333) and at most a quarter of the gates, PIs and POs a 32nd of the
    gates (16-1,000); SA0/SA1 on every gate output and input pin, collapsed."""
    import numpy as np
    rng = np.random.default_rng(seed + 7919)
    out = []
    for i in range(n_circuits):
        g = int(round(np.exp(rng.uniform(np.log(gates[0]), np.log(gates[1])))))
        lv = max(int(rng.integers(levels[0], levels[1] + 1)), -(-g // 1500))
        lv = max(2, min(lv, g // 4))
        io = int(min(1000, max(16, g // 32)))
        out.append(dict(n_gates=g, n_pi=io, n_po=io, n_levels=lv, p_fanin3=0.6,
                        seed=seed * 100003 + 5000 + i, faults="collapsed"))
    return out


def opentimer_dump(n_cells, n_pi, seed=0, loops=0, window=8, fanout_free=False, layers=None,
                   cell_types=None, pins=None):
    """Seeded OpenTimer-style netlist dump (the input of
    lsim_b200.opentimer.convert) over the cells of its pin table.

    Cells are created in order; each input comes from a PI or an earlier
    cell, drawn from the last ``window`` signals with probability 0.8, so
    that paths are deep.  ``fanout_free``: every signal drives at most one
    sink (the PI count bounds the cell count).  ``layers``: cells spread
    over that many layers, every input from the layer just before (layer 0
    being the PIs).  ``loops``: that many cells take one input -- a DFF's D,
    or the last input of a multi-input cell -- from a later cell (in
    ``layers`` mode from a later layer), which closes a cycle or adds an
    edge against the creation order.  Every signal left without a sink
    drives its own PO.  Names are fixed-width (pi*, po*, g*) so that no name
    is a prefix of another.  Edges, including the arcs inside each cell, are
    listed in a seeded random order.  ``pins``: the pin table to draw cells
    from (default: the converter's PIN_TABLE)."""
    import numpy as np
    from .opentimer import PIN_TABLE
    rng = np.random.default_rng(seed)
    table = PIN_TABLE if pins is None else pins
    kinds = sorted(table) if cell_types is None else list(cell_types)
    lib = {}
    for k in kinds:
        pins = table[k]
        ins = sorted((p for p in pins if pins[p] > 0), key=lambda p: pins[p])
        out = next(p for p in pins if pins[p] == 0)
        lib[k] = (k if k.endswith("X1") else k + "_X1", ins, out)
    pis = ["pi%05d" % i for i in range(n_pi)]
    cells = []  # (name, kind, [signal per input pin, None = loop input])
    layer_of = []
    sig = [(p, p) for p in pis]  # (source name in edges, element name)
    pool = list(range(len(sig)))  # signals without a sink (fanout-free mode)
    if layers:
        bounds = [0, n_pi] + [n_pi + (n_cells * (l + 1)) // layers for l in range(layers)]
    n_loop = 0
    for c in range(n_cells):
        name = "g%06d" % c
        kind = kinds[int(rng.integers(len(kinds)))]
        if fanout_free and len(pool) < len(lib[kind][1]) + (n_loop < loops):
            fits = [k for k in kinds if len(lib[k][1]) <= len(pool)]
            if not fits:
                break
            kind = fits[int(rng.integers(len(fits)))]
        n_in = len(lib[kind][1])
        want_loop = n_loop < loops and n_in >= 2 and rng.random() < 0.5
        src = []
        if layers:
            lay = next(l for l in range(layers) if n_pi + c < bounds[l + 2])
            lo, hi = bounds[lay], bounds[lay + 1]
            for _ in range(n_in):
                j = lo + int(rng.integers(hi - lo))
                while j in src and hi - lo > len(src):
                    j = lo + (j - lo + 1) % (hi - lo)
                src.append(j)
            want_loop = want_loop and lay + 1 < layers
            layer_of.append(lay)
        elif fanout_free:
            for _ in range(n_in):
                j = int(rng.integers(len(pool)))
                src.append(pool[j])
                pool[j] = pool[-1]
                pool.pop()
        else:
            for _ in range(n_in):
                if rng.random() < 0.8:
                    j = len(sig) - 1 - int(rng.integers(min(window, len(sig))))
                else:
                    j = int(rng.integers(len(sig)))
                while j in src:
                    j = (j + 1) % len(sig)
                src.append(j)
        if want_loop and c + 1 < n_cells:
            k = 0 if kind == "DFF" else n_in - 1
            if fanout_free:
                pool.append(src[k])
            src[k] = None
            n_loop += 1
        cells.append((name, kind, src))
        sig.append((name + ":" + lib[kind][2], name))
        pool.append(len(sig) - 1)
    used = set(s for _, _, src in cells for s in src if s is not None)
    for ci, (name, kind, src) in enumerate(cells):
        for k, s in enumerate(src):
            if s is not None:
                continue
            if layers:
                first = bounds[layer_of[ci] + 2] - n_pi
                cand = list(range(n_pi + first, n_pi + len(cells)))
            else:
                cand = list(range(n_pi + ci + 1, n_pi + len(cells)))
            if fanout_free:
                cand = [x for x in cand if x not in used]
            if not cand:  # no later cell free: a PI of its own
                pis.append("pi%05d" % len(pis))
                sig.append((pis[-1], pis[-1]))
                cand = [len(sig) - 1]
            s = cand[int(rng.integers(len(cand)))]
            src[k] = s
            used.add(s)
    # ids: PIs first (added PIs renumber nothing: sig keeps its indices)
    po_src = [s for s in range(len(sig)) if s not in used and ":" in sig[s][0]]
    pos = ["po%05d" % i for i in range(len(po_src))]
    edges = []
    for name, kind, src in cells:
        _, ins, out = lib[kind]
        for pin, s in zip(ins, src):
            edges.append((sig[s][0], name + ":" + pin))
            if not (kind == "DFF" and pin == "D"):
                edges.append((name + ":" + pin, name + ":" + out))
    for po, s in zip(pos, po_src):
        edges.append((sig[s][0], po))
    order = rng.permutation(len(edges))
    lines = ["module top;", "// Start PIs"] + ["input %s;" % p for p in pis] + [""]
    lines += ["// Start POs"] + ["output %s;" % p for p in pos] + [""]
    lines += ["// Start wires"] + ["wire n%s;" % name[1:] for name, _, _ in cells] + [""]
    lines += ["// Start cells"]
    for name, kind, src in cells:
        cell, ins, out = lib[kind]
        conn = ", ".join([".%s(%s)" % (p, sig[s][1]) for p, s in zip(ins, src)] +
                         [".%s(n%s)" % (out, name[1:])])
        lines.append("%s %s ( %s );" % (cell, name, conn))
    lines += ["endmodule", "", "digraph TimingGraph {"]
    lines += ['  "%s" -> "%s";' % edges[i] for i in order]
    lines += ["}", ""]
    return "\n".join(lines)
