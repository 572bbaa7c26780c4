"""Netlist import (lsim_b200.opentimer, the job of fsim/parser.py) against the
reference converter's recorded outputs, plus properties of the loop
breaking, and the converted netlists through the reader, the oracle and
(marked gpu) the GPU path."""
import json
import os
import subprocess
import sys
from collections import deque

import numpy as np
import pytest

from lsim_b200 import Simulator, gen, opentimer
from tests.conftest import GOLDEN, ROOT
from tests.oracle_lib import Oracle, Reference, ref_available

needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built here")

with open(os.path.join(GOLDEN, "opentimer_ref.json")) as _f:
    _FIX = json.load(_f)
DUMPS_REF = _FIX["dumps"]
REF = [dict(c, dump=DUMPS_REF[c["name"]]) for c in _FIX["cases"]]
COMPAT = [dict(c, dump=DUMPS_REF[c["name"]]) for c in _FIX["compat"]]


def canonical(ckt):
    ls = ckt.strip("\n").split("\n")
    n = int(ls[3])
    wires = []
    for line in ls[4:4 + n]:
        v = [int(x) for x in line.split()]
        assert len(v) == 3 + 2 * v[2]
        wires.append([v[0], v[1], v[2]] + sorted(zip(v[3::2], v[4::2])))
    return ls[:4], wires, ls[4 + n:]


def wires_of(ckt):
    ls = ckt.strip("\n").split("\n")
    n = int(ls[3])
    out = []
    for line in ls[4:4 + n]:
        v = [int(x) for x in line.split()]
        out.append(((v[0], v[1]), list(zip(v[3::2], v[4::2]))))
    return out


def is_acyclic(ckt):
    ls = ckt.strip("\n").split("\n")
    N = int(ls[0]) + int(ls[1]) + int(ls[2])
    indeg = [0] * N
    adj = [[] for _ in range(N)]
    for (src, _), sinks in wires_of(ckt):
        for dst, _ in sinks:
            adj[src].append(dst)
            indeg[dst] += 1
    q = deque(i for i in range(N) if indeg[i] == 0)
    seen = 0
    while q:
        u = q.popleft()
        seen += 1
        for v in adj[u]:
            indeg[v] -= 1
            if indeg[v] == 0:
                q.append(v)
    return seen == N


@pytest.mark.parametrize("case", [c for c in REF if c["name"] != "prefix_names"],
                         ids=lambda c: "%s-%s" % (c["name"], c["mode"]))
def test_matches_the_reference_converter(case):
    warnings = []
    got = opentimer.convert(case["dump"], case["mode"], warnings=warnings)
    assert canonical(got) == canonical(case["ckt"])
    assert len(warnings) == case["n_warnings"]
    if all(len(s) <= 1 for _, s in wires_of(got)):
        assert got == case["ckt"]  # nothing for a set to reorder: byte-identical


@pytest.mark.skipif("%d.%d" % sys.version_info[:2] != _FIX["python"],
                    reason="Python set order is specific to the interpreter version")
@pytest.mark.parametrize("case", COMPAT, ids=lambda c: "%s-%s" % (c["name"], c["mode"]))
def test_compat_mode_is_byte_identical_under_the_same_hash_seed(case, tmp_path):
    """Dumps whose reference output changes with the hash seed: in compat
    mode, run under the same PYTHONHASHSEED, the converter writes the
    reference's bytes (recorded for seeds 0, 5 and 11)."""
    src = tmp_path / "dump.txt"
    src.write_text(case["dump"])
    for seed, want in case["ckt"].items():
        dst = tmp_path / ("out%s.ckt" % seed)
        subprocess.run([sys.executable, "-m", "lsim_b200.opentimer", str(src), str(dst), case["mode"],
                        "--compat"], env=dict(os.environ, PYTHONHASHSEED=seed), cwd=ROOT,
                       check=True, capture_output=True)
        assert dst.read_text() == want, seed


def test_prefix_names_differ_only_where_documented():
    """The reference's prefix match (u1 also matches u12:A) drops the edge
    u5 -> u12:A along with the loop edge u5 -> u1:A2; here only the loop
    edge goes."""
    for mode in ("bfs", "dfs"):
        ref = [c for c in REF if c["name"] == "prefix_names" and c["mode"] == mode][0]
        got = opentimer.convert(ref["dump"], mode)
        g, r = wires_of(got), wires_of(ref["ckt"])
        assert [w[0] for w in g] == [w[0] for w in r]
        u5, u12 = 3, 4  # ids: a y u1 u5 u12
        for (src, gs), (_, rs) in zip(g, r):
            if src == (u5, 0):
                assert rs == [] and gs == [(u12, 1)]
            else:
                assert gs == rs


def test_sinks_keep_dump_order_and_output_is_deterministic():
    d = gen.opentimer_dump(300, 20, seed=5, loops=10)
    a = opentimer.convert(d, "bfs")
    assert a == opentimer.convert(d, "bfs")
    pis, pos, cells, edges = opentimer.parse_dump(d)
    names = pis + pos + [c[0] for c in cells]
    first = {}  # (driving pin, sink element) -> position of its first edge
    driver = {}  # element id -> its driving pin
    for k, (s, t) in enumerate(edges):
        if s.split(":")[0] != t.split(":")[0]:
            first.setdefault((s, t.split(":")[0]), k)
            driver[names.index(s.split(":")[0])] = s
    for (src, _), sinks in wires_of(a):
        order = [first[(driver[src], names[d])] for d, _ in sinks]
        assert order == sorted(order)


def test_loops_mode_keeps_acyclic_netlists_whole_and_breaks_every_cycle():
    d = gen.opentimer_dump(2000, 64, seed=7, window=12)
    pis, pos, cells, edges = opentimer.parse_dump(d)
    n_arcs = len({(s, t) for s, t in edges if s.split(":")[0] != t.split(":")[0]})
    whole = opentimer.convert(d, "loops")
    assert sum(len(s) for _, s in wires_of(whole)) == n_arcs
    assert is_acyclic(whole)
    cyc = gen.opentimer_dump(2000, 64, seed=8, window=12, loops=40)
    pis, pos, cells, edges = opentimer.parse_dump(cyc)
    n_arcs = len({(s, t) for s, t in edges if s.split(":")[0] != t.split(":")[0]})
    out = opentimer.convert(cyc, "loops")
    kept = sum(len(s) for _, s in wires_of(out))
    assert is_acyclic(out)
    assert n_arcs - 40 <= kept < n_arcs  # at most one cut per added loop input
    for mode in ("bfs", "dfs"):
        assert is_acyclic(opentimer.convert(cyc, mode))
        assert sum(len(s) for _, s in wires_of(opentimer.convert(cyc, mode))) < kept


def test_bfs_keeps_exactly_the_edges_into_the_next_layer():
    """With every element reached, "bfs" keeps an edge u -> v iff v's
    breadth-first depth is one more than u's, when no edge joins two
    elements of equal depth (a layered dump)."""
    d = gen.opentimer_dump(600, 16, seed=9, layers=12, loops=20)
    pis, pos, cells, edges = opentimer.parse_dump(d)
    arcs = {}
    for s, t in edges:
        a, b = s.split(":")[0], t.split(":")[0]
        if a != b:
            arcs.setdefault(a, set()).add(b)
    depth = {p: 0 for p in pis}
    q = deque(pis)
    while q:
        u = q.popleft()
        for v in arcs.get(u, ()):
            if v not in depth:
                depth[v] = depth[u] + 1
                q.append(v)
    names = pis + pos + [c[0] for c in cells]
    kept = {(names[s], names[t]) for (s, _), sinks in wires_of(opentimer.convert(d, "bfs"))
            for t, _ in sinks}
    want = {(u, v) for u in arcs for v in arcs[u] if depth[v] == depth[u] + 1}
    assert kept == want


def test_high_fanout_net_whose_sinks_were_all_taken():
    """A clock buffer reached after the 30,000 flip-flops it drives loses all
    of its edges in bfs mode; the removals take one pass over its sinks, not
    one pass per sink."""
    n = 30000
    lines = ["module top;", "// Start PIs", "input clk;", "input d;", "", "// Start POs"]
    lines += ["output po%05d;" % i for i in range(n)] + ["", "// Start wires", "", "// Start cells",
                                                        "INV_X1 i0 ( );", "INV_X1 i1 ( );",
                                                        "CLKBUF_X1 b0 ( );"]
    lines += ["DFF_X1 f%05d ( );" % i for i in range(n)] + ["endmodule", "", "digraph TimingGraph {"]
    lines += ['  "clk" -> "i0:A";', '  "i0:ZN" -> "i1:A";', '  "i1:ZN" -> "b0:A";']
    for i in range(n):
        lines += ['  "b0:Z" -> "f%05d:CK";' % i, '  "d" -> "f%05d:D";' % i,
                  '  "f%05d:Q" -> "po%05d";' % (i, i)]
    ckt = opentimer.convert("\n".join(lines + ["}", ""]), "bfs")
    w = dict(wires_of(ckt))
    b0 = 2 + n + 2  # ids: clk d, POs, i0 i1 b0, flip-flops
    assert w[(b0, 0)] == []
    assert len(w[(1, 0)]) == n and all(pin == 1 for _, pin in w[(1, 0)])


def test_nangate45_table_converts_without_fallbacks():
    """With the opt-in table, a dump over AND/OR 2-4, XOR2, XNOR2, BUF, MUX2
    and the reference's INV/NAND/NOR/AOI/OAI/DFF cells converts in strict
    mode; the netlist loads, MUX selects land on pin 5 and the oracle runs
    it."""
    table = dict(opentimer.PIN_TABLE)
    table.update(opentimer.NANGATE45_PINS)
    for k in ("AND2X1", "INVX1", "NAND3X1"):  # the reference's X1-suffixed variants
        table.pop(k)
    d = gen.opentimer_dump(1500, 40, seed=11, window=10, pins=table)  # acyclic: no input is cut
    warnings = []
    ckt = opentimer.convert(d, "loops", pin_table=opentimer.NANGATE45_PINS, strict=True,
                            warnings=warnings)
    assert all("unknown gate name" in w and w.startswith("BUF") for w in warnings)
    types = [int(t) for t in ckt.strip().split("\n")[-1].split()]
    assert 7 in types and 3 in types and 6 in types and 2 in types
    assert any(pin == 5 for _, sinks in wires_of(ckt) for _, pin in sinks)
    s = Simulator(-1)
    s.load_circuit(ckt)
    n_pi = int(ckt.split("\n")[0])
    o = Oracle(ckt, gen.faults(ckt, "outputs"), gen.patterns(n_pi, 300, seed=1))
    assert len(o.simulate()) > 0


def test_tables_and_errors():
    assert opentimer.gate_type("NAND2_X1") == 4 and opentimer.gate_type("XNOR2_X1") == 6
    assert opentimer.gate_type("AOI22_X2") == 4 and opentimer.gate_type("OAI21_X1") == 5
    assert opentimer.gate_type("DFF_X1") == 4 and opentimer.gate_type("CLKBUF_X3") == 8
    w = []
    assert opentimer.gate_type("BUF_X1", w) == 1 and len(w) == 1
    loose = [c for c in REF if c["name"] == "unknown_cells"][0]["dump"]
    with pytest.raises(ValueError, match="no pin number"):
        opentimer.convert(loose, strict=True)
    extra = {"MUX2": {"A": 1, "B": 2, "S": 5, "Z": 0}, "BUF": {"A": 1, "Z": 0},
             "XOR2": {"A": 1, "B": 2, "Z": 0}}
    ckt = opentimer.convert(loose, "loops", pin_table=extra, strict=True)
    assert canonical(ckt)[1][0] == [0, 0, 2, (5, 1), (7, 2)]
    with pytest.raises(ValueError, match="unknown mode"):
        opentimer.convert(loose, "xfs")
    with pytest.raises(ValueError, match="Start cells"):
        opentimer.convert(loose.replace("// Start cells", "// cells"))
    bad = loose.replace('"xr:Z" -> "z";', '"xr:Z" -> "nowhere:A";')
    with pytest.raises(ValueError, match="unknown gate:pin"):
        opentimer.convert(bad)
    with pytest.raises(ValueError, match="listed twice"):
        opentimer.convert(loose.replace("input s;", "input a;"))


def test_command_line(tmp_path):
    case = REF[0]
    src, dst = tmp_path / "d.txt", tmp_path / "o.ckt"
    src.write_text(case["dump"])
    assert opentimer.main([str(src), str(dst), case["mode"]]) == 0
    assert canonical(dst.read_text()) == canonical(case["ckt"])
    assert opentimer.main([str(src), str(dst)]) == 2
    assert opentimer.main([str(src), str(dst), "xfs"]) == 1
    assert opentimer.main([str(tmp_path / "missing"), str(dst), "bfs"]) == 1


DUMPS = [
    dict(n_cells=400, n_pi=24, seed=1, loops=12, mode="bfs"),
    dict(n_cells=400, n_pi=24, seed=2, loops=12, mode="dfs"),
    dict(n_cells=600, n_pi=32, seed=3, loops=20, window=16, mode="loops"),
    dict(n_cells=300, n_pi=12, seed=4, layers=10, loops=8, mode="bfs"),
    dict(n_cells=200, n_pi=220, seed=5, fanout_free=True, loops=6, mode="dfs"),
]


def _converted(cfg):
    cfg = dict(cfg)
    mode = cfg.pop("mode")
    ckt = opentimer.convert(gen.opentimer_dump(**cfg), mode)
    return ckt


@pytest.mark.parametrize("cfg", DUMPS, ids=lambda c: "%s-%d" % (c["mode"], c["seed"]))
def test_converted_netlists_load_in_the_reader(cfg):
    """Cut edges leave pin-slot gaps; the reader keeps the reference's
    meaning of them and reports the reference's levels."""
    ckt = _converted(cfg)
    s = Simulator(-1)
    s.load_circuit(ckt)
    ls = ckt.split("\n")
    assert s.num_PIs() == int(ls[0]) and s.num_POs() == int(ls[1])
    assert s.num_gates() == int(ls[2])
    o = Oracle(ckt, "0\n", "0\n")
    assert np.array_equal(s.levels(), o.levels())
    assert np.array_equal(s.num_gates_per_level(), o.per_level())
    assert np.array_equal(s.gate_idx_to_tpg_order_idx(), o.tpg())


def test_some_converted_netlists_are_not_level_sorted():
    """Element order (Kahn) and levels (1 + max over the pin slots) disagree
    when a slot gap hides an input: the case the schedule levels exist for."""
    unsorted = 0
    for cfg in DUMPS:
        lv = Oracle(_converted(cfg), "0\n", "0\n").levels().astype(np.int64)
        unsorted += bool(np.any(np.diff(lv) < 0))
    assert unsorted >= 2


@needs_ref
@pytest.mark.parametrize("cfg", DUMPS[:3], ids=lambda c: "%s-%d" % (c["mode"], c["seed"]))
def test_oracle_matches_the_live_reference_on_converted_netlists(cfg):
    ckt = _converted(cfg)
    n_pi = int(ckt.split("\n")[0])
    flst, ptn = gen.faults(ckt, "outputs"), gen.patterns(n_pi, 700, seed=3)
    o = Oracle(ckt, flst, ptn)
    F = len(o.faults)
    assert np.array_equal(o.simulate(0, F), Reference(ckt, flst, ptn).simulate(0, F))


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", DUMPS, ids=lambda c: "%s-%d" % (c["mode"], c["seed"]))
def test_converted_netlists_simulate_like_the_oracle(cfg):
    ckt = _converted(cfg)
    n_pi = int(ckt.split("\n")[0])
    flst = gen.faults(ckt, "pins")
    ptn = gen.patterns(n_pi, 3000, seed=cfg["seed"])
    sim = Simulator(0)
    sim.read_text(ckt, flst, ptn)
    sim.run()
    got = sim.results()
    ref = Oracle(ckt, flst, ptn).simulate()
    assert np.array_equal(got["detected"], ref["detected"])
    assert np.array_equal(got["first_pattern"], ref["first"])
    assert np.array_equal(got["count"], ref["count"])
