"""Device loader (fsimb_set_loader, lsim_b200/csrc/fsimb_loader.cu): the
netlist it builds equals the host reader's field for field -- element order,
levels, types, fanin (through the DOT text and the simulation results) --
and every text the host reader rejects is handed back to it, so errors do
not change.  Integer work: every comparison is bit-exact."""
import numpy as np
import pytest

from lsim_b200 import FsimbError, Simulator, gen, opentimer
from lsim_b200 import _lib
from tests.test_host import BAD_CKT

pytestmark = pytest.mark.gpu


def _load(ckt, mode, threads=0):
    s = Simulator(0)
    s.set_loader(mode, threads)
    s.load_circuit(ckt)
    return s


def _same_netlist(a, b):
    ia, ib = a.info(), b.info()
    for f in ("num_pis", "num_pos", "num_gates", "num_wires", "num_elements", "num_levels"):
        assert getattr(ia, f) == getattr(ib, f), f
    assert np.array_equal(a.gate_idx_to_tpg_order_idx(), b.gate_idx_to_tpg_order_idx())
    assert np.array_equal(a.levels(), b.levels())
    assert np.array_equal(a.num_gates_per_level(), b.num_gates_per_level())
    assert np.array_equal(a.types(), b.types())
    assert a.dot() == b.dot()  # fanin lists, in order


def _same_run(ckt, flst, ptn, threads=0):
    out = []
    for mode in ("host", "device"):
        s = Simulator(0)
        s.set_loader(mode, threads)
        s.read_text(ckt, flst, ptn)
        s.run()
        out.append(s)
    h, d = out
    assert d.load_info()["on_device"] == 1 and h.load_info()["on_device"] == 0
    assert np.array_equal(h.results(), d.results())
    assert np.array_equal(h.good_values(), d.good_values())
    _same_netlist(h, d)
    return d


CIRCUITS = {
    "c1": lambda: gen.workload("c1"),
    "mux_pins": lambda: gen.generate(n_gates=300, n_pi=10, n_po=8, n_levels=12, n_patterns=130,
                                     type_mask=gen.ALL_TYPES, seed=4, faults="pins"),
    "hubs": lambda: gen.generate(n_gates=5000, n_pi=50, n_po=50, n_levels=40, n_patterns=1000,
                                 seed=12, faults="collapsed", hub_frac=0.1, biased_pi_frac=0.5),
    "wide": lambda: gen.generate(n_gates=20000, n_pi=200, n_po=100, n_levels=10, n_patterns=2048,
                                 seed=8, faults="outputs"),
    "deep": lambda: gen.generate(n_gates=3000, n_pi=8, n_po=4, n_levels=300, n_patterns=640,
                                 seed=10, faults="outputs"),
}


@pytest.mark.parametrize("name", sorted(CIRCUITS))
def test_device_loader_builds_the_host_netlist(name):
    w = CIRCUITS[name]()
    d = _same_run(w["ckt"], w["flst"], w["ptn"], threads=5)
    li = d.load_info()
    assert li["waves"] == d.info().num_levels - 1 and li["threads"] == 5


def test_chunk_boundaries_and_whitespace():
    """Tokens split across tokenizer chunks, tabs, CR/LF, runs of blanks."""
    w = CIRCUITS["mux_pins"]()
    messy = w["ckt"].replace("\n", " \r\n\t").replace(" 0 ", "  0\t")
    for threads in (1, 2, 3, 7, 64):
        h, d = _load(w["ckt"], "host"), _load(messy, "device", threads)
        assert d.load_info()["on_device"] == 1
        _same_netlist(h, d)


def _split_lines(ckt):
    """The same circuit with every wire of two or more sinks written as two
    lines of the same source (insertion order is kept)."""
    ls = ckt.strip("\n").split("\n")
    n = int(ls[3])
    out, extra = [], 0
    for line in ls[4:4 + n]:
        v = line.split()
        k = int(v[2])
        if k >= 2:
            h = k // 2
            out.append(" ".join(v[:2] + [str(h)] + v[3:3 + 2 * h]))
            out.append(" ".join(v[:2] + [str(k - h)] + v[3 + 2 * h:]))
            extra += 1
        else:
            out.append(line)
    return "\n".join(ls[:3] + [str(n + extra)] + out + ls[4 + n:]) + "\n"


def test_sources_on_several_lines():
    w = CIRCUITS["hubs"]()
    ckt = _split_lines(w["ckt"])
    _same_run(ckt, w["flst"], w["ptn"], threads=3)


def test_converted_and_duplicate_pin_netlists():
    """Netlists from the OpenTimer converter (pin-slot gaps) and with a pin
    written twice: level-sorted ones are built on the device, the rest are
    handed back and still equal the host reader's."""
    handed = on_dev = 0
    for cfg in [dict(n_cells=400, n_pi=24, seed=1, loops=12, mode="bfs"),
                dict(n_cells=300, n_pi=12, seed=4, layers=10, loops=8, mode="bfs"),
                dict(n_cells=600, n_pi=32, seed=3, loops=20, window=16, mode="loops"),
                dict(n_cells=800, n_pi=40, seed=6, window=10, mode="loops")]:
        cfg = dict(cfg)
        mode = cfg.pop("mode")
        ckt = opentimer.convert(gen.opentimer_dump(**cfg), mode)
        n_pi = int(ckt.split("\n")[0])
        s = _load(ckt, "device")
        li = s.load_info()
        handed += li["handed_back"]
        on_dev += li["on_device"]
        _same_netlist(_load(ckt, "host"), s)
        flst, ptn = gen.faults(ckt, "pins"), gen.patterns(n_pi, 1000, seed=2)
        a, b = Simulator(0), Simulator(0)
        a.set_loader("host")
        b.set_loader("device")
        for x in (a, b):
            x.read_text(ckt, flst, ptn)
            x.run()
        assert np.array_equal(a.results(), b.results())
    assert handed >= 1 and on_dev >= 1
    # a pin written twice: the later write wins, both count as inputs
    ckt = "2 1 2 4\n0 0 2 3 1 4 1\n1 0 1 3 1\n3 0 1 4 2\n4 0 1 2 1\n1 4\n"
    h, d = _load(ckt, "host"), _load(ckt, "device")
    assert d.load_info()["on_device"] == 1
    _same_netlist(h, d)


@pytest.mark.parametrize("what", sorted(BAD_CKT))
def test_rejected_texts_keep_the_host_readers_error(what):
    errs = []
    for mode in ("host", "device"):
        s = Simulator(0)
        s.set_loader(mode, 2)
        with pytest.raises(FsimbError) as e:
            s.load_circuit(BAD_CKT[what])
        errs.append((e.value.code, str(e.value)))
    assert errs[0] == errs[1]
    assert errs[0][0] == _lib.ERR_PARSE


def test_auto_mode_and_loader_errors():
    w = CIRCUITS["c1"]()
    s = Simulator(0)
    s.load_circuit(w["ckt"])  # small text: the host reader
    assert s.load_info()["on_device"] == 0 and s.load_info()["handed_back"] == 0
    with pytest.raises(FsimbError) as e:
        s.set_loader("device", -1)
    assert e.value.code == _lib.ERR_ARG


def test_c3_size_circuit_loads_on_the_device():
    """2,000,000 gates (the stress configuration's circuit): same netlist,
    and the device loader is the automatic choice at this size."""
    cfg = {k: v for k, v in gen.WORKLOADS["c3"].items()
           if k in ("n_gates", "n_pi", "n_po", "n_levels", "p_fanin3", "seed", "hub_frac")}
    ckt = gen.circuit(**cfg)
    h = _load(ckt, "host")
    d = Simulator(0)
    d.load_circuit(ckt)
    li = d.load_info()
    assert li["on_device"] == 1
    ia = h.info()
    assert ia.num_elements == d.info().num_elements == 2010000
    assert np.array_equal(h.gate_idx_to_tpg_order_idx(), d.gate_idx_to_tpg_order_idx())
    assert np.array_equal(h.levels(), d.levels())
    assert np.array_equal(h.types(), d.types())
    assert h.dot() == d.dot()
    print("c3 load: host %.1f ms, device %.1f ms (tokenize %.1f ms on %d threads, device %.1f ms, "
          "%d waves)" % (h.load_info()["ms_total"], li["ms_total"], li["ms_tokenize"], li["threads"],
                         li["ms_device"], li["waves"]))
