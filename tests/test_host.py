"""Host logic of the product library without a GPU: the C ABI exports, the
reader (through a host-only handle) against the reference's golden answers,
input validation and error codes, and the fault-list generator."""
import os
import re

import numpy as np
import pytest

from lsim_b200 import Simulator, FsimbError, gen
from lsim_b200 import _lib
from tests.oracle_lib import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "fsimb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fsimb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = _declared()
    assert len(names) >= 25
    L = _lib.lib()
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, n


@pytest.mark.parametrize("t", range(7))
def test_reader_matches_test_basics(basics, t):
    c, a = basics["cases"][t], basics["answers"]
    sim = Simulator(-1)
    sim.read_text(c["ckt"], c["flst"], c["ptn"])
    nv = a["num_vars_ans"][t]
    assert (sim.num_PIs(), sim.num_POs(), sim.num_gates(), sim.num_wires(), sim.num_rounds()) == \
        tuple(nv)
    tpg = sim.gate_idx_to_tpg_order_idx()
    assert list(tpg) == a["tpg_ans"][t]
    assert list(sim.num_gates_per_level()) == a["num_gate_per_lvl_ans"][t]
    lv = sim.levels()
    n_pi, n_g = sim.num_PIs(), sim.num_gates()
    assert list(lv[:n_pi]) == a["pi_lvl_ans"][t]
    assert list(lv[n_pi:n_pi + n_g]) == a["gate_lvl_ans"][t]
    assert list(lv[n_pi + n_g:]) == a["po_lvl_ans"][t]
    site, pin, val = sim.faults()
    fa = a["fault_ans"][t]
    assert len(site) == a["fault_size_ans"][t]
    assert list(site) == [tpg[fa[2 * i]] for i in range(len(site))]
    assert list(val) == [fa[2 * i + 1] for i in range(len(site))]
    assert not pin.any()
    assert list(sim.patterns()[0]) == a["ptn_val_ans"][t][:n_pi]


def test_reader_matches_oracle_on_synthetic():
    w = gen.generate(n_gates=5000, n_pi=50, n_po=40, n_levels=30, n_patterns=1000, seed=3,
                     type_mask=gen.ALL_TYPES, faults="pins")
    sim = Simulator(-1)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    assert np.array_equal(sim.gate_idx_to_tpg_order_idx(), o.tpg())
    assert np.array_equal(sim.levels(), o.levels())
    assert np.array_equal(sim.num_gates_per_level(), o.per_level())
    assert np.array_equal(sim.types(), o.types())
    s, p, v = sim.faults()
    assert np.array_equal(s, o.faults["site"]) and np.array_equal(p, o.faults["pin"])
    assert np.array_equal(v, o.faults["value"])
    assert np.array_equal(sim.patterns().ravel(), o.words[:o.W * o.n_pi])


BAD_CKT = {
    "bad token": "1 1 1 2\n0 0 1 2 x\n",
    "pin out of range": "1 1 1 2\n0 0 1 2 7\n2 0 1 1 1\n0\n",
    "wire into a PI": "2 1 1 3\n0 0 1 1 1\n1 0 1 3 1\n3 0 1 2 1\n0\n",
    "wire out of a PO": "1 1 1 3\n0 0 1 2 1\n2 0 1 1 1\n1 0 1 2 2\n0\n",
    "unreachable gate": "1 1 2 2\n0 0 1 2 1\n2 0 1 1 1\n0 0\n",
    "cycle": "1 1 2 4\n0 0 1 2 1\n2 0 1 3 1\n3 0 2 2 2 1 1\n0 0\n1 0\n",
    "mux with two inputs": "2 1 1 3\n0 0 1 3 1\n1 0 1 3 2\n3 0 1 2 1\n7\n",
    "gate type out of range": "1 1 1 2\n0 0 1 2 1\n2 0 1 1 1\n12\n",
    "five inputs": "5 1 1 6\n0 0 1 6 1\n1 0 1 6 2\n2 0 1 6 3\n3 0 1 6 4\n4 0 1 6 1\n"
                   "6 0 1 5 1\n1\n",
    "truncated": "3 1 4 7\n7 0 1 5 1\n",
}


@pytest.mark.parametrize("what", sorted(BAD_CKT))
def test_malformed_circuits_are_rejected(what):
    sim = Simulator(-1)
    with pytest.raises(FsimbError) as e:
        sim.load_circuit(BAD_CKT[what])
    assert e.value.code == _lib.ERR_PARSE
    # the oracle restatement rejects the same inputs
    with pytest.raises(ValueError):
        Oracle(BAD_CKT[what], "0\n", "0\n")


def test_fault_and_pattern_errors(basics):
    c = basics["cases"][0]
    sim = Simulator(-1)
    sim.load_circuit(c["ckt"])
    with pytest.raises(FsimbError) as e:
        sim.set_fault_text("1\n99 0\n")
    assert e.value.code == _lib.ERR_PARSE
    with pytest.raises(FsimbError) as e:
        sim.set_fault_text("@pins\n1\n4 0 3\n")  # gate file id 4 has one input
    assert e.value.code == _lib.ERR_PARSE
    with pytest.raises(FsimbError) as e:
        sim.set_faults([99], [0], [1])
    assert e.value.code == _lib.ERR_ARG
    with pytest.raises(FsimbError) as e:
        sim.read_text(c["ckt"], c["flst"], "200\n1 2 3\n")  # 4 rounds, 3 words given
    assert e.value.code == _lib.ERR_PARSE
    sim.read_text(c["ckt"], c["flst"], c["ptn"])
    with pytest.raises(FsimbError) as e:
        sim.results()
    assert e.value.code == _lib.ERR_STATE
    with pytest.raises(FsimbError) as e:
        sim.run()
    assert e.value.code == _lib.ERR_CUDA


def test_missing_file_raises_like_the_reference(tmp_path):
    sim = Simulator(-1)
    with pytest.raises(RuntimeError, match="cannot open circut file"):
        sim.read(str(tmp_path / "nope.ckt"), str(tmp_path / "a"), str(tmp_path / "b"))


def test_generator_is_deterministic_and_sized():
    a = gen.workload("c1")
    b = gen.workload("c1")
    assert a == b
    sim = Simulator(-1)
    sim.read_text(a["ckt"], a["flst"], a["ptn"])
    i = sim.info()
    assert (i.num_gates, i.num_pis, i.num_pos, i.num_faults, i.num_patterns) == \
        (2000, 64, 64, 4000, 4096)
    assert i.num_levels == 32  # gate levels 1..30, POs at 31
    assert gen.workload("c1", seed=1)["ckt"] != a["ckt"]


def test_collapsed_faults_are_equivalent_classes():
    """Every fault of the uncollapsed list has the same per-pattern detection
    as some fault of the collapsed list, and collapsing keeps one fault per
    class: checked with the oracle's per-fault detection counts and first
    patterns, plus the equivalence rules on a circuit small enough to check
    every pair."""
    w = gen.generate(n_gates=120, n_pi=8, n_po=6, n_levels=8, n_patterns=640, seed=17,
                     faults="pins")
    coll = gen.faults(w["ckt"], "collapsed")
    full = Oracle(w["ckt"], w["flst"], w["ptn"])
    col = Oracle(w["ckt"], coll, w["ptn"])
    rf, rc = full.simulate(mode=0), col.simulate(mode=0)
    sig_full = {(int(a), int(b)) for a, b in zip(rf["count"], rf["first"])}
    sig_col = {(int(a), int(b)) for a, b in zip(rc["count"], rc["first"])}
    assert sig_full == sig_col
    assert len(col.faults) < len(full.faults)


def test_dot_matches_reference_visualization(basics):
    import json
    with open(os.path.join(ROOT, "tests", "golden", "test_basics_dot.json")) as f:
        dots = json.load(f)["cases"]
    for c, d in zip(basics["cases"], dots):
        sim = Simulator(-1)
        sim.read_text(c["ckt"], c["flst"], c["ptn"])
        assert sim.dot() == d["dot"], c["name"]


def test_batch_needs_a_gpu():
    """No CPU fallback: creating a batch without a usable device fails loudly."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lsim_b200 import Batch
    with pytest.raises(FsimbError) as e:
        Batch(0)
    assert e.value.code == _lib.ERR_CUDA


def test_batch_configs_follow_the_batched_configuration():
    cfgs = gen.batch_configs(256, seed=0)
    assert len(cfgs) == 256
    g = np.array([c["n_gates"] for c in cfgs])
    assert g.min() >= 500 and g.max() <= 50000
    assert np.median(g) < 10000  # log-uniform, not uniform
    assert all(10 <= c["n_levels"] <= 120 for c in cfgs)
    assert all(1024 <= c["n_patterns"] <= 16384 for c in cfgs)
    assert cfgs == gen.batch_configs(256, seed=0)


def test_serve_configs_follow_the_serving_configuration():
    cfgs = gen.serve_configs(32, seed=0)
    assert len(cfgs) == 32
    g = np.array([c["n_gates"] for c in cfgs])
    assert g.min() >= 1000 and g.max() <= 500000
    # levels at most 1,500 gates wide, so every circuit's sweep fits shared memory
    assert all(c["n_gates"] / c["n_levels"] <= 1500 for c in cfgs)
    assert cfgs == gen.serve_configs(32, seed=0)


def test_fault_costs_group_faults_that_share_a_sweep():
    from lsim_b200 import shard
    w = gen.generate(n_gates=3000, n_pi=30, n_po=20, n_levels=30, n_patterns=64, seed=9,
                     faults="pins")
    sim = Simulator(-1)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    site, pin, val = sim.faults()
    group, cost = sim.fault_costs()
    assert len(group) == len(site) and np.all(cost >= 1)
    # faults on one element always share a group, and a group has one cost
    for g in np.unique(group)[:200]:
        assert len(set(cost[group == g])) == 1
    by_site = {}
    for s, g in zip(site, group):
        assert by_site.setdefault(int(s), int(g)) == int(g)
    parts = shard.split_faults(group, cost, 3)
    allf = np.sort(np.concatenate(parts))
    assert np.array_equal(allf, np.arange(len(site)))      # every fault exactly once
    owners = {}
    for r, idx in enumerate(parts):
        for g in np.unique(group[idx]):
            assert owners.setdefault(int(g), r) == r        # a group is never split
    loads = []
    for idx in parts:
        _, first = np.unique(group[idx], return_index=True)
        loads.append(float(cost[idx][first].sum()))
    assert max(loads) <= 1.2 * min(loads) + cost.max()      # balanced


def test_shard_partitions_cover_everything_once():
    """Pattern blocks are contiguous, cut at 2,048-pattern tiles, disjoint and
    cover every round (ranks past the last tile get none); fault parts keep
    each sweep group on one rank and are balanced within the largest
    group's cost."""
    from lsim_b200 import shard
    for n_rounds in (1, 31, 32, 33, 1024, 1000):
        for world in (1, 2, 3, 4, 8, 64):
            blocks = [shard.round_block(n_rounds, r, world) for r in range(world)]
            at = 0
            for r0, r1 in blocks:
                if r1 > r0:  # an empty block may sit anywhere
                    assert r0 == at and r0 % 32 == 0 and (r1 % 32 == 0 or r1 == n_rounds)
                at = max(at, r1)
            assert at == n_rounds
            assert sum(r1 - r0 for r0, r1 in blocks) == n_rounds
    rng = np.random.default_rng(5)
    group = rng.integers(0, 300, size=5000)
    cost = rng.integers(1, 1000, size=5000)
    for world in (1, 2, 3, 8):
        parts = shard.split_faults(group, cost, world)
        allidx = np.concatenate(parts)
        assert len(allidx) == 5000 and len(np.unique(allidx)) == 5000
        owner = np.empty(5000, dtype=np.int64)
        for r, p in enumerate(parts):
            owner[p] = r
        for g in np.unique(group):
            assert len(np.unique(owner[group == g])) == 1
        gcost = {g: cost[group == g].max() for g in np.unique(group)}
        load = [sum(gcost[g] for g in np.unique(group[p])) for p in parts]
        assert max(load) - min(load) <= max(gcost.values())


def test_loader_selection_on_a_host_handle():
    """fsimb_set_loader / fsimb_get_load_info without a GPU: a host-only
    handle always uses the host reader, whatever mode is asked for."""
    s = Simulator(-1)
    with pytest.raises(FsimbError) as e:
        s.load_info()
    assert e.value.code == _lib.ERR_STATE
    for bad in ((3, 0), (-1, 0), (0, -2), (0, 5000)):
        rc = _lib.lib().fsimb_set_loader(s._h, *bad)
        assert rc == _lib.ERR_ARG
    w = gen.generate(n_gates=200, n_pi=8, n_po=8, n_levels=10, n_patterns=100, seed=3)
    for mode in ("auto", "host", "device"):
        s.set_loader(mode, 4)
        s.load_circuit(w["ckt"])
        li = s.load_info()
        assert li["on_device"] == 0 and li["handed_back"] == 0 and li["threads"] == 1
        assert li["ms_total"] >= 0
    with pytest.raises(KeyError):
        s.set_loader("gpu")


def test_element_accessors_like_the_reference():
    """pi(i) / gate(i) / po(i) / gates() (fsim/simulation.hpp:58-63) with
    ElementBase's idx() / level() / output_value(), and gateTypeToString."""
    from lsim_b200 import Simulator as S
    w = gen.generate(n_gates=120, n_pi=9, n_po=7, n_levels=8, n_patterns=100, seed=4,
                     type_mask=gen.ALL_TYPES)
    s = S(-1)
    s.read_text(w["ckt"], w["flst"], w["ptn"])
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    lv, ty = o.levels(), o.types()
    elems = [s.pi(i) for i in range(9)] + s.gates() + [s.po(i) for i in range(7)]
    assert [e.idx() for e in elems] == list(range(9 + 120 + 7))
    assert [e.level() for e in elems] == [int(x) for x in lv]
    assert [e.type for e in elems] == [int(x) for x in ty]
    assert all(e.output_value() == 0 for e in elems)  # before run()
    assert s.gate(5).idx() == 14 and s.po(0).idx() == 129
    assert [S.gateTypeToString(t) for t in range(12)] == [
        "INV", "AND", "OR", "XOR", "NAND", "NOR", "XNOR", "MUX", "CLKBUF", "PI", "PO", "UNKNOWN"]
    with pytest.raises(IndexError):
        s.pi(9)
    assert s.num_pos() == 7
