"""GPU path (through the C ABI) against the CPU oracle and the reference's
recorded outputs.  Integer work: every comparison is bit-exact."""
import numpy as np
import pytest

from lsim_b200 import Simulator, gen
from tests.oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def _run(w, **kw):
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    sim.run(**kw)
    return sim


def _assert_same(got, ref):
    assert np.array_equal(got["detected"], ref["detected"])
    assert np.array_equal(got["first_pattern"], ref["first"])
    assert np.array_equal(got["count"], ref["count"])
    assert np.array_equal(got["ref_last_round_flag"], ref["ref_flag"])
    assert np.array_equal(got["ref_last_rd"], ref["ref_rd"])


@pytest.mark.parametrize("t", range(7))
def test_unit_test_fixtures(basics, t):
    c = basics["cases"][t]
    a = basics["answers"]
    sim = _run(c)
    n_pi, n_g = sim.num_PIs(), sim.num_gates()
    assert list(sim.g_pi_results()) == a["pi_ans"][t]
    assert list(sim.g_gate_results()) == a["gate_ans"][t]
    assert list(sim.g_po_results()) == a["po_ans"][t]
    assert list(sim.found_fault_to_pattern()) == a["found_flst_2_ptn_ans"][t]
    assert n_pi == a["num_vars_ans"][t][0] and n_g == a["num_vars_ans"][t][2]
    _assert_same(sim.results(), Oracle(c["ckt"], c["flst"], c["ptn"]).simulate())


def test_reference_recorded_cases(ref_cases):
    for c in ref_cases["cases"]:
        sim = _run(c)
        r = sim.results()
        assert list(r["detected"]) == c["detected"], c["name"]
        assert list(r["first_pattern"]) == c["first"], c["name"]
        assert list(r["count"]) == c["count"], c["name"]
        assert list(sim.found_fault_to_pattern()) == c["table"], c["name"]
        assert list(sim.good_values()) == c["good_last"], c["name"]


CASES = {
    "c1": lambda: gen.workload("c1"),
    "mux_outputs": lambda: gen.generate(n_gates=300, n_pi=10, n_po=8, n_levels=12, n_patterns=200,
                                        type_mask=gen.ALL_TYPES, seed=3, faults="outputs"),
    "mux_pins": lambda: gen.generate(n_gates=300, n_pi=10, n_po=8, n_levels=12, n_patterns=130,
                                     type_mask=gen.ALL_TYPES, seed=4, faults="pins"),
    "pins_multi_tile": lambda: gen.generate(n_gates=500, n_pi=16, n_po=16, n_levels=15,
                                            n_patterns=4100, seed=5, faults="pins"),
    "collapsed_partial": lambda: gen.generate(n_gates=800, n_pi=20, n_po=10, n_levels=20,
                                              n_patterns=777, seed=6, faults="collapsed"),
    "wide_levels": lambda: gen.generate(n_gates=20000, n_pi=200, n_po=100, n_levels=10,
                                        n_patterns=2048, seed=8, faults="collapsed"),
    "deep_narrow": lambda: gen.generate(n_gates=3000, n_pi=8, n_po=4, n_levels=300,
                                        n_patterns=640, seed=10, faults="outputs"),
    "hubs": lambda: gen.generate(n_gates=5000, n_pi=50, n_po=50, n_levels=40, n_patterns=1000,
                                 seed=12, faults="collapsed", hub_frac=0.1, biased_pi_frac=0.5),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_synthetic_vs_oracle(name):
    w = CASES[name]()
    sim = _run(w)
    _assert_same(sim.results(), Oracle(w["ckt"], w["flst"], w["ptn"]).simulate())
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    assert np.array_equal(sim.good_values(0), o.good_values(0))


@pytest.mark.parametrize("M", [1, 2, 4, 8])
@pytest.mark.parametrize("threads", [32, 128, 512])
def test_sweep_shapes_agree(M, threads):
    w = gen.generate(n_gates=1500, n_pi=24, n_po=16, n_levels=25, n_patterns=2500, seed=31,
                     type_mask=gen.ALL_TYPES, faults="pins")
    ref = Oracle(w["ckt"], w["flst"], w["ptn"]).simulate()
    sim = _run(w, words_per_item=M, block_threads=threads)
    _assert_same(sim.results(), ref)


@pytest.mark.parametrize("M,threads,occ", [(2, 256, 3), (4, 128, 2), (8, 64, 4), (1, 512, 2)])
def test_ctas_per_sm_shapes_agree(M, threads, occ):
    """Several CTAs per SM (smaller record buffers) give the same results."""
    w = gen.generate(n_gates=1500, n_pi=24, n_po=16, n_levels=25, n_patterns=2500, seed=32,
                     type_mask=gen.ALL_TYPES, faults="pins")
    ref = Oracle(w["ckt"], w["flst"], w["ptn"]).simulate()
    sim = _run(w, words_per_item=M, block_threads=threads, ctas_per_sm=occ)
    _assert_same(sim.results(), ref)
    assert sim.stats()["ctas_per_sm"] >= 1


def test_autotuned_shape_agrees_and_is_kept():
    """The first tuned run times candidate shapes, later runs reuse the
    winner, and a new fault list is tuned again; results never change."""
    w = gen.generate(n_gates=4000, n_pi=40, n_po=30, n_levels=40, n_patterns=5000, seed=33,
                     type_mask=gen.ALL_TYPES, faults="collapsed")
    ref = Oracle(w["ckt"], w["flst"], w["ptn"]).simulate()
    sim = _run(w, tune=True)
    assert sim.stats()["ms_tune"] > 0
    _assert_same(sim.results(), ref)
    sim.run(tune=True)
    assert sim.stats()["ms_tune"] == 0
    _assert_same(sim.results(), ref)
    flst = gen.faults(w["ckt"], "outputs")
    sim.set_fault_text(flst)
    sim.run(tune=True)
    assert sim.stats()["ms_tune"] > 0
    _assert_same(sim.results(), Oracle(w["ckt"], flst, w["ptn"]).simulate())
    sim.run(tune=True, drop=True)
    r = sim.results()
    ref2 = Oracle(w["ckt"], flst, w["ptn"]).simulate()
    assert np.array_equal(r["first_pattern"], ref2["first"])


def test_drop_mode_first_pattern():
    w = gen.generate(n_gates=2000, n_pi=32, n_po=32, n_levels=30, n_patterns=20000, seed=41,
                     faults="collapsed", biased_pi_frac=0.7, p_one_biased=0.05)
    ref = Oracle(w["ckt"], w["flst"], w["ptn"]).simulate()
    sim = _run(w, drop=True)
    r = sim.results()
    assert np.array_equal(r["detected"], ref["detected"])
    assert np.array_equal(r["first_pattern"], ref["first"])
    # count covers the tile of first detection only: never above the full count
    assert np.all(r["count"] <= ref["count"])
    assert np.all((r["count"] > 0) == (ref["count"] > 0))


def test_edge_cases():
    # PI driving a PO directly, a dangling gate, a single pattern
    ckt = "2 2 2 4\n0 0 2 2 1 4 1\n1 0 2 4 2 5 1\n4 0 1 3 1\n5 0 0\n1 0\n"
    flst = "6\n0 0\n0 1\n4 0\n4 1\n5 1\n3 0\n"
    for P, ptn in [(1, "1\n1 0\n"), (64, "64\n%d %d\n" % (2**63 + 5, 77)), (65, "65\n3 5\n1 0\n")]:
        w = {"ckt": ckt, "flst": flst, "ptn": ptn}
        sim = _run(w)
        _assert_same(sim.results(), Oracle(ckt, flst, ptn).simulate())
    # no faults
    w = gen.generate(n_gates=50, n_pi=5, n_po=3, n_levels=5, n_patterns=100, seed=1)
    sim = Simulator(0)
    sim.read_text(w["ckt"], "0\n", w["ptn"])
    sim.run()
    assert len(sim.results()) == 0


def test_repeated_runs_and_reload():
    w1 = CASES["collapsed_partial"]()
    w2 = CASES["pins_multi_tile"]()
    sim = Simulator(0)
    for w in (w1, w2, w1):
        sim.read_text(w["ckt"], w["flst"], w["ptn"])
        sim.run()
        sim.run()
        _assert_same(sim.results(), Oracle(w["ckt"], w["flst"], w["ptn"]).simulate())
