"""The CPU oracle against the reference simulator itself: fixtures recorded by
running LSIM's fsim::Simulator (tests/golden/make_golden.py), and -- when the
reference was compiled into oracle/_ref here -- live comparisons."""
import numpy as np
import pytest

from lsim_b200 import gen
from tests.oracle_lib import Oracle, Reference, ref_available


def test_oracle_matches_recorded_reference(ref_cases):
    for c in ref_cases["cases"]:
        o = Oracle(c["ckt"], c["flst"], c["ptn"])
        for mode in (0, 1):
            r = o.simulate(mode=mode, threads=2)
            assert list(r["detected"]) == c["detected"], c["name"]
            assert list(r["first"]) == c["first"], c["name"]
            assert list(r["count"]) == c["count"], c["name"]
            table = np.empty(2 * len(r), dtype=np.uint64)
            table[0::2] = r["ref_flag"]
            table[1::2] = r["ref_rd"]
            assert list(table) == c["table"], c["name"]
        assert list(o.good_values()) == c["good_last"], c["name"]


def test_naive_and_cone_modes_agree():
    w = gen.generate(n_gates=300, n_pi=12, n_po=9, n_levels=12, n_patterns=333,
                     type_mask=gen.ALL_TYPES, seed=21, faults="pins")
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    a, b = o.simulate(mode=0), o.simulate(mode=1)
    assert np.array_equal(a, b)


needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built here")


@needs_ref
def test_oracle_matches_live_reference_c1_sample():
    w = gen.workload("c1")
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    ref = Reference(w["ckt"], w["flst"], w["ptn"])
    rng = np.random.default_rng(0)
    f0 = int(rng.integers(0, len(o.faults) - 64))
    a = o.simulate(f0, f0 + 64)
    b = ref.simulate(f0, f0 + 64, threads=4)
    assert np.array_equal(a, b)


@needs_ref
def test_reference_public_run_matches_harness():
    w = gen.generate(n_gates=150, n_pi=10, n_po=6, n_levels=10, n_patterns=300,
                     type_mask=gen.ALL_TYPES, seed=5, faults="outputs")
    ref = Reference(w["ckt"], w["flst"], w["ptn"])
    table, good = ref.run_table(mode=0)
    r = ref.simulate()
    assert list(table[0::2]) == list(r["ref_flag"])
    assert list(table[1::2]) == list(r["ref_rd"])
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    assert list(good) == list(o.good_values())


@needs_ref
def test_oracle_matches_reference_when_rounds_exceed_pis():
    # ceil(P/64) > nPI: the reference's row placement is undefined there, so
    # both sides load the rows in file order.
    w = gen.generate(n_gates=120, n_pi=3, n_po=4, n_levels=8, n_patterns=64 * 7 - 5, seed=9,
                     faults="outputs")
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    ref = Reference(w["ckt"], w["flst"], words=o.words, P=o.P, n_pi=o.n_pi)
    assert np.array_equal(o.simulate(), ref.simulate())


@needs_ref
def test_oracle_matches_reference_on_seeded_random_circuits():
    """48 small circuits drawn from one seed: every gate type (MUX included),
    fan-in up to 3, 1-4 levels back, partial last rounds, one to five
    rounds, output faults, at most as many POs as gates; also the
    reference's last-round table and good values."""
    rng = np.random.default_rng(2024)
    for case in range(48):
        n_gates = int(rng.integers(5, 400))
        n_pi = int(rng.integers(1, 24))
        # more POs than gates would drive a PO from a PI, where the reference
        # writes past its gate array (fsim/simulation.cpp:856-861)
        n_po = int(rng.integers(1, min(16, n_gates) + 1))
        n_levels = int(rng.integers(1, max(2, min(n_gates, 30))))
        P = int(rng.integers(1, 64 * min(5, n_pi) + 1))  # ceil(P/64) <= nPI: defined row placement
        mask = gen.ALL_TYPES if case % 2 else gen.BENCH_TYPES
        w = gen.generate(n_gates=n_gates, n_pi=n_pi, n_po=n_po, n_levels=n_levels, n_patterns=P,
                         type_mask=mask, seed=1000 + case, faults="outputs",
                         window=int(rng.integers(1, 5)))
        o = Oracle(w["ckt"], w["flst"], w["ptn"])
        ref = Reference(w["ckt"], w["flst"], w["ptn"])
        assert np.array_equal(o.simulate(), ref.simulate()), case
        table, good = ref.run_table(mode=0)
        r = o.simulate()
        assert list(table[0::2]) == list(r["ref_flag"]), case
        assert list(table[1::2]) == list(r["ref_rd"]), case
        assert list(good) == list(o.good_values()), case
