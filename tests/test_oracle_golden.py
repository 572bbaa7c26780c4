"""The CPU oracle against the reference's own unit-test answers
(unittests/test_basics.cpp:212-345): sizes, topological order, levels, fault
and pattern initialisation, good-machine words and the fault table."""
import numpy as np
import pytest

from tests.oracle_lib import Oracle


@pytest.mark.parametrize("t", range(7))
def test_oracle_matches_test_basics(basics, t):
    c = basics["cases"][t]
    a = basics["answers"]
    o = Oracle(c["ckt"], c["flst"], c["ptn"])
    nv = a["num_vars_ans"][t]
    assert (o.n_pi, o.n_po, o.n_gates, o.W) == (nv[0], nv[1], nv[2], nv[4])
    tpg = o.tpg()
    assert list(tpg) == a["tpg_ans"][t]
    assert list(o.per_level()) == a["num_gate_per_lvl_ans"][t]
    lv = o.levels()
    assert list(lv[:o.n_pi]) == a["pi_lvl_ans"][t]
    assert list(lv[o.n_pi:o.n_pi + o.n_gates]) == a["gate_lvl_ans"][t]
    assert list(lv[o.n_pi + o.n_gates:]) == a["po_lvl_ans"][t]
    fa = a["fault_ans"][t]
    assert len(o.faults) == a["fault_size_ans"][t]
    for i, f in enumerate(o.faults):
        assert f["site"] == tpg[fa[2 * i]]
        assert f["value"] == fa[2 * i + 1]
    assert list(o.words[:o.n_pi]) == a["ptn_val_ans"][t][:o.n_pi]
    g = o.good_values()
    assert list(g[:o.n_pi]) == a["pi_ans"][t]
    assert list(g[o.n_pi:o.n_pi + o.n_gates]) == a["gate_ans"][t]
    assert list(g[o.n_pi + o.n_gates:]) == a["po_ans"][t]
    for mode in (0, 1, 2):
        r = o.simulate(mode=mode, threads=1)
        table = np.empty(2 * len(r), dtype=np.uint64)
        table[0::2] = r["ref_flag"]
        table[1::2] = r["ref_rd"]
        assert list(table) == a["found_flst_2_ptn_ans"][t]


@pytest.mark.parametrize("seed,mask,kind,P", [(3, "all", "pins", 4493), (5, "bench", "collapsed", 777),
                                              (8, "all", "outputs", 130)])
def test_oracle_modes_agree(seed, mask, kind, P):
    """Full re-simulation (mode 0), the event-driven cone (mode 1) and the
    event-driven cone over chunks of rounds (mode 2) give the same results,
    partial last rounds and several chunks included."""
    from lsim_b200 import gen
    w = gen.generate(n_gates=400, n_pi=12, n_po=10, n_levels=14, n_patterns=P, seed=seed,
                     type_mask=gen.ALL_TYPES if mask == "all" else gen.BENCH_TYPES, faults=kind)
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    r0 = o.simulate(mode=0, threads=2)
    r1 = o.simulate(mode=1, threads=3)
    r2 = o.simulate(mode=2, threads=4)
    assert np.array_equal(r0, r1) and np.array_equal(r0, r2)
    half = o.W // 2
    assert np.array_equal(o.simulate(rd0=half, mode=2), o.simulate(rd0=half, mode=0))
