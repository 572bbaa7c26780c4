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
    for mode in (0, 1):
        r = o.simulate(mode=mode, threads=1)
        table = np.empty(2 * len(r), dtype=np.uint64)
        table[0::2] = r["ref_flag"]
        table[1::2] = r["ref_rd"]
        assert list(table) == a["found_flst_2_ptn_ans"][t]
