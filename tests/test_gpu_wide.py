"""Circuits whose live values do not fit in shared memory: the sweep keeps
each CTA's values in global memory instead (k_sweep_wide, chosen
automatically).  Bit-exact against the oracle on a generated circuit with
100,000-gate levels, on a converted netlist with 40,000-gate levels, and,
with the global-memory sweep forced, on the small synthetic cases."""
import numpy as np
import pytest

from lsim_b200 import FsimbError, Simulator, gen, opentimer
from tests.oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def _same(got, ref):
    assert np.array_equal(got["detected"], ref["detected"])
    assert np.array_equal(got["first_pattern"], ref["first"])
    assert np.array_equal(got["count"], ref["count"])
    assert np.array_equal(got["ref_last_round_flag"], ref["ref_flag"])


def _sample(sim, n, seed):
    """n faults spread over the levels of their sites and over output / pin faults."""
    site, pin, val = sim.faults()
    lev = sim.levels()[site.astype(np.int64)]
    rng = np.random.default_rng(seed)
    keys = lev * 2 + (pin > 0)
    groups = [np.nonzero(keys == k)[0] for k in np.unique(keys)]
    per = max(1, n // len(groups))
    pick = np.concatenate([rng.choice(g, size=min(per, len(g)), replace=False) for g in groups])
    pick = np.sort(pick)
    return site[pick], pin[pick], val[pick]


CASES = {
    "mux_pins": lambda: gen.generate(n_gates=300, n_pi=10, n_po=8, n_levels=12, n_patterns=130,
                                     type_mask=gen.ALL_TYPES, seed=4, faults="pins"),
    "collapsed_partial": lambda: gen.generate(n_gates=800, n_pi=20, n_po=10, n_levels=20,
                                              n_patterns=777, seed=6, faults="collapsed"),
    "hubs_two_tiles": lambda: gen.generate(n_gates=3000, n_pi=50, n_po=50, n_levels=30,
                                           n_patterns=4096, seed=12, faults="collapsed",
                                           hub_frac=0.1, biased_pi_frac=0.5),
}


@pytest.mark.parametrize("M", [1, 2])
@pytest.mark.parametrize("name", sorted(CASES))
def test_global_sweep_forced_vs_oracle(name, M):
    w = CASES[name]()
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    sim.run(sweep_variant="global", words_per_item=M)
    assert sim.stats()["sweep_variant"] == 2
    _same(sim.results(), Oracle(w["ckt"], w["flst"], w["ptn"]).simulate())


def test_100k_gate_levels_vs_oracle():
    w = gen.generate(n_gates=400000, n_pi=2000, n_po=2000, n_levels=4, n_patterns=256, seed=21,
                     faults="collapsed")
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    assert max(sim.num_gates_per_level()) >= 100000
    site, pin, val = _sample(sim, 3000, seed=1)
    sim.set_faults(site, pin, val)
    with pytest.raises(FsimbError) as e:
        sim.run(sweep_variant="shared")  # shared memory cannot hold these levels
    assert e.value.code == 7
    sim.run()
    assert sim.stats()["sweep_variant"] == 2
    o = Oracle(w["ckt"], "0\n", w["ptn"])
    o.set_faults(site, pin, val)
    _same(sim.results(), o.simulate(mode=2))


def test_converted_wide_netlist_vs_oracle():
    ckt = opentimer.convert(gen.opentimer_dump(120000, 50000, seed=3, layers=3), mode="loops")
    sim = Simulator(0)
    sim.load_circuit(ckt)
    assert max(sim.num_gates_per_level()[1:-1]) >= 40000
    fl = gen.faults(ckt, "collapsed")
    ptn = gen.patterns(sim.num_PIs(), 300, seed=5)
    sim.read_text(ckt, fl, ptn)
    site, pin, val = _sample(sim, 3000, seed=2)
    sim.set_faults(site, pin, val)
    sim.run()
    assert sim.stats()["sweep_variant"] == 2
    o = Oracle(ckt, "0\n", ptn)
    o.set_faults(site, pin, val)
    _same(sim.results(), o.simulate(mode=2))
