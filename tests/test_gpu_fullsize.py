"""The benchmark configurations at full size.

c2 (200,000 gates, 738,943 collapsed output + input-pin faults, 65,536
patterns): size-independent properties of every fault's result, and a
bit-exact comparison with the oracle on 1,024 faults stratified by the
level of their site, output / pin fault and fanout-free-region position
(the root itself or a member), over all 1,024 rounds.

c2 with MUX gates (the generator's full type set, 200,000 gates): faults
with a MUX downstream take exact sweeps; a stratified fault sample over a
4,096-pattern block, bit-exact against the oracle.

c3 (2,000,000 gates, 400 levels, hub fanouts, biased PIs): its collapsed
output + input-pin fault list sampled down to 4,000,000 faults (seeded),
count mode over one 2,048-pattern tile; properties of every result and a
stratified sample bit-exact against the oracle.
"""
import numpy as np
import pytest

from lsim_b200 import Simulator, gen
from tests.oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def _same(got, ref):
    assert np.array_equal(got["detected"], ref["detected"])
    assert np.array_equal(got["first_pattern"], ref["first"])
    assert np.array_equal(got["count"], ref["count"])
    assert np.array_equal(got["ref_last_round_flag"], ref["ref_flag"])


def _props(sim, r):
    P = sim.info().num_patterns
    det = r["detected"].astype(bool)
    assert np.array_equal(det, r["count"] > 0)
    assert np.all((r["first_pattern"] >= 0) == det)
    assert np.all(r["first_pattern"] < P)
    assert np.all(r["count"] <= P)
    assert np.all(r["ref_last_rd"] == sim.num_rounds() - 1)


def stratified(sim, n, seed, bins=8):
    """Indices of n faults spread evenly over strata: level bin of the site
    x output / pin fault x site is its fanout-free region's root or not."""
    site, pin, _ = sim.faults()
    lev = sim.levels()[site.astype(np.int64)].astype(np.int64)
    lbin = np.minimum(bins - 1, lev * bins // (lev.max() + 1))
    group, _ = sim.fault_costs()
    member = (group != site) & (group < sim.info().num_elements)
    key = (lbin * 2 + (pin > 0)) * 2 + member
    rng = np.random.default_rng(seed)
    strata = [np.nonzero(key == k)[0] for k in np.unique(key)]
    per = -(-n // len(strata))
    pick = np.concatenate([rng.choice(g, size=min(per, len(g)), replace=False) for g in strata])
    if len(pick) < n:  # small strata: fill up from the rest
        rest = np.setdiff1d(np.arange(len(site)), pick)
        pick = np.concatenate([pick, rng.choice(rest, size=n - len(pick), replace=False)])
    return np.sort(pick)


@pytest.fixture(scope="module")
def c2_run():
    w = gen.workload("c2")
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    sim.run()
    return w, sim, sim.results()


def test_c2_properties(c2_run):
    w, sim, r = c2_run
    _props(sim, r)


def test_c2_stratified_sample_vs_oracle(c2_run):
    w, sim, r = c2_run
    pick = stratified(sim, 1024, seed=1)
    site, pin, val = sim.faults()
    o = Oracle(w["ckt"], "0\n", w["ptn"])
    o.set_faults(site[pick], pin[pick], val[pick])
    ref = o.simulate(mode=2)  # all 1,024 rounds
    _same(r[pick], ref)
    assert (pin[pick] > 0).sum() >= 256 and (pin[pick] == 0).sum() >= 256


def test_c2_drop_mode_matches_count_mode(c2_run):
    w, sim, r = c2_run
    sim.run(drop=True)
    d = sim.results()
    assert np.array_equal(d["first_pattern"], r["first_pattern"])
    assert np.array_equal(d["detected"], r["detected"])


def test_c2_with_mux_gates_vs_oracle():
    cfg = dict(gen.WORKLOADS["c2"])
    cfg.update(type_mask=gen.ALL_TYPES, n_patterns=4096)
    w = gen.generate(**cfg)
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    pick = stratified(sim, 20000, seed=3)
    site, pin, val = sim.faults()
    sim.set_faults(site[pick], pin[pick], val[pick])
    sim.run()
    assert sim.stats()["n_exact_sweeps"] > 1000
    r = sim.results()
    _props(sim, r)
    sub = stratified(sim, 512, seed=4)
    s2, p2, v2 = sim.faults()
    o = Oracle(w["ckt"], "0\n", w["ptn"])
    o.set_faults(s2[sub], p2[sub], v2[sub])
    _same(r[sub], o.simulate(mode=2))


def test_c3_count_mode_sample_vs_oracle():
    w = gen.workload("c3", faults="collapsed", n_patterns=2048)
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    site, pin, val = sim.faults()
    keep = np.sort(np.random.default_rng(0).choice(len(site), size=4000000, replace=False))
    sim.set_faults(site[keep], pin[keep], val[keep])
    sim.run()
    r = sim.results()
    _props(sim, r)
    assert r["detected"].sum() > 1000000
    sub = stratified(sim, 256, seed=5)
    s2, p2, v2 = sim.faults()
    o = Oracle(w["ckt"], "0\n", w["ptn"])
    o.set_faults(s2[sub], p2[sub], v2[sub])
    _same(r[sub], o.simulate(mode=2))
