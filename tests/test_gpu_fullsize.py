"""The 200k-gate configuration at full size: size-independent properties plus
a sampled bit-exact comparison with the oracle (faults x all rounds)."""
import numpy as np
import pytest

from lsim_b200 import Simulator, gen
from tests.oracle_lib import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2_run():
    w = gen.workload("c2")
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    sim.run()
    return w, sim, sim.results()


def test_c2_properties(c2_run):
    w, sim, r = c2_run
    P = sim.info().num_patterns
    det = r["detected"].astype(bool)
    assert np.array_equal(det, r["count"] > 0)
    assert np.all((r["first_pattern"] >= 0) == det)
    assert np.all(r["first_pattern"] < P)
    assert np.all(r["count"] <= P)
    assert np.all(r["ref_last_rd"] == sim.num_rounds() - 1)


def test_c2_sample_vs_oracle(c2_run):
    w, sim, r = c2_run
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    rng = np.random.default_rng(1)
    # two contiguous blocks of 32 faults, all 1,024 rounds, cone-limited oracle
    for f0 in rng.integers(0, len(o.faults) - 32, size=2):
        f0 = int(f0)
        ref = o.simulate(f0, f0 + 32)
        assert np.array_equal(r["count"][f0:f0 + 32], ref["count"]), f0
        assert np.array_equal(r["first_pattern"][f0:f0 + 32], ref["first"]), f0
        assert np.array_equal(r["ref_last_round_flag"][f0:f0 + 32], ref["ref_flag"]), f0


def test_c2_drop_mode_matches_count_mode(c2_run):
    w, sim, r = c2_run
    sim.run(drop=True)
    d = sim.results()
    assert np.array_equal(d["first_pattern"], r["first_pattern"])
    assert np.array_equal(d["detected"], r["detected"])
    sim.run()
