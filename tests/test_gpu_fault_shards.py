"""Fault sharding on the GPU: the parts of a fault list (lsim_b200.shard),
simulated one after another on one GPU as separate ranks would, combine to
the results of the whole list (bit-exact)."""
import numpy as np
import pytest

from lsim_b200 import Simulator, gen, shard

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_fault_parts_combine_to_the_whole_list(world):
    w = gen.generate(n_gates=3000, n_pi=40, n_po=30, n_levels=40, n_patterns=4500, seed=61,
                     faults="pins", type_mask=gen.ALL_TYPES)
    full = Simulator(0)
    full.read_text(w["ckt"], w["flst"], w["ptn"])
    full.run()
    site, pin, val = full.faults()
    group, cost = full.fault_costs()
    parts = []
    for idx in shard.split_faults(group, cost, world):
        s = Simulator(0)
        s.read_text(w["ckt"], w["flst"], w["ptn"])
        s.set_faults(site[idx], pin[idx], val[idx])
        s.run()
        parts.append((idx, s.results()))
    got = shard.combine_fault_shards(parts, len(site))
    ref = full.results()
    for k in ("detected", "first_pattern", "count", "ref_last_round_flag", "ref_last_rd"):
        assert np.array_equal(got[k], ref[k]), k
