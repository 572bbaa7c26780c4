"""Batched mode (fsimb_batch_*): many circuits in one launch sequence give,
for every circuit, exactly the results of the CPU oracle and of the plain
per-circuit GPU path.  Integer work: every comparison is bit-exact."""
import numpy as np
import pytest

from lsim_b200 import Batch, Simulator, gen
from tests.oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def _same(got, ref):
    assert np.array_equal(got["detected"], ref["detected"])
    assert np.array_equal(got["first_pattern"], ref["first"])
    assert np.array_equal(got["count"], ref["count"])
    assert np.array_equal(got["ref_last_round_flag"], ref["ref_flag"])
    assert np.array_equal(got["ref_last_rd"], ref["ref_rd"])


# Mixed sizes, all gate types (MUX cones take the exact-fault sweeps), pin
# faults, partial last rounds, one to three 2,048-pattern tiles.
MIX = [
    dict(n_gates=300, n_pi=10, n_po=8, n_levels=12, n_patterns=200, type_mask=gen.ALL_TYPES,
         seed=3, faults="outputs"),
    dict(n_gates=300, n_pi=10, n_po=8, n_levels=12, n_patterns=130, type_mask=gen.ALL_TYPES,
         seed=4, faults="pins"),
    dict(n_gates=500, n_pi=16, n_po=16, n_levels=15, n_patterns=4100, seed=5, faults="pins"),
    dict(n_gates=800, n_pi=20, n_po=10, n_levels=20, n_patterns=1000, seed=6, faults="collapsed"),
    dict(n_gates=2000, n_pi=64, n_po=64, n_levels=30, n_patterns=4096, seed=0, faults="outputs"),
    dict(n_gates=40, n_pi=5, n_po=3, n_levels=6, n_patterns=37, seed=16, faults="outputs"),
    dict(n_gates=3000, n_pi=40, n_po=40, n_levels=60, n_patterns=6000, seed=7,
         type_mask=gen.ALL_TYPES, faults="collapsed"),
    dict(n_gates=1200, n_pi=30, n_po=20, n_levels=8, n_patterns=2048, seed=8, faults="pins"),
]


@pytest.fixture(scope="module")
def mix():
    ws = [gen.generate(**c) for c in MIX]
    refs = [Oracle(w["ckt"], w["flst"], w["ptn"]).simulate() for w in ws]
    return ws, refs


def _members(ws, device=-1):
    sims = []
    for w in ws:
        s = Simulator(device)
        s.read_text(w["ckt"], w["flst"], w["ptn"])
        sims.append(s)
    return sims


def test_batch_matches_oracle_and_plain_path(mix):
    ws, refs = mix
    sims = _members(ws)
    with Batch(0) as b:
        for s in sims:
            b.add(s)
        b.run()
        st = b.stats()
        assert st["n_circuits"] == len(ws) and st["graph_used"] == 1
        assert st["kernel_launches"] > 0
        for s, w, ref in zip(sims, ws, refs):
            got = s.results()
            _same(got, ref)
            plain = Simulator(0)
            plain.read_text(w["ckt"], w["flst"], w["ptn"])
            plain.run()
            assert np.array_equal(got, plain.results())
            assert np.array_equal(s.found_fault_to_pattern(), plain.found_fault_to_pattern())


def test_graph_replay_direct_launches_and_shapes_agree(mix):
    ws, refs = mix
    sims = _members(ws)
    with Batch(0) as b:
        for s in sims:
            b.add(s)
        b.run()
        first = [s.results().copy() for s in sims]
        b.run()  # graph replay
        assert all(np.array_equal(s.results(), f) for s, f in zip(sims, first))
        b.run(graph=False)
        st = b.stats()
        assert st["graph_used"] == 0 and st["ms_sweep"] > 0
        assert all(np.array_equal(s.results(), f) for s, f in zip(sims, first))
        assert len(b.classes()) == st["n_classes"] >= 1
        for graph in (True, False):
            b.run(concurrent=False, graph=graph)
            assert all(np.array_equal(s.results(), f) for s, f in zip(sims, first))
        for M, T, occ in [(1, 256, 1), (2, 512, 2), (8, 128, 1), (4, 64, 3)]:
            b.run(words_per_item=M, block_threads=T, ctas_per_sm=occ)
            assert all(np.array_equal(s.results(), f) for s, f in zip(sims, first)), (M, T, occ)
        b.run(tune=True)
        st = b.stats()
        assert st["ms_tune"] > 0
        assert all(np.array_equal(s.results(), f) for s, f in zip(sims, first))
        b.run(tune=True)
        assert b.stats()["ms_tune"] == 0  # the tuned shape is kept for this membership
    for s, ref in zip(sims, refs):
        _same(s.results(), ref)


def test_repeated_direct_runs_keep_launch_limits(mix):
    """A second run that reuses the layout launches every class within its
    kernel's shared-memory limit (the large member first, a small one last:
    choosing shapes queries the kernels with the small member's size)."""
    ws, refs = mix
    sims = _members([ws[6], ws[5]])
    with Batch(0) as b:
        for s in sims:
            b.add(s)
        for graph in (False, False, True, False):
            b.run(graph=graph, concurrent=False)
            _same(sims[0].results(), refs[6])
            _same(sims[1].results(), refs[5])


def test_member_changes_are_picked_up(mix):
    ws, refs = mix
    sims = _members(ws[:4])
    with Batch(0) as b:
        for s in sims:
            b.add(s)
        b.run()
        w = gen.generate(**dict(MIX[2], n_patterns=2500, seed=9))
        sims[1].read_text(w["ckt"], w["flst"], w["ptn"])
        b.run()
        _same(sims[1].results(), Oracle(w["ckt"], w["flst"], w["ptn"]).simulate())
        for i in (0, 2, 3):
            _same(sims[i].results(), refs[i])
        b.clear()
        assert len(b) == 0
        b.add(sims[3])
        b.run()
        _same(sims[3].results(), refs[3])


def test_device_handles_can_be_members(mix):
    ws, refs = mix
    sims = _members(ws[:3], device=0)
    sims[0].run()
    with Batch(0) as b:
        for s in sims:
            b.add(s)
        b.run()
    for s, ref in zip(sims, refs[:3]):
        _same(s.results(), ref)
    sims[1].run()  # plain run on a handle whose plan the batch built
    _same(sims[1].results(), refs[1])


def test_batch_errors():
    from lsim_b200 import FsimbError
    from lsim_b200 import _lib
    with Batch(0) as b:
        with pytest.raises(FsimbError) as e:
            b.run()
        assert e.value.code == _lib.ERR_STATE
        s = Simulator(-1)
        w = gen.generate(n_gates=50, n_pi=5, n_po=5, n_levels=5, n_patterns=64, seed=1)
        s.load_circuit(w["ckt"])
        b.add(s)
        with pytest.raises(FsimbError) as e:
            b.run()
        assert e.value.code == _lib.ERR_STATE
        with pytest.raises(FsimbError) as e:
            b.add(s)
        assert e.value.code == _lib.ERR_ARG
        with pytest.raises(FsimbError) as e:
            b.run(words_per_item=3)
        assert e.value.code == _lib.ERR_ARG


def test_c4_sample_batch_against_oracle():
    """32 circuits drawn like the 256-circuit batched configuration, smaller
    (500-5,000 gates, 1,024-4,096 patterns), every fault checked."""
    cfgs = gen.batch_configs(32, seed=1, gates=(500, 5000), patterns=(1024, 4096))
    ws = [gen.generate(**c) for c in cfgs]
    sims = _members(ws)
    with Batch(0) as b:
        for s in sims:
            b.add(s)
        b.run(tune=True)
        st = b.stats()
        assert st["fault_patterns"] == sum(len(s.results()) * s.info().num_patterns for s in sims)
    for s, w in zip(sims, ws):
        _same(s.results(), Oracle(w["ckt"], w["flst"], w["ptn"]).simulate())
