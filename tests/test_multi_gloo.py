"""Pattern sharding across 2 ranks (gloo, CPU): each rank simulates its block
of rounds (the CPU oracle stands in for the GPU here), lsim_b200.shard merges
the per-fault results, and the merge must equal one simulation of the whole
pattern block."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lsim_b200 import gen, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, w, q, dst=None):
    import torch.distributed as dist
    from tests.oracle_lib import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full = Oracle(w["ckt"], w["flst"], w["ptn"])
        words, P, first = shard.local_patterns(full.words, full.P, full.n_pi, rank, world)
        ptn = "%d\n" % P + "\n".join(" ".join(str(int(x)) for x in row) for row in words) + "\n"
        o = Oracle(w["ckt"], w["flst"], ptn)
        r = o.simulate(threads=2)
        res = np.zeros(len(r), dtype=[("detected", np.uint8), ("ref_last_round_flag", np.uint8),
                                      ("pad", np.uint8, 6), ("first_pattern", np.int64),
                                      ("count", np.uint64), ("ref_last_rd", np.uint64)])
        res["count"] = r["count"]
        res["first_pattern"] = r["first"]
        res["ref_last_round_flag"] = r["ref_flag"]
        r0, r1 = shard.round_block(full.W, rank, world)
        merged = shard.merge_results(res, first, r1 == full.W and r1 > r0, full.W, dst=dst)
        q.put((rank, None if merged is None else merged.tobytes()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("P,dst", [(64 * 40, None), (64 * 70 + 17, None), (64 * 70 + 17, 0)])
def test_pattern_shards_merge_to_full_block(P, dst):
    w = gen.generate(n_gates=300, n_pi=12, n_po=10, n_levels=12, n_patterns=P, seed=77,
                     faults="collapsed")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, w, q, dst)) for r in range(2)]
    for p in procs:
        p.start()
    outs = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from tests.oracle_lib import Oracle
    ref = Oracle(w["ckt"], w["flst"], w["ptn"]).simulate()
    dt = np.dtype([("detected", np.uint8), ("ref_last_round_flag", np.uint8), ("pad", np.uint8, 6),
                   ("first_pattern", np.int64), ("count", np.uint64), ("ref_last_rd", np.uint64)])
    if dst is not None:
        assert outs[1 - dst] is None
    for rank in range(2) if dst is None else [dst]:
        m = np.frombuffer(outs[rank], dtype=dt)
        assert np.array_equal(m["count"], ref["count"])
        assert np.array_equal(m["first_pattern"], ref["first"])
        assert np.array_equal(m["detected"], ref["detected"])
        assert np.array_equal(m["ref_last_round_flag"], ref["ref_flag"])
        assert np.array_equal(m["ref_last_rd"], ref["ref_rd"])


def _fault_worker(rank, world, port, w, q, dst=None):
    import torch.distributed as dist
    from lsim_b200 import Simulator
    from tests.oracle_lib import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        h = Simulator(-1)
        h.read_text(w["ckt"], w["flst"], w["ptn"])
        site, pin, val = h.faults()
        group, cost = h.fault_costs()
        idx = shard.split_faults(group, cost, world)[rank]
        o = Oracle(w["ckt"], "0\n", w["ptn"])
        o.set_faults(site[idx], pin[idx], val[idx])
        r = o.simulate(threads=2)
        res = np.zeros(len(r), dtype=_DT)
        res["count"] = r["count"]
        res["first_pattern"] = r["first"]
        res["ref_last_round_flag"] = r["ref_flag"]
        res["ref_last_rd"] = r["ref_rd"]
        merged = shard.merge_fault_shards(res, idx, len(site), h.info().num_rounds, dst=dst)
        q.put((rank, None if merged is None else merged.tobytes()))
    finally:
        dist.destroy_process_group()


_DT = np.dtype([("detected", np.uint8), ("ref_last_round_flag", np.uint8), ("pad", np.uint8, 6),
                ("first_pattern", np.int64), ("count", np.uint64), ("ref_last_rd", np.uint64)])


@pytest.mark.parametrize("dst", [None, 0, 1])
def test_fault_shards_merge_to_full_list(dst):
    """Each of 2 ranks simulates its part of the fault list over all patterns;
    the merge (gathered on every rank, or on rank dst only) equals one
    simulation of the whole list."""
    w = gen.generate(n_gates=400, n_pi=12, n_po=10, n_levels=14, n_patterns=64 * 9 + 5, seed=78,
                     faults="pins", type_mask=gen.ALL_TYPES)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fault_worker, args=(r, 2, port, w, q, dst)) for r in range(2)]
    for p in procs:
        p.start()
    outs = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from tests.oracle_lib import Oracle
    ref = Oracle(w["ckt"], w["flst"], w["ptn"]).simulate()
    if dst is not None:
        assert outs[1 - dst] is None
    for rank in range(2) if dst is None else [dst]:
        m = np.frombuffer(outs[rank], dtype=_DT)
        assert np.array_equal(m["count"], ref["count"])
        assert np.array_equal(m["first_pattern"], ref["first"])
        assert np.array_equal(m["detected"], ref["detected"])
        assert np.array_equal(m["ref_last_round_flag"], ref["ref_flag"])
        assert np.array_equal(m["ref_last_rd"], ref["ref_rd"])
