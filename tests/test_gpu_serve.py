"""Serving loop (fsimb_server_*): every request's results, computed in waves
mixed with other requests, equal the plain path's results for the same
circuit, faults and patterns run alone (integer work: bit-exact)."""
import threading

import numpy as np
import pytest

from lsim_b200 import FsimbError, Server, Simulator, gen
from lsim_b200 import _lib
from tests.oracle_lib import Oracle

pytestmark = pytest.mark.gpu

CIRCUITS = [
    dict(n_gates=3000, n_pi=40, n_po=40, n_levels=40, n_patterns=6000, seed=21,
         type_mask=gen.ALL_TYPES, faults="pins"),
    dict(n_gates=800, n_pi=20, n_po=12, n_levels=20, n_patterns=4100, seed=22, faults="collapsed"),
    dict(n_gates=12000, n_pi=64, n_po=64, n_levels=60, n_patterns=8192, seed=23, faults="outputs"),
    dict(n_gates=300, n_pi=10, n_po=8, n_levels=12, n_patterns=2100, seed=24,
         type_mask=gen.ALL_TYPES, faults="outputs"),
]


@pytest.fixture(scope="module")
def circuits():
    out = []
    for c in CIRCUITS:
        w = gen.generate(**c)
        h = Simulator(-1)
        h.read_text(w["ckt"], w["flst"], w["ptn"])
        site, pin, val = h.faults()
        out.append(dict(w=w, words=h.patterns(), P=h.info().num_patterns, n_pi=h.num_PIs(),
                        site=site, pin=pin, value=val))
    return out


def _requests(circuits, n, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n):
        ci = int(rng.integers(len(circuits)))
        c = circuits[ci]
        F = len(c["site"])
        k = int(rng.integers(1, min(F, 400) + 1))
        idx = np.sort(rng.choice(F, size=k, replace=False))
        rows = c["words"].shape[0]
        tiles = (rows + 31) // 32
        row0 = 32 * int(rng.integers(tiles))
        max_p = min(c["P"] - row0 * 64, 64 * (rows - row0))
        P = int(rng.integers(1, max_p + 1))
        reqs.append(dict(circuit=ci, site=c["site"][idx], pin=c["pin"][idx], value=c["value"][idx],
                         row0=row0, P=P))
    return reqs


def _plain(c, r):
    W = (r["P"] + 63) // 64
    s = Simulator(0)
    s.load_circuit(c["w"]["ckt"])
    s.set_faults(r["site"], r["pin"], r["value"])
    s.set_patterns(c["words"][r["row0"]:r["row0"] + W], r["P"])
    s.run()
    return s.results()


def _serve(circuits, reqs, threads=4, **kw):
    results = [None] * len(reqs)
    with Server(0, **kw) as srv:
        ids = [srv.add_circuit(c["w"]["ckt"], c["words"], c["P"]) for c in circuits]

        def client(lo):
            for i in range(lo, len(reqs), threads):
                r = reqs[i]
                t = srv.submit(ids[r["circuit"]], r["site"], r["value"], pin=r["pin"],
                               n_patterns=r["P"], row0=r["row0"])
                results[i] = t
            for i in range(lo, len(reqs), threads):
                results[i] = srv.wait(results[i])

        ts = [threading.Thread(target=client, args=(k,)) for k in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        st = srv.stats()
    return results, st


def test_each_result_is_the_same_alone_and_in_the_mix(circuits):
    reqs = _requests(circuits, 48, seed=1)
    got, st = _serve(circuits, reqs)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["latency_p99_ms"] >= st["latency_p50_ms"] > 0
    for r, g in zip(reqs, got):
        assert np.array_equal(g, _plain(circuits[r["circuit"]], r))


def test_results_match_the_oracle(circuits):
    reqs = _requests(circuits, 6, seed=2)
    got, _ = _serve(circuits, reqs, threads=2)
    for r, g in zip(reqs, got):
        c = circuits[r["circuit"]]
        W = (r["P"] + 63) // 64
        o = Oracle(c["w"]["ckt"], "0\n", "0\n")
        o.set_faults(r["site"], r["pin"], r["value"])
        o.set_patterns(c["words"][r["row0"]:r["row0"] + W], r["P"])
        ref = o.simulate()
        assert np.array_equal(g["detected"], ref["detected"])
        assert np.array_equal(g["first_pattern"], ref["first"])
        assert np.array_equal(g["count"], ref["count"])


def test_requests_with_their_own_patterns(circuits):
    rng = np.random.default_rng(3)
    with Server(0) as srv:
        ids = [srv.add_circuit(c["w"]["ckt"]) for c in circuits]  # no resident block
        tickets, reqs = [], []
        for ci, c in enumerate(circuits):
            P = int(rng.integers(64, 3000))
            W = (P + 63) // 64
            words = rng.integers(0, 2**63, size=(W, c["n_pi"]), dtype=np.uint64)
            k = min(len(c["site"]), 150)
            r = dict(circuit=ci, site=c["site"][:k], pin=c["pin"][:k], value=c["value"][:k],
                     words=words, P=P)
            reqs.append(r)
            tickets.append(srv.submit(ids[ci], r["site"], r["value"], pin=r["pin"], n_patterns=P,
                                      words=words))
        for r, t in zip(reqs, tickets):
            g = srv.wait(t)
            s = Simulator(0)
            s.load_circuit(circuits[r["circuit"]]["w"]["ckt"])
            s.set_faults(r["site"], r["pin"], r["value"])
            s.set_patterns(r["words"], r["P"])
            s.run()
            assert np.array_equal(g, s.results())
        with pytest.raises(FsimbError) as e:  # no resident block to take rows from
            srv.submit(ids[0], circuits[0]["site"][:3], circuits[0]["value"][:3], n_patterns=64)
        assert e.value.code == _lib.ERR_ARG


def test_small_slots_admit_by_footprint(circuits):
    """One slot of 48 MB: requests queue for room, run in many waves, and a
    request larger than a slot fails with FSIMB_ERR_LIMIT."""
    reqs = _requests(circuits, 24, seed=4)
    got, st = _serve(circuits, reqs, threads=3, slots=1, slot_bytes=48 << 20, max_wave_requests=4)
    assert st["waves"] >= 6 and st["mean_wave_requests"] <= 4
    for r, g in zip(reqs, got):
        assert np.array_equal(g, _plain(circuits[r["circuit"]], r))
    c = circuits[2]
    with Server(0, slots=1, slot_bytes=8 << 20) as srv:
        cid = srv.add_circuit(c["w"]["ckt"], c["words"], c["P"])
        t = srv.submit(cid, c["site"], c["value"], pin=c["pin"], n_patterns=c["P"])
        with pytest.raises(FsimbError) as e:
            srv.wait(t)
        assert e.value.code == _lib.ERR_LIMIT


def test_submit_errors(circuits):
    c = circuits[1]
    with Server(0) as srv:
        cid = srv.add_circuit(c["w"]["ckt"], c["words"], c["P"])
        for kw in (dict(row0=5, n_patterns=64), dict(row0=0, n_patterns=c["P"] + 64 * 40),
                   dict(row0=0, n_patterns=64, bad_site=True)):
            site = c["site"][:4].copy()
            if kw.pop("bad_site", False):
                site[0] = 10 ** 7
            with pytest.raises(FsimbError) as e:
                srv.submit(cid, site, c["value"][:4], **kw)
            assert e.value.code == _lib.ERR_ARG
        with pytest.raises(FsimbError) as e:
            srv.submit(cid + 7, c["site"][:4], c["value"][:4], n_patterns=64)
        assert e.value.code == _lib.ERR_ARG
        t = srv.submit(cid, c["site"][:4], c["value"][:4], n_patterns=64)
        assert srv.wait(t) is not None
