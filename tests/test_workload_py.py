"""The pure-Python workload generator (tests/workload_py.py) writes exactly
what the product generator (lsim_b200.gen, fsimb_gen.cpp) writes: the same
.ckt text, the same collapsed fault list and the same pattern words.  The
benchmark's reference arm builds its inputs with it, so that its process
loads no product library."""
import numpy as np
import pytest

from lsim_b200 import gen
from tests import workload_py as wp
from tests.oracle_lib import Oracle

CFGS = [
    dict(n_gates=500, n_pi=16, n_po=12, n_levels=14, p_fanin3=0.5, seed=3),
    dict(n_gates=3000, n_pi=64, n_po=64, n_levels=30, p_fanin3=0.6, seed=1, type_mask=gen.ALL_TYPES),
    dict(n_gates=2000, n_pi=40, n_po=50, n_levels=20, p_fanin3=0.6, seed=5, hub_frac=0.1),
    dict(n_gates=40, n_pi=8, n_po=30, n_levels=6, p_fanin3=0.2, seed=9),  # POs beyond the sinks
]


def _flst_arrays(text):
    toks = text.split()
    F = int(toks[1])
    a = np.array(toks[2:], dtype=np.int64).reshape(F, 3)
    return a[:, 0], a[:, 2], a[:, 1]


@pytest.mark.parametrize("cfg", CFGS)
def test_circuit_and_collapsed_faults_equal_the_product_generator(cfg):
    ckt = gen.circuit(**cfg)
    assert wp.circuit(**cfg) == ckt
    site, pin, val = _flst_arrays(gen.faults(ckt, "collapsed"))
    s, p, v = wp.collapsed_faults(wp._circuit(**cfg), Oracle(ckt, "0\n", "0\n").tpg())
    assert np.array_equal(s, site) and np.array_equal(p, pin) and np.array_equal(v, val)


@pytest.mark.parametrize("args", [(30, 1000, 4, 0.5, 0.2), (7, 64, 0, 0.0, 0.2), (5, 130, 2, 1.0, 0.3)])
def test_pattern_words_equal_the_product_generator(args):
    n_pi, P, seed, frac, p1 = args
    toks = gen.patterns(n_pi, P, seed=seed, biased_pi_frac=frac, p_one_biased=p1).split()
    want = np.array(toks[1:], dtype=np.uint64).reshape(-1, n_pi)
    assert np.array_equal(wp.pattern_words(n_pi, P, seed, frac, p1), want)
    assert np.array_equal(wp.pattern_words(n_pi, P, seed, frac, p1, rounds=1), want[:1])


def test_c2_inputs_match_the_benchmark_workload():
    w = gen.workload("c2")
    got = wp.c2_inputs(rounds=2, n_output_faults=16)
    assert got["ckt"] == w["ckt"]
    site, pin, val = _flst_arrays(w["flst"])
    assert got["n_faults"] == len(site)
    out = np.nonzero(pin == 0)[0][:16]
    want = "%d\n%s\n" % (len(out), "\n".join("%d %d" % (site[i], val[i]) for i in out))
    assert got["flst"] == want
    toks = w["ptn"].split(None, 2001)
    assert np.array_equal(got["words"], np.array(toks[1:2001], dtype=np.uint64).reshape(2, 1000))
