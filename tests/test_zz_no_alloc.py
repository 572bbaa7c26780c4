"""fsimb_good_po_noalloc: the entry point for callers that may not allocate
device memory (a memory budget fixed up front, or a loop that cannot take the
synchronisation of cudaMalloc/cudaFree).  Its PO words must equal the good
values of the regular entry point (fsimb_run + fsimb_good_values), bit for
bit, on two calls in a row that share its static scratch array.  This file is
collected last on purpose."""
import ctypes

import numpy as np
import pytest

from lsim_b200 import Simulator, gen
from lsim_b200 import _lib

pytestmark = pytest.mark.gpu


def _call(sim, words, n_words, n_po):
    import torch
    d_in = torch.from_numpy(np.ascontiguousarray(words).view(np.int64)).cuda()
    d_out = torch.zeros((n_words, n_po), dtype=torch.int64, device="cuda")
    code = _lib.lib().fsimb_good_po_noalloc(sim._h, ctypes.c_void_p(d_in.data_ptr()), n_words,
                                            ctypes.c_void_p(d_out.data_ptr()),
                                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(code, sim._h)
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(np.uint64)


def test_no_alloc_matches_regular_entry_point():
    w = gen.generate(n_gates=3000, n_pi=40, n_po=30, n_levels=25, n_patterns=3000, seed=91,
                     type_mask=gen.ALL_TYPES, faults="outputs")
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    sim.run()  # places the circuit on the device; the regular good values come from here
    n_pi, n_po, n_g = sim.num_PIs(), sim.num_POs(), sim.num_gates()
    P = sim.info().num_patterns
    words = sim.patterns()
    W = words.shape[0]
    # two calls in a row over different rounds and word counts
    for r0, r1 in [(0, 32), (32, W)]:
        out = _call(sim, words[r0:r1], r1 - r0, n_po)
        for k, rd in enumerate(range(r0, r1)):
            bits = 64 if P // (64 * (rd + 1)) else P % 64
            mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(~np.uint64(0))
            ref = sim.good_values(rd)[n_pi + n_g:]
            assert np.array_equal(out[k] & mask, ref), rd


def test_no_alloc_second_circuit_after_a_larger_one():
    """A smaller, different circuit called after a larger one through the same
    static array: nothing of the first circuit's values may leak into it."""
    big = gen.generate(n_gates=6000, n_pi=48, n_po=40, n_levels=30, n_patterns=2048, seed=93,
                       faults="outputs")
    small = gen.generate(n_gates=700, n_pi=20, n_po=15, n_levels=12, n_patterns=2048, seed=94,
                         type_mask=gen.ALL_TYPES, faults="outputs")
    sims = []
    for w in (big, small):
        s = Simulator(0)
        s.read_text(w["ckt"], w["flst"], w["ptn"])
        s.run()
        sims.append(s)
    for s in sims:
        words = s.patterns()[:32]
        out = _call(s, words, 32, s.num_POs())
        first_po = s.num_PIs() + s.num_gates()
        for rd in (0, 17, 31):
            assert np.array_equal(out[rd], s.good_values(rd)[first_po:]), rd


def test_no_alloc_rejects_out_of_range():
    w = gen.generate(n_gates=200, n_pi=8, n_po=6, n_levels=8, n_patterns=128, seed=5)
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    with pytest.raises(_lib.FsimbError) as e:  # circuit not yet on the device
        _call(sim, sim.patterns(), 2, 6)
    assert e.value.code == _lib.ERR_STATE
    sim.run()
    with pytest.raises(_lib.FsimbError) as e:
        _call(sim, np.zeros((33, 8), dtype=np.uint64), 33, 6)
    assert e.value.code == _lib.ERR_ARG
    big = gen.generate(n_gates=40000, n_pi=100, n_po=50, n_levels=30, n_patterns=64, seed=6)
    sim2 = Simulator(0)
    sim2.read_text(big["ckt"], big["flst"], big["ptn"])
    sim2.run()
    with pytest.raises(_lib.FsimbError) as e:
        _call(sim2, sim2.patterns(), 1, 50)
    assert e.value.code == _lib.ERR_LIMIT and "32768" in str(e.value)
