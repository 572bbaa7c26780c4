"""Fault dropping with an N-detect limit, and the bounded wait of the sweep
kernel.

N-detect: a fault leaves the simulation after the 2,048-pattern tile in
which its detection count reaches N; its first pattern is exact and its
count covers the patterns up to the end of that tile.  The expectation is
built from the oracle's per-tile results.

Bounded wait: with fsimb_opts.wait_test one sweep CTA waits on a barrier
that no copy completes.  The wait gives up after its time limit (20 ms),
the CTA lets its own record copies land and leaves, and the run fails with
FSIMB_ERR_CUDA and no results; the next run on the same handle succeeds."""
import numpy as np
import pytest

from lsim_b200 import FsimbError, Simulator, gen
from tests.oracle_lib import Oracle

pytestmark = pytest.mark.gpu

TILE_ROUNDS = 32


def _workload():
    return gen.generate(n_gates=1500, n_pi=24, n_po=20, n_levels=25, n_patterns=5 * 2048 + 100,
                        seed=31, faults="collapsed", biased_pi_frac=0.5)


def _per_tile(o):
    tiles = (o.W + TILE_ROUNDS - 1) // TILE_ROUNDS
    return [o.simulate(rd0=t * TILE_ROUNDS, rd1=min(o.W, (t + 1) * TILE_ROUNDS)) for t in range(tiles)]


@pytest.mark.parametrize("n_detect", [1, 3, 40])
def test_n_detect_drop_vs_oracle(n_detect):
    w = _workload()
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    sim.run(drop=True, n_detect=n_detect)
    got = sim.results()
    o = Oracle(w["ckt"], w["flst"], w["ptn"])
    full = o.simulate()
    tiles = _per_tile(o)
    cum = np.zeros(len(full), dtype=np.uint64)
    want = np.zeros(len(full), dtype=np.uint64)
    done = np.zeros(len(full), dtype=bool)
    for t in tiles:
        cum += t["count"]
        newly = ~done & (cum >= n_detect)
        want[newly] = cum[newly]
        done |= newly
    want[~done] = cum[~done]
    assert np.array_equal(got["count"], want)
    assert np.array_equal(got["first_pattern"], full["first"])
    assert np.array_equal(got["detected"], full["detected"])
    # some faults were dropped early and some ran to the end
    assert done.any() and (want < full["count"]).any()


def test_wait_limit_fails_the_run_and_the_handle_recovers():
    w = gen.generate(n_gates=2000, n_pi=32, n_po=32, n_levels=30, n_patterns=2048, seed=5,
                     faults="collapsed")
    sim = Simulator(0)
    sim.read_text(w["ckt"], w["flst"], w["ptn"])
    with pytest.raises(FsimbError) as e:
        sim.run(sweep_variant="shared", wait_test=True)
    assert e.value.code == 3  # FSIMB_ERR_CUDA
    assert "time limit" in str(e.value)
    with pytest.raises(FsimbError) as e2:
        sim.results()
    assert e2.value.code == 4  # FSIMB_ERR_STATE: results were discarded
    sim.run()
    ref = Oracle(w["ckt"], w["flst"], w["ptn"]).simulate()
    got = sim.results()
    assert np.array_equal(got["count"], ref["count"])
    assert np.array_equal(got["first_pattern"], ref["first"])
