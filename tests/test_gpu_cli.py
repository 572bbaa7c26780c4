"""The drop-in command-line tools (lsim_b200/bin) on the reference's unit-test
fixtures: `fsimb_simple` prints the same `arr[i] = v` good-machine words as
main/simple.cpp and writes per-fault results equal to the oracle's;
`fsimb_ma_partition` accepts MA_cuda_partition's arguments."""
import os
import subprocess

import numpy as np
import pytest

from lsim_b200 import build
from tests.oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def _write(tmp_path, c):
    paths = []
    for ext in ("ckt", "flst", "ptn"):
        p = tmp_path / ("c." + ext)
        p.write_text(c[ext])
        paths.append(str(p))
    return paths


@pytest.mark.parametrize("t", [0, 5, 6])
def test_simple_matches_reference_output(basics, tmp_path, t):
    build.build()
    c, a = basics["cases"][t], basics["answers"]
    ckt, flst, ptn = _write(tmp_path, c)
    out = tmp_path / "faults.txt"
    r = subprocess.run([os.path.join(build.BIN, "fsimb_simple"), ckt, flst, ptn, str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    arr = [int(line.split("=")[1]) for line in r.stdout.splitlines() if line.startswith("arr[")]
    assert arr == a["pi_ans"][t] + a["gate_ans"][t] + a["po_ans"][t]
    rows = [list(map(int, line.split())) for line in out.read_text().splitlines()[1:]]
    ref = Oracle(c["ckt"], c["flst"], c["ptn"]).simulate()
    assert [row[3] for row in rows] == list(ref["detected"])
    assert [row[4] for row in rows] == list(ref["first"])
    assert [row[5] for row in rows] == list(ref["count"])
    table = [v for row in rows for v in (row[6], row[7])]
    assert table == a["found_flst_2_ptn_ans"][t]
    dot = tmp_path / "g.dot"
    r = subprocess.run([os.path.join(build.BIN, "fsimb_simple"), ckt, flst, ptn, str(dot)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and dot.read_text().startswith("digraph G {")


def test_ma_partition_arguments(basics, tmp_path):
    build.build()
    ckt, flst, ptn = _write(tmp_path, basics["cases"][0])
    r = subprocess.run([os.path.join(build.BIN, "fsimb_ma_partition"), ckt, flst, ptn, "unused.hgr",
                        "unused.out", "2"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.count("run ") == 2
    r = subprocess.run([os.path.join(build.BIN, "fsimb_ma_partition"), ckt], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1 and "Usage" in r.stderr
