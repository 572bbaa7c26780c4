"""The header-only C++ mirror of fsim::Simulator (include/fsimb.hpp), built
and run like a reference caller: host-only reading and introspection here,
the full run on a GPU."""
import os
import subprocess

import pytest

from lsim_b200 import build
from tests.oracle_lib import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    build.build()
    exe = str(tmp_path_factory.mktemp("shim") / "shim_check")
    subprocess.check_call(["/usr/bin/g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "shim_check.cpp"), "-o", exe,
                           "-L" + build.HERE, "-lfsimb200", "-Wl,-rpath," + build.HERE])
    return exe


def _files(tmp_path, c):
    out = []
    for ext in ("ckt", "flst", "ptn"):
        p = tmp_path / ("c." + ext)
        p.write_text(c[ext])
        out.append(str(p))
    return out


def _parse(stdout):
    d = {}
    for line in stdout.splitlines():
        k, *v = line.split()
        d[k] = [int(x) for x in v]
    return d


@pytest.mark.parametrize("t", [0, 3, 6])
def test_shim_reads_like_the_reference(shim, basics, tmp_path, t):
    c, a = basics["cases"][t], basics["answers"]
    ckt, flst, ptn = _files(tmp_path, c)
    r = subprocess.run([shim, "-1", ckt, flst, ptn, str(tmp_path / "g.dot")], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    d = _parse(r.stdout)
    assert d["num"] == a["num_vars_ans"][t]
    assert d["tpg"] == a["tpg_ans"][t]
    assert d["per_level"] == a["num_gate_per_lvl_ans"][t]
    assert (tmp_path / "g.dot").read_text().startswith("digraph G {")
    n = sum(a["num_vars_ans"][t][:3])
    assert d["elem_idx"] == list(range(n))
    o = Oracle(c["ckt"], c["flst"], c["ptn"])
    assert d["elem_level"] == [int(x) for x in o.levels()]
    assert d["elem_type"] == [int(x) for x in o.types()]
    assert d["type_names_ok"] == [1]


def test_shim_missing_file_message(shim, tmp_path):
    r = subprocess.run([shim, "-1", str(tmp_path / "nope.ckt"), "a", "b", str(tmp_path / "g.dot")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    assert r.stdout.strip() == "error: cannot open circut file " + str(tmp_path / "nope.ckt")


@pytest.mark.gpu
@pytest.mark.parametrize("t", range(7))
def test_shim_runs_like_the_reference(shim, basics, tmp_path, t):
    c, a = basics["cases"][t], basics["answers"]
    ckt, flst, ptn = _files(tmp_path, c)
    r = subprocess.run([shim, "0", ckt, flst, ptn, str(tmp_path / "g.dot")], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    d = _parse(r.stdout)
    assert d["g_pi"] == a["pi_ans"][t]
    assert d["g_gate"] == a["gate_ans"][t]
    assert d["gate_output_values"] == d["g_gate"]
    assert d["g_po"] == a["po_ans"][t]
    assert d["found"] == a["found_flst_2_ptn_ans"][t]
