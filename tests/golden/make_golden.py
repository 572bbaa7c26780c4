"""Regenerates the golden fixtures in this folder.

1. ``test_basics_golden.json``: the seven netlist/fault/pattern fixtures and
   their answer tables, read as text from the reference's unit test
   (unittests/test_basics.cpp:8-345).  The C string literals there use
   backslash-newline continuations, which the compiler removes; the strings
   are stored as the compiler sees them.
2. ``test_basics_dot.json``: the reference's Graphviz output
   (Simulator::visualization_graph) for those seven fixtures.
3. ``ref_cases.json``: small synthetic circuits (all gate types including
   XNOR, CLKBUF and MUX, several rounds, partial last rounds) run through the
   reference's own simulator compiled into ``oracle/_ref`` (``make -C oracle
   ref``), recording per-fault detected / first / count, the reference's
   found_fault_to_pattern table and the last round's good values.

Run from the repository root with the reference tree named by
LSIM_REFERENCE (default: a ``reference`` directory beside the repository):  ``python tests/golden/make_golden.py``
"""
import ctypes
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("LSIM_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def _strip_comments(src):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _block(src, name):
    i = src.index(name)
    j = src.index("{", i)
    depth = 0
    for k in range(j, len(src)):
        if src[k] == "{":
            depth += 1
        elif src[k] == "}":
            depth -= 1
            if depth == 0:
                return src[j + 1:k]
    raise ValueError(name)


def _nums(s):
    return [int(x) for x in re.findall(r"\d+", s)]


def extract_test_basics():
    path = os.path.join(REF, "unittests", "test_basics.cpp")
    raw = open(path).read().replace("\\\n", "")
    names = re.findall(r"^\s*//\s*(\w+)\s*$", raw.split("test_cases{", 1)[1].split("};", 1)[0], re.M)
    src = _strip_comments(raw)
    body = _block(src, "test_cases{")
    strings = re.findall(r'"((?:[^"\\]|\\.)*)"', body)
    assert len(strings) == 21, len(strings)
    cases = []
    for i in range(7):
        cases.append({"name": names[i] if i < len(names) else "case%d" % i,
                      "ckt": strings[3 * i], "flst": strings[3 * i + 1], "ptn": strings[3 * i + 2]})
    answers = {}
    for key in ["num_vars_ans", "tpg_ans", "num_gate_per_lvl_ans", "pi_lvl_ans", "gate_lvl_ans",
                "po_lvl_ans", "fault_ans", "ptn_val_ans", "pi_ans", "gate_ans", "po_ans",
                "found_flst_2_ptn_ans"]:
        blk = _block(src, key + " =")
        answers[key] = [_nums(g) for g in re.findall(r"\{([^{}]*)\}", blk)]
        assert len(answers[key]) == 7, key
    for key in ["fault_size_ans", "ptn_size_ans"]:
        answers[key] = _nums(_block(src, key + " ="))
        assert len(answers[key]) == 7, key
    return {"source": "unittests/test_basics.cpp:8-345", "cases": cases, "answers": answers}


def ref_cases():
    """Synthetic cases through the reference simulator (oracle/_ref)."""
    sys.path.insert(0, ROOT)
    from lsim_b200 import gen
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libfsim_ref.so"))
    lib.ref_load_text.restype = ctypes.c_void_p
    lib.ref_load_text.argtypes = [ctypes.c_char_p, ctypes.c_size_t] * 3
    lib.ref_num.restype = ctypes.c_uint64
    lib.ref_num.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.ref_free.argtypes = [ctypes.c_void_p]
    lib.ref_run_table.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]

    class R(ctypes.Structure):
        _fields_ = [("detected", ctypes.c_uint8), ("ref_flag", ctypes.c_uint8),
                    ("pad", ctypes.c_uint8 * 6), ("first", ctypes.c_int64),
                    ("count", ctypes.c_uint64), ("ref_rd", ctypes.c_uint64)]
    lib.ref_simulate.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                 ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(R)]
    specs = [
        # name, gates, pi, po, levels, type mask, patterns, fault kind, seed
        ("all_types_mux", 60, 6, 4, 8, 0x1FF, 200, "outputs", 11),
        ("xnor_clkbuf_deep", 120, 8, 6, 20, (1 << 6) | (1 << 8) | (1 << 1) | (1 << 3), 130, "outputs", 12),
        ("mux_heavy", 80, 6, 5, 10, (1 << 7) | (1 << 0) | (1 << 2), 64, "outputs", 13),
        ("partial_round", 200, 10, 8, 12, 0x17F, 100, "outputs", 14),
        ("four_rounds", 300, 16, 12, 15, 0x17F, 256, "outputs", 15),
        ("single_partial", 40, 5, 3, 6, 0x17F, 37, "outputs", 16),
    ]
    out = []
    for name, g, pi, po, lv, mask, P, kind, seed in specs:
        w = gen.generate(n_gates=g, n_pi=pi, n_po=po, n_levels=lv, type_mask=mask, seed=seed,
                         n_patterns=P, faults=kind)
        ck, fl, pt = w["ckt"].encode(), w["flst"].encode(), w["ptn"].encode()
        h = lib.ref_load_text(ck, len(ck), fl, len(fl), pt, len(pt))
        F = lib.ref_num(h, 5)
        N = lib.ref_num(h, 0) + lib.ref_num(h, 1) + lib.ref_num(h, 2)
        R_ = lib.ref_num(h, 4)
        res = (R * F)()
        lib.ref_simulate(h, 0, F, 0, R_, 1, res)
        table = (ctypes.c_uint64 * (2 * F))()
        good = (ctypes.c_uint64 * N)()
        lib.ref_run_table(h, 0, 1, table, good)
        out.append({"name": name, "ckt": w["ckt"], "flst": w["flst"], "ptn": w["ptn"],
                    "detected": [r.detected for r in res], "first": [r.first for r in res],
                    "count": [r.count for r in res], "table": list(table), "good_last": list(good)})
        lib.ref_free(h)
    return {"source": "reference fsim::Simulator via oracle/_ref (oracle/ref_harness.cpp)",
            "cases": out}


def ref_dot(tb):
    """The reference's visualization_graph output for each unit-test fixture."""
    import tempfile
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libfsim_ref.so"))
    lib.ref_load_text.restype = ctypes.c_void_p
    lib.ref_load_text.argtypes = [ctypes.c_char_p, ctypes.c_size_t] * 3
    lib.ref_visualize.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    lib.ref_free.argtypes = [ctypes.c_void_p]
    out = []
    with tempfile.TemporaryDirectory() as d:
        for c in tb["cases"]:
            ck, fl, pt = c["ckt"].encode(), c["flst"].encode(), c["ptn"].encode()
            h = lib.ref_load_text(ck, len(ck), fl, len(fl), pt, len(pt))
            path = os.path.join(d, "g.dot")
            lib.ref_visualize(h, path.encode())
            out.append({"name": c["name"], "dot": open(path).read()})
            lib.ref_free(h)
    return {"source": "fsim::Simulator::visualization_graph via oracle/_ref", "cases": out}


def main():
    tb = extract_test_basics()
    with open(os.path.join(HERE, "test_basics_dot.json"), "w") as f:
        json.dump(ref_dot(tb), f, indent=1)
    with open(os.path.join(HERE, "test_basics_golden.json"), "w") as f:
        json.dump(tb, f, indent=1)
    rc = ref_cases()
    with open(os.path.join(HERE, "ref_cases.json"), "w") as f:
        json.dump(rc, f)
    print("wrote", len(tb["cases"]), "unit-test fixtures and", len(rc["cases"]), "reference cases")


if __name__ == "__main__":
    main()
