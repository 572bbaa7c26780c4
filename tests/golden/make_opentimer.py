"""Regenerates ``opentimer_ref.json``: OpenTimer-style dumps and the .ckt text
the reference converter (fsim/parser.py) writes for them.

The reference keeps each driving pin's sinks in a Python set, so its output
can change with the interpreter's hash seed.  Every case here is run under
several seeds (PYTHONHASHSEED) and kept only if all of them give the same
netlist -- wire lines in the same order with the same sinks, sink order
aside -- so that the fixture pins the reference's behaviour, not one hash
order.  The cases where that holds by construction:
  * fanout-free dumps (one sink per driving pin), with and without loops,
    in bfs and dfs mode;
  * layered dumps (every cell fed by the layer just before it; loop inputs
    from a deeper layer) in bfs mode: no edge joins two elements at the same
    breadth-first depth;
  * a small dump whose names are prefixes of one another (u1, u12), which
    records the reference's prefix match;
  * a small dump with cell types missing from the tables (pin 0 and the AND
    default, with the reference's warnings).

``compat`` records hold dumps whose output does depend on the hash seed
(fanout and equal-depth edges), with the reference's exact output under
PYTHONHASHSEED 0, 5 and 11 and the interpreter version that produced it:
the converter's compat mode must reproduce those bytes under the same seed
and interpreter.

Run from the repository root with the reference tree named by
LSIM_REFERENCE (default: a ``reference`` directory beside the repository):  ``python tests/golden/make_opentimer.py``
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("LSIM_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
sys.path.insert(0, ROOT)

from lsim_b200 import gen  # noqa: E402

SEEDS = (0, 1, 2, 3, 4, 5)

PREFIX_DUMP = """module top;
// Start PIs
input a;

// Start POs
output y;

// Start wires
wire n1;
wire n5;
wire n12;

// Start cells
NAND2_X1 u1 ( .A1(a), .A2(n5), .ZN(n1) );
INV_X1 u5 ( .A(n1), .ZN(n5) );
INV_X1 u12 ( .A(n5), .ZN(n12) );
endmodule

digraph TimingGraph {
  "a" -> "u1:A1";
  "u1:A1" -> "u1:ZN";
  "u1:A2" -> "u1:ZN";
  "u1:ZN" -> "u5:A";
  "u5:A" -> "u5:ZN";
  "u5:ZN" -> "u1:A2";
  "u5:ZN" -> "u12:A";
  "u12:A" -> "u12:ZN";
  "u12:ZN" -> "y";
}
"""

LOOSE_DUMP = """module top;
// Start PIs
input a;
input b;
input s;

// Start POs
output y;
output z;

// Start wires
wire m;
wire k;

// Start cells
MUX2_X1 mx ( .A(a), .B(b), .S(s), .Z(m) );
BUF_X2 bf ( .A(m), .Z(k) );
XOR2_X1 xr ( .A(k), .B(a), .Z(z) );
endmodule

digraph TimingGraph {
  "a" -> "mx:A";
  "b" -> "mx:B";
  "s" -> "mx:S";
  "mx:A" -> "mx:Z";
  "mx:Z" -> "bf:A";
  "bf:Z" -> "xr:A";
  "a" -> "xr:B";
  "bf:Z" -> "y";
  "xr:Z" -> "z";
}
"""


def cases():
    out = []
    for s in range(3):
        out.append(("tree_%d" % s, gen.opentimer_dump(24, 30, seed=s, fanout_free=True), ("bfs", "dfs")))
    for s in range(3):
        out.append(("tree_loops_%d" % s,
                    gen.opentimer_dump(30, 36, seed=10 + s, fanout_free=True, loops=4), ("bfs", "dfs")))
    for s in range(2):
        out.append(("layered_%d" % s, gen.opentimer_dump(40, 8, seed=20 + s, layers=6), ("bfs",)))
    for s in range(2):
        out.append(("layered_loops_%d" % s,
                    gen.opentimer_dump(48, 8, seed=30 + s, layers=6, loops=5), ("bfs",)))
    out.append(("prefix_names", PREFIX_DUMP, ("bfs", "dfs")))
    out.append(("unknown_cells", LOOSE_DUMP, ("bfs",)))
    return out


COMPAT_SEEDS = (0, 5, 11)


def compat_cases():
    out = [("fanout_%d" % s, gen.opentimer_dump(40 + 10 * s, 6 + s, seed=50 + s, loops=2 + s), ("bfs", "dfs"))
           for s in range(4)]
    out.append(("prefix_names", PREFIX_DUMP, ("bfs", "dfs")))
    return out


def canonical(ckt):
    """(header, wire lines with sorted sinks, type line) of .ckt text."""
    ls = ckt.strip("\n").split("\n")
    n = int(ls[3])
    wires = []
    for line in ls[4:4 + n]:
        v = [int(x) for x in line.split()]
        wires.append([v[0], v[1], v[2]] + sorted(zip(v[3::2], v[4::2])))
    return ls[:4], wires, ls[4 + n:]


def run_reference(dump, mode, seed, tmp):
    src = os.path.join(tmp, "dump.txt")
    dst = os.path.join(tmp, "out.ckt")
    with open(src, "w") as f:
        f.write(dump)
    r = subprocess.run([sys.executable, os.path.join(REF, "fsim", "parser.py"), src, dst, mode],
                       env=dict(os.environ, PYTHONHASHSEED=str(seed)), capture_output=True,
                       text=True, check=True)
    with open(dst) as f:
        return f.read(), r.stdout


def main():
    recs, dumps = [], {}
    with tempfile.TemporaryDirectory(dir=HERE) as tmp:
        for name, dump, modes in cases():
            for mode in modes:
                outs = [run_reference(dump, mode, s, tmp) for s in SEEDS]
                canon = [json.dumps(canonical(o[0])) for o in outs]
                if len(set(canon)) != 1:
                    raise SystemExit("%s/%s: the reference's output depends on the hash seed" %
                                     (name, mode))
                warnings = [ln for ln in outs[0][1].split("\n") if ln.startswith("Warning")]
                dumps[name] = dump
                recs.append(dict(name=name, mode=mode, ckt=outs[0][0], n_warnings=len(warnings)))
        compat = []
        for name, dump, modes in compat_cases():
            for mode in modes:
                outs = {str(sd): run_reference(dump, mode, sd, tmp)[0] for sd in COMPAT_SEEDS}
                dumps[name] = dump
                compat.append(dict(name=name, mode=mode, ckt=outs))
    path = os.path.join(HERE, "opentimer_ref.json")
    with open(path, "w") as f:
        json.dump(dict(source="fsim/parser.py run under PYTHONHASHSEED in %s" % (SEEDS,),
                       dumps=dumps, cases=recs, python="%d.%d" % sys.version_info[:2], compat=compat),
                  f, indent=0)
        f.write("\n")
    print("wrote %s: %d cases" % (path, len(recs)))


if __name__ == "__main__":
    main()
