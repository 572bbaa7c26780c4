"""OpenTimer netlist dumps to LSIM's .ckt text (the job of fsim/parser.py).

Input: the text OpenTimer writes for a gate-level design -- a "// Start
PIs" / "// Start POs" / "// Start wires" / "// Start cells" listing, then a
"digraph TimingGraph {" section of pin-to-pin edges ("u1:ZN" -> "u2:A1";).
Output: .ckt text with element ids PIs, POs, cells in listing order, one
wire line per driving pin, and the gate type of every cell.

What follows the reference converter (fsim/parser.py:11-31, 36-105,
140-227):
  * the section bounds (a PI/PO/wire section ends one line before the next
    marker, the cell section two lines before the graph, the graph two
    lines before the end of the file);
  * the cell tables: pin numbers by cell (the part of the cell type before
    '_'), output pin 0, inputs 1-4; gate type by the first matching prefix
    of INV, AND, OR, XOR, NAND, NOR, XNOR, MUX, CLKBUF, AOI21, AOI22, DFF,
    OAI21, OAI22 (the AOI cells become NAND, OAI cells NOR, DFF NAND), an
    unknown cell type becomes AND with a warning;
  * edges inside one cell are dropped; a PI is a source on pin 0, a PO a
    sink on pin 1; a cell pin missing from the tables is written as pin 0
    with a warning (strict=True makes it an error);
  * loop breaking, modes "bfs" and "dfs": a walk from the PIs in listing
    order (breadth-first or depth-first), each element taken once; an
    element's first output pin found among "", ":Z", ":ZN", ":Q", ":Y",
    ":QN" loses its edges to every element taken before it.  In "bfs" mode
    that keeps exactly the edges into the next breadth-first layer: besides
    every loop, it cuts each input that comes from an element deeper than
    the shallowest input of its cell.

Where it differs, on purpose:
  * the reference keeps each pin's sinks in a Python set, so their order --
    and, through the walk, which edges it removes -- changes with the
    interpreter's hash seed; here sinks keep the order of the dump, so the
    output is the same on every run (the two agree wherever the reference
    agrees with itself across hash seeds);
  * the reference removes the edges to every sink whose name merely starts
    with the taken element's name (u1 also matches u12:A); here the names
    must be equal;
  * compat=True (--compat) undoes the first two: sinks in Python sets and
    removal by prefix, so that the output is byte-identical to the
    reference's under the same interpreter and PYTHONHASHSEED;
  * mode "loops" (not in the reference) cuts only edges that close a
    cycle: a topological walk from the PIs that, whenever every element left
    waits on a cycle, cuts the unprocessed inputs of the waiting element
    that has the fewest.  An acyclic netlist converts unchanged; a cycle
    through one input of a cell costs that one input.
"""
import heapq
from collections import deque

# Pin numbers of each cell (fsim/parser.py:36-54).
PIN_TABLE = {
    "CLKBUF": {"A": 1, "Z": 0},
    "INV": {"A": 1, "ZN": 0},
    "AND2": {"A": 1, "B": 2, "Y": 0},
    "NAND2": {"A1": 1, "A2": 2, "ZN": 0},
    "NAND3": {"A1": 1, "A2": 2, "A3": 3, "ZN": 0},
    "NAND4": {"A1": 1, "A2": 2, "A3": 3, "A4": 4, "ZN": 0},
    "NOR2": {"A1": 1, "A2": 2, "ZN": 0},
    "NOR3": {"A1": 1, "A2": 2, "A3": 3, "ZN": 0},
    "NOR4": {"A1": 1, "A2": 2, "A3": 3, "A4": 4, "ZN": 0},
    "AOI21": {"A": 1, "B1": 2, "B2": 3, "ZN": 0},
    "AOI22": {"A1": 1, "A2": 2, "B1": 3, "B2": 4, "ZN": 0},
    "DFF": {"D": 1, "CK": 2, "Q": 0},
    "OAI21": {"A": 1, "B1": 2, "B2": 3, "ZN": 0},
    "OAI22": {"A1": 1, "A2": 2, "B1": 3, "B2": 4, "ZN": 0},
    "AND2X1": {"A": 1, "B": 2, "Y": 0},
    "INVX1": {"A": 1, "Y": 0},
    "NAND3X1": {"A": 1, "B": 2, "C": 3, "Y": 0},
}

# An opt-in table (convert(..., pin_table=NANGATE45_PINS)) for the cells of
# Nangate45-style libraries that the table above lacks or names otherwise
# (its AND2 has pins A, B, Y).  Inputs number 1-4 in pin order, a MUX's
# select is pin 5, the output is pin 0; BUF becomes a one-input AND, which
# is a buffer.  Not in the reference: with it a dump converts without
# pin-0 fallbacks.
NANGATE45_PINS = dict(
    {"AND%d" % n: dict({"A%d" % i: i for i in range(1, n + 1)}, ZN=0) for n in (2, 3, 4)},
    **{"OR%d" % n: dict({"A%d" % i: i for i in range(1, n + 1)}, ZN=0) for n in (2, 3, 4)},
    XOR2={"A": 1, "B": 2, "Z": 0},
    XNOR2={"A": 1, "B": 2, "ZN": 0},
    BUF={"A": 1, "Z": 0},
    MUX2={"A": 1, "B": 2, "S": 5, "Z": 0},
)

# Gate type by cell-type prefix, first match wins (fsim/parser.py:57-72,
# 82-88); GateType numbering of fsim/base_ppg.hpp.
TYPE_PREFIXES = [
    ("INV", 0), ("AND", 1), ("OR", 2), ("XOR", 3), ("NAND", 4), ("NOR", 5), ("XNOR", 6),
    ("MUX", 7), ("CLKBUF", 8), ("AOI21", 4), ("AOI22", 4), ("DFF", 4), ("OAI21", 5), ("OAI22", 5),
]

# Output pin names tried, in order, for an element's driving pin during the
# walk (fsim/parser.py:185).
OUTPUT_SUFFIXES = ["", ":Z", ":ZN", ":Q", ":Y", ":QN"]

MODES = ("bfs", "dfs", "loops")


def gate_type(cell_type, warnings=None):
    """Gate type number of a cell type such as NAND2_X1."""
    for prefix, t in TYPE_PREFIXES:
        if cell_type.startswith(prefix):
            return t
    if warnings is not None:
        warnings.append("%s is an unknown gate name: taken as AND" % cell_type)
    return 1


def _section(lines, marker):
    try:
        return lines.index(marker)
    except ValueError:
        raise ValueError("not an OpenTimer dump: no line %r" % marker) from None


def parse_dump(text):
    """(pis, pos, cells, edges) of a dump: names in listing order, cells as
    (name, cell type), edges as (from pin, to pin) in dump order
    (fsim/parser.py:11-34)."""
    lines = text.split("\n")
    i_pi = _section(lines, "// Start PIs")
    i_po = _section(lines, "// Start POs")
    i_wire = _section(lines, "// Start wires")
    i_cell = _section(lines, "// Start cells")
    i_graph = _section(lines, "digraph TimingGraph {")
    try:
        pis = [ln.split()[1][:-1] for ln in lines[i_pi + 1:i_po - 1]]
        pos = [ln.split()[1][:-1] for ln in lines[i_po + 1:i_wire - 1]]
        cells = [(ln.split()[1], ln.split()[0]) for ln in lines[i_cell + 1:i_graph - 2]]
    except IndexError:
        raise ValueError("a PI, PO or cell line has fewer than two words") from None
    edges = [tuple(part.strip(' ";') for part in ln.split(" -> "))
             for ln in lines[i_graph + 1:-2] if "->" in ln]
    for e in edges:
        if len(e) != 2:
            raise ValueError("edge line with %d arrows" % (len(e) - 1))
    return pis, pos, cells, edges


def _walk_reference(sinks, pis, po_set, mode, warnings):
    """Loop breaking of fsim/parser.py:163-211 (modes bfs / dfs)."""
    todo = deque(pis)
    taken = set()
    while todo:
        cur = todo.popleft() if mode == "bfs" else todo.pop()
        if cur in taken:
            continue
        taken.add(cur)
        key = next((cur + s for s in OUTPUT_SUFFIXES if cur + s in sinks), None)
        if key is None:
            if cur not in po_set and warnings is not None:
                warnings.append("no connection found for %s" % cur)
            continue
        # `taken` does not change while one element's sinks are looked at, so
        # the reference's removal per taken sink element is one pass here
        outs = [x.split(":")[0] for x in sinks[key]]
        drop = {out for out in outs if out in taken}
        if drop:
            sinks[key] = [x for x, out in zip(sinks[key], outs) if out not in drop]
        todo.extend(out for out in outs if out not in taken)


def _walk_compat(sinks, pis, po_set, mode, warnings):
    """The reference's walk step for step on its own data structure (sinks
    in Python sets, removal by name prefix, one rebuild per taken sink
    element), so that set iteration orders, and with them the output, are
    the reference's under the same interpreter and hash seed."""
    todo = deque(pis)
    taken = set()
    while todo:
        cur = todo.popleft() if mode == "bfs" else todo.pop()
        if cur in taken:
            continue
        taken.add(cur)
        key = next((cur + s for s in OUTPUT_SUFFIXES if cur + s in sinks), None)
        if key is None:
            if cur not in po_set and warnings is not None:
                warnings.append("no connection found for %s" % cur)
            continue
        for out in [x.split(":")[0] for x in sinks[key]]:
            if out in taken:
                sinks[key] = {x for x in sinks[key] if not x.startswith(out)}
            else:
                todo.append(out)


def _walk_loops(sinks, listing):
    """Cuts the fewest inputs it can to make the netlist acyclic: a
    topological walk (Kahn) from the elements without inputs, PIs first;
    when every element left waits on a cycle, the waiting element with the
    fewest inputs still unprocessed (first in `listing` order on ties; POs
    last, so that a PO keeps its driver) loses
    those inputs and the walk goes on.  Edges of an acyclic netlist are
    never cut."""
    out_arcs, in_arcs = {}, {}
    for key, lst in sinks.items():
        u = key.split(":")[0]
        for i, dst in enumerate(lst):
            out_arcs.setdefault(u, []).append((key, i))
            in_arcs.setdefault(dst.split(":")[0], []).append((key, i))
    rank = {n: k for k, n in enumerate(listing)}
    indeg = {v: len(a) for v, a in in_arcs.items()}
    todo = deque(n for n in listing if indeg.get(n, 0) == 0)
    waiting = [(d, rank[v], v) for v, d in indeg.items()]
    heapq.heapify(waiting)
    done, cut = set(), set()
    while True:
        while todo:
            u = todo.popleft()
            done.add(u)
            for arc in out_arcs.get(u, ()):
                if arc in cut:
                    continue
                v = sinks[arc[0]][arc[1]].split(":")[0]
                indeg[v] -= 1
                if indeg[v] == 0:
                    todo.append(v)
                else:
                    heapq.heappush(waiting, (indeg[v], rank[v], v))
        while waiting and (waiting[0][2] in done or indeg[waiting[0][2]] != waiting[0][0]):
            heapq.heappop(waiting)
        if not waiting:
            break
        _, _, v = heapq.heappop(waiting)
        for arc in in_arcs[v]:
            if arc[0].split(":")[0] not in done:
                cut.add(arc)
        indeg[v] = 0
        todo.append(v)
    for key in sinks:
        sinks[key] = [x for i, x in enumerate(sinks[key]) if (key, i) not in cut]


def convert(text, mode="bfs", pin_table=None, strict=False, warnings=None, compat=False):
    """.ckt text of an OpenTimer dump.
    mode: "bfs" or "dfs" (the reference's loop breaking) or "loops".
    pin_table: extra cells (name -> {pin: number}) beside PIN_TABLE.
    strict: an edge to a pin missing from the tables raises ValueError
    instead of being written as pin 0.
    warnings: a list that receives the notes the reference prints.
    compat: keep sinks in Python sets and remove them by name prefix, as
    the reference does: the output is then byte-identical to fsim/parser.py
    run by the same interpreter under the same PYTHONHASHSEED (bfs and dfs)."""
    if mode not in MODES:
        raise ValueError("unknown mode %r (bfs, dfs or loops)" % (mode,))
    if compat and mode == "loops":
        raise ValueError("compat reproduces the reference's bfs and dfs modes only")
    pins_of = dict(PIN_TABLE)
    if pin_table:
        pins_of.update(pin_table)
    pis, pos, cells, edges = parse_dump(text)

    ids = {}
    for name in pis + pos + [c[0] for c in cells]:
        if name in ids:
            raise ValueError("element %s listed twice" % name)
        ids[name] = len(ids)
    cell_kind = {name: ctype.split("_")[0] for name, ctype in cells}
    pi_set, po_set = set(pis), set(pos)
    types = [gate_type(ctype, warnings) for _, ctype in cells]

    # driving pin -> sinks, in dump order, each sink once (fsim/parser.py:94-102)
    sinks, seen = {}, set()
    for src, dst in edges:
        if src.split(":")[0] == dst.split(":")[0]:
            continue  # an arc inside one cell
        if compat:
            sinks.setdefault(src, set()).add(dst)
        elif (src, dst) not in seen:
            seen.add((src, dst))
            sinks.setdefault(src, []).append(dst)

    if compat:
        _walk_compat(sinks, pis, po_set, mode, warnings)
    elif mode == "loops":
        _walk_loops(sinks, pis + [c[0] for c in cells] + pos)
    else:
        _walk_reference(sinks, pis, po_set, mode, warnings)

    def pin_id(s):  # fsim/parser.py:140-160
        if ":" in s:
            name, pin = s.split(":", 1)
            if name not in ids:
                raise ValueError("%s is an unknown gate:pin" % s)
            kind = cell_kind.get(name)
            if kind is not None and kind in pins_of and pin in pins_of[kind]:
                return ids[name], pins_of[kind][pin]
            if strict:
                raise ValueError("no pin number for %s (cell type %s)" % (s, kind))
            if warnings is not None:
                warnings.append("%s for %s not found in the pin table: pin 0" % (pin, name))
            return ids[name], 0
        if s in pi_set:
            return ids[s], 0
        if s in po_set:
            return ids[s], 1
        raise ValueError("%s is an unknown gate:pin" % s)

    out = ["%d" % len(pis), "%d" % len(pos), "%d" % len(cells), "%d" % len(sinks)]
    for src, lst in sinks.items():
        parts = ["%d %d %d" % (pin_id(src) + (len(lst),))] + ["%d %d" % pin_id(d) for d in lst]
        out.append(" ".join(parts))
    out.append(" ".join(str(t) for t in types))
    return "\n".join(out) + "\n"


def convert_file(src, dst, mode="bfs", strict=False, compat=False):
    """fsim/parser.py's command line (python parser.py <in> <out> <mode>):
    python -m lsim_b200.opentimer <in> <out> <mode> [--compat].  Returns the
    warnings."""
    with open(src) as f:
        text = f.read()
    warnings = []
    ckt = convert(text, mode, strict=strict, warnings=warnings, compat=compat)
    with open(dst, "w") as f:
        f.write(ckt)
    return warnings


def main(argv=None):
    import sys
    argv = list(sys.argv[1:] if argv is None else argv)
    compat = "--compat" in argv
    if compat:
        argv.remove("--compat")
    if len(argv) != 3:
        print("usage: python -m lsim_b200.opentimer <dump> <out.ckt> <bfs|dfs|loops> [--compat]",
              file=sys.stderr)
        return 2
    try:
        for w in convert_file(argv[0], argv[1], argv[2], compat=compat):
            print("Warning:", w)
    except (OSError, ValueError) as e:
        print("error:", e, file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
