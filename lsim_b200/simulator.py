"""Python mirror of LSIM's ``fsim::Simulator`` (fsim/simulation.hpp:39-188).

Method names, argument meaning and error behaviour follow the reference:
``read(ckt, flst, ptn)`` takes three paths or three text streams and raises
``RuntimeError`` when a file cannot be opened (fsim/simulation.cpp:24-32);
``run(mode, num_threads)`` simulates every round and fault; the accessors
return the last round's good values, the ``found_fault_to_pattern`` table,
the topological index map and the level counts.  Every mode runs on the B200
through the C ABI; the reference's CPU modes are accepted for source
compatibility and mean the same GPU run.

Beyond the reference: ``results()`` returns, per fault, the detected flag,
the first detecting pattern and the detection count over all patterns.
"""
import ctypes
import enum
import io
import os

import numpy as np

from . import _lib
from ._lib import FsimbError, check

RESULT_DTYPE = np.dtype([("detected", np.uint8), ("ref_last_round_flag", np.uint8),
                         ("pad", np.uint8, 6), ("first_pattern", np.int64),
                         ("count", np.uint64), ("ref_last_rd", np.uint64)])


def _u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


# GateType names of fsim/base_ppg.hpp:19-32, as gateTypeToString gives them.
GATE_TYPE_NAMES = ["INV", "AND", "OR", "XOR", "NAND", "NOR", "XNOR", "MUX", "CLKBUF", "PI", "PO"]


class Element:
    """An element as ElementBase's public interface shows it
    (fsim/base_ppg.hpp:47-50): idx() is the topological index, level() the
    level; output_value() is the element's good-machine word of the last
    round after run() and 0 before (the reference leaves there the word of
    its last faulty-machine simulation).  `type` is the GateType number."""

    __slots__ = ("_idx", "_level", "type", "_value")

    def __init__(self, idx, level, type_, value):
        self._idx, self._level, self.type, self._value = idx, level, type_, value

    def idx(self):
        return self._idx

    def level(self):
        return self._level

    def output_value(self):
        return self._value

    def __repr__(self):
        return "Element(idx=%d, level=%d, type=%s)" % (self._idx, self._level,
                                                       Simulator.gateTypeToString(self.type))


class Simulator:
    class Mode(enum.IntEnum):
        SEQUENTIAL = 0
        PARALLEL_TF = 1
        PARALLEL_OMP = 2
        CUDA_B200 = 3

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        check(_lib.lib().fsimb_create(device, ctypes.byref(h)))
        self._h = h
        self._ran = False

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().fsimb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, code):
        check(code, self._h)

    # ------------------------------------------------------------ reading
    def read(self, ckt, flst, ptn):
        """Paths (str / PathLike) or text streams, like the two reference overloads."""
        if all(isinstance(x, (str, os.PathLike)) for x in (ckt, flst, ptn)):
            for p, what in ((ckt, "circut"), (flst, "fault"), (ptn, "pattern")):
                if not os.path.isfile(p):
                    raise RuntimeError("cannot open %s file %s" % (what, p))
            self._check(_lib.lib().fsimb_load_files(self._h, os.fsencode(ckt), os.fsencode(flst),
                                                    os.fsencode(ptn)))
        else:
            texts = [x.read() if isinstance(x, io.IOBase) or hasattr(x, "read") else x
                     for x in (ckt, flst, ptn)]
            self.read_text(*texts)
        self._ran = False

    def read_text(self, ckt, flst, ptn):
        b = [t.encode() if isinstance(t, str) else bytes(t) for t in (ckt, flst, ptn)]
        self._check(_lib.lib().fsimb_load_buffers(self._h, b[0], len(b[0]), b[1], len(b[1]),
                                                  b[2], len(b[2])))
        self._ran = False

    def set_loader(self, mode="auto", threads=0):
        """Circuit loader for the reads that follow: "auto" (device loader for
        texts of 4 MiB and more on a device handle), "host" or "device"."""
        m = {"auto": _lib.LOAD_AUTO, "host": _lib.LOAD_HOST, "device": _lib.LOAD_DEVICE}[mode]
        self._check(_lib.lib().fsimb_set_loader(self._h, m, int(threads)))

    def load_info(self):
        """How the last circuit was loaded (on_device, handed_back, threads,
        waves, ms_total, ms_tokenize, ms_device)."""
        li = _lib.LoadInfo()
        self._check(_lib.lib().fsimb_get_load_info(self._h, ctypes.byref(li)))
        return li.as_dict()

    def load_circuit(self, ckt):
        b = ckt.encode() if isinstance(ckt, str) else bytes(ckt)
        self._check(_lib.lib().fsimb_load_circuit(self._h, b, len(b)))

    def set_fault_text(self, flst):
        b = flst.encode() if isinstance(flst, str) else bytes(flst)
        self._check(_lib.lib().fsimb_set_fault_text(self._h, b, len(b)))

    def set_faults(self, site, pin, value):
        site = np.ascontiguousarray(site, dtype=np.uint32)
        pin = np.ascontiguousarray(pin, dtype=np.uint8)
        value = np.ascontiguousarray(value, dtype=np.uint8)
        n = len(site)
        self._check(_lib.lib().fsimb_set_faults(
            self._h, site.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
            pin.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            value.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n))

    def set_patterns(self, words, num_patterns):
        w = np.ascontiguousarray(words, dtype=np.uint64).ravel()
        self._check(_lib.lib().fsimb_set_patterns(self._h, _u64p(w), int(num_patterns)))

    # ------------------------------------------------------------ running
    SWEEP_VARIANTS = {"auto": 0, "shared": 1, "global": 2}

    def run(self, mode=Mode.CUDA_B200, num_threads=1, drop=False, words_per_item=0,
            block_threads=0, ctas_per_sm=0, tune=False, stream=None, n_detect=0,
            sweep_variant="auto", wait_test=False):
        """Simulates every fault against every pattern on the GPU.  drop: stop
        simulating a fault after the 2,048-pattern tile in which its count
        reaches n_detect (1 when 0).  sweep_variant: where a sweep keeps its
        live values ("auto", "shared" memory, "global" memory).  wait_test is
        a test hook (see fsimb_opts.wait_test)."""
        o = _lib.Opts(ctypes.sizeof(_lib.Opts), 1 if drop else 0, words_per_item, block_threads,
                      ctas_per_sm, 1 if tune else 0, stream, n_detect,
                      self.SWEEP_VARIANTS[sweep_variant], 1 if wait_test else 0, 0)
        self._check(_lib.lib().fsimb_run(self._h, ctypes.byref(o)))
        self._ran = True

    # ------------------------------------------------------------ results
    def info(self):
        i = _lib.Info()
        self._check(_lib.lib().fsimb_get_info(self._h, ctypes.byref(i)))
        return i

    def stats(self):
        s = _lib.Stats()
        self._check(_lib.lib().fsimb_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

    def results(self):
        n = self.info().num_faults
        out = np.zeros(n, dtype=RESULT_DTYPE)
        self._check(_lib.lib().fsimb_results(
            self._h, out.ctypes.data_as(ctypes.POINTER(_lib.FaultResult)), n))
        return out

    def found_fault_to_pattern(self):
        n = 2 * self.info().num_faults
        out = np.zeros(n, dtype=np.uint64)
        self._check(_lib.lib().fsimb_found_fault_to_pattern(self._h, _u64p(out), n))
        return out

    def good_values(self, round_=None):
        i = self.info()
        rd = i.num_rounds - 1 if round_ is None else round_
        out = np.zeros(i.num_elements, dtype=np.uint64)
        self._check(_lib.lib().fsimb_good_values(self._h, rd, _u64p(out), i.num_elements))
        return out

    def g_pi_results(self):
        return self.good_values()[: self.num_PIs()]

    def g_gate_results(self):
        return self.good_values()[self.num_PIs(): self.num_PIs() + self.num_gates()]

    def g_po_results(self):
        return self.good_values()[self.num_PIs() + self.num_gates():]

    # ------------------------------------------------------------ accessors
    def num_PIs(self):
        return self.info().num_pis

    def num_POs(self):
        return self.info().num_pos

    num_pos = num_POs

    def num_gates(self):
        return self.info().num_gates

    def num_wires(self):
        return self.info().num_wires

    def num_rounds(self):
        return self.info().num_rounds

    def pi(self, i):
        """fsim/simulation.hpp:58-63: the i-th PI, gate or PO as an Element."""
        return self._element(int(i), 0, self.num_PIs())

    def gate(self, i):
        return self._element(int(i), self.num_PIs(), self.num_gates())

    def po(self, i):
        return self._element(int(i), self.num_PIs() + self.num_gates(), self.num_POs())

    def gates(self):
        n_pi, n_g = self.num_PIs(), self.num_gates()
        lv, ty, val = self.levels(), self.types(), self._values()
        return [Element(t, int(lv[t]), int(ty[t]), int(val[t])) for t in range(n_pi, n_pi + n_g)]

    @staticmethod
    def gateTypeToString(t):
        """fsim/simulation.cpp:1127-1155."""
        t = int(t)
        return GATE_TYPE_NAMES[t] if 0 <= t < len(GATE_TYPE_NAMES) else "UNKNOWN"

    def _values(self):
        if self._ran and self.info().num_rounds:
            return self.good_values()
        return np.zeros(self.info().num_elements, dtype=np.uint64)

    def _element(self, i, first, count):
        if not 0 <= i < count:
            raise IndexError("element index out of range")
        t = first + i
        return Element(t, int(self.levels()[t]), int(self.types()[t]), int(self._values()[t]))

    def gate_idx_to_tpg_order_idx(self):
        n = self.info().num_elements
        out = np.zeros(n, dtype=np.uint64)
        self._check(_lib.lib().fsimb_topo_map(self._h, _u64p(out), n))
        return out

    def levels(self):
        n = self.info().num_elements
        out = np.zeros(n, dtype=np.uint64)
        self._check(_lib.lib().fsimb_levels(self._h, _u64p(out), n))
        return out

    def num_gates_per_level(self):
        n = self.info().num_levels
        out = np.zeros(n, dtype=np.uint64)
        self._check(_lib.lib().fsimb_gates_per_level(self._h, _u64p(out), n))
        return out

    def types(self):
        n = self.info().num_elements
        out = np.zeros(n, dtype=np.uint8)
        self._check(_lib.lib().fsimb_types(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n))
        return out

    def faults(self):
        """(site, pin, value) arrays; site is the topological index."""
        n = self.info().num_faults
        s = np.zeros(n, dtype=np.uint32)
        p = np.zeros(n, dtype=np.uint8)
        v = np.zeros(n, dtype=np.uint8)
        self._check(_lib.lib().fsimb_faults(
            self._h, s.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
            p.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            v.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n))
        return s, p, v

    def fault_costs(self):
        """(group, cost) per fault: faults with the same group share one sweep;
        cost estimates the group's work (see fsimb_fault_costs)."""
        n = self.info().num_faults
        g = np.zeros(n, dtype=np.uint64)
        c = np.zeros(n, dtype=np.uint64)
        self._check(_lib.lib().fsimb_fault_costs(self._h, _u64p(g), _u64p(c), n))
        return g, c

    def dot(self):
        """Graphviz text of the circuit (the reference's visualization_graph layout)."""
        ptr, n = ctypes.c_void_p(), ctypes.c_size_t()
        self._check(_lib.lib().fsimb_dot(self._h, ctypes.byref(ptr), ctypes.byref(n)))
        return _lib.take_text(ptr, n)

    def visualization_graph(self, output_file):
        """Writes dot() to a file, like fsim::Simulator::visualization_graph."""
        with open(output_file, "w") as f:
            f.write(self.dot())

    def patterns(self):
        i = self.info()
        out = np.zeros(i.num_rounds * i.num_pis, dtype=np.uint64)
        self._check(_lib.lib().fsimb_patterns(self._h, _u64p(out), len(out)))
        return out.reshape(i.num_rounds, i.num_pis)


__all__ = ["Simulator", "Element", "GATE_TYPE_NAMES", "FsimbError", "RESULT_DTYPE"]
