"""Test-side access to the CPU oracle (oracle/fsim_oracle.c) and, when it was
built, to the reference simulator harness (oracle/_ref/libfsim_ref.so).

Only tests, the smoke check and the benchmark's CPU-baseline leg use this
module; it is the checker, never the simulated path.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libfsim_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libfsim_ref.so")

RES_DTYPE = np.dtype([("detected", np.uint8), ("ref_flag", np.uint8), ("pad", np.uint8, 6),
                      ("first", np.int64), ("count", np.uint64), ("ref_rd", np.uint64)])
FAULT_DTYPE = np.dtype([("site", np.uint64), ("pin", np.uint32), ("value", np.uint32)])

_P = ctypes.c_void_p
_lib = None
_ref = None


def oracle_lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"])
        L = ctypes.CDLL(ORACLE_SO)
        L.or_parse_ckt.restype = _P
        L.or_parse_ckt.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t]
        L.or_free.argtypes = [_P]
        for n in ["or_num_elements", "or_num_pis", "or_num_pos", "or_num_gates", "or_num_levels"]:
            getattr(L, n).restype = ctypes.c_uint64
            getattr(L, n).argtypes = [_P]
        for n in ["or_tpg", "or_levels", "or_per_level"]:
            getattr(L, n).argtypes = [_P, _P]
        L.or_types.argtypes = [_P, _P]
        L.or_parse_flst.restype = ctypes.c_int64
        L.or_parse_flst.argtypes = [_P, ctypes.c_char_p, ctypes.c_size_t, _P, ctypes.c_size_t,
                                    ctypes.c_char_p, ctypes.c_size_t]
        L.or_parse_ptn.restype = ctypes.c_int64
        L.or_parse_ptn.argtypes = [_P, ctypes.c_char_p, ctypes.c_size_t, _P, ctypes.c_size_t,
                                   ctypes.c_char_p, ctypes.c_size_t]
        L.or_good_values.argtypes = [_P, _P, ctypes.c_uint64, ctypes.c_uint64, _P]
        L.or_results_init.argtypes = [_P, ctypes.c_size_t]
        L.or_simulate.argtypes = [_P, _P, ctypes.c_uint64, ctypes.c_uint64, _P, ctypes.c_uint64,
                                  ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, _P]
        _lib = L
    return _lib


class Oracle:
    """Parsed inputs + simulation through the C restatement."""

    def __init__(self, ckt, flst, ptn):
        L = oracle_lib()
        err = ctypes.create_string_buffer(256)
        ck = ckt.encode() if isinstance(ckt, str) else ckt
        self._nl = L.or_parse_ckt(ck, len(ck), err, 256)
        if not self._nl:
            raise ValueError(err.value.decode())
        self.N = L.or_num_elements(self._nl)
        self.n_pi = L.or_num_pis(self._nl)
        self.n_po = L.or_num_pos(self._nl)
        self.n_gates = L.or_num_gates(self._nl)
        self.n_levels = L.or_num_levels(self._nl)
        fl = flst.encode() if isinstance(flst, str) else flst
        cap = max(16, fl.count(b"\n") + len(fl.split()) + 16)
        self.faults = np.zeros(cap, dtype=FAULT_DTYPE)
        n = L.or_parse_flst(self._nl, fl, len(fl), self.faults.ctypes.data, cap, err, 256)
        if n < 0:
            raise ValueError(err.value.decode())
        self.faults = self.faults[:n].copy()
        pt = ptn.encode() if isinstance(ptn, str) else ptn
        toks = pt.split()
        P = int(toks[0]) if toks else 0
        W = (P + 63) // 64
        self.words = np.zeros(max(1, W * self.n_pi), dtype=np.uint64)
        p = L.or_parse_ptn(self._nl, pt, len(pt), self.words.ctypes.data, len(self.words), err, 256)
        if p < 0:
            raise ValueError(err.value.decode())
        self.P, self.W = P, W

    def set_faults(self, site, pin, value):
        """Faults by topological index (as fsimb_set_faults)."""
        f = np.zeros(len(site), dtype=FAULT_DTYPE)
        f["site"], f["pin"], f["value"] = site, pin, np.asarray(value) != 0
        self.faults = f

    def set_patterns(self, words, P):
        """Pattern words [ceil(P/64)][nPI] (as fsimb_set_patterns)."""
        self.P, self.W = P, (P + 63) // 64
        self.words = np.ascontiguousarray(np.asarray(words, dtype=np.uint64).ravel())
        if len(self.words) == 0:
            self.words = np.zeros(1, dtype=np.uint64)

    def __del__(self):
        if getattr(self, "_nl", None):
            oracle_lib().or_free(self._nl)
            self._nl = None

    def tpg(self):
        out = np.zeros(self.N, dtype=np.uint64)
        oracle_lib().or_tpg(self._nl, out.ctypes.data)
        return out

    def levels(self):
        out = np.zeros(self.N, dtype=np.uint64)
        oracle_lib().or_levels(self._nl, out.ctypes.data)
        return out

    def per_level(self):
        out = np.zeros(self.n_levels, dtype=np.uint64)
        oracle_lib().or_per_level(self._nl, out.ctypes.data)
        return out

    def types(self):
        out = np.zeros(self.N, dtype=np.uint8)
        oracle_lib().or_types(self._nl, out.ctypes.data)
        return out

    def good_values(self, rd=None):
        rd = self.W - 1 if rd is None else rd
        out = np.zeros(self.N, dtype=np.uint64)
        oracle_lib().or_good_values(self._nl, self.words.ctypes.data, self.P, rd, out.ctypes.data)
        return out

    def simulate(self, f0=0, f1=None, rd0=0, rd1=None, mode=1, threads=None):
        """Per-fault results over faults [f0,f1) and rounds [rd0,rd1)."""
        f1 = len(self.faults) if f1 is None else f1
        rd1 = self.W if rd1 is None else rd1
        threads = threads or min(32, os.cpu_count() or 1)
        res = np.zeros(max(0, f1 - f0), dtype=RES_DTYPE)
        L = oracle_lib()
        L.or_results_init(res.ctypes.data, len(res))
        L.or_simulate(self._nl, self.faults.ctypes.data, f0, f1, self.words.ctypes.data, self.P,
                      rd0, rd1, mode, threads, res.ctypes.data)
        return res


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_SO)
        L.ref_load_text.restype = _P
        L.ref_load_text.argtypes = [ctypes.c_char_p, ctypes.c_size_t] * 3
        L.ref_load_words.restype = _P
        L.ref_load_words.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                     ctypes.c_size_t, _P, ctypes.c_uint64, ctypes.c_uint64]
        L.ref_free.argtypes = [_P]
        L.ref_num.restype = ctypes.c_uint64
        L.ref_num.argtypes = [_P, ctypes.c_int]
        L.ref_arrays.argtypes = [_P, _P, _P, _P, _P, _P]
        L.ref_run_table.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P, _P]
        L.ref_simulate.argtypes = [_P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                   ctypes.c_uint64, ctypes.c_int, _P]
        L.ref_seconds.restype = ctypes.c_double
        L.ref_seconds.argtypes = [_P]
        _ref = L
    return _ref


class Reference:
    """LSIM's own simulator (compiled from the reference sources)."""

    def __init__(self, ckt, flst, ptn=None, words=None, P=None, n_pi=None):
        L = ref_lib()
        ck = ckt.encode() if isinstance(ckt, str) else ckt
        fl = flst.encode() if isinstance(flst, str) else flst
        if ptn is not None:
            pt = ptn.encode() if isinstance(ptn, str) else ptn
            self._h = L.ref_load_text(ck, len(ck), fl, len(fl), pt, len(pt))
        else:
            w = np.ascontiguousarray(words, dtype=np.uint64)
            self._words = w
            self._h = L.ref_load_words(ck, len(ck), fl, len(fl), w.ctypes.data, P, n_pi)
        self.F = L.ref_num(self._h, 5)
        self.N = L.ref_num(self._h, 0) + L.ref_num(self._h, 1) + L.ref_num(self._h, 2)
        self.rounds = L.ref_num(self._h, 4)

    def __del__(self):
        if getattr(self, "_h", None):
            ref_lib().ref_free(self._h)
            self._h = None

    def simulate(self, f0=0, f1=None, rd0=0, rd1=None, threads=1):
        f1 = self.F if f1 is None else f1
        rd1 = self.rounds if rd1 is None else rd1
        res = np.zeros(max(0, f1 - f0), dtype=RES_DTYPE)
        ref_lib().ref_simulate(self._h, f0, f1, rd0, rd1, threads, res.ctypes.data)
        self.seconds = ref_lib().ref_seconds(self._h)
        return res

    def run_table(self, mode=0, threads=1):
        table = np.zeros(2 * self.F, dtype=np.uint64)
        good = np.zeros(self.N, dtype=np.uint64)
        ref_lib().ref_run_table(self._h, mode, threads, table.ctypes.data, good.ctypes.data)
        return table, good
