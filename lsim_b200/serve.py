"""Serving loop: fault-simulation requests against resident circuits.

``Server`` wraps ``fsimb_server_*`` (include/fsimb.h).  Circuits are added
once (with an optional resident pattern block whose good-machine values stay
on the device); requests -- a fault subset and a range of the block's
patterns, or their own patterns -- are submitted from any thread and return
a ticket; ``wait(ticket)`` returns the per-fault results, equal to what
``Simulator.run()`` gives for the same circuit, faults and patterns.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import FsimbError, check
from .simulator import RESULT_DTYPE


def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Server:
    def __init__(self, device=0, slots=0, slot_bytes=0, max_wave_requests=0, planner_threads=0,
                 max_wave_ms=0):
        o = _lib.ServerOpts(ctypes.sizeof(_lib.ServerOpts), slots, slot_bytes, max_wave_requests,
                            planner_threads, max_wave_ms, 0)
        s = ctypes.c_void_p()
        check(_lib.lib().fsimb_server_create(device, ctypes.byref(o), ctypes.byref(s)), None,
              "fsimb_server_last_error")
        self._s = s
        self._n_faults = {}

    def close(self):
        if getattr(self, "_s", None):
            _lib.lib().fsimb_server_destroy(self._s)
            self._s = None

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
        check(code, self._s, "fsimb_server_last_error")

    def add_circuit(self, ckt, words=None, n_patterns=0):
        """Circuit text; optional resident pattern block (words [rows][nPI])."""
        b = ckt.encode() if isinstance(ckt, str) else ckt
        cid = ctypes.c_uint32()
        wp = None
        if words is not None:
            words = _arr(words, np.uint64)
            wp = words.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        self._check(_lib.lib().fsimb_server_add_circuit(self._s, b, len(b), wp, n_patterns,
                                                       ctypes.byref(cid)))
        return cid.value

    def submit(self, circuit, site, value, pin=None, n_patterns=0, row0=0, words=None):
        site = _arr(site, np.uint32)
        value = _arr(value, np.uint8)
        pin = None if pin is None else _arr(pin, np.uint8)
        r = _lib.Request()
        r.struct_size = ctypes.sizeof(_lib.Request)
        r.circuit = circuit
        r.site = site.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        r.pin = None if pin is None else pin.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        r.value = value.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        r.n_faults = len(site)
        r.n_patterns = n_patterns
        r.row0 = row0
        if words is not None:
            words = _arr(words, np.uint64)
            r.words = words.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        t = ctypes.c_uint64()
        self._check(_lib.lib().fsimb_server_submit(self._s, ctypes.byref(r), ctypes.byref(t)))
        self._n_faults[t.value] = len(site)
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        """Results of a ticket (numpy RESULT_DTYPE); None if not done in time."""
        n = self._n_faults[ticket]
        out = np.zeros(n, dtype=RESULT_DTYPE)
        code = _lib.lib().fsimb_server_wait(self._s, ticket,
                                           out.ctypes.data_as(ctypes.POINTER(_lib.FaultResult)),
                                           n, timeout_ms)
        if code == _lib.ERR_TIMEOUT:
            return None
        del self._n_faults[ticket]
        self._check(code)
        return out

    def stats(self):
        s = _lib.ServerStats()
        self._check(_lib.lib().fsimb_server_get_stats(self._s, ctypes.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        self._check(_lib.lib().fsimb_server_reset_stats(self._s))


__all__ = ["Server", "FsimbError"]
