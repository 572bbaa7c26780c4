"""Batched fault simulation: many circuits in one launch sequence.

``Batch`` wraps ``fsimb_batch_*`` (include/fsimb.h).  Members are
``Simulator`` objects loaded with circuit, faults and patterns -- host-only
ones (``Simulator(-1)``) are enough; after ``run()`` each member's
``results()`` / ``found_fault_to_pattern()`` hold its own results, equal to
what ``Simulator.run()`` gives for that circuit alone.
"""
import ctypes

from . import _lib
from ._lib import check


class Batch:
    def __init__(self, device=0):
        b = ctypes.c_void_p()
        check(_lib.lib().fsimb_batch_create(device, ctypes.byref(b)), None, "fsimb_batch_last_error")
        self._b = b
        self._members = []  # keeps the member handles alive while borrowed

    def close(self):
        if getattr(self, "_b", None):
            _lib.lib().fsimb_batch_destroy(self._b)
            self._b = None
            self._members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self._members)

    def _check(self, code):
        check(code, self._b, "fsimb_batch_last_error")

    def add(self, sim):
        self._check(_lib.lib().fsimb_batch_add(self._b, sim._h))
        self._members.append(sim)
        return len(self._members) - 1

    def clear(self):
        self._check(_lib.lib().fsimb_batch_clear(self._b))
        self._members = []

    def run(self, words_per_item=0, block_threads=0, ctas_per_sm=0, tune=False, graph=True,
            reupload=False, concurrent=True, stream=None):
        o = _lib.BatchOpts(ctypes.sizeof(_lib.BatchOpts), words_per_item, block_threads,
                           ctas_per_sm, 1 if tune else 0, 0 if graph else 1, 1 if reupload else 0,
                           0 if concurrent else 1, stream)
        self._check(_lib.lib().fsimb_batch_run(self._b, ctypes.byref(o)))
        for m in self._members:
            m._ran = True

    def stats(self):
        s = _lib.BatchStats()
        self._check(_lib.lib().fsimb_batch_get_stats(self._b, ctypes.byref(s)))
        return s.as_dict()

    def classes(self):
        """Sweep classes of the last run (shape, circuits, items, time)."""
        out = []
        i = 0
        while True:
            c = _lib.BatchClass()
            if _lib.lib().fsimb_batch_class_stats(self._b, i, ctypes.byref(c)) != 0:
                return out
            d = c.as_dict()
            ids = (ctypes.c_uint32 * max(1, c.n_circuits))()
            self._check(_lib.lib().fsimb_batch_class_members(self._b, i, ids, c.n_circuits))
            d["members"] = list(ids)[:c.n_circuits]
            out.append(d)
            i += 1

    @property
    def members(self):
        return list(self._members)
