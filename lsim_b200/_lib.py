"""ctypes binding of the C ABI in include/fsimb.h.

The shared library ``lsim_b200/libfsimb200.so`` is built in-tree from
``lsim_b200/csrc`` (``python -m lsim_b200.build``).  If it is missing it is
built on first use; if that fails the import fails -- there is no CPU
fallback for the simulation path.
"""
import ctypes
import os

from . import build as _build

HERE = os.path.dirname(os.path.abspath(__file__))

OK, ERR_ARG, ERR_PARSE, ERR_CUDA, ERR_STATE, ERR_NOMEM, ERR_IO, ERR_LIMIT, ERR_TIMEOUT = range(9)
_ERR_NAMES = {1: "ARG", 2: "PARSE", 3: "CUDA", 4: "STATE", 5: "NOMEM", 6: "IO", 7: "LIMIT",
              8: "TIMEOUT"}


class FsimbError(RuntimeError):
    """A failed C-ABI call: ``code`` is the FSIMB_ERR_* status."""

    def __init__(self, code, msg):
        super().__init__("FSIMB_ERR_%s: %s" % (_ERR_NAMES.get(code, str(code)), msg))
        self.code = code


class FaultResult(ctypes.Structure):
    _fields_ = [("detected", ctypes.c_uint8), ("ref_last_round_flag", ctypes.c_uint8),
                ("pad", ctypes.c_uint8 * 6), ("first_pattern", ctypes.c_int64),
                ("count", ctypes.c_uint64), ("ref_last_rd", ctypes.c_uint64)]


class Opts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("drop", ctypes.c_uint32),
                ("words_per_item", ctypes.c_uint32), ("block_threads", ctypes.c_uint32),
                ("ctas_per_sm", ctypes.c_uint32), ("tune", ctypes.c_uint32),
                ("stream", ctypes.c_void_p), ("n_detect", ctypes.c_uint32),
                ("sweep_variant", ctypes.c_uint32), ("wait_test", ctypes.c_uint32),
                ("pad", ctypes.c_uint32)]


class Info(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ["num_pis", "num_pos", "num_gates", "num_wires", "num_elements", "num_levels",
                 "num_faults", "num_patterns", "num_rounds"]]


class Stats(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in
                 ["ms_total", "ms_good", "ms_sweep", "ms_ffr", "ms_h2d", "ms_d2h"]] +
                [(n, ctypes.c_uint64) for n in
                 ["n_tiles", "n_stem_sweeps", "n_exact_sweeps", "n_traced_faults", "n_roots",
                  "sweep_items", "dense_gate_words", "sweep_alg_bytes", "good_gate_words",
                  "max_live"]] +
                [(n, ctypes.c_uint32) for n in
                 ["words_per_item", "block_threads", "blocks", "smem_bytes"]] +
                [("device_bytes", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64),
                 ("ms_compute", ctypes.c_double), ("bank_conflict_groups", ctypes.c_uint64),
                 ("bank_access_groups", ctypes.c_uint64), ("ms_tune", ctypes.c_double),
                 ("ctas_per_sm", ctypes.c_uint32), ("sweep_variant", ctypes.c_uint32),
                 ("hbm_bytes_per_tile", ctypes.c_uint64)])

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class LoadInfo(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_uint32) for n in ["on_device", "handed_back", "threads", "waves"]] +
                [(n, ctypes.c_double) for n in ["ms_total", "ms_tokenize", "ms_device"]])

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


LOAD_AUTO, LOAD_HOST, LOAD_DEVICE = 0, 1, 2


class GenConfig(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("seed", ctypes.c_uint64),
                ("n_gates", ctypes.c_uint32), ("n_pi", ctypes.c_uint32),
                ("n_po", ctypes.c_uint32), ("n_levels", ctypes.c_uint32),
                ("window", ctypes.c_uint32), ("p_fanin3", ctypes.c_double),
                ("type_mask", ctypes.c_uint32), ("hub_frac", ctypes.c_double),
                ("hub_fo_min", ctypes.c_uint32), ("hub_fo_max", ctypes.c_uint32),
                ("fo_min", ctypes.c_uint32), ("fo_max", ctypes.c_uint32),
                ("p_unused", ctypes.c_double), ("shuffle_ids", ctypes.c_int32)]


class BatchOpts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("words_per_item", ctypes.c_uint32),
                ("block_threads", ctypes.c_uint32), ("ctas_per_sm", ctypes.c_uint32),
                ("tune", ctypes.c_uint32), ("no_graph", ctypes.c_uint32),
                ("reupload", ctypes.c_uint32), ("serial_classes", ctypes.c_uint32),
                ("stream", ctypes.c_void_p)]


class BatchStats(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in
                 ["ms_total", "ms_h2d", "ms_compute", "ms_d2h", "ms_good", "ms_sweep", "ms_ffr",
                  "ms_tune", "ms_host_prep"]] +
                [(n, ctypes.c_uint64) for n in
                 ["n_circuits", "n_faults", "fault_patterns", "sweep_items", "ffr_units",
                  "exact_units", "good_units", "dense_gate_words", "sweep_alg_bytes",
                  "good_gate_words", "kernel_launches"]] +
                [(n, ctypes.c_uint32) for n in
                 ["graph_used", "n_classes", "words_per_item", "block_threads", "blocks",
                  "smem_bytes", "ctas_per_sm", "pad"]] +
                [("device_bytes", ctypes.c_uint64), ("h2d_bytes", ctypes.c_uint64),
                 ("d2h_bytes", ctypes.c_uint64)])

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "pad"}


class BatchClass(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_uint32) for n in
                 ["words_per_item", "block_threads", "blocks", "smem_bytes"]] +
                [("n_circuits", ctypes.c_uint64), ("sweep_items", ctypes.c_uint64),
                 ("max_live", ctypes.c_uint32), ("widest_level", ctypes.c_uint32),
                 ("ms_sweep", ctypes.c_double)])

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class ServerOpts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("slots", ctypes.c_uint32),
                ("slot_bytes", ctypes.c_uint64), ("max_wave_requests", ctypes.c_uint32),
                ("planner_threads", ctypes.c_uint32), ("max_wave_ms", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class Request(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("circuit", ctypes.c_uint32),
                ("site", ctypes.POINTER(ctypes.c_uint32)), ("pin", ctypes.POINTER(ctypes.c_uint8)),
                ("value", ctypes.POINTER(ctypes.c_uint8)), ("n_faults", ctypes.c_uint64),
                ("n_patterns", ctypes.c_uint64), ("row0", ctypes.c_uint64),
                ("words", ctypes.POINTER(ctypes.c_uint64))]


class ServerStats(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_uint64) for n in ["completed", "failed", "waves", "circuits"]] +
                [(n, ctypes.c_double) for n in
                 ["mean_wave_requests", "fault_patterns", "wall_ms", "ms_gpu_busy",
                  "latency_p50_ms", "latency_p99_ms", "latency_mean_ms", "latency_max_ms",
                  "queue_p50_ms", "queue_p99_ms", "wave_gpu_p50_ms", "wave_gpu_p99_ms"]] +
                [("resident_bytes", ctypes.c_uint64), ("slot_bytes", ctypes.c_uint64)])

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


# Every symbol the header declares, with its ctypes signature.
_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U64P = ctypes.POINTER(ctypes.c_uint64)
_U32P = ctypes.POINTER(ctypes.c_uint32)
_U8P = ctypes.POINTER(ctypes.c_uint8)
_CP = ctypes.c_char_p
_SZ = ctypes.c_size_t
SIGNATURES = {
    "fsimb_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    "fsimb_destroy": (ctypes.c_int, [_P]),
    "fsimb_last_error": (_CP, [_P]),
    "fsimb_load_files": (ctypes.c_int, [_P, _CP, _CP, _CP]),
    "fsimb_load_buffers": (ctypes.c_int, [_P, _CP, _SZ, _CP, _SZ, _CP, _SZ]),
    "fsimb_load_circuit": (ctypes.c_int, [_P, _CP, _SZ]),
    "fsimb_set_faults": (ctypes.c_int, [_P, _U32P, _U8P, _U8P, _U64]),
    "fsimb_set_fault_text": (ctypes.c_int, [_P, _CP, _SZ]),
    "fsimb_set_patterns": (ctypes.c_int, [_P, _U64P, _U64]),
    "fsimb_run": (ctypes.c_int, [_P, ctypes.POINTER(Opts)]),
    "fsimb_results": (ctypes.c_int, [_P, ctypes.POINTER(FaultResult), _U64]),
    "fsimb_found_fault_to_pattern": (ctypes.c_int, [_P, _U64P, _U64]),
    "fsimb_good_values": (ctypes.c_int, [_P, _U64, _U64P, _U64]),
    "fsimb_get_info": (ctypes.c_int, [_P, ctypes.POINTER(Info)]),
    "fsimb_set_loader": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
    "fsimb_get_load_info": (ctypes.c_int, [_P, ctypes.POINTER(LoadInfo)]),
    "fsimb_get_stats": (ctypes.c_int, [_P, ctypes.POINTER(Stats)]),
    "fsimb_topo_map": (ctypes.c_int, [_P, _U64P, _U64]),
    "fsimb_levels": (ctypes.c_int, [_P, _U64P, _U64]),
    "fsimb_gates_per_level": (ctypes.c_int, [_P, _U64P, _U64]),
    "fsimb_types": (ctypes.c_int, [_P, _U8P, _U64]),
    "fsimb_faults": (ctypes.c_int, [_P, _U32P, _U8P, _U8P, _U64]),
    "fsimb_patterns": (ctypes.c_int, [_P, _U64P, _U64]),
    "fsimb_fault_costs": (ctypes.c_int, [_P, _U64P, _U64P, _U64]),
    "fsimb_gen_circuit": (ctypes.c_int, [ctypes.POINTER(GenConfig), ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.POINTER(_SZ)]),
    "fsimb_gen_faults": (ctypes.c_int, [_CP, _SZ, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.POINTER(_SZ)]),
    "fsimb_gen_patterns": (ctypes.c_int, [_U64, _U64, _U64, ctypes.c_double, ctypes.c_double,
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(_SZ)]),
    "fsimb_free_text": (None, [ctypes.c_void_p]),
    "fsimb_dot": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(_SZ)]),
    "fsimb_good_po_noalloc": (ctypes.c_int, [_P, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                             ctypes.c_void_p]),
    "fsimb_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    "fsimb_batch_destroy": (ctypes.c_int, [_P]),
    "fsimb_batch_last_error": (_CP, [_P]),
    "fsimb_batch_add": (ctypes.c_int, [_P, _P]),
    "fsimb_batch_clear": (ctypes.c_int, [_P]),
    "fsimb_batch_size": (ctypes.c_int, [_P, _U64P]),
    "fsimb_batch_run": (ctypes.c_int, [_P, ctypes.POINTER(BatchOpts)]),
    "fsimb_batch_get_stats": (ctypes.c_int, [_P, ctypes.POINTER(BatchStats)]),
    "fsimb_batch_class_stats": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(BatchClass)]),
    "fsimb_batch_class_members": (ctypes.c_int, [_P, ctypes.c_uint32, _U32P, _U64]),
    "fsimb_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ServerOpts), ctypes.POINTER(_P)]),
    "fsimb_server_destroy": (ctypes.c_int, [_P]),
    "fsimb_server_last_error": (_CP, [_P]),
    "fsimb_server_add_circuit": (ctypes.c_int, [_P, _CP, _SZ, _U64P, _U64, _U32P]),
    "fsimb_server_submit": (ctypes.c_int, [_P, ctypes.POINTER(Request), _U64P]),
    "fsimb_server_wait": (ctypes.c_int, [_P, _U64, ctypes.POINTER(FaultResult), _U64, ctypes.c_int64]),
    "fsimb_server_get_stats": (ctypes.c_int, [_P, ctypes.POINTER(ServerStats)]),
    "fsimb_server_reset_stats": (ctypes.c_int, [_P]),
}

_lib = None


def lib():
    """Loads (building first if needed) the in-tree library."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            _build.build()
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code, handle=None, last_error="fsimb_last_error"):
    if code != OK:
        msg = getattr(lib(), last_error)(handle)
        raise FsimbError(code, msg.decode() if msg else "")


def take_text(ptr, n):
    try:
        return ctypes.string_at(ptr, n.value).decode()
    finally:
        lib().fsimb_free_text(ptr)
