"""ctypes binding of libqcb200 (the C ABI declared in include/qcb200.h).

The shared library is built in-tree (``quantumclifford.jl_b200/lib``).  There
is no fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libqcb200.so")

# status codes (enum qcb_status)
QCB_OK = 0
QCB_EDIM = 1
QCB_EBOUNDS = 2
QCB_EZEROQUBIT = 3
QCB_EARG = 4
QCB_EOOM = 5
QCB_EBUDGET = 6
QCB_ETIMEOUT = 7
QCB_ECUDA = 8
QCB_EBADSTRUCT = 9
QCB_EUNSUPPORTED = 10
QCB_ENOTREADY = 11


class QCBError(RuntimeError):
    """A libqcb200 call failed; ``status`` holds the qcb_status code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class DimensionMismatch(QCBError, ValueError):
    pass


class BoundsError(QCBError, IndexError):
    pass


class ArgumentError(QCBError, ValueError):
    pass


class BadDataStructure(QCBError):
    pass


_EXC = {
    QCB_EDIM: DimensionMismatch,
    QCB_EBOUNDS: BoundsError,
    QCB_EZEROQUBIT: ArgumentError,
    QCB_EARG: ArgumentError,
    QCB_EBADSTRUCT: BadDataStructure,
}


class qcb_op(ctypes.Structure):
    _fields_ = [
        ("opcode", ctypes.c_uint32),
        ("q1", ctypes.c_uint32),
        ("q2", ctypes.c_uint32),
        ("bit", ctypes.c_uint32),
        ("p", ctypes.c_double * 3),
    ]


OP_DTYPE = np.dtype(
    [("opcode", "<u4"), ("q1", "<u4"), ("q2", "<u4"), ("bit", "<u4"), ("p", "<f8", (3,))], align=True
)
assert OP_DTYPE.itemsize == ctypes.sizeof(qcb_op) == 40

EVENT_DTYPE = np.dtype([("op_index", "<u4"), ("pauli", "<u4"), ("shot", "<u8")], align=True)


class qcb_noise_source(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("seed", ctypes.c_uint64),
        ("shot_offset", ctypes.c_uint64),
        ("events", ctypes.c_void_p),
        ("n_events", ctypes.c_uint64),
        ("reset_planes", ctypes.c_void_p),
    ]


class qcb_batch_job(ctypes.Structure):
    _fields_ = [("frame", ctypes.c_void_p), ("program", ctypes.c_void_p), ("seed", ctypes.c_uint64),
                ("shot_offset", ctypes.c_uint64), ("tile", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class qcb_program_info(ctypes.Structure):
    _fields_ = [
        (name, ctypes.c_uint32)
        for name in (
            "nqubits", "nbits", "n_ops", "n_updates", "n_noise_sites", "n_resets", "n_segments", "n_flushes",
        )
    ]


_lib = None


def lib():
    """Load libqcb200 (once).  Raises if the library has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libqcb200.so not found at {LIB_PATH}; build it with `make -C quantumclifford.jl_b200` "
            "(or __graft_entry__.build())"
        )
    L = ctypes.CDLL(LIB_PATH)
    vp, u32, u64, i32, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_size_t
    P = ctypes.POINTER
    sig = {
        "qcb_init": ([ctypes.c_int], ctypes.c_int),
        "qcb_version": ([], ctypes.c_char_p),
        "qcb_last_error": ([ctypes.c_char_p, sz], ctypes.c_int),
        "qcb_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "qcb_device_synchronize": ([], ctypes.c_int),
        "qcb_launch_count": ([], u64),
        "qcb_program_compile": ([vp, sz, P(vp)], ctypes.c_int),
        "qcb_program_info_get": ([vp, P(qcb_program_info)], ctypes.c_int),
        "qcb_program_device_bytes": ([vp, P(u64)], ctypes.c_int),
        "qcb_program_destroy": ([vp], ctypes.c_int),
        "qcb_frame_create": ([u64, u32, u32, P(vp)], ctypes.c_int),
        "qcb_frame_destroy": ([vp], ctypes.c_int),
        "qcb_frame_shape": ([vp, P(u64), P(u32), P(u32)], ctypes.c_int),
        "qcb_frame_init_z": ([vp, u64, u64, vp], ctypes.c_int),
        "qcb_frame_init_z_planes": ([vp, vp, vp], ctypes.c_int),
        "qcb_frame_clear": ([vp, vp], ctypes.c_int),
        "qcb_frame_copy": ([vp, vp, vp], ctypes.c_int),
        "qcb_pftrajectories": ([vp, vp, P(qcb_noise_source), vp], ctypes.c_int),
        "qcb_frame_apply_ops": ([vp, vp, sz, P(qcb_noise_source), vp], ctypes.c_int),
        "qcb_frame_download_xzs": ([vp, vp, vp], ctypes.c_int),
        "qcb_frame_upload_xzs": ([vp, vp, vp], ctypes.c_int),
        "qcb_frame_download_measurements": ([vp, vp, vp], ctypes.c_int),
        "qcb_frame_upload_measurements": ([vp, vp, vp], ctypes.c_int),
        "qcb_frame_download_record_planes": ([vp, vp, vp], ctypes.c_int),
        "qcb_frame_download_planes": ([vp, vp, vp, vp], ctypes.c_int),
        "qcb_pftrajectories_host": ([vp, sz, u64, u64, u64, vp, vp], ctypes.c_int),
        "qcb_pftrajectories_fresh": ([vp, vp, u64, u64, vp], ctypes.c_int),
        "qcb_tune_set": ([ctypes.c_char_p, ctypes.c_int64], ctypes.c_int),
        "qcb_tableau_create": ([u32, u32, P(vp)], ctypes.c_int),
        "qcb_tableau_destroy": ([vp], ctypes.c_int),
        "qcb_tableau_shape": ([vp, P(u32), P(u32)], ctypes.c_int),
        "qcb_tableau_upload": ([vp, vp, vp, vp], ctypes.c_int),
        "qcb_tableau_download": ([vp, vp, vp, vp], ctypes.c_int),
        "qcb_tableau_copy": ([vp, vp, vp], ctypes.c_int),
        "qcb_mul_left_pauli": ([vp, vp, ctypes.c_int, vp, vp], ctypes.c_int),
        "qcb_mul_left_pauli_batch_noalloc": ([vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, vp],
                                             ctypes.c_int),
        "qcb_mul_left_row": ([vp, u32, u32, ctypes.c_int, vp], ctypes.c_int),
        "qcb_mul_rows": ([vp, u32, u32, vp, u32, u32, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp], ctypes.c_int),
        "qcb_mul_left_state": ([vp, ctypes.c_int, u32, u32, ctypes.c_int, vp], ctypes.c_int),
        "qcb_mul_left_tableau_pauli": ([vp, vp, ctypes.c_int, vp], ctypes.c_int),
        "qcb_prodphase": ([vp, u32, vp, u32, vp, vp], ctypes.c_int),
        "qcb_comm": ([vp, u32, vp, u32, vp, vp], ctypes.c_int),
        "qcb_canonicalize": ([vp, u32, u32, ctypes.c_int, P(i32), P(i32), vp], ctypes.c_int),
        "qcb_project": ([vp, ctypes.c_int, P(i32), vp, ctypes.c_int, ctypes.c_int, vp, vp, P(u32), vp], ctypes.c_int),
        "qcb_batch_create": ([vp, sz, P(vp)], ctypes.c_int),
        "qcb_batch_run": ([vp, vp], ctypes.c_int),
        "qcb_batch_status": ([vp], ctypes.c_int),
        "qcb_batch_destroy": ([vp], ctypes.c_int),
        "qcb_canon_batch_create": ([vp, sz, ctypes.c_int, u32, P(vp)], ctypes.c_int),
        "qcb_canon_batch_run": ([vp, vp], ctypes.c_int),
        "qcb_canon_batch_ranks": ([vp, vp, vp], ctypes.c_int),
        "qcb_canon_batch_destroy": ([vp], ctypes.c_int),
        "qcb_server_create": ([u64, u32, u64, P(vp)], ctypes.c_int),
        "qcb_server_submit": ([vp, vp, sz, u64, u64, P(u64)], ctypes.c_int),
        "qcb_server_preload": ([vp, vp, sz], ctypes.c_int),
        "qcb_server_query": ([vp, u64, P(i32), vp], ctypes.c_int),
        "qcb_server_next_done": ([vp, ctypes.c_double, P(u64), P(i32), vp], ctypes.c_int),
        "qcb_server_wait": ([vp, u64, ctypes.c_double], ctypes.c_int),
        "qcb_server_result": ([vp, u64, vp, P(u32)], ctypes.c_int),
        "qcb_server_release": ([vp, u64], ctypes.c_int),
        "qcb_server_destroy": ([vp], ctypes.c_int),
        "qcb_server_stats": ([vp, P(u64), P(u64), P(u32)], ctypes.c_int),
        "qcb_tune_tile": ([vp, P(u32), P(ctypes.c_float), vp], ctypes.c_int),
        "qcb_tune_walker": ([vp, ctypes.c_uint64, P(u32), P(u32), P(ctypes.c_float), vp], ctypes.c_int),
        "qcb_tune_walker_clear": ([], ctypes.c_int),
        "qcb_frame_measurement_columns": ([vp, vp, sz, vp, vp, vp], ctypes.c_int),
        "qcb_frame_syndrome_rows": ([vp, vp, sz, vp, ctypes.c_int, vp], ctypes.c_int),
        "qcb_evaluate_guesses": ([vp, vp, sz, vp, sz, vp, P(u64), vp], ctypes.c_int),
        "qcb_rowswap": ([vp, ctypes.c_int, u32, u32, ctypes.c_int, vp], ctypes.c_int),
        "qcb_expect": ([vp, ctypes.c_int, i32, vp, vp, vp], ctypes.c_int),
        "qcb_project_qubit": ([vp, ctypes.c_int, P(i32), u32, vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, vp, vp,
                               P(u32), vp], ctypes.c_int),
        "qcb_projectrand": ([vp, ctypes.c_int, P(i32), vp, u32, vp, ctypes.c_size_t, vp, vp, vp, P(u32), vp],
                            ctypes.c_int),
        "qcb_canonicalize_state": ([vp, ctypes.c_int, i32, ctypes.c_int, P(i32), P(i32), vp], ctypes.c_int),
        "qcb_canonicalize_rref": ([vp, ctypes.c_int, i32, vp, ctypes.c_size_t, ctypes.c_int, P(i32), vp], ctypes.c_int),
        "qcb_canonicalize_gott": ([vp, ctypes.c_int, P(i32), P(i32), vp, vp, vp], ctypes.c_int),
        "qcb_permutesystems": ([vp, vp, vp], ctypes.c_int),
        "qcb_generate": ([vp, vp, ctypes.c_int, P(i32), vp, u32, P(u32), vp], ctypes.c_int),
        "qcb_apply_gates": ([vp, vp, sz, ctypes.c_int, vp], ctypes.c_int),
        "qcb_apply_dense": ([vp, vp, ctypes.c_int, vp], ctypes.c_int),
        "qcb_debug_philox": ([vp, vp, vp], ctypes.c_int),
        "qcb_debug_program_dump": ([vp, sz, vp, sz, P(sz), vp, sz, P(sz), vp, vp, sz, P(sz), P(qcb_program_info)],
                                   ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def exported_symbols():
    """Names the C ABI declares (kept in sync with include/qcb200.h)."""
    lib()
    import re

    hdr = os.path.join(os.path.dirname(os.path.dirname(_HERE)), "include", "qcb200.h")
    if os.path.exists(hdr):
        txt = open(hdr).read()
        return sorted(set(re.findall(r"\b(qcb_[a-z0-9_]+)\s*\(", txt)))
    return []


def check(status: int) -> None:
    """Raise the exception matching a non-zero qcb_status."""
    if status == QCB_OK:
        return
    buf = ctypes.create_string_buffer(4096)
    lib().qcb_last_error(buf, 4096)
    msg = buf.value.decode(errors="replace")
    raise _EXC.get(status, QCBError)(status, msg)


_initialised = False


def ensure_init(device: int = 0) -> None:
    global _initialised
    if not _initialised:
        check(lib().qcb_init(device))
        _initialised = True


def ptr(a: np.ndarray) -> int:
    """Address of a C-contiguous numpy array (or torch tensor)."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data
