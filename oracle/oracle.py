"""ctypes wrapper of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker that tests/, __graft_entry__.smoke()
and the CPU-baseline leg of bench.py compare against.  The product never
imports this module.  All arrays use the reference's layouts (see
oracle.cpp).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")

OP_DTYPE = np.dtype(
    [("opcode", "<u4"), ("q1", "<u4"), ("q2", "<u4"), ("bit", "<u4"), ("p", "<f8", (3,))], align=True
)
EVENT_DTYPE = np.dtype([("op_index", "<u4"), ("pauli", "<u4"), ("shot", "<u8")], align=True)

KIND = {"Stabilizer": 0, "MixedStabilizer": 1, "Destabilizer": 2, "MixedDestabilizer": 3}

_L = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def L():
    global _L
    if _L is None:
        if not os.path.exists(SO):
            build()
        _L = ctypes.CDLL(SO)
        vp, u64, u32, sz, i = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_size_t, ctypes.c_int
        u8 = ctypes.c_uint8
        P = ctypes.POINTER
        sig = {
            "oracle_philox4x32_10": ([vp, vp, vp], None),
            "oracle_mul_left_words": ([vp, vp, sz, i], u8),
            "oracle_mul_left_pauli": ([vp, vp, vp, u8, sz, i], None),
            "oracle_prodphase": ([vp, vp, sz], u8),
            "oracle_comm": ([vp, vp, sz], u8),
            "oracle_mul_left_row": ([vp, vp, sz, sz, sz, i], None),
            "oracle_mul_rows": ([vp, vp, vp, vp, sz, sz, sz, sz, sz, i, i, i], None),
            "oracle_mul_left_tableau_pauli": ([vp, vp, sz, sz, vp, u8, i], None),
            "oracle_canonicalize": ([vp, vp, sz, u32, i, P(ctypes.c_int), P(ctypes.c_int)], None),
            "oracle_generate": ([vp, vp, vp, vp, sz, u32, i, vp, P(sz)], i),
            "oracle_project": ([i, vp, vp, sz, u32, P(ctypes.c_int), vp, u8, i, i, P(ctypes.c_int), P(ctypes.c_int)], i),
            "oracle_apply_gates": ([vp, vp, sz, u32, vp, sz, i], i),
            "oracle_apply_dense": ([vp, vp, sz, u32, vp, vp, i], None),
            "oracle_pftrajectories": ([vp, vp, u64, u32, u32, vp, sz, i, vp, u64, vp, u64, i], None),
            "oracle_frame_init_z": ([vp, u64, u32, vp, u64], None),
            "oracle_pftrajectories_philox": ([vp, vp, u64, u32, u32, vp, sz, u64, u64], None),
            "oracle_philox_init_z": ([vp, u64, u32, u64, u64], None),
            "oracle_evaluate_guesses": ([vp, vp, vp, u64, sz, sz], u64),
            "oracle_canonicalize_state": ([i, vp, vp, sz, u32, i, i, P(ctypes.c_int), P(ctypes.c_int)], None),
            "oracle_canonicalize_rref": ([i, vp, vp, sz, u32, i, vp, sz, i], i),
            "oracle_permutesystems": ([vp, sz, u32, vp], None),
            "oracle_canonicalize_gott": ([vp, vp, sz, u32, i, P(ctypes.c_int), P(ctypes.c_int), vp, vp], None),
            "oracle_project_cond": ([vp, vp, sz, u32, P(ctypes.c_int), u32, i, i, i, P(ctypes.c_int),
                                     P(ctypes.c_int)], None),
        }
        for name, (args, res) in sig.items():
            f = getattr(_L, name)
            f.argtypes = args
            f.restype = res
    return _L


def _p(a):
    return a.ctypes.data if a is not None and a.size else None


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    L().oracle_philox4x32_10(_p(c), _p(k), _p(out))
    return out


# ------------------------------------------------------------------ tableaux
def mul_left_pauli(r_xz, r_phase, l_xz, l_phase, phases=True):
    r = np.array(r_xz, dtype=np.uint64, copy=True)
    ph = np.array([r_phase], dtype=np.uint8)
    l = np.ascontiguousarray(l_xz, dtype=np.uint64)
    L().oracle_mul_left_pauli(_p(r), _p(ph), _p(l), int(l_phase), len(r), int(phases))
    return r, int(ph[0])


def mul_rows(s_ph, s_xz, t_ph, t_xz, s_row, count, t_row, t_step, right=False, phase_src=0, phases=True):
    """The mul_left!/mul_right! family on rows (1-based; see oracle.cpp).
    s is updated on copies: returns (phases, xzs).  Pass t_ph/t_xz = None for
    t = s (the source rows are read as they are when each target row is done)."""
    ph = np.array(s_ph, dtype=np.uint8, copy=True)
    xz = np.array(s_xz, dtype=np.uint64, copy=True)
    same = t_xz is None
    tx = xz if same else np.ascontiguousarray(t_xz, dtype=np.uint64)
    tp = ph if same else np.ascontiguousarray(t_ph, dtype=np.uint8)
    L().oracle_mul_rows(_p(xz), _p(ph), _p(tx), _p(tp), xz.shape[1], s_row, count, t_row, t_step, int(right),
                        int(phase_src), int(phases))
    return ph, xz


def prodphase(l_xz, l_ph, r_xz, r_ph):
    l = np.ascontiguousarray(l_xz, dtype=np.uint64)
    r = np.ascontiguousarray(r_xz, dtype=np.uint64)
    return (int(L().oracle_prodphase(_p(l), _p(r), len(l))) + l_ph + r_ph) & 3


def comm(l_xz, r_xz):
    l = np.ascontiguousarray(l_xz, dtype=np.uint64)
    r = np.ascontiguousarray(r_xz, dtype=np.uint64)
    return int(L().oracle_comm(_p(l), _p(r), len(l)))


def canonicalize(phases, xzs, n, use_phases=True):
    """Returns (phases, xzs, rx, rz) after _canonicalize!."""
    ph = np.array(phases, dtype=np.uint8, copy=True)
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    rx, rz = ctypes.c_int(), ctypes.c_int()
    L().oracle_canonicalize(_p(xz), _p(ph), len(ph), n, int(use_phases), ctypes.byref(rx), ctypes.byref(rz))
    return ph, xz, rx.value, rz.value


def canonicalize_state(kind, phases, xzs, n, rank=0, use_phases=True):
    """_canonicalize!(state) on a whole state tableau (the Destabilizer kinds
    carry their destabilizer rows along).  Returns (phases, xzs, rx, rz)."""
    ph = np.array(phases, dtype=np.uint8, copy=True)
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    rx, rz = ctypes.c_int(), ctypes.c_int()
    L().oracle_canonicalize_state(KIND[kind] if isinstance(kind, str) else kind, _p(xz), _p(ph), len(ph), n,
                                  int(rank), int(use_phases), ctypes.byref(rx), ctypes.byref(rz))
    return ph, xz, rx.value, rz.value


def canonicalize_rref(kind, phases, xzs, n, cols, rank=0, use_phases=True):
    """_canonicalize_rref!(state, cols) with 1-based cols.  Returns (phases, xzs, i)."""
    ph = np.array(phases, dtype=np.uint8, copy=True)
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    c = np.ascontiguousarray(cols, dtype=np.uint32)
    i = L().oracle_canonicalize_rref(KIND[kind] if isinstance(kind, str) else kind, _p(xz), _p(ph), len(ph), n,
                                     int(rank), _p(c), len(c), int(use_phases))
    return ph, xz, int(i)


def permutesystems(xzs, n, perm):
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    pm = np.ascontiguousarray(perm, dtype=np.uint32)
    L().oracle_permutesystems(_p(xz), xz.shape[0], n, _p(pm))
    return xz


def canonicalize_gott(phases, xzs, n, use_phases=True):
    """_canonicalize_gott!(stabilizer).  Returns (phases, xzs, r, s, xperm, zperm), perms 1-based."""
    ph = np.array(phases, dtype=np.uint8, copy=True)
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    r, s = ctypes.c_int(), ctypes.c_int()
    xp = np.zeros(max(n, 1), np.uint32)
    zp = np.zeros(max(n, 1), np.uint32)
    L().oracle_canonicalize_gott(_p(xz), _p(ph), len(ph), n, int(use_phases), ctypes.byref(r), ctypes.byref(s),
                                 _p(xp), _p(zp))
    return ph, xz, r.value, s.value, xp[:n], zp[:n]


def project_cond(phases, xzs, n, rank, qubit, basis, keep_result=True, use_phases=True):
    """project_cond! behind projectX!/projectZ!/projectY! (basis 1/2/3) on a
    MixedDestabilizer.  Returns (phases, xzs, rank, anticom, result), result -1 = nothing."""
    ph = np.array(phases, dtype=np.uint8, copy=True)
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    r = ctypes.c_int(rank)
    a, res = ctypes.c_int(), ctypes.c_int()
    L().oracle_project_cond(_p(xz), _p(ph), len(ph), n, ctypes.byref(r), int(qubit), int(basis), int(keep_result),
                            int(use_phases), ctypes.byref(a), ctypes.byref(res))
    return ph, xz, r.value, a.value, res.value


def evaluate_guesses(measured_faults, guesses, faults_matrix):
    """evaluate_guesses: fails / nsamples, on Bool matrices (samples x nlog,
    samples x k, nlog x k)."""
    m = np.asfortranarray(measured_faults, dtype=np.uint8)
    g = np.asfortranarray(guesses, dtype=np.uint8)
    f = np.asfortranarray(faults_matrix, dtype=np.uint8)
    S = g.shape[0]
    fails = L().oracle_evaluate_guesses(m.ctypes.data, g.ctypes.data, f.ctypes.data, S, f.shape[0], f.shape[1])
    return fails / S, int(fails)


def generate(p_xz, p_ph, phases, xzs, n, use_phases=True):
    p = np.array(p_xz, dtype=np.uint64, copy=True)
    pph = np.array([p_ph], dtype=np.uint8)
    ph = np.ascontiguousarray(phases, dtype=np.uint8)
    xz = np.ascontiguousarray(xzs, dtype=np.uint64)
    used = np.zeros(max(len(ph), 1) * 2 + 2, dtype=np.int32)
    nu = ctypes.c_size_t()
    ok = L().oracle_generate(_p(p), _p(pph), _p(xz), _p(ph), len(ph), n, int(use_phases), _p(used), ctypes.byref(nu))
    return bool(ok), p, int(pph[0]), [int(u) for u in used[: nu.value]]


def project(kind, phases, xzs, n, p_xz, p_ph, rank=0, keep_result=True, use_phases=True):
    """Returns (status, phases, xzs, rank, anticom, result) (result -1 = nothing)."""
    ph = np.array(phases, dtype=np.uint8, copy=True)
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    p = np.ascontiguousarray(p_xz, dtype=np.uint64)
    r = ctypes.c_int(rank)
    a, res = ctypes.c_int(), ctypes.c_int()
    st = L().oracle_project(KIND[kind] if isinstance(kind, str) else kind, _p(xz), _p(ph), len(ph), n,
                            ctypes.byref(r), _p(p), int(p_ph), int(keep_result), int(use_phases),
                            ctypes.byref(a), ctypes.byref(res))
    return st, ph, xz, r.value, a.value, res.value


def apply_gates(phases, xzs, n, ops, use_phases=True):
    ph = np.array(phases, dtype=np.uint8, copy=True)
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    o = np.ascontiguousarray(ops, dtype=OP_DTYPE)
    st = L().oracle_apply_gates(_p(xz), _p(ph), len(ph), n, _p(o), len(o), int(use_phases))
    assert st == 0, st
    return ph, xz


def apply_dense(phases, xzs, n, c_phases, c_xzs, use_phases=True):
    ph = np.array(phases, dtype=np.uint8, copy=True)
    xz = np.array(xzs, dtype=np.uint64, copy=True)
    cph = np.ascontiguousarray(c_phases, dtype=np.uint8)
    cxz = np.ascontiguousarray(c_xzs, dtype=np.uint64)
    L().oracle_apply_dense(_p(xz), _p(ph), len(ph), n, _p(cxz), _p(cph), int(use_phases))
    return ph, xz


# ------------------------------------------------------------------ frames
def frame_words(nq1):
    return 2 * ((nq1 + 63) // 64)


def pftrajectories_mask(ops, frames, qubits, nbits, init_z, reset_planes, events):
    """Reference-structured frame run in mask mode.  Returns (xzs [W', S], meas [S, nbits])."""
    nq1 = qubits + 1
    xzs = np.zeros((frame_words(nq1), frames), dtype=np.uint64)
    meas = np.zeros((nbits, frames), dtype=np.uint8)
    z = np.ascontiguousarray(init_z, dtype=np.uint32)
    L().oracle_frame_init_z(_p(xzs), frames, nq1, _p(z), 0)
    o = np.ascontiguousarray(ops, dtype=OP_DTYPE)
    ev = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    rp = np.ascontiguousarray(reset_planes, dtype=np.uint32)
    L().oracle_pftrajectories(_p(xzs), _p(meas), frames, nq1, nbits, _p(o), len(o), 1, _p(ev), len(ev), _p(rp), 0, 1)
    return xzs, meas.T.astype(bool)


def pftrajectories_rng(ops, frames, qubits, nbits, seed=1, threads=1, as_bool=True):
    """Reference-structured frame run with per-slice Xoshiro draws (the CPU
    baseline and the statistical comparison).  With as_bool=False the record
    is returned as the uint8 array [nbits, frames], which is the reference's
    column-major Bool matrix frames x nbits byte for byte (no conversion)."""
    nq1 = qubits + 1
    xzs = np.zeros((frame_words(nq1), frames), dtype=np.uint64)
    meas = np.zeros((nbits, frames), dtype=np.uint8)
    L().oracle_frame_init_z(_p(xzs), frames, nq1, None, seed)
    o = np.ascontiguousarray(ops, dtype=OP_DTYPE)
    L().oracle_pftrajectories(_p(xzs), _p(meas), frames, nq1, nbits, _p(o), len(o), 2, None, 0, None, seed,
                              int(threads))
    return xzs, (meas.T.astype(bool) if as_bool else meas)


def pftrajectories_philox(ops, frames, qubits, nbits, seed, shot_offset=0):
    """The device's Philox-mode procedure restated (bit-exact check)."""
    nq1 = qubits + 1
    xzs = np.zeros((frame_words(nq1), frames), dtype=np.uint64)
    meas = np.zeros((nbits, frames), dtype=np.uint8)
    L().oracle_philox_init_z(_p(xzs), frames, nq1, seed, shot_offset)
    o = np.ascontiguousarray(ops, dtype=OP_DTYPE)
    L().oracle_pftrajectories_philox(_p(xzs), _p(meas), frames, nq1, nbits, _p(o), len(o), seed, shot_offset)
    return xzs, meas.T.astype(bool)


def coding_mask(nq1):
    """Per-word masks of the coding bits of a frame row (padding excluded)."""
    wp = frame_words(nq1)
    half = wp // 2
    m = np.zeros(wp, dtype=np.uint64)
    for q in range(nq1):
        m[q >> 6] |= np.uint64(1 << (q & 63))
        m[half + (q >> 6)] |= np.uint64(1 << (q & 63))
    return m
