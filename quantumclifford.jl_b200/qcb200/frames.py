"""Pauli-frame sampling on the device (src/pauli_frames.jl, device side).

``PauliFrame(frames, qubits, measurements)`` allocates a device frame of
``qubits + 1`` qubits (the hidden ancilla of src/pauli_frames.jl:30-37) and
runs initZ! on it.  ``pftrajectories(frame, circuit)`` compiles the circuit
once and runs it with one kernel launch.  Randomness comes either from the
on-device Philox generator (``seed``) or, in mask mode, from a caller event
file (:class:`Masks`), which is how results are compared bit for bit.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import ops as _ops
from ._lib import (
    EVENT_DTYPE, check, ensure_init, lib, ptr, qcb_batch_job, qcb_noise_source, qcb_program_info,
)

QCB_NOISE_PHILOX = 0
QCB_NOISE_MASK = 1


class Program:
    """A compiled circuit (qcb_program)."""

    def __init__(self, circuit, nqubits: Optional[int] = None):
        """``nqubits``: the frame's qubit count, for NoiseOpAll (default: the
        highest qubit of the other ops)."""
        ensure_init()
        self.ops = _ops.to_array(circuit, nqubits)
        h = ctypes.c_void_p()
        check(lib().qcb_program_compile(ptr(self.ops) if len(self.ops) else None, len(self.ops), ctypes.byref(h)))
        self.handle = h
        self._destroy = lib().qcb_program_destroy
        info = qcb_program_info()
        check(lib().qcb_program_info_get(self.handle, ctypes.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in info._fields_}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None


@dataclass
class Masks:
    """Mask-mode randomness shared by the device and the oracle.

    init_z:       uint32 [qubits+1, ceil(S/32)]  initial Z bits (initZ!)
    reset_planes: uint32 [n_resets, ceil(S/32)]  rand(Bool) of each sMRZ/sMRX
    events:       EVENT_DTYPE records (op_index, pauli, shot)
    """

    init_z: np.ndarray
    reset_planes: np.ndarray
    events: np.ndarray


def sample_masks(circuit, frames: int, qubits: Optional[int] = None, seed: int = 0) -> Masks:
    """Draw a seeded event file for ``circuit`` over ``frames`` shots.

    Every noise site fires per frame with its reference probability
    (PauliNoise: X/Z/Y with px/pz/py; DepolarizationNoise(p): with probability
    p a uniform Pauli of the 4^k, identity included), so the file has the
    distribution of the reference's per-frame draws.
    """
    arr = _ops.to_array(circuit, qubits)  # NoiseOpAll over the frame's qubits
    qmax, _ = _ops.affected_counts(arr)
    nq1 = (qubits if qubits is not None else qmax) + 1
    rng = np.random.default_rng(seed)
    words = (frames + 31) // 32
    init_z = rng.integers(0, 2**32, size=(nq1, words), dtype=np.uint64).astype(np.uint32)
    n_resets = int(np.count_nonzero(np.isin(arr["opcode"], [_ops.OP["MRZ"], _ops.OP["MRX"]])))
    reset_planes = rng.integers(0, 2**32, size=(n_resets, words), dtype=np.uint64).astype(np.uint32)
    evs = []
    for k, o in enumerate(arr):
        oc = int(o["opcode"])
        if oc == _ops.OP["PAULI_NOISE"]:
            px, py, pz = (float(v) for v in o["p"])
            r = rng.random(frames)
            code = np.zeros(frames, dtype=np.uint32)
            code[r < px] = 1
            code[(r >= px) & (r < px + pz)] = 2
            code[(r >= px + pz) & (r < px + pz + py)] = 3
        elif oc in (_ops.OP["DEPOL1"], _ops.OP["DEPOL2"]):
            k_q = 2 if oc == _ops.OP["DEPOL2"] else 1
            hit = rng.random(frames) < float(o["p"][0])
            code = np.where(hit, rng.integers(0, 4**k_q, size=frames), 0).astype(np.uint32)
        else:
            continue
        shots = np.nonzero(code)[0]
        if len(shots):
            e = np.zeros(len(shots), dtype=EVENT_DTYPE)
            e["op_index"] = k
            e["pauli"] = code[shots]
            e["shot"] = shots
            evs.append(e)
    events = np.concatenate(evs) if evs else np.zeros(0, dtype=EVENT_DTYPE)
    return Masks(init_z, reset_planes, events)


def _noise_source(seed: int = 0, shot_offset: int = 0, masks: Optional[Masks] = None):
    n = qcb_noise_source()
    if masks is None:
        n.mode = QCB_NOISE_PHILOX
    else:
        n.mode = QCB_NOISE_MASK
        ev = np.ascontiguousarray(masks.events)
        rp = np.ascontiguousarray(masks.reset_planes)
        n.events = ptr(ev) if len(ev) else None
        n.n_events = len(ev)
        n.reset_planes = ptr(rp) if rp.size else None
        n._keep = (ev, rp)  # keep the buffers alive for the call
    n.seed = int(seed) & (2**64 - 1)
    n.shot_offset = int(shot_offset)
    return n


class PauliFrame:
    """A device Pauli frame: ``frames`` shots over ``qubits`` (+1 hidden ancilla)
    qubits with a ``measurements``-bit record."""

    def __init__(self, frames: int, qubits: int, measurements: int, *, seed: int = 0,
                 shot_offset: int = 0, masks: Optional[Masks] = None, init: bool = True):
        ensure_init()
        h = ctypes.c_void_p()
        check(lib().qcb_frame_create(int(frames), int(qubits), int(measurements), ctypes.byref(h)))
        self.handle = h
        self._destroy = lib().qcb_frame_destroy
        self.frames, self.qubits, self.nbits = int(frames), int(qubits), int(measurements)
        self.shot_offset = int(shot_offset)
        if init:
            self.initZ(seed=seed, masks=masks)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None

    def __len__(self):
        return self.frames

    @property
    def words(self) -> int:
        return (self.frames + 31) // 32

    def copy(self) -> "PauliFrame":
        """copy(frame) (src/pauli_frames.jl:17): a new device frame with the
        same x/z bits and record."""
        g = PauliFrame(self.frames, self.qubits, self.nbits, shot_offset=self.shot_offset, init=False)
        check(lib().qcb_frame_copy(g.handle, self.handle, None))
        return g

    def initZ(self, seed: int = 0, masks: Optional[Masks] = None):
        """initZ! (src/pauli_frames.jl:47-56)."""
        if masks is None:
            check(lib().qcb_frame_init_z(self.handle, int(seed), self.shot_offset, None))
        else:
            z = np.ascontiguousarray(masks.init_z, dtype=np.uint32)
            if z.shape != (self.qubits + 1, self.words):
                raise ValueError(f"init_z must have shape {(self.qubits + 1, self.words)}")
            check(lib().qcb_frame_init_z_planes(self.handle, ptr(z), None))
        return self

    def measurements(self) -> np.ndarray:
        """measurements(frame): Bool matrix frames x nbits (src/pauli_frames.jl:280)."""
        out = np.empty((self.nbits, self.frames), dtype=np.uint8)  # column-major frames x nbits
        if out.size:
            check(lib().qcb_frame_download_measurements(self.handle, ptr(out), None))
        return out.T.astype(bool)

    def set_measurements(self, meas: np.ndarray):
        """Load a Bool record matrix (frames x nbits) into the device record."""
        m = np.asfortranarray(np.asarray(meas, dtype=bool)).astype(np.uint8, order="F")
        if m.shape != (self.frames, self.nbits):
            raise ValueError(f"measurements must have shape {(self.frames, self.nbits)}")
        if m.size:
            check(lib().qcb_frame_upload_measurements(self.handle, m.ctypes.data, None))
        return self

    def record_planes(self) -> np.ndarray:
        out = np.empty((self.nbits, self.words), dtype=np.uint32)
        if out.size:
            check(lib().qcb_frame_download_record_planes(self.handle, ptr(out), None))
        return out

    def planes(self):
        x = np.empty((self.qubits + 1, self.words), dtype=np.uint32)
        z = np.empty((self.qubits + 1, self.words), dtype=np.uint32)
        check(lib().qcb_frame_download_planes(self.handle, ptr(x), ptr(z), None))
        return x, z

    def xzs(self) -> np.ndarray:
        """The frame tableau in the reference fastcolumn layout: uint64 array of
        shape (W', frames) (word-major, frames contiguous)."""
        wp = 2 * ((self.qubits + 1 + 63) // 64)
        out = np.empty((wp, self.frames), dtype=np.uint64)
        if out.size:
            check(lib().qcb_frame_download_xzs(self.handle, ptr(out), None))
        return out

    def set_xzs(self, xzs: np.ndarray):
        wp = 2 * ((self.qubits + 1 + 63) // 64)
        a = np.ascontiguousarray(xzs, dtype=np.uint64)
        if a.shape != (wp, self.frames):
            raise ValueError(f"xzs must have shape {(wp, self.frames)}")
        check(lib().qcb_frame_upload_xzs(self.handle, ptr(a), None))
        return self

    def measurement_columns(self, bits, reference=None) -> np.ndarray:
        """measurements(frame)[:, bits] (Bool, frames x len(bits)); with
        ``reference`` (the Register's record, one Bool per bit) it is
        measurements(register, frame)[:, bits] (src/pauli_frames.jl:289)."""
        b = np.ascontiguousarray(np.asarray(bits, dtype=np.int64).astype(np.uint32))
        out = np.empty((len(b), self.frames), dtype=np.uint8)  # column-major frames x nsel
        ref = None if reference is None else np.ascontiguousarray(np.asarray(reference, dtype=np.uint8))
        if ref is not None and len(ref) != self.nbits:
            raise ValueError("reference needs one entry per record bit")
        if out.size:
            check(lib().qcb_frame_measurement_columns(self.handle, ptr(b), len(b), ptr(ref) if ref is not None else None,
                                                      ptr(out), None))
        return out.T.astype(bool)

    def syndrome_rows(self, bits) -> np.ndarray:
        """The syndrome matrix a decoder consumes, shot-major and bit-packed:
        uint64 [frames, ceil(len(bits)/64)], bit b of word w = record bit
        bits[64w+b] of that shot."""
        b = np.ascontiguousarray(np.asarray(bits, dtype=np.int64).astype(np.uint32))
        out = np.zeros((self.frames, (len(b) + 63) // 64), dtype=np.uint64)
        if out.size:
            check(lib().qcb_frame_syndrome_rows(self.handle, ptr(b), len(b), ptr(out), 0, None))
        return out

    def apply(self, op, *, seed: int = 0, masks: Optional[Masks] = None):
        """apply!(frame, op) for one op or a short op list."""
        arr = _ops.to_array([op] if isinstance(op, (_ops.Op, _ops.NoiseOpAll)) else op, self.qubits)
        n = _noise_source(seed, self.shot_offset, masks)
        check(lib().qcb_frame_apply_ops(self.handle, ptr(arr), len(arr), ctypes.byref(n), None))
        return self


def pftrajectories(frame_or_circuit, circuit=None, *, trajectories: int = 5000, seed: int = 0,
                   masks: Optional[Masks] = None, threads: bool = True, program: Optional[Program] = None):
    """pftrajectories(frame, circuit) or pftrajectories(circuit; trajectories)
    (src/pauli_frames.jl:193-239).  ``threads`` is accepted for signature
    parity; the device path has one schedule."""
    if isinstance(frame_or_circuit, PauliFrame):
        frame = frame_or_circuit
        prog = program if program is not None else Program(circuit, frame.qubits)
    else:
        prog = program if program is not None else Program(frame_or_circuit)
        qmax, bmax = _ops.affected_counts(prog.ops)
        frame = PauliFrame(trajectories, qmax, bmax, seed=seed, masks=masks)
    n = _noise_source(seed, frame.shot_offset, masks)
    check(lib().qcb_pftrajectories(frame.handle, prog.handle, ctypes.byref(n), None))
    return frame


# `pauliframe!` is named in the task statement but does not exist in the
# reference; it is an alias of pftrajectories(frame, circuit).
pauliframe_ = pftrajectories


def measurements(frame: PauliFrame) -> np.ndarray:
    return frame.measurements()


def evaluate_guesses(frame: PauliFrame, logical_bits, guesses, faults_submatrix) -> float:
    """evaluate_guesses(measured_faults, guesses, faults_matrix)
    (src/ecc/decoder_pipeline.jl:172-190) with measured_faults =
    measurements(frame)[:, logical_bits], on the device: the fraction of
    shots whose guessed faults, through the faults matrix, miss a measured
    logical bit.  ``guesses``: Bool frames x k (a decoder's batchdecode
    output); ``faults_submatrix``: Bool nlog x k."""
    lb = np.ascontiguousarray(np.asarray(logical_bits, dtype=np.int64).astype(np.uint32))
    g = np.asfortranarray(np.asarray(guesses, dtype=np.uint8))
    f = np.asfortranarray(np.asarray(faults_submatrix, dtype=np.uint8))
    if g.shape[0] != frame.frames or f.shape != (len(lb), g.shape[1]):
        raise ValueError("guesses must be frames x k and the faults matrix len(logical_bits) x k")
    fails = ctypes.c_uint64()
    check(lib().qcb_evaluate_guesses(frame.handle, ptr(lb) if len(lb) else None, len(lb), g.ctypes.data if g.size else None,
                                     g.shape[1], f.ctypes.data if f.size else None, ctypes.byref(fails), None))
    return fails.value / frame.frames if frame.frames else 0.0


def pftrajectories_record(circuit, trajectories: int, seed: int = 0, shot_offset: int = 0,
                          out: Optional[np.ndarray] = None) -> np.ndarray:
    """One-call host API (qcb_pftrajectories_host): returns the record as
    shot-packed planes uint32 [nbits, ceil(trajectories/32)]."""
    ensure_init()
    arr = _ops.to_array(circuit)
    _, bmax = _ops.affected_counts(arr)
    words = (trajectories + 31) // 32
    if out is None:
        out = np.empty((bmax, words), dtype=np.uint32)
    check(lib().qcb_pftrajectories_host(ptr(arr), len(arr), int(trajectories), int(seed), int(shot_offset),
                                        ptr(out), None))
    return out


def unpack_record(planes: np.ndarray, frames: int) -> np.ndarray:
    """Shot-packed record planes -> Bool matrix frames x nbits."""
    b = np.unpackbits(planes.view(np.uint8).reshape(planes.shape[0], -1), axis=1, bitorder="little")
    return b[:, :frames].T.astype(bool)


def pack_record(meas: np.ndarray) -> np.ndarray:
    """Bool matrix frames x nbits -> shot-packed record planes uint32
    [nbits, ceil(frames/32)] (padding shots zero); inverse of unpack_record."""
    meas = np.asarray(meas)
    frames, nbits = meas.shape
    words = (frames + 31) // 32
    b = np.zeros((nbits, words * 32), dtype=np.uint8)
    b[:, :frames] = meas.T
    return np.packbits(b, axis=1, bitorder="little").view(np.uint32)


class Batch:
    """Many fresh sampling runs drained from one persistent launch
    (qcb_batch_*).  ``jobs``: (frame, program, seed[, shot_offset[, tile]])
    tuples; every frame gets initZ! and its circuit in Philox mode, so each
    result equals ``pftrajectories`` of that job alone with the same seed.
    ``run(stream)`` launches (capturable in a CUDA graph); ``status()``
    synchronises and raises on a device-side timeout."""

    def __init__(self, jobs):
        ensure_init()
        self.jobs = list(jobs)
        arr = (qcb_batch_job * max(len(self.jobs), 1))()
        for i, j in enumerate(self.jobs):
            frame, prog, seed = j[0], j[1], j[2]
            off = j[3] if len(j) > 3 else frame.shot_offset
            tile = j[4] if len(j) > 4 else 0
            arr[i] = qcb_batch_job(frame.handle, prog.handle, int(seed) & (2**64 - 1), int(off), int(tile), 0)
        h = ctypes.c_void_p()
        check(lib().qcb_batch_create(arr, len(self.jobs), ctypes.byref(h)))
        self.handle = h
        self._destroy = lib().qcb_batch_destroy

    def run(self, stream=None):
        check(lib().qcb_batch_run(self.handle, stream))
        return self

    def status(self):
        check(lib().qcb_batch_status(self.handle))
        return self

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None


def tune_tile(program: Program, stream=None):
    """The autotuner (qcb_tune_tile): the fastest tile width for the program's
    size class, recorded for later batches.  Returns (tile, us per column)."""
    t = ctypes.c_uint32()
    us = ctypes.c_float()
    check(lib().qcb_tune_tile(program.handle, ctypes.byref(t), ctypes.byref(us), stream))
    return t.value, us.value


def tune_walker(program: Program, frames: int, stream=None):
    """The plain walker's autotuner (qcb_tune_walker): the fastest (tile width,
    threads per CTA) for the program at `frames` shots, recorded for later
    fresh runs of that width.  Returns (tile, threads, ms per run)."""
    t = ctypes.c_uint32()
    th = ctypes.c_uint32()
    ms = ctypes.c_float()
    check(lib().qcb_tune_walker(program.handle, int(frames), ctypes.byref(t), ctypes.byref(th), ctypes.byref(ms),
                                stream))
    return t.value, th.value, ms.value


def tune_walker_clear():
    """Forget every pair the walker's autotuner recorded."""
    check(lib().qcb_tune_walker_clear())


class Server:
    """The serving loop (qcb_server_*): submit sampling requests at any time;
    a scheduler thread admits them against an HBM budget and a number of
    slots and runs them chunk by chunk with continuous batching.  Each
    request's record equals one plain fresh run with the same seed."""

    def __init__(self, hbm_budget_bytes: int, slots: int = 8, chunk_shots: int = 0):
        ensure_init()
        h = ctypes.c_void_p()
        check(lib().qcb_server_create(int(hbm_budget_bytes), int(slots), int(chunk_shots), ctypes.byref(h)))
        self.handle = h
        self._destroy = lib().qcb_server_destroy

    def submit(self, circuit, shots: int, seed: int) -> int:
        arr = _ops.to_array(circuit)
        t = ctypes.c_uint64()
        check(lib().qcb_server_submit(self.handle, ptr(arr) if len(arr) else None, len(arr), int(shots),
                                      int(seed) & (2**64 - 1), ctypes.byref(t)))
        return t.value

    def preload(self, circuit):
        """Compile a circuit into the resident program cache."""
        arr = _ops.to_array(circuit)
        check(lib().qcb_server_preload(self.handle, ptr(arr) if len(arr) else None, len(arr)))

    def query(self, ticket: int):
        """(state, (t_submit, t_admit, t_done)); state 0 queued, 1 running, 2 done."""
        st = ctypes.c_int32()
        times = np.zeros(3, np.float64)
        check(lib().qcb_server_query(self.handle, int(ticket), ctypes.byref(st), ptr(times)))
        return st.value, tuple(float(x) for x in times)

    def next_done(self, timeout: float = 600.0):
        """(ticket, state, (t_submit, t_admit, t_done)) of the next request to
        finish, in completion order (blocks without holding the GIL)."""
        t = ctypes.c_uint64()
        st = ctypes.c_int32()
        times = np.zeros(3, np.float64)
        check(lib().qcb_server_next_done(self.handle, float(timeout), ctypes.byref(t), ctypes.byref(st), ptr(times)))
        return t.value, st.value, tuple(float(x) for x in times)

    def wait(self, ticket: int, timeout: float = 600.0):
        check(lib().qcb_server_wait(self.handle, int(ticket), float(timeout)))

    def result(self, ticket: int, shots: int) -> np.ndarray:
        nb = ctypes.c_uint32()
        check(lib().qcb_server_result(self.handle, int(ticket), None, ctypes.byref(nb)))
        out = np.empty((nb.value, (shots + 31) // 32), dtype=np.uint32)
        if out.size:
            check(lib().qcb_server_result(self.handle, int(ticket), ptr(out), ctypes.byref(nb)))
        return out

    def release(self, ticket: int):
        check(lib().qcb_server_release(self.handle, int(ticket)))

    def stats(self):
        """(device bytes charged to the budget, of which resident programs,
        number of resident programs)."""
        used, prog = ctypes.c_uint64(), ctypes.c_uint64()
        n = ctypes.c_uint32()
        check(lib().qcb_server_stats(self.handle, ctypes.byref(used), ctypes.byref(prog), ctypes.byref(n)))
        return used.value, prog.value, n.value

    def close(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None

    def __del__(self):
        self.close()
