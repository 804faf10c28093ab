"""Tableaux, Pauli operators and the tableau hot path on the device.

Host objects use the reference layout (src/QuantumClifford.jl:145-151,
src/pauli_operator.jl:42-48): a row is ``W = 2*ceil(n/64)`` uint64 words, X
words then Z words; phases are uint8 mod 4 (0: +, 1: +i, 2: -, 3: -i).
``to_gpu`` moves them into library-owned device tableaux; the in-place
operations (``mul_left_``, ``canonicalize_``, ``project_``, ``generate_``,
``apply_``) run only on device objects, through the C ABI.
"""
from __future__ import annotations

import ctypes
import re
from typing import Optional

import numpy as np

from . import ops as _ops
from ._lib import QCB_EDIM, DimensionMismatch, check, ensure_init, lib, ptr

KIND = {"Stabilizer": 0, "MixedStabilizer": 1, "Destabilizer": 2, "MixedDestabilizer": 3}


def nwords(n: int) -> int:
    return 2 * ((n + 63) // 64)


class DeviceTableau:
    """Owner of a qcb_tableau handle."""

    def __init__(self, rows: int, nqubits: int):
        ensure_init()
        h = ctypes.c_void_p()
        check(lib().qcb_tableau_create(int(rows), int(nqubits), ctypes.byref(h)))
        self.handle = h
        self._destroy = lib().qcb_tableau_destroy
        self.rows, self.nqubits, self.W = int(rows), int(nqubits), nwords(nqubits)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None

    def upload(self, phases: np.ndarray, xzs: np.ndarray):
        ph = np.ascontiguousarray(phases, dtype=np.uint8)
        xz = np.ascontiguousarray(xzs, dtype=np.uint64)
        assert ph.shape == (self.rows,) and xz.shape == (self.rows, self.W)
        check(lib().qcb_tableau_upload(self.handle, ptr(ph) if ph.size else None, ptr(xz) if xz.size else None, None))

    def download(self):
        ph = np.empty(self.rows, dtype=np.uint8)
        xz = np.empty((self.rows, self.W), dtype=np.uint64)
        check(lib().qcb_tableau_download(self.handle, ptr(ph) if ph.size else None, ptr(xz) if xz.size else None, None))
        return ph, xz


class Tableau:
    """Rows of Pauli operators (host numpy arrays, reference layout), optionally
    mirrored by a device tableau (``self.dev``)."""

    def __init__(self, phases, nqubits: int, xzs):
        self.phases = np.ascontiguousarray(phases, dtype=np.uint8)
        self.nqubits = int(nqubits)
        self.xzs = np.ascontiguousarray(xzs, dtype=np.uint64).reshape(len(self.phases), nwords(nqubits))
        self.dev: Optional[DeviceTableau] = None

    # ----- construction helpers
    @classmethod
    def zeros(cls, rows: int, n: int) -> "Tableau":
        return cls(np.zeros(rows, np.uint8), n, np.zeros((rows, nwords(n)), np.uint64))

    @classmethod
    def from_bits(cls, phases, xs: np.ndarray, zs: np.ndarray) -> "Tableau":
        xs = np.asarray(xs, dtype=bool)
        zs = np.asarray(zs, dtype=bool)
        rows, n = xs.shape
        t = cls.zeros(rows, n)
        t.phases[:] = np.asarray(phases, dtype=np.uint8) & 3
        half = nwords(n) // 2
        if rows and n:
            pad = np.zeros((rows, half * 64), dtype=bool)
            for k, m in enumerate((xs, zs)):  # bit q of a half -> word q >> 6, bit q & 63
                pad[:, :n] = m
                t.xzs[:, k * half:(k + 1) * half] = np.packbits(pad, axis=1, bitorder="little").view("<u8")
        return t

    def bits(self):
        half = self.xzs.shape[1] // 2
        q = np.arange(self.nqubits)
        w, b = q >> 6, (q & 63).astype(np.uint64)
        xs = ((self.xzs[:, w] >> b) & np.uint64(1)).astype(bool)
        zs = ((self.xzs[:, half + w] >> b) & np.uint64(1)).astype(bool)
        return xs, zs

    def __len__(self):
        return len(self.phases)

    def copy(self) -> "Tableau":
        t = Tableau(self.phases.copy(), self.nqubits, self.xzs.copy())
        return t

    def __eq__(self, other) -> bool:
        return (
            isinstance(other, Tableau)
            and self.nqubits == other.nqubits
            and np.array_equal(self.phases, other.phases)
            and np.array_equal(self.xzs, other.xzs)
        )

    def __str__(self) -> str:
        xs, zs = self.bits()
        out = []
        for r in range(len(self)):
            s = {0: "+ ", 1: "+i", 2: "- ", 3: "-i"}[int(self.phases[r])]
            s += "".join("_XZY"[int(x) + 2 * int(z)] for x, z in zip(xs[r], zs[r]))
            out.append(s)
        return "\n".join(out)

    # ----- device mirror
    def to_gpu(self) -> "Tableau":
        if self.dev is None or self.dev.rows != len(self) or self.dev.nqubits != self.nqubits:
            self.dev = DeviceTableau(len(self), self.nqubits)
        self.dev.upload(self.phases, self.xzs)
        return self

    def to_cpu(self) -> "Tableau":
        if self.dev is not None:
            self.phases[:], self.xzs[:] = self.dev.download()
        return self

    def _need_dev(self) -> DeviceTableau:
        if self.dev is None:
            raise TypeError("this object lives on the host; call to_gpu() first (libqcb200 has no CPU path)")
        return self.dev


_PAULI_RE = re.compile(r"^\s*([+-]?)\s*(i?)\s*([XYZI_]+)\s*$")


def _parse_pauli(s: str):
    m = _PAULI_RE.match(s)
    if not m:
        raise ValueError(f"not a Pauli string: {s!r}")
    sign, im, body = m.groups()
    ph = (2 if sign == "-" else 0) + (1 if im else 0)
    xs = np.array([c in "XY" for c in body], dtype=bool)
    zs = np.array([c in "ZY" for c in body], dtype=bool)
    return ph & 3, xs, zs


class PauliOperator(Tableau):
    """A one-row tableau (src/pauli_operator.jl:42-48)."""

    @classmethod
    def from_str(cls, s: str) -> "PauliOperator":
        ph, xs, zs = _parse_pauli(s)
        t = Tableau.from_bits([ph], xs[None, :], zs[None, :])
        p = cls(t.phases, t.nqubits, t.xzs)
        return p

    @property
    def phase(self) -> int:
        return int(self.phases[0])

    @property
    def xz(self) -> np.ndarray:
        return self.xzs[0]


def P(s: str) -> PauliOperator:
    """P"..." string macro."""
    return PauliOperator.from_str(s)


def T(s: str) -> Tableau:
    """A tableau from whitespace/newline separated Pauli strings (S"..." / T"...")."""
    parts = re.findall(r"[+-]?\s*i?\s*[XYZI_]+", s)
    rows = [_parse_pauli(p) for p in parts]
    n = len(rows[0][1])
    return Tableau.from_bits([r[0] for r in rows], np.stack([r[1] for r in rows]), np.stack([r[2] for r in rows]))


class Stabilizer:
    """Stabilizer / MixedStabilizer / Destabilizer / MixedDestabilizer wrapper:
    a tableau plus the kind (and rank for the mixed kinds)."""

    kind = "Stabilizer"

    def __init__(self, tab: Tableau, rank: Optional[int] = None):
        self.tab = tab
        self.rank = rank

    def to_gpu(self):
        self.tab.to_gpu()
        return self

    def to_cpu(self):
        self.tab.to_cpu()
        return self

    def copy(self):
        return type(self)(self.tab.copy(), self.rank)

    @property
    def nqubits(self) -> int:
        return self.tab.nqubits

    def __eq__(self, other):
        return type(self) is type(other) and self.tab == other.tab and self.rank == other.rank

    def __str__(self):
        return str(self.tab)


class MixedStabilizer(Stabilizer):
    kind = "MixedStabilizer"


class Destabilizer(Stabilizer):
    kind = "Destabilizer"


class MixedDestabilizer(Stabilizer):
    kind = "MixedDestabilizer"


def S(s: str) -> Stabilizer:
    return Stabilizer(T(s))


def one_destabilizer(n: int) -> Destabilizer:
    """one(Destabilizer, n): destabilizers X_i, stabilizers Z_i."""
    xs = np.vstack([np.eye(n, dtype=bool), np.zeros((n, n), bool)])
    zs = np.vstack([np.zeros((n, n), bool), np.eye(n, dtype=bool)])
    return Destabilizer(Tableau.from_bits(np.zeros(2 * n), xs, zs))


def one_mixed_destabilizer(r: int, n: int) -> MixedDestabilizer:
    """one(MixedDestabilizer, r, n): X_i destabs / logical X, Z_i stabs / logical Z."""
    d = one_destabilizer(n)
    return MixedDestabilizer(d.tab, r)


def random_clifford_ops(n: int, depth: int, rng: np.random.Generator) -> list:
    """A random circuit of H, S and CNOT layers (used to make random states;
    the reference draws uniform Cliffords with Bravyi-Maslov, src/randoms.jl)."""
    ops = []
    for _ in range(depth):
        for q in range(1, n + 1):
            g = rng.integers(0, 3)
            if g == 0:
                ops.append(_ops.sHadamard(q))
            elif g == 1:
                ops.append(_ops.sPhase(q))
        perm = rng.permutation(n) + 1
        for k in range(0, n - 1, 2):
            ops.append(_ops.sCNOT(int(perm[k]), int(perm[k + 1])))
    return ops


# ------------------------------------------------------------------ hot path
def _tab(x) -> Tableau:
    return x.tab if isinstance(x, Stabilizer) else x


def _mul_rows(s, s_row, count, t, t_row, t_step, right, phase_src, phases):
    st, tt = _tab(s), _tab(t)
    ph = ctypes.c_uint8()
    check(lib().qcb_mul_rows(st._need_dev().handle, int(s_row), int(count), tt._need_dev().handle, int(t_row),
                             int(t_step), int(right), int(phase_src), int(phases),
                             ctypes.byref(ph) if count == 1 else None, None))
    if count == 1 and phases:
        st.phases[s_row - 1] = ph.value
    return s


def _mul_family(right: bool, a, args, phases: bool):
    """Method table of src/mul_leftright.jl:137-245 (and the device methods of
    ext/QuantumCliffordKAExt/mul_leftright.jl:101-460), 1-based rows."""
    if len(args) == 1 and isinstance(_tab(args[0]), PauliOperator) and not isinstance(_tab(a), PauliOperator):
        # mul_left!(s, p) / mul_right!(s, p): every row of s with p
        return _mul_rows(a, 1, len(_tab(a)), args[0], 1, 0, right, 0, phases)
    if len(args) == 1:  # PauliOperator with PauliOperator
        if _tab(a).nqubits != _tab(args[0]).nqubits:
            raise DimensionMismatch(QCB_EDIM, "The two Pauli operators should have the same length!")
        return _mul_rows(a, 1, 1, args[0], 1, 0, right, 0, phases)
    if len(args) == 2 and not isinstance(args[0], (int, np.integer)):
        # mul_left!(p::PauliOperator, s::Tableau/Stabilizer, i)
        return _mul_rows(a, 1, 1, args[0], int(args[1]), 0, right, 0, phases)
    if len(args) == 2:
        i, j = int(args[0]), int(args[1])
        if not right and isinstance(a, (Destabilizer, MixedDestabilizer)):
            # mul_left!(s::(Mixed)Destabilizer, i, j) (src/mul_leftright.jl:200-219)
            check(lib().qcb_mul_left_state(_tab(a)._need_dev().handle, KIND[a.kind], i, j, int(phases), None))
            return a
        # mul_left!(s, m, i) / mul_right!(s, m, i) on one tableau
        return _mul_rows(a, i, 1, a, j, 0, right, 0, phases)
    if len(args) == 3:
        # mul_left!(s::Tableau, m, t::Tableau, i): the reference adds s.phases[i]
        # (src/mul_leftright.jl:171-175, 183-187)
        m, t, i = int(args[0]), args[1], int(args[2])
        return _mul_rows(a, m, 1, t, i, 0, right, 1, phases)
    raise TypeError("no mul_left!/mul_right! method for these arguments")


def mul_left_(a, *args, phases: bool = True):
    """mul_left!(...) on device objects (src/mul_leftright.jl:137-229):
    mul_left!(r, l) (r <- l * r for PauliOperators), mul_left!(p, s, i),
    mul_left!(s, p) (every row), mul_left!(s, m, i), mul_left!(s, m, t, i),
    and mul_left!(::Destabilizer/::MixedDestabilizer, i, j).  Rows are
    1-based.  Returns the first argument."""
    if len(args) == 1 and isinstance(_tab(a), PauliOperator) and isinstance(_tab(args[0]), PauliOperator):
        rt, lt = _tab(a), _tab(args[0])
        ph = ctypes.c_uint8()
        check(lib().qcb_mul_left_pauli(rt._need_dev().handle, lt._need_dev().handle, int(phases), ctypes.byref(ph),
                                       None))
        rt.phases[0] = ph.value if phases else rt.phases[0]
        return a
    return _mul_family(False, a, args, phases)


def mul_right_(a, *args, phases: bool = True):
    """mul_right!(...) on device objects (src/mul_leftright.jl:128-245):
    mul_right!(l, r) (l <- l * r), mul_right!(p, s, i), mul_right!(s, p),
    mul_right!(s, m, i), mul_right!(s, m, t, i).  Rows are 1-based."""
    return _mul_family(True, a, args, phases)


def mul_left_row_(s, m: int, i: int, *, phases: bool = True):
    """mul_left!(s::Tableau, m, i) (1-based rows)."""
    check(lib().qcb_mul_left_row(_tab(s)._need_dev().handle, int(m), int(i), int(phases), None))
    return s


def prodphase(l, r, i: int = 1, j: int = 1) -> int:
    out = ctypes.c_uint8()
    check(lib().qcb_prodphase(_tab(l)._need_dev().handle, i, _tab(r)._need_dev().handle, j, ctypes.byref(out), None))
    return out.value


def comm(l, r, i: int = 1, j: int = 1) -> int:
    out = ctypes.c_uint8()
    check(lib().qcb_comm(_tab(l)._need_dev().handle, i, _tab(r)._need_dev().handle, j, ctypes.byref(out), None))
    return out.value


def _kind_rank(state):
    kind = KIND[state.kind if isinstance(state, Stabilizer) else "Stabilizer"]
    rank = state.rank if getattr(state, "rank", None) is not None else 0
    return kind, rank


def canonicalize_(state, *, phases: bool = True, ranks: bool = False):
    """canonicalize!(state; phases, ranks) (src/canonicalization.jl:92-133) on a
    device state; the Destabilizer kinds carry their destabilizer rows along
    (rowswap!/mul_left! on the state)."""
    dev = _tab(state)._need_dev()
    kind, rank = _kind_rank(state)
    rx, rz = ctypes.c_int32(), ctypes.c_int32()
    check(lib().qcb_canonicalize_state(dev.handle, kind, rank, int(phases), ctypes.byref(rx), ctypes.byref(rz), None))
    if ranks:
        return state, rx.value, rz.value
    return state


def canonicalize_rref_(state, colindices=None, *, phases: bool = True):
    """canonicalize_rref!(state[, colindices]; phases) (src/canonicalization.jl
    :150-185).  Returns (state, i) with the reference's 1-based index i."""
    dev = _tab(state)._need_dev()
    kind, rank = _kind_rank(state)
    if colindices is None:
        colindices = range(1, state.nqubits + 1)
    cols = np.ascontiguousarray(np.asarray(list(colindices), dtype=np.int64).astype(np.uint32))
    i = ctypes.c_int32()
    check(lib().qcb_canonicalize_rref(dev.handle, kind, rank, ptr(cols) if len(cols) else None, len(cols), int(phases),
                                      ctypes.byref(i), None))
    return state, i.value


def canonicalize_gott_(stabilizer, *, phases: bool = True):
    """canonicalize_gott!(stabilizer; phases) (src/canonicalization.jl:206-272).
    Returns (stabilizer, r, s, xperm, zperm), permutations 1-based."""
    if isinstance(stabilizer, Stabilizer) and stabilizer.kind != "Stabilizer":
        raise TypeError("canonicalize_gott! takes a Stabilizer")
    t = _tab(stabilizer)
    dev = t._need_dev()
    n = t.nqubits
    r, sz = ctypes.c_int32(), ctypes.c_int32()
    xp = np.zeros(max(n, 1), np.uint32)
    zp = np.zeros(max(n, 1), np.uint32)
    check(lib().qcb_canonicalize_gott(dev.handle, int(phases), ctypes.byref(r), ctypes.byref(sz), ptr(xp), ptr(zp),
                                      None))
    return stabilizer, r.value, sz.value, xp[:n].astype(np.int64), zp[:n].astype(np.int64)


def permutesystems_(state, perm):
    """permutesystems!(state, perm) (src/linalg.jl:7-17): qubit j of the result
    is qubit perm[j] (1-based) of the input."""
    dev = _tab(state)._need_dev()
    p = np.ascontiguousarray(np.asarray(perm, dtype=np.int64).astype(np.uint32))
    if len(p) != state.nqubits:
        raise ValueError("permutesystems!: the permutation needs one entry per qubit")
    check(lib().qcb_permutesystems(dev.handle, ptr(p) if len(p) else None, None))
    return state


_BASIS = {"X": 1, "Z": 2, "Y": 3}


def _project_qubit(state, basis, qubit, keep_result, phases):
    dev = _tab(state)._need_dev()
    kind, rank0 = _kind_rank(state)
    single = np.isscalar(qubit)
    qs = np.ascontiguousarray(np.atleast_1d(np.asarray(qubit, dtype=np.int64)).astype(np.uint32))
    k = len(qs)
    rank = ctypes.c_int32(rank0)
    anti = np.zeros(max(k, 1), dtype=np.int32)
    res = np.zeros(max(k, 1), dtype=np.int32)
    done = ctypes.c_uint32()
    check(lib().qcb_project_qubit(dev.handle, kind, ctypes.byref(rank), _BASIS[basis], ptr(qs) if k else None, k,
                                  int(keep_result), int(phases), ptr(anti), ptr(res), ctypes.byref(done), None))
    if isinstance(state, (MixedStabilizer, MixedDestabilizer)):
        state.rank = rank.value
    results = [None if v < 0 else int(v) for v in res[:k]]
    if single:
        return state, int(anti[0]), results[0]
    return state, [int(a) for a in anti[:k]], results


def projectX_(state, qubit, *, keep_result: bool = True, phases: bool = True):
    """projectX!(state, qubit) (src/project_trace_reset.jl:446-452); ``qubit``
    may be a sequence (projected in order, one launch)."""
    return _project_qubit(state, "X", qubit, keep_result, phases)


def projectZ_(state, qubit, *, keep_result: bool = True, phases: bool = True):
    """projectZ!(state, qubit) (src/project_trace_reset.jl:460-466)."""
    return _project_qubit(state, "Z", qubit, keep_result, phases)


def projectY_(state, qubit, *, keep_result: bool = True, phases: bool = True):
    """projectY!(state, qubit) (src/project_trace_reset.jl:474-480)."""
    return _project_qubit(state, "Y", qubit, keep_result, phases)


def _projectrand(state, paulis, basis, qubit, rng):
    dev = _tab(state)._need_dev()
    kind, rank0 = _kind_rank(state)
    rng = rng if rng is not None else np.random.default_rng()
    if paulis is not None:
        single = isinstance(paulis, PauliOperator)
        pt = _tab(paulis)
        if pt.dev is None:
            pt.to_gpu()
        k, qs, ph = len(pt), None, pt.dev.handle
    else:
        single = np.isscalar(qubit)
        qs = np.ascontiguousarray(np.atleast_1d(np.asarray(qubit, dtype=np.int64)).astype(np.uint32))
        k, ph = len(qs), None
    rp = (2 * rng.integers(0, 2, size=max(k, 1))).astype(np.uint8)  # rand((0x0, 0x2))
    rank = ctypes.c_int32(rank0)
    anti = np.zeros(max(k, 1), dtype=np.int32)
    res = np.zeros(max(k, 1), dtype=np.int32)
    done = ctypes.c_uint32()
    check(lib().qcb_projectrand(dev.handle, kind, ctypes.byref(rank), ph, _BASIS.get(basis, 0),
                                ptr(qs) if qs is not None and k else None, k, ptr(rp), ptr(anti), ptr(res),
                                ctypes.byref(done), None))
    if isinstance(state, (MixedStabilizer, MixedDestabilizer)):
        state.rank = rank.value
    results = [int(v) for v in res[:k]]
    return (state, results[0]) if single else (state, results)


def projectrand_(state, pauli, *, rng=None):
    """projectrand!(state, pauli) (src/project_trace_reset.jl:627-631): returns
    (state, result) with an undetermined outcome drawn from {0x0, 0x2}."""
    return _projectrand(state, pauli, None, None, rng)


def projectXrand_(state, qubit, *, rng=None):
    """projectXrand!(state, qubit) (src/project_trace_reset.jl:583-587)."""
    return _projectrand(state, None, "X", qubit, rng)


def projectZrand_(state, qubit, *, rng=None):
    """projectZrand!(state, qubit) (src/project_trace_reset.jl:598-602)."""
    return _projectrand(state, None, "Z", qubit, rng)


def projectYrand_(state, qubit, *, rng=None):
    """projectYrand!(state, qubit) (src/project_trace_reset.jl:613-617)."""
    return _projectrand(state, None, "Y", qubit, rng)


def project_(state, paulis, *, keep_result: bool = True, phases: bool = True):
    """project!(state, pauli; keep_result, phases) (src/project_trace_reset.jl:231-439).

    ``paulis``: one PauliOperator or a device Tableau of k Paulis projected in
    order.  Returns (state, anticom, result) with result None for `nothing`
    (lists when k > 1)."""
    t = _tab(state)
    dev = t._need_dev()
    single = isinstance(paulis, PauliOperator)
    pt = _tab(paulis)
    if pt.dev is None:
        pt.to_gpu()
    k = len(pt)
    kind = KIND[state.kind if isinstance(state, Stabilizer) else "Stabilizer"]
    rank = ctypes.c_int32(state.rank if getattr(state, "rank", None) is not None else 0)
    anti = np.zeros(k, dtype=np.int32)
    res = np.zeros(k, dtype=np.int32)
    done = ctypes.c_uint32()
    check(lib().qcb_project(dev.handle, kind, ctypes.byref(rank), pt.dev.handle, int(keep_result), int(phases),
                            ptr(anti), ptr(res), ctypes.byref(done), None))
    if isinstance(state, (MixedStabilizer, MixedDestabilizer)):
        state.rank = rank.value
    results = [None if v < 0 else int(v) for v in res]
    if single:
        return state, int(anti[0]), results[0]
    return state, [int(a) for a in anti], results


def rowswap_(state, i: int, j: int, *, phases: bool = True):
    """rowswap!(state, i, j; phases) (src/QuantumClifford.jl:899-927), 1-based
    rows of the stabilizer view (with the paired destabilizer rows for the
    Destabilizer kinds)."""
    dev = _tab(state)._need_dev()
    kind, _ = _kind_rank(state)
    check(lib().qcb_rowswap(dev.handle, kind, int(i), int(j), int(phases), None))
    return state


_EXPECT_VALUE = {-1: 0, 0: 1, 1: 1j, 2: -1, 3: -1j}


def expect(paulis, state):
    """expect(p, s) (src/project_trace_reset.jl:743-751): the expectation of
    a PauliOperator (or of each row of a device Tableau of Paulis, in one
    launch) on a device state, which is not modified.  Returns 0, 1, -1, 1j or
    -1j (a list for a Tableau of Paulis)."""
    dev = _tab(state)._need_dev()
    kind, rank = _kind_rank(state)
    single = isinstance(paulis, PauliOperator)
    pt = _tab(paulis)
    if pt.dev is None:
        pt.to_gpu()
    k = len(pt)
    out = np.zeros(max(k, 1), np.int32)
    check(lib().qcb_expect(dev.handle, kind, rank, pt.dev.handle, ptr(out), None))
    vals = [_EXPECT_VALUE[int(v)] for v in out[:k]]
    return vals[0] if single else vals


def generate_(pauli: PauliOperator, stab, *, phases: bool = True, saveindices: bool = True):
    """generate!(pauli, stabilizer) (src/project_trace_reset.jl:37-81) on device
    objects.  Returns None (nothing) or (pauli, used_indices)."""
    ok = ctypes.c_int32()
    cap = len(_tab(stab))
    used = np.zeros(max(cap, 1), dtype=np.int32)
    nu = ctypes.c_uint32()
    check(lib().qcb_generate(pauli._need_dev().handle, _tab(stab)._need_dev().handle, int(phases), ctypes.byref(ok),
                             ptr(used), cap, ctypes.byref(nu), None))
    if not ok.value:
        return None
    pauli.to_cpu()
    return (pauli, [int(u) for u in used[: nu.value]]) if saveindices else pauli


def apply_(state, op, *, phases: bool = True):
    """apply!(state, gate) for symbolic gates / gate lists, or dense
    apply!(state, c::CliffordOperator) when ``op`` is a CliffordOperator."""
    t = _tab(state)
    dev = t._need_dev()
    if isinstance(op, CliffordOperator):
        if op.tab.dev is None:
            op.tab.to_gpu()
        check(lib().qcb_apply_dense(dev.handle, op.tab.dev.handle, int(phases), None))
        return state
    arr = _ops.to_array([op] if isinstance(op, _ops.Op) else op)
    check(lib().qcb_apply_gates(dev.handle, ptr(arr), len(arr), int(phases), None))
    return state


class CliffordOperator:
    """Dense Clifford operator: a 2n-row tableau of the images of
    X_1..X_n, Z_1..Z_n (src/dense_cliffords.jl:42-56)."""

    def __init__(self, tab: Tableau):
        assert len(tab) == 2 * tab.nqubits
        self.tab = tab

    def to_gpu(self):
        self.tab.to_gpu()
        return self


def tCNOT() -> CliffordOperator:
    """C"XX IX ZI ZZ" (src/dense_cliffords.jl:222-244)."""
    return CliffordOperator(T("XX IX ZI ZZ"))


def tensor_pow(c: CliffordOperator, k: int) -> CliffordOperator:
    """tensor_pow (src/linalg.jl:303-309): k copies of c on disjoint qubits."""
    m = c.tab.nqubits
    n = m * k
    xs0, zs0 = c.tab.bits()
    xs = np.zeros((2 * n, n), bool)
    zs = np.zeros((2 * n, n), bool)
    ph = np.zeros(2 * n, np.uint8)
    for b in range(k):
        for r in range(m):
            for half in range(2):
                src = half * m + r
                dst = half * n + b * m + r
                xs[dst, b * m:(b + 1) * m] = xs0[src]
                zs[dst, b * m:(b + 1) * m] = zs0[src]
                ph[dst] = c.tab.phases[src]
    return CliffordOperator(Tableau.from_bits(ph, xs, zs))


class CanonBatch:
    """Many canonicalize! jobs (Stabilizer tableaux on the device) drained by
    persistent thread-block clusters in one launch (qcb_canon_batch_*); each
    result equals canonicalize_ of that tableau alone.  ``run(stream)`` is
    capturable in a CUDA graph; ``ranks()`` returns [(rx, rz)] in order."""

    def __init__(self, states, *, phases: bool = True, cluster: int = 0):
        self.states = list(states)
        handles = (ctypes.c_void_p * max(len(self.states), 1))()
        for i, st in enumerate(self.states):
            handles[i] = _tab(st)._need_dev().handle
        h = ctypes.c_void_p()
        check(lib().qcb_canon_batch_create(handles, len(self.states), int(phases), int(cluster), ctypes.byref(h)))
        self.handle = h
        self._destroy = lib().qcb_canon_batch_destroy

    def run(self, stream=None):
        check(lib().qcb_canon_batch_run(self.handle, stream))
        return self

    def ranks(self):
        k = len(self.states)
        rx = np.zeros(max(k, 1), np.int32)
        rz = np.zeros(max(k, 1), np.int32)
        check(lib().qcb_canon_batch_ranks(self.handle, ptr(rx), ptr(rz)))
        return [(int(a), int(b)) for a, b in zip(rx[:k], rz[:k])]

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None
