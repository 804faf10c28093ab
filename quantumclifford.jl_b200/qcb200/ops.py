"""Circuit operations with the reference's names and argument meaning.

Each constructor returns a record of the C ABI's ``qcb_op`` (1-based qubits,
1-based record bits, 0 = not recorded), validated like the Julia structs:
``sCNOT(q, q)`` raises ArgumentError, qubit 0 raises the NoZeroQubit error
(src/symbolic_cliffords.jl:88-101, 344-356; src/throws.jl:1).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Iterable, Optional, Sequence

import numpy as np

from ._lib import OP_DTYPE, ArgumentError, QCB_EARG, QCB_EZEROQUBIT

# opcodes (enum qcb_opcode)
OP = dict(
    NOP=0, I=1, H=2, S=3, SDAG=4, X=5, Y=6, Z=7, SQRTX=8, INVSQRTX=9, SQRTY=10, INVSQRTY=11,
    HXY=12, HYZ=13, CXYZ=14, CZYX=15, SQO=16,
    CNOT=32, CPHASE=33, SWAP=34, ZCX=35, ZCY=36, ZCZ=37, XCX=38, XCY=39, XCZ=40, YCX=41, YCY=42, YCZ=43,
    SWAPCX=44, INVSWAPCX=45, ISWAP=46, INVISWAP=47, CZSWAP=48, CXSWAP=49, ZCRY=50, INVZCRY=51,
    SQRTZZ=52, INVSQRTZZ=53, SQRTXX=54, INVSQRTXX=55, SQRTYY=56, INVSQRTYY=57,
    MZ=64, MRZ=65, MX=66, MRX=67, XOR=68, XOR_BITS=69,
    PAULI_NOISE=96, DEPOL1=97, DEPOL2=98,
)

NoZeroQubit = "Qubit indices start at 1 (NoZeroQubit)"


@dataclass(frozen=True)
class Op:
    opcode: int
    q1: int
    q2: int = 0
    bit: int = 0
    p: tuple = (0.0, 0.0, 0.0)

    @property
    def name(self) -> str:
        for k, v in OP.items():
            if v == self.opcode:
                return k
        return str(self.opcode)

    def is_noise(self) -> bool:
        return self.opcode >= OP["PAULI_NOISE"]

    def is_gate(self) -> bool:
        return self.opcode < OP["MZ"]


def _q(q: int) -> int:
    if q <= 0:
        raise ArgumentError(QCB_EZEROQUBIT, NoZeroQubit)
    return int(q)


def _one(name: str):
    code = OP[name]

    def make(q: int) -> Op:
        return Op(code, _q(q))

    make.__name__ = name
    return make


def _two(name: str):
    code = OP[name]

    def make(q1: int, q2: int) -> Op:
        _q(q1), _q(q2)
        if q1 == q2:
            raise ArgumentError(
                QCB_EARG,
                "Failed to create a two qubit gate because the two qubits it acts on have the same index. "
                "The qubit indices have to be different.",
            )
        return Op(code, int(q1), int(q2))

    make.__name__ = name
    return make


# single-qubit symbolic gates (src/symbolic_cliffords.jl:105-118)
sId1 = _one("I")
sHadamard = _one("H")
sPhase = _one("S")
sInvPhase = _one("SDAG")
sX = _one("X")
sY = _one("Y")
sZ = _one("Z")
sSQRTX = _one("SQRTX")
sInvSQRTX = _one("INVSQRTX")
sSQRTY = _one("SQRTY")
sInvSQRTY = _one("INVSQRTY")
sHadamardXY = _one("HXY")
sHadamardYZ = _one("HYZ")
sCXYZ = _one("CXYZ")
sCZYX = _one("CZYX")


def SingleQubitOperator(q, xx=None, xz=None, zx=None, zz=None, px=None, pz=None) -> Op:
    """SingleQubitOperator(q, xx, xz, zx, zz, px, pz) (src/symbolic_cliffords.jl
    :168-206): X -> (xx, xz) with sign px, Z -> (zx, zz) with sign pz.  Also
    SingleQubitOperator(gate) for a named single-qubit gate (the reference's
    conversion table, :207-221), and SingleQubitOperator(op, qubit)."""
    if isinstance(q, Op):
        if q.opcode == OP["SQO"]:
            return Op(OP["SQO"], _q(xx if xx is not None else q.q1), q.q2)
        f = _SQO_OF[q.opcode]
        return Op(OP["SQO"], _q(xx if xx is not None else q.q1), f)
    f = sum(int(bool(b)) << i for i, b in enumerate((xx, xz, zx, zz, px, pz)))
    return Op(OP["SQO"], _q(q), f)


def _sqo_flags(xx, xz, zx, zz, px, pz):
    return sum(int(b) << i for i, b in enumerate((xx, xz, zx, zz, px, pz)))


T_, F_ = True, False
_SQO_OF = {  # src/symbolic_cliffords.jl:207-221
    OP["H"]: _sqo_flags(F_, T_, T_, F_, F_, F_), OP["S"]: _sqo_flags(T_, T_, F_, T_, F_, F_),
    OP["SDAG"]: _sqo_flags(T_, T_, F_, T_, T_, F_), OP["I"]: _sqo_flags(T_, F_, F_, T_, F_, F_),
    OP["X"]: _sqo_flags(T_, F_, F_, T_, F_, T_), OP["Y"]: _sqo_flags(T_, F_, F_, T_, T_, T_),
    OP["Z"]: _sqo_flags(T_, F_, F_, T_, T_, F_), OP["CXYZ"]: _sqo_flags(T_, T_, T_, F_, F_, F_),
    OP["CZYX"]: _sqo_flags(F_, T_, T_, T_, F_, F_), OP["HXY"]: _sqo_flags(T_, T_, F_, T_, F_, T_),
    OP["HYZ"]: _sqo_flags(T_, F_, T_, T_, T_, F_), OP["SQRTX"]: _sqo_flags(T_, F_, T_, T_, F_, T_),
    OP["INVSQRTX"]: _sqo_flags(T_, F_, T_, T_, F_, F_), OP["SQRTY"]: _sqo_flags(F_, T_, T_, F_, T_, F_),
    OP["INVSQRTY"]: _sqo_flags(F_, T_, T_, F_, F_, T_),
}


def ClassicalXOR(bits, store) -> list:
    """ClassicalXOR(bits, store) (src/misc_ops.jl:198-205): record bit `store`
    <- XOR of record bits `bits` (1-based, at most 30).  The C ABI form: one
    XOR op (q1 = len(bits), bit = store) and the bits, three per XOR_BITS op."""
    bits = [int(b) for b in bits]
    if not 1 <= len(bits) <= 30:
        raise ArgumentError(QCB_EARG, "ClassicalXOR takes 1 to 30 bits")
    if store <= 0 or min(bits) <= 0:
        raise ArgumentError(QCB_EARG, "record bits start at 1")
    ops = [Op(OP["XOR"], len(bits), 0, int(store))]
    for i in range(0, len(bits), 3):
        b = bits[i:i + 3] + [0] * (3 - len(bits[i:i + 3]))
        ops.append(Op(OP["XOR_BITS"], b[0], b[1], b[2]))
    return ops


class _PauliMeasurementOps(list):
    """The lowered ops of one PauliMeasurement; `nqubits` is the length of its
    Pauli (affectedqubits(::PauliMeasurement) = 1:n, src/affectedqubits.jl:11)."""

    nqubits = 0


def PauliMeasurement(pauli, bit: int) -> list:
    """PauliMeasurement(pauli, bit) on a Pauli frame (src/pauli_frames.jl
    :118-134): through the hidden ancilla n+1 of an n-qubit Pauli, sXCZ / sCNOT
    / sYCX from each qubit with X / Z / Y onto it, then sMRZ(n+1, bit) (the
    sign's sX does not change a frame).  `pauli` is a string like "XIZY" (a
    leading sign is accepted) or an object with `bits()`/`nqubits` (a one-row
    Tableau)."""
    if isinstance(pauli, str):
        body = pauli.strip().lstrip("+-").lstrip("i")
        letters = [ch for ch in body if ch in "IXYZ_"]
    else:
        xs, zs = pauli.bits()
        letters = ["_XZY"[int(x) + 2 * int(z)] for x, z in zip(xs[0], zs[0])]
    n = len(letters)
    anc = n + 1
    ops = _PauliMeasurementOps()
    ops.nqubits = n
    for q, ch in enumerate(letters, start=1):
        if ch == "X":
            ops.append(Op(OP["XCZ"], q, anc))
        elif ch == "Z":
            ops.append(Op(OP["CNOT"], q, anc))
        elif ch == "Y":
            ops.append(Op(OP["YCX"], q, anc))
    ops.append(Op(OP["MRZ"], anc, 0, int(bit)))
    return ops


# two-qubit symbolic gates (src/symbolic_cliffords.jl:358-395)
sCNOT = _two("CNOT")
sCPHASE = _two("CPHASE")
sSWAP = _two("SWAP")
sZCX = _two("ZCX")
sZCY = _two("ZCY")
sZCZ = _two("ZCZ")
sXCX = _two("XCX")
sXCY = _two("XCY")
sXCZ = _two("XCZ")
sYCX = _two("YCX")
sYCY = _two("YCY")
sYCZ = _two("YCZ")
sSWAPCX = _two("SWAPCX")
sInvSWAPCX = _two("INVSWAPCX")
sISWAP = _two("ISWAP")
sInvISWAP = _two("INVISWAP")
sCZSWAP = _two("CZSWAP")
sCXSWAP = _two("CXSWAP")
sZCrY = _two("ZCRY")
sInvZCrY = _two("INVZCRY")
sSQRTZZ = _two("SQRTZZ")
sInvSQRTZZ = _two("INVSQRTZZ")
sSQRTXX = _two("SQRTXX")
sInvSQRTXX = _two("INVSQRTXX")
sSQRTYY = _two("SQRTYY")
sInvSQRTYY = _two("INVSQRTYY")


# measurements (src/symbolic_cliffords.jl:515-655)
def sMZ(q: int, bit: int = 0) -> Op:
    return Op(OP["MZ"], _q(q), 0, int(bit or 0))


def sMRZ(q: int, bit: int = 0) -> Op:
    return Op(OP["MRZ"], _q(q), 0, int(bit or 0))


def sMX(q: int, bit: int = 0) -> Op:
    return Op(OP["MX"], _q(q), 0, int(bit or 0))


def sMRX(q: int, bit: int = 0) -> Op:
    return Op(OP["MRX"], _q(q), 0, int(bit or 0))


# noise (src/noise.jl)
@dataclass(frozen=True)
class PauliNoise:
    px: float
    py: float
    pz: float


@dataclass(frozen=True)
class UnbiasedUncorrelatedNoise:
    p: float


@dataclass(frozen=True)
class DepolarizationNoise:
    p: float

    @staticmethod
    def from_two_qubit_error_probability(e: float) -> "DepolarizationNoise":
        """DepolarizationNoise(; two_qubit_error_probability=e) (src/noise.jl:53)."""
        return DepolarizationNoise(e * 16 / 15)


def NoiseOp(noise, indices: Sequence[int]) -> list:
    """NoiseOp(noise, indices): one op per qubit for Pauli noise (applynoise!
    loops over the indices, src/noise.jl:8-12), one op for depolarisation."""
    idx = [_q(q) for q in indices]
    if isinstance(noise, UnbiasedUncorrelatedNoise):
        noise = PauliNoise(noise.p / 3, noise.p / 3, noise.p / 3)
    if isinstance(noise, PauliNoise):
        return [Op(OP["PAULI_NOISE"], q, 0, 0, (float(noise.px), float(noise.py), float(noise.pz))) for q in idx]
    if isinstance(noise, DepolarizationNoise):
        if len(idx) == 1:
            return [Op(OP["DEPOL1"], idx[0], 0, 0, (float(noise.p), 0.0, 0.0))]
        if len(idx) == 2:
            if idx[0] == idx[1]:
                raise ArgumentError(QCB_EARG, "depolarising noise on a repeated qubit")
            return [Op(OP["DEPOL2"], idx[0], idx[1], 0, (float(noise.p), 0.0, 0.0))]
        raise ArgumentError(QCB_EARG, "DepolarizationNoise on frames supports 1 or 2 qubits")
    raise TypeError(f"unsupported noise model {noise!r}")


def PauliError(qubits, *p) -> list:
    """PauliError(q, p) / PauliError(q, px, py, pz) (src/noise.jl:145-171)."""
    qs = [qubits] if isinstance(qubits, (int, np.integer)) else list(qubits)
    if len(p) == 1:
        return NoiseOp(UnbiasedUncorrelatedNoise(float(p[0])), qs)
    if len(p) == 3:
        return NoiseOp(PauliNoise(*map(float, p)), qs)
    raise TypeError("PauliError(q, p) or PauliError(q, px, py, pz)")


@dataclass(frozen=True)
class NoiseOpAll:
    """NoiseOpAll(noise) (src/noise.jl:173-176, 192-195): the noise on every
    qubit 1..nqubits(frame) of the frame (hidden ancilla excluded,
    src/pauli_frames.jl:14).  Lowered by `flatten` once that count is known:
    `pftrajectories(frame, circuit)` passes the frame's.  Without a frame the
    highest qubit of the other ops is used, the frame the one-call form makes
    (the reference's `_create_pauliframe` has no qubit count for NoiseOpAll,
    src/affectedqubits.jl:22-24, and raises there)."""
    noise: object


def _is_two_qubit(o: Op) -> bool:
    return OP["CNOT"] <= o.opcode <= OP["INVSQRTYY"]


def NoisyGate(gate, noise) -> list:
    """NoisyGate(gate, noise) (src/noise.jl:178-190): the gate, then the
    noise on its qubits (affectedqubits(gate): both qubits of a two-qubit
    gate; 1..n for a PauliMeasurement of an n-qubit Pauli,
    src/affectedqubits.jl:5, 11)."""
    if isinstance(gate, _PauliMeasurementOps):
        return list(gate) + NoiseOp(noise, range(1, gate.nqubits + 1))
    ops = flatten([gate])
    if len(ops) != 1 or ops[0].is_noise() or ops[0].opcode in (OP["XOR"], OP["XOR_BITS"]):
        raise ArgumentError(QCB_EARG, "NoisyGate takes one single- or two-qubit gate or measurement")
    g = ops[0]
    return ops + NoiseOp(noise, (g.q1, g.q2) if _is_two_qubit(g) else (g.q1,))


def flatten(circuit: Iterable, nqubits: Optional[int] = None) -> list:
    """The circuit as a flat list of Op; NoiseOpAll becomes one noise op per
    qubit 1..n (n = nqubits, else the highest qubit of the other ops)."""
    out = []

    def walk(c):
        for o in c:
            if isinstance(o, (Op, NoiseOpAll)):
                out.append(o)
            else:
                walk(o)

    walk(circuit)
    if not any(isinstance(o, NoiseOpAll) for o in out):
        return out
    if nqubits is None:
        rest = [o for o in out if isinstance(o, Op)]
        nqubits = affected_counts(to_array(rest))[0] if rest else 1
    res = []
    for o in out:
        res.extend(NoiseOp(o.noise, range(1, int(nqubits) + 1)) if isinstance(o, NoiseOpAll) else [o])
    return res


def to_array(circuit: Iterable, nqubits: Optional[int] = None) -> np.ndarray:
    """Pack a circuit into a C-contiguous array of qcb_op records
    (``nqubits``: the frame's qubit count, for NoiseOpAll)."""
    if isinstance(circuit, np.ndarray) and circuit.dtype == OP_DTYPE:
        return np.ascontiguousarray(circuit)
    ops = flatten(circuit, nqubits)
    a = np.zeros(len(ops), dtype=OP_DTYPE)
    for i, o in enumerate(ops):
        a[i] = (o.opcode, o.q1, o.q2, o.bit, o.p)
    return a


def affected_counts(arr: np.ndarray) -> tuple[int, int]:
    """(qmax, bmax) as _create_pauliframe computes them (init = 1): the highest
    qubit of any op and the highest record bit (src/affectedqubits.jl)."""
    if len(arr) == 0:
        return 1, 1
    oc = arr["opcode"]
    one_q = ((oc >= OP["I"]) & (oc < OP["XOR"])) | (oc >= OP["PAULI_NOISE"])  # ops with a qubit q1
    two_q = ((oc >= OP["CNOT"]) & (oc <= OP["INVSQRTYY"])) | (oc == OP["DEPOL2"])   # and a second qubit q2
    pay = oc == OP["XOR_BITS"]                                                  # record bits in q1, q2, bit

    def top(v):
        return int(v.max()) if len(v) else 0

    qmax = max(1, top(arr["q1"][one_q]), top(arr["q2"][two_q]))
    bmax = max(1, top(arr["bit"][(oc >= OP["MZ"]) & (oc <= OP["XOR_BITS"])]), top(arr["q1"][pay]), top(arr["q2"][pay]))
    return qmax, bmax


def count_updates(arr: np.ndarray) -> int:
    """Clifford gates + measurements (noise not counted)."""
    return int(np.count_nonzero((arr["opcode"] > 0) & (arr["opcode"] < OP["XOR"])))
