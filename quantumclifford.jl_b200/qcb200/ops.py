"""Circuit operations with the reference's names and argument meaning.

Each constructor returns a record of the C ABI's ``qcb_op`` (1-based qubits,
1-based record bits, 0 = not recorded), validated like the Julia structs:
``sCNOT(q, q)`` raises ArgumentError, qubit 0 raises the NoZeroQubit error
(src/symbolic_cliffords.jl:88-101, 344-356; src/throws.jl:1).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Iterable, Sequence

import numpy as np

from ._lib import OP_DTYPE, ArgumentError, QCB_EARG, QCB_EZEROQUBIT

# opcodes (enum qcb_opcode)
OP = dict(
    NOP=0, I=1, H=2, S=3, SDAG=4, X=5, Y=6, Z=7, SQRTX=8, INVSQRTX=9, SQRTY=10, INVSQRTY=11,
    HXY=12, HYZ=13, CXYZ=14, CZYX=15,
    CNOT=32, CPHASE=33, SWAP=34, ZCX=35, ZCY=36, ZCZ=37, XCX=38, XCY=39, XCZ=40, YCX=41, YCY=42, YCZ=43,
    MZ=64, MRZ=65, MX=66, MRX=67,
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


def flatten(circuit: Iterable) -> list:
    out = []
    for o in circuit:
        if isinstance(o, Op):
            out.append(o)
        else:
            out.extend(flatten(o))
    return out


def to_array(circuit: Iterable) -> np.ndarray:
    """Pack a circuit into a C-contiguous array of qcb_op records."""
    if isinstance(circuit, np.ndarray) and circuit.dtype == OP_DTYPE:
        return np.ascontiguousarray(circuit)
    ops = flatten(circuit)
    a = np.zeros(len(ops), dtype=OP_DTYPE)
    for i, o in enumerate(ops):
        a[i] = (o.opcode, o.q1, o.q2, o.bit, o.p)
    return a


def affected_counts(arr: np.ndarray) -> tuple[int, int]:
    """(qmax, bmax) as _create_pauliframe computes them (init = 1)."""
    if len(arr) == 0:
        return 1, 1
    qmax = int(max(1, arr["q1"].max(), arr["q2"].max()))
    bmax = int(max(1, arr["bit"].max()))
    return qmax, bmax


def count_updates(arr: np.ndarray) -> int:
    """Clifford gates + measurements (noise not counted)."""
    return int(np.count_nonzero((arr["opcode"] > 0) & (arr["opcode"] < OP["PAULI_NOISE"])))
