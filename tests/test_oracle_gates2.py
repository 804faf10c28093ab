"""Pins of the two-qubit gate tables of src/symbolic_cliffords.jl:361-395
(SWAPCX ... InvSQRTYY) by group relations with the gates pinned elsewhere,
phases included, on random tableaux through the oracle (a wrong phase flag
or bit map in any entry breaks at least one relation):
inverse pairs compose to the identity; SWAPCX = SWAP then CNOT, CXSWAP =
CNOT then SWAP, CZSWAP = CZ then SWAP; ISWAP^2, SQRTZZ^2 = Z(x)Z,
SQRTXX^2 = X(x)X, SQRTYY^2 = Y(x)Y; SQRTXX = (H(x)H) SQRTZZ (H(x)H);
ZCrY = ZCY then sInvPhase on the control (a controlled +-iY), InvZCrY =
ZCY then sPhase."""
import numpy as np
import pytest

import oracle
from qcb200 import ops as O
from qcb200.randoms import random_destabilizer

N = 5


def apply(seq, ph, xz):
    arr = O.to_array([O.Op(O.OP[name], *qs) for name, qs in seq])
    return oracle.apply_gates(ph, xz, N, arr)


def states():
    rng = np.random.default_rng(2024)
    for _ in range(6):
        d = random_destabilizer(N, rng)
        ph = rng.integers(0, 4, 2 * N).astype(np.uint8)
        yield ph, d.tab.xzs.copy()


RELATIONS = {
    "inverse SWAPCX": ([("SWAPCX", (2, 4)), ("INVSWAPCX", (2, 4))], []),
    "inverse ISWAP": ([("ISWAP", (1, 3)), ("INVISWAP", (1, 3))], []),
    "inverse ZCrY": ([("ZCRY", (5, 2)), ("INVZCRY", (5, 2))], []),
    "inverse SQRTZZ": ([("SQRTZZ", (1, 2)), ("INVSQRTZZ", (1, 2))], []),
    "inverse SQRTXX": ([("SQRTXX", (3, 4)), ("INVSQRTXX", (3, 4))], []),
    "inverse SQRTYY": ([("SQRTYY", (4, 1)), ("INVSQRTYY", (4, 1))], []),
    "inverse CXSWAP": ([("CXSWAP", (2, 3)), ("SWAPCX", (2, 3))], []),
    "SWAPCX": ([("SWAPCX", (2, 4))], [("SWAP", (2, 4)), ("CNOT", (2, 4))]),
    "CXSWAP": ([("CXSWAP", (2, 4))], [("CNOT", (2, 4)), ("SWAP", (2, 4))]),
    "CZSWAP": ([("CZSWAP", (1, 5))], [("CPHASE", (1, 5)), ("SWAP", (1, 5))]),
    "ISWAP^2": ([("ISWAP", (1, 3)), ("ISWAP", (1, 3))], [("Z", (1, 0)), ("Z", (3, 0))]),
    "SQRTZZ^2": ([("SQRTZZ", (1, 2)), ("SQRTZZ", (1, 2))], [("Z", (1, 0)), ("Z", (2, 0))]),
    "SQRTXX^2": ([("SQRTXX", (3, 4)), ("SQRTXX", (3, 4))], [("X", (3, 0)), ("X", (4, 0))]),
    "SQRTYY^2": ([("SQRTYY", (4, 1)), ("SQRTYY", (4, 1))], [("Y", (4, 0)), ("Y", (1, 0))]),
    "InvSQRTYY^2": ([("INVSQRTYY", (4, 1)), ("INVSQRTYY", (4, 1))], [("Y", (4, 0)), ("Y", (1, 0))]),
    "SQRTXX = HH SQRTZZ HH": ([("SQRTXX", (2, 5))],
                              [("H", (2, 0)), ("H", (5, 0)), ("SQRTZZ", (2, 5)), ("H", (2, 0)), ("H", (5, 0))]),
    "ZCrY = ZCY Sdag": ([("ZCRY", (5, 2))], [("ZCY", (5, 2)), ("SDAG", (5, 0))]),
    "InvZCrY = ZCY S": ([("INVZCRY", (5, 2))], [("ZCY", (5, 2)), ("S", (5, 0))]),
}


@pytest.mark.parametrize("name", sorted(RELATIONS))
def test_two_qubit_gate_relations(orc, name):
    lhs, rhs = RELATIONS[name]
    for ph, xz in states():
        a = apply(lhs, ph, xz)
        b = apply(rhs, ph, xz) if rhs else (ph, xz)
        assert np.array_equal(a[1], b[1]), "bits"
        assert np.array_equal(a[0], b[0]), "phases"
