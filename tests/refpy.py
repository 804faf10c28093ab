"""A second, pure-Python restatement of the reference algorithms at the level
of Pauli strings (small sizes only; test infrastructure).

Phases are computed with the single-qubit product table (X*Y = iZ, Y*Z = iX,
Z*X = iY and the reverses with -i), a different method from the oracle's
Stim phase counters, so agreement pins the oracle's bit arithmetic.
Paulis are (phase, x list, z list) with phase the power of i.
"""
from __future__ import annotations

# exponent of i in sigma_a * sigma_b for single-qubit Paulis a, b in (x, z) form
_F = {}
for a in range(4):
    for b in range(4):
        _F[(a, b)] = 0
_X, _Z, _Y = (1, 0), (0, 1), (1, 1)


def _code(x, z):
    return x + 2 * z


_F[(_code(*_X), _code(*_Y))] = 1
_F[(_code(*_Y), _code(*_Z))] = 1
_F[(_code(*_Z), _code(*_X))] = 1
_F[(_code(*_Y), _code(*_X))] = 3
_F[(_code(*_Z), _code(*_Y))] = 3
_F[(_code(*_X), _code(*_Z))] = 3


def mul(l, r):
    """l * r (mul_left!(r, l) result)."""
    lp, lx, lz = l
    rp, rx, rz = r
    ph = lp + rp
    for a, b, c, d in zip(lx, lz, rx, rz):
        ph += _F[(_code(a, b), _code(c, d))]
    return (ph & 3, [a ^ c for a, c in zip(lx, rx)], [b ^ d for b, d in zip(lz, rz)])


def comm(l, r):
    s = 0
    for a, b, c, d in zip(l[1], l[2], r[1], r[2]):
        s ^= (b & c) ^ (a & d)
    return s


def canonicalize(rows, n, phases=True):
    """_canonicalize! on a list of Paulis; returns (rows, rx, rz)."""
    rows = [list(r) for r in rows]
    i = 0
    rx = 0
    for stage in (1, 2):
        for j in range(n):
            k = None
            for ii in range(i, len(rows)):
                if rows[ii][stage][j]:
                    k = ii
                    break
            if k is None:
                continue
            if phases:
                rows[k], rows[i] = rows[i], rows[k]
            else:
                pk, pi = rows[k][0], rows[i][0]
                rows[k], rows[i] = [pk] + rows[i][1:], [pi] + rows[k][1:]
            for m in range(len(rows)):
                if m != i and rows[m][stage][j]:
                    p = mul(rows[i], rows[m])
                    rows[m] = [p[0] if phases else rows[m][0], p[1], p[2]]
            i += 1
        if stage == 1:
            rx = i
    return rows, rx, i
