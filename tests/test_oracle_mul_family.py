"""The oracle's mul_left!/mul_right! row family (src/mul_leftright.jl:128-245)
pinned by the relations of test/test_mul_leftright.jl:3-20 and by the
product-table restatement (refpy): p1*p2 == mul_left!(copy(p2), p1) ==
mul_right!(copy(p1), p2); mul_left!(copy(p2), p1) == (-1)^comm(p1,p2) *
mul_right!(copy(p2), p1); Tableau row forms; the Destabilizer form
(:200-219) and the cross-tableau phase source (:171-175)."""
import numpy as np
import pytest

import oracle
import refpy
from qcb200.tableau import Tableau
from test_oracle_golden import _from_py, _to_py

SIZES = [1, 2, 10, 63, 64, 65, 127, 128, 129]


def rand_tab(rows, n, rng):
    return Tableau.from_bits(rng.integers(0, 4, rows), rng.random((rows, n)) < 0.5, rng.random((rows, n)) < 0.5)


@pytest.mark.parametrize("n", SIZES)
def test_pauli_products_left_and_right(orc, n):
    rng = np.random.default_rng(n)
    for _ in range(10):
        p1, p2 = rand_tab(1, n, rng), rand_tab(1, n, rng)
        want = _from_py([refpy.mul(_to_py(p1)[0], _to_py(p2)[0])], n)
        lph, lxz = oracle.mul_rows(p2.phases, p2.xzs, p1.phases, p1.xzs, 1, 1, 1, 0)
        rph, rxz = oracle.mul_rows(p1.phases, p1.xzs, p2.phases, p2.xzs, 1, 1, 1, 0, right=True)
        assert np.array_equal(lxz, want.xzs) and np.array_equal(rxz, want.xzs)
        assert lph[0] == want.phases[0] == rph[0]
        # mul_left!(copy(p2), p1) == (-1)^comm(p1, p2) * mul_right!(copy(p2), p1)
        r2ph, r2xz = oracle.mul_rows(p2.phases, p2.xzs, p1.phases, p1.xzs, 1, 1, 1, 0, right=True)
        c = refpy.comm(_to_py(p1)[0], _to_py(p2)[0])
        assert np.array_equal(r2xz, lxz) and (int(r2ph[0]) + 2 * c) % 4 == lph[0]


@pytest.mark.parametrize("n", [3, 64, 65, 130])
def test_tableau_row_forms(orc, n):
    rng = np.random.default_rng(100 + n)
    s = rand_tab(7, n, rng)
    p = rand_tab(1, n, rng)
    rows = _to_py(s)
    pp = _to_py(p)[0]
    # mul_left!(copy(s), p)[i] == p * s[i]; mul_right!(copy(s), p)[i] == s[i] * p
    lph, lxz = oracle.mul_rows(s.phases, s.xzs, p.phases, p.xzs, 1, 7, 1, 0)
    rph, rxz = oracle.mul_rows(s.phases, s.xzs, p.phases, p.xzs, 1, 7, 1, 0, right=True)
    assert _to_py(Tableau(lph, n, lxz)) == [refpy.mul(pp, r) for r in rows]
    assert _to_py(Tableau(rph, n, rxz)) == [refpy.mul(r, pp) for r in rows]
    # mul_left!(copy(p), s, i) == s[i] * p; mul_right!(copy(p), s, i) == p * s[i]
    for i in (1, 4, 7):
        a = oracle.mul_rows(p.phases, p.xzs, s.phases, s.xzs, 1, 1, i, 0)
        b = oracle.mul_rows(p.phases, p.xzs, s.phases, s.xzs, 1, 1, i, 0, right=True)
        assert _to_py(Tableau(*[a[0], n, a[1]])) == [refpy.mul(rows[i - 1], pp)]
        assert _to_py(Tableau(*[b[0], n, b[1]])) == [refpy.mul(pp, rows[i - 1])]
    # same tableau: mul_left!(s, m, i) = s[i] * s[m]; mul_right!(s, m, i) = s[m] * s[i]
    a = oracle.mul_rows(s.phases, s.xzs, None, None, 2, 1, 5, 0)
    b = oracle.mul_rows(s.phases, s.xzs, None, None, 2, 1, 5, 0, right=True)
    assert _to_py(Tableau(a[0], n, a[1]))[1] == refpy.mul(rows[4], rows[1])
    assert _to_py(Tableau(b[0], n, b[1]))[1] == refpy.mul(rows[1], rows[4])


def test_cross_tableau_phase_source(orc):
    """mul_left!(s, m, t, i) adds s.phases[i] (src/mul_leftright.jl:171-175):
    the product's bits, with the phase of s[i] in place of t[i]'s."""
    rng = np.random.default_rng(5)
    n = 20
    s, t = rand_tab(4, n, rng), rand_tab(4, n, rng)
    t2 = t.copy()
    t2.phases[:] = s.phases  # the same rows with s's phases
    q_ph, q_xz = oracle.mul_rows(s.phases, s.xzs, t.phases, t.xzs, 2, 1, 3, 0, phase_src=1)
    w_ph, w_xz = oracle.mul_rows(s.phases, s.xzs, t2.phases, t2.xzs, 2, 1, 3, 0, phase_src=0)
    assert np.array_equal(q_xz, w_xz) and np.array_equal(q_ph, w_ph)
    rows_s, rows_t2 = _to_py(s), _to_py(t2)
    assert _to_py(Tableau(q_ph, n, q_xz))[1] == refpy.mul(rows_t2[2], rows_s[1])
