"""Pins the CPU oracle against the reference's own known answers.

Every expected value below is written in the reference's doctests or tests
(file:line cited per case) or follows from its definitions; the pure-Python
restatement in tests/refpy.py (a different phase method) cross-checks the
rest on random inputs.
"""
import numpy as np
import pytest

import refpy
from qcb200 import P, S, T, ops as O
from qcb200.tableau import Tableau, nwords, one_destabilizer, random_clifford_ops


def tab_args(t):
    t = t.tab if hasattr(t, "tab") else t
    return t.phases.copy(), t.xzs.copy(), t.nqubits


def as_tab(ph, xzs, n):
    return Tableau(ph, n, xzs)


def test_philox_known_answers(orc):
    # Random123 known-answer vectors for Philox-4x32-10
    assert list(orc.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(orc.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(orc.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_prodphase_and_comm_doctests(orc):
    # src/QuantumClifford.jl:712-721
    zzz, xxx = P("ZZZ"), P("XXX")
    assert orc.prodphase(zzz.xz, 0, xxx.xz, 0) == 3
    assert orc.prodphase(xxx.xz, 0, zzz.xz, 0) == 1
    # test/test_paulis.jl:40
    assert orc.prodphase(P("XX").xz, 0, P("YY").xz, 0) == 2
    # src/QuantumClifford.jl:776-787 (comm doctest); test/test_paulis.jl:38-39
    assert orc.comm(P("ZZ").xz, P("XX").xz) == 0
    assert orc.comm(P("IZ").xz, P("XX").xz) == 1
    assert orc.comm(P("XX").xz, P("YY").xz) == 0
    assert orc.comm(P("XZ").xz, P("YZ").xz) == 1


def test_pauli_products_doctests(orc):
    # P"ZZZ"*P"XXX" == -iYYY (src/QuantumClifford.jl:712-715): mul_left!(copy(r), l) = l*r
    r, ph = orc.mul_left_pauli(P("XXX").xz, 0, P("ZZZ").xz, 0)
    assert ph == 3 and np.array_equal(r, P("YYY").xz)
    # P"XX"*P"ZZ" == -YY (src/QuantumClifford.jl:776-779)
    r, ph = orc.mul_left_pauli(P("ZZ").xz, 0, P("XX").xz, 0)
    assert ph == 2 and np.array_equal(r, P("YY").xz)


def canon(s, phases=True):
    ph, xz, n = tab_args(s)
    ph, xz, rx, rz = __import__("oracle").canonicalize(ph, xz, n, phases)
    return as_tab(ph, xz, n), rx, rz


def test_canonicalize_doctests(orc):
    # src/canonicalization.jl:9-86
    t, _, _ = canon(S("XXXX ZZII IZZI IIZZ"))
    assert t == T("+ XXXX + Z__Z + _Z_Z + __ZZ")
    t, _, _ = canon(S("XXXX IZZI IIZZ"))
    assert t == T("+ XXXX + _Z_Z + __ZZ")
    t, _, _ = canon(S("XXXX ZZII IZZI IZIZ IIZZ"))
    assert t == T("+ XXXX + Z__Z + _Z_Z + __ZZ + ____")
    s = S("-ZX XZ")
    t, _, _ = canon(s, phases=False)
    assert t == T("- XZ + ZX")
    t, _, _ = canon(s)
    assert t == T("+ XZ - ZX")
    t, rx, rz = canon(S("XXXX ZZII IZIZ ZIIZ"))
    assert (rx, rz) == (1, 3)
    assert t == T("+ XXXX + Z__Z + _Z_Z + ____")


def test_canonicalize_ten_qubit_golden(orc):
    # test/test_stabcanon.jl:5-26
    s = S("""- XZZZZ_____
            - _YZY___YX_
            - __XXZ__YX_
            + Z_Z_Y__YXZ
            + _____Z____
            + __________
            + __________
            + ______YYX_
            + __________
            + __________""")
    want = T("""- XZZZZ_____
            - _YZY___YX_
            - __XXZ__YX_
            + Z_Z_Y__YXZ
            + ______YYX_
            + _____Z____
            + __________
            + __________
            + __________
            + __________""")
    t, _, _ = canon(s)
    assert t == want


def proj(kind, state, pauli, rank=0, keep_result=True, phases=True):
    import oracle

    ph, xz, n = tab_args(state)
    st, ph, xz, rank, a, r = oracle.project(kind, ph, xz, n, pauli.xz, pauli.phase, rank, keep_result, phases)
    return st, as_tab(ph, xz, n), rank, a, (None if r < 0 else r)


def test_project_doctests(orc):
    # src/project_trace_reset.jl:110-137
    ghz, _, _ = canon(S("XXXX ZZII IZZI IIZZ"))
    st, t, _, a, r = proj("Stabilizer", ghz, P("ZIII"))
    assert t == T("+ Z___ + Z__Z + _Z_Z + __ZZ") and (a, r) == (1, None)
    t2, _, _ = canon(t)
    assert t2 == T("Z___ _Z__ __Z_ ___Z")
    # :139-160
    s, _, _ = canon(S("ZII IXI IIY"))
    assert s == T("+ _X_ + __Y + Z__")
    st, t, _, a, r = proj("Stabilizer", s, P("-ZII"))
    assert t == T("+ _X_ + __Y + Z__") and (a, r) == (0, 2)
    # :162-178: incomplete tableau, projector not generated -> anticom = rank + 1
    st, t, _, a, r = proj("Stabilizer", S("XZI IZI"), P("IIX"))
    assert t == T("+ X__ + _Z_") and (a, r) == (3, None)
    # :186-197  one(MixedStabilizer, 2, 3)
    ms = T("Z__ _Z_ __Z")
    st, t, rank, a, r = proj("MixedStabilizer", ms, P("IIX"), rank=2)
    assert rank == 3 and a == 3 and r is None
    assert as_tab(t.phases[:3], t.xzs[:3], 3) == T("+ Z__ + _Z_ + __X")
    # :199-225  one(MixedDestabilizer, 2, 3)
    md = one_destabilizer(3).tab
    st, t, rank, a, r = proj("MixedDestabilizer", md, P("IIX"), rank=2)
    assert rank == 3 and a == 3 and r is None
    assert as_tab(t.phases[:3], t.xzs[:3], 3) == T("+ X__ + _X_ + __Z")
    assert as_tab(t.phases[3:], t.xzs[3:], 3) == T("+ Z__ + _Z_ + __X")


def test_projection_tests(orc):
    # test/test_projections.jl:9-25
    s = S("XXX ZZI IZZ")
    st, t, _, a, r = proj("Stabilizer", s, P("ZII"))
    t2, _, _ = canon(t)
    assert a == 1 and r is None and t2 == T("ZII IZI IIZ")
    st, t, _, a, r = proj("Stabilizer", s, P("-XXX"))
    c, _, _ = canon(s)
    assert a == 0 and r == 2 and t == c
    st, t, _, a, r = proj("Stabilizer", s, P("-XXX"), keep_result=False)
    assert a == 0 and r is None and t == s.tab
    # test/test_projections.jl:66-96 (Stabilizer and MixedStabilizer parts)
    s = S(" XXX -ZZI")
    st, t, _, a, r = proj("Stabilizer", s, P("IZZ"))
    assert a == 3 and r is None
    big = Tableau.zeros(3, 3)
    big.phases[:2], big.xzs[:2] = s.tab.phases, s.tab.xzs
    st, t, rank, a, r = proj("MixedStabilizer", big, P("IZZ"), rank=2)
    assert rank == 3 and a == 3 and r is None
    st, t, _, a, r = proj("Stabilizer", s, P("ZZI"))
    assert a == 0 and r == 2
    st, t, rank, a, r = proj("MixedStabilizer", big, P("ZZI"), rank=2)
    assert rank == 2 and a == 0 and r == 2


def test_generate_doctests(orc):
    import oracle

    # src/project_trace_reset.jl:10-35
    ghz, _, _ = canon(S("XXXX ZZII IZZI IIZZ"))
    p = P("-ZIZI")
    ok, rest, ph, used = oracle.generate(p.xz, p.phase, ghz.phases, ghz.xzs, 4)
    assert ok and not rest.any() and ph == 2 and used == [2, 4]
    c, _, _ = canon(S("ZII"))
    assert not oracle.generate(P("XII").xz, 0, c.phases, c.xzs, 3)[0]
    c, _, _ = canon(S("XII"))
    assert oracle.generate(P("XII").xz, 0, c.phases, c.xzs, 3)[0]


def test_dense_tcnot_doctest(orc):
    import oracle

    # src/dense_cliffords.jl:4-22: tCNOT * S"XI IZ" == S"XX ZZ"
    c = T("XX IX ZI ZZ")
    s = T("XI IZ")
    ph, xz = oracle.apply_dense(s.phases, s.xzs, 2, c.phases, c.xzs)
    assert as_tab(ph, xz, 2) == T("+ XX + ZZ")


def _to_py(t):
    xs, zs = t.bits()
    return [(int(t.phases[r]), [int(v) for v in xs[r]], [int(v) for v in zs[r]]) for r in range(len(t))]


def _from_py(rows, n):
    import numpy as np

    return Tableau.from_bits([r[0] for r in rows], np.array([r[1] for r in rows], bool).reshape(len(rows), n),
                             np.array([r[2] for r in rows], bool).reshape(len(rows), n))


@pytest.mark.parametrize("n", [1, 2, 10, 63, 64, 65, 127, 128, 129])
def test_mul_left_against_table_method(orc, n):
    import oracle

    rng = np.random.default_rng(n)
    for _ in range(10):
        a = Tableau.from_bits(rng.integers(0, 4, 1), rng.random((1, n)) < 0.5, rng.random((1, n)) < 0.5)
        b = Tableau.from_bits(rng.integers(0, 4, 1), rng.random((1, n)) < 0.5, rng.random((1, n)) < 0.5)
        r, ph = oracle.mul_left_pauli(b.xzs[0], b.phases[0], a.xzs[0], a.phases[0])
        want = refpy.mul(_to_py(a)[0], _to_py(b)[0])
        got = _to_py(as_tab([ph], r[None, :], n))[0]
        assert got == (want[0], want[1], want[2])
        assert oracle.comm(a.xzs[0], b.xzs[0]) == refpy.comm(_to_py(a)[0], _to_py(b)[0])
        # prodphase is the phase of the product
        assert oracle.prodphase(a.xzs[0], a.phases[0], b.xzs[0], b.phases[0]) == want[0]


def random_stabilizer_tab(n, rng, depth=None):
    d = one_destabilizer(n)
    ops = O.to_array(random_clifford_ops(n, depth or max(4, n // 2), rng))
    import oracle

    ph, xz = oracle.apply_gates(d.tab.phases, d.tab.xzs, n, ops)
    full = as_tab(ph, xz, n)
    return full, as_tab(ph[n:], xz[n:], n)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 10, 17])
@pytest.mark.parametrize("phases", [True, False])
def test_canonicalize_against_table_method(orc, n, phases):
    rng = np.random.default_rng(100 + n)
    for rows in (n, max(1, n // 2), n + 2):
        _, st = random_stabilizer_tab(n, rng)
        t = Tableau.zeros(rows, n)
        k = min(rows, n)
        t.phases[:k], t.xzs[:k] = st.phases[:k], st.xzs[:k]
        if rows > n:  # redundant rows: products of existing ones
            for r in range(n, rows):
                t.xzs[r] = t.xzs[r - n] ^ t.xzs[(r - n + 1) % n]
        got, rx, rz = canon(t, phases)
        want, wrx, wrz = refpy.canonicalize(_to_py(t), n, phases)
        assert (rx, rz) == (wrx, wrz)
        assert got == _from_py(want, n)


GATES1 = ["I", "H", "S", "SDAG", "X", "Y", "Z", "SQRTX", "INVSQRTX", "SQRTY", "INVSQRTY", "HXY", "HYZ", "CXYZ", "CZYX"]
GATES2 = ["CNOT", "CPHASE", "SWAP", "ZCX", "ZCY", "ZCZ", "XCX", "XCY", "XCZ", "YCX", "YCY", "YCZ",
          "SWAPCX", "INVSWAPCX", "ISWAP", "INVISWAP", "CZSWAP", "CXSWAP", "ZCRY", "INVZCRY", "SQRTZZ", "INVSQRTZZ",
          "SQRTXX", "INVSQRTXX", "SQRTYY", "INVSQRTYY"]


@pytest.mark.parametrize("gate", GATES1 + GATES2)
def test_symbolic_gates_match_their_dense_form(orc, gate):
    """test/test_symcliff.jl:8-60: a symbolic gate and the dense operator built
    from its action on the generators act identically (phases included)."""
    import oracle

    n = 3
    code = O.OP[gate]
    q = [2, 3] if gate in GATES2 else [2]
    op = np.zeros(1, dtype=oracle.OP_DTYPE)
    op[0] = (code, q[0], q[1] if len(q) > 1 else 0, 0, (0, 0, 0))
    ident = one_destabilizer(n).tab  # rows X_1..X_n, Z_1..Z_n: the images define the operator
    cph, cxz = oracle.apply_gates(ident.phases, ident.xzs, n, op)
    rng = np.random.default_rng(7)
    for _ in range(5):
        _, st = random_stabilizer_tab(n, rng)
        st.phases[:] = rng.integers(0, 4, n)
        a_ph, a_xz = oracle.apply_gates(st.phases, st.xzs, n, op)
        d_ph, d_xz = oracle.apply_dense(st.phases, st.xzs, n, cph, cxz)
        assert np.array_equal(a_xz, d_xz)
        assert np.array_equal(a_ph, d_ph)


@pytest.mark.parametrize("gate", GATES1)
def test_single_qubit_operator_of_each_named_gate_acts_like_it(orc, gate):
    """SingleQubitOperator(g) (the reference's table, src/symbolic_cliffords.jl
    :207-221) acts like g on random tableaux, phases included
    (test/test_symcliff.jl compares them the same way)."""
    import oracle

    n = 3
    named = np.zeros(1, dtype=oracle.OP_DTYPE)
    named[0] = (O.OP[gate], 2, 0, 0, (0, 0, 0))
    sqo = O.to_array([O.SingleQubitOperator(O.Op(O.OP[gate], 2))])
    rng = np.random.default_rng(13)
    for _ in range(5):
        _, st = random_stabilizer_tab(n, rng)
        st.phases[:] = rng.integers(0, 4, n)
        a_ph, a_xz = oracle.apply_gates(st.phases, st.xzs, n, named)
        b_ph, b_xz = oracle.apply_gates(st.phases, st.xzs, n, sqo)
        assert np.array_equal(a_xz, b_xz)
        assert np.array_equal(a_ph, b_ph)


def test_frame_ghz_correlations(orc):
    """test/test_pauliframe.jl:30-52: GHZ records have row sums 0 or 3 and
    mean 1/2."""
    import oracle

    circ = O.to_array([O.sHadamard(1), O.sCNOT(1, 2), O.sCNOT(1, 3), O.sMZ(1, 1), O.sMZ(2, 2), O.sMZ(3, 3)])
    n = 200_000
    _, m = oracle.pftrajectories_rng(circ, n, 3, 3, seed=11, threads=4)
    tot = m.sum(axis=1)
    assert np.all(tot % 3 == 0)
    frac = tot.sum() / 3 / n
    assert 0.49 < frac < 0.51


def test_frame_repetition_syndrome(orc):
    """test/test_pauliframe.jl:2-27: an X error on qubit 2 flips both syndromes."""
    import oracle

    circ = O.to_array([O.sX(1), O.sCNOT(1, 2), O.sCNOT(1, 3)] + O.PauliError(2, 0.75) +
                      [O.sCNOT(1, 4), O.sCNOT(2, 4), O.sCNOT(2, 5), O.sCNOT(3, 5), O.sMZ(4, 1), O.sMZ(5, 2)])
    xzs, m = oracle.pftrajectories_rng(circ, 100, 5, 2, seed=3)
    half = xzs.shape[0] // 2
    for f in range(100):
        x2 = (xzs[0, f] >> np.uint64(1)) & np.uint64(1)
        z2 = (xzs[half, f] >> np.uint64(1)) & np.uint64(1)
        if x2 and not z2:
            x4 = (xzs[0, f] >> np.uint64(3)) & np.uint64(1)
            x5 = (xzs[0, f] >> np.uint64(4)) & np.uint64(1)
            assert x4 and x5 and m[f, 0] and m[f, 1]


def test_frame_reset_semantics(orc):
    """sMRZ records x, clears x and randomises z; sMZ with bit 0 is a no-op;
    sMX applies sHadamard and does not undo it (src/pauli_frames.jl:74-116)."""
    import oracle

    S_ = 64
    circ = O.to_array([O.sX(1), O.sMRZ(1, 1), O.sMZ(1, 2)])
    init_z = np.zeros((2, 2), np.uint32)
    reset = np.full((1, 2), 0xFFFFFFFF, np.uint32)
    ev = np.zeros(0, dtype=oracle.EVENT_DTYPE)
    xzs, m = oracle.pftrajectories_mask(circ, S_, 1, 2, init_z, reset, ev)
    # sX does not change frames; record is x = 0; after reset z is all ones
    assert not m.any()
    assert np.all(xzs[1] & np.uint64(1))
    # x error then measurement
    circ = O.to_array(O.PauliError(1, 1.0, 0, 0) + [O.sMZ(1, 1), O.sMZ(1, 0), O.sMX(1, 2)])
    ev = np.zeros(S_, dtype=oracle.EVENT_DTYPE)
    ev["op_index"], ev["pauli"], ev["shot"] = 0, 1, np.arange(S_)
    xzs, m = oracle.pftrajectories_mask(circ, S_, 1, 2, init_z, np.zeros((0, 2), np.uint32), ev)
    assert m[:, 0].all() and not m[:, 1].any()
    # after sMX the H stays applied: x moved to z
    assert np.all(xzs[1] & np.uint64(1)) and not np.any(xzs[0] & np.uint64(1))


# ------------------------------------------------------------------ state kinds, rref, gott, projectX/Y/Z
def random_mixed_destabilizer_tab(r, n, rng):
    """A random valid MixedDestabilizer tableau of rank r (one(MixedDestabilizer,
    r, n) under a random Clifford circuit): rows 0..n-1 destabilizers then
    logical X, rows n..2n-1 stabilizers then logical Z."""
    import oracle

    d = one_destabilizer(n)
    ops = O.to_array(random_clifford_ops(n, max(4, n // 2), rng))
    return oracle.apply_gates(d.tab.phases, d.tab.xzs, n, ops)


def symplectic_ok(xzs, n, r=None):
    """The pairing checks of destab_looks_good / mixed_destab_looks_good
    (src/misc.jl): rows i and n+j anticommute iff i == j, all other pairs
    commute."""
    import oracle

    rows = xzs.shape[0]
    for i in range(rows):
        for j in range(i + 1, rows):
            want = 1 if (rows == 2 * n and j == i + n) else 0
            if oracle.comm(xzs[i], xzs[j]) != want:
                return False
    return True


def stab_commutes(xzs):
    import oracle

    return all(oracle.comm(xzs[i], xzs[j]) == 0 for i in range(len(xzs)) for j in range(i + 1, len(xzs)))


@pytest.mark.parametrize("n", [1, 3, 10, 64, 65, 100])
@pytest.mark.parametrize("phases", [True, False])
def test_canonicalize_state_kinds_agree(orc, n, phases):
    # test/test_stabcanon.jl:44-72: canonicalize! and canonicalize_rref! give the
    # same stabilizer view for Stabilizer, MixedStabilizer, Destabilizer and
    # MixedDestabilizer, and the destabilizer kinds stay well formed
    rng = np.random.default_rng(500 + n)
    for r in sorted({n, max(1, n // 3), max(1, 2 * n // 3)}):
        ph, xz = random_mixed_destabilizer_tab(r, n, rng)
        sv = slice(n, n + r)
        c_ph, c_xz, rx, rz = orc.canonicalize(ph[sv], xz[sv], n, phases)
        kinds = [("MixedDestabilizer", ph, xz, r), ("MixedStabilizer", ph[sv], xz[sv], r)]
        if r == n:
            kinds += [("Destabilizer", ph, xz, 0), ("Stabilizer", ph[sv], xz[sv], 0)]
        for kind, p0, x0, rank in kinds:
            p1, x1, rx1, rz1 = orc.canonicalize_state(kind, p0, x0, n, rank, phases)
            off = n if "Destabilizer" in kind else 0
            assert np.array_equal(x1[off:off + r], c_xz) and (rx1, rz1) == (rx, rz), kind
            if phases:
                assert np.array_equal(p1[off:off + r], c_ph), kind
            if "Destabilizer" in kind:
                assert symplectic_ok(x1, n), kind
            cols = np.arange(1, n + 1)
            q1, y1, i1 = orc.canonicalize_rref(kind, p0, x0, n, cols, rank, phases)
            if kind == "MixedDestabilizer":
                want_view = y1[n:n + r].copy()
                want_i = i1
            else:
                assert np.array_equal(y1[off:off + r], want_view) and i1 == want_i, kind
            if "Destabilizer" in kind:
                assert symplectic_ok(y1, n), kind
            # canonicalize!(canonicalize_rref!(s)) == canonicalize!(s)
            # (test/test_stabcanon.jl:76-87)
            z_ph, z_xz, _, _ = orc.canonicalize(q1[off:off + r], y1[off:off + r], n, phases)
            assert np.array_equal(z_xz, c_xz), kind


def test_canonicalize_rref_partial_columns(orc):
    # canonicalize_rref!(state, colindices) on a subset, as traceout! uses it
    # (src/project_trace_reset.jl:643-660): pivots only in those columns, the
    # rows below the returned i are free of them
    rng = np.random.default_rng(7)
    n = 12
    ph, xz = random_mixed_destabilizer_tab(n, n, rng)
    cols = [3, 7, 8, 12]
    p1, x1, i = orc.canonicalize_rref("Stabilizer", ph[n:], xz[n:], n, cols)
    assert n - 2 * len(cols) <= i <= n  # the reference's `i`: rows i+1..n hold the pivots
    W = xz.shape[1]
    for row in range(i):  # rows 1..i (1-based) have no X or Z on the columns
        for c in cols:
            q = c - 1
            assert not (x1[row, q >> 6] >> np.uint64(q & 63)) & np.uint64(1)
            assert not (x1[row, W // 2 + (q >> 6)] >> np.uint64(q & 63)) & np.uint64(1)
    assert stab_commutes(x1)


@pytest.mark.parametrize("n", [1, 2, 5, 10, 63, 64, 65, 100])
def test_canonicalize_gott_invariants(orc, n):
    # test/test_stabcanon.jl:31-43: canonicalize!(permute(permute(s, p1), p2)) ==
    # canonicalize!(gott(s)), the result still a stabilizer; plus the standard
    # form it is named for (identity blocks in the X then Z pivot columns)
    rng = np.random.default_rng(900 + n)
    for rows in sorted({n, max(1, n // 3), max(1, 2 * n // 3)}):
        ph, xz = random_mixed_destabilizer_tab(rows, n, rng)
        s_ph, s_xz = ph[n:n + rows], xz[n:n + rows]
        g_ph, g_xz, r, s, xp, zp = orc.canonicalize_gott(s_ph, s_xz, n)
        assert sorted(xp) == list(range(1, n + 1)) and sorted(zp) == list(range(1, n + 1))
        p = orc.permutesystems(orc.permutesystems(s_xz, n, xp), n, zp)
        _, c1, _, _ = orc.canonicalize(s_ph, p, n)
        _, cg, _, _ = orc.canonicalize(g_ph, g_xz, n)
        assert np.array_equal(c1, cg)
        assert stab_commutes(g_xz)
        assert r + s <= rows
        W = xz.shape[1]
        bit = lambda row, half, q: int((g_xz[row, half * (W // 2) + (q >> 6)] >> np.uint64(q & 63)) & np.uint64(1))
        for a in range(r):
            assert [bit(a, 0, q) for q in range(r)] == [int(q == a) for q in range(r)]
        for a in range(s):
            assert [bit(r + a, 1, q) for q in range(r, r + s)] == [int(q == a) for q in range(s)]


@pytest.mark.parametrize("n", [1, 2, 3, 10, 64, 65, 100])
@pytest.mark.parametrize("phases", [True, False])
def test_project_xyz_equals_project_single_pauli(orc, n, phases):
    # test/test_projections.jl:291-317: project!(s, single_x(n, r)) ==
    # projectX!(s, r) (and Y, Z) on MixedDestabilizer(random_destabilizer(n), n÷2),
    # also after a first projection, with keep_result both ways
    rng = np.random.default_rng(1300 + n)
    W = nwords(n)
    for trial in range(4):
        rank = max(0, n // 2) if trial < 2 else n
        ph, xz = random_mixed_destabilizer_tab(rank, n, rng)
        for step in range(3):
            q = int(rng.integers(1, n + 1))
            basis = int(rng.integers(1, 4))
            keep = bool(rng.integers(2)) if trial % 2 else True
            p = np.zeros(W, np.uint64)
            if basis & 1:
                p[(q - 1) >> 6] |= np.uint64(1) << np.uint64((q - 1) & 63)
            if basis & 2:
                p[W // 2 + ((q - 1) >> 6)] |= np.uint64(1) << np.uint64((q - 1) & 63)
            st, ph1, xz1, r1, a1, res1 = orc.project("MixedDestabilizer", ph, xz, n, p, 0, rank, keep, phases)
            ph2, xz2, r2, a2, res2 = orc.project_cond(ph, xz, n, rank, q, basis, keep, phases)
            assert st == 0
            assert (r1, a1, res1) == (r2, a2, res2)
            assert np.array_equal(xz1, xz2) and np.array_equal(ph1, ph2)
            ph, xz, rank = ph2, xz2, r2


def test_project_xyz_known_answers(orc):
    # test/test_projections.jl:349-370: on S"XII -IZI IIY" the single-qubit
    # projections agree with project! of the Pauli: X1 -> 0x0, Z2 -> 0x2, Y3 -> 0x0
    # (destabilizers Z1, X2, Z3 pair with the three stabilizers)
    t = T("+Z__ +_X_ +__Z +X__ -_Z_ +__Y")
    for q, basis, want in [(1, 1, 0), (2, 2, 2), (3, 3, 0)]:
        _, _, rank, a, res = orc.project_cond(t.phases, t.xzs, 3, 3, q, basis)
        assert (rank, a, res) == (3, 0, want)


def test_evaluate_guesses_restatement(orc):
    # src/ecc/decoder_pipeline.jl:172-190 on small matrices, against the
    # definition: a sample fails when any row of faults . guess (mod 2)
    # differs from the measured logical bit
    rng = np.random.default_rng(4)
    for S, nlog, k in [(1, 1, 1), (50, 2, 7), (300, 4, 30)]:
        m = rng.random((S, nlog)) < 0.5
        g = rng.random((S, k)) < 0.5
        f = rng.random((nlog, k)) < 0.5
        frac, cnt = orc.evaluate_guesses(m, g, f)
        want = int(np.count_nonzero(((g.astype(int) @ f.T.astype(int)) % 2 != m).any(axis=1)))
        assert cnt == want and frac == want / S
    # a perfect decoder never fails
    g = rng.random((40, 6)) < 0.5
    f = rng.random((3, 6)) < 0.5
    assert orc.evaluate_guesses((g.astype(int) @ f.T.astype(int)) % 2 == 1, g, f)[1] == 0


def oracle_expect(kind, ph, xz, n, p_xz, p_ph, rank=0):
    """expect(p, s) = project!(copy(s), p) mapped (src/project_trace_reset.jl:743-751)."""
    st, _, _, _, a, r = orc_mod().project(kind, ph, xz, n, p_xz, p_ph, rank)
    assert st == 0
    return {-1: 0, 0: 1, 1: 1j, 2: -1, 3: -1j}[r]


def orc_mod():
    import oracle

    return oracle


def test_expect_known_answers(orc):
    # test/test_expect.jl:33-40: bell() with sX(2) applied is +XX, -ZZ
    st = S("+XX -ZZ").tab
    for pauli, want in [("XX", 1), ("ZZ", -1), ("XI", 0), ("ZI", 0), ("II", 1), ("-XX", -1), ("-iXX", -1j)]:
        p = P(pauli)
        assert oracle_expect("Stabilizer", st.phases, st.xzs, 2, p.xz, p.phase) == want, pauli
