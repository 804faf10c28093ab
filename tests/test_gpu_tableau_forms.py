"""GPU parity tests (through the C ABI) for the canonical forms and the
single-qubit projections: canonicalize! on every state kind (the
Destabilizer kinds carry their destabilizer rows), canonicalize_rref!,
canonicalize_gott!, permutesystems!, projectX!/Y!/Z! and the projectrand!
family, bit-exact with phases against the CPU oracle."""
import zlib

import numpy as np
import pytest

import oracle
from test_gpu_tableau import dev_random_destabilizer, _random_paulis  # noqa: E402
from qcb200.tableau import Tableau

pytestmark = pytest.mark.gpu

KINDS = ["Stabilizer", "MixedStabilizer", "Destabilizer", "MixedDestabilizer"]


def make_state(qcb, kind, d, n, rank):
    """The state of `kind` built from a random full destabilizer d; the mixed
    kinds get rank `rank` (MixedStabilizer keeps n rows, zero past the rank)."""
    if kind == "Stabilizer":
        tab = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
        return qcb.Stabilizer(tab.copy()), tab, 0
    if kind == "MixedStabilizer":
        tab = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
        tab.xzs[rank:] = 0
        tab.phases[rank:] = 0
        return qcb.MixedStabilizer(tab.copy(), rank), tab, rank
    if kind == "Destabilizer":
        return qcb.Destabilizer(d.tab.copy()), d.tab.copy(), 0
    return qcb.MixedDestabilizer(d.tab.copy(), rank), d.tab.copy(), rank


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [1, 5, 64, 65, 200, 1000])
@pytest.mark.parametrize("phases", [True, False])
def test_canonicalize_every_state_kind(qcb, kind, n, phases):
    rng = np.random.default_rng(zlib.crc32(f"canon{kind}{n}{phases}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    rank = max(1, (2 * n) // 3)
    st, tab, rank = make_state(qcb, kind, d, n, rank)
    st.to_gpu()
    _, rx, rz = qcb.canonicalize_(st, phases=phases, ranks=True)
    st.to_cpu()
    ph, xz, orx, orz = oracle.canonicalize_state(kind, tab.phases, tab.xzs, n, rank, phases)
    assert (rx, rz) == (orx, orz)
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


@pytest.mark.parametrize("kind", ["Destabilizer", "MixedDestabilizer"])
def test_canonicalize_tall_destabilizer_global_rows(qcb, kind):
    # n = 4000: the stabilizer and destabilizer rows no longer fit the
    # cluster's shared memory and stay in global memory
    n = 4000
    rng = np.random.default_rng(44)
    d = dev_random_destabilizer(qcb, n, rng, depth=6)
    st, tab, rank = make_state(qcb, kind, d, n, n - 7)
    st.to_gpu()
    qcb.canonicalize_(st)
    st.to_cpu()
    ph, xz, _, _ = oracle.canonicalize_state(kind, tab.phases, tab.xzs, n, rank, True)
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [1, 7, 64, 65, 300])
@pytest.mark.parametrize("phases", [True, False])
def test_canonicalize_rref(qcb, kind, n, phases):
    rng = np.random.default_rng(zlib.crc32(f"rref{kind}{n}{phases}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    for cols in (None, list(rng.permutation(n)[: max(1, n // 3)] + 1), [1] + list(range(n, 0, -2))):
        st, tab, rank = make_state(qcb, kind, d, n, max(1, n // 2))
        st.to_gpu()
        _, i = qcb.canonicalize_rref_(st, cols, phases=phases)
        st.to_cpu()
        c = np.arange(1, n + 1) if cols is None else np.asarray(cols)
        ph, xz, oi = oracle.canonicalize_rref(kind, tab.phases, tab.xzs, n, c, rank, phases)
        assert i == oi
        assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


@pytest.mark.parametrize("n", [1, 2, 10, 63, 64, 65, 300, 1000])
@pytest.mark.parametrize("phases", [True, False])
def test_canonicalize_gott(qcb, n, phases):
    rng = np.random.default_rng(zlib.crc32(f"gott{n}{phases}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    for rows in sorted({n, max(1, n // 3), max(1, 2 * n // 3)}):
        tab = Tableau(d.tab.phases[n:n + rows].copy(), n, d.tab.xzs[n:n + rows].copy())
        st = qcb.Stabilizer(tab.copy()).to_gpu()
        _, r, s, xp, zp = qcb.canonicalize_gott_(st, phases=phases)
        st.to_cpu()
        ph, xz, orr, os_, oxp, ozp = oracle.canonicalize_gott(tab.phases, tab.xzs, n, phases)
        assert (r, s) == (orr, os_)
        assert list(xp) == list(oxp) and list(zp) == list(ozp)
        assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


@pytest.mark.parametrize("n", [1, 3, 64, 65, 129, 1000])
def test_permutesystems(qcb, n):
    rng = np.random.default_rng(n)
    t = Tableau.from_bits(rng.integers(0, 4, 9), rng.random((9, n)) < 0.5, rng.random((9, n)) < 0.5)
    perm = rng.permutation(n) + 1
    g = qcb.Stabilizer(t.copy()).to_gpu()
    qcb.permutesystems_(g, perm)
    g.to_cpu()
    assert np.array_equal(g.tab.xzs, oracle.permutesystems(t.xzs, n, perm))
    assert np.array_equal(g.tab.phases, t.phases)
    with pytest.raises(qcb.QCBError):
        bad = perm.copy()
        bad[0] = bad[-1]
        qcb.permutesystems_(g, bad) if n > 1 else qcb.permutesystems_(g, [2])


def oracle_project_qubits(kind, tab, n, rank, qubits, basis, keep_result=True, phases=True):
    ph, xz = tab.phases.copy(), tab.xzs.copy()
    W = xz.shape[1]
    outs = []
    for q in qubits:
        if kind == "MixedDestabilizer":
            ph, xz, rank, a, r = oracle.project_cond(ph, xz, n, rank, q, basis, keep_result, phases)
        else:
            p = np.zeros(W, np.uint64)
            if basis & 1:
                p[(q - 1) >> 6] |= np.uint64(1) << np.uint64((q - 1) & 63)
            if basis & 2:
                p[W // 2 + ((q - 1) >> 6)] |= np.uint64(1) << np.uint64((q - 1) & 63)
            st, ph, xz, rank, a, r = oracle.project(kind, ph, xz, n, p, 0, rank, keep_result, phases)
            assert st == 0
        outs.append((a, None if r < 0 else r))
    return ph, xz, rank, outs


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [1, 5, 64, 65, 300])
@pytest.mark.parametrize("basis", ["X", "Y", "Z"])
def test_project_single_qubit(qcb, kind, n, basis):
    rng = np.random.default_rng(zlib.crc32(f"pq{kind}{n}{basis}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    st, tab, rank = make_state(qcb, kind, d, n, max(0, n // 2) if kind == "MixedDestabilizer" else max(1, n // 2))
    qubits = [int(q) for q in rng.integers(1, n + 1, size=25)]
    st.to_gpu()
    fn = {"X": qcb.projectX_, "Y": qcb.projectY_, "Z": qcb.projectZ_}[basis]
    _, anti, res = fn(st, qubits)
    st.to_cpu()
    ph, xz, orank, outs = oracle_project_qubits(kind, tab, n, rank, qubits, {"X": 1, "Z": 2, "Y": 3}[basis])
    assert list(zip(anti, res)) == outs
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)
    if kind.startswith("Mixed"):
        assert st.rank == orank


def test_project_single_qubit_flags(qcb):
    n = 40
    rng = np.random.default_rng(3)
    d = dev_random_destabilizer(qcb, n, rng)
    for kr, phs in ((False, True), (True, False), (False, False)):
        st, tab, rank = make_state(qcb, "MixedDestabilizer", d, n, 17)
        qubits = [int(q) for q in rng.integers(1, n + 1, size=30)]
        st.to_gpu()
        _, anti, res = qcb.projectY_(st, qubits, keep_result=kr, phases=phs)
        st.to_cpu()
        ph, xz, orank, outs = oracle_project_qubits("MixedDestabilizer", tab, n, rank, qubits, 3, kr, phs)
        assert list(zip(anti, res)) == outs and st.rank == orank
        assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


def test_project_single_qubit_known_answers(qcb):
    # test/test_projections.jl:349-370 on S"XII -IZI IIY" (destabilizers Z1, X2, Z3)
    for basis, q, want in [("X", 1, 0), ("Z", 2, 2), ("Y", 3, 0)]:
        st = qcb.MixedDestabilizer(qcb.T("+Z__ +_X_ +__Z +X__ -_Z_ +__Y"), 3).to_gpu()
        fn = {"X": qcb.projectX_, "Y": qcb.projectY_, "Z": qcb.projectZ_}[basis]
        _, a, r = fn(st, q)
        assert (a, r) == (0, want)


@pytest.mark.parametrize("kind", ["Stabilizer", "MixedStabilizer", "MixedDestabilizer"])
def test_projectrand(qcb, kind):
    n = 70
    rng = np.random.default_rng(zlib.crc32(kind.encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    st, tab, rank = make_state(qcb, kind, d, n, 30)
    qubits = [int(q) for q in rng.integers(1, n + 1, size=20)]
    st.to_gpu()
    _, res = qcb.projectZrand_(st, qubits, rng=np.random.default_rng(11))
    st.to_cpu()
    rp = 2 * np.random.default_rng(11).integers(0, 2, size=len(qubits))
    # the sequence, one projection at a time, with the same random signs
    ph, xz = tab.phases.copy(), tab.xzs.copy()
    off = n if kind == "MixedDestabilizer" else 0
    want = []
    for j, q in enumerate(qubits):
        ph, xz, rank, outs = oracle_project_qubits(kind, Tableau(ph, n, xz), n, rank, [q], 2)
        a, r = outs[0]
        if r is None:
            ph[off + a - 1] = rp[j]
            r = int(rp[j])
        want.append(r)
    assert res == want
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


def test_projectrand_paulis(qcb):
    n = 50
    rng = np.random.default_rng(12)
    d = dev_random_destabilizer(qcb, n, rng)
    st, tab, rank = make_state(qcb, "MixedDestabilizer", d, n, 20)
    paulis = _random_paulis(15, n, rng)
    st.to_gpu()
    _, res = qcb.projectrand_(st, paulis.copy().to_gpu(), rng=np.random.default_rng(5))
    st.to_cpu()
    rp = 2 * np.random.default_rng(5).integers(0, 2, size=15)
    ph, xz = tab.phases.copy(), tab.xzs.copy()
    want = []
    for j in range(15):
        s_, ph, xz, rank, a, r = oracle.project("MixedDestabilizer", ph, xz, n, paulis.xzs[j], paulis.phases[j], rank)
        if r < 0:
            ph[n + a - 1] = rp[j]
            r = int(rp[j])
        want.append(r)
    assert res == want and st.rank == rank
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


@pytest.mark.parametrize("kind", ["Destabilizer", "MixedDestabilizer"])
def test_project_large_tableau_global_rows(qcb, kind):
    # n = 3000: 6000 rows do not fit the cluster's shared memory, so the
    # projections run with the rows in global memory
    n = 3000
    rng = np.random.default_rng(77)
    d = dev_random_destabilizer(qcb, n, rng, depth=5)
    st, tab, rank = make_state(qcb, kind, d, n, n - 5)
    paulis = _random_paulis(6, n, rng)
    paulis.xzs[2] = d.tab.xzs[n + 3]  # a stabilizer row: the commuting branch
    st.to_gpu()
    _, anti, res = qcb.project_(st, paulis.copy().to_gpu())
    st.to_cpu()
    ph, xz = tab.phases.copy(), tab.xzs.copy()
    outs = []
    for j in range(6):
        s_, ph, xz, rank, a, r = oracle.project(kind, ph, xz, n, paulis.xzs[j], paulis.phases[j], rank)
        outs.append((a, None if r < 0 else r))
    assert list(zip(anti, res)) == outs
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 127, 128, 129, 300, 1000])
@pytest.mark.parametrize("phases", [True, False])
def test_canonicalize_by_panels_equals_column_steps(qcb, n, phases):
    # the 64-column panel kernel and the column-by-column kernel on the same
    # inputs, both against the oracle: full-rank, half-rank, redundant rows,
    # and rows that do not commute (random bits; the phases still follow the
    # reference's multiplication order)
    rng = np.random.default_rng(zlib.crc32(f"panel{n}{phases}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    stab = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
    cases = []
    for rows in sorted({n, max(1, n // 2), n + 3}):
        t = Tableau.zeros(rows, n)
        k = min(rows, n)
        t.phases[:k], t.xzs[:k] = stab.phases[:k], stab.xzs[:k]
        for r in range(n, rows):
            t.xzs[r] = t.xzs[r - n] ^ t.xzs[(r - n + 1) % n]
        cases.append(t)
    cases.append(Tableau.from_bits(rng.integers(0, 4, n + 5), rng.random((n + 5, n)) < 0.5, rng.random((n + 5, n)) < 0.5))
    try:
        for t in cases:
            ph, xz, orx, orz = oracle.canonicalize(t.phases, t.xzs, n, phases)
            for mode in (1, 2):
                qcb.check(qcb.lib().qcb_tune_set(b"canon_blocked", mode))
                s = qcb.Stabilizer(t.copy()).to_gpu()
                _, rx, rz = qcb.canonicalize_(s, phases=phases, ranks=True)
                s.to_cpu()
                assert (rx, rz) == (orx, orz), mode
                assert np.array_equal(s.tab.xzs, xz) and np.array_equal(s.tab.phases, ph), mode
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"canon_blocked", 0))


def test_canonicalize_by_panels_tall(qcb):
    # n = 4000: the panel kernel with the rows in global memory
    n = 4000
    rng = np.random.default_rng(4000)
    d = dev_random_destabilizer(qcb, n, rng, depth=6)
    t = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
    s = qcb.Stabilizer(t.copy()).to_gpu()
    _, rx, rz = qcb.canonicalize_(s, ranks=True)
    s.to_cpu()
    ph, xz, orx, orz = oracle.canonicalize(t.phases, t.xzs, n, True)
    assert (rx, rz) == (orx, orz)
    assert np.array_equal(s.tab.xzs, xz) and np.array_equal(s.tab.phases, ph)


def oracle_expect(kind, tab, n, p_xz, p_ph, rank=0):
    st, _, _, _, a, r = oracle.project(kind, tab.phases, tab.xzs, n, p_xz, p_ph, rank)
    assert st == 0
    return {-1: 0, 0: 1, 1: 1j, 2: -1, 3: -1j}[r]


def test_expect_known_answers_on_device(qcb):
    # test/test_expect.jl:33-40 (bell() with sX(2): +XX, -ZZ)
    st = qcb.S("+XX -ZZ").to_gpu()
    for pauli, want in [("XX", 1), ("ZZ", -1), ("XI", 0), ("ZI", 0), ("II", 1), ("-XX", -1), ("-iXX", -1j)]:
        assert qcb.expect(qcb.P(pauli), st) == want, pauli


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [1, 5, 64, 65, 300, 1000])
def test_expect_many_paulis(qcb, kind, n):
    # random Paulis (mostly 0) and group elements (products of stabilizer rows
    # with extra signs and factors of i): each against project! on a copy
    rng = np.random.default_rng(zlib.crc32(f"expect{kind}{n}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    st, tab, rank = make_state(qcb, kind, d, n, max(1, (2 * n) // 3))
    k = 48
    paulis = _random_paulis(k, n, rng)
    off = n if "Destabilizer" in kind else 0
    r = rank if kind.startswith("Mixed") else n
    for j in range(0, k, 2):
        acc, ph = np.zeros(tab.xzs.shape[1], np.uint64), 0
        for i in np.nonzero(rng.random(r) < 0.5)[0]:
            acc, ph = oracle.mul_left_pauli(acc, ph, tab.xzs[off + i], tab.phases[off + i])
        paulis.xzs[j] = acc
        paulis.phases[j] = (ph + int(rng.integers(0, 4))) & 3
    st.to_gpu()
    got = qcb.expect(paulis.copy().to_gpu(), st)
    st.to_cpu()
    assert np.array_equal(st.tab.xzs, tab.xzs) and np.array_equal(st.tab.phases, tab.phases)  # not modified
    want = [oracle_expect(kind, tab, n, paulis.xzs[j], paulis.phases[j], rank) for j in range(k)]
    assert got == want
    assert any(v != 0 for v in want)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("phases", [True, False])
def test_rowswap(qcb, kind, phases):
    # rowswap!(state, i, j; phases) (src/QuantumClifford.jl:899-927)
    n = 70
    rng = np.random.default_rng(zlib.crc32(f"swap{kind}{phases}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    st, tab, rank = make_state(qcb, kind, d, n, 40)
    st.to_gpu()
    want_x, want_p = tab.xzs.copy(), tab.phases.copy()
    off = n if "Destabilizer" in kind else 0
    for i, j in [(1, 2), (5, 40), (40, 5), (7, 7)]:
        qcb.rowswap_(st, i, j, phases=phases)
        rows = [(off + i - 1, off + j - 1)] + ([(i - 1, j - 1)] if off else [])
        for a, b in rows:
            want_x[[a, b]] = want_x[[b, a]]
            if phases:
                want_p[[a, b]] = want_p[[b, a]]
    st.to_cpu()
    assert np.array_equal(st.tab.xzs, want_x) and np.array_equal(st.tab.phases, want_p)
