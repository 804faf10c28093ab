"""GPU parity tests for the tableau kernels (through the C ABI), bit-exact
with phases against the CPU oracle."""
import zlib

import numpy as np
import pytest

import oracle
from test_gpu_frames import random_sqo  # noqa: E402
import qcb200
from qcb200 import ops as O
from qcb200.tableau import Tableau, one_destabilizer, random_clifford_ops

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 10, 63, 64, 65, 127, 128, 129]


def rand_tab(rows, n, rng):
    t = Tableau.from_bits(rng.integers(0, 4, rows), rng.random((rows, n)) < 0.5, rng.random((rows, n)) < 0.5)
    return t


def dev_random_destabilizer(qcb, n, rng, depth=None):
    """A random full-rank destabilizer: a random H/S/CNOT circuit applied on
    the device to one(Destabilizer, n) (the gate kernel is itself checked
    against the oracle below)."""
    d = one_destabilizer(n)
    d.to_gpu()
    ops = random_clifford_ops(n, depth or (2 * int(np.log2(max(n, 2))) + 8), rng)
    qcb.apply_(d, ops)
    d.to_cpu()
    return d


@pytest.mark.parametrize("n", SIZES + [1000, 100_000])
@pytest.mark.parametrize("phases", [True, False])
def test_mul_left_pauli(qcb, n, phases):
    rng = np.random.default_rng(n)
    for _ in range(3):
        a, b = rand_tab(1, n, rng), rand_tab(1, n, rng)
        ra = qcb.PauliOperator(b.phases.copy(), n, b.xzs.copy()).to_gpu()
        la = qcb.PauliOperator(a.phases.copy(), n, a.xzs.copy()).to_gpu()
        qcb.mul_left_(ra, la, phases=phases)
        ra.to_cpu()
        r, ph = oracle.mul_left_pauli(b.xzs[0], b.phases[0], a.xzs[0], a.phases[0], phases)
        assert np.array_equal(ra.xzs[0], r)
        assert ra.phases[0] == (ph if phases else b.phases[0])


def test_mul_left_pauli_large(qcb):
    n = 50_000_000
    rng = np.random.default_rng(5)
    W = 2 * ((n + 63) // 64)
    a = rng.integers(0, 2**63, size=(1, W), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=(1, W), dtype=np.uint64)
    b = rng.integers(0, 2**63, size=(1, W), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=(1, W), dtype=np.uint64)
    ra = qcb.PauliOperator(np.array([1], np.uint8), n, b.copy()).to_gpu()
    la = qcb.PauliOperator(np.array([2], np.uint8), n, a.copy()).to_gpu()
    qcb.mul_left_(ra, la)
    ra.to_cpu()
    r, ph = oracle.mul_left_pauli(b[0], 1, a[0], 2)
    assert ra.phases[0] == ph and np.array_equal(ra.xzs[0], r)


@pytest.mark.parametrize("n", [5, 64, 130])
def test_row_ops_prodphase_comm(qcb, n):
    rng = np.random.default_rng(n)
    t = rand_tab(6, n, rng)
    g = t.copy().to_gpu()
    qcb.mul_left_row_(g, 2, 5)
    g.to_cpu()
    ph, xz = t.phases.copy(), t.xzs.copy()
    oracle.L().oracle_mul_left_row(xz.ctypes.data, ph.ctypes.data, xz.shape[1], 2, 5, 1)
    assert np.array_equal(g.xzs, xz) and np.array_equal(g.phases, ph)
    p = rand_tab(1, n, rng)
    pg = qcb.PauliOperator(p.phases, n, p.xzs).to_gpu()
    g2 = t.copy().to_gpu()
    qcb.check(qcb.lib().qcb_mul_left_tableau_pauli(g2.dev.handle, pg.dev.handle, 1, None))
    g2.to_cpu()
    ph, xz = t.phases.copy(), t.xzs.copy()
    oracle.L().oracle_mul_left_tableau_pauli(xz.ctypes.data, ph.ctypes.data, 6, xz.shape[1], p.xzs.ctypes.data,
                                             int(p.phases[0]), 1)
    assert np.array_equal(g2.xzs, xz) and np.array_equal(g2.phases, ph)
    tg = t.copy().to_gpu()
    for i in range(1, 7):
        assert qcb.prodphase(pg, tg, 1, i) == oracle.prodphase(p.xzs[0], p.phases[0], t.xzs[i - 1], t.phases[i - 1])
        assert qcb.comm(pg, tg, 1, i) == oracle.comm(p.xzs[0], t.xzs[i - 1])


@pytest.mark.parametrize("n", [3, 70, 200])
def test_symbolic_gates_with_phases(qcb, n):
    rng = np.random.default_rng(n)
    t = rand_tab(2 * n, n, rng)
    gates = []
    g1 = ["I", "H", "S", "SDAG", "X", "Y", "Z", "SQRTX", "INVSQRTX", "SQRTY", "INVSQRTY", "HXY", "HYZ", "CXYZ", "CZYX"]
    g2 = ["CNOT", "CPHASE", "SWAP", "ZCX", "ZCY", "ZCZ", "XCX", "XCY", "XCZ", "YCX", "YCY", "YCZ",
          "SWAPCX", "INVSWAPCX", "ISWAP", "INVISWAP", "CZSWAP", "CXSWAP", "ZCRY", "INVZCRY", "SQRTZZ", "INVSQRTZZ",
          "SQRTXX", "INVSQRTXX", "SQRTYY", "INVSQRTYY"]
    for _ in range(300):
        u = rng.random()
        if u < 0.15:
            gates.append(random_sqo(int(rng.integers(1, n + 1)), rng))
        elif u < 0.5:
            gates.append(O.Op(O.OP[g1[rng.integers(len(g1))]], int(rng.integers(1, n + 1))))
        else:
            a, b = rng.choice(np.arange(1, n + 1), 2, replace=False)
            gates.append(O.Op(O.OP[g2[rng.integers(len(g2))]], int(a), int(b)))
    arr = O.to_array(gates)
    for phases in (True, False):
        g = t.copy().to_gpu()
        qcb.apply_(g, arr, phases=phases)
        g.to_cpu()
        ph, xz = oracle.apply_gates(t.phases, t.xzs, n, arr, phases)
        assert np.array_equal(g.xzs, xz) and np.array_equal(g.phases, ph)


@pytest.mark.parametrize("n", SIZES + [300, 1000])
@pytest.mark.parametrize("phases", [True, False])
def test_canonicalize_random_stabilizers(qcb, n, phases):
    rng = np.random.default_rng(1000 + n)
    d = dev_random_destabilizer(qcb, n, rng)
    stab = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
    for rows in sorted({n, max(1, n // 2), n + 3}):
        t = Tableau.zeros(rows, n)
        k = min(rows, n)
        t.phases[:k], t.xzs[:k] = stab.phases[:k], stab.xzs[:k]
        for r in range(n, rows):
            t.xzs[r] = t.xzs[r - n] ^ t.xzs[(r - n + 1) % n]
        s = qcb.Stabilizer(t.copy()).to_gpu()
        _, rx, rz = qcb.canonicalize_(s, phases=phases, ranks=True)
        s.to_cpu()
        ph, xz, orx, orz = oracle.canonicalize(t.phases, t.xzs, n, phases)
        assert (rx, rz) == (orx, orz)
        assert np.array_equal(s.tab.xzs, xz)
        assert np.array_equal(s.tab.phases, ph)


@pytest.mark.parametrize("n", [2000, 4000])
def test_canonicalize_benchmark_sizes(qcb, n):
    rng = np.random.default_rng(n)
    d = dev_random_destabilizer(qcb, n, rng)
    t = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
    s = qcb.Stabilizer(t.copy()).to_gpu()
    _, rx, rz = qcb.canonicalize_(s, ranks=True)
    s.to_cpu()
    ph, xz, orx, orz = oracle.canonicalize(t.phases, t.xzs, n, True)
    assert (rx, rz) == (orx, orz) == (rx, n)
    assert np.array_equal(s.tab.xzs, xz) and np.array_equal(s.tab.phases, ph)


def _random_paulis(k, n, rng, weight_uniform=True):
    ps = Tableau.zeros(k, n)
    for j in range(k):
        w = int(rng.integers(1, n + 1)) if weight_uniform else n
        qs = rng.choice(n, w, replace=False)
        kinds = rng.integers(1, 4, w)
        xs = np.zeros((1, n), bool)
        zs = np.zeros((1, n), bool)
        xs[0, qs] = (kinds & 1) > 0
        zs[0, qs] = (kinds & 2) > 0
        one = Tableau.from_bits([int(rng.integers(0, 2)) * 2], xs, zs)
        ps.phases[j], ps.xzs[j] = one.phases[0], one.xzs[0]
    return ps


def oracle_project_seq(kind, tab, paulis, n, rank=0, keep_result=True, phases=True):
    ph, xz = tab.phases.copy(), tab.xzs.copy()
    outs = []
    for j in range(len(paulis)):
        st, ph, xz, rank, a, r = oracle.project(kind, ph, xz, n, paulis.xzs[j], paulis.phases[j], rank,
                                                keep_result, phases)
        assert st == 0
        outs.append((a, None if r < 0 else r))
    return ph, xz, rank, outs


@pytest.mark.parametrize("kind", ["Stabilizer", "Destabilizer", "MixedDestabilizer", "MixedStabilizer"])
@pytest.mark.parametrize("n", [1, 5, 64, 65, 200])
def test_project_sequences(qcb, kind, n):
    rng = np.random.default_rng(zlib.crc32(f"{kind}{n}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    k = 40
    paulis = _random_paulis(k, n, rng)
    # mix in commuting / generated operators: stabilizer rows and their products
    for j in range(0, k, 5):
        paulis.xzs[j] = d.tab.xzs[n + (j % n)]
        paulis.phases[j] = (d.tab.phases[n + (j % n)] + 2 * (j % 2)) & 3
    rank = 0
    if kind == "Stabilizer":
        tab = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
        st = qcb.Stabilizer(tab.copy())
    elif kind == "MixedStabilizer":
        rank = max(1, n // 2)
        tab = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
        tab.xzs[rank:] = 0
        tab.phases[rank:] = 0
        st = qcb.MixedStabilizer(tab.copy(), rank)
    elif kind == "Destabilizer":
        tab = d.tab.copy()
        st = qcb.Destabilizer(tab.copy())
    else:
        rank = max(0, n - 2)
        tab = d.tab.copy()
        st = qcb.MixedDestabilizer(tab.copy(), rank)
    st.to_gpu()
    pg = paulis.copy().to_gpu()
    _, anti, res = qcb.project_(st, pg)
    st.to_cpu()
    ph, xz, orank, outs = oracle_project_seq(kind, tab, paulis, n, rank)
    assert list(zip(anti, res)) == outs
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)
    if kind.startswith("Mixed"):
        assert st.rank == orank


@pytest.mark.parametrize("kind", ["Stabilizer", "MixedStabilizer"])
@pytest.mark.parametrize("n", [5, 64, 200])
@pytest.mark.parametrize("keep_result,phases", [(True, True), (False, True), (True, False)])
def test_project_sequences_whole_gpu(qcb, kind, n, keep_result, phases):
    """project! of generic Paulis on Stabilizer / MixedStabilizer tableaux by
    the whole-GPU kernel (project_grid 1: a cooperative grid, two grid
    barriers per Pauli, the pivot row written one Pauli later), forced on
    small tableaux; sequences mixing anticommuting Paulis with stabilizer
    rows and their products (the commuting branch), bit for bit against the
    oracle."""
    rng = np.random.default_rng(zlib.crc32(f"grid{kind}{n}{keep_result}{phases}".encode()))
    d = dev_random_destabilizer(qcb, n, rng)
    k = 40
    paulis = _random_paulis(k, n, rng)
    for j in range(0, k, 5):
        paulis.xzs[j] = d.tab.xzs[n + (j % n)]
        paulis.phases[j] = (d.tab.phases[n + (j % n)] + 2 * (j % 2)) & 3
    for j in range(3, k, 7):  # the Pauli just projected, again
        paulis.xzs[j], paulis.phases[j] = paulis.xzs[j - 1], paulis.phases[j - 1]
    rank = 0
    tab = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
    if kind == "MixedStabilizer":
        rank = max(1, n // 2)
        tab.xzs[rank:] = 0
        tab.phases[rank:] = 0
        st = qcb.MixedStabilizer(tab.copy(), rank)
    else:
        st = qcb.Stabilizer(tab.copy())
    st.to_gpu()
    qcb.check(qcb.lib().qcb_tune_set(b"project_grid", 1))
    try:
        _, anti, res = qcb.project_(st, paulis.copy().to_gpu(), keep_result=keep_result, phases=phases)
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"project_grid", 0))
    st.to_cpu()
    ph, xz, orank, outs = oracle_project_seq(kind, tab, paulis, n, rank, keep_result, phases)
    assert list(zip(anti, res)) == outs
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)
    if kind == "MixedStabilizer":
        assert st.rank == orank


def test_project_keep_result_false_and_phases_false(qcb):
    n = 50
    rng = np.random.default_rng(8)
    d = dev_random_destabilizer(qcb, n, rng)
    paulis = _random_paulis(20, n, rng)
    for kr, phs in ((False, True), (True, False)):
        for kind in ("Stabilizer", "Destabilizer"):
            tab = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy()) if kind == "Stabilizer" else d.tab.copy()
            st = (qcb.Stabilizer if kind == "Stabilizer" else qcb.Destabilizer)(tab.copy()).to_gpu()
            _, anti, res = qcb.project_(st, paulis.copy().to_gpu(), keep_result=kr, phases=phs)
            st.to_cpu()
            ph, xz, _, outs = oracle_project_seq(kind, tab, paulis, n, 0, kr, phs)
            assert list(zip(anti, res)) == outs
            assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)


def test_project_bad_data_structure(qcb):
    # an incomplete Destabilizer cannot tell stabilized from logical operators
    n = 4
    d = one_destabilizer(n).tab
    t = Tableau(np.concatenate([d.phases[:2], d.phases[n:n + 2]]), n, np.vstack([d.xzs[:2], d.xzs[n:n + 2]]))
    st = qcb.Destabilizer(t).to_gpu()
    with pytest.raises(qcb.BadDataStructure):
        qcb.project_(st, qcb.P("IIZI").to_gpu())


@pytest.mark.parametrize("n", [4, 65, 300])
def test_generate(qcb, n):
    rng = np.random.default_rng(n)
    d = dev_random_destabilizer(qcb, n, rng)
    ph, xz, _, _ = oracle.canonicalize(d.tab.phases[n:], d.tab.xzs[n:], n)
    stab = Tableau(ph, n, xz).to_gpu()
    for j in range(6):
        if j % 2 == 0:  # a product of stabilizer rows: generated
            sel = rng.random(n) < 0.5
            p = Tableau.zeros(1, n)
            phase = 0
            for r in np.nonzero(sel)[0]:
                p.xzs[0], phase = oracle.mul_left_pauli(p.xzs[0], phase, xz[r], ph[r])
            p.phases[0] = phase
        else:
            p = _random_paulis(1, n, rng)
        pp = qcb.PauliOperator(p.phases.copy(), n, p.xzs.copy()).to_gpu()
        out = qcb.generate_(pp, qcb.Stabilizer(stab))
        ok, rest, rph, used = oracle.generate(p.xzs[0], p.phases[0], ph, xz, n)
        assert (out is not None) == ok
        if ok:
            assert out[1] == used and out[0].phases[0] == rph and not out[0].xzs.any()


@pytest.mark.parametrize("n", [2, 64, 129, 600, 1000, 1501, 3000])
def test_dense_apply(qcb, n):
    rng = np.random.default_rng(n)
    d = dev_random_destabilizer(qcb, n, rng)
    state = Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
    state.phases[:] = rng.integers(0, 4, n)
    if n % 2 == 0:
        c = qcb.tensor_pow(qcb.tCNOT(), n // 2)
    else:
        c = qcb.CliffordOperator(dev_random_destabilizer(qcb, n, rng).tab)
        c.tab.phases[:] = rng.integers(0, 4, 2 * n)
        c.to_gpu()  # the device copy must see the new phases
    for phases in (True, False):
        s = qcb.Stabilizer(state.copy()).to_gpu()
        qcb.apply_(s, c, phases=phases)
        s.to_cpu()
        ph, xz = oracle.apply_dense(state.phases, state.xzs, n, c.tab.phases, c.tab.xzs, phases)
        assert np.array_equal(s.tab.xzs, xz) and np.array_equal(s.tab.phases, ph)


def _canonicalize_with(qcb, t, phases, grid, lookahead):
    lib = qcb.lib()
    qcb.check(lib.qcb_tune_set(b"canon_grid", grid))
    qcb.check(lib.qcb_tune_set(b"canon_lookahead", lookahead))
    try:
        s = qcb.Stabilizer(t.copy()).to_gpu()
        _, rx, rz = qcb.canonicalize_(s, phases=phases, ranks=True)
        s.to_cpu()
    finally:
        qcb.check(lib.qcb_tune_set(b"canon_grid", 0))
        qcb.check(lib.qcb_tune_set(b"canon_lookahead", 1))
    return s, rx, rz


# (canon_grid, canon_lookahead): the whole GPU with look-ahead, the whole GPU
# with the search and the apply in turn, one cluster
SCHEDULES = [(1, 1), (1, 0), (2, 1)]


@pytest.mark.parametrize("grid,lookahead", SCHEDULES)
@pytest.mark.parametrize("n", [64, 97, 1000, 2100, 4000])
@pytest.mark.parametrize("phases", [True, False])
def test_canonicalize_panels_over_the_gpu(qcb, n, grid, lookahead, phases):
    """canonicalize! by panels with the per-row work spread over the GPU
    (canon_grid 1: with look-ahead, per panel one launch of the pivot steps
    beside the previous panel's grid-wide apply and one of the pivot rows and
    phase data beside the next panel's words; without, a one-CTA search
    launch and a grid-wide apply launch per panel) and on one cluster (2), on
    uniformly random stabilizer states, bit for bit with phases and ranks
    against the oracle, with phases tracked and not (the row swaps then leave
    the phases in place); also a rank-deficient view (repeated rows)."""
    from qcb200 import randoms

    rng = np.random.default_rng(n + grid)
    t = randoms.random_stabilizer(n, rng).tab
    if n == 97:  # duplicate rows: rank deficiency, columns without a pivot
        t.xzs[50:60] = t.xzs[10:20]
        t.phases[50:60] = t.phases[10:20]
    s, rx, rz = _canonicalize_with(qcb, t, phases, grid, lookahead)
    ph, xz, orx, orz = oracle.canonicalize(t.phases, t.xzs, n, phases)
    assert (rx, rz) == (orx, orz)
    assert np.array_equal(s.tab.xzs, xz) and np.array_equal(s.tab.phases, ph)


@pytest.mark.parametrize("lookahead", [1, 0])
@pytest.mark.parametrize("rows,n", [(300, 1000), (1500, 700), (700, 130), (1200, 1200)])
def test_canonicalize_panels_rectangular_views(qcb, rows, n, lookahead):
    """Views with fewer or more rows than qubits (random rows, commuting or
    not; rank-deficient when rows > 2n or rows repeat): the last pivot comes
    before the last panel, so the remaining panels find every position taken,
    or columns end without a pivot.  Whole-GPU panels with and without
    look-ahead, against the oracle."""
    rng = np.random.default_rng(rows * 7 + n + lookahead)
    t = rand_tab(rows, n, rng)
    if rows == 1200:  # low-weight rows and repeats: many panels without pivots
        t.xzs &= rng.integers(0, 2**63, t.xzs.shape, dtype=np.uint64) & rng.integers(0, 2**63, t.xzs.shape, dtype=np.uint64)
        t.xzs[600:900] = t.xzs[100:400]
    for phases in (True, False):
        s, rx, rz = _canonicalize_with(qcb, t, phases, 1, lookahead)
        ph, xz, orx, orz = oracle.canonicalize(t.phases, t.xzs, n, phases)
        assert (rx, rz) == (orx, orz)
        assert np.array_equal(s.tab.xzs, xz) and np.array_equal(s.tab.phases, ph)
