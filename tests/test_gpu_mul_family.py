"""The mul_left!/mul_right! family on the device (qcb_mul_rows,
qcb_mul_left_state) against the oracle, bit for bit with phases: every form
of src/mul_leftright.jl:137-245 and of the KA extension's device methods
(ext/QuantumCliffordKAExt/mul_leftright.jl:101-460), at word-boundary sizes
and one long row."""
import numpy as np
import pytest

import oracle
import qcb200
from qcb200.tableau import PauliOperator, Tableau

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 10, 63, 64, 65, 127, 128, 129, 1000]


def rand_tab(rows, n, rng):
    return Tableau.from_bits(rng.integers(0, 4, rows), rng.random((rows, n)) < 0.5, rng.random((rows, n)) < 0.5)


def pauli(t):
    return PauliOperator(t.phases.copy(), t.nqubits, t.xzs.copy())


def got(x):
    x.to_cpu()
    t = x.tab if isinstance(x, qcb200.Stabilizer) else x
    return t.phases.copy(), t.xzs.copy()


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("right", [False, True])
@pytest.mark.parametrize("phases", [True, False])
def test_pauli_and_row_forms(qcb, n, right, phases):
    rng = np.random.default_rng(n * 4 + right * 2 + phases)
    f = qcb.mul_right_ if right else qcb.mul_left_
    s, p, q = rand_tab(9, n, rng), rand_tab(1, n, rng), rand_tab(1, n, rng)
    # PauliOperator with PauliOperator
    a = pauli(p).to_gpu()
    f(a, pauli(q).to_gpu(), phases=phases)
    assert all(np.array_equal(x, y) for x, y in zip(got(a), oracle.mul_rows(p.phases, p.xzs, q.phases, q.xzs, 1, 1, 1, 0,
                                                                             right, 0, phases)))
    # PauliOperator with row i of a Tableau
    a = pauli(p).to_gpu()
    f(a, s.copy().to_gpu(), 6, phases=phases)
    assert all(np.array_equal(x, y) for x, y in zip(got(a), oracle.mul_rows(p.phases, p.xzs, s.phases, s.xzs, 1, 1, 6, 0,
                                                                             right, 0, phases)))
    # every row of a Stabilizer with a PauliOperator
    st = qcb.Stabilizer(s.copy()).to_gpu()
    f(st, pauli(q).to_gpu(), phases=phases)
    assert all(np.array_equal(x, y) for x, y in zip(got(st), oracle.mul_rows(s.phases, s.xzs, q.phases, q.xzs, 1, 9, 1, 0,
                                                                              right, 0, phases)))
    # rows m, i of one tableau
    t = s.copy().to_gpu()
    f(t, 3, 8, phases=phases)
    assert all(np.array_equal(x, y) for x, y in zip(got(t), oracle.mul_rows(s.phases, s.xzs, None, None, 3, 1, 8, 0,
                                                                             right, 0, phases)))
    # cross-tableau mul_left!(s, m, t, i) with the reference's s.phases[i]
    u = rand_tab(9, n, rng)
    t = s.copy().to_gpu()
    f(t, 2, u.copy().to_gpu(), 7, phases=phases)
    assert all(np.array_equal(x, y) for x, y in zip(got(t), oracle.mul_rows(s.phases, s.xzs, u.phases, u.xzs, 2, 1, 7, 0,
                                                                             right, 1, phases)))


@pytest.mark.parametrize("kind", ["Destabilizer", "MixedDestabilizer", "Stabilizer", "MixedStabilizer"])
@pytest.mark.parametrize("n", [5, 64, 200])
def test_mul_left_on_states(qcb, kind, n):
    """mul_left!(state, i, j) (src/mul_leftright.jl:194-219): the Destabilizer
    kinds update destabilizer j by destabilizer i (no phase) and stabilizer i
    by stabilizer j."""
    rng = np.random.default_rng(n)
    rows = 2 * n if "Destabilizer" in kind else n
    s = rand_tab(rows, n, rng)
    cls = getattr(qcb, kind)
    st = cls(s.copy(), n // 2 if kind.startswith("Mixed") else None).to_gpu()
    qcb.mul_left_(st, 2, n - 1)
    ph, xz = got(st)
    if "Destabilizer" in kind:
        w_ph, w_xz = oracle.mul_rows(s.phases, s.xzs, None, None, n - 1, 1, 2, 0, phases=False)
        w_ph, w_xz = oracle.mul_rows(w_ph, w_xz, None, None, n + 2, 1, 2 * n - 1, 0)
    else:
        w_ph, w_xz = oracle.mul_rows(s.phases, s.xzs, None, None, 2, 1, n - 1, 0)
    assert np.array_equal(xz, w_xz) and np.array_equal(ph, w_ph)


@pytest.mark.parametrize("right", [False, True])
def test_long_row_products(qcb, right):
    """3e7-qubit rows: the grid-stride path with 128-bit loads (even word
    count) and 64-bit loads (odd)."""
    rng = np.random.default_rng(9)
    for n in (30_000_000, 30_000_050):  # even and odd word counts
        W = 2 * ((n + 63) // 64)
        s = Tableau(rng.integers(0, 4, 2).astype(np.uint8), n, rng.integers(0, 2**63, size=(2, W), dtype=np.uint64))
        xs, zs = s.xzs[:, :W // 2], s.xzs[:, W // 2:]
        if n % 64:
            xs[:, -1] &= np.uint64((1 << (n % 64)) - 1)
            zs[:, -1] &= np.uint64((1 << (n % 64)) - 1)
        t = s.copy().to_gpu()
        (qcb.mul_right_ if right else qcb.mul_left_)(t, 1, 2)
        ph, xz = got(t)
        w_ph, w_xz = oracle.mul_rows(s.phases, s.xzs, None, None, 1, 1, 2, 0, right)
        assert np.array_equal(xz, w_xz) and np.array_equal(ph, w_ph)


def test_errors(qcb):
    rng = np.random.default_rng(1)
    a = pauli(rand_tab(1, 10, rng)).to_gpu()
    b = pauli(rand_tab(1, 11, rng)).to_gpu()
    with pytest.raises(qcb.DimensionMismatch):
        qcb.mul_right_(a, b)
    s = rand_tab(4, 10, rng).to_gpu()
    with pytest.raises(qcb.BoundsError):
        qcb.mul_left_(s, 5, 1)
