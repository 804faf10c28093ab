"""project! at the benchmarked tableau configuration: uniformly random
stabilizer states (random_stabilizer(n), Bravyi-Maslov) of n = 1000, 2000
and 4000 qubits, Stabilizer kind (src/project_trace_reset.jl:276-308), 1,000
random Paulis of weight ~ U{1..n}, bit for bit with phases against the
oracle.

  * chain: the 1,000 Paulis projected in order on one state by one call; some
    Paulis repeat the one before (that one is in the stabilizer group after
    its projection), which takes the commuting branch (canonicalize! +
    generate!, a determined result);
  * independent: each Pauli projected on a fresh copy of the state.
"""
import numpy as np
import pytest

import oracle
from qcb200 import randoms
from qcb200.tableau import Tableau

pytestmark = pytest.mark.gpu

K = 1000


def config_inputs(n, seed):
    rng = np.random.default_rng(seed)
    s = randoms.random_stabilizer(n, rng)
    ps = randoms.random_paulis(K, n, rng)
    return s.tab, ps


@pytest.mark.parametrize("n", [1000, 2000, 4000])
def test_project_chain_stabilizer(qcb, n):
    tab, ps = config_inputs(n, 31 + n)
    repeats = list(range(100, K, 100 if n < 4000 else 250))
    for j in repeats:
        ps.xzs[j], ps.phases[j] = ps.xzs[j - 1], ps.phases[j - 1]
    st = qcb.Stabilizer(tab.copy()).to_gpu()
    _, anti, res = qcb.project_(st, ps.copy().to_gpu())
    st.to_cpu()
    ph, xz = tab.phases.copy(), tab.xzs.copy()
    outs = []
    for j in range(K):
        code, ph, xz, _, a, r = oracle.project("Stabilizer", ph, xz, n, ps.xzs[j], ps.phases[j])
        assert code == 0
        outs.append((a, None if r < 0 else r))
    assert list(zip(anti, res)) == outs
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)
    # the repeated Paulis commute with the state and are determined
    assert all(anti[j] == 0 and res[j] is not None for j in repeats)
    assert sum(a != 0 for a in anti) >= K - len(repeats) - 5


@pytest.mark.parametrize("n", [1000, 2000, 4000])
def test_project_independent_stabilizer(qcb, n):
    tab, ps = config_inputs(n, 77 + n)
    pristine = qcb.Stabilizer(tab.copy()).to_gpu()
    work = qcb.Stabilizer(tab.copy()).to_gpu()
    lib = qcb.lib()
    k = 200 if n == 4000 else K
    for j in range(k):
        qcb.check(lib.qcb_tableau_copy(work.tab.dev.handle, pristine.tab.dev.handle, None))
        p = Tableau(ps.phases[j:j + 1].copy(), n, ps.xzs[j:j + 1].copy())
        _, a, r = qcb.project_(work, qcb.PauliOperator(p.phases, n, p.xzs).to_gpu())
        code, ph, xz, _, oa, orr = oracle.project("Stabilizer", tab.phases, tab.xzs, n, ps.xzs[j], ps.phases[j])
        assert (a, r) == (oa, None if orr < 0 else orr), j
        if j % 50 == 0:
            work.to_cpu()
            assert np.array_equal(work.tab.xzs, xz) and np.array_equal(work.tab.phases, ph), j
