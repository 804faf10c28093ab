"""Uniform random Cliffords (qcb200.randoms, Bravyi-Maslov Algorithm 2, the
method of src/randoms.jl:155-230): every sample is a valid destabilizer
tableau (symplectic: destabilizer i anticommutes with stabilizer i only),
and the symplectic part is uniform over Sp(2,2) (6 elements) and Sp(4,2)
(720 elements), checked by a chi-square test."""
import numpy as np
import pytest

from qcb200 import randoms


def symplectic_form(xzs, n):
    x, z = xzs[:, :n].astype(np.int64), xzs[:, n:].astype(np.int64)
    return (x @ z.T + z @ x.T) & 1


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 65, 200])
def test_random_destabilizer_is_symplectic(n):
    rng = np.random.default_rng(n)
    for _ in range(3 if n > 60 else 20):
        ph, xzs = randoms.random_destabilizer_bits(n, rng)
        omega = np.zeros((2 * n, 2 * n), np.int64)
        omega[:n, n:] = np.eye(n, dtype=np.int64)
        omega[n:, :n] = np.eye(n, dtype=np.int64)
        assert np.array_equal(symplectic_form(xzs, n), omega)
        assert set(np.unique(ph)) <= {0, 2}


@pytest.mark.parametrize("n,order,samples", [(1, 6, 6000), (2, 720, 36000)])
def test_symplectic_part_is_uniform(n, order, samples):
    rng = np.random.default_rng(100 + n)
    counts = {}
    for _ in range(samples):
        _, xzs = randoms.random_destabilizer_bits(n, rng, phases=False)
        k = xzs.tobytes()
        counts[k] = counts.get(k, 0) + 1
    assert len(counts) == order
    exp = samples / order
    chi2 = sum((c - exp) ** 2 / exp for c in counts.values())
    dof = order - 1
    # 5-sigma bound of the chi-square statistic (mean dof, variance 2 dof)
    assert chi2 < dof + 5 * np.sqrt(2 * dof), chi2


def test_random_stabilizer_shape_and_layout():
    rng = np.random.default_rng(5)
    s = randoms.random_stabilizer(130, rng)
    assert len(s.tab) == 130 and s.tab.nqubits == 130
    d = randoms.random_destabilizer(130, np.random.default_rng(5))
    assert np.array_equal(d.tab.xzs[130:], s.tab.xzs) and np.array_equal(d.tab.phases[130:], s.tab.phases)
    # padding bits past qubit 130 are zero (src/randoms.jl:13-24 keeps them clear)
    assert not (s.tab.xzs[:, 2] >> np.uint64(2)).any() and not (s.tab.xzs[:, 5] >> np.uint64(2)).any()
