"""Uniformly random Clifford operators and stabilizer states (host-side input
generation): random_destabilizer, random_stabilizer, random_clifford
(src/randoms.jl:155-230, 432-443).

Method: Bravyi & Maslov, "Hadamard-free circuits expose the structure of the
Clifford group" (IEEE Trans. Inf. Theory 67, 2021), Algorithm 2.  Every
Clifford is uniquely F1 . H(h) . S(perm) . F2 with F1, F2 Hadamard-free;
(h, perm) is drawn from the quantum Mallows distribution (their Algorithm 1)
and the free bits of F1, F2 uniformly under the uniqueness conditions, which
makes the Clifford uniform (up to the Pauli part, drawn as random row signs
as the reference does).  Written here in GF(2) matrix form: a Hadamard-free
Clifford F(Gamma, Delta) with Delta unit lower triangular and Gamma
symmetric has the symplectic matrix
    [[Delta, 0], [Gamma Delta, Delta^-T]]
acting on tableau rows (destabilizers 1..n, stabilizers n+1..2n; columns x
bits then z bits).  Products are exact float32 BLAS products reduced mod 2
(sums stay below 2^24 for n < 8 * 10^6).
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .tableau import CliffordOperator, Destabilizer, Stabilizer, Tableau


def quantum_mallows(n: int, rng: np.random.Generator):
    """(h, perm) from the quantum Mallows distribution (Bravyi-Maslov
    Algorithm 1): at step i, with m = n - i qubits left, a weight w in
    0..2m-1 with probability proportional to 2^-w; h_i = (w < m); the
    permutation takes the k-th remaining qubit, k = w if w < m else 2m-1-w."""
    left = list(range(n))
    h = np.zeros(n, dtype=bool)
    perm = np.zeros(n, dtype=np.int64)
    for i in range(n):
        m = n - i
        while True:  # truncated geometric(1/2), starting at 0
            w = int(rng.geometric(0.5)) - 1
            if w < 2 * m:
                break
        h[i] = w < m
        perm[i] = left.pop(w if w < m else 2 * m - 1 - w)
    return h, perm


def _mm2(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """GF(2) product of 0/1 matrices: an exact floating-point product reduced
    mod 2 (float64 on a CUDA device when one is present and the product is
    large -- input generation only -- else float32 BLAS on the host)."""
    if min(a.shape[0], b.shape[1]) >= 256 and _torch_cuda():
        import torch

        ta = torch.from_numpy(np.ascontiguousarray(a)).to("cuda", torch.float64)
        tb = torch.from_numpy(np.ascontiguousarray(b)).to("cuda", torch.float64)
        return (torch.matmul(ta, tb).to(torch.int64) & 1).to(torch.uint8).cpu().numpy()
    return (np.matmul(a.astype(np.float32), b.astype(np.float32)).astype(np.int64) & 1).astype(np.uint8)


_TORCH_CUDA = None


def _torch_cuda() -> bool:
    global _TORCH_CUDA
    if _TORCH_CUDA is None:
        try:
            import torch

            _TORCH_CUDA = bool(torch.cuda.is_available())
        except ImportError:
            _TORCH_CUDA = False
    return _TORCH_CUDA


def _unit_lower_inverse(low: np.ndarray) -> np.ndarray:
    """Inverse over GF(2) of a unit lower-triangular 0/1 matrix: by blocks,
    [[A, 0], [C, D]]^-1 = [[A^-1, 0], [D^-1 C A^-1, D^-1]] (signs vanish mod
    2), down to blocks of 128 rows done by forward substitution."""
    n = low.shape[0]
    if n > 128:
        h = n // 2
        ai = _unit_lower_inverse(low[:h, :h])
        di = _unit_lower_inverse(low[h:, h:])
        out = np.zeros((n, n), dtype=np.uint8)
        out[:h, :h] = ai
        out[h:, h:] = di
        out[h:, :h] = _mm2(_mm2(di, low[h:, :h]), ai)
        return out
    return _unit_lower_inverse_rows(low)


def _unit_lower_inverse_rows(low: np.ndarray) -> np.ndarray:
    """Forward substitution on bit-packed rows: row i of the inverse is e_i
    XOR the inverse rows j < i with low[i, j] = 1."""
    n = low.shape[0]
    words = (n + 63) // 64
    inv = np.zeros((n, words), dtype=np.uint64)
    for i in range(n):
        sel = np.flatnonzero(low[i, :i])
        if len(sel):
            inv[i] = np.bitwise_xor.reduce(inv[sel], axis=0)
        inv[i, i >> 6] ^= np.uint64(1 << (i & 63))
    bits = np.unpackbits(inv.view(np.uint8), axis=1, bitorder="little")[:, :n]
    return bits.astype(np.uint8)


def _hadamard_free(gamma: np.ndarray, delta: np.ndarray) -> np.ndarray:
    """Symplectic 2n x 2n matrix of F(Gamma, Delta)."""
    n = delta.shape[0]
    f = np.zeros((2 * n, 2 * n), dtype=np.uint8)
    f[:n, :n] = delta
    f[n:, :n] = _mm2(gamma, delta)
    f[n:, n:] = _unit_lower_inverse(delta).T
    return f


def _random_bits(rng, shape):
    return rng.integers(0, 2, size=shape, dtype=np.uint8)


def random_destabilizer_bits(n: int, rng: np.random.Generator, phases: bool = True):
    """A uniformly random n-qubit Clifford as (phases [2n], xzs 0/1 [2n, 2n]):
    rows are the images of X_1..X_n then Z_1..Z_n (destabilizers then
    stabilizers), columns x bits then z bits."""
    h, perm = quantum_mallows(n, rng)
    lo_r, lo_c = np.tril_indices(n, -1)
    # F2: unconstrained Delta' (unit lower) and Gamma' (symmetric)
    delta2 = np.eye(n, dtype=np.uint8)
    delta2[lo_r, lo_c] = _random_bits(rng, len(lo_r))
    gamma2 = np.zeros((n, n), dtype=np.uint8)
    g = _random_bits(rng, len(lo_r))
    gamma2[lo_r, lo_c] = g
    gamma2[lo_c, lo_r] = g
    gamma2[np.arange(n), np.arange(n)] = _random_bits(rng, n)
    # F1: free bits only where the canonical form allows them
    hr, hc = h[lo_r], h[lo_c]
    pr, pc = perm[lo_r], perm[lo_c]
    g_free = (hr & hc) | (hr & ~hc & (pr < pc)) | (~hr & hc & (pr > pc))
    d_free = (hr & hc & (pr > pc)) | (~hr & hc) | (~hr & ~hc & (pr < pc))
    delta1 = np.eye(n, dtype=np.uint8)
    delta1[lo_r, lo_c] = _random_bits(rng, len(lo_r)) & d_free
    gamma1 = np.zeros((n, n), dtype=np.uint8)
    g = _random_bits(rng, len(lo_r)) & g_free
    gamma1[lo_r, lo_c] = g
    gamma1[lo_c, lo_r] = g
    gamma1[np.arange(n), np.arange(n)] = _random_bits(rng, n) & h
    f1 = _hadamard_free(gamma1, delta1)
    f2 = _hadamard_free(gamma2, delta2)
    # U = H(h) . S(perm) . F2 on rows: permute, then swap x/z rows where h
    u = f2[np.concatenate([perm, perm + n])]
    hi = np.flatnonzero(h)
    u[np.concatenate([hi, hi + n])] = u[np.concatenate([hi + n, hi])]
    xzs = np.zeros((2 * n, 2 * n), dtype=np.uint8)
    xzs[:n] = _mm2(f1[:n, :n], u[:n])
    xzs[n:] = _mm2(f1[n:, :n], u[:n]) ^ _mm2(f1[n:, n:], u[n:])
    ph = (2 * _random_bits(rng, 2 * n)) if phases else np.zeros(2 * n, dtype=np.uint8)
    return ph.astype(np.uint8), xzs


def random_destabilizer(n: int, rng: Optional[np.random.Generator] = None, phases: bool = True) -> Destabilizer:
    """random_destabilizer(n) (src/randoms.jl:155-230): a uniformly random
    full-rank Destabilizer (host tableau, 2n rows)."""
    rng = np.random.default_rng() if rng is None else rng
    ph, xzs = random_destabilizer_bits(n, rng, phases)
    return Destabilizer(Tableau.from_bits(ph, xzs[:, :n].astype(bool), xzs[:, n:].astype(bool)))


def random_stabilizer(n: int, rng: Optional[np.random.Generator] = None, phases: bool = True) -> Stabilizer:
    """random_stabilizer(n) (src/randoms.jl:440): the stabilizer rows of a
    random_destabilizer(n), a uniformly random n-qubit stabilizer state."""
    d = random_destabilizer(n, rng, phases)
    return Stabilizer(Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy()))


def random_clifford(n: int, rng: Optional[np.random.Generator] = None, phases: bool = True) -> CliffordOperator:
    """random_clifford(n) (src/randoms.jl:427-430): a uniformly random n-qubit
    Clifford operator (images of X_1..X_n, Z_1..Z_n)."""
    return CliffordOperator(random_destabilizer(n, rng, phases).tab)


def random_paulis(k: int, n: int, rng: Optional[np.random.Generator] = None, *, weight: str = "uniform",
                  phases: bool = False) -> Tableau:
    """k random n-qubit Paulis as the rows of a host Tableau.  weight
    "uniform": the weight w ~ U{1..n}, then w distinct qubits, each X, Y or Z
    with probability 1/3 (the Pauli workload of the projection benchmarks);
    weight "full": every qubit I, X, Y or Z uniformly (random_pauli(n),
    src/randoms.jl:31-49).  phases: a random sign (0 or 2) per row, else 0."""
    rng = np.random.default_rng() if rng is None else rng
    xs = np.zeros((k, n), dtype=bool)
    zs = np.zeros((k, n), dtype=bool)
    for j in range(k):
        if weight == "uniform":
            w = int(rng.integers(1, n + 1))
            qs = rng.choice(n, w, replace=False)
            kinds = rng.integers(1, 4, w)
            xs[j, qs] = (kinds & 1) > 0
            zs[j, qs] = (kinds & 2) > 0
        elif weight == "full":
            kinds = rng.integers(0, 4, n)
            xs[j] = (kinds & 1) > 0
            zs[j] = (kinds & 2) > 0
        else:
            raise ValueError("weight must be 'uniform' or 'full'")
    ph = 2 * rng.integers(0, 2, k) if phases else np.zeros(k, dtype=np.int64)
    return Tableau.from_bits(ph, xs, zs)
