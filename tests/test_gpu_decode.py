"""GPU parity tests of the decoder hand-off (src/ecc/decoder_pipeline.jl
:163-190) through the C ABI: the syndrome / logical columns of the record,
the shot-major packed syndrome matrix, and evaluate_guesses, against the
oracle's record and its restatement of evaluate_guesses."""
import numpy as np
import pytest

import oracle
from qcb200 import circuits, ops as O

pytestmark = pytest.mark.gpu


def sampled(qcb, circ, frames, seed):
    arr = O.to_array(circ)
    qmax, bmax = O.affected_counts(arr)
    masks = qcb.sample_masks(arr, frames, qubits=qmax, seed=seed)
    f = qcb.PauliFrame(frames, qmax, bmax, masks=masks)
    qcb.pftrajectories(f, arr, masks=masks)
    _, om = oracle.pftrajectories_mask(arr, frames, qmax, bmax, masks.init_z, masks.reset_planes, masks.events)
    return f, om


def pack_rows(m):
    """Bool frames x nsel -> uint64 frames x ceil(nsel/64), bit b of word w = column 64w+b."""
    S, n = m.shape
    W = (n + 63) // 64
    pad = np.zeros((S, W * 64), dtype=np.uint8)
    pad[:, :n] = m
    return np.packbits(pad, axis=1, bitorder="little").view(np.uint64).reshape(S, W)


@pytest.mark.parametrize("frames", [1, 31, 33, 1000, 20_000])
def test_syndrome_and_logical_columns(qcb, frames):
    d = 5
    circ = circuits.rotated_surface_code_memory(d, d, 0.01)
    f, om = sampled(qcb, circ, frames, seed=frames)
    rng = np.random.default_rng(frames)
    nb = om.shape[1]
    syn = np.arange(1, nb - d * d + 1)            # the ancilla records of every round
    log = np.arange(nb - d * d + 1, nb + 1)       # the final data measurements
    for bits in (syn, log, rng.permutation(nb)[:77] + 1, np.array([nb, 1, nb])):
        got = f.measurement_columns(bits)
        assert np.array_equal(got, om[:, bits - 1])
        assert np.array_equal(f.syndrome_rows(bits), pack_rows(om[:, bits - 1]))
    ref = rng.random(nb) < 0.5
    assert np.array_equal(f.measurement_columns(syn, reference=ref), om[:, syn - 1] ^ ref[syn - 1])


def test_syndrome_rows_wide(qcb):
    # more selected bits than a CTA stages in shared memory (direct writes)
    c = []
    for k in range(13_000):
        q = 1 + k % 5
        c += O.PauliError(q, 0.2)
        c.append(O.sMZ(q, k + 1))
    f, om = sampled(qcb, c, 70, seed=3)
    bits = np.arange(1, 13_001)
    assert np.array_equal(f.syndrome_rows(bits), pack_rows(om))


@pytest.mark.parametrize("frames,k", [(1, 3), (100, 10), (5000, 97), (70_000, 242)])
def test_evaluate_guesses(qcb, frames, k):
    circ = circuits.rotated_surface_code_memory(3, 3, 0.05)
    f, om = sampled(qcb, circ, frames, seed=k)
    rng = np.random.default_rng(k)
    nb = om.shape[1]
    logical = rng.permutation(nb)[: min(4, nb)] + 1
    guesses = rng.random((frames, k)) < 0.1
    faults = rng.random((len(logical), k)) < 0.3
    got = qcb.evaluate_guesses(f, logical, guesses, faults)
    want, _ = oracle.evaluate_guesses(om[:, logical - 1], guesses, faults)
    assert got == want
    # no guessed faults: a shot fails exactly when a measured logical bit is set
    z = qcb.evaluate_guesses(f, logical, np.zeros((frames, k), bool), faults)
    assert z == np.count_nonzero(om[:, logical - 1].any(axis=1)) / frames
