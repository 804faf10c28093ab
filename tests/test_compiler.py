"""CPU tests of the circuit compiler: the device program, interpreted on the
host (tests/stream_emu.py), must reproduce the oracle bit for bit in mask
mode.  No GPU is involved: qcb_debug_program_dump compiles on the host."""
import numpy as np
import pytest

import oracle
import qcb200
import stream_emu
from qcb200 import circuits, ops as O

from test_gpu_frames import random_circuit, xor_chain_circuit  # noqa: E402  (shared generator; its GPU tests are marked)


def check_circuit(circ, frames, seed):
    arr = O.to_array(circ)
    qmax, bmax = O.affected_counts(arr)
    masks = qcb200.sample_masks(arr, frames, qubits=qmax, seed=seed)
    X, Z, rec, info = stream_emu.run_mask(arr, frames, qmax, bmax, masks)
    ox, om = oracle.pftrajectories_mask(arr, frames, qmax, bmax, masks.init_z, masks.reset_planes, masks.events)
    got = qcb200.unpack_record(rec, frames)
    assert np.array_equal(got, om)
    xzs = stream_emu.planes_to_xzs(X, Z, frames)
    m = oracle.coding_mask(qmax + 1)[:, None]
    assert np.array_equal(xzs & m, ox & m)
    return info


def test_repetition_code():
    info = check_circuit(circuits.repetition_code_memory(7, 7, 0.1), 300, 1)
    assert info["n_updates"] == 133


def test_surface_code_program_shape():
    info = check_circuit(circuits.rotated_surface_code_memory(5, 5, 0.02), 200, 2)
    # per round: four CNOT layers and the reset layer, a handful of flushes
    assert info["n_segments"] <= 5 * 6 + 2
    assert info["n_flushes"] <= 5 * 6 + 2


def test_surface_code_d11_segments():
    _, _, _, _, info = stream_emu.dump(circuits.rotated_surface_code_memory(11, 11, 1e-3))
    assert info["n_updates"] == 7601
    assert info["n_segments"] <= 11 * 6 + 2, info
    assert info["n_flushes"] <= 11 * 6 + 2, info


@pytest.mark.parametrize("seed", range(12))
def test_random_circuits(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 40))
    check_circuit(random_circuit(n, 300, rng, p=0.1), int(rng.integers(1, 200)), seed)


def test_relabels_and_noise_interleave():
    # noise between relabels on the same qubit, and measurements of relabelled qubits
    c = [O.sHadamard(1)] + O.PauliError(1, 0.3) + [O.sHadamard(1)] + O.PauliError(1, 0.3, 0.1, 0.2)
    c += [O.sCNOT(1, 2), O.sSQRTY(2)] + O.NoiseOp(O.DepolarizationNoise(0.5), (1, 2))
    c += [O.sMX(2, 1), O.sMRX(1, 2), O.sMZ(2, 3), O.sX(1), O.sMRZ(1, 4), O.sMZ(1, 2)]
    check_circuit(c, 500, 3)


def test_classical_xor_chains():
    info = check_circuit(xor_chain_circuit(np.random.default_rng(21)), 150, 4)
    assert info["n_flushes"] >= 1


def _records(stream):
    """(kind, count, continued, words) of every record of a device program,
    and the program's window size (carried by its WIN records)."""
    body = {1: lambda c: (2 * c + 3) // 4 * 4, 3: lambda c: (2 * c + 3) // 4 * 4, 4: lambda c: (2 * c + 3) // 4 * 4,
            6: lambda c: (2 * c + 3) // 4 * 4, 9: lambda c: (2 * c + 3) // 4 * 4, 5: lambda c: 4 * c,
            7: lambda c: 16 * c, 8: lambda c: 4 * c, 11: lambda c: 32 * c}
    out, pc, wins = [], 0, set()
    while pc < len(stream):
        h = int(stream[pc])
        kind, cnt = h >> 24, h & 0xFFFFFF
        if kind == 0:
            break
        if kind == 10:  # the stream continues in the next window; the count is its size
            wins.add(cnt)
            pc = pc // cnt * cnt + cnt
            continue
        n = body[kind](cnt)
        out.append((kind, cnt, int(stream[pc + 1]) & 1, 4 + n, pc))
        pc += 4 + n
    assert len(wins) <= 1 and wins <= {2048, 4096}
    win = wins.pop() if wins else len(stream)
    for r in out:
        assert r[4] // win == (r[4] + r[3] - 1) // win, "a record straddles a window"
    return out, win


@pytest.mark.parametrize("d", [3, 5, 11, 25])
def test_records_that_fit_a_window_are_not_split(d):
    """A split record is one more barrier-separated step of the walk, so the
    compiler starts a new window for a record that fits one instead of
    cutting it at the window edge; only longer records come in parts."""
    stream, _, _, _, info = stream_emu.dump(circuits.rotated_surface_code_memory(d, d, 1e-3))
    recs, win = _records(stream)
    if d >= 11:
        assert win == (4096 if d == 25 else 2048)  # 16 KB windows for the tall program only
    assert len(stream) % win == 0
    i = 0
    while i < len(recs):
        j = i
        while recs[j][2]:  # parts of one record: all but the last are marked continued
            assert recs[j + 1][0] == recs[i][0]
            j += 1
        total = 4 + sum(r[3] - 4 for r in recs[i:j + 1])
        if j > i:
            assert total > win - 4, (d, i, total)
        i = j + 1
    if d <= 11:
        assert not any(r[2] for r in recs)
    assert sum(1 for r in recs if r[0] == 8 and not r[2]) == info["n_flushes"]


def test_tall_program_runs_in_16k_windows():
    """A d=25 code (1,250 frame slots, 600-site flushes of 2,400 words) gets
    16 KB windows; interpreted on the host it reproduces the oracle."""
    circ = circuits.rotated_surface_code_memory(25, 2, 0.01)
    stream, _, _, _, _ = stream_emu.dump(circ)
    recs, win = _records(stream)
    assert win == 4096 and len(recs) > 10
    check_circuit(circ, 70, 8)


def test_noisy_gate_and_noise_op_all_lowering():
    """NoisyGate(g, noise) is g then the noise on g's qubits; NoiseOpAll(noise)
    is the noise on qubits 1..n of the frame (n given, else the highest qubit
    of the other ops, as _create_pauliframe sizes the frame)."""
    noise = O.UnbiasedUncorrelatedNoise(0.03)
    a = O.to_array([O.NoisyGate(O.sCNOT(2, 5), noise), O.NoisyGate(O.sHadamard(3), O.DepolarizationNoise(0.02)),
                    O.NoiseOpAll(noise), O.sMZ(4, 1)])
    b = O.to_array([O.sCNOT(2, 5), O.PauliError([2, 5], 0.03), O.sHadamard(3),
                    O.NoiseOp(O.DepolarizationNoise(0.02), [3]), O.PauliError([1, 2, 3, 4, 5], 0.03), O.sMZ(4, 1)])
    assert np.array_equal(a, b)
    c = O.to_array([O.NoiseOpAll(O.PauliNoise(0.01, 0.02, 0.03)), O.sMZ(2, 1)], nqubits=4)
    assert list(c["q1"][:4]) == [1, 2, 3, 4] and c["p"][0].tolist() == [0.01, 0.02, 0.03]
    with pytest.raises(qcb200.ArgumentError):
        O.NoisyGate(O.PauliError(1, 0.1), noise)
    # through the compiler and the stream emulator, bit for bit against the oracle
    check_circuit([O.sHadamard(q) for q in range(1, 7)] + [O.NoisyGate(O.sCNOT(1, 4), noise), O.NoiseOpAll(noise)]
                  + [O.sMZ(q, q) for q in range(1, 7)], 300, 3)


def test_sample_masks_lowers_noise_op_all_over_the_frame():
    """The event file of a circuit with NoiseOpAll refers to the ops of the
    lowering for the frame's qubit count, as pftrajectories(frame, circuit)
    compiles it."""
    noise = O.UnbiasedUncorrelatedNoise(0.3)
    circ = [O.sHadamard(1), O.NoiseOpAll(noise), O.sMZ(1, 1)]
    m = qcb200.sample_masks(circ, 256, qubits=6, seed=1)
    arr = O.to_array(circ, 6)
    assert len(arr) == 8 and m.init_z.shape[0] == 7
    assert set(np.unique(m.events["op_index"])) <= set(range(1, 7))
    assert len(np.unique(m.events["op_index"])) == 6  # p = 0.3 on 256 shots: every qubit's site fires


def test_noisy_gate_of_a_pauli_measurement():
    """NoisyGate(PauliMeasurement(P, b), noise): the measurement's ops, then
    the noise on qubits 1..n of its Pauli (affectedqubits(::PauliMeasurement)
    = 1:length(pauli), src/affectedqubits.jl:5, 11), as the Julia lowering
    does; bit for bit against the oracle through the compiler."""
    noise = O.UnbiasedUncorrelatedNoise(0.05)
    pm = O.PauliMeasurement("XIZY", 1)
    a = O.to_array([O.NoisyGate(pm, noise)])
    b = O.to_array(list(O.PauliMeasurement("XIZY", 1)) + O.PauliError([1, 2, 3, 4], 0.05))
    assert np.array_equal(a, b)
    circ = ([O.sHadamard(q) for q in range(1, 5)] + [O.NoisyGate(O.PauliMeasurement("XIZY", 1), noise)]
            + [O.sMZ(q, q + 1) for q in range(1, 5)])
    check_circuit(circ, 300, 4)
