"""GPU parity tests for the Pauli-frame engine (through the C ABI).

Bit-exact against the CPU oracle:
  * mask mode (shared seeded event file) against the reference-structured
    restatement: record and final frame (coding bits; reference padding bits
    are random and are not compared);
  * Philox mode against the oracle's restatement of the device procedure.
Statistical: Philox mode against the reference-structured per-frame draws,
per-detector rates within 5 sigma.
"""
import numpy as np
import pytest

import oracle
import qcb200
from qcb200 import circuits, ops as O

pytestmark = pytest.mark.gpu


def coding(xzs, nq1):
    return xzs & oracle.coding_mask(nq1)[:, None]


def run_mask(qcb, circ, frames, seed=0, qubits=None, nbits=None):
    arr = O.to_array(circ)
    qmax, bmax = O.affected_counts(arr)
    qubits = qubits or qmax
    nbits = nbits or bmax
    masks = qcb.sample_masks(arr, frames, qubits=qubits, seed=seed)
    f = qcb.PauliFrame(frames, qubits, nbits, masks=masks)
    qcb.pftrajectories(f, arr, masks=masks)
    ox, om = oracle.pftrajectories_mask(arr, frames, qubits, nbits, masks.init_z, masks.reset_planes, masks.events)
    return f, ox, om


def test_device_philox_matches_oracle(qcb):
    import ctypes

    for ctr, key in [([0, 0, 0, 0], [0, 0]), ([1, 2, 3, 4], [5, 6]), ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)]:
        c = (ctypes.c_uint32 * 4)(*ctr)
        k = (ctypes.c_uint32 * 2)(*key)
        out = (ctypes.c_uint32 * 4)()
        qcb.check(qcb.lib().qcb_debug_philox(c, k, out))
        assert list(out) == list(oracle.philox(ctr, key))


@pytest.mark.parametrize("frames", [10_000, 1, 31, 33, 1000])
def test_repetition_code_mask_mode_bit_exact(qcb, frames):
    circ = circuits.repetition_code_memory(7, 7, 1e-3 if frames == 10_000 else 0.2)
    f, ox, om = run_mask(qcb, circ, frames, seed=frames)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), 14), coding(ox, 14))


def test_surface_code_d11_mask_mode_bit_exact(qcb):
    circ = circuits.rotated_surface_code_memory(11, 11, 1e-3)
    f, ox, om = run_mask(qcb, circ, 10_000, seed=5)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), 242), coding(ox, 242))


# the invertible bit maps (xx, xz, zx, zz) of a single-qubit Clifford
SQO_MAPS = [(1, 0, 0, 1), (0, 1, 1, 0), (1, 1, 0, 1), (1, 0, 1, 1), (0, 1, 1, 1), (1, 1, 1, 0)]


def random_sqo(q, rng):
    m = SQO_MAPS[rng.integers(len(SQO_MAPS))]
    return O.SingleQubitOperator(q, *m, bool(rng.integers(2)), bool(rng.integers(2)))


def random_circuit(n, length, rng, p=0.05, nbits_start=1):
    g1 = ["H", "S", "SDAG", "X", "Y", "Z", "SQRTX", "INVSQRTX", "SQRTY", "INVSQRTY", "HXY", "HYZ", "CXYZ", "CZYX", "I"]
    g2 = ["CNOT", "CPHASE", "SWAP", "ZCX", "ZCY", "ZCZ", "XCX", "XCY", "XCZ", "YCX", "YCY", "YCZ",
          "SWAPCX", "INVSWAPCX", "ISWAP", "INVISWAP", "CZSWAP", "CXSWAP", "ZCRY", "INVZCRY", "SQRTZZ", "INVSQRTZZ",
          "SQRTXX", "INVSQRTXX", "SQRTYY", "INVSQRTYY"]
    c, bit = [], nbits_start
    for _ in range(length):
        k = rng.integers(0, 10)
        q = int(rng.integers(1, n + 1))
        if k < 3:
            if rng.random() < 0.25:
                c.append(random_sqo(q, rng))
            else:
                c.append(O.Op(O.OP[g1[rng.integers(len(g1))]], q))
        elif k < 6:
            q2 = int(rng.integers(1, n + 1))
            if q2 != q:
                c.append(O.Op(O.OP[g2[rng.integers(len(g2))]], q, q2))
        elif k == 6:
            meas = ["MZ", "MRZ", "MX", "MRX"][rng.integers(4)]
            b = bit if rng.random() < 0.8 else 0
            c.append(O.Op(O.OP[meas], q, 0, b))
            bit += 1
        elif k == 7:
            c += O.PauliError(q, *(rng.random(3) * p))
        elif k == 8:
            q2 = int(rng.integers(1, n + 1))
            if q2 != q:
                c += O.NoiseOp(O.DepolarizationNoise(p * 3), (q, q2))
        elif k == 9 and rng.random() < 0.5:
            if bit > 2 and rng.random() < 0.5:  # a detector-like XOR of earlier bits
                k_in = int(rng.integers(1, min(bit - 1, 12) + 1))
                c += O.ClassicalXOR([int(b) for b in rng.integers(1, bit, size=k_in)], bit)
            else:  # a random Pauli measured through the ancilla n+1
                c += O.PauliMeasurement("".join("IXZY"[int(v)] for v in rng.integers(0, 4, size=n)), bit)
            bit += 1
        else:
            c += O.NoiseOp(O.DepolarizationNoise(p * 2), (q,))
    c.append(O.sMZ(1, bit))
    return c


@pytest.mark.parametrize("seed", range(6))
def test_random_circuits_mask_mode_bit_exact(qcb, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 70))
    circ = random_circuit(n, 400, rng)
    frames = int(rng.integers(1, 3000))
    f, ox, om = run_mask(qcb, circ, frames, seed=seed)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), f.qubits + 1), coding(ox, f.qubits + 1))


def xor_chain_circuit(rng):
    """Stores among their own inputs, chains of XORs reading earlier stores,
    30-input XORs, XORs between measurements of the same round."""
    c = []
    for r in range(6):
        for q in range(1, 33):
            c.append(O.Op(O.OP["H"], q))
            c += O.PauliError(q, 0.1, 0.05, 0.02)
            c.append(O.sMZ(q, 32 * r + q))
        c += O.ClassicalXOR(list(range(32 * r + 1, 32 * r + 31)), 32 * r + 2)
        c += O.ClassicalXOR([32 * r + 2, 32 * r + 3], 32 * r + 3)
        c += O.ClassicalXOR([32 * r + 3], 200 + r)
        for _ in range(4):
            ins = [int(b) for b in rng.integers(1, 32 * r + 33, size=int(rng.integers(1, 31)))]
            c += O.ClassicalXOR(ins, int(rng.choice(ins)))
        c += O.PauliMeasurement("Z" + "I" * 31, 210 + r)
    return c


def test_classical_xor_chains_bit_exact(qcb):
    f, ox, om = run_mask(qcb, xor_chain_circuit(np.random.default_rng(21)), 2500, seed=4)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), f.qubits + 1), coding(ox, f.qubits + 1))


@pytest.mark.parametrize("nq", [1200, 3000])
def test_tall_frames_bit_exact(qcb, nq):
    # 1200 touched qubits: a narrow shared-memory tile (16..22 columns);
    # 3000: more than a 16-column tile holds, so the walker runs on the HBM planes
    rng = np.random.default_rng(9)
    circ = random_circuit(nq, 3000, rng, p=0.02)
    circ += [O.sCNOT(q, q + 1) for q in range(1, nq, 2)]
    f, ox, om = run_mask(qcb, circ, 700, seed=9)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), f.qubits + 1), coding(ox, f.qubits + 1))


@pytest.mark.parametrize("which", ["rep", "surface5", "random"])
def test_philox_mode_bit_exact_against_oracle_replica(qcb, which):
    rng = np.random.default_rng(1)
    if which == "rep":
        circ, frames = circuits.repetition_code_memory(7, 7, 0.05), 10_000
    elif which == "surface5":
        circ, frames = circuits.rotated_surface_code_memory(5, 5, 0.02), 4096
    else:
        circ, frames = random_circuit(40, 500, rng, p=0.1), 3000
    arr = O.to_array(circ)
    qmax, bmax = O.affected_counts(arr)
    seed = 0x1234_5678_9ABC
    f = qcb.pftrajectories(arr, trajectories=frames, seed=seed)
    ox, om = oracle.pftrajectories_philox(arr, frames, qmax, bmax, seed)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), qmax + 1), coding(ox, qmax + 1))


@pytest.mark.parametrize("mode", ["mask", "philox"])
def test_tall_program_16k_windows_bit_exact(qcb, mode):
    """d = 25 (1,250 frame slots, 600-site flushes longer than an 8 KB
    window): the program runs in 16 KB windows on 18-column tiles."""
    circ = circuits.rotated_surface_code_memory(25, 2, 0.01)
    if mode == "mask":
        f, ox, om = run_mask(qcb, circ, 1500, seed=25)
    else:
        arr = O.to_array(circ)
        qmax, bmax = O.affected_counts(arr)
        f = qcb.pftrajectories(arr, trajectories=3000, seed=2525)
        ox, om = oracle.pftrajectories_philox(arr, 3000, qmax, bmax, 2525)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), f.qubits + 1), coding(ox, f.qubits + 1))


@pytest.mark.parametrize("tile", [0, 8, 12, 16, 40, 106, 256])
@pytest.mark.parametrize("d,p", [(5, 0.004), (3, 0.015), (3, 1e-4)])
def test_philox_sparse_noise_any_tile_width(qcb, tile, d, p):
    # sparse sites (p_eff * 1024 <= 16): Binomial counts, distinct positions,
    # several events per group at p = 0.015; tiles of 12/16/40/106 columns cut
    # 1024-shot groups, which both neighbouring tiles draw; 8-column tiles are
    # the narrow tiles of tall programs
    arr = O.to_array(circuits.rotated_surface_code_memory(d, d, p))
    qmax, bmax = O.affected_counts(arr)
    frames = 9 * 1024 + 100
    qcb.check(qcb.lib().qcb_tune_set(b"walker_tile", tile))
    try:
        f = qcb.pftrajectories(arr, trajectories=frames, seed=99)
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"walker_tile", 0))
    ox, om = oracle.pftrajectories_philox(arr, frames, qmax, bmax, 99)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), qmax + 1), coding(ox, qmax + 1))


@pytest.mark.parametrize("tile", [8, 12, 16, 40, 106])
def test_mask_mode_any_tile_width(qcb, tile):
    circ = circuits.rotated_surface_code_memory(3, 3, 0.01)
    qcb.check(qcb.lib().qcb_tune_set(b"walker_tile", tile))
    try:
        f, ox, om = run_mask(qcb, circ, 5000, seed=tile)
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"walker_tile", 0))
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), f.qubits + 1), coding(ox, f.qubits + 1))


def test_shot_offset_shards_compose(qcb):
    circ = O.to_array(circuits.rotated_surface_code_memory(3, 3, 0.05))
    qmax, bmax = O.affected_counts(circ)
    full = qcb.PauliFrame(4096, qmax, bmax, seed=77)
    qcb.pftrajectories(full, circ, seed=77)
    parts = []
    for k in range(2):
        f = qcb.PauliFrame(2048, qmax, bmax, seed=77, shot_offset=2048 * k)
        qcb.pftrajectories(f, circ, seed=77)
        parts.append(f.measurements())
    assert np.array_equal(full.measurements(), np.vstack(parts))


def test_host_call_matches_frame_api(qcb):
    circ = O.to_array(circuits.rotated_surface_code_memory(5, 5, 1e-2))
    planes = qcb.pftrajectories_record(circ, 5000, seed=3)
    f = qcb.pftrajectories(circ, trajectories=5000, seed=3)
    assert np.array_equal(qcb.unpack_record(planes, 5000), f.measurements())
    assert np.array_equal(planes, f.record_planes())


@pytest.mark.parametrize("frames,offset", [(400_017, 0), (1_000_000, 3 * 1024)])
def test_host_call_chunked_copy_out_matches_one_launch(qcb, frames, offset):
    """The host call splits wide runs into shot chunks whose record columns
    are copied out while later chunks run; the record is that of one launch
    (a ragged last word, a shot offset, chunks of growing width)."""
    circ = O.to_array(circuits.rotated_surface_code_memory(3, 3, 1e-2))
    qmax, bmax = O.affected_counts(circ)
    planes = qcb.pftrajectories_record(circ, frames, seed=11, shot_offset=offset)
    f = qcb.PauliFrame(frames, qmax, bmax, seed=11, shot_offset=offset)
    qcb.pftrajectories(f, circ, seed=11)
    assert np.array_equal(planes, f.record_planes())
    assert planes.any()


def test_single_op_apply_equals_program(qcb):
    rng = np.random.default_rng(3)
    circ = O.flatten(random_circuit(12, 120, rng))
    arr = O.to_array(circ)
    qmax, bmax = O.affected_counts(arr)
    masks = qcb.sample_masks(arr, 500, qubits=qmax, seed=2)
    whole = qcb.PauliFrame(500, qmax, bmax, masks=masks)
    qcb.pftrajectories(whole, arr, masks=masks)
    step = qcb.PauliFrame(500, qmax, bmax, masks=masks)
    # apply op by op: remap events and reset planes to each single-op call
    # (a ClassicalXOR goes with its XOR_BITS payload ops)
    resets = 0
    k = 0
    while k < len(circ):
        op = circ[k]
        n = 1 + ((op.q1 + 2) // 3 if op.opcode == O.OP["XOR"] else 0)
        ev = masks.events[masks.events["op_index"] == k].copy()
        ev["op_index"] = 0
        nres = 1 if op.opcode in (O.OP["MRZ"], O.OP["MRX"]) else 0
        rp = masks.reset_planes[resets:resets + nres]
        resets += nres
        step.apply(circ[k:k + n], masks=qcb.Masks(masks.init_z, rp, ev))
        k += n
    assert np.array_equal(step.measurements(), whole.measurements())
    x1, z1 = step.planes()
    x2, z2 = whole.planes()
    assert np.array_equal(x1, x2) and np.array_equal(z1, z2)


def test_reference_layout_roundtrip(qcb):
    rng = np.random.default_rng(4)
    frames, qubits = 777, 130
    wp = 2 * ((qubits + 1 + 63) // 64)
    xzs = rng.integers(0, 2**63, size=(wp, frames), dtype=np.uint64) & oracle.coding_mask(qubits + 1)[:, None]
    f = qcb.PauliFrame(frames, qubits, 3, init=False)
    f.set_xzs(xzs)
    assert np.array_equal(f.xzs(), xzs)


def test_errors_are_reported_like_the_reference(qcb):
    f = qcb.PauliFrame(64, 3, 2)
    with pytest.raises(qcb.BoundsError):
        qcb.pftrajectories(f, [O.sCNOT(1, 5)])  # qubit 5 > 3 + hidden ancilla
    with pytest.raises(qcb.BoundsError):
        qcb.pftrajectories(f, [O.sMZ(1, 3)])
    qcb.pftrajectories(f, [O.sCNOT(1, 4)])  # the hidden ancilla is addressable
    bad = np.zeros(1, dtype=qcb.EVENT_DTYPE)
    with pytest.raises(qcb.ArgumentError):
        qcb.pftrajectories(f, [O.sX(1)], masks=qcb.Masks(np.zeros((4, 2), np.uint32), np.zeros((0, 2), np.uint32), bad))


def test_philox_statistics_match_reference_draws(qcb):
    """Per-detector rates of the d=5 memory circuit at 1e6 shots: Philox mode
    against the reference-structured per-frame draws, within 5 sigma."""
    d, frames = 5, 1_000_000
    circ = O.to_array(circuits.rotated_surface_code_memory(d, d, 5e-3))
    qmax, bmax = O.affected_counts(circ)
    planes = qcb.pftrajectories_record(circ, frames, seed=2024)
    dev = circuits.surface_code_detectors(qcb.unpack_record(planes, frames), d)
    _, om = oracle.pftrajectories_rng(circ, frames, qmax, bmax, seed=99, threads=8)
    ref = circuits.surface_code_detectors(om, d)
    p1, p2 = dev.mean(axis=0), ref.mean(axis=0)
    pbar = (p1 + p2) / 2
    sigma = np.sqrt(2 * pbar * (1 - pbar) / frames) + 1e-12
    z = np.abs(p1 - p2) / sigma
    assert z.max() < 5, (z.max(), p1[:5], p2[:5])
    assert p1.mean() > 0.005  # the noise is actually there
    # individual data measurements are uniformly random (initZ! / reset randomisation)
    rec = qcb.unpack_record(planes[-d * d:], frames)
    assert abs(rec.mean() - 0.5) < 0.01


def test_noisy_gate_and_noise_op_all_on_frames(qcb):
    """NoisyGate and NoiseOpAll through pftrajectories(frame, circuit): the
    frame's qubit count sizes NoiseOpAll (8 here, above the ops' highest
    qubit 5), bit for bit against the oracle on the lowered circuit."""
    noise = O.UnbiasedUncorrelatedNoise(0.05)
    circ = ([O.sHadamard(q) for q in range(1, 6)] + [O.NoisyGate(O.sCNOT(1, 4), noise), O.NoiseOpAll(noise)]
            + [O.sMZ(q, q) for q in range(1, 6)])
    masks = qcb.sample_masks(O.to_array(circ, 8), 4096, qubits=8, seed=6)
    f = qcb.PauliFrame(4096, 8, 5, masks=masks)
    qcb.pftrajectories(f, circ, masks=masks)
    arr = O.to_array(circ, 8)
    assert (arr["opcode"] == O.OP["PAULI_NOISE"]).sum() == 2 + 8
    ox, om = oracle.pftrajectories_mask(arr, 4096, 8, 5, masks.init_z, masks.reset_planes, masks.events)
    assert np.array_equal(f.measurements(), om)
    assert np.array_equal(coding(f.xzs(), 9), coding(ox, 9))


def test_frame_copy_is_independent(qcb):
    """copy(frame): same bits and record; later ops on the copy leave the
    original as it was."""
    circ = O.to_array(circuits.rotated_surface_code_memory(3, 3, 0.02))
    qmax, bmax = O.affected_counts(circ)
    f = qcb.pftrajectories(circ, trajectories=3000, seed=12)
    g = f.copy()
    assert np.array_equal(g.measurements(), f.measurements()) and np.array_equal(g.xzs(), f.xzs())
    before = f.xzs()
    g.apply([O.sHadamard(q) for q in range(1, qmax + 1)])
    assert np.array_equal(f.xzs(), before) and not np.array_equal(g.xzs(), before)
    with pytest.raises(qcb.DimensionMismatch):
        qcb.check(qcb.lib().qcb_frame_copy(qcb.PauliFrame(3000, qmax + 1, bmax).handle, f.handle, None))


@pytest.mark.parametrize("frames,nbits", [(1, 1), (33, 5), (1000, 49), (4096, 3)])
def test_measurements_upload_roundtrip(qcb, frames, nbits):
    """A reference frame's Bool record onto the device and back, and the run
    continues from it: bits the circuit does not write keep their values."""
    rng = np.random.default_rng(frames)
    m = rng.random((frames, nbits)) < 0.5
    f = qcb.PauliFrame(frames, 3, nbits, init=False)
    f.set_measurements(m)
    assert np.array_equal(f.measurements(), m)
    assert np.array_equal(f.record_planes(), qcb.pack_record(m))
    f.apply([O.sMZ(1, 1)])  # x starts at zero: bit 1 becomes false, the rest stay
    m2 = m.copy()
    m2[:, 0] = False
    assert np.array_equal(f.measurements(), m2)


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("which", ["d11", "d5_dense_mix", "d25_tall", "random"])
def test_presampled_noise_bit_exact(qcb, mode, which):
    """The noise of a Philox run drawn by the pre-sampler (mode 0, the
    default), in the walk (1), or pre-sampled with every bucket reporting an
    overflow so that the walk redraws it (2): the same record and frame, bit
    for bit against the oracle.  d5 at p = 0.02 mixes dense two-qubit sites
    (drawn in the walk) with sparse ones; d25 runs 16 KB windows."""
    rng = np.random.default_rng(5)
    if which == "d11":
        circ, frames = circuits.rotated_surface_code_memory(11, 3, 2e-3), 20_000
    elif which == "d5_dense_mix":
        circ, frames = circuits.rotated_surface_code_memory(5, 5, 0.02), 9 * 1024 + 77
    elif which == "d25_tall":
        circ, frames = circuits.rotated_surface_code_memory(25, 2, 0.01), 3000
    else:
        circ, frames = random_circuit(40, 500, rng, p=0.1), 3000
    arr = O.to_array(circ)
    qmax, bmax = O.affected_counts(arr)
    qcb.check(qcb.lib().qcb_tune_set(b"presample", mode))
    try:
        f = qcb.pftrajectories(arr, trajectories=frames, seed=4242)
        rec = f.measurements()
        xzs = f.xzs()
        planes = qcb.pftrajectories_record(arr, frames, seed=4242)  # the host call, chunked
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"presample", 0))
    ox, om = oracle.pftrajectories_philox(arr, frames, qmax, bmax, 4242)
    assert np.array_equal(rec, om)
    assert np.array_equal(coding(xzs, qmax + 1), coding(ox, qmax + 1))
    assert np.array_equal(qcb.unpack_record(planes, frames), om)


@pytest.mark.parametrize("frames", [1, 31, 4097, 300_001])
def test_measurements_download_chunks(qcb, frames):
    """measurements(frame) through the staged download: 32 MB chunks that
    cut bit rows (300,001 frames x 241 bits = 72 MB), ragged frame counts."""
    circ = O.to_array(circuits.rotated_surface_code_memory(11, 1, 1e-3))
    qmax, bmax = O.affected_counts(circ)
    f = qcb.pftrajectories(circ, trajectories=frames, seed=8)
    assert np.array_equal(f.measurements(), qcb.unpack_record(f.record_planes(), frames))


def test_chunked_presampled_run_equals_one_launch(qcb):
    """A Philox run whose noise pre-sampler scratch would pass its cap (d = 11
    at p = 1e-2, 2^23 shots: about 1.6 GB of event buckets) runs as column
    chunks of whole walker waves on two streams, each with its noise
    pre-sampled; record and frame equal the one-launch run that draws the
    noise in the walk, bit for bit, and its first 32k shots the oracle."""
    arr = O.to_array(circuits.rotated_surface_code_memory(11, 11, 1e-2))
    qmax, bmax = O.affected_counts(arr)
    shots = 1 << 23
    prog = qcb.Program(arr)
    got = []
    for mode in (0, 1):  # 0: chunked and pre-sampled; 1: one launch, noise in the walk
        qcb.check(qcb.lib().qcb_tune_set(b"presample", mode))
        try:
            f = qcb.PauliFrame(shots, qmax, bmax, init=False)
            qcb.check(qcb.lib().qcb_pftrajectories_fresh(f.handle, prog.handle, 99, 0, None))
            got.append((f.record_planes(), f.xzs()))
            del f
        finally:
            qcb.check(qcb.lib().qcb_tune_set(b"presample", 0))
    (p0, x0), (p1, x1) = got
    assert np.array_equal(p0, p1)
    cm = oracle.coding_mask(qmax + 1)[:, None]
    assert np.array_equal(x0 & cm, x1 & cm)
    n = 32 * 1024
    ox, om = oracle.pftrajectories_philox(arr, n, qmax, bmax, 99)
    assert np.array_equal(p0[:, : n // 32], qcb.pack_record(om))
    assert np.array_equal(x0[:, :n] & cm, ox & cm)


@pytest.mark.parametrize("narrow", [1, 0])
def test_tall_circuit_narrow_tiles(qcb, narrow):
    """A d = 33 surface code (2,177 qubits): a 16-column tile of every touched
    qubit does not fit shared memory, so the walker takes 8..14-column tiles
    (walker_narrow 1, the default) or walks the HBM planes (0); both bit-exact
    against the oracle, fresh Philox runs with pre-sampled noise."""
    arr = O.to_array(circuits.rotated_surface_code_memory(33, 2, 2e-3))
    qmax, bmax = O.affected_counts(arr)
    frames = 5 * 1024 + 300
    qcb.check(qcb.lib().qcb_tune_set(b"walker_narrow", narrow))
    try:
        f = qcb.pftrajectories(arr, trajectories=frames, seed=33)
        rec = f.measurements()
        xzs = f.xzs()
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"walker_narrow", 1))
    ox, om = oracle.pftrajectories_philox(arr, frames, qmax, bmax, 33)
    assert np.array_equal(rec, om)
    assert np.array_equal(coding(xzs, qmax + 1), coding(ox, qmax + 1))


def test_walker_autotuner_pairs_and_results(qcb):
    """qcb_tune_walker times (tile, threads per CTA) pairs for a program at a
    frame width and records the fastest; later fresh runs of that width take
    it, and their record and frame are still bit-exact against the oracle
    (any launch shape walks the same program on the same columns)."""
    arr = O.to_array(circuits.rotated_surface_code_memory(7, 7, 3e-3))
    qmax, bmax = O.affected_counts(arr)
    prog = qcb.Program(arr)
    frames = 20 * 1024 + 77
    try:
        tile, threads, ms = qcb.tune_walker(prog, frames)
        assert tile % 2 == 0 and 8 <= tile <= 256 and threads in (448, 512, 576, 640) and ms > 0
        f = qcb.PauliFrame(frames, qmax, bmax, init=False)
        qcb.check(qcb.lib().qcb_pftrajectories_fresh(f.handle, prog.handle, 71, 0, None))
        rec = f.measurements()
        xzs = f.xzs()
    finally:
        qcb.tune_walker_clear()
    ox, om = oracle.pftrajectories_philox(arr, frames, qmax, bmax, 71)
    assert np.array_equal(rec, om)
    assert np.array_equal(coding(xzs, qmax + 1), coding(ox, qmax + 1))
