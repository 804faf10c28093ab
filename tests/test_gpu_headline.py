"""Parity at the benchmarked configuration: the rotated surface-code memory
circuit, d = 11, 11 rounds, p = 1e-3, 1,000,000 shots, run by the same call
the benchmark times (qcb_pftrajectories_fresh on a preallocated frame, the
automatic tile width: 106 columns, 295 CTAs, 1024-shot noise groups
straddling tiles).

  * Philox mode, bit for bit: record and final frame (coding bits) against
    the oracle's restatement of the device procedure, run over the same
    1e6 shots in 32,768-shot slices on all host cores (the Philox counters
    depend only on the global shot group and column, so each slice is the
    matching part of one run).
  * Philox mode, statistically: per-detector rates of every Z-type detector
    (first round, consecutive rounds, last round against the data parity),
    every X-type detector (consecutive rounds) and the first-round X
    outcomes, against the reference-structured per-frame draws of the
    oracle (src/pauli_frames.jl:136-174, one rand() per frame per noise
    site) at 1e6 shots, within 5 sigma (the pattern of
    test/test_pauliframe.jl:24-43 and test/test_gpu.jl:116-133).
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle
import qcb200
from qcb200 import circuits, ops as O

pytestmark = pytest.mark.gpu

D, ROUNDS, P_NOISE, SHOTS = 11, 11, 1e-3, 1_000_000
SLICE = 32 * 1024


def threads():
    return max(1, min(32, os.cpu_count() or 1))


@pytest.fixture(scope="module")
def d11():
    arr = O.to_array(circuits.rotated_surface_code_memory(D, ROUNDS, P_NOISE))
    qmax, bmax = O.affected_counts(arr)
    assert O.count_updates(arr) == 7601 and (qmax, bmax) == (241, 1441)
    return arr, qmax, bmax


def run_fresh(qcb, arr, qmax, bmax, shots, seed, tile=0):
    """The benchmark's step: a fresh frame (initZ! fused) through the circuit."""
    prog = qcb.Program(arr)
    frame = qcb.PauliFrame(shots, qmax, bmax, init=False)
    qcb.check(qcb.lib().qcb_tune_set(b"walker_tile", tile))
    try:
        qcb.check(qcb.lib().qcb_pftrajectories_fresh(frame.handle, prog.handle, seed, 0, None))
        planes = frame.record_planes()
        xzs = frame.xzs()
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"walker_tile", 0))
    return planes, xzs


def check_philox_slices(arr, qmax, bmax, shots, seed, planes, xzs):
    cm = oracle.coding_mask(qmax + 1)[:, None]

    def one(off):
        n = min(SLICE, shots - off)
        ox, om = oracle.pftrajectories_philox(arr, n, qmax, bmax, seed, shot_offset=off)
        w0, nw = off // 32, (n + 31) // 32
        want = qcb200.pack_record(om)
        got = planes[:, w0:w0 + nw].copy()
        if n % 32:  # padding shots of the ragged last word are not part of the record
            m = np.uint32((1 << (n % 32)) - 1)
            got[:, -1] &= m
            want[:, -1] &= m
        rec_ok = np.array_equal(got, want)
        frame_ok = np.array_equal(xzs[:, off:off + n] & cm, ox & cm)
        return off, rec_ok, frame_ok

    with ThreadPoolExecutor(threads()) as ex:
        res = list(ex.map(one, range(0, shots, SLICE)))
    bad = [(off, r, f) for off, r, f in res if not (r and f)]
    assert not bad, f"slices differing from the oracle (offset, record ok, frame ok): {bad[:5]}"


def test_d11_philox_bit_exact_at_the_benchmark_config(qcb, d11):
    arr, qmax, bmax = d11
    seed = 1000  # the benchmark's first step seed
    planes, xzs = run_fresh(qcb, arr, qmax, bmax, SHOTS, seed)
    assert planes.shape == (1441, SHOTS // 32)
    check_philox_slices(arr, qmax, bmax, SHOTS, seed, planes, xzs)


@pytest.mark.parametrize("shots,tile", [(40_000, 106), (33_000, 40), (65_536, 256)])
def test_d11_philox_bit_exact_forced_tiles(qcb, d11, shots, tile):
    """Tiles that cut 1024-shot groups (106, 40 columns) and a group-aligned
    one (256), with ragged shot counts."""
    arr, qmax, bmax = d11
    planes, xzs = run_fresh(qcb, arr, qmax, bmax, shots, 77 + tile, tile=tile)
    check_philox_slices(arr, qmax, bmax, shots, 77 + tile, planes, xzs)


def test_d11_detector_rates_match_reference_draws(qcb, d11):
    arr, qmax, bmax = d11
    planes, _ = run_fresh(qcb, arr, qmax, bmax, SHOTS, 2024)
    dets = {b: circuits.surface_code_detector_bits(D, ROUNDS, b) for b in ("Z", "X", "X1")}
    dev = {b: circuits.detector_counts_from_planes(planes, SHOTS, v) for b, v in dets.items()}

    # the reference-structured run, in slices (different Xoshiro seeds per slice)
    ref = {b: np.zeros(len(v), np.int64) for b, v in dets.items()}
    chunk = 125_000
    for k, off in enumerate(range(0, SHOTS, chunk)):
        n = min(chunk, SHOTS - off)
        _, om = oracle.pftrajectories_rng(arr, n, qmax, bmax, seed=99 + k, threads=threads())
        p = qcb200.pack_record(om)
        del om
        for b, v in dets.items():
            ref[b] += circuits.detector_counts_from_planes(p, n, v)

    for b in dets:
        p1, p2 = dev[b] / SHOTS, ref[b] / SHOTS
        pbar = (p1 + p2) / 2
        sigma = np.sqrt(2 * pbar * (1 - pbar) / SHOTS) + 1e-12
        z = np.abs(p1 - p2) / sigma
        assert z.max() < 5, (b, float(z.max()), int(z.argmax()), p1[:6], p2[:6])
    # the noise is there, and the detectors are sparse at p = 1e-3
    for b in ("Z", "X"):
        assert 0.002 < dev[b].mean() / SHOTS < 0.05, (b, dev[b].mean() / SHOTS)
    assert np.all(np.abs(dev["X1"] / SHOTS - 0.5) < 0.005)
    assert len(dets["Z"]) == 60 * 12 and len(dets["X"]) == 60 * 10
