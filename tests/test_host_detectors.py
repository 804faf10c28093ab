"""CPU checks behind the headline parity tests: the detector definitions of
the memory-Z circuit (packed-plane counts equal the Bool-matrix detectors)
and the oracle's Philox procedure run in 1024-shot-aligned slices equals one
run over all the shots (what lets the GPU test check 1e6 shots in slices)."""
import numpy as np

import oracle
from qcb200 import circuits, ops as O
from qcb200 import pack_record


def test_detectors_from_planes_equal_bool_detectors():
    arr = O.to_array(circuits.rotated_surface_code_memory(5, 5, 0.01))
    q, b = O.affected_counts(arr)
    _, om = oracle.pftrajectories_philox(arr, 3001, q, b, 17)
    planes = pack_record(om)
    for basis in ("Z", "X", "X1"):
        bits = circuits.surface_code_detector_bits(5, 5, basis)
        want = circuits.surface_code_detectors(om, 5, basis=basis).sum(axis=0)
        assert np.array_equal(circuits.detector_counts_from_planes(planes, 3001, bits), want)
    assert len(circuits.surface_code_detector_bits(5, 5, "Z")) == 12 * 6
    assert len(circuits.surface_code_detector_bits(5, 5, "X")) == 12 * 4


def test_oracle_philox_slices_compose():
    arr = O.to_array(circuits.rotated_surface_code_memory(3, 3, 0.02))
    q, b = O.affected_counts(arr)
    frames = 5 * 1024 + 77
    ox, om = oracle.pftrajectories_philox(arr, frames, q, b, 9)
    parts = [oracle.pftrajectories_philox(arr, min(2048, frames - off), q, b, 9, shot_offset=off)
             for off in range(0, frames, 2048)]
    assert np.array_equal(np.vstack([p[1] for p in parts]), om)
    assert np.array_equal(np.hstack([p[0] for p in parts]), ox)
