"""CPU tests: the C ABI library loads and exports its header, host-side op
construction and validation, circuit generators, mask sampling, layouts."""
import ctypes
import os
import re

import numpy as np
import pytest

import qcb200
from qcb200 import circuits, ops as O
from qcb200._lib import ArgumentError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "qcb200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*|uint64_t)\s+(qcb_[a-z0-9_]+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(qcb200.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 40
    for s in syms:
        assert hasattr(lib, s), s


def test_binding_declares_every_symbol():
    qcb200.lib()  # loads without a GPU; no compute call
    from qcb200 import _lib

    src = open(_lib.__file__).read()
    for s in header_symbols():
        assert f'"{s}"' in src, s


def test_version_string_without_gpu():
    assert b"sm_100a" in qcb200.lib().qcb_version()


# every tuning / test knob of qcb_tune_set: (key, its default, a rejected value)
KNOBS = [("walker_tile", 0, 7), ("stage_withhold", 0, -1), ("presample", 0, 3), ("server_hash_bits", 0, 65),
         ("server_fill", 1, 2), ("walker_threads", 0, 65), ("canon_threads", 0, 33), ("canon_cluster", 0, 3),
         ("canon_blocked", 0, 3), ("canon_grid", 0, 3), ("canon_rpt", 0, 3), ("walker_narrow", 1, 2),
         ("walker_pdl", 1, 2), ("canon_pdl", 1, 2), ("canon_lookahead", 1, 2), ("gates_pdl", 1, 2),
         ("canon_apply_rows", 0, 7), ("project_grid", 0, 3), ("project_withhold", 0, 2), ("project_cluster", 0, 3)]


def test_tune_knobs_validate_without_gpu():
    """qcb_tune_set only records host settings: each documented knob takes
    its default back and rejects an out-of-range value with QCB_EARG; an
    unknown key is rejected too.  No device call is made."""
    lib = qcb200.lib()
    hdr = open(os.path.join(ROOT, "include", "qcb200.h")).read()
    for key, default, bad in KNOBS:
        assert f'"{key}"' in hdr, key  # documented beside qcb_tune_set
        assert lib.qcb_tune_set(key.encode(), default) == 0, key
        assert lib.qcb_tune_set(key.encode(), bad) == 4, (key, bad)  # QCB_EARG
        assert lib.qcb_tune_set(key.encode(), default) == 0, key
    assert lib.qcb_tune_set(b"no_such_knob", 0) == 4


def test_op_validation_matches_reference_constructors():
    with pytest.raises(ArgumentError):
        O.sCNOT(1, 1)
    with pytest.raises(ArgumentError):
        O.sHadamard(0)
    with pytest.raises(ArgumentError):
        O.sMZ(0, 1)
    a = O.to_array([O.sCNOT(1, 2), O.sMZ(3, 4)] + O.PauliError([1, 2], 0.3))
    assert a.dtype.itemsize == 40
    assert list(a["opcode"]) == [O.OP["CNOT"], O.OP["MZ"], O.OP["PAULI_NOISE"], O.OP["PAULI_NOISE"]]
    assert np.allclose(a["p"][2], [0.1, 0.1, 0.1])
    assert O.affected_counts(a) == (3, 4)


def test_depolarization_parameterisation():
    # DepolarizationNoise(; two_qubit_error_probability=e) = DepolarizationNoise(16e/15) (src/noise.jl:53)
    d = O.DepolarizationNoise.from_two_qubit_error_probability(1.5e-3)
    assert abs(d.p - 1.6e-3) < 1e-15
    (op,) = O.NoiseOp(d, (3, 5))
    assert op.opcode == O.OP["DEPOL2"] and (op.q1, op.q2) == (3, 5)


def test_repetition_code_counts():
    c = O.to_array(circuits.repetition_code_memory(7, 7, 1e-3))
    # 7 rounds x (6+6 CNOT + 6 MRZ) + 7 MZ = 133 updates; 49 record bits
    assert O.count_updates(c) == 133
    assert O.affected_counts(c) == (13, 49)
    assert np.count_nonzero(c["opcode"] == O.OP["PAULI_NOISE"]) == 49


def test_rotated_surface_code_counts():
    d = 11
    c = O.to_array(circuits.rotated_surface_code_memory(d, d, 1e-3))
    oc = c["opcode"]
    assert np.count_nonzero(oc == O.OP["CNOT"]) == 11 * 440
    assert np.count_nonzero(oc == O.OP["H"]) == 11 * 120
    assert np.count_nonzero(oc == O.OP["MRZ"]) == 11 * 120
    assert np.count_nonzero(oc == O.OP["MZ"]) == 121
    assert O.count_updates(c) == 7601
    assert O.affected_counts(c) == (241, 1441)
    assert np.count_nonzero(oc == O.OP["DEPOL2"]) == 4840
    assert np.count_nonzero(oc == O.OP["PAULI_NOISE"]) == 1320 + 1320


@pytest.mark.parametrize("d", [3, 5, 7, 11, 25])
def test_surface_code_layers_are_disjoint(d):
    plaq = circuits.rotated_surface_code_layout(d)
    assert len(plaq) == d * d - 1
    assert sum(1 for p in plaq if p[0] == "X") == (d * d - 1) // 2
    for layer in range(4):
        seen = set()
        for t, _, _, corners in plaq:
            key = (circuits.X_ORDER if t == "X" else circuits.Z_ORDER)[layer]
            if key in corners:
                assert corners[key] not in seen
                seen.add(corners[key])
    # stabilizers commute: X and Z plaquettes overlap on an even number of qubits
    xs = [set(p[3].values()) for p in plaq if p[0] == "X"]
    zs = [set(p[3].values()) for p in plaq if p[0] == "Z"]
    for a in xs:
        for b in zs:
            assert len(a & b) % 2 == 0


def test_sample_masks_shapes_and_rates():
    c = circuits.repetition_code_memory(5, 5, 0.3)
    m = qcb200.sample_masks(c, 10_000, seed=4)
    assert m.init_z.shape == (10, (10_000 + 31) // 32)
    assert m.reset_planes.shape == (20, (10_000 + 31) // 32)
    a = O.to_array(c)
    first_noise = int(np.nonzero(a["opcode"] == O.OP["PAULI_NOISE"])[0][0])
    ev = m.events[m.events["op_index"] == first_noise]
    assert abs(len(ev) / 10_000 - 0.3) < 0.03
    assert set(np.unique(ev["pauli"])) <= {1, 2, 3}


def test_unpack_record_roundtrip():
    rng = np.random.default_rng(0)
    frames = 100
    bools = rng.random((frames, 7)) < 0.5
    words = (frames + 31) // 32
    planes = np.zeros((7, words), np.uint32)
    for b in range(7):
        for f in range(frames):
            if bools[f, b]:
                planes[b, f >> 5] |= np.uint32(1 << (f & 31))
    assert np.array_equal(qcb200.unpack_record(planes, frames), bools)


def test_tableau_string_parsing_roundtrip():
    t = qcb200.T("- XZZZZ_____ + _YZY___YX_ -i__XXZ__YX_")
    assert list(t.phases) == [2, 0, 3]
    assert str(t).split("\n")[0] == "- XZZZZ_____"
    xs, zs = t.bits()
    assert xs[1, 1] and zs[1, 1]
