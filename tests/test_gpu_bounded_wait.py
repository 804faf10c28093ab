"""The walker's bounded staging wait (no fault, no trap): with the test knob
"stage_withhold" one program window is never staged, the wait gives up after
about a second, the kernel returns and the next synchronising call reports
QCB_ETIMEOUT.  The device stays usable: the next normal run on the same frame
is bit-exact against the oracle."""
import time

import numpy as np
import pytest

import oracle
import qcb200
from qcb200 import circuits, ops as O

pytestmark = pytest.mark.gpu

QCB_ETIMEOUT = 7


def test_withheld_window_times_out_and_the_device_recovers(qcb):
    arr = O.to_array(circuits.rotated_surface_code_memory(11, 11, 1e-3))
    qmax, bmax = O.affected_counts(arr)
    prog = qcb.Program(arr)
    lib = qcb.lib()
    frame = qcb.PauliFrame(64, qmax, bmax, init=False)  # one tile, one CTA
    qcb.check(lib.qcb_tune_set(b"stage_withhold", 5))
    try:
        t0 = time.perf_counter()
        qcb.check(lib.qcb_pftrajectories_fresh(frame.handle, prog.handle, 3, 0, None))
        with pytest.raises(qcb.QCBError) as ei:
            frame.record_planes()  # synchronises and reads the walker's status word
        waited = time.perf_counter() - t0
    finally:
        qcb.check(lib.qcb_tune_set(b"stage_withhold", 0))
    assert ei.value.status == QCB_ETIMEOUT
    assert 0.5 < waited < 30, waited
    # the same frame and device, a normal run: bit-exact
    qcb.check(lib.qcb_pftrajectories_fresh(frame.handle, prog.handle, 3, 0, None))
    planes = frame.record_planes()
    _, om = oracle.pftrajectories_philox(arr, 64, qmax, bmax, 3)
    assert np.array_equal(qcb.unpack_record(planes, 64), om)


def test_project_grid_barrier_times_out_and_the_device_recovers(qcb):
    """The whole-GPU project! kernel's bounded grid barrier: with the test
    knob "project_withhold" one CTA leaves before the first barrier, the
    others' waits give up after about a second and the call returns
    QCB_ETIMEOUT (the tableau is untouched: phase 1 writes only flags).  The
    next call on the same state is bit-exact against the oracle."""
    from qcb200 import randoms
    from qcb200.tableau import Tableau

    n = 64
    rng = np.random.default_rng(12)
    tab = randoms.random_stabilizer(n, rng).tab
    ps = randoms.random_paulis(5, n, rng)
    lib = qcb.lib()
    st = qcb.Stabilizer(tab.copy()).to_gpu()
    qcb.check(lib.qcb_tune_set(b"project_grid", 1))
    try:
        qcb.check(lib.qcb_tune_set(b"project_withhold", 1))
        try:
            t0 = time.perf_counter()
            with pytest.raises(qcb.QCBError) as ei:
                qcb.project_(st, ps.copy().to_gpu())
            waited = time.perf_counter() - t0
        finally:
            qcb.check(lib.qcb_tune_set(b"project_withhold", 0))
        assert ei.value.status == QCB_ETIMEOUT
        assert 0.2 < waited < 30, waited
        st.to_cpu()
        assert np.array_equal(st.tab.xzs, tab.xzs) and np.array_equal(st.tab.phases, tab.phases)
        st.to_gpu()
        _, anti, res = qcb.project_(st, ps.copy().to_gpu())
    finally:
        qcb.check(lib.qcb_tune_set(b"project_grid", 0))
    st.to_cpu()
    ph, xz = tab.phases.copy(), tab.xzs.copy()
    outs = []
    for j in range(5):
        code, ph, xz, _, a, r = oracle.project("Stabilizer", ph, xz, n, ps.xzs[j], ps.phases[j])
        assert code == 0
        outs.append((a, None if r < 0 else r))
    assert list(zip(anti, res)) == outs
    assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)
