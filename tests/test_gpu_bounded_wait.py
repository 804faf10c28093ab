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
