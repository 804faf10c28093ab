"""A stream of symbolic apply! calls, one launch per call and no
synchronisation in between, as a user's loop of apply!(state, gate) issues
them.  Each launch is a programmatic dependent of the launch before it on the
stream (knob "gates_pdl", on by default); the kernel reads the rows only after
its predecessor has completed, so the calls keep their order, also next to
plain launches of other kernels and when the stream is replayed from a CUDA
graph.  Bit-exact with phases against the oracle's sequence."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from qcb200 import ops as O
from qcb200._lib import check, ptr
from test_gpu_tableau import rand_tab

pytestmark = pytest.mark.gpu

G1 = ["H", "S", "SDAG", "X", "Y", "Z", "SQRTX", "SQRTY", "HXY", "CXYZ"]
G2 = ["CNOT", "CPHASE", "SWAP", "ZCY", "XCX", "YCZ", "ISWAP", "SQRTZZ", "CXSWAP", "INVSQRTYY"]


def random_gates(n, count, rng):
    gates = []
    for _ in range(count):
        if rng.random() < 0.4:
            gates.append(O.Op(O.OP[G1[rng.integers(len(G1))]], int(rng.integers(1, n + 1))))
        else:
            a, b = rng.choice(np.arange(1, n + 1), 2, replace=False)
            gates.append(O.Op(O.OP[G2[rng.integers(len(G2))]], int(a), int(b)))
    return gates


@pytest.mark.parametrize("pdl", [1, 0])
def test_single_gate_calls_in_a_stream(qcb, pdl):
    n = 1000
    rng = np.random.default_rng(500 + pdl)
    t = rand_tab(n, n, rng)
    gates = random_gates(n, 300, rng)
    lib = qcb.lib()
    check(lib.qcb_tune_set(b"gates_pdl", pdl))
    try:
        g = t.copy().to_gpu()
        h = g._need_dev().handle
        side = torch.cuda.Stream()
        sp = ctypes.c_void_p(side.cuda_stream)
        ph, xz = t.phases.copy(), t.xzs.copy()
        for k, op in enumerate(gates):
            arr = O.to_array([op])
            check(lib.qcb_apply_gates(h, ptr(arr), 1, 1, sp))
            ph, xz = oracle.apply_gates(ph, xz, n, arr, True)
            if k % 25 == 24:
                # a plain launch of another kernel in between: row s <- row 1 * row s
                s_row = 2 + k % 50
                check(lib.qcb_mul_rows(h, s_row, 1, h, 1, 0, 0, 0, 1, None, sp))
                ph, xz = oracle.mul_rows(ph, xz, None, None, s_row, 1, 1, 0)
        side.synchronize()
        g.to_cpu()
        assert np.array_equal(g.xzs, xz) and np.array_equal(g.phases, ph)
    finally:
        check(lib.qcb_tune_set(b"gates_pdl", 1))


def test_single_gate_calls_replayed_from_a_graph(qcb):
    n = 700
    rng = np.random.default_rng(77)
    t = rand_tab(n, n, rng)
    gates = [O.to_array([op]) for op in random_gates(n, 120, rng)]
    lib = qcb.lib()
    g = t.copy().to_gpu()
    h = g._need_dev().handle
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        cs = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        for arr in gates:
            check(lib.qcb_apply_gates(h, ptr(arr), 1, 1, cs))
    ph, xz = t.phases.copy(), t.xzs.copy()
    for _ in range(3):
        graph.replay()
        for arr in gates:
            ph, xz = oracle.apply_gates(ph, xz, n, arr, True)
    torch.cuda.synchronize()
    del graph
    g.to_cpu()
    assert np.array_equal(g.xzs, xz) and np.array_equal(g.phases, ph)
