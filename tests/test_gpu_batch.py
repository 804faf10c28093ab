"""GPU tests of the batched runner (qcb_batch_*): many fresh sampling jobs of
uneven size drained from one persistent launch give, job by job, exactly the
record and frame of the plain launch of that job alone; also under CUDA graph
replay, with explicit or tuned tile widths, and with shot offsets."""
import ctypes

import numpy as np
import pytest

from qcb200 import circuits, ops as O

pytestmark = pytest.mark.gpu


def make_jobs(qcb, rng, n, dmax=9, smax=4.7):
    jobs = []
    for i in range(n):
        d = int(rng.choice([x for x in (3, 5, 7, 9, 11, 13, 15) if x <= dmax]))
        p = float(10 ** rng.uniform(-4, -2))
        shots = int(10 ** rng.uniform(2, smax))
        prog = qcb.Program(circuits.rotated_surface_code_memory(d, d, p))
        qmax, bmax = O.affected_counts(prog.ops)
        seed = int(rng.integers(0, 2**63))
        off = 1024 * int(rng.integers(0, 4))
        jobs.append(dict(prog=prog, shots=shots, q=qmax, b=bmax, seed=seed, off=off))
    return jobs


def plain(qcb, j):
    f = qcb.PauliFrame(j["shots"], j["q"], j["b"], init=False, shot_offset=j["off"])
    qcb.check(qcb.lib().qcb_pftrajectories_fresh(f.handle, j["prog"].handle, j["seed"], j["off"], None))
    return f.record_planes(), f.planes()


def batched_frames(qcb, jobs, tiles=None):
    frames = [qcb.PauliFrame(j["shots"], j["q"], j["b"], init=False, shot_offset=j["off"]) for j in jobs]
    spec = [(f, j["prog"], j["seed"], j["off"], (tiles[i] if tiles else 0)) for i, (f, j) in enumerate(zip(frames, jobs))]
    return frames, qcb.Batch(spec)


def assert_same(qcb, frames, jobs):
    for f, j in zip(frames, jobs):
        rec, (x, z) = plain(qcb, j)
        x2, z2 = f.planes()
        assert np.array_equal(f.record_planes(), rec)
        assert np.array_equal(x2, x) and np.array_equal(z2, z)


def test_batch_equals_plain_launches(qcb):
    rng = np.random.default_rng(1)
    jobs = make_jobs(qcb, rng, 24)
    frames, b = batched_frames(qcb, jobs)
    b.run().status()
    assert_same(qcb, frames, jobs)


def test_batch_tile_widths_do_not_change_results(qcb):
    rng = np.random.default_rng(2)
    jobs = make_jobs(qcb, rng, 8, dmax=7)
    tiles = [16, 40, 106, 64, 18, 128, 32, 200]
    frames, b = batched_frames(qcb, jobs, tiles)
    b.run().status()
    assert_same(qcb, frames, jobs)


def test_batch_graph_replay_and_tuner(qcb):
    import torch

    rng = np.random.default_rng(3)
    jobs = make_jobs(qcb, rng, 12, dmax=11, smax=4.2)
    t, us = qcb.tune_tile(jobs[0]["prog"])
    assert 16 <= t <= 256 and t % 2 == 0 and us > 0
    frames, b = batched_frames(qcb, jobs)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.run(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    for _ in range(2):  # every replay is a fresh run of every job
        g.replay()
        torch.cuda.synchronize()
        b.status()
        assert_same(qcb, frames, jobs)
    del g


def test_batch_rejects_bad_jobs(qcb):
    rng = np.random.default_rng(4)
    jobs = make_jobs(qcb, rng, 1, dmax=3)
    f = qcb.PauliFrame(jobs[0]["shots"], jobs[0]["q"], jobs[0]["b"], init=False)
    with pytest.raises(qcb.QCBError):
        qcb.Batch([(f, jobs[0]["prog"], 1, 100)])  # shot_offset not a multiple of 1024
    with pytest.raises(qcb.QCBError):
        qcb.Batch([(f, jobs[0]["prog"], 1, 0, 7)])  # odd tile
    small = qcb.PauliFrame(100, 2, 1, init=False)
    with pytest.raises(qcb.QCBError):
        qcb.Batch([(small, jobs[0]["prog"], 1, 0)])  # the program needs more qubits
    assert qcb.Batch([]).run().status() is not None


@pytest.mark.parametrize("cluster", [0, 8, 16])
def test_canonicalize_batch_equals_single(qcb, cluster):
    import oracle
    from test_gpu_tableau import dev_random_destabilizer
    from qcb200.tableau import Tableau

    rng = np.random.default_rng(5 + cluster)
    srcs, states = [], []
    for k in range(24):
        n = int(rng.integers(10, 700)) if k % 8 else int(rng.integers(1800, 2600))  # some with rows in global memory
        d = dev_random_destabilizer(qcb, n, rng, depth=8)
        rows = n if k % 3 else max(1, n // 2)
        t = Tableau(d.tab.phases[n:n + rows].copy(), n, d.tab.xzs[n:n + rows].copy())
        srcs.append(t)
        states.append(qcb.Stabilizer(t.copy()).to_gpu())
    b = qcb.CanonBatch(states, cluster=cluster)
    b.run()
    ranks = b.ranks()
    for st, t, (rx, rz) in zip(states, srcs, ranks):
        st.to_cpu()
        ph, xz, orx, orz = oracle.canonicalize(t.phases, t.xzs, t.nqubits, True)
        assert (rx, rz) == (orx, orz)
        assert np.array_equal(st.tab.xzs, xz) and np.array_equal(st.tab.phases, ph)
    # a canonical tableau is a fixed point: running the batch again changes nothing
    b.run()
    assert b.ranks() == ranks
    for st in states:
        before = st.tab.xzs.copy()
        st.to_cpu()
        assert np.array_equal(st.tab.xzs, before)


def test_batch_with_a_tall_program_in_16k_windows(qcb):
    """A d=25 job (16 KB program windows) in one batch with small jobs
    (8 KB windows): the staging buffers take the larger size, every job
    still equals its plain launch."""
    rng = np.random.default_rng(25)
    jobs = make_jobs(qcb, rng, 5, dmax=5, smax=3.5)
    prog = qcb.Program(circuits.rotated_surface_code_memory(25, 2, 0.01))
    qmax, bmax = O.affected_counts(prog.ops)
    jobs.insert(2, dict(prog=prog, shots=2100, q=qmax, b=bmax, seed=77, off=2048))
    frames, b = batched_frames(qcb, jobs)
    b.run().status()
    assert_same(qcb, frames, jobs)
