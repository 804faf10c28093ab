"""GPU tests of the serving loop (qcb_server_*): requests submitted while
others run are admitted as slots and memory free up, overlap on the device
chunk by chunk, and each result is bit-identical alone and in the mix (and to
the plain fresh run of the same request)."""
import threading

import numpy as np
import pytest

from qcb200 import circuits, ops as O

pytestmark = pytest.mark.gpu


def plain_record(qcb, circ, shots, seed):
    prog = qcb.Program(circ)
    qmax, bmax = O.affected_counts(prog.ops)
    f = qcb.PauliFrame(shots, qmax, bmax, init=False)
    qcb.check(qcb.lib().qcb_pftrajectories_fresh(f.handle, prog.handle, seed, 0, None))
    return f.record_planes()


def requests(rng, n, dmax=7, smax=5.3):
    out = []
    for _ in range(n):
        d = int(rng.choice([x for x in (3, 5, 7, 9, 11) if x <= dmax]))
        p = float(10 ** rng.uniform(-4, -2))
        out.append((circuits.rotated_surface_code_memory(d, d, p), int(10 ** rng.uniform(2, smax)),
                    int(rng.integers(0, 2**63))))
    return out


def test_results_same_alone_and_in_the_mix(qcb):
    rng = np.random.default_rng(1)
    reqs = requests(rng, 12)
    srv = qcb.Server(hbm_budget_bytes=8 << 30, slots=4, chunk_shots=8192)
    tickets = [srv.submit(c, s, seed) for c, s, seed in reqs]
    for t in tickets:
        srv.wait(t)
    mixed = [srv.result(t, s) for t, (c, s, seed) in zip(tickets, reqs)]
    for t in tickets:
        srv.release(t)
    # alone: one request at a time through the same server, and the plain launch
    for (c, s, seed), m in zip(reqs[:5], mixed[:5]):
        t = srv.submit(c, s, seed)
        srv.wait(t)
        assert np.array_equal(srv.result(t, s), m)
        srv.release(t)
    for (c, s, seed), m in zip(reqs, mixed):
        assert np.array_equal(plain_record(qcb, c, s, seed), m)
    srv.close()


def test_admission_waits_for_memory_and_keeps_order(qcb):
    rng = np.random.default_rng(2)
    reqs = requests(rng, 6, dmax=5, smax=4.5)
    # a budget that holds about one request at a time
    srv = qcb.Server(hbm_budget_bytes=24 << 20, slots=4, chunk_shots=4096)
    tickets = [srv.submit(c, s, seed) for c, s, seed in reqs]
    admits = []
    for t in tickets:
        srv.wait(t)
        admits.append(srv.query(t)[1][1])
        srv.release(t)  # frees the record: the next one can be admitted
    assert admits == sorted(admits)  # first come, first served
    srv.close()


def test_request_larger_than_budget_fails(qcb):
    srv = qcb.Server(hbm_budget_bytes=1 << 20, slots=2)
    t = srv.submit(circuits.rotated_surface_code_memory(5, 5, 1e-3), 200_000, 1)
    with pytest.raises(qcb.QCBError):
        srv.wait(t)
    srv.release(t)
    srv.close()


def test_submissions_from_many_threads(qcb):
    rng = np.random.default_rng(3)
    reqs = requests(rng, 16, dmax=5, smax=4.0)
    srv = qcb.Server(hbm_budget_bytes=4 << 30, slots=6, chunk_shots=2048)
    tickets = [None] * len(reqs)

    def worker(i):
        c, s, seed = reqs[i]
        tickets[i] = srv.submit(c, s, seed)

    ths = [threading.Thread(target=worker, args=(i,)) for i in range(len(reqs))]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    for t, (c, s, seed) in zip(tickets, reqs):
        srv.wait(t)
        assert np.array_equal(srv.result(t, s), plain_record(qcb, c, s, seed))
        srv.release(t)
    srv.close()


def test_next_done_reports_each_request_once(qcb):
    rng = np.random.default_rng(6)
    reqs = requests(rng, 10, dmax=5, smax=4.0)
    srv = qcb.Server(hbm_budget_bytes=2 << 30, slots=3, chunk_shots=2048)
    tickets = {srv.submit(c, s, seed): (c, s, seed) for c, s, seed in reqs}
    seen = []
    for _ in range(len(reqs)):
        t, st, times = srv.next_done(60.0)
        assert st == 2 and times[0] <= times[1] <= times[2]
        c, s, seed = tickets[t]
        assert np.array_equal(srv.result(t, s), plain_record(qcb, c, s, seed))
        srv.release(t)
        seen.append(t)
    assert sorted(seen) == sorted(tickets)
    with pytest.raises(qcb.QCBError):
        srv.next_done(0.05)  # nothing left to report
    srv.close()


def test_program_cache_compares_ops_on_hash_collisions(qcb):
    """With the cache hash cut to one bit every circuit collides; the byte
    comparison on a hit still gives each request its own program."""
    rng = np.random.default_rng(7)
    reqs = requests(rng, 6, dmax=7, smax=4)
    qcb.check(qcb.lib().qcb_tune_set(b"server_hash_bits", 1))
    try:
        srv = qcb.Server(hbm_budget_bytes=4 << 30, slots=3, chunk_shots=4096)
        tickets = [srv.submit(c, s, seed) for c, s, seed in reqs]
        for t in tickets:
            srv.wait(t)
        got = [srv.result(t, s) for t, (c, s, seed) in zip(tickets, reqs)]
        assert srv.stats()[2] == len({O.to_array(c).tobytes() for c, _, _ in reqs})
        for t in tickets:
            srv.release(t)
        srv.close()
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"server_hash_bits", 0))
    for (c, s, seed), m in zip(reqs, got):
        assert np.array_equal(plain_record(qcb, c, s, seed), m)


def test_programs_count_against_the_budget(qcb):
    """Resident programs are charged to the HBM budget; preloading more than
    fits evicts the least recently used unused ones, and requests still run."""
    circs = [circuits.rotated_surface_code_memory(d, d, p) for d in (9, 11, 13) for p in (1e-3, 2e-3, 3e-3)]
    srv = qcb.Server(hbm_budget_bytes=1 << 20, slots=2, chunk_shots=1024)
    for c in circs:
        srv.preload(c)
        used, prog, n = srv.stats()
        assert used <= 1 << 20 and prog == used and n >= 1
    assert srv.stats()[2] < len(circs)  # some were evicted
    t = srv.submit(circs[0], 2000, 5)
    srv.wait(t)
    assert np.array_equal(srv.result(t, 2000), plain_record(qcb, circs[0], 2000, 5))
    used, prog, _ = srv.stats()
    assert used > prog  # the record is charged while it is held
    srv.release(t)
    assert srv.stats()[0] == srv.stats()[1]
    srv.close()


@pytest.mark.parametrize("fill", [1, 0])
def test_fill_gate_keeps_large_requests_in_order(qcb, fill):
    """server_fill 1: a request behind one whose chunks fill the GPU (2^21
    shots in chunks of whole walker waves near 2^17 shots) waits until that
    one is on its last chunk, which may leave SMs idle; server_fill 0 admits
    it at once.  Records equal the plain runs either way."""
    big = circuits.rotated_surface_code_memory(7, 7, 1e-3)
    small = circuits.rotated_surface_code_memory(3, 3, 1e-3)
    nbig = 16 << 17
    qcb.check(qcb.lib().qcb_tune_set(b"server_fill", fill))
    try:
        srv = qcb.Server(hbm_budget_bytes=8 << 30, slots=4, chunk_shots=1 << 17)
    finally:
        qcb.check(qcb.lib().qcb_tune_set(b"server_fill", 1))
    srv.preload(big)
    srv.preload(small)  # submissions then take no compile time
    tb = srv.submit(big, nbig, 5)
    ts = srv.submit(small, 2000, 6)
    srv.wait(tb)
    srv.wait(ts)
    _, admit_big, done_big = srv.query(tb)[1]
    admit_small = srv.query(ts)[1][1]
    # fill 1 holds the small one for all chunks of the big one but the last,
    # fill 0 lets it in while the first runs
    frac = (admit_small - admit_big) / (done_big - admit_big)
    if fill:
        assert frac > 0.5, frac
    else:
        assert frac < 0.3, frac
    assert np.array_equal(srv.result(tb, nbig), plain_record(qcb, big, nbig, 5))
    assert np.array_equal(srv.result(ts, 2000), plain_record(qcb, small, 2000, 6))
    srv.release(tb)
    srv.release(ts)
    srv.close()
