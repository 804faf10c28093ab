"""qcb_mul_left_pauli_batch_noalloc against the existing qcb_mul_left_pauli.

The no-alloc entry point keeps its phase accumulators in one static device
array that must be zero at every call; each case therefore runs two calls in
a row on fresh data and compares both with the per-pair handle-based entry
point.  The file sorts last so that the static array has also seen every
earlier test's use of the library.
"""
import ctypes

import numpy as np
import pytest

import oracle
from qcb200 import tableau as Q

pytestmark = pytest.mark.gpu


def random_pairs(rng, count, n):
    W = Q.nwords(n)
    xz = rng.integers(0, 2**64, size=(count, W), dtype=np.uint64)
    if n % 64:  # reference padding bits are zero
        pad = np.uint64((1 << (n % 64)) - 1)
        xz[:, W // 2 - 1] &= pad
        xz[:, W - 1] &= pad
    return xz, rng.integers(0, 4, size=count).astype(np.uint8)


def expected(rx, rp, lx, lp, n, phases):
    """The existing entry point, one pair at a time."""
    out_x, out_p = rx.copy(), rp.copy()
    for i in range(len(rp)):
        # copies: a Tableau keeps views of its arrays and mul_left_ writes the phase
        r = Q.Tableau(rp[i:i + 1].copy(), n, rx[i:i + 1].copy()).to_gpu()
        l = Q.Tableau(lp[i:i + 1].copy(), n, lx[i:i + 1].copy()).to_gpu()
        Q.mul_left_(r, l, phases=phases)
        out_p[i:i + 1], out_x[i:i + 1] = r.dev.download()
    return out_x, out_p


def noalloc(qcb, rx, rp, lx, lp, n, phases):
    import torch

    d_rx, d_rp = torch.from_numpy(rx.view(np.int64)).cuda(), torch.from_numpy(rp).cuda()
    d_lx, d_lp = torch.from_numpy(lx.view(np.int64)).cuda(), torch.from_numpy(lp).cuda()
    torch.cuda.synchronize()
    qcb.check(qcb.lib().qcb_mul_left_pauli_batch_noalloc(
        ctypes.c_void_p(d_rx.data_ptr()), ctypes.c_void_p(d_rp.data_ptr()), ctypes.c_void_p(d_lx.data_ptr()),
        ctypes.c_void_p(d_lp.data_ptr()), n, len(rp), int(phases), None))
    torch.cuda.synchronize()
    return d_rx.cpu().numpy().view(np.uint64), d_rp.cpu().numpy()


@pytest.mark.parametrize("n,count,phases", [(1, 5, True), (64, 37, True), (130, 37, True), (3000, 64, True),
                                            (3000, 64, False), (200, 4096, True)])
def test_noalloc_batch_matches_mul_left_pauli_two_calls(qcb, n, count, phases):
    rng = np.random.default_rng(n * 7919 + count)
    for _ in range(2):
        rx, rp = random_pairs(rng, count, n)
        lx, lp = random_pairs(rng, count, n)
        ex, ep = expected(rx, rp, lx, lp, n, phases)
        gx, gp = noalloc(qcb, rx, rp, lx, lp, n, phases)
        assert np.array_equal(gx, ex)
        assert np.array_equal(gp, ep if phases else rp)
        # and pinned to the CPU oracle directly, on the first pairs
        for i in range(min(count, 16)):
            ox, op = oracle.mul_left_pauli(rx[i], rp[i], lx[i], lp[i], phases)
            assert np.array_equal(gx[i], ox) and gp[i] == (op if phases else rp[i])


def test_noalloc_misaligned_words_and_a_side_stream(qcb):
    """Word arrays that start 8 bytes past a 16-byte boundary (even word
    count: the 64-bit load path) and a call on a non-default stream, two
    calls in a row, against the handle-based entry point."""
    import torch

    n, count = 640, 33  # 10 words per half: even
    rng = np.random.default_rng(77)
    side = torch.cuda.Stream()
    for _ in range(2):
        rx, rp = random_pairs(rng, count, n)
        lx, lp = random_pairs(rng, count, n)
        ex, ep = expected(rx, rp, lx, lp, n, True)
        # one spare word in front: the Pauli words start at an 8-byte offset
        d_rx = torch.zeros(rx.size + 1, dtype=torch.int64, device="cuda")
        d_lx = torch.zeros(lx.size + 1, dtype=torch.int64, device="cuda")
        d_rx[1:] = torch.from_numpy(rx.reshape(-1).view(np.int64)).cuda()
        d_lx[1:] = torch.from_numpy(lx.reshape(-1).view(np.int64)).cuda()
        d_rp, d_lp = torch.from_numpy(rp).cuda(), torch.from_numpy(lp).cuda()
        assert (d_rx.data_ptr() + 8) % 16 == 8
        torch.cuda.synchronize()
        qcb.check(qcb.lib().qcb_mul_left_pauli_batch_noalloc(
            ctypes.c_void_p(d_rx.data_ptr() + 8), ctypes.c_void_p(d_rp.data_ptr()), ctypes.c_void_p(d_lx.data_ptr() + 8),
            ctypes.c_void_p(d_lp.data_ptr()), n, count, 1, ctypes.c_void_p(side.cuda_stream)))
        side.synchronize()
        gx = d_rx[1:].cpu().numpy().view(np.uint64).reshape(rx.shape)
        assert np.array_equal(gx, ex) and np.array_equal(d_rp.cpu().numpy(), ep)
        assert int(d_rx[0].item()) == 0  # the spare word is untouched


def test_noalloc_rejects_batches_above_its_scratch(qcb):
    with pytest.raises(qcb.ArgumentError, match="exceeds the no-alloc scratch"):
        qcb.check(qcb.lib().qcb_mul_left_pauli_batch_noalloc(None, None, None, None, 64, 4097, 1, None))
