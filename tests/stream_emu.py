"""A NumPy interpreter of the device program (test infrastructure).

Runs the record stream that qcb_program_compile produces (dumped on the host
with qcb_debug_program_dump, no GPU involved) in mask mode, one uint32 word
per 32-shot column, with the same record semantics as the walker kernel.
Comparing it with the oracle checks the compiler (segmentation, relabels,
flush placement, reset grouping) on the CPU; the GPU tests then check the
kernel against the same oracle.
"""
from __future__ import annotations

import ctypes

import numpy as np

import qcb200
from qcb200 import ops as O
from qcb200._lib import check, lib, ptr, qcb_program_info

SEG_END, SEG_CNOT, SEG_H, SEG_S, SEG_G1, SEG_G2, SEG_MZ, SEG_MRZ, SEG_FLUSH, SEG_CZ, SEG_WIN, SEG_XOR = range(12)
BIT_NONE = 0xFFFFFFFF
MRZ_PAD = 0xFFFFFFFF
SITE_DTYPE = np.dtype([("kind", "<u4"), ("xa", "<u4"), ("za", "<u4"), ("xb", "<u4"), ("zb", "<u4"),
                       ("dense", "<u4"), ("pad", "<u4", (2,)), ("t", "<f8", (3,)), ("peff", "<f8"), ("q0", "<f8"),
                       ("r", "<f8")])
assert SITE_DTYPE.itemsize == 80


def dump(arr):
    L = lib()
    a = O.to_array(arr)
    sl, ns, nsl = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
    info = qcb_program_info()
    aptr = ptr(a) if len(a) else None
    check(L.qcb_debug_program_dump(aptr, len(a), None, 0, ctypes.byref(sl), None, 0, ctypes.byref(ns), None, None, 0,
                                   ctypes.byref(nsl), ctypes.byref(info)))
    stream = np.zeros(max(sl.value, 1), np.uint32)
    sites = np.zeros(max(ns.value, 1), SITE_DTYPE)
    sq = np.zeros(max(nsl.value, 1), np.uint32)
    sw = np.zeros(max(nsl.value, 1), np.uint32)
    check(L.qcb_debug_program_dump(aptr, len(a), ptr(stream), len(stream), ctypes.byref(sl), ptr(sites.view(np.uint8)),
                                   sites.nbytes, ctypes.byref(ns), ptr(sq), ptr(sw), len(sq), ctypes.byref(nsl),
                                   ctypes.byref(info)))
    return stream[: sl.value], sites[: ns.value], sq[: nsl.value], sw[: nsl.value], {f: getattr(info, f) for f, _ in info._fields_}


def gate1(op, x, z):
    X, Z = x.copy(), z.copy()
    if (op & 0xFF) == O.OP["SQO"]:
        f = op >> 8
        m = lambda b: np.uint32(0xFFFFFFFF if (f >> b) & 1 else 0)
        return (X & m(0)) ^ (Z & m(2)), (X & m(1)) ^ (Z & m(3))
    if op in (O.OP["H"], O.OP["SQRTY"], O.OP["INVSQRTY"]):
        return Z, X
    if op in (O.OP["HXY"], O.OP["S"], O.OP["SDAG"]):
        return X, X ^ Z
    if op in (O.OP["HYZ"], O.OP["SQRTX"], O.OP["INVSQRTX"]):
        return X ^ Z, Z
    if op == O.OP["CXYZ"]:
        return X ^ Z, X
    if op == O.OP["CZYX"]:
        return Z, X ^ Z
    return X, Z


def gate2(op, a, b, c, d):
    n = {k: v for k, v in O.OP.items()}
    if op == n["SWAP"]:
        return c, d, a, b
    if op in (n["CNOT"], n["ZCX"]):
        return a, b ^ d, c ^ a, d
    if op in (n["CPHASE"], n["ZCZ"]):
        return a, b ^ c, c, d ^ a
    if op == n["ZCY"]:
        return a, c ^ b ^ d, c ^ a, d ^ a
    if op == n["XCX"]:
        return d ^ a, b, c ^ b, d
    if op == n["XCY"]:
        return a ^ c ^ d, b, b ^ c, d ^ b
    if op == n["XCZ"]:
        return a ^ c, b, c, d ^ b
    if op == n["YCX"]:
        return a ^ d, d ^ b, a ^ b ^ c, d
    if op == n["YCY"]:
        return a ^ d ^ c, b ^ c ^ d, a ^ c ^ b, a ^ b ^ d
    if op == n["YCZ"]:
        return a ^ c, c ^ b, c, d ^ a ^ b
    if op == n["SWAPCX"]:
        return c, d ^ b, c ^ a, b
    if op in (n["INVSWAPCX"], n["CXSWAP"]):
        return c ^ a, d, a, d ^ b
    if op in (n["ISWAP"], n["INVISWAP"]):
        return c, a ^ d ^ c, a, a ^ c ^ b
    if op == n["CZSWAP"]:
        return c, d ^ a, a, c ^ b
    if op in (n["ZCRY"], n["INVZCRY"]):
        return a, a ^ b ^ c ^ d, a ^ c, a ^ d
    if op in (n["SQRTZZ"], n["INVSQRTZZ"]):
        return a, a ^ c ^ b, c, a ^ d ^ c
    if op in (n["SQRTXX"], n["INVSQRTXX"]):
        return b ^ d ^ a, b, b ^ c ^ d, d
    if op in (n["SQRTYY"], n["INVSQRTYY"]):
        return b ^ c ^ d, a ^ d ^ c, a ^ b ^ d, a ^ c ^ b
    raise ValueError(op)


def run_mask(arr, frames, qubits, nbits, masks):
    """Returns (x planes, z planes, record planes) as uint32 [n, words]."""
    stream, sites, sq, sw, info = dump(arr)
    words = (frames + 31) // 32
    nslots = len(sq) if info["nqubits"] else 0
    nq1 = qubits + 1
    X = np.zeros((nq1, words), np.uint32)
    Z = np.array(masks.init_z, dtype=np.uint32, copy=True)
    T = np.zeros((2 * max(nslots, 1), words), np.uint32)  # tile planes
    for s in range(nslots):
        T[2 * s] = X[sq[s]]
        T[2 * s + 1] = Z[sq[s]]
    rec = np.zeros((max(nbits, 1), words), np.uint32)
    # events bucketed by site
    a = O.to_array(arr)
    site_of_op = np.cumsum(np.isin(a["opcode"], [O.OP["PAULI_NOISE"], O.OP["DEPOL1"], O.OP["DEPOL2"]])) - 1
    ev_by_site = {}
    for e in masks.events:
        s = int(site_of_op[int(e["op_index"])])
        ev_by_site.setdefault(s, []).append((int(e["shot"]), int(e["pauli"])))
    WIN = 2048
    lo16 = lambda v: int(v) & 0xFFFF
    hi16 = lambda v: int(v) >> 16
    pc = 0
    while True:
        h = stream[pc: pc + 4]
        pc += 4
        kind, cnt = int(h[0]) >> 24, int(h[0]) & 0xFFFFFF
        if kind == SEG_END:
            break
        if kind == SEG_WIN:  # its count is the program's window size
            win = cnt or WIN
            pc = (pc - 4) // win * win + win
            continue
        if kind in (SEG_CNOT, SEG_CZ):
            e = stream[pc: pc + 2 * cnt].reshape(cnt, 2)
            pc += (2 * cnt + 3) // 4 * 4
            for a_, b_ in e:
                xa, za, xb, zb = lo16(a_), hi16(a_), lo16(b_), hi16(b_)
                if kind == SEG_CNOT:
                    T[xb] ^= T[xa]
                    T[za] ^= T[zb]
                else:
                    T[za] ^= T[xb]
                    T[zb] ^= T[xa]
        elif kind in (SEG_S, SEG_G1):
            e = stream[pc: pc + 2 * cnt].reshape(cnt, 2)
            pc += (2 * cnt + 3) // 4 * 4
            for a_, op in e:
                x, z = lo16(a_), hi16(a_)
                if kind == SEG_S:
                    T[z] ^= T[x]
                else:
                    T[x], T[z] = gate1(int(op), T[x], T[z])
        elif kind == SEG_G2:
            e = stream[pc: pc + 4 * cnt].reshape(cnt, 4)
            pc += 4 * cnt
            for a_, b_, op, _ in e:
                xa, za, xb, zb = lo16(a_), hi16(a_), lo16(b_), hi16(b_)
                T[xa], T[za], T[xb], T[zb] = gate2(int(op), T[xa].copy(), T[za].copy(), T[xb].copy(), T[zb].copy())
        elif kind == SEG_MZ:
            e = stream[pc: pc + 2 * cnt].reshape(cnt, 2)
            pc += (2 * cnt + 3) // 4 * 4
            for x, bit in e:
                rec[bit] = T[x]
        elif kind == SEG_MRZ:
            e = stream[pc: pc + 16 * cnt].reshape(cnt * 4, 4)
            pc += 16 * cnt
            for a_, bit, r, _ in e:
                if r == MRZ_PAD:
                    continue
                x, z = lo16(a_), hi16(a_)
                if bit != BIT_NONE:
                    rec[bit] = T[x]
                T[x] = 0
                T[z] ^= masks.reset_planes[r]
        elif kind == SEG_XOR:
            e = stream[pc: pc + 32 * cnt].reshape(cnt, 32)
            pc += 32 * cnt
            for row in e:
                v = np.zeros(words, np.uint32)
                for b in row[2: 2 + int(row[1])]:
                    v ^= rec[b]
                rec[row[0]] = v
        elif kind == SEG_FLUSH:
            e = stream[pc: pc + 4 * cnt].reshape(cnt, 4)
            pc += 4 * cnt
            for site, kc, pa, pb in e:
                for shot, code in ev_by_site.get(int(site), []):
                    w, b = shot >> 5, np.uint32(1 << (shot & 31))
                    if code & 1:
                        T[lo16(pa), w] ^= b
                    if code & 2:
                        T[hi16(pa), w] ^= b
                    if (int(kc) & 0xFF) == O.OP["DEPOL2"]:
                        if code & 4:
                            T[lo16(pb), w] ^= b
                        if code & 8:
                            T[hi16(pb), w] ^= b
        else:
            raise ValueError(f"unknown record kind {kind}")
    for s in range(nslots):
        X[sq[s]] = T[2 * s + sw[s]]
        Z[sq[s]] = T[2 * s + 1 - sw[s]]
    return X, Z, rec[:nbits], info


def planes_to_xzs(X, Z, frames):
    """Shot-packed planes -> reference fastcolumn xzs (W' x frames)."""
    nq1 = X.shape[0]
    wp = 2 * ((nq1 + 63) // 64)
    half = wp // 2
    out = np.zeros((wp, frames), np.uint64)
    f = np.arange(frames)
    for q in range(nq1):
        xb = ((X[q, f >> 5] >> (f & 31).astype(np.uint32)) & 1).astype(np.uint64)
        zb = ((Z[q, f >> 5] >> (f & 31).astype(np.uint32)) & 1).astype(np.uint64)
        out[q >> 6] |= xb << np.uint64(q & 63)
        out[half + (q >> 6)] |= zb << np.uint64(q & 63)
    return out
