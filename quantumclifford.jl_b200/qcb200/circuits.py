"""Circuit generators for the benchmark workloads, in the reference's op vocabulary.

repetition_code_memory:    distance-d repetition-code memory (d data + d-1
                           ancillas, d rounds), noise PauliError on the data
                           at the start of every round (the pattern of
                           src/ecc/decoder_pipeline.jl:103-104).
rotated_surface_code_memory: rotated surface code, memory-Z.  The reference
                           has no rotated-code generator (its Surface code is
                           the unrotated one, lib/QECCore/src/codes/quantum/
                           surface.jl:36-64); this one is written from the
                           standard layout.
"""
from __future__ import annotations

from . import ops as O


def repetition_code_memory(d: int = 7, rounds: int = 7, p: float = 1e-3) -> list:
    """Data qubits 1..d, ancillas d+1..2d-1.  Per round: PauliError(j, p) on
    every data qubit, sCNOT(i, d+i) and sCNOT(i+1, d+i) layers, sMRZ of the
    ancillas; then sMZ of the data.  Records: rounds*(d-1) + d bits."""
    c = []
    na = d - 1
    for r in range(rounds):
        for j in range(1, d + 1):
            c += O.PauliError(j, p)
        for i in range(1, na + 1):
            c.append(O.sCNOT(i, d + i))
        for i in range(1, na + 1):
            c.append(O.sCNOT(i + 1, d + i))
        for i in range(1, na + 1):
            c.append(O.sMRZ(d + i, na * r + i))
    for j in range(1, d + 1):
        c.append(O.sMZ(j, na * rounds + j))
    return c


def rotated_surface_code_layout(d: int):
    """Plaquettes of the rotated surface code.

    Data qubit (r, c), 0 <= r, c < d, is qubit r*d + c + 1.  Plaquette (i, j),
    0 <= i, j <= d, touches the data at (i-1, j-1) NW, (i-1, j) NE,
    (i, j-1) SW, (i, j) SE that exist.  Type X when i + j is even, else Z.
    Bulk plaquettes (1 <= i, j <= d-1) all exist; weight-2 boundary
    plaquettes exist for X on the top/bottom rows and for Z on the left/right
    columns.  Returns a list of (type, i, j, {corner: data qubit}).
    """
    plaq = []
    for i in range(d + 1):
        for j in range(d + 1):
            t = "X" if (i + j) % 2 == 0 else "Z"
            bulk = 1 <= i <= d - 1 and 1 <= j <= d - 1
            top_bottom = (i == 0 or i == d) and 1 <= j <= d - 1
            left_right = (j == 0 or j == d) and 1 <= i <= d - 1
            if not (bulk or (top_bottom and t == "X") or (left_right and t == "Z")):
                continue
            corners = {}
            for name, (di, dj) in (("NW", (-1, -1)), ("NE", (-1, 0)), ("SW", (0, -1)), ("SE", (0, 0))):
                r, cc = i + di, j + dj
                if 0 <= r < d and 0 <= cc < d:
                    corners[name] = r * d + cc + 1
            plaq.append((t, i, j, corners))
    return plaq


X_ORDER = ("NW", "NE", "SW", "SE")
Z_ORDER = ("NW", "SW", "NE", "SE")


def rotated_surface_code_memory(d: int = 11, rounds: int | None = None, p: float = 1e-3) -> list:
    """Memory-Z rotated surface code: d*d data, d*d-1 ancillas (X ancillas
    first).  Per round: sHadamard on X ancillas each followed by
    PauliError(a, p); four sCNOT layers in N/Z order (X check: ancilla ->
    data, Z check: data -> ancilla), each CNOT followed by two-qubit
    depolarising noise of error probability p; sHadamard on the X ancillas
    plus PauliError(a, p); measurement flips PauliError(a, p, 0, 0) and sMRZ
    on every ancilla.  Finally sMZ of all data.  Records: rounds*(d*d-1)+d*d."""
    rounds = d if rounds is None else rounds
    plaq = rotated_surface_code_layout(d)
    xs = [pq for pq in plaq if pq[0] == "X"]
    zs = [pq for pq in plaq if pq[0] == "Z"]
    order = xs + zs
    nd = d * d
    anc = {id(pq): nd + k + 1 for k, pq in enumerate(order)}
    xanc = [anc[id(pq)] for pq in xs]
    allanc = [anc[id(pq)] for pq in order]
    dep = O.DepolarizationNoise.from_two_qubit_error_probability(p)
    c = []
    na = len(order)
    for r in range(rounds):
        for a in xanc:
            c.append(O.sHadamard(a))
            c += O.PauliError(a, p)
        for layer in range(4):
            for pq in order:
                t, _, _, corners = pq
                key = (X_ORDER if t == "X" else Z_ORDER)[layer]
                if key not in corners:
                    continue
                a, q = anc[id(pq)], corners[key]
                if t == "X":
                    c.append(O.sCNOT(a, q))
                    c += O.NoiseOp(dep, (a, q))
                else:
                    c.append(O.sCNOT(q, a))
                    c += O.NoiseOp(dep, (q, a))
        for a in xanc:
            c.append(O.sHadamard(a))
            c += O.PauliError(a, p)
        for k, a in enumerate(allanc):
            c += O.PauliError(a, p, 0, 0)
            c.append(O.sMRZ(a, na * r + k + 1))
    for q in range(1, nd + 1):
        c.append(O.sMZ(q, na * rounds + q))
    return c


def surface_code_detector_bits(d: int, rounds: int | None = None, basis: str = "Z") -> list:
    """Detectors of the memory-Z circuit as lists of 0-based record bits whose
    XOR is the detector.

    basis "Z": per Z ancilla its first-round outcome, the XOR of consecutive
    rounds, and the last round against the data parity of its plaquette
    (deterministic in the noiseless circuit).  basis "X": per X ancilla the
    XOR of consecutive rounds (rounds 2..rounds; the first-round X outcome is
    random in a memory-Z experiment and the data are not measured in X).
    basis "X1": the first-round X outcomes alone (rate 1/2)."""
    rounds = d if rounds is None else rounds
    plaq = rotated_surface_code_layout(d)
    xs = [pq for pq in plaq if pq[0] == "X"]
    zs = [pq for pq in plaq if pq[0] == "Z"]
    na = len(xs) + len(zs)
    dets = []
    if basis == "Z":
        for k, pq in enumerate(zs):
            col = len(xs) + k
            dets.append([col])
            for r in range(1, rounds):
                dets.append([na * (r - 1) + col, na * r + col])
            dets.append([na * (rounds - 1) + col] + [na * rounds + q - 1 for q in pq[3].values()])
    elif basis == "X":
        for col in range(len(xs)):
            for r in range(1, rounds):
                dets.append([na * (r - 1) + col, na * r + col])
    elif basis == "X1":
        dets = [[col] for col in range(len(xs))]
    else:
        raise ValueError("basis must be 'Z', 'X' or 'X1'")
    return dets


def surface_code_detectors(record, d: int, rounds: int | None = None, basis: str = "Z"):
    """Detectors (surface_code_detector_bits) of the memory-Z circuit from a
    Bool record matrix (frames x bits).  Returns an int8 matrix frames x
    n_detectors."""
    import numpy as np

    rec = np.asarray(record, dtype=np.int8)
    dets = []
    for bits in surface_code_detector_bits(d, rounds, basis):
        v = rec[:, bits[0]].copy()
        for b in bits[1:]:
            v ^= rec[:, b]
        dets.append(v)
    return np.stack(dets, axis=1)


def detector_counts_from_planes(planes, frames: int, detectors: list):
    """Number of shots in which each detector fires, from shot-packed record
    planes (uint32 [nbits, words], bit s%32 of word s//32 = shot s).  Padding
    shots of the last word are masked off."""
    import numpy as np

    planes = np.asarray(planes, dtype=np.uint32)
    words = (frames + 31) // 32
    mask = np.full(words, 0xFFFFFFFF, dtype=np.uint32)
    if frames % 32:
        mask[-1] = np.uint32((1 << (frames % 32)) - 1)
    out = np.zeros(len(detectors), dtype=np.int64)
    for i, bits in enumerate(detectors):
        v = planes[bits[0], :words].copy()
        for b in bits[1:]:
            v ^= planes[b, :words]
        v &= mask
        out[i] = int(np.unpackbits(v.view(np.uint8)).sum())
    return out
