#!/usr/bin/env python3
"""Benchmark: Pauli-frame sampling of the d=11 rotated surface-code memory
circuit (121 data + 120 ancillas, 11 rounds, p = 1e-3 two-qubit
depolarising / single-qubit / measurement-flip noise), 1,000,000 shots per
GPU, one plain circuit launch per step.

Metric: frame-gate updates/s = (Clifford + measurement ops per shot, 7,601)
x shots / step time.  A step is one pftrajectories(circuit; trajectories)
over the shots: a fresh frame (initZ! from Philox) through the whole circuit,
the record and the final frame written to HBM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): shots are sharded by rank (weak scaling; each rank's
Philox counters use its global shot offset, so the union equals one big
run); there is no collective in the timed region.  Rank 0 prints one JSON
line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "quantumclifford.jl_b200"))

D = 11
ROUNDS = 11
P_NOISE = 1e-3
SHOTS_PER_GPU = 1_000_000
METRIC = "frame-gate updates/s, d=11 surface code"
UNIT = "updates/s"
WORKLOAD = "rotated surface-code memory d=11, 11 rounds, p=1e-3, 1e6 shots per GPU, plain one-circuit launch"

# Model bytes: the plane traffic an op-per-launch schedule must move (bits
# per shot read + written: CNOT 6, H 4, sMRZ 5, sMZ 2, initZ 1 per qubit):
# 11*(120*4 + 440*6 + 120*5) + 121*2 + 241 = 41,403 bits per shot.
MODEL_BITS_PER_SHOT = 11 * (120 * 4 + 440 * 6 + 120 * 5) + 121 * 2 + 241
# Compulsory HBM traffic of the fused kernel per shot: the record
# (1,441 bits) and the final frame (242 qubits x 2 bits).
RECORD_BITS = 11 * 120 + 121
FRAME_BITS = 2 * 242


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if "hbm_gbs" in d:
            return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6650 GB/s (no measured hbm_gbs in MEASURED_PEAKS.json)"


def clocks_snapshot(device_index: int = 0):
    """One nvidia-smi reading of the SM clock, its maximum and the throttle
    reasons (the launch-bound tableau timings are read right after their timed
    region: a sampler polling during a call of hundreds of launches stalls the
    launching thread and shows up as idle device time)."""
    try:
        r = subprocess.run(["nvidia-smi", "-i", str(device_index), f"--query-gpu={ClockSampler.FIELDS}",
                            "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=20)
    except (FileNotFoundError, subprocess.TimeoutExpired):
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "when": "after"}
    parts = [p.strip() for p in r.stdout.strip().split(",")]
    if len(parts) < 9:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unreadable"], "when": "after"}
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        sm, mx = float(parts[1]), float(parts[2])
    except ValueError:
        sm = mx = None
    return {"sm_mhz": sm, "sm_max_mhz": mx, "reasons": [nm for nm, v in zip(names, parts[5:9]) if v == "Active"],
            "when": "right after the timed calls"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _reference_circuit():
    from qcb200 import circuits, ops as O

    arr = O.to_array(circuits.rotated_surface_code_memory(D, ROUNDS, P_NOISE))
    qmax, bmax = O.affected_counts(arr)
    return arr, qmax, bmax, O.count_updates(arr)


def cpu_reference_step(arr, qmax, bmax, shots, seed, cores):
    """One step of the CPU path at the full configuration: the oracle port of
    pftrajectories(circuit; trajectories=shots, threads=true)
    (src/pauli_frames.jl:193-227: _create_pauliframe, initZ!, one pass over
    all frames per op, one rand() per frame per noise site, threads over frame
    slices, nthr = min(cores, shots / 100)), the frame and the Bool record
    (the reference's column-major Matrix{Bool}, 1.44 GB at 1e6 shots)
    allocated by the step as the reference allocates them.  Returns seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the checker, used here only as the timed CPU path

    t0 = time.perf_counter()
    xzs, meas = oracle.pftrajectories_rng(arr, shots, qmax, bmax, seed=seed, threads=cores, as_bool=False)
    dt = time.perf_counter() - t0
    del xzs, meas
    return dt


def cpu_baseline_run(shots: int = SHOTS_PER_GPU):
    """The oracle port timed on the host cores over the same workload as the
    GPU step (all 1e6 shots of the d=11 circuit): one untimed step on a
    small slice (pages the library in), then one full step."""
    arr, qmax, bmax, upd = _reference_circuit()
    cores = os.cpu_count() or 1
    cpu_reference_step(arr, qmax, bmax, min(shots, 20_000), 1, cores)
    dt = cpu_reference_step(arr, qmax, bmax, shots, 2, cores)
    threads = max(1, min(cores, shots // 100))
    return {"value": upd * shots / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"the full step: {shots} shots of the d=11 circuit (Xoshiro per-frame draws, Bool record "
                      f"allocated per step as the reference does), {dt:.2f} s wall on {threads} threads"}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (its Julia code cannot run
    here: no Julia; the oracle port restates it loop for loop) on all host
    cores, every step the full configuration (1e6 shots of the d=11
    circuit), W untimed then K timed steps, wall-clock per step."""
    if rank != 0:
        return
    arr, qmax, bmax, upd = _reference_circuit()
    cores = os.cpu_count() or 1
    threads = max(1, min(cores, SHOTS_PER_GPU // 100))
    times = []
    for i in range(args.warmup + args.steps):
        dt = cpu_reference_step(arr, qmax, bmax, SHOTS_PER_GPU, 1000 + i, cores)
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    v = upd * SHOTS_PER_GPU * len(times) / total
    sample = (f"every step the full configuration: {SHOTS_PER_GPU} shots of the d=11 circuit, Bool record "
              f"({SHOTS_PER_GPU * bmax / 1e9:.2f} GB) allocated per step; {threads} threads; step times "
              f"{min(times):.2f}-{max(times):.2f} s")
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": total / len(times) * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u64 qubit-packed frame words (the reference layout)",
           "data": "synthetic (seeded)", "impl": "reference",
           "config": {"workload": WORKLOAD, "shots_per_step": SHOTS_PER_GPU, "updates_per_shot": upd,
                      "path": "oracle port of pftrajectories(circuit; trajectories, threads=true); the Julia "
                              "reference cannot be installed or run here"},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# Published single-thread reference times (README of the reference, Ryzen 9
# 7950X, Julia 1.9.1), the denominators of vs_baseline for the tableau lines.
REF_MS = {"mul_left": 13.355, "canonicalize_1000": 8.536, "dense_apply": 17.010,
          "sCNOT": 3.043e-3, "project": 21.971e-3}


def bench_tableau(args):
    """Config-3 tableau kernels, one JSON line each: device time per call
    (CUDA events around the call only; state copies happen outside), the
    result checked against the oracle on the same input, and the oracle
    single-threaded on the host as cpu_baseline.  Random states are uniformly
    random stabilizer states (Bravyi-Maslov sampler, seeded)."""
    import torch
    import numpy as np
    import qcb200
    from qcb200 import tableau as Q
    from qcb200._lib import check, lib, ptr

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the checker and the timed CPU baseline only

    qcb200.ensure_init(0)
    L = lib()
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    peak, peak_kind = load_peaks()
    rng = np.random.default_rng(2024)

    def device_ms(fn, reps, setup=None, warm=3, warm_s=0.25):
        # warm-up: at least `warm` calls and `warm_s` seconds of them, so that
        # the SM clock is back up after the host-only oracle runs in between
        ts = []
        t0 = time.perf_counter()
        i = 0
        while i < warm or (time.perf_counter() - t0 < warm_s and i < 400):
            if setup:
                setup()
            fn()
            torch.cuda.synchronize()
            i += 1
        for _ in range(reps):
            if setup:
                setup()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        last_clocks[0] = clocks_snapshot(0)
        last_spread[0] = {"reps": len(ts), "min_ms": min(ts), "median_ms": statistics.median(ts), "max_ms": max(ts)}
        return statistics.median(ts)

    def cpu_ms(fn, reps=3):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t0) * 1e3)
        return statistics.median(ts)

    lines = []  # printed at the end
    last_clocks = [None]  # the clocks read right after the last timed region
    last_spread = [None]  # min / median / max of the last timed region's calls

    def emit(metric, key, ms, config, cpu, extra=None):
        out = {"metric": metric, "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": 3,
               "ms_per_step": ms, "higher_is_better": False, "scaling": "none",
               "vs_baseline": (ms / REF_MS[key]) if key in REF_MS else None, "dtype": "u64 bit rows + u8 phases",
               "data": "synthetic (seeded)", "config": config, "gpu_launches": None,
               "cpu_baseline": {"value": cpu, "unit": "ms", "cores": 1, "kind": "port",
                                "sample": "the oracle on the same input, one thread"}}
        out["clocks"] = last_clocks[0]
        out["spread"] = last_spread[0]
        if extra:
            out.update(extra)
        lines.append(out)

    only = set(x for x in (args.tableau_only or "").split(",") if x)

    def want(name):
        return not only or name in only

    def random_destabilizer(n):
        # uniformly random (Bravyi-Maslov), as random_destabilizer(n) in the reference
        return qcb200.random_destabilizer(n, rng)

    if want("mul_left"):
        # ---- mul_left! of two 1e9-qubit Paulis (HBM: read 2 x 250 MB, write 250 MB)
        n = 10**9
        W = Q.nwords(n)
        rx = rng.integers(0, 2**64, size=(1, W), dtype=np.uint64)
        lx = rng.integers(0, 2**64, size=(1, W), dtype=np.uint64)
        r = Q.Tableau(np.array([1], np.uint8), n, rx).to_gpu()
        l = Q.Tableau(np.array([2], np.uint8), n, lx).to_gpu()
        ms = device_ms(lambda: check(L.qcb_mul_left_pauli(r.dev.handle, l.dev.handle, 1, None, sp)), args.steps)
        # correctness of one call against the oracle on a 1e8-qubit slice (X and Z halves)
        m = 10**8
        Wm = Q.nwords(m)
        a = Q.Tableau(np.array([1], np.uint8), m, rx[:, :Wm].copy()).to_gpu()
        b = Q.Tableau(np.array([2], np.uint8), m, lx[:, :Wm].copy()).to_gpu()
        Q.mul_left_(a, b)
        a.to_cpu()
        ox, oph = oracle.mul_left_pauli(rx[0, :Wm], 1, lx[0, :Wm], 2)
        assert np.array_equal(a.xzs[0], ox) and int(a.phases[0]) == oph
        cpu = cpu_ms(lambda: oracle.mul_left_pauli(rx[0, :Wm], 1, lx[0, :Wm], 2)) * (n / m)
        traffic = 3 * W * 8
        emit("mul_left! of two 1e9-qubit Paulis", "mul_left", ms,
             {"workload": "mul_left! r <- l * r, n = 1e9 qubits (250 MB per Pauli), phases on", "l2": "750 MB > L2"},
             cpu, {"roofline": {"bound": "hbm", "achieved": traffic / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                "frac": traffic / (ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
                                "algorithmic_bytes_per_launch": traffic}})
        del r, l, a, b

    if want("canonicalize"):
        # ---- canonicalize! of random full-rank stabilizers
        sizes = [int(x) for x in args.canon_sizes.split(",") if x] if args.canon_sizes else [1000, 2000, 4000]
        for n in sizes:
            d = random_destabilizer(n)
            src = Q.Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
            work = Q.Tableau(src.phases.copy(), n, src.xzs.copy()).to_gpu()
            pristine = Q.DeviceTableau(n, n)
            pristine.upload(src.phases, src.xzs)
            ms = device_ms(lambda: check(L.qcb_canonicalize(work.dev.handle, 1, n, 1, None, None, sp)), args.steps,
                           setup=lambda: check(L.qcb_tableau_copy(work.dev.handle, pristine.handle, sp)))
            work.to_cpu()
            oph, oxz, _, _ = oracle.canonicalize(src.phases, src.xzs, n)
            assert np.array_equal(work.xzs, oxz) and np.array_equal(work.phases, oph)
            cpu = cpu_ms(lambda: oracle.canonicalize(src.phases, src.xzs, n), reps=1 if n > 2000 else 3)
            emit(f"canonicalize! of a random {n}-qubit stabilizer", f"canonicalize_{n}", ms,
                 {"workload": f"canonicalize!(random_stabilizer({n})), phases on", "rows": n}, cpu)

    if want("project"):
        # ---- project! of 1000 random Paulis (weight ~ U{1..n}) in sequence on
        # random_stabilizer(n), n = 1000 / 2000 / 4000 (Stabilizer kind: the
        # commuting branch runs canonicalize! + generate!), and on a random
        # 1000-qubit Destabilizer (the README's case)
        k = 1000
        for kind, n in (("Stabilizer", 1000), ("Stabilizer", 2000), ("Stabilizer", 4000), ("Destabilizer", 1000)):
            d = random_destabilizer(n)
            if kind == "Stabilizer":
                ph0, xz0 = d.tab.phases[n:].copy(), d.tab.xzs[n:].copy()
            else:
                ph0, xz0 = d.tab.phases.copy(), d.tab.xzs.copy()
            P = qcb200.random_paulis(k, n, rng).to_gpu()
            state = (Q.Stabilizer if kind == "Stabilizer" else Q.Destabilizer)(Q.Tableau(ph0.copy(), n, xz0.copy())).to_gpu()
            pristine = Q.DeviceTableau(len(ph0), n)
            pristine.upload(ph0, xz0)
            rank = ctypes.c_int32(0)
            anti = np.zeros(k, np.int32)
            res = np.zeros(k, np.int32)
            done = ctypes.c_uint32()
            ms = device_ms(lambda: check(L.qcb_project(state.tab.dev.handle, Q.KIND[kind], ctypes.byref(rank),
                                                       P.dev.handle, 1, 1, ptr(anti), ptr(res), ctypes.byref(done),
                                                       sp)),
                           max(7, args.steps // 2),
                           setup=lambda: check(L.qcb_tableau_copy(state.tab.dev.handle, pristine.handle, sp)))
            state.to_cpu()
            # the oracle: the same sequence on the host, one thread
            t0 = time.perf_counter()
            ph, xz = ph0.copy(), xz0.copy()
            outs = []
            for i in range(k):
                _, ph, xz, _, a_, r_ = oracle.project(kind, ph, xz, n, P.xzs[i], 0)
                outs.append((a_, r_))
            cpu = (time.perf_counter() - t0) * 1e3 / k
            assert [o[0] for o in outs] == list(anti) and [o[1] for o in outs] == list(res)
            assert np.array_equal(state.tab.xzs, xz) and np.array_equal(state.tab.phases, ph)
            key = "project" if kind == "Destabilizer" else f"project_stab_{n}"
            emit(f"project! of a random Pauli on a random {n}-qubit {kind}", key, ms / k,
                 {"workload": f"1000 random Paulis (weight ~ U{{1..n}}) projected in sequence on a random {n}-qubit "
                              f"{kind} by one call, per projection", "rows": len(ph0)}, cpu)

    if want("expect"):
        # ---- expect of 1000 random Paulis on a random 1000-qubit Destabilizer:
        # independent projections (each on its own copy), one launch, the
        # state unchanged; half of them are stabilizer-group elements
        n, k = 1000, 1000
        d = random_destabilizer(n)
        P = Q.Tableau.zeros(k, n)
        for i in range(k):
            if i % 2:
                w = int(rng.integers(1, n + 1))
                qs = rng.choice(n, w, replace=False)
                kinds = rng.integers(1, 4, size=w)
                xs = np.zeros((1, n), bool); zs = np.zeros((1, n), bool)
                xs[0, qs] = kinds & 1 == 1; zs[0, qs] = kinds & 2 == 2
                one = Q.Tableau.from_bits([0], xs, zs)
                P.xzs[i], P.phases[i] = one.xzs[0], 0
            else:
                acc, ph = np.zeros(d.tab.xzs.shape[1], np.uint64), 0
                for r in np.nonzero(rng.random(n) < 0.5)[0][:64]:
                    acc, ph = oracle.mul_left_pauli(acc, ph, d.tab.xzs[n + r], d.tab.phases[n + r])
                P.xzs[i], P.phases[i] = acc, ph
        Pg = P.copy().to_gpu()
        state = Q.Destabilizer(Q.Tableau(d.tab.phases.copy(), n, d.tab.xzs.copy())).to_gpu()
        out = np.zeros(k, np.int32)
        ms = device_ms(lambda: check(L.qcb_expect(state.tab.dev.handle, Q.KIND["Destabilizer"], 0, Pg.dev.handle,
                                                  ptr(out), sp)), args.steps)
        t0 = time.perf_counter()
        expected = []
        for i in range(k):
            st_, _, _, _, a_, r_ = oracle.project("Destabilizer", d.tab.phases, d.tab.xzs, n, P.xzs[i], P.phases[i])
            expected.append(r_)
        cpu = (time.perf_counter() - t0) * 1e3 / k
        assert list(out) == expected
        emit("expect of a random Pauli on a random 1000-qubit Destabilizer (independent projections)", "expect",
             ms / k, {"workload": "1000 Paulis (half random, half stabilizer-group elements) in one call, per Pauli",
                      "rows": 2 * n}, cpu)

    if want("dense_apply"):
        # ---- dense apply! of tensor_pow(tCNOT, 500) to a random 1000-qubit stabilizer
        n = 1000
        d = random_destabilizer(n)
        src = Q.Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
        work = Q.Tableau(src.phases.copy(), n, src.xzs.copy()).to_gpu()
        pristine = Q.DeviceTableau(n, n)
        pristine.upload(src.phases, src.xzs)
        c = Q.tensor_pow(Q.tCNOT(), 500).to_gpu()
        ms = device_ms(lambda: check(L.qcb_apply_dense(work.dev.handle, c.tab.dev.handle, 1, sp)), args.steps,
                       setup=lambda: check(L.qcb_tableau_copy(work.dev.handle, pristine.handle, sp)))
        work.to_cpu()
        oph, oxz = oracle.apply_dense(src.phases, src.xzs, n, c.tab.phases, c.tab.xzs)
        assert np.array_equal(work.xzs, oxz) and np.array_equal(work.phases, oph)
        cpu = cpu_ms(lambda: oracle.apply_dense(src.phases, src.xzs, n, c.tab.phases, c.tab.xzs))
        emit("dense apply! of tensor_pow(tCNOT, 500) to a random 1000-qubit stabilizer", "dense_apply", ms,
             {"workload": "apply!(random_stabilizer(1000), tensor_pow(tCNOT, 500)), phases on"}, cpu)

    if want("sCNOT"):
        n = 1000
        d = random_destabilizer(n)
        src = Q.Tableau(d.tab.phases[n:].copy(), n, d.tab.xzs[n:].copy())
        work = Q.Tableau(src.phases.copy(), n, src.xzs.copy()).to_gpu()
        pristine = Q.DeviceTableau(n, n)
        pristine.upload(src.phases, src.xzs)
        # ---- symbolic sCNOT(32, 504) on a random 1000-qubit stabilizer: the time
        # per call of a stream of calls (as a repeated apply! is timed on the
        # CPU), the K launches replayed from one CUDA graph so that the Python
        # call overhead is not in the timed region; the isolated call, host
        # overhead included, is reported beside it
        from qcb200 import ops as O
        gate = O.to_array([O.sCNOT(32, 504)])
        check(L.qcb_tableau_copy(work.dev.handle, pristine.handle, sp))
        single = device_ms(lambda: check(L.qcb_apply_gates(work.dev.handle, ptr(gate), 1, 1, sp)), max(args.steps, 50))
        check(L.qcb_tableau_copy(work.dev.handle, pristine.handle, sp))
        torch.cuda.synchronize()
        K = 1000  # even: sCNOT applied twice is the identity, so the state comes back
        graph = torch.cuda.CUDAGraph()
        n_before = L.qcb_launch_count()
        with torch.cuda.graph(graph):
            cs = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            for _ in range(K):
                check(L.qcb_apply_gates(work.dev.handle, ptr(gate), 1, 1, cs))
        per_graph = L.qcb_launch_count() - n_before
        ms = device_ms(lambda: graph.replay(), max(7, args.steps // 2)) / K
        work.to_cpu()
        assert np.array_equal(work.xzs, src.xzs) and np.array_equal(work.phases, src.phases)
        check(L.qcb_apply_gates(work.dev.handle, ptr(gate), 1, 1, sp))
        work.to_cpu()
        oph, oxz = oracle.apply_gates(src.phases, src.xzs, n, gate)
        assert np.array_equal(work.xzs, oxz) and np.array_equal(work.phases, oph)
        cpu = cpu_ms(lambda: oracle.apply_gates(src.phases, src.xzs, n, gate), reps=20)
        emit("symbolic apply! of sCNOT(32, 504) to a random 1000-qubit stabilizer", "sCNOT", ms,
             {"workload": "apply!(random_stabilizer(1000), sCNOT(32, 504)), per call of 1000 calls replayed from one "
                          "CUDA graph (one kernel launch each)"}, cpu,
             {"gpu_launches": per_graph, "single_call_ms": single,
              "single_call_note": "one call between CUDA events, Python ctypes overhead included"})
        del graph

    for out in lines:
        print(json.dumps(out), flush=True)


def bench_batch(args):
    """The batched mixed workload: 256 rotated surface-code sampling jobs
    (d uniform in {3,...,15}, rounds = d, p log-uniform in [1e-4, 1e-2], shots
    log-uniform in [1e3, 1e6]) plus 512 canonicalize! jobs on random
    stabilizers (n uniform in [100, 2000]), seeded.  Batched: one persistent
    sampling launch and one persistent canonicalize! launch on two streams,
    captured together in one CUDA graph, tile widths from the autotuner per
    size class.  Plain: the same 768 jobs as per-job launches in sequence.
    The value is frame-gate updates/s of the whole mix (all sampling updates
    over the time of everything, canonicalize! included)."""
    import torch
    import numpy as np
    import qcb200
    from qcb200 import circuits, ops as O
    from qcb200 import tableau as Q
    from qcb200._lib import check, lib

    qcb200.ensure_init(0)
    L = lib()
    rng = np.random.default_rng(0xBA7C4)
    t_setup = time.perf_counter()
    jobs = []
    for k in range(256):
        d = int(rng.choice([3, 5, 7, 9, 11, 13, 15]))
        p = float(10 ** rng.uniform(-4, -2))
        shots = int(round(10 ** rng.uniform(3, 6)))
        prog = qcb200.Program(circuits.rotated_surface_code_memory(d, d, p))
        qmax, bmax = O.affected_counts(prog.ops)
        frame = qcb200.PauliFrame(shots, qmax, bmax, init=False)
        jobs.append(dict(d=d, p=p, shots=shots, prog=prog, frame=frame, seed=int(rng.integers(0, 2**63))))
    updates = sum(j["prog"].info["n_updates"] * j["shots"] for j in jobs)
    # the autotuner: one tile width per size class (code distance)
    tuned = {}
    for j in jobs:
        if j["d"] not in tuned:
            tuned[j["d"]] = qcb200.tune_tile(j["prog"])[0]
    fbatch = qcb200.Batch([(j["frame"], j["prog"], j["seed"], 0) for j in jobs])
    # canonicalize! jobs: uniformly random stabilizer states (Bravyi-Maslov)
    canon_n = [int(n) for n in rng.integers(100, 2001, size=512)]
    pristine, work = [], []
    for n in canon_n:
        t = qcb200.random_stabilizer(n, rng).tab
        st = Q.Stabilizer(t).to_gpu()
        pristine.append(Q.Stabilizer(t.copy()).to_gpu())
        work.append(st)
    cbatch = Q.CanonBatch(work)
    setup_s = time.perf_counter() - t_setup

    def restore():
        for w, p0 in zip(work, pristine):
            check(L.qcb_tableau_copy(w.tab.dev.handle, p0.tab.dev.handle, None))

    main = torch.cuda.current_stream()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    n_cap = L.qcb_launch_count()
    with torch.cuda.graph(graph):
        cs = torch.cuda.current_stream()
        s1.wait_stream(cs)
        s2.wait_stream(cs)
        fbatch.run(ctypes.c_void_p(s1.cuda_stream))
        cbatch.run(ctypes.c_void_p(s2.cuda_stream))
        cs.wait_stream(s1)
        cs.wait_stream(s2)
    torch.cuda.synchronize()
    launches_per_replay = L.qcb_launch_count() - n_cap  # kernel nodes of the graph

    def timed(fn, steps, warm):
        ts = []
        for i in range(warm + steps):
            restore()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(main)
            fn()
            e1.record(main)
            torch.cuda.synchronize()
            if i >= warm:
                ts.append(e0.elapsed_time(e1))
        return statistics.median(ts), ts

    sp = ctypes.c_void_p(main.cuda_stream)

    def plain():
        for j in jobs:
            check(L.qcb_pftrajectories_fresh(j["frame"].handle, j["prog"].handle, j["seed"], 0, sp))
        for w in work:
            check(L.qcb_canonicalize(w.tab.dev.handle, 1, len(w.tab), 1, None, None, sp))

    sampler = ClockSampler(0)
    sampler.start()
    ms_b, _ = timed(lambda: graph.replay(), args.steps, args.warmup)
    ms_p, _ = timed(plain, max(3, args.steps // 4), 3)
    # the two halves alone, for the record
    ms_f, _ = timed(lambda: fbatch.run(sp), 3, 1)
    ms_c, _ = timed(lambda: cbatch.run(sp), 3, 1)
    clocks = sampler.stop()
    # every job of the last batched replay equals its plain launch: compare a sample
    restore()
    graph.replay()
    torch.cuda.synchronize()
    fbatch.status()
    want_rank = cbatch.ranks()
    for j in jobs[::37]:
        rec_b = j["frame"].record_planes()
        check(L.qcb_pftrajectories_fresh(j["frame"].handle, j["prog"].handle, j["seed"], 0, sp))
        torch.cuda.synchronize()
        assert np.array_equal(rec_b, j["frame"].record_planes()), "batched record differs from the plain launch"
    for k in range(0, 512, 97):
        work[k].to_cpu()
        got = work[k].tab.xzs.copy()
        check(L.qcb_tableau_copy(work[k].tab.dev.handle, pristine[k].tab.dev.handle, sp))
        _, rx, rz = Q.canonicalize_(work[k], ranks=True)
        work[k].to_cpu()
        assert np.array_equal(got, work[k].tab.xzs) and (rx, rz) == want_rank[k]
    v_b = updates / (ms_b / 1e3)
    v_p = updates / (ms_p / 1e3)
    out = {"metric": "frame-gate updates/s, batched mixed workload (256 surface-code circuits + 512 canonicalize!)",
           "value": v_b, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms_b, "higher_is_better": True, "scaling": "none", "vs_baseline": None,
           "dtype": "u32 bit planes (GF(2)) + u64 bit rows", "data": "synthetic (seeded)",
           "config": {"workload": "256 rotated surface-code memory circuits, d in {3..15}, rounds = d, p log-U[1e-4,1e-2], "
                                  "shots log-U[1e3,1e6] + 512 canonicalize! on uniformly random stabilizers n ~ U[100,2000]; one "
                                  "persistent sampling launch + one persistent canonicalize! launch in one CUDA graph",
                      "frame_updates": updates, "total_shots": sum(j["shots"] for j in jobs),
                      "tuned_tiles": {str(k): v for k, v in sorted(tuned.items())},
                      "l2": "no flush: the sampling jobs write ~%.1f GB of records per step" % (
                          sum(j["prog"].info["nbits"] * j["shots"] for j in jobs) / 8e9)},
           "gpu_launches": launches_per_replay,
           "plain": {"value": v_p, "ms_per_step": ms_p, "launches": len(jobs) + len(work)},
           "speedup_vs_plain": ms_p / ms_b, "sampling_alone_ms": ms_f, "canonicalize_alone_ms": ms_c,
           "clocks": clocks, "setup_s": setup_s}
    print(json.dumps(out), flush=True)


def bench_serve(args):
    """The serving loop: Poisson arrivals of sampling requests (rotated surface
    code, d uniform over odd 3..25, rounds = d, p log-uniform in [1e-4, 1e-2],
    shots log-uniform in [1e4, 1e7], seeded), admitted against a 64 GB HBM
    budget with programs and buffers resident on the device (compiled before
    the clock starts).  For each arrival rate the same requests go through
    (a) the continuous-batching server (8 slots, 2^20-shot chunks) and (b)
    serial plain execution (one slot, each request as one launch), with the
    same arrival times.  Latency = completion on the device - arrival; a
    client thread releases each record when it completes (no copy out).
    Reported: p50/p99 latency and aggregate frame-gate updates/s."""
    import numpy as np
    import qcb200
    from qcb200 import circuits, ops as O

    qcb200.ensure_init(0)
    rng = np.random.default_rng(0x5E7E)
    n_req = args.serve_requests
    reqs = []
    for _ in range(n_req):
        d = int(rng.choice(np.arange(3, 26, 2)))
        p = float(10 ** rng.uniform(-4, -2))
        shots = int(round(10 ** rng.uniform(4, 7)))
        circ = O.to_array(circuits.rotated_surface_code_memory(d, d, p))
        reqs.append(dict(d=d, shots=shots, ops=circ, seed=int(rng.integers(0, 2**63)),
                         updates=O.count_updates(circ) * shots))
    total_updates = sum(r["updates"] for r in reqs)
    budget = 64 << 30

    def run(server, lam, seed):
        arr_rng = np.random.default_rng(seed)
        gaps = arr_rng.exponential(1.0 / lam, size=n_req)
        t_arr = np.cumsum(gaps)
        tickets = [None] * n_req
        done = {}

        def reaper():
            # blocks in the library (no GIL held) until the next completion
            while len(done) < n_req:
                t, st, times = server.next_done(600.0)
                done[t] = times
                server.release(t)

        th = threading.Thread(target=reaper, daemon=True)
        th.start()
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            delay = t_arr[i] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets[i] = server.submit(r["ops"], r["shots"], r["seed"])
        th.join(timeout=600)
        lat = np.array([done[t][2] - done[t][0] for t in tickets])
        span = max(done[t][2] for t in tickets) - min(done[t][0] for t in tickets)
        return lat, span

    lams = [float(x) for x in args.serve_rates.split(",")]
    results = []
    srv = qcb200.Server(budget, slots=8, chunk_shots=1 << 20)
    ser = qcb200.Server(budget, slots=1, chunk_shots=1 << 24)  # one launch per request (shots <= 1e7)
    t_pre = time.perf_counter()
    for r in reqs:
        srv.preload(r["ops"])
        ser.preload(r["ops"])
    preload_s = time.perf_counter() - t_pre
    # warm-up: the buffers of the first requests through both servers
    for sv in (srv, ser):
        ts = [sv.submit(r["ops"], min(r["shots"], 1 << 16), r["seed"]) for r in reqs[:8]]
        for t in ts:
            sv.wait(t)
            sv.release(t)
    sampler = ClockSampler(0)
    sampler.start()
    for k, lam in enumerate(lams):
        lat_b, span_b = run(srv, lam, 100 + k)
        lat_s, span_s = run(ser, lam, 100 + k)
        results.append({"rate_per_s": lam,
                        "batched": {"p50_ms": float(np.percentile(lat_b, 50) * 1e3),
                                    "p99_ms": float(np.percentile(lat_b, 99) * 1e3),
                                    "updates_per_s": total_updates / span_b},
                        "serial_plain": {"p50_ms": float(np.percentile(lat_s, 50) * 1e3),
                                         "p99_ms": float(np.percentile(lat_s, 99) * 1e3),
                                         "updates_per_s": total_updates / span_s}})
    clocks = sampler.stop()
    srv.close()
    ser.close()
    head = results[-1]
    out = {"metric": "p99 latency of sampling requests, serving loop (Poisson arrivals)",
           "value": head["batched"]["p99_ms"], "unit": "ms", "n_gpus": 1, "steps": n_req, "warmup": 8,
           "ms_per_step": head["batched"]["p50_ms"], "higher_is_better": False, "scaling": "none",
           "vs_baseline": None, "dtype": "u32 bit planes (GF(2))", "data": "synthetic (seeded)",
           "config": {"workload": f"{n_req} requests: rotated surface code d in {{3,5,...,25}}, rounds = d, p log-U[1e-4,1e-2], "
                                  "shots log-U[1e4,1e7]; 64 GB HBM budget; continuous batching with 8 slots and 2^20-shot "
                                  "chunks vs serial plain (1 slot, one launch per request); value = p99 at the highest rate",
                      "total_updates": total_updates, "total_shots": sum(r["shots"] for r in reqs),
                      "preload_s": preload_s},
           "sweep": results, "clocks": clocks}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--shots", type=int, default=SHOTS_PER_GPU)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--walker-tile", type=int, default=0)
    ap.add_argument("--workload", default="frames", choices=["frames", "tableau", "batch", "serve"])
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--tableau-only", default="", help="comma list of mul_left,canonicalize,project,expect,dense_apply,sCNOT")
    ap.add_argument("--canon-sizes", default="", help="comma list of canonicalize! sizes (default 1000,2000,4000)")
    ap.add_argument("--serve-rates", default="25,50,100")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "tableau":
        if rank == 0:
            bench_tableau(args)
        return
    if args.workload == "batch":
        if rank == 0:
            bench_batch(args)
        return
    if args.workload == "serve":
        if rank == 0:
            bench_serve(args)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import qcb200
    from qcb200 import circuits, ops as O
    from qcb200._lib import check, lib, ptr

    qcb200.ensure_init(local)
    L = lib()
    if args.walker_tile:
        check(L.qcb_tune_set(b"walker_tile", args.walker_tile))
    arr = O.to_array(circuits.rotated_surface_code_memory(D, ROUNDS, P_NOISE))
    upd = O.count_updates(arr)
    assert upd == 7601
    shots = args.shots
    from qcb200.shard import max_over_ranks, shard_offset
    offset = shard_offset(rank, shots)  # Philox shot groups are 1024 shots
    prog = qcb200.Program(arr)
    qmax, bmax = O.affected_counts(arr)
    frame = qcb200.PauliFrame(shots, qmax, bmax, init=False)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def step(i):
        check(L.qcb_pftrajectories_fresh(frame.handle, prog.handle, 1000 + i, offset, sp))

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    n0 = L.qcb_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = L.qcb_launch_count() - n0
    ms = ev0.elapsed_time(ev1) / args.steps
    # a step is two kernels on one stream, the noise pre-sampler and the
    # walker (plus a memset of the bucket counts); the roofline is taken over
    # the step's event time (the launch list in profiles/ gives the shares)
    kernel_ms = ms

    # end to end through the public host API: the op list from host memory in
    # (compiled on the host when it changes; the compiled program, 0.2 MB at
    # d=11, copied host -> device from page-locked memory every call), the
    # record planes back to pinned host memory every call, copied out chunk by
    # chunk while later chunks run.
    words = (shots + 31) // 32
    rec_host = torch.empty((bmax, words), dtype=torch.int32, pin_memory=True)
    ops_host = arr  # numpy, host
    prog_bytes = ctypes.c_uint64()
    check(L.qcb_program_device_bytes(prog.handle, ctypes.byref(prog_bytes)))

    def e2e_step(i):
        check(L.qcb_pftrajectories_host(ptr(ops_host), len(ops_host), shots, 5000 + i, offset,
                                        rec_host.data_ptr(), sp))
    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize()
    e2e_steps = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        e2e_step(10 + i)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps

    # end to end through the drop-in output: pftrajectories(frame, circuit)
    # then measurements(frame), the reference's column-major Matrix{Bool}
    # (frames x nbits, one byte per bit: 1.44 GB at 1e6 shots) in pinned host
    # memory, every step
    bool_host = torch.empty((bmax, shots), dtype=torch.uint8, pin_memory=True)

    def bool_step(i):
        check(L.qcb_pftrajectories_fresh(frame.handle, prog.handle, 7000 + i, offset, sp))
        check(L.qcb_frame_download_measurements(frame.handle, ctypes.c_void_p(bool_host.data_ptr()), sp))
    bool_step(0)
    torch.cuda.synchronize()
    bool_steps = max(3, min(args.steps, 5))
    t0 = time.perf_counter()
    for i in range(bool_steps):
        bool_step(1 + i)
    torch.cuda.synchronize()
    bool_ms = (time.perf_counter() - t0) * 1e3 / bool_steps
    del bool_host
    clk = clocks.stop()

    if world > 1:
        ms, e2e_ms, bool_ms = max_over_ranks([ms, e2e_ms, bool_ms], device="cuda")

    total_updates = upd * shots * world
    value = total_updates / (ms / 1e3)
    e2e_value = total_updates / (e2e_ms / 1e3)
    peak, peak_kind = load_peaks()
    model_bytes = MODEL_BITS_PER_SHOT / 8 * shots
    hbm_bytes = (RECORD_BITS + FRAME_BITS) / 8 * shots
    achieved = model_bytes / (kernel_ms / 1e3) / 1e9
    # the walker moves the model bytes through shared memory: 128 B per SM
    # per clock at the sampled SM clock
    props = torch.cuda.get_device_properties(local)
    smem_gbs = props.multi_processor_count * 128 * (clk.get("sm_mhz") or 1965.0) * 1e6 / 1e9
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "walker_d11_traffic.json")
    if os.path.exists(tr_path):
        try:
            traffic = json.load(open(tr_path)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 bit planes (GF(2))", "data": "synthetic (seeded Philox noise)",
        "config": {"workload": WORKLOAD, "shots_per_gpu": shots, "updates_per_shot": upd,
                   "parallelism": f"shot-sharded x{world}",
                   "l2": "no flush: each step writes 240 MB (record + frame) > 126 MB L2; inputs are the 0.4 MB program"},
        "gpu_launches": int(launches),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(prog_bytes.value),
                "d2h_bytes_per_step": int(bmax * words * 4), "ms_per_step": e2e_ms,
                "api": "qcb_pftrajectories_host (one call: circuit + shots + seed in, record planes out)",
                "inputs": f"the {arr.nbytes}-byte op list is read from host memory and compared with the last "
                          "call's (compiled on the host when it differs); the compiled program "
                          f"({prog_bytes.value} bytes) is copied host -> device from page-locked memory every call"},
        "e2e_measurements": {"value": total_updates / (bool_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": int(bmax * shots), "ms_per_step": bool_ms,
                             "api": "pftrajectories(frame, circuit) + measurements(frame): qcb_pftrajectories_fresh "
                                    "then qcb_frame_download_measurements into the reference's column-major "
                                    "Bool matrix (one byte per bit) in pinned host memory",
                             "inputs": "the compiled program stays resident (compiled once per circuit, as the "
                                       "Julia extension caches it); seed per call"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one walker_kernel "
                                       "launch of this workload (profiles/walker_d11_traffic.json), not measured "
                                       "in this run",
                     "algorithmic_bytes_per_launch": model_bytes,
                     "timed": "the whole step (presample_kernel + walker_kernel), CUDA events on the launching stream",
                     "basis": "model plane bytes of an op-per-launch schedule (5,175 B/shot); the walker keeps the "
                              "frame on chip, so its compulsory DRAM bytes are the record + final frame",
                     "compulsory_dram_bytes_per_launch": hbm_bytes,
                     "compulsory_dram_frac": hbm_bytes / (kernel_ms / 1e3) / 1e9 / peak,
                     "smem_peak_gbs": smem_gbs, "smem_frac": achieved / smem_gbs},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline_run()
        except Exception as e:  # the oracle must be built on the box
            out["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
