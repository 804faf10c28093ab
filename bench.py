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
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


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


def cpu_baseline_run(target_cpu_seconds: float = 15.0):
    """The oracle port (reference loop structure: one pass over all frames per
    op, one rand() per frame per noise site, threads over frame slices) timed
    on the host cores on a bounded sample of the same circuit."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the checker, used here only as the timed CPU baseline
    from qcb200 import circuits, ops as O

    arr = O.to_array(circuits.rotated_surface_code_memory(D, ROUNDS, P_NOISE))
    qmax, bmax = O.affected_counts(arr)
    updates_per_shot = O.count_updates(arr)
    cores = os.cpu_count() or 1
    shots = 2000
    t0 = time.perf_counter()
    oracle.pftrajectories_rng(arr, shots, qmax, bmax, seed=1, threads=1)
    t1 = time.perf_counter() - t0
    # size the sample to about target_cpu_seconds of single-core work, spread over all cores
    sample = int(min(1_000_000, max(cores * 100, shots * target_cpu_seconds / max(t1, 1e-6))))
    t0 = time.perf_counter()
    oracle.pftrajectories_rng(arr, sample, qmax, bmax, seed=2, threads=cores)
    dt = time.perf_counter() - t0
    rate = updates_per_shot * sample / dt
    threads = max(1, min(cores, sample // 100))
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sample} shots of the d=11 circuit (Xoshiro per-frame draws), {dt:.2f} s wall on {threads} threads"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    cb = None
    times = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline_run(target_cpu_seconds=4.0)
        if i >= args.warmup:
            times.append(r["value"])
            cb = r
    v = statistics.median(times)
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 7601 * SHOTS_PER_GPU / v * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u32 bit planes", "data": "synthetic (seeded)", "impl": "reference",
           "config": {"workload": WORKLOAD, "sample": cb["sample"]},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": cb["cores"], "kind": cb["kind"], "sample": cb["sample"]},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

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
    offset = rank * ((shots + 1023) // 1024 * 1024)  # Philox shot groups are 1024 shots
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
    # the walker is the only kernel of a step: its event time is the launch duration
    kernel_ms = ms

    # end to end through the public host API: ops from host memory in, record
    # planes back to pinned host memory, every step.
    words = (shots + 31) // 32
    rec_host = torch.empty((bmax, words), dtype=torch.int32, pin_memory=True)
    ops_host = arr  # numpy, host
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
    clk = clocks.stop()

    if world > 1:
        t = torch.tensor([ms, e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms = float(t[0]), float(t[1])

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
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(arr.nbytes),
                "d2h_bytes_per_step": int(bmax * words * 4), "ms_per_step": e2e_ms},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)", "traffic": traffic,
                     "algorithmic_bytes_per_launch": model_bytes,
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
