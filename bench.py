#!/usr/bin/env python3
"""Benchmark of stwo's commit + FRI path on B200 (one JSON line on rank 0).

Workloads (seeded synthetic M31 data, values uniform in [0, P)):
  wide_fib_prove (default) Wide-Fibonacci STARK prove: 100 columns, 2^20 rows,
                 col[i+2] = col[i]^2 + col[i+1]^2, first two columns uniform
                 per row, default PcsConfig (pow 10, blowup 1, 3 queries, FRI
                 fold-by-2 to a last layer of degree 1), Blake2s channel.
                 A step is one whole proof from the two input columns to the
                 proof bytes.  Unit: proved trace cells / s (cells = 100 x 2^20).
  commit_uneven  512 columns, log sizes U{12..22}, blowup 2, one lifted
                 Blake2s tree (L = 24): interpolate -> evaluate -> leaves ->
                 nodes.  Unit: committed trace cells / s.
  commit_plain   32 columns of log 16, blowup 1, natural-order input:
                 interpolate (the bit reversal rides on the first IFFT pass's
                 loads) -> evaluate -> Merkle (L = 17).
  fri_heavy      one QM31 column of log 24: FRI commit + 70-query decommit.
  serving        Poisson stream of Wide-Fibonacci requests (p50/p99 latency).
  trace_fft      the prover's trace transforms alone (--n-cols x 2^--log-n-rows,
                 interpolate, then evaluate at --log-blowup): the kernels'
                 profile target.
  fri_fold       the stand-alone FriOps folds at log 24 (fold_circle_into_line,
                 fold_line) against HBM: their profile target.

The default line also carries, measured in the same run at N = 1, the plain
commit, the uneven commit's per-column / batched / graph forms, the FRI-heavy
commit with the stand-alone folds against HBM, and a 24-request serving stream
(skip with --no-extras).

A step is one commit of the whole trace.  `value` is device-timed with inputs
resident in HBM; `e2e` goes through the same public calls with the trace in
pinned host memory (H2D copy of the trace + D2H of the root inside every
step).  Multi-GPU runs are independent replicas (weak scaling, no collective).
`--impl reference` times the CPU restatement of stwo's SimdBackend (the
oracle port; Rust/SimdBackend itself cannot be built here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "stwo-metal_b200"))

P = (1 << 31) - 1
METRIC = "proved trace cells/s, batched vs per-column on B200 (bit-exact); p99 prove ms"


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------ workloads ----
def lifted_leaf_compressions(lde_logs, L):
    """Blake2s compressions of the lifted leaves as the staged leaf kernel
    runs them: 16-column group g of the columns sorted by size at the size of
    its largest column, the last group at the lifting size L."""
    logs = sorted(lde_logs)
    n_groups = (len(logs) + 15) // 16
    return sum(1 << (L if g + 1 == n_groups else logs[min(16 * g + 15, len(logs) - 1)]) for g in range(n_groups))


def workload_spec(name: str):
    if name == "commit_uneven":
        r = np.random.default_rng(3)
        logs = [int(x) for x in r.integers(12, 23, 512)]
        return dict(name=name, logs=logs, blowup=2, bitrev=False, seed=3)
    if name == "commit_plain":
        return dict(name=name, logs=[16] * 32, blowup=1, bitrev=True, seed=1)
    raise SystemExit(f"unknown workload {name}")


def make_columns(spec):
    r = np.random.default_rng(spec["seed"] + 1000)
    return [r.integers(0, P, 1 << l, dtype=np.uint32) for l in spec["logs"]]


# ---------------------------------------------------------- clock sampling --
class ClockSampler:
    """SM clocks and clock-event reasons of this rank's GPU, sampled during the
    timed region.  Reads NVML every 10 ms from a thread (the same counters as
    `nvidia-smi --query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.*`),
    so that a region of tens of milliseconds still gets several samples; falls
    back to an `nvidia-smi -lms 100` subprocess when NVML is not importable.
    Reads only: no clock or power setting is touched."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # nvmlClocksEventReason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.samples = []
        self.nvml = None
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
        return pynvml, h

    def _poll(self):
        nv, h = self.nvml
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop_flag.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM), int(get_reasons(h))))
            except Exception:
                pass
            self.stop_flag.wait(0.01)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
        except Exception:
            self.nvml = None
        if self.nvml is not None:
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            t0 = time.perf_counter()
            while not self.samples and time.perf_counter() - t0 < 1.0:
                time.sleep(0.001)
            self.samples.clear()  # keep only samples taken from here on
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_flag.set()
            self.t.join(timeout=1.0)
            got = list(self.samples)
            if not got:  # a region shorter than the period: one reading right at its end
                nv, h = self.nvml
                try:
                    get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                        nv.nvmlDeviceGetCurrentClocksThrottleReasons
                    got = [(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                            nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM), int(get_reasons(h)))]
                except Exception:
                    got = []
            reasons = sorted(nm for nm, bit in self.REASON_BITS.items() if any(r & bit for _, _, r in got))
            return {"sm_mhz": statistics.median(c for c, _, _ in got) if got else None,
                    "sm_max_mhz": max(m for _, m, _ in got) if got else None,
                    "reasons": reasons, "samples": len(got), "source": "nvml, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxes) if maxes else None,
                "reasons": sorted(reasons), "samples": len(sms), "source": "nvidia-smi, 100 ms"}


# ------------------------------------------------------------ dist helpers --
# Replicas only: every rank proves (or commits) its own copy of the workload,
# with no collective on the data path.  The only collectives are the barriers
# around the timed region and one all-reduce of the timing scalar; they run
# over NCCL when the ranks have GPUs, and over gloo otherwise (the CPU tests
# of this plumbing).
def dist_backend() -> str:
    import torch
    return "nccl" if torch.cuda.is_available() else "gloo"


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = dist_backend()
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank: float, ms_max: float, world: int) -> float:
    """Whole-job throughput of `world` replicas: all units over the slowest
    rank's time (weak scaling)."""
    return units_per_rank * world / (ms_max * 1e-3)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------- CPU reference ----
def cpu_commit_rate(spec, host_cols, budget_s=15.0, threads=None):
    """Oracle commit of a bounded sample of the workload's columns; returns
    (cells/s, sample description, threads)."""
    from oracle import ffi as oracle
    n_threads = oracle.set_threads(threads or os.cpu_count() or 1)
    blowup = spec["blowup"]
    maxlog = max(spec["logs"]) + blowup
    init, lg = oracle.canonic_half_coset_root(maxlog + 1)
    tw, itw = oracle.precompute_twiddles(init, lg)
    # sample: columns in workload order until ~1/16 of the cells (bounded)
    order = list(range(len(host_cols)))
    total = sum(c.size for c in host_cols)
    target = max(total // 16, host_cols[0].size)
    take, cells = [], 0
    for i in order:
        if cells >= target:
            break
        take.append(i)
        cells += host_cols[i].size
    cols = [host_cols[i] for i in take]
    L = max(spec["logs"][i] for i in take) + blowup
    reps, elapsed = 0, 0.0
    while elapsed < budget_s or reps == 0:
        t0 = time.perf_counter()
        src = [oracle.bit_reverse(c) for c in cols] if spec["bitrev"] else cols
        coeffs = oracle.interpolate_columns(src, itw)
        evals = oracle.evaluate_columns(coeffs, blowup, tw)
        oracle.merkle_build_layers(evals, L, staged=True)
        elapsed += time.perf_counter() - t0
        reps += 1
        if elapsed > budget_s / 3 and reps >= 1:
            break
    rate = reps * cells / elapsed
    return rate, f"{len(take)} of {len(host_cols)} columns ({cells} cells, lifted L={L}), {reps} rep(s)", n_threads


def run_reference(args, spec, world, rank):
    if rank != 0:
        return
    host_cols = make_columns(spec)
    from oracle import ffi as oracle
    n_threads = oracle.set_threads(os.cpu_count() or 1)
    rates = []
    for i in range(args.warmup + args.steps):
        rate, sample, n_threads = cpu_commit_rate(spec, host_cols, budget_s=4.0)
        if i >= args.warmup:
            rates.append(rate)
    value = statistics.median(rates)
    cells = sum(c.size for c in host_cols)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "committed trace cells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * cells / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 (M31)", "data": "synthetic (seeded numpy PCG64, uniform [0, 2^31-1))",
        "config": {"workload": spec["name"], "n_columns": len(spec["logs"]), "log_sizes": "U{12..22}"
                   if spec["name"] == "commit_uneven" else "16", "log_blowup": spec["blowup"],
                   "parallelism": f"replicas x{args.gpus}"},
        "cpu_baseline": {"value": value, "unit": "committed trace cells/s", "cores": n_threads, "kind": "port",
                         "sample": "per step: " + sample + "; SimdBackend restatement (C++, OpenMP, staged lifted leaves)"},
        "e2e": {"value": value, "unit": "committed trace cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- B200 ------
def run_b200(args, spec, world, rank, local):
    import torch
    from stwo_b200 import B200Backend, DeviceBuffer, DeviceColumn, ffi, layer_to_host
    from stwo_b200.backend import canonic_half_coset

    torch.cuda.set_device(local)
    ffi.init(local)
    stream = torch.cuda.Stream()
    be = B200Backend(stream.cuda_stream)
    logs, blowup = spec["logs"], spec["blowup"]
    host_cols = make_columns(spec)
    order = sorted(range(len(logs)), key=lambda i: logs[i])  # stable by length
    L = max(logs) + blowup
    init, lg = canonic_half_coset(L + 1)
    tree = be.precompute_twiddles(init, lg)
    inputs = [DeviceColumn.from_host(c, stream.cuda_stream) for c in host_cols]
    coeffs = [DeviceColumn(c.size, stream.cuda_stream) for c in host_cols]
    evals = [DeviceColumn(c.size << blowup, stream.cuda_stream) for c in host_cols]
    layers = [DeviceBuffer(32 << k, stream.cuda_stream) for k in range(L + 1)]
    evals_sorted = [evals[i] for i in order]
    cells = sum(c.size for c in host_cols)
    eval_cells = cells << blowup
    torch.cuda.synchronize()

    # Committer forms (commit_uneven): per-column launches, batched launches,
    # batched + CUDA graph; the pass plans of every size group are autotuned
    # first (process-wide, so every form below runs with them).
    cms, tuned = None, None
    if spec["name"] == "commit_uneven":
        from stwo_b200 import Committer, fft_get_plan
        cms = {"per_column": Committer(logs, blowup, tree, per_column=True, stream=stream.cuda_stream),
               "batched": Committer(logs, blowup, tree, stream=stream.cuda_stream),
               "batched_graph": Committer(logs, blowup, tree, graph=True, stream=stream.cuda_stream)}
        t_tune = time.perf_counter()
        cms["batched_graph"].autotune(inputs, coeffs, evals, reps=2)
        torch.cuda.synchronize()
        tuned = {"seconds": time.perf_counter() - t_tune,
                 "plans": {str(n): fft_get_plan(n) for n in sorted(set(logs))}}

    phases = ["bitrev", "ifft", "rfft", "leaves", "nodes"]

    def step(evs=None):
        if spec["bitrev"]:
            # natural-order trace: bit reversal + interpolation in one call,
            # the bit reversal fused into the first IFFT pass (no phase of its own)
            rec(evs, 0)
            be.interpolate_natural_into(inputs, coeffs, tree)
        else:
            rec(evs, 0)
            be.interpolate_columns_into(inputs, coeffs, tree)
        rec(evs, 1)
        be.evaluate_polynomials_into(coeffs, blowup, tree, evals)
        rec(evs, 2)
        be.build_leaves_layers(evals_sorted, L, layers)
        rec(evs, 3)
        be.build_nodes(layers)
        rec(evs, 4)

    import ctypes

    def ffi_ptr(b):
        return ctypes.c_void_p(b.ptr)

    def size_t(n):
        return ctypes.c_size_t(n)

    def rec(evs, i):
        if evs is not None:
            evs[i].record(stream)

    def new_events():
        return [torch.cuda.Event(enable_timing=True) for _ in range(6)]

    # correctness gate on the first step: the root must match the oracle for
    # commit_plain (whole workload) -- commit_uneven is checked by the tests.
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    root = bytes(layer_to_host(layers[0])[0])

    # ---- device-timed region ----
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    all_evs = [new_events() for _ in range(args.steps)]
    launches0 = ffi.launch_count()
    with torch.cuda.stream(stream):
        t_start.record(stream)
        for k in range(args.steps):
            evs = all_evs[k]
            evs[5].record(stream)
            step(evs)
        t_end.record(stream)
    torch.cuda.synchronize()
    launches = ffi.launch_count() - launches0
    ms = t_start.elapsed_time(t_end) / args.steps
    clocks = sampler.stop()
    barrier(world)
    ms = max_over_ranks(ms, world)
    phase_ms = {p: 0.0 for p in phases}
    for evs in all_evs:
        phase_ms["bitrev"] += evs[5].elapsed_time(evs[0])
        phase_ms["ifft"] += evs[0].elapsed_time(evs[1])
        phase_ms["rfft"] += evs[1].elapsed_time(evs[2])
        phase_ms["leaves"] += evs[2].elapsed_time(evs[3])
        phase_ms["nodes"] += evs[3].elapsed_time(evs[4])
    for p in phase_ms:
        phase_ms[p] /= args.steps

    # ---- e2e: host trace -> device -> commit -> root to host ----
    pinned = []
    for c in host_cols:
        t = torch.empty(c.size, dtype=torch.int32).pin_memory()
        t.numpy().view(np.uint32)[:] = c
        pinned.append(t)
    root_host = torch.empty(32, dtype=torch.uint8).pin_memory()
    h2d = sum(c.nbytes for c in host_cols)

    e2e_cm = None
    if spec["name"] == "commit_uneven":
        # the committer's host path: each size group's copies overlap the
        # transforms of the groups already on the device
        from stwo_b200 import Committer
        e2e_cm = Committer(logs, blowup, tree, stream=stream.cuda_stream)
        e2e_layers = e2e_cm.new_layers()
        e2e_root = e2e_layers[0]
    else:
        e2e_root = layers[0]

    def e2e_step():
        if e2e_cm is not None:
            e2e_cm.commit_from_host([t.data_ptr() for t in pinned], inputs, coeffs, evals, e2e_layers)
        else:
            for t, d in zip(pinned, inputs):
                ffi.call("stwo_b200_memcpy_h2d", ffi_ptr(d), ctypes.c_void_p(t.data_ptr()), size_t(d.nbytes),
                         be.stream)
            step()
        ffi.call("stwo_b200_memcpy_d2h", ctypes.c_void_p(root_host.data_ptr()), ffi_ptr(e2e_root), size_t(32),
                 be.stream)
        ffi.call("stwo_b200_stream_sync", be.stream)

    with torch.cuda.stream(stream):
        for _ in range(max(1, args.warmup // 2)):
            e2e_step()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    assert bytes(root_host.numpy()) == root, "e2e root differs from device-resident root"

    # Integer-pipe ceiling for the Blake2s op mix: register-only compression
    # chains on every SM (148 SMs x 8 blocks x 256 threads).
    probe_out = DeviceBuffer(64, stream.cuda_stream)
    pb, pit = 148 * 8, 256
    for _ in range(2):
        ffi.call("stwo_b200_blake2s_probe", ctypes.c_uint32(pb), ctypes.c_uint32(pit), ffi_ptr(probe_out), be.stream)
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        p0.record(stream)
        ffi.call("stwo_b200_blake2s_probe", ctypes.c_uint32(pb), ctypes.c_uint32(pit), ffi_ptr(probe_out), be.stream)
        p1.record(stream)
    torch.cuda.synchronize()
    probe_rate = pb * 256 * pit / (p0.elapsed_time(p1) * 1e-3)

    forms = None
    if cms is not None:
        forms = {}
        for name, cm in cms.items():
            with torch.cuda.stream(stream):
                for _ in range(args.warmup):
                    cm.commit(inputs, coeffs, evals, layers)
            torch.cuda.synchronize()
            l0 = ffi.launch_count()
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                f0.record(stream)
                for _ in range(args.steps):
                    cm.commit(inputs, coeffs, evals, layers)
                f1.record(stream)
            torch.cuda.synchronize()
            f_ms = max_over_ranks(f0.elapsed_time(f1) / args.steps, world)
            assert bytes(layer_to_host(layers[0])[0]) == root, f"{name} root differs"
            forms[name] = {"ms_per_step": f_ms, "committed_cells_per_s": cells / (f_ms * 1e-3),
                           "launches_per_step": (ffi.launch_count() - l0) / args.steps}
            cm.close()
        forms["batched_over_per_column"] = forms["per_column"]["ms_per_step"] / forms["batched"]["ms_per_step"]
        forms["graph_over_per_column"] = forms["per_column"]["ms_per_step"] / forms["batched_graph"]["ms_per_step"]
        forms["autotune"] = tuned

    if rank != 0:
        return
    hbm_peak, peak_kind = load_peaks()
    # algorithmic bytes per phase (inputs + outputs once; twiddles excluded)
    alg_bytes = {
        "bitrev": 0,  # fused into the first IFFT pass (natural-order loads)
        "ifft": 8 * cells,
        "rfft": 4 * cells + 4 * eval_cells,
        "leaves": 4 * eval_cells + 32 * (1 << L),
        "nodes": 32 * (1 << L) + 32 * ((1 << L) - 1),
    }
    dominant = max(("ifft", "rfft", "leaves", "nodes"), key=lambda p: phase_ms[p])
    compressions = lifted_leaf_compressions([x + blowup for x in logs], L)
    if dominant == "leaves":
        achieved = compressions / (phase_ms["leaves"] * 1e-3) / 1e9
        roof = {"bound": "int32", "kernel": "lifted_leaves_kernel", "achieved": achieved,
                "peak": probe_rate / 1e9, "unit": "G Blake2s compressions/s", "frac": achieved * 1e9 / probe_rate,
                "peak_kind": "measured in this run (register-only Blake2s chain, all SMs)", "traffic": None,
                "alg_compressions_per_step": compressions}
    else:
        achieved = alg_bytes[dominant] / (phase_ms[dominant] * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "peak_kind": peak_kind, "traffic": None,
                "alg_bytes_per_step": alg_bytes[dominant]}
    # the CPU baseline is measured at N = 1 only (replicas do the same work per rank)
    cpu_rate, cpu_sample, cpu_cores = (cpu_commit_rate(spec, host_cols, budget_s=10.0) if world == 1
                                       else (None, None, None))
    line = {
        "metric": METRIC,
        "value": replica_rate(cells, ms, world),
        "unit": "committed trace cells/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32 (M31)",
        "data": "synthetic (seeded numpy PCG64, uniform [0, 2^31-1))",
        "config": {"workload": spec["name"], "n_columns": len(logs), "total_trace_cells": cells,
                   "log_sizes": "U{12..22} seed 3" if spec["name"] == "commit_uneven" else "16",
                   "log_blowup": blowup, "lifting_log_size": L, "merkle": "lifted Blake2s",
                   "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {"value": replica_rate(cells, e2e_ms, world), "unit": "committed trace cells/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 32, "ms_per_step": e2e_ms},
        "roofline": roof,
        "phase_roofline": {p: (alg_bytes[p] / (phase_ms[p] * 1e-3) / 1e9 / hbm_peak) if phase_ms[p] > 0 else None
                           for p in ("ifft", "rfft")},
        "phases_ms": phase_ms,
        "blake2s_compressions_per_s": compressions / (phase_ms["leaves"] * 1e-3),
        "blake2s_probe_compressions_per_s": probe_rate,
        "cpu_baseline": ({"value": cpu_rate, "unit": "committed trace cells/s", "cores": cpu_cores, "kind": "port",
                          "sample": cpu_sample + "; SimdBackend restatement (C++ oracle, OpenMP, staged lifted leaves)"}
                         if world == 1 else None),
        "root": root.hex(),
    }
    if forms is not None:
        line["forms"] = forms
    print(json.dumps(line), flush=True)


# ------------------------------------------------------ Wide-Fibonacci -----
PROVE_PHASES = ["trace_gen", "trace_interpolate", "trace_evaluate", "trace_merkle", "composition",
                "composition_interpolate", "composition_evaluate", "composition_merkle", "oods_sampling",
                "quotients", "fri_merkle", "fri_fold", "grind", "decommit"]


def prove_spec(log_n=20, n_cols=100):
    return dict(name="wide_fib_prove", log_n=log_n, n_cols=n_cols, log_blowup=1, pow_bits=10, n_queries=3,
                log_last_layer=0, line_fold_step=1, seed=2)


def prove_inputs(spec):
    r = np.random.default_rng(spec["seed"])
    n = 1 << spec["log_n"]
    return r.integers(0, P, n, dtype=np.uint32), r.integers(0, P, n, dtype=np.uint32)


L2_BYTES = 126 << 20


def prove_l2_note(spec):
    trace = (spec["n_cols"] << spec["log_n"]) * 4
    sizes = f"{trace >> 20} MB trace, {2 * trace >> 20} MB evaluations"
    if trace > L2_BYTES:
        return f"inputs larger than L2 ({sizes}; no flush)"
    return f"inputs smaller than L2 ({sizes}; no flush: a small demonstration size, not the benchmark workload)"


def prove_config_json(spec, world):
    return {"workload": "wide_fib_prove", "n_columns": spec["n_cols"], "log_n_rows": spec["log_n"],
            "trace_cells": spec["n_cols"] << spec["log_n"], "log_blowup": spec["log_blowup"],
            "pow_bits": spec["pow_bits"], "n_queries": spec["n_queries"],
            "fri": "circle fold + line folds by 2 to last layer log degree 0",
            "channel": "Blake2sMerkleChannel", "inputs": "col0/col1 uniform [0, 2^31-1) per row, seed 2",
            "l2": prove_l2_note(spec),
            "twiddles": "resident on the device from prover creation (outside the timed region; the "
                        "reference harness precomputes them inside every sample; their device time is the "
                        "line's twiddle_precompute_ms)",
            "e2e_inputs": "the two seed columns (2 x 2^log_n_rows words) are copied per proof; the other "
                          "columns are generated on the device, as the Wide-Fibonacci trace is defined",
            "parallelism": f"replicas x{world}"}


def cpu_prove(spec, a, b, threads=None):
    """Full oracle prove of the workload on the host cores: (seconds, proof, threads)."""
    from oracle import ffi as oracle
    n_threads = oracle.set_threads(threads or os.cpu_count() or 1)
    cfg = oracle.wide_fib_config(spec["log_n"], spec["n_cols"], spec["log_blowup"], spec["pow_bits"],
                                 spec["n_queries"], spec["log_last_layer"], spec["line_fold_step"])
    t0 = time.perf_counter()
    proof = oracle.prove_wide_fib(cfg, a, b)
    return time.perf_counter() - t0, proof, n_threads


def run_prove_reference(args, world, rank):
    if rank != 0:
        return
    spec = prove_spec(args.log_n_rows, args.n_cols)
    a, b = prove_inputs(spec)
    cells = spec["n_cols"] << spec["log_n"]
    secs = []
    n_threads = 1
    for i in range(args.warmup + args.steps):
        t, _, n_threads = cpu_prove(spec, a, b)
        if i >= args.warmup:
            secs.append(t)
    med = statistics.median(secs)
    value = cells / med
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "proved trace cells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * med,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31/QM31)",
        "data": "synthetic (seeded numpy PCG64)", "config": prove_config_json(spec, args.gpus),
        "p50_prove_ms": 1000 * statistics.median(secs), "p99_prove_ms": 1000 * max(secs),
        "cpu_baseline": {"value": value, "unit": "proved trace cells/s", "cores": n_threads, "kind": "port",
                         "sample": f"each step: the whole Wide-Fibonacci {spec['n_cols']} x 2^{spec['log_n']} proof (SimdBackend restatement, "
                                   "C++ oracle, OpenMP)"},
        "e2e": {"value": value, "unit": "proved trace cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# DRAM bytes (read + written) of one trace interpolate + evaluate (2^20 ->
# 2^21 per column) measured by ncu on 40 columns -- fft_warp_contig_kernel<1>
# 172.0 + 120.7 MB, fft_warp_inv_fwd_kernel<10> 167.8 + 451.7 MB,
# fft_warp_contig_kernel<0> 347.7 + 275.4 MB -- scaled to the 100 columns of
# the proof.
TRACE_FFT_TRAFFIC_100x2e20 = (172.0 + 120.7 + 167.8 + 451.7 + 347.7 + 275.4) * 1e6 * 100 / 40


def twiddle_precompute_ms(log_size, stream, reps=5):
    """Device time of PolyOps::precompute_twiddles for CanonicCoset(log_size)
    .half_coset into preallocated buffers (CUDA events, after one warm-up)."""
    import ctypes
    import torch
    from stwo_b200 import B200Backend, DeviceColumn, ffi
    from stwo_b200.backend import canonic_half_coset
    be = B200Backend(stream.cuda_stream)
    init, lg = canonic_half_coset(log_size)
    tw, itw = DeviceColumn(1 << lg, stream.cuda_stream), DeviceColumn(1 << lg, stream.cuda_stream)

    def run():
        ffi.call("stwo_b200_precompute_twiddles", ctypes.c_uint64(init), ctypes.c_uint32(lg), ctypes.c_void_p(tw.ptr),
                 ctypes.c_void_p(itw.ptr), be.stream)

    run()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        a.record(stream)
        for _ in range(reps):
            run()
        b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def run_prove_b200(args, world, rank, local):
    import ctypes
    import torch
    from oracle import ffi as oracle
    from stwo_b200 import DeviceBuffer, DeviceColumn, WideFibProver, ffi, wide_fib_config

    torch.cuda.set_device(local)
    ffi.init(local)
    stream = torch.cuda.Stream()
    spec = prove_spec(args.log_n_rows, args.n_cols)
    a_host, b_host = prove_inputs(spec)
    cells = spec["n_cols"] << spec["log_n"]
    prover = WideFibProver(wide_fib_config(spec["log_n"], spec["n_cols"], spec["log_blowup"], spec["pow_bits"],
                                           spec["n_queries"], spec["log_last_layer"], spec["line_fold_step"]),
                           stream.cuda_stream)
    a = DeviceColumn.from_host(a_host, stream.cuda_stream)
    b = DeviceColumn.from_host(b_host, stream.cuda_stream)
    cap = 1 << 22
    buf = (ctypes.c_uint8 * cap)()
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        n = prover.prove_into(a.ptr, b.ptr, buf, cap)
    proof = bytes(buf[:n])
    verdict = oracle.verify_wide_fib(proof, spec["log_n"], spec["n_cols"])

    # ---- device-timed region: whole proofs, inputs resident in HBM ----
    # (phase events off here; the per-phase split is a separate pass below)
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches0 = ffi.launch_count()
    with torch.cuda.stream(stream):
        evs[0].record(stream)
        for k in range(args.steps):
            prover.prove_into(a.ptr, b.ptr, buf, cap)
            evs[k + 1].record(stream)
    torch.cuda.synchronize()
    launches = ffi.launch_count() - launches0
    clocks = sampler.stop()
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    ms = sum(step_ms) / args.steps
    # per-phase split: the same proofs again with CUDA events between phases
    # One proof in timing mode first (it captures the FRI graph variant that
    # records phase events, host work the device would wait on), then the
    # counters are reset and the measured proofs run.
    ffi.call("stwo_b200_prover_set_timing", prover.handle, ctypes.c_int(1))
    with torch.cuda.stream(stream):
        prover.prove_into(a.ptr, b.ptr, buf, cap)
    torch.cuda.synchronize()
    ffi.call("stwo_b200_prover_set_timing", prover.handle, ctypes.c_int(1))
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            prover.prove_into(a.ptr, b.ptr, buf, cap)
    torch.cuda.synchronize()
    phase = (ctypes.c_double * len(PROVE_PHASES))()
    nproofs = ctypes.c_uint32()
    ffi.call("stwo_b200_prover_phase_times", prover.handle, phase, ctypes.c_uint32(len(PROVE_PHASES)),
             ctypes.byref(nproofs))
    ffi.call("stwo_b200_prover_set_timing", prover.handle, ctypes.c_int(0))
    phase_ms = {nm: phase[i] / max(1, nproofs.value) for i, nm in enumerate(PROVE_PHASES)}
    barrier(world)
    ms_max = max_over_ranks(ms, world)

    # ---- e2e: host inputs (pinned) -> device -> proof bytes on the host ----
    pa = torch.empty(a_host.size, dtype=torch.int32).pin_memory()
    pb = torch.empty(b_host.size, dtype=torch.int32).pin_memory()
    pa.numpy().view(np.uint32)[:] = a_host
    pb.numpy().view(np.uint32)[:] = b_host
    sp = ctypes.c_void_p(stream.cuda_stream)

    def e2e_step():
        # the prover copies the pinned columns itself, chunk by chunk, and
        # generates each chunk's trace rows as it lands
        return prover.prove_host_into(pa.data_ptr(), pb.data_ptr(), buf, cap)

    with torch.cuda.stream(stream):
        e2e_step()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            n_e2e = e2e_step()
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    assert bytes(buf[:n_e2e]) == proof, "e2e proof differs from the device-resident proof"

    # Integer-pipe ceiling for Blake2s (register-only chains on all SMs).
    probe_out = DeviceBuffer(64, stream.cuda_stream)
    for _ in range(2):
        ffi.call("stwo_b200_blake2s_probe", ctypes.c_uint32(148 * 8), ctypes.c_uint32(256),
                 ctypes.c_void_p(probe_out.ptr), sp)
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        p0.record(stream)
        ffi.call("stwo_b200_blake2s_probe", ctypes.c_uint32(148 * 8), ctypes.c_uint32(256),
                 ctypes.c_void_p(probe_out.ptr), sp)
        p1.record(stream)
    torch.cuda.synchronize()
    probe_rate = 148 * 8 * 256 * 256 / (p0.elapsed_time(p1) * 1e-3)
    # Integer-issue ceiling of the M31 butterfly (register-only bfly2 chains,
    # 80 butterflies per thread and round, all SMs).
    bf_blocks, bf_iters = 148 * 8, 512
    for _ in range(2):
        ffi.call("stwo_b200_butterfly_probe", ctypes.c_uint32(bf_blocks), ctypes.c_uint32(bf_iters),
                 ctypes.c_void_p(probe_out.ptr), sp)
    with torch.cuda.stream(stream):
        p0.record(stream)
        ffi.call("stwo_b200_butterfly_probe", ctypes.c_uint32(bf_blocks), ctypes.c_uint32(bf_iters),
                 ctypes.c_void_p(probe_out.ptr), sp)
        p1.record(stream)
    torch.cuda.synchronize()
    bfly_rate = bf_blocks * 256 * bf_iters * 80 / (p0.elapsed_time(p1) * 1e-3)
    hbm_peak, peak_kind = load_peaks()

    # The rest of the metric, in the same run (N = 1 only; replica runs skip
    # it): the plain commit, the uneven commit's forms, the FRI-heavy commit
    # and a short serving stream.
    extras = {}
    if world == 1 and args.extras:
        prover.close()
        a.close()
        b.close()
        extras["commit_plain"] = extra_commit_plain(args, stream, world)
        extras["commit_uneven"] = extra_commit_uneven(args, stream, world, hbm_peak, probe_rate)
        extras["fri_heavy"] = extra_fri_heavy(args, stream, world, hbm_peak, probe_rate)
        torch.cuda.synchronize()
        extras["serving"] = measure_serving(24, 1, world, local, with_cpu=False)

    if rank != 0:
        return
    n, nc, lb = spec["log_n"], spec["n_cols"], spec["log_blowup"]
    rows, ev = 1 << n, 1 << (n + lb)
    # algorithmic bytes / compressions per phase (inputs + outputs once)
    # The interpolation's last pass runs in one kernel with the evaluation's
    # first, so the two trace FFT phases are rated together.
    ph = dict(phase_ms)
    ph["trace_fft"] = ph.get("trace_interpolate", 0) + ph.get("trace_evaluate", 0)
    alg = {
        "trace_gen": ("hbm", 8 * rows + 4 * nc * rows),
        "trace_fft": ("hbm", 8 * nc * rows + 4 * nc * rows + 4 * nc * ev),
        "trace_merkle": ("int32", ev * ((nc + 15) // 16) + ev - 1),
        "composition": ("hbm", 4 * nc * (2 * rows) + 16 * (2 * rows)),
        "quotients": ("hbm", 4 * (nc + 8) * ev + 16 * ev),
        "oods_sampling": ("hbm", 4 * (nc + 8) * rows),
    }
    timed = {k: v for k, v in alg.items() if ph.get(k, 0) > 0}
    dominant = max(timed, key=lambda k: ph[k])
    kind, amount = alg[dominant]
    if kind == "int32":
        achieved = amount / (ph[dominant] * 1e-3) / 1e9
        roof = {"bound": "int32", "kernel": dominant + " (lifted_leaves_kernel + node_layers_kernel)",
                "achieved": achieved, "peak": probe_rate / 1e9, "unit": "G Blake2s compressions/s",
                "frac": achieved * 1e9 / probe_rate,
                "peak_kind": "measured in this run (register-only Blake2s chain, all SMs)", "traffic": None,
                "alg_compressions_per_step": amount}
    else:
        achieved = amount / (ph[dominant] * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "peak_kind": peak_kind, "traffic": None,
                "alg_bytes_per_step": amount}
        if dominant == "trace_fft" and (n, nc, lb) == (20, 100, 1) and TRACE_FFT_TRAFFIC_100x2e20:
            # dram__bytes_read.sum + dram__bytes_write.sum of the three trace
            # FFT kernels, one ncu capture
            roof["traffic"] = TRACE_FFT_TRAFFIC_100x2e20
            roof["traffic_source"] = ("ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of the three "
                                      "trace FFT kernels on 40 columns of 2^20, scaled to 100 columns")
            roof["note"] = ("bound by integer issue, not HBM: the passes keep the ALU pipe 60-75% busy at about "
                            "8-10 instructions per M31 butterfly")
    # The trace FFTs against the butterfly ceiling: the interpolation runs n
    # layers of 2^(n-1) butterflies per column; the evaluation n layers of
    # 2^(n+lb-1) (its top lb layers only copy the zero-padded coefficients).
    fft_bflies = nc * n * ((1 << (n - 1)) + (1 << (n + lb - 1)))
    fft_ms = ph["trace_fft"]
    fft_issue = None
    if fft_ms > 0:
        fft_rate = fft_bflies / (fft_ms * 1e-3)
        fft_issue = {"bound": "int32 issue", "kernel": "trace interpolate + evaluate (fft_warp_contig_kernel, "
                     "fft_warp_inv_fwd_kernel)", "achieved": fft_rate / 1e9, "peak": bfly_rate / 1e9,
                     "unit": "G M31 butterflies/s", "frac": fft_rate / bfly_rate,
                     "peak_kind": "measured in this run (register-only butterfly chains, all SMs)",
                     "alg_butterflies_per_step": fft_bflies}
    phase_frac = {}
    for k, (kd, amt) in alg.items():
        if ph.get(k, 0) > 0:
            rate = amt / (ph[k] * 1e-3)
            phase_frac[k] = rate / (hbm_peak * 1e9) if kd == "hbm" else rate / probe_rate
    # The prover computes its twiddle tree (CanonicCoset(log_n + blowup + 1)
    # .half_coset) once at creation and keeps it resident, outside the timed
    # proofs; its device time is reported beside them.
    tw_ms = twiddle_precompute_ms(spec["log_n"] + spec["log_blowup"] + 1, stream)
    # the CPU baseline (and the byte comparison with it) is measured at N = 1 only
    cpu_s, cpu_proof, cpu_threads = cpu_prove(spec, a_host, b_host) if world == 1 else (None, None, None)
    srt = sorted(step_ms)
    line = {
        "metric": METRIC,
        "value": replica_rate(cells, ms_max, world),
        "unit": "proved trace cells/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32 (M31/QM31)",
        "data": "synthetic (seeded numpy PCG64)",
        "config": prove_config_json(spec, world),
        "p50_prove_ms": srt[len(srt) // 2],
        "p99_prove_ms": srt[min(len(srt) - 1, int(0.99 * len(srt)))],
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {"value": replica_rate(cells, e2e_ms, world), "unit": "proved trace cells/s",
                "h2d_bytes_per_step": int(a.nbytes + b.nbytes), "d2h_bytes_per_step": int(n_e2e),
                "ms_per_step": e2e_ms},
        "roofline": roof,
        "fft_issue_roofline": fft_issue,
        "phase_ms": phase_ms,
        "phase_roofline_frac": phase_frac,
        "twiddle_precompute_ms": tw_ms,
        "blake2s_probe_compressions_per_s": probe_rate,
        "butterfly_probe_per_s": bfly_rate,
        "proof_bytes": len(proof),
        "verifier": "accepted" if verdict is None else f"REJECTED: {verdict}",
        "bit_exact_vs_oracle": proof == cpu_proof if world == 1 else "checked at N=1",
        "cpu_baseline": ({"value": cells / cpu_s, "unit": "proved trace cells/s", "cores": cpu_threads,
                          "kind": "port",
                          "sample": f"one whole Wide-Fibonacci {spec['n_cols']} x 2^{spec['log_n']} proof (SimdBackend restatement, C++ oracle, "
                                    "OpenMP), same inputs; its proof bytes are compared with the GPU's"}
                         if world == 1 else None),
    }
    line.update(extras)
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ FRI-heavy -----
FRI_LOG, FRI_SEED, FRI_QUERIES = 24, 4, 70


def fri_config_json(world):
    return {"workload": "fri_heavy", "log_size": FRI_LOG, "n_queries": FRI_QUERIES,
            "folds": "circle-to-line, then line folds by 2 to log size 0; seeded QM31 alphas",
            "merkle": "lifted Blake2s tree per layer (24 trees)",
            "inputs": f"4 coordinate columns uniform [0, 2^31-1), alphas and positions seed {FRI_SEED}",
            "l2": "inputs larger than L2 (256 MB column; no flush)", "parallelism": f"replicas x{world}"}


def fri_units():
    # folded QM31 elements: every fold's input (2^24 + 2^23 + ... + 2)
    return (1 << (FRI_LOG + 1)) - 2


def cpu_fri(threads=None):
    from oracle import ffi as oracle
    n_threads = oracle.set_threads(threads or os.cpu_count() or 1)
    coords, alphas, queries = oracle.fri_inputs(FRI_LOG, FRI_SEED, FRI_QUERIES)
    t0 = time.perf_counter()
    proof = oracle.fri_prove_seeded(coords, FRI_LOG, alphas, queries)
    return time.perf_counter() - t0, proof, n_threads


def run_fri_reference(args, world, rank):
    if rank != 0:
        return
    secs, n_threads = [], 1
    for i in range(min(args.warmup, 1) + args.steps):
        t, _, n_threads = cpu_fri()
        if i >= min(args.warmup, 1):
            secs.append(t)
    med = statistics.median(secs)
    value = fri_units() / med
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "folded QM31 elements/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * med,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31/QM31)",
        "data": "synthetic (seeded numpy PCG64)", "config": fri_config_json(args.gpus),
        "cpu_baseline": {"value": value, "unit": "folded QM31 elements/s", "cores": n_threads, "kind": "port",
                         "sample": "each step: the whole log-24 FRI commit + 70-query decommit (SimdBackend "
                                   "restatement, C++ oracle, OpenMP)"},
        "e2e": {"value": value, "unit": "folded QM31 elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def blake2s_probe_rate(ffi, stream):
    """Integer-pipe ceiling for the Blake2s op mix: register-only compression
    chains on every SM (148 SMs x 8 blocks x 256 threads x 256 compressions)."""
    import ctypes
    import torch
    from stwo_b200 import DeviceBuffer
    sp = ctypes.c_void_p(stream.cuda_stream)
    probe_out = DeviceBuffer(64, stream.cuda_stream)
    for _ in range(2):
        ffi.call("stwo_b200_blake2s_probe", ctypes.c_uint32(148 * 8), ctypes.c_uint32(256),
                 ctypes.c_void_p(probe_out.ptr), sp)
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        p0.record(stream)
        ffi.call("stwo_b200_blake2s_probe", ctypes.c_uint32(148 * 8), ctypes.c_uint32(256),
                 ctypes.c_void_p(probe_out.ptr), sp)
        p1.record(stream)
    torch.cuda.synchronize()
    return 148 * 8 * 256 * 256 / (p0.elapsed_time(p1) * 1e-3)


def run_fri_b200(args, world, rank, local):
    import ctypes
    import torch
    from oracle import ffi as oracle
    from stwo_b200 import B200Backend, DeviceColumn, SeededFriProver, ffi

    torch.cuda.set_device(local)
    ffi.init(local)
    stream = torch.cuda.Stream()
    be = B200Backend(stream.cuda_stream)
    coords, alphas, queries = oracle.fri_inputs(FRI_LOG, FRI_SEED, FRI_QUERIES)
    init, lg = oracle.canonic_half_coset_root(FRI_LOG + 1)
    tree = be.precompute_twiddles(init, lg)
    fp = SeededFriProver(FRI_LOG, tree, stream=stream.cuda_stream)
    dev = [DeviceColumn.from_host(c, stream.cuda_stream) for c in coords]
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        proof = fp.prove(dev, alphas, queries)

    # ---- device-timed region: whole FRI commit + decommit, column resident ----
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches0 = ffi.launch_count()
    with torch.cuda.stream(stream):
        evs[0].record(stream)
        for k in range(args.steps):
            fp.prove(dev, alphas, queries)
            evs[k + 1].record(stream)
    torch.cuda.synchronize()
    launches = ffi.launch_count() - launches0
    clocks = sampler.stop()
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    ms = max_over_ranks(sum(step_ms) / args.steps, world)

    # ---- e2e: the column from pinned host memory, proof bytes to the host ----
    pinned = []
    for c in coords:
        t = torch.empty(c.size, dtype=torch.int32).pin_memory()
        t.numpy().view(np.uint32)[:] = c
        pinned.append(t)
    sp = ctypes.c_void_p(stream.cuda_stream)

    def e2e_step():
        for t, d in zip(pinned, dev):
            ffi.call("stwo_b200_memcpy_h2d", ctypes.c_void_p(d.ptr), ctypes.c_void_p(t.data_ptr()),
                     ctypes.c_size_t(d.nbytes), sp)
        return fp.prove(dev, alphas, queries)

    e2e_step()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            p_e2e = e2e_step()
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    assert p_e2e == proof, "e2e proof differs from the device-resident proof"
    probe_rate = blake2s_probe_rate(ffi, stream)

    if rank != 0:
        return
    # Dominant work: Blake2s (2^(k+1) - 1 compressions per tree of 2^k leaves,
    # one compression per 16-byte leaf); folds move 16 * 1.5 * 2^(k) bytes per
    # layer k and are a small share.
    compressions = sum((1 << (k + 1)) - 1 for k in range(1, FRI_LOG + 1))
    achieved = compressions / (ms * 1e-3) / 1e9
    roof = {"bound": "int32", "kernel": "Blake2s trees of every layer (lifted_leaves_kernel + node_layers_kernel)",
            "achieved": achieved, "peak": probe_rate / 1e9, "unit": "G Blake2s compressions/s",
            "frac": achieved * 1e9 / probe_rate,
            "peak_kind": "measured in this run (register-only Blake2s chain, all SMs)", "traffic": None,
            "alg_compressions_per_step": compressions,
            "note": "whole FRI step time (folds and decommit gather included) against the hash ceiling"}
    cpu_s, cpu_proof, cpu_threads = cpu_fri() if world == 1 else (None, None, None)  # N = 1 only
    units = fri_units()
    srt = sorted(step_ms)
    line = {
        "metric": METRIC, "value": replica_rate(units, ms, world), "unit": "folded QM31 elements/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31/QM31)",
        "data": "synthetic (seeded numpy PCG64)", "config": fri_config_json(world),
        "p50_ms": srt[len(srt) // 2], "p99_ms": srt[min(len(srt) - 1, int(0.99 * len(srt)))],
        "clocks": clocks, "gpu_launches": launches,
        "e2e": {"value": replica_rate(units, e2e_ms, world), "unit": "folded QM31 elements/s",
                "h2d_bytes_per_step": int(sum(d.nbytes for d in dev)), "d2h_bytes_per_step": len(proof),
                "ms_per_step": e2e_ms},
        "roofline": roof,
        "blake2s_probe_compressions_per_s": probe_rate,
        "proof_bytes": len(proof),
        "bit_exact_vs_oracle": proof == cpu_proof if world == 1 else "checked at N=1",
        "cpu_baseline": ({"value": units / cpu_s, "unit": "folded QM31 elements/s", "cores": cpu_threads,
                          "kind": "port",
                          "sample": "one whole log-24 FRI commit + 70-query decommit (SimdBackend restatement, C++ "
                                    "oracle, OpenMP), same inputs; its bytes are compared with the GPU's"}
                         if world == 1 else None),
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------- default-line extras -----
# The default run reports, beside the Wide-Fibonacci headline, the rest of the
# metric: the uneven 512-column commit in its batched, CUDA-graph and
# per-column forms (the "batched vs per-column" ratio), the FRI-heavy commit,
# and the FRI folds against HBM.  Bit-exactness at these sizes is checked
# against oracle digests committed in tests/golden/full_size_digests.json
# (made by tests/golden/make_full_size_digests.py; tests/test_gpu_full_size.py
# re-runs the oracle itself).
DIGESTS_PATH = os.path.join(ROOT, "tests", "golden", "full_size_digests.json")


def load_digests():
    if os.path.exists(DIGESTS_PATH):
        with open(DIGESTS_PATH) as f:
            return json.load(f)
    return {}


def fri_heavy_inputs(log_n=FRI_LOG, seed=FRI_SEED, n_queries=FRI_QUERIES):
    """The FRI-heavy inputs (numpy PCG64): 4 coordinate columns uniform in
    [0, P), one QM31 alpha per fold, sorted distinct query positions."""
    r = np.random.default_rng(seed)
    n = 1 << log_n
    coords = [r.integers(0, P, n, dtype=np.uint32) for _ in range(4)]
    alphas = r.integers(0, P, (log_n, 4), dtype=np.uint32)
    queries = np.unique(r.integers(0, n, n_queries, dtype=np.uint64))
    return coords, alphas, queries


def time_region(stream, fn, steps):
    """Mean device ms of `fn` over `steps` calls (CUDA events on `stream`)."""
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def extra_commit_uneven(args, stream, world, hbm_peak, probe_rate):
    """512 uneven columns (log 12..22, blowup 2, L = 24): per-column, batched
    and batched + graph committer forms, and the batched phases."""
    import torch
    from stwo_b200 import B200Backend, Committer, DeviceBuffer, DeviceColumn, fft_get_plan, ffi, layer_to_host
    from stwo_b200.backend import canonic_half_coset
    spec = workload_spec("commit_uneven")
    logs, blowup = spec["logs"], spec["blowup"]
    host_cols = make_columns(spec)
    be = B200Backend(stream.cuda_stream)
    L = max(logs) + blowup
    init, lg = canonic_half_coset(L + 1)
    tree = be.precompute_twiddles(init, lg)
    inputs = [DeviceColumn.from_host(c, stream.cuda_stream) for c in host_cols]
    coeffs = [DeviceColumn(c.size, stream.cuda_stream) for c in host_cols]
    evals = [DeviceColumn(c.size << blowup, stream.cuda_stream) for c in host_cols]
    layers = [DeviceBuffer(32 << k, stream.cuda_stream) for k in range(L + 1)]
    order = sorted(range(len(logs)), key=lambda i: logs[i])
    evals_sorted = [evals[i] for i in order]
    cells = sum(c.size for c in host_cols)
    eval_cells = cells << blowup
    del host_cols
    cms = {"per_column": Committer(logs, blowup, tree, per_column=True, stream=stream.cuda_stream),
           "batched": Committer(logs, blowup, tree, stream=stream.cuda_stream),
           "batched_graph": Committer(logs, blowup, tree, graph=True, stream=stream.cuda_stream)}
    torch.cuda.synchronize()
    t_tune = time.perf_counter()
    cms["batched_graph"].autotune(inputs, coeffs, evals, reps=2)
    torch.cuda.synchronize()
    tune_s = time.perf_counter() - t_tune
    steps = max(3, min(args.steps, 10))
    forms, roots = {}, {}
    for name, cm in cms.items():
        with torch.cuda.stream(stream):
            for _ in range(2):
                cm.commit(inputs, coeffs, evals, layers)
        torch.cuda.synchronize()
        l0 = ffi.launch_count()
        f_ms = max_over_ranks(time_region(stream, lambda: cm.commit(inputs, coeffs, evals, layers), steps), world)
        roots[name] = bytes(layer_to_host(layers[0])[0]).hex()
        forms[name] = {"ms_per_step": f_ms, "committed_cells_per_s": cells / (f_ms * 1e-3),
                       "launches_per_step": (ffi.launch_count() - l0) / steps}
        cm.close()
    # phases of the batched form through the per-op calls (the same launches)
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    phase_ms = {p: 0.0 for p in ("ifft", "rfft", "leaves", "nodes")}
    for _ in range(steps):
        with torch.cuda.stream(stream):
            marks[0].record(stream)
            be.interpolate_columns_into(inputs, coeffs, tree)
            marks[1].record(stream)
            be.evaluate_polynomials_into(coeffs, blowup, tree, evals)
            marks[2].record(stream)
            be.build_leaves_layers(evals_sorted, L, layers)
            marks[3].record(stream)
            be.build_nodes(layers)
            marks[4].record(stream)
        torch.cuda.synchronize()
        for i, ph in enumerate(phase_ms):
            phase_ms[ph] += marks[i].elapsed_time(marks[i + 1]) / steps
    root = bytes(layer_to_host(layers[0])[0]).hex()
    golden = load_digests().get("commit_uneven_root")
    alg = {"ifft": 8 * cells, "rfft": 4 * cells + 4 * eval_cells}
    compressions = lifted_leaf_compressions([x + blowup for x in logs], L)
    out = {
        "workload": "commit_uneven: 512 columns, log sizes U{12..22} seed 3, blowup 2, lifted Blake2s tree L=24",
        "committed_cells": cells,
        "forms": forms,
        "batched_over_per_column": forms["per_column"]["ms_per_step"] / forms["batched"]["ms_per_step"],
        "graph_over_per_column": forms["per_column"]["ms_per_step"] / forms["batched_graph"]["ms_per_step"],
        "phase_ms_batched": phase_ms,
        "phase_hbm_frac": {p: alg[p] / (phase_ms[p] * 1e-3) / (hbm_peak * 1e9) for p in alg},
        "leaves_vs_blake2s_ceiling": compressions / (phase_ms["leaves"] * 1e-3) / probe_rate,
        "autotune": {"seconds": tune_s, "plans": {str(n): fft_get_plan(n) for n in sorted(set(logs))}},
        "root": root,
        "roots_equal_across_forms": len(set(roots.values()) | {root}) == 1,
        "bit_exact_root_vs_oracle": (root == golden) if golden else "no oracle digest",
    }
    for x in inputs + coeffs + evals + layers:
        x.close()
    tree.twiddles.close()
    tree.itwiddles.close()
    return out


def extra_commit_plain(args, stream, world):
    """32 columns of log 16, natural order, blowup 1: interpolate (bit
    reversal in the first pass's loads), evaluate, lifted Blake2s tree."""
    from stwo_b200 import B200Backend, DeviceBuffer, DeviceColumn, layer_to_host
    from stwo_b200.backend import canonic_half_coset
    spec = workload_spec("commit_plain")
    logs, blowup = spec["logs"], spec["blowup"]
    host_cols = make_columns(spec)
    be = B200Backend(stream.cuda_stream)
    L = max(logs) + blowup
    init, lg = canonic_half_coset(L + 1)
    tree = be.precompute_twiddles(init, lg)
    inputs = [DeviceColumn.from_host(c, stream.cuda_stream) for c in host_cols]
    coeffs = [DeviceColumn(c.size, stream.cuda_stream) for c in host_cols]
    evals = [DeviceColumn(c.size << blowup, stream.cuda_stream) for c in host_cols]
    layers = [DeviceBuffer(32 << k, stream.cuda_stream) for k in range(L + 1)]

    def step():
        be.interpolate_natural_into(inputs, coeffs, tree)
        be.evaluate_polynomials_into(coeffs, blowup, tree, evals)
        be.build_leaves_layers(evals, L, layers)
        be.build_nodes(layers)

    for _ in range(3):
        step()
    steps = max(10, args.steps)
    ms = max_over_ranks(time_region(stream, step, steps), world)
    root = bytes(layer_to_host(layers[0])[0]).hex()
    golden = load_digests().get("commit_plain_root")
    cells = sum(c.size for c in host_cols)
    for x in inputs + coeffs + evals + layers:
        x.close()
    return {"workload": "commit_plain: 32 columns of log 16, natural order, blowup 1, lifted Blake2s tree L=17",
            "ms_per_step": ms, "committed_cells_per_s": cells / (ms * 1e-3), "root": root,
            "bit_exact_root_vs_oracle": (root == golden) if golden else "no oracle digest",
            "l2": "inputs smaller than L2 (8 MB trace; back-to-back steps, no flush): a latency figure"}


def extra_fri_heavy(args, stream, world, hbm_peak, probe_rate):
    """FRI-heavy commit + decommit (log 24, 70 queries) and the stand-alone
    FriOps folds at log 24 against HBM."""
    import hashlib
    from stwo_b200 import B200Backend, DeviceColumn, SeededFriProver
    from stwo_b200.backend import canonic_half_coset
    coords, alphas, queries = fri_heavy_inputs()
    be = B200Backend(stream.cuda_stream)
    init, lg = canonic_half_coset(FRI_LOG + 1)
    tree = be.precompute_twiddles(init, lg)
    half_init = canonic_half_coset(FRI_LOG)[0]  # the source domain's half coset (read below log 5 only)
    dev = [DeviceColumn.from_host(c, stream.cuda_stream) for c in coords]
    del coords
    fp = SeededFriProver(FRI_LOG, tree, stream=stream.cuda_stream)
    for _ in range(2):
        proof = fp.prove(dev, alphas, queries)
    steps = max(3, min(args.steps, 10))
    ms = max_over_ranks(time_region(stream, lambda: fp.prove(dev, alphas, queries), steps), world)
    fp.close()
    golden = load_digests().get("fri_heavy_sha256")
    folds = standalone_fold_roofline(stream, tree, dev, alphas[0], half_init, hbm_peak, steps=20)
    for x in dev:
        x.close()
    tree.twiddles.close()
    tree.itwiddles.close()
    compressions = sum((1 << (k + 1)) - 1 for k in range(1, FRI_LOG + 1))
    return {
        "workload": "fri_heavy: one QM31 column of log 24, circle fold + line folds by 2 to log 0, "
                    "70 query draws, seeded alphas",
        "ms_per_step": ms, "folded_elements_per_s": fri_units() / (ms * 1e-3),
        "trees_vs_blake2s_ceiling": compressions / (ms * 1e-3) / probe_rate,
        "bit_exact_vs_oracle": (hashlib.sha256(proof).hexdigest() == golden) if golden else "no oracle digest",
        "fold_roofline": folds,
    }


def standalone_fold_roofline(stream, tree, dev, alpha, half_init, hbm_peak, steps=20):
    """FriOps::fold_circle_into_line (2^k -> 2^(k-1), k = log size of `dev`)
    and FriOps::fold_line (2^(k-1) -> 2^(k-2)) through the C ABI, each timed
    alone with CUDA events, against HBM."""
    import ctypes
    from stwo_b200 import DeviceColumn, ffi
    from stwo_b200.backend import _ptr_array, _u32_array
    log_n = dev[0].log_size
    n = 1 << log_n
    line = [DeviceColumn(n >> 1, stream.cuda_stream) for _ in range(4)]
    out = [DeviceColumn(n >> 2, stream.cuda_stream) for _ in range(4)]
    sp = ctypes.c_void_p(stream.cuda_stream)
    a0 = _u32_array(alpha)

    def circle():
        ffi.call("stwo_b200_fold_circle_into_line", _ptr_array(line), _ptr_array(dev), ctypes.c_uint32(log_n),
                 ctypes.c_uint64(half_init), a0, ctypes.c_void_p(tree.itwiddles.ptr), ctypes.c_uint32(tree.log_size), sp)

    def fold():
        ffi.call("stwo_b200_fold_line", _ptr_array(line), ctypes.c_uint32(log_n - 1), a0, ctypes.c_uint32(1),
                 ctypes.c_void_p(tree.itwiddles.ptr), ctypes.c_uint32(tree.log_size), _ptr_array(out), sp)

    for _ in range(3):
        circle()
        fold()
    c_ms = time_region(stream, circle, steps)
    f_ms = time_region(stream, fold, steps)
    # algorithmic bytes: the circle fold reads 16 B per input and reads and
    # writes 16 B per output (dst <- dst * alpha^2 + f'); the line fold reads
    # 16 B per input and writes 16 B per output
    c_bytes = 16 * n + 32 * (n >> 1)
    f_bytes = 16 * (n >> 1) + 16 * (n >> 2)
    for x in line + out:
        x.close()
    return {
        f"fold_circle_into_line_log{log_n}": {"ms": c_ms, "alg_bytes": c_bytes,
                                              "achieved_gbs": c_bytes / (c_ms * 1e-3) / 1e9,
                                              "frac": c_bytes / (c_ms * 1e-3) / (hbm_peak * 1e9)},
        f"fold_line_log{log_n - 1}": {"ms": f_ms, "alg_bytes": f_bytes, "achieved_gbs": f_bytes / (f_ms * 1e-3) / 1e9,
                                      "frac": f_bytes / (f_ms * 1e-3) / (hbm_peak * 1e9)},
        "peak": hbm_peak, "unit": "GB/s",
        "kernels": "fold_circle_kernel, fold_line_kernel (the FriOps entry points; the prover's fused fold + "
                   "next-layer leaf hash kernels are in phase_roofline_frac)",
    }


def run_fri_fold_b200(args, world, rank, local):
    """The stand-alone FriOps folds at the FRI-heavy size (one QM31 column of
    log 24): the HBM-streaming kernels alone, for their roofline and profile."""
    import torch
    from stwo_b200 import B200Backend, DeviceColumn, ffi
    from stwo_b200.backend import canonic_half_coset
    torch.cuda.set_device(local)
    ffi.init(local)
    stream = torch.cuda.Stream()
    be = B200Backend(stream.cuda_stream)
    coords, alphas, _ = fri_heavy_inputs()
    init, lg = canonic_half_coset(FRI_LOG + 1)
    tree = be.precompute_twiddles(init, lg)
    dev = [DeviceColumn.from_host(c, stream.cuda_stream) for c in coords]
    torch.cuda.synchronize()
    launches0 = ffi.launch_count()
    r = standalone_fold_roofline(stream, tree, dev, alphas[0], canonic_half_coset(FRI_LOG)[0], load_peaks()[0],
                                 steps=args.steps)
    launches = ffi.launch_count() - launches0
    if rank != 0:
        return
    c = r[f"fold_circle_into_line_log{FRI_LOG}"]
    units = 1 << FRI_LOG
    print(json.dumps({
        "metric": METRIC, "value": replica_rate(units, c["ms"], world), "unit": "folded QM31 elements/s",
        "n_gpus": world, "steps": args.steps, "warmup": 3, "ms_per_step": c["ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31/QM31)", "data": "synthetic (seeded numpy PCG64)",
        "config": {"workload": "fri_fold", "log_size": FRI_LOG, "parallelism": f"replicas x{world}"},
        "gpu_launches": launches, "roofline": {"bound": "hbm", "kernel": "fold_circle_kernel",
                                               "achieved": c["achieved_gbs"], "peak": r["peak"], "unit": "GB/s",
                                               "frac": c["frac"], "traffic": None, "alg_bytes_per_step": c["alg_bytes"]},
        "folds": r}), flush=True)


# ------------------------------------------------------------- trace FFT ----
def trace_fft_setup(args):
    r = np.random.default_rng(1)
    return r.integers(0, P, 1 << args.log_n_rows, dtype=np.uint32)


def run_trace_fft_b200(args, world, rank, local):
    """The trace transforms of the prover alone: interpolate n_cols columns of
    2^log_n bit-reversed evaluations into coefficients, then evaluate them on
    the blowup domain.  Timed twice: as the one call the prover makes
    (stwo_b200_interpolate_evaluate_columns, whose interpolation's last pass
    and evaluation's first share a kernel at logs 20 and 21) -- the line's
    value -- and as the two trait calls (interpolate_columns, then
    evaluate_polynomials)."""
    import torch
    from stwo_b200 import B200Backend, DeviceColumn, ffi, fft_get_plan
    from stwo_b200.backend import canonic_half_coset
    torch.cuda.set_device(local)
    ffi.init(local)
    stream = torch.cuda.Stream()
    be = B200Backend(stream.cuda_stream)
    log_n, nc, lb = args.log_n_rows, args.n_cols, args.log_blowup
    init, lg = canonic_half_coset(log_n + lb + 1)
    tree = be.precompute_twiddles(init, lg)
    host = trace_fft_setup(args)
    evals = [DeviceColumn.from_host(host, stream.cuda_stream) for _ in range(nc)]
    coeffs = [DeviceColumn(1 << log_n, stream.cuda_stream) for _ in range(nc)]
    outs = [DeviceColumn(1 << (log_n + lb), stream.cuda_stream) for _ in range(nc)]
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        be.interpolate_columns_into(evals, coeffs, tree)
        be.evaluate_polynomials_into(coeffs, lb, tree, outs)
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ti = te = 0.0
    launches0 = ffi.launch_count()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            evs[0].record(stream)
            be.interpolate_columns_into(evals, coeffs, tree)
            evs[1].record(stream)
            be.evaluate_polynomials_into(coeffs, lb, tree, outs)
            evs[2].record(stream)
        torch.cuda.synchronize()
        ti += evs[0].elapsed_time(evs[1])
        te += evs[1].elapsed_time(evs[2])
    for _ in range(args.warmup):
        be.interpolate_evaluate_into(evals, coeffs, lb, tree, outs)
    torch.cuda.synchronize()
    tf = 0.0
    launches0 = ffi.launch_count()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            evs[0].record(stream)
            be.interpolate_evaluate_into(evals, coeffs, lb, tree, outs)
            evs[1].record(stream)
        torch.cuda.synchronize()
        tf += evs[0].elapsed_time(evs[1])
    launches = ffi.launch_count() - launches0
    ti, te = max_over_ranks(ti / args.steps, world), max_over_ranks(te / args.steps, world)
    tf = max_over_ranks(tf / args.steps, world)
    if rank != 0:
        return
    hbm_peak, peak_kind = load_peaks()
    n = 1 << log_n
    alg_i, alg_e = 8 * nc * n, 4 * nc * n + 4 * nc * (n << lb)
    bflies = nc * log_n * (n // 2 + (n << lb) // 2)
    cells = nc * n
    line = {
        "metric": METRIC, "value": replica_rate(cells, tf, world), "unit": "transformed trace cells/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tf,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31)",
        "data": "synthetic (seeded numpy PCG64)",
        "config": {"workload": "trace_fft", "n_columns": nc, "log_n_rows": log_n, "log_blowup": lb,
                   "parallelism": f"replicas x{world}"},
        "gpu_launches": launches,
        "two_calls_ms": {"interpolate": ti, "evaluate": te, "sum": ti + te},
        "pass_plan_layers": fft_get_plan(log_n),
        "two_calls_hbm_frac": {"interpolate": alg_i / (ti * 1e-3) / (hbm_peak * 1e9),
                               "evaluate": alg_e / (te * 1e-3) / (hbm_peak * 1e9)},
        "roofline": {"bound": "hbm", "kernel": "trace interpolate + evaluate (one call)",
                     "achieved": (alg_i + alg_e) / (tf * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                     "frac": (alg_i + alg_e) / (tf * 1e-3) / (hbm_peak * 1e9), "peak_kind": peak_kind,
                     "traffic": None, "alg_bytes_per_step": alg_i + alg_e},
        "butterflies_per_s": bflies / (tf * 1e-3),
    }
    print(json.dumps(line), flush=True)


def run_trace_fft_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import ffi as oracle
    n_threads = oracle.set_threads(os.cpu_count() or 1)
    log_n = args.log_n_rows
    init, lg = oracle.canonic_half_coset_root(log_n + args.log_blowup + 1)
    tw, itw = oracle.precompute_twiddles(init, lg)
    host = trace_fft_setup(args)
    k = max(1, min(args.n_cols, 8))  # a bounded sample of the columns per step
    secs = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        co = oracle.interpolate_columns([host] * k, itw)
        oracle.evaluate_columns(co, args.log_blowup, tw)
        if i >= args.warmup:
            secs.append(time.perf_counter() - t0)
    med = statistics.median(secs)
    value = k * (1 << log_n) / med
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "transformed trace cells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * med * args.n_cols / k,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31)",
        "data": "synthetic (seeded numpy PCG64)",
        "config": {"workload": "trace_fft", "n_columns": args.n_cols, "log_n_rows": log_n, "log_blowup": 1},
        "cpu_baseline": {"value": value, "unit": "transformed trace cells/s", "cores": n_threads, "kind": "port",
                         "sample": f"per step {k} of the {args.n_cols} columns (SimdBackend restatement, OpenMP)"},
        "e2e": {"value": value, "unit": "transformed trace cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# --------------------------------------------------------------- serving -----
SERVE_SEED, SERVE_SLOTS, SERVE_BUDGET = 5, 3, 120 << 30


def serving_requests(n):
    """Seeded prove requests: width U{64..256}, log_n_rows U{14..22}; inputs are
    generated per request from the request's own seed."""
    r = np.random.default_rng(SERVE_SEED)
    return [(int(r.integers(14, 23)), int(r.integers(64, 257)), 10_000 + i) for i in range(n)]


def serving_inputs(log_n, seed):
    r = np.random.default_rng(seed)
    n = 1 << log_n
    return r.integers(0, P, n, dtype=np.uint32), r.integers(0, P, n, dtype=np.uint32)


def run_stream(srv, reqs, inputs, arrivals):
    """Submits reqs at the given arrival offsets (seconds) to the server and
    collects every proof and its latency; returns (proofs, times, makespan_s, stats)."""
    from stwo_b200 import wide_fib_config
    tickets = [None] * len(reqs)
    t0 = time.perf_counter()
    for i, (ln, nc, _) in enumerate(reqs):
        delay = arrivals[i] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        a, b = inputs[i]
        tickets[i] = srv.submit(wide_fib_config(ln, nc), a, b)
    out = [srv.wait(t) for t in tickets]
    makespan = time.perf_counter() - t0
    return [o[0] for o in out], [o[1] for o in out], makespan, srv.stats()


def run_serving_b200(args, world, rank, local):
    import torch
    from stwo_b200 import ffi
    torch.cuda.set_device(local)
    ffi.init(local)
    line = measure_serving(max(24, 8 * args.steps), args.warmup, world, local, with_cpu=True)
    if rank != 0:
        return
    line.update({"steps": args.steps, "warmup": args.warmup})
    print(json.dumps(line), flush=True)


def measure_serving(n_req, warmup, world, local, with_cpu):
    """One Poisson stream of n_req seeded requests through the batched server
    and through serial proving on the same GPU (see the serving workload)."""
    import torch
    from oracle import ffi as oracle
    from stwo_b200 import ffi
    reqs = serving_requests(n_req)
    inputs = [serving_inputs(ln, sd) for ln, _, sd in reqs]
    cells = sum(nc << ln for ln, nc, _ in reqs)
    from stwo_b200 import ProveServer
    batched = ProveServer(SERVE_BUDGET, slots=SERVE_SLOTS)
    serial = ProveServer(SERVE_BUDGET, slots=1)
    # warm-up: the whole request list once through each server (resident
    # provers built up to the budget, kernels loaded, FRI graphs captured)
    for _ in range(max(1, min(warmup, 2))):
        run_stream(batched, reqs, inputs, [0.0] * n_req)
        run_stream(serial, reqs, inputs, [0.0] * n_req)
    # capacity: everything submitted at once, serial (1 slot) and batched
    barrier(world)
    torch.cuda.synchronize()
    p_ser, t_ser_sat, mk_ser, _ = run_stream(serial, reqs, inputs, [0.0] * n_req)
    p_sat, t_sat, mk_sat, st_sat = run_stream(batched, reqs, inputs, [0.0] * n_req)
    cap_batched = n_req / mk_sat
    # Poisson arrivals at 70% of the batched capacity, the same schedule for
    # the batched server and for serial proving.
    rate = 0.7 * cap_batched
    gaps = np.random.default_rng(SERVE_SEED + 1).exponential(1.0 / rate, n_req)
    arrivals = np.cumsum(gaps) - gaps[0]
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = ffi.launch_count()
    p_srv, t_srv, mk_srv, st_srv = run_stream(batched, reqs, inputs, arrivals)
    launches = ffi.launch_count() - launches0
    clocks = sampler.stop()
    p_ser2, t_ser2, mk_ser2, _ = run_stream(serial, reqs, inputs, arrivals)
    batched.close()
    serial.close()
    barrier(world)
    exact_mix = all(a == b for a, b in zip(p_srv, p_ser)) and all(a == b for a, b in zip(p_sat, p_ser))
    exact_serial = all(a == b for a, b in zip(p_ser2, p_ser))
    rejected = [i for i, (ln, nc, _) in enumerate(reqs)
                if oracle.verify_wide_fib(p_srv[i], ln, nc) is not None]

    def pct(xs, q):
        xs = sorted(xs)
        return xs[min(len(xs) - 1, int(q * len(xs)))]

    lat = [t["latency_ms"] for t in t_srv]
    lat_ser = [t["latency_ms"] for t in t_ser2]
    small = min(range(n_req), key=lambda i: reqs[i][1] << reqs[i][0])
    line = {
        "metric": METRIC, "value": cells / mk_srv * world, "unit": "proved trace cells/s",
        "n_gpus": world, "ms_per_step": 1000 * mk_srv,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31/QM31)",
        "data": "synthetic (seeded numpy PCG64)",
        "config": {"workload": "serving", "requests": n_req, "widths": "U{64..256}", "log_n_rows": "U{14..22}",
                   "seed": SERVE_SEED, "arrivals": "Poisson at 70% of the measured batched capacity",
                   "slots": SERVE_SLOTS, "hbm_budget_bytes": SERVE_BUDGET,
                   "step": f"one stream of {n_req} requests (host steady clock, submit to proof bytes)",
                   "parallelism": f"replicas x{world}"},
        "p50_latency_ms": pct(lat, 0.5), "p99_latency_ms": pct(lat, 0.99),
        "proofs_per_s": n_req / mk_srv,
        "serial": {"p50_latency_ms": pct(lat_ser, 0.5), "p99_latency_ms": pct(lat_ser, 0.99),
                   "proofs_per_s": n_req / mk_ser2, "saturated_proofs_per_s": n_req / mk_ser},
        "capacity_proofs_per_s": {"batched": cap_batched, "serial": n_req / mk_ser},
        "server_stats": st_srv,
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {"value": cells / mk_srv * world, "unit": "proved trace cells/s",
                "h2d_bytes_per_step": int(sum(8 << ln for ln, _, _ in reqs)),
                "d2h_bytes_per_step": int(sum(len(p) for p in p_srv)), "ms_per_step": 1000 * mk_srv},
        "bit_exact_mix_vs_alone": exact_mix and exact_serial,
        "verifier_rejected": rejected,
    }
    if with_cpu:
        # CPU baseline: the oracle proving the smallest request of the stream
        ln, nc, _ = reqs[small]
        a, b = inputs[small]
        n_threads = oracle.set_threads(os.cpu_count() or 1)
        t0 = time.perf_counter()
        cpu_proof = oracle.prove_wide_fib(oracle.wide_fib_config(ln, nc), a, b)
        cpu_s = time.perf_counter() - t0
        line["bit_exact_vs_oracle_sample"] = cpu_proof == p_srv[small]
        line["cpu_baseline"] = {"value": (nc << ln) / cpu_s, "unit": "proved trace cells/s", "cores": n_threads,
                                "kind": "port", "sample": f"the stream's smallest request ({nc} x 2^{ln}) proved by "
                                                          "the SimdBackend restatement (C++ oracle, OpenMP)"}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="wide_fib_prove",
                    choices=["wide_fib_prove", "commit_uneven", "commit_plain", "fri_heavy", "serving", "trace_fft",
                             "fri_fold"])
    ap.add_argument("--log-n-rows", type=int, default=20, help="wide_fib_prove: log2 of the trace rows")
    ap.add_argument("--n-cols", type=int, default=100, help="wide_fib_prove: trace columns")
    ap.add_argument("--log-blowup", type=int, default=1, help="trace_fft: log blowup of the evaluation")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="wide_fib_prove: skip the uneven-commit and FRI-heavy measurements of the default line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    try:
        if args.workload == "wide_fib_prove":
            if args.impl == "reference":
                run_prove_reference(args, world, rank)
            else:
                run_prove_b200(args, world, rank, local)
        elif args.workload == "serving":
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop; "
                                      "the oracle's per-proof rate is reported as cpu_baseline by the b200 arm"}))
            else:
                run_serving_b200(args, world, rank, local)
        elif args.workload == "fri_fold":
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "unavailable": "kernel profile target; the oracle's "
                                      "FRI rate is the fri_heavy workload's reference arm"}))
            else:
                run_fri_fold_b200(args, world, rank, local)
        elif args.workload == "trace_fft":
            if args.impl == "reference":
                run_trace_fft_reference(args, world, rank)
            else:
                run_trace_fft_b200(args, world, rank, local)
        elif args.workload == "fri_heavy":
            if args.impl == "reference":
                run_fri_reference(args, world, rank)
            else:
                run_fri_b200(args, world, rank, local)
        else:
            spec = workload_spec(args.workload)
            if args.impl == "reference":
                run_reference(args, spec, world, rank)
            else:
                run_b200(args, spec, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
