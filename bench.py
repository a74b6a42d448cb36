"""Benchmark of the B200 statevector engine: gates/s on the random-circuit
workload at n = 32, and trajectories/s of the batching form.

One step = one run of the seeded random layer circuit (n qubits, depth 20:
per layer one of H/S/T/SQRT_X/RZ on every qubit, then CZ on a random perfect
matching; n + n/2 gates per layer) on the device state.  The register is 32
qubits: 64 GiB in complex128 (plain path) or 32 GiB in complex64 (fused
precision form), far larger than L2, so no flush is needed between steps.

The trajectories/s part: one step = one run of 4096 noisy trajectories of
13..26-qubit registers (n = 16 + gen_range(0..7), depth 30, DEPOLARIZE2(1e-3)
after every CZ, M on every qubit) in the batching form's persistent kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  For N > 1 (torchrun, one rank per GPU) every rank runs
an independent replica with its own seed (weak scaling; the path has no
data exchange between replicas) and the time is the max over ranks.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "gates/s & %HBM peak, FP32-fused vs FP64, n=32 (1−F≤1e-6); trajectories/s"
FALLBACK_HBM_GBS = 6650.0


def _dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


RANK, WORLD, LOCAL_RANK = _dist_env()
if WORLD > 1 and "CUDA_VISIBLE_DEVICES" not in os.environ:
    # one GPU per rank: the engine uses device 0 of its own runtime
    os.environ["CUDA_VISIBLE_DEVICES"] = str(LOCAL_RANK)

sys.path.insert(0, ROOT)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from a committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, device_index: int = 0):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                idx = int(parts[0])
            except ValueError:
                continue
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            want = int(vis.split(",")[0]) if vis and vis.split(",")[0].isdigit() else device_index
            if idx != want:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                pass
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    if WORLD <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return dist


def max_over_ranks(dist, v: float) -> float:
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def pick_n(nb, want: int, precision_bytes: int, states: int) -> int:
    free = nb.device_info()["free_bytes"]
    n = want
    while n > 20 and states * (precision_bytes << n) + (6 << 30) > free:
        n -= 1
    return n


def host_mem_available() -> int:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def layer_sample_text(n: int, depth: int, seed: int, ones: int) -> str:
    """A sample of the random layer circuit with its own gate mix: from each
    layer in turn, its next one-qubit gates and CZ gates in the layer's 2:1
    ratio (`ones` one-qubit gates and ones // 2 CZ gates in all), in circuit
    order.  Run from |+>^n, every gate acts on a dense register."""
    from oracle import oracle as O

    lines = O.random_circuit_text(n, depth, seed).strip().split("\n")
    per = n + n // 2
    body = lines[1:]
    out, want1, want2 = [], ones, ones // 2
    for L in range(depth):
        layer = body[L * per:(L + 1) * per]
        one = [ln for ln in layer if not ln.startswith("CZ ")]
        two = [ln for ln in layer if ln.startswith("CZ ")]
        a, b = min(want1, len(one)), min(want2, len(two))
        out += one[:a] + two[:b]
        want1 -= a
        want2 -= b
        if want1 <= 0 and want2 <= 0:
            break
    return lines[0] + "\n" + "\n".join(out) + "\n"


def cpu_baseline(n_want: int, depth: int, seed: int, budget_s: float = 15.0):
    """The oracle (C++ restatement of the reference's StateVector, all host
    threads) on a bounded sample of the same workload: one-qubit gates and CZ
    gates of the same circuit in its 2:1 ratio, applied to a dense register
    (|+>^n), complex128.  The sample grows until it takes about budget_s."""
    from oracle import oracle as O

    avail = host_mem_available()
    n = n_want
    while n > 20 and (16 << n) * 1.3 > avail:
        n -= 1
    s = O.StateVector.plus_state(n)
    ones, elapsed, gates = 2, 0.0, 0
    while True:
        text = layer_sample_text(n, depth, seed, ones)
        c = O.Circuit(text)
        dt = s.run_gates_timed(c, c.num_gates)
        elapsed, gates = dt, c.num_gates
        if dt >= budget_s / 3 or ones >= 4 * n:
            break
        ones = max(ones + 2, int(ones * min(8.0, budget_s / 3 / max(dt, 1e-3))))
        ones += ones & 1
    n1 = sum(1 for ln in text.split("\n")[1:] if ln and not ln.startswith("CZ "))
    return {
        "value": gates / elapsed,
        "unit": "gates/s",
        "cores": O.lib().oracle_num_threads(),
        "kind": "port",
        "sample": f"oracle StateVector<C64> (complex128) at n={n}: {gates} gates of the random layer circuit "
                  f"(depth {depth}, seed {seed}) in its own mix ({n1} one-qubit, {gates - n1} CZ), on a dense "
                  f"register (|+>^n), in {elapsed:.1f} s"
                  + ("" if n == n_want else f" (n reduced from {n_want} to fit host memory)"),
        "n": n,
    }


def published_workload_text(n: int) -> str:
    """The reference's published StateVector workload (examples/bench.rs:120-137):
    H on every qubit, then for q in 0..n: T q, CX q (q+1)%n, CCZ q (q+1)%n (q+2)%n,
    RX(0.3) q."""
    h = "".join(f"H {q}\n" for q in range(n))
    layer = "".join(f"T {q}\nCX {q} {(q + 1) % n}\nCCZ {q} {(q + 1) % n} {(q + 2) % n}\nRX(0.3) {q}\n"
                    for q in range(n))
    return f"QUBITS {n}\n", h, layer


def published_workload_cpu(n: int = 22, reps: int = 3):
    """The same workload on the oracle (host threads): seconds for the 4n-gate layer
    and for one expectation of X0*Y3*Z5."""
    from oracle import oracle as O

    hdr, h, layer = published_workload_text(n)
    s = O.StateVector(n)
    s.run(O.Circuit(hdr + h), O.StdRng(0))
    c = O.Circuit(hdr + layer)
    t_layer = min(s.run_gates_timed(c, c.num_gates) for _ in range(reps))
    t0 = time.perf_counter()
    for _ in range(20):
        s.expectation("X0*Y3*Z5")
    t_exp = (time.perf_counter() - t0) / 20
    return {"layer_s": t_layer, "expectation_s": t_exp, "cores": O.lib().oracle_num_threads(), "kind": "port"}


def run_reference(args):
    """--impl reference: the reference's CPU path (the oracle port) on host cores."""
    if RANK != 0:
        return 0
    from oracle import oracle as O

    O.lib()
    vals = []
    sample = None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(args.n, args.depth, 1, budget_s=args.cpu_budget)
        if i >= args.warmup:
            vals.append(r["value"])
        sample = r
    v = statistics.median(vals)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "gates/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 / v,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"random layers n={sample['n']} depth {args.depth} seed 1 (complex128)",
                   "n": sample["n"], "depth": args.depth},
        "cpu_baseline": {"value": v, "unit": "gates/s", "cores": sample["cores"], "kind": "port",
                         "sample": sample["sample"]},
        "e2e": {"value": v, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_trajectories:
        tr = cpu_trajectories(30, 1e-3, args.cpu_budget * 2 / 3)
        tr.pop("results")
        line["trajectories"] = {"metric": "trajectories/s", "value": tr["value"], "unit": "trajectories/s",
                                "cpu_baseline": tr,
                                "e2e": {"value": tr["value"], "unit": "trajectories/s",
                                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_trajectories(depth: int, p: float, budget_s: float = 10.0, seed0: int = 1):
    """The oracle's noisy trajectories (FP64, the reference's StateVector
    semantics, all host threads) on the host cores: seeds seed0, seed0+1, ...
    until about budget_s seconds have passed.  `results` holds each one's
    (n, <Z0>/norm before the measurements, record)."""
    from oracle import oracle as O

    t0 = time.perf_counter()
    results = []
    while time.perf_counter() - t0 < budget_s:
        results.append(O.trajectory(seed0 + len(results), 16, 7, depth, p))
    dt = time.perf_counter() - t0
    done = len(results)
    return {"value": done / dt, "unit": "trajectories/s", "cores": O.lib().oracle_num_threads(), "kind": "port",
            "sample": f"oracle trajectories seeds {seed0}..{seed0 + done - 1} (n = 16 + gen_range(0..7), depth "
                      f"{depth}, DEPOLARIZE2({p}), M on every qubit) in {dt:.1f} s",
            "results": results}


def trajectory_fp64_reference(nb, count: int, seed0: int, depth: int, p: float, workers: int = 8):
    """<Z0>/<psi|psi> before the final measurements and the record of
    trajectories 0..count-1 (StdRng(seed0 + t)) on the plain complex128 path,
    from `workers` host threads (one register per size and thread, so the
    small registers' kernels overlap)."""
    import concurrent.futures as cf

    import numpy as np

    z = np.empty(count)
    rec = np.empty(count, dtype=np.uint64)

    def work(start):
        states, meas = {}, {}
        for t in range(start, count, workers):
            rng = nb.StdRng(seed0 + t)
            n = 16 + rng.gen_range(0, 7)
            c = nb.Circuit.random_layers_from(rng, n, depth, p, 0, 0)
            s = states.get(n)
            if s is None:
                s = states[n] = nb.GpuStateVector(n, nb.C128)
                meas[n] = nb.Circuit.parse(f"QUBITS {n}\n" + "".join(f"M {q}\n" for q in range(n)))
            else:
                s.set_basis(0)
            s.run(c, rng)
            z[t] = s.expectation(nb.Pauli(n, 0, 1, 0)).real / s.norm_sq().real
            r = s.run(meas[n], rng)
            rec[t] = sum(int(v) << k for k, v in enumerate(r))

    with cf.ThreadPoolExecutor(workers) as ex:
        list(ex.map(work, range(workers)))
    return z, rec


def trajectory_bench(nb, args, dist, peak, peak_kind):
    """The batching form: `count` noisy trajectories (trajectory t draws from
    StdRng(seed0 + t): n = 16 + gen_range(0..7), the random layer circuit of
    depth 30 with DEPOLARIZE2(1e-3) after every CZ, M on every qubit) in one
    persistent kernel.  A step is one run of the whole batch (one CUDA graph
    launch); states start at |0...0> in the kernel, the programs are resident."""
    count, depth, p = args.traj_count, 30, 1e-3
    seed0 = 1 + RANK * count
    t0 = time.perf_counter()
    tb = nb.TrajectoryBatch.random_layers(count, seed0, 16, 7, depth, p)
    build_s = time.perf_counter() - t0
    info = tb.info()
    if args.traj_launch:
        ctas, bufs = (int(v) for v in args.traj_launch.split(","))
        tb.set_config(ctas_per_sm=ctas, buffers=bufs)
    tb.run()  # tunes the planner's knobs per register size and the launch configuration on first use
    cfg = tb.config()
    sizes = sorted(set(int(v) for v in tb.qubits()))
    knobs = {str(n): tb.knobs(n) for n in sizes}
    for _ in range(args.warmup):
        tb.run()
    barrier(dist)
    ms = [tb.run() for _ in range(args.steps)]
    ms_mean = max_over_ranks(dist, statistics.mean(ms))
    value = WORLD * count / (ms_mean / 1e3)
    n_t, rec, z0, norm = tb.results()
    achieved = info["state_bytes"] / (ms_mean / 1e3) / 1e9
    out = {
        "metric": "trajectories/s",
        "value": value,
        "unit": "trajectories/s",
        "ms_per_step": ms_mean,
        "steps": args.steps,
        "warmup": args.warmup,
        "dtype": "f32 amplitudes (complex64), FP64 reductions",
        "config": {"workload": f"{count} noisy trajectories per GPU, n = 16 + gen_range(0..7), random layers "
                               f"depth {depth}, DEPOLARIZE2({p}) after every CZ, M on every qubit; "
                               f"StdRng(seed0 + t), seed0 = {seed0}",
                   "count": count, "depth": depth, "p": p, "launch": cfg,
                   "planner_knobs_by_size": {n: {"set": k["knob_set"], "window_step": k["window_step"],
                                                 "greedy_stages": k["greedy_stages"],
                                                 "timed_ms": [round(v, 3) for v in k["timed_ms"]]}
                                             for n, k in knobs.items()},
                   "l2": "about 1 TB of state traffic per step (no flush needed)"},
        "gpu_launches_per_step": 1,
        "plan": {k: info[k] for k in ("source_gates", "noise_events", "folded_ops", "passes", "tile_passes",
                                      "tile_stages", "program_bytes")},
        "roofline": {"bound": "hbm", "kernel": "k_batch", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": profiled_traffic("k_batch"),
                     "algorithmic_bytes_per_launch": info["state_bytes"]},
        "host_build_s": build_s,
    }
    # accuracy: every trajectory against a complex128 run of the same draws on the plain path
    if args.traj_check:
        t1 = time.perf_counter()
        check = min(count, args.traj_check)
        z_ref, rec_ref = trajectory_fp64_reference(nb, check, seed0, depth, p)
        zb = z0[:check]
        same = int((rec[:check] == rec_ref).sum())
        out["accuracy"] = {
            "reference": "plain complex128 path (FP64) per trajectory, same draws (StdRng(seed0 + t))",
            "trajectories": check,
            "mean_z0_error": abs(float(zb.mean()) - float(z_ref.mean())),
            "max_z0_error": float(abs(zb - z_ref).max()),
            "records_identical": f"{same}/{check}",
            "mean_norm_drift": float(abs(norm - 1.0).mean()),
            "check_s": round(time.perf_counter() - t1, 1),
        }
    if not args.no_e2e:
        def e2e_step():
            b = nb.TrajectoryBatch.random_layers(count, seed0, 16, 7, depth, p)  # host generation in
            b.set_config(ctas_per_sm=cfg["ctas_per_sm"], buffers=cfg["buffers"], order=cfg["order"])
            b.run()  # program upload, the graph, result copies
            return b.results()  # results out

        e2e_step()
        barrier(dist)
        t1 = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 2))
        for _ in range(e2e_steps):
            e2e_step()
        dt = max_over_ranks(dist, time.perf_counter() - t1)
        out["e2e"] = {"value": WORLD * e2e_steps * count / dt, "unit": "trajectories/s",
                      "h2d_bytes_per_step": info["program_bytes"], "d2h_bytes_per_step": count * 28,
                      "note": "per step: generate and compile the trajectories on the host, upload the "
                              "program, run, copy records, <Z0> and norms back; host wall clock"}
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        cpu = cpu_trajectories(depth, p, args.cpu_budget * 2 / 3, seed0)
        res = cpu.pop("results")
        if res:
            errs = [abs(z0[t] - zo) for t, (_, zo, _) in enumerate(res)]
            same = sum(int(rec[t]) == sum(int(v) << k for k, v in enumerate(ro)) for t, (_, _, ro) in enumerate(res))
            out["accuracy_oracle"] = {"reference": "the CPU oracle (FP64 restatement of StateVector) on the same "
                                                   "draws: the CPU baseline's trajectories",
                                      "trajectories": len(res), "max_z0_error": max(errs),
                                      "records_identical": f"{same}/{len(res)}"}
        out["cpu_baseline"] = cpu
    return out


FRAMES_PUBLISHED_MS = 31.0  # the reference's README: 100 000 shots of this circuit on a 16-thread desktop


def frames_bench(nb, args, dist, peak, peak_kind):
    """The reference's frame-sampler benchmark (examples/bench.rs:264-294):
    1000 qubits, 20 rounds of 500 CX + DEPOLARIZE2(1e-3) and 100 Z
    measurements (10 500 gates, 2000 measurements), 100 000 shots per step.
    A step is one sample_packed call: the host scan of the seven batches'
    random streams (noise hits, mask positions), their upload, the mask and
    frame kernels; the packed records stay on the device for `value` and come
    back to host memory for `e2e`.  The reference record (FrameSampler::new)
    is built once, outside the timed region, as the reference times it apart."""
    import numpy as np
    import torch

    shots = 100_000
    c = nb.Circuit.frames_workload(1000, 20, 100, 1e-3, 9)
    t0 = time.perf_counter()
    f = nb.FrameSampler(c, 0)
    new_s = time.perf_counter() - t0
    words = f.words(shots)
    d_out = torch.empty(f.m * words, dtype=torch.int64, device="cuda")
    rng = nb.StdRng(9 + RANK)

    def seeds():
        return [rng.next_u64() for _ in range((shots + f.BATCH - 1) // f.BATCH)]

    for _ in range(args.warmup):
        f.sample_packed_device(shots, seeds(), d_out.data_ptr(), d_out.numel())
    barrier(dist)
    kern, wall = [], []
    for _ in range(args.steps):
        sd = seeds()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        f.sample_packed_device(shots, sd, d_out.data_ptr(), d_out.numel())
        torch.cuda.synchronize()
        wall.append(time.perf_counter() - t1)
        kern.append(f.last_kernel_ms())
    ms = max_over_ranks(dist, 1e3 * statistics.mean(wall))
    kms = max_over_ranks(dist, statistics.mean(kern))
    masks = 1000 + 2000  # initial randomisations, then one per measurement
    alg = (masks + f.m) * words * 8  # masks written and read once, records written once
    out = {
        "metric": "shots/s",
        "value": WORLD * shots / (ms / 1e3),
        "unit": "shots/s",
        "ms_per_step": ms,
        "kernel_ms_per_step": kms,
        "published_ms": FRAMES_PUBLISHED_MS,
        "vs_published": round(FRAMES_PUBLISHED_MS / ms, 2),
        "config": {"workload": "frame-sampler benchmark: n=1000, 20 rounds x (500 CX + DEPOLARIZE2(0.001), 100 M), "
                               "10500 gates, 2000 measurements, 100000 shots (7 batches of 16384)",
                   "layers": f.num_layers, "reference_record_s": round(new_s, 3)},
        "roofline": {"bound": "hbm", "kernel": "k_frame_masks + k_frame_run",
                     "achieved": round(alg / (kms / 1e3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(alg / (kms / 1e3) / 1e9 / peak, 4), "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": alg,
                     "note": "frames live in shared memory; HBM carries only the masks and records, so the "
                             "kernels are bound by their dependency layers, not by HBM"},
        "gpu_launches_per_step": 2,
    }
    if not args.no_e2e:
        host = np.zeros((f.m, words), dtype=np.uint64)
        f.sample_packed_seeds(shots, seeds(), out=host)
        barrier(dist)
        t1 = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 3))
        for _ in range(e2e_steps):
            f.sample_packed_seeds(shots, seeds(), out=host)
        dt = max_over_ranks(dist, time.perf_counter() - t1)
        out["e2e"] = {"value": WORLD * e2e_steps * shots / dt, "unit": "shots/s", "h2d_bytes_per_step": None,
                      "d2h_bytes_per_step": host.nbytes,
                      "note": "per step: the same call with the packed records copied to host memory; "
                              "host wall clock"}
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_frames(c.to_text(), f.reference(), shots)
        out["vs_cpu"] = round(out["cpu_baseline"]["value"] and out["value"] / out["cpu_baseline"]["value"], 1)
    return out


def cpu_frames(text: str, reference, shots: int, reps: int = 2):
    """The oracle's restatement of frame.rs on the host cores, the same workload."""
    from oracle import oracle as O

    threads = max(1, min(os.cpu_count() or 1, 64))
    r = O.StdRng(9)
    times = []
    for _ in range(reps):
        seeds = [r.next_u64() for _ in range((shots + (1 << 14) - 1) >> 14)]
        t0 = time.perf_counter()
        O.frame_sample_packed(text, reference, shots, seeds, threads=threads)
        times.append(time.perf_counter() - t0)
    t = min(times)
    return {"value": shots / t, "unit": "shots/s", "cores": min(threads, (shots + (1 << 14) - 1) >> 14),
            "kind": "port", "sample": f"{shots} shots of the frame benchmark, {reps} runs, best"}


def config_rates(nb, peak, peak_kind):
    """The other sized workloads of the path, plain complex128 kernels, one GPU:
    C0 (n = 20, depth 40, with its readouts), C1 (n = 30, depth 20, M on the
    last 4 qubits) and C3 (n = 31: H on qubits 0..15, 2000 permutation and
    diagonal gates).  Gates/s from CUDA events on the state's stream; %HBM from
    the launch profiler's algorithmic bytes over a separate profiled run."""
    out = {}

    def measure(name, n, circuit, runs, extra=None, init_plus=False):
        s = nb.GpuStateVector.plus_state(n) if init_plus else nb.GpuStateVector(n)
        rng = nb.StdRng(11)
        if runs:
            s.run(circuit, rng)  # warm-up (and the gate graphs' capture)
            s.timer_start()
            for _ in range(runs):
                s.run(circuit, rng)
            ms = s.timer_stop() / runs
        s.profile(True)
        if not runs:  # one profiled run only (long circuits: plain kernels of milliseconds each)
            s.timer_start()
        s.run(circuit, rng)
        if not runs:
            ms = s.timer_stop()
        prof = s.profile_read()
        s.profile(False)
        pbytes = sum(v["bytes"] for v in prof.values())
        pms = sum(v["ms"] for v in prof.values())
        gates = circuit.num_gates
        r = {"n": n, "gates": gates, "ms_per_run": ms, "gates_per_s": gates / (ms / 1e3),
             "hbm_frac_of_kernel_time": round(pbytes / (pms / 1e3) / 1e9 / peak, 4) if pms else None,
             "peak_kind": peak_kind,
             "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 2),
                             "GBps": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6, 1)} for k, v in prof.items()}}
        if extra:
            r.update(extra(s))
        out[name] = r
        del s

    def c0_readouts(s):
        n = 20
        t0 = time.perf_counter()
        z = s.expectation(nb.Pauli.from_string(n, "Z0*Z1"))
        x = s.expectation(nb.Pauli.from_string(n, "X0*X5*Y9"))
        smp = s.sample(nb.StdRng(2), 4096)
        ridx = nb.StdRng(3)
        amps = s.amplitudes_at([ridx.gen_range(0, 1 << n) for _ in range(64)])
        return {"readouts_ms": (time.perf_counter() - t0) * 1e3, "readouts": "<Z0 Z1>, <X0 X5 Y9>, 4096 shots, "
                "64 amplitudes", "z0z1": z.real, "x0x5y9": x.real, "shots": int(smp.size), "amplitudes": len(amps)}

    measure("C0", 20, nb.Circuit.random_layers(20, 40, 1), 10, c0_readouts)
    measure("C1", 30, nb.Circuit.random_layers(30, 20, 1, 0.0, 26, 30), 2)
    c3 = nb.Circuit.reversible(31, 2000, 1)
    measure("C3", 31, c3, 0)
    # From |0...0> the register holds 2^16 nonzero amplitudes of 2^31, and the diagonal
    # kernels write only nonzero ones, so bytes per second of that run are not a
    # roofline.  The kernels' roofline is taken on a dense register instead: the
    # circuit's 2000 permutation and diagonal gates (without its Hadamard layer) from
    # |+>^31, where every amplitude stays nonzero.
    c3r = out["C3"]
    c3r["hbm_frac_of_kernel_time"] = None
    c3r["note"] = ("sparse register (2^16 of 2^31 amplitudes nonzero): per-kernel GB/s omitted; see "
                   "C3_dense_register for the kernels' roofline")
    c3r["kernels"] = {k: {"launches": v["launches"], "ms": v["ms"]} for k, v in c3r["kernels"].items()}
    c3d = nb.Circuit.parse("\n".join(l for l in c3.to_text().splitlines() if not l.startswith("H ")) + "\n")
    measure("C3_dense_register", 31, c3d, 0, init_plus=True)

    # the reference's published StateVector workload (examples/bench.rs:120-143; README.md:210-211:
    # 0.10 s for the 88-gate layer and 1.4 ms per expectation at n = 22 on a 16-thread desktop)
    n = 22
    hdr, h, layer = published_workload_text(n)
    s = nb.GpuStateVector(n)
    s.run(nb.Circuit.parse(hdr + h), nb.StdRng(0))
    lc = nb.Circuit.parse(hdr + layer)
    rng = nb.StdRng(0)
    s.timer_start()
    s.run(lc, rng)  # a circuit's first run launches kernel by kernel
    one_shot = s.timer_stop()
    s.run(lc, rng)  # the second captures its gate graph
    reps = 20
    s.timer_start()
    for _ in range(reps):
        s.run(lc, rng)
    replay = s.timer_stop() / reps
    pz = nb.Pauli.from_string(n, "X0*Y3*Z5")
    s.expectation(pz)
    t0 = time.perf_counter()
    for _ in range(20):
        s.expectation(pz)
    exp_s = (time.perf_counter() - t0) / 20
    del s
    pub = {"workload": "n=22 complex128: H on every qubit, then for q in 0..22: T q, CX q q+1, CCZ q q+1 q+2, "
                       "RX(0.3) q (88 gates); 20 expectations of X0*Y3*Z5",
           "layer_ms_first_run": one_shot, "layer_ms_replayed": replay, "layer_gates_per_s": 4 * n / (one_shot / 1e3),
           "expectation_ms": exp_s * 1e3,
           "published": {"layer_s": 0.10, "expectation_s": 1.4e-3, "hardware": "16-thread desktop (README.md:202)"},
           "vs_published_layer": 0.10 / (one_shot / 1e3), "vs_published_expectation": 1.4e-3 / exp_s}
    if RANK == 0 and WORLD == 1:
        cpu = published_workload_cpu(n)
        pub["cpu_oracle"] = cpu
        pub["vs_cpu_oracle_layer"] = cpu["layer_s"] / (one_shot / 1e3)
    out["published_n22"] = pub

    # the same C3 circuit on the sparse form (SparseVector: 2^16 entries instead of 2^31 amplitudes)
    sp = nb.GpuSparseVector(31)
    sp.run(c3, nb.StdRng(11))  # warm-up (stream-ordered pools, CUB temporaries)
    runs, t0 = 3, time.perf_counter()
    ms_dev = 0.0
    for _ in range(runs):
        sp = nb.GpuSparseVector(31)
        sp.timer_start()
        sp.run(c3, nb.StdRng(11))
        ms_dev += sp.timer_stop()
    wall = (time.perf_counter() - t0) * 1e3 / runs
    out["C3_sparse"] = {"n": 31, "gates": c3.num_gates, "entries": sp.num_entries(),
                        "ms_per_run": ms_dev / runs, "wall_ms_per_run": wall,
                        "gates_per_s": c3.num_gates / (ms_dev / runs / 1e3),
                        "speedup_vs_dense": out["C3"]["ms_per_run"] / (ms_dev / runs),
                        "note": "GpuSparseVector from |0>: device time of the run on its stream (the host waits "
                                "for entry counts after every normalisation); wall includes state creation"}
    del sp
    out["sparse_published_n1000"] = sparse_published_workload(nb)
    return out


def ripple_texts(n: int = 1000, inputs: int = 10):
    """The reference's published SparseVector workload (examples/bench.rs:245-262):
    H on `inputs` qubits of an n-qubit register, then for q in 0..n-2 CCX (q, q+1, q+2)
    and CX (q, q+2); the reference times the 2(n-2) ripple gates."""
    head = "\n".join([f"QUBITS {n}"] + [f"H {q}" for q in range(inputs)]) + "\n"
    body = "".join(f"CCX {q} {q + 1} {q + 2}\nCX {q} {q + 2}\n" for q in range(n - 2))
    return head, f"QUBITS {n}\n" + body


def sparse_published_workload(nb, reps: int = 5):
    """n = 1000 sparse register, 1024 superposed inputs, the 1996-gate CCX/CX ripple
    (README.md:214: 7 ms on a 16-thread desktop): device time of the ripple through
    GpuSparseVector.run (one launch per run of one-to-one gates), wall time of the same
    call, and the oracle's CPU restatement of the whole circuit on one host thread."""
    head, ripple = ripple_texts()
    ch, cr = nb.Circuit.parse(head), nb.Circuit.parse(ripple)
    pz = nb.Pauli.from_string(1000, "Z0*Z999")
    dev, wall, exp_ms = [], [], []
    for _ in range(reps + 1):
        sp = nb.GpuSparseVector(1000)
        sp.run(ch, nb.StdRng(1))
        sp.synchronize()
        t0 = time.perf_counter()
        sp.timer_start()
        sp.run(cr, nb.StdRng(1))
        dev.append(sp.timer_stop())
        wall.append((time.perf_counter() - t0) * 1e3)
        t1 = time.perf_counter()
        z = sp.expectation(pz)
        exp_ms.append((time.perf_counter() - t1) * 1e3)
    dev, wall, exp_ms = dev[1:], wall[1:], exp_ms[1:]  # the first run warms the pools
    out = {"workload": "n=1000 SparseVector: H on qubits 0..9, then CCX(q,q+1,q+2), CX(q,q+2) for q in 0..998 "
                       "(1996 timed gates, 1024 entries of 16 words)",
           "gates": cr.num_gates, "entries": sp.num_entries(),
           "ms_device": statistics.median(dev), "ms_wall": statistics.median(wall),
           "expectation_z0z999_ms_wall": statistics.median(exp_ms), "z0z999": z.real,
           "published": {"ripple_s": 0.007, "hardware": "16-thread desktop (README.md:202, :214)"},
           "vs_published_wall": 7.0 / statistics.median(wall)}
    try:
        from oracle import oracle as O

        O.build()
        t0 = time.perf_counter()
        O.WideSparse(head + ripple.split("\n", 1)[1], 1)
        out["cpu_oracle"] = {"s": time.perf_counter() - t0, "cores": 1, "kind": "port",
                             "sample": "the whole circuit (H's, ripple) on the oracle's restatement, parse included"}
    except Exception as e:  # the oracle is the baseline's checker only; its absence does not stop the bench
        out["cpu_oracle"] = {"unavailable": str(e)[:200]}
    return out


def timed_runs(nb, state, circuit, steps: int, warmup: int, fused: bool, dist):
    """Each step runs the circuit on the register the previous steps left.

    After the first warm-up step the register is dense (every amplitude
    nonzero), the regime of the CPU baseline (which starts from |+>^n) and of
    the algorithmic byte counts; starting every step from |0...0> would leave
    the first layers' registers sparse, where the diagonal kernels skip the
    writes of zero amplitudes.
    """
    rng = nb.StdRng(12345)

    def step():
        state.run_fused(circuit, rng) if fused else state.run(circuit, rng)

    for _ in range(warmup):
        step()
    state.synchronize()
    barrier(dist)
    state.timer_start()
    for _ in range(steps):
        step()
    ms = state.timer_stop()
    # one more step with the launch profiler on, for the per-kernel times and algorithmic
    # bytes of the roofline (its event records are kept out of the timed steps)
    state.profile(True)
    step()
    state.synchronize()
    prof = state.profile_read()
    state.profile(False)
    return ms, prof


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--qubits", type=int, default=32, dest="n")  # --qubits passes through torchrun
    ap.add_argument("--depth", type=int, default=20)
    ap.add_argument("--path", default="auto", choices=["auto", "plain", "fused"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--traj-count", type=int, default=4096)
    ap.add_argument("--traj-check", type=int, default=4096,
                    help="trajectories checked against complex128 plain-path runs (0: none)")
    ap.add_argument("--no-trajectories", action="store_true")
    ap.add_argument("--no-capacity", action="store_true", help="skip the n = 34 complex64 capacity run")
    ap.add_argument("--traj-launch", default="",
                    help="CTAS_PER_SM,BUFFERS: a fixed launch configuration of the batch kernel (default: tuned)")
    ap.add_argument("--no-configs", action="store_true", help="skip the C0, C1 and C3 plain-path rates")
    ap.add_argument("--no-frames", action="store_true", help="skip the frame-sampler benchmark")
    ap.add_argument("--frames-only", action="store_true", help="only the frame-sampler benchmark")
    ap.add_argument("--no-headline", action="store_true",
                    help="only the trajectories/s part (for profiling the batch kernel)")
    args = ap.parse_args()

    if args.impl == "reference":
        return run_reference(args)

    import ncsim_b200 as nb

    nb.lib()
    dist = dist_init()
    seed = 1 + RANK
    peak, peak_kind = measured_peaks()

    if args.frames_only:
        with ClockSampler() as fclk:
            fr = frames_bench(nb, args, dist, peak, peak_kind)
        fr["clocks"] = fclk.summary()
        if RANK == 0:
            print(json.dumps({"metric": METRIC, "n_gpus": WORLD, "frames": fr}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    if args.no_headline:
        with ClockSampler() as tclk:
            tr = trajectory_bench(nb, args, dist, peak, peak_kind)
        tr["clocks"] = tclk.summary()
        if RANK == 0:
            print(json.dumps({"metric": METRIC, "n_gpus": WORLD, "trajectories": tr}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    fused_ok = args.path in ("auto", "fused")
    if fused_ok:
        try:
            probe = nb.GpuStateVector(12, nb.C64)
            probe.run_fused(nb.Circuit.random_layers(12, 1, 1), nb.StdRng(0))
            del probe
        except nb.SimError:
            if args.path == "fused":
                raise
            fused_ok = False

    result = {}
    n = args.n
    if fused_ok:
        n = pick_n(nb, args.n, 8, 1)
        circuit = nb.Circuit.random_layers(n, args.depth, seed)
        st = nb.GpuStateVector(n, nb.C64)
        with ClockSampler() as clk:
            ms, prof = timed_runs(nb, st, circuit, args.steps, args.warmup, True, dist)
        headline = ("fused", st, ms, prof, clk)
    else:
        n = pick_n(nb, args.n, 16, 1)
        circuit = nb.Circuit.random_layers(n, args.depth, seed)
        st = nb.GpuStateVector(n, nb.C128)
        with ClockSampler() as clk:
            ms, prof = timed_runs(nb, st, circuit, args.steps, args.warmup, False, dist)
        headline = ("plain", st, ms, prof, clk)

    path, _, ms, prof, clk = headline
    del st, headline  # free the headline state before the comparison arms allocate
    gates = circuit.num_gates
    ms_max = max_over_ranks(dist, ms)
    value = WORLD * args.steps * gates / (ms_max / 1e3)
    launches = sum(v["launches"] for v in prof.values())
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"])
    dom_name, dom_v = dom
    achieved = dom_v["bytes"] / (dom_v["ms"] / 1e3) / 1e9
    total_bytes = sum(v["bytes"] for v in prof.values())
    overall = total_bytes / (ms / args.steps / 1e3) / 1e9  # the profiled step's bytes over one step's time
    traffic = profiled_traffic(dom_name)
    roofline = {
        "bound": "hbm",
        "kernel": dom_name,
        "achieved": round(achieved, 1),
        "peak": peak,
        "unit": "GB/s",
        "frac": round(achieved / peak, 4),
        "peak_kind": peak_kind,
        "traffic": traffic,
        "algorithmic_bytes_per_launch": dom_v["bytes"] / max(1, dom_v["launches"]),
        "launches": dom_v["launches"],
        "step_frac": round(overall / peak, 4),
    }
    result["kernels"] = {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                             "GBps": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6, 1)} for k, v in prof.items()}

    # The FP64 arm: the same circuit on the plain complex128 path.  Its first run from
    # |0...0> is also the reference of the fused result's fidelity; its second run, on
    # the dense register the first left, is timed (the regime of the fused steps).
    head = {}
    if path == "fused":
        ref = nb.GpuStateVector(n, nb.C128)
        ref.run(circuit, nb.StdRng(7))
        fz = nb.GpuStateVector(n, nb.C64)
        fz.run_fused(circuit, nb.StdRng(7))
        cmpd = ref.compare(fz)
        del fz
        ref.synchronize()
        ref.timer_start()
        ref.run(circuit, nb.StdRng(7))
        ms_p = ref.timer_stop()
        # the same run one kernel per gate (runs of gates not tiled into passes)
        ref.set_tile_passes(False)
        ref.timer_start()
        ref.run(circuit, nb.StdRng(7))
        ms_g = ref.timer_stop()
        del ref
        fp64 = gates / (ms_p / 1e3)
        fp64_g = gates / (ms_g / 1e3)
        head = {"fp64_gates_per_s": round(fp64, 2),
                "speedup_vs_fp64": round(value / WORLD / fp64, 3),
                "fp64_gate_by_gate_gates_per_s": round(fp64_g, 2),
                "speedup_vs_fp64_gate_by_gate": round(value / WORLD / fp64_g, 3),
                "infidelity": cmpd["infidelity"],
                "max_abs_err": cmpd["max_abs_diff"]}
        result["plain_fp64"] = {"gates_per_s": fp64, "ms_per_circuit": ms_p,
                                "gate_by_gate": {"gates_per_s": fp64_g, "ms_per_circuit": ms_g},
                                "note": "plain complex128 path, same circuit, dense register: runs of gates "
                                        "as tiled passes (the default), and one kernel per gate"}
        result["fidelity"] = {"infidelity": cmpd["infidelity"], "max_abs_diff": cmpd["max_abs_diff"],
                              "norm_fused": cmpd["norm_b"],
                              "reference": "plain complex128 run of the identical circuit from |0...0>"}

    # end to end through the C ABI: host circuit text in, readouts out
    e2e = None
    if not args.no_e2e:
        text = circuit.to_text()
        prec = nb.C64 if path == "fused" else nb.C128
        e2e_state = nb.GpuStateVector(n, prec)
        pz = nb.Pauli.from_string(n, "Z0*Z1")
        idx = list(range(0, 1 << n, (1 << n) // 64))[:64]

        def one_step():
            c = nb.Circuit.parse(text)  # host bytes in
            if path == "fused":
                e2e_state.run_fused(c, nb.StdRng(3))
            else:
                e2e_state.run(c, nb.StdRng(3))
            e = e2e_state.expectation(pz)  # results out
            a = e2e_state.amplitudes_at(idx)
            return e, a

        one_step()
        barrier(dist)
        t0 = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 2))
        for _ in range(e2e_steps):
            one_step()
        dt = max_over_ranks(dist, time.perf_counter() - t0)
        e2e = {"value": WORLD * e2e_steps * gates / dt, "unit": "gates/s",
               "h2d_bytes_per_step": len(text.encode()), "d2h_bytes_per_step": 16 + 16 * len(idx),
               "note": "per step: parse the circuit text, run it on the (dense) register, <Z0 Z1>, "
                       "64 amplitudes; host wall clock"}
        del e2e_state

    # capacity: the fused form at n = 34 (complex64, 128 GiB), beyond the reference's
    # n <= 30; its circuit and then the inverse circuit must bring |0...0> back
    if path == "fused" and not args.no_capacity:
        result["capacity"] = capacity_run(nb, args.depth)
        if "gates_per_s" in result["capacity"]:
            head["capacity_n34_gates_per_s"] = round(result["capacity"]["gates_per_s"], 2)

    cpu = None
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(n, args.depth, seed, args.cpu_budget)
        if "fp64_gates_per_s" in head:
            head["fp64_vs_cpu"] = round(head["fp64_gates_per_s"] / cpu["value"], 1)

    if not args.no_trajectories:
        with ClockSampler() as tclk:
            result["trajectories"] = trajectory_bench(nb, args, dist, peak, peak_kind)
        result["trajectories"]["clocks"] = tclk.summary()
        acc = result["trajectories"].get("accuracy")
        if acc:
            head["traj_mean_z0_error"] = acc["mean_z0_error"]
    if not args.no_configs and WORLD == 1:
        result["configs"] = config_rates(nb, peak, peak_kind)
    if not args.no_frames:
        with ClockSampler() as fclk:
            result["frames"] = frames_bench(nb, args, dist, peak, peak_kind)
        result["frames"]["clocks"] = fclk.summary()
        head["frames_shots_per_s"] = round(result["frames"]["value"], 1)

    clocks = clk.summary() if clk else None
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "gates/s",
        "n_gpus": WORLD,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
    }
    line.update(head)  # the short comparison keys early in the line
    line.update({
        "dtype": "f32" if path == "fused" else "f64",
        "data": "synthetic",
        "config": {
            "workload": f"random layers n={n} depth {args.depth} ({gates} gates), seed 1+rank, "
                        f"{'fused precision form, complex64' if path == 'fused' else 'plain one-kernel-per-gate path, complex128'}",
            "n": n,
            "depth": args.depth,
            "gates_per_step": gates,
            "path": path,
            "l2": "state larger than L2 (no flush needed)",
            "parallelism": f"replicas x{WORLD}",
        },
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        "gpu_launches": launches * args.steps,  # the profiled step launches what each timed step does
        "gpu_launches_per_step": launches,
    })
    line.update(result)
    if RANK == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def inverse_text(text: str) -> str:
    """The inverse of a random layer circuit: gates in reverse order, each replaced by its inverse."""
    inv = {"H": "H", "S": "S_DAG", "T": "T_DAG", "SQRT_X": "SQRT_X_DAG", "CZ": "CZ"}
    lines = text.strip().split("\n")
    out = [lines[0]]
    for ln in reversed(lines[1:]):
        name, rest = ln.split(" ", 1)
        out.append(f"RZ({-float(name[3:-1])!r}) {rest}" if name.startswith("RZ(") else f"{inv[name]} {rest}")
    return "\n".join(out) + "\n"


def capacity_run(nb, depth: int, n: int = 34):
    """The fused form at n = 34 (complex64, 128 GiB): the random layer circuit
    (device time on the state's stream), the norm after it, then the inverse
    circuit, after which the register should be |0...0> again."""
    free = nb.device_info()["free_bytes"]
    if free < (8 << n) + (4 << 30):
        return {"n": n, "skipped": f"needs {(8 << n) / 2**30:.0f} GiB, {free / 2**30:.0f} GiB free"}
    c = nb.Circuit.random_layers(n, depth, 1)
    ci = nb.Circuit.parse(inverse_text(c.to_text()))
    s = nb.GpuStateVector(n, nb.C64)
    s.run_fused(c, nb.StdRng(0))  # plans the circuit (host) and warms up
    s.set_basis(0)
    s.timer_start()
    _, st = s.run_fused(c, nb.StdRng(0))
    ms = s.timer_stop()
    nn = s.norm_sq().real
    s.run_fused(ci, nb.StdRng(0))
    back = 1.0 - abs(s.amplitude(0)) ** 2 / s.norm_sq().real  # normalised, as 1 - F
    del s
    return {"n": n, "precision": "complex64 (128 GiB)", "gates": c.num_gates, "passes": st.passes,
            "ms_per_circuit": ms, "gates_per_s": c.num_gates / (ms / 1e3), "norm_drift": abs(nn - 1.0),
            "round_trip_infidelity": back,
            "note": "from |0...0>: the circuit (timed), <psi|psi>, then its inverse; 1 - |<0|psi>|^2/<psi|psi> "
                    "after both"}


if __name__ == "__main__":
    sys.exit(main())
