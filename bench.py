#!/usr/bin/env python
"""Benchmark of the local-update hot path on B200.

Default workload (the configuration the headline metric is quoted on): 3D O(3)
Heisenberg model, 64^3 periodic cubic lattice, J = 1, beta = 0.693, FP32 unit
vectors drawn uniformly on the sphere from a seed; Metropolis with
UniformSphereN<3> alternating with Wolff cluster flips (uniform random axis).
One step = one Wolff flip + one Metropolis sweep with the observables (E, M)
reduced in FP64 on the device.  Units: site-updates = the sweep's sites plus the
flip's cluster sites.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl umc|reference]

Prints one JSON line (rank 0).  Multi-GPU (torchrun): every rank runs its own
replica chain (a single lattice does not shard), value = all ranks' units / the
slowest rank's device time ("weak" scaling).

The lattice (3 MiB) would otherwise stay in L2 between steps, so a 256 MiB
buffer is written between timed steps and only the steps are timed (CUDA
events on the chain's stream).
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
sys.path.insert(0, ROOT)

METRIC = "effective samples/s per B200 (learned+batched vs plain GPU); site-updates/s"
L_DEFAULT = 64
BETA = 0.693
PROFILES = os.path.join(ROOT, "profiles")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=4000)
    p.add_argument("--warmup", type=int, default=50)
    p.add_argument("--impl", choices=["umc", "reference"], default="umc")
    p.add_argument("--L", type=int, default=L_DEFAULT)
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    return p.parse_args()


def workload(L):
    return (f"O(3) Heisenberg {L}^3 periodic cubic, J=1, beta={BETA}, FP32 unit vectors uniform on S^2 "
            f"(keyed seed); step = 1 Wolff flip (UniformSphereN<3> axis) + 1 Metropolis sweep "
            f"(UniformSphereN<3>), E and M reduced in FP64 every step")


def rank_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# -------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: str):
        self.gpu = gpu  # nvidia-smi -i accepts the UUID, independent of CUDA_VISIBLE_DEVICES
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(kind: str, units: float):
    """DRAM bytes per launch of a kernel from the committed ncu summary
    (profiles/traffic.txt: '<kind> <bytes per unit>' lines), scaled to this
    launch's units, or None when no capture was summarised."""
    path = os.path.join(PROFILES, "traffic.txt")
    try:
        for line in open(path):
            f = line.split()
            if len(f) >= 2 and f[0] == kind:
                return float(f[1]) * units
    except OSError:
        pass
    return None


# ---------------------------------------------------------------- reference
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_o3(L, warmup, steps, threads):
    from oracle.oracle import Reference, have_reference

    if not have_reference():
        return None
    r = Reference()
    su, sec = r.bench_o3(L, BETA, warmup, steps, threads, 1)
    return su, sec


def run_reference(args):
    ws, rank, _ = rank_info()
    if rank != 0:
        return
    threads = cpu_threads()
    # a step of the stock CPU path is ~35 ms per thread at 64^3: bound the sample
    steps = max(1, min(args.steps, 200))
    warm = max(0, min(args.warmup, 3))
    res = reference_o3(args.L, warm, steps, threads)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libumc_ref.so was not built"}))
        return
    su, sec = res
    value = su / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "site-updates/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * sec / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload(args.L), "L": args.L, "beta": BETA, "chains": threads,
                   "note": "the reference's stock driver (driver.hpp) on the host cores, one independent chain per thread"},
        "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": threads, "kind": "reference",
                         "sample": f"{steps} steps x {threads} chains of {args.L}^3 after {warm} warm-up steps"},
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------- umc
def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    ws, rank, local = rank_info()
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    import universal_classical_montecarlo_b200 as umc

    L = args.L
    n = L**3
    g = umc.cubic_lattice(L, L, L)
    ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE,
                   wolff_axis=umc.AXIS_SPHERE, seed=1 + rank, device=local, max_records=8192)
    ch.randomize(1000 + rank)
    stream = torch.cuda.ExternalStream(ch.stream(), device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        if ws > 1:
            dist.barrier()

    # ---- warm-up
    ch.enqueue_hybrid(BETA, args.warmup)
    ch.fetch(8192)
    ch.kernel_stats(reset=True)

    # ---- timed region: K steps, L2 flushed between steps, steps timed on the chain's stream
    K = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    sampler = ClockSampler("GPU-" + str(torch.cuda.get_device_properties(local).uuid))
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)  # let the sampler attach before the work starts
    units = 0.0
    done = 0
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.fill_(k & 0xFF)
            starts[k].record(stream)
            ch.enqueue_hybrid(BETA, 1)
            ends[k].record(stream)
            done += 1
            if done == 4096:  # drain the record ring
                rec, sizes = ch.fetch(8192)
                units += len(rec) * n + float(sizes.sum())
                done = 0
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    rec, sizes = ch.fetch(8192)
    units += len(rec) * n + float(sizes.sum())
    launches = ch.kernel_stats(reset=True)
    gpu_launches = sum(v[0] for k, v in launches.items())
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))

    # ---- dominant kernel, timed live with events around each launch
    ch.set_timing(True)
    KP = min(K, 2000)
    with torch.cuda.stream(stream):
        for k in range(KP):
            flush.fill_(k & 0xFF)
            ch.enqueue_hybrid(BETA, 1)
            if (k + 1) % 4096 == 0:
                ch.fetch(8192)
    ch.fetch(8192)
    per_kind = ch.kernel_stats(reset=True)
    ch.set_timing(False)
    kind, (nl, ms) = max(((k, v) for k, v in per_kind.items() if v[0] > 0), key=lambda kv: kv[1][1])
    avg_s = ms / nl / 1e3
    # algorithmic bytes per launch: colour pass 36 B per site-update
    # (read own + neighbour class, write own; 12 B per FP32 3-vector), union-find
    # 68 B per site (field + CSR + label), flip 20 B per site (+ 12 B per flipped site)
    per_unit = {"metropolis": (36.0, n / 2), "wolff_union": (68.0, n), "wolff_flip": (20.0, n)}
    bpu, units_per_launch = per_unit.get(kind, (36.0, n / 2))
    achieved = bpu * units_per_launch / avg_s / 1e9
    peak, peak_src = measured_peak_hbm()
    traffic = profiled_traffic(kind, units_per_launch)

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        host.numpy()[:] = ch.get_field()
        KE = min(K, 300)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_units = 0.0
        for _ in range(KE):
            ch.set_field(host.numpy())  # H2D from pinned memory + layout kernel
            sz, r = ch.hybrid(BETA, 1)  # step + D2H of the record
            e_units += n + float(sz[0])
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        e2e = {"value": e_units / e2e_s, "unit": "site-updates/s", "h2d_bytes_per_step": n * 3 * 4,
               "d2h_bytes_per_step": 8 * 8 + 8, "steps": KE}

    # ---- aggregate over ranks
    max_ms, tot_units = total_ms, units
    if ws > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        u = torch.tensor([units], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
        max_ms, tot_units = float(t.item()), float(u.item())
        if e2e is not None:
            ev = torch.tensor([e2e["value"]], dtype=torch.float64, device="cuda")
            dist.all_reduce(ev, op=dist.ReduceOp.SUM)
            e2e["value"] = float(ev.item())

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = cpu_threads()
        est = reference_o3(L, 0, 1, 1)
        if est is not None:
            per_step = est[1]
            steps = max(2, int(args.cpu_seconds / max(per_step, 1e-4)))
            su, sec = reference_o3(L, 1, steps, threads)
            cpu = {"value": su / sec, "unit": "site-updates/s", "cores": threads, "kind": "reference",
                   "sample": f"{steps} steps x {threads} independent {L}^3 chains (reference stock driver, "
                             f"plain Pcg32), {sec:.1f} s"}

    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    value = tot_units / (max_ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": "site-updates/s", "n_gpus": ws, "steps": K,
        "warmup": args.warmup, "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload(L), "L": L, "beta": BETA, "parallelism": f"replicas x{ws}" if ws > 1 else "1 chain",
                   "l2": "flushed between timed steps (256 MiB write, outside the timed events)",
                   "units": "Metropolis site-updates + Wolff flipped sites",
                   "mean_cluster": float(sizes.mean()) if len(sizes) else None},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": kind, "avg_launch_us": avg_s * 1e6,
                     "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback 6.65 TB/s"},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "kernel_launches": {k: v[0] for k, v in launches.items() if v[0]},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
