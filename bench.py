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
# untimed hybrid steps from the random start before either arm is timed: at
# 64^3 and beta 0.693 the energy per site settles within about 500 steps
THERM_STEPS = 1000
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
    p.add_argument("--workload", choices=["o3", "ising", "su3", "xybatch", "u1batch", "u1learned", "userxy",
                                          "usero3", "usero3csr", "userwolff", "useru1", "useru1tables"],
                   default="o3",
                   help="o3: the headline configuration; ising / su3 / xybatch / userxy / usero3 / usero3csr: "
                        "secondary roofline runs (user*: user-written models through include/umc/device.cuh); "
                        "u1learned: the learned-proposal study (effective samples/s)")
    p.add_argument("--no-learned", action="store_true", help="skip the learned-proposal summary of the o3 line")
    return p.parse_args()


def workload(L):
    return (f"O(3) Heisenberg {L}^3 periodic cubic, J=1, beta={BETA}, FP32 unit vectors uniform on S^2 "
            f"(keyed seed); step = 1 Wolff flip (UniformSphereN<3> axis) + 1 Metropolis sweep "
            f"(UniformSphereN<3>), E and M reduced in FP64 every step")


def aggregate_ranks(dist, torch, device, total_ms, units, e2e_value=None):
    """Whole-job figures of a replicas run: the slowest rank's device time
    (max), the units all ranks processed (sum) and, when given, the sum of the
    ranks' end-to-end throughputs.  Every rank makes the same collective calls
    in the same order (e2e_value is None on all ranks or on none)."""
    t = torch.tensor([total_ms], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    e2e_sum = None
    if e2e_value is not None:
        ev = torch.tensor([e2e_value], dtype=torch.float64, device=device)
        dist.all_reduce(ev, op=dist.ReduceOp.SUM)
        e2e_sum = float(ev.item())
    return float(t.item()), float(u.item()), e2e_sum


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


def measured_peak_bf16():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def profiled_traffic(kind: str, units: float):
    """DRAM bytes per launch of a kernel from the committed ncu summary
    (profiles/traffic.txt: '<workload>:<kind> <bytes per launch>' lines), or
    None when no capture was summarised."""
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


def timing_reference():
    """(Reference, build) of the timed CPU baselines (oracle.timing_reference:
    the -O3 x86-64-v3 build of the reference harness where the host runs it),
    or (None, None)."""
    from oracle.oracle import timing_reference as tr

    got = tr()
    return got if got is not None else (None, None)


def reference_o3(L, warmup, steps, threads):
    r, build = timing_reference()
    if r is None:
        return None
    su, sec = r.bench_o3(L, BETA, warmup, steps, threads, 1)
    return su, sec, build


def run_reference(args):
    ws, rank, _ = rank_info()
    if rank != 0:
        return
    threads = cpu_threads()
    # a step of the stock CPU path is ~15-35 ms per thread at 64^3: bound the
    # sample; every chain first thermalises as the GPU arm's chain does
    steps = max(1, min(args.steps, 200))
    warm = max(0, min(args.warmup, 3))
    res = reference_o3(args.L, THERM_STEPS + warm, steps, threads)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libumc_ref.so was not built"}))
        return
    su, sec, build = res
    value = su / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "site-updates/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * sec / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload(args.L), "L": args.L, "beta": BETA, "chains": threads,
                   "note": "the reference's stock driver (driver.hpp) on the host cores, one independent chain per "
                           f"thread, built {build}",
                   "thermalisation": f"{THERM_STEPS} untimed steps per chain from its random start, then the "
                                     f"{warm} warm-up steps"},
        "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": threads, "kind": "reference",
                         "build": build,
                         "sample": f"{steps} steps x {threads} chains of {args.L}^3 after {THERM_STEPS + warm} "
                                   f"untimed steps"},
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ workloads
class O3Hybrid:
    """Headline workload: O(3) L^3, one Wolff flip + one Metropolis sweep per step."""

    name = "o3"
    unit = "site-updates/s"
    dtype = "f32"

    def __init__(self, umc, args, rank, local):
        self.L = args.L
        self.n = self.L**3
        g = umc.cubic_lattice(self.L, self.L, self.L)
        self.ch = umc.Chain(umc.MODEL_VECTOR, graph=g, components=3, coupling=1.0, proposal=umc.PROPOSAL_SPHERE,
                            wolff_axis=umc.AXIS_SPHERE, seed=1 + rank, device=local, max_records=8192)
        self.ch.randomize(1000 + rank)
        self.flush = True

    def thermalise(self):
        """THERM_STEPS untimed steps from the random start, so the timed steps
        see the configuration's equilibrium clusters; returns their mean size
        over the last 200 steps."""
        self.ch.enqueue_hybrid(BETA, THERM_STEPS)
        _, sizes = self.ch.fetch(8192)
        return float(sizes[-200:].mean())

    def describe(self):
        return workload(self.L)

    def enqueue(self, k):
        self.ch.enqueue_hybrid(BETA, k)

    def units(self, rec, sizes):
        return len(rec) * self.n + float(sizes.sum())

    def bytes_per_launch(self, kind):
        # algorithmic bytes: colour pass 36 B per site-update
        # (read own + neighbour class, write own; 12 B per FP32 3-vector);
        # Wolff: bond pass reads each site and its + neighbours once (12 B +
        # 4 B label write + 1 B crossing mask), flip reads label + spin (16 B)
        # fused step (one launch): sweep 36 B + bond/label pass 16 B (spins read
        # once, label written) + flip label read 4 B per site, and 24 B per
        # cluster site (the crossing-bond list is not counted)
        n = self.n
        c = getattr(self, "mean_cluster", 0.0)
        return {"metropolis": 36.0 * n / 2, "wolff_union": 17.0 * n, "wolff_flip": 4.0 * n + 24.0 * c,
                "wolff_merge": 1.0 * n, "fused": 56.0 * n + 24.0 * c}.get(kind, 36.0 * n / 2)

    def e2e(self, torch, K):
        """Every step starts from a configuration in pinned host memory: its
        3 MB upload (umc_chain_upload_async: copy stream, double-buffered
        staging) overlaps the step queued before it, and each step's record and
        cluster size stream back to pinned host memory as the step ends."""
        host = torch.empty((self.n, 3), dtype=torch.float32, pin_memory=True)
        host.numpy()[:] = self.ch.get_field()
        hn = host.numpy()
        self.ch.set_record_streaming(True)
        for _ in range(3):
            self.ch.upload_async(hn)
            self.ch.enqueue_hybrid(BETA, 1)
        self.ch.fetch(8)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            self.ch.upload_async(hn)
            self.ch.enqueue_hybrid(BETA, 1)
        _, sizes = self.ch.fetch(K)
        dt = time.perf_counter() - t0
        self.ch.set_record_streaming(False)
        u = K * self.n + float(sizes.sum())
        return {"value": u / dt, "unit": self.unit, "h2d_bytes_per_step": self.n * 12,
                "d2h_bytes_per_step": 8 * 8 + 8, "steps": K,
                "path": "umc_chain_upload_async + umc_hybrid_enqueue per step (upload overlaps the previous step), "
                        "records streamed to pinned host memory, one umc_chain_fetch at the end"}

    def cpu(self, seconds):
        est = reference_o3(self.L, 0, 1, 1)
        if est is None:
            return None
        threads = cpu_threads()
        steps = max(2, int(seconds / max(est[1], 1e-4)))
        su, sec, build = reference_o3(self.L, THERM_STEPS, steps, threads)
        return {"value": su / sec, "unit": self.unit, "cores": threads, "kind": "reference",
                         "build": build,
                "sample": f"{steps} steps x {threads} independent {self.L}^3 chains (reference stock driver, "
                          f"plain Pcg32) after {THERM_STEPS} untimed steps each, {sec:.1f} s"}


class IsingSweep:
    """Plain Ising Metropolis (Flip, J=1, beta=0.44) on an L x L lattice; step =
    one sweep.  At the default L = 32000 the int8 field is 0.95 GiB, far above L2
    (32768 would exceed the reference's uint32 bond count)."""

    name = "ising"
    unit = "site-updates/s"
    dtype = "i8"

    def __init__(self, umc, args, rank, local):
        self.L = args.L if args.L != L_DEFAULT else 32000
        self.n = self.L * self.L
        g = umc.square_lattice(self.L, self.L)
        self.ch = umc.Chain(umc.MODEL_ISING, graph=g, coupling=1, proposal=umc.PROPOSAL_FLIP, seed=1 + rank,
                            device=local, max_records=8192)
        self.ch.randomize(7 + rank)
        self.flush = self.n < (256 << 20)

    def describe(self):
        return (f"2D Ising {self.L}x{self.L} periodic, int8 spins, J=1, beta=0.44, Flip, random start; "
                f"step = 1 Metropolis sweep (packed checkerboard), E and M every sweep")

    def enqueue(self, k):
        self.ch.enqueue_metropolis(0.44, k)

    def units(self, rec, sizes):
        return len(rec) * self.n

    def bytes_per_launch(self, kind):
        return 3.0 * self.n / 2  # read own + other class, write own: 3 B per site-update

    def e2e(self, torch, K):
        host = torch.empty(self.n, dtype=torch.int8, pin_memory=True)
        host.numpy()[:] = self.ch.get_field()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            self.ch.set_field(host.numpy())
            self.ch.metropolis(0.44, 1)
        torch.cuda.synchronize()
        return {"value": K * self.n / (time.perf_counter() - t0), "unit": self.unit, "h2d_bytes_per_step": self.n,
                "d2h_bytes_per_step": 64, "steps": K}

    def cpu(self, seconds):
        r, build = timing_reference()
        if r is None:
            return None
        threads = cpu_threads()
        su, sec = r.bench_ising(64, 0.44, 10, 2000, threads, 1)
        return {"value": su / sec, "unit": self.unit, "cores": threads, "kind": "reference",
                         "build": build,
                "sample": f"2000 sweeps x {threads} independent 64x64 chains (reference stock driver)"}


class SU3Sweep:
    """SU(3) Wilson action on the L^4 hypercubic plaquette complex, beta = 5.7 in
    the model, SUShift width 0.2, 10 hits per link, reunitarisation and the FP64
    mean plaquette every sweep, Haar hot start; step = one sweep."""

    name = "su3"
    unit = "link-updates/s"
    dtype = "f32"

    def __init__(self, umc, args, rank, local):
        self.L = args.L if args.L != L_DEFAULT else 24
        cc = umc.hypercubic_plaquettes(self.L)
        self.n = cc.sites()
        self.ch = umc.Chain(umc.MODEL_SU, cells=cc, components=3, coupling=5.7, proposal=umc.PROPOSAL_SUSHIFT,
                            width=0.2, hits=10, seed=1 + rank, device=local, max_records=8192)
        self.ch.randomize(11 + rank)
        self.flush = True

    def describe(self):
        return (f"SU(3) Wilson action {self.L}^4 hypercubic_plaquettes, FP32 links, Haar start, beta=5.7, "
                f"SUShift 0.2, 10 hits per link, reunitarisation + FP64 mean plaquette every sweep")

    def enqueue(self, k):
        self.ch.enqueue_metropolis(1.0, k)

    def units(self, rec, sizes):
        return len(rec) * self.n

    def bytes_per_launch(self, kind):
        # per (mu, parity) pass: read 4.5 V links + write V/2 (72 B each) = 648 B per link-update
        return 648.0 * self.n / 8

    def e2e(self, torch, K):
        host = torch.empty((self.n, 18), dtype=torch.float32, pin_memory=True)
        host.numpy()[:] = self.ch.get_field()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            self.ch.set_field(host.numpy())
            self.ch.metropolis(1.0, 1)
        torch.cuda.synchronize()
        return {"value": K * self.n / (time.perf_counter() - t0), "unit": self.unit,
                "h2d_bytes_per_step": self.n * 72, "d2h_bytes_per_step": 64, "steps": K}

    def cpu(self, seconds):
        """The reference's SUGauge<3> with SUShift 0.2 and 10 hits per link
        (multi-hit through a window adapter), one chain per thread, timed on a
        window of each thread's lattice: a full 24^4 sweep of 10 hits takes
        about a minute per core, so the rate of a bounded window is reported."""
        r, build = timing_reference()
        if r is None:
            return None
        threads = cpu_threads()
        su, sec = r.bench_su3(self.L, 5.7, 0.2, 10, 2000, 1, 1, 1)
        window = max(2000, min(self.n, int(2000 * seconds / max(sec, 1e-4))))
        su, sec = r.bench_su3(self.L, 5.7, 0.2, 10, window, 1, threads, 1)
        return {"value": su / sec, "unit": self.unit, "cores": threads, "kind": "reference",
                         "build": build,
                "sample": f"{threads} independent {self.L}^4 chains (reference SUGauge<3>, SUShift 0.2, 10 hits per "
                          f"link, cold start), each timed on one pass over a window of {window} of its "
                          f"{self.n} links ({sec:.1f} s); the rate of a full sweep is extrapolated from it"}


class XYBatch:
    """Batched replica run: 32 ladders x 16 XY chains, L drawn per ladder from
    {16, 32, 64, 128, 256} (seeded), betas geometric on [0.8, 1.3], U1Shift 1.0,
    exchange every 10 sweeps; step = one segment (10 sweeps of every chain +
    one exchange round)."""

    name = "xybatch"
    unit = "site-updates/s"
    dtype = "f32"

    def __init__(self, umc, args, rank, local):
        np_ = __import__("numpy")
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rng = np_.random.default_rng(2024)
        self.Ls = rng.choice([16, 32, 64, 128, 256], size=32)
        R = 16
        self.betas = np_.stack([0.8 * (1.3 / 0.8) ** (np_.arange(R) / (R - 1))] * 32)
        # under torchrun the 32 ladders shard over the ranks (no exchange between
        # shards): the job's work is fixed, so the scaling is strong
        self.b = umc.Batch.shard(self.Ls, self.betas, rank, ws, coupling=1.0, width=1.0, sweeps_per_exchange=10,
                                 seed=1, device=local, max_records=8192)
        self.scaling = "strong" if ws > 1 else "weak"
        self.parallelism = f"ladders sharded over {ws} ranks" if ws > 1 else "1 GPU, 512 chains"
        self.Ls_all = self.Ls
        lo, hi = self.b.ladder_range
        self.Ls = self.Ls[lo:hi]
        self.b.randomize(17 + rank)
        self.n, _ = self.b.sites()
        self.L = int(self.Ls.max())
        self.flush = True
        self.ch = _BatchAsChain(self.b)

    def describe(self):
        counts = {int(L): int((self.Ls_all == L).sum()) for L in sorted(set(self.Ls_all.tolist()))}
        info = self.b.persistent_info()
        if info["enabled"]:
            form = (f"one persistent kernel per step ({info['grid']} CTAs of 1024 threads in clusters of "
                    f"{info['cluster']}, {info['ctas_per_sm']} per SM, {info['big_items']} cluster-swept chains, "
                    f"{info['items']} work items)")
        else:
            shapes = {L: self.b.config(L) for L in sorted(set(int(x) for x in self.Ls))}
            form = f"one kernel per side group + the exchange kernel, as one graph per step (shapes {shapes})"
        return (f"512 XY chains in 32 replica-exchange ladders of 16, L per ladder {counts} (ladders per L), "
                f"FP32 angles, J=1, betas geometric on [0.8, 1.3], U1Shift 1.0, swaps every 10 sweeps; "
                f"step = 10 sweeps of every chain + one exchange round, {form}; the faster form "
                f"measured at creation")

    def enqueue(self, k):
        self.b.enqueue(k)

    def units(self, rec, sizes):
        return len(rec) * self.n * 10

    def bytes_per_launch(self, kind):
        return 12.0 * self.n * 10  # 3 x 4 B per site-update

    def e2e(self, torch, K):
        import numpy as np_

        fields = [self.b.get_field(c) for c in range(self.b.n_chains)]
        pinned = [torch.from_numpy(f).pin_memory() for f in fields]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            for c, p in enumerate(pinned):
                self.b.set_field(c, p.numpy())
            self.b.run(1)
        torch.cuda.synchronize()
        return {"value": K * self.n * 10 / (time.perf_counter() - t0), "unit": self.unit,
                "h2d_bytes_per_step": self.n * 4, "d2h_bytes_per_step": self.b.n_chains * 64, "steps": K}

    def cpu(self, seconds):
        r, build = timing_reference()
        if r is None:
            return None
        threads = cpu_threads()
        su, sec = r.bench_xy(64, 1.0, 1.0, 2, 50, 1, 1)
        sweeps = max(10, int(seconds * 50 / max(sec, 1e-4)))
        su, sec = r.bench_xy(64, 1.0, 1.0, 2, sweeps, threads, 1)
        return {"value": su / sec, "unit": self.unit, "cores": threads, "kind": "reference",
                         "build": build,
                "sample": f"{sweeps} sweeps x {threads} independent 64x64 XY chains (reference PairModel + "
                          f"U1Shift, stock driver), {sec:.1f} s"}


# ------------------------------------------------------- learned U(1) study
LEARN_BETAS = (2.0, 4.0, 6.0, 8.0)


def _timed_sweeps(torch, b, n, net, chunk=100):
    """n sweeps of every chain of the batch in launches of `chunk` sweeps, each
    launch timed with CUDA events on the batch's stream and preceded (outside
    the events) by a 256 MiB write that evicts the chains from L2."""
    import numpy as np

    s = torch.cuda.ExternalStream(b.stream())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    recs, ms = [], 0.0
    done = 0
    torch.cuda.synchronize()
    while done < n:
        k = min(chunk, n - done)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            flush.fill_(done & 0xFF)
            e0.record(s)
            b.enqueue(k, net)
            e1.record(s)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        recs.append(b.fetch(k))
        done += k
    return np.concatenate(recs), ms / n


def _chain_ms_per_sweep(torch, ch, n):
    s = torch.cuda.ExternalStream(ch.stream())
    ch.enqueue_metropolis(1.0, 20)
    ch.fetch(8192)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    ch.enqueue_metropolis(1.0, n)
    e1.record(s)
    e1.synchronize()
    ch.fetch(8192)
    return e0.elapsed_time(e1) / n


def torus_plaquette(beta, n_plaq):
    """Exact <cos theta_p> of 2D U(1) (Wilson action) on a periodic torus of
    n_plaq plaquettes: Z = sum_n I_n(beta)^n_plaq (character expansion), so
    <P> = sum_n I_n^(n_plaq - 1) I_n' / sum_n I_n^n_plaq, I_n' = (I_{n-1} + I_{n+1}) / 2."""
    import numpy as np
    import scipy.special as sp

    ns = np.arange(-60, 61)
    li = np.log(sp.ive(ns, beta))
    ld = np.log(0.5 * (sp.ive(ns - 1, beta) + sp.ive(ns + 1, beta)))
    a = (n_plaq - 1) * li + ld
    b = n_plaq * li
    lse = lambda v: v.max() + np.log(np.exp(v - v.max()).sum())
    return float(np.exp(lse(a) - lse(b)))


def torus_plaquette_sectors(beta, n_plaq, charges, weights=None):
    """Exact <cos theta_p> of 2D U(1) on a periodic torus of n_plaq plaquettes
    within each topological sector Q of `charges` (Q = sum_p wrap(theta_p) /
    2 pi).  With the plaquette angles independent apart from sum_p theta_p =
    2 pi Q, Z_Q = int dk cos(2 pi k Q) c(k)^n_plaq with c(k) = (1/pi) int_0^pi
    e^{beta cos t} cos(k t) dt, and <P>_Q = int cos(2 pi k Q) c^(n-1) c' /
    int cos(2 pi k Q) c^n, c' = dc/dbeta; summed over Q with weights Z_Q this
    is torus_plaquette (Poisson summation turns the k integral into the sum
    over representations).  Local updates at large beta rarely change Q, so a
    chain's plaquette is compared with the sector values of the charges it
    visited.  Quadrature: Gauss-Legendre in t, trapezoid in k.  weights, if a
    dict, receives Z_Q / Z_0 for each Q."""
    import numpy as np

    t, w = np.polynomial.legendre.leggauss(400)
    t = 0.5 * np.pi * (t + 1.0)
    w = 0.5 * np.pi * w
    width = 12.0 * np.sqrt(max(beta, 1.0) / n_plaq)  # c^n decays as exp(-n k^2 / (2 beta))
    k = np.linspace(0.0, min(width, 4.0), 4001)
    e = np.exp(beta * (np.cos(t) - 1.0))                     # scaled by e^-beta
    ck = (np.cos(np.outer(k, t)) * e) @ w / np.pi
    dk = (np.cos(np.outer(k, t)) * (np.cos(t) * e)) @ w / np.pi
    if (ck <= 0).any():
        raise ValueError("c(k) changes sign inside the k range")
    lc = np.log(ck)
    base = n_plaq * lc[0]
    out = {}
    for Q in charges:
        cq = np.cos(2.0 * np.pi * k * Q)
        zn = np.trapezoid(cq * np.exp(n_plaq * lc - base), k)
        zd = np.trapezoid(cq * np.exp((n_plaq - 1) * lc - base) * dk, k)
        out[int(Q)] = float(zd / zn)
        if weights is not None:
            weights[int(Q)] = float(zn)
    if weights is not None and 0 in weights:
        z0 = weights[0]
        for q in weights:
            weights[q] /= z0
    return out


def sector_matched_plaquette(beta, n_plaq, charges):
    """The exact plaquette a sampler should show given the charges it visited:
    the mean over records of <P>_Q(record)."""
    import numpy as np

    q = np.rint(np.asarray(charges)).astype(int).ravel()
    vals, counts = np.unique(q, return_counts=True)
    table = torus_plaquette_sectors(beta, n_plaq, vals)
    return float(sum(table[int(v)] * c for v, c in zip(vals, counts)) / counts.sum())


def learned_study(umc, torch, betas=LEARN_BETAS, L=64, chains=444, n_configs=20000, train_steps=1500,
                  batch=16384, lr=3e-3, therm=20000, meas=4000, seed=1):
    """Effective independent samples per second of the plaquette P and the
    topological charge Q on 2D U(1) L x L, for plain U1Shift(0.5) Metropolis on
    one chain (the faster of the single-chain engine and the batch kernel with
    one chain), plain batched, and learned batched (the network trained on
    n_configs plain-chain configurations of the same beta).  Effective samples
    per second = chains x sweeps per second / (2 tau_int), tau_int pooled over
    the chains (umc.tau_int_multi)."""
    import numpy as np

    out = {}
    for beta in betas:
        t_start = time.perf_counter()
        # cold start (all angles 0), as the reference's U1Gauge constructs its
        # links (example/u1_gauge.hpp:23-25).  A hot start leaves each chain
        # with a topological charge of order sqrt(V / 12) that local updates
        # cannot shed at beta >= 6; the excess action then biases the
        # plaquette low by several standard errors.
        plain = umc.U1Batch(chains, L, beta, width=0.5, seed=seed, max_records=max(meas, 200))
        plain.run(therm, records=False)
        snaps = -(-n_configs // chains)
        net = umc.ProposalNet(seed + 7, max_configs=snaps * chains, L=L)
        for _ in range(snaps):
            plain.run(5, records=False)
            net.add_configs(plain)
        t0 = time.perf_counter()
        losses = net.train(train_steps, batch=batch, lr=lr)
        train_s = time.perf_counter() - t0
        learned = umc.U1Batch(chains, L, beta, seed=seed + 1, max_records=max(meas, 200))
        for c in range(chains):
            learned.set_field(c, plain.get_field(c))
        learned.run(20, net, records=False)
        rec_p, ms_p = _timed_sweeps(torch, plain, meas, None)
        rec_l, ms_l = _timed_sweeps(torch, learned, meas, net)
        one = umc.U1Batch(1, L, beta, width=0.5, seed=seed, max_records=1000)
        one.set_field(0, plain.get_field(0))
        _, ms_one = _timed_sweeps(torch, one, 1000, None, chunk=1000)
        ch = umc.Chain(umc.MODEL_U1, cells=umc.square_plaquettes(L), coupling=beta, proposal=umc.PROPOSAL_U1SHIFT,
                       width=0.5, seed=seed, max_records=8192)
        ch.set_field(plain.get_field(0))
        ms_chain = _chain_ms_per_sweep(torch, ch, 1000)
        ms_single = min(ms_one, ms_chain)
        row = {"ms_per_sweep": {"plain_single_chain": ms_single, "plain_single_chain_engine": ms_chain,
                                "plain_batch_kernel_one_chain": ms_one, "plain_batched": ms_p,
                                "learned_batched": ms_l},
               "acceptance": {"plain": float(rec_p[:, :, 3].mean() / (2 * L * L)),
                              "learned": float(rec_l[:, :, 3].mean() / (2 * L * L))},
               "train": {"configs": net.configs(), "steps": train_steps, "batch": batch, "lr": lr,
                         "loss_first": float(losses[0]), "loss_last": float(np.mean(losses[-20:])),
                         "seconds": train_s}}
        for name, idx in (("plaquette", 1), ("Q", 2)):
            tp, ep, wp = umc.tau_int_multi(rec_p[:, :, idx].T)
            tl, el, wl = umc.tau_int_multi(rec_l[:, :, idx].T)
            mp, ml = rec_p[:, :, idx].mean(0), rec_l[:, :, idx].mean(0)
            err = float(np.hypot(mp.std(ddof=1), ml.std(ddof=1)) / np.sqrt(chains))
            eff = {"plain_single_chain": 1e3 / ms_single / (2 * tp),
                   "plain_batched": chains * 1e3 / ms_p / (2 * tp),
                   "learned_batched": chains * 1e3 / ms_l / (2 * tl)}
            if name == "plaquette":
                exact = torus_plaquette(beta, L * L)
                row["exact_plaquette"] = exact
                row["z_vs_exact"] = {"plain": float((mp.mean() - exact) / (mp.std(ddof=1) / np.sqrt(chains))),
                                     "learned": float((ml.mean() - exact) / (ml.std(ddof=1) / np.sqrt(chains)))}
                # the known answer for the sectors each sampler visited (at
                # large beta local updates keep a chain near its charge)
                sp = sector_matched_plaquette(beta, L * L, rec_p[:, :, 2])
                sl = sector_matched_plaquette(beta, L * L, rec_l[:, :, 2])
                row["sector_matched_plaquette"] = {"plain": sp, "learned": sl}
                row["z_vs_sector_exact"] = {"plain": float((mp.mean() - sp) / (mp.std(ddof=1) / np.sqrt(chains))),
                                            "learned": float((ml.mean() - sl) / (ml.std(ddof=1) / np.sqrt(chains)))}
            row[name] = {"tau_int": {"plain": tp, "plain_err": ep, "learned": tl, "learned_err": el},
                         "tau_converged": {"plain": wp < meas // 2, "learned": wl < meas // 2},
                         "effective_samples_per_s": eff,
                         "learned_batched_over_plain_single": eff["learned_batched"] / eff["plain_single_chain"],
                         "learned_over_plain_at_equal_batch": eff["learned_batched"] / eff["plain_batched"],
                         "mean": {"plain": float(mp.mean()), "learned": float(ml.mean()),
                                  "z": float((ml.mean() - mp.mean()) / err) if err > 0 else 0.0}}
        row["seconds"] = time.perf_counter() - t_start
        out[f"beta={beta:g}"] = row
        for o in (plain, learned, one, net):
            o.close()
    return out


class _BatchAsChain:
    """The few chain methods the timing loop uses, for a batch."""

    def __init__(self, b):
        self.b = b
        self.timing = False

    def stream(self):
        return self.b.stream()

    def fetch(self, cap):
        rec = self.b.fetch(cap)
        return rec, __import__("numpy").zeros(len(rec))

    def kernel_stats(self, reset=False):
        _, k = self.b.sites()
        out = {"batch": (k - getattr(self, "_base", 0), 0.0)}
        if reset:
            self._base = k
        return out

    def set_timing(self, on):
        self.timing = on


class _U1AsChain:
    """The few chain methods the timing loop uses, for a U(1) batch."""

    def __init__(self, b):
        self.b = b

    def stream(self):
        return self.b.stream()

    def fetch(self, cap):
        rec = self.b.fetch(min(cap, self.b.max_records))
        return rec, __import__("numpy").zeros(len(rec))

    def kernel_stats(self, reset=False):
        _, k = self.b.counters()
        out = {"learned": (k - getattr(self, "_base", 0), 0.0)}
        if reset:
            self._base = k
        return out

    def set_timing(self, on):
        pass


class U1LearnedSweep:
    """The learned sampler alone: 444 2D U(1) 64x64 chains at beta 4, one
    learned sweep per step (MLP 3-64-64-16 in BF16 on tcgen05, von Mises
    mixture, MH), network weights from a fixed seed (untrained)."""

    name = "u1batch"
    unit = "link-updates/s"
    dtype = "bf16/f32"
    chains = 444

    def __init__(self, umc, args, rank, local):
        self.L = 64
        self.b = umc.U1Batch(self.chains, self.L, 4.0, width=0.5, seed=1 + rank, device=local, max_records=4096)
        self.b.run(200, records=False)
        self.net = umc.ProposalNet(3 + rank, device=local)
        self.n = self.chains * 2 * self.L * self.L
        self.flush = True
        self.ch = _U1AsChain(self.b)

    def describe(self):
        return (f"learned sampler: {self.chains} 2D U(1) {self.L}x{self.L} chains, beta 4, one learned sweep per step "
                f"(MLP 3-64-64-16 BF16 tcgen05, 4-component von Mises mixture, MH); network from a fixed seed")

    def enqueue(self, k):
        self.b.enqueue(k, self.net)

    def units(self, rec, sizes):
        return len(rec) * self.n

    def flops_per_launch(self, kind):
        return 10624.0 * self.n  # network forward per link-update (tensor cores)

    def bytes_per_launch(self, kind):
        return 20.0 * self.n

    def e2e(self, torch, K):
        return None

    def cpu(self, seconds):
        return None


# ------------------------------------------------ user-written device models
def _device_models_lib():
    """examples/device_models/libumc_device_models.so (built when stale)."""
    import ctypes as C

    sys.path.insert(0, os.path.join(ROOT, "examples", "device_models"))
    import build_device_models

    lib = C.CDLL(build_device_models.build())
    vp, d, u32, u64 = C.c_void_p, C.c_double, C.c_uint32, C.c_uint64
    lib.um_last_error.restype = C.c_char_p
    lib.um_session_create.argtypes = [C.c_int, vp, u32, u32, u32, d, d, d, u64, C.POINTER(vp)]
    lib.um_session_destroy.argtypes = [vp]
    lib.um_session_stream.argtypes = [vp]
    lib.um_session_stream.restype = vp
    lib.um_session_set_field.argtypes = [vp, vp]
    lib.um_session_get_field.argtypes = [vp, vp]
    lib.um_session_enqueue.argtypes = [vp, u64]
    lib.um_session_set_timing.argtypes = [vp, C.c_int]
    lib.um_session_stats.argtypes = [vp, C.POINTER(u64), C.POINTER(d), C.c_int]
    lib.um_session_energy.argtypes = [vp, C.POINTER(d)]
    lib.um_session_counters.argtypes = [vp, C.POINTER(u64), C.POINTER(u32)]
    lib.um_session_take_sizes.argtypes = [vp, vp, u64, C.POINTER(u64)]
    return lib


class _SessionAsChain:
    """The few chain methods the timing loop uses, for a device-model session."""

    def __init__(self, wl):
        self.wl = wl
        self.pending = 0

    def stream(self):
        return self.wl.lib.um_session_stream(self.wl.h)

    def fetch(self, cap):
        import ctypes as C

        import numpy as np

        self.kernel_stats(reset=False)  # waits for the stream, surfaces a device error
        rec = np.zeros((self.pending, 1))
        sizes = np.zeros(self.pending, np.uint64)
        got = C.c_uint64()
        self.wl.call(self.wl.lib.um_session_take_sizes(self.wl.h, sizes.ctypes.data, len(sizes), C.byref(got)))
        self.pending = 0
        return rec, sizes[:min(got.value, len(sizes))]

    def kernel_stats(self, reset=False):
        import ctypes as C

        n, ms = C.c_uint64(), C.c_double()
        self.wl.call(self.wl.lib.um_session_stats(self.wl.h, C.byref(n), C.byref(ms), int(reset)))
        return {getattr(self.wl, "kernel_name", "metropolis_sweeps"): (n.value, ms.value)}

    def set_timing(self, on):
        self.wl.call(self.wl.lib.um_session_set_timing(self.wl.h, int(on)))


class _UserSession:
    """A session of examples/device_models/user_models.cu: tables, field and
    the generic device Metropolis of include/umc/device.cuh for one user
    model; step = one sweep = one cooperative launch of metropolis_sweeps."""

    unit = "site-updates/s"

    def _open(self, umc, kind, graph, dims, J, beta, width, seed, field):
        import ctypes as C

        self.lib = _device_models_lib()
        h = C.c_void_p()
        self.call(self.lib.um_session_create(kind, graph, *dims, J, beta, width, seed, C.byref(h)))
        self.h = h
        self.field = field
        self.call(self.lib.um_session_set_field(self.h, self.field.ctypes.data))
        self.ch = _SessionAsChain(self)

    def call(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.um_last_error().decode())

    def enqueue(self, k):
        self.call(self.lib.um_session_enqueue(self.h, k))
        self.ch.pending += k

    def units(self, rec, sizes):
        return len(rec) * self.n

    def e2e(self, torch, K):
        import ctypes as C

        host = torch.from_numpy(self.field.copy()).pin_memory()
        e = C.c_double()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            self.call(self.lib.um_session_set_field(self.h, host.data_ptr()))
            self.enqueue(1)
            self.call(self.lib.um_session_energy(self.h, C.byref(e)))
        torch.cuda.synchronize()
        self.ch.fetch(0)
        blocks = min(1024, (self.n + 255) // 256)
        return {"value": K * self.n / (time.perf_counter() - t0), "unit": self.unit,
                "h2d_bytes_per_step": self.field.nbytes, "d2h_bytes_per_step": blocks * 8, "steps": K}


class UserXY(_UserSession):
    """The XY model on angles as PairModel<Angle, CosineTerm> with the
    AngleShift (U1Shift) proposal, FP64, from examples/device_models, on an
    L x L square_lattice (CSR bond table), J=1, beta=1.1, width 1.0, random
    start.  The reference runs the same model as PairModel<U1Dof, user term,
    PairGraph> through its stock Metropolis driver."""

    name = "userxy"
    dtype = "f64"

    def __init__(self, umc, args, rank, local):
        import numpy as np

        self.L = args.L if args.L != L_DEFAULT else 8192
        self.n = self.L * self.L
        self.g = umc.square_lattice(self.L, self.L)
        theta = np.random.default_rng(5 + rank).uniform(-np.pi, np.pi, self.n)
        self._open(umc, 0, self.g._h, (0, 0, 0), 1.0, 1.1, 1.0, 1 + rank, theta)
        self.flush = self.n * 8 < (256 << 20)

    def describe(self):
        return (f"user-written XY PairModel (CosineTerm + AngleShift, FP64, examples/device_models) on "
                f"{self.L}x{self.L} square_lattice, J=1, beta=1.1, width 1.0, random start; step = 1 Metropolis "
                f"sweep (one launch of the generic device kernel over the 2 colour classes)")

    def bytes_per_launch(self, kind):
        # per site-update: order 4 + offset 4 + 4 bonds 16 + field read as own
        # and as a neighbour 16 + write 8 = 48 B
        return 48.0 * self.n

    def cpu(self, seconds):
        r, build = timing_reference()
        if r is None:
            return None
        threads = cpu_threads()
        su, sec = r.bench_xy(256, 1.1, 1.0, 1, 5, 1, 1)
        sweeps = max(5, int(seconds * 5 / max(sec, 1e-4)))
        su, sec = r.bench_xy(256, 1.1, 1.0, 1, sweeps, threads, 1)
        return {"value": su / sec, "unit": self.unit, "cores": threads, "kind": "reference",
                         "build": build,
                "sample": f"{sweeps} sweeps x {threads} independent 256x256 XY chains (reference PairModel<U1Dof, "
                          f"user term> + U1Shift, stock driver), {sec:.1f} s"}


class UserO3(_UserSession):
    """A user-written FP32 Heisenberg pair term (DotTerm<float, 3> with an
    FP32 UniformSphereN<3>) on an L^3 periodic cubic lattice, J=1, beta=0.693,
    random unit start.  usero3: the table-free RegularLattice (neighbours
    computed, nothing about bonds read); usero3csr: the same model on the
    lattice's CSR tables (PairTables)."""

    dtype = "f32"

    def __init__(self, umc, args, rank, local, tables=False):
        import numpy as np

        self.tables = tables
        self.name = "usero3csr" if tables else "usero3"
        self.L = args.L if args.L != L_DEFAULT else 256
        self.n = self.L ** 3
        v = np.random.default_rng(9 + rank).normal(size=(self.n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        self._open(umc, 2 if tables else 1, None, (self.L, self.L, self.L), 1.0, 0.693, 0.0, 1 + rank,
                   np.ascontiguousarray(v, np.float32).reshape(-1))
        self.flush = self.n * 12 < (256 << 20)

    def describe(self):
        where = "PairTables (the lattice's CSR)" if self.tables else "RegularLattice (no bond tables)"
        return (f"user-written FP32 Heisenberg PairModel (DotTerm<float,3> + FP32 UniformSphereN<3>, "
                f"examples/device_models) on {self.L}^3 periodic cubic, {where}, J=1, beta=0.693, random start; "
                f"step = 1 Metropolis sweep (one launch of the generic device kernel)")

    def bytes_per_launch(self, kind):
        # 36 B per site-update (own 12 read, 12 as a neighbour, 12 write); the
        # tables add offset 4 + six bonds 24
        return (64.0 if self.tables else 36.0) * self.n

    def cpu(self, seconds):
        r, build = timing_reference()
        if r is None:
            return None
        threads = cpu_threads()
        su, sec = r.bench_pair_o3(32, 0.693, 1, 3, 1, 1)
        sweeps = max(3, int(seconds * 3 / max(sec, 1e-4)))
        su, sec = r.bench_pair_o3(32, 0.693, 1, sweeps, threads, 1)
        return {"value": su / sec, "unit": self.unit, "cores": threads, "kind": "reference",
                         "build": build,
                "sample": f"{sweeps} sweeps x {threads} independent 32^3 chains (reference PairModel<VectorDof<3>, "
                          f"HeisenbergTerm<3>> + UniformSphereN<3>, stock driver, FP64), {sec:.1f} s"}


class UserO3Csr(UserO3):
    def __init__(self, umc, args, rank, local):
        super().__init__(umc, args, rank, local, tables=True)


class UserIsingWolff(_UserSession):
    """A user-written Ising pair term in int32 on int8 spins (IsingBondTerm)
    with a fixed axis, driven by the generic device Wolff of
    include/umc/device.cuh on an L x L square_lattice's tables, J=1,
    beta=0.44, cold start; step = one cluster flip (bond activation,
    union-find labelling and the seed cluster's flip in one cooperative
    launch).  Units: flipped sites.  The reference runs
    Wolff<Ising, FixedAxis> through its stock driver."""

    name = "userwolff"
    dtype = "i8"

    def __init__(self, umc, args, rank, local):
        import numpy as np

        self.L = args.L if args.L != L_DEFAULT else 2048
        self.n = self.L * self.L
        self.g = umc.square_lattice(self.L, self.L)
        s = np.ones(self.n, np.int8)  # cold start, as Ising's constructor (example/ising.hpp:24)
        self._open(umc, 3, self.g._h, (0, 0, 0), 1.0, 0.44, 0.0, 1 + rank, s)
        self.kernel_name = "wolff_flips"
        self.flush = True  # field, parent array and tables (about 100 MB at 2048^2) fit in L2
        self.mean_cluster = 0.0

    def describe(self):
        return (f"user-written Ising PairModel (IsingBondTerm int32 on int8, UpAxis = FixedAxis, "
                f"examples/device_models) on {self.L}x{self.L} square_lattice tables, J=1, beta=0.44, cold "
                f"start; step = 1 Wolff flip of the generic device kernel; units = flipped sites")

    def units(self, rec, sizes):
        if len(sizes):
            self.mean_cluster = float(sizes.mean())
        return float(sizes.sum())

    def bytes_per_launch(self, kind):
        # per site and flip: parent init 4 + offset 4 + four bonds 16 + own and
        # neighbour spins 2 + parent read in the flip 4 = 30 B; per cluster
        # site the spin's read and write, 2 B
        return 30.0 * self.n + 2.0 * self.mean_cluster

    def e2e(self, torch, K):
        import ctypes as C

        # the chain's current (equilibrated) field, uploaded before every flip:
        # each step is one flip from the same state, like the timed steps
        host = torch.empty(self.n, dtype=torch.int8, pin_memory=True)
        self.call(self.lib.um_session_get_field(self.h, host.data_ptr()))
        self.ch.fetch(0)
        e = C.c_double()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            self.call(self.lib.um_session_set_field(self.h, host.data_ptr()))
            self.enqueue(1)
            self.call(self.lib.um_session_energy(self.h, C.byref(e)))
        torch.cuda.synchronize()
        _, sizes = self.ch.fetch(0)
        return {"value": float(sizes.sum()) / (time.perf_counter() - t0), "unit": self.unit,
                "h2d_bytes_per_step": self.field.nbytes, "d2h_bytes_per_step": 8 + min(1024, (self.n + 255) // 256) * 8,
                "steps": K}

    def cpu(self, seconds):
        r, build = timing_reference()
        if r is None:
            return None
        threads = cpu_threads()
        su, sec = r.bench_ising_wolff(256, 0.44, 50, 50, 1, 1)
        flips = max(50, int(seconds * 50 / max(sec, 1e-4)))
        su, sec = r.bench_ising_wolff(256, 0.44, 200, flips, threads, 1)
        return {"value": su / sec, "unit": self.unit, "cores": threads, "kind": "reference",
                         "build": build,
                "sample": f"{flips} flips x {threads} independent 256x256 Ising chains (reference Wolff<Ising, "
                          f"FixedAxis>, stock driver, 200 warm-up flips), {sec:.1f} s"}


class UserU1(_UserSession):
    """A user-written U(1) plaquette cell term (PlaquetteTerm, FP64: beta (1 -
    cos(t0 + t1 - t2 - t3))) with AngleShift 0.7 on L^4 hypercubic plaquettes,
    model beta 1.1, random start; step = one sweep (8 colour classes, one
    launch of the generic device kernel).  useru1: the table-free
    PlaquetteLattice (a link's plaquettes computed); useru1tables: the same
    on the library's cell and incidence tables (CellTables)."""

    unit = "link-updates/s"
    dtype = "f64"

    def __init__(self, umc, args, rank, local, tables=False):
        import numpy as np

        self.tables = tables
        self.name = "useru1tables" if tables else "useru1"
        self.L = args.L if args.L != L_DEFAULT else 48
        self.n = 4 * self.L ** 4
        theta = np.random.default_rng(21 + rank).uniform(-np.pi, np.pi, self.n)
        self._open(umc, 4 if tables else 5, None, (self.L, 0, 0), 1.1, 1.0, 0.7, 1 + rank, theta)
        self.flush = self.n * 8 < (256 << 20)

    def describe(self):
        where = "hypercubic_plaquettes tables (CellTables)" if self.tables else "PlaquetteLattice (no tables)"
        return (f"user-written U(1) plaquette term (FP64, examples/device_models) on {self.L}^4, {where}, model "
                f"beta 1.1, AngleShift 0.7, random start; step = 1 Metropolis sweep (one launch)")

    def bytes_per_launch(self, kind):
        # per (direction, parity) pass: read 4.5 V links and write V/2 (8 B
        # each) for V/2 link-updates = 80 B per link-update; the tables add
        # the offset 8, six (cell, slot) entries 30 and six cells' links 96
        return (214.0 if self.tables else 80.0) * self.n

    def cpu(self, seconds):
        r, build = timing_reference()
        if r is None:
            return None
        threads = cpu_threads()
        su, sec = r.bench_u1_cells(8, 1.1, 1.0, 0.7, 1, 2, 1, 1)
        sweeps = max(2, int(seconds * 2 / max(sec, 1e-4)))
        su, sec = r.bench_u1_cells(8, 1.1, 1.0, 0.7, 1, sweeps, threads, 1)
        return {"value": su / sec, "unit": self.unit, "cores": threads, "kind": "reference",
                         "build": build,
                "sample": f"{sweeps} sweeps x {threads} independent 8^4 chains (reference CellModel<U1Dof, "
                          f"U1PlaquetteTerm, CellComplex<4>> + U1Shift, stock driver, FP64), {sec:.1f} s"}


class UserU1Tables(UserU1):
    def __init__(self, umc, args, rank, local):
        super().__init__(umc, args, rank, local, tables=True)


WORKLOADS = {"o3": O3Hybrid, "ising": IsingSweep, "su3": SU3Sweep, "xybatch": XYBatch, "u1batch": U1LearnedSweep,
             "userxy": UserXY, "usero3": UserO3, "usero3csr": UserO3Csr, "userwolff": UserIsingWolff,
             "useru1": UserU1, "useru1tables": UserU1Tables}


def run_learned(args):
    """--workload u1learned: the full study, one JSON line."""
    import numpy as np
    import torch

    torch.cuda.set_device(0)
    import universal_classical_montecarlo_b200 as umc

    sampler = ClockSampler("GPU-" + str(torch.cuda.get_device_properties(0).uuid))
    sampler.start()
    time.sleep(0.3)
    study = learned_study(umc, torch, meas=args.steps if args.steps != 4000 else 4000)
    clocks = sampler.stop()
    eff = [row["plaquette"]["effective_samples_per_s"]["learned_batched"] for row in study.values()]
    line = {"metric": METRIC, "value": float(np.exp(np.mean(np.log(eff)))),
            "unit": "effective samples/s (plaquette, geometric mean over beta)", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "learned proposal on 2D U(1) 64x64, beta in {2,4,6,8}, 444 chains per batch, "
                                   "plain U1Shift 0.5 vs MLP 3-64-64-16 (BF16 tcgen05) 4-component von Mises "
                                   "mixture trained on 20000 plain-chain configurations per beta",
                       "l2": "256 MiB flush between timed launches of 100 sweeps"},
            "per_beta": study, "clocks": clocks}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------- umc
def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "u1learned":
        run_learned(args)
        return
    ws, rank, local = rank_info()
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    import universal_classical_montecarlo_b200 as umc

    wl = WORKLOADS[args.workload](umc, args, rank, local)
    therm_cluster = wl.thermalise() if hasattr(wl, "thermalise") else None
    ch = wl.ch
    stream = torch.cuda.ExternalStream(ch.stream(), device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if wl.flush else None

    def barrier():
        if ws > 1:
            dist.barrier()

    # ---- warm-up
    wl.enqueue(args.warmup)
    ch.fetch(8192)
    ch.kernel_stats(reset=True)

    # ---- timed region: K steps (L2 flushed between steps when the state fits
    # in L2), each step timed with CUDA events on the chain's stream
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
            if flush is not None:
                flush.fill_(k & 0xFF)
            starts[k].record(stream)
            wl.enqueue(1)
            ends[k].record(stream)
            done += 1
            if done == 4096:  # drain the record ring
                rec, sizes = ch.fetch(8192)
                units += wl.units(rec, sizes)
                done = 0
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    rec, sizes = ch.fetch(8192)
    units += wl.units(rec, sizes)
    launches = ch.kernel_stats(reset=True)
    gpu_launches = sum(v[0] for k, v in launches.items())
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))

    # ---- dominant kernel, timed live with events around each launch (for the
    # batch, one launch = the captured segment graph, timed by the step events)
    if wl.name == "xybatch":
        per_kind = {"batch": (K, total_ms)}
    elif wl.name == "u1batch":
        per_kind = {"learned": (K, total_ms)}
    elif len([k for k, v in launches.items() if v[0]]) == 1 and gpu_launches == K:
        # one launch per step: the step events time the kernel itself
        per_kind = {next(k for k, v in launches.items() if v[0]): (K, total_ms)}
    else:
        per_kind = None
    ch.set_timing(True)
    KP = min(K, 2000) if per_kind is None else 0
    with torch.cuda.stream(stream):
        for k in range(KP):
            if flush is not None:
                flush.fill_(k & 0xFF)
            wl.enqueue(1)
            if (k + 1) % 4096 == 0:
                ch.fetch(8192)
    if per_kind is None:
        ch.fetch(8192)
        per_kind = ch.kernel_stats(reset=True)
    ch.set_timing(False)
    if wl.name == "o3" and len(sizes):
        wl.mean_cluster = float(sizes.mean())
    kind, (nl, ms) = max(((k, v) for k, v in per_kind.items() if v[0] > 0 and k != "other"),
                         key=lambda kv: kv[1][1])
    avg_s = ms / nl / 1e3
    traffic = profiled_traffic(f"{wl.name}:{kind}", 1.0)
    if hasattr(wl, "flops_per_launch"):
        achieved = wl.flops_per_launch(kind) / avg_s / 1e12
        peak, peak_src = measured_peak_bf16()
        roof = {"bound": "tensor", "unit": "TFLOP/s",
                "peak_source": "of measured (MEASURED_PEAKS.json bf16_tflops)" if peak_src == "measured"
                else "of fallback 1.59 PFLOP/s"}
    else:
        achieved = wl.bytes_per_launch(kind) / avg_s / 1e9
        peak, peak_src = measured_peak_hbm()
        roof = {"bound": "hbm", "unit": "GB/s",
                "peak_source": "of measured (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                else "of fallback 6.65 TB/s"}

    # ---- end to end through the C ABI with host buffers
    e2e = None if args.no_e2e else wl.e2e(torch, min(K, 300))

    # ---- aggregate over ranks
    max_ms, tot_units = total_ms, units
    if ws > 1:
        max_ms, tot_units, e2e_sum = aggregate_ranks(dist, torch, "cuda", total_ms, units,
                                                     None if e2e is None else e2e["value"])
        if e2e is not None:
            e2e["value"] = e2e_sum

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = wl.cpu(args.cpu_seconds)

    # the learned-proposal study (2D U(1) 64x64, beta 2..8), summarised
    learned = None
    if rank == 0 and wl.name == "o3" and not args.no_learned:
        study = learned_study(umc, torch, meas=2000)
        learned = {"workload": "2D U(1) 64x64, 444 chains, U1Shift 0.5 vs learned 4-component von Mises mixture "
                               "(MLP 3-64-64-16, BF16 tcgen05), 20000 training configurations per beta",
                   "unit": "effective samples/s",
                   "per_beta": {b: {"learned_batched_over_plain_single": {o: row[o]["learned_batched_over_plain_single"]
                                                                          for o in ("plaquette", "Q")},
                                    "learned_over_plain_at_equal_batch": {o: row[o]["learned_over_plain_at_equal_batch"]
                                                                          for o in ("plaquette", "Q")},
                                    "effective_samples_per_s": {o: row[o]["effective_samples_per_s"]
                                                                for o in ("plaquette", "Q")},
                                    "tau_int": {o: row[o]["tau_int"] for o in ("plaquette", "Q")},
                                    "tau_converged": {o: row[o]["tau_converged"] for o in ("plaquette", "Q")},
                                    "z_vs_exact_plaquette": row["z_vs_exact"],
                                    "z_vs_sector_matched_plaquette": row["z_vs_sector_exact"],
                                    "acceptance": row["acceptance"]}
                                for b, row in study.items()}}

    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    value = tot_units / (max_ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": wl.unit, "n_gpus": ws, "steps": K,
        "warmup": args.warmup, "ms_per_step": max_ms / K, "higher_is_better": True,
        "scaling": getattr(wl, "scaling", "weak"),
        "vs_baseline": None, "dtype": wl.dtype, "data": "synthetic",
        "config": {"workload": wl.describe(), "L": wl.L, "parallelism": getattr(wl, "parallelism", None) or (f"replicas x{ws}" if ws > 1 else "1 chain"),
                   "l2": ("flushed between timed steps (256 MiB write, outside the timed events)" if wl.flush
                          else "state larger than L2, no flush"),
                   "mean_cluster": float(sizes.mean()) if len(sizes) and wl.name in ("o3", "userwolff") else None,
                   "thermalisation": (None if therm_cluster is None else
                                      f"{THERM_STEPS} untimed steps from the random start (mean cluster of the "
                                      f"last 200: {therm_cluster:.1f})")},
        "roofline": {"bound": roof["bound"], "achieved": achieved, "peak": peak, "unit": roof["unit"],
                     "frac": achieved / peak, "traffic": traffic, "kernel": kind, "avg_launch_us": avg_s * 1e6,
                     "peak_source": roof["peak_source"]},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "kernel_launches": {k: v[0] for k, v in launches.items() if v[0]},
        "kernel_ms": {k: round(v[1], 4) for k, v in per_kind.items() if v[0]},
        "clocks": clocks,
    }
    if learned is not None:
        line["learned_u1"] = learned
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
