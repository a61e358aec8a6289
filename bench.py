#!/usr/bin/env python
"""Benchmark of the single-GPU Barnes-Hut solve: Mparticles/s of one full build + upsweep + traversal.

Workload (default): N = 2^26 bodies i.i.d. uniform in [-1, 1]^3, masses 1/N, theta = 0.5, cartesian quadrupoles,
leaf bucket 64, 64-body target groups, fixed box [-1, 1]^3, FP32 with the FP64 steps of the design. The reference
P2P is singular for a body with itself at zero softening, so every body gets h = 1e-6 (the reference's own overflow
test does the same), far below the mean spacing 2.5e-3.

One "step" is one complete solve from unsorted, device-resident coordinates: SFC keys, radix sort, gathers, leaf
array, octree links, upsweep, target groups, traversal. Inputs (>> L2) are restored from a pristine copy before each
step, outside the timed interval of that step; each step is timed with CUDA events on the launching stream.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank solves its own system (replicas, weak scaling; a single system is not sharded).
`--impl reference` times the reference's own CPU implementation of the path (oracle/_ref, compiled from the
reference sources) on the host cores for a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

REFERENCE_PUBLISHED_MPS = 62.2  # reference, 1x A100, theta 0.5, 67 M particles (README.md:60)
P2P_FLOPS, M2P_FLOPS = 23, 65  # the reference's flop convention (ryoanji/test/demo.cu:108)
TRAV_DRAM_BYTES_2E24 = 1.289e9  # one traversal launch, uniform cube N=2^24, ncu dram bytes read + write
# bytes per body the build phases (keys, sort, permutation, leaves, upsweep) read and write in HBM
BUILD_BYTES_PER_BODY = {
    "keys": 12 + 8,                    # x, y, z in, key out
    "digit_histogram": 8,              # keys in
    "sort_passes": 8 * (12 + 12),      # 8 digit passes of (key, index) in and out
    "pack_records": 20 + 32,           # x, y, z, m, h in, 32-byte record out
    "gather_records": 4 + 32 + 20 + 32,  # index, record in; x, y, z, m, h and packed sources/targets out
    "leaves": 8,                       # sorted keys in
    "upsweep": 16 + 2,                 # packed bodies in; 64-byte node records out, about one node per 28 bodies
}
METRIC = "BH solve throughput (build + upsweep + traversal), theta 0.5, 1st-pct acc err vs FP64 direct"


def workload_config(args, world):
    return {"workload": f"uniform cube N=2^{args.log2n} in [-1,1]^3, masses 1/N, h=1e-6, theta={args.theta}, "
                        "cartesian quadrupole, bucket 64, groups 64, one full solve per step",
            "parallelism": "replicas" if world > 1 else "single GPU",
            "l2": "inputs of 256 MiB per array (> 126 MB L2) restored before every step",
            "vs_baseline_note": "published 62.2 Mparticles/s: reference on 1x A100, README.md:60"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--log2n", type=int, default=26)
    ap.add_argument("--theta", type=float, default=0.5)
    ap.add_argument("--accuracy-targets", type=int, default=16384)
    ap.add_argument("--cpu-log2n", type=int, default=22, help="CPU baseline sample size")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    ap.add_argument("--ensemble-systems", type=int, default=1024)
    ap.add_argument("--no-served", action="store_true", help="skip the served-stream leg")
    ap.add_argument("--no-plummer", action="store_true", help="skip the 2^24 Plummer sphere leg")
    ap.add_argument("--served-requests", type=int, default=48)
    ap.add_argument("--served-rate", type=float, default=24.0, help="Poisson arrival rate, requests per second")
    ap.add_argument("--served-repeats", type=int, default=3,
                    help="runs of each served-stream arm (alternating); the median-makespan run is reported")
    ap.add_argument("--served-max-step-bodies", type=int, default=None,
                    help="engine step cap in bodies (default: the library's; 0: every resident request each step)")
    ap.add_argument("--no-accuracy-matched", action="store_true")
    ap.add_argument("--no-precision", action="store_true", help="skip the precision-study leg (halos, periodic box)")
    ap.add_argument("--precision", action="store_true",
                    help="run the precision study (clustered halos and periodic box at theta 0.3/0.5/0.7) instead")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------------------ clocks

class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled while the timed region runs: NVML read queries every
    100 ms from a thread, or, where NVML is missing, an nvidia-smi subprocess at 200 ms. Nothing is set."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    # NVML clock-event reason bits of NAMES
    BITS = (0x8, 0x40, 0x20, 0x4)

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.source = None
        self.samples: list[tuple[float, float, set]] = []  # (sm MHz, max sm MHz, active reasons)
        self.lines: list[str] = []
        self._stop = threading.Event()
        self.thread = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            handle = pynvml.nvmlDeviceGetHandleByUUID(self.gpu_id)
            self.source = "nvml"
            self.thread = threading.Thread(target=self._poll_nvml, args=(pynvml, handle), daemon=True)
            self.thread.start()
            return self
        except Exception:  # no NVML binding or library: fall back to nvidia-smi
            self.source = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _poll_nvml(self, pynvml, handle):
        events = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        try:
            mx = float(pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM))
            while not self._stop.is_set():
                sm = float(pynvml.nvmlDeviceGetClockInfo(handle, pynvml.NVML_CLOCK_SM))
                bits = int(events(handle))
                self.samples.append((sm, mx, {n for n, b in zip(self.NAMES, self.BITS) if bits & b}))
                self._stop.wait(0.1)
        except Exception:
            pass
        finally:
            try:
                pynvml.nvmlShutdown()
            except Exception:
                pass

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        self._stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self) -> dict:
        samples = list(self.samples)
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm, mx = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            samples.append((sm, mx, {n for n, v in zip(self.NAMES, parts[4:8]) if v.lower().startswith("active")}))
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": self.source}
        reasons = set().union(*(r for _, _, r in samples))
        return {"sm_mhz": float(np.median([s for s, _, _ in samples])),
                "sm_max_mhz": float(max(m for _, m, _ in samples)), "reasons": sorted(reasons),
                "samples": len(samples), "source": self.source}


# ------------------------------------------------------------------------------------------------------ arms

def cpu_reference_solve(log2n: int, theta: float, seed: int = 0, library: str | None = None):
    """one solve of the reference's CPU path (oracle/_ref; @p library picks one of its builds) or, where it could not
    be built, the restated oracle; returns (kind, seconds, phase seconds)"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle, have_reference
    from ryoanji_b200 import datasets as ds
    kind = "reference" if have_reference() else "port"
    orc = Oracle(reference=(kind == "reference"), library=library)
    p = ds.uniform_cube(1 << log2n, seed=seed)
    t0 = time.perf_counter()
    u, *_ , sec = orc.solve(p.x, p.y, p.z, p.m, p.h, [-1, 1, -1, 1, -1, 1], bucket=64, theta=theta, G=1.0)
    dt = time.perf_counter() - t0
    return kind, dt, sec


def fastest_cpu_build(theta: float, log2n: int = 20):
    """the fastest build of the reference's CPU path on this host (one untimed solve of 2^log2n bodies each): the
    -O3 -fopenmp builds for the host's vector ISAs and the parity build. Returns (library, description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import have_reference, timing_builds, cpu_model
    if not have_reference():
        return None, f"restated oracle, g++ -O3 -fopenmp; {cpu_model()}"
    best = None
    for path, flags in timing_builds():
        _, dt, _ = cpu_reference_solve(log2n, theta, seed=1, library=path)
        if best is None or dt < best[0]:
            best = (dt, path, flags)
    return best[1], f"{best[2]} (fastest of {len(timing_builds())} builds on this host); {cpu_model()}"


def run_reference_arm(args, rank):
    if rank != 0:
        return
    library, build = fastest_cpu_build(args.theta, min(20, args.cpu_log2n))
    for _ in range(args.warmup):
        cpu_reference_solve(args.cpu_log2n, args.theta, seed=1, library=library)
    times = []
    kind = "port"
    for i in range(args.steps):
        kind, dt, _ = cpu_reference_solve(args.cpu_log2n, args.theta, seed=2 + i, library=library)
        times.append(dt)
    n = 1 << args.cpu_log2n
    value = n * len(times) / sum(times) / 1e6
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "Mparticles/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, args.gpus),
        "cpu_baseline": {"value": value, "unit": "Mparticles/s", "cores": cores, "kind": kind, "build": build,
                         "sample": f"each step: one full CPU solve (keys, sort, computeOctree, links, upsweep, "
                                   f"computeGravity) of N=2^{args.cpu_log2n} bodies of the same uniform-cube "
                                   f"distribution, OpenMP on {cores} threads"},
        "e2e": {"value": value, "unit": "Mparticles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    gpu = reference_gpu_plain(args)
    if gpu is not None:
        line["reference_gpu"] = gpu
    print(json.dumps(line), flush=True)


def reference_gpu_plain(args) -> dict | None:
    """the reference's own plain GPU path on this box's GPU (oracle/_ref/libryo_ref_gpu.so, compiled from the
    reference sources for sm_100a): TreeBuilder, the demo's upsweep, computeFixedGroups(64) and traverse
    (ryoanji/test/demo.cu:82-104, :171-190), on the uniform cube at 2^24 and 2^26 with h = 1e-6; device time per solve
    with CUDA events, inputs restored before every solve. None when no GPU or no such library is present."""
    import ctypes as C
    path = os.path.join(ROOT, "oracle", "_ref", "libryo_ref_gpu.so")
    try:
        import torch
        if not (os.path.exists(path) and torch.cuda.is_available()):
            return None
    except ImportError:
        return None
    lib = C.CDLL(path)
    lib.ref_gpu_solve_f32.restype = C.c_double
    lib.ref_gpu_solve_f32.argtypes = ([C.c_uint, C.c_float] + [C.c_void_p] * 5 + [C.c_size_t, C.c_void_p, C.c_float]
                                      + [C.c_void_p] * 6)
    dev = torch.device("cuda", 0)
    box = np.array([-1, 1, -1, 1, -1, 1], np.float32)
    out = {"workload": f"uniform cube in [-1,1]^3, masses 1/N, h=1e-6, theta={args.theta}, bucket 64, groups 64; "
                       "one build + upsweep + traverse per solve, on the GPU of this box"}
    for log2n in (24, 26):
        n = 1 << log2n
        gen = torch.Generator(device=dev)
        gen.manual_seed(1234)
        pristine = [torch.rand(n, device=dev, generator=gen) * 2 - 1 for _ in range(3)]
        m, h = torch.full((n,), 1.0 / n, device=dev), torch.full((n,), 1e-6, device=dev)
        work = [t.clone() for t in pristine]
        acc = [torch.zeros(n, device=dev) for _ in range(4)]
        stats = (C.c_uint64 * 5)()
        ms3 = (C.c_float * 3)()
        ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        times, parts = [], []
        for i in range(args.warmup + max(2, min(args.steps, 4))):
            for w, p in zip(work, pristine):
                w.copy_(p)
            for a in acc:
                a.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            lib.ref_gpu_solve_f32(64, C.c_float(args.theta), *[ptr(t) for t in work], ptr(m), ptr(h), n,
                                  box.ctypes.data_as(C.c_void_p), C.c_float(1.0), *[ptr(a) for a in acc], stats, ms3)
            e1.record()
            e1.synchronize()
            if i >= args.warmup:
                times.append(e0.elapsed_time(e1))
                parts.append(list(ms3))
        ms = float(np.mean(times))
        out[f"2^{log2n}"] = {"ms_per_solve": ms, "mparticles_per_s": n / (ms * 1e-3) / 1e6,
                             "phase_ms": dict(zip(("build", "upsweep", "groups_traverse"),
                                                  np.mean(parts, axis=0).round(3).tolist())),
                             "p2p_per_body": stats[0] / n, "m2p_per_body": stats[2] / n}
        del pristine, work, acc, m, h
        torch.cuda.empty_cache()
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import ryoanji_b200 as ryo

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = 1 << args.log2n
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    pristine = [torch.rand(n, device=dev, generator=gen) * 2 - 1 for _ in range(3)]
    pristine += [torch.full((n,), 1.0 / n, device=dev), torch.full((n,), 1e-6, device=dev)]
    work = [t.clone() for t in pristine]
    out = [torch.empty(n, device=dev) for _ in range(4)]
    ctx = ryo.Context(local_rank)
    params = ryo.SolveParams(theta=args.theta, bucket_size=64, group_size=64, box=ryo.Box.cube(-1.0, 1.0),
                             timing=True)
    peaks = ryo.measure_peaks(ctx)

    def restore():
        for w, p in zip(work, pristine):
            w.copy_(p)

    def solve():
        return ryo.solve(*work, *out, params=params, ctx=ctx)

    for _ in range(args.warmup):
        restore()
        solve()
    barrier()
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    launches0 = ryo.kernel_launches()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    results = []
    with ClockSampler(uuid) as clocks:
        barrier()
        for i in range(args.steps):
            restore()
            ev[i][0].record()
            results.append(solve())
            ev[i][1].record()
        barrier()
    launches = ryo.kernel_launches() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(sum(step_ms))
    value = world * n * args.steps / (total_ms * 1e-3) / 1e6
    res = results[-1]
    flops = P2P_FLOPS * res.sum_p2p + M2P_FLOPS * res.sum_m2p
    trav_ms = float(np.mean([r.ms["traverse"] for r in results]))
    achieved = flops / (trav_ms * 1e-3) / 1e12
    phase = {k: float(np.mean([r.ms[k] for r in results])) for k in ("sort", "tree", "upsweep", "traverse",
                                                                      "total")}

    line = {
        "metric": METRIC,
        "value": value, "unit": "Mparticles/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / world / REFERENCE_PUBLISHED_MPS, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, world),
        "phase_ms": phase,
        "interactions": {"p2p_per_body": res.sum_p2p / n, "m2p_per_body": res.sum_m2p / n, "max_p2p": res.max_p2p,
                         "max_m2p": res.max_m2p, "leaves": res.num_leaves, "nodes": res.num_nodes,
                         "retries": res.retries, "counted_tflops_traversal": achieved},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peaks["fp32_tflops"], "unit": "TFLOP/s",
                     "frac": achieved / peaks["fp32_tflops"],
                     "traffic": TRAV_DRAM_BYTES_2E24 * n / (1 << 24),
                     "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum of one traverseKernel launch "
                                     "captured with ncu on the same uniform cube at N=2^24 (1.027 GB + 0.262 GB), "
                                     "scaled by N/2^24; bytes per body are constant at fixed interactions per body",
                     "kernel": "traverseKernel (M2P + P2P), 23 flops per P2P and 65 per M2P per target",
                     "peak_source": "measured FP32 FMA peak of this GPU in this run (ryo_measure_peaks)",
                     "peak_fp32x2": peaks["fp32x2_tflops"]},
        "build_hbm": {"bytes_per_body": sum(BUILD_BYTES_PER_BODY.values()),
                      "gbs": sum(BUILD_BYTES_PER_BODY.values()) * n
                      / ((phase["sort"] + phase["tree"] + phase["upsweep"]) * 1e-3) / 1e9,
                      "peak_gbs": _measured_hbm(peaks),
                      "bytes_note": ", ".join(f"{k} {v}" for k, v in BUILD_BYTES_PER_BODY.items())},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }

    # accuracy against the FP64 direct sum on random targets of the last solve (sorted order)
    if args.accuracy_targets > 0:
        rng = np.random.default_rng(7)
        tgt = torch.from_numpy(rng.choice(n, args.accuracy_targets, replace=False)).to(dev)
        rp, rx, ry, rz = ryo.direct_targets_f64(tgt, *work)
        a = torch.stack([out[1][tgt], out[2][tgt], out[3][tgt]], 1).double()
        r = torch.stack([rx, ry, rz], 1)
        err = (torch.linalg.norm(a - r, dim=1) / torch.linalg.norm(r, dim=1)).cpu().numpy()
        pt, pd = float(out[0][tgt].double().sum()), float(rp.sum())
        line["accuracy"] = {"targets": args.accuracy_targets, "err_p99_1st_pct": float(np.percentile(err, 99)),
                            "err_max": float(err.max()), "err_median": float(np.median(err)),
                            "potential_sample_rel_diff": abs(pt - pd) / abs(pd),
                            "potential_energy_tree": res.potential_energy}

    # end to end through the public host-memory call (ryo_solve_host_f32): x, y, z, m, h from pinned host memory;
    # potential, acceleration and the permutation that maps them back to the input order into pinned host memory.
    # The call overlaps its copies with the solve and returns when every output is on the host.
    if not args.no_e2e:
        host_in = [t.cpu().pin_memory() for t in pristine]
        host_out = [torch.empty(n).pin_memory() for _ in range(4)]
        host_order = torch.empty(n, dtype=torch.int32).pin_memory()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def solve_host():
            return ryo.solve_host(*host_in, *host_out, params=params, order=host_order, ctx=ctx)

        for _ in range(2):
            solve_host()
        barrier()
        e0.record()
        for _ in range(args.steps):
            solve_host()
        e1.record()
        barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1))
        line["e2e"] = {"value": world * n * args.steps / (e2e_ms * 1e-3) / 1e6, "unit": "Mparticles/s",
                       "h2d_bytes_per_step": 5 * 4 * n, "d2h_bytes_per_step": 5 * 4 * n}

    if world == 1 and not args.no_accuracy_matched and args.accuracy_targets > 0:
        line["accuracy_matched"] = run_accuracy_matched(args, ctx, dev, work, out, pristine, n)
    if not args.no_ensemble:
        line["ensemble"] = run_ensemble(args, ctx, dev, rank, world, max_over_ranks)
    if not args.no_served:
        line["served"] = run_served(args, ctx, dev, rank, world, dist)
    if world == 1 and not args.no_plummer:
        line["plummer_2e24"] = run_plummer(args, ctx, dev)
    if world == 1 and not args.no_precision:
        line["precision"] = run_precision(args, ctx, dev)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        library, build = fastest_cpu_build(args.theta, min(20, args.cpu_log2n))
        kind, dt, sec = cpu_reference_solve(args.cpu_log2n, args.theta, seed=3, library=library)
        line["cpu_baseline"] = {"value": (1 << args.cpu_log2n) / dt / 1e6, "unit": "Mparticles/s",
                                "cores": os.cpu_count(), "kind": kind, "build": build,
                                "sample": f"one solve of N=2^{args.cpu_log2n} uniform cube (bounded sample), "
                                          f"OpenMP on {os.cpu_count()} threads; build/upsweep/gravity s = "
                                          f"{[round(float(s), 3) for s in sec]}"}
    if "accuracy" in line:
        acc = line["accuracy"]
        line["config"]["workload"] += (f"; measured 1st-pct acc err {acc['err_p99_1st_pct']:.2e} (max "
                                       f"{acc['err_max']:.2e}) vs FP64 direct on {acc['targets']} targets")
    # the compact summary goes last: it lands in the tail of the output that the driver keeps
    line["summary"] = summarize(line)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _r(v, digits=4):
    """round a float to a few significant digits for the summary"""
    if isinstance(v, float):
        return float(f"{v:.{digits}g}")
    if isinstance(v, dict):
        return {k: _r(x, digits) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [_r(x, digits) for x in v]
    return v


def summarize(line: dict) -> dict:
    """the figures of every leg in a few hundred characters, rounded"""
    s = {"mps": line["value"], "e2e_mps": line.get("e2e", {}).get("value"),
         "trav_frac_fp32": line["roofline"]["frac"], "build_hbm_frac": line["build_hbm"]["gbs"]
         / line["build_hbm"]["peak_gbs"] if line["build_hbm"].get("peak_gbs") else None,
         "phase_ms": line["phase_ms"],
         "per_body": [line["interactions"]["p2p_per_body"], line["interactions"]["m2p_per_body"]]}
    if "accuracy" in line:
        a = line["accuracy"]
        s["acc_theta_0.5"] = {"p99": a["err_p99_1st_pct"], "max": a["err_max"]}
    if "accuracy_matched" in line:
        a = line["accuracy_matched"]
        s["acc_matched"] = {"theta": a.get("theta"), "mps": a.get("value"), "p99": a.get("err_p99_1st_pct")}
    if "ensemble" in line:
        e = line["ensemble"]
        s["ensemble"] = {"batched_sps": e.get("batched", {}).get("solves_per_s"),
                         "plain_sps": e.get("plain_loop", {}).get("solves_per_s"), "x": e.get("speedup_solves_per_s")}
    if "served" in line:
        v = line["served"]
        s["served"] = {"x": v.get("speedup_solves_per_s"),
                       **{f"{arm}_{k}": v.get(arm, {}).get(k) for arm in ("served", "plain")
                          for k in ("solves_per_s", "latency_p50_s", "latency_p99_s")}}
    if "plummer_2e24" in line:
        p = line["plummer_2e24"]["fixed_groups"]
        s["plummer_2e24"] = {"mps": p["mparticles_per_s"], "p99": p["err_p99_1st_pct"], "max": p["err_max"]}
    if "precision" in line:
        s["precision"] = line["precision"].get("summary")
    return _r(s)


# ------------------------------------------------------------------------------------------------------ legs

def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_ensemble(args, ctx, dev, rank=0, world=1, max_over_ranks=lambda v: v) -> dict:
    """batched ensemble: independent Plummer systems (N = round(2^U[10, 18]), a ~ U[0.5, 2], eps = 0.01 a) solved in
    one launch per phase with autotuned bucket/group/stack, against a loop of the single-system solve. With several
    ranks each solves its LPT share of the systems; times are the maximum over ranks."""
    import torch
    import ryoanji_b200 as ryo
    from ryoanji_b200 import autotune
    from ryoanji_b200 import datasets as ds
    from ryoanji_b200.shard import lpt_partition, solve_cost
    all_sizes, all_radii = ds.ensemble_sizes(args.ensemble_systems, seed=5)
    total_systems, total_bodies = len(all_sizes), int(all_sizes.sum())
    all_bodies = ds.plummer_ensemble(all_sizes, all_radii, seed=5, device=dev)
    mine = lpt_partition([solve_cost(int(k)) for k in all_sizes], world)[rank]
    offs_all = np.concatenate([[0], np.cumsum(all_sizes)])
    idx = torch.cat([torch.arange(int(offs_all[i]), int(offs_all[i + 1]), device=dev) for i in mine])
    bodies = [b[idx].contiguous() for b in all_bodies]
    del all_bodies
    sizes = all_sizes[mine]
    n = int(sizes.sum())
    systems = [ryo.BatchSystem(int(k)) for k in sizes]
    base = ryo.SolveParams(theta=0.5)
    tuned, table = autotune.tune_batch(systems, bodies, base, ctx=ctx)
    work = [b.clone() for b in bodies[:5]]
    out = [torch.empty(n, device=dev) for _ in range(4)]

    def restore():
        for w, b in zip(work, bodies):
            w.copy_(b)

    steps = max(2, min(args.steps, 5))
    for _ in range(2):
        restore()
        ryo.solve_batch(systems, *work, *out, params=tuned, ctx=ctx)
    ms = 0.0
    for _ in range(steps):
        restore()
        e0, e1 = _events()
        e0.record()
        ryo.solve_batch(systems, *work, *out, params=tuned, ctx=ctx)
        e1.record()
        e1.synchronize()
        ms += e0.elapsed_time(e1)
    batched_ms = max_over_ranks(ms / steps)

    # the plain path: one single-system solve per system, same parameters
    offs = np.concatenate([[0], np.cumsum(sizes)])

    def plain_loop():
        for k in range(len(sizes)):
            sl = slice(int(offs[k]), int(offs[k + 1]))
            ryo.solve(*[w[sl] for w in work], *[o[sl] for o in out], params=tuned, ctx=ctx)

    restore()
    plain_loop()
    restore()
    e0, e1 = _events()
    e0.record()
    plain_loop()
    e1.record()
    e1.synchronize()
    plain_ms = max_over_ranks(e0.elapsed_time(e1))
    ns, n = total_systems, total_bodies
    return {"workload": f"{ns} Plummer systems, N=round(2^U[10,18]) ({n} bodies), a~U[0.5,2], eps=0.01a, theta 0.5, "
                        "quadrupole; one solve of every system per step"
                        + (f"; LPT shares over {world} GPUs, times = max over ranks" if world > 1 else ""),
            "autotuned": {"bucket": tuned.bucket_size, "group": tuned.group_size, "stack": tuned.stack_capacity,
                          "group_tolerance": tuned.group_tolerance,
                          "best_candidates_ms (bucket, group, stack, group tolerance, ms)":
                              [list(t) for t in sorted(table, key=lambda t: t[-1])[:3]], "candidates": len(table)},
            "batched": {"ms_per_step": batched_ms, "solves_per_s": ns / (batched_ms * 1e-3),
                        "mparticles_per_s": n / (batched_ms * 1e-3) / 1e6, "steps": steps},
            "plain_loop": {"ms_per_step": plain_ms, "solves_per_s": ns / (plain_ms * 1e-3),
                           "mparticles_per_s": n / (plain_ms * 1e-3) / 1e6},
            "speedup_solves_per_s": plain_ms / batched_ms}


def run_plummer(args, ctx, dev, log2n: int = 24) -> dict:
    """the plain path's second workload: one Plummer sphere of 2^24 equal masses (a = 1, total mass 1, eps = 0.01,
    radii resampled above 50 a, seeded), theta 0.5, quadrupole, bucket 64, one full solve per step with the inputs
    restored before each. Fixed groups of 64 (the reference demo's) and spatial groups (tolFactor 2); relative
    acceleration error against FP64 direct sums on 16,384 random targets."""
    import torch
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    n = 1 << log2n
    gen = torch.Generator(device=dev)
    gen.manual_seed(24)
    x, y, z, _, _, _ = ds.plummer_device(torch.ones(n, dtype=torch.float64, device=dev), gen, velocities=False)
    pristine = [t.float().contiguous() for t in (x, y, z)]
    pristine += [torch.full((n,), 1.0 / n, device=dev), torch.full((n,), 0.005, device=dev)]
    del x, y, z
    work = [t.clone() for t in pristine]
    out = [torch.empty(n, device=dev) for _ in range(4)]
    order = torch.empty(n, dtype=torch.int32, device=dev)
    rng = np.random.default_rng(3)
    tgt = torch.from_numpy(rng.choice(n, 16384, replace=False)).to(dev)
    _, rx, ry, rz = ryo.direct_targets_f64(tgt, *pristine)
    ref = torch.stack([rx, ry, rz], 1)
    res = {"workload": f"Plummer sphere N=2^{log2n}, a=1, M=1, eps=0.01 (h=0.005), rmax=50a, theta 0.5, quadrupole, "
                       "bucket 64, groups of 64; one full solve per step"}
    for label, tol in (("fixed_groups", 0.0), ("spatial_groups", 2.0)):
        params = ryo.SolveParams(theta=0.5, bucket_size=64, group_size=64, group_tolerance=tol, timing=True)
        times = []
        for i in range(6):
            for w, p in zip(work, pristine):
                w.copy_(p)
            e0, e1 = _events()
            e0.record()
            r = ryo.solve(*work, *out, params=params, order=order, ctx=ctx)
            e1.record()
            e1.synchronize()
            if i >= 3:
                times.append(e0.elapsed_time(e1))
        ms = sum(times) / len(times)
        inv = torch.empty_like(order)
        inv[order.long()] = torch.arange(n, dtype=torch.int32, device=dev)
        acc = torch.stack([a[inv[tgt].long()] for a in out[1:]], 1).double()
        err = (torch.linalg.norm(acc - ref, dim=1) / torch.linalg.norm(ref, dim=1)).cpu().numpy()
        res[label] = {"ms_per_step": ms, "mparticles_per_s": n / (ms * 1e-3) / 1e6, "groups": r.num_groups,
                      "phase_ms": {k: round(v, 3) for k, v in r.ms.items()},
                      "p2p_per_body": r.sum_p2p / n, "m2p_per_body": r.sum_m2p / n, "max_p2p": r.max_p2p,
                      "err_p99_1st_pct": float(np.percentile(err, 99)), "err_max": float(err.max()),
                      "err_median": float(np.median(err))}
    return res


def run_served(args, ctx, dev, rank=0, world=1, dist=None) -> dict:
    """served stream: open-loop Poisson arrivals of solve requests (N = round(2^U[12, 22]); 45% Plummer, 45% cube,
    10% periodic with Ewald; K ~ U{1..64} leapfrog steps, dt = 1e-3) through the engine, against the plain path
    taking the same requests one at a time in arrival order. Inputs come from pinned host memory and every request's
    final state goes back to the host in both arms."""
    import torch
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    from ryoanji_b200.shard import route_requests
    all_reqs = ds.served_requests(args.served_requests, seed=11, rate_per_s=args.served_rate)
    route = route_requests(all_reqs, world)
    reqs = [q for q, r in zip(all_reqs, route) if r == rank]
    host, result = {}, {}
    for q in reqs:
        host[q["tag"]] = [t.cpu().pin_memory() for t in ds.request_bodies(q, device=dev)]
        # the final state (x y z vx vy vz ax ay az p) of every request lands in pinned host memory in both arms
        result[q["tag"]] = torch.empty((10, q["n"]), dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()
    # both arms split each 64-body window spatially (tolFactor 2, the reference's production grouping): sparse
    # Plummer outskirts otherwise make wide groups
    params = ryo.SolveParams(theta=0.5, group_tolerance=2.0)
    periodic = ryo.Box(0.0, 1.0, 0.0, 1.0, 0.0, 1.0, boundary=(ryo.BOUNDARY_PERIODIC,) * 3)
    arrival = {q["tag"]: q["arrival"] for q in all_reqs}
    solves = sum(q["steps"] + 1 for q in all_reqs)
    body_solves = sum(q["n"] * (q["steps"] + 1) for q in all_reqs)

    def gather(done):
        # latencies of every rank's requests; the makespan is the latest completion on any rank
        if dist is None:
            return done
        parts = [None] * world
        dist.all_gather_object(parts, done)
        merged = {}
        for p in parts:
            merged.update(p)
        return merged

    def summary(done, t_end):
        done = gather(done)
        t_end = max(done.values())
        lat = np.array([done[k] - arrival[k] for k in arrival])
        return {"makespan_s": t_end, "solves_per_s": solves / t_end, "mparticles_per_s": body_solves / t_end / 1e6,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "latency_max_s": float(lat.max())}

    def serve_once():
        # served: the engine admits what has arrived at every step. Its two arenas are reserved at creation for 2^25
        # resident bodies (the stream peaks near 2.5e7), as a server sizes them at start-up.
        # the engine's solves record their phase times (CUDA events), to show where a step's device time goes
        eng = ryo.Engine(dataclasses.replace(params, timing=True), hbm_budget_bytes=120e9, ctx=ctx,
                         reserve_bodies=1 << 25, max_step_bodies=args.served_max_step_bodies)
        phase = np.zeros(6)
        outs = {}
        done = {}
        i = 0
        steps = 0
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        while len(done) < len(reqs):
            now = time.perf_counter() - t0
            while i < len(reqs) and reqs[i]["arrival"] <= now:
                q = reqs[i]
                x, y, z, m, h, vx, vy, vz = host[q["tag"]]
                eng.submit(q["tag"], x, y, z, m, h, vx, vy, vz, box=periodic if q["kind"] == "periodic" else None,
                           steps=q["steps"], dt=q["dt"], want_output=True, out=result[q["tag"]])
                i += 1
            st = eng.status()
            if st["queued"] == 0 and st["resident"] == 0:
                time.sleep(max(0.0, reqs[i]["arrival"] - (time.perf_counter() - t0)))
                continue
            info = eng.step()
            phase += np.array(info["ms"][:6])
            steps += 1
            for d in eng.poll():
                done[d["tag"]] = time.perf_counter() - t0
                outs[d["tag"]] = d
        served = summary(done, max(done.values(), default=0.0))
        served["engine_steps"] = steps
        # device time of the engine's batched solves by phase, summed over the steps: keys + sort + gather, leaves +
        # links, upsweep, groups + traversal, Ewald; share of the solves' total
        names = ("sort", "tree", "upsweep", "traverse", "ewald")
        served["solve_phase_ms"] = {k: round(float(v), 1) for k, v in zip(names + ("total",), phase)}
        served["solve_phase_share"] = {k: round(float(v / phase[5]), 4) if phase[5] > 0 else None
                                       for k, v in zip(names, phase)}
        served["max_step_bodies"] = ("library default" if args.served_max_step_bodies is None
                                     else args.served_max_step_bodies)
        drift = [abs(d["kinetic"] + d["potential"] - d["initial"]) / abs(d["initial"]) for d in outs.values()
                 if d["initial"] != 0]
        served["energy_drift_median"] = float(np.median(drift)) if drift else None
        eng.close()
        return served

    def plain_once():
        # plain: one request at a time, single-system solve and leapfrog on the device
        done = {}
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for q in reqs:
            wait = q["arrival"] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            x, y, z, m, h, vx, vy, vz = (t.to(dev, non_blocking=True) for t in host[q["tag"]])
            n = q["n"]
            p, ax, ay, az = (torch.empty(n, device=dev) for _ in range(4))
            pp = ryo.SolveParams(theta=0.5, box=periodic if q["kind"] == "periodic" else None, num_shells=1,
                                 group_tolerance=2.0)
            ryo.solve(x, y, z, m, h, p, ax, ay, az, params=pp, v=(vx, vy, vz), ctx=ctx)
            hdt, dt = 0.5 * q["dt"], q["dt"]
            for _ in range(q["steps"]):
                for v, a in ((vx, ax), (vy, ay), (vz, az)):
                    v.add_(a, alpha=hdt)
                for c, v in ((x, vx), (y, vy), (z, vz)):
                    c.add_(v, alpha=dt)
                    if q["kind"] == "periodic":
                        c.remainder_(1.0)
                ryo.solve(x, y, z, m, h, p, ax, ay, az, params=pp, v=(vx, vy, vz), ctx=ctx)
                for v, a in ((vx, ax), (vy, ay), (vz, az)):
                    v.add_(a, alpha=hdt)
            result[q["tag"]].copy_(torch.stack([x, y, z, vx, vy, vz, ax, ay, az, p]))
            done[q["tag"]] = time.perf_counter() - t0
        plain = summary(done, max(done.values(), default=0.0))
        return plain

    # the two arms alternate; each reports the run with its median makespan (arrival timing against step boundaries
    # makes single runs vary), and every run's makespan, p50 and p99 are listed
    runs_s, runs_p = [], []
    for _ in range(max(1, args.served_repeats)):
        runs_s.append(serve_once())
        runs_p.append(plain_once())
    pick = lambda runs: sorted(runs, key=lambda r: r["makespan_s"])[(len(runs) - 1) // 2]  # noqa: E731
    served, plain = pick(runs_s), pick(runs_p)
    brief = lambda runs: [[round(r["makespan_s"], 3), round(r["latency_p50_s"], 3),  # noqa: E731
                           round(r["latency_p99_s"], 3)] for r in runs]
    served["runs_makespan_p50_p99"] = brief(runs_s)
    plain["runs_makespan_p50_p99"] = brief(runs_p)
    return {"workload": f"{len(all_reqs)} requests, Poisson arrivals at {args.served_rate}/s, N=round(2^U[12,22]), "
                        "45% Plummer / 45% cube / 10% periodic+Ewald, K~U{1..64} KDK steps, dt=1e-3, theta 0.5, "
                        "spatial groups (tolFactor 2) in both arms, 120 GB admission budget"
                        + (f"; requests routed over {world} GPUs by estimated backlog" if world > 1 else ""),
            "solves": solves, "body_solves": body_solves, "served": served, "plain": plain,
            "speedup_solves_per_s": served["solves_per_s"] / plain["solves_per_s"],
            "h2d": "pinned host inputs copied per request",
            "d2h": "final state of every request copied back into pinned host memory"}


def run_accuracy_matched(args, ctx, dev, work, out, pristine, n) -> dict:
    """the lowest-cost theta (of a short list) whose 1st-percentile error meets 5e-4, timed like the main line"""
    import torch
    import ryoanji_b200 as ryo
    rng = np.random.default_rng(7)
    tgt = torch.from_numpy(rng.choice(n, 4096, replace=False)).to(dev)
    for theta in (0.45, 0.44, 0.43, 0.42, 0.41, 0.40, 0.38):
        params = ryo.SolveParams(theta=theta, bucket_size=64, group_size=64, box=ryo.Box.cube(-1.0, 1.0),
                                 timing=True)
        times = []
        for i in range(3):
            for w, p in zip(work, pristine):
                w.copy_(p)
            e0, e1 = _events()
            e0.record()
            ryo.solve(*work, *out, params=params, ctx=ctx)
            e1.record()
            e1.synchronize()
            if i:
                times.append(e0.elapsed_time(e1))
        rp, rx, ry, rz = ryo.direct_targets_f64(tgt, *work)
        a = torch.stack([out[1][tgt], out[2][tgt], out[3][tgt]], 1).double()
        r = torch.stack([rx, ry, rz], 1)
        err = (torch.linalg.norm(a - r, dim=1) / torch.linalg.norm(r, dim=1)).cpu().numpy()
        e99 = float(np.percentile(err, 99))
        if e99 <= 5e-4:
            ms = float(np.mean(times))
            return {"theta": theta, "targets": 4096, "err_p99_1st_pct": e99, "err_max": float(err.max()),
                    "ms_per_step": ms,
                    "value": n / (ms * 1e-3) / 1e6, "unit": "Mparticles/s",
                    "note": "theta lowered from 0.5 until the 1st-percentile error met 5e-4"}
    return {"theta": None, "note": "no theta in the list met 5e-4"}


def run_precision(args, ctx=None, dev=None) -> dict:
    """precision study: 64 Hernquist halos (N = 2^24) against FP64 direct sums on 16384 targets, and a periodic unit
    box (N = 2^22, Ewald defaults, one replica shell) against the FP64 particle-level Ewald sum on 1024 targets, at
    theta 0.3, 0.5 and 0.7; reports the 1st-percentile and maximum relative acceleration error and the relative error
    of the targets' summed potential. The net accelerations of a uniform periodic box are near zero, so its errors
    are also given normalised by the rms |a| of the reference (err_rms_norm_*)."""
    import torch
    import ryoanji_b200 as ryo
    from ryoanji_b200 import datasets as ds
    dev = dev or torch.device("cuda", 0)
    ctx = ctx or ryo.Context(0)
    out = {}

    def errors(ax, ay, az, pot, tgt, ref, periodic):
        rp, rx, ry, rz = ref
        a = torch.stack([ax[tgt], ay[tgt], az[tgt]], 1).double()
        r = torch.stack([rx, ry, rz], 1)
        err = (torch.linalg.norm(a - r, dim=1) / torch.linalg.norm(r, dim=1)).cpu().numpy()
        out = {"err_p99_1st_pct": float(np.percentile(err, 99)), "err_max": float(err.max()),
               "err_median": float(np.median(err))}
        if periodic:
            rms = float(torch.sqrt((r * r).sum(1).mean()))
            dn = (torch.linalg.norm(a - r, dim=1) / rms).cpu().numpy()
            out["err_rms_norm_p99"] = float(np.percentile(dn, 99))
            out["err_rms_norm_max"] = float(dn.max())
        pt = pot[tgt].double()
        if periodic:
            # periodic potentials are defined up to a constant, and the two Ewald forms place it differently
            # (the particle-level form includes every body's own image terms): compare after removing the mean
            off = float((pt - rp).mean())
            out["potential_offset_rel"] = off / float(rp.abs().mean())
            out["potential_rms_rel_after_offset"] = float(torch.sqrt(((pt - rp - off) ** 2).mean()) /
                                                          rp.abs().mean())
        else:
            out["potential_rel"] = abs(float(pt.sum()) - float(rp.sum())) / abs(float(rp.sum()))
        return out

    cases = [("hernquist_halos_2^24", ds.hernquist_halos(1 << 24, num_halos=64, seed=21), None, 16384),
             ("periodic_box_2^22", ds.periodic_box(1 << 22, seed=22), 1.0, 1024)]
    for name, p, L, nt in cases:
        base = [torch.from_numpy(a).to(dev) for a in (p.x, p.y, p.z, p.m, p.h)]
        n = p.n
        tgt_idx = None
        res = {}
        for theta in (0.3, 0.5, 0.7):
            work = [b.clone() for b in base]
            pot, ax, ay, az = (torch.empty(n, device=dev) for _ in range(4))
            box = ryo.Box(*p.box, boundary=(ryo.BOUNDARY_PERIODIC,) * 3) if L else None
            params = ryo.SolveParams(theta=theta, box=box, num_shells=1, timing=True)
            r = ryo.solve(*work, pot, ax, ay, az, params=params, ctx=ctx)
            if tgt_idx is None:
                # the sorted order is the same for every theta: pick targets and the FP64 reference once
                tgt_idx = torch.from_numpy(np.random.default_rng(5).choice(n, nt, replace=False)).to(dev)
                t0 = time.perf_counter()
                if L:
                    ref = ryo.ewald_targets_f64(tgt_idx, *work, L=L, ctx=ctx)
                else:
                    ref = ryo.direct_targets_f64(tgt_idx, *work)
                torch.cuda.synchronize()
                ref_s = time.perf_counter() - t0
            e = errors(ax, ay, az, pot, tgt_idx, ref, bool(L))
            e["solve_ms"] = r.ms["total"]
            e["p2p_per_body"] = r.sum_p2p / n
            e["m2p_per_body"] = r.sum_m2p / n
            res[f"theta_{theta}"] = e
        res["reference"] = ("FP64 particle-level Ewald sum (replica shells + every source's monopole correction)"
                            if L else "FP64 direct sum") + f" on {nt} targets, {ref_s:.1f} s"
        out[name] = res
    summ = {}
    for name, res in out.items():
        key = "err_rms_norm_p99" if "periodic" in name else "err_p99_1st_pct"
        summ[name.split("_")[0]] = {t.split("_")[1]: res[t][key] for t in res if t.startswith("theta_")}
    return {"precision_study": out, "dtype": "f32 bulk, FP64 upsweep/Ewald k-space/potential",
            "data": "synthetic, seeded",
            "summary": {"note": "hernquist: 1st-pct rel err; periodic: p99 err / rms|a|", **summ}}


def _measured_hbm(peaks):
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return peaks["copy_gbs"]


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.precision:
        if rank == 0:
            print(json.dumps(run_precision(args)), flush=True)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
