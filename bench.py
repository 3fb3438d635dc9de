#!/usr/bin/env python
"""Benchmark of the B200 certification hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload scene|plain] [--impl b200|reference]

A step is one pass of the hot path over one batch of seeded synthetic input:
  * scene (default): two 40,960-triangle UV spheres (FP64, rigid translation
    toward contact + per-vertex N(0, 1e-3) jitter) -> swept-AABB candidates ->
    exact VF/EE certificates of every candidate;
  * plain: 20,000 independent queries (10k VF + 10k EE).
metric: certified CCD queries/s (one query = one primitive certificate).

Timing: W untimed warm-up steps, then K steps each bracketed by CUDA events
on the launching stream, with a 512 MB L2 flush between steps (outside the
events); barrier + synchronize around the timed region; max over ranks.  The
e2e figure goes through the public API with the inputs copied from pinned
host memory and the results read back every step.  N > 1 runs N independent
replicas (weak scaling): the path has no exchange step.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (str(ROOT), str(ROOT / "p2c-ccd_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

L2_FLUSH_BYTES = 512 << 20


def _load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                mx = float(parts[2].split()[0])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------
# workloads


class PlainWorkload:
    """20,000 independent queries (10k vertex-face + 10k edge-edge)."""

    name = "plain"

    def __init__(self, device, rank: int):
        import torch

        from p2cccd_b200 import certify, workloads

        self.torch = torch
        self.certify = certify
        self.spec = workloads.PlainSpec(seed=workloads.DEFAULT_SEED + rank)
        w = workloads.plain_queries(self.spec)
        self.host = w
        self.cfg = certify.CertConfig(1e-6, 1e-6, 32)
        self.dev = device
        self.pt = certify.records_to_device(w["vf"], device)
        self.ee = certify.records_to_device(w["ee"], device)
        self.out_pt = torch.empty((len(w["vf"]), 72), dtype=torch.uint8, device=device)
        self.out_ee = torch.empty((len(w["ee"]), 72), dtype=torch.uint8, device=device)
        self.ws = certify.Workspace(device)
        # pinned host staging for the end-to-end path
        self.h_pt = torch.from_numpy(w["vf"].view("u1").reshape(-1, 240).copy()).pin_memory()
        self.h_ee = torch.from_numpy(w["ee"].view("u1").reshape(-1, 240).copy()).pin_memory()
        self.h_out_pt = torch.empty_like(self.out_pt, device="cpu").pin_memory()
        self.h_out_ee = torch.empty_like(self.out_ee, device="cpu").pin_memory()
        self.queries = len(w["vf"]) + len(w["ee"])
        self.launches_per_step = 1

    def config(self) -> dict:
        return {"workload": "plain exact CCD: 10,000 VF + 10,000 EE seeded FP64 queries (U[0,1]^3 endpoints, "
                            "N(0,0.05) displacement, 30% touching, 10% near-degenerate)",
                "queries_per_step": self.queries, "eps_time": self.cfg.eps_time, "eps_space": self.cfg.eps_space,
                "max_subdivision_depth": self.cfg.max_subdivision_depth, "seed": self.spec.seed}

    def step(self):
        self.certify.certify_batch2(self.pt, self.ee, 0.0, 1.0, self.cfg, self.out_pt, self.out_ee, self.ws)

    def step_e2e(self):
        self.pt.copy_(self.h_pt, non_blocking=True)
        self.ee.copy_(self.h_ee, non_blocking=True)
        self.step()
        self.h_out_pt.copy_(self.out_pt, non_blocking=True)
        self.h_out_ee.copy_(self.out_ee, non_blocking=True)

    def io_bytes(self) -> tuple[int, int]:
        return self.h_pt.numel() + self.h_ee.numel(), self.h_out_pt.numel() + self.h_out_ee.numel()

    def census(self) -> dict:
        return self.certify.census(self.pt, self.ee, 0.0, 1.0, self.cfg)["stats"]

    def cpu_reference(self, threads: int, budget_s: float) -> dict:
        """Reference C++ certifier (oracle/_ref, unchanged sources) on host cores."""
        import oracle

        done, t0 = 0, time.perf_counter()
        while True:
            for fam in ("vf", "ee"):
                oracle.ref_eval_batch(self.host[fam], 0.0, 1.0, self.cfg.eps_time, self.cfg.eps_space,
                                      self.cfg.max_subdivision_depth, threads=threads)
                done += len(self.host[fam])
            el = time.perf_counter() - t0
            if el >= budget_s:
                break
        return {"queries": done, "seconds": el,
                "sample": f"the full {self.queries}-query batch repeated {done // self.queries}x"}


WORKLOADS = {"plain": PlainWorkload}


# --------------------------------------------------------------------------


def _dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def _barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_steps(torch, fn, steps, flush, stream):
    times = []
    for _ in range(steps):
        flush.fill_(1)  # write > L2 between timed steps
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        e.synchronize()
        times.append(s.elapsed_time(e))
    return times


def run_b200(args) -> dict | None:
    import torch

    from p2cccd_b200 import certify

    world, rank, local = _dist_setup(args)
    dev = torch.device("cuda", local if world > 1 else 0)
    wl = WORKLOADS[args.workload](dev, rank)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        wl.step()
    torch.cuda.synchronize()
    _barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index if world > 1 else int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0))
    sampler.start()
    times = time_steps(torch, wl.step, args.steps, flush, stream)
    torch.cuda.synchronize()
    _barrier(world)
    clocks = sampler.stop()
    # e2e through the public API with pinned host buffers
    for _ in range(max(1, args.warmup)):
        wl.step_e2e()
    torch.cuda.synchronize()
    e2e_times = time_steps(torch, wl.step_e2e, args.steps, flush, stream)
    torch.cuda.synchronize()
    ms = statistics.mean(times)
    ms_max = _max_over_ranks(world, ms)
    e2e_ms = _max_over_ranks(world, statistics.mean(e2e_times))
    total_q = wl.queries * world
    value = total_q / (ms_max * 1e-3)
    e2e_value = total_q / (e2e_ms * 1e-3)
    census = wl.census()
    fp64_rate = certify.probe_fp64_rate(dev)
    kernel_ms = ms  # the step is one certification launch (plus a 112-byte scratch reset)
    achieved = census["fp64_ops"] / (kernel_ms * 1e-3)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = wl.cpu_reference(threads, args.cpu_budget)
        cpu = {"value": r["queries"] / r["seconds"], "unit": "queries/s", "cores": threads, "kind": "reference",
               "sample": r["sample"] + f" ({r['seconds']:.1f} s, {threads} threads over the reference's "
                                       "EvaluatePointTriangleInterval/EvaluateEdgeEdgeInterval)"}
    if rank != 0:
        return None
    h2d, d2h = wl.io_bytes()
    return {
        "metric": "certified CCD queries/s", "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "p50_ms": statistics.median(times), "p99_ms": sorted(times)[max(0, int(0.99 * len(times)) - 1)],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {**wl.config(), "l2": f"flushed between timed steps ({L2_FLUSH_BYTES >> 20} MB write)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": wl.launches_per_step * args.steps,
        "roofline": {"bound": "fp64", "achieved": achieved / 1e12, "peak": fp64_rate / 1e12, "unit": "TFLOP/s",
                     "frac": achieved / fp64_rate, "traffic": None,
                     "peak_source": "measured in-run: p2c_probe_fp64 (DMUL+DADD chains, no FMA)",
                     "kernel": "certify_records_kernel",
                     "algorithmic_fp64_ops_per_launch": census["fp64_ops"],
                     "nodes_per_launch": census["nodes_evaluated"]},
        "cpu_baseline": cpu,
        "clocks": clocks,
    }


def run_reference(args) -> dict | None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    import numpy as np  # noqa: F401

    import oracle
    from p2cccd_b200 import certify, workloads

    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libp2c_ref.so was not built"}
    threads = os.cpu_count() or 1
    if args.workload == "plain":
        spec = workloads.PlainSpec()
        w = workloads.plain_queries(spec)
        cfg = certify.CertConfig(1e-6, 1e-6, 32)
        nq = len(w["vf"]) + len(w["ee"])

        def step():
            for fam in ("vf", "ee"):
                oracle.ref_eval_batch(w[fam], 0.0, 1.0, cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth,
                                      threads=threads)
            return nq
        conf = {"workload": "plain exact CCD: 10,000 VF + 10,000 EE seeded FP64 queries", "queries_per_step": nq}
        sample = f"the full {nq}-query batch per step"
    else:
        raise SystemExit(f"unknown workload {args.workload}")
    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        q = step()
        times.append(time.perf_counter() - t0)
    ms = statistics.mean(times) * 1e3
    value = q / (ms * 1e-3)
    return {"metric": "certified CCD queries/s", "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": conf,
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="plain", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=10.0, help="seconds of reference CPU work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    line = run_reference(args) if args.impl == "reference" else run_b200(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and args.impl == "b200":
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
