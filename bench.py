#!/usr/bin/env python
"""Benchmark of the B200 certification hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload scene|plain|batch|cloth|serve|proxy|groups]
                    [--impl b200|reference]

A step is one pass of the hot path over one batch of seeded synthetic input:
  * scene (default): two 40,960-triangle UV spheres (FP64, rigid translation
    toward contact + per-vertex N(0, 1e-3) jitter) -> swept-AABB candidates ->
    exact VF/EE certificates of every candidate;
  * plain: 20,000 independent queries (10k VF + 10k EE);
  * batch, cloth, serve: many uneven scenes in one launch, the dense cloth
    any-hit stress case, a Poisson stream through the serving engine.
metric: certified CCD queries/s (one query = one primitive certificate).
  * proxy: a proxy scene (rigid bodies x patches x motion segments x time
    slabs) built, its raw hits and compacted candidates generated and the
    proposal feature rows of every candidate formed; metric: proxies/s.
  * groups: the candidate-group interface (run_native_dense_group_exact_early_stop)
    over 1M candidate rows in query groups; metric: rows/s.

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

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
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
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self, window: tuple[float, float] | None = None) -> dict:
        """Median SM clock and active throttle reasons of the samples taken
        inside ``window`` (epoch seconds); all samples if none fall in it."""
        import datetime

        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.12)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        parsed = []
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                sm = float(parts[2].split()[0])
                mx = float(parts[3].split()[0])
            except ValueError:
                continue
            parsed.append((ts, sm, mx, [n for n, v in zip(names, parts[6:10]) if v.lower() == "active"]))
        inside = [p for p in parsed if window and window[0] - 0.06 <= p[0] <= window[1] + 0.06]
        use = inside or parsed
        return {"sm_mhz": statistics.median(p[1] for p in use) if use else None,
                "sm_max_mhz": use[-1][2] if use else None,
                "reasons": sorted({r for p in use for r in p[3]}), "samples": len(use),
                "samples_in_timed_region": len(inside)}


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

    def e2e_pipelined(self, steps: int, flush, stream) -> list[float]:
        """End-to-end steps with the transfers overlapped (``overlapped_e2e``)
        over two sets of device records and results; the read-backs of both
        sets are checked to agree."""
        torch = self.torch
        if getattr(self, "set2", None) is None:
            self.set2 = (torch.empty_like(self.pt), torch.empty_like(self.ee), torch.empty_like(self.out_pt),
                         torch.empty_like(self.out_ee), self.certify.Workspace(self.dev))
        sets = ((self.pt, self.ee, self.out_pt, self.out_ee, self.ws), self.set2)
        host_out = [(self.h_out_pt, self.h_out_ee),
                    (torch.empty_like(self.h_out_pt).pin_memory(), torch.empty_like(self.h_out_ee).pin_memory())]

        def copy_in(i):
            sets[i][0].copy_(self.h_pt, non_blocking=True)
            sets[i][1].copy_(self.h_ee, non_blocking=True)

        def compute(i):
            pt, ee, opt, oee, ws = sets[i]
            self.certify.certify_batch2(pt, ee, 0.0, 1.0, self.cfg, opt, oee, ws)

        def copy_out(i):
            host_out[i][0].copy_(sets[i][2], non_blocking=True)
            host_out[i][1].copy_(sets[i][3], non_blocking=True)

        times = overlapped_e2e(torch, steps, flush, stream, copy_in, compute, copy_out)
        if steps >= 2 and not all(torch.equal(a, b) for a, b in zip(host_out[0], host_out[1])):
            raise RuntimeError("the alternating buffer sets returned different certificates")
        return times

    def io_bytes(self) -> tuple[int, int]:
        return self.h_pt.numel() + self.h_ee.numel(), self.h_out_pt.numel() + self.h_out_ee.numel()

    def census(self) -> dict:
        return self.certify.census(self.pt, self.ee, 0.0, 1.0, self.cfg)["stats"]

    def reference_gpu(self, steps: int) -> dict | None:
        """The reference's own GPU path on this batch: certificate_cuda.cu
        compiled unchanged for sm_100a (oracle/_ref), called the way its batch
        API runs (host records in, cudaMalloc + cudaMemcpy + one thread per
        primitive + cudaDeviceSynchronize + copy back + cudaFree per family)."""
        import oracle

        if not oracle.ref_cuda_available():
            return None
        c = self.cfg
        run = lambda fam: oracle.ref_cuda_eval_batch(self.host[fam], 0.0, 1.0, c.eps_time, c.eps_space,
                                                     c.max_subdivision_depth)
        for _ in range(2):
            run("vf"), run("ee")
        ts = []
        for _ in range(max(1, steps)):
            t0 = time.perf_counter()
            run("vf")
            run("ee")
            ts.append(time.perf_counter() - t0)
        ms = statistics.median(ts) * 1e3
        return {"value": self.queries / (ms * 1e-3), "unit": "queries/s", "ms_per_step": ms,
                "what": "the reference's CUDA batch certifier (certificate_cuda.cu, compiled unchanged for sm_100a: "
                        "malloc, copy, one thread per primitive, sync, copy back, free per call) on the same 20,000 "
                        "host records; its certificates are not parity truth (it stops at the first undecided leaf)"}

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


class SceneWorkload:
    """Two 40,960-triangle UV spheres (FP64), B translating toward A with
    per-vertex N(0, 1e-3) jitter: swept-AABB candidates (mesh-pair semantics:
    A x B pairs only) then certificates of every candidate."""

    name = "scene"

    def __init__(self, device, rank: int):
        import torch

        from p2cccd_b200 import certify, scenes
        from p2cccd_b200.scene import ScenePipeline

        self.torch = torch
        self.scene = scenes.two_spheres(seed=20261203 + rank)
        self.cfg = certify.CertConfig(1e-6, 1e-6, 32)
        self.pipe = ScenePipeline(self.scene, device, exclude_self=True, config=self.cfg)
        self.pipe.step_checked()
        self.pipe.fit_capacities()
        summ = self.pipe.step_checked()
        self.pipe.capture()
        self.n_vf, self.n_ee = summ["vf_certified"], summ["ee_certified"]
        self.queries = self.n_vf + self.n_ee
        self.first_summary = summ
        self.h_t0 = torch.from_numpy(self.scene["v_t0"].copy()).pin_memory()
        self.h_t1 = torch.from_numpy(self.scene["v_t1"].copy()).pin_memory()
        self.h_vf = torch.empty_like(self.pipe.vf_results, device="cpu").pin_memory()
        self.h_ee = torch.empty_like(self.pipe.ee_results, device="cpu").pin_memory()
        self.h_summary = torch.empty_like(self.pipe.summary, device="cpu").pin_memory()
        self.phase_events = []
        self.launches_per_step = None

    def config(self) -> dict:
        return scene_config(self.scene, self.cfg)

    def step(self):
        self.pipe.replay()  # the captured step: one graph launch

    def step_uncaptured(self):
        self.pipe.step()

    def step_phased(self):
        """The same step with events between the broad and the narrow phase."""
        torch = self.torch
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        self.pipe.candidates()
        e1.record()
        self.pipe.certify()
        e2.record()
        self.phase_events.append((e0, e1, e2))

    def step_e2e(self):
        self.pipe.v_t0.copy_(self.h_t0, non_blocking=True)
        self.pipe.v_t1.copy_(self.h_t1, non_blocking=True)
        self.pipe.replay()
        self.h_vf.copy_(self.pipe.vf_results, non_blocking=True)
        self.h_ee.copy_(self.pipe.ee_results, non_blocking=True)
        self.h_summary.copy_(self.pipe.summary, non_blocking=True)

    def e2e_pipelined(self, steps: int, flush, stream) -> list[float]:
        """End-to-end steps with the transfers overlapped (``overlapped_e2e``):
        two captured pipelines alternate; the read-backs of both are checked
        to agree (the same frames give the same certificates)."""
        torch = self.torch
        from p2cccd_b200.scene import ScenePipeline

        if getattr(self, "pipe2", None) is None:
            p2 = ScenePipeline(self.scene, self.pipe.v_t0.device, exclude_self=True, config=self.cfg)
            p2.step_checked()
            p2.fit_capacities()
            p2.step_checked()
            p2.capture()
            self.pipe2 = p2
        pipes = (self.pipe, self.pipe2)
        host_out = [(self.h_vf, self.h_ee, self.h_summary),
                    tuple(torch.empty_like(t, device="cpu").pin_memory()
                          for t in (self.pipe2.vf_results, self.pipe2.ee_results, self.pipe2.summary))]

        def copy_in(i):
            pipes[i].v_t0.copy_(self.h_t0, non_blocking=True)
            pipes[i].v_t1.copy_(self.h_t1, non_blocking=True)

        def copy_out(i):
            q = pipes[i]
            for d, src in zip(host_out[i], (q.vf_results, q.ee_results, q.summary)):
                d.copy_(src, non_blocking=True)

        times = overlapped_e2e(torch, steps, flush, stream, copy_in, lambda i: pipes[i].replay(), copy_out)
        if steps >= 2:  # the two pipelines certified the same frames: their certificates agree byte for byte
            rows = (self.n_vf, self.n_ee, None)  # result buffers hold spare capacity beyond the counts
            for name, r, a, b in zip(("vf", "ee", "summary"), rows, host_out[0], host_out[1]):
                if not torch.equal(a[:r] if r is not None else a, b[:r] if r is not None else b):
                    raise RuntimeError(f"the alternating pipelines returned different {name} results")
        return times

    def io_bytes(self) -> tuple[int, int]:
        return (self.h_t0.numel() * 8 + self.h_t1.numel() * 8,
                self.h_vf.numel() + self.h_ee.numel() + self.h_summary.numel())

    def census(self) -> dict:
        from p2cccd_b200 import certify

        vf_rec, ee_rec = self.pipe.materialize()
        return certify.census(certify.records_to_device(vf_rec, self.pipe.device),
                              certify.records_to_device(ee_rec, self.pipe.device), 0.0, 1.0, self.cfg)["stats"]

    def broad_phase_bytes(self) -> int:
        """Algorithmic bytes of candidate generation, B_bp = 48 V + 24 F + 16 E
        + 120 S + 8 P (S = V + F + E, P = pairs): vertex t0/t1 read, index
        read/write, box write, sort-key read/write and box re-read, pair write."""
        s = self.scene
        v, f, e = len(s["v_t0"]), len(s["faces"]), len(s["edges"])
        return 48 * v + 24 * f + 16 * e + 120 * (v + f + e) + 8 * self.queries

    def fused_ideal_bytes(self) -> int:
        """The floor of a fused broad phase that reads the scene once and
        writes the pairs: 48 B per vertex, 12 per face, 8 per edge, 8 per pair."""
        s = self.scene
        return 48 * len(s["v_t0"]) + 12 * len(s["faces"]) + 8 * len(s["edges"]) + 8 * self.queries

    def cpu_reference(self, threads: int, budget_s: float) -> dict:
        ref = ToolSceneStep(self.scene, self.cfg)
        q_sum, s_sum, rounds = 0, 0.0, 0
        t_start = time.perf_counter()
        while True:
            q, sec = ref.run()
            q_sum, s_sum, rounds = q_sum + q, s_sum + sec, rounds + 1
            if time.perf_counter() - t_start >= budget_s:
                break
        return {"queries": q_sum / rounds, "seconds": s_sum / rounds, "threads": 1,
                "sample": ref.describe() + f"; {rounds} whole step(s)"}


def scene_config(scene: dict, cfg) -> dict:
    """The scene workload's config, identical in both arms: built from the
    seeded scene alone (the candidate counts are reported per arm, beside it)."""
    sp = scene["spec"]
    return {"workload": "single-scene broad+narrow: two UV spheres of 40,960 triangles each (160 x 128 rings; "
                        "40,960 is not an icosphere level), FP64, B translating toward A "
                        f"(gap {sp['gap']}, approach {sp['approach']} per step) + per-vertex N(0,{sp['jitter']}) "
                        "jitter, swept-AABB candidates (A x B) then exact VF/EE certificates of every candidate",
            "vertices": int(len(scene["v_t0"])), "triangles": int(len(scene["faces"])),
            "edges": int(len(scene["edges"])), "eps_time": cfg.eps_time, "eps_space": cfg.eps_space,
            "max_subdivision_depth": cfg.max_subdivision_depth, "seed": sp["seed"]}


class ToolSceneStep:
    """One step of the reference's own scene path on the identical scene:
    the scene tool (tools/scene_object_envelope_native_ti_walltime.cpp, compiled
    unchanged) builds its candidates with SweepPairs / BuildVFCandidates /
    BuildEECandidates (:603-696) and certifies every candidate with its
    RunAllExactRows (:1239-1281), whose exact kernel answers with the reference
    certifier.  Single-threaded, as the tool is written.  PrepareScene (PLY
    frames in, swept boxes, edge list) runs once, outside the timed step."""

    def __init__(self, scene, cfg, exclude_self: bool = True):
        import oracle

        self.cfg = cfg
        t0 = time.perf_counter()
        self.tool = oracle.RefToolScene(scene["v_t0"], scene["v_t1"], scene["faces"], 0.0, exclude_self)
        self.prepare_s = time.perf_counter() - t0
        self.last = None

    def run(self) -> tuple[int, float]:
        c = self.cfg
        r = self.tool.time_all_exact(c.eps_time, c.eps_space, c.max_subdivision_depth)
        self.last = r
        return r["calls"], r["candidates_s"] + r["certify_s"]

    def describe(self) -> str:
        r = self.last or {}
        return ("the identical scene through the reference scene tool compiled unchanged: SweepPairs candidates + "
                "RunAllExactRows certificates of every candidate (reference certifier), 1 thread as written; "
                f"last step {r.get('candidates_s', 0.0):.3f} s candidates + {r.get('certify_s', 0.0):.4f} s "
                f"certificates, {r.get('calls', 0)} candidates; PrepareScene ({self.prepare_s:.2f} s incl. PLY "
                "frames) outside the step")


class BatchWorkload:
    """Batched uneven scenes: 256 independent two-sphere scenes, triangle
    counts log-uniform over 1k-200k (9.57M triangles), random rigid motion +
    jitter, every scene's swept-AABB candidates then the certificates of all
    their candidates in ONE persistent launch, the whole step one CUDA graph
    with an autotuned launch shape."""

    name = "batch"
    narrow_kernel = "batch_certify_kernel"

    def __init__(self, device, rank: int):
        import numpy as np
        import torch

        from p2cccd_b200 import certify, scenes
        from p2cccd_b200.batch import BatchPipeline

        self.torch = torch
        world = int(os.environ.get("WORLD_SIZE", "1"))
        if BATCH_PARTITION == "lpt":  # one batch split over the ranks by triangle count (strong scaling)
            from p2cccd_b200.batch import lpt_partition

            self.seed = 20261203
            everything = scenes.uneven_batch(BATCH_SCENES, seed=self.seed)
            self.share = lpt_partition([len(x["faces"]) for x in everything], world)[rank]
            self.scenes = [everything[i] for i in self.share]
        else:  # every rank its own batch (weak scaling)
            self.seed = 20261203 + rank
            self.scenes = scenes.uneven_batch(BATCH_SCENES, seed=self.seed)
        self.cfg = certify.CertConfig(1e-6, 1e-6, 32)
        self.bp = BatchPipeline(self.scenes, device, exclude_self=True, config=self.cfg, streams=8)
        self.bp.step_checked()
        self.bp.fit_capacities()
        summ = self.bp.step_checked()
        if AUTOTUNE_REPS > 0:
            self.tuning = self.bp.autotune(reps=AUTOTUNE_REPS)
        else:  # the library's default launch shape
            self.tuning = dict(self.bp.tuning.as_dict(), streams=self.bp.n_streams)
        self.bp.capture()
        self.summaries = summ
        self.queries = sum(x["vf_certified"] + x["ee_certified"] for x in summ)
        hits = np.array([x["collisions"] + x["undecided"] for x in summ], dtype=np.float64)
        cands = np.array([max(1, x["vf_certified"] + x["ee_certified"]) for x in summ], dtype=np.float64)
        self.hit_frac = hits / cands
        self.h_t0 = torch.empty_like(self.bp.v_t0, device="cpu").pin_memory()
        self.h_t1 = torch.empty_like(self.bp.v_t1, device="cpu").pin_memory()
        self.h_t0.copy_(self.bp.v_t0)
        self.h_t1.copy_(self.bp.v_t1)
        self.d2h = [(self.bp.vf_results, torch.empty_like(self.bp.vf_results, device="cpu").pin_memory()),
                    (self.bp.ee_results, torch.empty_like(self.bp.ee_results, device="cpu").pin_memory()),
                    (self.bp.summaries, torch.empty_like(self.bp.summaries, device="cpu").pin_memory())]
        self.phase_events = []

    def config(self) -> dict:
        tris = [s["spec"]["triangles"] for s in self.scenes]
        return {"workload": f"batched uneven scenes: {len(self.scenes)} independent two-UV-sphere scenes, triangle counts "
                            "log-uniform 1k-200k, random rigid motion (rotation + translation into contact, "
                            "penetration 0.25 f, f ~ U[5%, 40%]) + N(0,1e-3) jitter, FP64; per-scene swept-AABB "
                            "candidates then every candidate certified in one persistent launch, one CUDA graph",
                "scenes": len(self.scenes), "triangles": int(sum(tris)), "triangles_min": int(min(tris)),
                "triangles_max": int(max(tris)), "queries_per_step": self.queries,
                "contact_fraction_measured": {"min": float(self.hit_frac.min()), "mean": float(self.hit_frac.mean()),
                                              "max": float(self.hit_frac.max()),
                                              "definition": "(collisions + undecided) / candidates per scene"},
                "autotuned": {k: self.tuning[k] for k in ("blocks_per_sm", "fetch_limit", "helper_warps", "streams")},
                "eps_time": self.cfg.eps_time, "eps_space": self.cfg.eps_space,
                "max_subdivision_depth": self.cfg.max_subdivision_depth, "seed": self.seed}

    def step(self):
        self.bp.replay()

    def step_uncaptured(self):
        self.bp.step()

    def step_phased(self):
        torch = self.torch
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        self.bp.candidates()
        e1.record()
        self.bp.certify()
        e2.record()
        self.phase_events.append((e0, e1, e2))

    def step_e2e(self):
        self.bp.v_t0.copy_(self.h_t0, non_blocking=True)
        self.bp.v_t1.copy_(self.h_t1, non_blocking=True)
        self.bp.replay()
        for d, h in self.d2h:
            h.copy_(d, non_blocking=True)

    def e2e_pipelined(self, steps: int, flush, stream) -> list[float]:
        """End-to-end steps with the transfers overlapped (``overlapped_e2e``):
        two captured batch pipelines with the same launch shape alternate; the
        per-scene summaries read back from both are checked to agree."""
        torch = self.torch
        from p2cccd_b200.batch import BatchPipeline, BatchTuning

        if getattr(self, "bp2", None) is None:
            b2 = BatchPipeline(self.scenes, self.bp.device, exclude_self=True, config=self.cfg,
                               streams=self.bp.n_streams)
            b2.step_checked()
            b2.fit_capacities()
            b2.step_checked()
            t = self.bp.tuning
            b2.tuning = BatchTuning(t.blocks_per_sm, t.fetch_limit, t.helper_warps, 0)
            b2.capture()
            self.bp2 = b2
        pipes = (self.bp, self.bp2)
        host_out = [[h for _, h in self.d2h],
                    [torch.empty_like(d, device="cpu").pin_memory()
                     for d in (self.bp2.vf_results, self.bp2.ee_results, self.bp2.summaries)]]

        def copy_in(i):
            pipes[i].v_t0.copy_(self.h_t0, non_blocking=True)
            pipes[i].v_t1.copy_(self.h_t1, non_blocking=True)

        def copy_out(i):
            q = pipes[i]
            for d, h in zip((q.vf_results, q.ee_results, q.summaries), host_out[i]):
                h.copy_(d, non_blocking=True)

        times = overlapped_e2e(torch, steps, flush, stream, copy_in, lambda i: pipes[i].replay(), copy_out)
        if steps >= 2 and not torch.equal(host_out[0][2], host_out[1][2]):
            raise RuntimeError("the alternating batch pipelines returned different scene summaries")
        return times

    def io_bytes(self) -> tuple[int, int]:
        return self.h_t0.numel() * 8 + self.h_t1.numel() * 8, sum(h.numel() for _, h in self.d2h)

    def census(self) -> dict:
        import numpy as np

        from p2cccd_b200 import certify

        vf, ee = zip(*(self.bp.materialize(i) for i in range(self.bp.n)))
        vf, ee = np.concatenate(vf), np.concatenate(ee)
        return certify.census(certify.records_to_device(vf, self.bp.device),
                              certify.records_to_device(ee, self.bp.device), 0.0, 1.0, self.cfg)["stats"]

    def broad_phase_bytes(self) -> int:
        return sum(48 * len(s["v_t0"]) + 12 * len(s["faces"]) + 8 * len(s["edges"]) for s in self.scenes) + \
            8 * self.queries

    def cpu_reference(self, threads: int, budget_s: float) -> dict:
        return _batch_reference_sample(self.scenes, self.cfg, budget_s)


def _batch_reference_sample(scenes_list, cfg, budget_s: float, order=None, exclude_self: bool = True) -> dict:
    """The reference scene tool (compiled unchanged, 1 thread as written) on
    whole scenes of the batch, in batch order (or `order`), until budget_s:
    its sweep-and-prune candidates (self pairs excluded) then its
    every-candidate certificate rows (RunAllExactRows) of both families."""
    import oracle

    t_start = time.perf_counter()
    secs, calls, done, tris = 0.0, 0, 0, 0
    for i in (order if order is not None else range(len(scenes_list))):
        s = scenes_list[i]
        tool = oracle.RefToolScene(s["v_t0"], s["v_t1"], s["faces"], 0.0, exclude_self)
        r = tool.time_all_exact(cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth)
        secs += r["candidates_s"] + r["certify_s"]
        calls += r["calls"]
        done += 1
        tris += len(s["faces"])
        if time.perf_counter() - t_start >= budget_s:
            break
    return {"queries": calls, "seconds": secs, "threads": 1, "scenes": done,
            "sample": f"reference scene tool (SweepPairs candidates + RunAllExactRows, 1 thread as written) on "
                      f"{done} whole scene(s) of the batch ({tris} triangles, {calls} candidates)"}


class ClothWorkload:
    """Dense-contact stress: a 513 x 513 cloth grid (524,288 triangles)
    draped onto a 100,000-triangle UV sphere (250 x 200 rings) with a 1e-4
    initial gap, self pairs with adjacency exclusion, then the scheduled
    any-hit with fallback replay over object-pair groups with priorities from
    a seeded scheduler stub (proposal top-K 4096).  A query is one exact call
    of the procedure (proposal or fallback replay)."""

    name = "cloth"
    narrow_kernel = "anyhit_certify_kernel"

    def __init__(self, device, rank: int):
        import torch

        from p2cccd_b200 import certify, scenes
        from p2cccd_b200.scene import ScenePipeline

        self.torch = torch
        self.seed = 20261203 + rank
        if CLOTH_N == 513:
            self.scene = scenes.cloth_on_sphere(seed=self.seed)
        else:  # a smaller instance with the same proportions (profiling cases)
            k = max(8, int(round(250 * CLOTH_N / 513)))
            self.scene = scenes.cloth_on_sphere(n=CLOTH_N, sphere_lon=k, sphere_rings=max(6, (k * 4) // 5),
                                                seed=self.seed)
        self.cfg = certify.CertConfig(1e-6, 1e-6, 32)
        self.top_k = 4096
        self.pipe = ScenePipeline(self.scene, device, exclude_self=False, config=self.cfg, narrow="anyhit",
                                  top_k=self.top_k, scheduler_seed=self.seed, vf_capacity=1 << 20,
                                  ee_capacity=3 << 20)
        self.pipe.step_checked()
        self.pipe.fit_capacities()
        summ = self.pipe.step_checked()
        self.pipe.capture()
        self.first_summary = summ
        self.queries = summ["calls"]
        self.h_t0 = torch.from_numpy(self.scene["v_t0"].copy()).pin_memory()
        self.h_t1 = torch.from_numpy(self.scene["v_t1"].copy()).pin_memory()
        p = self.pipe
        self.d2h = [(p.anyhit_vf.hit, torch.empty_like(p.anyhit_vf.hit, device="cpu").pin_memory()),
                    (p.anyhit_ee.hit, torch.empty_like(p.anyhit_ee.hit, device="cpu").pin_memory()),
                    (p.anyhit_vf.group_detected, torch.empty_like(p.anyhit_vf.group_detected, device="cpu").pin_memory()),
                    (p.anyhit_ee.group_detected, torch.empty_like(p.anyhit_ee.group_detected, device="cpu").pin_memory()),
                    (p.anyhit_vf.summary, torch.empty_like(p.anyhit_vf.summary, device="cpu").pin_memory()),
                    (p.anyhit_ee.summary, torch.empty_like(p.anyhit_ee.summary, device="cpu").pin_memory())]
        self.phase_events = []

    def config(self) -> dict:
        sp = self.scene["spec"]
        s = self.first_summary
        return {"workload": f"dense-contact stress: {sp['cloth_n']} x {sp['cloth_n']} cloth grid "
                            f"({sp['cloth_triangles']:,} triangles) draped onto a {sp['sphere_triangles']:,}-triangle "
                            "UV sphere, 1e-4 initial gap, FP64, self pairs with "
                            "adjacency exclusion, swept-AABB candidates then scheduled any-hit with fallback replay "
                            "over object-pair groups (priorities from a seeded uniform scheduler stub, top-K "
                            f"{self.top_k}); a query is one exact call of the procedure",
                "vertices": int(len(self.scene["v_t0"])), "triangles": int(len(self.scene["faces"])),
                "edges": int(len(self.scene["edges"])), "candidates": s["candidates"],
                "groups": s["groups"], "detected_groups": s["detected_groups"],
                "proposal_calls": s["proposal_calls"], "fallback_calls": s["fallback_calls"],
                "speculative_certificates": s["speculative"], "queries_per_step": self.queries,
                "eps_time": self.cfg.eps_time, "eps_space": self.cfg.eps_space,
                "max_subdivision_depth": self.cfg.max_subdivision_depth, "seed": sp["seed"]}

    def step(self):
        self.pipe.replay()

    def step_uncaptured(self):
        self.pipe.step()

    def step_phased(self):
        torch = self.torch
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        self.pipe.candidates()
        e1.record()
        self.pipe.narrow_phase()
        e2.record()
        self.phase_events.append((e0, e1, e2))

    def step_e2e(self):
        self.pipe.v_t0.copy_(self.h_t0, non_blocking=True)
        self.pipe.v_t1.copy_(self.h_t1, non_blocking=True)
        self.pipe.replay()
        for d, h in self.d2h:
            h.copy_(d, non_blocking=True)

    def e2e_pipelined(self, steps: int, flush, stream) -> list[float]:
        """End-to-end steps with the transfers overlapped (``overlapped_e2e``):
        two captured any-hit pipelines alternate; their group decisions are
        checked to agree."""
        torch = self.torch
        from p2cccd_b200.scene import ScenePipeline

        if getattr(self, "pipe2", None) is None:
            p2 = ScenePipeline(self.scene, self.pipe.v_t0.device, exclude_self=False, config=self.cfg,
                               narrow="anyhit", top_k=self.top_k, scheduler_seed=self.seed, vf_capacity=1 << 20,
                               ee_capacity=3 << 20)
            p2.step_checked()
            p2.fit_capacities()
            p2.step_checked()
            p2.capture()
            self.pipe2 = p2
        pipes = (self.pipe, self.pipe2)

        def outs(q):
            return (q.anyhit_vf.hit, q.anyhit_ee.hit, q.anyhit_vf.group_detected, q.anyhit_ee.group_detected,
                    q.anyhit_vf.summary, q.anyhit_ee.summary)

        host_out = [[h for _, h in self.d2h], [torch.empty_like(d, device="cpu").pin_memory() for d in outs(self.pipe2)]]

        def copy_in(i):
            pipes[i].v_t0.copy_(self.h_t0, non_blocking=True)
            pipes[i].v_t1.copy_(self.h_t1, non_blocking=True)

        def copy_out(i):
            for d, h in zip(outs(pipes[i]), host_out[i]):
                h.copy_(d, non_blocking=True)

        times = overlapped_e2e(torch, steps, flush, stream, copy_in, lambda i: pipes[i].replay(), copy_out)
        # the group decisions are deterministic (how many speculative certificates ran is not)
        if steps >= 2 and not all(torch.equal(a, b) for a, b in zip(host_out[0][2:4], host_out[1][2:4])):
            raise RuntimeError("the alternating any-hit pipelines returned different group decisions")
        return times

    def io_bytes(self) -> tuple[int, int]:
        return self.h_t0.numel() * 8 + self.h_t1.numel() * 8, sum(h.numel() for _, h in self.d2h)

    def census(self) -> dict:
        """FP64 census of the calls the procedure makes (speculative
        certificates are device work beyond the algorithm, not counted)."""
        import numpy as np

        from p2cccd_b200 import certify

        vf_rec, ee_rec = self.pipe.materialize()
        ev_vf, _ = self.pipe.anyhit_vf.read_candidates(len(vf_rec))
        ev_ee, _ = self.pipe.anyhit_ee.read_candidates(len(ee_rec))
        vf_rec, ee_rec = vf_rec[ev_vf > 0], ee_rec[ev_ee > 0]
        return certify.census(certify.records_to_device(np.ascontiguousarray(vf_rec), self.pipe.device),
                              certify.records_to_device(np.ascontiguousarray(ee_rec), self.pipe.device), 0.0, 1.0,
                              self.cfg)["stats"]

    def broad_phase_bytes(self) -> int:
        s = self.scene
        return 48 * len(s["v_t0"]) + 12 * len(s["faces"]) + 8 * len(s["edges"]) + 8 * self.first_summary["candidates"]

    def cpu_reference(self, threads: int, budget_s: float) -> dict:
        return _cloth_reference_sample(self.cfg, self.top_k, budget_s)


def _cloth_reference_sample(cfg, top_k: int, budget_s: float) -> dict:
    """The reference scene tool (compiled unchanged; its Tight-Inclusion calls
    answered by the reference certifier), single-threaded as written, on the
    quarter-size instance of the cloth workload (257 x 257 cloth, 125 x 100
    sphere: 156,072 triangles): its sweep-and-prune candidates then its
    scheduled any-hit rows of both families.  Its candidate sweep grows
    faster than linearly, so the quarter-size rate favours the reference."""
    import oracle
    from p2cccd_b200 import scenes

    s = scenes.cloth_on_sphere(n=257, sphere_lon=125, sphere_rings=100)
    tool = oracle.RefToolScene(s["v_t0"], s["v_t1"], s["faces"], 0.0, False)
    t_start = time.perf_counter()
    secs, calls, rounds = 0.0, 0, 0
    while True:
        r = tool.time_step(top_k, cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth)
        secs += r["candidates_s"] + r["anyhit_vf_s"] + r["anyhit_ee_s"]
        calls += r["calls"]
        rounds += 1
        if time.perf_counter() - t_start >= budget_s:
            break
    return {"queries": calls / rounds, "seconds": secs / rounds, "threads": 1,
            "sample": f"reference scene tool (SweepPairs candidates + RunScheduledAnyHitRows, 1 thread) on the "
                      f"quarter-size cloth instance ({len(s['faces'])} triangles, {r['candidates']} candidates, "
                      f"{r['calls']} exact calls per step), {rounds} step(s)"}


class SceneReferenceSample:
    """The reference CPU path on the scene workload, in bounded slices.

    The reference mesh builder (BuildMeshExactCertificateQuery) is
    translation-only, so it runs on the translation-only form of the same
    scene: the two unjittered spheres, A at rest, B translating as in the
    step.  Its pair loops cost one identical swept-box test per pair, O(V*F +
    E^2) (~5.4e9 tests at full size), so it runs on sphere A restricted to the
    triangles whose x extent reaches B's swept bounding box (every candidate
    of the full query lies in it), cut into n_slices contiguous slices; a
    slice's build time is scaled by the exact ratio of pair tests full/sample
    and the reference certificates of every primitive it returns are timed in
    full on `threads` threads.
    """

    def __init__(self, scene, cfg, threads: int, n_slices: int = 1):
        import numpy as np

        from p2cccd_b200 import scenes

        sp = scene["spec"]
        self.cfg, self.threads = cfg, threads
        base, faces = scenes.uv_sphere(sp["n_lon"], sp["n_rings"])
        ang = 0.37
        rot = np.array([[np.cos(ang), 0.0, np.sin(ang)], [0.0, 1.0, 0.0], [-np.sin(ang), 0.0, np.cos(ang)]])
        self.vb = base @ rot.T
        self.fb = faces.astype(np.uint32)
        self.tb0 = np.array([2.0 + sp["gap"], 0.0, 0.0])
        self.tb1 = self.tb0 - np.array([sp["approach"], 0.0, 0.0])
        b_min_x = min((self.vb + self.tb0)[:, 0].min(), (self.vb + self.tb1)[:, 0].min())
        fa_s = faces[base[faces][:, :, 0].max(axis=1) >= b_min_x]
        ea_full = len(scenes.unique_edges(faces))
        nvb, nfb = len(self.vb), len(faces)
        tests_full = len(base) * nfb + nvb * len(faces) + ea_full * ea_full
        self.slices, tests_sample = [], 0
        for chunk in np.array_split(fa_s, max(1, n_slices)):
            used = np.unique(chunk)
            remap = -np.ones(len(base), np.int64)
            remap[used] = np.arange(len(used))
            fa = remap[chunk].astype(np.uint32)
            ea = len(scenes.unique_edges(fa.astype(np.int32)))
            tests_sample += len(used) * nfb + nvb * len(fa) + ea * ea_full
            self.slices.append((base[used], fa))
        self.n_faces_sample = len(fa_s)
        self.scale = tests_full / tests_sample

    def run(self, i: int) -> tuple[int, float, float]:
        """Slice i mod n_slices: (queries, extrapolated build seconds, certify seconds)."""
        import numpy as np

        import oracle

        va, fa = self.slices[i % len(self.slices)]
        z = np.zeros(3)
        t0 = time.perf_counter()
        pts, ees = oracle.ref_build_mesh_query(va, fa, z, z, self.vb, self.fb, self.tb0, self.tb1)
        t1 = time.perf_counter()
        c = self.cfg
        for rec in (pts, ees):
            if len(rec):
                oracle.ref_eval_batch(rec, 0.0, 1.0, c.eps_time, c.eps_space, c.max_subdivision_depth,
                                      threads=self.threads)
        t2 = time.perf_counter()
        return len(pts) + len(ees), (t1 - t0) * self.scale, t2 - t1

    def describe(self) -> str:
        return (f"translation-only form of the scene through the reference BuildMeshExactCertificateQuery on sphere "
                f"A's {self.n_faces_sample} triangles that reach B (in {len(self.slices)} slice(s)) vs the full "
                f"sphere B; build time x{self.scale:.1f} (= full/sample pair tests), plus reference certificates of "
                f"every candidate on {self.threads} threads")


def _scene_reference_sample(scene, cfg, budget_s: float, threads: int) -> dict:
    """Whole-sample rounds of SceneReferenceSample for about budget_s seconds."""
    ref = SceneReferenceSample(scene, cfg, threads, 1)
    t_start = time.perf_counter()
    q_sum, s_sum, rounds = 0, 0.0, 0
    while True:
        q, b, c = ref.run(0)
        q_sum += q
        s_sum += b + c
        rounds += 1
        if time.perf_counter() - t_start >= budget_s:
            break
    return {"queries": q_sum / rounds, "seconds": s_sum / rounds, "sample": ref.describe() + f"; {rounds} round(s)"}


WORKLOADS = {"plain": PlainWorkload, "scene": SceneWorkload, "cloth": ClothWorkload, "batch": BatchWorkload}


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
    """The slowest rank's value (all ranks call this in the same order)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(world, value: float) -> float:
    """All ranks' values added (all ranks call this in the same order)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def partition_rate(world: int, units_this_rank: float, ms_this_rank: float) -> tuple[float, float]:
    """Whole-job rate of one job split over N ranks (LPT): every rank's
    units over the slowest rank's time.  Every rank calls it."""
    units = _sum_over_ranks(world, units_this_rank)
    ms = _max_over_ranks(world, ms_this_rank)
    return units / (ms * 1e-3), ms


def replica_rate(world: int, units_per_rank: float, ms_per_rank: float) -> tuple[float, float]:
    """Whole-job rate of N replicas: all ranks' units over the slowest rank's
    time (max over ranks), and that time.  Every rank calls it."""
    ms = _max_over_ranks(world, ms_per_rank)
    return units_per_rank * world / (ms * 1e-3), ms


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


def overlapped_e2e(torch, steps, flush, stream, copy_in, compute, copy_out) -> list[float]:
    """End-to-end steps with the transfers overlapped on a copy stream, two
    buffer sets alternating: while step k computes on set k % 2, step k+1's
    inputs come in to the other set (``copy_in(slot)``) and step k-1's
    results go out of it (``copy_out(slot)``).  Every copy is issued after
    the start event of the step it overlaps and waited for before that step's
    end event, so each timed region holds its share of the transfers; a last
    region drains the final step's results and is spread over the steps.
    Returns per-step milliseconds."""
    cs = torch.cuda.Stream(stream.device)
    ev_in = [torch.cuda.Event(), torch.cuda.Event()]
    with torch.cuda.stream(cs):
        copy_in(0)
        ev_in[0].record(cs)
    times = []
    for k in range(steps + 1):
        flush.fill_(1)
        start, end, ev_x = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
                            torch.cuda.Event())
        start.record(stream)
        cs.wait_event(start)
        with torch.cuda.stream(cs):
            if k >= 1:
                copy_out((k - 1) % 2)
            if k + 1 < steps:  # the set step k-1 used, which is done with it
                copy_in((k + 1) % 2)
                ev_in[(k + 1) % 2].record(cs)
            ev_x.record(cs)
        if k < steps:
            stream.wait_event(ev_in[k % 2])
            compute(k % 2)
        stream.wait_event(ev_x)
        end.record(stream)
        end.synchronize()
        times.append(start.elapsed_time(end))
    drain = times.pop()
    return [t + drain / steps for t in times]


def count_kernels(torch, fn) -> tuple[int, dict]:
    """Kernels one call of fn launches (torch profiler / CUPTI), by name."""
    try:
        from torch.profiler import ProfilerActivity, profile

        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        names: dict[str, int] = {}
        for ev in prof.events():
            if getattr(ev, "device_type", None) is not None and "CUDA" in str(ev.device_type):
                nm = ev.name
                if "memcpy" in nm.lower() or "memset" in nm.lower():
                    continue
                names[nm] = names.get(nm, 0) + 1
        return sum(names.values()), names
    except Exception as exc:  # profiler unavailable: report unknown
        return -1, {"error": str(exc)}


def run_b200(args) -> dict | None:
    import torch

    from p2cccd_b200 import certify

    world, rank, local = _dist_setup(args)
    dev = torch.device("cuda", local if world > 1 else 0)
    wl = WORKLOADS[args.workload](dev, rank)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    gpu_index = dev.index if world > 1 else int((os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]) or 0)
    sampler = ClockSampler(gpu_index)
    sampler.start()
    for _ in range(args.warmup):
        wl.step()
    torch.cuda.synchronize()
    _barrier(world)
    torch.cuda.synchronize()
    t_begin = time.time()
    times = time_steps(torch, wl.step, args.steps, flush, stream)
    torch.cuda.synchronize()
    t_end = time.time()
    _barrier(world)
    clocks = sampler.stop((t_begin, t_end))
    # e2e through the public API with pinned host buffers
    for _ in range(max(1, args.warmup)):
        wl.step_e2e()
    torch.cuda.synchronize()
    e2e_serial_times = time_steps(torch, wl.step_e2e, args.steps, flush, stream)
    torch.cuda.synchronize()
    e2e_times = e2e_serial_times
    if hasattr(wl, "e2e_pipelined"):
        wl.e2e_pipelined(max(2, args.warmup), flush, stream)
        e2e_times = wl.e2e_pipelined(args.steps, flush, stream)
        torch.cuda.synchronize()
    ms = statistics.mean(times)
    split = args.workload == "batch" and BATCH_PARTITION == "lpt"
    rate = partition_rate if split else replica_rate
    value, ms_max = rate(world, wl.queries, ms)
    e2e_value, e2e_ms = rate(world, wl.queries, statistics.mean(e2e_times))
    n_kernels, kernel_names = count_kernels(torch, getattr(wl, "step_uncaptured", wl.step))
    census = wl.census()
    fp64_rate = certify.probe_fp64_rate(dev)
    peaks = _load_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hbm_src = "of measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "of fallback (6.65 TB/s)"
    fp64_roof = {"bound": "fp64", "peak": fp64_rate / 1e12, "unit": "TFLOP/s", "traffic": None,
                 "peak_source": "measured in-run: p2c_probe_fp64 (separately rounded DMUL+DADD chains)",
                 "algorithmic_fp64_ops_per_launch": census["fp64_ops"],
                 "nodes_per_launch": census["nodes_evaluated"]}
    phases = None
    if hasattr(wl, "step_phased"):
        wl.phase_events.clear()
        for _ in range(args.steps):
            flush.fill_(1)
            wl.step_phased()
        torch.cuda.synchronize()
        bp = statistics.mean(e0.elapsed_time(e1) for e0, e1, _ in wl.phase_events)
        npm = statistics.mean(e1.elapsed_time(e2) for _, e1, e2 in wl.phase_events)
        phases = {"broad_ms": bp, "narrow_ms": npm}
        bp_bytes = wl.broad_phase_bytes()
        broad_roof = {"bound": "hbm", "achieved": bp_bytes / (bp * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                      "frac": bp_bytes / (bp * 1e-3) / 1e9 / hbm_peak, "traffic": None,
                      "peak_source": hbm_src, "kernel": "candidate generation (boxes, sort, sweep)",
                      "algorithmic_bytes_per_step": bp_bytes, "bytes_formula": "48V + 24F + 16E + 120(V+F+E) + 8P"}
        if hasattr(wl, "fused_ideal_bytes"):
            broad_roof["fused_ideal_bytes_per_step"] = wl.fused_ideal_bytes()
        narrow = dict(fp64_roof, kernel=getattr(wl, "narrow_kernel", "certify_scene_kernel"),
                      achieved=census["fp64_ops"] / (npm * 1e-3) / 1e12,
                      frac=census["fp64_ops"] / (npm * 1e-3) / fp64_rate)
        roofline, secondary = (narrow, broad_roof) if npm >= bp else (broad_roof, narrow)
    else:
        roofline = dict(fp64_roof, kernel="certify_records_kernel", achieved=census["fp64_ops"] / (ms * 1e-3) / 1e12,
                        frac=census["fp64_ops"] / (ms * 1e-3) / fp64_rate)
        secondary = None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = wl.cpu_reference(threads, args.cpu_budget)
        cpu = {"value": r["queries"] / r["seconds"], "unit": "queries/s", "cores": r.get("threads", threads),
               "kind": "reference", "sample": r["sample"]}
        if hasattr(wl, "reference_gpu"):  # the reference's GPU path, a comparison row beside the CPU one
            cpu["reference_gpu"] = wl.reference_gpu(min(args.steps, 20))
    served = None
    if args.workload == "scene" and not args.no_served:
        served = serve_bench(args, dev, rank, args.cpu_budget if (cpu is not None) else None)
    if rank != 0:
        return None
    h2d, d2h = wl.io_bytes()
    line = {
        "metric": "certified CCD queries/s", "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "p50_ms": statistics.median(times), "p99_ms": sorted(times)[max(0, int(0.99 * len(times)) - 1)],
        "higher_is_better": True, "scaling": "strong" if split else "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {**wl.config(), "l2": f"flushed between timed steps ({L2_FLUSH_BYTES >> 20} MB write)",
                   "parallelism": (f"one batch LPT-packed over {world} ranks by triangle count" if split
                                   else f"replicas x{world}")},
        "queries_per_step": wl.queries,
        "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms, "pipelined": e2e_times is not e2e_serial_times,
                "serial_ms_per_step": statistics.mean(e2e_serial_times),
                "method": ("two buffer sets (captured pipelines for the scene) alternate; inputs in and results "
                           "out on a copy stream, overlapped with the neighbouring steps' compute; each transfer "
                           "inside the timed region of the step it overlaps"
                           if e2e_times is not e2e_serial_times else
                           "copy in, step, copy out, in order on one stream")},
        "gpu_launches": n_kernels * args.steps if n_kernels >= 0 else None,
        "kernels_per_step": kernel_names,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    if phases is not None:
        line["phases"] = phases
        line["roofline_secondary"] = secondary
    if served is not None:
        line["served"] = served
    if args.benchmark_rows:
        _write_benchmark_rows(args, wl, times, phases, census, line, dev)
    return line


def _write_benchmark_rows(args, wl, times, phases, census, line, dev) -> None:
    """The run as a BenchmarkRowV2 (the reference's export schema) in
    DIR/benchmark_v2.jsonl and .csv, from the device counters of the census
    launch and the per-step CUDA-event times."""
    import hashlib

    import torch

    from p2cccd_b200 import rows

    keys = ("collisions", "separations", "undecided", "vf_certified", "ee_certified")
    if isinstance(getattr(wl, "summaries", None), list):
        tot = {k: sum(int(x.get(k, 0)) for x in wl.summaries) for k in keys}
    elif getattr(wl, "first_summary", None) is not None:
        tot = {k: int(wl.first_summary.get(k, 0)) for k in keys}
    else:  # independent queries: the families of the batch
        tot = dict.fromkeys(keys, 0)
        tot["vf_certified"], tot["ee_certified"] = len(wl.host["vf"]), len(wl.host["ee"])
    extra = {}
    if tot["vf_certified"] + tot["ee_certified"] != wl.queries:  # exact calls not split by family (any-hit)
        tot["vf_certified"] = tot["ee_certified"] = 0
        extra = {"family_unknown_exact_calls": int(wl.queries), "exact_calls_total": int(wl.queries)}
    cfg = json.dumps(line["config"], sort_keys=True, default=str)
    row = rows.benchmark_row_v2(
        run_id=f"{args.workload}-{int(time.time())}", dataset_name="synthetic", scene_name=args.workload,
        method_name="b200", config_hash=hashlib.sha1(cfg.encode()).hexdigest()[:16],
        seed=int(line["config"].get("seed") or 0), query_count=int(wl.queries), latencies_ms=times,
        exact_ms=(phases or {}).get("narrow_ms", statistics.mean(times)), rt_ms=(phases or {}).get("broad_ms", 0.0),
        pt_exact_calls=tot["vf_certified"], ee_exact_calls=tot["ee_certified"],
        distance_evals=int(census.get("distance_evals", 0)), collisions=tot["collisions"],
        separations=tot["separations"], undecided=tot["undecided"],
        candidate_bytes=8 * int(wl.queries), vram_peak_bytes=torch.cuda.max_memory_allocated(dev), **extra)
    out = Path(args.benchmark_rows)
    rows.write_benchmark_v2_jsonl(out / "benchmark_v2.jsonl", [row])
    out.mkdir(parents=True, exist_ok=True)
    (out / "benchmark_v2.csv").write_text(rows.benchmark_csv([row]))


# --------------------------------------------------------------------------
# serving: a Poisson stream of mixed CCD steps through the continuous-batching engine


def _serve_pool(seed: int) -> list[tuple[str, dict, bool]]:
    """Meshes of the serving stream: the three scene kinds (two spheres,
    uneven-batch scene, cloth on sphere) at 10k-600k triangles."""
    from p2cccd_b200 import scenes

    pool = []
    for k, tris in enumerate((10_000, 25_000, 60_000, 150_000, 300_000, 600_000)):
        kind = ("spheres", "rigid", "cloth")[k % 3]
        if kind == "spheres":
            r = max(3, int(round((tris / 4 / 1.25) ** 0.5)))
            s = scenes.two_spheres(n_lon=max(4, int(round(tris / 4 / r))), n_rings=r, seed=seed + k)
            pool.append((f"{kind}{tris}", s, True))
        elif kind == "rigid":
            s = scenes.uneven_batch(1, tri_min=tris, tri_max=tris, seed=seed + k)[0]
            pool.append((f"{kind}{tris}", s, True))
        else:
            sphere = tris // 6
            r = max(6, int(round((sphere / 2 / 1.25) ** 0.5)))
            lon = max(8, int(round(sphere / 2 / r)))
            n = int(round(((tris - 2 * lon * r) / 2) ** 0.5)) + 1
            s = scenes.cloth_on_sphere(n=n, sphere_lon=lon, sphere_rings=r, seed=seed + k)
            pool.append((f"{kind}{tris}", s, False))
    for kind, tris in (("cloth", 300_000), ("spheres", 600_000), ("rigid", 10_000)):
        if kind == "cloth":
            s = scenes.cloth_on_sphere(n=353, sphere_lon=130, sphere_rings=100, seed=seed + 17)
        elif kind == "spheres":
            s = scenes.two_spheres(n_lon=432, n_rings=347, seed=seed + 18)
        else:
            s = scenes.uneven_batch(1, tri_min=tris, tri_max=tris, seed=seed + 19)[0]
        pool.append((f"{kind}{tris}b", s, kind != "cloth"))
    return pool


def _served_run(eng, reqs, torch) -> tuple[list, float]:
    """One stream through a server: wall seconds from the start to the last result."""
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done = eng.run(reqs)
    return done, time.perf_counter() - t0


def _tool_serve_sample(pool, cfg, budget_s: float) -> dict:
    """The reference scene tool (compiled unchanged: SweepPairs candidates +
    RunScheduledAnyHitRows with its random policy, top-K 4096, 1 thread as
    written) on whole steps of the serving meshes, smallest first, while the
    budget lasts."""
    import oracle

    done, secs, cands, calls, t_start = [], 0.0, 0, 0, time.perf_counter()
    for key, s, excl in sorted(pool, key=lambda p: len(p[1]["faces"])):
        tool = oracle.RefToolScene(s["v_t0"], s["v_t1"], s["faces"], 0.0, excl)
        r = tool.time_step(4096, cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth)
        done.append((key, len(s["faces"]), r["candidates_s"] + r["anyhit_vf_s"] + r["anyhit_ee_s"]))
        secs += done[-1][2]
        cands += r["candidates"]
        calls += r["calls"]
        if time.perf_counter() - t_start > budget_s:
            break
    return {"value": len(done) / secs, "unit": "steps/s", "cores": 1, "kind": "reference",
            "candidates_per_s": cands / secs, "exact_calls_per_s": calls / secs,
            "sample": "the reference scene tool (SweepPairs + RunScheduledAnyHitRows, random policy, top-K 4096, "
                      "1 thread as written) on one whole step of each of the smallest serving meshes: " +
                      ", ".join(f"{k} ({t} tris, {sec:.2f} s)" for k, t, sec in done)}


def serve_bench(args, dev, rank: int, cpu_budget: float | None) -> dict:
    """The serving stream: Poisson arrivals of CCD steps drawn from the
    two-sphere, rigid uneven-scene and cloth-on-sphere kinds at 10k-600k
    triangles, through the native server (p2c_serve_*), beside the plain path
    (each step alone through the single-scene pipeline, every candidate
    certified, host sync per step) on the same requests."""
    import numpy as np
    import torch

    from p2cccd_b200 import certify
    from p2cccd_b200.scene import ScenePipeline
    from p2cccd_b200.serve import Request, ServeEngine, latency_stats

    seed = 20261203 + rank
    cfg = certify.CertConfig(1e-6, 1e-6, 32)
    pool = _serve_pool(seed)
    host = {}
    for key, s, excl in pool:
        host[key] = (torch.from_numpy(np.ascontiguousarray(s["v_t0"])).pin_memory(),
                     torch.from_numpy(np.ascontiguousarray(s["v_t1"])).pin_memory(), len(s["faces"]), excl, s)
    keys = [k for k, _, _ in pool]
    rng = np.random.default_rng(seed)
    n_req = max(1, args.serve_requests)
    picks = [keys[int(rng.integers(len(keys)))] for _ in range(n_req)]
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, n_req))

    def stream(times):
        return [Request(rid=i, mesh=picks[i], v_t0=host[picks[i]][0], v_t1=host[picks[i]][1],
                        arrival_s=float(times[i]), seed=1000003 * i + 7) for i in range(n_req)]

    def engine(narrow):
        eng = ServeEngine(dev, config=cfg, slots=SERVE_SLOTS, max_group=SERVE_MAX_GROUP, narrow=narrow, top_k=4096,
                          memory_budget=int(args.serve_memory_gb * (1 << 30)))
        for key, s, excl in pool:
            eng.register_mesh(key, s, exclude_self=excl)
        warm = [Request(rid=-1 - i, mesh=k, v_t0=host[k][0], v_t1=host[k][1], arrival_s=0.0, seed=i)
                for i, k in enumerate(keys)]
        for _ in range(2):  # sizes every mesh's candidate state
            eng.run(warm)
        return eng

    sampler = ClockSampler(dev.index or 0)
    sampler.start()
    t_begin = time.time()
    out = {}
    for narrow in ("anyhit", "certify"):
        eng = engine(narrow)
        for _ in range(max(1, args.warmup // 2)):
            eng.run(stream(np.zeros(n_req))[: max(8, n_req // 8)])
        done, wall = _served_run(eng, stream(np.zeros(n_req)), torch)  # saturated: capacity
        st = eng.stats()
        cap = {"steps_per_s": n_req / wall, "candidates_per_s": sum(r.queries for r in done) / wall,
               "exact_calls_per_s": sum(r.calls for r in done) / wall, "wall_s": wall,
               "groups_run": st["groups"], "reruns": st["reruns"], "arena_peak_bytes": st["arena_peak"]}
        res = {"capacity": cap}
        if narrow == "anyhit":
            for tag, times in (("offered", arrivals),
                               ("sustainable", arrivals * max(1.0, args.serve_rate / (0.7 * cap["steps_per_s"])))):
                done_r, wall_r = _served_run(eng, stream(times), torch)
                tris = np.array([host[r.mesh][2] for r in done_r], dtype=np.float64)
                lat = np.array([r.latency_ms for r in done_r])
                per = lat / np.maximum(tris / 1e5, 1e-9)
                res[tag] = {"arrival_rate_per_s": n_req / float(times[-1]), "steps_per_s": n_req / wall_r,
                            **latency_stats(done_r),
                            "p50_ms_per_100k_tris": float(np.percentile(per, 50)),
                            "p99_ms_per_100k_tris": float(np.percentile(per, 99)),
                            "by_mesh": _latency_by_mesh(done_r, keys, host),
                            "admission_lag_p99_ms": float(np.percentile([r.admit_lag_ms for r in done_r], 99))}
        eng.close()
        out[narrow] = res
    t_end = time.time()
    clocks = sampler.stop((t_begin, t_end))
    # the plain path: each step alone, one at a time, every candidate certified
    plain_ms, ref_ms = {}, {}
    for key, s, excl in pool:
        if key not in picks:
            continue
        p = ScenePipeline(s, dev, exclude_self=excl, config=cfg)
        p.step_checked()
        p.fit_capacities()
        p.step_checked()
        ts = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p.v_t0.copy_(host[key][0], non_blocking=True)
            p.v_t1.copy_(host[key][1], non_blocking=True)
            p.step_checked()
            ts.append((time.perf_counter() - t0) * 1e3)
        plain_ms[key] = (statistics.median(ts), p.read_counts()[0] + p.read_counts()[1])
        if cpu_budget is not None:
            ref_ms[key] = _reference_gpu_step_ms(p, cfg)
        del p
    plain_s = sum(plain_ms[k][0] for k in picks) * 1e-3
    plain = {"steps_per_s": n_req / plain_s, "candidates_per_s": sum(plain_ms[k][1] for k in picks) / plain_s,
             "what": "each request alone, one at a time, through ScenePipeline.step_checked (single-scene broad "
                     "phase + certificates of every candidate, trajectories copied in from page-locked memory, "
                     "counts and summary read back: a host sync per step); per-mesh median of 3 steps, summed "
                     "over the stream's requests",
             "ms_per_step_by_mesh": {k: v[0] for k, v in plain_ms.items()}}
    block = {
        "workload": "serving stream: Poisson arrivals of CCD steps drawn uniformly from 9 meshes of the two-sphere, "
                    "rigid uneven-scene and cloth-on-sphere kinds (10k-600k triangles), through the native "
                    "continuous-batching server (p2c_serve_*): admission by slots and a device arena, one batched "
                    "candidate generation per group, then the scheduled any-hit with fallback replay (scores from "
                    "the seeded scheduler stub, top-K 4096) or certificates of every candidate",
        "requests": n_req, "offered_rate_per_s": args.serve_rate,
        "meshes": {k: int(host[k][2]) for k in keys}, "slots": SERVE_SLOTS, "max_group": SERVE_MAX_GROUP,
        "anyhit": out["anyhit"], "certify_all": out["certify"], "plain_path": plain,
        "served_over_plain": out["anyhit"]["capacity"]["steps_per_s"] / plain["steps_per_s"],
        "served_certify_all_over_plain": out["certify"]["capacity"]["steps_per_s"] / plain["steps_per_s"],
        "ratio_unit": "CCD steps/s on the same requests (capacity: every request arrives at once)",
        "e2e": "every served number is end to end: trajectories from page-locked host memory, summaries back",
        "clocks": clocks,
    }
    if cpu_budget is not None:
        block["cpu_baseline"] = _tool_serve_sample(pool, cfg, cpu_budget)
        if ref_ms and all(ref_ms.get(k) is not None for k in picks):
            ref_s = sum(ref_ms[k] for k in picks) * 1e-3
            ref = {"steps_per_s": n_req / ref_s, "queries_per_s": sum(plain_ms[k][1] for k in picks) / ref_s,
                   "ms_per_step_by_mesh": dict(ref_ms),
                   "what": "the reference's CUDA batch certifier (certificate_cuda.cu compiled unchanged for "
                           "sm_100a; host records in, malloc, copy, one thread per primitive, sync, copy back, "
                           "free per call) on every certificate query of each request (its candidates, generated "
                           "here: the reference has no GPU candidate generation), summed over the stream's "
                           "requests; certification only"}
            block["cpu_baseline"]["reference_gpu"] = ref
            block["served_over_reference_gpu"] = out["anyhit"]["capacity"]["steps_per_s"] / ref["steps_per_s"]
            block["served_certify_all_over_reference_gpu"] = (out["certify"]["capacity"]["steps_per_s"]
                                                              / ref["steps_per_s"])
    return block


def _latency_by_mesh(done, keys, host) -> dict:
    """p50 / p99 latency of each mesh's requests (its triangle count beside)."""
    import numpy as np

    out = {}
    for k in keys:
        lat = [r.latency_ms for r in done if r.mesh == k]
        if lat:
            out[k] = {"triangles": int(host[k][2]), "requests": len(lat), "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99))}
    return out


def _reference_gpu_step_ms(pipe, cfg) -> float | None:
    """Milliseconds the reference's CUDA batch path takes to certify every
    candidate of the pipeline's last step (median of 3), or None when that
    build is absent."""
    import oracle

    if not oracle.ref_cuda_available():
        return None
    vf, ee = pipe.materialize()
    run = lambda rec: oracle.ref_cuda_eval_batch(rec, 0.0, 1.0, cfg.eps_time, cfg.eps_space,
                                                 cfg.max_subdivision_depth) if len(rec) else None
    run(vf), run(ee)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        run(vf)
        run(ee)
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts) * 1e3


def run_serve(args) -> dict:
    import torch

    world, rank, local = _dist_setup(args)
    dev = torch.device("cuda", local if world > 1 else 0)
    blk = serve_bench(args, dev, rank, None if (args.no_cpu_baseline or rank != 0) else args.cpu_budget)
    cap = blk["anyhit"]["capacity"]
    value, ms = replica_rate(world, cap["candidates_per_s"] * cap["wall_s"], cap["wall_s"] * 1e3)
    if rank != 0:
        return None
    off = blk["anyhit"]["offered"]
    return {
        "metric": "served CCD candidates/s (every candidate decided: certified, or covered by its group's hit)",
        "value": value, "unit": "candidates/s", "n_gpus": world, "steps": 1, "warmup": args.warmup,
        "ms_per_step": ms, "p50_ms": off["p50_ms"], "p99_ms": off["p99_ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": blk["workload"], "requests_per_step": blk["requests"],
                   "arrival_rate_per_s": args.serve_rate, "parallelism": f"replicas x{world}",
                   "l2": "requests stream fresh trajectories from host memory"},
        "served": blk,
        "e2e": {"value": value, "unit": "candidates/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "what": blk["e2e"]},
        "gpu_launches": None, "roofline": None, "cpu_baseline": blk.get("cpu_baseline"), "clocks": blk["clocks"],
    }


PROXY_OBJECTS = 32  # rigid bodies of the proxy workload (--proxy-objects)
PROXY_PATCHES, PROXY_SEGMENTS, PROXY_SLABS = 200, 2, 4


def _proxy_input(objects: int, seed: int) -> dict:
    """The proxy-scene workload: ``objects`` rigid bodies of 200 patches in a
    box whose volume grows with the body count (constant density), 2 motion
    segments x 4 slabs each, rotating and drifting (swept AABBs and capsules)."""
    from p2cccd_b200 import scenes

    spread = 2.0 * (objects / 64.0) ** (1.0 / 3.0)
    return scenes.proxy_build_input(n_objects=objects, patches_per_object=PROXY_PATCHES, n_segments=PROXY_SEGMENTS,
                                    slabs=PROXY_SLABS, seed=seed, spread=spread)


def _proxy_config(inp: dict, n: int, raw: int, cand: int) -> dict:
    return {"workload": f"proxy-scene proposal data: {len(inp['objects'])} rigid bodies x {PROXY_PATCHES} patches x "
                        f"{PROXY_SEGMENTS} motion segments x {PROXY_SLABS} time slabs, bodies rotating and drifting "
                        "in a box of constant body density; BuildProxyScene (patch motion bounds, swept-AABB / "
                        "capsule proxies), raw hits and compacted candidates of the whole scene, density stats and "
                        "the 32-feature proposal rows of every candidate",
            "proxies_per_step": n, "raw_hits": raw, "candidates": cand, "objects": len(inp["objects"]),
            "seed": inp.get("seed")}


def _proxy_reference(inp: dict, budget_s: float) -> dict:
    """The reference's BuildProxyScene + GenerateRawCandidatesCpu +
    CompactRawCandidates + ComputeCandidateDensityStats +
    ExtractProposalFeatureRows (oracle/_ref, unchanged sources, 1 thread as
    written) on the same scene, whole scenes until budget_s has passed."""
    import oracle

    done, t0, runs = 0, time.perf_counter(), 0
    while True:
        sc = oracle.ref_build_proxy_scene(inp)
        oracle.ref_proposal_feature_rows(sc)
        done += sc["n"]
        runs += 1
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    return {"proxies": done, "seconds": el, "runs": runs}


def run_proxy(args) -> dict | None:
    import torch

    from p2cccd_b200.proxy import ProxyCandidates, ProxySceneBuild

    world, rank, local = _dist_setup(args)
    dev = torch.device("cuda", local if world > 1 else 0)
    inp = _proxy_input(PROXY_OBJECTS, 20261203 + rank)
    inp["seed"] = 20261203 + rank
    build = ProxySceneBuild(inp, dev, detail=False)
    scene = build.run_checked()
    cands = ProxyCandidates(scene, dev)
    raw, cand = cands.run_checked()
    n_raw, n_cand = len(raw), len(cand)
    cands.fit_capacity()  # buffers (and every sort over them) sized to the scene's hits
    cands.run_checked()

    def step():
        build.run()
        cands.run()
        cands.feature_rows_async()

    # end-to-end: patch arrays from pinned host memory in, counts and records back
    h_center = build.patch_center.cpu().pin_memory()
    h_radius = build.patch_radius.cpu().pin_memory()
    h_pid = build.patch_id.cpu().pin_memory()
    h_raw = torch.empty_like(cands.raw, device="cpu").pin_memory()
    h_cand = torch.empty_like(cands.cand, device="cpu").pin_memory()
    h_counts = torch.empty_like(cands.counts, device="cpu").pin_memory()
    cands.feature_rows()  # allocates the row buffers; checks the rows
    h_rows = torch.empty_like(cands.rows, device="cpu").pin_memory()

    def step_e2e():
        build.patch_center.copy_(h_center, non_blocking=True)
        build.patch_radius.copy_(h_radius, non_blocking=True)
        build.patch_id.copy_(h_pid, non_blocking=True)
        step()
        h_counts.copy_(cands.counts, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        nr, nc = int(h_counts[0]), int(h_counts[1])
        h_raw[:nr].copy_(cands.raw[:nr], non_blocking=True)
        h_cand[:nc].copy_(cands.cand[:nc], non_blocking=True)
        h_rows[:nc].copy_(cands.rows[:nc], non_blocking=True)

    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    sampler = ClockSampler(dev.index if world > 1 else 0)
    sampler.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _barrier(world)
    torch.cuda.synchronize()
    t_begin = time.time()
    times = time_steps(torch, step, args.steps, flush, stream)
    torch.cuda.synchronize()
    t_end = time.time()
    _barrier(world)
    clocks = sampler.stop((t_begin, t_end))
    for _ in range(max(1, args.warmup)):
        step_e2e()
    e2e_times = time_steps(torch, step_e2e, args.steps, flush, stream)
    # phases: build vs candidates
    ev = []
    for _ in range(args.steps):
        flush.fill_(1)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record()
        build.run()
        e[1].record()
        cands.run()
        e[2].record()
        cands.feature_rows_async()
        e[3].record()
        ev.append(e)
    torch.cuda.synchronize()
    build_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    cand_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    feat_ms = statistics.mean(e[2].elapsed_time(e[3]) for e in ev)
    n = build.n
    ms = statistics.mean(times)
    value, ms_max = replica_rate(world, n, ms)
    e2e_value, e2e_ms = replica_rate(world, n, statistics.mean(e2e_times))
    n_kernels, kernel_names = count_kernels(torch, step)
    peaks = _load_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hbm_src = "of measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "of fallback (6.65 TB/s)"
    n_patch = int(build.n_patch_entries)
    records = n // PROXY_PATCHES
    build_bytes = 36 * n_patch + 200 * records + 113 * n
    cand_bytes = 109 * n + 64 * n_raw + 80 * n_cand
    rl = {"bound": "hbm", "peak": hbm_peak, "unit": "GB/s", "traffic": None, "peak_source": hbm_src}
    cand_roof = dict(rl, kernel="proxy candidates (sorts, slab sweep, raw hits, compaction)",
                     achieved=cand_bytes / (cand_ms * 1e-3) / 1e9, frac=cand_bytes / (cand_ms * 1e-3) / 1e9 / hbm_peak,
                     algorithmic_bytes_per_step=cand_bytes,
                     bytes_per_unit="109 B read per proxy + 64 B per raw hit + 80 B per candidate written")
    build_roof = dict(rl, kernel="build_kernel (patch motion bounds and proxy bounds)",
                      achieved=build_bytes / (build_ms * 1e-3) / 1e9,
                      frac=build_bytes / (build_ms * 1e-3) / 1e9 / hbm_peak, algorithmic_bytes_per_step=build_bytes,
                      bytes_per_unit="36 B per patch + 200 B per slab record read, 113 B per proxy written")
    feat_bytes = 528 * n_cand
    feat_roof = dict(rl, kernel="proposal feature rows (density sorts, first-proxy lookup, rows_kernel)",
                     achieved=feat_bytes / (feat_ms * 1e-3) / 1e9, frac=feat_bytes / (feat_ms * 1e-3) / 1e9 / hbm_peak,
                     algorithmic_bytes_per_step=feat_bytes,
                     bytes_per_unit="80 B candidate + 2 x 96 B proxy read, 256 B row written per candidate")
    ranked = sorted(((cand_ms, cand_roof), (build_ms, build_roof), (feat_ms, feat_roof)), key=lambda x: -x[0])
    roofline, secondary = ranked[0][1], [r for _, r in ranked[1:]]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = _proxy_reference(inp, args.cpu_budget)
        cpu = {"value": r["proxies"] / r["seconds"], "unit": "proxies/s", "cores": 1, "kind": "reference",
               "sample": f"the same {n}-proxy scene, {r['runs']} whole run(s) of the reference build + all-pairs "
                         "candidates + compaction + density stats + feature rows (1 thread as written)"}
    if rank != 0:
        return None
    return {
        "metric": "proxy-scene proposal data: proxies/s", "value": value, "unit": "proxies/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "p50_ms": statistics.median(times), "p99_ms": sorted(times)[max(0, int(0.99 * len(times)) - 1)],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {**_proxy_config(inp, n, n_raw, n_cand),
                   "l2": f"flushed between timed steps ({L2_FLUSH_BYTES >> 20} MB write)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "proxies/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h_center.numel() * 8 + h_radius.numel() * 8 + h_pid.numel() * 4,
                "d2h_bytes_per_step": h_counts.numel() * 8 + 64 * n_raw + 80 * n_cand + 256 * n_cand},
        "gpu_launches": n_kernels * args.steps if n_kernels >= 0 else None,
        "kernels_per_step": kernel_names,
        "phases": {"build_ms": build_ms, "candidates_ms": cand_ms, "feature_rows_ms": feat_ms},
        "roofline": roofline, "roofline_secondary": secondary,
        "cpu_baseline": cpu, "clocks": clocks,
    }


GROUP_ROWS = 1_000_000  # rows of the candidate-group workload (--group-rows)
SERVE_SLOTS, SERVE_MAX_GROUP = 4, 16  # serving engine: groups in flight, requests per group
GROUP_CFG = {"threshold": 0.75, "limit": 3, "penalty": 0.22}  # the binding's defaults


def _groups_config(rows: dict, n_groups: int) -> dict:
    return {"workload": f"candidate-group interface: run_native_dense_group_exact_early_stop over "
                        f"{len(rows['query_id'])} candidate rows in {n_groups} query groups of log-uniform size "
                        f"1-256 (rows shuffled), 20% positive labels; uncertainty threshold 0.75, attempt limit 3, "
                        f"miss penalty 0.22 (the binding's defaults)",
            "rows_per_step": len(rows["query_id"]), "groups": n_groups}


def _groups_reference(rows: dict, budget_s: float) -> dict:
    """The reference's RunDenseGroupExactEarlyStop after its binding's row
    parse (oracle/_ref, unchanged sources, 1 thread as written), whole row
    sets until budget_s has passed."""
    import oracle

    done, runs, t0 = 0, 0, time.perf_counter()
    while True:
        oracle.ref_dense_group(rows, **GROUP_CFG)
        done += len(rows["query_id"])
        runs += 1
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    return {"rows": done, "seconds": el, "runs": runs}


def run_groups(args) -> dict | None:
    import numpy as np
    import torch

    from p2cccd_b200 import workloads
    from p2cccd_b200.dense_groups import DenseGroupEarlyStop, _ORDER, _query_bits, upload

    world, rank, local = _dist_setup(args)
    dev = torch.device("cuda", local if world > 1 else 0)
    rows = workloads.dense_group_rows(GROUP_ROWS, 20261203 + rank)
    n = len(rows["query_id"])
    qbits = _query_bits(rows["query_id"])
    tens = upload(rows, dev)
    runner = DenseGroupEarlyStop(n, dev)

    def step():
        runner.run(tens, n, query_bits=qbits, **GROUP_CFG)

    step()
    st = runner.result()
    n_groups = int(st["group_count"])
    host = {k: torch.from_numpy(rows[k].view(np.int64) if rows[k].dtype == np.uint64 else rows[k]).pin_memory()
            for k in _ORDER}
    h_stats = torch.empty_like(runner.stats, device="cpu").pin_memory()

    def step_e2e():  # rows from pinned host memory in, the stats back
        for k in _ORDER:
            tens[k].copy_(host[k], non_blocking=True)
        step()
        h_stats.copy_(runner.stats, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()

    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    sampler = ClockSampler(dev.index if world > 1 else 0)
    sampler.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _barrier(world)
    torch.cuda.synchronize()
    t_begin = time.time()
    times = time_steps(torch, step, args.steps, flush, stream)
    torch.cuda.synchronize()
    t_end = time.time()
    _barrier(world)
    clocks = sampler.stop((t_begin, t_end))
    for _ in range(max(1, args.warmup)):
        step_e2e()
    e2e_times = time_steps(torch, step_e2e, args.steps, flush, stream)
    ms = statistics.mean(times)
    value, ms_max = replica_rate(world, n, ms)
    e2e_value, e2e_ms = replica_rate(world, n, statistics.mean(e2e_times))
    n_kernels, kernel_names = count_kernels(torch, step)
    peaks = _load_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hbm_src = "of measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "of fallback (6.65 TB/s)"
    row_bytes = 128 * n  # query + candidate id, cost target, 8 trace doubles, 8 scores, 3 scores
    roofline = {"bound": "hbm", "peak": hbm_peak, "unit": "GB/s", "traffic": None, "peak_source": hbm_src,
                "kernel": "whole replay (parse, two stable sorts, gather, group walk, ordered folds)",
                "achieved": row_bytes / (ms * 1e-3) / 1e9, "frac": row_bytes / (ms * 1e-3) / 1e9 / hbm_peak,
                "algorithmic_bytes_per_step": row_bytes,
                "bytes_per_unit": "128 B per candidate row read once",
                "note": "the work totals are folded one term at a time in the reference's order "
                        "(bit-exact doubles): a dependent FP64 add chain per total"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = _groups_reference(rows, args.cpu_budget)
        cpu = {"value": r["rows"] / r["seconds"], "unit": "rows/s", "cores": 1, "kind": "reference",
               "sample": f"the same {n} rows, {r['runs']} whole run(s) of the binding's parse + "
                         "RunDenseGroupExactEarlyStop (1 thread as written)"}
    if rank != 0:
        return None
    return {
        "metric": "candidate-group early stop: rows/s", "value": value, "unit": "rows/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "p50_ms": statistics.median(times), "p99_ms": sorted(times)[max(0, int(0.99 * len(times)) - 1)],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {**_groups_config(rows, n_groups), "l2": f"flushed between timed steps ({L2_FLUSH_BYTES >> 20} MB write)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "rows/s", "ms_per_step": e2e_ms, "h2d_bytes_per_step": row_bytes,
                "d2h_bytes_per_step": int(h_stats.numel())},
        "gpu_launches": n_kernels * args.steps if n_kernels >= 0 else None,
        "kernels_per_step": kernel_names,
        "result": {"groups": n_groups, "learned_exact_calls": int(st["learned_exact_calls"]),
                   "learned_exact_work": float(st["learned_exact_work"]), "tp": int(st["tp"]), "fn": int(st["fn"])},
        "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
    }


BATCH_SCENES = 256  # scenes of the batch workload (--scenes)
BATCH_PARTITION = "replica"  # --partition: "replica" (each rank its own batch) or "lpt" (one batch split by LPT)
CLOTH_N = 513  # cloth grid of the cloth workload (--cloth-n; 513 = the dense-contact stress case)
AUTOTUNE_REPS = 3  # graph replays per autotuner trial of the batch workload (--autotune-reps; 0 = defaults)
REF_ARM_BUDGET_S = 150.0  # wall seconds of the whole reference arm (warm-up + timed steps)
REF_ARM_CAP_S = 600.0  # hard cap on a reference arm of whole steps (the scene tool's step is ~4 s)


def run_reference(args) -> dict | None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    import numpy as np

    import oracle
    from p2cccd_b200 import certify, scenes, workloads

    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libp2c_ref.so was not built"}
    if args.workload == "groups":
        from p2cccd_b200 import workloads as wl

        rows = wl.dense_group_rows(GROUP_ROWS, 20261203)
        budget = REF_ARM_BUDGET_S / max(1, args.steps + args.warmup)
        for _ in range(args.warmup):
            _groups_reference(rows, 0.0)
        runs = [_groups_reference(rows, budget) for _ in range(args.steps)]
        value = sum(r["rows"] for r in runs) / sum(r["seconds"] for r in runs)
        ms = sum(r["seconds"] for r in runs) / sum(r["runs"] for r in runs) * 1e3
        n_groups = int(oracle.ref_dense_group(rows, **GROUP_CFG)["group_count"])
        return {"metric": "candidate-group early stop: rows/s", "value": value, "unit": "rows/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": _groups_config(rows, n_groups), "impl": "reference",
                "cpu_baseline": {"value": value, "unit": "rows/s", "cores": 1, "kind": "reference",
                                 "sample": "whole row sets: the binding's row parse + RunDenseGroupExactEarlyStop, "
                                           "1 thread as written"},
                "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "proxy":
        inp = _proxy_input(PROXY_OBJECTS, 20261203)
        inp["seed"] = 20261203
        budget = REF_ARM_BUDGET_S / max(1, args.steps + args.warmup)
        for _ in range(args.warmup):
            _proxy_reference(inp, 0.0)
        runs = [_proxy_reference(inp, budget) for _ in range(args.steps)]
        n = sum(r["proxies"] for r in runs) / sum(r["runs"] for r in runs)
        value = sum(r["proxies"] for r in runs) / sum(r["seconds"] for r in runs)
        ms = sum(r["seconds"] for r in runs) / sum(r["runs"] for r in runs) * 1e3
        return {"metric": "proxy-scene proposal data: proxies/s", "value": value, "unit": "proxies/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {**_proxy_config(inp, int(n), -1, -1), "raw_hits": None, "candidates": None},
                "impl": "reference",
                "cpu_baseline": {"value": value, "unit": "proxies/s", "cores": 1, "kind": "reference",
                                 "sample": "whole scenes: BuildProxyScene + GenerateRawCandidatesCpu (all pairs) + "
                                           "CompactRawCandidates + ComputeCandidateDensityStats + "
                                           "ExtractProposalFeatureRows, 1 thread as written"},
                "e2e": {"value": value, "unit": "proxies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    threads = os.cpu_count() or 1
    cfg = certify.CertConfig(1e-6, 1e-6, 32)
    n_runs = max(1, args.steps + args.warmup)
    per_step_s = REF_ARM_BUDGET_S / n_runs  # wall time one step may take
    if args.workload == "plain":
        spec = workloads.PlainSpec()
        w = workloads.plain_queries(spec)
        nq = len(w["vf"]) + len(w["ee"])

        def step(i):
            t0 = time.perf_counter()
            for fam in ("vf", "ee"):
                oracle.ref_eval_batch(w[fam], 0.0, 1.0, cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth,
                                      threads=threads)
            return nq, time.perf_counter() - t0
        conf = {"workload": "plain exact CCD: 10,000 VF + 10,000 EE seeded FP64 queries"}
        sample = f"the full {nq}-query batch per step, {threads} threads over the reference certifier"
    elif args.workload == "scene" and args.scene_reference == "builder":
        scene = scenes.two_spheres()
        probe = SceneReferenceSample(scene, cfg, threads, 1)
        t0 = time.perf_counter()
        probe.run(0)
        n_slices = max(1, int(np.ceil((time.perf_counter() - t0) / per_step_s)))
        ref = SceneReferenceSample(scene, cfg, threads, n_slices)

        def step(i):
            q, b, c = ref.run(i)
            return q, b + c
        conf = {"workload": "single-scene broad+narrow: two 40,960-triangle UV spheres, translation-only form "
                            "(the reference mesh builder takes rigid translations only); EXTRAPOLATED from slices"}
        sample = ref.describe() + "; one slice per step"
    elif args.workload == "scene":
        scene = scenes.two_spheres()
        ref = ToolSceneStep(scene, cfg)

        def step(i):
            return ref.run()
        conf = scene_config(scene, cfg)
        threads = 1
        sample = None  # filled from the tool's last step
    elif args.workload in ("batch", "serve"):
        if args.workload == "batch":
            batch = scenes.uneven_batch(BATCH_SCENES)
            excl = [True] * len(batch)
        else:
            pool = _serve_pool(20261203)
            batch = [s for _, s, _ in pool]
            excl = [e for _, _, e in pool]
        by_size = sorted(range(len(batch)), key=lambda i: len(batch[i]["faces"]))
        chosen, spent = [], 0.0
        for i in by_size:  # smallest scenes first while their mean tool time fits the per-step budget
            r = _batch_reference_sample(batch, cfg, 0.0, order=[i], exclude_self=excl[i])
            if chosen and (spent + r["seconds"]) / (len(chosen) + 1) > per_step_s:
                break
            chosen.append(i)
            spent += r["seconds"]

        def step(i):
            j = chosen[i % len(chosen)]
            r = _batch_reference_sample(batch, cfg, 0.0, order=[j], exclude_self=excl[j])
            return r["queries"], r["seconds"]
        conf = {"workload": ("batched uneven scenes: 256 two-UV-sphere scenes, 1k-200k triangles"
                             if args.workload == "batch" else
                             "serving stream of mixed CCD steps (two spheres, rigid scenes, cloth), 10k-600k "
                             "triangles") + " (the reference scene tool, one scene per step)"}
        sample = (f"reference scene tool (SweepPairs candidates + RunAllExactRows, 1 thread as written), one whole "
                  f"scene per step cycling over the {len(chosen)} smallest scenes of the {args.workload} (up to "
                  f"{len(batch[chosen[-1]]['faces'])} triangles) whose mean step fits {per_step_s * 1e3:.0f} ms")
        threads = 1
    else:
        tool, n = None, None
        for cand in (17, 33, 65, 129, 257):  # largest instance whose step fits the per-step wall budget
            s_c = scenes.cloth_on_sphere(n=cand, sphere_lon=max(8, cand // 2), sphere_rings=max(6, (cand * 2) // 5))
            t_c = oracle.RefToolScene(s_c["v_t0"], s_c["v_t1"], s_c["faces"], 0.0, False)
            t0 = time.perf_counter()
            t_c.time_step(4096, cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth)
            if tool is not None and time.perf_counter() - t0 > per_step_s:
                break
            tool, n, n_tris = t_c, cand, len(s_c["faces"])

        def step(i):
            r = tool.time_step(4096, cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth)
            return r["calls"], r["candidates_s"] + r["anyhit_vf_s"] + r["anyhit_ee_s"]
        conf = {"workload": "dense-contact stress: cloth draped onto a UV sphere, self pairs, scheduled any-hit "
                            "with fallback replay (the reference scene tool)"}
        sample = (f"reference scene tool (SweepPairs candidates + RunScheduledAnyHitRows, 1 thread as written) on "
                  f"the {n} x {n} cloth instance ({n_tris} triangles; the full instance has 624,288), the largest "
                  f"whose step fits {per_step_s * 1e3:.0f} ms of wall time")
        threads = 1
    t_arm = time.perf_counter()
    for i in range(args.warmup):
        step(i)
    times, qs = [], []
    for i in range(args.steps):
        q, sec = step(args.warmup + i)
        times.append(sec)
        qs.append(q)
        if time.perf_counter() - t_arm > REF_ARM_CAP_S:
            break  # bounded run: the line reports how many steps were timed
    ms = statistics.mean(times) * 1e3
    value = sum(qs) / sum(times)
    if sample is None:
        sample = ref.describe() + f"; {len(times)} whole step(s) timed"
    line = {"metric": "certified CCD queries/s", "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": conf,
            "queries_per_step": statistics.mean(qs), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if len(times) < args.steps:
        line["steps_requested"] = args.steps
    return line


def _host_cpu() -> dict:
    """The host's CPU model and hardware threads (for the CPU baseline)."""
    model = ""
    try:
        with open("/proc/cpuinfo", encoding="utf-8") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model or None, "host_threads": os.cpu_count()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--workload", default="scene", choices=sorted(WORKLOADS) + ["serve", "proxy", "groups"])
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=10.0, help="seconds of reference CPU work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scenes", type=int, default=256, help="batch: number of scenes")
    ap.add_argument("--cloth-n", type=int, default=513, help="cloth: grid vertices per side (513 = the stress config)")
    ap.add_argument("--autotune-reps", type=int, default=3,
                    help="batch: graph replays per autotuner trial (0: the library's default launch shape)")
    ap.add_argument("--partition", default="replica", choices=["replica", "lpt"],
                    help="batch with --gpus N: every rank its own batch (weak scaling) or one batch packed onto the "
                         "ranks longest-processing-time first by triangle count (strong scaling)")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="serving: mean arrivals per second")
    ap.add_argument("--serve-requests", type=int, default=400, help="serving: requests per stream")
    ap.add_argument("--serve-memory-gb", type=float, default=32.0, help="serving: the server's device arena (GB)")
    ap.add_argument("--no-served", action="store_true", help="scene: leave out the serving block")
    ap.add_argument("--proxy-objects", type=int, default=32, help="proxy: rigid bodies of 200 patches x 8 slabs")
    ap.add_argument("--group-rows", type=int, default=1_000_000, help="groups: candidate rows per step")
    ap.add_argument("--serve-slots", type=int, default=4, help="serving: request groups in flight")
    ap.add_argument("--serve-max-group", type=int, default=16, help="serving: requests admitted per group")
    ap.add_argument("--scene-reference", default="tool", choices=["tool", "builder"],
                    help="reference arm of the scene: the scene tool's own SweepPairs path on the identical scene "
                         "(default) or the translation-only mesh builder, extrapolated from slices")
    ap.add_argument("--benchmark-rows", default=None, metavar="DIR",
                    help="also write the run as BenchmarkRowV2 JSONL / CSV (the reference's export schema) to DIR")
    args = ap.parse_args()
    global BATCH_SCENES, AUTOTUNE_REPS, CLOTH_N, PROXY_OBJECTS, GROUP_ROWS, SERVE_SLOTS, SERVE_MAX_GROUP
    global BATCH_PARTITION
    BATCH_PARTITION = args.partition
    PROXY_OBJECTS = max(2, args.proxy_objects)
    SERVE_SLOTS, SERVE_MAX_GROUP = max(1, args.serve_slots), max(1, args.serve_max_group)
    GROUP_ROWS = max(1, args.group_rows)
    BATCH_SCENES, AUTOTUNE_REPS = max(1, args.scenes), max(0, args.autotune_reps)
    CLOTH_N = max(9, args.cloth_n)
    if args.impl == "reference":
        line = run_reference(args)
    elif args.workload == "serve":
        line = run_serve(args)
    elif args.workload == "proxy":
        line = run_proxy(args)
    elif args.workload == "groups":
        line = run_groups(args)
    else:
        line = run_b200(args)
    if line is not None:
        if isinstance(line.get("cpu_baseline"), dict):
            line["cpu_baseline"].update(_host_cpu())
        print(json.dumps(line), flush=True)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and args.impl == "b200":
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
