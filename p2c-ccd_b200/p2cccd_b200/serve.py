"""Serving: continuous batching of CCD steps on one GPU.

A thin host layer over the library's native server (``p2c_serve_*`` in
``include/p2c_b200.h``): the runtime that admits requests, sizes groups by
device memory, drives one CUDA stream per slot and retires groups by event is
C++ inside the library; this module registers meshes, feeds a stream of
requests at their arrival times and collects the results.

A request is one CCD step of a registered mesh: its vertex trajectories over
the step in page-locked host memory.  The server keeps meshes and their
candidate state resident on the device and owns one device arena (allocated
at creation); requests that arrive while others run are admitted, in order,
as slots and arena ranges free up, and the groups on different slots overlap
on the device.  Each group is one batched candidate generation and then
either the certificates of every candidate (``narrow="certify"``) or the
scheduled any-hit with fallback replay (``narrow="anyhit"``): per object-pair
group, the top-K candidates by the scheduler's scores until the first hit,
then every other candidate of groups without a hit.  Scores come from the
seeded scheduler stub, keyed by candidate identity, so a step gets the same
answer alone and in any mix.  Latency is the device clock from the request's
admission to its group's completion, plus the host's admission lag behind
the nominal arrival time.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .anyhit import ANYHIT_SUMMARY_DTYPE
from .certify import CertConfig
from .records import INTERVAL_RESULT_DTYPE, QUERY_CERTIFICATE_DTYPE
from .scene import SUMMARY_DTYPE

NARROW = {"certify": 0, "anyhit": 1}


class ServeConfigC(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int32), ("max_group", ctypes.c_int32), ("narrow", ctypes.c_int32),
                ("top_k", ctypes.c_int32), ("memory_budget", ctypes.c_int64), ("undecided_capacity", ctypes.c_int64),
                ("cert", _lib.CertConfig), ("interval_t0", ctypes.c_double), ("interval_t1", ctypes.c_double)]


class ServeMeshC(ctypes.Structure):
    _fields_ = [("faces", ctypes.c_void_p), ("edges", ctypes.c_void_p), ("v_obj", ctypes.c_void_p),
                ("f_obj", ctypes.c_void_p), ("e_obj", ctypes.c_void_p), ("nv", ctypes.c_int64),
                ("nf", ctypes.c_int64), ("ne", ctypes.c_int64), ("n_obj", ctypes.c_int32),
                ("exclude_self", ctypes.c_int32), ("thickness", ctypes.c_double), ("vf_capacity", ctypes.c_int64),
                ("ee_capacity", ctypes.c_int64)]


class ServeRequestC(ctypes.Structure):
    _fields_ = [("mesh_id", ctypes.c_int32), ("pad", ctypes.c_int32), ("v_t0", ctypes.c_void_p),
                ("v_t1", ctypes.c_void_p), ("seed", ctypes.c_uint64), ("vf_results", ctypes.c_void_p),
                ("ee_results", ctypes.c_void_p), ("results_cap", ctypes.c_int64), ("undecided", ctypes.c_void_p),
                ("undecided_cap", ctypes.c_int64), ("group_detected", ctypes.c_void_p),
                ("groups_cap", ctypes.c_int64)]


SERVE_RESULT_DTYPE = np.dtype({
    "names": ["request_id", "status", "reruns", "latency_ms", "vf_candidates", "ee_candidates", "undecided_entries",
              "truncated", "certify", "anyhit"],
    "formats": ["<i8", "<i4", "<i4", "<f8", "<u8", "<u8", "<u8", "<u8", SUMMARY_DTYPE, (ANYHIT_SUMMARY_DTYPE, 2)],
    "offsets": [0, 8, 12, 16, 24, 32, 40, 48, 56, 168],
    "itemsize": 312,
})

SERVE_STATS_DTYPE = np.dtype([(k, "<u8") for k in (
    "admitted", "completed", "failed", "groups", "reruns", "pending", "in_flight", "candidates", "calls",
    "arena_bytes", "arena_in_use", "arena_peak")])


@dataclass
class Mesh:
    key: str
    mesh_id: int
    nv: int
    nf: int
    ne: int
    n_obj: int
    triangles: int


@dataclass
class Request:
    rid: int
    mesh: str
    v_t0: torch.Tensor  # page-locked host (nv, 3) float64
    v_t1: torch.Tensor
    arrival_s: float  # seconds after serving starts
    keep_results: bool = False
    seed: int = 0
    # filled by the engine
    status: int | None = None
    summary: dict | None = None          # certify: the Evaluate reduction of its candidates
    anyhit: dict | None = None           # any-hit: {"vf": summary, "ee": summary}
    results: tuple[np.ndarray, np.ndarray] | None = None
    undecided: np.ndarray | None = None  # certify: (family, pair position) of undecided certificates
    groups: tuple[np.ndarray, np.ndarray] | None = None  # any-hit: detected flags per object pair, VF and EE
    latency_ms: float | None = None
    admit_lag_ms: float = 0.0
    reruns: int = 0
    queries: int = 0                     # candidates of the step
    calls: int = 0                       # certificates the procedure called
    _out: dict = field(default_factory=dict)


class ServeEngine:
    """A native continuous-batching server (``p2c_serve_create``) on one GPU."""

    def __init__(self, device: str | torch.device = "cuda", *, config: CertConfig = CertConfig(),
                 interval: tuple[float, float] = (0.0, 1.0), slots: int = 4, max_group: int = 16,
                 memory_budget: int | None = None, narrow: str = "anyhit", top_k: int = 4096,
                 undecided_capacity: int = 1 << 14):
        if narrow not in NARROW:
            raise ValueError("narrow must be 'certify' or 'anyhit'")
        self.lib = _lib.load()
        self.device = torch.device(device)
        torch.cuda.set_device(self.device)
        self.config = config
        self.narrow = narrow
        self.interval = (float(interval[0]), float(interval[1]))
        cfg = ServeConfigC()
        cfg.slots, cfg.max_group, cfg.narrow, cfg.top_k = int(slots), int(max_group), NARROW[narrow], int(top_k)
        cfg.memory_budget = int(memory_budget or 0)
        cfg.undecided_capacity = int(undecided_capacity)
        cfg.cert = config.c()
        cfg.interval_t0, cfg.interval_t1 = self.interval
        self._cfg = cfg
        self._h = ctypes.c_void_p()
        _lib.check(self.lib.p2c_serve_create(ctypes.byref(cfg), ctypes.byref(self._h)))
        self.meshes: dict[str, Mesh] = {}
        self._keep: list = []  # host arrays of requests in flight
        self.done: list[Request] = []

    def close(self) -> None:
        if self._h:
            self.lib.p2c_serve_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- registration -----------------------------------------------------
    def register_mesh(self, key: str, scene: dict, *, exclude_self: bool = True, thickness: float = 0.0,
                      vf_capacity: int | None = None, ee_capacity: int | None = None) -> Mesh:
        arrs = {k: np.ascontiguousarray(scene[k], np.int32) for k in ("faces", "edges", "v_obj", "f_obj", "e_obj")}
        n_obj = int(max(arrs["v_obj"].max(initial=-1), arrs["f_obj"].max(initial=-1), arrs["e_obj"].max(initial=-1))
                    + 1)
        m = ServeMeshC()
        for k, a in arrs.items():
            setattr(m, k, a.ctypes.data if a.size else None)
        m.nv, m.nf, m.ne = len(scene["v_t0"]), len(arrs["faces"]), len(arrs["edges"])
        m.n_obj, m.exclude_self, m.thickness = max(1, n_obj), 1 if exclude_self else 0, float(thickness)
        m.vf_capacity, m.ee_capacity = int(vf_capacity or 0), int(ee_capacity or 0)
        mid = ctypes.c_int32(-1)
        _lib.check(self.lib.p2c_serve_register_mesh(self._h, ctypes.byref(m), ctypes.byref(mid)))
        mesh = Mesh(key, mid.value, m.nv, m.nf, m.ne, m.n_obj, m.nf)
        self.meshes[key] = mesh
        return mesh

    # -- requests ---------------------------------------------------------
    def admit(self, r: Request) -> int:
        """The request arrives now: queue it for admission; returns its id."""
        m = self.meshes[r.mesh]
        if not (r.v_t0.is_pinned() and r.v_t1.is_pinned()):
            raise ValueError("request trajectories must be page-locked host tensors")
        if r.v_t0.dtype != torch.float64 or tuple(r.v_t0.shape) != (m.nv, 3) or r.v_t1.shape != r.v_t0.shape:
            raise ValueError(f"request trajectories must be ({m.nv}, 3) float64")
        q = ServeRequestC()
        q.mesh_id, q.v_t0, q.v_t1, q.seed = m.mesh_id, r.v_t0.data_ptr(), r.v_t1.data_ptr(), int(r.seed) & (2**64 - 1)
        out = {}
        if r.keep_results:
            if self.narrow == "certify":
                cap = 16 * m.nf + 16 * m.ne + 4096
                out["vf"] = np.zeros(cap, dtype=INTERVAL_RESULT_DTYPE)
                out["ee"] = np.zeros(cap, dtype=INTERVAL_RESULT_DTYPE)
                out["uq"] = np.zeros(cap, dtype=np.uint64)
                q.vf_results, q.ee_results, q.results_cap = out["vf"].ctypes.data, out["ee"].ctypes.data, cap
                q.undecided, q.undecided_cap = out["uq"].ctypes.data, cap
            else:
                g = 2 * m.n_obj * m.n_obj
                out["groups"] = np.zeros(g, dtype=np.uint8)
                q.group_detected, q.groups_cap = out["groups"].ctypes.data, g
        r._out = out
        rid = ctypes.c_int64(-1)
        _lib.check(self.lib.p2c_serve_admit(self._h, ctypes.byref(q), ctypes.byref(rid)))
        return rid.value

    def poll(self, max_results: int = 256) -> np.ndarray:
        res = np.zeros(max_results, dtype=SERVE_RESULT_DTYPE)
        n = ctypes.c_int32(0)
        _lib.check(self.lib.p2c_serve_poll(self._h, res.ctypes.data, max_results, ctypes.byref(n)))
        return res[:n.value]

    def stats(self) -> dict:
        st = np.zeros(1, dtype=SERVE_STATS_DTYPE)
        _lib.check(self.lib.p2c_serve_read_stats(self._h, st.ctypes.data))
        return {k: int(st[0][k]) for k in SERVE_STATS_DTYPE.names}

    def _finish(self, r: Request, x) -> None:
        r.status = int(x["status"])
        r.reruns = int(x["reruns"])
        if r.status != 0:
            return
        r.latency_ms = float(x["latency_ms"]) + r.admit_lag_ms
        n_vf, n_ee = int(x["vf_candidates"]), int(x["ee_candidates"])
        r.queries = n_vf + n_ee
        if self.narrow == "certify":
            s = x["certify"]
            d = {k: int(s[k]) for k in SUMMARY_DTYPE.names if k != "query"}
            d["query"] = {k: s["query"][k].item() for k in QUERY_CERTIFICATE_DTYPE.names}
            r.summary = d
            r.calls = r.queries
            if r.keep_results:
                if int(x["truncated"]):
                    raise _lib.P2CError(f"request {r.rid}: outputs truncated ({int(x['truncated'])})")
                raw = lambda a, n: a.view(np.uint8).reshape(-1, 72)[:n].copy().view(INTERVAL_RESULT_DTYPE).reshape(-1)
                r.results = (raw(r._out["vf"], n_vf), raw(r._out["ee"], n_ee))  # bytes as written, padding too
                u = r._out["uq"][:int(x["undecided_entries"])]
                r.undecided = np.stack([(u >> np.uint64(63)).astype(np.int64) + 1,
                                        (u & np.uint64((1 << 63) - 1)).astype(np.int64)], 1)
        else:
            a = x["anyhit"]
            r.anyhit = {name: {k: int(a[f][k]) for k in ANYHIT_SUMMARY_DTYPE.names}
                        for f, name in ((0, "vf"), (1, "ee"))}
            r.calls = sum(v["proposal_calls"] + v["fallback_calls"] for v in r.anyhit.values())
            if r.keep_results:
                g = self.meshes[r.mesh].n_obj ** 2
                r.groups = (r._out["groups"][:g].copy(), r._out["groups"][g:].copy())
        r._out = {}

    def run(self, requests: list[Request], idle_sleep_s: float = 2e-5) -> list[Request]:
        """Serve requests (arrival_s relative to the start) to completion:
        each is admitted when its arrival time has passed, and the server is
        polled in between.  Returns the finished requests."""
        order = sorted(requests, key=lambda r: r.arrival_s)
        by_id: dict[int, Request] = {}
        done: list[Request] = []
        i = 0
        t0 = time.perf_counter()
        while len(done) < len(order):
            now = time.perf_counter() - t0
            while i < len(order) and order[i].arrival_s <= now:
                r = order[i]
                r.admit_lag_ms = max(0.0, (time.perf_counter() - t0 - r.arrival_s) * 1e3)
                by_id[self.admit(r)] = r
                i += 1
            got = self.poll()
            for x in got:
                r = by_id.pop(int(x["request_id"]))
                self._finish(r, x)
                if r.status != 0:
                    raise _lib.P2CError(f"request {r.rid} failed with status {r.status}: "
                                        f"{self.lib.p2c_last_error().decode()}")
                done.append(r)
            if not len(got):
                time.sleep(idle_sleep_s)
        self.done = done
        return done


def latency_stats(done: list[Request]) -> dict:
    lat = np.array([r.latency_ms for r in done], dtype=np.float64)
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}
