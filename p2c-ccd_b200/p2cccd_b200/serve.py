"""Serving: continuous batching of CCD steps on one GPU.

A ``ServeEngine`` keeps registered meshes (topology, object ids) and their
candidate state (the last candidate counts, which size the pair buffers)
resident on the GPU.  Requests are CCD steps of one registered mesh (its
vertex trajectories over the step, in pinned host memory) that arrive over
time.  ``pump`` admits arrived requests in arrival order while a slot is free
and the device memory the in-flight requests hold stays under the budget;
the requests admitted together form one group on the slot's own CUDA stream:

    host -> device copies of the trajectories,
    swept-AABB candidates of every request in one batched launch sequence
    (p2c_batch_candidates),
    ONE certification launch over the whole group (p2c_batch_certify), its
    undecided certificates appended to the group's fallback-replay queue,
    device -> host copies of the per-request summaries (and certificates),
    a completion event.

Groups on different slots overlap on the device, so requests that arrive
while others run are admitted as soon as a slot and memory free up.  A
request whose candidates outgrew its buffer is re-run with a larger one (its
mesh's candidate state grows), so every result is the complete certification
of the step: the same certificates as the request alone would get.
Latency is measured on the device clock from the request's arrival (placed
on the device timeline through an event recorded when serving starts) to the
completion event of its group.
"""
from __future__ import annotations

import collections
import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .batch import BATCH_SCENE_DTYPE, BatchTuning, scene_row
from .certify import CertConfig
from .records import INTERVAL_RESULT_DTYPE, QUERY_CERTIFICATE_DTYPE
from .scene import SUMMARY_DTYPE, SceneStruct


@dataclass
class Mesh:
    """A registered mesh: topology resident on the device plus its candidate state."""
    key: str
    nv: int
    nf: int
    ne: int
    faces: torch.Tensor
    edges: torch.Tensor
    v_obj: torch.Tensor
    f_obj: torch.Tensor
    e_obj: torch.Tensor
    n_obj: int
    exclude_self: bool
    thickness: float
    vf_cap: int
    ee_cap: int


@dataclass
class Request:
    rid: int
    mesh: str
    v_t0: torch.Tensor  # pinned host (nv, 3) float64
    v_t1: torch.Tensor
    arrival_s: float  # seconds after serving starts
    keep_results: bool = False
    # filled by the engine
    summary: dict | None = None
    results: tuple[np.ndarray, np.ndarray] | None = None
    undecided: np.ndarray | None = None  # (family, pair position) of undecided certificates (fallback replay)
    latency_ms: float | None = None
    reruns: int = 0
    queries: int = 0


@dataclass
class _Group:
    requests: list
    slot: int
    event: torch.cuda.Event
    bytes: int
    tensors: dict = field(default_factory=dict)


def _request_bytes(m: Mesh) -> int:
    """Device bytes one in-flight request holds: trajectories, pairs,
    certificates, and its share of the batched candidate workspace (about
    150 bytes per primitive plus 16 per pair slot)."""
    prims = m.nv + m.nf + m.ne
    return 48 * m.nv + (8 + 72) * (m.vf_cap + m.ee_cap) + 150 * prims + 16 * (m.vf_cap + m.ee_cap) + 4096


class ServeEngine:
    def __init__(self, device: str | torch.device = "cuda", *, config: CertConfig = CertConfig(),
                 interval: tuple[float, float] = (0.0, 1.0), slots: int = 4, max_group: int = 16,
                 memory_budget: int | None = None, tuning: BatchTuning | None = None,
                 undecided_capacity: int = 1 << 14):
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.config = config
        self.cfg_c = config.c()
        self.interval = (float(interval[0]), float(interval[1]))
        self.slots = max(1, int(slots))
        self.max_group = max(1, int(max_group))
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            memory_budget = int(free * 0.5)
        self.memory_budget = int(memory_budget)
        self.tuning = tuning if tuning is not None else BatchTuning(0, 0, 0, 0)
        self.undecided_capacity = max(1, int(undecided_capacity))
        self.meshes: dict[str, Mesh] = {}
        self.streams = [torch.cuda.Stream(self.device) for _ in range(self.slots)]
        self.busy: list[_Group | None] = [None] * self.slots
        self.pending: collections.deque = collections.deque()
        self.done: list[Request] = []
        self.in_flight_bytes = 0
        self.t0_event = None
        self.t0_host = None
        self.groups_run = 0

    # -- registration -----------------------------------------------------
    def register_mesh(self, key: str, scene: dict, *, exclude_self: bool = True, thickness: float = 0.0,
                      vf_capacity: int | None = None, ee_capacity: int | None = None) -> Mesh:
        d = self.device
        nf = len(scene["faces"])
        m = Mesh(key=key, nv=len(scene["v_t0"]), nf=nf, ne=len(scene["edges"]),
                 faces=torch.as_tensor(np.ascontiguousarray(scene["faces"], np.int32)).to(d),
                 edges=torch.as_tensor(np.ascontiguousarray(scene["edges"], np.int32)).to(d),
                 v_obj=torch.as_tensor(np.ascontiguousarray(scene["v_obj"], np.int32)).to(d),
                 f_obj=torch.as_tensor(np.ascontiguousarray(scene["f_obj"], np.int32)).to(d),
                 e_obj=torch.as_tensor(np.ascontiguousarray(scene["e_obj"], np.int32)).to(d),
                 n_obj=int(max(np.max(scene["v_obj"], initial=-1), np.max(scene["f_obj"], initial=-1),
                               np.max(scene["e_obj"], initial=-1)) + 1),
                 exclude_self=bool(exclude_self), thickness=float(thickness),
                 vf_cap=int(vf_capacity or max(1024, nf // 2)), ee_cap=int(ee_capacity or max(1024, nf)))
        self.meshes[key] = m
        return m

    # -- requests ---------------------------------------------------------
    def start(self) -> None:
        """Start the serving clock (request arrival times count from here)."""
        self.t0_event = torch.cuda.Event(enable_timing=True)
        self.t0_event.record(torch.cuda.current_stream(self.device))
        self.t0_host = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0_host

    def submit(self, req: Request) -> None:
        if req.mesh not in self.meshes:
            raise KeyError(f"mesh {req.mesh!r} is not registered")
        self.pending.append(req)

    def _admit(self) -> list[Request]:
        now = self.now()
        group, nbytes = [], 0
        while self.pending and len(group) < self.max_group:
            r = self.pending[0]
            if r.arrival_s > now:
                break
            b = _request_bytes(self.meshes[r.mesh])
            over = self.in_flight_bytes + nbytes + b > self.memory_budget
            if over and (group or self.in_flight_bytes > 0):
                break  # wait for memory to free up (a lone request is always admitted)
            group.append(self.pending.popleft())
            nbytes += b
        return group, nbytes

    def _launch(self, slot: int, group: list[Request], nbytes: int) -> None:
        d = self.device
        stream = self.streams[slot]
        stream.wait_stream(torch.cuda.current_stream(d))
        g = _Group(requests=group, slot=slot, event=torch.cuda.Event(enable_timing=True), bytes=nbytes)
        n = len(group)
        table = np.zeros(n, dtype=BATCH_SCENE_DTYPE)
        with torch.cuda.stream(stream):
            counts = torch.zeros((n, 4), dtype=torch.int64, device=d)
            keep = []
            for i, r in enumerate(group):
                m = self.meshes[r.mesh]
                v0 = torch.empty((m.nv, 3), dtype=torch.float64, device=d)
                v1 = torch.empty((m.nv, 3), dtype=torch.float64, device=d)
                v0.copy_(r.v_t0, non_blocking=True)
                v1.copy_(r.v_t1, non_blocking=True)
                vf = torch.empty(m.vf_cap, dtype=torch.int64, device=d)
                ee = torch.empty(m.ee_cap, dtype=torch.int64, device=d)
                rvf = torch.empty((m.vf_cap, 72), dtype=torch.uint8, device=d)
                ree = torch.empty((m.ee_cap, 72), dtype=torch.uint8, device=d)
                st = SceneStruct()
                st.v_t0, st.v_t1 = v0.data_ptr(), v1.data_ptr()
                st.faces, st.edges = m.faces.data_ptr(), m.edges.data_ptr()
                st.v_obj, st.f_obj, st.e_obj = m.v_obj.data_ptr(), m.f_obj.data_ptr(), m.e_obj.data_ptr()
                st.nv, st.nf, st.ne = m.nv, m.nf, m.ne
                st.thickness = m.thickness
                st.exclude_self = 1 if m.exclude_self else 0
                st.n_obj = m.n_obj
                table[i] = scene_row(st, vf.data_ptr(), ee.data_ptr(), m.vf_cap, m.ee_cap, counts.data_ptr() + 32 * i,
                                     rvf.data_ptr(), ree.data_ptr())
                keep.append((v0, v1, vf, ee, rvf, ree, None, (m.vf_cap, m.ee_cap)))
            h_table = torch.from_numpy(table.view(np.uint8).copy()).pin_memory()
            d_table = torch.empty_like(h_table, device=d)
            d_table.copy_(h_table, non_blocking=True)
            # every request's candidates in one batched launch sequence
            ws_bb = torch.empty(int(self.lib.p2c_batch_candidates_workspace_bytes(table.ctypes.data, n)),
                                dtype=torch.uint8, device=d)
            _lib.check(self.lib.p2c_batch_candidates(table.ctypes.data, d_table.data_ptr(), n, ws_bb.data_ptr(),
                                                     ws_bb.numel(), stream.cuda_stream))
            summaries = torch.empty((n, SUMMARY_DTYPE.itemsize), dtype=torch.uint8, device=d)
            ws_cert = torch.empty(int(self.lib.p2c_batch_certify_workspace_bytes(n)), dtype=torch.uint8, device=d)
            uq = torch.empty(self.undecided_capacity, dtype=torch.int64, device=d)
            _lib.check(self.lib.p2c_batch_certify(
                d_table.data_ptr(), n, self.interval[0], self.interval[1], ctypes.byref(self.cfg_c), 3,
                summaries.data_ptr(), uq.data_ptr(), self.undecided_capacity, ctypes.addressof(self.tuning),
                ws_cert.data_ptr(), ws_cert.numel(), stream.cuda_stream))
            h_sum = torch.empty(summaries.shape, dtype=torch.uint8).pin_memory()
            h_cnt = torch.empty(counts.shape, dtype=torch.int64).pin_memory()
            h_uq = torch.empty(uq.shape, dtype=torch.int64).pin_memory()
            h_sum.copy_(summaries, non_blocking=True)
            h_cnt.copy_(counts, non_blocking=True)
            h_uq.copy_(uq, non_blocking=True)
            h_res = []
            for r, k in zip(group, keep):
                if r.keep_results:
                    a = torch.empty(k[4].shape, dtype=torch.uint8).pin_memory()
                    b = torch.empty(k[5].shape, dtype=torch.uint8).pin_memory()
                    a.copy_(k[4], non_blocking=True)
                    b.copy_(k[5], non_blocking=True)
                    h_res.append((a, b))
                else:
                    h_res.append(None)
            g.event.record(stream)
        g.tensors = {"keep": keep, "h_table": h_table, "d_table": d_table, "summaries": summaries, "ws": ws_cert,
                     "ws_bb": ws_bb,
                     "counts": counts, "h_sum": h_sum, "h_cnt": h_cnt, "h_res": h_res, "uq": uq, "h_uq": h_uq}
        self.busy[slot] = g
        self.in_flight_bytes += nbytes
        self.groups_run += 1

    def _complete(self, slot: int) -> None:
        g = self.busy[slot]
        self.busy[slot] = None
        self.in_flight_bytes -= g.bytes
        t_done = self.t0_event.elapsed_time(g.event)  # ms after serving started
        cnt = g.tensors["h_cnt"].numpy()
        summ = g.tensors["h_sum"].numpy().reshape(-1).view(SUMMARY_DTYPE)
        n_uq = min(int(sum(int(x["undecided_queued"]) for x in summ)), self.undecided_capacity)
        uq = g.tensors["h_uq"].numpy()[:n_uq].view(np.uint64)
        uq_scene = (uq >> np.uint64(40)).astype(np.int64)
        rerun = []
        for i, r in enumerate(g.requests):
            m = self.meshes[r.mesh]
            vf_cap, ee_cap = g.tensors["keep"][i][7]
            n_vf, n_ee = int(cnt[i, 0]), int(cnt[i, 1])
            if cnt[i, 2] & 1:
                raise ValueError(f"request {r.rid}: scene trajectories must be finite")
            if n_vf > vf_cap or n_ee > ee_cap:
                m.vf_cap = max(m.vf_cap, int(n_vf * 1.25) + 1024)
                m.ee_cap = max(m.ee_cap, int(n_ee * 1.25) + 1024)
                r.reruns += 1
                rerun.append(r)
                continue
            # candidate state: the mesh's next requests get buffers fitted to
            # this step's counts (pair sorts and copies scale with capacity)
            m.vf_cap = min(m.vf_cap, int(n_vf * 1.25) + 1024)
            m.ee_cap = min(m.ee_cap, int(n_ee * 1.25) + 1024)
            s = summ[i]
            d = {k: int(s[k]) for k in SUMMARY_DTYPE.names if k != "query"}
            d["query"] = {k: s["query"][k].item() for k in QUERY_CERTIFICATE_DTYPE.names}
            if d["error_word"] & 1:
                raise _lib.P2CError("certification exceeded the device time budget (P2C_DEVICE_BUDGET_MS)")
            r.summary = d
            r.queries = n_vf + n_ee
            mine = uq[uq_scene == i]
            r.undecided = np.stack([((mine >> np.uint64(39)) & np.uint64(1)).astype(np.int64) + 1,
                                    (mine & np.uint64((1 << 39) - 1)).astype(np.int64)], 1)
            r.latency_ms = t_done - 1e3 * r.arrival_s
            if g.tensors["h_res"][i] is not None:
                a, b = g.tensors["h_res"][i]
                r.results = (a.numpy()[:n_vf].copy().view(INTERVAL_RESULT_DTYPE).reshape(-1),
                             b.numpy()[:n_ee].copy().view(INTERVAL_RESULT_DTYPE).reshape(-1))
            self.done.append(r)
        for r in reversed(rerun):
            self.pending.appendleft(r)

    def pump(self) -> bool:
        """Retire finished groups, then admit arrived requests into free
        slots.  Returns True while work is pending or in flight."""
        for s in range(self.slots):
            g = self.busy[s]
            if g is not None and g.event.query():
                self._complete(s)
        for s in range(self.slots):
            if self.busy[s] is not None:
                continue
            group, nbytes = self._admit()
            if not group:
                break
            self._launch(s, group, nbytes)
        return bool(self.pending) or any(g is not None for g in self.busy)

    def run(self, requests: list[Request], idle_sleep_s: float = 5e-5) -> list[Request]:
        """Serve a list of requests (arrival_s relative to the start) to completion."""
        self.done = []
        if self.t0_event is None:
            self.start()
        for r in sorted(requests, key=lambda r: r.arrival_s):
            self.submit(r)
        while self.pump():
            if all(g is not None for g in self.busy) or (self.pending and self.pending[0].arrival_s > self.now()):
                time.sleep(idle_sleep_s)
        torch.cuda.synchronize(self.device)
        return self.done


def latency_stats(done: list[Request]) -> dict:
    lat = np.array([r.latency_ms for r in done], dtype=np.float64)
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}
