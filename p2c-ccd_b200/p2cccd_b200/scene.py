"""Device-resident scenes: swept-AABB candidates and their certificates.

``ScenePipeline`` keeps a scene's vertex trajectories and topology on the GPU
and runs the hot path on the current torch stream without host
synchronisation: candidate generation (``p2c_scene_candidates``) then
certification of every candidate (``p2c_scene_certify``).  Pair buffers are
sized from the previous step; ``step_checked`` reads the counts back and
re-runs a step whose pair count outgrew its buffer.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .certify import CertConfig, _stream_ptr
from .records import INTERVAL_RESULT_DTYPE, QUERY_CERTIFICATE_DTYPE


class SceneStruct(ctypes.Structure):
    _fields_ = [("v_t0", ctypes.c_void_p), ("v_t1", ctypes.c_void_p), ("faces", ctypes.c_void_p),
                ("edges", ctypes.c_void_p), ("v_obj", ctypes.c_void_p), ("f_obj", ctypes.c_void_p),
                ("e_obj", ctypes.c_void_p), ("nv", ctypes.c_int64), ("nf", ctypes.c_int64), ("ne", ctypes.c_int64),
                ("thickness", ctypes.c_double), ("exclude_self", ctypes.c_int32), ("n_obj", ctypes.c_int32)]


SUMMARY_DTYPE = np.dtype({
    "names": ["query", "collisions", "separations", "undecided", "vf_certified", "ee_certified",
              "undecided_queued", "error_word"],
    "formats": [QUERY_CERTIFICATE_DTYPE, "<u8", "<u8", "<u8", "<u8", "<u8", "<u8", "<u8"],
    "offsets": [0, 56, 64, 72, 80, 88, 96, 104],
    "itemsize": 112,
})

ERR_BUDGET, ERR_OVERFLOW, ERR_GEOMETRY, ERR_UNDECIDED_FULL = 1, 2, 4, 8


class UndecidedOverflow(_lib.P2CError):
    """The undecided (fallback-replay) queue was too small: entries were
    counted but not written, so a replay list read from it would be
    incomplete.  ``step_checked`` re-runs with a larger queue instead."""


@dataclass
class SceneArrays:
    """Host (numpy) form of a scene."""
    v_t0: np.ndarray
    v_t1: np.ndarray
    faces: np.ndarray
    edges: np.ndarray
    v_obj: np.ndarray
    f_obj: np.ndarray
    e_obj: np.ndarray

    @classmethod
    def from_dict(cls, d: dict) -> "SceneArrays":
        return cls(*(np.ascontiguousarray(d[k]) for k in ("v_t0", "v_t1", "faces", "edges", "v_obj", "f_obj",
                                                          "e_obj")))


class ScenePipeline:
    """One scene resident on one GPU."""

    def __init__(self, scene: SceneArrays | dict, device: str | torch.device = "cuda", *,
                 thickness: float = 0.0, exclude_self: bool = True, config: CertConfig = CertConfig(),
                 interval: tuple[float, float] = (0.0, 1.0), family_mask: int = 3, sort_pairs: bool = True,
                 vf_capacity: int = 1 << 16, ee_capacity: int = 1 << 16, undecided_capacity: int = 1 << 14,
                 narrow: str = "certify", top_k: int = 4096, scheduler_seed: int = 0):
        """narrow = "certify": every candidate is certified (p2c_scene_certify);
        narrow = "anyhit": candidates are grouped by object pair and run
        through the scheduled any-hit with fallback replay
        (p2c_group_anyhit) with proposal size top_k and priority scores from
        the seeded scheduler stub (p2c_stub_scores: a uniform score per
        candidate identity, so a candidate ranks the same here and in a
        served batch)."""
        if isinstance(scene, dict):
            scene = SceneArrays.from_dict(scene)
        self.lib = _lib.load()
        self.device = torch.device(device)
        d = self.device
        self.v_t0 = torch.as_tensor(np.ascontiguousarray(scene.v_t0, dtype=np.float64)).to(d)
        self.v_t1 = torch.as_tensor(np.ascontiguousarray(scene.v_t1, dtype=np.float64)).to(d)
        self.faces = torch.as_tensor(np.ascontiguousarray(scene.faces, dtype=np.int32)).to(d)
        self.edges = torch.as_tensor(np.ascontiguousarray(scene.edges, dtype=np.int32)).to(d)
        self.v_obj = torch.as_tensor(np.ascontiguousarray(scene.v_obj, dtype=np.int32)).to(d)
        self.f_obj = torch.as_tensor(np.ascontiguousarray(scene.f_obj, dtype=np.int32)).to(d)
        self.e_obj = torch.as_tensor(np.ascontiguousarray(scene.e_obj, dtype=np.int32)).to(d)
        self.thickness = float(thickness)
        self.n_obj = int(max(scene.v_obj.max(initial=-1), scene.f_obj.max(initial=-1),
                             scene.e_obj.max(initial=-1)) + 1)
        self.exclude_self = bool(exclude_self)
        self.config = config
        self.interval = (float(interval[0]), float(interval[1]))
        self.family_mask = int(family_mask)
        self.sort_pairs = bool(sort_pairs)
        self.counts = torch.zeros(4, dtype=torch.int64, device=d)
        self.summary = torch.zeros(SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device=d)
        self.cert_ws = torch.empty(int(self.lib.p2c_scene_certify_workspace_bytes()), dtype=torch.uint8, device=d)
        self._alloc_undecided(undecided_capacity)
        if narrow not in ("certify", "anyhit"):
            raise ValueError("narrow must be 'certify' or 'anyhit'")
        self.narrow = narrow
        self.top_k = int(top_k)
        self.scheduler_seed = int(scheduler_seed)
        self._struct = SceneStruct()
        self._refresh_struct()
        self._alloc(vf_capacity, ee_capacity)

    # -- buffers ---------------------------------------------------------
    def _alloc_undecided(self, capacity: int) -> None:
        self.undecided_capacity = max(1, int(capacity))
        self.undecided_queue = torch.empty(self.undecided_capacity, dtype=torch.int64, device=self.device)
        self.graph = None

    def _refresh_struct(self):
        s = self._struct
        s.v_t0, s.v_t1 = self.v_t0.data_ptr(), self.v_t1.data_ptr()
        s.faces, s.edges = self.faces.data_ptr(), self.edges.data_ptr()
        s.v_obj, s.f_obj, s.e_obj = self.v_obj.data_ptr(), self.f_obj.data_ptr(), self.e_obj.data_ptr()
        s.nv, s.nf, s.ne = self.v_t0.shape[0], self.faces.shape[0], self.edges.shape[0]
        s.thickness = self.thickness
        s.exclude_self = 1 if self.exclude_self else 0
        s.n_obj = self.n_obj

    def _alloc(self, vf_cap: int, ee_cap: int):
        d = self.device
        self.vf_cap, self.ee_cap = max(1, int(vf_cap)), max(1, int(ee_cap))
        self.vf_pairs = torch.empty(self.vf_cap, dtype=torch.int64, device=d)
        self.ee_pairs = torch.empty(self.ee_cap, dtype=torch.int64, device=d)
        self.vf_results = torch.empty((self.vf_cap, 72), dtype=torch.uint8, device=d)
        self.ee_results = torch.empty((self.ee_cap, 72), dtype=torch.uint8, device=d)
        nbytes = self.lib.p2c_scene_candidates_workspace_bytes(self._struct.nv, self._struct.nf, self._struct.ne,
                                                               self.vf_cap, self.ee_cap)
        self.bp_ws = torch.empty(int(nbytes), dtype=torch.uint8, device=d)
        if self.narrow == "anyhit":
            from .anyhit import GroupAnyHit

            self.vf_scores = torch.zeros(self.vf_cap, dtype=torch.float64, device=d)
            self.ee_scores = torch.zeros(self.ee_cap, dtype=torch.float64, device=d)
            self.anyhit_vf = GroupAnyHit(self._struct, self.n_obj, "vf", self.vf_cap, d)
            self.anyhit_ee = GroupAnyHit(self._struct, self.n_obj, "ee", self.ee_cap, d)

    def update_positions(self, v_t0: torch.Tensor, v_t1: torch.Tensor) -> None:
        """Copy a new step's trajectories into the resident buffers (async)."""
        self.v_t0.copy_(v_t0, non_blocking=True)
        self.v_t1.copy_(v_t1, non_blocking=True)

    # -- hot path ---------------------------------------------------------
    def candidates(self) -> None:
        stream = _stream_ptr(self.device)
        _lib.check(self.lib.p2c_scene_candidates(ctypes.byref(self._struct), self.vf_pairs.data_ptr(), self.vf_cap,
                                                 self.ee_pairs.data_ptr(), self.ee_cap, self.counts.data_ptr(),
                                                 1 if self.sort_pairs else 0, self.bp_ws.data_ptr(),
                                                 self.bp_ws.numel(), stream))

    def certify(self) -> None:
        stream = _stream_ptr(self.device)
        cfg = self.config.c()
        _lib.check(self.lib.p2c_scene_certify(
            ctypes.byref(self._struct), self.vf_pairs.data_ptr(), self.vf_cap, self.ee_pairs.data_ptr(), self.ee_cap,
            self.counts.data_ptr(), self.interval[0], self.interval[1], ctypes.byref(cfg), self.family_mask,
            self.vf_results.data_ptr(), self.ee_results.data_ptr(), self.undecided_queue.data_ptr(),
            self.undecided_capacity, self.summary.data_ptr(), self.cert_ws.data_ptr(), self.cert_ws.numel(), stream))

    def anyhit(self) -> None:
        """Scheduled any-hit with fallback replay of both families (async),
        scores from the scheduler stub."""
        from .anyhit import stub_scores

        if self.family_mask & 1:
            stub_scores(self.vf_pairs, self.counts[0:1], 1, self.scheduler_seed, self.vf_scores)
        if self.family_mask & 2:
            stub_scores(self.ee_pairs, self.counts[1:2], 2, self.scheduler_seed, self.ee_scores)
        if self.family_mask & 1:
            self.anyhit_vf.run(self.vf_pairs, self.counts[0:1], self.vf_scores, self.top_k, self.config,
                               self.interval)
        if self.family_mask & 2:
            self.anyhit_ee.run(self.ee_pairs, self.counts[1:2], self.ee_scores, self.top_k, self.config,
                               self.interval)

    def narrow_phase(self) -> None:
        if self.narrow == "anyhit":
            self.anyhit()
        else:
            self.certify()

    def step(self) -> None:
        """Candidates then the narrow phase, asynchronous on the current stream."""
        self.candidates()
        self.narrow_phase()

    def capture(self) -> None:
        """Capture one step (candidates + certificates, ~60 launches) into a
        CUDA graph; ``replay`` then costs one graph launch.  Buffers and
        capacities are fixed at capture time: re-capture after growth."""
        self.graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self.step()
        torch.cuda.current_stream(self.device).wait_stream(side)
        with torch.cuda.graph(self.graph):
            self.step()
        self._graph_caps = (self.vf_cap, self.ee_cap)

    def replay(self) -> None:
        if getattr(self, "graph", None) is None or self._graph_caps != (self.vf_cap, self.ee_cap):
            self.capture()
        self.graph.replay()

    def read_counts(self) -> tuple[int, int, int]:
        c = self.counts.cpu().numpy()
        return int(c[0]), int(c[1]), int(c[2])

    def step_checked(self, max_retries: int = 3) -> dict:
        """Run a step; grow the pair buffers or the undecided queue and re-run
        if they overflowed; raise on non-finite geometry or an exhausted time
        budget.  Every returned step certified every candidate and queued
        every undecided one."""
        for _ in range(max_retries + 1):
            self.step()
            n_vf, n_ee, err = self.read_counts()
            if err & 1:
                raise ValueError("scene trajectories must be finite")
            if n_vf <= self.vf_cap and n_ee <= self.ee_cap:
                summ = self.read_summary() if self.narrow == "certify" else self.read_anyhit_summary()
                if summ["error_word"] & ERR_BUDGET:
                    raise _lib.P2CError("certification exceeded the device time budget (P2C_DEVICE_BUDGET_MS)")
                if self.narrow == "certify" and summ["error_word"] & ERR_UNDECIDED_FULL:
                    self._alloc_undecided(int(summ["undecided_queued"] * 1.25) + 1024)
                    continue
                return summ
            self._alloc(max(self.vf_cap, int(n_vf * 1.25) + 1024), max(self.ee_cap, int(n_ee * 1.25) + 1024))
        raise _lib.P2CError("pair buffers or the undecided queue kept overflowing")

    def read_anyhit_summary(self) -> dict:
        """Both families' any-hit summaries plus their sums."""
        out = {"vf": self.anyhit_vf.read_summary() if self.family_mask & 1 else None,
               "ee": self.anyhit_ee.read_summary() if self.family_mask & 2 else None}
        parts = [v for v in out.values() if v is not None]
        for k in ("candidates", "groups", "detected_groups", "proposal_calls", "fallback_calls", "speculative"):
            out[k] = sum(p[k] for p in parts)
        out["calls"] = out["proposal_calls"] + out["fallback_calls"]
        out["error_word"] = 0
        for p in parts:
            out["error_word"] |= p["error_word"]
        return out

    def fit_capacities(self, margin: float = 1.25, slack: int = 256) -> None:
        """Resize the pair buffers to the last candidate counts x margin +
        slack: the pair sorts, the any-hit sorts and the result buffers scale
        with the capacities, not the counts.  A later step whose counts grow
        past them needs ``step_checked``; a captured graph is re-captured."""
        n_vf, n_ee, _ = self.read_counts()
        self._alloc(int(n_vf * margin) + slack, int(n_ee * margin) + slack)
        self.graph = None

    def read_summary(self) -> dict:
        raw = self.summary.cpu().numpy().view(SUMMARY_DTYPE)[0]
        out = {k: int(raw[k]) for k in SUMMARY_DTYPE.names if k != "query"}
        out["query"] = {k: raw["query"][k].item() for k in QUERY_CERTIFICATE_DTYPE.names}
        return out

    def pairs(self) -> tuple[np.ndarray, np.ndarray]:
        n_vf, n_ee, _ = self.read_counts()
        return (self.vf_pairs[:n_vf].cpu().numpy().view(np.uint64),
                self.ee_pairs[:n_ee].cpu().numpy().view(np.uint64))

    def results(self) -> tuple[np.ndarray, np.ndarray]:
        n_vf, n_ee, _ = self.read_counts()
        r = lambda t, n: t[:n].cpu().numpy().view(INTERVAL_RESULT_DTYPE).reshape(-1)
        return r(self.vf_results, min(n_vf, self.vf_cap)), r(self.ee_results, min(n_ee, self.ee_cap))

    def materialize(self) -> tuple[np.ndarray, np.ndarray]:
        """Candidate pairs as reference primitive records (host arrays)."""
        from .records import EDGE_EDGE_DTYPE, POINT_TRIANGLE_DTYPE

        n_vf, n_ee, _ = self.read_counts()
        n_vf, n_ee = min(n_vf, self.vf_cap), min(n_ee, self.ee_cap)
        a = torch.empty((max(n_vf, 1), 240), dtype=torch.uint8, device=self.device)
        b = torch.empty((max(n_ee, 1), 240), dtype=torch.uint8, device=self.device)
        _lib.check(self.lib.p2c_scene_materialize(ctypes.byref(self._struct), self.vf_pairs.data_ptr(), n_vf,
                                                  self.ee_pairs.data_ptr(), n_ee, a.data_ptr(), b.data_ptr(),
                                                  _stream_ptr(self.device)))
        return (a[:n_vf].cpu().numpy().view(POINT_TRIANGLE_DTYPE).reshape(-1),
                b[:n_ee].cpu().numpy().view(EDGE_EDGE_DTYPE).reshape(-1))

    @property
    def undecided_entries(self) -> np.ndarray:
        """Undecided (fallback-replay) queue: (family - 1) << 63 | pair position.
        Raises ``UndecidedOverflow`` when the queue was too small for the
        step (the list would miss undecided candidates)."""
        summ = self.read_summary()
        n = summ["undecided_queued"]
        if summ["error_word"] & ERR_UNDECIDED_FULL or n > self.undecided_capacity:
            raise UndecidedOverflow(f"undecided queue overflow: {n} entries, capacity {self.undecided_capacity}")
        return self.undecided_queue[:n].cpu().numpy().view(np.uint64)
