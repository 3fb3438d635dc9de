"""Batched scenes: many independent scenes of uneven size per step.

``BatchPipeline`` keeps every scene resident on one GPU (one concatenated
buffer per array, scene-local indices) and runs a step as

* candidate generation of every scene (``p2c_scene_candidates``), fanned out
  over a few CUDA streams so small scenes overlap;
* ONE persistent certification launch over all scenes' candidates
  (``p2c_batch_certify``) with a per-scene CertificateEngine::Evaluate
  summary;

all of it captured into one CUDA graph.  ``autotune`` picks the certifier's
launch shape (blocks per SM, per-warp queue width, helper warps) and the
broad-phase stream count by timing graph replays of the actual batch.
"""
from __future__ import annotations

import ctypes
import itertools
import json
import os
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .certify import CertConfig, _stream_ptr
from .records import INTERVAL_RESULT_DTYPE, QUERY_CERTIFICATE_DTYPE
from .scene import ERR_UNDECIDED_FULL, SUMMARY_DTYPE, SceneStruct, UndecidedOverflow

BATCH_SCENE_DTYPE = np.dtype([
    ("v_t0", "<u8"), ("v_t1", "<u8"), ("faces", "<u8"), ("edges", "<u8"), ("vf_pairs", "<u8"),
    ("ee_pairs", "<u8"), ("vf_cap", "<i8"), ("ee_cap", "<i8"), ("counts", "<u8"), ("vf_results", "<u8"),
    ("ee_results", "<u8"), ("v_obj", "<u8"), ("f_obj", "<u8"), ("e_obj", "<u8"), ("nv", "<i8"), ("nf", "<i8"),
    ("ne", "<i8"), ("thickness", "<f8"), ("exclude_self", "<i4"), ("n_obj", "<i4"),
])
assert BATCH_SCENE_DTYPE.itemsize == 152


def scene_row(st, vf_pairs: int, ee_pairs: int, vf_cap: int, ee_cap: int, counts: int, vf_results: int,
              ee_results: int) -> tuple:
    """One p2c_batch_scene row from a SceneStruct and the scene's buffers."""
    return (st.v_t0, st.v_t1, st.faces, st.edges, vf_pairs, ee_pairs, vf_cap, ee_cap, counts, vf_results,
            ee_results, st.v_obj, st.f_obj, st.e_obj, st.nv, st.nf, st.ne, st.thickness, st.exclude_self, st.n_obj)


def lpt_partition(weights: list[float] | np.ndarray, n_bins: int) -> list[list[int]]:
    """Longest-processing-time-first packing of independent scenes onto
    n_bins GPUs: scenes by decreasing weight (triangle count), each to the
    least-loaded bin so far (ties: the lower bin); each bin's scenes in index
    order.  The most-loaded bin holds at most 4/3 of the optimum.  Every rank
    computes the same packing from the same weights, so no exchange is needed."""
    import heapq

    w = np.asarray(weights, dtype=np.float64)
    if n_bins < 1:
        raise ValueError("n_bins must be at least 1")
    heap = [(0.0, b) for b in range(n_bins)]
    bins: list[list[int]] = [[] for _ in range(n_bins)]
    for i in sorted(range(len(w)), key=lambda k: (-w[k], k)):
        load, b = heapq.heappop(heap)
        bins[b].append(i)
        heapq.heappush(heap, (load + float(w[i]), b))
    return [sorted(x) for x in bins]


def decode_batch_undecided(raw: np.ndarray) -> np.ndarray:
    """Entries (scene << 40 | (family - 1) << 39 | position) of a batch
    undecided queue as int64 rows (scene, family 1/2, pair position)."""
    u = np.asarray(raw).view(np.uint64)
    return np.stack([(u >> np.uint64(40)).astype(np.int64),
                     ((u >> np.uint64(39)) & np.uint64(1)).astype(np.int64) + 1,
                     (u & np.uint64((1 << 39) - 1)).astype(np.int64)], 1).reshape(-1, 3)


class BatchTuning(ctypes.Structure):
    _fields_ = [("blocks_per_sm", ctypes.c_int32), ("fetch_limit", ctypes.c_int32),
                ("helper_warps", ctypes.c_int32), ("reserved", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {"blocks_per_sm": self.blocks_per_sm, "fetch_limit": self.fetch_limit,
                "helper_warps": self.helper_warps}


def _pad(n: int, a: int = 32) -> int:
    return (n + a - 1) // a * a


class BatchPipeline:
    """Scenes (dicts of numpy arrays as ``scenes`` builds them) resident on one GPU."""

    def __init__(self, scenes: list[dict], device: str | torch.device = "cuda", *, thickness: float = 0.0,
                 exclude_self: bool = True, config: CertConfig = CertConfig(),
                 interval: tuple[float, float] = (0.0, 1.0), family_mask: int = 3, streams: int = 8,
                 undecided_capacity: int = 1 << 16, broad: str = "batched"):
        if not scenes:
            raise ValueError("a batch needs at least one scene")
        self.lib = _lib.load()
        self.device = d = torch.device(device)
        self.n = len(scenes)
        self.config = config
        self.interval = (float(interval[0]), float(interval[1]))
        self.family_mask = int(family_mask)
        self.thickness = float(thickness)
        self.exclude_self = bool(exclude_self)
        self.n_streams = max(1, int(streams))
        if broad not in ("batched", "per_scene"):
            raise ValueError("broad must be 'batched' or 'per_scene'")
        self.broad = broad
        self.tuning = BatchTuning(0, 0, 0, 0)
        # concatenated geometry; each scene's slice starts on a 256-byte boundary
        nv = [len(s["v_t0"]) for s in scenes]
        nf = [len(s["faces"]) for s in scenes]
        ne = [len(s["edges"]) for s in scenes]
        self.nv, self.nf, self.ne = nv, nf, ne
        self.v_off = np.concatenate([[0], np.cumsum([_pad(3 * x) for x in nv])]).astype(np.int64)
        self.f_off = np.concatenate([[0], np.cumsum([_pad(3 * x) for x in nf])]).astype(np.int64)
        self.e_off = np.concatenate([[0], np.cumsum([_pad(2 * x) for x in ne])]).astype(np.int64)
        self.vo_off = np.concatenate([[0], np.cumsum([_pad(x) for x in nv])]).astype(np.int64)
        self.fo_off = np.concatenate([[0], np.cumsum([_pad(x) for x in nf])]).astype(np.int64)
        self.eo_off = np.concatenate([[0], np.cumsum([_pad(x) for x in ne])]).astype(np.int64)
        h_t0 = np.zeros(self.v_off[-1]), np.zeros(self.v_off[-1])
        h_f = np.zeros(self.f_off[-1], np.int32)
        h_e = np.zeros(self.e_off[-1], np.int32)
        h_vo = np.zeros(self.vo_off[-1], np.int32)
        h_fo = np.zeros(self.fo_off[-1], np.int32)
        h_eo = np.zeros(self.eo_off[-1], np.int32)
        self.n_obj = []
        for i, s in enumerate(scenes):
            h_t0[0][self.v_off[i]:self.v_off[i] + 3 * nv[i]] = np.asarray(s["v_t0"], np.float64).ravel()
            h_t0[1][self.v_off[i]:self.v_off[i] + 3 * nv[i]] = np.asarray(s["v_t1"], np.float64).ravel()
            h_f[self.f_off[i]:self.f_off[i] + 3 * nf[i]] = np.asarray(s["faces"], np.int32).ravel()
            h_e[self.e_off[i]:self.e_off[i] + 2 * ne[i]] = np.asarray(s["edges"], np.int32).ravel()
            h_vo[self.vo_off[i]:self.vo_off[i] + nv[i]] = s["v_obj"]
            h_fo[self.fo_off[i]:self.fo_off[i] + nf[i]] = s["f_obj"]
            h_eo[self.eo_off[i]:self.eo_off[i] + ne[i]] = s["e_obj"]
            self.n_obj.append(int(max(np.max(s["v_obj"], initial=-1), np.max(s["f_obj"], initial=-1),
                                      np.max(s["e_obj"], initial=-1)) + 1))
        self.v_t0 = torch.from_numpy(h_t0[0]).to(d)
        self.v_t1 = torch.from_numpy(h_t0[1]).to(d)
        self.faces = torch.from_numpy(h_f).to(d)
        self.edges = torch.from_numpy(h_e).to(d)
        self.v_obj = torch.from_numpy(h_vo).to(d)
        self.f_obj = torch.from_numpy(h_fo).to(d)
        self.e_obj = torch.from_numpy(h_eo).to(d)
        self.structs = [SceneStruct() for _ in range(self.n)]
        for i in range(self.n):
            st = self.structs[i]
            st.v_t0 = self.v_t0.data_ptr() + 8 * int(self.v_off[i])
            st.v_t1 = self.v_t1.data_ptr() + 8 * int(self.v_off[i])
            st.faces = self.faces.data_ptr() + 4 * int(self.f_off[i])
            st.edges = self.edges.data_ptr() + 4 * int(self.e_off[i])
            st.v_obj = self.v_obj.data_ptr() + 4 * int(self.vo_off[i])
            st.f_obj = self.f_obj.data_ptr() + 4 * int(self.fo_off[i])
            st.e_obj = self.e_obj.data_ptr() + 4 * int(self.eo_off[i])
            st.nv, st.nf, st.ne = nv[i], nf[i], ne[i]
            st.thickness = self.thickness
            st.exclude_self = 1 if self.exclude_self else 0
            st.n_obj = self.n_obj[i]
        self.counts = torch.zeros((self.n, 4), dtype=torch.int64, device=d)
        self.summaries = torch.zeros((self.n, SUMMARY_DTYPE.itemsize), dtype=torch.uint8, device=d)
        self.cert_ws = torch.empty(int(self.lib.p2c_batch_certify_workspace_bytes(self.n)), dtype=torch.uint8,
                                   device=d)
        self._alloc_undecided(undecided_capacity)
        # first sizing of the pair buffers: about one candidate per triangle
        self._alloc([max(1024, x) for x in nf], [max(1024, 2 * x) for x in nf])

    # -- buffers ---------------------------------------------------------
    def _alloc_undecided(self, capacity: int) -> None:
        self.undecided_capacity = max(1, int(capacity))
        self.undecided_queue = torch.empty(self.undecided_capacity, dtype=torch.int64, device=self.device)
        self.graph = None

    def _alloc(self, vf_caps: list[int], ee_caps: list[int]) -> None:
        d = self.device
        self.vf_caps = [max(1, int(c)) for c in vf_caps]
        self.ee_caps = [max(1, int(c)) for c in ee_caps]
        self.vf_pair_off = np.concatenate([[0], np.cumsum([_pad(c) for c in self.vf_caps])]).astype(np.int64)
        self.ee_pair_off = np.concatenate([[0], np.cumsum([_pad(c) for c in self.ee_caps])]).astype(np.int64)
        self.vf_pairs = torch.empty(int(self.vf_pair_off[-1]), dtype=torch.int64, device=d)
        self.ee_pairs = torch.empty(int(self.ee_pair_off[-1]), dtype=torch.int64, device=d)
        self.vf_results = torch.empty((int(self.vf_pair_off[-1]), 72), dtype=torch.uint8, device=d)
        self.ee_results = torch.empty((int(self.ee_pair_off[-1]), 72), dtype=torch.uint8, device=d)
        ws = [int(self.lib.p2c_scene_candidates_workspace_bytes(self.nv[i], self.nf[i], self.ne[i], self.vf_caps[i],
                                                                 self.ee_caps[i])) for i in range(self.n)]
        self.bp_ws_off = np.concatenate([[0], np.cumsum([_pad(w, 256) for w in ws])]).astype(np.int64)
        self.bp_ws_bytes = ws
        self.bp_ws = torch.empty(int(self.bp_ws_off[-1]), dtype=torch.uint8, device=d)
        table = np.zeros(self.n, dtype=BATCH_SCENE_DTYPE)
        for i, st in enumerate(self.structs):
            table[i] = scene_row(st, self.vf_pairs.data_ptr() + 8 * int(self.vf_pair_off[i]),
                                 self.ee_pairs.data_ptr() + 8 * int(self.ee_pair_off[i]), self.vf_caps[i],
                                 self.ee_caps[i], self.counts.data_ptr() + 32 * i,
                                 self.vf_results.data_ptr() + 72 * int(self.vf_pair_off[i]),
                                 self.ee_results.data_ptr() + 72 * int(self.ee_pair_off[i]))
        self.table_host = table
        self.table = torch.from_numpy(table.view(np.uint8).copy()).to(d)
        self.bb_ws = torch.empty(int(self.lib.p2c_batch_candidates_workspace_bytes(table.ctypes.data, self.n)),
                                 dtype=torch.uint8, device=d)
        self.graph = None

    def update_positions(self, v_t0: torch.Tensor, v_t1: torch.Tensor) -> None:
        """Copy a new step's concatenated trajectories (layout of ``v_t0``) in (async)."""
        self.v_t0.copy_(v_t0, non_blocking=True)
        self.v_t1.copy_(v_t1, non_blocking=True)

    # -- hot path ---------------------------------------------------------
    def candidates(self) -> None:
        """Candidate generation of every scene: one batched launch sequence
        (``broad="batched"``, the default) or one p2c_scene_candidates per
        scene round-robin over side streams (``broad="per_scene"``)."""
        if self.broad == "batched":
            _lib.check(self.lib.p2c_batch_candidates(self.table_host.ctypes.data, self.table.data_ptr(), self.n,
                                                     self.bb_ws.data_ptr(), self.bb_ws.numel(),
                                                     _stream_ptr(self.device)))
            return
        self._candidates_per_scene()

    def _candidates_per_scene(self) -> None:
        main = torch.cuda.current_stream(self.device)
        if not hasattr(self, "_side") or len(self._side) != self.n_streams:
            self._side = [torch.cuda.Stream(self.device) for _ in range(self.n_streams)]
        for st in self._side:
            st.wait_stream(main)
        order = sorted(range(self.n), key=lambda i: -self.nf[i])  # largest first
        for k, i in enumerate(order):
            st = self._side[k % self.n_streams]
            _lib.check(self.lib.p2c_scene_candidates(
                ctypes.byref(self.structs[i]), self.vf_pairs.data_ptr() + 8 * int(self.vf_pair_off[i]),
                self.vf_caps[i], self.ee_pairs.data_ptr() + 8 * int(self.ee_pair_off[i]), self.ee_caps[i],
                self.counts.data_ptr() + 32 * i, 1, self.bp_ws.data_ptr() + int(self.bp_ws_off[i]),
                self.bp_ws_bytes[i], st.cuda_stream))
        for st in self._side:
            main.wait_stream(st)

    def certify(self) -> None:
        cfg = self.config.c()
        _lib.check(self.lib.p2c_batch_certify(
            self.table.data_ptr(), self.n, self.interval[0], self.interval[1], ctypes.byref(cfg), self.family_mask,
            self.summaries.data_ptr(), self.undecided_queue.data_ptr(), self.undecided_capacity,
            ctypes.addressof(self.tuning), self.cert_ws.data_ptr(), self.cert_ws.numel(), _stream_ptr(self.device)))

    def step(self) -> None:
        self.candidates()
        self.certify()

    def capture(self) -> None:
        """One CUDA graph for the whole step (all scenes' candidates, the one
        certification launch and the summaries)."""
        self.graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self.step()
        torch.cuda.current_stream(self.device).wait_stream(side)
        with torch.cuda.graph(self.graph):
            self.step()

    def replay(self) -> None:
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def read_counts(self) -> np.ndarray:
        return self.counts.cpu().numpy()

    def step_checked(self, max_retries: int = 3) -> list[dict]:
        """Run a step; grow the pair buffers of scenes that overflowed, or
        the shared undecided queue, and re-run."""
        for _ in range(max_retries + 1):
            self.step()
            c = self.read_counts()
            if np.any(c[:, 2] & 1):
                raise ValueError("scene trajectories must be finite")
            over_vf = c[:, 0] > np.array(self.vf_caps)
            over_ee = c[:, 1] > np.array(self.ee_caps)
            if not over_vf.any() and not over_ee.any():
                summ = self.read_summaries()
                if any(s["error_word"] & 1 for s in summ):
                    raise _lib.P2CError("certification exceeded the device time budget (P2C_DEVICE_BUDGET_MS)")
                queued = sum(s["undecided_queued"] for s in summ)
                if queued > self.undecided_capacity or any(s["error_word"] & ERR_UNDECIDED_FULL for s in summ):
                    self._alloc_undecided(int(queued * 1.25) + 1024)
                    continue
                return summ
            self._alloc([max(cap, int(n * 1.25) + 1024) if o else cap
                         for cap, n, o in zip(self.vf_caps, c[:, 0], over_vf)],
                        [max(cap, int(n * 1.25) + 1024) if o else cap
                         for cap, n, o in zip(self.ee_caps, c[:, 1], over_ee)])
        raise _lib.P2CError("pair buffers or the undecided queue kept overflowing")

    def fit_capacities(self, margin: float = 1.25, slack: int = 256) -> None:
        """Resize every scene's pair buffers to its last candidate count x
        margin + slack.  The pair sort and the result buffers scale with the
        capacities, not the counts, so a step after this costs less; a later
        step whose counts grow past the capacities needs ``step_checked``."""
        c = self.read_counts()
        self._alloc([int(n * margin) + slack for n in c[:, 0]], [int(n * margin) + slack for n in c[:, 1]])

    def read_summaries(self) -> list[dict]:
        raw = self.summaries.cpu().numpy().reshape(-1).view(SUMMARY_DTYPE)
        out = []
        for r in raw:
            d = {k: int(r[k]) for k in SUMMARY_DTYPE.names if k != "query"}
            d["query"] = {k: r["query"][k].item() for k in QUERY_CERTIFICATE_DTYPE.names}
            out.append(d)
        return out

    def pairs(self, i: int) -> tuple[np.ndarray, np.ndarray]:
        c = self.read_counts()[i]
        n_vf, n_ee = min(int(c[0]), self.vf_caps[i]), min(int(c[1]), self.ee_caps[i])
        a, b = int(self.vf_pair_off[i]), int(self.ee_pair_off[i])
        return (self.vf_pairs[a:a + n_vf].cpu().numpy().view(np.uint64),
                self.ee_pairs[b:b + n_ee].cpu().numpy().view(np.uint64))

    def results(self, i: int) -> tuple[np.ndarray, np.ndarray]:
        c = self.read_counts()[i]
        n_vf, n_ee = min(int(c[0]), self.vf_caps[i]), min(int(c[1]), self.ee_caps[i])
        a, b = int(self.vf_pair_off[i]), int(self.ee_pair_off[i])
        r = lambda t, o, n: t[o:o + n].cpu().numpy().view(INTERVAL_RESULT_DTYPE).reshape(-1)
        return r(self.vf_results, a, n_vf), r(self.ee_results, b, n_ee)

    def materialize(self, i: int) -> tuple[np.ndarray, np.ndarray]:
        """Scene i's candidate pairs as reference primitive records (host arrays)."""
        from .records import EDGE_EDGE_DTYPE, POINT_TRIANGLE_DTYPE

        c = self.read_counts()[i]
        n_vf, n_ee = min(int(c[0]), self.vf_caps[i]), min(int(c[1]), self.ee_caps[i])
        a = torch.empty((max(n_vf, 1), 240), dtype=torch.uint8, device=self.device)
        b = torch.empty((max(n_ee, 1), 240), dtype=torch.uint8, device=self.device)
        _lib.check(self.lib.p2c_scene_materialize(
            ctypes.byref(self.structs[i]), self.vf_pairs.data_ptr() + 8 * int(self.vf_pair_off[i]), n_vf,
            self.ee_pairs.data_ptr() + 8 * int(self.ee_pair_off[i]), n_ee, a.data_ptr(), b.data_ptr(),
            _stream_ptr(self.device)))
        return (a[:n_vf].cpu().numpy().view(POINT_TRIANGLE_DTYPE).reshape(-1),
                b[:n_ee].cpu().numpy().view(EDGE_EDGE_DTYPE).reshape(-1))

    def undecided_entries(self) -> np.ndarray:
        """The step's undecided (fallback-replay) entries of all scenes as
        (scene, family, pair position) rows, in queue order.  Raises
        ``UndecidedOverflow`` when the shared queue was too small."""
        summ = self.read_summaries()
        n = sum(s["undecided_queued"] for s in summ)
        if n > self.undecided_capacity or any(s["error_word"] & ERR_UNDECIDED_FULL for s in summ):
            raise UndecidedOverflow(f"undecided queue overflow: {n} entries, capacity {self.undecided_capacity}")
        return decode_batch_undecided(self.undecided_queue[:n].cpu().numpy())

    def certified_per_step(self) -> int:
        s = self.read_summaries()
        return sum(x["vf_certified"] + x["ee_certified"] for x in s)

    # -- autotuning ---------------------------------------------------------
    def _time_replays(self, reps: int) -> float:
        self.replay()
        torch.cuda.synchronize(self.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            self.graph.replay()
        e1.record()
        torch.cuda.synchronize(self.device)
        return e0.elapsed_time(e1) / reps

    def autotune(self, reps: int = 5, cache: str | os.PathLike | None = None) -> dict:
        """Time graph replays over a grid of launch shapes and keep the
        fastest: certifier blocks per SM x per-warp queue width x helper
        warps, then the broad-phase stream count.  The choice is cached in
        ``cache`` (JSON, keyed by device name and batch signature) when given."""
        key = None
        if cache is not None:
            sig = f"{torch.cuda.get_device_name(self.device)}|{self.n}|{sum(self.nf)}|{self.config}"
            key = sig
            path = Path(cache)
            if path.exists():
                known = json.loads(path.read_text())
                if key in known:
                    t = known[key]
                    self.tuning = BatchTuning(t["blocks_per_sm"], t["fetch_limit"], t["helper_warps"], 0)
                    self.n_streams = t["streams"]
                    self.graph = None
                    return dict(t, cached=True)
        trials = []
        for bps, fetch, helpers in itertools.product((0, 2, 3), (0, 4, 16), (0, 148, 592)):
            self.tuning = BatchTuning(bps, fetch, helpers, 0)
            self.graph = None
            trials.append((self._time_replays(reps), bps, fetch, helpers))
        trials.sort()
        _, bps, fetch, helpers = trials[0]
        self.tuning = BatchTuning(bps, fetch, helpers, 0)
        stream_trials = [(trials[0][0], self.n_streams)]
        if self.broad == "per_scene":  # the per-scene broad phase fans out over side streams
            stream_trials = []
            for ns in (1, 4, 8, 16):
                self.n_streams = ns
                self.graph = None
                stream_trials.append((self._time_replays(reps), ns))
            stream_trials.sort()
        self.n_streams = stream_trials[0][1]
        self.graph = None
        best = {"blocks_per_sm": bps, "fetch_limit": fetch, "helper_warps": helpers, "streams": self.n_streams,
                "broad": self.broad, "ms": stream_trials[0][0], "trials": len(trials) + len(stream_trials)}
        if key is not None:
            path = Path(cache)
            known = json.loads(path.read_text()) if path.exists() else {}
            known[key] = best
            path.write_text(json.dumps(known, indent=1))
        return best
