"""Candidates of a proxy scene on the device (p2c_proxy_candidates).

A proxy scene is the primitive list of a built ProxyScene
(rt_candidate/proxy_scene.h:29-46): per proxy its object, patch, time slab,
type, slab interval, AABB and motion bounds.  ``proxy_candidates`` returns
the reference's raw hits (GenerateRawCandidatesCpu) and compacted candidate
records (CompactRawCandidates) as numpy record arrays, byte for byte.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .certify import _stream_ptr
from .records import CANDIDATE_RECORD_DTYPE, DENSITY_DTYPE, FEATURE_ROW_DTYPE, RAW_HIT_DTYPE

ERR_INVALID_PROXY, ERR_MOTION_BOUND, ERR_OVERFLOW, ERR_ID_BITS, ERR_HIT_COUNT_OVERFLOW = 1, 2, 4, 8, 16

# ValidateRawHit's messages (rt_candidate/candidate_buffer.cpp:71-101) by the
# check number p2c_compact_raw_candidates reports
RAW_HIT_ERRORS = {1: "raw candidate hit is not marked valid", 2: "raw candidate query_id is required",
                  3: "raw candidate query_id must match ProxyScene.query_id",
                  4: "raw candidate proxy index is out of range",
                  5: "raw candidate cannot reference the same proxy twice",
                  6: "raw candidate pair_key does not match proxy indices",
                  7: "raw candidate must reference two different objects",
                  8: "raw candidate slab_id must match both proxy primitives",
                  9: "raw candidate motion_bound must be finite and non-negative"}


def _bits(max_id: int) -> int:
    """Width hint for ids up to max_id (at least 1 bit)."""
    return max(1, int(max_id).bit_length())


class ProxySceneStruct(ctypes.Structure):
    _fields_ = [("query_id", ctypes.c_uint64), ("n", ctypes.c_int64), ("object_id", ctypes.c_void_p),
                ("patch_id", ctypes.c_void_p), ("slab_id", ctypes.c_void_p), ("proxy_type", ctypes.c_void_p),
                ("t0", ctypes.c_void_p), ("t1", ctypes.c_void_p), ("bounds", ctypes.c_void_p),
                ("motion_bound", ctypes.c_void_p), ("slab_bits", ctypes.c_uint32), ("object_bits", ctypes.c_uint32),
                ("patch_bits", ctypes.c_uint32), ("pad0", ctypes.c_uint32)]


class ProxyCandidates:
    """A proxy scene resident on one GPU and its candidate buffers."""

    FIELDS = (("object_id", np.uint32), ("patch_id", np.uint32), ("slab_id", np.uint32), ("proxy_type", np.uint8),
              ("t0", np.float64), ("t1", np.float64), ("bounds", np.float64), ("motion_bound", np.float64))

    def __init__(self, scene: dict, device: str | torch.device = "cuda", raw_capacity: int | None = None):
        self.lib = _lib.load()
        self.device = d = torch.device(device)
        self.query_id = int(scene["query_id"])
        self.n = int(scene["n"])
        self.arrays = {}
        for k, dt in self.FIELDS:
            v = scene[k]
            if torch.is_tensor(v):  # already on the device (a built proxy scene)
                if v.device != d or not v.is_contiguous() or v.element_size() != np.dtype(dt).itemsize:
                    raise ValueError(f"proxy field {k}: expected a contiguous {np.dtype(dt)} tensor on {d}")
                self.arrays[k] = v
                continue
            a = np.ascontiguousarray(v, dtype=dt)
            self.arrays[k] = torch.from_numpy(a.view(np.uint8).copy()).to(d) if dt == np.uint32 else \
                torch.from_numpy(a).to(d)
        st = ProxySceneStruct()
        st.query_id, st.n = self.query_id, self.n
        for k, _ in self.FIELDS:
            setattr(st, k, self.arrays[k].data_ptr())
        # id widths: from the scene's own hint, or from host arrays; none for other device arrays
        hint = scene.get("id_bits")
        if hint is None and self.n and not any(torch.is_tensor(scene[k]) for k in ("slab_id", "object_id",
                                                                                   "patch_id")):
            hint = tuple(_bits(np.max(scene[k])) for k in ("slab_id", "object_id", "patch_id"))
        st.slab_bits, st.object_bits, st.patch_bits = hint or (0, 0, 0)
        self._struct = st
        self.counts = torch.zeros(4, dtype=torch.int64, device=d)
        self._alloc(max(1024, 4 * self.n) if raw_capacity is None else raw_capacity)


    def _alloc(self, cap: int) -> None:
        d = self.device
        self.cap = max(0, int(cap))  # 0: only count the hits
        self._filled = False  # no run has written the new buffers yet
        self.raw = torch.empty((self.cap, 64), dtype=torch.uint8, device=d)
        self.cand = torch.empty((self.cap, 80), dtype=torch.uint8, device=d)
        ws = int(self.lib.p2c_proxy_candidates_workspace_bytes(self.n, self.cap, self._struct.slab_bits))
        self.ws = torch.empty(ws, dtype=torch.uint8, device=d)

    def fit_capacity(self, margin: float = 1.25, slack: int = 1024) -> int:
        """Size the raw-hit and candidate buffers to the last run's raw hit
        count (x margin + slack): every sort and pass of the next runs covers
        that many entries.  Returns the new capacity."""
        n_raw = int(self.counts[0].item())
        self._alloc(int(n_raw * margin) + slack)
        return self.cap

    def run(self) -> None:
        """Enqueue candidate generation on the current stream (no host sync)."""
        _lib.check(self.lib.p2c_proxy_candidates(ctypes.byref(self._struct), self.raw.data_ptr(), self.cap,
                                                 self.cand.data_ptr(), self.counts.data_ptr(), self.ws.data_ptr(),
                                                 self.ws.numel(), _stream_ptr(self.device)))
        self._filled = True

    def compact(self, raw: np.ndarray) -> np.ndarray:
        """CompactRawCandidates on given raw hits of this scene
        (p2c_compact_raw_candidates): their candidate records, or ValueError
        with the reference's message for the first invalid hit."""
        hits = np.ascontiguousarray(raw, dtype=RAW_HIT_DTYPE)
        n = len(hits)
        d = self.device
        dh = torch.from_numpy(hits.view(np.uint8).reshape(-1).copy()).to(d) if n else None
        out = torch.empty((max(n, 1), 80), dtype=torch.uint8, device=d)
        counts = torch.zeros(4, dtype=torch.int64, device=d)
        ws = torch.empty(int(self.lib.p2c_compact_raw_candidates_workspace_bytes(self.n, n, self._struct.slab_bits)),
                         dtype=torch.uint8, device=d)
        _lib.check(self.lib.p2c_compact_raw_candidates(ctypes.byref(self._struct), dh.data_ptr() if n else None, n,
                                                       out.data_ptr(), counts.data_ptr(), ws.data_ptr(), ws.numel(),
                                                       _stream_ptr(d)))
        c = counts.cpu().numpy().view(np.uint64)
        if int(c[2]) & ERR_ID_BITS:  # a width hint was wrong: again without hints
            hint = (self._struct.slab_bits, self._struct.object_bits, self._struct.patch_bits)
            self._struct.slab_bits = self._struct.object_bits = self._struct.patch_bits = 0
            try:
                return self.compact(raw)
            finally:
                self._struct.slab_bits, self._struct.object_bits, self._struct.patch_bits = hint
        if int(c[2]) & ERR_INVALID_PROXY:
            raise ValueError("proxy scene fails validation (proxy type, finite t0 < t1, finite ordered bounds)")
        if n and int(c[3]) != 0xFFFFFFFFFFFFFFFF:
            raise ValueError(RAW_HIT_ERRORS[int(c[3]) & 15])
        if int(c[2]) & ERR_HIT_COUNT_OVERFLOW:
            raise ValueError("candidate rt_hit_count overflow during compaction")
        return out[:int(c[1])].cpu().numpy().view(CANDIDATE_RECORD_DTYPE).reshape(-1)

    def run_checked(self, max_retries: int = 3, raw_only: bool = False) -> tuple[np.ndarray, np.ndarray]:
        """Run; grow the buffers and re-run on overflow; raise on an invalid
        scene, and unless ``raw_only`` on a hit whose motion bound the
        reference's compaction rejects.  Returns (raw hits, candidates) as
        host record arrays (candidates empty when ``raw_only``)."""
        for _ in range(max_retries + 2):
            self.run()
            c = self.counts.cpu().numpy()
            n_raw, n_cand, err = int(c[0]), int(c[1]), int(c[2])
            if err & ERR_ID_BITS:  # a width hint was wrong: the run is void, drop the hints
                self._struct.slab_bits = self._struct.object_bits = self._struct.patch_bits = 0
                continue
            if err & ERR_INVALID_PROXY:
                raise ValueError("proxy scene fails validation (proxy type, finite t0 < t1, finite ordered bounds)")
            if err & ERR_MOTION_BOUND and not raw_only:
                raise ValueError("raw candidate motion_bound must be finite and non-negative")
            if raw_only:
                n_cand = 0
            if n_raw <= self.cap:
                raw = self.raw[:n_raw].cpu().numpy().view(RAW_HIT_DTYPE).reshape(-1)
                cand = self.cand[:n_cand].cpu().numpy().view(CANDIDATE_RECORD_DTYPE).reshape(-1)
                return raw, cand
            self._alloc(int(n_raw * 1.25) + 1024)
        raise _lib.P2CError("raw candidate buffer kept overflowing")

    def feature_rows_async(self) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """Enqueue the density stats and proposal feature rows of the last
        run's candidates (p2c_proposal_feature_rows, no host sync).  Returns
        device tensors (density 96 B, rows cap x 256 B, error word); rows
        [0, candidate count) are valid."""
        if not self._filled:
            raise RuntimeError("run() the candidates after (re)sizing the buffers before forming feature rows")
        d = self.device
        if getattr(self, "_rows_cap", -1) != self.cap:
            self.rows = torch.empty((max(self.cap, 1), 256), dtype=torch.uint8, device=d)
            self.density = torch.empty(96, dtype=torch.uint8, device=d)
            self.feature_error = torch.zeros(1, dtype=torch.int64, device=d)
            self.feature_ws = torch.empty(int(self.lib.p2c_proposal_feature_rows_workspace_bytes(self.n)),
                                          dtype=torch.uint8, device=d)
            self._rows_cap = self.cap
        _lib.check(self.lib.p2c_proposal_feature_rows(
            ctypes.byref(self._struct), self.cand.data_ptr(), self.cap, self.counts.data_ptr(),
            self.density.data_ptr(), self.rows.data_ptr(), self.feature_error.data_ptr(), self.feature_ws.data_ptr(),
            self.feature_ws.numel(), _stream_ptr(d)))
        return self.density, self.rows, self.feature_error

    def feature_rows(self) -> tuple[np.void, np.ndarray]:
        """Density stats (a DENSITY_DTYPE record) and proposal feature rows
        (FEATURE_ROW_DTYPE) of the last checked run's candidates; ValueError
        on an invalid candidate or one that maps to no proxy."""
        density, rows, err = self.feature_rows_async()
        n_cand = int(self.counts[1].item())
        e = int(err.item())
        if e & 1:
            raise ValueError("a CandidateRecord fails validation")
        if e & 2:
            raise ValueError("candidate does not map to proxy primitives")
        if e & 4:
            raise RuntimeError("a proxy id exceeds the scene's width hint")
        dens = density.cpu().numpy().view(DENSITY_DTYPE)[0]
        return dens, rows[:n_cand].cpu().numpy().view(FEATURE_ROW_DTYPE).reshape(-1)


def proxy_candidates(scene: dict, device: str | torch.device = "cuda") -> tuple[np.ndarray, np.ndarray]:
    return ProxyCandidates(scene, device).run_checked()


# ---------------------------------------------------------------------------
# proxy scene build (p2c_proxy_scene_build)

BUILD_ERRORS = ((1, "patch.local_center contains a non-finite value"),
                (2, "patch.radius must be finite and non-negative"),
                (4, "AABB contains a non-finite bound or its min exceeds its max"),
                (8, "capsule radius must be finite and non-negative"),
                (16, "proxy bounds contain a non-finite value or min exceeds max"))


class MotionSegmentStruct(ctypes.Structure):
    _fields_ = [("t0", ctypes.c_double), ("t1", ctypes.c_double), ("translation_t0", ctypes.c_double * 3),
                ("rotation_t0", ctypes.c_double * 4), ("translation_t1", ctypes.c_double * 3),
                ("rotation_t1", ctypes.c_double * 4)]


class ProxyObjectStruct(ctypes.Structure):
    _fields_ = [("object_id", ctypes.c_uint32), ("proxy_type", ctypes.c_uint32),
                ("slabs_per_motion_segment", ctypes.c_uint32), ("pad0", ctypes.c_uint32), ("eps_proxy", ctypes.c_double),
                ("patch_offset", ctypes.c_int64), ("n_patches", ctypes.c_int64), ("n_segments", ctypes.c_int64),
                ("segments", ctypes.c_void_p)]


class ProxyBuildOutStruct(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("object_id", "patch_id", "slab_id", "motion_segment_id", "proxy_type",
                                               "t0", "t1", "bounds", "motion_bound", "motion_detail",
                                               "capsule_radius")]


class ProxySceneBuild:
    """A ProxySceneBuildInput built into a device-resident proxy scene.

    ``inp`` is the dict of ``scenes.proxy_build_input``: ``query_id`` and
    ``objects``, each with object_id, proxy_type, slabs_per_motion_segment,
    eps_proxy, patch_id[P], local_center[P, 3], radius[P] and segments[M, 16]
    (t0, t1, translation_t0, rotation_t0 xyzw, translation_t1, rotation_t1).
    ``scene()`` returns the proxy arrays as device tensors, the input of
    ``ProxyCandidates`` without a host round trip."""

    def __init__(self, inp: dict, device: str | torch.device = "cuda", detail: bool = True):
        self.lib = _lib.load()
        self.device = d = torch.device(device)
        self.query_id = int(inp["query_id"])
        objs = inp["objects"]
        k = len(objs)
        self._segments = [np.ascontiguousarray(np.asarray(o["segments"], np.float64).reshape(-1, 16)) for o in objs]
        arr = (ProxyObjectStruct * max(k, 1))()
        off = 0
        for i, o in enumerate(objs):
            n_p = len(o["patch_id"])
            arr[i].object_id, arr[i].proxy_type = int(o["object_id"]), int(o["proxy_type"])
            arr[i].slabs_per_motion_segment, arr[i].eps_proxy = int(o["slabs_per_motion_segment"]), float(o["eps_proxy"])
            arr[i].patch_offset, arr[i].n_patches = off, n_p
            arr[i].n_segments = len(self._segments[i])
            arr[i].segments = self._segments[i].ctypes.data if len(self._segments[i]) else None
            off += n_p
        self._objects, self.n_objects = arr, k
        self.n_patch_entries = off
        max_slab = max((len(self._segments[i]) * int(o["slabs_per_motion_segment"]) - 1 for i, o in enumerate(objs)),
                       default=0)
        max_obj = max((int(o["object_id"]) for o in objs), default=0)
        max_patch = max((int(np.max(o["patch_id"])) for o in objs if len(o["patch_id"])), default=0)
        self.id_bits = (_bits(max(max_slab, 0)), _bits(max_obj), _bits(max_patch))
        cat = (lambda key, dt, w: np.ascontiguousarray(np.concatenate(
            [np.asarray(o[key], dt).reshape(-1, w) for o in objs]) if objs else np.zeros((0, w), dt)))
        self.patch_id = torch.from_numpy(cat("patch_id", np.uint32, 1).view(np.int32).reshape(-1)).to(d)
        self.patch_center = torch.from_numpy(cat("local_center", np.float64, 3)).to(d)
        self.patch_radius = torch.from_numpy(cat("radius", np.float64, 1).reshape(-1)).to(d)
        n = int(self.lib.p2c_proxy_scene_count(arr, k))
        if n < 0:
            raise ValueError(_lib.last_error())
        self.n = n
        self.out = {"object_id": torch.empty(n, dtype=torch.int32, device=d),
                    "patch_id": torch.empty(n, dtype=torch.int32, device=d),
                    "slab_id": torch.empty(n, dtype=torch.int32, device=d),
                    "motion_segment_id": torch.empty(n, dtype=torch.int32, device=d),
                    "proxy_type": torch.empty(n, dtype=torch.uint8, device=d),
                    "t0": torch.empty(n, dtype=torch.float64, device=d),
                    "t1": torch.empty(n, dtype=torch.float64, device=d),
                    "bounds": torch.empty((n, 6), dtype=torch.float64, device=d),
                    "motion_bound": torch.empty((n, 4), dtype=torch.float64, device=d)}
        if detail:
            self.out["motion_detail"] = torch.empty((n, 8), dtype=torch.float64, device=d)
            self.out["capsule_radius"] = torch.empty(n, dtype=torch.float64, device=d)
        st = ProxyBuildOutStruct()
        for f, _ in ProxyBuildOutStruct._fields_:
            setattr(st, f, self.out[f].data_ptr() if f in self.out else None)
        self._out_struct = st
        self.error_word = torch.zeros(1, dtype=torch.int64, device=d)
        self.ws = torch.empty(int(self.lib.p2c_proxy_scene_build_workspace_bytes(arr, k)), dtype=torch.uint8, device=d)

    def run(self) -> None:
        """Enqueue the build on the current stream (no host sync); raises
        ValueError for an invalid object, segment or slab partition."""
        _lib.check(self.lib.p2c_proxy_scene_build(
            self.query_id, self._objects, self.n_objects, self.patch_id.data_ptr(), self.patch_center.data_ptr(),
            self.patch_radius.data_ptr(), self.n_patch_entries, self.n, ctypes.byref(self._out_struct),
            self.error_word.data_ptr(), self.ws.data_ptr(), self.ws.numel(), _stream_ptr(self.device)))

    def run_checked(self) -> dict:
        """Build, then raise ValueError on a per-patch failure; returns
        ``scene()``."""
        self.run()
        e = int(self.error_word.item())
        for bit, msg in BUILD_ERRORS:
            if e & bit:
                raise ValueError(msg)
        return self.scene()

    def scene(self) -> dict:
        """The built proxies as device tensors (uint32 fields as int32), with
        the widths of their slab, object and patch ids."""
        sc = {"query_id": self.query_id, "n": self.n, "id_bits": self.id_bits}
        sc.update(self.out)
        return sc

    def to_host(self) -> dict:
        """The built proxies as numpy arrays with the reference's types."""
        sc = {"query_id": self.query_id, "n": self.n}
        for k, v in self.out.items():
            a = v.cpu().numpy()
            sc[k] = a.view(np.uint32) if a.dtype == np.int32 else a
        return sc


def runtime_feature_rows(candidates, primitive_count: int, raw_hit_count: int, compact_candidate_count: int,
                         masks: dict | None = None, device: str | torch.device = "cuda") -> np.ndarray:
    """Proposal feature rows from candidate records alone (the runtime form,
    p2c_runtime_feature_rows).  ``candidates``: CANDIDATE_RECORD_DTYPE records
    or a (n, 80) uint8 device tensor; ``masks``: query id -> conservative
    family mask.  Returns FEATURE_ROW_DTYPE records; ValueError on an invalid
    candidate or a zero primitive count."""
    lib = _lib.load()
    d = torch.device(device)
    if torch.is_tensor(candidates):
        cand = candidates.to(d).contiguous()
    else:
        a = np.ascontiguousarray(candidates).view(np.uint8).reshape(-1, 80)
        cand = torch.from_numpy(a.copy()).to(d)
    n = cand.shape[0]
    keys = sorted(int(k) for k in (masks or {}))
    mq = torch.tensor(np.array(keys, np.uint64).view(np.int64), device=d) if keys else None
    mv = torch.tensor(np.array([int(masks[k]) for k in keys], np.uint32).view(np.int32), device=d) if keys else None
    rows = torch.empty((max(n, 1), 256), dtype=torch.uint8, device=d)
    err = torch.zeros(1, dtype=torch.int64, device=d)
    _lib.check(lib.p2c_runtime_feature_rows(cand.data_ptr() if n else None, n, int(primitive_count), int(raw_hit_count),
                                            int(compact_candidate_count), mq.data_ptr() if keys else None,
                                            mv.data_ptr() if keys else None, len(keys), rows.data_ptr(), err.data_ptr(),
                                            _stream_ptr(d)))
    if int(err.item()) & 1:
        raise ValueError("a CandidateRecord fails validation")
    return rows[:n].cpu().numpy().view(FEATURE_ROW_DTYPE).reshape(-1)
