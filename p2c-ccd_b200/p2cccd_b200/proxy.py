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
from .records import CANDIDATE_RECORD_DTYPE, RAW_HIT_DTYPE

ERR_INVALID_PROXY, ERR_MOTION_BOUND, ERR_OVERFLOW = 1, 2, 4


class ProxySceneStruct(ctypes.Structure):
    _fields_ = [("query_id", ctypes.c_uint64), ("n", ctypes.c_int64), ("object_id", ctypes.c_void_p),
                ("patch_id", ctypes.c_void_p), ("slab_id", ctypes.c_void_p), ("proxy_type", ctypes.c_void_p),
                ("t0", ctypes.c_void_p), ("t1", ctypes.c_void_p), ("bounds", ctypes.c_void_p),
                ("motion_bound", ctypes.c_void_p)]


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
            a = np.ascontiguousarray(scene[k], dtype=dt)
            self.arrays[k] = torch.from_numpy(a.view(np.uint8).copy()).to(d) if dt == np.uint32 else \
                torch.from_numpy(a).to(d)
        st = ProxySceneStruct()
        st.query_id, st.n = self.query_id, self.n
        for k, _ in self.FIELDS:
            setattr(st, k, self.arrays[k].data_ptr())
        self._struct = st
        self.counts = torch.zeros(4, dtype=torch.int64, device=d)
        self._alloc(max(1024, 4 * self.n) if raw_capacity is None else raw_capacity)

    def _alloc(self, cap: int) -> None:
        d = self.device
        self.cap = max(0, int(cap))  # 0: only count the hits
        self.raw = torch.empty((self.cap, 64), dtype=torch.uint8, device=d)
        self.cand = torch.empty((self.cap, 80), dtype=torch.uint8, device=d)
        self.ws = torch.empty(int(self.lib.p2c_proxy_candidates_workspace_bytes(self.n, self.cap)), dtype=torch.uint8,
                              device=d)

    def run(self) -> None:
        """Enqueue candidate generation on the current stream (no host sync)."""
        _lib.check(self.lib.p2c_proxy_candidates(ctypes.byref(self._struct), self.raw.data_ptr(), self.cap,
                                                 self.cand.data_ptr(), self.counts.data_ptr(), self.ws.data_ptr(),
                                                 self.ws.numel(), _stream_ptr(self.device)))

    def run_checked(self, max_retries: int = 3, raw_only: bool = False) -> tuple[np.ndarray, np.ndarray]:
        """Run; grow the buffers and re-run on overflow; raise on an invalid
        scene, and unless ``raw_only`` on a hit whose motion bound the
        reference's compaction rejects.  Returns (raw hits, candidates) as
        host record arrays (candidates empty when ``raw_only``)."""
        for _ in range(max_retries + 1):
            self.run()
            c = self.counts.cpu().numpy()
            n_raw, n_cand, err = int(c[0]), int(c[1]), int(c[2])
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


def proxy_candidates(scene: dict, device: str | torch.device = "cuda") -> tuple[np.ndarray, np.ndarray]:
    return ProxyCandidates(scene, device).run_checked()
