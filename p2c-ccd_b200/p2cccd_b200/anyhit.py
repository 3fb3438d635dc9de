"""Scheduled any-hit over candidate groups with conservative fallback replay.

The device form of the scene tool's ``RunScheduledAnyHitRows``
(tools/scene_object_envelope_native_ti_walltime.cpp:1283-1410): groups are
unordered object pairs; each group's top-K candidates by the caller's scores
are certified in score order until the first hit, then every other candidate
of a group without a hit is replayed in candidate order until the first hit.
A hit is a certificate that is not a separation (collision, or undecided
under the conservative mapping).  Scores come from the caller's scheduler and
are consumed unchanged.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .certify import CertConfig, _stream_ptr

ANYHIT_SUMMARY_DTYPE = np.dtype([
    ("candidates", "<u8"), ("groups", "<u8"), ("detected_groups", "<u8"), ("proposal_calls", "<u8"),
    ("fallback_calls", "<u8"), ("fallback_groups", "<u8"), ("first_hit_rank_sum", "<u8"),
    ("speculative", "<u8"), ("error_word", "<u8"),
])

FAMILY = {"vf": 1, "ee": 2}

ERR_BUDGET, ERR_GEOMETRY, ERR_OBJECT, ERR_NAN_SCORE = 1, 4, 8, 16


class GroupAnyHit:
    """Workspace and outputs of ``p2c_group_anyhit`` for one family of one scene.

    ``scene_struct`` is the ``p2c_scene`` of a ``ScenePipeline`` (or any
    struct of that layout whose device arrays outlive this object).
    """

    def __init__(self, scene_struct, n_obj: int, family: str, capacity: int, device: str | torch.device = "cuda"):
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.scene_struct = scene_struct
        self.n_obj = int(n_obj)
        self.family = FAMILY[family]
        self.capacity = max(1, int(capacity))
        d = self.device
        nbytes = int(self.lib.p2c_group_anyhit_workspace_bytes(self.capacity, self.n_obj))
        if nbytes == 0:
            raise ValueError("scene n_obj must be at least 1 for candidate groups")
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=d)
        g = self.n_obj * self.n_obj
        self.evaluated = torch.zeros(self.capacity, dtype=torch.uint8, device=d)
        self.hit = torch.zeros(self.capacity, dtype=torch.uint8, device=d)
        self.group_detected = torch.zeros(g, dtype=torch.uint8, device=d)
        self.group_proposal_calls = torch.zeros(g, dtype=torch.int64, device=d)
        self.group_fallback_calls = torch.zeros(g, dtype=torch.int64, device=d)
        self.summary = torch.zeros(ANYHIT_SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device=d)

    def run(self, pairs: torch.Tensor, count: torch.Tensor, scores: torch.Tensor, top_k: int,
            config: CertConfig = CertConfig(), interval: tuple[float, float] = (0.0, 1.0)) -> None:
        """Enqueue the any-hit on the current stream (no host sync).

        ``pairs`` (int64, device) holds at least ``capacity`` entries of which
        the first ``min(count[0], capacity)`` are candidates; ``count`` is a
        device int64 tensor; ``scores`` (float64, device) is positional."""
        if pairs.numel() < self.capacity or scores.numel() < self.capacity:
            raise ValueError("pairs and scores must hold at least capacity entries")
        if scores.dtype != torch.float64 or pairs.dtype != torch.int64 or count.dtype != torch.int64:
            raise ValueError("pairs/count must be int64 and scores float64 device tensors")
        cfg = config.c()
        _lib.check(self.lib.p2c_group_anyhit(
            ctypes.byref(self.scene_struct), self.family, pairs.data_ptr(), self.capacity, count.data_ptr(),
            scores.data_ptr(), int(top_k), float(interval[0]), float(interval[1]), ctypes.byref(cfg),
            self.evaluated.data_ptr(), self.hit.data_ptr(), self.group_detected.data_ptr(),
            self.group_proposal_calls.data_ptr(), self.group_fallback_calls.data_ptr(), self.summary.data_ptr(),
            self.ws.data_ptr(), self.ws.numel(), _stream_ptr(self.device)))

    def read_summary(self) -> dict:
        s = self.summary.cpu().numpy().view(ANYHIT_SUMMARY_DTYPE)[0]
        return {k: int(s[k]) for k in ANYHIT_SUMMARY_DTYPE.names}

    def read_groups(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(detected, proposal calls, fallback calls) per group lo * n_obj + hi."""
        return (self.group_detected.cpu().numpy(), self.group_proposal_calls.cpu().numpy(),
                self.group_fallback_calls.cpu().numpy())

    def read_candidates(self, n: int) -> tuple[np.ndarray, np.ndarray]:
        """(evaluated phase 0/1/2, hit flag) of the first n candidates."""
        return self.evaluated[:n].cpu().numpy(), self.hit[:n].cpu().numpy()
