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


def stub_scores(pairs: torch.Tensor, count: torch.Tensor | None, family: int, seed: int,
                out: torch.Tensor) -> torch.Tensor:
    """Fill ``out`` (float64, device, positional over ``pairs``) with the
    seeded scheduler stub's scores (p2c_stub_scores): a uniform score per
    (seed, family, pair key).  Asynchronous on the current stream."""
    lib = _lib.load()
    cap = min(pairs.numel(), out.numel())
    _lib.check(lib.p2c_stub_scores(pairs.data_ptr(), None if count is None else count.data_ptr(), cap, int(family),
                                   int(seed) & ((1 << 64) - 1), out.data_ptr(), _stream_ptr(out.device)))
    return out


def stub_score_host(seed: int, family: int, key: int) -> float:
    """The stub's score of one candidate computed on the host (the same
    splitmix64 finaliser as the device), for checks."""
    m = (1 << 64) - 1
    x = (seed ^ ((key * 0x9E3779B97F4A7C15) & m) ^ ((family << 62) & m)) & m
    x = (x + 0x9E3779B97F4A7C15) & m
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & m
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & m
    x ^= x >> 31
    return (x >> 11) * (1.0 / 9007199254740992.0)


class BatchAnyHit:
    """Workspace and outputs of ``p2c_batch_anyhit`` for a batch scene table
    (``BATCH_SCENE_DTYPE`` rows, host copy and device copy).  One summary per
    (scene, family); scores from the scheduler stub with one seed per scene,
    or from per-(scene, family) device score tensors."""

    def __init__(self, table_host: np.ndarray, table_dev: torch.Tensor, family_mask: int = 3,
                 device: str | torch.device = "cuda", keep_candidates: bool = False):
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.table_host = table_host
        self.table_dev = table_dev
        self.n = len(table_host)
        self.family_mask = int(family_mask)
        d = self.device
        nbytes = int(self.lib.p2c_batch_anyhit_workspace_bytes(table_host.ctypes.data, self.n, self.family_mask))
        if nbytes == 0:
            raise ValueError("batch any-hit: invalid table or family mask")
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=d)
        self.summaries = torch.zeros((2 * self.n, ANYHIT_SUMMARY_DTYPE.itemsize), dtype=torch.uint8, device=d)
        caps = [(int(r["vf_cap"]) if family_mask & 1 else 0, int(r["ee_cap"]) if family_mask & 2 else 0)
                for r in table_host]
        self.n_obj = [int(r["n_obj"]) for r in table_host]
        groups = sum(k * k for k in self.n_obj) * ((family_mask & 1) + ((family_mask >> 1) & 1))
        self.cand_off = np.concatenate([[0], np.cumsum([c[0] for c in caps] + [c[1] for c in caps])]).astype(np.int64)
        self.group_off = np.concatenate([[0], np.cumsum([k * k if family_mask & 1 else 0 for k in self.n_obj] +
                                                        [k * k if family_mask & 2 else 0 for k in self.n_obj])])
        self.group_detected = torch.zeros(max(1, groups), dtype=torch.uint8, device=d)
        total = int(self.cand_off[-1])
        self.evaluated = torch.zeros(max(1, total), dtype=torch.uint8, device=d) if keep_candidates else None
        self.hit = torch.zeros(max(1, total), dtype=torch.uint8, device=d) if keep_candidates else None
        self.seeds = torch.zeros(self.n, dtype=torch.int64, device=d)

    def run(self, top_k: int, config: CertConfig = CertConfig(), interval: tuple[float, float] = (0.0, 1.0),
            seeds: torch.Tensor | None = None, scores_ptrs: torch.Tensor | None = None) -> None:
        """Enqueue on the current stream (no host sync)."""
        cfg = config.c()
        sd = self.seeds if seeds is None else seeds
        _lib.check(self.lib.p2c_batch_anyhit(
            self.table_host.ctypes.data, self.table_dev.data_ptr(), self.n, self.family_mask,
            None if scores_ptrs is None else scores_ptrs.data_ptr(), sd.data_ptr(), int(top_k), float(interval[0]),
            float(interval[1]), ctypes.byref(cfg), self.summaries.data_ptr(), self.group_detected.data_ptr(),
            None if self.evaluated is None else self.evaluated.data_ptr(),
            None if self.hit is None else self.hit.data_ptr(), self.ws.data_ptr(), self.ws.numel(),
            _stream_ptr(self.device)))

    def read_summaries(self) -> list[dict]:
        """Per scene: {"vf": summary, "ee": summary} (None for a family not run)."""
        raw = self.summaries.cpu().numpy().reshape(-1).view(ANYHIT_SUMMARY_DTYPE)
        out = []
        for s in range(self.n):
            row = {}
            for f, name in ((0, "vf"), (1, "ee")):
                row[name] = ({k: int(raw[2 * s + f][k]) for k in ANYHIT_SUMMARY_DTYPE.names}
                             if self.family_mask & (1 << f) else None)
            out.append(row)
        return out

    def group_detected_of(self, s: int, family: int) -> np.ndarray:
        """Scene s's detected flags of one family (n_obj * n_obj, index lo * n_obj + hi)."""
        k = (family - 1) * self.n + s
        a, b = int(self.group_off[k]), int(self.group_off[k + 1])
        return self.group_detected[a:b].cpu().numpy()

    def candidates_of(self, s: int, family: int, n: int) -> tuple[np.ndarray, np.ndarray]:
        """Scene s's (evaluated phase, hit) flags of its first n candidates of one family."""
        k = (family - 1) * self.n + s
        a = int(self.cand_off[k])
        return self.evaluated[a:a + n].cpu().numpy(), self.hit[a:a + n].cpu().numpy()


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
