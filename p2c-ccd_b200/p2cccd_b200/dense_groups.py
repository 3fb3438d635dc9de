"""The candidate-group early-stop replay on the device
(p2c_dense_group_early_stop): RunDenseGroupExactEarlyStop
(common/group_scheduler.cpp:60-239) over rows parsed as the binding
RunNativeDenseGroupExactEarlyStopOrThrow parses them
(bindings/py_module.cpp:1179-1311), with the result dict of that binding."""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from .certify import _stream_ptr
from .records import DENSE_GROUP_STATS_DTYPE

INTERVAL_BINS = 8  # kProposalIntervalBinCount

_ROW_ERRORS = {1: "dense group candidate ids must be non-zero",
               2: "dense group candidate contains a non-finite field"}


class DenseGroupConfigStruct(ctypes.Structure):
    _fields_ = [("uncertainty_fallback_threshold", ctypes.c_float),
                ("representative_attempt_limit", ctypes.c_uint32),
                ("interval_miss_penalty_scale", ctypes.c_double), ("preserve_input_order", ctypes.c_int32),
                ("query_bits", ctypes.c_int32)]


def _require(arrays: dict, key: str, dtype, shape: tuple) -> np.ndarray:
    """RequireArray1D / RequireArray2D (py_module.cpp:756-790): a forced cast
    to the element type, then the exact shape."""
    if key not in arrays or arrays[key] is None:
        raise ValueError("missing or invalid array field: " + key)
    try:
        a = np.ascontiguousarray(arrays[key], dtype=dtype)
    except (TypeError, ValueError):
        raise ValueError("missing or invalid array field: " + key) from None
    if a.shape != shape:
        raise ValueError(f"{key} must have shape [{', '.join(str(x) for x in shape)}]")
    return a


def parse_arrays(feature_arrays: dict, prediction_arrays: dict) -> dict:
    """The binding's array checks, in its order."""
    if "query_id" not in feature_arrays:
        raise ValueError("missing or invalid array field: query_id")
    n = len(feature_arrays["query_id"])
    return {"query_id": _require(feature_arrays, "query_id", np.uint64, (n,)),
            "candidate_id": _require(feature_arrays, "candidate_id", np.uint64, (n,)),
            "cost_target": _require(feature_arrays, "cost_target", np.float32, (n,)),
            "oracle_trace": _require(feature_arrays, "oracle_trace", np.float64, (n, 8)),
            "interval_scores": _require(prediction_arrays, "interval_scores", np.float32, (n, INTERVAL_BINS)),
            "priority_score": _require(prediction_arrays, "priority_score", np.float32, (n,)),
            "cost_score": _require(prediction_arrays, "cost_score", np.float32, (n,)),
            "uncertainty_score": _require(prediction_arrays, "uncertainty_score", np.float32, (n,))}


_ORDER = ("query_id", "candidate_id", "cost_target", "oracle_trace", "interval_scores", "priority_score", "cost_score",
          "uncertainty_score")


class DenseGroupEarlyStop:
    """Device buffers for up to ``capacity`` rows; ``run`` enqueues the replay
    on device tensors (no host sync) and leaves the stats in ``self.stats``."""

    def __init__(self, capacity: int, device: str | torch.device = "cuda"):
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.capacity = int(capacity)
        self.ws = torch.empty(int(self.lib.p2c_dense_group_early_stop_workspace_bytes(self.capacity)),
                              dtype=torch.uint8, device=self.device)
        self.stats = torch.zeros(DENSE_GROUP_STATS_DTYPE.itemsize, dtype=torch.uint8, device=self.device)

    def run(self, tensors: dict, n: int, *, threshold: float = 0.75, limit: int = 3, penalty: float = 0.22,
            preserve: bool = False, query_bits: int = 64) -> None:
        if n > self.capacity:
            raise ValueError(f"{n} rows exceed the capacity {self.capacity}")
        cfg = DenseGroupConfigStruct(float(np.float32(threshold)), int(limit), float(penalty), int(bool(preserve)),
                                     int(query_bits))
        ptrs = [tensors[k].data_ptr() if n else None for k in _ORDER]
        _lib.check(self.lib.p2c_dense_group_early_stop(int(n), *ptrs, ctypes.byref(cfg), self.stats.data_ptr(),
                                                       self.ws.data_ptr(), self.ws.numel(), _stream_ptr(self.device)))

    def result(self) -> np.void:
        st = self.stats.cpu().numpy().view(DENSE_GROUP_STATS_DTYPE)[0]
        if st["error_kind"]:
            raise ValueError(_ROW_ERRORS[int(st["error_kind"])])
        return st


def upload(rows: dict, device: str | torch.device = "cuda") -> dict:
    """Parsed host rows as device tensors (one copy each)."""
    d = torch.device(device)
    out = {}
    for k in _ORDER:
        a = rows[k]
        t = torch.from_numpy(a.view(np.int64) if a.dtype == np.uint64 else a)
        out[k] = t.to(d, non_blocking=False)
    return out


def _query_bits(q: np.ndarray) -> int:
    return max(1, int(q.max()).bit_length()) if len(q) else 1


def early_stop(feature_arrays: dict, prediction_arrays: dict, uncertainty_fallback_threshold: float = 0.75,
               representative_attempt_limit: int = 3, interval_miss_penalty_scale: float = 0.22,
               preserve_input_order: bool = False, device: str | torch.device = "cuda") -> dict:
    """RunNativeDenseGroupExactEarlyStopOrThrow's result dict from the device
    replay (totals bit-identical to the reference's; host timings measured
    here around the parse, the upload and the synchronised device run)."""
    if int(representative_attempt_limit) < 0:
        raise TypeError("representative_attempt_limit must be an unsigned 32-bit integer")
    t0 = time.perf_counter()
    rows = parse_arrays(feature_arrays, prediction_arrays)
    n = len(rows["query_id"])
    t1 = time.perf_counter()
    runner = DenseGroupEarlyStop(max(n, 1), device)
    tens = upload(rows, device) if n else {}
    t2 = time.perf_counter()
    runner.run(tens, n, threshold=uncertainty_fallback_threshold, limit=representative_attempt_limit,
               penalty=interval_miss_penalty_scale, preserve=preserve_input_order,
               query_bits=_query_bits(rows["query_id"]))
    st = runner.result()
    t3 = time.perf_counter()
    return result_dict(st, parse_ms=(t1 - t0) * 1e3, native_ms=(t3 - t1) * 1e3, upload_ms=(t2 - t1) * 1e3)


def result_dict(st: np.void, parse_ms: float = 0.0, native_ms: float = 0.0, upload_ms: float = 0.0) -> dict:
    """The binding's result dict (py_module.cpp:1264-1310) from the stats."""
    pos = int(st["positive_group_count"])
    npc, lec = int(st["no_proposal_exact_calls"]), int(st["learned_exact_calls"])
    npw, lew = float(st["no_proposal_exact_work"]), float(st["learned_exact_work"])
    out = {k: int(st[k]) for k in ("candidate_count", "group_count", "positive_group_count",
                                   "no_proposal_exact_calls")}
    out["no_proposal_exact_work"] = npw
    for k in ("learned_exact_calls", "learned_fallback_calls", "learned_interval_hit_count",
              "learned_interval_miss_count"):
        out[k] = int(st[k])
    out["learned_exact_work"] = lew
    out["first_positive_rank_mean"] = 0.0 if pos == 0 else float(st["first_positive_rank_sum"]) / float(pos)
    out["cost_weighted_first_positive_mean"] = (0.0 if pos == 0 else
                                                float(st["cost_before_first_positive_sum"]) / float(pos))
    for k in ("tp", "tn", "fp", "fn", "reordered_count", "high_uncertainty_group_count"):
        out[k] = int(st[k])
    out["parse_ms"] = float(parse_ms)
    out["schedule_ms"] = 0.0  # sort and walk are one device sequence; its time is exact_ms
    out["exact_ms"] = float(native_ms - upload_ms)
    out["native_driver_ms"] = float(native_ms)
    out["native_total_ms"] = float(parse_ms + native_ms)
    out["exact_call_reduction"] = 0.0 if npc == 0 else 1.0 - float(lec) / float(npc)
    out["exact_work_reduction"] = 0.0 if npw <= 0.0 else 1.0 - lew / npw
    return out


def ordered_sum(terms: torch.Tensor) -> torch.Tensor:
    """p2c_ordered_sum: the left-to-right double sum of non-negative terms (a
    CUDA float64 tensor), bit-identical to a sequential loop; returns a
    one-element device tensor (no host sync)."""
    lib = _lib.load()
    t = terms.contiguous()
    if t.dtype != torch.float64 or not t.is_cuda:
        raise TypeError("terms must be a CUDA float64 tensor")
    out = torch.empty(1, dtype=torch.float64, device=t.device)
    _lib.check(lib.p2c_ordered_sum(t.data_ptr() if t.numel() else None, t.numel(), out.data_ptr(),
                                   _stream_ptr(t.device)))
    return out
