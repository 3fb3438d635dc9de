"""Batch interval certificates on the GPU (device and host buffer forms).

Device form: primitives are a CUDA ``torch.uint8`` tensor of shape (n, 240)
holding reference-layout records; results come back as a CUDA ``torch.uint8``
tensor of shape (n, 72) (``records.INTERVAL_RESULT_DTYPE`` once on the host).
Work is enqueued on the current torch stream.

Host form: numpy record arrays in, numpy record arrays out, synchronous, with
library-owned device memory - the ownership model of the reference's
``evaluate_point_triangle_batch_cuda`` (cpp/bindings/py_module.cpp:1972-1983).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .records import (CERTIFY_STATS_DTYPE, EDGE_EDGE_DTYPE, FAMILY_EDGE_EDGE, FAMILY_POINT_TRIANGLE,
                      INTERVAL_RESULT_DTYPE, POINT_TRIANGLE_DTYPE)


@dataclass(frozen=True)
class CertConfig:
    """CertificateEngineConfig (certificate_engine.h:56-60) with its defaults."""
    eps_time: float = 1.0e-4
    eps_space: float = 1.0e-6
    max_subdivision_depth: int = 32

    def c(self) -> _lib.CertConfig:
        return _lib.make_config(self.eps_time, self.eps_space, self.max_subdivision_depth)


def _stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _as_records(t: torch.Tensor) -> torch.Tensor:
    if t.dtype != torch.uint8 or t.dim() != 2 or t.shape[1] != 240 or not t.is_contiguous():
        raise ValueError("primitive tensor must be a contiguous uint8 tensor of shape (n, 240)")
    if not t.is_cuda:
        raise ValueError("primitive tensor must live on a CUDA device")
    return t


def records_to_device(rec: np.ndarray, device: str | torch.device = "cuda") -> torch.Tensor:
    """Copy a numpy record array (240-byte records) to a CUDA uint8 tensor."""
    raw = np.ascontiguousarray(rec).view(np.uint8).reshape(len(rec), 240)
    return torch.from_numpy(raw).to(device)


def results_to_numpy(t: torch.Tensor) -> np.ndarray:
    """CUDA/CPU uint8 (n, 72) tensor -> INTERVAL_RESULT_DTYPE array."""
    return t.detach().cpu().contiguous().numpy().view(INTERVAL_RESULT_DTYPE).reshape(-1)


class Workspace:
    """Device scratch of one certification launch (owned by the caller)."""

    def __init__(self, device: torch.device):
        lib = _lib.load()
        self.bytes = int(lib.p2c_certify_workspace_bytes(0))
        self.buf = torch.empty(self.bytes, dtype=torch.uint8, device=device)

    def stats(self) -> np.ndarray:
        return self.buf[: CERTIFY_STATS_DTYPE.itemsize].cpu().numpy().view(CERTIFY_STATS_DTYPE)[0]


def certify_batch(prims: torch.Tensor, family: int, interval_t0: float = 0.0, interval_t1: float = 1.0,
                  config: CertConfig = CertConfig(), out: torch.Tensor | None = None,
                  workspace: Workspace | None = None) -> torch.Tensor:
    """Certify every primitive of one family; returns the (n, 72) result tensor.

    Asynchronous on the current stream.  Invalid primitives get an undecided
    InvalidInput record (``certify_batch_checked`` raises instead).
    """
    lib = _lib.load()
    prims = _as_records(prims)
    n = prims.shape[0]
    dev = prims.device
    if out is None:
        out = torch.empty((n, 72), dtype=torch.uint8, device=dev)
    ws = workspace if workspace is not None else Workspace(dev)
    cfg = config.c()
    fn = lib.p2c_certify_pt_batch if family == FAMILY_POINT_TRIANGLE else lib.p2c_certify_ee_batch
    _lib.check(fn(prims.data_ptr(), n, float(interval_t0), float(interval_t1), ctypes.byref(cfg),
                  out.data_ptr(), ws.buf.data_ptr(), ws.bytes, None, _stream_ptr(dev)))
    return out


def certify_batch2(pt: torch.Tensor, ee: torch.Tensor, interval_t0: float = 0.0, interval_t1: float = 1.0,
                   config: CertConfig = CertConfig(), out_pt: torch.Tensor | None = None,
                   out_ee: torch.Tensor | None = None, workspace: Workspace | None = None):
    """Both families in one launch; returns (pt results, ee results).  Asynchronous."""
    lib = _lib.load()
    pt, ee = _as_records(pt), _as_records(ee)
    dev = pt.device
    n_pt, n_ee = pt.shape[0], ee.shape[0]
    out_pt = torch.empty((n_pt, 72), dtype=torch.uint8, device=dev) if out_pt is None else out_pt
    out_ee = torch.empty((n_ee, 72), dtype=torch.uint8, device=dev) if out_ee is None else out_ee
    ws = workspace if workspace is not None else Workspace(dev)
    cfg = config.c()
    _lib.check(lib.p2c_certify_batch2(pt.data_ptr(), n_pt, ee.data_ptr(), n_ee, float(interval_t0),
                                      float(interval_t1), ctypes.byref(cfg), out_pt.data_ptr(),
                                      out_ee.data_ptr(), ws.buf.data_ptr(), ws.bytes, None, _stream_ptr(dev)))
    return out_pt, out_ee


def probe_fp64_rate(device: torch.device, iters: int = 4096, repeats: int = 5) -> float:
    """Measured FP64 (separately rounded mul + add) rate of this GPU, ops/s (best of repeats)."""
    lib = _lib.load()
    buf = torch.zeros(1, dtype=torch.float64, device=device)
    ops = ctypes.c_longlong(0)
    best = 0.0
    stream = _stream_ptr(device)
    for _ in range(repeats + 1):
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record()
        _lib.check(lib.p2c_probe_fp64(buf.data_ptr(), iters, ctypes.byref(ops), stream))
        end.record()
        end.synchronize()
        best = max(best, ops.value / (start.elapsed_time(end) * 1e-3))
    return best


def certify_batch_host(records: np.ndarray, interval_t0: float = 0.0, interval_t1: float = 1.0,
                       config: CertConfig = CertConfig()) -> np.ndarray:
    """Host-owned batch (the reference's ownership model); raises ValueError on invalid input."""
    lib = _lib.load()
    rec = np.ascontiguousarray(records)
    if rec.dtype == POINT_TRIANGLE_DTYPE:
        fn = lib.p2c_certify_pt_batch_host
    elif rec.dtype == EDGE_EDGE_DTYPE:
        fn = lib.p2c_certify_ee_batch_host
    else:
        raise ValueError("records must use POINT_TRIANGLE_DTYPE or EDGE_EDGE_DTYPE")
    out = np.zeros(len(rec), dtype=INTERVAL_RESULT_DTYPE)
    cfg = config.c()
    _lib.check(fn(rec.ctypes.data if len(rec) else None, len(rec), float(interval_t0), float(interval_t1),
                  ctypes.byref(cfg), out.ctypes.data if len(rec) else None))
    return out


def certify_batch_cpu(records: np.ndarray, interval_t0: float = 0.0, interval_t1: float = 1.0,
                      config: CertConfig = CertConfig()) -> np.ndarray:
    """The library's CPU certifier (p2c_certify_*_batch_cpu) on host records:
    the CPU side of the CPU/CUDA cross-check.  Never a fallback of the GPU path."""
    lib = _lib.load()
    rec = np.ascontiguousarray(records)
    fn = lib.p2c_certify_pt_batch_cpu if rec.dtype.names[0] == "point_id" else lib.p2c_certify_ee_batch_cpu
    out = np.zeros(len(rec), dtype=INTERVAL_RESULT_DTYPE)
    cfg = config.c()
    _lib.check(fn(rec.ctypes.data if len(rec) else None, len(rec), float(interval_t0), float(interval_t1),
                  ctypes.byref(cfg), out.ctypes.data if len(rec) else None))
    return out


def census(pt: torch.Tensor | None, ee: torch.Tensor | None, interval_t0: float = 0.0,
           interval_t1: float = 1.0, config: CertConfig = CertConfig()) -> dict:
    """Run the lane-local depth-first census launch (the reference's node set)
    and return its counters (nodes, distance evaluations, FP64 operations) and
    results.  Synchronous."""
    lib = _lib.load()
    dev = (pt if pt is not None else ee).device
    n_pt = 0 if pt is None else _as_records(pt).shape[0]
    n_ee = 0 if ee is None else _as_records(ee).shape[0]
    out_pt = torch.empty((n_pt, 72), dtype=torch.uint8, device=dev)
    out_ee = torch.empty((n_ee, 72), dtype=torch.uint8, device=dev)
    ws = Workspace(dev)
    cfg = config.c()
    _lib.check(lib.p2c_certify_census(pt.data_ptr() if n_pt else None, n_pt, ee.data_ptr() if n_ee else None,
                                      n_ee, float(interval_t0), float(interval_t1), ctypes.byref(cfg),
                                      out_pt.data_ptr() if n_pt else None, out_ee.data_ptr() if n_ee else None,
                                      ws.buf.data_ptr(), ws.bytes, None, _stream_ptr(dev)))
    torch.cuda.synchronize(dev)
    st = ws.stats()
    return {"stats": {k: int(st[k]) for k in CERTIFY_STATS_DTYPE.names}, "pt": out_pt, "ee": out_ee}
