"""Conservative refinement children on the device.

``refinement_children`` runs GenerateConservativeRefinementWorkItems
(cpp/certificate/certificate_engine.cpp:663-720) for a whole queue of
certified work items in one call (``p2c_refinement_children``): children come
back compacted in parent order with the ids the reference assigns when it is
called once per parent in order with the next free id.
"""
from __future__ import annotations

import torch

from . import _lib
from .certify import _stream_ptr


def refinement_children(t0: torch.Tensor, t1: torch.Tensor, depth: torch.Tensor, certs: torch.Tensor, *,
                        max_child_depth: int = 64, min_interval_width: float = 1e-4,
                        first_child_work_item_id: int = 1, sync: bool = True) -> dict:
    """Parents: float64 ``t0``/``t1``, uint16-valued ``depth`` (int32 tensor
    accepted), ``certs`` a (n, 56) uint8 tensor of query certificates, all on
    one CUDA device.  Returns device tensors ``parent``, ``t0``, ``t1``,
    ``depth``, ``work_item_id`` (capacity 2 n) plus ``count`` and, with
    ``sync``, the host ints ``n_children`` and ``error_word``."""
    lib = _lib.load()
    d = t0.device
    n = t0.numel()
    if certs.dtype != torch.uint8 or certs.dim() != 2 or certs.shape[1] != 56 or certs.shape[0] != n:
        raise ValueError("certs must be a (n, 56) uint8 tensor of query certificates")
    t0 = t0.contiguous().to(torch.float64)
    t1 = t1.contiguous().to(torch.float64)
    dep = depth.contiguous().to(torch.int32).to(torch.int16)  # 16-bit depths (values < 2^15 here)
    cap = max(1, 2 * n)
    out = {"parent": torch.empty(cap, dtype=torch.int64, device=d),
           "t0": torch.empty(cap, dtype=torch.float64, device=d),
           "t1": torch.empty(cap, dtype=torch.float64, device=d),
           "depth": torch.empty(cap, dtype=torch.int16, device=d),
           "work_item_id": torch.empty(cap, dtype=torch.int64, device=d),
           "count": torch.zeros(1, dtype=torch.int64, device=d)}
    err = torch.zeros(1, dtype=torch.int64, device=d)
    ws = torch.empty(max(1, int(lib.p2c_refinement_children_workspace_bytes(n))), dtype=torch.uint8, device=d)
    _lib.check(lib.p2c_refinement_children(
        n, t0.data_ptr(), t1.data_ptr(), dep.data_ptr(), certs.contiguous().data_ptr(), int(max_child_depth),
        float(min_interval_width), int(first_child_work_item_id), out["parent"].data_ptr(), out["t0"].data_ptr(),
        out["t1"].data_ptr(), out["depth"].data_ptr(), out["work_item_id"].data_ptr(), out["count"].data_ptr(),
        err.data_ptr(), ws.data_ptr(), ws.numel(), _stream_ptr(d)))
    if sync:
        out["n_children"] = int(out["count"].item())
        out["error_word"] = int(err.item())
    out["_keep"] = (t0, t1, dep, ws, err)
    return out
