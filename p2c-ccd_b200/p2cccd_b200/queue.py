"""Work queues on the GPU: many work items certified in one launch
(``p2c_certify_queries``), the device form of ProcessExactWorkQueueCpu /
CertificateEngine::Evaluate (cpp/certificate/certificate_engine.cpp:593-824).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .certify import CertConfig, _stream_ptr
from .records import EDGE_EDGE_DTYPE, INTERVAL_RESULT_DTYPE, POINT_TRIANGLE_DTYPE, QUERY_CERTIFICATE_DTYPE


def certify_work_items(pt_records: np.ndarray, pt_offsets: np.ndarray, ee_records: np.ndarray,
                       ee_offsets: np.ndarray, q_t0: np.ndarray, q_t1: np.ndarray, q_mask: np.ndarray,
                       config: CertConfig, device: str | torch.device = "cuda") -> dict:
    """Certify a queue given as flat record lists with CSR offsets per work item.

    Returns per work item a QUERY_CERTIFICATE_DTYPE record and per primitive
    the INTERVAL_RESULT_DTYPE results.  Synchronous (reads results back)."""
    lib = _lib.load()
    dev = torch.device(device)
    nq = len(q_t0)
    pt_offsets = np.ascontiguousarray(pt_offsets, dtype=np.int64)
    ee_offsets = np.ascontiguousarray(ee_offsets, dtype=np.int64)
    n_pt, n_ee = int(pt_offsets[-1]) if nq else 0, int(ee_offsets[-1]) if nq else 0
    pt_query = np.repeat(np.arange(nq, dtype=np.int64), np.diff(pt_offsets)) if nq else np.zeros(0, np.int64)
    ee_query = np.repeat(np.arange(nq, dtype=np.int64), np.diff(ee_offsets)) if nq else np.zeros(0, np.int64)

    def to_dev(a, dtype=None):
        a = np.ascontiguousarray(a if dtype is None else a.astype(dtype))
        if a.size == 0:
            return torch.empty(1, dtype=torch.uint8, device=dev)
        return torch.from_numpy(a.view(np.uint8).reshape(-1)).to(dev)

    pt = to_dev(pt_records.view(np.uint8) if len(pt_records) else np.zeros(0, np.uint8))
    ee = to_dev(ee_records.view(np.uint8) if len(ee_records) else np.zeros(0, np.uint8))
    d_ptq, d_eeq = to_dev(pt_query), to_dev(ee_query)
    d_pto, d_eeo = to_dev(pt_offsets), to_dev(ee_offsets)
    d_t0, d_t1 = to_dev(np.asarray(q_t0, np.float64)), to_dev(np.asarray(q_t1, np.float64))
    d_mask = to_dev(np.asarray(q_mask, np.uint32))
    out_pt = torch.empty((max(n_pt, 1), 72), dtype=torch.uint8, device=dev)
    out_ee = torch.empty((max(n_ee, 1), 72), dtype=torch.uint8, device=dev)
    certs = torch.empty((max(nq, 1), QUERY_CERTIFICATE_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    ws_bytes = int(lib.p2c_certify_queries_workspace_bytes(nq))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    cfg = config.c()
    _lib.check(lib.p2c_certify_queries(pt.data_ptr(), n_pt, d_ptq.data_ptr(), ee.data_ptr(), n_ee,
                                       d_eeq.data_ptr(), nq, d_pto.data_ptr(), d_eeo.data_ptr(), d_t0.data_ptr(),
                                       d_t1.data_ptr(), d_mask.data_ptr(), ctypes.byref(cfg), out_pt.data_ptr(),
                                       out_ee.data_ptr(), certs.data_ptr(), ws.data_ptr(), ws_bytes, None,
                                       _stream_ptr(dev)))
    torch.cuda.synchronize(dev)
    stats = ws[:48].cpu().numpy().view(np.uint64)
    if stats[5] != 0:
        raise _lib.P2CError("certification exceeded the device time budget (P2C_DEVICE_BUDGET_MS)")
    return {
        "certs": certs[:nq].cpu().numpy().view(QUERY_CERTIFICATE_DTYPE).reshape(-1),
        "pt_results": out_pt[:n_pt].cpu().numpy().view(INTERVAL_RESULT_DTYPE).reshape(-1),
        "ee_results": out_ee[:n_ee].cpu().numpy().view(INTERVAL_RESULT_DTYPE).reshape(-1),
    }


def empty_records(family: int) -> np.ndarray:
    return np.zeros(0, dtype=POINT_TRIANGLE_DTYPE if family == 1 else EDGE_EDGE_DTYPE)



def audit_rows(items, certs, first_event_id: int = 1, first_timestamp_us: int = 1, emit_dequeue: bool = True,
               device: str | torch.device = "cuda") -> np.ndarray:
    """The audit log of a certified queue, written on the device
    (p2c_audit_rows).  ``items``: AUDIT_ITEM_DTYPE records; ``certs``:
    QUERY_CERTIFICATE_DTYPE records or their (n, 64) uint8 device tensor.
    Returns AUDIT_ROW_DTYPE records; ValueError (with the first failing row
    index) when a row fails the reference's audit row validation."""
    from .records import AUDIT_ROW_DTYPE

    lib = _lib.load()
    dev = torch.device(device)
    items = np.ascontiguousarray(items)
    n = len(items)
    d_items = torch.from_numpy(items.view(np.uint8).reshape(-1).copy()).to(dev) if n else None
    if torch.is_tensor(certs):
        d_certs = certs.to(dev).contiguous()
    else:
        c = np.ascontiguousarray(certs)
        d_certs = torch.from_numpy(c.view(np.uint8).reshape(-1).copy()).to(dev) if n else None
    per = 2 if emit_dequeue else 1
    rows = torch.empty((max(per * n, 1), AUDIT_ROW_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    err = torch.zeros(2, dtype=torch.int64, device=dev)
    _lib.check(lib.p2c_audit_rows(d_items.data_ptr() if n else None, d_certs.data_ptr() if n else None, n,
                                  int(first_event_id), int(first_timestamp_us), 1 if emit_dequeue else 0,
                                  rows.data_ptr(), err.data_ptr(), _stream_ptr(dev)))
    e = err.cpu().numpy().view(np.uint64)
    out = rows[:per * n].cpu().numpy().view(AUDIT_ROW_DTYPE).reshape(-1)
    if e[0] & 1:
        raise AuditRowError(int(e[1]), out)
    return out


class AuditRowError(ValueError):
    """A row fails the reference's ValidateAuditLogRow; ``row`` is the first."""

    def __init__(self, row: int, rows: np.ndarray):
        super().__init__(f"audit row {row} fails validation")
        self.row, self.rows = row, rows
