"""p2c_certify_queries_static: the work-queue certifier for callers that
cannot allocate device memory (graph capture, frame loops that forbid
allocation, hosts that own all device memory under a budget).  Its scratch is
a fixed 1 MiB device array inside the library; this file checks, through the
C ABI, that two calls in a row give exactly what the workspace-taking entry
point gives on the same inputs, and that an oversized queue is refused.

The file is named to be collected last so that a run stopping at the first
failure has already run every other test; it also passes on its own.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P2C_STATIC_QUEUE_MAX_QUERIES = 26000  # include/p2c_b200.h


def _queue(seed: int, nq: int):
    from p2cccd_b200 import workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=600, n_ee=600, seed=seed))
    rng = np.random.default_rng(seed)
    masks = rng.integers(1, 4, nq).astype(np.uint32)
    n_pt = rng.integers(0, 6, nq) * (masks & 1)
    n_ee = rng.integers(0, 6, nq) * ((masks >> 1) & 1)
    t0 = rng.uniform(0.0, 0.4, nq)
    t1 = np.minimum(1.0, t0 + rng.uniform(0.0, 0.7, nq))
    pt = w["vf"][rng.integers(0, 600, int(n_pt.sum()))]
    ee = w["ee"][rng.integers(0, 600, int(n_ee.sum()))]
    pto = np.concatenate([[0], np.cumsum(n_pt)]).astype(np.int64)
    eeo = np.concatenate([[0], np.cumsum(n_ee)]).astype(np.int64)
    return pt, pto, ee, eeo, t0, t1, masks


def _to_dev(a, device):
    import torch

    a = np.ascontiguousarray(a)
    if a.size == 0:
        return torch.zeros(8, dtype=torch.uint8, device=device)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(device)


def _run(device, queue, static: bool):
    """One call through the C ABI; returns the raw output bytes."""
    import torch

    from p2cccd_b200 import _lib

    lib = _lib.load()
    pt, pto, ee, eeo, t0, t1, masks = queue
    nq = len(t0)
    n_pt, n_ee = int(pto[-1]), int(eeo[-1])
    ptq = np.repeat(np.arange(nq, dtype=np.int64), np.diff(pto))
    eeq = np.repeat(np.arange(nq, dtype=np.int64), np.diff(eeo))
    d = {k: _to_dev(v, device) for k, v in dict(pt=pt, ee=ee, ptq=ptq, eeq=eeq, pto=pto, eeo=eeo, t0=t0, t1=t1,
                                                   m=masks).items()}
    out_pt = torch.full((max(n_pt, 1), 72), 0xAB, dtype=torch.uint8, device=device)
    out_ee = torch.full((max(n_ee, 1), 72), 0xAB, dtype=torch.uint8, device=device)
    certs = torch.full((nq, 56), 0xAB, dtype=torch.uint8, device=device)
    cfg = _lib.make_config(1e-5, 1e-6, 32)
    stream = torch.cuda.current_stream(device).cuda_stream
    args = [d["pt"].data_ptr(), n_pt, d["ptq"].data_ptr(), d["ee"].data_ptr(), n_ee, d["eeq"].data_ptr(), nq,
            d["pto"].data_ptr(), d["eeo"].data_ptr(), d["t0"].data_ptr(), d["t1"].data_ptr(), d["m"].data_ptr(),
            ctypes.byref(cfg), out_pt.data_ptr(), out_ee.data_ptr(), certs.data_ptr()]
    if static:
        rc = lib.p2c_certify_queries_static(*args, None, stream)
    else:
        ws_bytes = int(lib.p2c_certify_queries_workspace_bytes(nq))
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
        rc = lib.p2c_certify_queries(*args, ws.data_ptr(), ws_bytes, None, stream)
    _lib.check(rc)
    torch.cuda.synchronize(device)
    return certs.cpu().numpy(), out_pt[:n_pt].cpu().numpy(), out_ee[:n_ee].cpu().numpy()


def test_static_scratch_matches_workspace_entry_point_twice(cuda_device):
    first = _queue(31, 400)
    second = _queue(47, 250)  # a different, smaller queue right after
    for queue in (first, second):
        want = _run(cuda_device, queue, static=False)
        got = _run(cuda_device, queue, static=True)
        for a, b in zip(want, got):
            np.testing.assert_array_equal(a, b)  # bit-identical, like every certificate test here
        assert (want[0][:, 0] <= 2).all()  # every work item got a certificate


def test_static_scratch_at_its_stated_maximum(cuda_device):
    """Exactly P2C_STATIC_QUEUE_MAX_QUERIES work items fit the array."""
    queue = _queue(53, P2C_STATIC_QUEUE_MAX_QUERIES)
    want = _run(cuda_device, queue, static=False)
    got = _run(cuda_device, queue, static=True)
    for a, b in zip(want, got):
        np.testing.assert_array_equal(a, b)


def test_static_scratch_refuses_oversized_queue(cuda_device):
    import torch

    from p2cccd_b200 import _lib

    lib = _lib.load()
    dummy = torch.zeros(64, dtype=torch.uint8, device=cuda_device)
    p = dummy.data_ptr()
    cfg = _lib.make_config(1e-5, 1e-6, 32)
    rc = lib.p2c_certify_queries_static(p, 0, p, p, 0, p, P2C_STATIC_QUEUE_MAX_QUERIES + 1, p, p, p, p, p,
                                        ctypes.byref(cfg), p, p, p, None, None)
    assert rc == _lib.P2C_ERR_INVALID
    assert "at most 26000 work items" in _lib.last_error()
