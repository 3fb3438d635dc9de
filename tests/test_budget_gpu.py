"""Failure detection without a GPU fault: the certifier's device time budget.

Every launch of the persistent certifier carries a time budget
(P2C_DEVICE_BUDGET_MS, read once per process).  When it runs out, every warp
leaves its loop at its next check, the launch ends normally, and the host
reports P2C_ERR_TIMEOUT with the budget message; the context stays usable, so
the next call certifies normally.  The case runs in a child process with a
1 ms budget on work that needs far longer (deep grazing trees), so nothing in
the parent's process is affected.  The reference's rule behind it: every
exact work item yields exactly one certificate or the call fails
(certificate_engine.cpp:553-591), never a silent partial answer."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import ctypes, json, sys
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/p2c-ccd_b200"]
import numpy as np
import torch
import oracle
from p2cccd_b200 import _lib, certify, records, workloads

lib = _lib.load()
rng = np.random.default_rng(3)
n = 2048
p0 = np.zeros((n, 4, 3)); p1 = np.zeros((n, 4, 3))
tri = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
p0[:, 1:, :] = tri; p1[:, 1:, :] = tri
h = 1e-6 * (1.0 + rng.uniform(1e-4, 1e-2, size=n))
p0[:, 0, :] = np.stack([rng.uniform(0.05, 0.3, n), rng.uniform(0.05, 0.3, n), h], 1)
p1[:, 0, :] = p0[:, 0, :] + np.stack([rng.uniform(0.1, 0.4, n), rng.uniform(0.1, 0.4, n), np.zeros(n)], 1)
deep = records.pack_primitives(p0, p1, np.arange(n), np.arange(n) + 100)
cfg = certify.CertConfig(1e-5, 1e-6, 32).c()
out = np.zeros(n, dtype=records.INTERVAL_RESULT_DTYPE)
rc = lib.p2c_certify_pt_batch_host(deep.ctypes.data, n, 0.0, 1.0, ctypes.byref(cfg), out.ctypes.data)
msg = lib.p2c_last_error().decode()
# the same device stays usable: a small batch right after certifies normally
w = workloads.plain_queries(workloads.PlainSpec(n_vf=256, n_ee=256, seed=9))
small = np.zeros(256, dtype=records.INTERVAL_RESULT_DTYPE)
cfg2 = certify.CertConfig(1e-6, 1e-6, 32).c()
rc2 = lib.p2c_certify_pt_batch_host(w["vf"].ctypes.data, 256, 0.0, 1.0, ctypes.byref(cfg2), small.ctypes.data)
cpu, st, _ = oracle.eval_batch(w["vf"], 0.0, 1.0, 1e-6, 1e-6, 32)
same = bool((small.view(np.uint8) == cpu.view(np.uint8)).all())
# the device entry point reports the budget in its stats' error word
dev = certify.records_to_device(deep, "cuda:0")
ws = certify.Workspace("cuda:0")
certify.certify_batch(dev, 1, 0.0, 1.0, certify.CertConfig(1e-5, 1e-6, 32), workspace=ws)
torch.cuda.synchronize()
err = int(ws.stats()["error_word"])
print(json.dumps({"rc": rc, "msg": msg, "rc_after": rc2, "after_equals_oracle": same, "device_error_word": err}))
"""


def test_device_time_budget_reports_timeout_and_recovers(cuda_device):
    env = dict(os.environ, P2C_DEVICE_BUDGET_MS="1")
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["rc"] == 4, out  # P2C_ERR_TIMEOUT
    assert "time budget" in out["msg"]
    assert out["rc_after"] == 0 and out["after_equals_oracle"], out
    assert out["device_error_word"] & 1, out
