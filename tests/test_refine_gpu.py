"""GPU parity of the device refinement children (p2c_refinement_children)
with the oracle's GenerateConservativeRefinementWorkItems restatement (itself
pinned to the reference in test_oracle.py), parent by parent in queue order."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _certs(status, toi, mode):
    from p2cccd_b200.records import QUERY_CERTIFICATE_DTYPE

    c = np.zeros(len(status), dtype=QUERY_CERTIFICATE_DTYPE)
    c["status"] = status
    c["toi_upper"] = toi
    c["next_refinement_mode"] = mode
    return c


@pytest.mark.parametrize("max_depth,min_width", [(64, 1e-4), (3, 1e-6), (8, 0.3)])
def test_refinement_children_match_oracle(cuda_device, oracle_mod, max_depth, min_width):
    from p2cccd_b200.refine import refinement_children

    rng = np.random.default_rng(11)
    n = 3000
    a = rng.uniform(0, 1, n)
    b = rng.uniform(0, 1, n)
    t0, t1 = np.minimum(a, b), np.maximum(a, b)
    t1[:50] = t0[:50]                                # zero-width parents
    t0[50:100] = np.minimum(t0[50:100], 1.0 - min_width)
    t1[50:100] = t0[50:100] + min_width              # about the minimum width (rounding decides)
    depth = rng.integers(0, 10, n).astype(np.int32)
    status = rng.integers(0, 3, n).astype(np.uint8)
    mode = rng.integers(0, 4, n).astype(np.uint8)
    toi = np.where(rng.random(n) < 0.3, rng.uniform(-0.5, 1.5, n), t0 + (t1 - t0) * rng.random(n))
    certs = _certs(status, toi, mode)
    dev = cuda_device
    first = 1000
    out = refinement_children(torch.from_numpy(t0).to(dev), torch.from_numpy(t1).to(dev),
                              torch.from_numpy(depth).to(dev),
                              torch.from_numpy(certs.view(np.uint8).reshape(n, 56).copy()).to(dev),
                              max_child_depth=max_depth, min_interval_width=min_width,
                              first_child_work_item_id=first)
    assert out["error_word"] == 0
    k = out["n_children"]
    got_parent = out["parent"][:k].cpu().numpy()
    got = np.stack([out["t0"][:k].cpu().numpy(), out["t1"][:k].cpu().numpy()], 1)
    exp_parent, exp = [], []
    for i in range(n):
        for c0, c1 in oracle_mod.refinement_children(t0[i], t1[i], int(depth[i]), int(status[i]), int(mode[i]),
                                                     toi[i], max_depth, min_width):
            exp_parent.append(i)
            exp.append((c0, c1))
    assert k == len(exp)
    assert np.array_equal(got_parent, np.array(exp_parent))
    assert np.array_equal(got.view(np.uint64), np.array(exp, dtype=np.float64).reshape(-1, 2).view(np.uint64))
    assert np.array_equal(out["depth"][:k].cpu().numpy(), depth[got_parent] + 1)
    assert np.array_equal(out["work_item_id"][:k].cpu().numpy(), first + np.arange(k))


def test_refinement_children_rejects_and_flags(cuda_device):
    from p2cccd_b200.refine import refinement_children

    dev = cuda_device
    t0 = torch.tensor([0.2, 0.7], dtype=torch.float64, device=dev)
    t1 = torch.tensor([0.6, 0.1], dtype=torch.float64, device=dev)  # second parent inverted
    depth = torch.zeros(2, dtype=torch.int32, device=dev)
    certs = torch.zeros((2, 56), dtype=torch.uint8, device=dev)  # collisions at toi 0
    with pytest.raises(ValueError):
        refinement_children(t0, t1, depth, certs, first_child_work_item_id=0)
    with pytest.raises(ValueError):
        refinement_children(t0, t1, depth, certs, min_interval_width=0.0)
    out = refinement_children(t0, t1, depth, certs)
    assert out["error_word"] == 1 and out["n_children"] == 0  # toi 0 clamps to t0: zero width
