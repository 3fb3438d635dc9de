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


def _summary_vs_row(summ, row):
    assert summ["proposal_calls"] == row["proposal_exact_calls"]
    assert summ["fallback_calls"] == row["fallback_exact_calls"]
    assert summ["detected_groups"] == row["hit_count"]
    assert summ["groups"] == row["group_count"]
    assert summ["fallback_groups"] == row["fallback_groups"]
    assert summ["first_hit_rank_sum"] == row["positive_first_hit_rank_sum"]


def test_cloth_on_sphere_full_size_anyhit(cuda_device, oracle_mod):
    """Vertex-face: the reference scene tool itself (its candidates, its
    random-policy scores, its RunScheduledAnyHitRows) against the device
    any-hit on the same candidates and scores.  Edge-edge (2.5 M candidates,
    whose tool sweep alone takes minutes on one core): the device's own
    candidates and the scheduler stub's scores, against the restated
    procedure (pinned to the tool on smaller scenes) over the reference
    certifier's decision for every candidate."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.anyhit import GroupAnyHit, stub_scores
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    if not oracle_mod.REF_TOOL_SO.exists():
        pytest.skip("reference scene tool library not built")
    cfg = CertConfig(A.CFG["eps_time"], A.CFG["eps_space"], A.CFG["max_depth"])
    s = scenes.cloth_on_sphere()
    assert len(s["faces"]) == 624_288
    tool = oracle_mod.RefToolScene(s["v_t0"], s["v_t1"], s["faces"], 0.0, False)
    d = dict(s)
    d.update(edges=tool.edges, e_obj=tool.e_obj, v_obj=tool.v_obj, f_obj=tool.f_obj, n_obj=tool.n_obj)
    pipe = ScenePipeline(d, cuda_device, exclude_self=False, config=cfg, vf_capacity=1 << 20, ee_capacity=1 << 22)
    # vertex-face through the tool
    vf = tool.candidates("vf")
    scores = tool.random_scores("vf", len(vf))
    row = tool.anyhit("vf", 4096, A.CFG["eps_time"], A.CFG["eps_space"], A.CFG["max_depth"])
    keys = ((vf[:, 0].astype(np.int64) << 32) | vf[:, 1].astype(np.int64))
    ah = GroupAnyHit(pipe._struct, pipe.n_obj, "vf", len(vf), cuda_device)
    ah.run(torch.from_numpy(keys).to(cuda_device), torch.tensor([len(vf)], device=cuda_device),
           torch.from_numpy(scores).to(cuda_device), 4096, cfg)
    torch.cuda.synchronize(cuda_device)
    summ = ah.read_summary()
    assert summ["candidates"] == len(vf) == row["all_exact_calls"] and summ["error_word"] == 0
    _summary_vs_row(summ, row)
    # edge-edge through the device broad phase, the stub and the restated procedure
    pipe.step_checked()
    n_ee = int(pipe.read_counts()[1])
    pairs = pipe.ee_pairs[:n_ee]
    sc = torch.empty(n_ee, dtype=torch.float64, device=cuda_device)
    stub_scores(pairs, None, 2, 97, sc)
    ah2 = GroupAnyHit(pipe._struct, pipe.n_obj, "ee", n_ee, cuda_device)
    ah2.run(pairs.contiguous(), torch.tensor([n_ee], device=cuda_device), sc, 4096, cfg)
    torch.cuda.synchronize(cuda_device)
    cands = _cands(pairs.cpu().numpy().view(np.uint64))
    rec = A.primitives(d, tool.edges, cands, "ee")
    res, st = oracle_mod.ref_eval_batch(rec, 0.0, 1.0, cfg.eps_time, cfg.eps_space, cfg.max_subdivision_depth,
                                        threads=16)
    hit = ((res["status"] != 1) | (st != 0)).astype(np.uint8)
    groups = A.groups_of(tool, cands, "ee")
    exp = A.expected(oracle_mod, groups, hit, sc.cpu().numpy(), tool.n_obj ** 2, 4096)
    summ2 = ah2.read_summary()
    assert summ2["candidates"] == n_ee > 2_000_000 and summ2["error_word"] == 0
    _summary_vs_row(summ2, exp["row"])
    det, pc, fc = ah2.read_groups()
    assert np.array_equal(det, exp["detected"]) and np.array_equal(pc, exp["proposal_calls"])
    assert np.array_equal(fc, exp["fallback_calls"])
