"""GPU parity of the candidate-group any-hit with fallback replay
(p2c_group_anyhit) against the reference scene tool's RunScheduledAnyHitRows
counts and the C restatement's per-group and per-candidate outcome."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import anyhit_case as A

pytestmark = pytest.mark.gpu


def _scene_with_tool_topology(s, tool):
    d = dict(s)
    d.update(edges=tool.edges, e_obj=tool.e_obj, v_obj=tool.v_obj, f_obj=tool.f_obj, n_obj=tool.n_obj)
    return d


def _run_device(pipe, kind, cands, scores, top_k, dev, capacity=None):
    from p2cccd_b200.anyhit import GroupAnyHit
    from p2cccd_b200.certify import CertConfig

    n = len(cands)
    cap = max(1, capacity or n)
    keys = np.zeros(cap, dtype=np.int64)
    keys[:n] = ((cands[:, 0].astype(np.int64) << 32) | cands[:, 1].astype(np.int64))
    sc = np.zeros(cap, dtype=np.float64)
    sc[:n] = scores
    ah = GroupAnyHit(pipe._struct, pipe.n_obj, kind, cap, dev)
    cfg = CertConfig(A.CFG["eps_time"], A.CFG["eps_space"], A.CFG["max_depth"])
    ah.run(torch.from_numpy(keys).to(dev), torch.tensor([n], dtype=torch.int64, device=dev),
           torch.from_numpy(sc).to(dev), top_k, cfg)
    torch.cuda.synchronize(dev)
    return ah


def _check(ah, exp, n, row=None):
    summ = ah.read_summary()
    assert summ["error_word"] == 0, summ
    assert summ["candidates"] == n
    det, pc, fc = ah.read_groups()
    assert np.array_equal(det, exp["detected"])
    assert np.array_equal(pc, exp["proposal_calls"])
    assert np.array_equal(fc, exp["fallback_calls"])
    ev, hit = ah.read_candidates(n)
    assert np.array_equal(ev > 0, exp["evaluated"] > 0)
    r = exp["row"]
    assert summ["proposal_calls"] == r["proposal_exact_calls"]
    assert summ["fallback_calls"] == r["fallback_exact_calls"]
    assert summ["detected_groups"] == r["hit_count"] == int(hit.sum())
    assert summ["groups"] == r["group_count"]
    assert summ["fallback_groups"] == r["fallback_groups"]
    assert summ["first_hit_rank_sum"] == r["positive_first_hit_rank_sum"]
    if row is not None:
        for k in ("exact_calls", "proposal_exact_calls", "fallback_exact_calls", "hit_count", "group_count",
                  "fallback_groups", "positive_first_hit_rank_sum"):
            assert r[k] == row[k], k
    return summ


SCENES = {
    "two_spheres": A.two_spheres_small,
    "cloth": A.cloth_small,
    "cluster5": lambda: A.sphere_cluster(7, 5),
    "cluster6": lambda: A.sphere_cluster(7, 6),
}


@pytest.mark.parametrize("scene", list(SCENES))
@pytest.mark.parametrize("kind", ["vf", "ee"])
@pytest.mark.parametrize("exclude_self", [False, True])
def test_device_anyhit_matches_reference_tool(cuda_device, oracle_mod, scene, kind, exclude_self):
    from p2cccd_b200.scene import ScenePipeline

    if not oracle_mod.REF_TOOL_SO.exists():
        pytest.skip("reference scene tool library not built")
    s = SCENES[scene]()
    tool, cands, scores, groups, hit = A.tool_case(oracle_mod, s, kind, 0.0, exclude_self)
    pipe = ScenePipeline(_scene_with_tool_topology(s, tool), cuda_device, exclude_self=exclude_self)
    for top_k in (0, 1, 5, 4096):
        exp = A.expected(oracle_mod, groups, hit, scores, tool.n_obj ** 2, top_k)
        row = tool.anyhit(kind, top_k, A.CFG["eps_time"], A.CFG["eps_space"], A.CFG["max_depth"])
        ah = _run_device(pipe, kind, cands, scores, top_k, cuda_device, capacity=len(cands) + 37)
        _check(ah, exp, len(cands), row)


def test_device_anyhit_after_device_broad_phase(cuda_device, oracle_mod):
    """Candidates straight from p2c_scene_candidates (sorted pairs), seeded
    scheduler scores, self pairs with adjacency exclusion, graph replay."""
    from p2cccd_b200.anyhit import GroupAnyHit
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    s = A.sphere_cluster(9, 11)
    pipe = ScenePipeline(s, cuda_device, exclude_self=False, config=CertConfig(**{
        "eps_time": A.CFG["eps_time"], "eps_space": A.CFG["eps_space"],
        "max_subdivision_depth": A.CFG["max_depth"]}))
    pipe.step_checked()
    vf, ee = pipe.pairs()
    cfg = CertConfig(A.CFG["eps_time"], A.CFG["eps_space"], A.CFG["max_depth"])
    gen = torch.Generator(device=cuda_device).manual_seed(1234)
    for kind, pairs_np, pairs_t, cap in (("vf", vf, pipe.vf_pairs, pipe.vf_cap), ("ee", ee, pipe.ee_pairs,
                                                                                    pipe.ee_cap)):
        n = len(pairs_np)
        scores = torch.rand(cap, dtype=torch.float64, device=cuda_device, generator=gen)
        count = pipe.counts[0:1] if kind == "vf" else pipe.counts[1:2]
        ah = GroupAnyHit(pipe._struct, pipe.n_obj, kind, cap, cuda_device)
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(cuda_device)
        side.wait_stream(torch.cuda.current_stream(cuda_device))
        with torch.cuda.stream(side):
            ah.run(pairs_t, count, scores, 3, cfg)
        torch.cuda.current_stream(cuda_device).wait_stream(side)
        with torch.cuda.graph(g):
            ah.run(pairs_t, count, scores, 3, cfg)
        for _ in range(2):
            g.replay()
        torch.cuda.synchronize(cuda_device)
        cands = np.stack([(pairs_np >> np.uint64(32)).astype(np.int64),
                          (pairs_np & np.uint64(0xffffffff)).astype(np.int64)], 1)
        if kind == "vf":
            oa, ob = s["v_obj"][cands[:, 0]], s["f_obj"][cands[:, 1]]
        else:
            oa, ob = s["e_obj"][cands[:, 0]], s["e_obj"][cands[:, 1]]
        groups = (np.minimum(oa, ob) * pipe.n_obj + np.maximum(oa, ob)).astype(np.int32)
        hit = A.hits(oracle_mod, s, s["edges"], cands, kind)
        exp = A.expected(oracle_mod, groups, hit, scores[:n].cpu().numpy(), pipe.n_obj ** 2, 3)
        summ = _check(ah, exp, n)
        assert summ["detected_groups"] > 1


@pytest.mark.parametrize("mode", ["ties", "signed_zero", "nan"])
def test_device_anyhit_score_edge_cases(cuda_device, oracle_mod, mode):
    """Equal scores rank the lower index first; -0 ties with +0; NaN ranks
    last and sets error bit 16."""
    from p2cccd_b200.scene import ScenePipeline

    if not oracle_mod.REF_TOOL_SO.exists():
        pytest.skip("reference scene tool library not built")
    s = A.sphere_cluster(7, 6)
    tool, cands, _, groups, hit = A.tool_case(oracle_mod, s, "vf", 0.0, False)
    n = len(cands)
    rng = np.random.default_rng(3)
    if mode == "ties":
        scores = rng.integers(0, 3, n).astype(np.float64)
    elif mode == "signed_zero":
        scores = np.where(rng.random(n) < 0.5, -0.0, 0.0)
    else:
        scores = rng.random(n)
        scores[rng.random(n) < 0.2] = np.nan
    pipe = ScenePipeline(_scene_with_tool_topology(s, tool), cuda_device, exclude_self=False)
    exp = A.expected(oracle_mod, groups, hit, np.where(np.isnan(scores), -np.inf, scores) if mode == "nan"
                     else np.abs(scores) if mode == "signed_zero" else scores, tool.n_obj ** 2, 4)
    ah = _run_device(pipe, "vf", cands, scores, 4, cuda_device)
    if mode == "nan":
        summ = ah.read_summary()
        assert summ["error_word"] == 16
        ah.summary.zero_()  # the outcome itself is still checked below
        det, pc, fc = ah.read_groups()
        assert np.array_equal(det, exp["detected"]) and np.array_equal(pc, exp["proposal_calls"])
        assert np.array_equal(fc, exp["fallback_calls"])
        ev, _ = ah.read_candidates(n)
        assert np.array_equal(ev > 0, exp["evaluated"] > 0)
    else:
        _check(ah, exp, n)


def test_device_anyhit_rejects_bad_arguments(cuda_device):
    from p2cccd_b200.anyhit import GroupAnyHit
    from p2cccd_b200.scene import ScenePipeline

    s = A.sphere_cluster(3, 2)
    pipe = ScenePipeline(s, cuda_device, exclude_self=False)
    ah = GroupAnyHit(pipe._struct, pipe.n_obj, "vf", 16, cuda_device)
    pairs = torch.zeros(16, dtype=torch.int64, device=cuda_device)
    count = torch.zeros(1, dtype=torch.int64, device=cuda_device)
    scores = torch.zeros(16, dtype=torch.float64, device=cuda_device)
    with pytest.raises(ValueError):
        ah.run(pairs, count, scores, -1)
    ah.run(pairs, count, scores, 4)  # zero candidates: empty outcome
    torch.cuda.synchronize(cuda_device)
    summ = ah.read_summary()
    assert summ["candidates"] == 0 and summ["groups"] == 0 and summ["error_word"] == 0
