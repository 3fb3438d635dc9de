"""GPU parity of the batched any-hit (p2c_batch_anyhit): every (scene,
family) of an uneven batch gets exactly the summary, group decisions and
per-candidate calls/hits that the single-scene any-hit (p2c_group_anyhit,
pinned to the reference scene tool's RunScheduledAnyHitRows in
test_anyhit_gpu.py) gives that scene alone with the same scores.  Scores come
from the seeded scheduler stub, a function of the candidate's identity."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import anyhit_case as A

pytestmark = pytest.mark.gpu


def _batch():
    from p2cccd_b200 import scenes

    out = scenes.uneven_batch(5, tri_min=300, tri_max=5000, seed=17)
    out += [A.sphere_cluster(7, 5), A.cloth_small(), A.two_spheres_small()]
    out.append(scenes.two_spheres(n_lon=12, n_rings=8, gap=5.0, approach=0.1))  # no candidates at all
    return out


def _exact(summary):
    """A summary without its speculation count: how many certificates were
    started before an earlier hit of their group landed depends on the
    device's timing, not on the procedure."""
    return None if summary is None else {k: v for k, v in summary.items() if k != "speculative"}


def test_stub_scores_equal_host_restatement(cuda_device):
    from p2cccd_b200.anyhit import stub_score_host, stub_scores

    rng = np.random.default_rng(1)
    keys = rng.integers(0, 1 << 62, 1000, dtype=np.int64)
    out = torch.empty(1000, dtype=torch.float64, device=cuda_device)
    for fam in (1, 2):
        stub_scores(torch.from_numpy(keys).to(cuda_device), torch.tensor([900], device=cuda_device), fam, 12345, out)
        got = out.cpu().numpy()
        exp = [stub_score_host(12345, fam, int(k)) for k in keys[:900]]
        assert np.array_equal(got[:900], np.array(exp)) and (got[900:] == 0.0).all()
        assert ((got[:900] >= 0.0) & (got[:900] < 1.0)).all()


@pytest.mark.parametrize("exclude_self,top_k", [(False, 3), (False, 0), (True, 1), (False, 4096)])
def test_batch_anyhit_equals_each_scene_alone(cuda_device, exclude_self, top_k):
    from p2cccd_b200.anyhit import BatchAnyHit, GroupAnyHit, stub_scores
    from p2cccd_b200.batch import BatchPipeline
    from p2cccd_b200.certify import CertConfig

    cfg = CertConfig(A.CFG["eps_time"], A.CFG["eps_space"], A.CFG["max_depth"])
    batch = _batch()
    bp = BatchPipeline(batch, cuda_device, config=cfg, exclude_self=exclude_self)
    bp.step_checked()  # sizes the pair buffers; candidates stay in them
    counts = bp.read_counts()
    ah = BatchAnyHit(bp.table_host, bp.table, 3, cuda_device, keep_candidates=True)
    seeds = torch.tensor([1000 + 7 * i for i in range(bp.n)], dtype=torch.int64, device=cuda_device)
    ah.run(top_k, cfg, seeds=seeds)
    torch.cuda.synchronize(cuda_device)
    summ = ah.read_summaries()
    total_calls = 0
    for i in range(bp.n):
        for fam, name, caps, off in ((1, "vf", bp.vf_caps, bp.vf_pair_off), (2, "ee", bp.ee_caps, bp.ee_pair_off)):
            cap = caps[i]
            pairs = (bp.vf_pairs if fam == 1 else bp.ee_pairs)[int(off[i]):int(off[i]) + cap]
            count = torch.tensor([int(counts[i, fam - 1])], dtype=torch.int64, device=cuda_device)
            scores = torch.empty(cap, dtype=torch.float64, device=cuda_device)
            stub_scores(pairs, count, fam, int(seeds[i]), scores)
            one = GroupAnyHit(bp.structs[i], bp.n_obj[i], name, cap, cuda_device)
            one.run(pairs, count, scores, top_k, cfg)
            torch.cuda.synchronize(cuda_device)
            alone = one.read_summary()
            assert _exact(summ[i][name]) == _exact(alone), (i, name, summ[i][name], alone)
            det, _, _ = one.read_groups()
            assert np.array_equal(ah.group_detected_of(i, fam), det), (i, name)
            n = min(int(counts[i, fam - 1]), cap)
            ev_a, hit_a = one.read_candidates(n)
            ev_b, hit_b = ah.candidates_of(i, fam, n)
            assert np.array_equal(ev_a, ev_b) and np.array_equal(hit_a, hit_b), (i, name)
            total_calls += alone["proposal_calls"] + alone["fallback_calls"]
    assert total_calls > 0
    if exclude_self:  # the far-apart spheres have candidates only between their own primitives
        assert summ[-1]["vf"]["candidates"] == 0 and summ[-1]["ee"]["candidates"] == 0


def test_batch_anyhit_caller_scores_and_one_family(cuda_device):
    """Per-(scene, family) score tensors from the caller are consumed
    unchanged: with the stub's own scores passed in, the result equals the
    stub run; with one family only, the other's summaries stay empty."""
    from p2cccd_b200.anyhit import BatchAnyHit, stub_scores
    from p2cccd_b200.batch import BatchPipeline
    from p2cccd_b200.certify import CertConfig

    cfg = CertConfig(A.CFG["eps_time"], A.CFG["eps_space"], A.CFG["max_depth"])
    batch = _batch()[:6]
    bp = BatchPipeline(batch, cuda_device, config=cfg, exclude_self=False)
    bp.step_checked()
    counts = torch.from_numpy(bp.read_counts()).to(cuda_device)
    ref = BatchAnyHit(bp.table_host, bp.table, 3, cuda_device)
    seeds = torch.arange(bp.n, dtype=torch.int64, device=cuda_device) * 31 + 5
    ref.run(2, cfg, seeds=seeds)
    keep, ptrs = [], []
    for i in range(bp.n):
        for fam, caps, off in ((1, bp.vf_caps, bp.vf_pair_off), (2, bp.ee_caps, bp.ee_pair_off)):
            pairs = (bp.vf_pairs if fam == 1 else bp.ee_pairs)[int(off[i]):int(off[i]) + caps[i]]
            sc = torch.empty(caps[i], dtype=torch.float64, device=cuda_device)
            stub_scores(pairs, counts[i, fam - 1:fam], fam, int(seeds[i]), sc)
            keep.append(sc)
            ptrs.append(sc.data_ptr())
    ptr_t = torch.tensor(ptrs, dtype=torch.int64, device=cuda_device)
    got = BatchAnyHit(bp.table_host, bp.table, 3, cuda_device)
    got.run(2, cfg, scores_ptrs=ptr_t)
    torch.cuda.synchronize(cuda_device)
    for a, b in zip(got.read_summaries(), ref.read_summaries()):
        assert _exact(a["vf"]) == _exact(b["vf"]) and _exact(a["ee"]) == _exact(b["ee"])
    vf_only = BatchAnyHit(bp.table_host, bp.table, 1, cuda_device)
    vf_only.run(2, cfg, seeds=seeds)
    torch.cuda.synchronize(cuda_device)
    for a, b in zip(vf_only.read_summaries(), ref.read_summaries()):
        assert _exact(a["vf"]) == _exact(b["vf"]) and a["ee"] is None
