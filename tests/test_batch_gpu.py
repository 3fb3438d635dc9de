"""GPU parity of batched scenes (p2c_batch_certify): every scene of an
uneven batch certified in one launch gets exactly the candidates, the
certificates and the Evaluate summary that the single-scene path gives, and
every certificate equals the oracle's byte for byte."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import anyhit_case as A

pytestmark = pytest.mark.gpu


def _small_batch(n=9, seed=7):
    from p2cccd_b200 import scenes

    return scenes.uneven_batch(n, tri_min=200, tri_max=6000, seed=seed)


def _cands(pairs):
    return np.stack([(pairs >> np.uint64(32)).astype(np.int64), (pairs & np.uint64(0xffffffff)).astype(np.int64)], 1)


def _bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1, 72)


@pytest.mark.parametrize("depth", [32, 4])
def test_batch_matches_single_scene_and_oracle(cuda_device, oracle_mod, depth):
    from p2cccd_b200.batch import BatchPipeline
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    cfg = CertConfig(1e-6, 1e-6, depth)
    batch = _small_batch()
    bp = BatchPipeline(batch, cuda_device, config=cfg, streams=3)
    summ = bp.step_checked()
    bp.capture()
    bp.replay()
    bp.replay()
    torch.cuda.synchronize(cuda_device)
    summ_graph = bp.read_summaries()
    assert summ_graph == summ
    total_undecided = 0
    for i, s in enumerate(batch):
        sp = ScenePipeline(s, cuda_device, config=cfg)
        single = sp.step_checked()
        assert summ[i] == single, i
        vf, ee = bp.pairs(i)
        svf, see = sp.pairs()
        assert np.array_equal(vf, svf) and np.array_equal(ee, see)
        rvf, ree = bp.results(i)
        srvf, sree = sp.results()
        assert np.array_equal(_bytes(rvf), _bytes(srvf)) and np.array_equal(_bytes(ree), _bytes(sree))
        for kind, pairs, res in (("vf", vf, rvf), ("ee", ee, ree)):
            if len(pairs) == 0:
                continue
            rec = A.primitives(s, s["edges"], _cands(pairs), kind)
            cpu, st, _ = oracle_mod.eval_batch(rec, 0.0, 1.0, cfg.eps_time, cfg.eps_space, depth)
            assert st.sum() == 0
            assert np.array_equal(_bytes(cpu), _bytes(res)), (i, kind)
        total_undecided += summ[i]["undecided"]
    # undecided queue: (scene << 40 | family << 39 | position), one entry per
    # undecided certificate of every scene, none twice (one queue shared by all scenes)
    assert sum(x["undecided_queued"] for x in summ) == total_undecided
    got = {tuple(int(v) for v in row) for row in bp.undecided_entries()}
    assert len(got) == total_undecided
    assert got == _undecided_set(bp)
    if depth == 4:
        assert sum(1 for x in summ if x["undecided"] > 0) >= 2  # several scenes share the queue


def _undecided_set(bp):
    out = set()
    for i in range(bp.n):
        for fam, res in ((1, bp.results(i)[0]), (2, bp.results(i)[1])):
            out |= {(i, fam, int(p)) for p in np.nonzero(res["status"] == 2)[0]}
    return out


def test_batch_undecided_queue_overflow_reruns(cuda_device):
    """A shared undecided queue smaller than the step's undecided
    certificates: the device marks the scenes whose entries were dropped
    (error bit 8), reading the queue raises, and step_checked re-runs with a
    larger queue so that the replay list is complete."""
    from p2cccd_b200.batch import BatchPipeline
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ERR_UNDECIDED_FULL, UndecidedOverflow

    cfg = CertConfig(1e-2, 1e-6, 4)  # coarse: many undecided certificates
    bp = BatchPipeline(_small_batch(), cuda_device, config=cfg, undecided_capacity=8)
    bp.step()
    summ = bp.read_summaries()
    queued = sum(x["undecided_queued"] for x in summ)
    assert queued > 8
    assert any(x["error_word"] & ERR_UNDECIDED_FULL for x in summ)
    with pytest.raises(UndecidedOverflow):
        bp.undecided_entries()
    summ = bp.step_checked()
    assert bp.undecided_capacity >= queued
    assert not any(x["error_word"] & ERR_UNDECIDED_FULL for x in summ)
    got = {tuple(int(v) for v in row) for row in bp.undecided_entries()}
    assert got == _undecided_set(bp) and len(got) == queued


def test_batch_autotune_keeps_results(cuda_device, tmp_path):
    from p2cccd_b200.batch import BatchPipeline
    from p2cccd_b200.certify import CertConfig

    cfg = CertConfig(1e-6, 1e-6, 32)
    bp = BatchPipeline(_small_batch(12, seed=3), cuda_device, config=cfg)
    summ = bp.step_checked()
    before = [tuple(map(_bytes, bp.results(i))) for i in range(bp.n)]
    bp.fit_capacities(margin=1.0, slack=0)  # exact-size buffers: same candidates and certificates
    assert bp.step_checked() == summ
    assert all(cap == int(n) for cap, n in zip(bp.vf_caps, bp.read_counts()[:, 0]) if n > 0)
    best = bp.autotune(reps=2, cache=tmp_path / "tune.json")
    assert best["ms"] > 0 and best["streams"] in (1, 4, 8, 16)
    cached = bp.autotune(reps=2, cache=tmp_path / "tune.json")
    assert cached.get("cached") is True
    bp.replay()
    torch.cuda.synchronize(cuda_device)
    assert bp.read_summaries() == summ
    for i in range(bp.n):
        after = tuple(map(_bytes, bp.results(i)))
        assert all(np.array_equal(a, b) for a, b in zip(before[i], after))


def test_batch_rejects_bad_arguments(cuda_device):
    from p2cccd_b200.batch import BatchPipeline, BatchTuning

    bp = BatchPipeline(_small_batch(2, seed=1), cuda_device)
    bp.tuning = BatchTuning(0, 33, 0, 0)
    with pytest.raises(ValueError):
        bp.certify()
    with pytest.raises(ValueError):
        BatchPipeline([], cuda_device)


@pytest.mark.parametrize("exclude_self,thickness", [(True, 0.0), (False, 0.0), (False, 2e-3)])
def test_batched_candidates_equal_per_scene(cuda_device, oracle_mod, exclude_self, thickness):
    """p2c_batch_candidates writes every scene's pair buffer (pairs sorted,
    ~0 padding) and counts exactly as p2c_scene_candidates does per scene,
    with self pairs, thickness, far-apart scenes with no candidates and
    scenes of many objects."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.batch import BatchPipeline
    from p2cccd_b200.certify import CertConfig

    batch = _small_batch(7, seed=21)
    batch += [A.sphere_cluster(6, 3), A.cloth_small()]
    far = scenes.two_spheres(n_lon=12, n_rings=8, gap=5.0, approach=0.1)  # no candidates at all
    batch.append(far)
    cfg = CertConfig(1e-6, 1e-6, 32)
    a = BatchPipeline(batch, cuda_device, config=cfg, exclude_self=exclude_self, thickness=thickness)
    b = BatchPipeline(batch, cuda_device, config=cfg, exclude_self=exclude_self, thickness=thickness,
                      broad="per_scene")
    sa, sb = a.step_checked(), b.step_checked()
    ca, cb = a.read_counts(), b.read_counts()
    assert np.array_equal(ca[:, :3], cb[:, :3])
    if exclude_self:  # the far-apart pair of spheres has no candidate between them
        assert ca[-1, 0] == 0 and ca[-1, 1] == 0
    for i in range(len(batch)):
        pa, pb = a.pairs(i), b.pairs(i)
        assert np.array_equal(pa[0], pb[0]) and np.array_equal(pa[1], pb[1]), i
        # padding after the pairs
        off, cap = int(a.vf_pair_off[i]), a.vf_caps[i]
        tail = a.vf_pairs[off + int(ca[i, 0]):off + cap].cpu().numpy().view(np.uint64)
        assert (tail == np.uint64(0xFFFFFFFFFFFFFFFF)).all()
    assert sa == sb
    # the oracle's pair sets for two of the scenes
    for i in (0, len(batch) - 3):
        s = batch[i]
        n_obj = int(s["n_obj"])
        allowed = oracle_mod.object_allowed(s["v_t0"], s["v_t1"], s["v_obj"], n_obj, thickness, exclude_self)
        vbox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], None, 1, thickness)
        fbox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], s["faces"], 3, thickness)
        ebox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], s["edges"], 2, thickness)
        valid = (s["v_obj"] >= 0).astype(np.uint8)
        vf = oracle_mod.vf_pairs(vbox, s["v_obj"], valid, fbox, s["f_obj"], s["faces"], allowed, "sweep")
        ee = oracle_mod.ee_pairs(ebox, s["e_obj"], s["edges"], allowed, "sweep")
        pa = a.pairs(i)
        assert np.array_equal(np.sort(vf), pa[0]) and np.array_equal(np.sort(ee), pa[1]), i
