"""Dummy proposal schedules: RunDummyProposalScheduleFromRuntimeCandidates
(proposal/proposal_policy.cpp:744-858, binding py_module.cpp:1009-1033) and
the external-batch schedule with its raw bypass (py_module.cpp:269-361),
against the reference compiled unchanged, byte for byte."""
from __future__ import annotations

import numpy as np
import pytest

from external_inputs import make_batch
from sched_inputs import make_inputs

CONFIGS = [{}, {"family_score_threshold": 0.6}, {"preserve_candidate_order": True},
           {"ood_abs_feature_threshold": 3.0, "first_work_item_id": 1000},
           {"fallback_interval_t0": 0.25, "fallback_interval_t1": 0.5, "family_score_threshold": -1.0}]


def _inputs(seed=3):
    cand, _, _, _ = make_inputs(seed)
    cand = cand.copy()
    cand["motion_bound"][5, 2] = 2e5  # out of distribution
    cand["rt_hit_count"][9] = 200000
    q = [int(x) for x in np.unique(cand["query_id"])]
    masks = {q[0]: 1}
    return cand, masks


def _need_ref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")


@pytest.mark.parametrize("cfg", CONFIGS)
@pytest.mark.parametrize("materialize", [True, False])
def test_restated_dummy_schedule_matches_reference(oracle_mod, cfg, materialize):
    _need_ref(oracle_mod)
    cand, masks = _inputs()
    n = len(cand)
    for m in (masks, {}, {int(cand["query_id"][0]): 0}, {int(cand["query_id"][0]): 2}):
        a = oracle_mod.ref_dummy_schedule(cand, 500, 700, n, m, materialize, **cfg)
        b = oracle_mod.dummy_schedule(cand, 500, 700, n, m, materialize, **cfg)
        assert [x.tobytes() == y.tobytes() for x, y in zip(a, b)] == [True] * 4


@pytest.mark.parametrize("fault,msg", [("schema", "CandidateRecord.schema_version is unsupported"),
                                       ("hits", "CandidateRecord.rt_hit_count is required"),
                                       ("motion", "CandidateRecord.motion_bound must contain finite non-negative"),
                                       ("type", "CandidateRecord.proxy_type_b must be a concrete proxy type")])
def test_candidate_messages_match_reference(oracle_mod, fault, msg):
    from p2cccd_b200.schedule import candidate_record_error

    _need_ref(oracle_mod)
    cand, masks = _inputs()
    k = 17
    if fault == "schema":
        cand["schema_version"][k] = 2
    elif fault == "hits":
        cand["rt_hit_count"][k] = 0
    elif fault == "motion":
        cand["motion_bound"][k, 1] = -1.0
    else:
        cand["proxy_type_b"][k] = 0
    with pytest.raises(ValueError, match=msg):
        oracle_mod.ref_dummy_schedule(cand, 500, 700, len(cand), masks)
    assert candidate_record_error(cand[k]).startswith(msg)


def test_bypass_restated_over_reference_candidates(oracle_mod):
    """The external-batch schedule takes the raw bypass (each query yields at
    most one candidate and has a single-family mask): one kRaw item per
    candidate in order, the family's mask, priority rt_hit_count."""
    _need_ref(oracle_mod)
    b = make_batch(80, 61, miss=0.2)
    cand, items, stats, rows, outs = oracle_mod.ref_external_dummy(b, True, first_work_item_id=50)
    c2, _, _, _ = oracle_mod.ref_external_batch(b)
    assert cand.tobytes() == c2.tobytes() and len(rows) == 0 and len(outs) == 0
    fam = dict(zip(oracle_mod.ref_external_batch(b)[1].tolist(), b["family"].tolist()))
    assert np.array_equal(items["parent_candidate_id"], cand["candidate_id"])
    assert np.array_equal(items["work_item_id"], np.arange(50, 50 + len(cand), dtype=np.uint64))
    assert np.array_equal(items["feature_family_mask"], [1 if fam[int(q)] == 0 else 2 for q in cand["query_id"]])
    assert np.array_equal(items["priority_score"], cand["rt_hit_count"].astype(np.float32))
    assert np.all(items["source"] == 0)
    assert stats["raw_candidate_count"] == stats["work_item_count"] == len(cand)
    assert stats["proposal_output_count"] == 0 and stats["monotonic_safe"] == 1


def test_bypass_skips_config_check_but_validates_items(oracle_mod):
    _need_ref(oracle_mod)
    b = make_batch(30, 62, miss=0.0)
    with pytest.raises(ValueError, match="interval must satisfy 0 <= interval_t0 <= interval_t1 <= 1"):
        oracle_mod.ref_external_dummy(b, fallback_interval_t0=0.8, fallback_interval_t1=0.2)
    cand, items, _, _, _ = oracle_mod.ref_external_dummy(b, conservative_feature_family_mask=0)
    assert len(items) == len(cand) > 0  # an invalid config mask is not looked at


# ---------------------------------------------------------------- on the GPU

@pytest.mark.gpu
@pytest.mark.parametrize("cfg", CONFIGS)
@pytest.mark.parametrize("materialize", [True, False])
def test_device_dummy_schedule_matches_reference(oracle_mod, cfg, materialize):
    from p2cccd_b200.schedule import dummy_schedule

    cand, masks = _inputs()
    n = len(cand)
    for m in (masks, {}, {int(cand["query_id"][0]): 0}):
        want = (oracle_mod.ref_dummy_schedule if oracle_mod.ref_available() else oracle_mod.dummy_schedule)(
            cand, 500, 700, n, m, materialize, **cfg)
        got = dummy_schedule(cand, 500, 700, n, m, materialize, **cfg)
        assert [x.tobytes() == y.tobytes() for x, y in zip(got, want)] == [True] * 4


@pytest.mark.gpu
def test_device_dummy_schedule_errors(oracle_mod):
    from p2cccd_b200.schedule import dummy_schedule

    cand, masks = _inputs()
    bad = cand.copy()
    bad["rt_hit_count"][40] = 0
    bad["schema_version"][60] = 3
    with pytest.raises(ValueError, match="CandidateRecord.rt_hit_count is required"):
        dummy_schedule(bad, 500, 700, len(bad), masks)
    with pytest.raises(ValueError, match="first_work_item_id must be non-zero"):
        dummy_schedule(cand, 500, 700, len(cand), masks, first_work_item_id=0)
    with pytest.raises(ValueError, match="CandidateDensityStats.proxy_count must be non-zero"):
        dummy_schedule(cand, 0, 700, len(cand), masks)


@pytest.mark.gpu
@pytest.mark.parametrize("seed,n,materialize", [(71, 60, False), (72, 500, True), (73, 1, False)])
def test_device_external_dummy_matches_reference(oracle_mod, seed, n, materialize):
    import p2cccd_cpp as cpp
    from p2cccd_b200.records import EXACT_WORK_ITEM_DTYPE

    b = make_batch(n, seed, miss=0.3)
    cfg = cpp.ProposalSchedulingConfig()
    cfg.first_work_item_id = 77
    res = cpp.generate_external_batch_dummy_proposal_schedule(b, config=cfg, materialize_artifacts=materialize)
    items = np.zeros(len(res.work_queue), dtype=EXACT_WORK_ITEM_DTYPE)
    for r, w in zip(items, res.work_queue):
        for k in ("work_item_id", "parent_candidate_id", "query_id", "slab_id", "patch_a_id", "patch_b_id",
                  "interval_t0", "interval_t1", "feature_family_mask", "topk_feature_ids_offset", "depth",
                  "priority_score"):
            r[k] = getattr(w, k)
        r["source"] = int(w.source)
    if oracle_mod.ref_available():
        cand, want, stats, _, _ = oracle_mod.ref_external_dummy(b, materialize, first_work_item_id=77)
        assert cpp._candidate_array(res.candidate_result.candidates).tobytes() == cand.tobytes()
        assert items.tobytes() == want.tobytes()
        assert res.stats.work_item_count == int(stats["work_item_count"]) == len(cand)
        assert res.stats.monotonic_safe and res.feature_rows == [] and res.proposal_outputs == []
    assert res.proposal_elapsed_ms >= 0.0


@pytest.mark.gpu
def test_device_external_dummy_item_check(oracle_mod):
    import p2cccd_cpp as cpp

    b = make_batch(30, 62, miss=0.0)
    cfg = cpp.ProposalSchedulingConfig()
    cfg.fallback_interval_t0, cfg.fallback_interval_t1 = 0.8, 0.2
    with pytest.raises(ValueError, match="interval must satisfy 0 <= interval_t0 <= interval_t1 <= 1"):
        cpp.generate_external_batch_dummy_proposal_schedule(b, config=cfg)
