"""CPU pin of the restated proxy-scene candidate generation (raw hits and
compaction) against the reference's GenerateRawCandidatesCpu and
CompactRawCandidates compiled unchanged, byte for byte."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("seed,dups,slabs", [(1, 0.0, 4), (2, 0.5, 3), (3, 0.3, 1), (4, 0.0, 8)])
def test_restated_proxy_candidates_match_reference(oracle_mod, seed, dups, slabs):
    from p2cccd_b200 import scenes

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=5, patches_per_object=30, n_slabs=slabs, seed=seed, duplicates=dups)
    r1, c1 = oracle_mod.ref_proxy_candidates(sc)
    r2, c2 = oracle_mod.proxy_candidates(sc)
    assert len(r1) > 0
    assert np.array_equal(r1.view(np.uint8), r2.view(np.uint8))
    assert np.array_equal(c1.view(np.uint8), c2.view(np.uint8))
    if dups:
        assert c1["rt_hit_count"].max() > 1


def _scene_object(sc):
    """A p2cccd_cpp.ProxyScene holding the primitives of a proxy-scene dict."""
    import p2cccd_cpp as cpp

    scene = cpp.ProxyScene()
    scene.query_id = int(sc["query_id"])
    for i in range(int(sc["n"])):
        p = cpp.ProxyPrimitive()
        p.proxy_id, p.object_id, p.patch_id = i, int(sc["object_id"][i]), int(sc["patch_id"][i])
        p.slab_id, p.proxy_type = int(sc["slab_id"][i]), cpp.ProxyType(int(sc["proxy_type"][i]))
        p.t0, p.t1 = float(sc["t0"][i]), float(sc["t1"][i])
        p.bounds.min, p.bounds.max = [float(x) for x in sc["bounds"][i, :3]], [float(x) for x in sc["bounds"][i, 3:]]
        mb = sc["motion_bound"][i]
        (p.motion_bound.translation_bound, p.motion_bound.rotation_angle, p.motion_bound.radial_motion_bound,
         p.motion_bound.conservative_radius) = (float(x) for x in mb)
        scene.primitives.append(p)
    return scene


def test_host_scene_validation_follows_reference():
    import p2cccd_cpp as cpp
    from p2cccd_b200 import scenes

    sc = scenes.proxy_scene(n_objects=3, patches_per_object=6, n_slabs=3, seed=2)
    obj = _scene_object(sc)
    assert cpp.validate_proxy_scene(obj) and cpp.validate_proxy_scene(sc)
    bad = _scene_object(sc)
    bad.primitives[4].proxy_id = 7
    with pytest.raises(ValueError, match="proxy_id"):
        cpp.validate_proxy_scene(bad)
    # one slab id with two intervals
    s2 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in sc.items()}
    k = int(np.nonzero(s2["slab_id"] == s2["slab_id"][0])[0][1])
    s2["t1"][k] = s2["t1"][k] + 1e-6
    with pytest.raises(ValueError, match="one global time interval"):
        cpp.validate_proxy_scene(s2)
    # overlapping slab intervals: stretch slab 0 into the next one
    s3 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in sc.items()}
    first = s3["t0"] == s3["t0"].min()
    s3["t1"][first] = s3["t1"][first] + 0.1
    with pytest.raises(ValueError, match="must not overlap"):
        cpp.validate_proxy_scene(s3)
    # a time tolerance of 1e-12 keeps touching slabs apart and nearly equal ends together
    s4 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in sc.items()}
    s4["t1"][first] = s4["t1"][first] + 5e-13
    assert cpp.validate_proxy_scene(s4)
    s5 = dict(sc, query_id=0)
    with pytest.raises(ValueError, match="query_id"):
        cpp.validate_proxy_scene(s5)


@pytest.mark.parametrize("seed", [1, 5])
def test_density_pair_count_closed_form(seed):
    import p2cccd_cpp as cpp
    from p2cccd_b200 import scenes
    from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE, RAW_HIT_DTYPE

    sc = scenes.proxy_scene(n_objects=4, patches_per_object=15, n_slabs=3, seed=seed)
    n, obj, slab = int(sc["n"]), sc["object_id"], sc["slab_id"]
    brute = sum(1 for i in range(n) for j in range(i + 1, n) if obj[i] != obj[j] and slab[i] == slab[j])
    d = cpp._density(sc, np.zeros(0, RAW_HIT_DTYPE), np.zeros(0, CANDIDATE_RECORD_DTYPE), cpp.RtCandidateTiming(),
                     "cpu_reference")
    assert d.cross_object_same_slab_pair_count == brute
    assert d.slab_count == 3 and d.object_count == 4 and d.proxy_count == n
    assert d.aabb_overlap_ratio == 0.0 and d.avg_rt_hits_per_candidate == 0.0


def test_host_slab_validation_agrees_with_reference(oracle_mod):
    import p2cccd_cpp as cpp
    from p2cccd_b200 import scenes

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    for stretch in (0.1, 1e-3, 5e-13, 0.0):
        sc = scenes.proxy_scene(n_objects=3, patches_per_object=6, n_slabs=3, seed=2)
        first = sc["t0"] == sc["t0"].min()
        sc["t1"][first] += stretch
        try:
            oracle_mod.ref_proxy_candidates(sc)
            ref_ok = True
        except Exception:
            ref_ok = False
        try:
            mine_ok = cpp.validate_proxy_scene(sc)
        except ValueError:
            mine_ok = False
        assert mine_ok == ref_ok, stretch


# ---- proxy scene build --------------------------------------------------------

def overlapping_build_input():
    """The reference's MakeOverlappingSceneInput (test_rt_candidate.cpp:49-94):
    a swept-AABB patch at x = 0 (object 10) and a capsule patch at x = 0.25
    (object 20), radius 0.2, both still over [0, 1] in 2 slabs, eps 0.05."""
    still = np.array([[0.0, 1.0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1]], np.float64)
    objs = []
    for oid, typ, pid, x in ((10, 1, 1, 0.0), (20, 2, 2, 0.25)):
        objs.append({"object_id": oid, "proxy_type": typ, "slabs_per_motion_segment": 2, "eps_proxy": 0.05,
                     "patch_id": np.array([pid], np.uint32), "local_center": np.array([[x, 0.0, 0.0]]),
                     "radius": np.array([0.2]), "segments": still.copy()})
    return {"query_id": 42, "objects": objs}


def _same(a, b, keys):
    return [k for k in keys if not np.array_equal(np.ascontiguousarray(a[k]).view(np.uint8),
                                                  np.ascontiguousarray(b[k]).view(np.uint8))]


@pytest.mark.parametrize("seed,objs,patches,segs,slabs", [(1, 8, 30, 3, 2), (2, 5, 50, 1, 4), (3, 12, 10, 2, 3)])
def test_build_restatement_matches_reference(oracle_mod, seed, objs, patches, segs, slabs):
    from p2cccd_b200 import scenes

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    inp = scenes.proxy_build_input(n_objects=objs, patches_per_object=patches, n_segments=segs, slabs=slabs,
                                   seed=seed)
    r, m = oracle_mod.ref_build_proxy_scene(inp), oracle_mod.build_proxy_scene(inp)
    assert r["n"] == m["n"] == objs * patches * segs * slabs
    assert _same(r, m, [k for k, _, _ in oracle_mod.BUILT_FIELDS]) == []


def test_build_known_answers(oracle_mod):
    """test_rt_candidate.cpp:98-156 on the restated build and candidates."""
    import p2cccd_cpp as cpp
    from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE, RAW_HIT_DTYPE

    sc = oracle_mod.build_proxy_scene(overlapping_build_input())
    assert sc["query_id"] == 42 and sc["n"] == 4
    assert cpp.validate_proxy_scene(sc)
    raw, cand = oracle_mod.proxy_candidates(sc)
    assert len(raw) == 2 and all(raw["flags"] & 3 == 3) and all(raw["motion_bound"][:, 3] > 0)
    assert len(cand) == 2 and all(cand["object_a_id"] == 10) and all(cand["object_b_id"] == 20)
    assert all(cand["rt_hit_count"] == 1) and all(cand["candidate_id"] != 0)
    d = cpp._density(sc, raw, cand, cpp.RtCandidateTiming(), "cpu_reference")
    assert (d.proxy_count, d.object_count, d.slab_count, d.cross_object_same_slab_pair_count, d.raw_hit_count,
            d.compact_candidate_count, d.aabb_overlap_ratio) == (4, 2, 2, 2, 2, 2, 1.0)
    if oracle_mod.ref_available():
        r = oracle_mod.ref_build_proxy_scene(overlapping_build_input())
        assert _same(r, sc, [k for k, _, _ in oracle_mod.BUILT_FIELDS]) == []


def _mutations():
    """(label, mutate(inp)) pairs, each an input BuildProxyScene rejects."""
    def obj(k, key, v):
        def f(inp):
            inp["objects"][k][key] = v
        return f

    def seg(k, col, v):
        def f(inp):
            inp["objects"][k]["segments"][0, col] = v
        return f

    def quat_zero(inp):
        inp["objects"][1]["segments"][0, 5:9] = 0.0

    def query0(inp):
        inp["query_id"] = 0

    return [("unknown proxy type", obj(0, "proxy_type", 0)),
            ("non-global slab grid", obj(1, "slabs_per_motion_segment", 3)),
            ("zero slabs", obj(0, "slabs_per_motion_segment", 0)),
            ("negative eps", obj(1, "eps_proxy", -1e-3)),
            ("nan eps", obj(1, "eps_proxy", float("nan"))),
            ("segment t0 >= t1", seg(0, 1, 0.0)),
            ("non-finite translation", seg(1, 3, float("inf"))),
            ("zero quaternion", quat_zero),
            ("non-finite quaternion", seg(0, 14, float("nan"))),
            ("query id 0", query0)]


def _reject_message(fn, inp):
    try:
        fn(inp)
    except ValueError as e:
        return str(e)
    return None


def _library_host_check(inp):
    """p2c_proxy_scene_build's host-side validation (it fails before any
    device work on these inputs; the output pointers are never touched)."""
    import ctypes

    from p2cccd_b200 import _lib
    from p2cccd_b200.proxy import ProxyBuildOutStruct, ProxyObjectStruct

    L = _lib.load()
    objs = inp["objects"]
    arr = (ProxyObjectStruct * len(objs))()
    keep, off = [], 0
    for i, o in enumerate(objs):
        s = np.ascontiguousarray(o["segments"], np.float64)
        keep.append(s)
        arr[i].object_id, arr[i].proxy_type = o["object_id"], o["proxy_type"]
        arr[i].slabs_per_motion_segment, arr[i].eps_proxy = o["slabs_per_motion_segment"], o["eps_proxy"]
        arr[i].patch_offset, arr[i].n_patches, arr[i].n_segments = off, len(o["patch_id"]), len(s)
        arr[i].segments = s.ctypes.data
        off += len(o["patch_id"])
    out = ProxyBuildOutStruct(*([16] * 11))
    rc = L.p2c_proxy_scene_build(int(inp["query_id"]), arr, len(objs), 16, 16, 16, off, 1 << 30, ctypes.byref(out),
                                 16, 16, 1 << 30, None)
    assert rc != 0, "expected a host-side rejection"
    return _lib.last_error()


def test_build_rejections_match_reference(oracle_mod):
    import copy

    import torch

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    for label, mutate in _mutations():
        inp = copy.deepcopy(overlapping_build_input())
        mutate(inp)
        ref_msg = _reject_message(oracle_mod.ref_build_proxy_scene, inp)
        assert ref_msg is not None, label
        assert _reject_message(oracle_mod.build_proxy_scene, inp) == ref_msg, label
        if not torch.cuda.is_available():  # the check never reaches the device; keep it off real devices anyway
            assert _library_host_check(inp) == ref_msg, label


# ---- proposal feature rows ---------------------------------------------------

@pytest.mark.parametrize("seed,dups,slabs", [(1, 0.0, 3), (2, 0.5, 3), (3, 0.2, 1), (4, 0.4, 6)])
def test_feature_rows_restatement_matches_reference(oracle_mod, seed, dups, slabs):
    """Density stats (ComputeCandidateDensityStats) and feature rows
    (ExtractProposalFeatureRows) restated, byte for byte with the reference;
    repeated patches exercise the first-proxy-in-scene-order lookup."""
    from p2cccd_b200 import scenes

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=5, patches_per_object=30, n_slabs=slabs, seed=seed, duplicates=dups)
    d_ref, rows_ref = oracle_mod.ref_proposal_feature_rows(sc)
    raw, cand = oracle_mod.proxy_candidates(sc)
    d = oracle_mod.candidate_density(sc, raw, cand)
    rows = oracle_mod.proposal_feature_rows(sc, cand, d)
    assert len(rows_ref) == len(cand) > 0
    assert d.tobytes() == d_ref.tobytes()
    assert np.array_equal(rows.view(np.uint8), rows_ref.view(np.uint8))


def test_feature_rows_known_properties(oracle_mod):
    """test_proposal_features.cpp:101-118 on the overlapping scene: one row per
    candidate, schema 1, the scene's query id, a one-hot interval target, both
    family targets set, a non-zero target mask, finite features."""
    sc = oracle_mod.build_proxy_scene(overlapping_build_input())
    raw, cand = oracle_mod.proxy_candidates(sc)
    rows = oracle_mod.proposal_feature_rows(sc, cand, oracle_mod.candidate_density(sc, raw, cand))
    assert len(rows) == len(cand) == 2
    assert all(rows["schema_version"] == 1) and all(rows["query_id"] == 42)
    assert np.array_equal(rows["interval_targets"].sum(1), np.ones(2, np.float32))
    assert np.all(rows["family_targets"][:, :2] == 1.0) and np.all(rows["target_mask"] != 0)
    assert np.all(np.isfinite(rows["features"]))
    # the two slabs of [0, 1]: interval bins 2 and 6 (centres 0.25 and 0.75)
    assert sorted(np.argmax(rows["interval_targets"], 1).tolist()) == [2, 6]


@pytest.mark.parametrize("masks", [None, {7: 1}, {7: 2}, {7: 0}, {8: 1}])
def test_runtime_feature_rows_restatement_matches_reference(oracle_mod, masks):
    """BuildProposalFeatureRowsFromRuntimeCandidates restated, byte for byte:
    no mask, point-triangle only, edge-edge only, a zero mask (both
    families) and another query's mask."""
    from p2cccd_b200 import scenes

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=5, patches_per_object=30, n_slabs=3, seed=2, duplicates=0.5)
    raw, cand = oracle_mod.proxy_candidates(sc)
    a = oracle_mod.ref_runtime_feature_rows(cand, int(sc["n"]), len(raw), len(cand), masks)
    b = oracle_mod.runtime_feature_rows(cand, int(sc["n"]), len(raw), len(cand), masks)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    # one proxy: overlap denominator 1; no candidates: ratios 0
    a1 = oracle_mod.ref_runtime_feature_rows(cand[:3], 1, 5, 0, masks)
    b1 = oracle_mod.runtime_feature_rows(cand[:3], 1, 5, 0, masks)
    assert np.array_equal(a1.view(np.uint8), b1.view(np.uint8))


def test_runtime_feature_rows_reject_zero_primitives(oracle_mod):
    import torch

    from p2cccd_b200 import _lib

    msg = "CandidateDensityStats.proxy_count must be non-zero"
    if oracle_mod.ref_available():
        with pytest.raises(ValueError, match=msg):
            oracle_mod.ref_runtime_feature_rows(np.zeros(0, np.uint8), 0, 0, 0)
    with pytest.raises(ValueError, match=msg):
        oracle_mod.runtime_feature_rows([], 0, 0, 0)
    if not torch.cuda.is_available():  # host-side check, before any device work
        with pytest.raises(ValueError, match=msg):
            _lib.check(_lib.load().p2c_runtime_feature_rows(None, 0, 0, 0, 0, None, None, 0, None, 16, None))


# ---- audit rows ---------------------------------------------------------------

@pytest.mark.parametrize("emit", [True, False])
def test_audit_rows_restatement_matches_reference(oracle_mod, emit):
    from audit_queue import make_queue

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    items, pts, pt_off, ees, ee_off = make_queue()
    certs, rows = oracle_mod.ref_process_queue(items, pts, pt_off, ees, ee_off, first_event_id=500,
                                               first_timestamp_us=800, emit_dequeue=emit)
    assert len(rows) == len(items) * (2 if emit else 1)
    assert (certs["reason_code"] == 3).sum() == 1  # the NaN primitive's item
    mine = oracle_mod.audit_rows(items, certs, 500, 800, emit)
    assert np.array_equal(mine.view(np.uint8), rows.view(np.uint8))


# ---- runtime exact work queue from proposals ---------------------------------

@pytest.mark.parametrize("cfg", [{}, {"preserve_candidate_order": True}, {"family_score_threshold": 0.6,
                                                                           "uncertainty_fallback_threshold": 0.5,
                                                                           "first_work_item_id": 1000,
                                                                           "conservative_feature_family_mask": 2,
                                                                           "fallback_interval_t0": 0.25,
                                                                           "fallback_interval_t1": 0.75}])
def test_schedule_restatement_matches_reference(oracle_mod, cfg):
    from sched_inputs import make_inputs

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    cand, rows, outs, _ = make_inputs()
    masks = {7: 1, 99: 2}
    ref_items, ref_stats = oracle_mod.ref_schedule_runtime(cand, rows, outs, masks, **cfg)
    items, stats = oracle_mod.schedule_runtime(cand, rows, outs, masks, 0, **cfg)
    assert np.array_equal(items.view(np.uint8), ref_items.view(np.uint8))
    assert stats.tobytes() == ref_stats.tobytes()
    assert ref_stats["missing_proposal_fallback_count"] == 6 and ref_stats["invalid_proposal_fallback_count"] >= 5
    assert ref_stats["ood_fallback_count"] >= 3 and ref_stats["high_uncertainty_fallback_count"] > 0
    if not cfg.get("preserve_candidate_order"):
        assert ref_stats["reordered_count"] > 0


def test_aligned_schedule_equals_candidate_schedule(oracle_mod):
    """The binding's aligned-array form on rows whose features[3] is the hit
    count (runtime rows) and outputs paired with them gives the reference's
    candidate-form queue."""
    from sched_inputs import make_inputs

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    cand, rows, _, outs_all = make_inputs(seed=4)
    ref_items, ref_stats = oracle_mod.ref_schedule_runtime(cand, rows, outs_all, {})
    items, stats = oracle_mod.schedule_runtime(cand, rows, outs_all, {}, 1)
    assert np.array_equal(items.view(np.uint8), ref_items.view(np.uint8))
    assert stats.tobytes() == ref_stats.tobytes()


def test_schedule_rejections_match_reference(oracle_mod):
    from sched_inputs import make_inputs

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    cand, rows, outs, _ = make_inputs(seed=5)
    cases = []
    bad = rows.copy(); bad["candidate_id"][1] = bad["candidate_id"][0]; cases.append((cand, bad, outs, {}))
    bad = outs.copy(); bad["candidate_id"][2] = 0; cases.append((cand, rows, bad, {}))
    bad = cand.copy(); bad["rt_hit_count"][4] = 0; cases.append((bad, rows, outs, {}))
    bad = cand.copy(); bad["candidate_id"][5] = bad["candidate_id"][6]; cases.append((bad, rows, outs, {}))
    cases.append((cand, rows, outs, {7: 4}))  # unknown family bit
    for c, r, o, m in cases:
        with pytest.raises(ValueError):
            oracle_mod.ref_schedule_runtime(c, r, o, m)
        with pytest.raises(ValueError):
            oracle_mod.schedule_runtime(c, r, o, m, 0)
    with pytest.raises(ValueError, match="first_work_item_id"):
        oracle_mod.ref_schedule_runtime(cand, rows, outs, {}, first_work_item_id=0)


def test_reference_compaction_of_its_own_hits(oracle_mod):
    """The compaction wrapper over given hits reproduces the reference's
    generated candidates when handed the reference's raw hits."""
    from p2cccd_b200 import scenes

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=5, patches_per_object=30, n_slabs=3, seed=7, duplicates=0.3)
    raw, cand = oracle_mod.ref_proxy_candidates(sc)
    got = oracle_mod.ref_compact_raw(sc, raw)
    assert got.tobytes() == cand.tobytes()
