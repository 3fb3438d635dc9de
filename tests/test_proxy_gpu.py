"""GPU parity of p2c_proxy_candidates with the reference's proxy candidate
generation (compiled unchanged): raw hits and candidate records byte for
byte, including compaction of repeated patches, capacity retries and an
invalid scene."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,dups,slabs,objs,patches", [(1, 0.0, 4, 6, 40), (2, 0.5, 3, 5, 60),
                                                           (3, 0.2, 1, 8, 200), (4, 0.0, 16, 3, 10)])
def test_device_proxy_candidates_match_reference(cuda_device, oracle_mod, seed, dups, slabs, objs, patches):
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=objs, patches_per_object=patches, n_slabs=slabs, seed=seed, duplicates=dups)
    ref_raw, ref_cand = oracle_mod.ref_proxy_candidates(sc)
    pc = ProxyCandidates(sc, cuda_device, raw_capacity=64)  # too small: retried with a larger buffer
    raw, cand = pc.run_checked()
    assert len(raw) == len(ref_raw) and len(cand) == len(ref_cand)
    assert np.array_equal(raw.view(np.uint8), ref_raw.view(np.uint8))
    assert np.array_equal(cand.view(np.uint8), ref_cand.view(np.uint8))


def test_device_proxy_candidates_flag_invalid_scene(cuda_device):
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates

    sc = scenes.proxy_scene(n_objects=3, patches_per_object=5, n_slabs=2, seed=9)
    sc["t1"][3] = sc["t0"][3]  # t0 < t1 broken
    with pytest.raises(ValueError):
        ProxyCandidates(sc, cuda_device).run_checked()
    sc = scenes.proxy_scene(n_objects=3, patches_per_object=5, n_slabs=2, seed=9)
    sc["query_id"] = 0
    with pytest.raises(ValueError):
        ProxyCandidates(sc, cuda_device).run()


def test_device_proxy_candidates_zero_capacity_counts_hits(cuda_device, oracle_mod):
    import numpy as np
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ERR_OVERFLOW, ProxyCandidates

    sc = scenes.proxy_scene(n_objects=4, patches_per_object=20, n_slabs=2, seed=3)
    n_ref = len(oracle_mod.proxy_candidates(sc)[0])
    pc = ProxyCandidates(sc, cuda_device, raw_capacity=0)
    pc.run()
    c = pc.counts.cpu().numpy()
    assert int(c[0]) == n_ref > 0 and int(c[1]) == 0 and int(c[2]) & ERR_OVERFLOW
    empty = dict(sc, n=0, **{k: np.asarray(sc[k])[:0] for k, _ in ProxyCandidates.FIELDS})
    raw, cand = ProxyCandidates(empty, cuda_device).run_checked()
    assert len(raw) == 0 and len(cand) == 0


def test_mirror_generate_candidates_for_proxy_scene(cuda_device, oracle_mod):
    import p2cccd_cpp as cpp
    from p2cccd_b200 import scenes
    from test_proxy_oracle import _scene_object

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=4, patches_per_object=25, n_slabs=3, seed=6, duplicates=0.4)
    ref_raw, ref_cand = oracle_mod.ref_proxy_candidates(sc)
    obj = _scene_object(sc)
    res = cpp.generate_candidates_for_proxy_scene(obj)
    assert res.backend_name == "cpu_reference" and res.density.backend_name == "cpu_reference"
    hits = res.raw_buffer.hits
    assert [h.pair_key for h in hits] == [int(x) for x in ref_raw["pair_key"]]
    assert [h.motion_bound for h in hits] == [[float(x) for x in r] for r in ref_raw["motion_bound"]]
    assert len(res.candidates) == len(ref_cand)
    for c, r in zip(res.candidates, ref_cand):
        assert (c.candidate_id, c.slab_id, c.object_a_id, c.patch_a_id, c.object_b_id, c.patch_b_id,
                int(c.proxy_type_a), int(c.proxy_type_b), c.rt_hit_count, c.flags) == \
            tuple(int(r[k]) for k in ("candidate_id", "slab_id", "object_a_id", "patch_a_id", "object_b_id",
                                      "patch_b_id", "proxy_type_a", "proxy_type_b", "rt_hit_count", "flags"))
    d = res.density
    assert d.raw_hit_count == len(ref_raw) and d.compact_candidate_count == len(ref_cand)
    assert d.avg_rt_hits_per_candidate == float(ref_cand["rt_hit_count"].sum()) / len(ref_cand)
    raw_only = cpp.generate_raw_candidates_cpu(obj)
    assert [h.pair_key for h in raw_only.hits] == [h.pair_key for h in hits]
    with pytest.raises(ValueError, match="OptiX"):
        cpp.generate_candidates_for_proxy_scene(obj, backend_name="optix")
    fb = cpp.generate_candidates_for_proxy_scene(obj, backend_name="optix_rt", allow_optix_cpu_fallback=True)
    assert fb.backend_name == "optix_cpu_fallback" and len(fb.candidates) == len(ref_cand)
    with pytest.raises(ValueError, match="match"):
        cpp.generate_candidates_for_proxy_scene(obj, query_id=obj.query_id + 1)
    with pytest.raises(ValueError, match="unsupported candidate backend"):
        cpp.generate_candidates_for_proxy_scene(obj, backend_name="embree")


def test_motion_bound_error_only_in_compaction(cuda_device):
    import p2cccd_cpp as cpp
    from p2cccd_b200 import scenes

    sc = scenes.proxy_scene(n_objects=3, patches_per_object=8, n_slabs=2, seed=4)
    sc["motion_bound"][:, 2] = 1e300  # finite as a double, infinite as the hit's float
    hits = cpp.generate_raw_candidates_cpu(sc).hits
    assert len(hits) > 0 and all(h.motion_bound[2] == float("inf") for h in hits)
    with pytest.raises(ValueError, match="motion_bound"):
        cpp.generate_candidates_for_proxy_scene(sc)


@pytest.mark.parametrize("seed,objs,patches,segs,slabs", [(1, 8, 30, 3, 2), (2, 5, 50, 1, 4), (7, 16, 120, 2, 3)])
def test_device_build_matches_reference(cuda_device, oracle_mod, seed, objs, patches, segs, slabs):
    """BuildProxyScene on the device: every output field byte for byte with
    the reference, then the device candidates of the device-resident scene."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates, ProxySceneBuild

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    inp = scenes.proxy_build_input(n_objects=objs, patches_per_object=patches, n_segments=segs, slabs=slabs,
                                   seed=seed)
    ref = oracle_mod.ref_build_proxy_scene(inp)
    b = ProxySceneBuild(inp, cuda_device)
    dev_scene = b.run_checked()
    got = b.to_host()
    assert got["n"] == ref["n"]
    for k, _, _ in oracle_mod.BUILT_FIELDS:
        assert np.array_equal(np.ascontiguousarray(got[k]).view(np.uint8),
                              np.ascontiguousarray(ref[k]).view(np.uint8)), k
    raw, cand = ProxyCandidates(dev_scene, cuda_device).run_checked()
    ref_raw, ref_cand = oracle_mod.ref_proxy_candidates(ref)
    assert np.array_equal(raw.view(np.uint8), ref_raw.view(np.uint8))
    assert np.array_equal(cand.view(np.uint8), ref_cand.view(np.uint8))


def test_device_build_known_answers_and_mirror(cuda_device, oracle_mod):
    """test_rt_candidate.cpp:98-156 through the p2cccd_cpp mirror objects."""
    import p2cccd_cpp as cpp
    from test_proxy_oracle import overlapping_build_input

    a = overlapping_build_input()
    inp = cpp.ProxySceneBuildInput()
    inp.query_id = a["query_id"]
    for o in a["objects"]:
        ob = cpp.ProxyObjectBuildInput()
        ob.object_id, ob.proxy_type = o["object_id"], cpp.ProxyType(o["proxy_type"])
        ob.slabs_per_motion_segment, ob.eps_proxy = o["slabs_per_motion_segment"], o["eps_proxy"]
        p = cpp.Patch()
        p.patch_id, p.local_center, p.radius = int(o["patch_id"][0]), o["local_center"][0].tolist(), 0.2
        ob.patches = [p]
        m = cpp.MotionSegment()
        m.pose_t0.translation = [0.0, 0.0, 0.0]
        m.pose_t1.translation = [0.0, 0.0, 0.0]
        ob.motion_segments = [m]
        inp.objects.append(ob)
    scene = cpp.build_proxy_scene(inp)
    assert scene.query_id == 42 and len(scene.primitives) == 4
    assert [p.proxy_id for p in scene.primitives] == [0, 1, 2, 3]
    cap = scene.primitives[2]
    assert cap.proxy_type == cpp.ProxyType.CAPSULE and cap.capsule.radius == 0.2 + 0.05
    assert cap.capsule.endpoint0 == [0.25, 0.0, 0.0]
    assert cpp.validate_proxy_scene(scene)
    res = cpp.generate_candidates_for_proxy_scene(scene)
    assert len(res.raw_buffer.hits) == 2 and len(res.candidates) == 2
    assert all(c.object_a_id == 10 and c.object_b_id == 20 and c.rt_hit_count == 1 for c in res.candidates)
    d = res.density
    assert (d.proxy_count, d.object_count, d.slab_count, d.cross_object_same_slab_pair_count,
            d.aabb_overlap_ratio) == (4, 2, 2, 2, 1.0)
    ref = oracle_mod.ref_build_proxy_scene(a)
    assert [p.bounds.min + p.bounds.max for p in scene.primitives] == ref["bounds"].tolist()
    bad = cpp.ProxySceneBuildInput()
    bad.query_id, bad.objects = 42, list(inp.objects)
    bad.objects[1] = cpp.ProxyObjectBuildInput()
    bad.objects[1].proxy_type, bad.objects[1].patches = cpp.ProxyType.UNKNOWN, [cpp.Patch()]
    bad.objects[1].motion_segments = [cpp.MotionSegment()]
    with pytest.raises(ValueError, match="concrete"):
        cpp.build_proxy_scene(bad)


def test_device_build_flags_bad_patches(cuda_device, oracle_mod):
    from test_proxy_oracle import overlapping_build_input
    from p2cccd_b200.proxy import ProxySceneBuild

    for key, value, msg in (("local_center", np.array([[np.nan, 0.0, 0.0]]), "local_center"),
                            ("radius", np.array([-0.1]), "radius")):
        a = overlapping_build_input()
        a["objects"][1][key] = value
        if oracle_mod.ref_available():
            with pytest.raises(ValueError, match=msg):
                oracle_mod.ref_build_proxy_scene(a)
        with pytest.raises(ValueError, match=msg):
            ProxySceneBuild(a, cuda_device).run_checked()


def test_fitted_capacity_keeps_results(cuda_device, oracle_mod):
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates

    sc = scenes.proxy_scene(n_objects=7, patches_per_object=90, n_slabs=5, seed=12, duplicates=0.3)
    ref_raw, ref_cand = oracle_mod.proxy_candidates(sc)
    pc = ProxyCandidates(sc, cuda_device)
    raw0, cand0 = pc.run_checked()
    assert pc.fit_capacity(margin=1.0, slack=0) == len(ref_raw)  # exactly full: no overflow
    raw1, cand1 = pc.run_checked()
    for raw, cand in ((raw0, cand0), (raw1, cand1)):
        assert np.array_equal(raw.view(np.uint8), ref_raw.view(np.uint8))
        assert np.array_equal(cand.view(np.uint8), ref_cand.view(np.uint8))


def test_wrong_id_width_hint_falls_back(cuda_device, oracle_mod):
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ERR_ID_BITS, ProxyCandidates

    sc = scenes.proxy_scene(n_objects=5, patches_per_object=50, n_slabs=6, seed=21, duplicates=0.2)
    ref_raw, ref_cand = oracle_mod.proxy_candidates(sc)
    for hint in ((2, 3, 6), (3, 1, 6), (3, 3, 4)):  # slab, object, patch ids wider than claimed
        pc = ProxyCandidates(dict(sc, id_bits=hint), cuda_device)
        pc.run()
        assert int(pc.counts[2].item()) & ERR_ID_BITS
        raw, cand = pc.run_checked()
        assert np.array_equal(raw.view(np.uint8), ref_raw.view(np.uint8))
        assert np.array_equal(cand.view(np.uint8), ref_cand.view(np.uint8))
    exact = ProxyCandidates(dict(sc, id_bits=(3, 3, 6)), cuda_device)  # max ids 5, 4, 49
    raw, cand = exact.run_checked()
    assert exact._struct.slab_bits == 3 and np.array_equal(cand.view(np.uint8), ref_cand.view(np.uint8))


@pytest.mark.parametrize("mode", ["table", "no_hint", "wide_slabs"])
def test_sweep_paths_agree(cuda_device, oracle_mod, mode):
    """The direct (slab, column) table (narrow slab ids) and the binary
    search over the sorted keys (no hint, or slab ids wider than the table)
    give the reference's hits."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates

    for seed, dups in ((31, 0.0), (32, 0.4)):
        sc = scenes.proxy_scene(n_objects=9, patches_per_object=70, n_slabs=5, seed=seed, duplicates=dups)
        if mode == "wide_slabs":
            sc["slab_id"] = (sc["slab_id"].astype(np.uint64) * 40_000_003 % (1 << 32)).astype(np.uint32)
        ref_raw, ref_cand = oracle_mod.proxy_candidates(sc)
        pc = ProxyCandidates(dict(sc, id_bits=(0, 0, 0)) if mode == "no_hint" else sc, cuda_device)
        raw, cand = pc.run_checked()
        table = 0 < pc._struct.slab_bits <= 6
        assert table == (mode == "table")
        assert np.array_equal(raw.view(np.uint8), ref_raw.view(np.uint8))
        assert np.array_equal(cand.view(np.uint8), ref_cand.view(np.uint8))


@pytest.mark.parametrize("seed,dups,hint", [(1, 0.0, True), (2, 0.5, True), (4, 0.4, False), (5, 0.0, False)])
def test_device_feature_rows_match_reference(cuda_device, oracle_mod, seed, dups, hint):
    """p2c_proposal_feature_rows: density stats and every 256-byte row byte for
    byte with the reference's ComputeCandidateDensityStats +
    ExtractProposalFeatureRows, with and without the id width hints."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=6, patches_per_object=40, n_slabs=4, seed=seed, duplicates=dups)
    d_ref, rows_ref = oracle_mod.ref_proposal_feature_rows(sc)
    pc = ProxyCandidates(sc if hint else dict(sc, id_bits=(0, 0, 0)), cuda_device)
    pc.run_checked()
    dens, rows = pc.feature_rows()
    assert dens.tobytes() == d_ref.tobytes()
    assert len(rows) == len(rows_ref) > 0
    assert np.array_equal(rows.view(np.uint8), rows_ref.view(np.uint8))


def test_device_feature_rows_of_a_built_scene(cuda_device, oracle_mod):
    """Build, candidates and feature rows all on the device, against the
    reference's build + generation + ExtractProposalFeatureRows."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates, ProxySceneBuild

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    inp = scenes.proxy_build_input(n_objects=10, patches_per_object=40, n_segments=2, slabs=3, seed=8)
    ref_scene = oracle_mod.ref_build_proxy_scene(inp)
    d_ref, rows_ref = oracle_mod.ref_proposal_feature_rows(ref_scene)
    pc = ProxyCandidates(ProxySceneBuild(inp, cuda_device).run_checked(), cuda_device)
    pc.run_checked()
    dens, rows = pc.feature_rows()
    assert dens.tobytes() == d_ref.tobytes()
    assert np.array_equal(rows.view(np.uint8), rows_ref.view(np.uint8))


def test_device_feature_rows_flag_bad_candidates(cuda_device):
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates

    sc = scenes.proxy_scene(n_objects=4, patches_per_object=20, n_slabs=2, seed=3)
    pc = ProxyCandidates(sc, cuda_device)
    pc.run_checked()
    pc.cand[0, 32:36] = 255  # patch_a_id of candidate 0: no proxy has it
    with pytest.raises(ValueError, match="map to proxy"):
        pc.feature_rows()
    pc.run_checked()
    pc.cand[1, 0] = 7  # schema_version of candidate 1
    with pytest.raises(ValueError, match="validation"):
        pc.feature_rows()
    pc.run_checked()
    dens, rows = pc.feature_rows()
    assert len(rows) == int(dens["compact_candidate_count"]) > 0


@pytest.mark.parametrize("masks", [None, {7: 1}, {7: 2}, {7: 0}])
def test_device_runtime_feature_rows_match_reference(cuda_device, oracle_mod, masks):
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates, runtime_feature_rows

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=6, patches_per_object=40, n_slabs=4, seed=6, duplicates=0.3)
    pc = ProxyCandidates(sc, cuda_device)
    raw, cand = pc.run_checked()
    ref = oracle_mod.ref_runtime_feature_rows(cand, int(sc["n"]), len(raw), len(cand), masks)
    got = runtime_feature_rows(cand, int(sc["n"]), len(raw), len(cand), masks, cuda_device)
    assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))
    # straight from the device candidates of the run
    got_dev = runtime_feature_rows(pc.cand[:len(cand)], int(sc["n"]), len(raw), len(cand), masks, cuda_device)
    assert np.array_equal(got_dev.view(np.uint8), ref.view(np.uint8))
    bad = cand.copy()
    bad["rt_hit_count"][2] = 0
    with pytest.raises(ValueError, match="validation"):
        runtime_feature_rows(bad, int(sc["n"]), len(raw), len(cand), masks, cuda_device)


def test_mirror_feature_row_functions(cuda_device, oracle_mod):
    import p2cccd_cpp as cpp
    from p2cccd_b200 import scenes
    from test_proxy_oracle import _scene_object

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    sc = scenes.proxy_scene(n_objects=4, patches_per_object=25, n_slabs=3, seed=9, duplicates=0.3)
    obj = _scene_object(sc)
    res = cpp.generate_candidates_for_proxy_scene(obj)
    _, ref_rows = oracle_mod.ref_proposal_feature_rows(sc)
    rows = cpp.extract_proposal_feature_rows(obj, res)
    assert len(rows) == len(ref_rows)
    for o, r in zip(rows, ref_rows):
        assert o.candidate_id == int(r["candidate_id"]) and o.features == [float(x) for x in r["features"]]
        assert o.interval_targets == [float(x) for x in r["interval_targets"]]
        assert (o.priority_target, o.cost_target, o.uncertainty_target) == \
            (float(r["priority_target"]), float(r["cost_target"]), float(r["uncertainty_target"]))
    masks = {int(sc["query_id"]): 2}
    n_raw, n_cand = len(res.raw_buffer.hits), len(res.candidates)
    ref_rt = oracle_mod.ref_runtime_feature_rows(cpp._candidate_array(res.candidates), int(sc["n"]), n_raw, n_cand,
                                                 masks)
    arrays = cpp.build_runtime_proposal_feature_arrays(res.candidates, int(sc["n"]), n_raw, n_cand, masks)
    assert arrays["schema_version"] == 1
    for k in ("features", "family_targets", "priority_target", "cost_target", "uncertainty_target", "candidate_id"):
        assert np.array_equal(arrays[k], ref_rt[k]), k
    rt_rows = cpp.build_runtime_proposal_feature_rows(res.candidates, int(sc["n"]), n_raw, n_cand, masks)
    assert [o.family_targets[:2] for o in rt_rows] == [[0.0, 1.0]] * n_cand
    with pytest.raises(ValueError, match="non-zero"):
        cpp.build_runtime_proposal_feature_rows(res.candidates, 0, n_raw, n_cand, masks)


def test_feature_rows_need_a_run_after_resizing(cuda_device):
    from p2cccd_b200 import scenes
    from p2cccd_b200.proxy import ProxyCandidates

    pc = ProxyCandidates(scenes.proxy_scene(n_objects=3, patches_per_object=10, n_slabs=2, seed=4), cuda_device)
    with pytest.raises(RuntimeError):
        pc.feature_rows()
    pc.run_checked()
    pc.fit_capacity()
    with pytest.raises(RuntimeError):
        pc.feature_rows()
    pc.run_checked()
    dens, rows = pc.feature_rows()
    assert len(rows) == int(dens["compact_candidate_count"])


@pytest.mark.parametrize("emit", [True, False])
def test_device_audit_rows_match_reference(cuda_device, oracle_mod, emit):
    """Certificates from the device queue path, then p2c_audit_rows: every
    80-byte AuditLogRow equal to the reference ProcessExactWorkQueueCpu's."""
    from audit_queue import make_queue
    from p2cccd_b200 import queue
    from p2cccd_b200.certify import CertConfig

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    items, pts, pt_off, ees, ee_off = make_queue()
    ref_certs, ref_rows = oracle_mod.ref_process_queue(items, pts, pt_off, ees, ee_off, 1e-6, 1e-6, 32, 500, 800,
                                                       emit)
    res = queue.certify_work_items(pts, pt_off, ees, ee_off, items["interval_t0"], items["interval_t1"],
                                   items["feature_family_mask"], CertConfig(1e-6, 1e-6, 32), cuda_device)
    certs = res["certs"]
    for k in ("status", "reason_code", "toi_upper", "safe_margin_lb", "next_refinement_mode"):
        assert np.array_equal(certs[k], ref_certs[k]), k
    rows = queue.audit_rows(items, certs, 500, 800, emit, cuda_device)
    assert np.array_equal(rows.view(np.uint8), ref_rows.view(np.uint8))


def test_mirror_queue_audit_log_matches_reference(cuda_device, oracle_mod):
    import p2cccd_cpp as cpp
    from audit_queue import make_queue

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    items, pts, pt_off, ees, ee_off = make_queue(n_items=40, seed=6)
    _, ref_rows = oracle_mod.ref_process_queue(items, pts, pt_off, ees, ee_off, 1e-6, 1e-6, 32, 7, 9, True)
    queries = []
    pt_objs = cpp._from_records(pts, 1)
    ee_objs = cpp._from_records(ees, 2)
    for k, it in enumerate(items):
        q = cpp.ExactCertificateQuery()
        w = q.work_item
        w.work_item_id, w.parent_candidate_id, w.query_id = (int(it[f]) for f in ("work_item_id", "candidate_id",
                                                                                  "query_id"))
        w.interval_t0, w.interval_t1 = float(it["interval_t0"]), float(it["interval_t1"])
        w.feature_family_mask, w.depth = int(it["feature_family_mask"]), int(it["depth"])
        w.priority_score = float(it["priority_score"])
        q.config.eps_time, q.config.eps_space, q.config.max_subdivision_depth = 1e-6, 1e-6, 32
        q.point_triangle_primitives = pt_objs[pt_off[k]:pt_off[k + 1]]
        q.edge_edge_primitives = ee_objs[ee_off[k]:ee_off[k + 1]]
        queries.append(q)
    cfg = cpp.ExactWorkQueueConfig()
    cfg.first_event_id, cfg.first_timestamp_us, cfg.emit_dequeue_events = 7, 9, True
    res = cpp.process_exact_work_queue_cpu(queries, cfg)
    assert len(res.audit_log) == len(ref_rows)
    for o, r in zip(res.audit_log, ref_rows):
        assert (o.event_id, o.query_id, o.candidate_id, o.work_item_id, int(o.stage), o.action, o.depth,
                o.timestamp_us) == tuple(int(r[k]) for k in ("event_id", "query_id", "candidate_id", "work_item_id",
                                                             "stage", "action", "depth", "timestamp_us"))
        assert (o.interval_t0, o.interval_t1, o.aux_value0, o.aux_value1) == \
            tuple(float(r[k]) for k in ("interval_t0", "interval_t1", "aux_value0", "aux_value1"))


@pytest.mark.parametrize("cfg", [{}, {"preserve_candidate_order": True}, {"family_score_threshold": 0.6,
                                                                           "uncertainty_fallback_threshold": 0.5,
                                                                           "first_work_item_id": 1000,
                                                                           "conservative_feature_family_mask": 2,
                                                                           "fallback_interval_t0": 0.25,
                                                                           "fallback_interval_t1": 0.75}])
def test_device_schedule_matches_reference(cuda_device, oracle_mod, cfg):
    """p2c_schedule_work_items: every 80-byte ExactWorkItem and the stats equal
    to the reference's ScheduleRuntimeExactWorkItemsFromProposals (candidate
    form), and the aligned-array form equal to it on paired inputs."""
    from p2cccd_b200.schedule import schedule_work_items
    from sched_inputs import make_inputs

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    cand, rows, outs, outs_all = make_inputs()
    masks = {7: 1, 99: 2}
    ref_items, ref_stats = oracle_mod.ref_schedule_runtime(cand, rows, outs, masks, **cfg)
    items, stats = schedule_work_items(cand, rows, outs, masks, 0, cuda_device, **cfg)
    assert np.array_equal(items.view(np.uint8), ref_items.view(np.uint8))
    assert stats.tobytes() == ref_stats.tobytes()
    ref_items, ref_stats = oracle_mod.ref_schedule_runtime(cand, rows, outs_all, masks, **cfg)
    items, stats = schedule_work_items(None, rows, outs_all, masks, 1, cuda_device, **cfg)
    assert np.array_equal(items.view(np.uint8), ref_items.view(np.uint8))
    assert stats.tobytes() == ref_stats.tobytes()


def test_device_schedule_rejections(cuda_device, oracle_mod):
    from p2cccd_b200.schedule import schedule_work_items
    from sched_inputs import make_inputs

    cand, rows, outs, outs_all = make_inputs(seed=5)
    cases = []
    bad = rows.copy(); bad["candidate_id"][1] = bad["candidate_id"][0]; cases.append((cand, bad, outs, {}, "rows"))
    bad = outs.copy(); bad["candidate_id"][2] = 0; cases.append((cand, rows, bad, {}, "outputs"))
    bad = cand.copy(); bad["rt_hit_count"][4] = 0; cases.append((bad, rows, outs, {}, "CandidateRecord"))
    bad = cand.copy(); bad["candidate_id"][5] = bad["candidate_id"][6]; cases.append((bad, rows, outs, {}, "duplicate"))
    cases.append((cand, rows, outs, {7: 4}, "feature family"))
    cases.append((cand, rows, outs, {7: 5}, "feature-family bits"))
    for c, r, o, m, msg in cases:
        with pytest.raises(ValueError, match=msg):
            schedule_work_items(c, r, o, m, 0, cuda_device)
        if oracle_mod.ref_available() and "family" in msg:  # the reference's own message for the same input
            with pytest.raises(ValueError) as ref_err:
                oracle_mod.ref_schedule_runtime(c, r, o, m)
            with pytest.raises(ValueError) as dev_err:
                schedule_work_items(c, r, o, m, 0, cuda_device)
            assert str(dev_err.value) == str(ref_err.value)
    swapped = outs_all.copy()
    swapped[[0, 1]] = swapped[[1, 0]]
    with pytest.raises(ValueError, match="preserve candidate_id order"):
        schedule_work_items(None, rows, swapped, {}, 1, cuda_device)
    with pytest.raises(ValueError, match="ood_abs_feature_threshold"):
        schedule_work_items(cand, rows, outs, {}, 0, cuda_device, ood_abs_feature_threshold=0.0)


def test_mirror_schedule_functions(cuda_device, oracle_mod):
    import p2cccd_cpp as cpp
    from sched_inputs import make_inputs

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    cand, rows, outs, outs_all = make_inputs(seed=6)
    masks = {7: 2}
    ref_items, ref_stats = oracle_mod.ref_schedule_runtime(cand, rows, outs, masks)
    cfg = cpp.ProposalSchedulingConfig()
    cand_objs = cpp._candidate_objects(cand)
    row_objs = cpp._row_objects(rows)
    out_objs = []
    for r in outs:
        o = cpp.ProposalOutput()
        o.candidate_id, o.interval_scores, o.family_scores = int(r["candidate_id"]), r["interval_scores"].tolist(), \
            r["family_scores"].tolist()
        o.priority_score, o.cost_score, o.uncertainty_score = (float(r[k]) for k in ("priority_score", "cost_score",
                                                                                     "uncertainty_score"))
        out_objs.append(o)
    queue, stats = cpp.schedule_runtime_exact_work_items(cand_objs, row_objs, out_objs, masks, cfg)
    assert [w.parent_candidate_id for w in queue] == [int(x) for x in ref_items["parent_candidate_id"]]
    assert [int(w.source) for w in queue] == [int(x) for x in ref_items["source"]]
    assert stats.fallback_count == int(ref_stats["fallback_count"]) and stats.monotonic_safe
    fa = cpp.build_runtime_proposal_feature_arrays(cand_objs, 100, 200, len(cand), masks)
    fa["features"] = rows["features"]  # the test rows (with out-of-distribution features)
    pa = {k: outs_all[k] for k in ("interval_scores", "family_scores", "priority_score", "cost_score",
                                   "uncertainty_score")}
    ref2, _ = oracle_mod.ref_schedule_runtime(cand, rows, outs_all, masks)
    q2, _ = cpp.schedule_runtime_exact_work_items_from_arrays(cand_objs, fa, pa, masks, cfg)
    assert [w.parent_candidate_id for w in q2] == [int(x) for x in ref2["parent_candidate_id"]]
    q3, s3 = cpp.schedule_runtime_exact_work_items_from_proposal_arrays(fa, pa, masks, cfg)
    assert [(w.parent_candidate_id, w.feature_family_mask, w.priority_score) for w in q3] == \
        [(int(r["parent_candidate_id"]), int(r["feature_family_mask"]), float(r["priority_score"])) for r in ref2]
    with pytest.raises(ValueError, match="must have shape"):
        cpp.schedule_runtime_exact_work_items_from_proposal_arrays(fa, dict(pa, priority_score=pa["priority_score"][:-1]),
                                                                   masks, cfg)


def _given_hits(oracle_mod, seed=11):
    from p2cccd_b200 import scenes

    sc = scenes.proxy_scene(n_objects=6, patches_per_object=40, n_slabs=3, seed=seed, duplicates=0.3)
    raw, _ = oracle_mod.proxy_candidates(sc)
    g = np.random.default_rng(seed)
    hits = np.concatenate([raw, raw[g.choice(len(raw), len(raw) // 3)]])  # repeated hits sum their counts
    hits = hits[g.permutation(len(hits))]  # the order of the hits does not matter
    hits["rt_hit_count"] = g.integers(1, 5, len(hits))
    hits["flags"] |= g.choice([0, 4, 8], len(hits)).astype(np.uint32)
    hits["motion_bound"] *= g.uniform(1.0, 2.0, (len(hits), 4)).astype(np.float32)
    return sc, hits


@pytest.mark.gpu
def test_device_compaction_of_given_hits(oracle_mod):
    from p2cccd_b200.proxy import ProxyCandidates

    sc, hits = _given_hits(oracle_mod)
    got = ProxyCandidates(sc, raw_capacity=0).compact(hits)
    if oracle_mod.ref_available():
        want = oracle_mod.ref_compact_raw(sc, hits)
        assert got.tobytes() == want.tobytes()
    assert got["rt_hit_count"].sum() == hits["rt_hit_count"].sum()
    raw, cand = oracle_mod.proxy_candidates(sc)  # the scene's own hits give its candidates
    assert ProxyCandidates(sc, raw_capacity=0).compact(raw).tobytes() == cand.tobytes()
    assert len(ProxyCandidates(sc, raw_capacity=0).compact(hits[:0])) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("fault", ["flags", "zero_query", "query", "index", "same", "pair_key", "object", "slab",
                                   "bound", "two", "overflow"])
def test_device_compaction_rejects_hits_like_reference(oracle_mod, fault):
    from p2cccd_b200.proxy import ProxyCandidates

    sc, hits = _given_hits(oracle_mod, seed=12)
    k = len(hits) // 2
    h = hits[k]
    obj = np.asarray(sc["object_id"])
    if fault == "flags":
        hits["flags"][k] &= ~np.uint32(1)
    elif fault == "zero_query":
        hits["query_id"][k] = 0
    elif fault == "query":
        hits["query_id"][k] = int(sc["query_id"]) + 1
    elif fault == "index":
        hits["proxy_b_index"][k] = int(sc["n"]) + 3
    elif fault == "same":
        hits["proxy_b_index"][k] = h["proxy_a_index"]
        hits["pair_key"][k] = (int(h["proxy_a_index"]) << 32) | int(h["proxy_a_index"])
    elif fault == "pair_key":
        hits["pair_key"][k] ^= 1
    elif fault == "object":
        a = int(h["proxy_a_index"])
        b = int(np.nonzero((obj == obj[a]) & (np.arange(len(obj)) != a))[0][0])
        hits["proxy_b_index"][k] = b
        hits["pair_key"][k] = (min(a, b) << 32) | max(a, b)
    elif fault == "slab":
        hits["slab_id"][k] += 1
    elif fault == "bound":
        hits["motion_bound"][k, 2] = -1.0
    elif fault == "two":  # the first invalid hit decides
        hits["motion_bound"][k, 0] = np.inf
        hits["flags"][k + 3] = 0
    else:  # summed counts beyond 32 bits
        dup = hits[k:k + 1].copy()
        dup["rt_hit_count"] = 0xFFFFFFFF
        hits = np.concatenate([hits, dup])
    with pytest.raises(ValueError) as err:
        ProxyCandidates(sc, raw_capacity=0).compact(hits)
    if oracle_mod.ref_available():
        with pytest.raises(ValueError) as ref_err:
            oracle_mod.ref_compact_raw(sc, hits)
        assert str(err.value) == str(ref_err.value)


@pytest.mark.gpu
def test_mirror_compact_raw_candidates(oracle_mod):
    import p2cccd_cpp as cpp

    sc, _ = _given_hits(oracle_mod, seed=13)
    buf = cpp.generate_raw_candidates_cpu(sc)
    got = cpp.compact_raw_candidates(sc, buf)
    want = cpp.generate_candidates_for_proxy_scene(sc).candidates
    assert cpp._candidate_array(got).tobytes() == cpp._candidate_array(want).tobytes()


@pytest.mark.gpu
def test_mirror_candidate_generator(oracle_mod):
    import p2cccd_cpp as cpp

    sc, _ = _given_hits(oracle_mod, seed=14)
    want = cpp._candidate_array(cpp.generate_candidates_for_proxy_scene(sc).candidates)
    gen = cpp.CandidateGenerator()
    assert cpp._candidate_array(gen.trace_candidates_for_proxy_scene(sc)).tobytes() == want.tobytes()
    cfg = cpp.CandidateGeneratorConfig()
    cfg.backend = cpp.CandidateBackend.OPTIX
    assert cpp.CandidateGenerator(cfg).trace_candidates_for_proxy_scene(sc) == []  # built without OptiX
    cfg.allow_optix_cpu_fallback = True
    got = cpp.CandidateGenerator(cfg).trace_candidates_for_proxy_scene(sc)
    assert cpp._candidate_array(got).tobytes() == want.tobytes()
