"""The reference's C++ known-answer tests, replayed through the p2cccd_cpp
mirror (every certificate computed on the GPU)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _vertex(m, fid, p0, p1):
    t = m.LinearVertexTrajectory()
    t.feature_id, t.position_t0, t.position_t1 = fid, list(p0), list(p1)
    return t


def _moving_point(m, z0, z1, pid=10, tid=20):  # test_certificate_engine.cpp:45-57
    p = m.PointTriangleIntervalPrimitive()
    p.point_id, p.triangle_id = pid, tid
    p.point = _vertex(m, pid, (0.25, 0.25, z0), (0.25, 0.25, z1))
    p.triangle_v0 = _vertex(m, 101, (0, 0, 0), (0, 0, 0))
    p.triangle_v1 = _vertex(m, 102, (1, 0, 0), (1, 0, 0))
    p.triangle_v2 = _vertex(m, 103, (0, 1, 0), (0, 1, 0))
    return p


def _moving_edge(m, z0, z1, a=30, b=40):  # :59-71
    p = m.EdgeEdgeIntervalPrimitive()
    p.edge_a_id, p.edge_b_id = a, b
    p.edge_a0 = _vertex(m, 201, (-1, 0, 0), (-1, 0, 0))
    p.edge_a1 = _vertex(m, 202, (1, 0, 0), (1, 0, 0))
    p.edge_b0 = _vertex(m, 301, (0, -1, z0), (0, -1, z1))
    p.edge_b1 = _vertex(m, 302, (0, 1, z0), (0, 1, z1))
    return p


def _cfg(m):
    c = m.CertificateEngineConfig()
    c.eps_time, c.eps_space, c.max_subdivision_depth = 1e-5, 1e-6, 32
    return c


def _item(m, mask, wid=9001):
    it = m.ExactWorkItem()
    it.work_item_id, it.parent_candidate_id, it.query_id = wid, 77, 1234
    it.patch_a_id, it.patch_b_id, it.feature_family_mask, it.priority_score = 1, 2, mask, 1.0
    return it


def test_interval_known_answers(cuda_device):
    import p2cccd_cpp as m

    r = m.evaluate_point_triangle_interval(_moving_point(m, 1.0, -3.0), 0.0, 1.0, _cfg(m))
    assert r.status == m.CertificateStatus.COLLISION and abs(r.toi_upper - 0.25) <= 1e-12
    assert (r.witness_family, r.witness_id_a, r.witness_id_b) == (1, 10, 20)
    r = m.evaluate_point_triangle_interval(_moving_point(m, 2.0, 2.0), 0.0, 1.0, _cfg(m))
    assert r.status == m.CertificateStatus.SEPARATION and r.covered_feature_mask == 1 and r.safe_margin_lb > 1.9
    r = m.evaluate_edge_edge_interval(_moving_edge(m, 1.0, -3.0), 0.0, 1.0, _cfg(m))
    assert r.status == m.CertificateStatus.COLLISION and abs(r.toi_upper - 0.25) <= 1e-12
    assert (r.witness_id_a, r.witness_id_b) == (30, 40)
    rs = m.evaluate_edge_edge_batch_cuda([_moving_edge(m, 1.0, -3.0), _moving_edge(m, 2.0, 2.0, 31, 41)], 0.0, 1.0,
                                         _cfg(m))
    assert [x.status for x in rs] == [m.CertificateStatus.COLLISION, m.CertificateStatus.SEPARATION]
    assert m.cross_check_cpu_cuda_exact([_moving_point(m, 1.0, -3.0), _moving_point(m, 2.0, 2.0, 11, 21)],
                                        [_moving_edge(m, 1.0, -3.0), _moving_edge(m, 2.0, 2.0, 31, 41)], 0.0, 1.0,
                                        _cfg(m), 1e-9)  # test_certificate_cuda.cpp:77-91
    bad = _moving_point(m, 1.0, -3.0)
    bad.point_id = -1
    with pytest.raises(ValueError, match="point-triangle primitive ids are required"):
        m.evaluate_point_triangle_interval(bad, 0.0, 1.0, _cfg(m))


def test_engine_and_work_queue_known_answers(cuda_device):
    """test_certificate_engine.cpp:161-287."""
    import p2cccd_cpp as m

    q1 = m.ExactCertificateQuery()
    q1.work_item, q1.config = _item(m, 1), _cfg(m)
    q1.point_triangle_primitives = [_moving_point(m, 1.0, -3.0)]
    c = m.evaluate_certificate_query_cpu(q1)
    assert c.status == m.CertificateStatus.COLLISION and abs(c.toi_upper - 0.25) <= 1e-12
    assert (c.witness_id_a, c.witness_id_b) == (10, 20) and c.next_refinement_mode == m.CertificateRefinementMode.NONE
    q2 = m.ExactCertificateQuery()
    q2.work_item, q2.config = _item(m, 3, 9002), _cfg(m)
    q2.point_triangle_primitives = [_moving_point(m, 2.0, 2.0)]
    q2.edge_edge_primitives = [_moving_edge(m, 2.0, 2.0)]
    c = m.CertificateEngine().evaluate_query(q2)
    assert c.status == m.CertificateStatus.SEPARATION and c.covered_feature_mask == 3 and c.safe_margin_lb > 1.9
    q3 = m.ExactCertificateQuery()
    q3.work_item, q3.config = _item(m, 1, 9003), _cfg(m)
    c = m.evaluate_certificate_query_cpu(q3)
    assert c.status == m.CertificateStatus.UNDECIDED and c.reason_code == m.CERTIFICATE_REASON_MISSING_GEOMETRY
    assert c.next_refinement_mode == m.CertificateRefinementMode.REQUEST_GEOMETRY
    qc = m.ExactWorkQueueConfig()
    qc.first_event_id, qc.first_timestamp_us = 500, 800
    sep = m.ExactCertificateQuery()
    sep.work_item, sep.config = _item(m, 2, 9002), _cfg(m)
    sep.edge_edge_primitives = [_moving_edge(m, 2.0, 2.0)]
    res = m.process_exact_work_queue_cpu([q1, sep, q3], qc)
    assert res.processed_count == 3 and len(res.certificates) == 3 and len(res.audit_log) == 6
    assert [c.status for c in res.certificates] == [0, 1, 2]
    assert res.certificates[2].next_refinement_mode == m.CertificateRefinementMode.REQUEST_GEOMETRY
    assert res.audit_log[0].action == m.EXACT_AUDIT_DEQUEUED and res.audit_log[1].action == m.EXACT_AUDIT_COLLISION
    assert res.audit_log[0].event_id == 500 and res.audit_log[-1].timestamp_us == 805
    assert m.validate_exact_work_queue_coverage([q1, sep, q3], res)
    incomplete = m.ExactWorkQueueResult()
    incomplete.processed_count = 1
    with pytest.raises(ValueError):
        m.validate_exact_work_queue_coverage([q1], incomplete)
    # an invalid primitive before any collision fails the query: InvalidInput
    bad = m.ExactCertificateQuery()
    bad.work_item, bad.config = _item(m, 1, 9004), _cfg(m)
    p = _moving_point(m, 2.0, 2.0)
    p.triangle_v1.position_t1 = [float("nan"), 0.0, 0.0]
    bad.point_triangle_primitives = [p, _moving_point(m, 1.0, -3.0)]
    res = m.process_exact_work_queue_cpu([bad], qc)
    assert res.certificates[0].reason_code == m.CERTIFICATE_REASON_INVALID_INPUT
    assert res.audit_log[1].action == m.EXACT_AUDIT_INVALID_INPUT
    with pytest.raises(ValueError, match="trajectories must be finite"):
        m.evaluate_certificate_query_cpu(bad)
    # ... but after the first collision it is never evaluated (early return)
    late = m.ExactCertificateQuery()
    late.work_item, late.config = _item(m, 1, 9005), _cfg(m)
    late.point_triangle_primitives = [_moving_point(m, 1.0, -3.0), p]
    assert m.evaluate_certificate_query_cpu(late).status == m.CertificateStatus.COLLISION


def test_work_queue_matches_oracle_aggregation(cuda_device, oracle_mod):
    import p2cccd_cpp as m
    from p2cccd_b200 import queue, workloads
    from p2cccd_b200.certify import CertConfig

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=800, n_ee=800, seed=13))
    rng = np.random.default_rng(2)
    nq = 300
    sizes_pt = rng.integers(0, 8, nq)
    sizes_ee = rng.integers(0, 8, nq)
    masks = rng.integers(1, 4, nq)
    sizes_pt[masks & 1 == 0] = 0
    sizes_ee[masks & 2 == 0] = 0
    t0 = rng.uniform(0, 0.5, nq)
    t1 = np.minimum(1.0, t0 + rng.uniform(0, 0.6, nq))
    pidx = rng.integers(0, 800, sizes_pt.sum())
    eidx = rng.integers(0, 800, sizes_ee.sum())
    pto = np.concatenate([[0], np.cumsum(sizes_pt)])
    eeo = np.concatenate([[0], np.cumsum(sizes_ee)])
    cfg = CertConfig(1e-5, 1e-6, 32)
    res = queue.certify_work_items(w["vf"][pidx], pto, w["ee"][eidx], eeo, t0, t1, masks.astype(np.uint32), cfg,
                                   cuda_device)
    for q in range(nq):
        a = w["vf"][pidx[pto[q]:pto[q + 1]]]
        b = w["ee"][eidx[eeo[q]:eeo[q + 1]]]
        ra, _, _ = oracle_mod.eval_batch(a, t0[q], t1[q], cfg.eps_time, cfg.eps_space, 32)
        rb, _, _ = oracle_mod.eval_batch(b, t0[q], t1[q], cfg.eps_time, cfg.eps_space, 32)
        exp = oracle_mod.aggregate(int(masks[q]), ra, rb, float(t1[q]))
        got = res["certs"][q]
        for k in ("status", "toi_upper", "safe_margin_lb", "witness_id_a", "witness_id_b", "reason_code",
                  "covered_feature_mask", "next_refinement_mode", "witness_index", "witness_family"):
            assert got[k] == exp[k], (q, k, got[k], exp[k])
        np.testing.assert_array_equal(res["pt_results"][pto[q]:pto[q + 1]].view(np.uint8), ra.view(np.uint8))
        np.testing.assert_array_equal(res["ee_results"][eeo[q]:eeo[q + 1]].view(np.uint8), rb.view(np.uint8))


def test_mesh_query_through_mirror_matches_reference_test(cuda_device):
    """test_mesh_exact_query.cpp:86-134."""
    import p2cccd_cpp as m

    mesh = m.Mesh()
    mesh.vertices_ref = [[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.0, 0.5, 0.0]]
    mesh.triangles = [[0, 1, 2]]
    item = _item(m, 3, 1)
    item.query_id = 11
    r = m.build_mesh_exact_certificate_query(mesh, [0, 0, 0], [0, 0, 0], mesh, [0, 0, 1], [0, 0, -1], item, _cfg(m),
                                             m.MeshExactBuildConfig())
    assert r.stats.point_triangle_kept_pairs > 0 and r.stats.edge_edge_kept_pairs > 0
    assert m.evaluate_certificate_query_cpu(r.query).status == m.CertificateStatus.COLLISION
    r = m.build_mesh_exact_certificate_query(mesh, [0, 0, 0], [0, 0, 0], mesh, [0, 0, 2], [0, 0, 2], item, _cfg(m),
                                             m.MeshExactBuildConfig())
    assert r.stats.point_triangle_kept_pairs == 0 and r.stats.edge_edge_kept_pairs == 0
    assert m.evaluate_certificate_query_cpu(r.query).status == m.CertificateStatus.UNDECIDED
    grid = m.Mesh()
    n = 8
    grid.vertices_ref = [[float(x), float(y), 0.0] for y in range(n + 1) for x in range(n + 1)]
    idx = lambda x, y: y * (n + 1) + x
    grid.triangles = [t for y in range(n) for x in range(n)
                      for t in ([idx(x, y), idx(x + 1, y), idx(x, y + 1)], [idx(x + 1, y), idx(x + 1, y + 1), idx(x, y + 1)])]
    bc = m.MeshExactBuildConfig()
    bc.prune_by_swept_aabb, bc.max_point_triangle_primitives = False, 64
    with pytest.raises(ValueError, match="point-triangle primitive budget exceeded"):
        m.build_mesh_exact_certificate_query(grid, [0, 0, 0], [0, 0, 0], grid, [0, 0, 0.1], [0, 0, 0.1], item,
                                             _cfg(m), bc)
