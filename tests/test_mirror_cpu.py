"""The p2cccd_cpp mirror exposes the reference module surface for this path
(names, defaults, enums, validators) without a GPU."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

import os

# the reference checkout (absent on the GPU box: the test is skipped there)
REF_PY = Path(os.environ.get("P2C_REFERENCE_ROOT", "/root/reference")) / "src" / "python"


def test_entry_points_and_defaults():
    import p2cccd_cpp as m

    for name in ("is_cuda_exact_built", "cuda_binding_status", "evaluate_point_triangle_batch_cuda",
                 "evaluate_edge_edge_batch_cuda", "cross_check_cpu_cuda_exact", "evaluate_point_triangle_interval",
                 "evaluate_edge_edge_interval", "evaluate_certificate_query_cpu", "process_exact_work_queue_cpu",
                 "validate_exact_work_queue_coverage", "generate_conservative_refinement_work_items",
                 "build_mesh_exact_certificate_query", "validate_certificate_result", "validate_exact_work_item",
                 "validate_audit_log_rows", "audit_log_rows_for_query"):
        assert callable(getattr(m, name)), name
    for cls in ("LinearVertexTrajectory", "PointTriangleIntervalPrimitive", "EdgeEdgeIntervalPrimitive",
                "CertificateEngineConfig", "ExactCertificateQuery", "PrimitiveIntervalResult"):
        assert hasattr(m, cls), cls
    c = m.CertificateEngineConfig()
    assert (c.eps_time, c.eps_space, c.max_subdivision_depth) == (1e-4, 1e-6, 32)  # certificate_engine.h:56-60
    assert m.CertificateStatus.Collision == m.CertificateStatus.COLLISION == 0
    t = m.LinearVertexTrajectory()
    assert t.feature_id == -1 and t.position_t0 == [0.0, 0.0, 0.0]
    with pytest.raises(TypeError):
        t.position_t0 = [1.0, 2.0]
    st = m.cuda_binding_status()
    assert st["cuda_exact_built"] and st["host_batch_exact_api"] and st["device_pointer_abi"]


def test_validators_raise_value_error_like_the_reference():
    import p2cccd_cpp as m

    item = m.ExactWorkItem()
    with pytest.raises(ValueError, match="ExactWorkItem.work_item_id is required"):
        m.validate_exact_work_item(item)
    item.work_item_id, item.parent_candidate_id, item.query_id, item.feature_family_mask = 1, 1, 1, 1
    assert m.validate_exact_work_item(item)
    item.interval_t1 = 2.0
    with pytest.raises(ValueError, match="interval must satisfy"):
        m.validate_exact_work_item(item)
    res = m.CertificateResult()
    res.work_item_id = res.query_id = 1
    with pytest.raises(ValueError, match="reason_code is required"):
        m.validate_certificate_result(res)


def test_refinement_children_match_reference_test():
    """test_certificate_engine.cpp:289-337, through the mirror (host logic)."""
    import p2cccd_cpp as m

    parent = m.ExactWorkItem()
    parent.work_item_id, parent.parent_candidate_id, parent.query_id = 9001, 77, 1234
    parent.feature_family_mask, parent.priority_score = 1, 1.0
    coll = m.CertificateResult()
    coll.work_item_id, coll.query_id, coll.status, coll.toi_upper = 9001, 1234, m.CertificateStatus.COLLISION, 0.25
    coll.witness_family, coll.witness_id_a, coll.witness_id_b = 1, 10, 20
    cfg = m.ExactRefinementConfig()
    cfg.first_child_work_item_id, cfg.min_interval_width = 10001, 1e-5
    kids = m.generate_conservative_refinement_work_items(parent, coll, cfg)
    assert len(kids) == 1 and kids[0].interval_t0 == 0.0 and kids[0].interval_t1 == 0.25
    assert kids[0].source == m.ProposalSource.REFINED
    und = m.CertificateResult()
    und.work_item_id, und.query_id, und.status = 9001, 1234, m.CertificateStatus.UNDECIDED
    und.reason_code, und.next_refinement_mode = 2, m.CertificateRefinementMode.BISECT_INTERVAL
    kids = m.generate_conservative_refinement_work_items(parent, und, cfg)
    assert [(k.interval_t0, k.interval_t1) for k in kids] == [(0.0, 0.5), (0.5, 1.0)]


@pytest.mark.skipif(not REF_PY.exists(), reason="reference checkout absent")
def test_reference_cuda_bindings_accept_the_mirror():
    """The reference's own p2cccd.cuda_bindings (read in place) sees a built,
    ready CUDA backend in this module."""
    sys.path.insert(0, str(REF_PY))
    try:
        import importlib

        cb = importlib.import_module("p2cccd.cuda_bindings")
        import p2cccd_cpp

        status = cb.get_cuda_binding_status(p2cccd_cpp)
        assert status.ready_for_cuda_execution and status.cuda_exact_built and status.device_pointer_abi
        assert status.backend_name == "b200_sm100a"
    finally:
        sys.path.remove(str(REF_PY))
        for k in [k for k in sys.modules if k == "p2cccd" or k.startswith("p2cccd.")]:
            del sys.modules[k]
