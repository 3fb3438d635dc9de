"""Pins the CPU oracle: the reference's own known answers, the golden fixtures
made from the reference, and byte equality with the reference sources
compiled unchanged (oracle/_ref)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "plain_sample.npz"


def _golden():
    return np.load(GOLDEN)


def _rec(raw, dtype):
    return np.ascontiguousarray(raw).view(dtype).reshape(-1)


# ---- known answers of the reference tests (test_certificate_engine.cpp) ----

def test_known_answer_point_triangle(oracle_mod):
    g = _golden()
    pt = _rec(g["ka_pt"], oracle_mod.PT)
    res, st, _ = oracle_mod.eval_batch(pt, 0.0, 1.0, 1e-5, 1e-6, 32)
    assert st.sum() == 0
    # :97-112 collision with toi 0.25 and witness (10, 20)
    assert res[0]["status"] == 0
    assert abs(res[0]["toi_upper"] - 0.25) <= 1e-12
    assert res[0]["witness_family"] == 1 and res[0]["witness_id_a"] == 10 and res[0]["witness_id_b"] == 20
    # :114-127 separation, mask = point-triangle, margin > 1.9
    assert res[1]["status"] == 1 and res[1]["covered_feature_mask"] == 1 and res[1]["safe_margin_lb"] > 1.9


def test_known_answer_edge_edge(oracle_mod):
    g = _golden()
    ee = _rec(g["ka_ee"], oracle_mod.EE)
    res, st, _ = oracle_mod.eval_batch(ee, 0.0, 1.0, 1e-5, 1e-6, 32)
    assert st.sum() == 0
    assert res[0]["status"] == 0 and abs(res[0]["toi_upper"] - 0.25) <= 1e-12
    assert res[0]["witness_family"] == 2 and res[0]["witness_id_a"] == 30 and res[0]["witness_id_b"] == 40
    assert res[1]["status"] == 1 and res[1]["covered_feature_mask"] == 2 and res[1]["safe_margin_lb"] > 1.9


def test_known_answer_aggregation(oracle_mod):
    g = _golden()
    pt = _rec(g["ka_pt"], oracle_mod.PT)
    ee = _rec(g["ka_ee"], oracle_mod.EE)
    rpt, _, _ = oracle_mod.eval_batch(pt, 0.0, 1.0, 1e-5, 1e-6, 32)
    ree, _, _ = oracle_mod.eval_batch(ee, 0.0, 1.0, 1e-5, 1e-6, 32)
    # :161-181 collision output
    c = oracle_mod.aggregate(1, rpt[:1], ree[:0])
    assert c["status"] == 0 and abs(c["toi_upper"] - 0.25) <= 1e-12 and c["next_refinement_mode"] == 0
    assert c["witness_id_a"] == 10 and c["witness_id_b"] == 20
    # :183-202 separation over both families, mask 3
    s = oracle_mod.aggregate(3, rpt[1:], ree[1:])
    assert s["status"] == 1 and s["covered_feature_mask"] == 3 and s["safe_margin_lb"] > 1.9
    # :204-217 undecided: family requested, no geometry
    u = oracle_mod.aggregate(1, rpt[:0], ree[:0])
    assert u["status"] == 2 and u["reason_code"] == 1 and u["next_refinement_mode"] == 2


def test_known_answer_refinement(oracle_mod):
    # :289-337
    assert oracle_mod.refinement_children(0.0, 1.0, 0, 0, 0, 0.25, 64, 1e-5) == [(0.0, 0.25)]
    assert oracle_mod.refinement_children(0.0, 1.0, 0, 2, 1, 1.0, 64, 1e-5) == [(0.0, 0.5), (0.5, 1.0)]
    assert oracle_mod.refinement_children(0.0, 1.0, 64, 2, 1, 1.0, 64, 1e-5) == []
    assert oracle_mod.refinement_children(0.0, 1e-6, 0, 2, 1, 1.0, 64, 1e-5) == []


# ---- golden fixtures produced by the reference ------------------------------

@pytest.mark.parametrize("tag,cfg", [("c6", (1e-6, 1e-6, 32)), ("cdef", (1e-4, 1e-6, 32))])
@pytest.mark.parametrize("fam", ["vf", "ee"])
def test_oracle_matches_golden(oracle_mod, tag, cfg, fam):
    g = _golden()
    dt = oracle_mod.PT if fam == "vf" else oracle_mod.EE
    rec = _rec(g[fam], dt)
    res, st, _ = oracle_mod.eval_batch(rec, 0.0, 1.0, *cfg)
    assert st.sum() == 0
    np.testing.assert_array_equal(res.view(np.uint8).reshape(-1, 72), g[f"{fam}_{tag}"])


# ---- byte equality with the reference compiled unchanged --------------------

needs_ref = pytest.mark.skipif(
    not __import__("oracle").ref_available(), reason="oracle/_ref not built (reference sources absent)")


@needs_ref
@pytest.mark.parametrize("cfg", [(1e-6, 1e-6, 32), (1e-4, 1e-6, 32), (1e-5, 1e-6, 8), (1e-3, 1e-4, 64)])
def test_oracle_equals_reference_plain_workload(oracle_mod, cfg):
    from p2cccd_b200 import workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=4000, n_ee=4000, seed=11))
    for fam in ("vf", "ee"):
        o, os_, _ = oracle_mod.eval_batch(w[fam], 0.0, 1.0, *cfg)
        r, rs = oracle_mod.ref_eval_batch(w[fam], 0.0, 1.0, *cfg)
        assert os_.sum() == 0 and rs.sum() == 0
        np.testing.assert_array_equal(o.view(np.uint8), r.view(np.uint8))


@needs_ref
@pytest.mark.parametrize("interval", [(0.25, 0.75), (0.3, 0.7), (0.0, 0.0), (1.0, 1.0), (0.1, 0.1000001)])
def test_oracle_equals_reference_subintervals(oracle_mod, interval):
    from p2cccd_b200 import workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=1000, n_ee=1000, seed=5))
    for fam in ("vf", "ee"):
        o, _, _ = oracle_mod.eval_batch(w[fam], interval[0], interval[1], 1e-6, 1e-6, 32)
        r, _ = oracle_mod.ref_eval_batch(w[fam], interval[0], interval[1], 1e-6, 1e-6, 32)
        np.testing.assert_array_equal(o.view(np.uint8), r.view(np.uint8))


@needs_ref
def test_oracle_error_messages_match_reference(oracle_mod):
    g = _golden()
    pt = _rec(g["ka_pt"], oracle_mod.PT).copy()
    bad_id = pt[:1].copy()
    bad_id["point_id"] = -1
    bad_nan = pt[:1].copy()
    bad_nan["triangle_v1"]["position_t1"][0, 2] = np.nan
    cases = [(bad_id, 0.0, 1.0, 1e-5, 1e-6), (bad_nan, 0.0, 1.0, 1e-5, 1e-6), (pt[:1], 0.0, 1.0, 0.0, 1e-6),
             (pt[:1], 0.0, 1.0, 1e-5, -1.0), (pt[:1], 0.5, 0.25, 1e-5, 1e-6), (pt[:1], 0.0, 1.5, 1e-5, 1e-6),
             (pt[:1], np.inf, 1.0, 1e-5, 1e-6)]
    for rec, t0, t1, et, es in cases:
        msg = oracle_mod.ref_eval_error(rec, t0, t1, et, es, 32)
        assert msg is not None
        _, st, _ = oracle_mod.eval_batch(rec, t0, t1, et, es, 32)
        assert st[0] == 1


@needs_ref
def test_oracle_aggregation_equals_reference(oracle_mod):
    from p2cccd_b200 import workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=600, n_ee=600, seed=3))
    rng = np.random.default_rng(0)
    for trial in range(40):
        a = rng.integers(0, 600, size=rng.integers(0, 12))
        b = rng.integers(0, 600, size=rng.integers(0, 12))
        mask = int(rng.integers(1, 4))
        pts, ees = w["vf"][a], w["ee"][b]
        rpt, _, _ = oracle_mod.eval_batch(pts, 0.0, 1.0, 1e-4, 1e-6, 32)
        ree, _, _ = oracle_mod.eval_batch(ees, 0.0, 1.0, 1e-4, 1e-6, 32)
        mine = oracle_mod.aggregate(mask, rpt, ree)
        theirs = oracle_mod.ref_evaluate_query(mask, pts, ees, 0.0, 1.0, 1e-4, 1e-6, 32)
        for f in ("status", "witness_family", "reason_code", "covered_feature_mask", "toi_upper",
                  "safe_margin_lb", "witness_id_a", "witness_id_b", "next_refinement_mode"):
            assert mine[f] == theirs[f], (trial, f)


@needs_ref
def test_oracle_refinement_equals_reference(oracle_mod):
    rng = np.random.default_rng(1)
    for _ in range(300):
        t0 = float(rng.uniform(0, 0.5))
        t1 = float(rng.uniform(t0, 1.0))
        st = int(rng.integers(0, 3))
        mode = int(rng.integers(0, 4)) if st == 2 else 0
        toi = float(rng.uniform(-0.2, 1.2)) if st == 0 else t1
        depth = int(rng.integers(0, 5))
        mw = float(10 ** rng.uniform(-6, -0.5))
        if st == 0:
            toi = float(np.clip(toi, t0, t1))
        a = oracle_mod.refinement_children(t0, t1, depth, st, mode, toi, 3, mw)
        b = oracle_mod.refinement_children(t0, t1, depth, st, mode, toi, 3, mw, use_ref=True)
        assert a == b


# ---- broad-phase oracle: sweep == brute force == the reference mesh query ---

def _two_meshes(seed=0, n=5, dz=(1.0, -1.0)):
    rng = np.random.default_rng(seed)
    va = rng.uniform(-1, 1, size=(n * n, 3))
    va[:, 2] *= 0.1
    faces = []
    for y in range(n - 1):
        for x in range(n - 1):
            i = y * n + x
            faces += [(i, i + 1, i + n), (i + 1, i + n + 1, i + n)]
    fa = np.array(faces, dtype=np.uint32)
    vb = rng.uniform(-1, 1, size=(n * n, 3))
    vb[:, 2] *= 0.1
    return va, fa, vb, fa.copy()


def _unique_edges(faces):
    e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
    e = np.sort(e, axis=1)
    return np.unique(e, axis=0)


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_pair_oracle_equals_reference_mesh_query(oracle_mod, seed):
    va, fa, vb, fb = _two_meshes(seed)
    ta0, ta1 = np.zeros(3), np.array([0.0, 0.0, 0.05])
    tb0, tb1 = np.array([0.1, 0.0, 0.3]), np.array([0.0, 0.1, -0.2])
    pts, ees = oracle_mod.ref_build_mesh_query(va, fa, ta0, ta1, vb, fb, tb0, tb1)
    # the same pairs as a two-object scene with self pairs excluded
    v_t0 = np.concatenate([va + ta0, vb + tb0])
    v_t1 = np.concatenate([va + ta1, vb + tb1])
    faces = np.concatenate([fa, fb + len(va)]).astype(np.int32)
    ea, eb = _unique_edges(fa), _unique_edges(fb)
    edges = np.concatenate([ea, eb + len(va)]).astype(np.int32)
    v_obj = np.repeat([0, 1], [len(va), len(vb)]).astype(np.int32)
    f_obj = np.repeat([0, 1], [len(fa), len(fb)]).astype(np.int32)
    e_obj = np.repeat([0, 1], [len(ea), len(eb)]).astype(np.int32)
    allowed = oracle_mod.object_allowed(v_t0, v_t1, v_obj, 2, 0.0, exclude_self=True)
    vbox = oracle_mod.swept_boxes(v_t0, v_t1, None, 1)
    fbox = oracle_mod.swept_boxes(v_t0, v_t1, faces, 3)
    ebox = oracle_mod.swept_boxes(v_t0, v_t1, edges, 2)
    for method in ("sweep", "brute"):
        vf = np.sort(oracle_mod.vf_pairs(vbox, v_obj, None, fbox, f_obj, faces, allowed, method))
        ee = np.sort(oracle_mod.ee_pairs(ebox, e_obj, edges, allowed, method))
        ref_vf = np.sort((pts["point_id"].astype(np.uint64) << np.uint64(32)) |
                         pts["triangle_id"].astype(np.uint64))
        ref_ee = np.sort((ees["edge_a_id"].astype(np.uint64) << np.uint64(32)) |
                         ees["edge_b_id"].astype(np.uint64))
        np.testing.assert_array_equal(vf, ref_vf)
        np.testing.assert_array_equal(ee, ref_ee)


def test_pair_sweep_equals_brute_with_self_pairs(oracle_mod):
    rng = np.random.default_rng(4)
    va, fa, vb, fb = _two_meshes(7, n=8)
    v_t0 = np.concatenate([va, vb])
    v_t1 = v_t0 + rng.normal(0, 0.05, size=v_t0.shape)
    faces = np.concatenate([fa, fb + len(va)]).astype(np.int32)
    edges = _unique_edges(faces).astype(np.int32)
    v_obj = np.repeat([0, 1], [len(va), len(vb)]).astype(np.int32)
    f_obj = v_obj[faces[:, 0]]
    e_obj = v_obj[edges[:, 0]]
    allowed = oracle_mod.object_allowed(v_t0, v_t1, v_obj, 2, 1e-3, exclude_self=False)
    vbox = oracle_mod.swept_boxes(v_t0, v_t1, None, 1, 1e-3)
    fbox = oracle_mod.swept_boxes(v_t0, v_t1, faces, 3, 1e-3)
    ebox = oracle_mod.swept_boxes(v_t0, v_t1, edges, 2, 1e-3)
    a = np.sort(oracle_mod.vf_pairs(vbox, v_obj, None, fbox, f_obj, faces, allowed, "sweep"))
    b = np.sort(oracle_mod.vf_pairs(vbox, v_obj, None, fbox, f_obj, faces, allowed, "brute"))
    np.testing.assert_array_equal(a, b)
    c = np.sort(oracle_mod.ee_pairs(ebox, e_obj, edges, allowed, "sweep"))
    d = np.sort(oracle_mod.ee_pairs(ebox, e_obj, edges, allowed, "brute"))
    np.testing.assert_array_equal(c, d)
    assert len(a) > 0 and len(c) > 0


def test_group_anyhit_oracle_small_case(oracle_mod):
    # 2 groups; group 0's top-2 misses, fallback finds the hit at candidate 4
    cand_group = np.array([0, 0, 1, 1, 0, 0])
    cand_hit = np.array([0, 0, 1, 0, 1, 1])
    top_offsets = np.array([0, 2, 4])
    top_index = np.array([1, 0, 3, 2])
    det, pc, fc, ev = oracle_mod.group_anyhit(cand_group, cand_hit, 2, top_offsets, top_index)
    assert det.tolist() == [1, 1]
    assert pc.tolist() == [2, 2] and fc.tolist() == [1, 0]
    assert ev.tolist() == [1, 1, 1, 1, 1, 0]
