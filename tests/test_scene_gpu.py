"""GPU parity of the scene path: candidate pair sets equal the CPU oracle's
(brute force and sort-and-sweep) and the reference's own
BuildMeshExactCertificateQuery; every candidate certificate equals the
oracle's byte for byte; the aggregate equals CertificateEngine::Evaluate."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grid_pair(seed=0, n=6):
    rng = np.random.default_rng(seed)
    va = rng.uniform(-1, 1, size=(n * n, 3))
    va[:, 2] *= 0.1
    faces = []
    for y in range(n - 1):
        for x in range(n - 1):
            i = y * n + x
            faces += [(i, i + 1, i + n), (i + 1, i + n + 1, i + n)]
    f = np.array(faces, dtype=np.int32)
    vb = rng.uniform(-1, 1, size=(n * n, 3))
    vb[:, 2] *= 0.1
    return va, f, vb, f.copy()


def _mesh_pair_scene(va, fa, ta0, ta1, vb, fb, tb0, tb1):
    from p2cccd_b200 import scenes

    ea, eb = scenes.unique_edges(fa), scenes.unique_edges(fb)
    return scenes.combine([(va + ta0, va + ta1, fa, ea), (vb + tb0, vb + tb1, fb, eb)])


def _oracle_pairs(oracle_mod, s, thickness, exclude_self, method="brute"):
    allowed = oracle_mod.object_allowed(s["v_t0"], s["v_t1"], s["v_obj"], s["n_obj"], thickness, exclude_self)
    vbox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], None, 1, thickness)
    fbox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], s["faces"], 3, thickness)
    ebox = oracle_mod.swept_boxes(s["v_t0"], s["v_t1"], s["edges"], 2, thickness)
    valid = (s["v_obj"] >= 0).astype(np.uint8)
    vf = oracle_mod.vf_pairs(vbox, s["v_obj"], valid, fbox, s["f_obj"], s["faces"], allowed, method)
    ee = oracle_mod.ee_pairs(ebox, s["e_obj"], s["edges"], allowed, method)
    return np.sort(vf), np.sort(ee)


def _bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1, 72)


def _check_results(oracle_mod, pipe, cfg):
    vf_rec, ee_rec = pipe.materialize()
    vf_res, ee_res = pipe.results()
    for rec, res in ((vf_rec, vf_res), (ee_rec, ee_res)):
        if len(rec) == 0:
            continue
        cpu, st, _ = oracle_mod.eval_batch(rec, pipe.interval[0], pipe.interval[1], cfg.eps_time, cfg.eps_space,
                                           cfg.max_subdivision_depth)
        assert st.sum() == 0
        bad = np.nonzero((_bytes(cpu) != _bytes(res)).any(axis=1))[0]
        assert bad.size == 0, f"{bad.size} certificates differ, first {bad[0]}: {res[bad[0]]} vs {cpu[bad[0]]}"
    return vf_rec, ee_rec, vf_res, ee_res


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_mesh_pair_candidates_equal_reference_mesh_query(cuda_device, oracle_mod, seed):
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    va, fa, vb, fb = _grid_pair(seed)
    ta0, ta1 = np.zeros(3), np.array([0.0, 0.0, 0.05])
    tb0, tb1 = np.array([0.1, 0.0, 0.3]), np.array([0.0, 0.1, -0.2])
    s = _mesh_pair_scene(va, fa, ta0, ta1, vb, fb, tb0, tb1)
    cfg = CertConfig(1e-5, 1e-6, 32)
    pipe = ScenePipeline(s, cuda_device, exclude_self=True, config=cfg, vf_capacity=64, ee_capacity=64)
    summ = pipe.step_checked()
    vf, ee = pipe.pairs()
    o_vf, o_ee = _oracle_pairs(oracle_mod, s, 0.0, True)
    np.testing.assert_array_equal(vf, o_vf)  # sorted ascending on the device
    np.testing.assert_array_equal(ee, o_ee)
    vf_rec, ee_rec, vf_res, ee_res = _check_results(oracle_mod, pipe, cfg)
    agg = oracle_mod.aggregate(3, vf_res, ee_res)
    for k in ("status", "toi_upper", "safe_margin_lb", "witness_id_a", "witness_id_b", "reason_code",
              "covered_feature_mask", "next_refinement_mode", "witness_index"):
        assert summ["query"][k] == agg[k], k
    if oracle_mod.ref_available():
        pts, ees = oracle_mod.ref_build_mesh_query(va, fa, ta0, ta1, vb, fb, tb0, tb1)
        np.testing.assert_array_equal(vf_rec["point_id"], pts["point_id"])
        np.testing.assert_array_equal(vf_rec["triangle_id"], pts["triangle_id"])
        np.testing.assert_array_equal(ee_rec["edge_a_id"], ees["edge_a_id"])
        np.testing.assert_array_equal(ee_rec["edge_b_id"], ees["edge_b_id"])
        for k in ("point", "triangle_v0", "triangle_v1", "triangle_v2"):
            np.testing.assert_array_equal(vf_rec[k]["position_t0"], pts[k]["position_t0"])
            np.testing.assert_array_equal(vf_rec[k]["position_t1"], pts[k]["position_t1"])
        q = oracle_mod.ref_evaluate_query(3, pts, ees, 0.0, 1.0, cfg.eps_time, cfg.eps_space, 32)
        assert summ["query"]["status"] == q["status"] and summ["query"]["toi_upper"] == q["toi_upper"]
        assert summ["query"]["witness_id_a"] == q["witness_id_a"]


@pytest.mark.parametrize("thickness", [0.0, 2e-3])
def test_self_pairs_with_adjacency_exclusion(cuda_device, oracle_mod, thickness):
    from p2cccd_b200 import scenes
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    rng = np.random.default_rng(11)
    va, fa, vb, fb = _grid_pair(5, n=9)
    s = _mesh_pair_scene(va, fa, 0.0, 0.0, vb, fb, 0.0, 0.0)
    s["v_t1"] = s["v_t1"] + rng.normal(0, 0.05, s["v_t1"].shape)
    # an isolated vertex (in no face) is never a candidate
    s["v_t0"] = np.concatenate([s["v_t0"], [[0.0, 0.0, 0.0]]])
    s["v_t1"] = np.concatenate([s["v_t1"], [[0.0, 0.0, 0.0]]])
    s["v_obj"] = np.concatenate([s["v_obj"], [-1]]).astype(np.int32)
    cfg = CertConfig(1e-4, 1e-6, 32)
    pipe = ScenePipeline(s, cuda_device, exclude_self=False, thickness=thickness, config=cfg, vf_capacity=16,
                         ee_capacity=16)
    pipe.step_checked()
    vf, ee = pipe.pairs()
    o_vf, o_ee = _oracle_pairs(oracle_mod, s, thickness, False, "brute")
    s_vf, s_ee = _oracle_pairs(oracle_mod, s, thickness, False, "sweep")
    np.testing.assert_array_equal(o_vf, s_vf)
    np.testing.assert_array_equal(vf, o_vf)
    np.testing.assert_array_equal(ee, o_ee)
    assert len(vf) > 0 and len(ee) > 0
    _check_results(oracle_mod, pipe, cfg)


def test_uv_spheres_small(cuda_device, oracle_mod):
    from p2cccd_b200 import scenes
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    s = scenes.two_spheres(n_lon=40, n_rings=30, gap=0.1, approach=0.3, seed=3)
    cfg = CertConfig(1e-6, 1e-6, 32)
    pipe = ScenePipeline(s, cuda_device, exclude_self=True, config=cfg)
    summ = pipe.step_checked()
    vf, ee = pipe.pairs()
    o_vf, o_ee = _oracle_pairs(oracle_mod, s, 0.0, True, "sweep")
    np.testing.assert_array_equal(vf, o_vf)
    np.testing.assert_array_equal(ee, o_ee)
    _, _, vf_res, ee_res = _check_results(oracle_mod, pipe, cfg)
    assert summ["vf_certified"] == len(vf) and summ["ee_certified"] == len(ee)
    assert summ["collisions"] == int((vf_res["status"] == 0).sum() + (ee_res["status"] == 0).sum())
    assert summ["query"]["status"] == 0  # the spheres meet during the step


def test_config2_scene_full_size(cuda_device, oracle_mod):
    """The bench scene (two 40,960-triangle spheres): pair sets equal the
    oracle sweep and every certificate equals the oracle's."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    s = scenes.two_spheres()
    cfg = CertConfig(1e-6, 1e-6, 32)
    pipe = ScenePipeline(s, cuda_device, exclude_self=True, config=cfg, vf_capacity=1 << 12, ee_capacity=1 << 12)
    pipe.step_checked()
    vf, ee = pipe.pairs()
    o_vf, o_ee = _oracle_pairs(oracle_mod, s, 0.0, True, "sweep")
    np.testing.assert_array_equal(vf, o_vf)
    np.testing.assert_array_equal(ee, o_ee)
    _check_results(oracle_mod, pipe, cfg)


@pytest.mark.parametrize("n_lon,n_rings", [(40, 30), (160, 128)])
def test_two_body_scene_with_the_counted_sort(cuda_device, oracle_mod, monkeypatch, n_lon, n_rings):
    """P2C_COUNT_SORT_MIN_PRIMS=0 ranks the kept boxes of any culled scene with
    the sort whose count is read on the device (by default only scenes above
    2^20 primitives): pair sets and certificates still equal the oracle's."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    monkeypatch.setenv("P2C_COUNT_SORT_MIN_PRIMS", "0")
    s = scenes.two_spheres(n_lon=n_lon, n_rings=n_rings, seed=5)
    cfg = CertConfig(1e-6, 1e-6, 32)
    pipe = ScenePipeline(s, cuda_device, exclude_self=True, config=cfg)
    pipe.step_checked()
    vf, ee = pipe.pairs()
    o_vf, o_ee = _oracle_pairs(oracle_mod, s, 0.0, True, "sweep")
    np.testing.assert_array_equal(vf, o_vf)
    np.testing.assert_array_equal(ee, o_ee)
    assert len(vf) > 0 and len(ee) > 0
    _check_results(oracle_mod, pipe, cfg)


def test_undecided_queue_and_invalid_geometry(cuda_device, oracle_mod):
    from p2cccd_b200 import scenes
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    s = scenes.two_spheres(n_lon=40, n_rings=30, gap=0.05, approach=0.2, seed=4)
    cfg = CertConfig(1e-2, 1e-6, 4)  # coarse: many undecided certificates
    pipe = ScenePipeline(s, cuda_device, exclude_self=True, config=cfg)
    summ = pipe.step_checked()
    vf_res, ee_res = pipe.results()
    expect = sorted([int(i) for i in np.nonzero(vf_res["status"] == 2)[0]] +
                    [(1 << 63) | int(i) for i in np.nonzero(ee_res["status"] == 2)[0]])
    assert summ["undecided"] == len(expect) > 0
    np.testing.assert_array_equal(np.sort(pipe.undecided_entries), np.array(expect, dtype=np.uint64))
    # a queue too small for the step: entries dropped, flagged, and the
    # checked step re-runs with a larger queue
    from p2cccd_b200.scene import ERR_UNDECIDED_FULL, UndecidedOverflow

    tiny = ScenePipeline(s, cuda_device, exclude_self=True, config=cfg, undecided_capacity=4)
    tiny.step()
    raw = tiny.read_summary()
    assert raw["undecided_queued"] == len(expect) and raw["error_word"] & ERR_UNDECIDED_FULL
    with pytest.raises(UndecidedOverflow):
        tiny.undecided_entries
    again = tiny.step_checked()
    assert again == summ and tiny.undecided_capacity >= len(expect)
    np.testing.assert_array_equal(np.sort(tiny.undecided_entries), np.array(expect, dtype=np.uint64))
    bad = dict(s)
    bad["v_t1"] = s["v_t1"].copy()
    bad["v_t1"][5, 1] = np.nan
    pipe2 = ScenePipeline(bad, cuda_device, exclude_self=True, config=cfg)
    with pytest.raises(ValueError, match="finite"):
        pipe2.step_checked()


@pytest.mark.parametrize("self_pairs", [False, True])
def test_small_pair_buffers_sort_like_large_ones(cuda_device, self_pairs):
    """Pair buffers of at most 8,192 entries take the one-launch block sort;
    the lists, padding, summary and certificates equal the device-wide sort's."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline

    s = (scenes.cloth_on_sphere(n=17, sphere_lon=24, sphere_rings=16, gap=1e-3, drop=0.05) if self_pairs
         else scenes.two_spheres(n_lon=40, n_rings=30))
    cfg = CertConfig(1e-6, 1e-6, 32)
    big = ScenePipeline(s, cuda_device, exclude_self=not self_pairs, config=cfg)
    sb = big.step_checked()
    small = ScenePipeline(s, cuda_device, exclude_self=not self_pairs, config=cfg)
    small.step_checked()
    small.fit_capacities(margin=1.0, slack=7)
    assert small.vf_cap <= 8192 and small.ee_cap <= 8192 and big.vf_cap > 8192
    ss = small.step_checked()
    assert ss == sb
    for a, b in zip(small.pairs(), big.pairs()):
        assert np.array_equal(a, b)
    for a, b in zip(small.results(), big.results()):
        assert np.array_equal(_bytes(a), _bytes(b))
    tail = small.vf_pairs[len(small.pairs()[0]):small.vf_cap].cpu().numpy().view(np.uint64)
    assert len(tail) == 7 and (tail == np.uint64(0xFFFFFFFFFFFFFFFF)).all()
