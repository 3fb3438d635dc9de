"""CPU pins of the candidate-group path against the reference scene tool
(tools/scene_object_envelope_native_ti_walltime.cpp compiled unchanged, its
Tight-Inclusion calls answered by the reference certifier):

* the C restatement of the scheduled any-hit with fallback replay
  (oracle_group_anyhit + proposal lists by score) reproduces the tool's
  RunScheduledAnyHitRows counts exactly;
* the restated sort-and-sweep candidate sets equal the tool's
  BuildVFCandidates / BuildEECandidates sets.
"""
from __future__ import annotations

import numpy as np
import pytest

import anyhit_case as A


@pytest.fixture(scope="module")
def tool_ready(oracle_mod):
    if not oracle_mod.REF_TOOL_SO.exists():
        pytest.skip("reference scene tool library not built (reference sources absent)")
    return oracle_mod


SCENES = {
    "two_spheres": A.two_spheres_small,
    "cloth": A.cloth_small,
    "cluster5": lambda: A.sphere_cluster(7, 5),
    "cluster6": lambda: A.sphere_cluster(7, 6),
}


@pytest.mark.parametrize("scene", list(SCENES))
@pytest.mark.parametrize("kind", ["vf", "ee"])
@pytest.mark.parametrize("exclude_self", [False, True])
def test_oracle_anyhit_matches_reference_tool(tool_ready, scene, kind, exclude_self):
    s = SCENES[scene]()
    tool, cands, scores, groups, hit = A.tool_case(tool_ready, s, kind, 0.0, exclude_self)
    for g in np.unique(groups):  # distinct inside each group: the proposal order is unambiguous
        assert len(np.unique(scores[groups == g])) == int((groups == g).sum())
    n_groups = tool.n_obj ** 2
    for top_k in (0, 1, 2, 5, 4096):
        exp = A.expected(tool_ready, groups, hit, scores, n_groups, top_k)
        row = tool.anyhit(kind, top_k, A.CFG["eps_time"], A.CFG["eps_space"], A.CFG["max_depth"])
        for field, value in exp["row"].items():
            assert value == row[field], (scene, kind, top_k, field, value, row[field])
        # detection equals the every-candidate truth: any-hit is exhaustive
        assert int(exp["detected"].sum()) == row["all_positive_groups"] == row["tp"]
        assert row["fn"] == 0 and row["fp"] == 0


def _keys(pairs: np.ndarray) -> np.ndarray:
    return np.sort((pairs[:, 0].astype(np.uint64) << np.uint64(32)) | pairs[:, 1].astype(np.uint64))


@pytest.mark.parametrize("scene", list(SCENES))
@pytest.mark.parametrize("exclude_self,thickness", [(False, 0.0), (True, 0.0), (False, 2e-3)])
def test_tool_candidate_sets_equal_oracle_sweep(tool_ready, scene, exclude_self, thickness):
    o = tool_ready
    s = SCENES[scene]()
    tool = o.RefToolScene(s["v_t0"], s["v_t1"], s["faces"], thickness, exclude_self)
    allowed = o.object_allowed(s["v_t0"], s["v_t1"], tool.v_obj, tool.n_obj, thickness, exclude_self)
    vbox = o.swept_boxes(s["v_t0"], s["v_t1"], None, 1, thickness)
    fbox = o.swept_boxes(s["v_t0"], s["v_t1"], s["faces"], 3, thickness)
    ebox = o.swept_boxes(s["v_t0"], s["v_t1"], tool.edges, 2, thickness)
    valid = (tool.v_obj >= 0).astype(np.uint8)
    vf = o.vf_pairs(vbox, tool.v_obj, valid, fbox, tool.f_obj, s["faces"], allowed, "sweep")
    ee = o.ee_pairs(ebox, tool.e_obj, tool.edges, allowed, "sweep")
    assert np.array_equal(np.sort(vf), _keys(tool.candidates("vf")))
    assert np.array_equal(np.sort(ee), _keys(tool.candidates("ee")))
