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
