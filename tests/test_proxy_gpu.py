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
