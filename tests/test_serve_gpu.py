"""GPU tests of the continuous-batching server (the native p2c_serve_* runtime
through its C ABI): every request's answer in the served mix equals the same
step run alone through the single-scene pipeline (itself pinned to the
oracle and the reference tool), in both modes - certificates of every
candidate, and the scheduled any-hit with fallback replay; requests admitted
by slots and arena memory overlap; overflowing buffers are re-run to
completion; a request that can never fit the arena fails alone."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1, 72)


def _meshes():
    from p2cccd_b200 import scenes

    import anyhit_case as A

    out = {
        "spheres": (scenes.two_spheres(n_lon=40, n_rings=30), True),
        "cloth": (scenes.cloth_on_sphere(n=33, sphere_lon=40, sphere_rings=30, gap=1e-3, drop=0.05), False),
        "cluster": (A.sphere_cluster(7, 5), False),
    }
    for i, s in enumerate(scenes.uneven_batch(3, tri_min=2000, tri_max=20000, seed=11)):
        out[f"batch{i}"] = (s, True)
    return out


def _requests(meshes, n, rng, keep=True, seed_base=0):
    from p2cccd_b200.serve import Request

    reqs, t = [], 0.0
    keys = list(meshes)
    for i in range(n):
        key = keys[int(rng.integers(len(keys)))]
        s, _ = meshes[key]
        jit = rng.normal(0.0, 1e-4, s["v_t1"].shape) if i else 0.0
        t += float(rng.exponential(2e-4))
        reqs.append(Request(rid=i, mesh=key, v_t0=torch.from_numpy(np.ascontiguousarray(s["v_t0"])).pin_memory(),
                            v_t1=torch.from_numpy(np.ascontiguousarray(s["v_t1"] + jit)).pin_memory(),
                            arrival_s=t, keep_results=keep, seed=seed_base + 13 * i))
    return reqs


def _alone(r, meshes, dev, cfg, narrow, top_k=4096):
    from p2cccd_b200.scene import ScenePipeline

    s, excl = meshes[r.mesh]
    alone = dict(s)
    alone["v_t0"], alone["v_t1"] = r.v_t0.numpy(), r.v_t1.numpy()
    sp = ScenePipeline(alone, dev, exclude_self=excl, config=cfg, narrow=narrow, top_k=top_k,
                       scheduler_seed=r.seed)
    return sp, sp.step_checked()


def _exact(summary):
    return {k: v for k, v in summary.items() if k != "speculative"}


def test_served_certificates_equal_alone(cuda_device):
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.serve import ServeEngine, latency_stats

    cfg = CertConfig(1e-6, 1e-6, 32)
    meshes = _meshes()
    eng = ServeEngine(cuda_device, config=cfg, slots=3, max_group=4, narrow="certify",
                      memory_budget=512 << 20)
    for key, (s, excl) in meshes.items():
        caps = (16, 16) if key == "batch0" else (None, None)  # its first step overflows and is re-run
        eng.register_mesh(key, s, exclude_self=excl, vf_capacity=caps[0], ee_capacity=caps[1])
    reqs = _requests(meshes, 36, np.random.default_rng(5))
    done = eng.run(reqs)
    assert len(done) == len(reqs)
    st = eng.stats()
    assert st["reruns"] > 0 and st["completed"] == len(reqs)
    assert st["groups"] < len(reqs) + st["reruns"]  # some groups held several requests
    assert latency_stats(done)["p50_ms"] > 0
    for r in done:
        sp, summ = _alone(r, meshes, cuda_device, cfg, "certify")
        assert r.summary == summ, r.rid
        a_vf, a_ee = sp.results()
        assert np.array_equal(_bytes(r.results[0]), _bytes(a_vf)), r.rid
        assert np.array_equal(_bytes(r.results[1]), _bytes(a_ee)), r.rid
        # the fallback-replay entries name exactly the undecided certificates
        und = {(1, int(p)) for p in np.nonzero(a_vf["status"] == 2)[0]} | \
              {(2, int(p)) for p in np.nonzero(a_ee["status"] == 2)[0]}
        assert {(int(f), int(p)) for f, p in r.undecided} == und, r.rid
    eng.close()


@pytest.mark.parametrize("top_k", [4096, 2])
def test_served_anyhit_equals_alone(cuda_device, top_k):
    """Any-hit mode: each request's per-family summaries (calls, hits,
    groups, fallback groups) and per-object-pair decisions equal the
    single-scene any-hit of the same step with the same scheduler seed."""
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.serve import ServeEngine

    cfg = CertConfig(1e-6, 1e-6, 32)
    meshes = _meshes()
    eng = ServeEngine(cuda_device, config=cfg, slots=3, max_group=5, narrow="anyhit", top_k=top_k,
                      memory_budget=512 << 20)
    for key, (s, excl) in meshes.items():
        caps = (16, 16) if key == "cloth" else (None, None)
        eng.register_mesh(key, s, exclude_self=excl, vf_capacity=caps[0], ee_capacity=caps[1])
    reqs = _requests(meshes, 30, np.random.default_rng(9), seed_base=77)
    done = eng.run(reqs)
    assert len(done) == len(reqs)
    calls = cands = 0
    for r in done:
        sp, summ = _alone(r, meshes, cuda_device, cfg, "anyhit", top_k)
        for fam in ("vf", "ee"):
            assert _exact(r.anyhit[fam]) == _exact(summ[fam]), (r.rid, fam, r.anyhit[fam], summ[fam])
        det_vf, _, _ = sp.anyhit_vf.read_groups()
        det_ee, _, _ = sp.anyhit_ee.read_groups()
        assert np.array_equal(r.groups[0], det_vf) and np.array_equal(r.groups[1], det_ee), r.rid
        calls += r.calls
        cands += r.queries
    assert 0 < calls <= cands
    eng.close()


def test_served_undecided_queue_overflow_reruns(cuda_device):
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.serve import ServeEngine

    cfg = CertConfig(1e-2, 1e-6, 4)  # coarse: many undecided certificates
    meshes = {k: v for k, v in _meshes().items() if k in ("spheres", "batch1")}
    eng = ServeEngine(cuda_device, config=cfg, slots=2, max_group=4, narrow="certify", undecided_capacity=4,
                      memory_budget=256 << 20)
    for key, (s, excl) in meshes.items():
        eng.register_mesh(key, s, exclude_self=excl)
    reqs = _requests(meshes, 8, np.random.default_rng(3))
    done = eng.run(reqs)
    assert eng.stats()["reruns"] > 0
    for r in done:
        sp, summ = _alone(r, meshes, cuda_device, cfg, "certify")
        assert r.summary["undecided"] == summ["undecided"] > 0
        assert len(r.undecided) == summ["undecided"]
    eng.close()


def test_memory_admission_and_a_request_too_large(cuda_device):
    """With a small arena, groups hold fewer requests and never more memory
    than the arena; a request that cannot fit the whole arena fails alone
    (P2C_ERR_CAPACITY) while the others complete."""
    from p2cccd_b200 import scenes
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.serve import Request, ServeEngine

    cfg = CertConfig(1e-6, 1e-6, 32)
    small = scenes.two_spheres(n_lon=24, n_rings=16)
    big = scenes.two_spheres(n_lon=300, n_rings=240)
    eng = ServeEngine(cuda_device, config=cfg, slots=4, max_group=8, narrow="anyhit", memory_budget=24 << 20)
    eng.register_mesh("small", small)
    eng.register_mesh("big", big)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    reqs = [Request(rid=i, mesh="small", v_t0=pin(small["v_t0"]), v_t1=pin(small["v_t1"]), arrival_s=0.0)
            for i in range(12)]
    rid_big = eng.admit(Request(rid=99, mesh="big", v_t0=pin(big["v_t0"]), v_t1=pin(big["v_t1"]), arrival_s=0.0))
    failed = []
    for _ in range(1000):
        for x in eng.poll():
            if int(x["status"]) != 0:
                assert int(x["status"]) == 3  # P2C_ERR_CAPACITY
                failed.append(int(x["request_id"]))
        if failed:
            break
    assert failed == [rid_big]
    done = eng.run(reqs)
    st = eng.stats()
    assert len(done) == 12 and all(r.status == 0 for r in done)
    assert st["arena_peak"] <= st["arena_bytes"] == 24 << 20
    assert len({r.anyhit["vf"]["detected_groups"] for r in done}) == 1
    eng.close()
