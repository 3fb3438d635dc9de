"""GPU tests of the continuous-batching server: every request's summary and
certificates in the served mix equal the same step certified alone (the
single-scene path, itself pinned to the oracle); requests admitted by memory
and slots overlap; overflowing candidate buffers are re-run to completion."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1, 72)


def _meshes():
    from p2cccd_b200 import scenes

    out = {
        "spheres": (scenes.two_spheres(n_lon=40, n_rings=30), True),
        "cloth": (scenes.cloth_on_sphere(n=33, sphere_lon=40, sphere_rings=30, gap=1e-3, drop=0.05), False),
    }
    for i, s in enumerate(scenes.uneven_batch(3, tri_min=2000, tri_max=20000, seed=11)):
        out[f"batch{i}"] = (s, True)
    return out


def _variant(s, k, rng):
    """Step k of a mesh: the scene's trajectories plus a small per-step offset."""
    jit = rng.normal(0.0, 1e-4, s["v_t1"].shape) if k else 0.0
    return s["v_t0"], s["v_t1"] + jit


def test_served_results_equal_alone(cuda_device):
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.scene import ScenePipeline
    from p2cccd_b200.serve import Request, ServeEngine, _request_bytes, latency_stats

    cfg = CertConfig(1e-6, 1e-6, 32)
    meshes = _meshes()
    rng = np.random.default_rng(5)
    eng = ServeEngine(cuda_device, config=cfg, slots=3, max_group=4)
    for key, (s, excl) in meshes.items():
        # tiny first capacities for one mesh: its first step overflows and is re-run
        caps = (16, 16) if key == "batch0" else (None, None)
        eng.register_mesh(key, s, exclude_self=excl, vf_capacity=caps[0], ee_capacity=caps[1])
    # memory budget of about 2.5 of the largest requests: admission also waits on memory
    eng.memory_budget = int(2.5 * max(_request_bytes(m) for m in eng.meshes.values()))
    reqs, t = [], 0.0
    keys = list(meshes)
    for i in range(36):
        key = keys[int(rng.integers(len(keys)))]
        s, _ = meshes[key]
        v0, v1 = _variant(s, i, rng)
        t += float(rng.exponential(2e-4))
        reqs.append(Request(rid=i, mesh=key, v_t0=torch.from_numpy(np.ascontiguousarray(v0)).pin_memory(),
                            v_t1=torch.from_numpy(np.ascontiguousarray(v1)).pin_memory(), arrival_s=t,
                            keep_results=True))
    done = eng.run(reqs)
    assert len(done) == len(reqs)
    assert sum(r.reruns for r in done) > 0
    assert eng.groups_run < len(reqs) + sum(r.reruns for r in done)  # some groups held several requests
    stats = latency_stats(done)
    assert stats["p50_ms"] > 0
    for r in done:
        s, excl = meshes[r.mesh]
        alone = dict(s)
        alone["v_t0"], alone["v_t1"] = r.v_t0.numpy(), r.v_t1.numpy()
        sp = ScenePipeline(alone, cuda_device, exclude_self=excl, config=cfg)
        summ = sp.step_checked()
        assert r.summary == summ, r.rid
        a_vf, a_ee = sp.results()
        assert np.array_equal(_bytes(r.results[0]), _bytes(a_vf)), r.rid
        assert np.array_equal(_bytes(r.results[1]), _bytes(a_ee)), r.rid
        # the fallback-replay entries name exactly the undecided certificates
        und = {(1, int(p)) for p in np.nonzero(a_vf["status"] == 2)[0]} | \
              {(2, int(p)) for p in np.nonzero(a_ee["status"] == 2)[0]}
        assert {(int(f), int(p)) for f, p in r.undecided} == und, r.rid


def test_memory_admission_serialises_when_budget_is_small(cuda_device):
    from p2cccd_b200.certify import CertConfig
    from p2cccd_b200.serve import Request, ServeEngine, _request_bytes

    cfg = CertConfig(1e-6, 1e-6, 32)
    meshes = _meshes()
    s, excl = meshes["spheres"]
    eng = ServeEngine(cuda_device, config=cfg, slots=4, max_group=8, memory_budget=1)
    eng.register_mesh("spheres", s, exclude_self=excl)
    v0 = torch.from_numpy(np.ascontiguousarray(s["v_t0"])).pin_memory()
    v1 = torch.from_numpy(np.ascontiguousarray(s["v_t1"])).pin_memory()
    reqs = [Request(rid=i, mesh="spheres", v_t0=v0, v_t1=v1, arrival_s=0.0) for i in range(6)]
    done = eng.run(reqs)
    # a lone request is always admitted, but never two at once under a 1-byte budget
    assert eng.groups_run == 6 + sum(r.reruns for r in done)
    assert len({r.summary["collisions"] for r in done}) == 1
