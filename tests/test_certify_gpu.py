"""GPU parity of the batch certifier: every 72-byte result equals the CPU
oracle's byte for byte (status, interval, toi, margin, witness, reason,
refinement mode, zero padding) - and the golden fixtures made by the
reference.  Calls go through the C ABI."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "plain_sample.npz"


def _gpu_certify(records, fam, t0, t1, cfg):
    import torch
    from p2cccd_b200 import certify

    dev = certify.records_to_device(records)
    out = certify.certify_batch(dev, fam, t0, t1, certify.CertConfig(*cfg))
    torch.cuda.synchronize()
    return certify.results_to_numpy(out)


def _bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1, 72)


def _assert_parity(gpu, cpu, records=None):
    g, c = _bytes(gpu), _bytes(cpu)
    bad = np.nonzero((g != c).any(axis=1))[0]
    if bad.size:
        i = bad[0]
        raise AssertionError(f"{bad.size} results differ; first at {i}: gpu={gpu[i]} cpu={cpu[i]}")


@pytest.mark.parametrize("cfg", [(1e-6, 1e-6, 32), (1e-4, 1e-6, 32), (1e-5, 1e-6, 8)])
def test_plain_workload_parity(cuda_device, oracle_mod, cfg):
    from p2cccd_b200 import workloads

    w = workloads.plain_queries()
    for fam_id, fam in ((1, "vf"), (2, "ee")):
        cpu, st, _ = oracle_mod.eval_batch(w[fam], 0.0, 1.0, *cfg)
        assert st.sum() == 0
        gpu = _gpu_certify(w[fam], fam_id, 0.0, 1.0, cfg)
        _assert_parity(gpu, cpu)


def test_golden_fixture_parity(cuda_device):
    from p2cccd_b200 import records

    g = np.load(GOLDEN)
    for tag, cfg in (("c6", (1e-6, 1e-6, 32)), ("cdef", (1e-4, 1e-6, 32))):
        for fam_id, fam, dt in ((1, "vf", records.POINT_TRIANGLE_DTYPE), (2, "ee", records.EDGE_EDGE_DTYPE)):
            rec = np.ascontiguousarray(g[fam]).view(dt).reshape(-1)
            gpu = _gpu_certify(rec, fam_id, 0.0, 1.0, cfg)
            np.testing.assert_array_equal(_bytes(gpu), g[f"{fam}_{tag}"])
    for fam_id, fam, dt in ((1, "ka_pt", records.POINT_TRIANGLE_DTYPE), (2, "ka_ee", records.EDGE_EDGE_DTYPE)):
        rec = np.ascontiguousarray(g[fam]).view(dt).reshape(-1)
        gpu = _gpu_certify(rec, fam_id, 0.0, 1.0, (1e-5, 1e-6, 32))
        np.testing.assert_array_equal(_bytes(gpu), g[f"{fam}_ka"])
        assert gpu[0]["status"] == 0 and abs(gpu[0]["toi_upper"] - 0.25) <= 1e-12


@pytest.mark.parametrize("interval", [(0.25, 0.75), (0.3, 0.7), (0.0, 0.0), (1.0, 1.0), (0.1, 0.1000001)])
def test_subinterval_parity(cuda_device, oracle_mod, interval):
    from p2cccd_b200 import workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=3000, n_ee=3000, seed=5))
    for fam_id, fam in ((1, "vf"), (2, "ee")):
        cpu, _, _ = oracle_mod.eval_batch(w[fam], interval[0], interval[1], 1e-6, 1e-6, 32)
        gpu = _gpu_certify(w[fam], fam_id, interval[0], interval[1], (1e-6, 1e-6, 32))
        _assert_parity(gpu, cpu)


def test_deep_grazing_queries_parity(cuda_device, oracle_mod):
    """Queries whose trees are wide and deep (distance hovering near eps_space
    along the whole interval) exercise donation between lanes and pruning."""
    from p2cccd_b200 import records

    rng = np.random.default_rng(3)
    n = 64
    p0 = np.zeros((n, 4, 3))
    p1 = np.zeros((n, 4, 3))
    tri = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    p0[:, 1:, :] = tri
    p1[:, 1:, :] = tri
    h = 1e-6 * (1.0 + rng.uniform(1e-4, 1e-2, size=n))
    p0[:, 0, :] = np.stack([rng.uniform(0.05, 0.3, n), rng.uniform(0.05, 0.3, n), h], 1)
    p1[:, 0, :] = p0[:, 0, :] + np.stack([rng.uniform(0.1, 0.4, n), rng.uniform(0.1, 0.4, n), np.zeros(n)], 1)
    # a few dip through the plane late in the step: collision after a wide tree
    dip = rng.uniform(size=n) < 0.3
    p1[dip, 0, 2] = -h[dip]
    rec = records.pack_primitives(p0, p1, np.arange(n), np.arange(n) + 100)
    cfg = (1e-5, 1e-6, 32)
    cpu, _, nodes = oracle_mod.eval_batch(rec, 0.0, 1.0, *cfg)
    assert nodes.max() > 100_000
    gpu = _gpu_certify(rec, 1, 0.0, 1.0, cfg)
    _assert_parity(gpu, cpu)
    # edge-edge: an edge sliding over a static edge at height ~eps_space
    q0 = np.zeros((n, 4, 3))
    q0[:, 0] = [-1.0, 0.0, 0.0]
    q0[:, 1] = [1.0, 0.0, 0.0]
    q0[:, 2] = np.stack([np.full(n, -0.5), rng.uniform(-1, -0.5, n), h], 1)
    q0[:, 3] = np.stack([np.full(n, 0.5), rng.uniform(-1, -0.5, n), h], 1)
    q1 = q0.copy()
    q1[:, 2:, 1] += 1.5
    q1[dip, 2:, 2] = -h[dip, None]
    rec = records.pack_primitives(q0, q1, np.arange(n), np.arange(n) + 100, family=2)
    cpu, _, nodes = oracle_mod.eval_batch(rec, 0.0, 1.0, *cfg)
    gpu = _gpu_certify(rec, 2, 0.0, 1.0, cfg)
    _assert_parity(gpu, cpu)


def test_host_buffer_api_parity_and_errors(cuda_device, oracle_mod):
    from p2cccd_b200 import certify, workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=2000, n_ee=2000, seed=9))
    for fam in ("vf", "ee"):
        cpu, _, _ = oracle_mod.eval_batch(w[fam], 0.0, 1.0, 1e-4, 1e-6, 32)
        gpu = certify.certify_batch_host(w[fam], 0.0, 1.0, certify.CertConfig())
        _assert_parity(gpu, cpu)
    # empty input: Ok with no results (certificate_cuda.cu:465-468)
    assert len(certify.certify_batch_host(w["vf"][:0])) == 0
    bad = w["vf"][:5].copy()
    bad["point_id"][3] = -1
    with pytest.raises(ValueError, match="point-triangle primitive ids are required"):
        certify.certify_batch_host(bad)
    bad = w["ee"][:5].copy()
    bad["edge_b1"]["position_t0"][2, 1] = np.inf
    with pytest.raises(ValueError, match="edge-edge primitive trajectories must be finite"):
        certify.certify_batch_host(bad)
    with pytest.raises(ValueError, match="0 <= t0 <= t1 <= 1"):
        certify.certify_batch_host(w["vf"][:5], 0.6, 0.5)
    with pytest.raises(ValueError, match="eps_time"):
        certify.certify_batch_host(w["vf"][:5], 0.0, 1.0, certify.CertConfig(eps_time=0.0))


def test_census_matches_oracle_node_count(cuda_device, oracle_mod):
    import torch
    from p2cccd_b200 import certify, workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=3000, n_ee=3000, seed=21))
    cfg = (1e-6, 1e-6, 32)
    cpu_pt, _, n_pt = oracle_mod.eval_batch(w["vf"], 0.0, 1.0, *cfg)
    cpu_ee, _, n_ee = oracle_mod.eval_batch(w["ee"], 0.0, 1.0, *cfg)
    res = certify.census(certify.records_to_device(w["vf"]), certify.records_to_device(w["ee"]), 0.0, 1.0,
                         certify.CertConfig(*cfg))
    assert res["stats"]["nodes_evaluated"] == int(n_pt.sum() + n_ee.sum())
    assert res["stats"]["queries"] == 6000
    assert res["stats"]["fp64_ops"] > 0 and res["stats"]["error_word"] == 0
    _assert_parity(certify.results_to_numpy(res["pt"]), cpu_pt)
    _assert_parity(certify.results_to_numpy(res["ee"]), cpu_ee)
    torch.cuda.synchronize()
