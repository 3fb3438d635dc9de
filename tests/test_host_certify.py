"""The library's CPU certifier (p2c_certify_*_batch_cpu, the CPU side of the
CPU/CUDA cross-check) equals the oracle byte for byte: all 72 result bytes,
on the plain workload at three configurations, the reference-made golden
fixtures, sub-intervals and deep grazing trees.  Runs without a GPU."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "plain_sample.npz"


def _bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1, 72)


@pytest.mark.parametrize("cfg", [(1e-6, 1e-6, 32), (1e-4, 1e-6, 32), (1e-5, 1e-6, 8)])
@pytest.mark.parametrize("interval", [(0.0, 1.0), (0.25, 0.75)])
def test_cpu_certifier_equals_oracle(oracle_mod, cfg, interval):
    from p2cccd_b200 import certify, workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=2000, n_ee=2000, seed=11))
    for fam in ("vf", "ee"):
        cpu, st, _ = oracle_mod.eval_batch(w[fam], interval[0], interval[1], *cfg)
        assert st.sum() == 0
        got = certify.certify_batch_cpu(w[fam], interval[0], interval[1], certify.CertConfig(*cfg))
        assert np.array_equal(_bytes(got), _bytes(cpu)), fam


def test_cpu_certifier_golden_and_deep_trees(oracle_mod):
    from p2cccd_b200 import certify, records

    g = np.load(GOLDEN)
    for tag, cfg in (("c6", (1e-6, 1e-6, 32)), ("cdef", (1e-4, 1e-6, 32))):
        for fam, dt in (("vf", records.POINT_TRIANGLE_DTYPE), ("ee", records.EDGE_EDGE_DTYPE)):
            rec = np.ascontiguousarray(g[fam]).view(dt).reshape(-1)
            got = certify.certify_batch_cpu(rec, 0.0, 1.0, certify.CertConfig(*cfg))
            np.testing.assert_array_equal(_bytes(got), g[f"{fam}_{tag}"])
    rng = np.random.default_rng(3)
    n = 16
    p0 = np.zeros((n, 4, 3))
    tri = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    p0[:, 1:, :] = tri
    p1 = p0.copy()
    h = 1e-6 * (1.0 + rng.uniform(1e-4, 1e-2, size=n))
    p0[:, 0, :] = np.stack([rng.uniform(0.05, 0.3, n), rng.uniform(0.05, 0.3, n), h], 1)
    p1[:, 0, :] = p0[:, 0, :] + np.stack([rng.uniform(0.1, 0.4, n), rng.uniform(0.1, 0.4, n), np.zeros(n)], 1)
    dip = rng.uniform(size=n) < 0.3
    p1[dip, 0, 2] = -h[dip]
    rec = records.pack_primitives(p0, p1, np.arange(n), np.arange(n) + 100)
    cpu, _, nodes = oracle_mod.eval_batch(rec, 0.0, 1.0, 1e-5, 1e-6, 32)
    assert nodes.max() > 100_000
    got = certify.certify_batch_cpu(rec, 0.0, 1.0, certify.CertConfig(1e-5, 1e-6, 32))
    assert np.array_equal(_bytes(got), _bytes(cpu))


def test_cpu_certifier_rejects_like_the_reference():
    from p2cccd_b200 import certify, workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=8, n_ee=8, seed=2))
    bad = w["vf"].copy()
    bad[3]["point_id"] = -1
    with pytest.raises(ValueError, match="point-triangle primitive ids are required"):
        certify.certify_batch_cpu(bad)
    bad = w["ee"].copy()
    bad[5]["edge_b0"]["position_t1"][1] = np.inf
    with pytest.raises(ValueError, match="edge-edge primitive trajectories must be finite"):
        certify.certify_batch_cpu(bad)
    with pytest.raises(ValueError, match="0 <= t0 <= t1 <= 1"):
        certify.certify_batch_cpu(w["vf"], 0.5, 0.25)


def test_cross_check_comparison_rules_catch_a_planted_difference(oracle_mod):
    """The comparison the cross-check applies (the reference's rules) flags
    a difference planted in a copy of the oracle's certificates."""
    import p2cccd_cpp as m
    from p2cccd_b200 import workloads

    w = workloads.plain_queries(workloads.PlainSpec(n_vf=200, n_ee=10, seed=4))
    cpu, _, _ = oracle_mod.eval_batch(w["vf"], 0.0, 1.0, 1e-6, 1e-6, 32)
    m._compare(cpu, cpu.copy(), 1e-6, "x")
    sep = int(np.nonzero(cpu["status"] == 1)[0][0])
    planted = cpu.copy()
    planted[sep]["safe_margin_lb"] += 1e-3
    with pytest.raises(ValueError, match="safe margin mismatch"):
        m._compare(cpu, planted, 1e-6, "x")
    planted = cpu.copy()
    planted[sep]["status"] = 2
    with pytest.raises(ValueError, match="status mismatch"):
        m._compare(cpu, planted, 1e-6, "x")
