"""The candidate-group early-stop replay (common/group_scheduler.cpp:60-239,
parse py_module.cpp:1179-1246): the restated replay against the reference
compiled unchanged on the CPU; the device replay against both on the GPU,
every total (the double work sums included) bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from dense_inputs import make_rows

CASES = [(1, 200, {}, {}), (2, 500, {"big_group": 60}, {"threshold": 0.9, "limit": 2, "penalty": 0.5}),
         (3, 300, {}, {"preserve": True}), (4, 50, {"n_groups": 2}, {"threshold": 0.3, "limit": 1, "penalty": 0.0}),
         (5, 0, {}, {}), (6, 1, {}, {}), (7, 2000, {"big_group": 700}, {"threshold": 0.97, "limit": 40}),
         (8, 400, {"ties": False, "zero_cost": 0.0}, {"threshold": 0.0})]

FIELDS = ("candidate_count", "group_count", "positive_group_count", "no_proposal_exact_calls",
          "no_proposal_exact_work", "learned_exact_calls", "learned_fallback_calls", "learned_interval_hit_count",
          "learned_interval_miss_count", "learned_exact_work", "first_positive_rank_sum",
          "cost_before_first_positive_sum", "tp", "tn", "fp", "fn", "reordered_count",
          "high_uncertainty_group_count")


def _same(a, b) -> list:
    """Fields whose values differ (doubles compared by their bits)."""
    bad = []
    for k in FIELDS:
        x, y = a[k], b[k]
        if isinstance(x, (float, np.floating)) or isinstance(y, (float, np.floating)):
            if np.float64(x).tobytes() != np.float64(y).tobytes():
                bad.append(k)
        elif int(x) != int(y):
            bad.append(k)
    return bad


@pytest.mark.parametrize("seed,n,kw,cfg", CASES)
def test_restated_replay_matches_reference(oracle_mod, seed, n, kw, cfg):
    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    rows = make_rows(n, seed, **kw)
    assert _same(oracle_mod.ref_dense_group(rows, **cfg), oracle_mod.dense_group(rows, **cfg)) == []


@pytest.mark.parametrize("fault,msg", [("qid", "dense group candidate ids must be non-zero"),
                                       ("cid", "dense group candidate ids must be non-zero"),
                                       ("trace", "dense group candidate contains a non-finite field"),
                                       ("prio", "dense group candidate contains a non-finite field"),
                                       ("overflow", "dense group candidate contains a non-finite field")])
def test_invalid_rows_match_reference(oracle_mod, fault, msg):
    rows = make_rows(40, 9)
    if fault == "qid":
        rows["query_id"][17] = 0
    elif fault == "cid":
        rows["candidate_id"][3] = 0
    elif fault == "trace":
        rows["oracle_trace"][5, 6] = np.inf
    elif fault == "prio":
        rows["priority_score"][22] = np.nan
    else:  # full * cost_target overflows to inf
        rows["oracle_trace"][8, 5] = 1e308
        rows["cost_target"][8] = np.float32(4.0)
    if oracle_mod.ref_available():
        with pytest.raises(ValueError, match=msg):
            oracle_mod.ref_dense_group(rows)
    with pytest.raises(ValueError, match=msg):
        oracle_mod.dense_group(rows)


@pytest.mark.parametrize("cfg,msg", [({"limit": 0}, "representative_attempt_limit must be positive"),
                                     ({"threshold": -0.5}, "uncertainty_fallback_threshold must be finite"),
                                     ({"threshold": float("inf")}, "uncertainty_fallback_threshold must be finite"),
                                     ({"penalty": float("nan")}, "interval_miss_penalty_scale must be finite")])
def test_invalid_config_messages(oracle_mod, cfg, msg):
    rows = make_rows(20, 10)
    if oracle_mod.ref_available():
        with pytest.raises(ValueError, match=msg):
            oracle_mod.ref_dense_group(rows, **cfg)
    with pytest.raises(ValueError, match=msg):
        oracle_mod.dense_group(rows, **cfg)


def test_array_checks():
    from p2cccd_b200.dense_groups import parse_arrays

    rows = make_rows(10, 11)
    feats = {k: rows[k] for k in ("query_id", "candidate_id", "cost_target", "oracle_trace")}
    preds = {k: rows[k] for k in ("interval_scores", "priority_score", "cost_score", "uncertainty_score")}
    assert parse_arrays(feats, preds)["oracle_trace"].shape == (10, 8)
    with pytest.raises(ValueError, match=r"oracle_trace must have shape \[10, 8\]"):
        parse_arrays(dict(feats, oracle_trace=rows["oracle_trace"][:, :7]), preds)
    with pytest.raises(ValueError, match=r"priority_score must have shape \[10\]"):
        parse_arrays(feats, dict(preds, priority_score=rows["priority_score"][:9]))
    with pytest.raises(ValueError, match="missing or invalid array field: cost_score"):
        parse_arrays(feats, {k: v for k, v in preds.items() if k != "cost_score"})


# ---------------------------------------------------------------- on the GPU

@pytest.mark.gpu
@pytest.mark.parametrize("seed,n,kw,cfg", CASES)
def test_device_replay_matches_reference(oracle_mod, seed, n, kw, cfg):
    from p2cccd_b200.dense_groups import DenseGroupEarlyStop, _query_bits, upload

    rows = make_rows(n, seed, **kw)
    want = oracle_mod.ref_dense_group(rows, **cfg) if oracle_mod.ref_available() else oracle_mod.dense_group(rows,
                                                                                                           **cfg)
    r = DenseGroupEarlyStop(max(n, 1))
    r.run(upload(rows) if n else {}, n, query_bits=_query_bits(rows["query_id"]), **cfg)
    assert _same(r.result(), want) == []


@pytest.mark.gpu
def test_device_replay_rejects_rows_like_reference():
    from p2cccd_b200.dense_groups import DenseGroupEarlyStop, upload

    rows = make_rows(300, 12)
    rows["priority_score"][250] = np.inf
    rows["query_id"][270] = 0
    r = DenseGroupEarlyStop(300)
    r.run(upload(rows), 300)
    with pytest.raises(ValueError, match="non-finite field"):  # row 250 comes first
        r.result()
    with pytest.raises(ValueError, match="representative_attempt_limit must be positive"):
        r.run(upload(rows), 300, limit=0)


@pytest.mark.gpu
def test_mirror_result_dict(oracle_mod):
    import p2cccd_cpp as cpp

    rows = make_rows(3000, 13, big_group=300)
    feats = {k: rows[k] for k in ("query_id", "candidate_id", "cost_target", "oracle_trace")}
    preds = {k: rows[k] for k in ("interval_scores", "priority_score", "cost_score", "uncertainty_score")}
    got = cpp.run_native_dense_group_exact_early_stop(feats, preds, 0.8, 3, 0.22, False)
    want = oracle_mod.dense_group(rows, threshold=0.8)
    for k in ("group_count", "learned_exact_calls", "tp", "fn", "reordered_count", "learned_exact_work",
              "no_proposal_exact_work"):
        assert got[k] == want[k], k
    pos = want["positive_group_count"]
    assert got["first_positive_rank_mean"] == want["first_positive_rank_sum"] / pos
    assert got["cost_weighted_first_positive_mean"] == want["cost_before_first_positive_sum"] / pos
    assert got["exact_work_reduction"] == 1.0 - want["learned_exact_work"] / want["no_proposal_exact_work"]
    assert got["native_total_ms"] >= got["parse_ms"] >= 0.0


@pytest.mark.gpu
def test_large_replay_against_reference(oracle_mod):
    """200k rows in 20k uneven groups: the device totals against the
    reference (the restatement is too slow at this size)."""
    from p2cccd_b200.dense_groups import DenseGroupEarlyStop, _query_bits, upload

    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")
    rows = make_rows(200_000, 14, n_groups=20_000, big_group=5000)
    want = oracle_mod.ref_dense_group(rows, threshold=0.93, limit=4)
    r = DenseGroupEarlyStop(200_000)
    r.run(upload(rows), 200_000, threshold=0.93, limit=4, query_bits=_query_bits(rows["query_id"]))
    assert _same(r.result(), want) == []


def _ordered_cases():
    """Non-negative term sequences that stress the ordered sum: wide dynamic
    range, exact half-ulp ties, runs of zeros (also in front), subnormals,
    terms that jump several binades, sums that round up to a power of two,
    an infinite term, and lengths around the 4,096-term chunk."""
    rng = np.random.default_rng(5)
    cases = [np.zeros(0), np.zeros(10), np.array([0.0, 0.0, 3.5]), np.array([2.0 ** -1074] * 5000)]
    for n in (1, 31, 4095, 4096, 4097, 12289, 50000):
        cases.append(rng.gamma(2.0, 3.0, n))
        cases.append(np.exp(rng.uniform(-40.0, 40.0, n)))
        cases.append(rng.integers(0, 64, n) * 2.0 ** rng.integers(-60, 10, n).astype(np.float64))
        z = rng.random(n)
        z[rng.random(n) < 0.4] = 0.0
        cases.append(z)
        cases.append(rng.integers(0, 3, n) * 0.5 + 2.0 ** 52 * (rng.random(n) < 0.05))
    ups = np.full(9000, 1.0)  # 2^53 + 1 + 1 + ... ties-to-even at every step
    ups[0] = 2.0 ** 53
    cases.append(ups)
    w = rng.random(6000) * 1e292
    w[0], w[3000], w[3001] = 1e300, 1e308, 1e308  # overflow to inf
    cases.append(w)
    w = rng.random(6000)
    w[4500] = np.inf
    cases.append(w)
    w = rng.random(5000)
    w[::7] = -0.0  # negative zeros add nothing
    w[:3] = -0.0
    cases.append(w)
    return cases


@pytest.mark.gpu
def test_ordered_sum_is_the_sequential_sum():
    import math

    import torch

    from p2cccd_b200.dense_groups import ordered_sum

    for i, c in enumerate(_ordered_cases()):
        want = 0.0
        for x in c.tolist():
            want += x
        got = float(ordered_sum(torch.from_numpy(np.ascontiguousarray(c, np.float64)).cuda()).item())
        assert (got == want and math.copysign(1.0, got) == math.copysign(1.0, want)) or \
            (math.isnan(got) and math.isnan(want)), (i, len(c), got, want)
