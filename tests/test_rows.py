"""The audit and benchmark row exports against the reference's own Python
serialization (golden text in tests/golden/rows.json, made by
tests/golden/make_row_golden.py): JSONL and CSV byte for byte, and the same
accept / reject verdicts of the row validator."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = json.loads((Path(__file__).parent / "golden" / "rows.json").read_text())


def _audit_array(values):
    from p2cccd_b200.records import AUDIT_ROW_DTYPE

    a = np.zeros(len(values), AUDIT_ROW_DTYPE)
    for r, v in zip(a, values):
        for k, x in v.items():
            r[k] = x
    return a


def test_audit_jsonl_matches_reference():
    from p2cccd_b200 import rows

    assert rows.audit_jsonl(_audit_array(GOLDEN["audit_values"])) == GOLDEN["audit_jsonl"]


def test_benchmark_rows_match_reference():
    from p2cccd_b200 import rows

    vals = GOLDEN["bench_values"]
    assert rows.benchmark_jsonl(vals) == GOLDEN["bench_jsonl"]
    assert rows.benchmark_csv(vals) == GOLDEN["bench_csv"]


def test_benchmark_validator_agrees_with_reference():
    from p2cccd_b200 import rows

    for v, accepted in zip(GOLDEN["invalid_values"], GOLDEN["invalid_accepted"]):
        v = {k: (float(x) if x in ("inf", "nan") else x) for k, x in v.items()}
        try:
            rows.validate_benchmark_row_v2(v)
            ok = True
        except rows.RowValidationError:
            ok = False
        assert ok == accepted, v


def test_benchmark_row_from_counters():
    from p2cccd_b200 import rows

    r = rows.benchmark_row_v2(run_id="r", dataset_name="synthetic", scene_name="s", method_name="b200",
                              config_hash="h", seed=1, query_count=1000, latencies_ms=[0.5, 0.4, 0.6, 0.45],
                              exact_ms=0.3, rt_ms=0.1, pt_exact_calls=600, ee_exact_calls=400, distance_evals=9000,
                              collisions=10, separations=980, undecided=10, candidate_bytes=8000,
                              vram_peak_bytes=3 << 20)
    assert r["exact_calls_total"] == 1000 and r["avg_exact_evals"] == 9.0 and r["vram_peak_mb"] == 3
    assert r["latency_min_ms"] == 0.4 and r["latency_max_ms"] == 0.6 and r["qps"] == pytest.approx(4000 / 1.95e-3)
    assert r["undecided_to_resolved_ratio"] == pytest.approx(10 / 990)
    line = rows.benchmark_jsonl([r])
    assert line.startswith('{"schema_version":3,"run_id":"r",') and line.endswith("}\n")
