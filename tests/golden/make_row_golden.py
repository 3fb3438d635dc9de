"""Generates tests/golden/rows.json with the reference's own Python
serialization (p2cccd.serialization / contracts / validators, imported from a
reference checkout): the JSONL text of a set of AuditLogRows and
BenchmarkRowV2s, the CSV text of the benchmark rows, and the reference's
accept / reject verdict on a set of invalid benchmark rows.

    python tests/golden/make_row_golden.py /path/to/reference
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent


def audit_values():
    vals = []
    for k in range(6):
        vals.append(dict(event_id=100 + k, query_id=3 + k % 2, candidate_id=77 * k + 1, work_item_id=5 + k,
                         stage=2 if k % 2 == 0 else 4, action=1 if k % 2 == 0 else 2 + k % 4, depth=k,
                         interval_t0=[0.0, 0.1, 1e-300, 0.25, 1 / 3, 0.5][k],
                         interval_t1=[1.0, 0.75, 0.3, 0.5, 2 / 3, 0.5][k], timestamp_us=900 + k,
                         aux_value0=[0.5, -1.25, 1e-12, 3.0, 0.1 + 0.2, 0.0][k], aux_value1=float(k % 4)))
    return vals


def bench_values():
    base = dict(schema_version=3, run_id="run-1", dataset_name="synthetic", scene_name="two_spheres",
                method_name="b200", config_hash="cfg", seed=7, query_count=4735, fn_count=0, fp_count=0,
                candidate_recall=1.0, avg_candidates=1.0, avg_exact_evals=12.5, avg_subdivision_depth=0.0,
                fallback_ratio=0.0, candidate_inflation_ratio=1.0, undecided_to_resolved_ratio=0.001,
                exact_queue_occupancy=0.0, rt_build_ms=0.0, rt_update_ms=0.0, rt_trace_ms=0.05, rt_ms=0.05,
                proposal_ms=0.0, exact_ms=0.27, total_ms=32.8, latency_min_ms=0.31, latency_p50_ms=0.328,
                latency_p90_ms=0.33, latency_p95_ms=0.331, latency_p99_ms=0.34, latency_max_ms=0.35,
                qps=14.4e6, family_point_triangle_exact_calls=3000, family_edge_edge_exact_calls=1735,
                family_conservative_exact_calls=0, family_unknown_exact_calls=0, exact_calls_total=4735,
                candidate_buffer_bandwidth_mb_s=1234.5, proposal_enqueue_dequeue_ms=0.0,
                total_tail_latency_ms=0.34, vram_peak_mb=512)
    second = dict(base, run_id="run-2", seed=-3, qps=1.0 / 3.0, latency_p50_ms=0.1 + 0.2, latency_min_ms=0.1,
                  fallback_ratio=0.25)
    return [base, second]


def invalid_values():
    b = bench_values()[0]
    return [dict(b, schema_version=2), dict(b, run_id=""), dict(b, query_count=0), dict(b, fn_count=5000),
            dict(b, candidate_recall=1.5), dict(b, qps=-1.0), dict(b, latency_p50_ms=0.2),
            dict(b, exact_calls_total=4734), dict(b, total_ms=float("inf")), dict(b, seed=1.5)]


def main(reference: str) -> None:
    sys.path.insert(0, str(Path(reference) / "src" / "python"))
    from p2cccd import contracts, serialization
    from p2cccd.validators import validate_contract

    audit = [contracts.AuditLogRow(**dict(v, stage=contracts.AuditStage(v["stage"]))) for v in audit_values()]
    bench = [contracts.BenchmarkRowV2(**v) for v in bench_values()]
    verdicts = []
    for v in invalid_values():
        try:
            validate_contract(contracts.BenchmarkRowV2(**v))
            verdicts.append(True)
        except Exception:
            verdicts.append(False)
    with tempfile.TemporaryDirectory() as d:
        serialization.write_benchmark_v2_csv(Path(d) / "b.csv", bench)
        csv_text = (Path(d) / "b.csv").read_text()
    out = {"audit_values": audit_values(), "audit_jsonl": "".join(serialization.to_json(r) + "\n" for r in audit),
           "bench_values": bench_values(), "bench_jsonl": "".join(serialization.to_json(r) + "\n" for r in bench),
           "bench_csv": csv_text, "invalid_values": [{k: (repr(v) if isinstance(v, float) and v != v or v in
                                                          (float("inf"),) else v) for k, v in iv.items()}
                                                     for iv in invalid_values()],
           "invalid_accepted": verdicts}
    (HERE / "rows.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "rows.json", "accepted:", verdicts)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("P2C_REFERENCE_ROOT", "/root/reference"))
