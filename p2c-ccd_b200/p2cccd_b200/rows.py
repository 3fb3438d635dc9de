"""Audit and benchmark rows in the reference's export formats.

``p2cccd.serialization`` (the reference's Python package) writes
``AuditLogRow`` and ``BenchmarkRowV2`` contracts as JSON lines: compact
separators, the contract's schema field order, enums as integers
(serialization.py:48-96), and CSV with a header in the same order
(:111-128).  The writers here produce the same bytes from the device outputs
(``AUDIT_ROW_DTYPE`` records of ``p2c_audit_rows``) and from a run's device
counters and timings, so downstream tooling that reads the reference's files
reads these.  The field lists are the reference's schemas
(contracts.py:120-132, 181-222, 295-...); ``validate_benchmark_row_v2``
restates validators.py:330-400.
"""
from __future__ import annotations

import csv
import io
import json
import math
from pathlib import Path
from typing import Iterable

import numpy as np

BENCHMARK_EXPORT_SCHEMA_VERSION = 3

AUDIT_ROW_FIELDS = ("event_id", "query_id", "candidate_id", "work_item_id", "stage", "action", "depth",
                    "interval_t0", "interval_t1", "timestamp_us", "aux_value0", "aux_value1")

# (name, kind): "u" unsigned, "i" signed, "f" float, "s" string
BENCHMARK_ROW_V2_FIELDS = (
    ("schema_version", "u"), ("run_id", "s"), ("dataset_name", "s"), ("scene_name", "s"), ("method_name", "s"),
    ("config_hash", "s"), ("seed", "i"), ("query_count", "u"), ("fn_count", "u"), ("fp_count", "u"),
    ("candidate_recall", "f"), ("avg_candidates", "f"), ("avg_exact_evals", "f"), ("avg_subdivision_depth", "f"),
    ("fallback_ratio", "f"), ("candidate_inflation_ratio", "f"), ("undecided_to_resolved_ratio", "f"),
    ("exact_queue_occupancy", "f"), ("rt_build_ms", "f"), ("rt_update_ms", "f"), ("rt_trace_ms", "f"),
    ("rt_ms", "f"), ("proposal_ms", "f"), ("exact_ms", "f"), ("total_ms", "f"), ("latency_min_ms", "f"),
    ("latency_p50_ms", "f"), ("latency_p90_ms", "f"), ("latency_p95_ms", "f"), ("latency_p99_ms", "f"),
    ("latency_max_ms", "f"), ("qps", "f"), ("family_point_triangle_exact_calls", "u"),
    ("family_edge_edge_exact_calls", "u"), ("family_conservative_exact_calls", "u"),
    ("family_unknown_exact_calls", "u"), ("exact_calls_total", "u"), ("candidate_buffer_bandwidth_mb_s", "f"),
    ("proposal_enqueue_dequeue_ms", "f"), ("total_tail_latency_ms", "f"), ("vram_peak_mb", "u"),
)

_U64 = (1 << 64) - 1
_U32 = (1 << 32) - 1


def _json_line(values: dict) -> str:
    return json.dumps(values, sort_keys=False, separators=(",", ":"))


def audit_row_dicts(rows: np.ndarray) -> list[dict]:
    """AUDIT_ROW_DTYPE records as the reference contract's plain dicts."""
    out = []
    for r in rows:
        d = {}
        for k in AUDIT_ROW_FIELDS:
            v = r[k]
            d[k] = float(v) if k in ("interval_t0", "interval_t1", "aux_value0", "aux_value1") else int(v)
        out.append(d)
    return out


def audit_jsonl(rows: np.ndarray) -> str:
    """The audit rows as write_audit_jsonl's text (one row per line)."""
    return "".join(_json_line(d) + "\n" for d in audit_row_dicts(rows))


def write_audit_jsonl(path: str | Path, rows: np.ndarray) -> None:
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    p.write_text(audit_jsonl(rows), encoding="utf-8", newline="\n")


class RowValidationError(ValueError):
    pass


def validate_benchmark_row_v2(row: dict) -> dict:
    """validate_benchmark_row_v2 (validators.py:330-400): types, ranges,
    non-empty names, monotonic latency percentiles, family call sums."""
    def fail(msg):
        raise RowValidationError(f"BenchmarkRowV2.{msg}")

    for name, kind in BENCHMARK_ROW_V2_FIELDS:
        v = row[name]
        if kind in ("u", "i"):
            if isinstance(v, bool) or not isinstance(v, int):
                fail(f"{name} must be an integer")
            lo, hi = (0, _U32 if name == "schema_version" else _U64) if kind == "u" else (-(1 << 63), (1 << 63) - 1)
            if not lo <= v <= hi:
                fail(f"{name} is out of range")
        elif kind == "f":
            if isinstance(v, bool) or not isinstance(v, (int, float)) or not math.isfinite(float(v)):
                fail(f"{name} must be finite")
            if float(v) < 0.0:
                fail(f"{name} must be non-negative")
        elif not isinstance(v, str) or (name != "schema_version" and not v):
            fail(f"{name} must be a non-empty string")
    if row["schema_version"] != BENCHMARK_EXPORT_SCHEMA_VERSION:
        fail("schema_version is unsupported")
    if row["query_count"] == 0:
        fail("query_count must be non-zero")
    if row["fn_count"] > row["query_count"]:
        fail("fn_count cannot exceed query_count")
    for name in ("candidate_recall", "fallback_ratio"):
        if float(row[name]) > 1.0:
            fail(f"{name} must lie in [0, 1]")
    lat = [float(row[k]) for k in ("latency_min_ms", "latency_p50_ms", "latency_p90_ms", "latency_p95_ms",
                                   "latency_p99_ms", "latency_max_ms")]
    if lat != sorted(lat):
        fail("latency percentiles must be monotonic")
    fam = sum(row[k] for k in ("family_point_triangle_exact_calls", "family_edge_edge_exact_calls",
                               "family_conservative_exact_calls", "family_unknown_exact_calls"))
    if fam != row["exact_calls_total"]:
        fail("exact_calls_total must equal family-wise exact calls")
    return row


def _percentile(sorted_ms: list[float], q: float) -> float:
    """Linear-interpolated percentile of sorted values (numpy's default)."""
    return float(np.percentile(np.asarray(sorted_ms, dtype=np.float64), q)) if sorted_ms else 0.0


def benchmark_row_v2(*, run_id: str, dataset_name: str, scene_name: str, method_name: str, config_hash: str,
                     seed: int, query_count: int, latencies_ms: Iterable[float], exact_ms: float, rt_ms: float = 0.0,
                     total_ms: float | None = None, pt_exact_calls: int = 0, ee_exact_calls: int = 0,
                     distance_evals: int = 0, collisions: int = 0, separations: int = 0, undecided: int = 0,
                     candidates: int | None = None, fallback_calls: int = 0, exact_calls: int | None = None,
                     candidate_bytes: int = 0, vram_peak_bytes: int = 0, **extra) -> dict:
    """A BenchmarkRowV2 from a run's device counters and CUDA-event timings.

    ``latencies_ms`` are per-step (or per-request) device times; ``qps`` is
    certified queries per second over their sum.  False negatives and
    positives are 0 by construction (certificates are the reference
    certifier's, bit for bit; there is no other ground truth in a synthetic
    run); candidate recall is 1 (every candidate is certified).  The device
    engine does not track subdivision depth, so avg_subdivision_depth is 0."""
    lat = sorted(float(x) for x in latencies_ms)
    total = float(sum(lat)) if total_ms is None else float(total_ms)
    cand = int(query_count if candidates is None else candidates)
    calls = int(pt_exact_calls + ee_exact_calls if exact_calls is None else exact_calls)
    row = {
        "schema_version": BENCHMARK_EXPORT_SCHEMA_VERSION, "run_id": run_id, "dataset_name": dataset_name,
        "scene_name": scene_name, "method_name": method_name, "config_hash": config_hash, "seed": int(seed),
        "query_count": int(query_count), "fn_count": 0, "fp_count": 0, "candidate_recall": 1.0,
        "avg_candidates": cand / max(1, int(query_count)),
        "avg_exact_evals": distance_evals / max(1, int(query_count)),
        "avg_subdivision_depth": 0.0,
        "fallback_ratio": fallback_calls / calls if calls else 0.0,
        "candidate_inflation_ratio": cand / max(1, int(query_count)),
        "undecided_to_resolved_ratio": undecided / (collisions + separations) if collisions + separations else 0.0,
        "exact_queue_occupancy": 0.0,
        "rt_build_ms": 0.0, "rt_update_ms": 0.0, "rt_trace_ms": float(rt_ms), "rt_ms": float(rt_ms),
        "proposal_ms": 0.0, "exact_ms": float(exact_ms), "total_ms": total,
        "latency_min_ms": lat[0] if lat else 0.0, "latency_p50_ms": _percentile(lat, 50),
        "latency_p90_ms": _percentile(lat, 90), "latency_p95_ms": _percentile(lat, 95),
        "latency_p99_ms": _percentile(lat, 99), "latency_max_ms": lat[-1] if lat else 0.0,
        "qps": int(query_count) * len(lat) / (total * 1e-3) if total > 0 else 0.0,
        "family_point_triangle_exact_calls": int(pt_exact_calls), "family_edge_edge_exact_calls": int(ee_exact_calls),
        "family_conservative_exact_calls": 0, "family_unknown_exact_calls": 0,
        "exact_calls_total": int(pt_exact_calls) + int(ee_exact_calls),
        "candidate_buffer_bandwidth_mb_s": candidate_bytes / 1e6 / (rt_ms * 1e-3) if rt_ms > 0 else 0.0,
        "proposal_enqueue_dequeue_ms": 0.0,
        "total_tail_latency_ms": _percentile(lat, 99),
        "vram_peak_mb": int(vram_peak_bytes) >> 20,
    }
    for k, v in extra.items():
        if k not in row:
            raise KeyError(f"BenchmarkRowV2 has no field {k}")
        row[k] = v
    return validate_benchmark_row_v2(row)


def benchmark_jsonl(rows: Iterable[dict]) -> str:
    """write_benchmark_v2_jsonl's text for validated rows."""
    return "".join(_json_line({k: validate_benchmark_row_v2(r)[k] for k, _ in BENCHMARK_ROW_V2_FIELDS}) + "\n"
                   for r in rows)


def benchmark_csv(rows: list[dict]) -> str:
    """write_benchmark_v2_csv's text (header in schema order)."""
    buf = io.StringIO()
    names = [k for k, _ in BENCHMARK_ROW_V2_FIELDS]
    w = csv.DictWriter(buf, fieldnames=names, lineterminator="\n")
    w.writeheader()
    for r in rows:
        w.writerow({k: validate_benchmark_row_v2(r)[k] for k in names})
    return buf.getvalue()


def write_benchmark_v2_jsonl(path: str | Path, rows: Iterable[dict]) -> None:
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    p.write_text(benchmark_jsonl(rows), encoding="utf-8", newline="\n")
