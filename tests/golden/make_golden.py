"""Generate the golden certificate fixtures from the reference itself.

Run in a checkout where oracle/_ref/libp2c_ref.so was built from the
reference sources (``make -C oracle ref``).  Writes ``plain_sample.npz``:
a seeded sample of the plain-query workload (vertex-face and edge-edge, with
constructed-touching and near-degenerate members) and the reference
certifier's 72-byte results for it under two configurations, plus the
reference's own known-answer fixtures (test_certificate_engine.cpp:45-71).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path[:0] = [str(ROOT), str(ROOT / "p2c-ccd_b200")]

import oracle  # noqa: E402
from p2cccd_b200 import workloads  # noqa: E402

CONFIGS = {"c6": (1e-6, 1e-6, 32), "cdef": (1e-4, 1e-6, 32)}


def known_answer_fixtures():
    """MovingPointStaticTriangle / MovingEdgeThroughStaticEdge of the reference tests."""
    pt = np.zeros(2, dtype=oracle.PT)
    for i, (z0, z1) in enumerate([(1.0, -3.0), (2.0, 2.0)]):
        pt[i]["point_id"], pt[i]["triangle_id"] = 10 + i, 20 + i
        pt[i]["point"] = (10 + i, (0.25, 0.25, z0), (0.25, 0.25, z1))
        pt[i]["triangle_v0"] = (101, (0, 0, 0), (0, 0, 0))
        pt[i]["triangle_v1"] = (102, (1, 0, 0), (1, 0, 0))
        pt[i]["triangle_v2"] = (103, (0, 1, 0), (0, 1, 0))
    ee = np.zeros(2, dtype=oracle.EE)
    for i, (z0, z1) in enumerate([(1.0, -3.0), (2.0, 2.0)]):
        ee[i]["edge_a_id"], ee[i]["edge_b_id"] = 30 + i, 40 + i
        ee[i]["edge_a0"] = (201, (-1, 0, 0), (-1, 0, 0))
        ee[i]["edge_a1"] = (202, (1, 0, 0), (1, 0, 0))
        ee[i]["edge_b0"] = (301, (0, -1, z0), (0, -1, z1))
        ee[i]["edge_b1"] = (302, (0, 1, z0), (0, 1, z1))
    return pt, ee


def main() -> None:
    w = workloads.plain_queries(workloads.PlainSpec(n_vf=512, n_ee=512, seed=7))
    ka_pt, ka_ee = known_answer_fixtures()
    out = {"vf": w["vf"].view(np.uint8).reshape(-1, 240), "ee": w["ee"].view(np.uint8).reshape(-1, 240),
           "ka_pt": ka_pt.view(np.uint8).reshape(-1, 240), "ka_ee": ka_ee.view(np.uint8).reshape(-1, 240)}
    for tag, cfg in CONFIGS.items():
        for fam in ("vf", "ee"):
            res, st = oracle.ref_eval_batch(w[fam], 0.0, 1.0, *cfg)
            assert st.sum() == 0
            out[f"{fam}_{tag}"] = res.view(np.uint8).reshape(-1, 72)
        for fam, rec in (("ka_pt", ka_pt), ("ka_ee", ka_ee)):
            res, st = oracle.ref_eval_batch(rec, 0.0, 1.0, 1e-5, 1e-6, 32)
            out[f"{fam}_ka"] = res.view(np.uint8).reshape(-1, 72)
    np.savez_compressed(HERE / "plain_sample.npz", **out)
    print("wrote", HERE / "plain_sample.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
