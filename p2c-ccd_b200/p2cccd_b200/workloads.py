"""Seeded synthetic CCD workloads (numpy Philox; seeds are part of each spec).

No public dataset is used: these generators stand in for the reference's
benchmark inputs with the stated shapes, sizes and value distributions.

* ``plain_queries``: the plain exact-CCD batch - independent vertex-face and
  edge-edge queries, endpoints U[0,1]^3, per-coordinate displacement
  N(0, 0.05); a fraction constructed to touch at t* ~ U[0,1] and a fraction
  near-degenerate (coplanar / collinear / parallel within 1e-9).
* scene generators (UV spheres, cloth) live in ``scenes.py``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .records import FAMILY_EDGE_EDGE, FAMILY_POINT_TRIANGLE, pack_primitives

DEFAULT_SEED = 20261203


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


@dataclass(frozen=True)
class PlainSpec:
    n_vf: int = 10_000
    n_ee: int = 10_000
    seed: int = DEFAULT_SEED
    touch_frac: float = 0.30
    degen_frac: float = 0.10
    disp_sigma: float = 0.05
    degen_eps: float = 1.0e-9


def _categories(g: np.random.Generator, n: int, spec: PlainSpec) -> np.ndarray:
    n_touch = int(round(spec.touch_frac * n))
    n_degen = int(round(spec.degen_frac * n))
    cat = np.zeros(n, dtype=np.int8)
    cat[:n_touch] = 1
    cat[n_touch:n_touch + n_degen] = 2
    return cat[g.permutation(n)]


def _vf(g: np.random.Generator, spec: PlainSpec) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    n = spec.n_vf
    p0 = g.uniform(0.0, 1.0, size=(n, 4, 3))
    p1 = p0 + g.normal(0.0, spec.disp_sigma, size=(n, 4, 3))
    cat = _categories(g, n, spec)
    # touching: shift the point's trajectory so that it lies on the triangle at t*
    idx = np.nonzero(cat == 1)[0]
    if idx.size:
        ts = g.uniform(0.0, 1.0, size=idx.size)[:, None]
        bary = g.dirichlet(np.ones(3), size=idx.size)
        tri_t = (1.0 - ts)[:, :, None] * p0[idx, 1:, :] + ts[:, :, None] * p1[idx, 1:, :]
        target = np.einsum("nk,nkc->nc", bary, tri_t)
        at_t = (1.0 - ts) * p0[idx, 0, :] + ts * p1[idx, 0, :]
        delta = target - at_t
        p0[idx, 0, :] += delta
        p1[idx, 0, :] += delta
    # near-degenerate: half coplanar (all four trajectories in one plane up to
    # 1e-9), half near-collinear triangles (triangle normal ~ 0)
    idx = np.nonzero(cat == 2)[0]
    if idx.size:
        half = idx[: idx.size // 2]
        rest = idx[idx.size // 2:]
        zc = g.uniform(0.0, 1.0, size=half.size)[:, None]
        p0[half, :, 2] = zc + g.normal(0.0, spec.degen_eps, size=(half.size, 4))
        p1[half, :, 2] = zc + g.normal(0.0, spec.degen_eps, size=(half.size, 4))
        a = p0[rest, 1, :]
        d = g.normal(0.0, 1.0, size=(rest.size, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        s = g.uniform(0.1, 0.5, size=(rest.size, 2))
        p0[rest, 2, :] = a + s[:, :1] * d + g.normal(0.0, spec.degen_eps, size=(rest.size, 3))
        p0[rest, 3, :] = a - s[:, 1:] * d + g.normal(0.0, spec.degen_eps, size=(rest.size, 3))
        p1[rest, 1:, :] = p0[rest, 1:, :] + (p1[rest, 1:2, :] - p0[rest, 1:2, :])
    ids_a = np.arange(n, dtype=np.int64)
    ids_b = np.arange(n, dtype=np.int64) + 1_000_000
    fid = np.arange(4 * n, dtype=np.int64).reshape(n, 4)
    return pack_primitives(p0, p1, ids_a, ids_b, fid, FAMILY_POINT_TRIANGLE), cat, fid


def _ee(g: np.random.Generator, spec: PlainSpec) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    n = spec.n_ee
    p0 = g.uniform(0.0, 1.0, size=(n, 4, 3))
    p1 = p0 + g.normal(0.0, spec.disp_sigma, size=(n, 4, 3))
    cat = _categories(g, n, spec)
    idx = np.nonzero(cat == 1)[0]
    if idx.size:
        ts = g.uniform(0.0, 1.0, size=idx.size)[:, None]
        sa = g.uniform(0.0, 1.0, size=idx.size)[:, None]
        sb = g.uniform(0.0, 1.0, size=idx.size)[:, None]
        pos = lambda k: (1.0 - ts) * p0[idx, k, :] + ts * p1[idx, k, :]
        on_a = (1.0 - sa) * pos(0) + sa * pos(1)
        on_b = (1.0 - sb) * pos(2) + sb * pos(3)
        delta = on_a - on_b
        p0[idx, 2:, :] += delta[:, None, :]
        p1[idx, 2:, :] += delta[:, None, :]
    # near-degenerate: half parallel edges (direction equal within 1e-9), half
    # a near-zero-length edge
    idx = np.nonzero(cat == 2)[0]
    if idx.size:
        half = idx[: idx.size // 2]
        rest = idx[idx.size // 2:]
        for p in (p0, p1):
            da = p[half, 1, :] - p[half, 0, :]
            scale = g.uniform(0.3, 1.5, size=(half.size, 1))
            p[half, 3, :] = p[half, 2, :] + scale * da + g.normal(0.0, spec.degen_eps, size=(half.size, 3))
            p[rest, 1, :] = p[rest, 0, :] + g.normal(0.0, spec.degen_eps, size=(rest.size, 3))
    ids_a = np.arange(n, dtype=np.int64) + 2_000_000
    ids_b = np.arange(n, dtype=np.int64) + 3_000_000
    fid = np.arange(4 * n, dtype=np.int64).reshape(n, 4) + 4 * spec.n_vf
    return pack_primitives(p0, p1, ids_a, ids_b, fid, FAMILY_EDGE_EDGE), cat, fid


def plain_queries(spec: PlainSpec = PlainSpec()) -> dict:
    """Returns {'vf': records, 'ee': records, 'vf_cat': ..., 'ee_cat': ...}
    (category 0 generic, 1 constructed touching, 2 near-degenerate)."""
    g = rng(spec.seed)
    vf, vf_cat, _ = _vf(g, spec)
    ee, ee_cat, _ = _ee(g, spec)
    return {"vf": vf, "ee": ee, "vf_cat": vf_cat, "ee_cat": ee_cat, "spec": spec}


def dense_group_rows(n_rows: int, seed: int = DEFAULT_SEED, max_group: int = 256) -> dict:
    """Rows of the candidate-group interface (the arrays
    run_native_dense_group_exact_early_stop reads) for ``n_rows`` candidates
    in query groups of log-uniform size 1..``max_group``, rows shuffled:
    labels (oracle_trace[:, 0]) positive for ~20% of candidates, full exact
    costs gamma-distributed (some zero or negative: replaced by 1 on the
    path), contact intervals inside [0, 1], eight interval scores, and
    priority / cost / uncertainty scores as a proposal model would emit."""
    g = rng(seed)
    sizes = []
    total = 0
    while total < n_rows:
        s = int(np.exp(g.uniform(0.0, np.log(max_group + 1.0))))
        s = max(1, min(s, n_rows - total))
        sizes.append(s)
        total += s
    q = np.repeat(np.arange(1, len(sizes) + 1, dtype=np.uint64) * np.uint64(7919), sizes)
    q = q[g.permutation(n_rows)]
    trace = np.zeros((n_rows, 8))
    trace[:, 0] = (g.random(n_rows) < 0.2).astype(np.float64)
    trace[:, 5] = g.gamma(2.0, 40.0, n_rows)
    trace[g.random(n_rows) < 0.01, 5] = 0.0
    c0 = g.random(n_rows)
    trace[:, 6] = c0
    trace[:, 7] = np.minimum(1.0, c0 + g.random(n_rows) * 0.25)
    return {"query_id": q, "candidate_id": np.arange(1, n_rows + 1, dtype=np.uint64),
            "cost_target": g.random(n_rows).astype(np.float32), "oracle_trace": trace,
            "interval_scores": g.normal(0.0, 1.0, (n_rows, 8)).astype(np.float32),
            "priority_score": g.normal(0.0, 1.0, n_rows).astype(np.float32),
            "cost_score": g.random(n_rows).astype(np.float32),
            "uncertainty_score": g.beta(2.0, 5.0, n_rows).astype(np.float32)}
