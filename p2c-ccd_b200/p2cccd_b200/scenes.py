"""Seeded synthetic scenes (FP64 vertex trajectories over one step).

* ``uv_sphere``: a closed UV sphere, ``n_lon`` longitudes x ``n_rings``
  interior latitude rings + 2 poles: 2 * n_lon * n_rings triangles.  160 x 128
  gives 40,960 triangles, 20,482 vertices and 61,440 edges (40,960 is not an
  icosphere level: 20 * 4^k gives 20,480 or 81,920).
* ``two_spheres``: two such spheres, B translating toward A so that they meet
  at mid-step, with per-vertex N(0, sigma) jitter at t0 and t1.
* ``cloth_on_sphere``: an n x n cloth grid draped onto a sphere with a small
  initial gap (the dense-contact stress scene).

A scene is a dict of numpy arrays: v_t0, v_t1 (nv, 3) f64; faces (nf, 3) i32;
edges (ne, 2) i32 (unique, sorted lexicographically per object, then offset);
v_obj / f_obj / e_obj i32 object ids.
"""
from __future__ import annotations

import numpy as np

from .workloads import rng


def uv_sphere(n_lon: int = 160, n_rings: int = 128, radius: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    lat = np.pi * np.arange(1, n_rings + 1) / (n_rings + 1)  # interior rings, poles excluded
    lon = 2.0 * np.pi * np.arange(n_lon) / n_lon
    st, ct = np.sin(lat)[:, None], np.cos(lat)[:, None]
    ring = np.stack([st * np.cos(lon)[None, :], st * np.sin(lon)[None, :], np.broadcast_to(ct, (n_rings, n_lon))],
                    axis=-1).reshape(-1, 3)
    verts = np.concatenate([[[0.0, 0.0, 1.0]], ring, [[0.0, 0.0, -1.0]]]) * radius
    north, south = 0, 1 + n_rings * n_lon

    def rv(r, j):  # ring r (0-based), longitude j
        return 1 + r * n_lon + (j % n_lon)

    faces = []
    j = np.arange(n_lon)
    faces.append(np.stack([np.full(n_lon, north), rv(0, j), rv(0, j + 1)], 1))
    for r in range(n_rings - 1):
        a, b, c, d = rv(r, j), rv(r, j + 1), rv(r + 1, j), rv(r + 1, j + 1)
        faces.append(np.stack([a, c, b], 1))
        faces.append(np.stack([b, c, d], 1))
    faces.append(np.stack([np.full(n_lon, south), rv(n_rings - 1, j + 1), rv(n_rings - 1, j)], 1))
    return verts, np.concatenate(faces).astype(np.int32)


def unique_edges(faces: np.ndarray) -> np.ndarray:
    """Unique undirected edges (min, max), sorted lexicographically - the order
    ExtractUniqueMeshEdges produces (cpp/certificate/mesh_exact_query.cpp:115-141)."""
    e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
    e = np.sort(e, axis=1)
    return np.unique(e, axis=0).astype(np.int32)


def combine(objects: list[tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]]) -> dict:
    """Stack objects (v_t0, v_t1, faces, edges) into one scene with offsets."""
    vt0, vt1, fs, es, vo, fo, eo = [], [], [], [], [], [], []
    off = 0
    for k, (a0, a1, f, e) in enumerate(objects):
        vt0.append(a0)
        vt1.append(a1)
        fs.append(f + off)
        es.append(e + off)
        vo.append(np.full(len(a0), k, np.int32))
        fo.append(np.full(len(f), k, np.int32))
        eo.append(np.full(len(e), k, np.int32))
        off += len(a0)
    return {"v_t0": np.ascontiguousarray(np.concatenate(vt0)), "v_t1": np.ascontiguousarray(np.concatenate(vt1)),
            "faces": np.concatenate(fs).astype(np.int32), "edges": np.concatenate(es).astype(np.int32),
            "v_obj": np.concatenate(vo), "f_obj": np.concatenate(fo), "e_obj": np.concatenate(eo),
            "n_obj": len(objects)}


def two_spheres(n_lon: int = 160, n_rings: int = 128, seed: int = 20261203, gap: float = 0.05,
                jitter: float = 1.0e-3, approach: float = 0.1) -> dict:
    """Sphere A at the origin, sphere B starting at x = 2 + gap and moving by
    -approach along x (contact near t = gap / approach); both spheres get
    independent N(0, jitter) per-vertex offsets at t0 and t1."""
    g = rng(seed)
    v, f = uv_sphere(n_lon, n_rings)
    e = unique_edges(f)
    # a fixed small rotation of B so the two tessellations are not aligned
    ang = 0.37
    rot = np.array([[np.cos(ang), 0.0, np.sin(ang)], [0.0, 1.0, 0.0], [-np.sin(ang), 0.0, np.cos(ang)]])
    vb = v @ rot.T
    a0 = v + g.normal(0.0, jitter, v.shape)
    a1 = v + g.normal(0.0, jitter, v.shape)
    cb0 = np.array([2.0 + gap, 0.0, 0.0])
    cb1 = cb0 - np.array([approach, 0.0, 0.0])
    b0 = vb + cb0 + g.normal(0.0, jitter, v.shape)
    b1 = vb + cb1 + g.normal(0.0, jitter, v.shape)
    s = combine([(a0, a1, f, e), (b0, b1, f, e)])
    s["spec"] = {"kind": "two_spheres", "n_lon": n_lon, "n_rings": n_rings, "seed": seed, "gap": gap,
                 "jitter": jitter, "approach": approach, "triangles_per_sphere": int(len(f))}
    return s


def cloth_on_sphere(n: int = 513, sphere_lon: int = 250, sphere_rings: int = 200, seed: int = 20261203,
                    gap: float = 1.0e-4, drop: float = 0.02, jitter: float = 1.0e-5) -> dict:
    """An n x n cloth grid (2 (n-1)^2 triangles) of side 3 centred over a unit
    sphere, its lowest point gap above the sphere at t0, falling by drop and
    draping (each vertex pulled toward the sphere surface) over the step."""
    g = rng(seed)
    sv, sf = uv_sphere(sphere_lon, sphere_rings)
    se = unique_edges(sf)
    xs = np.linspace(-1.5, 1.5, n)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    r2 = X ** 2 + Y ** 2
    top = np.sqrt(np.clip(1.0 - r2, 0.0, None))
    z0 = np.full_like(X, 1.0 + gap)
    # drape target: sphere surface inside the unit disc, sagging outside it
    z1 = np.where(r2 < 1.0, top + gap * 0.5, 1.0 + gap - drop - 0.5 * (np.sqrt(r2) - 1.0))
    z1 = np.minimum(z1, z0 - drop * 0.25)
    c0 = np.stack([X, Y, z0], -1).reshape(-1, 3) + g.normal(0, jitter, (n * n, 3))
    c1 = np.stack([X, Y, z1], -1).reshape(-1, 3) + g.normal(0, jitter, (n * n, 3))
    idx = np.arange(n * n).reshape(n, n)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[:-1, 1:].ravel(), idx[1:, :-1].ravel(), idx[1:, 1:].ravel()
    cf = np.concatenate([np.stack([a, b, c], 1), np.stack([b, d, c], 1)]).astype(np.int32)
    ce = unique_edges(cf)
    s0 = sv + g.normal(0, jitter, sv.shape)
    s1 = sv + g.normal(0, jitter, sv.shape)
    s = combine([(c0, c1, cf, ce), (s0, s1, sf, se)])
    s["spec"] = {"kind": "cloth_on_sphere", "cloth_n": n, "cloth_triangles": int(len(cf)),
                 "sphere_triangles": int(len(sf)), "seed": seed, "gap": gap, "drop": drop}
    return s


def _rotation(axis: np.ndarray, angle: float) -> np.ndarray:
    a = axis / np.linalg.norm(axis)
    k = np.array([[0.0, -a[2], a[1]], [a[2], 0.0, -a[0]], [-a[1], a[0], 0.0]])
    return np.eye(3) + np.sin(angle) * k + (1.0 - np.cos(angle)) * (k @ k)


def uneven_batch(n_scenes: int = 256, tri_min: float = 1.0e3, tri_max: float = 2.0e5, seed: int = 20261203,
                 jitter: float = 1.0e-3) -> list[dict]:
    """Independent two-sphere scenes of uneven size: total triangle counts
    log-uniform over [tri_min, tri_max]; each scene is two UV spheres of half
    that count, sphere A turning slightly (up to 0.02 rad) about a random
    axis, sphere B starting gap ~ U[0.01, 0.03] away along a random direction
    and moving rigidly (rotation up to 0.05 rad) toward A to a penetration
    depth of 0.25 f at t1, f ~ U[5%, 40%] the scene's contact parameter (the
    share of candidates that then hit is measured, not imposed);
    per-vertex N(0, jitter) at t0 and t1."""
    g = rng(seed)
    out = []
    for i in range(n_scenes):
        tris = float(np.exp(g.uniform(np.log(tri_min), np.log(tri_max))))
        rings = max(3, int(round(np.sqrt(tris / 5.0))))
        lon = max(4, int(round(tris / 2.0 / (2.0 * rings))))
        v, f = uv_sphere(lon, rings)
        e = unique_edges(f)
        frac = float(g.uniform(0.05, 0.40))
        gap = float(g.uniform(0.01, 0.03))
        u = g.normal(size=3)
        u /= np.linalg.norm(u)
        ra1 = _rotation(g.normal(size=3), float(g.uniform(0.0, 0.02)))
        rb0 = _rotation(g.normal(size=3), float(g.uniform(0.0, np.pi)))
        rb1 = _rotation(g.normal(size=3), float(g.uniform(0.0, 0.05))) @ rb0
        cb0 = (2.0 + gap) * u
        cb1 = (2.0 - 0.25 * frac) * u
        a0 = v + g.normal(0.0, jitter, v.shape)
        a1 = v @ ra1.T + g.normal(0.0, jitter, v.shape)
        b0 = v @ rb0.T + cb0 + g.normal(0.0, jitter, v.shape)
        b1 = v @ rb1.T + cb1 + g.normal(0.0, jitter, v.shape)
        s = combine([(a0, a1, f, e), (b0, b1, f, e)])
        s["spec"] = {"kind": "uneven_batch_scene", "index": i, "n_lon": lon, "n_rings": rings,
                     "triangles": int(2 * len(f)), "contact_parameter": frac, "gap": gap, "seed": seed}
        out.append(s)
    return out
