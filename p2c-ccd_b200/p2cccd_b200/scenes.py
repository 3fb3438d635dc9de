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


def proxy_scene(n_objects: int = 6, patches_per_object: int = 40, n_slabs: int = 4, seed: int = 20261203,
                query_id: int = 7, duplicates: float = 0.0) -> dict:
    """A proxy scene (the arrays p2c_proxy_scene reads): every object's patches
    as boxes in every time slab of a global partition of [0, 1], objects
    drifting toward each other so that patches of different objects overlap
    in some slabs; swept-AABB and capsule proxy types; motion bounds >= 0.
    ``duplicates`` adds that fraction of extra proxies repeating an existing
    (object, patch, slab) with other bounds, so that several raw hits
    compact into one candidate."""
    g = rng(seed)
    edges = np.linspace(0.0, 1.0, n_slabs + 1)
    rows = []
    for o in range(n_objects):
        center = g.uniform(-1.0, 1.0, 3)
        vel = -center * g.uniform(0.5, 1.0)
        ptype = 1 + (o % 2)
        offs = g.normal(0.0, 0.25, (patches_per_object, 3))
        half = g.uniform(0.02, 0.12, (patches_per_object, 3))
        for sl in range(n_slabs):
            t0, t1 = edges[sl], edges[sl + 1]
            c0, c1 = center + vel * t0, center + vel * t1
            for pch in range(patches_per_object):
                lo = np.minimum(c0, c1) + offs[pch] - half[pch]
                hi = np.maximum(c0, c1) + offs[pch] + half[pch]
                mb = g.uniform(0.0, 0.2, 4)
                rows.append((o, pch, sl, ptype, t0, t1, lo, hi, mb))
                if g.random() < duplicates:
                    d = g.normal(0.0, 0.03, 3)
                    rows.append((o, pch, sl, ptype, t0, t1, lo + d, hi + d, g.uniform(0.0, 0.2, 4)))
    n = len(rows)
    out = {"query_id": query_id, "n": n,
           "object_id": np.array([r[0] for r in rows], np.uint32),
           "patch_id": np.array([r[1] for r in rows], np.uint32),
           "slab_id": np.array([r[2] for r in rows], np.uint32),
           "proxy_type": np.array([r[3] for r in rows], np.uint8),
           "t0": np.array([r[4] for r in rows], np.float64),
           "t1": np.array([r[5] for r in rows], np.float64),
           "bounds": np.array([np.concatenate([r[6], r[7]]) for r in rows], np.float64).reshape(n, 6),
           "motion_bound": np.array([r[8] for r in rows], np.float64).reshape(n, 4)}
    perm = g.permutation(n)  # proxies in no particular order (proxy_id = index)
    for k in ("object_id", "patch_id", "slab_id", "proxy_type", "t0", "t1", "bounds", "motion_bound"):
        out[k] = np.ascontiguousarray(out[k][perm])
    return out


def _quat(axis, angle, scale=1.0):
    """Quaternion (x, y, z, w) of a rotation by ``angle`` about ``axis``,
    multiplied by ``scale`` (the builder normalises it)."""
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    return np.concatenate([axis * np.sin(0.5 * angle), [np.cos(0.5 * angle)]]) * scale


def proxy_build_input(n_objects: int = 6, patches_per_object: int = 60, n_segments: int = 2, slabs: int = 3,
                      seed: int = 20261203, query_id: int = 11, eps_proxy: float = 1e-3,
                      spread: float | None = None) -> dict:
    """A ProxySceneBuildInput as arrays: ``objects`` of rigid bodies whose
    patches (centres on a sphere about the body origin, small radii) move
    over piecewise rigid motion segments partitioning [0, 1] the same way for
    every object (so the slab ids form one global partition).  Bodies drift
    toward the origin while rotating; the rotations cover the slerp branch,
    the near-parallel lerp branch (a still body and a tiny rotation), a
    quaternion pair of opposite signs and quaternions of non-unit norm.
    Segment rows are t0, t1, translation_t0, rotation_t0 (x, y, z, w),
    translation_t1, rotation_t1.  With ``spread`` the bodies start anywhere
    in [-spread, spread]^3 and drift 0.1-0.4 in a random direction instead,
    a sparse scene where only neighbours meet."""
    g = rng(seed)
    cuts = np.linspace(0.0, 1.0, n_segments + 1)
    objects = []
    pid = 0
    for o in range(n_objects):
        if spread is None:
            start = g.uniform(-1.0, 1.0, 3)
            vel = -start * g.uniform(0.6, 1.1)
        else:
            start = g.uniform(-spread, spread, 3)
            vel = g.normal(size=3)
            vel *= g.uniform(0.1, 0.4) / np.linalg.norm(vel)
        axis = g.normal(size=3)
        spin = [g.uniform(0.5, 3.0), 0.0, 1e-3, g.uniform(0.5, 3.0)][o % 4]
        segs = np.zeros((n_segments, 16))
        for s in range(n_segments):
            a, b = cuts[s], cuts[s + 1]
            segs[s, 0:2] = a, b
            segs[s, 2:5] = start + vel * a
            segs[s, 5:9] = _quat(axis, spin * a, g.uniform(0.5, 2.0))
            segs[s, 9:12] = start + vel * b
            q1 = _quat(axis, spin * b, g.uniform(0.5, 2.0))
            segs[s, 12:16] = -q1 if o % 4 == 3 else q1  # same rotation, opposite sign
        radius_body = g.uniform(0.15, 0.35)
        d = g.normal(size=(patches_per_object, 3))
        centers = d / np.linalg.norm(d, axis=1, keepdims=True) * radius_body
        objects.append({"object_id": 100 + 3 * o, "proxy_type": 1 + (o % 2), "slabs_per_motion_segment": slabs,
                        "eps_proxy": eps_proxy,
                        "patch_id": np.arange(pid, pid + patches_per_object, dtype=np.uint32),
                        "local_center": np.ascontiguousarray(centers),
                        "radius": g.uniform(0.02, 0.08, patches_per_object), "segments": segs})
        pid += patches_per_object
    return {"query_id": query_id, "objects": objects}
