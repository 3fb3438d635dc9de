"""Triangle mesh loading, validation and centring (geometry/mesh_io.cpp)
against the reference's loaders compiled unchanged; the binding's row and
record validators."""
from __future__ import annotations

import numpy as np
import pytest


def _need_ref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")


def _same(oracle_mod, path, center=False):
    import p2cccd_cpp as cpp

    want = oracle_mod.ref_load_mesh(path, center=center)
    mesh = cpp.load_triangle_mesh(path)
    if center:
        mesh, c = cpp.center_mesh_at_aabb_center(mesh)
        assert np.array_equal(np.asarray(c), want[3])
    assert np.array_equal(np.asarray(mesh.vertices_ref, np.float64).reshape(-1, 3), want[0])
    assert np.array_equal(np.asarray(mesh.triangles, np.int64).reshape(-1, 3), want[1].astype(np.int64))
    assert list(mesh.patch_ids) == want[2].tolist()


OBJ_OK = {
    "tetra": "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1 2 3\nf 1 2 4\nf 1 3 4\nf 2 3 4\n",
    "quads": "# a cube face pair\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 1\nv 1 0 1\n"
             "f 1/1/1 2/2/2 3/3/3 4/4/4\nf 1 2 6 5 # comment\n",
    "negative": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf -3 -2 -1\nv 2 2 2\nf -4 -3 -1\n",
    "groups": "o a\nv 0 0 0\nv 1 0 0\nv 0 1 0\ng b\nf 1 2 3\n\nv 1e-3 .5 +2.5e1 7\nf 1 2 4\n",
}

OBJ_BAD = {
    "vertex": "v 0 0\nv 1 0 0\n",
    "zero_index": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n",
    "range": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n",
    "two": "v 0 0 0\nv 1 0 0\nf 1 2\n",
    "degenerate": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 2\n",
    "area": "v 0 0 0\nv 1 0 0\nv 2 0 0\nf 1 2 3\n",
    "empty": "# nothing\n",
    "letters": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 x 3\n",
    "partial": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2a 3\n",
    "nan": "v nan 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
}


@pytest.mark.parametrize("name", sorted(OBJ_OK))
def test_obj_loads_like_reference(oracle_mod, tmp_path, name):
    _need_ref(oracle_mod)
    p = tmp_path / f"{name}.obj"
    p.write_text(OBJ_OK[name])
    _same(oracle_mod, p)
    _same(oracle_mod, p, center=True)


@pytest.mark.parametrize("name", sorted(OBJ_BAD))
def test_obj_errors_like_reference(oracle_mod, tmp_path, name):
    import p2cccd_cpp as cpp

    _need_ref(oracle_mod)
    p = tmp_path / f"{name}.obj"
    p.write_text(OBJ_BAD[name])
    with pytest.raises(ValueError) as ref_err:
        oracle_mod.ref_load_mesh(p)
    with pytest.raises(ValueError) as err:
        cpp.load_triangle_mesh(p)
    assert str(err.value) == str(ref_err.value)


def _stl_triangles(seed: int) -> np.ndarray:
    """Triangles over a shared float vertex pool (so vertices merge), with a
    degenerate one, +0/-0 coordinates and a repeated triangle."""
    g = np.random.default_rng(seed)
    pool = g.normal(0, 1, (40, 3)).astype(np.float32)
    pool[3] = [0.0, 1.0, 2.0]
    pool[4] = [-0.0, 1.0, 2.0]
    tri = g.integers(0, 40, (60, 3))
    tri = tri[(tri[:, 0] != tri[:, 1]) & (tri[:, 0] != tri[:, 2]) & (tri[:, 1] != tri[:, 2])]
    tri = np.concatenate([tri, [[3, 4, 5], tri[0]]])
    return pool[tri]


def test_stl_binary_and_ascii_load_like_reference(oracle_mod, tmp_path):
    _need_ref(oracle_mod)
    t = _stl_triangles(3)
    rec = np.zeros(len(t), dtype=np.dtype([("f", "<f4", (12,)), ("a", "<u2")]))
    rec["f"][:, 3:] = t.reshape(-1, 9)
    b = tmp_path / "mesh.stl"
    b.write_bytes(b"\0" * 80 + np.uint32(len(t)).tobytes() + rec.tobytes())
    _same(oracle_mod, b)
    _same(oracle_mod, b, center=True)
    a = tmp_path / "mesh_ascii.STL"
    lines = ["solid m"]
    for tri in t:
        lines += ["facet normal 0 0 0", "outer loop"] + [f"vertex {x!r} {y!r} {z!r}" for x, y, z in tri.tolist()]
        lines += ["endloop", "endfacet"]
    a.write_text("\n".join(lines + ["endsolid m"]) + "\n")
    _same(oracle_mod, a)


def test_unknown_format_and_missing_file(oracle_mod, tmp_path):
    import p2cccd_cpp as cpp

    _need_ref(oracle_mod)
    for name in ("mesh.ply", "missing.obj", "missing.stl"):
        p = tmp_path / name
        if name.endswith(".ply"):
            p.write_text("ply\n")
        with pytest.raises(ValueError) as ref_err:
            oracle_mod.ref_load_mesh(p)
        with pytest.raises(ValueError) as err:
            cpp.load_triangle_mesh(p)
        assert str(err.value) == str(ref_err.value)


def test_validators():
    import p2cccd_cpp as cpp

    row = cpp.BenchmarkRow()
    with pytest.raises(ValueError, match="BenchmarkRow.query_count is required"):
        cpp.validate_benchmark_row(row)
    row.query_count, row.fn_count = 10, 11
    with pytest.raises(ValueError, match="fn_count cannot exceed query_count"):
        cpp.validate_benchmark_row(row)
    row.fn_count, row.candidate_recall = 0, 1.5
    with pytest.raises(ValueError, match=r"candidate_recall must be in \[0, 1\]"):
        cpp.validate_benchmark_row(row)
    row.candidate_recall, row.qps = 1.0, -1.0
    with pytest.raises(ValueError, match="BenchmarkRow.qps must be non-negative"):
        cpp.validate_benchmark_row(row)
    row.qps = 5.0
    assert cpp.validate_benchmark_row(row)
    rec = cpp.CandidateRecord()
    with pytest.raises(ValueError, match="CandidateRecord.candidate_id is required"):
        cpp.validate_candidate_record(rec)
    rec.candidate_id, rec.query_id, rec.rt_hit_count = 3, 4, 1
    rec.proxy_type_a = rec.proxy_type_b = cpp.ProxyType.SWEPT_AABB
    assert cpp.validate_candidate_record(rec)
    mesh = cpp.Mesh()
    mesh.vertices_ref, mesh.triangles = [[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 2]]
    mesh.patch_ids = [0, 0]
    with pytest.raises(ValueError, match="patch_ids must be empty or match triangle count"):
        cpp.validate_triangle_mesh(mesh)
